// Ray-driven projection kernels: exact line integrals of analytic ellipsoid phantoms (input
// generation) and a ray-marching forward projector through a voxel volume (consistency
// checks). Rays are built per detector pixel from the same per-view geometry the
// backprojector inverts, so a projection followed by backprojection uses one convention:
//   parallel kinds : origin s n + (0,0,z), direction (cos t, sin t, 0), n = (cos(t+pi/2), sin(t+pi/2), 0)
//   line / flat    : origin S, direction SDD e_w + u e_u + v e_v
//   arc / cylinder : origin S, direction cos(g) e_w + sin(g) e_u + (t / SDD) e_v
// with u = (c - c0) du, v = (r - r0) dv (src/cuda/geom/coord_trans_proj.cuh:142-150, the
// inverse of DCSToPCS).
#include "../../include/gct_fdk.h"
#include "project.hpp"

namespace gct {
namespace {

struct Ray {
    double o[3];
    double d[3];
};

__device__ Ray make_ray(const ProjView &pv, int kind, double du, double dv, int c, int r)
{
    Ray ray;
    const double u = (static_cast<double>(c) - pv.c0) * du;
    const double t = (static_cast<double>(r) - pv.r0) * dv;
    if (kind == GCT_GEOM_PARALLEL_1D || kind == GCT_GEOM_PARALLEL_2D || kind == GCT_GEOM_CONE_PARALLEL) {
        const double th = pv.extra;
        double sn, cs;
        sincos(th, &sn, &cs);
        // n = (cos(th + pi/2), sin(th + pi/2)) = (-sin th, cos th)
        double z = 0.0;
        if (kind == GCT_GEOM_PARALLEL_2D) z = -t;
        if (kind == GCT_GEOM_CONE_PARALLEL) z = -t * pv.zscale;
        ray.o[0] = -sn * u;
        ray.o[1] = cs * u;
        ray.o[2] = z;
        ray.d[0] = cs;
        ray.d[1] = sn;
        ray.d[2] = 0.0;
        return ray;
    }
    for (int i = 0; i < 3; ++i) ray.o[i] = pv.src[i];
    if (kind == GCT_GEOM_FAN_LINE || kind == GCT_GEOM_CONE_FLAT) {
        for (int i = 0; i < 3; ++i) ray.d[i] = pv.sdd * pv.ew[i] + u * pv.eu[i] + t * pv.ev[i];
    } else {
        double sg, cg;
        sincos(u, &sg, &cg);
        for (int i = 0; i < 3; ++i) ray.d[i] = cg * pv.ew[i] + sg * pv.eu[i] + (t / pv.sdd) * pv.ev[i];
    }
    return ray;
}

__global__ void phantom_kernel(const ProjView *__restrict__ views, int kind, int nv, int nr,
                               int nc, double du, double dv, const gct_ellipsoid *__restrict__ ell,
                               int ne, bool planar, float *__restrict__ out)
{
    const long long total = static_cast<long long>(nv) * nr * nc;
    for (long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
         idx += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int c = static_cast<int>(idx % nc);
        const long long vr = idx / nc;
        const int r = static_cast<int>(vr % nr);
        const int v = static_cast<int>(vr / nr);
        const Ray ray = make_ray(views[v], kind, du, dv, c, r);
        const double dn = sqrt(ray.d[0] * ray.d[0] + ray.d[1] * ray.d[1] + ray.d[2] * ray.d[2]);
        double sum = 0.0;
        for (int e = 0; e < ne; ++e) {
            const gct_ellipsoid E = ell[e];
            double sp, cp;
            sincos(E.phi, &sp, &cp);
            double p[3] = {ray.o[0] - E.center[0], ray.o[1] - E.center[1],
                           planar ? 0.0 : ray.o[2] - E.center[2]};
            double q[3] = {ray.d[0], ray.d[1], planar ? 0.0 : ray.d[2]};
            // rotate by -phi about z, then scale by the semi-axes
            const double px = (cp * p[0] + sp * p[1]) / E.semi_axes[0];
            const double py = (-sp * p[0] + cp * p[1]) / E.semi_axes[1];
            const double pz = p[2] / E.semi_axes[2];
            const double qx = (cp * q[0] + sp * q[1]) / E.semi_axes[0];
            const double qy = (-sp * q[0] + cp * q[1]) / E.semi_axes[1];
            const double qz = q[2] / E.semi_axes[2];
            const double A = qx * qx + qy * qy + qz * qz;
            const double B = px * qx + py * qy + pz * qz;
            const double C = px * px + py * py + pz * pz - 1.0;
            const double disc = B * B - A * C;
            if (disc > 0.0) sum += E.mu * 2.0 * sqrt(disc) / A * dn;
        }
        out[idx] = static_cast<float>(sum);
    }
}

// Trilinear sample with zero outside the grid; (x, y, z) in voxel-index units.
__device__ __forceinline__ float trilinear(const float *__restrict__ vol, int nx, int ny, int nz,
                                           float x, float y, float z)
{
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const int ix = static_cast<int>(fx), iy = static_cast<int>(fy), iz = static_cast<int>(fz);
    const float ax = x - fx, ay = y - fy, az = z - fz;
    float acc = 0.f;
#pragma unroll
    for (int dz = 0; dz < 2; ++dz) {
        const int zz = iz + dz;
        if (zz < 0 || zz >= nz) continue;
        const float wz = dz ? az : 1.f - az;
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
            const int yy = iy + dy;
            if (yy < 0 || yy >= ny) continue;
            const float wy = dy ? ay : 1.f - ay;
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int xx = ix + dx;
                if (xx < 0 || xx >= nx) continue;
                const float wx = dx ? ax : 1.f - ax;
                acc += wx * wy * wz * __ldg(vol + (static_cast<long long>(zz) * ny + yy) * nx + xx);
            }
        }
    }
    return acc;
}

__global__ void forward_kernel(const ProjView *__restrict__ views, int kind, int nv, int nr, int nc,
                               double du, double dv, const float *__restrict__ vol, VolBox box,
                               float step_vox, float *__restrict__ out)
{
    const long long total = static_cast<long long>(nv) * nr * nc;
    for (long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
         idx += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int c = static_cast<int>(idx % nc);
        const long long vr = idx / nc;
        const int r = static_cast<int>(vr % nr);
        const int v = static_cast<int>(vr / nr);
        Ray ray = make_ray(views[v], kind, du, dv, c, r);
        if (box.planar) {
            ray.o[2] = box.lo[2];
            ray.d[2] = 0.0;
        }
        const double dn = sqrt(ray.d[0] * ray.d[0] + ray.d[1] * ray.d[1] + ray.d[2] * ray.d[2]);
        double dir[3] = {ray.d[0] / dn, ray.d[1] / dn, ray.d[2] / dn};
        // slab intersection with the voxel-centre box extended by half a voxel
        double t0 = -1e300, t1 = 1e300;
        bool hit = true;
        for (int a = 0; a < 3; ++a) {
            if (box.planar && a == 2) continue;
            const double lo = box.lo[a] - 0.5 * box.w[a], hi = box.hi[a] + 0.5 * box.w[a];
            if (fabs(dir[a]) < 1e-15) {
                if (ray.o[a] < lo || ray.o[a] > hi) hit = false;
                continue;
            }
            double ta = (lo - ray.o[a]) / dir[a], tb = (hi - ray.o[a]) / dir[a];
            if (ta > tb) {
                const double tmp = ta;
                ta = tb;
                tb = tmp;
            }
            t0 = fmax(t0, ta);
            t1 = fmin(t1, tb);
        }
        float sum = 0.f;
        if (hit && t1 > t0) {
            const double wmin = box.planar ? fmin(box.w[0], box.w[1]) : fmin(box.w[0], fmin(box.w[1], box.w[2]));
            const double h = static_cast<double>(step_vox) * wmin;
            const long long ns = static_cast<long long>(ceil((t1 - t0) / h));
            for (long long s = 0; s < ns; ++s) {
                const double t = t0 + (static_cast<double>(s) + 0.5) * h;
                const float x = static_cast<float>((ray.o[0] + t * dir[0] - box.lo[0]) / box.w[0]);
                const float y = static_cast<float>((ray.o[1] + t * dir[1] - box.lo[1]) / box.w[1]);
                const float z = box.planar ? 0.f : static_cast<float>((ray.o[2] + t * dir[2] - box.lo[2]) / box.w[2]);
                sum += trilinear(vol, box.nx, box.ny, box.nz, x, y, z);
            }
            sum *= static_cast<float>(h);
        }
        out[idx] = sum;
    }
}

}  // namespace

void launch_phantom(const ProjView *views, int kind, int nv, int nr, int nc, double du, double dv,
                    const gct_ellipsoid *ell, int ne, bool planar, float *out, int num_sms,
                    cudaStream_t s)
{
    const long long total = static_cast<long long>(nv) * nr * nc;
    long long grid = (total + 255) / 256;
    if (grid > static_cast<long long>(num_sms) * 32) grid = static_cast<long long>(num_sms) * 32;
    if (grid < 1) grid = 1;
    phantom_kernel<<<static_cast<unsigned>(grid), 256, 0, s>>>(views, kind, nv, nr, nc, du, dv, ell, ne,
                                                               planar, out);
}

void launch_forward(const ProjView *views, int kind, int nv, int nr, int nc, double du, double dv,
                    const float *vol, const VolBox &box, float step_vox, float *out, int num_sms,
                    cudaStream_t s)
{
    const long long total = static_cast<long long>(nv) * nr * nc;
    long long grid = (total + 255) / 256;
    if (grid > static_cast<long long>(num_sms) * 32) grid = static_cast<long long>(num_sms) * 32;
    if (grid < 1) grid = 1;
    forward_kernel<<<static_cast<unsigned>(grid), 256, 0, s>>>(views, kind, nv, nr, nc, du, dv, vol, box,
                                                               step_vox, out);
}

}  // namespace gct
