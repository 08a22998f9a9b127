// Voxel-driven backprojection over padded bilinear quads.
//
// Replaces the per-view loop of reconFDKHighMem (src/cuda/recon/fdk_axial.cuh:189-193): there,
// every view is copied into a cudaArray and one launch per view reads it through a bilinear
// texture and does vol += val * w (src/cuda/recon/back_proj.cuh:16-104), a full volume
// read-modify-write per view. Here one launch covers a range of views: each thread owns one
// (x, y) column and zpt voxels along z, keeps their sums in registers across all views and
// writes the volume once. Per view, the column's detector column u, its bilinear split and the
// backprojection weight are computed once (they do not depend on z for circular trajectories),
// and each voxel costs one row coordinate, one 8- or 16-byte quad load and three lerps.
// Mappings follow projMapping (src/cuda/geom/coord_trans_proj.cuh:157-345) through per-view
// coefficients in voxel-index space that the host derives in FP64.
#include "../../include/gct_fdk.h"
#include "common.cuh"
#include "geometry.hpp"
#include "kernels.hpp"

namespace gct {
namespace {

constexpr int kViewsPerChunk = 128;
constexpr int kC = kCoefPerView;

// Coefficient layouts (per view, kCoefPerView floats):
//  affine     : [0..2] u0, ui, uj; [3..4] v0, vk; [5] wscale
//  projective : [0..3] U numerator; [4..7] V numerator; [8..11] denominator D; [12] wscale
//               u = U/D, v = V/D, weight = wscale / D^2
//  arc        : [0..3] A = e_u.d; [4..7] B = e_w.d; [8..11] T = e_v.d; [12] 1/dgamma; [13] c0;
//               [14] SDD/dv; [15] r0; [16] wscale
//               u = atan2(A, B)/dgamma + c0, v = SDD T / sqrt(A^2+B^2) / dv + r0,
//               weight = wscale / (A^2 + B^2 + T^2)
// Each affine form is c0 + ci*i + cj*j + ck*k in voxel indices.
__device__ __forceinline__ int wscale_slot(int family) { return family == 0 ? 5 : family == 1 ? 12 : 16; }

template <class Q>
__device__ __forceinline__ float bilerp(const typename Q::storage *col, int qpitch, float fu,
                                        float v, float vmax)
{
    v = fminf(fmaxf(v, -1.0f), vmax);
    int iv;
    float fv;
    split_coord(v, iv, fv);
    const float4 q = Q::unpack(Q::load(col + (iv + kQuadPad) * qpitch));
    const float top = fmaf(fu, q.y - q.x, q.x);
    const float bot = fmaf(fu, q.w - q.z, q.z);
    return fmaf(fv, bot - top, top);
}

template <int FAMILY, class Q, int ZPT, bool ZAFFINE>
__global__ void __launch_bounds__(256) bp_kernel(BpArgs a)
{
    __shared__ float4 s_coef[kViewsPerChunk * kC / 4];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k0 = blockIdx.z * ZPT;
    const bool active = i < a.nx && j < a.ny;
    const float fi = static_cast<float>(i), fj = static_cast<float>(j);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nthr = blockDim.x * blockDim.y;
    using S = typename Q::storage;
    const S *quads = static_cast<const S *>(a.quads);

    float acc[ZPT];
#pragma unroll
    for (int z = 0; z < ZPT; ++z) acc[z] = 0.f;

    for (int vc = 0; vc < a.v_count; vc += kViewsPerChunk) {
        const int nvc = min(kViewsPerChunk, a.v_count - vc);
        __syncthreads();
        const float4 *g = reinterpret_cast<const float4 *>(a.coefs + static_cast<long long>(a.v_begin + vc) * kC);
        for (int t = tid; t < nvc * kC / 4; t += nthr) s_coef[t] = __ldg(g + t);
        __syncthreads();
        if (a.vinv) {
            for (int t = tid; t < nvc; t += nthr)
                reinterpret_cast<float *>(s_coef)[t * kC + wscale_slot(FAMILY)] *= __ldg(a.vinv + a.v_begin + vc + t);
            __syncthreads();
        }
        if (!active) continue;
        for (int vv = 0; vv < nvc; ++vv) {
            const float *c = reinterpret_cast<const float *>(s_coef) + vv * kC;
            const S *view = quads + static_cast<long long>(a.v_begin + vc + vv) * a.qview;
            if (FAMILY == 0) {
                // parallel kinds: u = u0 + ui i + uj j, v = v0 + vk k, weight constant
                float u = fmaf(c[2], fj, fmaf(c[1], fi, c[0]));
                u = fminf(fmaxf(u, -1.0f), a.umax);
                int iu;
                float fu;
                split_coord(u, iu, fu);
                const S *col = view + iu + kQuadPad;
                const float w = c[5];
#pragma unroll
                for (int z = 0; z < ZPT; ++z) {
                    const float v = fmaf(c[4], static_cast<float>(k0 + z), c[3]);
                    acc[z] = fmaf(w, bilerp<Q>(col, a.qpitch, fu, v, a.vmax), acc[z]);
                }
            } else if (FAMILY == 1) {
                if (ZAFFINE) {
                    const float D = fmaf(c[10], fj, fmaf(c[9], fi, c[8]));
                    const float inv = rcp_approx(D);
                    float u = fmaf(c[2], fj, fmaf(c[1], fi, c[0])) * inv;
                    u = fminf(fmaxf(u, -1.0f), a.umax);
                    int iu;
                    float fu;
                    split_coord(u, iu, fu);
                    const S *col = view + iu + kQuadPad;
                    const float w = c[12] * inv * inv;
                    const float vs = c[7] * inv;
                    const float v0 = fmaf(c[7], static_cast<float>(k0), fmaf(c[6], fj, fmaf(c[5], fi, c[4]))) * inv;
#pragma unroll
                    for (int z = 0; z < ZPT; ++z) {
                        const float v = fmaf(vs, static_cast<float>(z), v0);
                        acc[z] = fmaf(w, bilerp<Q>(col, a.qpitch, fu, v, a.vmax), acc[z]);
                    }
                } else {
#pragma unroll
                    for (int z = 0; z < ZPT; ++z) {
                        const float fk = static_cast<float>(k0 + z);
                        const float D = fmaf(c[11], fk, fmaf(c[10], fj, fmaf(c[9], fi, c[8])));
                        const float inv = rcp_approx(D);
                        float u = fmaf(c[3], fk, fmaf(c[2], fj, fmaf(c[1], fi, c[0]))) * inv;
                        const float v = fmaf(c[7], fk, fmaf(c[6], fj, fmaf(c[5], fi, c[4]))) * inv;
                        u = fminf(fmaxf(u, -1.0f), a.umax);
                        int iu;
                        float fu;
                        split_coord(u, iu, fu);
                        acc[z] = fmaf(c[12] * inv * inv,
                                      bilerp<Q>(view + iu + kQuadPad, a.qpitch, fu, v, a.vmax), acc[z]);
                    }
                }
            } else {
                if (ZAFFINE) {
                    const float A = fmaf(c[2], fj, fmaf(c[1], fi, c[0]));
                    const float B = fmaf(c[6], fj, fmaf(c[5], fi, c[4]));
                    const float rho2 = fmaf(A, A, B * B);
                    float u = fmaf(atan2f(A, B), c[12], c[13]);
                    u = fminf(fmaxf(u, -1.0f), a.umax);
                    int iu;
                    float fu;
                    split_coord(u, iu, fu);
                    const S *col = view + iu + kQuadPad;
                    const float vs = c[14] * rsqrtf(rho2);
                    const float T0 = fmaf(c[11], static_cast<float>(k0), c[8]);
#pragma unroll
                    for (int z = 0; z < ZPT; ++z) {
                        const float T = fmaf(c[11], static_cast<float>(z), T0);
                        const float v = fmaf(vs, T, c[15]);
                        const float w = c[16] * rcp_approx(fmaf(T, T, rho2));
                        acc[z] = fmaf(w, bilerp<Q>(col, a.qpitch, fu, v, a.vmax), acc[z]);
                    }
                } else {
#pragma unroll
                    for (int z = 0; z < ZPT; ++z) {
                        const float fk = static_cast<float>(k0 + z);
                        const float A = fmaf(c[3], fk, fmaf(c[2], fj, fmaf(c[1], fi, c[0])));
                        const float B = fmaf(c[7], fk, fmaf(c[6], fj, fmaf(c[5], fi, c[4])));
                        const float T = fmaf(c[11], fk, fmaf(c[10], fj, fmaf(c[9], fi, c[8])));
                        const float rho2 = fmaf(A, A, B * B);
                        float u = fmaf(atan2f(A, B), c[12], c[13]);
                        u = fminf(fmaxf(u, -1.0f), a.umax);
                        int iu;
                        float fu;
                        split_coord(u, iu, fu);
                        const float v = fmaf(c[14] * rsqrtf(rho2), T, c[15]);
                        const float w = c[16] * rcp_approx(fmaf(T, T, rho2));
                        acc[z] = fmaf(w, bilerp<Q>(view + iu + kQuadPad, a.qpitch, fu, v, a.vmax), acc[z]);
                    }
                }
            }
        }
    }
    if (!active) return;
#pragma unroll
    for (int z = 0; z < ZPT; ++z) {
        const int k = k0 + z;
        if (k < a.nz) {
            const long long idx = (static_cast<long long>(k) * a.ny + j) * a.nx + i;
            a.vol[idx] = a.accumulate ? a.vol[idx] + acc[z] : acc[z];
        }
    }
}

template <int FAMILY, class Q, int ZPT>
void launch_zpt(const BpArgs &a, bool z_affine, dim3 grid, dim3 block, cudaStream_t s)
{
    if (z_affine || FAMILY == 0)
        bp_kernel<FAMILY, Q, ZPT, true><<<grid, block, 0, s>>>(a);
    else
        bp_kernel<FAMILY, Q, ZPT, false><<<grid, block, 0, s>>>(a);
}

template <int FAMILY, class Q>
void launch_q(const BpArgs &a, bool z_affine, int zpt, int bx, int by, cudaStream_t s)
{
    const dim3 block(bx, by);
    const dim3 grid((a.nx + bx - 1) / bx, (a.ny + by - 1) / by, (a.nz + zpt - 1) / zpt);
    switch (zpt) {
        case 1: launch_zpt<FAMILY, Q, 1>(a, z_affine, grid, block, s); break;
        case 2: launch_zpt<FAMILY, Q, 2>(a, z_affine, grid, block, s); break;
        case 4: launch_zpt<FAMILY, Q, 4>(a, z_affine, grid, block, s); break;
        case 8: launch_zpt<FAMILY, Q, 8>(a, z_affine, grid, block, s); break;
        default: launch_zpt<FAMILY, Q, 16>(a, z_affine, grid, block, s); break;
    }
}

}  // namespace

void launch_backproject(const BpArgs &a, int family, int storage, bool z_affine, int zpt, int bx,
                        int by, cudaStream_t s)
{
    if (storage == 0) {
        if (family == 0) launch_q<0, QuadF32>(a, z_affine, zpt, bx, by, s);
        else if (family == 1) launch_q<1, QuadF32>(a, z_affine, zpt, bx, by, s);
        else launch_q<2, QuadF32>(a, z_affine, zpt, bx, by, s);
    } else {
        if (family == 0) launch_q<0, QuadF16>(a, z_affine, zpt, bx, by, s);
        else if (family == 1) launch_q<1, QuadF16>(a, z_affine, zpt, bx, by, s);
        else launch_q<2, QuadF16>(a, z_affine, zpt, bx, by, s);
    }
}

}  // namespace gct
