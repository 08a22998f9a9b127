// Host-side FP64 geometry. Each function cites the reference routine whose behaviour it keeps;
// the arithmetic is done in double instead of the reference's float.
#include "geometry.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <functional>
#include <numeric>

namespace gct {

namespace {
constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 2.0 * kPi;

double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
double norm3(const double *a) { return std::sqrt(dot3(a, a)); }
void cross3(const double *a, const double *b, double *c)
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
}  // namespace

[[noreturn]] void fail(gct_status s, const std::string &msg) { throw GctError{s, msg}; }

Family family_of(gct_geom_kind kind)
{
    switch (kind) {
        case GCT_GEOM_PARALLEL_1D:
        case GCT_GEOM_PARALLEL_2D:
        case GCT_GEOM_CONE_PARALLEL: return Family::Affine;
        case GCT_GEOM_FAN_LINE:
        case GCT_GEOM_CONE_FLAT: return Family::Projective;
        case GCT_GEOM_FAN_ARC:
        case GCT_GEOM_CONE_CYL: return Family::Arc;
    }
    fail(GCT_ERR_INVALID_ARG, "unknown geometry kind");
}

bool is_2d_detector(gct_geom_kind kind) { return kind >= GCT_GEOM_PARALLEL_2D; }

// src/cpp/geom/utils.h:338-348 (wrapFrom0To2PI). The reference wraps FP32 angles against its FP32
// 2*pi, so an angle within one FP32 step (4.8e-7 rad) of 2*pi wraps to 0 there; the same band
// is snapped here so FP32-sourced angles (e.g. float(2*pi)) analyse identically in FP64.
double wrap_0_2pi(double a)
{
    while (a < 0.0) a += kTwoPi;
    if (std::fabs(a - kTwoPi) <= 4.8e-7) return 0.0;
    return (a >= kTwoPi) ? std::remainder(a, kTwoPi) : a;
}

// src/cpp/geom/utils.h:370-389 (quadrantIndex).
unsigned quadrant_index(double a)
{
    const double w = wrap_0_2pi(a);
    if (w >= 0.0 && w < kPi / 2.0) return 1u;
    if (w >= kPi / 2.0 && w < kPi) return 2u;
    if (w >= kPi && w < 1.5 * kPi) return 3u;
    return 4u;
}

// src/cpp/geom/rotation_geom.cpp:255-295 (Detail::rotAng).
double view_rot_angle(gct_geom_kind kind, const gct_view_geom &v)
{
    if (family_of(kind) == Family::Affine) return wrap_0_2pi(v.rot_ang);
    return wrap_0_2pi(std::atan2(v.src_pos[1], v.src_pos[0]));
}

// src/cpp/geom/rotation_geom.cpp:7-43 (Detail::rotDir).
bool rotation_dir(const std::vector<double> &ang, int *dir)
{
    if (ang.size() < 2) return false;
    const double a0 = wrap_0_2pi(ang[0]), a1 = wrap_0_2pi(ang[1]);
    const unsigned q0 = quadrant_index(a0), q1 = quadrant_index(a1);
    if (q0 == 1u && q1 == 4u) {
        *dir = GCT_ROT_CCW;
    } else if (q0 == 4u && q1 == 1u) {
        *dir = GCT_ROT_CW;
    } else {
        const double diff = a1 - a0;
        if (diff > 0.0)
            *dir = GCT_ROT_CW;
        else if (diff < 0.0)
            *dir = GCT_ROT_CCW;
        else
            return false;
    }
    return true;
}

// src/cpp/geom/rotation_geom.cpp:45-74 (Detail::relRotAngles).
bool rel_rot_angles(const std::vector<double> &ang, std::vector<double> *rel)
{
    int dir = 0;
    if (!rotation_dir(ang, &dir)) return false;
    rel->clear();
    rel->reserve(ang.size());
    const double first = ang.front();
    for (double a : ang) rel->push_back(wrap_0_2pi(dir == GCT_ROT_CCW ? first - a : a - first));
    return true;
}

// src/cpp/geom/rotation_geom.cpp:76-91 (Detail::rotAngIncr): mean of wrapped differences.
bool rot_ang_incr(const std::vector<double> &rel, double *incr)
{
    if (rel.empty()) return false;
    double sum = 0.0;
    for (size_t i = 0; i + 1 < rel.size(); ++i) sum += wrap_0_2pi(rel[i + 1] - rel[i]);
    *incr = sum / static_cast<double>(rel.size() - 1);
    return true;
}

// src/cpp/geom/rotation_geom.cpp:93-104 (Detail::rotAngRange).
bool rot_ang_range(const std::vector<double> &rel, double *range)
{
    double incr = 0.0;
    if (!rot_ang_incr(rel, &incr)) return false;
    *range = incr + *std::max_element(rel.begin(), rel.end());
    return true;
}

// src/cpp/geom/rotation_geom.cpp:106-134 (Detail::numProjPerRot).
bool num_proj_per_rot(const std::vector<double> &rel, unsigned *n)
{
    if (rel.empty() || rel.front() != 0.0) return false;
    for (size_t i = 1; i < rel.size(); ++i) {
        if (std::fabs(rel[i]) < 1e-6) {
            *n = static_cast<unsigned>(i);
            return true;
        }
    }
    *n = static_cast<unsigned>(rel.size());
    return true;
}

// src/cpp/geom/rotation_geom.h:90-115 (getRotationGeom).
bool rotation_info(const gct_ct_geom &g, RotationInfo *out)
{
    const auto kind = static_cast<gct_geom_kind>(g.kind);
    out->rot_ang.resize(g.num_views);
    for (unsigned v = 0; v < g.num_views; ++v) out->rot_ang[v] = view_rot_angle(kind, g.views[v]);
    if (!rotation_dir(out->rot_ang, &out->dir)) return false;
    if (!rel_rot_angles(out->rot_ang, &out->rel_rot_ang)) return false;
    if (!rot_ang_incr(out->rel_rot_ang, &out->incr)) return false;
    if (!rot_ang_range(out->rel_rot_ang, &out->range)) return false;
    if (!num_proj_per_rot(out->rel_rot_ang, &out->num_proj_per_rot)) return false;
    return true;
}

void check_ct_geom(const gct_ct_geom *g)
{
    if (!g) fail(GCT_ERR_INVALID_ARG, "geometry is NULL");
    if (g->kind < GCT_GEOM_PARALLEL_1D || g->kind > GCT_GEOM_CONE_FLAT)
        fail(GCT_ERR_INVALID_ARG, "unknown geometry kind " + std::to_string(g->kind));
    const auto kind = static_cast<gct_geom_kind>(g->kind);
    if (g->num_views == 0 || !g->views)
        fail(GCT_ERR_INVALID_ARG, "Empty collection of projection geometry.");
    if (g->det_row.num_samples == 0 || !(g->det_row.sampling_width > 0.0))
        fail(GCT_ERR_INVALID_ARG, "detector row sampler must have samples and a positive width");
    if (is_2d_detector(kind)) {
        if (g->det_col.num_samples == 0 || !(g->det_col.sampling_width > 0.0))
            fail(GCT_ERR_INVALID_ARG, "detector column sampler must have samples and a positive width");
    } else if (g->det_col.num_samples > 1) {
        fail(GCT_ERR_INVALID_ARG, "1D detector kinds take det_col.num_samples <= 1");
    }
    if (g->det_row.num_samples > 16384 || (is_2d_detector(kind) && g->det_col.num_samples > 65536))
        fail(GCT_ERR_NOT_SUPPORTED, "detector larger than 16384 columns or 65536 rows");
}

void check_vol_geom(const gct_vol_geom *v, bool volume_3d)
{
    if (!v) fail(GCT_ERR_INVALID_ARG, "volume geometry is NULL");
    // src/cpp/geom/recon_img_geom.h:57-70 (isSamplingValid).
    if (v->nx == 0 || v->ny == 0 || v->nz == 0)
        fail(GCT_ERR_INVALID_ARG, "The number of samples in any dimension cannot be zero.");
    if (!(v->dx > 0.0) || !(v->dy > 0.0) || (volume_3d && !(v->dz > 0.0)))
        fail(GCT_ERR_INVALID_ARG,
             "The sampling width of the image in any dimension cannot be zero or negative.");
    if (!volume_3d && v->nz != 1) fail(GCT_ERR_INVALID_ARG, "2D images take nz = 1");
}

// src/cpp/io/geom_reader/proj_geom_factory_params.cpp:8-108 with the cone-beam rotation of
// proj_geom_cb_factory.cpp:14-48 (R_z(dir*theta) applied to the basis u=(0,1,0), v=(0,0,-1),
// w=(-1,0,0) and to the source (SID, 0, -pitch*theta)) and the fan-beam reduction of
// proj_geom_fb_factory.cpp:13-45 (keep x, y; the fan-beam path drops the pitch).
gct_view_geom make_view(gct_geom_kind kind, const gct_geom_params &p, unsigned idx)
{
    gct_view_geom v{};
    const double theta = p.init_ang + p.ang_incr * static_cast<double>(idx);
    v.det_row_center = p.det_row_center;
    if (family_of(kind) == Family::Affine) {
        v.rot_ang = theta;
        if (kind != GCT_GEOM_PARALLEL_1D) v.det_col_center = p.det_col_center;
        if (kind == GCT_GEOM_CONE_PARALLEL) {
            v.src_det_dist = p.src_det_dist;
            v.src_iso_dist = p.src_iso_dist;
        }
        return v;
    }
    const bool fan = !is_2d_detector(kind);
    const double phi = static_cast<double>(p.rot_dir) * theta;
    const double c = std::cos(phi), s = std::sin(phi);
    const double pitch = fan ? 0.0 : p.hel_pitch;
    v.src_det_dist = p.src_det_dist;
    v.src_iso_dist = p.src_iso_dist;
    v.src_pos[0] = p.src_iso_dist * c;
    v.src_pos[1] = p.src_iso_dist * s;
    v.src_pos[2] = fan ? 0.0 : -pitch * theta;
    v.det_row_dir[0] = -s;
    v.det_row_dir[1] = c;
    v.det_row_dir[2] = 0.0;
    if (!fan) {
        v.det_col_center = p.det_col_center;
        v.det_col_dir[0] = 0.0;
        v.det_col_dir[1] = 0.0;
        v.det_col_dir[2] = -1.0;
    }
    if (kind == GCT_GEOM_FAN_ARC || kind == GCT_GEOM_CONE_CYL) {
        v.iso_ray_dir[0] = -c;
        v.iso_ray_dir[1] = -s;
        v.iso_ray_dir[2] = 0.0;
    }
    return v;
}

// src/cpp/recon/ramp_filter.h:22-56 (RampFilter::kernel, M(t), apodFact in ramp_filter.cpp:5-20)
// and src/cpp/recon/proj_filt_kernel.cpp:5-45 (projFiltKernel, (b/sin b)^2 for the arc).
std::vector<double> ramp_taps(gct_geom_kind kind, const gct_detector &det_row,
                              const gct_filt_params &fp)
{
    const int n = static_cast<int>(det_row.num_samples);
    const double a = fp.apod_func == GCT_APOD_HANN ? 0.5 : fp.apod_func == GCT_APOD_HAMMING ? 0.54 : 1.0;
    const double fc = fp.cut_off_freq;
    const double sw = det_row.sampling_width;
    auto M = [](double t) { return t == 0.0 ? 0.5 : std::sin(t) / t + (std::cos(t) - 1.0) / (t * t); };
    std::vector<double> h(n);
    const bool arc = kind == GCT_GEOM_FAN_ARC || kind == GCT_GEOM_CONE_CYL;
    for (int j = 0; j < n; ++j) {
        const int off = j - n / 2;
        const double nd = static_cast<double>(off);
        double c = (fc * fc / (2.0 * sw)) *
                   (a * M(fc * kPi * nd) + ((1.0 - a) / 2.0) * M(kPi * fc * nd + kPi) +
                    ((1.0 - a) / 2.0) * M(kPi * fc * nd - kPi));
        if (arc && off != 0) {
            const double beta = nd * sw;
            const double r = beta / std::sin(beta);
            c *= r * r;
        }
        h[j] = c;
    }
    return h;
}

// src/cuda/recon/parker_weighting.cuh:19-58 (fanAngle, fanAngleDet), :80-105 (parkerWeightFan),
// :132-176 (getParkerWeights; fan angles from view 0, relative angles reversed for CCW, weights
// only when the range exceeds pi) and :181-200 (parallel kinds: 1 or 0.5).
std::vector<double> parker_table(const gct_ct_geom &g, const RotationInfo &ri)
{
    const auto kind = static_cast<gct_geom_kind>(g.kind);
    const unsigned nc = g.det_row.num_samples, nv = g.num_views;
    std::vector<double> w(static_cast<size_t>(nc) * nv, 1.0);
    if (family_of(kind) == Family::Affine) {
        const bool half = ri.incr > 0.0 && ri.range <= ri.incr + kPi;
        std::fill(w.begin(), w.end(), half ? 1.0 : 0.5);
        return w;
    }
    if (!(ri.range > kPi)) return w;  // reference leaves these uninitialised; defined as 1 here
    const gct_view_geom &v0 = g.views[0];
    const bool arc = kind == GCT_GEOM_FAN_ARC || kind == GCT_GEOM_CONE_CYL;
    std::vector<double> gamma(nc);
    for (unsigned c = 0; c < nc; ++c) {
        const double t = (static_cast<double>(c) - v0.det_row_center) * g.det_row.sampling_width;
        gamma[c] = arc ? t : std::atan2(t, v0.src_det_dist);
    }
    std::vector<double> rel = ri.rel_rot_ang;
    if (ri.dir == GCT_ROT_CCW) std::reverse(rel.begin(), rel.end());
    const double phi = ri.range;
    for (unsigned v = 0; v < nv; ++v) {
        const double b = rel[v];
        for (unsigned c = 0; c < nc; ++c) {
            const double gm = gamma[c];
            const double t2 = 2.0 * gm + phi - kPi, t3 = 2.0 * gm + kPi, t4 = phi;
            double wt = 0.0;
            if (b >= 0.0 && b <= t2) {
                const double s = std::sin(kPi * b / (2.0 * (phi - kPi) + 4.0 * gm));
                wt = s * s;
            } else if (b >= t2 && b <= t3) {
                wt = 1.0;
            } else if (b >= t3 && b <= t4) {
                const double s = std::sin(kPi * (phi - b) / (2.0 * (phi - kPi) - 4.0 * gm));
                wt = s * s;
            }
            w[static_cast<size_t>(v) * nc + c] = wt;
        }
    }
    return w;
}

unsigned fft_length(unsigned n)
{
    const long need = std::max<long>(2L * n - 2 - n / 2, static_cast<long>(n) - 1 + n / 2);
    unsigned L = 256;  // the FFT filter runs transforms of 256 to 8192 points
    while (static_cast<long>(L) <= need) L *= 2u;
    return L;
}

std::vector<std::complex<double>> filter_spectrum(const std::vector<double> &taps, unsigned L)
{
    const int n = static_cast<int>(taps.size());
    std::vector<double> hc(L, 0.0);
    for (int j = 0; j < n; ++j) {
        const int off = j - n / 2;
        hc[static_cast<unsigned>((off % static_cast<int>(L) + static_cast<int>(L)) % static_cast<int>(L))] += taps[j];
    }
    std::vector<double> cs(L), sn(L);
    for (unsigned m = 0; m < L; ++m) {
        cs[m] = std::cos(kTwoPi * m / L);
        sn[m] = std::sin(kTwoPi * m / L);
    }
    std::vector<std::complex<double>> H(L);
    for (unsigned k = 0; k < L; ++k) {
        double re = 0.0, im = 0.0;
        for (unsigned m = 0; m < L; ++m) {
            if (hc[m] == 0.0) continue;
            const unsigned idx = static_cast<unsigned>((static_cast<unsigned long long>(k) * m) % L);
            re += hc[m] * cs[idx];
            im -= hc[m] * sn[idx];
        }
        H[k] = std::complex<double>(re / L, im / L);
    }
    return H;
}

// Per-view quantities as the reference's CTGeomDev stores them (src/cuda/geom/ct_geom_dev.cu:
// SID = |src_pos| for the fan and cone kinds (:84, :145, :302, :398), the fan-line iso-ray as
// rot90(det_row_dir) (:154), the flat detector normal as det_row_dir x det_col_dir (:407)).
ViewDerived derive_view(gct_geom_kind kind, const gct_ct_geom &g, unsigned vi)
{
    const gct_view_geom &v = g.views[vi];
    ViewDerived d;
    d.c0 = v.det_row_center;
    d.r0 = is_2d_detector(kind) ? v.det_col_center : 0.0;
    d.theta = v.rot_ang;
    const bool fan1d = kind == GCT_GEOM_FAN_ARC || kind == GCT_GEOM_FAN_LINE;
    switch (kind) {
        case GCT_GEOM_PARALLEL_1D:
        case GCT_GEOM_PARALLEL_2D: d.bp_const = 1.0; break;
        case GCT_GEOM_CONE_PARALLEL:
            d.sdd = v.src_det_dist;
            d.sid = v.src_iso_dist;
            d.bp_const = 1.0;
            break;
        default: {
            d.sdd = v.src_det_dist;
            for (int i = 0; i < 3; ++i) {
                d.src[i] = v.src_pos[i];
                d.eu[i] = v.det_row_dir[i];
            }
            if (fan1d) {
                d.src[2] = 0.0;
                d.eu[2] = 0.0;
            }
            d.sid = norm3(d.src);
            if (kind == GCT_GEOM_FAN_LINE) {
                d.ew[0] = -d.eu[1];
                d.ew[1] = d.eu[0];
                d.ew[2] = 0.0;
            } else if (kind == GCT_GEOM_CONE_FLAT) {
                for (int i = 0; i < 3; ++i) d.ev[i] = v.det_col_dir[i];
                cross3(d.eu, d.ev, d.ew);
            } else {  // arc kinds
                for (int i = 0; i < 3; ++i) d.ew[i] = v.iso_ray_dir[i];
                if (fan1d) d.ew[2] = 0.0;
                if (kind == GCT_GEOM_CONE_CYL)
                    for (int i = 0; i < 3; ++i) d.ev[i] = v.det_col_dir[i];
            }
            d.bp_const = (family_of(kind) == Family::Projective) ? d.sdd * d.sid : d.sid;
            break;
        }
    }
    return d;
}

// Per-view coefficients in voxel-index space (i, j, k) -> detector pixel coordinates.
// Voxel centres follow src/cuda/geom/coord_trans_img.cuh:52-66: first = mid - (n-1)*w/2.
// Mapping formulas follow src/cuda/geom/coord_trans_proj.cuh:157-345 (projMapping) with
// DCSToPCS (:142-145): pixel = coord / width + centre.
std::vector<float> bp_coefficients(const gct_ct_geom &g, const gct_vol_geom &vol,
                                   const std::vector<ViewDerived> &vd,
                                   const std::vector<double> &wscale, bool *z_affine,
                                   std::vector<double> *c64)
{
    const auto kind = static_cast<gct_geom_kind>(g.kind);
    const bool vol3d = is_2d_detector(kind);
    const double X0[3] = {vol.mid[0] - (vol.nx - 1.0) * vol.dx / 2.0,
                          vol.mid[1] - (vol.ny - 1.0) * vol.dy / 2.0,
                          vol3d ? vol.mid[2] - (vol.nz - 1.0) * vol.dz / 2.0 : 0.0};
    const double DX[3] = {vol.dx, vol.dy, vol3d ? vol.dz : 0.0};
    const double du = g.det_row.sampling_width;
    const double dv = vol3d ? g.det_col.sampling_width : 1.0;
    std::vector<double> cd(static_cast<size_t>(g.num_views) * kCoefPerView, 0.0);
    bool affine_z = true;
    // affine form of e . (X - S): value at (0,0,0) and slopes per index step.
    auto aff = [&](const double *e, const double *S, double *c4) {
        double base[3];
        for (int i = 0; i < 3; ++i) base[i] = X0[i] - S[i];
        c4[0] = dot3(e, base);
        for (int i = 0; i < 3; ++i) c4[1 + i] = e[i] * DX[i];
    };
    for (unsigned v = 0; v < g.num_views; ++v) {
        const ViewDerived &d = vd[v];
        double *c = &cd[static_cast<size_t>(v) * kCoefPerView];
        switch (family_of(kind)) {
            case Family::Affine: {
                // detCoordAxialParallel (coord_trans_proj.cuh:157-166): x cos(t+pi/2) + y sin(t+pi/2).
                const double t = d.theta + kPi / 2.0;
                const double ct = std::cos(t), st = std::sin(t);
                c[0] = (X0[0] * ct + X0[1] * st) / du + d.c0;
                c[1] = DX[0] * ct / du;
                c[2] = DX[1] * st / du;
                double vk = 0.0, v0 = 0.0;
                if (kind == GCT_GEOM_PARALLEL_2D) {  // t = -z
                    v0 = -X0[2] / dv + d.r0;
                    vk = -DX[2] / dv;
                } else if (kind == GCT_GEOM_CONE_PARALLEL) {  // t = -z * SDD / SID
                    const double m = d.sdd / d.sid;
                    v0 = -X0[2] * m / dv + d.r0;
                    vk = -DX[2] * m / dv;
                }
                c[3] = v0;
                c[4] = vk;
                c[5] = wscale[v];
                break;
            }
            case Family::Projective: {
                double U[4], V[4] = {0, 0, 0, 0}, D[4];
                aff(d.eu, d.src, U);
                aff(d.ew, d.src, D);
                if (vol3d) aff(d.ev, d.src, V);
                for (int i = 0; i < 4; ++i) {
                    c[i] = d.sdd / du * U[i] + d.c0 * D[i];
                    c[4 + i] = vol3d ? d.sdd / dv * V[i] + d.r0 * D[i] : 0.0;
                    c[8 + i] = D[i];
                }
                c[12] = wscale[v];
                if (U[3] != 0.0 || D[3] != 0.0) affine_z = false;
                break;
            }
            case Family::Arc: {
                double A[4], B[4], T[4] = {0, 0, 0, 0};
                aff(d.eu, d.src, A);
                aff(d.ew, d.src, B);
                if (vol3d) aff(d.ev, d.src, T);
                for (int i = 0; i < 4; ++i) {
                    c[i] = A[i];
                    c[4 + i] = B[i];
                    c[8 + i] = T[i];
                }
                c[12] = 1.0 / du;
                c[13] = d.c0;
                c[14] = vol3d ? d.sdd / dv : 0.0;
                c[15] = d.r0;
                c[16] = wscale[v];
                if (A[3] != 0.0 || B[3] != 0.0 || T[1] != 0.0 || T[2] != 0.0) affine_z = false;
                break;
            }
        }
    }
    *z_affine = affine_z;
    std::vector<float> out(cd.size());
    for (size_t n = 0; n < cd.size(); ++n) out[n] = static_cast<float>(cd[n]);
    if (c64) *c64 = std::move(cd);
    return out;
}

int quarter_turn_symmetry(gct_geom_kind kind, const std::vector<double> &c64, unsigned nv, unsigned nx,
                          unsigned ny, unsigned nz)
{
    if (nv < 4 || nv % 4 != 0 || nx != ny || nx % 2 != 0 || c64.size() != static_cast<size_t>(nv) * kCoefPerView)
        return 0;
    // Affine forms c0 + ci i + cj j + ck k of each family as slot indices (-1: absent), and the
    // per-view weight scale, which may differ between partner views. Every other slot must match.
    struct Form {
        int c0, ci, cj, ck;
    };
    std::vector<Form> forms;
    int free_slot = -1;
    switch (family_of(kind)) {
        case Family::Affine: forms = {{0, 1, 2, -1}, {3, 6, 7, 4}}; free_slot = 5; break;
        case Family::Projective: forms = {{0, 1, 2, 3}, {4, 5, 6, 7}, {8, 9, 10, 11}}; free_slot = 12; break;
        case Family::Arc: forms = {{0, 1, 2, 3}, {4, 5, 6, 7}, {8, 9, 10, 11}}; free_slot = 16; break;
    }
    bool in_form[kCoefPerView] = {};
    for (const Form &f : forms)
        for (int s : {f.c0, f.ci, f.cj, f.ck})
            if (s >= 0) in_form[s] = true;
    const double n1 = nx - 1.0, kRel = 1e-9;
    const unsigned q = nv / 4;
    for (int dir : {1, -1}) {
        bool ok = true;
        for (unsigned v = 0; ok && v + q < nv; ++v) {
            const double *a = &c64[static_cast<size_t>(v) * kCoefPerView];
            const double *b = &c64[static_cast<size_t>(v + q) * kCoefPerView];
            for (const Form &f : forms) {
                const double c0 = a[f.c0], ci = a[f.ci], cj = a[f.cj], ck = f.ck >= 0 ? a[f.ck] : 0.0;
                // b's form at R(i, j) equals a's at (i, j): R = (n-1-j, i) for +1, (j, n-1-i) for -1
                const double e0 = dir > 0 ? c0 + cj * n1 : c0 + ci * n1;
                const double ei = dir > 0 ? -cj : cj, ej = dir > 0 ? ci : -ci;
                const double scale = std::max({std::fabs(c0), std::fabs(ci) * nx, std::fabs(cj) * nx,
                                               std::fabs(ck) * nz, std::fabs(b[f.c0])});
                const double tol = kRel * scale;
                if (std::fabs(b[f.c0] - e0) > tol || std::fabs(b[f.ci] - ei) > tol || std::fabs(b[f.cj] - ej) > tol ||
                    (f.ck >= 0 && std::fabs(b[f.ck] - ck) > tol)) {
                    ok = false;
                    break;
                }
            }
            for (int s = 0; ok && s < kCoefPerView; ++s)
                if (!in_form[s] && s != free_slot &&
                    std::fabs(a[s] - b[s]) > kRel * std::max(std::fabs(a[s]), std::fabs(b[s])))
                    ok = false;
        }
        if (ok) return dir;
    }
    return 0;
}

bool z_mirror_symmetry(gct_geom_kind kind, const std::vector<double> &c64, unsigned nv, unsigned nr, unsigned nx,
                       unsigned ny, unsigned nz)
{
    if (nz < 2 || nz % 2 != 0 || nv == 0 || c64.size() != static_cast<size_t>(nv) * kCoefPerView) return false;
    const Family fam = family_of(kind);
    if (fam == Family::Arc) return false;
    const double K = nz - 1.0, m = nr - 1.0, kRel = 1e-9;
    for (unsigned v = 0; v < nv; ++v) {
        const double *c = &c64[static_cast<size_t>(v) * kCoefPerView];
        // v(i, j, k) + v(i, j, K - k) = m for every (i, j): the row form's constant, i and j parts
        double d0, di, dj, scale;
        if (fam == Family::Affine) {  // v = c3 + c6 i + c7 j + c4 k
            d0 = 2.0 * c[3] + c[4] * K - m;
            di = 2.0 * c[6];
            dj = 2.0 * c[7];
            scale = std::max({std::fabs(c[3]), std::fabs(c[4]) * nz, m});
        } else {  // v = (c4 + c5 i + c6 j + c7 k) / D, D = c8 + c9 i + c10 j (z-affine: c3 = c11 = 0)
            if (c[3] != 0.0 || c[11] != 0.0) return false;
            d0 = 2.0 * c[4] + c[7] * K - m * c[8];
            di = 2.0 * c[5] - m * c[9];
            dj = 2.0 * c[6] - m * c[10];
            scale = std::max({std::fabs(c[4]), std::fabs(c[7]) * nz, m * std::fabs(c[8]), std::fabs(c[5]) * nx,
                              std::fabs(c[6]) * ny, m * std::fabs(c[9]) * nx, m * std::fabs(c[10]) * ny});
        }
        const double tol = kRel * scale;
        if (std::fabs(d0) > tol || std::fabs(di) * nx > tol || std::fabs(dj) * ny > tol) return false;
    }
    return true;
}

// ---- projection matrices -----------------------------------------------------------------------

namespace {
void mat3_inverse(const double *a, double *inv)
{
    const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
    const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    if (!(std::fabs(det) > 0.0) || !std::isfinite(det)) fail(GCT_ERR_INVALID_ARG, "singular projection matrix");
    const double r = 1.0 / det;
    inv[0] = c00 * r;
    inv[1] = (a[2] * a[7] - a[1] * a[8]) * r;
    inv[2] = (a[1] * a[5] - a[2] * a[4]) * r;
    inv[3] = c01 * r;
    inv[4] = (a[0] * a[8] - a[2] * a[6]) * r;
    inv[5] = (a[2] * a[3] - a[0] * a[5]) * r;
    inv[6] = c02 * r;
    inv[7] = (a[1] * a[6] - a[0] * a[7]) * r;
    inv[8] = (a[0] * a[4] - a[1] * a[3]) * r;
}
void mat3_mul(const double *a, const double *b, double *c)
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) c[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
}
}  // namespace

// ProjectionMatrix(matrix) (src/cpp/geom/projection_matrix.cpp:4-62): with M the left 3 x 3 block,
// QR of M^-1 = Q U gives M = U^-1 Q^T, so K = U^-1 (upper triangular) and R = Q^T; signs are fixed
// so that K has a positive diagonal, K is normalised to K[2][2] = 1 and the source is
// -M^-1 times the fourth column. FP64 throughout (the reference keeps FP32 copies). The QR here is
// modified Gram-Schmidt on the three columns, which with the sign rule gives the same K and R as
// the reference's Householder QR.
ProjMatrix decompose_projection_matrix(const double *m)
{
    ProjMatrix pm{};
    std::copy(m, m + 12, pm.m);
    const double M[9] = {m[0], m[1], m[2], m[4], m[5], m[6], m[8], m[9], m[10]};
    double Mi[9];
    mat3_inverse(M, Mi);
    // columns of Mi -> Q (columns q0..q2) and U
    double q[3][3], U[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = 0; j < 3; ++j) {
        double a[3] = {Mi[j], Mi[3 + j], Mi[6 + j]};
        for (int k = 0; k < j; ++k) {
            const double r = q[k][0] * a[0] + q[k][1] * a[1] + q[k][2] * a[2];
            U[3 * k + j] = r;
            for (int t = 0; t < 3; ++t) a[t] -= r * q[k][t];
        }
        const double n = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        if (!(n > 0.0)) fail(GCT_ERR_INVALID_ARG, "singular projection matrix");
        U[3 * j + j] = n;
        for (int t = 0; t < 3; ++t) q[j][t] = a[t] / n;
    }
    double K[9];
    mat3_inverse(U, K);
    K[3] = K[6] = K[7] = 0.0;  // exactly upper triangular
    double R[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[3 * i + j] = q[i][j];  // R = Q^T: row i is column q_i
    for (int d = 0; d < 3; ++d) {
        const double sgn = std::copysign(1.0, K[4 * d]);
        for (int i = 0; i < 3; ++i) K[3 * i + d] *= sgn;  // K D
        for (int j = 0; j < 3; ++j) R[3 * d + j] *= sgn;  // D R
    }
    const double k22 = K[8];
    for (double &k : K) k /= k22;
    std::copy(K, K + 9, pm.K);
    std::copy(R, R + 9, pm.R);
    for (int i = 0; i < 3; ++i) pm.src[i] = -(Mi[3 * i] * m[3] + Mi[3 * i + 1] * m[7] + Mi[3 * i + 2] * m[11]);
    return pm;
}

// ProjectionMatrix(ProjGeom<DetFanLine, DetFanLine>, pix_width, pix_height)
// (projection_matrix.cpp:64-97): K from the source-detector distance in pixels and the centres,
// R from the detector directions and their cross product, M = K [R | -R src] scaled to M[2][3] = 1.
ProjMatrix compose_projection_matrix(const gct_view_geom &v, double pix_w, double pix_h)
{
    if (!(pix_w > 0.0) || !(pix_h > 0.0)) fail(GCT_ERR_INVALID_ARG, "pixel sizes must be positive");
    ProjMatrix pm{};
    const double K[9] = {v.src_det_dist / pix_w, 0.0, v.det_row_center, 0.0, v.src_det_dist / pix_h, v.det_col_center,
                         0.0, 0.0, 1.0};
    double w[3];
    cross3(v.det_row_dir, v.det_col_dir, w);
    const double R[9] = {v.det_row_dir[0], v.det_row_dir[1], v.det_row_dir[2], v.det_col_dir[0], v.det_col_dir[1],
                         v.det_col_dir[2], w[0], w[1], w[2]};
    double KR[9];
    mat3_mul(K, R, KR);
    double t[3];
    for (int i = 0; i < 3; ++i) t[i] = -(R[3 * i] * v.src_pos[0] + R[3 * i + 1] * v.src_pos[1] + R[3 * i + 2] * v.src_pos[2]);
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) pm.m[4 * i + j] = KR[3 * i + j];
        pm.m[4 * i + 3] = K[3 * i] * t[0] + K[3 * i + 1] * t[1] + K[3 * i + 2] * t[2];
    }
    const double s = pm.m[11];
    if (!(std::fabs(s) > 0.0)) fail(GCT_ERR_INVALID_ARG, "the source lies in the detector's plane through the origin");
    for (double &x : pm.m) x /= s;
    std::copy(K, K + 9, pm.K);
    std::copy(R, R + 9, pm.R);
    std::copy(v.src_pos, v.src_pos + 3, pm.src);
    return pm;
}

// ProjGeomFactory<DetFanLine, DetFanLine>::create(ProjectionMatrix)
// (src/cpp/io/geom_reader/proj_geom_factory_proj_mat.cpp:7-26): the flat-panel view of a matrix.
// As in the reference, the source-detector distance is the focal length in detector-row pixels
// (the caller multiplies by the pixel width).
gct_view_geom view_from_projection_matrix(const ProjMatrix &pm)
{
    gct_view_geom v{};
    v.src_det_dist = pm.K[0];
    v.det_row_center = pm.K[2];
    v.det_col_center = pm.K[5];
    for (int i = 0; i < 3; ++i) {
        v.src_pos[i] = pm.src[i];
        v.det_row_dir[i] = pm.R[i];
        v.det_col_dir[i] = pm.R[3 + i];
    }
    v.src_iso_dist = norm3(v.src_pos);
    v.rot_ang = view_rot_angle(GCT_GEOM_CONE_FLAT, v);
    return v;
}

// ---- spiral scans --------------------------------------------------------------------------------

// SpiralCTGeom's constructor (src/cpp/geom/spiral_ct_geom.h:30-50): a 2D detector, a positive
// number of projections per rotation, source z sorted either way and a positive pitch (the source
// z travel over one rotation / 2 pi).
SpiralInfo spiral_info(const gct_ct_geom &g)
{
    const auto kind = static_cast<gct_geom_kind>(g.kind);
    if (!is_2d_detector(kind) || family_of(kind) == Family::Affine)
        fail(GCT_ERR_NOT_SUPPORTED, "spiral scans need a cone-beam 2D detector (flat or cylindrical)");
    RotationInfo ri;
    if (!rotation_info(g, &ri)) fail(GCT_ERR_INVALID_ARG, "Invalid X-ray source trajectory.");
    if (ri.num_proj_per_rot == 0)
        fail(GCT_ERR_INVALID_ARG, "Invalid spiral CT geometry: number of projections per rotation should not be zero.");
    SpiralInfo si;
    si.npr = ri.num_proj_per_rot;
    si.src_z.resize(g.num_views);
    for (unsigned v = 0; v < g.num_views; ++v) si.src_z[v] = g.views[v].src_pos[2];
    if (!std::is_sorted(si.src_z.begin(), si.src_z.end()) &&
        !std::is_sorted(si.src_z.begin(), si.src_z.end(), std::greater<>()))
        fail(GCT_ERR_INVALID_ARG, "Invalid spiral CT geometry: the z-coordinate of source position should be sorted "
                                  "either in ascending or descending order.");
    if (si.npr >= g.num_views)
        fail(GCT_ERR_INVALID_ARG, "Invalid spiral CT geometry: the scan covers less than one rotation after the first");
    si.pitch = std::fabs(si.src_z.front() - si.src_z[si.npr]) / kTwoPi;
    if (!(si.pitch > 0.0))
        fail(GCT_ERR_INVALID_ARG, "Invalid spiral CT geometry: spiral pitch cannot be zero or negative.");
    return si;
}

// firstAndLastProjIndices (spiral_ct_geom.h:57-75): the view whose source z is nearest the slice
// (the first of equals), and the npr views starting npr / 2 before it. Signed here: the
// reference's unsigned first index wraps when it would be negative, and fdk_spiral.cuh:60-79 then
// does no work for the slice, as it does for first == 0 or last >= num_views.
void spiral_window(const SpiralInfo &si, double slice_pos, long long *first, long long *last)
{
    size_t mid = 0;
    double best = std::fabs(si.src_z[0] - slice_pos);
    for (size_t v = 1; v < si.src_z.size(); ++v) {
        const double d = std::fabs(si.src_z[v] - slice_pos);
        if (d < best) {
            best = d;
            mid = v;
        }
    }
    *first = static_cast<long long>(mid) - static_cast<long long>(si.npr / 2);
    *last = *first + si.npr;
}

}  // namespace gct

