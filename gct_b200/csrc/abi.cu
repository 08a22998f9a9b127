// C ABI of the FDK engine (include/gct_fdk.h): plans, execution, stage entry points and the
// host geometry functions. All failures become a gct_status plus a thread-local message.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gct_fdk.h"
#include "filter_gemm.hpp"
#include "plan.hpp"
#include "project.hpp"

thread_local std::string g_last_error;

gct_status set_error(gct_status s, const std::string &msg)
{
    g_last_error = msg;
    return s;
}

void cuda_check(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return;
    const gct_status s = (e == cudaErrorMemoryAllocation) ? GCT_ERR_OUT_OF_MEMORY : GCT_ERR_CUDA;
    cudaGetLastError();  // clear the sticky-free error state for the next call
    gct::fail(s, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {

bool orthonormal(const double *a, const double *b, double tol)
{
    auto dot = [](const double *x, const double *y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
    return std::fabs(dot(a, a) - 1.0) < tol && std::fabs(dot(b, b) - 1.0) < tol && std::fabs(dot(a, b)) < tol;
}

}  // namespace

namespace {

// FP16 value of x as the 16-bit pattern the GEMM buffers hold; `back` gets its value.
__nv_bfloat16 f16_bits(double x, double &back)
{
    const __half h = __float2half_rn(static_cast<float>(x));
    back = static_cast<double>(__half2float(h));
    __nv_bfloat16 b;
    std::memcpy(&b, &h, sizeof(b));
    return b;
}

// Tap pieces of the FP16 form (filter_gemm.cu): taps scaled by a power of two so that the largest
// is below 2^14; within the band |c - k| <= kGemmBand three FP16 pieces, beyond it the hi piece
// alone, and per output column c the parts dropped beyond the band added to its central tap (before
// that tap is split), so every column's sum of taps keeps its exact value.
void toeplitz_f16(gct_fdk_plan *p, const std::vector<double> &taps, std::vector<__nv_bfloat16> &bh,
                  std::vector<__nv_bfloat16> &bl, std::vector<__nv_bfloat16> &bll)
{
    double tmax = 0.0;
    for (double t : taps) tmax = std::max(tmax, std::fabs(t));
    int e = 0;
    if (tmax > 0.0) std::frexp(tmax, &e);  // tmax < 2^e
    const int sh = tmax > 0.0 ? std::min(100, std::max(-100, 14 - e)) : 0;
    const double st = std::ldexp(1.0, sh);
    p->tap_inv = static_cast<float>(std::ldexp(1.0, -sh));
    const int nc = p->nc, band = gct::kGemmBand;
    for (int n = 0; n < nc; ++n) {
        double comp = 0.0, back;
        for (int k = 0; k < nc; ++k) {
            const int m = n - k + nc / 2;
            if (m < 0 || m >= nc || std::abs(n - k) <= band) continue;
            const double t = taps[m] * st;
            bh[static_cast<size_t>(n) * p->Kp + k] = f16_bits(t, back);
            comp += t - back;
        }
        for (int k = std::max(0, n - band); k <= std::min(nc - 1, n + band); ++k) {
            const int m = n - k + nc / 2;
            if (m < 0 || m >= nc) continue;
            const double t = taps[m] * st + (k == n ? comp : 0.0);
            const size_t at = static_cast<size_t>(n) * p->Kp + k;
            double h, l, ll;
            bh[at] = f16_bits(t, h);
            bl[at] = f16_bits(t - h, l);
            bll[at] = f16_bits(t - h - l, ll);
        }
    }
}

void build_plan(gct_fdk_plan *p, const gct_ct_geom *g, const gct_vol_geom *vol,
                const gct_filt_params *filt, const gct_fdk_opts *opts)
{
    gct::check_ct_geom(g);
    const auto kind = static_cast<gct_geom_kind>(g->kind);
    gct::check_vol_geom(vol, gct::is_2d_detector(kind));
    p->kind = kind;
    p->family = gct::family_of(kind);
    p->views.assign(g->views, g->views + g->num_views);
    p->geom = *g;
    p->geom.views = p->views.data();
    if (!gct::is_2d_detector(kind)) p->geom.det_col = gct_detector{1u, 1.0};
    p->vol = *vol;
    p->filt = filt ? *filt : gct_filt_params{1.0, GCT_APOD_NONE};
    if (opts) p->opts = *opts;
    if (p->opts.filter != GCT_FILTER_FFT && p->opts.filter != GCT_FILTER_TOEPLITZ_BF16X3 &&
        p->opts.filter != GCT_FILTER_TOEPLITZ_BF16X4 && p->opts.filter != GCT_FILTER_TOEPLITZ_F16X2)
        gct::fail(GCT_ERR_INVALID_ARG, "unknown filter option");
    if (p->opts.storage != GCT_STORAGE_F32 && p->opts.storage != GCT_STORAGE_F16)
        gct::fail(GCT_ERR_INVALID_ARG, "unknown storage option");
    if (!gct::rotation_info(p->geom, &p->rot))
        gct::fail(GCT_ERR_INVALID_ARG, "Invalid X-ray source trajectory.");
    p->nv = static_cast<int>(g->num_views);
    p->nc = static_cast<int>(g->det_row.num_samples);
    p->nr = static_cast<int>(p->geom.det_col.num_samples);
    p->L = gct::fft_length(static_cast<unsigned>(p->nc));
    if (p->L > 8192) gct::fail(GCT_ERR_NOT_SUPPORTED, "detector rows longer than 5461 samples");

    // per-view derived geometry (FP64)
    std::vector<gct::ViewDerived> vd(p->nv);
    for (int v = 0; v < p->nv; ++v) {
        vd[v] = gct::derive_view(kind, p->geom, static_cast<unsigned>(v));
        if (p->family == gct::Family::Arc) {
            const bool ok = gct::is_2d_detector(kind) ? (orthonormal(vd[v].eu, vd[v].ew, 1e-6) &&
                                                         orthonormal(vd[v].eu, vd[v].ev, 1e-6) &&
                                                         orthonormal(vd[v].ew, vd[v].ev, 1e-6))
                                                      : orthonormal(vd[v].eu, vd[v].ew, 1e-6);
            if (!ok) gct::fail(GCT_ERR_NOT_SUPPORTED, "arc-detector views need an orthonormal detector basis");
        }
        if (p->family != gct::Family::Affine && !(vd[v].sid > 0.0 && vd[v].sdd > 0.0))
            gct::fail(GCT_ERR_INVALID_ARG, "source distances must be positive");
        if (kind == GCT_GEOM_CONE_PARALLEL && !(vd[v].sid > 0.0 && vd[v].sdd > 0.0))
            gct::fail(GCT_ERR_INVALID_ARG, "source distances must be positive");
    }
    // final scale of reconFDK (src/cuda/recon/fdk_axial.cuh:196-199): x rot_ang_incr if > 0
    const double dtheta = p->rot.incr > 0.0 ? p->rot.incr : 1.0;
    std::vector<double> wscale(p->nv);
    for (int v = 0; v < p->nv; ++v) wscale[v] = dtheta * vd[v].bp_const;
    std::vector<double> coefs64;
    std::vector<float> coefs = gct::bp_coefficients(p->geom, p->vol, vd, wscale, &p->z_affine, &coefs64);
    // 1D parallel kind: transpose, so that the detector coordinate u(x, y) = u0 + ui x + uj y becomes
    // the row coordinate v(i, k) = v0 + vi i + vk k of a one-column detector and image rows run
    // along the backprojector's z loop
    p->t1d = kind == GCT_GEOM_PARALLEL_1D;
    p->kx = static_cast<int>(vol->nx);
    p->ky = p->t1d ? 1 : static_cast<int>(vol->ny);
    p->kz = p->t1d ? static_cast<int>(vol->ny) : static_cast<int>(vol->nz);
    if (p->t1d) {
        for (int v = 0; v < static_cast<int>(g->num_views); ++v) {
            float *c = &coefs[static_cast<size_t>(v) * gct::kCoefPerView];
            const float u0 = c[0], ui = c[1], uj = c[2];
            c[0] = c[1] = c[2] = 0.0f;  // the single detector column
            c[3] = u0;
            c[6] = ui;
            c[4] = uj;
            c[7] = 0.0f;
        }
    }

    std::vector<float4> fview(p->nv);
    for (int v = 0; v < p->nv; ++v)
        fview[v] = make_float4(static_cast<float>(vd[v].c0), static_cast<float>(vd[v].r0),
                               static_cast<float>(vd[v].sdd), 0.f);
    if (p->opts.scan != GCT_SCAN_AXIAL && p->opts.scan != GCT_SCAN_SPIRAL)
        gct::fail(GCT_ERR_INVALID_ARG, "unknown scan option");
    p->spiral = p->opts.scan == GCT_SCAN_SPIRAL;
    gct::SpiralInfo spiral_si;
    if (p->spiral) spiral_si = gct::spiral_info(p->geom);  // validates like SpiralCTGeom
    // spiral scans: no Parker weights (fdk_spiral.cuh applies cosine weights and the filter only)
    std::vector<float> parker;
    if (p->spiral) {
        parker.assign(static_cast<size_t>(p->nv) * p->nc, 1.0f);
    } else {
        const std::vector<double> parker_d = gct::parker_table(p->geom, p->rot);
        parker.assign(parker_d.begin(), parker_d.end());
    }
    const std::vector<double> taps = gct::ramp_taps(kind, g->det_row, p->filt);
    double l1 = 0.0;
    for (double t : taps) l1 += std::fabs(t);
    p->l1 = static_cast<float>(l1);
    const auto Hd = gct::filter_spectrum(taps, p->L);
    std::vector<float2> H(p->L);
    for (unsigned k = 0; k < p->L; ++k)
        H[k] = make_float2(static_cast<float>(Hd[k].real()), static_cast<float>(Hd[k].imag()));

    cuda_check(cudaGetDevice(&p->device), "cudaGetDevice");
    cudaDeviceProp prop{};
    cuda_check(cudaGetDeviceProperties(&prop, p->device), "cudaGetDeviceProperties");
    p->num_sms = prop.multiProcessorCount;
    p->fview.upload(fview.data(), fview.size(), "plan geometry");
    p->parker.upload(parker.data(), parker.size(), "plan Parker table");
    p->H.upload(H.data(), H.size(), "plan filter spectrum");
    // status word of the plan's kernels (gct_fdk_plan_check): GEMM pipeline and FFT input waits
    p->gemm_err.alloc(1, "kernel status");
    cuda_check(cudaMemset(p->gemm_err.p, 0, sizeof(int)), "kernel status reset");
    p->coefs.upload(coefs.data(), coefs.size(), "plan backprojection coefficients");
    if (p->opts.filter != GCT_FILTER_FFT) {
        // B = T^T with T[k][c] = g(c - k): row n holds g(n - k); taps g(m) = taps[m + nc/2]
        p->Kp = gct::gemm_pad_k(p->nc);
        p->Np = gct::gemm_pad_n(p->nc);
        const bool four = p->opts.filter == GCT_FILTER_TOEPLITZ_BF16X4;
        const bool f16 = p->opts.filter == GCT_FILTER_TOEPLITZ_F16X2;
        std::vector<__nv_bfloat16> bh(static_cast<size_t>(p->Np) * p->Kp, __float2bfloat16(0.f)), bl(bh), bll;
        if (four || f16) bll = bh;
        if (f16) {
            toeplitz_f16(p, taps, bh, bl, bll);
        } else {
            for (int n = 0; n < p->nc; ++n)
                for (int k = 0; k < p->nc; ++k) {
                    const int m = n - k + p->nc / 2;
                    if (m < 0 || m >= p->nc) continue;
                    const double t = taps[m];
                    const __nv_bfloat16 hi = __float2bfloat16(static_cast<float>(t));
                    const double r1 = t - static_cast<double>(__bfloat162float(hi));
                    const __nv_bfloat16 lo = __float2bfloat16(static_cast<float>(r1));
                    const size_t at = static_cast<size_t>(n) * p->Kp + k;
                    bh[at] = hi;
                    bl[at] = lo;
                    if (four && std::abs(n - k) <= gct::kGemmBand)
                        bll[at] = __float2bfloat16(static_cast<float>(r1 - static_cast<double>(__bfloat162float(lo))));
                }
        }
        p->th.upload(bh.data(), bh.size(), "Toeplitz matrix (hi)");
        p->tl.upload(bl.data(), bl.size(), "Toeplitz matrix (lo)");
        if (four || f16) p->tll.upload(bll.data(), bll.size(), "Toeplitz matrix (third piece, central band)");
        const size_t rows = static_cast<size_t>(p->nv) * p->nr;
        p->xh.alloc(rows * p->Kp, "GEMM rows (hi)");
        p->xl.alloc(rows * p->Kp, "GEMM rows (lo)");
        if (four) p->xll.alloc(rows * p->Kp, "GEMM rows (third piece)");
        if (f16) p->grinv.alloc(rows, "GEMM row scales");
        p->ybuf.alloc(rows * p->nc, "GEMM filtered rows");
    }
    // backprojection launch shape
    const bool vol3d = gct::is_2d_detector(kind);
    // measured on B200 (512^3, 720 views, with the per-block view classes): 16 voxels per thread
    // with 8 x 16 blocks for FP16 quads (2047 GUPS; 8 voxels: 1855, 32: 1543) and with 4 x 16 blocks
    // for FP32 quads (1466 GUPS; 8 voxels on 4 x 32: 1425)
    const bool f16 = p->opts.storage == GCT_STORAGE_F16;
    // the transposed 1D parallel kind loops over image rows: 16 rows per thread, 128 x 1 blocks
    const int zpt3d = 16;
    p->zpt = p->opts.z_per_thread > 0 ? p->opts.z_per_thread : ((vol3d || p->t1d) ? zpt3d : 1);
    if (p->zpt != 1 && p->zpt != 2 && p->zpt != 4 && p->zpt != 8 && p->zpt != 16)
        gct::fail(GCT_ERR_INVALID_ARG, "z_per_thread must be 1, 2, 4, 8 or 16");
    p->bx = p->opts.block_x > 0 ? p->opts.block_x : (p->t1d ? 128 : vol3d ? (f16 ? 8 : 4) : 32);
    p->by = p->opts.block_y > 0 ? p->opts.block_y : (p->t1d ? 1 : vol3d ? 16 : 8);
    if (p->bx * p->by > 256 || p->bx * p->by < 32)
        gct::fail(GCT_ERR_INVALID_ARG, "backprojection block must hold 32..256 threads");
    // quarter-turn form: the z-affine column kernels (not the transposed 1D kind, whose kernel
    // grid is x by image rows); at most 8 voxels per thread, since each thread keeps four columns.
    // Measured on B200 (512^3, 720 views): FP16 quads 34.4 ms against 47.2 ms for the plain kernel
    // (8 voxels per thread, 2 x 32 blocks; 4 x 16: 35.5, 8 x 16: 36.6, 4 voxels: 36.9); FP32 quads
    // 88 ms against 64 ms (a 64-byte partner group per voxel), so AUTO takes it for FP16 storage
    // only and ON for both.
    const int so = p->opts.symmetry;
    if (so != GCT_SYMMETRY_AUTO && so != GCT_SYMMETRY_OFF && so != GCT_SYMMETRY_ON)
        gct::fail(GCT_ERR_INVALID_ARG, "unknown symmetry option");
    const bool want = so == GCT_SYMMETRY_ON || (so == GCT_SYMMETRY_AUTO && f16);
    if (want && !p->t1d && (p->family == gct::Family::Affine || p->z_affine))
        p->sym = gct::quarter_turn_symmetry(kind, coefs64, static_cast<unsigned>(p->nv), vol->nx, vol->ny,
                                            static_cast<unsigned>(p->kz));
    // z-mirror form of the column kernels (plans without the quarter-turn form, whose kernel has
    // its own sharing): each thread takes a segment of the lower half and its mirror voxels
    if (want && !p->sym && !p->t1d && !p->spiral && p->zpt % 2 == 0 &&
        (p->family == gct::Family::Affine || (p->family == gct::Family::Projective && p->z_affine)))
        p->mirror = gct::z_mirror_symmetry(kind, coefs64, static_cast<unsigned>(p->nv), static_cast<unsigned>(p->nr),
                                           vol->nx, vol->ny, static_cast<unsigned>(p->kz));
    // measured on B200 (512 x 512 x 384, 496 views of 1240 x 960, FP16 quads): 8 + 8 mirrored
    // voxels per thread 34.6 ms, 16 + 16 42.7 ms, 4 + 4 40.5 ms, the plain kernel 37.0 ms (16 voxels)
    // and 35.5 ms (8); FP32 quads 62.6 ms against 51.8 ms plain, so AUTO takes it for FP16 only
    if (p->mirror && p->opts.z_per_thread <= 0) p->zpt = 8;
    // quarter-turn stacks are prepared through FP32 rows (prepare_partners); the GEMM filter has
    // its row buffer already
    if (p->sym && !p->ybuf.p)
        p->ybuf.alloc(static_cast<size_t>(p->nv) * p->nr * p->nc, "filtered rows of quarter-turn stacks");
    if (p->spiral) {
        // one slice per thread along z: each slice has its own window of views
        p->sym = 0;
        p->zpt = 1;
        if (p->opts.block_x <= 0) p->bx = 32;
        if (p->opts.block_y <= 0) p->by = 8;
        std::vector<int2> win(p->kz);
        const double z0 = vol->mid[2] - (vol->nz - 1.0) * vol->dz / 2.0;
        for (int k = 0; k < p->kz; ++k) {
            long long first = 0, last = 0;
            gct::spiral_window(spiral_si, z0 + k * vol->dz, &first, &last);
            win[k] = (first > 0 && last < p->nv) ? make_int2(static_cast<int>(first), static_cast<int>(last - first))
                                                 : make_int2(0, 0);
        }
        p->slice_views.upload(win.data(), win.size(), "spiral slice windows");
    }
    p->zpt_sym = p->opts.z_per_thread > 0 ? std::min(p->zpt, 8) : (vol3d ? (f16 ? 8 : 4) : 1);
    p->bx_sym = p->opts.block_x > 0 ? p->bx : (vol3d ? (f16 ? 2 : 4) : 8);
    p->by_sym = p->opts.block_y > 0 ? p->by : (vol3d ? (f16 ? 32 : 16) : 8);
}

// Weighting and split of the rows of views [vb, vb + vc) into the plan's A pieces (row order:
// view-major, or partner-interleaved for `quarter` > 0). `fused_scales` (FP16 storage): the split
// also finds the view maxima, and the view scales follow it.
void split_rows(gct_fdk_plan *p, const float *proj, int vb, int vc, int quarter, cudaStream_t s,
                const StackRef *fused_scales)
{
    gct::SplitArgs sa;
    sa.proj = proj;
    sa.row0 = static_cast<long long>(vb) * p->nr;
    sa.rows = static_cast<long long>(vc) * p->nr;
    sa.nr = p->nr;
    sa.nc = p->nc;
    sa.Kp = p->Kp;
    sa.kind = p->kind;
    sa.du = static_cast<float>(p->geom.det_row.sampling_width);
    sa.dv = static_cast<float>(p->geom.det_col.sampling_width);
    sa.fview = p->fview.p;
    sa.parker = p->parker.p;
    sa.xh = p->xh.p;
    sa.xl = p->xl.p;
    sa.xll = p->xll.p;
    sa.amax = fused_scales ? fused_scales->amax : nullptr;
    sa.rinv = p->grinv.p;
    sa.tap_inv = p->tap_inv;
    sa.quarter = quarter;
    gct::launch_split(sa, p->num_sms, s);
    cuda_check(cudaGetLastError(), "split kernel launch");
    if (fused_scales) {  // the split found the view maxima: scales before the quads are written
        gct::launch_view_scales(fused_scales->amax + vb, vc, p->l1, fused_scales->vscale + vb, fused_scales->vinv + vb,
                                s);
        cuda_check(cudaGetLastError(), "view scale kernel");
    }
}

// The GEMM launch fields every form shares.
gct::GemmLaunch gemm_launch(const gct_fdk_plan *p)
{
    gct::GemmLaunch gl;
    gl.xh = p->xh.p;
    gl.xl = p->xl.p;
    gl.xll = p->xll.p;
    gl.tll = p->tll.p;
    gl.form = p->opts.filter == GCT_FILTER_TOEPLITZ_BF16X4 ? gct::kGemmBf16x4
              : p->opts.filter == GCT_FILTER_TOEPLITZ_F16X2  ? gct::kGemmF16x2
                                                             : gct::kGemmBf16x3;
    gl.rinv = p->grinv.p;
    gl.a_rows = static_cast<long long>(p->nv) * p->nr;
    gl.th = p->th.p;
    gl.tl = p->tl.p;
    gl.Np = p->Np;
    gl.Kp = p->Kp;
    gl.N = p->nc;
    gl.err = p->gemm_err.p;
    return gl;
}

// Toeplitz-GEMM form of run_filter: split, tcgen05 GEMM into FP32 rows, then quads (or the rows
// themselves for the plain output).
void run_filter_gemm(gct_fdk_plan *p, const float *proj, void *out, const float *vscale, int mode, int quarter,
                     int vb, int vc, cudaStream_t s, const StackRef *fused_scales)
{
    const long long row0 = static_cast<long long>(vb) * p->nr, rows = static_cast<long long>(vc) * p->nr;
    split_rows(p, proj, vb, vc, 0, s, fused_scales);
    gct::GemmLaunch gl = gemm_launch(p);
    if (mode == gct::kOutQuadF16 && quarter == 0 && !p->t1d && p->nc % 2 == 0 &&
        reinterpret_cast<uintptr_t>(out) % 16 == 0 && gct::gemm_quad_tiles(rows, 1) >= p->num_sms) {
        // view-major FP16 quads straight from the GEMM's epilogue
        gl.quads = out;
        gl.vscale = vscale;
        gl.nr = p->nr;
        gl.v_begin = vb;
        gl.v_count = vc;
        cuda_check(gct::launch_toeplitz_gemm(gl, p->num_sms, s), "Toeplitz GEMM launch (quads)");
        return;
    }
    gl.m_begin = static_cast<int>(row0);
    gl.M = static_cast<int>(rows);
    gl.Y = (mode == gct::kOutPlainF32 ? static_cast<float *>(out) : p->ybuf.p) + row0 * p->nc;
    gl.ldy = p->nc;
    cuda_check(gct::launch_toeplitz_gemm(gl, p->num_sms, s), "Toeplitz GEMM launch");
    if (mode == gct::kOutPlainF32) return;
    gct::QuadArgs qa;
    qa.Y = gl.Y;
    qa.ldy = p->nc;
    qa.v0 = vb;
    qa.nv = vc;
    qa.nr = p->nr;
    qa.nc = p->nc;
    qa.t1d = p->t1d ? 1 : 0;
    qa.vscale = (mode == gct::kOutQuadF16) ? vscale : nullptr;
    qa.out = out;
    qa.quarter = quarter;
    qa.err = p->gemm_err.p;
    gct::launch_quads_from_rows(qa, mode, p->num_sms, s);
    cuda_check(cudaGetLastError(), "quad kernel launch");
}

}  // namespace

// `out` is the view-0 address of the output; `vscale` (FP16 quads only) the view-0 scales;
// `quarter` the quad_layout of a quad output. `fused_scales` (Toeplitz form only, amax zeroed by
// the caller): the split pass also finds the view maxima and the scales follow it.
void run_filter(gct_fdk_plan *p, const float *proj, void *out, const float *vscale, int mode, int quarter, int vb,
                int vc, cudaStream_t s, const StackRef *fused_scales)
{
    if (vc <= 0) return;
    if (p->opts.filter != GCT_FILTER_FFT) {
        run_filter_gemm(p, proj, out, vscale, mode, quarter, vb, vc, s, fused_scales);
        return;
    }
    const long long pix = static_cast<long long>(p->nr) * p->nc;
    gct::FilterArgs fa;
    fa.proj = proj + vb * pix;
    fa.nv = vc;
    fa.nr = p->nr;
    fa.nc = p->nc;
    fa.kind = p->kind;
    fa.du = static_cast<float>(p->geom.det_row.sampling_width);
    fa.dv = static_cast<float>(p->geom.det_col.sampling_width);
    fa.fview = p->fview.p + vb;
    fa.parker = p->parker.p + static_cast<long long>(vb) * p->nc;
    fa.H = p->H.p;
    fa.err = p->gemm_err.p;
    fa.mode = mode;
    if (mode == gct::kOutPlainF32) {
        fa.out = static_cast<float *>(out) + vb * pix;
    } else {
        fa.out = out;
        fa.v0 = vb;
        fa.quarter = quarter;
    }
    fa.vscale = (mode == gct::kOutQuadF16) ? vscale + vb : nullptr;
    fa.t1d = (p->t1d && mode != gct::kOutPlainF32) ? 1 : 0;
    gct::launch_filter_fft(fa, static_cast<int>(p->L), p->num_sms, s);
    cuda_check(cudaGetLastError(), "filter kernel launch");
}

gct::BpArgs bp_args(const gct_fdk_plan *p, const StackRef &st, float *vol, int v_begin, int v_count)
{
    gct::BpArgs ba;
    ba.quads = st.quads;
    // the quad grid per view holds (nr + 4) x (nc + 4) entries in either orientation
    ba.qpitch = p->t1d ? gct::kT1dPitch : p->nc + 2 * gct::kQuadPad;
    ba.qview = static_cast<long long>(p->nr + 2 * gct::kQuadPad) * (p->nc + 2 * gct::kQuadPad);
    ba.coefs = p->coefs.p;
    ba.vinv = st.vinv;
    ba.v_begin = v_begin;
    ba.v_count = v_count;
    ba.quarter = st.quarter;
    ba.slice_views = p->slice_views.p;
    ba.vol = vol;
    ba.nx = p->kx;
    ba.ny = p->ky;
    ba.nz = p->kz;
    ba.umax = static_cast<float>(p->t1d ? 1 : p->nc);
    ba.vmax = static_cast<float>(p->t1d ? p->nc : p->nr);
    return ba;
}

namespace {
// View chunk of a split backprojection of `views` views (0: no split): a one-voxel-deep image
// whose launch of `blocks` blocks (`per_sm` resident per SM) fills less than one wave is split
// into the most parts (chunks of at least 8 views) whose blocks fit two whole waves.
int split_chunk(const gct_fdk_plan *p, long long blocks, int per_sm, int views)
{
    if (p->kz != 1 || p->spiral || p->t1d || blocks <= 0 || per_sm <= 0 || views < 16) return 0;
    const long long wave = static_cast<long long>(p->num_sms) * per_sm;
    if (blocks >= wave) return 0;
    const long long parts = std::min<long long>(2 * wave / blocks, views / 8);
    if (parts < 2) return 0;
    return static_cast<int>((views + parts - 1) / parts);
}

// Launches ba (vol, accumulate) through partial images when `chunk` > 0.
template <class Launch>
void launch_split(gct_fdk_plan *p, gct::BpArgs ba, int chunk, cudaStream_t s, Launch go)
{
    if (chunk <= 0) {
        go(ba);
        return;
    }
    const int parts = (ba.v_count + chunk - 1) / chunk;
    const long long n = static_cast<long long>(p->kx) * p->ky * p->kz;
    if (p->bp_part.n < static_cast<size_t>(parts) * n)
        p->bp_part.alloc(static_cast<size_t>(parts) * n, "partial images of a view-split backprojection");
    float *vol = ba.vol;
    const bool accumulate = ba.accumulate != 0;
    ba.vol = p->bp_part.p;
    ba.vchunk = chunk;
    ba.vol_stride = n;
    ba.accumulate = 0;
    go(ba);
    gct::launch_reduce_partials(p->bp_part.p, parts, n, vol, accumulate, s);
    cuda_check(cudaGetLastError(), "partial image reduction");
}
}  // namespace

void run_backproject(gct_fdk_plan *p, const StackRef &st, float *vol, int v_begin, int v_count,
                     bool accumulate, cudaStream_t s, bool split)
{
    if (st.quarter && v_begin == 0 && v_count == p->nv) {
        run_backproject_sym(p, st, vol, 0, p->nv / 4, accumulate, s, split);
        return;
    }
    gct::BpArgs ba = bp_args(p, st, vol, v_begin, v_count);
    ba.accumulate = accumulate ? 1 : 0;
    ba.mirror = (p->mirror && st.quarter == 0) ? 1 : 0;  // view-major stacks only
    const long long blocks = static_cast<long long>((p->kx + p->bx - 1) / p->bx) * ((p->ky + p->by - 1) / p->by);
    const int chunk =
        split ? split_chunk(p, blocks,
                            gct::backproject_blocks_per_sm(ba, static_cast<int>(p->family), p->opts.storage,
                                                           p->z_affine, false, p->zpt, p->bx * p->by),
                            v_count)
              : 0;
    launch_split(p, ba, chunk, s, [&](const gct::BpArgs &b) {
        gct::launch_backproject(b, static_cast<int>(p->family), p->opts.storage, p->z_affine, p->zpt, p->bx, p->by,
                                s);
        cuda_check(cudaGetLastError(), "backprojection kernel launch");
    });
}

void run_backproject_sym(gct_fdk_plan *p, const StackRef &st, float *vol, int b_begin, int b_count,
                         bool accumulate, cudaStream_t s, bool split)
{
    gct::BpArgs ba = bp_args(p, st, vol, b_begin, b_count);
    ba.accumulate = accumulate ? 1 : 0;
    ba.sym = p->sym;
    const int h = p->kx / 2;
    const long long blocks =
        static_cast<long long>((h + p->bx_sym - 1) / p->bx_sym) * ((h + p->by_sym - 1) / p->by_sym);
    const int chunk =
        split ? split_chunk(p, blocks,
                            gct::backproject_blocks_per_sm(ba, static_cast<int>(p->family), p->opts.storage, true,
                                                           true, p->zpt_sym, p->bx_sym * p->by_sym),
                            b_count)
              : 0;
    launch_split(p, ba, chunk, s, [&](const gct::BpArgs &b) {
        gct::launch_backproject_sym(b, static_cast<int>(p->family), p->opts.storage, p->zpt_sym, p->bx_sym,
                                    p->by_sym, s);
        cuda_check(cudaGetLastError(), "backprojection kernel launch");
    });
}

void check_range(const gct_fdk_plan *p, uint32_t vb, uint32_t vc)
{
    if (static_cast<uint64_t>(vb) + vc > static_cast<uint64_t>(p->nv))
        gct::fail(GCT_ERR_INVALID_ARG, "view range exceeds the number of views");
}

void *plan_workspace(gct_fdk_plan *p, void *workspace)
{
    if (workspace) return workspace;
    if (!p->work.p) p->work.alloc(p->workspace_bytes(), "plan workspace");
    return p->work.p;
}

namespace {
// FP16 storage: per-view maxima of views [vb, vb + vc) and their power-of-two scales.
void view_scales(gct_fdk_plan *p, const float *proj, const StackRef &st, int vb, int vc, cudaStream_t s)
{
    const long long pix = static_cast<long long>(p->nr) * p->nc;
    cuda_check(cudaMemsetAsync(st.amax + vb, 0, sizeof(float) * vc, s), "view maxima reset");
    gct::launch_view_absmax(proj + vb * pix, vc, pix, st.amax + vb, s);
    gct::launch_view_scales(st.amax + vb, vc, p->l1, st.vscale + vb, st.vinv + vb, s);
    cuda_check(cudaGetLastError(), "view scale kernels");
}
}  // namespace

void prepare(gct_fdk_plan *p, const float *proj, const StackRef &st, int vb, int vc, cudaStream_t s)
{
    if (!proj) gct::fail(GCT_ERR_INVALID_ARG, "NULL projection pointer");
    if (vc <= 0) return;
    const bool f16 = p->opts.storage == GCT_STORAGE_F16;
    const bool fuse = f16 && p->opts.filter != GCT_FILTER_FFT;  // the split pass finds the maxima
    if (fuse) cuda_check(cudaMemsetAsync(st.amax + vb, 0, sizeof(float) * vc, s), "view maxima reset");
    else if (f16) view_scales(p, proj, st, vb, vc, s);
    run_filter(p, proj, st.quads, st.vscale, f16 ? gct::kOutQuadF16 : gct::kOutQuadF32, st.quarter, vb, vc, s,
               fuse ? &st : nullptr);
}

void prepare_partners(gct_fdk_plan *p, const float *proj, const StackRef &st, int b, int n, cudaStream_t s)
{
    if (!proj) gct::fail(GCT_ERR_INVALID_ARG, "NULL projection pointer");
    const int m = st.quarter;
    if (n <= 0 || m <= 0) return;
    const bool f16 = p->opts.storage == GCT_STORAGE_F16;
    const bool whole = b == 0 && n == m;
    const bool fuse = f16 && p->opts.filter != GCT_FILTER_FFT;  // the split pass finds the maxima
    if (fuse && gct::gemm_quad_tiles(static_cast<long long>(n) * p->nr, 4) >= p->num_sms) {
        // FP16 quads from the Toeplitz GEMM: rows split in partner-interleaved order (with the view
        // maxima and scales), then one GEMM whose epilogue writes the partner groups
        for (int q = 0; q < (whole ? 1 : 4); ++q) {
            const int vb = whole ? 0 : b + q * m, vc = whole ? p->nv : n;
            cuda_check(cudaMemsetAsync(st.amax + vb, 0, sizeof(float) * vc, s), "view maxima reset");
            split_rows(p, proj, vb, vc, m, s, &st);
        }
        gct::GemmLaunch gl = gemm_launch(p);
        gl.quads = st.quads;
        gl.vscale = st.vscale;
        gl.quarter = m;
        gl.nr = p->nr;
        gl.v_begin = b;
        gl.v_count = n;
        cuda_check(gct::launch_toeplitz_gemm(gl, p->num_sms, s), "Toeplitz GEMM launch (partner quads)");
        return;
    }
    for (int q = 0; q < (whole ? 1 : 4); ++q) {
        const int vb = whole ? 0 : b + q * m, vc = whole ? p->nv : n;
        if (fuse) cuda_check(cudaMemsetAsync(st.amax + vb, 0, sizeof(float) * vc, s), "view maxima reset");
        else if (f16) view_scales(p, proj, st, vb, vc, s);
        run_filter(p, proj, p->ybuf.p, nullptr, gct::kOutPlainF32, 0, vb, vc, s, fuse ? &st : nullptr);
    }
    gct::QuadArgs qa;
    qa.Y = p->ybuf.p;
    qa.ldy = p->nc;
    qa.v0 = b;
    qa.nv = n;
    qa.nr = p->nr;
    qa.nc = p->nc;
    qa.vscale = f16 ? st.vscale : nullptr;
    qa.out = st.quads;
    qa.quarter = m;
    qa.err = p->gemm_err.p;
    gct::launch_quads_partners(qa, f16 ? gct::kOutQuadF16 : gct::kOutQuadF32, p->num_sms, s);
    cuda_check(cudaGetLastError(), "partner quad kernel launch");
}

void execute(gct_fdk_plan *p, const float *proj, float *vol, void *workspace, cudaStream_t s)
{
    if (!proj || !vol) gct::fail(GCT_ERR_INVALID_ARG, "NULL projection or volume pointer");
    const StackRef st = stack_of(p, plan_workspace(p, workspace));
    if (st.quarter) prepare_partners(p, proj, st, 0, st.quarter, s);
    else prepare(p, proj, st, 0, p->nv, s);
    run_backproject(p, st, vol, 0, p->nv, false, s);
}

// Host buffers through a plan. The upload of chunk c on the copy stream waits only for the
// previous call's filter of chunk c (its staging slot), and the volume download runs on a third
// stream into one of two device volumes, so consecutive calls overlap: one call's uploads run under
// the previous call's backprojections and one call's download under the next call's work. With
// `sync` the call returns when the volume is on the host; otherwise gct_fdk_host_sync waits.
void execute_host(gct_fdk_plan *p, const float *proj_host, float *vol_host, cudaStream_t s, bool sync)
{
    if (!proj_host || !vol_host) gct::fail(GCT_ERR_INVALID_ARG, "NULL projection or volume pointer");
    const size_t pix = static_cast<size_t>(p->nr) * p->nc;
    const size_t vol_n = static_cast<size_t>(p->vol.nx) * p->vol.ny * p->vol.nz;
    if (!p->host_proj.p) p->host_proj.alloc(pix * p->nv, "staging projections");
    const int slot = static_cast<int>(p->host_calls & 1u);
    DevBuf<float> &vbuf = slot ? p->host_vol2 : p->host_vol;
    if (!vbuf.p) vbuf.alloc(vol_n, "staging volume");
    const StackRef st = stack_of(p, plan_workspace(p, nullptr));
    if (!p->copy_stream) cuda_check(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking), "copy stream");
    if (!p->d2h_stream) cuda_check(cudaStreamCreateWithFlags(&p->d2h_stream, cudaStreamNonBlocking), "download stream");
    // About 8 chunks, at least 16 views each; a quarter-turn plan chunks its base views and takes
    // each chunk's partner views with it. (Measured and rejected at 512^3 / 720 views: splitting the
    // last quarter into chunks a quarter that size, to shorten the work after the last upload:
    // 74.8 against 61.2 ms per reconstruction, the small chunks' filter launches cost more.)
    const int parts = st.quarter ? 4 : 1, span = p->nv / parts;
    const int chunk = std::max(16 / parts, (span + 7) / 8);
    const int nchunks = (span + chunk - 1) / chunk;
    auto grow = [](std::vector<cudaEvent_t> &v, size_t n) {
        while (v.size() < n) {
            cudaEvent_t e;
            cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
            v.push_back(e);
        }
    };
    grow(p->chunk_events, nchunks);
    grow(p->prep_events, nchunks);
    for (cudaEvent_t *e : {&p->vol_free[0], &p->vol_free[1], &p->bp_done})
        if (!*e) cuda_check(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "event");
    for (int c = 0; c < nchunks; ++c) {
        const int vb = c * chunk, vc = std::min(chunk, span - vb);
        // the staging of chunk c is free once the previous call has filtered it (an event never
        // recorded lets the first call through)
        cuda_check(cudaStreamWaitEvent(p->copy_stream, p->prep_events[c], 0), "stream wait");
        for (int q = 0; q < parts; ++q) {
            const size_t v0 = static_cast<size_t>(vb + q * span);
            cuda_check(cudaMemcpyAsync(p->host_proj.p + v0 * pix, proj_host + v0 * pix, sizeof(float) * pix * vc,
                                       cudaMemcpyHostToDevice, p->copy_stream),
                       "projection upload");
        }
        cuda_check(cudaEventRecord(p->chunk_events[c], p->copy_stream), "event record");
        cuda_check(cudaStreamWaitEvent(s, p->chunk_events[c], 0), "stream wait");
        // this volume is free once the download two calls back has read it
        if (c == 0) cuda_check(cudaStreamWaitEvent(s, p->vol_free[slot], 0), "stream wait");
        if (st.quarter) prepare_partners(p, p->host_proj.p, st, vb, vc, s);
        else prepare(p, p->host_proj.p, st, vb, vc, s);
        cuda_check(cudaEventRecord(p->prep_events[c], s), "event record");
        if (st.quarter) run_backproject_sym(p, st, vbuf.p, vb, vc, c > 0, s);
        else run_backproject(p, st, vbuf.p, vb, vc, c > 0, s);
    }
    cuda_check(cudaEventRecord(p->bp_done, s), "event record");
    cuda_check(cudaStreamWaitEvent(p->d2h_stream, p->bp_done, 0), "stream wait");
    cuda_check(cudaMemcpyAsync(vol_host, vbuf.p, sizeof(float) * vol_n, cudaMemcpyDeviceToHost, p->d2h_stream),
               "volume download");
    cuda_check(cudaEventRecord(p->vol_free[slot], p->d2h_stream), "event record");
    ++p->host_calls;
    if (sync) cuda_check(cudaStreamSynchronize(p->d2h_stream), "reconstruction");
}

// Streaming FDK with a bounded device footprint for the projections: views go through two
// staging slots of `chunk` views (upload of the next chunk on the copy stream while the current
// one is filtered) into a view-major stack of one chunk, and each chunk is backprojected into the
// device volume (chunk 0 stores, later chunks add). Replaces reconFDKLowMem
// (src/cuda/recon/fdk_axial.cuh:91-149), which moves one view at a time with a synchronous copy.
void execute_host_budget(gct_fdk_plan *p, const float *proj_host, float *vol_host, uint64_t budget, cudaStream_t s)
{
    if (!proj_host || !vol_host) gct::fail(GCT_ERR_INVALID_ARG, "NULL projection or volume pointer");
    const size_t pix = static_cast<size_t>(p->nr) * p->nc;
    const size_t vol_n = static_cast<size_t>(p->vol.nx) * p->vol.ny * p->vol.nz;
    const bool f16 = p->opts.storage == GCT_STORAGE_F16;
    const size_t per_view = 2 * pix * sizeof(float) + p->view_bytes() + (f16 ? 3 * sizeof(float) : 0);
    const size_t chunk = std::min<size_t>(static_cast<size_t>(p->nv), (budget > 512 ? budget - 512 : 0) / per_view);
    if (chunk < 1)
        gct::fail(GCT_ERR_BUDGET, "one view needs " + std::to_string(per_view) + " bytes of streaming buffers; the budget is " +
                                      std::to_string(budget));
    if (p->stream_chunk != static_cast<int>(chunk)) {
        p->stream_stage.alloc(2 * chunk * pix, "streaming projection slots");
        p->stream_ws.alloc(((chunk * p->view_bytes() + 255) & ~static_cast<size_t>(255)) +
                               (f16 ? 3 * chunk * sizeof(float) : 0),
                           "streaming filtered-projection stack");
        p->stream_chunk = static_cast<int>(chunk);
    }
    if (!p->host_vol.p) p->host_vol.alloc(vol_n, "staging volume");
    if (!p->copy_stream) cuda_check(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking), "copy stream");
    // the device volume may still be downloading for an asynchronous host call
    if (p->vol_free[0]) cuda_check(cudaStreamWaitEvent(s, p->vol_free[0], 0), "stream wait");
    for (cudaEvent_t &e : p->stream_events)
        if (!e) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    cudaEvent_t *filled = p->stream_events, *freed = p->stream_events + 2;
    // the slots are free once everything earlier on `s` (a previous call) is done
    cuda_check(cudaEventRecord(freed[0], s), "event record");
    cuda_check(cudaEventRecord(freed[1], s), "event record");
    unsigned char *ws = p->stream_ws.p;
    float *scales = reinterpret_cast<float *>(ws + ((chunk * p->view_bytes() + 255) & ~static_cast<size_t>(255)));
    const int nchunks = static_cast<int>((p->nv + chunk - 1) / chunk);
    for (int c = 0; c < nchunks; ++c) {
        const int vb = c * static_cast<int>(chunk), vc = std::min(static_cast<int>(chunk), p->nv - vb);
        const int slot = c & 1;
        float *stage = p->stream_stage.p + slot * chunk * pix;
        cuda_check(cudaStreamWaitEvent(p->copy_stream, freed[slot], 0), "stream wait");
        cuda_check(cudaMemcpyAsync(stage, proj_host + static_cast<size_t>(vb) * pix, sizeof(float) * pix * vc,
                                   cudaMemcpyHostToDevice, p->copy_stream),
                   "projection upload");
        cuda_check(cudaEventRecord(filled[slot], p->copy_stream), "event record");
        cuda_check(cudaStreamWaitEvent(s, filled[slot], 0), "stream wait");
        // prepare() and run_backproject() address view v at view-0 bases: shifting them by vb views
        // puts this chunk at the start of the slot and of the chunk stack
        StackRef st;
        st.quads = reinterpret_cast<unsigned char *>(reinterpret_cast<uintptr_t>(ws) -
                                                     static_cast<uintptr_t>(vb) * p->view_bytes());
        if (f16) {
            st.amax = scales - vb;
            st.vscale = scales + chunk - vb;
            st.vinv = scales + 2 * chunk - vb;
        }
        const float *proj0 = reinterpret_cast<const float *>(reinterpret_cast<uintptr_t>(stage) -
                                                             static_cast<uintptr_t>(vb) * pix * sizeof(float));
        prepare(p, proj0, st, vb, vc, s);
        cuda_check(cudaEventRecord(freed[slot], s), "event record");
        run_backproject(p, st, p->host_vol.p, vb, vc, c > 0, s, false);  // within the byte budget
    }
    cuda_check(cudaMemcpyAsync(vol_host, p->host_vol.p, sizeof(float) * vol_n, cudaMemcpyDeviceToHost, s),
               "volume download");
    cuda_check(cudaStreamSynchronize(s), "reconstruction");
}

namespace {

struct PlanHolder {
    gct_fdk_plan *p = nullptr;
    ~PlanHolder() { delete p; }
};

}  // namespace

namespace {
// Device address of the allocation-free path's scratch array on `dev` (defined below).
unsigned char *noalloc_scratch(int dev);
}  // namespace

extern "C" {

int32_t gct_abi_version(void) { return GCT_FDK_ABI_VERSION; }

const char *gct_last_error_string(void) { return g_last_error.c_str(); }

gct_status gct_proj_geom_create(int32_t kind, const gct_geom_params *params, uint32_t proj_idx,
                                gct_view_geom *out)
{
    return guarded([&] {
        if (!params || !out) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        if (kind < GCT_GEOM_PARALLEL_1D || kind > GCT_GEOM_CONE_FLAT) gct::fail(GCT_ERR_INVALID_ARG, "unknown geometry kind");
        *out = gct::make_view(static_cast<gct_geom_kind>(kind), *params, proj_idx);
    });
}

namespace {
void export_matrix(const gct::ProjMatrix &pm, gct_proj_matrix *out)
{
    std::copy(pm.m, pm.m + 12, out->matrix);
    std::copy(pm.K, pm.K + 9, out->intrinsic);
    std::copy(pm.R, pm.R + 9, out->rotation);
    std::copy(pm.src, pm.src + 3, out->src_pos);
}
}  // namespace

gct_status gct_proj_matrix_decompose(const double *matrix, gct_proj_matrix *out)
{
    return guarded([&] {
        if (!matrix || !out) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        export_matrix(gct::decompose_projection_matrix(matrix), out);
    });
}

gct_status gct_proj_matrix_compose(const gct_view_geom *view, double pix_width_mm, double pix_height_mm,
                                   gct_proj_matrix *out)
{
    return guarded([&] {
        if (!view || !out) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        export_matrix(gct::compose_projection_matrix(*view, pix_width_mm, pix_height_mm), out);
    });
}

gct_status gct_proj_geom_from_matrix(const double *matrix, gct_view_geom *out)
{
    return guarded([&] {
        if (!matrix || !out) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        *out = gct::view_from_projection_matrix(gct::decompose_projection_matrix(matrix));
    });
}

gct_status gct_spiral_geom_check(const gct_ct_geom *geom, uint32_t *num_proj_per_rot, double *pitch_mm_per_rad)
{
    return guarded([&] {
        gct::check_ct_geom(geom);
        const gct::SpiralInfo si = gct::spiral_info(*geom);
        if (num_proj_per_rot) *num_proj_per_rot = si.npr;
        if (pitch_mm_per_rad) *pitch_mm_per_rad = si.pitch;
    });
}

gct_status gct_spiral_proj_indices(const gct_ct_geom *geom, double slice_pos_mm, int64_t *first, int64_t *last)
{
    return guarded([&] {
        gct::check_ct_geom(geom);
        if (!first || !last) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        long long f = 0, l = 0;
        gct::spiral_window(gct::spiral_info(*geom), slice_pos_mm, &f, &l);
        *first = f;
        *last = l;
    });
}

gct_status gct_rotation_geom_get(const gct_ct_geom *geom, gct_rotation_geom *out, double *rot_ang,
                                 double *rel_rot_ang)
{
    return guarded([&] {
        gct::check_ct_geom(geom);
        if (!out) gct::fail(GCT_ERR_INVALID_ARG, "NULL output");
        gct::RotationInfo ri;
        if (!gct::rotation_info(*geom, &ri)) gct::fail(GCT_ERR_INVALID_ARG, "Invalid X-ray source trajectory.");
        out->dir = ri.dir;
        out->rot_ang_incr = ri.incr;
        out->rot_ang_range = ri.range;
        out->num_proj_per_rot = ri.num_proj_per_rot;
        if (rot_ang) std::copy(ri.rot_ang.begin(), ri.rot_ang.end(), rot_ang);
        if (rel_rot_ang) std::copy(ri.rel_rot_ang.begin(), ri.rel_rot_ang.end(), rel_rot_ang);
    });
}

gct_status gct_is_valid_axial_recon(const gct_ct_geom *geom, uint32_t proj_num_cols,
                                    uint32_t proj_num_rows, uint32_t num_proj, int32_t verbose,
                                    int32_t *valid)
{
    return guarded([&] {
        gct::check_ct_geom(geom);
        if (!valid) gct::fail(GCT_ERR_INVALID_ARG, "NULL output");
        bool ok = true;
        const auto kind = static_cast<gct_geom_kind>(geom->kind);
        // checkProjDetConsistency (src/cpp/recon/check_validity.h:30-64)
        if (proj_num_cols != geom->det_row.num_samples) {
            ok = false;
            if (verbose)
                std::fprintf(stderr,
                             "Inconsistent projection and detector geometry data.\n"
                             "Number of columns of projection image:: %u\nNumber of detector columns:: %u\n",
                             proj_num_cols, geom->det_row.num_samples);
        }
        if (ok && gct::is_2d_detector(kind) && proj_num_rows != geom->det_col.num_samples) {
            ok = false;
            if (verbose)
                std::fprintf(stderr,
                             "Inconsistent projection and detector geometry data.\n"
                             "Number of rows of projection image:: %u\nNumber of detector rows:: %u\n",
                             proj_num_rows, geom->det_col.num_samples);
        }
        // checkProjViewConsistency (check_validity.h:77-108)
        if (ok && num_proj != geom->num_views) {
            ok = false;
            if (verbose) {
                std::fprintf(stderr, "%s\n",
                             num_proj > geom->num_views
                                 ? "Projection geometry parameters are not available for all projection images."
                                 : "Projection images are not available for all projection geometries.");
                std::fprintf(stderr, "Number of projection images:: %u\nNumber of projection geometry objects:: %u\n",
                             num_proj, geom->num_views);
            }
        }
        *valid = ok ? 1 : 0;
    });
}

gct_status gct_ramp_filter_taps(int32_t kind, const gct_detector *det_row,
                                const gct_filt_params *params, double *taps)
{
    return guarded([&] {
        if (!det_row || !taps) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        if (kind < GCT_GEOM_PARALLEL_1D || kind > GCT_GEOM_CONE_FLAT) gct::fail(GCT_ERR_INVALID_ARG, "unknown geometry kind");
        const gct_filt_params fp = params ? *params : gct_filt_params{1.0, GCT_APOD_NONE};
        const auto t = gct::ramp_taps(static_cast<gct_geom_kind>(kind), *det_row, fp);
        std::copy(t.begin(), t.end(), taps);
    });
}

gct_status gct_parker_weights(const gct_ct_geom *geom, float *weights)
{
    return guarded([&] {
        gct::check_ct_geom(geom);
        if (!weights) gct::fail(GCT_ERR_INVALID_ARG, "NULL output");
        gct::RotationInfo ri;
        if (!gct::rotation_info(*geom, &ri)) gct::fail(GCT_ERR_INVALID_ARG, "Invalid X-ray source trajectory.");
        const auto w = gct::parker_table(*geom, ri);
        for (size_t i = 0; i < w.size(); ++i) weights[i] = static_cast<float>(w[i]);
    });
}

gct_status gct_map_point(const gct_ct_geom *geom, const gct_vol_geom *vol, uint32_t view, const double ijk[3],
                         double xyz[3], double *col, double *row, double *weight)
{
    return guarded([&] {
        gct::check_ct_geom(geom);
        const auto kind = static_cast<gct_geom_kind>(geom->kind);
        const bool vol3d = gct::is_2d_detector(kind);
        gct::check_vol_geom(vol, vol3d);
        if (!ijk) gct::fail(GCT_ERR_INVALID_ARG, "NULL voxel index");
        if (view >= geom->num_views) gct::fail(GCT_ERR_INVALID_ARG, "view index out of range");
        gct_ct_geom g1 = *geom;
        g1.num_views = 1;
        g1.views = geom->views + view;
        if (!vol3d) g1.det_col = gct_detector{1u, 1.0};
        const gct::ViewDerived d = gct::derive_view(kind, g1, 0);
        bool za = true;
        const std::vector<float> c = gct::bp_coefficients(g1, *vol, {d}, {d.bp_const}, &za);
        const double i = ijk[0], j = ijk[1], k = vol3d ? ijk[2] : 0.0;
        auto aff = [&](int o) { return c[o] + c[o + 1] * i + c[o + 2] * j + c[o + 3] * k; };
        double u = 0, v = 0, w = 0;
        switch (gct::family_of(kind)) {
            case gct::Family::Affine:
                u = c[0] + c[1] * i + c[2] * j;
                v = c[3] + c[4] * k;
                w = c[5];
                break;
            case gct::Family::Projective: {
                const double D = aff(8);
                u = aff(0) / D;
                v = aff(4) / D;
                w = c[12] / (D * D);
                break;
            }
            case gct::Family::Arc: {
                const double A = aff(0), B = aff(4), T = aff(8);
                const double rho2 = A * A + B * B;
                u = std::atan2(A, B) * c[12] + c[13];
                v = c[14] * T / std::sqrt(rho2) + c[15];
                w = c[16] / (rho2 + T * T);
                break;
            }
        }
        if (col) *col = u;
        if (row) *row = v;
        if (weight) *weight = w;
        if (xyz) {
            xyz[0] = vol->mid[0] - (vol->nx - 1.0) * vol->dx / 2.0 + i * vol->dx;
            xyz[1] = vol->mid[1] - (vol->ny - 1.0) * vol->dy / 2.0 + j * vol->dy;
            xyz[2] = vol3d ? vol->mid[2] - (vol->nz - 1.0) * vol->dz / 2.0 + k * vol->dz : 0.0;
        }
    });
}

gct_status gct_fdk_plan_create(const gct_ct_geom *geom, const gct_vol_geom *vol,
                               const gct_filt_params *filt, const gct_fdk_opts *opts,
                               gct_fdk_plan **out)
{
    return guarded([&] {
        if (!out) gct::fail(GCT_ERR_INVALID_ARG, "NULL plan output");
        *out = nullptr;
        PlanHolder h;
        h.p = new gct_fdk_plan();
        build_plan(h.p, geom, vol, filt, opts);
        // The allocation-free path's scratch array sits in this file's module, which the CUDA
        // runtime loads lazily: looking its address up here commits it on the plan's device at
        // plan creation, so gct_fdk_execute_noalloc never loads it.
        noalloc_scratch(h.p->device);
        *out = h.p;
        h.p = nullptr;
    });
}

gct_status gct_fdk_plan_destroy(gct_fdk_plan *plan)
{
    return guarded([&] {
        if (!plan) return;
        DeviceGuard dg(plan->device);
        delete plan;
    });
}

gct_status gct_fdk_plan_workspace_bytes(const gct_fdk_plan *plan, uint64_t *bytes)
{
    return guarded([&] {
        if (!plan || !bytes) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        *bytes = plan->workspace_bytes();
    });
}

gct_status gct_fdk_plan_symmetry(const gct_fdk_plan *plan, int32_t *quarter_turn)
{
    return guarded([&] {
        if (!plan || !quarter_turn) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        *quarter_turn = plan->sym;
    });
}

gct_status gct_fdk_plan_z_mirror(const gct_fdk_plan *plan, int32_t *mirror)
{
    return guarded([&] {
        if (!plan || !mirror) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        *mirror = plan->mirror ? 1 : 0;
    });
}

gct_status gct_fdk_execute(gct_fdk_plan *plan, const float *proj_dev, float *vol_dev, void *workspace,
                           void *stream)
{
    return guarded([&] {
        if (!plan) gct::fail(GCT_ERR_INVALID_ARG, "NULL plan");
        DeviceGuard dg(plan->device);
        execute(plan, proj_dev, vol_dev, workspace, static_cast<cudaStream_t>(stream));
    });
}

gct_status gct_fdk_plan_check(gct_fdk_plan *plan)
{
    return guarded([&] {
        if (!plan) gct::fail(GCT_ERR_INVALID_ARG, "NULL plan");
        DeviceGuard dg(plan->device);
        cuda_check(cudaDeviceSynchronize(), "device synchronisation");
        if (!plan->gemm_err.p) return;
        int e = 0;
        cuda_check(cudaMemcpy(&e, plan->gemm_err.p, sizeof(int), cudaMemcpyDeviceToHost), "GEMM status read");
        if (e) {
            cuda_check(cudaMemset(plan->gemm_err.p, 0, sizeof(int)), "kernel status reset");
            if (e & gct::kFftWaitTimeout)
                gct::fail(GCT_ERR_TIMEOUT, "FFT filter: a projection row copy did not arrive within 2 s");
            if (e & gct::kQuadWaitTimeout)
                gct::fail(GCT_ERR_TIMEOUT, "quad formation: a filtered row copy did not arrive within 2 s");
            gct::fail(GCT_ERR_TIMEOUT, "Toeplitz GEMM pipeline wait timed out (stage " + std::to_string(e) + ")");
        }
    });
}

gct_status gct_fdk_filter(gct_fdk_plan *plan, const float *proj_dev, float *filtered_dev, void *stream)
{
    return guarded([&] {
        if (!plan || !proj_dev || !filtered_dev) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        DeviceGuard dg(plan->device);
        run_filter(plan, proj_dev, filtered_dev, nullptr, gct::kOutPlainF32, 0, 0, plan->nv,
                   static_cast<cudaStream_t>(stream));
    });
}

gct_status gct_fdk_prepare(gct_fdk_plan *plan, const float *proj_dev, void *workspace, uint32_t view_begin,
                           uint32_t view_count, void *stream)
{
    return guarded([&] {
        if (!plan) gct::fail(GCT_ERR_INVALID_ARG, "NULL plan");
        check_range(plan, view_begin, view_count);
        DeviceGuard dg(plan->device);
        const StackRef st = stack_of(plan, plan_workspace(plan, workspace));
        const auto s = static_cast<cudaStream_t>(stream);
        // a whole quarter-turn stack in one coalesced pass; partial ranges write their quads into
        // the interleaved layout one view at a time
        if (st.quarter && view_begin == 0 && view_count == static_cast<uint32_t>(plan->nv))
            prepare_partners(plan, proj_dev, st, 0, st.quarter, s);
        else
            prepare(plan, proj_dev, st, static_cast<int>(view_begin), static_cast<int>(view_count), s);
    });
}

gct_status gct_fdk_backproject(gct_fdk_plan *plan, const void *workspace, float *vol_dev, uint32_t view_begin,
                               uint32_t view_count, int32_t accumulate, void *stream)
{
    return guarded([&] {
        if (!plan || !vol_dev) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        check_range(plan, view_begin, view_count);
        DeviceGuard dg(plan->device);
        void *ws = workspace ? const_cast<void *>(workspace) : plan->work.p;
        if (!ws) gct::fail(GCT_ERR_INVALID_ARG, "no workspace: run gct_fdk_prepare first or pass one");
        run_backproject(plan, stack_of(plan, ws), vol_dev, static_cast<int>(view_begin), static_cast<int>(view_count),
                        accumulate != 0, static_cast<cudaStream_t>(stream));
    });
}

gct_status gct_fdk_execute_host(gct_fdk_plan *plan, const float *proj_host, float *vol_host, void *stream)
{
    return guarded([&] {
        if (!plan) gct::fail(GCT_ERR_INVALID_ARG, "NULL plan");
        DeviceGuard dg(plan->device);
        execute_host(plan, proj_host, vol_host, static_cast<cudaStream_t>(stream), true);
    });
}

gct_status gct_fdk_execute_host_async(gct_fdk_plan *plan, const float *proj_host, float *vol_host, void *stream)
{
    return guarded([&] {
        if (!plan) gct::fail(GCT_ERR_INVALID_ARG, "NULL plan");
        DeviceGuard dg(plan->device);
        execute_host(plan, proj_host, vol_host, static_cast<cudaStream_t>(stream), false);
    });
}

gct_status gct_fdk_host_sync(gct_fdk_plan *plan)
{
    return guarded([&] {
        if (!plan) gct::fail(GCT_ERR_INVALID_ARG, "NULL plan");
        DeviceGuard dg(plan->device);
        if (plan->d2h_stream) cuda_check(cudaStreamSynchronize(plan->d2h_stream), "reconstruction");
    });
}

}  // extern "C"

// ---- execution without device allocation ---------------------------------------------------
// Scratch of gct_fdk_execute_noalloc: filtered-projection quads of one chunk of views. The array
// lives on every device that loads the library. Host code must not pass its name to a kernel
// (on the host it is only a stand-in); the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[GCT_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxNoAllocDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_addr[kMaxNoAllocDevices] = {};

// Device address of the scratch on `dev` (the current device), looked up once per device.
unsigned char *noalloc_scratch(int dev)
{
    if (dev < 0 || dev >= kMaxNoAllocDevices) gct::fail(GCT_ERR_NOT_SUPPORTED, "device index beyond 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "scratch address lookup");
        g_noalloc_addr[dev] = p;
    }
    return static_cast<unsigned char *>(g_noalloc_addr[dev]);
}

void execute_noalloc(gct_fdk_plan *p, const float *proj, float *vol, cudaStream_t s)
{
    if (!proj || !vol) gct::fail(GCT_ERR_INVALID_ARG, "NULL projection or volume pointer");
    // per view: its quads and, for FP16 storage, three floats (maximum, scale, inverse scale)
    const size_t quads_per_view = p->view_bytes();
    const size_t scales_per_view = p->opts.storage == GCT_STORAGE_F16 ? 3 * sizeof(float) : 0;
    const size_t per_view = quads_per_view + scales_per_view;
    if (per_view + 256 > GCT_NOALLOC_SCRATCH_BYTES)
        gct::fail(GCT_ERR_BUDGET, "one view needs " + std::to_string(per_view) +
                                      " bytes of filtered-projection scratch; the allocation-free path holds " +
                                      std::to_string(GCT_NOALLOC_SCRATCH_BYTES) + " bytes");
    const int chunk =
        static_cast<int>(std::min<size_t>(static_cast<size_t>(p->nv), (GCT_NOALLOC_SCRATCH_BYTES - 256) / per_view));
    unsigned char *scratch = noalloc_scratch(p->device);
    // the chunk's scales follow its quads, 256-byte aligned
    float *scales = reinterpret_cast<float *>(
        scratch + ((static_cast<size_t>(chunk) * quads_per_view + 255) & ~static_cast<size_t>(255)));
    for (int vb = 0; vb < p->nv; vb += chunk) {
        const int vc = std::min(chunk, p->nv - vb);
        // prepare() and run_backproject() address view v at view-0 bases; shifting every base by
        // vb views puts this chunk at the start of its scratch region.
        StackRef st;
        st.quads = reinterpret_cast<unsigned char *>(reinterpret_cast<uintptr_t>(scratch) -
                                                     static_cast<uintptr_t>(vb) * quads_per_view);
        if (scales_per_view) {
            st.amax = scales - vb;
            st.vscale = scales + chunk - vb;
            st.vinv = scales + 2 * chunk - vb;
        }
        prepare(p, proj, st, vb, vc, s);
        run_backproject(p, st, vol, vb, vc, vb > 0, s, false);  // allocates nothing
    }
}
}  // namespace

extern "C" {

gct_status gct_fdk_execute_noalloc(gct_fdk_plan *plan, const float *proj_dev, float *vol_dev, void *stream)
{
    return guarded([&] {
        if (!plan) gct::fail(GCT_ERR_INVALID_ARG, "NULL plan");
        DeviceGuard dg(plan->device);
        execute_noalloc(plan, proj_dev, vol_dev, static_cast<cudaStream_t>(stream));
    });
}

gct_status gct_fdk_execute_host_budget(gct_fdk_plan *plan, const float *proj_host, float *vol_host,
                                       uint64_t device_bytes, void *stream)
{
    return guarded([&] {
        if (!plan) gct::fail(GCT_ERR_INVALID_ARG, "NULL plan");
        DeviceGuard dg(plan->device);
        execute_host_budget(plan, proj_host, vol_host, device_bytes, static_cast<cudaStream_t>(stream));
    });
}

gct_status gct_reconstruct_ex(const gct_ct_geom *geom, const gct_vol_geom *vol,
                              const gct_filt_params *filt, const gct_fdk_opts *opts,
                              const float *proj_host, float *vol_host)
{
    return guarded([&] {
        if (!proj_host || !vol_host) gct::fail(GCT_ERR_INVALID_ARG, "NULL projection or volume pointer");
        PlanHolder h;
        h.p = new gct_fdk_plan();
        build_plan(h.p, geom, vol, filt, opts);
        gct_fdk_plan *p = h.p;
        const size_t proj_n = static_cast<size_t>(p->nv) * p->nr * p->nc;
        const size_t vol_n = static_cast<size_t>(p->vol.nx) * p->vol.ny * p->vol.nz;
        // reconFDK's choice (src/cuda/recon/fdk_axial.cuh:68-89): all projections on the device
        // when they, the volume and the filtered stack need under 75 % of the device memory,
        // else the streaming path with half of the memory left after the volume
        size_t free_b = 0, total_b = 0;
        cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
        const double req = static_cast<double>(proj_n + vol_n) * sizeof(float) + static_cast<double>(p->workspace_bytes());
        if (req >= 0.75 * static_cast<double>(total_b)) {
            const size_t vol_b = vol_n * sizeof(float);
            execute_host_budget(p, proj_host, vol_host, free_b > vol_b ? (free_b - vol_b) / 2 : 0, nullptr);
            return;
        }
        DevBuf<float> dproj, dvol;
        dproj.alloc(proj_n, "projection stack");
        dvol.alloc(vol_n, "volume");
        cudaStream_t s = nullptr;
        cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
        std::unique_ptr<CUstream_st, void (*)(cudaStream_t)> sg(s, [](cudaStream_t x) { cudaStreamDestroy(x); });
        cuda_check(cudaMemcpyAsync(dproj.p, proj_host, proj_n * sizeof(float), cudaMemcpyHostToDevice, s),
                   "projection upload");
        execute(p, dproj.p, dvol.p, nullptr, s);
        cuda_check(cudaMemcpyAsync(vol_host, dvol.p, vol_n * sizeof(float), cudaMemcpyDeviceToHost, s),
                   "volume download");
        cuda_check(cudaStreamSynchronize(s), "reconstruction");
    });
}

gct_status gct_reconstruct(const gct_ct_geom *geom, const gct_vol_geom *vol, const float *proj_host,
                           float *vol_host)
{
    return gct_reconstruct_ex(geom, vol, nullptr, nullptr, proj_host, vol_host);
}

namespace {
std::vector<gct::ProjView> proj_views(const gct_ct_geom &g)
{
    const auto kind = static_cast<gct_geom_kind>(g.kind);
    std::vector<gct::ProjView> pv(g.num_views);
    for (unsigned v = 0; v < g.num_views; ++v) {
        const gct::ViewDerived d = gct::derive_view(kind, g, v);
        gct::ProjView &o = pv[v];
        for (int i = 0; i < 3; ++i) {
            o.src[i] = d.src[i];
            o.eu[i] = d.eu[i];
            o.ev[i] = d.ev[i];
            o.ew[i] = d.ew[i];
        }
        o.sdd = d.sdd;
        o.c0 = d.c0;
        o.r0 = d.r0;
        o.extra = d.theta;
        o.zscale = (kind == GCT_GEOM_CONE_PARALLEL) ? d.sid / d.sdd : 1.0;
    }
    return pv;
}
}  // namespace

gct_status gct_phantom_project(const gct_ct_geom *geom, const gct_ellipsoid *ellipsoids,
                               uint32_t num_ellipsoids, float *proj_dev, void *stream)
{
    return guarded([&] {
        gct::check_ct_geom(geom);
        if (!proj_dev || (num_ellipsoids && !ellipsoids)) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        const auto kind = static_cast<gct_geom_kind>(geom->kind);
        const auto pv = proj_views(*geom);
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        DevBuf<gct::ProjView> dv;
        DevBuf<gct_ellipsoid> de;
        dv.upload(pv.data(), pv.size(), "phantom geometry");
        de.upload(ellipsoids, num_ellipsoids, "phantom ellipsoids");
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int nr = gct::is_2d_detector(kind) ? static_cast<int>(geom->det_col.num_samples) : 1;
        gct::launch_phantom(dv.p, kind, static_cast<int>(geom->num_views), nr,
                            static_cast<int>(geom->det_row.num_samples), geom->det_row.sampling_width,
                            gct::is_2d_detector(kind) ? geom->det_col.sampling_width : 1.0, de.p,
                            static_cast<int>(num_ellipsoids), !gct::is_2d_detector(kind), proj_dev, sms, s);
        cuda_check(cudaGetLastError(), "phantom kernel launch");
        cuda_check(cudaStreamSynchronize(s), "phantom projection");  // buffers are freed on return
    });
}

gct_status gct_forward_project(const gct_ct_geom *geom, const gct_vol_geom *vol, const float *vol_dev,
                               float step_vox, float *proj_dev, void *stream)
{
    return guarded([&] {
        gct::check_ct_geom(geom);
        const auto kind = static_cast<gct_geom_kind>(geom->kind);
        const bool vol3d = gct::is_2d_detector(kind);
        gct::check_vol_geom(vol, vol3d);
        if (!vol_dev || !proj_dev) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        if (!(step_vox > 0.f)) gct::fail(GCT_ERR_INVALID_ARG, "step must be positive");
        const auto pv = proj_views(*geom);
        gct::VolBox box{};
        const unsigned n[3] = {vol->nx, vol->ny, vol->nz};
        const double w[3] = {vol->dx, vol->dy, vol3d ? vol->dz : 1.0};
        for (int a = 0; a < 3; ++a) {
            const double mid = (a == 2 && !vol3d) ? 0.0 : vol->mid[a];
            box.w[a] = w[a];
            box.lo[a] = mid - (n[a] - 1.0) * w[a] / 2.0;
            box.hi[a] = mid + (n[a] - 1.0) * w[a] / 2.0;
        }
        box.nx = static_cast<int>(vol->nx);
        box.ny = static_cast<int>(vol->ny);
        box.nz = static_cast<int>(vol->nz);
        box.planar = !vol3d;
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        DevBuf<gct::ProjView> dv;
        dv.upload(pv.data(), pv.size(), "projector geometry");
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int nr = vol3d ? static_cast<int>(geom->det_col.num_samples) : 1;
        gct::launch_forward(dv.p, kind, static_cast<int>(geom->num_views), nr,
                            static_cast<int>(geom->det_row.num_samples), geom->det_row.sampling_width,
                            vol3d ? geom->det_col.sampling_width : 1.0, vol_dev, box, step_vox, proj_dev, sms, s);
        cuda_check(cudaGetLastError(), "forward projector launch");
        cuda_check(cudaStreamSynchronize(s), "forward projection");
    });
}

}  // extern "C"
