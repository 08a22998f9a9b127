// Internal host interface of the FDK engine: the plan, device buffers, error plumbing and the
// stage functions shared by the C ABI (abi.cu), the batch engine (batch.cu) and the serving loop
// (server.cu). Not part of the public ABI.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/gct_fdk.h"
#include "geometry.hpp"
#include "kernels.hpp"

// Records msg as the calling thread's last error and returns s.
gct_status set_error(gct_status s, const std::string &msg);
// Throws gct::GctError (GCT_ERR_OUT_OF_MEMORY or GCT_ERR_CUDA) for a failed CUDA call.
void cuda_check(cudaError_t e, const char *what);

template <class F>
gct_status guarded(F &&f)
{
    try {
        f();
        return GCT_OK;
    } catch (const gct::GctError &e) {
        return set_error(e.status, e.msg);
    } catch (const std::bad_alloc &) {
        return set_error(GCT_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception &e) {
        return set_error(GCT_ERR_INVALID_ARG, e.what());
    }
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { reset(); }
    void reset()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count, const char *what)
    {
        reset();
        if (count == 0) return;
        cuda_check(cudaMalloc(reinterpret_cast<void **>(&p), count * sizeof(T)), what);
        n = count;
    }
    void upload(const T *host, size_t count, const char *what)
    {
        alloc(count, what);
        if (count) cuda_check(cudaMemcpy(p, host, count * sizeof(T), cudaMemcpyHostToDevice), what);
    }
};

struct gct_fdk_plan {
    int device = 0;
    int num_sms = 148;
    gct_geom_kind kind = GCT_GEOM_CONE_FLAT;
    gct::Family family = gct::Family::Projective;
    std::vector<gct_view_geom> views;
    gct_ct_geom geom{};
    gct_vol_geom vol{};
    gct_filt_params filt{};
    gct_fdk_opts opts{};
    gct::RotationInfo rot;
    bool z_affine = true;
    unsigned L = 0;
    int nv = 0, nr = 0, nc = 0;
    float l1 = 0.f;
    int zpt = 8, bx = 32, by = 8;
    // One-row 1D parallel detectors run transposed (kT1dPitch): the backprojector sees the image
    // as kx x 1 x kz voxels (z = image y) over a one-column detector of nc rows.
    bool t1d = false;
    int kx = 0, ky = 0, kz = 0;  // backprojector grid (the image's [z][y][x] memory either way)
    // Quarter-turn symmetry (+1 / -1 / 0, quarter_turn_symmetry): whole-scan backprojections then
    // run over the first quarter of the views and of the (x, y) columns, each thread serving the
    // four rotated columns from the four partner views, with zpt_sym voxels along z.
    int sym = 0, zpt_sym = 8, bx_sym = 8, by_sym = 16;
    // z-mirror symmetry (z_mirror_symmetry): column kernels over the lower half of the grid, each
    // thread also summing its mirror voxels
    bool mirror = false;
    // spiral scans: per-slice view windows (first, count); count 0 leaves the slice zero
    bool spiral = false;
    DevBuf<int2> slice_views;
    DevBuf<float4> fview;
    DevBuf<float> parker;
    DevBuf<float2> H;
    DevBuf<float> bp_part;  // partial images of view-split backprojections (run_backproject)
    DevBuf<float> coefs;
    DevBuf<unsigned char> work;
    // Toeplitz-GEMM filter: B = T^T split into 16-bit hi/lo pieces [Np][Kp] (BF16, or FP16 bit
    // patterns in the FP16 form), A rows [nv*nr][Kp], FP32 rows
    int Kp = 0, Np = 0;
    DevBuf<__nv_bfloat16> th, tl, xh, xl;
    DevBuf<__nv_bfloat16> xll, tll;  // four-term filter: third piece of the rows; third tap piece over the band
    DevBuf<float> grinv;             // FP16 form: per-row inverse scale of the GEMM rows
    float tap_inv = 1.f;             // FP16 form: inverse of the taps' power-of-two scale
    DevBuf<float> ybuf;
    DevBuf<int> gemm_err;  // kernel status word (GEMM pipeline and FFT input waits)
    // staging for gct_fdk_execute_host: projections, two device volumes (consecutive calls
    // alternate, so one call's download overlaps the next call's backprojection)
    DevBuf<float> host_proj, host_vol, host_vol2;
    cudaStream_t copy_stream = nullptr, d2h_stream = nullptr;
    std::vector<cudaEvent_t> chunk_events, prep_events;  // per chunk: upload done, filter done
    cudaEvent_t vol_free[2] = {nullptr, nullptr}, bp_done = nullptr;
    unsigned host_calls = 0;
    // bounded-memory streaming (gct_fdk_execute_host_budget): two projection slots of
    // stream_chunk views and a view-major stack of one chunk
    DevBuf<float> stream_stage;
    DevBuf<unsigned char> stream_ws;
    int stream_chunk = 0;
    cudaEvent_t stream_events[4] = {nullptr, nullptr, nullptr, nullptr};  // slot filled x2, slot free x2

    ~gct_fdk_plan()
    {
        for (cudaEvent_t e : chunk_events) cudaEventDestroy(e);
        for (cudaEvent_t e : prep_events) cudaEventDestroy(e);
        for (cudaEvent_t e : {vol_free[0], vol_free[1], bp_done})
            if (e) cudaEventDestroy(e);
        if (d2h_stream) cudaStreamDestroy(d2h_stream);
        for (cudaEvent_t e : stream_events)
            if (e) cudaEventDestroy(e);
        if (copy_stream) cudaStreamDestroy(copy_stream);
    }

    size_t quad_bytes() const { return opts.storage == GCT_STORAGE_F16 ? 8 : 16; }
    // Workspace layout: the quads of view v at v * view_bytes(), then (FP16 storage) the per-view
    // maxima, scales and inverse scales, nv floats each, from quad_region() on.
    size_t view_bytes() const
    {
        return static_cast<size_t>(nr + 2 * gct::kQuadPad) * (nc + 2 * gct::kQuadPad) * quad_bytes();
    }
    size_t quad_region() const { return (static_cast<size_t>(nv) * view_bytes() + 255) & ~static_cast<size_t>(255); }
    size_t scale_bytes() const { return opts.storage == GCT_STORAGE_F16 ? 3 * sizeof(float) * nv : 0; }
    size_t workspace_bytes() const { return quad_region() + scale_bytes(); }
};

// One filtered stack: the quads of view v at quads + v * view_bytes() and, for FP16 storage, the
// view's maximum, scale and inverse scale at amax[v], vscale[v], vinv[v]. All four are view-0
// addresses, so a chunk of views may live at a shifted base.
struct StackRef {
    unsigned char *quads = nullptr;
    float *amax = nullptr, *vscale = nullptr, *vinv = nullptr;
    int quarter = 0;  // quad_layout of the quads (kernels.hpp)
};

// A plan's stack in `workspace`. Quarter-turn plans interleave partner views (quad_layout) unless
// `view_major` asks for the plain layout, which the work-queue backprojector of batches and the
// server reads.
inline StackRef stack_of(const gct_fdk_plan *p, void *workspace, bool view_major = false)
{
    StackRef r;
    r.quads = static_cast<unsigned char *>(workspace);
    r.quarter = (p->sym && !view_major) ? p->nv / 4 : 0;
    if (p->opts.storage == GCT_STORAGE_F16) {
        r.amax = reinterpret_cast<float *>(r.quads + p->quad_region());
        r.vscale = r.amax + p->nv;
        r.vinv = r.vscale + p->nv;
    }
    return r;
}

// Stage functions (abi.cu). `out` / StackRef bases are view-0 addresses; [vb, vb + vc) is the
// view range worked on.
void run_filter(gct_fdk_plan *p, const float *proj, void *out, const float *vscale, int mode, int quarter, int vb,
                int vc, cudaStream_t s, const StackRef *fused_scales = nullptr);
void prepare(gct_fdk_plan *p, const float *proj, const StackRef &st, int vb, int vc, cudaStream_t s);
// Quarter-turn stacks (st.quarter > 0): base views [b, b + n) and their partners. FP16 storage
// with a Toeplitz filter: one GEMM whose epilogue writes the partner groups; otherwise through the
// plan's FP32 row buffer and one coalesced pass that writes them.
void prepare_partners(gct_fdk_plan *p, const float *proj, const StackRef &st, int b, int n, cudaStream_t s);
gct::BpArgs bp_args(const gct_fdk_plan *p, const StackRef &st, float *vol, int v_begin, int v_count);
// `split`: a one-voxel-deep image whose launch would leave most of the GPU idle is backprojected
// in view chunks into partial images (plan-owned, allocated on first use) and summed in chunk
// order; callers that must not allocate pass false.
void run_backproject_sym(gct_fdk_plan *p, const StackRef &st, float *vol, int b_begin, int b_count,
                         bool accumulate, cudaStream_t s, bool split = true);
void run_backproject(gct_fdk_plan *p, const StackRef &st, float *vol, int v_begin, int v_count, bool accumulate,
                     cudaStream_t s, bool split = true);
void check_range(const gct_fdk_plan *p, uint32_t vb, uint32_t vc);
void *plan_workspace(gct_fdk_plan *p, void *workspace);
