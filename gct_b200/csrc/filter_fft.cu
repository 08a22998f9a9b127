// Row-batched ramp filter: cosine and Parker weights fused into the load, a Stockham radix-4/2
// FFT convolution with the ramp spectrum in shared memory, and an epilogue that writes either
// plain FP32 rows or the padded bilinear-coefficient quads read by the backprojector. Two
// detector rows share one complex FFT (row a in the real part, row b in the imaginary part): the
// ramp taps are real, so the two convolutions stay separated.
//
// Replaces runCosWeighting (src/cuda/recon/cos_weighting.cuh:225-263), runParkerWeighting
// (src/cuda/recon/parker_weighting.cuh:202-230) and RampFilteringFFT::runFiltering
// (src/cuda/recon/ramp_filtering_fft.cuh:208-219): the reference pads to nextPow2(2N), runs
// cuFFT R2C/C2R and crops at N/2 in five passes over HBM; here the taps are placed circularly so
// the crop disappears, the shortest alias-free power of two (> 1.5 N) is used, and each row is
// read once and written once.
//
// Work split: one CTA per (view, segment of rows). A CTA walks its rows in order, keeps the
// previous filtered row in shared memory and writes the quad of row r once rows r and r + 1 are
// known, so every quad is written whole by one CTA. Each segment filters one extra row (the first
// row of the next segment) to close its last quad.
#include "../../include/gct_fdk.h"
#include "common.cuh"
#include "kernels.hpp"

namespace gct {
namespace {

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// Shared-memory index with one float2 of padding per 16: strided Stockham writes then spread
// over all banks.
__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }

// One Stockham stage (Govindaraju et al., SC'08). Butterfly j reads x[j + r L/R], multiplies by
// the twiddle W_{R Ns}^(r (j mod Ns)) and writes its R-point DFT to
// y[(j / Ns) Ns R + (j mod Ns) + r Ns]; after all stages the output is in natural order.
// Twiddles of a stage with span Ns live contiguously at tw[Ns + k], k < Ns.
// LAST fuses the pointwise product with the spectrum H and the conjugation that turns the next
// forward FFT into the inverse.
template <int L, int NT, bool LAST>
__device__ __forceinline__ void stage_r4(const float2 *src, float2 *dst, const float2 *tw, const float2 *H,
                                         int Ns, int tid)
{
    for (int j = tid; j < L / 4; j += NT) {
        const int k = j & (Ns - 1);
        float2 v0 = src[pad(j)], v1 = src[pad(j + L / 4)], v2 = src[pad(j + L / 2)], v3 = src[pad(j + 3 * L / 4)];
        if (Ns > 1) {
            const float2 w1 = tw[Ns + k];
            const float2 w2 = cmul(w1, w1);
            v1 = cmul(v1, w1);
            v2 = cmul(v2, w2);
            v3 = cmul(v3, cmul(w2, w1));
        }
        const float2 t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3);
        const float2 d = csub(v1, v3);
        const float2 t3 = make_float2(d.y, -d.x);  // -i * (v1 - v3)
        const int idx = (j - k) * 4 + k;
        float2 y[4] = {cadd(t0, t2), cadd(t1, t3), csub(t0, t2), csub(t1, t3)};
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            float2 o = y[r];
            if (LAST) {
                o = cmul(o, __ldg(H + idx + r * Ns));
                o.y = -o.y;
            }
            dst[pad(idx + r * Ns)] = o;
        }
    }
}

template <int L, int NT, bool LAST>
__device__ __forceinline__ void stage_r2(const float2 *src, float2 *dst, const float2 *tw, const float2 *H,
                                         int Ns, int tid)
{
    for (int j = tid; j < L / 2; j += NT) {
        const int k = j & (Ns - 1);
        float2 v0 = src[pad(j)], v1 = src[pad(j + L / 2)];
        if (Ns > 1) v1 = cmul(v1, tw[Ns + k]);
        const int idx = (j - k) * 2 + k;
        float2 y0 = cadd(v0, v1), y1 = csub(v0, v1);
        if (LAST) {
            y0 = cmul(y0, __ldg(H + idx));
            y0.y = -y0.y;
            y1 = cmul(y1, __ldg(H + idx + Ns));
            y1.y = -y1.y;
        }
        dst[pad(idx)] = y0;
        dst[pad(idx + Ns)] = y1;
    }
}

// Remaining stages of an L-point FFT whose first radix-4 stage (Ns = 1) is already in `a`.
// Ping-pongs between a and b; returns the buffer holding the result.
template <int LOG2L, int NT, bool FUSE_H>
__device__ __forceinline__ float2 *fft_rest(float2 *a, float2 *b, const float2 *tw, const float2 *H, int tid)
{
    constexpr int L = 1 << LOG2L;
    constexpr int NR4 = LOG2L / 2;
    float2 *src = a, *dst = b;
    int Ns = 4;
#pragma unroll
    for (int s = 1; s < NR4; ++s) {
        const bool last = (s == NR4 - 1) && !(LOG2L & 1);
        if (FUSE_H && last)
            stage_r4<L, NT, true>(src, dst, tw, H, Ns, tid);
        else
            stage_r4<L, NT, false>(src, dst, tw, H, Ns, tid);
        __syncthreads();
        float2 *t = src;
        src = dst;
        dst = t;
        Ns *= 4;
    }
    if (LOG2L & 1) {
        if (FUSE_H)
            stage_r2<L, NT, true>(src, dst, tw, H, Ns, tid);
        else
            stage_r2<L, NT, false>(src, dst, tw, H, Ns, tid);
        __syncthreads();
        float2 *t = src;
        src = dst;
        dst = t;
    }
    return src;
}

// First radix-4 stage of the inverse transform (input already conjugated in smem).
template <int L, int NT>
__device__ __forceinline__ void first_stage_smem(const float2 *src, float2 *dst, int tid)
{
    stage_r4<L, NT, false>(src, dst, nullptr, nullptr, 1, tid);
}

// Quad of rows (top, bot) at column c in the storage form of MODE (quad_f32 / quad_f16).
template <int MODE>
__device__ __forceinline__ void store_quad(void *out, long long qidx, float p00, float p01, float p10, float p11)
{
    if (MODE == kOutQuadF32)
        static_cast<float4 *>(out)[qidx] = quad_f32(p00, p01, p10, p11);
    else
        static_cast<uint2 *>(out)[qidx] = quad_f16(p00, p01, p10, p11);
}

// Writes quad row `r` (detector row r, padded index r + kQuadPad) of view v from the filtered
// rows `top` (row r) and `bot` (row r + 1); either may be NULL for a zero row. Values are scaled
// by `sc`. Rows read from the FFT buffer use its padded indexing and sign.
template <int MODE>
__device__ __forceinline__ void write_quad_row(const FilterArgs &a, int v, int r, const float *top,
                                               const float2 *bot, bool bot_imag, float sc, int tid, int nthr)
{
    const int nc = a.nc;
    const int qpitch = nc + 2 * kQuadPad;
    long long first;
    int step;
    quad_layout(a.v0 + v, static_cast<long long>(a.nr + 2 * kQuadPad) * qpitch, a.quarter, first, step);
    const long long row0 = first + static_cast<long long>(r + kQuadPad) * qpitch * step;
    auto tv = [&](int c) -> float { return (top && c >= 0 && c < nc) ? top[c] : 0.0f; };
    auto bv = [&](int c) -> float {
        if (!bot || c < 0 || c >= nc) return 0.0f;
        const float2 z = bot[pad(c)];
        return sc * (bot_imag ? -z.y : z.x);
    };
    for (int cq = tid; cq < qpitch; cq += nthr) {
        const int c = cq - kQuadPad;
        store_quad<MODE>(a.out, row0 + static_cast<long long>(cq) * step, tv(c), tv(c + 1), bv(c), bv(c + 1));
    }
}

// Transposed quad grid of view v of a one-row detector from its filtered, scaled row y (shared).
template <int MODE>
__device__ __forceinline__ void write_quads_t1d(const FilterArgs &a, int v, const float *y, int tid, int nthr)
{
    const int nc = a.nc, rows = nc + 2 * kQuadPad;
    const long long base = static_cast<long long>(a.v0 + v) * rows * kT1dPitch;
    auto yv = [&](int r) -> float { return (r >= 0 && r < nc) ? y[r] : 0.0f; };
    for (int e = tid; e < rows * kT1dPitch; e += nthr) {
        const int r = e / kT1dPitch - kQuadPad, c = e % kT1dPitch - kQuadPad;
        const float t = yv(r), b = yv(r + 1);
        if (c == 0)
            store_quad<MODE>(a.out, base + e, t, 0.0f, b, 0.0f);
        else if (c == -1)
            store_quad<MODE>(a.out, base + e, 0.0f, t, 0.0f, b);
        else
            store_quad<MODE>(a.out, base + e, 0.0f, 0.0f, 0.0f, 0.0f);
    }
}

template <int LOG2L, int MODE>
__global__ void __launch_bounds__(256) filter_fft_kernel(FilterArgs a, int seg_rows, int nseg)
{
    constexpr int L = 1 << LOG2L;
    constexpr int NT = (L / 4 < 256) ? L / 4 : 256;
    constexpr int LP = L + L / 16;
    extern __shared__ float2 smem[];
    float2 *tw = smem, *b0 = smem + L, *b1 = smem + L + LP;
    float *yprev = reinterpret_cast<float *>(smem + L + 2 * LP);
    const int tid = threadIdx.x;
    for (int m = tid; m < L; m += NT) tw[m] = a.twiddle[m];

    const int nc = a.nc, nr = a.nr;
    for (long long blk = blockIdx.x; blk < static_cast<long long>(a.nv) * nseg; blk += gridDim.x) {
        const int v = static_cast<int>(blk / nseg), s = static_cast<int>(blk - static_cast<long long>(v) * nseg);
        const int r0 = s * seg_rows, r1 = min(r0 + seg_rows, nr);
        const bool quads = MODE != kOutPlainF32;
        const int last_row = (quads && r1 < nr) ? r1 : r1 - 1;  // quads: one extra row closes the segment
        const float4 gv = __ldg(&a.fview[v]);
        const float *wpk = a.parker + static_cast<long long>(v) * nc;
        const float sc = (quads && a.vscale) ? a.vscale[v] : 1.0f;
        int prev_row = r0 - 1;
        bool have_prev = false;
        if (quads && s == 0 && !a.t1d) {
            write_quad_row<MODE>(a, v, -2, nullptr, nullptr, false, sc, tid, NT);
            for (int c = tid; c < nc; c += NT) yprev[c] = 0.0f;  // row -1 is zero
            have_prev = true;
        }
        __syncthreads();
        for (int ra = r0; ra <= last_row; ra += 2) {
            const bool has_b = ra + 1 <= last_row;
            const float *pa = a.proj + (static_cast<long long>(v) * nr + ra) * nc;
            const float *pb = pa + nc;
            // load, weight and first radix-4 stage straight from global memory
            for (int j = tid; j < L / 4; j += NT) {
                float2 x[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int k = j + q * (L / 4);
                    x[q] = make_float2(0.f, 0.f);
                    if (k < nc) {
                        const float w = __ldg(wpk + k);
                        x[q].x = __ldg(pa + k) * w * cos_weight_dev(a.kind, gv.x, gv.y, gv.z, a.du, a.dv, k, ra);
                        if (has_b) x[q].y = __ldg(pb + k) * w * cos_weight_dev(a.kind, gv.x, gv.y, gv.z, a.du, a.dv, k, ra + 1);
                    }
                }
                const float2 t0 = cadd(x[0], x[2]), t1 = csub(x[0], x[2]), t2 = cadd(x[1], x[3]);
                const float2 d = csub(x[1], x[3]);
                const float2 t3 = make_float2(d.y, -d.x);
                b0[pad(4 * j)] = cadd(t0, t2);
                b0[pad(4 * j + 1)] = cadd(t1, t3);
                b0[pad(4 * j + 2)] = csub(t0, t2);
                b0[pad(4 * j + 3)] = csub(t1, t3);
            }
            __syncthreads();
            float2 *spec = fft_rest<LOG2L, NT, true>(b0, b1, tw, a.H, tid);  // conj(FFT(x) H)
            float2 *other = (spec == b0) ? b1 : b0;
            first_stage_smem<L, NT>(spec, other, tid);
            __syncthreads();
            float2 *res = fft_rest<LOG2L, NT, false>(other, spec, tw, a.H, tid);  // conj of the filtered rows
            // rows: ra in .x, ra + 1 in -.y
            for (int h = 0; h < (has_b ? 2 : 1); ++h) {
                const int rr = ra + h;
                if (!quads) {
                    if (rr < r1) {
                        float *out = static_cast<float *>(a.out) + (static_cast<long long>(v) * nr + rr) * nc;
                        for (int c = tid; c < nc; c += NT) out[c] = h ? -res[pad(c)].y : res[pad(c)].x;
                    }
                    continue;
                }
                if (have_prev) write_quad_row<MODE>(a, v, prev_row, yprev, res, h == 1, sc, tid, NT);
                __syncthreads();
                for (int c = tid; c < nc; c += NT) yprev[c] = sc * (h ? -res[pad(c)].y : res[pad(c)].x);
                prev_row = rr;
                have_prev = true;
                __syncthreads();
            }
            __syncthreads();
        }
        if (quads && a.t1d) {  // one-row detector: the transposed grid from the filtered row
            write_quads_t1d<MODE>(a, v, yprev, tid, NT);
        } else if (quads && r1 == nr) {  // last segment: rows nr-1 (bottom neighbour zero), nr and nr+1
            write_quad_row<MODE>(a, v, nr - 1, yprev, nullptr, false, sc, tid, NT);
            write_quad_row<MODE>(a, v, nr, nullptr, nullptr, false, sc, tid, NT);
            write_quad_row<MODE>(a, v, nr + 1, nullptr, nullptr, false, sc, tid, NT);
        }
        __syncthreads();
    }
}

template <int LOG2L>
size_t smem_bytes_log2(int nc)
{
    constexpr int L = 1 << LOG2L;
    return (static_cast<size_t>(L) + 2 * (L + L / 16)) * sizeof(float2) + static_cast<size_t>(nc) * sizeof(float);
}

template <int LOG2L>
void launch_log2(const FilterArgs &a, int num_sms, cudaStream_t s)
{
    constexpr int L = 1 << LOG2L;
    constexpr int NT = (L / 4 < 256) ? L / 4 : 256;
    const size_t smem = smem_bytes_log2<LOG2L>(a.nc);
    // segments of about 64 rows (one extra filtered row each); shorter segments when views are few
    int seg_rows = 64;
    while (seg_rows > 2 && static_cast<long long>(a.nv) * ((a.nr + seg_rows - 1) / seg_rows) < 4LL * num_sms)
        seg_rows /= 2;
    if (seg_rows > a.nr) seg_rows = a.nr;
    const int nseg = (a.nr + seg_rows - 1) / seg_rows;
    long long grid = static_cast<long long>(a.nv) * nseg;
    const long long cap = static_cast<long long>(num_sms) * 64;
    if (grid > cap) grid = cap;
    auto go = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        kern<<<static_cast<unsigned>(grid), NT, smem, s>>>(a, seg_rows, nseg);
    };
    switch (a.mode) {
        case kOutPlainF32: go(filter_fft_kernel<LOG2L, kOutPlainF32>); break;
        case kOutQuadF32: go(filter_fft_kernel<LOG2L, kOutQuadF32>); break;
        default: go(filter_fft_kernel<LOG2L, kOutQuadF16>); break;
    }
}

__global__ void view_absmax_kernel(const float *__restrict__ proj, long long pix_per_view,
                                   float *amax)
{
    const int v = blockIdx.y;
    const float *p = proj + static_cast<long long>(v) * pix_per_view;
    float m = 0.f;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < pix_per_view;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        m = fmaxf(m, fabsf(__ldg(p + i)));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(amax + v), __float_as_int(m));
}

__global__ void view_scales_kernel(const float *amax, int nv, float l1, float *vscale, float *vinv)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    // quad coefficients are sums and differences of up to four filtered values: keep 4 * bound
    // below 2^14 so FP16 never overflows
    const float bound = 4.0f * amax[v] * l1;
    float e = 0.f;
    if (bound > 0.f && isfinite(bound)) e = fminf(fmaxf(floorf(log2f(16384.f / bound)), -100.f), 100.f);
    vscale[v] = exp2f(e);
    vinv[v] = exp2f(-e);
}

}  // namespace

size_t filter_fft_smem_bytes(int L, int nc)
{
    switch (L) {
        case 64: return smem_bytes_log2<6>(nc);
        case 128: return smem_bytes_log2<7>(nc);
        case 256: return smem_bytes_log2<8>(nc);
        case 512: return smem_bytes_log2<9>(nc);
        case 1024: return smem_bytes_log2<10>(nc);
        case 2048: return smem_bytes_log2<11>(nc);
        case 4096: return smem_bytes_log2<12>(nc);
        default: return smem_bytes_log2<13>(nc);
    }
}

void launch_filter_fft(const FilterArgs &a, int L, int num_sms, cudaStream_t s)
{
    switch (L) {
        case 64: launch_log2<6>(a, num_sms, s); break;
        case 128: launch_log2<7>(a, num_sms, s); break;
        case 256: launch_log2<8>(a, num_sms, s); break;
        case 512: launch_log2<9>(a, num_sms, s); break;
        case 1024: launch_log2<10>(a, num_sms, s); break;
        case 2048: launch_log2<11>(a, num_sms, s); break;
        case 4096: launch_log2<12>(a, num_sms, s); break;
        case 8192: launch_log2<13>(a, num_sms, s); break;
        default: break;  // rejected on the host
    }
}

void launch_view_absmax(const float *proj, int nv, long long pix_per_view, float *amax,
                        cudaStream_t s)
{
    long long bx = (pix_per_view + 256 * 8 - 1) / (256 * 8);
    if (bx > 64) bx = 64;
    if (bx < 1) bx = 1;
    view_absmax_kernel<<<dim3(static_cast<unsigned>(bx), nv), 256, 0, s>>>(proj, pix_per_view, amax);
}

void launch_view_scales(const float *amax, int nv, float l1, float *vscale, float *vinv,
                        cudaStream_t s)
{
    view_scales_kernel<<<(nv + 127) / 128, 128, 0, s>>>(amax, nv, l1, vscale, vinv);
}

}  // namespace gct
