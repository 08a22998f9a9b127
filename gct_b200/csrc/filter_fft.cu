// Row-batched ramp filter: cosine and Parker weights fused into the load, zero padding in
// shared memory, a Stockham radix-4/2 FFT convolution with the ramp spectrum, and an epilogue
// that writes either plain FP32 rows or the padded bilinear-quad layout used by the
// backprojector. Two detector rows share one complex FFT (row a in the real part, row b in
// the imaginary part): the ramp taps are real, so the two convolutions stay separated.
//
// Replaces runCosWeighting (src/cuda/recon/cos_weighting.cuh:225-263), runParkerWeighting
// (src/cuda/recon/parker_weighting.cuh:202-230) and RampFilteringFFT::runFiltering
// (src/cuda/recon/ramp_filtering_fft.cuh:208-219): the reference pads to nextPow2(2N), runs
// cuFFT R2C/C2R and crops at N/2; here the taps are placed circularly so the crop disappears and
// the shortest alias-free power of two (> 1.5 N) is used.
#include "../../include/gct_fdk.h"
#include "common.cuh"
#include "kernels.hpp"

namespace gct {
namespace {

// Cosine pre-weight of pixel (c, r) of a view, per geometry (src/cuda/recon/cos_weighting.cuh:
// 16-153). c0/r0 are the view's detector centres, du/dv the sampler widths.
__device__ __forceinline__ float cos_weight(int kind, float c0, float r0, float sdd, float du,
                                            float dv, int c, int r)
{
    switch (kind) {
        case GCT_GEOM_FAN_ARC: return cosf((static_cast<float>(c) - c0) * du);
        case GCT_GEOM_FAN_LINE: {
            const float u = (static_cast<float>(c) - c0) * du;
            return sdd * rsqrtf(u * u + sdd * sdd);
        }
        case GCT_GEOM_CONE_PARALLEL: {
            const float v = (static_cast<float>(r) - r0) * dv;
            return sdd * rsqrtf(v * v + sdd * sdd);
        }
        case GCT_GEOM_CONE_CYL: {
            const float g = (static_cast<float>(c) - c0) * du;
            const float v = (static_cast<float>(r) - r0) * dv;
            return cosf(g) * sdd * rsqrtf(v * v + sdd * sdd);
        }
        case GCT_GEOM_CONE_FLAT: {
            const float u = (static_cast<float>(c) - c0) * du;
            const float v = (static_cast<float>(r) - r0) * dv;
            return sdd * rsqrtf(u * u + v * v + sdd * sdd);
        }
        default: return 1.0f;  // parallel kinds
    }
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// One Stockham stage of radix R (4 or 2) with span Ns (Govindaraju et al., SC'08): butterfly j
// reads src[j + r L/R], applies the twiddle W_L^(r (j mod Ns) L/(Ns R)), and writes the R-point
// DFT to dst[(j / Ns) Ns R + (j mod Ns) + r Ns]. The output after all stages is in natural order.
template <int L, int NT>
__device__ __forceinline__ void stage_r4(const float2 *__restrict__ src, float2 *__restrict__ dst,
                                         const float2 *__restrict__ tw, int Ns, int tid)
{
#pragma unroll
    for (int j = tid; j < L / 4; j += NT) {
        const int k = j & (Ns - 1);
        float2 v0 = src[j], v1 = src[j + L / 4], v2 = src[j + L / 2], v3 = src[j + 3 * L / 4];
        if (Ns > 1) {
            const int step = k * (L / (4 * Ns));
            v1 = cmul(v1, tw[step]);
            v2 = cmul(v2, tw[2 * step]);
            v3 = cmul(v3, tw[3 * step]);
        }
        const float2 t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3);
        const float2 d = csub(v1, v3);
        const float2 t3 = make_float2(d.y, -d.x);  // -i * (v1 - v3)
        const int idx = (j - k) * 4 + k;
        dst[idx] = cadd(t0, t2);
        dst[idx + Ns] = cadd(t1, t3);
        dst[idx + 2 * Ns] = csub(t0, t2);
        dst[idx + 3 * Ns] = csub(t1, t3);
    }
}

template <int L, int NT>
__device__ __forceinline__ void stage_r2(const float2 *__restrict__ src, float2 *__restrict__ dst,
                                         const float2 *__restrict__ tw, int Ns, int tid)
{
#pragma unroll
    for (int j = tid; j < L / 2; j += NT) {
        const int k = j & (Ns - 1);
        float2 v0 = src[j], v1 = src[j + L / 2];
        if (Ns > 1) v1 = cmul(v1, tw[k * (L / (2 * Ns))]);
        const int idx = (j - k) * 2 + k;
        dst[idx] = cadd(v0, v1);
        dst[idx + Ns] = csub(v0, v1);
    }
}

// Forward FFT of L points from `a`; ping-pongs between a and b, returns the result buffer.
template <int LOG2L, int NT>
__device__ __forceinline__ float2 *fft(float2 *a, float2 *b, const float2 *tw, int tid)
{
    constexpr int L = 1 << LOG2L;
    float2 *src = a, *dst = b;
    int Ns = 1;
#pragma unroll
    for (int s = 0; s < LOG2L / 2; ++s) {
        stage_r4<L, NT>(src, dst, tw, Ns, tid);
        __syncthreads();
        float2 *t = src;
        src = dst;
        dst = t;
        Ns *= 4;
    }
    if (LOG2L & 1) {
        stage_r2<L, NT>(src, dst, tw, Ns, tid);
        __syncthreads();
        float2 *t = src;
        src = dst;
        dst = t;
    }
    return src;
}

template <int MODE>
__device__ __forceinline__ void store_row(const FilterArgs &a, long long row, const float2 *res,
                                          bool imag, int tid, int nthreads)
{
    const int nc = a.nc;
    if (MODE == kOutPlainF32) {
        float *out = static_cast<float *>(a.out) + row * nc;
        for (int c = tid; c < nc; c += nthreads) out[c] = imag ? -res[c].y : res[c].x;
        return;
    }
    const int v = static_cast<int>(row / a.nr);
    const int r = static_cast<int>(row - static_cast<long long>(v) * a.nr);
    const float sc = a.vscale ? a.vscale[v] : 1.0f;
    const int qpitch = nc + 2 * kQuadPad;
    const long long qview = static_cast<long long>(a.nr + 2 * kQuadPad) * qpitch;
    auto val = [&](int c) -> float {
        if (c < 0 || c >= nc) return 0.0f;
        return sc * (imag ? -res[c].y : res[c].x);
    };
    for (int cq = tid; cq < qpitch; cq += nthreads) {
        const int c = cq - kQuadPad;
        const float lo = val(c), hi = val(c + 1);
        const long long own = static_cast<long long>(v) * qview + static_cast<long long>(r + kQuadPad) * qpitch + cq;
        const long long prv = own - qpitch;
        if (MODE == kOutQuadF32) {
            float2 *q = reinterpret_cast<float2 *>(static_cast<float4 *>(a.out));
            const float2 pair = make_float2(lo, hi);
            const float2 zero = make_float2(0.f, 0.f);
            q[2 * own] = pair;          // own row: .xy
            q[2 * prv + 1] = pair;      // previous row: .zw
            if (r == 0) {
                q[2 * (prv - qpitch)] = zero;
                q[2 * (prv - qpitch) + 1] = zero;
                q[2 * prv] = zero;
            }
            if (r == a.nr - 1) {
                q[2 * own + 1] = zero;
                q[2 * (own + qpitch)] = zero;
                q[2 * (own + qpitch) + 1] = zero;
                q[2 * (own + 2 * qpitch)] = zero;
                q[2 * (own + 2 * qpitch) + 1] = zero;
            }
        } else {
            __half2 *q = reinterpret_cast<__half2 *>(static_cast<uint2 *>(a.out));
            const __half2 pair = __floats2half2_rn(lo, hi);
            const __half2 zero = __floats2half2_rn(0.f, 0.f);
            q[2 * own] = pair;
            q[2 * prv + 1] = pair;
            if (r == 0) {
                q[2 * (prv - qpitch)] = zero;
                q[2 * (prv - qpitch) + 1] = zero;
                q[2 * prv] = zero;
            }
            if (r == a.nr - 1) {
                q[2 * own + 1] = zero;
                q[2 * (own + qpitch)] = zero;
                q[2 * (own + qpitch) + 1] = zero;
                q[2 * (own + 2 * qpitch)] = zero;
                q[2 * (own + 2 * qpitch) + 1] = zero;
            }
        }
    }
}

template <int LOG2L, int MODE>
__global__ void __launch_bounds__(256) filter_fft_kernel(FilterArgs a)
{
    constexpr int L = 1 << LOG2L;
    constexpr int NT = (L / 4 < 256) ? L / 4 : 256;
    extern __shared__ float2 smem[];
    float2 *tw = smem, *b0 = smem + L, *b1 = smem + 2 * L;
    const int tid = threadIdx.x;
    for (int m = tid; m < L; m += NT) tw[m] = a.twiddle[m];

    const long long nrows = static_cast<long long>(a.nv) * a.nr;
    const long long npairs = (nrows + 1) / 2;
    const int nc = a.nc;
    for (long long p = blockIdx.x; p < npairs; p += gridDim.x) {
        const long long ra = 2 * p, rb = 2 * p + 1;
        const bool has_b = rb < nrows;
        const int va = static_cast<int>(ra / a.nr), r_a = static_cast<int>(ra - static_cast<long long>(va) * a.nr);
        const int vb = has_b ? static_cast<int>(rb / a.nr) : va;
        const int r_b = has_b ? static_cast<int>(rb - static_cast<long long>(vb) * a.nr) : 0;
        const float4 ga = __ldg(&a.fview[va]), gb = __ldg(&a.fview[vb]);
        const float *pa = a.proj + ra * nc, *pb = a.proj + rb * nc;
        const float *wa = a.parker + static_cast<long long>(va) * nc;
        const float *wb = a.parker + static_cast<long long>(vb) * nc;
        for (int k = tid; k < L; k += NT) {
            float2 z = make_float2(0.f, 0.f);
            if (k < nc) {
                z.x = __ldg(pa + k) * __ldg(wa + k) *
                      cos_weight(a.kind, ga.x, ga.y, ga.z, a.du, a.dv, k, r_a);
                if (has_b)
                    z.y = __ldg(pb + k) * __ldg(wb + k) *
                          cos_weight(a.kind, gb.x, gb.y, gb.z, a.du, a.dv, k, r_b);
            }
            b0[k] = z;
        }
        __syncthreads();
        float2 *res = fft<LOG2L, NT>(b0, b1, tw, tid);
        for (int k = tid; k < L; k += NT) {
            const float2 y = cmul(res[k], __ldg(&a.H[k]));
            res[k] = make_float2(y.x, -y.y);  // conj: the second forward FFT acts as the inverse
        }
        __syncthreads();
        float2 *other = (res == b0) ? b1 : b0;
        float2 *out = fft<LOG2L, NT>(res, other, tw, tid);
        // out holds conj(IFFT): row a in .x, row b in -.y
        store_row<MODE>(a, ra, out, false, tid, NT);
        if (has_b) store_row<MODE>(a, rb, out, true, tid, NT);
        __syncthreads();
    }
}

template <int LOG2L>
void launch_log2(const FilterArgs &a, int num_sms, cudaStream_t s)
{
    constexpr int L = 1 << LOG2L;
    constexpr int NT = (L / 4 < 256) ? L / 4 : 256;
    const size_t smem = 3ull * L * sizeof(float2);
    const long long npairs = (static_cast<long long>(a.nv) * a.nr + 1) / 2;
    const int per_sm = static_cast<int>((227 * 1024) / (smem + 1024));
    long long grid = static_cast<long long>(num_sms) * (per_sm > 0 ? per_sm : 1) * 4;
    if (grid > npairs) grid = npairs;
    if (grid < 1) grid = 1;
    switch (a.mode) {
        case kOutPlainF32:
            cudaFuncSetAttribute(filter_fft_kernel<LOG2L, kOutPlainF32>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
            filter_fft_kernel<LOG2L, kOutPlainF32><<<static_cast<unsigned>(grid), NT, smem, s>>>(a);
            break;
        case kOutQuadF32:
            cudaFuncSetAttribute(filter_fft_kernel<LOG2L, kOutQuadF32>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
            filter_fft_kernel<LOG2L, kOutQuadF32><<<static_cast<unsigned>(grid), NT, smem, s>>>(a);
            break;
        default:
            cudaFuncSetAttribute(filter_fft_kernel<LOG2L, kOutQuadF16>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
            filter_fft_kernel<LOG2L, kOutQuadF16><<<static_cast<unsigned>(grid), NT, smem, s>>>(a);
            break;
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
    const float bound = amax[v] * l1;
    float e = 0.f;
    if (bound > 0.f && isfinite(bound)) e = fminf(fmaxf(floorf(log2f(16384.f / bound)), -100.f), 100.f);
    vscale[v] = exp2f(e);
    vinv[v] = exp2f(-e);
}

}  // namespace

size_t filter_fft_smem_bytes(int L) { return 3ull * L * sizeof(float2); }

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
