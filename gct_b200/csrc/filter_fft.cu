// Row-batched ramp filter: cosine and Parker weights fused into the load, an FFT convolution with
// the ramp spectrum done in registers with radix-16 passes, and an epilogue that writes either
// plain FP32 rows or the padded bilinear-coefficient quads read by the backprojector. Two detector
// rows share one complex FFT (row a in the real part, row b in the imaginary part): the ramp taps
// are real, so the two convolutions stay separated.
//
// Replaces runCosWeighting (src/cuda/recon/cos_weighting.cuh:225-263), runParkerWeighting
// (src/cuda/recon/parker_weighting.cuh:202-230) and RampFilteringFFT::runFiltering
// (src/cuda/recon/ramp_filtering_fft.cuh:208-219): the reference pads to nextPow2(2N), runs
// cuFFT R2C/C2R and crops at N/2 in five passes over HBM; here the taps are placed circularly so
// the crop disappears, the shortest alias-free power of two (> 1.5 N) is used, and each row is
// read once and written once.
//
// Transform of length L = 2^LOG2L by T = L / 16 threads, 16 points per thread. Thread t holds
// x[t + T m], m = 0..15, in registers. The transform is a Stockham decomposition into passes of
// radix 16 (the last one radix 2^(LOG2L mod 4), or 16): a pass of radix R and span Ns takes, for
// butterfly j, the inputs x[j + r L / R] (r < R), multiplies input r by W_{R Ns}^{r (j mod Ns)} and
// writes its R-point DFT to y[(j - j mod Ns) R + (j mod Ns) + k Ns]. Each pass's butterflies run
// in one thread's registers; passes exchange through one shared-memory buffer (padded by one
// float2 per 16 so the strided accesses are bank-conflict free). The last pass leaves thread t
// with X[t + T m] in natural order, which is exactly the input set of the first pass of the next
// transform: the spectrum product and the inverse transform (a forward transform of the
// conjugate) follow without an exchange. Per row pair: four exchanges, no twiddle tables (each
// pass's twiddles are powers of one per-thread base computed at start).
//
// Work split: one CTA per (view, segment of quad rows) (or, for one-row detectors, per pair of
// views). A CTA walks its rows in pairs, keeps the filtered rows of the previous pair in shared
// memory and writes each quad row whole once its two detector rows are known.
#include <cstdint>

#include "../../include/gct_fdk.h"
#include "common.cuh"
#include "kernels.hpp"

namespace gct {
namespace {

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }  // times -i

// Shared-memory index with one float2 of padding per 16 entries.
__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }

// x times W_16^M = exp(-2 pi i M / 16) for a compile-time M (the exact constants cos(pi/8),
// sin(pi/8) and sqrt(1/2); multiples of a quarter turn are swaps and negations).
template <int M>
__device__ __forceinline__ float2 tw16(float2 x)
{
    constexpr int m = ((M % 16) + 16) % 16;
    constexpr float c1 = 0.923879532511286756f, s1 = 0.382683432365089772f, h = 0.707106781186547524f;
    if constexpr (m == 0) return x;
    else if constexpr (m == 4) return mul_mi(x);
    else if constexpr (m == 8) return make_float2(-x.x, -x.y);
    else if constexpr (m == 12) return make_float2(-x.y, x.x);
    else if constexpr (m == 2) return make_float2(h * (x.x + x.y), h * (x.y - x.x));
    else if constexpr (m == 6) return make_float2(h * (x.y - x.x), -h * (x.x + x.y));
    else if constexpr (m == 10) return make_float2(-h * (x.x + x.y), h * (x.x - x.y));
    else if constexpr (m == 14) return make_float2(h * (x.x - x.y), h * (x.x + x.y));
    else {
        // W = cos(2 pi m / 16) - i sin(2 pi m / 16)
        constexpr float cs = (m == 1 || m == 15) ? c1 : (m == 3 || m == 13) ? s1 : (m == 5 || m == 11) ? -s1 : -c1;
        constexpr float sn = (m == 1 || m == 7) ? s1 : (m == 3 || m == 5) ? c1 : (m == 9 || m == 15) ? -s1 : -c1;
        return make_float2(fmaf(x.x, cs, x.y * sn), fmaf(x.y, cs, -x.x * sn));
    }
}

// In-place DFTs with natural-order output.
__device__ __forceinline__ void dft2(float2 *x)
{
    const float2 a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
}

__device__ __forceinline__ void dft4v(float2 a0, float2 a1, float2 a2, float2 a3, float2 &y0, float2 &y1, float2 &y2,
                                      float2 &y3)
{
    const float2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = mul_mi(csub(a1, a3));
    y0 = cadd(t0, t2);
    y1 = cadd(t1, t3);
    y2 = csub(t0, t2);
    y3 = csub(t1, t3);
}

__device__ __forceinline__ void dft4(float2 *x) { dft4v(x[0], x[1], x[2], x[3], x[0], x[1], x[2], x[3]); }

// 8 = 4 x 2: inner DFT4 over x[2 n1 + n2], twiddle W_8^(n2 k1), outer DFT2.
__device__ __forceinline__ void dft8(float2 *x)
{
    float2 a0, a1, a2, a3, b0, b1, b2, b3;
    dft4v(x[0], x[2], x[4], x[6], a0, a1, a2, a3);
    dft4v(x[1], x[3], x[5], x[7], b0, b1, b2, b3);
    b1 = tw16<2>(b1);
    b2 = tw16<4>(b2);
    b3 = tw16<6>(b3);
    x[0] = cadd(a0, b0);
    x[4] = csub(a0, b0);
    x[1] = cadd(a1, b1);
    x[5] = csub(a1, b1);
    x[2] = cadd(a2, b2);
    x[6] = csub(a2, b2);
    x[3] = cadd(a3, b3);
    x[7] = csub(a3, b3);
}

// 16 = 4 x 4: inner DFT4 over x[4 n1 + n2], twiddle W_16^(n2 k1), outer DFT4 over n2.
__device__ __forceinline__ void dft16(float2 *x)
{
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) dft4v(x[n2], x[4 + n2], x[8 + n2], x[12 + n2], x[n2], x[4 + n2], x[8 + n2], x[12 + n2]);
    // x[n2 + 4 k1] now holds inner output k1 of column n2
    x[5] = tw16<1>(x[5]);
    x[9] = tw16<2>(x[9]);
    x[13] = tw16<3>(x[13]);
    x[6] = tw16<2>(x[6]);
    x[10] = tw16<4>(x[10]);
    x[14] = tw16<6>(x[14]);
    x[7] = tw16<3>(x[7]);
    x[11] = tw16<6>(x[11]);
    x[15] = tw16<9>(x[15]);
    float2 y[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
        dft4v(x[4 * k1], x[4 * k1 + 1], x[4 * k1 + 2], x[4 * k1 + 3], y[k1], y[k1 + 4], y[k1 + 8], y[k1 + 12]);
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = y[k];
}

// DFT16 of x whose entries 8..15 are zero: X[2k] = DFT8(x)[k], X[2k + 1] = DFT8(x[n] W_16^n)[k].
__device__ __forceinline__ void dft16_half(float2 *x)
{
    float2 e[8], o[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) e[n] = x[n];
    o[0] = x[0];
    o[1] = tw16<1>(x[1]);
    o[2] = tw16<2>(x[2]);
    o[3] = tw16<3>(x[3]);
    o[4] = tw16<4>(x[4]);
    o[5] = tw16<5>(x[5]);
    o[6] = tw16<6>(x[6]);
    o[7] = tw16<7>(x[7]);
    dft8(e);
    dft8(o);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        x[2 * k] = e[k];
        x[2 * k + 1] = o[k];
    }
}

template <int R>
__device__ __forceinline__ void dft(float2 *x)
{
    if constexpr (R == 16) dft16(x);
    else if constexpr (R == 8) dft8(x);
    else if constexpr (R == 4) dft4(x);
    else dft2(x);
}

// x[r] *= w^r, r = 1..R-1 (powers by squaring and products: at most five roundings deep).
template <int R>
__device__ __forceinline__ void twiddle(float2 *x, float2 w)
{
    if constexpr (R >= 2) x[1] = cmul(x[1], w);
    if constexpr (R >= 4) {
        const float2 w2 = cmul(w, w), w3 = cmul(w2, w);
        x[2] = cmul(x[2], w2);
        x[3] = cmul(x[3], w3);
        if constexpr (R >= 8) {
            const float2 w4 = cmul(w2, w2), w5 = cmul(w4, w), w6 = cmul(w4, w2), w7 = cmul(w4, w3);
            x[4] = cmul(x[4], w4);
            x[5] = cmul(x[5], w5);
            x[6] = cmul(x[6], w6);
            x[7] = cmul(x[7], w7);
            if constexpr (R >= 16) {
                const float2 w8 = cmul(w4, w4);
                x[8] = cmul(x[8], w8);
                x[9] = cmul(x[9], cmul(w8, w));
                x[10] = cmul(x[10], cmul(w8, w2));
                x[11] = cmul(x[11], cmul(w8, w3));
                x[12] = cmul(x[12], cmul(w8, w4));
                x[13] = cmul(x[13], cmul(w8, w5));
                x[14] = cmul(x[14], cmul(w8, w6));
                x[15] = cmul(x[15], cmul(w8, w7));
            }
        }
    }
}

// Pass structure of a transform of length 2^LOG2L.
template <int LOG2L>
struct Fft {
    static constexpr int L = 1 << LOG2L;
    static constexpr int T = L / 16;                  // threads per transform
    static constexpr int NPASS = (LOG2L + 3) / 4;
    static constexpr int RLAST = 1 << (LOG2L - 4 * (NPASS - 1));
    static constexpr int LP = L + L / 16;             // padded exchange buffer (float2)
    static constexpr int radix(int p) { return p < NPASS - 1 ? 16 : RLAST; }
    static constexpr int span(int p) { return 1 << (4 * p); }
};

// Per-thread twiddle bases: pass p >= 1 multiplies input r of butterfly 0 by base_p^r with
// base_p = W_{R Ns}^(t mod Ns); butterfly i of a last pass with several butterflies per thread
// uses base_p W_16^i (its j = t + i T is below Ns there).
template <int LOG2L>
struct Bases {
    float2 w[Fft<LOG2L>::NPASS];
    __device__ __forceinline__ void init(int t)
    {
        using F = Fft<LOG2L>;
        w[0] = make_float2(1.f, 0.f);
#pragma unroll
        for (int p = 1; p < F::NPASS; ++p) {
            const int ns = F::span(p), rn = F::radix(p) * ns;
            float s, c;
            // exp(-2 pi i k / (R Ns)) = cos - i sin of pi (2 k / (R Ns)); 2 k / (R Ns) is exact
            sincospif(2.0f * static_cast<float>(t & (ns - 1)) / static_cast<float>(rn), &s, &c);
            w[p] = make_float2(c, -s);
        }
    }
};

// Twiddles and DFT of butterflies I.. of pass P, whose inputs are in x (butterfly-major).
template <int LOG2L, int P, int I>
__device__ __forceinline__ void butterflies(float2 (&x)[16], float2 base)
{
    constexpr int R = Fft<LOG2L>::radix(P);
    twiddle<R>(x + I * R, tw16<I>(base));  // butterfly I's base: base W_16^I
    dft<R>(x + I * R);
    if constexpr (I + 1 < 16 / R) butterflies<LOG2L, P, I + 1>(x, base);
}

// One pass p >= 1: read inputs from the exchange buffer, twiddle, DFT. x is butterfly-major:
// x[i R + r] = input r of butterfly i, then output k at x[i R + k].
template <int LOG2L, int P>
__device__ __forceinline__ void pass_in(const float2 *buf, float2 (&x)[16], int t, float2 base)
{
    using F = Fft<LOG2L>;
    constexpr int R = F::radix(P), B = 16 / R, L = F::L, T = F::T;
#pragma unroll
    for (int i = 0; i < B; ++i)
#pragma unroll
        for (int r = 0; r < R; ++r) x[i * R + r] = buf[pad(t + i * T + r * (L / R))];
    butterflies<LOG2L, P, 0>(x, base);
}

// Writes the outputs of pass p (not the last) to the exchange buffer at their Stockham places.
template <int LOG2L, int P>
__device__ __forceinline__ void pass_out(float2 *buf, const float2 (&x)[16], int t)
{
    using F = Fft<LOG2L>;
    constexpr int R = F::radix(P), B = 16 / R, T = F::T, NS = F::span(P);
#pragma unroll
    for (int i = 0; i < B; ++i) {
        const int j = t + i * T;
        const int kk = j & (NS - 1);
        const int o = (j - kk) * R + kk;
#pragma unroll
        for (int k = 0; k < R; ++k) buf[pad(o + k * NS)] = x[i * R + k];
    }
}

// Natural order after the last pass: butterfly i's output k is X[t + T (i + k B)].
template <int LOG2L>
__device__ __forceinline__ void last_to_natural(float2 (&x)[16])
{
    constexpr int R = Fft<LOG2L>::RLAST, B = 16 / R;
    if constexpr (B > 1) {
        float2 y[16];
#pragma unroll
        for (int i = 0; i < B; ++i)
#pragma unroll
            for (int k = 0; k < R; ++k) y[i + k * B] = x[i * R + k];
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = y[m];
    }
}

// Full transform of x (natural order in: x[m] = v[t + T m]; natural order out). The first pass
// runs on the registers; HALF: x[8..15] are zero on entry.
template <int LOG2L, bool HALF>
__device__ __forceinline__ void transform(float2 (&x)[16], float2 *buf, int t, const Bases<LOG2L> &bs)
{
    using F = Fft<LOG2L>;
    static_assert(F::NPASS >= 2, "transforms of at least 64 points");
    if constexpr (HALF) dft16_half(x);
    else dft16(x);
    pass_out<LOG2L, 0>(buf, x, t);
    __syncthreads();
    pass_in<LOG2L, 1>(buf, x, t, bs.w[1]);
    if constexpr (F::NPASS > 2) {
        __syncthreads();
        pass_out<LOG2L, 1>(buf, x, t);
        __syncthreads();
        pass_in<LOG2L, 2>(buf, x, t, bs.w[2]);
    }
    if constexpr (F::NPASS > 3) {
        __syncthreads();
        pass_out<LOG2L, 2>(buf, x, t);
        __syncthreads();
        pass_in<LOG2L, 3>(buf, x, t, bs.w[3]);
    }
    __syncthreads();  // every thread is done reading the buffer before the next transform writes it
    last_to_natural<LOG2L>(x);
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

// Quad row qr (detector rows qr and qr + 1) of view v (stack index) from two shared rows stored
// with two zero entries before column 0 and a zero tail (row[c + 2] = y[c]); NULL = zero row.
template <int MODE>
__device__ __forceinline__ void write_quad_row(const FilterArgs &a, int v, int qr, const float *top, const float *bot,
                                               int t, int nthr)
{
    const int qpitch = a.nc + 2 * kQuadPad;
    long long first;
    int step;
    quad_layout(v, static_cast<long long>(a.nr + 2 * kQuadPad) * qpitch, a.quarter, first, step);
    const long long row0 = first + static_cast<long long>(qr + kQuadPad) * qpitch * step;
    for (int cq = t; cq < qpitch; cq += nthr) {
        const float p00 = top ? top[cq] : 0.f, p01 = top ? top[cq + 1] : 0.f;
        const float p10 = bot ? bot[cq] : 0.f, p11 = bot ? bot[cq + 1] : 0.f;
        store_quad<MODE>(a.out, row0 + static_cast<long long>(cq) * step, p00, p01, p10, p11);
    }
}

// Transposed quad grid of view v of a one-row detector from its filtered row y (shared, padded
// as above).
template <int MODE>
__device__ __forceinline__ void write_quads_t1d(const FilterArgs &a, int v, const float *y, int t, int nthr)
{
    const int nc = a.nc, rows = nc + 2 * kQuadPad;
    const long long base = static_cast<long long>(v) * rows * kT1dPitch;
    for (int e = t; e < rows * kT1dPitch; e += nthr) {
        const int r = e / kT1dPitch, c = e % kT1dPitch - kQuadPad;  // y[r - 2] is shared entry r
        const float tp = y[r], bt = y[r + 1];
        if (c == 0)
            store_quad<MODE>(a.out, base + e, tp, 0.0f, bt, 0.0f);
        else if (c == -1)
            store_quad<MODE>(a.out, base + e, 0.0f, tp, 0.0f, bt);
        else
            store_quad<MODE>(a.out, base + e, 0.0f, 0.0f, 0.0f, 0.0f);
    }
}

// Loads, weights and packs detector rows a (real part) and b (imaginary part) at columns t + T m;
// NULL rows are zero. Columns at or past nc are zero. SMEM: the rows are in shared memory (plain
// loads), else in global memory (read-only loads through the non-coherent path, which accepts
// global addresses only). The Parker rows ka, kb are always global.
template <int LOG2L, bool HALF, bool SMEM>
__device__ __forceinline__ void load_pair(const FilterArgs &a, float2 (&x)[16], const float *pa, const float *pb,
                                          const RowWeight &wa, const RowWeight &wb, const float *ka, const float *kb,
                                          int t)
{
    constexpr int T = Fft<LOG2L>::T;
    constexpr int MZ = HALF ? 8 : 11;  // nc <= L / 1.5 < 11 T
#pragma unroll
    for (int m = 0; m < 16; ++m) x[m] = make_float2(0.f, 0.f);
#pragma unroll
    for (int m = 0; m < MZ; ++m) {
        const int c = t + T * m;
        if (c < a.nc) {
            const float k = __ldg(ka + c);
            if (pa) x[m].x = (SMEM ? pa[c] : __ldg(pa + c)) * (wa.at(c) * k);
            if (pb) x[m].y = (SMEM ? pb[c] : __ldg(pb + c)) * (wb.at(c) * (kb == ka ? k : __ldg(kb + c)));
        }
    }
}

// Spectrum product and the conjugation that turns the next forward transform into the inverse:
// x <- conj(x H), H already scaled by 1 / L.
template <int LOG2L>
__device__ __forceinline__ void spectrum(float2 (&x)[16], const float2 *__restrict__ H, int t)
{
    constexpr int T = Fft<LOG2L>::T;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const float2 h = __ldg(H + t + T * m);
        const float2 z = cmul(x[m], h);
        x[m] = make_float2(z.x, -z.y);
    }
}

// Filters the detector rows pa (real part) and pb (imaginary part) (NULL = zero row; in shared
// memory with SMEM, else global) of views va and vb, rows ra and rb (for the weights), and leaves the filtered rows
// in natural order: row a in x[m].x, row b in -x[m].y at columns t + T m.
template <int LOG2L, bool HALF, bool SMEM>
__device__ __forceinline__ void filter_pair(const FilterArgs &a, float2 (&x)[16], float2 *buf, int t,
                                            const Bases<LOG2L> &bs, const float *pa, const float *pb, int va, int ra,
                                            int vb, int rb)
{
    const int ua = pa ? va : 0, ub = pb ? vb : ua;
    const float4 ga = __ldg(&a.fview[ua]), gb = __ldg(&a.fview[ub]);
    const RowWeight wa = row_weight(a.kind, ga.x, ga.y, ga.z, a.du, a.dv, ra);
    const RowWeight wb = row_weight(a.kind, gb.x, gb.y, gb.z, a.du, a.dv, rb);
    const float *ka = a.parker + static_cast<long long>(ua) * a.nc;
    const float *kb = a.parker + static_cast<long long>(ub) * a.nc;
    load_pair<LOG2L, HALF, SMEM>(a, x, pa, pb, wa, wb, ka, kb, t);
    // forward and inverse transform share one copy of the code (the fully unrolled transform is
    // large enough that two copies miss in the instruction cache)
#pragma unroll 1
    for (int k = 0; k < 2; ++k) {
        transform<LOG2L, false>(x, buf, t, bs);
        if (k == 0) spectrum<LOG2L>(x, a.H, t);
    }
}

// Writes the filtered rows held in x into two shared rows (padded: row[c + 2] = y[c]), scaled.
template <int LOG2L>
__device__ __forceinline__ void stage_rows(const float2 (&x)[16], float *ya, float *yb, float sa, float sb, int nc,
                                           int t)
{
    constexpr int T = Fft<LOG2L>::T;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const int c = t + T * m;
        if (c < nc) {
            ya[c + 2] = sa * x[m].x;
            yb[c + 2] = -sb * x[m].y;
        }
    }
}

// Resident blocks per SM asked of the compiler (caps registers at 65536 / (T * MINB)).
template <int LOG2L>
constexpr int fft_min_blocks()
{
    return Fft<LOG2L>::T >= 512 ? 1 : Fft<LOG2L>::T >= 256 ? 2 : Fft<LOG2L>::T >= 128 ? 4 : 8;
}

// ---- input pipeline --------------------------------------------------------------------------
// With BULK, the two raw rows of the next pair are copied into a shared stage by the tensor memory
// accelerator (cp.async.bulk, one thread) while the current pair is transformed; two stages, one
// mbarrier each. Every wait is bounded (2 s of %globaltimer): on a timeout the CTA records
// kFftWaitTimeout in a.err, waits (bounded) for its copies still in flight and returns.
constexpr unsigned long long kFftWaitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity)
{
    const unsigned long long t0 = now_ns();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (now_ns() - t0 > kFftWaitNs) return false;
    }
}

// The CTA's sequence of row pairs: items blockIdx.x, blockIdx.x + gridDim.x, ...; within an item
// (two-row detectors) pairs (ra, ra + 1) from its first row in steps of two. One-row detectors:
// item i is the pair of views (2 i, 2 i + 1), row 0.
struct PairSeq {
    int nv, nr, seg, nseg;
    long long items;
    bool quads, one_row;
    __device__ __forceinline__ int first_row(long long it) const
    {
        const int s = static_cast<int>(it % nseg);
        return quads ? -kQuadPad + s * seg : s * seg;
    }
    // end of the item's rows: quads: quad rows below it, pairs while ra <= end; plain: ra < end
    __device__ __forceinline__ int row_end(long long it) const
    {
        const int r0 = first_row(it);
        return quads ? min(r0 + seg, nr + kQuadPad) : min(r0 + seg, nr);
    }
    __device__ __forceinline__ bool in_item(long long it, int ra) const
    {
        return quads ? ra <= row_end(it) : ra < row_end(it);
    }
    __device__ __forceinline__ bool next(long long &it, int &ra) const
    {
        ra += 2;
        if (!one_row && in_item(it, ra)) return true;
        it += gridDim.x;
        if (it >= items) return false;
        ra = one_row ? 0 : first_row(it);
        return true;
    }
};

// Rows of pair (it, ra): views and rows of parts a and b; a view of -1 is a zero row.
struct PairRows {
    int va, ra, vb, rb;
};
__device__ __forceinline__ PairRows pair_rows(const PairSeq &q, long long it, int ra)
{
    PairRows p;
    if (q.one_row) {
        p.va = static_cast<int>(2 * it);
        p.vb = (2 * it + 1 < q.nv) ? static_cast<int>(2 * it + 1) : -1;
        p.ra = p.rb = 0;
        return p;
    }
    const int v = static_cast<int>(it / q.nseg);
    p.ra = ra;
    p.rb = ra + 1;
    p.va = (ra >= 0 && ra < q.nr) ? v : -1;
    p.vb = (p.rb >= 0 && p.rb < q.nr && (q.quads || p.rb < q.row_end(it))) ? v : -1;
    return p;
}

template <int LOG2L, int MODE, bool HALF, bool ONE_ROW, bool BULK>
__global__ void __launch_bounds__(Fft<LOG2L>::T, fft_min_blocks<LOG2L>())
    filter_fft_kernel(FilterArgs a, int seg, int nseg)
{
    using F = Fft<LOG2L>;
    constexpr int T = F::T;
    constexpr bool quads = MODE != kOutPlainF32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // layout: 2 mbarriers | exchange buffer (LP float2) | 3 padded rows | BULK: 2 stages x 2 rows
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem_raw);
    float2 *buf = reinterpret_cast<float2 *>(smem_raw + 16);
    const int rpitch = (a.nc + 2 * kQuadPad + 4) & ~3;  // padded shared row: 2 zeros, nc values, zeros
    float *rows = reinterpret_cast<float *>(buf + F::LP);
    float *stage = rows + 3 * rpitch;                   // [2 stages][2 rows][nc] raw rows (BULK)
    const int t = threadIdx.x;
    Bases<LOG2L> bs;
    bs.init(t);
    for (int e = t; e < 3 * rpitch; e += T) rows[e] = 0.f;
    if (BULK && t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bars)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bars + 1)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    float2 x[16];

    const long long items = ONE_ROW ? (a.nv + 1) / 2 : static_cast<long long>(a.nv) * nseg;
    const PairSeq q{a.nv, a.nr, seg, nseg, items, quads, ONE_ROW};
    const long long pix = static_cast<long long>(a.nr) * a.nc;
    const uint32_t row_bytes = static_cast<uint32_t>(a.nc) * 4u;
    int n_issued = 0, n_used = 0;  // pairs whose rows were copied into stages, and consumed

    long long it = blockIdx.x;
    int ra = (ONE_ROW || it >= items) ? 0 : q.first_row(it);
    bool have = it < items;
    long long cur_item = -1;
    int prev = 0, sa = 1, sb = 2;  // shared row slots (quads): previous pair's row b, this pair's a and b
    while (have) {
        const PairRows pr = pair_rows(q, it, ra);
        const bool present = pr.va >= 0 || pr.vb >= 0;
        long long it_n = it;
        int ra_n = ra;
        const bool have_n = q.next(it_n, ra_n);
        if constexpr (BULK) {
            // thread 0 copies the rows of this pair (unless already in flight) and of the next one
            for (int k = 0; k < 2; ++k) {
                const PairRows pi = k == 0 ? pr : pair_rows(q, it_n, ra_n);
                if (k == 0 ? !(present && n_issued == n_used) : !(have_n && (pi.va >= 0 || pi.vb >= 0))) continue;
                if (t == 0) {
                    const int st = n_issued & 1;
                    const uint32_t bar = smem_addr(bars + st);
                    const uint32_t bytes = row_bytes * ((pi.va >= 0) + (pi.vb >= 0));
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                                 : "memory");
                    if (pi.va >= 0)
                        asm volatile(
                            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                            ::"r"(smem_addr(stage + (2 * st) * a.nc)),
                            "l"(a.proj + pi.va * pix + static_cast<long long>(pi.ra) * a.nc), "r"(row_bytes), "r"(bar)
                            : "memory");
                    if (pi.vb >= 0)
                        asm volatile(
                            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                            ::"r"(smem_addr(stage + (2 * st + 1) * a.nc)),
                            "l"(a.proj + pi.vb * pix + static_cast<long long>(pi.rb) * a.nc), "r"(row_bytes), "r"(bar)
                            : "memory");
                }
                ++n_issued;
            }
        }
        if (it != cur_item) {
            cur_item = it;
            prev = 0, sa = 1, sb = 2;
        }
        if (present) {
            const float *pa = nullptr, *pb = nullptr;
            if constexpr (BULK) {
                const int st = n_used & 1;
                const bool ok = bar_wait(smem_addr(bars + st), (n_used >> 1) & 1);
                if (__syncthreads_or(!ok)) {
                    // the copies did not arrive: report, wait (bounded) for those still in flight, stop
                    if (t == 0) {
                        if (a.err) atomicOr(a.err, kFftWaitTimeout);
                        for (int k = n_used; k < n_issued; ++k) bar_wait(smem_addr(bars + (k & 1)), (k >> 1) & 1);
                    }
                    __syncthreads();
                    return;
                }
                if (pr.va >= 0) pa = stage + (2 * st) * a.nc;
                if (pr.vb >= 0) pb = stage + (2 * st + 1) * a.nc;
                ++n_used;
            } else {
                if (pr.va >= 0) pa = a.proj + pr.va * pix + static_cast<long long>(pr.ra) * a.nc;
                if (pr.vb >= 0) pb = a.proj + pr.vb * pix + static_cast<long long>(pr.rb) * a.nc;
            }
            filter_pair<LOG2L, HALF, BULK>(a, x, buf, t, bs, pa, pb, pr.va, pr.ra, pr.vb, pr.rb);  // holds barriers
        }
        if constexpr (!quads) {
            if (present) {
                float *out = static_cast<float *>(a.out);
#pragma unroll
                for (int m = 0; m < 16; ++m) {
                    const int c = t + T * m;
                    if (c < a.nc) {
                        if (pr.va >= 0) out[pr.va * pix + static_cast<long long>(pr.ra) * a.nc + c] = x[m].x;
                        if (pr.vb >= 0) out[pr.vb * pix + static_cast<long long>(pr.rb) * a.nc + c] = -x[m].y;
                    }
                }
            }
        } else if constexpr (ONE_ROW) {
            // each view's grid is written whole from its own row
            float *ya = rows, *yb = rows + rpitch;
            const float s_a = a.vscale ? a.vscale[pr.va] : 1.f, s_b = (a.vscale && pr.vb >= 0) ? a.vscale[pr.vb] : 1.f;
            stage_rows<LOG2L>(x, ya, yb, s_a, s_b, a.nc, t);
            __syncthreads();
            for (int h = 0; h < 2; ++h) {
                const int v = h ? pr.vb : pr.va;
                if (v < 0) continue;
                const float *y = h ? yb : ya;
                if (a.t1d) {
                    write_quads_t1d<MODE>(a, a.v0 + v, y, t, T);
                } else {
                    write_quad_row<MODE>(a, a.v0 + v, -2, nullptr, nullptr, t, T);
                    write_quad_row<MODE>(a, a.v0 + v, -1, nullptr, y, t, T);
                    write_quad_row<MODE>(a, a.v0 + v, 0, y, nullptr, t, T);
                    write_quad_row<MODE>(a, a.v0 + v, 1, nullptr, nullptr, t, T);
                    write_quad_row<MODE>(a, a.v0 + v, 2, nullptr, nullptr, t, T);
                }
            }
            __syncthreads();  // the shared rows are rewritten by the next pair
        } else {
            // quad rows [q0, q1) of view v: quad row r needs detector rows r and r + 1
            const int v = static_cast<int>(it / nseg);
            const int q0 = q.first_row(it), q1 = q.row_end(it);
            const float sc = a.vscale ? a.vscale[v] : 1.f;
            float *ya = rows + sa * rpitch, *yb = rows + sb * rpitch;
            if (present) {
                stage_rows<LOG2L>(x, ya, yb, sc, sc, a.nc, t);
            } else {
                __syncthreads();  // the previous pair's quad rows have been read from these slots
                for (int c = t; c < a.nc; c += T) ya[c + 2] = yb[c + 2] = 0.f;
            }
            __syncthreads();
            if (ra - 1 >= q0 && ra - 1 < q1) write_quad_row<MODE>(a, a.v0 + v, ra - 1, rows + prev * rpitch, ya, t, T);
            if (ra < q1) write_quad_row<MODE>(a, a.v0 + v, ra, ya, yb, t, T);
            // the next pair writes its rows into the slots of this pair's previous row and row a,
            // after the barriers of its transforms (or the one above)
            const int np = sb;
            sb = sa;
            sa = prev;
            prev = np;
        }
        it = it_n;
        ra = ra_n;
        have = have_n;
    }
}

// Shared memory of a CTA: two mbarriers, the exchange buffer, three padded rows and, with BULK,
// two stages of two raw rows.
template <int LOG2L>
size_t smem_bytes_log2(int nc, bool bulk)
{
    const int rpitch = (nc + 2 * kQuadPad + 4) & ~3;
    return 16 + static_cast<size_t>(Fft<LOG2L>::LP) * sizeof(float2) + 3 * static_cast<size_t>(rpitch) * sizeof(float) +
           (bulk ? 4 * static_cast<size_t>(nc) * sizeof(float) : 0);
}

template <int LOG2L, int MODE>
void launch_mode(const FilterArgs &a, int num_sms, cudaStream_t s)
{
    using F = Fft<LOG2L>;
    // rows are copied by the tensor memory accelerator when they start on 16-byte boundaries and
    // their length is a multiple of 16 bytes; otherwise each thread loads its columns directly
    const bool bulk = a.nc % 4 == 0 && reinterpret_cast<uintptr_t>(a.proj) % 16 == 0;
    const size_t smem = smem_bytes_log2<LOG2L>(a.nc, bulk);
    const bool half = a.nc <= F::L / 2;
    long long items;
    int seg = 0, nseg = 1;
    if (a.nr == 1) {
        items = (a.nv + 1) / 2;
    } else {
        // segments of about 64 rows (quad segments filter one extra pair to close their last quad
        // row); shorter segments when views are few; balanced lengths, even for quads
        const int rows = MODE == kOutPlainF32 ? a.nr : a.nr + 2 * kQuadPad;
        seg = 64;
        while (seg > 4 && static_cast<long long>(a.nv) * ((rows + seg - 1) / seg) < 8LL * num_sms) seg /= 2;
        nseg = (rows + seg - 1) / seg;
        seg = (rows + nseg - 1) / nseg;
        if (MODE != kOutPlainF32) seg = (seg + 1) & ~1;
        nseg = (rows + seg - 1) / seg;
        items = static_cast<long long>(a.nv) * nseg;
    }
    long long grid = items;
    const long long cap = static_cast<long long>(num_sms) * 32;
    if (grid > cap) grid = cap;
    if (grid < 1) grid = 1;
    auto go = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        kern<<<static_cast<unsigned>(grid), F::T, smem, s>>>(a, seg, nseg);
    };
    if (a.nr == 1) {
        if (!bulk) go(filter_fft_kernel<LOG2L, MODE, false, true, false>);
        else if (half) go(filter_fft_kernel<LOG2L, MODE, true, true, true>);
        else go(filter_fft_kernel<LOG2L, MODE, false, true, true>);
    } else {
        if (!bulk) go(filter_fft_kernel<LOG2L, MODE, false, false, false>);
        else if (half) go(filter_fft_kernel<LOG2L, MODE, true, false, true>);
        else go(filter_fft_kernel<LOG2L, MODE, false, false, true>);
    }
}

template <int LOG2L>
void launch_log2(const FilterArgs &a, int num_sms, cudaStream_t s)
{
    switch (a.mode) {
        case kOutPlainF32: launch_mode<LOG2L, kOutPlainF32>(a, num_sms, s); break;
        case kOutQuadF32: launch_mode<LOG2L, kOutQuadF32>(a, num_sms, s); break;
        default: launch_mode<LOG2L, kOutQuadF16>(a, num_sms, s); break;
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

void launch_filter_fft(const FilterArgs &a, int L, int num_sms, cudaStream_t s)
{
    switch (L) {
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
