// Voxel-driven backprojection over padded bilinear quads.
//
// Replaces the per-view loop of reconFDKHighMem (src/cuda/recon/fdk_axial.cuh:189-193): there,
// every view is copied into a cudaArray and one launch per view reads it through a bilinear
// texture and does vol += val * w (src/cuda/recon/back_proj.cuh:16-104), a full volume
// read-modify-write per view. Here one launch covers a range of views: each thread owns one
// (x, y) column and ZPT voxels along z, keeps their sums in registers across all views and
// writes the volume once.
//
// Column kernel (circular trajectories, "z-affine" geometry): per view, the column's detector
// column u, its bilinear split, the weight (projective and parallel kinds) and the row coordinate
// v(z) = v0 + z * vs are set up once. Each voxel then costs one FMA for v, a magic-number floor
// split, one IMAD.WIDE address, one 8- or 16-byte load of a bilinear-coefficient quad, two FMAs
// (one HFMA2 plus one FMA for FP16 storage) and the accumulate; pairs of voxels share packed
// FP32x2 instructions for the row split and the accumulate. A column segment whose rows all fall
// outside the detector contributes exactly zero (the reference's texture border) and is skipped;
// one that lies fully on the detector runs without per-voxel clamps.
//
// Mappings follow projMapping (src/cuda/geom/coord_trans_proj.cuh:157-345) through per-view
// coefficients in voxel-index space that the host derives in FP64.
#include "../../include/gct_fdk.h"
#include "common.cuh"
#include "geometry.hpp"
#include "kernels.hpp"

namespace gct {
namespace {

constexpr int kViewsPerChunk = 32;  // 2.5 KB of coefficients per block leaves L1 to the gathers
constexpr int kC = kCoefPerView;
constexpr float kShift = 12582912.0f;  // 1.5 * 2^23
constexpr int kShiftBits = 0x4B400000;  // bit pattern of kShift

// Coefficient layouts (per view, kCoefPerView floats):
//  affine     : [0..2] u0, ui, uj; [3..4] v0, vk; [5] wscale; [6..7] vi, vj (zero except for the
//               transposed one-row detector, where v is the detector coordinate)
//  projective : [0..3] U numerator; [4..7] V numerator; [8..11] denominator D; [12] wscale
//               u = U/D, v = V/D, weight = wscale / D^2
//  arc        : [0..3] A = e_u.d; [4..7] B = e_w.d; [8..11] T = e_v.d; [12] 1/dgamma; [13] c0;
//               [14] SDD/dv; [15] r0; [16] wscale
//               u = atan2(A, B)/dgamma + c0, v = SDD T / sqrt(A^2+B^2) / dv + r0,
//               weight = wscale / (A^2 + B^2 + T^2)
// Each affine form is c0 + ci*i + cj*j + ck*k in voxel indices.
__device__ __forceinline__ int wscale_slot(int family) { return family == 0 ? 5 : family == 1 ? 12 : 16; }

// Bilinear value of a stored coefficient quad (A, B, C, D) at column fraction fu in [0, 1] and
// centred row fraction fvc in [-0.5, 0.5]: (A + fu B) + fvc (C + fu D). The per-column form of fu
// (U) is precomputed once per view.
struct LerpF32 {
    using S = float4;
    using U = float;
    static __device__ __forceinline__ U ucol(float fu) { return fu; }
    static __device__ __forceinline__ float lerp(float4 q, U fu, float fvc)
    {
        return fmaf(fvc, fmaf(fu, q.w, q.z), fmaf(fu, q.y, q.x));
    }
};
struct LerpF16 {
    using S = uint2;  // .x = (A, C), .y = (B, D) as half2
    using U = __half2;
    static __device__ __forceinline__ U ucol(float fu) { return __float2half2_rn(fu); }
    static __device__ __forceinline__ float lerp(uint2 q, U fu2, float fvc)
    {
        const __half2 ac = *reinterpret_cast<__half2 *>(&q.x);
        const __half2 bd = *reinterpret_cast<__half2 *>(&q.y);
        const float2 e = __half22float2(__hfma2(fu2, bd, ac));  // (A + fu B, C + fu D)
        return fmaf(fvc, e.y, e.x);
    }
};
template <class Q> struct LerpOf;
template <> struct LerpOf<QuadF32> { using type = LerpF32; };
template <> struct LerpOf<QuadF16> { using type = LerpF16; };

struct ConstWeight {
    float w;
    __device__ __forceinline__ float at(int) const { return w; }
};
struct ArcWeight {  // wscale / (rho^2 + T(z)^2), T(z) = T0 + z tk
    float ws, rho2, T0, tk;
    __device__ __forceinline__ float at(int z) const
    {
        const float T = fmaf(tk, static_cast<float>(z), T0);
        return ws * rcp_approx(fmaf(T, T, rho2));
    }
};

// Accumulates one view into the ZPT voxels of a column. The row coordinate enters as
// vm(z) = v(z) - 0.5 = vm0 + z vs; the 1.5 * 2^23 shifter rounds it to the quad row iv (the
// floor of v, or v - 1 at integers) and leaves the centred fraction vm - iv in [-0.5, 0.5].
// `base` is arranged so that base + bits(t) * stride addresses quad row iv + kQuadPad, where
// bits(t) is the float bit pattern of the shifted coordinate.
// MIRROR (z-mirror plans, ZPT even): the column's mirror voxels nz - 1 - k sample row position
// nr - 1 - v, i.e. vm' = (nr - 2) - vm: quad row nr - 2 - iv with the centred fraction negated,
// addressed as mbase - bits(t) * stride; their sums go to accm. In clamped (mixed) columns the
// mirror coordinate is clamped and split on its own.
template <class L, int ZPT, bool CLAMP, bool MIRROR = false, class W>
__device__ __forceinline__ void column(unsigned long long base, int stride, typename L::U fu, float vm0, float vs,
                                       float vmax, const W &wt, float (&acc)[ZPT], unsigned long long mbase = 0,
                                       float (*accm)[ZPT] = nullptr)
{
    static_assert(!MIRROR || ZPT % 2 == 0, "mirror columns take voxel pairs");
    if constexpr (ZPT % 2 == 0) {
        // voxel pairs (z, z + 1): the row split and the accumulate run as packed FP32x2
        // operations (sm_100 FFMA2 / FADD2), element for element the same roundings as below
        const float2 shift = make_float2(kShift, kShift), mshift = make_float2(-kShift, -kShift);
        const float2 vs2 = make_float2(vs, vs), vm02 = make_float2(vm0, vm0);
#pragma unroll
        for (int z = 0; z < ZPT; z += 2) {
            float2 vm = __ffma2_rn(vs2, make_float2(static_cast<float>(z), static_cast<float>(z + 1)), vm02);
            float2 vmm = make_float2(0.f, 0.f);
            if (MIRROR && CLAMP) {
                vmm = make_float2(fminf(fmaxf((vmax - 2.0f) - vm.x, -1.5f), vmax - 0.5f),
                                  fminf(fmaxf((vmax - 2.0f) - vm.y, -1.5f), vmax - 0.5f));
            }
            if (CLAMP) {
                vm.x = fminf(fmaxf(vm.x, -1.5f), vmax - 0.5f);
                vm.y = fminf(fmaxf(vm.y, -1.5f), vmax - 0.5f);
            }
            const float2 t = __fadd2_rn(vm, shift);
            const float2 fl = __fadd2_rn(t, mshift);
            const float2 fvc = __ffma2_rn(fl, make_float2(-1.0f, -1.0f), vm);  // vm - fl, exact
            const auto *p0 = reinterpret_cast<const typename L::S *>(
                base + static_cast<unsigned long long>(static_cast<long long>(__float_as_int(t.x)) * stride));
            const auto *p1 = reinterpret_cast<const typename L::S *>(
                base + static_cast<unsigned long long>(static_cast<long long>(__float_as_int(t.y)) * stride));
            const float2 val = make_float2(L::lerp(__ldg(p0), fu, fvc.x), L::lerp(__ldg(p1), fu, fvc.y));
            const float2 r = __ffma2_rn(make_float2(wt.at(z), wt.at(z + 1)), val, make_float2(acc[z], acc[z + 1]));
            acc[z] = r.x;
            acc[z + 1] = r.y;
            if constexpr (MIRROR) {
                float2 valm;
                if constexpr (CLAMP) {
                    const float2 tm = __fadd2_rn(vmm, shift);
                    const float2 flm = __fadd2_rn(tm, mshift);
                    const float2 fvm = __ffma2_rn(flm, make_float2(-1.0f, -1.0f), vmm);
                    const auto *q0 = reinterpret_cast<const typename L::S *>(
                        base + static_cast<unsigned long long>(static_cast<long long>(__float_as_int(tm.x)) * stride));
                    const auto *q1 = reinterpret_cast<const typename L::S *>(
                        base + static_cast<unsigned long long>(static_cast<long long>(__float_as_int(tm.y)) * stride));
                    valm = make_float2(L::lerp(__ldg(q0), fu, fvm.x), L::lerp(__ldg(q1), fu, fvm.y));
                } else {
                    const auto *q0 = reinterpret_cast<const typename L::S *>(
                        mbase - static_cast<unsigned long long>(static_cast<long long>(__float_as_int(t.x)) * stride));
                    const auto *q1 = reinterpret_cast<const typename L::S *>(
                        mbase - static_cast<unsigned long long>(static_cast<long long>(__float_as_int(t.y)) * stride));
                    valm = make_float2(L::lerp(__ldg(q0), fu, -fvc.x), L::lerp(__ldg(q1), fu, -fvc.y));
                }
                float(&dm)[ZPT] = *accm;
                const float2 rm = __ffma2_rn(make_float2(wt.at(z), wt.at(z + 1)), valm, make_float2(dm[z], dm[z + 1]));
                dm[z] = rm.x;
                dm[z + 1] = rm.y;
            }
        }
    } else {
#pragma unroll
        for (int z = 0; z < ZPT; ++z) {
            float vm = fmaf(vs, static_cast<float>(z), vm0);
            if (CLAMP) vm = fminf(fmaxf(vm, -1.5f), vmax - 0.5f);
            const float t = vm + kShift;
            const float fvc = vm - (t - kShift);
            const auto *p = reinterpret_cast<const typename L::S *>(
                base + static_cast<unsigned long long>(static_cast<long long>(__float_as_int(t)) * stride));
            acc[z] = fmaf(wt.at(z), L::lerp(__ldg(p), fu, fvc), acc[z]);
        }
    }
}

// Block classes of one view (box_class): the block's voxels all project off the detector, all
// well inside it, or some of each.
constexpr int kBoxOff = 0, kBoxInside = 1, kBoxMixed = 2;

// cls == kBoxInside skips the per-column range tests: box_class has shown, with a margin, that
// every column of the block passes them, so the result is the same as with the tests.
// MIRROR: the column's mirror voxels as well (column(); accm), whose row segment is the mirror of
// this one's, so the same range decisions hold for both.
template <class L, int ZPT, bool MIRROR = false, class W>
__device__ __forceinline__ void column_dispatch(const typename L::S *view, int es, int qpitch, float u, float v0,
                                                float vs, float umax, float vmax, const W &wt, float (&acc)[ZPT],
                                                int cls = kBoxMixed, float (*accm)[ZPT] = nullptr)
{
    if (cls != kBoxInside && !(u >= -1.0f && u <= umax)) return;  // the column's rays miss the detector: zero
    int iu;
    float fu;
    split_coord(u, iu, fu);
    const float va = v0, vb = fmaf(vs, static_cast<float>(ZPT - 1), v0);
    const float lo = fminf(va, vb), hi = fmaxf(va, vb);
    if (cls != kBoxInside && (hi < -1.0f || lo > vmax)) return;  // the whole segment is off the detector
    const int stride = qpitch * es * static_cast<int>(sizeof(typename L::S));
    const unsigned long long base =
        reinterpret_cast<unsigned long long>(view + (iu + kQuadPad) * es) -
        static_cast<unsigned long long>(static_cast<long long>(kShiftBits - kQuadPad) * stride);
    const typename L::U fuc = L::ucol(fu);
    // mirror rows: base + bits' stride with bits' = (nr - 2 + 2 kShiftBits) - bits
    const unsigned long long mbase =
        MIRROR ? base + static_cast<unsigned long long>(
                            (static_cast<long long>(vmax) - 2 + 2LL * kShiftBits) * static_cast<long long>(stride))
               : 0ull;
    if (cls == kBoxInside || (lo >= -1.0f && hi <= vmax))
        column<L, ZPT, false, MIRROR>(base, stride, fuc, v0 - 0.5f, vs, vmax, wt, acc, mbase, accm);
    else
        column<L, ZPT, true, MIRROR>(base, stride, fuc, v0 - 0.5f, vs, vmax, wt, acc, mbase, accm);
}

// Classifies the block's voxel box [i0, i1] x [j0, j1] x [k0, k1] for one view of the affine or
// projective (z-affine) family. u and v are linear or linear-fractional in each index with a
// positive denominator over the box, so their extremes are at the corners; the tests keep a
// margin of 1/64 pixel so that the per-column values, computed with the same formulas, agree.
template <int FAMILY>
__device__ __forceinline__ int box_class(const float *c, float i0, float i1, float j0, float j1, float k0, float k1,
                                         float umax, float vmax)
{
    float ulo = 3.0e38f, uhi = -3.0e38f, vlo = 3.0e38f, vhi = -3.0e38f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float fi = (q & 1) ? i1 : i0, fj = (q & 2) ? j1 : j0;
        float u, va, vb;
        if (FAMILY == 0) {
            u = fmaf(c[2], fj, fmaf(c[1], fi, c[0]));
            const float V = fmaf(c[7], fj, fmaf(c[6], fi, c[3]));
            va = fmaf(c[4], k0, V);
            vb = fmaf(c[4], k1, V);
        } else {
            const float D = fmaf(c[10], fj, fmaf(c[9], fi, c[8]));
            if (!(D > 0.0f)) return kBoxMixed;
            const float inv = rcp_approx(D);
            u = fmaf(c[2], fj, fmaf(c[1], fi, c[0])) * inv;
            const float V = fmaf(c[6], fj, fmaf(c[5], fi, c[4]));
            va = fmaf(c[7], k0, V) * inv;
            vb = fmaf(c[7], k1, V) * inv;
        }
        ulo = fminf(ulo, u);
        uhi = fmaxf(uhi, u);
        vlo = fminf(vlo, fminf(va, vb));
        vhi = fmaxf(vhi, fmaxf(va, vb));
    }
    const float m = 1.0f / 64.0f;
    if (uhi < -1.0f - m || ulo > umax + m || vhi < -1.0f - m || vlo > vmax + m) return kBoxOff;
    if (ulo >= -1.0f + m && uhi <= umax - m && vlo >= -1.0f + m && vhi <= vmax - m) return kBoxInside;
    return kBoxMixed;
}

// Clamped bilinear sample at (u, v) for the per-voxel (non-z-affine) kernels.
template <class L>
__device__ __forceinline__ float sample(const typename L::S *view, int es, int qpitch, float u, float v, float umax,
                                        float vmax)
{
    u = fminf(fmaxf(u, -1.0f), umax);
    const float vm = fminf(fmaxf(v, -1.0f), vmax) - 0.5f;
    int iu;
    float fu;
    split_coord(u, iu, fu);
    const float t = vm + kShift;
    const int iv = __float_as_int(t) - kShiftBits;
    const float fvc = vm - (t - kShift);
    return L::lerp(__ldg(view + static_cast<long long>((iv + kQuadPad) * qpitch + iu + kQuadPad) * es), L::ucol(fu),
                   fvc);
}

// Backprojects views [a.v_begin, a.v_begin + a.v_count) into the column segment (i, j, k0 ..
// k0 + ZPT - 1) of the calling thread, staging VPS views of coefficients at a time in s_coef.
// Every thread of the block calls it (it holds block barriers); inactive threads only help to
// stage. mode: kStore writes the sums, kAccumulate adds them to the volume, kAtomic adds them
// with atomics (several blocks share the voxels).
// Voxel box of the calling block (active columns only; the full ZPT segment along z), used to
// classify each view for the whole block.
struct BlockBox {
    float i0, i1, j0, j1, k0, k1;
};

// ES is the entry step of the stack's quad_layout: 1 view-major, 4 interleaved partner views.
// MIRROR (z-mirror plans: affine or projective family, z-affine, ZPT even): the segment lies in
// the lower half of the grid and the thread also sums its mirror voxels nz - 1 - k.
template <int FAMILY, class Q, int ZPT, bool ZAFFINE, int ES = 1, bool MIRROR = false>
__device__ __forceinline__ void bp_column(const BpArgs &a, int i, int j, int k0, bool active, int vps,
                                          float4 *s_coef, int *s_cls, const BlockBox *s_box, int tid, int nthr,
                                          int mode)
{
    static_assert(!MIRROR || (ZAFFINE && FAMILY != 2 && ES == 1), "mirror columns: z-affine view-major stacks");
    constexpr bool kClassify = ZAFFINE && FAMILY != 2;
    using L = typename LerpOf<Q>::type;
    using S = typename L::S;
    const float fi = static_cast<float>(i), fj = static_cast<float>(j), fk0 = static_cast<float>(k0);
    const S *quads = static_cast<const S *>(a.quads);

    float acc[ZPT], accm[ZPT];
#pragma unroll
    for (int z = 0; z < ZPT; ++z) acc[z] = accm[z] = 0.f;

    for (int vc = 0; vc < a.v_count; vc += vps) {
        const int nvc = min(vps, a.v_count - vc);
        __syncthreads();
        const float4 *g = reinterpret_cast<const float4 *>(a.coefs + static_cast<long long>(a.v_begin + vc) * kC);
        for (int t = tid; t < nvc * kC / 4; t += nthr) s_coef[t] = __ldg(g + t);
        __syncthreads();
        if (a.vinv || kClassify) {
            for (int t = tid; t < nvc; t += nthr) {
                float *ct = reinterpret_cast<float *>(s_coef) + t * kC;
                if (a.vinv) ct[wscale_slot(FAMILY)] *= __ldg(a.vinv + a.v_begin + vc + t);
                if (kClassify)
                    s_cls[t] = box_class<FAMILY>(ct, s_box->i0, s_box->i1, s_box->j0, s_box->j1, s_box->k0, s_box->k1,
                                                 a.umax, a.vmax);
            }
            __syncthreads();
        }
        if (!active) continue;
        for (int vv = 0; vv < nvc; ++vv) {
            const int cls = kClassify ? s_cls[vv] : kBoxMixed;
            if (cls == kBoxOff) continue;  // exact: every column of the block would add zero
            const float *c = reinterpret_cast<const float *>(s_coef) + vv * kC;
            const long long v = a.v_begin + vc + vv;
            const S *view = ES == 1 ? quads + v * a.qview : quads + ((v % a.quarter) * a.qview * 4 + v / a.quarter);
            constexpr int es = ES;
            if (FAMILY == 0) {
                // parallel kinds: u = u0 + ui i + uj j, v = v0 + vi i + vj j + vk k, constant weight
                const float u = fmaf(c[2], fj, fmaf(c[1], fi, c[0]));
                const float v0 = fmaf(c[4], fk0, fmaf(c[7], fj, fmaf(c[6], fi, c[3])));
                column_dispatch<L, ZPT, MIRROR>(view, es, a.qpitch, u, v0, c[4], a.umax, a.vmax, ConstWeight{c[5]},
                                                acc, cls, MIRROR ? &accm : nullptr);
            } else if (FAMILY == 1) {
                if (ZAFFINE) {
                    const float D = fmaf(c[10], fj, fmaf(c[9], fi, c[8]));
                    const float inv = rcp_approx(D);
                    const float u = fmaf(c[2], fj, fmaf(c[1], fi, c[0])) * inv;
                    const float v0 = fmaf(c[7], fk0, fmaf(c[6], fj, fmaf(c[5], fi, c[4]))) * inv;
                    column_dispatch<L, ZPT, MIRROR>(view, es, a.qpitch, u, v0, c[7] * inv, a.umax, a.vmax,
                                                    ConstWeight{c[12] * inv * inv}, acc, cls,
                                                    MIRROR ? &accm : nullptr);
                } else {
#pragma unroll
                    for (int z = 0; z < ZPT; ++z) {
                        const float fk = fk0 + static_cast<float>(z);
                        const float D = fmaf(c[11], fk, fmaf(c[10], fj, fmaf(c[9], fi, c[8])));
                        const float inv = rcp_approx(D);
                        const float u = fmaf(c[3], fk, fmaf(c[2], fj, fmaf(c[1], fi, c[0]))) * inv;
                        const float v = fmaf(c[7], fk, fmaf(c[6], fj, fmaf(c[5], fi, c[4]))) * inv;
                        acc[z] = fmaf(c[12] * inv * inv, sample<L>(view, es, a.qpitch, u, v, a.umax, a.vmax), acc[z]);
                    }
                }
            } else {
                if (ZAFFINE) {
                    const float A = fmaf(c[2], fj, fmaf(c[1], fi, c[0]));
                    const float B = fmaf(c[6], fj, fmaf(c[5], fi, c[4]));
                    const float rho2 = fmaf(A, A, B * B);
                    const float u = fmaf(atan2f(A, B), c[12], c[13]);
                    const float vsr = c[14] * rsqrtf(rho2);
                    const float T0 = fmaf(c[11], fk0, c[8]);
                    column_dispatch<L, ZPT>(view, es, a.qpitch, u, fmaf(vsr, T0, c[15]), vsr * c[11], a.umax, a.vmax,
                                            ArcWeight{c[16], rho2, T0, c[11]}, acc);
                } else {
#pragma unroll
                    for (int z = 0; z < ZPT; ++z) {
                        const float fk = fk0 + static_cast<float>(z);
                        const float A = fmaf(c[3], fk, fmaf(c[2], fj, fmaf(c[1], fi, c[0])));
                        const float B = fmaf(c[7], fk, fmaf(c[6], fj, fmaf(c[5], fi, c[4])));
                        const float T = fmaf(c[11], fk, fmaf(c[10], fj, fmaf(c[9], fi, c[8])));
                        const float rho2 = fmaf(A, A, B * B);
                        const float u = fmaf(atan2f(A, B), c[12], c[13]);
                        const float v = fmaf(c[14] * rsqrtf(rho2), T, c[15]);
                        const float w = c[16] * rcp_approx(fmaf(T, T, rho2));
                        acc[z] = fmaf(w, sample<L>(view, es, a.qpitch, u, v, a.umax, a.vmax), acc[z]);
                    }
                }
            }
        }
    }
    if (!active) return;
    const int kend = MIRROR ? a.nz / 2 : a.nz;
#pragma unroll
    for (int z = 0; z < ZPT; ++z) {
        const int k = k0 + z;
        if (k < kend) {
            float *dst = a.vol + (static_cast<long long>(k) * a.ny + j) * a.nx + i;
            if (mode == kBpAtomic) atomicAdd(dst, acc[z]);
            else *dst = mode == kBpAccumulate ? *dst + acc[z] : acc[z];
            if constexpr (MIRROR) {
                float *dm = a.vol + (static_cast<long long>(a.nz - 1 - k) * a.ny + j) * a.nx + i;
                if (mode == kBpAtomic) atomicAdd(dm, accm[z]);
                else *dm = mode == kBpAccumulate ? *dm + accm[z] : accm[z];
            }
        }
    }
}

__device__ __forceinline__ BlockBox block_box(const BpArgs &a, int i0, int j0, int bx, int by, int k0, int zpt)
{
    return BlockBox{static_cast<float>(i0), static_cast<float>(min(i0 + bx, a.nx) - 1), static_cast<float>(j0),
                    static_cast<float>(min(j0 + by, a.ny) - 1), static_cast<float>(k0),
                    static_cast<float>(k0 + zpt - 1)};
}

// View-split launch (a.vchunk > 0): grid slice blockIdx.z takes its chunk of the view range and
// its own partial image; true when the launch is split.
__device__ __forceinline__ bool split_views(BpArgs &a)
{
    if (a.vchunk <= 0) return false;
    const int z = blockIdx.z, b = z * a.vchunk;
    a.v_begin += b;
    a.v_count = max(0, min(a.vchunk, a.v_count - b));
    a.vol += z * a.vol_stride;
    a.accumulate = 0;
    return true;
}

template <int FAMILY, class Q, int ZPT, bool ZAFFINE, int ES>
__global__ void __launch_bounds__(256) bp_kernel(BpArgs a)
{
    __shared__ float4 s_coef[kViewsPerChunk * kC / 4];
    __shared__ int s_cls[kViewsPerChunk];
    __shared__ BlockBox s_box;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    BpArgs la = a;
    const int k0 = split_views(la) ? 0 : blockIdx.z * ZPT;
    if (threadIdx.x == 0 && threadIdx.y == 0)
        s_box = block_box(a, blockIdx.x * blockDim.x, blockIdx.y * blockDim.y, blockDim.x, blockDim.y, k0, ZPT);
    if (a.slice_views) {  // spiral scans: this slice's rotation of views (ZPT == 1, uniform per block)
        const int2 w = a.slice_views[k0 < a.nz ? k0 : a.nz - 1];
        const int b = max(w.x, a.v_begin), e = min(w.x + w.y, a.v_begin + a.v_count);
        la.v_begin = b;
        la.v_count = max(0, e - b);
    }
    // the first barrier of bp_column orders the s_box store before any read
    bp_column<FAMILY, Q, ZPT, ZAFFINE, ES>(la, i, j, k0, i < a.nx && j < a.ny, kViewsPerChunk, s_coef, s_cls, &s_box,
                                           threadIdx.y * blockDim.x + threadIdx.x, blockDim.x * blockDim.y,
                                           a.accumulate ? kBpAccumulate : kBpStore);
}

// z-mirror plans (a.mirror): the grid covers the lower half of the volume along z; each thread's
// segment also serves its mirror voxels (bp_column MIRROR). Affine and projective z-affine
// families, view-major stacks, an even number of voxels per thread.
template <int FAMILY, class Q, int ZPT>
__global__ void __launch_bounds__(256) bp_mirror_kernel(BpArgs a)
{
    __shared__ float4 s_coef[kViewsPerChunk * kC / 4];
    __shared__ int s_cls[kViewsPerChunk];
    __shared__ BlockBox s_box;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k0 = blockIdx.z * ZPT;
    if (threadIdx.x == 0 && threadIdx.y == 0)
        s_box = block_box(a, blockIdx.x * blockDim.x, blockIdx.y * blockDim.y, blockDim.x, blockDim.y, k0, ZPT);
    // the first barrier of bp_column orders the s_box store before any read
    bp_column<FAMILY, Q, ZPT, true, 1, true>(a, i, j, k0, i < a.nx && j < a.ny, kViewsPerChunk, s_coef, s_cls, &s_box,
                                             threadIdx.y * blockDim.x + threadIdx.x, blockDim.x * blockDim.y,
                                             a.accumulate ? kBpAccumulate : kBpStore);
}

template <int FAMILY, class Q, int ZPT>
void launch_zpt(const BpArgs &a, bool z_affine, dim3 grid, dim3 block, cudaStream_t s)
{
    if constexpr (FAMILY != 2 && ZPT % 2 == 0) {
        if (a.mirror) {
            bp_mirror_kernel<FAMILY, Q, ZPT><<<grid, block, 0, s>>>(a);
            return;
        }
    }
    if (a.quarter)  // interleaved partner views: quarter-turn plans, which are z-affine
        bp_kernel<FAMILY, Q, ZPT, true, 4><<<grid, block, 0, s>>>(a);
    else if (z_affine || FAMILY == 0)
        bp_kernel<FAMILY, Q, ZPT, true, 1><<<grid, block, 0, s>>>(a);
    else
        bp_kernel<FAMILY, Q, ZPT, false, 1><<<grid, block, 0, s>>>(a);
}

template <int FAMILY, class Q>
void launch_q(const BpArgs &a, bool z_affine, int zpt, int bx, int by, cudaStream_t s)
{
    const dim3 block(bx, by);
    const int nz = a.mirror ? a.nz / 2 : a.nz;  // mirror launches cover the lower half
    const unsigned gz = a.vchunk > 0 ? (a.v_count + a.vchunk - 1) / a.vchunk : (nz + zpt - 1) / zpt;
    const dim3 grid((a.nx + bx - 1) / bx, (a.ny + by - 1) / by, gz);
    switch (zpt) {
        case 1: launch_zpt<FAMILY, Q, 1>(a, z_affine, grid, block, s); break;
        case 2: launch_zpt<FAMILY, Q, 2>(a, z_affine, grid, block, s); break;
        case 4: launch_zpt<FAMILY, Q, 4>(a, z_affine, grid, block, s); break;
        case 8: launch_zpt<FAMILY, Q, 8>(a, z_affine, grid, block, s); break;
        default: launch_zpt<FAMILY, Q, 16>(a, z_affine, grid, block, s); break;
    }
}

// ---- quarter-turn backprojection -----------------------------------------------------------
//
// On a full circular scan whose views come in quarter-turn partners (view v + q m, m = nv / 4, is
// view v turned by q quarter turns about the rotation axis) and a square, centred grid of even
// side n, view v + q m samples voxel column R^q(x) exactly where view v samples column x (R is a
// quarter turn of the grid, (i, j) -> (n-1-j, i) or (j, n-1-i); the host checks every view in
// FP64). A thread owns the four columns R^k(c), k = 0..3, of one first-quadrant column c. Per base
// view v it evaluates the detector coordinates of each of its columns (u, the weight, the row
// coordinates, their split and the quad offsets), and the evaluation at R^k(c) serves all four
// partners: partner q samples there for column R^(k+q)(c). The coordinate work is thus done once
// per four voxel-view updates; the loads, blends and accumulates are per update.

// Weight of partner q at voxel z: the partner's scale times a factor common to the four.
struct ConstWeight4 {
    float w[4];
    __device__ __forceinline__ float at(int q, int) const { return w[q]; }
};
struct ArcWeight4 {
    float ws[4];
    float rho2, T0, tk;
    __device__ __forceinline__ float at(int q, int z) const
    {
        const float T = fmaf(tk, static_cast<float>(z), T0);
        return ws[q] * rcp_approx(fmaf(T, T, rho2));
    }
};

// The four partner quads of one detector position in the quarter-turn layout (quad_layout): 32
// bytes (FP16) or 64 bytes (FP32), 32-byte aligned, read through the non-coherent path.
__device__ __forceinline__ void ldg_partners(unsigned long long p, uint2 (&o)[4])
{
    asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(o[0].x), "=r"(o[0].y), "=r"(o[1].x), "=r"(o[1].y), "=r"(o[2].x), "=r"(o[2].y), "=r"(o[3].x),
          "=r"(o[3].y)
        : "l"(p));
}
__device__ __forceinline__ void ldg_partners(unsigned long long p, float4 (&o)[4])
{
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(o[0].x), "=f"(o[0].y), "=f"(o[0].z), "=f"(o[0].w), "=f"(o[1].x), "=f"(o[1].y), "=f"(o[1].z),
          "=f"(o[1].w)
        : "l"(p));
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8+32];"
        : "=f"(o[2].x), "=f"(o[2].y), "=f"(o[2].z), "=f"(o[2].w), "=f"(o[3].x), "=f"(o[3].y), "=f"(o[3].z),
          "=f"(o[3].w)
        : "l"(p));
}

// column() for the four partners of one evaluation: `base` addresses the partner groups as in
// column(), and partner q accumulates into column (K + q) mod 4.
template <class L, int ZPT, int K, bool CLAMP, class W>
__device__ __forceinline__ void column4(unsigned long long base, int stride, typename L::U fu, float vm0, float vs,
                                        float vmax, const W &wt, float (&acc)[4][ZPT])
{
    if constexpr (ZPT % 2 == 0) {
        const float2 shift = make_float2(kShift, kShift), mshift = make_float2(-kShift, -kShift);
        const float2 vs2 = make_float2(vs, vs), vm02 = make_float2(vm0, vm0);
#pragma unroll
        for (int z = 0; z < ZPT; z += 2) {
            float2 vm = __ffma2_rn(vs2, make_float2(static_cast<float>(z), static_cast<float>(z + 1)), vm02);
            if (CLAMP) {
                vm.x = fminf(fmaxf(vm.x, -1.5f), vmax - 0.5f);
                vm.y = fminf(fmaxf(vm.y, -1.5f), vmax - 0.5f);
            }
            const float2 t = __fadd2_rn(vm, shift);
            const float2 fl = __fadd2_rn(t, mshift);
            const float2 fvc = __ffma2_rn(fl, make_float2(-1.0f, -1.0f), vm);
            typename L::S q0[4], q1[4];
            ldg_partners(base + static_cast<unsigned long long>(static_cast<long long>(__float_as_int(t.x)) * stride), q0);
            ldg_partners(base + static_cast<unsigned long long>(static_cast<long long>(__float_as_int(t.y)) * stride), q1);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float2 val = make_float2(L::lerp(q0[q], fu, fvc.x), L::lerp(q1[q], fu, fvc.y));
                float(&dst)[ZPT] = acc[(K + q) & 3];
                const float2 r =
                    __ffma2_rn(make_float2(wt.at(q, z), wt.at(q, z + 1)), val, make_float2(dst[z], dst[z + 1]));
                dst[z] = r.x;
                dst[z + 1] = r.y;
            }
        }
    } else {
#pragma unroll
        for (int z = 0; z < ZPT; ++z) {
            float vm = fmaf(vs, static_cast<float>(z), vm0);
            if (CLAMP) vm = fminf(fmaxf(vm, -1.5f), vmax - 0.5f);
            const float t = vm + kShift;
            const float fvc = vm - (t - kShift);
            typename L::S qv[4];
            ldg_partners(base + static_cast<unsigned long long>(static_cast<long long>(__float_as_int(t)) * stride), qv);
#pragma unroll
            for (int q = 0; q < 4; ++q)
                acc[(K + q) & 3][z] = fmaf(wt.at(q, z), L::lerp(qv[q], fu, fvc), acc[(K + q) & 3][z]);
        }
    }
}

// column_dispatch() for the four partners of one evaluation; group0 is the base view's grid of
// partner groups (four quads per detector position).
template <class L, int ZPT, int K, class W>
__device__ __forceinline__ void column4_dispatch(const typename L::S *group0, int qpitch, float u, float v0, float vs,
                                                 float umax, float vmax, const W &wt, float (&acc)[4][ZPT], int cls)
{
    if (cls != kBoxInside && !(u >= -1.0f && u <= umax)) return;
    int iu;
    float fu;
    split_coord(u, iu, fu);
    const float va = v0, vb = fmaf(vs, static_cast<float>(ZPT - 1), v0);
    const float lo = fminf(va, vb), hi = fmaxf(va, vb);
    if (cls != kBoxInside && (hi < -1.0f || lo > vmax)) return;
    const int stride = qpitch * 4 * static_cast<int>(sizeof(typename L::S));
    const unsigned long long base = reinterpret_cast<unsigned long long>(group0 + (iu + kQuadPad) * 4) -
                                    static_cast<unsigned long long>(static_cast<long long>(kShiftBits - kQuadPad) * stride);
    const typename L::U fuc = L::ucol(fu);
    if (cls == kBoxInside || (lo >= -1.0f && hi <= vmax))
        column4<L, ZPT, K, false>(base, stride, fuc, v0 - 0.5f, vs, vmax, wt, acc);
    else
        column4<L, ZPT, K, true>(base, stride, fuc, v0 - 0.5f, vs, vmax, wt, acc);
}

// One quarter turn of column (i, j) on a grid of side n: (n-1-j, i) for sym = +1, (j, n-1-i)
// for sym = -1.
__device__ __forceinline__ void turn(int sym, int n, int &i, int &j)
{
    const int ti = sym > 0 ? n - 1 - j : j, tj = sym > 0 ? i : n - 1 - i;
    i = ti;
    j = tj;
}
// The same turn of the index box [b.x, b.y] x [b.z, b.w].
__device__ __forceinline__ float4 turn_box(int sym, int n, float4 b)
{
    const float m = static_cast<float>(n - 1);
    return sym > 0 ? make_float4(m - b.w, m - b.z, b.x, b.y) : make_float4(b.z, b.w, m - b.y, m - b.x);
}

// Base view c (coefficients), evaluated at column (fi, fj) = R^K(c) of the thread; w holds the
// partners' weight scales.
template <int FAMILY, class L, int ZPT, int K>
__device__ __forceinline__ void sym_rotation(const BpArgs &a, const float *c, float4 w, const typename L::S *group0,
                                             float fi, float fj, float fk0, int cls, float (&acc)[4][ZPT])
{
    if (cls == kBoxOff) return;
    if (FAMILY == 0) {
        const float u = fmaf(c[2], fj, fmaf(c[1], fi, c[0]));
        const float v0 = fmaf(c[4], fk0, fmaf(c[7], fj, fmaf(c[6], fi, c[3])));
        column4_dispatch<L, ZPT, K>(group0, a.qpitch, u, v0, c[4], a.umax, a.vmax,
                                    ConstWeight4{{w.x, w.y, w.z, w.w}}, acc, cls);
    } else if (FAMILY == 1) {
        const float D = fmaf(c[10], fj, fmaf(c[9], fi, c[8]));
        const float inv = rcp_approx(D);
        const float u = fmaf(c[2], fj, fmaf(c[1], fi, c[0])) * inv;
        const float v0 = fmaf(c[7], fk0, fmaf(c[6], fj, fmaf(c[5], fi, c[4]))) * inv;
        const float i2 = inv * inv;
        column4_dispatch<L, ZPT, K>(group0, a.qpitch, u, v0, c[7] * inv, a.umax, a.vmax,
                                    ConstWeight4{{w.x * i2, w.y * i2, w.z * i2, w.w * i2}}, acc, cls);
    } else {
        const float A = fmaf(c[2], fj, fmaf(c[1], fi, c[0]));
        const float B = fmaf(c[6], fj, fmaf(c[5], fi, c[4]));
        const float rho2 = fmaf(A, A, B * B);
        const float u = fmaf(atan2f(A, B), c[12], c[13]);
        const float vsr = c[14] * rsqrtf(rho2);
        const float T0 = fmaf(c[11], fk0, c[8]);
        column4_dispatch<L, ZPT, K>(group0, a.qpitch, u, fmaf(vsr, T0, c[15]), vsr * c[11], a.umax, a.vmax,
                                    ArcWeight4{{w.x, w.y, w.z, w.w}, rho2, T0, c[11]}, acc, cls);
    }
}

// One block's tile of the quarter-turn form: first-quadrant columns [i0, i0 + bx) x [j0, j0 + by)
// and voxels [k0, k0 + ZPT) along z, over base views [a.v_begin, a.v_begin + a.v_count). tid is
// the thread's index in the block (column i0 + tid % bx, j0 + tid / bx); every thread of the block
// calls it (it holds block barriers). mode: kBpStore, kBpAccumulate or kBpAtomic for the four
// turned columns of each thread.
template <int FAMILY, class Q, int ZPT>
__device__ __forceinline__ void sym_tile(const BpArgs &a, int i0, int j0, int k0, int bx, int by, int tid, int nthr,
                                         int mode, float4 *s_coef, float4 *s_w, int *s_cls)
{
    using L = typename LerpOf<Q>::type;
    using S = typename L::S;
    constexpr bool kClassify = FAMILY != 2;
    const int n = a.nx, h = n / 2;
    const int i = i0 + tid % bx, j = j0 + tid / bx;
    const bool active = tid < bx * by && i < h && j < h;
    const float fk0 = static_cast<float>(k0);
    const S *quads = static_cast<const S *>(a.quads);
    const int wslot = wscale_slot(FAMILY);

    // the thread's four columns and the block's four boxes (active columns only)
    float fi[4], fj[4];
    {
        int ti = i, tj = j;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            fi[k] = static_cast<float>(ti);
            fj[k] = static_cast<float>(tj);
            turn(a.sym, n, ti, tj);
        }
    }
    const float4 box0 = make_float4(static_cast<float>(i0), static_cast<float>(min(i0 + bx, h) - 1),
                                    static_cast<float>(j0), static_cast<float>(min(j0 + by, h) - 1));
    const float bk0 = fk0, bk1 = static_cast<float>(k0 + ZPT - 1);

    float acc[4][ZPT];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int z = 0; z < ZPT; ++z) acc[q][z] = 0.f;

    for (int vc = 0; vc < a.v_count; vc += kViewsPerChunk) {
        const int nvc = min(kViewsPerChunk, a.v_count - vc);
        __syncthreads();
        const float4 *g = reinterpret_cast<const float4 *>(a.coefs + static_cast<long long>(a.v_begin + vc) * kC);
        for (int t = tid; t < nvc * kC / 4; t += nthr) s_coef[t] = __ldg(g + t);
        for (int t = tid; t < nvc; t += nthr) {
            float w[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const long long v = a.v_begin + vc + t + static_cast<long long>(q) * a.quarter;
                w[q] = __ldg(a.coefs + v * kC + wslot) * (a.vinv ? __ldg(a.vinv + v) : 1.0f);
            }
            s_w[t] = make_float4(w[0], w[1], w[2], w[3]);
        }
        __syncthreads();
        for (int t = tid; t < nvc; t += nthr) {
            int packed = 0;
            float4 b = box0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int cls = kClassify ? box_class<FAMILY>(reinterpret_cast<const float *>(s_coef) + t * kC, b.x,
                                                              b.y, b.z, b.w, bk0, bk1, a.umax, a.vmax)
                                          : kBoxMixed;
                packed |= cls << (2 * k);
                b = turn_box(a.sym, n, b);
            }
            s_cls[t] = packed;
        }
        __syncthreads();
        if (!active) continue;
        for (int vv = 0; vv < nvc; ++vv) {
            const int packed = s_cls[vv];
            if (packed == 0) continue;  // every turned box off the detector (kBoxOff == 0)
            // read from shared memory by each evaluation: copying them to registers once per base
            // view measured slower (128 registers, 37.0 against 34.4 ms at 512^3)
            const float *c = reinterpret_cast<const float *>(s_coef) + vv * kC;
            const float4 w = s_w[vv];
            // base views are below quarter, so their partner groups start at 4 qview per view
            const S *group0 = quads + static_cast<long long>(a.v_begin + vc + vv) * a.qview * 4;
            sym_rotation<FAMILY, L, ZPT, 0>(a, c, w, group0, fi[0], fj[0], fk0, packed & 3, acc);
            sym_rotation<FAMILY, L, ZPT, 1>(a, c, w, group0, fi[1], fj[1], fk0, (packed >> 2) & 3, acc);
            sym_rotation<FAMILY, L, ZPT, 2>(a, c, w, group0, fi[2], fj[2], fk0, (packed >> 4) & 3, acc);
            sym_rotation<FAMILY, L, ZPT, 3>(a, c, w, group0, fi[3], fj[3], fk0, (packed >> 6) & 3, acc);
        }
    }
    if (!active) return;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int ti = static_cast<int>(fi[q]), tj = static_cast<int>(fj[q]);
#pragma unroll
        for (int z = 0; z < ZPT; ++z) {
            const int k = k0 + z;
            if (k < a.nz) {
                float *dst = a.vol + (static_cast<long long>(k) * a.ny + tj) * a.nx + ti;
                if (mode == kBpAtomic) atomicAdd(dst, acc[q][z]);
                else *dst = mode == kBpAccumulate ? *dst + acc[q][z] : acc[q][z];
            }
        }
    }
}

template <int FAMILY, class Q, int ZPT>
__global__ void __launch_bounds__(256) bp_sym_kernel(BpArgs a)
{
    __shared__ float4 s_coef[kViewsPerChunk * kC / 4];
    __shared__ float4 s_w[kViewsPerChunk];  // weight scales of the four partners of each base view
    __shared__ int s_cls[kViewsPerChunk];   // box class of each of the block's four turned boxes, 2 bits each
    sym_tile<FAMILY, Q, ZPT>(a, blockIdx.x * blockDim.x, blockIdx.y * blockDim.y, blockIdx.z * ZPT, blockDim.x,
                             blockDim.y, threadIdx.y * blockDim.x + threadIdx.x, blockDim.x * blockDim.y,
                             a.accumulate ? kBpAccumulate : kBpStore, s_coef, s_w, s_cls);
}

// The view-split launch of bp_sym_kernel (a.vchunk > 0, one-voxel-deep images): its own kernel, so
// that the whole-volume kernel keeps its register allocation (the local copy of the arguments
// here took it from 128 to 102 registers, and 34.8 to 42.5 ms at 512^3 / 720 views).
template <int FAMILY, class Q, int ZPT>
__global__ void __launch_bounds__(256) bp_sym_split_kernel(BpArgs a)
{
    __shared__ float4 s_coef[kViewsPerChunk * kC / 4];
    __shared__ float4 s_w[kViewsPerChunk];
    __shared__ int s_cls[kViewsPerChunk];
    BpArgs la = a;
    split_views(la);
    sym_tile<FAMILY, Q, ZPT>(la, blockIdx.x * blockDim.x, blockIdx.y * blockDim.y, 0, blockDim.x, blockDim.y,
                             threadIdx.y * blockDim.x + threadIdx.x, blockDim.x * blockDim.y, kBpStore, s_coef, s_w,
                             s_cls);
}

template <int FAMILY, class Q>
void launch_sym_q(const BpArgs &a, int zpt, int bx, int by, cudaStream_t s)
{
    const int h = a.nx / 2;
    const dim3 block(bx, by);
    const unsigned gz = a.vchunk > 0 ? (a.v_count + a.vchunk - 1) / a.vchunk : (a.nz + zpt - 1) / zpt;
    const dim3 grid((h + bx - 1) / bx, (h + by - 1) / by, gz);
    if (a.vchunk > 0) {
        switch (zpt) {
            case 1: bp_sym_split_kernel<FAMILY, Q, 1><<<grid, block, 0, s>>>(a); break;
            case 2: bp_sym_split_kernel<FAMILY, Q, 2><<<grid, block, 0, s>>>(a); break;
            case 4: bp_sym_split_kernel<FAMILY, Q, 4><<<grid, block, 0, s>>>(a); break;
            default: bp_sym_split_kernel<FAMILY, Q, 8><<<grid, block, 0, s>>>(a); break;
        }
        return;
    }
    switch (zpt) {
        case 1: bp_sym_kernel<FAMILY, Q, 1><<<grid, block, 0, s>>>(a); break;
        case 2: bp_sym_kernel<FAMILY, Q, 2><<<grid, block, 0, s>>>(a); break;
        case 4: bp_sym_kernel<FAMILY, Q, 4><<<grid, block, 0, s>>>(a); break;
        default: bp_sym_kernel<FAMILY, Q, 8><<<grid, block, 0, s>>>(a); break;
    }
}

// ---- work-queue backprojection -----------------------------------------------------------

// Not inlined: each (family, storage, z depth) path gets its own register allocation instead of
// the union of all paths; the call happens once per work entry.
template <int FAMILY, class Q, int ZPT>
__device__ __noinline__ void queue_tile_z(const BpItem &it, const BpArgs &a, int tx, int ty, int tz, int tid,
                                             int mode, float4 *s_coef, int *s_cls, BlockBox *s_box)
{
    const int i0 = tx * it.bx, j0 = ty * it.by, k0 = tz * ZPT;
    const int i = i0 + tid % it.bx, j = j0 + tid / it.bx;
    const bool active = i < a.nx && j < a.ny;
    if (tid == 0) *s_box = block_box(a, i0, j0, it.bx, it.by, k0, ZPT);  // ordered by bp_column's first barrier
    if (FAMILY == 0 || it.z_affine)
        bp_column<FAMILY, Q, ZPT, true>(a, i, j, k0, active, it.vps, s_coef, s_cls, s_box, tid, kQueueThreads, mode);
    else
        bp_column<FAMILY, Q, ZPT, false>(a, i, j, k0, active, it.vps, s_coef, s_cls, s_box, tid, kQueueThreads, mode);
}

template <int FAMILY, class Q, int ZC>
__device__ __forceinline__ void queue_tile(const BpItem &it, const BpArgs &a, int tx, int ty, int tz, int tid,
                                           int mode, float4 *s_coef, int *s_cls, BlockBox *s_box)
{
    if constexpr (ZC == 0) {
        queue_tile_z<FAMILY, Q, 1>(it, a, tx, ty, tz, tid, mode, s_coef, s_cls, s_box);
        return;
    }
    switch (it.zpt) {
        case 1: queue_tile_z<FAMILY, Q, 1>(it, a, tx, ty, tz, tid, mode, s_coef, s_cls, s_box); break;
        case 4: queue_tile_z<FAMILY, Q, 4>(it, a, tx, ty, tz, tid, mode, s_coef, s_cls, s_box); break;
        case 8: queue_tile_z<FAMILY, Q, 8>(it, a, tx, ty, tz, tid, mode, s_coef, s_cls, s_box); break;
        default: queue_tile_z<FAMILY, Q, 16>(it, a, tx, ty, tz, tid, mode, s_coef, s_cls, s_box); break;
    }
}

// Persistent blocks take work entries in queue order from a global counter; each entry is one
// tile of one reconstruction over a range of views. The item descriptor is read once per entry
// into shared memory; all control flow below depends only on it, so it is uniform per block.
template <class Q, int ZC>
__global__ void __launch_bounds__(kQueueThreads, ZC == 0 ? 4 : 2)
    bp_queue_kernel(const BpItem *__restrict__ items, const BpWork *__restrict__ work, int n_work, int *counter)
{
    __shared__ float4 s_coef[kQueueMaxVps * kC / 4];
    __shared__ int s_cls[kQueueMaxVps];
    __shared__ BlockBox s_box;
    __shared__ BpItem s_item;
    __shared__ BpWork s_work;
    __shared__ int s_next;
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) s_next = atomicAdd(counter, 1);
        __syncthreads();
        const int w = s_next;
        if (w >= n_work) return;
        if (tid == 0) {
            s_work = work[w];
            s_item = items[s_work.item];
        }
        __syncthreads();
        const BpItem &it = s_item;
        BpArgs a = it.a;
        a.v_begin = s_work.v_begin;
        a.v_count = s_work.v_count;
        const int mode = s_work.mode;
        const int t = s_work.tile;
        const int tx = t % it.tiles_x, ty = (t / it.tiles_x) % it.tiles_y, tz = t / (it.tiles_x * it.tiles_y);
        if (it.family == 0) queue_tile<0, Q, ZC>(it, a, tx, ty, tz, tid, mode, s_coef, s_cls, &s_box);
        else if (it.family == 1) queue_tile<1, Q, ZC>(it, a, tx, ty, tz, tid, mode, s_coef, s_cls, &s_box);
        else queue_tile<2, Q, ZC>(it, a, tx, ty, tz, tid, mode, s_coef, s_cls, &s_box);
        __syncthreads();  // s_item / s_work / s_next are rewritten for the next entry
    }
}

// Quarter-turn items of the work queue: tile (tx, ty, tz) of first-quadrant columns.
template <int FAMILY, class Q, int ZPT>
__device__ __noinline__ void queue_sym_tile_z(const BpItem &it, const BpArgs &a, int tx, int ty, int tz, int tid,
                                              int mode, float4 *s_coef, float4 *s_w, int *s_cls)
{
    sym_tile<FAMILY, Q, ZPT>(a, tx * it.bx, ty * it.by, tz * ZPT, it.bx, it.by, tid, kQueueThreads, mode, s_coef, s_w,
                             s_cls);
}
template <int FAMILY, class Q>
__device__ __forceinline__ void queue_sym_tile(const BpItem &it, const BpArgs &a, int tx, int ty, int tz, int tid,
                                               int mode, float4 *s_coef, float4 *s_w, int *s_cls)
{
    if (it.zpt == 1) queue_sym_tile_z<FAMILY, Q, 1>(it, a, tx, ty, tz, tid, mode, s_coef, s_w, s_cls);
    else queue_sym_tile_z<FAMILY, Q, 8>(it, a, tx, ty, tz, tid, mode, s_coef, s_w, s_cls);
}

template <class Q>
__global__ void __launch_bounds__(kQueueThreads, 2)
    bp_queue_sym_kernel(const BpItem *__restrict__ items, const BpWork *__restrict__ work, int n_work, int *counter)
{
    __shared__ float4 s_coef[kViewsPerChunk * kC / 4];
    __shared__ float4 s_w[kViewsPerChunk];
    __shared__ int s_cls[kViewsPerChunk];
    __shared__ BpItem s_item;
    __shared__ BpWork s_work;
    __shared__ int s_next;
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) s_next = atomicAdd(counter, 1);
        __syncthreads();
        const int w = s_next;
        if (w >= n_work) return;
        if (tid == 0) {
            s_work = work[w];
            s_item = items[s_work.item];
        }
        __syncthreads();
        const BpItem &it = s_item;
        BpArgs a = it.a;
        a.v_begin = s_work.v_begin;
        a.v_count = s_work.v_count;
        const int mode = s_work.mode;
        const int t = s_work.tile;
        const int tx = t % it.tiles_x, ty = (t / it.tiles_x) % it.tiles_y, tz = t / (it.tiles_x * it.tiles_y);
        if (it.family == 0) queue_sym_tile<0, Q>(it, a, tx, ty, tz, tid, mode, s_coef, s_w, s_cls);
        else if (it.family == 1) queue_sym_tile<1, Q>(it, a, tx, ty, tz, tid, mode, s_coef, s_w, s_cls);
        else queue_sym_tile<2, Q>(it, a, tx, ty, tz, tid, mode, s_coef, s_w, s_cls);
        __syncthreads();  // s_item / s_work / s_next are rewritten for the next entry
    }
}

__global__ void reduce_partials_kernel(const float *__restrict__ part, int nparts, long long n, float *vol,
                                       int accumulate)
{
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        float t = accumulate ? vol[i] : 0.f;
        for (int c = 0; c < nparts; ++c) t += __ldg(part + c * n + i);
        vol[i] = t;
    }
}

}  // namespace

namespace {
template <class K>
int occupancy(K kern, int threads)
{
    int n = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, 0) == cudaSuccess ? n : 0;
}
template <int FAMILY, class Q, int ZPT>
int occupancy_zpt(const BpArgs &a, bool z_affine, bool sym, int threads)
{
    if (sym) return occupancy(bp_sym_split_kernel<FAMILY, Q, ZPT>, threads);  // asked for view-split launches
    if (a.quarter) return occupancy(bp_kernel<FAMILY, Q, ZPT, true, 4>, threads);
    if (z_affine || FAMILY == 0) return occupancy(bp_kernel<FAMILY, Q, ZPT, true, 1>, threads);
    return occupancy(bp_kernel<FAMILY, Q, ZPT, false, 1>, threads);
}
template <int FAMILY, class Q>
int occupancy_q(const BpArgs &a, bool z_affine, bool sym, int zpt, int threads)
{
    switch (zpt) {
        case 1: return occupancy_zpt<FAMILY, Q, 1>(a, z_affine, sym, threads);
        case 2: return occupancy_zpt<FAMILY, Q, 2>(a, z_affine, sym, threads);
        case 4: return occupancy_zpt<FAMILY, Q, 4>(a, z_affine, sym, threads);
        case 8: return occupancy_zpt<FAMILY, Q, 8>(a, z_affine, sym, threads);
        default: return sym ? 0 : occupancy_zpt<FAMILY, Q, 16>(a, z_affine, sym, threads);
    }
}
}  // namespace

int backproject_blocks_per_sm(const BpArgs &a, int family, int storage, bool z_affine, bool sym, int zpt, int threads)
{
    if (storage == 0) {
        if (family == 0) return occupancy_q<0, QuadF32>(a, z_affine, sym, zpt, threads);
        if (family == 1) return occupancy_q<1, QuadF32>(a, z_affine, sym, zpt, threads);
        return occupancy_q<2, QuadF32>(a, z_affine, sym, zpt, threads);
    }
    if (family == 0) return occupancy_q<0, QuadF16>(a, z_affine, sym, zpt, threads);
    if (family == 1) return occupancy_q<1, QuadF16>(a, z_affine, sym, zpt, threads);
    return occupancy_q<2, QuadF16>(a, z_affine, sym, zpt, threads);
}

void launch_reduce_partials(const float *part, int nparts, long long n, float *vol, bool accumulate, cudaStream_t s)
{
    long long grid = (n + 255) / 256;
    if (grid > 148LL * 16) grid = 148LL * 16;
    reduce_partials_kernel<<<static_cast<unsigned>(grid < 1 ? 1 : grid), 256, 0, s>>>(part, nparts, n, vol,
                                                                                      accumulate ? 1 : 0);
}

void launch_backproject_sym(const BpArgs &a, int family, int storage, int zpt, int bx, int by, cudaStream_t s)
{
    if (storage == 0) {
        if (family == 0) launch_sym_q<0, QuadF32>(a, zpt, bx, by, s);
        else if (family == 1) launch_sym_q<1, QuadF32>(a, zpt, bx, by, s);
        else launch_sym_q<2, QuadF32>(a, zpt, bx, by, s);
    } else {
        if (family == 0) launch_sym_q<0, QuadF16>(a, zpt, bx, by, s);
        else if (family == 1) launch_sym_q<1, QuadF16>(a, zpt, bx, by, s);
        else launch_sym_q<2, QuadF16>(a, zpt, bx, by, s);
    }
}

int queue_blocks_per_sm(int storage, int zclass)
{
    int n = 0;
    cudaError_t e;
    if (zclass == kQueueSymClass)
        e = storage == 0 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bp_queue_sym_kernel<QuadF32>, kQueueThreads, 0)
                         : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bp_queue_sym_kernel<QuadF16>, kQueueThreads, 0);
    else if (storage == 0)
        e = zclass == 0 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bp_queue_kernel<QuadF32, 0>, kQueueThreads, 0)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bp_queue_kernel<QuadF32, 1>, kQueueThreads, 0);
    else
        e = zclass == 0 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bp_queue_kernel<QuadF16, 0>, kQueueThreads, 0)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bp_queue_kernel<QuadF16, 1>, kQueueThreads, 0);
    return e == cudaSuccess ? n : 0;
}

void launch_backproject_queue(const BpItem *items, const BpWork *work, int n_work, int *counter, int storage,
                              int zclass, int grid, cudaStream_t s)
{
    if (zclass == kQueueSymClass) {
        if (storage == 0) bp_queue_sym_kernel<QuadF32><<<grid, kQueueThreads, 0, s>>>(items, work, n_work, counter);
        else bp_queue_sym_kernel<QuadF16><<<grid, kQueueThreads, 0, s>>>(items, work, n_work, counter);
        return;
    }
    if (storage == 0) {
        if (zclass == 0) bp_queue_kernel<QuadF32, 0><<<grid, kQueueThreads, 0, s>>>(items, work, n_work, counter);
        else bp_queue_kernel<QuadF32, 1><<<grid, kQueueThreads, 0, s>>>(items, work, n_work, counter);
    } else {
        if (zclass == 0) bp_queue_kernel<QuadF16, 0><<<grid, kQueueThreads, 0, s>>>(items, work, n_work, counter);
        else bp_queue_kernel<QuadF16, 1><<<grid, kQueueThreads, 0, s>>>(items, work, n_work, counter);
    }
}

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
