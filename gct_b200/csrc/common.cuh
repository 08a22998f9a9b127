// Shared device helpers for the FDK kernels (sm_100a).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gct_fdk.h"
#include "kernels.hpp"

namespace gct {

// Filtered projections are stored as padded "quads": entry (r, c) of view v holds the four
// bilinear taps p[r][c], p[r][c+1], p[r+1][c], p[r+1][c+1] of the filtered projection, so one
// 16-byte (FP32) or 8-byte (FP16) load serves one bilinear sample. The quad grid is padded by
// kQuadPad entries on every side and the padding holds zeros, which reproduces the reference's
// border-0 texture addressing (src/cuda/data/nd_array_texture.cuh:33-56) without branches.
// The padding width is kQuadPad (kernels.hpp).

// Storage tags of the backprojector: FP32 quads (float4, quad_f32) and FP16 quads (uint2, quad_f16).
struct QuadF32 {
    using storage = float4;
};
struct QuadF16 {
    using storage = uint2;
};

// Quad of taps p00 = p[r][c], p01 = p[r][c+1], p10 = p[r+1][c], p11 = p[r+1][c+1] in the centred
// form: value = (A + fu B) + fc (C + fu D) with fu in [0, 1] and fc = f - 1/2 in [-1/2, 1/2]:
//   A = (p00 + p10) / 2, B = (p01 + p11 - p00 - p10) / 2, C = p10 - p00, D = p11 - p01 - p10 + p00.
// The centred fraction keeps the FP16 products small: emulated on ramp-filtered noisy rows, an
// offset form (fraction in [1, 2), one operation fewer per sample) had three times the FP16 error.
__device__ __forceinline__ float4 quad_f32(float p00, float p01, float p10, float p11)
{
    const float l = p00 + p10, r = p01 + p11;
    return make_float4(0.5f * l, 0.5f * (r - l), p10 - p00, (p11 - p01) - (p10 - p00));
}

// FP16 storage of the same quad: half2 (A, C) in .x and half2 (B, D) in .y.
__device__ __forceinline__ uint2 quad_f16_of(float4 q)
{
    const __half2 lo = __floats2half2_rn(q.x, q.z), hi = __floats2half2_rn(q.y, q.w);
    uint2 u;
    u.x = *reinterpret_cast<const unsigned *>(&lo);
    u.y = *reinterpret_cast<const unsigned *>(&hi);
    return u;
}
__device__ __forceinline__ uint2 quad_f16(float p00, float p01, float p10, float p11)
{
    return quad_f16_of(quad_f32(p00, p01, p10, p11));
}

// floor(x) and x - floor(x) for |x| < 2^22 with three FP32 adds and one integer subtract:
// round-half-even of (x - 0.5) via the 1.5 * 2^23 shifter. For an integer x the split may
// return (x - 1, 1.0), which gives the same bilinear value.
__device__ __forceinline__ void split_coord(float x, int &i, float &f)
{
    const float t = (x - 0.5f) + 12582912.0f;
    i = __float_as_int(t) - 0x4B400000;
    f = x - (t - 12582912.0f);
}

// Cosine pre-weight of pixel (c, r) of a view, per geometry (src/cuda/recon/cos_weighting.cuh:
// 16-153). c0/r0 are the view's detector centres, du/dv the sampler widths.
__device__ __forceinline__ float cos_weight_dev(int kind, float c0, float r0, float sdd, float du,
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

// cos_weight_dev along one detector row r, with the kind's row-invariant parts taken once:
// w(c) = R cos(u) (arc, cylindrical) or S / sqrt(U2 u^2 + B) (line, flat, cone-parallel, parallel),
// u = (c - c0) du. The same weights as cos_weight_dev up to the rounding of the hoisted terms.
struct RowWeight {
    bool arc;
    float c0, du, S, U2, B, R;
    __device__ __forceinline__ float at(int c) const
    {
        const float u = (static_cast<float>(c) - c0) * du;
        return arc ? R * cosf(u) : S * rsqrtf(fmaf(U2 * u, u, B));
    }
};
__device__ __forceinline__ RowWeight row_weight(int kind, float c0, float r0, float sdd, float du, float dv, int r)
{
    const float v = (static_cast<float>(r) - r0) * dv;
    RowWeight w{false, c0, du, 1.f, 0.f, 1.f, 1.f};
    switch (kind) {
        case GCT_GEOM_FAN_ARC: w.arc = true; break;
        case GCT_GEOM_FAN_LINE: w.S = sdd, w.U2 = 1.f, w.B = sdd * sdd; break;
        case GCT_GEOM_CONE_PARALLEL: w.S = sdd, w.B = v * v + sdd * sdd; break;
        case GCT_GEOM_CONE_CYL: w.arc = true, w.R = sdd * rsqrtf(v * v + sdd * sdd); break;
        case GCT_GEOM_CONE_FLAT: w.S = sdd, w.U2 = 1.f, w.B = v * v + sdd * sdd; break;
        default: break;  // parallel kinds: 1 / sqrt(1) = 1
    }
    return w;
}

__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

}  // namespace gct
