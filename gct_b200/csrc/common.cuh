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

struct QuadF32 {
    using storage = float4;
    static __device__ __forceinline__ float4 load(const float4 *p) { return __ldg(p); }
    static __device__ __forceinline__ float4 unpack(float4 q) { return q; }
};

struct QuadF16 {
    using storage = uint2;  // four halves: (p00, p01) in .x, (p10, p11) in .y
    static __device__ __forceinline__ uint2 load(const uint2 *p) { return __ldg(p); }
    static __device__ __forceinline__ float4 unpack(uint2 q)
    {
        __half2 lo = *reinterpret_cast<__half2 *>(&q.x);
        __half2 hi = *reinterpret_cast<__half2 *>(&q.y);
        const float2 a = __half22float2(lo), b = __half22float2(hi);
        return make_float4(a.x, a.y, b.x, b.y);
    }
};

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

__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

}  // namespace gct
