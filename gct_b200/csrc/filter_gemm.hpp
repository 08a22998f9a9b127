// Launch interfaces of the Toeplitz-GEMM ramp filter (filter_gemm.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace gct {

int gemm_pad_k(int n);  // K padded to the 64-column tile
int gemm_pad_n(int n);  // N padded to the 256-column tile
constexpr int kGemmBand = 64;  // |c - k| of the band of the four-term and FP16 forms
// Split forms of the Toeplitz GEMM (filter_gemm.cu): three BF16 terms, four BF16 terms (third
// pieces over the band), FP16 rows in two pieces with scaled rows and taps (lo and third tap
// pieces over the band).
enum GemmForm : int { kGemmF16x2 = 2, kGemmBf16x3 = 3, kGemmBf16x4 = 4 };
size_t toeplitz_gemm_smem_bytes();

struct SplitArgs {
    const float *proj = nullptr;  // [views][nr][nc], full stack
    long long row0 = 0;           // first global row (view * nr + row)
    long long rows = 0;
    int nr = 0, nc = 0, Kp = 0;
    int kind = 0;
    float du = 0.f, dv = 0.f;
    const float4 *fview = nullptr;
    const float *parker = nullptr;
    // 16-bit pieces [all rows][Kp]: BF16, or FP16 bit patterns when rinv is set
    __nv_bfloat16 *xh = nullptr, *xl = nullptr;
    __nv_bfloat16 *xll = nullptr;                // third piece (four-term GEMM), or NULL
    float *amax = nullptr;                       // per-view max |raw value| (zeroed by the caller), or NULL
    float *rinv = nullptr;                       // FP16 form: per-row 1 / (row scale x tap scale), [all rows]
    float tap_inv = 1.f;                         // FP16 form: 1 / tap scale (a power of two)
    // quarter-turn stacks (quad_layout's quarter > 0): the pieces and rinv of view v's row r go to
    // the partner-interleaved A row ((v mod quarter) nr + r) 4 + v div quarter (gemm_partner_row)
    int quarter = 0;
};
void launch_split(const SplitArgs &a, int num_sms, cudaStream_t s);

struct GemmLaunch {
    const __nv_bfloat16 *xh = nullptr, *xl = nullptr;  // A: [a_rows][Kp] (FP16 bit patterns in the FP16 form)
    const __nv_bfloat16 *xll = nullptr;                // third piece of A (four-term form)
    int form = kGemmBf16x3;
    long long a_rows = 0;
    const __nv_bfloat16 *th = nullptr, *tl = nullptr;  // B = T^T: [Np][Kp]
    const __nv_bfloat16 *tll = nullptr;                // third piece of B, central band (four-term, FP16 forms)
    const float *rinv = nullptr;                       // FP16 form: per-row inverse scale, [a_rows]
    int Np = 0, Kp = 0;
    int m_begin = 0, M = 0, N = 0;
    float *Y = nullptr;  // row m_begin + i at Y + i * ldy
    int ldy = 0;
    int *err = nullptr;
    // Quad output (quads set): instead of FP32 rows the epilogue writes FP16 quads, in
    // quad_layout order, into the stack `quads` (view 0 address) with the per-view scales vscale:
    // quarter > 0 (A rows partner-interleaved): base views [v_begin, v_begin + v_count) and their
    // three partners; quarter = 0: views [v_begin, v_begin + v_count) of a view-major stack (quad
    // pitch nc + 4 even). m_begin / M are then ignored (taken from the views).
    void *quads = nullptr;
    const float *vscale = nullptr;
    int quarter = 0, nr = 0, v_begin = 0, v_count = 0;
};
// A row of view v's detector row r in a partner-interleaved GEMM (quarter > 0).
__host__ __device__ inline long long gemm_partner_row(long long v, int r, int nr, int quarter)
{
    return ((v % quarter) * nr + r) * 4 + v / quarter;
}
cudaError_t launch_toeplitz_gemm(const GemmLaunch &g, int num_sms, cudaStream_t s);
// M tiles of a quad-epilogue GEMM over `positions` detector-row positions of P partner rows each
// (one CTA takes whole M tiles, so fewer tiles than SMs leave SMs idle).
long long gemm_quad_tiles(long long positions, int P);

struct QuadArgs {
    const float *Y = nullptr;  // filtered rows of views [v0, v0 + nv), row stride ldy
    int ldy = 0;
    int v0 = 0, nv = 0, nr = 0, nc = 0;
    const float *vscale = nullptr;
    void *out = nullptr;       // quads of the full stack
    int quarter = 0;           // quad_layout (kernels.hpp)
    int t1d = 0;               // one-row detector: transposed quad grid (kernels.hpp, kT1dPitch)
    int *err = nullptr;        // plan status word: kQuadWaitTimeout when a row copy timed out
};
constexpr int kQuadWaitTimeout = 0x200;
void launch_quads_from_rows(const QuadArgs &a, int mode, int num_sms, cudaStream_t s);
// Quarter-turn stacks: the partner groups of base views [v0, v0 + nv) (quarter = nv of the stack
// / 4), from rows of all views at their stack positions in Y.
void launch_quads_partners(const QuadArgs &a, int mode, int num_sms, cudaStream_t s);

}  // namespace gct
