// Ramp filter as a Toeplitz GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// The reference filters each detector row by FFT convolution (src/cuda/recon/ramp_filtering_fft.cuh:
// 208-219). A row convolution with N taps is also the product of the row with an N x N Toeplitz
// matrix T[k][c] = g(c - k), so a whole projection stack is one GEMM Y = X T with
// M = views x rows, K = N = detector columns, FP32 accumulation in TMEM. Three split forms:
//   * BF16, three terms: X = Xh + Xl, T = Th + Tl (BF16 hi/lo parts), Y = Xh Th + Xh Tl + Xl Th
//     (the dropped Xl Tl term is ~2^-16 relative).
//   * BF16, four terms: X = Xh + Xl + Xll, Y = Xh Th + Xh Tl + Xl Th + Xll Th + Xh Tll, where Tll
//     is kept for |c - k| <= kBand only, and the Xll Th term also runs over the K blocks of that
//     band only (Xll is rounding noise 2^-16 below the values, so the far taps add nothing it
//     carries).
//   * FP16, two pieces of the rows: each row scaled by a power of two so that its largest value
//     is below 2^14, the taps likewise, X = Xh + Xl and T = Th + Tl + Tll in FP16 pieces, and
//     Y = Xh Th + (Xh Tl + Xl Th + Xh Tll over the band). Away from the diagonal a tap is its FP16
//     hi piece alone; what that drops is added to the central tap of the same output column, so
//     every column's DC response is exact to FP32 rounding. One full K pass instead of three.
// Two BF16 pieces hold a value to about 2^-17 relative, and ramp filtering removes the large
// smooth part of a projection, so residuals of that part are a large fraction of the filtered
// value: the two-piece BF16 taps keep a DC response error of about 1e-6 that multiplies the smooth
// part of every view alike and adds up over views. Relative RMS in a 512^3 volume with noisy
// 720-view input: three BF16 terms 1.1e-3 and four 7.9e-5 with FP16 quads; of that the filter
// alone (FP64 emulation of the forms on the two central slices) 4.0e-5 for four BF16 terms and
// 4.1e-6 for the FP16 form. Stages:
//   1. split_kernel: cosine x Parker weighting fused into the load, split into pieces (FP16: with
//      the row's scale, written beside the pieces), zero padding of K to a multiple of 64;
//   2. toeplitz_gemm_kernel: persistent, warp-specialised tcgen05 GEMM. Warp 0 issues TMA loads of
//      128 x 64 A tiles and 256 x 64 B tiles (128B swizzle) into a 4-stage shared-memory ring;
//      one thread of warp 1 issues tcgen05.mma (M 128, N 256, K 16) into one of two TMEM
//      accumulators of 256 FP32 columns; warps 2-5 drain the other accumulator with tcgen05.ld and
//      store FP32 rows (FP16 form: times the row's inverse scale) or, for FP16 stacks, the
//      backprojector's bilinear-coefficient quads themselves (pq_epilogue: partner groups of
//      quarter-turn stacks from partner-interleaved A rows, or view-major quads). An output
//      tile's K loop is the full-K segments of its form followed by its band segments.
//   3. otherwise quads_rows_kernel / quads_from_rows_kernel: the filtered rows become the quads
//      (FP32, or FP16 with the per-view scale).
// Every mbarrier wait is bounded (2 s of %globaltimer); on timeout the kernel records an error
// code, stops issuing work, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include "../../include/gct_fdk.h"
#include "common.cuh"
#include "filter_gemm.hpp"

namespace gct {
namespace {

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 4, UMMA_K = 16;
constexpr int kBand = kGemmBand;  // taps with |c - k| <= kBand carry the band pieces
constexpr uint32_t A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int TMEM_COLS = 512;  // two accumulators of BN FP32 columns
constexpr unsigned long long kWaitNs = 2000000000ull;

// ---- small PTX wrappers --------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// Bounded wait for phase `parity` of barrier `bar`; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    const unsigned long long t0 = global_ns();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (global_ns() - t0 > kWaitNs) return false;
    }
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int c0, int c1, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major operand tile written by TMA with 128B swizzle: 8-row atoms of 128 B rows, atoms 1024 B
// apart (SBO), LBO unused (1), descriptor version 1, layout type 2 (128B swizzle).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr)
{
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (1ull << 16) | (static_cast<uint64_t>(1024 >> 4) << 32) |
           (1ull << 46) | (2ull << 61);
}
// kind::f16 instruction descriptors: FP32 accumulator, A and B of one type (format 1 in both
// fields for BF16, 0 for FP16), both K-major, M = 128, N = 256.
constexpr uint32_t kIdescF16 = (1u << 4) | (static_cast<uint32_t>(BN >> 3) << 17) | (static_cast<uint32_t>(BM >> 4) << 24);
constexpr uint32_t kIdescBF16 = kIdescF16 | (1u << 7) | (1u << 10);

__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

#define GCT_LD32(r, taddr)                                                                                       \
    asm volatile(                                                                                                \
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17," \
        "%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"                                      \
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),          \
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),    \
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),  \
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])   \
        : "r"(taddr))

struct GemmParams {
    int M;          // rows (views x detector rows)
    int N;          // valid output columns (detector columns)
    int m_begin;    // first row of this launch in the A tensor
    int num_kb;     // K / 64 (padded K)
    int m_tiles, n_tiles;
    float *Y;       // [M][ldy] FP32, row m_begin + i at Y + i * ldy
    int ldy;
    int form;       // GemmForm
    const float *rinv;  // FP16 form: per-row inverse scale, indexed like the A rows
    int *err;       // set non-zero on a timed-out wait
    // quad epilogue (pq = P, the partner views per position: 4 for quarter-turn stacks with
    // partner-interleaved A rows, 1 for view-major stacks): M tile mb starts at A row
    // m_begin + pq_stride(P) mb and covers pq_rows(P) + 1 detector-row positions (P rows each) of
    // views from v_begin (base views for P = 4), the last one only as the lower neighbour of the
    // one before; `positions` = (base) views x nr
    int pq;
    uint2 *quads;          // FP16 quads of the stack (view 0), quad_layout with `quarter` (P = 4) or 0
    const float *vscale;   // per-view power-of-two scale of the stored values
    int quarter, nr, qpitch, v_begin;
    long long qview, positions;
};

// Quad tiles: BM / P positions x P partner rows, consecutive tiles overlapping by one position, so
// every quad row's lower detector row lies in the same tile as its upper one.
__host__ __device__ constexpr int pq_rows(int P) { return BM / P - 1; }
__host__ __device__ constexpr int pq_stride(int P) { return P * pq_rows(P); }

// Tile i of this CTA: (A row of its first row, first output column, N tile index); false past the
// last. Row tiles: every tile of the grid in turn. Quad tiles: whole M blocks per CTA with their N
// tiles in order, so that one epilogue thread sees a row's columns left to right.
__device__ __forceinline__ bool tile_at(const GemmParams &p, int i, int &m0, int &n0, int &mb)
{
    if (p.pq) {
        mb = blockIdx.x + (i / p.n_tiles) * gridDim.x;
        if (mb >= p.m_tiles) return false;
        m0 = p.m_begin + mb * pq_stride(p.pq);
        n0 = (i % p.n_tiles) * BN;
        return true;
    }
    const long long t = blockIdx.x + static_cast<long long>(i) * gridDim.x;
    if (t >= static_cast<long long>(p.m_tiles) * p.n_tiles) return false;
    mb = static_cast<int>(t / p.n_tiles);
    m0 = p.m_begin + mb * BM;
    n0 = static_cast<int>(t % p.n_tiles) * BN;
    return true;
}

// K blocks of the band segments for the output tile starting at column n0: the rows k with
// |c - k| <= kBand for some c in [n0, n0 + BN).
__device__ __forceinline__ void band_blocks(const GemmParams &p, int n0, int &kb0, int &kb1)
{
    if (p.form == kGemmBf16x3) {
        kb0 = kb1 = 0;
        return;
    }
    kb0 = max(0, (n0 - kBand) / BK);
    kb1 = min(p.num_kb, (n0 + BN + kBand + BK - 1) / BK);
}

// Full-K segments of a form, and its band segments per band K block.
__device__ __forceinline__ int full_segments(int form) { return form == kGemmF16x2 ? 1 : 3; }
__device__ __forceinline__ int band_segments(int form) { return form == kGemmF16x2 ? 3 : form == kGemmBf16x4 ? 2 : 0; }

// Operands of K step ks of a tile: A piece (0 hi, 1 lo, 2 third) and B piece (likewise) and the K
// block. Segments, full K then band:
//   BF16 three/four terms: Xh Th, Xh Tl, Xl Th | Xll Th, Xh Tll
//   FP16:                  Xh Th               | Xh Tl, Xl Th, Xh Tll
__device__ __forceinline__ void step_operands(const GemmParams &p, int ks, int kb0, int nband, int &pa, int &pb,
                                              int &kb)
{
    const int kfull = full_segments(p.form) * p.num_kb;
    int seg;
    if (ks < kfull) {
        seg = ks / p.num_kb;
        kb = ks - seg * p.num_kb;
    } else {
        const int bs = ks - kfull;
        const int j = bs / nband;
        kb = kb0 + (bs - j * nband);
        seg = full_segments(p.form) + j;
    }
    if (p.form == kGemmF16x2) {
        pa = seg == 2 ? 1 : 0;
        pb = seg == 1 ? 1 : seg == 3 ? 2 : 0;
    } else {
        pa = seg == 2 ? 1 : seg == 3 ? 2 : 0;
        pb = seg == 1 ? 1 : seg == 4 ? 2 : 0;
    }
}

__device__ __forceinline__ void epilogue_bar() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Quad column cq of quad row r of one partner (entry base + P cq) from its corner values, with
// the zero rows around a view: row -1 (lower row = detector row 0) and -2 above the first detector
// row, rows nr and nr + 1 below the last.
template <int P>
__device__ __forceinline__ void pq_store(const GemmParams &p, long long base, int cq, float lt, float rt, float lb,
                                         float rb, bool first_row, bool last_row)
{
    uint2 *o = p.quads + base + static_cast<long long>(P) * cq;
    const long long row = static_cast<long long>(P) * p.qpitch;
    *o = quad_f16(lt, rt, lb, rb);
    if (first_row) {
        o[-row] = quad_f16(0.f, 0.f, lt, rt);
        o[-2 * row] = make_uint2(0u, 0u);
    }
    if (last_row) {
        o[row] = make_uint2(0u, 0u);
        o[2 * row] = make_uint2(0u, 0u);
    }
}

// Quad epilogue of the four epilogue warps (TMEM lane quadrant q). TMEM lane t of a tile holds
// position t / P (partner t % P) of the tile's pq_rows(P) + 1 positions. Per 32-column chunk each
// thread scales its row (FP16 row scale x view scale, both powers of two), takes the next detector
// row of its partner from lane + P (a shuffle, or for the last P lanes the next quadrant's first
// P lanes through shared memory), and writes the quads of its position. P = 4: lanes 4i..4i+3
// store one 32-byte partner group per quad column; P = 1: each thread stores its own quad row,
// two quads per 16-byte store. Quads at a chunk's left edge take their left corners from the
// previous chunk (the previous N tile of the same M block, same thread). Every decision to stop is
// voted by all four warps, so the named barriers stay matched. Returns false on a timed-out wait.
template <int P>
__device__ bool pq_epilogue(const GemmParams &p, uint32_t tmem_base, int q, int lane, uint32_t tfull0,
                            uint32_t tempty0, float4 (*s_x)[4][4][9], int (*s_stop)[4], const volatile int *fail_flag)
{
    constexpr int kRows = pq_rows(P);
    const int trow = q * 32 + lane, pl = trow / P, k = trow % P;
    int acc = 0, tile_i = 0;
    uint32_t aphase = 0;
    for (int mb = blockIdx.x; mb < p.m_tiles; mb += gridDim.x) {
        const long long pos = static_cast<long long>(kRows) * mb + pl;
        const bool have = pos < p.positions;
        const int vl = have ? static_cast<int>(pos / p.nr) : 0;
        const int r = have ? static_cast<int>(pos - static_cast<long long>(vl) * p.nr) : 0;
        const bool writer = have && pl < kRows;
        const bool first_row = r == 0, last_row = r == p.nr - 1;
        const long long b = static_cast<long long>(p.v_begin) + vl;  // base view (P = 4) or view
        float rs = 0.f;
        if (have) {
            const long long arow =
                static_cast<long long>(p.m_begin) + static_cast<long long>(pq_stride(P)) * mb + trow;
            rs = (p.rinv ? __ldg(p.rinv + arow) : 1.0f) * __ldg(p.vscale + b + static_cast<long long>(k) * p.quarter);
        }
        const long long base = (b * p.qview + static_cast<long long>(r + kQuadPad) * p.qpitch) * P + k;
        float ct = 0.f, cb = 0.f;    // column c0 - 1 of this row and of the next one
        float ct2 = 0.f, cb2 = 0.f;  // column c0 - 2 (P = 1)
        for (int nt = 0; nt < p.n_tiles; ++nt, ++tile_i) {
            const bool ok = mbar_wait(tfull0 + 8u * acc, aphase);
            if (lane == 0) s_stop[tile_i & 1][q] = (!ok || *fail_flag) ? 1 : 0;
            epilogue_bar();
            const int *vote = s_stop[tile_i & 1];
            if (vote[0] | vote[1] | vote[2] | vote[3]) return ok;
            tc_fence_after();
#pragma unroll 1
            for (int ch = 0; ch < BN / 32; ++ch) {
                uint32_t rr[32];
                const uint32_t taddr =
                    tmem_base + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(acc * BN + ch * 32);
                GCT_LD32(rr, taddr);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                const int c0 = nt * BN + ch * 32;
                float v[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = c0 + j < p.N ? rs * __uint_as_float(rr[j]) : 0.f;
                float4(*xb)[9] = s_x[ch & 1][q];
                if (lane < P) {
#pragma unroll
                    for (int j = 0; j < 8; ++j) xb[lane][j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
                }
                epilogue_bar();
                float bt[32];
                if (lane >= 32 - P) {
                    const float4(*nb)[9] = s_x[ch & 1][(q + 1) & 3];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const float4 t4 = nb[lane - (32 - P)][j];
                        bt[4 * j] = t4.x, bt[4 * j + 1] = t4.y, bt[4 * j + 2] = t4.z, bt[4 * j + 3] = t4.w;
                    }
                }
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const float d = __shfl_down_sync(0xffffffffu, v[j], P);
                    if (lane < 32 - P) bt[j] = d;
                    if (last_row) bt[j] = 0.f;
                }
                const int lim = p.N + 3;  // last quad column
                if (writer && P == 4) {
                    if (c0 == 0) pq_store<P>(p, base, 0, 0.f, 0.f, 0.f, 0.f, first_row, last_row);
                    if (c0 + 32 <= lim && !first_row && !last_row) {
                        // interior rows, whole chunk: quads of columns c0 - 1 .. c0 + 30, each sharing
                        // its left sums with the quad before (the quad_f32 operations, unchanged)
                        uint2 *o = p.quads + base + 4LL * (c0 + 1);
                        float lp = ct + cb, cp = cb - ct;
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const float l = v[j] + bt[j], cc = bt[j] - v[j];
                            o[4 * j] = quad_f16_of(make_float4(0.5f * lp, 0.5f * (l - lp), cp, cc - cp));
                            lp = l;
                            cp = cc;
                        }
                    } else {
                        if (c0 + 1 <= lim) pq_store<P>(p, base, c0 + 1, ct, v[0], cb, bt[0], first_row, last_row);
#pragma unroll
                        for (int j = 0; j < 31; ++j)
                            if (c0 + 2 + j <= lim)
                                pq_store<P>(p, base, c0 + 2 + j, v[j], v[j + 1], bt[j], bt[j + 1], first_row, last_row);
                    }
                } else if (writer) {
                    // P = 1: quad columns c0 .. c0 + 31 (detector columns c0 - 2 .. c0 + 30), so that a
                    // pair of quads starts on a 16-byte boundary
                    if (c0 + 31 <= lim && !first_row && !last_row) {
                        uint4 *o = reinterpret_cast<uint4 *>(p.quads + base + c0);
                        float lp = ct2 + cb2, cp = cb2 - ct2;  // column c0 - 2
                        float l1 = ct + cb, c1 = cb - ct;      // column c0 - 1
                        const uint2 q0 = quad_f16_of(make_float4(0.5f * lp, 0.5f * (l1 - lp), cp, c1 - cp));
                        const float l2 = v[0] + bt[0], c2 = bt[0] - v[0];
                        const uint2 q1 = quad_f16_of(make_float4(0.5f * l1, 0.5f * (l2 - l1), c1, c2 - c1));
                        o[0] = make_uint4(q0.x, q0.y, q1.x, q1.y);
                        lp = l2;
                        cp = c2;
#pragma unroll
                        for (int j = 1; j < 16; ++j) {
                            const float la = v[2 * j - 1] + bt[2 * j - 1], ca = bt[2 * j - 1] - v[2 * j - 1];
                            const float lb = v[2 * j] + bt[2 * j], cb_ = bt[2 * j] - v[2 * j];
                            const uint2 qa = quad_f16_of(make_float4(0.5f * lp, 0.5f * (la - lp), cp, ca - cp));
                            const uint2 qb = quad_f16_of(make_float4(0.5f * la, 0.5f * (lb - la), ca, cb_ - ca));
                            o[j] = make_uint4(qa.x, qa.y, qb.x, qb.y);
                            lp = lb;
                            cp = cb_;
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            if (c0 + j > lim) continue;
                            const float lt = j == 0 ? ct2 : j == 1 ? ct : v[j - 2];
                            const float lb = j == 0 ? cb2 : j == 1 ? cb : bt[j - 2];
                            const float rt = j == 0 ? ct : v[j - 1], rb = j == 0 ? cb : bt[j - 1];
                            pq_store<P>(p, base, c0 + j, lt, rt, lb, rb, first_row, last_row);
                        }
                    }
                }
                ct2 = v[30];
                cb2 = bt[30];
                ct = v[31];
                cb = bt[31];
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(tempty0 + 8u * acc);
            if (++acc == 2) {
                acc = 0;
                aphase ^= 1;
            }
        }
        // quad columns past the last tile (the tile's last detector columns and the zero padding)
        if (writer) {
            const int np = p.n_tiles * BN;
            for (int cq = P == 4 ? np + 1 : np; cq <= p.N + 3; ++cq) {
                const int c = cq - 2;  // left detector column of the quad
                const float lt = c == np - 2 ? ct2 : c == np - 1 ? ct : 0.f;
                const float lb = c == np - 2 ? cb2 : c == np - 1 ? cb : 0.f;
                const float rt = c == np - 2 ? ct : 0.f, rb = c == np - 2 ? cb : 0.f;
                pq_store<P>(p, base, cq, lt, rt, lb, rb, first_row, last_row);
            }
        }
    }
    return true;
}

__global__ void __launch_bounds__(192, 1)
    toeplitz_gemm_kernel(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                         const __grid_constant__ CUtensorMap mAll, const __grid_constant__ CUtensorMap mBh,
                         const __grid_constant__ CUtensorMap mBl, const __grid_constant__ CUtensorMap mBll,
                         GemmParams p)
{
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
    // bars: full[STAGES], empty[STAGES], tfull[2], tempty[2]; then the TMEM base address
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * STAGES + 4);
    __shared__ int s_fail;
    const volatile int *fail_flag = &s_fail;  // re-read on every loop test
    // quad epilogue: the first P rows' values of each TMEM lane quadrant (two buffers) and the
    // per-tile stop votes of the four epilogue warps (two buffers)
    __shared__ float4 s_x[2][4][4][9];
    __shared__ int s_stop[2][4];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto full = [&](int s) { return smem_u32(bars + s); };
    auto empty = [&](int s) { return smem_u32(bars + STAGES + s); };
    auto tfull = [&](int a) { return smem_u32(bars + 2 * STAGES + a); };
    auto tempty = [&](int a) { return smem_u32(bars + 2 * STAGES + 2 + a); };

    if (threadIdx.x == 0) {
        s_fail = 0;
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(tfull(a), 1);
            mbar_init(tempty(a), 4);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int kfull = full_segments(p.form) * p.num_kb, nbseg = band_segments(p.form);
    const uint32_t idesc = p.form == kGemmF16x2 ? kIdescF16 : kIdescBF16;

    if (warp == 0) {
        if (lane == 0) {  // TMA producer
            int stage = 0;
            uint32_t phase = 0;
            int m0, n0, mb;
            for (int i = 0; tile_at(p, i, m0, n0, mb) && !*fail_flag; ++i) {
                int kb0, kb1;
                band_blocks(p, n0, kb0, kb1);
                const int nband = kb1 - kb0;
                const int ksteps = kfull + nbseg * nband;
                for (int ks = 0; ks < ksteps; ++ks) {
                    int pa, pb, kb;
                    step_operands(p, ks, kb0, nband, pa, pb, kb);
                    if (!mbar_wait(empty(stage), phase ^ 1)) {
                        atomicExch(&s_fail, 1);
                        break;
                    }
                    mbar_expect_tx(full(stage), STAGE_BYTES);
                    const uint32_t sa = smem_u32(smem + stage * STAGE_BYTES);
                    tma_load_2d(sa, pa == 2 ? &mAll : pa == 1 ? &mAl : &mAh, kb * BK, m0, full(stage));
                    tma_load_2d(sa + A_BYTES, pb == 2 ? &mBll : pb == 1 ? &mBl : &mBh, kb * BK, n0, full(stage));
                    if (++stage == STAGES) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            int stage = 0, acc = 0;
            uint32_t phase = 0, aphase = 0;
            int m0, n0, mb;
            for (int i = 0; tile_at(p, i, m0, n0, mb) && !*fail_flag; ++i) {
                if (!mbar_wait(tempty(acc), aphase ^ 1)) {
                    atomicExch(&s_fail, 2);
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem_base + static_cast<uint32_t>(acc * BN);
                int kb0, kb1;
                band_blocks(p, n0, kb0, kb1);
                const int ksteps = kfull + nbseg * (kb1 - kb0);
                bool ok = true;
                for (int ks = 0; ks < ksteps; ++ks) {
                    if (!mbar_wait(full(stage), phase)) {
                        atomicExch(&s_fail, 3);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = smem_u32(smem + stage * STAGE_BYTES);
                    const uint64_t da = smem_desc(sa), db = smem_desc(sa + A_BYTES);
#pragma unroll
                    for (int k = 0; k < BK / UMMA_K; ++k)  // +32 B along K per step: +2 in the address field
                        umma(d, da + 2 * k, db + 2 * k, idesc, (ks > 0 || k > 0) ? 1u : 0u);
                    umma_commit(empty(stage));
                    if (++stage == STAGES) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
                if (!ok) break;
                umma_commit(tfull(acc));
                if (++acc == 2) {
                    acc = 0;
                    aphase ^= 1;
                }
            }
        }
    } else if (p.pq) {  // epilogue warps 2..5, partner quads
        const int q = warp & 3;
        const bool ok = p.pq == 4 ? pq_epilogue<4>(p, tmem_base, q, lane, tfull(0), tempty(0), s_x, s_stop, fail_flag)
                                  : pq_epilogue<1>(p, tmem_base, q, lane, tfull(0), tempty(0), s_x, s_stop, fail_flag);
        if (!ok) atomicExch(&s_fail, 4);
    } else {  // epilogue warps 2..5: TMEM lane quadrant (warp % 4)
        const int q = warp & 3;
        int acc = 0;
        uint32_t aphase = 0;
        int m0, n0, mt;
        for (int i = 0; tile_at(p, i, m0, n0, mt) && !*fail_flag; ++i) {
            if (!mbar_wait(tfull(acc), aphase)) {
                atomicExch(&s_fail, 4);
                break;
            }
            tc_fence_after();
            const int row = mt * BM + q * 32 + lane;  // relative to m_begin
            float *yrow = p.Y + static_cast<long long>(row) * p.ldy;
            // FP16 form: undo the row and tap scales (powers of two, exact); 1 otherwise
            const float rs = (p.rinv && row < p.M) ? __ldg(p.rinv + p.m_begin + row) : 1.0f;
#pragma unroll 1
            for (int ch = 0; ch < BN / 32; ++ch) {
                uint32_t r[32];
                const uint32_t taddr = tmem_base + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(acc * BN + ch * 32);
                GCT_LD32(r, taddr);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                const int c0 = n0 + ch * 32;
                if (row < p.M) {
                    if (c0 + 32 <= p.N && (p.ldy & 3) == 0) {
                        float4 *dst = reinterpret_cast<float4 *>(yrow + c0);
#pragma unroll
                        for (int j = 0; j < 8; ++j)
                            dst[j] = make_float4(rs * __uint_as_float(r[4 * j]), rs * __uint_as_float(r[4 * j + 1]),
                                                 rs * __uint_as_float(r[4 * j + 2]), rs * __uint_as_float(r[4 * j + 3]));
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (c0 + j < p.N) yrow[c0 + j] = rs * __uint_as_float(r[j]);
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(tempty(acc));
            if (++acc == 2) {
                acc = 0;
                aphase ^= 1;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && s_fail) atomicExch(p.err, s_fail);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS) : "memory");
    }
}

// Cosine x Parker weighting and split of rows [row0, row0 + rows) into [rows][Kp]: two or three
// BF16 pieces per value, or (rinv set) two FP16 pieces of the value times the row's power-of-two
// scale, whose inverse times the tap scale's goes to rinv[row]. One warp per row (per-row
// view/row indices and geometry), four columns per lane step (one 16-byte load when rows are
// 16-byte aligned) stored as 8-byte words of four 16-bit pieces.
// With `amax`, the row's largest raw |p| also goes into amax[view] (atomic max of the bit
// pattern, non-negative floats), which replaces the separate view-maximum pass.
__device__ __forceinline__ uint2 bf16x4(float a, float b, float c, float d)
{
    const __nv_bfloat162 lo = __floats2bfloat162_rn(a, b), hi = __floats2bfloat162_rn(c, d);
    uint2 u;
    u.x = *reinterpret_cast<const unsigned *>(&lo);
    u.y = *reinterpret_cast<const unsigned *>(&hi);
    return u;
}
__device__ __forceinline__ float bf16_lo(unsigned w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(unsigned w) { return __uint_as_float(w & 0xffff0000u); }

// Weighted values x of columns [k, k + 4) of one row (zero beyond nc); m takes the max |raw|.
__device__ __forceinline__ void weighted4(const SplitArgs &a, const float *src, const float *pk, const RowWeight &rw,
                                          int k, bool vec, float (&x)[4], float &m)
{
    float raw[4], pw[4];
    if (vec && k + 3 < a.nc) {
        const float4 p4 = __ldg(reinterpret_cast<const float4 *>(src + k));
        const float4 w4 = __ldg(reinterpret_cast<const float4 *>(pk + k));
        raw[0] = p4.x, raw[1] = p4.y, raw[2] = p4.z, raw[3] = p4.w;
        pw[0] = w4.x, pw[1] = w4.y, pw[2] = w4.z, pw[3] = w4.w;
    } else {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const bool in = k + h < a.nc;
            raw[h] = in ? __ldg(src + k + h) : 0.f;
            pw[h] = in ? __ldg(pk + k + h) : 0.f;
        }
    }
#pragma unroll
    for (int h = 0; h < 4; ++h) {
        m = fmaxf(m, fabsf(raw[h]));
        x[h] = raw[h] * pw[h] * rw.at(k + h);
    }
}

__device__ __forceinline__ uint2 f16x4(float a, float b, float c, float d)
{
    const __half2 lo = __floats2half2_rn(a, b), hi = __floats2half2_rn(c, d);
    uint2 u;
    u.x = *reinterpret_cast<const unsigned *>(&lo);
    u.y = *reinterpret_cast<const unsigned *>(&hi);
    return u;
}

// Power-of-two scale that puts a row's largest |x| (xm, warp-uniform) in [2^13, 2^14); the row's
// 1 / (row scale x tap scale) goes to rinv[row].
__device__ __forceinline__ float row_scale_f16(const SplitArgs &a, long long row, float xm, int lane)
{
    int e = 0;
    if (xm > 0.f) frexpf(xm, &e);  // xm < 2^e
    const int sh = xm > 0.f ? min(100, max(-100, 14 - e)) : 0;
    if (lane == 0) a.rinv[row] = ldexpf(a.tap_inv, -sh);
    return ldexpf(1.0f, sh);
}

// x (already scaled) -> two FP16 pieces, stored at word k4 of the row
__device__ __forceinline__ void store_f16_pieces(const float (&x)[4], uint2 *dh, uint2 *dl, int k4)
{
    const uint2 hi = f16x4(x[0], x[1], x[2], x[3]);
    dh[k4] = hi;
    const __half2 h01 = *reinterpret_cast<const __half2 *>(&hi.x), h23 = *reinterpret_cast<const __half2 *>(&hi.y);
    // exact in FP32: x and its FP16 rounding are within one FP16 ulp
    dl[k4] = f16x4(x[0] - __low2float(h01), x[1] - __high2float(h01), x[2] - __low2float(h23), x[3] - __high2float(h23));
}

// One row of the FP16 form. NCH > 0 (rows of a multiple of 4 columns): every 16-byte load of the
// row is issued first (NCH words of four columns per lane, Kp <= 128 NCH) and the weighted values
// stay in registers between finding the row maximum and splitting; NCH == 0: two passes over the
// row, the second recomputing the weighted values.
template <int NCH>
__device__ __forceinline__ void split_f16_row(const SplitArgs &a, long long row, const float *src, const float *pk,
                                              const RowWeight &rw, bool vec, uint2 *dh, uint2 *dl, int lane, float &m)
{
    const int nk4 = a.Kp / 4;
    float xm = 0.f;
    if constexpr (NCH > 0) {
        float4 p4[NCH], w4[NCH];
#pragma unroll
        for (int c = 0; c < NCH; ++c) {  // columns past nc (K padding) read as zero
            const int k = 4 * (lane + 32 * c);
            const bool in = k < a.nc;
            p4[c] = in ? __ldg(reinterpret_cast<const float4 *>(src + k)) : make_float4(0.f, 0.f, 0.f, 0.f);
            w4[c] = in ? __ldg(reinterpret_cast<const float4 *>(pk + k)) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        float x[NCH][4];
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            const int k = 4 * (lane + 32 * c);
            const float raw[4] = {p4[c].x, p4[c].y, p4[c].z, p4[c].w}, pw[4] = {w4[c].x, w4[c].y, w4[c].z, w4[c].w};
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                m = fmaxf(m, fabsf(raw[h]));
                x[c][h] = raw[h] * pw[h] * rw.at(k + h);
                xm = fmaxf(xm, fabsf(x[c][h]));
            }
        }
        for (int o = 16; o > 0; o >>= 1) xm = fmaxf(xm, __shfl_xor_sync(0xffffffffu, xm, o));
        const float sc = row_scale_f16(a, row, xm, lane);
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            const int k4 = lane + 32 * c;
            if (k4 < nk4) {
#pragma unroll
                for (int h = 0; h < 4; ++h) x[c][h] *= sc;
                store_f16_pieces(x[c], dh, dl, k4);
            }
        }
    } else {
        for (int k4 = lane; k4 < nk4; k4 += 32) {
            float x[4];
            weighted4(a, src, pk, rw, 4 * k4, vec, x, m);
#pragma unroll
            for (int h = 0; h < 4; ++h) xm = fmaxf(xm, fabsf(x[h]));
        }
        for (int o = 16; o > 0; o >>= 1) xm = fmaxf(xm, __shfl_xor_sync(0xffffffffu, xm, o));
        const float sc = row_scale_f16(a, row, xm, lane);
        for (int k4 = lane; k4 < nk4; k4 += 32) {
            float x[4], mm = 0.f;
            weighted4(a, src, pk, rw, 4 * k4, vec, x, mm);
#pragma unroll
            for (int h = 0; h < 4; ++h) x[h] *= sc;
            store_f16_pieces(x, dh, dl, k4);
        }
    }
}

// NCH < 0: BF16 pieces; NCH >= 0: FP16 pieces (split_f16_row<NCH>), one instance per register
// footprint.
template <int NCH>
__global__ void split_kernel(SplitArgs a)
{
    const int lane = threadIdx.x & 31;
    const long long warp0 = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
    const bool vec = (a.nc & 3) == 0;
    for (long long rl = warp0; rl < a.rows; rl += nwarps) {
        const long long row = a.row0 + rl;
        const int v = static_cast<int>(row / a.nr), r = static_cast<int>(row - static_cast<long long>(v) * a.nr);
        const long long arow = a.quarter ? gemm_partner_row(v, r, a.nr, a.quarter) : row;  // A row
        const float4 gv = __ldg(&a.fview[v]);
        const RowWeight rw = row_weight(a.kind, gv.x, gv.y, gv.z, a.du, a.dv, r);
        const float *src = a.proj + row * a.nc;
        const float *pk = a.parker + static_cast<long long>(v) * a.nc;
        uint2 *dh = reinterpret_cast<uint2 *>(a.xh + arow * a.Kp);
        uint2 *dl = reinterpret_cast<uint2 *>(a.xl + arow * a.Kp);
        uint2 *dll = a.xll ? reinterpret_cast<uint2 *>(a.xll + arow * a.Kp) : nullptr;
        float m = 0.f;
        if (NCH >= 0) {
            split_f16_row<(NCH > 0 ? NCH : 0)>(a, arow, src, pk, rw, vec, dh, dl, lane, m);
        } else {
            for (int k4 = lane; k4 < a.Kp / 4; k4 += 32) {
                float x[4];
                weighted4(a, src, pk, rw, 4 * k4, vec, x, m);
                const uint2 hi = bf16x4(x[0], x[1], x[2], x[3]);
                dh[k4] = hi;
                const float r0 = x[0] - bf16_lo(hi.x), r1 = x[1] - bf16_hi(hi.x);  // exact in FP32
                const float r2 = x[2] - bf16_lo(hi.y), r3 = x[3] - bf16_hi(hi.y);
                const uint2 lo = bf16x4(r0, r1, r2, r3);
                dl[k4] = lo;
                if (dll)
                    dll[k4] = bf16x4(r0 - bf16_lo(lo.x), r1 - bf16_hi(lo.x), r2 - bf16_lo(lo.y), r3 - bf16_hi(lo.y));
            }
        }
        if (a.amax) {
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (lane == 0) atomicMax(reinterpret_cast<int *>(a.amax + v), __float_as_int(m));
        }
    }
}

// Filtered rows Y (row stride ldy) of views [v0, v0 + nv) -> bilinear-coefficient quads. One
// block per quad row (view, padded row), threads along the columns.
// One-row detector: each view's filtered row -> its transposed quad grid, one thread per entry.
template <int MODE>
__global__ void quads_t1d_kernel(QuadArgs a)
{
    const int rows = a.nc + 2 * kQuadPad;
    const long long n = static_cast<long long>(a.nv) * rows * kT1dPitch;
    for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
         e += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int vl = static_cast<int>(e / (rows * kT1dPitch));
        const int rem = static_cast<int>(e - static_cast<long long>(vl) * rows * kT1dPitch);
        const int r = rem / kT1dPitch - kQuadPad, c = rem % kT1dPitch - kQuadPad;
        const int v = a.v0 + vl;
        const float sc = a.vscale ? a.vscale[v] : 1.0f;
        const float *y = a.Y + static_cast<long long>(vl) * a.ldy;
        const float t = (r >= 0 && r < a.nc) ? sc * __ldg(y + r) : 0.f;
        const float b = (r + 1 >= 0 && r + 1 < a.nc) ? sc * __ldg(y + r + 1) : 0.f;
        const float p00 = c == 0 ? t : 0.f, p01 = c == -1 ? t : 0.f;
        const float p10 = c == 0 ? b : 0.f, p11 = c == -1 ? b : 0.f;
        const long long q = static_cast<long long>(v) * rows * kT1dPitch + rem;
        if (MODE == kOutQuadF32)
            static_cast<float4 *>(a.out)[q] = quad_f32(p00, p01, p10, p11);
        else
            static_cast<uint2 *>(a.out)[q] = quad_f16(p00, p01, p10, p11);
    }
}

template <int MODE>
__global__ void quads_from_rows_kernel(QuadArgs a)
{
    const int qpitch = a.nc + 2 * kQuadPad, qrows = a.nr + 2 * kQuadPad;
    const long long nrows = static_cast<long long>(a.nv) * qrows;
    for (long long qr = blockIdx.x; qr < nrows; qr += gridDim.x) {
        const int vl = static_cast<int>(qr / qrows);
        const int r = static_cast<int>(qr - static_cast<long long>(vl) * qrows) - kQuadPad;
        const int v = a.v0 + vl;
        const float sc = a.vscale ? a.vscale[v] : 1.0f;
        const float *top = (r >= 0 && r < a.nr) ? a.Y + (static_cast<long long>(vl) * a.nr + r) * a.ldy : nullptr;
        const float *bot = (r + 1 >= 0 && r + 1 < a.nr) ? a.Y + (static_cast<long long>(vl) * a.nr + r + 1) * a.ldy : nullptr;
        long long first;
        int step;
        quad_layout(v, static_cast<long long>(qrows) * qpitch, a.quarter, first, step);
        const long long qbase = first + static_cast<long long>(r + kQuadPad) * qpitch * step;
        for (int cq = threadIdx.x; cq < qpitch; cq += blockDim.x) {
            const int c = cq - kQuadPad;
            const bool c0 = c >= 0 && c < a.nc, c1 = c + 1 >= 0 && c + 1 < a.nc;
            const float p00 = (top && c0) ? sc * __ldg(top + c) : 0.f, p01 = (top && c1) ? sc * __ldg(top + c + 1) : 0.f;
            const float p10 = (bot && c0) ? sc * __ldg(bot + c) : 0.f, p11 = (bot && c1) ? sc * __ldg(bot + c + 1) : 0.f;
            const long long at = qbase + static_cast<long long>(cq) * step;
            if (MODE == kOutQuadF32)
                static_cast<float4 *>(a.out)[at] = quad_f32(p00, p01, p10, p11);
            else
                static_cast<uint2 *>(a.out)[at] = quad_f16(p00, p01, p10, p11);
        }
    }
}

// Quarter-turn stacks (quad_layout with quarter > 0): quads of base views [v0, v0 + nv) and their
// three partners from the filtered rows of all four (Y holds view v's row r at row v * nr + r).
// One block per (base view, padded row); each thread writes the whole group of four partner quads
// of one detector position (32 or 64 contiguous bytes), so the stores stay coalesced.
template <int MODE>
__global__ void quads_partners_kernel(QuadArgs a)
{
    const int qpitch = a.nc + 2 * kQuadPad, qrows = a.nr + 2 * kQuadPad;
    const long long nrows = static_cast<long long>(a.nv) * qrows;
    const long long qview = static_cast<long long>(qrows) * qpitch;
    for (long long qr = blockIdx.x; qr < nrows; qr += gridDim.x) {
        const int bl = static_cast<int>(qr / qrows);
        const int r = static_cast<int>(qr - static_cast<long long>(bl) * qrows) - kQuadPad;
        const int b = a.v0 + bl;
        const float *top[4], *bot[4];
        float sc[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const long long v = b + static_cast<long long>(q) * a.quarter;
            sc[q] = a.vscale ? a.vscale[v] : 1.0f;
            top[q] = (r >= 0 && r < a.nr) ? a.Y + (v * a.nr + r) * a.ldy : nullptr;
            bot[q] = (r + 1 >= 0 && r + 1 < a.nr) ? a.Y + (v * a.nr + r + 1) * a.ldy : nullptr;
        }
        const long long gbase = (static_cast<long long>(b) * qview + static_cast<long long>(r + kQuadPad) * qpitch) * 4;
        for (int cq = threadIdx.x; cq < qpitch; cq += blockDim.x) {
            const int c = cq - kQuadPad;
            const bool c0 = c >= 0 && c < a.nc, c1 = c + 1 >= 0 && c + 1 < a.nc;
            float4 g[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float p00 = (top[q] && c0) ? sc[q] * __ldg(top[q] + c) : 0.f;
                const float p01 = (top[q] && c1) ? sc[q] * __ldg(top[q] + c + 1) : 0.f;
                const float p10 = (bot[q] && c0) ? sc[q] * __ldg(bot[q] + c) : 0.f;
                const float p11 = (bot[q] && c1) ? sc[q] * __ldg(bot[q] + c + 1) : 0.f;
                g[q] = quad_f32(p00, p01, p10, p11);
            }
            const long long at = gbase + static_cast<long long>(cq) * 4;
            if (MODE == kOutQuadF32) {
                float4 *o = static_cast<float4 *>(a.out) + at;
#pragma unroll
                for (int q = 0; q < 4; ++q) o[q] = g[q];
            } else {
                uint2 h[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) h[q] = quad_f16_of(g[q]);
                uint4 *o = reinterpret_cast<uint4 *>(static_cast<uint2 *>(a.out) + at);
                o[0] = make_uint4(h[0].x, h[0].y, h[1].x, h[1].y);
                o[1] = make_uint4(h[2].x, h[2].y, h[3].x, h[3].y);
            }
        }
    }
}

// Quads from filtered FP32 rows, rolling form: a block takes (group b, segment of quad rows
// [q0, q1)); a group is P views (P = 1: view b of the launch; P = 4: base view v0 + b and its three
// quarter-turn partners, written as interleaved partner groups). Quad row q needs detector rows q
// and q + 1, so the block keeps three shared rows per view and has one thread copy each new row
// (cp.async.bulk, completion on the slot's mbarrier) while the current quad row is formed: every
// filtered row is read once per segment instead of twice. Rows outside the detector are zeros
// (no copy). Needs rows that start on 16-byte boundaries and hold a multiple of four floats; every
// wait is bounded (2 s): on a timeout the block sets kQuadWaitTimeout in a.err, waits (bounded) for
// its copies in flight and returns.
template <int MODE, int P>
__global__ void __launch_bounds__(256) quads_rows_kernel(QuadArgs a, int seg, int nseg)
{
    extern __shared__ __align__(16) unsigned char qsmem[];
    uint64_t *qbars = reinterpret_cast<uint64_t *>(qsmem);        // one mbarrier per slot
    const int rp = a.nc + 8;                                       // 4 zeros, nc values, 4 zeros
    float *rows = reinterpret_cast<float *>(qsmem + 32);           // [3 slots][P][rp]
    const int t = threadIdx.x, nt = blockDim.x;
    for (int e = t; e < 3 * P * rp; e += nt) rows[e] = 0.f;
    if (t == 0) {
        for (int k = 0; k < 3; ++k) mbar_init(smem_u32(qbars + k), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int qpitch = a.nc + 2 * kQuadPad, qrows = a.nr + 2 * kQuadPad;
    const long long qview = static_cast<long long>(qrows) * qpitch;
    const long long items = static_cast<long long>(a.nv) * nseg;
    const uint32_t row_bytes = static_cast<uint32_t>(a.nc) * 4u;
    // per slot (uniform over the block): copies completed so far (phase parity), row in the slot is zero
    int done[3] = {0, 0, 0};
    bool zero[3] = {true, true, true};
    int inflight = 0, inflight_slot[3] = {0, 0, 0};
    auto slot_of = [](int r) { return ((r % 3) + 3) % 3; };
    // Y row of view k of group b at detector row r
    auto yrow = [&](long long b, int k, int r) -> const float * {
        const long long v = P == 1 ? b : a.v0 + b + static_cast<long long>(k) * a.quarter;
        return a.Y + (v * a.nr + r) * static_cast<long long>(a.ldy);
    };
    auto issue = [&](long long b, int r) {
        const int sl = slot_of(r);
        zero[sl] = r < 0 || r >= a.nr;
        if (zero[sl]) return;
        if (t == 0) {
            const uint32_t bar = smem_u32(qbars + sl);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(bar, row_bytes * P);
#pragma unroll
            for (int k = 0; k < P; ++k)
                asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                             ::"r"(smem_u32(rows + (sl * P + k) * rp + 4)), "l"(yrow(b, k, r)), "r"(row_bytes),
                             "r"(bar)
                             : "memory");
        }
        inflight_slot[inflight++] = sl;
    };
    // waits for the copy into slot sl; false on timeout (uniform over the block)
    auto wait_slot = [&](int sl) -> bool {
        if (zero[sl]) return true;
        const bool ok = mbar_wait(smem_u32(qbars + sl), static_cast<uint32_t>(done[sl] & 1));
        if (ok) {
            ++done[sl];
            for (int k = 0; k < inflight; ++k)
                if (inflight_slot[k] == sl) {
                    inflight_slot[k] = inflight_slot[--inflight];
                    break;
                }
        }
        return !__syncthreads_or(!ok);
    };
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
        const long long b = it / nseg;
        const int q0 = -kQuadPad + static_cast<int>(it - b * nseg) * seg, q1 = min(q0 + seg, a.nr + kQuadPad);
        float scl[P];
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const long long v = P == 1 ? a.v0 + b : a.v0 + b + static_cast<long long>(k) * a.quarter;
            scl[k] = a.vscale ? a.vscale[v] : 1.0f;
        }
        long long first;
        int step;
        if (P == 1) quad_layout(a.v0 + b, qview, a.quarter, first, step);
        else first = (a.v0 + b) * qview * 4, step = 4;
        issue(b, q0);
        issue(b, q0 + 1);
        for (int q = q0; q < q1; ++q) {
            const bool ok = (q == q0 ? wait_slot(slot_of(q)) : true) && wait_slot(slot_of(q + 1));
            if (!ok) {
                if (t == 0) {
                    atomicOr(a.err, kQuadWaitTimeout);
                    for (int k = 0; k < inflight; ++k) {
                        const int sl = inflight_slot[k];
                        mbar_wait(smem_u32(qbars + sl), static_cast<uint32_t>(done[sl] & 1));
                        ++done[sl];
                    }
                }
                __syncthreads();
                return;
            }
            if (q + 2 <= q1) issue(b, q + 2);  // into the slot of row q - 1, read by the previous quad row
            const int st = slot_of(q), sb = slot_of(q + 1);
            const bool zt = zero[st], zb = zero[sb];
            const long long qbase = first + static_cast<long long>(q + kQuadPad) * qpitch * step;
            for (int cq = t; cq < qpitch; cq += nt) {
                const int c = cq - kQuadPad;  // shared index c + 4: columns -2 .. nc + 2 fall on zeros outside
                float4 g[P];
#pragma unroll
                for (int k = 0; k < P; ++k) {
                    const float *top = rows + (st * P + k) * rp + 4, *bot = rows + (sb * P + k) * rp + 4;
                    const float p00 = zt ? 0.f : scl[k] * top[c], p01 = zt ? 0.f : scl[k] * top[c + 1];
                    const float p10 = zb ? 0.f : scl[k] * bot[c], p11 = zb ? 0.f : scl[k] * bot[c + 1];
                    g[k] = quad_f32(p00, p01, p10, p11);
                }
                if constexpr (P == 4) {
                    const long long at = qbase + static_cast<long long>(cq) * 4;
                    if (MODE == kOutQuadF32) {
                        float4 *o = static_cast<float4 *>(a.out) + at;
#pragma unroll
                        for (int k = 0; k < 4; ++k) o[k] = g[k];
                    } else {
                        uint2 h[4];
#pragma unroll
                        for (int k = 0; k < 4; ++k) h[k] = quad_f16_of(g[k]);
                        uint4 *o = reinterpret_cast<uint4 *>(static_cast<uint2 *>(a.out) + at);
                        o[0] = make_uint4(h[0].x, h[0].y, h[1].x, h[1].y);
                        o[1] = make_uint4(h[2].x, h[2].y, h[3].x, h[3].y);
                    }
                } else {
                    const long long at = qbase + static_cast<long long>(cq) * step;
                    if (MODE == kOutQuadF32) static_cast<float4 *>(a.out)[at] = g[0];
                    else static_cast<uint2 *>(a.out)[at] = quad_f16_of(g[0]);
                }
            }
            __syncthreads();  // the slot of row q is rewritten by the copy issued in the next quad row
        }
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *ptr = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    }
    return fn;
}

// 2D 16-bit tensor [rows][cols] (cols contiguous), box cols_box x rows_box, 128B swizzle.
bool make_map(CUtensorMap *m, CUtensorMapDataType dt, const void *base, unsigned long long rows,
              unsigned long long cols, unsigned rows_box)
{
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {cols, rows};
    const cuuint64_t strides[1] = {cols * 2};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(BK), rows_box};
    const cuuint32_t estr[2] = {1, 1};
    return fn(m, dt, 2, const_cast<void *>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

long long gemm_quad_tiles(long long positions, int P) { return (positions + pq_rows(P) - 1) / pq_rows(P); }
int gemm_pad_k(int n) { return (n + BK - 1) / BK * BK; }
int gemm_pad_n(int n) { return (n + BN - 1) / BN * BN; }
size_t toeplitz_gemm_smem_bytes() { return STAGES * STAGE_BYTES + 1024 + 256; }

void launch_split(const SplitArgs &a, int num_sms, cudaStream_t s)
{
    long long grid = (a.rows + 7) / 8;  // 8 warps (rows) per block
    if (grid > static_cast<long long>(num_sms) * 16) grid = static_cast<long long>(num_sms) * 16;
    const unsigned g = static_cast<unsigned>(grid < 1 ? 1 : grid);
    const bool vec = (a.nc & 3) == 0;
    if (!a.rinv) split_kernel<-1><<<g, 256, 0, s>>>(a);
    else if (vec && a.Kp <= 128 * 8) split_kernel<8><<<g, 256, 0, s>>>(a);
    else if (vec && a.Kp <= 128 * 16) split_kernel<16><<<g, 256, 0, s>>>(a);
    else split_kernel<0><<<g, 256, 0, s>>>(a);
}

namespace {
// The rolling kernel, when every row starts on a 16-byte boundary (rows of a multiple of four floats
// from an aligned base) and a.err is set; false when it does not apply.
template <int P>
bool launch_quads_rows(const QuadArgs &a, int mode, int num_sms, cudaStream_t s)
{
    if (a.nc % 4 != 0 || a.ldy % 4 != 0 || reinterpret_cast<uintptr_t>(a.Y) % 16 != 0 || !a.err || a.nv <= 0)
        return false;
    const int seg = 32;
    const int nseg = (a.nr + 2 * kQuadPad + seg - 1) / seg;
    const size_t smem = 32 + 3 * static_cast<size_t>(P) * (a.nc + 8) * sizeof(float);
    if (smem > 200 * 1024) return false;
    long long grid = static_cast<long long>(a.nv) * nseg;
    if (grid > static_cast<long long>(num_sms) * 32) grid = static_cast<long long>(num_sms) * 32;
    auto go = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        kern<<<static_cast<unsigned>(grid), 256, smem, s>>>(a, seg, nseg);
    };
    if (mode == kOutQuadF32) go(quads_rows_kernel<kOutQuadF32, P>);
    else go(quads_rows_kernel<kOutQuadF16, P>);
    return true;
}
}  // namespace

void launch_quads_from_rows(const QuadArgs &a, int mode, int num_sms, cudaStream_t s)
{
    if (a.t1d) {
        const long long n = static_cast<long long>(a.nv) * (a.nc + 2 * kQuadPad) * kT1dPitch;
        long long grid = (n + 255) / 256;
        if (grid > static_cast<long long>(num_sms) * 32) grid = static_cast<long long>(num_sms) * 32;
        if (mode == kOutQuadF32)
            quads_t1d_kernel<kOutQuadF32><<<static_cast<unsigned>(grid < 1 ? 1 : grid), 256, 0, s>>>(a);
        else
            quads_t1d_kernel<kOutQuadF16><<<static_cast<unsigned>(grid < 1 ? 1 : grid), 256, 0, s>>>(a);
        return;
    }
    if (launch_quads_rows<1>(a, mode, num_sms, s)) return;
    long long grid = static_cast<long long>(a.nv) * (a.nr + 2 * kQuadPad);
    if (grid > static_cast<long long>(num_sms) * 32) grid = static_cast<long long>(num_sms) * 32;
    if (mode == kOutQuadF32)
        quads_from_rows_kernel<kOutQuadF32><<<static_cast<unsigned>(grid < 1 ? 1 : grid), 256, 0, s>>>(a);
    else
        quads_from_rows_kernel<kOutQuadF16><<<static_cast<unsigned>(grid < 1 ? 1 : grid), 256, 0, s>>>(a);
}

void launch_quads_partners(const QuadArgs &a, int mode, int num_sms, cudaStream_t s)
{
    if (launch_quads_rows<4>(a, mode, num_sms, s)) return;
    long long grid = static_cast<long long>(a.nv) * (a.nr + 2 * kQuadPad);
    if (grid > static_cast<long long>(num_sms) * 32) grid = static_cast<long long>(num_sms) * 32;
    if (mode == kOutQuadF32)
        quads_partners_kernel<kOutQuadF32><<<static_cast<unsigned>(grid < 1 ? 1 : grid), 256, 0, s>>>(a);
    else
        quads_partners_kernel<kOutQuadF16><<<static_cast<unsigned>(grid < 1 ? 1 : grid), 256, 0, s>>>(a);
}

cudaError_t launch_toeplitz_gemm(const GemmLaunch &g, int num_sms, cudaStream_t s)
{
    const bool four = g.form == kGemmBf16x4, f16 = g.form == kGemmF16x2;
    if (!(g.form == kGemmBf16x3 || (four && g.xll && g.tll) || (f16 && g.tll && g.rinv)))
        return cudaErrorInvalidValue;
    const CUtensorMapDataType dt = f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    CUtensorMap mAh, mAl, mAll, mBh, mBl, mBll;
    if (!make_map(&mAh, dt, g.xh, g.a_rows, g.Kp, BM) || !make_map(&mAl, dt, g.xl, g.a_rows, g.Kp, BM) ||
        !make_map(&mAll, dt, four ? g.xll : g.xl, g.a_rows, g.Kp, BM) ||
        !make_map(&mBh, dt, g.th, g.Np, g.Kp, BN) || !make_map(&mBl, dt, g.tl, g.Np, g.Kp, BN) ||
        !make_map(&mBll, dt, g.form == kGemmBf16x3 ? g.tl : g.tll, g.Np, g.Kp, BN))
        return cudaErrorInvalidValue;
    GemmParams p;
    p.M = g.M;
    p.N = g.N;
    p.m_begin = g.m_begin;
    p.num_kb = g.Kp / BK;
    p.m_tiles = (g.M + BM - 1) / BM;
    p.n_tiles = g.Np / BN;
    p.Y = g.Y;
    p.ldy = g.ldy;
    p.form = g.form;
    p.rinv = f16 ? g.rinv : nullptr;
    p.err = g.err;
    p.pq = g.quads ? (g.quarter > 0 ? 4 : 1) : 0;
    p.quads = static_cast<uint2 *>(g.quads);
    p.vscale = g.vscale;
    p.quarter = g.quarter;
    p.nr = g.nr;
    p.qpitch = g.N + 2 * kQuadPad;
    p.qview = static_cast<long long>(g.nr + 2 * kQuadPad) * p.qpitch;
    p.v_begin = g.v_begin;
    p.positions = static_cast<long long>(g.v_count) * g.nr;
    if (p.pq) {
        // partner stacks: base views of the quarter, A rows partner-interleaved; view-major
        // stacks: views of the stack, an even quad pitch (pairs of quads on 16-byte boundaries)
        const long long views = p.pq == 4 ? g.quarter : g.a_rows / (g.nr > 0 ? g.nr : 1);
        if (!g.vscale || g.nr <= 0 || g.v_count <= 0 || g.v_begin < 0 || g.v_begin + g.v_count > views ||
            (p.pq == 4 && static_cast<long long>(g.quarter) * 4 * g.nr != g.a_rows) ||
            (p.pq == 1 && (p.qpitch % 2 != 0 || reinterpret_cast<uintptr_t>(g.quads) % 16 != 0)))
            return cudaErrorInvalidValue;
        p.m_begin = g.v_begin * g.nr * p.pq;
        p.M = static_cast<int>(p.positions * p.pq);
        p.m_tiles = static_cast<int>((p.positions + pq_rows(p.pq) - 1) / pq_rows(p.pq));
    }
    const long long tiles = p.pq ? p.m_tiles : static_cast<long long>(p.m_tiles) * p.n_tiles;
    const int grid = tiles < num_sms ? static_cast<int>(tiles) : num_sms;
    const size_t smem = toeplitz_gemm_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(toeplitz_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    toeplitz_gemm_kernel<<<grid, 192, smem, s>>>(mAh, mAl, mAll, mBh, mBl, mBll, p);
    return cudaGetLastError();
}

}  // namespace gct
