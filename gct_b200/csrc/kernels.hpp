// Host-side launch interfaces of the FDK kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gct {

// Zero padding (entries per side) of the bilinear-quad layout of filtered projections.
constexpr int kQuadPad = 2;

enum FilterOut : int { kOutPlainF32 = 0, kOutQuadF32 = 1, kOutQuadF16 = 2 };

struct FilterArgs {
    const float *proj = nullptr;   // [nv][nr][nc] raw projections
    int nv = 0, nr = 0, nc = 0;
    int kind = 0;                  // gct_geom_kind
    float du = 0.f, dv = 0.f;      // row / column sampler widths
    const float4 *fview = nullptr; // per view: (det_row_center, det_col_center, sdd, 0)
    const float *parker = nullptr; // [nv][nc]
    const float2 *H = nullptr;     // [L] filter spectrum, scaled by 1/L
    int mode = kOutPlainF32;
    void *out = nullptr;           // plain: rows of views [0, nv); quads: view 0 of the stack (quad_layout)
    int v0 = 0;                    // quads: stack index of the first view filtered
    int quarter = 0;               // quads: quad_layout's quarter
    const float *vscale = nullptr; // per-view output scale for quads (nullable = 1)
    int t1d = 0;                   // one-row detectors: write the transposed quad grid (t1d_quad_layout)
    int *err = nullptr;            // plan status word: kFftWaitTimeout when an input copy timed out
};

// Status bits of the plan status word (gct_fdk_plan_check): Toeplitz GEMM pipeline stalls set
// small codes (the stage), the FFT filter's input copies kFftWaitTimeout.
constexpr int kFftWaitTimeout = 0x100;

// Where view v's quad grid (qview entries) lives in a stack: view after view (quarter = 0), or,
// for quarter-turn plans (quarter = nv / 4), with the four partner views v mod quarter + q quarter
// (q = 0..3) interleaved entry by entry, so that one 32-byte (FP16) or 64-byte (FP32) load brings
// all four partners of a detector position. Entry e of view v is at first + e * step.
__host__ __device__ inline void quad_layout(long long v, long long qview, int quarter, long long &first, int &step)
{
    if (quarter == 0) {
        first = v * qview;
        step = 1;
    } else {
        first = (v % quarter) * qview * 4 + v / quarter;
        step = 4;
    }
}

// Transposed quads of a one-row detector (1D parallel kind): the nc cells become the rows of a
// one-column image, so that the backprojector's row coordinate runs along the image's y axis (an
// affine function of the thread's loop index) and its column coordinate is the constant 0. Grid
// per view: (nc + 4) rows x 5 columns, entry (r, c) for r in [-2, nc + 2), c in [-2, 3); the quad
// at column 0 holds (y[r], 0, y[r + 1], 0) and at column -1 (0, y[r], 0, y[r + 1]).
constexpr int kT1dPitch = 1 + 2 * kQuadPad;

// Fused cosine + Parker weighting, zero padding, FFT convolution with the ramp filter and the
// epilogue into the requested layout. L is the power-of-two FFT length (256 to 8192).
void launch_filter_fft(const FilterArgs &a, int L, int num_sms, cudaStream_t s);

// Per-view |max| of the raw projections (amax must be zeroed) and the FP16 power-of-two scale
// that maps the bound amax * l1 (l1 = sum |taps|) below 2^14; writes vscale and 1/vscale.
void launch_view_absmax(const float *proj, int nv, long long pix_per_view, float *amax,
                        cudaStream_t s);
void launch_view_scales(const float *amax, int nv, float l1, float *vscale, float *vinv,
                        cudaStream_t s);

struct BpArgs {
    const void *quads = nullptr;
    int qpitch = 0;                // nc + 4
    long long qview = 0;           // (nr + 4) * (nc + 4)
    const float *coefs = nullptr;  // [nv][kCoefPerView]
    const float *vinv = nullptr;   // per-view scale of the stored values (nullable = 1)
    int v_begin = 0, v_count = 0;
    float *vol = nullptr;
    int nx = 0, ny = 0, nz = 0;
    float umax = 0.f, vmax = 0.f;  // nc, nr
    int accumulate = 0;
    int quarter = 0;  // quad_layout of the stack
    // spiral scans (one voxel per thread along z): slice k backprojects views [x, x + y) of
    // slice_views[k], intersected with [v_begin, v_begin + v_count)
    const int2 *slice_views = nullptr;
    // quarter-turn launches (quarter > 0): v_begin / v_count count base views, whose partners are
    // v + q * quarter (q = 1..3); sym (+1 / -1) is the turn that maps their voxel columns
    int sym = 0;
    // view-split launches of one-voxel-deep images (vchunk > 0, nz == 1): grid slice z takes views
    // [v_begin + z vchunk, + vchunk) and stores its sums at vol + z vol_stride (reduce_partials)
    int vchunk = 0;
    long long vol_stride = 0;
    // z-mirror launches (plans whose views map voxel (i, j, nz - 1 - k) to the mirror of (i, j, k)
    // about the detector's middle row, z_mirror_symmetry): column kernels over the lower half
    int mirror = 0;
};

// Resident blocks per SM of the backprojection kernel a launch of these options would use
// (sym: the quarter-turn kernel), for blocks of `threads` threads.
int backproject_blocks_per_sm(const BpArgs &a, int family, int storage, bool z_affine, bool sym, int zpt, int threads);
// vol[i] (+)= sum over c < nparts of part[c * n + i], in order of c (accumulate: add to vol).
void launch_reduce_partials(const float *part, int nparts, long long n, float *vol, bool accumulate, cudaStream_t s);

// Voxel-driven backprojection. family: 0 affine, 1 projective, 2 arc. storage: 0 f32, 1 f16.
// z_affine selects the column kernel (u and the denominator constant along z).
void launch_backproject(const BpArgs &a, int family, int storage, bool z_affine, int zpt,
                        int bx, int by, cudaStream_t s);

// Quarter-turn form (a.sym != 0, z-affine geometries, nx == ny even): threads cover the first
// quadrant of (x, y) columns; each evaluates the detector coordinates of its column once per base
// view and accumulates them into the column's four quarter-turn images from the four partner views.
void launch_backproject_sym(const BpArgs &a, int family, int storage, int zpt, int bx, int by, cudaStream_t s);

// How a block writes its sums: overwrite, add (views processed in order by successive launches)
// or add atomically (several blocks of one launch share the voxels; the volume starts at zero).
enum BpMode : int { kBpStore = 0, kBpAccumulate = 1, kBpAtomic = 2 };

// Work-queue backprojection: one persistent launch over the tiles of many reconstructions.
// A tile is the bx x by x zpt voxel box of one block (bx * by = 256 threads).
struct BpItem {
    BpArgs a;                  // v_begin / v_count / accumulate are taken from the work entry
    int family = 0, z_affine = 1, zpt = 8, bx = 8, by = 32;
    int vps = 32;              // views of coefficients staged per block barrier (<= kQueueMaxVps)
    int tiles_x = 0, tiles_y = 0, tiles_z = 0;
};
struct BpWork {
    int item = 0;              // index into the item array
    int tile = 0;              // x fastest, then y, then z
    int v_begin = 0, v_count = 0;
    int mode = kBpStore;
};
constexpr int kQueueThreads = 256;
constexpr int kQueueMaxVps = 64;    // views of coefficients staged per block barrier, at most
// Supported z-per-thread values of the queue kernels.
inline bool queue_zpt_ok(int zpt) { return zpt == 1 || zpt == 4 || zpt == 8 || zpt == 16; }
// Queue kernels by depth class, each compiled with its own register budget: class 0 runs tiles of
// one voxel per thread along z (2D images; needs many resident warps to hide its gather latency),
// class 1 tiles of 4, 8 or 16 (volumes; needs registers for its accumulators), class 2 the tiles
// of quarter-turn items (BpArgs.sym set, interleaved partner stacks): first-quadrant columns,
// 8 voxels per thread along z (1 for 2D images), view ranges counted in base views.
constexpr int kQueueClasses = 3;
constexpr int kQueueSymClass = 2;
inline bool sym_queue_zpt_ok(int zpt) { return zpt == 1 || zpt == 8; }
inline int queue_class(int zpt) { return zpt == 1 ? 0 : 1; }
// Blocks of a queue kernel resident per SM for the storage type (0 f32, 1 f16) and depth class.
int queue_blocks_per_sm(int storage, int zclass);
// Launches grid blocks that take work entries [0, n_work) in order from *counter (zeroed by the
// caller before the launch) until none are left. Every entry's item must be of the depth class.
void launch_backproject_queue(const BpItem *items, const BpWork *work, int n_work, int *counter, int storage,
                              int zclass, int grid, cudaStream_t s);

}  // namespace gct
