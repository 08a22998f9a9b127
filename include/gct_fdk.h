/*
 * gct_fdk.h -- C ABI of the B200-native FDK (Feldkamp-Davis-Kress) reconstruction engine.
 *
 * This is the drop-in boundary for GCT's axial FDK path. Every entry point below names the
 * reference interface it replaces (paths are relative to the satidev/gct project root).
 * The ABI uses plain C types only: pointers, sizes, doubles and PODs. No C++ or torch types
 * cross it, so a ctypes / cgo / JNI / N-API binding needs nothing but this file.
 *
 * Conventions
 *   - Every function returns gct_status. GCT_OK is 0. On failure, gct_last_error_string()
 *     returns a thread-local, human-readable message. The reference reports the same
 *     conditions with std::runtime_error / std::invalid_argument
 *     (src/cuda/utils/check_error.cu:6-36); the C++ header gct_fdk.hpp turns a non-OK
 *     status back into std::runtime_error.
 *   - Geometry is FP64 on the host. Projections and volumes are float32.
 *   - Projection stack layout: [view][row][col], col fastest
 *     (src/cpp/data/projection_stack.h:12-36). A 1D detector has one row.
 *   - Volume layout: [z][y][x], x fastest (src/cpp/data/recon_img.h:20-33). A 2D image has
 *     nz = 1.
 *   - "stream" arguments are cudaStream_t passed as void*; NULL is the legacy default stream.
 *   - Device pointers must live on the device that is current when the plan was created.
 */
#ifndef GCT_FDK_H
#define GCT_FDK_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define GCT_FDK_ABI_VERSION 1

typedef enum gct_status {
    GCT_OK = 0,
    GCT_ERR_INVALID_ARG = 1,   /* bad geometry, sizes or pointers */
    GCT_ERR_OUT_OF_MEMORY = 2, /* a device or host allocation failed */
    GCT_ERR_BUDGET = 3,        /* request does not fit the configured device-memory budget */
    GCT_ERR_TIMEOUT = 4,       /* a bounded wait ran out */
    GCT_ERR_CUDA = 5,          /* a CUDA runtime call failed */
    GCT_ERR_NOT_SUPPORTED = 6, /* option not available for this geometry or device */
    GCT_ERR_NOT_READY = 7,     /* asynchronous work still in flight (poll again) */
    GCT_ERR_CANCELLED = 8      /* request was cancelled before it ran */
} gct_status;

/* The seven axial detector configurations: GCT::Geom::ProjGeom<DetRow, DetCol...>
 * (src/cpp/geom/proj_geom.h:21-103), i.e. the seven reconstruct() overloads
 * (src/cuda/recon/recon_wrappers.cuh:15-43). */
typedef enum gct_geom_kind {
    GCT_GEOM_PARALLEL_1D = 0,   /* <DetParallel>                 -> 2D image */
    GCT_GEOM_FAN_ARC = 1,       /* <DetFanArc>                   -> 2D image */
    GCT_GEOM_FAN_LINE = 2,      /* <DetFanLine>                  -> 2D image */
    GCT_GEOM_PARALLEL_2D = 3,   /* <DetParallel, DetParallel>    -> 3D volume */
    GCT_GEOM_CONE_PARALLEL = 4, /* <DetParallel, DetFanLine>     -> 3D volume (rebinned) */
    GCT_GEOM_CONE_CYL = 5,      /* <DetFanArc, DetFanLine>       -> 3D volume */
    GCT_GEOM_CONE_FLAT = 6      /* <DetFanLine, DetFanLine>      -> 3D volume */
} gct_geom_kind;

/* Rotation direction: GCT::Geom::RotDir (src/cpp/geom/rotation_geom.h:10-14). */
typedef enum gct_rot_dir { GCT_ROT_CCW = -1, GCT_ROT_CW = 1 } gct_rot_dir;

/* Apodisation window: GCT::Recon::ApodFunc (src/cpp/io/parameters/filt_parameters.h:9-13). */
typedef enum gct_apod_func { GCT_APOD_NONE = 0, GCT_APOD_HANN = 1, GCT_APOD_HAMMING = 2 } gct_apod_func;

/* Uniform 1D detector sampler: GCT::Geom::Sampler1D (src/cpp/geom/sampling_info.h:144-153).
 * sampling_width is in mm for DetParallel / DetFanLine and in radians for DetFanArc. */
typedef struct gct_detector {
    uint32_t num_samples;
    double sampling_width;
} gct_detector;

/* Per-view projection geometry: the union of the ProjGeom<...> fields
 * (src/cpp/geom/proj_geom.h:21-103). Fields a kind does not use are ignored.
 *   PARALLEL_1D/2D : rot_ang, det_row_center (, det_col_center)
 *   CONE_PARALLEL  : rot_ang, src_det_dist, src_iso_dist, det_row_center, det_col_center
 *   FAN_LINE       : src_det_dist, det_row_center, src_pos[0..1], det_row_dir[0..1]
 *   FAN_ARC        : FAN_LINE fields + iso_ray_dir[0..1]
 *   CONE_FLAT      : src_det_dist, centres, src_pos, det_row_dir, det_col_dir
 *   CONE_CYL       : CONE_FLAT fields + iso_ray_dir
 * Distances in mm, angles in radians, centres in detector pixels. */
typedef struct gct_view_geom {
    double rot_ang;
    double det_row_center;
    double det_col_center;
    double src_det_dist;
    double src_iso_dist;
    double src_pos[3];
    double det_row_dir[3];
    double det_col_dir[3];
    double iso_ray_dir[3];
} gct_view_geom;

/* CT geometry of a scan: GCT::Geom::CTGeom / AxialCTGeom (src/cpp/geom/ct_geom.h:18-53,
 * src/cpp/geom/axial_ct_geom.h:8-13). det_col.num_samples must be 1 for the 1D kinds. */
typedef struct gct_ct_geom {
    int32_t kind; /* gct_geom_kind */
    gct_detector det_row;
    gct_detector det_col;
    uint32_t num_views;
    const gct_view_geom *views; /* num_views entries, host memory */
} gct_ct_geom;

/* Reconstruction grid: GCT::Geom::ReconImgGeom<2|3> (src/cpp/geom/recon_img_geom.h:15-30).
 * For a 2D image set nz = 1; dz and mid[2] are then ignored. */
typedef struct gct_vol_geom {
    uint32_t nx, ny, nz;
    double dx, dy, dz;
    double mid[3];
} gct_vol_geom;

/* Ramp-filter parameters: GCT::Recon::FiltParams (src/cpp/io/parameters/filt_parameters.h:14-18).
 * The reference's defaults are cut_off_freq = 1 and GCT_APOD_NONE. */
typedef struct gct_filt_params {
    double cut_off_freq;
    int32_t apod_func; /* gct_apod_func */
} gct_filt_params;

/* Rotation analysis: GCT::Geom::RotationGeom (src/cpp/geom/rotation_geom.h:16-24). */
typedef struct gct_rotation_geom {
    int32_t dir; /* gct_rot_dir */
    double rot_ang_incr;
    double rot_ang_range;
    uint32_t num_proj_per_rot;
} gct_rotation_geom;

/* Ideal circular-trajectory parameters: the union of Parallel1DProjGeomParams,
 * FanBeamProjGeomParams, Parallel2DProjGeomParams and ConeBeamProjGeomParams with their
 * RotationParams (src/cpp/io/parameters/proj_geom_params.h:16-58). */
typedef struct gct_geom_params {
    double det_row_center;
    double det_col_center;
    double src_det_dist;
    double src_iso_dist;
    int32_t rot_dir; /* gct_rot_dir */
    double init_ang;
    double ang_incr;
    uint32_t num_proj;
    double hel_pitch;
} gct_geom_params;

/* Execution options. Zero-initialise for defaults. */
enum {
    GCT_FILTER_FFT = 0,             /* own row-batched shared-memory FFT, FP32 arithmetic */
    GCT_FILTER_TOEPLITZ_BF16X3 = 1, /* 3-term split BF16 Toeplitz GEMM on tcgen05, FP32 accumulate */
    GCT_FILTER_TOEPLITZ_BF16X4 = 2, /* projections in three BF16 pieces and the central taps
                                     * (|c - k| <= 64) in three: three full GEMM terms plus two over
                                     * the diagonal band; removes the two-piece taps' DC error */
    GCT_FILTER_TOEPLITZ_F16X2 = 3   /* rows scaled per row into two FP16 pieces, taps in FP16: one
                                     * full GEMM term (hi x hi) plus three over the diagonal band,
                                     * the far taps' dropped parts folded into each column's
                                     * central tap so its DC response stays exact */
};
enum {
    GCT_STORAGE_F32 = 0, /* filtered projections kept in FP32 */
    GCT_STORAGE_F16 = 1  /* filtered projections kept in FP16 with a per-view power-of-two scale */
};
enum {
    /* Full scans whose views come in quarter-turn partners (view v + nv/4 is view v turned by 90
     * degrees about the rotation axis) on a square, even, centred grid can evaluate detector
     * coordinates once per four voxel-view updates, with the partner views' filtered projections
     * interleaved in the workspace. Detected on the host in FP64 at plan creation. AUTO uses it
     * with FP16 storage (where it is faster), ON with either storage, OFF never. */
    GCT_SYMMETRY_AUTO = 0,
    GCT_SYMMETRY_OFF = 1,
    GCT_SYMMETRY_ON = 2
};
enum {
    GCT_SCAN_AXIAL = 0,  /* circular scans: GCT::Recon::CUDA::reconFDK(AxialCTGeom) */
    /* spiral (helical) cone-beam scans, Wang's FDK: every z slice backprojects the one rotation of
     * views centred on the view whose source z is nearest the slice, with cosine weights and the
     * ramp filter but no Parker weights; slices whose rotation would start at view 0 or end at or
     * after the last view stay zero (GCT::Recon::CUDA::reconFDK(SpiralCTGeom),
     * src/cuda/recon/fdk_spiral.cuh:33-94; src/cpp/geom/spiral_ct_geom.h:30-95). */
    GCT_SCAN_SPIRAL = 1
};
typedef struct gct_fdk_opts {
    int32_t filter;        /* GCT_FILTER_* */
    int32_t storage;       /* GCT_STORAGE_* */
    int32_t z_per_thread;  /* backprojection voxels per thread along z; 0 = tuned default */
    int32_t block_x;       /* backprojection block shape; 0 = tuned default */
    int32_t block_y;
    int32_t symmetry;      /* GCT_SYMMETRY_* */
    int32_t scan;          /* GCT_SCAN_* */
    int32_t reserved[1];
} gct_fdk_opts;

typedef struct gct_fdk_plan gct_fdk_plan;

/* ---- version / errors ------------------------------------------------------------------ */
int32_t gct_abi_version(void);
const char *gct_last_error_string(void);

/* ---- geometry (host, FP64) ------------------------------------------------------------- */

/* Replaces GCT::Geom::ProjGeomFactory<DetRow, DetCol...>::create(params, proj_idx)
 * (src/cpp/io/geom_reader/proj_geom_factory_params.cpp:8-108, with the rotation of
 * src/cpp/io/geom_reader/proj_geom_cb_factory.cpp:14-48 and the fan-beam reduction of
 * src/cpp/io/geom_reader/proj_geom_fb_factory.cpp:13-45), evaluated in FP64. */
gct_status gct_proj_geom_create(int32_t kind, const gct_geom_params *params, uint32_t proj_idx,
                                gct_view_geom *out);

/* Projection matrix of a flat-panel view: GCT::Geom::ProjectionMatrix
 * (src/cpp/geom/projection_matrix.{h,cpp}), in FP64. matrix is 3 x 4 row-major; intrinsic K is
 * upper triangular with a positive diagonal and K[2][2] = 1 (focalLengthDetRow = K[0][0],
 * principalPointDetRow = K[0][2], principalPointDetCol = K[1][2]); rotation R holds the detector
 * row direction, column direction and their cross product as rows; src_pos is the focal spot. */
typedef struct gct_proj_matrix {
    double matrix[12];
    double intrinsic[9];
    double rotation[9];
    double src_pos[3];
} gct_proj_matrix;

/* ProjectionMatrix(matrix): RQ decomposition of the left 3 x 3 block (through QR of its
 * inverse) and the source position -M^-1 m4 (projection_matrix.cpp:4-62). */
gct_status gct_proj_matrix_decompose(const double *matrix, gct_proj_matrix *out);

/* ProjectionMatrix(ProjGeom<DetFanLine, DetFanLine>, pix_width_mm, pix_height_mm)
 * (projection_matrix.cpp:64-97): M = K [R | -R src], scaled so that M[2][3] = 1. view holds the
 * CONE_FLAT fields (src_det_dist in mm, centres in pixels, src_pos, det_row_dir, det_col_dir). */
gct_status gct_proj_matrix_compose(const gct_view_geom *view, double pix_width_mm, double pix_height_mm,
                                   gct_proj_matrix *out);

/* ProjGeomFactory<DetFanLine, DetFanLine>::create(ProjectionMatrix)
 * (src/cpp/io/geom_reader/proj_geom_factory_proj_mat.cpp:7-26): the CONE_FLAT view of a 3 x 4
 * matrix. As in the reference, src_det_dist is the focal length in detector-row pixels; multiply
 * it by the pixel width before use. src_iso_dist = |src_pos|. */
gct_status gct_proj_geom_from_matrix(const double *matrix, gct_view_geom *out);

/* GCT::Geom::SpiralCTGeom's checks (src/cpp/geom/spiral_ct_geom.h:30-50): a cone-beam 2D
 * detector, projections per rotation > 0, source z sorted either way and a positive pitch; returns
 * the projections per rotation and the pitch (source z travel per radian, mm). */
gct_status gct_spiral_geom_check(const gct_ct_geom *geom, uint32_t *num_proj_per_rot, double *pitch_mm_per_rad);

/* SpiralCTGeom::firstAndLastProjIndices (spiral_ct_geom.h:57-75): the views [first, last) of the
 * rotation centred on the view whose source z is nearest slice_pos_mm. Signed: first is negative
 * where the reference's unsigned index wraps. */
gct_status gct_spiral_proj_indices(const gct_ct_geom *geom, double slice_pos_mm, int64_t *first, int64_t *last);

/* Replaces GCT::Geom::getRotationGeom (src/cpp/geom/rotation_geom.h:90-115,
 * src/cpp/geom/rotation_geom.cpp:7-134). rot_ang / rel_rot_ang may be NULL; otherwise they
 * receive num_views angles each. Returns GCT_ERR_INVALID_ARG where the reference returns
 * std::nullopt (and CTGeom's constructor throws "Invalid X-ray source trajectory"). */
gct_status gct_rotation_geom_get(const gct_ct_geom *geom, gct_rotation_geom *out,
                                 double *rot_ang, double *rel_rot_ang);

/* Replaces GCT::Recon::isValidAxialRecon (src/cpp/recon/check_validity.h:66-75).
 * *valid receives 1 or 0; with verbose != 0 the reasons are printed to stderr. */
gct_status gct_is_valid_axial_recon(const gct_ct_geom *geom, uint32_t proj_num_cols,
                                    uint32_t proj_num_rows, uint32_t num_proj, int32_t verbose,
                                    int32_t *valid);

/* Replaces GCT::Recon::projFiltKernel / RampFilter::kernel
 * (src/cpp/recon/proj_filt_kernel.cpp:5-45, src/cpp/recon/ramp_filter.h:29-56): the
 * det_row.num_samples spatial taps, tap j at offset n = j - num_samples/2. FP64. */
gct_status gct_ramp_filter_taps(int32_t kind, const gct_detector *det_row,
                                const gct_filt_params *params, double *taps);

/* Replaces GCT::Recon::CUDA::getParkerWeights (src/cuda/recon/parker_weighting.cuh:132-200):
 * weights[view][col] (num_views x det_row.num_samples), window bounds in FP64. For fan and
 * cone kinds whose angular range is <= pi the reference leaves its buffer uninitialised
 * (parker_weighting.cuh:163-175); here those weights are defined as 1. */
gct_status gct_parker_weights(const gct_ct_geom *geom, float *weights);

/* Evaluates, on the host in double precision, the per-view backprojection coefficients the
 * kernels use (derived in FP64, stored as FP32) at fractional voxel index (i, j, k) of `vol`:
 * world position xyz (mm; src/cuda/geom/coord_trans_img.cuh:52-66), detector pixel coordinates
 * col/row (src/cuda/geom/coord_trans_proj.cuh:142-145 after projMapping :157-345) and the
 * backprojection weight (without the angular-increment scale). For the 1D kinds row is 0 and k
 * is ignored. Any pointer except geom/vol/ijk may be NULL. */
gct_status gct_map_point(const gct_ct_geom *geom, const gct_vol_geom *vol, uint32_t view,
                         const double ijk[3], double xyz[3], double *col, double *row,
                         double *weight);

/* ---- FDK plans (device) ---------------------------------------------------------------- */

/* Builds a reusable reconstruction plan on the current CUDA device: FP64 per-view geometry,
 * filter spectrum and Parker table, uploaded once. Replaces the per-call set-up inside
 * GCT::Recon::CUDA::reconFDK (src/cuda/recon/fdk_axial.cuh:68-205): CTGeomDev, the
 * RampFilteringFFT constructor and getParkerWeights. filt and opts may be NULL. */
gct_status gct_fdk_plan_create(const gct_ct_geom *geom, const gct_vol_geom *vol,
                               const gct_filt_params *filt, const gct_fdk_opts *opts,
                               gct_fdk_plan **out);
gct_status gct_fdk_plan_destroy(gct_fdk_plan *plan);

/* Synchronises the device and reports a failure recorded asynchronously by the plan's kernels:
 * GCT_ERR_TIMEOUT if a bounded pipeline wait of the Toeplitz-GEMM filter ran out. */
gct_status gct_fdk_plan_check(gct_fdk_plan *plan);

/* Device bytes of scratch that gct_fdk_execute needs: the filtered-projection stack and, for
 * FP16 storage, its per-view scales. A workspace carries everything the backprojection of one
 * prepared stack reads, so several stacks prepared with one plan into separate workspaces stay
 * independent. */
gct_status gct_fdk_plan_workspace_bytes(const gct_fdk_plan *plan, uint64_t *bytes);

/* Quarter-turn symmetry the plan found (GCT_SYMMETRY_AUTO): +1 when view v + nv/4 sees voxel
 * column (n-1-y, x) where view v sees (x, y), -1 for (y, n-1-x), 0 when the geometry has neither
 * or the option is off. No reference counterpart (an execution property of this engine). */
gct_status gct_fdk_plan_symmetry(const gct_fdk_plan *plan, int32_t *quarter_turn);

/* Mirror symmetry in z the plan found (GCT_SYMMETRY_AUTO with FP16 storage, or _ON): 1 when every
 * view maps voxel (x, y, nz-1-z) onto the same detector column and weight as (x, y, z) and onto
 * the row mirrored about the detector's middle row (source on the grid's middle plane, detector
 * centred on it, nz even), so that whole-volume backprojections without the quarter-turn form
 * evaluate each view once per voxel pair; 0 otherwise. No reference counterpart (an execution
 * property of this engine). */
gct_status gct_fdk_plan_z_mirror(const gct_fdk_plan *plan, int32_t *mirror);

/* Full FDK on device buffers, asynchronous on `stream`: fused cosine + Parker weighting and
 * ramp filtering, then backprojection and the angular-increment scale. proj_dev is
 * [view][row][col] float32, vol_dev receives [z][y][x] float32 (overwritten). workspace may be
 * NULL, in which case the plan allocates (once) and keeps its own. Replaces the device part of
 * reconFDKHighMem (src/cuda/recon/fdk_axial.cuh:151-205). */
gct_status gct_fdk_execute(gct_fdk_plan *plan, const float *proj_dev, float *vol_dev,
                           void *workspace, void *stream);

/* Stage entry points of the same plan, for tests and for callers that pipeline stages.
 * gct_fdk_filter writes the weighted, ramp-filtered projections as plain float32
 * [view][row][col] (what RampFilteringFFT::runFiltering leaves in the stack after
 * runCosWeighting and runParkerWeighting, src/cuda/recon/fdk_axial.cuh:165-171), without the
 * backprojection scales. */
gct_status gct_fdk_filter(gct_fdk_plan *plan, const float *proj_dev, float *filtered_dev,
                          void *stream);

/* The two device stages of gct_fdk_execute over a view range [view_begin, view_begin+count):
 *   gct_fdk_prepare      weights + ramp-filters those views of proj_dev (the full stack pointer)
 *                        into the workspace in the backprojector's layout;
 *   gct_fdk_backproject  backprojects those views of the workspace into vol_dev, overwriting it
 *                        (accumulate = 0) or adding to it (accumulate = 1), angular scale included.
 * Running prepare + backproject over all views equals gct_fdk_execute. Splitting the views lets a
 * caller overlap uploads of later views with work on earlier ones (the streaming replacement for
 * reconFDKLowMem, src/cuda/recon/fdk_axial.cuh:91-149). */
gct_status gct_fdk_prepare(gct_fdk_plan *plan, const float *proj_dev, void *workspace,
                           uint32_t view_begin, uint32_t view_count, void *stream);
gct_status gct_fdk_backproject(gct_fdk_plan *plan, const void *workspace, float *vol_dev,
                               uint32_t view_begin, uint32_t view_count, int32_t accumulate,
                               void *stream);

/* Host buffers through a plan: uploads proj_host in view chunks on a copy stream while earlier
 * chunks are filtered and backprojected (accumulating) on `stream`, then downloads the volume and
 * synchronises. Device staging buffers are owned by the plan and reused across calls. Pass pinned
 * host memory for the copies to overlap. */
gct_status gct_fdk_execute_host(gct_fdk_plan *plan, const float *proj_host, float *vol_host,
                                void *stream);

/* The same without the final wait: the call enqueues its uploads, filters, backprojections and
 * the volume download and returns. Consecutive calls on one plan overlap (a call's uploads run
 * under the previous call's backprojections, its download under the next call's work; two device
 * volumes alternate). proj_host and vol_host must stay valid and untouched until
 * gct_fdk_host_sync(plan) returns, which waits for every such call of the plan. */
gct_status gct_fdk_execute_host_async(gct_fdk_plan *plan, const float *proj_host, float *vol_host,
                                      void *stream);
gct_status gct_fdk_host_sync(gct_fdk_plan *plan);

/* Host buffers with a bounded device footprint for the projections (stacks larger than the
 * device): the views stream through two upload slots and a filtered stack of one chunk, where a
 * chunk is as many views as device_bytes holds (two float32 views plus one filtered view each),
 * and each chunk is backprojected into the plan's device volume. The volume itself must fit
 * besides. Replaces reconFDKLowMem (src/cuda/recon/fdk_axial.cuh:91-149), which the reference
 * picks when the whole stack needs 75 % of the device memory or more; gct_reconstruct_ex applies
 * the same rule and calls this path with half the memory left after the volume.
 * GCT_ERR_BUDGET if device_bytes holds no view. Synchronous on `stream`. */
gct_status gct_fdk_execute_host_budget(gct_fdk_plan *plan, const float *proj_host, float *vol_host,
                                       uint64_t device_bytes, void *stream);

/* Full FDK on device buffers without allocating device memory. No counterpart in the reference.
 * For callers that cannot allocate device memory when they reconstruct: a host application whose
 * own memory manager has already reserved the device's memory, or an acquisition loop that
 * forbids allocation once it is running. Such a caller creates the plan at start-up and then
 * calls this instead of gct_fdk_execute (which allocates its workspace on first use).
 * The filtered projections go through a fixed scratch array of GCT_NOALLOC_SCRATCH_BYTES
 * (64 MiB) that the library holds on every device that loads it, until the process exits; the
 * views are processed in chunks that fit it. A geometry whose single view needs more than that
 * is rejected with GCT_ERR_BUDGET. gct_fdk_plan_create looks up the scratch address
 * (cudaGetSymbolAddress) on the plan's device; the CUDA runtime loads the module that holds the
 * array lazily, so its 64 MiB are committed then, at plan creation, and never inside this call.
 * Kernel code is loaded by the CUDA driver at a kernel's first launch (lazy module loading, the
 * default since CUDA 12.2): a caller that must see no device allocation at all after start-up
 * makes one call at start-up, or sets CUDA_MODULE_LOADING=EAGER. All calls share the one scratch
 * array: calls whose GPU work overlaps (other streams, other threads, other plans) race on it and
 * must be serialised by the caller. Nothing in it needs to start at zero; each call overwrites
 * what it reads. Plans with the quarter-turn form run the plain backprojector on this path. */
#define GCT_NOALLOC_SCRATCH_BYTES (64ull << 20)
gct_status gct_fdk_execute_noalloc(gct_fdk_plan *plan, const float *proj_dev, float *vol_dev,
                                   void *stream);

/* Host-to-host drop-in: replaces void GCT::Recon::CUDA::reconstruct(cg, proj, vol)
 * (src/cuda/recon/recon_wrappers.cuh:15-43, recon_wrappers.cu:7-55). Synchronous, default
 * FiltParams, FP32 path; proj_host and vol_host are plain host arrays. */
gct_status gct_reconstruct(const gct_ct_geom *geom, const gct_vol_geom *vol,
                           const float *proj_host, float *vol_host);

/* Same as gct_reconstruct with explicit filter parameters and execution options. */
gct_status gct_reconstruct_ex(const gct_ct_geom *geom, const gct_vol_geom *vol,
                              const gct_filt_params *filt, const gct_fdk_opts *opts,
                              const float *proj_host, float *vol_host);

/* ---- batches (device) -------------------------------------------------------------------- */

/* Many reconstructions of uneven sizes and geometries in one persistent backprojection launch.
 * No counterpart in the reference, which reconstructs one stack per call
 * (src/cuda/recon/recon_wrappers.cuh:15-43) with one backprojection launch per view
 * (src/cuda/recon/fdk_axial.cuh:189-193).
 *
 * gct_fdk_batch_create takes the items (each: a plan, its device projections and its device
 * volume), allocates a workspace per item, picks each item's tile shape (z-voxels per thread,
 * block footprint, views per coefficient stage) with an on-device autotuner whose results are
 * cached per process, device and item shape, builds one work queue of (volume tile, view chunk)
 * entries per storage type, and captures the filter stages of all items (on up to four forked
 * streams) plus the queue launches as one CUDA graph. gct_fdk_batch_launch replays it on
 * `stream`: every item's volume is overwritten with its reconstruction, the values
 * gct_fdk_execute gives up to the order of the floating-point sums. The buffers and plans must
 * stay alive while the batch exists; items that share a plan run their filter stages one after
 * another. The batch uses the plans' filter scratch: do not run those plans elsewhere while a
 * launch is in flight. */
typedef struct gct_fdk_batch gct_fdk_batch;

typedef struct {
    gct_fdk_plan *plan;
    const float *proj_dev;    /* [view][row][col] */
    float *vol_dev;           /* [z][y][x], overwritten */
} gct_batch_item;

typedef struct {
    int32_t autotune;         /* 1: time tile shapes on the device (default); 0: fixed defaults */
    int32_t use_graph;        /* 1: replay a captured CUDA graph (default); 0: issue stage by stage */
    int32_t blocks_per_sm;    /* resident blocks of the queue kernel per SM; 0: its occupancy */
    int32_t reserved[5];
} gct_batch_opts;

typedef struct {
    int32_t z_per_thread, block_x, block_y, views_per_stage;
    int32_t view_split;       /* view chunks of the item's tiles (> 1: atomic accumulation) */
    double tuned_gups;        /* autotuner's measured rate of the chosen shape; 0 if untuned */
} gct_batch_item_config;

/* opts may be NULL (autotune, graph). */
gct_status gct_fdk_batch_create(const gct_batch_item *items, uint32_t count, const gct_batch_opts *opts,
                                gct_fdk_batch **out);
gct_status gct_fdk_batch_launch(gct_fdk_batch *batch, void *stream);
gct_status gct_fdk_batch_item_config(const gct_fdk_batch *batch, uint32_t item, gct_batch_item_config *out);
/* Work entries in the queues and voxel-view updates of one launch. */
gct_status gct_fdk_batch_work(const gct_fdk_batch *batch, uint64_t *work_entries, uint64_t *updates);
gct_status gct_fdk_batch_destroy(gct_fdk_batch *batch);

/* ---- serving (device) -------------------------------------------------------------------- */

/* A request loop with continuous batching. No counterpart in the reference (one synchronous
 * reconstruction per call, src/cuda/recon/recon_wrappers.cuh:15-43).
 *
 * gct_fdk_server_create reserves `memory_budget_bytes` of device memory once and starts a worker
 * thread on the current device. gct_fdk_server_submit queues a request (a plan, host projections
 * [view][row][col], a host volume [z][y][x] to fill) and returns a ticket; requests are admitted
 * in arrival order as soon as their projections, workspace and volume fit in the free part of the
 * budget and fewer than max_active are on the device. An admitted request is uploaded and
 * filtered on its own streams while others backproject; the backprojection runs in rounds, each
 * one persistent work-queue launch over the tiles of every active request, each request
 * contributing its next chunk of views (sized from its own shape only: about round_updates
 * voxel-view updates, at least 16 views). Requests arriving meanwhile join the next round. A
 * finished volume is copied back and its memory returned to the budget.
 *
 * Because a request's chunks and tile shape depend only on the request (and the process-wide
 * autotuner cache), its result is bit-identical whether it runs alone or among others. Host
 * buffers must stay valid until the request completes; pinned memory lets copies overlap. The
 * plan's filter scratch is used by the worker: do not run a plan elsewhere while the server holds
 * requests for it. */
typedef struct gct_fdk_server gct_fdk_server;

typedef struct {
    uint64_t memory_budget_bytes;   /* device bytes for admitted requests (required) */
    uint32_t max_active;            /* requests admitted at once; 0 = 64 */
    uint32_t autotune;              /* 1 = tile shapes from the autotuner (default 0 = fixed) */
    double round_updates;           /* voxel-view updates per request per round; 0 = 2e9 */
    int32_t reserved[4];
} gct_server_opts;

typedef enum {
    GCT_REQ_QUEUED = 0,
    GCT_REQ_RUNNING = 1,
    GCT_REQ_DONE = 2,
    GCT_REQ_FAILED = 3,
    GCT_REQ_CANCELLED = 4
} gct_req_state;

typedef struct {
    int32_t state;                  /* gct_req_state */
    int32_t status;                 /* gct_status of a failed request, else GCT_OK */
    double queued_ms;               /* submit -> admission */
    double latency_ms;              /* submit -> volume on the host */
    uint32_t rounds;                /* backprojection rounds the request took part in */
    uint32_t views_per_round;
} gct_request_info;

typedef struct {
    uint64_t submitted, completed, failed, cancelled, rejected;
    uint64_t rounds;                /* backprojection rounds launched */
    uint64_t peak_bytes;            /* most budget bytes in use at once */
    uint32_t peak_active;           /* most requests admitted at once */
    double p50_ms, p99_ms, mean_ms; /* latency of completed requests */
    double recons_per_s;            /* completed / (last completion - first submission) */
} gct_server_stats;

gct_status gct_fdk_server_create(const gct_server_opts *opts, gct_fdk_server **out);
/* GCT_ERR_BUDGET if the request alone exceeds the budget. */
gct_status gct_fdk_server_submit(gct_fdk_server *server, gct_fdk_plan *plan, const float *proj_host,
                                 float *vol_host, uint64_t *ticket);
gct_status gct_fdk_server_info(gct_fdk_server *server, uint64_t ticket, gct_request_info *info);
/* Blocks until the request is done, failed or cancelled (its status is returned) or timeout_ms
 * passes (GCT_ERR_NOT_READY); timeout_ms < 0 waits without limit. */
gct_status gct_fdk_server_wait(gct_fdk_server *server, uint64_t ticket, double timeout_ms);
/* Cancels a request that is still queued; GCT_ERR_NOT_READY if it was already admitted. */
gct_status gct_fdk_server_cancel(gct_fdk_server *server, uint64_t ticket);
gct_status gct_fdk_server_stats(gct_fdk_server *server, gct_server_stats *stats);
/* Finishes every request, stops the worker and releases the budget. */
gct_status gct_fdk_server_destroy(gct_fdk_server *server);

/* ---- projection (device) ---------------------------------------------------------------- */

/* Analytic phantom: an ellipsoid with centre c (mm), semi-axes a (mm), rotation angle
 * phi about z (radians) and attenuation mu (1/mm). For 2D kinds only x, y are used and the
 * ellipsoid acts as an ellipse. */
typedef struct gct_ellipsoid {
    double center[3];
    double semi_axes[3];
    double phi;
    double mu;
} gct_ellipsoid;

/* Exact line integrals of a sum of ellipsoids along every detector ray of the geometry,
 * written to proj_dev [view][row][col]. Generates the synthetic inputs of the benchmarks. The
 * reference has no counterpart (its inputs come from files). */
gct_status gct_phantom_project(const gct_ct_geom *geom, const gct_ellipsoid *ellipsoids,
                               uint32_t num_ellipsoids, float *proj_dev, void *stream);

/* Ray-driven forward projector of a voxel volume (trilinear samples every step_vox voxel
 * lengths along each ray), writing proj_dev [view][row][col]. Replaces the unfinished 1D
 * parallel ray-marcher of src/cuda/recon/forward_proj.cuh:13-102 for all seven kinds. */
gct_status gct_forward_project(const gct_ct_geom *geom, const gct_vol_geom *vol,
                               const float *vol_dev, float step_vox, float *proj_dev,
                               void *stream);

/* ---- array files (host) ---------------------------------------------------------------- */

/* Element types of array files: GCT::IO::ArrayElemType (src/cpp/io/metadata.h:10-22). */
typedef enum gct_elem_type {
    GCT_T_UINT8 = 0,
    GCT_T_INT8 = 1,
    GCT_T_UINT16 = 2,
    GCT_T_INT16 = 3,
    GCT_T_UINT32 = 4,
    GCT_T_INT32 = 5,
    GCT_T_UINT64 = 6,
    GCT_T_INT64 = 7,
    GCT_T_FLOAT = 8,
    GCT_T_DOUBLE = 9
} gct_elem_type;

/* GCT::IO::ArrayMetadata (src/cpp/io/metadata.h:24-30): one file's rows x columns x slices. */
typedef struct gct_array_metadata {
    uint32_t num_rows;
    uint32_t num_cols;
    uint32_t num_slices;
    int32_t type; /* gct_elem_type */
} gct_array_metadata;

/* Readers: GCT::IO::MetaImgFileReader (src/cpp/io/file_reader/meta_img_reader.cpp:10-165; .mha
 * with ElementDataFile = LOCAL, or a header naming a data file in its directory),
 * DenFileReader (den_file_reader.cpp: three uint16 then the data, the type from the file size)
 * and RawDataFileReader (raw_data_file_reader.h: the caller gives the metadata). */
typedef enum gct_file_format {
    GCT_FILE_META_IMAGE = 0,
    GCT_FILE_DEN = 1,
    GCT_FILE_RAW = 2
} gct_file_format;

/* ArrayFileReader::readMetadata (array_file_reader.h:25). For GCT_FILE_RAW, *md is the input
 * metadata and is returned unchanged once the file is found. */
gct_status gct_array_read_metadata(const char *filename, int32_t format, gct_array_metadata *md);

/* ArrayFileReader::readData<OpType> (array_file_reader.h:60-65): the data of the file, or with
 * `series` of every file in its directory tree with its extension and size in sorted order
 * (getAllFiles, src/cpp/io/file_utils.cpp:7-27), each element static_cast to out_type.
 * raw_md: metadata of GCT_FILE_RAW files (else ignored). *count (optional) receives the number of
 * elements; with out == NULL nothing else happens (a size query), else out_count must equal it.
 * Data sizes are checked exactly (readDataFromBinFile); a LOCAL MetaImage shorter than its header
 * promises is an error (the reference leaves the missing elements zero). */
gct_status gct_array_read(const char *filename, int32_t format, int32_t series, const gct_array_metadata *raw_md,
                          int32_t out_type, void *out, uint64_t out_count, uint64_t *count);

/* GCT::IO::ArrayFileWriter::write(MetaImgMetaData, data, filename)
 * (src/cpp/io/file_writer/meta_img_file_writer.h): the reference's header lines in its order;
 * a ".mha" name keeps the data after the header, any other writes <stem>.raw beside it. dim_size,
 * spacing and offset hold ndims (1..3) entries, x first; data holds count elements of `type`. */
gct_status gct_meta_image_write(const char *filename, uint32_t ndims, const uint32_t *dim_size,
                                const float *spacing, const float *offset, int32_t type, const void *data,
                                uint64_t count);

/* ArrayFileWriter::write(DenMetaData, ...) (den_file_writer.h): uint16 rows, columns, slices,
 * then the data. Dimensions above 65535 are rejected (the reference truncates them). */
gct_status gct_den_write(const char *filename, uint32_t num_rows, uint32_t num_cols, uint32_t num_slices,
                         int32_t type, const void *data, uint64_t count);

/* ArrayFileWriter::write(data, filename) (raw_data_file_writer.h): the bytes of the data. */
gct_status gct_raw_write(const char *filename, int32_t type, const void *data, uint64_t count);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif /* GCT_FDK_H */
