// Host-side FP64 geometry for the FDK engine: circular-trajectory factories, rotation analysis,
// validity checks, ramp taps, Parker table, filter spectrum and per-view backprojection
// coefficients. Everything here runs once per plan; the kernels only see the FP32 results.
#pragma once

#include <complex>
#include <string>
#include <vector>

#include "../../include/gct_fdk.h"

namespace gct {

// Mapping families shared by the kernels. The 1D-detector kinds reuse the 2D families with a
// single detector row whose row coordinate is identically 0.
enum class Family : int { Affine = 0, Projective = 1, Arc = 2 };

Family family_of(gct_geom_kind kind);
bool is_2d_detector(gct_geom_kind kind);

// Thrown by the host helpers; the ABI layer turns it into a status + message.
struct GctError {
    gct_status status;
    std::string msg;
};
[[noreturn]] void fail(gct_status s, const std::string &msg);

// Angle wrapping with the reference's semantics (src/cpp/geom/utils.h:322-348): add 2*pi while
// negative, then IEEE remainder() when >= 2*pi.
double wrap_0_2pi(double a);
unsigned quadrant_index(double a);  // src/cpp/geom/utils.h:350-367

struct RotationInfo {
    int dir = GCT_ROT_CW;
    double incr = 0.0;
    double range = 0.0;
    unsigned num_proj_per_rot = 0;
    std::vector<double> rot_ang;
    std::vector<double> rel_rot_ang;
};

// View rotation angle: wrapped rot_ang for parallel kinds, wrapped atan2 of the source
// position otherwise (src/cpp/geom/rotation_geom.cpp:255-295).
double view_rot_angle(gct_geom_kind kind, const gct_view_geom &v);
bool rotation_dir(const std::vector<double> &ang, int *dir);              // rotation_geom.cpp:7-43
bool rel_rot_angles(const std::vector<double> &ang, std::vector<double> *rel);  // :45-74
bool rot_ang_incr(const std::vector<double> &rel, double *incr);          // :76-91
bool rot_ang_range(const std::vector<double> &rel, double *range);        // :93-104
bool num_proj_per_rot(const std::vector<double> &rel, unsigned *n);       // :106-134
bool rotation_info(const gct_ct_geom &g, RotationInfo *out);              // rotation_geom.h:90-115

void check_ct_geom(const gct_ct_geom *g);   // structural checks, throws GctError
void check_vol_geom(const gct_vol_geom *v, bool volume_3d);

gct_view_geom make_view(gct_geom_kind kind, const gct_geom_params &p, unsigned idx);

// Spiral (helical) scans.
struct SpiralInfo {
    unsigned npr = 0;            // projections per rotation
    double pitch = 0.0;          // source z travel per radian (mm)
    std::vector<double> src_z;   // per view
};
SpiralInfo spiral_info(const gct_ct_geom &g);
void spiral_window(const SpiralInfo &si, double slice_pos, long long *first, long long *last);

// Projection matrices of flat-panel views (row-major 3 x 4 matrix, K, R, source), FP64.
struct ProjMatrix {
    double m[12], K[9], R[9], src[3];
};
ProjMatrix decompose_projection_matrix(const double *m);
ProjMatrix compose_projection_matrix(const gct_view_geom &v, double pix_w, double pix_h);
gct_view_geom view_from_projection_matrix(const ProjMatrix &pm);

std::vector<double> ramp_taps(gct_geom_kind kind, const gct_detector &det_row,
                              const gct_filt_params &fp);

// Parker (redundancy) weights [view][col]; see gct_parker_weights in gct_fdk.h.
std::vector<double> parker_table(const gct_ct_geom &g, const RotationInfo &ri);

// Smallest power of two L for which an L-point circular convolution of N samples with the
// N taps (offsets -N/2 .. N-1-N/2) equals the linear one on outputs 0..N-1.
unsigned fft_length(unsigned n);

// L-point spectrum of the circularly placed taps, scaled by 1/L.
std::vector<std::complex<double>> filter_spectrum(const std::vector<double> &taps, unsigned L);

// Per-view data used by the filter kernel (cosine weight) and the backprojector.
struct ViewDerived {
    double c0 = 0, r0 = 0;   // detector centres (pixels)
    double sdd = 0, sid = 0; // source-detector / source-isocentre distances (mm)
    double eu[3] = {0, 0, 0}, ev[3] = {0, 0, 0}, ew[3] = {0, 0, 0};
    double src[3] = {0, 0, 0};
    double theta = 0;        // rot_ang (parallel kinds)
    double bp_const = 1.0;   // constant factor of the backprojection weight folded into the filter
};
ViewDerived derive_view(gct_geom_kind kind, const gct_ct_geom &g, unsigned v);

// kCoefPerView floats per view; the layout depends on the family (see bp_kernels.cuh).
constexpr int kCoefPerView = 20;
std::vector<float> bp_coefficients(const gct_ct_geom &g, const gct_vol_geom &vol,
                                   const std::vector<ViewDerived> &vd,
                                   const std::vector<double> &wscale, bool *z_affine,
                                   std::vector<double> *c64 = nullptr);

// Quarter-turn symmetry of a circular scan on a square grid. Returns +1 when, for every view v
// below 3 nv / 4, view v + nv / 4 maps voxel column R(i, j) = (n - 1 - j, i) exactly where view v
// maps (i, j) (u, v and the weight up to the per-view weight scale), -1 for the opposite turn
// R(i, j) = (j, n - 1 - i), and 0 when neither holds (to 1e-9 of each form's range). c64 are the
// FP64 coefficients of bp_coefficients.
int quarter_turn_symmetry(gct_geom_kind kind, const std::vector<double> &c64, unsigned nv, unsigned nx,
                          unsigned ny, unsigned nz);

// Mirror symmetry in z of a z-affine axial scan (affine or projective family): true when, for
// every view, voxel (i, j, nz - 1 - k) projects onto the same column and weight as (i, j, k) and
// onto the detector row position mirrored about the detector's middle row, v' = nr - 1 - v (the
// source in the grid's middle plane, the detector's row centre on that plane), to 1e-9 of the
// form's range. c64 are the FP64 coefficients of bp_coefficients.
bool z_mirror_symmetry(gct_geom_kind kind, const std::vector<double> &c64, unsigned nv, unsigned nr, unsigned nx,
                       unsigned ny, unsigned nz);

}  // namespace gct
