// Launch interfaces of the ray-driven projection kernels (project.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/gct_fdk.h"

namespace gct {

// Per-view ray geometry in FP64 (device copy of the host derivation).
struct ProjView {
    double src[3];
    double eu[3], ev[3], ew[3];
    double sdd;
    double c0, r0;
    double extra;   // rotation angle (parallel kinds)
    double zscale;  // SID / SDD (cone-parallel)
};

// Voxel-centre bounding box of the reconstruction grid.
struct VolBox {
    double lo[3], hi[3], w[3];
    int nx, ny, nz;
    bool planar;  // 2D image: ignore z
};

void launch_phantom(const ProjView *views, int kind, int nv, int nr, int nc, double du, double dv,
                    const gct_ellipsoid *ell, int ne, bool planar, float *out, int num_sms,
                    cudaStream_t s);

void launch_forward(const ProjView *views, int kind, int nv, int nr, int nc, double du, double dv,
                    const float *vol, const VolBox &box, float step_vox, float *out, int num_sms,
                    cudaStream_t s);

}  // namespace gct
