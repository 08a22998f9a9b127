// gct_fdk.hpp -- header-only C++ layer over the C ABI in gct_fdk.h.
//
// Restores the reference's calling convention: failures throw std::runtime_error (as
// src/cuda/utils/check_error.cu:6-36 does), plans are RAII objects, and reconstruct() takes the
// geometry, the projection stack and the output image like GCT::Recon::CUDA::reconstruct
// (src/cuda/recon/recon_wrappers.cuh:15-43).
#pragma once

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "gct_fdk.h"

namespace gct {

inline void check(gct_status s)
{
    if (s != GCT_OK) throw std::runtime_error(std::string("gct_fdk: ") + gct_last_error_string());
}

// Geometry of an axial scan: detector samplers plus one record per view (owned).
struct CTGeom {
    gct_geom_kind kind = GCT_GEOM_CONE_FLAT;
    gct_detector det_row{0, 0.0};
    gct_detector det_col{1, 1.0};
    std::vector<gct_view_geom> views;

    gct_ct_geom c_view() const
    {
        gct_ct_geom g{};
        g.kind = kind;
        g.det_row = det_row;
        g.det_col = det_col;
        g.num_views = static_cast<uint32_t>(views.size());
        g.views = views.data();
        return g;
    }

    // ProjGeomFactory<DetRow, DetCol...>::create(params, i) for i < params.num_proj.
    static CTGeom from_params(gct_geom_kind kind, gct_detector det_row, gct_detector det_col,
                              const gct_geom_params &p)
    {
        CTGeom g;
        g.kind = kind;
        g.det_row = det_row;
        g.det_col = det_col;
        g.views.resize(p.num_proj);
        for (uint32_t i = 0; i < p.num_proj; ++i) check(gct_proj_geom_create(kind, &p, i, &g.views[i]));
        gct_rotation_geom rg{};
        const gct_ct_geom c = g.c_view();
        check(gct_rotation_geom_get(&c, &rg, nullptr, nullptr));  // throws for an invalid trajectory
        return g;
    }
};

// Host drop-in: vol receives nx*ny*nz floats ([z][y][x]); proj holds nv*nr*nc floats.
inline void reconstruct(const CTGeom &g, const gct_vol_geom &vol, const std::vector<float> &proj,
                        std::vector<float> &out, const gct_filt_params *filt = nullptr,
                        const gct_fdk_opts *opts = nullptr)
{
    const gct_ct_geom c = g.c_view();
    const size_t need = static_cast<size_t>(c.num_views) * c.det_col.num_samples * c.det_row.num_samples;
    if (proj.size() != need) throw std::invalid_argument("projection stack size does not match the geometry");
    out.resize(static_cast<size_t>(vol.nx) * vol.ny * vol.nz);
    check(gct_reconstruct_ex(&c, &vol, filt, opts, proj.data(), out.data()));
}

// Device plan (RAII).
class FdkPlan {
public:
    FdkPlan(const CTGeom &g, const gct_vol_geom &vol, const gct_filt_params *filt = nullptr,
            const gct_fdk_opts *opts = nullptr)
    {
        const gct_ct_geom c = g.c_view();
        check(gct_fdk_plan_create(&c, &vol, filt, opts, &plan_));
    }
    FdkPlan(const FdkPlan &) = delete;
    FdkPlan &operator=(const FdkPlan &) = delete;
    FdkPlan(FdkPlan &&o) noexcept : plan_(std::exchange(o.plan_, nullptr)) {}
    ~FdkPlan()
    {
        if (plan_) gct_fdk_plan_destroy(plan_);
    }

    uint64_t workspace_bytes() const
    {
        uint64_t b = 0;
        check(gct_fdk_plan_workspace_bytes(plan_, &b));
        return b;
    }
    void execute(const float *proj_dev, float *vol_dev, void *workspace = nullptr, void *stream = nullptr)
    {
        check(gct_fdk_execute(plan_, proj_dev, vol_dev, workspace, stream));
    }
    void execute_host(const float *proj_host, float *vol_host, void *stream = nullptr)
    {
        check(gct_fdk_execute_host(plan_, proj_host, vol_host, stream));
    }
    gct_fdk_plan *get() const { return plan_; }

private:
    gct_fdk_plan *plan_ = nullptr;
};

}  // namespace gct
