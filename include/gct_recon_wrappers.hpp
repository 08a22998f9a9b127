// gct_recon_wrappers.hpp -- satidev/gct's reconstruct() overloads on its own types, running on
// this library.
//
// The reference declares seven overloads GCT::Recon::CUDA::reconstruct(AxialCTGeom<...> const &,
// ProjectionStack<float, D> const &, ReconImg<float, D + 1> &) in
// src/cuda/recon/recon_wrappers.cuh:15-43 and defines them, plus a spiral overload on
// SpiralCTGeom<DetFanArc, DetFanLine> that its header does not declare, in
// src/cuda/recon/recon_wrappers.cu:7-63. This header declares the same eight functions with the
// same signatures and, in the one translation unit that defines GCT_RECON_WRAPPERS_DEFINE before
// including it, defines them over the C ABI of gct_fdk.h: the geometry records are copied field
// by field into gct_view_geom, the projections are passed as they are ([view][row][col]), the
// volume comes back through ReconImg::setData ([z][y][x]), and a non-OK status throws
// std::runtime_error with gct_last_error_string(), as the reference's checkError does
// (src/cuda/utils/check_error.cu:6-36). That translation unit replaces recon_wrappers.cu; the
// rest of the reference stays as it is. Needs the reference's src/ on the include path and
// links against libgct_fdk.so.
//
// Like the reference, gct_reconstruct chooses between the whole-stack and the bounded-memory path
// by its 75 % device-memory rule (src/cuda/recon/fdk_axial.cuh:68-89) and runs the FP32 path.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "cpp/data/projection_stack.h"
#include "cpp/data/recon_img.h"
#include "cpp/geom/axial_ct_geom.h"
#include "cpp/geom/detector_1d.h"
#include "cpp/geom/spiral_ct_geom.h"
#include "gct_fdk.h"

namespace GCT::Recon::CUDA
{
void reconstruct(Geom::AxialCTGeom<Geom::DetParallel> const &cg, Data::ProjectionStack<float, 1u> const &proj,
                 Data::ReconImg<float, 2u> &vol);
void reconstruct(Geom::AxialCTGeom<Geom::DetFanArc> const &cg, Data::ProjectionStack<float, 1u> const &proj,
                 Data::ReconImg<float, 2u> &vol);
void reconstruct(Geom::AxialCTGeom<Geom::DetFanLine> const &cg, Data::ProjectionStack<float, 1u> const &proj,
                 Data::ReconImg<float, 2u> &vol);
void reconstruct(Geom::AxialCTGeom<Geom::DetParallel, Geom::DetParallel> const &cg,
                 Data::ProjectionStack<float, 2u> const &proj, Data::ReconImg<float, 3u> &vol);
void reconstruct(Geom::AxialCTGeom<Geom::DetParallel, Geom::DetFanLine> const &cg,
                 Data::ProjectionStack<float, 2u> const &proj, Data::ReconImg<float, 3u> &vol);
void reconstruct(Geom::AxialCTGeom<Geom::DetFanArc, Geom::DetFanLine> const &cg,
                 Data::ProjectionStack<float, 2u> const &proj, Data::ReconImg<float, 3u> &vol);
void reconstruct(Geom::AxialCTGeom<Geom::DetFanLine, Geom::DetFanLine> const &cg,
                 Data::ProjectionStack<float, 2u> const &proj, Data::ReconImg<float, 3u> &vol);
void reconstruct(Geom::SpiralCTGeom<Geom::DetFanArc, Geom::DetFanLine> const &cg,
                 Data::ProjectionStack<float, 2u> const &proj, Data::ReconImg<float, 3u> &vol);
}  // namespace GCT::Recon::CUDA

#ifdef GCT_RECON_WRAPPERS_DEFINE
namespace GCT::Recon::CUDA
{
namespace GctB200
{
// gct_view_geom field groups of the seven ProjGeom specialisations (src/cpp/geom/proj_geom.h:21-103).
inline void put2(double *d, Geom::VecWCS<2u> const &v)
{
    d[0] = v.x.val;
    d[1] = v.y.val;
    d[2] = 0.0;
}
inline void put3(double *d, Geom::VecWCS<3u> const &v)
{
    d[0] = v.x.val;
    d[1] = v.y.val;
    d[2] = v.z.val;
}
inline gct_view_geom view(Geom::ProjGeom<Geom::DetParallel> const &p)
{
    gct_view_geom v{};
    v.rot_ang = p.rot_ang.val;
    v.det_row_center = p.det_row_center.val;
    return v;
}
inline gct_view_geom view(Geom::ProjGeom<Geom::DetFanArc> const &p)
{
    gct_view_geom v{};
    v.src_det_dist = p.src_det_dist.val;
    v.det_row_center = p.det_row_center.val;
    put2(v.src_pos, p.src_pos);
    put2(v.det_row_dir, p.det_row_dir);
    put2(v.iso_ray_dir, p.iso_ray_dir);
    return v;
}
inline gct_view_geom view(Geom::ProjGeom<Geom::DetFanLine> const &p)
{
    gct_view_geom v{};
    v.src_det_dist = p.src_det_dist.val;
    v.det_row_center = p.det_row_center.val;
    put2(v.src_pos, p.src_pos);
    put2(v.det_row_dir, p.det_row_dir);
    return v;
}
inline gct_view_geom view(Geom::ProjGeom<Geom::DetParallel, Geom::DetParallel> const &p)
{
    gct_view_geom v{};
    v.rot_ang = p.rot_ang.val;
    v.det_row_center = p.det_row_center.val;
    v.det_col_center = p.det_col_center.val;
    return v;
}
inline gct_view_geom view(Geom::ProjGeom<Geom::DetParallel, Geom::DetFanLine> const &p)
{
    gct_view_geom v{};
    v.src_det_dist = p.src_det_dist.val;
    v.src_iso_dist = p.src_iso_dist.val;
    v.rot_ang = p.rot_ang.val;
    v.det_row_center = p.det_row_center.val;
    v.det_col_center = p.det_col_center.val;
    return v;
}
inline gct_view_geom view(Geom::ProjGeom<Geom::DetFanArc, Geom::DetFanLine> const &p)
{
    gct_view_geom v{};
    v.src_det_dist = p.src_det_dist.val;
    v.det_row_center = p.det_row_center.val;
    v.det_col_center = p.det_col_center.val;
    put3(v.src_pos, p.src_pos);
    put3(v.det_row_dir, p.det_row_dir);
    put3(v.det_col_dir, p.det_col_dir);
    put3(v.iso_ray_dir, p.iso_ray_dir);
    return v;
}
inline gct_view_geom view(Geom::ProjGeom<Geom::DetFanLine, Geom::DetFanLine> const &p)
{
    gct_view_geom v{};
    v.src_det_dist = p.src_det_dist.val;
    v.det_row_center = p.det_row_center.val;
    v.det_col_center = p.det_col_center.val;
    put3(v.src_pos, p.src_pos);
    put3(v.det_row_dir, p.det_row_dir);
    put3(v.det_col_dir, p.det_col_dir);
    return v;
}

template <class Det>
gct_detector detector(Det const &d)
{
    return gct_detector{d.sampler.num_samples, static_cast<double>(d.sampler.sampling_width.val)};
}

inline gct_vol_geom volume(Geom::ReconImgGeom<2u> const &g)
{
    return gct_vol_geom{g.x.num_samples, g.y.num_samples, 1u, g.x.sampling_width.val, g.y.sampling_width.val, 1.0,
                        {g.mid_point.x.val, g.mid_point.y.val, 0.0}};
}
inline gct_vol_geom volume(Geom::ReconImgGeom<3u> const &g)
{
    return gct_vol_geom{g.x.num_samples,           g.y.num_samples,
                        g.z.num_samples,           g.x.sampling_width.val,
                        g.y.sampling_width.val,    g.z.sampling_width.val,
                        {g.mid_point.x.val, g.mid_point.y.val, g.mid_point.z.val}};
}

// One reconstruction of geometry cg (any CTGeom) of `kind` through gct_reconstruct_ex.
template <class CG, class Proj, class Vol>
void run(CG const &cg, gct_geom_kind kind, int32_t scan, Proj const &proj, Vol &vol)
{
    std::vector<gct_view_geom> views;
    views.reserve(cg.projGeom().size());
    for (auto const &p : cg.projGeom()) views.push_back(view(p));
    gct_ct_geom g{};
    g.kind = kind;
    g.det_row = detector(std::get<0>(cg.detGeom()));
    if constexpr (std::tuple_size_v<std::decay_t<decltype(cg.detGeom())>> > 1)
        g.det_col = detector(std::get<1>(cg.detGeom()));
    else
        g.det_col = gct_detector{1u, 1.0};
    g.num_views = static_cast<uint32_t>(views.size());
    g.views = views.data();
    const gct_vol_geom vg = volume(vol.geom());
    gct_fdk_opts opts{};
    opts.scan = scan;
    std::vector<float> out(vol.numElements());
    if (gct_reconstruct_ex(&g, &vg, nullptr, &opts, proj.elements().data(), out.data()) != GCT_OK)
        throw std::runtime_error(std::string("gct_reconstruct: ") + gct_last_error_string());
    vol.setData(std::move(out));
}
}  // namespace GctB200

void reconstruct(Geom::AxialCTGeom<Geom::DetParallel> const &cg, Data::ProjectionStack<float, 1u> const &proj,
                 Data::ReconImg<float, 2u> &vol)
{
    GctB200::run(cg, GCT_GEOM_PARALLEL_1D, GCT_SCAN_AXIAL, proj, vol);
}
void reconstruct(Geom::AxialCTGeom<Geom::DetFanArc> const &cg, Data::ProjectionStack<float, 1u> const &proj,
                 Data::ReconImg<float, 2u> &vol)
{
    GctB200::run(cg, GCT_GEOM_FAN_ARC, GCT_SCAN_AXIAL, proj, vol);
}
void reconstruct(Geom::AxialCTGeom<Geom::DetFanLine> const &cg, Data::ProjectionStack<float, 1u> const &proj,
                 Data::ReconImg<float, 2u> &vol)
{
    GctB200::run(cg, GCT_GEOM_FAN_LINE, GCT_SCAN_AXIAL, proj, vol);
}
void reconstruct(Geom::AxialCTGeom<Geom::DetParallel, Geom::DetParallel> const &cg,
                 Data::ProjectionStack<float, 2u> const &proj, Data::ReconImg<float, 3u> &vol)
{
    GctB200::run(cg, GCT_GEOM_PARALLEL_2D, GCT_SCAN_AXIAL, proj, vol);
}
void reconstruct(Geom::AxialCTGeom<Geom::DetParallel, Geom::DetFanLine> const &cg,
                 Data::ProjectionStack<float, 2u> const &proj, Data::ReconImg<float, 3u> &vol)
{
    GctB200::run(cg, GCT_GEOM_CONE_PARALLEL, GCT_SCAN_AXIAL, proj, vol);
}
void reconstruct(Geom::AxialCTGeom<Geom::DetFanArc, Geom::DetFanLine> const &cg,
                 Data::ProjectionStack<float, 2u> const &proj, Data::ReconImg<float, 3u> &vol)
{
    GctB200::run(cg, GCT_GEOM_CONE_CYL, GCT_SCAN_AXIAL, proj, vol);
}
void reconstruct(Geom::AxialCTGeom<Geom::DetFanLine, Geom::DetFanLine> const &cg,
                 Data::ProjectionStack<float, 2u> const &proj, Data::ReconImg<float, 3u> &vol)
{
    GctB200::run(cg, GCT_GEOM_CONE_FLAT, GCT_SCAN_AXIAL, proj, vol);
}
void reconstruct(Geom::SpiralCTGeom<Geom::DetFanArc, Geom::DetFanLine> const &cg,
                 Data::ProjectionStack<float, 2u> const &proj, Data::ReconImg<float, 3u> &vol)
{
    GctB200::run(cg, GCT_GEOM_CONE_CYL, GCT_SCAN_SPIRAL, proj, vol);
}
}  // namespace GCT::Recon::CUDA
#endif  // GCT_RECON_WRAPPERS_DEFINE
