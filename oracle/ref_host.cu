// Host-side harness over satidev/gct's own host-callable functions (TEST INFRASTRUCTURE ONLY).
//
// oracle/build_ref.sh compiles this file together with the reference sources, in place under the
// reference tree, into oracle/_ref/libgct_ref_host.so. The library exposes plain C entry points so
// that the tests and tests/golden/make_golden.py can evaluate the reference's FP32 arithmetic
// (ramp taps, rotation analysis, Parker and cosine weights, projMapping, voxel positions) and pin
// the FP64 oracle to it. The per-element math is the reference's; this file only marshals
// arguments, the way the reference's device-side copy (src/cuda/geom/ct_geom_dev.cu:7-447) and
// getParkerWeights (src/cuda/recon/parker_weighting.cuh:132-176) do.
#include <algorithm>
#include <cmath>
#include <vector>

#include "cpp/geom/axial_ct_geom.h"
#include "cpp/geom/ct_geom.h"
#include "cpp/geom/rotation_geom.h"
#include "cpp/recon/proj_filt_kernel.h"
#include "cuda/geom/coord_trans_img.cuh"
#include "cuda/geom/coord_trans_proj.cuh"
#include "cuda/recon/cos_weighting.cuh"
#include "cuda/recon/parker_weighting.cuh"

using namespace GCT;
using namespace GCT::Geom;

namespace {
Recon::FiltParams filt(float fc, int apod)
{
    Recon::FiltParams p{};
    p.cut_off_freq = fc;
    p.apod_func = apod == 1 ? Recon::ApodFunc::HANN : apod == 2 ? Recon::ApodFunc::HAMMING : Recon::ApodFunc::NONE;
    return p;
}

float norm2(float x, float y) { return std::sqrt(x * x + y * y); }
float norm3(const float *v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
}  // namespace

extern "C" {

// kind: 0 parallel (DetParallel), 1 arc (DetFanArc), 2 line (DetFanLine)
int ref_filter_taps(int kind, unsigned n, float width, float fc, int apod, float *out)
{
    std::vector<float> t;
    if (kind == 1) t = Recon::projFiltKernel(DetFanArc{EqAngSampler{n, Units::Radians{width}}}, filt(fc, apod));
    else if (kind == 2) t = Recon::projFiltKernel(DetFanLine{EqDistSampler{n, Units::MilliMeters{width}}}, filt(fc, apod));
    else t = Recon::projFiltKernel(DetParallel{EqDistSampler{n, Units::MilliMeters{width}}}, filt(fc, apod));
    std::copy(t.begin(), t.end(), out);
    return static_cast<int>(t.size());
}

// Rotation analysis of n parallel-beam views with the given rotation angles.
int ref_rotation(const float *ang, unsigned n, int *dir, float *incr, float *range, unsigned *nppr, float *rel)
{
    std::vector<ProjGeom<DetParallel>> pg(n);
    for (unsigned i = 0; i < n; ++i) pg[i].rot_ang = Units::Radians{ang[i]};
    const auto info = getRotationGeom(pg);
    if (!info) return -1;
    *dir = static_cast<int>(info->dir);
    *incr = info->rot_ang_incr.val;
    *range = info->rot_ang_range.val;
    *nppr = info->num_proj_per_rot;
    for (unsigned i = 0; i < n; ++i) rel[i] = info->rel_rot_ang[i].val;
    return 0;
}

float ref_parker_weight_fan(float fan, float det_fan, float rel, float range)
{
    return Recon::CUDA::Detail::parkerWeightFan(fan, det_fan, rel, range);
}

// Parker table [nv][nc] of a fan-beam scan (arc = 1: DetFanArc, else DetFanLine) given per-view
// source positions (x, y) and row directions, evaluated on the host with the reference's functions.
int ref_parker_table(int arc, unsigned nc, float width, unsigned nv, const float *src_xy, const float *row_xy,
                     float row_center, float sdd, float *out)
{
    auto run = [&](auto det) {
        using Det = decltype(det);
        std::vector<ProjGeom<Det>> pg(nv);
        for (unsigned v = 0; v < nv; ++v) {
            pg[v].src_det_dist = Units::MilliMeters{sdd};
            pg[v].det_row_center = Units::DetPixels{row_center};
            pg[v].src_pos = VecWCS<2u>{src_xy[2 * v], src_xy[2 * v + 1]};
            pg[v].det_row_dir = VecWCS<2u>{row_xy[2 * v], row_xy[2 * v + 1]};
            if constexpr (std::is_same_v<Det, DetFanArc>)
                pg[v].iso_ray_dir = VecWCS<2u>{-row_xy[2 * v + 1], row_xy[2 * v]};
        }
        const CTGeom<Det> cg{std::make_tuple(det), pg};
        const auto fan = Recon::CUDA::Detail::fanAngles(cg);
        const float det_fan = Recon::CUDA::Detail::fanAngleDet(det, cg.projGeom().front());
        std::vector<float> rel;
        for (const auto &a : cg.rotationGeom().rel_rot_ang) rel.push_back(a.val);
        if (cg.rotationGeom().dir == RotDir::CCW) std::reverse(rel.begin(), rel.end());
        const float range = cg.rotationGeom().rot_ang_range.val;
        for (unsigned v = 0; v < nv; ++v)
            for (unsigned c = 0; c < nc; ++c)
                out[v * nc + c] = Recon::CUDA::Detail::parkerWeightFan(fan[c], det_fan, rel[v], range);
        return 0;
    };
    if (arc) return run(DetFanArc{EqAngSampler{nc, Units::Radians{width}}});
    return run(DetFanLine{EqDistSampler{nc, Units::MilliMeters{width}}});
}

// Per-view record (floats): rot_ang, det_row_center, det_col_center, src_det_dist, src_iso_dist,
// src_pos[3], det_row_dir[3], det_col_dir[3], iso_ray_dir[3]; kind as gct_geom_kind.
// Fills one-view ProjGeomScanDev structs the way CTGeomDev does and evaluates cosWeight at
// (col, row) and projMapping at (x, y, z). Returns the backprojection weight.
float ref_view_eval(int kind, const float *r, float du, float dv, unsigned col, unsigned row, float x, float y,
                    float z, float *cosw, float *u_out, float *t_out)
{
    float rot = r[0], rc = r[1], cc = r[2], sdd = r[3], sid_p = r[4];
    const float *s = r + 5, *ru = r + 8, *rv = r + 11, *iso = r + 14;
    float w = 0.f;
    *t_out = 0.f;
    using namespace Geom::CUDA;
    switch (kind) {
        case 0: {
            ProjGeomScanDev<DetParallel> pg{&rot, &rc};
            DetParallel dr{EqDistSampler{1, Units::MilliMeters{du}}};
            *cosw = Recon::CUDA::Detail::cosWeight(&dr, &pg, 0, col);
            *u_out = projMapping(make_float2(x, y), &pg, 0, w);
            return w;
        }
        case 1: {
            float sid = norm2(s[0], s[1]);
            float2 sp = make_float2(s[0], s[1]), iv = make_float2(iso[0], iso[1]), rd = make_float2(ru[0], ru[1]);
            ProjGeomScanDev<DetFanArc> pg{&sdd, &sid, &rc, &sp, &iv, &rd};
            DetFanArc dr{EqAngSampler{1, Units::Radians{du}}};
            *cosw = Recon::CUDA::Detail::cosWeight(&dr, &pg, 0, col);
            *u_out = projMapping(make_float2(x, y), &pg, 0, w);
            return w;
        }
        case 2: {
            float sid = norm2(s[0], s[1]);
            float2 sp = make_float2(s[0], s[1]), rd = make_float2(ru[0], ru[1]), iv = make_float2(-ru[1], ru[0]);
            ProjGeomScanDev<DetFanLine> pg{&sdd, &sid, &rc, &sp, &rd, &iv};
            DetFanLine dr{EqDistSampler{1, Units::MilliMeters{du}}};
            *cosw = Recon::CUDA::Detail::cosWeight(&dr, &pg, 0, col);
            *u_out = projMapping(make_float2(x, y), &pg, 0, w);
            return w;
        }
        case 3: {
            ProjGeomScanDev<DetParallel, DetParallel> pg{&rot, &rc, &cc};
            DetParallel dr{EqDistSampler{1, Units::MilliMeters{du}}}, dc{EqDistSampler{1, Units::MilliMeters{dv}}};
            *cosw = Recon::CUDA::Detail::cosWeight(&dr, &dc, &pg, 0, col, row);
            const float2 d = projMapping(make_float3(x, y, z), &pg, 0, w);
            *u_out = d.x;
            *t_out = d.y;
            return w;
        }
        case 4: {
            ProjGeomScanDev<DetParallel, DetFanLine> pg{&sdd, &sid_p, &rot, &rc, &cc};
            DetParallel dr{EqDistSampler{1, Units::MilliMeters{du}}};
            DetFanLine dc{EqDistSampler{1, Units::MilliMeters{dv}}};
            *cosw = Recon::CUDA::Detail::cosWeight(&dr, &dc, &pg, 0, col, row);
            const float2 d = projMapping(make_float3(x, y, z), &pg, 0, w);
            *u_out = d.x;
            *t_out = d.y;
            return w;
        }
        case 5: {
            float sid = norm3(s);
            float3 sp = make_float3(s[0], s[1], s[2]), rd = make_float3(ru[0], ru[1], ru[2]);
            float3 cd = make_float3(rv[0], rv[1], rv[2]), iv = make_float3(iso[0], iso[1], iso[2]);
            ProjGeomScanDev<DetFanArc, DetFanLine> pg{&sdd, &sid, &rc, &cc, &sp, &rd, &cd, &iv};
            DetFanArc dr{EqAngSampler{1, Units::Radians{du}}};
            DetFanLine dc{EqDistSampler{1, Units::MilliMeters{dv}}};
            *cosw = Recon::CUDA::Detail::cosWeight(&dr, &dc, &pg, 0, col, row);
            const float2 d = projMapping(make_float3(x, y, z), &pg, 0, w);
            *u_out = d.x;
            *t_out = d.y;
            return w;
        }
        default: {
            float sid = norm3(s);
            float3 sp = make_float3(s[0], s[1], s[2]), rd = make_float3(ru[0], ru[1], ru[2]);
            float3 cd = make_float3(rv[0], rv[1], rv[2]);
            float3 sdir = make_float3(rd.y * cd.z - rd.z * cd.y, rd.z * cd.x - rd.x * cd.z, rd.x * cd.y - rd.y * cd.x);
            ProjGeomScanDev<DetFanLine, DetFanLine> pg{&sdd, &sid, &rc, &cc, &sp, &rd, &cd, &sdir,
                                                       nullptr, nullptr, nullptr};
            DetFanLine dr{EqDistSampler{1, Units::MilliMeters{du}}}, dc{EqDistSampler{1, Units::MilliMeters{dv}}};
            *cosw = Recon::CUDA::Detail::cosWeight(&dr, &dc, &pg, 0, col, row);
            const float2 d = projMapping(make_float3(x, y, z), &pg, 0, w);
            *u_out = d.x;
            *t_out = d.y;
            return w;
        }
    }
}

// voxPosWCS of voxel (i, j, k) of a 3D grid (src/cuda/geom/coord_trans_img.cuh:100-106).
void ref_vox_pos(unsigned nx, unsigned ny, unsigned nz, float dx, float dy, float dz, float mx, float my, float mz,
                 unsigned i, unsigned j, unsigned k, float *out)
{
    ReconImgGeom<3u> rg{EqDistSampler{nx, Units::MilliMeters{dx}}, EqDistSampler{ny, Units::MilliMeters{dy}},
                        EqDistSampler{nz, Units::MilliMeters{dz}}, VecWCS<3u>{mx, my, mz}};
    const float3 p = Geom::CUDA::voxPosWCS(&rg, make_uint3(i, j, k));
    out[0] = p.x;
    out[1] = p.y;
    out[2] = p.z;
}

}  // extern "C"
