// Runs satidev/gct's own CUDA FDK (GCT::Recon::CUDA::reconstruct, src/cuda/recon/recon_wrappers.cu)
// on a geometry and projection stack read from a file, and writes the volume.
// TEST INFRASTRUCTURE ONLY: built by oracle/build_ref.sh into oracle/_ref/ref_fdk from the
// reference sources in place; the GPU parity tests run it beside the engine on identical inputs.
//
// Input file (little endian): int32 kind, nc, nr, nv, nx, ny, nz; float32 du, dv, dx, dy, dz, mx,
// my, mz; nv records of 17 float32 (rot_ang, det_row_center, det_col_center, src_det_dist,
// src_iso_dist, src_pos[3], det_row_dir[3], det_col_dir[3], iso_ray_dir[3]); nv*nr*nc float32
// projections. Output file: nz*ny*nx float32 (nz = 1 for 2D images).
//
// The reference composes a projection matrix per flat-detector view (ct_geom_dev.cu:421-441) that no
// kernel reads; its constructor needs Eigen, so this harness defines it as leaving the matrix zero.
// The cross product used for the flat detector's normal (ct_geom_dev.cu:407) is computed here in
// FP32, as the reference's Eigen call would.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <stdexcept>
#include <vector>

#include "cpp/geom/axial_ct_geom.h"
#include "cpp/geom/geom_math.h"
#include "cpp/geom/projection_matrix.h"
#include "cpp/recon/check_validity.h"
#include "cuda/recon/recon_wrappers.cuh"

using namespace GCT;
using namespace GCT::Geom;

namespace GCT::Geom {
ProjectionMatrix::ProjectionMatrix(ProjGeom<DetFanLine, DetFanLine> const &, float, float) {}
namespace Math {
VecWCS<3u> crossProduct(VecWCS<3u> const &a, VecWCS<3u> const &b)
{
    return VecWCS<3u>{a.y.val * b.z.val - a.z.val * b.y.val, a.z.val * b.x.val - a.x.val * b.z.val,
                      a.x.val * b.y.val - a.y.val * b.x.val};
}
}  // namespace Math
}  // namespace GCT::Geom

namespace {
struct Rec {
    float rot, rc, cc, sdd, sid, s[3], ru[3], rv[3], iso[3];
};
VecWCS<2u> v2(const float *p) { return VecWCS<2u>{p[0], p[1]}; }
VecWCS<3u> v3(const float *p) { return VecWCS<3u>{p[0], p[1], p[2]}; }
Units::MilliMeters mm(float x) { return Units::MilliMeters{x}; }
Units::DetPixels px(float x) { return Units::DetPixels{x}; }

template <class PG>
PG make(const Rec &r);
template <> ProjGeom<DetParallel> make(const Rec &r) { return {Units::Radians{r.rot}, px(r.rc)}; }
template <> ProjGeom<DetFanArc> make(const Rec &r) { return {mm(r.sdd), px(r.rc), v2(r.s), v2(r.ru), v2(r.iso)}; }
template <> ProjGeom<DetFanLine> make(const Rec &r) { return {mm(r.sdd), px(r.rc), v2(r.s), v2(r.ru)}; }
template <> ProjGeom<DetParallel, DetParallel> make(const Rec &r) { return {Units::Radians{r.rot}, px(r.rc), px(r.cc)}; }
template <> ProjGeom<DetParallel, DetFanLine> make(const Rec &r)
{
    return {mm(r.sdd), mm(r.sid), Units::Radians{r.rot}, px(r.rc), px(r.cc)};
}
template <> ProjGeom<DetFanArc, DetFanLine> make(const Rec &r)
{
    return {mm(r.sdd), px(r.rc), px(r.cc), v3(r.s), v3(r.ru), v3(r.rv), v3(r.iso)};
}
template <> ProjGeom<DetFanLine, DetFanLine> make(const Rec &r)
{
    return {mm(r.sdd), px(r.rc), px(r.cc), v3(r.s), v3(r.ru), v3(r.rv)};
}

template <class Det> Det det(unsigned n, float w);
template <> DetParallel det(unsigned n, float w) { return DetParallel{EqDistSampler{n, mm(w)}}; }
template <> DetFanLine det(unsigned n, float w) { return DetFanLine{EqDistSampler{n, mm(w)}}; }
template <> DetFanArc det(unsigned n, float w) { return DetFanArc{EqAngSampler{n, Units::Radians{w}}}; }

struct Input {
    int kind, nc, nr, nv, nx, ny, nz;
    float du, dv, dx, dy, dz, mx, my, mz;
    std::vector<Rec> recs;
    std::vector<float> proj;
};

template <class DetRow>
std::vector<float> run1d(const Input &in)
{
    std::vector<ProjGeom<DetRow>> pg;
    for (const Rec &r : in.recs) pg.push_back(make<ProjGeom<DetRow>>(r));
    const AxialCTGeom<DetRow> cg{std::make_tuple(det<DetRow>(in.nc, in.du)), pg};
    Data::ProjectionStack<float, 1u> proj{Data::ProjSize<1u>{static_cast<unsigned>(in.nc)},
                                          static_cast<unsigned>(in.nv)};
    proj.setData(in.proj);
    const ReconImgGeom<2u> rg{EqDistSampler{static_cast<unsigned>(in.nx), mm(in.dx)},
                              EqDistSampler{static_cast<unsigned>(in.ny), mm(in.dy)}, VecWCS<2u>{in.mx, in.my}};
    Data::ReconImg<float, 2u> vol{rg};
    if (!Recon::isValidAxialRecon(cg, proj, true)) throw std::runtime_error("invalid reconstruction input");
    Recon::CUDA::reconstruct(cg, proj, vol);
    return vol.elements();
}

template <class DetRow, class DetCol>
std::vector<float> run2d(const Input &in)
{
    std::vector<ProjGeom<DetRow, DetCol>> pg;
    for (const Rec &r : in.recs) pg.push_back(make<ProjGeom<DetRow, DetCol>>(r));
    const AxialCTGeom<DetRow, DetCol> cg{std::make_tuple(det<DetRow>(in.nc, in.du), det<DetCol>(in.nr, in.dv)), pg};
    Data::ProjectionStack<float, 2u> proj{
        Data::ProjSize<2u>{static_cast<unsigned>(in.nc), static_cast<unsigned>(in.nr)}, static_cast<unsigned>(in.nv)};
    proj.setData(in.proj);
    const ReconImgGeom<3u> rg{EqDistSampler{static_cast<unsigned>(in.nx), mm(in.dx)},
                              EqDistSampler{static_cast<unsigned>(in.ny), mm(in.dy)},
                              EqDistSampler{static_cast<unsigned>(in.nz), mm(in.dz)}, VecWCS<3u>{in.mx, in.my, in.mz}};
    Data::ReconImg<float, 3u> vol{rg};
    if (!Recon::isValidAxialRecon(cg, proj, true)) throw std::runtime_error("invalid reconstruction input");
    Recon::CUDA::reconstruct(cg, proj, vol);
    return vol.elements();
}
}  // namespace

int main(int argc, char **argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
        return 2;
    }
    try {
        std::ifstream f(argv[1], std::ios::binary);
        Input in{};
        int32_t hdr[7];
        float fl[8];
        f.read(reinterpret_cast<char *>(hdr), sizeof(hdr));
        f.read(reinterpret_cast<char *>(fl), sizeof(fl));
        in.kind = hdr[0], in.nc = hdr[1], in.nr = hdr[2], in.nv = hdr[3], in.nx = hdr[4], in.ny = hdr[5], in.nz = hdr[6];
        in.du = fl[0], in.dv = fl[1], in.dx = fl[2], in.dy = fl[3], in.dz = fl[4], in.mx = fl[5], in.my = fl[6],
        in.mz = fl[7];
        in.recs.resize(in.nv);
        f.read(reinterpret_cast<char *>(in.recs.data()), sizeof(Rec) * in.nv);
        in.proj.resize(static_cast<size_t>(in.nv) * in.nr * in.nc);
        f.read(reinterpret_cast<char *>(in.proj.data()), sizeof(float) * in.proj.size());
        if (!f) throw std::runtime_error("short input file");
        std::vector<float> out;
        switch (in.kind) {
            case 0: out = run1d<DetParallel>(in); break;
            case 1: out = run1d<DetFanArc>(in); break;
            case 2: out = run1d<DetFanLine>(in); break;
            case 3: out = run2d<DetParallel, DetParallel>(in); break;
            case 4: out = run2d<DetParallel, DetFanLine>(in); break;
            case 5: out = run2d<DetFanArc, DetFanLine>(in); break;
            case 6: out = run2d<DetFanLine, DetFanLine>(in); break;
            default: throw std::runtime_error("unknown kind");
        }
        std::ofstream o(argv[2], std::ios::binary);
        o.write(reinterpret_cast<const char *>(out.data()), sizeof(float) * out.size());
        return o ? 0 : 1;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_fdk: %s\n", e.what());
        return 1;
    }
}
