// Calls GCT::Recon::CUDA::reconstruct on the reference's own types, with the definitions of
// include/gct_recon_wrappers.hpp (this library in place of the reference's recon_wrappers.cu):
// the check that the drop-in compiles against satidev/gct's headers, and what its overloads
// return on the GPU. TEST INFRASTRUCTURE ONLY: built by oracle/build_ref.sh into
// oracle/_ref/ref_wrappers where the reference tree exists.
//
//   ref_wrappers [--spiral] input.bin output.bin
//
// Input: the format of ref_input.hpp (the same files ref_fdk reads). Output: nz*ny*nx float32.
// The reference's callers validate first (isValidAxialRecon, src/cpp/recon/check_validity.h:
// 66-75); so does this program.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>

#include "cpp/recon/check_validity.h"
#include "ref_input.hpp"

#define GCT_RECON_WRAPPERS_DEFINE
#include "gct_recon_wrappers.hpp"

using namespace ref_input;

namespace {

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
    int a = 1;
    if (a < argc && std::strcmp(argv[a], "--spiral") == 0) {
        // The spiral overload's parameter type, SpiralCTGeom, cannot be constructed in the
        // reference: its constructor does not compile (src/cpp/geom/spiral_ct_geom.h:81-94). The
        // overload is declared and defined by gct_recon_wrappers.hpp all the same.
        std::fprintf(stderr, "ref_wrappers: SpiralCTGeom cannot be constructed from the reference's sources\n");
        return 3;
    }
    if (argc - a != 2) {
        std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
        return 2;
    }
    try {
        const Input in = read_input(argv[a]);
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
        std::ofstream o(argv[a + 1], std::ios::binary);
        o.write(reinterpret_cast<const char *>(out.data()), sizeof(float) * out.size());
        return o ? 0 : 1;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_wrappers: %s\n", e.what());
        return 1;
    }
}
