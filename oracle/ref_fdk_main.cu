// Runs satidev/gct's own CUDA FDK (GCT::Recon::CUDA::reconstruct, src/cuda/recon/recon_wrappers.cu)
// on a geometry and projection stack read from a file, and writes the volume.
// TEST INFRASTRUCTURE ONLY: built by oracle/build_ref.sh into oracle/_ref/ref_fdk from the
// reference sources in place; the GPU parity tests run it beside the engine on identical inputs.
//
//   ref_fdk [--repeat K] in.bin out.bin       the reference's reconstruct() (K runs, wall times on
//                                             stderr: host buffers in and out, as the reference does)
//   ref_fdk --spiral in.bin out.bin           its spiral FDK (fdk_spiral.cuh:33-94, cylindrical
//                                             detector, kind 5) through its own stage functions;
//                                             see fdk_spiral_stages for why not its overload
//   ref_fdk --bp MODE in.bin out.bin          the reference's stage sequence of reconFDKHighMem
//                                             (fdk_axial.cuh:151-205: its cosine and Parker weights,
//                                             its cuFFT ramp filter, its projMapping/DCSToPCS per voxel
//                                             and view, view by view), except that the texture fetch
//                                             of backProjKern (back_proj.cuh:16-79) is replaced by a
//                                             bilinear interpolation of the same filtered view in
//                                             global memory: MODE exact (FP32 weights) or texture
//                                             (the texture unit's 1/256 weight rule, see lerp2).
//                                             This isolates the texture unit's weight quantisation
//                                             from everything else.
//   ref_fdk --texprobe in.bin out.bin         fetches through the reference's own texture objects
//                                             (NDArrayTexture, nd_array_texture.cuh:33-56, filled by
//                                             copyDevToDevTexture) at given coordinates. Input: int32
//                                             dim (1 or 2), width, height, n; float32 texels
//                                             [height][width]; float32 n (x, y) coordinates as passed
//                                             to tex1D / tex2D. Output: n float32 fetched values.
//
// Input file: the format of ref_input.hpp. Output file: nz*ny*nx float32 (nz = 1 for 2D images).
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
#include "cuda/recon/fdk_axial.cuh"
#include "ref_input.hpp"

#include <chrono>
#include <cstring>
#include <string>


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
using namespace ref_input;

// ---- bilinear interpolation in place of the texture fetch (--bp) ------------------------------
enum BpMode { kBpExact = 0, kBpTexture = 1 };

__device__ __forceinline__ float q256(float v) { return floorf(v * 256.f + 0.5f) * (1.f / 256.f); }

__device__ __forceinline__ float texel(const float *img, int w, int h, int i, int j)
{
    return (i >= 0 && i < w && j >= 0 && j < h) ? img[static_cast<size_t>(j) * w + i] : 0.f;  // border 0
}

// Bilinear sample at texture coordinates (tx, ty) (the values passed to tex1D / tex2D, which
// include the reference's +0.5: the linear filter interpolates between texels floor(t - 0.5) and
// floor(t - 0.5) + 1). kBpExact: FP32 weights. kBpTexture: the texture unit's rule as measured
// through the reference's own texture objects (tests/golden/tex_probe.npz): the sample position
// snaps to the nearest 1/256 of a texel on each axis, and the corner weight a b also snaps to the
// nearest 1/256, the other three weights being a - w11, b - w11 and 1 - a - b + w11.
__device__ float lerp2(const float *img, int w, int h, float tx, float ty, int mode)
{
    float x = tx - 0.5f, y = ty - 0.5f;
    if (mode == kBpTexture) {
        x = q256(x);
        y = q256(y);
    }
    const float fx = floorf(x), fy = floorf(y);
    const int i = static_cast<int>(fx), j = static_cast<int>(fy);
    const float a = x - fx, b = y - fy;
    const float w11 = mode == kBpTexture ? q256(a * b) : a * b;
    const float w01 = a - w11, w10 = b - w11, w00 = 1.f - a - b + w11;
    return w00 * texel(img, w, h, i, j) + w01 * texel(img, w, h, i + 1, j) + w10 * texel(img, w, h, i, j + 1) +
           w11 * texel(img, w, h, i + 1, j + 1);
}

// backProjKern (back_proj.cuh:16-42) with the fetch replaced by lerp2 on the view in memory.
template <typename DetRow>
__global__ void bp_manual_2d(DetRow const *dr, Geom::CUDA::ProjGeomScanDev<DetRow> const *pg, unsigned proj_idx,
                             const float *view, int nc, Geom::ReconImgGeom<2u> const *rg, float *img, int mode)
{
    const unsigned col_idx = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned row_idx = blockIdx.y * blockDim.y + threadIdx.y;
    if (col_idx >= rg->x.num_samples || row_idx >= rg->y.num_samples) return;
    using namespace GCT::Geom::CUDA;
    const auto pix = pixPosWCS(rg, uint2{col_idx, row_idx});
    auto w = 1.0f;
    const auto det = projMapping(pix, pg, proj_idx, w);
    const auto p = DCSToPCS(det, dr->sampler.sampling_width.val, pg->det_row_center[proj_idx]);
    img[row_idx * rg->x.num_samples + col_idx] += lerp2(view, nc, 1, p + 0.5f, 0.5f, mode) * w;
}

// backProjKern (back_proj.cuh:44-79) with the fetch replaced by lerp2 on the view in memory.
template <typename DetRow, typename DetCol>
__global__ void bp_manual_3d(DetRow const *dr, DetCol const *dc, Geom::CUDA::ProjGeomScanDev<DetRow, DetCol> const *pg,
                             unsigned proj_idx, const float *view, int nc, int nr, Geom::ReconImgGeom<3u> const *rg,
                             float *vol, int mode)
{
    const unsigned col_idx = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned row_idx = blockIdx.y * blockDim.y + threadIdx.y;
    const unsigned slice_idx = blockIdx.z * blockDim.z + threadIdx.z;
    if (col_idx >= rg->x.num_samples || row_idx >= rg->y.num_samples || slice_idx >= rg->z.num_samples) return;
    using namespace GCT::Geom::CUDA;
    const auto pos = voxPosWCS(rg, uint3{col_idx, row_idx, slice_idx});
    auto w = 1.0f;
    const auto det = projMapping(pos, pg, proj_idx, w);
    const auto col = DCSToPCS(det.x, dr->sampler.sampling_width.val, pg->det_row_center[proj_idx]);
    const auto row = DCSToPCS(det.y, dc->sampler.sampling_width.val, pg->det_col_center[proj_idx]);
    const size_t at = (static_cast<size_t>(slice_idx) * rg->y.num_samples + row_idx) * rg->x.num_samples + col_idx;
    vol[at] += lerp2(view, nc, nr, col + 0.5f, row + 0.5f, mode) * w;
}
}  // namespace

namespace GCT::Recon::CUDA {
// reconFDKHighMem (fdk_axial.cuh:151-205) step for step through the reference's own functions,
// with bp_manual_* in place of backProjVoxDriven.
template <typename DetRow, typename... DetCol>
std::vector<float> fdk_manual_bp(Geom::AxialCTGeom<DetRow, DetCol...> const &cg_host,
                                 Data::ProjectionStack<float, Data::projDim<DetCol...>()> const &proj_all_host,
                                 Geom::ReconImgGeom<Data::reconImgDim<DetCol...>()> const &rg_host, int mode)
{
    constexpr auto proj_dim = Data::projDim<DetCol...>();
    constexpr auto recon_dim = Data::reconImgDim<DetCol...>();
    auto const ct_geom_dev = Geom::CUDA::CTGeomDev<DetRow, DetCol...>{cg_host};
    auto proj_dev = Data::CUDA::ProjectionStack<float, proj_dim, Data::CUDA::DevMem<float>>{
        proj_all_host.projSize(), proj_all_host.numProj()};
    Data::CUDA::copyHostToDev(proj_all_host.elements(), proj_dev);
    {
        runCosWeighting(ct_geom_dev, proj_dev);
        auto const parker_weights = CUDA::getParkerWeights(cg_host);
        runParkerWeighting(parker_weights, proj_dev);
        auto const num_rows_filt = Data::numProjRows(proj_all_host.projSize()) * proj_all_host.numProj();
        auto rf = RampFilteringFFT{std::get<0>(cg_host.detGeom()), FiltParams{}, num_rows_filt};
        rf.runFiltering(proj_dev);
    }
    auto img_dev = Data::CUDA::ReconImg<float, recon_dim, Data::CUDA::DevMem<float>>{rg_host};
    img_dev.setVal(0.0f);
    auto const config = GCT::CUDA::execConfig(img_dev.dimensions());
    const auto &dg = ct_geom_dev.detGeom();
    const int nc = static_cast<int>(std::get<0>(cg_host.detGeom()).sampler.num_samples);
    const size_t pix = Data::numProjPixels(proj_all_host.projSize());
    for (auto proj_idx = 0u; proj_idx < proj_all_host.numProj(); proj_idx++) {
        const float *view = proj_dev.dataPointer() + proj_idx * pix;
        if constexpr (recon_dim == 2u) {
            bp_manual_2d<<<config.first, config.second>>>(dg.detRow(), ct_geom_dev.projGeom(), proj_idx, view, nc,
                                                          img_dev.geom(), img_dev.dataPointer(), mode);
        } else {
            const int nr = static_cast<int>(pix / nc);
            bp_manual_3d<<<config.first, config.second>>>(dg.detRow(), dg.detCol(), ct_geom_dev.projGeom(), proj_idx,
                                                          view, nc, nr, img_dev.geom(), img_dev.dataPointer(), mode);
        }
        GCT::CUDA::checkErrorKernel("manual backprojection");
    }
    auto const rot_ang_incr = cg_host.rotationGeom().rot_ang_incr;
    if (rot_ang_incr > Geom::Units::Radians{0.0f}) img_dev *= rot_ang_incr.val;
    auto pixel_data = std::vector<float>(img_dev.numElements());
    Data::CUDA::copyDevToHost(img_dev, pixel_data);
    return pixel_data;
}

// The reference's spiral FDK, reconFDK(SpiralCTGeom, ...) (fdk_spiral.cuh:33-94), run through its
// own stage functions in its order (per slice: cosine weights, cuFFT ramp filter, texture copy and
// backProjVoxDriven for each view of the slice's window, x rot_ang_incr). SpiralCTGeom itself
// cannot be constructed: its constructor does not compile (spiral_ct_geom.h:81-94 pushes a
// Units::MilliMeters into a std::vector<float> and passes one to std::fabs), so the geometry is
// the CTGeom base it would hold and the window rule firstAndLastProjIndices
// (spiral_ct_geom.h:57-75) is restated: the view whose FP32 source z is nearest the slice (the
// first of equals), num_proj_per_rot / 2 views before it in unsigned arithmetic, and
// num_proj_per_rot views from there; fdk_spiral.cuh:75 reconstructs the slice only when the
// first index is above 0 and the last below the number of views.
template <typename DetRow, typename DetCol>
std::vector<float> fdk_spiral_stages(Geom::CTGeom<DetRow, DetCol> const &geom_host,
                                     Data::ProjectionStack<float, 2u> const &proj_all_host,
                                     Geom::ReconImgGeom<3u> const &vol_geom)
{
    auto const geom_dev = Geom::CUDA::CTGeomDev<DetRow, DetCol>{geom_host};
    auto rf = RampFilteringFFT{std::get<0>(geom_host.detGeom()), FiltParams{},
                               Data::numProjRows(proj_all_host.projSize())};
    auto proj_dev = Data::CUDA::Projection<float, 2u, Data::CUDA::DevMem<float>>{proj_all_host.projSize()};
    auto proj_tex = Data::CUDA::NDArrayTexture<float, 2u>{projSizeToArr(proj_all_host.projSize())};
    std::vector<float> src_z;
    for (auto const &p : geom_host.projGeom()) src_z.push_back(p.src_pos.z.val);
    const unsigned npr = geom_host.rotationGeom().num_proj_per_rot;
    if (npr == 0u) throw std::runtime_error("not a spiral scan: zero projections per rotation");
    auto const first_slice_pos = Geom::leftEndPointPos(vol_geom.mid_point.z.val, vol_geom.z.num_samples,
                                                       vol_geom.z.sampling_width.val);
    std::vector<float> out;
    for (auto slice_idx = 0u; slice_idx < vol_geom.z.num_samples; slice_idx++) {
        auto const slice_pos = first_slice_pos + static_cast<float>(slice_idx) * vol_geom.z.sampling_width.val;
        auto vg_slice = vol_geom;
        vg_slice.z.num_samples = 1u;
        vg_slice.mid_point.z.val = slice_pos;
        auto img_dev = Data::CUDA::ReconImg<float, 3u, Data::CUDA::DevMem<float>>{vg_slice};
        img_dev.setVal(0.0f);
        unsigned mid = 0u;
        for (unsigned i = 1u; i < src_z.size(); ++i)
            if (std::fabs(src_z[i] - slice_pos) < std::fabs(src_z[mid] - slice_pos)) mid = i;
        const unsigned first = mid - npr / 2u, last = first + npr;
        if (first > 0u && last < proj_all_host.numProj()) {
            for (auto proj_idx = first; proj_idx < last; proj_idx++) {
                auto const num_pix_proj = Data::numProjPixels(proj_all_host.projSize());
                Data::CUDA::copyHostToDev(proj_all_host.elements(), proj_dev, proj_idx * num_pix_proj, 0u,
                                          num_pix_proj);
                runCosWeighting(geom_dev, proj_idx, proj_dev);
                rf.runFiltering(proj_dev);
                Data::CUDA::copyDevToDevTexture(proj_dev, proj_tex);
                CUDA::backProjVoxDriven(geom_dev, proj_idx, proj_tex, img_dev);
            }
        }
        img_dev *= geom_host.rotationGeom().rot_ang_incr.val;
        std::vector<float> slice(img_dev.numElements());
        Data::CUDA::copyDevToHost(img_dev, slice);
        out.insert(out.end(), slice.begin(), slice.end());
    }
    return out;
}
}  // namespace GCT::Recon::CUDA

namespace {
// ---- texture probe (--texprobe) ----------------------------------------------------------------
// Source array for the reference's copyDevToDevTexture: plain device floats.
struct DevFloats {
    using value_type = float;
    const float *p;
    size_t n;
    size_t numElements() const { return n; }
    const float *dataPointer() const { return p; }
};

__global__ void tex_fetch_1d(cudaTextureObject_t t, const float *xy, int n, float *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = tex1D<float>(t, xy[2 * i]);
}

__global__ void tex_fetch_2d(cudaTextureObject_t t, const float *xy, int n, float *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = tex2D<float>(t, xy[2 * i], xy[2 * i + 1]);
}

void cuda_ok(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

int texprobe(const char *in_path, const char *out_path)
{
    std::ifstream f(in_path, std::ios::binary);
    int32_t hdr[4];
    f.read(reinterpret_cast<char *>(hdr), sizeof(hdr));
    const int dim = hdr[0], w = hdr[1], h = hdr[2], n = hdr[3];
    if (!f || (dim != 1 && dim != 2) || w <= 0 || h <= 0 || n <= 0 || (dim == 1 && h != 1))
        throw std::runtime_error("bad texprobe header");
    std::vector<float> texels(static_cast<size_t>(w) * h), xy(2 * static_cast<size_t>(n));
    f.read(reinterpret_cast<char *>(texels.data()), sizeof(float) * texels.size());
    f.read(reinterpret_cast<char *>(xy.data()), sizeof(float) * xy.size());
    if (!f) throw std::runtime_error("short texprobe file");
    float *d_tex = nullptr, *d_xy = nullptr, *d_out = nullptr;
    cuda_ok(cudaMalloc(&d_tex, sizeof(float) * texels.size()), "cudaMalloc");
    cuda_ok(cudaMalloc(&d_xy, sizeof(float) * xy.size()), "cudaMalloc");
    cuda_ok(cudaMalloc(&d_out, sizeof(float) * n), "cudaMalloc");
    cuda_ok(cudaMemcpy(d_tex, texels.data(), sizeof(float) * texels.size(), cudaMemcpyHostToDevice), "copy");
    cuda_ok(cudaMemcpy(d_xy, xy.data(), sizeof(float) * xy.size(), cudaMemcpyHostToDevice), "copy");
    const DevFloats src{d_tex, texels.size()};
    if (dim == 1) {
        Data::CUDA::NDArrayTexture<float, 1u> tex{{static_cast<unsigned>(w)}};
        Data::CUDA::copyDevToDevTexture(src, tex);
        tex_fetch_1d<<<(n + 255) / 256, 256>>>(tex.texObject(), d_xy, n, d_out);
        cuda_ok(cudaDeviceSynchronize(), "texture fetch");
    } else {
        Data::CUDA::NDArrayTexture<float, 2u> tex{{static_cast<unsigned>(w), static_cast<unsigned>(h)}};
        Data::CUDA::copyDevToDevTexture(src, tex);
        tex_fetch_2d<<<(n + 255) / 256, 256>>>(tex.texObject(), d_xy, n, d_out);
        cuda_ok(cudaDeviceSynchronize(), "texture fetch");
    }
    std::vector<float> out(n);
    cuda_ok(cudaMemcpy(out.data(), d_out, sizeof(float) * n, cudaMemcpyDeviceToHost), "copy");
    cudaFree(d_tex);
    cudaFree(d_xy);
    cudaFree(d_out);
    std::ofstream o(out_path, std::ios::binary);
    o.write(reinterpret_cast<const char *>(out.data()), sizeof(float) * out.size());
    return o ? 0 : 1;
}

struct Options {
    int bp_mode = -1;  // -1: the reference's reconstruct()
    int repeat = 1;
    bool spiral = false;
};

template <class F>
void timed(const Options &opt, F &&f)
{
    for (int k = 0; k < opt.repeat; ++k) {
        const auto t0 = std::chrono::steady_clock::now();
        f();
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        std::fprintf(stderr, "ref_fdk: reconstruct %.3f ms\n", ms);
    }
}

template <class DetRow>
std::vector<float> run1d(const Input &in, const Options &opt)
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
    if (opt.bp_mode >= 0) return Recon::CUDA::fdk_manual_bp(cg, proj, rg, opt.bp_mode);
    timed(opt, [&] { Recon::CUDA::reconstruct(cg, proj, vol); });
    return vol.elements();
}

template <class DetRow, class DetCol>
std::vector<float> run2d(const Input &in, const Options &opt)
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
    if (opt.spiral) {
        if constexpr (std::is_same_v<DetRow, DetFanArc> && std::is_same_v<DetCol, DetFanLine>) {
            const CTGeom<DetRow, DetCol> base{std::make_tuple(det<DetRow>(in.nc, in.du), det<DetCol>(in.nr, in.dv)),
                                              pg};
            return Recon::CUDA::fdk_spiral_stages(base, proj, rg);
        }
        throw std::runtime_error("the reference's spiral FDK takes a cylindrical detector only");
    }
    if (!Recon::isValidAxialRecon(cg, proj, true)) throw std::runtime_error("invalid reconstruction input");
    if (opt.bp_mode >= 0) return Recon::CUDA::fdk_manual_bp(cg, proj, rg, opt.bp_mode);
    timed(opt, [&] { Recon::CUDA::reconstruct(cg, proj, vol); });
    return vol.elements();
}
}  // namespace

int main(int argc, char **argv)
{
    Options opt;
    bool probe = false;
    int a = 1;
    try {
        for (; a < argc && std::strncmp(argv[a], "--", 2) == 0; ++a) {
            const std::string o = argv[a];
            if (o == "--texprobe") {
                probe = true;
            } else if (o == "--spiral") {
                opt.spiral = true;
            } else if (o == "--repeat" && a + 1 < argc) {
                opt.repeat = std::max(1, std::atoi(argv[++a]));
            } else if (o == "--bp" && a + 1 < argc) {
                const std::string m = argv[++a];
                opt.bp_mode = m == "exact" ? kBpExact : m == "texture" ? kBpTexture : -2;
                if (opt.bp_mode < 0) throw std::runtime_error("unknown --bp mode " + m);
            } else {
                throw std::runtime_error("unknown option " + o);
            }
        }
        if (argc - a != 2) {
            std::fprintf(stderr, "usage: %s [--texprobe | --spiral | --bp exact|texture] [--repeat K] "
                                 "input.bin output.bin\n", argv[0]);
            return 2;
        }
        if (probe) return texprobe(argv[a], argv[a + 1]);
        const Input in = read_input(argv[a]);
        if (opt.spiral && in.kind != 5) throw std::runtime_error("--spiral needs kind 5 (cylindrical detector)");
        std::vector<float> out;
        switch (in.kind) {
            case 0: out = run1d<DetParallel>(in, opt); break;
            case 1: out = run1d<DetFanArc>(in, opt); break;
            case 2: out = run1d<DetFanLine>(in, opt); break;
            case 3: out = run2d<DetParallel, DetParallel>(in, opt); break;
            case 4: out = run2d<DetParallel, DetFanLine>(in, opt); break;
            case 5: out = run2d<DetFanArc, DetFanLine>(in, opt); break;
            case 6: out = run2d<DetFanLine, DetFanLine>(in, opt); break;
            default: throw std::runtime_error("unknown kind");
        }
        std::ofstream o(argv[a + 1], std::ios::binary);
        o.write(reinterpret_cast<const char *>(out.data()), sizeof(float) * out.size());
        return o ? 0 : 1;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_fdk: %s\n", e.what());
        return 1;
    }
}
