// Shared by the reference harnesses ref_fdk_main.cu and ref_wrappers_main.cpp (TEST
// INFRASTRUCTURE ONLY): the input file format and the reference's own geometry types built from
// it. Input file (little endian): int32 kind, nc, nr, nv, nx, ny, nz; float32 du, dv, dx, dy, dz,
// mx, my, mz; nv records of 17 float32 (rot_ang, det_row_center, det_col_center, src_det_dist,
// src_iso_dist, src_pos[3], det_row_dir[3], det_col_dir[3], iso_ray_dir[3]); nv*nr*nc float32
// projections.
#pragma once

#include <cstdint>
#include <fstream>
#include <stdexcept>
#include <vector>

#include "cpp/geom/axial_ct_geom.h"

namespace ref_input {
using namespace GCT;
using namespace GCT::Geom;

struct Rec {
    float rot, rc, cc, sdd, sid, s[3], ru[3], rv[3], iso[3];
};
inline VecWCS<2u> v2(const float *p) { return VecWCS<2u>{p[0], p[1]}; }
inline VecWCS<3u> v3(const float *p) { return VecWCS<3u>{p[0], p[1], p[2]}; }
inline Units::MilliMeters mm(float x) { return Units::MilliMeters{x}; }
inline Units::DetPixels px(float x) { return Units::DetPixels{x}; }

template <class PG>
PG make(const Rec &r);
template <> inline ProjGeom<DetParallel> make(const Rec &r) { return {Units::Radians{r.rot}, px(r.rc)}; }
template <> inline ProjGeom<DetFanArc> make(const Rec &r) { return {mm(r.sdd), px(r.rc), v2(r.s), v2(r.ru), v2(r.iso)}; }
template <> inline ProjGeom<DetFanLine> make(const Rec &r) { return {mm(r.sdd), px(r.rc), v2(r.s), v2(r.ru)}; }
template <> inline ProjGeom<DetParallel, DetParallel> make(const Rec &r)
{
    return {Units::Radians{r.rot}, px(r.rc), px(r.cc)};
}
template <> inline ProjGeom<DetParallel, DetFanLine> make(const Rec &r)
{
    return {mm(r.sdd), mm(r.sid), Units::Radians{r.rot}, px(r.rc), px(r.cc)};
}
template <> inline ProjGeom<DetFanArc, DetFanLine> make(const Rec &r)
{
    return {mm(r.sdd), px(r.rc), px(r.cc), v3(r.s), v3(r.ru), v3(r.rv), v3(r.iso)};
}
template <> inline ProjGeom<DetFanLine, DetFanLine> make(const Rec &r)
{
    return {mm(r.sdd), px(r.rc), px(r.cc), v3(r.s), v3(r.ru), v3(r.rv)};
}

template <class Det> Det det(unsigned n, float w);
template <> inline DetParallel det(unsigned n, float w) { return DetParallel{EqDistSampler{n, mm(w)}}; }
template <> inline DetFanLine det(unsigned n, float w) { return DetFanLine{EqDistSampler{n, mm(w)}}; }
template <> inline DetFanArc det(unsigned n, float w) { return DetFanArc{EqAngSampler{n, Units::Radians{w}}}; }

struct Input {
    int kind, nc, nr, nv, nx, ny, nz;
    float du, dv, dx, dy, dz, mx, my, mz;
    std::vector<Rec> recs;
    std::vector<float> proj;
};

inline Input read_input(const char *path)
{
    std::ifstream f(path, std::ios::binary);
    Input in{};
    int32_t hdr[7];
    float fl[8];
    f.read(reinterpret_cast<char *>(hdr), sizeof(hdr));
    f.read(reinterpret_cast<char *>(fl), sizeof(fl));
    in.kind = hdr[0], in.nc = hdr[1], in.nr = hdr[2], in.nv = hdr[3], in.nx = hdr[4], in.ny = hdr[5], in.nz = hdr[6];
    in.du = fl[0], in.dv = fl[1], in.dx = fl[2], in.dy = fl[3], in.dz = fl[4], in.mx = fl[5], in.my = fl[6],
    in.mz = fl[7];
    if (!f || in.nv <= 0 || in.nc <= 0 || in.nr <= 0) throw std::runtime_error("bad input header");
    in.recs.resize(in.nv);
    f.read(reinterpret_cast<char *>(in.recs.data()), sizeof(Rec) * in.nv);
    in.proj.resize(static_cast<size_t>(in.nv) * in.nr * in.nc);
    f.read(reinterpret_cast<char *>(in.proj.data()), sizeof(float) * in.proj.size());
    if (!f) throw std::runtime_error("short input file");
    return in;
}
}  // namespace ref_input
