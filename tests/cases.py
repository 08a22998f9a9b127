"""Geometry cases shared by the tests: one builder per reference detector configuration.

The parameters follow the reference's FDK integration tests (test/cuda/recon/fdk_axial_tests.cu:
15-537) scaled down so the FP64 oracle finishes in seconds: 360 or fewer views over 360 degrees,
detector centres at (n - 1) / 2, SID/SDD 500/1000 or 1000/1536, 1 mm voxels.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

import gct_b200 as g
from oracle import oracle as orc

KINDS = ["parallel_1d", "fan_arc", "fan_line", "parallel_2d", "cone_parallel", "cone_cyl", "cone_flat"]

# seeded ellipses / ellipsoids (cx, cy, cz, ax, ay, az, phi, mu)
PHANTOM = [
    (0.0, 0.0, 0.0, 40.0, 34.0, 30.0, 0.0, 0.020),
    (-12.0, 8.0, 4.0, 9.0, 14.0, 10.0, 0.4, 0.012),
    (15.0, -10.0, -6.0, 7.0, 5.0, 8.0, -0.7, -0.008),
    (3.0, 18.0, 2.0, 4.0, 6.0, 5.0, 1.1, 0.015),
]


@dataclass
class Case:
    name: str
    cg: g.AxialCTGeom
    og: orc.Geometry
    vg: g.ReconImgGeom
    ov: orc.Volume


def make_case(name: str, nv: int = 120, nc: int = 96, nr: int = 24, n: int = 48, nz: int = 8,
              rot_dir: g.RotDir = g.RotDir.CW, range_rad: float = 2 * math.pi, init_ang: float = 0.0,
              vox: float = 1.0, mid=(0.0, 0.0, 0.0), reference_sizes: bool = False) -> Case:
    """With reference_sizes, the detector widths are those of the reference's FDK integration
    tests (parallel 0.8961 mm, arc 0.0017922 rad, line and flat 2.0 mm, rows 1.14 mm)."""
    incr = range_rad / nv
    c0, r0 = (nc - 1) / 2.0, (nr - 1) / 2.0
    rot = g.RotationParams(rot_dir, init_ang, incr, nv)
    w_par = 0.8961 if reference_sizes else 0.9
    w_arc = 0.0017922 if reference_sizes else 0.11 / nc * 2.0
    if name == "parallel_1d":
        det = (g.DetParallel(nc, w_par),)
        params = g.Parallel1DProjGeomParams(c0, rot)
    elif name == "fan_arc":
        det = (g.DetFanArc(nc, w_arc),)
        params = g.FanBeamProjGeomParams(c0, rot, 1000.0, 500.0)
    elif name == "fan_line":
        det = (g.DetFanLine(nc, 2.0),)
        params = g.FanBeamProjGeomParams(c0, rot, 1536.0, 1000.0)
    elif name == "parallel_2d":
        det = (g.DetParallel(nc, w_par), g.DetParallel(nr, 1.14))
        params = g.Parallel2DProjGeomParams(c0, rot, r0)
    elif name == "cone_parallel":
        det = (g.DetParallel(nc, w_par), g.DetFanLine(nr, 1.14))
        params = g.ConeBeamProjGeomParams(c0, rot, 1536.0, 1000.0, r0)
    elif name == "cone_cyl":
        det = (g.DetFanArc(nc, w_arc), g.DetFanLine(nr, 1.14))
        params = g.ConeBeamProjGeomParams(c0, rot, 1000.0, 500.0, r0)
    elif name == "cone_flat":
        det = (g.DetFanLine(nc, 2.0), g.DetFanLine(nr, 2.0))
        params = g.ConeBeamProjGeomParams(c0, rot, 1000.0, 500.0, r0)
    else:
        raise KeyError(name)
    cg = g.AxialCTGeom.from_params(det, params)
    kind = int(cg.kind)
    og = orc.Geometry(kind, nc, det[0].sampling_width, cg.views, nr if len(det) > 1 else 1,
                      det[1].sampling_width if len(det) > 1 else 1.0)
    if len(det) > 1:
        vg = g.ReconImgGeom(g.EqDistSampler(n, vox), g.EqDistSampler(n, vox), g.EqDistSampler(nz, vox), mid)
        ov = orc.Volume(n, n, nz, vox, vox, vox, tuple(mid))
    else:
        vg = g.ReconImgGeom(g.EqDistSampler(n, vox), g.EqDistSampler(n, vox), None, mid[:2])
        ov = orc.Volume(n, n, 1, vox, vox, 1.0, (mid[0], mid[1], 0.0))
    return Case(name, cg, og, vg, ov)


def oracle_projections(case: Case, scale: float = 1.0) -> np.ndarray:
    """Float32 line integrals (FP64 oracle) of PHANTOM with positions and sizes scaled by `scale`."""
    ph = np.array(PHANTOM)
    ph[:, :6] *= scale
    ph[:, 7] /= scale  # keep line integrals of the same order
    return orc.phantom(case.og, ph).astype(np.float32)


def make_spiral_case(name: str = "cone_cyl", npr: int = 60, turns: int = 3, pitch: float = 1.0, nc: int = 96,
                     nr: int = 24, n: int = 48, nz: int = 16, rot_dir: g.RotDir = g.RotDir.CW) -> Case:
    """Helical cone-beam scan: `turns` rotations of `npr` views, source z = -pitch * angle (mm per
    radian); the grid is centred on the middle of the helix so that the slices near both ends have
    no complete rotation of views (the spiral FDK leaves them zero)."""
    incr = 2 * math.pi / npr
    rot = g.RotationParams(rot_dir, 0.0, incr, npr * turns, pitch)
    c0, r0 = (nc - 1) / 2.0, (nr - 1) / 2.0
    if name == "cone_cyl":
        det = (g.DetFanArc(nc, 0.11 / nc * 2.0), g.DetFanLine(nr, 1.14))
        params = g.ConeBeamProjGeomParams(c0, rot, 1000.0, 500.0, r0)
    elif name == "cone_flat":
        det = (g.DetFanLine(nc, 2.0), g.DetFanLine(nr, 2.0))
        params = g.ConeBeamProjGeomParams(c0, rot, 1000.0, 500.0, r0)
    else:
        raise KeyError(name)
    views = g.ProjGeomFactory(*(type(d) for d in det)).create_all(params)
    cg = g.SpiralCTGeom(det, views)
    og = orc.Geometry(int(cg.kind), nc, det[0].sampling_width, cg.views, nr, det[1].sampling_width)
    zmid = -pitch * incr * (npr * turns - 1) / 2.0
    vg = g.ReconImgGeom(g.EqDistSampler(n, 1.0), g.EqDistSampler(n, 1.0), g.EqDistSampler(nz, 1.5), (0.0, 0.0, zmid))
    ov = orc.Volume(n, n, nz, 1.0, 1.0, 1.5, (0.0, 0.0, zmid))
    return Case(name + "_spiral", cg, og, vg, ov)


def spiral_projections(case: Case) -> np.ndarray:
    """Line integrals of PHANTOM stretched along z to cover the helix, centred on the grid."""
    ph = np.array(PHANTOM)
    ph[:, 2] = ph[:, 2] * 0.5 + case.ov.mid[2]
    ph[:, 5] *= 1.5
    return orc.phantom(case.og, ph).astype(np.float32)
