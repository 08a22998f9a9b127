"""Spiral (helical) geometry checks and per-slice view windows on the host.

SpiralCTGeom (src/cpp/geom/spiral_ct_geom.h:30-95): the constructor's checks, the pitch and
firstAndLastProjIndices; the windows are compared with the oracle's restatement of the same rule.
"""
import math

import numpy as np
import pytest

import gct_b200 as g
from cases import make_spiral_case
from oracle import oracle as orc


@pytest.mark.parametrize("name", ["cone_cyl", "cone_flat"])
def test_spiral_geometry(name):
    case = make_spiral_case(name, pitch=1.25)
    assert case.cg.num_proj_per_rot == 60
    assert case.cg.spiral_pitch == pytest.approx(1.25, rel=1e-9)


@pytest.mark.parametrize("rot_dir", [g.RotDir.CW, g.RotDir.CCW])
def test_windows_match_oracle(rot_dir):
    case = make_spiral_case(rot_dir=rot_dir, nz=40)
    wins = orc.spiral_windows(case.og, case.ov)
    z0 = case.ov.mid[2] - (case.ov.nz - 1) * case.ov.dz / 2.0
    nv = case.cg.num_views
    valid = 0
    for k, w in enumerate(wins):
        first, last = case.cg.first_and_last_proj_indices(z0 + k * case.ov.dz)
        assert last - first == 60
        if w is None:
            assert not (first > 0 and last < nv)
        else:
            assert (first, last) == w
            valid += 1
    assert 0 < valid < len(wins)  # some slices reconstruct, the ends do not


def test_window_rule_below_the_scan():
    case = make_spiral_case()
    first, last = case.cg.first_and_last_proj_indices(+1000.0)  # nearest view: view 0
    assert (first, last) == (-30, 30)


def test_invalid_spirals():
    det = (g.DetFanArc(96, 0.11 / 48), g.DetFanLine(24, 1.14))
    rot = g.RotationParams(g.RotDir.CW, 0.0, 2 * math.pi / 60, 180, 0.0)
    params = g.ConeBeamProjGeomParams(47.5, rot, 1000.0, 500.0, 11.5)
    views = g.ProjGeomFactory(g.DetFanArc, g.DetFanLine).create_all(params)
    with pytest.raises(g.GctError, match="pitch cannot be zero"):
        g.SpiralCTGeom(det, views)
    rot = g.RotationParams(g.RotDir.CW, 0.0, 2 * math.pi / 60, 180, 1.0)
    views = g.ProjGeomFactory(g.DetFanArc, g.DetFanLine).create_all(
        g.ConeBeamProjGeomParams(47.5, rot, 1000.0, 500.0, 11.5))
    shuffled = views.copy()
    shuffled[[10, 11]] = shuffled[[11, 10]]
    with pytest.raises(g.GctError, match="sorted"):
        g.SpiralCTGeom(det, shuffled)
    with pytest.raises(g.GctError, match="less than one rotation"):
        g.SpiralCTGeom(det, views[:60])
    fan = g.ProjGeomFactory(g.DetFanLine).create_all(g.FanBeamProjGeomParams(47.5, rot, 1000.0, 500.0))
    with pytest.raises(g.GctError, match="2D detector"):
        g.SpiralCTGeom((g.DetFanLine(96, 2.0),), fan)
