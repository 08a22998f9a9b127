"""The reference's own known-answer tests, restated, against the engine's host geometry (C ABI)
and the FP64 oracle. No GPU needed.

Sources (satidev/gct): test/cuda/geom/coord_trans_proj_test.cu:9-395,
test/cpp/geom/proj_geom_factory_params_test.cpp:12-312, test/cpp/geom/rotation_geom_test.cpp:11-202,
test/cuda/recon/parker_weighting_test.cu:57-100, test/cuda/geom/coord_trans_img_test.cu:6-66, with the
fixture of test/cpp/geom/proj_geom_params_test_fix.h:11-101 (4 views, pi/2 apart, starting at pi/2,
centres 256 / 257, SID 500, SDD 1000, detectors 512 x 1.0).
"""
import math

import numpy as np
import pytest

import gct_b200 as g
from oracle import oracle as orc

PI = math.pi
EPS = 1e-4  # fixture threshold of the reference (proj_geom_params_test_fix.h:24)


def fixture_params(kind: g.GeomKind):
    rot = g.RotationParams(g.RotDir.CW, PI / 2, PI / 2, 4, 0.0)
    if kind == g.GeomKind.PARALLEL_1D:
        return g.Parallel1DProjGeomParams(256.0, rot)
    if kind in (g.GeomKind.FAN_ARC, g.GeomKind.FAN_LINE):
        return g.FanBeamProjGeomParams(256.0, rot, 1000.0, 500.0)
    if kind == g.GeomKind.PARALLEL_2D:
        return g.Parallel2DProjGeomParams(256.0, rot, 257.0)
    return g.ConeBeamProjGeomParams(256.0, rot, 1000.0, 500.0, 257.0)


DETS = {
    g.GeomKind.PARALLEL_1D: (g.DetParallel(512, 1.0),),
    g.GeomKind.FAN_ARC: (g.DetFanArc(512, 1.0),),
    g.GeomKind.FAN_LINE: (g.DetFanLine(512, 1.0),),
    g.GeomKind.PARALLEL_2D: (g.DetParallel(512, 1.0), g.DetParallel(512, 1.0)),
    g.GeomKind.CONE_PARALLEL: (g.DetParallel(512, 1.0), g.DetFanLine(512, 1.0)),
    g.GeomKind.CONE_CYL: (g.DetFanArc(512, 1.0), g.DetFanLine(512, 1.0)),
    g.GeomKind.CONE_FLAT: (g.DetFanLine(512, 1.0), g.DetFanLine(512, 1.0)),
}


def fixture_geom(kind):
    det = DETS[kind]
    return g.AxialCTGeom.from_params(det, fixture_params(kind))


def oracle_geom(cg):
    det = cg.det_geom()
    return orc.Geometry(int(cg.kind), det[0].num_samples, det[0].sampling_width, cg.views,
                        det[1].num_samples if len(det) > 1 else 1, det[1].sampling_width if len(det) > 1 else 1.0)


# A 1 mm grid of odd size centred on the origin: voxel index c maps to world 0.
GRID3 = g.ReconImgGeom(g.EqDistSampler(9, 1.0), g.EqDistSampler(9, 1.0), g.EqDistSampler(9, 1.0), (0.0, 0.0, 0.0))
GRID2 = g.ReconImgGeom(g.EqDistSampler(9, 1.0), g.EqDistSampler(9, 1.0), None, (0.0, 0.0))


def engine_map(cg, xyz):
    """Detector coordinates in mm/rad (DCS) and weight of world point xyz via the engine's coefficients."""
    grid = GRID3 if cg.is_3d else GRID2
    ijk = [4.0 + xyz[0], 4.0 + xyz[1], 4.0 + (xyz[2] if len(xyz) > 2 else 0.0)]
    pos, col, row, w = g.map_point(cg, grid, 2, ijk)
    v = cg.views[2]
    det = cg.det_geom()
    u = (col - v["det_row_center"]) * det[0].sampling_width
    t = (row - v["det_col_center"]) * det[1].sampling_width if cg.is_3d else 0.0
    return u, t, w, pos


# ---- coord_trans_proj_test.cu -------------------------------------------------------------------

def test_dcs_pcs_known_answers():
    # DCSToPCS(4, 2, 3) = 5, DCSToPCS(-4, 2, 3) = 1; PCSToDCS(5, 2, 3) = 4, PCSToDCS(1, 2, 3) = -4
    dcs_to_pcs = lambda d, w, c: d / w + c
    pcs_to_dcs = lambda p, w, c: (p - c) * w
    assert dcs_to_pcs(4.0, 2.0, 3.0) == 5.0 and dcs_to_pcs(-4.0, 2.0, 3.0) == 1.0
    assert pcs_to_dcs(5.0, 2.0, 3.0) == 4.0 and pcs_to_dcs(1.0, 2.0, 3.0) == -4.0
    # the same conversions inside the engine: a 2 mm detector with centre 3
    rot = g.RotationParams(g.RotDir.CW, 0.0, PI / 2, 4)
    cg = g.AxialCTGeom.from_params((g.DetParallel(8, 2.0),), g.Parallel1DProjGeomParams(3.0, rot))
    grid = g.ReconImgGeom(g.EqDistSampler(9, 1.0), g.EqDistSampler(9, 1.0), None, (0.0, 0.0))
    # view 0: s = y, so world y = 4 maps to pixel 4/2 + 3 = 5 and y = -4 to 1
    assert g.map_point(cg, grid, 0, [4.0, 8.0])[1] == pytest.approx(5.0)
    assert g.map_point(cg, grid, 0, [4.0, 0.0])[1] == pytest.approx(1.0)


@pytest.mark.parametrize("theta,x,y,expect", [(0.0, 0.0, 0.0, 0.0), (0.0, 1.0, 3.0, 3.0), (PI / 2, 1.0, 3.0, -1.0)])
def test_det_coord_axial_parallel(theta, x, y, expect):
    rot = g.RotationParams(g.RotDir.CW, theta, 0.1, 2)
    cg = g.AxialCTGeom.from_params((g.DetParallel(64, 1.0),), g.Parallel1DProjGeomParams(10.0, rot))
    grid = g.ReconImgGeom(g.EqDistSampler(9, 1.0), g.EqDistSampler(9, 1.0), None, (0.0, 0.0))
    col = g.map_point(cg, grid, 0, [4.0 + x, 4.0 + y])[1]
    assert col - 10.0 == pytest.approx(expect, abs=1e-5)
    og = oracle_geom(cg)
    assert orc.proj_mapping(og, 0, [x, y])[0] == pytest.approx(expect, abs=1e-12)


@pytest.mark.parametrize("kind", list(g.GeomKind))
def test_proj_mapping_origin_and_symmetry(kind):
    cg = fixture_geom(kind)
    og = oracle_geom(cg)
    # third projection: rotation angle 270 degrees
    assert cg.rotation_geom().rot_ang[2] == pytest.approx(4.7123889923, abs=1e-6)
    u0, t0, w0, _ = engine_map(cg, [0.0, 0.0, 0.0])
    assert u0 == pytest.approx(0.0, abs=1e-4) and t0 == pytest.approx(0.0, abs=1e-4)
    ou, ot, ow = orc.proj_mapping(og, 2, [0.0, 0.0, 0.0])
    assert ou == pytest.approx(0.0, abs=1e-12) and ot == pytest.approx(0.0, abs=1e-12)
    expected_w = {g.GeomKind.CONE_CYL: 0.002, g.GeomKind.CONE_FLAT: 2.0, g.GeomKind.PARALLEL_1D: 1.0,
                  g.GeomKind.PARALLEL_2D: 1.0, g.GeomKind.CONE_PARALLEL: 1.0,
                  g.GeomKind.FAN_ARC: 1.0 / 500.0, g.GeomKind.FAN_LINE: 1000.0 / 500.0}[kind]
    assert w0 == pytest.approx(expected_w, rel=1e-6)
    assert ow == pytest.approx(expected_w, rel=1e-12)
    # (2, 0, 2) and (-2, 0, -2): axial coordinate odd, longitudinal coordinate odd with z anti-parallel
    up, tp, _, _ = engine_map(cg, [2.0, 0.0, 2.0])
    un, tn, _, _ = engine_map(cg, [-2.0, 0.0, -2.0])
    assert up > un and abs(up) == pytest.approx(abs(un), rel=1e-5)
    if cg.is_3d:
        assert tp < tn and abs(tp) == pytest.approx(abs(tn), rel=1e-5)
    oup, otp, _ = orc.proj_mapping(og, 2, [2.0, 0.0, 2.0])
    oun, otn, _ = orc.proj_mapping(og, 2, [-2.0, 0.0, -2.0])
    assert oup > oun and abs(oup) == pytest.approx(abs(oun), rel=1e-12)
    if cg.is_3d:
        assert otp < otn


def test_parallel_1d_mapping_values():
    cg = fixture_geom(g.GeomKind.PARALLEL_1D)
    # view 2 at 270 degrees: s = x cos(360) + y sin(360) = x
    assert engine_map(cg, [2.0, 0.0])[0] == pytest.approx(2.0, abs=1e-5)
    assert engine_map(cg, [-2.0, 0.0])[0] == pytest.approx(-2.0, abs=1e-5)


# ---- proj_geom_factory_params_test.cpp --------------------------------------------------------

def _vec_eq(a, b, eps=EPS):
    return all(abs(x - y) <= eps or abs(x - y) <= eps * max(abs(x), abs(y)) for x, y in zip(a, b))


@pytest.mark.parametrize("kind", list(g.GeomKind))
def test_factory_basis_vectors(kind):
    params = fixture_params(kind)
    fac = g.ProjGeomFactory(*(type(d) for d in DETS[kind]))
    v2, v3 = fac.create(params, 2), fac.create(params, 3)
    if kind in (g.GeomKind.PARALLEL_1D, g.GeomKind.PARALLEL_2D, g.GeomKind.CONE_PARALLEL):
        assert v2.rot_ang == pytest.approx(3 * PI / 2) and v3.rot_ang == pytest.approx(2 * PI)
        assert v2.det_row_center == 256.0
        if kind != g.GeomKind.PARALLEL_1D:
            assert v2.det_col_center == 257.0
        if kind == g.GeomKind.CONE_PARALLEL:
            assert v2.src_det_dist == 1000.0 and v2.src_iso_dist == 500.0
        return
    three = kind in (g.GeomKind.CONE_CYL, g.GeomKind.CONE_FLAT)
    n = 3 if three else 2
    assert v2.src_det_dist == 1000.0 and v2.det_row_center == 256.0
    assert math.hypot(*v2.src_pos[:n]) == pytest.approx(500.0)
    # 270 degrees: source on -y, row direction +x, iso ray +y, column direction -z
    assert _vec_eq(v2.src_pos[:n], [0.0, -500.0, 0.0][:n])
    assert _vec_eq(v2.det_row_dir[:n], [1.0, 0.0, 0.0][:n])
    # 0 degrees: source on +x, row direction +y, iso ray -x
    assert _vec_eq(v3.src_pos[:n], [500.0, 0.0, 0.0][:n])
    assert _vec_eq(v3.det_row_dir[:n], [0.0, 1.0, 0.0][:n])
    if three:
        assert _vec_eq(v2.det_col_dir, [0.0, 0.0, -1.0]) and _vec_eq(v3.det_col_dir, [0.0, 0.0, -1.0])
        if kind == g.GeomKind.CONE_FLAT:
            assert _vec_eq(np.cross(v2.det_row_dir, v2.det_col_dir), [0.0, 1.0, 0.0])
            assert _vec_eq(np.cross(v3.det_row_dir, v3.det_col_dir), [-1.0, 0.0, 0.0])
    if kind in (g.GeomKind.FAN_ARC, g.GeomKind.CONE_CYL):
        assert _vec_eq(v2.iso_ray_dir[:n], [0.0, 1.0, 0.0][:n])
        assert _vec_eq(v3.iso_ray_dir[:n], [-1.0, 0.0, 0.0][:n])
    if kind == g.GeomKind.FAN_LINE:  # rot90(det_row_dir) is the source-detector direction
        r2, r3 = v2.det_row_dir, v3.det_row_dir
        assert _vec_eq([-r2[1], r2[0]], [0.0, 1.0]) and _vec_eq([-r3[1], r3[0]], [-1.0, 0.0])


@pytest.mark.parametrize("kind", list(g.GeomKind))
def test_factory_matches_oracle(kind):
    params = fixture_params(kind)
    cg = fixture_geom(kind)
    rot = params.rot
    ov = orc.make_views(int(kind), 4, params.det_row_center, getattr(params, "det_col_center", 0.0),
                        getattr(params, "src_det_dist", 0.0), getattr(params, "src_iso_dist", 0.0), int(rot.dir),
                        rot.init_ang, rot.ang_incr, rot.hel_pitch)
    for name in ov.dtype.names:
        np.testing.assert_array_equal(cg.views[name], ov[name])


# ---- rotation_geom_test.cpp ---------------------------------------------------------------------

def _parallel_geom(deg_angles):
    views = np.zeros(len(deg_angles), dtype=g.VIEW_DTYPE)
    views["rot_ang"] = np.radians(deg_angles)
    views["det_row_center"] = 1.0
    return views


def _rotation(deg_angles):
    return g.AxialCTGeom((g.DetParallel(4, 1.0),), _parallel_geom(deg_angles)).rotation_geom()


@pytest.mark.parametrize("angles", [[1, 2, 3], [-10, -9, -8], [358, 0, 2], [361, 2, 3]])
def test_clockwise(angles):
    assert _rotation(angles).dir == g.RotDir.CW
    assert orc.rot_dir(np.radians(angles)) == 1


@pytest.mark.parametrize("angles", [[3, 2, 1], [-10, -12, -14], [2, 0, 358], [3, 361, 359]])
def test_counter_clockwise(angles):
    assert _rotation(angles).dir == g.RotDir.CCW
    assert orc.rot_dir(np.radians(angles)) == -1


@pytest.mark.parametrize("angles", [[-10, -10, -14], [0]])
def test_no_rotation_direction(angles):
    with pytest.raises(g.GctError, match="Invalid X-ray source trajectory"):
        _rotation(angles)
    assert orc.rot_dir(np.radians(angles)) == 0


@pytest.mark.parametrize("angles,expect", [([180, 360, 540, 0], [0, 180, 0, 180]),
                                           ([0, 540, 360, 180], [0, 180, 0, 180]),
                                           ([90, 270, 90], [0, 180, 0])])
def test_relative_angles(angles, expect):
    rel = _rotation(angles).rel_rot_ang
    np.testing.assert_allclose(np.degrees(rel), expect, atol=1e-3)


def test_relative_angles_invalid_when_stationary():
    with pytest.raises(g.GctError):
        _rotation([0, 360, 0, 360])


def test_increment_and_range():
    assert np.degrees(_rotation([3, 2, 1]).rot_ang_incr) == pytest.approx(1.0)
    r = _rotation([90, 270, 90])
    assert np.degrees(r.rot_ang_incr) == pytest.approx(180.0)
    assert np.degrees(r.rot_ang_range) == pytest.approx(360.0)
    full = _rotation(list(range(360)))
    assert np.degrees(full.rot_ang_range) == pytest.approx(360.0)
    assert full.num_proj_per_rot == 360


def test_num_proj_per_rot():
    assert _rotation([0, 180, 360, 0]).num_proj_per_rot == 2
    assert _rotation([0, 57.29577951308232, 114.59155902616465]).num_proj_per_rot == 3


@pytest.mark.parametrize("kind", list(g.GeomKind))
def test_rotation_info_of_fixture(kind):
    r = fixture_geom(kind).rotation_geom()
    assert r.dir == g.RotDir.CW
    assert r.rot_ang_incr == pytest.approx(PI / 2, rel=EPS)
    assert r.rot_ang_range == pytest.approx(2 * PI, rel=EPS)
    assert r.num_proj_per_rot == 4
    np.testing.assert_allclose(r.rot_ang, [PI / 2, PI, 3 * PI / 2, 0.0], atol=EPS)
    np.testing.assert_allclose(r.rel_rot_ang, [0.0, PI / 2, PI, 3 * PI / 2], atol=EPS)


# ---- parker_weighting_test.cu -------------------------------------------------------------------

def _fan_arc_geom(range_deg, start_deg, rot_dir):
    det = (g.DetFanArc(512, 0.0017922),)
    nv = 360
    rot = g.RotationParams(rot_dir, math.radians(start_deg), math.radians(range_deg) / nv, nv)
    params = g.FanBeamProjGeomParams((512 - 1) / 2.0, rot, 1000.0, 500.0)
    return g.AxialCTGeom.from_params(det, params)


@pytest.mark.parametrize("start", [45, 90, 180, 270, 360])
@pytest.mark.parametrize("rng", [200, 250, 360])
@pytest.mark.parametrize("rot_dir", [g.RotDir.CW, g.RotDir.CCW])
def test_parker_weights_in_unit_interval(start, rng, rot_dir):
    cg = _fan_arc_geom(rng, start, rot_dir)
    w = g.parker_weights(cg)
    assert np.all(w >= 0.0) and np.all(w <= 1.0)
    ow = orc.parker(oracle_geom(cg))
    np.testing.assert_allclose(w, ow, atol=1e-6)


@pytest.mark.parametrize("start", [90, 180, 270, 360])
def test_parker_weights_independent_of_start(start):
    ref = g.parker_weights(_fan_arc_geom(360, 0, g.RotDir.CW))
    np.testing.assert_allclose(g.parker_weights(_fan_arc_geom(360, start, g.RotDir.CW)), ref, atol=1e-5)


@pytest.mark.parametrize("rng", [90, 180, 270, 360])
def test_parker_weights_depend_on_range(rng):
    ref = g.parker_weights(_fan_arc_geom(255, 90, g.RotDir.CW))
    assert not np.array_equal(ref, g.parker_weights(_fan_arc_geom(rng, 90, g.RotDir.CW)))


def test_parker_parallel_weights():
    half = g.AxialCTGeom((g.DetParallel(8, 1.0),), _parallel_geom(np.arange(180.0)))
    full = g.AxialCTGeom((g.DetParallel(8, 1.0),), _parallel_geom(np.arange(360.0)))
    assert np.all(g.parker_weights(half) == 1.0)
    assert np.all(g.parker_weights(full) == 0.5)


# ---- coord_trans_img_test.cu --------------------------------------------------------------------

def test_voxel_positions():
    assert g.ReconImgGeom(g.EqDistSampler(256, 1.0), g.EqDistSampler(256, 1.0)).first_voxel_pos()[0] == -127.5
    geo2 = g.ReconImgGeom(g.EqDistSampler(1025, 1.0), g.EqDistSampler(513, 2.0), None, (1.0, 2.0))
    assert geo2.first_voxel_pos() == (-511.0, -510.0)
    geo3 = g.ReconImgGeom(g.EqDistSampler(1025, 1.0), g.EqDistSampler(513, 2.0), g.EqDistSampler(11, 4.0),
                          (1.0, 2.0, 3.0))
    assert geo3.first_voxel_pos() == pytest.approx((-511.0, -510.0, -17.0))
    # the engine's voxel centres (map_point) agree
    cg = fixture_geom(g.GeomKind.CONE_FLAT)
    xyz = g.map_point(cg, geo3, 0, [0, 0, 0])[0]
    np.testing.assert_allclose(xyz, [-511.0, -510.0, -17.0])
    geo = g.ReconImgGeom(g.EqDistSampler(512, 2.0), g.EqDistSampler(256, 1.0), None, (0.0, 0.0))
    xyz = g.map_point(fixture_geom(g.GeomKind.FAN_LINE), geo, 0, [0, 0])[0]
    np.testing.assert_allclose(xyz[:2], [-511.0, -127.5])
