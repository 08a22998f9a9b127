"""Pins the FP64 oracle and the engine's host geometry to golden vectors recorded from
satidev/gct's own host-callable functions (tests/golden/make_golden.py, built from the reference
sources by oracle/build_ref.sh). The reference computes in FP32, so the comparisons allow FP32
rounding. No GPU needed; the fixture file travels with the tests."""
from pathlib import Path

import numpy as np
import pytest

import gct_b200 as g
from oracle import oracle as orc

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "ref_host_vectors.npz")
KIND_1D = {0: g.GeomKind.PARALLEL_1D, 1: g.GeomKind.FAN_ARC, 2: g.GeomKind.FAN_LINE}


def test_ramp_taps_match_reference():
    off = 0
    for kind, n, width, fc, apod in GOLD["taps_cases"]:
        n = int(n)
        ref = GOLD["taps_values"][off:off + n]
        off += n
        gk = KIND_1D[int(kind)]
        det = (g.DetParallel if kind == 0 else g.DetFanArc if kind == 1 else g.DetFanLine)(n, float(np.float32(width)))
        eng = g.ramp_filter_taps(gk, det, float(np.float32(fc)), g.ApodFunc(int(apod)))
        ora = orc.ramp_taps(int(gk), n, float(np.float32(width)), float(np.float32(fc)), int(apod))
        scale = np.abs(ref).max()
        np.testing.assert_allclose(eng, ref, rtol=0, atol=2e-6 * scale)
        np.testing.assert_allclose(ora, ref, rtol=0, atol=2e-6 * scale)


def _wrap_diff(a, b):
    d = np.abs(np.asarray(a) - np.asarray(b))
    return np.minimum(d, np.abs(d - 2 * np.pi))


def test_rotation_analysis_matches_reference():
    off = 0
    for n, rc, d, incr, rng, nppr in GOLD["rot_results"]:
        n = int(n)
        ang = GOLD["rot_angles"][off:off + n].astype(np.float64)
        rel_ref = GOLD["rot_rel"][off:off + n]
        off += n
        views = np.zeros(n, dtype=g.VIEW_DTYPE)
        views["rot_ang"] = ang
        views["det_row_center"] = 1.0
        og = orc.Geometry(0, 4, 1.0, views)
        ora = orc.rotation(og)
        if rc != 0:
            with pytest.raises(g.GctError):
                g.AxialCTGeom((g.DetParallel(4, 1.0),), views)
            assert ora is None
            continue
        r = g.AxialCTGeom((g.DetParallel(4, 1.0),), views).rotation_geom()
        assert int(r.dir) == int(d) and ora[0] == int(d)
        assert r.rot_ang_incr == pytest.approx(incr, abs=2e-5) and ora[1] == pytest.approx(incr, abs=2e-5)
        assert r.rot_ang_range == pytest.approx(rng, abs=5e-5) and ora[2] == pytest.approx(rng, abs=5e-5)
        assert r.num_proj_per_rot == int(nppr) and ora[3] == int(nppr)
        assert _wrap_diff(r.rel_rot_ang, rel_ref).max() < 5e-5
        assert _wrap_diff(ora[5], rel_ref).max() < 5e-5


def test_parker_tables_match_reference():
    off = 0
    for arc, nc, width, nv, start, rng, rot_dir in GOLD["parker_cases"]:
        nc, nv = int(nc), int(nv)
        ref = GOLD["parker_values"][off:off + nc * nv].reshape(nv, nc)
        off += nc * nv
        det = (g.DetFanArc if arc else g.DetFanLine)(nc, float(np.float32(width)))
        rot = g.RotationParams(g.RotDir(int(rot_dir)), np.radians(start), np.radians(rng) / nv, nv)
        cg = g.AxialCTGeom.from_params((det,), g.FanBeamProjGeomParams((nc - 1) / 2.0, rot, 1000.0, 500.0))
        eng = g.parker_weights(cg)
        og = orc.Geometry(int(cg.kind), nc, det.sampling_width, cg.views)
        np.testing.assert_allclose(eng, ref, atol=2e-4)
        np.testing.assert_allclose(orc.parker(og), ref, atol=2e-4)


@pytest.mark.parametrize("kind", range(7))
def test_cosine_weights_and_mapping_match_reference(kind):
    inp, outp = GOLD["view_inputs"], GOLD["view_outputs"]
    sel = inp[:, 0] == kind
    for row_in, row_out in zip(inp[sel], outp[sel]):
        _, du, dv, col, row, x, y, z = row_in[:8]
        rec = row_in[8:]
        cosw_ref, u_ref, t_ref, w_ref = row_out
        views = np.zeros(1, dtype=g.VIEW_DTYPE)
        views["rot_ang"], views["det_row_center"], views["det_col_center"] = rec[0], rec[1], rec[2]
        views["src_det_dist"], views["src_iso_dist"] = rec[3], rec[4]
        views["src_pos"], views["det_row_dir"], views["det_col_dir"], views["iso_ray_dir"] = \
            rec[5:8], rec[8:11], rec[11:14], rec[14:17]
        du, dv = float(np.float32(du)), float(np.float32(dv))
        og = orc.Geometry(kind, 512, du, views, 256, dv)
        assert orc.cos_weight(og, 0, int(row), int(col)) == pytest.approx(cosw_ref, rel=2e-6)
        u, t, w = orc.proj_mapping(og, 0, [x, y, z])
        scale_u = 1e-2 if kind in (1, 5) else 1.0   # radians vs mm
        assert u == pytest.approx(u_ref, rel=1e-4, abs=2e-4 * scale_u)
        assert t == pytest.approx(t_ref, rel=1e-4, abs=2e-4)
        assert w == pytest.approx(w_ref, rel=1e-4)
        # the engine's coefficient form at the same point (grid centred on it, voxel 0)
        det = {0: (g.DetParallel(512, du),), 1: (g.DetFanArc(512, du),), 2: (g.DetFanLine(512, du),),
               3: (g.DetParallel(512, du), g.DetParallel(256, dv)), 4: (g.DetParallel(512, du), g.DetFanLine(256, dv)),
               5: (g.DetFanArc(512, du), g.DetFanLine(256, dv)), 6: (g.DetFanLine(512, du), g.DetFanLine(256, dv))}[kind]
        if kind in (0, 3, 4):
            cg = g.AxialCTGeom(det, np.concatenate([views, views]) if False else _two_views(views))
        else:
            cg = g.AxialCTGeom(det, _two_views(views))
        if len(det) > 1:
            grid = g.ReconImgGeom(g.EqDistSampler(1, 1.0), g.EqDistSampler(1, 1.0), g.EqDistSampler(1, 1.0), (x, y, z))
        else:
            grid = g.ReconImgGeom(g.EqDistSampler(1, 1.0), g.EqDistSampler(1, 1.0), None, (x, y))
        _, ecol, erow, ew = g.map_point(cg, grid, 0, [0.0, 0.0, 0.0])
        eu = (ecol - rec[1]) * du
        et = (erow - rec[2]) * dv if len(det) > 1 else 0.0
        bp_const = {0: 1.0, 3: 1.0, 4: 1.0}.get(kind)
        if bp_const is None:
            sid = np.linalg.norm(rec[5:7] if kind in (1, 2) else rec[5:8])
            bp_const = rec[3] * sid if kind in (2, 6) else sid
        assert eu == pytest.approx(u_ref, rel=2e-4, abs=5e-3 * scale_u)
        assert et == pytest.approx(t_ref, rel=2e-4, abs=5e-3)
        assert ew * 1.0 == pytest.approx(w_ref, rel=2e-4)


def _two_views(views):
    """A second view 1 degree further so the rotation analysis of a one-view test is defined."""
    two = np.concatenate([views, views])
    th = 0.0175
    c, s = np.cos(th), np.sin(th)
    rz = np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])
    two[1]["rot_ang"] = views[0]["rot_ang"] + th
    for f in ("src_pos", "det_row_dir", "det_col_dir", "iso_ray_dir"):
        two[1][f] = rz @ views[0][f]
    return two


def test_voxel_positions_match_reference():
    for case, ref in zip(GOLD["vox_inputs"], GOLD["vox_outputs"]):
        nx, ny, nz, dx, dy, dz, mx, my, mz, i, j, k = case
        grid = g.ReconImgGeom(g.EqDistSampler(int(nx), dx), g.EqDistSampler(int(ny), dy),
                              g.EqDistSampler(int(nz), dz), (mx, my, mz))
        cg = g.AxialCTGeom.from_params((g.DetFanLine(8, 1.0), g.DetFanLine(8, 1.0)), g.ConeBeamProjGeomParams(
            3.5, g.RotationParams(g.RotDir.CW, 0.0, 0.1, 3), 1000.0, 500.0, 3.5))
        xyz = g.map_point(cg, grid, 0, [i, j, k])[0]
        np.testing.assert_allclose(xyz, ref, rtol=1e-6, atol=1e-4)
