"""Projection matrices of flat-panel views: decomposition, composition, the view factory and the
matrix file reader, against satidev/gct's own tests.

Known answers: test/cpp/io/projection_matrix_test.cpp (matrix -> principal points 307.5 / 239.5,
focal length 1200 / 0.616 pixels, source (0, -785, 0), R = [[1,0,0],[0,0,-1],[0,1,0]]) and
test/cpp/geom/proj_geom_factory_proj_mat_test.cpp (the view: rotation angle 3 pi / 2, SDD 1200 mm
after scaling by the pixel size, row direction (1,0,0), column direction (0,0,-1)). The reference
checks these in FP32 to 1e-6 relative; the engine decomposes in FP64, so the bar here is 1e-12.
"""
import math

import numpy as np
import pytest

import gct_b200 as g
from gct_b200 import io

REF_MATRIX = np.array([[2.48159483828274, 0.39171974522293, 0.0000, 307.5],
                       [0, 0.305095541401274, -2.48159483828274, 239.5],
                       [0, 0.00127388535031847, 0.0000, 1.0000]])
PIX = 0.616


def test_known_decomposition():
    pm = g.ProjectionMatrix(REF_MATRIX)
    assert pm.principal_point_det_row() == pytest.approx(307.5, rel=1e-12)
    assert pm.principal_point_det_col() == pytest.approx(239.5, rel=1e-12)
    assert pm.focal_length_det_row() == pytest.approx(1200.0 / PIX, rel=1e-12)
    src = pm.src_pos()
    assert np.linalg.norm(src) == pytest.approx(785.0, rel=1e-12)
    assert np.allclose(src, [0.0, -785.0, 0.0], rtol=0, atol=1e-9)
    assert np.allclose(pm.rotation_matrix(), [[1, 0, 0], [0, 0, -1], [0, 1, 0]], rtol=0, atol=1e-12)
    k = pm.intrinsic_matrix()
    assert np.allclose(k, [[1200 / PIX, 0, 307.5], [0, 1200 / PIX, 239.5], [0, 0, 1]], rtol=1e-12, atol=1e-12)


def test_known_factory_view_and_recomposition():
    pm = g.ProjectionMatrix(REF_MATRIX)
    pg = g.ProjGeomFactory(g.DetFanLine, g.DetFanLine).create(pm)
    assert pg.rot_ang == pytest.approx(3 * math.pi / 2, abs=1e-12)
    assert pg.src_det_dist * PIX == pytest.approx(1200.0, rel=1e-12)  # SDD in pixels, as in the reference
    assert (pg.det_row_center, pg.det_col_center) == (pytest.approx(307.5), pytest.approx(239.5))
    assert np.allclose(pg.det_row_dir, [1, 0, 0], atol=1e-12)
    assert np.allclose(pg.det_col_dir, [0, 0, -1], atol=1e-12)
    pg.src_det_dist *= PIX
    comp = g.ProjectionMatrix.compose(pg, PIX, PIX)
    assert comp.focal_length_det_row() == pytest.approx(pm.focal_length_det_row(), rel=1e-12)
    assert comp.principal_point_det_row() == pytest.approx(pm.principal_point_det_row(), rel=1e-12)
    assert comp.principal_point_det_col() == pytest.approx(pm.principal_point_det_col(), rel=1e-12)
    assert np.allclose(comp.matrix(), REF_MATRIX, rtol=1e-12, atol=1e-12)


def _views(n=24, tilt=0.0):
    rot = g.RotationParams(g.RotDir.CCW, 0.3, 2 * math.pi / n, n)
    params = g.ConeBeamProjGeomParams(511.5, rot, 1200.0, 750.0, 383.5)
    cg = g.AxialCTGeom.from_params((g.DetFanLine(1024, 0.4), g.DetFanLine(768, 0.3)), params)
    views = cg.views.copy()
    if tilt:
        for v in views:  # roll each detector in its own plane
            u, c = np.array(v["det_row_dir"]), np.array(v["det_col_dir"])
            v["det_row_dir"] = math.cos(tilt) * u + math.sin(tilt) * c
            v["det_col_dir"] = -math.sin(tilt) * u + math.cos(tilt) * c
    return cg, views


@pytest.mark.parametrize("tilt", [0.0, 0.07])
def test_compose_decompose_round_trip(tilt):
    cg, views = _views(tilt=tilt)
    fac = g.ProjGeomFactory(g.DetFanLine, g.DetFanLine)
    for rec in views:
        pg = g.ProjGeom.from_record(rec)
        pm = g.ProjectionMatrix.compose(pg, 0.4, 0.3)
        back = fac.create(g.ProjectionMatrix(pm.matrix()))
        assert back.src_det_dist * 0.4 == pytest.approx(pg.src_det_dist, rel=1e-12)
        assert back.det_row_center == pytest.approx(pg.det_row_center, rel=1e-12, abs=1e-9)
        assert back.det_col_center == pytest.approx(pg.det_col_center, rel=1e-12, abs=1e-9)
        for f in ("src_pos", "det_row_dir", "det_col_dir"):
            assert np.allclose(getattr(back, f), getattr(pg, f), rtol=1e-12, atol=1e-9), f


@pytest.mark.parametrize("scale", [3.5, -0.25])
def test_matrix_scale(scale):
    # the decomposition fixes K's diagonal positive and nothing else, as the reference does: a
    # negative scale of the matrix flips R (det -1), K and the source do not change
    a, b = g.ProjectionMatrix(REF_MATRIX), g.ProjectionMatrix(REF_MATRIX * scale)
    assert np.allclose(a.intrinsic_matrix(), b.intrinsic_matrix(), rtol=1e-12, atol=1e-9)
    assert np.allclose(np.sign(scale) * a.rotation_matrix(), b.rotation_matrix(), rtol=1e-12, atol=1e-12)
    assert np.allclose(a.src_pos(), b.src_pos(), rtol=1e-12, atol=1e-9)


def test_singular_matrix_rejected():
    m = REF_MATRIX.copy()
    m[:, 1] = m[:, 0]
    with pytest.raises(g.GctError, match="singular"):
        g.ProjectionMatrix(m)


def test_proj_mat_reader(tmp_path):
    cg, views = _views(n=8)
    mats = np.stack([g.ProjectionMatrix.compose(g.ProjGeom.from_record(v), 0.4, 0.3).matrix() for v in views])
    io.write_meta_image([4, 3, len(mats)], [1, 1, 1], [0, 0, 0], mats, str(tmp_path / "pmat.mha"))
    got = io.ProjMatReader.read(io.MetaImgFileReader(str(tmp_path / "pmat.mha")))
    assert len(got) == len(mats)
    for m, pm in zip(mats, got):
        assert np.allclose(pm.matrix(), m / m[2, 3], rtol=1e-12, atol=1e-12)
    io.write_meta_image([5, 3, 2], [1, 1, 1], [0, 0, 0], np.zeros(30), str(tmp_path / "bad.mha"))
    with pytest.raises(ValueError, match="12 elements"):
        io.ProjMatReader.read(io.MetaImgFileReader(str(tmp_path / "bad.mha")))
