"""C ABI checks that need no GPU: exported symbols, header hygiene, host-side errors and the
absence of a CPU fallback."""
import ctypes as C
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import gct_b200 as g
from gct_b200 import _lib

REPO = Path(__file__).resolve().parents[1]
HEADER = REPO / "include" / "gct_fdk.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:gct_status|int32_t|const char \*)\s*\*?\s*(gct_\w+)\s*\(", text, flags=re.M)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.library_path())], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (gct_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    lib = _lib.load()
    for n in names:
        assert hasattr(lib, n)
    assert set(_lib.SIGNATURES) <= set(names)


def test_only_abi_symbols_are_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.library_path())], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (\w+)", out))
    assert exported == set(declared_functions())


@pytest.mark.parametrize("lang,flags", [("c", ["-std=c11"]), ("c++", ["-std=c++17"])])
def test_header_compiles_standalone(tmp_path, lang, flags):
    cc = shutil.which("gcc") if lang == "c" else shutil.which("g++")
    src = tmp_path / ("t.c" if lang == "c" else "t.cpp")
    inc = '#include "gct_fdk.h"\n' if lang == "c" else '#include "gct_fdk.hpp"\n'
    src.write_text(inc + "int main(void) { return gct_abi_version() == GCT_FDK_ABI_VERSION ? 0 : 1; }\n")
    subprocess.run([cc, *flags, "-Wall", "-Werror", "-fsyntax-only", "-I", str(REPO / "include"), str(src)], check=True)


def test_abi_version():
    assert _lib.load().gct_abi_version() == 1


def _views(n, kind=g.GeomKind.CONE_FLAT):
    params = g.ConeBeamProjGeomParams(7.5, g.RotationParams(g.RotDir.CW, 0.0, 2 * np.pi / n, n), 1000.0, 500.0, 3.5)
    return g.ProjGeomFactory(g.DetFanLine, g.DetFanLine).create_all(params)


def test_invalid_trajectory_message():
    views = _views(4)
    views[:] = views[0]  # stationary source
    with pytest.raises(g.GctError, match="Invalid X-ray source trajectory"):
        g.AxialCTGeom((g.DetFanLine(16, 1.0), g.DetFanLine(8, 1.0)), views)


def test_empty_geometry_rejected():
    geom = _lib.gct_ct_geom()
    geom.kind = int(g.GeomKind.CONE_FLAT)
    geom.det_row = _lib.gct_detector(16, 1.0)
    geom.det_col = _lib.gct_detector(8, 1.0)
    geom.num_views = 0
    out = _lib.gct_rotation_geom()
    st = _lib.load().gct_rotation_geom_get(C.byref(geom), C.byref(out), None, None)
    assert st == 1
    assert b"Empty collection of projection geometry" in _lib.load().gct_last_error_string()


def test_bad_kind_and_null_pointers():
    lib = _lib.load()
    v = _lib.gct_view_geom()
    p = _lib.gct_geom_params()
    assert lib.gct_proj_geom_create(9, C.byref(p), 0, C.byref(v)) == 1
    assert lib.gct_proj_geom_create(0, None, 0, C.byref(v)) == 1
    assert lib.gct_fdk_plan_destroy(None) == 0


def test_zero_sized_image_rejected():
    cg = g.AxialCTGeom((g.DetFanLine(16, 1.0), g.DetFanLine(8, 1.0)), _views(4))
    bad = g.ReconImgGeom(g.EqDistSampler(0, 1.0), g.EqDistSampler(4, 1.0), g.EqDistSampler(4, 1.0))
    with pytest.raises(g.GctError, match="number of samples"):
        g.map_point(cg, bad, 0, [0, 0, 0])
    with pytest.raises(ValueError):
        g.ReconImg(g.ReconImgGeom(g.EqDistSampler(4, 0.0), g.EqDistSampler(4, 1.0)))


def test_is_valid_axial_recon():
    # src/cpp/recon/check_validity.h:66-75: detector size and view count must match
    cg = g.AxialCTGeom((g.DetFanLine(16, 1.0), g.DetFanLine(8, 1.0)), _views(4))
    assert g.is_valid_axial_recon(cg, g.ProjectionStack(16, 4, 8))
    assert not g.is_valid_axial_recon(cg, g.ProjectionStack(15, 4, 8))
    assert not g.is_valid_axial_recon(cg, g.ProjectionStack(16, 4, 9))
    assert not g.is_valid_axial_recon(cg, g.ProjectionStack(16, 5, 8))
    assert not g.is_valid_axial_recon(cg, g.ProjectionStack(16, 3, 8))


def test_projection_stack_rejects_zero_sizes():
    with pytest.raises(ValueError):
        g.ProjectionStack(0, 4, 8)
    with pytest.raises(ValueError):
        g.ProjectionStack(16, 0)


def test_unknown_detector_configuration():
    with pytest.raises(TypeError):
        g.kind_of((g.DetFanLine, g.DetFanArc))


def test_no_cpu_fallback_without_a_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    cg = g.AxialCTGeom((g.DetFanLine(16, 1.0), g.DetFanLine(8, 1.0)), _views(8))
    vg = g.ReconImgGeom(g.EqDistSampler(4, 1.0), g.EqDistSampler(4, 1.0), g.EqDistSampler(4, 1.0))
    with pytest.raises(g.GctError, match="GCT_ERR_CUDA"):
        g.FdkPlan(cg, vg)
    vol = g.ReconImg(vg)
    with pytest.raises(g.GctError):
        g.reconstruct(cg, g.ProjectionStack(16, 8, 8), vol)


def test_empty_batch_rejected():
    lib = _lib.load()
    out = C.c_void_p()
    assert lib.gct_fdk_batch_create(None, 0, None, C.byref(out)) == 1
    assert not out.value
    assert b"empty batch" in lib.gct_last_error_string()
