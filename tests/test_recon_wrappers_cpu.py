"""The drop-in overloads' error path on a machine without a CUDA device: the library returns a
non-OK status and the overload throws std::runtime_error carrying gct_last_error_string(), the
reference's convention (src/cuda/utils/check_error.cu:6-36); the harness reports the exception.
Also checks that include/gct_recon_wrappers.hpp declares exactly the reference's overloads."""
import re
import subprocess
from pathlib import Path

import pytest

from cases import make_case, oracle_projections

REPO = Path(__file__).resolve().parents[1]
REF_WRAPPERS = REPO / "oracle" / "_ref" / "ref_wrappers"


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_overload_throws_runtime_error_without_a_device(tmp_path):
    if not REF_WRAPPERS.exists():
        pytest.skip("oracle/_ref/ref_wrappers not built")
    from test_reference_gpu import write_input
    case = make_case("fan_line", nv=24)
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    write_input(case, oracle_projections(case), inp)
    res = subprocess.run([str(REF_WRAPPERS), str(inp), str(out)], capture_output=True, text=True, timeout=120)
    assert res.returncode == 1
    assert "ref_wrappers: gct_reconstruct:" in res.stderr


def test_header_declares_the_reference_overloads():
    text = (REPO / "include" / "gct_recon_wrappers.hpp").read_text()
    decl = text[:text.index("#ifdef GCT_RECON_WRAPPERS_DEFINE")]
    sigs = re.findall(r"void reconstruct\((Geom::\w+<[^>]*>) const &cg,\s*Data::ProjectionStack<float, (\d)u> const &proj,"
                      r"\s*Data::ReconImg<float, (\d)u> &vol\);", decl)
    kinds = {s[0] for s in sigs}
    assert len(sigs) == 8 and len(kinds) == 8
    for geom, pd, vd in sigs:
        assert int(vd) == int(pd) + 1
    assert "Geom::SpiralCTGeom<Geom::DetFanArc, Geom::DetFanLine>" in kinds
