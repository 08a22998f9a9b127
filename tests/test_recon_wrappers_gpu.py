"""The drop-in C++ boundary: satidev/gct's seven GCT::Recon::CUDA::reconstruct overloads on its own
types (AxialCTGeom, ProjectionStack, ReconImg; src/cuda/recon/recon_wrappers.cuh:15-43), defined
by include/gct_recon_wrappers.hpp over this library's C ABI.

oracle/_ref/ref_wrappers is compiled against the reference's own headers (oracle/build_ref.sh)
with those definitions in place of the reference's recon_wrappers.cu, builds the reference's
typed geometry, projection stack and image from the harness input file (the geometry in FP32, as
the reference stores it), validates them with the reference's isValidAxialRecon and calls
reconstruct(). Its volume must equal this library's reconstruction of the same FP32-rounded
geometry through gct_fdk_execute: the same FP32 path, so the only difference allowed is the
pairing of one-row detectors' rows into transforms across the host path's view chunks
(<= 1e-6 relative RMS). It must also stay within the FP32 parity bound of the FP64 oracle
(1e-4).
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import gct_b200 as g
from cases import KINDS, make_case, oracle_projections
from conftest import rel_rms
from oracle import oracle as orc
from test_reference_gpu import write_input

pytestmark = pytest.mark.gpu
REF_WRAPPERS = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "ref_wrappers"


@pytest.fixture(scope="module")
def wrappers():
    if not REF_WRAPPERS.exists():
        pytest.skip("oracle/_ref/ref_wrappers not built (run oracle/build_ref.sh where the reference tree exists)")
    return REF_WRAPPERS


def _fp32_geometry(case):
    views = case.cg.views.copy()
    for f in views.dtype.names:
        views[f] = views[f].astype(np.float32).astype(np.float64)
    return g.AxialCTGeom(case.cg.det_geom(), views)


@pytest.mark.parametrize("kind", KINDS)
def test_typed_overloads_reconstruct_like_the_engine(kind, wrappers, tmp_path):
    import torch
    case = make_case(kind)
    proj = oracle_projections(case)
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    write_input(case, proj, inp)
    res = subprocess.run([str(wrappers), str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr[-2000:]
    got = np.fromfile(out, dtype=np.float32).reshape(case.vg.shape)
    cg32 = _fp32_geometry(case)
    vol = torch.empty(case.vg.shape, dtype=torch.float32, device="cuda")
    with g.FdkPlan(cg32, case.vg) as plan:
        plan.execute(torch.from_numpy(proj).cuda(), vol)
    torch.cuda.synchronize()
    ref = vol.cpu().numpy()
    e = rel_rms(got, ref)
    exact = orc.fdk(case.og, case.ov, proj).reshape(got.shape)
    print(f"{kind}: typed overload vs engine {e:.2e}, vs FP64 oracle {rel_rms(got, exact):.2e}")
    assert e <= 1e-6
    assert rel_rms(got, exact) <= 1e-4
