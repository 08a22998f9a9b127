"""gct_fdk_execute_noalloc: the FDK entry point that allocates no device memory.

It serves callers that cannot allocate device memory while they reconstruct (a host whose own
memory manager has reserved the device, an acquisition loop that forbids allocation after
start-up). Its filtered projections go through a fixed 64 MiB scratch array held by the library,
in chunks of views. This file is collected last so that a failure here does not hide the other
tests. The result must equal gct_fdk_execute's within the FP32 tolerance of the other tests, on
two calls in a row (the scratch keeps the previous call's contents).
"""
import ctypes as C
import math

import numpy as np
import pytest

import gct_b200 as g
from gct_b200 import _lib

pytestmark = pytest.mark.gpu


def _plan_case(storage):
    import torch
    nv, nc, nr, n, nz = 40, 1024, 256, 96, 24  # FP32: 4.3 MB of quads per view, 15 views per chunk
    rot = g.RotationParams(g.RotDir.CW, 0.0, 2 * math.pi / nv, nv)
    params = g.ConeBeamProjGeomParams((nc - 1) / 2, rot, 1200.0, 750.0, (nr - 1) / 2)
    cg = g.AxialCTGeom.from_params((g.DetFanLine(nc, 0.4), g.DetFanLine(nr, 0.4)), params)
    vg = g.ReconImgGeom(g.EqDistSampler(n, 1.0), g.EqDistSampler(n, 1.0), g.EqDistSampler(nz, 1.0))
    proj = torch.empty((nv, nr, nc), dtype=torch.float32, device="cuda")
    g.phantom_project(cg, [(0.0, 0.0, 0.0, 40.0, 35.0, 30.0, 0.0, 0.02), (8.0, -5.0, 3.0, 10.0, 6.0, 7.0, 0.6, 0.01)],
                      proj)
    # view chunks run the plain column kernel; execute() runs the same kernel over all views when
    # the quarter-turn form is off, so the comparison below sees the chunking alone
    plan = g.FdkPlan(cg, vg, opts=g.FdkOptions(storage=storage, symmetry=g.SYMMETRY_OFF))
    return plan, proj, vg


def _noalloc(plan, proj, vol):
    import torch
    lib = _lib.load()
    st = lib.gct_fdk_execute_noalloc(plan._handle, C.c_void_p(proj.data_ptr()), C.c_void_p(vol.data_ptr()),
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(st)


@pytest.mark.parametrize("storage", [g.STORAGE_F32, g.STORAGE_F16])
def test_noalloc_matches_execute_twice(storage):
    import torch
    plan, proj, vg = _plan_case(storage)
    assert plan.workspace_bytes > 64 << 20  # the views do not fit the scratch at once: chunks run
    ref = torch.empty(vg.shape, dtype=torch.float32, device="cuda")
    plan.execute(proj, ref)
    torch.cuda.synchronize()
    r = ref.cpu().numpy().astype(np.float64)
    for _ in range(2):
        out = torch.full(vg.shape, float("nan"), dtype=torch.float32, device="cuda")
        _noalloc(plan, proj, out)
        torch.cuda.synchronize()
        o = out.cpu().numpy().astype(np.float64)
        assert np.isfinite(o).all()
        # Views are summed chunk by chunk, and fewer views per call make the filter pair rows
        # differently inside its complex FFTs. With FP32 storage only rounding order differs
        # (1e-6); with FP16 storage those 1e-7 differences can flip a half-precision rounding,
        # so the FP32-path parity tolerance of the other tests (1e-4) applies.
        tol = 1e-6 if storage == g.STORAGE_F32 else 1e-4
        rel = np.sqrt(np.mean((o - r) ** 2) / np.mean(r ** 2))
        assert rel <= tol, rel
        assert np.abs(o - r).max() <= 10 * tol * np.abs(r).max()
    plan.close()


def test_noalloc_rejects_views_beyond_the_scratch():
    import torch
    nv, nc, nr = 2, 4096, 1100  # FP32 quads of one view: 1104 * 4100 * 16 B > 64 MiB
    rot = g.RotationParams(g.RotDir.CW, 0.0, math.pi / 2, nv)
    params = g.ConeBeamProjGeomParams((nc - 1) / 2, rot, 1200.0, 750.0, (nr - 1) / 2)
    cg = g.AxialCTGeom.from_params((g.DetFanLine(nc, 0.1), g.DetFanLine(nr, 0.1)), params)
    vg = g.ReconImgGeom(g.EqDistSampler(8, 1.0), g.EqDistSampler(8, 1.0), g.EqDistSampler(8, 1.0))
    plan = g.FdkPlan(cg, vg)
    proj = torch.zeros((nv, nr, nc), dtype=torch.float32, device="cuda")
    vol = torch.zeros(vg.shape, dtype=torch.float32, device="cuda")
    with pytest.raises(g.GctError, match="GCT_ERR_BUDGET"):
        _noalloc(plan, proj, vol)
    plan.close()
