"""gct_fdk_execute_noalloc: the FDK entry point that allocates no device memory.

It serves callers that cannot allocate device memory while they reconstruct (a host whose own
memory manager has reserved the device, an acquisition loop that forbids allocation after
start-up). Its filtered projections go through a fixed 64 MiB scratch array held by the library,
in chunks of views; the array is committed when a plan is created, so the calls themselves leave
the device's free memory unchanged. This file is collected last so that a failure here does not
hide the other tests.

Checked on freshly created plans, for two calls in a row (the scratch keeps the previous call's
contents): the device's free memory does not change across the calls; the result equals
gct_fdk_execute's (FP32 storage 1e-6: only the order of the view chunks' sums differs; FP16
storage 1e-4: a 1e-7 difference can flip a half-precision rounding) and the FP64 oracle's (FP32
1e-4, FP16 1e-3, the tolerances of the other parity tests). Covered: the FFT filter and the
FP16-split Toeplitz GEMM (whose chunks start at row offsets inside the GEMM), FP32 and FP16
storage, and a plan with the quarter-turn form (execute() runs the quarter-turn backprojector,
this path the plain one: they differ by FP32 coordinate rounding, within the FP16 tolerance).
"""
import ctypes as C
import math

import numpy as np
import pytest

import gct_b200 as g
from gct_b200 import _lib
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

NV, NC, NR, N, NZ = 40, 1024, 256, 96, 24  # FP32: 4.3 MB of quads per view, 15 views per chunk
ELL = [(0.0, 0.0, 0.0, 40.0, 35.0, 30.0, 0.0, 0.02), (8.0, -5.0, 3.0, 10.0, 6.0, 7.0, 0.6, 0.01)]


def _geometry():
    rot = g.RotationParams(g.RotDir.CW, 0.0, 2 * math.pi / NV, NV)
    params = g.ConeBeamProjGeomParams((NC - 1) / 2, rot, 1200.0, 750.0, (NR - 1) / 2)
    cg = g.AxialCTGeom.from_params((g.DetFanLine(NC, 0.4), g.DetFanLine(NR, 0.4)), params)
    vg = g.ReconImgGeom(g.EqDistSampler(N, 1.0), g.EqDistSampler(N, 1.0), g.EqDistSampler(NZ, 1.0))
    return cg, vg


@pytest.fixture(scope="module")
def case():
    import torch
    cg, vg = _geometry()
    proj = torch.empty((NV, NR, NC), dtype=torch.float32, device="cuda")
    g.phantom_project(cg, ELL, proj)
    torch.cuda.synchronize()
    og = orc.Geometry(int(cg.kind), NC, 0.4, cg.views, NR, 0.4)
    exact = orc.fdk(og, orc.Volume(N, N, NZ), proj.cpu().numpy()).reshape(vg.shape)
    return cg, vg, proj, exact


def _noalloc(plan, proj, vol):
    import torch
    lib = _lib.load()
    st = lib.gct_fdk_execute_noalloc(plan._handle, C.c_void_p(proj.data_ptr()), C.c_void_p(vol.data_ptr()),
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(st)


def _rel(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))


FORMS = [
    ("fft-f32", dict(filter=g.FILTER_FFT, storage=g.STORAGE_F32, symmetry=g.SYMMETRY_OFF), 1e-6, 1e-4),
    ("fft-f16", dict(filter=g.FILTER_FFT, storage=g.STORAGE_F16, symmetry=g.SYMMETRY_OFF), 1e-4, 1e-3),
    ("gemm16-f32", dict(filter=g.FILTER_TOEPLITZ_F16X2, storage=g.STORAGE_F32, symmetry=g.SYMMETRY_OFF), 1e-6, 1e-4),
    ("gemm16-f16", dict(filter=g.FILTER_TOEPLITZ_F16X2, storage=g.STORAGE_F16, symmetry=g.SYMMETRY_OFF), 1e-4, 1e-3),
    ("gemm16-f16-quarter-turn", dict(filter=g.FILTER_TOEPLITZ_F16X2, storage=g.STORAGE_F16,
                                     symmetry=g.SYMMETRY_AUTO), 1e-4, 1e-3),
]


@pytest.mark.parametrize("name,opts,tol_exec,tol_oracle", FORMS, ids=[f[0] for f in FORMS])
def test_noalloc_fresh_plan_twice(case, name, opts, tol_exec, tol_oracle):
    import torch
    cg, vg, proj, exact = case
    # a first call on another plan loads the kernels' code (lazy module loading), so that the
    # measured calls below see only what the entry point itself does
    with g.FdkPlan(cg, vg, opts=g.FdkOptions(**opts)) as warm:
        tmp = torch.empty(vg.shape, dtype=torch.float32, device="cuda")
        _noalloc(warm, proj, tmp)
        torch.cuda.synchronize()
        del tmp
    plan = g.FdkPlan(cg, vg, opts=g.FdkOptions(**opts))
    if name.endswith("quarter-turn"):
        assert plan.quarter_turn != 0
    assert plan.workspace_bytes > 64 << 20  # the views do not fit the scratch at once: chunks run
    outs = [torch.full(vg.shape, float("nan"), dtype=torch.float32, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for o in outs:
        _noalloc(plan, proj, o)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes across two calls"
    plan.check()
    ref = torch.empty(vg.shape, dtype=torch.float32, device="cuda")
    plan.execute(proj, ref)  # allocates the workspace, after the measured calls
    torch.cuda.synchronize()
    r = ref.cpu().numpy().astype(np.float64)
    for o in outs:
        got = o.cpu().numpy().astype(np.float64)
        assert np.isfinite(got).all()
        e = _rel(got, r)
        assert e <= tol_exec, f"{name}: vs execute {e:.3e}"
        assert np.abs(got - r).max() <= 10 * tol_exec * np.abs(r).max()
        eo = _rel(got, exact)
        assert eo <= tol_oracle, f"{name}: vs FP64 oracle {eo:.3e}"
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
