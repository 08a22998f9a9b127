"""GPU parity of the FDK engine against the FP64 oracle, all seven geometries.

Tolerances (relative RMS over the grid, against the FP64 oracle on identical float32 inputs):
  * FP32 path (FFT filter, FP32 quads)        <= 1e-4
  * mixed path (FFT filter, FP16 quads)        <= 1e-3
  * filter stage alone (weights + ramp filter) <= 1e-5
"""
import math

import numpy as np
import pytest

import gct_b200 as g
from cases import KINDS, make_case, oracle_projections
from conftest import rel_rms
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _run(case, proj_np, storage=g.STORAGE_F32, zpt=0, filt=None, sym=g.SYMMETRY_AUTO):
    import torch
    proj = torch.from_numpy(proj_np).cuda()
    vol = torch.empty(case.vg.shape, dtype=torch.float32, device="cuda")
    with g.FdkPlan(case.cg, case.vg, filt=filt,
                   opts=g.FdkOptions(storage=storage, z_per_thread=zpt, symmetry=sym)) as plan:
        plan.execute(proj, vol)
        torch.cuda.synchronize()
    return vol.cpu().numpy()


@pytest.mark.parametrize("sym", [g.SYMMETRY_ON, g.SYMMETRY_OFF])
@pytest.mark.parametrize("kind", KINDS)
def test_fdk_fp32_matches_oracle(kind, sym):
    case = make_case(kind)
    proj = oracle_projections(case)
    got = _run(case, proj, sym=sym)
    ref = orc.fdk(case.og, case.ov, proj).reshape(got.shape)
    err = rel_rms(got, ref)
    assert err <= 1e-4, f"{kind}: relRMS {err:.3e}"
    assert np.abs(got - ref).max() <= 1e-3 * np.abs(ref).max()


@pytest.mark.parametrize("sym", [g.SYMMETRY_AUTO, g.SYMMETRY_OFF])
@pytest.mark.parametrize("kind", KINDS)
def test_fdk_fp16_storage_matches_oracle(kind, sym):
    case = make_case(kind)
    proj = oracle_projections(case)
    got = _run(case, proj, storage=g.STORAGE_F16, sym=sym)
    ref = orc.fdk(case.og, case.ov, proj).reshape(got.shape)
    err = rel_rms(got, ref)
    assert err <= 1e-3, f"{kind}: relRMS {err:.3e}"


@pytest.mark.parametrize("kind", KINDS)
def test_filter_stage_matches_oracle(kind):
    import torch
    case = make_case(kind)
    proj = oracle_projections(case)
    dproj = torch.from_numpy(proj).cuda()
    out = torch.empty_like(dproj)
    with g.FdkPlan(case.cg, case.vg) as plan:
        plan.filter(dproj, out)
        torch.cuda.synchronize()
    ref = orc.filter_stack(case.og, proj).reshape(out.shape)
    assert rel_rms(out.cpu().numpy(), ref) <= 1e-5


@pytest.mark.parametrize("kind", ["fan_arc", "cone_flat", "cone_cyl", "parallel_2d", "parallel_1d"])
@pytest.mark.parametrize("zpt", [1, 4, 8, 16])
def test_z_per_thread_variants_agree(kind, zpt):
    case = make_case(kind, nz=10)
    proj = oracle_projections(case)
    base = _run(case, proj, zpt=1)
    got = _run(case, proj, zpt=zpt)
    assert rel_rms(got, base) <= 1e-6


@pytest.mark.parametrize("kind", ["cone_flat", "cone_cyl", "fan_line"])
def test_ccw_short_scan_with_parker(kind):
    # short scan: pi + fan angle + margin, counter-clockwise, starting at 90 degrees
    case = make_case(kind, nv=100, range_rad=math.pi + 0.5, rot_dir=g.RotDir.CCW, init_ang=math.pi / 2)
    proj = oracle_projections(case)
    got = _run(case, proj)
    ref = orc.fdk(case.og, case.ov, proj).reshape(got.shape)
    assert rel_rms(got, ref) <= 1e-4


def test_odd_sizes_and_offset_grid():
    case = make_case("cone_flat", nv=37, nc=75, nr=13, n=21, nz=7, mid=(3.0, -2.0, 1.5), vox=1.3)
    proj = oracle_projections(case)
    got = _run(case, proj, zpt=4)
    ref = orc.fdk(case.og, case.ov, proj).reshape(got.shape)
    assert rel_rms(got, ref) <= 1e-4


def _rolled_tilted(views, roll, tilt):
    """Rolls each detector in its plane and tilts it about the row axis: the row coordinate and
    the denominator then depend on z, which selects the general (per-voxel) kernels."""
    out = views.copy()
    for v in out:
        u = np.array(v["det_row_dir"])
        col = np.array(v["det_col_dir"])
        u, col = math.cos(roll) * u + math.sin(roll) * col, -math.sin(roll) * u + math.cos(roll) * col
        w = np.cross(u, col)
        col = math.cos(tilt) * col + math.sin(tilt) * w
        v["det_row_dir"] = u
        v["det_col_dir"] = col
        if np.any(v["iso_ray_dir"]):
            v["iso_ray_dir"] = np.cross(u, col)
    return out


@pytest.mark.parametrize("kind", ["cone_flat", "cone_cyl"])
def test_rolled_tilted_detector_general_kernel(kind):
    case = make_case(kind, nv=60)
    tilt = 0.004 if kind == "cone_flat" else 0.0  # the arc kinds need an orthonormal basis
    views = _rolled_tilted(case.cg.views, 0.05, tilt)
    cg = g.AxialCTGeom(case.cg.det_geom(), views)
    og = orc.Geometry(case.og.kind, case.og.nc, case.og.du, cg.views, case.og.nr, case.og.dv)
    case2 = type(case)(case.name, cg, og, case.vg, case.ov)
    proj = oracle_projections(case2)
    got = _run(case2, proj)
    ref = orc.fdk(og, case.ov, proj).reshape(got.shape)
    assert rel_rms(got, ref) <= 1e-4


def test_host_reconstruct_matches_plan():
    case = make_case("cone_flat")
    proj = oracle_projections(case)
    vol = g.ReconImg(case.vg)
    g.reconstruct(case.cg, g.ProjectionStack(case.cg.num_cols, case.cg.num_views, case.cg.num_rows, proj), vol)
    dev = _run(case, proj)
    assert np.array_equal(vol.elements, dev)


def test_deterministic():
    case = make_case("cone_cyl")
    proj = oracle_projections(case)
    a = _run(case, proj)
    b = _run(case, proj)
    assert np.array_equal(a, b)


def test_hann_filter_matches_oracle():
    case = make_case("fan_line")
    proj = oracle_projections(case)
    filt = g.FiltParams(0.8, g.ApodFunc.HANN)
    got = _run(case, proj, filt=filt)
    ref = orc.fdk(case.og, case.ov, proj, cut_off=0.8, apod=1).reshape(got.shape)
    assert rel_rms(got, ref) <= 1e-4


def test_texture_lerp_difference_is_quantified():
    # The reference samples through the texture unit, whose lerp weights carry 8 fractional
    # bits. The oracle emulates that; the exact-bilinear engine differs from it by more than it
    # differs from the exact oracle.
    case = make_case("cone_flat")
    proj = oracle_projections(case)
    got = _run(case, proj)
    exact = orc.fdk(case.og, case.ov, proj).reshape(got.shape)
    tex8 = orc.fdk(case.og, case.ov, proj, lerp_bits=8).reshape(got.shape)
    e_exact, e_tex = rel_rms(got, exact), rel_rms(got, tex8)
    assert e_exact < e_tex
    assert e_tex <= 5e-3


@pytest.mark.parametrize("storage", [g.STORAGE_F32, g.STORAGE_F16])
def test_two_workspaces_one_plan(storage):
    # A workspace carries a whole prepared stack (quads and FP16 view scales): preparing a second
    # stack into another workspace must not change what the first one backprojects.
    import torch
    case = make_case("cone_flat")
    p1 = oracle_projections(case)
    p2 = (p1 * 3.0 + 0.5).astype(np.float32)
    with g.FdkPlan(case.cg, case.vg, opts=g.FdkOptions(storage=storage)) as plan:
        nbytes = plan.workspace_bytes
        ws = [torch.empty(nbytes, dtype=torch.uint8, device="cuda") for _ in range(2)]
        d = [torch.from_numpy(p).cuda() for p in (p1, p2)]
        vols = [torch.empty(case.vg.shape, dtype=torch.float32, device="cuda") for _ in range(2)]
        plan.prepare(d[0], ws[0])
        plan.prepare(d[1], ws[1])
        plan.backproject(vols[0], ws[0])
        plan.backproject(vols[1], ws[1])
        alone = [torch.empty_like(vols[0]) for _ in range(2)]
        plan.execute(d[0], alone[0])
        plan.execute(d[1], alone[1])
        torch.cuda.synchronize()
    for a, b in zip(vols, alone):
        assert torch.equal(a, b)


def test_flat_panel_views_from_projection_matrices():
    # views rebuilt from 3 x 4 projection matrices (compose, then the factory of a decomposed
    # matrix, source-detector distance scaled by the pixel width) reconstruct like the views they
    # came from: FP64 geometry equal to 1e-12, so the FP32 results agree to rounding
    case = make_case("cone_flat")
    proj = oracle_projections(case)
    du, dv = (d.sampling_width for d in case.cg.det_geom())
    fac = g.ProjGeomFactory(g.DetFanLine, g.DetFanLine)
    views = case.cg.views.copy()
    for i in range(len(views)):
        pm = g.ProjectionMatrix.compose(g.ProjGeom.from_record(views[i]), du, dv)
        pg = fac.create(g.ProjectionMatrix(pm.matrix()))
        pg.src_det_dist *= du
        views[i] = pg.to_record()
    cg = g.AxialCTGeom(case.cg.det_geom(), views)
    case2 = type(case)(case.name, cg, case.og, case.vg, case.ov)
    got, base = _run(case2, proj), _run(case, proj)
    assert rel_rms(got, base) <= 1e-6
    ref = orc.fdk(case.og, case.ov, proj).reshape(got.shape)
    assert rel_rms(got, ref) <= 1e-4


@pytest.mark.parametrize("storage", [g.STORAGE_F32, g.STORAGE_F16])
def test_streaming_budget_path(storage):
    # a budget of a few views: many chunks through the two upload slots; view-major chunk stacks
    # and the plain kernel, so against execute() with the quarter-turn form off only the chunked
    # summation differs (rounding; FP16 scale roundings can flip: 1e-5)
    import torch
    case = make_case("cone_flat")
    proj = oracle_projections(case)
    with g.FdkPlan(case.cg, case.vg, opts=g.FdkOptions(storage=storage, symmetry=g.SYMMETRY_OFF)) as plan:
        dev = torch.empty(case.vg.shape, dtype=torch.float32, device="cuda")
        plan.execute(torch.from_numpy(proj).cuda(), dev)
        torch.cuda.synchronize()
        pix = case.cg.num_rows * case.cg.num_cols
        per_view = 2 * pix * 4 + (case.cg.num_rows + 4) * (case.cg.num_cols + 4) * (16 if storage == g.STORAGE_F32 else 8)
        out = np.empty(case.vg.shape, np.float32)
        plan.execute_host_budget(proj, out, 7 * per_view + 4096)
        assert rel_rms(out, dev.cpu().numpy()) <= (1e-6 if storage == g.STORAGE_F32 else 1e-5)
        again = np.empty_like(out)
        plan.execute_host_budget(proj, again, 7 * per_view + 4096)
        assert np.array_equal(out, again)
        with pytest.raises(g.GctError, match="budget"):
            plan.execute_host_budget(proj, out, per_view // 2)


@pytest.mark.parametrize("storage", [g.STORAGE_F32, g.STORAGE_F16])
def test_async_host_calls_overlap_and_match(storage):
    # three back-to-back asynchronous calls with different inputs and outputs (two device volumes
    # alternate, uploads wait per chunk) give the synchronous results
    case = make_case("cone_flat")
    proj = oracle_projections(case)
    inputs = [proj, (proj * 2.0).astype(np.float32), (proj + 0.5).astype(np.float32)]
    with g.FdkPlan(case.cg, case.vg, opts=g.FdkOptions(storage=storage)) as plan:
        ref = []
        for p in inputs:
            out = np.empty(case.vg.shape, np.float32)
            plan.execute_host(p, out)
            ref.append(out)
        outs = [np.full(case.vg.shape, np.nan, np.float32) for _ in inputs]
        for p, o in zip(inputs, outs):
            plan.execute_host_async(p, o)
        plan.host_sync()
    for o, r in zip(outs, ref):
        assert np.array_equal(o, r)


@pytest.mark.parametrize("storage,sym,tol", [(g.STORAGE_F32, g.SYMMETRY_OFF, 1e-6), (g.STORAGE_F16, g.SYMMETRY_OFF, 1e-6),
                                             (g.STORAGE_F16, g.SYMMETRY_ON, 1e-5)])
@pytest.mark.parametrize("kind", ["fan_line", "fan_arc"])
def test_view_split_images_match_unsplit(kind, storage, sym, tol):
    """One-voxel-deep images small enough to leave most of the GPU idle are backprojected in view
    chunks into partial images that are summed in chunk order (execute, backproject). The
    allocation-free entry point launches the plain kernel unsplit: with the same kernel the two
    differ only by the grouping of the sum over views (relative RMS <= 1e-6); against the
    quarter-turn kernel (symmetry on) by its FP32 coordinate rounding as well (<= 1e-5, the
    tolerance of the quarter-turn tests). A split backproject with accumulate adds onto the image
    already there (the split image itself, giving twice it)."""
    import ctypes as C
    import torch
    from gct_b200 import _lib
    case = make_case(kind, nv=360, n=64)
    proj = torch.from_numpy(oracle_projections(case)).cuda()
    with g.FdkPlan(case.cg, case.vg, opts=g.FdkOptions(storage=storage, symmetry=sym)) as plan:
        assert (plan.quarter_turn != 0) == (sym == g.SYMMETRY_ON)
        split = torch.full(case.vg.shape, float("nan"), dtype=torch.float32, device="cuda")
        plan.execute(proj, split)
        whole = torch.full(case.vg.shape, float("nan"), dtype=torch.float32, device="cuda")
        lib = _lib.load()
        _lib.check(lib.gct_fdk_execute_noalloc(plan._handle, C.c_void_p(proj.data_ptr()),
                                               C.c_void_p(whole.data_ptr()),
                                               C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        acc = split.clone()
        plan.prepare(proj)
        plan.backproject(acc, accumulate=True)
        plan.check()
        torch.cuda.synchronize()
    s, w, a = split.cpu().numpy(), whole.cpu().numpy(), acc.cpu().numpy()
    assert np.isfinite(s).all()
    assert rel_rms(s, w) <= tol
    assert rel_rms(a, 2.0 * s) <= 1e-6
