"""Quarter-turn backprojection (full scans in quarter-turn view partners on a square, even,
centred grid) against the plain column kernel and the FP64 oracle.

Tolerances (relative RMS): quarter-turn vs plain kernel of the same plan options <= 1e-5 (the
rotated columns take their detector coordinates from the base view's FP32 coefficients instead of
their own; the coefficients agree to FP32 rounding); against the FP64 oracle as for the engine
(1e-4 FP32 quads, 1e-3 FP16 quads); chunked host-buffer path vs one launch <= 1e-5 (the sum over
chunks is rounded once per chunk, and the partial sums of ramp-filtered views cancel heavily, so
their rounding is large against the final value: measured 1.9e-6 with FP16 quads).
"""
import math

import numpy as np
import pytest

import gct_b200 as g
from cases import make_case, oracle_projections
from conftest import rel_rms
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

SYM_KINDS = ["fan_arc", "fan_line", "parallel_2d", "cone_parallel", "cone_cyl", "cone_flat"]


def _plan(case, storage=g.STORAGE_F32, sym=g.SYMMETRY_ON, zpt=0, filt=g.FILTER_FFT):
    return g.FdkPlan(case.cg, case.vg, opts=g.FdkOptions(storage=storage, symmetry=sym, z_per_thread=zpt,
                                                         filter=filt))


def _execute(plan, case, proj):
    import torch
    vol = torch.full(case.vg.shape, float("nan"), dtype=torch.float32, device="cuda")
    plan.execute(torch.from_numpy(proj).cuda(), vol)
    torch.cuda.synchronize()
    return vol.cpu().numpy()


@pytest.mark.parametrize("kind", SYM_KINDS)
def test_detected_on_full_scans(kind):
    cw = make_case(kind)
    ccw = make_case(kind, rot_dir=g.RotDir.CCW, init_ang=0.3)
    with _plan(cw) as a, _plan(ccw) as b, _plan(cw, sym=g.SYMMETRY_OFF) as off:
        assert a.quarter_turn in (1, -1) and b.quarter_turn in (1, -1)
        assert off.quarter_turn == 0


def test_auto_takes_it_for_fp16_storage_only():
    case = make_case("cone_flat")
    with _plan(case, g.STORAGE_F16, sym=g.SYMMETRY_AUTO) as a, _plan(case, g.STORAGE_F32, sym=g.SYMMETRY_AUTO) as b:
        assert a.quarter_turn != 0
        assert b.quarter_turn == 0


@pytest.mark.parametrize("case_kw", [
    dict(n=21, nz=7),                          # odd grid side
    dict(mid=(3.0, -2.0, 1.5)),                # grid off the rotation axis
    dict(nv=122),                              # views not in quarter-turn partners
    dict(nv=100, range_rad=math.pi + 0.5),     # short scan
])
def test_not_detected(case_kw):
    case = make_case("cone_flat", **case_kw)
    with _plan(case) as p:
        assert p.quarter_turn == 0
    with _plan(make_case("parallel_1d")) as p:  # the transposed 1D kind keeps its own kernel
        assert p.quarter_turn == 0


@pytest.mark.parametrize("storage", [g.STORAGE_F32, g.STORAGE_F16])
@pytest.mark.parametrize("kind", SYM_KINDS)
def test_matches_plain_kernel_and_oracle(kind, storage):
    for rot in (g.RotDir.CW, g.RotDir.CCW):
        case = make_case(kind, rot_dir=rot, init_ang=0.2)
        proj = oracle_projections(case)
        with _plan(case, storage) as ps, _plan(case, storage, sym=g.SYMMETRY_OFF) as pp:
            assert ps.quarter_turn != 0
            got, plain = _execute(ps, case, proj), _execute(pp, case, proj)
        assert rel_rms(got, plain) <= 1e-5, (kind, rot)
        ref = orc.fdk(case.og, case.ov, proj).reshape(got.shape)
        tol = 1e-4 if storage == g.STORAGE_F32 else 1e-3
        assert rel_rms(got, ref) <= tol, (kind, rot)


@pytest.mark.parametrize("kind", ["cone_flat", "cone_cyl", "fan_arc"])
def test_z_per_thread_variants_agree(kind):
    case = make_case(kind, nz=10)
    proj = oracle_projections(case)
    outs = []
    for zpt in (1, 2, 4, 8):
        with _plan(case, zpt=zpt) as p:
            assert p.quarter_turn != 0
            outs.append(_execute(p, case, proj))
    for o in outs[1:]:
        assert rel_rms(o, outs[0]) <= 1e-6


@pytest.mark.parametrize("storage", [g.STORAGE_F32, g.STORAGE_F16])
def test_host_buffer_path_chunks_base_views(storage):
    case = make_case("cone_flat", nv=240)
    proj = oracle_projections(case)
    with _plan(case, storage) as p:
        dev = _execute(p, case, proj)
        host = np.empty(case.vg.shape, np.float32)
        p.execute_host(proj, host)
    assert rel_rms(host, dev) <= 1e-5


def test_partial_view_range_uses_plain_kernel():
    # prepare + backproject over two halves accumulate the same volume as one execute
    import torch
    case = make_case("cone_flat")
    proj = oracle_projections(case)
    with _plan(case) as p:
        full = _execute(p, case, proj)
        dproj = torch.from_numpy(proj).cuda()
        vol = torch.zeros(case.vg.shape, dtype=torch.float32, device="cuda")
        half = case.cg.num_views // 2
        p.prepare(dproj)
        p.backproject(vol, view_begin=0, view_count=half)
        p.backproject(vol, view_begin=half, view_count=case.cg.num_views - half, accumulate=True)
        torch.cuda.synchronize()
        assert rel_rms(vol.cpu().numpy(), full) <= 1e-5


@pytest.mark.parametrize("storage", [g.STORAGE_F32, g.STORAGE_F16])
def test_prepare_in_parts_matches_whole(storage):
    # partial prepares write single views into the interleaved stack; a whole prepare writes the
    # partner groups from FP32 rows in one pass: the same quads up to the order of one scaling,
    # which can flip an FP16 rounding (measured 3e-6 with FP16 storage)
    import torch
    case = make_case("cone_flat")
    proj = oracle_projections(case)
    with _plan(case, storage) as p:
        full = _execute(p, case, proj)
        dproj = torch.from_numpy(proj).cuda()
        half = case.cg.num_views // 2 + 3
        p.prepare(dproj, view_begin=0, view_count=half)
        p.prepare(dproj, view_begin=half, view_count=case.cg.num_views - half)
        vol = torch.full(case.vg.shape, float("nan"), dtype=torch.float32, device="cuda")
        p.backproject(vol)
        torch.cuda.synchronize()
        assert rel_rms(vol.cpu().numpy(), full) <= (1e-6 if storage == g.STORAGE_F32 else 1e-5)


def test_toeplitz_filter_with_quarter_turns():
    case = make_case("cone_flat")
    proj = oracle_projections(case)
    with _plan(case, g.STORAGE_F16, filt=g.FILTER_TOEPLITZ_BF16X4) as p:
        assert p.quarter_turn != 0
        got = _execute(p, case, proj)
        p.check()
    ref = orc.fdk(case.og, case.ov, proj).reshape(got.shape)
    assert rel_rms(got, ref) <= 1e-3


TOEPLITZ_FORMS = [g.FILTER_TOEPLITZ_F16X2, g.FILTER_TOEPLITZ_BF16X3, g.FILTER_TOEPLITZ_BF16X4]


def _quads_from_rows(y, vscale, quarter):
    """FP16 partner groups of a quarter-turn stack from FP32 filtered rows y [nv][nr][nc]: the
    quad formula of the engine (quad (R, cq) from rows R - 2, R - 1 and columns cq - 2, cq - 1 of
    the zero-padded view, values times the view's power-of-two scale, A C B D in FP16), arranged
    [base view][quad row][quad column][partner][A, C, B, D] as the stack stores them."""
    nv, nr, nc = y.shape
    out = np.empty((quarter, nr + 4, nc + 4, 4, 4), np.float16)
    for v in range(nv):
        yp = np.zeros((nr + 5, nc + 5), np.float32)
        yp[2:nr + 2, 2:nc + 2] = np.float32(vscale[v]) * y[v]
        p00, p01 = yp[:nr + 4, :nc + 4], yp[:nr + 4, 1:nc + 5]
        p10, p11 = yp[1:nr + 5, :nc + 4], yp[1:nr + 5, 1:nc + 5]
        left, right = p00 + p10, p01 + p11
        half = np.float32(0.5)
        quad = np.stack([half * left, p10 - p00, half * (right - left), (p11 - p01) - (p10 - p00)], axis=-1)
        out[v % quarter, :, :, v // quarter, :] = quad.astype(np.float16)
    return out


# Sizes: the quads come from the GEMM's epilogue when the launch has at least one M tile per SM
# (148 on a B200): 31 positions per tile for partner stacks, 127 rows for view-major ones, so the
# stacks below hold 120 views x 160 rows (or 18400 one-row views); the small cases take the
# FP32-row path and must give the same stack.
QUAD_CASES = [("cone_flat", 96, 160, 120), ("cone_flat", 254, 160, 120), ("cone_cyl", 256, 161, 120),
              ("cone_flat", 300, 160, 120), ("fan_line", 130, 1, 18400), ("cone_flat", 96, 24, 120),
              ("fan_line", 130, 1, 120)]


@pytest.mark.parametrize("filt", TOEPLITZ_FORMS)
@pytest.mark.parametrize("kind,nc,nr,nv", QUAD_CASES)
def test_gemm_partner_quads_are_the_quads_of_the_filtered_rows(kind, nc, nr, nv, filt):
    """FP16 quarter-turn stacks with a Toeplitz filter take their partner groups straight from the
    GEMM's epilogue (TMEM -> quads). The stack must hold, bit for bit, the quads formed from the
    same GEMM's plain filtered rows (gct_fdk_filter) with the view scales of the stack: the row and
    view scales are powers of two, so the two orders of scaling round identically. Every entry of
    the stack is written (the workspace starts as 0xFF bytes)."""
    import torch
    case = make_case(kind, nc=nc, nr=nr, n=32, nv=nv)
    proj = oracle_projections(case)
    with _plan(case, g.STORAGE_F16, filt=filt) as p:
        assert p.quarter_turn != 0
        dproj = torch.from_numpy(proj).cuda()
        ws = torch.full((p.workspace_bytes,), 0xFF, dtype=torch.uint8, device="cuda")
        p.prepare(dproj, workspace=ws)
        rows = torch.empty((nv, case.cg.num_rows, case.cg.num_cols), dtype=torch.float32, device="cuda")
        p.filter(dproj, rows)
        p.check()
        torch.cuda.synchronize()
        wsb = ws.cpu().numpy()
        quad_bytes = nv * (nr + 4) * (nc + 4) * 8
        region = (quad_bytes + 255) // 256 * 256
        vscale = wsb[region + 4 * nv:region + 8 * nv].view(np.float32)
        got = wsb[:quad_bytes].view(np.uint16).reshape(nv // 4, nr + 4, nc + 4, 4, 4)
        want = _quads_from_rows(rows.cpu().numpy(), vscale, nv // 4).view(np.uint16)
        bad = np.argwhere(got != want)
        assert bad.size == 0, f"{len(bad)} differing halves, first at {bad[:4].tolist()}"


@pytest.mark.parametrize("filt", TOEPLITZ_FORMS)
def test_gemm_partner_quads_in_chunks_match_whole(filt):
    """The host-buffer path prepares base views in chunks (each with its partners, one GEMM each);
    the volume equals the one-launch execute to the chunked sums' rounding."""
    case = make_case("cone_flat", nv=240)
    proj = oracle_projections(case)
    with _plan(case, g.STORAGE_F16, filt=filt) as p:
        dev = _execute(p, case, proj)
        host = np.empty(case.vg.shape, np.float32)
        p.execute_host(proj, host)
        p.check()
    assert rel_rms(host, dev) <= 1e-5


@pytest.mark.parametrize("filt", TOEPLITZ_FORMS)
@pytest.mark.parametrize("kind,nc,nr,nv", QUAD_CASES[:4] + [("fan_line", 130, 1, 18800), ("cone_flat", 97, 160, 120),
                                                          ("cone_flat", 96, 24, 120)])
def test_gemm_view_major_quads_are_the_quads_of_the_filtered_rows(kind, nc, nr, nv, filt):
    """FP16 stacks without quarter turns (view after view) take their quads straight from the GEMM's
    epilogue too when the quad pitch nc + 4 is even and the launch is large enough (one thread per detector row, two quads per
    16-byte store); an odd pitch (nc = 97) goes through FP32 rows and the quad pass. Either way the
    stack holds, bit for bit, the quads of the plain filtered rows with the view scales."""
    import torch
    case = make_case(kind, nc=nc, nr=nr, n=32, nv=nv)
    proj = oracle_projections(case)
    with _plan(case, g.STORAGE_F16, sym=g.SYMMETRY_OFF, filt=filt) as p:
        assert p.quarter_turn == 0
        dproj = torch.from_numpy(proj).cuda()
        ws = torch.full((p.workspace_bytes,), 0xFF, dtype=torch.uint8, device="cuda")
        p.prepare(dproj, workspace=ws)
        rows = torch.empty((nv, case.cg.num_rows, case.cg.num_cols), dtype=torch.float32, device="cuda")
        p.filter(dproj, rows)
        p.check()
        torch.cuda.synchronize()
        wsb = ws.cpu().numpy()
        quad_bytes = nv * (nr + 4) * (nc + 4) * 8
        region = (quad_bytes + 255) // 256 * 256
        vscale = wsb[region + 4 * nv:region + 8 * nv].view(np.float32)
        got = wsb[:quad_bytes].view(np.uint16).reshape(nv, nr + 4, nc + 4, 4)
        # one partner group per view: the view-major stack is the partner layout with quarter = nv
        want = _quads_from_rows(rows.cpu().numpy(), vscale, nv)[:, :, :, 0, :].view(np.uint16)
        bad = np.argwhere(got != want)
        assert bad.size == 0, f"{len(bad)} differing halves, first at {bad[:4].tolist()}"


# ---- z-mirror form -----------------------------------------------------------------------------
# A short scan has no quarter-turn partners, but with the source on the grid's middle plane and the
# detector centred on it every view maps voxel (x, y, nz - 1 - z) to the same column and weight as
# (x, y, z) and to the mirrored detector row: the column kernels then run over the lower half of
# the grid and each evaluation of a view serves a voxel pair. Results differ from the plain kernel
# by FP32 coordinate rounding only (the mirror sample takes its row split from its partner's).

def _short(kind="cone_flat", **kw):
    return make_case(kind, nv=100, range_rad=math.pi + 0.5, **kw)


@pytest.mark.parametrize("kind", ["cone_flat", "parallel_2d", "cone_parallel"])
def test_z_mirror_detected(kind):
    case = _short(kind)
    with _plan(case, g.STORAGE_F16, sym=g.SYMMETRY_AUTO) as a, _plan(case, g.STORAGE_F32, sym=g.SYMMETRY_AUTO) as b, \
            _plan(case, g.STORAGE_F32, sym=g.SYMMETRY_ON) as c, _plan(case, g.STORAGE_F16, sym=g.SYMMETRY_OFF) as d:
        assert a.quarter_turn == 0 and a.z_mirror == 1
        assert b.z_mirror == 0 and c.z_mirror == 1 and d.z_mirror == 0


@pytest.mark.parametrize("case_kw", [dict(nz=7), dict(mid=(0.0, 0.0, 1.5)), dict(kind="cone_cyl")])
def test_z_mirror_not_detected(case_kw):
    kw = dict(case_kw)
    kind = kw.pop("kind", "cone_flat")
    case = _short(kind, **kw)
    with _plan(case, g.STORAGE_F16, sym=g.SYMMETRY_AUTO) as p:
        assert p.z_mirror == 0


def test_quarter_turn_takes_precedence_over_z_mirror():
    case = make_case("cone_flat")
    with _plan(case, g.STORAGE_F16, sym=g.SYMMETRY_AUTO) as p:
        assert p.quarter_turn != 0 and p.z_mirror == 0


@pytest.mark.parametrize("storage", [g.STORAGE_F32, g.STORAGE_F16])
@pytest.mark.parametrize("case_kw", [dict(kind="cone_flat"), dict(kind="parallel_2d"),
                                     dict(kind="cone_parallel"), dict(kind="cone_flat", nz=48)])
def test_z_mirror_matches_plain_kernel_and_oracle(case_kw, storage):
    """nz = 48 reaches past the detector's rows (clamped, mixed and off blocks)."""
    kw = dict(case_kw)
    case = _short(kw.pop("kind"), **kw)
    proj = oracle_projections(case)
    with _plan(case, storage, sym=g.SYMMETRY_ON) as pm, _plan(case, storage, sym=g.SYMMETRY_OFF) as pp:
        assert pm.z_mirror == 1
        got = _execute(pm, case, proj)
        plain = _execute(pp, case, proj)
    assert np.isfinite(got).all()
    assert rel_rms(got, plain) <= 1e-5
    ref = orc.fdk(case.og, case.ov, proj).reshape(got.shape)
    assert rel_rms(got, ref) <= (1e-4 if storage == g.STORAGE_F32 else 1e-3)


def test_z_mirror_accumulate_and_host_chunks():
    import torch
    case = _short()
    proj = oracle_projections(case)
    with _plan(case, g.STORAGE_F16, sym=g.SYMMETRY_AUTO) as p:
        assert p.z_mirror == 1
        dev = _execute(p, case, proj)
        host = np.empty(case.vg.shape, np.float32)
        p.execute_host(proj, host)
        acc = torch.from_numpy(dev).cuda()
        p.prepare(torch.from_numpy(proj).cuda())
        p.backproject(acc, accumulate=True)
        torch.cuda.synchronize()
        twice = acc.cpu().numpy()
    assert rel_rms(host, dev) <= 1e-5
    assert rel_rms(twice, 2.0 * dev) <= 1e-6
