"""Batched persistent FDK (one work-queue launch over many reconstructions, CUDA graph replay)
against the per-plan entry point and the FP64 oracle.

Tolerances (relative RMS): batch vs gct_fdk_execute of the same plan <= 1e-5 (the queue kernel
may pick another tile shape, which changes FP32 rounding of the row coordinate only); view-split
items accumulate with atomics, whose order varies, <= 1e-5; batch vs the FP64 oracle as for the
engine (1e-4 FP32 quads, 1e-3 FP16 quads).
"""
import numpy as np
import pytest

import gct_b200 as g
from cases import KINDS, make_case, oracle_projections
from conftest import rel_rms
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _dev(case, storage=g.STORAGE_F32, filt=g.FILTER_FFT):
    import torch
    proj = oracle_projections(case)
    plan = g.FdkPlan(case.cg, case.vg, opts=g.FdkOptions(storage=storage, filter=filt, symmetry=g.SYMMETRY_OFF))
    dproj = torch.from_numpy(proj).cuda()
    vol = torch.full(case.vg.shape, float("nan"), dtype=torch.float32, device="cuda")
    return plan, dproj, vol, proj


def _alone(plan, dproj, shape):
    import torch
    out = torch.empty(shape, dtype=torch.float32, device="cuda")
    plan.execute(dproj, out)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_batch_all_kinds_match_execute_and_oracle():
    import torch
    cases = [make_case(k) for k in KINDS]
    items = [_dev(c) for c in cases]
    with g.FdkBatch([(p, d, v) for p, d, v, _ in items]) as batch:
        batch.launch()
        torch.cuda.synchronize()
        n_work, updates = batch.work()
        assert n_work > 0
        assert updates == sum(int(np.prod(c.vg.shape)) * c.cg.num_views for c in cases)
        for i, (case, (plan, dproj, vol, proj)) in enumerate(zip(cases, items)):
            got = vol.cpu().numpy()
            assert rel_rms(got, _alone(plan, dproj, case.vg.shape)) <= 1e-5, case.name
            ref = orc.fdk(case.og, case.ov, proj).reshape(got.shape)
            assert rel_rms(got, ref) <= 1e-4, case.name
            cfg = batch.item_config(i)
            assert cfg["z_per_thread"] in (1, 4, 8, 16)
            assert cfg["block"][0] * cfg["block"][1] == 256
    for p, *_ in items:
        p.close()


def test_batch_mixed_storage_and_shared_plan():
    import torch
    case = make_case("cone_cyl")
    p32, d32, v32, _ = _dev(case)
    p16, d16, v16, _ = _dev(case, storage=g.STORAGE_F16)
    # a second stack through the same FP16 plan
    d16b = d16 * 2.0 + 0.25
    v16b = torch.empty_like(v16)
    with g.FdkBatch([(p32, d32, v32), (p16, d16, v16), (p16, d16b, v16b)]) as batch:
        batch.launch()
        torch.cuda.synchronize()
        assert rel_rms(v32.cpu().numpy(), _alone(p32, d32, case.vg.shape)) <= 1e-5
        assert rel_rms(v16.cpu().numpy(), _alone(p16, d16, case.vg.shape)) <= 1e-5
        assert rel_rms(v16b.cpu().numpy(), _alone(p16, d16b, case.vg.shape)) <= 1e-5
    for p in (p32, p16):
        p.close()


def test_batch_view_split_single_item():
    # one small item: its tiles are too few for the grid, so views are split into chunks that
    # accumulate atomically into a zeroed volume
    import torch
    case = make_case("cone_flat")
    plan, dproj, vol, proj = _dev(case)
    with g.FdkBatch([(plan, dproj, vol)]) as batch:
        assert batch.item_config(0)["view_split"] > 1
        batch.launch()
        torch.cuda.synchronize()
        a = vol.cpu().numpy()
        batch.launch()  # replay overwrites: the volume is zeroed inside the graph
        torch.cuda.synchronize()
        b = vol.cpu().numpy()
    assert rel_rms(a, _alone(plan, dproj, case.vg.shape)) <= 1e-5
    assert rel_rms(a, b) <= 1e-6
    plan.close()


def test_batch_graph_and_direct_issue_agree():
    import torch
    cases = [make_case("fan_arc"), make_case("parallel_2d"), make_case("cone_parallel")]
    items = [_dev(c, storage=g.STORAGE_F16) for c in cases]
    outs = []
    for use_graph in (True, False):
        with g.FdkBatch([(p, d, v) for p, d, v, _ in items], use_graph=use_graph, autotune=False) as batch:
            batch.launch()
            torch.cuda.synchronize()
            outs.append([v.cpu().numpy() for _, _, v, _ in items])
    for a, b in zip(*outs):
        assert rel_rms(a, b) <= 1e-6
    for case, (plan, dproj, _, _), got in zip(cases, items, outs[0]):
        assert rel_rms(got, _alone(plan, dproj, case.vg.shape)) <= 1e-5, case.name
    for p, *_ in items:
        p.close()


@pytest.mark.parametrize("filt", [g.FILTER_TOEPLITZ_BF16X4, g.FILTER_TOEPLITZ_F16X2])
def test_batch_toeplitz_filter_items(filt):
    case = make_case("cone_flat")
    plan, dproj, vol, proj = _dev(case, storage=g.STORAGE_F16, filt=filt)
    with g.FdkBatch([(plan, dproj, vol)]) as batch:
        batch.launch()
        plan.check()
        got = vol.cpu().numpy()
    ref = orc.fdk(case.og, case.ov, proj).reshape(got.shape)
    assert rel_rms(got, ref) <= 1e-3
    plan.close()


def test_batch_quarter_turn_items():
    # FP16 plans of full scans on square centred grids keep their interleaved partner stacks and
    # run in the quarter-turn queue; against execute() of the same plans (the quarter-turn
    # kernel, with another tile shape): <= 1e-5; a single-item batch of 240 views splits its 60
    # base views into atomic chunks (at least 16 base views each)
    import torch
    kinds = ["cone_flat", "cone_cyl", "fan_arc", "cone_parallel", "parallel_2d"]
    cases = [make_case(k) for k in kinds]
    items = []
    for c in cases:
        proj = oracle_projections(c)
        plan = g.FdkPlan(c.cg, c.vg, opts=g.FdkOptions(storage=g.STORAGE_F16))
        assert plan.quarter_turn != 0
        items.append((plan, torch.from_numpy(proj).cuda(),
                      torch.full(c.vg.shape, float("nan"), dtype=torch.float32, device="cuda"), proj))
    for tune in (True, False):
        with g.FdkBatch([(p, d, v) for p, d, v, _ in items], autotune=tune) as batch:
            batch.launch()
            torch.cuda.synchronize()
            for i, (case, (plan, dproj, vol, proj)) in enumerate(zip(cases, items)):
                got = vol.cpu().numpy()
                assert rel_rms(got, _alone(plan, dproj, case.vg.shape)) <= 1e-5, case.name
                ref = orc.fdk(case.og, case.ov, proj).reshape(got.shape)
                assert rel_rms(got, ref) <= 1e-3, case.name
                assert batch.item_config(i)["z_per_thread"] == (1 if case.name == "fan_arc" else 8)
    for p, *_ in items:
        p.close()
    case = make_case("cone_flat", nv=240)
    proj = oracle_projections(case)
    with g.FdkPlan(case.cg, case.vg, opts=g.FdkOptions(storage=g.STORAGE_F16)) as plan:
        dproj = torch.from_numpy(proj).cuda()
        vol = torch.full(case.vg.shape, float("nan"), dtype=torch.float32, device="cuda")
        with g.FdkBatch([(plan, dproj, vol)]) as batch:
            assert batch.item_config(0)["view_split"] > 1
            batch.launch()
            torch.cuda.synchronize()
            assert rel_rms(vol.cpu().numpy(), _alone(plan, dproj, case.vg.shape)) <= 1e-5
