"""Serving loop (continuous batching over a device-memory budget) on the GPU.

Tolerances: a request's volume is bit-identical alone and in a mix (its view chunks, tile shape
and summation order depend only on the request); against gct_fdk_execute of the same plan, which
sums all views before one store, the chunked accumulation differs by rounding only: <= 1e-6
relative RMS.
"""
import time

import numpy as np
import pytest

import gct_b200 as g
from cases import make_case, oracle_projections
from conftest import rel_rms
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

MB = 1 << 20


def _request(kind, storage=g.STORAGE_F16, scale=1.0, filt=g.FILTER_FFT, **kw):
    case = make_case(kind, **kw)
    proj = (oracle_projections(case) * np.float32(scale)).astype(np.float32)
    # the server runs the work-queue kernel; execute() of a plan with the quarter-turn form off runs
    # the same per-column arithmetic, which the 1e-6 comparisons below rely on
    plan = g.FdkPlan(case.cg, case.vg, opts=g.FdkOptions(storage=storage, symmetry=g.SYMMETRY_OFF, filter=filt))
    return case, plan, proj


def _execute(plan, case, proj):
    import torch
    out = torch.empty(case.vg.shape, dtype=torch.float32, device="cuda")
    plan.execute(torch.from_numpy(proj).cuda(), out)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_alone_and_in_mix_are_identical():
    a_case, a_plan, a_proj = _request("cone_flat", nv=120)
    others = [_request("fan_line"), _request("cone_cyl", storage=g.STORAGE_F32), _request("parallel_2d"),
              _request("cone_flat", scale=2.0, nv=120), _request("fan_arc")]
    # small rounds so every request spans several rounds and shares them with the others
    with g.FdkServer(512 * MB, round_updates=2e5) as srv:
        alone = np.empty(a_case.vg.shape, np.float32)
        t = srv.submit(a_plan, a_proj, alone)
        srv.wait(t)
        assert srv.info(t)["rounds"] > 1
        outs = [np.empty(c.vg.shape, np.float32) for c, _, _ in others]
        mixed = np.empty(a_case.vg.shape, np.float32)
        tickets = [srv.submit(p, pr, o) for (c, p, pr), o in zip(others[:3], outs[:3])]
        tm = srv.submit(a_plan, a_proj, mixed)
        tickets += [srv.submit(p, pr, o) for (c, p, pr), o in zip(others[3:], outs[3:])]
        for tk in tickets + [tm]:
            srv.wait(tk)
        ref = _execute(a_plan, a_case, a_proj)
        bad = np.argwhere(np.abs(alone - ref) > 1e-5 * np.abs(ref).max())
        assert rel_rms(alone, ref) <= 1e-6, f"alone differs from execute at {bad[:3].tolist()} of {len(bad)}"
        bad = np.argwhere(np.abs(mixed - ref) > 1e-5 * np.abs(ref).max())
        assert rel_rms(mixed, ref) <= 1e-6, f"mixed differs from execute at {bad[:3].tolist()} of {len(bad)}"
        for (c, p, pr), o in zip(others, outs):
            assert rel_rms(o, _execute(p, c, pr)) <= 1e-6, c.name
        assert np.array_equal(alone, mixed)
        st = srv.stats()
        assert st["completed"] == 1 + len(others) + 1 and st["failed"] == 0
        assert st["peak_active"] >= 2
        assert st["p50_ms"] > 0 and st["p99_ms"] >= st["p50_ms"]
    for _, p, _ in others + [(a_case, a_plan, a_proj)]:
        p.close()


def test_toeplitz_filter_requests():
    # requests whose plans filter with the Toeplitz GEMM forms: the server filters their view
    # chunks one at a time (the FP16 form's row scales are per row, so chunking changes nothing)
    reqs = [_request("cone_flat", nv=120, filt=g.FILTER_TOEPLITZ_F16X2),
            _request("cone_cyl", filt=g.FILTER_TOEPLITZ_BF16X4), _request("fan_line")]
    with g.FdkServer(512 * MB, round_updates=2e5) as srv:
        outs = [np.empty(c.vg.shape, np.float32) for c, _, _ in reqs]
        tickets = [srv.submit(p, pr, o) for (c, p, pr), o in zip(reqs, outs)]
        for tk in tickets:
            srv.wait(tk)
        assert srv.info(tickets[0])["rounds"] > 1
    for (c, p, pr), o in zip(reqs, outs):
        assert rel_rms(o, _execute(p, c, pr)) <= 1e-5, c.name
        ref = orc.fdk(c.og, c.ov, pr).reshape(o.shape)
        assert rel_rms(o, ref) <= 1e-3, c.name
        p.close()


def test_budget_admission_and_rejection():
    case, plan, proj = _request("cone_flat", nv=120)
    vol_bytes = int(np.prod(case.vg.shape)) * 4
    need = proj.nbytes + plan.workspace_bytes + vol_bytes
    budget = int(2.5 * need) + 4096  # room for two requests at a time
    with g.FdkServer(budget) as srv:
        outs = [np.empty(case.vg.shape, np.float32) for _ in range(6)]
        tickets = [srv.submit(plan, proj, o) for o in outs]
        for t in tickets:
            srv.wait(t)
        for o in outs[1:]:
            assert np.array_equal(o, outs[0])
        st = srv.stats()
        assert st["peak_active"] <= 2
        assert st["peak_bytes"] <= budget
        assert st["completed"] == 6
    big = _request("cone_flat", nv=120, n=96, nz=64)
    with g.FdkServer(need) as srv:
        with pytest.raises(g.GctError) as e:
            srv.submit(big[1], big[2], np.empty(big[0].vg.shape, np.float32))
        assert e.value.status == 3  # GCT_ERR_BUDGET
        assert srv.stats()["rejected"] == 1
    plan.close()
    big[1].close()


def test_cancel_queued_request():
    case, plan, proj = _request("cone_flat", nv=120)
    need = proj.nbytes + plan.workspace_bytes + int(np.prod(case.vg.shape)) * 4
    with g.FdkServer(need + 4096, max_active=1) as srv:
        outs = [np.empty(case.vg.shape, np.float32) for _ in range(4)]
        tickets = [srv.submit(plan, proj, o) for o in outs]
        cancelled = 0
        for t in tickets[1:]:
            try:
                srv.cancel(t)
                cancelled += 1
            except g.GctError as e:
                assert e.status == 7  # already admitted
        srv.wait(tickets[0])
        for t in tickets[1:]:
            assert srv.info(t)["state"] in ("cancelled", "done", "running")
        assert srv.stats()["cancelled"] == cancelled
    plan.close()


def test_poisson_arrivals_report_latency():
    reqs = [_request("fan_line"), _request("cone_cyl"), _request("cone_flat", nv=120)]
    rng = np.random.default_rng(3)
    with g.FdkServer(1024 * MB) as srv:
        tickets = []
        for _ in range(30):
            c, p, pr = reqs[rng.choice(3, p=[0.7, 0.25, 0.05])]
            tickets.append(srv.submit(p, pr, np.empty(c.vg.shape, np.float32)))
            time.sleep(rng.exponential(0.002))
        for t in tickets:
            srv.wait(t)
        st = srv.stats()
        assert st["completed"] == 30
        assert st["recons_per_s"] > 0
        assert st["p99_ms"] >= st["p50_ms"] > 0
    for _, p, _ in reqs:
        p.close()


def test_quarter_turn_requests_alone_and_in_mix():
    # FP16 plans of full scans keep their interleaved partner stacks in the server and run in the
    # quarter-turn queue: identical alone and in a mix, and against execute() of the same plan (the
    # quarter-turn kernel, same per-thread sums in another chunking) within rounding
    def request(kind, scale=1.0, **kw):
        case = make_case(kind, **kw)
        proj = (oracle_projections(case) * np.float32(scale)).astype(np.float32)
        plan = g.FdkPlan(case.cg, case.vg, opts=g.FdkOptions(storage=g.STORAGE_F16))
        assert plan.quarter_turn != 0
        return case, plan, proj

    a_case, a_plan, a_proj = request("cone_cyl", nv=240)
    others = [request("fan_arc"), request("cone_flat", scale=2.0), request("cone_parallel")]
    with g.FdkServer(512 * MB, round_updates=2e5) as srv:
        alone = np.empty(a_case.vg.shape, np.float32)
        t = srv.submit(a_plan, a_proj, alone)
        srv.wait(t)
        assert srv.info(t)["rounds"] > 1
        outs = [np.empty(c.vg.shape, np.float32) for c, _, _ in others]
        mixed = np.empty(a_case.vg.shape, np.float32)
        tickets = [srv.submit(p, pr, o) for (c, p, pr), o in zip(others[:2], outs[:2])]
        tm = srv.submit(a_plan, a_proj, mixed)
        tickets += [srv.submit(p, pr, o) for (c, p, pr), o in zip(others[2:], outs[2:])]
        for tk in tickets + [tm]:
            srv.wait(tk)
        assert np.array_equal(alone, mixed)
        assert rel_rms(alone, _execute(a_plan, a_case, a_proj)) <= 1e-5
        for (c, p, pr), o in zip(others, outs):
            assert rel_rms(o, _execute(p, c, pr)) <= 1e-5, c.name
    for _, p, _ in [(a_case, a_plan, a_proj)] + others:
        p.close()
