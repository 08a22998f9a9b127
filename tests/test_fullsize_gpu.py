"""Full-size workloads (the benchmark's flat cone 512^3 / 720 views and the short scan 512 x 512 x
384 / 496 views on a 1240 x 960 detector) through properties that do not need the whole FP64
oracle volume.

* Sampled-voxel parity: 4200 voxels (6 slices x 700) against the FP64 oracle, which filters only
  the detector rows those voxels touch: FP32 path <= 1e-4, mixed path <= 1e-3 relative RMS.
* Linearity: FDK(a p1 + b p2) = a FDK(p1) + b FDK(p2). The FP32 path is linear up to rounding
  (<= 1e-5); the mixed path's per-view FP16 scales depend on the data, so <= 1e-3.
* The host-buffer paths (synchronous, asynchronous, bounded memory) reconstruct what a device
  call does: <= 1e-6 (chunked summation) for FP32 quads.
"""
import numpy as np
import pytest

import bench
import gct_b200 as g
from conftest import rel_rms

pytestmark = pytest.mark.gpu


def _setup(config):
    import torch
    cfg = bench.CONFIGS[config]
    cg, vg = bench.make_geometry(cfg)
    proj = bench.make_projections(cg, cfg, 1234, torch.device("cuda"))
    return cfg, cg, vg, proj


def _run(plan, proj, vg):
    import torch
    vol = torch.empty(vg.shape, dtype=torch.float32, device="cuda")
    plan.execute(proj, vol)
    torch.cuda.synchronize()
    return vol


@pytest.mark.parametrize("config", ["cone512", "short384"])
def test_sampled_voxels_and_linearity(config):
    import torch
    cfg, cg, vg, proj = _setup(config)
    mixed = g.FdkOptions(filter=g.FILTER_TOEPLITZ_F16X2, storage=g.STORAGE_F16)
    with g.FdkPlan(cg, vg) as p32, g.FdkPlan(cg, vg, opts=mixed) as p16:
        vols = {"fp32": _run(p32, proj, vg), "mixed": _run(p16, proj, vg)}
        errs, n = bench.oracle_errors(cg, cfg, proj, vols, 1234)
        assert n == 4200
        assert errs["fp32"]["rel_rms"] <= 1e-4, errs
        assert errs["mixed"]["rel_rms"] <= 1e-3, errs
        # linearity, with a second input of a different phantom
        proj2 = bench.make_projections(cg, cfg, 99, torch.device("cuda"))
        combo = 0.75 * proj - 1.5 * proj2
        for name, plan, tol in (("fp32", p32, 1e-5), ("mixed", p16, 1e-3)):
            lhs = _run(plan, combo, vg).double()
            rhs = 0.75 * vols[name].double() - 1.5 * _run(plan, proj2, vg).double()
            err = float(((lhs - rhs).pow(2).mean() / rhs.pow(2).mean()).sqrt())
            assert err <= tol, (name, err)


def test_host_paths_at_full_size():
    import torch
    cfg, cg, vg, proj = _setup("cone512")
    host_proj = torch.empty(proj.shape, dtype=torch.float32, pin_memory=True)
    host_proj.copy_(proj)
    hp = host_proj.numpy()
    with g.FdkPlan(cg, vg) as plan:
        dev = _run(plan, proj, vg).cpu().numpy()
        outs = [np.empty(vg.shape, np.float32) for _ in range(3)]
        plan.execute_host(hp, outs[0])
        plan.execute_host_async(hp, outs[1])
        plan.host_sync()
        plan.execute_host_budget(hp, outs[2], 4 << 30)
    for o in outs:
        assert rel_rms(o, dev) <= 1e-6
