"""Host logic of bench.py: the reference arm's geometry and its independence from the engine.

The reference arm (`--impl reference`) times the FP64 oracle on the host cores. Its geometry is
built by the oracle's own view factory, so the arm loads no engine code; these tests pin that
geometry to the engine's factory on every workload, and check in a fresh process that a
reference-arm run never imports gct_b200 and prints the same metric string as the GPU arm.
"""
import json
import subprocess
import sys

import numpy as np
import pytest

from conftest import REPO

sys.path.insert(0, str(REPO))
import bench  # noqa: E402


@pytest.mark.parametrize("name", sorted(bench.CONFIGS))
def test_oracle_geometry_equals_engine_geometry(name):
    cfg = bench.CONFIGS[name]
    cg, _ = bench.make_geometry(cfg)
    og = bench.oracle_geometry(cfg)
    assert og.kind == int(cg.kind) and og.nc == cg.num_cols and og.nv == cg.num_views
    for f in ("rot_ang", "det_row_center", "det_col_center", "src_det_dist", "src_iso_dist", "src_pos",
              "det_row_dir", "det_col_dir", "iso_ray_dir"):
        np.testing.assert_allclose(og.views[f], cg.views[f], rtol=0, atol=1e-9, err_msg=f)


def test_row_cut_shifts_the_row_centre():
    cfg = bench.CONFIGS["cone256"]
    lo, hi = bench.sample_rows(cfg["nr"])
    og = bench.oracle_geometry(cfg, lo, hi)
    assert og.nr == hi - lo
    np.testing.assert_allclose(og.views["det_col_center"], (cfg["nr"] - 1) / 2.0 - lo)


def test_reference_arm_loads_no_engine_code():
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--config', 'fan256', "
            "'--steps', '1', '--warmup', '0']; runpy.run_path('bench.py', run_name='__main__'); "
            "assert not any(m == 'gct_b200' or m.startswith('gct_b200.') for m in sys.modules), 'engine imported'")
    res = subprocess.run([sys.executable, "-c", code], cwd=str(REPO), capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr[-2000:]
    line = json.loads(res.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
