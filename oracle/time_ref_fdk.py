"""Times satidev/gct's own CUDA FDK (oracle/_ref/ref_fdk: GCT::Recon::CUDA::reconstruct compiled from
its sources for sm_100a) on one of bench.py's workloads, on the same GPU, for context beside the
engine's numbers. TEST INFRASTRUCTURE: measures the reference; nothing of the engine runs inside
the timed calls.

    python oracle/time_ref_fdk.py --config fan256 [--repeat 3]

The workload's projections (bench.py's seeded phantom, made on the GPU) are written in the
harness's input format (oracle/ref_input.hpp) to a temporary file; ref_fdk runs reconstruct()
--repeat times in one process and reports each call's wall time (host projections in, host
volume out, as the reference's API works: its allocation, copies, per-view texture copies and
launches, cuFFT plan). Prints one JSON line: the times, the voxel x view updates per second of
the fastest call and the relative RMS distance from the engine's FP32 reconstruction.
"""
from __future__ import annotations

import argparse
import json
import re
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[1]
# run as a script, this file's own directory would shadow the oracle package
sys.path[:] = [p for p in sys.path if Path(p or ".").resolve() != Path(__file__).resolve().parent]
sys.path.insert(0, str(REPO / "tests"))
sys.path.insert(0, str(REPO))


def main():
    import torch
    import bench
    import gct_b200 as g
    from test_reference_gpu import write_input

    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="fan256", choices=sorted(bench.CONFIGS))
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--split", action="store_true",
                    help="also run the reference's stage sequence with an exact fetch (ref_fdk --bp exact) and "
                         "report the texture's share of the engine/reference distance")
    args = ap.parse_args()
    cfg = bench.CONFIGS[args.config]
    cg, vg = bench.make_geometry(cfg)
    proj = bench.make_projections(cg, cfg, args.seed, torch.device("cuda", 0))
    vol = torch.empty(vg.shape, dtype=torch.float32, device="cuda")
    with g.FdkPlan(cg, vg) as plan:
        plan.execute(proj, vol)
    torch.cuda.synchronize()
    engine = vol.cpu().numpy().astype(np.float64)
    host = proj.cpu().numpy()
    del proj, vol
    torch.cuda.empty_cache()
    case = type("Case", (), {"cg": cg, "vg": vg})()
    with tempfile.TemporaryDirectory() as td:
        inp, out = Path(td) / "in.bin", Path(td) / "out.bin"
        write_input(case, host, inp)
        res = subprocess.run([str(REPO / "oracle" / "_ref" / "ref_fdk"), "--repeat", str(args.repeat), str(inp),
                              str(out)], capture_output=True, text=True, timeout=3600)
        if res.returncode != 0:
            raise SystemExit(res.stderr[-2000:])
        ref = np.fromfile(out, dtype=np.float32).astype(np.float64).reshape(engine.shape)
        ref_exact = None
        if args.split:
            r2 = subprocess.run([str(REPO / "oracle" / "_ref" / "ref_fdk"), "--bp", "exact", str(inp), str(out)],
                                capture_output=True, text=True, timeout=3600)
            if r2.returncode != 0:
                raise SystemExit(r2.stderr[-2000:])
            ref_exact = np.fromfile(out, dtype=np.float32).astype(np.float64).reshape(engine.shape)
    times = [float(m) for m in re.findall(r"reconstruct ([0-9.]+) ms", res.stderr)]
    rel = lambda a, b: float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))
    nx, ny, nz = cfg["n"]
    updates = nx * ny * nz * cfg["nv"]
    print(json.dumps({"workload": args.config, "reference_reconstruct_ms": times,
                      "reference_gups_best": updates / (min(times) / 1000.0) / 1e9,
                      "rel_rms_vs_engine_fp32": rel(ref, engine),
                      "split": None if ref_exact is None else {
                          "lerp_part_ref_vs_ref_exact_fetch": rel(ref, ref_exact),
                          "engine_fp32_vs_ref_exact_fetch": rel(engine, ref_exact)},
                      "note": "wall time of GCT::Recon::CUDA::reconstruct per call, host buffers in and out"}))


if __name__ == "__main__":
    main()
