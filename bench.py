#!/usr/bin/env python
"""FDK benchmark: backprojection GUPS and recons/s on one or more B200s.

Workload (default ``cone512``): flat-panel cone-beam full scan, 512^3 volume at 0.5 mm, 720 views
over 360 degrees, 1024 x 768 detector at 0.4 mm, SOD 750 mm, SDD 1200 mm. Input: analytic line
integrals of 16 seeded random ellipsoids (FP64 on the device, cast to float32) with Poisson noise
at 1e5 incident photons per ray. A step is one full FDK reconstruction (weighting + ramp filter +
backprojection) of that input, resident in HBM. Inputs (2.26 GB) and the volume (537 MB) exceed the
126 MB L2, so no flush is needed between steps.

``value`` is GUPS (voxel x view updates per second, all GPUs) of the mixed-precision path (FP16
filtered storage with per-view scale, FP32 accumulation); the plain FP32 path is timed in the same
run (``fp32``). Errors are relative RMS / max against the FP64 CPU oracle on sampled voxels.

``--impl reference`` times the reference's CPU path. The reference (satidev/gct) has no CPU FDK,
so its stand-in is the FP64 oracle port (oracle/), run on all host cores on a bounded sample of the
same workload.

Multi-GPU: every rank reconstructs its own copy of the workload (independent reconstructions,
weak scaling, no collective on the data path); times are max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

CONFIGS = {
    "cone512": dict(kind="cone_flat", nv=720, nc=1024, nr=768, du=0.4, dv=0.4, sod=750.0, sdd=1200.0,
                    n=(512, 512, 512), vox=0.5, range=2 * math.pi, n_ell=16, i0=1e5,
                    label="flat-panel cone-beam full scan, 512^3 at 0.5 mm, 720 views, 1024x768 at 0.4 mm, "
                          "SOD 750, SDD 1200"),
    "cone256": dict(kind="cone_flat", nv=360, nc=512, nr=384, du=0.8, dv=0.8, sod=750.0, sdd=1200.0,
                    n=(256, 256, 256), vox=1.0, range=2 * math.pi, n_ell=16, i0=1e5,
                    label="flat-panel cone-beam full scan, 256^3 at 1 mm, 360 views, 512x384 at 0.8 mm, "
                          "SOD 750, SDD 1200 (profiling-size case)"),
    "short384": dict(kind="cone_flat", nv=496, nc=1240, nr=960, du=0.3, dv=0.3, sod=785.0, sdd=1200.0,
                     n=(512, 512, 384), vox=0.5, range=None, n_ell=16, i0=None,
                     label="flat-panel cone-beam short scan (pi + fan), 512x512x384, 496 views, 1240x960 at 0.3 mm, "
                           "SOD 785, SDD 1200"),
    "short256": dict(kind="cone_flat", nv=248, nc=620, nr=480, du=0.6, dv=0.6, sod=785.0, sdd=1200.0,
                     n=(256, 256, 192), vox=1.0, range=None, n_ell=16, i0=None,
                     label="flat-panel cone-beam short scan (pi + fan), 256x256x192, 248 views, 620x480 at 0.6 mm, "
                           "SOD 785, SDD 1200 (profiling-size case of short384)"),
    "fan256": dict(kind="fan_line", nv=360, nc=512, nr=1, du=1.2, dv=1.0, sod=570.0, sdd=1040.0,
                   n=(256, 256, 1), vox=1.0, range=2 * math.pi, n_ell=10, i0=None, phantom="water_disk",
                   label="fan-beam line detector full scan, 256^2 at 1 mm, 360 views, 512 cells at 1.2 mm, "
                         "SOD 570, SDD 1040"),
}


# Batched mix (C4, 48 reconstructions). Choices the mix leaves open are fixed here and echoed in
# the JSON line: 2D parallel N x N with 1.42 N cells (FOV 250 mm); fan arc 672 channels over a
# 0.907 rad fan (SOD 570, SDD 1040) into 512^2 at 0.9 mm; cylindrical cone 64 x 896 (arc 0.0011
# rad, rows 1.0 mm, SOD 600, SDD 1100) and cone-parallel (rebinned) 64 x 736 at 0.65 mm, both into
# 512 x 512 x 64 at 0.9 x 0.9 x 0.55 mm, 1152 views each.
BATCH48_2D = [(256, 180), (512, 360), (1024, 900), (2048, 1800)]
BATCH48_LABEL = ("48 uneven reconstructions in one persistent launch: 24 x 2D parallel (256-2048 px, 180-1800 "
                 "views), 8 x fan arc 672 ch x 1152 views -> 512^2, 8 x cylindrical cone 64x896 x 1152 views -> "
                 "512x512x64, 8 x cone-parallel 64x736 x 1152 views -> 512x512x64")
# Serving mix (C5): 70 % 2D fan (line detector, 768 cells at 1.0 mm, SOD 570, SDD 1040, 720 views ->
# 512^2 at 0.8 mm), 25 % cylindrical cone (the C4 geometry -> 512 x 512 x 64), 5 % flat cone 512^3
# (the cone512 workload); 80 GB budget, mixed precision (FP16 quads; the flat cone with the
# FP16-split Toeplitz filter, the others with the FFT filter).
SERVE_LABEL = ("Poisson arrivals, mix 70/25/5: 2D fan 512^2 x 720 views / cylindrical cone 512x512x64 x 1152 "
               "views / flat cone 512^3 x 720 views, 80 GB budget, mixed precision")
EXTRA_CONFIGS = ["batch48", "serve"]

# The headline metric, identical on both arms (the GPU arm and --impl reference).
METRIC = "FDK backprojection GUPS & recons/s, mixed-precision vs plain FP32 at stated FP64 error"


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["gct", "reference"], default="gct")
    ap.add_argument("--config", choices=sorted(CONFIGS) + EXTRA_CONFIGS, default="cone512")
    ap.add_argument("--serve-requests", type=int, default=160, help="requests per arrival rate (serve)")
    ap.add_argument("--serve-loads", type=str, default="0.3,0.6,0.9",
                    help="arrival rates as fractions of the measured capacity (serve)")
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--zpt", type=int, default=0, help="backprojection z per thread (0 = default)")
    ap.add_argument("--mixed-filter", choices=["gemm16", "gemm4", "gemm3", "fft"], default="gemm16",
                    help="ramp filter of the mixed path: split Toeplitz GEMM on tcgen05 with rows in two FP16 "
                         "pieces (one full term + three over the diagonal band), split-BF16 in the four-term "
                         "form (three pieces of rows and central taps) or three terms, or the FFT")
    ap.add_argument("--symmetry", choices=["auto", "off", "on"], default="auto",
                    help="quarter-turn and z-mirror backprojection forms: auto (FP16 storage, when the scan has "
                         "them), off, on")
    ap.add_argument("--no-error", action="store_true", help="skip the FP64 oracle error check")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--profile-path", choices=["mixed", "fp32"], default=None,
                    help="profiling run: build and time only this path's plan (a smaller device footprint for "
                         "ncu captures) and print its stage times instead of the benchmark line")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------------
# workload

def make_geometry(cfg):
    import gct_b200 as g
    nv, nc, nr = cfg["nv"], cfg["nc"], cfg["nr"]
    rng = cfg["range"]
    if rng is None:  # short scan: pi + full fan angle
        rng = math.pi + 2.0 * math.atan(nc * cfg["du"] / 2.0 / cfg["sdd"])
    rot = g.RotationParams(g.RotDir.CW, 0.0, rng / nv, nv)
    if cfg["kind"] == "cone_flat":
        det = (g.DetFanLine(nc, cfg["du"]), g.DetFanLine(nr, cfg["dv"]))
        params = g.ConeBeamProjGeomParams((nc - 1) / 2.0, rot, cfg["sdd"], cfg["sod"], (nr - 1) / 2.0)
    else:
        det = (g.DetFanLine(nc, cfg["du"]),)
        params = g.FanBeamProjGeomParams((nc - 1) / 2.0, rot, cfg["sdd"], cfg["sod"])
    cg = g.AxialCTGeom.from_params(det, params)
    nx, ny, nz = cfg["n"]
    v = cfg["vox"]
    if cfg["kind"] == "cone_flat":
        vg = g.ReconImgGeom(g.EqDistSampler(nx, v), g.EqDistSampler(ny, v), g.EqDistSampler(nz, v), (0.0, 0.0, 0.0))
    else:
        vg = g.ReconImgGeom(g.EqDistSampler(nx, v), g.EqDistSampler(ny, v), None, (0.0, 0.0))
    return cg, vg


# Water disk of the fan-beam workload: radius 120 mm (the configuration's "120 mm water disk" read
# as a radius, the only reading in which its ellipses of semi-axes up to 100 mm fit inside), water
# at 0.0193 / mm (about 70 keV).
WATER_DISK_RADIUS_MM = 120.0
WATER_MU_PER_MM = 0.0193


def water_disk_ellipses(n_ell, seed):
    """Seeded 2D phantom: a water disk plus n_ell ellipses with semi-axes U[5, 100] mm, added
    attenuation U[0.01, 0.05] / mm and random rotation, each inside the disk."""
    rs = np.random.RandomState(seed)
    R = WATER_DISK_RADIUS_MM
    ell = [(0.0, 0.0, 0.0, R, R, 1.0, 0.0, WATER_MU_PER_MM)]
    for _ in range(n_ell):
        a, b = rs.uniform(5.0, 100.0, size=2)
        room = max(R - max(a, b), 0.0)
        r, t = room * math.sqrt(rs.uniform()), rs.uniform(0, 2 * math.pi)
        ell.append((r * math.cos(t), r * math.sin(t), 0.0, a, b, 1.0, rs.uniform(0, math.pi), rs.uniform(0.01, 0.05)))
    return ell


def make_ellipsoids(cfg, seed):
    """Seeded phantom (mm, 1/mm): the water disk with ellipses for the fan-beam workload, else a
    water-like body plus random inner ellipsoids."""
    if cfg.get("phantom") == "water_disk":
        return water_disk_ellipses(cfg["n_ell"], seed)
    rs = np.random.RandomState(seed)
    nx, ny, nz = cfg["n"]
    half = 0.5 * cfg["vox"] * min(nx, ny)
    halfz = 0.5 * cfg["vox"] * nz if nz > 1 else half
    ell = [(0.0, 0.0, 0.0, 0.80 * half, 0.65 * half, 0.75 * halfz, 0.0, 0.019)]
    for _ in range(cfg["n_ell"] - 1):
        r = 0.55 * half * math.sqrt(rs.uniform())
        t = rs.uniform(0, 2 * math.pi)
        cz = rs.uniform(-0.5, 0.5) * halfz
        a = rs.uniform(5.0, 0.25 * half, size=3)
        ell.append((r * math.cos(t), r * math.sin(t), cz, a[0], a[1], min(a[2], 0.4 * halfz), rs.uniform(0, math.pi),
                    rs.uniform(0.01, 0.05) - 0.03))
    return ell


def make_projections(cg, cfg, seed, device):
    import torch
    import gct_b200 as g
    proj = torch.empty((cg.num_views, cg.num_rows, cg.num_cols), dtype=torch.float32, device=device)
    g.phantom_project(cg, make_ellipsoids(cfg, seed), proj)
    if cfg["i0"]:
        gen = torch.Generator(device=device)
        gen.manual_seed(seed)
        lam = cfg["i0"] * torch.exp(-proj.double())
        counts = torch.poisson(lam, generator=gen).clamp_(min=1.0)
        proj = (-torch.log(counts / cfg["i0"])).float()
        del lam, counts
    torch.cuda.synchronize()
    return proj.contiguous()


# ---------------------------------------------------------------------------------------------
# CPU oracle leg (reference arm and cpu_baseline)

def sample_rows(nr: int) -> tuple:
    """Detector rows [lo, hi) that the two central z-slices of a centred grid project onto."""
    lo = max(0, (nr - 1) // 2 - 7)
    return lo, min(nr, lo + 16)


def oracle_geometry(cfg, row_lo: int = 0, row_hi: int | None = None):
    """The workload's geometry built by the FP64 oracle's own view factory (no gct_b200), with the
    detector cut to rows [row_lo, row_hi) (a shifted row centre; identical for voxels whose
    projections stay inside those rows)."""
    from oracle import oracle as orc
    nv, nc, nr = cfg["nv"], cfg["nc"], cfg["nr"]
    rng = cfg["range"]
    if rng is None:  # short scan: pi + full fan angle
        rng = math.pi + 2.0 * math.atan(nc * cfg["du"] / 2.0 / cfg["sdd"])
    kind = orc.KIND[cfg["kind"]]
    row_hi = nr if row_hi is None else row_hi
    views = orc.make_views(kind, nv, (nc - 1) / 2.0, (nr - 1) / 2.0 - row_lo, cfg["sdd"], cfg["sod"], 1, 0.0,
                           rng / nv)
    if kind >= 3:
        return orc.Geometry(kind, nc, cfg["du"], views, row_hi - row_lo, cfg["dv"])
    return orc.Geometry(kind, nc, cfg["du"], views)


def oracle_sample(cfg, seed, proj_rows=None):
    """Bounded CPU sample: FP64 oracle FDK of the two central z-slices (all x, y) over all views.

    The detector is cut to the rows those slices project onto (geometry with a shifted row
    centre, identical for these voxels). Projections are the given device rows, or generated by
    the FP64 oracle phantom with numpy Poisson noise when None. Uses the oracle alone."""
    from oracle import oracle as orc
    nx, ny, nz = cfg["n"]
    k0 = nz // 2 - 1
    is3d = orc.KIND[cfg["kind"]] >= 3
    r_lo, r_hi = sample_rows(cfg["nr"]) if is3d else (0, 1)
    og = oracle_geometry(cfg, r_lo, r_hi)
    if proj_rows is None:
        p = orc.phantom(og, np.array(make_ellipsoids(cfg, seed)))
        if cfg["i0"]:
            rs = np.random.RandomState(seed)
            cnt = np.maximum(rs.poisson(cfg["i0"] * np.exp(-p)), 1.0)
            p = -np.log(cnt / cfg["i0"])
        proj_rows = p.astype(np.float32)
    nslab = 2 if nz > 1 else 1
    ov = orc.Volume(nx, ny, nz, cfg["vox"], cfg["vox"], cfg["vox"], (0.0, 0.0, 0.0))
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    vox = np.concatenate([np.stack([ii.ravel(), jj.ravel(), np.full(ii.size, k0 + s if nz > 1 else 0)], 1)
                          for s in range(nslab)]).astype(np.uint32)
    threads = os.cpu_count() or 1
    t = time.perf_counter()
    orc.fdk(og, ov, proj_rows, voxels=vox, use_fft=True, threads=threads)
    dt = time.perf_counter() - t
    updates = len(vox) * og.nv
    sample = (f"FP64 oracle FDK of {nslab} central z-slice(s) ({nx}x{ny}x{nslab} voxels) over all {og.nv} "
              f"views" + (f", detector rows {r_lo}-{r_hi - 1} (the rows those slices touch)" if is3d else "")
              + f", {threads} threads")
    return updates / dt / 1e9, threads, sample, (r_lo, r_hi)


def run_reference(args, cfg, rank):
    if rank != 0:
        return
    for _ in range(args.warmup):
        oracle_sample(cfg, args.seed)
    vals = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        v, threads, sample, _ = oracle_sample(cfg, args.seed)
        vals.append(v)
    wall = time.perf_counter() - t0
    value = float(np.median(vals))
    nx, ny, nz = cfg["n"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": "GUPS", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * wall / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.config, "description": cfg["label"], "volume": list(cfg["n"]),
                   "views": cfg["nv"], "detector": [cfg["nc"], cfg["nr"]]},
        "cpu_baseline": {"value": value, "unit": "GUPS", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "satidev/gct has no CPU FDK; the FP64 oracle port stands in for its CPU path",
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# GPU arm

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.path = Path(tempfile.mkstemp(prefix="clocks_", suffix=".csv")[1])
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(gpu_index)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        self.path.unlink(missing_ok=True)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# DRAM bytes per voxel-view update of the backprojectors, from ncu captures (dram__bytes_read.sum +
# dram__bytes_write.sum of one launch on the cone256 profiling case, divided by its updates). These
# are recorded figures, not measured by this run; the summary file names the command.
NCU_DRAM_BYTES_PER_UPDATE = {
    "bp_sym_kernel f16": (0.55, "profiles/backproject_sym_cone512_f16.md"),
}


def rooflines(cfg, updates, mixed, fp32, quarter, hbm, peak_kind, sm_mhz, num_sms, workload):
    """Roofline entries of the timed kernels.

    Backprojectors: the four bilinear taps of an update (8 B in FP16 quads, 16 B in FP32 quads)
    come through the SM's L1 data path from L1 and L2 (each quad is reused along rays), so the
    bound is that path, 128 B per clock per SM (nominal), not HBM; their compulsory HBM bytes
    (filtered stack read once, volume written once) are reported beside it.
    FFT filter: HBM-bound; algorithmic bytes 4 B read per detector pixel plus the padded quads
    written (16 B FP32). All achieved figures are per-launch bytes over the CUDA-event time of the
    stage on the launching stream."""
    nx, ny, nz = cfg["n"]
    nv, nc, nr = cfg["nv"], cfg["nc"], cfg["nr"]
    l1_peak = 128.0 * num_sms * sm_mhz * 1e6 / 1e9
    vox_bytes = 4.0 * nx * ny * nz
    quads = float(nv) * (nr + 4) * (nc + 4)  # padded quad grid per view
    out = {}
    for name, res, b_upd, kern in (("backproject_mixed", mixed, 8,
                                    "bp_sym_kernel (quarter-turn partners, FP16 quads)" if quarter
                                    else "bp_kernel (FP16 quads)"),
                                   ("backproject_fp32", fp32, 16, "bp_kernel (FP32 quads)")):
        t = res["bp_ms"] / 1000.0
        ach = updates * b_upd / t / 1e9
        comp = quads * b_upd + vox_bytes
        e = {"bound": "l1", "kernel": kern, "achieved": ach, "peak": l1_peak, "unit": "GB/s",
             "frac": ach / l1_peak, "peak_source": "nominal 128 B/clk per SM x SMs x median SM clock under load",
             "algorithmic_bytes_per_update": b_upd, "traffic": None,
             "hbm_compulsory": {"bytes": comp, "achieved": comp / t / 1e9, "peak": hbm, "unit": "GB/s",
                                "frac": comp / t / 1e9 / hbm, "peak_source": peak_kind}}
        key = "bp_sym_kernel f16" if (name == "backproject_mixed" and quarter) else None
        if key in NCU_DRAM_BYTES_PER_UPDATE and workload in ("cone512", "cone256"):
            per, src = NCU_DRAM_BYTES_PER_UPDATE[key]
            e["traffic_ncu"] = {"bytes_per_launch": per * updates, "bytes_per_update": per, "source": src}
        out[name] = e
    t = fp32["filt_ms"] / 1000.0
    fb = float(nv) * nr * nc * 4 + quads * 16
    out["filter_fft_fp32"] = {"bound": "hbm", "kernel": "filter_fft_kernel (FP32 quads)", "achieved": fb / t / 1e9,
                              "peak": hbm, "unit": "GB/s", "frac": fb / t / 1e9 / hbm, "peak_source": peak_kind,
                              "algorithmic_bytes": fb, "traffic": None}
    return out


def sample_voxels(cfg, seed):
    nx, ny, nz = cfg["n"]
    rs = np.random.RandomState(seed + 7)
    ks = np.linspace(nz // 8, nz - 1 - nz // 8, 6).astype(int) if nz > 1 else np.zeros(1, int)
    pts = []
    for k in ks:
        ii = rs.randint(0, nx, 700)
        jj = rs.randint(0, ny, 700)
        pts.append(np.stack([ii, jj, np.full(700, k)], 1))
    return np.concatenate(pts).astype(np.uint32)


def oracle_errors(cg, cfg, proj_dev, vols, seed):
    """relRMS / max error of each device volume against the FP64 oracle on sampled voxels."""
    from oracle import oracle as orc
    vox = sample_voxels(cfg, seed)
    proj = proj_dev.cpu().numpy()
    og = orc.Geometry(int(cg.kind), cg.num_cols, cg.det_geom()[0].sampling_width, cg.views,
                      cg.num_rows, cg.det_geom()[1].sampling_width if cg.is_3d else 1.0)
    nx, ny, nz = cfg["n"]
    ov = orc.Volume(nx, ny, nz, cfg["vox"], cfg["vox"], cfg["vox"], (0.0, 0.0, 0.0))
    ref = orc.fdk(og, ov, proj, voxels=vox, use_fft=True)
    out = {}
    for name, vol in vols.items():
        v = vol.reshape(-1)
        flat = (vox[:, 2].astype(np.int64) * ny + vox[:, 1]) * nx + vox[:, 0]
        got = v[flat].double().cpu().numpy() if hasattr(v, "cpu") else v[flat]
        out[name] = {"rel_rms": float(np.sqrt(np.mean((got - ref) ** 2) / np.mean(ref ** 2))),
                     "max_rel": float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))}
    return out, len(vox)


def sampled_oracle_error(cg, c, proj, vol, seed, nvox=2000):
    """relRMS / max error of one reconstruction (host arrays) against the FP64 oracle on nvox
    sampled voxels (3D volumes: the two central slices, detector cut to the rows those slices
    project onto), with the oracle's time for them as a CPU rate (voxel x view updates / s)."""
    from oracle import oracle as orc
    nx, ny, nz = c["n"]
    rs = np.random.RandomState(seed)
    is3d = cg.is_3d
    k = np.full(nvox, 0) if nz <= 1 else (nz // 2 - 1 + (np.arange(nvox) % 2))
    vox = np.stack([rs.randint(0, nx, nvox), rs.randint(0, ny, nvox), k], 1).astype(np.uint32)
    views = cg.views.copy()
    r_lo, r_hi = (sample_rows(cg.num_rows) if is3d else (0, 1))
    if is3d:
        views["det_col_center"] -= r_lo
    det = cg.det_geom()
    og = orc.Geometry(int(cg.kind), cg.num_cols, det[0].sampling_width, views, (r_hi - r_lo) if is3d else 1,
                      det[1].sampling_width if is3d else 1.0)
    vz = c.get("voxz", c["vox"])
    ov = orc.Volume(nx, ny, max(nz, 1), c["vox"], c["vox"], vz, (0.0, 0.0, 0.0))
    rows = np.ascontiguousarray(proj[:, r_lo:r_hi, :]) if is3d else proj
    threads = os.cpu_count() or 1
    t = time.perf_counter()
    ref = orc.fdk(og, ov, rows, voxels=vox, use_fft=True, threads=threads)
    dt = time.perf_counter() - t
    flat = (vox[:, 2].astype(np.int64) * ny + vox[:, 1]) * nx + vox[:, 0]
    got = np.asarray(vol, dtype=np.float64).reshape(-1)[flat]
    err = {"voxels": int(nvox), "rel_rms": float(np.sqrt(np.mean((got - ref) ** 2) / np.mean(ref ** 2))),
           "max_rel": float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))}
    return err, len(vox) * cg.num_views / dt / 1e9, threads


def time_plan(plan, proj, vol, steps, warmup, stream, dist):
    """Times `steps` full FDKs: returns (total seconds max over ranks, mean filter ms, mean BP ms)."""
    import torch
    for _ in range(warmup):
        plan.prepare(proj, stream=stream)
        plan.backproject(vol, stream=stream)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    start.record(stream)
    for s in range(steps):
        ev[s][0].record(stream)
        plan.prepare(proj, stream=stream)
        ev[s][1].record(stream)
        plan.backproject(vol, stream=stream)
        ev[s][2].record(stream)
    stop.record(stream)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    total = start.elapsed_time(stop) / 1000.0
    filt = float(np.mean([e[0].elapsed_time(e[1]) for e in ev]))
    bp = float(np.mean([e[1].elapsed_time(e[2]) for e in ev]))
    if dist:
        total = max_over_ranks(total, "cuda")
    return total, filt, bp


def time_plans_interleaved(plans, proj, vols, steps, warmup, stream, dist):
    """Times `steps` full FDKs of each plan with the plans' steps interleaved (plan a step, plan b
    step, ...), so that every path runs under the same clocks and power state; each step is
    device-timed with CUDA events on the launching stream. Returns {name: (seconds of that plan's
    steps, max over ranks; mean filter ms; mean BP ms)}."""
    import torch
    for _ in range(warmup):
        for name, plan in plans.items():
            plan.prepare(proj, stream=stream)
            plan.backproject(vols[name], stream=stream)
    ev = {name: [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)] for name in plans}
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    for s in range(steps):
        for name, plan in plans.items():
            e = ev[name][s]
            e[0].record(stream)
            plan.prepare(proj, stream=stream)
            e[1].record(stream)
            plan.backproject(vols[name], stream=stream)
            e[2].record(stream)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    out = {}
    for name in plans:  # every rank takes the same reductions in the same order
        total = sum(e[0].elapsed_time(e[2]) for e in ev[name]) / 1000.0
        if dist:
            total = max_over_ranks(total, "cuda")
        out[name] = (total, float(np.mean([e[0].elapsed_time(e[1]) for e in ev[name]])),
                     float(np.mean([e[1].elapsed_time(e[2]) for e in ev[name]])))
    return out


def max_over_ranks(value: float, device) -> float:
    """The job's time for a per-rank time: the maximum over all ranks (every rank calls this)."""
    import torch
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank: float, world: int, steps: int, seconds: float) -> float:
    """Whole-job rate of `world` independent replicas, each processing units_per_rank per step,
    over the max-over-ranks time."""
    return units_per_rank * world * steps / seconds


def run_gct(args, cfg, rank, world, local_rank):
    import torch
    import gct_b200 as g
    dist = world > 1
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    cg, vg = make_geometry(cfg)
    nx, ny, nz = cfg["n"]
    updates = nx * ny * nz * cg.num_views
    proj = make_projections(cg, cfg, args.seed + rank, device)
    stream = torch.cuda.current_stream()
    mixed_filter = {"gemm16": g.FILTER_TOEPLITZ_F16X2, "gemm4": g.FILTER_TOEPLITZ_BF16X4,
                    "gemm3": g.FILTER_TOEPLITZ_BF16X3, "fft": g.FILTER_FFT}[args.mixed_filter]
    sym = {"auto": g.SYMMETRY_AUTO, "off": g.SYMMETRY_OFF, "on": g.SYMMETRY_ON}[args.symmetry]
    opts = {"mixed": g.FdkOptions(filter=mixed_filter, storage=g.STORAGE_F16, z_per_thread=args.zpt, symmetry=sym),
            "fp32": g.FdkOptions(filter=g.FILTER_FFT, storage=g.STORAGE_F32, z_per_thread=args.zpt, symmetry=sym)}
    if args.profile_path:
        plan = g.FdkPlan(cg, vg, opts=opts[args.profile_path])
        vol = torch.empty(vg.shape, dtype=torch.float32, device=device)
        total, filt_ms, bp_ms = time_plan(plan, proj, vol, args.steps, args.warmup, stream, dist)
        plan.check()
        if rank == 0:
            print(json.dumps({"profile_path": args.profile_path, "workload": args.config, "steps": args.steps,
                              "ms_per_step": 1000.0 * total / args.steps, "stages_ms": {"filter": filt_ms,
                                                                                         "backproject": bp_ms},
                              "quarter_turn": plan.quarter_turn}), flush=True)
        plan.close()
        return
    plans = {k: g.FdkPlan(cg, vg, opts=o) for k, o in opts.items()}
    mixed_quarter_turn = plans["mixed"].quarter_turn
    vols = {k: torch.empty(vg.shape, dtype=torch.float32, device=device) for k in plans}
    for k, p in plans.items():
        p.execute(proj, vols[k], stream=stream)
    torch.cuda.synchronize()

    errors, nsamp = (None, 0)
    if rank == 0 and not args.no_error:
        errors, nsamp = oracle_errors(cg, cfg, proj, vols, args.seed)

    # the two paths' steps alternate, so that the comparison sees one set of clocks (timed one
    # after the other, the second path ran under the first one's power cap)
    sampler = ClockSampler(local_rank)
    timed = time_plans_interleaved({"fp32": plans["fp32"], "mixed": plans["mixed"]}, proj, vols, args.steps,
                                   args.warmup, stream, dist)
    clocks = sampler.stop()
    results = {}
    for name, (total, filt_ms, bp_ms) in timed.items():
        results[name] = dict(total=total, filt_ms=filt_ms, bp_ms=bp_ms,
                             gups=replica_rate(updates, world, args.steps, total) / 1e9)

    e2e = None
    if not args.no_e2e:
        plan = plans["mixed"]
        host_proj = torch.empty(proj.shape, dtype=torch.float32, pin_memory=True)
        host_proj.copy_(proj)
        host_vol = torch.empty(vg.shape, dtype=torch.float32, pin_memory=True)
        hp, hv = host_proj.numpy(), host_vol.numpy()
        def host_run(asynchronous):
            # every step uploads its projections from pinned host memory and downloads its volume;
            # the asynchronous calls overlap one step's uploads and download with its neighbours'
            for _ in range(max(1, args.warmup)):
                (plan.execute_host_async if asynchronous else plan.execute_host)(hp, hv, stream=stream)
            plan.host_sync()
            if dist:
                torch.distributed.barrier()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                (plan.execute_host_async if asynchronous else plan.execute_host)(hp, hv, stream=stream)
            plan.host_sync()
            t = time.perf_counter() - t0
            return max_over_ranks(t, device) if dist else t
        te = host_run(True)
        ts = host_run(False)
        e2e = {"value": replica_rate(updates, world, args.steps, te) / 1e9, "unit": "GUPS",
               "h2d_bytes_per_step": int(proj.numel() * 4), "d2h_bytes_per_step": int(host_vol.numel() * 4),
               "ms_per_step": 1000.0 * te / args.steps,
               "path": "gct_fdk_execute_host_async per step (pinned host buffers), gct_fdk_host_sync at the end",
               "one_call_at_a_time": {"value": replica_rate(updates, world, args.steps, ts) / 1e9, "unit": "GUPS",
                                      "ms_per_step": 1000.0 * ts / args.steps, "path": "gct_fdk_execute_host"}}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        # same sampled rows of the device input, so the baseline reconstructs identical data
        r_lo, r_hi = sample_rows(cg.num_rows)
        rows = proj[:, r_lo:r_hi, :].contiguous().cpu().numpy()
        v, threads, sample, _ = oracle_sample(cfg, args.seed, proj_rows=rows)
        cpu = {"value": v, "unit": "GUPS", "cores": threads, "kind": "port", "sample": sample}

    if rank != 0:
        return
    hbm, peak_kind = measured_peaks()
    mixed = results["mixed"]
    rl = rooflines(cfg, updates, mixed, results["fp32"], mixed_quarter_turn, hbm, peak_kind,
                   (clocks or {}).get("sm_mhz") or 1965.0,
                   torch.cuda.get_device_properties(local_rank).multi_processor_count, args.config)
    line = {
        "metric": METRIC, "value": mixed["gups"], "precision": "mixed (FP16 filtered storage, FP32 accumulation)",
        "unit": "GUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * mixed["total"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32-accumulate/f16-storage", "data": "synthetic",
        "config": {"workload": args.config, "description": cfg["label"], "volume": list(cfg["n"]),
                   "views": cfg["nv"], "detector": [cfg["nc"], cfg["nr"]], "phantom": (f"{cfg['n_ell']} seeded ellipses in a {WATER_DISK_RADIUS_MM:g} mm radius water disk"
                               if cfg.get("phantom") == "water_disk" else f"{cfg['n_ell']} seeded ellipsoids"),
                   "noise": f"Poisson I0={cfg['i0']:g}" if cfg["i0"] else "none", "l2": "inputs larger than L2, no flush",
                   "timing": "mixed and FP32 steps interleaved, each device-timed with CUDA events",
                   "parallelism": f"replicas x{world}"},
        "recons_per_s": world * args.steps / mixed["total"],
        "stages_ms": {"filter": mixed["filt_ms"], "backproject": mixed["bp_ms"]},
        "quarter_turn": {"mixed": mixed_quarter_turn, "fp32": plans["fp32"].quarter_turn},
        "fp32": {"value": results["fp32"]["gups"], "unit": "GUPS",
                 "recons_per_s": world * args.steps / results["fp32"]["total"],
                 "stages_ms": {"filter": results["fp32"]["filt_ms"], "backproject": results["fp32"]["bp_ms"]}},
        "speedup_mixed_vs_fp32": mixed["gups"] / results["fp32"]["gups"],
        "error_vs_fp64_oracle": ({"voxels": nsamp, **errors} if errors else None),
        "roofline": rl["backproject_mixed"],
        "rooflines": {k: v for k, v in rl.items() if k != "backproject_mixed"},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clocks,
        # per mixed step: GEMM forms split (with the view maxima), view scales, GEMM (writing the
        # partner quads of quarter-turn stacks itself), quads (view-major stacks), backprojection;
        # FFT: view maxima, view scales, FFT filter, (partner quads), backprojection
        "gpu_launches": (5 if (args.mixed_filter != "fft") != bool(mixed_quarter_turn) else 4) * args.steps,
        "mixed_filter": {"gemm16": "split-FP16 Toeplitz GEMM on tcgen05, 1 full term + 3 banded (rows scaled per row "
                                   "in two FP16 pieces, central taps in three, far taps' dropped parts folded into "
                                   "the central tap)",
                         "gemm4": "split-BF16 Toeplitz GEMM on tcgen05, 3 full terms + 2 banded (rows and central "
                                  "taps in three BF16 pieces)",
                         "gemm3": "split-BF16 Toeplitz GEMM on tcgen05, 3 terms",
                         "fft": "shared-memory FFT"}[args.mixed_filter],
    }
    print(json.dumps(line), flush=True)


def batch48_items():
    items = []
    for i in range(24):
        n, nv = BATCH48_2D[i % 4]
        items.append(dict(kind="parallel_1d", nv=nv, nc=int(math.ceil(1.42 * n)), nr=1, du=250.0 / n, dv=1.0,
                          n=(n, n, 1), vox=250.0 / n, voxz=1.0, n_ell=10))
    for _ in range(8):
        items.append(dict(kind="fan_arc", nv=1152, nc=672, nr=1, du=0.907 / 672, dv=1.0, sod=570.0, sdd=1040.0,
                          n=(512, 512, 1), vox=0.9, voxz=1.0, n_ell=10))
    for _ in range(8):
        items.append(cyl_item())
    for _ in range(8):
        items.append(dict(kind="cone_parallel", nv=1152, nc=736, nr=64, du=0.65, dv=1.0, sod=600.0, sdd=1100.0,
                          n=(512, 512, 64), vox=0.9, voxz=0.55, n_ell=16))
    return items


def cyl_item():
    return dict(kind="cone_cyl", nv=1152, nc=896, nr=64, du=0.0011, dv=1.0, sod=600.0, sdd=1100.0,
                n=(512, 512, 64), vox=0.9, voxz=0.55, n_ell=16)


def make_geometry2(c):
    """Full-scan geometry of a batch or serving item, any of the seven kinds' factories."""
    import gct_b200 as g
    nv, nc, nr = c["nv"], c["nc"], c["nr"]
    rot = g.RotationParams(g.RotDir.CW, 0.0, 2 * math.pi / nv, nv)
    c0, r0 = (nc - 1) / 2.0, (nr - 1) / 2.0
    k = c["kind"]
    if k == "parallel_1d":
        det, params = (g.DetParallel(nc, c["du"]),), g.Parallel1DProjGeomParams(c0, rot)
    elif k == "fan_arc":
        det, params = (g.DetFanArc(nc, c["du"]),), g.FanBeamProjGeomParams(c0, rot, c["sdd"], c["sod"])
    elif k == "fan_line":
        det, params = (g.DetFanLine(nc, c["du"]),), g.FanBeamProjGeomParams(c0, rot, c["sdd"], c["sod"])
    elif k == "cone_cyl":
        det = (g.DetFanArc(nc, c["du"]), g.DetFanLine(nr, c["dv"]))
        params = g.ConeBeamProjGeomParams(c0, rot, c["sdd"], c["sod"], r0)
    elif k == "cone_parallel":
        det = (g.DetParallel(nc, c["du"]), g.DetFanLine(nr, c["dv"]))
        params = g.ConeBeamProjGeomParams(c0, rot, c["sdd"], c["sod"], r0)
    elif k == "cone_flat":
        det = (g.DetFanLine(nc, c["du"]), g.DetFanLine(nr, c["dv"]))
        params = g.ConeBeamProjGeomParams(c0, rot, c["sdd"], c["sod"], r0)
    else:
        raise KeyError(k)
    cg = g.AxialCTGeom.from_params(det, params)
    nx, ny, nz = c["n"]
    if nr > 1:
        vg = g.ReconImgGeom(g.EqDistSampler(nx, c["vox"]), g.EqDistSampler(ny, c["vox"]),
                            g.EqDistSampler(nz, c["voxz"]), (0.0, 0.0, 0.0))
    else:
        vg = g.ReconImgGeom(g.EqDistSampler(nx, c["vox"]), g.EqDistSampler(ny, c["vox"]), None, (0.0, 0.0))
    return cg, vg


def item_projections(cg, c, seed, device):
    import torch
    import gct_b200 as g
    proj = torch.empty((cg.num_views, cg.num_rows, cg.num_cols), dtype=torch.float32, device=device)
    g.phantom_project(cg, make_ellipsoids(dict(n=c["n"], vox=c["vox"], n_ell=c["n_ell"]), seed), proj)
    return proj


def device_timed(fn, steps, warmup, stream, dist, device):
    import torch
    for _ in range(warmup):
        fn()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    start.record(stream)
    for _ in range(steps):
        fn()
    stop.record(stream)
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    total = start.elapsed_time(stop) / 1000.0
    if dist:
        total = max_over_ranks(total, device)
    return total


def run_batch(args, rank, world, local_rank):
    """C4: 48 uneven reconstructions as one batch (filters on forked streams + one persistent
    work-queue backprojection, replayed as a CUDA graph), against the same 48 plans run one after
    another through gct_fdk_execute."""
    import torch
    import gct_b200 as g
    dist = world > 1
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream()
    specs = batch48_items()
    plans, projs, vols = [], [], []
    updates = 0
    for i, c in enumerate(specs):
        cg, vg = make_geometry2(c)
        projs.append(item_projections(cg, c, args.seed + 17 * i + rank, device))
        plans.append(g.FdkPlan(cg, vg, opts=g.FdkOptions(filter=g.FILTER_FFT, storage=g.STORAGE_F16)))
        vols.append(torch.empty(vg.shape, dtype=torch.float32, device=device))
        updates += int(np.prod(c["n"])) * c["nv"]
    torch.cuda.synchronize()
    t_build = time.perf_counter()
    batch = g.FdkBatch(list(zip(plans, projs, vols)))
    t_build = time.perf_counter() - t_build
    n_work, upd = batch.work()
    assert upd == updates
    sampler = ClockSampler(local_rank)
    t_batch = device_timed(lambda: batch.launch(stream=stream), args.steps, args.warmup, stream, dist, device)
    clocks = sampler.stop()
    batch_vols = [v.clone() for v in vols]
    errors, cpu = None, None
    if rank == 0 and not args.no_error:
        # one item of each geometry class, checked against the FP64 oracle on sampled voxels
        errors, rates, threads = {}, [], 1
        seen = set()
        for i, c in enumerate(specs):
            key = f"{c['kind']} {c['n'][0]}x{c['n'][1]}x{c['n'][2]} nv={c['nv']}"
            if c["kind"] in seen or (c["kind"] == "parallel_1d" and c["n"][0] != 1024):
                continue
            seen.add(c["kind"])
            cg_i, _ = make_geometry2(c)
            err, rate, threads = sampled_oracle_error(cg_i, c, projs[i].cpu().numpy(), batch_vols[i].cpu().numpy(),
                                                      args.seed + i)
            errors[key] = err
            rates.append(rate)
        cpu = {"value": float(np.median(rates)), "unit": "GUPS", "cores": threads, "kind": "port",
               "sample": "FP64 oracle FDK of 2000 sampled voxels (3D: the two central slices) of one item per "
                         f"geometry class, all views, {threads} threads; median over the classes"}

    def sequential():
        for p, pr, v in zip(plans, projs, vols):
            p.execute(pr, v, stream=stream)
    t_seq = device_timed(sequential, args.steps, args.warmup, stream, dist, device)
    diff = max(float(((a - b).norm() / b.norm().clamp_min(1e-30)).item()) for a, b in zip(batch_vols, vols))
    configs = {}
    for i, c in enumerate(specs):
        configs[f"{c['kind']} {c['n'][0]}x{c['n'][1]}x{c['n'][2]} nv={c['nv']}"] = batch.item_config(i)
    batch.close()
    for p in plans:
        p.close()
    if rank != 0:
        return
    line = {
        "metric": "FDK batched backprojection GUPS (voxel x view updates / s), 48 mixed reconstructions",
        "value": replica_rate(updates, world, args.steps, t_batch) / 1e9, "unit": "GUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t_batch / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32-accumulate/f16-storage", "data": "synthetic",
        "config": {"workload": "batch48", "description": BATCH48_LABEL, "items": len(specs),
                   "filter": "shared-memory FFT", "l2": "inputs larger than L2, no flush",
                   "parallelism": f"replicas x{world}"},
        "recons_per_s": world * len(specs) * args.steps / t_batch,
        "sequential": {"value": replica_rate(updates, world, args.steps, t_seq) / 1e9, "unit": "GUPS",
                       "ms_per_step": 1000.0 * t_seq / args.steps,
                       "path": "the same 48 plans through gct_fdk_execute one after another"},
        "speedup_batch_vs_sequential": t_seq / t_batch,
        "max_rel_diff_batch_vs_sequential": diff,
        "work_entries": n_work, "batch_build_s": t_build, "tile_configs": configs,
        "clocks": clocks, "gpu_launches": (3 * len(specs) + 1) * args.steps,
        "error_vs_fp64_oracle": errors, "cpu_baseline": cpu, "e2e": None,
    }
    print(json.dumps(line), flush=True)


def run_serve(args, rank, world, local_rank):
    """C5: Poisson arrivals of the 70/25/5 mix into the serving loop (80 GB budget) at several
    arrival rates, host buffers in and out; p50/p99 latency and recons/s per rate."""
    import threading
    import torch
    import gct_b200 as g
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    kinds = [
        ("fan2d", 0.70, dict(kind="fan_line", nv=720, nc=768, nr=1, du=1.0, dv=1.0, sod=570.0, sdd=1040.0,
                             n=(512, 512, 1), vox=0.8, voxz=1.0, n_ell=10), g.FILTER_FFT, 64),
        ("cyl", 0.25, cyl_item(), g.FILTER_FFT, 24),
        ("flat", 0.05, dict(kind="cone_flat", nv=720, nc=1024, nr=768, du=0.4, dv=0.4, sod=750.0, sdd=1200.0,
                            n=(512, 512, 512), vox=0.5, voxz=0.5, n_ell=16), g.FILTER_TOEPLITZ_F16X2, 6),
    ]
    cls = []
    for i, (name, frac, c, filt, nbuf) in enumerate(kinds):
        cg, vg = make_geometry2(c)
        proj = item_projections(cg, c, args.seed + i, device)
        hp = torch.empty(proj.shape, dtype=torch.float32, pin_memory=True)
        hp.copy_(proj)
        del proj
        plan = g.FdkPlan(cg, vg, opts=g.FdkOptions(filter=filt, storage=g.STORAGE_F16))
        outs = [torch.empty(vg.shape, dtype=torch.float32, pin_memory=True).numpy() for _ in range(nbuf)]
        cls.append(dict(name=name, frac=frac, plan=plan, proj=hp.numpy(), outs=outs,
                        updates=int(np.prod(c["n"])) * c["nv"]))
    torch.cuda.empty_cache()
    srv = g.FdkServer(80 << 30)

    def run_load(rate, nreq, seed):
        rng = np.random.default_rng(seed)
        picks = rng.choice(len(cls), size=nreq, p=[k["frac"] for k in cls])
        gaps = rng.exponential(1.0 / rate, size=nreq) if rate > 0 else np.zeros(nreq)
        owner = {}   # (class, buffer) -> ticket still using it
        nxt = [0] * len(cls)
        tickets = []
        t0 = time.perf_counter()
        due = t0
        for k, gap in zip(picks, gaps):
            due += gap
            now = time.perf_counter()
            if due > now:
                time.sleep(due - now)
            b = nxt[k]
            nxt[k] = (b + 1) % len(cls[k]["outs"])
            prev = owner.get((k, b))
            if prev is not None:
                srv.wait(prev)
            t = srv.submit(cls[k]["plan"], cls[k]["proj"], cls[k]["outs"][b])
            owner[(k, b)] = t
            tickets.append((k, t))
        for _, t in tickets:
            srv.wait(t)
        span = time.perf_counter() - t0
        lat = {}
        for k, t in tickets:
            lat.setdefault(cls[k]["name"], []).append(srv.info(t)["latency_ms"])
        allv = np.concatenate([np.array(v) for v in lat.values()])
        upd = sum(cls[k]["updates"] for k, _ in tickets)
        return {"offered_per_s": rate, "requests": nreq, "recons_per_s": nreq / span, "gups": upd / span / 1e9,
                "p50_ms": float(np.percentile(allv, 50)), "p99_ms": float(np.percentile(allv, 99)),
                "per_class": {n: {"n": len(v), "p50_ms": float(np.percentile(v, 50)),
                                  "p99_ms": float(np.percentile(v, 99))} for n, v in lat.items()}}

    # capacity: everything submitted at once (closed loop), after a warm-up pass
    run_load(0, 24, args.seed + 99)
    sat = run_load(0, args.serve_requests, args.seed + 100)
    cap = sat["recons_per_s"]
    sampler = ClockSampler(local_rank)
    loads = []
    for j, f in enumerate(float(x) for x in args.serve_loads.split(",")):
        loads.append(dict(load=f, **run_load(f * cap, args.serve_requests, args.seed + 200 + j)))
    clocks = sampler.stop()
    errors, cpu = None, None
    if rank == 0 and not args.no_error:
        errors, rates, threads = {}, [], 1
        for i, (name, frac, c, filt, nbuf) in enumerate(kinds):
            k = cls[i]
            cg_i, _ = make_geometry2(c)
            # the class's buffer 0 holds a completed reconstruction of the class's projections
            err, rate, threads = sampled_oracle_error(cg_i, c, k["proj"], k["outs"][0], args.seed + i)
            errors[name] = err
            rates.append(rate)
        cpu = {"value": float(np.median(rates)), "unit": "GUPS", "cores": threads, "kind": "port",
               "sample": "FP64 oracle FDK of 2000 sampled voxels (3D: the two central slices) of each request "
                         f"class, all views, {threads} threads; median over the classes"}
    st = srv.stats()
    srv.close()
    for k in cls:
        k["plan"].close()
    if rank != 0:
        return
    mid = loads[len(loads) // 2]
    line = {
        "metric": "FDK serving recons/s with p50/p99 latency (continuous batching, 1 GPU)",
        "value": mid["recons_per_s"], "unit": "recons/s", "n_gpus": world, "steps": args.serve_requests,
        "warmup": 24, "ms_per_step": 1000.0 / mid["recons_per_s"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32-accumulate/f16-storage", "data": "synthetic",
        "config": {"workload": "serve", "description": SERVE_LABEL, "budget_bytes": 80 << 30,
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2, no flush"},
        "p50_ms": mid["p50_ms"], "p99_ms": mid["p99_ms"], "capacity": sat, "loads": loads,
        "server": {"rounds": st["rounds"], "peak_active": st["peak_active"], "peak_bytes": st["peak_bytes"]},
        "e2e": {"value": mid["recons_per_s"], "unit": "recons/s", "path": "host buffers in and out through the server"},
        "clocks": clocks, "error_vs_fp64_oracle": errors, "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.config in EXTRA_CONFIGS:
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": f"the {args.config} workload has no CPU leg; "
                                  "the reference arm runs on the cone512 workload"}), flush=True)
            return
        if world > 1:
            import datetime
            import torch
            torch.cuda.set_device(local_rank)
            torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                                 device_id=torch.device("cuda", local_rank))
        try:
            (run_batch if args.config == "batch48" else run_serve)(args, rank, world, local_rank)
        finally:
            if world > 1:
                import torch
                torch.distributed.destroy_process_group()
        return
    cfg = CONFIGS[args.config]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, cfg, rank)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local_rank))
    try:
        run_gct(args, cfg, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
