"""Generates tests/golden/ref_host_vectors.npz from satidev/gct's own host-callable functions.

Run after ``bash oracle/build_ref.sh`` (which compiles the reference sources under the reference
tree into oracle/_ref/libgct_ref_host.so):

    python tests/golden/make_golden.py

The vectors are the reference's FP32 outputs for seeded inputs: ramp-filter taps, rotation
analysis, Parker tables, cosine weights, projMapping coordinates/weights and voxel positions. The
tests compare the FP64 oracle and the engine's host geometry against them.
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
LIB = REPO / "oracle" / "_ref" / "libgct_ref_host.so"
OUT = HERE / "ref_host_vectors.npz"

F = C.POINTER(C.c_float)


def load():
    lib = C.CDLL(str(LIB))
    lib.ref_filter_taps.argtypes = [C.c_int, C.c_uint, C.c_float, C.c_float, C.c_int, F]
    lib.ref_rotation.argtypes = [F, C.c_uint, C.POINTER(C.c_int), F, F, C.POINTER(C.c_uint), F]
    lib.ref_parker_weight_fan.argtypes = [C.c_float] * 4
    lib.ref_parker_weight_fan.restype = C.c_float
    lib.ref_parker_table.argtypes = [C.c_int, C.c_uint, C.c_float, C.c_uint, F, F, C.c_float, C.c_float, F]
    lib.ref_view_eval.argtypes = [C.c_int, F, C.c_float, C.c_float, C.c_uint, C.c_uint, C.c_float, C.c_float,
                                  C.c_float, F, F, F]
    lib.ref_view_eval.restype = C.c_float
    lib.ref_vox_pos.argtypes = [C.c_uint] * 3 + [C.c_float] * 6 + [C.c_uint] * 3 + [F]
    lib.ref_vox_pos.restype = None
    return lib


def fp(a):
    return a.ctypes.data_as(F)


def fan_views(nv, start, rng, rot_dir, sid):
    """Fan-beam views of an ideal circular scan (source at R_z(dir*theta)(SID, 0))."""
    th = start + rng / nv * np.arange(nv)
    phi = rot_dir * th
    src = np.stack([sid * np.cos(phi), sid * np.sin(phi)], 1).astype(np.float32)
    row = np.stack([-np.sin(phi), np.cos(phi)], 1).astype(np.float32)
    return src, row


def main():
    lib = load()
    rs = np.random.RandomState(20231025)
    out = {}

    # ramp-filter taps: (kind, n, width, cut-off, apodisation)
    tap_cases = []
    taps = []
    for kind, width in [(0, 0.8961), (1, 0.0017922), (2, 2.0)]:
        for n in (511, 512, 1024):
            for fc, apod in [(1.0, 0), (0.8, 1), (0.6, 2)]:
                t = np.zeros(n, np.float32)
                lib.ref_filter_taps(kind, n, width, fc, apod, fp(t))
                tap_cases.append((kind, n, width, fc, apod))
                taps.append(t)
    out["taps_cases"] = np.array(tap_cases, dtype=np.float64)
    out["taps_values"] = np.concatenate(taps)

    # rotation analysis of angle sequences (degrees -> float radians)
    seqs = [[1, 2, 3], [-10, -9, -8], [358, 0, 2], [361, 2, 3], [3, 2, 1], [-10, -12, -14], [2, 0, 358],
            [3, 361, 359], [180, 360, 540, 0], [0, 540, 360, 180], [90, 270, 90], [0, 180, 360, 0]]
    for _ in range(8):
        n = rs.randint(5, 40)
        start = rs.uniform(-400, 400)
        step = rs.choice([-1, 1]) * rs.uniform(0.3, 20)
        seqs.append(list(start + step * np.arange(n)))
    rot_rows, rel_all = [], []
    for s in seqs:
        a = np.radians(np.array(s, dtype=np.float64)).astype(np.float32)
        d, nppr = C.c_int(), C.c_uint()
        incr, rng = C.c_float(), C.c_float()
        rel = np.zeros(len(a), np.float32)
        rc = lib.ref_rotation(fp(a), len(a), C.byref(d), C.byref(incr), C.byref(rng), C.byref(nppr), fp(rel))
        rot_rows.append((len(a), rc, d.value, incr.value, rng.value, nppr.value))
        rel_all.append(rel)
    out["rot_angles"] = np.concatenate([np.radians(np.array(s, dtype=np.float64)).astype(np.float32) for s in seqs])
    out["rot_results"] = np.array(rot_rows, dtype=np.float64)
    out["rot_rel"] = np.concatenate(rel_all)

    # Parker tables of fan-beam scans (arc and line detectors)
    pk_cases, pk_vals = [], []
    nc, nv = 48, 120
    for arc, width in [(1, 0.0017922 * 10), (0, 2.0 * 10)]:
        for start, rng_deg, rot_dir in [(0, 360, 1), (90, 360, 1), (45, 250, 1), (270, 200, -1), (180, 250, -1),
                                        (0, 215, 1)]:
            src, row = fan_views(nv, math.radians(start), math.radians(rng_deg), rot_dir, 500.0)
            w = np.zeros(nv * nc, np.float32)
            lib.ref_parker_table(arc, nc, width, nv, fp(np.ascontiguousarray(src)), fp(np.ascontiguousarray(row)),
                                 (nc - 1) / 2.0, 1000.0, fp(w))
            pk_cases.append((arc, nc, width, nv, start, rng_deg, rot_dir))
            pk_vals.append(w)
    out["parker_cases"] = np.array(pk_cases, dtype=np.float64)
    out["parker_values"] = np.concatenate(pk_vals)

    # per-view cosine weight, projMapping and weight at random points, all seven kinds
    recs, ev = [], []
    for kind in range(7):
        for _ in range(60):
            th = rs.uniform(0, 2 * math.pi)
            phi = th * rs.choice([-1, 1])
            sid, sdd = rs.uniform(400, 800), rs.uniform(900, 1500)
            r = np.zeros(17, np.float32)
            r[0] = th
            r[1], r[2] = rs.uniform(100, 400), rs.uniform(50, 200)
            r[3], r[4] = sdd, sid
            r[5:8] = [sid * math.cos(phi), sid * math.sin(phi), rs.uniform(-5, 5) if kind >= 5 else 0.0]
            r[8:11] = [-math.sin(phi), math.cos(phi), 0.0]
            r[11:14] = [0.0, 0.0, -1.0]
            r[14:17] = [-math.cos(phi), -math.sin(phi), 0.0]
            du = {0: 0.9, 1: 0.0018, 2: 1.2, 3: 0.9, 4: 0.9, 5: 0.0018, 6: 0.4}[kind]
            dv = 1.14
            col, row = rs.randint(0, 512), rs.randint(0, 256)
            x, y, z = rs.uniform(-120, 120, 3)
            cw, u, t = C.c_float(), C.c_float(), C.c_float()
            w = lib.ref_view_eval(kind, fp(r), du, dv, col, row, x, y, z, C.byref(cw), C.byref(u), C.byref(t))
            recs.append(np.concatenate([[kind, du, dv, col, row, x, y, z], r]))
            ev.append((cw.value, u.value, t.value, w))
    out["view_inputs"] = np.array(recs, dtype=np.float64)
    out["view_outputs"] = np.array(ev, dtype=np.float64)

    # voxel positions
    vp_in, vp_out = [], []
    for case in [(256, 256, 256, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0, 0, 0), (1025, 513, 11, 1.0, 2.0, 4.0, 1.0, 2.0, 3.0, 0, 0, 0),
                 (512, 512, 512, 0.5, 0.5, 0.5, 0.0, 0.0, 0.0, 511, 17, 300), (37, 41, 7, 1.3, 0.7, 2.1, 3.0, -2.0, 1.5, 5, 40, 6)]:
        o = np.zeros(3, np.float32)
        lib.ref_vox_pos(*case, fp(o))
        vp_in.append(case)
        vp_out.append(o)
    out["vox_inputs"] = np.array(vp_in, dtype=np.float64)
    out["vox_outputs"] = np.array(vp_out, dtype=np.float64)

    np.savez_compressed(OUT, **out)
    print(OUT, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
