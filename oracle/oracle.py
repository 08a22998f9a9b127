"""ctypes wrapper of the FP64 CPU oracle (fdk_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker for tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg. It depends on numpy and the C oracle only, not on the gct_b200 package.

Geometry is passed as (kind, detector samplers, per-view records). The per-view record layout is
the 17 doubles of the reference's ProjGeom fields: rot_ang, det_row_center, det_col_center,
src_det_dist, src_iso_dist, src_pos[3], det_row_dir[3], det_col_dir[3], iso_ray_dir[3].
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "fdk_oracle.c"
LIB = HERE / "_build" / "liboracle.so"

VIEW_DTYPE = np.dtype([
    ("rot_ang", "<f8"), ("det_row_center", "<f8"), ("det_col_center", "<f8"),
    ("src_det_dist", "<f8"), ("src_iso_dist", "<f8"), ("src_pos", "<f8", 3),
    ("det_row_dir", "<f8", 3), ("det_col_dir", "<f8", 3), ("iso_ray_dir", "<f8", 3),
])

# lerp_bits=8 emulates the texture unit's linear filter as measured through the reference's own
# texture objects (tests/golden/tex_probe.npz): sample positions snap to the nearest 1/256 texel
# and the bilinear corner weight a b to the nearest 1/256; ref_fdk --bp texture is the same rule.

KIND = {"parallel_1d": 0, "fan_arc": 1, "fan_line": 2, "parallel_2d": 3, "cone_parallel": 4,
        "cone_cyl": 5, "cone_flat": 6}


class _Geom(C.Structure):
    _fields_ = [("kind", C.c_int), ("nc", C.c_uint), ("du", C.c_double), ("nr", C.c_uint),
                ("dv", C.c_double), ("nv", C.c_uint), ("views", C.c_void_p)]


class _Vol(C.Structure):
    _fields_ = [("nx", C.c_uint), ("ny", C.c_uint), ("nz", C.c_uint), ("dx", C.c_double),
                ("dy", C.c_double), ("dz", C.c_double), ("mx", C.c_double), ("my", C.c_double),
                ("mz", C.c_double)]


_lib = None
_lock = threading.Lock()


def build(force: bool = False) -> Path:
    """Compile the oracle with gcc into oracle/_build/liboracle.so."""
    LIB.parent.mkdir(exist_ok=True)
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        tmp = LIB.with_suffix(".so.tmp")
        subprocess.run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-pthread", str(SRC), "-o", str(tmp), "-lm"],
                       check=True)
        os.replace(tmp, LIB)
    return LIB


def load() -> C.CDLL:
    global _lib
    with _lock:
        if _lib is None:
            if not LIB.exists():
                build()
            lib = C.CDLL(str(LIB))
            vp, dp = C.c_void_p, C.POINTER(C.c_double)
            lib.or_make_view.argtypes = [C.c_int, dp, C.c_uint, vp]
            lib.or_rotation.argtypes = [C.POINTER(_Geom), C.POINTER(C.c_int), dp, dp, C.POINTER(C.c_uint), dp, dp]
            lib.or_rot_dir.argtypes = [dp, C.c_uint]
            lib.or_ramp_taps.argtypes = [C.c_int, C.c_uint, C.c_double, C.c_double, C.c_int, dp]
            lib.or_ramp_taps.restype = None
            lib.or_cos_weight.argtypes = [C.POINTER(_Geom), C.c_uint, C.c_uint, C.c_uint]
            lib.or_cos_weight.restype = C.c_double
            lib.or_parker.argtypes = [C.POINTER(_Geom), dp]
            lib.or_filter.argtypes = [C.POINTER(_Geom), vp, C.c_double, C.c_int, C.c_int, dp, C.c_int]
            lib.or_filter_np.argtypes = [C.POINTER(_Geom), vp, C.c_double, C.c_int, C.c_int, dp, C.c_int]
            lib.or_backproject.argtypes = [C.POINTER(_Geom), C.POINTER(_Vol), dp, vp, C.c_long, C.c_int, dp, C.c_int]
            lib.or_fdk.argtypes = [C.POINTER(_Geom), C.POINTER(_Vol), vp, C.c_double, C.c_int, C.c_int, vp,
                                   C.c_long, C.c_int, dp, C.c_int]
            lib.or_proj_mapping.argtypes = [C.POINTER(_Geom), C.c_uint, dp, dp, dp]
            lib.or_proj_mapping.restype = C.c_double
            lib.or_phantom.argtypes = [C.POINTER(_Geom), dp, C.c_uint, dp]
            lib.or_phantom.restype = None
            lib.or_tex_fetch.argtypes = [dp, C.c_uint, C.c_uint, C.c_double, C.c_double, C.c_int]
            lib.or_tex_fetch.restype = C.c_double
            lib.or_gauss_project.argtypes = [C.POINTER(_Geom), dp, C.c_uint, dp]
            lib.or_gauss_project.restype = None
            _lib = lib
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class Geometry:
    kind: int
    nc: int
    du: float
    views: np.ndarray          # VIEW_DTYPE records
    nr: int = 1
    dv: float = 1.0

    def __post_init__(self):
        self.views = np.ascontiguousarray(self.views, dtype=VIEW_DTYPE)
        self._s = _Geom(self.kind, self.nc, self.du, self.nr if self.kind >= 3 else 1,
                        self.dv if self.kind >= 3 else 1.0, len(self.views), self.views.ctypes.data)

    @property
    def nv(self) -> int:
        return len(self.views)

    @property
    def shape(self) -> tuple:
        return (self.nv, self.nr if self.kind >= 3 else 1, self.nc)


@dataclass
class Volume:
    nx: int
    ny: int
    nz: int = 1
    dx: float = 1.0
    dy: float = 1.0
    dz: float = 1.0
    mid: tuple = (0.0, 0.0, 0.0)

    def struct(self) -> _Vol:
        return _Vol(self.nx, self.ny, self.nz, self.dx, self.dy, self.dz, *self.mid)

    @property
    def shape(self) -> tuple:
        return (self.nz, self.ny, self.nx)


def make_views(kind: int, n: int, det_row_center: float, det_col_center: float = 0.0,
               src_det_dist: float = 0.0, src_iso_dist: float = 0.0, rot_dir: int = 1,
               init_ang: float = 0.0, ang_incr: float = 0.0, hel_pitch: float = 0.0) -> np.ndarray:
    p = np.array([det_row_center, det_col_center, src_det_dist, src_iso_dist, rot_dir, init_ang, ang_incr,
                  hel_pitch], dtype=np.float64)
    out = np.zeros(n, dtype=VIEW_DTYPE)
    lib = load()
    for i in range(n):
        lib.or_make_view(kind, _dp(p), i, out[i:i + 1].ctypes.data)
    return out


def rotation(g: Geometry):
    """(dir, incr, range, num_proj_per_rot, rot_ang, rel_rot_ang) or None."""
    d, n = C.c_int(0), C.c_uint(0)
    incr, rng = C.c_double(0), C.c_double(0)
    rot = np.zeros(g.nv)
    rel = np.zeros(g.nv)
    rc = load().or_rotation(C.byref(g._s), C.byref(d), C.byref(incr), C.byref(rng), C.byref(n), _dp(rot), _dp(rel))
    if rc != 0:
        return None
    return d.value, incr.value, rng.value, n.value, rot, rel


def rot_dir(angles) -> int:
    a = np.ascontiguousarray(angles, dtype=np.float64)
    return load().or_rot_dir(_dp(a), len(a))


def ramp_taps(kind: int, n: int, width: float, cut_off: float = 1.0, apod: int = 0) -> np.ndarray:
    t = np.zeros(n)
    load().or_ramp_taps(kind, n, width, cut_off, apod, _dp(t))
    return t


def parker(g: Geometry) -> np.ndarray:
    w = np.zeros((g.nv, g.nc))
    if load().or_parker(C.byref(g._s), _dp(w)) != 0:
        raise ValueError("invalid trajectory")
    return w


def cos_weight(g: Geometry, v: int, r: int, c: int) -> float:
    return load().or_cos_weight(C.byref(g._s), v, r, c)


def filter_stack(g: Geometry, proj: np.ndarray, cut_off: float = 1.0, apod: int = 0, use_fft: bool = False,
                 threads: int | None = None, parker: bool = True) -> np.ndarray:
    p = np.ascontiguousarray(proj, dtype=np.float32).reshape(g.shape)
    out = np.zeros(g.shape)
    fn = load().or_filter if parker else load().or_filter_np
    rc = fn(C.byref(g._s), p.ctypes.data, cut_off, apod, int(use_fft), _dp(out), threads or os.cpu_count())
    if rc != 0:
        raise ValueError("invalid trajectory")
    return out


def backproject(g: Geometry, vol: Volume, filtered: np.ndarray, lerp_bits: int = 0,
                threads: int | None = None) -> np.ndarray:
    f = np.ascontiguousarray(filtered, dtype=np.float64).reshape(g.shape)
    out = np.zeros(vol.shape)
    load().or_backproject(C.byref(g._s), C.byref(vol.struct()), _dp(f), None, 0, lerp_bits, _dp(out),
                          threads or os.cpu_count())
    return out


def fdk(g: Geometry, vol: Volume, proj: np.ndarray, voxels: np.ndarray | None = None, cut_off: float = 1.0,
        apod: int = 0, lerp_bits: int = 0, use_fft: bool | None = None, threads: int | None = None) -> np.ndarray:
    """FP64 FDK of the whole grid ([z][y][x]) or of the listed (i, j, k) voxels (1D result)."""
    p = np.ascontiguousarray(proj, dtype=np.float32).reshape(g.shape)
    if use_fft is None:
        use_fft = g.nc > 256
    if voxels is None:
        out = np.zeros(vol.shape)
        vp, n = None, 0
    else:
        vox = np.ascontiguousarray(voxels, dtype=np.uint32).reshape(-1, 3)
        out = np.zeros(len(vox))
        vp, n = vox.ctypes.data, len(vox)
    rc = load().or_fdk(C.byref(g._s), C.byref(vol.struct()), p.ctypes.data, cut_off, apod, int(use_fft), vp, n,
                       lerp_bits, _dp(out), threads or os.cpu_count())
    if rc != 0:
        raise ValueError("oracle FDK failed (invalid trajectory or allocation)")
    return out


def spiral_windows(g: Geometry, vol: Volume) -> list:
    """Per z slice, the views [first, last) the spiral FDK backprojects, or None for a slice it
    leaves zero. Restates src/cpp/geom/spiral_ct_geom.h:57-75 (firstAndLastProjIndices: the view
    whose source z is nearest the slice, the first of equals, and the num_proj_per_rot views
    starting num_proj_per_rot / 2 before it) and src/cuda/recon/fdk_spiral.cuh:60-79 (a slice
    is reconstructed only when first > 0 and last < num_views; the reference's unsigned first
    index wraps below zero, which also leaves the slice zero)."""
    rot = rotation(g)
    if rot is None or rot[3] == 0:
        raise ValueError("invalid spiral trajectory")
    npr = rot[3]
    z = np.array([v["src_pos"][2] for v in g.views], dtype=np.float64)
    z0 = vol.mid[2] - (vol.nz - 1) * vol.dz / 2.0
    out = []
    for k in range(vol.nz):
        mid = int(np.argmin(np.abs(z - (z0 + k * vol.dz))))
        first = mid - npr // 2
        last = first + npr
        out.append((first, last) if (first > 0 and last < g.nv) else None)
    return out


def fdk_spiral(g: Geometry, vol: Volume, proj: np.ndarray, cut_off: float = 1.0, apod: int = 0,
               threads: int | None = None) -> np.ndarray:
    """FP64 spiral FDK ([z][y][x]): cosine weights and the ramp filter on every view (no Parker
    weights), then per slice the backprojection of its window of views with the final angular
    increment scale (src/cuda/recon/fdk_spiral.cuh:33-94)."""
    filt = filter_stack(g, proj, cut_off, apod, use_fft=g.nc > 256, threads=threads, parker=False)
    out = np.zeros(vol.shape)
    z0 = vol.mid[2] - (vol.nz - 1) * vol.dz / 2.0
    for k, w in enumerate(spiral_windows(g, vol)):
        if w is None:
            continue
        first, last = w
        gs = Geometry(g.kind, g.nc, g.du, g.views[first:last], g.nr, g.dv)
        vs = Volume(vol.nx, vol.ny, 1, vol.dx, vol.dy, vol.dz, (vol.mid[0], vol.mid[1], z0 + k * vol.dz))
        out[k] = backproject(gs, vs, filt[first:last], threads=threads)[0]
    return out


def proj_mapping(g: Geometry, v: int, X) -> tuple:
    """(u, t, weight): detector coordinates (mm or rad, before pixel conversion) of point X."""
    x = np.ascontiguousarray(list(X) + [0.0] * (3 - len(X)), dtype=np.float64)
    u, t = C.c_double(0), C.c_double(0)
    w = load().or_proj_mapping(C.byref(g._s), v, _dp(x), C.byref(u), C.byref(t))
    return u.value, t.value, w


def phantom(g: Geometry, ellipsoids) -> np.ndarray:
    e = np.ascontiguousarray(np.asarray(ellipsoids, dtype=np.float64).reshape(-1, 8))
    out = np.zeros(g.shape)
    load().or_phantom(C.byref(g._s), _dp(e), len(e), _dp(out))
    return out


def gauss_project(g: Geometry, blobs) -> np.ndarray:
    """Exact line integrals of isotropic Gaussian blobs (cx, cy, cz, sigma, amplitude)."""
    b = np.ascontiguousarray(np.asarray(blobs, dtype=np.float64).reshape(-1, 5))
    out = np.zeros(g.shape)
    load().or_gauss_project(C.byref(g._s), _dp(b), len(b), _dp(out))
    return out


def gauss_volume(vol: Volume, blobs, planar: bool = False) -> np.ndarray:
    """The blobs' density sampled at the voxel centres ([z][y][x]); planar: the z = 0 plane."""
    b = np.asarray(blobs, dtype=np.float64).reshape(-1, 5)
    x = vol.mid[0] - (vol.nx - 1) * vol.dx / 2.0 + np.arange(vol.nx) * vol.dx
    y = vol.mid[1] - (vol.ny - 1) * vol.dy / 2.0 + np.arange(vol.ny) * vol.dy
    z = np.zeros(1) if planar else vol.mid[2] - (vol.nz - 1) * vol.dz / 2.0 + np.arange(vol.nz) * vol.dz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    out = np.zeros(Z.shape)
    for cx, cy, cz, s, a in b:
        r2 = (X - cx) ** 2 + (Y - cy) ** 2 + (0.0 if planar else (Z - cz) ** 2)
        out += a * np.exp(-r2 / (2.0 * s * s))
    return out


def tex_fetch(texels: np.ndarray, xy: np.ndarray, lerp_bits: int = 8) -> np.ndarray:
    """The oracle's bilinear fetch of texels [h][w] at texture coordinates xy (n x 2, texel
    centres at integer + 0.5), border 0; lerp_bits=8 is the texture unit's rule."""
    t = np.ascontiguousarray(texels, dtype=np.float64)
    h, w = t.shape
    lib = load()
    return np.array([lib.or_tex_fetch(_dp(t), w, h, float(x), float(y), lerp_bits) for x, y in np.asarray(xy)])
