"""GCT geometry types over the C ABI (host, FP64).

Mirrors the reference's geometry API so that callers of GCT find the same objects:

* detectors ``DetParallel``, ``DetFanArc``, ``DetFanLine`` (src/cpp/geom/detector_1d.h:10-25)
* circular-trajectory parameters (src/cpp/io/parameters/proj_geom_params.h:16-58)
* ``ProjGeomFactory(DetRow[, DetCol]).create(params, proj_idx)``
  (src/cpp/io/geom_reader/proj_geom_factory_params.cpp:8-108)
* ``AxialCTGeom(det_geom, proj_geom)`` with its ``RotationGeom`` (src/cpp/geom/ct_geom.h:18-53,
  src/cpp/geom/rotation_geom.h:16-115)
* ``ReconImgGeom``, ``ProjectionStack``, ``ReconImg`` (src/cpp/geom/recon_img_geom.h:15-90,
  src/cpp/data/projection_stack.h:12-36, src/cpp/data/recon_img.h:20-61)
* ``is_valid_axial_recon`` (src/cpp/recon/check_validity.h:66-75)

Unlike the reference (FP32 throughout), every geometric quantity is kept in double precision.
"""
from __future__ import annotations

import ctypes as C
import enum
import math
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import _lib


class RotDir(enum.IntEnum):
    CCW = -1
    CW = 1


class ApodFunc(enum.IntEnum):
    NONE = 0
    HANN = 1
    HAMMING = 2


class GeomKind(enum.IntEnum):
    PARALLEL_1D = 0
    FAN_ARC = 1
    FAN_LINE = 2
    PARALLEL_2D = 3
    CONE_PARALLEL = 4
    CONE_CYL = 5
    CONE_FLAT = 6


@dataclass(frozen=True)
class _Det:
    num_samples: int
    sampling_width: float


class DetParallel(_Det):
    """1D detector for parallel-beam projection; sampling width in mm."""


class DetFanArc(_Det):
    """1D arc-shaped detector for fan-beam projection; sampling width in radians."""


class DetFanLine(_Det):
    """1D line-shaped detector for fan-beam projection; sampling width in mm."""


_KIND_OF = {
    (DetParallel,): GeomKind.PARALLEL_1D,
    (DetFanArc,): GeomKind.FAN_ARC,
    (DetFanLine,): GeomKind.FAN_LINE,
    (DetParallel, DetParallel): GeomKind.PARALLEL_2D,
    (DetParallel, DetFanLine): GeomKind.CONE_PARALLEL,
    (DetFanArc, DetFanLine): GeomKind.CONE_CYL,
    (DetFanLine, DetFanLine): GeomKind.CONE_FLAT,
}


def kind_of(det_types: Sequence[type]) -> GeomKind:
    """Geometry kind of a (DetRow[, DetCol]) type pair; only the seven reference overloads exist."""
    key = tuple(det_types)
    if key not in _KIND_OF:
        names = ", ".join(t.__name__ for t in key)
        raise TypeError(f"no axial reconstruction for detector configuration <{names}>")
    return _KIND_OF[key]


@dataclass
class RotationParams:
    dir: RotDir = RotDir.CW
    init_ang: float = 0.0
    ang_incr: float = 0.0
    num_proj: int = 0
    hel_pitch: float = 0.0


@dataclass
class Parallel1DProjGeomParams:
    det_row_center: float = 0.0
    rot: RotationParams = field(default_factory=RotationParams)


@dataclass
class FanBeamProjGeomParams:
    det_row_center: float = 0.0
    rot: RotationParams = field(default_factory=RotationParams)
    src_det_dist: float = 0.0
    src_iso_dist: float = 0.0


@dataclass
class Parallel2DProjGeomParams:
    det_row_center: float = 0.0
    rot: RotationParams = field(default_factory=RotationParams)
    det_col_center: float = 0.0


@dataclass
class ConeBeamProjGeomParams:
    det_row_center: float = 0.0
    rot: RotationParams = field(default_factory=RotationParams)
    src_det_dist: float = 0.0
    src_iso_dist: float = 0.0
    det_col_center: float = 0.0


# numpy mirror of gct_view_geom (one record per view)
VIEW_DTYPE = np.dtype([
    ("rot_ang", "<f8"), ("det_row_center", "<f8"), ("det_col_center", "<f8"),
    ("src_det_dist", "<f8"), ("src_iso_dist", "<f8"), ("src_pos", "<f8", 3),
    ("det_row_dir", "<f8", 3), ("det_col_dir", "<f8", 3), ("iso_ray_dir", "<f8", 3),
])
assert VIEW_DTYPE.itemsize == C.sizeof(_lib.gct_view_geom)


@dataclass
class ProjGeom:
    """Per-view projection geometry: union of the reference's ProjGeom<...> fields."""
    rot_ang: float = 0.0
    det_row_center: float = 0.0
    det_col_center: float = 0.0
    src_det_dist: float = 0.0
    src_iso_dist: float = 0.0
    src_pos: tuple = (0.0, 0.0, 0.0)
    det_row_dir: tuple = (0.0, 0.0, 0.0)
    det_col_dir: tuple = (0.0, 0.0, 0.0)
    iso_ray_dir: tuple = (0.0, 0.0, 0.0)

    def to_record(self):
        rec = np.zeros((), dtype=VIEW_DTYPE)
        for name in VIEW_DTYPE.names:
            rec[name] = getattr(self, name)
        return rec

    @classmethod
    def from_record(cls, rec) -> "ProjGeom":
        vals = {}
        for name in VIEW_DTYPE.names:
            v = rec[name]
            vals[name] = tuple(float(x) for x in v) if np.ndim(v) else float(v)
        return cls(**vals)


def _params_struct(params) -> _lib.gct_geom_params:
    p = _lib.gct_geom_params()
    p.det_row_center = float(params.det_row_center)
    p.det_col_center = float(getattr(params, "det_col_center", 0.0))
    p.src_det_dist = float(getattr(params, "src_det_dist", 0.0))
    p.src_iso_dist = float(getattr(params, "src_iso_dist", 0.0))
    p.rot_dir = int(params.rot.dir)
    p.init_ang = float(params.rot.init_ang)
    p.ang_incr = float(params.rot.ang_incr)
    p.num_proj = int(params.rot.num_proj)
    p.hel_pitch = float(params.rot.hel_pitch)
    return p


class ProjectionMatrix:
    """GCT::Geom::ProjectionMatrix (src/cpp/geom/projection_matrix.{h,cpp}) in FP64: a 3 x 4
    flat-panel projection matrix with its intrinsic matrix K (upper triangular, positive diagonal,
    K[2][2] = 1), rotation R (rows: detector row direction, column direction, their cross product)
    and source position."""

    def __init__(self, matrix):
        m = np.ascontiguousarray(np.asarray(matrix, dtype=np.float64).reshape(12))
        out = _lib.gct_proj_matrix()
        _lib.check(_lib.load().gct_proj_matrix_decompose(m.ctypes.data_as(C.POINTER(C.c_double)), C.byref(out)))
        self._set(out)

    def _set(self, s: _lib.gct_proj_matrix) -> None:
        self._matrix = np.array(s.matrix[:], dtype=np.float64).reshape(3, 4)
        self._k = np.array(s.intrinsic[:], dtype=np.float64).reshape(3, 3)
        self._r = np.array(s.rotation[:], dtype=np.float64).reshape(3, 3)
        self._src = np.array(s.src_pos[:], dtype=np.float64)

    @classmethod
    def compose(cls, pg: ProjGeom, pix_width_mm: float, pix_height_mm: float) -> "ProjectionMatrix":
        """ProjectionMatrix(ProjGeom<DetFanLine, DetFanLine>, pix_width_mm, pix_height_mm)."""
        v = _lib.gct_view_geom.from_buffer_copy(pg.to_record().tobytes())
        out = _lib.gct_proj_matrix()
        _lib.check(_lib.load().gct_proj_matrix_compose(C.byref(v), float(pix_width_mm), float(pix_height_mm),
                                                       C.byref(out)))
        obj = cls.__new__(cls)
        obj._set(out)
        return obj

    def matrix(self) -> np.ndarray:
        return self._matrix.copy()

    def intrinsic_matrix(self) -> np.ndarray:
        return self._k.copy()

    def rotation_matrix(self) -> np.ndarray:
        return self._r.copy()

    def src_pos(self) -> np.ndarray:
        return self._src.copy()

    def principal_point_det_row(self) -> float:
        return float(self._k[0, 2])

    def principal_point_det_col(self) -> float:
        return float(self._k[1, 2])

    def focal_length_det_row(self) -> float:
        """Source-detector distance in detector-row pixels."""
        return float(self._k[0, 0])


class ProjGeomFactory:
    """``ProjGeomFactory(DetRow[, DetCol]).create(params, proj_idx)``, and for flat panels
    ``create(ProjectionMatrix)`` (src/cpp/io/geom_reader/proj_geom_factory_proj_mat.cpp:7-26)."""

    def __init__(self, *det_types: type):
        self.kind = kind_of(det_types)

    def create(self, params, proj_idx: int | None = None) -> ProjGeom:
        out = _lib.gct_view_geom()
        lib = _lib.load()
        if isinstance(params, ProjectionMatrix):
            if self.kind != GeomKind.CONE_FLAT:
                raise TypeError("projection matrices describe flat-panel (DetFanLine, DetFanLine) views")
            m = np.ascontiguousarray(params.matrix().reshape(12))
            _lib.check(lib.gct_proj_geom_from_matrix(m.ctypes.data_as(C.POINTER(C.c_double)), C.byref(out)))
        else:
            _lib.check(lib.gct_proj_geom_create(int(self.kind), C.byref(_params_struct(params)),
                                                int(proj_idx), C.byref(out)))
        rec = np.frombuffer(bytearray(out), dtype=VIEW_DTYPE)[0]
        return ProjGeom.from_record(rec)

    def create_all(self, params) -> np.ndarray:
        """All ``params.rot.num_proj`` views as a VIEW_DTYPE array."""
        n = int(params.rot.num_proj)
        arr = np.zeros(n, dtype=VIEW_DTYPE)
        ps = _params_struct(params)
        lib = _lib.load()
        buf = (_lib.gct_view_geom * max(n, 1))()
        for i in range(n):
            _lib.check(lib.gct_proj_geom_create(int(self.kind), C.byref(ps), i, C.byref(buf[i])))
        if n:
            arr[:] = np.frombuffer(bytearray(buf), dtype=VIEW_DTYPE)[:n]
        return arr


@dataclass
class RotationGeom:
    dir: RotDir
    rot_ang_incr: float
    rot_ang_range: float
    num_proj_per_rot: int
    rot_ang: np.ndarray
    rel_rot_ang: np.ndarray


class AxialCTGeom:
    """Geometry of an axial CT scan: detector tuple + per-view projection geometry.

    ``det_geom`` is a tuple ``(DetRow,)`` or ``(DetRow, DetCol)`` of detector instances;
    ``proj_geom`` is a sequence of ``ProjGeom`` or a ``VIEW_DTYPE`` array. Raises
    ``GctError`` ("Invalid X-ray source trajectory.") like the reference's constructor.
    """

    def __init__(self, det_geom: tuple, proj_geom):
        self._det = tuple(det_geom)
        self.kind = kind_of(type(d) for d in self._det)
        if isinstance(proj_geom, np.ndarray) and proj_geom.dtype == VIEW_DTYPE:
            self._views = np.ascontiguousarray(proj_geom)
        else:
            self._views = np.array([pg.to_record() for pg in proj_geom], dtype=VIEW_DTYPE)
        self._struct = self._make_struct()
        self._rot = self._rotation()

    @classmethod
    def from_params(cls, det_geom: tuple, params) -> "AxialCTGeom":
        views = ProjGeomFactory(*(type(d) for d in det_geom)).create_all(params)
        return cls(det_geom, views)

    def _make_struct(self) -> _lib.gct_ct_geom:
        g = _lib.gct_ct_geom()
        g.kind = int(self.kind)
        g.det_row = _lib.gct_detector(self._det[0].num_samples, self._det[0].sampling_width)
        if len(self._det) > 1:
            g.det_col = _lib.gct_detector(self._det[1].num_samples, self._det[1].sampling_width)
        else:
            g.det_col = _lib.gct_detector(1, 1.0)
        g.num_views = len(self._views)
        g.views = self._views.ctypes.data_as(C.POINTER(_lib.gct_view_geom))
        return g

    def _rotation(self) -> RotationGeom:
        n = len(self._views)
        rot = np.zeros(max(n, 1))
        rel = np.zeros(max(n, 1))
        out = _lib.gct_rotation_geom()
        dp = C.POINTER(C.c_double)
        _lib.check(_lib.load().gct_rotation_geom_get(C.byref(self._struct), C.byref(out),
                                                     rot.ctypes.data_as(dp), rel.ctypes.data_as(dp)))
        return RotationGeom(RotDir(out.dir), out.rot_ang_incr, out.rot_ang_range, out.num_proj_per_rot,
                            rot[:n], rel[:n])

    def det_geom(self) -> tuple:
        return self._det

    def proj_geom(self) -> list[ProjGeom]:
        return [ProjGeom.from_record(r) for r in self._views]

    @property
    def views(self) -> np.ndarray:
        return self._views

    def rotation_geom(self) -> RotationGeom:
        return self._rot

    @property
    def num_views(self) -> int:
        return len(self._views)

    @property
    def num_cols(self) -> int:
        return self._det[0].num_samples

    @property
    def num_rows(self) -> int:
        return self._det[1].num_samples if len(self._det) > 1 else 1

    @property
    def is_3d(self) -> bool:
        return len(self._det) > 1

    def struct(self) -> _lib.gct_ct_geom:
        return self._struct


CTGeom = AxialCTGeom


class SpiralCTGeom(AxialCTGeom):
    """Geometry of a spiral (helical) cone-beam scan: GCT::Geom::SpiralCTGeom
    (src/cpp/geom/spiral_ct_geom.h:9-95). The constructor checks what the reference's does
    (projections per rotation > 0, source z sorted either way, positive pitch)."""

    def __init__(self, det_geom: tuple, proj_geom):
        super().__init__(det_geom, proj_geom)
        npr, pitch = C.c_uint32(0), C.c_double(0.0)
        _lib.check(_lib.load().gct_spiral_geom_check(C.byref(self.struct()), C.byref(npr), C.byref(pitch)))
        self.num_proj_per_rot = int(npr.value)
        self.spiral_pitch = float(pitch.value)  # source z travel per radian (mm)

    def first_and_last_proj_indices(self, slice_pos_mm: float) -> tuple:
        """[first, last) of the rotation of views centred on the view nearest the slice (first may
        be negative where the reference's unsigned index wraps)."""
        f, l = C.c_int64(0), C.c_int64(0)
        _lib.check(_lib.load().gct_spiral_proj_indices(C.byref(self.struct()), float(slice_pos_mm), C.byref(f),
                                                       C.byref(l)))
        return int(f.value), int(l.value)


@dataclass(frozen=True)
class EqDistSampler:
    num_samples: int
    sampling_width: float


@dataclass
class ReconImgGeom:
    """Reconstruction grid: x, y (, z) samplers and the mid point (mm)."""
    x: EqDistSampler
    y: EqDistSampler
    z: EqDistSampler | None = None
    mid_point: tuple = (0.0, 0.0, 0.0)

    @property
    def dim(self) -> int:
        return 3 if self.z is not None else 2

    @property
    def shape(self) -> tuple:
        """Array shape in [z][y][x] order (z omitted for 2D)."""
        if self.z is None:
            return (self.y.num_samples, self.x.num_samples)
        return (self.z.num_samples, self.y.num_samples, self.x.num_samples)

    def struct(self) -> _lib.gct_vol_geom:
        v = _lib.gct_vol_geom()
        v.nx, v.ny = self.x.num_samples, self.y.num_samples
        v.dx, v.dy = self.x.sampling_width, self.y.sampling_width
        if self.z is None:
            v.nz, v.dz = 1, 1.0
        else:
            v.nz, v.dz = self.z.num_samples, self.z.sampling_width
        mp = tuple(self.mid_point) + (0.0,) * (3 - len(self.mid_point))
        v.mid = (C.c_double * 3)(*mp)
        return v

    def first_voxel_pos(self) -> tuple:
        """Centre of voxel (0, 0[, 0]) (src/cpp/geom/recon_img_geom.h:72-90)."""
        s = [self.x, self.y] + ([self.z] if self.z is not None else [])
        return tuple(self.mid_point[i] - (s[i].num_samples - 1) * s[i].sampling_width / 2.0
                     for i in range(len(s)))


class ProjectionStack:
    """Stack of 1D or 2D projections, float32 [view][row][col] (1D: [view][col])."""

    def __init__(self, num_cols: int, num_proj: int, num_rows: int | None = None, data=None):
        if num_cols == 0 or num_proj == 0 or num_rows == 0:
            raise ValueError("Projections size or number of projections cannot be zero.")
        self.num_cols, self.num_rows, self.num_proj = num_cols, num_rows, num_proj
        shape = (num_proj, num_cols) if num_rows is None else (num_proj, num_rows, num_cols)
        if data is None:
            self.elements = np.zeros(shape, dtype=np.float32)
        else:
            self.elements = np.ascontiguousarray(np.asarray(data, dtype=np.float32).reshape(shape))

    @property
    def dim(self) -> int:
        return 1 if self.num_rows is None else 2


class ReconImg:
    """2D or 3D reconstructed image, float32 [z][y][x] (2D: [y][x])."""

    def __init__(self, geom: ReconImgGeom):
        if any(s.num_samples == 0 for s in [geom.x, geom.y] + ([geom.z] if geom.z else [])):
            raise ValueError("The number of samples in any dimension cannot be zero.")
        if any(s.sampling_width <= 0 for s in [geom.x, geom.y] + ([geom.z] if geom.z else [])):
            raise ValueError("The sampling width of the image in any dimension cannot be zero or negative.")
        self.geom = geom
        self.elements = np.zeros(geom.shape, dtype=np.float32)


def is_valid_axial_recon(cg: AxialCTGeom, proj: ProjectionStack, verbose: bool = False) -> bool:
    valid = C.c_int32(0)
    rows = proj.num_rows if proj.num_rows is not None else 1
    _lib.check(_lib.load().gct_is_valid_axial_recon(C.byref(cg.struct()), proj.num_cols, rows,
                                                    proj.num_proj, int(verbose), C.byref(valid)))
    return bool(valid.value)


def ramp_filter_taps(kind: GeomKind, det_row, cut_off_freq: float = 1.0,
                     apod_func: ApodFunc = ApodFunc.NONE) -> np.ndarray:
    taps = np.zeros(det_row.num_samples)
    fp = _lib.gct_filt_params(cut_off_freq, int(apod_func))
    d = _lib.gct_detector(det_row.num_samples, det_row.sampling_width)
    _lib.check(_lib.load().gct_ramp_filter_taps(int(kind), C.byref(d), C.byref(fp),
                                                taps.ctypes.data_as(C.POINTER(C.c_double))))
    return taps


def parker_weights(cg: AxialCTGeom) -> np.ndarray:
    """Redundancy weights [view][col] (getParkerWeights)."""
    w = np.zeros((cg.num_views, cg.num_cols), dtype=np.float32)
    _lib.check(_lib.load().gct_parker_weights(C.byref(cg.struct()), w.ctypes.data_as(C.POINTER(C.c_float))))
    return w


def map_point(cg: AxialCTGeom, vol_geom: ReconImgGeom, view: int, ijk) -> tuple:
    """(xyz, col, row, weight) of fractional voxel index ``ijk`` in ``view``, evaluated on the host
    from the same per-view coefficients the backprojection kernels use."""
    dp = C.POINTER(C.c_double)
    idx = np.zeros(3)
    idx[:len(ijk)] = ijk
    xyz = np.zeros(3)
    col, row, w = C.c_double(), C.c_double(), C.c_double()
    _lib.check(_lib.load().gct_map_point(C.byref(cg.struct()), C.byref(vol_geom.struct()), int(view),
                                         idx.ctypes.data_as(dp), xyz.ctypes.data_as(dp), C.byref(col),
                                         C.byref(row), C.byref(w)))
    return xyz, col.value, row.value, w.value


def deg(x: float) -> float:
    return x * math.pi / 180.0
