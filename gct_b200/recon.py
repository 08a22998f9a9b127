"""FDK reconstruction over the C ABI.

``reconstruct(cg, proj, vol)`` is the drop-in for ``GCT::Recon::CUDA::reconstruct``
(src/cuda/recon/recon_wrappers.cuh:15-43): host arrays in, host array out, synchronous.

``FdkPlan`` is the device-resident form: geometry, filter spectrum and Parker table are built
once (FP64 on the host) and reused; ``execute`` runs on caller-owned CUDA buffers on a stream.
Torch tensors are accepted as device buffers (torch only provides memory and streams here; the
arithmetic is the library's CUDA kernels). There is no CPU fallback: without a CUDA device the
calls fail.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from dataclasses import dataclass

import numpy as np

from . import _lib
from .geometry import ApodFunc, AxialCTGeom, ProjectionStack, ReconImg, ReconImgGeom, SpiralCTGeom

FILTER_FFT = 0
FILTER_TOEPLITZ_BF16X3 = 1
FILTER_TOEPLITZ_BF16X4 = 2
FILTER_TOEPLITZ_F16X2 = 3
STORAGE_F32 = 0
STORAGE_F16 = 1
SYMMETRY_AUTO = 0
SYMMETRY_OFF = 1
SYMMETRY_ON = 2
SCAN_AXIAL = 0
SCAN_SPIRAL = 1


@dataclass
class FiltParams:
    """Ramp-filter parameters (src/cpp/io/parameters/filt_parameters.h:14-18)."""
    cut_off_freq: float = 1.0
    apod_func: ApodFunc = ApodFunc.NONE

    def struct(self) -> _lib.gct_filt_params:
        return _lib.gct_filt_params(float(self.cut_off_freq), int(self.apod_func))


@dataclass
class FdkOptions:
    filter: int = FILTER_FFT
    storage: int = STORAGE_F32
    z_per_thread: int = 0
    block_x: int = 0
    block_y: int = 0
    symmetry: int = SYMMETRY_AUTO
    scan: int = SCAN_AXIAL

    def struct(self) -> _lib.gct_fdk_opts:
        o = _lib.gct_fdk_opts()
        o.filter, o.storage, o.z_per_thread = self.filter, self.storage, self.z_per_thread
        o.block_x, o.block_y, o.symmetry, o.scan = self.block_x, self.block_y, self.symmetry, self.scan
        return o


def _ptr(x) -> int:
    """Device pointer of a torch tensor (or an int address)."""
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if not x.is_cuda:
            raise ValueError("expected a CUDA tensor")
        if not x.is_contiguous() or x.dtype.itemsize != 4:
            raise ValueError("expected a contiguous float32 CUDA tensor")
        return x.data_ptr()
    raise TypeError(f"unsupported buffer type {type(x)!r}")


def _ws(workspace):
    if workspace is None:
        return None
    return C.c_void_p(workspace.data_ptr() if hasattr(workspace, "data_ptr") else int(workspace))


def _stream(stream) -> int | None:
    if stream is None:
        try:
            import torch
            return torch.cuda.current_stream().cuda_stream
        except Exception:  # pragma: no cover - torch without CUDA
            return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def reconstruct(cg: AxialCTGeom, proj, vol, filt: FiltParams | None = None,
                opts: FdkOptions | None = None) -> None:
    """Host-to-host FDK: ``proj`` is a ProjectionStack (or float32 array [view][row][col]),
    ``vol`` a ReconImg whose ``elements`` receive the result. A SpiralCTGeom selects the spiral
    FDK (reconFDK(SpiralCTGeom), src/cuda/recon/fdk_spiral.cuh:33-94)."""
    pe = proj.elements if isinstance(proj, ProjectionStack) else np.ascontiguousarray(proj, dtype=np.float32)
    if not (pe.flags.c_contiguous and pe.dtype == np.float32):
        pe = np.ascontiguousarray(pe, dtype=np.float32)
    expect = cg.num_views * cg.num_rows * cg.num_cols
    if pe.size != expect:
        raise ValueError(f"projection stack has {pe.size} values, geometry needs {expect}")
    ve = vol.elements if isinstance(vol, ReconImg) else vol
    geom = vol.geom if isinstance(vol, ReconImg) else None
    if geom is None:
        raise TypeError("vol must be a ReconImg")
    fp = C.POINTER(C.c_float)
    lib = _lib.load()
    o = opts or FdkOptions()
    if isinstance(cg, SpiralCTGeom):
        o = dataclasses.replace(o, scan=SCAN_SPIRAL)
    _lib.check(lib.gct_reconstruct_ex(C.byref(cg.struct()), C.byref(geom.struct()),
                                      C.byref((filt or FiltParams()).struct()), C.byref(o.struct()),
                                      pe.ctypes.data_as(fp), ve.ctypes.data_as(fp)))


class FdkPlan:
    """Reusable device plan for one geometry / grid / option set."""

    def __init__(self, cg: AxialCTGeom, vol_geom: ReconImgGeom, filt: FiltParams | None = None,
                 opts: FdkOptions | None = None):
        self.cg = cg
        self.vol_geom = vol_geom
        self.opts = opts or FdkOptions()
        self._lib = _lib.load()
        self._handle = C.c_void_p()
        _lib.check(self._lib.gct_fdk_plan_create(C.byref(cg.struct()), C.byref(vol_geom.struct()),
                                                 C.byref((filt or FiltParams()).struct()),
                                                 C.byref(self.opts.struct()), C.byref(self._handle)))

    @property
    def workspace_bytes(self) -> int:
        n = C.c_uint64(0)
        _lib.check(self._lib.gct_fdk_plan_workspace_bytes(self._handle, C.byref(n)))
        return int(n.value)

    @property
    def quarter_turn(self) -> int:
        """+1 / -1 when whole-scan backprojections use the quarter-turn symmetry, else 0."""
        t = C.c_int32(0)
        _lib.check(self._lib.gct_fdk_plan_symmetry(self._handle, C.byref(t)))
        return int(t.value)

    @property
    def z_mirror(self) -> int:
        """1 when whole-volume backprojections pair each voxel with its mirror in z, else 0."""
        t = C.c_int32(0)
        _lib.check(self._lib.gct_fdk_plan_z_mirror(self._handle, C.byref(t)))
        return int(t.value)

    def execute(self, proj, vol, workspace=None, stream=None) -> None:
        _lib.check(self._lib.gct_fdk_execute(self._handle, C.c_void_p(_ptr(proj)), C.c_void_p(_ptr(vol)),
                                             _ws(workspace), C.c_void_p(_stream(stream))))

    def prepare(self, proj, workspace=None, view_begin: int = 0, view_count: int | None = None,
                stream=None) -> None:
        """Weights and ramp-filters views [view_begin, view_begin + view_count) into the workspace."""
        n = self.cg.num_views - view_begin if view_count is None else view_count
        _lib.check(self._lib.gct_fdk_prepare(self._handle, C.c_void_p(_ptr(proj)), _ws(workspace), view_begin, n,
                                             C.c_void_p(_stream(stream))))

    def backproject(self, vol, workspace=None, view_begin: int = 0, view_count: int | None = None,
                    accumulate: bool = False, stream=None) -> None:
        """Backprojects the prepared views into ``vol`` (overwrite, or add with ``accumulate``)."""
        n = self.cg.num_views - view_begin if view_count is None else view_count
        _lib.check(self._lib.gct_fdk_backproject(self._handle, _ws(workspace), C.c_void_p(_ptr(vol)), view_begin,
                                                 n, int(accumulate), C.c_void_p(_stream(stream))))

    def execute_host(self, proj: np.ndarray, vol: np.ndarray, stream=None) -> None:
        """Host arrays in and out through the plan's pipelined upload path (synchronous)."""
        fp = C.POINTER(C.c_float)
        for a in (proj, vol):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous):
                raise TypeError("expected contiguous float32 numpy arrays")
        if proj.size != self.cg.num_views * self.cg.num_rows * self.cg.num_cols:
            raise ValueError("projection array does not match the geometry")
        if vol.size != int(np.prod(self.vol_geom.shape)):
            raise ValueError("volume array does not match the grid")
        _lib.check(self._lib.gct_fdk_execute_host(self._handle, proj.ctypes.data_as(fp), vol.ctypes.data_as(fp),
                                                  C.c_void_p(_stream(stream))))

    def execute_host_async(self, proj: np.ndarray, vol: np.ndarray, stream=None) -> None:
        """As execute_host without the final wait; consecutive calls overlap. The arrays must stay
        untouched until host_sync()."""
        fp = C.POINTER(C.c_float)
        for a in (proj, vol):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous):
                raise TypeError("expected contiguous float32 numpy arrays")
        if proj.size != self.cg.num_views * self.cg.num_rows * self.cg.num_cols:
            raise ValueError("projection array does not match the geometry")
        if vol.size != int(np.prod(self.vol_geom.shape)):
            raise ValueError("volume array does not match the grid")
        _lib.check(self._lib.gct_fdk_execute_host_async(self._handle, proj.ctypes.data_as(fp), vol.ctypes.data_as(fp),
                                                        C.c_void_p(_stream(stream))))

    def host_sync(self) -> None:
        """Waits for every execute_host_async call of this plan."""
        _lib.check(self._lib.gct_fdk_host_sync(self._handle))

    def execute_host_budget(self, proj: np.ndarray, vol: np.ndarray, device_bytes: int, stream=None) -> None:
        """Host arrays in and out with at most `device_bytes` of device buffers for the projections
        (streamed in chunks of views; synchronous)."""
        fp = C.POINTER(C.c_float)
        for a in (proj, vol):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous):
                raise TypeError("expected contiguous float32 numpy arrays")
        if proj.size != self.cg.num_views * self.cg.num_rows * self.cg.num_cols:
            raise ValueError("projection array does not match the geometry")
        if vol.size != int(np.prod(self.vol_geom.shape)):
            raise ValueError("volume array does not match the grid")
        _lib.check(self._lib.gct_fdk_execute_host_budget(self._handle, proj.ctypes.data_as(fp), vol.ctypes.data_as(fp),
                                                         int(device_bytes), C.c_void_p(_stream(stream))))

    def filter(self, proj, out, stream=None) -> None:
        _lib.check(self._lib.gct_fdk_filter(self._handle, C.c_void_p(_ptr(proj)), C.c_void_p(_ptr(out)),
                                            C.c_void_p(_stream(stream))))

    def check(self) -> None:
        """Synchronises and raises GctError if the plan's kernels recorded a failure."""
        _lib.check(self._lib.gct_fdk_plan_check(self._handle))

    def close(self) -> None:
        if self._handle:
            _lib.check(self._lib.gct_fdk_plan_destroy(self._handle))
            self._handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class FdkBatch:
    """Many reconstructions in one persistent backprojection launch, replayed as a CUDA graph.

    ``items`` is a sequence of ``(plan, proj, vol)`` with device buffers (torch CUDA tensors or
    addresses); every ``launch`` overwrites each ``vol`` with its reconstruction. The plans and
    buffers must outlive the batch. No counterpart in the reference (one stack per call).
    """

    def __init__(self, items, autotune: bool = True, use_graph: bool = True, blocks_per_sm: int = 0):
        self._lib = _lib.load()
        self._handle = C.c_void_p()
        self._keep = list(items)
        arr = (_lib.gct_batch_item * len(self._keep))()
        for i, (plan, proj, vol) in enumerate(self._keep):
            arr[i].plan = plan._handle
            arr[i].proj_dev = _ptr(proj)
            arr[i].vol_dev = _ptr(vol)
        opts = _lib.gct_batch_opts()
        opts.autotune, opts.use_graph, opts.blocks_per_sm = int(autotune), int(use_graph), int(blocks_per_sm)
        _lib.check(self._lib.gct_fdk_batch_create(arr, len(self._keep), C.byref(opts), C.byref(self._handle)))

    def launch(self, stream=None) -> None:
        _lib.check(self._lib.gct_fdk_batch_launch(self._handle, C.c_void_p(_stream(stream))))

    def item_config(self, i: int) -> dict:
        c = _lib.gct_batch_item_config()
        _lib.check(self._lib.gct_fdk_batch_item_config(self._handle, i, C.byref(c)))
        return {"z_per_thread": c.z_per_thread, "block": (c.block_x, c.block_y),
                "views_per_stage": c.views_per_stage, "view_split": c.view_split, "tuned_gups": c.tuned_gups}

    def work(self) -> tuple[int, int]:
        """(work entries, voxel-view updates) of one launch."""
        n, u = C.c_uint64(), C.c_uint64()
        _lib.check(self._lib.gct_fdk_batch_work(self._handle, C.byref(n), C.byref(u)))
        return n.value, u.value

    def close(self) -> None:
        if self._handle:
            _lib.check(self._lib.gct_fdk_batch_destroy(self._handle))
            self._handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


REQ_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}


class FdkServer:
    """Request loop with continuous batching over a device-memory budget (gct_fdk_server_*).

    ``submit(plan, proj, vol)`` takes host float32 arrays ([view][row][col] in, [z][y][x] out),
    keeps references to them until the request finishes and returns a ticket. Pinned arrays
    (e.g. from ``torch.empty(..., pin_memory=True).numpy()``) let the copies overlap.
    No counterpart in the reference (one synchronous reconstruction per call).
    """

    def __init__(self, memory_budget_bytes: int, max_active: int = 0, autotune: bool = False,
                 round_updates: float = 0.0):
        self._lib = _lib.load()
        self._handle = C.c_void_p()
        self._keep = {}
        o = _lib.gct_server_opts()
        o.memory_budget_bytes, o.max_active, o.autotune = int(memory_budget_bytes), int(max_active), int(autotune)
        o.round_updates = float(round_updates)
        _lib.check(self._lib.gct_fdk_server_create(C.byref(o), C.byref(self._handle)))

    def submit(self, plan, proj: np.ndarray, vol: np.ndarray) -> int:
        fp = C.POINTER(C.c_float)
        for a in (proj, vol):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous):
                raise TypeError("expected contiguous float32 numpy arrays")
        t = C.c_uint64()
        _lib.check(self._lib.gct_fdk_server_submit(self._handle, plan._handle, proj.ctypes.data_as(fp),
                                                   vol.ctypes.data_as(fp), C.byref(t)))
        self._keep[t.value] = (plan, proj, vol)
        return t.value

    def wait(self, ticket: int, timeout_ms: float = -1.0) -> None:
        """Blocks until the request finishes; raises GctError if it failed, was cancelled or timed out."""
        st = self._lib.gct_fdk_server_wait(self._handle, ticket, float(timeout_ms))
        if st != _lib.GCT_ERR_NOT_READY:
            self._keep.pop(ticket, None)
        _lib.check(st)

    def info(self, ticket: int) -> dict:
        i = _lib.gct_request_info()
        _lib.check(self._lib.gct_fdk_server_info(self._handle, ticket, C.byref(i)))
        return {"state": REQ_STATES.get(i.state, i.state), "status": i.status, "queued_ms": i.queued_ms,
                "latency_ms": i.latency_ms, "rounds": i.rounds, "views_per_round": i.views_per_round}

    def cancel(self, ticket: int) -> None:
        _lib.check(self._lib.gct_fdk_server_cancel(self._handle, ticket))
        self._keep.pop(ticket, None)

    def stats(self) -> dict:
        s = _lib.gct_server_stats()
        _lib.check(self._lib.gct_fdk_server_stats(self._handle, C.byref(s)))
        return {k: getattr(s, k) for k, _ in _lib.gct_server_stats._fields_}

    def close(self) -> None:
        if self._handle:
            _lib.check(self._lib.gct_fdk_server_destroy(self._handle))
            self._handle = C.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def ellipsoid_array(ellipsoids) -> "C.Array":
    """ellipsoids: iterable of (cx, cy, cz, ax, ay, az, phi, mu)."""
    ell = list(ellipsoids)
    arr = (_lib.gct_ellipsoid * max(len(ell), 1))()
    for i, e in enumerate(ell):
        arr[i].center = (C.c_double * 3)(*e[0:3])
        arr[i].semi_axes = (C.c_double * 3)(*e[3:6])
        arr[i].phi = e[6]
        arr[i].mu = e[7]
    return arr, len(ell)


def phantom_project(cg: AxialCTGeom, ellipsoids, out, stream=None) -> None:
    """Analytic line integrals of ellipsoids into ``out`` (CUDA float32 [view][row][col])."""
    arr, n = ellipsoid_array(ellipsoids)
    _lib.check(_lib.load().gct_phantom_project(C.byref(cg.struct()), arr, n, C.c_void_p(_ptr(out)),
                                               C.c_void_p(_stream(stream))))


def forward_project(cg: AxialCTGeom, vol_geom: ReconImgGeom, vol, out, step_vox: float = 0.5,
                    stream=None) -> None:
    """Ray-driven forward projection of a device volume into ``out``."""
    _lib.check(_lib.load().gct_forward_project(C.byref(cg.struct()), C.byref(vol_geom.struct()),
                                               C.c_void_p(_ptr(vol)), float(step_vox), C.c_void_p(_ptr(out)),
                                               C.c_void_p(_stream(stream))))
