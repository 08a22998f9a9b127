"""gct_b200: B200-native FDK reconstruction with GCT's geometry and reconstruct() API.

The compute path is the CUDA library ``libgct_fdk.so`` (sm_100a) behind the C ABI in
``include/gct_fdk.h``; this package is its Python host mirror.
"""
from ._lib import GctError, load as load_library, library_path
from .geometry import (ApodFunc, AxialCTGeom, ConeBeamProjGeomParams, CTGeom, DetFanArc, DetFanLine,
                       DetParallel, EqDistSampler, FanBeamProjGeomParams, GeomKind, Parallel1DProjGeomParams,
                       Parallel2DProjGeomParams, ProjectionMatrix, ProjectionStack, ProjGeom, ProjGeomFactory,
                       ReconImg, ReconImgGeom, RotationGeom, RotationParams, RotDir, SpiralCTGeom,
                       is_valid_axial_recon, kind_of, map_point, parker_weights, ramp_filter_taps, VIEW_DTYPE)
from .recon import (FILTER_FFT, FILTER_TOEPLITZ_BF16X3, FILTER_TOEPLITZ_BF16X4, FILTER_TOEPLITZ_F16X2,
                    SCAN_AXIAL, SCAN_SPIRAL, STORAGE_F16,
                    STORAGE_F32, SYMMETRY_AUTO, SYMMETRY_OFF, SYMMETRY_ON, FdkBatch, FdkOptions, FdkPlan, FdkServer,
                    FiltParams, forward_project, phantom_project, reconstruct)

from . import io

__all__ = [name for name in dir() if not name.startswith("_")]
