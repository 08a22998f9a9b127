"""Array files: MetaImage (.mha / .mhd + .raw), Dennerlein (.den) and raw binaries.

Host mirror of GCT::IO (src/cpp/io): the readers MetaImgFileReader, DenFileReader and
RawDataFileReader (readMetadata / readData), ProjectionReader::read, ProjMatReader::read, the
writers ArrayFileWriter::write for each format and the image writer write(ReconImg, filename)
(src/cpp/io/img_writer/img_writer.{h,cpp}). Parsing, conversion and writing run in the native
library (gct_array_* in include/gct_fdk.h); this module shapes the arrays.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from .geometry import ProjectionMatrix, ProjectionStack, ReconImg


class ArrayElemType(enum.IntEnum):
    """GCT::IO::ArrayElemType (src/cpp/io/metadata.h:10-22)."""
    T_UINT8 = 0
    T_INT8 = 1
    T_UINT16 = 2
    T_INT16 = 3
    T_UINT32 = 4
    T_INT32 = 5
    T_UINT64 = 6
    T_INT64 = 7
    T_FLOAT = 8
    T_DOUBLE = 9


_NP = {ArrayElemType.T_UINT8: np.uint8, ArrayElemType.T_INT8: np.int8, ArrayElemType.T_UINT16: np.uint16,
       ArrayElemType.T_INT16: np.int16, ArrayElemType.T_UINT32: np.uint32, ArrayElemType.T_INT32: np.int32,
       ArrayElemType.T_UINT64: np.uint64, ArrayElemType.T_INT64: np.int64, ArrayElemType.T_FLOAT: np.float32,
       ArrayElemType.T_DOUBLE: np.float64}


def elem_type_of(dtype) -> ArrayElemType:
    dt = np.dtype(dtype)
    for t, d in _NP.items():
        if np.dtype(d) == dt:
            return t
    raise TypeError(f"no array-file element type for {dt}")


_META_IMAGE, _DEN, _RAW = 0, 1, 2


@dataclass
class ArrayMetadata:
    """GCT::IO::ArrayMetadata (src/cpp/io/metadata.h:24-30): one file's rows x columns x slices."""
    num_rows: int
    num_cols: int
    num_slices: int
    type: ArrayElemType

    def struct(self) -> _lib.gct_array_metadata:
        return _lib.gct_array_metadata(self.num_rows, self.num_cols, self.num_slices, int(self.type))

    @classmethod
    def from_struct(cls, s: _lib.gct_array_metadata) -> "ArrayMetadata":
        return cls(int(s.num_rows), int(s.num_cols), int(s.num_slices), ArrayElemType(s.type))


class _ArrayFileReader:
    """ArrayFileReader (src/cpp/io/file_reader/array_file_reader.h): metadata of one file and
    the data of the file, or of the series of files beside it."""
    _format = _META_IMAGE

    def __init__(self, filename: str, series: bool = False):
        self.filename = os.fspath(filename)
        self.series = bool(series)
        if not os.path.exists(self.filename):
            raise FileNotFoundError(f"File {self.filename} is not found.")
        self._raw_md = None

    def _md_arg(self):
        return C.byref(self._raw_md.struct()) if self._raw_md is not None else None

    def read_metadata(self) -> ArrayMetadata:
        lib = _lib.load()
        md = self._raw_md.struct() if self._raw_md is not None else _lib.gct_array_metadata()
        _lib.check(lib.gct_array_read_metadata(self.filename.encode(), self._format, C.byref(md)))
        return ArrayMetadata.from_struct(md)

    def read_data(self, dtype=np.float32) -> np.ndarray:
        """All elements (of every series member, in order) converted to `dtype` element by
        element as C++ static_cast does; a flat array."""
        lib = _lib.load()
        n = C.c_uint64(0)
        name = self.filename.encode()
        _lib.check(lib.gct_array_read(name, self._format, int(self.series), self._md_arg(), 0, None, 0, C.byref(n)))
        out = np.empty(int(n.value), dtype=_NP[elem_type_of(dtype)])
        _lib.check(lib.gct_array_read(name, self._format, int(self.series), self._md_arg(), int(elem_type_of(dtype)),
                                      out.ctypes.data_as(C.c_void_p), out.size, None))
        return out


class MetaImgFileReader(_ArrayFileReader):
    """MetaImgFileReader (src/cpp/io/file_reader/meta_img_reader.cpp:10-165)."""
    _format = _META_IMAGE


class DenFileReader(_ArrayFileReader):
    """DenFileReader (src/cpp/io/file_reader/den_file_reader.cpp)."""
    _format = _DEN


class RawDataFileReader(_ArrayFileReader):
    """RawDataFileReader (src/cpp/io/file_reader/raw_data_file_reader.h): headerless files whose
    metadata the caller gives."""
    _format = _RAW

    def __init__(self, filename: str, md: ArrayMetadata, series: bool = False):
        super().__init__(filename, series)
        self._raw_md = md


class ProjectionReader:
    """ProjectionReader<FileReader>::read (src/cpp/io/proj_reader/projection_reader.{h,cpp}): a
    file of 1D projections holds rows x slices projections of num_cols cells; a file of 2D
    projections holds slices projections of rows x columns."""

    @staticmethod
    def read(reader: _ArrayFileReader, dim: int) -> ProjectionStack:
        md = reader.read_metadata()
        data = reader.read_data(np.float32)
        if dim == 1:
            return ProjectionStack(md.num_cols, data.size // md.num_cols, data=data)
        if dim == 2:
            return ProjectionStack(md.num_cols, data.size // (md.num_cols * md.num_rows), md.num_rows, data=data)
        raise ValueError("projections are 1D or 2D")


class ProjMatReader:
    """ProjMatReader<FileReader>::read (src/cpp/io/geom_reader/proj_mat_reader.h:9-45): a file
    of num_slices 3 x 4 projection matrices (12 elements each, row-major), read as doubles."""

    @staticmethod
    def read(reader: _ArrayFileReader) -> list[ProjectionMatrix]:
        md = reader.read_metadata()
        data = reader.read_data(np.float64)
        n = md.num_slices
        if data.size != 12 * n:
            raise ValueError(f"Error during the reading of projection matrix file {reader.filename}.\n"
                             "There should be 12 elements in each projection matrix.")
        return [ProjectionMatrix(data[12 * i: 12 * i + 12]) for i in range(n)]


def _contig(data) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(data))
    elem_type_of(a.dtype)
    return a


def write_meta_image(dim_size, spacing, offset, data, filename: str) -> None:
    """ArrayFileWriter::write(MetaImgMetaData, data, filename) (meta_img_file_writer.h): x first
    in dim_size / spacing / offset; '.mha' keeps the data after the header, other names write
    '<stem>.raw' beside it."""
    a = _contig(data)
    nd = len(dim_size)
    if not (len(spacing) == len(offset) == nd):
        raise ValueError("dim_size, spacing and offset need one entry per dimension")
    ds = (C.c_uint32 * nd)(*[int(d) for d in dim_size])
    sp = (C.c_float * nd)(*[float(v) for v in spacing])
    of = (C.c_float * nd)(*[float(v) for v in offset])
    _lib.check(_lib.load().gct_meta_image_write(os.fspath(filename).encode(), nd, ds, sp, of,
                                                int(elem_type_of(a.dtype)), a.ctypes.data_as(C.c_void_p), a.size))


def write_den(num_rows: int, num_cols: int, num_slices: int, data, filename: str) -> None:
    """ArrayFileWriter::write(DenMetaData, data, filename) (den_file_writer.h)."""
    a = _contig(data)
    _lib.check(_lib.load().gct_den_write(os.fspath(filename).encode(), num_rows, num_cols, num_slices,
                                         int(elem_type_of(a.dtype)), a.ctypes.data_as(C.c_void_p), a.size))


def write_raw(data, filename: str) -> None:
    """ArrayFileWriter::write(data, filename) (raw_data_file_writer.h)."""
    a = _contig(data)
    _lib.check(_lib.load().gct_raw_write(os.fspath(filename).encode(), int(elem_type_of(a.dtype)),
                                         a.ctypes.data_as(C.c_void_p), a.size))


def write(img: ReconImg, filename: str) -> None:
    """write(ReconImg, filename) (src/cpp/io/img_writer/img_writer.{h,cpp}): '.den' with rows = y,
    columns = x, slices = z (1 for 2D); '.mha' / '.mhd' with DimSize x y [z], the sampling widths
    and the first voxel's position as Offset. Other extensions are not written (the reference
    prints a message; here a ValueError)."""
    ext = os.path.splitext(os.fspath(filename))[1].lower()
    g = img.geom
    samplers = [g.x, g.y] + ([g.z] if g.z is not None else [])
    if ext == ".den":
        write_den(g.y.num_samples, g.x.num_samples, g.z.num_samples if g.z is not None else 1, img.elements,
                  filename)
    elif ext in (".mha", ".mhd"):
        write_meta_image([s.num_samples for s in samplers], [s.sampling_width for s in samplers],
                         list(g.first_voxel_pos())[:len(samplers)], img.elements, filename)
    else:
        raise ValueError("Currently images can be saved to den or meta image file.")


def read_image(filename: str, series: bool = False) -> np.ndarray:
    """Convenience: a MetaImage or Dennerlein file as float32 [slices][rows][cols]."""
    ext = os.path.splitext(os.fspath(filename))[1].lower()
    reader = DenFileReader(filename, series) if ext == ".den" else MetaImgFileReader(filename, series)
    md = reader.read_metadata()
    return reader.read_data(np.float32).reshape(-1, md.num_rows, md.num_cols)
