"""Generates tests/golden/io/: array files written by satidev/gct's own writers and what its own
readers return for them and for hand-written headers.

Run after ``bash oracle/build_ref.sh`` (which compiles the reference's src/cpp/io sources under
the reference tree into oracle/_ref/libgct_ref_io.so):

    python tests/golden/make_io_golden.py

Every array is seeded and a few dozen elements long, so the fixtures stay small. `expected.npz`
holds, per file, the reference reader's metadata (rows, cols, slices, ArrayElemType) and its
readData<double>() values; `inputs.npz` holds the arrays and header values given to the
reference writers, so the tests can write the same files with the engine and compare bytes.
"""
from __future__ import annotations

import ctypes as C
import shutil
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
LIB = REPO / "oracle" / "_ref" / "libgct_ref_io.so"
OUT = HERE / "io"

KIND = {np.float32: 0, np.uint16: 1, np.int16: 2, np.float64: 3, np.uint8: 4}


def load():
    lib = C.CDLL(str(LIB))
    lib.ref_io_error.restype = C.c_char_p
    lib.ref_io_write_meta_image.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_uint), C.POINTER(C.c_float),
                                            C.POINTER(C.c_float), C.c_int, C.c_void_p, C.c_size_t]
    lib.ref_io_write_den.argtypes = [C.c_char_p, C.c_uint, C.c_uint, C.c_uint, C.c_int, C.c_void_p, C.c_size_t]
    lib.ref_io_read_metadata.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_uint)]
    lib.ref_io_read_f64.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_size_t,
                                    C.POINTER(C.c_size_t)]
    return lib


def check(lib, rc):
    if rc != 0:
        raise RuntimeError(lib.ref_io_error().decode())


def main():
    lib = load()
    if OUT.exists():
        shutil.rmtree(OUT)
    (OUT / "series").mkdir(parents=True)
    rs = np.random.RandomState(7)
    inputs, expected = {}, {}

    def write_mi(name, arr, dims, spacing, offset):
        a = np.ascontiguousarray(arr)
        nd = len(dims)
        check(lib, lib.ref_io_write_meta_image(str(OUT / name).encode(), nd, (C.c_uint * nd)(*dims),
                                               (C.c_float * nd)(*spacing), (C.c_float * nd)(*offset),
                                               KIND[a.dtype.type], a.ctypes.data_as(C.c_void_p), a.size))
        key = name.replace("/", "__")
        inputs[key + "__data"] = a
        inputs[key + "__dims"] = np.array(dims, np.uint32)
        inputs[key + "__spacing"] = np.array(spacing, np.float32)
        inputs[key + "__offset"] = np.array(offset, np.float32)

    def write_den(name, arr, rows, cols, slices):
        a = np.ascontiguousarray(arr)
        check(lib, lib.ref_io_write_den(str(OUT / name).encode(), rows, cols, slices, KIND[a.dtype.type],
                                        a.ctypes.data_as(C.c_void_p), a.size))
        inputs[name + "__data"] = a
        inputs[name + "__dims"] = np.array([rows, cols, slices], np.uint32)

    def record(name, fmt, series=False):
        md = (C.c_uint * 4)()
        check(lib, lib.ref_io_read_metadata(str(OUT / name).encode(), fmt, md))
        out = np.zeros(4096, np.float64)
        n = C.c_size_t(0)
        check(lib, lib.ref_io_read_f64(str(OUT / name).encode(), fmt, int(series),
                                       out.ctypes.data_as(C.POINTER(C.c_double)), out.size, C.byref(n)))
        key = name.replace("/", "__") + ("__series" if series else "")
        expected[key + "__md"] = np.array(list(md), np.uint32)
        expected[key + "__data"] = out[: n.value].copy()

    # the reference's writers
    write_mi("f32_3d.mha", rs.randn(4, 2, 3).astype(np.float32), [3, 2, 4], [0.5, 0.25, 1.0], [-1.5, 2.0, 0.75])
    write_mi("u16_2d.mhd", rs.randint(0, 60000, (2, 3)).astype(np.uint16), [3, 2], [0.8, 0.8], [0.0, -3.2])
    write_mi("i16_3d.mha", rs.randint(-30000, 30000, (2, 3, 5)).astype(np.int16), [5, 3, 2], [1, 1, 1], [0, 0, 0])
    write_mi("f64_2d.mha", rs.randn(3, 4), [4, 3], [0.125, 3.0], [1e-3, -7.25])
    write_mi("u8_3d.mhd", rs.randint(0, 255, (3, 2, 2)).astype(np.uint8), [2, 2, 3], [2, 2, 2], [1, 2, 3])
    write_den("f32.den", rs.randn(4, 2, 3).astype(np.float32), 2, 3, 4)
    write_den("u16.den", rs.randint(0, 60000, (1, 3, 5)).astype(np.uint16), 3, 5, 1)
    write_den("f64.den", rs.randn(2, 2, 2), 2, 2, 2)
    write_den("u8.den", rs.randint(0, 255, (2, 4, 3)).astype(np.uint8), 4, 3, 2)
    for k in range(3):  # a series: same extension and size, sorted names
        write_mi(f"series/s{k:02d}.mha", (rs.randn(2, 2, 3) + 10 * k).astype(np.float32), [3, 2, 2],
                 [1, 1, 1], [0, 0, 0])

    # hand-written headers: tag order, extra tags, spaces the reference's parser allows
    body = rs.randn(3, 4).astype(np.float32)
    hdr = ("ObjectType = Image\nNDims = 2\nCompressedData = False\nElementSpacing = 1 1\n"
           "DimSize =   4   3\nAnatomicalOrientation = RAI\nElementType = MET_FLOAT\nElementDataFile = LOCAL\n")
    (OUT / "hand_2d.mha").write_bytes(hdr.encode() + body.tobytes())
    inputs["hand_2d.mha__data"] = body
    body = rs.randint(-100, 100, (2, 2, 3)).astype(np.int32)
    (OUT / "hand_i32.raw").write_bytes(body.tobytes())
    (OUT / "hand_i32.mhd").write_text("NDims = 3\nDimSize = 3 2 2\nElementType = MET_INT\n"
                                      "ElementDataFile = hand_i32.raw\n")
    inputs["hand_i32.mhd__data"] = body

    for name in ["f32_3d.mha", "u16_2d.mhd", "i16_3d.mha", "f64_2d.mha", "u8_3d.mhd", "hand_2d.mha",
                 "hand_i32.mhd", "series/s00.mha"]:
        record(name, 0)
    record("series/s00.mha", 0, series=True)
    for name in ["f32.den", "u16.den", "f64.den", "u8.den"]:
        record(name, 1)
    np.savez(OUT / "inputs.npz", **inputs)
    np.savez(OUT / "expected.npz", **expected)
    print(f"wrote {sorted(p.name for p in OUT.rglob('*') if p.is_file())}")


if __name__ == "__main__":
    main()
