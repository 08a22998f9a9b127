"""Array files (MetaImage, Dennerlein, raw) against satidev/gct's own readers and writers.

The fixtures under tests/golden/io/ were written by the reference's writers, and expected.npz holds
what the reference's readers return for them (tests/golden/make_io_golden.py, run against the
reference sources compiled by oracle/build_ref.sh). Bar: bit-exact metadata, values and bytes.
"""
import os
import shutil
from pathlib import Path

import numpy as np
import pytest

import gct_b200 as g
from gct_b200 import io

GOLD = Path(__file__).resolve().parent / "golden" / "io"
EXP = np.load(GOLD / "expected.npz")
INP = np.load(GOLD / "inputs.npz")

MI_FILES = ["f32_3d.mha", "u16_2d.mhd", "i16_3d.mha", "f64_2d.mha", "u8_3d.mhd", "hand_2d.mha", "hand_i32.mhd",
            "series/s00.mha"]
DEN_FILES = ["f32.den", "u16.den", "f64.den", "u8.den"]


def _md_tuple(md):
    return [md.num_rows, md.num_cols, md.num_slices, int(md.type)]


@pytest.mark.parametrize("name", MI_FILES + DEN_FILES)
def test_reader_matches_reference_reader(name):
    reader = (io.DenFileReader if name.endswith(".den") else io.MetaImgFileReader)(str(GOLD / name))
    key = name.replace("/", "__")
    assert _md_tuple(reader.read_metadata()) == EXP[key + "__md"].tolist()
    got = reader.read_data(np.float64)
    assert np.array_equal(got, EXP[key + "__data"])


def test_series_matches_reference_reader():
    reader = io.MetaImgFileReader(str(GOLD / "series" / "s00.mha"), series=True)
    assert _md_tuple(reader.read_metadata()) == EXP["series__s00.mha__series__md"].tolist()
    assert np.array_equal(reader.read_data(np.float64), EXP["series__s00.mha__series__data"])
    assert reader.read_data(np.float64).size == 3 * 12


@pytest.mark.parametrize("name", ["f32_3d.mha", "u16_2d.mhd", "i16_3d.mha", "f64_2d.mha", "u8_3d.mhd"])
def test_meta_image_writer_bytes_match_reference_writer(name, tmp_path):
    out = tmp_path / name
    io.write_meta_image(INP[name + "__dims"], INP[name + "__spacing"], INP[name + "__offset"], INP[name + "__data"],
                        str(out))
    assert out.read_bytes() == (GOLD / name).read_bytes()
    if name.endswith(".mhd"):
        raw = Path(name).stem + ".raw"
        assert (tmp_path / raw).read_bytes() == (GOLD / raw).read_bytes()


@pytest.mark.parametrize("name", DEN_FILES)
def test_den_writer_bytes_match_reference_writer(name, tmp_path):
    rows, cols, slices = INP[name + "__dims"].tolist()
    io.write_den(rows, cols, slices, INP[name + "__data"], str(tmp_path / name))
    assert (tmp_path / name).read_bytes() == (GOLD / name).read_bytes()


@pytest.mark.parametrize("dtype", [np.uint8, np.int8, np.uint16, np.int16, np.uint32, np.int32, np.uint64, np.int64,
                                   np.float32, np.float64])
def test_round_trip_every_element_type(dtype, tmp_path):
    rs = np.random.RandomState(3)
    a = (rs.randn(3, 4, 5) * 50).astype(dtype)
    io.write_meta_image([5, 4, 3], [1, 1, 1], [0, 0, 0], a, str(tmp_path / "a.mha"))
    r = io.MetaImgFileReader(str(tmp_path / "a.mha"))
    assert r.read_metadata().type == io.elem_type_of(dtype)
    assert np.array_equal(r.read_data(dtype), a.ravel())
    # element-wise static_cast to another type, like readData<OpType>
    assert np.array_equal(r.read_data(np.float64), a.ravel().astype(np.float64))
    io.write_raw(a, str(tmp_path / "a.raw"))
    md = io.ArrayMetadata(4, 5, 3, io.elem_type_of(dtype))
    assert np.array_equal(io.RawDataFileReader(str(tmp_path / "a.raw"), md).read_data(dtype), a.ravel())


def test_reader_errors(tmp_path):
    with pytest.raises(FileNotFoundError):
        io.MetaImgFileReader(str(tmp_path / "missing.mha"))
    bad = tmp_path / "bad.mha"
    bad.write_text("NDims = 2\nDimSize = 2 2\nElementType = MET_HALF\nElementDataFile = LOCAL\n")
    with pytest.raises(g.GctError, match="not a valid ElementType"):
        io.MetaImgFileReader(str(bad)).read_metadata()
    nodata = tmp_path / "nodata.mhd"
    nodata.write_text("NDims = 2\nDimSize = 2 2\nElementType = MET_FLOAT\nElementDataFile = absent.raw\n")
    with pytest.raises(g.GctError, match="is not found"):
        io.MetaImgFileReader(str(nodata)).read_data()
    # a raw data file of the wrong size
    shutil.copy(GOLD / "u16_2d.mhd", tmp_path / "u16_2d.mhd")
    (tmp_path / "u16_2d.raw").write_bytes((GOLD / "u16_2d.raw").read_bytes()[:-2])
    with pytest.raises(g.GctError, match="data bytes"):
        io.MetaImgFileReader(str(tmp_path / "u16_2d.mhd")).read_data()
    # a LOCAL file shorter than its header promises
    (tmp_path / "short.mha").write_bytes((GOLD / "f32_3d.mha").read_bytes()[:-4])
    with pytest.raises(g.GctError, match="fewer data bytes"):
        io.MetaImgFileReader(str(tmp_path / "short.mha")).read_data()


def test_writer_errors(tmp_path):
    a = np.zeros((2, 3), np.float32)
    with pytest.raises(g.GctError, match="Mismatch in the number of elements"):
        io.write_meta_image([3, 3], [1, 1], [0, 0], a, str(tmp_path / "x.mha"))
    with pytest.raises(g.GctError, match="Mismatch in the number of elements"):
        io.write_den(2, 2, 1, a, str(tmp_path / "x.den"))
    with pytest.raises(g.GctError, match="16-bit"):
        io.write_den(70000, 1, 1, np.zeros(70000, np.float32), str(tmp_path / "x.den"))
    with pytest.raises(g.GctError, match="not writable"):
        io.write_raw(a, str(tmp_path / "no_such_dir" / "x.raw"))


def test_projection_reader_shapes(tmp_path):
    # 1D projections: rows x slices projections of num_cols cells; 2D: slices projections
    a = np.arange(2 * 3 * 5, dtype=np.float32).reshape(2, 3, 5)
    io.write_meta_image([5, 3, 2], [1, 1, 1], [0, 0, 0], a, str(tmp_path / "p.mha"))
    r = io.MetaImgFileReader(str(tmp_path / "p.mha"))
    p1 = io.ProjectionReader.read(r, 1)
    assert (p1.num_cols, p1.num_proj, p1.num_rows) == (5, 6, None)
    p2 = io.ProjectionReader.read(r, 2)
    assert (p2.num_cols, p2.num_proj, p2.num_rows) == (5, 2, 3)
    assert np.array_equal(p2.elements, a)


def test_image_writer_headers(tmp_path):
    vg = g.ReconImgGeom(g.EqDistSampler(4, 0.5), g.EqDistSampler(3, 0.25), g.EqDistSampler(2, 2.0), (1.0, -2.0, 0.5))
    img = g.ReconImg(vg)
    img.elements[:] = np.random.RandomState(1).randn(*img.elements.shape).astype(np.float32)
    io.write(img, str(tmp_path / "v.mha"))
    text = (tmp_path / "v.mha").read_bytes().split(b"ElementDataFile = LOCAL\n")[0].decode()
    x0, y0, z0 = vg.first_voxel_pos()
    assert "DimSize = 4 3 2\n" in text
    assert "ElementSpacing = 0.500000 0.250000 2.000000\n" in text
    assert f"Offset = {x0:f} {y0:f} {z0:f}\n" in text
    assert np.array_equal(io.read_image(str(tmp_path / "v.mha")), img.elements)
    io.write(img, str(tmp_path / "v.den"))
    r = io.DenFileReader(str(tmp_path / "v.den"))
    assert _md_tuple(r.read_metadata()) == [3, 4, 2, int(io.ArrayElemType.T_FLOAT)]
    assert np.array_equal(io.read_image(str(tmp_path / "v.den")), img.elements)
    with pytest.raises(ValueError):
        io.write(img, str(tmp_path / "v.tif"))
