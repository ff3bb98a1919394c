"""TIFF raster files of the reference's pixel types (tops_tiff_write /
tops_tiff_read): round trips, the file layout other readers expect, big-endian
input and the formats that are refused.  No GPU."""
import struct

import numpy as np
import pytest


def _rand(kind, h, w, seed=0):
    rng = np.random.default_rng(seed)
    if kind == "cint16":
        return rng.integers(-32768, 32767, (h, w, 2), dtype=np.int16)
    if kind == "float32":
        return rng.standard_normal((h, w)).astype(np.float32)
    return (rng.standard_normal((h, w)) + 1j * rng.standard_normal((h, w))).astype(np.complex64)


@pytest.mark.parametrize("kind", ["cint16", "float32", "complex64"])
@pytest.mark.parametrize("shape", [(1, 1), (37, 1001), (700, 1000)])
def test_round_trip(T, tmp_path, kind, shape):
    a = _rand(kind, *shape)
    p = tmp_path / f"{kind}.tif"
    T.tiff_write(p, a)
    b = T.tiff_read(p)
    assert b.dtype == a.dtype and b.shape == a.shape
    assert np.array_equal(b.view(np.uint8), a.view(np.uint8))


def test_layout_and_pitch(T, tmp_path):
    import ctypes as C
    a = _rand("complex64", 300, 513, 4)
    wide = np.zeros((300, 600), np.complex64)
    wide[:, :513] = a
    p = tmp_path / "pitched.tif"
    T.check(T.lib.tops_tiff_write(str(p).encode(), 3, 513, 300, C.c_void_p(wide.ctypes.data),
                                  wide.strides[0]), "write")
    raw = p.read_bytes()
    assert raw[:4] == b"II*\x00"
    ifd = struct.unpack_from("<I", raw, 4)[0]
    n = struct.unpack_from("<H", raw, ifd)[0]
    tags = {}
    for i in range(n):
        tag, ty, cnt, val = struct.unpack_from("<HHII", raw, ifd + 2 + 12 * i)
        tags[tag] = (ty, cnt, val & 0xFFFF if ty == 3 and cnt == 1 else val)
    assert tags[256][2] == 513 and tags[257][2] == 300
    assert tags[258][2] == 64 and tags[339][2] == 6 and tags[259][2] == 1
    assert np.array_equal(T.tiff_read(p), a)


def test_pil_reads_float32(T, tmp_path):
    Image = pytest.importorskip("PIL.Image")
    a = _rand("float32", 50, 70, 2)
    p = tmp_path / "coh.tif"
    T.tiff_write(p, a)
    assert np.array_equal(np.asarray(Image.open(p)), a)


def _big_endian_tiff(path, a):
    """A one-strip big-endian float32 TIFF written by hand."""
    h, w = a.shape
    data = a.astype(">f4").tobytes()
    ifd = 8 + len(data)
    entries = [(256, 4, 1, w), (257, 4, 1, h), (258, 3, 1, 32), (259, 3, 1, 1), (262, 3, 1, 1),
               (273, 4, 1, 8), (277, 3, 1, 1), (278, 4, 1, h), (279, 4, 1, len(data)),
               (339, 3, 1, 3)]
    out = b"MM" + struct.pack(">HI", 42, ifd) + data + struct.pack(">H", len(entries))
    for tag, ty, cnt, val in entries:
        v = struct.pack(">HH", val, 0) if ty == 3 else struct.pack(">I", val)
        out += struct.pack(">HHI", tag, ty, cnt) + v
    path.write_bytes(out + struct.pack(">I", 0))


def test_big_endian_input(T, tmp_path):
    a = _rand("float32", 20, 33, 3)
    p = tmp_path / "be.tif"
    _big_endian_tiff(p, a)
    assert np.array_equal(T.tiff_read(p), a)


def test_refuses_compressed_and_unknown(T, tmp_path):
    a = _rand("float32", 10, 10, 5)
    p = tmp_path / "c.tif"
    T.tiff_write(p, a)
    raw = bytearray(p.read_bytes())
    ifd = struct.unpack_from("<I", raw, 4)[0]
    n = struct.unpack_from("<H", raw, ifd)[0]
    for i in range(n):
        at = ifd + 2 + 12 * i
        if struct.unpack_from("<H", raw, at)[0] == 259:
            struct.pack_into("<H", raw, at + 8, 5)   # LZW
    q = tmp_path / "lzw.tif"
    q.write_bytes(bytes(raw))
    with pytest.raises(T.TopsError):
        T.tiff_read(q)
    with pytest.raises(T.TopsError):
        T.tiff_read(tmp_path / "missing.tif")
    with pytest.raises(TypeError):
        T.tiff_write(tmp_path / "x.tif", np.zeros((2, 2), np.float64))


def test_int16_and_georef_round_trip(T, tmp_path):
    """An int16 raster with a north-up geotransform (a DEM) reads back with
    the geotransform GDAL would give it."""
    a = (np.arange(30 * 41).reshape(30, 41) - 700).astype(np.int16)
    gt = [10.5, 1 / 3600, 0.0, 45.25, 0.0, -1 / 3600]
    p = tmp_path / "dem.tif"
    T.tiff_write_georef(p, a, gt)
    assert np.array_equal(T.tiff_read(p), a)
    assert np.array_equal(T.tiff_georef(p), np.array(gt))
    f = np.random.default_rng(1).normal(0, 300, (17, 23)).astype(np.float32)
    T.tiff_write_georef(tmp_path / "f.tif", f, gt)
    assert np.array_equal(T.tiff_read(tmp_path / "f.tif"), f)


def test_georef_pixel_is_point(T, tmp_path):
    """A PixelIsPoint raster's origin moves half a pixel up and left, as
    GDAL reports it (GTRasterTypeGeoKey 1025 = 2)."""
    a = np.zeros((8, 8), np.int16)
    gt = [10.0, 0.5, 0.0, 40.0, 0.0, -0.25]
    p = tmp_path / "pt.tif"
    T.tiff_write_georef(p, a, gt)
    raw = bytearray(p.read_bytes())
    key = np.array([1025, 0, 1, 1], "<u2").tobytes()
    i = raw.index(key)
    raw[i:i + 8] = np.array([1025, 0, 1, 2], "<u2").tobytes()
    p.write_bytes(bytes(raw))
    assert np.allclose(T.tiff_georef(p), [10.0 - 0.25, 0.5, 0.0, 40.0 + 0.125, 0.0, -0.25])


def test_georef_refusals(T, tmp_path):
    a = np.zeros((4, 4), np.float32)
    T.tiff_write(tmp_path / "plain.tif", a)
    with pytest.raises(T.TopsError):
        T.tiff_georef(tmp_path / "plain.tif")
    with pytest.raises(T.TopsError):   # south-up or rotated transforms are not written
        T.tiff_write_georef(tmp_path / "x.tif", a, [0, 1, 0, 0, 0, 1])
