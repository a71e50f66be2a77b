"""The image writers against azimuth's own OutputPixelsToPNG / BMP / TGA / JPG
(src/azimuth_main.cpp:1460-1618, stb_image_write inside the reference
harness): the same 8-bit pixels, decoded with Pillow, must come back from
both; the BMP pixel rows are byte for byte the same; JPEG (lossy) is compared
by its error against the source.  The EXR writer is checked by parsing the
file (OpenEXR is not in the image, so azimuth's own EXR path cannot run)."""
import os
import struct

import numpy as np
import pytest

import azimuth_b200 as az
import oracle_lib as ol

PIL = pytest.importorskip("PIL.Image")

needs_ref = pytest.mark.skipif(not ol.have_ref(), reason="reference harness not built")


def _images():
    rng = np.random.default_rng(7)
    noise = rng.integers(0, 256, (23, 37, 3), dtype=np.uint8)        # odd width: BMP row padding
    h, w = 48, 200                                                   # runs longer than a TGA packet
    y, x = np.mgrid[0:h, 0:w]
    smooth = np.stack([(x * 255 // (w - 1)), (y * 255 // (h - 1)), ((x + y) % 64) * 4], -1).astype(np.uint8)
    smooth[10:20, 30:170] = (200, 40, 10)
    return {"noise": noise, "smooth": smooth, "single": np.array([[[1, 2, 3]]], np.uint8)}


def _colours(rgb8):
    # float colours whose (u8)(Clamp01(c) * 255) are the given bytes
    c = ((rgb8.astype(np.float32) + np.float32(0.5)) / np.float32(255.0)).astype(np.float32)
    back = (np.clip(c, 0, 1) * np.float32(255.0)).astype(np.float32).astype(np.uint8)
    assert np.array_equal(back, rgb8)
    return c


def _ref_file(rgb8, fmt, tmp_path, name):
    c = np.ascontiguousarray(_colours(rgb8))
    path = str(tmp_path / name)
    h, w = rgb8.shape[:2]
    assert ol.ref().azref_write_image(c.ctypes.data, w, h, fmt, path.encode()) == 1
    return path


def _decode(path):
    with PIL.open(path) as im:
        return np.asarray(im.convert("RGB"))


@needs_ref
@pytest.mark.parametrize("name", ["noise", "smooth", "single"])
@pytest.mark.parametrize("fmt,ext", [(az.FILE_PNG, "png"), (az.FILE_BMP, "bmp"), (az.FILE_TGA, "tga")])
def test_lossless_formats_match_azimuth(tmp_path, name, fmt, ext):
    rgb8 = _images()[name]
    ours = str(tmp_path / ("ours." + ext))
    az.write_image(ours, rgb8, fmt)
    ref = _ref_file(rgb8, fmt, tmp_path, "ref." + ext)
    a, b = _decode(ours), _decode(ref)
    assert np.array_equal(a, rgb8)
    assert np.array_equal(b, rgb8)
    if fmt == az.FILE_BMP:
        ob, rb = open(ours, "rb").read(), open(ref, "rb").read()
        off_o, off_r = struct.unpack_from("<I", ob, 10)[0], struct.unpack_from("<I", rb, 10)[0]
        # width, height, planes, bits per pixel, compression of the info header
        assert struct.unpack_from("<iiHHI", ob, 18) == struct.unpack_from("<iiHHI", rb, 18)
        h, w = rgb8.shape[:2]
        stride = (3 * w + 3) & ~3
        assert ob[off_o:off_o + stride * h] == rb[off_r:off_r + stride * h]
    if fmt == az.FILE_TGA and name == "smooth":
        # run-length packets make the file smaller than the raw pixels
        assert os.path.getsize(ours) < 18 + rgb8.size


@needs_ref
def test_jpeg_error_matches_azimuths(tmp_path):
    rgb8 = _images()["smooth"]
    ours = str(tmp_path / "ours.jpg")
    az.write_image(ours, rgb8, az.FILE_JPG)
    ref = _ref_file(rgb8, az.FILE_JPG, tmp_path, "ref.jpg")
    a, b = _decode(ours).astype(int), _decode(ref).astype(int)
    ea, eb = np.abs(a - rgb8), np.abs(b - rgb8)
    # quality 100: both within a few levels of the source, ours no worse than azimuth's
    assert ea.max() <= 6 and ea.mean() <= 1.0
    assert ea.mean() <= eb.mean() + 0.5
    assert np.abs(a - b).mean() <= 1.5


def test_jpeg_quality_trades_size_for_error(tmp_path):
    rgb8 = _images()["smooth"]
    errs, sizes = [], []
    for q in (30, 75, 100):
        p = str(tmp_path / ("q%d.jpg" % q))
        az.write_image(p, rgb8, quality=q)
        errs.append(np.abs(_decode(p).astype(int) - rgb8).mean())
        sizes.append(os.path.getsize(p))
    assert errs[0] > errs[1] > errs[2] and sizes[0] < sizes[1] < sizes[2]


def _read_exr(path):
    b = open(path, "rb").read()
    assert struct.unpack_from("<II", b, 0) == (20000630, 2)
    pos, attrs = 8, {}
    while b[pos] != 0:
        e = b.index(b"\0", pos)
        name = b[pos:e].decode()
        e2 = b.index(b"\0", e + 1)
        typ = b[e + 1:e2].decode()
        size = struct.unpack_from("<i", b, e2 + 1)[0]
        attrs[name] = (typ, b[e2 + 5:e2 + 5 + size])
        pos = e2 + 5 + size
    pos += 1
    x0, y0, x1, y1 = struct.unpack_from("<iiii", attrs["dataWindow"][1])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    offs = struct.unpack_from("<%dQ" % h, b, pos)
    out = np.zeros((h, w, 3), np.float16)
    for y in range(h):
        ly, n = struct.unpack_from("<ii", b, offs[y])
        assert ly == y and n == w * 6
        line = np.frombuffer(b, np.float16, 3 * w, offs[y] + 8).reshape(3, w)
        out[y] = line[::-1].T       # channels stored B, G, R
    return attrs, out


def test_exr_holds_the_half_values(tmp_path):
    rng = np.random.default_rng(3)
    rgb = rng.uniform(-2, 3e4, (9, 13, 3)).astype(np.float32)
    rgb[0, 0] = (1e-6, 7e-8, 70000.0)     # a subnormal, a value below half the smallest one, an overflow
    rgb[0, 1] = (0.0, -0.0, 65504.0)
    p = str(tmp_path / "a.exr")
    az.write_exr(p, rgb)
    attrs, got = _read_exr(p)
    assert attrs["compression"] == ("compression", b"\x00")
    assert attrs["channels"][0] == "chlist"
    with np.errstate(over="ignore"):
        want = rgb.astype(np.float16)
    assert np.array_equal(got.view(np.uint16), want.view(np.uint16))


def test_exr_sibling_names_follow_azimuth():
    assert az.exr_sibling_path("out/img.png") == "out/img.exr"
    assert az.exr_sibling_path("a.b.jpeg") == "a.b.exrg"
    assert az.exr_sibling_path("noext") == "nexrt"
    assert az.exr_sibling_path("x.pn") is None


def test_invalid_arguments_are_status_codes(tmp_path):
    with pytest.raises(az.AzError):
        az.write_image(str(tmp_path / "a.png"), np.zeros((2, 2, 3), np.uint8), 9)
    with pytest.raises(az.AzError):
        az.write_image(str(tmp_path / "no" / "such" / "dir.png"), np.zeros((2, 2, 3), np.uint8), az.FILE_PNG)
