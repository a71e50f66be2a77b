"""ctypes access to the oracle libraries (test infrastructure only).

* ``ref()``:  azimuth's own render code compiled by oracle/build.py
  (oracle/_ref/libazref.so).  Present where the reference sources were
  available at build time; the built file travels with the repository.
* ``port()``: the C restatement oracle/az_oracle.c (oracle/lib/libazoracle.so),
  compiled on demand with gcc.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(REPO, "oracle", "_ref", "libazref.so")
REF_FAST_SO = os.path.join(REPO, "oracle", "_ref", "libazref_fast.so")
PORT_SO = os.path.join(REPO, "oracle", "lib", "libazoracle.so")

_ref = {}
_port = None


class Vec2u(C.Structure):
    _fields_ = [("x", C.c_uint32), ("y", C.c_uint32)]


class Scissor(C.Structure):
    _fields_ = [("Max", Vec2u), ("Min", Vec2u)]


def have_ref(fast=False):
    return os.path.exists(REF_FAST_SO if fast else REF_SO)


def ref(fast=False):
    path = REF_FAST_SO if fast else REF_SO
    if path not in _ref:
        L = C.CDLL(path)
        vp, u32, i32, u64 = C.c_void_p, C.c_uint32, C.c_int32, C.c_uint64
        L.azref_set_seed.argtypes = [u64]
        L.azref_output_pixels.argtypes = [vp, u32, u32, vp, C.c_float, u32, C.c_char_p]
        L.azref_output_pixels.restype = i32
        L.azref_output_pixels_fmt.argtypes = [vp, u32, u32, vp, C.c_float, u32, i32, C.c_char_p]
        L.azref_output_pixels_fmt.restype = i32
        L.azref_write_image.argtypes = [vp, u32, u32, i32, C.c_char_p]
        L.azref_write_image.restype = i32
        L.azref_produce_image.argtypes = [vp, vp, vp, vp, Scissor, i32, i32, u32]
        L.azref_closest_hit.argtypes = [vp, vp, u32, i32, C.c_float, vp, vp, vp, vp, vp, i32]
        L.azref_sample_radiance.argtypes = [vp, vp, vp, vp, Scissor, i32, u32]
        L.azref_set_perlin_gradients.argtypes = [vp]
        L.azref_get_perlin_gradients.argtypes = [vp]
        L.azref_construct_bvh.argtypes = [vp, vp, u32]
        L.azref_construct_bvh_triangles.argtypes = [vp, vp, u32]
        L.azref_sample_perlin.argtypes = [vp, C.c_float, C.c_float, C.c_float]
        L.azref_sample_perlin.restype = C.c_float
        L.azref_random01.restype = C.c_float
        L.azref_light_contribution.argtypes = [vp, vp, vp, vp, vp, C.c_float, C.c_float, C.c_float, vp]
        L.azref_sizeof_entity.restype = u32
        _ref[path] = L
    return _ref[path]


def port():
    global _port
    if _port is None:
        src = os.path.join(REPO, "oracle", "az_oracle.c")
        if not os.path.exists(PORT_SO) or os.path.getmtime(PORT_SO) < os.path.getmtime(src):
            subprocess.check_call([sys.executable, os.path.join(REPO, "oracle", "build.py")])
        L = C.CDLL(PORT_SO)
        vp, u32, i32, u64 = C.c_void_p, C.c_uint32, C.c_int32, C.c_uint64
        L.azo_set_order.argtypes = [i32]
        L.azo_output_pixels.argtypes = [vp, u32, u32, vp, C.c_float, u32, vp, vp]
        L.azo_output_pixels.restype = i32
        L.azo_set_gradients.argtypes = [vp]
        L.azo_produce_image.argtypes = [vp, vp, vp, vp, Scissor, i32, i32, u64, i32]
        L.azo_render_samples.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, u32, i32, u64]
        L.azo_closest_hit.argtypes = [vp, vp, u32, i32, C.c_float, vp, vp, vp, vp, i32]
        L.azo_u01.argtypes = [u64, u32, u32, u32, u32, u32]
        L.azo_u01.restype = C.c_float
        L.azo_philox.argtypes = [vp, u32, u32, vp]
        L.azo_sample_perlin.argtypes = [vp, C.c_float, C.c_float, C.c_float]
        L.azo_sample_perlin.restype = C.c_float
        # evaluation order of paired draws in the oracle build: all three pairs
        # right to left (pinned by tests/test_oracle_pin.py)
        L.azo_set_order(7)
        _port = L
    return _port


def scissor_of(scene, rows=None, cols=None):
    w, h = scene.resolution()
    r0, r1 = rows if rows else (0, h)
    c0, c1 = cols if cols else (0, w)
    return Scissor(Vec2u(c1, r1), Vec2u(c0, r0))


def output_pixels(film, tonemap, inv_gamma, srgb, kind="ref", tmpdir="/tmp"):
    """azimuth's OutputPixelsToFile post-processing of a film (H, W, 4): (colours (H, W, 3) float32, the
    8-bit values azimuth writes).  kind "ref" runs azimuth's own function (writing a BMP it then
    discards), "port" the C restatement."""
    import tempfile
    from azimuth_b200._native import Tonemap
    h, w = film.shape[:2]
    tm = Tonemap()
    tm.KeyValue, tm.BurnoutPercentage, tm.Saturation, tm.Operator = tonemap
    if kind == "ref":
        px = np.ascontiguousarray(film, np.float32).copy()
        fd, path = tempfile.mkstemp(suffix=".bmp", dir=tmpdir)
        os.close(fd)
        try:
            ok = ref().azref_output_pixels(px.ctypes.data, w, h, C.byref(tm), inv_gamma, srgb, path.encode())
        finally:
            os.unlink(path)
        assert ok == 1
        rgb = np.ascontiguousarray(px[..., :3])
        rgb8 = (np.clip(rgb, 0.0, 1.0) * np.float32(255.0)).astype(np.float32).astype(np.uint8)
        return rgb, rgb8
    rgb = np.zeros((h, w, 3), np.float32)
    rgb8 = np.zeros((h, w, 3), np.uint8)
    port().azo_output_pixels(np.ascontiguousarray(film, np.float32).ctypes.data, w, h, C.byref(tm), inv_gamma, srgb,
                             rgb.ctypes.data, rgb8.ctypes.data)
    return rgb, rgb8


def ref_film(scene, seed=0, threads=None, scissor=None, fast=False, filter_type=None):
    """azimuth's ProduceImageInLinearSpace over the scissor (film numpy (H, W, 4))."""
    L = ref(fast)
    w, h = scene.resolution()
    film = np.zeros((h, w, 4), np.float32)
    L.azref_set_seed(seed)
    if scene.perlin_gradients:
        L.azref_set_perlin_gradients(scene.perlin_gradients)
    ft = scene.filter_type if filter_type is None else filter_type
    L.azref_produce_image(film.ctypes.data, scene.scene_ptr, scene.camera_ptr, scene.epsilons_ptr,
                          scissor or scissor_of(scene), ft, 0, threads or os.cpu_count())
    return film


def ref_samples(scene, seed=0, threads=None, scissor=None):
    """azimuth's colour of every camera sample of the scissor (before ComputeSampleWeight), as an array
    (samples, 4) in the order sample number * scissor pixels + pixel (row-major in the scissor)."""
    L = ref()
    sc = scissor or scissor_of(scene)
    w, h = scene.resolution()
    rows = min(sc.Max.y, h) - sc.Min.y
    cols = min(sc.Max.x, w) - sc.Min.x
    k = int(np.sqrt(np.float32(scene.sample_count())))   # (u32)Sqrt((f32)SampleCount)
    out = np.zeros((k * k * rows * cols, 4), np.float32)
    L.azref_set_seed(seed)
    if scene.perlin_gradients:
        L.azref_set_perlin_gradients(scene.perlin_gradients)
    L.azref_sample_radiance(out.ctypes.data, scene.scene_ptr, scene.camera_ptr, scene.epsilons_ptr, sc, 0,
                            threads or os.cpu_count())
    return out


def port_film(scene, seed=0, threads=None, scissor=None, filter_type=None):
    L = port()
    w, h = scene.resolution()
    film = np.zeros((h, w, 4), np.float32)
    if scene.perlin_gradients:
        L.azo_set_gradients(scene.perlin_gradients)
    ft = scene.filter_type if filter_type is None else filter_type
    L.azo_produce_image(film.ctypes.data, scene.scene_ptr, scene.camera_ptr, scene.epsilons_ptr,
                        scissor or scissor_of(scene), ft, 0, seed, threads or os.cpu_count())
    return film


def closest_hit(lib_kind, scene, rays, cull=0, eps=0.0, threads=None):
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[0]
    hit = np.zeros(n, np.uint32)
    uid = np.zeros(n, np.uint32)
    face = np.zeros(n, np.uint32)
    t = np.zeros(n, np.float32)
    if lib_kind == "ref":
        pnuv = np.zeros((n, 8), np.float32)
        ref().azref_closest_hit(scene.scene_ptr, rays.ctypes.data, n, cull, eps, hit.ctypes.data, uid.ctypes.data,
                                face.ctypes.data, t.ctypes.data, pnuv.ctypes.data, threads or os.cpu_count())
    else:
        port().azo_closest_hit(scene.scene_ptr, rays.ctypes.data, n, cull, eps, hit.ctypes.data, uid.ctypes.data,
                               face.ctypes.data, t.ctypes.data, threads or os.cpu_count())
    return hit, uid, face, t


def film_compare(a, b, rel=1e-4):
    """Per-pixel comparison of two films (H, W, 4).

    Returns (fraction of pixels whose every channel agrees within `rel`
    relative to max(|b|, 1e-3 * mean |b|), max relative error over the agreeing
    pixels, relMSE of the resolved images)."""
    floor = 1e-3 * max(float(np.abs(b[..., :3]).mean()), 1e-12)
    den = np.maximum(np.abs(b), floor)
    err = np.abs(a - b) / den
    ok = (err <= rel).all(axis=-1)
    wa = np.maximum(a[..., 3:4], 1e-12)
    wb = np.maximum(b[..., 3:4], 1e-12)
    ia, ib = a[..., :3] / wa, b[..., :3] / wb
    relmse = float(np.mean((ia - ib) ** 2 / (ib ** 2 + 1e-2)))
    return float(ok.mean()), float(err[ok].max()) if ok.any() else float("inf"), relmse
