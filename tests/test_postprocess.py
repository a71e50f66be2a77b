"""Film post-processing (normalisation, photographic tone mapping, gamma/sRGB,
8-bit conversion; src/azimuth_main.cpp:1620-1760): the C restatement against
azimuth's own OutputPixelsToFile (bit for bit), and the GPU against azimuth."""
import numpy as np
import pytest

import azimuth_b200 as az
import oracle_lib as ol

SETTINGS = [
    ("photographic_srgb", (0.18, 1.0, 1.0, 1), 1.0 / 2.2, 1),
    ("photographic_gamma_saturated", (0.36, 5.0, 0.7, 1), 1.0 / 2.2, 0),
    ("none_srgb", (0.18, 1.0, 1.0, 0), 1.0 / 2.4, 1),
]


def _film():
    # a rendered film with an uneven weight per pixel (Gaussian filter)
    scene = az.generate_scene(az.SCENE_FEATURES, seed=2, width=48, height=40, spp=4)
    return ol.port_film(scene, seed=3)


@pytest.mark.skipif(not ol.have_ref(), reason="azimuth's compiled reference is not built here")
@pytest.mark.parametrize("name,tm,inv_gamma,srgb", SETTINGS, ids=[s[0] for s in SETTINGS])
def test_restatement_matches_azimuth_bit_for_bit(name, tm, inv_gamma, srgb):
    film = _film()
    r_rgb, r_8 = ol.output_pixels(film, tm, inv_gamma, srgb, kind="ref")
    p_rgb, p_8 = ol.output_pixels(film, tm, inv_gamma, srgb, kind="port")
    assert np.array_equal(r_rgb.view(np.uint32), p_rgb.view(np.uint32))
    assert np.array_equal(r_8, p_8)


@pytest.mark.gpu
@pytest.mark.parametrize("name,tm,inv_gamma,srgb", SETTINGS, ids=[s[0] for s in SETTINGS])
def test_gpu_postprocess_matches_azimuth(gpu, name, tm, inv_gamma, srgb):
    import torch
    film = _film()
    h, w = film.shape[:2]
    kind = "ref" if ol.have_ref() else "port"
    r_rgb, r_8 = ol.output_pixels(film, tm, inv_gamma, srgb, kind=kind)
    d_film = torch.from_numpy(film).cuda()
    rgb = torch.zeros((h, w, 3), device="cuda")
    rgb8 = torch.zeros((h, w, 3), device="cuda", dtype=torch.uint8)
    az.postprocess(d_film.data_ptr(), w, h, key_value=tm[0], burnout=tm[1], saturation=tm[2],
                   photographic=bool(tm[3]), inv_gamma=inv_gamma, srgb=bool(srgb), rgb_ptr=rgb.data_ptr(),
                   rgb8_ptr=rgb8.data_ptr())
    g_rgb, g_8 = rgb.cpu().numpy(), rgb8.cpu().numpy()
    # CUDA's logf/powf and the double log-average sum differ from glibc's and
    # azimuth's float sum in the last bits
    assert np.allclose(g_rgb, r_rgb, rtol=1e-4, atol=1e-6)
    diff = np.abs(g_8.astype(np.int32) - r_8.astype(np.int32))
    assert diff.max() <= 1 and (diff == 0).mean() >= 0.995
    # the film itself is left as it was
    assert np.array_equal(d_film.cpu().numpy(), film)


@pytest.mark.gpu
def test_gpu_postprocess_linear_output_is_the_normalised_film(gpu):
    import torch
    film = _film()
    h, w = film.shape[:2]
    d_film = torch.from_numpy(film).cuda()
    rgb = torch.zeros((h, w, 3), device="cuda")
    az.postprocess(d_film.data_ptr(), w, h, linear=True, rgb_ptr=rgb.data_ptr())
    assert np.array_equal(rgb.cpu().numpy(), (film[..., :3] / film[..., 3:4]).astype(np.float32))


@pytest.mark.gpu
@pytest.mark.skipif(not ol.have_ref(), reason="azimuth's compiled reference is not built here")
@pytest.mark.parametrize("fmt,ext", [(az.FILE_PNG, "png"), (az.FILE_BMP, "bmp"), (az.FILE_TGA, "tga")])
def test_gpu_output_pixels_to_file_matches_azimuths_file(gpu, tmp_path, fmt, ext):
    """az_gpu_output_pixels_to_file against azimuth's OutputPixelsToFile writing the same format."""
    import ctypes as C
    import torch
    from PIL import Image
    from azimuth_b200._native import Tonemap
    film = _film()
    h, w = film.shape[:2]
    ours, ref = str(tmp_path / ("ours." + ext)), str(tmp_path / ("ref." + ext))
    d_film = torch.from_numpy(film).cuda()
    az.output_pixels_to_file(ours, d_film.data_ptr(), w, h, fmt, save_exr=True)
    tm = Tonemap()
    tm.KeyValue, tm.BurnoutPercentage, tm.Saturation, tm.Operator = 0.18, 1.0, 1.0, 1
    px = np.ascontiguousarray(film, np.float32).copy()
    assert ol.ref().azref_output_pixels_fmt(px.ctypes.data, w, h, C.byref(tm), 1.0 / 2.2, 1, fmt, ref.encode()) == 1
    a = np.asarray(Image.open(ours).convert("RGB")).astype(np.int32)
    b = np.asarray(Image.open(ref).convert("RGB")).astype(np.int32)
    diff = np.abs(a - b)
    assert diff.max() <= 1 and (diff == 0).mean() >= 0.995
    # the EXR beside it: the normalised colours times 255 as halves
    from test_image_io import _read_exr
    _, got = _read_exr(str(tmp_path / "ours.exr"))
    want = ((film[..., :3] / film[..., 3:4]).astype(np.float32) * np.float32(255.0)).astype(np.float16)
    assert np.array_equal(got.view(np.uint16), want.view(np.uint16))
