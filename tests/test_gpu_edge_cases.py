"""Boundary cases of the render entry points: empty and oversize scissors, a
1x1 image, sample counts that are not squares, depth 0, the resolution and
depth limits, and invalid arguments (status codes, no trap)."""
import ctypes as C

import numpy as np
import pytest

import azimuth_b200 as az
import oracle_lib as ol

pytestmark = pytest.mark.gpu

MAX_DEPTH_OFFSET = 1384 + 1320 + 16     # offsetof(az_scene, MaxRecursionDepth), see include/az_abi.h


def _sc(c0, r0, c1, r1):
    return az.Scissor(az.Vec2u(c1, r1), az.Vec2u(c0, r0))


def _oracle(scene, seed, scissor=None):
    return ol.ref_film(scene, seed=seed, scissor=scissor) if ol.have_ref() else ol.port_film(scene, seed=seed, scissor=scissor)


def test_empty_scissor_renders_nothing(gpu):
    scene = az.generate_scene(az.SCENE_CORNELL, width=16, height=16, spp=4)
    film = az.produce_image(scene, scissor=_sc(0, 5, 16, 5), seed=1)
    assert not film.any()


def test_scissor_past_the_image_is_clamped(gpu):
    scene = az.generate_scene(az.SCENE_CORNELL, width=24, height=20, spp=4)
    a = az.produce_image(scene, scissor=_sc(10, 12, 1000, 1000), seed=2)
    b = az.produce_image(scene, scissor=_sc(10, 12, 24, 20), seed=2)
    # equal up to the order of the film's float atomics
    assert ol.film_compare(a, b, 1e-4)[0] == 1.0 and np.array_equal(a[..., 3], b[..., 3])
    assert not a[:12].any() and not a[:, :10].any() and a[12:, 10:, 3].all()


def test_one_pixel_image_matches_the_oracle(gpu):
    scene = az.generate_scene(az.SCENE_CORNELL, width=1, height=1, spp=9)
    g = az.produce_image(scene, seed=3)
    r = _oracle(scene, 3)
    assert ol.film_compare(g, r, 1e-4)[0] == 1.0


def test_sample_count_is_floored_to_a_square(gpu):
    scene = az.generate_scene(az.SCENE_CORNELL, width=8, height=8, spp=8)     # 2 x 2 samples per pixel
    film = az.produce_image(scene, seed=4, filter_type=0)
    assert np.all(film[..., 3] == 4.0)


def test_depth_zero_matches_the_oracle(gpu):
    scene = az.generate_scene(az.SCENE_FEATURES, width=24, height=24, spp=4)
    depth = C.c_uint32.from_address(scene.scene_ptr + MAX_DEPTH_OFFSET)
    assert depth.value == scene.max_depth()
    depth.value = 0
    g = az.produce_image(scene, seed=5)
    r = _oracle(scene, 5)
    assert ol.film_compare(g, r, 1e-4)[0] >= 0.999


def test_limits_and_invalid_arguments_return_status_codes(gpu):
    import torch
    scene = az.generate_scene(az.SCENE_CORNELL, width=8, height=8, spp=1)
    with az.GpuScene(scene) as g:
        film = torch.zeros((8, 8, 4), device="cuda")
        with pytest.raises(az.AzError, match="AZ_ERR_INVALID_ARGUMENT"):
            g.render_device(film.data_ptr(), variant=az.LAUNCH_VARIANTS + 1)
        with pytest.raises(az.AzError, match="AZ_ERR_INVALID_ARGUMENT"):
            g.render_device(None)
        depth = C.c_uint32.from_address(scene.scene_ptr + MAX_DEPTH_OFFSET)
        depth.value = 62      # 63 tree levels: one more than the wave counters hold
        with az.GpuScene(scene) as deep:
            with pytest.raises(az.AzError, match="AZ_ERR_UNSUPPORTED"):
                deep.render_device(film.data_ptr())
        depth.value = 5
        g.render_device(film.data_ptr(), seed=1)      # the scene is still usable after the errors
        assert film[..., 3].sum().item() == 64.0
    with pytest.raises(az.AzError, match="AZ_ERR_INVALID_ARGUMENT"):
        az.GpuScene(scene, bvh_width=3)
    wide = az.generate_scene(az.SCENE_CORNELL, width=65536, height=1, spp=1)
    with az.GpuScene(wide) as g:
        with pytest.raises(az.AzError, match="AZ_ERR_INVALID_ARGUMENT"):
            g.render_device(film.data_ptr())
