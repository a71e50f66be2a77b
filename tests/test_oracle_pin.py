"""Pins the C restatement (oracle/az_oracle.c) to azimuth's own compiled code.

Both are compiled with the same flags and call the same libm, so on one
thread their films must be identical bit for bit.  Also pins the evaluation
order of azimuth's paired Random01() draws inside one expression (camera
lens, area-light point, glossy perturbation): GCC takes the second one first.
"""
import numpy as np
import pytest

import azimuth_b200 as az
import oracle_lib as ol

pytestmark = pytest.mark.skipif(not ol.have_ref(), reason="reference oracle not built (needs the reference sources)")

SCENES = [
    ("cornell", az.SCENE_CORNELL, dict(width=24, height=24, spp=4)),
    ("features", az.SCENE_FEATURES, dict(width=24, height=24, spp=4)),
    ("env_spheres", az.SCENE_ENV_SPHERES, dict(width=24, height=16, spp=4, env_width=64, env_height=32)),
    ("dense_mesh", az.SCENE_DENSE_MESH, dict(width=16, height=16, spp=4, detail=3)),
    ("motion_env", az.SCENE_MOTION_ENV, dict(width=24, height=16, spp=4, detail=300, env_width=64, env_height=32)),
]


@pytest.mark.parametrize("name,sid,kw", SCENES, ids=[s[0] for s in SCENES])
def test_restatement_film_is_bit_identical(name, sid, kw):
    scene = az.generate_scene(sid, seed=1, **kw)
    r = ol.ref_film(scene, seed=9, threads=1)
    p = ol.port_film(scene, seed=9, threads=1)
    assert np.array_equal(r.view(np.uint32), p.view(np.uint32))


def test_draw_order_of_paired_random01_calls():
    # the feature scene has a thin lens, an area light and a glossy mirror;
    # only the right-to-left order (7) reproduces azimuth's film
    scene = az.generate_scene(az.SCENE_FEATURES, seed=1, width=20, height=20, spp=4)
    r = ol.ref_film(scene, seed=4, threads=1)
    L = ol.port()
    try:
        for order in range(8):
            L.azo_set_order(order)
            p = ol.port_film(scene, seed=4, threads=1)
            assert np.array_equal(r, p) == (order == 7), order
    finally:
        L.azo_set_order(7)


def test_restatement_closest_hit_matches_reference():
    scene = az.generate_scene(az.SCENE_FEATURES, seed=2, width=8, height=8, spp=1)
    rng = np.random.default_rng(0)
    n = 20000
    o = rng.uniform(0.02, 0.98, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d, rng.uniform(0, 1, (n, 1))], axis=1).astype(np.float32)
    a = ol.closest_hit("ref", scene, rays)
    b = ol.closest_hit("port", scene, rays)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
