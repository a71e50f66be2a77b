"""Committed golden fixtures (tests/golden/, written by make_golden.py from
azimuth's own compiled code): films of ProduceImageInLinearSpace on one
thread with OutputPixelsToFile's colours and bytes, and nearest hits of
RayEntityIntersection.  The C restatement must reproduce them bit for bit on
the CPU, and the GPU within the bars of the live parity tests, so parity is
pinned even where the compiled reference is not available."""
import glob
import os

import numpy as np
import pytest

import azimuth_b200 as az
import oracle_lib as ol

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILMS = sorted(glob.glob(os.path.join(GOLDEN, "film_*.npz")))
HITS = sorted(glob.glob(os.path.join(GOLDEN, "hits_*.npz")))
TONEMAP = ((0.18, 1.0, 1.0, 1), 1.0 / 2.2, 1)


def _scene(g):
    kw = {k[4:]: int(g[k]) for k in g.files if k.startswith("gen_")}
    return az.generate_scene(int(g["scene_id"]), **kw)


def _id(path):
    return os.path.basename(path)[:-4]


def test_fixtures_are_present():
    assert len(FILMS) >= 3 and len(HITS) >= 3


@pytest.mark.parametrize("path", FILMS, ids=[_id(p) for p in FILMS])
def test_restatement_reproduces_golden_film(path):
    g = np.load(path)
    sc = _scene(g)
    try:
        film = ol.port_film(sc, seed=int(g["seed"]), threads=1)
    finally:
        sc.close()
    assert np.array_equal(film.view(np.uint32), g["film"].view(np.uint32))
    rgb, rgb8 = ol.output_pixels(g["film"].copy(), *TONEMAP, kind="port")
    assert np.array_equal(rgb.view(np.uint32), g["rgb"].view(np.uint32))
    assert np.array_equal(rgb8, g["rgb8"])


@pytest.mark.parametrize("path", HITS, ids=[_id(p) for p in HITS])
def test_restatement_reproduces_golden_hits(path):
    g = np.load(path)
    sc = _scene(g)
    try:
        hit, uid, face, t = ol.closest_hit("port", sc, g["rays"], threads=1)
    finally:
        sc.close()
    assert np.array_equal(hit, g["hit"]) and np.array_equal(uid, g["uid"]) and np.array_equal(face, g["face"])
    assert np.array_equal(t.view(np.uint32), g["t"].view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("path", FILMS, ids=[_id(p) for p in FILMS])
def test_gpu_film_matches_golden(gpu, path):
    g = np.load(path)
    sc = _scene(g)
    try:
        film = az.produce_image(sc, seed=int(g["seed"]))
        other = az.produce_image(sc, seed=int(g["seed"]) + 1)   # an independent realisation
    finally:
        sc.close()
    ok, _, relmse = ol.film_compare(film, g["film"], 1e-4)
    _, _, noise = ol.film_compare(other, g["film"], 1e-4)
    assert np.allclose(film[..., 3], g["film"][..., 3], rtol=1e-5, atol=1e-6)
    # same bars as the live parity tests: a last-bit difference (CUDA's versus
    # glibc's transcendental functions) may send a rare path elsewhere
    assert ok >= 0.95 and relmse <= 0.05 * noise


@pytest.mark.gpu
@pytest.mark.parametrize("path", HITS, ids=[_id(p) for p in HITS])
def test_gpu_hits_match_golden(gpu, path):
    g = np.load(path)
    sc = _scene(g)
    try:
        with az.GpuScene(sc) as gs:
            hit, uid, face, t = gs.closest_hit(g["rays"])
    finally:
        sc.close()
    same = (hit == g["hit"]) & (uid == g["uid"]) & (face == g["face"])
    # a mismatch is an exact or near tie between two primitives at the same distance
    near = ~same & (hit == 1) & (g["hit"] == 1) & np.isclose(t, g["t"], rtol=1e-5, atol=1e-7)
    assert (~same & ~near).sum() <= 2
    assert near.sum() <= max(2, int(1e-3 * len(hit)))
    assert np.array_equal(t[same].view(np.uint32), g["t"][same].view(np.uint32))
