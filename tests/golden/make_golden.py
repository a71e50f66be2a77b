"""Writes the golden fixtures of tests/golden/ from azimuth's own code.

    python tests/golden/make_golden.py

Needs the compiled reference (oracle/build.py builds oracle/_ref/libazref.so
from the reference sources); the fixtures let the parity tests run where it
is not available.  Every input is a seeded scene of the library's own
generators (azimuth ships no scenes or test vectors):

  film_<scene>.npz      ProduceImageInLinearSpace on one thread (a fixed
                        order of the film sums): film (H, W, 4) float32, and
                        OutputPixelsToFile's colours and bytes of that film
  hits_<scene>.npz      RayEntityIntersection on the scene root for seeded
                        rays: hit flag, UniqueEntityID, face id, t
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

import azimuth_b200 as az  # noqa: E402
import oracle_lib as ol  # noqa: E402

# (name, scene id, generator arguments, render seed)
FILMS = [("cornell", az.SCENE_CORNELL, dict(seed=0, width=32, height=32, spp=4), 3),
         ("features", az.SCENE_FEATURES, dict(seed=2, width=24, height=20, spp=4), 5),
         ("env_spheres", az.SCENE_ENV_SPHERES, dict(seed=1, width=24, height=16, spp=4), 7)]
HITS = [("cornell", az.SCENE_CORNELL, dict(seed=0, width=8, height=8, spp=1), (-1.0, 1.0)),
        ("dense_mesh", az.SCENE_DENSE_MESH, dict(seed=0, width=8, height=8, spp=1, detail=3), (-1.0, 1.0)),
        ("motion_env", az.SCENE_MOTION_ENV, dict(seed=0, width=8, height=8, spp=1, detail=200), (0.0, 10.0))]
TONEMAP = ((0.18, 1.0, 1.0, 1), 1.0 / 2.2, 1)


def rays(n, seed, lo, hi):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d, rng.uniform(0, 1, (n, 1)).astype(np.float32)], axis=1)


def main():
    assert ol.have_ref(), "build the reference first: python oracle/build.py"
    for name, sid, kw, seed in FILMS:
        sc = az.generate_scene(sid, **kw)
        film = ol.ref_film(sc, seed=seed, threads=1)
        rgb, rgb8 = ol.output_pixels(film, *TONEMAP, kind="ref")
        np.savez_compressed(os.path.join(HERE, "film_%s.npz" % name), film=film, rgb=rgb, rgb8=rgb8,
                            scene_id=sid, seed=seed, **{"gen_" + k: v for k, v in kw.items()})
        sc.close()
    for name, sid, kw, span in HITS:
        sc = az.generate_scene(sid, **kw)
        r = rays(2048, sid + 17, *span)
        hit, uid, face, t = ol.closest_hit("ref", sc, r, threads=1)
        np.savez_compressed(os.path.join(HERE, "hits_%s.npz" % name), rays=r, hit=hit, uid=uid, face=face, t=t,
                            scene_id=sid, **{"gen_" + k: v for k, v in kw.items()})
        sc.close()


if __name__ == "__main__":
    main()
