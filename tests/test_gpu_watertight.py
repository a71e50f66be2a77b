"""The watertight triangle test (AZ_FLAG_WATERTIGHT), the production
alternative to azimuth's Cramer test (src/azimuth_main.cpp:147-243).

* Rays from inside the closed, displaced icosphere of the dense-mesh scene,
  aimed exactly at its vertices and at the midpoints of its edges -- where a
  ray meets two to six triangles at a shared edge or vertex -- must all hit
  the icosphere: none may slip between its triangles to the walls behind.
  The same rays under the Cramer test are counted too (its -1e-6 barycentric
  tolerance also closes most gaps, by overlapping neighbours instead).
* On random rays the two tests must find the same primitives, except where two
  primitives lie at the same distance (a shared edge or vertex, where each
  test may keep a different one), and the distances agree to float rounding
  (99.9% within 1e-5 relative; grazing hits, where the two formulas divide by
  a small determinant, within 1e-2).
* A watertight render of the dense mesh matches the Cramer render pixel for
  pixel up to the few paths that take the other side of a tie.
"""
import numpy as np
import pytest

import azimuth_b200 as az
from test_gpu_closest_hit import random_rays

pytestmark = pytest.mark.gpu

ICOSPHERE_UIDS = set(range(4, 11))   # the seven per-BRDF meshes of the icosphere


def _targets(scene):
    """Icosphere centre, its vertices and the midpoints of its edges (float64)."""
    v, f, _, descs = scene.soup_arrays()
    ico = [d for d in descs if d["unique_entity_id"] in ICOSPHERE_UIDS]
    assert len(ico) == 7 and all(np.allclose(np.array(d["transform"]).reshape(4, 4), np.eye(4)) for d in ico)
    faces = np.concatenate([f[d["face_base"]:d["face_base"] + d["face_count"]] for d in ico])
    used = np.unique(faces)
    verts = v[used].astype(np.float64)
    centre = verts.mean(axis=0)
    edges = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
    edges = np.unique(np.sort(edges, axis=1), axis=0)
    mids = 0.5 * (v[edges[:, 0]].astype(np.float64) + v[edges[:, 1]].astype(np.float64))
    return centre, verts, mids


def _rays_towards(centre, pts):
    d = pts - centre
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    o = np.broadcast_to(centre, d.shape)
    return np.concatenate([o, d, np.zeros((len(d), 1))], axis=1).astype(np.float32)


def test_rays_through_shared_vertices_and_edges_never_escape(gpu):
    scene = az.generate_scene(az.SCENE_DENSE_MESH, seed=5, width=8, height=8, spp=1, detail=5)
    centre, verts, mids = _targets(scene)
    rays = _rays_towards(centre, np.concatenate([verts, mids]))
    with az.GpuScene(scene) as g:
        wh, wu, _, _ = g.closest_hit(rays, flags=az.FLAG_WATERTIGHT)
        ch, cu, _, _ = g.closest_hit(rays)
    escaped_wt = int(((wh == 0) | ~np.isin(wu, list(ICOSPHERE_UIDS))).sum())
    escaped_cr = int(((ch == 0) | ~np.isin(cu, list(ICOSPHERE_UIDS))).sum())
    print("watertight: %d rays at %d vertices and %d edge midpoints; escaped: watertight %d, Cramer %d" % (
        len(rays), len(verts), len(mids), escaped_wt, escaped_cr))
    assert escaped_wt == 0


@pytest.mark.parametrize("name,sid,kw,lo,hi", [
    ("cornell", az.SCENE_CORNELL, {}, (-0.45, 0.05, -0.45), (0.45, 0.95, 0.45)),
    ("dense_mesh", az.SCENE_DENSE_MESH, dict(detail=6), (-0.45, 0.05, -0.45), (0.45, 0.95, 0.45)),
    ("interior", az.SCENE_INTERIOR, dict(detail=8), (0.5, 0.2, 0.5), (24.0, 3.8, 7.5)),
], ids=["cornell", "dense_mesh", "interior"])
def test_watertight_ids_agree_with_cramer(gpu, name, sid, kw, lo, hi):
    scene = az.generate_scene(sid, seed=5, width=8, height=8, spp=1, **kw)
    rays = random_rays(200000, lo, hi, seed=7 + len(name))
    with az.GpuScene(scene) as g:
        wh, wu, wf, wt = g.closest_hit(rays, flags=az.FLAG_WATERTIGHT)
        ch, cu, cf, ct = g.closest_hit(rays)
    both = (wh == 1) & (ch == 1)
    same = both & (wu == cu) & (wf == cf)
    differ = (wh != ch) | (both & ~same)
    tie = both & ~same & (np.abs(wt - ct) <= 1e-5 * np.maximum(np.abs(ct), 1e-6))
    print("watertight vs Cramer, %s: %d rays, %d hits, differing ids %d (at equal distance %d)" % (
        name, len(rays), int(ch.sum()), int(differ.sum()), int(tie.sum())))
    assert (differ & ~tie).sum() <= max(2, int(2e-5 * len(rays)))
    assert tie.sum() <= int(1e-3 * len(rays))
    # the same distance up to rounding (a few ulps), more at grazing incidence
    rel = np.abs(wt[same].astype(np.float64) - ct[same]) / np.maximum(np.abs(ct[same]), 1e-6)
    print("  relative distance difference: median %.2e, 99.9%% %.2e, max %.2e" % (
        np.median(rel), np.quantile(rel, 0.999), rel.max()))
    assert np.quantile(rel, 0.999) <= 1e-5 and rel.max() <= 1e-2


def test_watertight_render_matches_cramer(gpu):
    import torch
    scene = az.generate_scene(az.SCENE_DENSE_MESH, seed=1, width=64, height=64, spp=4, detail=6)
    w, h = scene.resolution()
    films = []
    with az.GpuScene(scene) as g:
        for flags in (0, az.FLAG_WATERTIGHT):
            film = torch.zeros((h, w, 4), device="cuda")
            st = g.render_device(film.data_ptr(), seed=3, stats=True, flags=flags)
            assert st["samples"] == w * h * 4
            films.append(film.cpu().numpy())
    a, b = films
    assert np.isfinite(b).all() and np.allclose(a[..., 3], b[..., 3], rtol=1e-5)
    floor = 1e-3 * float(np.abs(a[..., :3]).mean())
    err = (np.abs(b - a)[..., :3] / np.maximum(np.abs(a[..., :3]), floor)).max(axis=-1)
    print("watertight render: pixels within 1e-3 of the Cramer render: %.4f" % float((err <= 1e-3).mean()))
    assert (err <= 1e-3).mean() >= 0.97
