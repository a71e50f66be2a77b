"""The scene build on the GPU (LBVH, wide collapse, primitive gather):
az_gpu_scene_info's figures, the effect of the hierarchy's shape, and that two
builds of one scene are identical (same nearest hits, bit for bit)."""
import numpy as np
import pytest

import azimuth_b200 as az

pytestmark = pytest.mark.gpu


def _rays(n, seed, lo=-1.0, hi=1.0):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    t = rng.uniform(0.0, 1.0, (n, 1)).astype(np.float32)
    return np.concatenate([o, d, t], axis=1)


@pytest.fixture(scope="module")
def dense():
    sc = az.generate_scene(az.SCENE_DENSE_MESH, seed=0, width=64, height=64, spp=1, detail=5)
    yield sc
    sc.close()


def test_scene_info_reports_the_build(gpu, dense):
    with az.GpuScene(dense) as g:
        info = g.info()
    assert info["triangles"] == dense.triangle_count
    assert info["spheres"] == dense.sphere_count
    assert info["bvh_width"] == 8 and info["bvh_leaf"] == 2
    # every wide node holds at least two children, so there are fewer nodes than triangles
    assert 0 < info["wide_nodes"] < info["triangles"]
    assert info["bvh_depth"] >= 2 and info["hierarchies"] >= 2
    # 48 + 80 bytes per triangle plus 80 per node at least; build scratch is freed
    assert info["device_bytes"] >= info["triangles"] * 128 + info["wide_nodes"] * 80
    assert info["device_bytes"] < info["triangles"] * 400 + (64 << 20)
    assert info["bvh_ms"] > 0.0 and info["total_ms"] >= info["bvh_ms"]


def test_wider_nodes_make_a_shallower_hierarchy(gpu, dense):
    got = {}
    for w in (2, 4, 8):
        with az.GpuScene(dense, bvh_width=w) as g:
            got[w] = g.info()
    assert got[2]["wide_nodes"] > got[4]["wide_nodes"] > got[8]["wide_nodes"]
    assert got[2]["bvh_depth"] > got[4]["bvh_depth"] > got[8]["bvh_depth"]
    # binary nodes: about one per leaf of <= 2 triangles
    assert got[2]["wide_nodes"] >= got[2]["triangles"] // 2 - 1
    for leaf in (1, 3):
        with az.GpuScene(dense, bvh_leaf=leaf) as g:
            info = g.info()
        assert (info["wide_nodes"] > got[8]["wide_nodes"]) == (leaf == 1)


@pytest.mark.parametrize("scene_id", [az.SCENE_CORNELL, az.SCENE_DENSE_MESH, az.SCENE_MOTION_ENV, az.SCENE_INTERIOR])
def test_two_builds_give_identical_hits(gpu, scene_id):
    kw = {"detail": 4} if scene_id in (az.SCENE_DENSE_MESH, az.SCENE_INTERIOR) else {}
    sc = az.generate_scene(scene_id, seed=3, width=32, height=32, spp=1, **kw)
    try:
        span = {az.SCENE_MOTION_ENV: (0.0, 10.0), az.SCENE_INTERIOR: (0.5, 3.5)}.get(scene_id, (-1.0, 1.0))
        rays = _rays(1 << 15, seed=scene_id, lo=span[0], hi=span[1])
        outs = []
        for _ in range(2):
            with az.GpuScene(sc) as g:
                outs.append((g.info()["wide_nodes"],) + g.closest_hit(rays))
        assert outs[0][0] == outs[1][0]
        for a, b in zip(outs[0][1:], outs[1][1:]):
            assert np.array_equal(a, b)
        assert outs[0][1].any()   # the rays do hit something
    finally:
        sc.close()


@pytest.mark.parametrize("scene_id", [az.SCENE_DENSE_MESH, az.SCENE_MOTION_ENV])
def test_ploc_and_lbvh_find_the_same_hits(gpu, scene_id):
    kw = {"detail": 5} if scene_id == az.SCENE_DENSE_MESH else {}
    sc = az.generate_scene(scene_id, seed=5, width=32, height=32, spp=1, **kw)
    try:
        span = (0.0, 10.0) if scene_id == az.SCENE_MOTION_ENV else (-1.0, 1.0)
        rays = _rays(1 << 15, seed=11, lo=span[0], hi=span[1])
        with az.GpuScene(sc, bvh_builder=az.BVH_LBVH) as a, az.GpuScene(sc, bvh_builder=az.BVH_PLOC) as b:
            assert a.info()["bvh_builder"] == az.BVH_LBVH and b.info()["bvh_builder"] == az.BVH_PLOC
            ha, hb = a.closest_hit(rays), b.closest_hit(rays)
        same = (ha[0] == hb[0]) & (ha[1] == hb[1]) & (ha[2] == hb[2]) & (ha[3] == hb[3])
        assert same.mean() >= 0.999
        assert np.array_equal(ha[3][~same], hb[3][~same])   # exact-distance ties only
    finally:
        sc.close()


def test_ploc_visits_fewer_nodes(gpu, dense):
    import torch
    w, h = dense.resolution()
    film = torch.zeros((h, w, 4), device="cuda")
    visits = {}
    for builder in (az.BVH_LBVH, az.BVH_PLOC):
        with az.GpuScene(dense, bvh_builder=builder) as g:
            st = g.render_device(film.data_ptr(), seed=1, stats=True, flags=az.FLAG_COUNT_TRAVERSAL)
            visits[builder] = (st["node_visits"] + st["prim_visits"] + st["shadow_node_visits"] +
                               st["shadow_prim_visits"]) / (st["extend_rays"] + st["shadow_rays"])
    assert visits[az.BVH_PLOC] < visits[az.BVH_LBVH]
