"""Per-path radiance parity with azimuth on the benchmark configurations.

Every camera sample's radiance -- the value azimuth's
ProduceImageInLinearSpace hands to ComputeSampleWeight
(src/azimuth_main.cpp:1365-1391) -- from az_gpu_render_samples against
azimuth's own code (oracle/_ref/libazref.so, whose patched ComputeSampleWeight
reports each sample), with the same counter-RNG keys on both sides:

* the Cornell box at its full benchmark size (256x256, 16 spp, depth 5,
  uniform hemisphere sampling: 1,048,576 paths);
* a band of the dense-mesh benchmark frame (the full 1,310,720-triangle
  icosphere, 1024x1024 camera, 8 rows x 512 columns through the icosphere,
  64 spp, depth 8, cosine sampling + area-light NEE: 262,144 paths).

Bar per path: |gpu - ref| <= 1e-4 * max(|ref|, floor) in every channel, floor
= 1e-3 of the mean sample radiance.  Paths above the bar are split by size:
"rounding" (relative error up to 1e-2: CUDA's transcendental functions differ
from glibc's in the last bits, and a path of up to nine vertices compounds
them) and "branch flips" (above 1e-2: some
vertex of the path tree found a different primitive, at a near tie or for a
direction a few ulps off).  Both counts are printed and bounded.
"""
import numpy as np
import pytest

import azimuth_b200 as az
import oracle_lib as ol

pytestmark = pytest.mark.gpu

REL = 1e-4


def per_path(scene, seed, scissor=None):
    import torch
    sc = scissor or ol.scissor_of(scene)
    w, h = scene.resolution()
    rows = min(sc.Max.y, h) - sc.Min.y
    cols = min(sc.Max.x, w) - sc.Min.x
    k = int(np.sqrt(np.float32(scene.sample_count())))
    n = k * k * rows * cols
    with az.GpuScene(scene) as g:
        buf = torch.zeros((n, 4), device="cuda", dtype=torch.float32)
        g.render_samples(buf.data_ptr(), scissor=az.Scissor(az.Vec2u(sc.Max.x, sc.Max.y), az.Vec2u(sc.Min.x, sc.Min.y)),
                         seed=seed)
        torch.cuda.synchronize()
        gpu = buf.cpu().numpy()
    ref = ol.ref_samples(scene, seed=seed, scissor=sc)
    floor = 1e-3 * max(float(np.abs(ref[:, :3]).mean()), 1e-12)
    err = (np.abs(gpu[:, :3] - ref[:, :3]) / np.maximum(np.abs(ref[:, :3]), floor)).max(axis=1)
    ok = err <= REL
    rounding = (err > REL) & (err <= 1e-2)
    flips = err > 1e-2
    return {"paths": n, "within": float(ok.mean()), "rounding": int(rounding.sum()), "flips": int(flips.sum()),
            "max_rounding_err": float(err[rounding].max()) if rounding.any() else 0.0,
            "nonzero": float((np.abs(ref[:, :3]).sum(axis=1) > 0).mean())}


@pytest.mark.skipif(not ol.have_ref(), reason="needs azimuth's compiled code (oracle/_ref)")
def test_per_path_cornell_full_size(gpu):
    scene = az.generate_scene(az.SCENE_CORNELL, seed=0)
    assert scene.resolution() == (256, 256) and scene.sample_count() == 16 and scene.max_depth() == 5
    r = per_path(scene, seed=11)
    print("per-path C0 256x256x16: %s" % r)
    assert r["paths"] == 256 * 256 * 16
    assert r["within"] >= 0.995
    assert r["flips"] <= 0.002 * r["paths"]


@pytest.mark.skipif(not ol.have_ref(), reason="needs azimuth's compiled code (oracle/_ref)")
def test_per_path_dense_mesh_band(gpu):
    scene = az.generate_scene(az.SCENE_DENSE_MESH, seed=0)
    assert scene.triangle_count == 1310732 and scene.resolution() == (1024, 1024)
    sc = ol.scissor_of(scene, rows=(508, 516), cols=(256, 768))
    r = per_path(scene, seed=11, scissor=sc)
    print("per-path C1 band 8x512x64: %s" % r)
    assert r["paths"] == 8 * 512 * 64
    assert r["within"] >= 0.98
    assert r["flips"] <= 0.01 * r["paths"]
