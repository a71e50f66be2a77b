"""Batched jobs and graph replay of the wave launches: each job's film equals
the film of the same render made on its own."""
import numpy as np
import pytest

import azimuth_b200 as az
import oracle_lib as ol

pytestmark = pytest.mark.gpu


def test_graph_replay_renders_the_same_film(gpu):
    import torch
    scene = az.generate_scene(az.SCENE_FEATURES, seed=4, width=40, height=32, spp=9)
    w, h = scene.resolution()
    with az.GpuScene(scene) as g:
        stream = torch.cuda.Stream()           # graphs are captured on a non-default stream
        films = []
        for flags in (az.FLAG_NO_GRAPH, 0, 0):
            f = torch.zeros((h, w, 4), device="cuda")
            # 1000-sample waves: the graph is replayed for every wave (and the seed changes per call)
            st = g.render_device(f.data_ptr(), seed=9, stream=stream.cuda_stream, stats=True, flags=flags,
                                 chunk_samples=1024)
            assert st["chunks"] >= 10
            films.append(f.cpu().numpy())
        for f in films[1:]:
            assert ol.film_compare(f, films[0], 1e-4)[0] == 1.0
        # another seed through the same captured graph
        f2 = torch.zeros((h, w, 4), device="cuda")
        g.render_device(f2.data_ptr(), seed=10, stream=stream.cuda_stream, chunk_samples=1024)
        f3 = torch.zeros((h, w, 4), device="cuda")
        g.render_device(f3.data_ptr(), seed=10, stream=stream.cuda_stream, chunk_samples=1024, flags=az.FLAG_NO_GRAPH)
        assert ol.film_compare(f2.cpu().numpy(), f3.cpu().numpy(), 1e-4)[0] == 1.0
        assert ol.film_compare(f2.cpu().numpy(), films[0], 1e-4)[0] < 0.9   # different samples


@pytest.mark.parametrize("tiles", [False, True], ids=["streams", "tile_waves"])
def test_batch_jobs_equal_their_own_renders(gpu, tiles):
    import torch
    rng = np.random.default_rng(5)
    specs = [(az.SCENE_CORNELL, dict(width=64, height=48, spp=4)),
             (az.SCENE_DENSE_MESH, dict(width=96, height=64, spp=16, detail=3)),
             (az.SCENE_FEATURES, dict(width=32, height=32, spp=1)),
             (az.SCENE_MOTION_ENV, dict(width=80, height=45, spp=4, detail=300, env_width=64, env_height=32)),
             (az.SCENE_INTERIOR, dict(width=48, height=27, spp=9, detail=3)),
             (az.SCENE_CORNELL, dict(width=200, height=120, spp=36))]
    scenes, gscenes, films, jobs = [], [], [], []
    for k, (sid, kw) in enumerate(specs):
        sc = az.generate_scene(sid, seed=k, **kw)
        gs = az.GpuScene(sc)
        w, h = sc.resolution()
        f = torch.zeros((h, w, 4), device="cuda")
        scenes.append(sc)
        gscenes.append(gs)
        films.append(f)
        jobs.append({"gpu_scene": gs, "film_ptr": f.data_ptr(), "seed": int(rng.integers(1 << 30))})
    guide = az.Guide(gscenes[4], seed=3)
    jobs[4]["guide"] = guide
    # tiles: the five plain jobs (five scenes) share tile waves on one stream, the guided job runs beside
    per, st = az.render_batch(jobs, streams=3, chunk_samples=4096, tiles=tiles)
    assert st["jobs"] == len(jobs) and st["failed"] == 0 and st["streams"] == 3
    assert all(p["status"] == 0 for p in per)
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["gpu_ms"] + 1e-3
    assert st["samples"] == sum(p["samples"] for p in per)
    for k, j in enumerate(jobs):
        w, h = scenes[k].resolution()
        ref = torch.zeros((h, w, 4), device="cuda")
        if k == 4:
            guide.render(ref.data_ptr(), train=False, seed=j["seed"], chunk_samples=4096)
        else:
            gscenes[k].render_device(ref.data_ptr(), seed=j["seed"], chunk_samples=4096)
        ok = ol.film_compare(films[k].cpu().numpy(), ref.cpu().numpy(), 1e-4)[0]
        assert ok == 1.0, (k, ok)
    guide.close()
    for gs in gscenes:
        gs.close()
