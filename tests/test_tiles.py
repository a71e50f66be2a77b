"""az_gpu_render_tiles: jobs rendered together in shared waves, every wave's
camera kernel pulling 4096-sample tiles of all jobs from a device work queue.
Each job's film must equal what az_gpu_render adds for that job alone (same
seed, same samples; only the order of float atomics differs), for jobs that
differ in camera, resolution, spp, scissor, filter and seed, and for jobs of
different scenes in the same waves (every queue entry carries its scene)."""
import ctypes as C

import numpy as np
import pytest

import azimuth_b200 as az
import oracle_lib as ol

CAMERA_BYTES = 396          # sizeof(az_camera), include/az_abi.h
RESOLUTION, SAMPLES = 340, 384


def camera_copy(scene, width, height, spp):
    """A copy of the scene's camera with another resolution and sample count."""
    buf = (C.c_ubyte * CAMERA_BYTES)()
    C.memmove(buf, scene.camera_ptr, CAMERA_BYTES)
    addr = C.addressof(buf)
    C.c_uint32.from_address(addr + RESOLUTION).value = width
    C.c_uint32.from_address(addr + RESOLUTION + 4).value = height
    C.c_uint32.from_address(addr + SAMPLES).value = spp
    return buf


def test_header_declares_the_entry_point():
    assert hasattr(az.lib(), "az_gpu_render_tiles") and callable(az.render_tiles)


@pytest.mark.gpu
@pytest.mark.parametrize("scene_id", [az.SCENE_CORNELL, az.SCENE_FEATURES])
def test_tile_render_gives_every_job_its_own_render(gpu, scene_id):
    import torch
    sc = az.generate_scene(scene_id, seed=4, width=40, height=30, spp=4)
    try:
        cams = [None, camera_copy(sc, 57, 21, 9), camera_copy(sc, 8, 8, 1), camera_copy(sc, 96, 70, 16)]
        specs = []   # (camera buffer or None, width, height, scissor or None, filter, seed)
        full = lambda w, h: az.Scissor(az.Vec2u(w, h), az.Vec2u(0, 0))   # noqa: E731
        specs.append((None, 40, 30, None, sc.filter_type, 11))
        specs.append((cams[1], 57, 21, full(57, 21), az.FILTER_GAUSSIAN, 12))
        specs.append((cams[2], 8, 8, full(8, 8), az.FILTER_BOX, 13))
        specs.append((cams[3], 96, 70, az.Scissor(az.Vec2u(90, 61), az.Vec2u(5, 3)), az.FILTER_BOX, 14))
        specs.append((None, 40, 30, az.Scissor(az.Vec2u(40, 12), az.Vec2u(0, 0)), az.FILTER_GAUSSIAN, 15))
        with az.GpuScene(sc) as g:
            tiled, alone, jobs = [], [], []
            for cam, w, h, scis, filt, seed in specs:
                f = torch.zeros((h, w, 4), device="cuda")
                tiled.append(f)
                job = {"gpu_scene": g, "film_ptr": f.data_ptr(), "filter_type": filt, "seed": seed}
                if cam is not None:
                    job["camera_ptr"] = C.addressof(cam)
                if scis is not None:
                    job["scissor"] = scis
                jobs.append(job)
                a = torch.zeros((h, w, 4), device="cuda")
                g.render_device(a.data_ptr(), camera_ptr=C.addressof(cam) if cam is not None else None,
                                scissor=scis, filter_type=filt, seed=seed)
                alone.append(a)
            torch.cuda.synchronize()
            # a small wave size, so that waves hold tiles of several jobs and jobs span waves
            per, stats = az.render_tiles(jobs, chunk_samples=3 * 4096)
            torch.cuda.synchronize()
        want_samples = [40 * 30 * 4, 57 * 21 * 9, 8 * 8 * 1, 85 * 58 * 16, 40 * 12 * 4]
        assert [p["samples"] for p in per] == want_samples and stats["samples"] == sum(want_samples)
        assert all(p["status"] == 0 for p in per) and stats["gpu_ms"] > 0
        assert max(p["done_ms"] for p in per) <= stats["gpu_ms"] + 1e-3
        for k, (t, a) in enumerate(zip(tiled, alone)):
            t, a = t.cpu().numpy(), a.cpu().numpy()
            assert a[..., 3].sum() > 0, k
            assert ol.film_compare(t, a, 1e-4)[0] == 1.0, k
    finally:
        sc.close()


@pytest.mark.gpu
def test_tile_render_of_several_scenes_gives_every_job_its_own_render(gpu):
    import torch
    # the benchmark generators' scenes (small sizes): Cornell box (uniform sampling, box filter,
    # depth 5), dense mesh (7 BRDFs, cosine sampling, Gaussian filter, depth 8), moving spheres with an
    # HDR map (dielectrics, environment light, depth 12), plus the features scene (textures, every
    # light type) and a second Cornell box of another depth
    specs = [(az.SCENE_CORNELL, dict(width=40, height=30, spp=4)),
             (az.SCENE_DENSE_MESH, dict(width=48, height=36, spp=4, detail=4)),
             (az.SCENE_MOTION_ENV, dict(width=64, height=36, spp=4, detail=300)),
             (az.SCENE_FEATURES, dict(width=32, height=24, spp=9)),
             (az.SCENE_CORNELL, dict(width=24, height=24, spp=16, max_depth=9))]
    scenes = [az.generate_scene(sid, seed=7 + k, **kw) for k, (sid, kw) in enumerate(specs)]
    gss = [az.GpuScene(s) for s in scenes]
    try:
        tiled, alone, jobs = [], [], []
        for k, (s, g) in enumerate(zip(scenes, gss)):
            w, h = s.resolution()
            f = torch.zeros((h, w, 4), device="cuda")
            tiled.append(f)
            jobs.append({"gpu_scene": g, "film_ptr": f.data_ptr(), "seed": 20 + k})
            a = torch.zeros((h, w, 4), device="cuda")
            g.render_device(a.data_ptr(), seed=20 + k)
            alone.append(a)
        # the second job twice more, with other seeds: one scene for several jobs of the wave
        for k in (1, 2):
            w, h = scenes[1].resolution()
            f = torch.zeros((h, w, 4), device="cuda")
            tiled.append(f)
            jobs.append({"gpu_scene": gss[1], "film_ptr": f.data_ptr(), "seed": 40 + k})
            a = torch.zeros((h, w, 4), device="cuda")
            gss[1].render_device(a.data_ptr(), seed=40 + k)
            alone.append(a)
        torch.cuda.synchronize()
        # small waves: every wave holds tiles of several scenes
        per, stats = az.render_tiles(jobs, chunk_samples=2 * 4096)
        torch.cuda.synchronize()
        assert all(p["status"] == 0 for p in per)
        for k, (t, a) in enumerate(zip(tiled, alone)):
            t, a = t.cpu().numpy(), a.cpu().numpy()
            assert a[..., 3].sum() > 0, k
            assert ol.film_compare(t, a, 1e-4)[0] == 1.0, k
    finally:
        for g in gss:
            g.close()
        for s in scenes:
            s.close()


@pytest.mark.gpu
def test_tile_render_rejects_guides(gpu):
    import torch
    a = az.generate_scene(az.SCENE_CORNELL, seed=1, width=16, height=16, spp=1)
    try:
        with az.GpuScene(a) as ga:
            f = torch.zeros((16, 16, 4), device="cuda")
            with az.Guide(ga) as guide:
                with pytest.raises(az.AzError):
                    az.render_tiles([{"gpu_scene": ga, "film_ptr": f.data_ptr(), "guide": guide}])
    finally:
        a.close()


def test_tile_entry_checks_its_arguments_before_the_device():
    lib = az.lib()
    st = az.BatchStats()
    assert lib.az_gpu_render_tiles(None, 0, None, C.byref(st)) == 0          # nothing to render
    assert lib.az_gpu_render_tiles(None, 3, None, C.byref(st)) != 0          # jobs missing
    jobs = (az.Job * 1)()                                                    # a job without a scene
    assert lib.az_gpu_render_tiles(jobs, 1, None, C.byref(st)) != 0
