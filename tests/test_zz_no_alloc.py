"""The allocation-free render entry point, az_gpu_render_noalloc.

Some callers cannot allocate device memory while they render: hosts whose
caching allocator has already reserved the GPU's memory (a cudaMalloc from
the library would fail or fragment the host's pool), plug-in hosts that
forbid their plug-ins to allocate, and real-time loops on a fixed memory
budget.  For them the render's wave queues live in one static device array of
8.7 MiB instead of buffers the library allocates.  This file checks, through
the C-ABI, that two calls in a row give the film the regular az_gpu_render
gives (within the 1e-4 relative bar of the parity tests), that the second
call leaves free device memory unchanged, that a wave larger than the static
array is refused with a clear error, that a wave whose queues overflow the
array is run again with fewer samples and still gives the regular film, that
environment importance sampling is honoured and that flags needing buffers of
their own are refused.

It is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import azimuth_b200 as az

pytestmark = pytest.mark.gpu


def _noalloc(gs, film, scene, seed, chunk=0, flags=0):
    o = az.make_opts(scene, seed=seed, device=0, chunk_samples=chunk, flags=flags)
    return az.lib().az_gpu_render_noalloc(gs._h, film.data_ptr(), scene.camera_ptr, scene.epsilons_ptr,
                                          az.full_scissor(scene), scene.filter_type, 0, C.byref(o))


def _rel_err(a, b):
    floor = 1e-3 * max(float(np.abs(b[..., :3]).mean()), 1e-12)
    return float((np.abs(a - b) / np.maximum(np.abs(b), floor)).max())


def test_noalloc_matches_render_on_two_calls(gpu):
    import torch
    # every light type, textures, glossy mirror, dielectric: many tree branches
    # per sample, so the render spans several static waves
    scene = az.generate_scene(az.SCENE_FEATURES, seed=3, width=96, height=80, spp=4)
    w, h = scene.resolution()
    with az.GpuScene(scene) as gs:
        ref = torch.zeros((h, w, 4), device="cuda", dtype=torch.float32)
        gs.render_device(ref.data_ptr(), seed=7, stats=True)
        ref = ref.cpu().numpy()
        assert ref[..., 3].sum() > 0
        free_before = None
        for call in range(2):
            film = torch.zeros((h, w, 4), device="cuda", dtype=torch.float32)
            torch.cuda.synchronize()
            if call == 1:
                free_before = torch.cuda.mem_get_info()[0]
            rc = _noalloc(gs, film, scene, seed=7)
            assert rc == 0, az.lib().az_gpu_last_error()
            torch.cuda.synchronize()
            if call == 1:
                assert torch.cuda.mem_get_info()[0] == free_before
            got = film.cpu().numpy()
            assert np.isfinite(got).all()
            assert _rel_err(got, ref) <= 1e-4


def test_noalloc_refuses_a_wave_beyond_its_static_array(gpu):
    import torch
    scene = az.generate_scene(az.SCENE_CORNELL, seed=0, width=16, height=16, spp=4)
    with az.GpuScene(scene) as gs:
        film = torch.zeros((16, 16, 4), device="cuda", dtype=torch.float32)
        rc = _noalloc(gs, film, scene, seed=1, chunk=16385)
        assert rc == 1
        assert b"16384" in az.lib().az_gpu_last_error()
        assert float(film.abs().sum()) == 0.0
        # the largest allowed wave still renders
        assert _noalloc(gs, film, scene, seed=1, chunk=16384) == 0
        torch.cuda.synchronize()
        assert float(film[..., 3].sum()) == 16 * 16 * 4


def _branching_cornell():
    """Cornell box at 64x64, 4 spp, MaxRecursionDepth 1 whose every material is
    also a mirror and a dielectric: each hit spawns scatter, mirror,
    refraction and reflection rays, four children per sample, more than the
    1.5 queue entries per sample that a wave's queues hold."""
    scene = az.generate_scene(az.SCENE_CORNELL, seed=0, width=64, height=64, spp=4, max_depth=1)
    materials = C.c_void_p.from_address(scene.scene_ptr + 1360).value    # az_scene.Materials
    count = C.c_uint32.from_address(scene.scene_ptr + 2708).value        # az_scene.MaterialCount
    for k in range(count):
        m = materials + 96 * k                                           # az_material, 96 bytes
        (C.c_float * 3).from_address(m + 52)[:] = [0.5, 0.5, 0.5]        # MirrorReflectance
        (C.c_float * 3).from_address(m + 64)[:] = [0.9, 0.9, 0.9]        # Transparency
        C.c_float.from_address(m + 76).value = 1.5                       # RefractionIndex
    return scene


def test_noalloc_reruns_a_wave_whose_queues_overflow(gpu):
    import torch
    scene = _branching_cornell()
    w, h = scene.resolution()
    with az.GpuScene(scene) as gs:
        ref = torch.zeros((h, w, 4), device="cuda", dtype=torch.float32)
        st = gs.render_device(ref.data_ptr(), seed=5, stats=True, chunk_samples=16384)
        # the regular render's queues of the same capacity overflow too
        assert st["retries"] >= 1
        ref = ref.cpu().numpy()
        film = torch.zeros((h, w, 4), device="cuda", dtype=torch.float32)
        rc = _noalloc(gs, film, scene, seed=5, chunk=16384)
        assert rc == 0, az.lib().az_gpu_last_error()
        got = film.cpu().numpy()
        assert float(got[..., 3].sum()) == w * h * 4   # every sample splatted once
        assert _rel_err(got, ref) <= 1e-4


def test_noalloc_environment_importance_and_refused_flags(gpu):
    import torch
    scene = az.generate_scene(az.SCENE_ENV_SPHERES, seed=2, width=48, height=32, spp=4)
    w, h = scene.resolution()
    with az.GpuScene(scene) as gs:
        ref = torch.zeros((h, w, 4), device="cuda", dtype=torch.float32)
        gs.render_device(ref.data_ptr(), seed=9, flags=az.FLAG_ENV_IMPORTANCE)
        plain = torch.zeros((h, w, 4), device="cuda", dtype=torch.float32)
        gs.render_device(plain.data_ptr(), seed=9)
        film = torch.zeros((h, w, 4), device="cuda", dtype=torch.float32)
        rc = _noalloc(gs, film, scene, seed=9, flags=az.FLAG_ENV_IMPORTANCE)
        assert rc == 0, az.lib().az_gpu_last_error()
        got, ref, plain = film.cpu().numpy(), ref.cpu().numpy(), plain.cpu().numpy()
        assert _rel_err(got, ref) <= 1e-4
        assert _rel_err(got, plain) > 1e-3    # the flag changed the estimator
        for flag in (az.FLAG_COUNT_TRAVERSAL, az.FLAG_TIME_STAGES, az.FLAG_ORDER_SHADOW, az.FLAG_ORDER_EXTEND):
            film.zero_()
            assert _noalloc(gs, film, scene, seed=9, flags=flag) == 1
            assert b"az_gpu_render_noalloc does not take" in az.lib().az_gpu_last_error()
            assert float(film.abs().sum()) == 0.0
