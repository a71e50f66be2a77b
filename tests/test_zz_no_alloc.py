"""The allocation-free render entry point, az_gpu_render_noalloc.

Some callers cannot allocate device memory while they render: code that runs
inside CUDA stream capture (cudaMalloc is not permitted there), hosts whose
caching allocator owns all device memory, and real-time loops on a fixed
memory budget.  For them the render's wave queues live in one static device
array of 8.7 MiB instead of buffers the library allocates.  This file checks,
through the C-ABI, that two calls in a row give the film the regular
az_gpu_render gives (within the 1e-4 relative bar of the parity tests), that
the second call leaves free device memory unchanged, and that a wave larger
than the static array is refused with a clear error.

It is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import azimuth_b200 as az

pytestmark = pytest.mark.gpu


def _noalloc(gs, film, scene, seed, chunk=0):
    o = az.make_opts(scene, seed=seed, device=0, chunk_samples=chunk)
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
