"""Failure paths of the render, made on the host (no GPU fault is involved).

The root of a scene's hierarchy is rewritten so that its first inner child is
the root itself and every child box spans the whole node: every query then
re-enters the root forever.  The traversal is bounded (a step limit per query
and a fixed stack that refuses pushes beyond it), so the kernels stop, flag
the error in the wave counters, and the render returns AZ_ERR_CUDA with the
"corrupt hierarchy" message instead of hanging; the CUDA context stays usable
and a fresh scene renders normally afterwards.  The rewritten child index
points at valid nodes (the root and its real children after it), so every
read stays in bounds.
"""
import ctypes as C

import numpy as np
import pytest

import azimuth_b200 as az

pytestmark = pytest.mark.gpu


def _driver():
    cu = C.CDLL("libcuda.so.1")
    cu.cuMemcpyHtoD_v2.argtypes = [C.c_uint64, C.c_void_p, C.c_size_t]
    cu.cuMemcpyDtoH_v2.argtypes = [C.c_void_p, C.c_uint64, C.c_size_t]
    return cu


def test_looping_hierarchy_returns_corrupt_status(gpu):
    import torch
    torch.zeros(1, device="cuda")   # the primary context is current on this thread
    torch.cuda.synchronize()
    cu = _driver()
    # the dense mesh at 1,280 triangles: one top-level group, whose root queries enter directly
    scene = az.generate_scene(az.SCENE_DENSE_MESH, seed=0, width=8, height=8, spp=1, max_depth=1, detail=3)
    gs = az.GpuScene(scene)
    try:
        arr = gs.arrays()
        root = arr["single_group_root"] if arr["single_group_root"] != 0xFFFFFFFF else arr["tlas_root"]
        assert root != 0xFFFFFFFF and root + 8 <= arr["wide_node_count"]
        node = np.zeros(20, np.uint32)   # one 80-byte wide node
        base = arr["wide_nodes"] + 80 * root
        assert cu.cuMemcpyDtoH_v2(node.ctypes.data, base, 80) == 0
        imask = int(node[3]) >> 24
        assert imask != 0, "the root has inner children"
        # first inner child := the node itself (the others become the real children at root + k), and
        # every child box the whole node (quantised low bounds 0, high bounds 255), so every ray that
        # reaches the root hits the looping child
        node[4] = root
        node[8:14] = 0x00000000
        node[14:20] = 0xFFFFFFFF
        assert cu.cuMemcpyHtoD_v2(base, node.ctypes.data, 80) == 0
        film = torch.zeros((8, 8, 4), device="cuda", dtype=torch.float32)
        with pytest.raises(az.AzError) as ei:
            gs.render_device(film.data_ptr(), seed=1)
        assert ei.value.code == 4   # AZ_ERR_CUDA
        assert b"corrupt hierarchy" in az.lib().az_gpu_last_error()
    finally:
        gs.close()
    # the context is still healthy: a fresh scene renders every sample
    torch.cuda.synchronize()
    with az.GpuScene(scene) as g2:
        film = torch.zeros((8, 8, 4), device="cuda", dtype=torch.float32)
        g2.render_device(film.data_ptr(), seed=1)
        torch.cuda.synchronize()
        assert float(film[..., 3].sum()) > 0.0 and np.isfinite(film.cpu().numpy()).all()
