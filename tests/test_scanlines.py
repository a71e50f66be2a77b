"""One frame over several ranks (azimuth_b200.scanlines): RenderScene's
scanline split (src/azimuth_main.cpp:1815-1867) with a band per rank, then one
reduce of the films.  The band arithmetic and the exchange run on CPU gloo
ranks; on the GPU, bands rendered separately must add up to the full frame."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

import azimuth_b200 as az
from azimuth_b200.scanlines import band_scissor, scanline_band

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("height,world", [(1, 1), (7, 2), (1024, 8), (1080, 7), (3, 5)])
def test_bands_cover_every_row_once_like_renderscene(height, world):
    bands = [scanline_band(r, world, height) for r in range(world)]
    assert bands[0][0] == 0 and bands[-1][1] == height
    assert all(a[1] == b[0] for a, b in zip(bands, bands[1:]))
    sizes = [b - a for a, b in bands]
    # RenderScene: height // world rows each, the first height % world threads one more
    assert sizes == [height // world + (1 if r < height % world else 0) for r in range(world)]
    sc = band_scissor(640, height, world - 1, world)
    assert (sc.Min.x, sc.Max.x, sc.Min.y, sc.Max.y) == (0, 640, bands[-1][0], bands[-1][1])


def test_band_of_a_rank_outside_the_world_is_an_error():
    with pytest.raises(ValueError):
        scanline_band(2, 2, 10)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    from azimuth_b200.scanlines import render_frame_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    film = torch.zeros((9, 5, 4), dtype=torch.float32)

    def fake_render(sc):
        # this rank's rows, plus a filter footprint reaching one row into the next band
        film[sc.Min.y:sc.Max.y] += rank + 1.0
        if sc.Max.y < film.shape[0]:
            film[sc.Max.y] += 0.25

    render_frame_over_ranks(None, film, group=None, render=fake_render)
    if rank == 0:
        out["film"] = film.numpy().copy()
    dist.barrier()
    dist.destroy_process_group()


def test_ranks_sum_their_bands_into_rank_zero():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    film = out["film"]
    # 9 rows over 2 ranks: rows 0-4 rank 0 (value 1), rows 5-8 rank 1 (value 2); rank 0's footprint
    # adds 0.25 to row 5
    want = np.array([1, 1, 1, 1, 1, 2.25, 2, 2, 2], np.float32)[:, None, None] * np.ones((9, 5, 4), np.float32)
    assert np.array_equal(film, want)


@pytest.mark.gpu
def test_bands_rendered_apart_add_up_to_the_frame(gpu):
    import torch
    sc = az.generate_scene(az.SCENE_CORNELL, seed=2, width=48, height=37, spp=4, filter=az.FILTER_GAUSSIAN)
    try:
        assert sc.filter_type == az.FILTER_GAUSSIAN   # footprints cross the bands' edges
        w, h = sc.resolution()
        full = torch.zeros((h, w, 4), device="cuda")
        bands = torch.zeros((h, w, 4), device="cuda")
        with az.GpuScene(sc) as g:
            g.render_device(full.data_ptr(), seed=7)
            for r in range(3):
                g.render_device(bands.data_ptr(), scissor=band_scissor(w, h, r, 3), seed=7)
        torch.cuda.synchronize()
        a, b = full.cpu().numpy(), bands.cpu().numpy()
    finally:
        sc.close()
    assert a[..., 3].min() > 0
    # the same samples with the same random numbers; only the order of float additions differs
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6)
