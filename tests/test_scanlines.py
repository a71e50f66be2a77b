"""One frame over several ranks (azimuth_b200.scanlines): equal ranges of the
camera-sample sequence per rank (the default) or RenderScene's scanline split
(src/azimuth_main.cpp:1815-1867) with a band per rank, then one reduce of the
films.  The split arithmetic and the exchange run on CPU gloo ranks; on the
GPU, parts rendered separately must add up to the full frame."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

import azimuth_b200 as az
from azimuth_b200.scanlines import band_scissor, sample_range, scanline_band

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
    with pytest.raises(ValueError):
        sample_range(3, 3, 10)


@pytest.mark.parametrize("total,world", [(1, 1), (10, 3), (1024 * 1024 * 64, 8), (5, 7)])
def test_sample_ranges_cover_every_sample_once_and_balance(total, world):
    parts = [sample_range(r, world, total) for r in range(world)]
    assert parts[0][0] == 0 and parts[-1][1] == total
    assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
    sizes = [b - a for a, b in parts]
    assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out, split):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    from azimuth_b200.scanlines import render_frame_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    film = torch.zeros((9, 5, 4), dtype=torch.float32)

    def fake_render(sc, part, parts):
        if split == "scanlines":
            # this rank's rows, plus a filter footprint reaching one row into the next band
            assert parts == 0
            film[sc.Min.y:sc.Max.y] += rank + 1.0
            if sc.Max.y < film.shape[0]:
                film[sc.Max.y] += 0.25
        else:
            # every pixel, this rank's share of its samples
            assert (sc.Min.y, sc.Max.y, sc.Min.x, sc.Max.x) == (0, 9, 0, 5) and (part, parts) == (rank, world)
            film.add_(10.0 ** rank)

    render_frame_over_ranks(None, film, group=None, render=fake_render, split=split)
    if rank == 0:
        out["film"] = film.numpy().copy()
    dist.barrier()
    dist.destroy_process_group()


def _run_ranks(world, split):
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out, split)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return out["film"]


def test_ranks_sum_their_sample_parts_into_rank_zero():
    film = _run_ranks(2, "samples")
    # both ranks render every pixel: 1 + 10
    assert np.array_equal(film, np.full((9, 5, 4), 11.0, np.float32))


def test_ranks_sum_their_bands_into_rank_zero():
    film = _run_ranks(2, "scanlines")
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


@pytest.mark.gpu
def test_sample_parts_rendered_apart_add_up_to_the_frame(gpu):
    import torch
    sc = az.generate_scene(az.SCENE_CORNELL, seed=2, width=48, height=37, spp=9, filter=az.FILTER_GAUSSIAN)
    try:
        w, h = sc.resolution()
        full = torch.zeros((h, w, 4), device="cuda")
        parts = torch.zeros((h, w, 4), device="cuda")
        with az.GpuScene(sc) as g:
            st = g.render_device(full.data_ptr(), seed=7, stats=True)
            n = 0
            for r in range(4):
                s = g.render_device(parts.data_ptr(), seed=7, stats=True, sample_part=r, sample_parts=4)
                first, last = sample_range(r, 4, w * h * 9)
                assert s["samples"] == last - first
                n += s["samples"]
            assert n == st["samples"] == w * h * 9
            with pytest.raises(az.AzError):
                g.render_device(parts.data_ptr(), seed=7, sample_part=4, sample_parts=4)
        torch.cuda.synchronize()
        a, b = full.cpu().numpy(), parts.cpu().numpy()
    finally:
        sc.close()
    assert a[..., 3].min() > 0
    # the same samples with the same random numbers; only the order of float additions differs
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6)
