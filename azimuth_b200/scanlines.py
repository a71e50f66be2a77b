"""One frame over several GPUs: azimuth's scanline split of RenderScene
(src/azimuth_main.cpp:1815-1867), which hands each host thread a band of
rows, with one band per rank (one process per GPU) instead, then one sum of the
bands' films into rank 0's film.

The random numbers of a camera sample are keyed by (seed, pixel, sample), not
by the thread or rank that renders it, so with the same seed on every rank the
assembled frame is the frame one GPU renders (up to the order of float
additions where a band's filter footprint reaches into its neighbour's rows:
those contributions meet in the sum).  The sum is the only exchange: one
reduce of W*H*16 bytes over NCCL after the bands are rendered.
"""
from ._native import Scissor, Vec2u


def scanline_band(rank, world, height):
    """Rows [first, last) of `rank`: RenderScene's split of `height` rows over `world` workers, the first
    height % world of them one row more (src/azimuth_main.cpp:1823-1835)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    per, residual = divmod(height, world)
    first = rank * per + min(rank, residual)
    return first, first + per + (1 if rank < residual else 0)


def band_scissor(width, height, rank, world):
    """The az_scissor of `rank`'s band: all columns of its rows."""
    first, last = scanline_band(rank, world, height)
    return Scissor(Vec2u(width, last), Vec2u(0, first))


def render_frame_over_ranks(gpu_scene, film, seed=0, group=None, render=None):
    """Renders `rank`'s band of `gpu_scene`'s camera into `film` (a zeroed torch tensor (H, W, 4) float32
    on this rank's GPU) and sums every rank's film into rank 0's; returns the film, which on rank 0 then
    holds the whole frame.  Every rank of `group` calls it with the same seed.  `render(scissor)`
    replaces the GPU render (tests run the exchange on CPU ranks with it)."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    h, w = int(film.shape[0]), int(film.shape[1])
    sc = band_scissor(w, h, rank, world)
    if render is not None:
        render(sc)
    else:
        # the render is queued on torch's current stream, which the collective waits for
        gpu_scene.render_device(film.data_ptr(), scissor=sc, seed=seed,
                                stream=torch.cuda.current_stream(film.device).cuda_stream)
    dist.reduce(film, dst=0, group=group)
    return film
