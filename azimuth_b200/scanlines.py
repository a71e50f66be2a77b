"""One frame over several GPUs, one process per GPU, and one sum of the films.

Two ways to split the frame's camera samples over the ranks:

* "samples" (the default): rank r renders part r of `world` equal ranges of
  the frame's camera-sample sequence (sample number x pixels, pixels
  fastest), i.e. about spp / world samples of every pixel.  Every rank sees
  the whole image, so the ranks carry equal loads whatever the image content.
* "scanlines": azimuth's own split of RenderScene (src/azimuth_main.cpp:
  1815-1867), which hands each host thread a contiguous band of rows, with
  one band per rank.  Bands through expensive geometry (the dense mesh's
  icosphere) load their ranks more than bands of floor and ceiling.

The random numbers of a camera sample are keyed by (seed, pixel, sample), not
by the thread or rank that renders it, so with the same seed on every rank the
summed frame is the frame one GPU renders, up to the order of float additions
(every pixel's samples meet in the sum).  The sum is the only exchange: one
reduce of W*H*16 bytes into rank 0 over NCCL after the parts are rendered.
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


def sample_range(rank, world, total):
    """Camera samples [first, last) of `rank` when `total` samples are split into `world` equal parts, the
    first total % world parts one sample longer (the library's az_render_opts.sample_part arithmetic)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    per, residual = divmod(total, world)
    first = rank * per + min(rank, residual)
    return first, first + per + (1 if rank < residual else 0)


def render_frame_over_ranks(gpu_scene, film, seed=0, group=None, render=None, split="samples"):
    """Renders `rank`'s share of `gpu_scene`'s camera into `film` (a zeroed torch tensor (H, W, 4) float32
    on this rank's GPU) and sums every rank's film into rank 0's; returns the film, which on rank 0 then
    holds the whole frame.  Every rank of `group` calls it with the same seed and split.
    `render(scissor, part, parts)` replaces the GPU render (tests run the exchange on CPU ranks with it)."""
    import torch
    import torch.distributed as dist
    if split not in ("samples", "scanlines"):
        raise ValueError("split must be 'samples' or 'scanlines'")
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    h, w = int(film.shape[0]), int(film.shape[1])
    if split == "scanlines":
        sc, part, parts = band_scissor(w, h, rank, world), 0, 0
    else:
        sc, part, parts = Scissor(Vec2u(w, h), Vec2u(0, 0)), rank, world
    if render is not None:
        render(sc, part, parts)
    else:
        # the render is queued on torch's current stream, which the collective waits for
        gpu_scene.render_device(film.data_ptr(), scissor=sc, seed=seed, sample_part=part, sample_parts=parts,
                                stream=torch.cuda.current_stream(film.device).cuda_stream)
    dist.reduce(film, dst=0, group=group)
    return film
