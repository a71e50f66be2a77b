"""Many small jobs of one scene: tile waves (az_gpu_render_tiles) against
per-job renders on concurrent streams (az_gpu_render_batch).

    python -m azimuth_b200.tiles_eval [--jobs 256] [--streams 8] [--seed 0]

The scene is the dense-mesh config (1.3 M triangles).  Every job renders the
scene's camera at its own resolution, log-uniform over 32^2 .. 256^2 pixels,
with a square sample count from 1 to 64 and its own seed.  Reported:
aggregate Mpaths/s (all jobs' camera samples / device time) of both forms,
and that every job's film holds the same total filter weight in both.
"""
import argparse
import ctypes as C
import json
import math
import sys

import numpy as np

CAMERA_BYTES = 396              # sizeof(az_camera), include/az_abi.h
RESOLUTION, SAMPLES = 340, 384


def camera_copy(scene, width, height, spp):
    buf = (C.c_ubyte * CAMERA_BYTES)()
    C.memmove(buf, scene.camera_ptr, CAMERA_BYTES)
    addr = C.addressof(buf)
    C.c_uint32.from_address(addr + RESOLUTION).value = width
    C.c_uint32.from_address(addr + RESOLUTION + 4).value = height
    C.c_uint32.from_address(addr + SAMPLES).value = spp
    return buf


def run(n_jobs=256, streams=8, seed=0, log=lambda m: print(m, file=sys.stderr, flush=True)):
    import torch
    import azimuth_b200 as az
    rng = np.random.default_rng(seed)
    scene = az.generate_scene(az.SCENE_DENSE_MESH, seed=seed)
    specs = []
    for j in range(n_jobs):
        pixels = math.exp(rng.uniform(math.log(32 * 32), math.log(256 * 256)))
        w = h = max(8, int(round(math.sqrt(pixels))))
        spp = int(rng.integers(1, 9)) ** 2
        specs.append((w, h, spp, int(seed * 100003 + j)))
    cams = [camera_copy(scene, w, h, spp) for w, h, spp, _ in specs]
    samples = sum(w * h * spp for w, h, spp, _ in specs)
    out = {"jobs": n_jobs, "camera_samples": samples, "scene": "dense mesh, 1,310,720 + 12 triangles"}
    with az.GpuScene(scene) as g:
        def jobs_for(films):
            return [{"gpu_scene": g, "film_ptr": f.data_ptr(), "camera_ptr": C.addressof(c),
                     "scissor": az.Scissor(az.Vec2u(w, h), az.Vec2u(0, 0)), "seed": s}
                    for f, c, (w, h, spp, s) in zip(films, cams, specs)]
        films_b = [torch.zeros((h, w, 4), device="cuda") for w, h, _, _ in specs]
        films_t = [torch.zeros((h, w, 4), device="cuda") for w, h, _, _ in specs]
        # warm-up of both paths on a copy of the job list (queues, graphs)
        az.render_batch(jobs_for(films_b), streams=streams)
        az.render_tiles(jobs_for(films_t))
        for f in films_b + films_t:
            f.zero_()
        torch.cuda.synchronize()
        _, sb = az.render_batch(jobs_for(films_b), streams=streams)
        _, st = az.render_tiles(jobs_for(films_t))
        torch.cuda.synchronize()
        weight_b = np.array([float(f[..., 3].sum()) for f in films_b])
        weight_t = np.array([float(f[..., 3].sum()) for f in films_t])
    out["streams"] = {"streams": streams, "gpu_ms": sb["gpu_ms"], "Mpaths_per_s": samples / sb["gpu_ms"] / 1e3,
                      "p50_ms": sb["p50_ms"], "p99_ms": sb["p99_ms"]}
    out["tiles"] = {"gpu_ms": st["gpu_ms"], "Mpaths_per_s": samples / st["gpu_ms"] / 1e3,
                    "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"]}
    out["same_filter_weight"] = bool(np.allclose(weight_b, weight_t, rtol=1e-5))
    log("tiles %.1f Mpaths/s vs streams %.1f Mpaths/s" % (out["tiles"]["Mpaths_per_s"],
                                                          out["streams"]["Mpaths_per_s"]))
    scene.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=256)
    ap.add_argument("--streams", type=int, default=8)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    print(json.dumps(run(args.jobs, args.streams, args.seed)))


if __name__ == "__main__":
    main()
