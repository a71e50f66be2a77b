"""Batched uneven render jobs (config 4) through az_gpu_render_batch.

    python -m azimuth_b200.batch_eval [--jobs 256] [--streams 8] [--seed 0]

Each job draws its scene uniformly from the generators of configs 0-2
(Cornell box; dense mesh with a 1.3 M-triangle icosphere; 10,000 moving
spheres with an HDR environment map) with its own seed; resolution
log-uniform over 64^2 .. 1024^2 pixels with aspect ratio uniform in
[1, 16/9]; samples per pixel log-uniform in [1, 256] (azimuth renders the
largest square at or below); depth uniform in 5..16; odd jobs render with a
path guide that trains while rendering.  Scene generation and upload happen
before the timed batch.  Reported: aggregate Mpaths/s (all jobs' camera
samples / device time from the batch start to the last completion), job
completion-time p50 / p99 (jobs shortest first on `--streams` streams), the
same batch largest first and on one stream for comparison, and the batch with
its plain jobs in multi-scene tile waves (one persistent chain of launches
pulling 4096-sample tiles of every plain job from a device work queue) while
the other streams take the guided jobs.  After the tile-wave batch, eight of
its plain jobs are rendered again one at a time (a batch of one job) and the
relMSE of each tile-wave film against that film is reported: the tile waves
trace the same samples, so the images agree to float summation order.
"""
import argparse
import json
import math
import sys
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np


def job_specs(n, seed):
    rng = np.random.default_rng(seed)
    specs = []
    for j in range(n):
        pixels = math.exp(rng.uniform(math.log(64 * 64), math.log(1024 * 1024)))
        aspect = rng.uniform(1.0, 16.0 / 9.0)
        h = max(8, int(round(math.sqrt(pixels / aspect))))
        w = max(8, int(round(h * aspect)))
        spp = int(round(math.exp(rng.uniform(0.0, math.log(256.0)))))
        depth = int(rng.integers(5, 17))
        specs.append({"config": int(rng.integers(0, 3)), "seed": int(seed * 100003 + j), "width": w, "height": h,
                      "spp": max(1, spp), "max_depth": depth, "guided": j % 2 == 1})
    return specs


def run(n_jobs=256, streams=8, seed=0, log=lambda m: print(m, file=sys.stderr, flush=True)):
    import torch
    import azimuth_b200 as az
    import ctypes as C
    specs = job_specs(n_jobs, seed)
    t0 = time.time()

    def prepare(s):
        # generate, upload, keep copies of the camera and epsilons, release the host scene
        sc = az.generate_scene(s["config"], seed=s["seed"], width=s["width"], height=s["height"], spp=s["spp"],
                               max_depth=s["max_depth"])
        gs = az.GpuScene(sc)
        cam = C.create_string_buffer(C.string_at(sc.camera_ptr, 396), 396)
        eps = C.create_string_buffer(C.string_at(sc.epsilons_ptr, 8), 8)
        info = {"resolution": sc.resolution(), "filter_type": sc.filter_type, "triangles": int(sc.triangle_count),
                "spheres": int(sc.sphere_count), "scissor": az.full_scissor(sc)}
        sc.close()
        return gs, cam, eps, info
    with ThreadPoolExecutor(max_workers=8) as ex:
        prepared = list(ex.map(prepare, specs))
    gen_s = time.time() - t0
    upload_s = 0.0
    log("generated and uploaded %d scenes in %.1f s" % (n_jobs, gen_s))
    gscenes = [p[0] for p in prepared]
    films, guides, jobs = [], [], []
    for k, (s, (gs, cam, eps, info)) in enumerate(zip(specs, prepared)):
        w, h = info["resolution"]
        f = torch.zeros((h, w, 4), device="cuda")
        films.append(f)
        j = {"gpu_scene": gs, "film_ptr": f.data_ptr(), "seed": s["seed"], "camera_ptr": C.addressof(cam),
             "epsilons_ptr": C.addressof(eps), "filter_type": info["filter_type"], "scissor": info["scissor"],
             "_keep": (cam, eps)}
        if s["guided"]:
            gd = az.Guide(gs, seed=s["seed"])
            guides.append(gd)
            j["guide"] = gd
            j["train"] = True
        jobs.append(j)
    torch.cuda.synchronize()
    out = {"jobs": n_jobs, "generate_and_upload_s": gen_s,
           "triangles": int(sum(p[3]["triangles"] for p in prepared)),
           "spheres": int(sum(p[3]["spheres"] for p in prepared)),
           "configs": [int(sum(1 for s in specs if s["config"] == c)) for c in range(3)]}
    for label, nstreams, lf, tiles in (("tiles", streams, True, True), ("concurrent", streams, False, False),
                                       ("concurrent_largest_first", streams, True, False),
                                       ("one_stream", 1, False, False)):
        for f in films:
            f.zero_()
        torch.cuda.synchronize()
        per, st = az.render_batch(jobs, streams=nstreams, largest_first=lf, tiles=tiles)
        done = np.array([p["done_ms"] for p in per])
        out[label] = {"streams": st["streams"], "gpu_ms": st["gpu_ms"], "samples": st["samples"],
                      "mpaths_per_s": st["samples"] / (st["gpu_ms"] / 1000.0) / 1e6,
                      "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "failed": st["failed"],
                      "guided_p50_ms": float(np.median(done[1::2])), "plain_p50_ms": float(np.median(done[0::2]))}
        if tiles:
            check = [k for k, s in enumerate(specs) if not s["guided"]][:8]
            snap = {k: films[k].clone() for k in check}
            worst = 0.0
            for k in check:
                films[k].zero_()
                az.render_batch([jobs[k]], streams=1)
                torch.cuda.synchronize()
                a = snap[k][..., :3] / snap[k][..., 3:].clamp_min(1e-30)
                b = films[k][..., :3] / films[k][..., 3:].clamp_min(1e-30)
                worst = max(worst, float(((a - b) ** 2 / (b ** 2 + 1e-2)).mean()))
            out[label]["equal_image_check"] = {"jobs": len(check), "max_relmse_vs_own_render": worst}
        log("%s: %s" % (label, json.dumps(out[label])))
    for gd in guides:
        gd.close()
    for gs in gscenes:
        gs.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=256)
    ap.add_argument("--streams", type=int, default=8)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args()
    print(json.dumps(run(a.jobs, a.streams, a.seed)), flush=True)


if __name__ == "__main__":
    main()
