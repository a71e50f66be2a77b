"""Every benchmark config at its full size on one GPU.

    python -m azimuth_b200.configs_eval [--configs 0,1,2,3] [--frames 3]

C0 Cornell box, C1 dense mesh, C2 moving spheres with an HDR environment
map, C3 interior, each at the generator's default size (the configs' sizes).
The scene is built, az_gpu_autotune_scene picks the hierarchy shape and the
launch configurations, then the best of `--frames` frames (device time) is
reported with the frame's camera samples (paths), extension queries (path
segments) and all rays (extension and shadow queries) per second.
"""
import argparse
import json
import sys
import time

CONFIGS = {0: "SCENE_CORNELL", 1: "SCENE_DENSE_MESH", 2: "SCENE_MOTION_ENV", 3: "SCENE_INTERIOR"}


def run(configs=(0, 1, 2, 3), frames=3, log=lambda m: print(m, file=sys.stderr, flush=True)):
    import torch
    import azimuth_b200 as az
    out = {}
    for c in configs:
        sc = az.generate_scene(getattr(az, CONFIGS[c]), seed=0)
        w, h = sc.resolution()
        film = torch.zeros((h, w, 4), device="cuda")
        with az.GpuScene(sc) as g:
            t0 = time.time()
            width, variant, band_ms = g.autotune_scene(seed=0)
            tune_s = time.time() - t0
            info = g.info()
            best = None
            for f in range(frames):
                film.zero_()
                st = g.render_device(film.data_ptr(), seed=f, stats=True)
                if best is None or st["gpu_ms"] < best["gpu_ms"]:
                    best = st
        s = best["gpu_ms"] / 1e3
        out["C%d" % c] = {"scene": CONFIGS[c], "width": w, "height": h, "spp": sc.sample_count(),
                          "max_depth": sc.max_depth(), "frame_ms": best["gpu_ms"],
                          "Mpaths_per_s": best["samples"] / s / 1e6,
                          "Msegments_per_s": best["extend_rays"] / s / 1e6,
                          "Mrays_per_s": (best["extend_rays"] + best["shadow_rays"]) / s / 1e6,
                          "waves": best["chunks"], "bvh_width": width, "variant": variant,
                          "shadow_variant": info["shadow_variant"], "queue_order": info["queue_order"],
                          "autotune_s": tune_s}
        log("C%d: %.1f ms, %.0f Mpaths/s, %.0f M segments/s" % (c, best["gpu_ms"], out["C%d" % c]["Mpaths_per_s"],
                                                               out["C%d" % c]["Msegments_per_s"]))
        sc.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--configs", default="0,1,2,3")
    ap.add_argument("--frames", type=int, default=3)
    a = ap.parse_args()
    print(json.dumps(run(tuple(int(x) for x in a.configs.split(",")), a.frames)))


if __name__ == "__main__":
    main()
