"""Equal-time comparison of the guided and the plain GPU renderer.

    python -m azimuth_b200.guiding_eval [--width 480 --height 270 --detail 49 --ref-spp 4096 --pass-spp 4]
    python -m azimuth_b200.guiding_eval --width 1920 --height 1080 --ref-file REF.npz --ref-spp 8192 --ref-only
    python -m azimuth_b200.guiding_eval --width 1920 --height 1080 --ref-file REF.npz --ref-spp 0 --runs 5

Workload: the interior scene (three 8x4x8 rooms joined by 1x2 doorways,
Perlin-displaced panels and clutter, ~4 M triangles at the default detail,
one 1x1 light in room 1, camera in room 3, depth 10).  A converged reference
is accumulated in FP64 from plain renders (`--ref-spp` samples per pixel, in
renders of 1024 samples per pixel); with `--ref-file` the reference's mean
(rounded to float32 for the file: 6e-8 relative, far below the noise of any
reference) and its sample count are kept in that file and every run adds
`--ref-spp` more in FP64, so a reference of many thousand samples per pixel
can be built over several runs (`--ref-only` stops after that).
Then each renderer runs passes of `--pass-spp` samples per pixel until
`--passes`; after every pass the running average's relMSE against the
reference, mean over pixels and channels of (x - ref)^2 / (ref^2 + 1e-2), is
recorded with the GPU time spent so far (CUDA events; the guide's inference,
recording and training included).  Both renderers run with their buffers
already allocated: the plain renderer's by the reference renders, the
guided renderer's (proposals, records) by one training and one inference
render of a throwaway guide before the timed passes.  The guided renderer trains during the
first `--train-passes` passes and keeps every pass in its average (all are
unbiased).  Reported: both curves and the time the guided renderer needs to
reach the plain renderer's final relMSE, as a fraction of the plain time.
With `--runs R` the comparison is repeated R times against the same
reference, run r drawing its passes' random numbers and the guide's initial
weights from seeds of its own (`--ref-spp 0` with `--ref-file` adds no
reference samples).
"""
import argparse
import json
import sys
import time

import numpy as np


def _relmse(img, ref):
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))


def _time_to(curve, target):
    """First time (linear interpolation in log relMSE) at which curve reaches target."""
    prev_t, prev_e = 0.0, None
    for t, e in curve:
        if e <= target:
            if prev_e is None or prev_e <= e:
                return t
            a = (np.log(prev_e) - np.log(target)) / (np.log(prev_e) - np.log(e))
            return prev_t + a * (t - prev_t)
        prev_t, prev_e = t, e
    return None


def _log(msg):
    print(msg, file=sys.stderr, flush=True)


def _camera_with_spp(scene, spp):
    """A copy of the scene's camera (az_camera, 396 bytes) with another sample count."""
    import ctypes as C
    buf = (C.c_ubyte * 396)()
    C.memmove(buf, scene.camera_ptr, 396)
    C.c_uint32.from_address(C.addressof(buf) + 384).value = spp   # az_camera.SampleCount
    return buf


def run(width=480, height=270, detail=49, ref_spp=4096, pass_spp=4, passes=64, train_passes=16, seed=0,
        log=_log, ref_file=None, ref_only=False, runs=1, guide_kw=None):
    import torch
    import azimuth_b200 as az
    t0 = time.time()
    scene = az.generate_scene(az.SCENE_INTERIOR, seed=seed, width=width, height=height, spp=pass_spp, detail=detail)
    gen_s = time.time() - t0
    w, h = scene.resolution()
    spp = int(int(scene.sample_count() ** 0.5) ** 2)
    film = torch.zeros((h, w, 4), device="cuda")
    out = {"workload": "interior (3 rooms, %d triangles), %dx%d, depth %d" % (scene.triangle_count, w, h,
                                                                                scene.max_depth()),
           "pass_spp": spp, "passes": passes, "train_passes": train_passes, "generate_s": gen_s}
    with az.GpuScene(scene) as g:
        stream = torch.cuda.current_stream()

        def one(render):
            film.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            render()
            e1.record(stream)
            torch.cuda.synchronize()
            f = film.cpu().numpy().astype(np.float64)
            return f[..., :3] / np.maximum(f[..., 3:4], 1e-30), e0.elapsed_time(e1) / 1000.0

        # converged reference: FP64 sum of plain renders of 1024 spp (or fewer), each
        # with its own seeds; the image is the sum over the renders' sample count
        import ctypes as C
        import os
        ref_sum, ref_n, ref_runs = np.zeros((h, w, 3)), 0, 0
        if ref_file and os.path.exists(ref_file):
            z = np.load(ref_file)
            assert tuple(z["shape"]) == (h, w, 3) and int(z["detail"]) == detail and int(z["seed"]) == seed
            ref_n, ref_runs = int(z["spp"]), int(z["runs"])
            ref_sum = z["mean"].astype(np.float64) * ref_n
        per = min(1024, max(1, ref_spp))
        cam = _camera_with_spp(scene, per)
        per = int(int(per ** 0.5) ** 2)
        t_ref = 0.0
        assert ref_spp > 0 or ref_n > 0, "--ref-spp 0 needs a reference file with samples"
        for k in range(ref_spp // per if ref_spp > 0 else 0):
            s = 100000 + 1000 * ref_runs + k
            img, dt = one(lambda: g.render_device(film.data_ptr(), camera_ptr=C.addressof(cam), seed=s,
                                                  stream=stream.cuda_stream))
            ref_sum += img * per
            ref_n += per
            t_ref += dt
        ref_runs += 1 if ref_spp > 0 else 0
        if ref_file and ref_spp > 0:
            np.savez(ref_file, mean=(ref_sum / ref_n).astype(np.float32), spp=ref_n, runs=ref_runs,
                     shape=np.array([h, w, 3]), detail=detail, seed=seed)
        ref = ref_sum / ref_n
        out["reference"] = {"spp": ref_n, "gpu_s_this_run": t_ref, "runs": ref_runs, "mean": float(ref.mean()),
                            "file": ref_file}
        log("reference: %d spp (%.1f s GPU in this run)" % (ref_n, t_ref))
        if ref_only:
            return out

        guide_kw = dict(guide_kw or {})
        out["guide_config"] = guide_kw
        # the plain renderer's wave queues were allocated by the reference renders; let the guided
        # renderer's proposal and record buffers be allocated outside its timed passes as well
        with az.Guide(g, seed=seed + 7777, **guide_kw) as warm:
            one(lambda: warm.render(film.data_ptr(), train=True, seed=999999, stream=stream.cuda_stream, stats=False))
            one(lambda: warm.render(film.data_ptr(), train=False, seed=999998, stream=stream.cuda_stream,
                                    stats=False))
        results = []
        for rn in range(runs):
            base = 7919 * rn   # run rn's pass seeds (run 0: passes 0, 1, ...)
            curves = {}
            # plain
            acc = np.zeros_like(ref)
            t, curve = 0.0, []
            for k in range(passes):
                img, dt = one(lambda: g.render_device(film.data_ptr(), seed=base + k, stream=stream.cuda_stream))
                acc += img
                t += dt
                curve.append((t, _relmse(acc / (k + 1), ref)))
            curves["plain"] = curve
            # guided (trains during the first passes)
            res = {"run": rn}
            with az.Guide(g, seed=seed + rn, **guide_kw) as guide:
                acc = np.zeros_like(ref)
                t, curve = 0.0, []
                for k in range(passes):
                    tr = k < train_passes
                    img, dt = one(lambda: guide.render(film.data_ptr(), train=tr, seed=base + k,
                                                       stream=stream.cuda_stream, stats=False))
                    acc += img
                    t += dt
                    curve.append((t, _relmse(acc / (k + 1), ref)))
                curves["guided"] = curve
                res["guide_steps"] = guide.info()["steps"]
            target = curves["plain"][-1][1]
            t_plain = curves["plain"][-1][0]
            t_guided = _time_to(curves["guided"], target)
            res["plain"] = {"gpu_s": t_plain, "relmse": target, "s_per_pass": t_plain / passes}
            res["guided"] = {"gpu_s": curves["guided"][-1][0], "relmse": curves["guided"][-1][1],
                             "s_per_pass": curves["guided"][-1][0] / passes,
                             "time_to_plain_relmse_s": t_guided}
            res["time_ratio_at_equal_relmse"] = (t_guided / t_plain) if t_guided is not None else None
            res["relmse_ratio_at_equal_passes"] = curves["guided"][-1][1] / target
            res["curves"] = {k: [[round(a, 5), b] for a, b in v] for k, v in curves.items()}
            log("run %d: time ratio %s, relMSE plain %.5g guided %.5g" % (
                rn, res["time_ratio_at_equal_relmse"], target, res["guided"]["relmse"]))
            results.append(res)
    if runs == 1:
        out.update(results[0])
    else:
        out["runs"] = results
        out["time_ratios"] = [r["time_ratio_at_equal_relmse"] for r in results]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=480)
    ap.add_argument("--height", type=int, default=270)
    ap.add_argument("--detail", type=int, default=49)
    ap.add_argument("--ref-spp", type=int, default=4096)
    ap.add_argument("--pass-spp", type=int, default=4)
    ap.add_argument("--passes", type=int, default=64)
    ap.add_argument("--train-passes", type=int, default=16)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--ref-file", default=None, help="npz keeping the FP64 reference sum across runs")
    ap.add_argument("--ref-only", action="store_true", help="only add --ref-spp samples to the reference")
    ap.add_argument("--runs", type=int, default=1, help="comparisons against the same reference")
    ap.add_argument("--steps-per-wave", type=int, default=0, help="Adam steps per training wave (0: the default)")
    ap.add_argument("--learning-rate", type=float, default=0.0)
    ap.add_argument("--record-samples", type=int, default=0)
    a = ap.parse_args()
    kw = {k: v for k, v in (("steps_per_wave", a.steps_per_wave), ("learning_rate", a.learning_rate),
                            ("record_samples", a.record_samples)) if v}
    res = run(a.width, a.height, a.detail, a.ref_spp, a.pass_spp, a.passes, a.train_passes, a.seed,
              ref_file=a.ref_file, ref_only=a.ref_only, runs=a.runs, guide_kw=kw)
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
