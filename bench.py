"""Benchmark: Mpaths/s of azimuth's render path on B200 (dense-mesh workload).

Workload (one "step" = one frame): the dense-mesh scene -- the Cornell walls and
area light around a seeded, Perlin-displaced icosphere of 1,310,720 triangles
whose faces are split round-robin over azimuth's seven BRDF models -- at
1024x1024, 64 samples per pixel, MaxRecursionDepth 8, cosine importance
sampling with area-light next-event estimation and the Gaussian film filter.
Data are synthetic (seeded generator), the scene is built in azimuth's own
structs.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

GPU arm: the scene is uploaded once (az_gpu_scene_create); each step renders
the frame into a device film with az_gpu_render; K steps are timed with CUDA
events on the render stream, between a barrier and a synchronize, max over
ranks.  Each rank renders its own frame with its own seed (weak scaling, no
collective on the data path).  `e2e` repeats the measurement through
az_gpu_render_host, the host-film entry point, with the film copied in and out
every step.

Reference arm (--impl reference): azimuth's own ProduceImageInLinearSpace
(oracle/_ref/libazref_fast.so, the -O3 -ffast-math build) on all host cores,
each step a bounded sample of the same frame (8 rows x 32 pixels spread over
the image, all 64 samples and full depth), rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "Mpaths/s on 1 B200; equal-time relMSE guided vs plain GPU vs FP64 converged"
WORKLOAD = "dense mesh + importance sampling: 1,310,720-triangle Perlin-displaced icosphere in a Cornell box, " \
           "7 BRDFs, 1024x1024, 64 spp, depth 8, cosine sampling + area-light NEE, Gaussian filter"
SCENE_ARGS = dict(scene_id=1, seed=0)
# DRAM read + write per query of the two traversal kernels on this scene, from
# one single-pass ncu capture (dram__bytes_read.sum + dram__bytes_write.sum)
# of every k_extend / k_shadow launch of one 256x256, 16-spp frame (one wave of
# 2^20 samples): the capture's bytes over the frame's queries
DRAM_BYTES_PER_QUERY = {"k_extend": 207.1, "k_shadow": 246.2}
PROFILE_NOTE = "profiles/traversal_dram_dense_mesh_256x256_16spp.md, profiles/k_extend_k_shadow_dense_mesh_256x256_16spp.md"
# issue statistics of the two traversal kernels from the ncu capture of that small case
ISSUE = {"k_extend": {"threads_per_warp_instruction": 8.63, "issue_active_pct": 57.1, "warps_active_pct": 36.2},
         "k_shadow": {"threads_per_warp_instruction": 8.47, "issue_active_pct": 56.2, "warps_active_pct": 34.3}}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--chunk", type=int, default=0, help="camera samples per wave (0 = library default)")
    ap.add_argument("--split", action="store_true",
                    help="N>1: render ONE frame per step over the ranks (equal parts of its camera samples, "
                         "then an NCCL reduce of the films into rank 0) instead of one frame per rank")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip az_gpu_autotune_scene (BVH width and traversal launch variant) before timing")
    return ap.parse_args()


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        return self.summary()

    def summary(self):
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                mhz.append(float(r[1]))
                mx = float(r[2])
                for k, name in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


def reference_sample_scissors(w, h):
    """8 rows spread over the frame, 32 columns each at spread positions."""
    out = []
    for k in range(8):
        row = (2 * k + 1) * h // 16
        col = ((5 * k + 3) % 16) * w // 16
        out.append((row, row + 1, col, col + 32))
    return out


def run_reference_sample(scene, steps, warmup, threads):
    """azimuth's ProduceImageInLinearSpace over the bounded sample; returns paths/s and seconds."""
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import oracle_lib as ol
    fast = ol.have_ref(fast=True)
    kind = "reference" if fast else "port"
    w, h = scene.resolution()
    spp = int(int(scene.sample_count() ** 0.5) ** 2)
    boxes = reference_sample_scissors(w, h)
    paths_per_step = sum((r1 - r0) * (c1 - c0) for r0, r1, c0, c1 in boxes) * spp

    def one_step(seed):
        for r0, r1, c0, c1 in boxes:
            sc = ol.scissor_of(scene, rows=(r0, r1), cols=(c0, c1))
            if fast:
                ol.ref_film(scene, seed=seed, threads=threads, scissor=sc, fast=True)
            else:
                ol.port_film(scene, seed=seed, threads=threads, scissor=sc)

    for i in range(warmup):
        one_step(100 + i)
    t0 = time.monotonic()
    for i in range(steps):
        one_step(i)
    dt = time.monotonic() - t0
    return paths_per_step * steps / dt, dt, paths_per_step, kind


def reference_arm(args):
    import azimuth_b200 as az
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    scene = az.generate_scene(SCENE_ARGS["scene_id"], seed=SCENE_ARGS["seed"])
    pps, dt, per_step, kind = run_reference_sample(scene, args.steps, args.warmup, threads)
    value = pps / 1e6
    sample = "per step: 8 rows x 32 px spread over the 1024x1024 frame, 64 spp, depth 8 (%d paths)" % per_step
    out = {"metric": METRIC, "value": value, "unit": "Mpaths/s", "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / max(args.steps, 1),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded generator, azimuth structs)",
           "config": {"workload": WORKLOAD, "parallelism": "host threads (%d)" % threads, "sample": sample},
           "cpu_baseline": {"value": value, "unit": "Mpaths/s", "cores": threads, "kind": kind, "sample": sample},
           "e2e": {"value": value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


def seed_base(rank):
    return 1000 * rank


def max_over_ranks(dist, value, device):
    """The largest of every rank's `value` (a time), on every rank; `value` itself without a process group."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(world, units_per_rank, steps, seconds):
    """Whole-job throughput: every rank's units over the slowest rank's time (weak scaling)."""
    return world * units_per_rank * steps / seconds


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)

    import numpy as np
    import torch
    import azimuth_b200 as az

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    scene = az.generate_scene(SCENE_ARGS["scene_id"], seed=SCENE_ARGS["seed"])
    w, h = scene.resolution()
    spp = int(int(scene.sample_count() ** 0.5) ** 2)
    paths_per_frame = w * h * spp
    t0 = time.time()
    gs = az.GpuScene(scene, device=local)
    torch.cuda.synchronize()
    upload_s = time.time() - t0
    # az_gpu_scene_info: host flattening, uploads and the GPU BVH build of this first build
    build = {k: (round(v, 2) if isinstance(v, float) else v) for k, v in gs.info().items()}
    tune = None
    if not args.no_autotune:
        # the autotuner's sweep (BVH width 8/4/2 x launch variants) on a band of the frame
        t0 = time.time()
        tw, tv, tms = gs.autotune_scene(seed=seed_base(rank))
        tune = {"bvh_width": tw, "variant": tv, "shadow_variant": gs.info()["shadow_variant"], "band_ms": tms,
                "seconds": time.time() - t0}

    # a stream of our own: the wave launches are captured and replayed as CUDA
    # graphs, which the legacy default stream does not allow
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream
    film = torch.zeros((h, w, 4), device="cuda", dtype=torch.float32)
    # one frame over the ranks needs the same random numbers on every rank
    seed = seed_base(0) if (args.split and world > 1) else seed_base(rank)

    split = args.split and world > 1

    def step(i, flags=0, stats=False):
        if not split:
            return gs.render_device(film.data_ptr(), seed=seed + i, stream=sptr, flags=flags, stats=stats,
                                    chunk_samples=args.chunk)
        # one frame over the ranks: this rank's part of the camera-sample sequence, then one
        # NCCL reduce of the films into rank 0 (azimuth_b200.scanlines, "samples" split)
        film.zero_()
        st_ = gs.render_device(film.data_ptr(), seed=seed + i, stream=sptr, flags=flags, stats=stats,
                               chunk_samples=args.chunk, sample_part=rank, sample_parts=world)
        dist.reduce(film, dst=0)
        return st_

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    launches = 0
    extend_ms = 0.0
    extend_launches = 0
    seg = shadow = 0
    for i in range(args.steps):
        st = step(args.warmup + i, stats=True)
        launches += st["kernel_launches"]
        seg += st["extend_rays"]
        shadow += st["shadow_rays"]
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    # stage split from one more frame outside the timed region (events between
    # the stages; direct launches instead of the graph)
    stg = step(args.warmup + args.steps, flags=az.FLAG_TIME_STAGES, stats=True)
    extend_ms = stg["extend_ms"] * args.steps
    extend_launches = stg["extend_launches"] * args.steps
    stages = {"extend_ms": stg["extend_ms"], "shade_ms": stg["shade_ms"], "shadow_ms": stg["shadow_ms"],
              "frame_ms": stg["gpu_ms"]}
    ms = max_over_ranks(dist, ms, "cuda")
    if dist:
        dist.barrier()
    ms_per_step = ms / args.steps
    # weak scaling: every rank's frame; split: one frame per step over all ranks
    value = aggregate(1 if split else world, paths_per_frame, args.steps, ms / 1000.0) / 1e6

    # end to end through the host-film entry point (film in and out every step)
    host_film = torch.zeros((h, w, 4), dtype=torch.float32).pin_memory()
    hf = host_film.numpy()
    gs.render_host(hf, seed=seed, stream=sptr, chunk_samples=args.chunk)   # warm the host-film path
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.monotonic()
    e_steps = args.steps   # as many frames as the device-timed region
    for i in range(e_steps):
        gs.render_host(hf, seed=seed + i, stream=sptr, chunk_samples=args.chunk)
    e2e_s = time.monotonic() - t0
    e2e_s = max_over_ranks(dist, e2e_s, "cuda")
    e2e = {"value": aggregate(world, paths_per_frame, e_steps, e2e_s) / 1e6, "unit": "Mpaths/s",
           "h2d_bytes_per_step": int(w * h * 16), "d2h_bytes_per_step": int(w * h * 16), "steps": e_steps,
           "api": "az_gpu_render_host (device scene resident, host film copied in and out)"}

    # rooflines of the two traversal kernels: algorithmic bytes from a counting
    # pass over one frame (node and primitive visits of each query kind, counted
    # by the kernels themselves), time per launch from the stage-timed frame
    cnt = step(0, flags=az.FLAG_COUNT_TRAVERSAL, stats=True)
    torch.cuda.synchronize()

    # the production triangle test (AZ_FLAG_WATERTIGHT) on the same frame, outside
    # the timed region: one frame to capture its graphs, then one timed frame
    wt = {}
    for i in range(2):
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        s_ = step(args.warmup + i, flags=az.FLAG_WATERTIGHT, stats=True)
        a1.record(stream)
        torch.cuda.synchronize()
        wt = {"ms_per_frame": a0.elapsed_time(a1), "segments_per_s": world * s_["extend_rays"] / (
            a0.elapsed_time(a1) / 1000.0), "test": "watertight (Woop, Benthin and Wald 2013) instead of azimuth's"}
    wt["ms_per_frame"] = max_over_ranks(dist, wt["ms_per_frame"], "cuda")
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    launches_per_frame = max(1, stg["extend_launches"])
    ext_q, sh_q = max(1, cnt["extend_rays"]), max(1, cnt["shadow_rays"])
    # closest hit, per query: ray read (32 B) + hit written (16 B); 80 B per wide node, 48 B per triangle
    ext_bytes = cnt["extend_rays"] * (32 + 16) + cnt["node_visits"] * 80 + cnt["prim_visits"] * 48
    # visibility, per query: origin, direction and contribution read (48 B) + kind (4 B) + one 16-byte sum
    # for a visible sample (counted for every query); the same node and triangle bytes
    sh_bytes = cnt["shadow_rays"] * (48 + 4 + 16) + cnt["shadow_node_visits"] * 80 + cnt["shadow_prim_visits"] * 48
    per_launch_ext_ms = stg["extend_ms"] / launches_per_frame
    per_launch_sh_ms = stg["shadow_ms"] / launches_per_frame
    ext_achieved = ext_bytes / launches_per_frame / (per_launch_ext_ms / 1000.0) / 1e9
    sh_achieved = sh_bytes / launches_per_frame / (per_launch_sh_ms / 1000.0) / 1e9
    # DRAM read + write per query from a single-pass ncu capture of every launch
    # of one small frame of the same scene (DRAM_BYTES_PER_QUERY), scaled to a
    # launch of this frame by its query count
    dense = SCENE_ARGS["scene_id"] == az.SCENE_DENSE_MESH
    ext_traffic = (DRAM_BYTES_PER_QUERY["k_extend"] * ext_q / launches_per_frame
                   if dense and DRAM_BYTES_PER_QUERY["k_extend"] else None)
    sh_traffic = (DRAM_BYTES_PER_QUERY["k_shadow"] * sh_q / launches_per_frame
                  if dense and DRAM_BYTES_PER_QUERY["k_shadow"] else None)
    limiter = ("instruction issue of divergent traversal, not HBM: about 8 of 32 lanes active per warp "
               "instruction, DRAM traffic a quarter of the algorithmic bytes (%s)" % PROFILE_NOTE)
    roofline = {"bound": "hbm", "achieved": ext_achieved, "peak": hbm, "unit": "GB/s", "frac": ext_achieved / hbm,
                "traffic": ext_traffic, "traffic_unit": "DRAM bytes per launch (ncu, scaled from a small frame)",
                "algorithmic_bytes_per_launch": ext_bytes / launches_per_frame,
                "kernel": "k_extend (closest-hit traversal)", "limiter": limiter, "issue": ISSUE["k_extend"],
                "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650",
                "bytes_per_segment": ext_bytes / ext_q,
                "node_visits_per_segment": cnt["node_visits"] / ext_q,
                "prim_visits_per_segment": cnt["prim_visits"] / ext_q,
                "launch_ms": per_launch_ext_ms,
                "extend_share_of_serial_frame": stg["extend_ms"] / max(stg["gpu_ms"], 1e-9)}
    roofline_shadow = {"bound": "hbm", "achieved": sh_achieved, "peak": hbm, "unit": "GB/s",
                       "frac": sh_achieved / hbm, "traffic": sh_traffic,
                       "traffic_unit": "DRAM bytes per launch (ncu, scaled from a small frame)",
                       "algorithmic_bytes_per_launch": sh_bytes / launches_per_frame,
                       "kernel": "k_shadow (visibility, any hit)", "limiter": limiter, "issue": ISSUE["k_shadow"],
                       "bytes_per_query": sh_bytes / sh_q,
                       "node_visits_per_query": cnt["shadow_node_visits"] / sh_q,
                       "prim_visits_per_query": cnt["shadow_prim_visits"] / sh_q,
                       "launch_ms": per_launch_sh_ms,
                       "shadow_share_of_serial_frame": stg["shadow_ms"] / max(stg["gpu_ms"], 1e-9)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            # four seeds of the sample: about 10-15 s of work on the GPU box's host cores
            pps, dt, per_step, kind = run_reference_sample(scene, 4, 0, threads)
            cpu = {"value": pps / 1e6, "unit": "Mpaths/s", "cores": threads, "kind": kind,
                   "sample": "4 x (8 rows x 32 px spread over the frame, 64 spp, depth 8: %d paths), "
                             "azimuth -O3 -ffast-math build" % per_step, "seconds": dt}
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "Mpaths/s", "cores": 0, "kind": "unavailable", "sample": str(ex)}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
               "scaling": "strong" if split else "weak",
               "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, azimuth structs)",
               "config": {"workload": WORKLOAD, "triangles": int(scene.triangle_count), "width": w, "height": h,
                          "spp": spp, "max_depth": scene.max_depth(),
                          "paths_per_step_per_gpu": paths_per_frame // world if split else paths_per_frame,
                          "parallelism": ("split%d (one frame per step: equal parts of its camera samples per "
                                          "GPU, one NCCL reduce of the films)" % world) if split else
                                         "dp%d (one frame per GPU, own seed)" % world,
                          "l2": "inputs larger than L2 (scene %.0f MB on device)" % (
                              gs.info()["device_bytes"] / 1e6),
                          "scene_upload_s": upload_s, "scene_build": build, "autotune": tune},
               "segments_per_s": world * seg / (ms / 1000.0), "rays_per_s": world * (seg + shadow) / (ms / 1000.0),
               "gpu_launches": int(launches), "stages_one_frame": stages, "e2e": e2e, "roofline": roofline,
               "roofline_shadow": roofline_shadow, "watertight_mode": wt,
               "clocks": clk}
        if cpu:
            out["cpu_baseline"] = cpu
        print(json.dumps(out), flush=True)
    gs.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
