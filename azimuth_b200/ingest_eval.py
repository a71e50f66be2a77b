"""Time to a renderable device scene: azimuth's finished structs vs the mesh soup.

    python -m azimuth_b200.ingest_eval [--scenes 1,3]

For each scene (default: the dense mesh, 1.31 M triangles, and the interior,
3.96 M triangles, at their default sizes) and each path, one JSON line:
`structs` generates the scene as azimuth's importer leaves it (post-processed
meshes and 288-byte entity BVHs) and builds it with az_gpu_scene_create;
`soup` generates only the importer's arrays (AZ_GEN_SOUP_ONLY) and builds with
az_gpu_scene_create_from_meshes (post-processing on the GPU).  Times are host
wall clock around each call after a synchronize; az_gpu_scene_info's split is
included.
"""
import argparse
import json
import time


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", default="1,3")
    a = ap.parse_args(argv)
    import torch
    import azimuth_b200 as az
    torch.zeros(1, device="cuda")
    torch.cuda.synchronize()
    names = {az.SCENE_DENSE_MESH: "dense_mesh", az.SCENE_INTERIOR: "interior", az.SCENE_CORNELL: "cornell",
             az.SCENE_MOTION_ENV: "motion_env"}
    for sid in [int(s) for s in a.scenes.split(",")]:
        for path in ("structs", "soup"):
            t0 = time.time()
            sc = az.generate_scene(sid, seed=0, soup_only=(path == "soup"))
            t1 = time.time()
            g = az.GpuScene(sc, from_soup=(path == "soup"))
            torch.cuda.synchronize()
            t2 = time.time()
            info = {k: (round(v, 2) if isinstance(v, float) else v) for k, v in g.info().items()}
            print(json.dumps({"scene": names.get(sid, str(sid)), "path": path, "generate_s": round(t1 - t0, 3),
                              "gpu_scene_s": round(t2 - t1, 3), "ready_s": round(t2 - t0, 3), "info": info}),
                  flush=True)
            g.close()
            sc.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
