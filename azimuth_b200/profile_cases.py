"""Small, fixed workloads for profiling the kernels (ncu captures).

    python -m azimuth_b200.profile_cases dense_mesh [--variant V] [--frames F]
    python -m azimuth_b200.profile_cases guide_interior [--frames F]
    python -m azimuth_b200.profile_cases guide_interior_full [--frames F]

dense_mesh: the dense-mesh scene (1,310,720-triangle displaced icosphere in
the Cornell box, 7 BRDFs, depth 8) at 256x256 and 16 samples per pixel, one
wave per frame, traversal launch variant V (default: the library's).
guide_interior: the interior scene (detail 12, about 250 k triangles) at
320x180, 4 samples per pixel; the first frame trains the path guide, the
rest render with it.
guide_interior_full: the same at the guided comparison's size (detail 49,
about 4 M triangles, 1920x1080, 4 samples per pixel).
"""
import argparse
import sys


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["dense_mesh", "guide_interior", "guide_interior_full"])
    ap.add_argument("--variant", type=int, default=0)
    ap.add_argument("--frames", type=int, default=2)
    a = ap.parse_args(argv)
    import torch
    import azimuth_b200 as az
    if a.case == "dense_mesh":
        sc = az.generate_scene(az.SCENE_DENSE_MESH, seed=0, width=256, height=256, spp=16)
    elif a.case == "guide_interior":
        sc = az.generate_scene(az.SCENE_INTERIOR, seed=0, width=320, height=180, spp=4, detail=12)
    else:
        sc = az.generate_scene(az.SCENE_INTERIOR, seed=0, width=1920, height=1080, spp=4, detail=49)
    w, h = sc.resolution()
    film = torch.zeros((h, w, 4), device="cuda")
    with az.GpuScene(sc) as g:
        if a.case == "dense_mesh":
            for i in range(a.frames):
                st = g.render_device(film.data_ptr(), seed=i, stats=True, variant=a.variant)
                print(i, st["gpu_ms"], st["extend_rays"], st["shadow_rays"], flush=True)
        else:
            with az.Guide(g, seed=0) as guide:
                for i in range(a.frames):
                    st = guide.render(film.data_ptr(), train=(i == 0), seed=i, stats=True)
                    print(i, st["gpu_ms"], st["extend_rays"], st["shadow_rays"], flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
