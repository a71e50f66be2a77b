"""Build the native library ``azimuth_b200/libazimuth_b200.so`` in-tree.

Host C++ (scene assembly, generators, the RenderScene-style host API) is
compiled with g++ and ``-ffp-contract=off`` so its float sums round like
azimuth's; CUDA sources are compiled by nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``), side by side.  CUDA files are
compiled without FMA contraction (``--fmad=false``: primitive tests, mesh
ingestion, BVH quantisation and the post-process round like azimuth's scalar
code), except the ones in ``CONTRACTED``, whose results are compared within a
tolerance and feed no bit-exact distance: the path guide.  (The shading stage
stays uncontracted: contraction changed the finite differences of Perlin bump
mapping enough to move textured pixels beyond the 1e-4 parity bar.)  The result links the CUDA
runtime statically, so the library needs only the driver and the system zlib
at run time.

Usage: python -m azimuth_b200.build [--force] [--debug]
"""
import argparse
import concurrent.futures
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libazimuth_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# CUDA files compiled with FMA contraction (see above)
CONTRACTED = {"az_guide.cu"}
INCLUDES = ["-I", os.path.join(REPO, "include"), "-I", os.path.join(CSRC, "host"), "-I", os.path.join(CSRC, "cuda")]


def _run(cmd):
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout)
        raise RuntimeError("build failed: " + " ".join(cmd))
    return proc.stdout


def _headers():
    hs = glob.glob(os.path.join(REPO, "include", "*.h"))
    hs += glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True)
    hs += glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
    return hs


def _newer(src, obj, headers):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or any(os.path.getmtime(h) > t for h in headers)


def build(force=False, debug=False, verbose=False):
    headers = _headers()
    sources = glob.glob(os.path.join(CSRC, "host", "*.cpp")) + glob.glob(os.path.join(CSRC, "cuda", "*.cu"))
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(f) <= t for f in sources + headers):
            return LIB   # up to date (object files need not be present)
    os.makedirs(OBJ, exist_ok=True)
    objs = []
    opt = ["-O0", "-g"] if debug else ["-O2"]
    for src in sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp"))):
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        if force or _newer(src, obj, headers):
            _run(["g++", "-std=c++17", "-fPIC", "-c", "-Wall", "-Wno-unused-function", "-ffp-contract=off"]
                 + opt + INCLUDES + ["-I", "/usr/local/cuda/include", src, "-o", obj])
        objs.append(obj)
    cu_srcs = sorted(glob.glob(os.path.join(CSRC, "cuda", "*.cu")))
    jobs = []
    for src in cu_srcs:
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        if force or _newer(src, obj, headers):
            fmad = "--fmad=true" if os.path.basename(src) in CONTRACTED else "--fmad=false"
            cmd = [NVCC, "-std=c++17", "-c", "-Xcompiler", "-fPIC,-ffp-contract=off", "-lineinfo", "-O3",
                   fmad] + ARCH + INCLUDES
            cmd += ["-Xptxas", "-v"] if verbose else []
            cmd += ["-DAZ_DEBUG_CHECKS=1"] if debug else []
            jobs.append(cmd + [src, "-o", obj])
        objs.append(obj)
    # the CUDA files compile independently: one nvcc per file, side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for out in ex.map(_run, jobs):
            if verbose:
                sys.stdout.write(out)
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        if cu_srcs:
            _run([NVCC, "-shared", "-cudart", "static"] + ARCH + objs + ["-o", LIB, "-lpthread", "-lz"])
        else:
            _run(["g++", "-shared"] + objs + ["-o", LIB, "-lz"])
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="print ptxas register/spill report")
    a = ap.parse_args()
    print(build(a.force, a.debug, a.verbose))


if __name__ == "__main__":
    main()
