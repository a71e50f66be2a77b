"""Build recipe for the oracle (test infrastructure).

Two libraries come out of it:

* ``oracle/_ref/libazref.so`` (+ ``libazref_fast.so``): azimuth's own render
  code, compiled from the reference checkout after the mechanical edits of
  ``oracle/patch_reference.py``, linked with ``oracle/ref_harness.cpp``.
  ``libazref.so`` is the parity build (-O2, IEEE, no FMA contraction);
  ``libazref_fast.so`` is the speed build (-O3 -ffast-math), the nearest GCC
  analogue of azimuth's MSVC ``/O2 /fp:fast`` release flags (build.bat:26,40).
  Needs the reference sources, so it only runs where they exist; the built
  files travel with the repository to the GPU box.
* ``oracle/lib/libazoracle.so``: the CPU restatement ``oracle/az_oracle.c``
  (plain C, no reference code), built wherever gcc exists.

Usage: python oracle/build.py [--reference DIR] [--force]
(DIR defaults to $AZIMUTH_REFERENCE, else ../reference beside the repository.)
"""
import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF_OUT = os.path.join(HERE, "_ref")
PORT_OUT = os.path.join(HERE, "lib")
# the reference checkout: AZIMUTH_REFERENCE, else the checkout beside the
# repository (../reference), else /root/reference
DEFAULT_REFERENCE = os.environ.get("AZIMUTH_REFERENCE") or next(
    (d for d in (os.path.join(os.path.dirname(REPO), "reference"), "/root/reference")
     if os.path.isdir(os.path.join(d, "src"))), "/root/reference")

PARITY_FLAGS = ["-O2", "-ffp-contract=off", "-fno-strict-aliasing"]
# x86-64-v3 (AVX2/FMA) rather than -march=native: the library is built here and
# also runs on the GPU box's host CPU.
SPEED_FLAGS = ["-O3", "-ffast-math", "-march=x86-64-v3", "-fno-strict-aliasing"]


def _run(cmd):
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout)
        raise RuntimeError("oracle build failed: " + " ".join(cmd[:3]) + " ...")
    return proc.stdout


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_reference(reference=DEFAULT_REFERENCE, force=False):
    """Patch and compile the reference render code into oracle/_ref."""
    src = os.path.join(reference, "src")
    inc = os.path.join(reference, "include")
    if not os.path.isdir(src):
        return None
    patched = os.path.join(REF_OUT, "src")
    harness = os.path.join(HERE, "ref_harness.cpp")
    shim = os.path.join(HERE, "shim")
    deps = [harness, os.path.join(HERE, "patch_reference.py"), os.path.join(HERE, "az_rng_oracle.h"),
            os.path.join(REPO, "include", "az_abi.h"), os.path.join(REPO, "include", "az_xmlreader.h"),
            os.path.join(REPO, "include", "azimuth_gpu.h")]
    deps += [os.path.join(d, f) for d, _, files in os.walk(shim) for f in files]
    outputs = {"libazref.so": PARITY_FLAGS, "libazref_fast.so": SPEED_FLAGS}
    if not force and not any(_stale(os.path.join(REF_OUT, o), deps) for o in outputs):
        return os.path.join(REF_OUT, "libazref.so")
    if os.path.isdir(patched):
        shutil.rmtree(patched)
    os.makedirs(REF_OUT, exist_ok=True)
    _run([sys.executable, os.path.join(HERE, "patch_reference.py"), src, patched])
    for out, flags in outputs.items():
        cmd = ["g++", "-std=c++14", "-shared", "-fPIC", "-fopenmp", "-fpermissive", "-w"] + flags + [
            "-I", patched, "-I", shim, "-I", HERE, "-I", os.path.join(REPO, "include"), "-I", inc,
            "-include", os.path.join(shim, "az_oracle_compat.h"),
            "-Dmain=azimuth_main", harness, "-o", os.path.join(REF_OUT, out), "-lpthread"]
        _run(cmd)
    return os.path.join(REF_OUT, "libazref.so")


def build_port(force=False):
    """Compile the C restatement oracle/az_oracle.c into oracle/lib."""
    srcs = [os.path.join(HERE, "az_oracle.c")]
    if not os.path.exists(srcs[0]):
        return None
    deps = srcs + [os.path.join(HERE, "az_rng_oracle.h"), os.path.join(REPO, "include", "az_abi.h")]
    os.makedirs(PORT_OUT, exist_ok=True)
    out = os.path.join(PORT_OUT, "libazoracle.so")
    if force or _stale(out, deps):
        _run(["gcc", "-std=gnu11", "-shared", "-fPIC", "-fopenmp", "-Wall", "-Wno-unused-function"]
             + PARITY_FLAGS + ["-I", HERE, "-I", os.path.join(REPO, "include")]
             + srcs + ["-o", out, "-lm"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build_reference(args.reference, args.force))
    print(build_port(args.force))


if __name__ == "__main__":
    main()
