"""Build the in-tree CUDA library aprl_b200/libaprl_b200.so for sm_100a.

The FP64 drop-in kernels are compiled without FMA contraction
(--fmad=false) so their arithmetic follows the reference's operation order.

Usage: python -m aprl_b200.build [--force]
"""
import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUTPUT = os.path.join(HERE, "libaprl_b200.so")
SOURCES = ["run.cu", "fields.cu", "particles.cu", "ledger.cu", "selffield.cu", "scan.cu"]
HEADERS = ["common.cuh", "dd.cuh", "fields.cuh", "ledger.cuh", "particles.cuh", "selffield.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def flags():
    # Kernel templates are instantiated in fields.cu / particles.cu and
    # launched from run.cu: keep their host stubs externally visible.
    return ["-std=c++17", "-O3", "-lineinfo", "--fmad=false", "-Xcompiler",
            "-fPIC", "-static-global-template-stub=false",
            "-I", os.path.join(REPO, "include")] + ARCH


# The bounds-checked variant: every field, current, orbit-sum, CPML-history
# and inlet-plane index of the step's kernels is tested before the access; an
# index outside its array raises the run's device error instead of touching
# memory (never a trap).  Slower; for testing.
CHECKED_OUTPUT = os.path.join(HERE, "libaprl_b200_checked.so")


def _build_library(output, objdir, extra, force, verbose):
    deps = ([os.path.join(CSRC, s) for s in SOURCES + HEADERS] +
            [os.path.join(REPO, "include", "aprl_gpu.h"), os.path.abspath(__file__)])
    if (not force and os.path.exists(output) and
            all(os.path.getmtime(d) <= os.path.getmtime(output) for d in deps)):
        return output
    os.makedirs(objdir, exist_ok=True)
    objects = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [nvcc(), "-rdc=false", "-c", os.path.join(CSRC, src), "-o", obj] + flags() + extra
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        objects.append(obj)
    cmd = [nvcc(), "-shared", "-o", output] + objects + ARCH + ["-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return output


def build(force=False, verbose=True):
    return _build_library(OUTPUT, os.path.join(HERE, "_build"), [], force, verbose)


def build_checked(force=False, verbose=True):
    return _build_library(CHECKED_OUTPUT, os.path.join(HERE, "_build_checked"),
                          ["-DAPRL_GPU_BOUNDS_CHECK"], force, verbose)


def main(argv=None):
    parser = argparse.ArgumentParser()
    parser.add_argument("--force", action="store_true")
    args = parser.parse_args(argv)
    build(force=args.force)
    build_checked(force=args.force)


if __name__ == "__main__":
    sys.exit(main())
