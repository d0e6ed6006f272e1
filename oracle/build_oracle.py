"""Build the CPU checkers under oracle/ (test infrastructure only).

* oracle/libpic_oracle.so -- the plain-C restatement (oracle/pic_oracle.c),
  always built.
* oracle/_ref/libaprl_ref.so -- the reference's own hot-path translation
  units, compiled straight from the APRL sources with a single-rank MPI
  stand-in (oracle/ref/mpi_shim), a stand-in for the three FFTW calls of the
  blocked Cowan reference (oracle/ref/fftw_shim: the type-I sine transform
  by direct sums) and the driver in oracle/ref/ref_harness.cpp.
  Built only where the APRL source tree is present; the built library then
  travels with the repository copy.

The APRL source tree (its src/ folder) is taken from --reference-src, else
from the environment variable APRL_REFERENCE_SRC, else from a checkout named
`reference` beside this repository (../reference/src).

Usage: python oracle/build_oracle.py [--reference-src DIR]
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def default_reference_src():
    return os.environ.get("APRL_REFERENCE_SRC") or os.path.join(
        os.path.dirname(REPO), "reference", "src")

# The hot-path translation units of APRL 2.1 that compile against the MPI
# stand-in (the remaining ones need HDF5, yaml-cpp or FFTW).
REFERENCE_UNITS = [
    "eb_field", "eb_cpml", "eb_deposition", "eb_particles", "boostframe",
    "eb_sources", "compute_threads", "source_coupling",
    "moving_window_fields", "particle_boundary", "pending_particle_queue",
    "eb_initial_field", "transverse_reference_current", "blocked_cowan_reference",
]


def run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_oracle():
    src = os.path.join(HERE, "pic_oracle.c")
    out = os.path.join(HERE, "libpic_oracle.so")
    deps = [src, os.path.join(HERE, "pic_oracle.h"),
            os.path.join(REPO, "include", "aprl_gpu.h")]
    if newer(out, deps):
        run(["gcc", "-O2", "-std=c11", "-D_GNU_SOURCE", "-ffp-contract=off",
             "-fPIC", "-shared", "-Wall", "-o", out, src, "-lm"])
    return out


def build_reference(reference_src):
    if not os.path.isdir(reference_src):
        print(f"reference sources not found at {reference_src}; "
              "oracle/_ref not rebuilt", flush=True)
        return None
    outdir = os.path.join(HERE, "_ref")
    objdir = os.path.join(outdir, "obj")
    os.makedirs(objdir, exist_ok=True)
    shim = os.path.join(HERE, "ref", "mpi_shim")
    fftw = os.path.join(HERE, "ref", "fftw_shim")
    flags = ["-std=c++14", "-O2", "-fopenmp", "-DAPRL_HAS_OPENMP=1",
             "-DAPRL_HAS_MOVING_WINDOW=1", "-fPIC", "-I", shim, "-I", fftw,
             "-I", reference_src, "-I", os.path.join(REPO, "include")]
    objects = []
    headers = [os.path.join(reference_src, f) for f in os.listdir(reference_src)
               if f.endswith(".h")]
    for unit in REFERENCE_UNITS:
        src = os.path.join(reference_src, unit + ".cpp")
        obj = os.path.join(objdir, unit + ".o")
        if newer(obj, [src] + headers):
            run(["g++"] + flags + ["-c", src, "-o", obj])
        objects.append(obj)
    for src in [os.path.join(HERE, "ref", "ref_harness.cpp"),
                os.path.join(shim, "mpi_shim.cpp"),
                os.path.join(fftw, "fftw_shim.cpp")]:
        obj = os.path.join(objdir, os.path.basename(src).replace(".cpp", ".o"))
        if newer(obj, [src, os.path.join(shim, "mpi.h"), os.path.join(fftw, "fftw3.h"),
                       os.path.join(REPO, "include", "aprl_gpu.h")] + headers):
            run(["g++"] + flags + ["-c", src, "-o", obj])
        objects.append(obj)
    out = os.path.join(outdir, "libaprl_ref.so")
    if newer(out, objects):
        run(["g++", "-shared", "-fopenmp", "-o", out] + objects)
    return out


def main(argv=None):
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference-src", default=None)
    args = parser.parse_args(argv)
    build_oracle()
    build_reference(args.reference_src or default_reference_src())


if __name__ == "__main__":
    sys.exit(main())
