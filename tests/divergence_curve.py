"""Per-step divergence of the GPU runs from the reference over a long run.

Not a test (pytest does not collect it): a measurement that runs the drift
configuration (64x64x256 cells, 100k particles, linear-binomial3, FP64) for
`--steps` coupled steps with five runs in lock step -- the reference's own
translation units (oracle/_ref; the plain-C oracle where they were not
built), two GPU runs with the default FP64-atomic current sum (A, B) and two
with the bit-reproducible fixed-point sum (D1, D2) -- and writes, per step,
the largest relative difference over the fields E, B and the particle
positions and momenta (each array's max |a - b| / max |b|) of

  A vs reference, D1 vs reference   (GPU against the reference)
  A vs B, D1 vs D2                  (GPU against GPU: summation order only)

as one JSON object per line to `--out`.

    python tests/divergence_curve.py --steps 200 --out gpurun_out/curve.jsonl
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import checkers  # noqa: E402
from aprl_b200 import native, workloads  # noqa: E402


def snapshot(run):
    fields = [run.get_field(a) for a in range(6)]
    p = run.get_particles()
    return fields, p


NAMES = ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "x", "y", "z", "ux", "uy", "uz")


def per_array(a, b):
    """max |a - b| / max |b| for each field component and particle coordinate."""
    out = [checkers.max_relative(x, y) for x, y in zip(a[0], b[0])]
    if not np.array_equal(a[1]["id"], b[1]["id"]):
        return [float("inf")] * len(NAMES)
    out += [checkers.max_relative(a[1][k], b[1][k]) for k in ("x", "y", "z", "ux", "uy", "uz")]
    return out


def vector_rel(a, b):
    """The field differences against the largest magnitude of the whole E
    (or B) field, max over components; particles as in per_array."""
    out = []
    for group in ((0, 1, 2), (3, 4, 5)):
        scale = max(float(np.max(np.abs(b[0][c]))) for c in group)
        diff = max(float(np.max(np.abs(a[0][c] - b[0][c]))) for c in group)
        out.append(diff / scale if scale else diff)
    return out


def max_rel(a, b):
    return max(per_array(a, b))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--out", default="divergence.jsonl")
    args = ap.parse_args(argv)
    w = workloads.drift_c1(steps=args.steps + 2)
    if checkers.reference_available():
        binding = checkers.reference()
        binding.lib.ref_set_threads(os.cpu_count() or 1)
        name = "reference"
    else:
        binding = checkers.oracle()
        name = "oracle"
    ref = checkers.run(binding, w)
    lib = native.load()
    det_cfg = workloads.with_determinism(w.config)
    runs = {"A": native.Run(lib, w.config).load_workload(w),
            "B": native.Run(lib, w.config).load_workload(w),
            "D1": native.Run(lib, det_cfg).load_workload(w),
            "D2": native.Run(lib, det_cfg).load_workload(w)}
    t0 = time.time()
    with open(args.out, "w") as f:
        for step in range(1, args.steps + 1):
            ref.step(1)
            for r in runs.values():
                r.step(1)
            s = {k: snapshot(r) for k, r in runs.items()}
            so = snapshot(ref)
            arrays = {"A_ref": per_array(s["A"], so), "D1_ref": per_array(s["D1"], so),
                      "A_B": per_array(s["A"], s["B"]), "D1_D2": per_array(s["D1"], s["D2"])}
            row = {"step": step, "against": name}
            row.update({k: max(v) for k, v in arrays.items()})
            row.update({k + "_worst": NAMES[int(np.argmax(v))] for k, v in arrays.items()})
            row.update({k + "_arrays": dict(zip(NAMES, v)) for k, v in arrays.items()})
            row["A_ref_EB_vector"] = vector_rel(s["A"], so)
            row["D1_ref_EB_vector"] = vector_rel(s["D1"], so)
            row["A_B_EB_vector"] = vector_rel(s["A"], s["B"])
            row.update({
                "particles": int(ref.stats()["particles"]),
                "iterations_equal": all(r.stats()["iterations"] == ref.stats()["iterations"]
                                        for r in runs.values()),
                "elapsed_s": round(time.time() - t0, 1)})
            f.write(json.dumps(row) + "\n")
            f.flush()
            if step % 10 == 0 or step == 1:
                print(json.dumps({k: v for k, v in row.items() if not k.endswith("_arrays")}),
                      flush=True)


if __name__ == "__main__":
    main()
