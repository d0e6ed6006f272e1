"""Generate the golden fixtures of tests/golden from the reference's own
translation units (oracle/_ref/libaprl_ref.so, built from the APRL sources by
oracle/build_oracle.py).  Each fixture holds the complete input of a small
seeded moving-window run (configuration, particles, held-injection state,
inlet reference table, start fields) and the reference's state after the
case's coupled steps.

Usage: python tests/golden/make_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import checkers  # noqa: E402
from aprl_b200 import workloads  # noqa: E402

CASES = {
    "binomial3_dipole": dict(nx=12, ny=12, nz=24, particles=120, steps=2,
                             shape="linear-binomial3", cpml=2, fields=False),
    "quintic_dipole": dict(nx=12, ny=12, nz=24, particles=100, steps=2,
                           shape="quintic-compensated", cpml=2, fields=False),
    # held lab-plane injection: pending, held and active particles
    "binomial3_stream": dict(nx=12, ny=12, nz=24, particles=160, steps=8,
                             shape="linear-binomial3", cpml=2, upstream_cells=12),
}


def workload(name):
    case = CASES[name]
    if "upstream_cells" in case:
        return workloads.streaming_case(**case)
    return workloads.small_case(**case)


def save(name, path):
    w = workload(name)
    r = checkers.run(checkers.reference(), w)
    r.step(CASES[name]["steps"])
    s = checkers.state(r)
    out = {"config": np.frombuffer(bytes(w.config), dtype=np.uint8),
           "steps": np.array(CASES[name]["steps"])}
    for k, v in w.particles.items():
        out["in_p_" + k] = v
    if getattr(w, "held", None) is not None:
        out["in_held"] = w.held
        frozen, beta = r.get_held()
        out["out_held_frozen"] = frozen
        out["out_held_beta"] = beta
    for a, t in enumerate(w.reference):
        out[f"in_ref_{a}"] = t
    for a, f in enumerate(w.fields):
        out[f"in_field_{a}"] = f
    for a, f in enumerate(s["fields"]):
        out[f"out_field_{a}"] = f
    for h, v in enumerate(s["histories"]):
        out[f"out_hist_{h}"] = v
    for k, v in s["particles"].items():
        out["out_p_" + k] = v
    for k, v in s["carriers"].items():
        out["out_c_" + k] = v
    for k in ("iterations", "total_iterations", "exits", "carriers", "particles",
              "pending", "admitted", "activations", "held"):
        out["out_stat_" + k] = np.array(s["stats"][k])
    np.savez_compressed(path, **out)


if __name__ == "__main__":
    if not checkers.reference_available():
        sys.exit("oracle/_ref/libaprl_ref.so is not built")
    for name in CASES:
        save(name, os.path.join(HERE, name + ".npz"))
        print("wrote", name)
