"""The oracle reproduces, bit for bit, fixtures generated from the
reference's own translation units (tests/golden/make_golden.py); the CUDA
path reproduces them to the FP64 drop-in tolerance."""
import os

import numpy as np
import pytest

import checkers
from aprl_b200 import abi, native

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["binomial3_dipole", "quintic_dipole", "binomial3_stream"]
STATS = ("iterations", "total_iterations", "exits", "carriers", "particles",
         "pending", "admitted", "activations", "held")


def load_case(name):
    d = np.load(os.path.join(HERE, name + ".npz"))
    cfg = abi.RunConfig.from_bytes(d["config"].tobytes())
    return cfg, d


def run_from_fixture(binding, cfg, d):
    r = native.Run(binding, cfg)
    r.set_reference([d[f"in_ref_{a}"] for a in range(6)])
    for a in range(9):
        if f"in_field_{a}" in d.files:
            r.set_field(a, d[f"in_field_{a}"])
    r.set_particles({k[5:]: d[k] for k in d.files if k.startswith("in_p_")})
    if "in_held" in d.files:
        r.set_held(d["in_held"], d["in_p_beta_held"])
    return r


def check_held(r, d):
    if "out_held_frozen" in d.files:
        frozen, beta = r.get_held()
        np.testing.assert_array_equal(frozen, d["out_held_frozen"])
        np.testing.assert_array_equal(beta, d["out_held_beta"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference_fixture(name):
    cfg, d = load_case(name)
    r = run_from_fixture(checkers.oracle(), cfg, d)
    r.step(int(d["steps"]))
    s = checkers.state(r)
    for a in range(6):
        np.testing.assert_array_equal(s["fields"][a], d[f"out_field_{a}"])
    for h in range(12):
        np.testing.assert_array_equal(s["histories"][h], d[f"out_hist_{h}"])
    for k, v in s["particles"].items():
        np.testing.assert_array_equal(v, d["out_p_" + k])
    for k, v in s["carriers"].items():
        np.testing.assert_array_equal(v, d["out_c_" + k])
    for k in STATS:
        assert s["stats"][k] == int(d["out_stat_" + k])
    check_held(r, d)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_matches_reference_fixture(name):
    """J is accumulated with FP64 atomics: 1e-12 relative, integers exact."""
    cfg, d = load_case(name)
    r = run_from_fixture(native.load(), cfg, d)
    r.step(int(d["steps"]))
    s = checkers.state(r)
    for a in range(6):
        assert checkers.max_relative(s["fields"][a], d[f"out_field_{a}"]) <= 1e-12
    for h in range(12):
        assert checkers.max_relative(s["histories"][h], d[f"out_hist_{h}"]) <= 1e-12
    np.testing.assert_array_equal(s["particles"]["id"], d["out_p_id"])
    for k in ("x", "y", "z", "ux", "uy", "uz"):
        assert checkers.max_relative(s["particles"][k], d["out_p_" + k]) <= 1e-12
    for k in STATS:
        assert s["stats"][k] == int(d["out_stat_" + k])
    check_held(r, d)
