"""RelativisticBorisPusher::push (src/eb_particles.cpp:99-139, 207-216)
through the C ABI (aprl_boris_push).

The oracle's restatement equals the reference's own translation unit bit for
bit on seeded particles and fields; the GPU equals the oracle bit for bit
(same operation order, no FMA contraction).  The gyro-phase check restates
verification/core_checks.cpp:665-714: a 1 T gyration of an electron with
u = 2 over one cyclotron period in 32 and 64 steps -- phase error below
6e-3 at 64 steps, second-order convergence (ratio above 3.7), and gamma
conserved to 2e-14.
"""
import ctypes as C
import math

import numpy as np
import pytest

import checkers
from aprl_b200 import abi, native

E_CHARGE = 1.602176634e-19
E_MASS = 9.1093837139e-31


def seeded(count=500, seed=7):
    rng = np.random.default_rng(seed)
    p = {"x": rng.uniform(-1e-4, 1e-4, count), "y": rng.uniform(-1e-4, 1e-4, count),
         "z": rng.uniform(0, 1e-3, count),
         "ux": rng.normal(0, 3, count), "uy": rng.normal(0, 3, count),
         "uz": rng.normal(50, 20, count),
         "q": rng.choice([-1.0, 1.0], count) * E_CHARGE * rng.uniform(1, 1e4, count),
         "m": E_MASS * rng.uniform(1, 1e4, count)}
    p["m"] = np.abs(p["q"]) / E_CHARGE * E_MASS
    e = rng.normal(0, 1e8, (count, 3))
    b = rng.normal(0, 2.0, (count, 3))
    return p, e, b


def push(binding, p, e, b, dt):
    out = {k: np.array(v, dtype=np.float64) for k, v in p.items()}
    d = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    e = np.ascontiguousarray(e, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    binding("boris_push", out["x"].size, d(out["x"]), d(out["y"]), d(out["z"]), d(out["ux"]),
            d(out["uy"]), d(out["uz"]), d(out["q"]), d(out["m"]), d(e), d(b), dt)
    return out


def gyration(binding, steps):
    """verification/core_checks.cpp:670-694 through aprl_boris_push."""
    u0 = np.array([2.0, 0.0, 0.0])
    gamma0 = math.sqrt(1.0 + 4.0)
    omega = E_CHARGE / (E_MASS * gamma0)
    dt = 2.0 * math.pi / omega / steps
    p = {"x": np.zeros(1), "y": np.zeros(1), "z": np.zeros(1), "ux": u0[:1].copy(),
         "uy": np.zeros(1), "uz": np.zeros(1), "q": np.array([-E_CHARGE]),
         "m": np.array([E_MASS])}
    for _ in range(steps):
        p = push(binding, p, np.zeros((1, 3)), np.array([[0.0, 0.0, 1.0]]), dt)
    u = np.array([p["ux"][0], p["uy"][0], p["uz"][0]])
    phase = abs(math.atan2(u[1], u[0]))
    gamma = checkers.oracle().lib.oracle_gamma(u.ctypes.data_as(C.POINTER(C.c_double)))
    return phase, abs(gamma - gamma0) / gamma0


def test_oracle_gyration_pins():
    coarse, fine = gyration(checkers.oracle(), 32), gyration(checkers.oracle(), 64)
    assert fine[0] < 6.0e-3
    assert coarse[0] / fine[0] > 3.7
    assert coarse[1] < 2.0e-14 and fine[1] < 2.0e-14


@pytest.mark.skipif(not checkers.reference_available(),
                    reason="reference translation units not built")
def test_oracle_equals_reference_bitwise():
    p, e, b = seeded()
    o = push(checkers.oracle(), p, e, b, 3.3e-15)
    r = push(checkers.reference(), p, e, b, 3.3e-15)
    for k in o:
        np.testing.assert_array_equal(o[k], r[k])


@pytest.mark.parametrize("binding", ["oracle", "reference"])
def test_invalid_parameters_are_refused(binding):
    if binding == "reference" and not checkers.reference_available():
        pytest.skip("reference translation units not built")
    lib = checkers.oracle() if binding == "oracle" else checkers.reference()
    p, e, b = seeded(4)
    p["m"][2] = 0.0
    with pytest.raises(native.AprlError) as info:
        push(lib, p, e, b, 1e-15)
    assert info.value.status == abi.APRL_ERR_INVALID_ARGUMENT
    assert info.value.message == "Invalid SI particle pusher parameters"


@pytest.mark.gpu
def test_gpu_equals_oracle_bitwise():
    p, e, b = seeded(20000, seed=11)
    g = push(native.load(), p, e, b, 3.3e-15)
    o = push(checkers.oracle(), p, e, b, 3.3e-15)
    for k in o:
        np.testing.assert_array_equal(g[k], o[k])


@pytest.mark.gpu
def test_gpu_gyration_pins_and_refusal():
    coarse, fine = gyration(native.load(), 32), gyration(native.load(), 64)
    assert fine[0] < 6.0e-3 and coarse[0] / fine[0] > 3.7
    assert coarse[1] < 2.0e-14 and fine[1] < 2.0e-14
    p, e, b = seeded(4)
    with pytest.raises(native.AprlError) as info:
        push(native.load(), p, e, b, -1.0)
    assert info.value.message == "Invalid SI particle pusher parameters"
