"""The bit-reproducible mode (aprl_run_config.deterministic): every deposit
contribution is rounded once to a 128-bit fixed point and summed with
integer reductions, so J -- and with it every field, particle and carrier --
comes out with the same bits from one run to the next, whatever order the
GPU's atomics take.  The cell sort (stable radix sort), the compactions and
the residual sums are ordered in both modes.

Parity with the oracle holds to the FP64 drop-in tolerance in this mode as
well: the fixed-point sum differs from the reference's serial binary64 sum
of the same contributions by the latter's own rounding."""
import numpy as np
import pytest

import checkers
from aprl_b200 import native, workloads
from test_gpu_parity import compare_state

pytestmark = pytest.mark.gpu


def gpu_run(w):
    return native.Run(native.load(), w.config).load_workload(w)


def deterministic(w):
    w.config = workloads.with_determinism(w.config)
    return w


def assert_bitwise_equal(a, b):
    sa, sb = checkers.state(a), checkers.state(b)
    for x, y in zip(sa["fields"], sb["fields"]):
        np.testing.assert_array_equal(x, y)
    for x, y in zip(sa["histories"], sb["histories"]):
        np.testing.assert_array_equal(x, y)
    for k in sa["particles"]:
        np.testing.assert_array_equal(sa["particles"][k], sb["particles"][k])
    for k in sa["carriers"]:
        np.testing.assert_array_equal(sa["carriers"][k], sb["carriers"][k])
    for k, v in sa["stats"].items():
        assert v == sb["stats"][k], k
    for c in (6, 7, 8):
        np.testing.assert_array_equal(a.get_field(c), b.get_field(c))


@pytest.mark.parametrize("shape", ["linear-binomial3", "quintic-compensated"])
def test_two_runs_give_the_same_bits(shape):
    """Two runs of a grid whose bunch sheds CPML carriers and leaves through
    the exit plane: identical bits after every step."""
    w = deterministic(workloads.small_case(nx=32, ny=24, nz=80, particles=4000, steps=8,
                                           shape=shape, z_fraction=(0.02, 0.99),
                                           margin_cells=1))
    a, b = gpu_run(w), gpu_run(w)
    for _ in range(8):
        a.step(1)
        b.step(1)
        assert_bitwise_equal(a, b)
    assert a.stats()["carriers"] > 0 and a.stats()["exits"] > 0


def test_held_injection_with_charge_matched_inlet_gives_the_same_bits():
    w = deterministic(workloads.streaming_case(steps=10))
    w.config.inlet_charge_match = 1
    a, b = gpu_run(w), gpu_run(w)
    a.step(10)
    b.step(10)
    assert_bitwise_equal(a, b)
    assert a.stats()["admitted"] > 0


def test_fp32_mixed_gives_the_same_bits():
    w = deterministic(workloads.small_case(nx=32, ny=24, nz=80, particles=4000, steps=6,
                                           z_fraction=(0.02, 0.99), margin_cells=1))
    w.config = workloads.with_precision(w.config, "fp32-mixed")
    a, b = gpu_run(w), gpu_run(w)
    a.step(6)
    b.step(6)
    assert_bitwise_equal(a, b)


@pytest.mark.parametrize("shape", ["linear-binomial3", "quintic-compensated"])
def test_deterministic_mode_matches_oracle(shape):
    w = deterministic(workloads.small_case(nx=32, ny=24, nz=80, particles=4000, steps=8,
                                           shape=shape, z_fraction=(0.02, 0.99),
                                           margin_cells=1))
    g, o = gpu_run(w), checkers.run(checkers.oracle(), w)
    for _ in range(8):
        g.step(1)
        o.step(1)
        compare_state(g, o)


def test_held_injection_deterministic_matches_oracle():
    w = deterministic(workloads.streaming_case(steps=10))
    w.config.inlet_charge_match = 1
    g, o = gpu_run(w), checkers.run(checkers.oracle(), w)
    for _ in range(10):
        g.step(1)
        o.step(1)
        compare_state(g, o)
