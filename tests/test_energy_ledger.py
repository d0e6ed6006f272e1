"""The moving-window energy ledger (aprl_run_enable_energy_ledger /
aprl_run_energy_ledger).

The oracle restates MovingWindowFieldEnergyLedger and the ledger record's
field and particle sums (src/moving_window_fields.cpp:206-218, 265-290,
387-437, 444-516; src/simulation.cpp:3308-3340, 3591-3604) in long double,
with the reference's loop order.  It is pinned to the reference's own
MovingWindowFields ledger and EBFieldGrid cell operators (oracle/_ref) bit
for bit.  The CUDA path sums the same binary64 terms in double-double, in
another order; its values must agree to 1e-13 of the scale of each group of
quantities (energies, powers, particle sums), which is far below any
physical change of the ledger and far above the last-bit differences of a
long double versus a double-double sum.
"""
import numpy as np
import pytest

import checkers
from aprl_b200 import native, workloads

STEPS = 5
ENERGY_KEYS = ["inlet_overwrite_energy", "inserted_energy", "cropped_energy",
               "remap_energy", "field_energy_interior"]
COUNT_KEYS = ["overwrite_events", "flux_steps", "remap_steps", "particles"]
PARTICLE_KEYS = ["particle_kinetic", "particle_total", "represented_electrons"]
BOUND = 1e-13


def ledger_run(binding, w):
    run = checkers.run(binding, w)
    run.enable_energy_ledger()
    return run


def assert_close(a, b, bound=BOUND):
    for key in COUNT_KEYS:
        assert a[key] == b[key], key
    energies = ENERGY_KEYS + ["outward_energy"]
    scale = max(max(abs(np.asarray(b[k], dtype=float)).max() for k in energies), 1e-300)
    for k in energies:
        np.testing.assert_allclose(a[k], b[k], rtol=0, atol=bound * scale, err_msg=k)
    pscale = max(np.abs(b["boundary_power"]).max(), 1e-300)
    np.testing.assert_allclose(a["boundary_power"], b["boundary_power"], rtol=0,
                               atol=bound * pscale)
    for k in PARTICLE_KEYS:
        np.testing.assert_allclose(a[k], b[k], rtol=bound, atol=0, err_msg=k)


def test_oracle_ledger_is_nonzero_and_balanced_in_count():
    w = workloads.small_case(steps=STEPS)
    run = ledger_run(checkers.oracle(), w)
    before = run.energy_ledger()
    assert before["flux_steps"] == 0 and before["field_energy_interior"] > 0
    run.step(STEPS)
    led = run.energy_ledger()
    assert led["flux_steps"] == led["remap_steps"] == led["overwrite_events"] == STEPS
    assert led["inserted_energy"] > 0 and led["cropped_energy"] > 0
    assert led["remap_energy"] == pytest.approx(led["inserted_energy"] - led["cropped_energy"],
                                                rel=1e-12, abs=1e-12 * led["inserted_energy"])
    assert any(v != 0 for v in led["outward_energy"])
    assert led["particle_total"] > led["particle_kinetic"] > 0
    assert led["particles"] == run.particle_count()


def test_ledger_must_be_enabled_before_the_first_step():
    w = workloads.small_case(steps=2)
    run = checkers.run(checkers.oracle(), w)
    run.step(1)
    with pytest.raises(native.AprlError):
        run.enable_energy_ledger()


@pytest.mark.skipif(not checkers.reference_available(),
                    reason="reference translation units not built")
@pytest.mark.parametrize("shape", ["linear-binomial3", "quintic-compensated"])
def test_oracle_ledger_matches_reference_bitwise(shape):
    w = workloads.small_case(steps=STEPS, shape=shape)
    o = ledger_run(checkers.oracle(), w)
    r = ledger_run(checkers.reference(), w)
    assert o.energy_ledger() == r.energy_ledger()
    for _ in range(STEPS):
        o.step(1)
        r.step(1)
        assert o.energy_ledger() == r.energy_ledger()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32-mixed"])
def test_gpu_ledger_matches_oracle(precision):
    w = workloads.small_case(steps=STEPS)
    w.config = workloads.with_precision(w.config, precision)
    g = ledger_run(native.load(), w)
    o = ledger_run(checkers.oracle(), workloads.small_case(steps=STEPS))
    assert_close(g.energy_ledger(), o.energy_ledger())
    for _ in range(STEPS):
        g.step(1)
        o.step(1)
        if precision == "fp64":
            assert_close(g.energy_ledger(), o.energy_ledger())
    if precision == "fp32-mixed":
        # Binary32 gathers move the particles by ~1e-9 relative; the ledger
        # itself is summed the same way.
        assert_close(g.energy_ledger(), o.energy_ledger(), bound=1e-6)


@pytest.mark.gpu
def test_gpu_ledger_by_seams_and_disabled_run_unchanged():
    """The ledger follows seam-driven steps too, and a run without the
    ledger steps to the same state (up to the order of the FP64 current
    atomics, which differs between any two GPU runs)."""
    w = workloads.small_case(steps=3, particles=300)
    a = ledger_run(native.load(), w)
    b = ledger_run(native.load(), w)
    plain = checkers.run(native.load(), w)
    a.step(3)
    plain.step(3)
    for _ in range(3):
        b.advance_magnetic()
        b.preview_electric()
        for _ in range(3):
            b.coupling_trial()
        b.commit_electric()
        b.shift()
    la = a.energy_ledger()
    assert la["flux_steps"] == 3
    for x, y in zip(checkers.state(a)["fields"], checkers.state(plain)["fields"]):
        assert checkers.max_relative(x, y) <= 1e-12
    lb = b.energy_ledger()
    assert lb["flux_steps"] == 3
    assert lb["field_energy_interior"] > 0


@pytest.mark.gpu
def test_gpu_ledger_after_fields_replaced_between_steps():
    """A field written between steps changes the next step's start power:
    the ledger must measure the written fields, as the reference's begin
    does."""
    w = workloads.small_case(steps=4, particles=300)
    g = ledger_run(native.load(), w)
    o = ledger_run(checkers.oracle(), w)
    for run in (g, o):
        run.step(2)
    ex = o.get_field(0) * 1.01
    for run in (g, o):
        run.set_field(0, ex)
        run.step(2)
    assert_close(g.energy_ledger(), o.energy_ledger())
