"""The initial self-field solve (aprl_run_initialize_self_field,
EBGaussFieldInitializer::initialize, src/eb_initial_field.cpp:829-1095).

The oracle restates the initializer in long double with the reference's loop
orders and is pinned to the reference's own translation unit bit for bit
(fields and report), for the three models, with the transverse-CPML padding
and the held longitudinal velocity, and in its error path.  The CUDA path
deposits the charge with FP64 atomics and sums every dot product in
double-double, so its conjugate-gradient iterates differ from the oracle's
by roundoff: E and B must agree to 1e-9 of their largest value, the
iteration count to within one, the report's sums to 1e-12 (energies 1e-9).
"""
import numpy as np
import pytest

import checkers
from aprl_b200 import abi, native, workloads

MODELS = ["relativistic-poisson", "electrostatic-poisson", "cowan-relativistic-poisson"]
FIELD_BOUND = 1e-9


def solve(binding, w, **options):
    run = checkers.run(binding, w)
    report = run.initialize_self_field(abi.self_field_config(w.config, **options))
    return run, report, [run.get_field(a) for a in range(6)]


@pytest.mark.skipif(not checkers.reference_available(),
                    reason="reference translation units not built")
@pytest.mark.parametrize("energy", [5.11e6, 8.84e6])
@pytest.mark.parametrize("model", MODELS)
def test_oracle_matches_reference_bitwise(model, energy):
    w = workloads.self_field_case(energy)
    _, ro, fo = solve(checkers.oracle(), w, model=model)
    _, rr, fr = solve(checkers.reference(), w, model=model)
    assert ro == rr
    for a, b in zip(fo, fr):
        np.testing.assert_array_equal(a, b)


@pytest.mark.skipif(not checkers.reference_available(),
                    reason="reference translation units not built")
def test_oracle_matches_reference_with_cpml_sources_and_held_velocity():
    w = workloads.self_field_case(8.84e6, margin_cells=-1)
    opts = dict(include_transverse_cpml_particles=True, hold_transverse_until_activation=True)
    _, ro, fo = solve(checkers.oracle(), w, **opts)
    _, rr, fr = solve(checkers.reference(), w, **opts)
    assert ro == rr and ro["transverse_poisson_padding_cells"] == 2
    for a, b in zip(fo, fr):
        np.testing.assert_array_equal(a, b)


def test_oracle_gauss_law_and_charge_touching_the_boundary():
    w = workloads.self_field_case(8.84e6)
    _, rep, _ = solve(checkers.oracle(), w)
    assert rep["relative_residual"] <= 4e-10
    assert rep["total_charge"] == pytest.approx(np.sum(w.particles["charge"]), rel=1e-14)
    inside_cpml = workloads.self_field_case(8.84e6, margin_cells=-1)
    with pytest.raises(native.AprlError, match="touches the static zero-potential"):
        solve(checkers.oracle(), inside_cpml)


def assert_close(g, o):
    (rg, fg), (ro, fo) = g, o
    assert abs(int(rg["iterations"]) - int(ro["iterations"])) <= 1
    for key in ("total_charge", "mean_beta_z", "mean_beta_transverse"):
        assert rg[key] == pytest.approx(ro[key], rel=1e-12, abs=1e-15)
    for key in ("rms_position_cells", "centre_padding_rms"):
        np.testing.assert_allclose(rg[key], ro[key], rtol=1e-12)
    for key in ("initial_electric_energy", "initial_magnetic_energy"):
        assert rg[key] == pytest.approx(ro[key], rel=1e-9, abs=1e-30)
    assert rg["relative_residual"] <= 4e-10
    assert rg["static_field_guard_cells"] == ro["static_field_guard_cells"]
    assert rg["temporary_bytes"] == ro["temporary_bytes"]
    for a, b in zip(fg, fo):
        assert checkers.max_relative(a, b) <= FIELD_BOUND


@pytest.mark.gpu
@pytest.mark.parametrize("energy", [5.11e6, 8.84e6])
@pytest.mark.parametrize("model", MODELS)
def test_gpu_matches_oracle(model, energy):
    w = workloads.self_field_case(energy)
    _, rg, fg = solve(native.load(), w, model=model)
    _, ro, fo = solve(checkers.oracle(), w, model=model)
    assert_close((rg, fg), (ro, fo))


@pytest.mark.gpu
def test_gpu_with_cpml_sources_and_held_velocity_then_steps():
    w = workloads.self_field_case(8.84e6, margin_cells=-1)
    opts = dict(include_transverse_cpml_particles=True, hold_transverse_until_activation=True)
    run, rg, fg = solve(native.load(), w, **opts)
    _, ro, fo = solve(checkers.oracle(), w, **opts)
    assert_close((rg, fg), (ro, fo))
    # The run steps on from the solved fields like the oracle does.
    w2 = workloads.self_field_case(8.84e6)
    g, _, _ = solve(native.load(), w2)
    o, _, _ = solve(checkers.oracle(), w2)
    g.step(2)
    o.step(2)
    for a in range(6):
        assert checkers.max_relative(g.get_field(a), o.get_field(a)) <= FIELD_BOUND


@pytest.mark.gpu
def test_gpu_reports_charge_touching_the_boundary():
    w = workloads.self_field_case(8.84e6, margin_cells=-1)
    run = checkers.run(native.load(), w)
    with pytest.raises(native.AprlError, match="touches the static zero-potential"):
        run.initialize_self_field(abi.self_field_config(w.config))


def test_oracle_rejects_the_relativistic_bunch_like_the_reference():
    """A 1 GeV bunch boosted to gamma 10 moves at beta_z ~ 1 in the box: the
    Cowan operator fails its positive-definiteness bound on z, in the
    reference and the oracle alike, with the reference's message."""
    cfg = workloads.make_config(32, 32, 64, 5e-6, 5e-6, 2e-6, 10, 10.0, "linear-binomial3", 4,
                                magnets=[])
    bunch = workloads.gaussian_bunch(cfg, 500, 100e-12, 1e9, 50e-6, 20e-6, 1e-6, 1e-4, seed=17,
                                     margin_cells=2)
    w = workloads.Workload("relativistic", cfg, bunch, workloads.synthetic_reference(cfg), [],
                           steps=4)
    messages = []
    bindings = [checkers.oracle()] + ([checkers.reference()] if checkers.reference_available()
                                      else [])
    for binding in bindings:
        with pytest.raises(native.AprlError, match="positive-definiteness bound on axis 2") as e:
            solve(binding, w)
        messages.append(str(e.value).split(": ", 1)[1])
    assert len(set(messages)) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("energy", [5.11e6, 8.84e6])
@pytest.mark.parametrize("model", MODELS)
def test_gpu_modal_solve_matches_the_oracle_initializer(model, energy):
    """The transverse-mode direct solve (solver="modal", the blocked Cowan
    reference's method) on the same box gives the CG initializer's fields to
    the CG's own tolerance (the reference holds its modal reference to the
    initializer the same way, verification/blocked_cowan_reference_checks.cpp:61-130)."""
    w = workloads.self_field_case(energy)
    _, rg, fg = solve(native.load(), w, model=model, solver="modal")
    _, ro, fo = solve(checkers.oracle(), w, model=model)
    assert rg["iterations"] == 0
    assert rg["relative_residual"] <= 1e-11
    for a, b in zip(fg, fo):
        assert checkers.max_relative(a, b) <= FIELD_BOUND
    assert rg["total_charge"] == pytest.approx(ro["total_charge"], rel=1e-12)


@pytest.mark.gpu
def test_gpu_modal_solve_with_cpml_sources_and_held_velocity():
    w = workloads.self_field_case(8.84e6, margin_cells=-1)
    opts = dict(include_transverse_cpml_particles=True, hold_transverse_until_activation=True)
    _, rg, fg = solve(native.load(), w, solver="modal", **opts)
    _, ro, fo = solve(checkers.oracle(), w, **opts)
    assert rg["transverse_poisson_padding_cells"] == 2
    for a, b in zip(fg, fo):
        assert checkers.max_relative(a, b) <= FIELD_BOUND
