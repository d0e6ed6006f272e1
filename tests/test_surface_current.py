"""The reference's equivalent surface current
(mesh.moving_window.reference_surface_current; TransverseReferenceCurrent,
src/transverse_reference_current.h:12-28, .cpp:19-28, 46-63, 104-118).

Jz += curl_z(B_ref)/mu0 of the prepared reference, lerped to the step, at
the points of the physical region's four transverse faces, after every
trial's deposit and before the commit (src/simulation_source_coupling.cpp:44,
src/simulation.cpp:548-561).  The oracle restates it; the reference harness
writes the prepared values in the reference's own file format and lets the
reference's class apply them, so the oracle is pinned bit for bit to the
reference's apply.  The GPU follows the oracle to the FP64 tolerance."""
import numpy as np
import pytest

import checkers
from aprl_b200 import abi, native, workloads
from test_gpu_parity import compare_state

SHAPES = ["linear-binomial3", "quintic-compensated"]


def case(shape, steps=4):
    return workloads.with_reference_surface_current(workloads.small_case(steps=steps, shape=shape))


def without(w):
    cfg = abi.RunConfig.from_buffer_copy(bytes(w.config))
    cfg.reference_surface_current = 0
    return workloads.Workload(w.name, cfg, w.particles, w.reference, w.fields, steps=w.steps)


@pytest.mark.skipif(not checkers.reference_available(),
                    reason="reference translation units not built")
@pytest.mark.parametrize("shape", SHAPES)
def test_oracle_matches_reference_bitwise(shape):
    w = case(shape)
    o, r = checkers.run(checkers.oracle(), w), checkers.run(checkers.reference(), w)
    for _ in range(4):
        o.step(1)
        r.step(1)
        for a in range(6):
            np.testing.assert_array_equal(o.get_field(a), r.get_field(a))
        po, pr = o.get_particles(), r.get_particles()
        for k in po:
            np.testing.assert_array_equal(po[k], pr[k])


def test_the_current_changes_the_fields():
    w = case("linear-binomial3")
    on, off = checkers.run(checkers.oracle(), w), checkers.run(checkers.oracle(), without(w))
    on.step(2)
    off.step(2)
    assert max(checkers.max_relative(on.get_field(a), off.get_field(a)) for a in range(6)) > 1e-9


def test_a_reference_shorter_than_the_window_is_refused():
    w = workloads.small_case(steps=4)
    w.config.reference_surface_current = 1     # reference table covers the inlet planes only
    r = checkers.run(checkers.oracle(), w)
    with pytest.raises(native.AprlError) as info:
        r.step(1)
    assert info.value.status == abi.APRL_ERR_OUT_OF_RANGE
    assert info.value.message == "Reference surface-current query outside domain"


@pytest.mark.gpu
@pytest.mark.parametrize("deterministic", [False, True])
@pytest.mark.parametrize("shape", SHAPES)
def test_gpu_matches_oracle(shape, deterministic):
    w = case(shape)
    w.config = workloads.with_determinism(w.config, deterministic)
    g = native.Run(native.load(), w.config).load_workload(w)
    o = checkers.run(checkers.oracle(), w)
    for _ in range(4):
        g.step(1)
        o.step(1)
        compare_state(g, o)


@pytest.mark.gpu
def test_gpu_refuses_a_reference_shorter_than_the_window():
    w = workloads.small_case(steps=4)
    w.config.reference_surface_current = 1
    g = native.Run(native.load(), w.config).load_workload(w)
    with pytest.raises(native.AprlError) as info:
        g.step(1)
    assert info.value.status == abi.APRL_ERR_OUT_OF_RANGE
    assert info.value.message.startswith("Reference surface-current query outside domain")


@pytest.mark.skipif(not checkers.reference_available(),
                    reason="reference translation units not built")
@pytest.mark.parametrize("shape", SHAPES)
def test_file_writer_matches_the_references_own_prepare(shape, tmp_path):
    """The harness writes the prepared surface current from reference
    tables; the reference's own TransverseReferenceCurrent::prepare reads
    its BlockedCowanReference.  Over the same blocked reference of a bunch
    (the run's shaped source, as the moving window prepares both) the two
    give the same values bit for bit."""
    import test_prepared_reference as prepared
    w = prepared.covering_case()
    w.config.shape = abi.SHAPES[shape]
    reference, tables = checkers.surface_current_pin(w.config, w.particles, 0.5,
                                                     str(tmp_path / "blocked"))
    assert reference.shape == tables.shape and np.abs(reference).max() > 0.0
    assert np.array_equal(reference, tables)
    assert not (tmp_path / "blocked").exists()
