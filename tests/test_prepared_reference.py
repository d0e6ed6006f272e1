"""The inlet reference prepared on the GPU (aprl_run_prepare_reference).

The reference prepares its inlet supply with BlockedCowanReference, a modal
solve of the Cowan relativistic Poisson problem on the whole reference grid
that its own check holds to the Cowan initializer on the same grid within
the CG tolerance (verification/blocked_cowan_reference_checks.cpp:61-130);
its translation unit needs FFTW and is not built here.  The GPU path runs the
initializer itself on the reference grid.  Its tables must equal the
oracle's initializer on that grid (pinned bit for bit to the reference's
EBGaussFieldInitializer, tests/test_self_field.py) to the tolerance of the
self-field tests, and a run stepping on them must follow the oracle stepping
on the oracle's tables.
"""
import numpy as np
import pytest

import checkers
from aprl_b200 import abi, native, workloads

BOUND = 1e-9


def covering_case():
    """The self-field case with a reference grid that also covers the window
    (upstream supply, window and a 4-cell margin), as a prepared reference of
    the whole bunch's field must."""
    w = workloads.self_field_case(8.84e6)
    w.config.reference_nz = w.config.initial_offset + w.config.nz + 4
    w.reference = []
    return w


def reference_grid(cfg):
    big = abi.RunConfig.from_buffer_copy(bytes(cfg))
    big.nz = cfg.reference_nz
    big.initial_offset = 0
    return big


def oracle_tables(w):
    big = reference_grid(w.config)
    run = native.Run(checkers.oracle(), big)
    run.set_particles(w.particles)
    report = run.initialize_self_field(abi.self_field_config(big))
    return [run.get_field(a) for a in range(6)], report


def test_reference_grid_holds_the_window():
    w = covering_case()
    cfg = w.config
    assert cfg.reference_nz >= cfg.nz + cfg.initial_offset
    tables, report = oracle_tables(w)
    assert report["relative_residual"] <= 4e-10
    assert [t.shape for t in tables] == [abi.reference_shape(cfg, a)[::-1] for a in range(6)]


@pytest.mark.gpu
def test_gpu_prepared_reference_matches_the_oracle_and_steps():
    w = covering_case()
    cfg = w.config
    tables, expected = oracle_tables(w)
    g = native.Run(native.load(), cfg)
    g.set_particles(w.particles)
    report = g.prepare_reference(w.particles, abi.self_field_config(cfg))
    assert abs(int(report["iterations"]) - int(expected["iterations"])) <= 1
    for a in range(6):
        assert checkers.max_relative(g.get_reference(a), tables[a]) <= BOUND
    o = native.Run(checkers.oracle(), cfg)
    o.set_reference(tables)
    o.set_particles(w.particles)
    g.step(3)
    o.step(3)
    for a in range(6):
        assert checkers.max_relative(g.get_field(a), o.get_field(a)) <= BOUND
    assert g.stats()["particles"] == o.stats()["particles"]
