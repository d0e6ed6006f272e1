"""The inlet reference prepared on the GPU (aprl_run_prepare_reference).

The reference prepares its inlet supply with BlockedCowanReference, a modal
solve of the Cowan relativistic Poisson problem on the whole reference grid
that its own check holds to the Cowan initializer on the same grid within
the CG tolerance (verification/blocked_cowan_reference_checks.cpp:61-130).
Its translation unit is built into oracle/_ref over a stand-in for the three
FFTW calls it makes (oracle/ref/fftw_shim: the type-I sine transform by
direct sums), so the oracle's initializer is held to the reference's own
blocked solve here, with the CIC source and with the shaped source the
moving window uses (the run's shape), and the GPU's open-transverse-wall
reference is held to the reference's own open solve.  The GPU path runs the initializer
(CG or the same modal solve) on the reference grid; its tables must equal
the oracle's to the tolerance of the self-field tests, and a run stepping on
them must follow the oracle stepping on the oracle's tables.
"""
import numpy as np
import pytest

import checkers
from aprl_b200 import abi, native, workloads

BOUND = 1e-9
# GPU against the reference's own open-wall solve: both are direct solves of
# the same lifted problem (sine sums against FFTW's transform stand-in,
# block sums against serial Coulomb sums), so only rounding separates them.
OPEN_BOUND = 1e-11


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


def oracle_tables(w, source_shape="cic"):
    big = reference_grid(w.config)
    run = native.Run(checkers.oracle(), big)
    run.set_particles(w.particles)
    report = run.initialize_self_field(abi.self_field_config(big, source_shape=source_shape))
    return [run.get_field(a) for a in range(6)], report


def blocked_tables(w, report, shaped, directory, open_transverse=False):
    """The reference's own BlockedCowanReference on the same reference grid,
    with the initializer's mean beta_z and guards (as the moving window
    prepares it, src/simulation_moving_window.cpp:145-148)."""
    big = reference_grid(w.config)
    sf = abi.self_field_config(big)
    return checkers.blocked_reference(w.config, w.particles, report["mean_beta_z"],
                                      [sf.guard_cells[a] for a in range(3)], 8, shaped,
                                      str(directory), open_transverse=open_transverse)


def wide_case():
    """A 48 x 48 x 64 grid with the bunch near its axis: about 20 cells from
    the outer transverse faces, the open-wall table is sampled on a coarse
    grid and interpolated (the reference's checked error about 1e-11), not
    evaluated at every node."""
    w = workloads.self_field_case(8.84e6, nx=48, ny=48, nz=64, particles=2000)
    w.config.reference_nz = w.config.initial_offset + w.config.nz + 4
    w.reference = []
    return w


def support_touching_case(shape):
    """The covering case with one particle whose shaped support reaches a
    zero-potential face while its CIC support stays inside: the binomial3
    x weights (nodes floor(x)-1 ..) reach the face x = guard, the quintic
    z basis (nodes floor(z)-5 ..) the lower z face."""
    w = covering_case()
    cfg = w.config
    cfg.shape = shape
    w.particles = dict(w.particles)
    if shape == abi.SHAPE_LINEAR_BINOMIAL3:
        x = np.array(w.particles["x"], dtype=np.float64)
        x[0] = cfg.reference_origin[0] + (cfg.cpml_cells_x + 1.5) * cfg.dx
        w.particles["x"] = x
    else:
        z = np.array(w.particles["z"], dtype=np.float64)
        z[0] = cfg.reference_origin[2] + 3.5 * cfg.dz
        w.particles["z"] = z
    return w


SHAPES = [abi.SHAPE_LINEAR_BINOMIAL3, abi.SHAPE_QUINTIC_COMPENSATED]


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


@pytest.mark.skipif(not checkers.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("source", ["cic", "run-shape"])
def test_oracle_prepared_reference_matches_the_references_blocked_solve(shape, source, tmp_path):
    """The reference's BlockedCowanReference (its deposit, sine-mode and
    Thomas solve and native E/B, built over the FFTW stand-in) against the
    oracle's initializer with the same source, to the CG tolerance as the
    reference's own check holds them (verification/
    blocked_cowan_reference_checks.cpp:61-130)."""
    w = covering_case()
    w.config.shape = shape
    tables, report = oracle_tables(w, source)
    directory = tmp_path / "blocked"
    blocked, summary = blocked_tables(w, report, source != "cic", directory)
    for a in range(6):
        assert checkers.max_relative(blocked[a], tables[a]) <= BOUND, a
    assert summary[2] > 0.0 and summary[3] > 0.0  # positive Thomas pivots and modes
    assert abs(summary[1] - summary[0]) <= 1e-12 * abs(summary[0])  # charge conserved
    assert not directory.exists()


@pytest.mark.skipif(not checkers.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("shape", SHAPES)
def test_shaped_source_touching_the_guard_is_refused_like_the_reference(shape, tmp_path):
    w = support_touching_case(shape)
    big = reference_grid(w.config)
    run = native.Run(checkers.oracle(), big)
    run.set_particles(w.particles)
    with pytest.raises(native.AprlError) as oracle_error:
        run.initialize_self_field(abi.self_field_config(big, source_shape="run-shape"))
    with pytest.raises(native.AprlError) as reference_error:
        blocked_tables(w, {"mean_beta_z": 0.5}, True, tmp_path / "blocked")
    for e in (oracle_error.value, reference_error.value):
        assert e.status == abi.APRL_ERR_INVALID_ARGUMENT
        assert e.message.startswith("Reference charge support touches Dirichlet surface")
    # the CIC source of the same bunch stays inside the box
    run.initialize_self_field(abi.self_field_config(big))


def test_shaped_source_has_no_cpml_padding():
    w = covering_case()
    big = reference_grid(w.config)
    run = native.Run(checkers.oracle(), big)
    run.set_particles(w.particles)
    with pytest.raises(native.AprlError) as e:
        run.initialize_self_field(abi.self_field_config(
            big, source_shape="run-shape", include_transverse_cpml_particles=True))
    assert e.value.status == abi.APRL_ERR_INVALID_ARGUMENT


@pytest.mark.gpu
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("solver", ["cg", "modal"])
def test_gpu_shaped_prepared_reference_matches_the_oracle(shape, solver):
    w = covering_case()
    cfg = w.config
    cfg.shape = shape
    tables, expected = oracle_tables(w, "run-shape")
    g = native.Run(native.load(), cfg)
    g.set_particles(w.particles)
    g.prepare_reference(w.particles, abi.self_field_config(cfg, solver=solver,
                                                           source_shape="run-shape"))
    for a in range(6):
        assert checkers.max_relative(g.get_reference(a), tables[a]) <= BOUND, a


@pytest.mark.gpu
@pytest.mark.parametrize("shape", SHAPES)
def test_gpu_shaped_source_touching_the_guard_is_refused(shape):
    w = support_touching_case(shape)
    g = native.Run(native.load(), w.config)
    g.set_particles(w.particles)
    with pytest.raises(native.AprlError) as e:
        g.prepare_reference(w.particles, abi.self_field_config(w.config,
                                                               source_shape="run-shape"))
    assert e.value.status == abi.APRL_ERR_INVALID_ARGUMENT
    assert e.value.message.startswith("Reference charge support touches Dirichlet surface")


@pytest.mark.gpu
@pytest.mark.skipif(not checkers.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("source", ["cic", "run-shape"])
def test_gpu_open_transverse_reference_matches_the_references_blocked_solve(shape, source,
                                                                           tmp_path):
    """The open-transverse-wall reference (mesh.moving_window.
    open_transverse_reference): the GPU's wall table, lifted modal solve and
    face smoothing against the reference's own BlockedCowanReference with
    openTransverse on the same grid, source and beta."""
    w = covering_case()
    cfg = w.config
    cfg.shape = shape
    g = native.Run(native.load(), cfg)
    g.set_particles(w.particles)
    report = g.prepare_reference(w.particles, abi.self_field_config(
        cfg, solver="modal", source_shape=source, open_transverse=True))
    directory = tmp_path / "blocked"
    blocked, summary = blocked_tables(w, report, source != "cic", directory, open_transverse=True)
    for a in range(6):
        assert checkers.max_relative(g.get_reference(a), blocked[a]) <= OPEN_BOUND, a
    assert not directory.exists()


@pytest.mark.gpu
@pytest.mark.skipif(not checkers.reference_available(), reason="oracle/_ref not built")
def test_gpu_open_transverse_reference_interpolated_wall_matches(tmp_path):
    w = wide_case()
    cfg = w.config
    g = native.Run(native.load(), cfg)
    g.set_particles(w.particles)
    report = g.prepare_reference(w.particles, abi.self_field_config(
        cfg, solver="modal", source_shape="run-shape", open_transverse=True))
    blocked, summary = blocked_tables(w, report, True, tmp_path / "blocked",
                                      open_transverse=True)
    assert 0.0 < summary[4] < 2e-7 and summary[5] == 0  # interpolated, no direct fallback
    for a in range(6):
        assert checkers.max_relative(g.get_reference(a), blocked[a]) <= OPEN_BOUND, a


@pytest.mark.gpu
def test_gpu_open_transverse_reference_refuses_what_the_reference_refuses():
    w = covering_case()
    cfg = w.config
    g = native.Run(native.load(), cfg)
    g.set_particles(w.particles)
    for kwargs in ({"solver": "cg"}, {"solver": "modal", "include_transverse_cpml_particles": True}):
        with pytest.raises(native.AprlError) as e:
            g.prepare_reference(w.particles, abi.self_field_config(cfg, open_transverse=True,
                                                                   **kwargs))
        assert e.value.status == abi.APRL_ERR_INVALID_ARGUMENT
    c = abi.self_field_config(cfg, solver="modal", open_transverse=True)
    c.guard_cells[2] = 1
    with pytest.raises(native.AprlError) as e:
        g.prepare_reference(w.particles, c)
    assert e.value.message == "Open transverse reference requires only transverse CPML"
