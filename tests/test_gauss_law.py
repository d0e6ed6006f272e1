"""Discrete Gauss law, eps0 div E - rho, on the device (aprl_run_gauss_law).

The Ampere update adds the plain Yee curl of B, whose discrete divergence
vanishes, and the current of each shape's deposit conserves its node
charge density (F3 x binomial3 for linear-binomial3; linear x, y and the
quintic node basis in z for quintic-compensated, whose Jz uses the edge
basis); so G = eps0 div E - rho at the interior nodes (away
from the CPML, the PEC faces and the inlet plane) keeps its value through a
step up to roundoff.  The restatement of rho and div E in numpy
(tests/checkers.py) is checked for that property on the oracle; the CUDA
reduction must reproduce it node by node on the GPU's own state and show
the same property.
"""
import numpy as np
import pytest

import checkers
from aprl_b200 import native, workloads

BOUND = 1e-13   # |G_after - G_before| / max |rho| at the inner nodes (measured 1e-15)


SHAPES = ["linear-binomial3", "quintic-compensated"]


def interior_case(shape="linear-binomial3"):
    return workloads.small_case(steps=2, particles=300, z_fraction=(0.3, 0.6), seed=11,
                                shape=shape)


def numpy_gauss(run, cfg):
    st = run.stats()
    origin = (cfg.reference_origin[0], cfg.reference_origin[1], st["origin_z"])
    return checkers.gauss_residual(cfg, origin, run.get_particles(),
                                   run.get_field(0), run.get_field(1), run.get_field(2))


def inner(cfg, a, margin=2):
    cx, cy = cfg.cpml_cells_x, cfg.cpml_cells_y
    return a[margin:cfg.nz + 1 - margin, cy + margin:cfg.ny + 1 - cy - margin,
             cx + margin:cfg.nx + 1 - cx - margin]


def step_by_seams(run):
    run.advance_magnetic()
    run.preview_electric()
    for _ in range(3):
        run.coupling_trial()
    run.commit_electric()


@pytest.mark.parametrize("shape", SHAPES)
def test_oracle_step_keeps_gauss_law(shape):
    w = interior_case(shape)
    cfg = w.config
    run = checkers.run(checkers.oracle(), w)
    g0, rho0 = numpy_gauss(run, cfg)
    step_by_seams(run)
    g1, rho1 = numpy_gauss(run, cfg)
    scale = max(np.abs(rho0).max(), np.abs(rho1).max())
    assert scale > 0 and np.abs(inner(cfg, g0)).max() > 1e3 * BOUND * scale
    assert np.abs(inner(cfg, g1 - g0)).max() <= BOUND * scale


@pytest.mark.gpu
@pytest.mark.parametrize("shape", SHAPES)
def test_gpu_gauss_law_matches_numpy_and_is_kept_by_a_step(shape):
    w = interior_case(shape)
    cfg = w.config
    run = checkers.run(native.load(), w)
    s0, d0 = run.gauss_law(residual=True)
    g0, rho0 = numpy_gauss(run, cfg)
    scale = np.abs(rho0).max()
    assert s0["outside"] == 0
    assert np.abs(d0 - g0).max() <= 1e-13 * scale
    assert s0["max_charge_density"] == pytest.approx(scale, rel=1e-13)
    assert s0["total_charge"] == pytest.approx(np.sum(w.particles["charge"]), rel=1e-12)
    lo = inner(cfg, g0, margin=1)
    assert s0["interior_nodes"] == lo.size
    assert s0["max_residual"] == pytest.approx(np.abs(lo).max(), rel=1e-12)
    assert s0["rms_residual"] == pytest.approx(np.sqrt(np.mean(lo ** 2)), rel=1e-12)
    step_by_seams(run)
    s1, d1 = run.gauss_law(residual=True)
    assert np.abs(inner(cfg, d1 - d0)).max() <= BOUND * scale
