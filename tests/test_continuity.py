"""Discrete charge continuity of one coupled step's current.

The linear-binomial3 current of a chord is charge-conserving against the
charge density of the same shape (F3 node weights in x, linear in y,
binomial3 in z; verification/transverse_binomial_checks.cpp:12-66).  Over a
whole fixed-point trial, with every particle inside the trusted region, the
deposited J therefore satisfies

    (rho(end positions) - rho(start positions)) / dt + div J = 0

node by node up to roundoff (the reference's continuity audit,
verification/held_cut_bunch_probe.cpp:121-135).  The test drives the
operator seams (advance, preview, three trials, commit) so J and the
particle states belong to the same trial, and checks the oracle and the CUDA
path alike; on the GPU the current is summed with FP64 atomics in any order.
"""
import math

import numpy as np
import pytest

import checkers
from aprl_b200 import native, workloads

BOUND = 1e-12  # relative to max |rho| / dt


def continuity(cfg, origin, before, after, jx, jy, jz):
    r0, pad = checkers.charge_density(cfg, origin, before)
    r1, _ = checkers.charge_density(cfg, origin, after)
    drho = (r1 - r0)[pad:-pad, pad:-pad, pad:-pad] / cfg.dt  # nodes 0..n
    div = np.zeros_like(drho)
    # Jx (nz+1, ny+1, nx): x-edges between nodes i and i+1
    div[:, :, :-1] -= jx / cfg.dx
    div[:, :, 1:] += jx / cfg.dx
    div[:, :-1, :] -= jy / cfg.dy
    div[:, 1:, :] += jy / cfg.dy
    div[:-1, :, :] -= jz / cfg.dz
    div[1:, :, :] += jz / cfg.dz
    residual = drho - div
    scale = max(np.max(np.abs(r0)), np.max(np.abs(r1))) / cfg.dt
    return np.max(np.abs(residual)) / scale


def one_step_by_seams(run):
    run.advance_magnetic()
    run.preview_electric()
    for _ in range(3):
        run.coupling_trial()
    run.commit_electric()


def interior_case():
    # A compact bunch in the middle of the window: no exit-plane crossing and
    # no CPML entry in the first step.
    return workloads.small_case(steps=2, particles=300, z_fraction=(0.3, 0.6), seed=11)


def check(binding):
    w = interior_case()
    run = native.Run(binding, w.config).load_workload(w)
    before = run.get_particles()
    one_step_by_seams(run)
    st = run.stats()
    assert st["exits"] == 0 and sum(st["cpml_entries"]) == 0 and st["carriers"] == 0
    after = run.get_particles()
    np.testing.assert_array_equal(before["id"], after["id"])
    cfg = w.config
    origin = (cfg.reference_origin[0], cfg.reference_origin[1], st["origin_z"])
    jx, jy, jz = (run.get_field(a) for a in (6, 7, 8))
    assert np.max(np.abs(jz)) > 0.0
    return continuity(cfg, origin, before, after, jx, jy, jz)


def test_oracle_step_current_conserves_charge():
    assert check(checkers.oracle()) <= BOUND


@pytest.mark.gpu
def test_gpu_step_current_conserves_charge():
    assert check(native.load()) <= BOUND
