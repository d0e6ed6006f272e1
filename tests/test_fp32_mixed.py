"""FP32-mixed mode against the FP64 oracle.

The mode runs the field gathers in binary32 (weights, the orbit-averaged E
and B they read, and their accumulation) and everything else in binary64.
Its error is measured against the FP64 oracle on the same seeded input: the
lab detector-plane field (relative L2 over the plane, target 1e-5), the
particle states (same ids in the same order), and the grid fields.
"""
import numpy as np
import pytest

import checkers
from aprl_b200 import abi, native, workloads

DETECTOR_BOUND = 1e-5   # relative L2 over the plane, E and B separately
PARTICLE_BOUND = 1e-6   # relative to each coordinate's largest magnitude
FIELD_BOUND = 1e-3      # max node error relative to the component's maximum


def detector_error(a, b):
    a, b = a.reshape(-1, 6), b.reshape(-1, 6)
    return (np.linalg.norm(a[:, :3] - b[:, :3]) / np.linalg.norm(b[:, :3]),
            np.linalg.norm(a[:, 3:] - b[:, 3:]) / np.linalg.norm(b[:, 3:]))


def test_oracle_rejects_fp32_config():
    w = workloads.small_case(steps=2)
    with pytest.raises(native.AprlError):
        native.Run(checkers.oracle(), workloads.with_precision(w.config, "fp32-mixed"))


def test_precision_copy_sets_tolerances():
    w = workloads.small_case(steps=2)
    c = workloads.with_precision(w.config, "fp32-mixed")
    assert c.precision == abi.PRECISION_FP32_MIXED
    assert c.force_tolerance == workloads.FP32_FORCE_TOLERANCE
    assert workloads.with_precision(c, "fp64").force_tolerance == 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("shape", ["linear-binomial3", "quintic-compensated"])
def test_fp32_mixed_detector_field_within_target(shape):
    w = workloads.small_case(steps=10, shape=shape)
    o = checkers.run(checkers.oracle(), w)
    g = native.Run(native.load(), workloads.with_precision(w.config, "fp32-mixed")).load_workload(w)
    o.step(8)
    g.step(8)
    cfg = w.config
    for f in (0.3, 0.5, 0.7):
        z = cfg.boost_gamma * (f * cfg.nz * cfg.dz)
        e, b = detector_error(g.sample_field_plane(z), o.sample_field_plane(z))
        assert e <= DETECTOR_BOUND and b <= DETECTOR_BOUND, (f, e, b)
    pg, po = g.get_particles(), o.get_particles()
    np.testing.assert_array_equal(pg["id"], po["id"])
    for k in ("x", "y", "z", "ux", "uy", "uz"):
        assert checkers.max_relative(pg[k], po[k]) <= PARTICLE_BOUND, k
    for a in range(6):
        assert checkers.max_relative(g.get_field(a), o.get_field(a)) <= FIELD_BOUND, a
    st = g.stats()
    assert st["exits"] == o.stats()["exits"] and st["particles"] == o.stats()["particles"]


@pytest.mark.gpu
def test_fp32_mixed_held_injection_matches_oracle():
    w = workloads.streaming_case(steps=12)
    o = checkers.run(checkers.oracle(), w)
    g = native.Run(native.load(), workloads.with_precision(w.config, "fp32-mixed")).load_workload(w)
    o.step(12)
    g.step(12)
    so, sg = o.stats(), g.stats()
    for k in ("admitted", "activations", "held", "particles", "pending"):
        assert sg[k] == so[k], k
    pg, po = g.get_particles(), o.get_particles()
    np.testing.assert_array_equal(pg["id"], po["id"])
    for k in ("x", "y", "z", "ux", "uy", "uz"):
        assert checkers.max_relative(pg[k], po[k]) <= PARTICLE_BOUND, k
