"""The plain-C oracle against the reference's own translation units.

oracle/_ref/libaprl_ref.so is compiled from the APRL sources
(EBFieldGrid, EBConvolutionalPML, MovingWindowFields,
ConservativeSourceCoupling, longitudinal_shape, ChargeConservingCurrentDepositor,
ParticleCPMLRegion, ParticleOpenBoundary, BoostFrameTransform,
SIFieldSourceSet).  The oracle must reproduce it bit for bit: whole coupled
steps (fields, CPML histories, particles, carriers, counters) and the single
operators."""
import ctypes as C

import numpy as np
import pytest

import checkers
from aprl_b200 import abi, workloads

pytestmark = pytest.mark.skipif(not checkers.reference_available(),
                                reason="reference translation units not built")


def assert_states_identical(a, b):
    for x, y in zip(a["fields"], b["fields"]):
        np.testing.assert_array_equal(x, y)
    for x, y in zip(a["histories"], b["histories"]):
        np.testing.assert_array_equal(x, y)
    for k in a["particles"]:
        np.testing.assert_array_equal(a["particles"][k], b["particles"][k])
    for k in a["carriers"]:
        np.testing.assert_array_equal(a["carriers"][k], b["carriers"][k])
    assert a["stats"] == b["stats"]


MAGNETS = {
    "dipole": lambda: [workloads.dipole(1.0)],
    "none": lambda: [],
    "undulator": lambda: [workloads.planar_undulator(1.0, 0.03, -1.0, 100)],
    "quadrupole-dipole": lambda: [workloads.dipole(0.5, angle=0.3), _quadrupole()],
}


def _quadrupole():
    m = abi.Magnet()
    m.type = abi.MAGNET_QUADRUPOLE
    m.center[2] = -5.0
    m.length = 50.0
    m.quadrupole_gradient = 20.0
    m.polarization_angle = 0.2
    m.cos_angle = np.cos(0.2)
    m.sin_angle = np.sin(0.2)
    return m


@pytest.mark.parametrize("shape", ["linear-binomial3", "quintic-compensated"])
@pytest.mark.parametrize("magnets", sorted(MAGNETS))
def test_steps_bit_identical(shape, magnets):
    w = workloads.small_case(steps=4, shape=shape, magnets=MAGNETS[magnets]())
    o = checkers.run(checkers.oracle(), w)
    r = checkers.run(checkers.reference(), w)
    for _ in range(4):
        o.step(1)
        r.step(1)
        assert_states_identical(checkers.state(o), checkers.state(r))


def test_operator_sequence_bit_identical():
    """Each seam separately: magnetic, preview, trials, commit, shift."""
    w = workloads.small_case(steps=3, particles=300)
    o = checkers.run(checkers.oracle(), w)
    r = checkers.run(checkers.reference(), w)
    for run in (o, r):
        run.advance_magnetic()
    for a in range(6):
        np.testing.assert_array_equal(o.get_field(a), r.get_field(a))
    for run in (o, r):
        run.preview_electric()
    for a in range(3):
        np.testing.assert_array_equal(o.get_field(a), r.get_field(a))
    for _ in range(3):
        np.testing.assert_array_equal(o.coupling_trial(), r.coupling_trial())
        for a in range(9):
            np.testing.assert_array_equal(o.get_field(a), r.get_field(a))
    for run in (o, r):
        run.commit_electric()
        run.shift()
    assert_states_identical(checkers.state(o), checkers.state(r))


def test_carrier_heavy_run_bit_identical():
    w = workloads.small_case(nx=24, ny=20, nz=48, particles=1500, steps=6,
                             z_fraction=(0.02, 0.995), margin_cells=0)
    o = checkers.run(checkers.oracle(), w)
    r = checkers.run(checkers.reference(), w)
    o.step(6)
    r.step(6)
    so, sr = checkers.state(o), checkers.state(r)
    assert so["stats"]["exits"] > 0 and so["stats"]["carriers"] > 0
    assert_states_identical(so, sr)


def test_cowan_coefficients_identical():
    o, r = checkers.oracle(), checkers.reference()
    for dx, dy, dz in [(5e-6, 5e-6, 2e-6), (1.0, 1.0, 1.0), (3e-6, 7e-6, 1e-6)]:
        a = (C.c_double * 12)()
        b = (C.c_double * 12)()
        o("cowan_coefficients", dx, dy, dz, a)
        r("cowan_coefficients", dx, dy, dz, b)
        assert list(a) == list(b)


@pytest.mark.parametrize("shape", ["linear-binomial3", "quintic-compensated"])
def test_shape_weights_identical(shape):
    """151 seeded chords, as verification/transverse_binomial_checks.cpp:19-27."""
    cfg = workloads.make_config(22, 22, 22, 1.0, 1.0, 1.0, 3, 10.0, shape, 2)
    rng = np.random.default_rng(20031)
    origin = np.zeros(3)
    for path in range(151):
        a = rng.uniform(6.0, 15.0, 3)
        b = a + rng.uniform(-2.1, 2.1, 3)
        if path == 0:
            a, b = np.full(3, 8.0), np.full(3, 11.0)
        if path == 1:
            a = np.full(3, 10.0)
            b = a.copy()
        if path == 2:
            a, b = np.full(3, 9.5), np.full(3, 7.5)
        wo = checkers.shape_weights(checkers.oracle(), cfg, origin, a, b)
        wr = checkers.shape_weights(checkers.reference(), cfg, origin, a, b)
        for x, y in zip(wo, wr):
            np.testing.assert_array_equal(x, y)


def test_momentum_identical():
    lib_o, lib_r = checkers.oracle().lib, checkers.reference().lib
    rng = np.random.default_rng(7)
    d = lambda v: (C.c_double * 3)(*v)
    for _ in range(500):
        u = rng.normal(0.0, 50.0, 3)
        e = rng.normal(0.0, 1e9, 3)
        b = rng.normal(0.0, 2.0, 3)
        q, m = -1.6e-19 * 6e3, 9.1e-31 * 6e3
        h = rng.uniform(1e-16, 1e-13)
        uo, ur = d(u), d(u)
        io = lib_o.oracle_momentum(uo, d(e), d(b), q, m, h, 0.0)
        ir = lib_r.ref_momentum(ur, d(e), d(b), q, m, h, 0.0)
        assert io == ir
        assert list(uo) == list(ur)
        assert lib_o.oracle_gamma(d(u)) == lib_r.ref_gamma(d(u))


@pytest.mark.parametrize("shape", ["linear-binomial3", "quintic-compensated"])
def test_held_injection_bit_identical(shape):
    """Pending extraction, admission, frozen source support, activation kinks
    and upstream admission clips against the reference's
    PendingParticleQueue and prepareParticle path."""
    w = workloads.streaming_case(shape=shape, steps=12)
    o = checkers.run(checkers.oracle(), w)
    r = checkers.run(checkers.reference(), w)
    assert o.stats()["pending"] == r.stats()["pending"] > 0
    for _ in range(w.steps):
        o.step(1)
        r.step(1)
        assert_states_identical(checkers.state(o), checkers.state(r))
        for x, y in zip(o.get_held(), r.get_held()):
            np.testing.assert_array_equal(x, y)
    s = o.stats()
    assert s["admitted"] > 0 and s["activations"] > 0
