"""Known-answer pins of the oracle, restated from the reference's own tests
(no reference build needed):

* F3 discrete continuity of the wide-shape current, 151 seeded chords,
  bound 5e-13 (verification/transverse_binomial_checks.cpp:12-66);
* Cowan-z normalisation and stable-dispersion factorisation to 1e-12
  (src/eb_field.cpp:910-942);
* Lapenta-Markidis energy theorem: m c^2 (gamma1 - gamma0) equals the work
  q E . dx of the mean-velocity step, and a pure magnetic field conserves
  gamma (src/source_coupling_math.h:269-293).
"""
import ctypes as C
import math

import numpy as np
import pytest

import checkers
from aprl_b200 import workloads

C_LIGHT = 299792458.0


def _f3_node(f):
    return np.array([0.25 * (1.0 - f), 0.5 - 0.25 * f, 0.25 + 0.25 * f, 0.25 * f])


def _binomial3_z(z):
    cell = math.floor(z)
    f = z - cell
    v = np.zeros(4)
    for k, w in zip((-1, 0, 1), (0.25, 0.5, 0.25)):
        v[k + 1] += w * (1.0 - f)
        v[k + 2] += w * f
    return int(cell) - 1, v


def test_f3_current_continuity_151_chords():
    n = 22
    cfg = workloads.make_config(n, n, n, 1.0, 1.0, 1.0, 3, 10.0, "linear-binomial3", 2)
    rng = np.random.default_rng(20031)
    worst = 0.0
    for path in range(151):
        a = rng.uniform(6.0, 15.0, 3)
        b = a + rng.uniform(-2.1, 2.1, 3)
        if path == 0:
            a, b = np.full(3, 8.0), np.full(3, 11.0)
        if path == 2:
            a, b = np.full(3, 9.5), np.full(3, 7.5)
        axis, index, weight = checkers.shape_weights(checkers.oracle(), cfg, np.zeros(3), a, b)
        J = np.zeros((3, n, n, n))  # [axis][k][j][i]
        for ax, (i, j, k), w in zip(axis, index, weight):
            J[ax, k, j, i] += w
        rho = np.zeros((n, n, n))
        for sign, x in ((-1.0, a), (1.0, b)):
            i, j = math.floor(x[0]), math.floor(x[1])
            wx = _f3_node(x[0] - i)
            fy = x[1] - j
            first, wz = _binomial3_z(x[2])
            for u in range(4):
                for v in range(2):
                    for t in range(4):
                        rho[first + t, j + v, i - 1 + u] += sign * wx[u] * (fy if v else 1.0 - fy) * wz[t]
        d = b - a
        div = (d[0] * (J[0, 1:, 1:, 1:] - J[0, 1:, 1:, :-1]) +
               d[1] * (J[1, 1:, 1:, 1:] - J[1, 1:, :-1, 1:]) +
               d[2] * (J[2, 1:, 1:, 1:] - J[2, :-1, 1:, 1:]))
        worst = max(worst, float(np.max(np.abs(rho[1:, 1:, 1:] + div))))
    assert worst < 5e-13


def test_cowan_normalisation_and_factorisation():
    o = checkers.oracle()
    for dx, dy, dz in [(5e-6, 5e-6, 2e-6), (1.0, 1.0, 1.0), (3e-6, 7e-6, 1e-6)]:
        c = (C.c_double * 12)()
        o("cowan_coefficients", dx, dy, dz, c)
        alpha, beta = c[0:3], c[3:6]
        dxy, dyz, dzx = c[6], c[7], c[8]
        rx, ry, rz = c[9], c[10], c[11]
        norm = [alpha[0] + 2 * beta[1] + 2 * beta[2] + 4 * dyz,
                alpha[1] + 2 * beta[2] + 2 * beta[0] + 4 * dzx,
                alpha[2] + 2 * beta[0] + 2 * beta[1] + 4 * dxy]
        fact = [4 * ((beta[2] + 2 * dzx) / rz + (beta[1] + 2 * dxy) / ry),
                4 * ((beta[0] + 2 * dxy) / rx + (beta[2] + 2 * dyz) / rz),
                4 * ((beta[1] + 2 * dyz) / ry + (beta[0] + 2 * dzx) / rx),
                16 * (dyz / (ry * rz) + dzx / (rz * rx) + dxy / (rx * ry))]
        for v in norm + fact:
            assert abs(v - 1.0) <= 1e-12


def test_cowan_rejects_dz_not_smallest():
    o = checkers.oracle()
    c = (C.c_double * 12)()
    assert o.fn["cowan_coefficients"](1e-6, 5e-6, 2e-6, c) == 1


def test_lapenta_markidis_energy_theorem():
    lib = checkers.oracle().lib
    rng = np.random.default_rng(11)
    d = lambda v: (C.c_double * 3)(*v)
    q, m = -1.602176634e-19 * 1e3, 9.1093837139e-31 * 1e3
    for _ in range(300):
        u0 = rng.normal(0.0, 30.0, 3)
        e = rng.normal(0.0, 1e10, 3)
        b = rng.normal(0.0, 3.0, 3)
        h = 1e-14
        u = d(u0)
        assert lib.oracle_momentum(u, d(e), d(b), q, m, h, 0.0) > 0
        u1 = np.array(list(u))
        g0 = lib.oracle_gamma(d(u0))
        g1 = lib.oracle_gamma(d(u1))
        dx = h * C_LIGHT * (u0 + u1) / (g0 + g1)
        work = q * np.dot(e, dx)
        lhs = m * C_LIGHT ** 2 * (g1 - g0)
        assert abs(lhs - work) <= 1e-9 * max(abs(work), m * C_LIGHT ** 2 * 1e-6)
        # pure magnetic rotation conserves gamma
        u = d(u0)
        assert lib.oracle_momentum(u, d([0.0, 0.0, 0.0]), d(b), q, m, h, 0.0) > 0
        assert abs(lib.oracle_gamma(u) - g0) <= 4e-15 * g0
