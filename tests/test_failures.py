"""Failures injected from the host, and the errors they raise.

Every failure here is made by the caller's data -- a fixed point that is
never allowed to converge, an active particle placed inside the CPML, a
non-finite field value, a carrier with a non-finite or superluminal velocity
-- never by a fault on the device: the kernels record the first error code
in a status word that the host reads after the trial, and the entry point
returns the reference's exception type (as a status) and message.  After
such an error the device stays usable (the next run steps normally).

The oracle and the reference's own translation units raise the same
status and message for each case (the CPU tests); the GPU raises what the
oracle raises (the GPU tests).

Reference anchors: the fixed point's failure message
(src/simulation_source_coupling.cpp:54), ParticleCPMLRegion::firstEntry's
non-finite and start-in-CPML checks (src/particle_boundary.cpp:115-122), the
64-cut crossing budget (src/longitudinal_shape.h:102) and the
Lapenta-Markidis root check (src/source_coupling_math.h:272-293).
"""
import re

import numpy as np
import pytest

import checkers
from aprl_b200 import abi, native, workloads


def no_convergence():
    w = workloads.small_case(steps=3)
    w.config.force_tolerance = 0.0   # force < 0 never holds: all 64 trials run
    return w, lambda r: None


def particle_in_cpml():
    w = workloads.small_case(steps=3)

    def mutate(r):
        p = r.get_particles()
        p["x"][0] = w.config.reference_origin[0] + 1.5 * w.config.dx   # inside the 4-cell CPML
        r.set_particles(p)
    return w, mutate


def nan_field():
    w = workloads.small_case(steps=3)

    def mutate(r):
        f = r.get_field(0)
        f[5, 8, 8] = np.nan
        r.set_field(0, f)
    return w, mutate


def carrier(w, position_cells, velocity_cells):
    cfg = w.config
    pos = np.array([[cfg.reference_origin[0] + position_cells[0] * cfg.dx,
                     cfg.reference_origin[1] + position_cells[1] * cfg.dy,
                     position_cells[2] * cfg.dz]])
    vel = np.array([[velocity_cells[0] * cfg.dx / cfg.dt, velocity_cells[1] * cfg.dy / cfg.dt,
                     velocity_cells[2] * cfg.dz / cfg.dt]])
    return {"position": pos, "velocity": vel, "charge": np.array([-1e-15]),
            "weight": np.array([0.5])}


def nan_carrier():
    w = workloads.small_case(steps=3)
    return w, lambda r: r.set_carriers(carrier(w, (1.5, 8.5, 20), (np.nan, 0.0, 0.0)))


def crossing_budget():
    # 40 cells in x and 40 in y within one step: 80 cell-plane cuts
    w = workloads.small_case(nx=64, ny=64, nz=40, particles=100, steps=3)
    return w, lambda r: r.set_carriers(carrier(w, (2.5, 2.5, 20), (40.0, 40.0, 0.0)))


CASES = {
    "no_convergence": (no_convergence, abi.APRL_ERR_NOT_CONVERGED,
                       "Conservative source coupling failed at step 1"),
    "particle_in_cpml": (particle_in_cpml, abi.APRL_ERR_OUT_OF_RANGE,
                         "Active particle starts inside the non-physical CPML region"),
    "nan_field": (nan_field, abi.APRL_ERR_RUNTIME, "Nonphysical local mean-gamma root"),
    "nan_carrier": (nan_carrier, abi.APRL_ERR_RUNTIME,
                    "Particle trajectory contains a non-finite coordinate"),
    "crossing_budget": (crossing_budget, abi.APRL_ERR_RUNTIME,
                        "Quintic orbit exceeds crossing budget"),
}


def failure(binding, case):
    make, _, _ = CASES[case]
    w, mutate = make()
    r = checkers.run(binding, w)
    mutate(r)
    with pytest.raises(native.AprlError) as info:
        r.step(1)
    return info.value


HISTORY = re.compile(r"^Conservative source coupling failed at step (\d+): force=(\S+) "
                     r"work=(\S+) iterations=(\d+) history\(force/work\)=((?: \S+/\S+)*)$")


@pytest.mark.parametrize("case", sorted(CASES))
def test_oracle_raises_the_reference_error(case):
    err = failure(checkers.oracle(), case)
    _, status, message = CASES[case]
    assert err.status == status
    assert str(err.message).startswith(message)
    if case == "no_convergence":
        m = HISTORY.match(err.message)
        assert m and int(m.group(4)) == 64 and len(m.group(5).split()) == 64


@pytest.mark.skipif(not checkers.reference_available(),
                    reason="reference translation units not built")
@pytest.mark.parametrize("case", sorted(CASES))
def test_reference_raises_the_same_error(case):
    err = failure(checkers.reference(), case)
    _, status, message = CASES[case]
    assert err.status == status
    assert str(err.message).startswith(message.split(" at step")[0])


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_gpu_raises_what_the_oracle_raises(case):
    got = failure(native.load(), case)
    want = failure(checkers.oracle(), case)
    assert got.status == want.status
    if case == "no_convergence":
        mg, mw = HISTORY.match(got.message), HISTORY.match(want.message)
        assert mg and mw and mg.group(4) == mw.group(4) == "64"
        hg, hw = mg.group(5).split(), mw.group(5).split()
        assert len(hg) == len(hw) == 64
        # the first two trials' force and work (well above roundoff) agree
        for a, b in zip(hg[:2], hw[:2]):
            for x, y in zip(a.split("/"), b.split("/")):
                assert abs(float(x) - float(y)) <= 1e-5 * abs(float(y))
    else:
        # the library adds the index of the first failing element
        assert got.message.startswith(want.message)


@pytest.mark.gpu
def test_device_stays_usable_after_errors():
    for case in sorted(CASES):
        failure(native.load(), case)
    w = workloads.small_case(steps=3)
    g = native.Run(native.load(), w.config).load_workload(w)
    o = checkers.run(checkers.oracle(), w)
    g.step(2)
    o.step(2)
    from test_gpu_parity import compare_state
    compare_state(g, o)
