"""The bounds-checked build (libaprl_b200_checked.so, -DAPRL_GPU_BOUNDS_CHECK).

In that build every field, current, orbit-sum, CPML-history and inlet-plane
index of the step's kernels is tested against its array before the access;
an index outside raises the run's device error ("Array index outside its
array"), and the access is redirected to element 0, so the check itself
never touches memory outside an array and never traps.  The counterpart of
the reference's DIRECT_EB_BOUNDS_CHECK build (CMakeLists.txt:49-50,
src/eb_field.h:134-141).

The tests run whole coupled steps on grids of at most 16 cells per axis
(plus a longer one for the moving window's ring wrap), both shapes, with
carriers, exits and held injection: no index leaves its array, and the
results are the product library's (the oracle's to 1e-12).
"""
import pytest

import checkers
from aprl_b200 import native, workloads
from test_c1_parity import compare
from test_gpu_parity import compare_state

CASES = {
    "binomial3": dict(nx=16, ny=16, nz=16, particles=300, steps=4),
    "quintic": dict(nx=16, ny=16, nz=16, particles=300, steps=4, shape="quintic-compensated"),
    "carriers": dict(nx=16, ny=16, nz=16, particles=600, steps=6, z_fraction=(0.02, 0.99),
                     margin_cells=1),
    "ring_wrap": dict(nx=12, ny=12, nz=20, particles=200, steps=24),
}


def test_checked_library_exports_the_abi():
    from test_abi import declared_functions
    lib = native.load_checked().lib
    missing = [n for n in declared_functions() if getattr(lib, n, None) is None]
    assert not missing, missing


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_steps_stay_inside_every_array(case):
    w = workloads.small_case(cpml=3, **CASES[case])
    g = native.Run(native.load_checked(), w.config).load_workload(w)
    o = checkers.run(checkers.oracle(), w)
    for _ in range(w.steps):
        g.step(1)     # raises on a device error, a bounds violation included
        o.step(1)
    # Over two dozen steps the nearly vanishing Bz of these bunches is held
    # against |B|, as in the full-size parity test.
    compare(g, o, case)
    assert g.stats()["device_error"] == 0


@pytest.mark.gpu
def test_held_injection_stays_inside_every_array():
    w = workloads.streaming_case(nx=16, ny=16, nz=16, particles=300, steps=8, cpml=3,
                                 upstream_cells=10)
    w.config.inlet_charge_match = 1
    g = native.Run(native.load_checked(), w.config).load_workload(w)
    o = checkers.run(checkers.oracle(), w)
    for _ in range(w.steps):
        g.step(1)
        o.step(1)
    compare_state(g, o)
