"""aprl_run_sample_field_plane_noalloc against aprl_run_sample_field_plane.

The no-allocation variant serves callers that may not allocate device memory
while a run is stepping (a framework's caching allocator already holds the
free memory, or the loop must not take cudaFree's device-wide
synchronisation).  It stages the plane in a fixed array built into the
library instead of a buffer the run allocates, so it must return the same
values as the allocating call, on consecutive calls that reuse the array,
and refuse planes larger than the array.

This file is named to be collected last: a run that stops at the first
failure has already run every other test.  Its first call on the device
performs the one-time address look-up, so it passes alone in a fresh process
as well as after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import checkers
from aprl_b200 import abi, native, workloads

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def sample(binding, run, name, lab_z):
    cfg = run.config
    out = np.full(6 * cfg.nx * cfg.ny, np.nan)
    inside = C.c_int(-1)
    binding(name, run.handle, lab_z, out.ctypes.data_as(C.POINTER(C.c_double)),
            out.size, C.byref(inside))
    return out, inside.value


def test_noalloc_plane_matches_allocating_call_twice_in_a_row():
    w = workloads.small_case(steps=3)
    b = native.load()
    run = native.Run(b, w.config).load_workload(w)
    run.step(2)
    cfg = w.config
    planes = [cfg.boost_gamma * (f * cfg.nz * cfg.dz) for f in (0.3, 0.6)]
    expected = [sample(b, run, "run_sample_field_plane", z) for z in planes]
    # Two calls in a row through the fixed array, each against the
    # allocating call at the same plane.
    got = [sample(b, run, "run_sample_field_plane_noalloc", z) for z in planes]
    for (e, e_inside), (g, g_inside) in zip(expected, got):
        assert e_inside == g_inside == 1
        assert np.all(np.isfinite(g))
        assert checkers.max_relative(g, e) <= RTOL
    # The two planes differ, so the second call did not read the first's data.
    assert checkers.max_relative(expected[0][0], expected[1][0]) > 0.0
    # A plane beyond the window: same *inside answer, output untouched.
    far = cfg.boost_gamma * (10.0 * cfg.nz * cfg.dz)
    assert sample(b, run, "run_sample_field_plane", far)[1] == 0
    out, inside = sample(b, run, "run_sample_field_plane_noalloc", far)
    assert inside == 0 and np.all(np.isnan(out))


def test_noalloc_plane_rejects_planes_beyond_its_array():
    cells = 288  # 6 * 288 * 288 values > APRL_NOALLOC_PLANE_MAX_VALUES
    assert 6 * cells * cells > 393216
    cfg = workloads.make_config(cells, cells, 4, 5e-6, 5e-6, 2e-6, 2, 10.0,
                                "linear-binomial3", 1)
    b = native.load()
    run = native.Run(b, cfg)
    with pytest.raises(native.AprlError) as err:
        sample(b, run, "run_sample_field_plane_noalloc", 0.0)
    assert err.value.status == abi.APRL_ERR_OUT_OF_RANGE
    assert "393216" in str(err.value)
