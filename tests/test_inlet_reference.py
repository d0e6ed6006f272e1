"""Non-finite inlet reference values.

The reference throws "Non-finite moving-window inlet" when an inlet query
returns a non-finite value (src/moving_window_fields.cpp:204).  The oracle
checks at the query too.  The GPU path cannot raise from a kernel, so it
checks every value when the host hands the table over (aprl_run_set_reference
and aprl_run_set_reference_planes) and refuses the upload with the same
message, before any byte reaches the device.  A refused upload leaves the
device table as it was.
"""
import numpy as np
import pytest

import checkers
from aprl_b200 import native, workloads

MESSAGE = "Non-finite moving-window inlet"
BAD = [np.nan, -np.nan, np.inf, -np.inf]


def poisoned(table, position, value):
    out = np.array(table, copy=True)
    out.reshape(-1)[position] = value
    return out


def test_oracle_rejects_a_non_finite_inlet_at_the_query():
    w = workloads.small_case(steps=2)
    reference = [np.full_like(t, np.nan) for t in w.reference]
    run = native.Run(checkers.oracle(), w.config)
    run.set_reference(reference)
    run.set_particles(w.particles)
    with pytest.raises(native.AprlError, match=MESSAGE):
        run.step(1)
    run.close()


@pytest.mark.gpu
@pytest.mark.parametrize("value", BAD)
def test_gpu_refuses_a_non_finite_table(value):
    w = workloads.small_case(nx=32, ny=32, steps=2)
    assert w.reference[2].size > 4097  # crosses a 4096-value check chunk
    run = native.Run(native.load(), w.config)
    for position in (0, 4095, 4096, w.reference[2].size - 1):
        tables = list(w.reference)
        tables[2] = poisoned(tables[2], position, value)
        with pytest.raises(native.AprlError, match=MESSAGE):
            run.set_reference(tables)
    run.close()


@pytest.mark.gpu
def test_gpu_refused_planes_leave_the_table_unchanged():
    w = workloads.small_case(steps=4)
    good = checkers.run(native.load(), w)
    refused = checkers.run(native.load(), w)
    for a in range(6):
        planes = poisoned(w.reference[a][:3], w.reference[a][:3].size - 1, np.inf)
        with pytest.raises(native.AprlError, match=MESSAGE):
            refused.set_reference_planes(a, 0, planes)
        # finite planes of the same table are accepted
        refused.set_reference_planes(a, 0, w.reference[a][:3])
    good.step(w.steps)
    refused.step(w.steps)
    for a in range(6):
        assert checkers.max_relative(refused.get_field(a), good.get_field(a)) <= 1e-12
    good.close()
    refused.close()
