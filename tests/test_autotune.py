"""The autotuner of the grid kernels' launch shapes (aprl_run_tuning).

For a grid extent the process has not seen, the first steps time every
candidate shape of the Cowan magnetic, preview, orbit-sum and commit
kernels twice (real launches of those steps) and then keep the fastest.
Every candidate computes each node the same way, so the choice changes no
bit of a result: a bit-reproducible run stepped while the candidates are
being measured ends with the bits of a run of the same request stepped
after the choice was made."""
import numpy as np
import pytest

import checkers
from aprl_b200 import native, workloads

pytestmark = pytest.mark.gpu


def case():
    # An extent no other test uses, so that its tuning starts here.
    w = workloads.small_case(nx=20, ny=18, nz=44, particles=500, steps=12)
    w.config = workloads.with_determinism(w.config)
    return w


def test_choices_are_made_and_change_no_bit():
    w = case()
    first = native.Run(native.load(), w.config).load_workload(w)
    assert first.tuning()["decided"] == [False] * 4
    first.step(12)
    t = first.tuning()
    assert t["decided"] == [True] * 4, t
    assert t["cowan_planes_per_block"] in (2, 4, 8, 16)
    for k in range(4):
        assert all(ms > 0.0 for ms in t["candidate_ms"][k])
    second = native.Run(native.load(), w.config).load_workload(w)
    second.step(12)
    a, b = checkers.state(first), checkers.state(second)
    for x, y in zip(a["fields"] + a["histories"], b["fields"] + b["histories"]):
        np.testing.assert_array_equal(x, y)
    for k in a["particles"]:
        np.testing.assert_array_equal(a["particles"][k], b["particles"][k])
    assert a["stats"] == b["stats"]
