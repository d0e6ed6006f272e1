"""The parameter-scan server (aprl_scan_*): continuous batching of
independent runs on one GPU.

Each result must be the result of the same request run alone, within the
stated tolerance: runs share nothing but the GPU, so only the summation order
of the J atomics differs (FP64: 1e-12 relative; FP32-mixed: 1e-6 relative
detector-plane L2).  Admission follows the device budget (a budget that
holds one run at a time serialises the runs in FIFO order) and requests that
arrive while others run overlap with them.
"""
import numpy as np
import pytest

import checkers
from aprl_b200 import abi, native, workloads

STEPS = 6


def draws(count, precision, seed=7):
    return [workloads.scan_draw(i, seed=seed, steps=STEPS, precision=precision,
                                cells_min=(32, 32, 32), cells_max=(48, 48, 64),
                                particles_range=(200, 2000))
            for i in range(count)]


def plain_detector(w):
    """The same request through the plain run API on the default stream."""
    run = native.Run(native.load(), w.config)
    run.allocate_reference()
    run.set_particles(w.particles)
    run.step(STEPS)
    return run.sample_field_plane(workloads.detector_plane_lab_z(w.config)), run.stats()


def submit_all(scan, ws):
    return [scan.submit(w.config, w.particles, STEPS,
                        detector_lab_z=workloads.detector_plane_lab_z(w.config)) for w in ws]


def rel_l2(a, b):
    a, b = np.asarray(a).ravel(), np.asarray(b).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_footprint_grows_with_grid_particles_and_precision():
    b = native.load()
    small = workloads.make_config(32, 32, 32, 5e-6, 5e-6, 2e-6, 8, 10.0,
                                  "linear-binomial3", 10)
    big = workloads.make_config(64, 64, 128, 5e-6, 5e-6, 2e-6, 8, 10.0,
                                "linear-binomial3", 10)
    f = {}
    for name, cfg in (("small", small), ("big", big)):
        for n in (1000, 100000):
            out = __import__("ctypes").c_uint64()
            b("scan_footprint", __import__("ctypes").byref(cfg), n,
              __import__("ctypes").byref(out))
            f[name, n] = out.value
    assert f["small", 1000] < f["small", 100000] < f["big", 100000]
    assert f["big", 1000] > f["small", 1000]
    mixed = workloads.with_precision(big, "fp32-mixed")
    out = __import__("ctypes").c_uint64()
    b("scan_footprint", __import__("ctypes").byref(mixed), 1000,
      __import__("ctypes").byref(out))
    assert out.value < f["big", 1000]


@pytest.mark.gpu
@pytest.mark.parametrize("group", [1, 4])
@pytest.mark.parametrize("precision,bound", [("fp64", 1e-12), ("fp32-mixed", 1e-6)])
def test_each_result_is_the_same_alone_and_in_the_mix(precision, bound, group):
    """group: runs each worker steps in lock step (aprl_runs_step)."""
    ws = draws(6, precision)
    alone = [plain_detector(w) for w in ws]
    scan = native.Scan(native.load(), slots=4 if group == 1 else 2, runs_per_slot=group)
    tickets = submit_all(scan, ws)
    results = [scan.wait(t) for t in tickets]
    scan.close()
    for w, (det, st), r in zip(ws, alone, results):
        assert r["state"] == abi.SCAN_DONE and r["status"] == abi.APRL_OK, r["message"]
        assert rel_l2(r["detector"], det) <= bound
        assert r["stats"]["step"] == STEPS
        assert r["stats"]["particles"] == st["particles"]
        assert r["stats"]["exits"] == st["exits"]
    # Requests submitted together ran at the same time on different slots.
    spans = sorted((r["start_s"], r["finish_s"]) for r in results)
    assert any(b0 < a1 for (a0, a1), (b0, b1) in zip(spans, spans[1:]))
    if group == 1:
        assert len({r["slot"] for r in results}) > 1


@pytest.mark.gpu
def test_lock_step_gives_each_run_its_own_bits():
    """aprl_runs_step: three different runs (bit-reproducible current sum)
    stepped in lock step end with the bits each gets stepped alone."""
    import ctypes
    ws = draws(3, "fp64", seed=5)
    for w in ws:
        w.config = workloads.with_determinism(w.config)
    def start(w):
        run = native.Run(native.load(), w.config)
        run.allocate_reference()
        run.set_particles(w.particles)
        return run
    alone = []
    for w in ws:
        r = start(w)
        r.step(STEPS)
        alone.append(checkers.state(r))
    runs = [start(w) for w in ws]
    handles = (ctypes.c_void_p * len(runs))(*[r.handle for r in runs])
    statuses = (ctypes.c_int * len(runs))()
    native.load()("runs_step", handles, len(runs), STEPS, statuses)
    assert list(statuses) == [0] * len(runs)
    for r, a in zip(runs, alone):
        b = checkers.state(r)
        for x, y in zip(a["fields"] + a["histories"], b["fields"] + b["histories"]):
            np.testing.assert_array_equal(x, y)
        for k in a["particles"]:
            np.testing.assert_array_equal(a["particles"][k], b["particles"][k])
        assert a["stats"] == b["stats"]


@pytest.mark.gpu
def test_budget_admits_one_run_at_a_time_in_fifo_order():
    ws = draws(3, "fp64", seed=11)
    scan0 = native.Scan(native.load(), slots=1)
    biggest = max(scan0.footprint(w.config, w.particles["x"].size) for w in ws)
    scan0.close()
    scan = native.Scan(native.load(), budget_bytes=biggest + 1, slots=3)
    tickets = submit_all(scan, ws)
    results = [scan.wait(t) for t in tickets]
    scan.close()
    for r in results:
        assert r["status"] == abi.APRL_OK, r["message"]
    for prev, nxt in zip(results, results[1:]):
        assert nxt["start_s"] >= prev["finish_s"]      # never two at once
    assert [r["start_s"] for r in results] == sorted(r["start_s"] for r in results)


@pytest.mark.gpu
def test_failed_request_reports_and_others_finish():
    ws = draws(3, "fp64", seed=13)
    bad = abi.RunConfig.from_buffer_copy(bytes(ws[1].config))
    bad.substeps = 0
    scan = native.Scan(native.load(), slots=2)
    tickets = [scan.submit(ws[0].config, ws[0].particles, STEPS),
               scan.submit(bad, ws[1].particles, STEPS),
               scan.submit(ws[2].config, ws[2].particles, STEPS)]
    results = [scan.wait(t) for t in tickets]
    scan.close()
    assert results[0]["status"] == abi.APRL_OK and results[2]["status"] == abi.APRL_OK
    assert results[1]["status"] == abi.APRL_ERR_INVALID_ARGUMENT
    assert "substep" in results[1]["message"].lower()


@pytest.mark.gpu
def test_request_larger_than_budget_is_refused():
    w = draws(1, "fp64")[0]
    scan = native.Scan(native.load(), budget_bytes=1 << 20, slots=1)
    with pytest.raises(native.AprlError) as err:
        scan.submit(w.config, w.particles, STEPS)
    scan.close()
    assert err.value.status == abi.APRL_ERR_OUT_OF_RANGE


@pytest.mark.gpu
def test_runs_growing_their_lists_beside_each_other_stay_intact():
    """Sixteen requests, four at a time, three times over, whose carrier
    lists outgrow their first reservation mid-run (up to ~12k carriers)
    while other runs are created and destroyed beside them.  A run's memory
    comes from a pool shared by all runs, and a list that grows is copied
    and its old storage freed in the run's stream order; a copy issued
    outside that order (on the legacy default stream) once let another run
    take the old storage while it was still being read, which corrupted
    particles and carriers ("Active particle fell behind moving inlet",
    "Invalid CPML carrier current weight").  Every request must finish, and
    every repetition must give the same detector plane."""
    steps = 40
    ws = [workloads.scan_draw(i, seed=11, steps=steps, precision="fp32-mixed",
                              cells_min=(40, 40, 48), cells_max=(72, 72, 128),
                              particles_range=(2.0e4, 1.5e5)) for i in range(16)]
    planes = []
    for _ in range(3):
        scan = native.Scan(native.load(), slots=4)
        tickets = [scan.submit(w.config, w.particles, steps,
                               detector_lab_z=workloads.detector_plane_lab_z(w.config))
                   for w in ws]
        results = [scan.wait(t) for t in tickets]
        scan.close()
        for r in results:
            assert r["status"] == abi.APRL_OK, r["message"]
        planes.append([r["detector"] for r in results])
    assert max(r["stats"]["carriers"] for r in results) > 4096   # the lists did grow
    for later in planes[1:]:
        for a, b in zip(later, planes[0]):
            if b is not None:
                assert rel_l2(a, b) <= 1e-6
