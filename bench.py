"""Benchmark of the B200 PIC step on the dipole-radiation workload.

`python bench.py --gpus N --steps K --warmup W` runs one independent run per
GPU (replicas: a moving-window run does not shard without z-slab halos), W
untimed steps, then K timed steps bracketed by a barrier and a device
synchronise, timed with CUDA events on the run's stream; rank 0 prints one
JSON line.  `--impl reference` times the reference's own CPU translation
units (oracle/_ref, built from the APRL sources) on the host cores instead.

Workload: 128x128x512 cells (dx = dy = 5 um, dz = 2 um, c dt = dz), 10-cell
transverse CPML, linear-binomial3, a uniform 1 T lab dipole seen in a
gamma = 10 boosted frame, and a seeded 1 GeV, 100 pC Gaussian bunch of 1M
macro-particles (sigma_xy = 50 um, sigma_z = 20 um lab, 1 um emittance,
1e-4 energy spread) truncated to the window's trusted region.  Fields start
at zero; the inlet reference is a smooth seeded analytic table.
"""
import argparse
import contextlib
import csv
import io
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

from aprl_b200 import abi, native, workloads  # noqa: E402

METRIC = "particle-steps/s"


def parse_args(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["dipole", "drift", "undulator"], default="dipole",
                   help="dipole: 128x128x512, 1M particles (the headline); drift: "
                        "64x64x256, 100k; undulator: 128x128x2048, 4M, FP32-mixed")
    p.add_argument("--particles", type=int, default=None)
    p.add_argument("--shape", default="linear-binomial3")
    p.add_argument("--precision", choices=["fp64", "fp32-mixed"], default=None)
    p.add_argument("--deterministic", action="store_true",
                   help="sum the current in the bit-reproducible fixed-point mode")
    p.add_argument("--no-fp32-arm", action="store_true",
                   help="skip the FP32-mixed comparison pass of an FP64 run")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-other-configs", action="store_true",
                   help="skip the drift, quintic and bit-reproducible step rates")
    p.add_argument("--no-scan", action="store_true",
                   help="skip the batched-ensemble and served-scan measurements")
    p.add_argument("--ensemble-runs", type=int, default=64)
    p.add_argument("--ensemble-steps", type=int, default=100)
    p.add_argument("--scan-requests", type=int, default=64, help="requests per arrival rate")
    p.add_argument("--scan-steps", type=int, default=500)
    p.add_argument("--scan-rates", default="5,10,20,50",
                   help="Poisson arrival rates (requests per second), comma-separated")
    p.add_argument("--scan-slots", type=int, default=4, help="scan worker threads")
    p.add_argument("--scan-group", type=int, default=8,
                   help="runs each worker steps in lock step")
    p.add_argument("--cpu-sample-seconds", type=float, default=20.0)
    p.add_argument("--initial-self-field", choices=["auto", "on", "off"], default="auto",
                   help="start from the Cowan initial self-field (auto: on for the undulator "
                        "workload; the dipole and drift bunches, beta_z ~ 1 in the box, are "
                        "rejected by the reference's own initializer)")
    p.add_argument("--no-self-field", action="store_true",
                   help="skip the timing of the initial self-field solve")
    p.add_argument("--energy-ledger", choices=["auto", "on", "off"], default="auto",
                   help="keep the moving-window energy ledger during the timed steps "
                        "(auto: on for the undulator workload)")
    args = p.parse_args(argv)
    if args.initial_self_field == "auto":
        args.initial_self_field = args.workload == "undulator"
    else:
        args.initial_self_field = args.initial_self_field == "on"
    if args.energy_ledger == "auto":
        args.energy_ledger = args.workload == "undulator"
    else:
        args.energy_ledger = args.energy_ledger == "on"
    defaults = {"dipole": (1_000_000, "fp64"), "drift": (100_000, "fp64"),
                "undulator": (4_000_000, "fp32-mixed")}[args.workload]
    if args.particles is None:
        args.particles = defaults[0]
    if args.precision is None:
        args.precision = defaults[1]
    if args.workload != "dipole":
        # the scan objects and the CPU slice belong to the dipole headline
        args.no_scan = True
        args.no_cpu_baseline = True
    return args


WORKLOADS = {
    "dipole": (lambda steps, args, seed: workloads.dipole_c2(
        steps=steps, particles=args.particles, shape=args.shape, seed=seed,
        precision=args.precision), "uniform 1 T lab dipole"),
    "drift": (lambda steps, args, seed: workloads.drift_c1(
        steps=steps, particles=args.particles, shape=args.shape, seed=seed,
        precision=args.precision), "none (free drift)"),
    "undulator": (lambda steps, args, seed: workloads.undulator_c3(
        steps=steps, particles=args.particles, shape=args.shape, seed=seed,
        precision=args.precision), "planar undulator, period 3 cm, K = 1"),
}


def over_ranks(times, counts, world, device="cuda"):
    """The job's figures from every rank's: the maximum of `times` (a run
    ends when its slowest replica does) and the sums of `counts` (the units
    all replicas processed).  One rank: the inputs unchanged.  The same
    collective steps on every rank, in the same order."""
    import torch
    import torch.distributed as dist
    vals = torch.tensor([float(t) for t in times] + [float(c) for c in counts],
                        dtype=torch.float64, device=device)
    if world <= 1:
        return [float(t) for t in times], [int(c) for c in counts]
    mx = vals.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    sm = vals.clone()
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    n = len(times)
    return ([mx[i].item() for i in range(n)],
            [int(round(sm[n + i].item())) for i in range(len(counts))])


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
@contextlib.contextmanager
def clock_sampler(index):
    """nvidia-smi clocks and throttle reasons during the timed region."""
    fields = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    proc = None
    try:
        proc = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={fields}",
                                 "--format=csv,noheader,nounits", "-lms", "200"],
                                stdout=out, stderr=subprocess.DEVNULL)
    except OSError:
        proc = None
    result = {}
    try:
        yield result
    finally:
        if proc is not None:
            proc.terminate()
            try:
                proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                proc.kill()
        out.flush()
        out.seek(0)
        rows = [r for r in csv.reader(io.StringIO(out.read())) if len(r) >= 9]
        out.close()
        os.unlink(out.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for name, value in zip(names, r[5:9]):
                if value.strip().lower() == "active":
                    reasons.add(name)
        result.update({"sm_mhz": statistics.median(sm) if sm else None,
                       "sm_max_mhz": max(mx) if mx else None,
                       "reasons": sorted(reasons), "samples": len(sm)})


def algorithmic_bytes(kernel, cfg, particles, carriers):
    """Unique-state bytes one launch must move (FP64).  Gather/deposit
    stencil traffic is not counted: it is cache traffic for cell-local
    particles."""
    n_cells = cfg.nx * cfg.ny * cfg.nz
    if kernel == "cowan_magnetic":      # read 3 E, read+write 3 B
        return 9 * 8 * n_cells
    if kernel == "electric_preview":    # read 3 E^n and 3 B, write 3 E* and, with particles
        return (12 if particles else 9) * 8 * n_cells   # in the window, the orbit sum E* + E^n
    if kernel == "electric_commit":     # read J; E* += -dt/eps0 J only where J != 0
        return 3 * 8 * n_cells          # (that part depends on the bunch; not counted)
    if kernel == "push_deposit":        # read x,u,q,m,nextE/B; write x1,u1,usedE/B,work,flags,
        return particles * (64 + 48 + 48 + 48 + 8 + 2 + 49)   # and the chord (b, e, mode)
    if kernel == "chord_deposit":       # read the chord (b, e), q, mode; J updates are L2 reductions
        return particles * (48 + 8 + 1)
    if kernel == "residual":            # read x0,x1,q,m,usedE/B,work; write nextE/B
        return particles * (48 + 16 + 48 + 8 + 48)
    if kernel == "guess_gather":        # read x,u,flags; write nextE/B
        return particles * (48 + 1 + 48)
    if kernel == "orbit_sum":           # read E*, J, E^n; write S, per E node
        return 4 * 8 * 3 * n_cells
    if kernel == "carrier":             # read + write 8 words
        return carriers * 128
    return None


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from
# one-kernel ncu captures of the default workload -- dipole, 128x128x512
# cells, 1M particles, linear-binomial3, FP64 -- with a cold L2.  The grid
# passes move the same bytes for any bunch on this grid; the particle
# kernels' traffic is mostly the fields over the bunch's region, which does
# not grow with the particle count, so they have a figure only at 1M.
GRID_TRAFFIC = {"cowan_magnetic": 669_778_944, "orbit_sum": 791_749_632,
                "electric_preview": 845_800_448, "electric_commit": 280_096_512}
PARTICLE_TRAFFIC = {"chord_deposit": 118_682_624, "push_deposit": 252_511_232,
                    "residual": 287_908_096, "guess_gather": 191_039_744}
PARTICLE_TRAFFIC_CONFIG = {"workload": "dipole", "shape": "linear-binomial3",
                           "precision": "fp64", "particles": 1_000_000,
                           "deterministic": False}


# L2 reduction sectors per particle of one chord_deposit launch: ncu
# lts__t_sectors_srcunit_tex_op_red on the dipole workload (the unmerged
# one-reduction-per-visit deposit of the same chords took 90.4 at 250k).
RED_SECTORS_PER_PARTICLE = {250_000: 45.5, 1_000_000: 21.3}


PROBE_SOURCE = os.path.join(REPO, "bench_probe.cu")
PROBE_OUTPUT = os.path.join(REPO, "bench_probe.so")


def build_probe(force=False, verbose=True):
    """The benchmark's measurement probe (bench_probe.so, sm_100a)."""
    if (not force and os.path.exists(PROBE_OUTPUT) and
            os.path.getmtime(PROBE_SOURCE) <= os.path.getmtime(PROBE_OUTPUT)):
        return PROBE_OUTPUT
    from aprl_b200 import build as product_build
    cmd = [product_build.nvcc(), "-shared", "-o", PROBE_OUTPUT, PROBE_SOURCE, "-std=c++17",
           "-O3", "-Xcompiler", "-fPIC"] + product_build.ARCH
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return PROBE_OUTPUT


def atomic_peak(integer=False):
    """Measured L2 reduction rate of this GPU (bench_probe.cu): every lane
    adds to its own 32-byte sector of a 16 MB window, neighbouring lanes on
    neighbouring sectors, as the cell-sorted deposit's reductions land; best
    of 5 launches, in G reductions/s.  Binary64 adds (the default deposit),
    or 64-bit integer adds (the deterministic deposit)."""
    import ctypes
    lib = ctypes.CDLL(build_probe(verbose=False))
    rate = ctypes.c_double()
    probe = lib.aprl_probe_integer_reduction_rate if integer else lib.aprl_probe_reduction_rate
    if probe(16, 5, ctypes.byref(rate)) != 0:
        return None
    return rate.value / 1e9


def measured_traffic(kernel, args):
    """Measured DRAM bytes of one launch of `kernel` on this run's
    configuration, or None where none was measured."""
    if args.workload != "dipole":
        return None
    if kernel in GRID_TRAFFIC:
        return GRID_TRAFFIC[kernel]
    if kernel in PARTICLE_TRAFFIC and all(
            getattr(args, key) == value for key, value in PARTICLE_TRAFFIC_CONFIG.items()):
        return PARTICLE_TRAFFIC[kernel]
    return None


# ---------------------------------------------------------------------------
def reference_planes_for_step(cfg, step):
    """Native reference z planes the inlet queries of one step touch:
    begin (offset-1, step), preview (offset, step+1), shift (offset-1, step+1)."""
    offset = cfg.initial_offset - step
    zs = [offset - 1 - cfg.translation_beta * step,
          offset - cfg.translation_beta * (step + 1),
          offset - 1 - cfg.translation_beta * (step + 1)]
    lo = max(0, int(math.floor(min(zs))))
    hi = int(math.floor(max(zs))) + 1
    return lo, hi


def run_ours(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    K, W = args.steps, args.warmup
    total_steps = W + 2 * K + 4
    make, magnet = WORKLOADS[args.workload]
    w = make(total_steps, args, 17 + rank)
    if args.deterministic:
        w.config = workloads.with_determinism(w.config)
    cfg = w.config
    lib = native.load()

    def start_run():
        """A run of the workload after its W warm-up steps."""
        run = native.Run(lib, cfg, stream=stream.cuda_stream)
        run.set_reference(w.reference)
        run.set_particles(w.particles)
        initial_fields = "zero"
        if args.initial_self_field:
            report = run.initialize_self_field(abi.self_field_config(
                cfg, hold_transverse_until_activation=True))
            initial_fields = (f"cowan-relativistic-poisson self-field ({report['iterations']} "
                              f"CG iterations, beta_z {report['mean_beta_z']:.3f})")
        if args.energy_ledger:
            run.enable_energy_ledger()
        for _ in range(W):
            run.step(1)
        run.synchronize()
        run.b("run_reset_iteration_stats", run.handle)
        return run, initial_fields

    # Autotuning of the grid kernels' launch shapes, untimed: a run of the
    # same grid steps until the process-wide choices for this grid extent are
    # made (each candidate timed twice on real steps); every later run of the
    # extent, the timed ones included, launches with the choices.
    tune_run = native.Run(lib, cfg, stream=stream.cuda_stream)
    tune_run.set_reference(w.reference)
    tune_run.set_particles(w.particles)
    tuning_steps = 0
    while tuning_steps < 16 and not all(tune_run.tuning()["decided"]):
        tune_run.step(1)
        tuning_steps += 1
    tuning = tune_run.tuning()
    tuning["steps"] = tuning_steps
    tune_run.close()

    run, initial_fields = start_run()

    # ---- device-resident timed region ------------------------------------
    launches0 = run.launch_count()
    particle_steps = 0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with clock_sampler(local) as clocks:
        start.record(stream)
        for _ in range(K):
            particle_steps += run.particle_count()
            run.step(1)
        stop.record(stream)
        torch.cuda.synchronize()
    elapsed_ms = start.elapsed_time(stop)
    if world > 1:
        dist.barrier()
    launches = run.launch_count() - launches0
    stats = run.stats()

    # ---- per-kernel times: the same K steps replayed from the same start,
    # with a CUDA event pair around every launch on its stream.  The events
    # cost about 0.24 ms of host enqueue per dipole step, so the timed region
    # above runs without them and the kernel table and roofline come from
    # this replay.
    run.close()
    run, _ = start_run()
    run.profile_enable(True)
    torch.cuda.synchronize()
    p_start, p_stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p_start.record(stream)
    for _ in range(K):
        run.step(1)
    p_stop.record(stream)
    torch.cuda.synchronize()
    profiled_ms = p_start.elapsed_time(p_stop)
    profile = run.profile_read()
    run.profile_enable(False)

    # ---- end to end through the C ABI with host buffers -------------------
    # A second run of the same workload, from the same start and warm-up, so
    # that both legs time the same K steps (the cost of a step changes as the
    # run goes on, so steps W+K.. are not a like-for-like comparison).
    run.close()
    run, _ = start_run()
    # The inlet reference table lives in pinned host memory (48 MB on the
    # dipole grid); each step uploads the native planes that step's inlet
    # queries touch.  Step k+1's planes are uploaded between
    # aprl_run_step_begin and aprl_run_step_end of step k, so their host-side
    # finiteness check and their PCIe transfer (on the run's copy stream) run
    # while step k's trials run on the GPU; the planes take effect in stream
    # order behind those trials.  K steps, K uploads, all inside the timed
    # region (the first one before the loop).
    pinned_ref = []
    for table in w.reference:
        host = torch.empty(table.shape, dtype=torch.float64, pin_memory=True).numpy()
        np.copyto(host, table)
        pinned_ref.append(host)

    def upload(step):
        lo, hi = reference_planes_for_step(cfg, step)
        sent = 0
        for a in range(6):
            planes = pinned_ref[a][lo:hi + 1]
            run.set_reference_planes(a, lo, planes)
            sent += planes.nbytes
        return sent

    # The detector plane of step k is queued without a wait into one of two
    # page-locked buffers; step k+1's own trial read-back waits for the
    # stream, so the plane is read on the host while step k+1's tail runs.
    # The last plane is completed by the synchronize before the stop event.
    detectors = [torch.empty((cfg.ny, cfg.nx, 6), dtype=torch.float64,
                             pin_memory=True).numpy() for _ in range(2)]
    detector_lab_z = cfg.boost_gamma * (0.5 * cfg.nz * cfg.dz)
    e2e_particle_steps, h2d, d2h = 0, 0, 0
    planes_read, planes_finite = 0, True
    step0 = run.stats()["step"]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e_start, e_stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    wall0 = time.perf_counter()
    e_start.record(stream)
    h2d += upload(step0)
    inside = [False, False]
    for i in range(K):
        e2e_particle_steps += run.particle_count()
        # Step i runs between begin and end; meanwhile the host checks and
        # queues step i+1's planes and reads step i-2's detector plane (its
        # copy completed before step i-1's trials were read back; its buffer
        # is refilled only by step i's plane, queued after step_end).
        run.step_begin()
        if i + 1 < K:
            h2d += upload(step0 + i + 1)
        if i > 1 and inside[i % 2]:
            planes_finite &= bool(np.isfinite(detectors[i % 2]).all())
            planes_read += 1
        run.step_end()
        inside[i % 2] = run.sample_field_plane_async(detector_lab_z, detectors[i % 2])
        d2h += detectors[0].nbytes + 8 * 24  # plane + stats block
        run.stats()
    run.synchronize()
    for last in (K - 2, K - 1):  # the two planes the loop has not read yet
        if last >= 0 and inside[last % 2]:
            planes_finite &= bool(np.isfinite(detectors[last % 2]).all())
            planes_read += 1
    e_stop.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e_start.elapsed_time(e_stop)
    e2e_wall_ms = (time.perf_counter() - wall0) * 1e3
    ledger = run.energy_ledger() if args.energy_ledger else None
    fp32_arm = None
    if args.precision == "fp64" and not args.no_fp32_arm:
        fp32_arm = time_fp32_arm(args, w, stream, run, detector_lab_z, world)

    # max over ranks, totals over ranks
    (elapsed_ms, e2e_ms), (particle_steps, e2e_particle_steps) = over_ranks(
        [elapsed_ms, e2e_ms], [particle_steps, e2e_particle_steps], world)
    run.close()
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return

    value = particle_steps / (elapsed_ms * 1e-3)
    e2e_value = e2e_particle_steps / (e2e_ms * 1e-3)
    peak, peak_kind = measured_peaks()
    dominant = max(profile.items(), key=lambda kv: kv[1][0]) if profile else None
    roofline = None
    if dominant:
        name, (ms, count) = dominant
        per_launch_ms = ms / max(count, 1)
        mean_particles = particle_steps / max(K, 1)
        algo = algorithmic_bytes(name, cfg, mean_particles, stats["carriers"])
        achieved = algo / (per_launch_ms * 1e-3) / 1e9 if algo else None
        roofline = {"bound": "hbm", "kernel": name,
                    "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": (achieved / peak) if achieved else None,
                    "peak_source": peak_kind,
                    "traffic": measured_traffic(name, args),
                    "traffic_source": "ncu DRAM bytes of a one-kernel capture of this "
                                      "workload at 1M particles, cold L2 "
                                      "(profiles/dram_traffic_dipole_128x128x512_1M.md)",
                    "bytes_per_launch": algo, "ms_per_launch": per_launch_ms,
                    "launches": count,
                    "timing": "CUDA events around every launch on its stream, in a replay "
                              "of the timed steps from the same start"}
    atomic_roofline = None
    if "chord_deposit" in profile and world == 1:
        ms, count = profile["chord_deposit"]
        per_launch_ms = ms / max(count, 1)
        mean_particles = particle_steps / max(K, 1)
        # sectors per particle measured nearest this particle count
        key = min(RED_SECTORS_PER_PARTICLE, key=lambda n: abs(math.log(n / max(mean_particles, 1))))
        per_particle = RED_SECTORS_PER_PARTICLE[key]
        achieved_atomic = per_particle * mean_particles / (per_launch_ms * 1e-3) / 1e9
        peak_atomic = atomic_peak(integer=bool(args.deterministic))
        atomic_roofline = {
            "kernel": "chord_deposit",
            "bound": "l2-int64-atomics" if args.deterministic else "l2-fp64-atomics",
            "achieved": achieved_atomic, "peak": peak_atomic, "unit": "G reductions/s",
            "frac": achieved_atomic / peak_atomic if peak_atomic else None,
            "peak_source": "measured here: one reduction per lane per 32-byte sector, "
                           "neighbouring sectors, 16 MB window (bench_probe.cu)",
            "reductions_per_particle": per_particle,
            "reductions_measured_at_particles": key,
            "note": "whole chord_deposit launch time"}
    total_ms = max(sum(x[0] for x in profile.values()), 1e-12)
    kernels = {}
    for k, v in profile.items():
        entry = {"ms": v[0], "launches": v[1], "share": v[0] / total_ms}
        algo = algorithmic_bytes(k, cfg, particle_steps / max(K, 1), stats["carriers"])
        if algo and v[1]:
            gbs = algo / (v[0] / v[1] * 1e-3) / 1e9
            entry.update({"bytes_per_launch": algo, "achieved_gbs": gbs, "hbm_frac": gbs / peak})
        traffic = measured_traffic(k, args)
        if traffic and v[1]:
            # DRAM bytes one launch moved (ncu) over its mean launch time here
            entry.update({"dram_bytes_per_launch": traffic,
                          "dram_gbs": traffic / (v[0] / v[1] * 1e-3) / 1e9})
        kernels[k] = entry
    line = {
        "metric": METRIC, "value": value, "unit": "particle-steps/s",
        "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": elapsed_ms / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic (seeded Gaussian bunch, analytic inlet reference)",
        "config": {"workload": w.name, "cells": [cfg.nx, cfg.ny, cfg.nz],
                   "particles": args.particles, "shape": args.shape,
                   "precision": "fp64-drop-in" if args.precision == "fp64" else "fp32-mixed",
                   "magnet": magnet,
                   "boost_gamma": cfg.boost_gamma, "parallelism": f"replicas{world}",
                   "energy_ledger": bool(args.energy_ledger),
                   "initial_fields": initial_fields,
                   "l2": "inputs larger than L2 (fields + particles > 126 MB)"},
        "fixed_point_trials": {"mean": stats["total_iterations"] / max(K, 1),
                               "max": stats["max_iterations"]},
        "particles_end": stats["particles"], "carriers_end": stats["carriers"],
        "e2e": {"value": e2e_value, "unit": "particle-steps/s",
                "h2d_bytes_per_step": h2d // max(K, 1),
                "d2h_bytes_per_step": d2h // max(K, 1),
                "wall_ms_per_step": e2e_wall_ms / K,
                "detector_planes_read": planes_read,
                "detector_planes_finite": planes_finite,
                "path": "aprl_run_set_reference_planes (pinned table), aprl_run_step, "
                        "aprl_run_sample_field_plane_async (pinned, double-buffered)"},
        "gpu_launches": launches,
        "autotune": tuning,
        "roofline": roofline,
        "atomic_roofline": atomic_roofline,
        "kernels": kernels,
        "kernel_timing": {"how": "CUDA events around every launch on its stream, in a replay "
                                 "of the K timed steps from the same start and warm-up",
                          "profiled_ms_per_step": profiled_ms / K},
        "clocks": {"sm_mhz": clocks.get("sm_mhz"), "sm_max_mhz": clocks.get("sm_max_mhz"),
                   "reasons": clocks.get("reasons", [])},
    }
    if ledger:
        line["energy_ledger"] = {
            "steps": ledger["flux_steps"],
            "field_energy_interior_J": ledger["field_energy_interior"],
            "outward_energy_J": sum(ledger["outward_energy"]),
            "remap_energy_J": ledger["remap_energy"],
            "inlet_overwrite_energy_J": ledger["inlet_overwrite_energy"],
            "particle_kinetic_J": ledger["particle_kinetic"]}
    if fp32_arm:
        line["fp32_mixed"] = fp32_arm
    if world == 1 and not args.no_scan:
        line.update(scan_benchmarks(args))
    if world == 1 and args.workload == "dipole" and not args.no_self_field:
        line.update(self_field_benchmark(args, stream))
    if world == 1 and args.workload == "dipole" and not args.no_other_configs:
        line["other_configs"] = other_configs(args, stream)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    print(json.dumps(line), flush=True)


def other_configs(args, stream):
    """Device-resident step rates of the other single-GPU configurations,
    W warm-up and K timed steps each (CUDA events on the run's stream): the
    plain FP64 drift (64x64x256, 100k), the dipole workload with the
    quintic-compensated shape, in FP64 and FP32-mixed, the dipole workload
    in the bit-reproducible current mode, and the planar-undulator workload
    (128x128x2048, 4M, FP32-mixed, from its Cowan self-field, with the
    energy ledger)."""
    import torch
    K, W = args.steps, args.warmup
    quintic = lambda: workloads.dipole_c2(steps=W + K + 4, particles=args.particles,
                                          shape="quintic-compensated", seed=17)
    cases = {
        "drift_64x64x256_100k_binomial3_fp64": (lambda: workloads.drift_c1(
            steps=W + K + 4, particles=100_000, seed=17), {}),
        "dipole_128x128x512_1M_quintic_fp64": (quintic, {}),
        "dipole_128x128x512_1M_quintic_fp32_mixed": (quintic, {"precision": "fp32-mixed"}),
        "dipole_128x128x512_1M_binomial3_fp64_deterministic": (lambda: workloads.dipole_c2(
            steps=W + K + 4, particles=args.particles, seed=17), {"deterministic": True}),
        "undulator_128x128x2048_4M_binomial3_fp32_mixed": (lambda: workloads.undulator_c3(
            steps=W + K + 4, particles=4_000_000, seed=17, precision="fp32-mixed"),
            {"self_field": True, "ledger": True}),
    }
    out = {}
    lib = native.load()
    for name, (make, options) in cases.items():
        w = make()
        cfg = w.config
        if options.get("deterministic"):
            cfg = workloads.with_determinism(cfg)
        if options.get("precision"):
            cfg = workloads.with_precision(cfg, options["precision"])
        run = native.Run(lib, cfg, stream=stream.cuda_stream)
        run.set_reference(w.reference)
        run.set_particles(w.particles)
        if options.get("self_field"):
            run.initialize_self_field(abi.self_field_config(
                cfg, hold_transverse_until_activation=True))
        if options.get("ledger"):
            run.enable_energy_ledger()
        for _ in range(W):
            run.step(1)
        run.synchronize()
        run.b("run_reset_iteration_stats", run.handle)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ps = 0
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(K):
            ps += run.particle_count()
            run.step(1)
        stop.record(stream)
        torch.cuda.synchronize()
        ms = start.elapsed_time(stop)
        stats = run.stats()
        run.close()
        out[name] = {"value": ps / (ms * 1e-3), "unit": "particle-steps/s",
                     "ms_per_step": ms / K, "steps": K, "warmup": W,
                     "cells": list(w.description["cells"]),
                     "particles": int(w.particles["x"].size),
                     "fixed_point_trials_mean": stats["total_iterations"] / max(K, 1)}
        if options.get("self_field"):
            out[name]["initial_fields"] = "cowan-relativistic-poisson self-field"
        if options.get("ledger"):
            out[name]["energy_ledger"] = True
        del w, run
    return out


def time_fp32_arm(args, w, stream, fp64_run, detector_lab_z, world):
    """The same workload in the FP32-mixed mode: W warm-up and K timed steps
    (CUDA events, inputs resident), then untimed steps up to the FP64 run's
    step, where the lab detector planes of the two runs are compared."""
    import torch
    import torch.distributed as dist
    K, W = args.steps, args.warmup
    cfg = workloads.with_precision(w.config, "fp32-mixed")
    run = native.Run(native.load(), cfg, stream=stream.cuda_stream)
    run.set_reference(w.reference)
    run.set_particles(w.particles)
    for _ in range(W):
        run.step(1)
    run.synchronize()
    run.b("run_reset_iteration_stats", run.handle)
    particle_steps = 0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(K):
        particle_steps += run.particle_count()
        run.step(1)
    stop.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop)
    stats = run.stats()
    (ms,), (particle_steps,) = over_ranks([ms], [particle_steps], world)
    while run.stats()["step"] < fp64_run.stats()["step"]:
        run.step(1)
    mixed = run.sample_field_plane(detector_lab_z).reshape(-1, 6)
    exact = fp64_run.sample_field_plane(detector_lab_z).reshape(-1, 6)
    err = [float(np.linalg.norm(mixed[:, s] - exact[:, s]) / max(np.linalg.norm(exact[:, s]), 1e-300))
           for s in (slice(0, 3), slice(3, 6))]
    run.close()
    return {"value": particle_steps / (ms * 1e-3), "unit": "particle-steps/s",
            "ms_per_step": ms / K,
            "fixed_point_trials": {"mean": stats["total_iterations"] / max(K, 1),
                                   "max": stats["max_iterations"]},
            "tolerances": {"force": cfg.force_tolerance, "work": cfg.work_tolerance},
            "detector_rel_l2_vs_fp64": {"E": err[0], "B": err[1],
                                        "step": int(fp64_run.stats()["step"])}}


# ---------------------------------------------------------------------------
# Batched ensemble (64-run class) and served scan (Poisson arrivals): seeded
# draws of independent drift/dipole runs (grid 32^3 .. 128x128x512, 1e4 ..
# 5e5 particles log-uniform, 0 .. 1.5 T, 10 .. 200 pC, sigma_z 10 .. 50 um,
# vacuum inlet).  The FP32-mixed form goes through the scan server; the
# baseline is the plain FP64 drop-in path, one run at a time.  Times are host
# wall clock around whole runs (each run ends with a device-to-host read of
# its detector plane, so no device work is outstanding at the clock reads).
def _rel_l2(a, b):
    a, b = np.asarray(a).ravel(), np.asarray(b).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _plain_fp64(lib, w, steps):
    cfg = workloads.with_precision(w.config, "fp64")
    run = native.Run(lib, cfg)
    run.allocate_reference()
    run.set_particles(w.particles)
    run.step(steps)
    det = run.sample_field_plane(workloads.detector_plane_lab_z(cfg))
    run.close()
    return det


def _percentiles(values):
    v = np.sort(np.asarray(values, dtype=np.float64))
    return {"p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99))}


SELF_FIELD_SMALL = {"cells": (48, 48, 128), "particles": 50_000, "energy_ev": 8.84e6}


def self_field_benchmark(args, stream):
    """The initial self-field solve (Cowan relativistic Poisson, tolerance
    1e-10) on the dipole grid with 1M particles at beta_z ~ 0.5, timed with
    CUDA events on the run's stream; the conjugate-gradient iterations move
    88 algorithmic bytes per lattice node (apply: read d, write Ad;
    update: read x, d, r, Ad, write x, r; direction: read r, d, write d)."""
    import torch
    w = workloads.self_field_c2(particles=args.particles)
    run = native.Run(native.load(), w.config, stream=stream.cuda_stream)
    run.set_particles(w.particles)
    config = abi.self_field_config(w.config)
    run.initialize_self_field(config)          # warm-up (allocation paths, module load)
    # Three timed solves from the same particles; the median is reported
    # (repeat solves in one process vary by up to ~40 % from box to box).
    solves = []
    for _ in range(3):
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        report = run.initialize_self_field(config)
        stop.record(stream)
        torch.cuda.synchronize()
        solves.append(start.elapsed_time(stop))
    ms = statistics.median(solves)
    # The same solve by transverse modes (sine transforms in x and y, one
    # tridiagonal system along z per mode): the direct method of the
    # reference's blocked Cowan reference, on the same operator and box.
    modal_config = abi.self_field_config(w.config, solver="modal")
    run.initialize_self_field(modal_config)
    modal = []
    for _ in range(3):
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        modal_report = run.initialize_self_field(modal_config)
        stop.record(stream)
        torch.cuda.synchronize()
        modal.append(start.elapsed_time(stop))
    modal_fields = [run.get_field(a) for a in range(6)]
    run.initialize_self_field(config)
    cg_fields = [run.get_field(a) for a in range(6)]
    modal_vs_cg = max(float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)
                      for a, b in zip(modal_fields, cg_fields))
    run.close()
    # The small case the CPU baseline also solves.
    sw = workloads.self_field_case(SELF_FIELD_SMALL["energy_ev"], nx=SELF_FIELD_SMALL["cells"][0],
                                   ny=SELF_FIELD_SMALL["cells"][1], nz=SELF_FIELD_SMALL["cells"][2],
                                   particles=SELF_FIELD_SMALL["particles"])
    small = native.Run(native.load(), sw.config, stream=stream.cuda_stream)
    small.load_workload(sw)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    small_report = small.initialize_self_field(abi.self_field_config(sw.config))
    small_ms = (time.perf_counter() - t0) * 1e3
    small.close()
    cfg = w.config
    nodes = (cfg.nx + 1) * (cfg.ny + 1) * cfg.nz
    iterations = report["iterations"]
    return {"initial_self_field": {
        "workload": w.name, "model": "cowan-relativistic-poisson", "tolerance": 1e-10,
        "particles": args.particles, "ms": ms, "ms_solves": solves, "iterations": iterations,
        "ms_per_iteration": ms / max(iterations, 1),
        "cg_bytes_per_iteration": 88 * nodes,
        "cg_gbs_upper_bound": 88 * nodes * iterations / (ms * 1e-3) / 1e9,
        "gauss_relative_residual": report["relative_residual"],
        "mean_beta_z": report["mean_beta_z"],
        "modal": {"ms": statistics.median(modal), "ms_solves": modal,
                  "gauss_relative_residual": modal_report["relative_residual"],
                  "fields_vs_cg_max_relative": modal_vs_cg},
        "small": {"workload": sw.name, "particles": SELF_FIELD_SMALL["particles"],
                  "ms_wall": small_ms, "iterations": small_report["iterations"]}}}


def scan_benchmarks(args):
    """The batched ensemble (64 seeded drift/dipole runs submitted at once)
    and the served scan (Poisson arrivals at each rate), FP32-mixed through
    the scan server (worker threads each stepping a group of runs in lock
    step) against the plain FP64 path one run at a time."""
    lib = native.load()
    out = {}
    # -- batched ensemble: every run submitted at once ---------------------
    draws = [workloads.scan_draw(i, seed=4, steps=args.ensemble_steps, precision="fp32-mixed")
             for i in range(args.ensemble_runs)]
    # Untimed warm-up: one batched pass of the same draws.  It loads the
    # kernels both paths use, tunes every grid extent's launch shapes (the
    # choices are process-wide) and grows the device memory pool, so that
    # both timed passes below run warm, as a serving process does.
    warm = native.Scan(lib, slots=args.scan_slots, runs_per_slot=args.scan_group)
    for t in [warm.submit(w.config, w.particles, args.ensemble_steps) for w in draws]:
        warm.wait(t)
    warm.close()
    t0 = time.perf_counter()
    exact = [_plain_fp64(lib, w, args.ensemble_steps) for w in draws]
    sequential_s = time.perf_counter() - t0
    scan = native.Scan(lib, slots=args.scan_slots, runs_per_slot=args.scan_group)
    t0 = time.perf_counter()
    tickets = [scan.submit(w.config, w.particles, args.ensemble_steps,
                           detector_lab_z=workloads.detector_plane_lab_z(w.config))
               for w in draws]
    results = [scan.wait(t) for t in tickets]
    batched_s = time.perf_counter() - t0
    scan.close()
    failed = [r["message"] for r in results if r["status"] != 0]
    errors = [_rel_l2(r["detector"], e) for r, e in zip(results, exact)
              if r["status"] == 0 and r["detector"] is not None and e is not None]
    out["batched_ensemble"] = {
        "runs": args.ensemble_runs, "steps": args.ensemble_steps, "slots": args.scan_slots,
        "runs_per_slot": args.scan_group,
        "warm_up": "one untimed batched pass of the same draws before both timed passes",
        "fp32_mixed_batched_solves_per_s": args.ensemble_runs / batched_s,
        "fp64_sequential_solves_per_s": args.ensemble_runs / sequential_s,
        "speedup": sequential_s / batched_s,
        "detector_rel_l2_vs_fp64": {"max": max(errors) if errors else None,
                                    "median": float(np.median(errors)) if errors else None},
        "failed": failed[:3]}
    # -- served scan: Poisson arrivals at each rate ---------------------------
    reqs = [workloads.scan_draw(100 + i, seed=5, steps=args.scan_steps, precision="fp32-mixed")
            for i in range(args.scan_requests)]

    def serve(arrivals, precision, slots, group):
        scan = native.Scan(lib, slots=slots, runs_per_slot=group)
        t_start = time.perf_counter()
        tickets = []
        for at, w in zip(arrivals, reqs):
            delay = at - (time.perf_counter() - t_start)
            if delay > 0:
                time.sleep(delay)
            cfg = workloads.with_precision(w.config, precision)
            tickets.append(scan.submit(cfg, w.particles, args.scan_steps,
                                       detector_lab_z=workloads.detector_plane_lab_z(cfg)))
        res = [scan.wait(t) for t in tickets]
        span = time.perf_counter() - t_start
        scan.close()
        return res, span

    served = []
    for rate in [float(x) for x in args.scan_rates.split(",") if x]:
        rng = np.random.default_rng(5)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, args.scan_requests))
        mixed, mixed_span = serve(arrivals, "fp32-mixed", args.scan_slots, args.scan_group)
        plain, plain_span = serve(arrivals, "fp64", 1, 1)
        errs = [_rel_l2(m["detector"], p["detector"]) for m, p in zip(mixed, plain)
                if m["status"] == 0 and p["status"] == 0 and m["detector"] is not None]
        served.append({
            "rate_req_per_s": rate, "requests": args.scan_requests,
            "arrival_span_s": float(arrivals[-1]),
            "fp32_mixed": {"solves_per_s": args.scan_requests / mixed_span,
                           "latency_ms": _percentiles([r["total_ms"] for r in mixed]),
                           "failed": sum(r["status"] != 0 for r in mixed)},
            "fp64_sequential": {"solves_per_s": args.scan_requests / plain_span,
                                "latency_ms": _percentiles([r["total_ms"] for r in plain]),
                                "failed": sum(r["status"] != 0 for r in plain)},
            "throughput_ratio": plain_span / mixed_span,
            "detector_rel_l2_vs_fp64": {"max": max(errs) if errs else None}})
    out["served_scan"] = {"steps": args.scan_steps, "slots": args.scan_slots,
                          "runs_per_slot": args.scan_group, "inlet": "vacuum (zero reference)",
                          "rates": served}
    return out


def reference_workload(args, steps, seed=17):
    """The benchmark workload itself (same grid, bunch, seed and inlet as the
    GPU arm's rank 0), for the reference's CPU translation units."""
    make, _ = WORKLOADS[args.workload]
    return make(steps, args, seed)


def _cpu_checker():
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import checkers
    if checkers.reference_available():
        b = checkers.reference()
        b.lib.ref_set_threads(os.cpu_count() or 1)
        return b, "reference", os.cpu_count() or 1
    return checkers.oracle(), "port", 1


def cpu_baseline(args):
    binding, kind, cores = _cpu_checker()
    steps = 3
    w = reference_workload(args, steps + 2)
    run = native.Run(binding, w.config).load_workload(w)
    run.step(1)  # warm-up
    done, ps, t0 = 0, 0, time.perf_counter()
    while done < steps:
        ps += run.particle_count()
        run.step(1)
        done += 1
        if time.perf_counter() - t0 > args.cpu_sample_seconds:
            break
    elapsed = time.perf_counter() - t0
    run.close()
    out = {"value": ps / elapsed, "unit": "particle-steps/s", "cores": cores, "kind": kind,
           "sample": f"{done} steps (after one warm-up step) of the full workload, "
                     f"{w.description['cells']} cells with {w.particles['x'].size} particles"}
    # The initial self-field solve of the same checker on the small solve
    # case that the GPU leg also times (initial_self_field.small).
    sw = workloads.self_field_case(SELF_FIELD_SMALL["energy_ev"], nx=SELF_FIELD_SMALL["cells"][0],
                                   ny=SELF_FIELD_SMALL["cells"][1], nz=SELF_FIELD_SMALL["cells"][2],
                                   particles=SELF_FIELD_SMALL["particles"])
    srun = native.Run(binding, sw.config).load_workload(sw)
    t0 = time.perf_counter()
    report = srun.initialize_self_field(abi.self_field_config(sw.config))
    out["initial_self_field_small"] = {"ms": (time.perf_counter() - t0) * 1e3,
                                       "iterations": report["iterations"], "cores": 1,
                                       "kind": kind, "sample": sw.name}
    srun.close()
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    binding, kind, cores = _cpu_checker()
    K, W = args.steps, args.warmup
    w = reference_workload(args, K + W + 2)
    run = native.Run(binding, w.config).load_workload(w)
    for _ in range(W):
        run.step(1)
    ps = 0
    t0 = time.perf_counter()
    for _ in range(K):
        ps += run.particle_count()
        run.step(1)
    elapsed = time.perf_counter() - t0
    stats = run.stats()
    run.close()
    value = ps / elapsed
    sample = (f"each step: one reference step of the full workload, "
              f"{w.description['cells']} cells with {w.particles['x'].size} particles")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "particle-steps/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": K, "warmup": W,
        "ms_per_step": elapsed * 1e3 / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w.name, "cells": list(w.description["cells"]),
                   "particles": args.particles, "shape": args.shape,
                   "precision": "fp64-drop-in" if args.precision == "fp64" else "fp32-mixed",
                   "magnet": WORKLOADS[args.workload][1], "boost_gamma": w.config.boost_gamma,
                   "parallelism": "replicas1", "same_config": True},
        "fixed_point_trials": {"mean": stats["total_iterations"] / max(K + W, 1),
                               "max": stats["max_iterations"]},
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores,
                         "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def launch_replicas(args, argv):
    """`--gpus N` without a launcher: start N ranks (one per GPU) through
    torch.distributed.run on this node and pass rank 0's line through."""
    import socket
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1",
           "--master-port", str(port), os.path.abspath(__file__)] + list(argv)
    return subprocess.call(cmd)


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    args = parse_args(argv)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(launch_replicas(args, argv))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
