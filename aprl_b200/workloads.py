"""Seeded synthetic workloads in the shapes of the benchmark configurations.

A workload is a run configuration (aprl_run_config), a box-frame particle
snapshot, a prepared inlet-reference table and initial fields.  Nothing here
reads a dataset: the electron bunch is drawn with the reference's own
deterministic generator (splitmix64 + Box-Muller,
src/particle_initializer.cpp:24-107) in the laboratory frame and mapped to
the boosted frame at box time zero; the inlet reference is a smooth seeded
analytic field in place of the FFTW-prepared modal reference
(src/blocked_cowan_reference.h:59-98), which is one-time initialisation.

Geometry follows the moving-window setup of
src/simulation_moving_window.cpp:53-117: the window starts at reference
cell `initial_offset`, moves one cell toward -z per step (c dt = dz), the
fixed-lab exit plane sits `right_margin` cells below the upper face, and
transverse CPML only.
"""
from dataclasses import dataclass, field
import math

import numpy as np

from . import abi

C_LIGHT = 299792458.0
ELEMENTARY_CHARGE = 1.602176634e-19
ELECTRON_MASS = 9.1093837139e-31
ELECTRON_REST_EV = 0.51099895000e6


# --------------------------------------------------------------------------
# deterministic sampler (src/particle_initializer.cpp:24-50)
def _splitmix64(v):
    v = (v + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    v = ((v ^ (v >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9))
    v = ((v ^ (v >> np.uint64(27))) * np.uint64(0x94D049BB133111EB))
    return v ^ (v >> np.uint64(31))


def _uniform_open(seed, particle, component):
    with np.errstate(over="ignore"):
        mixed = _splitmix64(np.uint64(seed) ^ _splitmix64(
            particle + np.uint64(0x100000001B3) * np.uint64(component)))
    mantissa = (mixed >> np.uint64(11)) | np.uint64(1)
    value = mantissa.astype(np.float64) * (1.0 / 9007199254740992.0)
    return np.minimum(value, 1.0 - np.finfo(np.float64).eps)


def gaussian(seed, particles, pair):
    """Standard normal deviates for particle indices `particles`."""
    with np.errstate(over="ignore"):
        first = _uniform_open(seed, particles, 2 * pair)
        second = _uniform_open(seed, particles, 2 * pair + 1)
    return np.sqrt(-2.0 * np.log(first)) * np.cos(2.0 * math.pi * second)


# --------------------------------------------------------------------------
# Lorentz helpers (src/boostframe.cpp:57-170)
def gamma_beta_from_gamma(gamma):
    return math.sqrt(gamma - 1.0) * math.sqrt(gamma + 1.0)


def gamma_from_proper_velocity(u):
    scale = np.maximum(1.0, np.max(np.abs(u), axis=-1))
    inv = 1.0 / scale
    s = u * inv[..., None]
    return scale * np.sqrt(inv * inv + np.sum(s * s, axis=-1))


def proper_velocity_lab_to_box(u_lab, boost_gamma):
    """Light-front longitudinal transform, vectorised
    (BoostFrameTransform::properVelocityLabToBox)."""
    gb = gamma_beta_from_gamma(boost_gamma)
    rapidity = boost_gamma + gb
    gamma = gamma_from_proper_velocity(u_lab)
    mt2 = u_lab[:, 0] * u_lab[:, 0] + (u_lab[:, 1] * u_lab[:, 1] + 1.0)
    positive = np.where(u_lab[:, 2] >= 0.0, gamma + u_lab[:, 2],
                        mt2 / (gamma - u_lab[:, 2]))
    positive = positive / rapidity
    out = u_lab.copy()
    out[:, 2] = 0.5 * (positive - mt2 / positive)
    return out


# --------------------------------------------------------------------------
@dataclass
class Workload:
    name: str
    config: abi.RunConfig
    particles: dict            # x y z ux uy uz charge mass id (numpy arrays)
    reference: list            # 6 arrays in native (k, j, i) layout
    fields: list = field(default_factory=list)  # 9 arrays or [] for zero
    steps: int = 0             # steps the reference table covers
    description: dict = field(default_factory=dict)


# Fixed-point stopping rule of the FP32-mixed mode.  Its binary32 gathers
# put a floor under the trial-to-trial residual (force ~1e-10, relative work
# ~1e-9), so the binary64 tolerances 1e-13 / 1e-8 cannot be met; 1e-9 / 1e-5
# stop at the minimum two trials.
FP32_FORCE_TOLERANCE = 1.0e-9
FP32_WORK_TOLERANCE = 1.0e-5


def with_precision(cfg, precision):
    """A copy of `cfg` in the given precision ("fp64" or "fp32-mixed"), with
    that precision's fixed-point tolerances."""
    out = abi.RunConfig.from_buffer_copy(bytes(cfg))
    out.precision = abi.PRECISIONS[precision] if isinstance(precision, str) else precision
    if out.precision == abi.PRECISION_FP32_MIXED:
        out.force_tolerance = FP32_FORCE_TOLERANCE
        out.work_tolerance = FP32_WORK_TOLERANCE
    else:
        out.force_tolerance = 1.0e-13
        out.work_tolerance = 1.0e-8
    return out


def with_determinism(cfg, deterministic=True):
    """A copy of `cfg` with the bit-reproducible current summation on or off."""
    out = abi.RunConfig.from_buffer_copy(bytes(cfg))
    out.deterministic = 1 if deterministic else 0
    return out


def with_reference_surface_current(w):
    """`w` with the reference's equivalent surface current on: the prepared
    reference then has to cover the whole window over the run (the current
    is sampled at every window plane), so its table is extended to
    initial_offset + nz + 2 planes and drawn again."""
    cfg = abi.RunConfig.from_buffer_copy(bytes(w.config))
    cfg.reference_surface_current = 1
    cfg.reference_nz = max(cfg.reference_nz, cfg.initial_offset + cfg.nz + 2)
    return Workload(w.name + "-surface-current", cfg, w.particles, synthetic_reference(cfg),
                    w.fields, steps=w.steps, description=dict(w.description))


def make_config(nx, ny, nz, dx, dy, dz, cpml_cells, boost_gamma, shape,
                steps, substeps=1, magnets=(), right_margin=None,
                translation_beta=1.0, release_cells=6):
    """Run configuration of a moving window with `steps` of inlet reference."""
    cfg = abi.RunConfig()
    cfg.nx, cfg.ny, cfg.nz = nx, ny, nz
    cfg.dx, cfg.dy, cfg.dz = dx, dy, dz
    cfg.dt = dz / C_LIGHT
    cfg.cpml_cells_x = cpml_cells
    cfg.cpml_cells_y = cpml_cells
    cfg.cpml_polynomial_order = 3.0
    cfg.cpml_target_reflection = 1.0e-8
    cfg.cpml_kappa_max = 8.0
    cfg.cpml_alpha_fraction = 0.0
    cfg.shape = abi.SHAPES[shape] if isinstance(shape, str) else shape
    cfg.substeps = substeps
    cfg.max_trials = 64
    cfg.force_tolerance = 1.0e-13
    cfg.work_tolerance = 1.0e-8
    gb = gamma_beta_from_gamma(boost_gamma)
    cfg.boost_gamma = boost_gamma
    cfg.boost_gamma_beta = gb
    cfg.boost_beta = gb / boost_gamma
    cfg.lab_time_origin = 0.0
    cfg.lab_z_origin = 0.0
    cfg.box_z_origin = 0.0
    cfg.translation_beta = translation_beta
    # The inlet queries reach z = offset - 1 - translation_beta*step >= 0
    # over `steps` steps (src/simulation_moving_window.cpp:97-104).
    offset = int(math.ceil((1.0 + translation_beta) * (steps + 1))) + 2
    cfg.initial_offset = offset
    cfg.reference_nz = offset + 2
    cfg.reference_origin[0] = -0.5 * nx * dx
    cfg.reference_origin[1] = -0.5 * ny * dy
    cfg.reference_origin[2] = -offset * dz      # window starts at box z = 0
    if right_margin is None:
        right_margin = 8 + int(math.ceil((1.0 - cfg.boost_beta) * steps))
    safe_exit = (nz - right_margin) * dz          # box z at t = 0
    # labZFromBoxZT(safe_exit, 0) = labZOrigin + gamma*(z - boxZOrigin)
    cfg.exit_lab_z = cfg.lab_z_origin + boost_gamma * (safe_exit - cfg.box_z_origin)
    # Held particles release at a fixed lab plane `release_cells` above the
    # window inlet at t = 0 (startCell = release - lowerGuardCells,
    # src/simulation_moving_window.cpp:83).
    cfg.activation_plane_lab_z = cfg.lab_z_origin + boost_gamma * (release_cells * dz)
    cfg.maximum_step = steps
    cfg.n_magnets = len(magnets)
    for n, m in enumerate(magnets):
        cfg.magnets[n] = m
    return cfg


def dipole(field_t, center_z=-10.0, length=100.0, angle=0.0):
    m = abi.Magnet()
    m.type = abi.MAGNET_UNIFORM_DIPOLE
    m.center[2] = center_z
    m.length = length
    m.peak_field = field_t
    m.polarization_angle = angle
    m.fringe_relative_cutoff = 1.0e-9
    m.wave_number = 0.0
    m.fringe_extent = 0.0
    m.cos_angle = math.cos(angle)
    m.sin_angle = math.sin(angle)
    return m


def planar_undulator(k_parameter, period, entrance_z, periods, angle=0.0):
    """SIMagneticElement::planarUndulatorFromK (src/eb_sources.cpp:290-307)."""
    m = abi.Magnet()
    m.type = abi.MAGNET_PLANAR_UNDULATOR
    m.gaussian_fringe = 1
    m.center[2] = entrance_z
    m.period = period
    m.length = periods * period
    m.peak_field = (k_parameter * 2.0 * math.pi * ELECTRON_MASS * C_LIGHT /
                    (ELEMENTARY_CHARGE * period))
    m.polarization_angle = angle
    m.fringe_relative_cutoff = 1.0e-9
    m.wave_number = 2.0 * math.pi / period
    m.fringe_extent = math.sqrt(-2.0 * math.log(1.0e-9)) / m.wave_number
    m.cos_angle = math.cos(angle)
    m.sin_angle = math.sin(angle)
    return m


def held_beta_z(u_lab, boost_gamma):
    """BoostFrameTransform::heldLongitudinalBetaZ for a lab proper velocity:
    keep only lab u_z, boost it, beta = u/hypot(1, u)
    (src/boostframe.cpp:96-107)."""
    gb = gamma_beta_from_gamma(boost_gamma)
    uz = u_lab[:, 2]
    g = np.sqrt(1.0 + uz * uz)
    positive = np.where(uz >= 0.0, g + uz, 1.0 / (g - uz)) / (boost_gamma + gb)
    u_box = 0.5 * (positive - 1.0 / positive)
    return u_box / np.hypot(1.0, u_box)


def gaussian_bunch(cfg, count, charge_c, energy_ev, sigma_xy, sigma_z_lab,
                   emittance_n, energy_spread, seed=17, margin_cells=3,
                   z_fraction=(0.05, 0.95), z_range=None, uniform_z=False):
    """Box-frame snapshot of a lab-frame Gaussian electron bunch, truncated
    to the moving window's trusted particle region (inside the transverse
    CPML by `margin_cells`, above the inlet guard, below the exit plane).
    uniform_z: the window holds a slice of a bunch much longer than it, so z
    is drawn uniformly over the slice (seeded random longitudinal phases)."""
    gamma_lab = energy_ev / ELECTRON_REST_EV
    u0 = gamma_beta_from_gamma(gamma_lab)
    boost = cfg.boost_gamma
    beta_b = cfg.boost_beta
    sigma_z_box = sigma_z_lab * boost * (1.0 + beta_b)
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    x_lo = cfg.reference_origin[0] + (cfg.cpml_cells_x + margin_cells) * cfg.dx
    x_hi = cfg.reference_origin[0] + (nx - cfg.cpml_cells_x - margin_cells) * cfg.dx
    y_lo = cfg.reference_origin[1] + (cfg.cpml_cells_y + margin_cells) * cfg.dy
    y_hi = cfg.reference_origin[1] + (ny - cfg.cpml_cells_y - margin_cells) * cfg.dy
    exit_box = cfg.exit_lab_z / boost
    z_lo = 2.0 * cfg.dz + z_fraction[0] * (exit_box - 2.0 * cfg.dz)
    z_hi = 2.0 * cfg.dz + z_fraction[1] * (exit_box - 2.0 * cfg.dz)
    if z_range is not None:
        z_lo, z_hi = z_range
    z_center = 0.5 * (z_lo + z_hi)

    if not (x_lo < x_hi and y_lo < y_hi and z_lo < z_hi):
        raise ValueError("the trusted particle region of this window is empty")
    kept = []
    total = 0
    index = np.uint64(0)
    block = max(4 * count, 4096)
    for _ in range(64):
        if total >= count:
            break
        ids = np.arange(int(index), int(index) + block, dtype=np.uint64)
        index = np.uint64(int(index) + block)
        x = sigma_xy * gaussian(seed, ids, 0)
        y = sigma_xy * gaussian(seed, ids, 1)
        if uniform_z:
            z = z_lo + (z_hi - z_lo) * _uniform_open(seed ^ 0x5DEECE66D, ids, 7)
        else:
            z = z_center + sigma_z_box * gaussian(seed, ids, 2)
        pseed = seed ^ 0xD6E8FEB86659FD93
        sigma_u = emittance_n / sigma_xy
        ux = sigma_u * gaussian(pseed, ids, 0)
        uy = sigma_u * gaussian(pseed, ids, 1)
        uz = u0 * (1.0 + energy_spread * gaussian(pseed, ids, 2))
        ok = ((x > x_lo) & (x < x_hi) & (y > y_lo) & (y < y_hi) &
              (z > z_lo) & (z < z_hi))
        sel = np.nonzero(ok)[0][: count - total]
        kept.append((ids[sel], x[sel], y[sel], z[sel], ux[sel], uy[sel], uz[sel]))
        total += sel.size
    if total < count:
        raise ValueError("the bunch barely overlaps the trusted particle region")
    cols = [np.concatenate(c) for c in zip(*kept)]
    ids, x, y, z, ux, uy, uz = cols
    u_lab = np.stack([ux, uy, uz], axis=1)
    u_box = proper_velocity_lab_to_box(u_lab, boost)
    electrons = charge_c / ELEMENTARY_CHARGE
    per = electrons / count
    beta_held = held_beta_z(u_lab, boost)
    return {
        "beta_held": np.ascontiguousarray(beta_held),
        "x": np.ascontiguousarray(x), "y": np.ascontiguousarray(y),
        "z": np.ascontiguousarray(z),
        "ux": np.ascontiguousarray(u_box[:, 0]),
        "uy": np.ascontiguousarray(u_box[:, 1]),
        "uz": np.ascontiguousarray(u_box[:, 2]),
        "charge": np.full(count, -ELEMENTARY_CHARGE * per),
        "mass": np.full(count, ELECTRON_MASS * per),
        "id": (ids + np.uint64(1)).astype(np.uint64),
    }


def synthetic_reference(cfg, amplitude=1.0e3, seed=5):
    """Smooth seeded analytic inlet reference, native layout (k, j, i)."""
    rng = np.random.default_rng(seed)
    out = []
    for a in range(6):
        nx_c, ny_c, nz_c = abi.reference_shape(cfg, a)
        phase = rng.uniform(0.0, 2.0 * math.pi, size=3)
        i = np.arange(nx_c)[None, None, :]
        j = np.arange(ny_c)[None, :, None]
        k = np.arange(nz_c)[:, None, None]
        value = (np.sin(2 * math.pi * (i + 0.5) / nx_c + phase[0]) *
                 np.cos(2 * math.pi * (j + 0.25) / ny_c + phase[1]) *
                 np.cos(2 * math.pi * k / 37.0 + phase[2]))
        scale = amplitude if a < 3 else amplitude / C_LIGHT
        out.append(np.ascontiguousarray((scale * value).astype(np.float64)))
    return out


def synthetic_fields(cfg, amplitude=1.0e4, seed=11):
    """Smooth seeded E/B start fields (J zero), native layout (k, j, i)."""
    rng = np.random.default_rng(seed)
    out = []
    for a in range(9):
        shape = abi.field_shape(cfg, a)
        if a >= 6:
            out.append(np.zeros(shape[::-1]))
            continue
        phase = rng.uniform(0.0, 2.0 * math.pi, size=3)
        i = np.arange(shape[0])[None, None, :]
        j = np.arange(shape[1])[None, :, None]
        k = np.arange(shape[2])[:, None, None]
        value = (np.sin(2 * math.pi * i / 13.0 + phase[0]) *
                 np.sin(2 * math.pi * j / 11.0 + phase[1]) *
                 np.cos(2 * math.pi * k / 17.0 + phase[2]))
        scale = amplitude if a < 3 else amplitude / C_LIGHT
        out.append(np.ascontiguousarray(scale * value))
    return out


# --------------------------------------------------------------------------
# named workloads (benchmark configurations and small parity cases)
def drift_c1(steps=200, particles=100_000, shape="linear-binomial3", seed=17,
             precision="fp64"):
    """Plain FP64 drift: 64x64x256 cells, dx=dy=5 um, dz=2 um, 8-cell CPML."""
    cfg = with_precision(make_config(64, 64, 256, 5e-6, 5e-6, 2e-6, 8, 10.0, shape, steps),
                         precision)
    bunch = gaussian_bunch(cfg, particles, 100e-12, 1e9, 50e-6, 20e-6, 1e-6,
                           1e-4, seed=seed)
    return Workload("drift-64x64x256", cfg, bunch, synthetic_reference(cfg),
                    steps=steps,
                    description={"cells": [64, 64, 256], "particles": particles,
                                 "shape": shape, "boost_gamma": 10.0})


def dipole_c2(steps=2000, particles=1_000_000, shape="linear-binomial3",
              seed=17, precision="fp64"):
    """Dipole bending radiation: 128x128x512 cells, 10-cell CPML, 1 T lab
    dipole, boost gamma 10."""
    cfg = with_precision(make_config(128, 128, 512, 5e-6, 5e-6, 2e-6, 10, 10.0, shape,
                                     steps, magnets=[dipole(1.0)]), precision)
    bunch = gaussian_bunch(cfg, particles, 100e-12, 1e9, 50e-6, 20e-6, 1e-6,
                           1e-4, seed=seed)
    return Workload("dipole-128x128x512", cfg, bunch, synthetic_reference(cfg),
                    steps=steps,
                    description={"cells": [128, 128, 512], "particles": particles,
                                 "shape": shape, "boost_gamma": 10.0,
                                 "dipole_T": 1.0, "precision": precision})


def undulator_c3(steps=5000, particles=4_000_000, shape="linear-binomial3", seed=17,
                 precision="fp32-mixed"):
    """Planar-undulator beam: period 3 cm, K = 1, gamma_lab 3000 (energy
    spread 1e-4, sigma_xy 30 um, sigma_z 50 um lab), boosted to the
    undulator-resonant frame gamma_b = gamma / sqrt(1 + K^2/2)
    (utilities/undulator_resonance.cpp:155-157); 128x128x2048 cells.  In that
    frame the bunch is far longer than the window, so the window holds a
    slice with uniformly random longitudinal phases (shot noise)."""
    k_parameter, gamma_lab = 1.0, 3000.0
    boost = gamma_lab / math.sqrt(1.0 + 0.5 * k_parameter ** 2)
    cfg = with_precision(make_config(128, 128, 2048, 4e-6, 4e-6, 1e-6, 10, boost, shape, steps,
                                     magnets=[planar_undulator(k_parameter, 0.03, -1.0, 1000)]),
                         precision)
    # weight ~355 per macro-particle
    charge = 355.0 * particles * ELEMENTARY_CHARGE
    bunch = gaussian_bunch(cfg, particles, charge, gamma_lab * ELECTRON_REST_EV, 30e-6, 50e-6,
                           1e-6, 1e-4, seed=seed, uniform_z=True)
    return Workload("undulator-128x128x2048", cfg, bunch, synthetic_reference(cfg),
                    steps=steps,
                    description={"cells": [128, 128, 2048], "particles": particles,
                                 "shape": shape, "boost_gamma": boost,
                                 "undulator": {"period_m": 0.03, "K": k_parameter},
                                 "precision": precision})


def split_held(cfg, bunch):
    """Frozen flags for held lab-plane injection: particles below the
    activation plane's box position at t = 0 are held (src/eb_bunch.cpp)."""
    release_box = (cfg.activation_plane_lab_z - cfg.lab_z_origin) / cfg.boost_gamma
    return (bunch["z"] < release_box).astype(np.uint8)


def streaming_case(nx=16, ny=16, nz=40, particles=600, steps=12,
                   shape="linear-binomial3", magnets=None, seed=5, cpml=4,
                   upstream_cells=24, margin_cells=2):
    """A bunch straddling the inlet: pending upstream, held between the
    inlet and the activation plane, active above it."""
    if magnets is None:
        magnets = [dipole(1.0)]
    cfg = make_config(nx, ny, nz, 5e-6, 5e-6, 2e-6, cpml, 10.0, shape, steps,
                      magnets=magnets)
    exit_box = cfg.exit_lab_z / cfg.boost_gamma
    z_range = (-upstream_cells * cfg.dz, 0.8 * exit_box)
    bunch = gaussian_bunch(cfg, particles, 20e-12, 1e9, 12e-6, 10e-6, 1e-6,
                           1e-4, seed=seed, z_range=z_range,
                           margin_cells=margin_cells)
    w = Workload(f"stream-{nx}x{ny}x{nz}", cfg, bunch, synthetic_reference(cfg),
                 synthetic_fields(cfg), steps=steps,
                 description={"cells": [nx, ny, nz], "particles": particles,
                              "shape": shape, "held_injection": True})
    w.held = split_held(cfg, bunch)
    return w


def small_case(nx=16, ny=16, nz=40, particles=400, steps=6,
               shape="linear-binomial3", magnets=None, seed=3, cpml=4,
               fields=True, z_fraction=(0.05, 0.95), margin_cells=2):
    """A grid the serial oracle steps in well under a second."""
    if magnets is None:
        magnets = [dipole(1.0)]
    cfg = make_config(nx, ny, nz, 5e-6, 5e-6, 2e-6, cpml, 10.0, shape, steps,
                      magnets=magnets)
    bunch = gaussian_bunch(cfg, particles, 20e-12, 1e9, 12e-6, 10e-6, 1e-6,
                           1e-4, seed=seed, z_fraction=z_fraction,
                           margin_cells=margin_cells)
    return Workload(f"small-{nx}x{ny}x{nz}", cfg, bunch,
                    synthetic_reference(cfg),
                    synthetic_fields(cfg) if fields else [], steps=steps,
                    description={"cells": [nx, ny, nz], "particles": particles,
                                 "shape": shape})


def self_field_case(energy_ev=8.84e6, nx=16, ny=16, nz=40, particles=400, seed=3,
                    margin_cells=2, steps=6):
    """A bunch whose box-frame mean velocity is moderate (lab energy near the
    boost's: 5.11 MeV gives beta_z ~ 0, 8.84 MeV ~ 0.5), the regime the
    initial self-field solve is meant for."""
    cfg = make_config(nx, ny, nz, 5e-6, 5e-6, 2e-6, 4, 10.0, "linear-binomial3", steps,
                      magnets=[])
    bunch = gaussian_bunch(cfg, particles, 20e-12, energy_ev, 12e-6, 10e-6, 1e-6, 1e-4,
                           seed=seed, margin_cells=margin_cells)
    return Workload(f"self-field-{nx}x{ny}x{nz}", cfg, bunch, synthetic_reference(cfg), [],
                    steps=steps, description={"energy_ev": energy_ev})


def self_field_c2(particles=1_000_000, seed=17, energy_ev=8.84e6):
    """The dipole grid (128x128x512 cells, 10-cell CPML, boost gamma 10) with
    a 100 pC bunch moving at beta_z ~ 0.5 in the box (8.84 MeV lab): the
    initial self-field solve's regime."""
    cfg = make_config(128, 128, 512, 5e-6, 5e-6, 2e-6, 10, 10.0, "linear-binomial3", 8,
                      magnets=[])
    bunch = gaussian_bunch(cfg, particles, 100e-12, energy_ev, 50e-6, 20e-6, 1e-6, 1e-4,
                           seed=seed)
    return Workload("self-field-128x128x512", cfg, bunch, synthetic_reference(cfg), [],
                    steps=8, description={"cells": [128, 128, 512], "particles": particles,
                                          "energy_ev": energy_ev})


# ---------------------------------------------------------------------------
# Batched ensemble and served scan: seeded draws of independent runs.
def scan_draw(index, seed=2024, steps=500, precision="fp32-mixed",
              shape="linear-binomial3", cells_min=(32, 32, 32), cells_max=(128, 128, 512),
              particles_range=(1.0e4, 5.0e5)):
    """Request `index` of a seeded parameter scan of drift/dipole runs: grid
    extents uniform in [cells_min, cells_max], particle count log-uniform in
    particles_range, lab dipole field uniform in [0, 1.5] T, bunch charge
    uniform in [10, 200] pC, lab sigma_z uniform in [10, 50] um.  The inlet
    is the vacuum (zero) reference.  Smallest useful extent: 2*(8+3)+2 cells
    transversely (CPML plus particle margin)."""
    rng = np.random.default_rng([seed, index])
    nx = int(rng.integers(cells_min[0], cells_max[0] + 1))
    ny = int(rng.integers(cells_min[1], cells_max[1] + 1))
    nz = int(rng.integers(cells_min[2], cells_max[2] + 1))
    lo, hi = math.log10(particles_range[0]), math.log10(particles_range[1])
    particles = int(round(10.0 ** rng.uniform(lo, hi)))
    bend = float(rng.uniform(0.0, 1.5))
    charge = float(rng.uniform(10e-12, 200e-12))
    sigma_z = float(rng.uniform(10e-6, 50e-6))
    magnets = [dipole(bend)] if bend > 0.0 else []
    cfg = with_precision(make_config(nx, ny, nz, 5e-6, 5e-6, 2e-6, 8, 10.0, shape, steps,
                                     magnets=magnets), precision)
    # sigma_xy is 50 um, narrowed on small grids to a quarter of the trusted
    # transverse width so the bunch is not mostly truncated.
    trusted = (min(nx, ny) - 2 * (8 + 3)) * 5e-6
    sigma_xy = min(50e-6, 0.25 * trusted)
    bunch = gaussian_bunch(cfg, particles, charge, 1e9, sigma_xy, sigma_z, 1e-6, 1e-4,
                           seed=seed * 1000 + index)
    return Workload(f"scan-{index}-{nx}x{ny}x{nz}", cfg, bunch, None, steps=steps,
                    description={"cells": [nx, ny, nz], "particles": particles,
                                 "dipole_T": bend, "charge_C": charge,
                                 "sigma_z_m": sigma_z, "precision": precision})


def detector_plane_lab_z(cfg, fraction=0.5):
    """A fixed lab detector plane `fraction` of the way up the initial window."""
    return cfg.lab_z_origin + cfg.boost_gamma * (fraction * cfg.nz * cfg.dz)
