"""ctypes mirror of the plain-data types in include/aprl_gpu.h.

Only data layouts live here; the loader for the CUDA library is in
aprl_b200/native.py.
"""
import ctypes as C

APRL_OK = 0
APRL_ERR_INVALID_ARGUMENT = 1
APRL_ERR_OUT_OF_RANGE = 2
APRL_ERR_RUNTIME = 3
APRL_ERR_NOT_CONVERGED = 4
APRL_ERR_CUDA = 5
APRL_ERR_UNSUPPORTED = 6

STATUS_NAMES = {
    APRL_OK: "ok",
    APRL_ERR_INVALID_ARGUMENT: "invalid_argument",
    APRL_ERR_OUT_OF_RANGE: "out_of_range",
    APRL_ERR_RUNTIME: "runtime_error",
    APRL_ERR_NOT_CONVERGED: "not_converged",
    APRL_ERR_CUDA: "cuda_error",
    APRL_ERR_UNSUPPORTED: "unsupported",
}

SHAPE_LINEAR_BINOMIAL3 = 0
SHAPE_QUINTIC_COMPENSATED = 1
SHAPES = {"linear-binomial3": SHAPE_LINEAR_BINOMIAL3,
          "quintic-compensated": SHAPE_QUINTIC_COMPENSATED}

PRECISION_FP64 = 0
PRECISION_FP32_MIXED = 1
PRECISIONS = {"fp64": PRECISION_FP64, "fp32-mixed": PRECISION_FP32_MIXED}

MAGNET_PLANAR_UNDULATOR = 0
MAGNET_UNIFORM_DIPOLE = 1
MAGNET_QUADRUPOLE = 2
MAX_MAGNETS = 4

# Field component order of the ABI: Ex Ey Ez Bx By Bz Jx Jy Jz.
COMPONENTS = ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Jx", "Jy", "Jz")


class Magnet(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("gaussian_fringe", C.c_int32),
        ("center", C.c_double * 3),
        ("length", C.c_double),
        ("period", C.c_double),
        ("peak_field", C.c_double),
        ("polarization_angle", C.c_double),
        ("fringe_relative_cutoff", C.c_double),
        ("quadrupole_gradient", C.c_double),
        ("wave_number", C.c_double),
        ("fringe_extent", C.c_double),
        ("cos_angle", C.c_double),
        ("sin_angle", C.c_double),
    ]


class RunConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_uint64), ("ny", C.c_uint64), ("nz", C.c_uint64),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("dt", C.c_double),
        ("cpml_cells_x", C.c_uint64), ("cpml_cells_y", C.c_uint64),
        ("cpml_polynomial_order", C.c_double),
        ("cpml_target_reflection", C.c_double),
        ("cpml_kappa_max", C.c_double),
        ("cpml_alpha_fraction", C.c_double),
        ("shape", C.c_int32),
        ("substeps", C.c_uint32),
        ("max_trials", C.c_uint32),
        ("precision", C.c_uint32),
        ("force_tolerance", C.c_double),
        ("work_tolerance", C.c_double),
        ("boost_gamma", C.c_double), ("boost_beta", C.c_double),
        ("boost_gamma_beta", C.c_double),
        ("lab_time_origin", C.c_double), ("lab_z_origin", C.c_double),
        ("box_z_origin", C.c_double),
        ("reference_origin", C.c_double * 3),
        ("initial_offset", C.c_int64),
        ("reference_nz", C.c_uint64),
        ("translation_beta", C.c_double),
        ("exit_lab_z", C.c_double),
        ("activation_plane_lab_z", C.c_double),
        ("maximum_step", C.c_uint64),
        ("n_magnets", C.c_uint32),
        ("inlet_charge_match", C.c_uint32),
        ("magnets", Magnet * MAX_MAGNETS),
        ("deterministic", C.c_uint32),
        ("reference_surface_current", C.c_uint32),
    ]

    @classmethod
    def from_bytes(cls, raw):
        """A config from its raw bytes; fields appended after an older layout
        was written (the deterministic flag) read as zero."""
        raw = bytes(raw)
        if len(raw) < C.sizeof(cls):
            raw = raw + bytes(C.sizeof(cls) - len(raw))
        return cls.from_buffer_copy(raw)


class StepStats(C.Structure):
    _fields_ = [
        ("step", C.c_uint64),
        ("iterations", C.c_uint32),
        ("max_iterations", C.c_uint32),
        ("total_iterations", C.c_uint64),
        ("force", C.c_double),
        ("work", C.c_double),
        ("particles", C.c_uint64),
        ("carriers", C.c_uint64),
        ("exits", C.c_uint64),
        ("exit_charge", C.c_double),
        ("cpml_entries", C.c_uint64 * 6),
        ("cpml_entry_charge", C.c_double * 6),
        ("carrier_outer", C.c_uint64 * 6),
        ("carrier_outer_charge", C.c_double * 6),
        ("cropped_carriers", C.c_uint64),
        ("cropped_charge", C.c_double),
        ("window_offset", C.c_int64),
        ("origin_z", C.c_double),
        ("time_box", C.c_double),
        ("device_error", C.c_uint32),
        ("reserved", C.c_uint32),
        ("pending", C.c_uint64),
        ("admitted", C.c_uint64),
        ("activations", C.c_uint64),
        ("held", C.c_uint64),
    ]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            value = getattr(self, name)
            if isinstance(value, C.Array):
                value = list(value)
            out[name] = value
        return out


class EnergyLedger(C.Structure):
    """aprl_energy_ledger: the moving-window energy ledger and the field and
    particle energy sums of the current state (joules, watts)."""
    _fields_ = [
        ("inlet_overwrite_energy", C.c_double),
        ("inserted_energy", C.c_double),
        ("cropped_energy", C.c_double),
        ("remap_energy", C.c_double),
        ("outward_energy", C.c_double * 6),
        ("overwrite_events", C.c_uint64),
        ("flux_steps", C.c_uint64),
        ("remap_steps", C.c_uint64),
        ("field_energy_interior", C.c_double),
        ("boundary_power", C.c_double * 6),
        ("particle_kinetic", C.c_double),
        ("particle_total", C.c_double),
        ("represented_electrons", C.c_double),
        ("particles", C.c_uint64),
    ]

    as_dict = StepStats.as_dict


class GaussLaw(C.Structure):
    """aprl_gauss_law: eps0 div E - rho over the nodes of the current state."""
    _fields_ = [
        ("max_residual", C.c_double),
        ("rms_residual", C.c_double),
        ("max_charge_density", C.c_double),
        ("total_charge", C.c_double),
        ("interior_nodes", C.c_uint64),
        ("outside", C.c_uint64),
    ]

    as_dict = StepStats.as_dict


SELF_FIELD_MODELS = {"relativistic-poisson": 0, "electrostatic-poisson": 1,
                     "cowan-relativistic-poisson": 2}


class SelfFieldConfig(C.Structure):
    """aprl_self_field_config: EBGaussFieldInitializer::initialize's controls."""
    _fields_ = [
        ("model", C.c_int32),
        ("include_transverse_cpml_particles", C.c_int32),
        ("hold_transverse_until_activation", C.c_int32),
        ("solver", C.c_int32),
        ("relative_tolerance", C.c_double),
        ("maximum_mean_transverse_beta", C.c_double),
        ("maximum_iterations", C.c_uint64),
        ("guard_cells", C.c_uint64 * 3),
        ("source_shape", C.c_int32),
        ("open_transverse", C.c_int32),
    ]


SOURCE_SHAPES = {"cic": 0, "run-shape": 1}


class SelfFieldReport(C.Structure):
    """aprl_self_field_report: EBGaussInitializationReport."""
    _fields_ = [
        ("iterations", C.c_uint64),
        ("relative_residual", C.c_double),
        ("maximum_gauss_residual", C.c_double),
        ("total_charge", C.c_double),
        ("mean_beta_z", C.c_double),
        ("mean_beta_transverse", C.c_double),
        ("initial_electric_energy", C.c_double),
        ("initial_magnetic_energy", C.c_double),
        ("rms_position_cells", C.c_double * 3),
        ("centre_padding_rms", C.c_double * 3),
        ("static_field_guard_cells", C.c_uint64 * 3),
        ("transverse_poisson_padding_cells", C.c_uint64),
        ("temporary_bytes", C.c_uint64),
    ]

    as_dict = StepStats.as_dict


def self_field_config(run_config, model="cowan-relativistic-poisson", tolerance=1e-10,
                      maximum_iterations=20000, maximum_mean_transverse_beta=0.05,
                      include_transverse_cpml_particles=False,
                      hold_transverse_until_activation=False, solver="cg",
                      source_shape="cic", open_transverse=False):
    """The initializer controls with the CPML cells as the static guard;
    solver "cg" (the reference's initializer) or "modal" (transverse sine
    modes and a tridiagonal solve along z per mode); source_shape "cic"
    (the initializer's charge) or "run-shape" (the shaped source of the
    moving window's prepared reference); open_transverse: the potential
    extends to the outer transverse faces, held there at the free-space
    potential of the charge (needs solver "modal")."""
    c = SelfFieldConfig()
    c.solver = {"cg": 0, "modal": 1}[solver]
    c.source_shape = SOURCE_SHAPES[source_shape]
    c.open_transverse = int(open_transverse)
    c.model = SELF_FIELD_MODELS[model]
    c.include_transverse_cpml_particles = int(include_transverse_cpml_particles)
    c.hold_transverse_until_activation = int(hold_transverse_until_activation)
    c.relative_tolerance = tolerance
    c.maximum_mean_transverse_beta = maximum_mean_transverse_beta
    c.maximum_iterations = maximum_iterations
    c.guard_cells[0] = run_config.cpml_cells_x
    c.guard_cells[1] = run_config.cpml_cells_y
    c.guard_cells[2] = 0
    return c


def field_shape(config, component):
    """Yee extents (nx_c, ny_c, nz_c) of an ABI component (x fastest)."""
    cells = (config.nx, config.ny, config.nz)
    electric = component < 3 or component >= 6
    axis = component % 3
    return tuple(cells[d] + ((d != axis) if electric else (d == axis))
                 for d in range(3))


def reference_shape(config, component):
    """Extents of one prepared-reference component over reference_nz cells."""
    nx_c, ny_c, _ = field_shape(config, component)
    return (nx_c, ny_c,
            config.reference_nz + (1 if component in (0, 1, 5) else 0))


def history_shape(config, index):
    """(slots, layers, row) of CPML history `index` (0..11), or None when the
    term is inactive (z-derivative histories under the moving window)."""
    pairs = ((0, 1), (0, 2), (1, 2), (1, 0), (2, 0), (2, 1))
    comp, der = pairs[index % 6]
    if der == 2:
        return None
    electric = index >= 6
    shape = field_shape(config, comp if electric else 3 + comp)
    cells = config.cpml_cells_x if der == 0 else config.cpml_cells_y
    # makeProfile marks 2*cells active points on each derivative axis
    # (cells on each side) for magnetic (half-integer) positions and
    # 2*cells (+0) for electric nodes: the node at the thickness edge has
    # zero depth and is inactive.
    slots = 2 * cells
    row = shape[1] if der == 0 else shape[0]
    return (slots, shape[2], row)


# Parameter-scan server (aprl_scan_*).
SCAN_QUEUED, SCAN_RUNNING, SCAN_DONE = 0, 1, 2


class ScanConfig(C.Structure):
    _fields_ = [("device_budget_bytes", C.c_uint64),
                ("max_slots", C.c_uint32),
                ("runs_per_slot", C.c_uint32)]


_PD = C.POINTER(C.c_double)


class ScanRequest(C.Structure):
    _fields_ = [("config", RunConfig),
                ("steps", C.c_uint64),
                ("particles", C.c_size_t),
                ("x", _PD), ("y", _PD), ("z", _PD),
                ("ux", _PD), ("uy", _PD), ("uz", _PD),
                ("charge", _PD), ("mass", _PD),
                ("id", C.POINTER(C.c_uint64)),
                ("frozen", C.POINTER(C.c_uint8)),
                ("frozen_beta_z", _PD),
                ("reference", _PD * 6),
                ("detector_lab_z", C.c_double),
                ("detector", _PD)]


class ScanResult(C.Structure):
    _fields_ = [("state", C.c_int32),
                ("status", C.c_int32),
                ("detector_inside", C.c_int32),
                ("slot", C.c_int32),
                ("footprint_bytes", C.c_uint64),
                ("queued_ms", C.c_double),
                ("run_ms", C.c_double),
                ("total_ms", C.c_double),
                ("submit_s", C.c_double),
                ("start_s", C.c_double),
                ("finish_s", C.c_double),
                ("stats", StepStats),
                ("message", C.c_char * 256)]


class Tuning(C.Structure):
    """aprl_tuning: the autotuner's launch shapes for one grid extent."""
    _fields_ = [("decided", C.c_int32),
                ("cowan_planes_per_block", C.c_uint32),
                ("preview_block", C.c_uint32 * 2),
                ("orbit_block", C.c_uint32 * 2),
                ("commit_block", C.c_uint32 * 2),
                ("candidate_ms", (C.c_float * 4) * 4)]

    def as_dict(self):
        return {"decided": [bool(self.decided >> k & 1) for k in range(4)],
                "cowan_planes_per_block": self.cowan_planes_per_block,
                "preview_block": list(self.preview_block),
                "orbit_block": list(self.orbit_block),
                "commit_block": list(self.commit_block),
                "candidate_ms": [list(row) for row in self.candidate_ms]}
