"""ctypes binding of the C ABI (include/aprl_gpu.h) and a thin Python handle.

`load()` opens the in-tree CUDA library aprl_b200/libaprl_b200.so and fails
loudly when it is missing: there is no CPU fallback.  `bind()` declares the
ABI signatures on any library that exports them under a given prefix, and
`Run` drives one handle through the reference-shaped operator sequence.
"""
import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libaprl_b200.so")

_D = C.POINTER(C.c_double)
_U64 = C.POINTER(C.c_uint64)
_I32 = C.POINTER(C.c_int32)
_I64 = C.POINTER(C.c_int64)
_SZ = C.POINTER(C.c_size_t)

# name -> (restype, argtypes) with the handle type as `H`.
_H = object()
_SIGNATURES = {
    "last_error": (C.c_char_p, []),
    "magnet_prepare": (C.c_int, [C.POINTER(abi.Magnet)]),
    "cowan_coefficients": (C.c_int, [C.c_double, C.c_double, C.c_double, _D]),
    "runs_step": (C.c_int, [C.POINTER(C.c_void_p), C.c_size_t, C.c_uint32, C.POINTER(C.c_int)]),
    "boris_push": (C.c_int, [C.c_size_t, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D, C.c_double]),
    "run_destroy": (C.c_int, [_H]),
    "run_set_reference": (C.c_int, [_H, C.c_uint, _D, C.c_size_t]),
    "run_set_reference_planes": (C.c_int, [_H, C.c_uint, C.c_uint64, C.c_uint64, _D]),
    "run_set_field": (C.c_int, [_H, C.c_uint, _D, C.c_size_t]),
    "run_get_field": (C.c_int, [_H, C.c_uint, _D, C.c_size_t]),
    "run_history_length": (C.c_int, [_H, C.c_uint, _U64]),
    "run_set_history": (C.c_int, [_H, C.c_uint, _D, C.c_size_t]),
    "run_get_history": (C.c_int, [_H, C.c_uint, _D, C.c_size_t]),
    "run_set_particles": (C.c_int, [_H, C.c_size_t, _D, _D, _D, _D, _D, _D,
                                    _D, _D, _U64, C.c_int]),
    "run_particle_count": (C.c_int, [_H, _SZ]),
    "run_set_held": (C.c_int, [_H, C.c_size_t, C.POINTER(C.c_uint8), _D]),
    "run_get_held": (C.c_int, [_H, C.c_size_t, C.POINTER(C.c_uint8), _D, _SZ]),
    "run_get_particles": (C.c_int, [_H, C.c_size_t, _D, _D, _D, _D, _D, _D,
                                    _D, _D, _U64, _SZ]),
    "run_carrier_count": (C.c_int, [_H, _SZ]),
    "run_get_carriers": (C.c_int, [_H, C.c_size_t, _D, _D, _D, _D, _SZ]),
    "run_set_carriers": (C.c_int, [_H, C.c_size_t, _D, _D, _D, _D]),
    "run_advance_magnetic": (C.c_int, [_H]),
    "run_preview_electric": (C.c_int, [_H]),
    "run_coupling_trial": (C.c_int, [_H, _D]),
    "run_commit_electric": (C.c_int, [_H]),
    "run_shift": (C.c_int, [_H]),
    "run_step": (C.c_int, [_H, C.c_uint32]),
    "run_step_begin": (C.c_int, [_H]),
    "run_step_end": (C.c_int, [_H]),
    "run_get_stats": (C.c_int, [_H, C.POINTER(abi.StepStats)]),
    "run_tuning": (C.c_int, [_H, C.POINTER(abi.Tuning)]),
    "run_enable_energy_ledger": (C.c_int, [_H, C.c_int]),
    "run_energy_ledger": (C.c_int, [_H, C.POINTER(abi.EnergyLedger)]),
    "run_initialize_self_field": (C.c_int, [_H, C.POINTER(abi.SelfFieldConfig),
                                            C.POINTER(abi.SelfFieldReport)]),
    "run_get_slot_fields": (C.c_int, [_H, C.c_size_t, _D, _D, _D, _D, _SZ]),
    "run_sample_field_plane": (C.c_int, [_H, C.c_double, _D, C.c_size_t,
                                         C.POINTER(C.c_int)]),
}
_PRODUCT_ONLY = {
    "abi_version": (C.c_int, []),
    "run_synchronize": (C.c_int, [_H]),
    "run_profile_enable": (C.c_int, [_H, C.c_int]),
    "run_profile_read": (C.c_int, [_H, _D, _U64, C.c_uint, C.POINTER(C.c_uint)]),
    "kernel_name": (C.c_char_p, [C.c_uint]),
    "run_launch_count": (C.c_int, [_H, _U64]),
    "run_reset_iteration_stats": (C.c_int, [_H]),
    "run_sample_field_plane_noalloc": (C.c_int, [_H, C.c_double, _D, C.c_size_t,
                                                 C.POINTER(C.c_int)]),
    "run_sample_field_plane_async": (C.c_int, [_H, C.c_double, _D, C.c_size_t,
                                               C.POINTER(C.c_int)]),
    "run_gauss_law": (C.c_int, [_H, C.POINTER(abi.GaussLaw), _D, C.c_size_t]),
    "run_prepare_reference": (C.c_int, [_H, C.c_size_t, _D, _D, _D, _D, _D, _D, _D, _D,
                                        C.POINTER(abi.SelfFieldConfig),
                                        C.POINTER(abi.SelfFieldReport)]),
    "run_get_reference": (C.c_int, [_H, C.c_uint, _D, C.c_size_t]),
    "scan_footprint": (C.c_int, [C.POINTER(abi.RunConfig), C.c_size_t, _U64]),
    "scan_create": (C.c_int, [C.POINTER(abi.ScanConfig), C.POINTER(C.c_void_p)]),
    "scan_submit": (C.c_int, [C.c_void_p, C.POINTER(abi.ScanRequest), _U64]),
    "scan_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_double,
                            C.POINTER(abi.ScanResult)]),
    "scan_destroy": (C.c_int, [C.c_void_p]),
}


class AprlError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


class Binding:
    """The ABI functions of one library, keyed by their unprefixed names."""

    def __init__(self, lib, prefix, product):
        self.lib = lib
        self.prefix = prefix
        self.product = product
        self.fn = {}
        sigs = dict(_SIGNATURES)
        if product:
            sigs.update(_PRODUCT_ONLY)
        for name, (res, args) in sigs.items():
            f = getattr(lib, prefix + name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = [C.c_void_p if a is _H else a for a in args]
            self.fn[name] = f
        create = getattr(lib, prefix + "run_create")
        create.restype = C.c_int
        if product:
            create.argtypes = [C.POINTER(abi.RunConfig), C.c_void_p,
                               C.POINTER(C.c_void_p)]
        else:
            create.argtypes = [C.POINTER(abi.RunConfig), C.POINTER(C.c_void_p)]
        self.fn["run_create"] = create

    def error(self):
        msg = self.fn["last_error"]()
        return msg.decode() if msg else ""

    def check(self, status):
        if status != abi.APRL_OK:
            raise AprlError(status, self.error())

    def __call__(self, name, *args):
        self.check(self.fn[name](*args))


def bind(lib, prefix, product=False):
    return Binding(lib, prefix, product)


_PRODUCT = None


def load():
    """The product library; raises when it has not been built."""
    global _PRODUCT
    if _PRODUCT is None:
        if not os.path.exists(LIBRARY_PATH):
            raise ImportError(
                f"aprl_b200 CUDA library not built: {LIBRARY_PATH} is missing "
                "(run `python -m aprl_b200.build`); there is no CPU fallback")
        _PRODUCT = bind(C.CDLL(LIBRARY_PATH), "aprl_", product=True)
    return _PRODUCT


CHECKED_LIBRARY_PATH = os.path.join(_HERE, "libaprl_b200_checked.so")
_CHECKED = None


def load_checked():
    """The bounds-checked build of the library (every field, current and
    history index tested on the device; an index outside its array is a
    device error, never an access).  For tests; raises when not built."""
    global _CHECKED
    if _CHECKED is None:
        if not os.path.exists(CHECKED_LIBRARY_PATH):
            raise ImportError(f"bounds-checked library not built: {CHECKED_LIBRARY_PATH} "
                              "(run `python -m aprl_b200.build`)")
        _CHECKED = bind(C.CDLL(CHECKED_LIBRARY_PATH), "aprl_", product=True)
    return _CHECKED


def _ptr(array, ctype=C.c_double):
    return array.ctypes.data_as(C.POINTER(ctype))


class Run:
    """One aprl_run (or a checker's run) driven through the ABI."""

    def __init__(self, binding, config, stream=None):
        self.b = binding
        self.config = config
        handle = C.c_void_p()
        if binding.product:
            binding.check(binding.fn["run_create"](C.byref(config),
                                                   C.c_void_p(stream or 0),
                                                   C.byref(handle)))
        else:
            binding.check(binding.fn["run_create"](C.byref(config),
                                                   C.byref(handle)))
        self.handle = handle

    def close(self):
        if self.handle:
            self.b("run_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state ----------------------------------------------------------
    def set_reference(self, tables):
        for a, t in enumerate(tables):
            t = np.ascontiguousarray(t, dtype=np.float64)
            self.b("run_set_reference", self.handle, a, _ptr(t), t.size)

    def allocate_reference(self):
        """Zero-filled device table, to be streamed with set_reference_planes."""
        for a in range(6):
            n = int(np.prod(abi.reference_shape(self.config, a)))
            self.b("run_set_reference", self.handle, a, None, n)

    def set_reference_planes(self, component, first, planes):
        """planes: array (count, ny_c, nx_c) of native planes from `first`."""
        a = np.ascontiguousarray(planes, dtype=np.float64)
        self.b("run_set_reference_planes", self.handle, component, first,
               a.shape[0], _ptr(a))

    def set_field(self, component, array):
        a = np.ascontiguousarray(array, dtype=np.float64)
        self.b("run_set_field", self.handle, component, _ptr(a), a.size)

    def get_field(self, component):
        shape = abi.field_shape(self.config, component)
        out = np.empty(shape[::-1])
        self.b("run_get_field", self.handle, component, _ptr(out), out.size)
        return out

    def history_length(self, index):
        n = C.c_uint64()
        self.b("run_history_length", self.handle, index, C.byref(n))
        return n.value

    def get_history(self, index):
        out = np.empty(self.history_length(index))
        if out.size:
            self.b("run_get_history", self.handle, index, _ptr(out), out.size)
        return out

    def set_history(self, index, array):
        a = np.ascontiguousarray(array, dtype=np.float64)
        self.b("run_set_history", self.handle, index, _ptr(a), a.size)

    def set_particles(self, p, reset_carriers=True):
        cols = [np.ascontiguousarray(p[k], dtype=np.float64)
                for k in ("x", "y", "z", "ux", "uy", "uz", "charge", "mass")]
        ids = np.ascontiguousarray(p["id"], dtype=np.uint64)
        self.b("run_set_particles", self.handle, ids.size,
               *[_ptr(c) for c in cols], _ptr(ids, C.c_uint64),
               1 if reset_carriers else 0)

    def set_held(self, frozen, beta):
        """Frozen flags + held speeds for the current list, then the
        pending-queue extraction."""
        f = np.ascontiguousarray(frozen, dtype=np.uint8)
        b = np.ascontiguousarray(beta, dtype=np.float64)
        self.b("run_set_held", self.handle, f.size, _ptr(f, C.c_uint8), _ptr(b))

    def get_held(self):
        n = self.particle_count()
        f = np.empty(n, dtype=np.uint8)
        b = np.empty(n)
        count = C.c_size_t()
        self.b("run_get_held", self.handle, n, _ptr(f, C.c_uint8), _ptr(b), C.byref(count))
        return f, b

    def particle_count(self):
        n = C.c_size_t()
        self.b("run_particle_count", self.handle, C.byref(n))
        return n.value

    def get_particles(self):
        n = self.particle_count()
        out = {k: np.empty(n) for k in ("x", "y", "z", "ux", "uy", "uz",
                                        "charge", "mass")}
        out["id"] = np.empty(n, dtype=np.uint64)
        count = C.c_size_t()
        self.b("run_get_particles", self.handle, n,
               *[_ptr(out[k]) for k in ("x", "y", "z", "ux", "uy", "uz",
                                        "charge", "mass")],
               _ptr(out["id"], C.c_uint64), C.byref(count))
        return out

    def carrier_count(self):
        n = C.c_size_t()
        self.b("run_carrier_count", self.handle, C.byref(n))
        return n.value

    def get_carriers(self):
        n = self.carrier_count()
        out = {"position": np.empty((n, 3)), "velocity": np.empty((n, 3)),
               "charge": np.empty(n), "weight": np.empty(n)}
        count = C.c_size_t()
        self.b("run_get_carriers", self.handle, n, _ptr(out["position"]),
               _ptr(out["velocity"]), _ptr(out["charge"]),
               _ptr(out["weight"]), C.byref(count))
        return out

    def set_carriers(self, c):
        pos = np.ascontiguousarray(c["position"], dtype=np.float64)
        vel = np.ascontiguousarray(c["velocity"], dtype=np.float64)
        q = np.ascontiguousarray(c["charge"], dtype=np.float64)
        w = np.ascontiguousarray(c["weight"], dtype=np.float64)
        self.b("run_set_carriers", self.handle, q.size, _ptr(pos), _ptr(vel),
               _ptr(q), _ptr(w))

    def load_workload(self, workload):
        self.set_reference(workload.reference)
        for a, f in enumerate(workload.fields):
            self.set_field(a, f)
        self.set_particles(workload.particles)
        held = getattr(workload, "held", None)
        if held is not None:
            self.set_held(held, workload.particles["beta_held"])
        return self

    # -- operators ------------------------------------------------------
    def advance_magnetic(self):
        self.b("run_advance_magnetic", self.handle)

    def preview_electric(self):
        self.b("run_preview_electric", self.handle)

    def coupling_trial(self):
        res = (C.c_double * 4)()
        self.b("run_coupling_trial", self.handle, res)
        return list(res)

    def commit_electric(self):
        self.b("run_commit_electric", self.handle)

    def shift(self):
        self.b("run_shift", self.handle)

    def step(self, steps=1):
        self.b("run_step", self.handle, steps)

    def step_begin(self):
        """Queue one step's magnetic update, preview and first trials and
        return without waiting (aprl_run_step_begin)."""
        self.b("run_step_begin", self.handle)

    def step_end(self):
        """Finish the step begun by step_begin (aprl_run_step_end)."""
        self.b("run_step_end", self.handle)

    def tuning(self):
        t = abi.Tuning()
        self.b("run_tuning", self.handle, C.byref(t))
        return t.as_dict()

    def stats(self):
        s = abi.StepStats()
        self.b("run_get_stats", self.handle, C.byref(s))
        return s.as_dict()

    def enable_energy_ledger(self, enabled=True):
        self.b("run_enable_energy_ledger", self.handle, int(enabled))

    def initialize_self_field(self, config):
        """EBGaussFieldInitializer::initialize on the run's particles; returns
        the report as a dict (config: abi.SelfFieldConfig)."""
        out = abi.SelfFieldReport()
        self.b("run_initialize_self_field", self.handle, C.byref(config), C.byref(out))
        return out.as_dict()

    def energy_ledger(self):
        out = abi.EnergyLedger()
        self.b("run_energy_ledger", self.handle, C.byref(out))
        return out.as_dict()

    def prepare_reference(self, particles, config):
        """The inlet reference tables from the Cowan self-field of `particles`
        on the reference grid (aprl_run_prepare_reference)."""
        p = {k: np.ascontiguousarray(particles[k], dtype=np.float64)
             for k in ("x", "y", "z", "ux", "uy", "uz", "charge", "mass")}
        out = abi.SelfFieldReport()
        self.b("run_prepare_reference", self.handle, p["x"].size, _ptr(p["x"]), _ptr(p["y"]),
               _ptr(p["z"]), _ptr(p["ux"]), _ptr(p["uy"]), _ptr(p["uz"]), _ptr(p["charge"]),
               _ptr(p["mass"]), C.byref(config), C.byref(out))
        return out.as_dict()

    def get_reference(self, component):
        nx_c, ny_c, nz_c = abi.reference_shape(self.config, component)
        out = np.empty((nz_c, ny_c, nx_c))
        self.b("run_get_reference", self.handle, component, _ptr(out), out.size)
        return out

    def gauss_law(self, residual=False):
        """Summary dict, and with residual=True also G per node [k][j][i]."""
        cfg = self.config
        out = abi.GaussLaw()
        if residual:
            nodes = np.empty((cfg.nz + 1, cfg.ny + 1, cfg.nx + 1))
            self.b("run_gauss_law", self.handle, C.byref(out), _ptr(nodes), nodes.size)
            return out.as_dict(), nodes
        self.b("run_gauss_law", self.handle, C.byref(out), None, 0)
        return out.as_dict()

    def slot_fields(self):
        n = self.particle_count_slots()
        out = {k: np.empty((n, 3)) for k in ("used_e", "used_b", "next_e",
                                             "next_b")}
        count = C.c_size_t()
        self.b("run_get_slot_fields", self.handle, n, _ptr(out["used_e"]),
               _ptr(out["used_b"]), _ptr(out["next_e"]), _ptr(out["next_b"]),
               C.byref(count))
        return out

    def particle_count_slots(self):
        """Slots are sized by the particle list at the last preview; with all
        output pointers NULL the call only reports that count."""
        count = C.c_size_t()
        self.b("run_get_slot_fields", self.handle, 0, None, None, None, None,
               C.byref(count))
        return count.value

    def sample_field_plane(self, lab_z):
        cfg = self.config
        out = np.empty((cfg.ny, cfg.nx, 6))
        inside = C.c_int()
        self.b("run_sample_field_plane", self.handle, lab_z, _ptr(out),
               out.size, C.byref(inside))
        return out if inside.value else None

    # -- product-only ---------------------------------------------------
    def sample_field_plane_async(self, lab_z, out):
        """Queue the detector plane's copy into `out` (a C-contiguous
        (ny, nx, 6) float64 array, best page-locked) and return whether the
        plane is inside the window; `out` holds the values once the run's
        stream has passed the copy (synchronize(), or the next step)."""
        cfg = self.config
        if out.shape != (cfg.ny, cfg.nx, 6) or out.dtype != np.float64 or \
                not out.flags["C_CONTIGUOUS"]:
            raise ValueError("detector buffer must be a C-contiguous (ny, nx, 6) float64 array")
        inside = C.c_int()
        self.b("run_sample_field_plane_async", self.handle, lab_z, _ptr(out),
               out.size, C.byref(inside))
        return bool(inside.value)

    def synchronize(self):
        self.b("run_synchronize", self.handle)

    def profile_enable(self, enabled=True):
        self.b("run_profile_enable", self.handle, 1 if enabled else 0)

    def profile_read(self):
        cap = 64
        ms = (C.c_double * cap)()
        launches = (C.c_uint64 * cap)()
        n = C.c_uint()
        self.b("run_profile_read", self.handle, ms, launches, cap, C.byref(n))
        names = [self.b.fn["kernel_name"](i).decode() for i in range(n.value)]
        return {names[i]: (ms[i], launches[i]) for i in range(n.value)
                if launches[i]}

    def launch_count(self):
        n = C.c_uint64()
        self.b("run_launch_count", self.handle, C.byref(n))
        return n.value


class Scan:
    """A parameter-scan server (aprl_scan_*): independent runs admitted by
    device footprint into `slots` concurrent streams of one GPU."""

    def __init__(self, binding, budget_bytes=0, slots=4, runs_per_slot=1):
        self.b = binding
        cfg = abi.ScanConfig(int(budget_bytes), int(slots), int(runs_per_slot))
        handle = C.c_void_p()
        binding("scan_create", C.byref(cfg), C.byref(handle))
        self.handle = handle
        self._inputs = {}

    def footprint(self, config, particles):
        out = C.c_uint64()
        self.b("scan_footprint", C.byref(config), particles, C.byref(out))
        return out.value

    def submit(self, config, particles, steps, reference=None, held=None,
               detector_lab_z=None):
        """Queue one run; the arrays stay referenced until wait() returns it."""
        keep = {}

        def arr(a, dtype=np.float64):
            a = np.ascontiguousarray(a, dtype=dtype)
            keep[len(keep)] = a
            return a

        q = abi.ScanRequest()
        q.config = config
        q.steps = int(steps)
        n = int(np.asarray(particles["x"]).size)
        q.particles = n
        for name in ("x", "y", "z", "ux", "uy", "uz", "charge", "mass"):
            setattr(q, name, _ptr(arr(particles[name])))
        q.id = _ptr(arr(particles["id"], np.uint64), C.c_uint64)
        if held is not None:
            q.frozen = _ptr(arr(held[0], np.uint8), C.c_uint8)
            q.frozen_beta_z = _ptr(arr(held[1]))
        if reference is not None:
            for a in range(6):
                q.reference[a] = _ptr(arr(reference[a]))
        detector = None
        if detector_lab_z is not None:
            detector = arr(np.full(6 * config.nx * config.ny, np.nan))
            q.detector_lab_z = float(detector_lab_z)
            q.detector = _ptr(detector)
        ticket = C.c_uint64()
        self.b("scan_submit", self.handle, C.byref(q), C.byref(ticket))
        self._inputs[ticket.value] = (keep, detector)
        return ticket.value

    def wait(self, ticket, timeout=3600.0):
        """The request's result as a dict (state, status, times, stats,
        detector) once done, or its state when the timeout expired first."""
        res = abi.ScanResult()
        self.b("scan_wait", self.handle, ticket, float(timeout), C.byref(res))
        out = {name: getattr(res, name) for name, _ in abi.ScanResult._fields_
               if name not in ("stats", "message")}
        out["message"] = res.message.decode(errors="replace")
        if res.state == abi.SCAN_DONE:
            out["stats"] = res.stats.as_dict()
            _, detector = self._inputs.pop(ticket)
            out["detector"] = detector if res.detector_inside else None
        return out

    def close(self):
        if self.handle:
            self.b("scan_destroy", self.handle)
            self.handle = None
            self._inputs.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
