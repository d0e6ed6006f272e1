"""Loaders for the CPU checkers under oracle/ (test infrastructure only).

The plain-C oracle (oracle/libpic_oracle.so) and, where it was built, the
reference's own translation units (oracle/_ref/libaprl_ref.so) export the
same ABI as the product under the prefixes `oracle_` and `ref_`.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

from aprl_b200 import abi, native  # noqa: E402

ORACLE_PATH = os.path.join(REPO, "oracle", "libpic_oracle.so")
REFERENCE_PATH = os.path.join(REPO, "oracle", "_ref", "libaprl_ref.so")

_oracle = None
_reference = None


def oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_PATH):
            subprocess.check_call([sys.executable,
                                   os.path.join(REPO, "oracle", "build_oracle.py")])
        lib = C.CDLL(ORACLE_PATH)
        _oracle = native.bind(lib, "oracle_")
        f = lib.oracle_shape_weights
        f.restype = C.c_long
        f.argtypes = [C.POINTER(abi.RunConfig), C.POINTER(C.c_double),
                      C.POINTER(C.c_double), C.POINTER(C.c_double),
                      C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                      C.POINTER(C.c_double), C.c_long]
        f = lib.oracle_momentum
        f.restype = C.c_int
        f.argtypes = [C.POINTER(C.c_double)] * 3 + [C.c_double] * 4
        f = lib.oracle_gamma
        f.restype = C.c_double
        f.argtypes = [C.POINTER(C.c_double)]
    return _oracle


def reference_available():
    return os.path.exists(REFERENCE_PATH)


def reference():
    global _reference
    if _reference is None:
        lib = C.CDLL(REFERENCE_PATH)
        _reference = native.bind(lib, "ref_")
        f = lib.ref_shape_weights
        f.restype = C.c_long
        f.argtypes = [C.POINTER(abi.RunConfig), C.POINTER(C.c_double),
                      C.POINTER(C.c_double), C.POINTER(C.c_double),
                      C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                      C.POINTER(C.c_double), C.c_long]
        f = lib.ref_momentum
        f.restype = C.c_int
        f.argtypes = [C.POINTER(C.c_double)] * 3 + [C.c_double] * 4
        f = lib.ref_gamma
        f.restype = C.c_double
        f.argtypes = [C.POINTER(C.c_double)]
        f = lib.ref_set_threads
        f.restype = C.c_int
        f.argtypes = [C.c_uint]
        f = lib.ref_blocked_reference
        f.restype = C.c_int
        f.argtypes = [C.POINTER(abi.RunConfig), C.c_size_t] + [C.POINTER(C.c_double)] * 4 + \
            [C.c_double, C.POINTER(C.c_uint64), C.c_uint64, C.c_int, C.c_int, C.c_char_p,
             C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_double)]
        f = lib.ref_surface_current_pin
        f.restype = C.c_int
        f.argtypes = [C.POINTER(abi.RunConfig), C.c_size_t] + [C.POINTER(C.c_double)] * 4 + \
            [C.c_double, C.c_uint64, C.c_char_p, C.POINTER(C.c_double),
             C.POINTER(C.c_double), C.c_size_t, C.POINTER(C.c_size_t)]
    return _reference


def surface_current_pin(cfg, particles, beta, directory):
    """The equivalent surface current per reference plane and point from the
    reference's own TransverseReferenceCurrent::prepare over its own
    BlockedCowanReference, and from the harness's writer fed that
    reference's Bx, By tables: (from_reference, from_tables), each
    [plane][point]."""
    lib = reference()
    cols = [np.ascontiguousarray(particles[k], dtype=np.float64) for k in ("x", "y", "z", "charge")]
    capacity = (cfg.reference_nz + 1) * 2 * (cfg.nx + cfg.ny + 2)
    a = np.zeros(capacity)
    b = np.zeros(capacity)
    count = C.c_size_t()
    lib.check(lib.lib.ref_surface_current_pin(
        C.byref(cfg), len(cols[0]), *[c.ctypes.data_as(C.POINTER(C.c_double)) for c in cols],
        float(beta), 8, directory.encode(), a.ctypes.data_as(C.POINTER(C.c_double)),
        b.ctypes.data_as(C.POINTER(C.c_double)), capacity, C.byref(count)))
    n = cfg.reference_nz * count.value
    return a[:n].reshape(cfg.reference_nz, -1), b[:n].reshape(cfg.reference_nz, -1)


def blocked_reference(cfg, particles, beta, guards, block_layers, shaped, directory,
                      open_transverse=False):
    """The reference's own BlockedCowanReference (built over the FFTW
    stand-in) on cfg's reference grid: the six native tables and its report
    (source charge, deposited charge, minimum pivot, minimum mode
    eigenvalue, open-wall interpolation error, open-wall fallback tiles).
    shaped: deposit with the run's own shape instead of CIC;
    open_transverse: the open-transverse-wall variant."""
    lib = reference()
    n = len(particles["x"])
    cols = [np.ascontiguousarray(particles[k], dtype=np.float64) for k in ("x", "y", "z", "charge")]
    tables = [np.zeros(abi.reference_shape(cfg, a)[::-1]) for a in range(6)]
    ptrs = (C.POINTER(C.c_double) * 6)(*[t.ctypes.data_as(C.POINTER(C.c_double)) for t in tables])
    g = (C.c_uint64 * 3)(*guards)
    report = (C.c_double * 6)()
    lib.check(lib.lib.ref_blocked_reference(
        C.byref(cfg), n, *[c.ctypes.data_as(C.POINTER(C.c_double)) for c in cols],
        float(beta), g, int(block_layers), 1 if shaped else 0, 1 if open_transverse else 0,
        directory.encode(), ptrs, report))
    return tables, list(report)


def shape_weights(binding, config, origin, begin, end, capacity=8192):
    axis = np.empty(capacity, dtype=np.int32)
    index = np.empty((capacity, 3), dtype=np.int64)
    weight = np.empty(capacity)
    f = getattr(binding.lib, binding.prefix + "shape_weights")
    d = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))
    n = f(C.byref(config), d(origin), d(begin), d(end),
          axis.ctypes.data_as(C.POINTER(C.c_int32)),
          index.ctypes.data_as(C.POINTER(C.c_int64)),
          weight.ctypes.data_as(C.POINTER(C.c_double)), capacity)
    if n < 0:
        raise native.AprlError(abi.APRL_ERR_RUNTIME, binding.error())
    return axis[:n], index[:n], weight[:n]


def run(binding, workload):
    return native.Run(binding, workload.config).load_workload(workload)


def state(run_handle, histories=True):
    """Everything observable after a step, as numpy arrays."""
    out = {"fields": [run_handle.get_field(a) for a in range(6)],
           "particles": run_handle.get_particles(),
           "carriers": run_handle.get_carriers(),
           "stats": run_handle.stats()}
    if histories:
        out["histories"] = [run_handle.get_history(h) for h in range(12)]
    return out


def max_relative(a, b):
    """max |a-b| / max |b| (0 when both vanish)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.shape != b.shape:
        raise AssertionError(f"shape mismatch {a.shape} vs {b.shape}")
    if a.size == 0:
        return 0.0
    scale = np.max(np.abs(b))
    diff = np.max(np.abs(a - b))
    if scale == 0.0:
        return float(diff)
    return float(diff / scale)


# ---------------------------------------------------------------------------
# Node charge density and the discrete Gauss law (numpy restatements).
def _f3_node(f):
    return np.stack([0.25 * (1.0 - f), 0.5 - 0.25 * f, 0.25 + 0.25 * f, 0.25 * f])


def _quintic_node(f):
    """The quintic-compensated node basis (longitudinal_shape.h:48-54) for
    cell-relative offsets f: 12 weights per particle, nodes cell-5 .. cell+6."""
    n = np.zeros((6, f.size))
    n[0] = 1.0
    for j in range(1, 6):
        saved = np.zeros(f.size)
        for k in range(j):
            t = n[k] / j
            n[k] = saved + (k + 1 - f) * t
            saved = (f + j - k - 1) * t
        n[j] = saved
    p = 5.0
    a = p / 6.0
    b = 3 * p / 40.0 + p * (p - 1) / 72.0
    d = 5 * p / 112.0 + p * (p - 1) / 80.0 + p * (p - 1) * (p - 2) / 1296.0
    c = [-d / 64.0, b / 16.0 + 3 * d / 32.0, -a / 4.0 - b / 4.0 - 15 * d / 64.0,
         1 + a / 2.0 + 3 * b / 8.0 + 5 * d / 16.0, -a / 4.0 - b / 4.0 - 15 * d / 64.0,
         b / 16.0 + 3 * d / 32.0, -d / 64.0]
    v = np.zeros((12, f.size))
    for j in range(6):
        for k in range(7):
            v[j + k] += n[j] * c[k]
    return v


def charge_density(cfg, origin, p, pad=6):
    """The node charge density the run's current conserves, [k][j][i] with
    `pad` extra nodes on every side (index pad is node 0): for
    linear-binomial3 F3 in x, linear in y, binomial3 in z
    (verification/transverse_binomial_checks.cpp:12-66); for
    quintic-compensated linear in x and y and the quintic node basis in z."""
    if cfg.shape == 0:
        return _binomial3_density(cfg, origin, p, pad)
    rho = np.zeros((cfg.nz + 1 + 2 * pad, cfg.ny + 1 + 2 * pad, cfg.nx + 1 + 2 * pad))
    x = (p["x"] - origin[0]) / cfg.dx
    y = (p["y"] - origin[1]) / cfg.dy
    z = (p["z"] - origin[2]) / cfg.dz
    i = np.floor(x).astype(int)
    j = np.floor(y).astype(int)
    k = np.floor(z).astype(int)
    fx, fy = x - i, y - j
    wz = _quintic_node(z - k)
    q = p["charge"] / (cfg.dx * cfg.dy * cfg.dz)
    for u in range(2):
        wx = fx if u else 1.0 - fx
        for v in range(2):
            wy = fy if v else 1.0 - fy
            for t in range(12):
                np.add.at(rho, (k - 5 + t + pad, j + v + pad, i + u + pad),
                          q * wx * wy * wz[t])
    return rho, pad


def _binomial3_density(cfg, origin, p, pad):
    rho = np.zeros((cfg.nz + 1 + 2 * pad, cfg.ny + 1 + 2 * pad, cfg.nx + 1 + 2 * pad))
    x = (p["x"] - origin[0]) / cfg.dx
    y = (p["y"] - origin[1]) / cfg.dy
    z = (p["z"] - origin[2]) / cfg.dz
    i = np.floor(x).astype(int)
    j = np.floor(y).astype(int)
    k = np.floor(z).astype(int)
    wx = _f3_node(x - i)            # nodes i-1 .. i+2
    fy = y - j
    fz = z - k
    wz = np.zeros((4, x.size))      # binomial3 over nodes k-1 .. k+2
    for s, w in zip((-1, 0, 1), (0.25, 0.5, 0.25)):
        wz[s + 1] += w * (1.0 - fz)
        wz[s + 2] += w * fz
    q = p["charge"] / (cfg.dx * cfg.dy * cfg.dz)
    for u in range(4):
        for v in range(2):
            wy = fy if v else 1.0 - fy
            for t in range(4):
                np.add.at(rho, (k - 1 + t + pad, j + v + pad, i - 1 + u + pad),
                          q * wx[u] * wy * wz[t])
    return rho, pad


def gauss_residual(cfg, origin, p, ex, ey, ez):
    """eps0 div E - rho at every node [k][j][i]; edges outside the grid are
    zero (ex, ey, ez in the [k][j][i] arrays of get_field)."""
    eps0 = 8.8541878128e-12
    rho, pad = charge_density(cfg, origin, p)
    rho = rho[pad:-pad, pad:-pad, pad:-pad]
    shape = rho.shape
    dx = np.zeros(shape)
    dx[:, :, :-1] += ex
    dx[:, :, 1:] -= ex
    dy = np.zeros(shape)
    dy[:, :-1, :] += ey
    dy[:, 1:, :] -= ey
    dz = np.zeros(shape)
    dz[:-1, :, :] += ez
    dz[1:, :, :] -= ez
    div = dx / cfg.dx + dy / cfg.dy + dz / cfg.dz
    return eps0 * div - rho, rho
