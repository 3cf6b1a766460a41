"""ctypes binding of the C ABI declared in include/pkde_b200.h.

The shared library is built in-tree (``parallelkde.jl_b200/lib/libpkde_b200.so``) by
``parallelkde.jl_b200/build.py``.  There is no CPU fallback: if the library or a CUDA
device is missing, every compute call raises.
"""
import ctypes
import math
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libpkde_b200.so")

PKDE_OK, PKDE_EINVAL, PKDE_ENOMEM, PKDE_ECUDA, PKDE_EUNSUPPORTED = 0, 1, 2, 3, 4
PKDE_DEVICE_INPUT = 1
PKDE_DEVICE_OUTPUT = 2

# every symbol include/pkde_b200.h declares
EXPORTED = [
    "pkde_create", "pkde_destroy", "pkde_last_error", "pkde_version",
    "pkde_gradepro_default_params", "pkde_gradepro_estimate", "pkde_gradepro_estimate_batch", "pkde_dirac_sequence",
    "pkde_dirac_sequence_noalloc",
    "pkde_fft", "pkde_scaled_vmr", "pkde_identify_convergence", "pkde_set_profiling", "pkde_get_stats",
    "pkde_set_step_path", "pkde_rot_estimate", "pkde_serve_config", "pkde_submit", "pkde_wait",
    "pkde_find_grid", "pkde_normalize_density", "pkde_set_autotune",
    "pkde_boot_index", "pkde_set_wait_limit", "pkde_set_fault", "pkde_diag_divide",
]

PHASES = ["binning", "forward_fft", "step_fft", "step_vmr", "step_means", "other"]


class PkdeStats(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_uint64), ("phase_launches", ctypes.c_uint64 * 6),
                ("phase_ms", ctypes.c_double * 6)]


class PkdeGrid(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("dims", ctypes.c_int64 * 4), ("lo", ctypes.c_double * 4),
                ("hi", ctypes.c_double * 4), ("h", ctypes.c_double * 4)]


class PkdeGradeproParams(ctypes.Structure):
    _fields_ = [("grid", PkdeGrid), ("n_bootstraps", ctypes.c_int32), ("n_steps", ctypes.c_int32),
                ("bw_step", ctypes.c_double), ("bw_final", ctypes.c_double * 4),
                ("alpha_s", ctypes.c_double), ("alpha_os", ctypes.c_double), ("eps", ctypes.c_double)]


class ArgumentError(ValueError):
    """Raised where the reference throws ArgumentError."""


class CudaLibraryError(RuntimeError):
    pass


_lib = None
_lock = threading.Lock()
_ctx = {}


def load():
    """Load the shared library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CudaLibraryError(f"CUDA library not built: {LIB_PATH} is missing (run parallelkde.jl_b200/build.py)")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i32, i64, u32, u64, dbl = (ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32,
                                   ctypes.c_uint64, ctypes.c_double)
    lib.pkde_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int]
    lib.pkde_destroy.argtypes = [vp]
    lib.pkde_last_error.argtypes = [vp]
    lib.pkde_last_error.restype = ctypes.c_char_p
    lib.pkde_version.restype = ctypes.c_char_p
    lib.pkde_gradepro_default_params.argtypes = [ctypes.POINTER(PkdeGradeproParams), i32]
    lib.pkde_gradepro_estimate.argtypes = [vp, ctypes.POINTER(PkdeGradeproParams), vp, i64, vp, u64, vp, vp, u32, vp]
    lib.pkde_gradepro_estimate_batch.argtypes = [vp, i32, ctypes.POINTER(PkdeGradeproParams), vp, vp, vp, vp, vp,
                                                 vp, u32, vp]
    lib.pkde_dirac_sequence.argtypes = [vp, ctypes.POINTER(PkdeGrid), vp, i64, vp, i32, u64, vp, vp, vp, u32, vp]
    lib.pkde_dirac_sequence_noalloc.argtypes = [vp, ctypes.POINTER(PkdeGrid), vp, i64, vp, i32, u64, vp, vp, vp,
                                                vp]
    lib.pkde_fft.argtypes = [vp, i32, vp, vp, i32, i32, u32, vp]
    lib.pkde_scaled_vmr.argtypes = [vp, i64, i32, vp, vp, i32, vp, vp, i64, vp, u32, vp]
    lib.pkde_identify_convergence.argtypes = [vp, i64, vp, vp, vp, vp, vp, dbl, dbl, i64, i64, vp, vp, vp, vp, u32, vp]
    lib.pkde_set_profiling.argtypes = [vp, ctypes.c_int]
    lib.pkde_set_step_path.argtypes = [vp, ctypes.c_int]
    lib.pkde_set_autotune.argtypes = [vp, ctypes.c_int]
    lib.pkde_find_grid.argtypes = [vp, i32, vp, i64, vp, vp, vp, ctypes.POINTER(PkdeGrid), u32, vp]
    lib.pkde_normalize_density.argtypes = [vp, vp, i64, dbl, u32, vp]
    lib.pkde_rot_estimate.argtypes = [vp, ctypes.POINTER(PkdeGrid), i32, vp, i64, vp, u32, vp]
    lib.pkde_get_stats.argtypes = [vp, ctypes.POINTER(PkdeStats), ctypes.c_int]
    lib.pkde_set_wait_limit.argtypes = [vp, i64]
    lib.pkde_set_fault.argtypes = [vp, i32]
    lib.pkde_diag_divide.argtypes = [vp, vp, vp, vp, i64, u32, vp]
    lib.pkde_boot_index.argtypes = [u64, i64, i64, i64]
    lib.pkde_boot_index.restype = i64
    for name in EXPORTED:
        getattr(lib, name).restype = getattr(lib, name).restype or ctypes.c_int
    _lib = lib
    return lib


def context(device=0):
    """Per-device context (created on first use, kept until exit)."""
    lib = load()
    with _lock:
        if device not in _ctx:
            h = ctypes.c_void_p()
            rc = lib.pkde_create(ctypes.byref(h), int(device))
            if rc != PKDE_OK:
                raise CudaLibraryError(f"pkde_create(device={device}) failed with status {rc} (no usable CUDA device?)")
            _ctx[device] = h
        return _ctx[device]


def check(rc, ctx):
    if rc == PKDE_OK:
        return
    msg = load().pkde_last_error(ctx).decode(errors="replace")
    if rc == PKDE_EINVAL:
        raise ArgumentError(msg)
    raise CudaLibraryError(f"status {rc}: {msg}")


def make_grid_struct(lo, hi, h, dims):
    g = PkdeGrid()
    g.ndim = len(dims)
    for j in range(len(dims)):
        g.dims[j] = int(dims[j])
        g.lo[j] = float(lo[j])
        g.hi[j] = float(hi[j])
        g.h[j] = float(h[j])
    return g


def make_params(grid_struct, n_bootstraps=100, n_steps=None, bw_step=None, bw_final=None, alpha_s=None,
                alpha_os=None, eps=None):
    p = PkdeGradeproParams()
    load().pkde_gradepro_default_params(ctypes.byref(p), grid_struct.ndim)
    p.grid = grid_struct
    p.n_bootstraps = int(n_bootstraps)
    p.n_steps = int(n_steps) if n_steps is not None else 0
    nan = math.nan
    p.bw_step = float(bw_step) if bw_step is not None else nan
    if bw_final is None:
        vals = [nan] * 4
    elif np.isscalar(bw_final):
        vals = [float(bw_final)] * grid_struct.ndim + [nan] * (4 - grid_struct.ndim)
    else:
        vals = [float(v) for v in bw_final] + [nan] * (4 - len(bw_final))
    for j in range(4):
        p.bw_final[j] = vals[j]
    p.alpha_s = float(alpha_s) if alpha_s is not None else nan
    p.alpha_os = float(alpha_os) if alpha_os is not None else nan
    p.eps = float(eps) if eps is not None else nan
    return p


PKDE_PROFILE_OFF, PKDE_PROFILE_ALL, PKDE_PROFILE_STEPS = 0, 1, 2


def set_profiling(enable, device=0):
    """True / PKDE_PROFILE_ALL: time every launch per phase; PKDE_PROFILE_STEPS: only
    the bandwidth-step phases; False / PKDE_PROFILE_OFF: launch counts only."""
    ctx = context(device)
    check(load().pkde_set_profiling(ctx, int(enable)), ctx)


PKDE_STEPS_AUTO, PKDE_STEPS_PER_STEP_LAUNCH = 0, 1


def set_step_path(path, device=0):
    """PKDE_STEPS_AUTO (default) or PKDE_STEPS_PER_STEP_LAUNCH (the plain form)."""
    ctx = context(device)
    check(load().pkde_set_step_path(ctx, int(path)), ctx)


def set_autotune(enable, device=0):
    """Per-shape autotuning of the step engine's schedule (on by default)."""
    ctx = context(device)
    check(load().pkde_set_autotune(ctx, int(bool(enable))), ctx)


DEFAULT_WAIT_LIMIT = 20_000_000


def set_wait_limit(polls, device=0):
    """Polls a step-engine dependency wait makes before the launch gives up (default
    20,000,000, about 1-2 s); the call then fails with 'a dependency wait timed out'."""
    ctx = context(device)
    check(load().pkde_set_wait_limit(ctx, int(polls)), ctx)


PKDE_FAULT_NONE, PKDE_FAULT_AFTER_BINNING = 0, 1


def set_fault(point, device=0):
    """Arm a one-shot host-side fault at `point` (tests of the error paths)."""
    ctx = context(device)
    check(load().pkde_set_fault(ctx, int(point)), ctx)


def diag_divide(num, den, device=0):
    """num / den (float64 arrays) with the quotient the step engine uses."""
    num = np.ascontiguousarray(num, dtype=np.float64)
    den = np.ascontiguousarray(den, dtype=np.float64)
    if num.shape != den.shape:
        raise ValueError("num and den must have the same shape")
    out = np.empty_like(num)
    ctx = context(device)
    check(load().pkde_diag_divide(ctx, num.ctypes.data, den.ctypes.data, out.ctypes.data, num.size, 0, None), ctx)
    return out


def get_stats(device=0, reset=False):
    """Kernel launches and per-phase device milliseconds since the last reset."""
    st = PkdeStats()
    rc = load().pkde_get_stats(context(device), ctypes.byref(st), int(bool(reset)))
    if rc != PKDE_OK:
        raise CudaLibraryError(f"pkde_get_stats failed with status {rc}")
    return dict(launches=int(st.launches),
                phase_launches={p: int(st.phase_launches[i]) for i, p in enumerate(PHASES)},
                phase_ms={p: float(st.phase_ms[i]) for i, p in enumerate(PHASES)})


def ptr(a):
    """Address of a numpy array or a CUDA torch tensor."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()
