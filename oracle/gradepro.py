"""TEST INFRASTRUCTURE ONLY: FP64 CPU restatement of ParallelKDE.jl's ``:gradepro`` path.

This module is the oracle.  Only ``tests/``, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline leg may import it; the product path (the CUDA library and its host mirror)
never does.  It restates the reference's ``device=:cpu, method=:serial`` Float64 path line
by line (citations are ``file:line`` within the reference project):

* grid      : src/Grids/Grids.jl:217 (t0 = h/2), :225-231 (fftgrid), :252-300 (find_grid)
* binning   : src/StatisticsPropagation/DirectSpace.jl:97-145, 196-242, 479-498
              (C restatement in ``binning.c``; ``dirac_numpy`` below is the same
              arithmetic in NumPy for small cases and cross-checks the C code)
* forward   : src/StatisticsPropagation/FourierSpace.jl:25-52 (unnormalised forward FFT)
* propagate : src/StatisticsPropagation/FourierSpace.jl:215-262
* inverse   : src/StatisticsPropagation/FourierSpace.jl:445-472 (ifft, scaled by 1/G)
* VMR       : src/StatisticsPropagation/DirectSpace.jl:526-584
* means     : src/StatisticsPropagation/DirectSpace.jl:747-764
* converge  : src/StatisticsPropagation/DirectSpace.jl:829-871, 975-1031, 1092-1100
* ladder    : src/DensityEstimators/GradeProEstimator.jl:740-796, 860-905, 954-966,
              1074-1089;  silverman_rule DirectSpace.jl:1102-1111
* main loop : src/DensityEstimators/GradeProEstimator.jl:968-1060 (incl. replace_nans!)
* :rot      : src/DensityEstimators/RoTEstimator.jl:24-49 (rule-of-thumb times),
              :55-75 (time = rule - h/2), :143-148, 159-172, 177-201, 203-265
              (identity binning, FFT, one propagation, inverse FFT, |.|)

Layout: the reference is column-major with grid axis 1 fastest.  Arrays here are
C-ordered with shape (n_N, ..., n_1) [bootstrap axis first when present], so the flat
index is the reference's linear index.  FFTs use scipy.fft (pocketfft) in FP64; FFTW
itself is not available, so FFT rounding is matched only to FP64 accuracy.

Deliberate difference: the reference's VMR scale uses ``n_samples^3`` in Int64, which
wraps for n >= 2^21 (a constant offset in log space that cancels in every difference
the convergence test takes, and that makes the reference throw for some n).  The
oracle uses the exact n^3 in FP64.

Added output (not in the reference): ``selected_step`` per grid point = the last
0-based step s at which ``density := means`` happened (``more_stable`` in
find_stability, DirectSpace.jl:1024-1030), or S (number of steps) when the point was
filled by replace_nans! from the final step's means.
"""
import ctypes
import math
import os
from dataclasses import dataclass, field
from fractions import Fraction

import numpy as np
import scipy.fft as sfft

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            build_oracle()
        lib = ctypes.CDLL(path)
        for fn in (lib.oracle_dirac, lib.oracle_dirac_ext):
            fn.restype = ctypes.c_int
            fn.argtypes = [
                ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        _LIB = lib
    return _LIB


def build_oracle():
    """Compile binning.c into oracle/_build/liboracle.so (IEEE semantics, no FMA)."""
    import subprocess
    out = os.path.join(_HERE, "_build")
    os.makedirs(out, exist_ok=True)
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
           "-o", os.path.join(out, "liboracle.so"), os.path.join(_HERE, "binning.c"), "-lm"]
    subprocess.check_call(cmd)


# --------------------------------------------------------------------------- grids
@dataclass
class Grid:
    """Uniform grid: per axis low bound, high bound, spacing and point count."""
    lo: np.ndarray
    hi: np.ndarray
    h: np.ndarray
    dims: tuple

    @property
    def ndim(self):
        return len(self.dims)

    @property
    def size(self):
        return int(np.prod(self.dims))

    @property
    def shape_c(self):
        """C-order array shape (n_N, ..., n_1)."""
        return tuple(reversed(self.dims))


def range_step(lo, hi, n):
    """Step of Julia's ``range(lo, stop=hi, length=n)``: the exact quotient
    (hi - lo)/(n - 1) rounded once to FP64 (Julia carries the step in TwicePrecision)."""
    return float((Fraction(hi) - Fraction(lo)) / (n - 1))


def grid_from_ranges(ranges):
    """ranges: sequence of (lo, hi, n) per axis (like ``range(lo, hi, length=n)``)."""
    lo = np.array([float(r[0]) for r in ranges])
    hi = np.array([float(r[1]) for r in ranges])
    dims = tuple(int(r[2]) for r in ranges)
    h = np.array([range_step(a, b, n) for a, b, n in zip(lo, hi, dims)])
    return Grid(lo, hi, h, dims)


def grid_from_steps(ranges):
    """ranges: sequence of (lo, step, hi) like Julia's ``lo:step:hi`` literal ranges."""
    lo = np.array([float(r[0]) for r in ranges])
    h = np.array([float(r[1]) for r in ranges])
    dims = tuple(int(math.floor((float(r[2]) - float(r[0])) / float(r[1]) + 1e-9)) + 1 for r in ranges)
    hi = np.array([float(r[2]) for r in ranges])
    return Grid(lo, hi, h, dims)


def find_grid(data, grid_bounds=None, grid_dims=None, grid_steps=None, grid_padding=None):
    """Grids.jl:252-300.  data: (N, n) array."""
    data = np.asarray(data, dtype=np.float64)
    ndim = data.shape[0]
    if grid_bounds is None:
        grid_bounds = [(float(row.min()), float(row.max())) for row in data]
    if grid_padding is None:
        grid_padding = [0.1 * abs(b[1] - b[0]) for b in grid_bounds]
    grid_bounds = [(b[0] - p, b[1] + p) for b, p in zip(grid_bounds, grid_padding)]
    if grid_steps is None and grid_dims is None:
        grid_dims = tuple(150 for _ in range(ndim))
    if grid_dims is not None:
        return grid_from_ranges([(b[0], b[1], n) for b, n in zip(grid_bounds, grid_dims)])
    ranges = []
    for b, s in zip(grid_bounds, grid_steps):
        n = int(math.floor((b[1] - b[0]) / s)) + 1
        ranges.append((b[0], s, b[0] + (n - 1) * s))
    lo = np.array([r[0] for r in ranges])
    h = np.array([float(r[1]) for r in ranges])
    hi = np.array([r[2] for r in ranges])
    return Grid(lo, hi, h, tuple(int(round((r[2] - r[0]) / r[1])) + 1 for r in ranges))


def initial_bandwidth(grid):
    """Grids.jl:217."""
    return grid.h / 2


def fftgrid_axes(grid):
    """Grids.jl:225-231: per axis 2pi * fftfreq(n, 1/h), i.e. m * (2pi * ((1/h)/n))."""
    ks = []
    for n, h in zip(grid.dims, grid.h):
        mult = (2 * math.pi) * ((1.0 / h) / n)
        m = np.arange(n, dtype=np.float64)
        nneg = (n - 1) // 2 + 1
        m[nneg:] -= n
        ks.append(m * mult)
    return ks


# ------------------------------------------------------------------------ bandwidths
def silverman_rule(data):
    """DirectSpace.jl:1102-1111."""
    data = np.asarray(data, dtype=np.float64)
    ndim, n = data.shape
    stds = np.sqrt(np.var(data, axis=1, ddof=1))
    prefactor = (4 / ((ndim + 2) * n)) ** (1 / (ndim + 4))
    return prefactor * stds


def get_time(time_final, n_steps=None, time_step=None):
    """GradeProEstimator.jl:860-905 (CPU).  Returns (times (S, N), dt (N,))."""
    time_final = np.asarray(time_final, dtype=np.float64)
    if n_steps is not None:
        dt = time_final / n_steps
        times = np.stack([dt * i for i in range(0, n_steps + 1)])
        return times, dt
    if time_step is not None:
        ts = np.full(time_final.shape, float(time_step)) if np.isscalar(time_step) \
            else np.asarray(time_step, dtype=np.float64)
        if np.any(ts > time_final) or np.any(ts <= 0):
            raise ValueError("Invalid time step")
        n_steps = int(np.min(np.floor(time_final / ts)))
        times = np.stack([ts * i for i in range(0, n_steps + 1)])
        return times, ts
    return get_time(time_final, n_steps=250)


def _julia_round(x):
    """round(Int, x) with ties to even (Julia RoundNearest)."""
    return int(round(x))


def calculate_duration_steps(time_max, dt, alpha_s=0.0, alpha_os=0.1):
    """GradeProEstimator.jl:954-966."""
    if alpha_s < 0 or alpha_s > 1 or alpha_os < 0 or alpha_os > 1:
        raise ValueError("Fraction must be in the range [0, 1]")
    n_steps = np.asarray(time_max) / np.asarray(dt)
    buf = alpha_s * n_steps
    stop = alpha_os * n_steps
    return _julia_round(float(np.sum(buf)) / buf.size), _julia_round(float(np.sum(stop)) / stop.size)


def calculate_dlogt(t0_sq, t, t_prev=None):
    """GradeProEstimator.jl:1074-1089."""
    if t_prev is None:
        det_prev = _prod(t0_sq)
    else:
        det_prev = _prod(t0_sq + t_prev ** 2)
    det_curr = _prod(t0_sq + t ** 2)
    return math.log(det_curr / det_prev)


def _prod(v):
    p = float(v[0])
    for x in v[1:]:
        p = p * float(x)
    return p


def default_params(ndim):
    """Defaults of GradeProEstimator.jl:705, 754-766 and DensityState eps (:541-550)."""
    return dict(alpha_s=0.0 if ndim == 1 else 0.06, alpha_os=0.1, eps=2.0 if ndim == 1 else -0.5)


# --------------------------------------------------------------------------- binning
def check_data(data, grid):
    """DirectSpace.jl:479-498."""
    data = np.asarray(data)
    for j in range(grid.ndim):
        x = data[j]
        if np.any((x >= grid.hi[j]) | (x <= grid.lo[j])):
            raise ValueError("Data points lie beyond grid. Remove them or increase grid boundaries.")


def dirac(data, grid, idx, include_var=True, nthreads=1, extended=False):
    """Binning through the C restatement.  data (N, n); idx (B, n) int32 1-based.
    Returns (M, V) real arrays of shape (B,) + grid.shape_c (V None if not include_var).
    extended: the same terms summed in long double and rounded once (a more exact binning
    than the reference's sequential FP64 sums)."""
    data = np.ascontiguousarray(np.asarray(data, dtype=np.float64).T)  # (n, N) == N x n col-major
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    B, n = idx.shape
    if data.shape[0] != n and B > 0:
        pass
    G = grid.size
    M = np.zeros((B, G), dtype=np.float64)
    V = np.zeros((B, G), dtype=np.float64) if include_var else None
    dims = np.array(grid.dims, dtype=np.int64)
    fn = _lib().oracle_dirac_ext if extended else _lib().oracle_dirac
    rc = fn(grid.ndim, dims.ctypes.data, grid.lo.ctypes.data, grid.hi.ctypes.data,
                             grid.h.ctypes.data, data.ctypes.data, data.shape[0], idx.ctypes.data, B,
                             M.ctypes.data, V.ctypes.data if V is not None else None, int(nthreads))
    if rc == 1:
        raise ValueError("Data points lie beyond grid. Remove them or increase grid boundaries.")
    if rc != 0:
        raise ValueError(f"oracle_dirac failed with code {rc}")
    shp = (B,) + grid.shape_c
    return M.reshape(shp), (V.reshape(shp) if V is not None else None)


def dirac_numpy(data, grid, idx, include_var=True):
    """Same arithmetic as binning.c in NumPy (np.add.at accumulates in index order)."""
    data = np.asarray(data, dtype=np.float64)
    check_data(data, grid)
    idx = np.asarray(idx)
    B, n = idx.shape
    N = grid.ndim
    G = grid.size
    sp = grid.h[0]
    for j in range(1, N):
        sp = sp * grid.h[j]
    denom = float(n) * (sp * sp)
    stride = [1]
    for j in range(1, N):
        stride.append(stride[-1] * grid.dims[j - 1])
    M = np.zeros((B, G))
    V = np.zeros((B, G)) if include_var else None
    for b in range(B):
        x = data[:, idx[b] - 1]  # (N, n)
        delta = x - grid.lo[:, None]
        il = np.floor(delta / grid.h[:, None]).astype(np.int64)
        rh = np.fmod(delta, grid.h[:, None])
        rl = grid.h[:, None] - rh
        cells = []
        terms = []
        for c in range(1 << N):
            pl = None
            ph = None
            cell = np.zeros(n, dtype=np.int64)
            for j in range(N):
                lower = (c >> (N - 1 - j)) & 1
                if lower:
                    pl = rl[j] if pl is None else pl * rl[j]
                    cell += il[j] * stride[j]
                else:
                    ph = rh[j] if ph is None else ph * rh[j]
                    cell += (il[j] + 1) * stride[j]
            pl = np.ones(n) if pl is None else pl
            ph = np.ones(n) if ph is None else ph
            cells.append(cell)
            terms.append((pl * ph) / denom)
        # draw-major, corner-minor order, as in the reference loop
        cells = np.stack(cells, axis=1).reshape(-1)
        terms = np.stack(terms, axis=1).reshape(-1)
        np.add.at(M[b], cells, terms)
        if include_var:
            np.add.at(V[b], cells, terms * terms)
    shp = (B,) + grid.shape_c
    return M.reshape(shp), (V.reshape(shp) if V is not None else None)


# ------------------------------------------------------------------- fourier space
def _spatial_axes(arr, batched):
    nd = arr.ndim - (1 if batched else 0)
    return tuple(range(arr.ndim - nd, arr.ndim))


_FFT_LIB = {"lib": "pocketfft"}


def _fftn(arr, axes, workers, inverse):
    """scipy.fft (pocketfft), or with _FFT_LIB["lib"] == "mkl" torch's CPU FFT (Intel
    MKL's DFT): another FP64 FFT implementation, for the rounding-stability variants."""
    if _FFT_LIB["lib"] == "mkl" and arr.dtype == np.complex128:
        import torch
        t = torch.from_numpy(np.ascontiguousarray(arr))
        out = (torch.fft.ifftn if inverse else torch.fft.fftn)(t, dim=axes)
        return out.numpy()
    return (sfft.ifftn if inverse else sfft.fftn)(arr, axes=axes, workers=workers)


def fourier_statistics(arr, workers=1):
    """FourierSpace.jl:25-52: unnormalised forward FFT over the grid axes (batched)."""
    return _fftn(arr, _spatial_axes(arr, True), workers, False)


def propagator(grid, t):
    """exp(-0.5 * sum_i (k_i t_i)^2), summed in axis order 1..N (FourierSpace.jl:228-234).
    Returned in C-order grid shape."""
    ks = fftgrid_axes(grid)
    acc = None
    for i in range(grid.ndim):
        term = (ks[i] * t[i]) ** 2
        shape = [1] * grid.ndim
        shape[grid.ndim - 1 - i] = grid.dims[i]
        term = term.reshape(shape)
        acc = (0.0 + term) if acc is None else acc + term
    return np.exp(-0.5 * acc)


def propagate_statistics(M0, V0, grid, t, t0):
    """FourierSpace.jl:215-241.  Complex x real products done per component."""
    p = propagator(grid, t)
    det_t0 = _prod(t0)
    det_t = math.sqrt(_prod(t0 ** 2 + t ** 2))
    Mt = (M0.real * p) + 1j * (M0.imag * p)
    sp = np.sqrt(p)
    Vt = (((V0.real * sp) * det_t0) / det_t) + 1j * (((V0.imag * sp) * det_t0) / det_t)
    return Mt, Vt


def propagate_means(M0, grid, t):
    """FourierSpace.jl:242-262."""
    p = propagator(grid, t)
    return (M0.real * p) + 1j * (M0.imag * p)


def ifourier_statistics(arr, batched=True, workers=1):
    """FourierSpace.jl:445-472: inverse FFT scaled by 1/G."""
    return _fftn(arr, _spatial_axes(arr, batched), workers, True)


# ------------------------------------------------------------------ direct space
def _fused_vmr(Mt, Vt, t, t0, n_samples):
    """scaled_vmr with fused multiply-adds (one rounding: long double intermediates
    rounded once to FP64) where the GPU library fuses: m = |M| (1/n), v = fma(-m, m,
    |V| (1/n)), the Welford updates mean = fma(delta, 1/i, mean) and m2 = fma(delta,
    x - mean, m2)."""
    ld = np.longdouble
    inv_n = 1.0 / float(n_samples)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        m = np.sqrt(Mt.real ** 2 + Mt.imag ** 2) * inv_n
        a = np.sqrt(Vt.real ** 2 + Vt.imag ** 2) * inv_n
        v = (a.astype(ld) - m.astype(ld) * m.astype(ld)).astype(np.float64)
        vmr = v / m
        B = vmr.shape[0]
        mean = np.zeros(vmr.shape[1:])
        m2 = np.zeros(vmr.shape[1:])
        for i in range(1, B + 1):
            x = vmr[i - 1]
            delta = x - mean
            mean = (delta.astype(ld) * ld(1.0 / i) + mean.astype(ld)).astype(np.float64)
            m2 = (delta.astype(ld) * (x - mean).astype(ld) + m2.astype(ld)).astype(np.float64)
        scaling = _prod(t ** 2 + t0 ** 2) ** (3 / 2) * float(n_samples ** 3)
        vv = scaling * m2 / (B - 1)
    out = np.full(vv.shape, np.nan)
    fin = np.isfinite(vv)
    out[fin] = np.log(vv[fin])
    return out


def scaled_vmr(Mt, Vt, t, t0, n_samples):
    """DirectSpace.jl:526-584.  Mt, Vt: complex (B, ...) after the inverse FFT."""
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        sk = np.sqrt(Mt.real ** 2 + Mt.imag ** 2) / n_samples
        s2k = np.sqrt(Vt.real ** 2 + Vt.imag ** 2) / n_samples - sk ** 2
        vmr = s2k / sk
        B = vmr.shape[0]
        mean = np.zeros(vmr.shape[1:])
        m2 = np.zeros(vmr.shape[1:])
        for i in range(1, B + 1):
            x = vmr[i - 1]
            delta = x - mean
            mean = mean + delta / i
            m2 = m2 + delta * (x - mean)
        scaling = _prod(t ** 2 + t0 ** 2) ** (3 / 2) * float(n_samples ** 3)
        v = scaling * m2 / (B - 1)
    out = np.full(v.shape, np.nan)
    fin = np.isfinite(v)
    out[fin] = np.log(v[fin])
    return out


def full_means(Mt):
    """DirectSpace.jl:747-764."""
    return np.sqrt(Mt.real ** 2 + Mt.imag ** 2)


@dataclass
class DensityState:
    """GradeProEstimator.jl:515-563."""
    eps: float
    steps_low: int
    steps_over: int
    shape: tuple
    minima: np.ndarray = None
    counters_low: np.ndarray = None
    counters_over: np.ndarray = None
    low_flags: np.ndarray = None
    f_prev1: np.ndarray = None
    f_prev2: np.ndarray = None

    def __post_init__(self):
        self.minima = np.full(self.shape, np.nan)
        self.counters_low = np.zeros(self.shape, dtype=np.uint16)
        self.counters_over = np.zeros(self.shape, dtype=np.uint16)
        self.low_flags = np.zeros(self.shape, dtype=bool)
        self.f_prev1 = np.full(self.shape, np.nan)
        self.f_prev2 = np.full(self.shape, np.nan)


def identify_convergence(density, means, f, f1, f2, dlogt, eps, steps_low, steps_over,
                         minima, counters_low, counters_over, low_flags):
    """DirectSpace.jl:829-871 + find_stability :975-1031, vectorised.  Mutates the state
    arrays and ``density`` in place; returns the ``more_stable`` mask."""
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        d1 = np.log(np.abs((f - f1) / (2 * dlogt)))
        d2 = np.log(np.abs((f - 2 * f1 + f2) / (dlogt * dlogt)))
    below = d2 < eps
    minnan = np.isnan(minima)
    not_low = ~low_flags
    a = not_low & below
    a_upd = a & ((d1 < minima) | minnan) & (counters_over.astype(np.int64) <= steps_over)
    a_inc = a & ~a_upd
    b = not_low & ~below
    c = low_flags & below & minnan
    more_stable = a_upd | c
    new_min = np.where(more_stable, d1, minima)
    counters_over[a_upd] = 0
    counters_over[a_inc] = counters_over[a_inc] + np.uint16(1)
    counters_low[b] = counters_low[b] + np.uint16(1)
    flip = b & (counters_low.astype(np.int64) > steps_low)
    low_flags[flip] = True
    new_min[flip] = np.nan
    minima[...] = new_min
    density[more_stable] = means[more_stable]
    return more_stable


# --------------------------------------------------------------------- estimator
@dataclass
class GradeProResult:
    density: np.ndarray
    selected_step: np.ndarray
    times: np.ndarray
    steps_low: int
    steps_over: int
    eps: float
    vmr_trace: list = field(default_factory=list)
    means_trace: list = field(default_factory=list)


def ladder(data, grid, n_steps=None, bw_step=None, bw_final=None, alpha_s=None, alpha_os=None, eps=None):
    """Host-side set-up of GradeProEstimator.jl:740-796: times, steps_low/over, eps."""
    ndim = grid.ndim
    d = default_params(ndim)
    alpha_s = d["alpha_s"] if alpha_s is None else alpha_s
    alpha_os = d["alpha_os"] if alpha_os is None else alpha_os
    eps = d["eps"] if eps is None else eps
    if bw_final is None:
        bw_final = silverman_rule(data)
    elif np.isscalar(bw_final):
        bw_final = np.full(ndim, float(bw_final))
    times, dt = get_time(np.asarray(bw_final, dtype=np.float64), n_steps=n_steps, time_step=bw_step)
    steps_low, steps_over = calculate_duration_steps(times[-1], dt, alpha_s=alpha_s, alpha_os=alpha_os)
    return times, steps_low, steps_over, float(eps)


def _r2c_propagate(Mb_hat, Vb_hat, grid, t, t0):
    """propagate_statistics on half spectra (last C axis = grid axis 1 halved)."""
    h1 = grid.dims[0] // 2 + 1
    p = propagator(grid, t)[..., :h1]
    det_t0 = _prod(t0)
    det_t = math.sqrt(_prod(t0 ** 2 + t ** 2))
    Mt = (Mb_hat.real * p) + 1j * (Mb_hat.imag * p)
    sp = np.sqrt(p)
    Vt = None
    if Vb_hat is not None:
        Vt = (((Vb_hat.real * sp) * det_t0) / det_t) + 1j * (((Vb_hat.imag * sp) * det_t0) / det_t)
    return Mt, Vt


def propagator_separable(grid, t):
    """exp(-0.5 sum_i (k_i t_i)^2) as the product of per-axis factors exp(-0.5 (k_i t_i)^2)
    (the same mathematics, other rounding), and its square root as the product of the
    per-axis square roots."""
    ks = fftgrid_axes(grid)
    p = None
    sp = None
    for i in range(grid.ndim):
        e = np.exp(-0.5 * (ks[i] * t[i]) ** 2)
        shape = [1] * grid.ndim
        shape[grid.ndim - 1 - i] = grid.dims[i]
        e = e.reshape(shape)
        p = e if p is None else p * e
        sp = np.sqrt(e) if sp is None else sp * np.sqrt(e)
    return p, sp


def estimate_gradepro(data, grid, idx, n_steps=None, bw_step=None, bw_final=None, alpha_s=None,
                      alpha_os=None, eps=None, workers=1, keep_trace=False, dirac_fn=None, fft_mode="c2c",
                      variant=None):
    """GradeProEstimator.jl:700-735 + :968-1060 (``estimate!``) on the CPU in FP64.

    data: (N, n) float64; idx: (B, n) int32 1-based bootstrap draws.
    fft_mode "c2c" follows the reference (complex transforms of the real arrays, |.| of
    the complex result); "r2c" uses real-input transforms instead -- the same
    mathematics with different FP64 rounding, used to tell which grid points' decisions
    are decided by rounding noise (see ``stable_points``).  `variant` (c2c only) names
    another FP64 implementation of the same mathematics, for the same purpose (each is
    deterministic, like any real implementation):
      "paired"     two bootstraps' real arrays in one complex transform, |Re| and |Im| as
                   their magnitudes (the GPU library's pairing);
      "sep"        the propagator as a product of per-axis factors (also the GPU's);
      "paired-sep" both;
      "longdouble" every transform and the VMR in 80-bit extended precision;
      "jitter-K"   the forward spectra multiplied once by (1 + u g), g standard normal
                   from seed K, u = 2^-53: the rounding of another forward transform;
      "xbin"       the binned sums accumulated in long double and rounded once (a more
                   exact binning, like the GPU library's fixed-point sums);
      "gpu-like"   xbin, paired and sep together;
      "mkl", "mkl-gpu-like"  as c2c and gpu-like, every transform by Intel MKL's DFT
                   (torch's CPU FFT) instead of pocketfft;
      "gpu-fma"    gpu-like with the VMR numerator and the Welford updates fused (one
                   rounding each, as the GPU library computes them).
    keep_trace: True keeps every step's log-VMR variance and means, "f" only the former.
    Returns GradeProResult with density/selected_step in C-order grid shape."""
    if variant is not None and variant.startswith("mkl"):
        _FFT_LIB["lib"] = "mkl"
        try:
            return estimate_gradepro(data, grid, idx, n_steps, bw_step, bw_final, alpha_s, alpha_os, eps, workers,
                                     keep_trace, dirac_fn, fft_mode, None if variant == "mkl" else variant[4:])
        finally:
            _FFT_LIB["lib"] = "pocketfft"
    data = np.asarray(data, dtype=np.float64)
    n = data.shape[1]
    if idx.shape[0] < 2:
        raise ValueError("at least 2 bootstraps are needed for a variance")
    binner = dirac if dirac_fn is None else dirac_fn
    bkw = dict(extended=True, nthreads=workers) if variant in ("xbin", "gpu-like", "gpu-fma") else {}
    Mb, Vb = binner(data, grid, idx, include_var=True, **bkw)
    ident = np.arange(1, n + 1, dtype=np.int32).reshape(1, n)
    Mf, _ = binner(data, grid, ident, include_var=False, **bkw)
    if fft_mode == "r2c":
        return _estimate_r2c(data, grid, Mb, Vb, Mf, n, n_steps, bw_step, bw_final, alpha_s, alpha_os, eps,
                             workers, keep_trace)
    cdt = np.clongdouble if variant == "longdouble" else np.complex128
    paired = variant in ("paired", "paired-sep", "gpu-like", "gpu-fma")
    if paired:  # z = M_b + i M_b+1 (odd B: the last one alone), w likewise
        B = Mb.shape[0]
        zs = [Mb[b] + 1j * (Mb[b + 1] if b + 1 < B else 0.0) for b in range(0, B, 2)]
        ws = [Vb[b] + 1j * (Vb[b + 1] if b + 1 < B else 0.0) for b in range(0, B, 2)]
        Mb_hat = fourier_statistics(np.stack(zs), workers)
        Vb_hat = fourier_statistics(np.stack(ws), workers)
    else:
        Mb_hat = fourier_statistics(Mb.astype(cdt), workers)
        Vb_hat = fourier_statistics(Vb.astype(cdt), workers)
    Mf_hat = fourier_statistics(Mf.astype(cdt), workers)[0]
    if variant is not None and variant.startswith("jitter-"):
        jr = np.random.default_rng(int(variant[7:]))
        for a in (Mb_hat, Vb_hat, Mf_hat):
            a *= 1.0 + 2.0 ** -53 * jr.standard_normal(a.shape)
    times, steps_low, steps_over, eps = ladder(data, grid, n_steps, bw_step, bw_final, alpha_s, alpha_os, eps)
    t0 = initial_bandwidth(grid)
    t0_sq = t0 ** 2
    shape = grid.shape_c
    st = DensityState(eps, steps_low, steps_over, shape)
    density = np.full(shape, np.nan)
    selected = np.full(shape, -1, dtype=np.int32)
    res = GradeProResult(density, selected, times, steps_low, steps_over, eps)
    means = None
    for s, t in enumerate(times):
        if variant in ("sep", "paired-sep", "gpu-like", "gpu-fma"):
            p, sp = propagator_separable(grid, t)
            c = _prod(t0) / math.sqrt(_prod(t0 ** 2 + t ** 2))
            Mt = Mb_hat * p
            Vt = Vb_hat * (sp * c)
            Ft = Mf_hat * p
        else:
            Mt, Vt = propagate_statistics(Mb_hat, Vb_hat, grid, t, t0)
            Ft = propagate_means(Mf_hat, grid, t)
        Mt = ifourier_statistics(Mt, True, workers)
        Vt = ifourier_statistics(Vt, True, workers)
        Ft = ifourier_statistics(Ft, False, workers)
        if paired:  # back to one real array per bootstrap: |Re| and |Im| of each pair
            B = Mb.shape[0]
            Mt = np.stack([np.abs(Mt[b // 2].real if b % 2 == 0 else Mt[b // 2].imag) for b in range(B)]) + 0j
            Vt = np.stack([np.abs(Vt[b // 2].real if b % 2 == 0 else Vt[b // 2].imag) for b in range(B)]) + 0j
        f = (_fused_vmr if variant == "gpu-fma" else scaled_vmr)(Mt, Vt, t, t0, n)
        means = full_means(Ft)
        if variant == "longdouble":
            f = f.astype(np.float64)
            means = means.astype(np.float64)
        dlogt = calculate_dlogt(t0_sq, t) if s == 0 else calculate_dlogt(t0_sq, t, times[s - 1])
        ms = identify_convergence(density, means, f, st.f_prev1, st.f_prev2, dlogt, st.eps, st.steps_low,
                                  st.steps_over, st.minima, st.counters_low, st.counters_over, st.low_flags)
        selected[ms] = s
        st.f_prev2 = st.f_prev1.copy()
        st.f_prev1 = f.copy()
        if keep_trace:
            res.vmr_trace.append(f)
            if keep_trace != "f":
                res.means_trace.append(means)
    nan = np.isnan(density)
    density[nan] = means[nan]
    selected[selected < 0] = len(times)
    res.selected_step = selected
    return res


def _estimate_r2c(data, grid, Mb, Vb, Mf, n, n_steps, bw_step, bw_final, alpha_s, alpha_os, eps, workers,
                  keep_trace):
    ax = tuple(range(1, 1 + grid.ndim))
    Mb_hat = sfft.rfftn(Mb, axes=ax, workers=workers)
    Vb_hat = sfft.rfftn(Vb, axes=ax, workers=workers)
    Mf_hat = sfft.rfftn(Mf, axes=ax, workers=workers)
    times, steps_low, steps_over, eps = ladder(data, grid, n_steps, bw_step, bw_final, alpha_s, alpha_os, eps)
    t0 = initial_bandwidth(grid)
    t0_sq = t0 ** 2
    shape = grid.shape_c
    st = DensityState(eps, steps_low, steps_over, shape)
    density = np.full(shape, np.nan)
    selected = np.full(shape, -1, dtype=np.int32)
    res = GradeProResult(density, selected, times, steps_low, steps_over, eps)
    means = None
    for s, t in enumerate(times):
        Mt, Vt = _r2c_propagate(Mb_hat, Vb_hat, grid, t, t0)
        Mt = sfft.irfftn(Mt, s=shape, axes=ax, workers=workers)
        Vt = sfft.irfftn(Vt, s=shape, axes=ax, workers=workers)
        f = scaled_vmr(Mt + 0j, Vt + 0j, t, t0, n)
        Ft, _ = _r2c_propagate(Mf_hat, None, grid, t, t0)
        means = np.abs(sfft.irfftn(Ft, s=shape, axes=ax, workers=workers)[0])
        dlogt = calculate_dlogt(t0_sq, t) if s == 0 else calculate_dlogt(t0_sq, t, times[s - 1])
        ms = identify_convergence(density, means, f, st.f_prev1, st.f_prev2, dlogt, st.eps, st.steps_low,
                                  st.steps_over, st.minima, st.counters_low, st.counters_over, st.low_flags)
        selected[ms] = s
        st.f_prev2 = st.f_prev1.copy()
        st.f_prev1 = f.copy()
        if keep_trace:
            res.vmr_trace.append(f)
            if keep_trace != "f":
                res.means_trace.append(means)
    nan = np.isnan(density)
    density[nan] = means[nan]
    selected[selected < 0] = len(times)
    res.selected_step = selected
    return res


def select_from_trace(f_steps, times, t0, steps_low, steps_over, eps):
    """The selected step of every point from a sequence of log-VMR-variance arrays alone
    (the decisions of identify_convergence depend on f only; the means only fill the
    density).  f_steps yields one array per step, any shape (e.g. samples x grid
    points); returns int32 steps with the estimator's convention (len(times) where no
    step was selected).  Same loop as estimate_gradepro."""
    t0_sq = np.asarray(t0) ** 2
    st = None
    selected = None
    for s, f in enumerate(f_steps):
        if st is None:
            st = DensityState(eps, steps_low, steps_over, f.shape)
            selected = np.full(f.shape, -1, dtype=np.int32)
            dummy = np.zeros(f.shape)
        dlogt = calculate_dlogt(t0_sq, times[s]) if s == 0 else calculate_dlogt(t0_sq, times[s], times[s - 1])
        ms = identify_convergence(dummy, dummy, f, st.f_prev1, st.f_prev2, dlogt, st.eps, st.steps_low,
                                  st.steps_over, st.minima, st.counters_low, st.counters_over, st.low_flags)
        selected[ms] = s
        st.f_prev2 = st.f_prev1
        st.f_prev1 = f.copy()
    selected[selected < 0] = len(times)
    return selected


def stable_points(ref, alt):
    """Grid points whose outcome does not depend on FP64 rounding: the reference-faithful
    run ``ref`` and a run ``alt`` with different rounding (fft_mode="r2c") select the same
    bandwidth step.  The reference's decision at the other points is set by rounding
    noise -- typically at cells that are empty at t = 0, where the VMR is 0/0 up to
    FFT round-off -- so no implementation can reproduce it."""
    return ref.selected_step == alt.selected_step


# ------------------------------------------------------------------------- :rot
def rot_time(data, rule="scott"):
    """propagation_time of the rules of thumb (RoTEstimator.jl:24-49): factor * the
    per-axis standard deviations (diag of Statistics.cov, divisor n - 1)."""
    data = np.asarray(data, dtype=np.float64)
    ndim, n = data.shape
    if rule == "silverman":
        factor = (n * (ndim + 2) / 4) ** (-1 / (ndim + 4))
    elif rule == "scott":
        factor = n ** (-1 / (ndim + 4))
    else:
        raise ValueError(f"Rule of thumb {rule} not implemented.")
    return factor * np.sqrt(np.var(data, axis=1, ddof=1))


def estimate_rot(data, grid, rule="scott"):
    """The :rot estimator on the CPU (RoTEstimator.jl:143-148, 159-201, 203-230):
    binning of every sample once (means only), unnormalised forward FFT, propagation by
    t = rule-of-thumb time - h/2 (RoTEstimator.jl:64-66), inverse FFT scaled by 1/G,
    density = |.|.  Returns the density in C-order grid shape."""
    data = np.asarray(data, dtype=np.float64)
    n = data.shape[1]
    ident = np.arange(1, n + 1, dtype=np.int32)[None]
    M, _ = dirac(data, grid, ident, include_var=False)
    Mh = fourier_statistics(M.astype(complex))[0]
    t = rot_time(data, rule) - initial_bandwidth(grid)
    Mt = propagate_means(Mh, grid, t)
    return np.abs(ifourier_statistics(Mt, batched=False))


def normalize_density(density, grid):
    """ParallelKDE.jl:192-194: density ./= sum(density) * prod(spacings)."""
    return density / (np.sum(density) * _prod(grid.h))
