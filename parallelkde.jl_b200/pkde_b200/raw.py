"""Thin wrappers of the individual C-ABI entry points (host NumPy arrays or CUDA torch
tensors).  These mirror the reference's internal functions that its own tests call
(initialize_dirac_sequence, fourier_statistics!/ifourier_statistics!,
calculate_scaled_vmr!, identify_convergence!)."""
import ctypes

import numpy as np

from ._lib import (PKDE_DEVICE_INPUT, PKDE_DEVICE_OUTPUT, ArgumentError, PkdeGradeproParams, check, context, load,
                   make_grid_struct,
                   make_params, ptr)


def _is_dev(a):
    return a is not None and not isinstance(a, np.ndarray)


def dirac_sequence(grid, data, bootstrap_idxs=None, n_bootstraps=None, seed=0, include_var=True, device_id=0,
                   counts=True):
    """Binning of bootstrap resamples (DirectSpace.jl:289-362, arithmetic of :196-287).

    data: N x n float64.  bootstrap_idxs: (B, n) int32 1-based or None (seeded draws, or
    the identity when n_bootstraps == 0).  Returns (means, sq, counts) as arrays of shape
    (B,) + reversed(grid dims) (the identity has B = 1 and sq = None)."""
    lib = load()
    ctx = context(device_id)
    data = np.ascontiguousarray(np.asarray(data, dtype=np.float64))
    if data.ndim == 1:
        data = data.reshape(1, -1)
    N, n = data.shape
    if bootstrap_idxs is not None:
        idx = np.ascontiguousarray(bootstrap_idxs, dtype=np.int32)
        B = idx.shape[0]
    else:
        idx = None
        B = 0 if n_bootstraps is None else int(n_bootstraps)
    slots = max(B, 1)
    G = int(np.prod(grid.dims))
    gs = make_grid_struct(grid.lo, grid.hi, grid.h, grid.dims)
    M = np.empty((slots, G))
    V = np.empty((slots, G)) if include_var and B > 0 else None
    C = np.empty((slots, G), dtype=np.uint32) if counts else None
    dt = np.ascontiguousarray(data.T)
    rc = lib.pkde_dirac_sequence(ctx, ctypes.byref(gs), ptr(dt), n, ptr(idx), B, int(seed), ptr(M), ptr(V), ptr(C),
                                 0, None)
    check(rc, ctx)
    shp = (slots,) + tuple(reversed(grid.dims))
    return M.reshape(shp), (V.reshape(shp) if V is not None else None), (C.reshape(shp) if C is not None else None)


def fft(arr, direction, device_id=0):
    """In-place-style N-D FFT over all axes but the first (batch) of a complex128 array of
    C-order shape (B, n_N, ..., n_1).  direction -1: forward unnormalised; +1: inverse / G."""
    lib = load()
    ctx = context(device_id)
    a = np.array(arr, dtype=np.complex128, order="C", copy=True)
    dims = np.array(list(reversed(a.shape[1:])), dtype=np.int64)
    rc = lib.pkde_fft(ctx, len(dims), ptr(dims), ptr(a), a.shape[0], int(direction), 0, None)
    check(rc, ctx)
    return a


def scaled_vmr(means, sq, t, t0, n_samples, device_id=0):
    """calculate_scaled_vmr! (DirectSpace.jl:526-584) of complex (B, ...) arrays; returns
    the grid-shaped log scaled variance of the VMR."""
    lib = load()
    ctx = context(device_id)
    m = np.ascontiguousarray(np.asarray(means, dtype=np.complex128))
    s = np.ascontiguousarray(np.asarray(sq, dtype=np.complex128))
    B = m.shape[0]
    G = int(np.prod(m.shape[1:]))
    t = np.ascontiguousarray(np.asarray(t, dtype=np.float64).reshape(-1))
    t0 = np.ascontiguousarray(np.asarray(t0, dtype=np.float64).reshape(-1))
    out = np.empty(G)
    rc = lib.pkde_scaled_vmr(ctx, G, B, ptr(m), ptr(s), len(t), ptr(t), ptr(t0), int(n_samples), ptr(out), 0, None)
    check(rc, ctx)
    return out.reshape(m.shape[1:])


def identify_convergence(density, means, vmr_current, vmr_prev1, vmr_prev2, dlogt, eps, steps_low, steps_over,
                         minima, counters_low, counters_over, low_density_flags, device_id=0):
    """identify_convergence! (DirectSpace.jl:829-973): updates density, minima, counters
    and flags in place (host NumPy arrays of equal size)."""
    lib = load()
    ctx = context(device_id)
    G = density.size
    arrs = [density, means, vmr_current, vmr_prev1, vmr_prev2, minima]
    for a in arrs:
        if a.dtype != np.float64 or not a.flags.c_contiguous or a.size != G:
            raise ArgumentError("float64 contiguous arrays of equal size expected")
    for a, dt in ((counters_low, np.uint16), (counters_over, np.uint16), (low_density_flags, np.bool_)):
        if a.dtype != dt or not a.flags.c_contiguous or a.size != G:
            raise ArgumentError("counter/flag arrays of the grid size expected")
    rc = lib.pkde_identify_convergence(ctx, G, ptr(density), ptr(means), ptr(vmr_current), ptr(vmr_prev1),
                                       ptr(vmr_prev2), float(dlogt), float(eps), int(steps_low), int(steps_over),
                                       ptr(minima), ptr(counters_low), ptr(counters_over), ptr(low_density_flags), 0,
                                       None)
    check(rc, ctx)


def gradepro_device(grid, data_dev, n_samples, density_dev, selected_dev=None, idx_dev=None, seed=0, stream=None,
                    device_id=0, **kwargs):
    """estimate with device-resident inputs/outputs (CUDA torch tensors):
    data_dev (n, N) float64 contiguous (== N x n column-major), density_dev (G,) float64."""
    lib = load()
    ctx = context(device_id)
    gs = make_grid_struct(grid.lo, grid.hi, grid.h, grid.dims)
    p = make_params(gs, **kwargs)
    flags = PKDE_DEVICE_INPUT | PKDE_DEVICE_OUTPUT
    rc = lib.pkde_gradepro_estimate(ctx, ctypes.byref(p), ptr(data_dev), int(n_samples), ptr(idx_dev),
                                    int(seed) & (2**64 - 1), ptr(density_dev), ptr(selected_dev), flags, stream)
    check(rc, ctx)


def gradepro_host(grid, data, density_out, selected_out=None, idx=None, seed=0, stream=None, device_id=0,
                  **kwargs):
    """estimate with host inputs/outputs (NumPy arrays, pinned or pageable): data (n, N)
    float64 contiguous; density_out (G,) float64."""
    lib = load()
    ctx = context(device_id)
    gs = make_grid_struct(grid.lo, grid.hi, grid.h, grid.dims)
    p = make_params(gs, **kwargs)
    rc = lib.pkde_gradepro_estimate(ctx, ctypes.byref(p), ptr(data), int(data.shape[0]), ptr(idx),
                                    int(seed) & (2**64 - 1), ptr(density_out), ptr(selected_out), 0, stream)
    check(rc, ctx)


def gradepro_batch(jobs, device=False, stream=None, device_id=0):
    """Several estimations in one pkde_gradepro_estimate_batch call.

    jobs: list of dicts with keys grid, data, density, and optionally selected, idx, seed
    and the keyword arguments of make_params (n_bootstraps, n_steps, bw_step, bw_final,
    alpha_s, alpha_os, eps).  device=False: host NumPy arrays (data (n, N) float64
    C-contiguous, density (G,) float64, selected (G,) int32, idx (B, n) int32);
    device=True: CUDA torch tensors of the same shapes."""
    lib = load()
    ctx = context(device_id)
    count = len(jobs)
    params = (PkdeGradeproParams * count)()
    keys = ("n_bootstraps", "n_steps", "bw_step", "bw_final", "alpha_s", "alpha_os", "eps")
    vp = ctypes.c_void_p
    data_p, idx_p, dens_p, sel_p = (vp * count)(), (vp * count)(), (vp * count)(), (vp * count)()
    n_arr = (ctypes.c_int64 * count)()
    seeds = (ctypes.c_uint64 * count)()
    any_idx = any_sel = False
    for e, j in enumerate(jobs):
        g = j["grid"]
        params[e] = make_params(make_grid_struct(g.lo, g.hi, g.h, g.dims), **{k: j[k] for k in keys if k in j})
        data_p[e] = ptr(j["data"])
        n_arr[e] = int(j["data"].shape[0])
        dens_p[e] = ptr(j["density"])
        seeds[e] = int(j.get("seed", 0)) & (2**64 - 1)
        if j.get("idx") is not None:
            idx_p[e] = ptr(j["idx"])
            any_idx = True
        if j.get("selected") is not None:
            sel_p[e] = ptr(j["selected"])
            any_sel = True
    flags = (PKDE_DEVICE_INPUT | PKDE_DEVICE_OUTPUT) if device else 0
    rc = lib.pkde_gradepro_estimate_batch(ctx, count, params, data_p, n_arr, idx_p if any_idx else None, seeds,
                                          dens_p, sel_p if any_sel else None, flags, stream)
    check(rc, ctx)


def rot(grid, data, rule="scott", density=None, device=False, stream=None, device_id=0):
    """The :rot estimator through pkde_rot_estimate.  data: (n, N) float64 C-contiguous
    (host NumPy, or a CUDA tensor with device=True); returns the density (G,)."""
    lib = load()
    ctx = context(device_id)
    rules = {"scott": 0, "silverman": 1}
    r = rules.get(str(rule).lstrip(":"), -1)
    gs = make_grid_struct(grid.lo, grid.hi, grid.h, grid.dims)
    G = int(np.prod(grid.dims))
    if density is None:
        density = np.empty(G)
    flags = (PKDE_DEVICE_INPUT | PKDE_DEVICE_OUTPUT) if device else 0
    rc = lib.pkde_rot_estimate(ctx, ctypes.byref(gs), r, ptr(data), int(data.shape[0]), ptr(density), flags, stream)
    check(rc, ctx)
    return density


def find_grid_device(data, grid_dims=None, grid_steps=None, grid_padding=None, device=False, stream=None,
                     device_id=0):
    """find_grid (Grids.jl:252-300) with the extrema reduced on the GPU: data (n, N)
    float64 C-contiguous host array, or a CUDA tensor with device=True.  Returns a Grid."""
    from .grids import Grid
    from ._lib import PkdeGrid
    lib = load()
    ctx = context(device_id)
    n, N = int(data.shape[0]), int(data.shape[1])
    dims = None if grid_dims is None else np.ascontiguousarray(grid_dims, dtype=np.int64)
    steps = None if grid_steps is None else np.ascontiguousarray(grid_steps, dtype=np.float64)
    pad = None if grid_padding is None else np.ascontiguousarray(grid_padding, dtype=np.float64)
    g = PkdeGrid()
    rc = lib.pkde_find_grid(ctx, N, ptr(data), n, ptr(dims), ptr(steps), ptr(pad), ctypes.byref(g),
                            PKDE_DEVICE_INPUT if device else 0, stream)
    check(rc, ctx)
    return Grid([g.lo[j] for j in range(N)], [g.hi[j] for j in range(N)], [g.dims[j] for j in range(N)],
                [g.h[j] for j in range(N)])


def normalize_density(density, dx, device=False, stream=None, device_id=0):
    """density /= sum(density) * dx in place, FP64 sum on the GPU (ParallelKDE.jl:189-202)."""
    lib = load()
    ctx = context(device_id)
    G = int(np.prod(density.shape))
    rc = lib.pkde_normalize_density(ctx, ptr(density), G, float(dx), PKDE_DEVICE_INPUT if device else 0, stream)
    check(rc, ctx)
    return density
