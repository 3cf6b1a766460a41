"""Host-side mirror of ParallelKDE.jl's user API and estimator plugin interface for the
``device=:cuda`` ``:gradepro`` path, over the C ABI (include/pkde_b200.h).

Names, argument meaning and error behaviour follow the reference:
  initialize_estimation / estimate_density / get_density   src/ParallelKDE.jl:102-226
  add_estimator / estimator_lookup / estimate              src/DensityEstimators/DensityEstimators.jl:31-115
  initialize_kde / bootstrap_indices / set_nan_density     src/KDEs/KDEs.jl:62-206
``estimate_density!`` is spelled ``estimate_density`` (no ``!`` in Python); ArgumentError
is ``pkde_b200.ArgumentError`` (a ValueError).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import ArgumentError, check, context, load, make_grid_struct, make_params, ptr
from .grids import AVAILABLE_DEVICES, Grid, find_grid, initialize_grid

DEVICE_IMPLEMENTATIONS = {"cpu": set(), "cuda": {"cuda"}}
DEFAULT_IMPLEMENTATIONS = {"cuda": "cuda"}


def ensure_valid_implementation(device, method):
    """Devices.jl:125-133 (the CPU methods live in the reference, not here)."""
    if method not in DEVICE_IMPLEMENTATIONS.get(device, set()):
        raise ArgumentError(f"Invalid implementation {method} for device {device}")
    return True


# ---------------------------------------------------------------------------- KDE
class KDE:
    """Samples (N x n, FP64) and the density on the grid (KDEs.jl:44-47, CuKDE).

    ``samples`` holds the same values as an (n, N) C-contiguous array -- the N x n
    column-major layout the C ABI reads -- made once here, like the reference's one H2D
    copy in initialize_kde (KDEs.jl:94-111); ``pin()`` moves it to page-locked memory."""

    def __init__(self, data, dims):
        self.data = data
        if hasattr(data, "is_cuda"):  # samples already on the GPU stay there
            self.samples = data.double().t().contiguous()
        else:
            self.samples = np.ascontiguousarray(np.asarray(data).T)
        self.density = np.full(tuple(reversed(dims)), np.nan)
        self.dims = tuple(dims)
        self._pinned = None

    @property
    def ndim(self):
        return len(self.dims)

    def pin(self):
        """Keep the samples in page-locked host memory (faster host-to-device copies)."""
        if not isinstance(self.samples, np.ndarray):
            return self
        import torch
        t = torch.empty(self.samples.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = self.samples
        dp = torch.empty(self.density.shape, dtype=torch.float64, pin_memory=True)
        dp.numpy()[...] = self.density
        self._pinned = (t, dp)
        self.samples = t.numpy()
        self.density = dp.numpy()
        return self

    def density_out(self):
        """A flat FP64 view of ``density`` the library can write into directly, or None
        when ``density`` was replaced by an array of another layout."""
        d = self.density
        if isinstance(d, np.ndarray) and d.dtype == np.float64 and d.flags.c_contiguous and d.flags.writeable:
            return d.reshape(-1)
        return None


def _as_samples(data):
    if isinstance(data, (list, tuple)) and len(data) and np.ndim(data[0]) == 1:
        data = np.stack([np.asarray(v, dtype=np.float64) for v in data], axis=1)
    if hasattr(data, "is_cuda"):
        return data
    a = np.asarray(data, dtype=np.float64)
    if a.ndim == 1:
        a = a.reshape(1, -1)
    if a.ndim != 2:
        raise ArgumentError("Data must be a matrix or vector.")
    return np.ascontiguousarray(a)


def initialize_kde(data, dims, device="cuda"):
    """KDEs.jl:62-111."""
    if device not in AVAILABLE_DEVICES:
        raise ArgumentError(f"Invalid device: {device}")
    if device != "cuda":
        raise ArgumentError("this package implements the device=:cuda path only")
    a = _as_samples(data)
    if a.shape[0] != len(dims):
        raise ArgumentError(f"Data must have {len(dims)} dimensions")
    return KDE(a, dims)


def get_nsamples(kde):
    return int(kde.data.shape[1])


def get_data(kde):
    return kde.data


def set_density(kde, density):
    kde.density[...] = density


def set_nan_density(kde):
    kde.density[...] = np.nan


def bootstrap_indices(kde, n_bootstraps, seed=0):
    """n x B 1-based draws (KDEs.jl:182-206) from the library's counter-based generator,
    returned as a (B, n) int32 array (= column-major n x B).  B = 0 gives the identity."""
    n = get_nsamples(kde)
    if n_bootstraps < 0:
        raise ArgumentError("Number of bootstraps must be non-negative")
    if n_bootstraps == 0:
        return np.arange(1, n + 1, dtype=np.int32).reshape(1, n)
    lib = load()
    out = np.empty((n_bootstraps, n), dtype=np.int32)
    for b in range(n_bootstraps):
        out[b] = [lib.pkde_boot_index(seed, n, b, j) + 1 for j in range(n)]
    return out


# ------------------------------------------------------------------ estimation
class DensityEstimation:
    """ParallelKDE.jl:75-78."""

    def __init__(self, kde, grid):
        self.kde = kde
        self.grid = grid
        self.selected_step = None


def initialize_estimation(data, grid=False, grid_ranges=None, dims=None, grid_bounds=None, grid_padding=None,
                          device="cuda"):
    """ParallelKDE.jl:102-158."""
    a = _as_samples(data)
    if device not in AVAILABLE_DEVICES:
        raise ArgumentError(f"Invalid device: {device}")
    if device != "cuda":
        raise ArgumentError("this package implements the device=:cuda path only")
    if isinstance(grid, bool):
        if grid:
            if grid_ranges is not None:
                grid = initialize_grid(grid_ranges, device=device)
            elif isinstance(a, np.ndarray) or grid_bounds is not None:
                host = a if isinstance(a, np.ndarray) else a.double().cpu().numpy()
                grid = find_grid(host, grid_bounds=grid_bounds, grid_dims=dims, grid_padding=grid_padding,
                                 device=device)
            else:  # samples already on the GPU: extrema reduced there (pkde_find_grid)
                from . import raw
                grid = raw.find_grid_device(a.double().t().contiguous(), grid_dims=dims, grid_padding=grid_padding,
                                            device=True, device_id=a.device.index or 0)
        else:
            grid = None
    elif getattr(grid, "device", device) != device:
        raise ArgumentError("Grid must be of the same device as the KDE.")
    if grid is None and dims is None:
        raise ArgumentError("Grid must be required if dims is not specified.")
    if grid is not None:
        dims = grid.dims
    return DensityEstimation(initialize_kde(a, dims, device=device), grid)


def has_grid(est):
    return est.grid is not None


def get_grid(est):
    return est.grid


def get_density(est, normalize=False, dx=None):
    """ParallelKDE.jl:189-202: with normalize, density /= sum(density) * prod(spacings)
    (or dx), the sum in FP64 on the GPU (pkde_normalize_density)."""
    from . import raw
    d = est.kde.density
    if normalize and has_grid(est):
        raw.normalize_density(np.ascontiguousarray(d) if not d.flags.c_contiguous else d, float(np.prod(est.grid.h)))
    elif normalize and dx is not None:
        raw.normalize_density(d, float(dx))
    elif normalize:
        raise ArgumentError("Normalization requires a grid or dx to be specified.")
    return d


# -------------------------------------------------------------- estimator plugins
class AbstractEstimator:
    """DensityEstimators.jl:29; subclasses implement initialize_estimator/estimate."""

    @classmethod
    def initialize_estimator(cls, kde, **kwargs):
        raise ArgumentError("Estimator not implemented")

    def estimate(self, kde, **kwargs):
        raise ArgumentError("Estimator not implemented")


estimator_lookup = {}


def add_estimator(key, value):
    """DensityEstimators.jl:37-45."""
    if key in estimator_lookup:
        raise ArgumentError(f"Key {key} already exists")
    estimator_lookup[key] = value


def estimate(estimator_name, kde, method=None, **kwargs):
    """DensityEstimators.jl:58-84: look up, validate the implementation, run."""
    if estimator_name not in estimator_lookup:
        raise ArgumentError(f"Estimator {estimator_name} not registered")
    cls = estimator_lookup[estimator_name]
    device = "cuda"
    if method is None:
        method = DEFAULT_IMPLEMENTATIONS[device]
    ensure_valid_implementation(device, method)
    est = cls.initialize_estimator(kde, method=method, **kwargs)
    est.estimate(kde, method=method, **kwargs)


class GradeProEstimator(AbstractEstimator):
    """The ``:gradepro`` estimator (GradeProEstimator.jl:684-858) on the B200 library."""

    KWARGS = ("grid", "n_bootstraps", "bw_step", "bw_final", "n_steps", "alpha_s", "alpha_os", "eps", "seed",
              "bootstrap_idxs", "stream", "device_id")

    def __init__(self, grid, params, seed, idx, stream, device_id):
        self.grid = grid
        self.params = params
        self.seed = seed
        self.idx = idx
        self.stream = stream
        self.device_id = device_id
        self.selected_step = None

    @classmethod
    def initialize_estimator(cls, kde, method="cuda", grid=None, n_bootstraps=100, bw_step=None, n_steps=None,
                             bw_final=None, alpha_s=None, alpha_os=None, eps=None, seed=0, bootstrap_idxs=None,
                             stream=None, device_id=0, **unused):
        for k in unused:
            if k not in cls.KWARGS:
                raise ArgumentError(f"unknown keyword argument {k}")
        if grid is None:
            raise ArgumentError("the :gradepro estimator needs a grid")
        if n_bootstraps < 0:
            raise ArgumentError("Number of boostraps must be positive.")
        gs = make_grid_struct(grid.lo, grid.hi, grid.h, grid.dims)
        p = make_params(gs, n_bootstraps, n_steps, bw_step, bw_final, alpha_s, alpha_os, eps)
        idx = None
        if bootstrap_idxs is not None:
            idx = np.ascontiguousarray(bootstrap_idxs, dtype=np.int32)
            if idx.shape != (n_bootstraps, get_nsamples(kde)):
                raise ArgumentError("bootstrap_idxs must have shape (n_bootstraps, n_samples)")
        return cls(grid, p, seed, idx, stream, device_id)

    def estimate(self, kde, method="cuda", **unused):
        ctx = context(self.device_id)
        lib = load()
        G = int(np.prod(self.grid.dims))
        direct = kde.density_out()
        dens = direct if direct is not None and direct.size == G else np.empty(G, dtype=np.float64)
        sel = np.empty(G, dtype=np.int32)
        data_t = kde.samples  # (n, N) C-contiguous == N x n column-major
        flags, idx = 0, self.idx
        if not isinstance(data_t, np.ndarray):  # device samples: device inputs, host outputs
            flags = _lib.PKDE_DEVICE_INPUT
            if idx is not None:
                import torch
                idx = torch.from_numpy(idx).to(data_t.device)
        rc = lib.pkde_gradepro_estimate(ctx, ctypes.byref(self.params), ptr(data_t), data_t.shape[0],
                                        ptr(idx), int(self.seed) & (2**64 - 1), ptr(dens), ptr(sel), flags,
                                        self.stream)
        check(rc, ctx)
        if dens is not direct:
            kde.density[...] = dens.reshape(kde.density.shape)
        self.selected_step = sel.reshape(kde.density.shape)


add_estimator("gradepro", GradeProEstimator)


class RoTEstimator(AbstractEstimator):
    """The ``:rot`` estimator (RoTEstimator.jl:107-201) on the B200 library: one
    propagation of the binned samples by the rule-of-thumb bandwidth (``:scott``, the
    reference's default, or ``:silverman``; RoTEstimator.jl:24-49, :117-124)."""

    RULES = {"scott": 0, "silverman": 1}
    KWARGS = ("grid", "rule_of_thumb", "stream", "device_id")

    def __init__(self, grid, rule, stream, device_id):
        self.grid = grid
        self.rule = rule
        self.stream = stream
        self.device_id = device_id

    @classmethod
    def initialize_estimator(cls, kde, method="cuda", grid=None, rule_of_thumb="scott", stream=None, device_id=0,
                             **unused):
        for k in unused:
            if k not in cls.KWARGS:
                raise ArgumentError(f"unknown keyword argument {k}")
        if grid is None:
            raise ArgumentError("the :rot estimator needs a grid")
        rule = str(rule_of_thumb).lstrip(":")
        if rule not in cls.RULES:
            raise ArgumentError(f"Rule of thumb {rule} not implemented.")
        return cls(grid, rule, stream, device_id)

    def estimate(self, kde, method="cuda", **unused):
        ctx = context(self.device_id)
        lib = load()
        G = int(np.prod(self.grid.dims))
        direct = kde.density_out()
        dens = direct if direct is not None and direct.size == G else np.empty(G, dtype=np.float64)
        data_t = kde.samples
        flags = 0 if isinstance(data_t, np.ndarray) else _lib.PKDE_DEVICE_INPUT
        gs = make_grid_struct(self.grid.lo, self.grid.hi, self.grid.h, self.grid.dims)
        rc = lib.pkde_rot_estimate(ctx, ctypes.byref(gs), self.RULES[self.rule], ptr(data_t), data_t.shape[0],
                                   ptr(dens), flags, self.stream)
        check(rc, ctx)
        if dens is not direct:
            kde.density[...] = dens.reshape(kde.density.shape)


add_estimator("rot", RoTEstimator)


def estimate_density(est, estimation_method, **kwargs):
    """estimate_density! (ParallelKDE.jl:211-226)."""
    set_nan_density(est.kde)
    cls = estimator_lookup.get(estimation_method)
    if cls is None:
        raise ArgumentError(f"Estimator {estimation_method} not registered")
    method = kwargs.pop("method", None) or "cuda"
    ensure_valid_implementation("cuda", method)
    if has_grid(est):
        kwargs["grid"] = est.grid
    inst = cls.initialize_estimator(est.kde, method=method, **kwargs)
    inst.estimate(est.kde, method=method)
    est.selected_step = getattr(inst, "selected_step", None)
