"""The ParallelKDEpy surface over the B200 library.

ParallelKDEpy is the Python wrapper of ParallelKDE.jl that the reference's benchmark
notebook drives (paper/benchmark_time.ipynb):

    grid = pkde.Grid(dim * [(lb, hb, n_points)], device=device)
    est = pkde.DensityEstimation(data, grid=grid, device=device)   # data: n x dim
    est.estimate_density("gradepro")
    density = est.get_density()
    mesh = grid.to_meshgrid(); grid.shape

The same calls work here with ``import pkde_b200.parallelkdepy as pkde`` (device
"cuda" only; the estimators are "gradepro" and "rot", optionally spelled ":gradepro").
Arrays follow the grid's axis order: ``grid.shape == (n_1, ..., n_N)``,
``to_meshgrid()`` gives N arrays of that shape (``indexing="ij"``) and ``get_density()``
returns density[i_1, ..., i_N] at (x_1[i_1], ..., x_N[i_N]).
"""
import numpy as np

from . import api
from ._lib import ArgumentError
from .grids import initialize_grid


class Grid:
    """A uniform grid from per-axis (low, high, n_points) ranges."""

    def __init__(self, ranges, device="cuda"):
        if device != "cuda":
            raise ArgumentError("this package implements the device=:cuda path only")
        self._grid = initialize_grid([tuple(r) for r in ranges], device=device)
        self.device = device

    @property
    def shape(self):
        return tuple(self._grid.dims)

    @property
    def ndim(self):
        return self._grid.ndim

    def spacings(self):
        return self._grid.spacings()

    def bounds(self):
        return self._grid.bounds()

    def to_meshgrid(self):
        """N coordinate arrays of shape (n_1, ..., n_N)."""
        axes = [self._grid.axis_coordinates(j) for j in range(self._grid.ndim)]
        return list(np.meshgrid(*axes, indexing="ij"))


class DensityEstimation:
    """Samples (n x dim, one sample per row) and a grid; estimate_density runs an
    estimator of the library, get_density returns the density on the grid."""

    def __init__(self, data, grid=None, dims=None, device="cuda"):
        x = np.asarray(data, dtype=np.float64)
        if x.ndim == 1:
            x = x[:, None]
        if x.ndim != 2:
            raise ArgumentError("Data must be a matrix or vector.")
        g = grid._grid if isinstance(grid, Grid) else grid
        if g is None:
            self._est = api.initialize_estimation(x.T, grid=True, dims=dims, device=device)
        else:
            self._est = api.initialize_estimation(x.T, grid=g, device=device)
        self.grid = grid

    def estimate_density(self, method="gradepro", **kwargs):
        api.estimate_density(self._est, str(method).lstrip(":"), **kwargs)
        return self

    def get_density(self, normalize=False):
        d = api.get_density(self._est, normalize=normalize)
        return np.ascontiguousarray(d.T)

    @property
    def selected_step(self):
        s = self._est.selected_step
        return None if s is None else np.ascontiguousarray(s.T)
