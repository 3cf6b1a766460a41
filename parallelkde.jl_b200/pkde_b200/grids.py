"""Uniform grids, mirroring src/Grids/Grids.jl.

A grid is described by per-axis (lo, hi, n) with spacing h = (hi - lo)/(n - 1); on the
device only this descriptor exists (the reference's CuGrid materialises an N x G
coordinate array, Grids.jl:95-134; here coordinates are produced on demand).
"""
import math
from fractions import Fraction

import numpy as np

from ._lib import ArgumentError

AVAILABLE_DEVICES = ("cpu", "cuda")


def _range_step(lo, hi, n):
    """Step of Julia's ``range(lo, stop=hi, length=n)``: (hi - lo)/(n - 1) computed
    exactly and rounded once."""
    return float((Fraction(hi) - Fraction(lo)) / (n - 1))


class Grid:
    """Uniform grid on the CUDA device (Grids.jl:95-134, CuGrid)."""

    def __init__(self, lo, hi, dims, h=None, device="cuda"):
        self.lo = np.asarray(lo, dtype=np.float64).reshape(-1)
        self.hi = np.asarray(hi, dtype=np.float64).reshape(-1)
        self.dims = tuple(int(d) for d in dims)
        if not (len(self.lo) == len(self.hi) == len(self.dims)):
            raise ArgumentError("Elements of ranges must implement 'step' method.")
        if h is None:
            h = [_range_step(a, b, n) for a, b, n in zip(self.lo, self.hi, self.dims)]
        self.h = np.asarray(h, dtype=np.float64).reshape(-1)
        self.device = device

    # Grids.jl:141-217
    @property
    def ndim(self):
        return len(self.dims)

    @property
    def size(self):
        return self.dims

    def __len__(self):
        return int(np.prod(self.dims))

    def spacings(self):
        return self.h.copy()

    def bounds(self):
        """2 x N matrix [low; high] (Grids.jl:196)."""
        return np.stack([self.lo, self.hi])

    def low_bounds(self):
        return self.lo.copy()

    def high_bounds(self):
        return self.hi.copy()

    def initial_bandwidth(self):
        """Half the spacing per axis (Grids.jl:217)."""
        return self.h / 2

    def axis_coordinates(self, j):
        n = self.dims[j]
        return self.lo[j] + self.h[j] * np.arange(n, dtype=np.float64)

    def get_coordinates(self):
        """N x n_1 x ... x n_N coordinate array, column-major like the reference
        (returned as a C-ordered array of shape (N, n_N, ..., n_1))."""
        axes = [self.axis_coordinates(j) for j in range(self.ndim)]
        mesh = np.meshgrid(*reversed(axes), indexing="ij")
        return np.stack(list(reversed(mesh)))

    def fftgrid(self):
        """Per-axis 2 pi fftfreq(n, 1/h) (Grids.jl:225-238)."""
        out = []
        for n, h in zip(self.dims, self.h):
            mult = (2 * math.pi) * ((1.0 / h) / n)
            m = np.arange(n, dtype=np.float64)
            m[(n - 1) // 2 + 1:] -= n
            out.append(m * mult)
        return out

    def __repr__(self):
        return f"Grid(dims={self.dims}, lo={self.lo.tolist()}, hi={self.hi.tolist()}, device={self.device!r})"


def _check_device(device):
    if device not in AVAILABLE_DEVICES:
        raise ArgumentError(f"Invalid device: {device}")


def initialize_grid(ranges, device="cuda"):
    """Grids.jl:38-50.  ``ranges``: per axis a (lo, hi, n) tuple or a uniform 1-D array."""
    _check_device(device)
    if device != "cuda":
        raise ArgumentError("this package implements the device=:cuda path only")
    lo, hi, dims, hs = [], [], [], []
    for r in ranges:
        if isinstance(r, tuple) and len(r) == 3:
            a, b, n = float(r[0]), float(r[1]), int(r[2])
            lo.append(a), hi.append(b), dims.append(n), hs.append(_range_step(a, b, n))
        else:
            v = np.asarray(r, dtype=np.float64)
            if v.ndim != 1 or v.size < 2:
                raise ArgumentError("Elements of ranges must implement 'step' method.")
            d = np.diff(v)
            if not np.allclose(d, d[0], rtol=1e-9, atol=0):
                raise ArgumentError("Elements of ranges must implement 'step' method.")
            lo.append(v[0]), hi.append(v[-1]), dims.append(v.size), hs.append(_range_step(v[0], v[-1], v.size))
    return Grid(lo, hi, dims, hs, device)


def find_grid(data, grid_bounds=None, grid_dims=None, grid_steps=None, grid_padding=None, device="cuda"):
    """Grids.jl:252-300.  data: N x n array (one column per sample)."""
    data = np.asarray(data, dtype=np.float64)
    if data.ndim == 1:
        data = data.reshape(1, -1)
    ndim = data.shape[0]
    if grid_bounds is None:
        grid_bounds = [(float(row.min()), float(row.max())) for row in data]
    if grid_padding is None:
        grid_padding = [0.1 * abs(b[1] - b[0]) for b in grid_bounds]
    bounds = [(b[0] - p, b[1] + p) for b, p in zip(grid_bounds, grid_padding)]
    if grid_steps is None and grid_dims is None:
        grid_dims = tuple(150 for _ in range(ndim))
    if grid_dims is not None:
        return initialize_grid([(b[0], b[1], int(n)) for b, n in zip(bounds, grid_dims)], device=device)
    ranges = []
    for b, s in zip(bounds, grid_steps):
        n = int(math.floor((b[1] - b[0]) / s)) + 1
        ranges.append((b[0], b[0] + (n - 1) * s, n))
    return initialize_grid(ranges, device=device)
