"""Known-answer cases restated from the reference's own test suite (shared by the oracle
tests and the GPU parity tests).  Citations are file:line in ParallelKDE.jl."""
import math

import numpy as np


def dirac_kat_expected(n_dims):
    """test/directspace_tests.jl:1-41 (calculate_test_sequences): samples at 0.05 and
    0.15 on -5:0.1:5 per axis, bootstrap matrix [1 2; 2 1].  Returns (M, V) of C-order
    shape (2, 101, ..., 101)."""
    spacing_squared = (0.1 ** n_dims) ** 2
    shape = (2,) + (101,) * n_dims
    M = np.zeros(shape)
    V = np.zeros(shape)
    for lo_idx in (51, 52):  # 1-based lower index of sample 1 and sample 2
        term = (0.05 ** n_dims) / (2 * spacing_squared)
        for corner in np.ndindex(*(2,) * n_dims):
            cell = tuple(lo_idx - 1 + c for c in reversed(corner))
            for b in range(2):
                M[(b,) + cell] += term
                V[(b,) + cell] += term ** 2
    return M, V


def dirac_kat_inputs(n_dims):
    data = np.array([[0.05] * n_dims, [0.15] * n_dims]).T  # N x 2
    idx = np.array([[1, 2], [2, 1]], dtype=np.int32)  # (B, n): bootstrap 1 = (1, 2), 2 = (2, 1)
    return data, idx


def vmr_formula(test_mean, test_var, time_final=1.0, time_initial=0.0, n_samples=2):
    """test/directspace_tests.jl:47-61 (calculate_test_vmr); arrays (B, ...)."""
    n_dims = test_mean.ndim - 1
    means = np.abs(test_mean) / n_samples
    var = np.abs(test_var) / n_samples - means ** 2
    vmr = var / means
    scaling = (time_final ** 2 + time_initial ** 2) ** n_dims
    scaling = scaling ** 1.5 * n_samples ** 3
    v = scaling * np.var(vmr, axis=0, ddof=1)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(np.isfinite(v), np.log(np.where(np.isfinite(v), v, 1.0)), np.nan)


def snapshot(n_dims, stage, steps_low, steps_over):
    """test/directspace_tests.jl:69-129 (make_snapshot, CPU)."""
    shape = (101,) * n_dims
    f = lambda v: np.full(shape, v, dtype=np.float64)
    if stage == "low_density_recon":
        s = dict(cur=f(1.0e6), p1=f(0.8), p2=f(1.0e6), minima=np.zeros(shape), cl=np.full(shape, steps_low, np.uint16),
                 co=np.zeros(shape, np.uint16), flags=np.zeros(shape, bool))
    elif stage == "low_density_stop":
        s = dict(cur=f(1.0), p1=f(0.99), p2=f(1.0), minima=f(np.nan), cl=np.full(shape, steps_low + 1, np.uint16),
                 co=np.zeros(shape, np.uint16), flags=np.ones(shape, bool))
    elif stage == "high_density_update":
        s = dict(cur=f(1.00005), p1=f(1.0), p2=f(1.00005), minima=np.zeros(shape), cl=np.zeros(shape, np.uint16),
                 co=np.zeros(shape, np.uint16), flags=np.zeros(shape, bool))
    elif stage == "high_density_noupdate":
        s = dict(cur=f(1.01), p1=f(1.0), p2=f(1.01), minima=f(-5.0), cl=np.zeros(shape, np.uint16),
                 co=np.zeros(shape, np.uint16), flags=np.zeros(shape, bool))
    else:
        raise ValueError(stage)
    return s


def snapshot_expectations(stage, density, s, steps_low):
    """The assertions of test/directspace_tests.jl:276-367."""
    if stage == "low_density_recon":
        return [np.all(np.isnan(density)), np.all(np.isnan(s["minima"])), np.all(s["cl"] == steps_low + 1),
                np.all(s["co"] == 0), np.all(s["flags"])]
    if stage == "low_density_stop":
        return [np.all(density == 1), not np.any(s["minima"] == 0), np.all(s["cl"] == steps_low + 1),
                np.all(s["co"] == 0), np.all(s["flags"])]
    if stage == "high_density_update":
        return [np.all(density == 1), np.all(s["minima"] <= 0), np.all(s["cl"] == 0), np.all(s["co"] == 0),
                not np.any(s["flags"])]
    if stage == "high_density_noupdate":
        return [np.all(np.isnan(density)), np.all(s["minima"] == -5.0), np.all(s["cl"] == 0), np.all(s["co"] == 1),
                not np.any(s["flags"])]
    raise ValueError(stage)


STAGES = ["low_density_recon", "low_density_stop", "high_density_update", "high_density_noupdate"]


def gaussian_kde_on_grid(data, axes, bw):
    """test/fourierspace_tests.jl:1-25 (initialize_density): sum of isotropic normal pdfs
    of std ``bw`` divided by n, and the sum of their squares.  axes: per-axis coordinates
    (axis 1 first); returns C-order arrays (n_N, ..., n_1)."""
    n = data.shape[1]
    N = data.shape[0]
    dens = 0.0
    dens2 = 0.0
    mesh = np.meshgrid(*reversed(axes), indexing="ij")
    coords = list(reversed(mesh))
    norm = (2 * math.pi * bw * bw) ** (-N / 2)
    for i in range(n):
        r2 = 0.0
        for j in range(N):
            r2 = r2 + (coords[j] - data[j, i]) ** 2
        k = norm * np.exp(-0.5 * r2 / (bw * bw)) / n
        dens = dens + k
        dens2 = dens2 + k * k
    return dens, dens2


def normal_pdf_grid(axes):
    mesh = np.meshgrid(*reversed(axes), indexing="ij")
    r2 = sum(m * m for m in mesh)
    return (2 * math.pi) ** (-len(axes) / 2) * np.exp(-0.5 * r2)


def mise(f1, f2, dx):
    """test/test_utils.jl:24-28."""
    return float(np.sum((f1 - f2) ** 2) * dx / f1.size)
