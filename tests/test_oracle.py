"""The FP64 oracle pinned against the known answers and identities of the reference's
own test suite (ParallelKDE.jl test/*.jl).  CPU only."""
import math

import numpy as np
import pytest

import _kat
from oracle.rng import bootstrap_indices


@pytest.mark.parametrize("n_dims", [1, 2, 3])
def test_dirac_known_answer(oracle, n_dims):
    """directspace_tests.jl:193-208: exact cells 51/52 and 52/53, equal corner weights."""
    grid = oracle.grid_from_steps([(-5.0, 0.1, 5.0)] * n_dims)
    data, idx = _kat.dirac_kat_inputs(n_dims)
    M, V = oracle.dirac(data, grid, idx)
    eM, eV = _kat.dirac_kat_expected(n_dims)
    # Julia's isapprox default: norm(x - y) <= sqrt(eps) * max(norm(x), norm(y))
    assert np.linalg.norm(M - eM) <= 1.5e-8 * np.linalg.norm(eM)
    assert np.linalg.norm(V - eV) <= 1.5e-8 * np.linalg.norm(eV)
    M2, V2 = oracle.dirac_numpy(data, grid, idx)
    assert np.array_equal(M, M2) and np.array_equal(V, V2)


@pytest.mark.parametrize("n_dims", [2, 3])
def test_dirac_asymmetric_corners(oracle, n_dims):
    """A sample off the cell midpoint: each corner weight is the product of the
    remainders of the opposite side (the CPU arithmetic, DirectSpace.jl:227-237)."""
    grid = oracle.grid_from_steps([(-1.0, 0.25, 1.0)] * n_dims)
    x = np.array([0.1, -0.3, 0.55, 0.7][:n_dims]).reshape(n_dims, 1)
    idx = np.array([[1]], dtype=np.int32)
    M, V = oracle.dirac(x, grid, idx)
    h = 0.25
    lo = np.floor((x[:, 0] + 1.0) / h).astype(int)
    rh = np.fmod(x[:, 0] + 1.0, h)
    rl = h - rh
    expect = np.zeros(grid.shape_c)
    for corner in np.ndindex(*(2,) * n_dims):
        w = 1.0
        cell = []
        for j in range(n_dims):
            upper = corner[j]
            w *= rh[j] if upper else rl[j]
            cell.append(lo[j] + upper)
        expect[tuple(reversed(cell))] += w / (h ** n_dims) ** 2
    assert np.allclose(M[0], expect, rtol=1e-14, atol=0)
    assert np.allclose(V[0], expect ** 2, rtol=1e-14, atol=0)
    # a full resample distributes total weight 1/prod(h) per draw
    assert math.isclose(M[0].sum(), 1.0 / h ** n_dims, rel_tol=1e-14)


def test_dirac_rejects_out_of_grid(oracle):
    """check_data, DirectSpace.jl:479-498."""
    grid = oracle.grid_from_steps([(-1.0, 0.1, 1.0)])
    for bad in (1.0, -1.0, 1.5):
        with pytest.raises(ValueError, match="beyond grid"):
            oracle.dirac(np.array([[0.0, bad]]), grid, np.array([[1, 2]], dtype=np.int32))


@pytest.mark.parametrize("n_dims", [1, 2, 3])
def test_scaled_vmr_formula(oracle, n_dims):
    """directspace_tests.jl:210-230: random complex 50^N x 5, t = 1, t0 = 0, n = 2."""
    rng = np.random.default_rng(100 + n_dims)
    shape = (5,) + (50,) * n_dims
    mk = lambda: rng.random(shape) + 1j * rng.random(shape)
    var, mean = mk(), mk()
    expect = _kat.vmr_formula(mean, var)
    got = oracle.scaled_vmr(mean, var, np.full(n_dims, 1.0), np.full(n_dims, 0.0), 2)
    fin = np.isfinite(expect)
    assert np.array_equal(fin, np.isfinite(got))
    assert np.linalg.norm(got[fin] - expect[fin]) <= 1.5e-8 * np.linalg.norm(expect[fin])


@pytest.mark.parametrize("n_dims", [1, 2, 3])
def test_full_means(oracle, n_dims):
    """directspace_tests.jl:232-245: means = |sk|."""
    rng = np.random.default_rng(7)
    a = rng.random((50,) * n_dims) + 1j * rng.random((50,) * n_dims)
    assert np.allclose(oracle.full_means(a), np.abs(a), rtol=1e-15)


@pytest.mark.parametrize("n_dims", [1, 2, 3])
@pytest.mark.parametrize("stage", _kat.STAGES)
def test_convergence_snapshots(oracle, n_dims, stage):
    """directspace_tests.jl:247-368: dlogt 0.1, eps 2, steps_low 3, steps_over 30."""
    steps_low, steps_over = 3, 30
    s = _kat.snapshot(n_dims, stage, steps_low, steps_over)
    density = np.full(s["cur"].shape, np.nan)
    means = np.ones(s["cur"].shape)
    oracle.identify_convergence(density, means, s["cur"], s["p1"], s["p2"], 0.1, 2.0, steps_low, steps_over,
                                s["minima"], s["cl"], s["co"], s["flags"])
    assert all(_kat.snapshot_expectations(stage, density, s, steps_low))


@pytest.mark.parametrize("n_dims", [1, 2])
def test_fourier_gaussian_identity(oracle, n_dims):
    """fourierspace_tests.jl:27-96: the FFT of a Gaussian KDE of bandwidth 0.2 propagated
    by t = 0.2 is the FFT of the KDE of bandwidth sqrt(2 * 0.2^2); the inverse FFT
    recovers it."""
    rng = np.random.default_rng(5)
    data = rng.standard_normal((n_dims, 100))
    grid = oracle.grid_from_steps([(-5.0, 0.1, 5.0)] * n_dims)
    axes = [grid.lo[j] + grid.h[j] * np.arange(grid.dims[j]) for j in range(n_dims)]
    d0, d02 = _kat.gaussian_kde_on_grid(data, axes, 0.2)
    M0 = oracle.fourier_statistics(d0.astype(complex)[None])
    V0 = oracle.fourier_statistics(d02.astype(complex)[None])
    assert np.allclose(M0[0], np.fft.fftn(d0), rtol=1e-12, atol=1e-12 * np.abs(M0).max())
    d1, d12 = _kat.gaussian_kde_on_grid(data, axes, math.sqrt(2 * 0.2 ** 2))
    t = np.full(n_dims, 0.2)
    Mt, Vt = oracle.propagate_statistics(M0, V0, grid, t, t)
    F1, F12 = np.fft.fftn(d1), np.fft.fftn(d12)
    assert np.linalg.norm(Mt[0] - F1) <= 1.5e-8 * np.linalg.norm(F1)
    assert np.linalg.norm(Vt[0] - F12) <= 1e-6 * np.linalg.norm(F12)
    m = np.abs(oracle.ifourier_statistics(Mt))[0]
    v = np.abs(oracle.ifourier_statistics(Vt))[0]
    assert np.linalg.norm(m - d1) <= 1.5e-8 * np.linalg.norm(d1)
    assert np.linalg.norm(v - d12) <= 1e-6 * np.linalg.norm(d12)


@pytest.mark.parametrize("n_dims", [1, 2, 3])
def test_grid_and_fftgrid(oracle, n_dims):
    """grid_tests.jl:1-36."""
    grid = oracle.grid_from_steps([(-1.0, 0.1, 1.0)] * n_dims)
    assert grid.dims == (21,) * n_dims
    assert np.all(grid.h == 0.1) and np.all(grid.lo == -1.0) and np.all(grid.hi == 1.0)
    for k in oracle.fftgrid_axes(grid):
        assert np.allclose(k, 2 * np.pi * np.fft.fftfreq(21, 0.1), rtol=1e-14)
    data = np.array([[-1.0] * n_dims, [1.0] * n_dims]).T
    g2 = oracle.find_grid(data)
    assert np.allclose(g2.lo, -1.2, rtol=0, atol=1e-15) and np.allclose(g2.hi, 1.2, rtol=0, atol=1e-15)
    assert np.allclose(oracle.initial_bandwidth(grid), 0.05)


@pytest.mark.parametrize("n_dims", [1, 2, 3])
def test_time_ladder(oracle, n_dims):
    """gradepro_tests.jl:166-177: get_time(fill(2.0), time_step=0.2)."""
    times, dt = oracle.get_time(np.full(n_dims, 2.0), time_step=0.2)
    assert np.all(times[0] == 0.0) and np.all(times[-1] == 2.0) and np.all(dt == 0.2)
    times, dt = oracle.get_time(np.full(n_dims, 1.0))
    assert times.shape == (251, n_dims)
    with pytest.raises(ValueError):
        oracle.get_time(np.full(n_dims, 1.0), time_step=2.0)


def test_duration_steps(oracle):
    """calculate_duration_steps (GradeProEstimator.jl:954-966) with the defaults."""
    assert oracle.calculate_duration_steps(np.array([1.0]), np.array([1.0 / 250]), 0.0, 0.1) == (0, 25)
    assert oracle.calculate_duration_steps(np.array([1.0, 2.0]), np.array([1.0 / 200, 2.0 / 200]), 0.06, 0.1) == (12, 20)
    assert oracle.calculate_duration_steps(np.array([1.0] * 3), np.array([1.0 / 150] * 3), 0.06, 0.1) == (9, 15)
    with pytest.raises(ValueError):
        oracle.calculate_duration_steps(np.array([1.0]), np.array([0.1]), -0.1, 0.1)


def test_dlogt_first_step_is_zero(oracle):
    t0sq = np.array([0.01, 0.04])
    assert oracle.calculate_dlogt(t0sq, np.zeros(2)) == 0.0


def test_bootstrap_generator_range():
    """kde_tests.jl:18-21: indices lie in 1:n."""
    idx = bootstrap_indices(3, 100, 2)
    assert idx.shape == (2, 100) and idx.min() >= 1 and idx.max() <= 100
    idx2 = bootstrap_indices(3, 100, 2)
    assert np.array_equal(idx, idx2)
    assert not np.array_equal(idx, bootstrap_indices(4, 100, 2))


def test_mise_1d(oracle):
    """gradepro_tests.jl:485-511 (1-D): n = 10,000 N(0,1), 300 points on [-6, 6],
    reference defaults (100 bootstraps, 251 bandwidths): MISE < 5e-5."""
    rng = np.random.default_rng(2024)
    x = rng.standard_normal((1, 10_000))
    grid = oracle.grid_from_ranges([(-6.0, 6.0, 300)])
    idx = bootstrap_indices(9, 10_000, 100)
    res = oracle.estimate_gradepro(x, grid, idx, workers=4)
    axes = [grid.lo[0] + grid.h[0] * np.arange(300)]
    truth = _kat.normal_pdf_grid(axes)
    assert _kat.mise(res.density, truth, float(grid.h[0])) < 5e-5
    assert np.all(np.isfinite(res.density))
    assert res.selected_step.min() >= 0 and res.selected_step.max() <= 251


# ------------------------------------------------------------------------- :rot
@pytest.mark.parametrize("n_dims", [1, 2])
@pytest.mark.parametrize("rule", ["silverman", "scott"])
def test_rot_mise(oracle, n_dims, rule):
    """rulesofthumb_tests.jl:96-125: 1000 N(0, I) samples, 300 points per axis on [-6, 6],
    MISE against the true density below 1e-3."""
    rng = np.random.default_rng(10 + n_dims)
    x = rng.standard_normal((n_dims, 1000))
    grid = oracle.grid_from_ranges([(-6.0, 6.0, 300)] * n_dims)
    d = oracle.estimate_rot(x, grid, rule)
    axes = np.meshgrid(*([np.linspace(-6.0, 6.0, 300)] * n_dims), indexing="ij")
    truth = np.exp(-0.5 * sum(a ** 2 for a in axes)) / (2 * np.pi) ** (n_dims / 2)
    assert d.shape == truth.shape and not np.any(np.isnan(d))
    assert _kat.mise(d, truth, float(np.prod(grid.h))) < 1e-3


def test_rot_times(oracle):
    """RoTEstimator.jl:24-49: Scott n^(-1/(N+4)), Silverman (n (N+2)/4)^(-1/(N+4)), times
    the standard deviations (divisor n - 1)."""
    rng = np.random.default_rng(3)
    x = rng.standard_normal((3, 500)) * np.array([[1.0], [2.0], [0.5]])
    sd = np.std(x, axis=1, ddof=1)
    assert np.allclose(oracle.rot_time(x, "scott"), 500 ** (-1 / 7) * sd, rtol=1e-14)
    assert np.allclose(oracle.rot_time(x, "silverman"), (500 * 5 / 4) ** (-1 / 7) * sd, rtol=1e-14)
    with pytest.raises(ValueError, match="not implemented"):
        oracle.rot_time(x, "plugin")
