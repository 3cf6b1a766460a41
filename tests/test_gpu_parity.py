"""Parity of the CUDA path (through the C ABI) with the FP64 oracle and the reference's
known answers.  Needs a B200 and the built library."""
import math

import numpy as np
import pytest

import _kat
from oracle.rng import bootstrap_indices

pytestmark = pytest.mark.gpu


def _grid_pk(pk, og_grid):
    return pk.Grid(og_grid.lo, og_grid.hi, og_grid.dims, og_grid.h)


def _lower_cell_counts(oracle, data, grid, idx):
    """Exact draws per lower cell (NumPy restatement of DirectSpace.jl:219-221)."""
    N = grid.ndim
    out = np.zeros((idx.shape[0], grid.size), dtype=np.uint32)
    stride = np.cumprod([1] + list(grid.dims[:-1]))
    for b in range(idx.shape[0]):
        x = data[:, idx[b] - 1]
        il = np.floor((x - grid.lo[:, None]) / grid.h[:, None]).astype(np.int64)
        cell = (il * stride[:, None]).sum(axis=0)
        out[b] = np.bincount(cell, minlength=grid.size).astype(np.uint32)
    return out.reshape((idx.shape[0],) + grid.shape_c)


@pytest.mark.parametrize("n_dims", [1, 2, 3])
def test_dirac_known_answer(pk, oracle, n_dims):
    """directspace_tests.jl:374-389 (GPU): the same cells and weights as on the CPU."""
    from pkde_b200 import raw
    og_grid = oracle.grid_from_steps([(-5.0, 0.1, 5.0)] * n_dims)
    data, idx = _kat.dirac_kat_inputs(n_dims)
    M, V, C = raw.dirac_sequence(_grid_pk(pk, og_grid), data, idx)
    eM, eV = _kat.dirac_kat_expected(n_dims)
    assert np.linalg.norm(M - eM) <= 1e-13 * np.linalg.norm(eM)
    assert np.linalg.norm(V - eV) <= 1e-13 * np.linalg.norm(eV)
    oM, oV = oracle.dirac(data, og_grid, idx)
    assert np.max(np.abs(M - oM)) <= 1e-14 * np.max(oM)
    assert int(C.sum()) == 4


@pytest.mark.parametrize("n_dims,dims,n,B", [(1, (257,), 5000, 6), (2, (40, 33), 20000, 5), (3, (17, 12, 20), 8000, 4),
                                            (4, (7, 9, 6, 8), 3000, 3)])
def test_dirac_counts_bit_exact(pk, oracle, n_dims, dims, n, B):
    """Random samples and explicit draws: integer counts per cell bit-exact, weights within
    fixed-point rounding of the FP64 oracle (<= 1e-14 of the largest cell)."""
    from pkde_b200 import raw
    rng = np.random.default_rng(n_dims)
    data = rng.standard_normal((n_dims, n))
    og_grid = oracle.find_grid(data, grid_dims=dims)
    idx = bootstrap_indices(77, n, B)
    M, V, C = raw.dirac_sequence(_grid_pk(pk, og_grid), data, idx)
    oM, oV = oracle.dirac(data, og_grid, idx)
    assert np.array_equal(C, _lower_cell_counts(oracle, data, og_grid, idx))
    assert np.max(np.abs(M - oM)) <= 1e-14 * np.max(oM)
    assert np.max(np.abs(V - oV)) <= 1e-14 * np.max(oV)
    # seeded draws on the device == the oracle's generator
    M2, V2, C2 = raw.dirac_sequence(_grid_pk(pk, og_grid), data, None, n_bootstraps=B, seed=77)
    assert np.array_equal(C2, C) and np.array_equal(M2, M) and np.array_equal(V2, V)
    # identity resample (B = 0)
    Mi, _, Ci = raw.dirac_sequence(_grid_pk(pk, og_grid), data, None, n_bootstraps=0)
    oMi, _ = oracle.dirac(data, og_grid, np.arange(1, n + 1, dtype=np.int32)[None], include_var=False)
    assert np.max(np.abs(Mi - oMi)) <= 1e-14 * np.max(oMi) and int(Ci.sum()) == n


def test_dirac_rejects_out_of_grid(pk, oracle):
    from pkde_b200 import raw
    g = _grid_pk(pk, oracle.grid_from_steps([(-1.0, 0.1, 1.0)]))
    for bad in (1.0, -1.0, 7.0):
        with pytest.raises(pk.ArgumentError, match="beyond grid"):
            raw.dirac_sequence(g, np.array([[0.0, bad]]), np.array([[1, 2]], dtype=np.int32))
    with pytest.raises(pk.ArgumentError):
        raw.dirac_sequence(g, np.array([[0.0, 0.5]]), np.array([[1, 3]], dtype=np.int32))


@pytest.mark.parametrize("shape", [(3, 1024), (2, 101), (2, 21, 21), (1, 48, 40), (2, 12, 30, 7), (1, 5, 6, 7, 8),
                                   (1, 4096), (1, 512, 512), (1, 96, 80, 48)])
def test_fft_matches_numpy(pk, shape):
    from pkde_b200 import raw
    rng = np.random.default_rng(len(shape))
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    axes = tuple(range(1, len(shape)))
    fwd = raw.fft(x, -1)
    ref = np.fft.fftn(x, axes=axes)
    assert np.linalg.norm(fwd - ref) <= 1e-14 * math.log2(x[0].size + 1) * np.linalg.norm(ref)
    inv = raw.fft(ref, +1)
    assert np.linalg.norm(inv - x) <= 1e-14 * math.log2(x[0].size + 1) * np.linalg.norm(x)


@pytest.mark.parametrize("n_dims", [1, 2, 3])
def test_scaled_vmr(pk, oracle, n_dims):
    """directspace_tests.jl:391-415 (GPU): random complex 50^N x 5, t = 1, t0 = 0, n = 2."""
    from pkde_b200 import raw
    rng = np.random.default_rng(200 + n_dims)
    shape = (5,) + (50,) * n_dims
    var = rng.random(shape) + 1j * rng.random(shape)
    mean = rng.random(shape) + 1j * rng.random(shape)
    got = raw.scaled_vmr(mean, var, np.full(n_dims, 1.0), np.full(n_dims, 0.0), 2)
    want = oracle.scaled_vmr(mean, var, np.full(n_dims, 1.0), np.full(n_dims, 0.0), 2)
    fin = np.isfinite(want)
    assert np.array_equal(fin, np.isfinite(got))
    assert np.max(np.abs(got[fin] - want[fin])) <= 1e-13 * np.max(np.abs(want[fin]))
    assert np.linalg.norm(got[fin] - _kat.vmr_formula(mean, var)[fin]) <= 1.5e-8 * np.linalg.norm(want[fin])


@pytest.mark.parametrize("n_dims", [1, 2, 3])
@pytest.mark.parametrize("stage", _kat.STAGES)
def test_convergence_snapshots(pk, n_dims, stage):
    """directspace_tests.jl:433-554 (GPU snapshots), FP64 on the device."""
    from pkde_b200 import raw
    steps_low, steps_over = 3, 30
    s = _kat.snapshot(n_dims, stage, steps_low, steps_over)
    density = np.full(s["cur"].shape, np.nan)
    means = np.ones(s["cur"].shape)
    raw.identify_convergence(density.reshape(-1), means.reshape(-1), s["cur"].reshape(-1), s["p1"].reshape(-1),
                             s["p2"].reshape(-1), 0.1, 2.0, steps_low, steps_over, s["minima"].reshape(-1),
                             s["cl"].reshape(-1), s["co"].reshape(-1), s["flags"].reshape(-1))
    assert all(_kat.snapshot_expectations(stage, density, s, steps_low))


class Parity:
    """GPU result vs the reference-faithful oracle run (fft_mode c2c).  A second oracle run
    with different FP64 rounding (fft_mode r2c) marks the grid points whose reference
    outcome is set by rounding noise; parity is asserted exactly on the others."""

    def __init__(self, est, ref, alt, density):
        self.stable = ref.selected_step == alt.selected_step
        self.sel = est.selected_step
        self.rel = float(np.linalg.norm(density - ref.density) / np.linalg.norm(ref.density))
        self.rel_alt = float(np.linalg.norm(alt.density - ref.density) / np.linalg.norm(ref.density))
        self.agree = float(np.mean(self.sel == ref.selected_step))
        self.agree_alt = float(np.mean(self.stable))
        st = self.stable
        self.agree_stable = float(np.mean(self.sel[st] == ref.selected_step[st]))
        both = st & (self.sel == ref.selected_step)
        self.rel_stable = float(np.linalg.norm(density[both] - ref.density[both]) / np.linalg.norm(ref.density[both]))
        self.flips = int(np.sum(self.sel != ref.selected_step))
        self.flips_alt = int(np.sum(~st))

    def report(self, tag):
        print(f"{tag}: rel L2 {self.rel:.2e} (oracle r2c vs c2c {self.rel_alt:.2e}); selected agree {self.agree:.5f} "
              f"(oracle r2c vs c2c {self.agree_alt:.5f}); on rounding-stable points agree {self.agree_stable:.6f}, "
              f"rel L2 {self.rel_stable:.2e}")

    def check(self):
        G = self.sel.size
        # identical densities wherever the selected step agrees (FP64 round-off only)
        assert self.rel_stable <= 1e-10
        # the GPU flips no more decisions than a second FP64 implementation of the
        # reference does (decisions within round-off of the threshold are coin flips)
        assert self.flips <= 1.5 * self.flips_alt + 0.001 * G + 2
        assert self.agree_stable >= 1.0 - 3.0 * (1.0 - self.agree_alt) - 0.001


def _compare(pk, oracle, data, og_grid, B, n_steps=None, idx_seed=5, **kw):
    idx = bootstrap_indices(idx_seed, data.shape[1], B)
    est = pk.initialize_estimation(data, grid=_grid_pk(pk, og_grid))
    pk.estimate_density(est, "gradepro", n_bootstraps=B, n_steps=n_steps, bootstrap_idxs=idx, **kw)
    ref = oracle.estimate_gradepro(data, og_grid, idx, n_steps=n_steps, workers=4, **kw)
    alt = oracle.estimate_gradepro(data, og_grid, idx, n_steps=n_steps, workers=4, fft_mode="r2c", **kw)
    par = Parity(est, ref, alt, pk.get_density(est))
    par.report(f"N={og_grid.ndim} dims={og_grid.dims} B={B}")
    return par


@pytest.mark.parametrize("n_dims,dims,n,B,steps", [(1, (256,), 4000, 10, 60), (2, (48, 40), 20000, 8, 50),
                                                   (3, (16, 20, 12), 20000, 6, 30), (4, (8, 6, 10, 7), 20000, 4, 20),
                                                   (2, (64, 32), 20000, 8, 40), (2, (256, 128), 50000, 5, 30),
                                                   (3, (16, 32, 16), 20000, 6, 30), (2, (2048, 16), 20000, 4, 20),
                                                   (4, (16, 16, 16, 16), 30000, 4, 12),
                                                   # mixed-radix engine tiles (N = 3 or 5 times a power of two)
                                                   (2, (96, 80), 30000, 6, 30), (2, (24, 320), 20000, 4, 20),
                                                   (3, (48, 40, 24), 30000, 4, 15), (2, (384, 192), 40000, 4, 12)])
def test_estimate_matches_oracle(pk, oracle, n_dims, dims, n, B, steps):
    rng = np.random.default_rng(10 + n_dims)
    data = rng.standard_normal((n_dims, n))
    og_grid = oracle.find_grid(data, grid_dims=dims)
    _compare(pk, oracle, data, og_grid, B, steps).check()


def test_estimate_odd_bootstraps_and_prime_grid(pk, oracle):
    rng = np.random.default_rng(3)
    data = rng.standard_normal((2, 5000))
    og_grid = oracle.find_grid(data, grid_dims=(21, 101))
    _compare(pk, oracle, data, og_grid, 5, 30).check()


def test_estimate_kwargs(pk, oracle):
    """bw_step / bw_final / alpha / eps keyword arguments reach the ladder."""
    rng = np.random.default_rng(4)
    data = rng.standard_normal((2, 4000))
    og_grid = oracle.find_grid(data, grid_dims=(32, 36))
    _compare(pk, oracle, data, og_grid, 6, None, bw_step=0.01, bw_final=0.3, alpha_s=0.1, alpha_os=0.2,
             eps=-0.3).check()
    with pytest.raises(pk.ArgumentError, match="Invalid time step"):
        est2 = pk.initialize_estimation(data, grid=_grid_pk(pk, og_grid))
        pk.estimate_density(est2, "gradepro", n_bootstraps=4, bw_step=1.0, bw_final=0.3)


def test_estimate_errors(pk, oracle):
    rng = np.random.default_rng(0)
    data = rng.standard_normal((1, 500))
    g = pk.Grid([-1.0], [1.0], (64,))
    est = pk.initialize_estimation(data, grid=g)
    with pytest.raises(pk.ArgumentError, match="beyond grid"):
        pk.estimate_density(est, "gradepro", n_bootstraps=4, n_steps=10)
    g2 = pk.find_grid(data, grid_dims=(64,))
    est = pk.initialize_estimation(data, grid=g2)
    with pytest.raises(pk.ArgumentError):
        pk.estimate_density(est, "gradepro", n_bootstraps=1, n_steps=10)
    with pytest.raises(pk.ArgumentError):
        pk.estimate_density(est, "gradepro", method="serial")


def test_estimate_deterministic(pk):
    rng = np.random.default_rng(1)
    data = rng.standard_normal((2, 30000))
    outs = []
    for _ in range(2):
        est = pk.initialize_estimation(data, grid=True, dims=(64, 48))
        pk.estimate_density(est, "gradepro", n_bootstraps=6, n_steps=40, seed=123)
        outs.append((pk.get_density(est).copy(), est.selected_step.copy()))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("n_dims", [1, 2])
def test_mise(pk, n_dims):
    """gradepro_tests.jl:513-540 (GPU): n = 10,000 N(0, I), 300 points per axis on
    [-6, 6], reference defaults; MISE < 5e-5."""
    rng = np.random.default_rng(2024 + n_dims)
    data = rng.standard_normal((n_dims, 10_000))
    g = pk.initialize_grid([(-6.0, 6.0, 300)] * n_dims)
    est = pk.initialize_estimation(data, grid=g)
    pk.estimate_density(est, "gradepro", seed=9)
    axes = [g.axis_coordinates(j) for j in range(n_dims)]
    truth = _kat.normal_pdf_grid(axes)
    m = _kat.mise(pk.get_density(est), truth, float(np.prod(g.h)))
    print(f"MISE {n_dims}-D: {m:.3e}")
    assert m < 5e-5
