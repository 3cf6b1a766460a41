"""The :rot estimator on the device (pkde_rot_estimate) against the FP64 oracle's
restatement of RoTEstimator.jl, and the reference's own acceptance test through the
host API.  Needs a B200."""
import numpy as np
import pytest

import _kat

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,n", [((300,), 1000), ((256,), 5000), ((64, 48), 20000), ((17, 12, 20), 8000),
                                    ((8, 6, 10, 7), 3000)])
@pytest.mark.parametrize("rule", ["scott", "silverman"])
def test_rot_matches_oracle(pk, oracle, dims, n, rule):
    from pkde_b200 import raw
    rng = np.random.default_rng(len(dims) * 7 + n)
    x = rng.standard_normal((len(dims), n))
    og_grid = oracle.find_grid(x, grid_dims=dims)
    grid = pk.Grid(og_grid.lo, og_grid.hi, og_grid.dims, og_grid.h)
    d = raw.rot(grid, np.ascontiguousarray(x.T), rule)
    ref = oracle.estimate_rot(x, og_grid, rule).reshape(-1)
    assert np.max(np.abs(d - ref)) <= 1e-12 * np.max(ref)


@pytest.mark.parametrize("n_dims", [1, 2])
@pytest.mark.parametrize("rule", ["silverman", "scott"])
def test_rot_api_mise(pk, oracle, n_dims, rule):
    """rulesofthumb_tests.jl:127-155 (GPU): MISE < 1e-3 on N(0, I) through
    initialize_estimation / estimate_density(:rot) / get_density."""
    rng = np.random.default_rng(40 + n_dims)
    x = rng.standard_normal((n_dims, 1000))
    est = pk.initialize_estimation(x, grid=True, grid_ranges=[(-6.0, 6.0, 300)] * n_dims, device="cuda")
    pk.estimate_density(est, "rot", rule_of_thumb=rule)
    d = pk.get_density(est)
    axes = np.meshgrid(*([np.linspace(-6.0, 6.0, 300)] * n_dims), indexing="ij")
    truth = np.exp(-0.5 * sum(a ** 2 for a in axes)) / (2 * np.pi) ** (n_dims / 2)
    assert not np.any(np.isnan(d))
    assert _kat.mise(d, truth, float(np.prod(est.grid.h))) < 1e-3


def test_rot_errors_and_device_pointers(pk, oracle):
    import torch
    from pkde_b200 import raw
    rng = np.random.default_rng(1)
    x = rng.standard_normal((2, 4000))
    og_grid = oracle.find_grid(x, grid_dims=(32, 40))
    grid = pk.Grid(og_grid.lo, og_grid.hi, og_grid.dims, og_grid.h)
    with pytest.raises(pk.ArgumentError, match="not implemented"):
        raw.rot(grid, np.ascontiguousarray(x.T), "plugin")
    est = pk.initialize_estimation(x, grid=grid, device="cuda")
    with pytest.raises(pk.ArgumentError, match="not implemented"):
        pk.estimate_density(est, "rot", rule_of_thumb="plugin")
    bad = np.ascontiguousarray(x.T).copy()
    bad[5, 1] = og_grid.hi[1] + 1.0
    with pytest.raises(pk.ArgumentError, match="beyond grid"):
        raw.rot(grid, bad, "scott")
    host = raw.rot(grid, np.ascontiguousarray(x.T), "scott")
    dd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()
    out = torch.empty(host.shape, dtype=torch.float64, device="cuda")
    raw.rot(grid, dd, "scott", density=out, device=True, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), host)


def test_parallelkdepy_surface_estimates(pk):
    """paper/benchmark_time.ipynb's ParallelKDE class: Grid, DensityEstimation(data n x
    dim), estimate_density(method), get_density() -- same numbers as the main API."""
    import pkde_b200.parallelkdepy as pkdepy
    rng = np.random.default_rng(5)
    data = rng.standard_normal((3000, 2))
    grid = pkdepy.Grid(2 * [(-8.0, 8.0, 64)], device="cuda")
    for method in ("gradepro", ":rot"):
        est = pkdepy.DensityEstimation(data, grid=grid, device="cuda")
        kw = dict(n_bootstraps=8, n_steps=20) if method == "gradepro" else {}
        est.estimate_density(method, **kw)
        d = est.get_density()
        assert d.shape == grid.shape
        ref = pk.initialize_estimation(data.T, grid=True, grid_ranges=2 * [(-8.0, 8.0, 64)], device="cuda")
        pk.estimate_density(ref, method.lstrip(":"), **kw)
        assert np.array_equal(d, pk.get_density(ref).T)
