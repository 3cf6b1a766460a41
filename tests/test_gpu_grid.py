"""find_grid from device-resident samples (pkde_find_grid) and the normalised density
with the FP64 sum on the GPU (pkde_normalize_density).  Needs a B200."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ndim", [1, 2, 3, 4])
def test_find_grid_on_device_equals_host(pk, ndim):
    import torch
    from pkde_b200 import raw
    rng = np.random.default_rng(ndim)
    x = rng.standard_normal((ndim, 50_000)) * rng.uniform(0.1, 30.0, size=(ndim, 1)) + rng.uniform(-5, 5, (ndim, 1))
    cases = [dict(grid_dims=(37, 64, 20, 9)[:ndim]), dict(), dict(grid_dims=(100,) * ndim, grid_padding=[0.5] * ndim),
             dict(grid_steps=[0.37, 0.5, 1.1, 2.0][:ndim])]
    dev = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()
    for kw in cases:
        host = pk.find_grid(x, **kw)
        for g in (raw.find_grid_device(np.ascontiguousarray(x.T), **kw), raw.find_grid_device(dev, device=True, **kw)):
            assert g.dims == host.dims, kw
            assert np.array_equal(g.lo, host.lo) and np.array_equal(g.hi, host.hi), kw
            assert np.array_equal(g.h, host.h), (kw, g.h, host.h)


def test_initialize_estimation_from_device_samples(pk):
    import torch
    rng = np.random.default_rng(3)
    x = rng.standard_normal((2, 5000))
    est_d = pk.initialize_estimation(torch.from_numpy(x).cuda(), grid=True, dims=(48, 40), device="cuda")
    est_h = pk.initialize_estimation(x, grid=True, dims=(48, 40), device="cuda")
    assert est_d.grid.dims == est_h.grid.dims and np.array_equal(est_d.grid.h, est_h.grid.h)
    # the estimation reads the samples from device memory, same result as from the host
    for method, kw in (("gradepro", dict(n_bootstraps=6, n_steps=15, seed=2)), ("rot", {})):
        pk.estimate_density(est_d, method, **kw)
        pk.estimate_density(est_h, method, **kw)
        assert np.array_equal(pk.get_density(est_d), pk.get_density(est_h))


def test_normalized_density(pk):
    import torch
    from pkde_b200 import raw
    rng = np.random.default_rng(4)
    x = rng.standard_normal((2, 8000))
    est = pk.initialize_estimation(x, grid=True, dims=(64, 48), device="cuda")
    pk.estimate_density(est, "gradepro", n_bootstraps=6, n_steps=20)
    d = pk.get_density(est).copy()
    dx = float(np.prod(est.grid.h))
    n = pk.get_density(est, normalize=True)
    ref = d / (np.sum(d) * dx)
    assert np.max(np.abs(n - ref)) <= 1e-14 * np.max(ref)
    assert abs(np.sum(n) * dx - 1.0) < 1e-13
    t = torch.from_numpy(d.copy()).cuda()
    raw.normalize_density(t, dx, device=True, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy(), n)
    with pytest.raises(pk.ArgumentError, match="Normalization requires"):
        raw.normalize_density(d.copy(), 0.0)
