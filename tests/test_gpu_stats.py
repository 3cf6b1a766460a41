"""Launch accounting and the profiling levels of pkde_set_profiling, and the public API
writing into a page-locked density.  Needs a B200."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _estimate(pk, level):
    from pkde_b200 import _lib, raw
    rng = np.random.default_rng(11)
    x = np.ascontiguousarray(rng.standard_normal((3000, 2)))
    grid = pk.find_grid(x.T, grid_dims=(64, 48))
    d, s = np.empty(64 * 48), np.empty(64 * 48, dtype=np.int32)
    _lib.get_stats(0, reset=True)
    _lib.set_profiling(level, 0)
    try:
        raw.gradepro_host(grid, x, d, s, seed=3, n_bootstraps=8, n_steps=20)
    finally:
        _lib.set_profiling(_lib.PKDE_PROFILE_OFF, 0)
    return _lib.get_stats(0, reset=True), d


def test_profiling_levels(pk):
    from pkde_b200 import _lib
    _estimate(pk, _lib.PKDE_PROFILE_OFF)  # the first call of a shape runs the autotuner's trials
    full, d_full = _estimate(pk, _lib.PKDE_PROFILE_ALL)
    steps, d_steps = _estimate(pk, _lib.PKDE_PROFILE_STEPS)
    off, d_off = _estimate(pk, _lib.PKDE_PROFILE_OFF)
    # timing never changes results, and launch counts are kept at every level
    assert np.array_equal(d_full, d_steps) and np.array_equal(d_full, d_off)
    assert full["launches"] == steps["launches"] == off["launches"] > 0
    assert full["phase_ms"]["binning"] > 0 and full["phase_ms"]["step_vmr"] > 0
    assert steps["phase_ms"]["binning"] == 0 and steps["phase_ms"]["forward_fft"] == 0
    assert steps["phase_ms"]["step_vmr"] > 0
    assert all(v == 0 for v in off["phase_ms"].values())


def test_profiling_level_out_of_range(pk):
    from pkde_b200 import _lib
    with pytest.raises(pk.ArgumentError):
        _lib.set_profiling(3, 0)


def test_api_writes_pinned_density(pk):
    """pin() moves the samples and the density to page-locked memory; estimate_density
    writes the density in place, with the same values as without pin()."""
    rng = np.random.default_rng(5)
    x = rng.standard_normal((2, 4000))
    a = pk.initialize_estimation(x, grid=True, dims=(40, 56), device="cuda")
    b = pk.initialize_estimation(x, grid=True, dims=(40, 56), device="cuda")
    b.kde.pin()
    before = b.kde.density
    for est in (a, b):
        pk.estimate_density(est, "gradepro", n_bootstraps=6, n_steps=12, seed=4)
    assert pk.get_density(b) is before
    assert np.array_equal(pk.get_density(a), pk.get_density(b))
    assert np.array_equal(a.selected_step, b.selected_step)
