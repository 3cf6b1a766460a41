"""The C-ABI library loads and exports every entry point include/pkde_b200.h declares;
host-only entry points behave; the host API validates arguments like the reference.
No GPU needed (no compute call is made)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "pkde_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char \*)\s*(pkde_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    import importlib.util
    spec = importlib.util.spec_from_file_location("pkde_build", os.path.join(REPO, "parallelkde.jl_b200", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build()
    import pkde_b200
    return pkde_b200.load()


def test_header_and_binding_agree():
    from pkde_b200 import _lib
    assert declared_symbols() == sorted(_lib.EXPORTED)


def test_library_exports_every_symbol(lib):
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_version_and_defaults(lib):
    from pkde_b200._lib import PkdeGradeproParams
    assert b"sm_100a" in lib.pkde_version()
    for nd, eps, alpha_s in ((1, 2.0, 0.0), (2, -0.5, 0.06)):
        p = PkdeGradeproParams()
        assert lib.pkde_gradepro_default_params(ctypes.byref(p), nd) == 0
        assert p.n_bootstraps == 100 and p.n_steps == 0 and np.isnan(p.eps) and np.isnan(p.bw_final[0])
    assert lib.pkde_gradepro_default_params(ctypes.byref(PkdeGradeproParams()), 5) == 1


def test_boot_index_matches_oracle_generator(lib):
    from oracle.rng import bootstrap_indices
    for seed, n, B in ((0, 17, 3), (12345, 1000, 2), (2**63 + 5, 999_983, 1)):
        idx = bootstrap_indices(seed, n, B, one_based=False)
        for b in range(B):
            for j in list(range(5)) + [n - 1]:
                assert lib.pkde_boot_index(seed, n, b, j) == idx[b, j]
    assert lib.pkde_boot_index(1, 0, 0, 0) == -1


def test_struct_layout_matches_header(lib):
    from pkde_b200._lib import PkdeGradeproParams, PkdeGrid
    assert ctypes.sizeof(PkdeGrid) == 8 + 4 * 8 * 4
    assert ctypes.sizeof(PkdeGradeproParams) == ctypes.sizeof(PkdeGrid) + 8 + 8 + 32 + 24


def test_host_api_validation():
    import pkde_b200 as pk
    x = np.random.default_rng(0).standard_normal((2, 50))
    with pytest.raises(pk.ArgumentError):
        pk.initialize_estimation(x, grid=True, dims=(20, 20), device="cpu")
    with pytest.raises(pk.ArgumentError):
        pk.initialize_estimation(x, grid=True, dims=(20, 20), device="tpu")
    with pytest.raises(pk.ArgumentError):
        pk.initialize_estimation(x, grid=False)
    est = pk.initialize_estimation(x, grid=True, dims=(20, 30))
    assert est.grid.dims == (20, 30) and pk.has_grid(est)
    assert np.all(np.isnan(pk.get_density(est)))
    with pytest.raises(pk.ArgumentError):
        pk.estimate_density(est, "nope")
    with pytest.raises(pk.ArgumentError):
        pk.ensure_valid_implementation("cuda", "serial")
    with pytest.raises(pk.ArgumentError):
        pk.add_estimator("gradepro", pk.GradeProEstimator)
    assert "gradepro" in pk.estimator_lookup
    est2 = pk.initialize_estimation(x, grid=False, dims=(5, 5))
    assert not pk.has_grid(est2)


def test_find_grid_and_normalisation():
    import pkde_b200 as pk
    data = np.array([[-1.0, 1.0], [-1.0, 1.0]])
    g = pk.find_grid(data, grid_dims=(11, 21))
    assert np.allclose(g.low_bounds(), -1.2) and np.allclose(g.high_bounds(), 1.2)
    assert g.dims == (11, 21) and np.allclose(g.spacings(), [2.4 / 10, 2.4 / 20])
    assert np.allclose(g.initial_bandwidth(), g.spacings() / 2)
    k = g.fftgrid()
    assert np.allclose(k[0], 2 * np.pi * np.fft.fftfreq(11, 2.4 / 10))
    # normalisation runs on the GPU (tests/test_gpu_grid.py); without a grid or dx it
    # is an ArgumentError before any device work (ParallelKDE.jl:198-199)
    est = pk.initialize_estimation(data, dims=(11, 21))
    with pytest.raises(pk.ArgumentError, match="Normalization requires"):
        pk.get_density(est, normalize=True)
    gg = pk.initialize_grid([np.linspace(-5, 5, 101)])
    assert gg.dims == (101,) and np.isclose(gg.h[0], 0.1)


def test_parallelkdepy_surface_grid():
    """The ParallelKDEpy Grid of the reference's benchmark notebook: shape in axis order,
    meshgrid with indexing "ij"."""
    import pkde_b200.parallelkdepy as pkdepy
    g = pkdepy.Grid(2 * [(-8.0, 8.0, 33)] + [(-1.0, 1.0, 5)], device="cuda")
    assert g.shape == (33, 33, 5)
    m = g.to_meshgrid()
    assert len(m) == 3 and m[0].shape == (33, 33, 5)
    assert m[0][4, 0, 0] == -8.0 + 4 * 0.5 and m[2][0, 0, 4] == 1.0
    with pytest.raises(pkdepy.ArgumentError):
        pkdepy.Grid([(-1.0, 1.0, 5)], device="cpu")
