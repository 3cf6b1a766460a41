"""Edge cases of the :gradepro path against the FP64 oracle: the smallest sample and
bootstrap counts, the smallest grids, the longest lines each tile path takes, grids whose
axes fall to different tile paths, and the plain form on the same inputs.  Needs a B200."""
import numpy as np
import pytest

from test_gpu_parity import _compare

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_dims,dims,n,B,steps", [
    (1, (8,), 2, 2, 5),            # two samples, two bootstraps, a tiny 1-D grid (launch path)
    (2, (2, 2), 5, 2, 4),          # the smallest 2-D grid (2 points per axis)
    (2, (3, 5), 40, 3, 6),         # odd bootstrap count, prime axes (generic radix)
    (3, (2, 3, 4), 60, 2, 5),      # tiny 3-D
    (1, (4096,), 3000, 4, 10),     # longest 1-D line of the step-parallel path
    (2, (2048, 8), 5000, 3, 8),    # longest register-tile axis 1
    (2, (16, 768), 4000, 2, 8),    # longest mixed-radix axis (3 * 256) as a column axis
    (2, (640, 16), 4000, 2, 8),    # 5 * 128 as axis 1 (final pass)
    (2, (17, 4096), 3000, 2, 6),   # axis longer than the engine takes: launch path
    (3, (16, 48, 8), 6000, 3, 8),  # register, mixed-radix and generic axes in one grid
])
def test_edge_shapes_match_oracle(pk, oracle, n_dims, dims, n, B, steps):
    rng = np.random.default_rng(sum(dims) + n)
    data = rng.standard_normal((n_dims, n))
    og_grid = oracle.find_grid(data, grid_dims=dims)
    par = _compare(pk, oracle, data, og_grid, B, n_steps=steps)
    par.check()


def test_bw_step_ladder_and_explicit_bandwidth(pk, oracle):
    """bw_step / bw_final keyword paths (GradeProEstimator.jl:860-905) on an engine shape."""
    rng = np.random.default_rng(3)
    data = rng.standard_normal((2, 8000))
    og_grid = oracle.find_grid(data, grid_dims=(64, 48))
    _compare(pk, oracle, data, og_grid, 4, n_steps=None, bw_step=0.02, bw_final=[0.3, 0.25]).check()


def test_plain_form_on_edge_shapes(pk, oracle):
    """The launch-per-step form and the engine on shapes that take different tile paths:
    identical densities to FP64 round-off wherever the selected steps agree, and no more
    disagreement in the selected steps than between two FP64 implementations of the
    reference (the oracle with complex and with real-input transforms) on the same draws:
    on sparse grids many decisions sit within round-off of the threshold."""
    from pkde_b200 import _lib, raw
    from oracle.rng import bootstrap_indices
    rng = np.random.default_rng(9)
    for dims in ((16, 768), (640, 16), (16, 48, 8)):
        x = rng.standard_normal((len(dims), 20000))
        og_grid = oracle.find_grid(x, grid_dims=dims)
        grid = pk.Grid(og_grid.lo, og_grid.hi, og_grid.dims, og_grid.h)
        idx = bootstrap_indices(4, x.shape[1], 8)
        G = int(np.prod(dims))
        out = []
        for path in (_lib.PKDE_STEPS_AUTO, _lib.PKDE_STEPS_PER_STEP_LAUNCH):
            _lib.set_step_path(path)
            try:
                d, s = np.empty(G), np.empty(G, dtype=np.int32)
                raw.gradepro_host(grid, np.ascontiguousarray(x.T), d, s, idx=idx, n_bootstraps=8, n_steps=10)
            finally:
                _lib.set_step_path(_lib.PKDE_STEPS_AUTO)
            out.append((d, s))
        ref = oracle.estimate_gradepro(x, og_grid, idx, n_steps=10, workers=4)
        alt = oracle.estimate_gradepro(x, og_grid, idx, n_steps=10, workers=4, fft_mode="r2c")
        flips_oracle = int(np.sum(np.asarray(ref.selected_step).reshape(-1) != np.asarray(alt.selected_step).reshape(-1)))
        same = out[0][1] == out[1][1]
        assert int(np.sum(~same)) <= 1.5 * flips_oracle + 0.001 * G + 2, (dims, int(np.sum(~same)), flips_oracle)
        assert np.linalg.norm((out[0][0] - out[1][0])[same]) <= 1e-10 * np.linalg.norm(out[1][0][same])
