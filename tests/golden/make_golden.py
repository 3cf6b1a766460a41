"""Generate the golden fixtures of the :gradepro parity tests from the FP64 oracle.

    python tests/golden/make_golden.py

Each fixture holds the inputs (samples, grid, bootstrap-draw seed, keyword arguments)
and the oracle's outputs (density, selected bandwidth step) of one small
estimation, plus a second oracle run with real-input transforms (fft_mode "r2c") whose
agreement with the first marks the grid points whose outcome is fixed by the
reference's arithmetic rather than by FP64 round-off.  The bootstrap draws are not
stored: they are oracle.rng.bootstrap_indices(idx_seed, n, n_bootstraps), the same
integer stream the CUDA library generates (pkde_boot_index).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import gradepro as og  # noqa: E402
from oracle.rng import bootstrap_indices  # noqa: E402

CASES = [
    # name, ndim, dims, n, B, n_steps, seed, extra kwargs
    ("c1_like_1d", 1, (1024,), 10_000, 100, None, 11, {}),
    ("gmm_2d_64x48", 2, (64, 48), 20_000, 16, 60, 12, {}),
    ("gauss_2d_pow2_128x64", 2, (128, 64), 40_000, 8, 50, 13, {}),
    ("gauss_3d_16x20x12", 3, (16, 20, 12), 20_000, 6, 30, 14, {}),
    ("gauss_4d_8x6x10x7", 4, (8, 6, 10, 7), 20_000, 4, 20, 15, {}),
    ("kwargs_2d_32x36", 2, (32, 36), 4_000, 6, None, 16, dict(bw_step=0.01, bw_final=0.3, alpha_s=0.1,
                                                             alpha_os=0.2, eps=-0.3)),
]


def samples(ndim, n, seed):
    rng = np.random.default_rng(seed)
    if ndim == 2:
        w = rng.random(n) < 0.6
        x = rng.standard_normal((2, n))
        x[:, ~w] = x[:, ~w] * 0.5 + np.array([[2.0], [1.0]])
        return x
    return rng.standard_normal((ndim, n))


def make(case):
    name, ndim, dims, n, B, n_steps, seed, kw = case
    x = samples(ndim, n, seed)
    grid = og.find_grid(x, grid_dims=dims, grid_padding=[3 * float(np.std(x[0], ddof=1))] if ndim == 1 else None)
    idx = bootstrap_indices(seed, n, B)
    ref = og.estimate_gradepro(x, grid, idx, n_steps=n_steps, workers=4, **kw)
    alt = og.estimate_gradepro(x, grid, idx, n_steps=n_steps, workers=4, fft_mode="r2c", **kw)
    out = dict(data=x, lo=grid.lo, hi=grid.hi, h=grid.h, dims=np.array(grid.dims), idx_seed=seed, n_bootstraps=B,
               n_steps=-1 if n_steps is None else n_steps, density=ref.density, selected=ref.selected_step,
               selected_alt=alt.selected_step)
    for k, v in kw.items():
        out["kw_" + k] = v
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    stable = float(np.mean(ref.selected_step == alt.selected_step))
    print(f"{name}: G={grid.size} S={len(ref.times)} stable={stable:.4f}")


if __name__ == "__main__":
    for c in CASES:
        make(c)
