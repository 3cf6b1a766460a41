"""Generate the golden fixtures of the :gradepro parity tests from the FP64 oracle.

    python tests/golden/make_golden.py

Each fixture holds the inputs (samples, grid, bootstrap-draw seed, keyword arguments)
and the oracle's outputs (density, selected bandwidth step) of one small
estimation, plus a second oracle run with real-input transforms (fft_mode "r2c") whose
agreement with the first marks the grid points whose outcome is fixed by the
reference's arithmetic rather than by FP64 round-off.  The bootstrap draws are not
stored: they are oracle.rng.bootstrap_indices(idx_seed, n, n_bootstraps), the same
integer stream the CUDA library generates (pkde_boot_index).

    python tests/golden/make_golden.py --configs [c1 c2 c3]

makes the fixtures of the benchmarked configurations instead (config_c1/c2/c3.npz), and

    python tests/golden/make_golden.py --stable c2 paired,sep,longdouble,jitter-1

adds to one of them the grid points whose outcome rounding decides (where other FP64
implementations of the same mathematics select another step; see add_stability).  The configuration fixtures:
the samples are not stored but regenerated from the seeded generators of
pkde_b200.workloads (a SHA-256 of the sample bytes guards against drift), and the
bootstrap seed is the one bench.py uses for its first timed estimation.  The 3-D
density is stored in float32 (16 MB in float64; float32 keeps ~6e-8 relative, far
inside the 1e-5 tolerance), selected steps in int16.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "parallelkde.jl_b200"))

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


# The benchmarked configurations: name, workload generator, bootstrap count, bandwidth
# steps (None: the reference's default 250), density storage type.  Bootstrap seed 0 is
# bench.py's first timed estimation on rank 0 (multi.estimation_seed(0, 0)).
CONFIGS = {
    "c1": ("gaussian_1d", 100, None, np.float64),
    "c2": ("gmm_2d", 64, 200, np.float64),
    "c3": ("banana_t_3d", 32, 150, np.float32),
}
CONFIG_SEED = 0


def config_inputs(name):
    """Samples (N, n) and grid spec of a benchmarked configuration, regenerated."""
    from pkde_b200 import workloads as W
    gen, B, n_steps, _ = CONFIGS[name]
    x, spec = getattr(W, gen)()
    return x, spec, B, n_steps


def sample_digest(x):
    return hashlib.sha256(np.ascontiguousarray(x, dtype=np.float64).tobytes()).hexdigest()


def make_config(name, workers):
    import time
    x, spec, B, n_steps = config_inputs(name)
    grid = og.find_grid(x, grid_dims=spec["dims"], grid_padding=spec.get("grid_padding"))
    idx = bootstrap_indices(CONFIG_SEED, x.shape[1], B)
    t0 = time.time()
    ref = og.estimate_gradepro(x, grid, idx, n_steps=n_steps, workers=workers)
    t1 = time.time()
    alt = og.estimate_gradepro(x, grid, idx, n_steps=n_steps, workers=workers, fft_mode="r2c")
    t2 = time.time()
    dt = CONFIGS[name][3]
    rel_alt = float(np.linalg.norm(alt.density - ref.density) / np.linalg.norm(ref.density))
    agree_alt = float(np.mean(ref.selected_step == alt.selected_step))
    np.savez_compressed(os.path.join(HERE, f"config_{name}.npz"), workload=CONFIGS[name][0],
                        sample_sha256=sample_digest(x), lo=grid.lo, hi=grid.hi, h=grid.h, dims=np.array(grid.dims),
                        idx_seed=CONFIG_SEED, n_bootstraps=B, n_steps=-1 if n_steps is None else n_steps,
                        density=ref.density.astype(dt), selected=ref.selected_step.astype(np.int16),
                        selected_alt=alt.selected_step.astype(np.int16), rel_alt=rel_alt, agree_alt=agree_alt,
                        oracle_seconds=t1 - t0, workers=workers)
    print(f"config_{name}: G={grid.size} S={len(ref.times)} oracle {t1 - t0:.0f} s (r2c {t2 - t1:.0f} s) on "
          f"{workers} threads; r2c vs c2c rel L2 {rel_alt:.2e}, agree {agree_alt:.5f}", flush=True)


def add_stability(name, variants, workers):
    """Add to config_<name>.npz the grid points whose selected step depends on FP64
    rounding: those where any other FP64 implementation of the same mathematics -- the
    real-input-transform run already in the fixture and the oracle's `variant`s
    (estimate_gradepro: paired transforms, separable propagator, long double, jittered
    forward spectra) -- selects another step than the reference-faithful run.  Stored
    bit-packed as `unstable`, with each variant's agreement in `variant_agree`."""
    import time
    path = os.path.join(HERE, f"config_{name}.npz")
    z = dict(np.load(path))
    x, spec, B, n_steps = config_inputs(name)
    grid = og.Grid(z["lo"], z["hi"], z["h"], tuple(int(d) for d in z["dims"]))
    idx = bootstrap_indices(int(z["idx_seed"]), x.shape[1], B)
    ref_sel = z["selected"].astype(np.int32).reshape(-1)
    unstable = ref_sel != z["selected_alt"].astype(np.int32).reshape(-1)
    agrees = []
    for v in variants:
        t0 = time.time()
        r = og.estimate_gradepro(x, grid, idx, n_steps=n_steps, workers=workers, variant=v)
        sel = r.selected_step.reshape(-1)
        agrees.append(float(np.mean(sel == ref_sel)))
        unstable |= sel != ref_sel
        print(f"config_{name}: {v} agree {agrees[-1]:.5f}, unstable so far {np.mean(unstable):.5f} "
              f"({time.time() - t0:.0f} s)", flush=True)
        z["unstable"] = np.packbits(unstable)
        z["variants"] = np.array(variants[:len(agrees)])
        z["variant_agree"] = np.array(agrees)
        for k in ("ens_members", "ens_agree"):
            z.pop(k, None)
        np.savez_compressed(path, **z)


if __name__ == "__main__":
    if "--stable" in sys.argv:
        i = sys.argv.index("--stable")
        add_stability(sys.argv[i + 1], sys.argv[i + 2].split(","), os.cpu_count() or 1)
    elif "--configs" in sys.argv:
        names = [a for a in sys.argv[sys.argv.index("--configs") + 1:] if not a.startswith("-")] or list(CONFIGS)
        for nm in names:
            make_config(nm, os.cpu_count() or 1)
    else:
        for c in CASES:
            make(c)
