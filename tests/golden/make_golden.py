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
import math
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


def add_sampled_stability(name, trace_variants, samples, heldout, workers, seed=1, batch=16, cache=None,
                          target=1e-4):
    """Extend the fixture's rounding-unstable set with sampled rounding realisations.

    A union over a handful of FP64 implementations under-covers the points whose decision
    is set by rounding: where the reference's log-VMR variance f sits at the noise floor
    (empty or nearly empty cells; many steps, so that the second difference divides a
    rounding-level wobble by a small dlogt^2) each implementation's decision is a coin
    flip of its own, and the union of k flip sets keeps growing with k.

    The reference's trace F0 (steps x points) and the traces F_i of the `trace_variants`
    give k rounding differences D_i = F_i - F0, each with the step-to-step correlation of
    real rounding.  Each sample replays the selection on F0 + sum_i c_i D_i, c ~ N(0, 1/k)
    (the variance of one more independent implementation's difference from the
    reference), so a point's flip frequency over the samples estimates the probability q
    that an independent FP64 implementation selects another step there.  The unstable set
    is the variants' own flips plus the points ranked highest by the frequency in one half
    of the samples, as few as leave an expected flip rate <= `target` (a tenth of the
    0.1 % that parity allows; on C1's ~1,000 points 0.1 expected flips, where one flip near
    the mode already moves the density by 2e-4 relative L2) on the remaining, stable
    points, that rate estimated from the other half: ranked and scored by the same counts,
    the points kept as stable are the ones whose count came out low, and their residual
    is underestimated (by 3x on C2).  `rounding_rate` (the mean of q over the grid: the expected
    flip rate of an independent implementation) is recorded beside the whole-grid flip
    rates of the `heldout` implementations (real ones, run afterwards and not used to
    build the set) as a calibration check, with their agreement on the stable points.
    `cache`: a directory for the traces and the held-out selections (re-runs reuse them)."""
    import time
    path = os.path.join(HERE, f"config_{name}.npz")
    z = dict(np.load(path))
    x, spec, B, n_steps = config_inputs(name)
    grid = og.Grid(z["lo"], z["hi"], z["h"], tuple(int(d) for d in z["dims"]))
    idx = bootstrap_indices(int(z["idx_seed"]), x.shape[1], B)
    ref_sel = z["selected"].astype(np.int32).reshape(-1)
    G = ref_sel.size
    real = np.unpackbits(z["unstable_real"] if "unstable_real" in z else z["unstable"])[:G].astype(bool)
    t_start = time.time()
    cpath = (lambda tag: os.path.join(cache, f"cache_{name}_{tag}.npy")) if cache else None

    def trace(v):
        """(selected steps, trace as steps x points) of the oracle run `v` (None: c2c)."""
        if cpath and os.path.exists(cpath(f"F_{v}")):
            return np.load(cpath(f"sel_{v}")), np.load(cpath(f"F_{v}"), mmap_mode="r")
        r = og.estimate_gradepro(x, grid, idx, n_steps=n_steps, workers=workers, variant=v, keep_trace="f")
        sel = r.selected_step.reshape(-1).astype(np.int32)
        F = np.stack([f.reshape(-1) for f in r.vmr_trace])
        del r
        if cpath:
            np.save(cpath(f"sel_{v}"), sel)
            np.save(cpath(f"F_{v}"), F)
        print(f"config_{name}: trace {v} ({time.time() - t_start:.0f} s)", flush=True)
        return sel, F

    sel0, F0 = trace(None)
    assert np.array_equal(sel0, ref_sel), "reference trace does not reproduce the fixture"
    S = F0.shape[0]
    D = np.empty((len(trace_variants), S, G), dtype=np.float32)
    for i, v in enumerate(trace_variants):
        sel, Fv = trace(v)
        real |= sel != ref_sel
        for s in range(S):
            d = np.asarray(Fv[s]) - F0[s]
            d[~np.isfinite(d)] = 0.0
            D[i, s] = d
        del Fv
    times, steps_low, steps_over, eps = og.ladder(x, grid, n_steps)
    t0 = og.initial_bandwidth(grid)
    rng = np.random.default_rng(seed)
    k = len(trace_variants)
    flips = np.zeros((2, G), dtype=np.int32)  # the two halves of the samples
    done = 0
    while done < samples:
        m = min(batch, samples - done)
        C = (rng.standard_normal((m, k)) / math.sqrt(k)).astype(np.float32)
        steps = (np.asarray(F0[s])[None, :] + (C @ D[:, s, :]).astype(np.float64) for s in range(S))
        sel = og.select_from_trace(steps, times, t0, steps_low, steps_over, eps)
        flips[0 if done < samples // 2 else 1] += np.sum(sel != ref_sel[None, :], axis=0).astype(np.int32)
        done += m
        print(f"config_{name}: {done} samples, mean flip rate {flips.sum() / (done * G):.5f} "
              f"({time.time() - t_start:.0f} s)", flush=True)
    half = (samples // 2 + batch - 1) // batch * batch  # the first half: whole batches
    qa = flips[0] / float(half)
    qb = flips[1] / float(samples - half)
    q = flips.sum(0) / float(samples)
    # the fewest points of highest qa that leave sum(qb) / |stable| <= target on the rest
    order = np.argsort(-qa, kind="stable")
    rest = np.cumsum(qb[order][::-1])[::-1]  # rest[j]: sum of qb over order[j:]
    nstable = G - np.arange(G)
    ok = np.nonzero(rest <= target * nstable)[0]
    cut = int(ok[0]) if ok.size else G
    sampled = np.zeros(G, dtype=bool)
    sampled[order[:cut]] = True
    unstable = sampled | real
    stable = ~unstable
    print(f"config_{name}: sampled set {np.mean(sampled):.5f}, union {np.mean(unstable):.5f}, expected flip rate "
          f"on the stable points {qb[stable].sum() / max(stable.sum(), 1):.6f}, over the grid {q.mean():.5f}", flush=True)
    hagree = []
    for v in heldout:
        if cpath and os.path.exists(cpath(f"sel_{v}")):
            sel = np.load(cpath(f"sel_{v}"))
        else:
            r = og.estimate_gradepro(x, grid, idx, n_steps=n_steps, workers=workers, variant=v)
            sel = r.selected_step.reshape(-1).astype(np.int32)
            del r
            if cpath:
                np.save(cpath(f"sel_{v}"), sel)
        hagree.append([float(np.mean(sel == ref_sel)), float(np.mean(sel[stable] == ref_sel[stable]))])
        print(f"config_{name}: held-out {v} agree {hagree[-1][0]:.5f}, on the stable points "
              f"{hagree[-1][1]:.5f} ({time.time() - t_start:.0f} s)", flush=True)
    z["unstable_real"] = np.packbits(real)
    z["unstable"] = np.packbits(unstable)
    z["trace_variants"] = np.array(trace_variants)
    z["rounding_samples"] = np.int64(samples)
    z["rounding_seed"] = np.int64(seed)
    z["rounding_target"] = np.float64(target)
    z["rounding_rate"] = np.float64(q.mean())
    z["rounding_rate_stable"] = np.float64(qb[stable].sum() / max(stable.sum(), 1))
    z["heldout"] = np.array(list(heldout))
    z["heldout_agree"] = np.array(hagree).reshape(-1, 2)
    np.savez_compressed(path, **z)


if __name__ == "__main__":
    if "--sampled" in sys.argv:
        i = sys.argv.index("--sampled")
        cache = sys.argv[sys.argv.index("--cache") + 1] if "--cache" in sys.argv else None
        add_sampled_stability(sys.argv[i + 1], sys.argv[i + 2].split(","), int(sys.argv[i + 3]),
                              [v for v in sys.argv[i + 4].split(",") if v], os.cpu_count() or 1, cache=cache)
    elif "--stable" in sys.argv:
        i = sys.argv.index("--stable")
        add_stability(sys.argv[i + 1], sys.argv[i + 2].split(","), os.cpu_count() or 1)
    elif "--configs" in sys.argv:
        names = [a for a in sys.argv[sys.argv.index("--configs") + 1:] if not a.startswith("-")] or list(CONFIGS)
        for nm in names:
            make_config(nm, os.cpu_count() or 1)
    else:
        for c in CASES:
            make(c)
