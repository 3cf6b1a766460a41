"""The batched form (pkde_gradepro_estimate_batch): estimations of different dimensions,
grid sizes, sample and bootstrap counts in one call.  Each estimation's density and
selected steps are identical, bit for bit, to what the one-estimation entry point gives
for it alone; one member is also checked against the FP64 oracle.  Needs a B200."""
import numpy as np
import pytest

from oracle.rng import bootstrap_indices

pytestmark = pytest.mark.gpu


def _mix(pk, seed=5):
    """(grid, data (N x n), kwargs) for a spread of paths: 1-D step-parallel, 2-D/3-D
    power-of-two engine, 2-D non-power-of-two, 4-D."""
    rng = np.random.default_rng(seed)
    cases = [
        ((512,), 3000, 16, 40),
        ((64, 32), 5000, 8, 30),
        ((48, 40), 4000, 6, 25),
        ((16, 32, 16), 6000, 4, 20),
        ((128, 64), 20000, 12, 35),
        ((1024,), 800, 10, 50),
        ((8, 6, 10, 7), 2500, 3, 12),
        ((32, 32), 1500, 2, 15),
    ]
    out = []
    for dims, n, B, steps in cases:
        x = rng.standard_normal((len(dims), n)) * rng.uniform(0.5, 2.0)
        grid = pk.find_grid(x, grid_dims=dims)
        out.append((grid, x, dict(n_bootstraps=B, n_steps=steps)))
    return out


def _alone(pk, grid, x, kw, seed):
    from pkde_b200 import raw
    G = int(np.prod(grid.dims))
    dens = np.empty(G)
    sel = np.empty(G, dtype=np.int32)
    raw.gradepro_host(grid, np.ascontiguousarray(x.T), dens, sel, seed=seed, **kw)
    return dens, sel


def _batch_jobs(mix):
    jobs = []
    for e, (grid, x, kw) in enumerate(mix):
        G = int(np.prod(grid.dims))
        jobs.append(dict(grid=grid, data=np.ascontiguousarray(x.T), density=np.empty(G),
                         selected=np.empty(G, dtype=np.int32), seed=100 + e, **kw))
    return jobs


def test_batch_equals_alone(pk):
    from pkde_b200 import raw
    mix = _mix(pk)
    jobs = _batch_jobs(mix)
    raw.gradepro_batch(jobs)
    for e, (grid, x, kw) in enumerate(mix):
        d, s = _alone(pk, grid, x, kw, seed=100 + e)
        assert np.array_equal(jobs[e]["density"], d, equal_nan=True), f"estimation {e} {grid.dims}"
        assert np.array_equal(jobs[e]["selected"], s), f"estimation {e} {grid.dims}"
        assert np.all(np.isfinite(d))


def test_batch_order_and_subsets(pk):
    """The same estimation in a different position and with other neighbours."""
    from pkde_b200 import raw
    mix = _mix(pk)
    jobs = _batch_jobs(mix)
    raw.gradepro_batch(jobs)
    sub = [mix[4], mix[1], mix[0]]
    seeds = [104, 101, 100]
    jobs2 = _batch_jobs(sub)
    for j, sd in zip(jobs2, seeds):
        j["seed"] = sd
    raw.gradepro_batch(jobs2)
    for j2, e in zip(jobs2, (4, 1, 0)):
        assert np.array_equal(j2["density"], jobs[e]["density"])
        assert np.array_equal(j2["selected"], jobs[e]["selected"])


def test_batch_member_matches_oracle(pk, oracle):
    from pkde_b200 import raw
    mix = _mix(pk)
    grid, x, kw = mix[1]
    n = x.shape[1]
    idx = bootstrap_indices(9, n, kw["n_bootstraps"])
    jobs = _batch_jobs(mix)
    jobs[1]["idx"] = idx
    raw.gradepro_batch(jobs)
    og_grid = oracle.Grid(grid.lo, grid.hi, grid.h, grid.dims)
    ref = oracle.estimate_gradepro(x, og_grid, idx, n_steps=kw["n_steps"])
    d = jobs[1]["density"]
    rd = np.asarray(ref.density).reshape(-1)
    rel = np.linalg.norm(d - rd) / np.linalg.norm(rd)
    agree = np.mean(jobs[1]["selected"] == np.asarray(ref.selected_step).reshape(-1))
    assert rel < 1e-6 and agree > 0.99, (rel, agree)


def test_batch_device_pointers(pk):
    import torch
    from pkde_b200 import raw
    mix = _mix(pk)[:4]
    host = _batch_jobs(mix)
    raw.gradepro_batch(host)
    dev = []
    for j in host:
        dev.append(dict(grid=j["grid"], data=torch.from_numpy(j["data"]).cuda(),
                        density=torch.empty(j["density"].shape, dtype=torch.float64, device="cuda"),
                        selected=torch.empty(j["selected"].shape, dtype=torch.int32, device="cuda"),
                        seed=j["seed"], n_bootstraps=j["n_bootstraps"], n_steps=j["n_steps"]))
    raw.gradepro_batch(dev, device=True, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    for h, d in zip(host, dev):
        assert np.array_equal(d["density"].cpu().numpy(), h["density"])
        assert np.array_equal(d["selected"].cpu().numpy(), h["selected"])


def test_batch_error_names_estimation(pk):
    from pkde_b200 import raw
    mix = _mix(pk)[:3]
    jobs = _batch_jobs(mix)
    bad = jobs[2]["data"].copy()
    bad[0, 0] = jobs[2]["grid"].hi[0] + 1.0  # beyond the grid
    jobs[2]["data"] = bad
    with pytest.raises(pk.ArgumentError, match=r"estimation 2: Data points lie beyond grid"):
        raw.gradepro_batch(jobs)
    # the context is still usable
    ok = _batch_jobs(mix[:2])
    raw.gradepro_batch(ok)
    assert np.all(np.isfinite(ok[0]["density"]))


@pytest.mark.parametrize("dims,n,B,steps", [((48, 40), 6000, 8, 30), ((64, 32), 6000, 8, 30),
                                             ((16, 20, 12), 5000, 6, 20), ((96, 96), 20000, 16, 40)])
def test_plain_form_agrees_with_engine(pk, dims, n, B, steps):
    """The launch-per-step form (PKDE_STEPS_PER_STEP_LAUNCH) and the step engine: same
    densities to FP64 round-off wherever the selected steps agree, and (nearly) the same
    selected steps."""
    from pkde_b200 import _lib
    rng = np.random.default_rng(sum(dims))
    x = rng.standard_normal((len(dims), n))
    grid = pk.find_grid(x, grid_dims=dims)
    kw = dict(n_bootstraps=B, n_steps=steps)
    d_auto, s_auto = _alone(pk, grid, x, kw, seed=3)
    _lib.set_step_path(_lib.PKDE_STEPS_PER_STEP_LAUNCH)
    try:
        d_plain, s_plain = _alone(pk, grid, x, kw, seed=3)
    finally:
        _lib.set_step_path(_lib.PKDE_STEPS_AUTO)
    same = s_auto == s_plain
    assert same.mean() >= 0.99
    rel = np.linalg.norm((d_auto - d_plain)[same]) / np.linalg.norm(d_plain[same])
    assert rel <= 1e-10, rel


def test_autotune_keeps_results_and_caches(pk, tmp_path, monkeypatch):
    """The per-shape schedule search changes time only: results with autotuning on and
    off are identical; the chosen schedule is appended to PKDE_TUNE_CACHE."""
    import ctypes
    from pkde_b200 import _lib
    lib = _lib.load()
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("PKDE_TUNE_CACHE", str(cache))
    rng = np.random.default_rng(12)
    x = rng.standard_normal((2, 6000))
    grid = pk.find_grid(x, grid_dims=(64, 48))
    p = _lib.make_params(_lib.make_grid_struct(grid.lo, grid.hi, grid.h, grid.dims), 10, 20)
    data = np.ascontiguousarray(x.T)
    outs = []
    for tune in (0, 1):
        ctx = ctypes.c_void_p()
        assert lib.pkde_create(ctypes.byref(ctx), 0) == 0
        assert lib.pkde_set_autotune(ctx, tune) == 0
        d = np.empty(grid.dims[0] * grid.dims[1])
        s = np.empty(d.size, dtype=np.int32)
        rc = lib.pkde_gradepro_estimate(ctx, ctypes.byref(p), _lib.ptr(data), data.shape[0], None, 3, _lib.ptr(d),
                                        _lib.ptr(s), 0, None)
        assert rc == 0
        outs.append((d, s))
        lib.pkde_destroy(ctx)
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    lines = cache.read_text().split()
    assert lines and lines[0] == "2x64x48:p5" and len(lines) == 4


@pytest.mark.parametrize("dims", [(64, 48), (16, 32, 16), (24, 20, 12)])
def test_engine_schedules_keep_results(pk, monkeypatch, dims):
    """Every schedule the autotuner may pick (pipeline delay 1..4, ring-slot sizes from one
    pair per group up to all pairs, tiles per item) gives the same densities and steps."""
    import ctypes
    from pkde_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(len(dims))
    x = rng.standard_normal((len(dims), 5000))
    grid = pk.find_grid(x, grid_dims=dims)
    p = _lib.make_params(_lib.make_grid_struct(grid.lo, grid.hi, grid.h, grid.dims), 10, 24)
    data = np.ascontiguousarray(x.T)
    G = int(np.prod(dims))
    ctx = ctypes.c_void_p()
    assert lib.pkde_create(ctypes.byref(ctx), 0) == 0
    outs = []
    try:
        assert lib.pkde_set_autotune(ctx, 0) == 0
        for delay, slot_mb, tpi in ((2, 32, 2), (1, 1, 1), (1, 32, 4), (3, 1, 8), (4, 2, 2)):
            monkeypatch.setenv("PKDE_ENGINE_DELAY", str(delay))
            monkeypatch.setenv("PKDE_ENGINE_SLOT_MB", str(slot_mb))
            monkeypatch.setenv("PKDE_ENGINE_TPI", str(tpi))
            d, s = np.empty(G), np.empty(G, dtype=np.int32)
            rc = lib.pkde_gradepro_estimate(ctx, ctypes.byref(p), _lib.ptr(data), data.shape[0], None, 5, _lib.ptr(d),
                                            _lib.ptr(s), 0, None)
            _lib.check(rc, ctx)
            outs.append((d, s))
    finally:
        lib.pkde_destroy(ctx)
    for d, s in outs[1:]:
        assert np.array_equal(d, outs[0][0]) and np.array_equal(s, outs[0][1])


def test_wide_ring_slots_keep_results(pk, monkeypatch):
    """Ring slots above 64 MB, holding all bootstrap pairs of a step in one group (what the
    autotuner picks for large grids), give the same result as narrow slots of one or a
    few pairs per group."""
    import ctypes
    from pkde_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(21)
    x = rng.standard_normal((2, 20000))
    dims = (256, 256)
    grid = pk.find_grid(x, grid_dims=dims)
    B = 80  # 40 pairs x 2 arrays x 1 MB = 80 MB per group of all pairs
    p = _lib.make_params(_lib.make_grid_struct(grid.lo, grid.hi, grid.h, grid.dims), B, 12)
    data = np.ascontiguousarray(x.T)
    G = int(np.prod(dims))
    ctx = ctypes.c_void_p()
    assert lib.pkde_create(ctypes.byref(ctx), 0) == 0
    outs = []
    try:
        assert lib.pkde_set_autotune(ctx, 0) == 0
        for slot_mb, tpi in ((128, 4), (2, 2), (8, 4), (48, 2)):
            monkeypatch.setenv("PKDE_ENGINE_SLOT_MB", str(slot_mb))
            monkeypatch.setenv("PKDE_ENGINE_TPI", str(tpi))
            d, s = np.empty(G), np.empty(G, dtype=np.int32)
            rc = lib.pkde_gradepro_estimate(ctx, ctypes.byref(p), _lib.ptr(data), data.shape[0], None, 9, _lib.ptr(d),
                                            _lib.ptr(s), 0, None)
            _lib.check(rc, ctx)
            outs.append((d, s))
    finally:
        lib.pkde_destroy(ctx)
    for d, s in outs[1:]:
        assert np.array_equal(d, outs[0][0]) and np.array_equal(s, outs[0][1])


def test_batch_packed_into_several_launches(pk, monkeypatch):
    """When the estimations' tuned ring slots together exceed the memory budget, a batch call
    packs them into consecutive engine launches that fit (PKDE_RING_BUDGET_MB caps the
    budget: with 1 MB every estimation gets a launch of its own).  The results equal each
    estimation's alone result, bit for bit.  N-D estimations only: the 1-D step path's
    launches count in the same phase."""
    from pkde_b200 import _lib, raw
    mix = [m for m in _mix(pk) if len(m[0].dims) >= 2]
    alone = [_alone(pk, grid, x, kw, seed=100 + e) for e, (grid, x, kw) in enumerate(mix)]  # also tunes

    def engine_launches(jobs):
        _lib.get_stats(0, reset=True)
        _lib.set_profiling(_lib.PKDE_PROFILE_STEPS, 0)
        try:
            raw.gradepro_batch(jobs)
        finally:
            _lib.set_profiling(_lib.PKDE_PROFILE_OFF, 0)
        return _lib.get_stats(0, reset=True)["phase_launches"]["step_vmr"]

    jobs = _batch_jobs(mix)
    assert engine_launches(jobs) <= 2  # the lean and the mixed-radix instantiation
    monkeypatch.setenv("PKDE_RING_BUDGET_MB", "1")
    packed = _batch_jobs(mix)
    assert engine_launches(packed) == len(mix)
    for e, (d, s) in enumerate(alone):
        assert np.array_equal(packed[e]["density"], d, equal_nan=True), f"estimation {e}"
        assert np.array_equal(packed[e]["selected"], s), f"estimation {e}"
        assert np.array_equal(jobs[e]["density"], d, equal_nan=True), f"estimation {e}"
