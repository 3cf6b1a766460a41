"""Contexts driven from several host threads at once (what the serving lanes do): the
shared-memory size a kernel may use is a property of the kernel for the whole process,
so launches of shapes with different needs from concurrent threads must never see a
limit another thread lowered.  Every result equals the same estimation run alone.
Needs a B200."""
import ctypes
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# engine shapes of different shared-memory needs (register, mixed-radix and generic
# tiles), a forward-FFT axis of 1000 points, and a 1-D grid
SHAPES = [(256, 128), (48, 40), (96, 24), (1000, 8), (2048,), (16, 32, 16)]


def _case(pk, i):
    rng = np.random.default_rng(100 + i)
    dims = SHAPES[i % len(SHAPES)]
    x = rng.standard_normal((len(dims), 3000 + 500 * i))
    return pk.find_grid(x, grid_dims=dims), np.ascontiguousarray(x.T)


def _run(pk, ctx, grid, xt, seed):
    from pkde_b200 import _lib
    lib = _lib.load()
    p = _lib.make_params(_lib.make_grid_struct(grid.lo, grid.hi, grid.h, grid.dims), n_bootstraps=6, n_steps=16)
    G = int(np.prod(grid.dims))
    d, s = np.empty(G), np.empty(G, dtype=np.int32)
    rc = lib.pkde_gradepro_estimate(ctx, ctypes.byref(p), _lib.ptr(xt), xt.shape[0], None, seed, _lib.ptr(d),
                                    _lib.ptr(s), 0, None)
    _lib.check(rc, ctx)
    return d, s


def test_concurrent_contexts_match_alone(pk):
    from pkde_b200 import _lib
    lib = _lib.load()
    cases = [_case(pk, i) for i in range(len(SHAPES))]
    alone = [_run(pk, _lib.context(0), g, xt, 7 + i) for i, (g, xt) in enumerate(cases)]
    ctxs = []
    for _ in range(2):
        h = ctypes.c_void_p()
        assert lib.pkde_create(ctypes.byref(h), 0) == 0
        ctxs.append(h)
    errors, results = [], {}

    def worker(k):
        j = None
        try:
            for rep in range(4):
                for i in range(len(cases)):
                    j = (i + 3 * k + rep) % len(cases)  # the threads walk the shapes out of phase
                    g, xt = cases[j]
                    results[(k, rep, j)] = _run(pk, ctxs[k], g, xt, 7 + j)
        except Exception as e:  # reported on the main thread
            errors.append(f"thread {k}, shape {SHAPES[j]}: {e!r}")

    try:
        threads = [threading.Thread(target=worker, args=(k,)) for k in range(2)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    finally:
        for h in ctxs:
            lib.pkde_destroy(h)
    assert not errors, errors
    assert len(results) == 2 * 4 * len(cases)
    for (k, rep, j), (d, s) in results.items():
        assert np.array_equal(d, alone[j][0]) and np.array_equal(s, alone[j][1]), (k, rep, SHAPES[j])
