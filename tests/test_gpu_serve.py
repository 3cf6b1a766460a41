"""Serving with continuous batching (pkde_submit / pkde_wait): requests submitted from
several threads while others are on the GPU; each result is identical to a
one-request call; a bad request fails alone.  Needs a B200."""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(pk, count, seed):
    rng = np.random.default_rng(seed)
    shapes = [(512,), (64, 32), (48, 40), (16, 32, 16), (1024,), (8, 6, 10, 7), (96, 96), (20, 24, 16)]
    out = []
    for i in range(count):
        dims = shapes[i % len(shapes)]
        n = int(rng.integers(800, 20000))
        x = rng.standard_normal((len(dims), n)) * rng.uniform(0.5, 2.0)
        grid = pk.find_grid(x, grid_dims=dims)
        out.append(dict(grid=grid, data=x, n_bootstraps=int(rng.integers(2, 12)), n_steps=int(rng.integers(10, 40)),
                        seed=1000 + i))
    return out


def _alone(r):
    from pkde_b200 import raw
    G = int(np.prod(r["grid"].dims))
    d = np.empty(G)
    s = np.empty(G, dtype=np.int32)
    raw.gradepro_host(r["grid"], np.ascontiguousarray(r["data"].T), d, s, seed=r["seed"],
                      n_bootstraps=r["n_bootstraps"], n_steps=r["n_steps"])
    return d, s


def test_served_results_equal_alone(pk):
    from pkde_b200.serve import Server
    srv = Server()
    reqs = _requests(pk, 24, 1)
    tickets = [None] * len(reqs)

    def producer(k):
        rng = np.random.default_rng(k)
        for i in range(k, len(reqs), 3):
            r = reqs[i]
            tickets[i] = srv.submit(r["grid"], r["data"], n_bootstraps=r["n_bootstraps"], n_steps=r["n_steps"],
                                    seed=r["seed"])
            time.sleep(float(rng.uniform(0, 0.004)))

    th = [threading.Thread(target=producer, args=(k,)) for k in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    results = [srv.wait(t) for t in tickets]
    for r, res in zip(reqs, results):
        assert res["status"] == 0, res["message"]
        d, s = _alone(r)
        assert np.array_equal(res["density"].reshape(-1), d)
        assert np.array_equal(res["selected_step"].reshape(-1), s)
        assert res["total_ms"] >= res["run_ms"] > 0 and res["queue_ms"] >= 0
    assert max(res["batch_size"] for res in results) >= 2  # later arrivals were batched


def test_served_bad_request_fails_alone(pk):
    from pkde_b200.serve import Server
    srv = Server()
    reqs = _requests(pk, 6, 2)
    bad = reqs[3]["data"].copy()
    bad[0, 0] = reqs[3]["grid"].hi[0] + 1.0
    reqs[3]["data"] = bad
    tickets = [srv.submit(r["grid"], r["data"], n_bootstraps=r["n_bootstraps"], n_steps=r["n_steps"], seed=r["seed"])
               for r in reqs]
    results = [srv.wait(t) for t in tickets]
    assert results[3]["status"] == 1 and "beyond grid" in results[3]["message"]
    for i in (0, 1, 2, 4, 5):
        assert results[i]["status"] == 0, results[i]["message"]
        d, s = _alone(reqs[i])
        assert np.array_equal(results[i]["density"].reshape(-1), d)
    with pytest.raises(pk.ArgumentError, match="unknown ticket"):
        srv.wait(tickets[0])
    with pytest.raises(pk.ArgumentError):
        srv.submit(reqs[0]["grid"], reqs[0]["data"], n_bootstraps=1)  # parameter error at submit
