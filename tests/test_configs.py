"""Parity on the benchmarked configurations, at the stated tolerance: densities within
1e-5 relative L2 of the FP64 oracle and the same selected bandwidth step on >= 99.9 % of
the grid points.

Fixtures (tests/golden/config_c1/c2/c3.npz, made by ``make_golden.py --configs``): the
oracle's density and selected steps for
  C1: 1-D N(0,1), 10,000 samples, 1,024 points on [min - 3 sd, max + 3 sd], B = 100,
      the default 250 bandwidth steps;
  C2: 2-D 3-component GMM, 1,000,000 samples, 512 x 512, B = 64, 200 steps;
  C3: 3-D banana + Student-t(3), 4,000,000 samples, 128^3, B = 32, 150 steps;
with the bootstrap draws of seed 0 (bench.py's first timed estimation), plus the
selected steps of a second FP64 oracle run with real-input transforms.  Where the two
oracle runs select the same step, the outcome is fixed by the reference's arithmetic
(rounding-stable points); elsewhere a decision sits within FP64 round-off of the
threshold and is set by the last bits of the transforms.

Asserted per configuration:
* on the rounding-stable points: relative L2 <= 1e-5 and agreement >= 99.9 %;
* on the whole grid as well, wherever the oracle's own second FP64 run meets those
  numbers (C2, C3; not C1, where the two oracle runs differ by 1.2e-4 relative L2);
* where the GPU and the oracle select the same step the densities agree to FP64
  round-off (1e-10; 1e-7 for C3, whose fixture stores the density in float32).
The samples are regenerated from pkde_b200.workloads (a SHA-256 guards the bytes)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import config_parity as cp  # noqa: E402
CONFIGS = ["c1", "c2", "c3"]
REL_L2 = 1e-5
AGREE = 0.999


def _fixture(name):
    z = cp.load(name)
    if z is None:
        pytest.skip(f"fixture {cp.fixture_path(name)} not generated")
    return z


_inputs = cp.samples
parity = cp.parity


@pytest.mark.parametrize("name", CONFIGS)
def test_fixture_inputs_regenerate(name):
    """The seeded generators still give the fixture's samples (CPU)."""
    z = _fixture(name)
    x = _inputs(z)
    assert x.shape[0] == len(z["dims"])


def test_oracle_reproduces_c1(oracle):
    """C1 is small enough to re-run the oracle on the CPU: bit-identical steps."""
    from oracle.rng import bootstrap_indices
    z = _fixture("c1")
    x = _inputs(z)
    grid = oracle.Grid(z["lo"], z["hi"], z["h"], tuple(int(d) for d in z["dims"]))
    idx = bootstrap_indices(int(z["idx_seed"]), x.shape[1], int(z["n_bootstraps"]))
    res = oracle.estimate_gradepro(x, grid, idx, n_steps=None, workers=2)
    assert np.array_equal(res.selected_step.astype(np.int16), z["selected"])
    assert np.max(np.abs(res.density - z["density"])) <= 1e-13 * np.max(z["density"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", CONFIGS)
def test_config_parity(pk, name):
    z = _fixture(name)
    x = _inputs(z)
    dims = tuple(int(d) for d in z["dims"])
    grid = pk.Grid(z["lo"], z["hi"], dims, z["h"])
    n_steps = int(z["n_steps"])
    est = pk.initialize_estimation(x, grid=grid)
    pk.estimate_density(est, "gradepro", n_bootstraps=int(z["n_bootstraps"]), n_steps=None if n_steps < 0 else n_steps,
                        seed=int(z["idx_seed"]))
    p = parity(pk.get_density(est), est.selected_step, z)
    print(f"{name}: " + ", ".join(f"{k} {v:.3g}" for k, v in p.items()))
    # the stated tolerance on the rounding-stable points
    assert p["rel_l2_stable"] <= REL_L2
    assert p["agree_stable"] >= AGREE
    # on the whole grid wherever a second FP64 implementation of the reference meets it
    if p["oracle_r2c_rel_l2"] <= REL_L2 and p["oracle_r2c_agree"] >= AGREE:
        assert p["rel_l2"] <= REL_L2
        assert p["agree"] >= AGREE
    assert p["rel_l2_same_step"] <= (1e-7 if z["density"].dtype == np.float32 else 1e-10)
