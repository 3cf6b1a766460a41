"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from the FP64
oracle): the oracle still reproduces them (CPU), and the CUDA path matches them through
the C ABI, with explicit draws and with the device's own seeded draws (GPU)."""
import glob
import os

import numpy as np
import pytest

from oracle.rng import bootstrap_indices

HERE = os.path.dirname(os.path.abspath(__file__))
# the benchmarked configurations (config_*.npz) have their own tests (test_configs.py)
FIXTURES = sorted(p for p in glob.glob(os.path.join(HERE, "golden", "*.npz"))
                  if not os.path.basename(p).startswith("config_"))


def load(path):
    z = np.load(path)
    kw = {k[3:]: float(z[k]) for k in z.files if k.startswith("kw_")}
    n_steps = int(z["n_steps"])
    return z, kw, (None if n_steps < 0 else n_steps)


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_reproduces_fixture(oracle, path):
    z, kw, n_steps = load(path)
    grid = oracle.Grid(z["lo"], z["hi"], z["h"], tuple(int(d) for d in z["dims"]))
    if grid.size > 5000:
        pytest.skip("large fixture: checked on the GPU runs")
    idx = bootstrap_indices(int(z["idx_seed"]), z["data"].shape[1], int(z["n_bootstraps"]))
    res = oracle.estimate_gradepro(z["data"], grid, idx, n_steps=n_steps, workers=2, **kw)
    assert np.array_equal(res.selected_step, z["selected"])
    assert np.max(np.abs(res.density - z["density"])) <= 1e-13 * np.max(z["density"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_cuda_matches_fixture(pk, path):
    z, kw, n_steps = load(path)
    dims = tuple(int(d) for d in z["dims"])
    grid = pk.Grid(z["lo"], z["hi"], dims, z["h"])
    B = int(z["n_bootstraps"])
    n = z["data"].shape[1]
    idx = bootstrap_indices(int(z["idx_seed"]), n, B)
    outs = []
    for explicit in (True, False):
        est = pk.initialize_estimation(z["data"], grid=grid)
        extra = dict(bootstrap_idxs=idx) if explicit else dict(seed=int(z["idx_seed"]))
        pk.estimate_density(est, "gradepro", n_bootstraps=B, n_steps=n_steps, **kw, **extra)
        outs.append((pk.get_density(est).copy(), est.selected_step.copy()))
    # the device's seeded draws are the same integer stream as the explicit ones
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    dens, sel = outs[0]
    ref_sel, alt_sel, ref_d = z["selected"], z["selected_alt"], z["density"]
    stable = ref_sel == alt_sel
    flips_alt = int(np.sum(~stable))
    flips = int(np.sum(sel != ref_sel))
    both = stable & (sel == ref_sel)
    rel_both = float(np.linalg.norm(dens[both] - ref_d[both]) / np.linalg.norm(ref_d[both]))
    rel = float(np.linalg.norm(dens - ref_d) / np.linalg.norm(ref_d))
    print(f"{os.path.basename(path)}: rel L2 {rel:.2e}, flips {flips} (oracle r2c vs c2c {flips_alt}), "
          f"rel L2 where the step agrees {rel_both:.2e}")
    assert rel_both <= 1e-10
    assert flips <= 1.5 * flips_alt + 0.001 * sel.size + 2
