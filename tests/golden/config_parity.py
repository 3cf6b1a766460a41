"""Parity of a :gradepro result against the fixture of a benchmarked configuration
(config_c1/c2/c3.npz, made by make_golden.py --configs).  Used by tests/test_configs.py
and by bench.py (outside its timed region) to state the error of the estimation it
timed.  Reads only the committed fixture; the samples are regenerated from the seeded
generators of pkde_b200.workloads and checked against the fixture's SHA-256."""
import hashlib
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def fixture_path(name):
    return os.path.join(HERE, f"config_{name}.npz")


def load(name):
    """The fixture of configuration `name` ("c1", "c2", "c3"), or None if absent."""
    p = fixture_path(name)
    return np.load(p) if os.path.exists(p) else None


def samples(z):
    """The configuration's samples (N, n), regenerated; raises if they drifted."""
    from pkde_b200 import workloads as W
    x, _ = getattr(W, str(z["workload"]))()
    if hashlib.sha256(np.ascontiguousarray(x, dtype=np.float64).tobytes()).hexdigest() != str(z["sample_sha256"]):
        raise RuntimeError(f"samples of {z['workload']} differ from the fixture's")
    return x


def parity(dens, sel, z):
    """Error figures of (density, selected steps) against the fixture: whole grid,
    rounding-stable points and points where the result selects the oracle's step.  A
    point is rounding-stable when no other FP64 implementation of the same mathematics
    selects another step there than the reference-faithful run: the oracle's real-input
    transform run, its deterministic variants (make_golden.py --stable) and the sampled
    rounding realisations built from their traces (make_golden.py --sampled), whose set
    is validated by implementations held out of it (`heldout`, `heldout_agree`)."""
    ref_d = z["density"].astype(np.float64).reshape(-1)
    ref_s = z["selected"].astype(np.int32).reshape(-1)
    alt_s = z["selected_alt"].astype(np.int32).reshape(-1)
    dens = np.asarray(dens, dtype=np.float64).reshape(-1)
    sel = np.asarray(sel).reshape(-1)
    if "unstable" in z.files:  # the variants and sampled realisations (make_golden.py)
        stable = ~np.unpackbits(z["unstable"], count=ref_s.size).astype(bool)
    else:
        stable = ref_s == alt_s
    same = sel == ref_s
    both = stable & same
    nrm = lambda a: float(np.linalg.norm(a))
    return dict(
        rel_l2=nrm(dens - ref_d) / nrm(ref_d),
        max_abs=float(np.max(np.abs(dens - ref_d))),
        max_rel=float(np.max(np.abs(dens - ref_d)) / np.max(np.abs(ref_d))),
        agree=float(np.mean(same)),
        rel_l2_stable=nrm(dens[stable] - ref_d[stable]) / nrm(ref_d[stable]),
        agree_stable=float(np.mean(same[stable])),
        stable_fraction=float(np.mean(stable)),
        rel_l2_same_step=nrm(dens[both] - ref_d[both]) / nrm(ref_d[both]),
        oracle_r2c_rel_l2=float(z["rel_alt"]),
        oracle_r2c_agree=float(z["agree_alt"]),
    )
