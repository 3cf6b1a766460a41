"""Seeded synthetic sample sets with the shapes and distributions of the benchmark
configurations (the reference publishes no dataset; its own benchmark draws N(0, I)).

Every generator returns a float64 array of shape (N, n) -- the reference's N x n sample
matrix, one column per sample -- plus the grid specification it is estimated on.
"""
import math

import numpy as np


def gaussian_1d(n=10_000, seed=0):
    """1-D N(0,1); grid of 1,024 points on [min - 3 sd, max + 3 sd]."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((1, n))
    sd = float(np.std(x[0], ddof=1))
    pad = 3.0 * sd
    return x, dict(dims=(1024,), grid_padding=[pad])


def gmm_2d(n=1_000_000, seed=1, dims=(512, 512)):
    """2-D three-component mixture: weights 0.5/0.3/0.2, means (0,0), (3,2), (-2,3),
    covariances [[1,.6],[.6,1]], 0.5 I, [[2,-.8],[-.8,1]]; default 10 % padding."""
    rng = np.random.default_rng(seed)
    w = np.array([0.5, 0.3, 0.2])
    mus = np.array([[0.0, 0.0], [3.0, 2.0], [-2.0, 3.0]])
    covs = np.array([[[1.0, 0.6], [0.6, 1.0]], [[0.5, 0.0], [0.0, 0.5]], [[2.0, -0.8], [-0.8, 1.0]]])
    comp = rng.choice(3, size=n, p=w)
    out = np.empty((n, 2))
    for c in range(3):
        sel = comp == c
        out[sel] = rng.multivariate_normal(mus[c], covs[c], size=int(sel.sum()))
    return out.T.copy(), dict(dims=tuple(dims))


def banana_t_3d(n=4_000_000, seed=2, dims=(128, 128, 128)):
    """3-D: 70 % banana (x ~ N(0,1), y = 0.5 x^2 + N(0, 0.3^2), z ~ N(0,1)) and 30 %
    isotropic Student-t with 3 degrees of freedom; default 10 % padding (the grid
    encloses every sample, as the reference's bounds check requires)."""
    rng = np.random.default_rng(seed)
    nb = int(round(0.7 * n))
    nt = n - nb
    x = rng.standard_normal(nb)
    y = 0.5 * x * x + 0.3 * rng.standard_normal(nb)
    z = rng.standard_normal(nb)
    ban = np.stack([x, y, z], axis=1)
    g = rng.standard_normal((nt, 3))
    chi = rng.chisquare(3, size=nt)
    tt = g / np.sqrt(chi / 3.0)[:, None]
    out = np.concatenate([ban, tt], axis=0)
    rng.shuffle(out, axis=0)
    return out.T.copy(), dict(dims=tuple(dims))


def random_mixture(ndim, n, rng, n_comp=None):
    """Gaussian mixture with 1-4 random components (random means, scales, weights)."""
    k = int(rng.integers(1, 5)) if n_comp is None else n_comp
    w = rng.dirichlet(np.ones(k))
    comp = rng.choice(k, size=n, p=w)
    mus = rng.uniform(-3, 3, size=(k, ndim))
    out = np.empty((n, ndim))
    for c in range(k):
        sel = comp == c
        a = rng.normal(size=(ndim, ndim)) * 0.4 + np.eye(ndim) * rng.uniform(0.4, 1.2)
        out[sel] = mus[c] + rng.standard_normal((int(sel.sum()), ndim)) @ a.T
    return out.T.copy()


def batched_mix(count=256, seed=3, n_range=(1e3, 1e6), n_steps=100, n_boot=32):
    """Uneven estimations: dims uniform in {1,2,3}, samples log-uniform, grids 256-4096
    (1-D), 128^2-512^2 (2-D), 32^3-96^3 (3-D)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        ndim = int(rng.integers(1, 4))
        n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
        if ndim == 1:
            g = (int(2 ** rng.integers(8, 13)),)
        elif ndim == 2:
            s = int(rng.choice([128, 192, 256, 320, 384, 512]))
            g = (s, s)
        else:
            s = int(rng.choice([32, 48, 64, 80, 96]))
            g = (s, s, s)
        out.append(dict(data=random_mixture(ndim, n, rng), dims=g, n_steps=n_steps, n_bootstraps=n_boot))
    return out


def served_mix(count=48, seed=4, n_range=(1e3, 4e6), n_steps=100, n_boot=32):
    """Served requests: dims uniform in 1..4, samples log-uniform in n_range from random
    1-4 component Gaussian mixtures, grids 256-4096 (1-D), 128^2-512^2 (2-D), 32^3-128^3
    (3-D), 16^4-48^4 (4-D)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        ndim = int(rng.integers(1, 5))
        n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
        if ndim == 1:
            g = (int(2 ** rng.integers(8, 13)),)
        elif ndim == 2:
            s = int(rng.choice([128, 192, 256, 320, 384, 512]))
            g = (s, s)
        elif ndim == 3:
            s = int(rng.choice([32, 48, 64, 96, 128]))
            g = (s, s, s)
        else:
            s = int(rng.choice([16, 24, 32, 48]))
            g = (s, s, s, s)
        out.append(dict(data=random_mixture(ndim, n, rng), dims=g, n_steps=n_steps, n_bootstraps=n_boot))
    return out


def batched_small_mix(count=256, seed=5, n_range=(1e3, 1e4), n_steps=100, n_boot=32):
    """Small estimations, where one estimation alone cannot fill the GPU: dims 1 or 2,
    samples log-uniform in n_range, grids 256-1024 (1-D) and 64^2-128^2 (2-D)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        ndim = int(rng.integers(1, 3))
        n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
        if ndim == 1:
            g = (int(2 ** rng.integers(8, 11)),)
        else:
            s = int(rng.choice([64, 96, 128]))
            g = (s, s)
        out.append(dict(data=random_mixture(ndim, n, rng), dims=g, n_steps=n_steps, n_bootstraps=n_boot))
    return out
