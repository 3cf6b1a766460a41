"""TEST INFRASTRUCTURE ONLY: the seeded bootstrap-index generator, restated on the CPU.

The reference draws bootstrap resamples with Julia's ``rand(1:n, n, B)``
(src/KDEs/KDEs.jl:182-191) and, on CUDA, ``CUDA.rand(Int32)`` + ``mod1``
(src/KDEs/KDEs.jl:192-206).  Neither stream can be reproduced outside Julia, so the
C ABI accepts explicit indices, or a seed for this counter-based generator, which the
CUDA library evaluates with the same integer arithmetic (``pkde_boot_index`` in
``csrc/pkde_common.cuh``).  Draw ``j`` of bootstrap ``b`` is

    x = seed + (b*n + j + 1) * 0x9E3779B97F4A7C15        (mod 2**64)
    z = splitmix64 finaliser of x                         (Vigna's published mixer)
    idx = ((z >> 32) * n) >> 32                           (0-based, in [0, n))

and the reference's 1-based index is ``idx + 1``.  Integer arithmetic only: the CPU and
GPU streams are bit-identical.
"""
import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(x):
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = x
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def bootstrap_indices(seed, n_samples, n_bootstraps, one_based=True):
    """Return a (n_bootstraps, n_samples) int32 array: row b is bootstrap column b of the
    reference's n x B index matrix (column-major n x B == C-order (B, n))."""
    n = int(n_samples)
    if n < 1 or n >= 2**31:
        raise ValueError("n_samples must be in [1, 2^31)")
    if n_bootstraps == 0:
        idx = np.arange(n, dtype=np.int64).reshape(1, n)
        return (idx + (1 if one_based else 0)).astype(np.int32)
    out = np.empty((n_bootstraps, n), dtype=np.int32)
    ctr = np.arange(1, n + 1, dtype=np.uint64)
    s = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
    with np.errstate(over="ignore"):
        for b in range(n_bootstraps):
            x = s + (np.uint64(b * n) + ctr) * _GOLDEN
            z = splitmix64(x)
            v = ((z >> np.uint64(32)) * np.uint64(n)) >> np.uint64(32)
            out[b] = v.astype(np.int64) + (1 if one_based else 0)
    return out
