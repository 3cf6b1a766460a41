"""The allocation-free binning entry point (pkde_dirac_sequence_noalloc).

It serves callers that cannot allocate device memory -- a framework whose caching
allocator owns the GPU, or a caller that must not make cudaMalloc/cudaFree calls, which
synchronise the whole device -- by keeping its scratch in a fixed array inside the
library (the call itself still blocks: it synchronises its stream twice).  This test calls it through the C ABI twice in a row and checks each result
against the allocating entry point (pkde_dirac_sequence) with the tolerances of the other
binning tests (counts bit-exact, sums within 1e-14 of the largest cell), and that device
memory use does not change across a call.  The file name sorts last so that a run that
stops at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from oracle.rng import bootstrap_indices

pytestmark = pytest.mark.gpu


def _case(seed, ndim, dims, n, B):
    rng = np.random.default_rng(seed)
    data = rng.standard_normal((ndim, n))
    idx = bootstrap_indices(seed, n, B)
    return data, idx


def test_noalloc_matches_allocating_entry_point(pk):
    import torch
    from pkde_b200 import _lib, raw
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    cases = [(101, 2, (40, 33), 12000, 5), (202, 3, (17, 12, 20), 9000, 4)]
    free_after = []
    for seed, ndim, dims, n, B in cases:
        data, idx = _case(seed, ndim, dims, n, B)
        grid = pk.find_grid(data, grid_dims=dims)
        M_ref, V_ref, C_ref = raw.dirac_sequence(grid, data, idx)  # allocating entry point
        G = int(np.prod(dims))
        d_data = torch.from_numpy(np.ascontiguousarray(data.T)).to(dev)
        d_idx = torch.from_numpy(np.ascontiguousarray(idx)).to(dev)
        d_m = torch.empty(B * G, dtype=torch.float64, device=dev)
        d_v = torch.empty(B * G, dtype=torch.float64, device=dev)
        d_c = torch.empty(B * G, dtype=torch.int32, device=dev)
        gs = _lib.make_grid_struct(grid.lo, grid.hi, grid.h, grid.dims)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(0)[0]
        rc = lib.pkde_dirac_sequence_noalloc(None, ctypes.byref(gs), d_data.data_ptr(), n, d_idx.data_ptr(), B, 0,
                                             d_m.data_ptr(), d_v.data_ptr(), d_c.data_ptr(), None)
        assert rc == 0, lib.pkde_last_error(None)
        torch.cuda.synchronize()
        free_after.append((free_before, torch.cuda.mem_get_info(0)[0]))
        shp = M_ref.shape
        M = d_m.cpu().numpy().reshape(shp)
        V = d_v.cpu().numpy().reshape(shp)
        C = d_c.cpu().numpy().view(np.uint32).reshape(shp)
        assert np.array_equal(C, C_ref)
        assert np.max(np.abs(M - M_ref)) <= 1e-14 * np.max(M_ref)
        assert np.max(np.abs(V - V_ref)) <= 1e-14 * np.max(V_ref)
    # the second call finds the scratch address already looked up: no device memory taken
    assert free_after[1][0] == free_after[1][1]


def test_noalloc_rejects_sizes_beyond_its_scratch(pk):
    import torch
    from pkde_b200 import _lib
    lib = _lib.load()
    n = 16385
    data = np.random.default_rng(0).standard_normal((1, n))
    grid = pk.find_grid(data, grid_dims=(64,))
    gs = _lib.make_grid_struct(grid.lo, grid.hi, grid.h, grid.dims)
    d_data = torch.from_numpy(np.ascontiguousarray(data.T)).cuda()
    d_m = torch.empty(64, dtype=torch.float64, device="cuda")
    ctx = _lib.context(0)
    rc = lib.pkde_dirac_sequence_noalloc(ctx, ctypes.byref(gs), d_data.data_ptr(), n, None, 0, 0, d_m.data_ptr(), None,
                                         None, None)
    assert rc == _lib.PKDE_EINVAL
    assert b"16384" in lib.pkde_last_error(ctx)
    # without a context the message is kept for pkde_last_error(NULL), per thread
    rc = lib.pkde_dirac_sequence_noalloc(None, ctypes.byref(gs), d_data.data_ptr(), n, None, 0, 0, d_m.data_ptr(),
                                         None, None, None)
    assert rc == _lib.PKDE_EINVAL
    assert b"16384" in lib.pkde_last_error(None)
