"""The allocation-free divergence statistics (ffx_divergence_stats_static).

Some callers cannot allocate device memory when they need the statistics (a
host that has handed its device memory to its own pool, a real-time callback
that must not call cudaMalloc, a C caller with no allocator). This entry point
keeps its scratch in a fixed array inside the library. Here it is called
through the C ABI twice in a row, on different data, and each result is
compared with the workspace-based ffx_divergence_stats. The file name sorts
last so a run that stops at the first failure has already run everything else;
the test also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from fluxfx_b200 import _native as N

pytestmark = pytest.mark.gpu

def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _workspace_stats(lib, before, after):
    n = before.numel()
    ws = torch.zeros(lib.ffx_divergence_stats_workspace(n) // 8 + 1, dtype=torch.float64, device='cuda')
    out = torch.zeros(8, dtype=torch.float64, device='cuda')
    N.check(lib.ffx_divergence_stats(n, _ptr(before), _ptr(after), _ptr(out), _ptr(ws), ws.numel() * 8, None))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_static_scratch_stats_match_workspace_stats_on_two_calls():
    lib = N.load()
    rng = np.random.default_rng(99)
    out = torch.zeros(8, dtype=torch.float64, device='cuda')
    for n in (1_000_003, 70_001):        # second call is smaller: stale partials must not leak in
        before = torch.as_tensor(rng.normal(size=n).astype(np.float32)).cuda()
        after = torch.as_tensor((rng.normal(size=n) * 1e-3).astype(np.float32)).cuda()
        expected = _workspace_stats(lib, before, after)
        out.fill_(-1.0)
        N.check(lib.ffx_divergence_stats_static(n, _ptr(before), _ptr(after), _ptr(out), None))
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert got[6] == n and got[7] == 0
        # the same kernels with the same block count: the results must be identical
        assert np.array_equal(got, expected), (got, expected)
        assert got[2] == np.abs(before.cpu().numpy().astype(np.float64)).max()


def test_static_scratch_rejects_invalid_counts_and_pointers():
    lib = N.load()
    x = torch.zeros(4, device='cuda')
    out = torch.zeros(8, dtype=torch.float64, device='cuda')
    for count in (0, -5):
        assert lib.ffx_divergence_stats_static(count, _ptr(x), _ptr(x), _ptr(out), None) == N.FFX_ERR_INVALID
        assert b'must be at least 1' in lib.ffx_last_error()
    assert lib.ffx_divergence_stats_static(4, None, _ptr(x), _ptr(out), None) == N.FFX_ERR_INVALID
    assert b'NULL pointer' in lib.ffx_last_error()
