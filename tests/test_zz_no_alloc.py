"""The allocation-free merge entry point, checked through the C ABI.

piro_csrgeam3_noalloc exists for callers that cannot give the library device
memory: it runs the same v.grad merge as piro_csrgeam3 with the scan scratch
held in a fixed array inside the library.  Its results must equal those of
piro_csrgeam3 (which takes caller workspace) exactly -- the outputs are
integer structures and single products -- on consecutive calls that reuse the
shared array.  This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _grad3(torch, ops, n, scheme):
    return [ops.csr_gradient(*n, scheme, a, 2.0) for a in range(3)]


def _call_noalloc(lib, torch, N, G, v):
    nnz = sum(int(g[2].numel()) for g in G)
    rp = torch.full((N + 1,), -7, dtype=torch.int32, device="cuda")
    col = torch.full((nnz,), -7, dtype=torch.int32, device="cuda")
    val = torch.full((nnz,), float("nan"), dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    st = lib.piro_csrgeam3_noalloc(N, G[0][0].data_ptr(), G[0][1].data_ptr(), G[0][2].data_ptr(),
                                   G[1][0].data_ptr(), G[1][1].data_ptr(), G[1][2].data_ptr(),
                                   G[2][0].data_ptr(), G[2][1].data_ptr(), G[2][2].data_ptr(), v.data_ptr(),
                                   rp.data_ptr(), col.data_ptr(), val.data_ptr(), s)
    assert st == 0, lib.piro_last_error()
    torch.cuda.synchronize()
    return rp, col, val


def test_noalloc_merge_matches_workspace_merge_on_consecutive_calls(cuda):
    import torch
    from piro_b200 import ops
    from piro_b200._lib import lib
    L = lib()
    rng = np.random.default_rng(42)
    # two calls in a row with different sizes, schemes and velocities: the
    # second reuses (and must not be disturbed by) what the first left behind
    for n, scheme in [((40, 36, 30), 1), ((64, 50, 45), 3)]:
        N = n[0] * n[1] * n[2]
        G = _grad3(torch, ops, n, scheme)
        v = torch.from_numpy(rng.standard_normal(3 * N).astype(np.float32)).cuda()
        want = ops.csrgeam3(N, *G, v)
        got = _call_noalloc(L, torch, N, G, v)
        assert torch.equal(got[0], want[0])
        assert torch.equal(got[1], want[1])
        assert torch.equal(got[2].view(torch.int32), want[2].view(torch.int32))


def test_noalloc_rejects_rows_beyond_its_scratch(cuda):
    from piro_b200._lib import lib
    L = lib()
    too_many = 16777216 + 1
    st = L.piro_csrgeam3_noalloc(too_many, *([None] * 13), None)
    assert st == 1  # PIRO_ERR_ARG, before any device work
    assert b"16777216" in L.piro_last_error()
