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


def test_noalloc_call_moves_no_device_memory(cuda):
    """The property the entry point exists for: once its first call on the
    device has loaded the library's scratch array, a call changes neither the
    device's free memory nor what torch's allocator holds."""
    import torch
    from piro_b200 import ops
    from piro_b200._lib import lib
    L = lib()
    n = (48, 40, 36)
    N = n[0] * n[1] * n[2]
    G = _grad3(torch, ops, n, 3)
    v = torch.from_numpy(np.random.default_rng(5).standard_normal(3 * N).astype(np.float32)).cuda()
    nnz = sum(int(g[2].numel()) for g in G)
    outs = [(torch.empty(N + 1, dtype=torch.int32, device="cuda"), torch.empty(nnz, dtype=torch.int32, device="cuda"),
             torch.empty(nnz, dtype=torch.float32, device="cuda")) for _ in range(2)]
    s = torch.cuda.current_stream().cuda_stream
    args = [g.data_ptr() for grad in G for g in grad] + [v.data_ptr()]

    def call(o):
        st = L.piro_csrgeam3_noalloc(N, *args, o[0].data_ptr(), o[1].data_ptr(), o[2].data_ptr(), s)
        assert st == 0, L.piro_last_error()
        torch.cuda.synchronize()
    call(outs[0])  # the first call on the device (module load, address lookup)
    free0, _ = torch.cuda.mem_get_info()
    alloc0, res0 = torch.cuda.memory_allocated(), torch.cuda.memory_reserved()
    call(outs[1])
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert torch.cuda.memory_allocated() == alloc0 and torch.cuda.memory_reserved() == res0
    for a, b in zip(outs[0], outs[1]):
        assert torch.equal(a.view(torch.int32), b.view(torch.int32))


def test_noalloc_merge_at_its_row_limit_vs_oracle(cuda, oracle):
    """16,777,216 rows (the 256^3 gradients): the scan scratch is nearly full
    (4,096 scan blocks); the merge must equal the oracle's csrgeam3 exactly."""
    import torch
    from piro_b200 import ops
    from piro_b200._lib import lib
    L = lib()
    n = (256, 256, 256)
    N = n[0] * n[1] * n[2]
    assert N == 16777216
    G = _grad3(torch, ops, n, 1)
    v_h = np.random.default_rng(7).standard_normal(3 * N).astype(np.float32)
    v = torch.from_numpy(v_h).cuda()
    got = _call_noalloc(L, torch, N, G, v)
    Gh = [tuple(t.cpu().numpy() for t in g) for g in G]
    del G
    want = oracle.csrgeam3(N, Gh[0], Gh[1], Gh[2], v_h)
    assert np.array_equal(got[0].cpu().numpy(), want[0])
    assert np.array_equal(got[1].cpu().numpy(), want[1])
    assert np.array_equal(got[2].cpu().numpy().view(np.uint32), want[2].view(np.uint32))


def test_noalloc_rejects_rows_beyond_its_scratch(cuda):
    from piro_b200._lib import lib
    L = lib()
    too_many = 16777216 + 1
    st = L.piro_csrgeam3_noalloc(too_many, *([None] * 13), None)
    assert st == 1  # PIRO_ERR_ARG, before any device work
    assert b"16777216" in L.piro_last_error()
    st = L.piro_csrgeam3_noalloc(1000, *([None] * 13), None)
    assert st == 1 and b"null pointer" in L.piro_last_error()
