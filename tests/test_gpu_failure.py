"""Failure detection without a GPU fault: the bounded device waits give up.

piro_set_wait_limit(0) makes every bounded wait (the grid barriers of the
persistent backward-Euler kernel and of the batched step, the stage waits of
the TMA-staged matrix-free step) run out at its first poll, as a wait whose
flag never comes would after its bound.  The call must then report
PIRO_ERR_CUDA with its message, every block must have left the kernel, and
the CUDA context must stay usable: with the limit restored the same objects,
and fresh ones, give the oracle's results.  Nothing here faults, traps or
hangs a GPU: a timed-out wait raises a flag and returns."""
import numpy as np
import pytest

from conftest import f32_bits_equal

pytestmark = pytest.mark.gpu
PIRO_ERR_CUDA = 6


@pytest.fixture
def wait_limit():
    from piro_b200._lib import lib
    L = lib()

    def set_(polls):
        assert L.piro_set_wait_limit(polls) == 0
    yield set_
    L.piro_set_wait_limit(-1)


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("variant", ["resident", "global"])
def test_persistent_be_barrier_gives_up(cuda, oracle, wait_limit, monkeypatch, variant):
    import torch
    from piro_b200 import ops
    from piro_b200._lib import lib
    nx, ny, nz = 40, 32, 24
    N = nx * ny * nz
    rng = np.random.default_rng(4)
    alpha = np.exp(rng.standard_normal(N)).astype(np.float32)
    dt = np.float32(50.0 / (6.0 * alpha.max()))
    L = oracle.laplacian(nx, ny, nz, 3, np.float32(1.0))
    Ls = (L[0], L[1], oracle.csr_rowscale(N, L[0], L[2], alpha))
    I = (np.arange(N + 1, dtype=np.int32), np.arange(N, dtype=np.int32), np.ones(N, np.float32))
    A = oracle.csrgeam2(N, I, np.float32(-dt), Ls)
    b = rng.random(N, dtype=np.float32)
    inter = np.zeros((nz, ny, nx), bool)
    inter[1:-1, 1:-1, 1:-1] = True
    b[~inter.ravel()] = 0.0
    u64, _, _ = oracle.be_cg_f64(nx, ny, nz, A, alpha, b, rtol=1e-13)
    monkeypatch.setenv("PIRO_BE_PERSISTENT", "1" if variant == "resident" else "g")
    Ad, ad = tuple(dev(torch, a) for a in A), dev(torch, alpha)
    s = ops.BESolver(nx, ny, nz, Ad, ad, stencil=(dt, 1.0))
    assert s.persistent_variant == variant
    x = torch.empty(N, dtype=torch.float32, device="cuda")
    wait_limit(0)
    info = s.solve(dev(torch, b), x, rtol=1e-8, strict=False)
    assert info.status == PIRO_ERR_CUDA
    assert b"grid barrier timed out" in lib().piro_last_error()
    wait_limit(-1)
    for sv in (s, ops.BESolver(nx, ny, nz, Ad, ad, stencil=(dt, 1.0))):
        info = sv.solve(dev(torch, b), x, rtol=1e-8)
        assert info.status == 0 and info.rel_residual <= 1e-8
        err = np.abs(x.cpu().numpy().astype(np.float64) - u64).max() / np.abs(u64).max()
        assert err < 1e-6, err
        sv.close()


def test_staged_stencil_stage_wait_gives_up(cuda, oracle, wait_limit):
    import torch
    from piro_b200 import ops
    from piro_b200._lib import PiroError
    nx = ny = nz = 64  # the TMA-staged kernel (16 <= nx <= 256, nx divides 2048)
    N = nx * ny * nz
    rng = np.random.default_rng(9)
    u = rng.random(N, dtype=np.float32)
    alpha = np.exp(rng.standard_normal(N)).astype(np.float32)
    ud, ad = dev(torch, u), dev(torch, alpha)
    out = torch.zeros(N, dtype=torch.float32, device="cuda")
    wait_limit(0)
    ops.stencil_fe_step(nx, ny, nz, 0.01, ud, out, alpha=ad)
    with pytest.raises(PiroError) as e:
        ops.stencil_check()
    assert e.value.status == PIRO_ERR_CUDA and "stage wait timed out" in str(e.value)
    wait_limit(-1)
    ops.stencil_check()  # the flag was cleared by the report
    ops.stencil_fe_step(nx, ny, nz, 0.01, ud, out, alpha=ad)
    ops.stencil_check()
    want = oracle.stencil_fe(nx, ny, nz, np.float32(0.01), u, alpha=alpha)
    assert f32_bits_equal(out.cpu().numpy(), want)


def test_batched_barrier_gives_up(cuda, wait_limit):
    from piro_b200 import ops
    from piro_b200 import workloads as W
    from piro_b200._lib import PiroError
    cfg = W.batched(seed=7, count=10, lo=8, hi=22)
    assert (cfg["scheme"] == 1).any()  # backward-Euler members: the lockstep rounds wait at grid barriers
    B = ops.Batch(cfg["n"], cfg["alpha"], cfg["dt"], cfg["scheme"])
    u0 = W.pack_batch(cfg["fields"], B.offsets, B.total)
    B.set_fields(u0)
    wait_limit(0)
    with pytest.raises(PiroError) as e:
        B.step(1)
    assert e.value.status == PIRO_ERR_CUDA and "grid barrier timed out" in str(e.value)
    wait_limit(-1)
    B.set_fields(u0)
    B.step(1)
    one = B.get_fields()
    B.set_fields(u0)
    B.step(2)  # the pair graph, captured with the restored limit
    info = B.member_info()
    assert np.all(info["status"] == 0)
    C = ops.Batch(cfg["n"], cfg["alpha"], cfg["dt"], cfg["scheme"])
    C.set_fields(u0)
    C.step(1)
    assert np.array_equal(C.get_fields(), one)  # same step as a fresh batch
    B.close()
    C.close()
