"""The benchmark configurations' own workloads, checked end to end against
the oracle: the 32^3 forward-Euler heat run (bit-exact after 100 steps) and
upwind advection through the csrgeam-merged matrix (bit-exact)."""
import numpy as np
import pytest

from conftest import f32_bits_equal

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_heat_fe_32_hundred_steps_bit_exact(cuda, oracle):
    import torch
    from piro_b200 import fe, workloads as W
    c = W.heat_fe_32()
    nx, ny, nz = c["n"]
    N = nx * ny * nz
    A = oracle.laplacian(nx, ny, nz, 3, np.float32(1.0))
    As = (A[0], A[1], oracle.csr_rowscale(N, A[0], A[2], c["alpha"]))
    ref = oracle.fe_csr(nx, ny, nz, As, c["dt"], c["u0"], c["steps"])
    run = fe.FeRunner(nx, ny, nz, dev(torch, c["alpha"]), float(c["dt"]))
    u = run.run(dev(torch, c["u0"]), c["steps"], graph=True)
    assert f32_bits_equal(u.cpu().numpy(), ref)
    # structure of the 32^3 matrix: nnz and the 10.0 boundary entries
    assert run.A[2].numel() == 223232
    assert int((run.A_unscaled_tens == 10).sum()) == 5768


@pytest.mark.parametrize("n,steps", [(24, 30), (41, 12)])
def test_advection_merged_operator_bit_exact(cuda, oracle, n, steps):
    import torch
    from piro_b200 import fe, workloads as W
    c = W.advection(n)
    N = n ** 3
    G = oracle.gradient3(n, n, n, 1, c["gnorm"])
    D = oracle.csrgeam3(N, *G, c["v"])
    ref = oracle.fe_csr(n, n, n, D, c["dt"], c["u0"], steps)
    run = fe.AdvectionRunner(n, n, n, dev(torch, c["v"]), float(c["dt"]), float(c["gnorm"]))
    u = run.run(dev(torch, c["u0"]), steps, graph=True)
    assert f32_bits_equal(u.cpu().numpy(), ref)
