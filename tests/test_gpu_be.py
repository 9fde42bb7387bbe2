"""Backward Euler on the device against FP64 oracle solves."""
import numpy as np
import pytest

from conftest import f32_bits_equal

pytestmark = pytest.mark.gpu


def h(t):
    return t.cpu().numpy()


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def be_matrix(oracle, nx, ny, nz, alpha, dt):
    N = nx * ny * nz
    L = oracle.laplacian(nx, ny, nz, 3, np.float32(1.0))
    Ls = (L[0], L[1], oracle.csr_rowscale(N, L[0], L[2], alpha))
    I = (np.arange(N + 1, dtype=np.int32), np.arange(N, dtype=np.int32), np.ones(N, np.float32))
    return oracle.csrgeam2(N, I, np.float32(-dt), Ls)


@pytest.mark.parametrize("n,contrast", [((18, 18, 18), 0.0), ((34, 30, 26), 1.5)])
def test_be_pcg_reaches_fp64_residual(cuda, oracle, n, contrast):
    import torch
    from piro_b200 import ops
    nx, ny, nz = n
    N = nx * ny * nz
    rng = np.random.default_rng(7)
    alpha = np.exp(contrast * rng.standard_normal(N)).astype(np.float32)
    dt = np.float32(50.0 / (6.0 * alpha.max()))
    A = be_matrix(oracle, nx, ny, nz, alpha, dt)
    b = rng.random(N, dtype=np.float32)
    # boundary values stay b (Dirichlet); make them zero like the configs
    inter = np.zeros((nz, ny, nx), bool)
    inter[1:-1, 1:-1, 1:-1] = True
    b[~inter.ravel()] = 0.0
    u64, its, rel = oracle.be_cg_f64(nx, ny, nz, A, alpha, b, rtol=1e-13)
    assert its > 0 and rel < 1e-12
    Ad = tuple(dev(torch, a) for a in A)
    s = ops.BESolver(nx, ny, nz, Ad, dev(torch, alpha))
    x = torch.empty(N, dtype=torch.float32, device="cuda")
    info = s.solve(dev(torch, b), x, rtol=1e-8)
    assert info.status == 0 and info.rel_residual <= 1e-8
    # error of the FP32 field against the FP64-only solve
    xs = h(x).astype(np.float64)
    err = np.abs(xs - u64).max() / np.abs(u64).max()
    assert err < 1e-6, err
    s.close()


def test_be_jli_matches_oracle(cuda, oracle):
    import torch
    from piro_b200 import ops
    nx, ny, nz = 10, 10, 33
    N = nx * ny * nz
    A = oracle.laplacian(nx, ny, nz, 2, np.float32(1.0))
    rng = np.random.default_rng(3)
    b = rng.random(N, dtype=np.float32)
    xr, itr = oracle.be_jli(nx, ny, nz, A, np.float32(0.001), b)
    x, it = ops.be_jli(nx, ny, nz, tuple(dev(torch, a) for a in A), 0.001, dev(torch, b))
    assert it == itr
    np.testing.assert_allclose(h(x), xr, rtol=1e-6, atol=1e-6)
