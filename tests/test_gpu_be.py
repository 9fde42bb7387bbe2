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


@pytest.mark.parametrize("n,contrast", [((18, 18, 18), 0.0), ((34, 30, 26), 1.5), ((40, 33, 35), 1.0), ((13, 11, 9), 0.5)])
@pytest.mark.parametrize("inner", ["csr", "stencil", "stencil-persistent"])
def test_be_pcg_reaches_fp64_residual(cuda, oracle, n, contrast, inner, monkeypatch):
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
    monkeypatch.setenv("PIRO_BE_PERSISTENT", "1" if inner == "stencil-persistent" else "0")
    s = ops.BESolver(nx, ny, nz, Ad, dev(torch, alpha), stencil=(dt, 1.0) if inner != "csr" else None)
    assert s.inner_operator == inner
    x = torch.empty(N, dtype=torch.float32, device="cuda")
    info = s.solve(dev(torch, b), x, rtol=1e-8)
    assert info.status == 0 and info.rel_residual <= 1e-8
    assert np.array_equal(h(x)[~inter.ravel()], b[~inter.ravel()])  # boundary held at b
    # error of the FP32 field against the FP64-only solve
    xs = h(x).astype(np.float64)
    err = np.abs(xs - u64).max() / np.abs(u64).max()
    assert err < 1e-6, err
    s.close()


@pytest.mark.parametrize("persist", ["0", "1"])
def test_be_nonzero_dirichlet_boundary(cuda, oracle, monkeypatch, persist):
    """Boundary values enter the interior system through A's interior-boundary
    block (including the 10.0 entries): the FP64 oracle and the device agree."""
    import torch
    from piro_b200 import ops
    nx, ny, nz = 20, 17, 15
    N = nx * ny * nz
    rng = np.random.default_rng(11)
    alpha = np.exp(0.7 * rng.standard_normal(N)).astype(np.float32)
    dt = np.float32(20.0 / (6.0 * alpha.max()))
    A = be_matrix(oracle, nx, ny, nz, alpha, dt)
    b = (rng.random(N, dtype=np.float32) + np.float32(0.5)).astype(np.float32)
    u64, _, _ = oracle.be_cg_f64(nx, ny, nz, A, alpha, b, rtol=1e-13)
    monkeypatch.setenv("PIRO_BE_PERSISTENT", persist)
    s = ops.BESolver(nx, ny, nz, tuple(dev(torch, a) for a in A), dev(torch, alpha), stencil=(dt, 1.0))
    x = torch.empty(N, dtype=torch.float32, device="cuda")
    info = s.solve(dev(torch, b), x, rtol=1e-8)
    assert info.status == 0 and info.rel_residual <= 1e-8
    err = np.abs(h(x).astype(np.float64) - u64).max() / np.abs(u64).max()
    assert err < 1e-6, err
    s.close()


def test_stencil_operator_rejected_for_other_schemes(cuda, oracle):
    """The matrix-free inner operator is only taken when A's interior block
    is the central stencil; an upwind-assembled A falls back to CSR."""
    import torch
    from piro_b200 import ops
    nx, ny, nz = 12, 11, 10
    N = nx * ny * nz
    alpha = np.full(N, 0.5, np.float32)
    L = oracle.laplacian(nx, ny, nz, 1, np.float32(1.0))
    Ls = (L[0], L[1], oracle.csr_rowscale(N, L[0], L[2], alpha))
    I = (np.arange(N + 1, dtype=np.int32), np.arange(N, dtype=np.int32), np.ones(N, np.float32))
    A = oracle.csrgeam2(N, I, np.float32(-0.1), Ls)
    s = ops.BESolver(nx, ny, nz, tuple(dev(torch, a) for a in A), dev(torch, alpha), stencil=(0.1, 1.0))
    assert s.inner_operator == "csr"
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
