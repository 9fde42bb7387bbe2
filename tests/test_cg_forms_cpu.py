"""The CG iteration of the persistent backward-Euler kernel, restated in
numpy and checked against textbook Jacobi-PCG on the same system.

The kernel's resident form does not run PCG as written: phase A forms
q = A p by the recurrence q = A z + beta q_old, stores no r (phase B forms
r = z A_rr - a q from the cell's z), and defers d += a p to the next phase A.
In exact arithmetic these are the same iterates; the test shows it in FP64
(the iterates agree to rounding) and that the FP32 form converges like FP32
PCG.  The system is the interior SPD form S = diag(alpha)^-1 A_II of
A = I - dt diag(alpha) L, as the solver uses it.
"""
import numpy as np
import pytest
import scipy.sparse as sp


def _system(oracle, n, dt, seed):
    nx, ny, nz = n
    N = nx * ny * nz
    rng = np.random.default_rng(seed)
    alpha = (np.exp(1.2 * rng.standard_normal(N)) * 0.01).astype(np.float32)
    L = oracle.laplacian(nx, ny, nz, 3, np.float32(1.0))
    Ls = (L[0], L[1], oracle.csr_rowscale(N, L[0], L[2], alpha))
    I = (np.arange(N + 1, dtype=np.int32), np.arange(N, dtype=np.int32), np.ones(N, np.float32))
    A = oracle.csrgeam2(N, I, np.float32(-dt), Ls)
    M = sp.csr_matrix((A[2].astype(np.float64), A[1], A[0]), shape=(N, N))
    x, y, z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    inter = ((x > 0) & (x < nx - 1) & (y > 0) & (y < ny - 1) & (z > 0) & (z < nz - 1)).transpose(2, 1, 0).reshape(-1)
    Aii = M[inter][:, inter].tocsr()
    a = alpha[inter].astype(np.float64)
    b = rng.random(int(inter.sum()))
    return Aii, a, b


def _pcg(Aii, a, b, iters, dtype):
    """Textbook Jacobi-PCG on S x = b/alpha with the alpha-weighted inner product."""
    A = Aii.astype(dtype)
    diag = A.diagonal()
    w = (1.0 / a).astype(dtype)
    x = np.zeros_like(b, dtype=dtype)
    r = b.astype(dtype).copy()
    z = r / diag
    p = z.copy()
    rz = np.dot(r * w, z)
    xs = []
    for _ in range(iters):
        q = A @ p
        alpha_k = rz / np.dot(p * w, q)
        x = x + alpha_k * p
        r = r - alpha_k * q
        z = r / diag
        rzn = np.dot(r * w, z)
        xs.append(x.copy())
        if not rzn > 0:  # converged to the last bit
            break
        p = z + (rzn / rz) * p
        rz = rzn
    return xs


def _kernel_form(Aii, a, b, iters, dtype):
    """The resident kernel's iteration: q by recurrence, r = z A_rr - a q,
    d += a p one phase A later."""
    A = Aii.astype(dtype)
    diag = A.diagonal()
    w = (1.0 / a).astype(dtype)
    d = np.zeros_like(b, dtype=dtype)
    z = (b.astype(dtype)) / diag  # the sweep's first z (x = 0: r = b)
    p = np.zeros_like(d)
    q = np.zeros_like(d)
    rz = np.dot(z * diag * w, z)
    beta, fa_prev = dtype(0), dtype(0)
    xs = []
    for _ in range(iters):
        # phase A
        d = d + fa_prev * p
        q = A @ z + beta * q
        p = z + beta * p
        pq = np.dot(p * w, q)
        fa = rz / pq
        # phase B
        r = z * diag - fa * q
        z = r / diag
        rzn = np.dot(r * w, z)
        xs.append(d + fa * p)  # the correction with this iteration's deferred term
        if not rzn > 0:  # converged to the last bit
            break
        beta = rzn / rz
        rz = rzn
        fa_prev = fa
    return xs


@pytest.mark.parametrize("n,dt", [((14, 12, 10), 8.0), ((10, 16, 13), 60.0)])
def test_kernel_cg_form_equals_pcg_in_fp64(oracle, n, dt):
    Aii, a, b = _system(oracle, n, dt, 41)
    ref = _pcg(Aii, a, b, 25, np.float64)
    got = _kernel_form(Aii, a, b, 25, np.float64)
    scale = np.abs(ref[-1]).max()
    for k in (0, 4, 12, 24):
        assert np.abs(got[k] - ref[k]).max() <= 1e-10 * scale, k


def test_kernel_cg_form_converges_like_fp32_pcg(oracle):
    Aii, a, b = _system(oracle, (16, 14, 12), 40.0, 42)
    x64 = sp.linalg.spsolve(Aii.tocsc(), b)
    err = []
    for form in (_pcg, _kernel_form):
        xs = form(Aii, a, b, 60, np.float32)
        e = [np.abs(x.astype(np.float64) - x64).max() / np.abs(x64).max() for x in xs]
        err.append(e)
        assert min(e) <= 1e-5
    # the same error history, to FP32 rounding, while the error is above it
    for k in range(0, min(30, len(err[0]), len(err[1])), 5):
        assert abs(err[0][k] - err[1][k]) <= 1e-3 * err[0][k] + 1e-6, k


@pytest.mark.parametrize("n,scheme", [((9, 8, 7), 3), ((12, 6, 10), 3)])
def test_matrix_free_residual_with_side_matrix_equals_csr(oracle, n, scheme):
    """The FP64 residual the stencil solver forms without streaming A: on
    interior rows the 7-point stencil over interior neighbours with the
    coefficients fl(1 + fl(-dt fl(alpha vself))) and fl(-dt fl(alpha vnb)),
    plus the row's entries in boundary columns copied from A (PIRO's 10.0
    values among them), with x = b on the boundary -- equals b - A x."""
    nx, ny, nz = n
    N = nx * ny * nz
    rng = np.random.default_rng(43)
    dt = np.float32(5.0)
    alpha = (np.exp(rng.standard_normal(N)) * 0.01).astype(np.float32)
    L = oracle.laplacian(nx, ny, nz, scheme, np.float32(1.0))
    Ls = (L[0], L[1], oracle.csr_rowscale(N, L[0], L[2], alpha))
    I = (np.arange(N + 1, dtype=np.int32), np.arange(N, dtype=np.int32), np.ones(N, np.float32))
    A = oracle.csrgeam2(N, I, -dt, Ls)
    M = sp.csr_matrix((A[2].astype(np.float64), A[1], A[0]), shape=(N, N))
    x3, y3, z3 = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    to_flat = lambda a3: a3.transpose(2, 1, 0).reshape(-1)
    X, Y, Z = to_flat(x3), to_flat(y3), to_flat(z3)
    inter = (X > 0) & (X < nx - 1) & (Y > 0) & (Y < ny - 1) & (Z > 0) & (Z < nz - 1)
    b = rng.random(N).astype(np.float32)
    x = np.where(inter, rng.standard_normal(N), b.astype(np.float64))
    want = b.astype(np.float64) - M @ x
    # the side matrix: entries of interior rows in boundary columns, exactly A's
    side = M.multiply(inter[:, None]).tocsr()
    side = side[:, ~inter] @ x[~inter]
    vself, vnb = np.float32(-6.0), np.float32(1.0)
    cd = (np.float32(1.0) + (-dt) * (alpha * vself)).astype(np.float64)
    co = ((-dt) * (alpha * vnb)).astype(np.float64)
    sxy = nx * ny
    nb = np.zeros(N)
    for off, ok in ((-1, X > 1), (1, X < nx - 2), (-nx, Y > 1), (nx, Y < ny - 2), (-sxy, Z > 1), (sxy, Z < nz - 2)):
        idx = np.arange(N) + off
        nb += np.where(ok & inter, x[np.clip(idx, 0, N - 1)], 0.0)
    got = b.astype(np.float64) - (cd * x + co * nb + side)
    assert np.abs(got[inter] - want[inter]).max() <= 1e-12 * np.abs(want[inter]).max()
