"""Scheme 27: the hash-table LU against PIRO's own factorization
(tests/golden/ht_lu.npz, made by tests/golden/make_lu_golden.py from the
reference build), and the solve that scheme 27 gains here."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("n,suffix", [((6, 5, 4), ""), ((5, 5, 5), ""), ((7, 6, 5), ""), ((6, 5, 4), "_ts30011")])
def test_ht_lu_matches_reference(cuda, n, suffix):
    import torch
    from piro_b200 import ops
    g = np.load(os.path.join(HERE, "golden", "ht_lu.npz"))
    nx, ny, nz = n
    tag = f"{nx}x{ny}x{nz}{suffix}"
    N, ts = nx * ny * nz, int(g[f"ts_{tag}"])
    A = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
    keys, vals = ops.ht_build(N, *A, ts)
    assert np.array_equal(keys.cpu().numpy(), g[f"keys0_{tag}"].astype(np.int64))
    assert np.array_equal(vals.cpu().numpy(), g[f"vals0_{tag}"])
    ops.ht_lu_reference(N, keys, vals, ts)
    torch.cuda.synchronize()
    k = keys.cpu().numpy()
    assert np.array_equal(k, g[f"keys_{tag}"].astype(np.int64))  # slots, fill-in order and deletions
    live = k >= 0
    assert np.array_equal(vals.cpu().numpy()[live], g[f"vals_{tag}"][live])  # bit for bit


def test_ht_lu_full_table_is_reported(cuda):
    from piro_b200 import ops
    from piro_b200._lib import PiroError
    nx = ny = nz = 6
    N = nx * ny * nz
    A = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
    ts = A[2].numel() + 7  # no room for the fill-in
    keys, vals = ops.ht_build(N, *A, ts)
    with pytest.raises(PiroError) as e:
        ops.ht_lu_reference(N, keys, vals, ts)
    assert e.value.status == 4  # PIRO_ERR_TABLE_FULL


def _fp32_nopivot_berr(Ad, b):
    """Backward error of a plain FP32 elimination without pivoting (numpy), the
    yardstick for a matrix whose elements grow during the elimination."""
    import scipy.linalg as sl
    N = Ad.shape[0]
    U = Ad.astype(np.float32)
    for k in range(N - 1):
        f = U[k + 1:, k] / U[k, k]
        U[k + 1:, k + 1:] -= np.outer(f, U[k, k + 1:]).astype(np.float32)
        U[k + 1:, k] = f
    y = sl.solve_triangular(np.tril(U, -1) + np.eye(N, dtype=np.float32), b, lower=True, unit_diagonal=True)
    x = sl.solve_triangular(np.triu(U), y).astype(np.float64)
    return np.abs(Ad @ x - b).max() / (np.abs(Ad).sum(1).max() * np.abs(x).max())


# dt 0.05: well conditioned (cond ~ 10); dt 0.7: PIRO's 10.0 boundary entries
# make the elements grow ~1e4 during elimination without pivoting
@pytest.mark.parametrize("n,dt", [((8, 7, 6), 0.05), ((12, 10, 9), 0.05), ((8, 7, 6), 0.7), ((12, 10, 9), 0.7),
                                  ((40, 3, 3), 0.05), ((3, 3, 40), 0.05)])
def test_ht_lu_solve(cuda, n, dt):
    import torch
    from piro_b200 import ops
    nx, ny, nz = n
    N = nx * ny * nz
    L = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
    bw = nx * ny
    ts = ops.ht_table_size(L[2].numel(), N, 1)
    keys, vals = ops.ht_build(N, *L, ts)  # the operator's table: the factor scales and shifts it
    A = ops.csrgeam2(N, ops.csr_identity(N), -dt, L)  # I - dt L, all rows
    Ad = np.zeros((N, N))
    rp, col, val = (t.cpu().numpy() for t in A)
    for r in range(N):
        for k in range(rp[r], rp[r + 1]):
            Ad[r, col[k]] += val[k]
    cond = np.linalg.cond(Ad)
    lu = ops.HtLu(N, bw, keys, vals, ts, 1.0, -dt)
    rng = np.random.default_rng(3)
    for _ in range(2):
        b = rng.random(N).astype(np.float32)
        x = lu.solve(torch.from_numpy(b).cuda()).cpu().numpy().astype(np.float64)
        ref = np.linalg.solve(Ad, b.astype(np.float64))
        berr = np.abs(Ad @ x - b).max() / (np.abs(Ad).sum(1).max() * np.abs(x).max())
        if dt == 0.05:
            assert berr <= 2e-6
            assert np.abs(x - ref).max() <= 4 * cond * 6e-8 * np.abs(ref).max()
        else:
            assert berr <= 4 * _fp32_nopivot_berr(Ad, b)


def test_ht_lu_factor_matches_elimination(cuda):
    """The band after the factor: U and the multipliers of an FP32
    elimination without pivoting in the same operation order, bit for bit."""
    import torch
    from piro_b200 import ops
    nx, ny, nz = 6, 5, 4
    N, bw, dt = nx * ny * nz, nx * ny, np.float32(0.05)
    L = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
    ts = ops.ht_table_size(L[2].numel(), N, 1)
    keys, vals = ops.ht_build(N, *L, ts)
    lu = ops.HtLu(N, bw, keys, vals, ts, 1.0, float(-dt))
    W = 2 * bw + 1
    band = lu.band[: N * W * 4].view(torch.float32).cpu().numpy().reshape(N, W)
    rp, col, val = (t.cpu().numpy() for t in L)
    U = np.zeros((N, N), np.float32)
    for r in range(N):
        for k in range(rp[r], rp[r + 1]):
            U[r, col[k]] = np.float32(-dt) * val[k]
        U[r, r] = np.float32(1.0) + U[r, r]
    for k in range(N - 1):
        f = U[k + 1:, k] / U[k, k]
        U[k + 1:, k + 1:] -= np.outer(f, U[k, k + 1:]).astype(np.float32)
        U[k + 1:, k] = f
    got = np.zeros((N, N), np.float32)
    for r in range(N):
        for d in range(-bw, bw + 1):
            if 0 <= r + d < N:
                got[r, r + d] = band[r, d + bw]
    assert np.array_equal(got, U), np.abs(got - U).max()


def test_ht_lu_zero_pivot_is_reported(cuda):
    """PIRO's boundary quirk puts 10.0 at (0, 0) of the Laplacian; with
    dt = 0.1 (FP32) A(0, 0) = 1 - dt*10 is exactly zero and elimination
    without pivoting cannot go on."""
    from piro_b200 import ops
    from piro_b200._lib import PiroError
    nx, ny, nz = 8, 7, 6
    N = nx * ny * nz
    L = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
    ts = ops.ht_table_size(L[2].numel(), N, 1)
    keys, vals = ops.ht_build(N, *L, ts)
    with pytest.raises(PiroError, match="zero pivot at row 0") as e:
        ops.HtLu(N, nx * ny, keys, vals, ts, 1.0, -0.1)
    assert e.value.status == 12  # PIRO_ERR_ZERO_PIVOT


def test_ht_lu_entry_outside_band_is_reported(cuda):
    from piro_b200 import ops
    from piro_b200._lib import PiroError
    nx, ny, nz = 6, 5, 4
    N = nx * ny * nz
    L = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
    ts = ops.ht_table_size(L[2].numel(), N, 1)
    keys, vals = ops.ht_build(N, *L, ts)
    with pytest.raises(PiroError, match="outside the bandwidth") as e:
        ops.HtLu(N, nx, keys, vals, ts, 1.0, -0.05)  # the z neighbours sit nx*ny away
    assert e.value.status == 1
