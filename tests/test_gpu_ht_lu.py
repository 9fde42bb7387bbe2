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


def _dense(ops, n, dt):
    """I - dt L as the FP64 dense matrix the factor builds (FP32 table values
    and FP32 dt, products and sums in FP64)."""
    nx, ny, nz = n
    N = nx * ny * nz
    L = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
    rp, col, val = (t.cpu().numpy() for t in L)
    Ad = np.zeros((N, N))
    for r in range(N):
        for k in range(rp[r], rp[r + 1]):
            Ad[r, col[k]] += float(np.float32(-dt)) * float(val[k])
        Ad[r, r] += 1.0
    return L, Ad


# dt 0.05: well conditioned (cond ~ 7, no row exchanges); dt 0.7: PIRO's 10.0
# boundary entries exceed the diagonal (an unpivoted elimination grows the
# elements ~1e4; here 155 and 468 row exchanges, cond up to 1.6e8); dt 0.1:
# A(0, 0) = 1 - 0.1*10 vanishes (to -1.5e-8 with dt in FP32; exactly 0 in an
# FP32 elimination), so the first pivot must be exchanged.
# pivots: compare the pivot rows with LAPACK's dgetrf (scipy) where its choice
# is not a near-tie in that matrix.
@pytest.mark.parametrize("n,dt,pivots", [((8, 7, 6), 0.05, True), ((12, 10, 9), 0.05, True), ((8, 7, 6), 0.7, True),
                                         ((12, 10, 9), 0.7, False), ((8, 7, 6), 0.1, True), ((6, 5, 4), 0.1, True),
                                         ((40, 3, 3), 0.05, True), ((3, 3, 40), 0.05, True)])
def test_ht_lu_pivoted_fp64_solve(cuda, n, dt, pivots):
    import scipy.linalg as sl
    import torch
    from piro_b200 import ops
    nx, ny, nz = n
    N = nx * ny * nz
    L, Ad = _dense(ops, n, dt)
    ts = ops.ht_table_size(L[2].numel(), N, 1)
    keys, vals = ops.ht_build(N, *L, ts)  # the operator's table: the factor scales and shifts it
    lu = ops.HtLu(N, nx * ny, keys, vals, ts, 1.0, -dt)
    if pivots:
        assert np.array_equal(lu.pivots(), sl.lu_factor(Ad)[1])
    cond = np.linalg.cond(Ad)
    rng = np.random.default_rng(3)
    for _ in range(2):  # the factor serves several solves
        b = rng.random(N).astype(np.float32)
        x = lu.solve(torch.from_numpy(b).cuda()).cpu().numpy().astype(np.float64)
        ref = np.linalg.solve(Ad, b.astype(np.float64))
        # FP64 factor and solve: the error is the FP32 rounding of x plus cond * eps64
        assert np.abs(x - ref).max() <= (1.2e-7 + 64 * cond * 1.2e-16) * np.abs(ref).max(), (cond,)


def test_ht_lu_singular_matrix_is_reported(cuda):
    """A column with no nonzero at or below the diagonal: PIRO_ERR_ZERO_PIVOT
    (shift 0, scale 0: the zero matrix)."""
    from piro_b200 import ops
    from piro_b200._lib import PiroError
    nx, ny, nz = 8, 7, 6
    N = nx * ny * nz
    L = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
    ts = ops.ht_table_size(L[2].numel(), N, 1)
    keys, vals = ops.ht_build(N, *L, ts)
    with pytest.raises(PiroError, match="singular matrix: column 0") as e:
        ops.HtLu(N, nx * ny, keys, vals, ts, 0.0, 0.0)
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


@pytest.mark.parametrize("n,dt", [((8, 7, 6), 0.7), ((12, 10, 9), 0.05), ((3, 3, 40), 0.05), ((3, 3, 20), 0.7),
                                  ((40, 3, 3), 0.1), ((9, 9, 9), 0.7)])
def test_ht_lu_panels_equal_column_launches(cuda, n, dt, monkeypatch):
    """The blocked factorization (16-column panels, or 8/4 for wide bands)
    gives the band, the multipliers and the pivots of the column-by-column
    launches bit for bit (PIRO_LU_UNBLOCKED=1 selects those)."""
    from piro_b200 import ops
    nx, ny, nz = n
    N = nx * ny * nz
    bw = nx * ny
    L = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
    ts = ops.ht_table_size(L[2].numel(), N, 1)
    keys, vals = ops.ht_build(N, *L, ts)
    band_bytes = 8 * N * (3 * bw + 1)
    lc_off = (band_bytes + 255) // 256 * 256
    blk = ops.HtLu(N, bw, keys, vals, ts, 1.0, -dt)
    monkeypatch.setenv("PIRO_LU_UNBLOCKED", "1")
    col = ops.HtLu(N, bw, keys, vals, ts, 1.0, -dt)
    assert np.array_equal(blk.pivots(), col.pivots())
    # the band (zeroed before the factorization, every entry defined)
    a, b = blk.band[:band_bytes].cpu().numpy(), col.band[:band_bytes].cpu().numpy()
    assert np.array_equal(a, b), int(np.count_nonzero(a != b))
    # the multipliers of step r: Lc[r][t - 1] for t <= min(bw, N - 1 - r)
    la = blk.band[lc_off:lc_off + 8 * N * bw].cpu().numpy().view(np.float64).reshape(N, bw)
    lb = col.band[lc_off:lc_off + 8 * N * bw].cpu().numpy().view(np.float64).reshape(N, bw)
    span = np.minimum(bw, N - 1 - np.arange(N))
    defined = np.arange(bw)[None, :] < span[:, None]
    assert np.array_equal(la[defined].view(np.uint64), lb[defined].view(np.uint64))


@pytest.mark.parametrize("n,dt", [((8, 7, 6), 0.7), ((12, 10, 9), 0.05), ((3, 3, 40), 0.1)])
def test_ht_lu_ring_and_global_solves_agree(cuda, n, dt, monkeypatch):
    """The solve with y in a shared-memory ring and the one with y in global
    memory (PIRO_LU_NO_RING=1, the form bands wider than the ring take) give
    the same bits; both match an FP64 dense solve."""
    import torch
    from piro_b200 import ops
    nx, ny, nz = n
    N = nx * ny * nz
    L, Ad = _dense(ops, n, dt)
    ts = ops.ht_table_size(L[2].numel(), N, 1)
    keys, vals = ops.ht_build(N, *L, ts)
    lu = ops.HtLu(N, nx * ny, keys, vals, ts, 1.0, -dt)
    b = torch.from_numpy(np.random.default_rng(5).random(N).astype(np.float32)).cuda()
    x_ring = lu.solve(b).cpu().numpy()
    monkeypatch.setenv("PIRO_LU_NO_RING", "1")
    x_glob = lu.solve(b).cpu().numpy()
    assert np.array_equal(x_ring.view(np.uint32), x_glob.view(np.uint32))
    ref = np.linalg.solve(Ad, b.cpu().numpy().astype(np.float64))
    cond = np.linalg.cond(Ad)
    assert np.abs(x_ring - ref).max() <= (1.2e-7 + 64 * cond * 1.2e-16) * np.abs(ref).max()
