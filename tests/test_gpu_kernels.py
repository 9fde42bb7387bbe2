"""CUDA path vs the oracle and the reference-made golden fixtures.

Integer structures and the reference-order FP32 kernels must match bit for
bit; the warp-segmented COO SpMV and the matrix-free stencil are checked at
FP32 tolerance (1e-5 relative on the stepped field)."""
import hashlib

import numpy as np
import pytest

from conftest import f32_bits_equal

pytestmark = pytest.mark.gpu
SCHEMES = (1, 2, 3)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def h(t):
    return t.cpu().numpy()


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("tag_l", ["h1", "h37"])
def test_laplacian_and_gradient_vs_golden(cuda, golden_grids, tag_l):
    from piro_b200 import ops
    for (nx, ny, nz), g in golden_grids:
        for s in SCHEMES:
            t = f"s{s}_{tag_l}"
            rp, col, val = ops.csr_laplacian(nx, ny, nz, s, g[f"norm_{tag_l}"])
            assert np.array_equal(h(rp), g[f"csr_rowptr_{t}"]), (nx, ny, nz, s)
            assert np.array_equal(h(col), g[f"csr_col_{t}"])
            assert f32_bits_equal(h(val), g[f"csr_val_{t}"])
            rows, ccol, cval = ops.coo_laplacian(nx, ny, nz, s, g[f"norm_{tag_l}"])
            assert np.array_equal(h(rows), g[f"coo_rows_{t}"])
            assert np.array_equal(h(ccol), g[f"coo_col_{t}"])
            assert f32_bits_equal(h(cval), g[f"coo_val_{t}"])
            for a in range(3):
                grp, gcol, gval = ops.csr_gradient(nx, ny, nz, s, a, g[f"gnorm_{tag_l}"])
                assert np.array_equal(h(grp), g[f"grad{a}_rowptr_{t}"])
                assert np.array_equal(h(gcol), g[f"grad{a}_col_{t}"])
                assert f32_bits_equal(h(gval), g[f"grad{a}_val_{t}"])


def test_large_grids_by_hash(cuda, oracle, golden_hashes):
    from piro_b200 import ops
    for hh in golden_hashes:
        nx, ny, nz = hh["n"]
        rp, col, val = ops.csr_laplacian(nx, ny, nz, hh["scheme"], oracle.laplacian_norm(nx - 2, nx))
        assert sha(h(rp)) == hh["rowptr"] and sha(h(col)) == hh["col"] and sha(h(val)) == hh["val"]
        for a in range(3):
            G = ops.csr_gradient(nx, ny, nz, hh["scheme"], a, oracle.gradient_norm(nx - 2, nx))
            assert sha(h(G[0])) == hh["grad"][a]["rowptr"] and sha(h(G[1])) == hh["grad"][a]["col"]
            assert sha(h(G[2])) == hh["grad"][a]["val"]


@pytest.mark.parametrize("n", [(64, 64, 64), (100, 37, 53), (3, 3, 3), (3, 40, 5)])
def test_assembly_vs_oracle_ragged(cuda, oracle, n):
    from piro_b200 import ops
    nx, ny, nz = n
    for s in SCHEMES:
        rp, col, val = ops.csr_laplacian(nx, ny, nz, s, 0.37)
        orp, ocol, oval = oracle.laplacian(nx, ny, nz, s, 0.37)
        assert np.array_equal(h(rp), orp) and np.array_equal(h(col), ocol) and f32_bits_equal(h(val), oval)
        rows, _, _ = ops.coo_laplacian(nx, ny, nz, s, 0.37)
        assert np.array_equal(h(rows), np.repeat(np.arange(nx * ny * nz, dtype=np.int32), np.diff(orp)))


def test_face_lists_and_setbc(cuda, golden_grids):
    import torch
    from piro_b200 import ops
    for (nx, ny, nz), g in golden_grids:
        idx, fs = ops.face_lists(nx, ny, nz)
        assert np.array_equal(h(idx), g["bc_idx"])
        N = nx * ny * nz
        src = torch.arange(N, dtype=torch.float32, device="cuda")
        dst = torch.zeros(N, dtype=torch.float32, device="cuda")
        ops.set_bc(idx, src, dst)
        want = np.zeros(N, np.float32)
        want[g["bc_idx"]] = g["bc_idx"].astype(np.float32)
        assert np.array_equal(h(dst), want)


def test_step_kernels_vs_golden(cuda, golden_grids):
    import torch
    from piro_b200 import ops
    for (nx, ny, nz), g in golden_grids:
        N = nx * ny * nz
        for s in SCHEMES:
            t = f"s{s}_h1"
            A = tuple(dev(torch, g[f"csr_{k}_{t}"]) for k in ("rowptr", "col", "val"))
            u, c0 = dev(torch, g[f"in_u_{t}"]), dev(torch, g[f"in_c0_{t}"])
            out = c0.clone()
            ops.csr_fe_step(nx, ny, nz, A, 0.01, u, out)
            assert f32_bits_equal(h(out), g[f"spmvcsr_{t}"])
            out = c0.clone()
            ops.csr_i1(nx, ny, nz, A, 0.01, u, out)
            assert f32_bits_equal(h(out), g[f"spmvcsr_i1_{t}"])
            coo = tuple(dev(torch, g[f"coo_{k}_{t}"]) for k in ("rows", "col", "val"))
            out = torch.empty(N, dtype=torch.float32, device="cuda")
            ops.coo_spmv(N, coo, 0.01, u, out)
            np.testing.assert_allclose(h(out), g[f"spmvcoo_{t}"], rtol=1e-5, atol=1e-6)
            rowstart = ops.coo_row_index(N, coo[0])
            assert np.array_equal(h(rowstart), g[f"csr_rowptr_{t}"])  # the row index is the CSR row pointer
            ops.coo_step_indexed(N, rowstart, coo[1], coo[2], 0.01, u, out)
            np.testing.assert_allclose(h(out), g[f"spmvcoo_{t}"], rtol=1e-5, atol=1e-6)
            keys = dev(torch, g[f"ht_keys_{t}"].astype(np.int64))
            hv = dev(torch, g[f"ht_vals_{t}"])
            ops.ht_spmv(nx, ny, nz, keys, hv, 0.01, u, out)
            assert f32_bits_equal(h(out), g[f"spmvht_{t}"])
            order = ops.ht_row_order(N, keys.numel())
            assert np.array_equal(np.sort(h(order)), np.arange(N))  # a permutation of the rows
            out2 = torch.full_like(out, float("nan"))
            ops.ht_spmv_ordered(nx, ny, nz, keys, hv, 0.01, order, u, out2)
            assert f32_bits_equal(h(out2), g[f"spmvht_{t}"])
            out2.fill_(float("nan"))
            ops.ht_spmv_staged(nx, ny, nz, keys, hv, 0.01, order, ops.ht_stage(N), u, out2)
            assert f32_bits_equal(h(out2), g[f"spmvht_{t}"])
            val = A[2].clone()
            ops.csr_rowscale(A[0], val, dev(torch, g[f"in_alpha_{t}"]))
            assert f32_bits_equal(h(val), g[f"spmdsm_{t}"])


def test_coo_bad_rows_are_errors(cuda, golden_grids):
    """Both COO entry points turn a row id outside [0, N) and row ids that do
    not ascend into PIRO_ERR_ARG (SpMVCOO.cl matches no row outside [0, N);
    the warp-segmented sum is only whole rows when the ids ascend), and the
    library stays usable: the next call with good input matches the fixture."""
    import torch
    from piro_b200 import ops
    from piro_b200._lib import PiroError
    (nx, ny, nz), g = golden_grids[0]
    N = nx * ny * nz
    t = "s3_h1"
    rows, col, val = (g[f"coo_{k}_{t}"] for k in ("rows", "col", "val"))
    u = dev(torch, g[f"in_u_{t}"])
    out = torch.empty(N, dtype=torch.float32, device="cuda")
    bad_range = rows.copy()
    bad_range[len(rows) // 2] = N  # one entry's row past the last row
    bad_order = rows.copy()
    k = int(np.argmax(np.diff(rows) > 0))  # first row change: swap the ids around it
    bad_order[k], bad_order[k + 1] = bad_order[k + 1], bad_order[k]
    for bad in (bad_range, bad_order):
        coo = (dev(torch, bad), dev(torch, col), dev(torch, val))
        for fe in (False, True):
            with pytest.raises(PiroError) as e:
                ops.coo_spmv(N, coo, 0.01, u, out, fe=fe)
            assert e.value.status == 1  # PIRO_ERR_ARG
        with pytest.raises(PiroError) as e:
            ops.coo_row_index(N, coo[0])
        assert e.value.status == 1
    neg = rows.copy()
    neg[0] = -1
    with pytest.raises(PiroError):
        ops.coo_spmv(N, (dev(torch, neg), dev(torch, col), dev(torch, val)), 0.01, u, out)
    coo = (dev(torch, rows), dev(torch, col), dev(torch, val))
    ops.coo_spmv(N, coo, 0.01, u, out)
    np.testing.assert_allclose(h(out), g[f"spmvcoo_{t}"], rtol=1e-5, atol=1e-6)


def test_csr_and_coo_steps_on_wide_rows_bitexact(cuda, oracle):
    """Rows longer than 32 entries are summed by their whole warp (coalesced
    entry loads, terms added in storage order through a shuffle chain), the
    rest one row per thread: the result must equal SpMVCSR.cl's / SpMVCOO.cl's
    sequential sums bit for bit whatever the mix of lengths in a warp."""
    import torch
    from piro_b200 import ops
    nx, ny, nz = 18, 16, 14
    N = nx * ny * nz
    rng = np.random.default_rng(21)
    lengths = rng.choice([0, 1, 3, 7, 31, 32, 33, 64, 100, 257, 1000], size=N,
                         p=[.05, .05, .1, .3, .05, .05, .1, .1, .1, .07, .03]).astype(np.int64)
    lengths[5] = 5000  # one very long row
    lengths[[0, N - 2, N - 1]] = 0  # rows without entries at both ends
    rp = np.zeros(N + 1, np.int64)
    rp[1:] = np.cumsum(lengths)
    nnz = int(rp[-1])
    col = rng.integers(0, N, size=nnz).astype(np.int32)  # unsorted, with repeats
    val = rng.standard_normal(nnz).astype(np.float32)
    A = (rp.astype(np.int32), col, val)
    u = rng.standard_normal(N).astype(np.float32)
    c0 = rng.standard_normal(N).astype(np.float32)
    dt = np.float32(0.013)
    want = oracle.spmv_csr_fe(nx, ny, nz, A, dt, u, c0)
    Ad = tuple(dev(torch, a) for a in A)
    out = dev(torch, c0)
    ops.csr_fe_step(nx, ny, nz, Ad, dt, dev(torch, u), out)
    assert f32_bits_equal(h(out), want)
    rows = np.repeat(np.arange(N, dtype=np.int32), lengths)
    want_coo = oracle.spmv_coo(N, (rows, col, val), dt, u)
    ops.coo_step_indexed(N, Ad[0], Ad[1], Ad[2], dt, dev(torch, u), out)
    assert f32_bits_equal(h(out), want_coo)
    # the segmented sum (8 entries per lane, rows across lanes and 256-entry
    # spans): FP32 tolerance, since it adds in another order
    coo = (dev(torch, rows), Ad[1], Ad[2])
    ops.coo_spmv(N, coo, dt, dev(torch, u), out)
    scale = np.abs(val).reshape(-1).max() * np.abs(u).max() * lengths.max() * abs(float(dt))
    np.testing.assert_allclose(h(out), want_coo, rtol=1e-5, atol=1e-6 * scale)
    assert np.all(h(out)[lengths == 0] == 0.0)
    # the fused forward-Euler form, and the same bits on every run (the parts of
    # rows that cross spans are added in span order, not by atomics)
    runs = []
    for _ in range(3):
        o = torch.full_like(out, float("nan"))
        ops.coo_spmv(N, coo, dt, dev(torch, u), o, fe=True)
        runs.append(h(o))
    np.testing.assert_allclose(runs[0], u + want_coo, rtol=1e-5, atol=1e-6 * scale)
    assert np.array_equal(runs[0][lengths == 0], u[lengths == 0])
    assert all(np.array_equal(runs[0], r) for r in runs[1:])


def test_csrgeam3_vs_golden(cuda, golden_grids):
    import torch
    from piro_b200 import ops
    for (nx, ny, nz), g in golden_grids:
        N = nx * ny * nz
        for s in SCHEMES:
            t = f"s{s}_h1"
            G = [tuple(dev(torch, g[f"grad{a}_{k}_{t}"]) for k in ("rowptr", "col", "val")) for a in range(3)]
            D = ops.csrgeam3(N, *G, dev(torch, g[f"in_v_{t}"]))
            assert np.array_equal(h(D[0]), g[f"geam_rowptr_{t}"])
            assert np.array_equal(h(D[1]), g[f"geam_col_{t}"])
            assert f32_bits_equal(h(D[2]), g[f"geam_val_{t}"])


@pytest.mark.parametrize("n", [(40, 40, 40), (129, 65, 33)])
def test_csrgeam3_and_geam2_vs_oracle_large(cuda, oracle, n):
    import torch
    from piro_b200 import ops
    nx, ny, nz = n
    N = nx * ny * nz
    rng = np.random.default_rng(5)
    for s in SCHEMES:
        G = oracle.gradient3(nx, ny, nz, s, np.float32(2.0))
        v = rng.standard_normal(3 * N).astype(np.float32)
        ref = oracle.csrgeam3(N, *G, v)
        Gd = [tuple(dev(torch, a) for a in gg) for gg in G]
        D = ops.csrgeam3(N, *Gd, dev(torch, v))
        assert np.array_equal(h(D[0]), ref[0]) and np.array_equal(h(D[1]), ref[1]) and f32_bits_equal(h(D[2]), ref[2])
        # A + beta*B: I - dt*diag(alpha)*L
        L = oracle.laplacian(nx, ny, nz, s, np.float32(1.0))
        alpha = (rng.random(N, dtype=np.float32) + np.float32(0.1)).astype(np.float32)
        Ls = (L[0], L[1], oracle.csr_rowscale(N, L[0], L[2], alpha))
        I = (np.arange(N + 1, dtype=np.int32), np.arange(N, dtype=np.int32), np.ones(N, np.float32))
        ref2 = oracle.csrgeam2(N, I, np.float32(-0.7), Ls)
        Ld = tuple(dev(torch, a) for a in Ls)
        Id = ops.csr_identity(N)
        D2 = ops.csrgeam2(N, Id, -0.7, Ld)
        assert np.array_equal(h(D2[0]), ref2[0]) and np.array_equal(h(D2[1]), ref2[1])
        assert f32_bits_equal(h(D2[2]), ref2[2])


@pytest.mark.parametrize("n", [(12, 10, 9), (20, 20, 20), (64, 64, 64)])
@pytest.mark.parametrize("policy", [0, 1])
def test_ht_build_slots_vs_oracle(cuda, oracle, n, policy):
    from piro_b200 import ops
    nx, ny, nz = n
    N = nx * ny * nz
    for s in SCHEMES:
        A = ops.csr_laplacian(nx, ny, nz, s, 1.0)
        nnz = A[2].numel()
        if policy == 0:
            if N > 18000:
                continue  # the reference formula is only defined below N ~ 18.6k
            ts = ops.ht_table_size(nnz, N, 0)
            assert ts == oracle.ht_table_size_reference(nnz, N)
        else:
            ts = ops.ht_table_size(nnz, N, 1)
        keys, vals = ops.ht_build(N, *A, ts)
        okeys, ovals = oracle.ht_build(N, h(A[0]), h(A[1]), h(A[2]), ts)
        assert np.array_equal(h(keys), okeys), (n, s, policy)
        assert f32_bits_equal(h(vals), ovals)


def test_ht_build_vs_golden_and_table_full(cuda, golden_grids):
    import torch
    from piro_b200 import ops
    from piro_b200._lib import PiroError
    for (nx, ny, nz), g in golden_grids:
        N = nx * ny * nz
        for s in SCHEMES:
            t = f"s{s}_h1"
            A = tuple(dev(torch, g[f"csr_{k}_{t}"]) for k in ("rowptr", "col", "val"))
            keys, vals = ops.ht_build(N, *A, int(g[f"ht_ts_{t}"]))
            assert np.array_equal(h(keys).astype(np.int32), g[f"ht_keys_{t}"])
            assert f32_bits_equal(h(vals), g[f"ht_vals_{t}"])
    A = ops.csr_laplacian(6, 5, 4, 3, 1.0)
    with pytest.raises(PiroError, match="TABLE_FULL"):
        ops.ht_build(120, *A, 100)  # 692 keys into 100 slots


@pytest.mark.parametrize("n", [(32, 32, 32), (50, 41, 37)])
def test_fe_steps_match_oracle(cuda, oracle, n):
    """Repeated Solve() steps on CSR (bit-exact), HT (bit-exact) and COO
    (1e-5 relative), with setBC restoring face values each step."""
    import torch
    from piro_b200 import ops
    nx, ny, nz = n
    N = nx * ny * nz
    rng = np.random.default_rng(0)
    u0 = rng.random(N, dtype=np.float32)
    alpha = np.full(N, 0.01, np.float32)
    dt = np.float32(0.2 / (6 * 0.01))
    A = oracle.laplacian(nx, ny, nz, 3, np.float32(1.0))
    As = (A[0], A[1], oracle.csr_rowscale(N, A[0], A[2], alpha))
    steps = 20
    ref = oracle.fe_csr(nx, ny, nz, As, dt, u0, steps)
    Ad = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
    ops.csr_rowscale(Ad[0], Ad[2], dev(torch, alpha))
    idx, _ = ops.face_lists(nx, ny, nz)
    u = dev(torch, u0)
    bc = u.clone()
    out = torch.empty_like(u)
    for _ in range(steps):
        out.zero_()
        ops.csr_fe_step(nx, ny, nz, Ad, dt, u, out)
        ops.set_bc(idx, bc, out)
        u, out = out, u
    assert f32_bits_equal(h(u), ref)
    # HT (build policy) and COO forward Euler
    ts = ops.ht_table_size(As[2].size, N, 1)
    keys, vals = ops.ht_build(N, *Ad, ts)
    okeys, ovals = oracle.ht_build(N, As[0], As[1], As[2], ts)
    ref_ht = oracle.fe_ht(nx, ny, nz, okeys, ovals, dt, u0, 3)
    u = dev(torch, u0)
    out = torch.empty_like(u)
    for _ in range(3):
        ops.ht_spmv(nx, ny, nz, keys, vals, dt, u, out, fe=True)
        ops.set_bc(idx, bc, out)
        u, out = out, u
    assert f32_bits_equal(h(u), ref_ht)
    order = ops.ht_row_order(N, ts)
    u = dev(torch, u0)
    for _ in range(3):
        ops.ht_spmv_ordered(nx, ny, nz, keys, vals, dt, order, u, out, fe=True)
        ops.set_bc(idx, bc, out)
        u, out = out, u
    assert f32_bits_equal(h(u), ref_ht)
    stage = ops.ht_stage(N)
    u = dev(torch, u0)
    for _ in range(3):
        ops.ht_spmv_staged(nx, ny, nz, keys, vals, dt, order, stage, u, out, fe=True)
        ops.set_bc(idx, bc, out)
        u, out = out, u
    assert f32_bits_equal(h(u), ref_ht)
    coo = ops.coo_laplacian(nx, ny, nz, 3, 1.0)
    rows_np = h(coo[0])
    coo_s = (coo[0], coo[1], dev(torch, oracle.csr_rowscale(N, A[0], h(coo[2]), alpha)))
    ref_coo = oracle.fe_coo(nx, ny, nz, (rows_np, h(coo[1]), h(coo_s[2])), dt, u0, 3)
    u = dev(torch, u0)
    for _ in range(3):
        ops.coo_spmv(N, coo_s, dt, u, out, fe=True)
        ops.set_bc(idx, bc, out)
        u, out = out, u
    np.testing.assert_allclose(h(u), ref_coo, rtol=1e-5, atol=1e-6)
    # the row-indexed step adds each row's products in entry order, as
    # SpMVCOO.cl does, then dt * sum and u + that (addVectors.cl): bit-exact
    rowstart = ops.coo_row_index(N, coo_s[0])
    u = dev(torch, u0)
    for _ in range(3):
        ops.coo_step_indexed(N, rowstart, coo_s[1], coo_s[2], dt, u, out, fe=True)
        ops.set_bc(idx, bc, out)
        u, out = out, u
    assert f32_bits_equal(h(u), ref_coo)
    bad = coo_s[0].flip(0).contiguous()
    with pytest.raises(Exception, match="not sorted"):
        ops.coo_row_index(N, bad)


# nx in {16, 32, 64, 128, 256} takes the TMA-staged path (partial row blocks,
# one-plane z runs); other nx % 4 == 0 the float4 path (48, 4, 8); the rest
# the z-march
@pytest.mark.parametrize("n", [(48, 40, 36), (33, 9, 17), (3, 3, 3), (70, 12, 5), (64, 8, 5), (4, 4, 4), (8, 3, 3),
                               (16, 130, 6), (32, 70, 11), (128, 19, 33), (256, 10, 3), (64, 64, 64)])
def test_stencil_matches_oracle(cuda, oracle, n):
    import torch
    from piro_b200 import ops
    nx, ny, nz = n
    N = nx * ny * nz
    rng = np.random.default_rng(1)
    u = rng.random(N, dtype=np.float32)
    alpha = np.exp(rng.standard_normal(N)).astype(np.float32)
    ref = oracle.stencil_fe(nx, ny, nz, 0.01, u, alpha, idx2=1.0, idy2=0.25, idz2=4.0)
    out = torch.empty(N, dtype=torch.float32, device="cuda")
    ops.stencil_fe_step(nx, ny, nz, 0.01, dev(torch, u), out, alpha=dev(torch, alpha), idx2=1.0, idy2=0.25, idz2=4.0)
    assert f32_bits_equal(h(out), ref)
    ref = oracle.stencil_fe(nx, ny, nz, 0.01, u)
    ops.stencil_fe_step(nx, ny, nz, 0.01, dev(torch, u), out)
    assert f32_bits_equal(h(out), ref)
    ops.stencil_check()


def test_vector_ops_and_dot(cuda, oracle):
    import torch
    from piro_b200 import ops
    rng = np.random.default_rng(2)
    b = rng.random(10007, dtype=np.float32) + np.float32(0.5)
    c = rng.random(10007, dtype=np.float32) + np.float32(0.5)
    bd, cd = dev(torch, b), dev(torch, c)
    for op in range(4):
        want = np.zeros_like(b)
        oracle.lib().or_vec_binary(op, len(b), b, c, want)
        assert f32_bits_equal(h(ops.vec_op(op, bd, cd)), want)
        oracle.lib().or_vec_constant(op, len(b), np.float32(1.7), c, want)
        assert f32_bits_equal(h(ops.vec_op_scalar(op, 1.7, cd)), want)
    a2, c2 = b.copy(), c.copy()
    oracle.lib().or_urf(len(a2), a2, c2, np.float32(0.7))
    ad, cd2 = dev(torch, b), dev(torch, c)
    ops.vec_urf(ad, cd2, 0.7)
    assert f32_bits_equal(h(ad), a2) and f32_bits_equal(h(cd2), c2)
    for n in (0, 1, 1000, 3 * 10 ** 6 + 17):
        x = rng.standard_normal(n).astype(np.float32)
        y = rng.standard_normal(n).astype(np.float32)
        got = ops.dot_f64(dev(torch, x), dev(torch, y)) if n else 0.0
        want = float(np.dot(x.astype(np.float64), y.astype(np.float64)))
        assert abs(got - want) <= 1e-12 * max(1.0, np.abs(x.astype(np.float64) * y).sum())


@pytest.mark.parametrize("n", [(12, 10, 9), (3, 3, 3), (33, 17, 5)])
def test_fused_fe_step_with_bc(cuda, n):
    """piro_csr_fe_step_bc = zero-filled result + SpMVCSR step + setBC, bit for bit."""
    import torch
    from piro_b200 import ops
    nx, ny, nz = n
    N = nx * ny * nz
    rng = np.random.default_rng(4)
    u = torch.from_numpy(rng.random(N, dtype=np.float32)).cuda()
    memD = torch.from_numpy(rng.random(N, dtype=np.float32)).cuda()
    A = ops.csr_laplacian(nx, ny, nz, 3, 1.0)
    ops.csr_rowscale(A[0], A[2], torch.from_numpy(np.exp(rng.standard_normal(N)).astype(np.float32)).cuda())
    idx, _ = ops.face_lists(nx, ny, nz)
    ref = torch.zeros(N, device="cuda")
    ops.csr_fe_step(nx, ny, nz, A, 0.013, u, ref)
    ops.set_bc(idx, memD, ref)
    got = torch.full((N,), float("nan"), device="cuda")
    ops.csr_fe_step_bc(nx, ny, nz, A, 0.013, u, memD, got)
    assert f32_bits_equal(h(got), h(ref))
    ref = torch.zeros(N, device="cuda")
    ops.csr_fe_step(nx, ny, nz, A, 0.013, u, ref)
    got.fill_(float("nan"))
    ops.csr_fe_step_bc(nx, ny, nz, A, 0.013, u, None, got)  # no [BC]: faces stay 0
    assert f32_bits_equal(h(got), h(ref))


@pytest.mark.parametrize("n,load", [((40, 36, 30), 0.97), ((33, 17, 9), 0.5), ((3, 7, 64), 0.9)])
def test_ht_ordered_and_staged_steps_on_crowded_tables(cuda, oracle, n, load):
    """On tables with long probe runs (97% full), with deleted keys (-2, which
    a lookup walks past) and with odd sizes, the home-slot-ordered and the
    two-pass HT steps equal the row-major probing step bit for bit."""
    import torch
    from piro_b200 import ops
    nx, ny, nz = n
    N = nx * ny * nz
    rng = np.random.default_rng(11)
    A = ops.csr_laplacian(nx, ny, nz, 1, 1.0)
    nnz = int(A[2].numel())
    ts = int(nnz / load) | 1
    keys, vals = ops.ht_build(N, *A, ts)
    vals.copy_(torch.from_numpy(rng.standard_normal(ts).astype(np.float32)).cuda())
    order = ops.ht_row_order(N, ts)
    stage = ops.ht_stage(N)
    u = dev(torch, rng.random(N, dtype=np.float32))
    want = torch.empty_like(u)
    got = torch.empty_like(u)
    for trial in range(2):
        if trial == 1:  # delete a tenth of the keys: every reader sees them as absent
            kh = h(keys)
            live = np.flatnonzero(kh >= 0)
            kh[rng.choice(live, size=len(live) // 10, replace=False)] = -2
            keys.copy_(torch.from_numpy(kh).cuda())
        ops.ht_spmv(nx, ny, nz, keys, vals, 0.37, u, want, fe=True)
        got.fill_(float("nan"))
        ops.ht_spmv_ordered(nx, ny, nz, keys, vals, 0.37, order, u, got, fe=True)
        assert f32_bits_equal(h(got), h(want)), trial
        got.fill_(float("nan"))
        ops.ht_spmv_staged(nx, ny, nz, keys, vals, 0.37, order, stage, u, got, fe=True)
        assert f32_bits_equal(h(got), h(want)), trial
