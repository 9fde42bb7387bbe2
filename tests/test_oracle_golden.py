"""The CPU oracle against fixtures produced by PIRO's own code (tests/golden/,
made by tests/golden/make_golden.py from oracle/_ref).  These pin the oracle
before it is used to check the CUDA path."""
import hashlib

import numpy as np
import pytest

from conftest import f32_bits_equal

SCHEMES = (1, 2, 3)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("tag_l", ["h1", "h37"])
def test_laplacian_csr_coo_bit_exact(oracle, golden_grids, tag_l):
    for (nx, ny, nz), g in golden_grids:
        norm = g[f"norm_{tag_l}"]
        for s in SCHEMES:
            t = f"s{s}_{tag_l}"
            rp, col, val = oracle.laplacian(nx, ny, nz, s, norm, "csr")
            assert np.array_equal(rp, g[f"csr_rowptr_{t}"]), (nx, ny, nz, s)
            assert np.array_equal(col, g[f"csr_col_{t}"])
            assert f32_bits_equal(val, g[f"csr_val_{t}"])
            rows, ccol, cval = oracle.laplacian(nx, ny, nz, s, norm, "coo")
            assert np.array_equal(rows, g[f"coo_rows_{t}"])
            assert np.array_equal(ccol, g[f"coo_col_{t}"])
            assert f32_bits_equal(cval, g[f"coo_val_{t}"])


@pytest.mark.parametrize("tag_l", ["h1", "h37"])
def test_gradient_bit_exact(oracle, golden_grids, tag_l):
    for (nx, ny, nz), g in golden_grids:
        for s in SCHEMES:
            t = f"s{s}_{tag_l}"
            G = oracle.gradient3(nx, ny, nz, s, g[f"gnorm_{tag_l}"])
            for a in range(3):
                assert np.array_equal(G[a][0], g[f"grad{a}_rowptr_{t}"])
                assert np.array_equal(G[a][1], g[f"grad{a}_col_{t}"])
                assert f32_bits_equal(G[a][2], g[f"grad{a}_val_{t}"])


def test_ht_slots_bit_exact(oracle, golden_grids):
    for (nx, ny, nz), g in golden_grids:
        N = nx * ny * nz
        for s in SCHEMES:
            t = f"s{s}_h1"
            rp, col, val = g[f"csr_rowptr_{t}"], g[f"csr_col_{t}"], g[f"csr_val_{t}"]
            ts = oracle.ht_table_size_reference(len(val), N)
            assert ts == int(g[f"ht_ts_{t}"])
            keys, vals = oracle.ht_build(N, rp, col, val, ts)
            assert np.array_equal(keys.astype(np.int32), g[f"ht_keys_{t}"])
            assert f32_bits_equal(vals, g[f"ht_vals_{t}"])


def test_step_kernels_bit_exact(oracle, golden_grids):
    for (nx, ny, nz), g in golden_grids:
        N = nx * ny * nz
        for s in SCHEMES:
            t = f"s{s}_h1"
            A = (g[f"csr_rowptr_{t}"], g[f"csr_col_{t}"], g[f"csr_val_{t}"])
            u, c0, v, alpha = g[f"in_u_{t}"], g[f"in_c0_{t}"], g[f"in_v_{t}"], g[f"in_alpha_{t}"]
            dt = np.float32(0.01)
            assert f32_bits_equal(oracle.spmv_csr_fe(nx, ny, nz, A, dt, u, c0), g[f"spmvcsr_{t}"])
            assert f32_bits_equal(oracle.spmv_csr_i1(nx, ny, nz, A, dt, u, c0), g[f"spmvcsr_i1_{t}"])
            coo = (g[f"coo_rows_{t}"], g[f"coo_col_{t}"], g[f"coo_val_{t}"])
            assert f32_bits_equal(oracle.spmv_coo(N, coo, dt, u), g[f"spmvcoo_{t}"])
            keys = g[f"ht_keys_{t}"].astype(np.int64)
            assert f32_bits_equal(oracle.spmv_ht(N, keys, g[f"ht_vals_{t}"], dt, u), g[f"spmvht_{t}"])
            assert f32_bits_equal(oracle.csr_rowscale(N, A[0], A[2], alpha), g[f"spmdsm_{t}"])
            G = [(g[f"grad{a}_rowptr_{t}"], g[f"grad{a}_col_{t}"], g[f"grad{a}_val_{t}"]) for a in range(3)]
            D = oracle.csrgeam3(N, *G, v)
            assert np.array_equal(D[0], g[f"geam_rowptr_{t}"])
            assert np.array_equal(D[1], g[f"geam_col_{t}"])
            assert f32_bits_equal(D[2], g[f"geam_val_{t}"])


def test_boundary_lists_and_stencil(oracle, golden_grids):
    for (nx, ny, nz), g in golden_grids:
        idx, fs = oracle.face_lists(nx, ny, nz)
        assert np.array_equal(idx.astype(np.int32), g["bc_idx"])
        assert np.array_equal(np.diff(fs), g["bc_face_len"])
        # setbc wrote face f's value onto face f's cells (values 0.5 .. 5.5)
        field = g["bc_field"]
        for f in range(6):
            assert np.all(field[idx[fs[f]:fs[f + 1]]] == np.float32(0.5 + f))
        # matrix-free step: oracle u + dt*lap vs laplacianscalar.cl's dt*lap
        ub, ref = g["lapscalar_in"], g["lapscalar_out"]
        st = oracle.stencil_fe(nx, ny, nz, np.float32(0.05), ub)
        inter = np.zeros((nz, ny, nx), bool)
        inter[1:-1, 1:-1, 1:-1] = True
        inter = inter.ravel()
        np.testing.assert_allclose((st - ub)[inter], ref[inter], rtol=0, atol=2e-6)


def test_jli_matches_reference_kernels(oracle, golden_grids):
    for (nx, ny, nz), g in golden_grids:
        A = oracle.laplacian(nx, ny, nz, 2, np.float32(1.0))
        x, it = oracle.be_jli(nx, ny, nz, A, np.float32(0.001), g["jli_b"])
        assert it == int(g["jli_iters"])
        assert f32_bits_equal(x, g["jli_x"])


def test_large_grid_hashes(oracle, golden_hashes):
    """32^3 (the forward-Euler config), 34^3 and a ragged grid: nnz, the
    number of 10.0 boundary entries and SHA-256 of every array."""
    for h in golden_hashes:
        nx, ny, nz = h["n"]
        norm = oracle.laplacian_norm(nx - 2, nx)
        rp, col, val = oracle.laplacian(nx, ny, nz, h["scheme"], norm)
        assert len(val) == h["nnz"] and int((val == 10).sum()) == h["n_ten"]
        assert sha(rp) == h["rowptr"] and sha(col) == h["col"] and sha(val) == h["val"]
        G = oracle.gradient3(nx, ny, nz, h["scheme"], oracle.gradient_norm(nx - 2, nx))
        for a in range(3):
            assert sha(G[a][0]) == h["grad"][a]["rowptr"] and sha(G[a][1]) == h["grad"][a]["col"]
            assert sha(G[a][2]) == h["grad"][a]["val"]
    c1 = [h for h in golden_hashes if h["n"] == [32, 32, 32] and h["scheme"] == 3][0]
    assert c1["nnz"] == 223232 and c1["n_ten"] == 5768


def test_step_count_float_loop(oracle):
    # while (time < TotalTime) with float time (src/solve.cpp:17-18,45)
    assert oracle.step_count(0.001, 0.001) == 1
    assert oracle.step_count(0.2, 0.001) == 200 or oracle.step_count(0.2, 0.001) == 201
    t, n = np.float32(0), 0
    while t < np.float32(0.2):
        t = np.float32(t + np.float32(0.001))
        n += 1
    assert oracle.step_count(0.2, 0.001) == n


def test_ht_table_size_reference_sign(oracle):
    # the reference formula turns negative above N ~ 18.6k (27^3 = 19683)
    assert oracle.ht_table_size_reference(7 * 125 - 150, 125) == 4795
    assert oracle.ht_table_size_reference(7 * 19683, 19683) <= 0


def test_initial_conditions_bit_exact(oracle):
    """Gaussian / Coulomb / UniformVector against Piro::initialcondition."""
    import os
    from case_oracle import floats, read_ini
    from conftest import GOLDEN, ROOT
    g = dict(np.load(os.path.join(GOLDEN, "initial_conditions.npz")))
    dist = read_ini(os.path.join(ROOT, "tests", "cases", "IC", "distribution.ini"))
    for key in g:
        if not key.startswith("ic_"):
            continue
        _, kind, dims = key.split("_")
        nx, ny, nz = map(int, dims.split("x"))
        l = g[f"l_{dims}"]
        if kind == "Gaussian":
            d = dist["Gaussian"]
            got = oracle.ic_gaussian(nx, ny, nz, l, np.float32(d["Scalefactor"]), floats(d["Sigma"]), floats(d["Median"]))
        elif kind == "Coulomb":
            d = dist["Coulomb"]
            got = oracle.ic_coulomb(nx, ny, nz, l, floats(d["center"]), np.float32(d["Z"]), np.float32(d["e"]),
                                    np.float32(d["epsilon_0"]))
        else:
            d = dist["Vector"]
            got = oracle.ic_uniform_vector(nx * ny * nz, floats(d["Direction"]), floats(d["Value"])[0])
        assert f32_bits_equal(got, g[key]), key


def test_case_oracle_runs_every_test_case(oracle):
    """The oracle-composed case runner itself (used by the GPU case tests)."""
    import os
    from case_oracle import run_case
    from conftest import ROOT
    assets = os.path.join(ROOT, "tests", "cases")
    r = run_case(assets, "heat_fe_csr.ini")
    assert r["steps"] == 10 and r["n"] == (16, 14, 12)
    # the face values of field 1 are restored by setBC every step; edges stay 0
    idx, fs = oracle.face_lists(16, 14, 12)
    T = r["fields"][1]
    assert np.all(T[idx[fs[5]:fs[6]]] == np.float32(1.0))
    assert T[0] == 0.0


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["ref_available"]).ref_available(),
                    reason="the reference build (oracle/_ref) is absent")
def test_reference_spmv_over_threads_equals_sequential(oracle):
    """The CPU baseline runs PIRO's SpMVCSR/SpMVCOO/SpMVHT NDRanges over the
    OpenMP threads; every work-item writes only its own row, so the result
    must equal the sequential NDRange bit for bit."""
    R = oracle.Ref()
    nx, ny, nz = 9, 8, 7
    N = nx * ny * nz
    A = oracle.laplacian(nx, ny, nz, 3, np.float32(1.0))
    u = np.random.default_rng(2).random(N).astype(np.float32)
    seq = R.spmvcsr(nx, ny, nz, A, 0.01, u, np.zeros(N, np.float32))
    assert np.array_equal(seq.view(np.uint32), R.spmv_par("csr", nx, ny, nz, A, 0.01, u).view(np.uint32))
    rows = np.repeat(np.arange(N, dtype=np.int32), np.diff(A[0]))
    seq = R.spmvcoo(nx, ny, nz, (rows, A[1], A[2]), 0.01, u)
    par = R.spmv_par("coo", nx, ny, nz, (rows, A[1], A[2]), 0.01, u)
    assert np.array_equal(seq.view(np.uint32), par.view(np.uint32))
    ts = oracle.ht_table_size_build(len(A[2]))
    keys, vals = oracle.ht_build(N, *A, ts)
    seq = R.spmvht(N, keys.astype(np.int32), vals, 0.01, u)
    par = R.spmv_par("ht", nx, ny, nz, (keys.astype(np.int32), vals), 0.01, u)
    assert np.array_equal(seq.view(np.uint32), par.view(np.uint32))


@pytest.mark.parametrize("n,dt", [((12, 10, 9), 3.0), ((9, 14, 11), 40.0)])
def test_fp64_cg_matches_direct_solve(oracle, n, dt):
    """The oracle's FP64 Jacobi-PCG, the reference every backward-Euler result
    is checked against, equals a direct sparse solve of the same system
    (A = I - dt diag(alpha) L assembled by the oracle's own csrgeam2 and row
    scale, interior unknowns, boundary held at b) to 1e-10."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    nx, ny, nz = n
    N = nx * ny * nz
    rng = np.random.default_rng(31)
    alpha = np.exp(rng.standard_normal(N)).astype(np.float32) * np.float32(0.01)
    L = oracle.laplacian(nx, ny, nz, 3, np.float32(1.0))
    Ls = (L[0], L[1], oracle.csr_rowscale(N, L[0], L[2], alpha))
    I = (np.arange(N + 1, dtype=np.int32), np.arange(N, dtype=np.int32), np.ones(N, np.float32))
    A = oracle.csrgeam2(N, I, np.float32(-dt), Ls)
    b = rng.random(N).astype(np.float32)
    u, its, rel = oracle.be_cg_f64(nx, ny, nz, A, alpha, b, rtol=1e-13)
    M = sp.csr_matrix((A[2].astype(np.float64), A[1], A[0]), shape=(N, N))
    x, y, z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    inter = ((x > 0) & (x < nx - 1) & (y > 0) & (y < ny - 1) & (z > 0) & (z < nz - 1)).transpose(2, 1, 0).reshape(-1)
    bb = b.astype(np.float64)
    want = bb.copy()
    want[inter] = spla.spsolve(M[inter][:, inter].tocsc(), bb[inter] - M[inter][:, ~inter] @ bb[~inter])
    assert rel <= 1e-13
    assert np.abs(u - want).max() <= 1e-10 * np.abs(want).max()
