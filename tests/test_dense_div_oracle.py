"""The oracle's DENSE format and divergence operator against fixtures made by
PIRO's own code (tests/golden/make_dense_div_golden.py)."""
import os

import numpy as np

from conftest import ROOT, f32_bits_equal

G = os.path.join(ROOT, "tests", "golden", "dense_div.npz")
NX, NY, NZ = 6, 5, 4
N = NX * NY * NZ


def _dense(g, s):
    A = np.zeros((N, N), np.float32)
    A[g[f"dense_rows_s{s}"], g[f"dense_cols_s{s}"]] = g[f"dense_vals_s{s}"]
    return A


def test_dense_laplacian_and_step(oracle):
    g = np.load(G)
    for s in (1, 2, 3):
        A = oracle.dense_laplacian(NX, NY, NZ, s, g["lap_norm"])
        assert f32_bits_equal(A, _dense(g, s)), s
        c, d = oracle.fe_dense(A, g["dt"], g["u"])
        assert f32_bits_equal(c, g[f"dense_C_s{s}"]) and f32_bits_equal(d, g[f"dense_D_s{s}"]), s


def test_dense_uw_dw_diagonal_is_the_last_assignment(oracle):
    """uw/dw assign the replaced neighbour onto the diagonal after -6/norm."""
    A = oracle.dense_laplacian(NX, NY, NZ, 1, np.float32(1.0))
    d = np.diag(A)
    assert d[N - 1] == np.float32(-6.0) and np.all(d[:N - 1] == np.float32(1.0))
    A = oracle.dense_laplacian(NX, NY, NZ, 2, np.float32(1.0))
    d = np.diag(A)
    assert d[0] == np.float32(-6.0) and np.all(d[1:] == np.float32(1.0))


def test_divergence_intended_and_literal(oracle):
    g = np.load(G)
    for s in (1, 2, 3):
        D3 = oracle.div3(NX, NY, NZ, s, g["grad_norm"])
        rp, col, val = oracle.csrgeam3(N, *D3, g["vel"])
        assert np.array_equal(rp, g[f"div_rp_s{s}"]) and np.array_equal(col, g[f"div_col_s{s}"])
        assert f32_bits_equal(val, g[f"div_val_s{s}"])
        rp, col, val = oracle.csrgeam3(N, *D3, np.ones(3 * N, np.float32))
        assert np.array_equal(rp, g[f"divlit_rp_s{s}"]) and np.array_equal(col, g[f"divlit_col_s{s}"])
        assert f32_bits_equal(val, g[f"divlit_val_s{s}"])
