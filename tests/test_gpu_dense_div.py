"""DENSE format (Data 1) and the divergence operator (sim 2) on the device,
against fixtures from PIRO's own code and the oracle, bit for bit."""
import os

import numpy as np
import pytest

from conftest import ROOT, f32_bits_equal

pytestmark = pytest.mark.gpu
G = os.path.join(ROOT, "tests", "golden", "dense_div.npz")
NX, NY, NZ = 6, 5, 4
N = NX * NY * NZ


@pytest.mark.parametrize("s", [1, 2, 3])
def test_dense_laplacian_and_step_match_reference(cuda, s):
    import torch
    from piro_b200 import ops
    g = np.load(G)
    A = ops.dense_laplacian(NX, NY, NZ, s, float(g["lap_norm"]))
    ref = np.zeros((N, N), np.float32)
    ref[g[f"dense_rows_s{s}"], g[f"dense_cols_s{s}"]] = g[f"dense_vals_s{s}"]
    assert f32_bits_equal(A.cpu().numpy(), ref)
    out = ops.dense_fe_step(A, float(g["dt"]), torch.from_numpy(g["u"]).cuda())
    assert f32_bits_equal(out.cpu().numpy(), g[f"dense_D_s{s}"])


# N % 4 == 0 takes the bulk-copy path (120 rows in the fixture test, 5760 and
# 4352 here: the 256-column shape; 14240 = 445 row blocks of 32, where one
# round of 6 CTAs/SM beats two rounds of 3 on 148 SMs: the 128-column shape);
# 105 and 3267 the 4-byte cp.async path
@pytest.mark.parametrize("n", [(7, 5, 3), (20, 18, 16), (33, 9, 11), (17, 16, 16), (89, 20, 8)])
def test_dense_step_matches_oracle(cuda, oracle, n):
    """Ragged sizes (N not a multiple of the 32-row or 256-column tiles) and a
    larger matrix (N = 5760, 133 MB)."""
    import torch
    from piro_b200 import ops
    nx, ny, nz = n
    norm = oracle.laplacian_norm(9, nx)
    A = ops.dense_laplacian(nx, ny, nz, 3, float(norm))
    Ah = oracle.dense_laplacian(nx, ny, nz, 3, norm)
    assert f32_bits_equal(A.cpu().numpy(), Ah)
    u = np.random.default_rng(5).standard_normal(nx * ny * nz).astype(np.float32)
    out = ops.dense_fe_step(A, 0.013, torch.from_numpy(u).cuda())
    ops.dense_check()
    assert f32_bits_equal(out.cpu().numpy(), oracle.fe_dense(Ah, 0.013, u)[1])


@pytest.mark.parametrize("s", [1, 2, 3])
def test_divergence_merge_matches_reference(cuda, s):
    import torch
    from piro_b200 import ops
    g = np.load(G)
    D3 = [ops.csr_gradient(NX, NY, NZ, s, a, float(g["grad_norm"])) for a in range(3)]
    for vel, key in ((g["vel"], "div"), (np.ones(3 * N, np.float32), "divlit")):
        rp, col, val = ops.csrgeam3(N, *D3, torch.from_numpy(vel).cuda())
        assert np.array_equal(rp.cpu().numpy(), g[f"{key}_rp_s{s}"])
        assert np.array_equal(col.cpu().numpy(), g[f"{key}_col_s{s}"])
        assert f32_bits_equal(val.cpu().numpy(), g[f"{key}_val_s{s}"])


def test_continuity_literal_mode(cuda, oracle):
    """alpha_mode 1: the velocity scaling dropped, as the reference's SpMSCSR
    launches never run."""
    from case_oracle import run_case
    from piro_b200.case import Case
    assets = os.path.join(ROOT, "tests", "cases")
    ref = run_case(assets, "cont_fe.ini", alpha_mode=1)
    c = Case(assets, "cont_fe.ini", alpha_mode=1)
    assert c.solve() == ref["steps"]
    assert f32_bits_equal(c.get("rho"), ref["fields"][1])
    c.close()


def test_continuity_operator_spelling(cuda):
    """ddt_r("rho") = div("rho", "u") as solve.cpp:35 writes it equals piro_solve."""
    from piro_b200.case import Case, process, scalarMatrix
    assets = os.path.join(ROOT, "tests", "cases")
    a = Case(assets, "cont_fe.ini")
    a.solve()
    b = Case(assets, "cont_fe.ini")
    solver = process(b)
    time, dt, total = np.float32(0), np.float32(b.info.timestep), np.float32(b.info.totaltime)
    while time < total:
        scalarMatrix(solver.ddt_r("rho").assign(solver.div("rho", "u"))).Solve(float(time))
        time = np.float32(time + dt)
    assert f32_bits_equal(a.get("rho"), b.get("rho"))
