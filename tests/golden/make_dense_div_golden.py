"""Generate tests/golden/dense_div.npz from PIRO's own code (oracle/_ref):

- DENSE Laplacian (Piro::DENSE::stencils::laplacian_*, stencils.cpp:431-570)
  for the three space schemes, and one DENSE forward-Euler step
  (SpMVDENSE.cl + addVectors.cl, kernelprocess.cpp:42-66) on a seeded field;
- the divergence operator (Piro::CSR::div's div_*_x/y/z matrices,
  operatordivergenceCSR.cpp:21-101) merged as kernelmethods::csrgeam_2 does
  (kernelcsrgeam.cpp:88-207): "intended" with every matrix row-scaled by the
  velocity component (what SpMSCSR.cl means: csrgeam_3.cl's arithmetic), and
  "literal" with no scaling (the reference's SpMSCSR launches set their int
  arguments with sizeof(cl_mem) and never run on a conformant OpenCL).

    make -C oracle ref && python tests/golden/make_dense_div_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402

GRID = (6, 5, 4)
L0 = 5.0          # [Mesh] l along x
DT = np.float32(0.01)


def main() -> None:
    R = O.Ref()
    nx, ny, nz = GRID
    N = nx * ny * nz
    rng = np.random.default_rng(7)
    u = rng.standard_normal(N).astype(np.float32)
    vel = rng.standard_normal(3 * N).astype(np.float32)
    out = {"u": u, "vel": vel, "dt": DT, "lap_norm": O.laplacian_norm(L0, nx), "grad_norm": O.gradient_norm(L0, nx)}
    for s in (1, 2, 3):
        A = R.dense_laplacian(nx, ny, nz, s, out["lap_norm"])
        nzr, nzc = np.nonzero(A)
        out[f"dense_rows_s{s}"] = nzr.astype(np.int32)
        out[f"dense_cols_s{s}"] = nzc.astype(np.int32)
        out[f"dense_vals_s{s}"] = A[nzr, nzc]
        c, d = R.fe_dense(A, DT, u)
        out[f"dense_C_s{s}"], out[f"dense_D_s{s}"] = c, d
        D3 = R.div3(nx, ny, nz, s, out["grad_norm"])
        rp, col, val = R.csrgeam(N, *D3, vel)
        k = int(rp[N])
        out[f"div_rp_s{s}"], out[f"div_col_s{s}"], out[f"div_val_s{s}"] = rp, col[:k], val[:k]
        rp2, col2, val2 = R.csrgeam2_merge(N, *D3)
        out[f"divlit_rp_s{s}"], out[f"divlit_col_s{s}"], out[f"divlit_val_s{s}"] = rp2, col2, val2
        print(f"scheme {s}: dense nnz {len(nzr)}, div nnz {k}")
    np.savez_compressed(os.path.join(HERE, "dense_div.npz"), **out)


if __name__ == "__main__":
    main()
