"""Generate the golden fixtures in tests/golden/ from PIRO's own code.

Run where the PIRO source tree is present, named by PIRO_REF_DIR:

    PIRO_REF_DIR=<PIRO tree> make -C oracle ref && python tests/golden/make_golden.py

Every array stored here is produced by the reference itself -- its host
stencil/hash/boundary routines and its .cl kernels compiled for the CPU
(oracle/_ref/libpiro_ref.so, built by oracle/Makefile).  The oracle
restatement is NOT used to make fixtures; tests check the oracle and the CUDA
path against these files.  Inputs are seeded (numpy default_rng).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402

GRIDS = [(6, 5, 4), (5, 5, 5), (7, 7, 7), (10, 10, 10)]
HASH_GRIDS = [(32, 32, 32), (34, 34, 34), (20, 12, 17)]


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    R = O.Ref()
    rng = np.random.default_rng(20240601)
    manifest = {"grids": [], "hashes": []}
    for (nx, ny, nz) in GRIDS:
        N = nx * ny * nz
        data = {}
        for l0 in (nx - 2, 3.7):
            norm = O.laplacian_norm(l0, nx)
            gnorm = O.gradient_norm(l0, nx)
            tag_l = "h1" if l0 == nx - 2 else "h37"
            data[f"norm_{tag_l}"] = np.float32(norm)
            data[f"gnorm_{tag_l}"] = np.float32(gnorm)
            for s in (1, 2, 3):
                t = f"s{s}_{tag_l}"
                rp, col, val = R.laplacian(nx, ny, nz, s, norm, "csr")
                data[f"csr_rowptr_{t}"], data[f"csr_col_{t}"], data[f"csr_val_{t}"] = rp, col, val
                rows, ccol, cval = R.laplacian(nx, ny, nz, s, norm, "coo")
                data[f"coo_rows_{t}"], data[f"coo_col_{t}"], data[f"coo_val_{t}"] = rows, ccol, cval
                G = R.gradient3(nx, ny, nz, s, gnorm)
                for a, (grp, gcol, gval) in enumerate(G):
                    data[f"grad{a}_rowptr_{t}"], data[f"grad{a}_col_{t}"], data[f"grad{a}_val_{t}"] = grp, gcol, gval
                if tag_l == "h1":
                    TS = O.ht_table_size_reference(len(val), N)
                    data[f"ht_ts_{t}"] = np.int64(TS)
                    keys, vals = R.ht_insert_all(N, rp, col, val, TS)
                    data[f"ht_keys_{t}"], data[f"ht_vals_{t}"] = keys, vals
                    # seeded inputs and one application of each step kernel
                    u = rng.random(N, dtype=np.float32)
                    c0 = rng.random(N, dtype=np.float32)
                    v = rng.standard_normal(3 * N).astype(np.float32)
                    alpha = (rng.random(N, dtype=np.float32) + np.float32(0.5)).astype(np.float32)
                    dt = np.float32(0.01)
                    data[f"in_u_{t}"], data[f"in_c0_{t}"], data[f"in_v_{t}"], data[f"in_alpha_{t}"] = u, c0, v, alpha
                    data[f"spmvcsr_{t}"] = R.spmvcsr(nx, ny, nz, (rp, col, val), dt, u, c0)
                    data[f"spmvcsr_i1_{t}"] = R.spmvcsr_i1(nx, ny, nz, (rp, col, val), dt, u, c0)
                    data[f"spmvcoo_{t}"] = R.spmvcoo(nx, ny, nz, (rows, ccol, cval), dt, u)
                    data[f"spmvht_{t}"] = R.spmvht(N, keys, vals, dt, u)
                    data[f"spmdsm_{t}"] = R.spmdsm(N, (rp, col, val), alpha)
                    D = R.csrgeam(N, G[0], G[1], G[2], v)
                    k = int(D[0][-1])
                    data[f"geam_rowptr_{t}"], data[f"geam_col_{t}"], data[f"geam_val_{t}"] = D[0], D[1][:k], D[2][:k]
        # boundary lists and the field after setbc(), from bc::initbc
        with tempfile.TemporaryDirectory() as td:
            os.makedirs(os.path.join(td, "assets"))
            with open(os.path.join(td, "assets", "setup.ini"), "w") as f:
                f.write("[BC]\ntype = 0 0 0 0 0 0\nproperty = T T T T T T\nvalues = 0.5 1.5 2.5 3.5 4.5 5.5\n")
            idx, flen, field = R.initbc(nx, ny, nz, td)
        data["bc_idx"], data["bc_face_len"], data["bc_field"] = idx, flen, field
        # laplacianscalar.cl applied to a seeded field
        ub = rng.random(N, dtype=np.float32)
        data["lapscalar_in"] = ub
        data["lapscalar_out"] = R.laplacianscalar(nx, ny, nz, ub, np.float32(0.05))
        # JLI iterations (scheme 12/40) composed from the reference kernels
        rp, col, val = R.laplacian(nx, ny, nz, 2, np.float32(1.0), "csr")
        b = rng.random(N, dtype=np.float32)
        x = b.copy()
        old = np.float32(0.0)
        its = 0
        for it in range(1000):
            r = R.spmvcsr_i1(nx, ny, nz, (rp, col, val), np.float32(0.001), x, np.zeros(N, np.float32))
            r = R.sub(b, r)
            x, r = R.urf(x, r, 1.0)
            s = np.float32(0.0)
            for t_ in r:
                s = np.float32(s + t_ * t_)
            res = np.float32(np.sqrt(s)) / np.float32(np.sqrt(np.float32(N)))
            its = it + 1
            if (res - old) * (res - old) < np.float32(1e-5):
                break
            old = res
        data["jli_b"], data["jli_x"], data["jli_iters"] = b, x, np.int64(its)
        name = f"grid_{nx}x{ny}x{nz}.npz"
        np.savez_compressed(os.path.join(HERE, name), **data)
        manifest["grids"].append({"file": name, "n": [nx, ny, nz]})
    # Initial conditions from Piro::initialcondition (src/ic.cpp), with the
    # test cases' IC/distribution.ini.
    ic = {}
    with tempfile.TemporaryDirectory() as td:
        os.makedirs(os.path.join(td, "assets", "IC"))
        src = os.path.join(os.path.dirname(HERE), "cases", "IC", "distribution.ini")
        with open(src) as f, open(os.path.join(td, "assets", "IC", "distribution.ini"), "w") as g:
            g.write(f.read())
        for (nx, ny, nz), l in [((16, 14, 12), (14, 12, 10)), ((11, 10, 9), (9, 8, 7)), ((7, 6, 5), (5, 4, 3.5))]:
            for kind in ("Gaussian", "Coulomb", "UniformVector"):
                ic[f"ic_{kind}_{nx}x{ny}x{nz}"] = R.initialcondition(nx, ny, nz, l, td, kind)
                ic[f"l_{nx}x{ny}x{nz}"] = np.asarray(l, np.float32)
    np.savez_compressed(os.path.join(HERE, "initial_conditions.npz"), **ic)
    # Large grids: only hashes and counts (arrays would bloat the repository).
    for (nx, ny, nz) in HASH_GRIDS:
        for s in (1, 2, 3):
            norm = O.laplacian_norm(nx - 2, nx)
            rp, col, val = R.laplacian(nx, ny, nz, s, norm, "csr")
            G = R.gradient3(nx, ny, nz, s, O.gradient_norm(nx - 2, nx))
            manifest["hashes"].append({
                "n": [nx, ny, nz], "scheme": s, "nnz": int(len(val)), "n_ten": int((val == 10).sum()),
                "rowptr": sha(rp), "col": sha(col), "val": sha(val),
                "grad": [{"rowptr": sha(g[0]), "col": sha(g[1]), "val": sha(g[2]), "nnz": int(len(g[2]))} for g in G],
            })
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main()
