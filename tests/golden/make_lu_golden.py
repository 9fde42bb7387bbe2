"""Generate tests/golden/ht_lu.npz: scheme 27's factorization of the
Laplacian hash table by PIRO's own code (oracle/_ref: methods::sethash,
methods::lookup/lookupandset fill-in, lu_decompHT.cl rounds), for two small
grids (central scheme, h = 1) and tables of a given size (the last one too
large for the single-block shared-memory path).

    make -C oracle ref && python tests/golden/make_lu_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402

CASES = [((6, 5, 4), 4099), ((5, 5, 5), 4507), ((7, 6, 5), 16411), ((6, 5, 4), 30011)]


def main() -> None:
    R = O.Ref()
    out = {}
    for (nx, ny, nz), ts in CASES:
        N = nx * ny * nz
        rp, col, val = R.laplacian(nx, ny, nz, 3, np.float32(1.0), "csr")
        keys, vals = R.ht_insert_all(N, rp, col, val, ts)
        tag = f"{nx}x{ny}x{nz}" + ("" if ts < 30000 else f"_ts{ts}")
        out[f"keys0_{tag}"], out[f"vals0_{tag}"] = keys.copy(), vals.copy()
        R.ht_lu(N, keys, vals, ts)
        out[f"keys_{tag}"], out[f"vals_{tag}"] = keys, vals
        out[f"ts_{tag}"] = np.int64(ts)
        print(tag, ts, int((keys >= 0).sum()), int((keys == -2).sum()))
    np.savez_compressed(os.path.join(HERE, "ht_lu.npz"), **out)


if __name__ == "__main__":
    main()
