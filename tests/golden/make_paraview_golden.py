"""Generate tests/golden/paraview_*.npz: the ParaView files PIRO's own writer
(Piro::paraview::writevth, built into oracle/_ref by `make -C oracle ref`)
produces for two test cases after their full time loop.  The fields come from
the oracle-composed case run (tests/case_oracle.py), whose steps match the
reference kernels bit for bit on these paths.

    make -C oracle ref && python tests/golden/make_paraview_golden.py
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402
from tests import case_oracle as CO  # noqa: E402

CASES = ["heat_fe_csr.ini", "adv_fe.ini"]


def main() -> None:
    R = O.Ref()
    assets = os.path.join(ROOT, "tests", "cases")
    for case in CASES:
        cfg = CO.read_ini(os.path.join(assets, case))
        run = CO.run_case(assets, case)
        nx, ny, nz = run["n"]
        sim = cfg["Simulation"]
        nconst = len(sim["Constants"].split(" "))
        nscal = len(sim["Scalars"].split(" "))
        types = [0] * nconst + [1] * nscal + [2] * len(sim.get("Vectors", "").split())
        fields = [(nm, t, v) for nm, t, v in zip(run["names"], types, run["fields"])]
        o = [int(float(v)) for v in cfg["Mesh"]["o"].split()]
        s = [int(float(v)) for v in cfg["Mesh"]["s"].split()]
        ts = run["steps"] - 1
        with tempfile.TemporaryDirectory() as d:
            vth, vti = R.paraview(nx, ny, nz, o, s, d, cfg["File"]["casename"], ts, fields)
        np.savez_compressed(os.path.join(HERE, "paraview_" + case.replace(".ini", "") + ".npz"),
                            vth=np.frombuffer(vth.encode(), np.uint8), vti=np.frombuffer(vti.encode(), np.uint8),
                            timestep=np.int64(ts))
        print(case, ts, len(vth), len(vti))


if __name__ == "__main__":
    main()
