"""ParaView output (piro_write_paraview) against the files PIRO's own writer
produces for the same fields (tests/golden/paraview_*.npz, made by
tests/golden/make_paraview_golden.py from the reference build): byte for byte."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ASSETS = os.path.join(HERE, "cases")


def _golden(case):
    d = np.load(os.path.join(HERE, "golden", "paraview_" + case.replace(".ini", "") + ".npz"))
    return bytes(d["vth"]).decode(), bytes(d["vti"]).decode(), int(d["timestep"])


def _read(root, case, ts):
    mesh = os.path.join(root, case, "mesh")
    with open(os.path.join(mesh, f"mesh_{ts:05d}.vth")) as f:
        vth = f.read()
    with open(os.path.join(mesh, "level", f"{ts:05d}_level_0.vti")) as f:
        vti = f.read()
    return vth, vti


@pytest.mark.parametrize("case", ["heat_fe_csr.ini", "adv_fe.ini"])
def test_paraview_matches_reference_writer(cuda, tmp_path, case):
    from piro_b200.case import Case
    vth_ref, vti_ref, ts = _golden(case)
    c = Case(ASSETS, case)
    steps = c.solve()
    assert steps - 1 == ts
    c.write_paraview(str(tmp_path), ts)
    vth, vti = _read(str(tmp_path), case, ts)
    assert vth == vth_ref
    assert vti == vti_ref
    c.close()


def test_paraview_every_save_step(cuda, tmp_path):
    from piro_b200.case import Case
    case = "heat_fe_csr.ini"
    vth_ref, vti_ref, ts = _golden(case)
    c = Case(ASSETS, case)
    c.set_output(str(tmp_path))
    steps = c.solve()
    level = os.path.join(str(tmp_path), case, "mesh", "level")
    assert sorted(os.listdir(level)) == [f"{k:05d}_level_0.vti" for k in range(steps)]  # Save = 1
    assert _read(str(tmp_path), case, ts) == (vth_ref, vti_ref)
    c.close()
