"""The context layer of the C ABI (PIRO's operator API over a case .ini),
run end to end and compared with an oracle-composed run of the same case."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, f32_bits_equal

pytestmark = pytest.mark.gpu
ASSETS = os.path.join(ROOT, "tests", "cases")

# case, exact (bit-for-bit) or relative tolerance
CASES = [
    ("heat_fe_csr.ini", None),     # FE, central, CSR, alpha applied by SpMDSM's row scale
    ("heat_fe_uw.ini", None),      # FE, upwind Laplacian (duplicate columns), Coulomb IC
    ("heat_fe_ht.ini", None),      # FE, hash table (reference table size), downwind
    ("heat_fe_coo.ini", None),     # FE, COO through the row index (SpMVCOO.cl's per-row entry order)
    ("adv_fe.ini", None),          # advection: vector & gradient (csrgeam), upwind
    ("heat_be_jli.ini", 1e-6),     # BE, the reference's JLI iteration (FP64 residual sums)
    ("heat_be_pcg.ini", 1e-6),     # BE, FP32 PCG in FP64 refinement vs an FP64 solve
    ("heat_be_lu.ini", 1e-5),      # BE, scheme 27: FP32 banded LU in the hash table vs an FP64 solve
    ("heat_fe_dense.ini", None),   # FE, DENSE (N x N), downwind: SpMVDENSE's sequential sums
    ("cont_fe.ini", None),         # continuity: div(rho, u), central
]


@pytest.mark.parametrize("name,tol", CASES)
def test_case_solve_matches_oracle(cuda, oracle, name, tol):
    from case_oracle import run_case
    from piro_b200.case import Case
    ref = run_case(ASSETS, name)
    c = Case(ASSETS, name)
    steps = c.solve()
    assert steps == ref["steps"]
    got = c.get(ref["names"][1])
    want = ref["fields"][1]
    if tol is None:
        assert f32_bits_equal(got, want), np.abs(got - want).max()
    else:
        np.testing.assert_allclose(got, want, rtol=tol, atol=tol * np.abs(want).max())
    c.close()


def test_scheme27_as_the_reference_runs(cuda, oracle):
    """lu_mode 1: PIRO's factorization on the first step, a zero result field
    with the boundary values put back (the 5^3 case of Test/LUDecomp.ini)."""
    from case_oracle import run_case
    from piro_b200.case import Case
    ref = run_case(ASSETS, "heat_lu_ref.ini", lu_mode=1)
    c = Case(ASSETS, "heat_lu_ref.ini", lu_mode=1)
    assert c.solve() == ref["steps"] == 3
    assert f32_bits_equal(c.get("T"), ref["fields"][1])
    assert c.get("T").max() == 1.0
    c.close()


def test_operator_spelling_equals_solve_loop(cuda):
    """process / scalarMatrix calls, as solve.cpp writes them, give the same
    field as piro_solve."""
    from piro_b200.case import Case, process, scalarMatrix
    a = Case(ASSETS, "adv_fe.ini")
    a.solve()
    b = Case(ASSETS, "adv_fe.ini")
    solver = process(b)
    time, dt, total = np.float32(0), np.float32(b.info.timestep), np.float32(b.info.totaltime)
    while time < total:
        UEqn = scalarMatrix(solver.ddt_r("U").assign(solver.vector("v") & solver.gradient("U")))
        UEqn.Solve(float(time))
        time = np.float32(time + dt)
    assert f32_bits_equal(a.get("U"), b.get("U"))


def test_exported_operator_is_the_assembled_laplacian(cuda, oracle):
    from piro_b200.case import Case, process
    c = Case(ASSETS, "heat_fe_uw.ini")
    op = process(c).laplacian("T", "Alpha")
    rp, col, val = c.export_csr(op)
    nx, ny, nz = c.info.nx, c.info.ny, c.info.nz
    orp, ocol, oval = oracle.laplacian(nx, ny, nz, 1, oracle.laplacian_norm(9, nx))
    oval = oracle.csr_rowscale(nx * ny * nz, orp, oval, np.full(nx * ny * nz, 0.1, np.float32))
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol) and f32_bits_equal(val, oval)


def test_config_errors_are_status_codes(cuda, tmp_path):
    from piro_b200._lib import PiroError
    from piro_b200.case import Case
    with pytest.raises(PiroError, match="CONFIG"):
        Case(str(tmp_path), "missing.ini")
    bad = tmp_path / "bad.ini"
    bad.write_text(open(os.path.join(ASSETS, "heat_fe_csr.ini")).read().replace("Time = 11", "Time = eleven"))
    (tmp_path / "IC").mkdir()
    (tmp_path / "IC" / "distribution.ini").write_text(open(os.path.join(ASSETS, "IC", "distribution.ini")).read())
    with pytest.raises(PiroError, match="Time"):
        Case(str(tmp_path), "bad.ini")


def test_cpp_host_driver(cuda, tmp_path):
    """A C++ driver written against include/piro.hpp (the solve.cpp spelling)
    links the library and reproduces the Python context's fields."""
    from piro_b200 import _lib
    from piro_b200.case import Case
    exe = tmp_path / "run_case"
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "run_case.cpp"), "-L", os.path.dirname(_lib.LIB_PATH),
                           "-lpiro_b200", f"-Wl,-rpath,{os.path.dirname(_lib.LIB_PATH)}", "-o", str(exe)])
    for name, var in [("heat_fe_csr.ini", "T"), ("adv_fe.ini", "U")]:
        out = tmp_path / (name + ".raw")
        subprocess.check_call([str(exe), ASSETS, name, str(out)])
        got = np.fromfile(out, np.float32)
        c = Case(ASSETS, name)
        c.solve()
        assert f32_bits_equal(got, c.get(var))
