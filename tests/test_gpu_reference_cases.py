"""PIRO's own example cases (Test/HeatEq.ini, Test/AdvEq.ini,
Test/LUDecomp.ini, which maketest.sh:101-130 runs) end to end through the
context layer of the C ABI, against an oracle-composed run of the same case.

The case and asset files are rebuilt from tests/golden/reference_cases.json
(made from the PIRO tree by make_reference_cases.py), as maketest.sh lays
them out: the case file beside setup.ini in a copy of dependencies/assets.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, f32_bits_equal

pytestmark = pytest.mark.gpu


def write_ini(path, sections):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        for sec, kv in sections.items():
            f.write(f"[{sec}]\n")
            for k, v in kv.items():
                f.write(f"{k} = {v}".rstrip() + "\n")
            f.write("\n")


@pytest.fixture(scope="module")
def assets(tmp_path_factory):
    with open(os.path.join(GOLDEN, "reference_cases.json")) as f:
        d = json.load(f)
    root = tmp_path_factory.mktemp("piro_assets")
    for rel, sections in d["assets"].items():
        write_ini(os.path.join(root, *rel.split("/")), sections)
    for name, sections in d["cases"].items():
        write_ini(os.path.join(root, name), sections)
    return str(root)


# case, lu_mode, exact (None) or relative tolerance
CASES = [
    ("HeatEq.ini", 0, 1e-6),    # 10x10x31, backward Euler, downwind, JLI (solver.ini), top face at 1.0
    ("AdvEq.ini", 0, None),     # 31^3, v & grad(U), upwind, forward Euler, v = 100 * (0, 0, -1)
    ("LUDecomp.ini", 1, None),  # 3^3, scheme 27 in the hash table as the reference runs it
    ("LUDecomp.ini", 0, 1e-5),  # the same case solved (banded LU) against an FP64 solve
]


@pytest.mark.parametrize("name,lu_mode,tol", CASES)
def test_reference_case_matches_oracle(cuda, oracle, assets, name, lu_mode, tol):
    from case_oracle import run_case
    from piro_b200.case import Case
    ref = run_case(assets, name, lu_mode=lu_mode)
    c = Case(assets, name, lu_mode=lu_mode)
    steps = c.solve()
    assert steps == ref["steps"] and steps >= 1
    var = ref["names"][1]
    got, want = c.get(var), ref["fields"][1]
    assert np.all(np.isfinite(got))
    if tol is None:
        assert f32_bits_equal(got, want), np.abs(got - want).max()
    else:
        np.testing.assert_allclose(got, want, rtol=tol, atol=tol * np.abs(want).max())
    c.close()
