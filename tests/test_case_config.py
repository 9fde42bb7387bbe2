"""The case front end's error handling: piro_open reads the .ini files and
computes the initial values before its first CUDA call, so a malformed case
reports PIRO_ERR_CONFIG (with the offending section or key in the message)
on any machine, GPU or not.  Mirrors the reference's preprocess
(src/preprocess.cpp:20-208), which throws on a missing parameter and exits on
an invalid one."""
from __future__ import annotations

import json
import os
import shutil

import pytest

from conftest import ROOT

ASSETS = os.path.join(ROOT, "tests", "cases")


def case_dir(tmp_path, text=None, name="case.ini", ic=True):
    """A copy of the assets directory with one case file (the CSR heat case,
    optionally rewritten) and, unless ic is False, the IC parameters."""
    if ic:
        shutil.copytree(os.path.join(ASSETS, "IC"), tmp_path / "IC")
    for f in ("setup.ini", "solver.ini"):
        shutil.copy(os.path.join(ASSETS, f), tmp_path / f)
    shutil.copytree(os.path.join(ASSETS, "Data"), tmp_path / "Data")
    src = open(os.path.join(ASSETS, "heat_fe_csr.ini")).read()
    (tmp_path / name).write_text(src if text is None else text(src))
    return str(tmp_path), name


def open_error(assets, name):
    from piro_b200._lib import PiroError
    from piro_b200.case import Case
    with pytest.raises(PiroError) as e:
        Case(assets, name)
    return e.value


def test_missing_case_file(tmp_path):
    e = open_error(str(tmp_path), "missing.ini")
    assert "CONFIG" in str(e) and "missing.ini" in str(e)


@pytest.mark.parametrize("old,new,word", [
    ("Time = 11", "Time = eleven", "Time"),        # [Schemes] Time is an integer
    ("Time = 11", "", "Time"),                     # a required key is missing
    ("Timestep = 0.5", "Timestep = half", "Timestep"),
    ("n = 14 12 10", "n = 14 12", "Mesh"),         # [Mesh] n needs three values
    ("filename = Gaussian", "filename = Bessel", "Bessel"),  # unknown initial condition
    ("Values = 0.1", "Values = ", "Values"),       # a constant without a value
])
def test_malformed_case_is_a_config_error(tmp_path, old, new, word):
    assets, name = case_dir(tmp_path, lambda s: s.replace(old, new))
    e = open_error(assets, name)
    assert "CONFIG" in str(e) and word in str(e), str(e)


def test_missing_initial_condition_file(tmp_path):
    assets, name = case_dir(tmp_path, ic=False)
    e = open_error(assets, name)
    assert "CONFIG" in str(e) and "distribution.ini" in str(e), str(e)


def test_valid_case_without_a_gpu_fails_loudly(tmp_path):
    """A well-formed case gets past the parser; with no GPU the first CUDA
    call fails with PIRO_ERR_CUDA -- there is no CPU fallback."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the case opens")
    assets, name = case_dir(tmp_path)
    e = open_error(assets, name)
    assert "PIRO_ERR_CUDA" in str(e), str(e)


@pytest.mark.parametrize("name", ["HeatEq.ini", "AdvEq.ini", "LUDecomp.ini"])
def test_reference_cases_parse(tmp_path, name):
    """PIRO's own example cases (Test/*.ini, run by maketest.sh from a copy of
    dependencies/assets with the case file placed beside setup.ini; rebuilt
    here from tests/golden/reference_cases.json) get through the front end:
    with no GPU the first failure is the first CUDA call, never the parser."""
    import torch
    from test_gpu_reference_cases import write_ini
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the case would open")
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_cases.json")) as f:
        d = json.load(f)
    assets = tmp_path / "assets"
    for rel, sections in d["assets"].items():
        write_ini(os.path.join(assets, *rel.split("/")), sections)
    write_ini(os.path.join(assets, name), d["cases"][name])
    e = open_error(str(assets), name)
    assert "PIRO_ERR_CUDA" in str(e), str(e)
