"""Extract PIRO's own example cases into tests/golden/reference_cases.json.

Run where the PIRO source tree is present, named by PIRO_REF_DIR:

    PIRO_REF_DIR=<PIRO tree> python tests/golden/make_reference_cases.py

maketest.sh:101-130 runs Test/HeatEq.ini, Test/AdvEq.ini and Test/LUDecomp.ini
from a copy of dependencies/assets with the case file placed beside setup.ini.
The GPU machine has no PIRO tree, so this script stores what those runs read:
every key of the three case files and of the asset files (setup.ini,
solver.ini, Data/hashtable.ini, IC/distribution.ini), parsed by the rules of
PIRO's IniReader (src/fileutilities.cpp:124-183: comment lines dropped, keys
and values stripped of spaces).  tests/test_gpu_reference_cases.py writes them
back out as .ini files and runs the cases end to end.
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))                   # tests/ (case_oracle)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))  # the repository root (oracle)

CASES = ["HeatEq.ini", "AdvEq.ini", "LUDecomp.ini"]
ASSETS = ["setup.ini", "solver.ini", os.path.join("Data", "hashtable.ini"), os.path.join("IC", "distribution.ini")]


def main() -> None:
    from case_oracle import read_ini
    ref = os.environ.get("PIRO_REF_DIR", "")
    if not ref or not os.path.isdir(os.path.join(ref, "Test")):
        raise SystemExit("set PIRO_REF_DIR to the PIRO source tree")
    out = {"source": "PIRO Test/*.ini and dependencies/assets, parsed by IniReader's rules", "cases": {},
           "assets": {}}
    for name in CASES:
        out["cases"][name] = read_ini(os.path.join(ref, "Test", name))
    for rel in ASSETS:
        out["assets"][rel.replace(os.sep, "/")] = read_ini(os.path.join(ref, "dependencies", "assets", rel))
    path = os.path.join(HERE, "reference_cases.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", path)


if __name__ == "__main__":
    main()
