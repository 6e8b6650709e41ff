"""The C-ABI library loads and exports every symbol include/sg_api.h declares
(no compute calls: this file runs without a GPU)."""
import os
import re
import subprocess

import subgraph_b200 as sg
from subgraph_b200._lib import EXPORTS

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "sg_api.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(sg_[a-z0-9_]+)\s*\(", txt)))


def test_header_and_binding_agree():
    assert sorted(EXPORTS) == declared_symbols()


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", sg.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\s[TW]\s(sg_\w+)$", out, flags=re.M))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing


def test_library_loads_and_reports_errors():
    L = sg.lib()
    assert L.sg_version().decode().startswith("subgraph_b200")
    assert L.sg_estimate(None, 0, 3, 1, None) == 1
    assert "bad argument" in L.sg_last_error().decode()

