"""The C-ABI library loads and exports every symbol include/mbx_b200.h declares (CPU)."""
import ctypes
import os
import re

import pytest

from mbx_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "mbx_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(mbx_\w+)\s*\(", text, re.M)))


def test_header_declares_the_abi():
    syms = declared_symbols()
    for s in ("mbx_create", "mbx_energy", "mbx_evaluate", "mbx_poly", "mbx_nmers", "mbx_evaluate_dcoef"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    if not os.path.exists(capi.LIB_PATH):
        pytest.fail("libmbx_b200.so is not built; run python -m mbx_b200.build")
    L = ctypes.CDLL(capi.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert capi.lib().mbx_version().decode().startswith("mbx_b200")


def test_evaluator_info_without_gpu():
    for name in capi.EVALUATORS:
        nb, nreal, nv, nc = capi.evaluator_info(name)
        assert nb in (2, 3) and nreal > 0 and nv > 0 and nc > 0
    with pytest.raises(capi.MBXError):
        capi.evaluator_info("nope")
