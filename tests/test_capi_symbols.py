"""The C-ABI library loads and exports every symbol include/pybrown_b200.h declares (no GPU calls)."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pybrown_b200.h")


def declared_symbols():
    with open(HEADER) as f:
        src = "\n".join(ln for ln in f.read().splitlines() if not ln.lstrip().startswith("#"))
    return re.findall(r"PBG_API\s+[A-Za-z_ ]+?\**\s*\**([A-Za-z_][A-Za-z0-9_]*)\s*\(", src)


def test_header_declares_reference_abi():
    names = set(declared_symbols())
    for ref in ("RPY_M_matrix", "RPY_Smith_M_matrix", "JO_2B_R_matrix", "JO_R_lubrication_correction_matrix",
                "pointer_pbc_matrix", "pointer_immobile_pbc_matrix", "check_overlaps"):
        assert ref in names


def test_library_exports_every_declared_symbol():
    from pybrown_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.pbg_version() >= 10000
