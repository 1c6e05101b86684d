"""The C-ABI library loads without a GPU and exports every function that
include/fastiso_b200.h declares; the Python bindings cover the same set."""
import ctypes as C
import pathlib
import re

from fastiso_b200 import abi

ROOT = pathlib.Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "fastiso_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(fi_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for must in ("fi_create", "fi_init", "fi_rhs", "fi_run", "fi_init_integrator", "fi_step", "fi_destroy",
                 "fi_rhs_noalloc", "fi_ensemble_create", "fi_ensemble_step", "fi_set_tiles"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(abi.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_match_the_header():
    assert set(declared_functions()) == set(abi.exported_symbols())
