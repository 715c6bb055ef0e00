"""CPU checks of the drop-in boundary: the sm_100a library loads without a GPU and exports
every entry point that include/*.h declares (no compute call is made here)."""
import ctypes
import glob
import os
import re

import ceos_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(hdr).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(ceos_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ["ceos_create", "ceos_pattern", "ceos_slot_map", "ceos_evaluate", "ceos_evaluate_device",
                 "ceos_commit_state", "ceos_last_error", "ceos_destroy", "ceos_analysis"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(ceos_b200.LIBPATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_bad_arguments_rejected_without_gpu():
    """Argument validation happens before any device call."""
    lib = ceos_b200.lib()
    h = ctypes.c_void_p()
    assert lib.ceos_create(None, None, 0, 0, 0, ctypes.byref(h)) == -1
    assert lib.ceos_pattern(None, None, None, None, None, None) == -1


def test_fortran_module_binds_exported_symbols():
    """include/ceos_gpu_mod.f90 (the ISO_C_BINDING module a Fortran host uses) binds only symbols the
    library exports, and its derived types match the C structs field by field."""
    src = open(os.path.join(ROOT, "include", "ceos_gpu_mod.f90")).read()
    names = set(re.findall(r'bind\(C,\s*name="(ceos_[a-z0-9_]+)"\)', src))
    assert {"ceos_create", "ceos_pattern", "ceos_evaluate", "ceos_commit_state", "ceos_last_error",
            "ceos_destroy"} <= names
    lib = ctypes.CDLL(ceos_b200.LIBPATH)
    assert all(hasattr(lib, n) for n in names), names
    assert "integer(c_int) :: n_nodes, n_elem" in src and "type(c_ptr) :: X, conn, mat_id" in src
    assert "integer(c_int) :: model, per_element, n_params" in src and "type(c_ptr) :: params" in src
    assert max(len(ln) for ln in src.splitlines()) <= 132  # free-form source line limit
