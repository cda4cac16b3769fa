"""The C-ABI library loads (no GPU needed) and exports every function that
include/cm_b200.h declares, with the Python binding declaring each one."""
import ctypes
import os
import re

import pytest

from contactmechanics_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cm_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cm_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "cm_ccg_solve" in names and "cm_apply" in names and "cm_plan_create" in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} not bound in _lib.SIGNATURES"


def test_status_strings():
    assert _lib.status_string(_lib.CM_ERR_NAN) == "nan encountered."
    assert "different signs" in _lib.status_string(_lib.CM_ERR_BISECT)
    assert _lib.load_library().cm_version().decode().startswith("cm_b200")


def test_struct_sizes_match_header_layout():
    # cm_plan_desc: 4 ints, 4 doubles, int, 2 doubles, 3 ints (natural alignment)
    assert ctypes.sizeof(_lib.PlanDesc) == 4 * 4 + 4 * 8 + 8 + 2 * 8 + 16
    assert ctypes.sizeof(_lib.CcgResult) % 8 == 0


def test_product_path_refuses_without_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("has a GPU")
    import contactmechanics_b200 as cm
    with pytest.raises(_lib.CudaLibraryError):
        cm.PeriodicFFTElasticHalfSpace((8, 8), 1.0, (1.0, 1.0))
