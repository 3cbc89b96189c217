"""The C-ABI shared library on a host without a GPU: it loads, exports every
entry point include/tpicb200.h declares (and tpic_b200._lib binds), and the
compute path fails loudly instead of falling back to the CPU."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import pytest

from tpic_b200 import _lib

HEADER = Path(__file__).resolve().parent.parent / "include" / "tpicb200.h"


def declared_functions() -> set:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return set(re.findall(r"\b(tpicb200_[a-z0-9_]+)\s*\(", text))


def test_header_declares_the_path():
    names = declared_functions()
    for stage in ("tpicb200_mover", "tpicb200_sort", "tpicb200_sort_binned", "tpicb200_deposit",
                  "tpicb200_deposit_species", "tpicb200_fold_periodic", "tpicb200_mass_apply",
                  "tpicb200_field_solve", "tpicb200_field_advance", "tpicb200_energy", "tpicb200_cycle"):
        assert stage in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.EXPORTS) == declared_functions()


def test_version_and_error_strings():
    lib = _lib.load()
    assert lib.tpicb200_version().decode().startswith("tpicb200")
    assert isinstance(lib.tpicb200_last_error(), bytes)


def test_no_cpu_fallback_without_a_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    grid = _lib.Grid(4, 4, 4, 1.0, 1.0, 1.0)
    opts = _lib.Options(0.1, 0.5, 1.0, 1e-8, 30, 100, _lib.PRECISION_MIXED, 1000, _lib.MASS_LAYOUT_RECORDS)
    handle = C.c_void_p()
    status = lib.tpicb200_create(C.byref(grid), C.byref(opts), C.byref(handle))
    assert status == _lib.BACKEND_FAILURE
    assert "no CUDA device" in lib.tpicb200_last_error().decode()
    assert not handle.value
    with pytest.raises(_lib.TpicError):
        _lib.check(status)


def test_invalid_arguments_are_rejected_before_any_device_work():
    lib = _lib.load()
    assert lib.tpicb200_destroy(None) == _lib.SUCCESS
    assert lib.tpicb200_mover(None, 1.0, None, None, None, None, None) == _lib.INVALID_ARGUMENT
    assert lib.tpicb200_cycle(None, None, 1, None, None) == _lib.INVALID_ARGUMENT
