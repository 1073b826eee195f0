"""The C-ABI library builds, loads and exports every entry point declared in include/wtbgpu.h."""
import os
import re

import pytest

from wantibexos_b200 import build as B
from wantibexos_b200 import wtbgpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "wtbgpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(wtbg_[a-z0-9_]+)\s*\(", txt)))


def test_header_lists_all_bound_symbols():
    assert declared_symbols() == sorted(wtbgpu.EXPORTS)


def test_library_loads_and_exports():
    B.build()
    lib = wtbgpu.load_library()
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_create_without_device_reports_status():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import ctypes as C
    lib = wtbgpu.load_library()
    h = C.c_void_p()
    assert lib.wtbg_create(C.byref(h), 0) == -9
    assert lib.wtbg_error_string(-9) == b"no CUDA device"
    with pytest.raises(wtbgpu.WtbgError):
        wtbgpu.Context(0)
