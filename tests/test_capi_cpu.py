"""CPU checks of the C-ABI library: it loads without a GPU and exports every
function the public header declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "eqtl_b200.h")


def header_functions():
    src = open(HDR).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(eqtl_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_function():
    from eqtl_b200 import build, capi
    build.build_lib()
    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [f for f in header_functions() if not hasattr(lib, f)]
    assert not missing, missing


def test_binding_covers_header():
    from eqtl_b200 import capi
    assert sorted(capi.EXPORTS) == header_functions()


def test_open_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from eqtl_b200 import capi
    with pytest.raises(capi.EqtlError):
        capi.Context(0)
