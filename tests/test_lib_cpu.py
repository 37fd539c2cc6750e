"""The C-ABI library: loads without a GPU and exports every declared symbol."""
import os
import re

import pytest

from ddfmm_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "ddfmm.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(ddfmm_\w+)\s*\(", src, re.M)))


def test_header_declares_the_binding():
    assert set(declared_functions()) == set(_lib.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_create_rejects_bad_arguments(lib):
    import ctypes as C
    import numpy as np
    pos = np.zeros((4, 3))
    out = C.c_void_p()
    dp = C.POINTER(C.c_double)
    rc = lib.ddfmm_session_create(pos.ctypes.data_as(dp), 4, 7, 1, 4, 4.0, None, 100, 8, 4, b"a", b"b", 0,
                                  C.byref(out))
    assert rc == 1 and b"kernel" in lib.ddfmm_last_error()
    rc = lib.ddfmm_session_create(pos.ctypes.data_as(dp), 4, 0, 5, 4, 4.0, None, 100, 8, 4, b"a", b"b", 0,
                                  C.byref(out))
    assert rc == 1 and b"ACCU" in lib.ddfmm_last_error()
    assert lib.ddfmm_eval(None, None, None) == 1


def test_no_gpu_reports_cuda_error(lib):
    pytest.importorskip("torch")
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import ctypes as C
    import numpy as np
    pos = np.zeros((4, 3))
    out = C.c_void_p()
    rc = lib.ddfmm_session_create(pos.ctypes.data_as(C.POINTER(C.c_double)), 4, 0, 1, 4, 4.0, None, 100, 8, 4,
                                  b"a", b"b", 0, C.byref(out))
    assert rc == 2
