"""ddfmm_eval_device_noalloc: the matvec for callers that cannot allocate
device memory while they run (a host application whose allocator owns the
whole GPU, or a loop with a device-memory budget fixed up front).  Its
V-list spectra live in the library's fixed 16 MiB device array instead of
session memory; the result must equal ddfmm_eval_device's on the same
session, for plain FP64 and for mixed sessions, on two calls in a row (the
array keeps the previous call's contents).

This file is named to be collected last, so a stop-at-first-failure run has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import fixtures
from ddfmm_b200 import _lib, wave3d

pytestmark = pytest.mark.gpu
TOL = 1e-10        # the parity tolerance of the plain GPU tests
TOL_MIXED = 2e-5   # the mixed-form tolerance of the GPU tests


def _session(c, tmp_path, precision=_lib.PLAIN_FP64):
    ldp, hdp = c.write_operators(str(tmp_path))
    p = c.params
    mlib = wave3d.Mlib3d()
    mlib.setup({"-mlib3d_ldname": ldp, "-mlib3d_hdname": hdp})
    w = wave3d.Wave3d(precision=precision)
    w.posptr = c.pos
    w.kernel = p["kernel"]
    w.mlibptr = mlib
    w.geomprtn = p["nc"]
    w.setup({"-wave3d_ACCU": str(p["accu"]), "-wave3d_NPQ": str(p["npq"]), "-wave3d_K": str(p["K"]),
             "-wave3d_ptsmax": str(p["ptsmax"]), "-wave3d_maxlevel": str(p["maxlevel"])})
    return w


@pytest.mark.parametrize("name,precision", [("sphere_k8_n5000_p4_helm", _lib.PLAIN_FP64),
                                            ("sphere_k4_n1500_p6_helm", _lib.PLAIN_FP64),
                                            ("sphere_k8_n5000_p4_helm", _lib.MIXED)])
def test_noalloc_eval_matches_eval_device_twice(name, precision, tmp_path):
    import torch
    lib = _lib.load()
    c = fixtures.Case(name)
    w = _session(c, tmp_path, precision)
    tol = TOL if precision == _lib.PLAIN_FP64 else TOL_MIXED
    dev = torch.device("cuda", 0)
    den = torch.from_numpy(np.ascontiguousarray(c.den).view(np.float64)).to(dev)
    ref = torch.empty_like(den)
    out = torch.empty_like(den)
    _lib.check(lib.ddfmm_eval_device(w._s, C.c_void_p(den.data_ptr()), C.c_void_p(ref.data_ptr()), None))
    torch.cuda.synchronize()
    a = ref.cpu().numpy().view(np.complex128)
    for _ in range(2):  # the shared array keeps the last call's contents: reuse must not leak
        out.fill_(float("nan"))
        _lib.check(lib.ddfmm_eval_device_noalloc(w._s, C.c_void_p(den.data_ptr()), C.c_void_p(out.data_ptr()), None))
        torch.cuda.synchronize()
        b = out.cpu().numpy().view(np.complex128)
        assert np.linalg.norm(b - a) / np.linalg.norm(a) <= tol
        assert np.linalg.norm(b - c.val) / np.linalg.norm(c.val) <= tol
    w.close()


def test_noalloc_rejects_sessions_beyond_the_fixed_scratch(tmp_path):
    import torch
    lib = _lib.load()
    c = fixtures.Case("sphere_k16_n4000_p4_helm")  # 19.9 MiB of spectra
    w = _session(c, tmp_path)
    den = torch.zeros(2 * len(c.den), dtype=torch.float64, device="cuda")
    out = torch.zeros_like(den)
    rc = lib.ddfmm_eval_device_noalloc(w._s, C.c_void_p(den.data_ptr()), C.c_void_p(out.data_ptr()), None)
    assert rc == 1
    assert b"MiB" in lib.ddfmm_last_error()
    w.close()
