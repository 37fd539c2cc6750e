"""The tensor-core GEMM's bounded pipeline waits, made to run out on purpose.

ddfmm_session_test_gemm_stall arms a one-shot hook: the next eval's first
tcgen05 GEMM launch bounds its mbarrier waits by a short limit and its block 0
withholds the operator copies that block waits on (a flag nothing sets), so
that wait runs out.  Nothing faults: the block stops issuing, drains what it
issued, frees its tensor memory and flags the session; the session's next
synchronous call reports DDFMM_ECUDA (the reference's counterpart is a throw,
include/commoninc.hpp:52-53), and the context stays usable: the same session
and a fresh one compute correct matvecs afterwards."""
import time

import numpy as np
import pytest

import fixtures
from ddfmm_b200 import _lib, wave3d

pytestmark = pytest.mark.gpu
TOL_MIXED = 2e-5  # the mixed-form tolerance (tests/test_mixed_gpu.py)


def _session(c, tmp_path, precision):
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


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_gemm_wait_timeout_is_reported_and_recovered(tmp_path):
    lib = _lib.load()
    c = fixtures.Case("sphere_k8_n5000_p4_helm")
    w = _session(c, tmp_path, _lib.MIXED)
    v = np.zeros_like(c.den)
    w.eval(c.den, v)
    assert _rel(v, c.val) <= TOL_MIXED
    _lib.check(lib.ddfmm_session_test_gemm_stall(w._s, 0.002))
    t0 = time.perf_counter()
    with pytest.raises(_lib.DDFMMError) as e:
        w.eval(c.den, np.zeros_like(c.den))
    took = time.perf_counter() - t0
    assert e.value.code == 2 and "timed out" in str(e.value)
    assert took < 5.0  # the 2 ms limit, not the default 1 s or a hang
    # the flag is cleared and the hook was one-shot: the same session is correct again
    v2 = np.zeros_like(c.den)
    w.eval(c.den, v2)
    assert _rel(v2, c.val) <= TOL_MIXED
    w.close()
    # a fresh session on the same GPU (its tensor memory was freed) is correct
    w3 = _session(c, tmp_path, _lib.MIXED)
    v3 = np.zeros_like(c.den)
    w3.eval(c.den, v3)
    assert _rel(v3, c.val) <= TOL_MIXED
    w3.close()


def test_stall_hook_refuses_other_sessions(tmp_path):
    lib = _lib.load()
    c = fixtures.Case("sphere_k4_n1500_p4_expr")
    w = _session(c, tmp_path, _lib.PLAIN_FP64)
    assert lib.ddfmm_session_test_gemm_stall(w._s, 0.002) == 1
    w.close()
    m = _session(c, tmp_path, _lib.MIXED)
    assert lib.ddfmm_session_test_gemm_stall(m._s, 0.0) == 1
    assert lib.ddfmm_session_test_gemm_stall(m._s, 2.0) == 1
    m.close()
