"""Mixed-precision form: complex FP32 storage, 3xTF32 tensor-core
translations with FP32 accumulation, FP32 near field on FP64 differences.
MIXED runs the translations on tcgen05 (accumulators in tensor memory),
MIXED_MMA_SYNC on the warp-level mma.sync path; both are held to the bar.

Tolerance: the mixed result differs from the reference's FP64 result by FP32
rounding through ~10 chained translations; bar 2e-5 relative l2 (the method
error itself is 4e-4 at ACCU 1, 1e-6 at ACCU 2, 1e-8 at ACCU 3), and its error
against the FP64 direct sum stays within 2e-5 of the reference's.  At ACCU 3
(P = 8) this needs the mixed form's truncated low-frequency pseudo-inverse
(singular values below 1e-7 of the largest dropped)."""
import numpy as np
import pytest

import fixtures
from ddfmm_b200 import _lib, wave3d

pytestmark = pytest.mark.gpu
TOL_MIXED = 2e-5


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


@pytest.mark.parametrize("name", ["sphere_k8_n5000_p4_helm", "sphere_k4_n1500_p6_helm", "sphere_k16_n4000_p4_helm",
                                  "cluster_k4_n1500_p4_helm_m8", "sphere_k4_n1500_p4_expr", "sphere_k4_n1500_p8_helm"])
def test_mixed_close_to_reference(name, tmp_path):
    c = fixtures.Case(name)
    w = _session(c, tmp_path, _lib.MIXED)
    val = np.zeros_like(c.den)
    w.eval(c.den, val)
    rel = np.linalg.norm(val - c.val) / np.linalg.norm(c.val)
    print("mixed %s: rel l2 vs reference %.3e" % (name, rel))
    assert rel <= TOL_MIXED, rel
    relerr = w.check(c.den, val, c.chk)
    assert abs(relerr - c.relerr) <= TOL_MIXED + 1e-3 * c.relerr, (relerr, c.relerr)
    # complex64 in, complex64 out gives the same matvec (up to FP32 rounding:
    # atomic accumulation orders differ from run to run)
    v64 = np.zeros(len(c.den), dtype=np.complex64)
    w.eval(c.den.astype(np.complex64), v64)
    d = np.linalg.norm(v64 - val) / np.linalg.norm(val)
    print("mixed %s: complex64 I/O vs complex128 I/O %.3e" % (name, d))
    assert d <= TOL_MIXED
    w.close()


@pytest.mark.parametrize("name", ["sphere_k8_n5000_p4_helm", "sphere_k4_n1500_p6_helm", "cluster_k4_n1500_p4_helm_m8"])
def test_tcgen05_and_mma_sync_translations_agree(name, tmp_path):
    """Same FP32 form, two tensor-core paths: they differ only by FP32
    accumulation order (both 3xTF32 products with FP32 sums)."""
    c = fixtures.Case(name)
    vals = {}
    for prec in (_lib.MIXED, _lib.MIXED_MMA_SYNC):
        w = _session(c, tmp_path, prec)
        v = np.zeros_like(c.den)
        w.eval(c.den, v)
        vals[prec] = v
        rel = np.linalg.norm(v - c.val) / np.linalg.norm(c.val)
        print("precision %d %s: rel l2 vs reference %.3e" % (prec, name, rel))
        assert rel <= TOL_MIXED, rel
        w.close()
    d = np.linalg.norm(vals[_lib.MIXED] - vals[_lib.MIXED_MMA_SYNC]) / np.linalg.norm(c.val)
    print("tcgen05 vs mma.sync %s: %.3e" % (name, d))
    assert d <= TOL_MIXED


def test_c64_entry_points_refuse_plain_sessions(tmp_path):
    c = fixtures.Case("sphere_k4_n1500_p4_expr")
    w = _session(c, tmp_path, _lib.PLAIN_FP64)
    with pytest.raises(_lib.DDFMMError) as e:
        w.eval(c.den.astype(np.complex64), np.zeros(len(c.den), dtype=np.complex64))
    assert e.value.code == 1
    w.close()
