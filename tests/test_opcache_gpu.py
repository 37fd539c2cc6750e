"""Packed translation operators shared across sessions (process-wide cache,
mixed form): a second session on the same operator files, kernel and
accuracy reuses the first one's packed M2M / L2L / M2L / E2 operators, takes
less device memory, and computes the same matvec; it keeps working after the
first one is closed.  Sessions that differ in accuracy level share nothing.

Tolerance: both sessions run the same arithmetic on the same packed
operators; FP32 atomic accumulation order may differ (bar 1e-6 relative)."""
import numpy as np
import pytest

from ddfmm_b200 import _lib, wave3d
from ddfmm_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_second_session_shares_packed_operators():
    w1 = wl.sphere(8, 5000, accu=1, seed=0)
    w2 = wl.ellipsoid(8, 5000, accu=1, seed=4)  # another geometry, same operator files
    a = wave3d.from_workload(w1, precision=_lib.MIXED)
    b = wave3d.from_workload(w2, precision=_lib.MIXED)
    b1 = wave3d.from_workload(w2, precision=_lib.MIXED)  # identical to b
    sa, sb, sb1 = a.stats(), b.stats(), b1.stats()
    print("device GB: first %.3f, second geometry %.3f, repeat %.3f; setup s %.2f %.2f %.2f"
          % (sa["device_bytes"] / 1e9, sb["device_bytes"] / 1e9, sb1["device_bytes"] / 1e9,
             sa["setup_seconds"], sb["setup_seconds"], sb1["setup_seconds"]))
    assert sb1["device_bytes"] < sa["device_bytes"]
    den = w2.densities(np.complex64)
    vb = np.zeros(w2.N, dtype=np.complex64)
    vb1 = np.zeros(w2.N, dtype=np.complex64)
    b.eval(den, vb)
    b1.eval(den, vb1)
    assert _rel(vb1, vb) <= 1e-6
    # accuracy against the FP64 direct sum is that of the mixed form
    relerr = b1.check(den.astype(np.complex128), vb1.astype(np.complex128), w2.check_ids())
    print("shared-operator session relerr vs FP64 direct %.3e" % relerr)
    assert relerr < 1e-3
    a.close()
    b.close()
    vb2 = np.zeros(w2.N, dtype=np.complex64)
    b1.eval(den, vb2)  # the operators it shares outlive their creators
    assert _rel(vb2, vb) <= 1e-6
    b1.close()


def test_different_accuracy_shares_nothing():
    p4 = wave3d.from_workload(wl.sphere(4, 1500, accu=1), precision=_lib.MIXED)
    p6a = wave3d.from_workload(wl.sphere(4, 1500, accu=2), precision=_lib.MIXED)
    s6a = p6a.stats()["device_bytes"]
    p4.close()
    p6a.close()
    p6b = wave3d.from_workload(wl.sphere(4, 1500, accu=2), precision=_lib.MIXED)
    assert p6b.stats()["device_bytes"] == s6a  # nothing left to share once both are closed
    p6b.close()
