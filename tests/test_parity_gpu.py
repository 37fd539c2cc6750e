"""GPU plain FP64 form against the reference's own output (golden fixtures).

Bar (north star): relative l2 difference <= 1e-10 on identical points,
densities and operators, through the C-ABI (Wave3d mirror)."""
import numpy as np
import pytest

import fixtures
from ddfmm_b200 import wave3d

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _session(c, tmp_path):
    ldp, hdp = c.write_operators(str(tmp_path))
    p = c.params
    mlib = wave3d.Mlib3d()
    mlib.setup({"-mlib3d_ldname": ldp, "-mlib3d_hdname": hdp})
    w = wave3d.Wave3d()
    w.posptr = c.pos
    w.kernel = p["kernel"]
    w.mlibptr = mlib
    w.geomprtn = p["nc"]
    w.setup({"-wave3d_ACCU": str(p["accu"]), "-wave3d_NPQ": str(p["npq"]), "-wave3d_K": str(p["K"]),
             "-wave3d_ptsmax": str(p["ptsmax"]), "-wave3d_maxlevel": str(p["maxlevel"])})
    return w


@pytest.mark.parametrize("name", fixtures.case_names())
def test_matches_reference_output(name, tmp_path):
    c = fixtures.Case(name)
    w = _session(c, tmp_path)
    val = np.zeros_like(c.den)
    w.eval(c.den, val)
    rel = np.linalg.norm(val - c.val) / np.linalg.norm(c.val)
    worst = np.max(np.abs(val - c.val)) / np.max(np.abs(c.val))
    print("parity %s: rel l2 %.3e, max %.3e" % (name, rel, worst))
    assert rel <= TOL and worst <= 10 * TOL, (rel, worst)
    # Wave3d::check against the FP64 direct sum reproduces the reference's relerr
    relerr = w.check(c.den, val, c.chk)
    assert abs(relerr - c.relerr) <= 1e-6 * max(c.relerr, 1e-12) + 1e-12, (relerr, c.relerr)
    w.close()


def test_repeated_eval_does_not_accumulate(tmp_path):
    c = fixtures.Case("cluster_k4_n1500_p4_helm_m8")
    w = _session(c, tmp_path)
    a = np.zeros_like(c.den)
    b = np.zeros_like(c.den)
    w.eval(c.den, a)
    w.eval(c.den, b)
    assert np.linalg.norm(a - b) / np.linalg.norm(a) < 1e-14
    w.close()
