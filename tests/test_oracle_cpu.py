"""The oracle pinned against the reference.

* the numpy restatement (oracle/restate.py) reproduces the reference
  binary's outputs stored in the golden fixtures, and its tree counts;
* the FFTW / BLAS stand-ins of the reference build agree with numpy.
"""
import os
import subprocess
import time

import numpy as np
import pytest

import fixtures
import restate

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIMTEST = os.path.join(ROOT, "oracle", "_ref", "shimtest")

@pytest.fixture(autouse=True, scope="module")
def _one_blas_thread():
    # the restatement multiplies many tiny matrices: BLAS threads only thrash
    from threadpoolctl import threadpool_limits
    with threadpool_limits(1):
        yield


CASES = ["sphere_k4_n1500_p4_expr", "sphere_k4_n1500_p6_helm", "cluster_k4_n1500_p4_helm_m8",
         "ellipsoid_k8_n3000_p4_helm", "sphere_k8_n5000_p4_helm"]


def _oracle(c, tmp_path):
    ldp, hdp = c.write_operators(str(tmp_path))
    p = c.params
    return restate.Wave3dOracle(c.pos, p["K"], p["nc"], p["ptsmax"], p["maxlevel"], p["accu"], p["kernel"],
                                restate.read_ld(ldp), restate.read_hd(hdp), p["npq"])


@pytest.mark.parametrize("name", CASES)
def test_restatement_matches_reference(name, tmp_path):
    c = fixtures.Case(name)
    o = _oracle(c, tmp_path)
    total, empty, boxes, dirs = o.counts()
    assert (total, empty) == (c.ref_total_boxes, c.ref_deleted)
    assert boxes == c.ref_boxes and dirs == c.ref_dirs
    t = time.time()
    val = o.eval(c.den)
    rel = np.linalg.norm(val - c.val) / np.linalg.norm(c.val)
    assert rel < 1e-12, rel
    truth = o.direct(c.den, c.chk)
    relerr = np.linalg.norm(truth - val[c.chk]) / np.linalg.norm(val[c.chk])
    assert abs(relerr - c.relerr) <= 1e-6 * c.relerr


def test_restatement_coincident_points_use_r_equals_one():
    """src/kernel3d.cpp:47-49: r < 1e-8 is replaced by 1, so G(p, p) = exp(2 pi i)."""
    K = restate.kernel(np.zeros((3, 1)), np.zeros((3, 1)), 0)
    assert abs(K[0, 0] - 1.0) < 1e-15
    K = restate.kernel(np.zeros((3, 1)), np.full((3, 1), 1e-9), 1)
    assert abs(K[0, 0] - 1.0) < 1e-15


@pytest.mark.skipif(not os.access(SHIMTEST, os.X_OK), reason="oracle not built (make -C oracle)")
@pytest.mark.parametrize("n", [8, 12, 16])
def test_fftw_and_blas_shims_match_numpy(n):
    rng = np.random.default_rng(n)
    g = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
    m, k = 7, 5
    A = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
    x = rng.standard_normal(k) + 1j * rng.standard_normal(k)
    y = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    # the shim reads row-major (FFTW order); feed g in C order
    lines = [str(n)] + ["%.17g %.17g" % (v.real, v.imag) for v in g.ravel(order="C")]
    lines += ["%d %d" % (m, k)] + ["%.17g %.17g" % (v.real, v.imag) for v in A.ravel(order="F")]
    lines += ["%.17g %.17g" % (v.real, v.imag) for v in x] + ["%.17g %.17g" % (v.real, v.imag) for v in y]
    out = subprocess.run([SHIMTEST], input="\n".join(lines), capture_output=True, text=True, check=True).stdout
    vals = np.array([complex(float(a), float(b)) for a, b in (l.split() for l in out.split("\n") if l)])
    N = n ** 3
    fwd, bwd, gemv = vals[:N].reshape((n, n, n)), vals[N:2 * N].reshape((n, n, n)), vals[2 * N:]
    assert np.abs(fwd - np.fft.fftn(g)).max() <= 1e-12 * np.abs(np.fft.fftn(g)).max()
    assert np.abs(bwd - np.fft.ifftn(g) * N).max() <= 1e-12 * np.abs(bwd).max()
    assert np.abs(gemv - (A @ x + y)).max() <= 1e-13 * np.abs(gemv).max()
