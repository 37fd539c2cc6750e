"""Batched evaluation of several independent instances (merged
multi-instance launches, one CUDA graph): every instance's result in the
batch equals its result evaluated alone, for the whole batch and for
subsets, and instances left out are not touched.

Tolerance: batch and single runs execute the same arithmetic; only the order
of FP32 atomic accumulations may differ, so the results agree to FP32
rounding (bar 1e-5 relative l2, observed ~1e-7)."""
import numpy as np
import pytest

import fixtures
from ddfmm_b200 import _lib, wave3d

pytestmark = pytest.mark.gpu
TOL = 1e-5
CASES = ["sphere_k8_n5000_p4_helm", "sphere_k4_n1500_p4_expr", "cluster_k4_n1500_p4_helm_m8",
         "ellipsoid_k8_n3000_p4_helm", "sphere_k16_n4000_p4_helm"]


def _session(c, tmp_path, i):
    d = tmp_path / ("ops%d" % i)
    d.mkdir()
    ldp, hdp = c.write_operators(str(d))
    p = c.params
    mlib = wave3d.Mlib3d()
    mlib.setup({"-mlib3d_ldname": ldp, "-mlib3d_hdname": hdp})
    w = wave3d.Wave3d(precision=_lib.MIXED)
    w.posptr = c.pos
    w.kernel = p["kernel"]
    w.mlibptr = mlib
    w.geomprtn = p["nc"]
    w.setup({"-wave3d_ACCU": str(p["accu"]), "-wave3d_NPQ": str(p["npq"]), "-wave3d_K": str(p["K"]),
             "-wave3d_ptsmax": str(p["ptsmax"]), "-wave3d_maxlevel": str(p["maxlevel"])})
    return w


@pytest.fixture(scope="module")
def setup(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("batch")
    cases = [fixtures.Case(n) for n in CASES]
    waves = [_session(c, tmp, i) for i, c in enumerate(cases)]
    rng = np.random.default_rng(3)
    dens = [(rng.standard_normal(len(c.den)) + 1j * rng.standard_normal(len(c.den))).astype(np.complex64)
            for c in cases]
    alone = []
    for w, d in zip(waves, dens):
        v = np.zeros(len(d), dtype=np.complex64)
        w.eval(d, v)
        alone.append(v)
    b = wave3d.Batch(waves)
    yield cases, waves, dens, alone, b
    b.close()
    for w in waves:
        w.close()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_batch_matches_each_instance_alone(setup):
    cases, waves, dens, alone, b = setup
    print("batch of %d instances: %d launches per matvec" % (len(waves), b.launches()))
    for rep in range(2):  # the second call replays the captured graph
        vals = [np.zeros(len(d), dtype=np.complex64) for d in dens]
        b.eval(dens, vals)
        for n, v, a in zip(CASES, vals, alone):
            r = _rel(v, a)
            print("rep %d %s: batch vs alone %.3e" % (rep, n, r))
            assert r <= TOL, (n, r)


def test_batch_subset_leaves_others_untouched(setup):
    cases, waves, dens, alone, b = setup
    sel = [1, 3]
    vals = [np.full(len(d), 7 + 7j, dtype=np.complex64) for d in dens]
    b.eval([d if i in sel else None for i, d in enumerate(dens)], vals)
    for i in range(len(dens)):
        if i in sel:
            assert _rel(vals[i], alone[i]) <= TOL, (i, _rel(vals[i], alone[i]))
        else:
            assert np.all(vals[i] == 7 + 7j)
    # and the full batch again afterwards
    vals = [np.zeros(len(d), dtype=np.complex64) for d in dens]
    b.eval(dens, vals)
    for i in range(len(dens)):
        assert _rel(vals[i], alone[i]) <= TOL


def test_batch_is_closer_to_reference_than_tolerance(setup):
    # each instance's batched result stays within the mixed-form bar of the
    # reference's own FP64 output for the fixture densities
    cases, waves, dens, alone, b = setup
    fdens = [c.den.astype(np.complex64) for c in cases]
    vals = [np.zeros(len(d), dtype=np.complex64) for d in fdens]
    b.eval(fdens, vals)
    for n, c, v in zip(CASES, cases, vals):
        r = _rel(v.astype(np.complex128), c.val)
        print("%s: batch vs reference %.3e" % (n, r))
        assert r <= 2e-5, (n, r)
