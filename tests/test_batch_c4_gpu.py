"""A batch shaped like the batched-instances configuration: 16 independent
spheres and ellipsoids with K drawn from {4, 8, 16, 32} (N = 25 pi K^2, up to
80k points each), P = 6, complex64 N(0,1) densities, mixed form, evaluated
as one batch (merged multi-instance launches replayed as one CUDA graph).

Each instance's batched value is checked three ways:
  * against the same session evaluated alone (same arithmetic; only the
    order of FP32 atomic sums differs): 1e-5 relative l2;
  * against the plain FP64 GPU form of the same instance (itself equal to
    the reference's output to 1e-10, tests/test_parity*.py): the mixed
    tolerance 2e-5;
  * against the FP64 direct sum at 200 seeded targets (the accuracy check of
    Wave3d::check, src/wave3d_check.cpp:22-100): 1e-4."""
import numpy as np
import pytest

from ddfmm_b200 import _lib, wave3d
from ddfmm_b200 import workloads as wl

pytestmark = pytest.mark.gpu
TOL_ALONE = 1e-5
TOL_MIXED = 2e-5
TOL_DIRECT = 1e-4


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def mix():
    rng = np.random.default_rng(64)
    Ks = [int(k) for k in rng.permutation([4, 8, 16, 32] * 4)]
    ws = wl.instance_mix(Ks, 300)
    waves = [wave3d.from_workload(w, precision=_lib.MIXED) for w in ws]
    yield Ks, ws, waves
    for w in waves:
        w.close()


def test_c4_shaped_batch(mix):
    Ks, ws, waves = mix
    rng = np.random.default_rng(5)
    dens = [(rng.standard_normal(w.N) + 1j * rng.standard_normal(w.N)).astype(np.complex64) for w in ws]
    alone = []
    for wv, d in zip(waves, dens):
        v = np.zeros(len(d), dtype=np.complex64)
        wv.eval(d, v)
        alone.append(v)
    b = wave3d.Batch(waves)
    try:
        print("batch of %d instances (K %s, %d points): %d launches per matvec"
              % (len(ws), Ks, sum(w.N for w in ws), b.launches()))
        for rep in range(2):  # capture, then replay of the graph
            vals = [np.zeros(len(d), dtype=np.complex64) for d in dens]
            b.eval(dens, vals)
            for k, (v, a) in enumerate(zip(vals, alone)):
                r = _rel(v, a)
                assert r <= TOL_ALONE, (k, Ks[k], r)
    finally:
        b.close()
    worst_plain = worst_direct = 0.0
    for k, (w, wv, d, v) in enumerate(zip(ws, waves, dens, vals)):
        p = wave3d.from_workload(w, precision=_lib.PLAIN_FP64)
        ref = np.zeros(w.N, dtype=np.complex128)
        p.eval(d.astype(np.complex128), ref)
        e = p.check(d.astype(np.complex128), v.astype(np.complex128), w.check_ids())
        p.close()
        r = _rel(v.astype(np.complex128), ref)
        worst_plain, worst_direct = max(worst_plain, r), max(worst_direct, e)
        print("instance %d (%s K=%d N=%d): batch vs plain FP64 %.3e, vs FP64 direct %.3e"
              % (k, w.geometry, Ks[k], w.N, r, e))
        assert r <= TOL_MIXED, (k, r)
        assert e <= TOL_DIRECT, (k, e)
    print("worst: vs plain FP64 %.3e, vs direct %.3e" % (worst_plain, worst_direct))
