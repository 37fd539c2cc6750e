"""The C++ operator precompute (ddfmm_precompute_operators) against the numpy
restatement in ddfmm_b200.precompute, and its files run through the
reference binary.

The two generators draw different random samples and use different (equally
valid) factorizations, so the high-frequency factors are compared by what
they must deliver -- the far-field approximation error of each wedge, at the
EPS of its accuracy level (matlab/aug3d_hghdata.m:47-54) -- and by their
skeleton ranks; the low-frequency surfaces and FFT'd tensors are compared
directly.
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

from ddfmm_b200 import _lib, formats, geometry, precompute

EPS = {1: 1e-4, 2: 1e-6, 3: 1e-8}


def _gen(tmp_path, kind, accu, wmax, threads=0, ld=True, hd=True, tag=""):
    ldp = str(tmp_path / ("ld%s.bin" % tag)) if ld else None
    hdp = str(tmp_path / ("hd%s.bin" % tag)) if hd else None
    precompute.native_operators(kind, accu, wmax, ldp, hdp, threads)
    return ldp, hdp


def _children_sources(hd, W, n, P):
    """The children's source collection of wedge n (aug3d_hghdata.m:94-102)."""
    pspre = precompute._surface_grid(W / 2, P) if W == 1 else hd[W / 2][precompute._hgh_predir(n)].uep
    sgs = np.array([[(-1) ** (1 - ((t >> d) & 1)) for d in range(3)] for t in range(8)], dtype=float).T * W / 4
    return np.unique(np.hstack([pspre + sgs[:, t:t + 1] for t in range(8)]).T, axis=0).T


def _far_targets(rng, W, n, count=300):
    """Random points of the wedge's cone at distances D..5D, D = W^2 + W."""
    Cw, D = 4 * W, W * W + W
    the = (rng.random(count) * 2 - 1 + n[0]) / Cw * math.pi / 4
    phi = (rng.random(count) * 2 - 1 + n[1]) / Cw * math.pi / 4
    rho = D + rng.random(count) * 4 * D
    t = np.sqrt(np.tan(the) ** 2 + np.tan(phi) ** 2 + 1)
    return np.vstack([np.tan(the) / t * rho, np.tan(phi) / t * rho, rho / t])


def _wedge_error(e, ps, tgt, den, kind):
    ex = precompute.kernel_matrix(tgt, ps, kind) @ den
    E1, E2, E3 = e.uc2ue
    ap = precompute.kernel_matrix(tgt, e.uep, kind) @ (E1 @ (E2 @ (E3 @ (precompute.kernel_matrix(e.ucp, ps, kind) @ den))))
    return np.linalg.norm(ap - ex) / np.linalg.norm(ex)


@pytest.mark.parametrize("kind,accu", [(0, 1), (1, 1), (0, 2)])
def test_lowfreq_matches_numpy(tmp_path, kind, accu):
    ldp, _ = _gen(tmp_path, kind, accu, 1, hd=False)
    ld = formats.read_ld(ldp)
    assert sorted(ld) == [2.0 ** e for e in range(-7, 0)]
    rng = np.random.default_rng(0)
    for W in (2.0 ** -7, 0.125, 0.5):
        e, ref = ld[W], precompute.lowfreq_entry(accu, W, kind)
        # surfaces: the same grid arithmetic, bit for bit
        assert np.array_equal(e.uep, ref.uep) and np.array_equal(e.ucp, ref.ucp)
        assert set(e.ue2dc) == set(ref.ue2dc) and len(e.ue2dc) == 316
        for k, t in ref.ue2dc.items():
            assert np.abs(e.ue2dc[k] - t).max() <= 1e-13 * np.abs(t).max()
        # the pseudo-inverse: same rank, same far-field accuracy of the equivalent density
        assert e.uc2ue[0].shape == ref.uc2ue[0].shape
        src = (rng.random((3, 20)) - 0.5) * 0.9 * W
        tgt = rng.normal(size=(3, 50))
        tgt = tgt / np.linalg.norm(tgt, axis=0) * 4 * W
        exact = precompute.kernel_matrix(tgt, src, kind)
        b = precompute.kernel_matrix(e.ucp, src, kind)
        errs = []
        for f in (e, ref):
            X = f.uc2ue[0] @ (f.uc2ue[1] * f.uc2ue[2])
            ap = precompute.kernel_matrix(tgt, f.uep, kind) @ (X @ b)
            errs.append(np.linalg.norm(ap - exact) / np.linalg.norm(exact))
        assert errs[0] <= 2 * errs[1] + 1e-9, errs


@pytest.mark.parametrize("kind", [0, 1])
def test_highfreq_wedges_reach_eps(tmp_path, kind):
    accu, wmax = 1, 2
    _, hdp = _gen(tmp_path, kind, accu, wmax, ld=False)
    hd = formats.read_hd(hdp)
    ref = precompute.highfreq_levels(accu, kind, wmax, workers=1)
    P = precompute.accu_to_p(accu)
    rng = np.random.default_rng(1)
    for W in (1.0, 2.0):
        assert sorted(hd[W]) == sorted(ref[W])  # the same canonical wedges (aug3d_hghdata.m:42-45)
        for n, e in hd[W].items():
            r1, r2 = e.uep.shape[1], e.ucp.shape[1]
            assert [m.shape for m in e.uc2ue] == [(r1, r1), (r1, r2), (r2, r2)]
            f = ref[W][n]
            # skeleton ranks within 10% of the numpy restatement's
            assert abs(r1 - f.uep.shape[1]) <= 0.1 * f.uep.shape[1] + 2
            assert abs(r2 - f.ucp.shape[1]) <= 0.1 * f.ucp.shape[1] + 2
            ps = _children_sources(hd, W, n, P)
            den = rng.normal(size=ps.shape[1]) + 1j * rng.normal(size=ps.shape[1])
            err = _wedge_error(e, ps, _far_targets(rng, W, n), den, kind)
            assert err < 10 * EPS[accu], (W, n, err)
            # skeleton points are children's source points (uep) / far-field targets (ucp)
            assert set(map(tuple, e.uep.T)) <= set(map(tuple, ps.T))


def test_accu2_wedge_sample_reaches_eps(tmp_path):
    """ACCU 2 at widths 1 and 2, every wedge."""
    accu, kind = 2, 0
    _, hdp = _gen(tmp_path, kind, accu, 2, ld=False)
    hd = formats.read_hd(hdp)
    rng = np.random.default_rng(2)
    for W, lev in hd.items():
        for n, e in lev.items():
            ps = _children_sources(hd, W, n, 6)
            den = rng.normal(size=ps.shape[1]) + 1j * rng.normal(size=ps.shape[1])
            assert _wedge_error(e, ps, _far_targets(rng, W, n), den, kind) < 10 * EPS[accu]


def test_files_are_independent_of_thread_count(tmp_path):
    a = _gen(tmp_path, 0, 1, 2, threads=1, tag="1")
    b = _gen(tmp_path, 0, 1, 2, threads=4, tag="4")
    for p, q in zip(a, b):
        assert open(p, "rb").read() == open(q, "rb").read()


def test_files_pass_the_operator_check(tmp_path, lib):
    ldp, hdp = _gen(tmp_path, 1, 1, 2)
    nl, nh = C.c_int(), C.c_int()
    _lib.check(lib.ddfmm_operators_check(ldp.encode(), hdp.encode(), 1, C.byref(nl), C.byref(nh)))
    assert nl.value == 7 and nh.value == 3 + 10


def test_bad_arguments(tmp_path, lib):
    p = str(tmp_path / "x.bin").encode()
    assert lib.ddfmm_precompute_operators(2, 1, 1, 1, p, None, 0) == 1      # kernel
    assert lib.ddfmm_precompute_operators(0, 4, 1, 1, p, None, 0) == 1      # ACCU
    assert lib.ddfmm_precompute_operators(0, 1, 3, 1, p, None, 0) == 1      # wmax not a power of two
    assert lib.ddfmm_precompute_operators(0, 1, 1, 1, None, None, 0) == 1   # nothing to write
    bad = str(tmp_path / "no_such_dir" / "ld.bin").encode()
    assert lib.ddfmm_precompute_operators(0, 1, 1, 1, bad, None, 0) == 3    # DDFMM_ESETUP
    assert b"cannot write" in lib.ddfmm_last_error()


def test_reference_binary_runs_on_native_operators(tmp_path):
    """The reference's own eval (oracle/_ref) on a K=4 sphere with operator
    files from the C++ precompute reaches the accuracy of ACCU 1 against its
    own direct sum (Wave3d::check)."""
    import run_ref
    if not run_ref.available():
        pytest.skip("reference oracle not built (make -C oracle)")
    K, N = 4.0, 1500
    ldp, hdp = _gen(tmp_path, 0, 1, max(1, int(round(K / geometry.cells_for(K)))))
    pos = geometry.sphere_points(N, K)
    den = geometry.densities(N)
    out = run_ref.run(pos, den, K=K, accu=1, kernel=0, nc=geometry.cells_for(K), maxlevel=geometry.maxlevel_for(K),
                      ld_path=ldp, hd_path=hdp, chk=geometry.check_ids(N, 50), timeout=600)
    assert out["relerr"] < 1e-3, out["relerr"]
