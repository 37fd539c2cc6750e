"""Reference binary formats (include/serialize.hpp) and the precompute."""
import os

import numpy as np

import fixtures
from ddfmm_b200 import formats, geometry, precompute


def test_pos_den_roundtrip(tmp_path):
    pos = geometry.sphere_points(100, 4.0)
    den = geometry.densities(100)
    formats.write_pos(tmp_path / "pos", pos)
    formats.write_den(tmp_path / "den", den)
    k, p, owner = formats.read_pos(tmp_path / "pos")
    assert np.array_equal(k, np.arange(100)) and np.array_equal(p, pos) and list(owner) == [0, 100]
    k, v, owner = formats.read_val(tmp_path / "den")
    assert np.array_equal(v, den)
    # int count + (int key, 3 doubles) records + owner vector
    assert os.path.getsize(tmp_path / "pos") == 4 + 100 * 28 + 4 + 8


def test_operator_files_roundtrip(tmp_path):
    c = fixtures.Case("sphere_k4_n1500_p6_helm")
    ldp, hdp = c.write_operators(str(tmp_path))
    ld = formats.read_ld(ldp)
    hd = formats.read_hd(hdp)
    assert set(ld) == {0.5}
    e = ld[0.5]
    assert e.uep.shape == (3, 152) and len(e.ue2dc) == 316
    assert all(t.shape == (12, 12, 12) for t in e.ue2dc.values())
    for lev in hd.values():
        for key, h in lev.items():
            r1, r2 = h.uep.shape[1], h.ucp.shape[1]
            assert [m.shape for m in h.uc2ue] == [(r1, r1), (r1, r2), (r2, r2)]


def test_lowfreq_surfaces_follow_matlab_grid():
    e = precompute.lowfreq_entry(1, 0.5, 0)
    assert e.uep.shape == (3, 56)
    assert np.isclose(np.abs(e.uep).max(), 0.25) and np.isclose(np.abs(e.ucp).max(), 0.75)
    # pseudo-inverse factors reproduce K(ucp, uep)^+
    M = precompute.kernel_matrix(e.ucp, e.uep, 0)
    pinv = e.uc2ue[0] @ (e.uc2ue[1][:, 0][:, None] * e.uc2ue[2])
    assert np.linalg.norm(M @ pinv @ M - M) / np.linalg.norm(M) < 1e-8


def test_highfreq_factors_are_low_rank_of_far_field():
    """E1 E2 E3 applied to a check potential reproduces the far field of a
    source inside the child boxes (aug3d_hghdata.m:238)."""
    hd = precompute.highfreq_levels(1, 0, 1, workers=1)
    (n, h), = [(k, v) for k, v in hd[1.0].items() if k == (1, 3, 4)]
    rng = np.random.default_rng(1)
    src = rng.uniform(-0.45, 0.45, (3, 20))
    q = rng.standard_normal(20) + 1j * rng.standard_normal(20)
    upchk = precompute.kernel_matrix(h.ucp, src, 0) @ q
    E1, E2, E3 = h.uc2ue
    ued = E1 @ (E2 @ (E3 @ upchk))
    # far target in the wedge (direction ~ (1,3,4)/C)
    d = np.array([1, 3, 4.0]) * np.tan(np.pi / 16) / 1.0
    trg = (np.array([np.tan(1 / 4 * np.pi / 4), np.tan(3 / 4 * np.pi / 4), 1.0]) * 5.0)[:, None]
    exact = precompute.kernel_matrix(trg, src, 0) @ q
    approx = precompute.kernel_matrix(trg, h.uep, 0) @ ued
    assert abs(exact - approx).max() / abs(exact).max() < 1e-3
