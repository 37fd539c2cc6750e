"""Host octree and interaction lists against the reference's own printout.

The reference's Wave3d::eval prints the total and empty box counts, the
boxes with points per level and the summed directional far-list sizes per
level (src/wave3d_eval.cpp:345-372); the golden fixtures recorded them from
the reference binary.  The native library's host-only tree builder must
reproduce every number (no GPU needed)."""
import numpy as np
import pytest

import fixtures
from ddfmm_b200 import _lib


@pytest.mark.parametrize("name", fixtures.case_names())
def test_tree_counts_match_reference(name):
    c = fixtures.Case(name)
    p = c.params
    st = _lib.tree_stats(c.pos, p["K"], p["ptsmax"], p["maxlevel"], p["nc"], p["npq"])
    assert st["total_boxes"] == c.ref_total_boxes
    assert st["empty_boxes"] == c.ref_deleted
    assert {L["level"]: L["boxes"] for L in st["levels"]} == c.ref_boxes
    assert {L["level"]: L["far_pairs"] for L in st["levels"]} == c.ref_dirs


def test_tree_adaptive_case_has_all_list_kinds():
    c = fixtures.Case("cluster_k4_n1500_p4_helm_m8")
    p = c.params
    st = _lib.tree_stats(c.pos, p["K"], p["ptsmax"], p["maxlevel"], p["nc"], p["npq"])
    tot = {k: sum(L[k] for L in st["levels"]) for k in ("u_pairs", "v_pairs", "w_pairs", "x_pairs")}
    assert all(v > 0 for v in tot.values()), tot
    # non-leaf low-frequency boxes exist (LF M2M / L2L are exercised)
    assert any(L["width"] < 1 and L["boxes"] > L["leaves"] for L in st["levels"])


def test_tree_lists_independent_of_host_threads(monkeypatch):
    """The lists are built level by level with the boxes of a level spread over
    host threads; every count must be the same on one thread and on several
    (a K=16 sphere: levels large enough to be split)."""
    from ddfmm_b200 import workloads as wl
    w = wl.sphere(16, None, accu=2)
    out = []
    for n in ("1", "4"):
        monkeypatch.setenv("DDFMM_HOST_THREADS", n)
        out.append(_lib.tree_stats(w.points(), 16, 100, w.maxlevel, 8, 4))
    assert out[0] == out[1]
    assert sum(L["far_pairs"] for L in out[0]["levels"]) > 0 and sum(L["v_pairs"] for L in out[0]["levels"]) > 0


def test_tree_rejects_point_outside_root_box():
    pos = np.array([[0.0, 0.0, 0.0], [2.5, 0.0, 0.0]])
    with pytest.raises(_lib.DDFMMError) as e:
        _lib.tree_stats(pos, 4.0, 100, 8, 4)
    assert "outside" in str(e.value)


def test_tree_rejects_bad_cell_count():
    with pytest.raises(_lib.DDFMMError):
        _lib.tree_stats(np.zeros((4, 3)), 4.0, 100, 8, 3)
