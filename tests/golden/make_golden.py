"""Regenerate the golden fixtures by running the reference binary.

Needs oracle/_ref/ref_eval (``make -C oracle``, built from the reference's
sources).  For each case: generate the inputs and operator files, run the
reference's Wave3d::setup + eval + check, and store inputs, result, relerr
and the exact operator factors in tests/golden/<case>.npz.

    python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

import fixtures  # noqa: E402
import run_ref  # noqa: E402
from ddfmm_b200 import formats  # noqa: E402
from ddfmm_b200 import workloads as wl  # noqa: E402

CASES = {
    # the reference's CPU-runnable configuration: sphere K=8, N=5000, P=4
    "sphere_k8_n5000_p4_helm": wl.sphere(8, 5000, accu=1),
    "sphere_k4_n1500_p4_expr": wl.sphere(4, 1500, accu=1, kernel=1),
    "sphere_k4_n1500_p6_helm": wl.sphere(4, 1500, accu=2),
    "cluster_k4_n1500_p4_helm_m8": wl.cluster(4, 1500, accu=1, ptsmax=8),
    "ellipsoid_k8_n3000_p4_helm": wl.ellipsoid(8, 3000, accu=1),
    "sphere_k16_n4000_p4_helm": wl.sphere(16, 4000, accu=1),
    "sphere_k4_n1500_p8_helm": wl.sphere(4, 1500, accu=3),
}


def lf_widths(pos, K, ptsmax, maxlevel, nc):
    """Widths of the low-frequency boxes the tree will hold, following the
    split rule of src/wave3d_setup.cpp:156-157 (boxes at or above the unit
    level always split when non-empty; below it when > ptsmax points)."""
    unit = int(round(math.log2(K)))
    lvl = int(round(math.log2(nc)))
    u = (pos + K / 2) / K
    active = np.ones(len(pos), dtype=bool)
    widths = set()
    while active.any():
        idx = np.floor(u[active] * (1 << lvl)).astype(np.int64)
        key = (idx[:, 0] << 40) | (idx[:, 1] << 20) | idx[:, 2]
        uk, inv, cnt = np.unique(key, return_inverse=True, return_counts=True)
        W = K / (1 << lvl)
        if W < 1 - 1e-12:
            widths.add(W)
        split = (lvl <= unit) | ((cnt > ptsmax) & (lvl < maxlevel - 1))
        keep = split[inv]
        sub = np.nonzero(active)[0]
        active[sub[~keep]] = False
        lvl += 1
    return sorted(widths)


def parse_counts(log):
    """The reference's own tree printout (src/wave3d_eval.cpp:345-372):
    total / deleted boxes, boxes with points per level, and the summed
    directional interaction-list sizes per level."""
    import re
    m = re.search(r"Deleting (\d+) out of (\d+) total boxes", log)
    boxes = [(int(a), int(b)) for a, b in re.findall(r"boxes: \((\d+), (\d+)\)", log)]
    dirs = [(int(a), int(b)) for a, b in re.findall(r"dirs: \((\d+), (\d+)\)", log)]
    return dict(ref_deleted=int(m.group(1)), ref_total_boxes=int(m.group(2)),
                ref_boxes=np.array(boxes, dtype=np.int64).reshape(-1, 2),
                ref_dirs=np.array(dirs, dtype=np.int64).reshape(-1, 2))


def make(name, w):
    ld_path, hd_path = w.operators()
    r = run_ref.run_workload(w, chk=True)
    pos, den = w.points(), w.densities()
    ld = formats.read_ld(ld_path)
    # only the high-frequency widths this tree uses (the file may hold wider ones)
    hd = {W: e for W, e in formats.read_hd(hd_path).items() if W <= w.wmax}
    widths = lf_widths(pos, w.K, w.ptsmax, w.maxlevel, w.nc)
    params = dict(K=w.K, accu=w.accu, kernel=w.kernel, ptsmax=w.ptsmax, maxlevel=w.maxlevel, nc=w.nc,
                  npq=w.npq, workload=w.name, ref_eval_s=r["eval_s"])
    fixtures.pack(os.path.join(HERE, name + ".npz"), params, pos, den, r["val"], w.check_ids(),
                  r["relerr"], ld, hd, widths, parse_counts(r["log"]))
    print("%-32s N=%-6d eval %.2fs relerr %.3e  LF widths %s" % (name, w.N, r["eval_s"], r["relerr"], widths))


if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES)
    for n in names:
        make(n, CASES[n])
