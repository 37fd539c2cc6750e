"""Full-size golden fixture: the reference's matvec on the K=64, P=6 sphere.

Runs the reference binary (oracle/_ref/ref_eval, built by ``make -C oracle``)
once on the 321,699-point sphere with the operator files of
ddfmm_b200/_operators (about 40 minutes on one core), and stores a compact
summary of its output in tests/golden/full/sphere_k64_p6_helm.npz:

* ``ids`` / ``val``: the reference's values at 4096 seeded point ids;
* ``wsum``: three seeded random complex weightings of the whole output
  vector (sum_i w_i val_i), ``norm``: its l2 norm;
* ``ld_sha256`` / ``hd_sha256``: the operator files it ran with (the
  skeleton factors are machine dependent, so the comparison is only
  meaningful with the same files);
* ``relerr`` / ``eval_s``: what the reference's own check printed.

    python tests/golden/make_full.py [--val saved.npy --eval-s S --relerr R]

``--val`` reuses the output vector of an identical earlier run of
``oracle/run_ref.run_workload(workloads.LARGE, chk=True)``.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from ddfmm_b200 import workloads as wl  # noqa: E402

OUT = os.path.join(HERE, "full", "sphere_k64_p6_helm.npz")
NSAMPLE = 4096


def sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 24), b""):
            h.update(chunk)
    return h.hexdigest()


def weights(n):
    """The three seeded complex weight vectors of the checksums."""
    g = np.random.default_rng(20261203)
    return g.standard_normal((3, n)) + 1j * g.standard_normal((3, n))


def sample_ids(n):
    return np.sort(np.random.default_rng(7).choice(n, NSAMPLE, replace=False))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--val")
    ap.add_argument("--eval-s", type=float)
    ap.add_argument("--relerr", type=float)
    a = ap.parse_args()
    w = wl.LARGE
    ld, hd = w.operators()
    if a.val:
        val, eval_s, relerr = np.load(a.val), a.eval_s, a.relerr
    else:
        import run_ref
        r = run_ref.run_workload(w, chk=True)
        val, eval_s, relerr = r["val"], r["eval_s"], r["relerr"]
    assert val.shape == (w.N,)
    ids = sample_ids(w.N)
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    np.savez_compressed(OUT, ids=ids, val=val[ids], wsum=weights(w.N) @ val, norm=np.linalg.norm(val),
                        relerr=np.array(relerr), eval_s=np.array(eval_s), workload=np.array(w.name),
                        ld_sha256=np.array(sha256(ld)), hd_sha256=np.array(sha256(hd)))
    print("wrote", OUT, "eval_s", eval_s, "relerr", relerr)


if __name__ == "__main__":
    main()
