"""Golden fixtures: outputs of the reference binary on small seeded cases.

Each ``<case>.npz`` (written by make_golden.py from the reference's own
Wave3d::eval, built by oracle/Makefile) holds the inputs, the reference's
result ``val`` and its ``relerr``, and the operator factors the reference
ran with.  The pseudo-inverse / skeleton factors (LF uc2ue, HF uep/ucp/E1-3)
are stored bit-exactly because they are ill-conditioned and machine
dependent; the FFT'd LF translation tensors are a well-conditioned function
of the geometry and are regenerated with ddfmm_b200.precompute.
"""
from __future__ import annotations

import json
import os

import numpy as np

from ddfmm_b200 import formats, precompute

HERE = os.path.dirname(os.path.abspath(__file__))


def case_names():
    return sorted(f[:-4] for f in os.listdir(HERE) if f.endswith(".npz"))


def pack(path, params, pos, den, val, chk, relerr, ld, hd, ld_widths, counts):
    arrs = dict(pos=pos, den=den, val=val, chk=chk, relerr=np.array(relerr),
                params=np.array(json.dumps(params)), **counts)
    for W in ld_widths:
        e = ld[W]
        tag = "ld_%r" % W
        arrs[tag + "_uep"] = e.uep
        arrs[tag + "_ucp"] = e.ucp
        for i, m in enumerate(e.uc2ue):
            arrs[tag + "_uc2ue%d" % i] = m
    for W, lev in hd.items():
        for key, e in lev.items():
            tag = "hd_%r_%d_%d_%d" % ((W,) + tuple(key))
            arrs[tag + "_uep"] = e.uep
            arrs[tag + "_ucp"] = e.ucp
            for i, m in enumerate(e.uc2ue):
                arrs[tag + "_E%d" % (i + 1)] = m
    np.savez_compressed(path, **arrs)


class Case:
    def __init__(self, name):
        z = np.load(os.path.join(HERE, name + ".npz"))
        self.name = name
        self.params = json.loads(str(z["params"]))
        self.pos = z["pos"]
        self.den = z["den"]
        self.val = z["val"]
        self.chk = z["chk"]
        self.relerr = float(z["relerr"])
        self.ref_total_boxes = int(z["ref_total_boxes"])
        self.ref_deleted = int(z["ref_deleted"])
        self.ref_boxes = {int(a): int(b) for a, b in z["ref_boxes"]}
        self.ref_dirs = {int(a): int(b) for a, b in z["ref_dirs"]}
        self._z = z

    def write_operators(self, dirpath):
        """Reconstitute ld/hd files in the reference format under dirpath."""
        z = self._z
        p = self.params
        P = precompute.accu_to_p(p["accu"])
        ld = {}
        for k in z.files:
            if k.startswith("ld_") and k.endswith("_uep"):
                W = float(k[3:-4])
                tag = k[:-4]
                fresh = precompute.lowfreq_entry(p["accu"], W, p["kernel"])
                ld[W] = formats.LowFreqEntry(z[tag + "_uep"], z[tag + "_ucp"],
                                             [z[tag + "_uc2ue%d" % i] for i in range(3)], fresh.ue2dc)
                assert fresh.uep.shape[1] == P ** 3 - (P - 2) ** 3
        hd = {}
        for k in z.files:
            if k.startswith("hd_") and k.endswith("_uep"):
                parts = k.split("_")
                W = float(parts[1])
                key = (int(parts[2]), int(parts[3]), int(parts[4]))
                tag = k[:-4]
                hd.setdefault(W, {})[key] = formats.HighFreqEntry(
                    z[tag + "_uep"], z[tag + "_ucp"], [z[tag + "_E%d" % i] for i in (1, 2, 3)])
        ldp = os.path.join(dirpath, "ld.bin")
        hdp = os.path.join(dirpath, "hd.bin")
        formats.write_ld(ldp, ld)
        formats.write_hd(hdp, hd)
        return ldp, hdp
