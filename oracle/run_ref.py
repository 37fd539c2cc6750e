"""Run the reference binary (oracle/_ref/ref_eval, built by oracle/Makefile)
on a workload and read back its result.  Test infrastructure only: nothing
in the product imports this module.

The reference reads pos/den per rank from data/<name>_<rank>_<size> and the
shared files (operators, geomprtn, chk) from data/<name>
(src/parallel.cpp:33,81), so each run gets a scratch directory with a data/
folder holding exactly those files.
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_EVAL = os.path.join(HERE, "_ref", "ref_eval")


def available() -> bool:
    return os.access(REF_EVAL, os.X_OK)


def write_case(dirpath, pos, den, nc, chk, ld_path, hd_path):
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    from ddfmm_b200 import formats
    data = os.path.join(dirpath, "data")
    os.makedirs(data, exist_ok=True)
    formats.write_pos(os.path.join(data, "pos_0_1"), pos)
    formats.write_den(os.path.join(data, "den_0_1"), den)
    formats.write_geomprtn(os.path.join(data, "geomprtn"), nc)
    formats.write_chk(os.path.join(data, "chk"), chk)
    for src, name in ((ld_path, "ld.bin"), (hd_path, "hd.bin")):
        dst = os.path.join(data, name)
        try:
            os.symlink(os.path.abspath(src), dst)
        except OSError:
            shutil.copy(src, dst)


def run(pos, den, *, K, accu, kernel, nc, maxlevel, ld_path, hd_path, chk=None,
        ptsmax=100, npq=4, timeout=None, workdir=None):
    """Returns dict(val=complex array in id order, setup_s, eval_s, relerr)."""
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    from ddfmm_b200 import formats
    if not available():
        raise RuntimeError("reference oracle not built: run make -C oracle")
    tmp = workdir or tempfile.mkdtemp(prefix="ddfmm_ref_")
    try:
        chk_ids = np.asarray(chk if chk is not None else [0], dtype=np.int32)
        write_case(tmp, pos, den, nc, chk_ids, ld_path, hd_path)
        args = [REF_EVAL, "-posfile", "pos", "-denfile", "den", "-geomprtn", "geomprtn",
                "-valfile", "val", "-kernel", str(kernel),
                "-mlib3d_NPQ", str(npq), "-mlib3d_ldname", "ld.bin", "-mlib3d_hdname", "hd.bin",
                "-wave3d_ACCU", str(accu), "-wave3d_NPQ", str(npq), "-wave3d_K", repr(float(K)),
                "-wave3d_ctr", "0 0 0", "-wave3d_ptsmax", str(ptsmax),
                "-wave3d_maxlevel", str(maxlevel)]
        if chk is not None:
            args += ["-chkfile", "chk"]
        p = subprocess.run(args, cwd=tmp, capture_output=True, text=True, timeout=timeout)
        m = re.search(r"REF_EVAL setup_s=(\S+) eval_s=(\S+) n=(\d+) relerr=(\S+)", p.stdout)
        if p.returncode != 0 or not m:
            raise RuntimeError("reference run failed (rc=%d):\n%s\n%s" % (p.returncode, p.stdout[-2000:], p.stderr[-2000:]))
        keys, val, _ = formats.read_val(os.path.join(tmp, "data", "val_0_1"))
        if not np.array_equal(keys, np.arange(len(val))):
            raise RuntimeError("reference val keys are not 0..N-1")
        return dict(val=val, setup_s=float(m.group(1)), eval_s=float(m.group(2)),
                    relerr=float(m.group(4)), log=p.stdout + p.stderr)
    finally:
        if workdir is None:
            shutil.rmtree(tmp, ignore_errors=True)


def run_workload(w, chk=True, timeout=None, workdir=None):
    ld, hd = w.operators()
    return run(w.points(), w.densities(), K=w.K, accu=w.accu, kernel=w.kernel, nc=w.nc,
               maxlevel=w.maxlevel, ld_path=ld, hd_path=hd,
               chk=w.check_ids() if chk else None, ptsmax=w.ptsmax, npq=w.npq,
               timeout=timeout, workdir=workdir)
