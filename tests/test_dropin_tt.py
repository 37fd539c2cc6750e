"""The reference's own driver, unmodified, on the GPU path.

oracle/_ref/tt_dropin is the reference's src/tt.cpp compiled against the
drop-in include/ddfmm_ref/wave3d.hpp (put ahead of the reference's headers
on the include path) and linked with libddfmm_b200.so in place of the
reference's wave3d*.cpp; ParVec<int, cpx, PtPrtn>, Mlib3d, Kernel3d and the
file I/O (src/parallel.cpp) are the reference's.  Built by oracle/Makefile.

Run like the reference (src/tt.cpp:43-198): files under data/, options as
"-key value" pairs; it writes data/val_0_1 and prints the RESULT block with
the relative error Ea of the FMM against the FP64 direct sum at the check ids.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import fixtures
import run_ref
from ddfmm_b200 import formats

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TT = os.path.join(ROOT, "oracle", "_ref", "tt_dropin")
TOL = 1e-10


def _need_binary():
    if not os.access(TT, os.X_OK):
        pytest.skip("oracle/_ref/tt_dropin is not built (make -C oracle with the reference sources)")


def _run(c, tmp_path, timeout=600):
    p = c.params
    ldp, hdp = c.write_operators(str(tmp_path / "ops"))
    run_ref.write_case(str(tmp_path), c.pos, c.den, p["nc"], np.asarray(c.chk, dtype=np.int32), ldp, hdp)
    args = [TT, "-posfile", "pos", "-denfile", "den", "-geomprtn", "geomprtn", "-valfile", "val",
            "-chkfile", "chk", "-kernel", str(p["kernel"]), "-mlib3d_NPQ", str(p["npq"]),
            "-mlib3d_ldname", "ld.bin", "-mlib3d_hdname", "hd.bin", "-wave3d_ACCU", str(p["accu"]),
            "-wave3d_NPQ", str(p["npq"]), "-wave3d_K", repr(float(p["K"])), "-wave3d_ctr", "0 0 0",
            "-wave3d_ptsmax", str(p["ptsmax"]), "-wave3d_maxlevel", str(p["maxlevel"])]
    return subprocess.run(args, cwd=str(tmp_path), capture_output=True, text=True, timeout=timeout)


def test_dropin_without_gpu_throws_like_the_reference(tmp_path):
    """No device: Wave3d::setup reports the library's reason and throws, as
    the reference's SAFE_FUNC_EVAL does; tt (built with RELEASE) then ends
    abnormally before writing any value."""
    _need_binary()
    pytest.importorskip("torch")
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    os.makedirs(tmp_path / "ops")
    r = _run(fixtures.Case("sphere_k4_n1500_p4_expr"), tmp_path)
    assert r.returncode != 0
    assert "Wave3d: no CUDA device" in r.stderr
    assert "Done reading mlib" in r.stderr  # the reference's Mlib3d read both operator files first
    assert not os.path.exists(tmp_path / "data" / "val_0_1")


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sphere_k8_n5000_p4_helm", "cluster_k4_n1500_p4_helm_m8"])
def test_reference_driver_on_the_gpu_matches_the_reference(name, tmp_path):
    _need_binary()
    c = fixtures.Case(name)
    os.makedirs(tmp_path / "ops")
    r = _run(c, tmp_path)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    keys, val, _ = formats.read_val(str(tmp_path / "data" / "val_0_1"))
    assert np.array_equal(keys, np.arange(len(c.den)))
    rel = np.linalg.norm(val - c.val) / np.linalg.norm(c.val)
    print("tt_dropin %s: rel l2 vs reference %.3e" % (name, rel))
    assert rel <= TOL, rel
    m = re.search(r"^Ea\s+(\S+)", r.stdout, re.M)
    assert m, r.stdout
    ea = float(m.group(1))
    assert abs(ea - c.relerr) <= 2e-6 * c.relerr + 1e-12, (ea, c.relerr)
