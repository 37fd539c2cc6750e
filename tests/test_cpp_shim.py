"""The header-only C++ drop-in (include/ddfmm_wave3d.hpp) used the way the
reference's tt driver uses Wave3d (src/tt.cpp:103-185)."""
import os
import subprocess

import numpy as np
import pytest

import fixtures

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "ddfmm_b200")


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("shim") / "shim_main")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-o", out,
                    os.path.join(ROOT, "tests", "cpp", "shim_main.cpp"), os.path.join(LIBDIR, "libddfmm_b200.so"),
                    "-Wl,-rpath," + LIBDIR], check=True)
    return out


def test_shim_compiles_and_throws_like_the_reference(shim):
    pytest.importorskip("torch")
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    r = subprocess.run([shim, "--no-gpu"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "setup threw" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sphere_k8_n5000_p4_helm", "cluster_k4_n1500_p4_helm_m8"])
def test_shim_matches_reference(shim, name, tmp_path):
    c = fixtures.Case(name)
    ldp, hdp = c.write_operators(str(tmp_path))
    p = c.params
    c.pos.astype("<f8").tofile(tmp_path / "pos.bin")
    c.den.astype("<c16").tofile(tmp_path / "den.bin")
    c.chk.astype("<f8").tofile(tmp_path / "chk.bin")
    with open(tmp_path / "opts.txt", "w") as f:
        for k, v in {"-mlib3d_ldname": ldp, "-mlib3d_hdname": hdp, "-kernel": p["kernel"], "-geomprtn": p["nc"],
                     "-wave3d_ACCU": p["accu"], "-wave3d_NPQ": p["npq"], "-wave3d_K": p["K"],
                     "-wave3d_ptsmax": p["ptsmax"], "-wave3d_maxlevel": p["maxlevel"]}.items():
            f.write("%s %s\n" % (k, v))
    r = subprocess.run([shim, str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    val = np.fromfile(tmp_path / "val.bin", dtype="<c16")
    rel = np.linalg.norm(val - c.val) / np.linalg.norm(c.val)
    assert rel <= 1e-10, rel
    relerr = float(r.stdout.split()[-1])
    assert abs(relerr - c.relerr) <= 1e-6 * c.relerr
