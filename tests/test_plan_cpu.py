"""Host-only pieces of the launch plan (ddfmm_b200/csrc/plan.hpp: V-list sum
groups, M2L far pairs, M2M / E2 / E2^T / L2L column lists), checked without a
GPU by a C++ driver linked against the library."""
import os
import subprocess

import pytest

from ddfmm_b200 import geometry

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "ddfmm_b200")


@pytest.fixture(scope="module")
def plan_test(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("plan") / "plan_test")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(LIBDIR, "csrc"), "-o", out,
                    os.path.join(ROOT, "tests", "cpp", "plan_test.cpp"), os.path.join(LIBDIR, "libddfmm_b200.so"),
                    "-Wl,-rpath," + LIBDIR], check=True)
    return out


# Order-sensitive hashes of the V-list groups and the M2M / E2 / E2^T / L2L
# column lists, recorded from the first (sequential) implementation of both:
# the parallel construction must give the same problems and columns in the
# same order.
PLAN_HASHES = {("sphere", 8.0): "4e1721f80f4e06ca", ("sphere", 16.0): "e421a66932133880",
               ("ellipsoid", 8.0): "f481e0411765727f", ("cluster", 4.0): "4950994f63afc9ab"}


@pytest.mark.parametrize("geom,K,N,ptsmax", [("sphere", 8.0, 5027, 100), ("sphere", 16.0, 20106, 100),
                                             ("ellipsoid", 8.0, 3000, 100), ("cluster", 4.0, 1500, 8)])
def test_plan_pieces_cover_every_pair_once(plan_test, tmp_path, geom, K, N, ptsmax):
    pos = {"sphere": geometry.sphere_points, "ellipsoid": geometry.ellipsoid_points,
           "cluster": geometry.cluster_points}[geom](N, K)
    path = tmp_path / "pos.bin"
    pos.astype("<f8").tofile(path)
    r = subprocess.run([plan_test, str(path), str(len(pos)), repr(K), str(geometry.cells_for(K)),
                        str(geometry.maxlevel_for(K)), str(ptsmax)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    words = r.stdout.split()
    assert words[0] == "ok" and int(words[2]) > 0, r.stdout
    assert words[words.index("hash") + 1] == PLAN_HASHES[(geom, K)], r.stdout
    if K >= 8:  # trees with high-frequency levels
        assert int(words[6]) > 0 and int(words[8]) > 0, r.stdout
