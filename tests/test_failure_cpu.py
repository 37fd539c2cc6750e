"""Failure paths that need no GPU: bad operator files and out-of-range options.

The reference throws `new std::exception()` from SAFE_FUNC_EVAL / CHECK_TRUE
(include/commoninc.hpp:52-53) when Mlib3d::setup cannot read its files
(src/mlib3d.cpp:70-103, deserialize in include/serialize.hpp) and when
Wave3d::setup meets an option it cannot use (src/wave3d.cpp:145-158); the C
ABI returns DDFMM_ESETUP (3) and DDFMM_EINVAL (1) in those places, and the
Python mirror raises DDFMMError with that code."""
import ctypes as C
import os

import numpy as np
import pytest

import fixtures
from ddfmm_b200 import _lib, formats, wave3d

EINVAL, ESETUP = 1, 3


@pytest.fixture(scope="module")
def ops(tmp_path_factory):
    """Valid ld / hd files of the K=8, ACCU 1 reference fixture."""
    d = tmp_path_factory.mktemp("ops")
    return fixtures.Case("sphere_k8_n5000_p4_helm").write_operators(str(d))


def _check(lib, ld, hd, accu=1):
    nl, nh = C.c_int(), C.c_int()
    rc = lib.ddfmm_operators_check(ld.encode(), hd.encode(), accu, C.byref(nl), C.byref(nh))
    return rc, lib.ddfmm_last_error().decode(), nl.value, nh.value


def test_valid_files_pass(lib, ops):
    rc, msg, nl, nh = _check(lib, *ops)
    assert rc == 0, msg
    assert nl >= 1 and nh > 0


def test_missing_file(lib, ops, tmp_path):
    rc, msg, _, _ = _check(lib, str(tmp_path / "nope.bin"), ops[1])
    assert rc == ESETUP and "cannot open" in msg


@pytest.mark.parametrize("which", [0, 1])
@pytest.mark.parametrize("keep", [0.0, 0.5, 0.999])
def test_truncated_file(lib, ops, tmp_path, which, keep):
    src = ops[which]
    raw = open(src, "rb").read()
    cut = tmp_path / "cut.bin"
    cut.write_bytes(raw[:int(len(raw) * keep)])
    paths = list(ops)
    paths[which] = str(cut)
    rc, msg, _, _ = _check(lib, *paths)
    assert rc == ESETUP, msg
    assert "truncated" in msg or "bad dimension" in msg


@pytest.mark.parametrize("which", [0, 1])
def test_trailing_bytes(lib, ops, tmp_path, which):
    raw = open(ops[which], "rb").read()
    longer = tmp_path / "long.bin"
    longer.write_bytes(raw + b"\0" * 8)
    paths = list(ops)
    paths[which] = str(longer)
    rc, msg, _, _ = _check(lib, *paths)
    assert rc == ESETUP and "trailing" in msg


def test_files_of_another_accuracy_level(lib, ops):
    """ACCU 1 files (P = 4: 56 surface points, 8^3 tensors) for an ACCU 2 run."""
    rc, msg, _, _ = _check(lib, *ops, accu=2)
    assert rc == ESETUP and "ACCU" in msg


def test_inconsistent_low_frequency_factors(lib, ops, tmp_path):
    ld = formats.read_ld(ops[0])
    W = sorted(ld)[0]
    e = ld[W]
    e.uc2ue[0] = e.uc2ue[0][:, :-1]  # v loses a column: r no longer matches 1/sigma and U^H
    bad = tmp_path / "ld_bad.bin"
    formats.write_ld(str(bad), ld)
    rc, msg, _, _ = _check(lib, str(bad), ops[1])
    assert rc == ESETUP and "uc2ue" in msg


def test_inconsistent_high_frequency_factors(lib, ops, tmp_path):
    hd = formats.read_hd(ops[1])
    W = sorted(hd)[0]
    key = sorted(hd[W])[0]
    e = hd[W][key]
    e.uc2ue[1] = e.uc2ue[1][:-1, :]  # E2 loses a row: no longer r1 x r2
    bad = tmp_path / "hd_bad.bin"
    formats.write_hd(str(bad), hd)
    rc, msg, _, _ = _check(lib, ops[0], str(bad))
    assert rc == ESETUP and "E1/E2/E3" in msg


def test_operator_check_arguments(lib, ops):
    assert lib.ddfmm_operators_check(None, ops[1].encode(), 1, None, None) == EINVAL
    assert lib.ddfmm_operators_check(ops[0].encode(), ops[1].encode(), 4, None, None) == EINVAL


@pytest.mark.parametrize("opt,value,word", [("ACCU", "0", b"ACCU"), ("ACCU", "4", b"ACCU"), ("NPQ", "3", b"NPQ"),
                                            ("K", "0.5", b"K must"), ("ptsmax", "0", b"ptsmax"),
                                            ("maxlevel", "0", b"maxlevel")])
def test_options_out_of_range(lib, ops, opt, value, word):
    """Wave3d::setup options outside what the method supports: rejected before
    any device work, with the option named."""
    c = fixtures.Case("sphere_k8_n5000_p4_helm")
    mlib = wave3d.Mlib3d()
    mlib.setup({"-mlib3d_ldname": ops[0], "-mlib3d_hdname": ops[1]})
    w = wave3d.Wave3d()
    w.posptr = c.pos
    w.kernel = 0
    w.mlibptr = mlib
    w.geomprtn = 8
    opts = {"-wave3d_ACCU": "1", "-wave3d_NPQ": "4", "-wave3d_K": "8", "-wave3d_ptsmax": "100",
            "-wave3d_maxlevel": "10"}
    opts["-wave3d_" + opt] = value
    with pytest.raises(_lib.DDFMMError) as e:
        w.setup(opts)
    assert e.value.code == EINVAL
    assert word.decode() in str(e.value)


def test_partition_must_fit_the_box(lib, ops):
    """geomprtn cells narrower than one wavelength (src/wave3d_setup.cpp:307)."""
    pos = np.zeros((4, 3))
    out = C.c_void_p()
    rc = lib.ddfmm_session_create(pos.ctypes.data_as(C.POINTER(C.c_double)), 4, 0, 1, 4, 8.0, None, 100, 8, 16,
                                  ops[0].encode(), ops[1].encode(), 0, C.byref(out))
    assert rc == EINVAL and b"ncell" in lib.ddfmm_last_error()


def test_mlib_setup_requires_both_files(tmp_path):
    m = wave3d.Mlib3d()
    with pytest.raises(_lib.DDFMMError) as e:
        m.setup({"-mlib3d_ldname": str(tmp_path / "a"), "-mlib3d_hdname": str(tmp_path / "b")})
    assert e.value.code == ESETUP
    assert not os.path.exists(tmp_path / "a")
