"""ctypes binding of libddfmm_b200.so (include/ddfmm.h).

There is no fallback: if the shared library is missing or cannot be loaded
this module raises, and every eval runs the CUDA kernels of that library.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libddfmm_b200.so")

EXPORTS = (
    "ddfmm_session_create", "ddfmm_eval", "ddfmm_eval_device", "ddfmm_direct",
    "ddfmm_session_stats", "ddfmm_session_destroy", "ddfmm_last_error", "ddfmm_tree_stats",
    "ddfmm_profile_enable", "ddfmm_profile_read", "ddfmm_eval_device_noalloc",
    "ddfmm_session_create_ex", "ddfmm_eval_c64", "ddfmm_eval_device_c64",
    "ddfmm_batch_create", "ddfmm_batch_eval_c64", "ddfmm_batch_eval_device_c64", "ddfmm_batch_launches",
    "ddfmm_batch_destroy", "ddfmm_server_create", "ddfmm_server_add_session", "ddfmm_server_session_state",
    "ddfmm_server_remove_session", "ddfmm_server_submit", "ddfmm_server_wait", "ddfmm_server_poll",
    "ddfmm_server_get_stats", "ddfmm_server_destroy", "ddfmm_operators_check", "ddfmm_session_test_gemm_stall",
    "ddfmm_precompute_operators",
)
PLAIN_FP64, MIXED, MIXED_MMA_SYNC = 0, 1, 2


class ddfmm_server_stats(C.Structure):
    _fields_ = [("requests", C.c_longlong), ("ticks", C.c_longlong), ("mean_batch", C.c_double),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double), ("busy_s", C.c_double),
                ("used_bytes", C.c_longlong), ("admitted", C.c_int), ("waiting", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ddfmm_stats(C.Structure):
    _fields_ = [
        ("n_points", C.c_int), ("n_boxes", C.c_int), ("n_leaves", C.c_int), ("n_lf_boxes", C.c_int),
        ("u_pairs", C.c_longlong), ("u_interactions", C.c_longlong), ("v_pairs", C.c_longlong),
        ("w_pairs", C.c_longlong), ("x_pairs", C.c_longlong),
        ("hf_up_nodes", C.c_longlong), ("hf_down_nodes", C.c_longlong), ("hf_far_pairs", C.c_longlong),
        ("m2l_matrices", C.c_longlong), ("gemm_launches", C.c_longlong), ("kernel_launches", C.c_longlong),
        ("flops_gemm", C.c_double), ("fft_spectra_bytes", C.c_longlong), ("setup_seconds", C.c_double),
        ("device_bytes", C.c_longlong), ("ops_seconds", C.c_double), ("tree_seconds", C.c_double),
        ("plan_seconds", C.c_double), ("tune_seconds", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ddfmm_tree_level(C.Structure):
    _fields_ = [("level", C.c_int), ("width", C.c_double), ("boxes", C.c_int), ("leaves", C.c_int),
                ("far_pairs", C.c_longlong), ("out_dirs", C.c_longlong), ("inc_dirs", C.c_longlong),
                ("u_pairs", C.c_longlong), ("v_pairs", C.c_longlong), ("w_pairs", C.c_longlong),
                ("x_pairs", C.c_longlong)]


class ddfmm_profile_entry(C.Structure):
    _fields_ = [("label", C.c_char * 32), ("kernel", C.c_char * 32), ("launches", C.c_int), ("ms", C.c_double),
                ("flops", C.c_double), ("bytes", C.c_double)]


_lib = None


def load():
    """Load the library once; raise if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libddfmm_b200.so is not built (run python -m ddfmm_b200.build or __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    dp = C.POINTER(C.c_double)
    lib.ddfmm_session_create.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, dp, C.c_int,
                                         C.c_int, C.c_int, C.c_char_p, C.c_char_p, C.c_int,
                                         C.POINTER(C.c_void_p)]
    lib.ddfmm_session_create.restype = C.c_int
    lib.ddfmm_session_create_ex.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, dp, C.c_int,
                                            C.c_int, C.c_int, C.c_char_p, C.c_char_p, C.c_int, C.c_int,
                                            C.POINTER(C.c_void_p)]
    lib.ddfmm_session_create_ex.restype = C.c_int
    fp = C.POINTER(C.c_float)
    lib.ddfmm_eval_c64.argtypes = [C.c_void_p, fp, fp]
    lib.ddfmm_eval_c64.restype = C.c_int
    lib.ddfmm_eval_device_c64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ddfmm_eval_device_c64.restype = C.c_int
    lib.ddfmm_eval.argtypes = [C.c_void_p, dp, dp]
    lib.ddfmm_eval.restype = C.c_int
    lib.ddfmm_eval_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ddfmm_eval_device.restype = C.c_int
    lib.ddfmm_eval_device_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ddfmm_eval_device_noalloc.restype = C.c_int
    lib.ddfmm_direct.argtypes = [C.c_void_p, dp, C.POINTER(C.c_int), C.c_int, dp]
    lib.ddfmm_direct.restype = C.c_int
    lib.ddfmm_session_stats.argtypes = [C.c_void_p, C.POINTER(ddfmm_stats)]
    lib.ddfmm_session_stats.restype = C.c_int
    lib.ddfmm_session_destroy.argtypes = [C.c_void_p]
    lib.ddfmm_session_destroy.restype = C.c_int
    lib.ddfmm_tree_stats.argtypes = [dp, C.c_int, C.c_double, dp, C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(ddfmm_tree_level)]
    lib.ddfmm_tree_stats.restype = C.c_int
    lib.ddfmm_profile_enable.argtypes = [C.c_void_p, C.c_int]
    lib.ddfmm_profile_enable.restype = C.c_int
    lib.ddfmm_profile_read.argtypes = [C.c_void_p, C.POINTER(ddfmm_profile_entry), C.c_int, C.POINTER(C.c_int),
                                       C.c_int]
    lib.ddfmm_profile_read.restype = C.c_int
    lib.ddfmm_last_error.argtypes = []
    lib.ddfmm_last_error.restype = C.c_char_p
    ip = C.POINTER(C.c_int)
    lib.ddfmm_operators_check.argtypes = [C.c_char_p, C.c_char_p, C.c_int, ip, ip]
    lib.ddfmm_operators_check.restype = C.c_int
    lib.ddfmm_precompute_operators.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_char_p, C.c_int]
    lib.ddfmm_precompute_operators.restype = C.c_int
    lib.ddfmm_session_test_gemm_stall.argtypes = [C.c_void_p, C.c_double]
    lib.ddfmm_session_test_gemm_stall.restype = C.c_int
    vpp = C.POINTER(C.c_void_p)
    lib.ddfmm_batch_create.argtypes = [vpp, C.c_int, vpp]
    lib.ddfmm_batch_create.restype = C.c_int
    lib.ddfmm_batch_eval_c64.argtypes = [C.c_void_p, vpp, vpp]
    lib.ddfmm_batch_eval_c64.restype = C.c_int
    lib.ddfmm_batch_eval_device_c64.argtypes = [C.c_void_p, vpp, vpp, C.c_void_p]
    lib.ddfmm_batch_eval_device_c64.restype = C.c_int
    lib.ddfmm_batch_launches.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    lib.ddfmm_batch_launches.restype = C.c_int
    lib.ddfmm_batch_destroy.argtypes = [C.c_void_p]
    lib.ddfmm_batch_destroy.restype = C.c_int
    lib.ddfmm_server_create.argtypes = [C.c_int, C.c_double, vpp]
    lib.ddfmm_server_add_session.argtypes = [C.c_void_p, dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, dp,
                                             C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_char_p,
                                             C.POINTER(C.c_int)]
    lib.ddfmm_server_session_state.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    lib.ddfmm_server_remove_session.argtypes = [C.c_void_p, C.c_int]
    lib.ddfmm_server_submit.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_longlong)]
    lib.ddfmm_server_wait.argtypes = [C.c_void_p, C.c_longlong, C.c_double, C.POINTER(C.c_int)]
    lib.ddfmm_server_poll.argtypes = [C.c_void_p, C.c_longlong, C.POINTER(C.c_int)]
    lib.ddfmm_server_get_stats.argtypes = [C.c_void_p, C.POINTER(ddfmm_server_stats), C.c_int]
    lib.ddfmm_server_destroy.argtypes = [C.c_void_p]
    for f in ("ddfmm_server_create", "ddfmm_server_add_session", "ddfmm_server_session_state",
              "ddfmm_server_remove_session", "ddfmm_server_submit", "ddfmm_server_wait", "ddfmm_server_poll",
              "ddfmm_server_get_stats", "ddfmm_server_destroy"):
        getattr(lib, f).restype = C.c_int
    _lib = lib
    return lib


class DDFMMError(RuntimeError):
    """Raised where the reference throws (include/commoninc.hpp:52-53)."""

    def __init__(self, code, msg):
        super().__init__("ddfmm status %d: %s" % (code, msg))
        self.code = code


def tree_stats(pos, K, ptsmax, maxlevel, ncell, npq=4, ctr=(0.0, 0.0, 0.0)):
    """Host-only octree / list statistics (no GPU involved)."""
    lib = load()
    pos = __import__("numpy").ascontiguousarray(pos, dtype="float64").reshape(-1, 3)
    levels = (ddfmm_tree_level * 64)()
    tot, emp, nl = C.c_int(), C.c_int(), C.c_int()
    c3 = (C.c_double * 3)(*ctr)
    check(lib.ddfmm_tree_stats(pos.ctypes.data_as(C.POINTER(C.c_double)), pos.shape[0], float(K), c3, ptsmax,
                               maxlevel, ncell, npq, C.byref(tot), C.byref(emp), C.byref(nl), levels))
    out = [{k: getattr(levels[i], k) for k, _ in ddfmm_tree_level._fields_} for i in range(nl.value)]
    return dict(total_boxes=tot.value, empty_boxes=emp.value, levels=out)


def check(rc):
    if rc != 0:
        raise DDFMMError(rc, load().ddfmm_last_error().decode(errors="replace"))
