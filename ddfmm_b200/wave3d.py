"""Host-side mirror of the reference's Wave3d / Mlib3d interface.

Usage follows the reference driver (src/tt.cpp:103-185):

    mlib = Mlib3d("mlib3d_"); mlib.kernel = kernel; mlib.setup(opts)
    wave = Wave3d("wave3d_")
    wave.posptr = pos            # (N, 3) float64, point ids 0..N-1
    wave.kernel = kernel
    wave.mlibptr = mlib
    wave.geomprtn = nc           # cells per edge of the partition tensor
    wave.setup(opts)             # -wave3d_ACCU/NPQ/K/ctr/ptsmax/maxlevel
    wave.eval(den, val)          # val[:] = FMM matvec of den
    relerr = wave.check(den, val, chkkeys)

ParVec<int, cpx, PtPrtn> becomes a complex128 array indexed by point id.
Failures raise DDFMMError where the reference throws std::exception.
Every eval runs on the GPU through libddfmm_b200.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import _lib


def _opt(opts, key, default, conv):
    v = opts.get(key)
    return conv(v) if v is not None else default


class Mlib3d:
    """Operator library handle: the ld/hd files named by -<prefix>ldname and
    -<prefix>hdname (src/mlib3d.cpp:70-103).  The files are read by the
    native library when a Wave3d session is set up."""

    def __init__(self, prefix="mlib3d_"):
        self.prefix = prefix
        self.kernel = 0
        self.NPQ = 4
        self.ldname = None
        self.hdname = None

    def setup(self, opts):
        p = "-" + self.prefix
        self.NPQ = _opt(opts, p + "NPQ", self.NPQ, int)
        self.ldname = _opt(opts, p + "ldname", self.ldname, str)
        self.hdname = _opt(opts, p + "hdname", self.hdname, str)
        for f in (self.ldname, self.hdname):
            if not f or not os.path.exists(f):
                raise _lib.DDFMMError(3, "operator file not found: %r" % (f,))
        return 0


class Wave3d:
    """precision: _lib.PLAIN_FP64 (every pass in FP64), _lib.MIXED (complex
    FP32 storage, 3xTF32 translations on tcgen05, FP32 near field) or
    _lib.MIXED_MMA_SYNC (the same with the translations on mma.sync)."""

    def __init__(self, prefix="wave3d_", device=0, precision=0):
        self.prefix = prefix
        self.precision = precision
        self.posptr = None
        self.kernel = 0
        self.mlibptr = None
        self.geomprtn = None
        self.ACCU = 1
        self.NPQ = 4
        self.K = 64.0
        self.ctr = (0.0, 0.0, 0.0)
        self.ptsmax = 100
        self.maxlevel = None
        self.device = device
        self._s = None
        self._n = 0

    # src/wave3d_setup.cpp:21-97
    def setup(self, opts):
        lib = _lib.load()
        p = "-" + self.prefix
        self.ACCU = _opt(opts, p + "ACCU", self.ACCU, int)
        self.NPQ = _opt(opts, p + "NPQ", self.NPQ, int)
        self.K = _opt(opts, p + "K", self.K, float)
        self.ctr = _opt(opts, p + "ctr", self.ctr, lambda s: tuple(float(x) for x in s.split()))
        self.ptsmax = _opt(opts, p + "ptsmax", self.ptsmax, int)
        self.maxlevel = _opt(opts, p + "maxlevel", self.maxlevel, int)
        if self.maxlevel is None:
            raise _lib.DDFMMError(1, "-%smaxlevel is required" % self.prefix)
        if self.posptr is None or self.mlibptr is None or self.geomprtn is None:
            raise _lib.DDFMMError(1, "posptr, mlibptr and geomprtn must be set before setup")
        pos = np.ascontiguousarray(self.posptr, dtype=np.float64).reshape(-1, 3)
        nc = self.geomprtn if isinstance(self.geomprtn, int) else int(np.asarray(self.geomprtn).shape[0])
        self.close()
        ctr = (C.c_double * 3)(*self.ctr)
        out = C.c_void_p()
        rc = lib.ddfmm_session_create_ex(pos.ctypes.data_as(C.POINTER(C.c_double)), pos.shape[0],
                                         int(self.kernel), self.ACCU, self.NPQ, self.K, ctr, self.ptsmax,
                                         self.maxlevel, nc, self.mlibptr.ldname.encode(),
                                         self.mlibptr.hdname.encode(), self.device, int(self.precision),
                                         C.byref(out))
        _lib.check(rc)
        self._s = out
        self._n = pos.shape[0]
        return 0

    def _need(self):
        if self._s is None:
            raise _lib.DDFMMError(1, "setup() has not been called")

    # src/wave3d_eval.cpp:299-415
    def eval(self, den, val):
        """val[:] = matvec(den).  val's dtype picks the I/O: complex128 always,
        complex64 on mixed sessions."""
        self._need()
        c64 = isinstance(val, np.ndarray) and val.dtype == np.complex64
        dt = np.complex64 if c64 else np.complex128
        d = np.ascontiguousarray(den, dtype=dt)
        if d.shape != (self._n,):
            raise _lib.DDFMMError(1, "den must hold %d complex values" % self._n)
        if not (isinstance(val, np.ndarray) and val.dtype == dt and val.shape == (self._n,)
                and val.flags.c_contiguous):
            raise _lib.DDFMMError(1, "val must be a contiguous complex128 (or, mixed, complex64) array of "
                                     "length %d" % self._n)
        if c64:
            fp = C.POINTER(C.c_float)
            _lib.check(_lib.load().ddfmm_eval_c64(self._s, d.ctypes.data_as(fp), val.ctypes.data_as(fp)))
        else:
            dp = C.POINTER(C.c_double)
            _lib.check(_lib.load().ddfmm_eval(self._s, d.ctypes.data_as(dp), val.ctypes.data_as(dp)))
        return 0

    def eval_device(self, den_ptr, val_ptr, stream_ptr=None, c64=False):
        """den_ptr / val_ptr: device addresses of N complex128 values
        (complex64 with c64=True, mixed sessions only)."""
        self._need()
        f = _lib.load().ddfmm_eval_device_c64 if c64 else _lib.load().ddfmm_eval_device
        _lib.check(f(self._s, C.c_void_p(den_ptr), C.c_void_p(val_ptr),
                     C.c_void_p(stream_ptr) if stream_ptr else None))

    def direct(self, den, ids):
        """FP64 direct sum at the given point ids."""
        self._need()
        d = np.ascontiguousarray(den, dtype=np.complex128)
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        out = np.zeros(ids.shape[0], dtype=np.complex128)
        dp = C.POINTER(C.c_double)
        _lib.check(_lib.load().ddfmm_direct(self._s, d.ctypes.data_as(dp), ids.ctypes.data_as(C.POINTER(C.c_int)),
                                            ids.shape[0], out.ctypes.data_as(dp)))
        return out

    # src/wave3d_check.cpp:22-100: relerr = |direct - fmm| / |fmm| at chkkeys
    def check(self, den, val, chkkeys):
        ids = np.asarray(chkkeys, dtype=np.int32)
        truth = self.direct(den, ids)
        fmm = np.asarray(val)[ids]
        return float(np.linalg.norm(truth - fmm) / np.linalg.norm(fmm))

    def stats(self):
        self._need()
        st = _lib.ddfmm_stats()
        _lib.check(_lib.load().ddfmm_session_stats(self._s, C.byref(st)))
        return st.as_dict()

    def profile(self, on=True):
        self._need()
        _lib.check(_lib.load().ddfmm_profile_enable(self._s, 1 if on else 0))

    def profile_read(self, reset=True):
        """Per-pass totals since the last reset: {label: dict(kernel, launches, ms, flops, bytes)}, in the
        order the eval first launches each label."""
        self._need()
        arr = (_lib.ddfmm_profile_entry * 64)()
        n = C.c_int()
        _lib.check(_lib.load().ddfmm_profile_read(self._s, arr, 64, C.byref(n), 1 if reset else 0))
        return {arr[i].label.decode(): dict(kernel=arr[i].kernel.decode(), launches=arr[i].launches, ms=arr[i].ms,
                                            flops=arr[i].flops, bytes=arr[i].bytes) for i in range(n.value)}

    def close(self):
        if self._s is not None:
            _lib.load().ddfmm_session_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Several mixed-form Wave3d instances evaluated together (merged
    multi-instance launches replayed as one CUDA graph).  The instances must
    stay open while the batch is used."""

    def __init__(self, waves):
        self.waves = list(waves)
        for w in self.waves:
            w._need()
        arr = (C.c_void_p * len(self.waves))(*[w._s for w in self.waves])
        out = C.c_void_p()
        _lib.check(_lib.load().ddfmm_batch_create(arr, len(self.waves), C.byref(out)))
        self._b = out

    def launches(self):
        n = C.c_int()
        _lib.check(_lib.load().ddfmm_batch_launches(self._b, C.byref(n)))
        return n.value

    def eval(self, dens, vals):
        """vals[i][:] = matvec_i(dens[i]) for every i with dens[i] is not None
        (complex64 arrays); the others are not computed."""
        n = len(self.waves)
        keep = []
        dp = (C.c_void_p * n)()
        vp = (C.c_void_p * n)()
        for i, (d, v) in enumerate(zip(dens, vals)):
            if d is None:
                continue
            d = np.ascontiguousarray(d, dtype=np.complex64)
            if d.shape != (self.waves[i]._n,) or v.dtype != np.complex64 or v.shape != d.shape:
                raise _lib.DDFMMError(1, "instance %d needs complex64 arrays of %d entries" % (i, self.waves[i]._n))
            if not v.flags.c_contiguous:
                raise _lib.DDFMMError(1, "val arrays must be contiguous")
            keep.append(d)
            dp[i] = d.ctypes.data
            vp[i] = v.ctypes.data
        _lib.check(_lib.load().ddfmm_batch_eval_c64(self._b, dp, vp))

    def eval_device(self, den_ptrs, val_ptrs, stream=None):
        """Device complex64 arrays (integer pointers, None = not computed)."""
        n = len(self.waves)
        dp = (C.c_void_p * n)(*[p if p else None for p in den_ptrs])
        vp = (C.c_void_p * n)(*[p if p else None for p in val_ptrs])
        _lib.check(_lib.load().ddfmm_batch_eval_device_c64(self._b, dp, vp, C.c_void_p(stream) if stream else None))

    def close(self):
        if getattr(self, "_b", None) is not None:
            _lib.load().ddfmm_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Matvec server (ddfmm_server_*): mixed-form sessions admitted against a
    device-memory budget, pending requests batched across sessions each tick."""
    WAITING, ADMITTED, REJECTED, REMOVED, FAILED = range(5)

    def __init__(self, budget_bytes, device=0):
        out = C.c_void_p()
        _lib.check(_lib.load().ddfmm_server_create(device, float(budget_bytes), C.byref(out)))
        self._sv = out
        self._n = {}
        self._inflight = {}

    def add_session(self, pos, kernel, ldname, hdname, opts, geomprtn, prefix="wave3d_"):
        """Arguments as Wave3d/Mlib3d: points (n x 3), kernel type, operator files,
        the -wave3d_* options and geomprtn (cells per edge)."""
        p = "-" + prefix
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        ctr = _opt(opts, p + "ctr", (0.0, 0.0, 0.0), lambda s: tuple(float(x) for x in s.split()))
        maxlevel = _opt(opts, p + "maxlevel", None, int)
        if maxlevel is None:
            raise _lib.DDFMMError(1, "-%smaxlevel is required" % prefix)
        nc = geomprtn if isinstance(geomprtn, int) else int(np.asarray(geomprtn).shape[0])
        c3 = (C.c_double * 3)(*ctr)
        sid = C.c_int()
        dp = C.POINTER(C.c_double)
        _lib.check(_lib.load().ddfmm_server_add_session(
            self._sv, pos.ctypes.data_as(dp), pos.shape[0], int(kernel), _opt(opts, p + "ACCU", 1, int),
            _opt(opts, p + "NPQ", 4, int), _opt(opts, p + "K", 64.0, float), c3, _opt(opts, p + "ptsmax", 100, int),
            maxlevel, nc, ldname.encode(), hdname.encode(), C.byref(sid)))
        self._n[sid.value] = pos.shape[0]
        return sid.value

    def add_workload(self, w):
        ld, hd = w.operators()
        return self.add_session(w.points(), w.kernel, ld, hd, w.options(), w.nc)

    def state(self, sid):
        st = C.c_int()
        _lib.check(_lib.load().ddfmm_server_session_state(self._sv, sid, C.byref(st)))
        return st.value

    def wait_admitted(self, sids, timeout=600.0):
        """Block until none of sids is waiting; returns their states."""
        t0 = time.time()
        while True:
            st = [self.state(s) for s in sids]
            if all(x != self.WAITING for x in st) or time.time() - t0 > timeout:
                return st
            time.sleep(0.01)

    def remove(self, sid):
        _lib.check(_lib.load().ddfmm_server_remove_session(self._sv, sid))

    def submit(self, sid, den, val):
        """Queue val[:] = matvec_sid(den) (complex64 arrays); returns a ticket."""
        d = np.ascontiguousarray(den, dtype=np.complex64)
        if d.shape != (self._n[sid],) or val.dtype != np.complex64 or val.shape != d.shape or \
                not val.flags.c_contiguous:
            raise _lib.DDFMMError(1, "session %d needs complex64 arrays of %d entries" % (sid, self._n[sid]))
        t = C.c_longlong()
        _lib.check(_lib.load().ddfmm_server_submit(self._sv, sid, d.ctypes.data, val.ctypes.data, C.byref(t)))
        self._inflight[t.value] = (d, val)  # keep the arrays alive until completion
        return t.value

    def wait(self, ticket, timeout=60.0):
        done = C.c_int()
        try:
            _lib.check(_lib.load().ddfmm_server_wait(self._sv, ticket, float(timeout), C.byref(done)))
        except _lib.DDFMMError:
            self._inflight.pop(ticket, None)
            raise
        if done.value:
            self._inflight.pop(ticket, None)
        return bool(done.value)

    def stats(self, reset=False):
        st = _lib.ddfmm_server_stats()
        _lib.check(_lib.load().ddfmm_server_get_stats(self._sv, C.byref(st), 1 if reset else 0))
        return st.as_dict()

    def close(self):
        if getattr(self, "_sv", None) is not None:
            _lib.load().ddfmm_server_destroy(self._sv)
            self._sv = None
            self._inflight.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def from_workload(w, device=0, precision=0):
    """Set up a Wave3d for a workloads.Workload (operators created on demand)."""
    ld, hd = w.operators()
    mlib = Mlib3d()
    mlib.kernel = w.kernel
    mlib.setup({"-mlib3d_ldname": ld, "-mlib3d_hdname": hd, "-mlib3d_NPQ": str(w.npq)})
    wave = Wave3d(device=device, precision=precision)
    wave.posptr = w.points()
    wave.kernel = w.kernel
    wave.mlibptr = mlib
    wave.geomprtn = w.nc
    wave.setup(w.options())
    return wave
