"""Reader/writer for the reference's raw little-endian binary formats.

The reference serialises everything with include/serialize.hpp:
  * int = 4 bytes, double = 8 bytes, cpx = 2 doubles (serialize.hpp:53-110)
  * Index3 = 3 ints, Point3 = 3 doubles (serialize.hpp:114-150)
  * std::vector / std::set / std::map = int count + elements
    (serialize.hpp:155-245); a map is written in ascending key order
  * DblNumMat / CpxNumMat = int m, int n + column-major data
    (serialize.hpp:444-620; layout include/nummat.hpp:104-112)
  * CpxNumTns = int m, n, p + data with i fastest (include/numtns.hpp:104-117)
  * NumVec<T> / NumTns<T> of objects = dims + serialised elements, first
    index fastest (serialize.hpp:622-711)
  * ParVec<Key,Data,Prtn> = map<Key,Data> + the partition's owner vector
    (include/parvec.hpp:533-550; PtPrtn::ownerinfo is a vector<int> of prefix
    offsets, include/wave3d.hpp:40-57)

The operator files follow matlab/aug3d_script.m:36-84:
  ld: map<double, (DblNumMat uep, DblNumMat ucp, NumVec<CpxNumMat> uc2ue,
                   NumTns<CpxNumTns> ue2dc)>     (src/mlib3d.cpp:361-379)
  hd: map<double, map<Index3, (DblNumMat uep, DblNumMat ucp,
                               NumVec<CpxNumMat> uc2ue)>> (src/mlib3d.cpp:382-405)
"""
from __future__ import annotations

import io
import struct
from dataclasses import dataclass, field

import numpy as np


# ---------------------------------------------------------------- writers
class Writer:
    def __init__(self, f):
        self.f = f

    def int(self, v: int):
        self.f.write(struct.pack("<i", int(v)))

    def double(self, v: float):
        self.f.write(struct.pack("<d", float(v)))

    def dblmat(self, a):
        a = np.asarray(a, dtype=np.float64)
        if a.ndim == 1:
            a = a.reshape(-1, 1)
        m, n = a.shape
        self.int(m)
        self.int(n)
        self.f.write(np.asfortranarray(a).tobytes(order="F"))

    def cpxmat(self, a):
        a = np.asarray(a, dtype=np.complex128)
        if a.ndim == 1:
            a = a.reshape(-1, 1)
        m, n = a.shape
        self.int(m)
        self.int(n)
        self.f.write(np.asfortranarray(a).tobytes(order="F"))

    def cpxtns(self, a):
        if a is None:
            for _ in range(3):
                self.int(0)
            return
        a = np.asarray(a, dtype=np.complex128)
        m, n, p = a.shape
        self.int(m)
        self.int(n)
        self.int(p)
        self.f.write(np.asfortranarray(a).tobytes(order="F"))

    def inttns(self, a):
        a = np.asarray(a, dtype=np.int32)
        m, n, p = a.shape
        self.int(m)
        self.int(n)
        self.int(p)
        self.f.write(np.asfortranarray(a).tobytes(order="F"))

    def intvec(self, a):
        a = np.asarray(a, dtype=np.int32).ravel()
        self.int(a.size)
        self.f.write(a.tobytes())


class Reader:
    def __init__(self, buf: bytes):
        self.b = memoryview(buf)
        self.o = 0

    def _take(self, n):
        if self.o + n > len(self.b):
            raise ValueError("truncated file: need %d bytes at offset %d of %d" % (n, self.o, len(self.b)))
        v = self.b[self.o:self.o + n]
        self.o += n
        return v

    def int(self):
        return struct.unpack("<i", self._take(4))[0]

    def double(self):
        return struct.unpack("<d", self._take(8))[0]

    def _dims(self, k):
        d = [self.int() for _ in range(k)]
        if any(x < 0 for x in d):
            raise ValueError("negative dimension %r at offset %d" % (d, self.o))
        return d

    def dblmat(self):
        m, n = self._dims(2)
        return np.frombuffer(self._take(8 * m * n), dtype=np.float64).reshape((m, n), order="F").copy()

    def cpxmat(self):
        m, n = self._dims(2)
        return np.frombuffer(self._take(16 * m * n), dtype=np.complex128).reshape((m, n), order="F").copy()

    def cpxtns(self):
        m, n, p = self._dims(3)
        if m * n * p == 0:
            return None
        return np.frombuffer(self._take(16 * m * n * p), dtype=np.complex128).reshape((m, n, p), order="F").copy()

    def inttns(self):
        m, n, p = self._dims(3)
        return np.frombuffer(self._take(4 * m * n * p), dtype=np.int32).reshape((m, n, p), order="F").copy()

    def intvec(self):
        (m,) = self._dims(1)
        return np.frombuffer(self._take(4 * m), dtype=np.int32).copy()

    def done(self):
        return self.o == len(self.b)


# ------------------------------------------------------------ operator files
@dataclass
class LowFreqEntry:
    """One low-frequency width (src/mlib3d.hpp LowFreqEntry)."""
    uep: np.ndarray                 # 3 x n  equivalent points
    ucp: np.ndarray                 # 3 x n  check points
    uc2ue: list                     # [v (n x r), is (r x 1), up (r x n)]
    ue2dc: dict = field(default_factory=dict)  # (a,b,c) in 0..6 -> (2P)^3 tensor


@dataclass
class HighFreqEntry:
    """One canonical wedge at one width (src/mlib3d.hpp HghFreqDirEntry)."""
    uep: np.ndarray                 # 3 x r1 skeleton source points
    ucp: np.ndarray                 # 3 x r2 skeleton target points
    uc2ue: list                     # [E1 (r1 x r1), E2 (r1 x r2), E3 (r2 x r2)]


def write_ld(path, ld: dict):
    """ld: {W: LowFreqEntry}; written as map<double, LowFreqEntry>."""
    with open(path, "wb") as f:
        w = Writer(f)
        w.int(len(ld))
        for W in sorted(ld):
            e = ld[W]
            w.double(W)
            w.dblmat(e.uep)
            w.dblmat(e.ucp)
            w.int(3)
            for m in e.uc2ue:
                w.cpxmat(m)
            w.int(7)
            w.int(7)
            w.int(7)
            for c in range(7):
                for b in range(7):
                    for a in range(7):
                        w.cpxtns(e.ue2dc.get((a, b, c)))


def read_ld(path) -> dict:
    r = Reader(open(path, "rb").read())
    out = {}
    for _ in range(r.int()):
        W = r.double()
        uep = r.dblmat()
        ucp = r.dblmat()
        nv = r.int()
        uc2ue = [r.cpxmat() for _ in range(nv)]
        dims = r._dims(3)
        ue2dc = {}
        for c in range(dims[2]):
            for b in range(dims[1]):
                for a in range(dims[0]):
                    t = r.cpxtns()
                    if t is not None:
                        ue2dc[(a, b, c)] = t
        out[W] = LowFreqEntry(uep, ucp, uc2ue, ue2dc)
    if not r.done():
        raise ValueError("trailing bytes in %s" % path)
    return out


def _index3_key(d):
    return tuple(int(x) for x in d)


def write_hd(path, hd: dict):
    """hd: {W: {(a,b,c): HighFreqEntry}}; map<double, map<Index3, entry>>.
    Index3 keys are ordered lexicographically (include/vec3t.hpp:98-107)."""
    with open(path, "wb") as f:
        w = Writer(f)
        w.int(len(hd))
        for W in sorted(hd):
            w.double(W)
            inner = hd[W]
            w.int(len(inner))
            for key in sorted(inner, key=_index3_key):
                e = inner[key]
                for x in key:
                    w.int(x)
                w.dblmat(e.uep)
                w.dblmat(e.ucp)
                w.int(3)
                for m in e.uc2ue:
                    w.cpxmat(m)


def read_hd(path) -> dict:
    r = Reader(open(path, "rb").read())
    out = {}
    for _ in range(r.int()):
        W = r.double()
        inner = {}
        for _ in range(r.int()):
            key = (r.int(), r.int(), r.int())
            uep = r.dblmat()
            ucp = r.dblmat()
            nv = r.int()
            inner[key] = HighFreqEntry(uep, ucp, [r.cpxmat() for _ in range(nv)])
        out[W] = inner
    if not r.done():
        raise ValueError("trailing bytes in %s" % path)
    return out


# ------------------------------------------------------------ point files
def write_pos(path, pos: np.ndarray):
    """ParVec<int,Point3,PtPrtn> for one rank: map id->Point3, then the
    owner vector [0, N] (matlab/new_data.m:205-216)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    n = pos.shape[0]
    rec = np.zeros(n, dtype=[("k", "<i4"), ("p", "<f8", (3,))])
    rec["k"] = np.arange(n, dtype=np.int32)
    rec["p"] = pos
    with open(path, "wb") as f:
        f.write(struct.pack("<i", n))
        f.write(rec.tobytes())
        f.write(struct.pack("<iii", 2, 0, n))


def write_den(path, den: np.ndarray):
    """ParVec<int,cpx,PtPrtn> for one rank (matlab/new_data.m:218-229)."""
    den = np.ascontiguousarray(den, dtype=np.complex128).ravel()
    n = den.size
    rec = np.zeros(n, dtype=[("k", "<i4"), ("v", "<c16")])
    rec["k"] = np.arange(n, dtype=np.int32)
    rec["v"] = den
    with open(path, "wb") as f:
        f.write(struct.pack("<i", n))
        f.write(rec.tobytes())
        f.write(struct.pack("<iii", 2, 0, n))


def _read_parvec(path, dtype):
    buf = open(path, "rb").read()
    (n,) = struct.unpack_from("<i", buf, 0)
    rec = np.frombuffer(buf, dtype=[("k", "<i4"), ("v", dtype)], count=n, offset=4)
    r = Reader(buf)
    r.o = 4 + rec.nbytes
    owner = r.intvec()
    if not r.done():
        raise ValueError("trailing bytes in %s" % path)
    order = np.argsort(rec["k"], kind="stable")
    return rec["k"][order].copy(), rec["v"][order].copy(), owner


def read_pos(path):
    keys, v, owner = _read_parvec(path, ("<f8", (3,)))
    return keys, v, owner


def read_val(path):
    """ParVec<int,cpx,PtPrtn> as written by tt (src/tt.cpp:159-166)."""
    keys, v, owner = _read_parvec(path, "<c16")
    return keys, v, owner


def write_geomprtn(path, nc: int):
    """IntNumTns of owner ranks per cell; all zeros for one rank."""
    with open(path, "wb") as f:
        Writer(f).inttns(np.zeros((nc, nc, nc), dtype=np.int32))


def write_chk(path, ids):
    with open(path, "wb") as f:
        Writer(f).intvec(ids)


def read_chk(path):
    return Reader(open(path, "rb").read()).intvec()
