"""CPU restatement of the reference's Wave3d setup + eval, in numpy.

TEST INFRASTRUCTURE ONLY: the checker, never the thing measured or shipped.
Nothing in the product (ddfmm_b200/, include/) imports this module.

It restates, with its own data structures, the reference's single-rank
algorithm for this path:
  * tree and lists: Wave3d::setup_tree / setup_tree_callowlist /
    setup_tree_calhghlist / setup_tree_find / setup_tree_adjacent
    (src/wave3d_setup.cpp:100-477)
  * direction geometry: nml2dir / ParentDir / ChildDir / BoxCenter
    (src/wave3d.cpp:43-142), canonical wedges: HighFetchIndex3Sort /
    HighFetchShuffle / predir (src/mlib3d.cpp:283-357)
  * operator fetches: Mlib3d::{Upward,Downward}{Low,High}Fetch
    (src/mlib3d.cpp:106-280)
  * passes: EvalUpwardLow (src/wave3d_eval.cpp:418-490), the recursive
    high-frequency upward / downward passes (:721-854, :876-1040),
    EvalDownwardLow with U/V/W/X lists (:493-718), eval (:299-415)
  * kernel: Kernel3d::kernel (src/kernel3d.cpp:26-107), r := 1 below 1e-8
  * check: Wave3d::check's direct sum (src/wave3d_check.cpp:22-100)
It reads the operator files in the reference's binary format with its own
reader.  Pinned against the reference binary's outputs in
tests/test_oracle_cpu.py (golden fixtures).
"""
from __future__ import annotations

import math
import struct
from collections import deque

import numpy as np

TWO_PI = 2.0 * math.pi
PTS, TERMINAL = 1, 2


# ------------------------------------------------------------------ files
class _In:
    def __init__(self, path):
        self.b = open(path, "rb").read()
        self.o = 0

    def i(self):
        v = struct.unpack_from("<i", self.b, self.o)[0]
        self.o += 4
        return v

    def d(self):
        v = struct.unpack_from("<d", self.b, self.o)[0]
        self.o += 8
        return v

    def arr(self, dtype, n):
        a = np.frombuffer(self.b, dtype=dtype, count=n, offset=self.o).copy()
        self.o += a.nbytes
        return a

    def dmat(self):
        m, n = self.i(), self.i()
        return self.arr("<f8", m * n).reshape((m, n), order="F")

    def cmat(self):
        m, n = self.i(), self.i()
        return self.arr("<c16", m * n).reshape((m, n), order="F")

    def ctns(self):
        m, n, p = self.i(), self.i(), self.i()
        a = self.arr("<c16", m * n * p)
        return a.reshape((m, n, p), order="F") if a.size else None


def read_ld(path):
    """map<double, (uep, ucp, uc2ue[3], ue2dc 7x7x7)>  (src/mlib3d.cpp:361-379)"""
    r = _In(path)
    out = {}
    for _ in range(r.i()):
        W = r.d()
        uep, ucp = r.dmat(), r.dmat()
        uc2ue = [r.cmat() for _ in range(r.i())]
        dims = (r.i(), r.i(), r.i())
        t = {}
        for c in range(dims[2]):
            for b in range(dims[1]):
                for a in range(dims[0]):
                    x = r.ctns()
                    if x is not None:
                        t[(a, b, c)] = x
        out[W] = (uep, ucp, uc2ue, t)
    return out


def read_hd(path):
    """map<double, map<Index3, (uep, ucp, uc2ue[3])>>  (src/mlib3d.cpp:382-405)"""
    r = _In(path)
    out = {}
    for _ in range(r.i()):
        W = r.d()
        lev = {}
        for _ in range(r.i()):
            key = (r.i(), r.i(), r.i())
            uep, ucp = r.dmat(), r.dmat()
            lev[key] = (uep, ucp, [r.cmat() for _ in range(r.i())])
        out[W] = lev
    return out


# ------------------------------------------------------------------ kernel
def kernel(trg, src, kind):
    """Kernel3d::kernel: 3 x M targets, 3 x N sources -> M x N."""
    x = trg[0][:, None] - src[0][None, :]
    y = trg[1][:, None] - src[1][None, :]
    z = trg[2][:, None] - src[2][None, :]
    r2 = x * x + y * y + z * z
    r2[r2 < 1e-8 * 1e-8] = 1.0
    r = np.sqrt(r2)
    ph = np.exp(1j * (TWO_PI * r))
    if kind == 0:
        return ph / r
    if kind == 1:
        return ph
    raise ValueError("unknown kernel type")


# ------------------------------------------------------------------ directions
def linfty(d):
    return max(abs(v) for v in d)


def parent_dir(d):
    C = linfty(d)
    B = C // 2
    midx = [k for k in range(3) if abs(d[k]) == C][-1]
    r = []
    for v in d:
        t = int((v + C - 1) / 2)  # C++ integer division (operand >= 0)
        r.append(2 * (t // 2) + 1 - B)
    r[midx] = d[midx] // 2 if d[midx] >= 0 else -((-d[midx]) // 2)
    return tuple(r)


def child_dirs(d):
    C = linfty(d)
    o = [k for k in range(3) if abs(d[k]) != C]
    res = []
    for a in (0, 1):
        for b in (0, 1):
            t = [2 * v for v in d]
            t[o[0]] += 2 * a - 1
            t[o[1]] += 2 * b - 1
            res.append(tuple(t))
    return res


def index3_sort(val):
    sgn = [(-1 if v < 0 else 1) for v in val]
    v = [abs(x) for x in val]
    upp = max(v) + 1
    srt, prm = [0, 0, 0], [0, 0, 0]
    for d in range(3):
        mi, mv = d, v[d]
        for e in range(3):
            if v[e] < mv:
                mv, mi = v[e], e
        srt[d], prm[d] = mv, mi
        v[mi] = upp
    return tuple(srt), sgn, prm


def shuffle(pts, prm, sgn):
    res = np.empty_like(pts)
    for d in range(3):
        res[prm[d]] = pts[d]
    for d in range(3):
        res[d] = sgn[d] * res[d]
    return res


def shifted(ind, W):
    a, b, c = (ind >> 2) & 1, (ind >> 1) & 1, ind & 1
    return np.array([(a - 0.5) * W / 2, (b - 0.5) * W / 2, (c - 0.5) * W / 2])[:, None]


CHILD = [((i >> 2) & 1, (i >> 1) & 1, i & 1) for i in range(8)]


# ------------------------------------------------------------------ oracle
class Box:
    __slots__ = ("tag", "pts", "U", "V", "W", "X", "near", "far", "out", "inc")

    def __init__(self, pts):
        self.tag = 0
        self.pts = pts
        self.U, self.V, self.W, self.X, self.near = [], [], [], [], []
        self.far = {}
        self.out, self.inc = set(), set()


class Wave3dOracle:
    def __init__(self, pos, K, ncell, ptsmax, maxlevel, accu, kind, ld, hd, npq=4, ctr=(0.0, 0.0, 0.0)):
        self.pos = np.asarray(pos, dtype=np.float64)
        self.K, self.nc, self.ptsmax, self.maxlevel = float(K), ncell, ptsmax, maxlevel
        self.P = {1: 4, 2: 6, 3: 8}[accu]
        self.kind, self.npq, self.ctr = kind, npq, np.asarray(ctr, dtype=np.float64)
        self.ld, self.hd = ld, hd
        self.boxes = {}
        self.setup_tree()

    # ---- geometry
    def width(self, key):
        return self.K / (1 << key[0])

    def center(self, key):
        tmp = 1 << key[0]
        return np.array([self.ctr[d] - self.K / 2 + (key[1 + d] + 0.5) / tmp * self.K for d in range(3)])

    def unitlevel(self):
        return int(round(math.log(self.K) / math.log(2)))

    def cell_level(self):
        return int(round(math.log(self.nc) / math.log(2)))

    def nml2dir(self, n, W):
        C = self.npq * int(round(W))
        B = C // 2
        midx, mval = 0, abs(n[0])
        for d in (1, 2):
            if mval < abs(n[d]):
                midx, mval = d, abs(n[d])
        val = [math.atan(n[d] / mval) for d in range(3)]
        ang = (math.pi / 2) / C
        res = []
        for d in range(3):
            t = int(math.floor(val[d] / ang))
            res.append(2 * min(max(t, -B), B - 1) + 1)
        res[midx] = C * int(round(val[midx]))
        return tuple(res)

    @staticmethod
    def child(key, ind):
        a, b, c = CHILD[ind]
        return (key[0] + 1, 2 * key[1] + a, 2 * key[2] + b, 2 * key[3] + c)

    @staticmethod
    def adjacent(me, yo):
        md = max(me[0], yo[0])
        sm, sy = 1 << (md - me[0]), 1 << (md - yo[0])
        rad = sm + sy
        dif = [abs((2 * me[1 + d] + 1) * sm - (2 * yo[1 + d] + 1) * sy) for d in range(3)]
        return all(x <= rad for x in dif) and max(dif) == rad

    def find(self, key):
        cl = self.cell_level()
        while key[0] != cl:
            if key in self.boxes:
                return key
            key = (key[0] - 1, key[1] // 2, key[2] // 2, key[3] // 2)
        return key if key in self.boxes else None

    # ---- setup (src/wave3d_setup.cpp:100-299)
    def setup_tree(self):
        K, nc, lvl = self.K, self.nc, self.cell_level()
        idx = np.floor(nc * ((self.pos - self.ctr + K / 2) / K)).astype(np.int64)
        if idx.min() < 0 or idx.max() >= nc:
            raise ValueError("point outside the root box")
        cells = {}
        for pid in range(len(self.pos)):
            cells.setdefault(tuple(idx[pid]), []).append(pid)
        q = deque()
        for a in range(nc):
            for b in range(nc):
                for c in range(nc):
                    q.append(((lvl, a, b, c), cells.get((a, b, c), [])))
        ul = self.unitlevel()
        while q:
            key, pts = q.popleft()
            box = Box(pts)
            if pts:
                box.tag |= PTS
            if (key[0] <= ul and pts) or (len(pts) > self.ptsmax and key[0] < self.maxlevel - 1):
                cc = self.center(key)
                ch = [[] for _ in range(8)]
                for pid in pts:
                    p = self.pos[pid]
                    ch[(p[0] >= cc[0]) * 4 + (p[1] >= cc[1]) * 2 + (p[2] >= cc[2])].append(pid)
                for ind in range(8):
                    q.append((self.child(key, ind), ch[ind]))
                box.pts = []
            else:
                box.tag |= TERMINAL
            self.boxes[key] = box
        self.order = sorted(self.boxes)
        for key in self.order:
            b = self.boxes[key]
            if b.tag & PTS:
                if self.width(key) < 1 - 1e-12:
                    self.lowlist(key)
                else:
                    self.highlist(key)
        for key in self.order:
            b = self.boxes[key]
            W = self.width(key)
            if not (W > 1 - 1e-12 and b.tag & PTS):
                continue
            if key[0] != lvl:
                par = self.boxes[(key[0] - 1, key[1] // 2, key[2] // 2, key[3] // 2)]
                b.out |= {parent_dir(d) for d in par.out}
                b.inc |= {parent_dir(d) for d in par.inc}
            cc = self.center(key)
            for lst in b.far.values():
                for o in lst:
                    t = self.center(o) - cc
                    b.out.add(self.nml2dir(t / np.sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]), W))
                    t = cc - self.center(o)
                    b.inc.add(self.nml2dir(t / np.sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]), W))

    def lowlist(self, key):
        cur = self.boxes[key]
        U, V, Wl, X = set(), set(), set(), set()
        par = (key[1] // 2, key[2] // 2, key[3] // 2)
        L = 1 << key[0]
        rng = [range(max(2 * par[d] - 2, 0), min(2 * par[d] + 4, L)) for d in range(3)]
        term = cur.tag & TERMINAL
        for i in rng[0]:
            for j in rng[1]:
                for k in rng[2]:
                    if (i, j, k) == key[1:]:
                        continue
                    res = self.find((key[0], i, j, k))
                    if res is None:
                        continue
                    rb = self.boxes[res]
                    adj = self.adjacent(res, key)
                    if res[0] < key[0] and rb.tag & PTS:
                        if not adj:
                            X.add(res)
                        elif term:
                            U.add(res)
                    if res[0] == key[0]:
                        if not adj:
                            if rb.tag & PTS:
                                V.add(res)
                        elif term:
                            rest = deque([res])
                            while rest:
                                f = rest.popleft()
                                fb = self.boxes[f]
                                a2 = self.adjacent(f, key)
                                if not a2 and fb.tag & PTS:
                                    Wl.add(f)
                                if a2 and fb.tag & TERMINAL and fb.tag & PTS:
                                    U.add(f)
                                if a2 and not fb.tag & TERMINAL:
                                    rest.extend(self.child(f, ind) for ind in range(8))
        if term and cur.tag & PTS:
            U.add(key)
        cur.U, cur.V, cur.W, cur.X = sorted(U), sorted(V), sorted(Wl), sorted(X)

    def highlist(self, key):
        cur = self.boxes[key]
        cc = self.center(key)
        W = self.width(key)
        thr = W * W + W - 1e-12
        if key[0] == self.cell_level():
            cands = [k for k in self.order if k[0] == key[0]]
        else:
            par = self.boxes[(key[0] - 1, key[1] // 2, key[2] // 2, key[3] // 2)]
            cands = [self.child(t, ind) for t in par.near for ind in range(8)]
        for o in cands:
            if not self.boxes[o].tag & PTS:
                continue
            diff = cc - self.center(o)
            n = math.sqrt(diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2])
            if n >= thr:
                cur.far.setdefault(self.nml2dir(diff / n, W), []).append(o)
            else:
                cur.near.append(o)

    # ---- operator fetches (src/mlib3d.cpp:106-280)
    def hf_entry(self, W, d):
        srt, sgn, prm = index3_sort(d)
        uep, ucp, uc2ue = self.hd[W][srt]
        return shuffle(uep, prm, sgn), shuffle(ucp, prm, sgn), uc2ue

    # ---- eval (src/wave3d_eval.cpp:299-415)
    def eval(self, den):
        den = np.asarray(den, dtype=np.complex128)
        live = {k: b for k, b in self.boxes.items() if b.tag & PTS}
        leafpts = {k: np.array(b.pts, dtype=np.int64) for k, b in live.items() if b.tag & TERMINAL}
        upeq, dnchk, extval = {}, {}, {k: np.zeros(len(p), complex) for k, p in leafpts.items()}
        dirup, dirdn = {}, {}
        ldmap, hdmap = {}, {}
        for key in self.order:
            if key not in live:
                continue
            W = self.width(key)
            if W < 1 - 1e-12:
                ldmap.setdefault(W, []).append(key)
            else:
                for d in sorted(live[key].out):
                    hdmap.setdefault(d, ([], []))[0].append(key)
                for d in sorted(live[key].inc):
                    hdmap.setdefault(d, ([], []))[1].append(key)
        kind = self.kind
        # low-frequency upward, widths ascending
        for W in sorted(ldmap):
            uep, ucp, (v, is_, up), _ = self.ld[W]
            chd = {}
            for key in ldmap[W]:
                c = self.center(key)[:, None]
                if key in leafpts:
                    p = leafpts[key]
                    chk = kernel(ucp + c, self.pos[p].T, kind) @ den[p]
                else:
                    chk = np.zeros(ucp.shape[1], complex)
                    for ind in range(8):
                        ck = self.child(key, ind)
                        if ck in live:
                            if ind not in chd:
                                chd[ind] = kernel(ucp, self.ld[W / 2][0] + shifted(ind, W), kind)
                            chk += chd[ind] @ upeq[ck]
                upeq[key] = v @ ((up @ chk) * is_[:, 0])
        # high-frequency upward, pre-order over wedge refinements
        def up_rec(W, d):
            if d not in hdmap:
                return
            uep, ucp, (E1, E2, E3) = self.hf_entry(W, d)
            if W == 1.0:
                uepchd = self.ld[W / 2][0]
            else:
                uepchd = self.hf_entry(W / 2, parent_dir(d))[0]
            mats = {}
            for key in hdmap[d][0]:
                chk = np.zeros(ucp.shape[1], complex)
                for ind in range(8):
                    ck = self.child(key, ind)
                    if ck not in live:
                        continue
                    if ind not in mats:
                        mats[ind] = kernel(ucp, uepchd + shifted(ind, W), kind)
                    x = upeq[ck] if W == 1.0 else dirup[(ck, parent_dir(d))]
                    chk += mats[ind] @ x
                dirup[(key, d)] = E1 @ (E2 @ (E3 @ chk))
            for cd in child_dirs(d):
                up_rec(2 * W, cd)

        def down_rec(W, d):
            if d not in hdmap:
                return
            for cd in child_dirs(d):
                down_rec(2 * W, cd)
            uep, ucp, (E1, E2, E3) = self.hf_entry(W, d)
            dep, dcp = -ucp, -uep
            if W == 1.0:
                dcpchd = self.ld[W / 2][0]
            else:
                dcpchd = -self.hf_entry(W / 2, parent_dir(d))[0]
            mats, m2l = {}, {}
            for key in hdmap[d][1]:
                ct = self.center(key)
                dcv = dirdn.get((key, d))
                for s in live[key].far.get(d, []):
                    off = ct - self.center(s)
                    ok = tuple(np.round(off / W).astype(int))
                    if ok not in m2l:  # K(dcp + c_t, uep + c_s) depends on c_t - c_s only
                        m2l[ok] = kernel(dcp + ct[:, None], uep + self.center(s)[:, None], kind)
                    contrib = m2l[ok] @ dirup[(s, d)]
                    dcv = contrib if dcv is None else dcv + contrib
                dneq = E3.T @ (E2.T @ (E1.T @ dcv))
                for ind in range(8):
                    ck = self.child(key, ind)
                    if ck not in live:
                        continue
                    if ind not in mats:
                        mats[ind] = kernel(dcpchd + shifted(ind, W), dep, kind)
                    tgt = dnchk if W == 1.0 else dirdn
                    kk = ck if W == 1.0 else (ck, parent_dir(d))
                    tgt[kk] = tgt.get(kk, 0) + mats[ind] @ dneq

        base = sorted(d for d in hdmap if linfty(d) // self.npq == 1)
        for d in base:
            up_rec(1.0, d)
        for d in base:
            down_rec(1.0, d)
        # low-frequency downward, widths descending
        for W in sorted(ldmap, reverse=True):
            uep, ucp, (v, is_, up), tns = self.ld[W]
            P, G = self.P, 2 * self.P
            step = W / (P - 1)
            gi = [tuple(int(round((uep[d, k] + W / 2) / step)) + P for d in range(3)) for k in range(uep.shape[1])]
            spec = {}
            chd = {}
            for key in ldmap[W]:
                b = live[key]
                c = self.center(key)[:, None]
                chk = dnchk.get(key, np.zeros(uep.shape[1], complex))
                if key in leafpts:
                    p = leafpts[key]
                    for s in b.U:
                        q = leafpts[s]
                        extval[key] += kernel(self.pos[p].T, self.pos[q].T, kind) @ den[q]
                if b.V:
                    acc = np.zeros((G, G, G), complex)
                    for s in b.V:
                        if s not in spec:
                            g = np.zeros((G, G, G), complex)
                            for k, ijk in enumerate(gi):
                                g[ijk] = upeq[s][k]
                            spec[s] = np.fft.fftn(g)
                        o = tuple(int(round(x)) + 3 for x in (self.center(key) - self.center(s)) / W)
                        acc += spec[s] * tns[o]
                    val = np.fft.ifftn(acc)  # = unnormalised backward DFT / G^3
                    chk = chk + np.array([val[ijk] for ijk in gi])
                for s in b.W:
                    sb = live[s]
                    if s in leafpts and len(leafpts[s]) < uep.shape[1]:
                        q = leafpts[s]
                        extval[key] += kernel(self.pos[leafpts[key]].T, self.pos[q].T, kind) @ den[q]
                    else:
                        coef = self.width(s) / W
                        extval[key] += kernel(self.pos[leafpts[key]].T, coef * uep + self.center(s)[:, None],
                                              kind) @ upeq[s]
                for s in b.X:
                    q = leafpts[s]
                    if key in leafpts and len(leafpts[key]) < uep.shape[1]:
                        extval[key] += kernel(self.pos[leafpts[key]].T, self.pos[q].T, kind) @ den[q]
                    else:
                        chk = chk + kernel(uep + c, self.pos[q].T, kind) @ den[q]
                dneq = up.T @ ((v.T @ chk) * is_[:, 0])
                if key in leafpts:
                    extval[key] += kernel(self.pos[leafpts[key]].T, ucp + c, kind) @ dneq
                else:
                    for ind in range(8):
                        ck = self.child(key, ind)
                        if ck in live:
                            if ind not in chd:
                                chd[ind] = kernel(self.ld[W / 2][0] + shifted(ind, W), ucp, kind)
                            dnchk[ck] = dnchk.get(ck, 0) + chd[ind] @ dneq
        val = np.zeros(len(self.pos), complex)
        for key, p in leafpts.items():
            val[p] = extval[key]
        return val

    def direct(self, den, ids):
        """Wave3d::check's FP64 direct sum at the given ids."""
        ids = np.asarray(ids)
        return kernel(self.pos[ids].T, self.pos.T, self.kind) @ np.asarray(den, dtype=np.complex128)

    def counts(self):
        """What Wave3d::eval prints about the tree (src/wave3d_eval.cpp:345-372)."""
        boxes, dirs = {}, {}
        empty = 0
        for k, b in self.boxes.items():
            if not b.tag & PTS:
                empty += 1
                continue
            boxes[k[0]] = boxes.get(k[0], 0) + 1
            dirs[k[0]] = dirs.get(k[0], 0) + sum(len(v) for v in b.far.values())
        return len(self.boxes), empty, boxes, dirs
