"""FP64 translation-operator precompute, written in the reference's format.

The reference builds its operators offline in MATLAB (matlab/aug3d_script.m,
aug3d_lowdata.m, aug3d_hghdata.m) and ships none, so this module restates
that procedure with numpy/scipy (LAPACK SVD and pivoted QR, qhull hulls):

  * low frequency, widths 2^-7..2^-1 (aug3d_script.m:25): equivalent and
    check surfaces of a P^3 grid, the SVD pseudo-inverse of K(ucp, uep) split
    as {V, 1/sigma, U^H} (aug3d_lowdata.m:35-61), and the 316 FFT'd M2L
    tensors on a (2P)^3 wrap-around grid (aug3d_lowdata.m:81-105);
  * high frequency, widths 2^0..: per canonical wedge (a,b,C), a <= b odd,
    randomised pivoted-QR skeletons of the far-field interaction plus the
    middle factor G (aug3d_hghdata.m:18-284).

The MATLAB draws with an unseeded ``rand``; here every random draw comes
from a numpy Generator seeded per (kernel, ACCU, W, wedge), so the files are
reproducible.  The same files feed the reference binary and this project's
GPU path, which is what makes a bit-level parity comparison possible.

Both kernels are supported (KERNEL_HELM=0: exp(2 pi i r)/r, KERNEL_EXPR=1:
exp(2 pi i r); include/kernel3d.hpp:24-27).  The MATLAB only ever wrote
helm files (matlab/kernel3d.m:31).
"""
from __future__ import annotations

import hashlib
import math
import os
from concurrent.futures import ProcessPoolExecutor

import numpy as np
import scipy.linalg as sla
from scipy.spatial import ConvexHull

from . import formats

TPK = 2.0 * math.pi
KERNEL_HELM = 0
KERNEL_EXPR = 1


def accu_to_p(accu: int) -> int:
    """src/wave3d.cpp:145-158 / aug3d_lowdata.m:23-29."""
    if accu not in (1, 2, 3):
        raise ValueError("ACCU must be 1, 2 or 3 (got %r)" % (accu,))
    return {1: 4, 2: 6, 3: 8}[accu]


def kernel_matrix(trg: np.ndarray, src: np.ndarray, kind: int) -> np.ndarray:
    """Dense kernel matrix, trg/src given as 3 x M / 3 x N (matlab/kernel3d.m).
    The precompute never evaluates coincident pairs, so no r=0 guard."""
    d = trg[:, :, None] - src[:, None, :]
    r = np.sqrt(np.einsum("imn,imn->mn", d, d))
    if kind == KERNEL_HELM:
        return np.exp(1j * TPK * r) / r
    if kind == KERNEL_EXPR:
        return np.exp(1j * TPK * r)
    raise ValueError("unknown kernel type %r" % (kind,))


def _surface_grid(L: float, P: int) -> np.ndarray:
    """Surface nodes of a P^3 grid on [-L/2, L/2]^3 in ndgrid (x fastest)
    order (aug3d_lowdata.m:35-41)."""
    v = np.linspace(-L / 2, L / 2, P)
    z, y, x = np.meshgrid(v, v, v, indexing="ij")
    pp = np.vstack([x.ravel(), y.ravel(), z.ravel()])
    good = np.max(np.abs(pp), axis=0) == L / 2
    return pp[:, good]


# ------------------------------------------------------------- low frequency
def lowfreq_entry(accu: int, W: float, kind: int) -> formats.LowFreqEntry:
    """aug3d_lowdata.m:18-115."""
    P = accu_to_p(accu)
    uep = _surface_grid(W, P)
    ucp = _surface_grid(3 * W, P)
    M = kernel_matrix(ucp, uep, kind)
    U, s, Vh = np.linalg.svd(M, full_matrices=False)
    gd = s > 1e-16 * s[0]
    U, s, Vh = U[:, gd], s[gd], Vh[gd, :]
    uc2ue = [Vh.conj().T, (1.0 / s).astype(np.complex128).reshape(-1, 1), U.conj().T]
    step = W / (P - 1)
    t = np.concatenate([np.arange(P), np.arange(-P, 0)]) * step
    gz, gy, gx = np.meshgrid(t, t, t, indexing="ij")
    grid = np.vstack([gx.ravel(), gy.ravel(), gz.ravel()])
    ue2dc = {}
    for c in range(7):
        for b in range(7):
            for a in range(7):
                sa, sb, sc = a - 3, b - 3, c - 3
                if abs(sa) > 1 or abs(sb) > 1 or abs(sc) > 1:
                    pc = grid + (np.array([sa, sb, sc], dtype=np.float64) * W)[:, None]
                    col = kernel_matrix(pc, np.zeros((3, 1)), kind)[:, 0]
                    tns = col.reshape((2 * P, 2 * P, 2 * P), order="F")
                    ue2dc[(a, b, c)] = np.fft.fftn(tns)
    return formats.LowFreqEntry(uep, ucp, uc2ue, ue2dc)


# ------------------------------------------------------------ high frequency
def _hgh_dir(ns: np.ndarray, C: int) -> np.ndarray:
    """aug3d_hghdata_dir.m: continuous wedge coordinates of unit vectors."""
    t = np.max(np.abs(ns), axis=0)
    return np.arctan(ns / t) / (math.pi / 4) * C


def _hgh_predir(n):
    """aug3d_hghdata_predir.m (the same map as src/mlib3d.cpp:283-303 for a
    canonical wedge)."""
    C = max(abs(x) for x in n)
    r = [((x + C - 1) // 2) for x in n]
    r = [2 * (x // 2) + 1 - C // 2 for x in r]
    r[2] = n[2] // 2
    return tuple(r)


def _unique_rows(pts: np.ndarray) -> np.ndarray:
    """MATLAB unique(pts','rows')': sorted ascending by x, then y, then z."""
    return np.unique(pts.T, axis=0).T


def _hull_vertices(pts: np.ndarray) -> np.ndarray:
    return np.unique(ConvexHull(pts.T).simplices.ravel())


def _hull_facet_points(pts: np.ndarray) -> np.ndarray:
    """MATLAB play(:, convhulln(play')): facet vertices, repeated."""
    simp = ConvexHull(pts.T).simplices
    return pts[:, simp.T.ravel()]


_HF_PARAMS = {1: (1e-4, 70, 4, 2400), 2: (1e-6, 120, 5, 2400), 3: (1e-8, 160, 6, 4800)}


def _sample_sorted(rng, n_pick, total):
    """MATLAB sort(ceil(rand(1,n)*(total-n))) + [1:n], made 0-based."""
    r = np.sort(np.ceil(rng.random(n_pick) * (total - n_pick)).astype(np.int64))
    return r + np.arange(1, n_pick + 1) - 1


def _wedge(args):
    accu, W, kind, n, pspre, ptpre, seed = args
    EPS, rr, RT, NT = _HF_PARAMS[accu]
    rng = np.random.default_rng(seed)
    D = W * W + W
    DP = (2 * W) ** 2 + 2 * W
    C = 4 * W
    # far-field box centres in the positive octant and their wedge coordinates
    tmp = np.arange(0, 5 * D + 1e-9, W)
    sz, sy, sx = np.meshgrid(tmp, tmp, tmp, indexing="ij")
    sfts = np.vstack([sx.ravel(), sy.ravel(), sz.ravel()])
    sr = np.sqrt((sfts ** 2).sum(0))
    sfts = sfts[:, (sr >= D - 1e-8) & (sr <= 5 * D)]
    ns = _hgh_dir(sfts / np.sqrt((sfts ** 2).sum(0)), C)
    # source and target collections of the 8 children (aug3d_hghdata.m:96-113)
    cz, cy, cx = np.meshgrid([-W / 4, W / 4], [-W / 4, W / 4], [-W / 4, W / 4], indexing="ij")
    sgs = np.vstack([cx.ravel(), cy.ravel(), cz.ravel()])
    pscol = _unique_rows(np.hstack([pspre + sgs[:, t:t + 1] for t in range(8)]))
    ptcol = _unique_rows(np.hstack([ptpre + sgs[:, t:t + 1] for t in range(8)]))
    ps = pscol
    salw = _hull_vertices(ps)
    # targets (aug3d_hghdata.m:121-175)
    tol = 1.0 + 1e-8
    good = (np.abs(ns[0] - n[0]) <= tol) & (np.abs(ns[1] - n[1]) <= tol) & (np.abs(ns[2] - n[2]) <= 1e-8)
    sss = sfts[:, good]
    if sss.shape[1] == 0:
        raise RuntimeError("wedge %r at W=%g has no far-field centres" % (n, W))
    bz, by, bx = np.meshgrid([-W / 2, W / 2], [-W / 2, W / 2], [-W / 2, W / 2], indexing="ij")
    corners = np.vstack([bx.ravel(), by.ravel(), bz.ravel()])
    play = []
    for k in range(sss.shape[1]):
        c = sss[:, k:k + 1]
        play.append((1 if np.linalg.norm(c) < DP - 1e-8 else 3) * corners + c)
    play = np.hstack(play)
    pt0 = _hull_facet_points(play)
    dis = np.sqrt((sss ** 2).sum(0))
    mindis = dis.min()
    pt1 = _unique_rows(np.hstack([ptcol + sss[:, k:k + 1] for k in np.nonzero(dis < mindis + 1e-8)[0]]))
    u = play / np.sqrt((play ** 2).sum(0))
    thes = np.arctan2(u[0], u[2])
    phis = np.arctan2(u[1], u[2])
    the_rng = (thes.min(), thes.max())
    phi_rng = (phis.min(), phis.max())
    a, b = n[0], n[1]
    if (the_rng[0] > (a - 1) / C * math.pi / 4 or the_rng[1] < (a + 1) / C * math.pi / 4
            or phi_rng[0] > (b - 1) / C * math.pi / 4 or phi_rng[1] < (b + 1) / C * math.pi / 4):
        raise RuntimeError("wedge %r at W=%g: sample cone does not cover the wedge" % (n, W))
    rho_rng = (mindis - W / 2, 6 * D)
    the = rng.random(NT) * (the_rng[1] - the_rng[0]) + the_rng[0]
    phi = rng.random(NT) * (phi_rng[1] - phi_rng[0]) + phi_rng[0]
    rho = rng.random(NT) * (rho_rng[1] - rho_rng[0]) + rho_rng[0]
    t = np.sqrt(np.tan(the) ** 2 + np.tan(phi) ** 2 + 1)
    pt2 = np.vstack([np.tan(the) / t * rho, np.tan(phi) / t * rho, 1 / t * rho])
    talw2 = pt2[:, _hull_vertices(pt2)]
    pt = _unique_rows(np.hstack([pt0, pt1, pt2]))
    talw_pts = _unique_rows(np.hstack([pt0, pt1, talw2]))
    # indices of talw points inside pt (MATLAB intersect(...,'rows'))
    lookup = {tuple(row): i for i, row in enumerate(pt.T)}
    talw = np.array(sorted(lookup[tuple(row)] for row in talw_pts.T if tuple(row) in lookup), dtype=np.int64)
    # randomised pivoted QR skeletons (aug3d_hghdata.m:177-238)
    M, N = pt.shape[1], ps.shape[1]
    sz1 = rr * RT
    sz2 = rr * RT * RT
    nr = int(round(sz1 * math.sqrt(M / N)))
    rs = np.arange(M) if nr > M else _sample_sorted(rng, nr, M)
    rs = np.unique(np.concatenate([rs, talw]))
    M1 = kernel_matrix(pt[:, rs], ps, kind)
    _, R1, E1 = sla.qr(M1, mode="economic", pivoting=True)
    gd = np.abs(np.diag(R1)) > EPS * abs(R1[0, 0])
    idx1 = E1[:len(gd)][gd]
    psidx = ps[:, idx1]
    Q1, R1 = np.linalg.qr(kernel_matrix(pt, psidx, kind))
    nc = sz1
    cs = np.arange(N) if nc > N else _sample_sorted(rng, nc, N)
    cs = np.unique(np.concatenate([cs, salw, idx1]))
    M2 = kernel_matrix(pt, ps[:, cs], kind)
    _, R2, E2 = sla.qr(M2.conj().T, mode="economic", pivoting=True)
    gd = np.abs(np.diag(R2)) > EPS * abs(R2[0, 0])
    idx2 = E2[:len(gd)][gd]
    ptidx = pt[:, idx2]
    Q2, R2 = np.linalg.qr(kernel_matrix(ptidx, ps, kind).conj().T)
    nc = sz2
    cs = np.arange(N) if nc > N else _sample_sorted(rng, nc, N)
    cs = np.unique(np.concatenate([idx1, cs]))
    nr = sz2
    rs = np.arange(M) if nr > M else _sample_sorted(rng, nr, M)
    rs = np.unique(np.concatenate([idx2, rs]))
    M3 = kernel_matrix(pt[:, rs], ps[:, cs], kind)
    G = np.linalg.pinv(Q1[rs, :]) @ M3 @ np.linalg.pinv(Q2[cs, :].conj().T)
    E1m = sla.solve_triangular(R1, np.eye(R1.shape[0], dtype=np.complex128))
    E3m = sla.solve_triangular(R2.conj().T, np.eye(R2.shape[0], dtype=np.complex128), lower=True)
    return n, formats.HighFreqEntry(psidx.copy(), ptidx.copy(), [E1m, G, E3m])


def _worker_init():
    # one BLAS thread per worker process: the wedges are the parallelism
    from threadpoolctl import threadpool_limits
    threadpool_limits(1)


def _seed(kind, accu, W, n):
    h = hashlib.sha256(("ddfmm-hf|%d|%d|%r|%r" % (kind, accu, W, tuple(n))).encode()).digest()
    return int.from_bytes(h[:8], "little")


def highfreq_levels(accu: int, kind: int, wmax: int, workers: int | None = None) -> dict:
    """aug3d_script.m:53-66 + aug3d_hghdata.m for W = 1, 2, ..., wmax."""
    P = accu_to_p(accu)
    out = {}
    prev = None
    W = 1
    workers = workers or max(1, (os.cpu_count() or 1))
    while W <= wmax:
        C = 4 * W
        uns = sorted({tuple(sorted((a, b, C))) for a in range(1, C, 2) for b in range(1, C, 2)})
        jobs = []
        for n in uns:
            if W == 1:
                pg = _surface_grid(W / 2, P)
                pspre, ptpre = pg, pg
            else:
                e = prev[_hgh_predir(n)]
                pspre, ptpre = e.uep, -e.uep
            jobs.append((accu, W, kind, n, pspre, ptpre, _seed(kind, accu, W, n)))
        if workers > 1 and len(jobs) > 1:
            import multiprocessing as mp
            with ProcessPoolExecutor(max_workers=min(workers, len(jobs)),
                                     mp_context=mp.get_context("spawn"),
                                     initializer=_worker_init) as ex:
                res = list(ex.map(_wedge, jobs))
        else:
            res = [_wedge(j) for j in jobs]
        level = {n: e for n, e in res}
        for n, e in level.items():
            r1, r2 = e.uep.shape[1], e.ucp.shape[1]
            if max(r1, r2) > 400:
                raise RuntimeError("wedge %r at W=%d has rank %d > DVMAX=400 (src/wave3d_eval.cpp:25)"
                                   % (n, W, max(r1, r2)))
        out[float(W)] = level
        prev = level
        W *= 2
    return out


def lowfreq_levels(accu: int, kind: int) -> dict:
    return {2.0 ** e: lowfreq_entry(accu, 2.0 ** e, kind) for e in range(-7, 0)}


def operator_paths(cache_dir: str, kind: int, accu: int, wmax: int):
    name = "helm" if kind == KERNEL_HELM else "expr"
    return (os.path.join(cache_dir, "%s3d_ld_%d.bin" % (name, accu)),
            os.path.join(cache_dir, "%s3d_hd_%d_4_w%d.bin" % (name, accu, wmax)))


def ensure_operators(cache_dir: str, kind: int, accu: int, wmax: int, workers: int | None = None):
    """Create (once) and return the (ld, hd) operator file paths for HF
    widths 1..wmax.  Files are written atomically."""
    os.makedirs(cache_dir, exist_ok=True)
    ld_path, hd_path = operator_paths(cache_dir, kind, accu, wmax)
    # a file built for wider boxes holds every narrower width too
    w = max(1, wmax)
    while not os.path.exists(hd_path) and w <= 64:
        w *= 2
        cand = operator_paths(cache_dir, kind, accu, w)[1]
        if os.path.exists(cand):
            hd_path = cand
    if not os.path.exists(ld_path):
        tmp = ld_path + ".tmp%d" % os.getpid()
        formats.write_ld(tmp, lowfreq_levels(accu, kind))
        os.replace(tmp, ld_path)
    if not os.path.exists(hd_path):
        tmp = hd_path + ".tmp%d" % os.getpid()
        formats.write_hd(tmp, highfreq_levels(accu, kind, max(1, wmax), workers))
        os.replace(tmp, hd_path)
    return ld_path, hd_path
