"""Matvec server: sessions admitted against a device-memory budget,
continuous batching of pending requests across sessions.

The bar for "the same alone and in the mix": a request's value equals the
matvec of the same session evaluated on its own (single-session mixed form)
to FP32 rounding of differently ordered atomic sums, 1e-5 relative l2
(observed ~1e-7)."""
import threading
import time

import numpy as np
import pytest

import fixtures
from ddfmm_b200 import _lib, wave3d

pytestmark = pytest.mark.gpu
TOL = 1e-5
CASES = ["sphere_k8_n5000_p4_helm", "sphere_k4_n1500_p4_expr", "cluster_k4_n1500_p4_helm_m8",
         "sphere_k16_n4000_p4_helm"]


def _opts(c):
    p = c.params
    return {"-wave3d_ACCU": str(p["accu"]), "-wave3d_NPQ": str(p["npq"]), "-wave3d_K": str(p["K"]),
            "-wave3d_ptsmax": str(p["ptsmax"]), "-wave3d_maxlevel": str(p["maxlevel"])}


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("serve")
    out = []
    rng = np.random.default_rng(11)
    for i, n in enumerate(CASES):
        c = fixtures.Case(n)
        d = tmp / ("ops%d" % i)
        d.mkdir()
        ldp, hdp = c.write_operators(str(d))
        mlib = wave3d.Mlib3d()
        mlib.setup({"-mlib3d_ldname": ldp, "-mlib3d_hdname": hdp})
        w = wave3d.Wave3d(precision=_lib.MIXED)
        w.posptr, w.kernel, w.mlibptr, w.geomprtn = c.pos, c.params["kernel"], mlib, c.params["nc"]
        w.setup(_opts(c))
        dens = [(rng.standard_normal(len(c.den)) + 1j * rng.standard_normal(len(c.den))).astype(np.complex64)
                for _ in range(6)]
        alone = []
        for dd in dens:
            v = np.zeros(len(dd), dtype=np.complex64)
            w.eval(dd, v)
            alone.append(v)
        out.append(dict(case=c, ld=ldp, hd=hdp, dens=dens, alone=alone, bytes=w.stats()["device_bytes"]))
        w.close()
    return out


def _add(sv, e):
    c = e["case"]
    return sv.add_session(c.pos, c.params["kernel"], e["ld"], e["hd"], _opts(c), c.params["nc"])


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_each_result_same_alone_and_in_the_mix(cases):
    sv = wave3d.Server(budget_bytes=1e12)
    sids = [_add(sv, e) for e in cases]
    assert sv.wait_admitted(sids) == [sv.ADMITTED] * len(sids)
    # a burst: every request of every session queued at once -> ticks carry several sessions
    vals = {}
    tickets = []
    for k, (sid, e) in enumerate(zip(sids, cases)):
        for r, d in enumerate(e["dens"]):
            v = np.zeros(len(d), dtype=np.complex64)
            vals[(k, r)] = v
            tickets.append(sv.submit(sid, d, v))
    for t in tickets:
        assert sv.wait(t, 120.0)
    burst = sv.stats(reset=True)
    print("burst: %d requests in %d ticks (mean batch %.2f), p50 %.2f ms p99 %.2f ms"
          % (burst["requests"], burst["ticks"], burst["mean_batch"], burst["p50_ms"], burst["p99_ms"]))
    assert burst["requests"] == len(tickets)
    assert burst["mean_batch"] >= 2.0
    for (k, r), v in vals.items():
        assert _rel(v, cases[k]["alone"][r]) <= TOL, (k, r, _rel(v, cases[k]["alone"][r]))
    # random arrivals from one thread per session: each result still equals the alone one
    errs = []

    def client(k, sid, e):
        rng = np.random.default_rng(100 + k)
        for rep in range(3):
            for r, d in enumerate(e["dens"]):
                time.sleep(rng.exponential(0.002))
                v = np.zeros(len(d), dtype=np.complex64)
                t = sv.submit(sid, d, v)
                if not sv.wait(t, 120.0):
                    errs.append((k, r, "timeout"))
                    continue
                rel = _rel(v, e["alone"][r])
                if rel > TOL:
                    errs.append((k, r, rel))

    th = [threading.Thread(target=client, args=(k, sid, e)) for k, (sid, e) in enumerate(zip(sids, cases))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    mix = sv.stats()
    print("random arrivals: %d requests in %d ticks (mean batch %.2f), p50 %.2f ms p99 %.2f ms"
          % (mix["requests"], mix["ticks"], mix["mean_batch"], mix["p50_ms"], mix["p99_ms"]))
    assert not errs, errs
    assert mix["requests"] == 3 * sum(len(e["dens"]) for e in cases)
    sv.close()


def test_admission_by_device_memory_budget(cases):
    a, b, c = cases[0], cases[1], cases[3]
    # a and b fit together, c fits once a is gone, but not next to both
    budget = b["bytes"] + c["bytes"] + a["bytes"] // 2
    assert a["bytes"] + b["bytes"] <= budget < a["bytes"] + b["bytes"] + c["bytes"]
    sv = wave3d.Server(budget_bytes=budget)
    sa, sb = _add(sv, a), _add(sv, b)
    assert sv.wait_admitted([sa, sb]) == [sv.ADMITTED, sv.ADMITTED]
    sc = _add(sv, c)
    time.sleep(0.5)
    assert sv.state(sc) == sv.WAITING  # does not fit next to a and b
    # a and b keep serving meanwhile
    v = np.zeros(len(b["dens"][0]), dtype=np.complex64)
    assert sv.wait(sv.submit(sb, b["dens"][0], v), 60.0)
    assert _rel(v, b["alone"][0]) <= TOL
    sv.remove(sa)
    assert sv.wait_admitted([sc]) == [sv.ADMITTED]
    assert sv.state(sa) == sv.REMOVED
    v = np.zeros(len(c["dens"][2]), dtype=np.complex64)
    assert sv.wait(sv.submit(sc, c["dens"][2], v), 60.0)
    assert _rel(v, c["alone"][2]) <= TOL
    with pytest.raises(_lib.DDFMMError):
        sv.submit(sa, a["dens"][0], np.zeros(len(a["dens"][0]), dtype=np.complex64))
    st = sv.stats()
    assert st["used_bytes"] <= budget
    sv.close()
    # a session larger than the whole budget is rejected
    sv = wave3d.Server(budget_bytes=a["bytes"] // 2)
    sa = _add(sv, a)
    assert sv.wait_admitted([sa]) == [sv.REJECTED]
    sv.close()


def test_k64_sphere_in_the_mix():
    """The served configuration's largest session -- the K=64 sphere, 321,699
    points -- admitted under the 30 GB budget next to K=8, 16 and 32 sessions:
    bursts and random arrivals from one client per session, every result
    equal to the same session's matvec evaluated alone."""
    from ddfmm_b200 import workloads as wl
    ws = [wl.LARGE] + wl.instance_mix([8, 16, 32], 1)
    rng = np.random.default_rng(17)
    dens = [[(rng.standard_normal(w.N) + 1j * rng.standard_normal(w.N)).astype(np.complex64) for _ in range(3)]
            for w in ws]
    alone = []
    for w, ds in zip(ws, dens):
        m = wave3d.from_workload(w, precision=_lib.MIXED)
        out = []
        for d in ds:
            v = np.zeros(w.N, dtype=np.complex64)
            m.eval(d, v)
            out.append(v)
        m.close()
        alone.append(out)
    sv = wave3d.Server(budget_bytes=30e9)
    sids = [sv.add_workload(w) for w in ws]
    assert sv.wait_admitted(sids) == [sv.ADMITTED] * len(sids)
    vals, tickets = {}, []
    for k, sid in enumerate(sids):
        for r, d in enumerate(dens[k]):
            v = np.zeros(len(d), dtype=np.complex64)
            vals[(k, r)] = v
            tickets.append(sv.submit(sid, d, v))
    for t in tickets:
        assert sv.wait(t, 120.0)
    burst = sv.stats(reset=True)
    print("K=64 mix burst: %d requests in %d ticks (mean batch %.2f), p50 %.2f ms p99 %.2f ms"
          % (burst["requests"], burst["ticks"], burst["mean_batch"], burst["p50_ms"], burst["p99_ms"]))
    assert burst["mean_batch"] >= 2.0
    for (k, r), v in vals.items():
        assert _rel(v, alone[k][r]) <= TOL, (k, r, _rel(v, alone[k][r]))
    errs = []

    def client(k, sid):
        crng = np.random.default_rng(200 + k)
        for rep in range(2):
            for r, d in enumerate(dens[k]):
                time.sleep(crng.exponential(0.005))
                v = np.zeros(len(d), dtype=np.complex64)
                if not sv.wait(sv.submit(sid, d, v), 120.0):
                    errs.append((k, r, "timeout"))
                    continue
                if _rel(v, alone[k][r]) > TOL:
                    errs.append((k, r, _rel(v, alone[k][r])))

    th = [threading.Thread(target=client, args=(k, sid)) for k, sid in enumerate(sids)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    mix = sv.stats()
    print("K=64 mix random arrivals: %d requests, mean batch %.2f, p50 %.2f ms p99 %.2f ms"
          % (mix["requests"], mix["mean_batch"], mix["p50_ms"], mix["p99_ms"]))
    assert not errs, errs
    sv.close()
