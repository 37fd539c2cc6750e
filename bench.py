#!/usr/bin/env python
"""Throughput of the directional FMM matvec (Wave3d::eval) on B200.

Workload: the large single instance -- points uniform by area on a sphere of
diameter K=64 wavelengths (N = 321,699, about 25 per square wavelength),
kernel exp(ir)/r, P=6 (ACCU 2), NPQ 4, ptsmax 100, complex128 N(0,1)
densities, seed 0.  One step = one matvec with fresh densities on a fixed
geometry (setup excluded, reported separately).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs its own replica of the instance on its GPU
(independent matvecs, no collective on the data path): weak scaling.
Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FMM matvecs/sec & points/sec at stated rel. err vs FP64 direct; p50/p99 latency"
CAP_FRACTION = 64  # the reference's bounded sample: a 1/64 spherical cap of the same sphere


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="large", choices=["large", "medium", "small"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-json", default=None, help="write the per-pass profile here")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision form measurement")
    ap.add_argument("--no-served", action="store_true", help="skip the continuous-batching server measurement")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the 64 uneven instances evaluated as one batch")
    ap.add_argument("--ellipsoid-table", default=None,
                    help="only tabulate the mixed form on the ellipsoid (K=128, N=900k by default) for the given "
                         "ACCU levels and kernels, optionally K and the form (mixed or plain), e.g. '1,2:0,1' or "
                         "'1,2,3:0:64:plain'")
    ap.add_argument("--mixed-mma-sync", action="store_true",
                    help="also measure the mixed form with its translations on the mma.sync path")
    return ap.parse_args()


def workload(name):
    from ddfmm_b200 import workloads as wl
    return {"large": wl.LARGE, "medium": wl.MEDIUM, "small": wl.SMALL}[name]


def max_over_ranks(x, ws, dev=None):
    """The largest value of x over all ranks; every rank calls it (a collective)."""
    if ws == 1:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(ms_per_step, ws):
    """matvec/s of the whole job: every rank evaluates its own instance (a
    replica) in each step, and a step lasts as long as the slowest rank's."""
    return ws * 1e3 / ms_per_step


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def fp64_peak_tflops(torch, dev):
    """Measured FP64 GEMM throughput (cuBLAS DGEMM via torch.matmul) as the
    denominator of the FP64 roofline; the driver's peak file has no FP64 entry."""
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def cap_directions(n):
    """n directions spread over the sphere (golden-angle spiral): the centres
    of the reference's sample caps."""
    i = np.arange(n) + 0.5
    z = 1.0 - 2.0 * i / n
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = np.pi * (3.0 - np.sqrt(5.0)) * i
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


def reference_step(w, nproc, timeout=900):
    """One step of the reference arm: nproc processes at once, one per host
    core, each running the reference binary (oracle/_ref/ref_eval, built from
    the reference's sources; Wave3d::eval timed with a steady clock) on the
    points of the workload's sphere inside a different 1/CAP_FRACTION
    spherical cap, with the workload's K, P, NPQ, ptsmax, maxlevel and
    operator files.  One eval per process (the reference's eval is not
    re-entrant).  Returns (total sample points, the longest eval seconds)."""
    from concurrent.futures import ThreadPoolExecutor
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import run_ref
    if not run_ref.available():
        raise RuntimeError("reference binary not built (make -C oracle)")
    pos, den = w.points(), w.densities()
    R = np.linalg.norm(pos, axis=1).max()
    ld, hd = w.operators()
    masks = [pos @ d >= R * (1 - 2.0 / CAP_FRACTION) for d in cap_directions(nproc)]

    def one(m):
        r = run_ref.run(pos[m], den[m], K=w.K, accu=w.accu, kernel=w.kernel, nc=w.nc, maxlevel=w.maxlevel,
                        ld_path=ld, hd_path=hd, ptsmax=w.ptsmax, npq=w.npq, timeout=timeout)
        return int(m.sum()), r["eval_s"]

    with ThreadPoolExecutor(nproc) as ex:
        res = list(ex.map(one, masks))
    return sum(n for n, _ in res), max(t for _, t in res)


def reference_procs():
    return max(1, min(CAP_FRACTION, host_cores()))


def sample_desc(w, nproc, npts):
    return ("reference Wave3d::eval (oracle/_ref/ref_eval, the reference's own sources built with its "
            "makeinc/wave4 flags against a one-rank MPI stand-in, an O(n^2) DFT stand-in for FFTW and naive "
            "BLAS; it has no threads) in %d processes at once, one per host core, each on the points of the "
            "workload's K=%g sphere inside a different 1/%d spherical cap (%d points in all per step, about %d "
            "each; same P/NPQ/ptsmax/maxlevel/operators); points/s = those points / the longest eval. Per point "
            "a cap is cheaper than the whole sphere (shorter far-field lists): one core took 2481 s for the "
            "whole %d-point matvec (130 points/s, tests/golden/full)"
            % (nproc, w.K, CAP_FRACTION, npts, npts // max(1, nproc), w.N))


def bench_config(w):
    """The config both arms report: the workload itself."""
    return {"workload": w.name, "geometry": w.geometry, "K": w.K, "N": w.N, "P": w.P,
            "kernel": "exp(ir)/r" if w.kernel == 0 else "exp(ir)", "npq": w.npq, "ptsmax": w.ptsmax,
            "l2": "inputs larger than L2 (one matvec's device working set is many times the 126 MB L2; "
                  "fresh densities each step, cycled over 4 inputs)"}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    w = workload(args.workload)
    nproc = reference_procs()
    steps = []
    for i in range(args.warmup + args.steps):
        steps.append(reference_step(w, nproc))
    timed = steps[args.warmup:] if len(steps) > args.warmup else steps
    sec = float(np.median([t for _, t in timed]))
    npts = timed[0][0]
    pps = npts / sec
    line = {"metric": METRIC, "impl": "reference", "value": pps, "unit": "points/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic", "config": bench_config(w),
            "cpu_baseline": {"value": pps, "unit": "points/s", "cores": nproc, "kind": "reference",
                             "sample": sample_desc(w, nproc, npts)},
            "e2e": {"value": pps, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def gemm_traffic(kernel, algorithmic_bytes):
    """DRAM bytes (read + write) per launch of the GEMM kernel, scaled from the
    small-case ncu capture committed under profiles/: the width-1 M2M launch of
    a K=16 sphere, whose DRAM bytes over its algorithmic bytes give the ratio
    applied to this workload's algorithmic bytes per launch.  None without the
    capture."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "gemm_dram_traffic_sphere_K16_P6.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.split()
        if f and not line.startswith("#") and f[0] == kernel:
            return (float(f[3]) + float(f[4])) / float(f[2]) * algorithmic_bytes
    return None


def measure_mixed(w, wave_args, steps, warmup, dev, chk, ws, profile_json=None, precision=None):
    """The mixed-precision form on the same workload: complex64 densities on
    the device, 3xTF32 translations (tcgen05 by default, or the mma.sync
    path); reports matvec/s, its error vs the FP64 direct sum and latency
    percentiles."""
    import torch
    from ddfmm_b200 import _lib, wave3d
    (local,) = wave_args
    precision = _lib.MIXED if precision is None else precision
    t0 = time.perf_counter()
    m = wave3d.from_workload(w, device=local, precision=precision)
    setup_s = time.perf_counter() - t0
    den = w.densities(np.complex64)
    rng = np.random.default_rng(7)
    dens = [den] + [(rng.standard_normal(w.N) + 1j * rng.standard_normal(w.N)).astype(np.complex64)
                    for _ in range(3)]
    den_d = [torch.from_numpy(np.ascontiguousarray(d).view(np.float32)).to(dev) for d in dens]
    val_d = torch.empty(2 * w.N, dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream
    for i in range(warmup):
        m.eval_device(den_d[i % 4].data_ptr(), val_d.data_ptr(), sp, c64=True)
    m.eval_device(den_d[0].data_ptr(), val_d.data_ptr(), sp, c64=True)
    stream.synchronize()
    v = val_d.cpu().numpy().view(np.complex64).astype(np.complex128)
    relerr = m.check(den.astype(np.complex128), v, chk)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    if profile_json:
        m.profile(True)
    for i in range(steps):
        with torch.cuda.stream(stream):
            ev[i][0].record(stream)
        m.eval_device(den_d[i % 4].data_ptr(), val_d.data_ptr(), sp, c64=True)
        with torch.cuda.stream(stream):
            ev[i][1].record(stream)
    stream.synchronize()
    if profile_json:
        prof = m.profile_read(reset=True)
        m.profile(False)
        json.dump({k: dict(v, ms_per_step=v["ms"] / steps) for k, v in prof.items()}, open(profile_json, "w"),
                  indent=1)
    lat = np.array([a.elapsed_time(b) for a, b in ev])
    ms = max_over_ranks(ev[0][0].elapsed_time(ev[-1][1]) / steps, ws, dev)
    # roofline of the dominant kernel from a separate event-profiled pass (the timed
    # steps above run without per-launch events)
    m.profile(True)
    for i in range(3):
        m.eval_device(den_d[i % 4].data_ptr(), val_d.data_ptr(), sp, c64=True)
    stream.synchronize()
    prof = m.profile_read(reset=True)
    m.profile(False)
    gk = {"launches": 0, "ms": 0.0, "flops": 0.0, "bytes": 0.0}
    for e in prof.values():
        if e["kernel"] in ("umma_cgemm_kernel", "zgemm_kernel"):
            gk["launches"] += e["launches"]
            gk["ms"] += e["ms"]
            gk["flops"] += e["flops"]
            gk["bytes"] += e["bytes"]
    roof = None
    if gk["ms"] > 0:
        peaks = measured_peaks()
        algo = gk["flops"] / (gk["ms"] * 1e-3) / 1e12  # complex flops (8 per complex MAC) / s
        executed = 3.0 * algo  # 3xTF32: three TF32 products per complex product
        if "bf16_tflops_sustained" in peaks:
            peak, src = peaks["bf16_tflops_sustained"] / 2, "MEASURED_PEAKS.json bf16_tflops_sustained / 2"
        else:
            peak, src = 1400.0 / 2, "fallback 1.4 PFLOP/s bf16 sustained / 2"
        kname = "umma_cgemm_kernel" if precision == _lib.MIXED else "cgemm_kernel"
        roof = {"bound": "tensor", "kernel": kname,
                "achieved": executed, "peak": peak, "unit": "TFLOP/s", "frac": executed / peak,
                "traffic": gemm_traffic(kname, 0.5 * gk["bytes"] / max(1, gk["launches"])),
                "traffic_note": "DRAM read + write bytes per launch: this workload's algorithmic bytes per launch "
                                "(complex64 columns and operators: algorithmic_bytes) times the DRAM / algorithmic "
                                "ratio of an ncu capture of the width-1 M2M launch on a K=16 sphere "
                                "(profiles/gemm_dram_traffic_sphere_K16_P6.txt)",
                "algorithmic_bytes": 0.5 * gk["bytes"] / max(1, gk["launches"]),
                "algorithmic_complex_tflops": algo, "launches": gk["launches"] // 3,
                "peak_source": src + " (dense TF32 runs at half the BF16 rate on B200's tensor cores)",
                "note": "executed = 3 x algorithmic (hi*hi + lo*hi + hi*lo TF32 products)"}
    m.close()
    gemm = "tcgen05" if precision == _lib.MIXED else "mma.sync"
    passes = {lab: {"ms_per_step": e["ms"] / 3, "launches_per_step": e["launches"] / 3, "kernel": e["kernel"]}
              for lab, e in sorted(prof.items(), key=lambda kv: -kv[1]["ms"])}
    return {"value": whole_job_rate(ms, ws), "unit": "matvec/s", "ms_per_step": ms,
            "dtype": "c64 (3xTF32 translations on %s)" % gemm,
            "relerr_vs_fp64_direct": relerr, "setup_s": setup_s, "roofline": roof,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "passes": passes}


def instance_mix(Ks, seed0):
    from ddfmm_b200 import workloads as wl
    return wl.instance_mix(Ks, seed0)


def served_workloads():
    """16 sessions: the bench sphere (K=64, N=321,699) and 15 spheres /
    ellipsoids with K cycling over 8, 16, 32, 64."""
    from ddfmm_b200 import workloads as wl
    return [wl.LARGE] + instance_mix([(8, 16, 32, 64)[j % 4] for j in range(15)], 1)


def measure_served(large_plain_e2e_s, budget_gb=30.0, closed_s=4.0, poisson_s=4.0):
    """Continuous-batching server (mixed form) on the served mix against the
    plain FP64 form serving the same requests one at a time."""
    import threading
    from ddfmm_b200 import _lib, wave3d
    ws_list = served_workloads()
    t0 = time.perf_counter()
    sv = wave3d.Server(budget_bytes=budget_gb * 1e9)
    sids = [sv.add_workload(w) for w in ws_list]
    states = sv.wait_admitted(sids, timeout=240.0)
    admit_s = time.perf_counter() - t0
    live = [(sid, w) for sid, w, st in zip(sids, ws_list, states) if st == sv.ADMITTED]
    rng = np.random.default_rng(5)
    dens = {sid: (rng.standard_normal(w.N) + 1j * rng.standard_normal(w.N)).astype(np.complex64) for sid, w in live}
    # closed loop: one request outstanding per session
    sv.stats(reset=True)
    stop = time.perf_counter() + closed_s
    counts = {}

    def client(sid, w):
        v = np.zeros(w.N, dtype=np.complex64)
        n = 0
        while time.perf_counter() < stop:
            t = sv.submit(sid, dens[sid], v)
            sv.wait(t, 120.0)
            n += 1
        counts[sid] = n

    th = [threading.Thread(target=client, args=lw) for lw in live]
    tc = time.perf_counter()
    for t in th:
        t.start()
    for t in th:
        t.join()
    closed_wall = time.perf_counter() - tc
    cst = sv.stats(reset=True)
    closed_rate = cst["requests"] / closed_wall
    # open loop: Poisson arrivals at half the saturated rate, sessions drawn uniformly
    lam = 0.5 * closed_rate
    arrivals = []
    tickets = []
    t_end = time.perf_counter() + poisson_s
    t_next = time.perf_counter()
    while True:
        t_next += rng.exponential(1.0 / lam)
        if t_next > t_end:
            break
        dt = t_next - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        k = int(rng.integers(len(live)))
        sid, w = live[k]
        v = np.zeros(w.N, dtype=np.complex64)
        tickets.append((sv.submit(sid, dens[sid], v), v))
        arrivals.append((t_next, k))
    for t, v in tickets:
        sv.wait(t, 120.0)
    pst = sv.stats(reset=True)
    used_gb = sv.stats()["used_bytes"] / 1e9
    sv.close()
    # plain FP64 per request: end-to-end service time of each session (host arrays in and out)
    service = []
    for sid, w in live:
        if w.name == ws_list[0].name:
            service.append(large_plain_e2e_s)
            continue
        p = wave3d.from_workload(w, precision=_lib.PLAIN_FP64)
        d = dens[sid].astype(np.complex128)
        v = np.zeros(w.N, dtype=np.complex128)
        p.eval(d, v)
        ts = []
        for _ in range(5):
            a = time.perf_counter()
            p.eval(d, v)
            ts.append(time.perf_counter() - a)
        p.close()
        service.append(float(np.median(ts)))
    plain_closed_rate = len(live) / sum(service)
    # the same Poisson arrivals served one at a time in arrival order
    free_at, lat = 0.0, []
    for ta, k in arrivals:
        start = max(ta, free_at)
        free_at = start + service[k]
        lat.append((free_at - ta) * 1e3)
    lat = np.array(lat) if lat else np.zeros(1)
    return {"sessions": len(live), "waiting": len(sids) - len(live), "budget_gb": budget_gb,
            "device_gb_used": used_gb, "admission_s": admit_s,
            "mix": "K=64 sphere N=321699 + 15 spheres/ellipsoids, K cycling 8, 16, 32, 64 (N = 25 pi K^2), P=6",
            "admitted_K": sorted(int(w.K) for _, w in live),
            "saturated": {"value": closed_rate, "unit": "matvec/s", "mean_batch": cst["mean_batch"],
                          "p50_ms": cst["p50_ms"], "p99_ms": cst["p99_ms"]},
            "poisson": {"rate_per_s": lam, "requests": pst["requests"], "mean_batch": pst["mean_batch"],
                        "p50_ms": pst["p50_ms"], "p99_ms": pst["p99_ms"]},
            "plain_fp64_per_request": {"value": plain_closed_rate, "unit": "matvec/s",
                                       "poisson_p50_ms": float(np.percentile(lat, 50)),
                                       "poisson_p99_ms": float(np.percentile(lat, 99)),
                                       "how": "measured end-to-end service time per session, requests served one at a "
                                              "time in arrival order"},
            "speedup_saturated": closed_rate / plain_closed_rate,
            "io": "host complex64 arrays in and out of the server (pinned staging, H2D/D2H inside each request)"}


def create_sessions(ws_list, precision, workers=8):
    """Sessions for every workload, created by a pool of threads (the C calls
    release the interpreter lock); the widest instance first and alone, so
    that the others find its translation operators in the shared cache."""
    from concurrent.futures import ThreadPoolExecutor
    from ddfmm_b200 import wave3d
    first = max(range(len(ws_list)), key=lambda i: ws_list[i].K)
    out = [None] * len(ws_list)
    out[first] = wave3d.from_workload(ws_list[first], precision=precision)
    with ThreadPoolExecutor(workers) as ex:
        futs = {i: ex.submit(wave3d.from_workload, w, 0, precision) for i, w in enumerate(ws_list) if i != first}
        for i, f in futs.items():
            out[i] = f.result()
    return out


def measure_batched(steps=5):
    """64 independent instances (K drawn from 4, 8, 16, 32; spheres and
    ellipsoids; N = 25 pi K^2; P=6) evaluated as one batch (merged
    multi-instance launches, one CUDA graph) against the same instances one
    after another, mixed and plain FP64; device-resident densities."""
    import torch
    from ddfmm_b200 import _lib, wave3d
    rng = np.random.default_rng(64)
    Ks = [int(k) for k in rng.choice([4, 8, 16, 32], 64)]
    ws_list = instance_mix(Ks, 100)
    t0 = time.perf_counter()
    waves = create_sessions(ws_list, _lib.MIXED)
    setup_s = time.perf_counter() - t0
    dev_gb = sum(wv.stats()["device_bytes"] for wv in waves) / 1e9
    b = wave3d.Batch(waves)
    dens = [torch.from_numpy(w.densities(np.complex64).view(np.float32)).cuda() for w in ws_list]
    vals = [torch.empty_like(d) for d in dens]
    dp = [d.data_ptr() for d in dens]
    vp = [v.data_ptr() for v in vals]
    st = torch.cuda.Stream()
    for _ in range(3):
        b.eval_device(dp, vp, st.cuda_stream)
    st.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(st):
        e0.record(st)
    for _ in range(steps):
        b.eval_device(dp, vp, st.cuda_stream)
    with torch.cuda.stream(st):
        e1.record(st)
    st.synchronize()
    batch_ms = e0.elapsed_time(e1) / steps
    # one after another, mixed
    for wv, d, v in zip(waves, dens, vals):
        wv.eval_device(d.data_ptr(), v.data_ptr(), st.cuda_stream, c64=True)
    st.synchronize()
    with torch.cuda.stream(st):
        e0.record(st)
    for _ in range(steps):
        for wv, d, v in zip(waves, dens, vals):
            wv.eval_device(d.data_ptr(), v.data_ptr(), st.cuda_stream, c64=True)
    with torch.cuda.stream(st):
        e1.record(st)
    st.synchronize()
    seq_ms = e0.elapsed_time(e1) / steps
    launches = b.launches()
    b.close()
    for wv in waves:
        wv.close()
    # one after another, plain FP64 (created three at a time ahead of their timing, then closed)
    from concurrent.futures import ThreadPoolExecutor
    plain_ms = 0.0
    with ThreadPoolExecutor(3) as ex:
        futs = [ex.submit(wave3d.from_workload, w, 0, _lib.PLAIN_FP64) for w in ws_list[:3]]
        for i, w in enumerate(ws_list):
            p = futs[i].result()
            if i + 3 < len(ws_list):
                futs.append(ex.submit(wave3d.from_workload, ws_list[i + 3], 0, _lib.PLAIN_FP64))
            d = torch.from_numpy(w.densities().view(np.float64)).cuda()
            v = torch.empty_like(d)
            p.eval_device(d.data_ptr(), v.data_ptr(), st.cuda_stream)
            st.synchronize()
            with torch.cuda.stream(st):
                e0.record(st)
            for _ in range(steps):
                p.eval_device(d.data_ptr(), v.data_ptr(), st.cuda_stream)
            with torch.cuda.stream(st):
                e1.record(st)
            st.synchronize()
            plain_ms += e0.elapsed_time(e1) / steps
            p.close()
    n = len(ws_list)
    return {"instances": n, "K_counts": {str(k): Ks.count(k) for k in (4, 8, 16, 32)},
            "points": int(sum(w.N for w in ws_list)), "setup_s": setup_s, "device_gb": dev_gb,
            "launches_per_batch_matvec": launches,
            "batched": {"value": n * 1e3 / batch_ms, "unit": "matvec/s", "ms_per_batch": batch_ms},
            "mixed_one_by_one": {"value": n * 1e3 / seq_ms, "unit": "matvec/s", "ms_per_round": seq_ms},
            "plain_fp64_one_by_one": {"value": n * 1e3 / plain_ms, "unit": "matvec/s", "ms_per_round": plain_ms},
            "speedup_vs_plain": plain_ms / batch_ms, "speedup_vs_mixed_one_by_one": seq_ms / batch_ms}


def ellipsoid_table(accus, kernels, K=128, steps=3, form="mixed"):
    """The mixed form on the ellipsoid with semi-axes 0.5, 0.25, 0.125 of a root
    box of K wavelengths (K=128: N = 900,000 uniform by area, 55 points per
    square wavelength; other K at the same density), complex64 N(0,1)
    densities, for each kernel and accuracy level: matvec/s and the relative
    error against the FP64 direct sum at 200 seeded targets."""
    import torch
    from ddfmm_b200 import _lib, wave3d, workloads as wl
    rows = []
    for kernel in kernels:
        for accu in accus:
            w = wl.ellipsoid(K, int(round(900000 * (K / 128.0) ** 2)), accu=accu, kernel=kernel)
            t0 = time.perf_counter()
            w.operators()
            ops_s = time.perf_counter() - t0
            t0 = time.perf_counter()
            mixed = form == "mixed"
            m = wave3d.from_workload(w, precision=_lib.MIXED if mixed else _lib.PLAIN_FP64)
            setup_s = time.perf_counter() - t0
            den = w.densities(np.complex64 if mixed else np.complex128)
            d = torch.from_numpy(den.view(np.float32 if mixed else np.float64)).cuda()
            v = torch.empty_like(d)
            st = torch.cuda.Stream()
            m.eval_device(d.data_ptr(), v.data_ptr(), st.cuda_stream, c64=mixed)
            st.synchronize()
            val = v.cpu().numpy().view(np.complex64 if mixed else np.complex128).astype(np.complex128)
            relerr = m.check(den.astype(np.complex128), val, w.check_ids())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(st):
                e0.record(st)
            for _ in range(steps):
                m.eval_device(d.data_ptr(), v.data_ptr(), st.cuda_stream, c64=mixed)
            with torch.cuda.stream(st):
                e1.record(st)
            st.synchronize()
            ms = e0.elapsed_time(e1) / steps
            stt = m.stats()
            rows.append({"form": form, "kernel": "exp(ir)/r" if kernel == 0 else "exp(ir)", "ACCU": accu, "P": w.P,
                         "K": K, "N": w.N,
                         "relerr_vs_fp64_direct": relerr, "ms_per_matvec": ms, "matvec_per_s": 1e3 / ms,
                         "setup_s": setup_s, "operator_files_s": ops_s, "device_gb": stt["device_bytes"] / 1e9})
            m.close()
            print(json.dumps(rows[-1]), flush=True)
    return rows


def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from ddfmm_b200 import wave3d
    w = workload(args.workload)
    w.operators()
    t0 = time.perf_counter()
    wave = wave3d.from_workload(w, device=local)
    setup_s = time.perf_counter() - t0
    st = wave.stats()
    den = w.densities()
    chk = w.check_ids()
    # device-resident inputs (value) -----------------------------------------
    rng = np.random.default_rng(1 + rank)
    n_inputs = 4  # fresh densities per step, cycled
    dens = [den] + [(rng.standard_normal(w.N) + 1j * rng.standard_normal(w.N)) for _ in range(n_inputs - 1)]
    den_d = [torch.from_numpy(np.ascontiguousarray(d).view(np.float64)).to(dev) for d in dens]
    val_d = torch.empty(2 * w.N, dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream
    for i in range(args.warmup):
        wave.eval_device(den_d[i % n_inputs].data_ptr(), val_d.data_ptr(), sp)
    stream.synchronize()
    # accuracy of this path against the FP64 direct sum at 200 targets
    wave.eval_device(den_d[0].data_ptr(), val_d.data_ptr(), sp)
    stream.synchronize()
    val0 = val_d.cpu().numpy().view(np.complex128)
    relerr = wave.check(den, val0, chk)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    # the timed steps run as a caller runs them: no per-launch events
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                ev[i][0].record(stream)
            wave.eval_device(den_d[i % n_inputs].data_ptr(), val_d.data_ptr(), sp)
            with torch.cuda.stream(stream):
                ev[i][1].record(stream)
        stream.synchronize()
    torch.cuda.synchronize(dev)
    if ws > 1:
        torch.distributed.barrier()
    lat = np.array([a.elapsed_time(b) for a, b in ev])
    total_ms = ev[0][0].elapsed_time(ev[-1][1])
    ms_per_step = max_over_ranks(total_ms / args.steps, ws, dev)
    value = whole_job_rate(ms_per_step, ws)
    # per-pass profile from a separate pass of event-bracketed launches
    prof_steps = 3
    wave.profile(True)
    for i in range(prof_steps):
        wave.eval_device(den_d[i % n_inputs].data_ptr(), val_d.data_ptr(), sp)
    stream.synchronize()
    prof = wave.profile_read(reset=True)
    wave.profile(False)
    # end to end through the public API with pinned host buffers ---------------
    den_h = torch.from_numpy(np.ascontiguousarray(den).view(np.float64)).pin_memory()
    val_h = torch.empty(2 * w.N, dtype=torch.float64).pin_memory()
    dh = den_h.numpy().view(np.complex128)
    vh = val_h.numpy().view(np.complex128)
    wave.eval(dh, vh)
    e2e_steps = max(1, min(args.steps, 5))
    if ws > 1:
        torch.distributed.barrier()
    t1 = time.perf_counter()
    for _ in range(e2e_steps):
        wave.eval(dh, vh)
    e2e_s = max_over_ranks((time.perf_counter() - t1) / e2e_steps, ws, dev)
    e2e_relerr = float(np.linalg.norm(vh - val0) / np.linalg.norm(val0))
    # roofline of the dominant kernel -------------------------------------------
    by_kernel = {}
    for lab, e in prof.items():
        # one kernel, whatever launch shape the autotuner chose for the pass
        k = by_kernel.setdefault(e["kernel"].split("<")[0], dict(ms=0.0, launches=0, flops=0.0, bytes=0.0))
        for f in ("ms", "launches", "flops", "bytes"):
            k[f] += e[f]
    dom = max(by_kernel, key=lambda k: by_kernel[k]["ms"])
    dk = by_kernel[dom]
    peaks = measured_peaks()
    if dom == "zgemm_kernel" or dom.startswith("pt"):
        peak = fp64_peak_tflops(torch, dev)
        achieved = dk["flops"] / (dk["ms"] * 1e-3) / 1e12
        roof = {"bound": "tensor", "pipe": "FP64 DMMA (mma.sync.m8n8k4.f64)", "kernel": dom, "achieved": achieved,
                "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": gemm_traffic(dom, dk["bytes"] / max(1, dk["launches"])),
                "traffic_note": "DRAM read + write bytes per launch: this workload's algorithmic bytes per launch "
                                "(algorithmic_bytes) times the DRAM / algorithmic ratio of an ncu capture of the "
                                "width-1 M2M launch on a K=16 sphere (profiles/gemm_dram_traffic_sphere_K16_P6.txt)",
                "algorithmic_bytes": dk["bytes"] / max(1, dk["launches"]),
                "peak_source": "measured cuBLAS DGEMM 4096^3 on this GPU (FP64 has no entry in MEASURED_PEAKS.json)",
                "launches": dk["launches"]}
    else:
        peak = peaks.get("hbm_gbs", 6650.0)
        achieved = dk["bytes"] / (dk["ms"] * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s",
                "launches": dk["launches"]}
    passes = {lab: {"ms_per_step": e["ms"] / prof_steps, "launches_per_step": e["launches"] / prof_steps,
                    "gflop_per_step": e["flops"] / prof_steps / 1e9, "kernel": e["kernel"]}
              for lab, e in sorted(prof.items(), key=lambda kv: -kv[1]["ms"])}
    # kernels of this library per matvec: the passes (memsets are not kernels) plus gather and scatter
    launches_per_step = sum(e["launches"] for lab, e in prof.items() if e["kernel"] != "memset") // prof_steps + 2
    clocks = clk.summary()
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and args.workload == "large":
        nproc = reference_procs()
        try:
            npts, sec = reference_step(w, nproc)
            cpu = {"value": npts / sec, "unit": "points/s", "cores": nproc, "kind": "reference",
                   "sample": "one step: " + sample_desc(w, nproc, npts)}
        except Exception as ex:  # the reference binary travels with the tree; report when it does not
            cpu = {"value": None, "unit": "points/s", "cores": nproc, "kind": "reference",
                   "sample": "unavailable: %s" % ex}
    mixed = None
    if not args.no_mixed:
        mixed = measure_mixed(w, wave_args=(local,), steps=args.steps, warmup=args.warmup, dev=dev, chk=chk, ws=ws,
                              profile_json=(args.profile_json + ".mixed") if args.profile_json else None)
    served = None
    if not args.no_served and ws == 1 and args.workload == "large":
        served = measure_served(e2e_s)
    batched = measure_batched() if not args.no_batched and ws == 1 and args.workload == "large" else None
    mixed_mma = None
    if args.mixed_mma_sync:
        from ddfmm_b200 import _lib
        mixed_mma = measure_mixed(w, wave_args=(local,), steps=args.steps, warmup=args.warmup, dev=dev, chk=chk,
                                  ws=ws, precision=_lib.MIXED_MMA_SYNC,
                                  profile_json=(args.profile_json + ".mma_sync") if args.profile_json else None)
    if args.profile_json and rank == 0:
        json.dump({"passes": passes, "by_kernel": by_kernel, "stats": st}, open(args.profile_json, "w"), indent=1)
    if rank == 0:
        line = {"metric": METRIC, "value": value * w.N, "unit": "points/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "c128", "data": "synthetic",
                "matvec_per_sec": value, "relerr_vs_fp64_direct": relerr,
                "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
                "config": bench_config(w),
                "form": "plain FP64", "parallelism": "replicas" if ws > 1 else "single GPU", "setup_s": setup_s,
                "setup_split_s": {k: st[k] for k in ("ops_seconds", "tree_seconds", "plan_seconds", "tune_seconds")},
                "device_gb": st["device_bytes"] / 1e9,
                "e2e": {"value": whole_job_rate(1e3 * e2e_s, ws) * w.N, "unit": "points/s",
                        "h2d_bytes_per_step": 16 * w.N, "d2h_bytes_per_step": 16 * w.N,
                        "matvec_per_sec": whole_job_rate(1e3 * e2e_s, ws), "rel_diff_vs_device_path": e2e_relerr},
                "roofline": roof, "gpu_launches": int(launches_per_step * args.steps),
                "clocks": clocks, "cpu_baseline": cpu, "mixed_form": mixed, "passes": passes}
        if mixed_mma:
            line["mixed_form_mma_sync"] = mixed_mma
        if served:
            line["served"] = served
        if batched:
            line["batched"] = batched
        print(json.dumps(line), flush=True)
    wave.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    if args.ellipsoid_table:
        parts = args.ellipsoid_table.split(":")
        K = int(parts[2]) if len(parts) > 2 else 128
        form = parts[3] if len(parts) > 3 else "mixed"
        rows = ellipsoid_table([int(x) for x in parts[0].split(",")], [int(x) for x in parts[1].split(",")], K,
                               form=form)
        print(json.dumps({"ellipsoid_table": rows, "config": "ellipsoid semi-axes 0.5/0.25/0.125 K, K=%d, "
                          "55 points per square wavelength, NPQ 4, ptsmax 100, mixed form, complex64 N(0,1) "
                          "densities, 200 check targets" % K}))
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
