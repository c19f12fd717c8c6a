"""Benchmark of the multi-sphere T-matrix GMRES solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload medium|small]
                    [--operator direct|mlfmm] [--fmm-convention 0|1]

One step = one complete solve (GMRES to the workload's tolerance) of the seeded synthetic
scene.  The default workload is the 2000-sphere lognormal cluster (40 um cube, per-sphere
Wiscombe truncation, GMRES(50) to 1e-8, FP64, one x-polarised plane wave along +z).  With N > 1
(torchrun, one process per GPU) every rank solves its own replica: the path has no exchange
step, so there is no collective on the data path ("scaling": "weak").

Printed JSON line (rank 0):
  value      solves/s of the whole job with the scene resident in HBM (device-timed, max over
             ranks), e2e the same through the public API with host buffers (scene upload,
             solve, solution download inside the timed region);
  roofline   the operator kernel k_direct (>95% of the solve): achieved FP64 FLOP/s from the
             algorithmic flop count per launch and its CUDA-event time, against the FP64
             cuBLAS DGEMM rate measured in the same run;
  cpu_baseline  the FP64 oracle (restated reference algorithm, exact Xu translation
             coefficients recomputed for every pair as the reference does) timed on this
             host's cores on a bounded random sample of sphere pairs, extrapolated to solves/s.
--impl reference prints the same line for that CPU implementation alone.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# the reference's headline metric names the ML-FMM operator; lines that run the direct all-pairs
# operator (exact, the default) say so in the metric text
METRIC_MLFMM = "MLFMM-GMRES solves/s, p50/p99 latency at 1e-6 rel err vs plain FP64 on 1 B200"
METRIC = ("GMRES solves/s with the direct all-pairs T-matrix operator (in place of the ML-FMM), p50/p99 latency "
          "at 1e-6 rel err vs plain FP64 on 1 B200")

# Operator applications one solve of the default workload takes (GMRES(50) to 1e-8 with the
# initial residual and one explicit residual per restart), measured by the GPU arm; the CPU
# reference arm scales its per-matvec time by it.
MATVECS_PER_SOLVE = {"medium": 90, "small": None}


def workload_scene(name):
    from itofoggysim_b200 import scene as S
    if name == "small":
        return S.small_cluster()
    return S.medium_cluster()


def algorithmic_flops(sc):
    """FP64 flops of one direct-operator application, as written: per ordered pair (j <- l)
    two rotations (source degrees nu <= p_l, target degrees n <= p_j; a and b parts; a real
    d-matrix times a complex vector = 4 flops per term) and the axial step (4 complex MACs per
    (k, n, nu), 8 flops each); plus the T-matrix scaling 2 P_j complex multiplies per sphere."""
    p = sc.p_of_sphere().astype(np.int64)
    N = len(p)
    pv = np.arange(0, int(p.max()) + 1)
    rot = np.cumsum((2 * pv + 1) ** 2) - 1          # sum_{n=1..p} (2n+1)^2
    # axial terms: sum over k = -min..min of (#n >= max(1,|k|), n <= pj) (#nu >= max(1,|k|), nu <= pl)
    ps = np.unique(p)
    ax = {}
    for a in ps:
        for b in ps:
            mn = min(a, b)
            s = 0
            for k in range(-mn, mn + 1):
                lo = max(1, abs(k))
                s += (a - lo + 1) * (b - lo + 1)
            ax[(a, b)] = s
    cnt = {v: int(np.sum(p == v)) for v in ps}
    total = 0.0
    for a in ps:
        for b in ps:
            pairs = cnt[a] * cnt[b] - (cnt[a] if a == b else 0)
            total += pairs * (4.0 * 2 * (rot[b] + rot[a]) + 8.0 * 4 * ax[(a, b)])
    total += 8.0 * float(np.sum(2 * p * (p + 2)))
    return total


def translation_flops(pt, ps):
    """Flops of one translation from a degree-ps expansion to a degree-pt one, counted as in
    algorithmic_flops (two rotations and the axial step)."""
    rot = lambda p: sum((2 * n + 1) ** 2 for n in range(1, p + 1))
    mn = min(pt, ps)
    ax = sum((pt - max(1, abs(k)) + 1) * (ps - max(1, abs(k)) + 1) for k in range(-mn, mn + 1))
    return 4.0 * 2 * (rot(ps) + rot(pt)) + 8.0 * 4 * ax


def _morton(c, l):
    n = 0
    for b in range(l):
        for d in range(3):
            n |= ((c[d] >> b) & 1) << (3 * b + (2 - d))
    return n


def _demorton(n, l):
    c = [0, 0, 0]
    for b in range(l):
        for d in range(3):
            c[d] |= ((n >> (3 * b + (2 - d))) & 1) << b
    return c


def fmm_flops(sc, uindex, lmin, lmax, row_rule):
    """Flops of one ML-FMM operator application from the tree the library built (per-sphere box
    index at l_max): aggregation, M2M, M2L over the interaction lists, L2L, box-to-sphere and the
    near field, each translation counted by translation_flops, plus the T-matrix scaling."""
    p = sc.p_of_sphere().astype(int)
    pg = int(sc.n_range[1])
    lmin = min(lmin, lmax)
    boxes = {l: set(int(u) >> (3 * (lmax - l)) for u in uindex) for l in range(lmin, lmax + 1)}
    tp = translation_flops(pg, pg)
    total = 0.0
    total += sum(translation_flops(pg, int(pi)) for pi in p if not row_rule or pi >= pg)
    total += sum(len(boxes[l]) for l in range(lmin + 1, lmax + 1)) * tp * 2     # M2M and L2L
    for l in range(lmin, lmax + 1):
        hi = (1 << l) - 1
        for nb in boxes[l]:
            c = _demorton(nb, l)
            own = {_morton([c[0] + dx, c[1] + dy, c[2] + dz], l)
                   for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)
                   if all(0 <= c[d] + v <= hi for d, v in enumerate((dx, dy, dz)))}
            pc = _demorton(nb >> 3, l - 1) if l > 0 else [0, 0, 0]
            phi = (1 << (l - 1)) - 1 if l > 0 else -1
            par = {_morton([pc[0] + dx, pc[1] + dy, pc[2] + dz], l - 1)
                   for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)
                   if l > 0 and all(0 <= pc[d] + v <= phi for d, v in enumerate((dx, dy, dz)))}
            i4 = {(q << 3) | ch for q in par for ch in range(8)} - own
            total += len(i4 & boxes[l]) * tp
    leaf = [int(u) for u in uindex]
    total += sum(translation_flops(int(pj), pg) for pj in p)
    members = {}
    for j, b in enumerate(leaf):
        members.setdefault(b, []).append(j)
    hi = (1 << lmax) - 1
    for b, js in members.items():
        c = _demorton(b, lmax)
        near = []
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    q = [c[0] + dx, c[1] + dy, c[2] + dz]
                    if all(0 <= v <= hi for v in q):
                        near += members.get(_morton(q, lmax), [])
        for j in js:
            total += sum(translation_flops(int(p[j]), int(p[l])) for l in near if l != j)
    total += 8.0 * float(np.sum(2 * p * (p + 2)))
    return total


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(np.max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def measure_fp64_peak(torch, dev):
    """cuBLAS DGEMM 8192^3 (float64 torch.matmul), best of 5, TFLOP/s."""
    return measure_gemm_peak(torch, dev, torch.float64)


def measure_fp32_peak(torch, dev):
    """cuBLAS SGEMM 8192^3 on the CUDA cores (float32 torch.matmul with TF32 off), best of 5,
    TFLOP/s."""
    keep = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        return measure_gemm_peak(torch, dev, torch.float32)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = keep


def measure_gemm_peak(torch, dev, dtype):
    n = 8192
    a = torch.randn(n, n, dtype=dtype, device=dev)
    b = torch.randn(n, n, dtype=dtype, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def cpu_sample(sc, budget_s=15.0, seed=0):
    """Time the oracle (reference algorithm, translation blocks recomputed per pair) on random
    ordered sphere pairs for about budget_s seconds on all host cores; returns seconds per
    operator application (extrapolated over all N (N - 1) pairs) and the sample size."""
    from oracle import oracle as O
    P = O.Problem(sc)
    rng = np.random.default_rng(seed)
    x = P.vector_b()
    N = sc.n_spheres
    done, elapsed = 0, 0.0
    batch = max(os.cpu_count() or 1, 1)
    while elapsed < budget_s and done < N * (N - 1):
        t = rng.integers(0, N, batch)
        s = (t + rng.integers(1, N, batch)) % N
        t0 = time.perf_counter()
        P.pairs_apply(x, t, s)
        elapsed += time.perf_counter() - t0
        done += batch
    per_pair = elapsed / done
    return per_pair * N * (N - 1), done, elapsed


def cpu_cached_sample():
    """The cached CPU mode of the reference algorithm: the oracle's operator with the translation blocks of
    every ordered pair built once and kept (bit-identical to recomputing them), timed on all host cores
    for the 64-sphere cluster, where the cache fits (4032 pairs x 2 blocks of 255^2 complex, 8.4 GB).  Returns seconds per cached application and the seconds the cache took to build."""
    from oracle import oracle as O
    from itofoggysim_b200 import scene as S
    sc = S.small_cluster()
    P = O.Problem(sc)
    x = P.vector_b()
    t0 = time.perf_counter()
    P.matvec_rows(x, 0, sc.n_spheres, cache=True)
    build = time.perf_counter() - t0
    reps = []
    for _ in range(3):
        t0 = time.perf_counter()
        P.matvec_rows(x, 0, sc.n_spheres, cache=True)
        reps.append(time.perf_counter() - t0)
    return float(np.median(reps)), build, sc


def cached_scale(sc_from, sc_to):
    """Ratio of the cached operator's work between two scenes: a cached application is one dense
    (2 P_j x 2 P_l) block product per ordered pair, so its cost goes with sum_{j != l} P_j P_l."""
    def w(sc):
        p = sc.p_of_sphere().astype(np.float64)
        P = p * (p + 2)
        return float(P.sum() ** 2 - (P * P).sum())
    return w(sc_to) / w(sc_from)


def cached_bytes(sc):
    """Bytes of every ordered pair's two translation blocks A, B: 2 x P_j P_l x 16."""
    p = sc.p_of_sphere().astype(np.float64)
    P = p * (p + 2)
    return 32.0 * float(P.sum() ** 2 - (P * P).sum())


def job_rate(local_ms, units, world, torch, dev, dist):
    """Whole-job rate of replicas: every rank processed `units` in local_ms of its own device
    time; the job's time is the slowest rank's, so rate = world * units / max over ranks.
    Returns (rate per second, max_ms)."""
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    return world * units / (max_ms * 1e-3), max_ms


def percentile(v, q):
    return float(np.percentile(np.asarray(v), q)) if len(v) else None


def run_reference(args, rank, world):
    if rank != 0:
        return
    sc = workload_scene(args.workload)
    matvecs = MATVECS_PER_SOLVE[args.workload] or args.matvecs_per_solve
    cores = os.cpu_count()
    times, per_mv = [], []
    for i in range(args.warmup + args.steps):
        s_mv, pairs, el = cpu_sample(sc, budget_s=args.cpu_budget / max(1, args.steps), seed=i)
        if i >= args.warmup:
            per_mv.append(s_mv)
            times.append(s_mv * matvecs)
    sps = 1.0 / float(np.mean(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": sps, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(times)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_of(sc, args),
        "cpu_baseline": {"value": sps, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": "%d random sphere pairs per step, exact Xu translations recomputed per pair "
                                   "(reference algorithm), extrapolated x N(N-1) pairs x %d matvecs/solve"
                                   % (pairs, matvecs)},
        "e2e": {"value": sps, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_serving(args):
    """A seeded Poisson stream of solve requests (itofoggysim_b200.scene.serving_request) submitted
    at their arrival times to the solve server; value = requests completed per second of the
    stream's makespan, latency = submission to completion per request.  The same stream run one
    request at a time gives the plain-path comparison."""
    from itofoggysim_b200 import scene as S
    from itofoggysim_b200.server import SolveServer
    rng = np.random.default_rng(42)
    reqs = [S.serving_request(rng) for _ in range(args.warmup + args.steps)]
    gaps = np.random.default_rng(43).exponential(1.0 / 50.0, len(reqs))

    prec = 1 if args.precision == "mixed" else 0

    def stream(concurrent, prec):
        with SolveServer(max_concurrent=concurrent) as srv:
            for sc in reqs[:args.warmup]:
                srv.wait(srv.submit(sc, rhs_per_wave=True, precision=prec))
            t0 = time.perf_counter()
            ids, t_arr = [], t0
            for sc, gap in zip(reqs[args.warmup:], gaps[args.warmup:]):
                t_arr += gap
                dt = t_arr - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                ids.append(srv.submit(sc, rhs_per_wave=True, precision=prec))
            infos = [srv.wait(i)[0] for i in ids]
            span = time.perf_counter() - t0
        ok = [i for i in infos if i["state"] == 2]
        lat = [i["ms_latency"] for i in ok]
        return dict(solves_s=len(ok) / span, p50_ms=percentile(lat, 50), p99_ms=percentile(lat, 99),
                    done=len(ok), failed=len(infos) - len(ok), makespan_s=span,
                    rhs=int(sum(i["nrhs"] for i in ok)), iterations=int(sum(i["stats"]["iterations"] for i in ok)))

    co = stream(args.concurrent, prec)
    # the plain FP64 path one request at a time
    one = stream(1, 0)
    timed = reqs[args.warmup:]
    line = {
        "metric": METRIC, "value": co["solves_s"], "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": co["makespan_s"] * 1e3 / max(1, args.steps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 translations, f64 Krylov and residuals" if prec else "f64", "data": "synthetic",
        "config": {"workload": "serving stream: 50-500 lognormal spheres per request, 1-16 right-hand sides", "requests": args.steps,
                   "arrivals": "Poisson, 50 per s", "spheres": [int(min(r.n_spheres for r in timed)),
                                                                 int(max(r.n_spheres for r in timed))],
                   "rhs_total": co["rhs"], "gmres_tolerance": 1e-6, "concurrent": args.concurrent,
                   "admission": "FIFO by device footprint",
                   "solve": "a request's right-hand sides as one block (foggy_solve_block), %s"
                            % ("mixed precision" if prec else "FP64"),
                   "one_at_a_time": "the same stream, FP64, one request at a time"},
        "latency_ms": {"p50": co["p50_ms"], "p99": co["p99_ms"]},
        "serving": co, "one_at_a_time": one,
    }
    print(json.dumps(line), flush=True)


def fibonacci_waves(n_dir):
    """n_dir incidence directions on a Fibonacci sphere (z_i = 1 - (2i+1)/n, phi_i = i pi (3 - sqrt 5))
    times the two polarisations TM (Jones (1, 0)) and TE (Jones (0, 1))."""
    i = np.arange(n_dir)
    th = np.arccos(1.0 - (2.0 * i + 1.0) / n_dir)
    ph = np.mod(i * math.pi * (3.0 - math.sqrt(5.0)), 2.0 * math.pi)
    th2, ph2 = np.repeat(th, 2), np.repeat(ph, 2)
    jones = np.tile([[1.0, 0.0, 0.0, 0.0], [0.0, 0.0, 1.0, 0.0]], (n_dir, 1))
    n = 2 * n_dir
    return dict(wave_theta=th2, wave_phi=ph2, jones=jones, wave_g=np.ones(n), wave_phase=np.zeros(n),
                wave_d0=np.zeros((n, 3)))


def run_multi_rhs(args):
    """Several right-hand sides of one scene through foggy_solve_rhs: the 64-sphere cluster (the
    small workload) under 64 Fibonacci directions x 2 polarisations = 128 right-hand sides, GMRES
    to 1e-6; value = right-hand sides solved per second (device time)."""
    import torch
    from itofoggysim_b200 import scene as S, solver
    sc = S.small_cluster()
    sc = S.Scene(**{**sc.__dict__, **fibonacci_waves(64), "gmres_tolerance": 1e-6, "name": "small_cluster_64_rhs128"})
    with solver.MultiSphereSolver(sc) as s:
        for _ in range(args.warmup):
            s.solve_rhs()
        torch.cuda.synchronize()
        tot_ms, iters = 0.0, 0
        for _ in range(args.steps):
            x, cs, st = s.solve_rhs()
            tot_ms += st["ms_total"]
            iters += st["iterations"]
    nrhs = sc.n_waves
    line = {
        "metric": METRIC, "value": nrhs * args.steps / (tot_ms * 1e-3), "unit": "rhs solves/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "64-sphere cluster x 128 right-hand sides (64 Fibonacci directions "
                               "x TM/TE)", "rhs": nrhs, "gmres_tolerance": 1e-6,
                   "solver": "one GMRES per right-hand side on a shared operator and pair tables"},
        "iterations_per_rhs": iters / (args.steps * nrhs),
        "c_ext_range": [float(cs[:, 1].min()), float(cs[:, 1].max())],
    }
    print(json.dumps(line), flush=True)


def block_scene(n_spheres):
    """The 20,000-sphere 128-right-hand-side scene's shape at n_spheres: lognormal water spheres (median 0.6 um, sigma_ln 0.3,
    clipped to 0.2-1.5 um) at the number density of 20,000 spheres in a 90 um cube, 64 Fibonacci
    directions x TM/TE = 128 right-hand sides, GMRES(30) to 1e-6."""
    from itofoggysim_b200 import scene as S
    box = 90.0 * (n_spheres / 20000.0) ** (1.0 / 3.0)
    sc = S.medium_cluster(seed=4, n=n_spheres, box=box)
    return S.Scene(**{**sc.__dict__, **fibonacci_waves(64), "gmres_tolerance": 1e-6, "gmres_restart": 30,
                      "tree_l_max": 0, "name": "lognormal_%d_rhs128" % n_spheres})


def run_block(args):
    """The 128 right-hand sides of one scene solved as one block in mixed precision
    (foggy_solve_block: FP32 translation arithmetic in the Arnoldi steps, FP64 restart residuals,
    every operator application shared by the block), against the plain FP64 path (one FP64 GMRES per
    right-hand side, foggy_solve_rhs) on the same scene.  value = right-hand sides solved per second
    (device time of the block solve); errors of every right-hand side against the FP64 solutions."""
    import ctypes as C
    import torch
    from itofoggysim_b200 import _native as N, solver
    dev = torch.device("cuda", 0)
    sc = block_scene(args.spheres)
    nrhs = sc.n_waves
    # the plain FP64 path, one GMRES per right-hand side (the reference's one run per illumination)
    with solver.MultiSphereSolver(sc) as s:
        x64, cs64, st64 = s.solve_rhs()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    with solver.MultiSphereSolver(sc, precision=1) as s:
        for _ in range(args.warmup):
            s.solve_block()
        torch.cuda.synchronize()
        ms, launches, its = [], 0, []
        with ClockSampler(0) as clk:
            for _ in range(args.steps):
                flush.zero_()
                x, cs, it, be, st = s.solve_block()
                ms.append(st["ms_total"])
                launches += st["kernel_launches"]
                its.append(int(it.sum()))
            torch.cuda.synchronize()
        tiles = s.block_tiles(nrhs, precision=1)
        # the FP32 block operator alone on the 128 solutions (device buffers, CUDA events)
        xd = torch.from_numpy(np.ascontiguousarray(x).reshape(-1).view(np.float64).copy()).to(dev)
        yd = torch.empty_like(xd)
        s.L.foggy_matvec_block(s.h, nrhs, 1, C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()), N.FOGGY_MEM_DEVICE)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        N.check(s.L.foggy_matvec_block(s.h, nrhs, 1, C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()),
                                       N.FOGGY_MEM_DEVICE), s.h)
        e1.record()
        torch.cuda.synchronize()
        t_op = e0.elapsed_time(e1)
        del xd, yd
    # end to end through the public API: scene from host memory, the block solve, solutions to host
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with solver.MultiSphereSolver(sc, precision=1) as s2:
        xh, _, _, _, _ = s2.solve_block()
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3
    h2d = (sc.centres.nbytes + sc.param_index.nbytes + sc.refractive_index.nbytes + sc.radius.nbytes
           + sc.n_range_param.nbytes + 6 * 8 * nrhs)
    del flush
    torch.cuda.empty_cache()
    g = g_layout(sc)
    rel = [float(np.linalg.norm((x[r] - x64[r]) / g) / np.linalg.norm(x64[r] / g)) for r in range(nrhs)]
    cext = [float(abs(cs[r, 1] - cs64[r, 1]) / abs(cs64[r, 1])) for r in range(nrhs)]
    peak = measure_fp32_peak(torch, dev)
    flops = algorithmic_flops(sc) * nrhs
    achieved = flops / (t_op * 1e-3) / 1e12
    value = nrhs * len(ms) / (float(np.sum(ms)) * 1e-3)
    plain = nrhs / (st64["ms_total"] * 1e-3)
    p = sc.p_of_sphere()
    line = {
        "metric": METRIC, "value": value, "unit": "rhs solves/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": float(np.mean(ms)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 translations, f64 Krylov and residuals", "data": "synthetic",
        "config": {"workload": sc.name, "spheres": sc.n_spheres, "p_max": int(p.max()), "p_median": float(np.median(p)),
                   "rhs": nrhs, "gmres_restart": sc.gmres_restart, "gmres_tolerance": sc.gmres_tolerance,
                   "solver": "batched GMRES, one Krylov space per right-hand side, block operator",
                   "matvec": "direct (all pairs, rotation-axial-rotation), right-hand-side tiles per CTA",
                   "l2": "Krylov block exceeds L2; 256 MB L2 flush between steps"},
        "plain_fp64": {"rhs_per_s": plain, "ms_total": st64["ms_total"], "iterations": st64["iterations"],
                       "solver": "foggy_solve_rhs: one FP64 GMRES per right-hand side"},
        "speedup_vs_plain_fp64": value / plain,
        "iterations_total": its[-1], "max_rel_coefficient_error": max(rel), "max_c_ext_rel_error": max(cext),
        "tiles": {"fp32_per_launch": tiles[:, 3].tolist()},
        "roofline": {"bound": "fp32", "compute": "FP32 CUDA-core pipe (packed fma.rn.f32x2); no tensor-core instruction",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                     "kernel": "k_direct_block<cplxf> (one block application of 128 vectors)",
                     "flops_per_launch": flops, "ms_per_launch": t_op,
                     "peak_source": "cuBLAS FP32 SGEMM 8192^3 (TF32 off) measured in this run"},
        "e2e": {"value": nrhs / (e2e_ms * 1e-3), "unit": "rhs solves/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(xh.nbytes)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def run_operator(args):
    """Operator applications alone, for timing and ncu captures: the lognormal scene of --spheres
    (the 2000-sphere cube's volume fraction), --rhs vectors (the right-hand sides of its plane
    wave), FP64 or FP32 translations (--precision), through foggy_matvec (one vector) or
    foggy_matvec_block.  One untimed application builds the pair tables and tunes the tiles; the
    CUDA profiler is started after it, so `ncu --profile-from-start off` captures the timed ones."""
    import ctypes as C
    import torch
    from itofoggysim_b200 import _native as N, scene as S, solver
    dev = torch.device("cuda", 0)
    n = args.spheres
    sc = S.medium_cluster(n=n, box=40.0 * (n / 2000.0) ** (1.0 / 3.0))
    prec = 1 if args.precision == "mixed" else 0
    with solver.MultiSphereSolver(sc, precision=prec) as s:
        b = np.tile(s.get_vector_b(), (args.rhs, 1))
        xd = torch.from_numpy(b.reshape(-1).view(np.float64).copy()).to(dev)
        yd = torch.empty_like(xd)

        def apply():
            if args.rhs == 1 and prec == 0:
                s.matvec_device(xd.data_ptr(), yd.data_ptr())
            else:
                N.check(s.L.foggy_matvec_block(s.h, args.rhs, prec, C.c_void_p(xd.data_ptr()),
                                               C.c_void_p(yd.data_ptr()), N.FOGGY_MEM_DEVICE), s.h)

        t0 = time.perf_counter()
        apply()
        torch.cuda.synchronize()
        ms_first = (time.perf_counter() - t0) * 1e3   # wall time: pair tables, tile tuning, one application
        if args.solve:
            # one GMRES(50) solve to 1e-8 instead (mixed precision: FP32 operator in the Arnoldi steps)
            s.set_restart(50)
            s.set_tolerance(1e-8)
            torch.cuda.profiler.start()
            _, st = s.solve()
            torch.cuda.profiler.stop()
            print(json.dumps({"workload": "operator", "spheres": n, "solve": args.precision,
                              "ms_total": st["ms_total"], "iterations": st["iterations"],
                              "backward_error": st["backward_error"]}), flush=True)
            return
        torch.cuda.profiler.start()
        out = []
        for _ in range(args.applications):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            apply()
            e1.record()
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1))
        torch.cuda.profiler.stop()
    flops = algorithmic_flops(sc) * args.rhs
    print(json.dumps({"workload": "operator", "spheres": n, "rhs": args.rhs, "precision": args.precision,
                      "ms_first_application": ms_first,
                      "ms_per_application": out, "ms_per_rhs": float(np.mean(out)) / args.rhs,
                      "tflops": flops / (float(np.mean(out)) * 1e-3) / 1e12}), flush=True)


def long_wave_scene(n):
    """n water spheres of radius 0.1-0.3 um at lambda = 6 um, 0.04 spheres per um^3 (boxes a fraction
    of a wavelength to a few wavelengths), global order 8: the regime where the reference's ML-FMM
    expansion is accurate."""
    from itofoggysim_b200 import scene as S
    rng = np.random.default_rng(7)
    box = (n / 0.04) ** (1.0 / 3.0)
    return S.make_scene(rng.uniform(0.1, 0.3, n), box, 5, lambda_0=6.0, n_max=8, z_coupling=3,
                        reference_row_rule=False, name="long_wave_%d" % n)


def run_fmm_scale(args):
    """The direct operator against the ML-FMM (consistent convention, --fmm-digits per-level orders or
    the global order) on long_wave_scene(--spheres): device time per application (median of
    --applications after one untimed one) and the relative difference of the two results."""
    import torch
    from itofoggysim_b200 import solver
    dev = torch.device("cuda", 0)
    sc = long_wave_scene(args.spheres)
    out = {"workload": "fmm_scale", "spheres": args.spheres, "fmm_digits": args.fmm_digits}
    ys = {}
    for name, kw in (("direct", {}), ("mlfmm", dict(use_ml_fmm=True, fmm_convention=1, fmm_digits=args.fmm_digits))):
        with solver.MultiSphereSolver(sc, **kw) as s:
            b = s.get_vector_b()
            xd = torch.from_numpy(b.view(np.float64).copy()).to(dev)
            yd = torch.empty_like(xd)
            s.matvec_device(xd.data_ptr(), yd.data_ptr())
            torch.cuda.synchronize()
            ts = []
            for _ in range(max(1, args.applications)):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                s.matvec_device(xd.data_ptr(), yd.data_ptr())
                e1.record()
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            ys[name] = yd.cpu().numpy().view(np.complex128)
            out[name + "_ms"] = float(np.median(ts))
    out["speedup"] = out["direct_ms"] / out["mlfmm_ms"]
    out["rel_diff"] = float(np.linalg.norm(ys["mlfmm"] - ys["direct"]) / np.linalg.norm(ys["direct"]))
    print(json.dumps(out), flush=True)


def g_layout(sc):
    g = np.array([math.sqrt(math.factorial(n + m) / math.factorial(n - m))
                  for n in range(1, sc.n_range[1] + 1) for m in range(-n, n + 1)])
    return np.tile(np.concatenate([g, g]), sc.n_spheres)


def run_mixed(args):
    """The workload solved with the FP32 operator in the Arnoldi steps and FP64 true residuals
    (the 2000-sphere lognormal scene); value = solves/s (device time), with the relative error
    of the coefficients and of C_ext against one FP64 solve of the same scene.  The roofline is
    that of the FP32 operator: its mean application time is the operator time of a solve less its
    FP64 residual applications (timed in the FP64 solve), over its Arnoldi steps."""
    import torch
    from itofoggysim_b200 import solver
    dev = torch.device("cuda", 0)
    sc = workload_scene(args.workload)
    with solver.MultiSphereSolver(sc) as s:
        x64, st64 = s.solve()
        c64 = s.cross_sections(x64)
    ms64_per_mv = st64["ms_matvec"] / st64["matvecs"]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    with solver.MultiSphereSolver(sc, precision=1) as s:
        for _ in range(args.warmup):
            s.solve()
        torch.cuda.synchronize()
        ms, its, mvs, ms32, launches = [], [], [], [], 0
        with ClockSampler(0) as clk:
            for _ in range(args.steps):
                flush.zero_()
                x, st = s.solve()
                ms.append(st["ms_total"])
                its.append(st["iterations"])
                mvs.append(st["matvecs"])
                n64 = st["matvecs"] - st["iterations"]
                ms32.append((st["ms_matvec"] - n64 * ms64_per_mv) / st["iterations"])
                launches += st["kernel_launches"] + 1
            torch.cuda.synchronize()
        c = s.cross_sections(x)
    # end to end through the public API: scene from host memory, solution back to host
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with solver.MultiSphereSolver(sc, precision=1) as s2:
        xh, _ = s2.solve()
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3
    h2d = (sc.centres.nbytes + sc.param_index.nbytes + sc.refractive_index.nbytes + sc.radius.nbytes
           + sc.n_range_param.nbytes + 6 * 8 * sc.n_waves)
    del flush
    torch.cuda.empty_cache()
    peak = measure_fp32_peak(torch, dev)
    flops = algorithmic_flops(sc)
    t32 = float(np.mean(ms32))
    achieved = flops / (t32 * 1e-3) / 1e12
    line = {
        "metric": METRIC, "value": 1e3 / float(np.mean(ms)), "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": float(np.mean(ms)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 translations, f64 residuals", "data": "synthetic",
        "config": {"workload": sc.name + " mixed precision", "gmres_restart": sc.gmres_restart,
                   "gmres_tolerance": sc.gmres_tolerance,
                   "fp32_pair_tables": "tcgen05 kind::tf32 3xTF32 products (k_pair_tc), built once per handle "
                                       "before the timed solves; inside the e2e leg",
                   "l2": "Krylov basis exceeds L2; 256 MB L2 flush between steps"},
        "fp64": {"ms_per_solve": st64["ms_total"], "iterations": st64["iterations"],
                 "ms_per_operator": ms64_per_mv},
        "iterations": its[-1], "matvecs": mvs[-1], "backward_error": st["backward_error"],
        "rel_coefficient_error": float(np.linalg.norm(x - x64) / np.linalg.norm(x64)),
        "c_ext_rel_error": float(abs(c[1] - c64[1]) / abs(c64[1])),
        "roofline": {"bound": "fp32", "compute": "FP32 CUDA-core pipe (FFMA); no tensor-core instruction",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None, "kernel": "k_direct<cplxf> (+k_direct_finish)",
                     "flops_per_launch": flops, "ms_per_launch": t32,
                     "peak_source": "cuBLAS FP32 SGEMM 8192^3 (TF32 off) measured in this run (no FP32 figure "
                                    "in MEASURED_PEAKS.json)"},
        "e2e": {"value": 1e3 / e2e_ms, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(xh.nbytes)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def config_of(sc, args):
    p = sc.p_of_sphere()
    return {"workload": sc.name, "spheres": sc.n_spheres, "p_max": int(p.max()), "p_median": float(np.median(p)),
            "unknowns_ragged": sc.ragged_unknowns(),
            "matvec": ("ML-FMM, %s passes, every box at the global order" %
                       ("reference" if args.fmm_convention == 0 else "consistent") if args.operator == "mlfmm"
                       else "direct (all pairs, rotation-axial-rotation)"),
            "z_coupling": "h_n^(1)" if sc.z_coupling == 3 else "j_n", "gmres_restart": sc.gmres_restart,
            "gmres_tolerance": sc.gmres_tolerance, "rhs": 1, "parallelism": "replicas x%d" % args.gpus,
            "l2": "Krylov basis (restart+1 vectors) exceeds L2; 256 MB L2 flush between steps"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="medium", choices=["medium", "small", "serving", "multi_rhs", "block",
                                                             "operator", "fmm_scale"],
                    help="serving: a request stream through the solve server; block: 128 right-hand sides of "
                         "one lognormal scene as one mixed-precision block (their own JSON lines)")
    ap.add_argument("--spheres", type=int, default=500, help="spheres of the block and operator workloads' scenes")
    ap.add_argument("--rhs", type=int, default=1, help="vectors per application of the operator workload")
    ap.add_argument("--applications", type=int, default=2, help="timed applications of the operator workload")
    ap.add_argument("--solve", action="store_true", help="operator workload: one GMRES solve instead")
    ap.add_argument("--concurrent", type=int, default=3, help="co-resident requests of the serving workload")
    ap.add_argument("--operator", default="direct", choices=["direct", "mlfmm"],
                    help="mlfmm: the ML-FMM passes (fmm_convention below) instead of all pairs")
    ap.add_argument("--fmm-convention", type=int, default=0, choices=[0, 1])
    ap.add_argument("--fmm-digits", type=float, default=0.0,
                    help="fmm_scale workload: per-level ML-FMM orders for this many digits (0: the global order)")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU sampling")
    ap.add_argument("--matvecs-per-solve", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-cached", action="store_true",
                    help="also time the oracle with cached translation blocks (about a minute of CPU)")
    ap.add_argument("--cpu-mlfmm", action="store_true",
                    help="with --operator mlfmm: also time one application of the oracle's ML-FMM (the "
                         "reference's passes, translations recomputed exactly; minutes of CPU)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="mixed: FP32 Arnoldi operator, FP64 true residuals (its own JSON line, with errors "
                         "against an FP64 solve)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.precision == "mixed" and args.workload not in ("operator", "block", "serving"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no mixed-precision solve"}),
                  flush=True)
        elif rank == 0:
            run_mixed(args)
        return

    if args.workload == "multi_rhs":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "CPU reference arm times the single-RHS workloads"}),
                  flush=True)
        elif rank == 0:
            run_multi_rhs(args)
        return

    if args.workload == "fmm_scale":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "operator comparison mode of the GPU arm"}),
                  flush=True)
        elif rank == 0:
            run_fmm_scale(args)
        return

    if args.workload == "operator":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "operator timing mode of the GPU arm"}), flush=True)
        elif rank == 0:
            run_operator(args)
        return

    if args.workload == "block":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "CPU reference arm times the single-RHS workloads"}),
                  flush=True)
        elif rank == 0:
            run_block(args)
        return

    if args.workload == "serving":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving layer"}), flush=True)
        elif rank == 0:
            run_serving(args)
        return

    if args.impl == "reference":
        if not args.matvecs_per_solve and not MATVECS_PER_SOLVE[args.workload]:
            args.matvecs_per_solve = 1
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    from itofoggysim_b200 import solver

    sc = workload_scene(args.workload)
    fmm = args.operator == "mlfmm"
    mk = lambda: solver.MultiSphereSolver(sc, device=local, use_ml_fmm=fmm, fmm_convention=args.fmm_convention)
    s = mk()
    n = s.n
    xbuf = torch.empty(2 * n, dtype=torch.float64, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def step():
        return s.solve_device(xbuf.data_ptr())

    for _ in range(args.warmup):
        st = step()
    torch.cuda.synchronize()

    lat, mv_ms, mv_count, iters, launches = [], 0.0, 0, [], 0
    with ClockSampler(local) as clk:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e_all0 = torch.cuda.Event(enable_timing=True)
        e_all1 = torch.cuda.Event(enable_timing=True)
        total_ms = 0.0
        for _ in range(args.steps):
            flush.zero_()
            st = step()
            lat.append(st["ms_total"])
            total_ms += st["ms_total"]
            mv_ms += st["ms_matvec"]
            mv_count += st["matvecs"]
            iters.append(st["iterations"])
            launches += st["kernel_launches"] + 1
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    value, max_ms = job_rate(total_ms, args.steps, world, torch, dev, dist)
    x_dev = xbuf.cpu().numpy().view(np.complex128)
    berr = s.get_backward_error()
    tree = s.build_tree() if fmm else None
    # the timed handle's pair tables take most of HBM; free them so the end-to-end handle gets
    # the same operator path
    s.close()
    del xbuf
    torch.cuda.empty_cache()

    # end to end through the public API: scene from host memory, solution back to host
    e2e_ms = []
    h2d = 0
    for i in range(max(1, min(args.steps, 2))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with mk() as s2:
            xh, _ = s2.solve()
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    h2d = (sc.centres.nbytes + sc.param_index.nbytes + sc.refractive_index.nbytes + sc.radius.nbytes
           + sc.n_range_param.nbytes + 6 * 8 * sc.n_waves)
    d2h = xh.nbytes
    e2e_value, _ = job_rate(float(np.mean(e2e_ms)), 1, world, torch, dev, dist)

    result = None
    if rank == 0:
        peak = measure_fp64_peak(torch, dev)
        flops = (fmm_flops(sc, tree[0], tree[2], tree[3], sc.reference_row_rule) if fmm
                 else algorithmic_flops(sc))
        avg_mv = mv_ms / max(mv_count, 1)
        achieved = flops / (avg_mv * 1e-3) / 1e12
        traffic = None
        tf = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tf):
            with open(tf) as f:
                traffic = json.load(f).get(sc.name + ("_mlfmm" if fmm else ""))
        result = {
            "metric": METRIC_MLFMM if fmm else METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(sc, args),
            "latency_ms": {"p50": percentile(lat, 50), "p99": percentile(lat, 99)},
            "solve": {"iterations": iters, "matvecs_per_solve": mv_count // args.steps,
                      "backward_error": berr, "ms_operator_per_solve": mv_ms / args.steps},
            "roofline": {"bound": "fp64", "compute": "FP64 CUDA-core pipe (DFMA); no tensor-core instruction",
                         "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                         "kernel": ("k_translate (ML-FMM passes) + k_direct_finish" if fmm
                                    else "k_direct (+k_direct_finish)"), "flops_per_launch": flops,
                         "ms_per_launch": avg_mv,
                         "peak_source": "cuBLAS FP64 DGEMM 8192^3 measured in this run (no FP64 figure in "
                                        "MEASURED_PEAKS.json)"},
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        if not args.no_cpu:
            s_mv, pairs, el = cpu_sample(sc, budget_s=args.cpu_budget)
            per_solve = s_mv * (mv_count / args.steps)
            result["cpu_baseline"] = {
                "value": 1.0 / per_solve, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
                "sample": "%d random sphere pairs (%.1f s), exact Xu translations recomputed per pair as the "
                          "reference does, extrapolated x N(N-1) pairs x %d matvecs/solve"
                          % (pairs, el, mv_count // args.steps)}
        if args.cpu_cached:
            t_c, t_build, sc_small = cpu_cached_sample()
            per_solve_c = t_c * cached_scale(sc_small, sc) * (mv_count / args.steps)
            result["cpu_baseline_cached"] = {
                "value": 1.0 / per_solve_c, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
                "sample": "oracle operator with every pair's translation blocks cached "
                          "(oracle-direct-cached), %.3f s per application of the 64-sphere cluster (cache built in "
                          "%.1f s), scaled by sum_{j!=l} P_j P_l to this scene and x %d matvecs/solve; this "
                          "scene's cache (two P_j x P_l complex blocks per ordered pair) would need "
                          "%.1f GB" % (t_c, t_build, mv_count // args.steps, cached_bytes(sc) / 1e9)}
        if fmm and args.cpu_mlfmm:
            from oracle import oracle as O
            P = O.Problem(sc)
            xo = P.vector_b()
            t0 = time.perf_counter()
            P.fmm_matvec(xo, l_max=sc.tree_l_max, convention=args.fmm_convention, z_gt_r=3)
            t_f = time.perf_counter() - t0
            result["cpu_baseline_mlfmm"] = {
                "value": 1.0 / (t_f * (mv_count / args.steps)), "unit": "solves/s", "cores": os.cpu_count(),
                "kind": "port",
                "sample": "one whole application of the oracle's ML-FMM (oracle-mlfmm: the reference's "
                          "passes and lists, every translation's coefficients recomputed exactly), %.1f s, x %d "
                          "matvecs/solve" % (t_f, mv_count // args.steps)}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


if __name__ == "__main__":
    main()
