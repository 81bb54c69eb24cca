"""Benchmark: n = 2^20 H-matvec GB/s on one B200 (the large 1-D H-matvec
workload: uniform grid on [0,10], Cauchy kernel 1/(1+(x-y)^2), MaxBlock 512,
MinBlock 64, MaxRank 16, ACA tolerance 1e-8, N(0,1) right-hand side).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One step = one single-RHS H-matvec y = H x through the library.  `value` is
the algorithmic bytes of a matvec (every stored factor and dense entry once,
plus x and y) divided by the device time of a step, inputs resident in HBM;
the factor pool (~100 GB in FP64) is far larger than L2, so no flush is
needed between steps.  `e2e` is the same metric through hm_matvec with host
(pinned) buffers, the 8 MB host->device copy of x and device->host copy of y
inside the timed region.

Multi-GPU (--gpus N): one H of n = 2^20 row-sharded over the ranks (strong
scaling): every rank builds and multiplies only its rows (shards balanced by
the bytes they stream), and one NCCL all-gather of the row shards leaves the
full H*x on every rank each step; the job time is the max over ranks.
--replicas runs N independent copies instead (weak scaling).

--impl reference times the reference algorithm's CPU path (the C restatement
of hmat_matvec! in oracle/, FP64, all host threads) on a bounded sample of
the same workload: the leaves touching a band of rows, built by the same
restatement of aca2.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "hmatrix.jl_b200"))

METRIC = "n=2^20 H-matvec GB/s"
UNIT = "GB/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--storage", default="f64", choices=["f64", "f32", "bf16"])
    ap.add_argument("--no-precisions", action="store_true",
                    help="skip the FP32 / BF16 factor legs (single RHS and tensor-core multi-RHS)")
    ap.add_argument("--no-kmeans", action="store_true", help="skip the matvec on the reference's KMeans tree")
    ap.add_argument("--no-c4", action="store_true", help="skip the gradient (adjoint) leg")
    ap.add_argument("--c4-n", type=int, default=1 << 17, help="size of the gradient leg")
    ap.add_argument("--c5", action="store_true",
                    help="also run the 2-D point-cloud leg (mixed H-LU, GMRES-based refinement, adjoint solve)")
    ap.add_argument("--c5-n", type=int, default=1 << 18, help="size of the 2-D leg")
    ap.add_argument("--c5-eps-lu", type=float, default=1e-8,
                    help="LU truncation of the 2-D leg (1e-6 breaks the LU down at n=2^18: below 1e-3/|H| only)")
    ap.add_argument("--cpu-rows", type=int, default=4096, help="rows of the CPU baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-lu", action="store_true", help="skip the H-LU + solve leg")
    ap.add_argument("--lu-n", type=int, default=1 << 16, help="size of the H-LU + solve leg")
    ap.add_argument("--rhs", default="16,64",
                    help="column counts of the multi-RHS matvec leg (comma separated; empty to skip)")
    ap.add_argument("--replicas", action="store_true",
                    help="with --gpus N > 1: N independent copies of H instead of row shards of one H")
    ap.add_argument("--batch", type=int, default=256,
                    help="problems of the batched uneven H-LU + solve leg (0: skip)")
    ap.add_argument("--batch-nthreads", type=int, default=0, help="host threads of the batched calls (0: auto)")
    return ap.parse_args()


def workload(n):
    return {"workload": "large 1-D H-matvec, n=%d uniform grid on [0,10]" % n, "n": n,
            "kernel": "1/(1+(x-y)^2)", "MaxBlock": 512, "MinBlock": 64, "MaxRank": 16,
            "aca_tol": 1e-8, "cons": "aca2 (Adj=I)", "tree": "median bisection",
            "rhs": "1 column N(0,1), seed 1",
            "l2": "no flush: inputs (factor pool) far larger than the 126 MB L2"}


# --------------------------------------------------------------------------
# clocks sampled during the timed region
# --------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the first query initialises NVML, which can hold the driver for a
            # while: let it finish before anything is timed
            t0 = time.time()
            while not self.lines and time.time() - t0 < 10 and self.proc.poll() is None:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        self.m0 = 0

    def mark(self):
        """Start of the timed region: samples before it are not reported."""
        self.m0 = len(self.lines)

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        use = self.lines[self.m0:] or self.lines[-1:]
        for ln in use:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_byte():
    """DRAM bytes per algorithmic byte of each matvec phase from the committed
    ncu summary (profiles/matvec_traffic.json), if present."""
    try:
        with open(os.path.join(ROOT, "profiles", "matvec_traffic.json")) as f:
            return json.load(f)
    except Exception:
        return None


# --------------------------------------------------------------------------
# CPU baseline: the C restatement of aca2 + hmat_matvec! on a band of rows
# --------------------------------------------------------------------------
def cpu_sample_gbs(n, rows, target_s=12.0, max_reps=200, nthreads=0):
    from hmatrix.cluster import construct_cluster
    from oracle.hm_oracle_c import Sample
    c = construct_cluster(np.linspace(0, 10, n), 64, "bisect")
    tree = {"s": c.s, "e": c.e, "left": c.left, "right": c.right}
    r0 = n // 2 - rows // 2
    S = Sample(1, 1.0, c.X, tree, 64, 512, 16, 1e-8, r0, r0 + rows, nthreads=nthreads)
    x = np.random.default_rng(1).standard_normal(n)
    S.matvec(x)
    t0 = time.perf_counter()
    reps = 0
    while reps < max_reps:
        S.matvec(x)
        reps += 1
        if time.perf_counter() - t0 > target_s:
            break
    dt = (time.perf_counter() - t0) / reps
    gbs = S.bytes_per_matvec() / dt / 1e9
    return gbs, S.threads, ("leaves of the %d rows [%d,%d) of the n=%d matrix (%d leaves, %.2f GB FP64), "
                            "%d matvecs" % (rows, r0, r0 + rows, n, len(S.lv), 8 * S.stored / 1e9, reps)), dt


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    gbs, thr, sample, dt = cpu_sample_gbs(a.n, a.cpu_rows, target_s=max(2.0, 0.5 * a.steps))
    # each step: one matvec of the sample (bounded), reported as GB/s
    line = {"metric": METRIC, "value": gbs, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak" if a.replicas else "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload(a.n),
            "impl": "reference",
            "cpu_baseline": {"value": gbs, "unit": UNIT, "cores": thr, "kind": "port", "sample": sample},
            "e2e": {"value": gbs, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------
def build(n, storage, shard=None):
    """The benchmark H-matrix; with shard = (rank, world), this rank's row shard."""
    import hmatrix as hm
    prm = hm.Params(Geom=np.linspace(0, 10, n), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64,
                    MaxRank=16, ConsMethod="aca2", εComp=1e-8, Tree="bisect",
                    Storage={"f64": hm.F64, "f32": hm.F32, "bf16": hm.BF16}[storage],
                    Device=int(os.environ.get("LOCAL_RANK", "0")))
    t0 = time.perf_counter()
    if shard is not None:
        from hmatrix.shard import ShardedHmat
        S = ShardedHmat(prm, shard[0], shard[1])
        S.H.shard = S
        return S.c, S.H, time.perf_counter() - t0
    c, H = hm.NewHmat(prm)
    return c, H, time.perf_counter() - t0


def job_time(ms_local, dist, device):
    """Time of the whole job: the max over ranks of each rank's own time (the
    job ends when the slowest replica does).  `device` is "cuda" under NCCL
    and "cpu" under gloo."""
    if dist is None:
        return ms_local
    import torch
    t = torch.tensor([ms_local], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(bytes_per_rank, world, ms):
    """Whole-job throughput in GB/s: every rank streams its own replica."""
    return world * bytes_per_rank / (ms * 1e-3) / 1e9


def measure(H, a, torch, dist, world, shard=False):
    import ctypes as C
    from hmatrix import _lib
    L = _lib.lib()
    n = H.n
    dev = torch.cuda.current_device()
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randn(n, generator=g, device="cuda", dtype=torch.float64)
    y = torch.empty_like(x)
    st = torch.cuda.current_stream()
    sp = C.c_void_p(st.cuda_stream or 1)   # torch's default stream is cudaStreamLegacy
    flags = _lib.HM_FLAG_DEVICE_PTRS

    from hmatrix.shard import gather_rows

    def step():
        _lib.check(L.hm_matvec(H._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), 1, 0, flags, sp))
        if shard:                            # every rank's rows -> the full H*x on every rank
            gather_rows(y, H.shard.splits, H.shard.rank, dist)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    # per-phase device times (events between the launches)
    ms3 = (C.c_float * 3)()
    ph = np.zeros(3)
    for _ in range(3):
        _lib.check(L.hm_matvec_profile(H._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), 0, sp, ms3))
        ph += np.array(ms3[:])
    ph /= 3
    clocks = Clocks(dev)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for _ in range(2):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.mark()
    e0.record(st)
    for _ in range(a.steps):
        step()
    e1.record(st)
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = job_time(e0.elapsed_time(e1) / a.steps, dist, "cuda")
    if dist is not None:
        dist.barrier()
    # end to end with host pinned buffers: through the C ABI's host-pointer path
    # on one GPU; with shards, x copied in, the shard's matvec, the all-reduce
    # and y copied out, every step
    xh = x.cpu().pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    xd, yd = torch.empty_like(x), torch.empty_like(x)

    def e2e_step():
        if not shard:
            _lib.check(L.hm_matvec(H._h, C.c_void_p(xh.data_ptr()), C.c_void_p(yh.data_ptr()), 1, 0, 0, None))
            return
        xd.copy_(xh, non_blocking=True)
        _lib.check(L.hm_matvec(H._h, C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()), 1, 0, flags, sp))
        gather_rows(yd, H.shard.splits, H.shard.rank, dist)
        yh.copy_(yd, non_blocking=True)
        torch.cuda.synchronize()
    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ke = max(3, a.steps // 2)
    for _ in range(ke):
        e2e_step()
    e2e_ms = job_time((time.perf_counter() - t0) / ke * 1e3, dist, "cuda")
    # accuracy: 4096 sampled rows against exact FP64 kernel rows (dense oracle)
    rows = np.sort(np.random.default_rng(2).choice(n, 4096, replace=False))
    ex = H.exact_rows(rows, x.cpu().numpy())
    got = y.cpu().numpy()[rows]
    rel = float(np.linalg.norm(got - ex) / np.linalg.norm(ex))
    return ms, ph, ck, e2e_ms, rel


def multi_rhs_leg(H, cols, steps, torch, bytes_1, exact_rows=False):
    """H*X for X of c N(0,1) columns (seed 1): device time per call (CUDA
    events over `steps` calls after 3 warm-up calls), the factor bytes
    streamed per second, the equivalent single-column rate (c x the bytes
    of one column's matvec per second), and the agreement with the
    single-column kernel on the first and last columns.  FP32/BF16 factors
    run on the tensor cores; exact_rows adds the error of the first column
    against exact FP64 kernel rows (the dense FullMat oracle, 1024 rows)."""
    import ctypes as C
    from hmatrix import _lib
    L = _lib.lib()
    st = torch.cuda.current_stream()
    sp = C.c_void_p(st.cuda_stream or 1)
    info = H.info()
    out = {}
    for c in cols:
        g = torch.Generator(device="cuda").manual_seed(1)
        X = torch.randn(c, H.n, generator=g, device="cuda", dtype=torch.float64)   # column-major n x c
        Y = torch.empty_like(X)

        def step():
            _lib.check(L.hm_matvec(H._h, C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()), c, 0,
                                   _lib.HM_FLAG_DEVICE_PTRS, sp))
        for _ in range(3):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            step()
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        y1 = torch.empty(H.n, device="cuda", dtype=torch.float64)
        err = 0.0
        for j in (0, c - 1):
            _lib.check(L.hm_matvec(H._h, C.c_void_p(X[j].data_ptr()), C.c_void_p(y1.data_ptr()), 1, 0,
                                   _lib.HM_FLAG_DEVICE_PTRS, sp))
            torch.cuda.synchronize()
            err = max(err, float(torch.linalg.norm(Y[j] - y1) / torch.linalg.norm(y1)))
        flops = 2.0 * c * (info.rk_entries + info.dense_entries)
        out[str(c)] = {"ms": ms, "factor_GB/s": bytes_1 / (ms * 1e-3) / 1e9,
                       "equiv_single_column_GB/s": c * bytes_1 / (ms * 1e-3) / 1e9,
                       "GFLOP/s": flops / (ms * 1e-3) / 1e9, "rel_diff_vs_single_column": err}
        if exact_rows:
            from hmatrix import _lib as _l
            rows = np.sort(np.random.default_rng(2).choice(H.n, 1024, replace=False))
            ex = H.exact_rows(rows, X[0].cpu().numpy())
            out[str(c)]["rel_err_vs_exact_fp64_rows"] = float(np.linalg.norm(Y[0].cpu().numpy()[rows] - ex)
                                                               / np.linalg.norm(ex))
            _l.check(L.hm_status(H._h, sp))
        del X, Y
        torch.cuda.empty_cache()
    return out


def lu_solve_leg(n, torch):
    """H-LU + H\\y on the largest problem of the batched 1-D configuration
    (n points on [0,10], 1/(1+(x-y)^2) + delta_xy, MaxBlock 256, MinBlock 32,
    MaxRank 12, one N(0,1) right-hand side): the FP64 factorisation as in the
    reference (eps_trunc 1e-10) against a cheaper low-accuracy factorisation
    (eps_trunc 1e-3 inside the LU: the fastest total of a sweep over 1e-6 .. 1e-2
    at this size), both refined with the FP64 H-matvec to a
    relative residual <= 1e-10."""
    import hmatrix as hm
    out = {"config": {"n": n, "kernel": "1/(1+(x-y)^2) + delta_xy", "MaxBlock": 256, "MinBlock": 32,
                      "MaxRank": 12, "aca_tol": 1e-10, "target_relres": 1e-10, "tree": "median bisection"}}
    y = np.random.default_rng(3).standard_normal(n)
    # one small untimed factorisation and solve first: the library's one-time
    # set-up (module loading, cuBLAS handles) stays out of the timed legs
    wprm = hm.Params(Geom=np.linspace(0, 10, 4096), Kernel=hm.Cauchy(1.0), MaxBlock=256, MinBlock=32,
                     MaxRank=12, ConsMethod="aca2", εComp=1e-10, Tree="bisect", Shift=1.0,
                     Device=torch.cuda.current_device())
    wc, wH = hm.NewHmat(wprm)
    wH.lu_()
    wH.solve_refined(np.ones(4096), tol=1e-10, max_iter=5)
    del wH
    for name, epslu in (("fp64", 0.0), ("mixed", 1e-3)):
        prm = hm.Params(Geom=np.linspace(0, 10, n), Kernel=hm.Cauchy(1.0), MaxBlock=256, MinBlock=32,
                        MaxRank=12, ConsMethod="aca2", εComp=1e-10, Tree="bisect", Shift=1.0, εTruncLU=epslu,
                        Device=torch.cuda.current_device())
        c, H = hm.NewHmat(prm)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L = hm.lu(H)
        t1 = time.perf_counter()
        x, it, rr = L.solve_refined(y, tol=1e-10, max_iter=20)
        t2 = time.perf_counter()
        r = H * x - y
        out[name] = {"lu_s": t1 - t0, "solve_refined_s": t2 - t1, "total_s": t2 - t0, "refine_steps": it,
                     "relres": float(np.linalg.norm(r) / np.linalg.norm(y)), "eps_trunc_lu": epslu or 1e-10}
        del L, H
        torch.cuda.empty_cache()
    out["mixed_speedup"] = out["fp64"]["total_s"] / out["mixed"]["total_s"]
    return out


LU_CPU_N = 8192          # bounded size of the CPU H-LU sample (the oracle takes ~3 s there)


def lu_params(n):
    """Parameters of the H-LU legs: n points on [0,10], MaxBlock 256, MinBlock 32,
    MaxRank 12, aca2 at 1e-10, median-bisection tree (kernel and shift apart)."""
    return dict(Geom=np.linspace(0, 10, n), MaxBlock=256, MinBlock=32, MaxRank=12, ConsMethod="aca2",
                εComp=1e-10, Tree="bisect")


def oracle_lu_sample(n):
    """The reference's lu! and \\ (src/hlu.jl:465-562) as restated in FP64 numpy by
    the oracle, timed on the host cores (numpy's BLAS on every thread) on the LU
    leg's matrix at a bounded size n: 1/(1+(x-y)^2) + I, no refinement."""
    import os
    from oracle import hm_oracle as O
    y = np.random.default_rng(3).standard_normal(n)
    prm = O.Params(Kernel=O.kernel_cauchy(), **lu_params(n))
    _, H = O.NewHmat(prm)
    H = O.add_identity(H, 1.0)
    t0 = time.perf_counter()
    L = O.lu(H, prm)
    t1 = time.perf_counter()
    x = O.solve(L, y)
    t2 = time.perf_counter()
    rr = float(np.linalg.norm(O.matvec(H, x) - y) / np.linalg.norm(y))
    try:
        cores = len(os.sched_getaffinity(0))
    except Exception:
        cores = os.cpu_count() or 1
    return {"n": n, "lu_s": t1 - t0, "solve_s": t2 - t1, "total_s": t2 - t0, "relres": rr, "cores": cores,
            "kind": "port", "sample": "lu! + \\ of the FP64 oracle (numpy/BLAS) at n=%d" % n}


def lu_cpu_beside_gpu(n, torch):
    """The CPU sample of oracle_lu_sample next to the GPU's FP64 lu(H) + H\\y of the
    same matrix (no refinement on either side)."""
    import hmatrix as hm
    cpu = oracle_lu_sample(n)
    y = np.random.default_rng(3).standard_normal(n)
    _, H = hm.NewHmat(hm.Params(Kernel=hm.Cauchy(1.0), Shift=1.0, Device=torch.cuda.current_device(),
                                **lu_params(n)))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L = hm.lu(H)
    t1 = time.perf_counter()
    x = L.solve(y)
    t2 = time.perf_counter()
    rr = float(np.linalg.norm(H * x - y) / np.linalg.norm(y))
    gpu = {"n": n, "lu_s": t1 - t0, "solve_s": t2 - t1, "total_s": t2 - t0, "relres": rr}
    return {"cpu": cpu, "gpu": gpu, "gpu_speedup": cpu["total_s"] / gpu["total_s"]}


def batched_problems(count, seed=3, nmin=2 ** 10, nmax=2 ** 16):
    """The batched uneven 1-D problems: n = round(2^U(log2 nmin, log2 nmax)),
    points sorted U[0, L] with L ~ U[5, 20], K = 1/(1+((x-y)/l)^2) + delta_xy
    with l ~ U[0.5, 2], one N(0,1) right-hand side each."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(2 ** rng.uniform(np.log2(nmin), np.log2(nmax))))
        L = rng.uniform(5, 20)
        ell = rng.uniform(0.5, 2)
        x = np.sort(rng.uniform(0, L, n))
        out.append((x, ell, rng.standard_normal(n)))
    return out


def oracle_batch_sample(count, budget_s=15.0, nmax=8192):
    """The oracle's FP64 lu! + \\ (src/hlu.jl:465-562, numpy BLAS on every host
    thread) on a bounded sample of the batched problems: in problem order, those
    of n <= nmax, until budget_s of CPU time is spent; per-problem times, no
    refinement."""
    import os
    from oracle import hm_oracle as O
    rows = []
    spent = 0.0
    for i, (x, ell, y) in enumerate(batched_problems(count)):
        if len(x) > nmax:
            continue
        prm = O.Params(Geom=x, Kernel=O.kernel_cauchy(ell), MaxBlock=256, MinBlock=32, MaxRank=12,
                       ConsMethod="aca2", εComp=1e-10, Tree="bisect")
        _, H = O.NewHmat(prm)
        H = O.add_identity(H, 1.0)
        t0 = time.perf_counter()
        L = O.lu(H, prm)
        xs = O.solve(L, y)
        dt = time.perf_counter() - t0
        rr = float(np.linalg.norm(O.matvec(H, xs) - y) / np.linalg.norm(y))
        rows.append({"problem": i, "n": len(x), "s": dt, "relres": rr})
        spent += dt
        if spent >= budget_s:
            break
    try:
        cores = len(os.sched_getaffinity(0))
    except Exception:
        cores = os.cpu_count() or 1
    return rows, cores


def batch_cpu_beside_gpu(count, torch):
    """The CPU sample of oracle_batch_sample next to the GPU's FP64 lu(H) + H\\y of
    the same problems, one at a time (no refinement on either side)."""
    import hmatrix as hm
    rows, cores = oracle_batch_sample(count)
    probs = batched_problems(count)
    gpu_total = 0.0
    for r in rows:
        x, ell, y = probs[r["problem"]]
        prm = hm.Params(Geom=x, Kernel=hm.Cauchy(ell), MaxBlock=256, MinBlock=32, MaxRank=12,
                        ConsMethod="aca2", εComp=1e-10, Tree="bisect", Shift=1.0,
                        Device=torch.cuda.current_device())
        _, H = hm.NewHmat(prm)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L = hm.lu(H)
        xs = L.solve(y)
        dt = time.perf_counter() - t0
        r["gpu_s"] = dt
        r["gpu_relres"] = float(np.linalg.norm(H * xs - y) / np.linalg.norm(y))
        gpu_total += dt
        del L, H
    cpu_total = sum(r["s"] for r in rows)
    return {"kind": "port", "cores": cores, "problems": rows, "cpu_total_s": cpu_total, "gpu_total_s": gpu_total,
            "gpu_speedup": cpu_total / gpu_total if gpu_total > 0 else None,
            "sample": "lu! + \\ of the FP64 oracle (numpy/BLAS) on the first %d batched problems of n <= 8192 "
                      "(about 15 s of host time), beside the GPU's FP64 lu(H) + H\\y of the same problems" % len(rows)}


def batch_leg(count, torch, nthreads=0, budget_gb=90.0, rank=0, world=1, dist=None):
    """All problems factored (lu!) and solved with FP64 refinement to a
    relative residual <= 1e-10 through the batched entry points, in waves
    whose factor memory (about 2.5 n^2 bytes a problem) fits the budget.
    Timed: factorisation + refined solve of every problem (host right-hand
    sides in, solutions out); construction is not timed.  With world > 1 the
    problems are split over the ranks by predicted cost (no exchange between
    ranks); the job time is the max over ranks."""
    import hmatrix as hm
    from hmatrix.shard import problem_cost, split_problems
    probs = batched_problems(count)
    mine = split_problems([problem_cost(len(p[0]), 256) for p in probs], world)[rank]
    waves, cur, acc = [], [], 0.0
    for i in mine:
        x = probs[i][0]
        need = 2.5 * len(x) ** 2 / 1e9
        if cur and acc + need > budget_gb:
            waves.append(cur)
            cur, acc = [], 0.0
        cur.append(i)
        acc += need
    if cur:
        waves.append(cur)
    out = {"config": {"problems": count, "sum_n": int(sum(len(p[0]) for p in probs)),
                      "n_range": [int(min(len(p[0]) for p in probs)), int(max(len(p[0]) for p in probs))],
                      "kernel": "1/(1+((x-y)/l)^2) + delta_xy", "MaxBlock": 256, "MinBlock": 32, "MaxRank": 12,
                      "aca_tol": 1e-10, "target_relres": 1e-10, "tree": "median bisection", "waves": len(waves),
                      "host_threads": nthreads or "auto",
                      "split": ("%d ranks by predicted cost, no exchange" % world) if world > 1 else "1 GPU"}}
    dev = "cuda" if dist is not None and dist.get_backend() == "nccl" else "cpu"
    for name, epslu in (("fp64", 0.0), ("mixed", 1e-6)):
        t_all, worst, steps = 0.0, 0.0, 0
        if dist is not None:
            dist.barrier()
        for w in waves:
            Hs, ys = [], []
            for i in w:
                x, ell, y = probs[i]
                prm = hm.Params(Geom=x, Kernel=hm.Cauchy(ell), MaxBlock=256, MinBlock=32, MaxRank=12,
                                ConsMethod="aca2", εComp=1e-10, Tree="bisect", Shift=1.0, εTruncLU=epslu,
                                Device=torch.cuda.current_device())
                Hs.append(hm.NewHmat(prm)[1])
                ys.append(y)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            hm.lu_batch_(Hs, nthreads)
            xs, it, rr = hm.solve_refined_batch(Hs, ys, tol=1e-10, max_iter=20, nthreads=nthreads)
            t_all += time.perf_counter() - t0
            worst = max(worst, float(rr.max()))
            steps = max(steps, int(it.max()))
            del Hs, xs
            torch.cuda.empty_cache()
        t_all = job_time(t_all * 1e3, dist, dev) * 1e-3
        worst = job_time(worst, dist, dev)              # max over ranks
        steps = int(job_time(float(steps), dist, dev))
        out[name] = {"total_s": t_all, "max_relres": worst, "max_refine_steps": steps,
                     "eps_trunc_lu": epslu or 1e-10}
    out["mixed_speedup"] = out["fp64"]["total_s"] / out["mixed"]["total_s"]
    return out


def kmeans_leg(a, torch, peak):
    """The large 1-D matvec on the reference's own cluster tree: KMeans
    bisection (src/cluster.jl:196-256, the same sklearn call, subtrees on a
    pool of host processes), FP64 factors.  The tree build and the H-matrix
    construction are timed apart from the matvec."""
    import hmatrix as hm
    from hmatrix.cluster import construct_cluster
    n = a.n
    t0 = time.perf_counter()
    c = construct_cluster(np.linspace(0, 10, n), 64, "kmeans")
    t_tree = time.perf_counter() - t0
    prm = hm.Params(Geom=np.linspace(0, 10, n), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64, MaxRank=16,
                    ConsMethod="aca2", εComp=1e-8, Device=torch.cuda.current_device())
    t0 = time.perf_counter()
    H = hm.new_on_cluster(prm, c)
    t_build = time.perf_counter() - t0
    info = H.info()
    _, tune_choice = H.autotune(1, calls=3)
    ms, ph, ck, e2e_ms, rel = measure(H, a, torch, None, 1)
    bytes_mv = 8 * info.rk_entries + 8 * info.dense_entries + 16 * n
    sz = c.e - c.s
    leaf = c.left < 0
    gbs = bytes_mv / (ms * 1e-3) / 1e9
    out = {"tree": "kmeans (src/cluster.jl:196-256)", "tree_s": t_tree, "build_s": t_build,
           "leaf_clusters": int(leaf.sum()), "leaf_sizes": [int(sz[leaf].min()), int(sz[leaf].max())],
           "n_rk": info.n_rk, "n_dense": info.n_dense, "rk_entries": info.rk_entries,
           "dense_entries": info.dense_entries, "max_rank": info.max_rank, "algorithmic_bytes": bytes_mv,
           "ms_per_matvec": ms, "GB/s": gbs, "frac_of_peak": gbs / peak, "phase_ms": [float(v) for v in ph],
           "e2e_GB/s": bytes_mv / (e2e_ms * 1e-3) / 1e9, "rel_err_vs_exact_fp64_rows": rel, "clocks": ck,
           "autotune": tune_choice}
    del H
    torch.cuda.empty_cache()
    return out


def gradient_leg(n, torch):
    """The differentiation configuration: n points on [0,10], Gaussian kernel
    exp(-(x-y)^2/(2 l^2)) + sigma2 I with l = 0.7, sigma2 = 1e-2, MaxRank 24,
    ACA tolerance 1e-10, b ~ N(0,1), loss L = b'(H\b) + |H b|^2.  Gradients
    in b, l and sigma2 from the adjoint kernels (transposed matvec, transposed
    solve on the stored LU, H-matrix of dK/dl), checked against central finite
    differences of the H-path loss (step 1e-6 for l and sigma2; the H-matrices
    at l +- h reuse the pivots of H, so their factors move smoothly with l)."""
    import hmatrix as hm
    from hmatrix.autodiff import KernelOperator

    def prm(ell=0.7, s2=1e-2, keep=False):
        return hm.Params(Geom=np.linspace(0, 10, n), Kernel=hm.Gauss(ell), MaxBlock=512, MinBlock=64, MaxRank=24,
                         ConsMethod="aca2", εComp=1e-10, Tree="bisect", Shift=s2, KeepPivots=keep,
                         Device=torch.cuda.current_device())

    def loss(op, bb):
        with torch.no_grad():
            t = torch.tensor(bb, device="cuda")
            return float(torch.dot(t, op.solve(t)) + torch.sum(op.matvec(t) ** 2))

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    op = KernelOperator(prm(keep=True), refine_tol=1e-13)
    t_build = time.perf_counter() - t0
    b0 = np.random.default_rng(4).standard_normal(n)
    b = torch.tensor(b0, device="cuda", requires_grad=True)
    t0 = time.perf_counter()
    L = torch.dot(b, op.solve(b)) + torch.sum(op.matvec(b) ** 2)
    L.backward()
    torch.cuda.synchronize()
    t_grad = time.perf_counter() - t0
    gb, gl, gs = b.grad.cpu().numpy(), float(op.p.grad), float(op.sigma2.grad)
    d = np.random.default_rng(5).standard_normal(n)
    hb = 1e-3
    fd_b = (loss(op, b0 + hb * d) - loss(op, b0 - hb * d)) / (2 * hb)
    h = 1e-6
    fd_s = (loss(KernelOperator(prm(s2=1e-2 + h), cluster=op.c, refine_tol=1e-13), b0)
            - loss(KernelOperator(prm(s2=1e-2 - h), cluster=op.c, refine_tol=1e-13), b0)) / (2 * h)
    fd_l = (loss(KernelOperator(prm(ell=0.7 + h), like=op, refine_tol=1e-13), b0)
            - loss(KernelOperator(prm(ell=0.7 - h), like=op, refine_tol=1e-13), b0)) / (2 * h)
    return {"config": {"n": n, "kernel": "exp(-(x-y)^2/(2 l^2)) + sigma2 I", "l": 0.7, "sigma2": 1e-2,
                       "MaxRank": 24, "aca_tol": 1e-10, "loss": "b'(H\\b) + |H b|^2", "fd_step": h,
                       "tree": "median bisection"},
            "loss": float(L.detach()), "build_s": t_build, "forward_backward_s": t_grad,
            "grad_l": gl, "fd_l": fd_l, "rel_err_l": abs(fd_l - gl) / abs(gl),
            "grad_sigma2": gs, "fd_sigma2": fd_s, "rel_err_sigma2": abs(fd_s - gs) / abs(gs),
            "rel_err_b_directional": abs(fd_b - gb @ d) / abs(gb @ d),
            "target": 1e-6}


def c5_leg(n, eps_lu, torch):
    """The 2-D point cloud: n points i.i.d. uniform in [0,1]^2 (seed 5), coordinate
    bisection, 1/(1+|x-y|^2) + 1e-3 I, MaxBlock 512, MinBlock 64, MaxRank 32, ACA
    tolerance 1e-9, 8 N(0,1) right-hand sides.  Mixed-precision H-LU (truncation
    eps_lu: FP32 recompression cores from 1e-6 on), then GMRES-based refinement
    (compensated FP64 residual, GMRES preconditioned by the H-LU) to a relative
    residual <= 1e-10, then the adjoint (transposed) solve the same way.  The
    errors against the dense FP64 oracle are measured on 1024 sampled rows of
    K + 1e-3 I (exact kernel rows)."""
    import hmatrix as hm
    rng = np.random.default_rng(5)
    G = rng.uniform(0, 1, (n, 2))
    prm = hm.Params(Geom=G, Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64, MaxRank=32, ConsMethod="aca2",
                    εComp=1e-9, Tree="bisect", Shift=1e-3, εTruncLU=eps_lu, Device=torch.cuda.current_device())
    t0 = time.perf_counter()
    c, H = hm.NewHmat(prm)
    t_build = time.perf_counter() - t0
    info = H.info()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    try:
        L = hm.lu(H)
    except hm.HmError as e:
        # a truncation above 1e-3/|H| perturbs the Schur complements by more
        # than the shift: a diagonal tile loses its pivots
        return {"config": {"n": n, "eps_trunc_lu": eps_lu}, "build_s": t_build,
                "lu_error": str(e)[:300], "lu_s_until_error": time.perf_counter() - t0}
    t_lu = time.perf_counter() - t0
    B = rng.standard_normal((n, 8))
    rows = np.sort(np.random.default_rng(7).choice(n, 1024, replace=False))
    out = {"config": {"n": n, "kernel": "1/(1+|x-y|^2) + 1e-3 I", "MaxBlock": 512, "MinBlock": 64, "MaxRank": 32,
                      "aca_tol": 1e-9, "eps_trunc_lu": eps_lu, "rhs": 8, "tree": "coordinate bisection",
                      "refinement": "GMRES-IR (compensated residual, GMRES(30) preconditioned by the H-LU)"},
           "build_s": t_build, "lu_s": t_lu, "n_rk": info.n_rk, "max_rank": info.max_rank,
           "lu_tiles": L.info().lu_tiles, "fp32_core": eps_lu >= 1e-6}
    for name, trans in (("solve", False), ("adjoint_solve", True)):
        t0 = time.perf_counter()
        worst, steps, dense_err = 0.0, 0, 0.0
        for j in range(B.shape[1]):
            x, it, rr = hm.gmres_ir(H, L, B[:, j], tol=1e-10, trans=trans)
            worst = max(worst, rr)
            steps = max(steps, it)
            if not trans:
                ex = H.exact_rows(rows, x)            # rows of (K + 1e-3 I) x, FP64 dense oracle
                dense_err = max(dense_err, float(np.linalg.norm(ex - B[rows, j]) / np.linalg.norm(B[rows, j])))
        out[name] = {"s": time.perf_counter() - t0, "max_relres": worst, "max_outer_steps": steps}
        if not trans:
            out[name]["rel_residual_vs_dense_rows"] = dense_err
    del L, H
    torch.cuda.empty_cache()
    return out


def run_ours(a):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    import hmatrix as hm
    shard = world > 1 and not a.replicas
    c, H, t_build = build(a.n, a.storage, (rank, world) if shard else None)
    info = H.info()
    # launch shapes from the autotuner, on this matrix (untimed)
    tune_table, tune_choice = H.autotune(1, calls=5)
    ms, ph, ck, e2e_ms, rel = measure(H, a, torch, dist, world, shard)
    eb = {"f64": 8, "f32": 4, "bf16": 2}[a.storage]
    deb = 8 if a.storage == "f64" else 4
    bytes_mv = eb * info.rk_entries + deb * info.dense_entries + 16 * a.n
    if shard:
        # strong scaling: one H over all ranks; its bytes are the sum of the shards'
        tb = torch.tensor([float(eb * info.rk_entries + deb * info.dense_entries)], device="cuda")
        dist.all_reduce(tb)
        bytes_mv = float(tb.item()) + 16 * a.n
        value = bytes_mv / (ms * 1e-3) / 1e9
        e2e = bytes_mv / (e2e_ms * 1e-3) / 1e9
    else:
        value = job_value(bytes_mv, world, ms)
        e2e = job_value(bytes_mv, world, e2e_ms)
    peak, peak_kind = peaks()
    # dominant kernel: the phase with the larger device time; its algorithmic
    # bytes: phase 1 streams the B factors (+x segments from L2), phase 2 the
    # A factors, the dense leaves, and writes y.
    half_rk = eb * info.rk_entries / 2.0
    p_bytes = [24.0 * a.n, half_rk, half_rk + deb * info.dense_entries + 8 * a.n]
    dom = int(np.argmax(ph))
    dom_name = ["xcopy", "mv_phase1_kernel", "mv_phase2_kernel"][dom]
    achieved = p_bytes[dom] / (ph[dom] * 1e-3) / 1e9
    tr = traffic_per_byte()
    traffic = None
    if tr and dom_name in tr:
        traffic = tr[dom_name] * p_bytes[dom]
    multi = None
    cols = [int(v) for v in a.rhs.split(",") if v.strip()]
    if cols and world == 1:
        multi = multi_rhs_leg(H, cols, max(3, min(a.steps, 10)), torch, bytes_mv)
    extra = {}
    if not a.no_precisions and world == 1:
        # FP32 / BF16 factors: single-RHS matvec (FP32 partial sums) and the
        # tensor-core multi-RHS product, each against exact FP64 rows
        for s in ("f32", "bf16"):
            if s == a.storage:
                continue
            del H
            H = None
            torch.cuda.empty_cache()
            _, H2, tb2 = build(a.n, s)
            i2 = H2.info()
            ms2, ph2, _, _, rel2 = measure(H2, a, torch, None, 1)
            eb2 = {"f32": 4, "bf16": 2}[s]
            b2 = eb2 * i2.rk_entries + 4 * i2.dense_entries + 16 * a.n
            extra[s] = {"GB/s": b2 / (ms2 * 1e-3) / 1e9, "ms_per_step": ms2, "frac_of_peak": b2 / (ms2 * 1e-3) / 1e9 / peak,
                        "rel_err_4096_rows": rel2, "phase_ms": [float(v) for v in ph2], "build_s": tb2}
            if cols:
                tuned = {}
                for cc in cols:                 # the tensor-core column block for each width
                    tt, ch = H2.autotune(cc, calls=3)
                    tuned[str(cc)] = {"choice": ch["tc_nc"], "ms": {k: v for k, v in tt.items() if k.startswith("tc_")}}
                extra[s]["autotune"] = tuned
                mr = multi_rhs_leg(H2, cols, max(3, min(a.steps, 10)), torch, b2, exact_rows=True)
                for v in mr.values():
                    # the factors stream once per call: the HBM floor is their bytes
                    v["frac_of_hbm_floor"] = v["factor_GB/s"] / peak
                extra[s]["multi_rhs_tensor_cores"] = mr
            del H2
            torch.cuda.empty_cache()
    lu = None
    if not a.no_lu and world == 1:
        H = None
        torch.cuda.empty_cache()
        lu = lu_solve_leg(a.lu_n, torch)
        if not a.no_cpu:
            try:
                lu["cpu_baseline"] = lu_cpu_beside_gpu(LU_CPU_N, torch)
            except Exception as e:          # the CPU sample never costs the bench line
                lu["cpu_baseline"] = {"error": repr(e)[:300]}
    batch = None
    if a.batch > 0:
        H = None
        torch.cuda.empty_cache()
        batch = batch_leg(a.batch, torch, a.batch_nthreads, rank=rank, world=world, dist=dist)
        if not a.no_cpu and world == 1:
            try:
                batch["cpu_baseline"] = batch_cpu_beside_gpu(a.batch, torch)
            except Exception as e:          # the CPU sample never costs the bench line
                batch["cpu_baseline"] = {"error": repr(e)[:300]}
            torch.cuda.empty_cache()
    c5 = None
    if a.c5 and world == 1:
        H = None
        torch.cuda.empty_cache()
        c5 = c5_leg(a.c5_n, a.c5_eps_lu, torch)
    c4 = None
    if not a.no_c4 and world == 1:
        H = None
        torch.cuda.empty_cache()
        c4 = gradient_leg(a.c4_n, torch)
    # the KMeans-tree matrix (180 GB of FP64 factors at n = 2^20) last: run
    # before the H-LU legs it left the FP64 factorisation timed at twice its
    # time in a fresh process
    kmeans = None
    if not a.no_kmeans and world == 1:
        H = None
        torch.cuda.empty_cache()
        kmeans = kmeans_leg(a, torch, peak)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    cpu = None
    if not a.no_cpu and world == 1:
        gbs, thr, sample, _ = cpu_sample_gbs(a.n, a.cpu_rows)
        cpu = {"value": gbs, "unit": UNIT, "cores": thr, "kind": "port", "sample": sample}
        try:                                # the reference's own mode: one thread
            g1, _, s1, _ = cpu_sample_gbs(a.n, a.cpu_rows, target_s=4.0, nthreads=1)
            cpu["single_thread"] = {"value": g1, "unit": UNIT, "cores": 1, "sample": s1}
        except Exception as e:
            cpu["single_thread"] = {"error": repr(e)[:300]}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak" if a.replicas else "strong",
            "vs_baseline": None, "dtype": a.storage, "data": "synthetic",
            "config": dict(workload(a.n), storage=a.storage, parallelism=("%d row shards, NCCL all-gather of y" % world) if shard
                        else ("replicas" if world > 1 else "1 GPU")),
            "clocks": ck,
            "autotune": {"choice": tune_choice, "single_column_ms": tune_table},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * a.n, "d2h_bytes_per_step": 8 * a.n,
                    "ms_per_step": e2e_ms},
            "gpu_launches": 3 * a.steps,
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "algorithmic_bytes": p_bytes[dom], "ms": float(ph[dom])},
            "matvec_frac_of_peak": value / world / peak,
            "phase_ms": [float(v) for v in ph],
            "cpu_baseline": cpu,
            "accuracy": {"rel_err_vs_exact_fp64_rows": rel, "rows": 4096},
            "structure": {"n_rk": info.n_rk, "n_dense": info.n_dense, "rk_entries": info.rk_entries,
                          "dense_entries": info.dense_entries, "max_rank": info.max_rank,
                          "algorithmic_bytes": bytes_mv, "build_s": t_build},
            "multi_rhs": multi,
            "reduced_precision": extra or None,
            "kmeans_tree": kmeans,
            "gradients": c4,
            "point_cloud_2d": c5,
            "lu_solve": lu,
            "batched_lu_solve": batch}
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
