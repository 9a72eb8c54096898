"""Benchmark of the batched NUFHT on B200: forward H c plus adjoint H^T y.

Metric (the reference's headline): Gpts*cols/s = 2 (N + M) B / (t_fwd + t_adj).
Workload: nu = 0; N = M = 1e6 sources r and targets k drawn as 1000 (1 - U[0,1)) and sorted;
B = 32 columns of c ~ N(0,1) (seed 1, plus the rank); tol 1e-8.  One step = one forward
transform on (r -> k) and one adjoint transform on (k -> r) of B columns each.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--precision mixed-averaged|mixed|fp64]

Precision: mixed-averaged (default) runs the asymptotic boxes in FP32 and reports the
forward output's error against FP64 direct sums at sampled targets beside the planner's
worst-case FP32 bound (a column concentrated on one source); mixed keeps FP64 wherever that
bound exceeds tol / 4 (at tol 1e-8 this workload then runs in FP64); fp64 is the plain form.
The plain FP64 form is always timed beside a mixed one.

Under torchrun each rank transforms its own B columns with the same grids (weak scaling,
no data-path collective); the reported time is the maximum over ranks.  Rank 0 prints one
JSON line.  --impl reference times the reference's CPU path (its own planner and driver,
compiled from its sources into oracle/_ref, over the oracle's evaluators) on the host cores.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gpts*cols/s fwd+adjoint at tol 1e-8, mixed vs plain FP64 GPU, vs host CPU"
UNIT = "Gpts*cols/s"


def make_inputs(N, M, B, seed):
    rng = np.random.default_rng(1)
    r = np.sort(1000.0 * (1.0 - rng.random(N)))
    k = np.sort(1000.0 * (1.0 - rng.random(M)))
    crng = np.random.default_rng(1 + seed)
    c = crng.standard_normal((B, N))  # column t = row t (column-major N x B)
    y = crng.standard_normal((B, M))
    return r, k, c, y


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
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
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_from_profiles(kernel):
    """DRAM bytes per launch of `kernel` at this workload from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic_cfg2.json")) as f:
            t = json.load(f)
        return t.get(kernel)
    except Exception:
        return None


class StdoutToStderr:
    """Route C-level writes to stdout (the reference prints when it loads its tables) to
    stderr, so that stdout carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def run_cpu_reference(N, M, B_sample, runs, threads):
    """The reference's CPU path: oracle/_ref (the reference's own planner and nufht_batch,
    compiled from its sources, over the oracle's evaluators with the type-3 NUFFT), or the
    oracle's restatement of the driver when oracle/_ref is absent, on `threads` host threads.
    Planning (once per direction) is outside the timed region, as the reference's benchmark
    notebook times nufht_batch.  Returns (seconds per fwd+adj step of each run, kind)."""
    import oracle
    oracle.set_threads(threads)
    r, k, c, y = make_inputs(N, M, B_sample, 0)
    cF = np.asfortranarray(c.T)
    yF = np.asfortranarray(y.T)
    kind = "reference" if oracle.ref_available() else "port"
    if kind == "reference":
        from nufht_b200 import _lib as L
        R = oracle.ref()
        R.oracle_set_type3_mode(oracle.T3_NUFFT)
        R.oracle_set_threads(threads)
        plans = []
        for (a, b) in ((r, k), (k, r)):
            p = L.NufhtPlan()
            opt = R.nufht_default_options()
            opt.tol = 1e-8
            rc = R.nufht_plan_init(ctypes.byref(p), 0.0, a.ctypes.data_as(ctypes.c_void_p), len(a),
                                   b.ctypes.data_as(ctypes.c_void_p), len(b), ctypes.byref(opt))
            assert rc == 0, rc
            plans.append(p)
        gF = np.zeros((M, B_sample), order="F")
        hF = np.zeros((N, B_sample), order="F")

        def step():
            R.nufht_batch(ctypes.byref(plans[0]), cF.ctypes.data_as(ctypes.c_void_p), N,
                          gF.ctypes.data_as(ctypes.c_void_p), M, B_sample, None)
            R.nufht_batch(ctypes.byref(plans[1]), yF.ctypes.data_as(ctypes.c_void_p), M,
                          hF.ctypes.data_as(ctypes.c_void_p), N, B_sample, None)
    else:
        def step():
            oracle.nufht_batch(0.0, r, k, cF, 1e-8, mode=oracle.T3_NUFFT)
            oracle.nufht_batch(0.0, k, r, yF, 1e-8, mode=oracle.T3_NUFFT)
    times = []
    for _ in range(runs):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    if kind == "reference":
        for p in plans:
            R.nufht_plan_free(ctypes.byref(p))
    return times, kind


def cpu_baseline_leg(N, M, B, runs):
    """CPU baseline of the workload on this box's host: the reference's path on all host
    threads (OpenMP over columns and the 2(K+1) type-3 transforms of a box; `value`) and on
    one thread (faithful to the reference, whose only parallel construct is a critical
    section and whose FINUFFT calls run with nthreads = 1), each the median of `runs` steps
    of forward + adjoint on a sample of the columns."""
    cores = os.cpu_count() or 1
    B_all = max(1, min(B, 8))
    with StdoutToStderr():
        t_all, kind = run_cpu_reference(N, M, B_all, runs, cores)
        t_one, _ = run_cpu_reference(N, M, 1, runs, 1)
    v_all = 2.0 * (N + M) * B_all / statistics.median(t_all) / 1e9
    v_one = 2.0 * (N + M) * 1 / statistics.median(t_one) / 1e9
    return {"value": v_all, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": "%d of %d columns of the workload, fwd+adj, median of %d steps, planning excluded; "
                      "type-3 transforms by the oracle's NUFFT (eps = tol) in place of FINUFFT" % (B_all, B, runs),
            "runs_s": t_all,
            "single_thread": {"value": v_one, "unit": UNIT, "cores": 1, "kind": kind,
                              "sample": "1 of %d columns, fwd+adj, median of %d steps" % (B, runs),
                              "runs_s": t_one}}


def batch_problems(rng, count, nmax=100_000):
    """The batching workload: `count` independent transforms with nu in {0, 1/2, 1, 2, 7/2, 10},
    N and M log-uniform integers in [1e3, nmax], r and k uniform on (0, R] and (0, K] with R, K
    log-uniform in [10, 1e3], 1-16 columns of N(0,1), tol in {1e-4, 1e-8, 1e-12}."""
    out = []
    for _ in range(count):
        nu = float(rng.choice([0.0, 0.5, 1.0, 2.0, 3.5, 10.0]))
        N = int(10.0 ** rng.uniform(3, np.log10(nmax)))
        M = int(10.0 ** rng.uniform(3, np.log10(nmax)))
        R = 10.0 ** rng.uniform(1, 3)
        K = 10.0 ** rng.uniform(1, 3)
        r = np.sort(R * (1.0 - rng.random(N)))
        k = np.sort(K * (1.0 - rng.random(M)))
        B = int(rng.integers(1, 17))
        tol = float(rng.choice([1e-4, 1e-8, 1e-12]))
        out.append((nu, r, k, B, tol, rng.standard_normal((B, N))))
    return out


def batch_figure(dev, st, steps):
    """256 independent transforms (the batching workload) in one CUDA-graph launch, against the
    same plans launched one after another on one stream: Gpts*cols/s = sum (N + M) B / t for one
    (forward) transform of every problem, device time with CUDA events."""
    import torch
    from nufht_b200 import DevicePlan
    from nufht_b200.batch import TransformBatch
    probs = batch_problems(np.random.default_rng(4), 256)
    t0 = time.perf_counter()
    plans = [DevicePlan(nu, r, k, tol) for nu, r, k, B, tol, c in probs]
    plan_s = time.perf_counter() - t0
    items = [(p, torch.tensor(c, device=dev)) for p, (nu, r, k, B, tol, c) in zip(plans, probs)]
    outs = [torch.empty((c.shape[0], p.n), dtype=torch.float64, device=dev) for p, c in items]
    t0 = time.perf_counter()
    tb = TransformBatch(items)
    create_s = time.perf_counter() - t0
    work = float(sum((len(r) + len(k)) * B for nu, r, k, B, tol, c in probs))

    def timed(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    def sequential():
        for (p, c), o in zip(items, outs):
            p.execute_columns(c, o, st)

    ms_graph = timed(lambda: tb.launch(st), steps)
    ms_seq = timed(sequential, max(1, steps // 2))
    info = tb.info()
    tb.close()
    for p in plans:
        p.close()
    return {"workload": "256 transforms: nu in {0,1/2,1,2,7/2,10}, N,M log-uniform in [1e3,1e5], "
                        "R,K log-uniform in [10,1e3], 1-16 columns, tol in {1e-4,1e-8,1e-12}; one forward each",
            "unit": UNIT, "value": work / (ms_graph * 1e-3) / 1e9, "ms": ms_graph,
            "sequential": {"value": work / (ms_seq * 1e-3) / 1e9, "ms": ms_seq},
            "graph_over_sequential": ms_seq / ms_graph, "branches": info["branches"],
            "kernel_nodes": info["kernel_nodes"], "planning_s": plan_s, "batch_create_s": create_s}


def planning_figure(dev):
    """Planning cost (host wall-clock, device-side box partition) of this workload's forward
    plan (1e6 x 1e6, nu = 0, tol 1e-8) and of the 4e6 x 4e6 order-100 stress grids, beside
    the first and a later transform of 32 columns."""
    import torch
    from nufht_b200 import DevicePlan
    out = {}
    rng = np.random.default_rng(1)
    r = np.sort(1000.0 * (1.0 - rng.random(1_000_000)))
    k = np.sort(1000.0 * (1.0 - rng.random(1_000_000)))
    rng = np.random.default_rng(100)
    n = 4_000_000
    means = np.array([200.0, 800.0, 1500.0])
    rr = np.sort(np.clip(np.abs(rng.normal(means[rng.integers(0, 3, n)], 50.0)), 1e-9, 2000.0))
    kk = np.sort(2000.0 * (1.0 - rng.random(n)))
    for name, a, b, nu, kw in (("1e6_nu0", r, k, 0.0, {}), ("4e6_nu100", rr, kk, 100.0, {"extended_tables": True})):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        p = DevicePlan(nu, a, b, 1e-8, mixed="averaged", **kw)
        torch.cuda.synchronize(dev)
        create_ms = (time.perf_counter() - t0) * 1e3
        st = p.stats()
        c = torch.randn((32, len(a)), dtype=torch.float64, device=dev)
        times = []
        for _ in range(3):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            p.execute_columns(c)
            torch.cuda.synchronize(dev)
            times.append((time.perf_counter() - t0) * 1e3)
        out[name] = {"plan_create_ms": create_ms, "partition_ms": st[15], "work_lists_ms": st[16],
                     "tables_upload_ms": st[17], "partition_on_device": bool(st[18]),
                     "first_transform_ms": times[0], "transform_ms": min(times[1:])}
        p.close()
        del c
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="mixed-averaged", choices=["fp64", "mixed", "mixed-averaged"])
    ap.add_argument("--n", type=int, default=1000000)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the batching and planning figures")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    N = M = args.n
    B = args.batch
    tol = 1e-8
    workload = "nu=0, N=M=%d uniform on (0,1000], batch %d, tol 1e-8, forward + adjoint" % (N, B)
    config = {"workload": workload, "nu": 0, "N": N, "M": M, "batch_per_gpu": B, "tol": tol,
              "global_batch": B * world, "precision": args.precision,
              "parallelism": "dp%d (independent column blocks per GPU, no collective)" % world,
              "l2": "inputs larger than L2 (c %d MB, y %d MB; NUFFT grids and records larger still)"
                    % (8 * N * B // 2**20, 8 * M * B // 2**20)}
    cores = os.cpu_count() or 1

    if args.impl == "reference":
        if rank != 0:
            return
        cpu = cpu_baseline_leg(N, M, B, 3)
        value = cpu["value"]
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
                "steps": 3, "warmup": 0, "ms_per_step": 2.0 * (N + M) * min(B, 8) / value / 1e6,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded numpy draws with the workload's shapes)", "config": config,
                "cpu_baseline": cpu,
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=dev)
        pg = True
    from nufht_b200 import DevicePlan
    from nufht_b200 import _lib as L
    lib = L.lib()
    mixed_arg = {"fp64": False, "mixed": True, "mixed-averaged": "averaged"}[args.precision]
    r, k, c_h, y_h = make_inputs(N, M, B, rank)
    pf = DevicePlan(0.0, r, k, tol, mixed=mixed_arg, device=local)
    pa = DevicePlan(0.0, k, r, tol, mixed=mixed_arg, device=local)
    mixed = bool(pf.info()["mixed"])  # asymptotic boxes in FP32
    c = torch.tensor(c_h, device=dev)
    y = torch.tensor(y_h, device=dev)
    g = torch.empty((B, M), dtype=torch.float64, device=dev)
    h = torch.empty((B, N), dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream(dev)

    def step():
        pf.execute_columns(c, g, st)
        pa.execute_columns(y, h, st)

    def barrier():
        if pg:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(max(args.warmup, 3)):
        step()
    barrier()
    launches0 = lib.nufht_b200_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(st)
        for _ in range(args.steps):
            step()
        e1.record(st)
        barrier()
    launches = lib.nufht_b200_launch_count() - launches0
    ms = e0.elapsed_time(e1) / args.steps
    if pg:
        t = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    value = 2.0 * (N + M) * B * world / (ms * 1e-3) / 1e9

    # The plain FP64 form of the same method on the same inputs, for the mixed/FP64 ratio.
    fp64 = None
    if args.precision != "fp64":
        qf = DevicePlan(0.0, r, k, tol, mixed=False, device=local)
        qa = DevicePlan(0.0, k, r, tol, mixed=False, device=local)

        def step64():
            qf.execute_columns(c, g, st)
            qa.execute_columns(y, h, st)

        for _ in range(max(args.warmup, 3)):
            step64()
        barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(st)
        for _ in range(args.steps):
            step64()
        f1.record(st)
        barrier()
        ms64 = f0.elapsed_time(f1) / args.steps
        if pg:
            t = torch.tensor([ms64], device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms64 = float(t.item())
        fp64 = {"value": 2.0 * (N + M) * B * world / (ms64 * 1e-3) / 1e9, "ms_per_step": ms64,
                "mixed_over_fp64": ms64 / ms}
        qf.close()
        qa.close()

    # Per-kernel device times over a second run of the same steps (CUDA events on the
    # launching stream around each phase), for the roofline of the dominant kernel.
    lib.nufht_b200_set_phase_timing(1)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize(dev)
    lib.nufht_b200_set_phase_timing(0)
    phases = {kk: v / args.steps for kk, v in L.phase_times().items()}

    # End to end through the reference-facing C ABI: nufht_plan_init / nufht_batch with host
    # buffers (pinned), the copies inside the timed region.  The precision of that entry
    # point is chosen with NUFHT_B200_PRECISION (read when a plan first runs).
    os.environ["NUFHT_B200_PRECISION"] = args.precision
    plans = []
    for (a, b) in ((r, k), (k, r)):
        p = L.NufhtPlan()
        opt = L.options(tol=tol)
        assert lib.nufht_plan_init(ctypes.byref(p), 0.0, L.dptr(a), len(a), L.dptr(b), len(b), ctypes.byref(opt)) == 0
        plans.append(p)
    cp = torch.tensor(c_h).pin_memory()
    yp = torch.tensor(y_h).pin_memory()
    gp = torch.empty((B, M), dtype=torch.float64).pin_memory()
    hp = torch.empty((B, N), dtype=torch.float64).pin_memory()

    def e2e_step():
        rc1 = lib.nufht_batch(ctypes.byref(plans[0]), ctypes.c_void_p(cp.data_ptr()), N,
                              ctypes.c_void_p(gp.data_ptr()), M, B, None)
        rc2 = lib.nufht_batch(ctypes.byref(plans[1]), ctypes.c_void_p(yp.data_ptr()), M,
                              ctypes.c_void_p(hp.data_ptr()), N, B, None)
        assert rc1 == 0 and rc2 == 0

    for _ in range(2):
        e2e_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    barrier()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if pg:
        t = torch.tensor([e2e_s], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    for p in plans:
        lib.nufht_plan_free(ctypes.byref(p))
    e2e = {"value": 2.0 * (N + M) * B * world / e2e_s / 1e9, "unit": UNIT,
           "h2d_bytes_per_step": 8 * (N * B + M * B), "d2h_bytes_per_step": 8 * (M * B + N * B),
           "api": "nufht_plan_init + nufht_batch (C ABI) on pinned host buffers"}

    # Roofline of the dominant kernel (the phase with the largest device time).
    hbm, hbm_kind = peaks()
    sf = np.zeros(21)
    sa = np.zeros(21)
    lib.nufht_b200_plan_stats(pf._h, sf.ctypes.data_as(L.c_double_p), 21)
    lib.nufht_b200_plan_stats(pa._h, sa.ctypes.data_as(L.c_double_p), 21)
    V = sf[10] * B
    gb = 8.0 if mixed else 16.0  # bytes per complex grid value (FP32 / FP64)
    ev = gb / 2  # bytes per value of the arithmetic type
    # algorithmic bytes per fwd+adj step (both plans): spreading reads the source records and
    # each box's packed coefficients and writes the grid (the packing pass reads c once and
    # writes its packed copy); interpolation reads the grid cells its stencils reach and the
    # target records, and adds one value per target and column into g
    npts = {id(sf): N, id(sa): M}
    byts = {
        "asy_spread": sum(s[19] + ev * s[0] * B + gb * s[2] * V + (8.0 + ev) * npts[id(s)] * B for s in (sf, sa)),
        "asy_fft": sum(2 * gb * s[2] * V for s in (sf, sa)),
        "asy_interp": sum(gb * s[8] * V + s[20] + 8.0 * s[1] * B for s in (sf, sa)),
    }
    flops = {
        "asy_spread": sum(4.0 * s[3] * V for s in (sf, sa)),
        "asy_interp": sum(4.0 * s[4] * V for s in (sf, sa)),
        "dir": sum(2.0 * s[5] * B for s in (sf, sa)),
    }
    dom = max(phases, key=lambda kk: phases[kk])
    kname = {"asy_spread": "k_asy_spread", "asy_interp": "k_asy_interp", "asy_fft": "cufft",
             "dir": "k_dir", "loc_proj": "k_loc_proj", "loc_eval": "k_loc_eval", "zero": "memset"}[dom]
    fp64_peak = ctypes.c_double(0.0)
    lib.nufht_b200_fp64_peak(ctypes.byref(fp64_peak))
    t_dom = phases[dom] * 1e-3  # per step (2 launches: forward and adjoint plan)
    ach_gbs = byts.get(dom, 0.0) / t_dom / 1e9 if t_dom > 0 else 0.0
    roofline = {"kernel": kname, "bound": "hbm", "achieved": ach_gbs, "peak": hbm, "unit": "GB/s",
                "frac": ach_gbs / hbm, "peak_source": hbm_kind + " (MEASURED_PEAKS.json hbm_gbs)"
                if hbm_kind == "measured" else "fallback",
                "traffic": traffic_from_profiles(kname),
                "algorithmic_bytes_per_launch": byts.get(dom, 0.0) / 2,
                "avg_launch_ms": phases[dom] / 2}
    if dom in flops and (not mixed or dom == "dir"):
        ach_tf = flops[dom] / t_dom / 1e12
        roofline["fp64"] = {"achieved": ach_tf, "peak": fp64_peak.value, "unit": "TFLOP/s",
                            "frac": ach_tf / fp64_peak.value if fp64_peak.value > 0 else None,
                            "peak_source": "measured FP64 FMA probe (nufht_b200_fp64_peak)"}
    elif dom in flops:
        # single-precision spreading / interpolation: issue-bound on packed FP32 FMAs
        fp32_peak = ctypes.c_double(0.0)
        lib.nufht_b200_fp32_peak(ctypes.byref(fp32_peak))
        ach_tf = flops[dom] / t_dom / 1e12
        roofline["fp32"] = {"achieved": ach_tf, "peak": fp32_peak.value, "unit": "TFLOP/s",
                            "frac": ach_tf / fp32_peak.value if fp32_peak.value > 0 else None,
                            "peak_source": "measured FP32 packed-FMA probe (nufht_b200_fp32_peak)"}

    # Accuracy of this run's forward output: error against the oracle's exact FP64 direct sums
    # (every source, no expansion, Kahan-compensated, on the host cores; the checker, outside
    # every timed region) at 64 sampled targets, per column over ||c_t||_1, beside the
    # planner's worst-case bound for FP32 rounding (per ||c||_1).
    import oracle
    oracle.set_threads(cores)
    pf.execute_columns(c, g, st)
    torch.cuda.synchronize(dev)
    idx = np.sort(np.random.default_rng(7).choice(M, 64, replace=False))
    ex = oracle.direct_sum(0.0, r, k, c_h.T, idx)
    got = g[:, torch.tensor(idx, device=dev)].cpu().numpy().T
    err = float((np.abs(got - ex).max(axis=0) / np.abs(c_h).sum(axis=1)).max())
    accuracy = {"max_err_over_l1": err, "over_tol": err / tol, "targets_sampled": 64,
                "reference": "oracle FP64 direct sums (all sources, host) at sampled targets of the forward transform",
                "fp32_worst_case_bound_over_l1": float(pf.stats()[14]) if mixed else None}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_leg(N, M, B, 3)

    extra = None
    if rank == 0 and world == 1 and not args.no_extra:
        extra = {"batch_256": batch_figure(dev, st, args.steps), "planning": planning_figure(dev)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if not mixed else "f32/f64",
                "data": "synthetic (seeded numpy draws with the workload's shapes)", "config": config,
                "clocks": clk.summary(), "e2e": e2e, "gpu_launches": int(launches),
                "phases_ms_per_step": phases, "roofline": roofline, "cpu_baseline": cpu,
                "fp64_form": fp64, "accuracy": accuracy, "plan": pf.info(), "extra": extra}
        print(json.dumps(line))
    pf.close()
    pa.close()
    if pg:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
