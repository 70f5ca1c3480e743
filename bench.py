#!/usr/bin/env python
"""Benchmark: time to an FP64 true relative residual ||b - A x|| / ||b|| <=
1e-8 on one B200, BiCGSTAB(4) on the 3D convection-diffusion 7-point upwind
stencil, 128^3 grid (n = 2,097,152, nnz = 14,581,760), b = A x_true with
x_true ~ U[-1, 1] (seed 1).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Our arm prints one JSON line:
  value        time-to-solution (s) of the headline solve with A, b, x
               resident in HBM (CUDA events on the launching stream, max over
               ranks); the headline solve is the best available GPU mode,
               named in config.mode, and the plain FP64 GPU solve is reported
               beside it (plain_fp64_s);
  e2e          the same solve through the public bksp.h call with host
               arrays (upload of the CSR operator, b and x0 from pinned host
               memory and download of x inside the timed region);
  roofline     the SpMV kernel (dominant kernel) timed alone with CUDA events
               over the same operator, algorithmic bytes / duration vs the
               measured HBM copy bandwidth;
  cpu_baseline the reference (aldente39/bksp compiled from source with gcc +
               OpenBLAS, oracle/_ref) on this host's cores, one full solve.
  modes        every GPU mode with its time, iterations, FP64 true residual
               and relative error against x_true;
With --gpus N > 1 each rank solves its own replica (one system does not
shard without a halo exchange per product and an all-reduce per dot):
value is the max over ranks.

--impl reference times the reference CPU implementation instead: each step
runs a bounded number of outer iterations; value = measured time per outer
iteration x the iteration count of one full reference solve (run once,
untimed, in warm-up).
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

T0 = time.perf_counter()


def log(msg):
    """Progress on stderr (stdout carries only the JSON line)."""
    print(f"[bench {time.perf_counter() - T0:7.1f} s] {msg}", file=sys.stderr, flush=True)


METRIC = "time to 1e-8 FP64 true residual: learned-precond mixed vs plain FP64, same B200"
TOL_TRUE = 1e-8
L_DEG = 4
NX = 128


def args_():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--nx", type=int, default=NX)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--workload", default="convdiff3d",
                   choices=["convdiff3d", "kappa_batch", "configs", "complex",
                            "spmv_general"],
                   help="kappa_batch: the batched workload (64 kappa-diffusion "
                        "systems, BiCGSTAB(2)); configs: the other survey "
                        "configurations through the bksp.h calls; complex: "
                        "the complex solvers against the compiled reference's; "
                        "spmv_general: every SpMV kernel on the benchmark "
                        "operator under a random symmetric permutation (no "
                        "diagonal form); "
                        "each prints one JSON line of its own")
    p.add_argument("--batch-count", type=int, default=64)
    p.add_argument("--reference-solve-worker", action="store_true",
                   help=argparse.SUPPRESS)
    p.add_argument("--x-out", default=None, help=argparse.SUPPRESS)
    p.add_argument("--complex-reference-worker", default=None,
                   help=argparse.SUPPRESS)
    p.add_argument("--profile", default=None,
                   choices=["plain_fp64", "mixed_none", "mixed_learned", "spmv",
                            "block_cg", "persist_cg", "zbicgstabl", "spmv_perm"],
                   help="profiling driver: set up, run one warm solve, then "
                        "one solve (or SpMV launches) between "
                        "cudaProfilerStart/Stop, print nothing else")
    return p.parse_args()


def usable_cores():
    """Host cores this process may run on: its CPU affinity, capped by a
    cgroup CPU quota (containers often see every core of the machine but
    may use only a share; more OpenMP/BLAS threads than that thrash)."""
    try:
        n = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        n = os.cpu_count() or 1
    quota = None
    try:
        with open("/sys/fs/cgroup/cpu.max") as f:
            q, per = f.read().split()[:2]
            if q != "max":
                quota = float(q) / float(per)
    except (OSError, ValueError):
        try:
            with open("/sys/fs/cgroup/cpu/cpu.cfs_quota_us") as f:
                q = float(f.read())
            with open("/sys/fs/cgroup/cpu/cpu.cfs_period_us") as f:
                per = float(f.read())
            if q > 0:
                quota = q / per
        except (OSError, ValueError):
            quota = None
    if quota is not None:
        n = min(n, max(1, int(quota)))
    return max(1, n)


def reference_full_solve(nx, timeout, x_out=None):
    """One full reference dbicgstabl solve (oracle/_ref) on usable_cores()
    threads, in a child process bounded by `timeout` seconds; the child
    writes its solution to `x_out` (.npy) when given.  Returns
    (seconds, ret, cores) or (None, reason, cores)."""
    cores = usable_cores()
    env = dict(os.environ, OPENBLAS_NUM_THREADS=str(cores), OMP_NUM_THREADS=str(cores))
    cmd = [sys.executable, os.path.abspath(__file__),
           "--reference-solve-worker", "--nx", str(nx)]
    if x_out:
        cmd += ["--x-out", x_out]
    try:
        out = subprocess.run(cmd, env=env, capture_output=True, text=True,
                             timeout=timeout)
        d = json.loads(out.stdout.strip().splitlines()[-1])
        return d["s"], d["ret"], cores
    except subprocess.TimeoutExpired:
        return None, f"timed out after {timeout} s", cores
    except (ValueError, IndexError, KeyError) as e:
        return None, f"failed: {e}", cores


def reference_solve_worker(nx, x_out=None):
    from oracle import ref as R
    rp, c, v, n, b, _ = problem(nx)
    A = R.Matrix(rp, c, v, n)
    t0 = time.perf_counter()
    ret, outs, _ = R.call("dbicgstabl", A, b, L_DEG, TOL_TRUE, 10000, np.zeros(n))
    dt = time.perf_counter() - t0
    x = outs[-1]
    if x_out:
        np.save(x_out, x)
    print(json.dumps({"s": dt, "ret": int(ret)}), flush=True)
    return 0


def problems_module():
    """bksp_b200/problems.py loaded by file path: the synthetic-problem
    generators are plain NumPy, and importing them through the package would
    load the CUDA library (the package's __init__ does), which the
    reference arm's process must not map."""
    import importlib.util
    name = "_bksp_problems"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(ROOT, "bksp_b200", "problems.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def problem(nx):
    """The operator (CSR), b = A x_true and x_true."""
    P = problems_module()
    rp, c, v, n = P.convdiff3d(nx)
    xt = P.uniform(n, 1)
    b = P.csr_matvec(rp, c, v, xt)
    return rp, c, v, n, b, xt


def workload_config(nx, n, nnz):
    return {"workload": f"bicgstabl{L_DEG}_convdiff3d_{nx}^3",
            "n": n, "nnz": nnz, "l": L_DEG, "tol_true_residual": TOL_TRUE,
            "rhs": "b = A x_true, x_true ~ U[-1,1] seed 1",
            "l2": ("solve inputs larger than L2 (FP64 CSR %.0f MB); kernel timings "
                   "after a 384 MB write + read of a flush buffer before each launch")
                  % ((nnz * 12 + 4 * n) / 1e6),
            "parallelism": "replicas"}


# ----------------------------------------------------------- reference arm

def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cores = usable_cores()
    os.environ["OPENBLAS_NUM_THREADS"] = str(cores)
    os.environ["OMP_NUM_THREADS"] = str(cores)
    # Full solve once (warm-up, untimed, child process bounded in time): the
    # reference's iteration count.
    full_s, ret_full, cores = reference_full_solve(a.nx, timeout=420)
    if full_s is None:
        print(json.dumps({"impl": "reference",
                          "unavailable": f"reference full solve {ret_full} "
                                         f"on {cores} host threads"}), flush=True)
        return 0
    iters_full = ret_full + 1 if ret_full >= 0 else 10000
    from oracle import ref as R
    rp, c, v, n, b, _ = problem(a.nx)
    A = R.Matrix(rp, c, v, n)
    sample = 8
    for _ in range(max(a.warmup - 1, 0)):
        R.call("dbicgstabl", A, b, L_DEG, 1e-300, sample, np.zeros(n))
    times = []
    for _ in range(a.steps):
        t0 = time.perf_counter()
        R.call("dbicgstabl", A, b, L_DEG, 1e-300, sample, np.zeros(n))
        times.append(time.perf_counter() - t0)
    per_iter = float(np.mean(times)) / sample
    value = per_iter * iters_full
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * float(np.mean(times)), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(a.nx, n, int(rp[-1])),
        "cpu_baseline": {"value": value, "unit": "s", "cores": cores,
                         "kind": "reference",
                         "sample": f"{sample} outer iterations per step, "
                                   f"extrapolated: per-iteration time x the "
                                   f"{iters_full} iterations of one full "
                                   f"solve ({full_s:.1f} s wall, ret {ret_full})"},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "reference_full_solve_s": full_s,
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ our arm

class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,"
         "clocks.mem")

    def __init__(self, index):
        self.index = index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.p is None:
            return
        time.sleep(0.25)
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
            out, _ = self.p.communicate()
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.rows.append(f)

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if r[5 + i].lower() == "active"})
        mem = [float(r[9]) for r in self.rows
               if len(r) > 9 and r[9].replace(".", "").isdigit()]
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "mem_mhz": float(np.median(mem)) if mem else None,
                "samples": len(self.rows)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def run_ours(a):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    import bksp_b200 as B

    rp, c, v, n, b_h, xt_h = problem(a.nx)
    nnz = int(rp[-1])
    Ah = B.CsrMatrix(rp, c, v)
    G = B.GpuMatrix(Ah, B.FP32)
    log(f"operator uploaded (n={n}, nnz={nnz}, variant {G.variant()})")
    dev = torch.device("cuda", local)
    b = torch.from_numpy(b_h).to(dev)
    xt = torch.from_numpy(xt_h).to(dev)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    # A dedicated (non-default) stream: the library orders its work on it and
    # the CUDA events below are recorded on it.
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def plain_step(method=None):
        def f():
            x.zero_()
            return G.solve(B.BICGSTABL_FAST if method is None else method,
                           b.data_ptr(), x.data_ptr(), TOL_TRUE, 10000,
                           l=L_DEG, stream=sp)
        return f

    def timed(step, k):
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ms, last = [], None
        for _ in range(k):
            ev0.record(stream)
            last = step()
            ev1.record(stream)
            ev1.synchronize()
            ms.append(ev0.elapsed_time(ev1))
        return ms, last

    def max_over_ranks(val):
        if world == 1:
            return val
        t = torch.tensor([val], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # Learned preconditioner: trained once on small systems of the same
    # family (setup, outside the timed region); the MLP inference that turns
    # the operator's rows into M runs inside every timed solve.
    from bksp_b200 import problems as P
    t0 = time.perf_counter()
    model = B.SpaiModel(seed=3)
    train_mats = [B.GpuMatrix(B.CsrMatrix(*P.convdiff3d(nt)[:3]), B.FP32)
                  for nt in (12, 16, 24)]
    train_loss = model.train(train_mats, epochs=200, probes=8, lr=3e-3, seed=7)
    for m_ in train_mats:
        m_.close()
    train_s = time.perf_counter() - t0
    log(f"preconditioner trained ({train_s:.2f} s)")

    def mixed_step(precond, mdl=None):
        def f():
            x.zero_()
            return G.solve_mixed(b.data_ptr(), x.data_ptr(), l=L_DEG,
                                 target=TOL_TRUE, precond=precond, model=mdl,
                                 stream=sp)
        return f

    if a.profile:
        return profile_run(a, torch, G, b, x, sp, plain_step, mixed_step, B, n,
                           model)

    modes = {}
    for name, step in (("plain_fp64", plain_step()),
                       ("plain_fp64_mgs", plain_step(B.BICGSTABL)),
                       ("mixed_none", mixed_step(B.PRECOND_NONE)),
                       ("mixed_jacobi", mixed_step(B.PRECOND_JACOBI)),
                       ("mixed_learned", mixed_step(B.PRECOND_LEARNED, model))):
        for _ in range(a.warmup):
            step()
        barrier()
        if name == "mixed_learned":
            with Clocks(local) as clk:
                ms, (ret_m, st_m) = timed(step, a.steps)
        else:
            ms, (ret_m, st_m) = timed(step, a.steps)
        barrier()
        tr = G.true_residual(b.data_ptr(), x.data_ptr(), sp)
        xe = float(torch.linalg.vector_norm(x - xt) / torch.linalg.vector_norm(xt))
        log(f"mode {name}: {np.mean(ms):.2f} ms, ret {ret_m}")
        modes[name] = {"s": max_over_ranks(float(np.mean(ms))) / 1e3,
                       "ret": ret_m, "true_residual": tr, "x_rel_error": xe,
                       "iters": st_m.get("iters", st_m.get("hist_len")),
                       "launches": int(st_m["launches"]),
                       "alg_bytes": int(st_m["alg_bytes"])}
    mode = "mixed_learned"
    step_ms = modes[mode]["s"] * 1e3
    plain_ms = modes["plain_fp64"]["s"] * 1e3
    ret, true_res = modes[mode]["ret"], modes[mode]["true_residual"]
    launches = modes[mode]["launches"] * a.steps

    # Dominant kernel alone: SpMV over the same operator, FP64 and FP32.
    xs64 = torch.rand(n, dtype=torch.float64, device=dev)
    ys64 = torch.empty(n, dtype=torch.float64, device=dev)
    xs32 = xs64.float()
    ys32 = torch.empty(n, dtype=torch.float32, device=dev)
    reps = 30
    tuned = G.variant()
    # The FP32 diagonal form with its vectors (78 MB) fits in L2: every
    # timed launch follows a 384 MB write and a read of the same buffer
    # (the read leaves L2 holding clean lines of that buffer, so the timed
    # launch neither hits its own data nor pays for writing back the
    # flush's dirty lines), and only the launch is inside the events.
    l2_flush = torch.empty(384 << 20, dtype=torch.uint8, device=dev)

    def time_spmv(xx, yy, f32):
        for _ in range(5):
            G.spmv(xx.data_ptr(), yy.data_ptr(), f32, sp)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        tot = 0.0
        for k in range(reps):
            l2_flush.fill_(k & 255)
            l2_flush.max()
            e0.record(stream)
            G.spmv(xx.data_ptr(), yy.data_ptr(), f32, sp)
            e1.record(stream)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / reps

    variants = {}
    for var_id, vname in G.SPMV_VARIANTS.items():
        G.variant(var_id)
        variants[vname] = {"fp64_ms": time_spmv(xs64, ys64, False),
                           "fp32_ms": time_spmv(xs32, ys32, True)}
    G.variant(tuned)
    kern = {"spmv_fp64": variants[G.SPMV_VARIANTS[tuned]]["fp64_ms"],
            "spmv_fp32": variants[G.SPMV_VARIANTS[tuned]]["fp32_ms"]}
    wv = 8 if mode == "plain_fp64" else 4
    fp = "fp64" if wv == 8 else "fp32"
    vname = G.SPMV_VARIANTS[tuned]
    kname = f"spmv_{vname}_{fp}"
    ndia = len(G.diagonals())
    if vname == "dia" and ndia:
        # Diagonal form: the stored diagonals (zero where a row lacks one),
        # one mask byte per row, x and y once.
        alg_bytes = ndia * wv * n + n + 2 * wv * n
    else:
        # CSR: values + column indices, row pointers, x and y once.
        alg_bytes = nnz * (wv + 4) + 4 * (n + 1) + 2 * wv * n
    csr_bytes = nnz * (wv + 4) + 4 * (n + 1) + 2 * wv * n
    peak, peak_kind = peaks()
    # Whole solve: the algorithmic bytes of every kernel the solve launched
    # (the library's per-launch count, stats["alg_bytes"]) over its time.
    for m_ in modes.values():
        m_["achieved_gbs"] = m_["alg_bytes"] / m_["s"] / 1e9
    solve_roof = {"bound": "hbm", "mode": mode, "alg_bytes": modes[mode]["alg_bytes"],
                  "achieved": modes[mode]["achieved_gbs"], "peak": peak,
                  "unit": "GB/s", "frac": modes[mode]["achieved_gbs"] / peak,
                  "peak_kind": peak_kind}
    launch_ms = kern["spmv_" + fp]
    achieved = alg_bytes / (launch_ms * 1e-3) / 1e9
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            traffic = json.load(f).get(kname)
    except (OSError, ValueError):
        traffic = None

    # End to end through bksp.h with host arrays (pinned).  The pinned
    # tensors are kept referenced for as long as their NumPy views are used.
    pinned_keep = [torch.from_numpy(np.ascontiguousarray(arr)).pin_memory()
                   for arr in (rp, c, v, b_h, np.zeros(n))]
    rp_p, c_p, v_p, b_p, x_p = [t.numpy() for t in pinned_keep]
    Ap = B.CsrMatrix(rp_p, c_p, v_p)
    e2e_ms, e2e_rets = [], []
    for i in range(a.warmup + a.steps):
        x_p[:] = 0.0
        if world > 1:
            dist.barrier()
        with B.record() as st_e:
            t0 = time.perf_counter()
            r_e2e = B.dbicgstabl_mixed(Ap, b_p, x_p, l=L_DEG, target=TOL_TRUE,
                                       precond=B.PRECOND_LEARNED, model=model)
            dt = time.perf_counter() - t0
        e2e_rets.append(r_e2e)
        if i >= a.warmup:
            e2e_ms.append(dt * 1e3)
    e2e_s = max_over_ranks(float(np.mean(e2e_ms))) / 1e3
    log(f"e2e: {e2e_s * 1e3:.1f} ms, rets {e2e_rets}")
    e2e_true = float(np.linalg.norm(b_h - P.csr_matvec(rp, c, v, x_p)) /
                     np.linalg.norm(b_h))
    e2e_xerr = float(np.linalg.norm(x_p - xt_h) / np.linalg.norm(xt_h))
    # CSR operator (FP64 values), b and x0; everything else (structure scan,
    # diagonal form, the learned preconditioner's slot map) is built on the
    # GPU.
    h2d = 4 * (n + 1) + 12 * nnz + 16 * n
    d2h = 8 * n

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(a.nx, x_ours=x_p, x_true=xt_h)
        log(f"cpu baseline: {cpu}")

    if rank == 0:
        line = {
            "metric": METRIC, "value": step_ms / 1e3, "unit": "s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": step_ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if mode == "plain_fp64" else "f32+f64",
            "data": "synthetic",
            "config": workload_config(a.nx, n, nnz),
            "mode": mode,
            "ret": ret, "true_residual": true_res,
            "plain_fp64_s": plain_ms / 1e3,
            "speedup_vs_plain_fp64": plain_ms / step_ms,
            "modes": modes,
            "spai_training": {"s": train_s, "final_loss": train_loss,
                              "systems": "convdiff3d 12^3, 16^3, 24^3",
                              "epochs": 200, "probes": 8},
            "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ret": r_e2e, "rets": e2e_rets,
                    "iters": st_e.get("hist_len"), "true_residual": e2e_true,
                    "x_rel_error": e2e_xerr,
                    "call_ms": st_e.get("total_ms"), "solve_ms": st_e.get("solve_ms")},
            "roofline": {"bound": "hbm", "kernel": kname,
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic,
                         "traffic_source": "profiles/traffic.json (ncu DRAM "
                                           "bytes of one launch, committed)",
                         "alg_bytes": alg_bytes,
                         "csr_alg_bytes": csr_bytes,
                         "launch_ms": launch_ms,
                         "variant": vname, "diagonals": ndia,
                         "spmv_variants_ms": variants},
            "solve_roofline": solve_roof,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    G.close()
    model.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def profile_run(a, torch, G, b, x, sp, plain_step, mixed_step, B, n, model):
    """One region between cudaProfilerStart/Stop, for ncu
    (--profile-from-start off)."""
    if a.profile == "spmv":
        x64 = torch.rand(n, dtype=torch.float64, device=b.device)
        y64 = torch.empty_like(x64)
        x32 = x64.float()
        y32 = torch.empty_like(x32)
        for _ in range(3):
            G.spmv(x64.data_ptr(), y64.data_ptr(), False, sp)
            G.spmv(x32.data_ptr(), y32.data_ptr(), True, sp)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        for _ in range(3):
            G.spmv(x64.data_ptr(), y64.data_ptr(), False, sp)
            G.spmv(x32.data_ptr(), y32.data_ptr(), True, sp)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        return 0
    step = {"plain_fp64": plain_step(),
            "mixed_none": mixed_step(B.PRECOND_NONE),
            "mixed_learned": mixed_step(B.PRECOND_LEARNED, model)}[a.profile]
    ret, st = step()          # warm: graph instantiation, features, pools
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    ret, st = step()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(f"profiled {a.profile}: ret {ret} launches {st['launches']}", flush=True)
    return 0


def cpu_baseline(nx, x_ours=None, x_true=None):
    """One full reference solve on this host (oracle/_ref), on every usable
    core, bounded to a few minutes.  With `x_ours` (the end-to-end solution)
    the reference's solution is compared with it and with x_true."""
    import tempfile
    from oracle import ref as R
    cores = usable_cores()
    if not R.available():
        return {"value": None, "unit": "s", "cores": cores, "kind": "reference",
                "sample": "oracle/_ref not built"}
    with tempfile.TemporaryDirectory() as td:
        xf = os.path.join(td, "x_ref.npy") if x_ours is not None else None
        dt, ret, cores = reference_full_solve(nx, timeout=300, x_out=xf)
        out = {"value": dt, "unit": "s", "cores": cores, "kind": "reference",
               "sample": f"one full dbicgstabl(l={L_DEG}) solve to tol {TOL_TRUE} "
                         f"(ret {ret}), {cores} threads"}
        if xf and dt is not None and os.path.exists(xf):
            xr = np.load(xf)
            out["x_rel_error"] = float(np.linalg.norm(xr - x_true) / np.linalg.norm(x_true))
            out["e2e_x_rel_diff_vs_reference"] = float(
                np.linalg.norm(np.asarray(x_ours) - xr) / np.linalg.norm(xr))
    return out


def run_batch(a):
    """The batched workload: 64 systems -div(kappa grad u) = f, 7-point
    finite volumes on L^3 grids, L ~ U{32..96} (seed 4), kappa = exp(GRF),
    f ~ N(0,1); time to an FP64 true relative residual of 1e-8 on every
    system.  value: mixed-precision BiCGSTAB(2) with the learned SPAI
    preconditioner (trained beforehand on the configuration's 256 smaller
    systems of the same family, seeds 1000+i, in four rounds whose logged
    iteration counts on three held-out systems pick the kept parameters),
    one CUDA-graph loop per system on eight host
    threads; plain_fp64_s: FP64 BiCGSTAB(2) on the Jacobi right-scaled
    systems A D^-1 y = b, x = D^-1 y, batched the same way; the modes also
    time both as one persistent launch for the whole batch (*_persistent)
    and the learned solve one system at a time (mixed_learned_sequential)."""
    import torch
    import torch.distributed as dist
    import bksp_b200 as B
    from bksp_b200 import problems as P
    from bksp_b200 import shard
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    # Multi-GPU: the systems are independent, so each rank solves its share
    # of the batch (balanced by stored entries, computed identically on every
    # rank); only the timings are reduced (max over ranks).
    edges = P.kappa_batch_edges(a.batch_count)
    mine = shard.my_share([7.0 * float(L) ** 3 for L in edges], world, rank)
    t0 = time.perf_counter()
    systems = P.kappa_batch(count=a.batch_count, indices=set(mine))
    gen_s = time.perf_counter() - t0
    ntot_all = int(sum(int(L) ** 3 for L in edges))
    ntot = sum(s[3] for s in systems)
    nnz = sum(int(s[0][-1]) for s in systems)
    t0 = time.perf_counter()
    mats = [B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32) for rp, c, v, n, b in systems]
    bs = [torch.from_numpy(s[4]).to(dev) for s in systems]
    xs = [torch.zeros_like(b) for b in bs]
    # Jacobi right-scaled copies for the FP64 comparator.
    scaled, dinv = [], []
    for rp, c, v, n, b in systems:
        rows = np.repeat(np.arange(n), np.diff(rp))
        d = np.zeros(n)
        d[rows[c == rows]] = v[c == rows]
        scaled.append(B.GpuMatrix(B.CsrMatrix(rp, c, v / d[c])))
        dinv.append(torch.from_numpy(1.0 / d).to(dev))
    upload_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    model = B.SpaiModel(seed=3)
    Ls = np.random.default_rng(999).integers(16, 33, 256)
    train = [B.GpuMatrix(B.CsrMatrix(*P.kappa_diffusion3d(int(L), 1000 + i)[:3]), B.FP32)
             for i, L in enumerate(Ls)]
    # Held-out probe systems (seeds 5000+i) whose logged iteration counts
    # choose among the training rounds.
    probe = []
    for i, L in enumerate((20, 28, 36)):
        prp, pc, pv, pn = P.kappa_diffusion3d(L, 5000 + i)[:4]
        probe.append((B.CsrMatrix(prp, pc, pv), np.random.default_rng(5100 + i).standard_normal(pn)))
    tlog = model.train_logged(train, probe, rounds=4, epochs=25, probes=8,
                              lr=3e-3, seed=7, l=2)
    loss = tlog["rounds"][tlog["best_round"]]["loss"] if tlog["best_round"] >= 0 else None
    for m in train:
        m.close()
    train_s = time.perf_counter() - t0
    torch.cuda.synchronize()

    def timed(fn, k):
        ms, last = [], None
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for _ in range(k):
            for x in xs:
                x.zero_()
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            e0.record()
            last = fn()
            e1.record()
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        t = float(np.mean(ms))
        if world > 1:
            tt = torch.tensor([t], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        return t, last

    def learned(workers=0):
        return lambda: B.solve_mixed_batch(mats, [b.data_ptr() for b in bs],
                                           [x.data_ptr() for x in xs], l=2,
                                           target=TOL_TRUE, precond=B.PRECOND_LEARNED,
                                           model=model, workers=workers)

    def plain(workers=0):
        return lambda: B.solve_batch(scaled, B.BICGSTABL_FAST, [b.data_ptr() for b in bs],
                                     [x.data_ptr() for x in xs], TOL_TRUE, 20000, l=2,
                                     workers=workers)

    def worst_true_res(scale):
        w = 0.0
        for (rp, c, v, n, b), x, di in zip(systems, xs, dinv):
            xh = (x * di if scale else x).cpu().numpy()
            r = b - P.csr_matvec(rp, c, v, xh)
            w = max(w, float(np.linalg.norm(r) / np.linalg.norm(b)))
        return w

    res = {}
    # workers=8: eight host threads, one CUDA-graph loop per system (the
    # default); workers=-1: every system in one persistent launch;
    # workers=1: one system after the other.
    for name, fn, k, scale in (("plain_fp64", plain(8), a.steps, True),
                               ("plain_fp64_persistent", plain(-1), a.steps, True),
                               ("mixed_learned_sequential", learned(1), 1, False),
                               ("mixed_learned_persistent", learned(-1), a.steps, False),
                               ("mixed_learned", learned(8), a.steps, False)):
        for _ in range(a.warmup if k > 1 else 0):
            for x in xs:
                x.zero_()
            fn()
        if name == "mixed_learned":
            with Clocks(local) as clk:
                ms, (ret, st) = timed(fn, k)
        else:
            ms, (ret, st) = timed(fn, k)
        its = [s["hist_len"] for s in st]
        stats = [worst_true_res(scale), -min(its), max(its), float(sum(its)),
                 float(len(its)), float(sum(s["launches"] for s in st)),
                 0.0 if ret == 0 else 1.0]
        if world > 1:
            t = torch.tensor(stats, dtype=torch.float64, device=dev)
            for i, op in enumerate((dist.ReduceOp.MAX, dist.ReduceOp.MAX, dist.ReduceOp.MAX,
                                    dist.ReduceOp.SUM, dist.ReduceOp.SUM, dist.ReduceOp.SUM,
                                    dist.ReduceOp.MAX)):
                ti = t[i:i + 1].clone()
                dist.all_reduce(ti, op=op)
                stats[i] = float(ti.item())
        res[name] = {"s": ms / 1e3, "ret": ret if stats[6] == 0 else -1,
                     "worst_true_residual": stats[0],
                     "iters_min": int(-stats[1]), "iters_max": int(stats[2]),
                     "iters_mean": stats[3] / stats[4],
                     "launches": int(stats[5])}
    if rank != 0:
        for m in mats + scaled:
            m.close()
        model.close()
        if world > 1:
            dist.destroy_process_group()
        return 0
    line = {
        "metric": "time to 1e-8 FP64 true residual on every system of the batch",
        "value": res["mixed_learned"]["s"], "unit": "s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": res["mixed_learned"]["s"] * 1e3, "higher_is_better": False,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": f"kappa_batch_{a.batch_count}", "systems": a.batch_count,
                   "rows": ntot_all, "rows_rank0": ntot, "nnz_rank0": nnz, "l": 2,
                   "edge": "U{32..96} seed 4",
                   "parallelism": f"systems sharded over {world} GPU(s), no exchange",
                   "kappa": "exp(GRF), corr 0.1, var 1", "rhs": "N(0,1)",
                   "l2": "inputs larger than L2 (FP64 CSR %.0f MB)" % ((nnz * 12 + 4 * ntot) / 1e6)},
        "plain_fp64_s": res["plain_fp64"]["s"],
        "speedup_vs_plain_fp64": res["plain_fp64"]["s"] / res["mixed_learned"]["s"],
        "modes": res,
        "spai_training": {"s": train_s, "final_loss": loss, "systems": "256 kappa, L U{16..32}",
                          "logged_iterations": tlog,
                          "epochs": 100, "probes": 8},
        "setup_s": {"generate": gen_s, "upload": upload_s},
        "clocks": clk.summary(),
        "gpu_launches": res["mixed_learned"]["launches"],
    }
    print(json.dumps(line), flush=True)
    for m in mats + scaled:
        m.close()
    model.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_configs(a):
    """The survey's configurations 1, 3 and 4, each as plain FP64 against
    mixed precision, both to an FP64 true relative residual of 1e-8 (every
    column / every shift):

    * cfg 1: CG on the 2D Poisson 64^2 operator (b ~ U[-1,1], seed 0),
      device-resident (CUDA events, median of five) and through the bksp.h
      host-array calls (one triangle stored); mixed = FP32 vectors, FP64
      reliable replacement, the learned preconditioner symmetrised (trained
      beforehand on 16^2..32^2 Poisson systems, outside the timing); the
      compiled reference's bksp_dcg beside it;
    * cfg 3: Block CG and Block BiCGSTAB(2), 16 Gaussian right-hand sides
      (seed 2), 3D Poisson 64^3 and 128^3, through dblcg / dblbicgstabl and
      their mixed counterparts (FP64 refinement around FP32 inner solves);
      the second of two calls is timed (the first includes the one-time
      block-product autotuning and the loop's graph capture);
    * cfg 4: shifted BiCGSTAB(4), 32 shifts 1e-3..1, 2D convection-diffusion
      1024^2, dshbicgstabl against bksp_dshbicgstabl_mixed (FP32 shift
      vectors, per-shift FP64 polishing).

    Prints one JSON line; worst residuals are recomputed on the host in FP64."""
    import scipy.sparse as sp
    import torch
    import bksp_b200 as B
    from bksp_b200 import problems as P
    res = {}

    def host_run(fn, reps=2):
        for _ in range(reps):
            with B.record() as st:
                t0 = time.perf_counter()
                r = fn()
                dt = time.perf_counter() - t0
        return r, dt, st

    def pair(name, plain, mixed):
        p_, m_ = res[name]["plain_fp64"], res[name]["mixed"]
        res[name]["speedup_mixed_vs_plain"] = p_["solve_s"] / m_["solve_s"]
        log(f"{name}: {res[name]}")

    # ---- cfg 1
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp_ = stream.cuda_stream
    rp, c, v, n = P.poisson2d(64)
    A = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = P.uniform(n, 0)
    mats = [B.GpuMatrix(B.CsrMatrix(*P.poisson2d(k)[:3]), B.FP32) for k in (16, 24, 32)]
    model = B.SpaiModel(seed=5)
    model.train(mats, epochs=150, probes=8, lr=3e-3, seed=9)
    for m_ in mats:
        m_.close()
    G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)
    bd = torch.from_numpy(b).cuda()
    xd = torch.zeros_like(bd)

    def dev_time(f, k=5):
        for _ in range(3):
            f()
        ms = []
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for _ in range(k):
            e0.record(stream)
            r = f()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.median(ms)) / 1e3, r

    def resid(x):
        return float(np.linalg.norm(b - A @ x) / np.linalg.norm(b))

    def plain1():
        xd.zero_()
        return G.solve(B.CG, bd.data_ptr(), xd.data_ptr(), 1e-8, 10000, stream=sp_)
    t, (r, st) = dev_time(plain1)
    e1 = {"solve_s": t, "ret": r, "true_residual": resid(xd.cpu().numpy()),
          "launches": st["launches"]}
    out = {}
    for pc, nm in ((0, "mixed_none"), (2, "mixed")):
        def mixed1():
            xd.zero_()
            return G.solve_mixed(bd.data_ptr(), xd.data_ptr(), target=1e-8, precond=pc,
                                 model=model, stream=sp_, method="cg")
        t, (r, st) = dev_time(mixed1)
        out[nm] = {"solve_s": t, "ret": r, "true_residual": resid(xd.cpu().numpy()),
                   "launches": st["launches"], "replacements": st["replacements"]}
    lrp, lc, lv, _ = P.lower_triangle(rp, c, v, n)
    A1 = B.CsrMatrix(lrp, lc, lv, symmetric=True)
    xh = np.zeros(n)
    r, dt, _ = host_run(lambda: (xh.fill(0.0), B.bksp_dcg(A1, b, 1e-8, 10000, xh))[1])
    e1["e2e_s"] = dt
    xh2 = np.zeros(n)
    r, dt, _ = host_run(lambda: (xh2.fill(0.0), B.dcg_mixed(A1, b, xh2, precond=B.PRECOND_LEARNED,
                                                           model=model))[1])
    out["mixed"]["e2e_s"] = dt
    res["cfg1_cg_poisson64"] = {"plain_fp64": e1, **out}
    from oracle import ref as R
    if R.available():
        Ar = R.Matrix(lrp, lc, lv, n, symmetric=True)
        t0 = time.perf_counter()
        r = R.call("bksp_dcg", Ar, b, 1e-8, 10000, np.zeros(n))[0]
        res["cfg1_cg_poisson64"]["reference_cpu"] = {"ret": int(r), "s": time.perf_counter() - t0}
    pair("cfg1_cg_poisson64", None, None)
    G.close()
    model.close()

    # ---- cfg 3
    for nx in (64, 128):
        rp, c, v, n = P.poisson3d(nx)
        lrp, lc, lv, _ = P.lower_triangle(rp, c, v, n)
        Af = sp.csr_matrix((v, c, rp), shape=(n, n))
        Bm = np.random.default_rng(2).standard_normal((n, 16))
        As = B.CsrMatrix(lrp, lc, lv, symmetric=True)
        Ag = B.CsrMatrix(rp, c, v)

        def worst(X):
            return float(max(np.linalg.norm(Bm[:, k] - Af @ X[:, k]) / np.linalg.norm(Bm[:, k])
                             for k in range(16)))
        for meth, plain, mixed in (
                ("blcg", lambda X: B.dblcg(As, Bm, 1e-8, 5000, X),
                 lambda X: B.dblcg_mixed(As, Bm, X, inner_tol=1e-3)),
                ("blbicgstabl2", lambda X: B.dblbicgstabl(Ag, Bm, 2, 1e-8, 5000, X),
                 lambda X: B.dblbicgstabl_mixed(Ag, Bm, 2, X, inner_tol=1e-3))):
            name = f"cfg3_{meth}_poisson{nx}"
            res[name] = {}
            for mode, fn in (("plain_fp64", plain), ("mixed", mixed)):
                X = np.zeros((n, 16))
                r, dt, st = host_run(lambda: (X.fill(0.0), fn(X))[1], reps=2)
                res[name][mode] = {"ret": r, "solve_s": st["solve_ms"] / 1e3, "e2e_s": dt,
                                   "worst_true_residual": worst(X)}
            pair(name, None, None)

    # ---- cfg 4
    rp, c, v, n = P.convdiff2d(1024)
    Af = sp.csr_matrix((v, c, rp), shape=(n, n))
    b = P.uniform(n, 3)
    sig = P.log_shifts(32)
    A4 = B.CsrMatrix(rp, c, v)
    nb = np.linalg.norm(b)

    def worst4(x):
        r_ = [np.linalg.norm(b - Af @ x[:n]) / nb] + [
            np.linalg.norm(b - (Af @ x[(k + 1) * n:(k + 2) * n] + s_ * x[(k + 1) * n:(k + 2) * n])) / nb
            for k, s_ in enumerate(sig)]
        return float(max(r_))
    name = "cfg4_shbicgstabl4_convdiff1024_32shifts"
    res[name] = {}
    for mode, fn in (("plain_fp64", lambda x: B.dshbicgstabl(A4, b, 4, sig, 1e-8, 5000, x)),
                     ("mixed", lambda x: B.dshbicgstabl_mixed(A4, b, 4, sig, x))):
        x = np.zeros(33 * n)
        r, dt, st = host_run(lambda: (x.fill(0.0), fn(x))[1])
        res[name][mode] = {"ret": r, "solve_s": st["solve_ms"] / 1e3, "e2e_s": dt,
                           "worst_true_residual": worst4(x),
                           "polish_iterations": st["inner_iters"] if mode == "mixed" else 0}
    pair(name, None, None)
    print(json.dumps({"workload": "configs", "unit": "s",
                      "metric": "time to 1e-8 FP64 true residual, plain FP64 vs mixed",
                      "results": res}), flush=True)
    return 0


def run_spmv_general(a):
    """Every SpMV kernel on the 3D convection-diffusion --nx^3 operator under
    a seeded random symmetric permutation (problems.permuted: same rows and
    entries, no diagonal form), hot, CUDA events over 50 launches: time and
    fraction of the measured copy bandwidth on the CSR algorithmic bytes
    nnz (w + 4) + 4 (n + 1) + 2 w n.  Prints one JSON line."""
    import torch
    import bksp_b200 as B
    P = problems_module()
    rp, c, v, n = P.permuted(*P.convdiff3d(a.nx))
    G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)
    tuned = G.variant()
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp_ = stream.cuda_stream
    x64 = torch.rand(n, dtype=torch.float64, device="cuda")
    y64 = torch.empty_like(x64)
    x32 = x64.float()
    y32 = torch.empty_like(x32)
    peak = peaks()[0]
    nnz = int(rp[-1])
    out = {}
    for vid, name in G.SPMV_VARIANTS.items():
        if name == "dia":
            continue
        G.variant(vid)
        row = {}
        for f32, xx, yy, w in ((False, x64, y64, 8), (True, x32, y32, 4)):
            for _ in range(5):
                G.spmv(xx.data_ptr(), yy.data_ptr(), f32, sp_)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(50):
                G.spmv(xx.data_ptr(), yy.data_ptr(), f32, sp_)
            e1.record(stream)
            e1.synchronize()
            us = e0.elapsed_time(e1) / 50 * 1e3
            alg = nnz * (w + 4) + 4 * (n + 1) + 2 * w * n
            key = "fp32" if f32 else "fp64"
            row[key + "_us"] = us
            row[key + "_frac"] = alg / (us * 1e-6) / 1e9 / peak
        out[name] = row
    G.variant(tuned)
    G.close()
    # The block product (s = 16) on the unpermuted operator, both kernels:
    # algorithmic bytes = the format's matrix bytes + X once + Y once.
    rp, c, v, n = P.convdiff3d(a.nx)
    G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)
    nd = len(G.diagonals())
    spmm = {}
    for f32, w, dt in ((False, 8, torch.float64), (True, 4, torch.float32)):
        X = torch.rand(n * 16, dtype=dt, device="cuda")
        Y = torch.empty_like(X)
        for kern, name in ((0, "dia"), (1, "csr")):
            for _ in range(3):
                G.spmm(16, X.data_ptr(), Y.data_ptr(), f32, kern, sp_)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(20):
                G.spmm(16, X.data_ptr(), Y.data_ptr(), f32, kern, sp_)
            e1.record(stream)
            e1.synchronize()
            us = e0.elapsed_time(e1) / 20 * 1e3
            mat = nd * w * n + n if name == "dia" else nnz * (w + 4) + 4 * (n + 1)
            alg = mat + 2 * 16 * w * n
            key = f"{name}_{'fp32' if f32 else 'fp64'}"
            spmm[key + "_us"] = us
            spmm[key + "_frac"] = alg / (us * 1e-6) / 1e9 / peak
    line = {"metric": "SpMV time on an operator without a diagonal form",
            "workload": f"permuted convdiff3d {a.nx}^3", "n": n, "nnz": nnz,
            "peak_gbs": peak, "autotuned": G.SPMV_VARIANTS[tuned],
            "variants": out, "timing": "hot, CUDA events, 50 launches",
            "spmm_s16_unpermuted": spmm}
    print(json.dumps(line), flush=True)
    G.close()
    return 0


def complex_reference_worker(spec):
    """One compiled-reference complex solve (oracle/_ref) in this process;
    prints {"s": seconds, "ret": ret}."""
    from oracle import ref as R
    P = problems_module()
    d = json.loads(spec)
    rp, c, v, n = P.complex_convdiff3d(d["nx"])
    A = R.ZMatrix(rp, c, v, n)
    b = P.complex_uniform(n, 3)
    m = d["method"]
    t0 = time.perf_counter()
    if m == "zbicg":
        ret, _, _ = R.zcall("zbicg", A, b, 1e-8, d["max_iter"], np.zeros(n, complex))
    elif m == "zshbicgstabl":
        sig = P.complex_shifts(d["ns"])
        ret, _, _ = R.zcall("zshbicgstabl", A, b, d["l"], sig, d["ns"], 1e-8,
                            d["max_iter"], np.zeros(n * (d["ns"] + 1), complex))
    else:
        Bm = np.random.default_rng(7).uniform(-1, 1, (n, d["s"])) \
            + 1j * np.random.default_rng(8).uniform(-1, 1, (n, d["s"]))
        ret, _, _ = R.zcall("zblbicgstabl", A, Bm, d["l"], 1e-8, d["max_iter"],
                            np.zeros((n, d["s"]), complex))
    print(json.dumps({"s": time.perf_counter() - t0, "ret": int(ret)}), flush=True)
    return 0


def run_complex(a):
    """The complex solvers on the complex 3D convection-diffusion operator
    (complex_convdiff3d, --nx^3, seeded right-hand sides), each to a relative
    residual of 1e-8 through the bksp.h calls: GPU device time of the call
    (bksp_gpu_record) and its FP64 true residual, beside the compiled
    reference's complex solver on this host's cores (a child process, the
    same call; zbicgstabl has no reference timing: its reference result
    depends on stack contents).  Prints one JSON line."""
    import scipy.sparse as sp
    import bksp_b200 as B
    P = problems_module()
    nx = a.nx if a.nx != NX else 64
    rp, c, v, n = P.complex_convdiff3d(nx)
    As = sp.csr_matrix((v, c, rp), shape=(n, n))
    A = B.ZCsrMatrix(rp, c, v)
    b = P.complex_uniform(n, 3)
    ns, s_blk = 8, 8
    sig = P.complex_shifts(ns)
    rng7, rng8 = np.random.default_rng(7), np.random.default_rng(8)
    Bm = rng7.uniform(-1, 1, (n, s_blk)) + 1j * rng8.uniform(-1, 1, (n, s_blk))
    cores = usable_cores()
    out = {}

    def gpu(name, fn, check):
        best = None
        for _ in range(3):
            with B.record() as st:
                ret, xv = fn()
            if best is None or st["solve_ms"] < best[0]:
                best = (st["solve_ms"], ret, st["total_ms"], st["launches"], xv)
        ms, ret, tot, launches, xv = best
        out[name] = {"gpu_solve_s": ms / 1e3, "gpu_call_s": tot / 1e3, "ret": ret,
                     "launches": launches, "worst_true_residual": check(xv)}

    def ref(name, spec, budget=600):
        env = dict(os.environ, OPENBLAS_NUM_THREADS=str(cores),
                   OMP_NUM_THREADS=str(cores))
        cmd = [sys.executable, os.path.abspath(__file__),
               "--complex-reference-worker", json.dumps(spec)]
        try:
            r = subprocess.run(cmd, env=env, capture_output=True, text=True,
                               timeout=budget)
            d = json.loads(r.stdout.strip().splitlines()[-1])
            out[name]["reference_s"] = d["s"]
            out[name]["reference_ret"] = d["ret"]
            out[name]["gpu_speedup_vs_reference"] = d["s"] / out[name]["gpu_call_s"]
        except (subprocess.TimeoutExpired, ValueError, IndexError, KeyError) as e:
            out[name]["reference_s"] = None
            out[name]["reference_note"] = f"not measured: {type(e).__name__}"

    def tr(x, sigma=0.0):
        return float(np.linalg.norm(b - As @ x - sigma * x) / np.linalg.norm(b))

    def run_zbicg():
        x = np.zeros(n, complex)
        return B.zbicg(A, b, 1e-8, 5000, x), x
    gpu("zbicg", run_zbicg, tr)
    ref("zbicg", {"method": "zbicg", "nx": nx, "max_iter": 5000})

    def run_zbl():
        x = np.zeros(n, complex)
        return B.zbicgstabl(A, b, 4, 1e-8, 5000, x), x
    gpu("zbicgstabl4", run_zbl, tr)

    def run_zsh():
        x = np.zeros(n * (ns + 1), complex)
        return B.zshbicgstabl(A, b, 4, sig, 1e-8, 5000, x), x
    gpu("zshbicgstabl4_8shifts", run_zsh, lambda x: max(
        [tr(x[:n])] + [tr(x[(k + 1) * n:(k + 2) * n], sg) for k, sg in enumerate(sig)]))
    ref("zshbicgstabl4_8shifts", {"method": "zshbicgstabl", "nx": nx, "l": 4,
                                  "ns": ns, "max_iter": 5000})

    def run_zblk():
        X = np.zeros((n, s_blk), complex)
        return B.zblbicgstabl(A, Bm, 2, 1e-8, 5000, X), X
    gpu("zblbicgstabl2_s8", run_zblk, lambda X: max(
        float(np.linalg.norm(Bm[:, j] - As @ X[:, j]) / np.linalg.norm(Bm[:, j]))
        for j in range(s_blk)))
    ref("zblbicgstabl2_s8", {"method": "zblbicgstabl", "nx": nx, "l": 2,
                             "s": s_blk, "max_iter": 5000})
    line = {"metric": "complex solves to a relative residual of 1e-8",
            "workload": f"complex_convdiff3d_{nx}^3", "n": n, "nnz": int(rp[-1]),
            "reference_cores": cores, "methods": out}
    print(json.dumps(line), flush=True)
    return 0


def profile_small(a):
    """Profiling drivers that need no headline set-up: block_cg = five Block
    CG iterations (16 Gaussian right-hand sides, 3D Poisson --nx^3; run with
    BKSP_GPU_LOOP=poll so a launch list sees every kernel); persist_cg = one
    CG solve of the 2D Poisson 64^2 system as a persistent launch."""
    import bksp_b200 as B
    P = problems_module()
    if a.profile == "spmv_perm":
        import torch
        rp, c, v, n = P.permuted(*P.convdiff3d(a.nx))
        G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)
        x64 = torch.rand(n, dtype=torch.float64, device="cuda")
        y64 = torch.empty_like(x64)
        x32 = x64.float()
        y32 = torch.empty_like(x32)
        for var in (0, 8):
            G.variant(var)
            for _ in range(2):
                G.spmv(x64.data_ptr(), y64.data_ptr(), False)
                G.spmv(x32.data_ptr(), y32.data_ptr(), True)
        torch.cuda.synchronize()
        print(f"profiled spmv_perm {a.nx}^3", flush=True)
        G.close()
        return 0
    if a.profile == "zbicgstabl":
        rp, c, v, n = P.complex_convdiff3d(a.nx)
        A = B.ZCsrMatrix(rp, c, v)
        b = P.complex_uniform(n, 3)
        x = np.zeros(n, complex)
        ret = B.zbicgstabl(A, b, 4, 1e-10, 3, x)
        print(f"profiled zbicgstabl {a.nx}^3: ret {ret}", flush=True)
        return 0
    if a.profile == "block_cg":
        rp, c, v, n = P.poisson3d(a.nx)
        lrp, lc, lv, _ = P.lower_triangle(rp, c, v, n)
        Bm = np.random.default_rng(2).standard_normal((n, 16))
        X = np.zeros((n, 16))
        ret = B.dblcg(B.CsrMatrix(lrp, lc, lv, symmetric=True), Bm, 1e-8, 5, X)
        print(f"profiled block_cg {a.nx}^3: ret {ret}", flush=True)
        return 0
    import torch
    torch.cuda.set_device(0)
    rp, c, v, n = P.poisson2d(64)
    G = B.GpuMatrix(B.CsrMatrix(rp, c, v), B.FP32)
    b = torch.from_numpy(P.uniform(n, 0)).cuda()
    x = torch.zeros_like(b)
    with B.loop_mode(1):
        for _ in range(2):
            x.zero_()
            ret, st = G.solve(B.CG, b.data_ptr(), x.data_ptr(), 1e-10, 10000)
    print(f"profiled persist_cg: ret {ret} launches {st['launches']}", flush=True)
    G.close()
    return 0


def main():
    a = args_()
    if a.reference_solve_worker:
        return reference_solve_worker(a.nx, a.x_out)
    if a.complex_reference_worker:
        return complex_reference_worker(a.complex_reference_worker)
    if a.profile in ("block_cg", "persist_cg", "zbicgstabl", "spmv_perm"):
        return profile_small(a)
    if a.impl == "reference":
        return run_reference(a)
    if a.workload == "kappa_batch":
        return run_batch(a)
    if a.workload == "configs":
        return run_configs(a)
    if a.workload == "complex":
        return run_complex(a)
    if a.workload == "spmv_general":
        return run_spmv_general(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
