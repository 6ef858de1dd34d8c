#!/usr/bin/env python3
"""Benchmark of the matrix-free DG SIPG vmult (one JSON line on rank 0).

Workload (one step = one vmult dst = A src): DG SIPG Poisson, degree 3 (20
DoF/tet), 32^3 hexes x 6 Kuhn tets = 196,608 affine tets, 3,932,160 DoFs;
interior vertices jittered by U[-0.1h, 0.1h] (mt19937_64 seed 0); src uniform
in [-1,1] (numpy PCG64 seed 1); penalty (p+1)(p+d)/d * surface/volume.
The same operator in FP32 is measured beside the FP64 headline.

--impl ours (default): the CUDA path through the C ABI; L2 (126 MB) is
flushed before every timed vmult by writing a 256 MB buffer and then reading
another 256 MB buffer (so the vmult starts with none of its data in L2 and no
dirty lines of the flush left to write back), and only the vmult is inside
the CUDA events.
--impl reference: the reference's optimized algorithm on the host cores
(oracle/fast.cpp: cells and faces in 8-lane SIMD batches, 4 batches per dense
shape-matrix product, face groups by local face numbers, OpenMP threads over
contiguous cell ranges), on the same mesh built by the oracle's own generator
(oracle/mesh.c), each step one full vmult.  The product library is not loaded.

N > 1 (torchrun): every rank runs its own replica of the workload (the
north-star path is a single-GPU operator; no data-path collective), timing is
the max over ranks, value is the sum of DoFs over ranks / that time.  With
--dd the ranks instead share one 32 x 32 x 32N mesh, domain-decomposed, and
exchange ghost cells over NCCL in every vmult (simplex-benchmarks_b200/
distributed.py).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (os.path.join(ROOT, "simplex-benchmarks_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

N_HEX, DEGREE, JITTER = 32, 3, 0.1
METRIC = "vmult DoF/s (FP64 vs mixed); Poisson solve time to 1e-8 (MG vs learned)"
WORKLOAD = "DG SIPG Poisson vmult, P3 on 32^3 x 6 Kuhn tets (196,608 cells, 3,932,160 DoFs), jitter 0.1h"
# DRAM bytes (read + written) of one launch of the apply kernel on this
# workload: dram__bytes_read.sum + dram__bytes_write.sum of an ncu capture
# (profiles/dg_apply_kernel_p3_fp64_32cube.md)
APPLY_KERNEL = "dg_apply_kernel<3,1,false,128,double,1,false,true,1>"
APPLY_TRAFFIC_BYTES = 100.57e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-solve", action="store_true", help="skip the multigrid solve measurement")
    ap.add_argument("--no-extra", action="store_true", help="skip the CG (configs 1, 1L) and batch (config 4) lines")
    ap.add_argument("--no-learned", action="store_true", help="skip training and timing the learned smoother")
    ap.add_argument("--dd", action="store_true",
                    help="domain decomposition instead of replicas: one 32^3 x 6-tet DG P3 block per rank of a "
                         "32 x 32 x 32N mesh, halo exchange over NCCL every vmult")
    ap.add_argument("--case", choices=["cg-p2-64", "cg-p3-64", "cg-p1-128", "cg-p2-128", "mlp-64", "dg-p3-32",
                                       "solve-p3-64"],
                    help="run one small kernel workload (for profiling) instead of the benchmark")
    ap.add_argument("--variant", type=int, default=0,
                    help="kernel variant of --case dg-p3-32, or of the FP32 operator of a cg-* case (0: default)")
    return ap.parse_args()


def max_over_ranks(value, device):
    """The largest `value` over the ranks of the default process group (the
    timed region ends when the slowest rank ends); the value itself without one."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu, interval=0.02):
        self.gpu = gpu
        self.interval = interval
        self.proc = None
        self.samples = []  # (sm_mhz, max_mhz, reasons)
        self.nvml = None

    def _poll(self):
        import pynvml as nv
        h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        bits = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}
        while not self.stop.is_set():
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            self.samples.append((float(sm), float(mx), [k for k, v in bits.items() if r & v]))
            time.sleep(self.interval)

    def __enter__(self):
        try:
            import threading
            import pynvml as nv
            nv.nvmlInit()
            self.nvml = nv
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.nvml:
            time.sleep(2 * self.interval)
            self.stop.set()
            self.thread.join(timeout=5)
            return
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        sm, mx, reasons = [], None, set()
        for f, m, rs in self.samples:
            sm.append(f)
            mx = m
            reasons.update(rs)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self.nvml else "nvidia-smi"}


class L2Flush:
    """Evicts L2 (126 MB) on a stream: writes a 256 MB buffer, then reads a
    second 256 MB buffer (a sum into a one-element tensor), so the next kernel
    starts with none of its data in L2 and the flush's own dirty lines are
    already written back."""

    def __init__(self):
        import torch
        n = 256 * 1024 * 1024 // 4
        self.wbuf = torch.empty(n, dtype=torch.float32, device="cuda")
        self.rbuf = torch.ones(n, dtype=torch.float32, device="cuda")
        self.acc = torch.empty(1, dtype=torch.float32, device="cuda")

    def __call__(self, on=None):
        import torch
        with torch.cuda.stream(on if on is not None else torch.cuda.current_stream()):
            self.wbuf.fill_(1.0)
            torch.sum(self.rbuf, dim=0, keepdim=True, out=self.acc)


def timed_steps(fn, steps, warmup, stream, flush=None):
    """Per-step device time (ms) of fn() with CUDA events on `stream`; flush(s)
    writes the L2-sized buffer on stream s, the timing stream, so that it ends
    before the timed work starts."""
    import torch
    for _ in range(warmup):
        if flush:
            flush(stream)
        fn()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with torch.cuda.stream(stream):
        for a, b in ev:
            if flush:
                flush(stream)
            a.record(stream)
            fn()
            b.record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def fp64_peak_tflops():
    """Measured FP64 throughput of cuBLAS DGEMM (8192^3, best of 5), TF/s."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2 * n ** 3 / best / 1e12


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def build_problem(precision):
    import numpy as np
    import simplexfem as sf
    mesh = sf.Mesh(N_HEX, jitter=JITTER, seed=0)
    op = sf.Operator(mesh, DEGREE, "dg", precision)
    x = np.random.default_rng(1).uniform(-1.0, 1.0, op.m())
    return mesh, op, x


def cpu_solve_baseline(b, repeats=2):
    """The same solve on the host cores: the matrix-free MG-CG restatement
    (oracle/fast_mg.py: optimized SIMD/OpenMP level operators, Chebyshev(3)-
    Jacobi, nodal transfers, direct coarse solve, FP64 CG to 1e-8) on the same
    load vector; best of `repeats` solves after the set-up."""
    import torch
    import fast_mg
    t0 = time.perf_counter()
    mg = fast_mg.FastMG(64, 3)
    setup = time.perf_counter() - t0
    bt = torch.from_numpy(b)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        _, its = mg.solve(bt.clone(), rtol=1e-8)
        times.append(time.perf_counter() - t0)
    L = mg.levels[-1]
    return {"ms": 1e3 * min(times), "iterations": its, "setup_s": setup, "cores": L.op.threads,
            "kind": "port", "sample": f"{repeats} full solves of the same problem ({L.n} DoFs) on {L.op.threads} "
                                      f"threads ({L.op.isa}), matrix-free levels by the optimized CPU restatement"}


def mg_solve_bench(repeats=5, learned=True, cpu_baseline=True):
    """Poisson solve to rel. residual 1e-8: CG P3 on 64^3 x 6 tets (7,189,057 DoFs),
    f = sum of 8 sin(k.x), k ~ U[1,6]^3 (PCG64 seed 2); FP64 outer CG preconditioned by
    the hybrid p(3-2-1)/h(64-32-16-8-4) multigrid with Chebyshev(3)-Jacobi smoothing and a
    CUDA-graph V-cycle; levels in FP32 (mixed; CUDA-core, and TF32 tensor-core
    contractions for the CG levels) vs FP64."""
    import torch
    import simplexfem as sf
    mesh = sf.Mesh(64)
    op = sf.Operator(mesh, 3, "cg", "fp64")
    b = sf.rhs(op, sf.sine_modes_rhs())
    x = op.initialize_dof_vector()
    out = {"workload": "CG P3 Poisson, 64^3 x 6 Kuhn tets, 7,189,057 DoFs, rel. residual 1e-8",
           "dofs": op.m()}
    for prec, tc in (("fp64", False), ("fp32", False), ("fp32", True)):
        mg = sf.Multigrid(op, precision=prec, smoother_degree=3, tensor_cores=tc)
        cg = sf.SolverCG(op, mg)
        cg.solve(x, b, rtol=1e-8)  # warm-up (graph capture)
        times, its = [], None
        for _ in range(repeats):
            x.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = cg.solve(x, b, rtol=1e-8)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
            its = r["iterations"]
            assert r["status"] == 0
        key = "fp64_mg" if prec == "fp64" else ("mixed_tf32_mg" if tc else "mixed_mg")
        out[key] = {"ms": 1e3 * min(times), "ms_median": 1e3 * statistics.median(times), "iterations": its,
                    "dofs_per_s": op.m() / min(times)}
        del cg, mg
    if cpu_baseline:
        out["cpu_baseline"] = cpu_solve_baseline(b.cpu().numpy())
    if learned:
        # config 5: the finest-level smoother replaced by the per-cell MLP, trained
        # here on residual/error pairs of MG-CG solves on 16^3 and 32^3 meshes
        # (random sine loads, seeds 1000+, 200k samples), tcgen05 inference,
        # flexible CG, Chebyshev fallback on a poor cycle
        t0 = time.perf_counter()
        mlp = sf.MLP(seed=1)
        info = mlp.generate_and_train(epochs=20)
        train_s = time.perf_counter() - t0
        mg = sf.Multigrid(op, precision="fp32", smoother_degree=3)
        mg.set_learned_smoother(mlp, fallback=True)
        cg = sf.SolverCG(op, mg, flexible=True)
        cg.solve(x, b, rtol=1e-8)
        times = []
        for _ in range(repeats):
            x.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = cg.solve(x, b, rtol=1e-8)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
            assert r["status"] == 0
        out["mixed_learned_mg"] = {
            "ms": 1e3 * min(times), "ms_median": 1e3 * statistics.median(times), "iterations": r["iterations"],
            "fallback_iteration": r["fallback_iteration"], "dofs_per_s": op.m() / min(times),
            "train_seconds": train_s, "train_samples": info["samples"], "loss_first": info["loss_first"],
            "loss_last": info["loss_last"], "bounded_wait_timeouts": int(mlp.timed_out())}
        del cg, mg
    # DG (SIPG) P3 on 32^3 x 6 tets solved with the p/c/h multigrid (cph: CG P3
    # right below DG P3), FP32 levels, FP64 outer CG, random load (seed 3)
    mesh_dg = sf.Mesh(32)
    opd = sf.Operator(mesh_dg, 3, "dg", "fp64")
    bd = torch.tensor(__import__("numpy").random.default_rng(3).uniform(-1, 1, opd.m()), device="cuda")
    xd = opd.initialize_dof_vector()
    for ct, name in ((0, "dg_mg_phc"), (1, "dg_mg_cph")):
        mg = sf.Multigrid(opd, precision="fp32", smoother_degree=3, c_transfer=ct)
        cg = sf.SolverCG(opd, mg)
        cg.solve(xd, bd, rtol=1e-8)
        times = []
        for _ in range(repeats):
            xd.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = cg.solve(xd, bd, rtol=1e-8)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
            assert r["status"] == 0
        out[name] = {"workload": "DG SIPG P3, 32^3 x 6 tets (3,932,160 DoFs), mixed MG-CG to 1e-8",
                     "ms": 1e3 * min(times), "iterations": r["iterations"]}
        del cg, mg
    return out


def cg_vmult_bench(steps, warmup, flush):
    """Config 1: CG P2 Poisson on 16^3 x 6 tets (jitter 0.1h, seed 0), src U[-1,1]
    (seed 1) zeroed at constrained DoFs, FP64: 100 vmults replayed from one CUDA
    graph, best of 5 replays.  Config 1L: CG P2 on 128^3 x 6 tets (16,974,593 DoFs),
    FP64 and FP32, L2 flushed before every timed vmult: the HBM-bound case."""
    import numpy as np
    import torch
    import simplexfem as sf
    out = {}
    s = torch.cuda.Stream()
    mesh = sf.Mesh(16, jitter=JITTER, seed=0)
    op = sf.Operator(mesh, 2, "cg", "fp64")
    x = np.random.default_rng(1).uniform(-1.0, 1.0, op.m())
    x[op.constrained().astype(bool)] = 0.0
    src = torch.tensor(x, device="cuda")
    dst = op.initialize_dof_vector()
    with torch.cuda.stream(s):
        for _ in range(3):
            op.vmult(dst, src, s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        for _ in range(100):
            op.vmult(dst, src, s)
    best = 1e30
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(s):
            a.record(s)
            g.replay()
            b.record(s)
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    del g
    out["config1"] = {"workload": "CG P2 Poisson vmult, 16^3 x 6 tets (24,576 cells, 35,937 DoFs), FP64, "
                                  "100 vmults in one CUDA graph, best of 5",
                      "dofs_per_s": 100 * op.m() / (best / 1e3), "us_per_vmult": best * 10.0}
    del op, mesh
    hbm, _ = measured_peaks()
    mesh = sf.Mesh(128, jitter=JITTER, seed=0)
    for prec in ("fp64", "fp32"):
        op = sf.Operator(mesh, 2, "cg", prec)
        tune = op.autotune(reps=10, use_cache=False)
        src = torch.rand(op.m(), dtype=op.dtype, device="cuda") * 2 - 1
        dst = op.initialize_dof_vector()
        t = timed_steps(lambda: op.vmult(dst, src, s), steps, warmup, s, flush)
        ms = statistics.mean(t)
        _, alg = op.work()
        out["config1L_" + prec] = {
            "workload": "CG P2 Poisson vmult, 128^3 x 6 tets (12,582,912 cells, 16,974,593 DoFs), L2 flushed",
            "dofs_per_s": op.m() / (ms / 1e3), "us_per_vmult": ms * 1e3,
            "alg_gbs": alg / (ms / 1e3) / 1e9, "hbm_frac": alg / (ms / 1e3) / 1e9 / hbm,
            "kernel_variant": tune["variant"], "variant_us": tune["us"]}
        del op, src, dst
    return out


def spmv_bench(steps, warmup, flush):
    """The reference's assembled-matrix comparison (CG/cells_batched/
    application.cc:1944-1988): CG P2 on 64^3 x 6 tets (jitter 0.1h), FP64, the
    matrix-free vmult against the same operator assembled into a device CSR
    matrix (fem_csr_spmv), L2 flushed before every timed product."""
    import numpy as np
    import torch
    import simplexfem as sf
    mesh = sf.Mesh(64, jitter=JITTER, seed=0)
    op = sf.Operator(mesh, 2, "cg", "fp64")
    A = sf.CSRMatrix(op)
    x = np.random.default_rng(1).uniform(-1.0, 1.0, op.m())
    src = torch.tensor(x, device="cuda")
    y1, y2 = op.initialize_dof_vector(), op.initialize_dof_vector()
    s = torch.cuda.Stream()
    t_mf = timed_steps(lambda: op.vmult(y1, src, s), steps, warmup, s, flush)
    t_sp = timed_steps(lambda: A.vmult(y2, src, s), steps, warmup, s, flush)
    torch.cuda.synchronize()
    diff = float(torch.linalg.norm(y1 - y2) / torch.linalg.norm(y1))
    sp_bytes = A.nnz * 12 + (A.m + 1) * 8 + 2 * 8 * A.m
    out = {"workload": "CG P2 Poisson, 64^3 x 6 tets (2,146,689 DoFs), FP64, L2 flushed",
           "matrix_free_us": 1e3 * statistics.mean(t_mf), "spmv_us": 1e3 * statistics.mean(t_sp),
           "nnz_per_row": A.nnz / A.m, "spmv_bytes": sp_bytes,
           "spmv_gbs": sp_bytes / (statistics.mean(t_sp) / 1e3) / 1e9, "rel_diff": diff}
    del A
    return out


def batch_bench(steps, warmup, flush):
    """Config 4: 32 independent Helmholtz-like DG P2 x 3-component problems on
    uneven meshes n_i = 8 + floor(32 i / 31) (8^3 .. 40^3 hexes x 6 tets,
    110,213,460 DoFs in total), src_i ~ U[-1,1] (seeds 100 + i); one persistent
    launch per pass for all 32, kernel shape picked by the autotuner; against the
    same 32 vmults launched one after another."""
    import numpy as np
    import torch
    import simplexfem as sf
    sizes = [8 + (32 * i) // 31 for i in range(32)]
    meshes = [sf.Mesh(n) for n in sizes]
    s = torch.cuda.Stream()
    out = {"workload": "32 Helmholtz DG P2 x 3 comps problems, n_i = 8 + floor(32 i/31) hexes/dir"}
    for prec in ("fp64", "fp32"):
        ops = [sf.Operator(m, 2, "helmholtz", prec) for m in meshes]
        total = sum(o.m() for o in ops)
        xs = [torch.tensor(np.random.default_rng(100 + i).uniform(-1.0, 1.0, o.m()), dtype=o.dtype, device="cuda")
              for i, o in enumerate(ops)]
        ys = [o.initialize_dof_vector() for o in ops]
        b = sf.Batch(ops)
        tune = b.autotune(reps=5, use_cache=False)
        tb = timed_steps(lambda: b.vmult(ys, xs, s), steps, warmup, s, flush)

        def one_by_one():
            for o, x_, y_ in zip(ops, xs, ys):
                o.vmult(y_, x_, s)
        ts = timed_steps(one_by_one, steps, warmup, s, flush)
        out[prec] = {"dofs": total, "batched_dofs_per_s": total / (statistics.mean(tb) / 1e3),
                     "batched_ms": statistics.mean(tb), "sequential_ms": statistics.mean(ts),
                     "autotuned_variant": tune["variant"], "variant_us": tune["us"]}
        del ops, xs, ys, b
    return out


def fast_problem():
    """The headline workload built by the oracle alone: its own Kuhn mesh
    generator and the optimized CPU restatement of the reference's vmult."""
    import numpy as np
    import fast
    import oracle as orc
    mesh = orc.KuhnMesh(N_HEX, jitter=JITTER, seed=0)
    op = fast.FastOperator(mesh, DEGREE, orc.DG)
    x = np.random.default_rng(1).uniform(-1.0, 1.0, op.n)
    return op, x


def cpu_baseline(target_seconds=10.0):
    """The optimized CPU restatement on this host's cores, full vmults of the
    same workload for about `target_seconds`."""
    import numpy as np
    op, x = fast_problem()
    y = np.empty(op.n)
    op.vmult(x, y)
    t0 = time.perf_counter()
    op.vmult(x, y)
    one = time.perf_counter() - t0
    reps = max(1, int(target_seconds / max(one, 1e-6)))
    t0 = time.perf_counter()
    for _ in range(reps):
        op.vmult(x, y)
    dt = time.perf_counter() - t0
    return {"value": op.n * reps / dt, "unit": "DoF/s", "cores": op.threads, "kind": "port",
            "sample": f"{reps} full FP64 DG P3 vmults of the same workload ({op.n} DoFs each), {dt:.1f} s; "
                      f"optimized restatement of the reference's vmult ({op.isa}, {op.lanes} lanes, "
                      f"{op.n_cell_points}/{op.n_face_points} cell/face points), OpenMP over {op.threads} "
                      f"threads; mesh from the oracle's own generator"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import numpy as np
    op, x = fast_problem()
    y = np.empty(op.n)
    for _ in range(args.warmup):
        op.vmult(x, y)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        op.vmult(x, y)
        times.append(time.perf_counter() - t0)
    assert np.isfinite(y).all()
    total = sum(times)
    value = op.n * args.steps / total
    sample = (f"one full FP64 DG P3 vmult per step ({op.n} DoFs): optimized restatement of the reference's "
              f"vmult ({op.isa}, {op.lanes} lanes, {op.n_cell_points}/{op.n_face_points} cell/face points), "
              f"OpenMP over {op.threads} threads; mesh from the oracle's own generator")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "DoF/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "scope": "rank 0 only, host cores"},
            "cpu_baseline": {"value": value, "unit": "DoF/s", "cores": op.threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "DoF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "gpu_launches": 0}
    print(json.dumps(line), flush=True)


def run_dd(args):
    """Weak scaling of the domain-decomposed DG P3 vmult: the mesh is 32 x 32 x
    32N hexes x 6 tets (jitter 0.1h) split into N contiguous Morton ranges, one
    per rank; every step is one ghost update (NCCL point-to-point) and one
    local vmult; time = max over ranks of the device time."""
    import numpy as np
    import torch
    import torch.distributed as dist
    import simplexfem as sf
    import distributed as fd
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    import datetime
    dist.init_process_group("nccl" if world > 1 else "gloo", timeout=datetime.timedelta(seconds=120),
                            **({"device_id": torch.device("cuda", local)} if world > 1 else {}))
    mesh = sf.Mesh((N_HEX, N_HEX, N_HEX * world), jitter=JITTER, seed=0)
    dop = fd.DistributedOperator(mesh, DEGREE, "dg", "fp64")
    xg = torch.tensor(np.random.default_rng(1).uniform(-1.0, 1.0, dop.partition.n_global), device="cuda")
    x = dop.scatter(xg)
    y = dop.initialize_dof_vector()
    flush = L2Flush()
    for _ in range(args.warmup):
        dop.vmult(y, x)
    dist.barrier()
    torch.cuda.synchronize()
    total = 0.0
    for _ in range(args.steps):
        flush()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        dop.vmult(y, x)
        b.record()
        torch.cuda.synchronize()
        total += a.elapsed_time(b)
    dist.barrier()
    total_ms = max_over_ranks(total, "cuda")
    value = dop.partition.n_global * args.steps / (total_ms / 1e3)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "DoF/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"DG SIPG Poisson vmult, P3 on 32 x 32 x {32 * world} x 6 Kuhn tets, "
                                       f"domain-decomposed over {world} ranks", "parallelism": f"dd{world}",
                           "l2": "flushed before every timed vmult (256 MB write, then 256 MB read of another buffer)"},
                "gpu_launches": 2 * args.steps}
        print(json.dumps(line), flush=True)
    dist.barrier()
    dist.destroy_process_group()


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    stream = torch.cuda.Stream()
    flush = L2Flush()

    mesh, op, x = build_problem("fp64")
    src = torch.tensor(x, device="cuda")
    dst = op.initialize_dof_vector()
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- headline: FP64 vmult, L2 flushed before every step
    barrier()
    with ClockSampler(local) as clk:
        t64 = timed_steps(lambda: op.vmult(dst, src, stream), args.steps, args.warmup, stream, flush)
    barrier()
    total_ms = max_over_ranks(sum(t64), "cuda")
    value = op.m() * args.steps * world / (total_ms / 1e3)

    # ---- per-kernel times (dominant kernel for the roofline)
    t_trace = timed_steps(lambda: op.vmult_phase(dst, src, 1, stream), args.steps, 2, stream, flush)
    t_apply = timed_steps(lambda: op.vmult_phase(dst, src, 2, stream), args.steps, 2, stream, flush)

    # ---- FP32 operator on the same mesh and input
    op32 = __import__("simplexfem").Operator(mesh, DEGREE, "dg", "fp32")
    src32 = src.float()
    dst32 = op32.initialize_dof_vector()
    t32 = timed_steps(lambda: op32.vmult(dst32, src32, stream), args.steps, args.warmup, stream, flush)
    value32 = op.m() * args.steps * world / (sum(t32) / 1e3)

    # ---- end to end through the public API on host vectors: fem_op_vmult_host
    # over K vectors (pinned host src -> device -> vmult -> host dst, the copies
    # of consecutive vectors overlapped), one call timed with CUDA events
    hsrc = torch.tensor(x).pin_memory()
    hdst = torch.empty(op.m(), dtype=torch.float64).pin_memory()
    for _ in range(args.warmup):
        op.vmult_host([hdst], [hsrc], stream)
    torch.cuda.synchronize()
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ea.record(stream)
    op.vmult_host([hdst] * args.steps, [hsrc] * args.steps, stream)
    eb.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(ea.elapsed_time(eb), "cuda")
    e2e_value = op.m() * args.steps * world / (e2e_ms / 1e3)
    nbytes = op.m() * 8
    op.vmult(dst, src, stream)
    torch.cuda.synchronize()
    assert torch.equal(hdst, dst.cpu()), "host-vector vmult differs from the device vmult"

    # the same copies without overlap: one vector at a time on one stream
    def e2e_serial_step():
        with torch.cuda.stream(stream):
            src.copy_(hsrc, non_blocking=True)
            op.vmult(dst, src, stream)
            hdst.copy_(dst, non_blocking=True)

    te2e_serial = timed_steps(e2e_serial_step, args.steps, args.warmup, stream, None)
    e2e_serial_value = op.m() * args.steps * world / (max_over_ranks(sum(te2e_serial), "cuda") / 1e3)

    # parity of the timed result against the oracle is covered by the tests;
    # here a cheap self-check that the benchmarked output is finite
    assert bool(torch.isfinite(dst).all())

    flops, alg_bytes = op.work()
    hbm, peak_src = measured_peaks()
    apply_ms = statistics.mean(t_apply)
    achieved_gbs = alg_bytes / (apply_ms / 1e3) / 1e9
    vm_ms = statistics.mean(t64)
    fp64_peak = fp64_peak_tflops() if rank == 0 else None
    solve = (mg_solve_bench(learned=not args.no_learned, cpu_baseline=not args.no_cpu_baseline)
             if (rank == 0 and not args.no_solve) else None)
    extra_cfg = None
    if rank == 0 and not args.no_extra:
        extra_cfg = cg_vmult_bench(min(args.steps, 100), 3, flush)
        extra_cfg["config4"] = batch_bench(min(args.steps, 20), 3, flush)
        extra_cfg["spmv"] = spmv_bench(min(args.steps, 50), 3, flush)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "DoF/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "precision": "fp64 (fp32 variant in extra)",
                       "l2": "flushed before every timed vmult (256 MB write, then 256 MB read of another buffer)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "e2e": {"value": e2e_value, "unit": "DoF/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes,
                    "how": "fem_op_vmult_host over `steps` host vectors (pinned), copies of consecutive "
                           "vectors overlapped with the apply; one vector at a time on one stream: "
                           f"{e2e_serial_value:.4g} DoF/s"},
            "roofline": {"bound": "hbm", "kernel": APPLY_KERNEL,
                         "achieved": achieved_gbs, "peak": hbm, "unit": "GB/s",
                         "frac": achieved_gbs / hbm, "traffic": APPLY_TRAFFIC_BYTES,
                         "note": f"algorithmic bytes of one vmult ({alg_bytes:.4g} B) over the apply kernel's "
                                 f"mean time; peak {peak_src} (copy); traffic = dram bytes read + written per "
                                 f"launch of the apply kernel in an ncu capture of this workload"},
            "fp64": {"achieved_tflops": flops / (vm_ms / 1e3) / 1e12, "peak_tflops_dgemm": fp64_peak,
                     "frac": (flops / (vm_ms / 1e3) / 1e12) / fp64_peak if fp64_peak else None,
                     "flops_per_vmult": flops},
            "kernels_ms": {"dg_trace_tma_kernel": statistics.mean(t_trace), "dg_apply_kernel": apply_ms,
                           "vmult": vm_ms},
            "extra": {"fp32_value": value32, "fp32_ms_per_step": sum(t32) / args.steps},
            "solve": solve,
            "configs": extra_cfg,
            "clocks": clk.summary(),
            "gpu_launches": 2 * args.steps,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_case(name, reps=3, variant=0):
    """One small workload of a single kernel family, for profiling (ncu -k ...):
    cg-p2-64 / cg-p3-64 / cg-p1-128 / cg-p2-128: CG vmults (default kernel variant, FP64 and
    FP32) on 64^3 or 128^3 x 6 tets, jitter 0.1h; mlp-64: eager V-cycles of the
    mixed multigrid with the learned finest-level smoother on CG P3 64^3
    (untrained network: the kernels do the same work); dg-p3-32: FP64 vmults of
    the headline DG P3 32^3 workload with kernel variant `variant`.  For the
    cg-* cases `variant` sets the kernel of the FP32 operator (e.g. 8: TF32
    tensor cores per cube).  solve-p3-64: the kernel timeline of one mixed
    MG-CG solve of the config-3 problem (CUPTI through torch.profiler): per
    kernel its launches and device time, and the time between kernels."""
    import torch
    import simplexfem as sf
    out = {"case": name}
    if name == "dg-p3-32":
        mesh = sf.Mesh(N_HEX, jitter=JITTER, seed=0)
        op = sf.Operator(mesh, DEGREE, "dg", "fp64")
        if variant:
            op.set_kernel_variant(variant)
        x = torch.rand(op.m(), dtype=op.dtype, device="cuda")
        y = op.initialize_dof_vector()
        for _ in range(reps):
            op.vmult(y, x)
        torch.cuda.synchronize()
        out.update({"m": op.m(), "variant": variant, "finite": bool(torch.isfinite(y).all())})
    elif name.startswith("cg-"):
        p, n = int(name[4]), int(name.split("-")[2])
        mesh = sf.Mesh(n, jitter=JITTER, seed=0)
        for prec in ("fp64", "fp32"):
            op = sf.Operator(mesh, p, "cg", prec)
            if variant and prec == "fp32":
                op.set_kernel_variant(variant)
            x = torch.rand(op.m(), dtype=op.dtype, device="cuda")
            y = op.initialize_dof_vector()
            for _ in range(reps):
                op.vmult(y, x)
            torch.cuda.synchronize()
            out[prec] = {"m": op.m(), "finite": bool(torch.isfinite(y).all())}
    elif name == "mlp-64":
        mesh = sf.Mesh(64)
        op = sf.Operator(mesh, 3, "cg", "fp64")
        mg = sf.Multigrid(op, precision="fp32", use_graph=False)
        mlp = sf.MLP(seed=1)
        mg.set_learned_smoother(mlp, fallback=False)
        b = torch.rand(op.m(), dtype=torch.float64, device="cuda")
        x = op.initialize_dof_vector()
        for _ in range(reps):
            mg.vmult(x, b)
        torch.cuda.synchronize()
        out["finite"] = bool(torch.isfinite(x).all())
        out["timed_out"] = mlp.timed_out()
    elif name == "solve-p3-64":
        from torch.profiler import profile, ProfilerActivity
        mesh = sf.Mesh(64)
        op = sf.Operator(mesh, 3, "cg", "fp64")
        b = sf.rhs(op, sf.sine_modes_rhs())
        x = op.initialize_dof_vector()
        mg = sf.Multigrid(op, precision="fp32", smoother_degree=3)
        cg = sf.SolverCG(op, mg)
        cg.solve(x, b, rtol=1e-8)  # warm-up (graph capture)
        plain = []
        for _ in range(reps):
            x.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = cg.solve(x, b, rtol=1e-8)
            torch.cuda.synchronize()
            plain.append(1e3 * (time.perf_counter() - t0))
        x.zero_()
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            r = cg.solve(x, b, rtol=1e-8)
            torch.cuda.synchronize()
        ev = sorted((e.time_range.start, e.time_range.end, e.name) for e in prof.events()
                    if e.device_type == torch.autograd.DeviceType.CUDA)
        busy, cur_s, cur_e = 0.0, None, None
        for s0, e0, _ in ev:
            if cur_e is None or s0 > cur_e:
                if cur_e is not None:
                    busy += cur_e - cur_s
                cur_s, cur_e = s0, e0
            else:
                cur_e = max(cur_e, e0)
        if cur_e is not None:
            busy += cur_e - cur_s
        span = (max(e for _, e, _ in ev) - ev[0][0]) if ev else 0.0
        per = {}
        for s0, e0, n in ev:
            c, t = per.get(n, (0, 0.0))
            per[n] = (c + 1, t + e0 - s0)
        top = sorted(per.items(), key=lambda kv: -kv[1][1])[:20]
        out.update({"iterations": r["iterations"], "solve_ms": [round(t, 2) for t in plain],
                    "launches": len(ev), "span_us": round(span, 1), "busy_us": round(busy, 1),
                    "gaps_us": round(span - busy, 1),
                    "kernels": [{"name": n[:100], "launches": c, "us": round(t, 1),
                                 "share_of_busy": round(t / busy, 3) if busy else None}
                                for n, (c, t) in top]})
    else:
        raise SystemExit(f"unknown case {name}")
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.case:
        run_case(args.case, variant=args.variant)
        return
    if args.impl == "reference":
        run_reference(args)
    elif args.dd:
        run_dd(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
