"""Benchmark of the BoSSS linear-solver hot path on B200.

Workload (one "step"): one complete solve of the 3-D SIP Poisson system on 64^3 hexahedra, p = 3 (Np = 20,
5,242,880 unknowns, 1,810,432 blocks of 20x20 in FP64), seeded 16-mode sine right-hand side, to relative residual
1e-10 with FlexGMRES(30) preconditioned by one 3-level p-multigrid V-cycle (p = 3 -> 2 -> 1, block-Jacobi
smoothing, 10 post-smoother sweeps).  `value` is the time to that residual for the fastest available path
(FP32 preconditioner inside FP64 FGMRES), `plain_fp64` the same for the all-FP64 path, and `spmv` the stand-alone
FP64 block SpMV on the same matrix, 100 repeats.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one process per GPU) every rank solves its own copy of the system: the path has no
exchange step at one system per GPU, so ranks are independent replicas and no collective runs on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-1e-10 residual & iters: learned+mixed vs plain FP64 GPU; SpMV GB/s"
WORKLOAD = "SIP DG Poisson 3-D 64^3 hex, p=3 (Np=20, 5.24M DOF), FlexGMRES(30) + 3-level p-MG (3->2->1), BJ smoothing"
TOL = 1e-10
# p-multigrid settings shared by every path (PmgConfig.cs:80-245 with UseILU = false; the coarsest p = 1 level,
# a direct solve in the reference, is block-Jacobi PCG to 0.1 reduction, at most 60 iterations)
SOLVER_PARAMS = dict(NoOfPostSmootherSweeps=10, BlockJacobiIterations=1, CoarseSolver="pcg", CoarseTolerance=0.1,
                     CoarseMaxIterations=60, SubLevelReduction=0.1, SubLevelMaxIterations=100)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=64, help="cells per direction")
    ap.add_argument("--p", type=int, default=3)
    ap.add_argument("--spmv-repeats", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--spmv-only", action="store_true",
                    help="only the stand-alone SpMV timing (profiling runs; prints a short JSON line)")
    ap.add_argument("--seed", type=int, default=0)
    return ap.parse_args()


def levels_for(p: int):
    from bosss_b200.assembly import np_of
    return tuple(np_of(3, q) for q in range(p, 0, -1))


def spmv_bytes(s) -> int:
    """Algorithmic bytes of one y = A*x: blocks, column indices, row pointers (int64), x once, y written."""
    return s.nnzb * s.Np * s.Np * 8 + s.nnzb * 4 + (s.nb + 1) * 8 + 2 * s.N * 8


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._proc = None

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                           "--format=csv,noheader,nounits", "-lms", "200"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (FileNotFoundError, OSError):
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def max_over_ranks(v: float, ws: int) -> float:
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ----------------------------------------------------------------------------------------------------------------
# CPU side: the oracle (CPU restatement of the reference algorithms), used as baseline only
# ----------------------------------------------------------------------------------------------------------------
class CpuReference:
    """The CPU restatement of the reference algorithms (oracle/), set up once on the workload.

    One sample = one SpMV plus one FGMRES solve limited to its first restart test (two preconditioner
    applications = two outer iterations); the per-iteration time times the iteration count the solve needs
    projects the time to 1e-10.  Reported as a baseline only.
    """

    def __init__(self, s, threads: int):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        self.O = O
        self.threads = O.set_threads(threads)
        self.s = s
        self.B = O.Bsr.of(s)
        t0 = time.perf_counter()
        vals, L = O.change_of_basis(self.B)
        self.t_cob = time.perf_counter() - t0

        class T:
            Np, row_ptr, col_idx, values = s.Np, s.row_ptr, s.col_idx, vals
        self.Bt = O.Bsr.of(T)
        self._keep = (vals, L)
        self.bt = np.einsum("cij,cj->ci", L.reshape(-1, s.Np, s.Np), s.rhs.reshape(-1, s.Np)).reshape(-1)
        cfg = O.SolverConfig(solver=O.FGMRES_PMG, tol=TOL, top_mode=O.TERM_RELATIVE, level_keep=levels_for(s.p),
                             coarse_kind=O.COARSE_PCG, coarse_tol=SOLVER_PARAMS["CoarseTolerance"],
                             coarse_max_iter=SOLVER_PARAMS["CoarseMaxIterations"],
                             sub_reduction=SOLVER_PARAMS["SubLevelReduction"],
                             sub_max_iter=SOLVER_PARAMS["SubLevelMaxIterations"], max_iter=1, min_iter=0)
        t0 = time.perf_counter()
        self.solver = O.PersistentSolver(self.Bt, cfg)
        self.t_setup = time.perf_counter() - t0
        self.x = np.random.default_rng(0).standard_normal(s.N)
        self.y = np.zeros(s.N)

    def sample(self, iters_needed: int | None):
        t0 = time.perf_counter()
        self.O.spmv(self.B, 1.0, self.x, 0.0, self.y)
        t_spmv = time.perf_counter() - t0
        t0 = time.perf_counter()
        r = self.solver.solve(self.bt)
        t_solve = time.perf_counter() - t0
        t_iter = t_solve / max(r.iterations, 1)
        out = {"t_spmv": t_spmv, "spmv_gbs": spmv_bytes(self.s) / t_spmv / 1e9, "t_change_of_basis": self.t_cob,
               "t_solver_setup": self.t_setup, "t_outer_iteration": t_iter, "sample_iterations": r.iterations,
               "threads": self.threads}
        if iters_needed:
            out["projected_time_to_tol"] = t_iter * iters_needed
        return out


def run_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from bosss_b200 import assembly as A
    threads = os.cpu_count() or 1
    s = A.poisson_3d(args.n, args.p, seed=args.seed)
    iters = _reference_iterations(args)
    ref = CpuReference(s, threads)
    samples = []
    for i in range(args.warmup + args.steps):
        r = ref.sample(iters)
        if i >= args.warmup:
            samples.append(r)
    v = statistics.median([r["projected_time_to_tol"] for r in samples])
    threads = ref.threads
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded sine-mode RHS, assembled SIP operator)",
        "config": {"workload": WORKLOAD, "l2": "inputs larger than L2 (5.8 GB matrix)"},
        "cpu_baseline": {"value": v, "unit": "s", "cores": threads, "kind": "port",
                         "sample": f"per step: one SpMV and an FGMRES solve stopped at its first test (2 outer "
                                   f"iterations = 2 V-cycles), per-iteration time x {iters} iterations (the CPU "
                                   f"restatement's own count on this system); SpMV {samples[-1]['spmv_gbs']:.1f} GB/s"},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "detail": samples[-1],
    }
    print(json.dumps(line), flush=True)


def _reference_iterations(args):
    """Outer iteration count of the oracle on this system (committed with the script that produced it)."""
    path = os.path.join(ROOT, "tests", "golden", "c2_oracle_solve.json")
    if os.path.exists(path) and args.n == 64 and args.p == 3 and args.seed == 0:
        return int(json.load(open(path))["iterations"])
    return 9


# ----------------------------------------------------------------------------------------------------------------
# GPU side
# ----------------------------------------------------------------------------------------------------------------
def run_ours(args):
    import torch
    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from bosss_b200 import assembly as A
    from bosss_b200 import native as nat
    from bosss_b200.solvers import BlockMsrMatrix, FGMRESConfig, MultigridOperator, PmgConfig
    nat.check(nat.lib().bsgpu_set_device(local))

    s = A.poisson_3d(args.n, args.p, seed=args.seed)
    M = BlockMsrMatrix.from_system(s)
    t0 = time.perf_counter()
    op = MultigridOperator(M)
    torch.cuda.synchronize()
    t_cob = time.perf_counter() - t0
    Aop = op.OperatorMatrix

    # --- SpMV alone (dominant kernel): CUDA events on the launching stream
    x = torch.randn(s.N, dtype=torch.float64, device=dev)
    y = torch.zeros_like(x)
    stream = torch.cuda.current_stream()
    for _ in range(5):
        Aop.SpMV(1.0, x, 0.0, y)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.spmv_repeats)]
    for i in range(args.spmv_repeats):
        ev[2 * i].record(stream)
        Aop.SpMV(1.0, x, 0.0, y)
        ev[2 * i + 1].record(stream)
    torch.cuda.synchronize()
    spmv_ms = [ev[2 * i].elapsed_time(ev[2 * i + 1]) for i in range(args.spmv_repeats)]
    spmv_avg = sum(spmv_ms) / len(spmv_ms)
    nbytes = spmv_bytes(s)
    spmv_gbs = nbytes / (spmv_avg * 1e-3) / 1e9
    # FP32 copy (preconditioner operator)
    A32 = Aop.ToSingle()
    x32 = x.float()
    y32 = torch.zeros_like(x32)
    for _ in range(5):
        A32.SpMV(1.0, x32, 0.0, y32)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.spmv_repeats):
        A32.SpMV(1.0, x32, 0.0, y32)
    e1.record(stream)
    torch.cuda.synchronize()
    spmv32_ms = e0.elapsed_time(e1) / args.spmv_repeats
    nbytes32 = s.nnzb * s.Np * s.Np * 4 + s.nnzb * 4 + (s.nb + 1) * 8 + 2 * s.N * 4
    del A32, x32, y32
    if args.spmv_only:
        print(json.dumps({"spmv_fp64_gbs": spmv_gbs, "spmv_fp64_ms": spmv_avg, "bytes": nbytes,
                          "spmv_fp32_gbs": nbytes32 / (spmv32_ms * 1e-3) / 1e9, "n": args.n, "p": args.p}))
        return

    pmg = PmgConfig(DegreeHierarchy=levels_for(args.p), **SOLVER_PARAMS)
    mk = lambda mixed: FGMRESConfig(ConvergenceCriterion=TOL, termination="relative", MaxKrylovDim=30,
                                    Preconditioners=[pmg], MixedPrecision=mixed).CreateInstance(op)
    fast = mk(True)
    plain = mk(False)
    B = torch.from_numpy(s.rhs).to(dev)
    X = torch.zeros_like(B)

    def solve(slv):
        X.zero_()
        slv.Solve(X, B)
        return slv

    # plain FP64 path: one warm-up, two timed
    solve(plain)
    plain_t = []
    for _ in range(2):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        solve(plain)
        b.record(stream)
        torch.cuda.synchronize()
        plain_t.append(a.elapsed_time(b) * 1e-3)
    plain_iters = plain.ThisLevelIterations
    plain_res = _true_relres(Aop, op, X, B, s)
    x_plain = X.clone()

    for _ in range(args.warmup):
        solve(fast)
    torch.cuda.synchronize()
    barrier(ws)
    launches0 = nat.launch_count()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            solve(fast)
        b.record(stream)
        torch.cuda.synchronize()
    launches = nat.launch_count() - launches0
    t_fast = a.elapsed_time(b) * 1e-3 / args.steps
    barrier(ws)
    t_fast_max = max_over_ranks(t_fast, ws)
    fast_iters = fast.ThisLevelIterations
    fast_res = _true_relres(Aop, op, X, B, s)
    sol_diff = (torch.linalg.norm(X - x_plain) / torch.linalg.norm(x_plain)).item()

    # --- end to end through the public API with host (pinned) buffers
    bh = torch.from_numpy(s.rhs).pin_memory()
    xh = torch.zeros(s.N, dtype=torch.float64).pin_memory()
    bn, xn = bh.numpy(), xh.numpy()
    e2e = []
    for i in range(1 + min(args.steps, 3)):
        xn[:] = 0.0
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fast.Solve(xn, bn)
        b.record(stream)
        torch.cuda.synchronize()
        if i > 0:
            e2e.append(a.elapsed_time(b) * 1e-3)
    e2e_t = max_over_ranks(sum(e2e) / len(e2e), ws)

    clocks = clk.summary()
    if rank != 0:
        return
    cpu = None
    if not args.no_cpu_baseline and ws == 1:
        threads = os.cpu_count() or 1
        try:
            cpu = CpuReference(s, threads).sample(plain_iters)
            threads = cpu["threads"]
            cpu_line = {"value": cpu["projected_time_to_tol"], "unit": "s", "cores": threads, "kind": "port",
                        "sample": "CPU restatement: FGMRES solve stopped at its first test (2 V-cycles), "
                                  f"per-iteration time x {plain_iters} iterations (the GPU FP64 count); one SpMV "
                                  f"at {cpu['spmv_gbs']:.1f} GB/s",
                        "detail": cpu}
        except Exception as e:  # the baseline is reported only
            cpu_line = {"value": None, "unit": "s", "cores": threads, "kind": "port", "sample": f"failed: {e}"}
    else:
        cpu_line = None
    peaks = _peaks()
    line = {
        "metric": METRIC, "value": t_fast_max, "unit": "s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_fast_max * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (outer) / f32 (preconditioner)",
        "data": "synthetic (seeded 16-mode sine RHS, SIP operator assembled in-repo)",
        "config": {"workload": WORKLOAD, "dof": s.N, "blocks": s.nnzb, "tol": TOL,
                   "l2": "inputs larger than L2 (5.8 GB FP64 matrix per SpMV)",
                   "parallelism": f"replicas x{ws}"},
        "iters": fast_iters, "final_relres": fast_res,
        "plain_fp64": {"value": max_over_ranks(min(plain_t), 1), "unit": "s", "iters": plain_iters,
                       "final_relres": plain_res},
        "speedup_vs_plain_fp64": min(plain_t) / t_fast_max,
        "rel_diff_vs_plain_fp64_solution": sol_diff,
        "spmv": {"gbs": spmv_gbs, "ms": spmv_avg, "bytes": nbytes, "repeats": args.spmv_repeats,
                 "fp32_gbs": nbytes32 / (spmv32_ms * 1e-3) / 1e9, "fp32_ms": spmv32_ms},
        "setup": {"change_of_basis_s": t_cob},
        "roofline": {"bound": "hbm", "achieved": spmv_gbs, "peak": peaks[0], "unit": "GB/s",
                     "frac": spmv_gbs / peaks[0], "traffic": _traffic_per_launch(),
                     "kernel": "spmv_uniform_kernel<double,20,2,0> (FP64 block SpMV, 64^3 p=3)",
                     "peak_source": peaks[1]},
        "e2e": {"value": e2e_t, "unit": "s", "h2d_bytes_per_step": 2 * s.N * 8, "d2h_bytes_per_step": s.N * 8},
        "gpu_launches": launches,
        "clocks": clocks,
        "cpu_baseline": cpu_line,
    }
    print(json.dumps(line), flush=True)


def _true_relres(Aop, op, X, B, s):
    """|B - A X| / |B| in the original basis (A = the assembled matrix)."""
    import torch
    r = B.clone()
    op.BaseMatrix.SpMV(-1.0, X, 1.0, r)
    return (torch.linalg.norm(r) / torch.linalg.norm(B)).item()


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    return 6650.0, "fallback 6.65 TB/s (of fallback)"


def _traffic_per_launch():
    p = os.path.join(ROOT, "profiles", "spmv_traffic.json")
    if os.path.exists(p):
        return json.load(open(p)).get("bytes_per_launch")
    return None


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
