"""Many independent systems on one GPU: one solver handle (with its own CUDA stream) per system, several host
threads driving them at once.

The reference solves independent systems one after another, each with its own ``ISolverSmootherTemplate``
instance (``UniSolver.Solve``, ``UniSolver.cs:588,623``).  Here a wave of systems is set up on the calling thread
(device allocations and factorisations), then solved concurrently: every ``GpuSolver.Solve`` call releases the
interpreter lock inside the C library, and each handle's kernels run on its own stream, so the small systems of a
batch fill the GPU together.  Setup and teardown stay on the calling thread so that no allocation runs while
another thread is capturing a CUDA graph.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, Iterable, List, Optional

import numpy as np


@dataclass
class BatchResult:
    index: int
    dof: int
    setup_s: float
    solve_s: float          # wall time of this system's solve while the others of its wave ran beside it
    iterations: int
    converged: bool
    relres: float
    info: dict = field(default_factory=dict)


@dataclass
class BatchSummary:
    results: List[BatchResult]
    solve_wall_s: float     # sum over waves of the wave's solve makespan
    setup_wall_s: float

    @property
    def dof(self) -> int:
        return sum(r.dof for r in self.results)

    def percentile(self, q: float, key: str = "solve_s") -> float:
        return float(np.percentile([getattr(r, key) for r in self.results], q))

    def as_dict(self) -> dict:
        return {"problems": len(self.results), "dof": self.dof, "solve_wall_s": self.solve_wall_s,
                "setup_wall_s": self.setup_wall_s,
                "dof_per_s_solve": self.dof / self.solve_wall_s if self.solve_wall_s > 0 else None,
                "dof_per_s_with_setup": self.dof / (self.solve_wall_s + self.setup_wall_s),
                "latency_p50_s": self.percentile(50), "latency_p99_s": self.percentile(99),
                "setup_p50_s": self.percentile(50, "setup_s"), "setup_p99_s": self.percentile(99, "setup_s"),
                "iterations_p50": float(np.percentile([r.iterations for r in self.results], 50)),
                "iterations_max": max(r.iterations for r in self.results),
                "all_converged": all(r.converged for r in self.results),
                "relres_max": max(r.relres for r in self.results),
                # set-up phases summed over the problems (matrix upload and layout, change of basis, solvers of
                # every configuration with their factorisations, autotuning and graph recordings)
                "setup_phases_s": {k: float(sum(r.info.get(k, 0.0) for r in self.results))
                                   for k in ("matrix_s", "change_of_basis_s", "solvers_s")}}


class BatchSolver:
    """Solves a stream of systems in waves of ``concurrency``.

    ``make_solver(op)`` returns a ``GpuSolver`` for a ``MultigridOperator``, or a dict {name: GpuSolver} to solve
    every system with several configurations (each configuration runs as its own concurrent wave, one after the
    other, from a zero initial guess).  ``prepare(op, system)`` (optional) runs after the operator is built, e.g.
    to set the cell graph of the learned stage.
    """

    def __init__(self, make_solver: Callable, concurrency: int = 8, prepare: Optional[Callable] = None,
                 device: str = "cuda", one_graph: Iterable[str] = ()):
        if concurrency < 1:
            raise ValueError("concurrency must be at least 1")
        self.make_solver = make_solver
        self.concurrency = concurrency
        self.prepare = prepare
        self.device = device
        # configuration names whose waves run as one CUDA graph (GpuBatch; their solvers are created with
        # FGMRESConfig(Graph="solve")); the other configurations run from host threads
        self.one_graph = set(one_graph)

    def _setup(self, system):
        import torch
        from .solvers import BlockMsrMatrix, MultigridOperator
        t0 = time.perf_counter()
        M = BlockMsrMatrix.from_system(system)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        op = MultigridOperator(M)
        if self.prepare is not None:
            self.prepare(op, system)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        slv = self.make_solver(op)
        slvs = slv if isinstance(slv, dict) else {"": slv}
        B = torch.from_numpy(np.ascontiguousarray(system.rhs, np.float64)).to(self.device)
        X = {k: torch.zeros_like(B) for k in slvs}
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        return dict(M=M, op=op, slv=slvs, B=B, X=X, setup_s=t3 - t0, dof=int(system.N),
                    phases={"matrix_s": t1 - t0, "change_of_basis_s": t2 - t1, "solvers_s": t3 - t2})

    @staticmethod
    def _collect(name, wave, times, results, on_result):
        import torch
        for i, w in wave:
            r = w["B"].clone()
            w["M"].SpMV(-1.0, w["X"][name], 1.0, r)
            rel = (torch.linalg.norm(r) / torch.linalg.norm(w["B"])).item()
            slv = w["slv"][name]
            res = BatchResult(index=i, dof=w["dof"], setup_s=w["setup_s"], solve_s=times[i],
                              iterations=slv.ThisLevelIterations, converged=slv.Converged, relres=rel,
                              info=dict(w.get("phases", {})))
            results.setdefault(name, []).append(res)
            if on_result is not None:
                on_result(name, res, w)

    def run(self, systems: Iterable, on_result: Optional[Callable] = None) -> Dict[str, BatchSummary]:
        """Returns one summary per configuration name ("" for a single solver).  Per-system solve_s: the host wall
        time of its Solve call (threads), or the device time from the wave's graph launch to the end of its branch
        (one-graph waves)."""
        results: Dict[str, List[BatchResult]] = {}
        solve_wall: Dict[str, float] = {}
        setup_wall = 0.0
        it = iter(systems)
        index = 0
        while True:
            wave = []
            t0 = time.perf_counter()
            for sysm in it:
                wave.append((index, self._setup(sysm)))
                index += 1
                if len(wave) == self.concurrency:
                    break
            if not wave:
                break
            setup_wall += time.perf_counter() - t0
            for name in wave[0][1]["slv"]:
                times = {}
                errors = []
                if name in self.one_graph:
                    from .solvers import GpuBatch
                    t1 = time.perf_counter()
                    gb = GpuBatch([w["slv"][name] for _, w in wave])  # records the wave's graph (set-up)
                    setup_wall += time.perf_counter() - t1
                    a = time.perf_counter()
                    try:
                        gb.Solve([w["X"][name] for _, w in wave], [w["B"] for _, w in wave])
                    finally:
                        lat = gb.Latencies()
                        gb.Dispose()
                    solve_wall[name] = solve_wall.get(name, 0.0) + time.perf_counter() - a
                    for (i, _), sec in zip(wave, lat):
                        times[i] = sec
                    self._collect(name, wave, times, results, on_result)
                    continue

                def work(i, w, key):
                    try:
                        a = time.perf_counter()
                        w["slv"][key].Solve(w["X"][key], w["B"])
                        times[i] = time.perf_counter() - a
                    except Exception as e:  # re-raised on the calling thread
                        errors.append(e)

                threads = [threading.Thread(target=work, args=(i, w, name)) for i, w in wave]
                a = time.perf_counter()
                for t in threads:
                    t.start()
                for t in threads:
                    t.join()
                solve_wall[name] = solve_wall.get(name, 0.0) + time.perf_counter() - a
                if errors:
                    raise errors[0]
                self._collect(name, wave, times, results, on_result)
            for i, w in wave:
                for slv in w["slv"].values():
                    slv.Dispose()
                w["op"].Dispose()
                w["M"].Dispose()
            del wave
        return {k: BatchSummary(results=v, solve_wall_s=solve_wall[k], setup_wall_s=setup_wall)
                for k, v in results.items()}
