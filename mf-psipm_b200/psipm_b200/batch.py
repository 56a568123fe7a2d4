"""Serving many small LPs at once on one GPU.

The batched configuration asks for many uneven LPs from the random-LP
generator (m ~ U{500..5,000}, n = 3m) solved together and compared with the
same LPs solved one after another.  Each LP keeps its own handle, stream and
device-resident PS-IPM loop (``ipm_device.psipm_solve_resident``); ``workers``
host threads each take the next LP from a queue, so up to ``workers`` LPs are
in flight at once.  Every C-ABI call releases the interpreter lock while it
waits for its stream, and every handle's persistent kernels use a share of
the GPU (``psipm_set_grid``), so the LPs' kernels run side by side instead of
one LP's launches idling the rest of the GPU.

:func:`solve_batch` returns per-LP wall times (submission to result) and the
aggregate LPs per second; :func:`solve_sequential` is the baseline, one LP
at a time with the whole GPU.  :func:`autotune` picks the schedule (LPs in
flight and each LP's share of the persistent grid) by timing candidates on a
sample of the batch.
"""

from __future__ import annotations

import queue
import threading
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np


@dataclass
class BatchResult:
    seconds: float                      # wall time of the whole batch
    lp_seconds: List[float]             # per LP: start of its solve to its result
    status: List[str]
    objectives: List[float]
    pcg_iterations: List[int]
    workers: int
    errors: List[str] = field(default_factory=list)

    @property
    def lps_per_second(self) -> float:
        return len(self.lp_seconds) / self.seconds if self.seconds > 0 else float("nan")

    def percentile(self, q: float) -> float:
        return float(np.percentile(np.asarray(self.lp_seconds), q))


def _solve_one(lp, tol: float, device: int, grid_blocks: int):
    from .ipm_device import psipm_solve_resident
    from .kkt import GpuSpectralStableColumnPreconditioner

    solver = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, device=device)
    try:
        if grid_blocks:
            solver.dev.set_grid(grid_blocks)
        sol = psipm_solve_resident(lp, solver, tol=tol)
        return sol.status, float(sol.obj), int(sol.pcg_iterations)
    finally:
        solver.close()


def solve_batch(lps, workers: int = 8, tol: float = 1e-8, device: int = 0,
                grid_blocks: Optional[int] = None) -> BatchResult:
    """Solve ``lps`` with ``workers`` LPs in flight; ``grid_blocks`` per LP
    (default: the GPU's co-resident grid divided among the workers)."""
    import torch

    torch.cuda.set_device(device)
    if grid_blocks is None:
        sms = torch.cuda.get_device_properties(device).multi_processor_count
        grid_blocks = max(8, (4 * sms) // max(1, workers))
    n = len(lps)
    status: List[str] = [""] * n
    objs = [float("nan")] * n
    its = [0] * n
    secs = [0.0] * n
    errors: List[str] = []
    todo: "queue.Queue[int]" = queue.Queue()
    for k in range(n):
        todo.put(k)
    lock = threading.Lock()

    def work():
        torch.cuda.set_device(device)
        while True:
            try:
                k = todo.get_nowait()
            except queue.Empty:
                return
            t0 = time.perf_counter()
            try:
                status[k], objs[k], its[k] = _solve_one(lps[k], tol, device, grid_blocks)
            except Exception as exc:  # reported, the other LPs go on
                status[k] = "error"
                with lock:
                    errors.append(f"LP {k}: {exc}")
            secs[k] = time.perf_counter() - t0

    t0 = time.perf_counter()
    threads = [threading.Thread(target=work, daemon=True) for _ in range(max(1, workers))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    return BatchResult(time.perf_counter() - t0, secs, status, objs, its, workers, errors)


def solve_sequential(lps, tol: float = 1e-8, device: int = 0) -> BatchResult:
    """The baseline: one LP at a time, each with the whole GPU."""
    return solve_batch(lps, workers=1, tol=tol, device=device, grid_blocks=0)


@dataclass
class Schedule:
    workers: int        # LPs in flight
    grid_blocks: int    # persistent-kernel blocks per LP (psipm_set_grid; 0 = the whole co-resident grid)
    lps_per_second: float
    trials: List[dict] = field(default_factory=list)


def schedule_candidates(sms: int, max_workers: int = 16) -> List[tuple]:
    """(workers, grid_blocks) pairs the tuner times: 1, 2, 4, ... LPs in flight,
    each with its share of the co-resident grid (4 blocks per SM divided among
    them) and with half that share."""
    out = []
    w = 1
    while w <= max_workers:
        share = max(8, (4 * sms) // w)
        out.append((w, 0 if w == 1 else share))
        if w > 1 and share // 2 >= 8:
            out.append((w, share // 2))
        w *= 2
    return out


def autotune(lps, sample: int = 16, candidates: Optional[List[tuple]] = None, tol: float = 1e-8,
             device: int = 0, run=None) -> Schedule:
    """Choose the batch schedule by timing each candidate on the same sample.

    The sample is ``sample`` LPs spread over the batch (every k-th, so their
    sizes follow the batch's distribution); each candidate solves the whole
    sample with :func:`solve_batch`, and the schedule with the most LPs per
    second wins (ties: fewer workers).  ``run(lps, workers, grid_blocks)``
    replaces :func:`solve_batch` (tests use a timing model).
    """
    if not lps:
        raise ValueError("no LPs to tune on")
    if candidates is None:
        import torch

        sms = torch.cuda.get_device_properties(device).multi_processor_count
        candidates = schedule_candidates(sms)
    if run is None:
        def run(sub, workers, grid_blocks):
            return solve_batch(sub, workers=workers, tol=tol, device=device, grid_blocks=grid_blocks)
    step = max(1, len(lps) // max(1, sample))
    sub = list(lps[::step])[:max(1, sample)]
    best, trials = None, []
    for workers, grid_blocks in candidates:
        res = run(sub, workers, grid_blocks)
        rate = res.lps_per_second
        trials.append(dict(workers=workers, grid_blocks=grid_blocks, lps_per_second=rate,
                           optimal=sum(st == "optimal" for st in res.status)))
        if best is None or rate > best[2] * (1.0 + 1e-9):
            best = (workers, grid_blocks, rate)
    return Schedule(best[0], best[1], best[2], trials)
