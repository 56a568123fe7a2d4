#!/usr/bin/env python3
"""Time to 1e-8 relative KKT residual with the B200 inner solve.

Workload (one step): a full PS-IPM solve, to relative KKT residual 1e-8
(primal, dual and gap, psipm_active_pool.py:2561-2637), of the seeded
synthetic min-cost-flow LP on a 200 x 250 directed grid plus 10% random
long-range arcs (m = 49,999 grounded rows, n = 219,010 arcs, all boxed),
with the spectral stable-column preconditioned normal equations solved on
the device in FP64.

Keys of the JSON line:
* value      seconds per LP solve with A already resident on the device
             (CUDA events on the library's stream around K solves); the
             PS-IPM loop keeps its vectors on the device (ipm_device.py);
* e2e        the same solve through the public API from host arrays
             (solve_standard): handle creation (A uploaded), c, b, u and the
             starting point uploaded, the solution copied back to the host;
* roofline   the persistent PCG kernel (k_pcg): algorithmic bytes of all
             its launches / its CUDA-event time, against the measured HBM
             copy bandwidth;
* spmv       the operator pair H p = A (w o (A' p)) + delta p inside k_pcg:
             its algorithmic bytes per product / its time per product (the
             kernel's own clock marks), against the same bandwidth;
* learned_selector  the same solve with the learned active-column selector
             (psipm_b200.learned, trained on solver traces of other seeds of
             this LP family) over --selector-steps solves; `value` stays the
             plain spectral rule;
* learned_fp32  the metric's other arm: the learned selector with the FP32
             preconditioner (FP64 PCG around an FP32 factor whose large
             fronts' updates run on the tensor cores, FP32 sweeps) over
             --fp32-steps solves, each bounded by --fp32-time-limit seconds
             (a solve that hits it reports status "time-limit");
* cpu_baseline  the CPU oracle (reference algorithm, SuperLU stand-in
             factor) timed on a bounded sample of the same LP (its first K
             outer iterations), next to the device's time for the same K
             outer iterations (same_work); the reference's complete solve,
             measured once elsewhere, is reported beside it, labelled.

``--impl reference`` times that CPU implementation alone (rank 0).
Multi-GPU: one process per GPU (torchrun), each solving its own seeded
instance (weak scaling, no collective on the data path); times are the max
over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "mf-psipm_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "time to 1e-8 rel. KKT residual (PS-IPM, device normal-equations PCG)"
WORKLOAD = ("min-cost flow LP, 200x250 directed grid (both orientations) + 10% random long-range arcs, "
            "m=49,999 grounded rows, n=219,010 boxed arcs, nnz=438,005; spectral stable-column "
            "preconditioner, FP64")
HBM_FALLBACK = 6650.0
# DRAM traffic of k_pcg, from one ncu capture on a B200 of the 151st k_pcg launch
# of `python bench.py --steps 1 --warmup 0 --no-cpu-baseline --selector none --fp32-steps 0`:
#   ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum
#       --clock-control none -k regex:k_pcg -s 150 -c 1 ...
# read 14,438,526,720 B + written 167,321,344 B in 10.243744 ms.  The bench scales
# this rate by its own average launch duration to give bytes per launch.
KPCG_DRAM_BYTES_PER_S = (14_438_526_720 + 167_321_344) / 0.010243744


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--workload", choices=("grid", "batch"), default="grid",
                    help="grid: the 200x250 network LP (the default line); batch: uneven random LPs "
                         "served several at a time, against the same LPs one after another")
    ap.add_argument("--count", type=int, default=256, help="LPs of the batch workload")
    ap.add_argument("--workers", type=int, default=8,
                    help="LPs in flight in the batch workload (0: choose the schedule with psipm_b200.batch.autotune "
                         "on 16 LPs of the batch, outside the timed region)")
    ap.add_argument("--rows", type=int, default=200)
    ap.add_argument("--cols", type=int, default=250)
    ap.add_argument("--cpu-sample-outer", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--selector", default="default",
                    help="learned column selector model for the learned arm ('default': the packaged model, "
                         "'none': no learned arm)")
    ap.add_argument("--selector-window", type=float, default=None)
    ap.add_argument("--selector-steps", type=int, default=3)
    ap.add_argument("--fp32-steps", type=int, default=1,
                    help="solves of the FP32 arm (learned selector + FP32 factor on the tensor cores)")
    ap.add_argument("--fp32-time-limit", type=float, default=60.0,
                    help="seconds per FP32-arm solve before it is reported as a time limit")
    return ap.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", HBM_FALLBACK)), "measured"
    return HBM_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_lp(args, rank: int):
    from psipm_b200 import synthetic

    return synthetic.grid_network(args.rows, args.cols, seed=1000 + rank)


def cpu_oracle_sample(lp, tol, outer, seconds_limit=25.0):
    """Reference algorithm (oracle) on the first `outer` outer iterations,
    stopped after `seconds_limit` seconds."""
    from oracle import ipm as OI
    from oracle import stable as OS

    t0 = time.perf_counter()
    solver = OS.SpectralOracle(lp.A, protected=~lp.pos)
    sol = OI.psipm_solve(lp, solver, tol=tol, max_outer=outer, time_limit=seconds_limit)
    seconds = time.perf_counter() - t0
    return seconds, max(1, sol.inner_iter), sol


def blas_threads() -> int:
    try:
        from threadpoolctl import threadpool_info

        info = threadpool_info()
        return int(max((i.get("num_threads", 1) for i in info), default=1))
    except Exception:
        return os.cpu_count() or 1


def flush_l2():
    import torch

    buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    buf.fill_(1.0)
    torch.cuda.synchronize()
    del buf


REFERENCE_RESULT = os.path.join(ROOT, "tests", "golden", "grid_200x250_result.json")


def reference_full_solve(args):
    """The unmodified reference's complete solve of this LP to 1e-8, measured
    once by tests/golden/make_golden.py (SuperLU stand-in factor) on the
    machine named in the file; reported beside the bounded sample, never as
    the sample's value."""
    if (args.rows, args.cols) != (200, 250) or not os.path.exists(REFERENCE_RESULT):
        return None
    with open(REFERENCE_RESULT) as f:
        d = json.load(f)
    return {"seconds": d["seconds"], "cpu_count": d.get("cpu_count"), "outer_iterations": d["outer_iter"],
            "pcg_iterations": d["pcg_iterations"], "objective": d["obj"], "status": d["status"],
            "note": "measured once by tests/golden/make_golden.py, not on this host"}


def sample_text(args, seconds):
    return (f"oracle (reference algorithm, SuperLU stand-in factor) on the first {args.cpu_sample_outer} "
            f"PS-IPM outer iterations of the same LP: {seconds:.2f} s measured here; the device's time for "
            f"the same {args.cpu_sample_outer} outer iterations is in same_work")


def run_reference(args, rank, world):
    if rank != 0:
        return None
    lp = make_lp(args, 0)
    threads = blas_threads()
    samples = []
    for step in range(args.warmup + args.steps):
        seconds, inner, sol = cpu_oracle_sample(lp, args.tol, args.cpu_sample_outer, seconds_limit=1e9)
        if step >= args.warmup:
            samples.append(seconds)
    mean = sum(samples) / len(samples)
    line = {
        "metric": METRIC, "value": mean, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * mean, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": WORKLOAD, "tol": args.tol,
                   "sample": f"first {args.cpu_sample_outer} PS-IPM outer iterations (bounded sample; a "
                             f"complete solve takes tens of minutes on the CPU)"},
        "cpu_baseline": {"value": mean, "unit": "s", "cores": threads, "kind": "port",
                         "sample": sample_text(args, mean)},
        "e2e": {"value": mean, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_full_solve": reference_full_solve(args),
    }
    return line


def load_selector(args):
    """The learned arm's model and window: the packaged model (trained on
    solver traces of other seeds of the same LP family) unless told otherwise."""
    if args.selector == "none":
        return None, 0.0
    from psipm_b200.learned import DEFAULT_MODEL, DEFAULT_WINDOW, SelectorModel

    path = DEFAULT_MODEL if args.selector == "default" else args.selector
    if not os.path.exists(path):
        return None, 0.0
    model = SelectorModel.load(path)
    model.path = path
    window = DEFAULT_WINDOW if args.selector_window is None else args.selector_window
    return model, window


def run_ours(args, rank, world, local_rank):
    import torch

    from psipm_b200.ipm_device import psipm_solve_resident, solve_standard
    from psipm_b200.device import NormalEquationsDevice
    from psipm_b200.replicas import max_over_ranks
    from psipm_b200.kkt import GpuSpectralStableColumnPreconditioner

    torch.cuda.set_device(local_rank)
    lp = make_lp(args, rank)
    m, n = lp.A.shape
    dev = NormalEquationsDevice(lp.A, device=local_rank)

    def one_solve(selector=None, window=0.0):
        solver = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, dev=dev, selector=selector,
                                                       selector_window=window)
        sol = psipm_solve_resident(lp, solver, tol=args.tol)
        if sol.status != "optimal":
            raise RuntimeError(f"solve ended {sol.status}")
        return sol, solver

    for _ in range(args.warmup):
        one_solve()
        flush_l2()
    dist = world > 1
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank)
    sampler.start()
    launches0 = dev.kernel_launches
    total = 0.0
    sols = []
    pcg_s = pcg_b = hp_s = 0.0
    pcg_launches = pcg_its = 0
    for _ in range(args.steps):
        torch.cuda.synchronize()
        dev.timer_start()
        sol, solver = one_solve()
        total += dev.timer_stop()
        sols.append(sol)
        pcg_s += solver.device_seconds
        pcg_b += solver.pcg_bytes
        pcg_launches += solver.pcg_launches
        pcg_its += solver.pcg_total_iterations
        hp_s += float(solver.pcg_phase_seconds[0])
        flush_l2()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = dev.kernel_launches - launches0
    per_step = max_over_ranks(total / args.steps)
    # ---- learned column selector (same LP, same timing; the plain rule is `value`) ----
    learned = None
    model, window = load_selector(args)
    if model is not None and args.selector_steps > 0:
        lt, lpcg, lfb, lref = 0.0, 0, 0, 0
        for _ in range(args.selector_steps):
            torch.cuda.synchronize()
            dev.timer_start()
            sol_l, solver_l = one_solve(model, window)
            lt += dev.timer_stop()
            lpcg += solver_l.pcg_total_iterations
            lfb += solver_l.selector_fallbacks
            lref += solver_l.learned_refreshes
            flush_l2()
        k = args.selector_steps
        learned = {"value": max_over_ranks(lt / k), "unit": "s", "steps": k, "model": os.path.basename(model.path),
                   "window": window, "pcg_iterations_per_step": lpcg / k, "learned_refreshes_per_step": lref / k,
                   "fallbacks_per_step": lfb / k, "objective": sol_l.obj, "status": sol_l.status,
                   "speedup_vs_plain": per_step / max_over_ranks(lt / k)}
    # ---- learned selector + FP32 factor and sweeps (the metric's other arm) ----
    fp32 = None
    if args.fp32_steps > 0:
        from psipm_b200 import _lib

        dev32 = NormalEquationsDevice(lp.A, device=local_rank, precision=_lib.FP32_PRECOND)
        ft, fpcg, fstatus, fobj = 0.0, 0, [], None
        try:
            for _ in range(args.fp32_steps):
                torch.cuda.synchronize()
                dev32.timer_start()
                solver32 = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, dev=dev32,
                                                                 precision=_lib.FP32_PRECOND, selector=model,
                                                                 selector_window=window)
                sol32 = psipm_solve_resident(lp, solver32, tol=args.tol, time_limit=args.fp32_time_limit)
                ft += dev32.timer_stop()
                fpcg += solver32.pcg_total_iterations
                fstatus.append(sol32.status)
                fobj = sol32.obj
                flush_l2()
        finally:
            dev32.close()
        k = args.fp32_steps
        fp32 = {"value": max_over_ranks(ft / k), "unit": "s", "steps": k,
                "precision": "FP32_PRECOND (FP64 PCG, FP32 factor with 3xTF32 tensor-core updates, FP32 sweeps)",
                "selector": os.path.basename(model.path) if model is not None else None,
                "status": fstatus, "objective": fobj, "pcg_iterations_per_step": fpcg / k,
                "time_limit_s": args.fp32_time_limit,
                "speedup_vs_plain_fp64": per_step / max_over_ranks(ft / k)}
    # ---- end to end through the public API, host buffers ----------------------
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sol_e2e, solver_e2e = solve_standard(lp, tol=args.tol, device=local_rank)
    x_host = np.array(sol_e2e.x)
    torch.cuda.synchronize()
    e2e = time.perf_counter() - t0
    h2d = (8 * (n + 1) + 12 * lp.A.nnz) + solver_e2e.h2d_bytes
    d2h = 8 * solver_e2e.candidates.size + solver_e2e.d2h_bytes
    solver_e2e.close()
    e2e = max_over_ranks(e2e)
    peak, peak_kind = measured_peaks()
    achieved = pcg_b / pcg_s / 1e9 if pcg_s > 0 else None
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None,
            "traffic": (KPCG_DRAM_BYTES_PER_S * pcg_s / pcg_launches) if pcg_launches else None,
            "traffic_note": "bytes per average k_pcg launch: the DRAM rate of one ncu-captured launch "
                            "(dram__bytes_read.sum + dram__bytes_write.sum) x this run's mean launch time",
            "kernel": "k_pcg", "peak_source": f"{peak_kind} hbm_gbs",
            "pcg_launches": pcg_launches, "pcg_iterations": pcg_its,
            "pcg_seconds_per_step": pcg_s / args.steps,
            "note": "the operator (~10 MB) is L2-resident and the factor panels (0.6-1 GB read per "
                    "preconditioner application) stream from HBM; the supernodal sweeps below the two "
                    "top tree levels are latency bound, so the HBM fraction stays low"}
    from psipm_b200.roofline import hp_bytes

    b_hp = hp_bytes(m, n, lp.A.nnz)
    hp_gbs = b_hp * pcg_its / hp_s / 1e9 if hp_s > 0 else None
    spmv = {"bound": "hbm", "achieved": hp_gbs, "peak": peak, "unit": "GB/s",
            "frac": (hp_gbs / peak) if hp_gbs else None, "bytes_per_product": b_hp,
            "us_per_product": 1e6 * hp_s / pcg_its if pcg_its else None,
            "kernel": "k_pcg operator phases: H p = A (w o (A' p)) + delta p with its dot-product reduction",
            "timing": "the PCG kernel's own %globaltimer marks (block 0) around each iteration's operator "
                      "pass, summed over the timed solves",
            "note": "this LP's operator (A twice, w, t, p, q: ~20 MB) stays in L2, so the HBM figure is a "
                    "byte rate, not DRAM traffic"}
    line = None
    if rank == 0:
        sol0 = sols[-1]
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            # the same bounded work on both sides: the first K outer iterations
            torch.cuda.synchronize()
            dev.timer_start()
            solver_s = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, dev=dev)
            sol_s = psipm_solve_resident(lp, solver_s, tol=args.tol, max_outer=args.cpu_sample_outer)
            gpu_same = dev.timer_stop()
            seconds, inner, sol_c = cpu_oracle_sample(lp, args.tol, args.cpu_sample_outer, seconds_limit=1e9)
            cpu = {"value": seconds, "unit": "s", "cores": blas_threads(), "kind": "port",
                   "sample": sample_text(args, seconds),
                   "same_work": {"outer_iterations": args.cpu_sample_outer, "cpu_s": seconds, "gpu_s": gpu_same,
                                 "ratio": seconds / gpu_same if gpu_same > 0 else None,
                                 "cpu_inner_iterations": int(sol_c.inner_iter),
                                 "gpu_inner_iterations": int(sol_s.inner_iter)},
                   "reference_full_solve": reference_full_solve(args)}
        line = {
            "metric": METRIC, "value": per_step, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * per_step, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "tol": args.tol, "l2": "256 MB L2 flush between steps",
                       "outer_iterations": sol0.outer_iter, "inner_iterations": sol0.inner_iter,
                       "objective": sol0.obj, "status": sol0.status,
                       "pcg_iterations_per_step": pcg_its / args.steps},
            "roofline": roof,
            "spmv": spmv,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "learned_selector": learned,
            "learned_fp32": fp32,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "lp_per_s": world / per_step,
        }
    return line


def run_batch(args, rank, world, local_rank):
    """Uneven random LPs (m ~ U{500..5000}, n = 3m, seeded) on this rank's GPU:
    the whole batch with --workers LPs in flight, then the same LPs one after
    another; value = batched LPs per second (nnz-balanced shares per rank)."""
    import torch

    from psipm_b200 import synthetic
    from psipm_b200.batch import autotune, solve_batch, solve_sequential
    from psipm_b200.replicas import max_over_ranks, partition_by_nnz

    torch.cuda.set_device(local_rank)
    lps = synthetic.random_lp_batch(count=args.count, seed=4000)
    mine = [lps[k] for k in partition_by_nnz([lp.A.nnz for lp in lps], world)[rank]]
    workers, grid_blocks, tuned = args.workers, None, None
    if workers <= 0:  # the tuner's trials also warm the device up
        tuned = autotune(mine, sample=16, device=local_rank)
        workers, grid_blocks = tuned.workers, tuned.grid_blocks
    else:
        solve_batch(mine[: min(len(mine), workers)], workers=workers, device=local_rank)  # warm-up
    bat = solve_batch(mine, workers=workers, device=local_rank, grid_blocks=grid_blocks)
    seconds = max_over_ranks(bat.seconds)
    seq = solve_sequential(mine, device=local_rank) if world == 1 else None
    if rank != 0:
        return None
    return {
        "metric": "LPs solved to 1e-8 per second (batched serving)", "value": len(lps) / seconds,
        "unit": "LP/s", "n_gpus": world, "steps": 1, "warmup": 1, "ms_per_step": 1e3 * seconds,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{len(lps)} uneven random LPs, m ~ U{{500..5000}}, n = 3m, 5 nonzeros per column, "
                               f"seeds 4001..{4000 + len(lps)}", "workers": workers, "grid_blocks": grid_blocks,
                   "tol": 1e-8},
        "autotune": None if tuned is None else {"workers": tuned.workers, "grid_blocks": tuned.grid_blocks,
                                                 "trials": tuned.trials},
        "p50_s": bat.percentile(50), "p99_s": bat.percentile(99),
        "optimal": sum(s == "optimal" for s in bat.status), "errors": bat.errors[:5],
        "sequential": None if seq is None else {"value": seq.lps_per_second, "p50_s": seq.percentile(50),
                                                "p99_s": seq.percentile(99), "seconds": seq.seconds},
    }


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = world > 1
    if dist:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                             device_id=torch.device("cuda", local_rank))
    try:
        if args.impl == "reference":
            line = run_reference(args, rank, world)
        elif args.workload == "batch":
            line = run_batch(args, rank, world, local_rank)
        else:
            line = run_ours(args, rank, world, local_rank)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
