"""Learned active-column selector: model, device training, solver traces.

The reference chooses the preconditioner's active columns by a leverage
score with a diagonal (Jacobi) approximation of ``H`` (``_scores`` /
``_refresh_core``, psipm_stable_preconditioner.py:293-371).  This module adds
a small network that re-scores the candidate columns before the same refresh
step, trained to predict each column's *true* leverage
``w_j a_j' H^{-1} a_j`` from six per-column inputs (log theta, log nnz,
log column norm, log mu, previous core membership and the rule's own log
score).  A second output, averaged over the candidates, votes for the
factor's first diagonal-shift index.

* :class:`SelectorModel` holds the parameters (FP32 master copy; the solver
  uses the BF16-rounded weights and FP32 biases).
* :class:`DeviceTrainer` trains it with the library's own CUDA kernels
  (``psipm_mlp_grad_dev`` / ``psipm_mlp_adam_dev``); PyTorch only provides
  the device buffers.
* :func:`collect_traces` runs the device solver with the plain spectral rule
  on an LP and records, at every core refresh, the inputs of a sample of
  candidates and their true leverage, estimated on the device by Hutchinson
  probes of ``D^{1/2} A' H^{-1} A D^{1/2}`` with ``H`` factored exactly (a
  second handle whose core holds every candidate).

The solver side (``kkt.GpuSpectralStableColumnPreconditioner(selector=...)``)
falls back to the plain rule whenever a learned core turns out poor by the
reference's own signals (psipm_spectral_preconditioner.py:420-467).

Command line (training on solver traces, on a GPU)::

    python -m psipm_b200.learned --rows 200 --cols 250 --train 0-19 --out model.npz
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import time
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np

from . import _lib

N_IN, N_HID, N_OUT = _lib.MLP_INPUTS, 64, 2
N_WEIGHTS, N_BIASES, N_PARAMS = _lib.MLP_WEIGHTS, _lib.MLP_BIASES, _lib.MLP_PARAMS
# packaged model: trained on device traces of 200 x 250 grid networks (seeds 1100-1111)
DEFAULT_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "selector_grid.npz")
DEFAULT_WINDOW = 0.0


def _bf16_bits(x: np.ndarray) -> np.ndarray:
    bits = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return (((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


class SelectorModel:
    """Parameters of the 6 -> 64 -> 64 -> 2 selector network."""

    def __init__(self, params: Optional[np.ndarray] = None, seed: int = 0):
        if params is None:
            rng = np.random.default_rng(seed)
            p = np.zeros(N_PARAMS, dtype=np.float32)
            off = 0
            for rows, cols in ((N_HID, N_IN), (N_HID, N_HID), (N_OUT, N_HID)):  # He initialisation
                p[off:off + rows * cols] = rng.normal(0.0, np.sqrt(2.0 / cols), rows * cols)
                off += rows * cols
            params = p
        self.params = np.ascontiguousarray(params, dtype=np.float32).copy()
        if self.params.size != N_PARAMS:
            raise ValueError("wrong number of selector parameters")

    @property
    def weights_bf16(self) -> np.ndarray:
        return _bf16_bits(self.params[:N_WEIGHTS])

    @property
    def biases(self) -> np.ndarray:
        return np.ascontiguousarray(self.params[N_WEIGHTS:], dtype=np.float32)

    def save(self, path: str, **meta) -> None:
        np.savez_compressed(path, params=self.params, meta=json.dumps(meta))

    @classmethod
    def load(cls, path: str) -> "SelectorModel":
        with np.load(path) as d:
            return cls(d["params"])


class DeviceTrainer:
    """Adam training of a :class:`SelectorModel` on the device.

    The gradient kernel runs ``blocks`` blocks of ``PSIPM_MLP_TILE`` threads
    and adds their partial gradients in block order, so a training run is
    repeatable bit for bit for a given data order.
    """

    def __init__(self, model: SelectorModel, device: int = 0, blocks: int = 148, lr: float = 1e-3,
                 beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8, decay: float = 0.0):
        import torch

        self.torch = torch
        self.lib = _lib.load()
        self.model = model
        self.dev = torch.device("cuda", device)
        self.blocks = int(blocks)
        self.lr, self.beta1, self.beta2, self.eps, self.decay = lr, beta1, beta2, eps, decay
        f32 = dict(dtype=torch.float32, device=self.dev)
        self.master = torch.tensor(model.params, **f32)
        self.m1 = torch.zeros(N_PARAMS, **f32)
        self.m2 = torch.zeros(N_PARAMS, **f32)
        self.grad = torch.zeros(N_PARAMS, **f32)
        self.loss = torch.zeros(1, **f32)
        self.part = torch.zeros(self.blocks * N_PARAMS, **f32)
        self.loss_part = torch.zeros(self.blocks, **f32)
        self.w = torch.tensor(model.weights_bf16.view(np.int16), dtype=torch.int16, device=self.dev)
        self.b = torch.tensor(model.biases, **f32)
        self.step_count = 0

    @staticmethod
    def _p(t):
        return ctypes.c_void_p(t.data_ptr())

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def gradient(self, x, y, c0: float = 1.0, c1: float = 0.0, scale: Optional[float] = None):
        """Loss and gradient over device tensors x[count][6], y[count][2] (no update)."""
        count = int(x.shape[0])
        scale = 1.0 / count if scale is None else scale
        status = self.lib.psipm_mlp_grad_dev(count, self._p(x), self._p(y), float(c0), float(c1), self._p(self.w),
                                             self._p(self.b), self.blocks, self._p(self.part),
                                             self._p(self.loss_part), float(scale), self._p(self.grad),
                                             self._p(self.loss), self._stream())
        if status != _lib.OK:
            raise RuntimeError(f"psipm_mlp_grad_dev failed ({status})")
        return self.loss, self.grad

    def step(self, x, y, c0: float = 1.0, c1: float = 0.0) -> None:
        self.gradient(x, y, c0, c1)
        self.step_count += 1
        status = self.lib.psipm_mlp_adam_dev(self._p(self.master), self._p(self.m1), self._p(self.m2),
                                             self._p(self.grad), float(self.lr), float(self.beta1),
                                             float(self.beta2), float(self.eps), self.step_count,
                                             float(self.decay), self._p(self.w), self._p(self.b),
                                             self._stream())
        if status != _lib.OK:
            raise RuntimeError(f"psipm_mlp_adam_dev failed ({status})")

    def forward(self, x):
        out = self.torch.empty((int(x.shape[0]), N_OUT), dtype=self.torch.float32, device=self.dev)
        status = self.lib.psipm_mlp_forward_dev(int(x.shape[0]), self._p(x), self._p(self.w), self._p(self.b),
                                                self._p(out), self._stream())
        if status != _lib.OK:
            raise RuntimeError(f"psipm_mlp_forward_dev failed ({status})")
        return out

    def fit(self, x: np.ndarray, y: np.ndarray, epochs: int = 10, batch: int = 65536, c0: float = 1.0,
            c1: float = 0.05, seed: int = 0, lr_decay: float = 0.85) -> List[float]:
        """Mini-batch Adam over host arrays (copied to the device once); returns
        the mean loss of every epoch (each batch's loss before its step)."""
        torch = self.torch
        xd = torch.tensor(np.ascontiguousarray(x, dtype=np.float32), device=self.dev)
        yd = torch.tensor(np.ascontiguousarray(y, dtype=np.float32), device=self.dev)
        rng = np.random.default_rng(seed)
        history = []
        for _ in range(epochs):
            order = torch.tensor(rng.permutation(xd.shape[0]), device=self.dev)
            total, batches = 0.0, 0
            for beg in range(0, xd.shape[0], batch):
                idx = order[beg:beg + batch]
                self.step(xd.index_select(0, idx).contiguous(), yd.index_select(0, idx).contiguous(), c0, c1)
                total += float(self.loss.item())
                batches += 1
            history.append(total / max(1, batches))
            self.lr *= lr_decay
        self.model.params = self.master.cpu().numpy().copy()
        return history


# ---------------------------------------------------------------------------
# traces
@dataclass
class Trace:
    features: np.ndarray  # (samples, 6) float32
    targets: np.ndarray   # (samples, 2) float32: true leverage, shift index of the next factor
    refreshes: int
    solve: dict


def true_leverage(A, at_csr, theta, delta, label_dev, columns, probes: int, rng) -> np.ndarray:
    """Hutchinson estimate of diag(D^{1/2} A' H^{-1} A D^{1/2}) at `columns`,
    H = A D A' + delta I factored exactly on `label_dev` (core = every candidate)."""
    n = A.shape[1]
    label_dev.set_theta(theta, delta)
    label_dev.factor(delta, 0)
    sw = np.sqrt(1.0 / theta)
    acc = np.zeros(n)
    for _ in range(probes):
        s = rng.choice(np.array([-1.0, 1.0]), n)
        z = label_dev.apply(A @ (sw * s))
        acc += s * (sw * (at_csr @ z))
    return acc[columns] / probes


def collect_traces(lp, samples_per_refresh: int = 20000, probes: int = 48, seed: int = 0, device: int = 0,
                   tol: float = 1e-8, max_refreshes: Optional[int] = None, solver_options: Optional[dict] = None
                   ) -> Trace:
    """Solve `lp` on the device with the plain rule and record, at every core
    refresh, (inputs, true leverage) for a random sample of candidates and
    the diagonal-shift index the following factorisation used."""
    from .device import NormalEquationsDevice
    from .ipm_device import psipm_solve_resident
    from .kkt import GpuSpectralStableColumnPreconditioner

    rng = np.random.default_rng(seed)
    A = lp.A.tocsc()
    at_csr = A.T.tocsr()
    solver = GpuSpectralStableColumnPreconditioner(A, protected=~lp.pos, device=device, **(solver_options or {}))
    label = NormalEquationsDevice(A, device=device)
    label.set_core(label.candidates)
    feats: List[np.ndarray] = []
    targs: List[np.ndarray] = []
    pending: List[int] = []

    def hook(kkt):
        if max_refreshes is not None and len(feats) >= max_refreshes:
            return
        x = kkt.dev.mlp_features(kkt.mu)
        theta = kkt.dev.get_theta()
        cand = kkt.candidates
        take = rng.choice(cand.size, size=min(samples_per_refresh, cand.size), replace=False)
        try:
            lev = true_leverage(A, at_csr, theta, kkt.delta_now, label, cand[take], probes, rng)
        except Exception:
            return  # the exact factor needed more than the ladder's largest shift: skip this refresh
        y = np.zeros((take.size, 2), dtype=np.float32)
        y[:, 0] = lev
        feats.append(x[take])
        targs.append(y)
        pending.append(len(targs) - 1)

    def after_factor(kkt, shift_index):
        while pending:
            targs[pending.pop()][:, 1] = shift_index

    solver.trace_hook = hook
    solver.factor_hook = after_factor
    try:
        sol = psipm_solve_resident(lp, solver, tol=tol)
        info = dict(status=sol.status, obj=sol.obj, outer=sol.outer_iter, inner=sol.inner_iter,
                    pcg=sol.pcg_iterations, n_fact=sol.n_fact)
    finally:
        solver.close()
        label.close()
    if not feats:
        return Trace(np.zeros((0, N_IN), np.float32), np.zeros((0, 2), np.float32), 0, info)
    return Trace(np.concatenate(feats), np.concatenate(targs), len(feats), info)


def train_selector(traces: List[Trace], epochs: int = 12, seed: int = 0, device: int = 0, lr: float = 2e-3,
                   batch: int = 65536, target: str = "linear") -> Dict:
    """Train a fresh model on the pooled traces; returns the model and the loss
    history.  target "linear" regresses the true leverage itself, "log" its
    logarithm (floored at 1e-4), which weighs the ordering of small leverages
    as much as that of large ones."""
    x = np.concatenate([t.features for t in traces])
    y = np.concatenate([t.targets for t in traces]).copy()
    if target == "log":
        y[:, 0] = np.log(np.maximum(y[:, 0], 1e-4))
    model = SelectorModel(seed=seed)
    trainer = DeviceTrainer(model, device=device, lr=lr)
    history = trainer.fit(x, y, epochs=epochs, batch=batch, seed=seed)
    return dict(model=model, history=history, samples=int(x.shape[0]))


def compare(lp, model: SelectorModel, tol: float = 1e-8, device: int = 0, solver_options=None,
            windows=(0.0,)) -> Dict:
    """Solve `lp` with the plain rule and with the selector (plus its fallback),
    both device-resident; returns time, PCG iterations and outcome of each."""
    from .ipm_device import psipm_solve_resident
    from .kkt import GpuSpectralStableColumnPreconditioner

    out = {}
    arms = [("rule", None, 0.0)] + [("learned" if w <= 1.0 else f"learned_window{w:g}", model, w) for w in windows]
    for name, sel, window in arms:
        solver = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, device=device, selector=sel,
                                                       selector_window=window, **(solver_options or {}))
        try:
            solver.dev.timer_start()
            sol = psipm_solve_resident(lp, solver, tol=tol)
            seconds = solver.dev.timer_stop()
            out[name] = dict(status=sol.status, obj=sol.obj, seconds=seconds, pcg=sol.pcg_iterations,
                             outer=sol.outer_iter, inner=sol.inner_iter, n_fact=sol.n_fact,
                             learned_refreshes=solver.learned_refreshes, fallbacks=solver.selector_fallbacks,
                             res_p=sol.res_p, res_d=sol.res_d, gap=sol.gap)
        finally:
            solver.close()
    return out


def _seeds(text: str) -> List[int]:
    lo, _, hi = text.partition("-")
    return list(range(int(lo), int(hi or lo) + 1))


def main(argv=None) -> None:
    from . import synthetic

    ap = argparse.ArgumentParser(description="train the learned column selector on solver traces")
    ap.add_argument("--rows", type=int, default=200)
    ap.add_argument("--cols", type=int, default=250)
    ap.add_argument("--train", default="0-19", help="training seeds (grid_network seed = 1000 + s + 100)")
    ap.add_argument("--test", default="0-1", help="held-out seeds (seed = 1000 + s + 500)")
    ap.add_argument("--samples", type=int, default=20000)
    ap.add_argument("--probes", type=int, default=48)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--out", required=True)
    ap.add_argument("--report", default=None)
    ap.add_argument("--model", default=None, help="evaluate this model instead of training one")
    ap.add_argument("--windows", default="0", help="comma-separated selector windows to compare")
    ap.add_argument("--target", default="linear", choices=("linear", "log"))
    args = ap.parse_args(argv)
    windows = tuple(float(w) for w in args.windows.split(","))
    if args.model:
        model = SelectorModel.load(args.model)
        report = dict(model=args.model, held_out={})
        for s in _seeds(args.test):
            lp = synthetic.grid_network(args.rows, args.cols, seed=1500 + s)
            report["held_out"][s] = compare(lp, model, windows=windows)
            print(f"held-out seed {s}: {report['held_out'][s]}", flush=True)
        if args.report:
            with open(args.report, "w") as f:
                json.dump(report, f, indent=1)
        return
    t0 = time.time()
    traces = []
    for s in _seeds(args.train):
        lp = synthetic.grid_network(args.rows, args.cols, seed=1100 + s)
        traces.append(collect_traces(lp, samples_per_refresh=args.samples, probes=args.probes, seed=s))
        print(f"trace seed {s}: {traces[-1].refreshes} refreshes, {traces[-1].features.shape[0]} samples, "
              f"solve {traces[-1].solve}", flush=True)
    result = train_selector(traces, epochs=args.epochs, target=args.target)
    print(f"trained on {result['samples']} samples, loss by epoch {result['history']}", flush=True)
    result["model"].save(args.out, rows=args.rows, cols=args.cols, train=args.train, samples=result["samples"],
                         history=result["history"], target=args.target, probes=args.probes)
    report = dict(train=args.train, samples=result["samples"], history=result["history"], held_out={},
                  trace_seconds=time.time() - t0)
    for s in _seeds(args.test):
        lp = synthetic.grid_network(args.rows, args.cols, seed=1500 + s)
        report["held_out"][s] = compare(lp, result["model"], windows=windows)
        print(f"held-out seed {s}: {report['held_out'][s]}", flush=True)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()

