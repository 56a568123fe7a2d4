"""Generate the golden fixtures by running the unmodified reference.

Run in a container that has the reference checked out (read-only), giving
its directory with ``--reference`` or the ``PSIPM_REFERENCE`` environment
variable:

    python tests/golden/make_golden.py --reference PATH [--only NAME]

The reference needs ``sksparse.cholmod`` (CHOLMOD), which is not installed
in this image; ``tests/golden/cholmod_standin`` provides the same API on top
of SciPy's SuperLU and is put first on ``sys.path``.  So every fixture is
"reference code + SuperLU stand-in factor".

For each seeded instance the script wraps the reference's
``SpectralStableColumnPreconditioner`` (psipm_spectral_preconditioner.py:143)
so that every ``factorize`` and ``solve`` call records its inputs and
outputs, runs ``psipm_solve`` (psipm_active_pool.py:2277) to tolerance 1e-8
and writes ``<name>.npz`` next to this script: the LP, the first
``KEEP_CALLS`` factorize/solve records (theta, delta, scores at refresh,
core, r1, r2, dx, dy, PCG iterations and tolerance), every core the
refreshes produced, and the final iterate and status.
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
KEEP_CALLS = 8

INSTANCES = {
    "random_m300": ("random_lp", dict(m=300, n=900, seed=0)),
    "grid_20x25": ("grid_network", dict(rows=20, cols=25, seed=1000)),
    "cover_m200": ("set_cover", dict(m=200, n=10_000, seed=2000)),
    # four dense columns (1,100 entries each): the Woodbury extraction path
    "dense_m1200": ("random_lp_dense", dict(m=1200, n=3600, seed=7)),
    # the full-size random LP (m = 2,000, n = 6,000, 5 nonzeros per column) with the
    # reference's default options: m > 1,500, so the stable core path runs as is
    "random_m2000": ("random_lp", dict(m=2000, n=6000, seed=0)),
}
# per-instance option overrides and number of recorded calls
INSTANCE_OPTIONS = {"random_m2000": {}}
INSTANCE_KEEP = {"random_m2000": 4}
# full solves recorded as a summary only (no per-call vectors): the 200 x 250 grid
# network LP that the benchmark solves (seed 1000), with the reference's defaults
RESULTS = {"grid_200x250_result": ("grid_network", dict(rows=200, cols=250, seed=1000))}
# plus hsd_m1600 (make_hsd): the V3.1 HSD preconditioner surface, and
# hsd_newton_m1600 (make_hsd_newton): the V3.1 reduced HSD Newton system
# the small instances use the stable core path (the exact-preconditioner
# gate, psipm_stable_preconditioner.py:202-207, would otherwise switch it off)
OPTIONS = dict(full_preconditioner_row_threshold=10)


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=os.environ.get("PSIPM_REFERENCE"))
    parser.add_argument("--only", default=None)
    args = parser.parse_args()
    if not args.reference:
        parser.error("give the reference's directory with --reference or PSIPM_REFERENCE")
    sys.path.insert(0, os.path.join(HERE, "cholmod_standin"))
    sys.path.insert(0, args.reference)
    sys.path.insert(0, os.path.join(REPO, "mf-psipm_b200"))
    import psipm_active_pool as PS
    import psipm_spectral_preconditioner as SSP
    from psipm_b200 import synthetic

    class Recording(SSP.SpectralStableColumnPreconditioner):
        def __init__(self, *a, **k):
            super().__init__(*a, **k)
            self.rec_factor = []
            self.rec_solve = []
            self.rec_cores = []
            self._pending_scores = None

        def _scores(self, weights, delta):
            s = super()._scores(weights, delta)
            self._pending_scores = (np.array(weights), float(delta), np.array(s))
            return s

        def _refresh_core(self, weights, delta, stable, force_backbone=False):
            super()._refresh_core(weights, delta, stable, force_backbone)
            self.rec_cores.append(self.core.copy())

        keep = KEEP_CALLS

        def factorize(self, theta, delta):
            self._pending_scores = None
            core_before = self.core.copy()
            super().factorize(theta, delta)
            if len(self.rec_factor) < self.keep:
                self.rec_factor.append(dict(
                    theta=np.array(theta), delta=float(delta), core_before=core_before,
                    core=self.core.copy(), scores=(None if self._pending_scores is None
                                                   else self._pending_scores[2]),
                    factor_age=int(self.factor_age), core_target=int(self.core_target)))

        def solve(self, r1, r2):
            dx, dy = super().solve(r1, r2)
            if len(self.rec_solve) < self.keep:
                self.rec_solve.append(dict(
                    r1=np.array(r1), r2=np.array(r2), dx=np.array(dx), dy=np.array(dy),
                    theta=np.array(self.theta), delta=float(self.delta), core=self.core.copy(),
                    iterations=int(self.cg_iterations[-1]), tolerance=float(self.cg_tolerances[-1])))
            return dx, dy

    for name, (family, kwargs) in INSTANCES.items():
        if args.only and name != args.only:
            continue
        lp0 = getattr(synthetic, family)(**kwargs)
        lp = PS.StandardLP(c=lp0.c, A=lp0.A, b=lp0.b, u=lp0.u, pos=lp0.pos, box=lp0.box)
        options = INSTANCE_OPTIONS.get(name, OPTIONS)
        solver = Recording(lp.A, protected=~lp.pos, **options)
        solver.keep = INSTANCE_KEEP.get(name, KEEP_CALLS)
        sol = PS.psipm_solve(lp, kkt="spectral-stable-pcg", kkt_solver=solver, tol=1e-8, printlevel=0)
        out = dict(
            family=family, kwargs=repr(kwargs), options=repr(options),
            A_data=lp.A.data, A_indices=lp.A.indices, A_indptr=lp.A.indptr,
            A_shape=np.array(lp.A.shape), b=lp.b, c=lp.c, u=lp.u, pos=lp.pos, box=lp.box,
            x=sol.x, y=sol.y, z=sol.z, w=sol.w, obj=sol.obj, status=sol.status,
            res_p=sol.res_p, res_d=sol.res_d, mu=sol.mu,
            pcg_iterations=sol.pcg_iterations, cg_iterations=np.array(solver.cg_iterations),
            core_sizes=np.array(solver.core_sizes), n_fact=solver.n_fact,
            candidates=solver.candidates, matching_columns=solver.matching_columns,
            low_rank_columns=np.asarray(solver.low_rank_columns, dtype=np.int64),
            n_factor_calls=len(solver.rec_factor), n_solve_calls=len(solver.rec_solve),
            n_cores=len(solver.rec_cores),
        )
        for i, rec in enumerate(solver.rec_factor):
            for key, value in rec.items():
                if value is not None:
                    out[f"f{i}_{key}"] = value
        for i, rec in enumerate(solver.rec_solve):
            for key, value in rec.items():
                out[f"s{i}_{key}"] = value
        for i, core in enumerate(solver.rec_cores):
            out[f"core{i}"] = core
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{name}: {sol.status} obj {sol.obj!r} pcg {sol.pcg_iterations} "
              f"-> {os.path.getsize(path) / 1e6:.2f} MB")

    for name, (family, kwargs) in RESULTS.items():
        if args.only == name:  # long (about 40 minutes on 8 cores): only on request
            make_result(PS, SSP, synthetic, name, family, kwargs)
    if args.only in (None, "tree_grid_20x25"):
        make_tree(synthetic)
    if args.only in (None, "hsd_m1600"):
        make_hsd(PS, synthetic)
    if args.only in (None, "hsd_newton_m1600"):
        make_hsd_newton(synthetic)
    if args.only in (None, "crash_masks"):
        make_crash(PS, synthetic)


CRASH_CASES = {
    "cover_a": ("set_cover", dict(m=300, n=6000, seed=2101)),
    "cover_b": ("set_cover", dict(m=120, n=2000, kmin=1, kmax=4, seed=2102)),
    "cover_c": ("set_cover", dict(m=500, n=20000, zipf=1.5, seed=2103)),
    "random": ("random_lp", dict(m=100, n=300, seed=2104)),  # not a covering LP: no crash
    "cover_unbounded": ("set_cover", dict(m=200, n=4000, seed=2105)),  # upper bounds dropped: implied caps
}


def crash_lp(synthetic, name, family, kwargs):
    """The LP of a crash case (the test rebuilds it the same way)."""
    lp = getattr(synthetic, family)(**kwargs)
    if name.endswith("_unbounded"):
        lp.u[:] = np.inf
        lp.box[:] = False
        lp.c[np.diff(lp.A.tocsc().indptr) > 1] *= 1.0 + np.arange(int((np.diff(lp.A.tocsc().indptr) > 1).sum())) % 3
    return lp


def make_crash(PS, synthetic):
    """The reference's covering crash support (_covering_crash_mask,
    psipm_active_pool.py:3436-3533) on a few covering LPs and one LP it must
    decline; the LPs are rebuilt from the generator's arguments."""
    out = {}
    for name, (family, kwargs) in CRASH_CASES.items():
        lp0 = crash_lp(synthetic, name, family, kwargs)
        lp = PS.StandardLP(c=lp0.c, A=lp0.A, b=lp0.b, u=lp0.u, pos=lp0.pos, box=lp0.box)
        mask = PS._covering_crash_mask(lp)
        out[f"{name}_family"] = family
        out[f"{name}_kwargs"] = repr(kwargs)
        out[f"{name}_none"] = mask is None
        out[f"{name}_mask"] = np.zeros(0, dtype=bool) if mask is None else np.asarray(mask, dtype=bool)
        print(f"crash {name}: {'none' if mask is None else int(mask.sum())} of {lp.A.shape[1]} columns")
    path = os.path.join(HERE, "crash_masks.npz")
    np.savez_compressed(path, **out)
    print(f"crash_masks -> {os.path.getsize(path) / 1e3:.1f} kB")


def make_result(PS, SSP, synthetic, name, family, kwargs):
    """Full reference solve to 1e-8 with default options, kept as a JSON summary:
    the outcome (status, objective, residuals, iteration counts), the outer
    iteration history and the per-call PCG counts and core sizes, plus a
    fingerprint of the generated LP so that a test can check that it solves
    the same instance."""
    import json
    import time

    lp0 = getattr(synthetic, family)(**kwargs)
    lp = PS.StandardLP(c=lp0.c, A=lp0.A, b=lp0.b, u=lp0.u, pos=lp0.pos, box=lp0.box)
    solver = SSP.SpectralStableColumnPreconditioner(lp.A, protected=~lp.pos)
    t0 = time.perf_counter()
    sol = PS.psipm_solve(lp, kkt="spectral-stable-pcg", kkt_solver=solver, tol=1e-8, printlevel=0)
    seconds = time.perf_counter() - t0
    cx = float(lp.c @ sol.x)
    ibox = np.flatnonzero(lp.box)
    gap = abs(cx - (float(lp.b @ sol.y) - float(sol.w[ibox] @ lp.u[ibox]))) / (1.0 + abs(cx))
    out = dict(
        family=family, kwargs=kwargs, tol=1e-8, status=sol.status, obj=float(sol.obj),
        res_p=float(sol.res_p), res_d=float(sol.res_d), mu=float(sol.mu), gap=gap,
        outer_iter=int(sol.outer_iter), inner_iter=int(sol.inner_iter),
        pcg_iterations=int(sol.pcg_iterations), n_fact=int(solver.n_fact),
        cg_iterations=[int(v) for v in solver.cg_iterations],
        core_sizes=[int(v) for v in solver.core_sizes],
        history=[{k: float(v) for k, v in h.items() if isinstance(v, (int, float))} for h in sol.history],
        seconds=seconds, cpu_count=os.cpu_count(),
        fingerprint=dict(shape=list(lp.A.shape), nnz=int(lp.A.nnz), c_sum=float(lp.c.sum()),
                         b_abs_sum=float(np.abs(lp.b).sum()), u_sum=float(lp.u[ibox].sum())),
    )
    path = os.path.join(HERE, f"{name}.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(f"{name}: {sol.status} obj {sol.obj!r} outer {sol.outer_iter} pcg {sol.pcg_iterations} "
          f"in {seconds:.0f} s")


def make_tree(synthetic):
    """V3.1 network surface: NetworkTopology.from_incidence and TreePreconditioner
    (psipm_v3_1_hsd.py:495-610, 715-785) on an ungrounded 20 x 25 grid network,
    with a random active-column set containing the protected forest arcs:
    the forest, then three factorisations (random weights, delta) each with
    two solves, and the HSD _pcg (:1015-1063) with the tree as preconditioner."""
    import psipm_v3_1_hsd as H

    lp = synthetic.grid_network(20, 25, seed=1001, ground=False)
    A = lp.A.tocsc()
    topo = H.NetworkTopology.from_incidence(A)
    rng = np.random.default_rng(23)
    active = np.flatnonzero(topo.protected | (rng.random(A.shape[1]) < 0.6))
    pre = H.TreePreconditioner(topo, active)
    out = dict(A_data=A.data, A_indices=A.indices, A_indptr=A.indptr, A_shape=np.array(A.shape),
               parent=topo.parent, depth=topo.depth, tree_child=topo.tree_child, protected=topo.protected,
               root=topo.root, components=topo.components, active=active)
    Aa = A[:, active]
    for call in range(3):
        D = np.exp(rng.uniform(-6.0, 6.0, active.size))
        delta = float(10.0 ** rng.uniform(-10, -4))
        pre.factor(D, delta)
        out.update({f"c{call}_D": D, f"c{call}_delta": delta, f"c{call}_pivot": pre.pivot.copy(),
                    f"c{call}_multiplier": pre.multiplier.copy()})
        for k in range(2):
            rhs = rng.standard_normal(A.shape[0])
            out[f"c{call}_rhs{k}"] = rhs
            out[f"c{call}_sol{k}"] = pre.solve(rhs)

        def matvec(v, D=D, delta=delta):
            return Aa @ (D * (Aa.T @ v)) + delta * v

        rhs = Aa @ (D * rng.standard_normal(active.size))
        x, it, mv, ok, _ = H._pcg(matvec, rhs, pre, 1e-10, 1000, np.inf)
        out.update({f"c{call}_pcg_rhs": rhs, f"c{call}_pcg_x": x, f"c{call}_pcg_iterations": it,
                    f"c{call}_pcg_ok": ok})
    path = os.path.join(HERE, "tree_grid_20x25.npz")
    np.savez_compressed(path, **out)
    print(f"tree_grid_20x25: depth {int(topo.depth.max())}, active {active.size}, PCG "
          f"{[int(out[f'c{i}_pcg_iterations']) for i in range(3)]} -> {os.path.getsize(path) / 1e6:.2f} MB")


def make_hsd(PS, synthetic):
    """V3.1 HSD surface: StableColumnPreconditioner.factor + _pcg
    (psipm_v3_1_hsd.py:823-989, 1015-1063) on a random LP with m > 1500, so
    the stable core path (not the exact small-row gate) is taken."""
    import psipm_v3_1_hsd as H

    lp = synthetic.random_lp(1600, 4800, seed=5)
    A = lp.A
    rng = np.random.default_rng(20)
    options = H.V3Options(generic_preconditioner="stable")
    pre = H.StableColumnPreconditioner(A, options)
    out = dict(A_data=A.data, A_indices=A.indices, A_indptr=A.indptr, A_shape=np.array(A.shape))
    for call in range(3):
        D = np.exp(rng.uniform(-6.0, 6.0, A.shape[1]))
        delta = 1e-8
        pre.factor(D, delta)
        rhs = A @ (D * rng.standard_normal(A.shape[1]))

        def matvec(v, D=D, delta=delta):
            return A @ (D * (A.T @ v)) + delta * v

        x, it, mv, ok, _ = H._pcg(matvec, rhs, pre, 1e-10, options.pcg_max_iterations, np.inf)
        pre.record_iterations(it, 0.0, ok)
        out.update({f"c{call}_D": D, f"c{call}_delta": delta, f"c{call}_rhs": rhs, f"c{call}_x": x,
                    f"c{call}_iterations": it, f"c{call}_matvecs": mv, f"c{call}_ok": ok,
                    f"c{call}_core": pre.impl.core.copy(), f"c{call}_n_fact": pre.impl.n_fact})
    path = os.path.join(HERE, "hsd_m1600.npz")
    np.savez_compressed(path, **out)
    print(f"hsd_m1600: iterations {[int(out[f'c{i}_iterations']) for i in range(3)]} "
          f"-> {os.path.getsize(path) / 1e6:.2f} MB")


def hsd_newton_inputs(A, b, rng):
    """Seeded HSD iterate, embedding and boxes for one active-column set (shared
    with the tests, which rebuild the same D from the stored iterate)."""
    m, n = A.shape
    boxed = rng.random(n) < 0.3
    tau, kappa = 0.8, 0.3
    x = rng.uniform(0.1, 2.0, n)
    z = rng.uniform(0.1, 2.0, n)
    upper = np.where(boxed, (x + rng.uniform(0.2, 2.0, n)) / tau, np.inf)
    w = np.where(boxed, rng.uniform(0.1, 2.0, n), 0.0)
    bar_b = b - A @ x / tau
    bar_c = rng.standard_normal(n)
    bar_g = float(rng.standard_normal())
    return dict(x=x, z=z, w=w, upper=upper, tau=tau, kappa=kappa, bar_b=bar_b, bar_c=bar_c, bar_g=bar_g)


def hsd_weights(x, z, w, upper, tau, rho, floor):
    """D as the HSD step loop forms it (psipm_v3_1_hsd.py:1694-1695, 1718-1721)."""
    boxed = np.isfinite(upper)
    slack = np.ones_like(x)
    slack[boxed] = upper[boxed] * tau - x[boxed]
    ratio = np.zeros_like(x)
    ratio[boxed] = w[boxed] / slack[boxed]
    return 1.0 / np.maximum(rho + z / x + ratio, floor), slack


def make_hsd_newton(synthetic):
    """V3.1 HSDNewtonSystem (psipm_v3_1_hsd.py:1066-1264) over the reference's
    StableColumnPreconditioner: two systems (the second at a moved iterate, so the
    preconditioner's lagged-reuse policy runs), each with an affine direction
    and a corrector direction shaped like the step loop's (:1734-1791)."""
    import psipm_v3_1_hsd as H

    lp = synthetic.random_lp(1600, 4800, seed=6)
    A, b = lp.A.tocsc(), lp.b
    m, n = A.shape
    c = lp.c
    rng = np.random.default_rng(41)
    # growth_amortization 0 makes the core-growth rule (:954-984) independent of
    # the measured PCG and factor times, so the fixture is reproducible
    options = H.V3Options(generic_preconditioner="stable", generic_growth_amortization=0.0)
    pre = H.StableColumnPreconditioner(A, options)
    stats = H.LinearStats()
    base = hsd_newton_inputs(A, b, rng)
    out = dict(A_data=A.data, A_indices=A.indices, A_indptr=A.indptr, A_shape=np.array(A.shape), c=c, b=b,
               upper=base["upper"], delta=options.delta, eta=options.eta, zeta=options.zeta,
               rho=options.rho, floor=options.regularization_floor, pcg_tolerance=1e-10,
               pcg_max_iterations=options.pcg_max_iterations,
               growth_amortization=options.generic_growth_amortization)
    for sys_i in range(2):
        it = dict(base)
        if sys_i:
            boxed = np.isfinite(base["upper"])
            it["x"] = base["x"] * np.where(boxed, 1.0, np.exp(rng.uniform(-0.5, 0.5, n)))
            it["z"] = base["z"] * np.exp(rng.uniform(-0.5, 0.5, n))
        D, slack = hsd_weights(it["x"], it["z"], it["w"], it["upper"], it["tau"], options.rho,
                               options.regularization_floor)
        state = H.HSDState(x=it["x"], y=np.zeros(m), z=it["z"], w=it["w"], tau=it["tau"], kappa=it["kappa"],
                           theta=1.0, x_center=it["x"].copy(), y_center=np.zeros(m), tau_center=it["tau"],
                           theta_center=1.0)
        emb = H.HSDEmbedding(bar_b=it["bar_b"], bar_c=it["bar_c"], bar_g=it["bar_g"], alpha=1.0)
        system = H.HSDNewtonSystem(A, c, it["upper"], b, D, options.delta, options.eta, state, emb, pre, 1e-10,
                                   options, np.inf, stats)
        boxed = np.isfinite(it["upper"])
        rd, rp = rng.standard_normal(n), rng.standard_normal(m)
        rg, rn = float(rng.standard_normal()), float(rng.standard_normal())
        affine_rhs = (-rd, -rp, -rg, -rn, -it["x"] * it["z"], np.where(boxed, -slack * it["w"], 0.0),
                      -it["tau"] * it["kappa"])
        aff = system.direction(*affine_rhs)
        ds = np.zeros(n)
        ds[boxed] = it["upper"][boxed] * aff[4] - aff[0][boxed]
        smu = 0.1 * float(it["x"] @ it["z"]) / n
        corr_rhs = (np.zeros(n), np.zeros(m), 0.0, 0.0, smu - aff[0] * aff[2],
                    np.where(boxed, smu - ds * aff[3], 0.0), smu - aff[4] * aff[6])
        cor = system.direction(*corr_rhs)
        out[f"s{sys_i}_x"], out[f"s{sys_i}_z"] = it["x"], it["z"]
        for key in ("w", "tau", "kappa", "bar_b", "bar_c", "bar_g"):
            out[f"s{sys_i}_{key}"] = it[key]
        out[f"s{sys_i}_D"] = D
        out[f"s{sys_i}_core"] = pre.impl.core.copy()
        out[f"s{sys_i}_n_fact"] = pre.impl.n_fact
        for d_i, (rhs, res) in enumerate(((affine_rhs, aff), (corr_rhs, cor))):
            tag = f"s{sys_i}d{d_i}"
            for k, v in enumerate(rhs):
                out[f"{tag}_rhs{k}"] = v
            for k, name in enumerate(("dx", "dy", "dz", "dw", "dtau", "dtheta", "dkappa", "ok")):
                out[f"{tag}_{name}"] = res[k]
        out[f"s{sys_i}_stats"] = np.array([stats.solves, stats.iterations, stats.max_iterations, stats.matvecs,
                                           stats.failures])
    path = os.path.join(HERE, "hsd_newton_m1600.npz")
    np.savez_compressed(path, **out)
    print(f"hsd_newton_m1600: stats {out['s1_stats'].tolist()} ok "
          f"{[bool(out[f's{i}d{j}_ok']) for i in range(2) for j in range(2)]} "
          f"-> {os.path.getsize(path) / 1e6:.2f} MB")


if __name__ == "__main__":
    main()
