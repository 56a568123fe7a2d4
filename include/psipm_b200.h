/*
 * psipm_b200 — B200-native normal-equations inner solve for PS-IPM / HSD.
 *
 * C ABI of libpsipm_b200.so.  Plain pointers and sizes only; every array
 * argument is HOST memory unless the function name ends in _dev.  One handle
 * owns one LP's device data (A, A^T, weights, core, factor, PCG workspace)
 * and one CUDA stream; calls on a handle must come from one host thread at a
 * time and are synchronous on return.
 *
 * The operations replace the arithmetic of the reference's KKT solver
 * objects (StefanoCipolla/MF-PSIPM):
 *   SpectralStableColumnPreconditioner   psipm_spectral_preconditioner.py:143-752
 *   StableActiveColumnPreconditioner     psipm_stable_preconditioner.py:113-517
 *   NormalEquations (factor/apply)       psipm_active_pool.py:720-996
 *   V3.1 _pcg / HSDNewtonSystem.matvec   psipm_v3_1_hsd.py:1015-1063, 1136-1137
 * The refresh/refactor policy, statistics and exceptions of those classes
 * stay in the host wrapper (psipm_b200/kkt.py), which maps every nonzero
 * status to the reference's KKTSolveError.
 */
#ifndef PSIPM_B200_H
#define PSIPM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define PSIPM_OK 0
#define PSIPM_ERR_ARGUMENT (-1)   /* invalid size, pointer or option */
#define PSIPM_ERR_CUDA (-2)       /* a CUDA runtime call failed */
#define PSIPM_ERR_NOT_PD (-3)     /* Cholesky failed at every diagonal shift */
#define PSIPM_ERR_STATE (-4)      /* call order (e.g. apply before factor) */
#define PSIPM_ERR_BOUNDS (-5)     /* a device index check tripped */
#define PSIPM_ERR_TIMEOUT (-6)    /* a device loop hit its deadline */
#define PSIPM_ERR_MEMORY (-7)     /* device allocation failed */
#define PSIPM_ERR_SYMBOLIC (-8)   /* symbolic analysis rejected the pattern */
#define PSIPM_ERR_UNSUPPORTED (-9)

typedef struct psipm_handle psipm_handle;

/* PCG variants (the two reference loops) */
#define PSIPM_PCG_SPECTRAL 0 /* psipm_spectral_preconditioner.py:469-581 */
#define PSIPM_PCG_HSD 1      /* psipm_v3_1_hsd.py:1015-1063 */

/* precision of the PCG inner iterations */
#define PSIPM_FP64 0         /* everything in FP64 */
#define PSIPM_FP32_REFINED 1 /* FP32 SpMV/factor/solves inside FP64 refinement sweeps; when a sweep
                                stops reducing the FP64 residual the solve finishes with FP64 PCG
                                around the FP32 preconditioner */
#define PSIPM_FP32_PRECOND 2 /* FP64 PCG (operator, vectors) with the preconditioner's factor and
                                triangular solves in FP32 */

typedef struct {
    int32_t info;            /* reference KrylovResult.info: 0 ok, >0 limit, -1..-7 breakdown */
    int32_t iterations;      /* PCG iterations (sum over refinement sweeps) */
    int32_t matvecs;         /* H·p products, true-residual ones included */
    int32_t replacements;    /* residual replacements */
    int32_t residual_checks; /* true-residual verifications */
    int32_t n_alpha;         /* entries written to alphas[] (current Lanczos run) */
    int32_t n_beta;          /* entries written to betas[] */
    int32_t n_history;       /* entries written to history[] */
    int32_t refinements;     /* FP64 refinement sweeps (FP32_REFINED only) */
    int32_t ok;              /* converged (spectral variant: info == 0) */
    double relative_residual;/* ||rhs - H x|| / max(1, ||rhs||) in FP64 */
    double seconds;          /* device time of the call (CUDA events) */
    double phase_seconds[4]; /* device time by phase: [0] H·p passes, [1] vector
                                updates, [2] preconditioner applies, [3] setup and
                                true-residual checks (%globaltimer, block 0) */
} psipm_pcg_info;

typedef struct {
    int32_t nsupernodes;
    int32_t nlevels;
    int32_t max_front;
    int32_t symbolic_analyses; /* cumulative */
    int64_t nnz_factor;        /* stored entries of L */
    double flops;              /* numeric factorisation flops */
    double symbolic_seconds;   /* last host symbolic analysis */
    double factor_seconds;     /* last numeric factorisation (device) */
} psipm_factor_info;

/* ---- lifetime -------------------------------------------------------------
 * A is m x n in CSC (colptr[n+1], rowidx[nnz], values[nnz]); indices sorted
 * within columns, no duplicates (the reference canonicalises A the same way,
 * psipm_active_pool.py:781-784).  Replaces NormalEquations.__init__ and the
 * candidate bookkeeping of StableActiveColumnPreconditioner.__init__
 * (psipm_stable_preconditioner.py:162-201).  `device` is the CUDA ordinal. */
int psipm_create(int64_t m, int64_t n, int64_t nnz, const int64_t* colptr,
                 const int32_t* rowidx, const double* values, int32_t device,
                 int32_t precision, psipm_handle** out);
void psipm_destroy(psipm_handle* h);
const char* psipm_last_error(const psipm_handle* h);

/* ---- F3 extracted dense columns ----------------------------------------------
 * Declare the (sorted) columns that the factor leaves out and corrects by
 * Woodbury, as low_rank_normal_columns chose them (psipm_active_pool.py:691-718,
 * at most PSIPM_LOW_RANK_MAX): they leave the candidate set and the assembled
 * diagonal (A_factor), the scores' diagonal adds A2_low_rank w_L
 * (psipm_stable_preconditioner.py:298-303), and every successful psipm_factor
 * prepares B = P_base^{-1} A_L and the Cholesky factor of
 * Theta_L + A_L^T B (psipm_active_pool.py:906-947), which every apply then
 * uses (:949-956).  Call once, before any core and before set_theta; FP64 only. */
#define PSIPM_LOW_RANK_MAX 8
int psipm_set_low_rank(psipm_handle* h, const int64_t* cols, int64_t q);

/* Number and (global, ascending) indices of the candidate columns: columns
 * with at least two nonzeros (psipm_stable_preconditioner.py:169-172). */
int64_t psipm_num_candidates(const psipm_handle* h);
int psipm_get_candidates(const psipm_handle* h, int64_t* out);

/* ---- weights ----------------------------------------------------------------
 * theta[n] (host).  Stores theta and w = 1/theta on the device; replaces
 * `self._weights = 1.0 / theta` (psipm_stable_preconditioner.py:399) and the
 * `self.theta = theta` of every factorize. */
int psipm_set_theta(psipm_handle* h, const double* theta, double delta);

/* ---- S3 leverage scores -----------------------------------------------------
 * scores[ncand] = w_C * (A2_C^T (1/max(A2 w + max(delta,tiny), tiny))) /
 * (1 + fill_weight * q(q-1)/2), bit-identical to _scores
 * (psipm_stable_preconditioner.py:293-309).  Either output may be NULL. */
int psipm_scores(psipm_handle* h, double fill_weight, double* scores, double* diagonal);

/* ---- S1/S4 core refresh -----------------------------------------------------
 * New core from the current scores, as _refresh_core does
 * (psipm_stable_preconditioner.py:311-371): mandatory columns, the top
 * floor(retention*target) of the old core (if stable), trimming, and the top
 * remaining candidates; ties broken by candidate index.  mandatory_local are
 * sorted candidate-local positions.  core_out (capacity ncand) receives the
 * sorted global column indices; *retained the fraction of the old core kept.
 * psipm_scores must have been called for the current weights. */
int psipm_refresh_core(psipm_handle* h, int64_t target, double retention, int32_t stable,
                       const int64_t* mandatory_local, int64_t nmandatory,
                       int64_t* core_out, int64_t* ncore, double* retained);
/* Deterministic preconditioner applications (on != 0): the partial sums of
 * the triangular sweeps go to their own slots and are added in a fixed
 * order, so a PCG and a whole IPM solve take the same trajectory, bit for
 * bit, on every run.  Off (the default): FP64 atomics, faster; the order of
 * the additions, and so the last bits and possibly an iteration count, can
 * change between runs.  Every other reduction of the library has a fixed
 * order in both modes. */
int psipm_set_deterministic(psipm_handle* h, int32_t on);
/* Grid of this handle's persistent kernels (PCG, apply, operator): `blocks`
 * thread blocks (at most the co-resident maximum chosen at creation; 0 goes
 * back to it).  Several handles that solve small LPs concurrently on their
 * own streams each take a share of the GPU this way (psipm_b200.batch).  Not
 * with extracted dense columns (PSIPM_ERR_STATE). */
int psipm_set_grid(psipm_handle* h, int32_t blocks);
/* Arithmetic of the FP32 factor's large fronts (PSIPM_FP32_REFINED and
 * PSIPM_FP32_PRECOND handles; the FP64 factor always runs on the CUDA cores):
 * `passes` 3 (the default) factors them in panels of 256 columns whose
 * trailing updates run on the tensor cores as 3xTF32 products (hi*hi + hi*lo
 * + lo*hi of a TF32 head and its FP32 remainder: FP32-level products, FP32
 * accumulation); 1 uses the TF32 heads alone; 0 keeps the CUDA-core blocked
 * kernels.  The reference factors with CHOLMOD in FP64
 * (psipm_active_pool.py:839-897); this switch has no counterpart there.
 * Takes effect at the next psipm_factor. */
int psipm_set_factor_tc(psipm_handle* h, int32_t passes);
/* Straddling ties of the top-k selections (psipm_refresh_core, psipm_top_k).
 * The reference selects with np.argpartition (psipm_stable_preconditioner.py:
 * 97-110), whose pick among equal scores that straddle the cut depends on
 * NumPy's build; this library takes them by ascending candidate index.  A
 * selection "straddles" when the keys equal to its threshold outnumber the
 * slots left for them.  out[4] = {selections that straddled (cumulative),
 * tied keys at the last straddling threshold, slots they competed for,
 * selections run (cumulative)}. */
int psipm_tie_info(const psipm_handle* h, int64_t* out);
/* Install an explicit core (sorted global column indices). */
int psipm_set_core(psipm_handle* h, const int64_t* core, int64_t ncore);
/* Top-`count` candidates among those with mask[i]!=0 (NULL mask: all) by
 * (score desc, index asc), finite scores only — the reference's _top_k
 * (psipm_stable_preconditioner.py:97-110) — written as ascending local
 * indices to out (capacity count); *nout receives how many. */
int psipm_top_k(psipm_handle* h, const double* scores, int64_t nscores, const uint8_t* mask,
                int64_t count, int64_t* out, int64_t* nout);

/* ---- F1/F2 factor -------------------------------------------------------------
 * Assemble P = A_C diag(w_C) A_C^T + diag(max(A2 w - diag_C, 0) + delta),
 * Jacobi-scale it to unit diagonal and factor it on the device, trying the
 * diagonal shifts (0,1e-14,...,1e-2) from index `start_shift` on
 * (psipm_active_pool.py:839-897).  The symbolic analysis is redone when the
 * core changed since the last one.  *shift_index receives the shift used. */
int psipm_factor(psipm_handle* h, double delta, int32_t start_shift, int32_t* shift_index,
                 psipm_factor_info* info);

/* ---- H4 preconditioner apply: z = P^{-1} r (psipm_active_pool.py:903-904) */
int psipm_apply(psipm_handle* h, const double* r, double* z);

/* ---- H3 operator: y = A diag(w) A^T v + delta v
 * (psipm_stable_preconditioner.py:434-438, psipm_v3_1_hsd.py:1136-1137) */
int psipm_matvec(psipm_handle* h, const double* v, double* y);

/* ---- H2/H2b PCG on H with P as preconditioner ---------------------------------
 * variant PSIPM_PCG_SPECTRAL restates psipm_spectral_preconditioner.py:469-581
 * (initial guess P^{-1} rhs, residual replacement every `replacement`
 * iterations, breakdown codes); PSIPM_PCG_HSD restates psipm_v3_1_hsd.py:1015-1063.
 * alphas/betas (capacity maxit) receive the current Lanczos run,
 * history (capacity maxit+2) the explicit relative residuals; any may be NULL.
 * residual (m, may be NULL) receives rhs - H x. */
int psipm_pcg(psipm_handle* h, const double* rhs, double tol, int32_t maxit, int32_t variant,
              int32_t replacement, double gap_tolerance, double* x, double* residual,
              double* alphas, double* betas, double* history, psipm_pcg_info* info);

/* Wall-clock budget of every later PCG launch of this handle, in seconds
 * (0: none).  The HSD variant tests it after each iteration's convergence
 * test, like the deadline of psipm_v3_1_hsd.py:1054-1055, and returns the
 * current x with ok = 0 when it has passed; the spectral variant stops with
 * info = -8 (no reference code).  A budget of 1e-9 s stops after the first
 * iteration, as the reference does when it starts past its deadline. */
int psipm_set_pcg_budget(psipm_handle* h, double seconds);

/* ---- H1 Newton solve ------------------------------------------------------------
 * w = r1/theta; rhs = r2 - A w; dy = PCG(rhs); dx = w + (A^T dy)/theta
 * (psipm_spectral_preconditioner.py:651-752 without the host policy). */
int psipm_solve(psipm_handle* h, const double* r1, const double* r2, double tol, int32_t maxit,
                int32_t variant, int32_t replacement, double gap_tolerance, double* dx,
                double* dy, double* residual, double* alphas, double* betas, double* history,
                psipm_pcg_info* info);

/* ---- device-pointer variants (no host copies) ----------------------------------- */
int psipm_solve_dev(psipm_handle* h, const double* r1_dev, const double* r2_dev, double tol,
                    int32_t maxit, int32_t variant, int32_t replacement, double gap_tolerance,
                    double* dx_dev, double* dy_dev, psipm_pcg_info* info);

/* ---- device-resident PS-IPM inner loop ------------------------------------------
 * The reference's prox_eval (psipm_active_pool.py:1947-2271) and the outer
 * KKT measures of psipm_solve (:2559-2637) do their O(n) arithmetic in NumPy
 * and pass theta, r1, r2 across the KKT boundary and dx, dy back.  These
 * entry points keep the whole iterate in device memory instead: the handle
 * holds the LP data (c, b, u, pos, box), the iterate (x, y, z, w, s), the
 * proximal centre (xk, yk, zk, wk), the residuals (rd, rp), the
 * complementarity targets (rmz, rmw), a direction D = (dx, dy, dz, dw) and a
 * corrector C = (dxc, dyc, dzc, dwc).  The host keeps only the scalars the
 * loop branches on.  Sums add block partials in block order (the same bits
 * on every run); minima and maxima are exact.  */

/* Upload c[n], b[m], u[n] and the masks pos[n], box[n] (0/1 bytes) and
 * allocate the vectors (psipm_active_pool.py:2389-2392). */
int psipm_ipm_load(psipm_handle* h, const double* c, const double* b, const double* u,
                   const uint8_t* pos, const uint8_t* box);
/* Host <-> device copies of one vector set (x[n], y[m], z[n], w[n]):
 * which = 0 the iterate (x, y, z, w), 1 the centre (xk, yk, zk, wk),
 * 2 the direction D (dx, dy, dz, dw), 3 the corrector C (dxc, dyc, dzc, dwc). */
int psipm_ipm_put(psipm_handle* h, int32_t which, const double* x, const double* y,
                  const double* z, const double* w);
int psipm_ipm_get(psipm_handle* h, int32_t which, double* x, double* y, double* z, double* w);
/* to_centre = 1: centre <- iterate (psipm_active_pool.py:2670-2672).  to_centre = 0:
 * iterate <- centre, s = 1, then the box floors x = clip(x, x_floor, u - s_floor),
 * s = max(u - x, s_floor) on box columns (:1963-1967, sync_box :1860-1872). */
int psipm_ipm_copy(psipm_handle* h, int32_t to_centre);
/* Proximal residuals of the iterate (:1984-1993): rd = -(c - A^T y - z + w + rho (x - xk)),
 * rp = -(A x - b + delta (y - yk)) stay on the device; out[6] =
 * {sum_pos x z + sum_box s w, |gp|^2, |rp|^2, |rd|^2, |x - xk|^2, |y - yk|^2} with
 * g = c - A^T y + rho (x - xk) and gp = x - clip(x - g, 0, u) on pos, g elsewhere. */
int psipm_ipm_residuals(psipm_handle* h, double rho, double delta, double* out);
/* theta = theta_min + pos z/x + box w/s, non-finite entries -> theta_cap, clipped to
 * [theta_min, theta_cap] (:2014-2020), written as the handle's theta; then the
 * same as psipm_set_theta(h, theta, delta) without the host copy. */
int psipm_ipm_theta(psipm_handle* h, double theta_min, double theta_cap, double delta);
/* Complementarity targets rmz (pos), rmw (box):
 *   kind 0: -x z + p[0], -s w + p[0]                     (:2063-2087)
 *   kind 1: p[0] - dx dz, p[0] - ds dw, ds = -dx          (Mehrotra, :2113-2114)
 *   kind 2: Gondzio, p = {ta_x, ta_z, mu_target, beta_min, beta_max}:
 *           prod = (x + ta_x dx)(z + ta_z dz) (and (s - ta_x dx)(w + ta_z dw)),
 *           clip(clip(prod, bmin mu, bmax mu) - prod, -bmax mu, 2 bmax mu)  (:2180-2197) */
int psipm_ipm_targets(psipm_handle* h, int32_t kind, const double* params);
/* One Newton system (newton(), :2042-2056): r1 = rd + rmz/x - rmw/s, r2 = rp
 * into D (corrector = 0), or r1 = rmz/x - rmw/s, r2 = 0 into C (corrector = 1);
 * (dx, dy) = psipm_solve_dev(r1, r2, ...), dz = (rmz - z dx)/x on pos,
 * dw = (rmw + w dx)/s on box.  *finite = 0 when dx, dy, dz or dw holds a
 * non-finite entry.  alphas/betas/history (may be NULL) and info as in
 * psipm_solve. */
int psipm_ipm_newton(psipm_handle* h, int32_t corrector, double tol, int32_t maxit,
                     int32_t variant, int32_t replacement, double gap_tolerance, double* alphas,
                     double* betas, double* history, int32_t* finite, psipm_pcg_info* info);
/* Starting point on the device (_starting_point, psipm_active_pool.py:4122-4304,
 * the default legacy projection).  With theta = 1 and delta = 1 factored
 * (psipm_factor after the caller's policy chose the core), two projections:
 * psipm_ipm_start_solve(which = 0) solves with r1 = 0, r2 = b and keeps
 * x = A^T dy; which = 1 solves with r1 = 0, r2 = A c and keeps y = dy
 * (alphas/betas/history/info and *finite as in psipm_ipm_newton).  Then
 * psipm_ipm_start(solved) forms the start in the iterate: solved = 0 (a
 * factorisation or a projection failed) starts from x = y = 0; non-finite x or
 * y is replaced by zeros; the primal bound shifts, the dual estimate
 * r = c - A^T y (y scaled by 0.95 when |r| < 0.05 |c|), the dual slack shifts,
 * the complementarity-levelling shifts and the boxed projection follow the
 * reference.  Sums fold block partials in a fixed order (the same start on
 * every run).  out[5] (may be NULL) = {xshift1, zshift1, xshift2, zshift2,
 * 1 if y was scaled}. */
int psipm_ipm_start_solve(psipm_handle* h, int32_t which, double tol, int32_t maxit, int32_t variant,
                          int32_t replacement, double gap_tolerance, double* alphas, double* betas,
                          double* history, int32_t* finite, psipm_pcg_info* info);
int psipm_ipm_start(psipm_handle* h, int32_t solved, double* out);
/* Step to the boundary (_step_to_boundary, :1831-1837) along d = D (with_corrector
 * = 0) or d = D + gamma C: out[0] = min(1, min_{pos,dx<0} -x/dx, min_{box,ds<0} -s/ds),
 * out[1] = min(1, min_{pos,dz<0} -z/dz, min_{box,dw<0} -w/dw); ds = -dx. */
int psipm_ipm_steps(psipm_handle* h, int32_t with_corrector, double gamma, double* out);
/* *out = sum_pos (x + ax dx)(z + az dz) + sum_box (s - ax dx)(w + az dw) along
 * d = D or D + gamma C (trial mu, :2109-2110 and :2124-2128). */
int psipm_ipm_complementarity(psipm_handle* h, int32_t with_corrector, double gamma,
                              double alpha_x, double alpha_z, double* out);
/* D += gamma C (the accepted corrector, :2142-2145 and :2200-2203). */
int psipm_ipm_accept(psipm_handle* h, double gamma);
/* x += ax dx, y += az dy, z += az dz, w += az dw, then the box floors (:2231-2236). */
int psipm_ipm_update(psipm_handle* h, double alpha_x, double alpha_z);
/* Outer KKT measures (:2561-2599) after the box floors on the iterate:
 * out[6] = {max|b - A x|, max|c - A^T y - z + w|, c.x, b.y, sum_box w u,
 * sum_pos x z + sum_box s w}. */
int psipm_ipm_metrics(psipm_handle* h, double* out);
/* Lag bound of the spectral rule (psipm_spectral_preconditioner.py:396-410):
 * psipm_lag_reference keeps the current weights w = 1/theta as the reference;
 * psipm_lag_ratio returns out = {max r, min r} over r = w / max(w_ref, tiny),
 * or {inf, 0} if some r is not finite and positive. */
int psipm_lag_reference(psipm_handle* h);
int psipm_lag_ratio(psipm_handle* h, double* out);

/* ---- R2 MINRES fallback ---------------------------------------------------------
 * The reference's _minres (psipm_spectral_preconditioner.py:583-637), used by
 * solve (:717-737) when PCG broke down or stagnated: preconditioned MINRES on
 * the augmented system [diag(theta) A^T; A -delta I] [dx; q] = [r1; r2] with
 * the preconditioner diag(1/theta, P^{-1}) of the current factor, internal
 * tolerance max(eps, min(tol, 1e-8)), at most three refinement sweeps on the
 * true residual; dy = -q.  info: iterations (all sweeps), relative_residual
 * (true, over max(1, ||[r1; r2]||)), ok = 1 when it is <= max(2 tol,
 * fail_tol) (the reference's acceptance), info = 0 then, else maxit or -1.
 * FP64 handles only.  psipm_ipm_minres does the same for the device-resident
 * Newton system that psipm_ipm_newton(corrector) just failed to solve, and
 * fills D (or C) and the dual directions like it. */
int psipm_minres(psipm_handle* h, const double* r1, const double* r2, double tol, int32_t maxit,
                 double fail_tol, double* dx, double* dy, psipm_pcg_info* info);
int psipm_ipm_minres(psipm_handle* h, int32_t corrector, double tol, int32_t maxit, double fail_tol,
                     int32_t* finite, psipm_pcg_info* info);

/* ---- diagnostics ---------------------------------------------------------------- */
/* Device-side stopwatch on the handle's stream (CUDA events): start records
 * an event; stop records a second one, waits for it and returns the elapsed
 * seconds.  Everything the handle launches in between is inside the interval. */
int psipm_timer_start(psipm_handle* h);
/* One preconditioner apply with a %globaltimer stamp after every grid barrier
 * (stamps[0] at entry; *count stamps written, at most cap), and the average
 * cost of one grid barrier of the persistent kernels in *barrier_ns (may be NULL). */
int psipm_debug_apply_trace(psipm_handle* h, const double* r, double* z, int64_t* stamps, int32_t cap,
                            int32_t* count, int32_t* barrier_ns);
int psipm_timer_stop(psipm_handle* h, double* seconds);
/* Timeout path of the persistent kernels' grid barrier, without a fault:
 * `count` barriers with a poll limit of `polls` per wait, where block
 * `skip_block` (-1: none) returns without arriving, so the other blocks' first
 * wait runs out and sets the handle's timeout flag; every later wait then gives
 * up within a few polls.  Returns PSIPM_ERR_TIMEOUT when a wait ran out (the
 * handle stays usable), PSIPM_OK otherwise; *seconds is the host time of the
 * launch. */
int psipm_debug_barrier_timeout(psipm_handle* h, int32_t count, int32_t polls, int32_t skip_block,
                                double* seconds);
/* Test hook of the tensor-core trailing update alone, on GPU `device`:
 * f_out = f_in (column-major r x r, FP32) with
 *   F[i, j] -= sum_{k < kb} F[i, k0 + k] F[j, k0 + k]  for k0 + kb <= j <= i < r, j < jend,
 * computed by the kernel the FP32 factor uses (passes 3 or 1 as in
 * psipm_set_factor_tc).  Host buffers; no handle. */
int psipm_debug_syrk_tc(int32_t device, int32_t r, int32_t k0, int32_t kb, int32_t jend, int32_t passes,
                        const float* f_in, float* f_out);
/* Shape of the current symbolic factor by height level (out[8 * l + .] for
 * l < min(cap, *nlevels)): {supernodes, fused single-warp supernodes,
 * supernodes cut into GEMV tasks, forward tasks, backward tasks,
 * panel entries sum r*c, front rows sum r, largest r}. */
int psipm_debug_levels(const psipm_handle* h, int64_t* out, int32_t cap, int32_t* nlevels);
/* Kernels launched by this handle since creation (all of them are this
 * library's own kernels). */
int64_t psipm_kernel_launches(const psipm_handle* h);
/* Time of the last PCG's phases on the device (seconds): [0] H·p,
 * [1] preconditioner apply, [2] vector ops; filled only when profiling is on. */
int psipm_set_profiling(psipm_handle* h, int32_t on);

/* ---- network tree-plus-diagonal preconditioner ------------------------------------
 * The V3.1 TreePreconditioner (psipm_v3_1_hsd.py:715-785) for incidence
 * matrices (exactly two entries per column): psipm_set_tree installs the
 * spanning forest of NetworkTopology.from_incidence (:495-610) -- parent[m]
 * (-1 at roots), depth[m], and per column the child end of a forest arc or -1
 * (tree_child[n]) -- and switches the handle from the supernodal factor to
 * the tree (FP64 handles only; psipm_factor then refuses).
 * psipm_tree_factor(weights = D[n], delta) forms the pivots and multipliers
 * level by level (:732-760); every later apply and PCG of the handle uses the
 * tree solve (:762-776).  Factor and solve perform the reference's operations
 * in its order, so their results are bit-identical.  psipm_tree_get copies
 * pivot[m] and multiplier[m] (either may be NULL) to the host.  The PCG's
 * operator still uses the weights of psipm_set_theta. */
int psipm_set_tree(psipm_handle* h, const int32_t* parent, const int32_t* depth, const int32_t* tree_child);
int psipm_tree_factor(psipm_handle* h, const double* weights, double delta);
int psipm_tree_get(psipm_handle* h, double* pivot, double* multiplier);

/* ---- HSD pricing over all columns -------------------------------------------------
 * The pricing round of the V3.1 HSD loop (psipm_v3_1_hsd.py:2101-2158):
 * violation = A^T y - c tau over every column of the handle's A (products and
 * sums in index order, no contraction: bit-identical to SciPy's product), the
 * inactive columns (active[j] == 0) whose violation exceeds `threshold`
 * (the caller passes pricing_tolerance * max(tau, 1e-12)), and among them
 * the `batch` largest violations (pricing_batch; the reference's argpartition,
 * ties by ascending index here).  psipm_price_load stores c[n] once per LP.
 * candidates (capacity min(n, batch)) receive ascending column indices,
 * violation[n] (may be NULL) the full vector for the caller's reduced costs. */
int psipm_price_load(psipm_handle* h, const double* c);
int psipm_price(psipm_handle* h, const double* y, double tau, const uint8_t* active, double threshold,
                int64_t batch, double* violation, int64_t* candidates, int64_t* ncandidates);

/* ---- learned active-column selector ---------------------------------------------
 * No counterpart in the reference code: a 6 -> 64 -> 64 -> 2 perceptron per
 * candidate column whose first output re-scores the candidates before the
 * rule's own core refresh (psipm_refresh_core keeps its mandatory, retention
 * and trimming steps, psipm_stable_preconditioner.py:311-371) and whose second
 * output, averaged over the candidates, votes for the factor's first shift
 * index.  Inputs per column: log theta, log nnz, log |a_j|, log mu, previous
 * core membership and the spectral rule's log score (_scores,
 * psipm_stable_preconditioner.py:293-309).  Weights are BF16 (uint16 bit
 * patterns), biases FP32, arithmetic FP32.  Parameter order: W1[64][6],
 * W2[64][64], W3[2][64] (the PSIPM_MLP_WEIGHTS BF16 values), then b1[64],
 * b2[64], b3[2] (the PSIPM_MLP_BIASES FP32 values); gradients and the FP32
 * master copy use the same order over all PSIPM_MLP_PARAMS values. */
#define PSIPM_MLP_INPUTS 6
#define PSIPM_MLP_WEIGHTS 4608
#define PSIPM_MLP_BIASES 130
#define PSIPM_MLP_PARAMS 4738
#define PSIPM_MLP_TILE 128
/* Copy of the handle's current theta[n] (set by psipm_set_theta or
 * psipm_ipm_theta) to the host. */
int psipm_get_theta(psipm_handle* h, double* theta);
/* Features of every candidate for the current weights and core (psipm_scores
 * must have run): x[ncand][6] (host). */
int psipm_mlp_features(psipm_handle* h, double mu, float* x);
/* Replace the handle's scores by the network's (host weights w, biases b);
 * with keep > 0 only the rule's `keep` best candidates (by the scores in
 * place) keep a score, the others become -inf and no selection takes them.
 * *shift_vote (may be NULL) receives the mean second output. */
int psipm_mlp_scores(psipm_handle* h, const uint16_t* w, const float* b, double mu, int64_t keep,
                     double* shift_vote);
/* Device-pointer kernels for training, on `stream`; they allocate nothing.
 * forward: out[count][2] for x[count][6].
 * grad: loss = scale * sum_i c0 (out0_i - y0_i)^2 + c1 (out1_i - y1_i)^2 for
 * targets y[count][2], and its gradient w.r.t. every parameter (weights as
 * the BF16 values in use) into grad[PSIPM_MLP_PARAMS]; `blocks` blocks of
 * PSIPM_MLP_TILE threads each write one partial (part[blocks][PSIPM_MLP_PARAMS],
 * loss_part[blocks]) and the partials are added in block order, so the result
 * does not depend on scheduling.
 * adam: one Adam step (bias corrections for step `step` >= 1, decoupled
 * weight decay `decay` on the weights) on the FP32 master copy, which is then
 * rounded into w (BF16) and copied into b. */
int psipm_mlp_forward_dev(int64_t count, const float* x, const uint16_t* w, const float* b, float* out,
                          void* stream);
int psipm_mlp_grad_dev(int64_t count, const float* x, const float* y, float c0, float c1, const uint16_t* w,
                       const float* b, int32_t blocks, float* part, float* loss_part, float scale, float* grad,
                       float* loss, void* stream);
int psipm_mlp_adam_dev(float* master, float* m1, float* m2, const float* grad, float lr, float beta1,
                       float beta2, float eps, int32_t step, float decay, uint16_t* w, float* b, void* stream);

/* ---- allocation-free operator product -------------------------------------------
 * No counterpart in the reference: an addition for callers that cannot
 * allocate device memory (a host framework that owns the whole device pool,
 * code that may not call cudaMalloc/cudaFree because they synchronise the
 * device, a solver with a fixed, declared memory footprint).
 *   y = A diag(w) A^T v + delta v
 * Every argument except `delta` and `stream` is a DEVICE pointer owned by the
 * caller: A^T in CSR (at_ptr[n+1], at_idx, at_val: i.e. A in CSC) and A in
 * CSR (a_ptr[m+1], a_idx, a_val), w[n], v[m], y[m].  The intermediate
 * w o (A^T v) uses a fixed device array inside the library instead of an
 * allocation, so n may be at most PSIPM_STATIC_SCRATCH_MAX columns
 * (PSIPM_ERR_ARGUMENT otherwise).  The kernels run on `stream` (a
 * cudaStream_t, NULL for the default stream) and the call returns without
 * waiting for them.  The first call on a device looks up the array's device
 * address and must come before any stream capture; calls must not cross a
 * cudaDeviceReset of that device (the cached address would be stale).  All
 * calls share the one array and it keeps the last call's contents (each call
 * writes what it reads, nothing needs clearing); calls whose kernels overlap
 * on the GPU race.  A launch error already pending in the caller's context
 * makes the call return PSIPM_ERR_CUDA without launching (the error stays
 * pending). */
#define PSIPM_STATIC_SCRATCH_MAX (1ll << 20)
int psipm_normal_matvec_static(int64_t m, int64_t n, const int32_t* at_ptr, const int32_t* at_idx,
                               const double* at_val, const int32_t* a_ptr, const int32_t* a_idx,
                               const double* a_val, const double* w, double delta, const double* v,
                               double* y, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PSIPM_B200_H */
