// C ABI of libpsipm_b200 (declared in include/psipm_b200.h).
//
// Each entry point validates its arguments, runs on the handle's stream,
// synchronises before returning and converts any failure into a status code
// (the message is kept for psipm_last_error).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "common.cuh"
#include "factor_tc.h"
#include "kernels_factor.cuh"
#include "kernels_ipm.cuh"
#include "kernels_mlp.cuh"
#include "kernels_pcg.cuh"
#include "kernels_select.cuh"
#include "symbolic.h"

using namespace psipm;

namespace {

const double kShifts[8] = {0.0, 1e-14, 1e-12, 1e-10, 1e-8, 1e-6, 1e-4, 1e-2};
// fronts with more rows than this are factored by the multi-CTA blocked path
int kBigFront = 192;
// supernodes with at least this many columns use the split triangular solve
int kBigSolve = 96;

// The two thresholds can be lowered through the environment
// (PSIPM_BIG_FRONT, PSIPM_BIG_SOLVE) so that small test problems exercise
// the large-front and split-solve code paths.
void read_thresholds() {
    if (const char* v = std::getenv("PSIPM_BIG_FRONT")) kBigFront = std::max(1, std::atoi(v));
    if (const char* v = std::getenv("PSIPM_BIG_SOLVE")) kBigSolve = std::max(1, std::atoi(v));
}


template <typename T>
struct FactorStore {
    DevBuf<T> ms, G, update, front, xp, yp, dscp, GT, fvec, dinv;
    DevBuf<T> fslots, eslots, bslots;  // fixed-order accumulation slots of the apply
};

template <typename T>
struct PcgStore {
    DevBuf<T> rhs, x, r, z, p, q, t, tr, chunk_part, w, at_val, a_val;
};

// Work vectors of the MINRES fallback (n + m entries each).
struct MinresWork {
    DevBuf<double> x, rhs, cr, corr, r1, r2, y, v, w, w1, w2, t, dot;
};

// Device-resident PS-IPM state: LP data, iterate (x, y, z, w, s), proximal
// centre (xk, yk, zk, wk), residuals, complementarity targets, the Newton
// direction D = (dx, dy, dz, dw) and the corrector C = (dxc, dyc, dzc, dwc).
struct IpmStore {
    bool loaded = false;
    DevBuf<double> c, b, u;
    DevBuf<unsigned char> pos, box;
    DevBuf<double> x, y, z, w, s, xk, yk, zk, wk;
    DevBuf<double> rd, rp, rmz, rmw, r1, zero_m, aty, ax;
    DevBuf<double> dx, dy, dz, dw, dxc, dyc, dzc, dwc;
    DevBuf<double> red, wref, part;  // part: per-block partial sums (kIpmPartStride per sum)
    DevBuf<unsigned long long> redu;
    DevBuf<int> flag;
    bool have_ref = false;
};

}  // namespace

struct psipm_handle {
    int device = 0;
    int precision = PSIPM_FP64;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, tv0 = nullptr, tv1 = nullptr;
    int64_t m = 0, n = 0, nnz = 0;
    std::string err;
    int64_t launches = 0;
    int num_sms = 0;
    int coop_blocks = 0;
    int coop_max = 0;  // the largest co-resident grid of the persistent kernels
    bool deterministic = false;  // fixed-order accumulation in the preconditioner apply
    int factor_tc = 3;           // FP32 big fronts: tensor-core updates (3 = 3xTF32, 1 = TF32, 0 = CUDA cores)

    // A in CSC on the host (needed by the symbolic analysis)
    std::vector<int64_t> colptr;
    std::vector<int32_t> rowidx;
    std::vector<double> val;
    std::vector<int64_t> cand;

    // device matrix
    DevBuf<int> at_ptr, at_idx, a_ptr, a_idx;
    DevBuf<double> at_val, a_val;
    DevBuf<int> short_rows, long_rows, long_chunk_ptr, chunk_beg, chunk_end, chunk_row;
    int64_t short_nnz = 0;
    int n_short = 0, n_long = 0, n_chunks = 0, vw = 32;
    long long pcg_budget_ns = 0;  // psipm_set_pcg_budget (0: none)
    DevBuf<long long> d_cand;

    // weights and scores
    DevBuf<double> theta, w, diag_full, inv, scores;
    double delta = 0.0;
    bool have_theta = false;
    bool scores_valid = false;

    // core
    std::vector<int64_t> core;
    DevBuf<long long> d_core;
    DevBuf<unsigned char> core_flags;  // candidate-local membership of the current core
    bool core_dirty = true;            // core changed since the last symbolic analysis

    // symbolic
    Symbolic sym;
    bool have_symbolic = false;
    int n_symbolic = 0;
    double symbolic_seconds = 0.0;
    DevBuf<int> s_perm, s_iperm, s_first, s_rows, s_child_ptr, s_child_list, s_relind, s_level_sn;
    DevBuf<int> s_ent_col, s_ent_rowpos, s_ent_row, s_ent_colg, s_contrib_col;
    DevBuf<long long> s_rowptr, s_panel_off, s_update_off, s_uvec_off, s_entptr, s_ent_ptr,
        s_diag_entry, s_front_off;
    DevBuf<double> s_contrib_val;
    DevBuf<int> fwd_ptr_d, bwd_ptr_d;
    DevBuf<FwdTask> fwd_tasks_d;
    DevBuf<BwdTask> bwd_tasks_d;
    std::vector<int> fwd_ptr, bwd_ptr;
    DevBuf<int> fown_d, fdst_d;  // forward-sweep push maps (prec_apply)
    // fixed-order accumulation of the apply: per front row / update row / column
    DevBuf<int> frow_nch_d, ecnt_d, brow_nch_d, fcount_d, ecount_d, bcount_d;
    DevBuf<long long> frow_slot_d, eslot_off_d, uslot_d, brow_slot_d;
    int64_t nfslots = 0, neslots = 0, nbslots = 0;
    std::vector<int> fdst_host;  // fdst of the current analysis (slot maps are built from it)
    bool slots_ready = false;
    std::vector<int> solve_big_sn;        // supernodes with a transposed panel
    std::vector<int64_t> gt_off_host;
    DevBuf<long long> gt_off_d;
    int64_t front_total = 0;
    // per level: fronts factored one per CTA (small) and by the multi-CTA path (big)
    std::vector<int> small_ptr, small_sn, big_ptr, big_sn;
    std::vector<int64_t> front_off_host;
    DevBuf<int> small_sn_d;

    // numeric
    DevBuf<double> pval, dscp64;
    FactorStore<double> f64;
    FactorStore<float> f32;          // FP32_REFINED: factor and solve panels in FP32
    DevBuf<float> at_valf, a_valf, wf;
    bool have_factor = false;
    double factor_seconds = 0.0;
    DevBuf<int> fail;

    // PCG
    PcgStore<double> p64;
    PcgStore<float> p32;
    DevBuf<double> x64, r64, rhs64, t64, norm64, norm_part;  // FP64 refinement (FP32_REFINED)
    DevBuf<double> achunk;                                  // chunk sums of the long rows (a_times)
    DevBuf<double> part;
    DevBuf<int> ctrl, iout;
    DevBuf<unsigned int> gbar;  // grid barrier words of the persistent kernels
    DevBuf<int> gbar_err;       // set when a barrier wait timed out
    bool coop_used = false;     // a persistent kernel ran in the current entry point
    DevBuf<double> dout, alphas, betas, history;
    DevBuf<double> r1, r2, dx, dy, wr1;

    // PS-IPM vectors
    IpmStore ipm;
    MinresWork minres;

    // F3: extracted dense columns and their Woodbury correction
    std::vector<int64_t> lr_cols;
    std::vector<int> lr_ptr_host, lr_row_host;
    std::vector<double> lr_val_host;
    DevBuf<unsigned char> lr_mask;          // n: 1 on the extracted columns
    DevBuf<int> lr_ptr, lr_row;             // their CSC slices (q + 1, nnz)
    DevBuf<double> lr_val, lr_B, lr_chol;   // values; B = P_base^{-1} A_L (m x q); core Cholesky (q x q)
    DevBuf<double> d_lr, diag_score, lr_part;
    bool lr_ready = false;

    // selection scratch
    DevBuf<unsigned char> flag_a, flag_b, flag_c, mand_flags;
    DevBuf<int> eq, eqscan;
    DevBuf<unsigned int> hist;
    DevBuf<unsigned long long> counter;
    // network tree-plus-diagonal preconditioner (psipm_set_tree / psipm_tree_factor)
    bool tree_mode = false, tree_ready = false;
    int tree_levels = 0;
    DevBuf<int> t_level_ptr, t_level_nodes, t_parent, t_kid_ptr, t_kids, t_fptr, t_fcol, t_sptr, t_scol, t_cptr,
        t_ccol;
    DevBuf<double> t_D, t_diag, t_tw, t_piv, t_mult, t_pivot, t_val;
    std::vector<int> t_level_ptr_host, t_level_nodes_host;
    // HSD pricing: costs of all columns and per-round buffers
    DevBuf<double> price_c, price_y, price_v;
    DevBuf<unsigned char> price_active, price_elig, price_pick;
    bool have_price_c = false;
    // straddling ties (keys equal to the selection threshold outnumber the
    // slots left for them): cumulative count, and the last one's sizes
    int64_t tie_straddles = 0, tie_tied = 0, tie_slots = 0, selections = 0;
};

namespace {

#define LAUNCH(h, ...)                \
    do {                              \
        __VA_ARGS__;                  \
        PSIPM_CHECK_LAUNCH();         \
        ++(h)->launches;              \
    } while (0)

int fail_code(psipm_handle* h, const Failure& f) {
    if (h) h->err = f.what();
    return f.code;
}

template <typename F>
int guarded(psipm_handle* h, F&& body) {
    if (!h) return PSIPM_ERR_ARGUMENT;
    try {
        PSIPM_CUDA(cudaSetDevice(h->device));
        body();
        PSIPM_CUDA(cudaStreamSynchronize(h->stream));
        if (h->coop_used) {
            h->coop_used = false;
            int timed_out = 0;
            PSIPM_CUDA(cudaMemcpy(&timed_out, h->gbar_err.p, sizeof(int), cudaMemcpyDeviceToHost));
            if (timed_out) throw Failure(PSIPM_ERR_TIMEOUT, "a grid barrier wait of a persistent kernel timed out");
        }
        return PSIPM_OK;
    } catch (const Failure& f) {
        // a failed allocation or launch also sets the runtime's last error; clear
        // it so that it is not reported again by this handle's next launch check
        (void)cudaGetLastError();
        return fail_code(h, f);
    } catch (const std::bad_alloc&) {
        h->err = "host allocation failed";
        return PSIPM_ERR_MEMORY;
    } catch (const std::exception& e) {
        h->err = e.what();
        return PSIPM_ERR_ARGUMENT;
    }
}

inline int blocks_for(int64_t n, int threads) { return (int)std::max<int64_t>(1, (n + threads - 1) / threads); }

void require(bool cond, int code, const char* msg) {
    if (!cond) throw Failure(code, msg);
}

// ---------------------------------------------------------------------------
// device layout of A
void build_matrix(psipm_handle* h) {
    const int64_t m = h->m, n = h->n, nnz = h->nnz;
    // A^T CSR == A CSC
    std::vector<int> at_ptr(n + 1);
    for (int64_t j = 0; j <= n; ++j) at_ptr[j] = (int)h->colptr[j];
    h->at_ptr.upload(at_ptr, h->stream);
    h->at_idx.upload(h->rowidx.data(), nnz, h->stream);
    h->at_val.upload(h->val.data(), nnz, h->stream);
    // A CSR (column indices ascending within a row)
    std::vector<int> a_ptr(m + 1, 0), a_idx(nnz);
    std::vector<double> a_val(nnz);
    for (int64_t k = 0; k < nnz; ++k) ++a_ptr[h->rowidx[k] + 1];
    for (int64_t i = 0; i < m; ++i) a_ptr[i + 1] += a_ptr[i];
    {
        std::vector<int> f(a_ptr.begin(), a_ptr.end() - 1);
        for (int64_t j = 0; j < n; ++j)
            for (int64_t k = h->colptr[j]; k < h->colptr[j + 1]; ++k) {
                int i = h->rowidx[k];
                a_idx[f[i]] = (int)j;
                a_val[f[i]] = h->val[k];
                ++f[i];
            }
    }
    h->a_ptr.upload(a_ptr, h->stream);
    h->a_idx.upload(a_idx, h->stream);
    h->a_val.upload(a_val, h->stream);
    if (h->precision == PSIPM_FP32_REFINED) {
        std::vector<float> af(a_val.begin(), a_val.end()), atf(h->val.begin(), h->val.end());
        h->a_valf.upload(af, h->stream);
        h->at_valf.upload(atf, h->stream);
        PSIPM_CUDA(cudaStreamSynchronize(h->stream));
    }
    // short / long rows
    std::vector<int> shortr, longr, lcp{0}, cb, ce, crow;
    int64_t short_nnz = 0, short_cnt = 0;
    for (int64_t i = 0; i < m; ++i) {
        int len = a_ptr[i + 1] - a_ptr[i];
        if (len > kLongRow) {
            longr.push_back((int)i);
            for (int b = a_ptr[i]; b < a_ptr[i + 1]; b += kLongRow) {
                cb.push_back(b);
                ce.push_back(std::min(b + kLongRow, a_ptr[i + 1]));
                crow.push_back((int)i);
            }
            lcp.push_back((int)cb.size());
        } else {
            shortr.push_back((int)i);
            short_nnz += len;
            ++short_cnt;
        }
    }
    double avg = short_cnt ? (double)short_nnz / (double)short_cnt : 1.0;
    int vw = 1;
    while (vw < 32 && vw < avg) vw <<= 1;
    h->vw = vw;
    h->n_short = (int)shortr.size();
    h->n_long = (int)longr.size();
    h->n_chunks = (int)cb.size();
    h->short_rows.upload(shortr, h->stream);
    h->long_rows.upload(longr, h->stream);
    h->long_chunk_ptr.upload(lcp, h->stream);
    h->chunk_beg.upload(cb, h->stream);
    h->chunk_end.upload(ce, h->stream);
    h->chunk_row.upload(crow, h->stream);
    h->short_nnz = short_nnz;
    // candidates: columns with at least two nonzeros
    h->cand.clear();
    for (int64_t j = 0; j < n; ++j)
        if (h->colptr[j + 1] - h->colptr[j] >= 2) h->cand.push_back(j);
    std::vector<long long> cl(h->cand.begin(), h->cand.end());
    h->d_cand.upload(cl, h->stream);
}

template <typename T>
SpmvLayout spmv_layout(psipm_handle* h) {
    SpmvLayout s;
    s.m = (int)h->m;
    s.n = (int)h->n;
    s.at_ptr = h->at_ptr.p;
    s.at_idx = h->at_idx.p;
    s.a_ptr = h->a_ptr.p;
    s.a_idx = h->a_idx.p;
    s.vw = h->vw;
    s.short_rows = h->short_rows.p;
    s.n_short = h->n_short;
    s.long_rows = h->long_rows.p;
    s.n_long = h->n_long;
    s.long_chunk_ptr = h->long_chunk_ptr.p;
    s.chunk_beg = h->chunk_beg.p;
    s.chunk_end = h->chunk_end.p;
    s.n_chunks = h->n_chunks;
    return s;
}

// The barrier words are cleared before every persistent launch (a timed-out
// wait can leave the arrival count behind); the timeout flag once per entry point.
void prepare_barrier(psipm_handle* h) {
    h->gbar.reserve(2);
    h->gbar_err.reserve(1);
    PSIPM_CUDA(cudaMemsetAsync(h->gbar.p, 0, 2 * sizeof(unsigned int), h->stream));
    if (!h->coop_used) PSIPM_CUDA(cudaMemsetAsync(h->gbar_err.p, 0, sizeof(int), h->stream));
    h->coop_used = true;
}

GridBarrier grid_barrier(psipm_handle* h) {
    h->gbar.reserve(2);
    h->gbar_err.reserve(1);
    GridBarrier b;
    b.bar = h->gbar.p;
    b.err = h->gbar_err.p;
    return b;
}

FactorStore<double>& fstore(psipm_handle* h, const double*) { return h->f64; }
FactorStore<float>& fstore(psipm_handle* h, const float*) { return h->f32; }
PcgStore<double>& pstore(psipm_handle* h, const double*) { return h->p64; }
PcgStore<float>& pstore(psipm_handle* h, const float*) { return h->p32; }
const double* at_values(psipm_handle* h, const double*) { return h->at_val.p; }
const float* at_values(psipm_handle* h, const float*) { return h->at_valf.p; }
const double* a_values(psipm_handle* h, const double*) { return h->a_val.p; }
const float* a_values(psipm_handle* h, const float*) { return h->a_valf.p; }
const double* weights(psipm_handle* h, const double*) { return h->w.p; }
const float* weights(psipm_handle* h, const float*) { return h->wf.p; }

// Slot maps of the deterministic apply, built on first use after each
// symbolic analysis (handles that never ask for determinism pay nothing).
void build_slot_maps(psipm_handle* h) {
    const Symbolic& s = h->sym;
    cudaStream_t st = h->stream;
    const std::vector<int>& fdst = h->fdst_host;
// slots of the fixed-order accumulation (kernels_pcg.cuh, slot_arrive):
    //  forward: every GEMV task writes one partial per row of its 4-row group;
    //  update rows: one slot per (child update row -> parent front row), in
    //  ascending child and row order; backward: one partial per covering task
    const int64_t nfront = std::max<int64_t>(1, s.sn_rowptr[s.ns]);
    std::vector<int> frow_nch(nfront, 0), ecnt(nfront, 0), brow_nch(std::max<int64_t>(1, h->m), 0);
    std::vector<long long> frow_slot(nfront, 0), eslot_off(nfront + 1, 0), brow_slot(std::max<int64_t>(1, h->m), 0);
    std::vector<long long> uslot(std::max<int64_t>(1, s.uvec_off[s.ns]), 0);
    int64_t nf = 0, nb = 0;
    for (int sn = 0; sn < s.ns; ++sn) {
        const int first = s.sn_first[sn], c = s.sn_first[sn + 1] - first;
        const int64_t rb = s.sn_rowptr[sn];
        const int r = (int)(s.sn_rowptr[sn + 1] - rb);
        if (r <= kSmallRows && c <= 32) continue;  // fused: rows written directly
        const int cch = (c + kApplyChunk - 1) / kApplyChunk;
        for (int i0 = 0; i0 < r; i0 += kApplyRows) {
            const int i1 = std::min(r, i0 + kApplyRows);
            const int nch = (i1 - 1 < c) ? (i1 - 1) / kApplyChunk + 1 : cch;
            for (int ii = i0; ii < i1; ++ii) {
                frow_nch[rb + ii] = nch;
                frow_slot[rb + ii] = nf;
                nf += nch;
            }
        }
        const int rch = (r + kApplyChunk - 1) / kApplyChunk;
        for (int j0 = 0; j0 < c; j0 += kApplyRows) {
            const int nch = rch - j0 / kApplyChunk;
            for (int jj = j0; jj < std::min(c, j0 + kApplyRows); ++jj) {
                brow_nch[first + jj] = nch;
                brow_slot[first + jj] = nb;
                nb += nch;
            }
        }
    }
    for (int64_t u = 0; u < s.uvec_off[s.ns]; ++u)
        if (fdst[u] >= 0) ++ecnt[fdst[u]];
    for (int64_t g = 0; g < nfront; ++g) eslot_off[g + 1] = eslot_off[g] + ecnt[g];
    {
        std::vector<long long> fill(eslot_off.begin(), eslot_off.end() - 1);
        for (int64_t u = 0; u < s.uvec_off[s.ns]; ++u)  // children ascending, rows ascending
            if (fdst[u] >= 0) uslot[u] = fill[fdst[u]]++;
    }
    h->nfslots = std::max<int64_t>(1, nf);
    h->nbslots = std::max<int64_t>(1, nb);
    h->neslots = std::max<int64_t>(1, eslot_off[nfront]);
    h->frow_nch_d.upload(frow_nch, st);
    h->frow_slot_d.upload(frow_slot, st);
    h->ecnt_d.upload(ecnt, st);
    h->eslot_off_d.upload(eslot_off, st);
    h->uslot_d.upload(uslot, st);
    h->brow_nch_d.upload(brow_nch, st);
    h->brow_slot_d.upload(brow_slot, st);
    h->fcount_d.zero(nfront, st);
    h->ecount_d.zero(nfront, st);
    h->bcount_d.zero(std::max<int64_t>(1, h->m), st);

    h->slots_ready = true;
}

// A multifrontal workspace above this size is given back after every
// factorisation (the PCG that follows does not use it); smaller ones stay
// allocated for the next factorisation.
constexpr int64_t kKeepWorkspaceBytes = int64_t(16) << 30;

template <typename T>
void release_workspace(FactorStore<T>& fs) {
    if ((int64_t)((fs.update.n + fs.front.n) * sizeof(T)) > kKeepWorkspaceBytes) {
        fs.update.release();
        fs.front.release();
    }
}

template <typename T, typename P = T>
PcgArgs<T, P> pcg_args(psipm_handle* h) {
    const T* tag = nullptr;
    const P* ptag = nullptr;
    PcgArgs<T, P> a;
    a.sp = spmv_layout<T>(h);
    a.at_val = at_values(h, tag);
    a.a_val = a_values(h, tag);
    a.w = weights(h, tag);
    a.delta = (T)h->delta;
    a.gb = grid_barrier(h);
    a.budget_ns = h->pcg_budget_ns;
    PrecLayout<P>& pc = a.pc;
    pc.m = (int)h->m;
    FactorStore<P>& fs = fstore(h, ptag);
    if (h->have_symbolic) {
        pc.perm = h->s_perm.p;
        pc.iperm = h->s_iperm.p;
        pc.dscp = fs.dscp.p;
        pc.G = fs.G.p;
        pc.panel_off = h->s_panel_off.p;
        pc.sn_first = h->s_first.p;
        pc.sn_rowptr = h->s_rowptr.p;
        pc.sn_rows = h->s_rows.p;
        pc.uvec_off = h->s_uvec_off.p;
        pc.fown = h->fown_d.p;
        pc.fdst = h->fdst_d.p;
        pc.deterministic = h->deterministic ? 1 : 0;
        if (h->deterministic) {
            if (!h->slots_ready) build_slot_maps(h);
            fs.fslots.reserve(h->nfslots);
            fs.eslots.reserve(h->neslots);
            fs.bslots.reserve(h->nbslots);
        }
        pc.frow_nch = h->frow_nch_d.p;
        pc.frow_slot = h->frow_slot_d.p;
        pc.fcount = h->fcount_d.p;
        pc.fslots = fs.fslots.p;
        pc.ecnt = h->ecnt_d.p;
        pc.eslot_off = h->eslot_off_d.p;
        pc.uslot = h->uslot_d.p;
        pc.ecount = h->ecount_d.p;
        pc.eslots = fs.eslots.p;
        pc.brow_nch = h->brow_nch_d.p;
        pc.brow_slot = h->brow_slot_d.p;
        pc.bcount = h->bcount_d.p;
        pc.bslots = fs.bslots.p;
        pc.nfront = h->sym.sn_rowptr[h->sym.ns];
        pc.nlevels = h->sym.nlevels;
        pc.fwd_ptr = h->fwd_ptr_d.p;
        pc.fwd_tasks = h->fwd_tasks_d.p;
        pc.bwd_ptr = h->bwd_ptr_d.p;
        pc.bwd_tasks = h->bwd_tasks_d.p;
        pc.xp = fs.xp.p;
        pc.yp = fs.yp.p;
        pc.fvec = fs.fvec.p;
        pc.GT = fs.GT.p;
        pc.gt_off = h->s_panel_off.p;
        if (h->lr_ready) {
            pc.lr_q = (int)h->lr_cols.size();
            pc.lr_ptr = h->lr_ptr.p;
            pc.lr_row = h->lr_row.p;
            pc.lr_val = h->lr_val.p;
            pc.lr_B = h->lr_B.p;
            pc.lr_chol = h->lr_chol.p;
            pc.lr_part = h->lr_part.p;
        }
    }
    if (h->tree_ready) {
        TreeLayout& t = pc.tree;
        t.m = (int)h->m;
        t.nlevels = h->tree_levels;
        t.level_ptr = h->t_level_ptr.p;
        t.level_nodes = h->t_level_nodes.p;
        t.parent = h->t_parent.p;
        t.kid_ptr = h->t_kid_ptr.p;
        t.kids = h->t_kids.p;
        t.mult = h->t_mult.p;
        t.pivot = h->t_pivot.p;
        t.val = h->t_val.p;
    }
    PcgStore<T>& st = pstore(h, tag);
    const int64_t m = h->m, n = h->n;
    st.x.reserve(m);
    st.r.reserve(m);
    st.z.reserve(m);
    st.p.reserve(m);
    st.q.reserve(m);
    st.t.reserve(n);
    st.tr.reserve(m);
    st.rhs.reserve(m);
    st.chunk_part.reserve(std::max(1, h->n_chunks));
    h->part.reserve((size_t)2 * 4 * std::max(1, h->coop_blocks));
    h->ctrl.reserve(4);
    h->iout.reserve(16);
    h->dout.reserve(8);
    a.x = st.x.p;
    a.r = st.r.p;
    a.z = st.z.p;
    a.p = st.p.p;
    a.q = st.q.p;
    a.t = st.t.p;
    a.tr = st.tr.p;
    a.chunk_part = st.chunk_part.p;
    a.part = h->part.p;
    a.ctrl = h->ctrl.p;
    a.iout = h->iout.p;
    a.dout = h->dout.p;
    return a;
}

size_t pcg_smem() { return (size_t)kPcgWarps * kStageChunk * sizeof(double); }  // covers float too

// the persistent kernels take more than the default 48 KB of dynamic shared memory
void set_pcg_smem_attributes() {
    const int bytes = (int)pcg_smem();
    const void* fns[] = {(const void*)k_pcg<double, double>, (const void*)k_pcg<double, float>,
                         (const void*)k_pcg<float, float>,  (const void*)k_apply<double, double>,
                         (const void*)k_apply<double, float>, (const void*)k_matvec<double, double>};
    for (const void* fn : fns)
        PSIPM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
}

void launch_coop(psipm_handle* h, const void* fn, void** args) {
    prepare_barrier(h);
    dim3 grid(h->coop_blocks), block(kPcgThreads);
    PSIPM_CUDA(cudaLaunchCooperativeKernel(fn, grid, block, args, pcg_smem(), h->stream));
    ++h->launches;
}

// ---------------------------------------------------------------------------
// symbolic analysis of the current core and upload of its arrays
void analyse(psipm_handle* h) {
    auto t0 = std::chrono::steady_clock::now();
    h->have_symbolic = false;  // until the new analysis and its device arrays are complete
    read_thresholds();
    SymbolicOptions opt;
    Symbolic S;
    std::vector<int64_t> core(h->core.begin(), h->core.end());
    int rc = build_symbolic((int32_t)h->m, h->n, h->colptr.data(), h->rowidx.data(), h->val.data(),
                            core.data(), (int64_t)core.size(), opt, S);
    if (rc != 0) throw Failure(PSIPM_ERR_SYMBOLIC, "symbolic analysis failed with code " + std::to_string(rc));
    h->sym = std::move(S);
    Symbolic& s = h->sym;
    cudaStream_t st = h->stream;
    h->s_perm.upload(s.perm, st);
    h->s_iperm.upload(s.iperm, st);
    h->s_first.upload(s.sn_first, st);
    h->s_rows.upload(s.sn_rows, st);
    h->s_child_ptr.upload(s.child_ptr, st);
    h->s_child_list.upload(s.child_list, st);
    h->s_relind.upload(s.relind, st);
    h->s_level_sn.upload(s.level_sn, st);
    h->s_ent_col.upload(s.ent_col, st);
    h->s_ent_rowpos.upload(s.ent_rowpos, st);
    h->s_contrib_col.upload(s.contrib_col, st);
    h->s_contrib_val.upload(s.contrib_val, st);
    auto up64 = [&](DevBuf<long long>& d, const std::vector<int64_t>& v) {
        std::vector<long long> t(v.begin(), v.end());
        d.upload(t, st);
        PSIPM_CUDA(cudaStreamSynchronize(st));
    };
    up64(h->s_rowptr, s.sn_rowptr);
    up64(h->s_panel_off, s.panel_off);
    up64(h->s_update_off, s.update_off);
    up64(h->s_uvec_off, s.uvec_off);
    up64(h->s_entptr, s.sn_entptr);
    up64(h->s_ent_ptr, s.ent_ptr);
    up64(h->s_diag_entry, s.diag_entry);
    // entry row/col in permuted numbering (for the Jacobi scaling)
    std::vector<int> er(s.nentries), ec(s.nentries);
    for (int64_t e = 0; e < s.nentries; ++e) {
        int sn = s.ent_sn[e];
        ec[e] = s.sn_first[sn] + s.ent_col[e];
        er[e] = s.sn_rows[s.sn_rowptr[sn] + s.ent_rowpos[e]];
    }
    h->s_ent_row.upload(er, st);
    h->s_ent_colg.upload(ec, st);
    // front workspace offsets per level
    std::vector<int64_t> foff(s.ns, 0);
    int64_t fmax_total = 0;
    for (int l = 0; l < s.nlevels; ++l) {
        int64_t off = 0;
        for (int q = s.level_ptr[l]; q < s.level_ptr[l + 1]; ++q) {
            int sn = s.level_sn[q];
            int64_t r = s.sn_rowptr[sn + 1] - s.sn_rowptr[sn];
            foff[sn] = off;
            off += r * r;
        }
        fmax_total = std::max(fmax_total, off);
    }
    h->front_total = fmax_total;
    h->front_off_host = foff;
    up64(h->s_front_off, foff);
    // triangular-solve tasks per level (kernels_pcg.cuh, prec_apply): fused
    // single-warp tasks for small supernodes, 2-D GEMV tasks of kApplyRows
    // rows x kApplyChunk contraction entries for the others (all-zero blocks
    // of the triangular L11^{-1} skipped)
    std::vector<FwdTask> ft;
    std::vector<BwdTask> bt;
    h->fwd_ptr.assign(s.nlevels + 1, 0);
    h->bwd_ptr.assign(s.nlevels + 1, 0);
    for (int l = 0; l < s.nlevels; ++l) {
        for (int q = s.level_ptr[l]; q < s.level_ptr[l + 1]; ++q) {
            const int sn = s.level_sn[q];
            const int first = s.sn_first[sn];
            const int c = s.sn_first[sn + 1] - first;
            const int r = (int)(s.sn_rowptr[sn + 1] - s.sn_rowptr[sn]);
            FwdTask f{};
            f.f = s.sn_rowptr[sn];
            f.u = s.uvec_off[sn];
            f.first = first;
            f.c = c;
            f.s = -1;
            BwdTask b{};
            b.rb = s.sn_rowptr[sn];
            b.first = first;
            b.c = c;
            b.r = r;
            b.s = -1;
            if (r <= kSmallRows && c <= 32) {
                f.s = sn;
                b.s = sn;
                ft.push_back(f);
                bt.push_back(b);
                continue;
            }
            for (int i0 = 0; i0 < r; i0 += kApplyRows) {
                f.i0 = i0;
                f.i1 = std::min(r, i0 + kApplyRows);
                f.g = s.panel_off[sn] + (int64_t)i0 * c;
                for (int j0 = 0; j0 < c; j0 += kApplyChunk) {
                    if (f.i1 - 1 < c && j0 > f.i1 - 1) break;  // above the diagonal of L11^{-1}
                    f.j0 = j0;
                    ft.push_back(f);
                }
            }
            for (int j0 = 0; j0 < c; j0 += kApplyRows) {
                b.j0 = j0;
                b.j1 = std::min(c, j0 + kApplyRows);
                b.g = s.panel_off[sn] + (int64_t)j0 * r;
                for (int i0 = 0; i0 < r; i0 += kApplyChunk) {
                    if (std::min(r, i0 + kApplyChunk) - 1 < j0) continue;  // rows above the block's first column
                    b.i0 = i0;
                    bt.push_back(b);
                }
            }
        }
        h->fwd_ptr[l + 1] = (int)ft.size();
        h->bwd_ptr[l + 1] = (int)bt.size();
    }
    // push targets of the forward sweep: pivot rows carry their permuted
    // column (fown), update-vector rows their position in the parent (fdst)
    require(s.sn_rowptr[s.ns] < (int64_t)INT32_MAX, PSIPM_ERR_UNSUPPORTED, "front rows exceed int32");
    {
        std::vector<int> fown(std::max<int64_t>(1, s.sn_rowptr[s.ns]), -1);
        std::vector<int> fdst(std::max<int64_t>(1, s.uvec_off[s.ns]), -1);
        for (int sn = 0; sn < s.ns; ++sn) {
            const int first = s.sn_first[sn], c = s.sn_first[sn + 1] - first;
            const int64_t rb = s.sn_rowptr[sn], r = s.sn_rowptr[sn + 1] - rb;
            for (int q = 0; q < c; ++q) fown[rb + q] = first + q;
            const int par = s.sn_parent[sn];
            for (int64_t q = c; q < r; ++q) {
                const int64_t e = s.uvec_off[sn] + (q - c);
                fdst[e] = par >= 0 ? (int)(s.sn_rowptr[par] + s.relind[e]) : -1;
            }
        }
        h->fown_d.upload(fown, st);
        h->fdst_d.upload(fdst, st);
        h->fdst_host = std::move(fdst);
        h->slots_ready = false;
    }
    // per level: fronts factored one per CTA (small) or by the multi-CTA path (big)
    h->small_ptr.assign(s.nlevels + 1, 0);
    h->big_ptr.assign(s.nlevels + 1, 0);
    h->small_sn.clear();
    h->big_sn.clear();
    for (int l = 0; l < s.nlevels; ++l) {
        for (int q = s.level_ptr[l]; q < s.level_ptr[l + 1]; ++q) {
            int sn = s.level_sn[q];
            int r = (int)(s.sn_rowptr[sn + 1] - s.sn_rowptr[sn]);
            if (r > kBigFront)
                h->big_sn.push_back(sn);
            else
                h->small_sn.push_back(sn);
        }
        h->small_ptr[l + 1] = (int)h->small_sn.size();
        h->big_ptr[l + 1] = (int)h->big_sn.size();
    }
    h->small_sn_d.upload(h->small_sn, st);
    h->fwd_ptr_d.upload(h->fwd_ptr, st);
    h->bwd_ptr_d.upload(h->bwd_ptr, st);
    h->fwd_tasks_d.upload(ft, st);
    h->bwd_tasks_d.upload(bt, st);
    // numeric storage (entries are assembled in FP64, the factor lives in the
    // handle's precision)
    h->pval.reserve(std::max<int64_t>(1, s.nentries));
    auto reserve_factor = [&](auto& fs) {
        fs.ms.fit(std::max<int64_t>(1, s.nentries));
        fs.G.fit(std::max<int64_t>(1, s.panel_total));
        fs.GT.fit(std::max<int64_t>(1, s.panel_total));
        fs.xp.reserve(h->m);
        fs.yp.reserve(h->m);
        fs.dscp.reserve(h->m);
        fs.fvec.reserve(std::max<int64_t>(1, s.sn_rowptr[s.ns]));
    };
    if (h->precision != PSIPM_FP64)
        reserve_factor(h->f32);
    else
        reserve_factor(h->f64);
    h->dscp64.reserve(h->m);
    h->fail.reserve(1);
    PSIPM_CUDA(cudaStreamSynchronize(st));
    h->have_symbolic = true;
    h->have_factor = false;
    h->core_dirty = false;
    ++h->n_symbolic;
    h->symbolic_seconds =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void compute_weights(psipm_handle* h) {
    const int64_t n = h->n, m = h->m;
    h->w.reserve(n);
    h->diag_full.reserve(m);
    LAUNCH(h, k_weights<<<blocks_for(n, 256), 256, 0, h->stream>>>(n, h->theta.p, h->w.p));
    const bool lr = !h->lr_cols.empty();
    LAUNCH(h, k_diag_full<<<blocks_for(m, 256), 256, 0, h->stream>>>(
                  (int)m, h->a_ptr.p, h->a_idx.p, h->a_val.p, h->w.p, lr ? h->lr_mask.p : nullptr,
                  h->diag_full.p));
    if (lr) {
        // scores see A2_factor w_F + A2_low_rank w_L (psipm_stable_preconditioner.py:298-303)
        h->d_lr.zero(m, h->stream);
        h->diag_score.reserve(m);
        for (size_t a = 0; a < h->lr_cols.size(); ++a) {
            const int nnz = h->lr_ptr_host[a + 1] - h->lr_ptr_host[a];
            LAUNCH(h, k_diag_lr_column<<<blocks_for(nnz, 256), 256, 0, h->stream>>>(
                          nnz, h->lr_row.p + h->lr_ptr_host[a], h->lr_val.p + h->lr_ptr_host[a], h->w.p,
                          (long long)h->lr_cols[a], h->d_lr.p));
        }
        LAUNCH(h, k_add_rn<<<blocks_for(m, 256), 256, 0, h->stream>>>((int)m, h->diag_full.p, h->d_lr.p,
                                                                      h->diag_score.p));
    }
    if (h->precision == PSIPM_FP32_REFINED) {
        h->wf.reserve(n);
        LAUNCH(h, k_cast<float><<<blocks_for(n, 256), 256, 0, h->stream>>>(n, h->w.p, h->wf.p));
    }
}


// Columns per panel of the FP32 tensor-core path: the trailing update's K.
constexpr int kTcPanel = 256;

// one large front by the multi-CTA blocked path (kernels_factor.cuh)
template <typename T>
void factor_big_front(psipm_handle* h, int sn, const FactorArgs<T>& fa) {
    const Symbolic& s = h->sym;
    cudaStream_t st = h->stream;
    const int r = (int)(s.sn_rowptr[sn + 1] - s.sn_rowptr[sn]);
    const int c = s.sn_first[sn + 1] - s.sn_first[sn];
    // front offsets live on the device; the host keeps its own copy
    T* F = fa.front + h->front_off_host[sn];
    PSIPM_CUDA(cudaMemsetAsync(F, 0, (size_t)r * r * sizeof(T), st));
    const long long e0 = s.sn_entptr[sn], e1 = s.sn_entptr[sn + 1];
    if (e1 > e0)
        LAUNCH(h, k_front_scatter<T><<<std::min(blocks_for(e1 - e0, 256), 4096), 256, 0, st>>>(
                      F, r, e0, e1, fa.ent_col, fa.ent_rowpos, fa.ms, fa.eta));
    for (int ci = s.child_ptr[sn]; ci < s.child_ptr[sn + 1]; ++ci) {
        const int ch = s.child_list[ci];
        const int rc = (int)(s.uvec_off[ch + 1] - s.uvec_off[ch]);
        if (rc <= 0) continue;
        const long long n2 = (long long)rc * rc;
        LAUNCH(h, k_front_extend_add<T><<<std::min(blocks_for(n2, 256), 8192), 256, 0, st>>>(
                      F, r, fa.update + s.update_off[ch], rc, fa.relind + s.uvec_off[ch]));
    }
    const size_t trsm_smem = kNB * (kNB + 1) * sizeof(T);
    const size_t syrk_smem = 2 * kNB * (kNB + 1) * sizeof(T);
    // Cholesky of the diagonal block at k0 and the rows below it
    auto panel_step = [&](int k0, int kb) {
        LAUNCH(h, k_potrf_diag<T><<<1, 256, 0, st>>>(F, r, k0, kb, fa.fail));
        const int rows = r - k0 - kb;
        if (rows > 0)
            LAUNCH(h, k_trsm_panel<T><<<blocks_for(rows, kTrsmRows), kTrsmRows, trsm_smem, st>>>(F, r, k0, kb));
        return rows;
    };
    bool tensor_cores = false;
    if constexpr (std::is_same<T, float>::value) tensor_cores = h->factor_tc > 0;
    if (!tensor_cores) {
        for (int k0 = 0; k0 < c; k0 += kNB) {
            const int kb = std::min(kNB, c - k0);
            const int rows = panel_step(k0, kb);
            if (rows <= 0) continue;
            const int ntile = (rows + 63) / 64;
            LAUNCH(h, k_syrk_update<T><<<ntile * (ntile + 1) / 2, 256, syrk_smem, st>>>(F, r, k0, kb, ntile));
        }
    } else if constexpr (std::is_same<T, float>::value) {
        // two-level blocking: panels of kTcPanel columns factored by kNB-wide
        // steps whose updates stay inside the panel, then one tensor-core
        // update of the whole trailing matrix with K = the panel width
        for (int kp = 0; kp < c; kp += kTcPanel) {
            const int kpe = std::min(c, kp + kTcPanel);
            for (int k0 = kp; k0 < kpe; k0 += kNB) {
                const int kb = std::min(kNB, kpe - k0);
                if (panel_step(k0, kb) > 0 && k0 + kb < kpe) {
                    syrk_update_tc(F, r, k0, kb, kpe, h->factor_tc, fa.fail, st);
                    ++h->launches;
                }
            }
            if (kpe < r) {
                syrk_update_tc(F, r, kp, kpe - kp, r, h->factor_tc, fa.fail, st);
                ++h->launches;
            }
        }
    }
    if (r > c) {
        const long long n2 = (long long)(r - c) * (r - c);
        LAUNCH(h, k_extract_update<T><<<std::min(blocks_for(n2, 256), 8192), 256, 0, st>>>(
                      F, r, c, fa.update + s.update_off[sn]));
    }
    // G = [I; L21] L11^{-1} by column blocks from the right (kernels_factor.cuh)
    T* G = fa.G + s.panel_off[sn];
    const int nblk = (c + kGB - 1) / kGB;
    const size_t g_smem = 2 * kGB * (kGB + 1) * sizeof(T);
    LAUNCH(h, k_diag_block_inv<T><<<nblk, kGB, kGB * (kGB + 1) * sizeof(T), st>>>(F, r, c, fa.dinv));
    LAUNCH(h, k_g_init<T><<<dim3((c + 31) / 32, (r + 31) / 32), dim3(32, 8), 0, st>>>(F, r, c, fa.dinv, G));
    if (r > c)
        LAUNCH(h, k_g_convert<T><<<blocks_for(r - c, kGB), 256, g_smem, st>>>(r, c, fa.dinv, nblk - 1, G));
    for (int jb = nblk - 1; jb >= 1; --jb)
        LAUNCH(h, k_g_update<T><<<dim3(blocks_for(r - jb * kGB, kGB), jb), 256, g_smem, st>>>(F, r, c, fa.dinv, jb,
                                                                                           G));
    dim3 tgrid((c + 31) / 32, (r + 31) / 32), tblock(32, 8);
    LAUNCH(h, k_transpose_panel<T><<<tgrid, tblock, 0, st>>>(fa.G + s.panel_off[sn], r, c, fa.GT + s.panel_off[sn]));
}


// F1 in FP64 (bit-reproducible entries and Jacobi scale), then the factor in
// precision T with the shift ladder; returns the shift index used or -1.
template <typename T>
int factor_numeric(psipm_handle* h, double delta, int start_shift) {
    const T* tag = nullptr;
    Symbolic& s = h->sym;
    cudaStream_t st = h->stream;
    FactorStore<T>& fs = fstore(h, tag);
    // multifrontal workspace: update matrices, one level's fronts, the
    // diagonal-block inverses of a big front
    fs.update.fit(std::max<int64_t>(1, s.update_total));
    fs.front.fit(std::max<int64_t>(1, h->front_total));
    fs.dinv.reserve((int64_t)(s.max_cols / kGB + 1) * kGB * kGB);
    if (s.nentries)
        LAUNCH(h, k_assemble_entries<<<blocks_for(s.nentries, 256), 256, 0, st>>>(
                      s.nentries, h->s_ent_ptr.p, h->s_contrib_col.p, h->s_contrib_val.p, h->d_core.p, h->w.p,
                      h->pval.p));
    LAUNCH(h, k_diag_fix<<<blocks_for(h->m, 256), 256, 0, st>>>((int)h->m, h->s_diag_entry.p, h->s_perm.p,
                                                                 h->diag_full.p, delta, h->pval.p, h->dscp64.p));
    if (s.nentries)
        LAUNCH(h, k_scale_entries<T><<<blocks_for(s.nentries, 256), 256, 0, st>>>(
                      s.nentries, h->s_ent_row.p, h->s_ent_colg.p, h->pval.p, h->dscp64.p, fs.ms.p));
    LAUNCH(h, k_cast<T><<<blocks_for(h->m, 256), 256, 0, st>>>(h->m, h->dscp64.p, fs.dscp.p));
    FactorArgs<T> fa;
    fa.sn_first = h->s_first.p;
    fa.sn_rowptr = h->s_rowptr.p;
    fa.panel_off = h->s_panel_off.p;
    fa.update_off = h->s_update_off.p;
    fa.uvec_off = h->s_uvec_off.p;
    fa.child_ptr = h->s_child_ptr.p;
    fa.child_list = h->s_child_list.p;
    fa.relind = h->s_relind.p;
    fa.sn_entptr = h->s_entptr.p;
    fa.ent_col = h->s_ent_col.p;
    fa.ent_rowpos = h->s_ent_rowpos.p;
    fa.ms = fs.ms.p;
    fa.G = fs.G.p;
    fa.GT = fs.GT.p;
    fa.update = fs.update.p;
    fa.front = fs.front.p;
    fa.dinv = fs.dinv.p;
    fa.front_off = h->s_front_off.p;
    fa.fail = h->fail.p;
    require((int)h->small_ptr.size() == s.nlevels + 1 && (int)h->big_ptr.size() == s.nlevels + 1 &&
                h->small_ptr[s.nlevels] + h->big_ptr[s.nlevels] == s.ns,
            PSIPM_ERR_STATE, "level tables do not match the symbolic factor");
    for (int k = start_shift; k < 8; ++k) {
        fa.eta = kShifts[k];
        PSIPM_CUDA(cudaMemsetAsync(h->fail.p, 0, sizeof(int), st));
        for (int l = 0; l < s.nlevels; ++l) {
            int cnt = h->small_ptr[l + 1] - h->small_ptr[l];
            if (cnt)
                LAUNCH(h, k_factor_level<T><<<cnt, kFactorThreads, 0, st>>>(fa, h->small_sn_d.p + h->small_ptr[l]));
            for (int q = h->big_ptr[l]; q < h->big_ptr[l + 1]; ++q) factor_big_front<T>(h, h->big_sn[q], fa);
        }
        int failed = 0;
        PSIPM_CUDA(cudaMemcpyAsync(&failed, h->fail.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        PSIPM_CUDA(cudaStreamSynchronize(st));
        if (failed & kTcErrWait) {
            release_workspace(fs);
            throw Failure(PSIPM_ERR_CUDA, "tensor-core front update: completion wait expired");
        }
        if (!failed) {
            release_workspace(fs);
            return k;
        }
    }
    release_workspace(fs);
    return -1;
}

// ---------------------------------------------------------------------------
// radix top-k among eligible entries; sets out_flag[i] = 1 for the selected
void select_top(psipm_handle* h, const double* score, const unsigned char* mask, int64_t nsc,
                int64_t count, unsigned char* out_flag) {
    if (count <= 0 || nsc == 0) return;
    ++h->selections;
    cudaStream_t st = h->stream;
    h->counter.reserve(1);
    PSIPM_CUDA(cudaMemsetAsync(h->counter.p, 0, sizeof(unsigned long long), st));
    const int gb = std::min(blocks_for(nsc, kSelectThreads), 4 * std::max(1, h->num_sms));
    LAUNCH(h, k_count_eligible<<<gb, kSelectThreads, 0, st>>>(nsc, score, mask, h->counter.p));
    unsigned long long nel = 0;
    PSIPM_CUDA(cudaMemcpyAsync(&nel, h->counter.p, sizeof(nel), cudaMemcpyDeviceToHost, st));
    PSIPM_CUDA(cudaStreamSynchronize(st));
    h->eq.reserve(nsc);
    h->eqscan.reserve(nsc);
    if ((int64_t)nel <= count) {
        LAUNCH(h, k_mark_threshold<<<blocks_for(nsc, 256), 256, 0, st>>>(nsc, score, mask, 0ull, 1,
                                                                          out_flag, h->eq.p));
        return;
    }
    unsigned long long prefix = 0, pmask = 0;
    int64_t need = count;
    h->hist.reserve(256);
    std::vector<unsigned int> hh(256);
    for (int shift = 56; shift >= 0; shift -= 8) {
        PSIPM_CUDA(cudaMemsetAsync(h->hist.p, 0, 256 * sizeof(unsigned int), st));
        LAUNCH(h, k_radix_hist<<<gb, kSelectThreads, 0, st>>>(nsc, score, mask, shift, prefix, pmask,
                                                               h->hist.p));
        PSIPM_CUDA(cudaMemcpyAsync(hh.data(), h->hist.p, 256 * sizeof(unsigned int),
                                   cudaMemcpyDeviceToHost, st));
        PSIPM_CUDA(cudaStreamSynchronize(st));
        int64_t cum = 0;
        int b = 255;
        for (; b >= 0; --b) {
            if (cum + (int64_t)hh[b] >= need) break;
            cum += hh[b];
        }
        if (b < 0) throw Failure(PSIPM_ERR_BOUNDS, "radix select lost track of the threshold");
        need -= cum;
        prefix |= (unsigned long long)b << shift;
        pmask |= 0xffull << shift;
    }
    // keys > prefix selected; first `need` equal keys by index
    LAUNCH(h, k_mark_threshold<<<blocks_for(nsc, 256), 256, 0, st>>>(nsc, score, mask, prefix, 0,
                                                                      out_flag, h->eq.p));
    // exclusive scan of eq on the host (ties are rare and the array is modest)
    std::vector<int> eqh(nsc);
    PSIPM_CUDA(cudaMemcpyAsync(eqh.data(), h->eq.p, nsc * sizeof(int), cudaMemcpyDeviceToHost, st));
    PSIPM_CUDA(cudaStreamSynchronize(st));
    int acc = 0;
    for (int64_t i = 0; i < nsc; ++i) {
        int v = eqh[i];
        eqh[i] = acc;
        acc += v;
    }
    if (acc > need) {  // the cut falls inside a run of equal keys: the index rule decides
        ++h->tie_straddles;
        h->tie_tied = acc;
        h->tie_slots = need;
    }
    h->eqscan.upload(eqh, st);
    LAUNCH(h, k_mark_ties<<<blocks_for(nsc, 256), 256, 0, st>>>(nsc, h->eq.p, h->eqscan.p, need, out_flag));
}

int64_t count_flags(psipm_handle* h, const unsigned char* flags, int64_t n) {
    std::vector<unsigned char> f(n);
    if (n) PSIPM_CUDA(cudaMemcpyAsync(f.data(), flags, n, cudaMemcpyDeviceToHost, h->stream));
    PSIPM_CUDA(cudaStreamSynchronize(h->stream));
    int64_t c = 0;
    for (auto v : f) c += v;
    return c;
}

std::vector<unsigned char> download_flags(psipm_handle* h, const unsigned char* flags, int64_t n) {
    std::vector<unsigned char> f(n);
    if (n) PSIPM_CUDA(cudaMemcpyAsync(f.data(), flags, n, cudaMemcpyDeviceToHost, h->stream));
    PSIPM_CUDA(cudaStreamSynchronize(h->stream));
    return f;
}

void set_core_internal(psipm_handle* h, std::vector<int64_t> newcore) {
    if (newcore != h->core) {
        h->core = std::move(newcore);
        h->core_dirty = true;
    }
    std::vector<long long> c(h->core.begin(), h->core.end());
    h->d_core.upload(c, h->stream);
    // candidate-local flags
    const int64_t nc = (int64_t)h->cand.size();
    std::vector<unsigned char> f(nc, 0);
    for (int64_t g : h->core) {
        auto it = std::lower_bound(h->cand.begin(), h->cand.end(), g);
        if (it != h->cand.end() && *it == g) f[it - h->cand.begin()] = 1;
    }
    h->core_flags.upload(f, h->stream);
}

template <typename T, typename P = T>
void run_pcg(psipm_handle* h, const T* rhs_dev, double tol, int maxit, int variant, int replacement,
             double gap_tol, psipm_pcg_info* info) {
    require(h->have_factor, PSIPM_ERR_STATE, "pcg before a successful factor");
    PcgArgs<T, P> a = pcg_args<T, P>(h);
    a.rhs = rhs_dev;
    a.variant = variant;
    a.maxit = maxit;
    a.replacement = replacement;
    a.tol = tol;
    a.gap_tol = gap_tol;
    h->alphas.reserve(std::max(1, maxit));
    h->betas.reserve(std::max(1, maxit));
    h->history.reserve(maxit + 2);
    a.alphas = h->alphas.p;
    a.betas = h->betas.p;
    a.history = h->history.p;
    PSIPM_CUDA(cudaMemsetAsync(h->ctrl.p, 0, 4 * sizeof(int), h->stream));
    void* args[] = {&a};
    PSIPM_CUDA(cudaEventRecord(h->ev0, h->stream));
    launch_coop(h, (const void*)k_pcg<T, P>, args);
    PSIPM_CUDA(cudaEventRecord(h->ev1, h->stream));
    int io[16];
    double dd[8];
    PSIPM_CUDA(cudaMemcpyAsync(io, h->iout.p, 9 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    PSIPM_CUDA(cudaMemcpyAsync(dd, h->dout.p, 6 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    PSIPM_CUDA(cudaStreamSynchronize(h->stream));
    float ms = 0.f;
    PSIPM_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    if (info) {
        std::memset(info, 0, sizeof(*info));
        info->info = io[0];
        info->iterations = io[1];
        info->matvecs = io[2];
        info->replacements = io[3];
        info->residual_checks = io[4];
        info->n_alpha = io[5];
        info->n_beta = io[6];
        info->n_history = io[7];
        info->ok = io[8];
        info->relative_residual = dd[0];
        info->seconds = ms * 1e-3;
        for (int q = 0; q < 4; ++q) info->phase_seconds[q] = dd[2 + q];
    }
}

void copy_out(psipm_handle* h, double* host, const double* dev, int64_t n) {
    if (host && n) PSIPM_CUDA(cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
}

__global__ void k_scatter_column(int nnz, const int* __restrict__ rows, const double* __restrict__ vals,
                                 double* __restrict__ dense) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nnz) dense[rows[e]] = vals[e];
}

// F3: after a numeric factorisation, the Woodbury data for the extracted dense
// columns (psipm_active_pool.py:906-947): B = P_base^{-1} A_L by q applies of
// the base factor, the core C = A_L^T B + Theta_L (symmetrised) and its
// Cholesky factor with the relative shift ladder (0, 1e-14, ..., 1e-8).
void prepare_low_rank(psipm_handle* h) {
    require(h->precision == PSIPM_FP64, PSIPM_ERR_UNSUPPORTED, "dense-column extraction is FP64 only");
    const int q = (int)h->lr_cols.size();
    const int64_t m = h->m;
    cudaStream_t st = h->stream;
    h->lr_B.reserve((int64_t)q * m);
    DevBuf<double> dense;
    dense.reserve(m);
    PcgArgs<double, double> a = pcg_args<double, double>(h);  // lr_ready is false: the base apply
    for (int c = 0; c < q; ++c) {
        const int nnz = h->lr_ptr_host[c + 1] - h->lr_ptr_host[c];
        PSIPM_CUDA(cudaMemsetAsync(dense.p, 0, m * sizeof(double), st));
        LAUNCH(h, k_scatter_column<<<blocks_for(nnz, 256), 256, 0, st>>>(nnz, h->lr_row.p + h->lr_ptr_host[c],
                                                                         h->lr_val.p + h->lr_ptr_host[c], dense.p));
        const double* in = dense.p;
        double* out = h->lr_B.p + (int64_t)c * m;
        void* args[] = {&a, (void*)&in, (void*)&out};
        launch_coop(h, (const void*)k_apply<double, double>, args);
    }
    std::vector<double> B((size_t)q * m), th(q);
    PSIPM_CUDA(cudaMemcpyAsync(B.data(), h->lr_B.p, B.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    for (int c = 0; c < q; ++c)
        PSIPM_CUDA(cudaMemcpyAsync(&th[c], h->theta.p + h->lr_cols[c], sizeof(double), cudaMemcpyDeviceToHost, st));
    PSIPM_CUDA(cudaStreamSynchronize(st));
    std::vector<double> core((size_t)q * q, 0.0);
    for (int c = 0; c < q; ++c)
        for (int d = 0; d < q; ++d) {
            double acc = 0.0;
            for (int e = h->lr_ptr_host[c]; e < h->lr_ptr_host[c + 1]; ++e)
                acc += h->lr_val_host[e] * B[(size_t)d * m + h->lr_row_host[e]];
            core[(size_t)c * q + d] = acc;
        }
    for (int c = 0; c < q; ++c) core[(size_t)c * q + c] += th[c];
    for (int c = 0; c < q; ++c)
        for (int d = 0; d < c; ++d) {
            const double v = 0.5 * (core[(size_t)c * q + d] + core[(size_t)d * q + c]);
            core[(size_t)c * q + d] = core[(size_t)d * q + c] = v;
        }
    double scale = 1.0;
    for (int c = 0; c < q; ++c) scale = std::max(scale, std::fabs(core[(size_t)c * q + c]));
    for (double rel : {0.0, 1e-14, 1e-12, 1e-10, 1e-8}) {
        std::vector<double> L((size_t)q * q, 0.0);
        bool ok = true;
        for (int i = 0; i < q && ok; ++i)
            for (int j = 0; j <= i; ++j) {
                double v = core[(size_t)i * q + j] + (i == j ? rel * scale : 0.0);
                for (int k = 0; k < j; ++k) v -= L[(size_t)i * q + k] * L[(size_t)j * q + k];
                if (i == j) {
                    if (!(v > 0.0)) {
                        ok = false;
                        break;
                    }
                    L[(size_t)i * q + i] = std::sqrt(v);
                } else {
                    L[(size_t)i * q + j] = v / L[(size_t)j * q + j];
                }
            }
        if (!ok) continue;
        h->lr_chol.upload(L, st);
        PSIPM_CUDA(cudaStreamSynchronize(st));
        h->lr_ready = true;
        return;
    }
    h->have_factor = false;
    throw Failure(PSIPM_ERR_NOT_PD, "low-rank correction is not positive definite");
}

}  // namespace

namespace {
const double* solve_normal(psipm_handle* h, const double* rhs, double tol, int maxit, int variant, int replacement,
                           double gap_tol, psipm_pcg_info* info);
}  // namespace

// ===========================================================================
extern "C" {

int psipm_create(int64_t m, int64_t n, int64_t nnz, const int64_t* colptr, const int32_t* rowidx,
                 const double* values, int32_t device, int32_t precision, psipm_handle** out) {
    if (!out || m <= 0 || n < 0 || nnz < 0 || !colptr || (nnz && (!rowidx || !values)))
        return PSIPM_ERR_ARGUMENT;
    if (m >= (1ll << 31) || n >= (1ll << 31) || nnz >= (1ll << 31)) return PSIPM_ERR_UNSUPPORTED;
    if (precision != PSIPM_FP64 && precision != PSIPM_FP32_REFINED && precision != PSIPM_FP32_PRECOND)
        return PSIPM_ERR_ARGUMENT;
    *out = nullptr;
    if (colptr[0] != 0 || colptr[n] != nnz) return PSIPM_ERR_ARGUMENT;
    for (int64_t j = 0; j < n; ++j) {
        if (colptr[j + 1] < colptr[j]) return PSIPM_ERR_ARGUMENT;
        for (int64_t k = colptr[j]; k < colptr[j + 1]; ++k) {
            if (rowidx[k] < 0 || rowidx[k] >= m) return PSIPM_ERR_ARGUMENT;
            if (k > colptr[j] && rowidx[k] <= rowidx[k - 1]) return PSIPM_ERR_ARGUMENT;
        }
    }
    std::unique_ptr<psipm_handle> h(new psipm_handle());
    h->device = device;
    h->precision = precision;
    h->m = m;
    h->n = n;
    h->nnz = nnz;
    h->colptr.assign(colptr, colptr + n + 1);
    h->rowidx.assign(rowidx, rowidx + nnz);
    h->val.assign(values, values + nnz);
    int rc = guarded(h.get(), [&]() {
        int ndev = 0;
        PSIPM_CUDA(cudaGetDeviceCount(&ndev));
        require(device >= 0 && device < ndev, PSIPM_ERR_ARGUMENT, "no such CUDA device");
        PSIPM_CUDA(cudaSetDevice(device));
        PSIPM_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        PSIPM_CUDA(cudaEventCreate(&h->ev0));
        PSIPM_CUDA(cudaEventCreate(&h->ev1));
        PSIPM_CUDA(cudaEventCreate(&h->tv0));
        PSIPM_CUDA(cudaEventCreate(&h->tv1));
        cudaDeviceProp prop;
        PSIPM_CUDA(cudaGetDeviceProperties(&prop, device));
        h->num_sms = prop.multiProcessorCount;
        require(prop.cooperativeLaunch, PSIPM_ERR_UNSUPPORTED, "device lacks cooperative launch");
        set_pcg_smem_attributes();
        PSIPM_CUDA(cudaFuncSetAttribute(k_trsm_panel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(2 * kNB * (kNB + 1) * sizeof(float))));
        PSIPM_CUDA(cudaFuncSetAttribute(k_syrk_update<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(2 * kNB * (kNB + 1) * sizeof(float))));
        PSIPM_CUDA(cudaFuncSetAttribute(k_trsm_panel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(2 * kNB * (kNB + 1) * sizeof(double))));
        PSIPM_CUDA(cudaFuncSetAttribute(k_syrk_update<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(2 * kNB * (kNB + 1) * sizeof(double))));
        PSIPM_CUDA(cudaFuncSetAttribute(k_g_update<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(2 * kGB * (kGB + 1) * sizeof(double))));
        PSIPM_CUDA(cudaFuncSetAttribute(k_g_convert<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(2 * kGB * (kGB + 1) * sizeof(double))));
        PSIPM_CUDA(cudaFuncSetAttribute(k_diag_block_inv<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)((2 * kGB * (kGB + 1) + 4 * kGB) * sizeof(double))));
        int per_sm = 0;
        PSIPM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg<double, double>, kPcgThreads,
                                                                 pcg_smem()));
        int per_sm2 = 0;
        PSIPM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, k_apply<double, double>, kPcgThreads,
                                                                 pcg_smem()));
        int per_sm3 = 0;
        PSIPM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm3, k_matvec<double, double>, kPcgThreads,
                                                                 pcg_smem()));
        int per_sm4 = 0;
        PSIPM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm4, k_pcg<float, float>, kPcgThreads, pcg_smem()));
        int per_sm5 = 0;
        PSIPM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm5, k_pcg<double, float>, kPcgThreads, pcg_smem()));
        per_sm = std::min(std::min(std::min(per_sm, per_sm2), std::min(per_sm3, per_sm4)), per_sm5);
        require(per_sm >= 1, PSIPM_ERR_UNSUPPORTED, "PCG kernel does not fit on an SM");
        // blocks per SM of the persistent kernels (PSIPM_BLOCKS_PER_SM overrides)
        int want = 4;
        if (const char* v = std::getenv("PSIPM_BLOCKS_PER_SM")) want = std::max(1, std::atoi(v));
        h->coop_blocks = std::min(per_sm, want) * h->num_sms;
        h->coop_max = h->coop_blocks;
        build_matrix(h.get());
    });
    if (rc != PSIPM_OK) {
        std::string msg = h->err;
        // keep the handle so the caller can read the message
        *out = h.release();
        return rc;
    }
    *out = h.release();
    return PSIPM_OK;
}

void psipm_destroy(psipm_handle* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->tv0) cudaEventDestroy(h->tv0);
    if (h->tv1) cudaEventDestroy(h->tv1);
    cudaStream_t s = h->stream;
    delete h;
    if (s) cudaStreamDestroy(s);
}

const char* psipm_last_error(const psipm_handle* h) { return h ? h->err.c_str() : "null handle"; }

int psipm_set_low_rank(psipm_handle* h, const int64_t* cols, int64_t q) {
    if (q < 0 || q > PSIPM_LOW_RANK_MAX || (q && !cols)) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        if ((int64_t)h->lr_cols.size() == q && std::equal(h->lr_cols.begin(), h->lr_cols.end(), cols)) return;
        require(!h->have_symbolic && h->core.empty(), PSIPM_ERR_STATE, "set_low_rank after a core was set");
        require(q == 0 || h->precision == PSIPM_FP64, PSIPM_ERR_UNSUPPORTED, "dense-column extraction is FP64 only");
        for (int64_t t = 0; t < q; ++t)
            require(cols[t] >= 0 && cols[t] < h->n && (t == 0 || cols[t] > cols[t - 1]), PSIPM_ERR_ARGUMENT,
                    "low-rank columns must be sorted, distinct and in range");
        const int64_t n = h->n;
        cudaStream_t st = h->stream;
        h->lr_cols.assign(cols, cols + q);
        std::vector<unsigned char> mask(std::max<int64_t>(1, n), 0);
        h->lr_ptr_host.assign(1, 0);
        h->lr_row_host.clear();
        h->lr_val_host.clear();
        for (int64_t t = 0; t < q; ++t) {
            const int64_t j = cols[t];
            mask[j] = 1;
            for (int64_t e = h->colptr[j]; e < h->colptr[j + 1]; ++e) {
                h->lr_row_host.push_back(h->rowidx[e]);
                h->lr_val_host.push_back(h->val[e]);
            }
            h->lr_ptr_host.push_back((int)h->lr_row_host.size());
        }
        h->lr_mask.upload(mask, st);
        h->lr_ptr.upload(h->lr_ptr_host, st);
        h->lr_row.upload(h->lr_row_host.empty() ? std::vector<int>(1, 0) : h->lr_row_host, st);
        h->lr_val.upload(h->lr_val_host.empty() ? std::vector<double>(1, 0.0) : h->lr_val_host, st);
        h->lr_part.reserve((int64_t)std::max(1, h->coop_blocks) * kLowRankMax);
        h->lr_ready = false;
        // the candidates of the factor exclude the extracted columns (psipm_stable_preconditioner.py:169-172)
        h->cand.clear();
        for (int64_t j = 0; j < n; ++j)
            if (!mask[j] && h->colptr[j + 1] - h->colptr[j] >= 2) h->cand.push_back(j);
        std::vector<long long> cl(h->cand.begin(), h->cand.end());
        h->d_cand.upload(cl, st);
        h->have_theta = false;
    });
}

int64_t psipm_num_candidates(const psipm_handle* h) { return h ? (int64_t)h->cand.size() : -1; }

int psipm_get_candidates(const psipm_handle* h, int64_t* out) {
    if (!h || !out) return PSIPM_ERR_ARGUMENT;
    std::copy(h->cand.begin(), h->cand.end(), out);
    return PSIPM_OK;
}

int psipm_set_theta(psipm_handle* h, const double* theta, double delta) {
    if (!theta) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        h->theta.upload(theta, h->n, h->stream);
        h->delta = delta;
        compute_weights(h);
        h->have_theta = true;
        h->scores_valid = false;
    });
}

int psipm_scores(psipm_handle* h, double fill_weight, double* scores, double* diagonal) {
    return guarded(h, [&]() {
        require(h->have_theta, PSIPM_ERR_STATE, "scores before set_theta");
        const int64_t m = h->m, nc = (int64_t)h->cand.size();
        const double tiny = 2.2250738585072014e-308;
        h->inv.reserve(m);
        h->scores.reserve(std::max<int64_t>(1, nc));
        const double* diag = h->lr_cols.empty() ? h->diag_full.p : h->diag_score.p;
        LAUNCH(h, k_inv_diag<<<blocks_for(m, 256), 256, 0, h->stream>>>((int)m, diag,
                                                                        std::max(h->delta, tiny), h->inv.p));
        if (nc)
            LAUNCH(h, k_scores<<<blocks_for(nc, 256), 256, 0, h->stream>>>(
                          nc, h->d_cand.p, h->at_ptr.p, h->at_idx.p, h->at_val.p, h->w.p, h->inv.p,
                          fill_weight, h->scores.p));
        h->scores_valid = true;
        copy_out(h, scores, h->scores.p, nc);
        copy_out(h, diagonal, diag, m);
    });
}

int psipm_top_k(psipm_handle* h, const double* scores, int64_t nscores, const uint8_t* mask, int64_t count,
                int64_t* out, int64_t* nout) {
    if (!scores || nscores < 0 || !out || !nout) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        DevBuf<double> sc;
        DevBuf<unsigned char> mk, fl;
        sc.upload(scores, nscores, h->stream);
        if (mask) mk.upload(mask, nscores, h->stream);
        fl.zero(std::max<int64_t>(1, nscores), h->stream);
        select_top(h, sc.p, mask ? mk.p : nullptr, nscores, count, fl.p);
        auto f = download_flags(h, fl.p, nscores);
        int64_t k = 0;
        for (int64_t i = 0; i < nscores; ++i)
            if (f[i]) out[k++] = i;
        *nout = k;
    });
}

int psipm_refresh_core(psipm_handle* h, int64_t target, double retention, int32_t stable,
                       const int64_t* mandatory_local, int64_t nmandatory, int64_t* core_out, int64_t* ncore,
                       double* retained) {
    if (nmandatory < 0 || (nmandatory && !mandatory_local) || !core_out || !ncore) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        require(h->scores_valid, PSIPM_ERR_STATE, "refresh before scores");
        cudaStream_t st = h->stream;
        const int64_t nc = (int64_t)h->cand.size();
        target = std::min(target, nc);
        for (int64_t q = 0; q < nmandatory; ++q)
            require(mandatory_local[q] >= 0 && mandatory_local[q] < nc && (q == 0 || mandatory_local[q] > mandatory_local[q - 1]),
                    PSIPM_ERR_ARGUMENT, "mandatory positions must be sorted candidate-local indices");
        const int64_t nn = std::max<int64_t>(1, nc);
        h->flag_a.zero(nn, st);  // fixed
        h->flag_b.zero(nn, st);  // scratch selection
        h->flag_c.zero(nn, st);  // mask
        h->mand_flags.zero(nn, st);
        DevBuf<long long> mand;
        {
            std::vector<long long> mv(mandatory_local, mandatory_local + nmandatory);
            mand.upload(mv, st);
        }
        if (nmandatory) {
            LAUNCH(h, k_set_flags<<<blocks_for(nmandatory, 256), 256, 0, st>>>(nmandatory, mand.p, 1, h->flag_a.p));
            LAUNCH(h, k_set_flags<<<blocks_for(nmandatory, 256), 256, 0, st>>>(nmandatory, mand.p, 1, h->mand_flags.p));
        }
        const int64_t old_size = (int64_t)h->core.size();
        bool have_old = old_size > 0 && h->core_flags.p && h->core_flags.n >= (size_t)nc;
        if (stable && have_old && target) {
            int64_t keep = std::min<int64_t>(old_size, std::max<int64_t>(0, (int64_t)std::floor(retention * (double)target)));
            if (keep) {
                select_top(h, h->scores.p, h->core_flags.p, nc, keep, h->flag_b.p);
                LAUNCH(h, k_flag_op<<<blocks_for(nc, 256), 256, 0, st>>>(nc, h->flag_a.p, h->flag_b.p, 1, h->flag_a.p));
            }
        }
        int64_t nfixed = count_flags(h, h->flag_a.p, nc);
        if (nfixed > target) {
            if (nmandatory >= target) {
                PSIPM_CUDA(cudaMemsetAsync(h->flag_a.p, 0, nc, st));
                if (target)
                    LAUNCH(h, k_set_flags<<<blocks_for(target, 256), 256, 0, st>>>(target, mand.p, 1, h->flag_a.p));
            } else {
                // optional = fixed & ~mandatory; keep the best (target - |mandatory|)
                LAUNCH(h, k_flag_op<<<blocks_for(nc, 256), 256, 0, st>>>(nc, h->flag_a.p, h->mand_flags.p, 0, h->flag_c.p));
                PSIPM_CUDA(cudaMemsetAsync(h->flag_b.p, 0, nc, st));
                select_top(h, h->scores.p, h->flag_c.p, nc, target - nmandatory, h->flag_b.p);
                LAUNCH(h, k_flag_op<<<blocks_for(nc, 256), 256, 0, st>>>(nc, h->mand_flags.p, h->flag_b.p, 1, h->flag_a.p));
            }
            nfixed = count_flags(h, h->flag_a.p, nc);
        }
        const int64_t remaining = target - nfixed;
        if (remaining > 0) {
            // available = ~fixed (fixed scores count as -inf, i.e. not eligible)
            std::vector<unsigned char> fa = download_flags(h, h->flag_a.p, nc);
            for (auto& v : fa) v = !v;
            h->flag_c.upload(fa, st);
            PSIPM_CUDA(cudaMemsetAsync(h->flag_b.p, 0, nc, st));
            select_top(h, h->scores.p, h->flag_c.p, nc, remaining, h->flag_b.p);
            LAUNCH(h, k_flag_op<<<blocks_for(nc, 256), 256, 0, st>>>(nc, h->flag_a.p, h->flag_b.p, 1, h->flag_a.p));
        }
        std::vector<unsigned char> nf = download_flags(h, h->flag_a.p, nc);
        std::vector<unsigned char> of = have_old ? download_flags(h, h->core_flags.p, nc)
                                                 : std::vector<unsigned char>(nc, 0);
        std::vector<int64_t> newcore;
        int64_t inter = 0;
        for (int64_t i = 0; i < nc; ++i) {
            if (nf[i]) newcore.push_back(h->cand[i]);
            if (nf[i] && of[i]) ++inter;
        }
        if (retained) *retained = old_size ? (double)inter / (double)std::max<int64_t>(1, old_size) : 1.0;
        std::copy(newcore.begin(), newcore.end(), core_out);
        *ncore = (int64_t)newcore.size();
        set_core_internal(h, std::move(newcore));
    });
}

int psipm_set_deterministic(psipm_handle* h, int32_t on) {
    if (!h) return PSIPM_ERR_ARGUMENT;
    h->deterministic = on != 0;
    return PSIPM_OK;
}

int psipm_set_factor_tc(psipm_handle* h, int32_t passes) {
    if (!h || (passes != 0 && passes != 1 && passes != 3)) return PSIPM_ERR_ARGUMENT;
    h->factor_tc = passes;
    return PSIPM_OK;
}

int psipm_set_grid(psipm_handle* h, int32_t blocks) {
    if (!h || blocks < 0) return PSIPM_ERR_ARGUMENT;
    if (h->lr_ready || !h->lr_cols.empty()) return PSIPM_ERR_STATE;  // lr_part is sized for the grid
    h->coop_blocks = blocks == 0 ? h->coop_max : std::min(blocks, h->coop_max);
    return PSIPM_OK;
}

int psipm_tie_info(const psipm_handle* h, int64_t* out) {
    if (!h || !out) return PSIPM_ERR_ARGUMENT;
    out[0] = h->tie_straddles;
    out[1] = h->tie_tied;
    out[2] = h->tie_slots;
    out[3] = h->selections;
    return PSIPM_OK;
}

int psipm_set_core(psipm_handle* h, const int64_t* core, int64_t ncore) {
    if (ncore < 0 || (ncore && !core)) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        std::vector<int64_t> c(core, core + ncore);
        for (int64_t q = 0; q < ncore; ++q)
            require(c[q] >= 0 && c[q] < h->n && (q == 0 || c[q] > c[q - 1]), PSIPM_ERR_ARGUMENT,
                    "core must hold sorted, distinct column indices");
        set_core_internal(h, std::move(c));
    });
}

int psipm_factor(psipm_handle* h, double delta, int32_t start_shift, int32_t* shift_index,
                 psipm_factor_info* info) {
    if (start_shift < 0 || start_shift > 7) return PSIPM_ERR_ARGUMENT;
    int status = guarded(h, [&]() {
        require(h->have_theta, PSIPM_ERR_STATE, "factor before set_theta");
        require(!h->tree_mode, PSIPM_ERR_STATE, "the handle uses the tree preconditioner (psipm_tree_factor)");
        h->have_factor = false;  // until this factorisation succeeds (a failed one leaves no factor)
        int used = -1;
        Symbolic& s = h->sym;
        cudaStream_t st = h->stream;
        try {
            if (h->core_dirty || !h->have_symbolic) analyse(h);
            h->delta = delta;
            PSIPM_CUDA(cudaEventRecord(h->ev0, st));
            used = h->precision != PSIPM_FP64 ? factor_numeric<float>(h, delta, start_shift)
                                              : factor_numeric<double>(h, delta, start_shift);
        } catch (const Failure& f) {
            if (f.code == PSIPM_ERR_MEMORY) {
                // give every factor buffer back, so that a smaller core fits
                // next time; the next factorisation analyses afresh
                (void)cudaStreamSynchronize(st);
                auto drop = [](auto& fs) {
                    fs.ms.release();
                    fs.G.release();
                    fs.GT.release();
                    fs.update.release();
                    fs.front.release();
                    fs.fvec.release();
                    fs.dinv.release();
                };
                drop(h->f64);
                drop(h->f32);
                h->have_symbolic = false;
            }
            throw;
        }
        PSIPM_CUDA(cudaEventRecord(h->ev1, st));
        PSIPM_CUDA(cudaEventSynchronize(h->ev1));
        float ms = 0.f;
        PSIPM_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
        h->factor_seconds = ms * 1e-3;
        if (shift_index) *shift_index = used;
        if (info) {
            info->nsupernodes = s.ns;
            info->nlevels = s.nlevels;
            info->max_front = s.max_front;
            info->symbolic_analyses = h->n_symbolic;
            info->nnz_factor = s.nnz_L;
            info->flops = s.flops;
            info->symbolic_seconds = h->symbolic_seconds;
            info->factor_seconds = h->factor_seconds;
        }
        if (used < 0) {
            h->have_factor = false;
            throw Failure(PSIPM_ERR_NOT_PD, "Cholesky failed even with a 1e-2 shift");
        }
        PSIPM_CUDA(cudaStreamSynchronize(st));
        h->have_factor = true;
        h->lr_ready = false;
        if (!h->lr_cols.empty()) prepare_low_rank(h);
    });
    return status;
}

int psipm_apply(psipm_handle* h, const double* r, double* z) {
    if (!r || !z) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        require(h->have_factor, PSIPM_ERR_STATE, "apply before a successful factor");
        h->r1.upload(r, h->m, h->stream);
        h->r2.reserve(h->m);
        if (h->precision != PSIPM_FP64) {
            PcgArgs<double, float> a = pcg_args<double, float>(h);
            const double* in = h->r1.p;
            double* outp = h->r2.p;
            void* args[] = {&a, (void*)&in, (void*)&outp};
            launch_coop(h, (const void*)k_apply<double, float>, args);
        } else {
            PcgArgs<double, double> a = pcg_args<double, double>(h);
            const double* in = h->r1.p;
            double* outp = h->r2.p;
            void* args[] = {&a, (void*)&in, (void*)&outp};
            launch_coop(h, (const void*)k_apply<double, double>, args);
        }
        copy_out(h, z, h->r2.p, h->m);
    });
}

int psipm_matvec(psipm_handle* h, const double* v, double* y) {
    if (!v || !y) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        require(h->have_theta, PSIPM_ERR_STATE, "matvec before set_theta");
        PcgArgs<double, double> a = pcg_args<double, double>(h);  // the operator is applied in FP64 here
        PSIPM_CUDA(cudaMemcpyAsync(h->p64.p.p, v, h->m * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        void* args[] = {&a};
        launch_coop(h, (const void*)k_matvec<double, double>, args);
        copy_out(h, y, h->p64.q.p, h->m);
    });
}

int psipm_pcg(psipm_handle* h, const double* rhs, double tol, int32_t maxit, int32_t variant, int32_t replacement,
              double gap_tolerance, double* x, double* residual, double* alphas, double* betas, double* history,
              psipm_pcg_info* info) {
    if (!rhs || !x || maxit < 0 || (variant != PSIPM_PCG_SPECTRAL && variant != PSIPM_PCG_HSD))
        return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        h->rhs64.upload(rhs, h->m, h->stream);
        psipm_pcg_info local;
        const double* xd = solve_normal(h, h->rhs64.p, tol, maxit, variant, replacement, gap_tolerance, &local);
        copy_out(h, x, xd, h->m);
        if (residual) copy_out(h, residual, h->r64.p, h->m);
        copy_out(h, alphas, h->alphas.p, local.n_alpha);
        copy_out(h, betas, h->betas.p, local.n_beta);
        copy_out(h, history, h->history.p, local.n_history);
        if (info) *info = local;
    });
}

}  // extern "C"

// ---- H1 solve --------------------------------------------------------------
namespace {

// y[rows[r]] = (row rows[r] of CSR M) . v, W lanes per listed row
template <int W>
__global__ void k_list_rows(int nrows, const int* __restrict__ rows, const int* __restrict__ ptr,
                            const int* __restrict__ idx, const double* __restrict__ val,
                            const double* __restrict__ v, double* __restrict__ y) {
    constexpr int kRowsPerWarp = 32 / W;
    const int lane = threadIdx.x & (W - 1);
    const int sub = (threadIdx.x & 31) / W;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = warp * kRowsPerWarp; base < nrows; base += nwarps * kRowsPerWarp) {
        const long long r = base + sub;
        const int i = r < nrows ? rows[r] : 0;
        double acc = 0.0;
        if (r < nrows)
            for (int k = ptr[i] + lane; k < ptr[i + 1]; k += W) acc += val[k] * v[idx[k]];
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, W);
        if (lane == 0 && r < nrows) y[i] = acc;
    }
}

// long rows: one warp per kLongRow-entry chunk writes the chunk's sum; then
// one warp per long row adds its chunk sums in a fixed order (lane-strided,
// then a butterfly), so y is the same on every run
__global__ void k_chunk_rows(int nchunks, const int* __restrict__ cbeg, const int* __restrict__ cend,
                             const int* __restrict__ idx, const double* __restrict__ val,
                             const double* __restrict__ v, double* __restrict__ part) {
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long c = warp; c < nchunks; c += nwarps) {
        double acc = 0.0;
        for (int k = cbeg[c] + lane; k < cend[c]; k += 32) acc += val[k] * v[idx[k]];
        acc = warp_sum(acc);
        if (lane == 0) part[c] = acc;
    }
}
__global__ void k_long_rows(int nlong, const int* __restrict__ rows, const int* __restrict__ chunk_ptr,
                            const double* __restrict__ part, double* __restrict__ y) {
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long l = warp; l < nlong; l += nwarps) {
        double acc = 0.0;
        for (int c = chunk_ptr[l] + lane; c < chunk_ptr[l + 1]; c += 32) acc += part[c];
        acc = warp_sum(acc);
        if (lane == 0) y[rows[l]] = acc;
    }
}

// out = sum of part[0 .. n) in a fixed order (one block)
__global__ void k_fold_sum(long long n, const double* __restrict__ part, double* __restrict__ out) {
    __shared__ double scratch[32];
    double acc = 0.0;
    for (long long k = threadIdx.x; k < n; k += blockDim.x) acc += part[k];
    acc = block_sum(acc, scratch);
    if (threadIdx.x == 0) *out = acc;
}

// y = A v (m rows, FP64) for any row lengths: the short rows by sub-warps
// sized to their mean length, the long rows in chunks whose sums a warp per
// row adds in a fixed order, so y is the same on every run.
void a_times(psipm_handle* h, const double* v, double* y) {
    cudaStream_t st = h->stream;
    const int ns = h->n_short;
    if (ns) {
        const double mean = (double)h->short_nnz / ns;
        const int grid = (int)std::min<int64_t>(std::max<int64_t>(1, ns / 8), (int64_t)h->num_sms * 16);
        if (mean <= 3.0)
            LAUNCH(h, k_list_rows<1><<<grid, 256, 0, st>>>(ns, h->short_rows.p, h->a_ptr.p, h->a_idx.p, h->a_val.p, v, y));
        else if (mean <= 12.0)
            LAUNCH(h, k_list_rows<4><<<grid, 256, 0, st>>>(ns, h->short_rows.p, h->a_ptr.p, h->a_idx.p, h->a_val.p, v, y));
        else if (mean <= 48.0)
            LAUNCH(h, k_list_rows<8><<<grid, 256, 0, st>>>(ns, h->short_rows.p, h->a_ptr.p, h->a_idx.p, h->a_val.p, v, y));
        else
            LAUNCH(h, k_list_rows<32><<<grid, 256, 0, st>>>(ns, h->short_rows.p, h->a_ptr.p, h->a_idx.p, h->a_val.p, v, y));
    }
    if (h->n_long) {
        h->achunk.reserve(std::max(1, h->n_chunks));
        const int grid = (int)std::min<int64_t>(blocks_for((int64_t)h->n_chunks * 32, 256), (int64_t)h->num_sms * 16);
        LAUNCH(h, k_chunk_rows<<<grid, 256, 0, st>>>(h->n_chunks, h->chunk_beg.p, h->chunk_end.p, h->a_idx.p,
                                                     h->a_val.p, v, h->achunk.p));
        LAUNCH(h, k_long_rows<<<blocks_for((int64_t)h->n_long * 32, 256), 256, 0, st>>>(
                      h->n_long, h->long_rows.p, h->long_chunk_ptr.p, h->achunk.p, y));
    }
}

__global__ void k_sub(long long n, const double* __restrict__ b, const double* __restrict__ a,
                      double* __restrict__ out) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) out[i] = b[i] - a[i];
}

__global__ void k_div(long long n, const double* __restrict__ a, const double* __restrict__ b,
                      double* __restrict__ out) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[i] / b[i];
}

// dx_j = wr1_j + (sum_i A_ij dy_i) / theta_j
__global__ void k_dx(long long n, const int* __restrict__ ptr, const int* __restrict__ idx,
                     const double* __restrict__ val, const double* __restrict__ dy,
                     const double* __restrict__ wr1, const double* __restrict__ theta,
                     double* __restrict__ dx) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= n) return;
    double s = 0.0;
    for (int k = ptr[j]; k < ptr[j + 1]; ++k) s += val[k] * dy[idx[k]];
    dx[j] = wr1[j] + s / theta[j];
}

// t = w o (A^T x)  (FP64, one thread per column)
__global__ void k_at_w(long long n, const int* __restrict__ ptr, const int* __restrict__ idx,
                       const double* __restrict__ val, const double* __restrict__ w, const double* __restrict__ x,
                       double* __restrict__ t) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= n) return;
    double s = 0.0;
    for (int k = ptr[j]; k < ptr[j + 1]; ++k) s += val[k] * x[idx[k]];
    t[j] = w[j] * s;
}

// r = rhs - (A t + delta x)   (FP64, one warp per row); per-warp partials of r.r
__global__ void k_residual(long long m, const int* __restrict__ ptr, const int* __restrict__ idx,
                           const double* __restrict__ val, const double* __restrict__ t, double delta,
                           const double* __restrict__ x, const double* __restrict__ rhs, double* __restrict__ r,
                           double* __restrict__ norm2) {
    const int lane = threadIdx.x & 31;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    double acc = 0.0;
    for (long long i = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; i < m; i += warps) {
        double s = 0.0;
        for (int k = ptr[i] + lane; k < ptr[i + 1]; k += 32) s += val[k] * t[idx[k]];
        s = warp_sum(s);
        if (lane == 0) {
            const double ri = rhs[i] - (s + delta * x[i]);
            r[i] = ri;
            acc += ri * ri;
        }
    }
    acc = warp_sum(acc);
    if (lane == 0) norm2[(blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5] = acc;
}

__global__ void k_scale_narrow(long long m, const double* __restrict__ r, double s, float* __restrict__ out) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < m) out[i] = (float)(r[i] * s);
}

__global__ void k_axpy64(long long m, const double* __restrict__ d, double* __restrict__ x) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < m) x[i] += d[i];
}

__global__ void k_axpy_widen(long long m, double a, const float* __restrict__ d, double* __restrict__ x) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < m) x[i] += a * (double)d[i];
}

// r64 = rhs64 - H x64 in FP64; returns ||r64||
double fp64_residual(psipm_handle* h, const double* rhs, const double* x) {
    const int64_t m = h->m, n = h->n;
    cudaStream_t st = h->stream;
    h->t64.reserve(n);
    h->r64.reserve(m);
    h->norm64.reserve(1);
    LAUNCH(h, k_at_w<<<blocks_for(n, 256), 256, 0, st>>>(n, h->at_ptr.p, h->at_idx.p, h->at_val.p, h->w.p, x,
                                                          h->t64.p));
    const int rows = (int)std::min<int64_t>(blocks_for(m * 32, 256), 8 * std::max(1, h->num_sms));
    h->norm_part.reserve((size_t)rows * 8);
    LAUNCH(h, k_residual<<<rows, 256, 0, st>>>(m, h->a_ptr.p, h->a_idx.p, h->a_val.p, h->t64.p, h->delta, x, rhs,
                                               h->r64.p, h->norm_part.p));
    LAUNCH(h, k_fold_sum<<<1, 256, 0, st>>>((long long)rows * 8, h->norm_part.p, h->norm64.p));
    double nrm2 = 0.0;
    PSIPM_CUDA(cudaMemcpyAsync(&nrm2, h->norm64.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    PSIPM_CUDA(cudaStreamSynchronize(st));
    return std::sqrt(nrm2);
}

// Solve H x = rhs (rhs FP64 on the device) to relative residual tol.
// FP64 mode: one persistent PCG.  FP32_REFINED: iterative refinement in FP64
// around FP32 persistent PCG sweeps on the normalised residual:
//   x = 0; repeat { r = rhs - H x (FP64); stop if |r|/scale <= tol;
//                   d = PCG32(r/|r|, tol_in); x += |r| d }
// Returns the device pointer of x (FP64).
const double* solve_normal(psipm_handle* h, const double* rhs, double tol, int maxit, int variant, int replacement,
                           double gap_tol, psipm_pcg_info* info) {
    require(h->have_factor, PSIPM_ERR_STATE, "solve before a successful factor");
    if (h->precision != PSIPM_FP32_REFINED) {
        if (h->precision == PSIPM_FP32_PRECOND)
            run_pcg<double, float>(h, rhs, tol, maxit, variant, replacement, gap_tol, info);
        else
            run_pcg<double, double>(h, rhs, tol, maxit, variant, replacement, gap_tol, info);
        h->r64.reserve(h->m);
        PSIPM_CUDA(cudaMemcpyAsync(h->r64.p, h->p64.tr.p, h->m * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        return h->p64.x.p;
    }
    const int64_t m = h->m;
    cudaStream_t st = h->stream;
    h->x64.zero(m, st);
    PcgStore<float>& s32 = h->p32;
    pcg_args<float, float>(h);  // sizes the FP32 work vectors
    double rnorm = fp64_residual(h, rhs, h->x64.p);
    const double rhs_norm = rnorm;
    const double scale = variant == PSIPM_PCG_HSD ? rhs_norm : std::max(1.0, rhs_norm);
    const double target = variant == PSIPM_PCG_HSD ? std::max(tol * rhs_norm, 64.0 * 2.220446049250313e-16 * rhs_norm)
                                                   : tol * scale;
    psipm_pcg_info total;
    std::memset(&total, 0, sizeof(total));
    psipm_pcg_info first;
    std::memset(&first, 0, sizeof(first));
    int sweeps = 0;
    int last_info = 0;
    const int max_sweeps = 8;
    int budget = maxit;
    while (rnorm > target && sweeps < max_sweeps && budget > 0 && rnorm > 0.0) {
        LAUNCH(h, k_scale_narrow<<<blocks_for(m, 256), 256, 0, st>>>(m, h->r64.p, 1.0 / rnorm, s32.rhs.p));
        const double inner = std::min(0.5, std::max(1e-5, 0.5 * target / rnorm));
        psipm_pcg_info one;
        run_pcg<float, float>(h, s32.rhs.p, inner, budget, variant, replacement, gap_tol, &one);
        if (sweeps == 0) first = one;
        last_info = one.info;
        total.iterations += one.iterations;
        total.matvecs += one.matvecs + 1;
        total.replacements += one.replacements;
        total.residual_checks += one.residual_checks + 1;
        total.seconds += one.seconds;
        for (int q = 0; q < 4; ++q) total.phase_seconds[q] += one.phase_seconds[q];
        budget -= std::max(1, one.iterations);
        LAUNCH(h, k_axpy_widen<<<blocks_for(m, 256), 256, 0, st>>>(m, rnorm, s32.x.p, h->x64.p));
        const double before = rnorm;
        rnorm = fp64_residual(h, rhs, h->x64.p);
        ++sweeps;
        if (!std::isfinite(rnorm)) break;
        if (rnorm > 0.1 * before && rnorm > target) {
            // FP32 arithmetic cannot reduce this residual further (the
            // operator's rounding error is comparable to it): finish with an
            // FP64 PCG around the FP32 preconditioner, from the current x.
            psipm_pcg_info tail;
            pcg_args<double, double>(h);  // sizes the FP64 work vectors
            PSIPM_CUDA(cudaMemcpyAsync(h->p64.rhs.p, h->r64.p, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
            const double tail_tol = std::max(1e-16, std::min(0.5, target / std::max(rnorm, 1e-300)));
            run_pcg<double, float>(h, h->p64.rhs.p, tail_tol, std::max(1, budget), PSIPM_PCG_HSD, replacement,
                                   gap_tol, &tail);
            total.iterations += tail.iterations;
            total.matvecs += tail.matvecs;
            total.seconds += tail.seconds;
            for (int q = 0; q < 4; ++q) total.phase_seconds[q] += tail.phase_seconds[q];
            LAUNCH(h, k_axpy64<<<blocks_for(m, 256), 256, 0, st>>>(m, h->p64.x.p, h->x64.p));
            rnorm = fp64_residual(h, rhs, h->x64.p);
            ++sweeps;
            last_info = tail.ok ? 0 : tail.info;
            break;
        }
    }
    if (info) {
        *info = total;
        info->n_alpha = first.n_alpha;  // Lanczos data of the first (longest) sweep
        info->n_beta = first.n_beta;
        info->n_history = first.n_history;
        info->refinements = sweeps;
        info->relative_residual = scale > 0.0 ? rnorm / scale : 0.0;
        const bool converged = rnorm <= target;
        info->ok = converged ? 1 : 0;
        info->info = converged ? 0 : (last_info != 0 ? last_info : maxit);
    }
    return h->x64.p;
}

void solve_device(psipm_handle* h, const double* r1d, const double* r2d, double tol, int maxit, int variant,
                  int replacement, double gap_tol, double* dxd, psipm_pcg_info* info, const double** dy_out) {
    const int64_t m = h->m, n = h->n;
    cudaStream_t st = h->stream;
    h->wr1.reserve(n);
    h->rhs64.reserve(m);
    LAUNCH(h, k_div<<<blocks_for(n, 256), 256, 0, st>>>(n, r1d, h->theta.p, h->wr1.p));
    // rhs = r2 - A (r1 / theta)
    a_times(h, h->wr1.p, h->rhs64.p);
    LAUNCH(h, k_sub<<<blocks_for(m, 256), 256, 0, st>>>(m, r2d, h->rhs64.p, h->rhs64.p));
    const double* dy = solve_normal(h, h->rhs64.p, tol, maxit, variant, replacement, gap_tol, info);
    LAUNCH(h, k_dx<<<blocks_for(n, 256), 256, 0, st>>>(n, h->at_ptr.p, h->at_idx.p, h->at_val.p, dy, h->wr1.p,
                                                        h->theta.p, dxd));
    *dy_out = dy;
}

}  // namespace

extern "C" {

int psipm_solve(psipm_handle* h, const double* r1, const double* r2, double tol, int32_t maxit, int32_t variant,
                int32_t replacement, double gap_tolerance, double* dx, double* dy, double* residual, double* alphas,
                double* betas, double* history, psipm_pcg_info* info) {
    if (!r1 || !r2 || !dx || !dy || maxit < 0) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        require(h->have_factor, PSIPM_ERR_STATE, "solve before a successful factor");
        h->r1.upload(r1, h->n, h->stream);
        h->r2.upload(r2, h->m, h->stream);
        h->dx.reserve(h->n);
        psipm_pcg_info local;
        const double* dyd = nullptr;
        solve_device(h, h->r1.p, h->r2.p, tol, maxit, variant, replacement, gap_tolerance, h->dx.p, &local, &dyd);
        copy_out(h, dx, h->dx.p, h->n);
        copy_out(h, dy, dyd, h->m);
        if (residual) copy_out(h, residual, h->r64.p, h->m);
        copy_out(h, alphas, h->alphas.p, local.n_alpha);
        copy_out(h, betas, h->betas.p, local.n_beta);
        copy_out(h, history, h->history.p, local.n_history);
        if (info) *info = local;
    });
}

int psipm_solve_dev(psipm_handle* h, const double* r1_dev, const double* r2_dev, double tol, int32_t maxit,
                    int32_t variant, int32_t replacement, double gap_tolerance, double* dx_dev, double* dy_dev,
                    psipm_pcg_info* info) {
    if (!r1_dev || !r2_dev || !dx_dev || !dy_dev || maxit < 0) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        require(h->have_factor, PSIPM_ERR_STATE, "solve before a successful factor");
        const double* dyd = nullptr;
        solve_device(h, r1_dev, r2_dev, tol, maxit, variant, replacement, gap_tolerance, dx_dev, info, &dyd);
        PSIPM_CUDA(cudaMemcpyAsync(dy_dev, dyd, h->m * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    });
}

int64_t psipm_kernel_launches(const psipm_handle* h) { return h ? h->launches : -1; }

int psipm_debug_apply_trace(psipm_handle* h, const double* r, double* z, int64_t* stamps, int32_t cap,
                            int32_t* count, int32_t* barrier_ns) {
    if (!r || !z || !stamps || cap <= 0 || !count) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        require(h->have_factor, PSIPM_ERR_STATE, "apply before a successful factor");
        require(h->precision == PSIPM_FP64, PSIPM_ERR_UNSUPPORTED, "apply trace is FP64 only");
        PcgArgs<double, double> a = pcg_args<double, double>(h);
        DevBuf<long long> tr;
        tr.zero(cap, h->stream);
        a.pc.trace = tr.p;
        a.pc.trace_cap = cap;
        h->r1.upload(r, h->m, h->stream);
        h->r2.reserve(h->m);
        const double* in = h->r1.p;
        double* outp = h->r2.p;
        void* args[] = {&a, (void*)&in, (void*)&outp};
        launch_coop(h, (const void*)k_apply<double, double>, args);
        copy_out(h, z, h->r2.p, h->m);
        std::vector<long long> host(cap);
        PSIPM_CUDA(cudaMemcpyAsync(host.data(), tr.p, cap * sizeof(long long), cudaMemcpyDeviceToHost, h->stream));
        PSIPM_CUDA(cudaStreamSynchronize(h->stream));
        int n = 0;
        for (; n < cap && host[n] != 0; ++n) stamps[n] = host[n];
        *count = n;
        if (barrier_ns) {
            DevBuf<long long> out;
            out.zero(1, h->stream);
            int iters = 1000;
            long long* op = out.p;
            GridBarrier gb = grid_barrier(h);
            int skip = -1;
            void* bargs[] = {&iters, &op, &gb, &skip};
            prepare_barrier(h);
            PSIPM_CUDA(cudaLaunchCooperativeKernel((const void*)k_barrier_probe, dim3(h->coop_blocks),
                                                   dim3(kPcgThreads), bargs, 0, h->stream));
            ++h->launches;
            long long ns = 0;
            PSIPM_CUDA(cudaMemcpyAsync(&ns, out.p, sizeof(ns), cudaMemcpyDeviceToHost, h->stream));
            PSIPM_CUDA(cudaStreamSynchronize(h->stream));
            *barrier_ns = (int32_t)(ns / iters);
        }
    });
}

int psipm_debug_barrier_timeout(psipm_handle* h, int32_t count, int32_t polls, int32_t skip_block,
                                double* seconds) {
    if (!h || count <= 0 || polls <= 0 || !seconds) return PSIPM_ERR_ARGUMENT;
    *seconds = 0.0;
    return guarded(h, [&]() {
        require(skip_block < h->coop_blocks, PSIPM_ERR_ARGUMENT, "skip_block outside the grid");
        DevBuf<long long> out;
        out.zero(1, h->stream);
        long long* op = out.p;
        GridBarrier gb = grid_barrier(h);
        gb.polls = (unsigned int)polls;
        int skip = skip_block;
        void* bargs[] = {&count, &op, &gb, &skip};
        prepare_barrier(h);
        const auto t0 = std::chrono::steady_clock::now();
        PSIPM_CUDA(cudaLaunchCooperativeKernel((const void*)k_barrier_probe, dim3(h->coop_blocks),
                                               dim3(kPcgThreads), bargs, 0, h->stream));
        ++h->launches;
        PSIPM_CUDA(cudaStreamSynchronize(h->stream));
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    });
}

int psipm_debug_syrk_tc(int32_t device, int32_t r, int32_t k0, int32_t kb, int32_t jend, int32_t passes,
                        const float* f_in, float* f_out) {
    if (r <= 0 || k0 < 0 || kb <= 0 || k0 + kb > r || jend > r || (passes != 1 && passes != 3) || !f_in ||
        !f_out)
        return PSIPM_ERR_ARGUMENT;
    try {
        PSIPM_CUDA(cudaSetDevice(device));
        cudaStream_t st;
        PSIPM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        struct StreamGuard {
            cudaStream_t s;
            ~StreamGuard() { cudaStreamDestroy(s); }
        } guard{st};
        const size_t bytes = (size_t)r * r * sizeof(float);
        DevBuf<float> F;
        DevBuf<int> err;
        F.upload(f_in, (size_t)r * r, st);
        err.zero(1, st);
        syrk_update_tc(F.p, r, k0, kb, jend, passes, err.p, st);
        int e = 0;
        PSIPM_CUDA(cudaMemcpyAsync(f_out, F.p, bytes, cudaMemcpyDeviceToHost, st));
        PSIPM_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        PSIPM_CUDA(cudaStreamSynchronize(st));
        return e ? PSIPM_ERR_TIMEOUT : PSIPM_OK;
    } catch (const Failure& f) {
        (void)cudaGetLastError();
        return f.code;
    } catch (...) {
        return PSIPM_ERR_CUDA;
    }
}

int psipm_debug_levels(const psipm_handle* h, int64_t* out, int32_t cap, int32_t* nlevels) {
    if (!h || !out || !nlevels || cap < 0) return PSIPM_ERR_ARGUMENT;
    if (!h->have_symbolic) return PSIPM_ERR_STATE;
    const Symbolic& s = h->sym;
    *nlevels = s.nlevels;
    for (int l = 0; l < s.nlevels && l < cap; ++l) {
        int64_t* o = out + 8 * (int64_t)l;
        std::memset(o, 0, 8 * sizeof(int64_t));
        o[0] = s.level_ptr[l + 1] - s.level_ptr[l];
        for (int q = s.level_ptr[l]; q < s.level_ptr[l + 1]; ++q) {
            const int sn = s.level_sn[q];
            const int64_t c = s.sn_first[sn + 1] - s.sn_first[sn];
            const int64_t r = s.sn_rowptr[sn + 1] - s.sn_rowptr[sn];
            if (r <= kSmallRows && c <= 32) ++o[1];
            o[5] += r * c;
            o[6] += r;
            o[7] = std::max<int64_t>(o[7], r);
        }
        o[2] = o[0] - o[1];
        o[3] = h->fwd_ptr[l + 1] - h->fwd_ptr[l];
        o[4] = h->bwd_ptr[l + 1] - h->bwd_ptr[l];
    }
    return PSIPM_OK;
}

int psipm_timer_start(psipm_handle* h) {
    return guarded(h, [&]() { PSIPM_CUDA(cudaEventRecord(h->tv0, h->stream)); });
}

int psipm_timer_stop(psipm_handle* h, double* seconds) {
    if (!seconds) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        PSIPM_CUDA(cudaEventRecord(h->tv1, h->stream));
        PSIPM_CUDA(cudaEventSynchronize(h->tv1));
        float ms = 0.f;
        PSIPM_CUDA(cudaEventElapsedTime(&ms, h->tv0, h->tv1));
        *seconds = ms * 1e-3;
    });
}

int psipm_set_pcg_budget(psipm_handle* h, double seconds) {
    if (!h || !(seconds >= 0.0)) return PSIPM_ERR_ARGUMENT;
    // round up so that any positive budget stays positive; cap at ~290 years
    const double ns = std::ceil(std::min(seconds, 9.0e18 * 1e-9) * 1e9);
    h->pcg_budget_ns = (long long)ns;
    return PSIPM_OK;
}

int psipm_set_profiling(psipm_handle* h, int32_t on) {
    (void)on;
    return h ? PSIPM_OK : PSIPM_ERR_ARGUMENT;
}

}  // extern "C"

// ===========================================================================
// Device-resident PS-IPM vectors (kernels_ipm.cuh).  The inner loop of the
// reference's prox_eval (psipm_active_pool.py:1947-2271) keeps x, y, z, w, s,
// the residuals and the directions in NumPy; here they stay in HBM and the
// host only sees the scalars the loop branches on.
namespace {

constexpr int kIpmThreads = 256;

int ipm_grid(const psipm_handle* h, int64_t n) {
    return (int)std::min<int64_t>({blocks_for(n, kIpmThreads), (int64_t)std::max(1, h->num_sms) * 8,
                                   (int64_t)kIpmPartStride});
}

void ipm_require(const psipm_handle* h) {
    require(h->ipm.loaded, PSIPM_ERR_STATE, "IPM vectors used before psipm_ipm_load");
}

// y = M v with M in CSR (rows, ptr, idx, val); lanes per row from the mean row length
void spmv_csr(psipm_handle* h, int64_t rows, int64_t nnz, const int* ptr, const int* idx, const double* val,
              const double* v, double* y) {
    const double mean = rows ? (double)nnz / (double)rows : 0.0;
    const int grid = (int)std::min<int64_t>(std::max<int64_t>(1, rows / 8), (int64_t)h->num_sms * 16);
    cudaStream_t st = h->stream;
    if (mean <= 3.0)
        LAUNCH(h, k_spmv_rows<1><<<grid, kIpmThreads, 0, st>>>(rows, ptr, idx, val, v, y));
    else if (mean <= 12.0)
        LAUNCH(h, k_spmv_rows<4><<<grid, kIpmThreads, 0, st>>>(rows, ptr, idx, val, v, y));
    else if (mean <= 48.0)
        LAUNCH(h, k_spmv_rows<8><<<grid, kIpmThreads, 0, st>>>(rows, ptr, idx, val, v, y));
    else
        LAUNCH(h, k_spmv_rows<32><<<grid, kIpmThreads, 0, st>>>(rows, ptr, idx, val, v, y));
}

void ipm_reset(psipm_handle* h, int nred, int nu, unsigned long long uval) {
    if (nred)
        PSIPM_CUDA(cudaMemsetAsync(h->ipm.part.p, 0, (size_t)nred * kIpmPartStride * sizeof(double), h->stream));
    LAUNCH(h, k_ipm_reset<<<1, 32, 0, h->stream>>>(h->ipm.red.p, nred, h->ipm.redu.p, nu, uval, h->ipm.flag.p));
}

// the sums' block partials -> red[0 .. nred), in block order
void ipm_fold(psipm_handle* h, int nred) {
    LAUNCH(h, k_ipm_fold<<<1, 32, 0, h->stream>>>(nred, h->ipm.part.p, h->ipm.red.p));
}

unsigned long long bits_of(double v) {
    unsigned long long b;
    std::memcpy(&b, &v, sizeof(b));
    return b;
}

double from_bits(unsigned long long b) {
    double v;
    std::memcpy(&v, &b, sizeof(v));
    return v;
}

// A^T y into aty and A x into ax for the current iterate
void ipm_products(psipm_handle* h) {
    IpmStore& I = h->ipm;
    spmv_csr(h, h->n, h->nnz, h->at_ptr.p, h->at_idx.p, h->at_val.p, I.y.p, I.aty.p);
    a_times(h, I.x.p, I.ax.p);
}

template <typename U>
void read_back(psipm_handle* h, U* host, const U* dev, int count) {
    PSIPM_CUDA(cudaMemcpyAsync(host, dev, count * sizeof(U), cudaMemcpyDeviceToHost, h->stream));
    PSIPM_CUDA(cudaStreamSynchronize(h->stream));
}

// which: 0 iterate (x, y, z, w), 1 centre (xk, yk, zk, wk), 2 direction D, 3 corrector C
void ipm_set(IpmStore& I, int which, double*& x, double*& y, double*& z, double*& w) {
    switch (which) {
        case 0: x = I.x.p, y = I.y.p, z = I.z.p, w = I.w.p; break;
        case 1: x = I.xk.p, y = I.yk.p, z = I.zk.p, w = I.wk.p; break;
        case 2: x = I.dx.p, y = I.dy.p, z = I.dz.p, w = I.dw.p; break;
        default: x = I.dxc.p, y = I.dyc.p, z = I.dzc.p, w = I.dwc.p; break;
    }
}

}  // namespace

extern "C" {

int psipm_ipm_load(psipm_handle* h, const double* c, const double* b, const double* u, const uint8_t* pos,
                   const uint8_t* box) {
    if (!c || !b || !u || !pos || !box) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        const int64_t n = h->n, m = h->m;
        IpmStore& I = h->ipm;
        cudaStream_t st = h->stream;
        I.c.upload(c, n, st);
        I.b.upload(b, m, st);
        I.u.upload(u, n, st);
        I.pos.upload(pos, n, st);
        I.box.upload(box, n, st);
        for (DevBuf<double>* v : {&I.x, &I.z, &I.w, &I.s, &I.xk, &I.zk, &I.wk, &I.rd, &I.rmz, &I.rmw, &I.r1,
                                  &I.aty, &I.dx, &I.dz, &I.dw, &I.dxc, &I.dzc, &I.dwc, &I.wref})
            v->zero(n, st);
        for (DevBuf<double>* v : {&I.y, &I.yk, &I.rp, &I.zero_m, &I.ax, &I.dy, &I.dyc}) v->zero(m, st);
        I.red.zero(8, st);
        I.part.zero((size_t)8 * kIpmPartStride, st);
        I.redu.zero(4, st);
        I.flag.zero(1, st);
        I.loaded = true;
        I.have_ref = false;
    });
}

int psipm_ipm_put(psipm_handle* h, int32_t which, const double* x, const double* y, const double* z,
                  const double* w) {
    if (!x || !y || !z || !w || which < 0 || which > 3) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        ipm_require(h);
        double *dx, *dy, *dz, *dw;
        ipm_set(h->ipm, which, dx, dy, dz, dw);
        cudaStream_t st = h->stream;
        PSIPM_CUDA(cudaMemcpyAsync(dx, x, h->n * sizeof(double), cudaMemcpyHostToDevice, st));
        PSIPM_CUDA(cudaMemcpyAsync(dy, y, h->m * sizeof(double), cudaMemcpyHostToDevice, st));
        PSIPM_CUDA(cudaMemcpyAsync(dz, z, h->n * sizeof(double), cudaMemcpyHostToDevice, st));
        PSIPM_CUDA(cudaMemcpyAsync(dw, w, h->n * sizeof(double), cudaMemcpyHostToDevice, st));
    });
}

int psipm_ipm_get(psipm_handle* h, int32_t which, double* x, double* y, double* z, double* w) {
    if (which < 0 || which > 3) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        ipm_require(h);
        double *dx, *dy, *dz, *dw;
        ipm_set(h->ipm, which, dx, dy, dz, dw);
        copy_out(h, x, dx, h->n);
        copy_out(h, y, dy, h->m);
        copy_out(h, z, dz, h->n);
        copy_out(h, w, dw, h->n);
    });
}

int psipm_ipm_copy(psipm_handle* h, int32_t to_centre) {
    return guarded(h, [&]() {
        ipm_require(h);
        IpmStore& I = h->ipm;
        cudaStream_t st = h->stream;
        const int g = blocks_for(std::max(h->n, h->m), kIpmThreads);
        if (to_centre) {
            LAUNCH(h, k_ipm_copy<<<g, kIpmThreads, 0, st>>>(h->n, h->m, I.x.p, I.y.p, I.z.p, I.w.p, I.xk.p, I.yk.p,
                                                           I.zk.p, I.wk.p));
        } else {
            LAUNCH(h, k_ipm_copy<<<g, kIpmThreads, 0, st>>>(h->n, h->m, I.xk.p, I.yk.p, I.zk.p, I.wk.p, I.x.p, I.y.p,
                                                           I.z.p, I.w.p));
            LAUNCH(h, k_ipm_sync_box<<<blocks_for(h->n, kIpmThreads), kIpmThreads, 0, st>>>(h->n, I.x.p, I.s.p,
                                                                                             I.u.p, I.box.p));
        }
    });
}

int psipm_ipm_residuals(psipm_handle* h, double rho, double delta, double* out) {
    if (!out) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        ipm_require(h);
        IpmStore& I = h->ipm;
        cudaStream_t st = h->stream;
        const int64_t n = h->n, m = h->m;
        ipm_products(h);
        ipm_reset(h, 8, 0, 0ull);
        LAUNCH(h, k_ipm_residual_n<<<ipm_grid(h, n), kIpmThreads, 0, st>>>(
                      n, I.c.p, I.aty.p, I.x.p, I.z.p, I.w.p, I.xk.p, I.u.p, I.pos.p, rho, I.rd.p,
                      I.part.p + 1 * kIpmPartStride));
        LAUNCH(h, k_ipm_residual_m<<<ipm_grid(h, m), kIpmThreads, 0, st>>>(m, I.ax.p, I.b.p, I.y.p, I.yk.p, delta,
                                                                            I.rp.p, I.part.p + 1 * kIpmPartStride));
        LAUNCH(h, k_ipm_comp<<<ipm_grid(h, n), kIpmThreads, 0, st>>>(
                      n, I.x.p, I.s.p, I.z.p, I.w.p, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0.0, 0.0,
                      0.0, I.pos.p, I.box.p, I.part.p));
        ipm_fold(h, 6);
        read_back(h, out, I.red.p, 6);
    });
}

int psipm_ipm_theta(psipm_handle* h, double theta_min, double theta_cap, double delta) {
    return guarded(h, [&]() {
        ipm_require(h);
        IpmStore& I = h->ipm;
        h->theta.reserve(h->n);
        LAUNCH(h, k_ipm_theta<<<blocks_for(h->n, kIpmThreads), kIpmThreads, 0, h->stream>>>(
                      h->n, I.x.p, I.z.p, I.w.p, I.s.p, I.pos.p, I.box.p, theta_min, theta_cap, h->theta.p));
        h->delta = delta;
        compute_weights(h);
        h->have_theta = true;
        h->scores_valid = false;
    });
}

int psipm_ipm_targets(psipm_handle* h, int32_t kind, const double* params) {
    if (!params || kind < 0 || kind > 2) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        ipm_require(h);
        IpmStore& I = h->ipm;
        const int g = blocks_for(h->n, kIpmThreads);
        cudaStream_t st = h->stream;
        if (kind == 0)
            LAUNCH(h, k_ipm_targets<<<g, kIpmThreads, 0, st>>>(h->n, I.x.p, I.s.p, I.z.p, I.w.p, params[0], I.pos.p,
                                                              I.box.p, I.rmz.p, I.rmw.p));
        else if (kind == 1)
            LAUNCH(h, k_ipm_mehrotra<<<g, kIpmThreads, 0, st>>>(h->n, I.dx.p, I.dz.p, I.dw.p, params[0], I.pos.p,
                                                               I.box.p, I.rmz.p, I.rmw.p));
        else
            LAUNCH(h, k_ipm_gondzio<<<g, kIpmThreads, 0, st>>>(h->n, I.x.p, I.s.p, I.z.p, I.w.p, I.dx.p, I.dz.p,
                                                              I.dw.p, params[0], params[1], params[2], params[3],
                                                              params[4], I.pos.p, I.box.p, I.rmz.p, I.rmw.p));
    });
}

int psipm_ipm_newton(psipm_handle* h, int32_t corrector, double tol, int32_t maxit, int32_t variant,
                     int32_t replacement, double gap_tolerance, double* alphas, double* betas, double* history,
                     int32_t* finite, psipm_pcg_info* info) {
    if (maxit < 0 || !finite) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        ipm_require(h);
        require(h->have_factor, PSIPM_ERR_STATE, "solve before a successful factor");
        IpmStore& I = h->ipm;
        cudaStream_t st = h->stream;
        const int64_t n = h->n, m = h->m;
        double* dx = corrector ? I.dxc.p : I.dx.p;
        double* dy = corrector ? I.dyc.p : I.dy.p;
        double* dz = corrector ? I.dzc.p : I.dz.p;
        double* dw = corrector ? I.dwc.p : I.dw.p;
        LAUNCH(h, k_ipm_r1<<<blocks_for(n, kIpmThreads), kIpmThreads, 0, st>>>(
                      n, corrector ? nullptr : I.rd.p, I.rmz.p, I.rmw.p, I.x.p, I.s.p, I.pos.p, I.box.p, I.r1.p));
        psipm_pcg_info local;
        const double* dyd = nullptr;
        solve_device(h, I.r1.p, corrector ? I.zero_m.p : I.rp.p, tol, maxit, variant, replacement, gap_tolerance, dx,
                     &local, &dyd);
        PSIPM_CUDA(cudaMemcpyAsync(dy, dyd, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
        PSIPM_CUDA(cudaMemsetAsync(I.flag.p, 0, sizeof(int), st));
        LAUNCH(h, k_ipm_dual_dirs<<<blocks_for(std::max(n, m), kIpmThreads), kIpmThreads, 0, st>>>(
                      n, m, I.rmz.p, I.rmw.p, I.x.p, I.z.p, I.w.p, I.s.p, dx, dy, I.pos.p, I.box.p, dz, dw,
                      I.flag.p));
        int bad = 0;
        PSIPM_CUDA(cudaMemcpyAsync(&bad, I.flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        copy_out(h, alphas, h->alphas.p, local.n_alpha);
        copy_out(h, betas, h->betas.p, local.n_beta);
        copy_out(h, history, h->history.p, local.n_history);
        PSIPM_CUDA(cudaStreamSynchronize(st));
        *finite = bad ? 0 : 1;
        if (info) *info = local;
    });
}

int psipm_ipm_start_solve(psipm_handle* h, int32_t which, double tol, int32_t maxit, int32_t variant,
                          int32_t replacement, double gap_tolerance, double* alphas, double* betas, double* history,
                          int32_t* finite, psipm_pcg_info* info) {
    if (maxit < 0 || !finite || (which != 0 && which != 1)) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        ipm_require(h);
        require(h->have_factor, PSIPM_ERR_STATE, "solve before a successful factor");
        IpmStore& I = h->ipm;
        cudaStream_t st = h->stream;
        const int64_t n = h->n, m = h->m;
        PSIPM_CUDA(cudaMemsetAsync(I.r1.p, 0, n * sizeof(double), st));
        // which 0: r2 = b, x = A^T dy (= dx at theta = 1, r1 = 0); which 1: r2 = A c, y = dy
        if (which == 1) a_times(h, I.c.p, I.ax.p);
        psipm_pcg_info local;
        const double* dyd = nullptr;
        solve_device(h, I.r1.p, which == 0 ? I.b.p : I.ax.p, tol, maxit, variant, replacement, gap_tolerance,
                     I.dx.p, &local, &dyd);
        PSIPM_CUDA(cudaMemcpyAsync(which == 0 ? I.x.p : I.y.p, which == 0 ? I.dx.p : dyd,
                                   (which == 0 ? n : m) * sizeof(double), cudaMemcpyDeviceToDevice, st));
        PSIPM_CUDA(cudaMemsetAsync(I.flag.p, 0, sizeof(int), st));
        LAUNCH(h, k_start_finite<<<blocks_for(std::max(n, m), kIpmThreads), kIpmThreads, 0, st>>>(
                      n, m, I.dx.p, dyd, I.flag.p));
        int bad = 0;
        PSIPM_CUDA(cudaMemcpyAsync(&bad, I.flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        copy_out(h, alphas, h->alphas.p, local.n_alpha);
        copy_out(h, betas, h->betas.p, local.n_beta);
        copy_out(h, history, h->history.p, local.n_history);
        PSIPM_CUDA(cudaStreamSynchronize(st));
        *finite = bad ? 0 : 1;
        if (info) *info = local;
    });
}

int psipm_ipm_start(psipm_handle* h, int32_t solved, double* out) {
    return guarded(h, [&]() {
        ipm_require(h);
        IpmStore& I = h->ipm;
        cudaStream_t st = h->stream;
        const int64_t n = h->n, m = h->m;
        const int g = ipm_grid(h, std::max(n, m));
        DevBuf<double> part, xl, xu, r;
        part.reserve((size_t)kStartSlots * g);
        xl.reserve(n);
        xu.reserve(n);
        r.reserve(n);
        std::vector<double> hp((size_t)kStartSlots * g);
        // fold slot k of the last kernel's partials in block order
        auto fold = [&](int nslots) {
            read_back(h, hp.data(), part.p, nslots * g);
        };
        auto sum_of = [&](int k) {
            double v = 0.0;
            for (int b = 0; b < g; ++b) v += hp[(size_t)k * g + b];
            return v;
        };
        auto max_of = [&](int k) {
            double v = 0.0;
            for (int b = 0; b < g; ++b) v = std::max(v, hp[(size_t)k * g + b]);
            return v;
        };
        if (!solved) {  // factorisation or a projection failed: x = y = 0 (:4182-4187)
            PSIPM_CUDA(cudaMemsetAsync(I.x.p, 0, n * sizeof(double), st));
            PSIPM_CUDA(cudaMemsetAsync(I.y.p, 0, m * sizeof(double), st));
        }
        // non-finite x or y is replaced by zeros (:4190-4193)
        for (int pass = 0; pass < 2; ++pass) {
            LAUNCH(h, k_start_bounds<<<g, kIpmThreads, 0, st>>>(n, m, I.x.p, I.y.p, I.u.p, I.pos.p, I.box.p, xl.p,
                                                                 xu.p, part.p));
            fold(4);
            const bool xbad = max_of(0) != 0.0, ybad = max_of(3) != 0.0;
            if (!xbad && !ybad) break;
            require(pass == 0, PSIPM_ERR_BOUNDS, "starting point: zeroed x or y still not finite");
            if (xbad) PSIPM_CUDA(cudaMemsetAsync(I.x.p, 0, n * sizeof(double), st));
            if (ybad) PSIPM_CUDA(cudaMemsetAsync(I.y.p, 0, m * sizeof(double), st));
        }
        const double xinfeas = std::max(max_of(1), max_of(2));
        const double xshift1 = 1.0 + 1.5 * xinfeas;
        // dual estimate (:4200-4206)
        spmv_csr(h, n, h->nnz, h->at_ptr.p, h->at_idx.p, h->at_val.p, I.y.p, I.aty.p);
        LAUNCH(h, k_start_dual_norms<<<g, kIpmThreads, 0, st>>>(n, I.c.p, I.aty.p, r.p, part.p));
        fold(2);
        const double cnorm = std::sqrt(sum_of(0));
        int scaled = 0;
        if (cnorm > 0.0 && std::sqrt(sum_of(1)) < 0.05 * cnorm) {
            LAUNCH(h, k_start_scale<<<blocks_for(m, kIpmThreads), kIpmThreads, 0, st>>>(m, 0.95, I.y.p));
            spmv_csr(h, n, h->nnz, h->at_ptr.p, h->at_idx.p, h->at_val.p, I.y.p, I.aty.p);
            LAUNCH(h, k_start_dual_norms<<<g, kIpmThreads, 0, st>>>(n, I.c.p, I.aty.p, r.p, part.p));
            scaled = 1;
        }
        const int c_zero = cnorm == 0.0;
        LAUNCH(h, k_start_slacks<<<g, kIpmThreads, 0, st>>>(n, r.p, xshift1, c_zero, I.pos.p, I.box.p, xl.p, xu.p,
                                                             I.z.p, I.w.p, part.p));
        fold(2);
        const double zinfeas = std::max(max_of(0), max_of(1));
        const double zshift1 = c_zero ? 0.0 : 1.0 + 1.5 * zinfeas;
        LAUNCH(h, k_start_sums<<<g, kIpmThreads, 0, st>>>(n, zshift1, I.pos.p, I.box.p, xl.p, xu.p, I.z.p, I.w.p,
                                                           part.p));
        fold(6);
        const double xsum = 1.0 + sum_of(0) + sum_of(1);
        const double zsum = 1.0 + sum_of(2) + sum_of(3);
        const double mu0 = 1.0 + sum_of(4) + sum_of(5);
        double xshift2 = zsum > 0.0 ? 0.5 * mu0 / zsum : 0.0;
        double zshift2 = xsum > 0.0 ? 0.5 * mu0 / xsum : 0.0;
        if (!(std::isfinite(xshift2) && xshift2 > 0.0)) xshift2 = 0.0;
        if (!(std::isfinite(zshift2) && zshift2 > 0.0)) zshift2 = 0.0;
        LAUNCH(h, k_start_final<<<blocks_for(n, kIpmThreads), kIpmThreads, 0, st>>>(
                      n, xshift2, zshift2, I.u.p, I.pos.p, I.box.p, xl.p, xu.p, I.x.p, I.z.p, I.w.p));
        PSIPM_CUDA(cudaStreamSynchronize(st));
        if (out) {
            out[0] = xshift1;
            out[1] = zshift1;
            out[2] = xshift2;
            out[3] = zshift2;
            out[4] = scaled;
        }
    });
}

int psipm_ipm_steps(psipm_handle* h, int32_t with_corrector, double gamma, double* out) {
    if (!out) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        ipm_require(h);
        IpmStore& I = h->ipm;
        ipm_reset(h, 0, 2, bits_of(1.0));
        const bool c = with_corrector != 0;
        LAUNCH(h, k_ipm_steps<<<ipm_grid(h, h->n), kIpmThreads, 0, h->stream>>>(
                      h->n, I.x.p, I.s.p, I.z.p, I.w.p, I.dx.p, I.dz.p, I.dw.p, c ? I.dxc.p : nullptr,
                      c ? I.dzc.p : nullptr, c ? I.dwc.p : nullptr, gamma, I.pos.p, I.box.p, I.redu.p));
        unsigned long long b[2];
        read_back(h, b, I.redu.p, 2);
        out[0] = from_bits(b[0]);
        out[1] = from_bits(b[1]);
    });
}

int psipm_ipm_complementarity(psipm_handle* h, int32_t with_corrector, double gamma, double alpha_x, double alpha_z,
                              double* out) {
    if (!out) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        ipm_require(h);
        IpmStore& I = h->ipm;
        ipm_reset(h, 1, 0, 0ull);
        const bool c = with_corrector != 0;
        LAUNCH(h, k_ipm_comp<<<ipm_grid(h, h->n), kIpmThreads, 0, h->stream>>>(
                      h->n, I.x.p, I.s.p, I.z.p, I.w.p, I.dx.p, I.dz.p, I.dw.p, c ? I.dxc.p : nullptr,
                      c ? I.dzc.p : nullptr, c ? I.dwc.p : nullptr, gamma, alpha_x, alpha_z, I.pos.p, I.box.p,
                      I.part.p));
        ipm_fold(h, 1);
        read_back(h, out, I.red.p, 1);
    });
}

int psipm_ipm_accept(psipm_handle* h, double gamma) {
    return guarded(h, [&]() {
        ipm_require(h);
        IpmStore& I = h->ipm;
        LAUNCH(h, k_ipm_accept<<<blocks_for(std::max(h->n, h->m), kIpmThreads), kIpmThreads, 0, h->stream>>>(
                      h->n, h->m, I.dx.p, I.dy.p, I.dz.p, I.dw.p, I.dxc.p, I.dyc.p, I.dzc.p, I.dwc.p, gamma));
    });
}

int psipm_ipm_update(psipm_handle* h, double alpha_x, double alpha_z) {
    return guarded(h, [&]() {
        ipm_require(h);
        IpmStore& I = h->ipm;
        LAUNCH(h, k_ipm_update<<<blocks_for(std::max(h->n, h->m), kIpmThreads), kIpmThreads, 0, h->stream>>>(
                      h->n, h->m, I.x.p, I.y.p, I.z.p, I.w.p, I.s.p, I.u.p, I.box.p, I.dx.p, I.dy.p, I.dz.p, I.dw.p,
                      alpha_x, alpha_z));
    });
}

int psipm_ipm_metrics(psipm_handle* h, double* out) {
    if (!out) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        ipm_require(h);
        IpmStore& I = h->ipm;
        cudaStream_t st = h->stream;
        LAUNCH(h, k_ipm_sync_box<<<blocks_for(h->n, kIpmThreads), kIpmThreads, 0, st>>>(h->n, I.x.p, I.s.p, I.u.p,
                                                                                         I.box.p));
        ipm_products(h);
        ipm_reset(h, 4, 2, 0ull);
        LAUNCH(h, k_ipm_outer_n<<<ipm_grid(h, h->n), kIpmThreads, 0, st>>>(h->n, I.c.p, I.aty.p, I.x.p, I.z.p, I.w.p,
                                                                            I.s.p, I.u.p, I.pos.p, I.box.p, I.part.p,
                                                                            I.redu.p));
        LAUNCH(h, k_ipm_outer_m<<<ipm_grid(h, h->m), kIpmThreads, 0, st>>>(h->m, I.ax.p, I.b.p, I.y.p, I.part.p,
                                                                            I.redu.p));
        ipm_fold(h, 4);
        double sums[4];
        unsigned long long mx[2];
        PSIPM_CUDA(cudaMemcpyAsync(sums, I.red.p, sizeof(sums), cudaMemcpyDeviceToHost, st));
        read_back(h, mx, I.redu.p, 2);
        out[0] = from_bits(mx[0]);
        out[1] = from_bits(mx[1]);
        for (int q = 0; q < 4; ++q) out[2 + q] = sums[q];
    });
}

int psipm_lag_reference(psipm_handle* h) {
    return guarded(h, [&]() {
        ipm_require(h);
        require(h->have_theta, PSIPM_ERR_STATE, "lag reference before set_theta");
        PSIPM_CUDA(cudaMemcpyAsync(h->ipm.wref.p, h->w.p, h->n * sizeof(double), cudaMemcpyDeviceToDevice,
                                   h->stream));
        h->ipm.have_ref = true;
    });
}

int psipm_lag_ratio(psipm_handle* h, double* out) {
    if (!out) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        ipm_require(h);
        require(h->have_theta && h->ipm.have_ref, PSIPM_ERR_STATE, "lag ratio without a reference");
        IpmStore& I = h->ipm;
        ipm_reset(h, 0, 2, bits_of(INFINITY));
        LAUNCH(h, k_ipm_reset<<<1, 32, 0, h->stream>>>(nullptr, 0, I.redu.p, 1, 0ull, nullptr));
        LAUNCH(h, k_lag_ratio<<<ipm_grid(h, h->n), kIpmThreads, 0, h->stream>>>(h->n, h->w.p, I.wref.p, I.redu.p,
                                                                                 I.flag.p));
        unsigned long long b[2];
        int bad = 0;
        PSIPM_CUDA(cudaMemcpyAsync(&bad, I.flag.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        read_back(h, b, I.redu.p, 2);
        out[0] = bad ? INFINITY : from_bits(b[0]);
        out[1] = bad ? 0.0 : from_bits(b[1]);
    });
}

}  // extern "C"

// ===========================================================================
// MINRES fallback on the augmented system (psipm_spectral_preconditioner.py:
// 583-637): K [dx; q] = [r1; r2] with K = [diag(theta) A^T; A -delta I],
// preconditioned by diag(1/theta, P^{-1}), three refinement sweeps on the true
// residual; the direction is (dx, dy = -q).  The Krylov recurrences are
// preconditioned MINRES (Paige and Saunders, 1975): every vector lives on the
// device (n + m entries, the y part at offset n), the host keeps the scalars.
namespace {

__global__ void k_aug_finish(long long n, long long m, const double* __restrict__ theta, double delta,
                             const double* __restrict__ v, double* __restrict__ y) {
    // y holds [A^T v_y ; A v_x]; add theta o v_x and -delta v_y
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j < n) y[j] += theta[j] * v[j];
    else if (j < n + m) y[j] -= delta * v[j];
}

__global__ void k_lincomb(long long len, double a, const double* __restrict__ x, double b,
                          const double* __restrict__ y, double c, const double* __restrict__ z,
                          double* __restrict__ out) {
    // out = a x + b y + c z (y, z may be null)
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= len) return;
    double v = a * x[j];
    if (y) v += b * y[j];
    if (z) v += c * z[j];
    out[j] = v;
}

__global__ void k_dot(long long len, const double* __restrict__ x, const double* __restrict__ y,
                      double* __restrict__ out) {
    __shared__ double scratch[32];
    double acc = 0.0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < len;
         j += (long long)gridDim.x * blockDim.x)
        acc += x[j] * y[j];
    acc = block_sum(acc, scratch);
    if (threadIdx.x == 0) out[blockIdx.x] = acc;  // one partial per block
}

struct MinresState {
    psipm_handle* h;
    MinresWork& W;
    int64_t n, m, len;

    void aug_matvec(const double* v, double* out) {  // out = K v
        spmv_csr(h, n, h->nnz, h->at_ptr.p, h->at_idx.p, h->at_val.p, v + n, out);
        a_times(h, v, out + n);
        LAUNCH(h, k_aug_finish<<<blocks_for(len, kIpmThreads), kIpmThreads, 0, h->stream>>>(n, m, h->theta.p,
                                                                                               h->delta, v, out));
    }
    void precondition(const double* v, double* out) {  // out = diag(1/theta, P^-1) v
        LAUNCH(h, k_div<<<blocks_for(n, 256), 256, 0, h->stream>>>(n, v, h->theta.p, out));
        PcgArgs<double, double> a = pcg_args<double, double>(h);
        const double* in = v + n;
        double* o = out + n;
        void* args[] = {&a, (void*)&in, (void*)&o};
        launch_coop(h, (const void*)k_apply<double, double>, args);
    }
    void lincomb(double a, const double* x, double b, const double* y, double c, const double* z, double* out) {
        LAUNCH(h, k_lincomb<<<blocks_for(len, kIpmThreads), kIpmThreads, 0, h->stream>>>(len, a, x, b, y, c, z,
                                                                                           out));
    }
    double dot(const double* x, const double* y) {
        const int g = ipm_grid(h, len);
        W.dot.reserve((size_t)g + 1);
        LAUNCH(h, k_dot<<<g, kIpmThreads, 0, h->stream>>>(len, x, y, W.dot.p + 1));
        LAUNCH(h, k_fold_sum<<<1, 256, 0, h->stream>>>(g, W.dot.p + 1, W.dot.p));
        double v = 0.0;
        read_back(h, &v, W.dot.p, 1);
        return v;
    }

    // preconditioned MINRES on K x = b from x = 0; returns the stop code
    // (1, 2 converged; 6 iteration limit; -1 a preconditioner that is not
    // positive definite) and adds the iterations to *its.
    int minres(const double* b, double* x, double rtol, int maxit, int* its) {
        const double eps = 2.220446049250313e-16;
        cudaStream_t st = h->stream;
        // the rotating vectors are pointers into fixed buffers
        double *R1 = W.r1.p, *R2 = W.r2.p, *Wn = W.w.p, *W1 = W.w1.p, *W2 = W.w2.p;
        PSIPM_CUDA(cudaMemsetAsync(x, 0, len * sizeof(double), st));
        PSIPM_CUDA(cudaMemcpyAsync(R1, b, len * sizeof(double), cudaMemcpyDeviceToDevice, st));
        precondition(R1, W.y.p);
        double beta1 = dot(R1, W.y.p);
        if (beta1 < 0.0) return -1;
        if (beta1 == 0.0) return 0;
        beta1 = std::sqrt(beta1);
        PSIPM_CUDA(cudaMemcpyAsync(R2, R1, len * sizeof(double), cudaMemcpyDeviceToDevice, st));
        PSIPM_CUDA(cudaMemsetAsync(Wn, 0, len * sizeof(double), st));
        PSIPM_CUDA(cudaMemsetAsync(W2, 0, len * sizeof(double), st));
        double oldb = 0.0, beta = beta1, dbar = 0.0, epsln = 0.0, phibar = beta1, cs = -1.0, sn = 0.0;
        double tnorm2 = 0.0, ynorm2 = 0.0;
        int istop = 6;
        for (int itn = 1; itn <= maxit; ++itn) {
            ++*its;
            const double s = 1.0 / beta;
            lincomb(s, W.y.p, 0.0, nullptr, 0.0, nullptr, W.v.p);          // v = y / beta
            aug_matvec(W.v.p, W.y.p);                                      // y = K v
            if (itn >= 2) lincomb(1.0, W.y.p, -beta / oldb, R1, 0.0, nullptr, W.y.p);
            const double alfa = dot(W.v.p, W.y.p);
            lincomb(1.0, W.y.p, -alfa / beta, R2, 0.0, nullptr, W.y.p);
            std::swap(R1, R2);                                             // r1 = r2, r2 = y
            PSIPM_CUDA(cudaMemcpyAsync(R2, W.y.p, len * sizeof(double), cudaMemcpyDeviceToDevice, st));
            precondition(R2, W.y.p);
            oldb = beta;
            const double b2 = dot(R2, W.y.p);
            if (b2 < 0.0) return -1;
            beta = std::sqrt(b2);
            tnorm2 += alfa * alfa + oldb * oldb + beta * beta;
            // previous rotation, then the new one
            const double oldeps = epsln;
            const double delta = cs * dbar + sn * alfa;
            const double gbar = sn * dbar - cs * alfa;
            epsln = sn * beta;
            dbar = -cs * beta;
            const double root = std::sqrt(gbar * gbar + dbar * dbar);
            const double gamma = std::max(std::sqrt(gbar * gbar + beta * beta), eps);
            cs = gbar / gamma;
            sn = beta / gamma;
            const double phi = cs * phibar;
            phibar = sn * phibar;
            // w = (v - oldeps w1 - delta w2) / gamma with (w1, w2) = (w2, w); x += phi w
            std::swap(W1, W2);
            std::swap(W2, Wn);
            lincomb(1.0 / gamma, W.v.p, -oldeps / gamma, W1, -delta / gamma, W2, Wn);
            lincomb(1.0, x, phi, Wn, 0.0, nullptr, x);
            ynorm2 = dot(x, x);
            const double anorm = std::sqrt(tnorm2), ynorm = std::sqrt(ynorm2);
            const double test1 = phibar / std::max(anorm * ynorm, 1e-300);
            const double test2 = root / std::max(anorm, 1e-300);
            if (test2 <= rtol) istop = 2;
            if (test1 <= rtol) istop = 1;
            if (istop != 6) return istop;
        }
        return 6;
    }
};

// the reference's _minres: refinement sweeps on the true residual
void minres_solve(psipm_handle* h, const double* r1d, const double* r2d, double tol, int maxit, double fail_tol,
                  double* dxd, double* dyd, psipm_pcg_info* info) {
    const int64_t n = h->n, m = h->m, len = n + m;
    MinresWork& W = h->minres;
    for (DevBuf<double>* b : {&W.x, &W.rhs, &W.cr, &W.corr, &W.r1, &W.r2, &W.y, &W.v, &W.w, &W.w1, &W.w2, &W.t})
        b->reserve(len);
    W.dot.reserve(1);
    MinresState S{h, W, n, m, len};
    cudaStream_t st = h->stream;
    PSIPM_CUDA(cudaMemcpyAsync(W.rhs.p, r1d, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    PSIPM_CUDA(cudaMemcpyAsync(W.rhs.p + n, r2d, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
    PSIPM_CUDA(cudaMemsetAsync(W.x.p, 0, len * sizeof(double), st));
    const double scale = std::max(1.0, std::sqrt(S.dot(W.rhs.p, W.rhs.p)));
    const double target = std::max(2.0 * tol, fail_tol);
    const double rtol = std::max(2.220446049250313e-16, std::min(tol, 1e-8));
    int its = 0, code = maxit, stop = 0;
    double rel = 0.0;
    for (int sweep = 0; sweep < 3; ++sweep) {
        S.aug_matvec(W.x.p, W.t.p);
        S.lincomb(1.0, W.rhs.p, -1.0, W.t.p, 0.0, nullptr, W.cr.p);
        rel = std::sqrt(S.dot(W.cr.p, W.cr.p)) / scale;
        if (std::isfinite(rel) && rel <= target) {
            code = 0;
            break;
        }
        stop = S.minres(W.cr.p, W.corr.p, rtol, maxit, &its);
        S.lincomb(1.0, W.x.p, 1.0, W.corr.p, 0.0, nullptr, W.x.p);
        code = stop < 0 ? -1 : (stop == 6 ? maxit : 0);
        if (stop < 0) break;
    }
    S.aug_matvec(W.x.p, W.t.p);
    S.lincomb(1.0, W.rhs.p, -1.0, W.t.p, 0.0, nullptr, W.cr.p);
    rel = std::sqrt(S.dot(W.cr.p, W.cr.p)) / scale;
    const bool accepted = std::isfinite(rel) && rel <= target;
    PSIPM_CUDA(cudaMemcpyAsync(dxd, W.x.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    LAUNCH(h, k_lincomb<<<blocks_for(m, kIpmThreads), kIpmThreads, 0, st>>>(m, -1.0, W.x.p + n, 0.0, nullptr, 0.0,
                                                                            nullptr, dyd));
    if (info) {
        std::memset(info, 0, sizeof(*info));
        info->iterations = its;
        info->info = accepted ? 0 : code;
        info->ok = accepted ? 1 : 0;
        info->relative_residual = rel;
    }
}

}  // namespace

extern "C" {

int psipm_minres(psipm_handle* h, const double* r1, const double* r2, double tol, int32_t maxit, double fail_tol,
                 double* dx, double* dy, psipm_pcg_info* info) {
    if (!r1 || !r2 || !dx || !dy || maxit <= 0) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        require(h->have_factor, PSIPM_ERR_STATE, "minres before a successful factor");
        require(h->precision == PSIPM_FP64, PSIPM_ERR_UNSUPPORTED, "the MINRES fallback is FP64 only");
        h->r1.upload(r1, h->n, h->stream);
        h->r2.upload(r2, h->m, h->stream);
        h->dx.reserve(h->n);
        h->dy.reserve(h->m);
        minres_solve(h, h->r1.p, h->r2.p, tol, maxit, fail_tol, h->dx.p, h->dy.p, info);
        copy_out(h, dx, h->dx.p, h->n);
        copy_out(h, dy, h->dy.p, h->m);
    });
}

int psipm_ipm_minres(psipm_handle* h, int32_t corrector, double tol, int32_t maxit, double fail_tol, int32_t* finite,
                     psipm_pcg_info* info) {
    if (maxit <= 0 || !finite) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        ipm_require(h);
        require(h->have_factor, PSIPM_ERR_STATE, "minres before a successful factor");
        require(h->precision == PSIPM_FP64, PSIPM_ERR_UNSUPPORTED, "the MINRES fallback is FP64 only");
        IpmStore& I = h->ipm;
        cudaStream_t st = h->stream;
        const int64_t n = h->n, m = h->m;
        double* dx = corrector ? I.dxc.p : I.dx.p;
        double* dy = corrector ? I.dyc.p : I.dy.p;
        double* dz = corrector ? I.dzc.p : I.dz.p;
        double* dw = corrector ? I.dwc.p : I.dw.p;
        // r1 as the preceding psipm_ipm_newton built it
        LAUNCH(h, k_ipm_r1<<<blocks_for(n, kIpmThreads), kIpmThreads, 0, st>>>(
                      n, corrector ? nullptr : I.rd.p, I.rmz.p, I.rmw.p, I.x.p, I.s.p, I.pos.p, I.box.p, I.r1.p));
        minres_solve(h, I.r1.p, corrector ? I.zero_m.p : I.rp.p, tol, maxit, fail_tol, dx, dy, info);
        PSIPM_CUDA(cudaMemsetAsync(I.flag.p, 0, sizeof(int), st));
        LAUNCH(h, k_ipm_dual_dirs<<<blocks_for(std::max(n, m), kIpmThreads), kIpmThreads, 0, st>>>(
                      n, m, I.rmz.p, I.rmw.p, I.x.p, I.z.p, I.w.p, I.s.p, dx, dy, I.pos.p, I.box.p, dz, dw,
                      I.flag.p));
        int bad = 0;
        read_back(h, &bad, I.flag.p, 1);
        *finite = bad ? 0 : 1;
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Learned active-column selector (kernels_mlp.cuh)
extern "C" {

int psipm_mlp_forward_dev(int64_t count, const float* x, const uint16_t* w, const float* b, float* out,
                          void* stream) {
    if (count < 0 || (count && (!x || !out)) || !w || !b) return PSIPM_ERR_ARGUMENT;
    if (count == 0) return PSIPM_OK;
    if ((count + 255) / 256 > 0x7fffffffLL) return PSIPM_ERR_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int grid = (int)((count + 255) / 256);
    k_mlp_forward<<<grid, 256, 0, st>>>(count, x, reinterpret_cast<const __nv_bfloat16*>(w), b, out);
    return cudaGetLastError() == cudaSuccess ? PSIPM_OK : PSIPM_ERR_CUDA;
}

int psipm_mlp_grad_dev(int64_t count, const float* x, const float* y, float c0, float c1, const uint16_t* w,
                       const float* b, int32_t blocks, float* part, float* loss_part, float scale, float* grad,
                       float* loss, void* stream) {
    if (count <= 0 || !x || !y || !w || !b || blocks <= 0 || !part || !loss_part || !grad || !loss)
        return PSIPM_ERR_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMlpGradSmem) !=
        cudaSuccess)
        return PSIPM_ERR_CUDA;
    k_mlp_grad<<<blocks, kMlpTile, kMlpGradSmem, st>>>(count, x, y, c0, c1,
                                                       reinterpret_cast<const __nv_bfloat16*>(w), b, part,
                                                       loss_part);
    k_mlp_reduce<<<(kMlpParams + 255) / 256, 256, 0, st>>>(blocks, part, loss_part, scale, grad, loss);
    return cudaGetLastError() == cudaSuccess ? PSIPM_OK : PSIPM_ERR_CUDA;
}

int psipm_mlp_adam_dev(float* master, float* m1, float* m2, const float* grad, float lr, float beta1, float beta2,
                       float eps, int32_t step, float decay, uint16_t* w, float* b, void* stream) {
    if (!master || !m1 || !m2 || !grad || !w || !b || step <= 0) return PSIPM_ERR_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float bc1 = 1.0f - std::pow(beta1, (float)step), bc2 = 1.0f - std::pow(beta2, (float)step);
    k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(master, m1, m2, grad, lr, beta1, beta2, eps, bc1, bc2,
                                                         decay, reinterpret_cast<__nv_bfloat16*>(w), b);
    return cudaGetLastError() == cudaSuccess ? PSIPM_OK : PSIPM_ERR_CUDA;
}

int psipm_get_theta(psipm_handle* h, double* theta) {
    if (!theta) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        require(h->have_theta, PSIPM_ERR_STATE, "no weights yet");
        copy_out(h, theta, h->theta.p, h->n);
    });
}

int psipm_mlp_features(psipm_handle* h, double mu, float* x) {
    if (!x) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        require(h->scores_valid, PSIPM_ERR_STATE, "features before scores");
        const int64_t nc = (int64_t)h->cand.size();
        if (!nc) return;
        DevBuf<float> xd;
        xd.reserve(nc * kMlpIn);
        const unsigned char* flags = (h->core_flags.p && h->core_flags.n >= (size_t)nc) ? h->core_flags.p : nullptr;
        LAUNCH(h, k_mlp_features<<<blocks_for(nc, 256), 256, 0, h->stream>>>(
                      nc, h->d_cand.p, h->at_ptr.p, h->at_val.p, h->theta.p, h->scores.p, flags, mu, xd.p));
        PSIPM_CUDA(cudaMemcpyAsync(x, xd.p, nc * kMlpIn * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        PSIPM_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int psipm_mlp_scores(psipm_handle* h, const uint16_t* w, const float* b, double mu, int64_t keep,
                     double* shift_vote) {
    if (!w || !b) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        require(h->scores_valid, PSIPM_ERR_STATE, "learned scores before the rule's scores");
        const int64_t nc = (int64_t)h->cand.size();
        if (!nc) return;
        cudaStream_t st = h->stream;
        DevBuf<float> xd, out, bd;
        DevBuf<uint16_t> wd;
        xd.reserve(nc * kMlpIn);
        out.reserve(nc * kMlpOut);
        wd.upload(w, kMlpWeights, st);
        bd.upload(b, kMlpBiases, st);
        const unsigned char* flags = (h->core_flags.p && h->core_flags.n >= (size_t)nc) ? h->core_flags.p : nullptr;
        LAUNCH(h, k_mlp_features<<<blocks_for(nc, 256), 256, 0, st>>>(nc, h->d_cand.p, h->at_ptr.p, h->at_val.p,
                                                                       h->theta.p, h->scores.p, flags, mu, xd.p));
        const int grid = (int)((nc + 255) / 256);
        LAUNCH(h, k_mlp_forward<<<grid, 256, 0, st>>>(nc, xd.p, reinterpret_cast<const __nv_bfloat16*>(wd.p), bd.p,
                                                      out.p));
        // keep > 0: only the rule's `keep` best candidates stay eligible (the others
        // become -inf, which no selection takes); the network orders them
        const unsigned char* allow = nullptr;
        DevBuf<unsigned char> top;
        if (keep > 0 && keep < nc) {
            top.zero(nc, st);
            select_top(h, h->scores.p, nullptr, nc, keep, top.p);
            allow = top.p;
        }
        LAUNCH(h, k_mlp_take_scores<<<blocks_for(nc, 256), 256, 0, st>>>(nc, out.p, allow, h->scores.p));
        std::vector<float> o(2 * nc);
        PSIPM_CUDA(cudaMemcpyAsync(o.data(), out.p, 2 * nc * sizeof(float), cudaMemcpyDeviceToHost, st));
        PSIPM_CUDA(cudaStreamSynchronize(st));
        if (shift_vote) {
            double v = 0.0;
            for (int64_t c = 0; c < nc; ++c) v += o[2 * c + 1];
            *shift_vote = v / (double)nc;
        }
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// HSD pricing over all columns (psipm_v3_1_hsd.py:2101-2158)
extern "C" {

int psipm_price_load(psipm_handle* h, const double* c) {
    if (!c) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        h->price_c.upload(c, h->n, h->stream);
        h->have_price_c = true;
    });
}

int psipm_price(psipm_handle* h, const double* y, double tau, const uint8_t* active, double threshold,
                int64_t batch, double* violation, int64_t* candidates, int64_t* ncandidates) {
    if (!y || !active || batch < 0 || !candidates || !ncandidates) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        require(h->have_price_c, PSIPM_ERR_STATE, "pricing before psipm_price_load");
        const int64_t n = h->n;
        cudaStream_t st = h->stream;
        h->price_y.upload(y, h->m, st);
        h->price_active.upload(active, n, st);
        h->price_v.reserve(std::max<int64_t>(1, n));
        h->price_elig.reserve(std::max<int64_t>(1, n));
        h->price_pick.zero(std::max<int64_t>(1, n), st);
        if (n)
            LAUNCH(h, k_price<<<blocks_for(n, 256), 256, 0, st>>>(n, h->at_ptr.p, h->at_idx.p, h->at_val.p,
                                                                   h->price_y.p, h->price_c.p, tau,
                                                                   h->price_active.p, threshold, h->price_v.p,
                                                                   h->price_elig.p));
        // eligible columns, the `batch` largest violations among them (index rule on ties)
        select_top(h, h->price_v.p, h->price_elig.p, n, batch, h->price_pick.p);
        std::vector<unsigned char> pick = download_flags(h, h->price_pick.p, n);
        int64_t k = 0;
        for (int64_t j = 0; j < n; ++j)
            if (pick[j]) candidates[k++] = j;
        *ncandidates = k;
        copy_out(h, violation, h->price_v.p, n);
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Network tree-plus-diagonal preconditioner (psipm_v3_1_hsd.py:715-785)
extern "C" {

int psipm_set_tree(psipm_handle* h, const int32_t* parent, const int32_t* depth, const int32_t* tree_child) {
    if (!parent || !depth || !tree_child) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        const int64_t m = h->m, n = h->n;
        require(h->precision == PSIPM_FP64, PSIPM_ERR_UNSUPPORTED, "the tree preconditioner is FP64 only");
        int maxd = 0;
        for (int64_t i = 0; i < m; ++i) {
            require(depth[i] >= 0 && depth[i] < m, PSIPM_ERR_ARGUMENT, "depth out of range");
            require(parent[i] >= -1 && parent[i] < m, PSIPM_ERR_ARGUMENT, "parent out of range");
            require((parent[i] < 0) == (depth[i] == 0), PSIPM_ERR_ARGUMENT, "roots are the nodes at depth 0");
            if (parent[i] >= 0)
                require(depth[parent[i]] == depth[i] - 1, PSIPM_ERR_ARGUMENT, "a parent is one level up");
            maxd = std::max(maxd, (int)depth[i]);
        }
        // every column: exactly two entries; its first and second row
        std::vector<int> first(n), second(n);
        for (int64_t j = 0; j < n; ++j) {
            require(h->colptr[j + 1] - h->colptr[j] == 2, PSIPM_ERR_ARGUMENT,
                    "the tree preconditioner needs exactly two entries per column");
            first[j] = h->rowidx[h->colptr[j]];
            second[j] = h->rowidx[h->colptr[j] + 1];
            const int c = tree_child[j];
            require(c == -1 || ((c == first[j] || c == second[j]) && parent[c] == (c == first[j] ? second[j] : first[j])),
                    PSIPM_ERR_ARGUMENT, "tree_child must name the arc's child end in the forest");
        }
        const int L = maxd + 1;
        // nodes by level (ascending within a level), children lists, arc lists
        std::vector<int> lptr(L + 1, 0), lnodes(m), kptr(m + 1, 0), kids;
        for (int64_t i = 0; i < m; ++i) ++lptr[depth[i] + 1];
        for (int l = 0; l < L; ++l) lptr[l + 1] += lptr[l];
        {
            std::vector<int> f(lptr.begin(), lptr.end() - 1);
            for (int64_t i = 0; i < m; ++i) lnodes[f[depth[i]]++] = (int)i;
        }
        for (int64_t i = 0; i < m; ++i)
            if (parent[i] >= 0) ++kptr[parent[i] + 1];
        for (int64_t i = 0; i < m; ++i) kptr[i + 1] += kptr[i];
        kids.resize(kptr[m]);
        {
            std::vector<int> f(kptr.begin(), kptr.end() - 1);
            for (int64_t i = 0; i < m; ++i)
                if (parent[i] >= 0) kids[f[parent[i]]++] = (int)i;
        }
        auto lists = [&](const std::vector<int>& key, std::vector<int>& ptr, std::vector<int>& col) {
            ptr.assign(m + 1, 0);
            for (int64_t j = 0; j < n; ++j)
                if (key[j] >= 0) ++ptr[key[j] + 1];
            for (int64_t i = 0; i < m; ++i) ptr[i + 1] += ptr[i];
            col.resize(ptr[m]);
            std::vector<int> f(ptr.begin(), ptr.end() - 1);
            for (int64_t j = 0; j < n; ++j)
                if (key[j] >= 0) col[f[key[j]]++] = (int)j;
        };
        std::vector<int> fptr, fcol, sptr, scol, cptr, ccol, tc(tree_child, tree_child + n);
        lists(first, fptr, fcol);
        lists(second, sptr, scol);
        lists(tc, cptr, ccol);
        cudaStream_t st = h->stream;
        h->t_level_ptr.upload(lptr, st);
        h->t_level_nodes.upload(lnodes, st);
        std::vector<int> par(parent, parent + m);
        h->t_parent.upload(par, st);
        h->t_kid_ptr.upload(kptr, st);
        h->t_kids.upload(kids.empty() ? std::vector<int>{0} : kids, st);
        h->t_fptr.upload(fptr, st);
        h->t_fcol.upload(fcol, st);
        h->t_sptr.upload(sptr, st);
        h->t_scol.upload(scol, st);
        h->t_cptr.upload(cptr, st);
        h->t_ccol.upload(ccol.empty() ? std::vector<int>{0} : ccol, st);
        for (DevBuf<double>* v : {&h->t_diag, &h->t_tw, &h->t_piv, &h->t_mult, &h->t_pivot, &h->t_val})
            v->reserve(std::max<int64_t>(1, m));
        h->t_D.reserve(std::max<int64_t>(1, n));
        h->t_level_ptr_host = lptr;
        h->t_level_nodes_host = lnodes;
        h->tree_levels = L;
        h->tree_mode = true;
        h->tree_ready = false;
        h->have_factor = false;
        PSIPM_CUDA(cudaStreamSynchronize(st));
    });
}

int psipm_tree_factor(psipm_handle* h, const double* weights, double delta) {
    if (!weights) return PSIPM_ERR_ARGUMENT;
    return guarded(h, [&]() {
        require(h->tree_mode, PSIPM_ERR_STATE, "tree factor before psipm_set_tree");
        const int m = (int)h->m;
        cudaStream_t st = h->stream;
        h->t_D.upload(weights, h->n, st);
        LAUNCH(h, k_tree_diag<<<blocks_for(m, 256), 256, 0, st>>>(m, delta, h->t_fptr.p, h->t_fcol.p, h->t_sptr.p,
                                                                   h->t_scol.p, h->t_cptr.p, h->t_ccol.p, h->t_D.p,
                                                                   h->t_diag.p, h->t_tw.p));
        for (int l = h->tree_levels - 1; l >= 0; --l) {
            const int beg = h->t_level_ptr_host[l], cnt = h->t_level_ptr_host[l + 1] - beg;
            if (cnt)
                LAUNCH(h, k_tree_pivots<<<blocks_for(cnt, 256), 256, 0, st>>>(
                              cnt, h->t_level_nodes.p + beg, l > 0, h->t_kid_ptr.p, h->t_kids.p, h->t_diag.p,
                              h->t_tw.p, h->t_piv.p, h->t_mult.p));
        }
        const double floor = std::max(delta * 1.0e-8, 2.2250738585072014e-308);
        LAUNCH(h, k_tree_floor<<<blocks_for(m, 256), 256, 0, st>>>(m, floor, h->t_piv.p, h->t_pivot.p));
        h->tree_ready = true;
        h->have_factor = true;
    });
}

int psipm_tree_get(psipm_handle* h, double* pivot, double* multiplier) {
    return guarded(h, [&]() {
        require(h->tree_ready, PSIPM_ERR_STATE, "no tree factor");
        copy_out(h, pivot, h->t_pivot.p, h->m);
        copy_out(h, multiplier, h->t_mult.p, h->m);
    });
}

}  // extern "C"
