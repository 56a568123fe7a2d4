// Host-side symbolic analysis of the active-core normal matrix
//     P = A_C diag(w_C) A_C^T + diag(drop) + delta I      (m x m, SPD)
// for the supernodal multifrontal Cholesky that runs on the GPU.
//
// The reference factors P with CHOLMOD (psipm_active_pool.py:839-897 via
// psipm_stable_preconditioner.py:373-395); its symbolic analysis is redone
// whenever the pattern of P changes.  Here the same event (a new core) runs
// this analysis:
//   1. pattern of P from the core columns of A,
//   2. fill-reducing ordering: approximate minimum degree (default) or
//      nested dissection by BFS level-structure separators,
//   3. elimination tree, postorder, column counts (row-subtree method),
//   4. fundamental supernodes + relaxed amalgamation,
//   5. supernode row structures, extend-add maps, a height-level schedule,
//   6. the expanded product: for every stored entry of L's pattern that P
//      touches, the list of (core column, a_ik * a_jk) contributions.
#pragma once

#include <cstdint>
#include <vector>

namespace psipm {

struct Symbolic {
    int32_t m = 0;
    std::vector<int32_t> perm;   // perm[new] = old row index
    std::vector<int32_t> iperm;  // iperm[old] = new

    // supernodes (in permuted column order, postordered)
    int32_t ns = 0;
    std::vector<int32_t> sn_first;   // ns+1: first column of each supernode
    std::vector<int64_t> sn_rowptr;  // ns+1: offsets into sn_rows
    std::vector<int32_t> sn_rows;    // permuted row indices; first c_s are the columns
    std::vector<int32_t> sn_parent;  // -1 for roots
    std::vector<int32_t> sn_level;   // height: 0 for leaves
    int32_t nlevels = 0;
    std::vector<int32_t> level_ptr;  // nlevels+1 offsets into level_sn
    std::vector<int32_t> level_sn;   // supernodes grouped by level (ascending)

    // storage offsets (in scalars)
    std::vector<int64_t> panel_off;   // ns+1: G panel r_s x c_s (row-major)
    std::vector<int64_t> update_off;  // ns+1: update matrix (r_s-c_s)^2 (column-major)
    std::vector<int64_t> uvec_off;    // ns+1: update vector (r_s-c_s)

    // children (CSR over supernodes, in ascending order)
    std::vector<int32_t> child_ptr;   // ns+1
    std::vector<int32_t> child_list;
    // relative index of each below-row of a supernode in its parent's row list
    // (indexed like uvec_off)
    std::vector<int32_t> relind;

    // expanded product for assembling P in factor order
    // entries sorted by (supernode, column, row position)
    int64_t nentries = 0;
    std::vector<int32_t> ent_sn;       // supernode of the entry's column
    std::vector<int32_t> ent_col;      // local column within the supernode
    std::vector<int32_t> ent_rowpos;   // position of the row within the supernode rows
    std::vector<int64_t> ent_ptr;      // nentries+1 into contrib
    std::vector<int32_t> contrib_col;  // core-local column index k (0..ncore-1)
    std::vector<double> contrib_val;   // a_ik * a_jk
    std::vector<int64_t> sn_entptr;    // ns+1 into entries
    std::vector<int64_t> diag_entry;   // m: entry index of the diagonal of permuted row i

    // statistics
    int64_t nnz_L = 0;        // stored entries of the supernodal L (incl. explicit zeros)
    int64_t panel_total = 0;  // sum r_s c_s
    int64_t update_total = 0; // sum (r_s-c_s)^2
    int64_t uvec_total = 0;   // sum (r_s-c_s)
    int32_t max_front = 0;    // max r_s
    int32_t max_cols = 0;     // max c_s
    double flops = 0.0;       // numeric factorisation flops (approx.)
};

struct SymbolicOptions {
    int32_t leaf_size = 64;        // nested-dissection leaf size
    int32_t relax_small = 4;       // always merge supernodes up to this many columns
    int32_t relax_medium = 16;     // merge up to this many columns if zeros <= 80%
    int32_t relax_large = 48;      // merge up to this many columns if zeros <= 10%
    int32_t ordering = 0;          // 0 approximate minimum degree, 1 natural, 2 nested dissection
};

// Build the symbolic factor for the core columns `core` (sorted, global
// column indices) of A given in CSC (colptr[n+1], rowidx[nnz], val[nnz]).
// Returns 0 on success, a negative value on invalid input (-14: a host
// allocation failed).  Analyses with more than 2^18 expanded-product keys build
// the expanded product on up to 8 host threads; the result does not depend on
// the thread count.
int build_symbolic(int32_t m, int64_t n, const int64_t* colptr, const int32_t* rowidx,
                   const double* val, const int64_t* core, int64_t ncore,
                   const SymbolicOptions& opt, Symbolic& out);

}  // namespace psipm
