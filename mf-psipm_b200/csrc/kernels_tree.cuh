// Tree-plus-diagonal preconditioner for network LPs (V3.1 TreePreconditioner,
// psipm_v3_1_hsd.py:715-785).
//
// The incidence graph's BFS spanning forest (parent, depth) is fixed per LP.
// For the active arcs with weights D the preconditioner is the exact LDL'
// factor of  diag(delta + sum of D over the arcs at each node) with the
// off-diagonal entries of the tree arcs only:
//   factor (levels bottom-up): piv_p = diag_p - sum_{children c} e_c^2 / max(piv_c, tiny)
//                               mult_c = -e_c / max(piv_c, tiny),   e_c = D summed over the tree arcs into c
//                               pivot  = max(piv, max(delta 1e-8, tiny))
//   solve  (levels bottom-up): v_p += -mult_c v_c over the children c
//           v /= pivot
//          (levels top-down):  v_c -= mult_c v_parent(c)
// The reference scatters into parents with np.add.at in ascending node
// order; here every parent gathers its children in ascending order, with the
// same operations and no contraction, so both the factor and a solve are
// bit-identical to the reference.  The node lists per level, the children
// lists and the arc lists per node are built once on the host.
#pragma once

#include "common.cuh"

namespace psipm {

struct TreeLayout {
    int m = 0;
    int nlevels = 0;                   // max depth + 1
    const int* level_ptr = nullptr;    // nlevels + 1 offsets into level_nodes
    const int* level_nodes = nullptr;  // nodes by depth, ascending within a level
    const int* parent = nullptr;       // -1 at roots
    const int* kid_ptr = nullptr;      // m + 1: children of each node, ascending
    const int* kids = nullptr;
    const double* mult = nullptr;
    const double* pivot = nullptr;
    double* val = nullptr;             // m: work vector of the solve
};

// diag_i = (delta + sum_{arcs a, first(a) = i} D_a) + sum_{arcs a, second(a) = i} D_a,
// tw_i = sum_{tree arcs a into i} D_a (each sum sequential, ascending arc order)
__global__ void k_tree_diag(int m, double delta, const int* __restrict__ fptr, const int* __restrict__ fcol,
                            const int* __restrict__ sptr, const int* __restrict__ scol,
                            const int* __restrict__ cptr, const int* __restrict__ ccol,
                            const double* __restrict__ D, double* __restrict__ diag, double* __restrict__ tw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    double b1 = 0.0, b2 = 0.0, e = 0.0;
    for (int k = fptr[i]; k < fptr[i + 1]; ++k) b1 = __dadd_rn(b1, D[fcol[k]]);
    for (int k = sptr[i]; k < sptr[i + 1]; ++k) b2 = __dadd_rn(b2, D[scol[k]]);
    for (int k = cptr[i]; k < cptr[i + 1]; ++k) e = __dadd_rn(e, D[ccol[k]]);
    diag[i] = __dadd_rn(__dadd_rn(delta, b1), b2);
    tw[i] = e;
}

// one level of the factor: the level's pivots from their children, and (below
// the roots) their multipliers
__global__ void k_tree_pivots(int count, const int* __restrict__ nodes, int with_mult,
                              const int* __restrict__ kid_ptr, const int* __restrict__ kids,
                              const double* __restrict__ diag, const double* __restrict__ tw,
                              double* __restrict__ piv, double* __restrict__ mult) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    const double tiny = 2.2250738585072014e-308;
    const int p = nodes[q];
    double v = diag[p];
    for (int k = kid_ptr[p]; k < kid_ptr[p + 1]; ++k) {
        const int c = kids[k];
        const double e = tw[c];
        v = __dadd_rn(v, __ddiv_rn(-__dmul_rn(e, e), fmax(piv[c], tiny)));
    }
    piv[p] = v;
    mult[p] = with_mult ? __ddiv_rn(-tw[p], fmax(v, tiny)) : 0.0;
}

__global__ void k_tree_floor(int m, double floor, const double* __restrict__ piv, double* __restrict__ pivot) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) pivot[i] = fmax(piv[i], floor);
}

}  // namespace psipm
