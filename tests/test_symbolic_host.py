"""The host symbolic analysis (mf-psipm_b200/csrc/symbolic.cpp), without a GPU.

A small C++ driver built here against symbolic.cpp runs ``build_symbolic`` on
the cores the reference chose for the golden fixtures and writes every array
of the result.  Checks, for each core:

* the ordering is a permutation and ``iperm`` its inverse;
* the supernodes partition the columns, each supernode's row list starts with
  its own columns and continues with sorted rows below them;
* the supernodal tree is postordered (parent after child) and the levels are
  heights (0 at leaves, 1 + the highest child);
* every below-row of a supernode appears in its parent's row list at the
  recorded relative index (the extend-add map);
* the supernodal structure contains the structural Cholesky factor of
  ``P = A_C A_C' + D`` in the chosen order (computed here by symbolic
  elimination);
* the expanded product assembles ``A_C diag(w) A_C'`` exactly (lower triangle,
  permuted) for random weights, and every diagonal has an entry.
"""

import os
import shutil
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import ROOT

DRIVER = r'''
#include <cstdio>
#include <cstdint>
#include <vector>
#include "symbolic.h"
using namespace psipm;
template <typename T> std::vector<T> rd(FILE* f) {
    int64_t n = 0; if (fread(&n, 8, 1, f) != 1) return {};
    std::vector<T> v(n); if (n && fread(v.data(), sizeof(T), n, f) != (size_t)n) v.clear(); return v;
}
template <typename T> void wr(FILE* f, const std::vector<T>& v) {
    int64_t n = (int64_t)v.size(); fwrite(&n, 8, 1, f); if (n) fwrite(v.data(), sizeof(T), n, f);
}
int main(int argc, char** argv) {
    FILE* in = fopen(argv[1], "rb");
    auto mv = rd<int64_t>(in); auto colptr = rd<int64_t>(in); auto rowidx = rd<int32_t>(in);
    auto val = rd<double>(in); auto core = rd<int64_t>(in);
    fclose(in);
    Symbolic S; SymbolicOptions opt; opt.ordering = (int)mv[1];
    int rc = build_symbolic((int32_t)mv[0], (int64_t)colptr.size() - 1, colptr.data(), rowidx.data(), val.data(),
                            core.data(), (int64_t)core.size(), opt, S);
    FILE* out = fopen(argv[2], "wb");
    wr(out, std::vector<int64_t>{rc, S.ns, S.nlevels, S.nnz_L});
    wr(out, S.perm); wr(out, S.iperm); wr(out, S.sn_first); wr(out, S.sn_rowptr); wr(out, S.sn_rows);
    wr(out, S.sn_parent); wr(out, S.sn_level); wr(out, S.uvec_off); wr(out, S.relind);
    wr(out, S.ent_sn); wr(out, S.ent_col); wr(out, S.ent_rowpos); wr(out, S.ent_ptr); wr(out, S.contrib_col);
    wr(out, S.contrib_val); wr(out, S.diag_entry);
    fclose(out);
    return rc == 0 ? 0 : 1;
}
'''

FIELDS = [("head", np.int64), ("perm", np.int32), ("iperm", np.int32), ("sn_first", np.int32),
          ("sn_rowptr", np.int64), ("sn_rows", np.int32), ("sn_parent", np.int32), ("sn_level", np.int32),
          ("uvec_off", np.int64), ("relind", np.int32), ("ent_sn", np.int32), ("ent_col", np.int32),
          ("ent_rowpos", np.int32), ("ent_ptr", np.int64), ("contrib_col", np.int32), ("contrib_val", np.float64),
          ("diag_entry", np.int64)]


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("symbolic")
    src = d / "driver.cpp"
    src.write_text(DRIVER)
    exe = d / "driver"
    csrc = os.path.join(ROOT, "mf-psipm_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", csrc, str(src), os.path.join(csrc, "symbolic.cpp"), "-o",
                    str(exe)], check=True)
    return d, exe


def run_symbolic(driver, A, core, ordering=0):
    d, exe = driver
    inp, out = d / "in.bin", d / "out.bin"
    with open(inp, "wb") as f:
        for arr, dt in ((np.array([A.shape[0], ordering]), np.int64), (A.indptr, np.int64),
                        (A.indices, np.int32), (A.data, np.float64), (core, np.int64)):
            a = np.ascontiguousarray(arr, dtype=dt)
            np.array([a.size], dtype=np.int64).tofile(f)
            a.tofile(f)
    subprocess.run([str(exe), str(inp), str(out)], check=True)
    res = {}
    with open(out, "rb") as f:
        for name, dt in FIELDS:
            n = int(np.fromfile(f, dtype=np.int64, count=1)[0])
            res[name] = np.fromfile(f, dtype=dt, count=n)
    return res


def structural_cholesky(P):
    """Column patterns of L for the SPD pattern P (lower, natural order) by
    symbolic elimination: struct(L_j) = struct(P_j) | union of children."""
    m = P.shape[0]
    Pl = sp.tril(P, -1).tocsc()
    cols = [set(Pl.indices[Pl.indptr[j]:Pl.indptr[j + 1]].tolist()) for j in range(m)]
    for j in range(m):
        if cols[j]:
            parent = min(cols[j])
            cols[parent] |= {i for i in cols[j] if i > parent}
    return cols


def cases(golden):
    for name in ("random_m300", "grid_20x25", "cover_m200", "dense_m1200"):
        g = golden(name)
        A = sp.csc_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=tuple(int(v) for v in g["A_shape"]))
        A.sum_duplicates()
        A.sort_indices()
        n_cores = int(g["n_cores"])
        for i in sorted({0, n_cores // 2, n_cores - 1}):
            yield f"{name}/core{i}", A, np.asarray(g[f"core{i}"], dtype=np.int64)


@pytest.mark.parametrize("ordering", [0, 2])
def test_symbolic_structure(driver, golden, ordering):
    rng = np.random.default_rng(3)
    checked = 0
    for label, A, core in cases(golden):
        S = run_symbolic(driver, A, core, ordering)
        rc, ns = int(S["head"][0]), int(S["head"][1])
        assert rc == 0, label
        m = A.shape[0]
        perm, iperm = S["perm"], S["iperm"]
        assert np.array_equal(np.sort(perm), np.arange(m)) and np.array_equal(iperm[perm], np.arange(m)), label
        first, rowptr, rows = S["sn_first"], S["sn_rowptr"], S["sn_rows"]
        assert first[0] == 0 and first[-1] == m and np.all(np.diff(first) > 0), label
        col2sn = np.repeat(np.arange(ns), np.diff(first))
        parent, level = S["sn_parent"], S["sn_level"]
        height = np.zeros(ns, dtype=np.int64)
        for s in range(ns):
            c = first[s + 1] - first[s]
            rs = rows[rowptr[s]:rowptr[s + 1]]
            assert np.array_equal(rs[:c], np.arange(first[s], first[s + 1])), (label, s)
            below = rs[c:]
            assert np.all(np.diff(below) > 0) and (below.size == 0 or below[0] >= first[s + 1]), (label, s)
            p = parent[s]
            if p < 0:
                assert below.size == 0, (label, s)
                continue
            assert p > s, (label, s)
            prow = rows[rowptr[p]:rowptr[p + 1]]
            rel = S["relind"][S["uvec_off"][s]:S["uvec_off"][s + 1]]
            assert np.array_equal(prow[rel], below), (label, s)
            height[p] = max(height[p], height[s] + 1)
        assert np.array_equal(level, height), label
        # structural Cholesky factor of P (permuted) inside the supernodal pattern
        Ac = A[:, core]
        P = (Ac @ Ac.T + sp.eye(m)).tocsc()
        Pp = P[perm][:, perm].tocsc()
        Lcols = structural_cholesky(Pp)
        for j in range(m):
            s = col2sn[j]
            allowed = set(rows[rowptr[s]:rowptr[s + 1]].tolist())
            assert Lcols[j] <= allowed, (label, j)
        # expanded product = A_C diag(w) A_C' (lower triangle, permuted order)
        w = rng.uniform(0.5, 2.0, core.size)
        M = (Ac @ sp.diags(w) @ Ac.T).tocsc()[perm][:, perm]
        lower = sp.tril(M).tocoo()
        want = {(int(i), int(j)): float(v) for i, j, v in zip(lower.row, lower.col, lower.data)}
        got = {}
        ent_ptr, ccol, cval = S["ent_ptr"], S["contrib_col"], S["contrib_val"]
        for e in range(S["ent_sn"].size):
            s = S["ent_sn"][e]
            j = first[s] + S["ent_col"][e]
            i = rows[rowptr[s] + S["ent_rowpos"][e]]
            got[(int(i), int(j))] = float(np.dot(cval[ent_ptr[e]:ent_ptr[e + 1]], w[ccol[ent_ptr[e]:ent_ptr[e + 1]]]))
        for key, v in want.items():
            assert key in got and abs(got[key] - v) <= 1e-12 * max(1.0, abs(v)), (label, key)
        assert all(abs(v) == 0.0 or key in want for key, v in got.items()), label
        de = S["diag_entry"]
        assert np.all(de >= 0), label
        for i in range(m):
            s = S["ent_sn"][de[i]]
            assert first[s] + S["ent_col"][de[i]] == i and rows[rowptr[s] + S["ent_rowpos"][de[i]]] == i
        checked += 1
    assert checked >= 10


def test_threaded_expanded_product(driver):
    """A core large enough (> 2^18 expanded-product keys) for the threaded
    construction: repeated runs give identical arrays, and the expanded product
    still assembles A_C diag(w) A_C' exactly."""
    from psipm_b200 import synthetic

    A = synthetic.grid_network(120, 160, seed=7).A.tocsc()
    A.sum_duplicates()
    A.sort_indices()
    core = np.flatnonzero(np.diff(A.indptr) >= 2).astype(np.int64)
    q = np.diff(A.indptr)[core]
    assert int((q * (q + 1) // 2).sum()) + A.shape[0] > (1 << 18)
    S1 = run_symbolic(driver, A, core)
    S2 = run_symbolic(driver, A, core)
    for name, _ in FIELDS:
        assert np.array_equal(S1[name], S2[name]), name
    S = S1
    assert int(S["head"][0]) == 0
    first, rowptr, rows = S["sn_first"], S["sn_rowptr"], S["sn_rows"]
    ent_ptr = S["ent_ptr"]
    j = first[S["ent_sn"]] + S["ent_col"]
    i = rows[rowptr[S["ent_sn"]] + S["ent_rowpos"]]
    w = np.random.default_rng(5).uniform(0.5, 2.0, core.size)
    counts = np.diff(ent_ptr)
    owner = np.repeat(np.arange(counts.size), counts)
    vals = np.bincount(owner, weights=S["contrib_val"] * w[S["contrib_col"]], minlength=counts.size)
    got = sp.coo_matrix((vals, (i, j)), shape=(A.shape[0],) * 2).tocsr()
    Ac = A[:, core]
    perm = S["perm"]
    want = sp.tril((Ac @ sp.diags(w) @ Ac.T).tocsc()[perm][:, perm]).tocsr()
    diff = abs(got - want)
    assert diff.max() <= 1e-12 * max(1.0, abs(want).max())
    assert got.nnz >= want.nnz
