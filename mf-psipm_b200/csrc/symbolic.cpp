// Host-side symbolic analysis for the GPU multifrontal Cholesky of the
// active-core normal matrix.  See symbolic.h for the pipeline.
#include "symbolic.h"

#include <algorithm>
#include <cstring>
#include <numeric>
#include <thread>
#include <utility>

namespace psipm {

namespace {

struct Graph {
    int32_t n = 0;
    std::vector<int64_t> xadj;  // n+1
    std::vector<int32_t> adj;   // symmetric, no self loops, sorted per row
};

// Pattern of A_C A_C^T without the diagonal, in original row indices.
Graph core_graph(int32_t m, const int64_t* colptr, const int32_t* rowidx, const int64_t* core,
                 int64_t ncore) {
    Graph g;
    g.n = m;
    std::vector<int64_t> deg(m + 1, 0);
    for (int64_t t = 0; t < ncore; ++t) {
        int64_t k = core[t];
        int64_t q = colptr[k + 1] - colptr[k];
        for (int64_t a = colptr[k]; a < colptr[k + 1]; ++a) deg[rowidx[a]] += q - 1;
    }
    g.xadj.assign(m + 1, 0);
    for (int32_t i = 0; i < m; ++i) g.xadj[i + 1] = g.xadj[i] + deg[i];
    std::vector<int32_t> raw(g.xadj[m]);
    std::vector<int64_t> fill(g.xadj.begin(), g.xadj.end() - 1);
    for (int64_t t = 0; t < ncore; ++t) {
        int64_t k = core[t];
        for (int64_t a = colptr[k]; a < colptr[k + 1]; ++a)
            for (int64_t b = colptr[k]; b < colptr[k + 1]; ++b)
                if (a != b) raw[fill[rowidx[a]]++] = rowidx[b];
    }
    // sort + unique per row
    std::vector<int64_t> nx(m + 1, 0);
    for (int32_t i = 0; i < m; ++i) {
        auto b = raw.begin() + g.xadj[i], e = raw.begin() + g.xadj[i + 1];
        std::sort(b, e);
        auto u = std::unique(b, e);
        nx[i + 1] = nx[i] + (u - b);
    }
    g.adj.resize(nx[m]);
    for (int32_t i = 0; i < m; ++i) {
        std::copy(raw.begin() + g.xadj[i], raw.begin() + g.xadj[i] + (nx[i + 1] - nx[i]),
                  g.adj.begin() + nx[i]);
    }
    g.xadj.swap(nx);
    return g;
}

// Nested dissection by BFS level structures.  Positions are assigned from
// the top of each subset's range: separator last, then the two sides.
void nested_dissection(const Graph& g, int32_t leaf, std::vector<int32_t>& order) {
    const int32_t n = g.n;
    order.assign(n, -1);
    std::vector<int32_t> part(n, 0);     // task label of each vertex
    std::vector<int32_t> level(n, -1);   // BFS level scratch
    std::vector<int32_t> queue(n);
    struct Task {
        std::vector<int32_t> verts;
        int32_t lo, label;
        bool connected = false;
    };
    std::vector<Task> stack;
    int32_t next_label = 1;
    {
        Task t;
        t.verts.resize(n);
        std::iota(t.verts.begin(), t.verts.end(), 0);
        t.lo = 0;
        t.label = 0;
        stack.push_back(std::move(t));
    }
    auto bfs = [&](int32_t src, int32_t label, std::vector<int32_t>& out_levels_ptr,
                   int32_t& count) {
        // fills queue[0..count) in BFS order, level[] for visited vertices
        int32_t head = 0, tail = 0;
        queue[tail++] = src;
        level[src] = 0;
        out_levels_ptr.clear();
        out_levels_ptr.push_back(0);
        int32_t cur = 0;
        while (head < tail) {
            int32_t v = queue[head];
            if (level[v] != cur) {
                out_levels_ptr.push_back(head);
                cur = level[v];
            }
            ++head;
            for (int64_t e = g.xadj[v]; e < g.xadj[v + 1]; ++e) {
                int32_t u = g.adj[e];
                if (part[u] == label && level[u] < 0) {
                    level[u] = level[v] + 1;
                    queue[tail++] = u;
                }
            }
        }
        out_levels_ptr.push_back(tail);
        count = tail;
    };
    std::vector<int32_t> lptr;
    while (!stack.empty()) {
        Task t = std::move(stack.back());
        stack.pop_back();
        const int32_t sz = (int32_t)t.verts.size();
        if (sz == 0) continue;
        for (int32_t v : t.verts) part[v] = t.label;
        if (!t.connected) {
            // split into connected components, each becomes its own task
            std::vector<std::vector<int32_t>> comps;
            int32_t cnt_c = 0;
            for (int32_t v0 : t.verts) {
                if (level[v0] >= 0) continue;
                bfs(v0, t.label, lptr, cnt_c);
                comps.emplace_back(queue.begin(), queue.begin() + cnt_c);
            }
            for (int32_t v : t.verts) level[v] = -1;
            if (comps.size() > 1) {
                int32_t lo2 = t.lo;
                for (auto& cv : comps) {
                    Task tc;
                    tc.lo = lo2;
                    lo2 += (int32_t)cv.size();
                    tc.verts = std::move(cv);
                    tc.label = next_label++;
                    tc.connected = true;
                    stack.push_back(std::move(tc));
                }
                continue;
            }
        }
        // start vertex: minimum degree
        int32_t src = t.verts[0];
        for (int32_t v : t.verts)
            if (g.xadj[v + 1] - g.xadj[v] < g.xadj[src + 1] - g.xadj[src]) src = v;
        int32_t count = 0;
        int32_t ecc = -1;
        for (int round = 0; round < 4; ++round) {
            bfs(src, t.label, lptr, count);
            int32_t d = (int32_t)lptr.size() - 2;
            // reset levels for next round
            if (d <= ecc) {
                break;
            }
            ecc = d;
            // candidate: min degree vertex in last level
            int32_t best = queue[lptr[d]];
            for (int32_t q = lptr[d]; q < lptr[d + 1]; ++q) {
                int32_t v = queue[q];
                if (g.xadj[v + 1] - g.xadj[v] < g.xadj[best + 1] - g.xadj[best]) best = v;
            }
            for (int32_t q = 0; q < count; ++q) level[queue[q]] = -1;
            if (best == src) break;
            src = best;
        }
        for (int32_t q = 0; q < count; ++q) level[queue[q]] = -1;
        bfs(src, t.label, lptr, count);
        std::vector<int32_t> comp(queue.begin(), queue.begin() + count);
        const int32_t d = (int32_t)lptr.size() - 2;
        const int32_t lo = t.lo;
        if (count <= leaf || d < 2) {
            // leaf: reverse BFS order keeps the band narrow; place as is
            for (int32_t q = 0; q < count; ++q) {
                order[lo + q] = comp[q];
                level[comp[q]] = -1;
            }
            continue;
        }
        // choose the separator level
        int32_t bestk = -1;
        double bestcost = 1e300;
        for (int32_t k = 1; k < d; ++k) {
            int32_t below = lptr[k];
            int32_t sep = lptr[k + 1] - lptr[k];
            int32_t above = count - lptr[k + 1];
            double bal = (double)std::min(below, above) / (double)std::max(1, below + above);
            if (bal < 0.15) continue;
            double cost = (double)sep / (0.25 + bal);
            if (cost < bestcost) {
                bestcost = cost;
                bestk = k;
            }
        }
        if (bestk < 0) {
            // no balanced level: take the level nearest the median
            for (int32_t k = 1; k < d; ++k)
                if (lptr[k + 1] * 2 >= count) {
                    bestk = k;
                    break;
                }
            if (bestk < 0) bestk = d / 2;
        }
        // classify: 0 = A (levels < k), 1 = S, 2 = B
        std::vector<int8_t> side(count);
        std::vector<int32_t> where(count);
        for (int32_t q = 0; q < count; ++q) {
            int32_t v = comp[q];
            side[q] = level[v] < bestk ? 0 : (level[v] == bestk ? 1 : 2);
        }
        // thinning: separator vertices without neighbours in B move to A,
        // then those without neighbours in A move to B
        std::vector<int32_t> pos_of(0);
        for (int32_t q = 0; q < count; ++q) level[comp[q]] = q;  // reuse as position
        for (int pass = 0; pass < 2; ++pass) {
            int8_t other = pass == 0 ? 2 : 0;
            int8_t dest = pass == 0 ? 0 : 2;
            for (int32_t q = 0; q < count; ++q) {
                if (side[q] != 1) continue;
                int32_t v = comp[q];
                bool touches = false;
                for (int64_t e = g.xadj[v]; e < g.xadj[v + 1] && !touches; ++e) {
                    int32_t u = g.adj[e];
                    if (part[u] == t.label && side[level[u]] == other) touches = true;
                }
                if (!touches) side[q] = dest;
            }
        }
        for (int32_t q = 0; q < count; ++q) level[comp[q]] = -1;
        Task ta, tb;
        std::vector<int32_t> sep;
        for (int32_t q = 0; q < count; ++q) {
            if (side[q] == 0)
                ta.verts.push_back(comp[q]);
            else if (side[q] == 2)
                tb.verts.push_back(comp[q]);
            else
                sep.push_back(comp[q]);
        }
        if (ta.verts.empty() || tb.verts.empty()) {
            // degenerate split: order the component as a leaf
            for (int32_t q = 0; q < count; ++q) order[lo + q] = comp[q];
            continue;
        }
        ta.lo = lo;
        tb.lo = lo + (int32_t)ta.verts.size();
        int32_t slo = tb.lo + (int32_t)tb.verts.size();
        for (size_t q = 0; q < sep.size(); ++q) order[slo + q] = sep[q];
        ta.label = next_label++;
        tb.label = next_label++;
        stack.push_back(std::move(ta));
        stack.push_back(std::move(tb));
    }
}


// Approximate minimum degree on the quotient graph (Amestoy, Davis & Duff,
// SIAM J. Matrix Anal. Appl. 17(4), 1996): elements absorb the elements of
// the pivot, external degrees are bounded by the AMD approximation, and
// indistinguishable variables are merged into supervariables by hashing.
uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

void amd_order(const Graph& g, std::vector<int32_t>& order) {
    const int32_t n = g.n;
    order.clear();
    order.reserve(n);
    enum : int8_t { VAR = 0, ELEM = 1, ABSORBED = 2, MERGED = 3 };
    std::vector<std::vector<int32_t>> V(n), E(n), L(n), merged(n);
    std::vector<int32_t> nv(n, 1);
    std::vector<int64_t> deg(n, 0);
    std::vector<int8_t> status(n, VAR);
    std::vector<int64_t> wval(n, 0);
    std::vector<int64_t> esize(n, 0);  // sum of nv over an element's variables
    std::vector<int32_t> wstamp(n, -1), mark(n, -1);
    for (int32_t i = 0; i < n; ++i) {
        V[i].assign(g.adj.begin() + g.xadj[i], g.adj.begin() + g.xadj[i + 1]);
        deg[i] = (int64_t)V[i].size();
    }
    // degree buckets (doubly linked)
    std::vector<int32_t> head(n + 1, -1), nxt(n, -1), prv(n, -1);
    auto bucket_of = [&](int32_t i) { return (int32_t)std::min<int64_t>(deg[i], n); };
    auto insert = [&](int32_t i) {
        int32_t d = bucket_of(i);
        nxt[i] = head[d];
        prv[i] = -1;
        if (head[d] >= 0) prv[head[d]] = i;
        head[d] = i;
    };
    auto remove = [&](int32_t i) {
        int32_t d = bucket_of(i);
        if (prv[i] >= 0)
            nxt[prv[i]] = nxt[i];
        else
            head[d] = nxt[i];
        if (nxt[i] >= 0) prv[nxt[i]] = prv[i];
        nxt[i] = prv[i] = -1;
    };
    for (int32_t i = 0; i < n; ++i) insert(i);
    int64_t eliminated = 0;
    int32_t mindeg = 0, tag = 0, step = 0;
    std::vector<int32_t> Lp;
    std::vector<std::pair<uint64_t, int32_t>> hashes;
    // variables and elements share one index space (both are graph nodes)
    std::vector<int32_t> setmark(n, 0);
    int32_t setstamp = 0;
    while (eliminated < n) {
        while (mindeg <= n && head[mindeg] < 0) ++mindeg;
        if (mindeg > n) break;
        const int32_t p = head[mindeg];
        remove(p);
        ++tag;
        ++step;
        mark[p] = tag;
        Lp.clear();
        for (int32_t e : E[p]) {
            if (status[e] != ELEM) continue;
            for (int32_t v : L[e])
                if (status[v] == VAR && mark[v] != tag) {
                    mark[v] = tag;
                    Lp.push_back(v);
                }
            status[e] = ABSORBED;
            std::vector<int32_t>().swap(L[e]);
        }
        for (int32_t v : V[p])
            if (status[v] == VAR && mark[v] != tag) {
                mark[v] = tag;
                Lp.push_back(v);
            }
        status[p] = ELEM;
        std::vector<int32_t>().swap(V[p]);
        std::vector<int32_t>().swap(E[p]);
        eliminated += nv[p];
        order.push_back(p);
        for (int32_t q : merged[p]) order.push_back(q);
        std::vector<int32_t>().swap(merged[p]);
        int64_t degLp = 0;
        for (int32_t i : Lp) degLp += nv[i];
        // prune the element lists of the new element's variables, and
        // w(e) = |Le \ Lp| for the other elements touching Lp.  w(e) starts
        // from |Le|, which never changes while e lives: a variable leaves Le
        // only as a pivot (which absorbs e) or by merging into a variable of Le.
        for (int32_t i : Lp) {
            remove(i);
            std::vector<int32_t>& Ei = E[i];
            size_t w = 0;
            for (int32_t e : Ei) {
                if (status[e] != ELEM) continue;
                Ei[w++] = e;
                if (wstamp[e] != step) {
                    wstamp[e] = step;
                    wval[e] = esize[e];
                }
                wval[e] -= nv[i];
            }
            Ei.resize(w);
            Ei.push_back(p);
        }
        // prune the variable lists (drop eliminated variables and those of Lp,
        // now reached through p), approximate external degrees, aggressive
        // absorption, and the supervariable hash of each variable's final
        // (V, E) lists.  An element
        // with w(e) <= 0 is a subset of Lp and is absorbed by the first variable
        // that meets it; w(e) is fixed for the step, so whether an element of
        // E[i] survives the step is known when i is visited.  The hash is a sum
        // of mixed indices, so it needs no sorted lists; equal hashes are
        // confirmed by marking one variable's lists and scanning the other's.
        hashes.clear();
        for (int32_t i : Lp) {
            int64_t dext = degLp - nv[i];
            uint64_t hl = 0;
            std::vector<int32_t>& Vi = V[i];
            size_t wv = 0;
            for (int32_t v : Vi) {
                if (status[v] != VAR || mark[v] == tag) continue;
                Vi[wv++] = v;
                dext += nv[v];
                hl += mix64((uint64_t)v);
            }
            Vi.resize(wv);
            std::vector<int32_t>& Ei = E[i];
            size_t w = 0;
            for (int32_t e : Ei) {
                if (e != p) {
                    if (status[e] != ELEM) continue;  // absorbed earlier in this pass
                    if (wval[e] <= 0) {
                        status[e] = ABSORBED;
                        std::vector<int32_t>().swap(L[e]);
                        continue;
                    }
                    dext += wval[e];
                }
                Ei[w++] = e;
                hl += mix64((uint64_t)e ^ 0x5bd1e9955bd1e995ull);
            }
            Ei.resize(w);
            int64_t bound = deg[i] + degLp - nv[i];
            deg[i] = std::max<int64_t>(0, std::min<int64_t>({dext, bound, (int64_t)n - eliminated}));
            hashes.emplace_back((uint64_t)wv * 0x9e3779b97f4a7c15ull + (uint64_t)w + hl, i);
        }
        std::sort(hashes.begin(), hashes.end());
        auto same_lists = [&](int32_t i, int32_t j) {
            if (V[i].size() != V[j].size() || E[i].size() != E[j].size()) return false;
            ++setstamp;
            for (int32_t v : V[i]) setmark[v] = setstamp;
            for (int32_t e : E[i]) setmark[e] = setstamp;
            for (int32_t v : V[j])
                if (setmark[v] != setstamp) return false;
            for (int32_t e : E[j])
                if (setmark[e] != setstamp) return false;
            return true;
        };
        for (size_t a = 0; a < hashes.size();) {
            size_t b = a;
            while (b < hashes.size() && hashes[b].first == hashes[a].first) ++b;
            for (size_t x = a; x < b; ++x) {
                int32_t i = hashes[x].second;
                if (status[i] != VAR) continue;
                for (size_t y = x + 1; y < b; ++y) {
                    int32_t j = hashes[y].second;
                    if (status[j] != VAR) continue;
                    if (same_lists(i, j)) {
                        nv[i] += nv[j];
                        merged[i].push_back(j);
                        for (int32_t q : merged[j]) merged[i].push_back(q);
                        std::vector<int32_t>().swap(merged[j]);
                        deg[i] = std::max<int64_t>(0, deg[i] - nv[j]);
                        nv[j] = 0;
                        status[j] = MERGED;
                        std::vector<int32_t>().swap(V[j]);
                        std::vector<int32_t>().swap(E[j]);
                    }
                }
            }
            a = b;
        }
        {
            size_t w = 0;
            for (int32_t i : Lp)
                if (status[i] == VAR) Lp[w++] = i;
            Lp.resize(w);
        }
        L[p] = Lp;
        esize[p] = degLp;
        for (int32_t i : Lp) {
            insert(i);
            mindeg = std::min(mindeg, bucket_of(i));
        }
    }
}

// Host threads for a symbolic analysis of `work` expanded-product keys: one
// below 2^18, else up to 8.
int host_threads(int64_t work) {
    if (work < (int64_t(1) << 18)) return 1;
    const unsigned hc = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(hc ? hc : 1u, 8u));
}

// f(thread, lo, hi) on `nthreads` contiguous ranges of [0, n), one per host
// thread (the calling thread takes the first).  f must not throw.
template <typename F>
void run_chunks(int nthreads, int64_t n, F f) {
    if (nthreads <= 1 || n <= 1) {
        f(0, 0, n);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(f, t, n * t / nthreads, n * (t + 1) / nthreads);
    f(0, 0, n / nthreads);
    for (auto& th : pool) th.join();
}

}  // namespace

int build_symbolic(int32_t m, int64_t n, const int64_t* colptr, const int32_t* rowidx,
                   const double* val, const int64_t* core, int64_t ncore,
                   const SymbolicOptions& opt, Symbolic& S) {
    if (m <= 0 || n < 0 || ncore < 0) return -1;
    for (int64_t t = 0; t < ncore; ++t) {
        if (core[t] < 0 || core[t] >= n) return -2;
        if (t && core[t] <= core[t - 1]) return -3;
    }
    S = Symbolic();
    S.m = m;
    Graph g = core_graph(m, colptr, rowidx, core, ncore);

    // ---- ordering ---------------------------------------------------------
    std::vector<int32_t> order;
    if (opt.ordering == 1) {
        order.resize(m);
        std::iota(order.begin(), order.end(), 0);
    } else if (opt.ordering == 2) {
        nested_dissection(g, std::max(2, opt.leaf_size), order);
    } else {
        amd_order(g, order);
    }
    {
        // the ordering must be a permutation
        std::vector<char> seen(m, 0);
        if ((int32_t)order.size() != m) return -4;
        for (int32_t v : order) {
            if (v < 0 || v >= m || seen[v]) return -5;
            seen[v] = 1;
        }
    }
    std::vector<int32_t> iperm(m);
    for (int32_t k = 0; k < m; ++k) iperm[order[k]] = k;

    // ---- elimination tree on the permuted graph ---------------------------
    auto permuted_lower = [&](const std::vector<int32_t>& ip, std::vector<int64_t>& lx,
                              std::vector<int32_t>& la) {
        // for each new index k: neighbours j < k (sorted)
        lx.assign(m + 1, 0);
        for (int32_t v = 0; v < m; ++v) {
            int32_t k = ip[v];
            for (int64_t e = g.xadj[v]; e < g.xadj[v + 1]; ++e)
                if (ip[g.adj[e]] < k) ++lx[k + 1];
        }
        for (int32_t k = 0; k < m; ++k) lx[k + 1] += lx[k];
        la.resize(lx[m]);
        std::vector<int64_t> f(lx.begin(), lx.end() - 1);
        for (int32_t v = 0; v < m; ++v) {
            int32_t k = ip[v];
            for (int64_t e = g.xadj[v]; e < g.xadj[v + 1]; ++e) {
                int32_t j = ip[g.adj[e]];
                if (j < k) la[f[k]++] = j;
            }
        }
        for (int32_t k = 0; k < m; ++k) std::sort(la.begin() + lx[k], la.begin() + lx[k + 1]);
    };
    std::vector<int64_t> lx;
    std::vector<int32_t> la;
    permuted_lower(iperm, lx, la);
    std::vector<int32_t> parent(m, -1), ancestor(m, -1);
    for (int32_t k = 0; k < m; ++k) {
        for (int64_t e = lx[k]; e < lx[k + 1]; ++e) {
            int32_t i = la[e];
            while (i != -1 && i < k) {
                int32_t inext = ancestor[i];
                ancestor[i] = k;
                if (inext == -1) parent[i] = k;
                i = inext;
            }
        }
    }
    // ---- postorder -------------------------------------------------------
    std::vector<int32_t> head(m, -1), next(m, -1), post(m), stackv;
    for (int32_t k = m - 1; k >= 0; --k)
        if (parent[k] != -1) {
            next[k] = head[parent[k]];
            head[parent[k]] = k;
        }
    {
        int32_t cnt = 0;
        for (int32_t r = 0; r < m; ++r) {
            if (parent[r] != -1) continue;
            stackv.push_back(r);
            while (!stackv.empty()) {
                int32_t p = stackv.back();
                int32_t c = head[p];
                if (c == -1) {
                    stackv.pop_back();
                    post[p] = cnt++;
                } else {
                    head[p] = next[c];
                    stackv.push_back(c);
                }
            }
        }
    }
    S.perm.resize(m);
    S.iperm.resize(m);
    for (int32_t v = 0; v < m; ++v) S.iperm[v] = post[iperm[v]];
    for (int32_t v = 0; v < m; ++v) S.perm[S.iperm[v]] = v;
    std::vector<int32_t> par(m, -1);
    for (int32_t k = 0; k < m; ++k) par[post[k]] = parent[k] == -1 ? -1 : post[parent[k]];
    permuted_lower(S.iperm, lx, la);

    // ---- column counts (row subtrees) -------------------------------------
    // Column count of j = number of row subtrees T_i (i >= j) that contain j.
    // Each T_i is described by weights on the tree: +1 at each of its leaves,
    // -1 at the lowest common ancestor of consecutive leaves (in postorder) and
    // -1 at the parent of i; the sum of the weights over the subtree of j is
    // then 1 if j is in T_i and 0 otherwise (the skeleton method of Gilbert,
    // Ng and Peyton, 1994).  Nodes are in postorder, so first[j] (smallest
    // node of j's subtree) and the least common ancestors come from one pass
    // with a union-find of the finished nodes: O(nnz(A)) instead of O(nnz(L)).
    std::vector<int64_t> cnt(m, 0);
    {
        std::vector<int32_t> first(m, -1);
        for (int32_t k = 0; k < m; ++k)
            for (int32_t j = k; j != -1 && first[j] == -1; j = par[j]) first[j] = k;
        // rows i > j of column j (transpose of the lower pattern)
        std::vector<int64_t> ux(m + 1, 0);
        for (int64_t e = 0; e < lx[m]; ++e) ++ux[la[e] + 1];
        for (int32_t k = 0; k < m; ++k) ux[k + 1] += ux[k];
        std::vector<int32_t> ua(lx[m]);
        {
            std::vector<int64_t> f(ux.begin(), ux.end() - 1);
            for (int32_t i = 0; i < m; ++i)
                for (int64_t e = lx[i]; e < lx[i + 1]; ++e) ua[f[la[e]]++] = i;
        }
        std::vector<int32_t> maxfirst(m, -1), prevleaf(m, -1), uf(m);
        std::iota(uf.begin(), uf.end(), 0);
        auto find = [&](int32_t u) {
            int32_t r = u;
            while (uf[r] != r) r = uf[r];
            while (uf[u] != r) {
                const int32_t nx = uf[u];
                uf[u] = r;
                u = nx;
            }
            return r;
        };
        auto leaf = [&](int32_t i, int32_t j) {  // is j a leaf of T_i?
            if (first[j] <= maxfirst[i]) return;
            maxfirst[i] = first[j];
            ++cnt[j];
            if (prevleaf[i] != -1) --cnt[find(prevleaf[i])];
            prevleaf[i] = j;
        };
        for (int32_t j = 0; j < m; ++j) {
            for (int64_t e = ux[j]; e < ux[j + 1]; ++e) leaf(ua[e], j);
            leaf(j, j);  // the diagonal: T_j = {j} when j has no earlier neighbour
            if (par[j] != -1) {
                --cnt[par[j]];
                uf[j] = par[j];
            }
        }
        for (int32_t j = 0; j < m; ++j)
            if (par[j] != -1) cnt[par[j]] += cnt[j];
    }
    std::vector<int32_t> nchild(m, 0);
    for (int32_t k = 0; k < m; ++k)
        if (par[k] != -1) ++nchild[par[k]];

    // ---- fundamental supernodes -------------------------------------------
    std::vector<int32_t> fs;  // first columns
    for (int32_t j = 0; j < m; ++j) {
        bool extend = j > 0 && par[j - 1] == j && cnt[j - 1] == cnt[j] + 1 && nchild[j] == 1;
        if (!extend) fs.push_back(j);
    }
    int32_t nf = (int32_t)fs.size();
    fs.push_back(m);
    std::vector<int32_t> col2f(m);
    for (int32_t s = 0; s < nf; ++s)
        for (int32_t j = fs[s]; j < fs[s + 1]; ++j) col2f[j] = s;
    // relaxed amalgamation (merge a supernode into its parent when it is the
    // parent's last child and the merged block stays dense enough)
    std::vector<int32_t> f_first(nf), f_ncols(nf), f_parent(nf);
    std::vector<int64_t> f_nrows(nf);
    std::vector<double> f_zeros(nf, 0.0);
    std::vector<int32_t> alias(nf);
    for (int32_t s = 0; s < nf; ++s) {
        f_first[s] = fs[s];
        f_ncols[s] = fs[s + 1] - fs[s];
        f_nrows[s] = cnt[fs[s]];
        int32_t last = fs[s + 1] - 1;
        f_parent[s] = par[last] == -1 ? -1 : col2f[par[last]];
        alias[s] = s;
    }
    auto entries = [](double c, double r) { return c * r - c * (c - 1.0) / 2.0; };
    for (int32_t s = 0; s + 1 < nf; ++s) {
        int32_t p = f_parent[s];
        if (p != s + 1) continue;  // only the last child is contiguous with its parent
        double cc = f_ncols[s], rc = (double)f_nrows[s];
        double cp = f_ncols[p], rp = (double)f_nrows[p];
        double cm = cc + cp, rm = cc + rp;
        double em = entries(cm, rm);
        double zm = f_zeros[s] + f_zeros[p] + em - entries(cc, rc) - entries(cp, rp);
        double frac = zm / em;
        bool merge = cm <= opt.relax_small || (cm <= opt.relax_medium && frac <= 0.8) ||
                     (cm <= opt.relax_large && frac <= 0.1) || frac <= 0.05;
        if (merge) {
            f_first[p] = f_first[s];
            f_ncols[p] = (int32_t)cm;
            f_nrows[p] = (int64_t)rm;
            f_zeros[p] = zm;
            alias[s] = p;
            f_ncols[s] = 0;  // dead
        }
    }
    // renumber live supernodes
    std::vector<int32_t> newid(nf, -1);
    int32_t ns = 0;
    for (int32_t s = 0; s < nf; ++s)
        if (f_ncols[s] > 0) newid[s] = ns++;
    S.ns = ns;
    S.sn_first.resize(ns + 1);
    for (int32_t s = 0; s < nf; ++s)
        if (f_ncols[s] > 0) S.sn_first[newid[s]] = f_first[s];
    S.sn_first[ns] = m;
    std::vector<int32_t> col2sn(m);
    for (int32_t s = 0; s < ns; ++s)
        for (int32_t j = S.sn_first[s]; j < S.sn_first[s + 1]; ++j) col2sn[j] = s;
    S.sn_parent.assign(ns, -1);
    for (int32_t s = 0; s < ns; ++s) {
        int32_t last = S.sn_first[s + 1] - 1;
        S.sn_parent[s] = par[last] == -1 ? -1 : col2sn[par[last]];
    }
    // children lists
    S.child_ptr.assign(ns + 1, 0);
    for (int32_t s = 0; s < ns; ++s)
        if (S.sn_parent[s] >= 0) ++S.child_ptr[S.sn_parent[s] + 1];
    for (int32_t s = 0; s < ns; ++s) S.child_ptr[s + 1] += S.child_ptr[s];
    S.child_list.resize(S.child_ptr[ns]);
    {
        std::vector<int32_t> f(S.child_ptr.begin(), S.child_ptr.end() - 1);
        for (int32_t s = 0; s < ns; ++s)
            if (S.sn_parent[s] >= 0) S.child_list[f[S.sn_parent[s]]++] = s;
    }
    // ---- supernode row structures -----------------------------------------
    // upper adjacency (rows > k of column k) is the transpose of la
    std::vector<int64_t> ux(m + 1, 0);
    for (int64_t e = 0; e < (int64_t)la.size(); ++e) ++ux[la[e] + 1];
    for (int32_t k = 0; k < m; ++k) ux[k + 1] += ux[k];
    std::vector<int32_t> ua(la.size());
    {
        std::vector<int64_t> f(ux.begin(), ux.end() - 1);
        for (int32_t i = 0; i < m; ++i)
            for (int64_t e = lx[i]; e < lx[i + 1]; ++e) ua[f[la[e]]++] = i;
    }
    S.sn_rowptr.assign(ns + 1, 0);
    std::vector<std::vector<int32_t>> rows(ns);
    std::vector<int32_t> mark(m, -1);
    for (int32_t s = 0; s < ns; ++s) {
        int32_t f0 = S.sn_first[s], f1 = S.sn_first[s + 1];
        std::vector<int32_t>& R = rows[s];
        for (int32_t j = f0; j < f1; ++j) {
            R.push_back(j);
            mark[j] = s;
        }
        for (int32_t j = f0; j < f1; ++j)
            for (int64_t e = ux[j]; e < ux[j + 1]; ++e) {
                int32_t i = ua[e];
                if (i >= f1 && mark[i] != s) {
                    mark[i] = s;
                    R.push_back(i);
                }
            }
        for (int32_t c = S.child_ptr[s]; c < S.child_ptr[s + 1]; ++c) {
            const std::vector<int32_t>& C = rows[S.child_list[c]];
            int32_t cc = S.sn_first[S.child_list[c] + 1] - S.sn_first[S.child_list[c]];
            for (size_t q = cc; q < C.size(); ++q) {
                int32_t i = C[q];
                if (i >= f1 && mark[i] != s) {
                    mark[i] = s;
                    R.push_back(i);
                }
            }
        }
        std::sort(R.begin() + (f1 - f0), R.end());
        S.sn_rowptr[s + 1] = S.sn_rowptr[s] + (int64_t)R.size();
    }
    S.sn_rows.resize(S.sn_rowptr[ns]);
    for (int32_t s = 0; s < ns; ++s)
        std::copy(rows[s].begin(), rows[s].end(), S.sn_rows.begin() + S.sn_rowptr[s]);
    // ---- offsets, levels, relative indices --------------------------------
    S.panel_off.assign(ns + 1, 0);
    S.update_off.assign(ns + 1, 0);
    S.uvec_off.assign(ns + 1, 0);
    S.sn_level.assign(ns, 0);
    for (int32_t s = 0; s < ns; ++s) {
        int64_t c = S.sn_first[s + 1] - S.sn_first[s];
        int64_t r = S.sn_rowptr[s + 1] - S.sn_rowptr[s];
        S.panel_off[s + 1] = S.panel_off[s] + r * c;
        S.update_off[s + 1] = S.update_off[s] + (r - c) * (r - c);
        S.uvec_off[s + 1] = S.uvec_off[s] + (r - c);
        S.nnz_L += c * r - c * (c - 1) / 2;
        S.max_front = std::max<int32_t>(S.max_front, (int32_t)r);
        S.max_cols = std::max<int32_t>(S.max_cols, (int32_t)c);
        double cd = (double)c, rd = (double)(r - c);
        S.flops += cd * cd * cd / 3.0 + cd * cd * rd + cd * rd * rd;
        int32_t lev = 0;
        for (int32_t q = S.child_ptr[s]; q < S.child_ptr[s + 1]; ++q)
            lev = std::max(lev, S.sn_level[S.child_list[q]] + 1);
        S.sn_level[s] = lev;
        S.nlevels = std::max(S.nlevels, lev + 1);
    }
    S.panel_total = S.panel_off[ns];
    S.update_total = S.update_off[ns];
    S.uvec_total = S.uvec_off[ns];
    S.level_ptr.assign(S.nlevels + 1, 0);
    for (int32_t s = 0; s < ns; ++s) ++S.level_ptr[S.sn_level[s] + 1];
    for (int32_t l = 0; l < S.nlevels; ++l) S.level_ptr[l + 1] += S.level_ptr[l];
    S.level_sn.resize(ns);
    {
        std::vector<int32_t> f(S.level_ptr.begin(), S.level_ptr.end() - 1);
        for (int32_t s = 0; s < ns; ++s) S.level_sn[f[S.sn_level[s]]++] = s;
    }
    S.relind.resize(S.uvec_total);
    for (int32_t s = 0; s < ns; ++s) {
        int32_t p = S.sn_parent[s];
        int64_t c = S.sn_first[s + 1] - S.sn_first[s];
        int64_t r = S.sn_rowptr[s + 1] - S.sn_rowptr[s];
        if (p < 0) {
            if (r != c) return -10;  // a root has no rows below its columns
            continue;
        }
        const int32_t* pr = S.sn_rows.data() + S.sn_rowptr[p];
        int64_t pn = S.sn_rowptr[p + 1] - S.sn_rowptr[p];
        for (int64_t q = c; q < r; ++q) {
            int32_t row = S.sn_rows[S.sn_rowptr[s] + q];
            const int32_t* it = std::lower_bound(pr, pr + pn, row);
            if (it == pr + pn || *it != row) {
                // rows of the parent's columns are not sorted with the rest
                int32_t pf = S.sn_first[p];
                if (row >= pf && row < S.sn_first[p + 1])
                    S.relind[S.uvec_off[s] + q - c] = row - pf;
                else
                    return -11;
            } else {
                S.relind[S.uvec_off[s] + q - c] = (int32_t)(it - pr);
            }
        }
    }
    // ---- expanded product -------------------------------------------------
    struct Key {
        int64_t pos;   // global position key: (sn, col, rowpos) linearised
        int32_t k;     // core-local column
        int32_t s;     // supernode of the position
        double v;
    };
    // linearised front position: sn_rowptr-based column-major within the
    // panel: panel_off[s] + rowpos * c + col  (row-major panel index).
    // Large analyses split the key generation, the supernode scatter and the
    // per-supernode sorts over host threads; every thread owns a fixed range
    // and writes fixed slots, so the result is the sequential one.
    std::vector<int64_t> kofs(ncore + 1, 0);
    for (int64_t t = 0; t < ncore; ++t) {
        const int64_t q = colptr[core[t] + 1] - colptr[core[t]];
        kofs[t + 1] = kofs[t] + q * (q + 1) / 2;
    }
    const int64_t ncol_keys = kofs[ncore];
    std::vector<Key> keys((size_t)(ncol_keys + m));
    const int nthreads = host_threads(ncol_keys + m);
    std::vector<int> thread_rc(nthreads, 0);
    run_chunks(nthreads, ncore, [&](int tid, int64_t lo, int64_t hi) {
      try {
        std::vector<std::pair<int32_t, double>> col;
        for (int64_t t = lo; t < hi; ++t) {
            int64_t kk = core[t];
            col.clear();
            for (int64_t a = colptr[kk]; a < colptr[kk + 1]; ++a)
                col.emplace_back(S.iperm[rowidx[a]], val[a]);
            std::sort(col.begin(), col.end());
            int64_t out = kofs[t];
            for (size_t a = 0; a < col.size(); ++a)
                for (size_t b = a; b < col.size(); ++b) {
                    int32_t j = col[a].first, i = col[b].first;  // j <= i
                    int32_t s = col2sn[j];
                    const int32_t* sr = S.sn_rows.data() + S.sn_rowptr[s];
                    int64_t rn = S.sn_rowptr[s + 1] - S.sn_rowptr[s];
                    int32_t c = S.sn_first[s + 1] - S.sn_first[s];
                    int64_t rp;
                    if (i < S.sn_first[s + 1]) {
                        rp = i - S.sn_first[s];
                    } else {
                        const int32_t* it = std::lower_bound(sr + c, sr + rn, i);
                        if (it == sr + rn || *it != i) {
                            thread_rc[tid] = -12;
                            return;
                        }
                        rp = it - sr;
                    }
                    int64_t pos = S.panel_off[s] + rp * c + (j - S.sn_first[s]);
                    keys[out++] = {pos, (int32_t)t, s, col[a].second * col[b].second};
                }
        }
      } catch (...) {
        thread_rc[tid] = -14;  // host allocation failed
      }
    });
    for (int rc : thread_rc)
        if (rc) return rc;
    // every diagonal entry exists even without contributions
    for (int32_t i = 0; i < m; ++i) {
        int32_t s = col2sn[i];
        int32_t c = S.sn_first[s + 1] - S.sn_first[s];
        int64_t rp = i - S.sn_first[s];
        keys[ncol_keys + i] = {S.panel_off[s] + rp * c + rp, -1, s, 0.0};
    }
    // order by (position, column): a stable counting sort by supernode (positions
    // of different supernodes do not interleave), then a sort inside each
    // supernode's short run.  The scatter is stable across threads: thread t's
    // keys of a supernode go after those of threads < t.
    {
        const int64_t nk = (int64_t)keys.size();
        std::vector<std::vector<int64_t>> cnt(nthreads, std::vector<int64_t>(ns + 1, 0));
        run_chunks(nthreads, nk, [&](int tid, int64_t lo, int64_t hi) {
            std::vector<int64_t>& c = cnt[tid];
            for (int64_t q = lo; q < hi; ++q) ++c[keys[q].s];
        });
        std::vector<int64_t> bptr(ns + 1, 0);
        {
            int64_t run = 0;
            for (int32_t t = 0; t < ns; ++t) {
                bptr[t] = run;
                for (int tid = 0; tid < nthreads; ++tid) {
                    const int64_t v = cnt[tid][t];
                    cnt[tid][t] = run;  // this thread's first slot for supernode t
                    run += v;
                }
            }
            bptr[ns] = run;
        }
        std::vector<Key> sorted(keys.size());
        run_chunks(nthreads, nk, [&](int tid, int64_t lo, int64_t hi) {
            std::vector<int64_t>& f = cnt[tid];
            for (int64_t q = lo; q < hi; ++q) sorted[f[keys[q].s]++] = keys[q];
        });
        auto less = [](const Key& a, const Key& b) { return a.pos < b.pos || (a.pos == b.pos && a.k < b.k); };
        // supernode ranges of about equal key counts per thread
        std::vector<int32_t> sbeg(nthreads + 1, ns);
        sbeg[0] = 0;
        for (int tid = 1, t = 0; tid < nthreads; ++tid) {
            const int64_t goal = nk * tid / nthreads;
            while (t < ns && bptr[t] < goal) ++t;
            sbeg[tid] = t;
        }
        run_chunks(nthreads, nthreads, [&](int, int64_t lo, int64_t hi) {
            for (int64_t part = lo; part < hi; ++part)
                for (int32_t t = sbeg[part]; t < sbeg[part + 1]; ++t)
                    std::sort(sorted.begin() + bptr[t], sorted.begin() + bptr[t + 1], less);
        });
        keys.swap(sorted);
    }
    // distinct positions -> entries
    S.ent_ptr.clear();
    S.contrib_col.clear();
    S.contrib_val.clear();
    std::vector<int64_t> ent_pos;
    for (size_t q = 0; q < keys.size(); ++q) {
        if (q == 0 || keys[q].pos != keys[q - 1].pos) {
            ent_pos.push_back(keys[q].pos);
            S.ent_ptr.push_back((int64_t)S.contrib_col.size());
        }
        if (keys[q].k >= 0) {
            S.contrib_col.push_back(keys[q].k);
            S.contrib_val.push_back(keys[q].v);
        }
    }
    S.ent_ptr.push_back((int64_t)S.contrib_col.size());
    S.nentries = (int64_t)ent_pos.size();
    S.ent_sn.resize(S.nentries);
    S.ent_col.resize(S.nentries);
    S.ent_rowpos.resize(S.nentries);
    S.diag_entry.assign(m, -1);
    S.sn_entptr.assign(ns + 1, 0);
    {
        int32_t s = 0;
        for (int64_t e = 0; e < S.nentries; ++e) {
            int64_t pos = ent_pos[e];
            while (S.panel_off[s + 1] <= pos) ++s;
            int32_t c = S.sn_first[s + 1] - S.sn_first[s];
            int64_t local = pos - S.panel_off[s];
            S.ent_sn[e] = s;
            S.ent_col[e] = (int32_t)(local % c);
            S.ent_rowpos[e] = (int32_t)(local / c);
            if (S.ent_rowpos[e] == S.ent_col[e]) S.diag_entry[S.sn_first[s] + S.ent_col[e]] = e;
            ++S.sn_entptr[s + 1];
        }
        for (int32_t q = 0; q < ns; ++q) S.sn_entptr[q + 1] += S.sn_entptr[q];
    }
    for (int32_t i = 0; i < m; ++i)
        if (S.diag_entry[i] < 0) return -13;
    return 0;
}

}  // namespace psipm
