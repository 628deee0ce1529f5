// Presolve and decomposition before the anneal (host only): the reductions
// UltimateSolver::solve applies first (src/solver/ultimate.rs:161-218).
//  - first-order persistency to a fixpoint (src/presolve/mod.rs:54-105),
//  - probing persistency (mod.rs:125-180),
//  - roof duality / QPBO strong persistencies by max-flow on the implication
//    network (src/presolve/qpbo.rs:40-293), on the clamp-reduced model
//    (mod.rs:330-381),
//  - their union (full_presolve, mod.rs:279-324),
//  - connected components of the free-variable graph (mod.rs:189-218).
// The fixings decide which sites the device anneals, so the algorithms are
// followed step for step: the same f64 arithmetic, the same Dinic edge order
// and residual epsilon, the same visiting orders.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <deque>
#include <limits>
#include <vector>

#include "ie_host.h"

namespace ie {
namespace {

constexpr int8_t kFree = -1;

// A QUBO in CSR form (both triangles, reference row order).
struct Csr {
    size_t n = 0;
    std::vector<double> lin, val;
    std::vector<size_t> row, col;
};

Csr from_problem(const ie_problem* p) {
    Csr m;
    m.n = (size_t)p->num_vars;
    m.lin.assign(p->linear, p->linear + m.n);
    m.row.resize(m.n + 1);
    for (size_t i = 0; i <= m.n; i++) m.row[i] = (size_t)p->row_offsets[i];
    const size_t nnz = m.row[m.n];
    m.col.resize(nnz);
    m.val.assign(p->values, p->values + nnz);
    for (size_t e = 0; e < nnz; e++) m.col[e] = (size_t)p->col_indices[e];
    return m;
}

// mod.rs:54-105: state[i] = fixed value or kFree.
std::vector<int8_t> first_order(const Csr& m, const std::vector<std::pair<size_t, int8_t>>& assume) {
    std::vector<double> h = m.lin;
    std::vector<int8_t> st(m.n, kFree);
    for (const auto& a : assume) st[a.first] = a.second;
    for (const auto& a : assume)
        if (a.second == 1)
            for (size_t e = m.row[a.first]; e < m.row[a.first + 1]; e++) h[m.col[e]] += m.val[e];
    for (bool changed = true; changed;) {
        changed = false;
        for (size_t i = 0; i < m.n; i++) {
            if (st[i] != kFree) continue;
            double lo = h[i], hi = h[i];
            for (size_t e = m.row[i]; e < m.row[i + 1]; e++) {
                if (st[m.col[e]] != kFree) continue;
                if (m.val[e] < 0.0) lo += m.val[e];
                else hi += m.val[e];
            }
            if (lo >= 0.0) {
                st[i] = 0;
                changed = true;
            } else if (hi <= 0.0) {
                st[i] = 1;
                for (size_t e = m.row[i]; e < m.row[i + 1]; e++) h[m.col[e]] += m.val[e];
                changed = true;
            }
        }
    }
    return st;
}

bool has(const std::vector<std::pair<size_t, int8_t>>& v, size_t i) {
    for (const auto& a : v)
        if (a.first == i) return true;
    return false;
}

// mod.rs:125-180: a variable fixed to the same value under both case splits
// of another is fixed; repeated until nothing is added. Returns the
// assumptions (clamps included, in the reference's order).
std::vector<std::pair<size_t, int8_t>> probing(const Csr& m, std::vector<std::pair<size_t, int8_t>> assume) {
    for (;;) {
        const std::vector<int8_t> base = first_order(m, assume);
        std::vector<std::pair<size_t, int8_t>> fixed, newly;
        for (size_t i = 0; i < m.n; i++)
            if (base[i] != kFree) fixed.push_back({i, base[i]});
        for (size_t i = 0; i < m.n; i++) {
            if (base[i] != kFree) continue;
            auto a = fixed;
            a.push_back({i, 0});
            const std::vector<int8_t> b0 = first_order(m, a);
            a.back().second = 1;
            const std::vector<int8_t> b1 = first_order(m, a);
            for (size_t j = 0; j < m.n; j++) {
                if (j == i || base[j] != kFree) continue;
                if (b0[j] != kFree && b0[j] == b1[j] && !has(newly, j)) newly.push_back({j, b0[j]});
            }
        }
        const size_t before = assume.size();
        for (const auto* src : {&fixed, &newly})
            for (const auto& a : *src)
                if (!has(assume, a.first)) assume.push_back(a);
        if (assume.size() == before) return assume;
    }
}

// Dinic max-flow on f64 capacities with the residual epsilon of qpbo.rs:42.
struct MaxFlow {
    static constexpr double kEps = 1e-9;
    std::vector<std::vector<size_t>> out;  // node -> arc ids, in insertion order
    std::vector<size_t> head;              // arc -> target node
    std::vector<double> cap;
    std::vector<int> depth;
    std::vector<size_t> next_arc;

    explicit MaxFlow(size_t nodes) : out(nodes), depth(nodes), next_arc(nodes) {}

    void arc(size_t u, size_t v, double c) {
        out[u].push_back(head.size());
        head.push_back(v);
        cap.push_back(c);
        out[v].push_back(head.size());
        head.push_back(u);
        cap.push_back(0.0);
    }

    bool layer(size_t s, size_t t) {
        std::fill(depth.begin(), depth.end(), -1);
        std::deque<size_t> q{s};
        depth[s] = 0;
        while (!q.empty()) {
            const size_t u = q.front();
            q.pop_front();
            for (size_t a : out[u])
                if (cap[a] > kEps && depth[head[a]] < 0) {
                    depth[head[a]] = depth[u] + 1;
                    q.push_back(head[a]);
                }
        }
        return depth[t] >= 0;
    }

    double push(size_t u, size_t t, double f) {
        if (u == t) return f;
        for (; next_arc[u] < out[u].size(); next_arc[u]++) {
            const size_t a = out[u][next_arc[u]], v = head[a];
            if (cap[a] > kEps && depth[v] == depth[u] + 1) {
                const double d = push(v, t, std::min(f, cap[a]));
                if (d > kEps) {
                    cap[a] -= d;
                    cap[a ^ 1] += d;
                    return d;
                }
            }
        }
        return 0.0;
    }

    void run(size_t s, size_t t) {
        while (layer(s, t)) {
            std::fill(next_arc.begin(), next_arc.end(), 0);
            while (push(s, t, std::numeric_limits<double>::infinity()) > kEps) {
            }
        }
    }

    // nodes reachable from s along residual arcs (reverse = against them)
    std::vector<char> reach(size_t s, bool reverse) const {
        const size_t nn = out.size();
        std::vector<std::vector<size_t>> adj(nn);
        for (size_t u = 0; u < nn; u++)
            for (size_t a : out[u])
                if (cap[a] > kEps) {
                    if (reverse) adj[head[a]].push_back(u);
                    else adj[u].push_back(head[a]);
                }
        std::vector<char> seen(nn, 0);
        std::deque<size_t> q{s};
        seen[s] = 1;
        while (!q.empty()) {
            const size_t u = q.front();
            q.pop_front();
            for (size_t v : adj[u])
                if (!seen[v]) {
                    seen[v] = 1;
                    q.push_back(v);
                }
        }
        return seen;
    }
};

// qpbo.rs:155-275: posiform of E / scale on the implication network of 2n
// literals (x_i = 2i, its complement 2i + 1) plus T = 2n and F = 2n + 1; after
// the max flow, x_i is fixed when its literal and complement fall on definite
// opposite sides of the residual cut.
std::vector<int8_t> roof_duality(const Csr& m) {
    const size_t n = m.n;
    if (n == 0) return {};
    const size_t T = 2 * n, F = 2 * n + 1;
    auto bar = [&](size_t lit) { return lit == T ? F : (lit == F ? T : lit ^ 1); };
    double scale = 0.0;
    for (size_t i = 0; i < n; i++) {
        scale = std::max(scale, std::fabs(m.lin[i]));
        for (size_t e = m.row[i]; e < m.row[i + 1]; e++) scale = std::max(scale, std::fabs(m.val[e]));
    }
    if (!(scale > 0.0)) scale = 1.0;
    MaxFlow g(2 * n + 2);
    auto quad = [&](size_t u, size_t v, double c) {
        if (c > MaxFlow::kEps) {
            g.arc(u, bar(v), c);
            g.arc(v, bar(u), c);
        }
    };
    auto linear = [&](size_t u, double c) {
        if (c >= 0.0) {
            if (c > MaxFlow::kEps) {
                g.arc(u, F, c);
                g.arc(T, bar(u), c);
            }
        } else {
            g.arc(bar(u), F, -c);
            g.arc(T, u, -c);
        }
    };
    for (size_t i = 0; i < n; i++) linear(2 * i, m.lin[i] / scale);
    for (size_t i = 0; i < n; i++)
        for (size_t e = m.row[i]; e < m.row[i + 1]; e++) {
            const size_t j = m.col[e];
            if (i >= j) continue;
            const double w = m.val[e] / scale;
            if (w >= 0.0) {
                quad(2 * i, 2 * j, w);
            } else {
                linear(2 * i, w);
                quad(2 * i, 2 * j + 1, -w);
            }
        }
    g.run(T, F);
    const std::vector<char> src_side = g.reach(T, false), sink_side = g.reach(F, true);
    std::vector<int8_t> out(n, kFree);
    for (size_t i = 0; i < n; i++) {
        const size_t p = 2 * i, q = 2 * i + 1;
        if (src_side[p] && sink_side[q]) out[i] = 1;
        else if (sink_side[p] && src_side[q]) out[i] = 0;
    }
    return out;
}

// mod.rs:330-381: the free variables' QUBO with clamped-1 neighbours folded
// into the linear terms; rows sorted by (reduced) column.
Csr reduce_by_clamps(const Csr& m, const std::vector<int8_t>& clamp, std::vector<size_t>& free) {
    free.clear();
    std::vector<size_t> g2l(m.n, SIZE_MAX);
    for (size_t i = 0; i < m.n; i++)
        if (clamp[i] == kFree) {
            g2l[i] = free.size();
            free.push_back(i);
        }
    Csr r;
    r.n = free.size();
    r.lin.resize(r.n);
    r.row.assign(1, 0);
    std::vector<std::pair<size_t, double>> rowbuf;
    for (size_t li = 0; li < r.n; li++) {
        const size_t gi = free[li];
        double h = m.lin[gi];
        rowbuf.clear();
        for (size_t e = m.row[gi]; e < m.row[gi + 1]; e++) {
            const size_t j = m.col[e];
            if (clamp[j] == kFree) rowbuf.push_back({g2l[j], m.val[e]});
            else if (clamp[j] == 1) h += m.val[e];
        }
        r.lin[li] = h;
        std::stable_sort(rowbuf.begin(), rowbuf.end(),
                         [](const std::pair<size_t, double>& a, const std::pair<size_t, double>& b) {
                             return a.first < b.first;
                         });
        for (const auto& x : rowbuf) {
            r.col.push_back(x.first);
            r.val.push_back(x.second);
        }
        r.row.push_back(r.col.size());
    }
    return r;
}

}  // namespace
}  // namespace ie

using namespace ie;

extern "C" {

ie_status ie_presolve(const ie_problem* problem, const uint64_t* clamp_idx, const int8_t* clamp_val,
                      uint64_t n_clamps, uint64_t* out_idx, int8_t* out_val, uint64_t* n_out) {
    if (!problem || !n_out || (n_clamps && (!clamp_idx || !clamp_val))) return fail(IE_ERR_INVALID, "NULL argument");
    if (problem->num_vars && (!problem->linear || !problem->row_offsets)) return fail(IE_ERR_INVALID, "NULL argument");
    const Csr m = from_problem(problem);
    if (m.row[m.n] && (!problem->col_indices || !problem->values)) return fail(IE_ERR_INVALID, "NULL argument");
    for (size_t e = 0; e < m.col.size(); e++)
        if (m.col[e] >= m.n) return fail(IE_ERR_INVALID, "column index out of range");
    std::vector<std::pair<size_t, int8_t>> assume;
    std::vector<int8_t> clamp(m.n, kFree);
    std::vector<char> user(m.n, 0);
    for (uint64_t k = 0; k < n_clamps; k++) {
        if (clamp_idx[k] >= m.n || (clamp_val[k] != 0 && clamp_val[k] != 1))
            return fail(IE_ERR_INVALID, "clamp index or value out of range");
        assume.push_back({(size_t)clamp_idx[k], clamp_val[k]});
        clamp[clamp_idx[k]] = clamp_val[k];
        user[clamp_idx[k]] = 1;
    }
    // strong persistencies of the clamp-reduced model
    std::vector<size_t> free;
    const Csr red = reduce_by_clamps(m, clamp, free);
    const std::vector<int8_t> qp = roof_duality(red);
    for (size_t li = 0; li < qp.size(); li++) {
        const size_t gi = free[li];
        if (qp[li] != kFree && !user[gi] && !has(assume, gi)) assume.push_back({gi, qp[li]});
    }
    // probing on top, then the union without the user's clamps
    const std::vector<std::pair<size_t, int8_t>> probed = probing(m, assume);
    for (const auto& a : probed)
        if (!user[a.first] && !has(assume, a.first)) assume.push_back(a);
    uint64_t k = 0;
    for (const auto& a : assume) {
        if (user[a.first]) continue;
        if (out_idx) out_idx[k] = a.first;
        if (out_val) out_val[k] = a.second;
        k++;
    }
    *n_out = k;
    return IE_OK;
}

ie_status ie_connected_components(const ie_problem* problem, const uint8_t* active, uint64_t* component,
                                  uint64_t* n_components) {
    if (!problem || !active || !component || !n_components) return fail(IE_ERR_INVALID, "NULL argument");
    const Csr m = from_problem(problem);
    for (size_t e = 0; e < m.col.size(); e++)
        if (m.col[e] >= m.n) return fail(IE_ERR_INVALID, "column index out of range");
    std::fill(component, component + m.n, UINT64_MAX);
    uint64_t c = 0;
    std::vector<size_t> stack;
    for (size_t s = 0; s < m.n; s++) {
        if (!active[s] || component[s] != UINT64_MAX) continue;
        component[s] = c;
        stack.push_back(s);
        while (!stack.empty()) {
            const size_t v = stack.back();
            stack.pop_back();
            for (size_t e = m.row[v]; e < m.row[v + 1]; e++) {
                const size_t j = m.col[e];
                if (m.val[e] != 0.0 && active[j] && component[j] == UINT64_MAX) {
                    component[j] = c;
                    stack.push_back(j);
                }
            }
        }
        c++;
    }
    *n_components = c;
    return IE_OK;
}

}  // extern "C"
