// The 2-opt escape finisher of UltimateSolver (use_2opt) on the host:
// steepest-descent 1-opt with incremental gains (src/solver/local_search.rs:
// 19-57), then the steepest improving 2-flip along the coupling graph's edges
// (:83-121; pairs without a coupling can never improve a 1-opt minimum), flipped
// and descended again until neither exists (:123-143). The reference runs it
// on the host after the anneal; it is sequential by nature (one flip depends
// on the last) and touches O(nnz) per step.
#include <cstdint>
#include <vector>

#include "ie_host.h"

namespace ie {
namespace {

struct Qubo {
    uint64_t n;
    const double* lin;
    const uint64_t* row;
    const uint64_t* col;
    const double* val;
    double offset;
};

// compute_single_flip_gains (local_search.rs:61-74): g_i = (1 - 2 x_i) *
// (lin_i + sum_j w_ij x_j), f64 in CSR order.
void flip_gains(const Qubo& m, const int8_t* x, std::vector<double>& g) {
    g.assign(m.n, 0.0);
    for (uint64_t i = 0; i < m.n; i++) {
        double field = m.lin[i];
        for (uint64_t e = m.row[i]; e < m.row[i + 1]; e++) field += m.val[e] * (double)x[m.col[e]];
        g[i] = (1.0 - 2.0 * (double)x[i]) * field;
    }
}

// local_search.rs:19-57: steepest flip below -1e-12 with the lowest index on
// ties, incremental neighbour updates.
void one_opt(const Qubo& m, int8_t* x, const uint8_t* clamped, std::vector<double>& g) {
    flip_gains(m, x, g);
    for (;;) {
        uint64_t bi = UINT64_MAX;
        double bg = -1e-12;
        for (uint64_t i = 0; i < m.n; i++)
            if (!(clamped && clamped[i]) && g[i] < bg) {
                bi = i;
                bg = g[i];
            }
        if (bi == UINT64_MAX) return;
        const double dir = 1.0 - 2.0 * (double)x[bi];
        x[bi] = (int8_t)(1 - x[bi]);
        g[bi] = -bg;
        for (uint64_t e = m.row[bi]; e < m.row[bi + 1]; e++) {
            const uint64_t j = m.col[e];
            g[j] += (1.0 - 2.0 * (double)x[j]) * m.val[e] * dir;
        }
    }
}

double energy(const Qubo& m, const int8_t* x) {  // src/core/hubo.rs:176-189
    double e = m.offset;
    for (uint64_t i = 0; i < m.n; i++) {
        if (x[i] != 1) continue;
        e += m.lin[i];
        for (uint64_t k = m.row[i]; k < m.row[i + 1]; k++)
            if (x[m.col[k]] == 1) e += m.val[k] * 0.5;
    }
    return e;
}

}  // namespace
}  // namespace ie

using namespace ie;

extern "C" {

ie_status ie_two_opt(const ie_problem* problem, int8_t* state, const uint8_t* is_clamped, double* improvement) {
    if (!problem || (!state && problem->num_vars)) return fail(IE_ERR_INVALID, "NULL argument");
    const Qubo m{problem->num_vars, problem->linear, problem->row_offsets, problem->col_indices, problem->values,
                 problem->energy_offset};
    if (m.n && (!m.lin || !m.row || (m.row[m.n] && (!m.col || !m.val)))) return fail(IE_ERR_INVALID, "NULL argument");
    for (uint64_t e = 0; m.n && e < m.row[m.n]; e++)
        if (m.col[e] >= m.n) return fail(IE_ERR_INVALID, "column index out of range");
    for (uint64_t i = 0; i < m.n; i++)
        if (state[i] != 0 && state[i] != 1) return fail(IE_ERR_INVALID, "state entries must be 0 or 1");
    const double e0 = energy(m, state);
    std::vector<double> g;
    for (;;) {
        one_opt(m, state, is_clamped, g);
        flip_gains(m, state, g);  // recomputed after the descent (local_search.rs:131)
        uint64_t bu = UINT64_MAX, bv = 0;
        double best = 0.0;
        for (uint64_t u = 0; u < m.n; u++) {
            if (is_clamped && is_clamped[u]) continue;
            const double su = 1.0 - 2.0 * (double)state[u];
            for (uint64_t e = m.row[u]; e < m.row[u + 1]; e++) {
                const uint64_t v = m.col[e];
                if (v <= u || (is_clamped && is_clamped[v])) continue;
                const double sv = 1.0 - 2.0 * (double)state[v];
                const double d = g[u] + g[v] + m.val[e] * su * sv;
                if (d < -1e-12 && (bu == UINT64_MAX || d < best)) {
                    bu = u;
                    bv = v;
                    best = d;
                }
            }
        }
        if (bu == UINT64_MAX) break;
        state[bu] = (int8_t)(1 - state[bu]);
        state[bv] = (int8_t)(1 - state[bv]);
    }
    const double d = e0 - energy(m, state);
    if (improvement) *improvement = d > 0.0 ? d : 0.0;
    return IE_OK;
}

}  // extern "C"
