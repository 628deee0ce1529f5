// The finishers of UltimateSolver after the anneal, on the host as in the
// reference. The 2-opt escape finisher (use_2opt):
// steepest-descent 1-opt with incremental gains (src/solver/local_search.rs:
// 19-57), then the steepest improving 2-flip along the coupling graph's edges
// (:83-121; pairs without a coupling can never improve a 1-opt minimum), flipped
// and descended again until neither exists (:123-143). The reference runs it
// on the host after the anneal; it is sequential by nature (one flip depends
// on the last) and touches O(nnz) per step. The path-relinking finisher
// (use_path_relinking, ultimate.rs:436-479 with src/solver/elite.rs): an elite
// archive of the field's replicas, greedy relinks between every pair of
// elites, each polished by 1-opt; the best state wins.
#include <algorithm>
#include <cstdint>
#include <limits>
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

size_t hamming(const int8_t* a, const int8_t* b, uint64_t n) {
    size_t d = 0;
    for (uint64_t i = 0; i < n; i++) d += a[i] != b[i];
    return d;
}

// EliteArchive (src/solver/elite.rs:21-123): at most `cap` solutions sorted by
// energy (stable), pairwise at least `min_h` apart; a candidate within the
// radius of an entry replaces the first such entry only when strictly better
// (by 1e-12), otherwise it enters when there is room or it beats the worst.
struct Elites {
    size_t cap, min_h;
    uint64_t n;
    std::vector<std::pair<double, std::vector<int8_t>>> e;

    void sort_trim() {
        std::stable_sort(e.begin(), e.end(), [](const std::pair<double, std::vector<int8_t>>& a,
                                                const std::pair<double, std::vector<int8_t>>& b) {
            return a.first < b.first;
        });
        if (e.size() > cap) e.resize(cap);
    }

    void insert(const int8_t* x, double energy) {
        const size_t radius = min_h > 0 ? min_h : 1;
        for (auto& entry : e)
            if (hamming(entry.second.data(), x, n) < radius) {
                if (energy < entry.first - 1e-12) {
                    entry = {energy, std::vector<int8_t>(x, x + n)};
                    sort_trim();
                }
                return;
            }
        if (e.size() < cap || energy < e.back().first - 1e-12) {
            e.push_back({energy, std::vector<int8_t>(x, x + n)});
            sort_trim();
        }
    }
};

// path_relink (elite.rs:133-181): from source toward target, each step flips
// the differing variable of lowest gain (lowest position on ties, the list
// kept by swap-remove), tracking the energy; the best state on the path.
std::vector<int8_t> path_relink(const Qubo& m, const std::vector<int8_t>& src, const std::vector<int8_t>& dst) {
    std::vector<int8_t> x(src), best(src);
    double e = energy(m, x.data());
    double best_e = e;
    std::vector<double> g;
    flip_gains(m, x.data(), g);
    std::vector<uint64_t> diff;
    for (uint64_t i = 0; i < m.n; i++)
        if (src[i] != dst[i]) diff.push_back(i);
    while (!diff.empty()) {
        size_t pick = 0;
        double bg = std::numeric_limits<double>::infinity();
        for (size_t k = 0; k < diff.size(); k++)
            if (g[diff[k]] < bg - 1e-15) {
                bg = g[diff[k]];
                pick = k;
            }
        const uint64_t i = diff[pick];
        diff[pick] = diff.back();
        diff.pop_back();
        const double dir = 1.0 - 2.0 * (double)x[i];
        e += g[i];
        x[i] = (int8_t)(1 - x[i]);
        g[i] = -g[i];
        for (uint64_t k = m.row[i]; k < m.row[i + 1]; k++) {
            const uint64_t j = m.col[k];
            g[j] += (1.0 - 2.0 * (double)x[j]) * m.val[k] * dir;
        }
        if (e < best_e) {
            best_e = e;
            best = x;
        }
    }
    return best;
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

ie_status ie_path_relink(const ie_problem* problem, const uint64_t* words, uint64_t cells,
                         const uint8_t* is_clamped, int8_t* state, double* energy_out) {
    if (!problem || (!state && problem->num_vars) || (!words && cells && problem->num_vars))
        return fail(IE_ERR_INVALID, "NULL argument");
    const Qubo m{problem->num_vars, problem->linear, problem->row_offsets, problem->col_indices, problem->values,
                 problem->energy_offset};
    if (m.n && (!m.lin || !m.row || (m.row[m.n] && (!m.col || !m.val)))) return fail(IE_ERR_INVALID, "NULL argument");
    for (uint64_t e = 0; m.n && e < m.row[m.n]; e++)
        if (m.col[e] >= m.n) return fail(IE_ERR_INVALID, "column index out of range");
    // ultimate.rs:436-479: the archive (8 entries, radius max(n / 10, 1)) of
    // the current state and every replica of the field, cell-major
    Elites arch{8, std::max<size_t>((size_t)(m.n / 10), 1), m.n, {}};
    const double e_cur = energy(m, state);
    arch.insert(state, e_cur);
    std::vector<int8_t> buf(m.n);
    for (uint64_t c = 0; c < cells; c++)
        for (uint32_t r = 0; r < 64; r++) {
            for (uint64_t v = 0; v < m.n; v++) buf[v] = (int8_t)((words[c * m.n + v] >> r) & 1u);
            arch.insert(buf.data(), energy(m, buf.data()));
        }
    std::vector<int8_t> best(state, state + m.n);
    double best_e = e_cur;
    std::vector<double> g;
    for (size_t i = 0; i < arch.e.size(); i++)
        for (size_t j = i + 1; j < arch.e.size(); j++) {
            std::vector<int8_t> x = path_relink(m, arch.e[i].second, arch.e[j].second);
            one_opt(m, x.data(), is_clamped, g);
            const double e = energy(m, x.data());
            if (e < best_e) {
                best_e = e;
                best = x;
            }
        }
    std::copy(best.begin(), best.end(), state);
    if (energy_out) *energy_out = best_e;
    return IE_OK;
}

}  // extern "C"
