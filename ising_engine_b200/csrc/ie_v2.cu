// engine_v2 (S2) state backend on the device: the integer bit-sliced state of
// src/engine_v2/backends/sparse_bitslice.rs:19-346 with the MetropolisSweep
// (src/engine_v2/operators/metropolis_sweep.rs:95-146), GibbsColorSweep
// (src/engine_v2/operators/gibbs_color_sweep.rs:119-165) and ReplicaExchange
// (src/engine_v2/operators/replica_exchange.rs:61-110) operators, behind the
// per-sweep seam ie_v2_* of include/ising_b200.h.
//
// Layout: spins[site * w + word] (u64, bit b = replica 64 * word + b, the
// reference's planes), read by the kernels as u32 halves so a warp owns 32
// replicas of a site; energies as int64 per replica. The reference keeps an
// integer local-field ledger; here a site's field lin + sum_j w_j x_j is
// gathered from the neighbours' planes when the site is visited. Both are
// exact integers, so every dE equals the ledger's.
//
// MetropolisSweep draws one gen::<f64>() per (site, replica) in chromatic
// order, every sweep: draw ((sweep * n + position) * r + replica) of the
// operator's stream, computed directly from its index (ChaCha8 is a counter
// generator), so all sites of one colour (never neighbours) and all replicas
// are decided at once. Acceptance d <= 0, or u < exp(-d / t): for integer d
// that is (draw >> 11) < ceil(exp(-d / t) * 2^53), tabulated on the host
// with libm exp, the function the reference calls.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/ising_b200.h"
#include "ie_device.cuh"
#include "ie_host.h"

using namespace ie;

namespace {

struct V2Dev {
    uint32_t n, r, w, w2;  // sites, replicas, u64 words per site, u32 words per site
    const uint32_t* row;
    const uint32_t* col;
    const int32_t* wt;
    const int32_t* lin;
    const uint32_t* order;  // chromatic order (position -> site)
    uint64_t* spins;
    unsigned long long* energies;  // int64 per replica
    unsigned long long* counter;   // accepted moves
    // Metropolis thresholds per temperature index ti = replica % n_temps
    const uint64_t* thr;
    const uint64_t* thr_off;
    const uint64_t* thr_max;
    const uint64_t* thr_und;
    uint32_t n_temps;
    // exchange tables per pair (k, k+1)
    const uint64_t* xtab;
    const uint64_t* xoff;
    const uint64_t* xdmax;
    const uint64_t* xdund;
    const double* dbeta;
    uint64_t* pmask;  // bit k: pair (k, k+1) swapped in this round
};

struct Key {
    uint32_t k[8];
};

// One colour of one sweep: warp = (32-replica group g = blockIdx.y, positions
// strided over the grid).
__global__ void __launch_bounds__(128) v2_metropolis_color(V2Dev D, Key key, uint32_t p_begin, uint32_t p_end,
                                                           uint64_t draw0) {
    const uint32_t g = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t rep = g * 32 + lane;
    const bool valid = rep < D.r;
    const uint32_t* planes = reinterpret_cast<const uint32_t*>(D.spins);
    uint32_t* own = reinterpret_cast<uint32_t*>(D.spins);
    const uint32_t ti = valid ? rep % D.n_temps : 0;
    const uint64_t t_off = D.thr_off[ti], t_max = D.thr_max[ti], t_und = D.thr_und[ti];
    long long eacc = 0;
    unsigned long long acc_count = 0;
    for (uint32_t p = p_begin + warp; p < p_end; p += nwarps) {
        const uint32_t site = D.order[p];
        int32_t h = D.lin[site];
        const uint32_t e1 = D.row[site + 1];
        for (uint32_t e = D.row[site]; e < e1; e++) {
            const uint32_t word = planes[(size_t)D.col[e] * D.w2 + g];
            h += ((word >> lane) & 1u) ? D.wt[e] : 0;
        }
        const uint32_t ownw = planes[(size_t)site * D.w2 + g];
        const int32_t d = ((ownw >> lane) & 1u) ? -h : h;
        bool accept = false;
        if (valid) {
            if (d <= 0) {
                accept = true;  // the draw is consumed but not needed
            } else {
                const uint64_t ad = (uint64_t)d;
                const uint64_t th = ad <= t_max ? D.thr[t_off + ad - 1] : (ad <= t_und ? 1ull : 0ull);
                if (th) {
                    const uint64_t u = chacha8_draw(key.k, draw0 + (uint64_t)p * D.r + rep) >> 11;
                    accept = u < th;
                }
            }
        }
        const uint32_t mask = __ballot_sync(0xffffffffu, accept);
        if (lane == 0) {
            own[(size_t)site * D.w2 + g] = ownw ^ mask;
            acc_count += __popc(mask);
        }
        if (accept) eacc += d;
    }
    if (valid && eacc) atomicAdd(D.energies + rep, (unsigned long long)eacc);
    if (lane == 0 && acc_count) atomicAdd(D.counter, acc_count);
}

// GibbsColorSweep thresholds of one temperature: P(x = 1) = 1 / (1 + exp(b h))
// as ceil(P * 2^53) for integer fields h, so that u < P <=> (draw >> 11) < T.
struct GParam {
    int64_t lo;      // field of tab entry 0
    uint64_t off;    // first entry in the table
    uint64_t len;    // entries
    uint64_t below;  // T for h < lo
    uint64_t above;  // T for lo + len <= h <= und
    int64_t und;     // h > und: P == 0, T == 0
};

__device__ __forceinline__ uint64_t gibbs_threshold(const GParam& P, const uint64_t* tab, int32_t h) {
    const int64_t rel = (int64_t)h - P.lo;
    if (rel < 0) return P.below;
    if ((uint64_t)rel < P.len) return tab[P.off + rel];
    return h <= P.und ? P.above : 0ull;
}

// One colour of one Gibbs sweep, same decomposition as v2_metropolis_color:
// replica's new spin is 1 iff its draw is below the threshold of its field.
__global__ void __launch_bounds__(128) v2_gibbs_color(V2Dev D, const GParam* gp, const uint64_t* gtab, Key key,
                                                      uint32_t p_begin, uint32_t p_end, uint64_t draw0) {
    const uint32_t g = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t rep = g * 32 + lane;
    const bool valid = rep < D.r;
    const uint32_t* planes = reinterpret_cast<const uint32_t*>(D.spins);
    uint32_t* own = reinterpret_cast<uint32_t*>(D.spins);
    GParam P = gp[valid ? rep % D.n_temps : 0];
    constexpr uint64_t kOne = 1ull << 53;
    long long eacc = 0;
    unsigned long long acc_count = 0;
    for (uint32_t p = p_begin + warp; p < p_end; p += nwarps) {
        const uint32_t site = D.order[p];
        int32_t h = D.lin[site];
        const uint32_t e1 = D.row[site + 1];
        for (uint32_t e = D.row[site]; e < e1; e++) {
            const uint32_t word = planes[(size_t)D.col[e] * D.w2 + g];
            h += ((word >> lane) & 1u) ? D.wt[e] : 0;
        }
        const uint32_t ownw = planes[(size_t)site * D.w2 + g];
        const bool x = (ownw >> lane) & 1u;
        bool flip = false;
        if (valid) {
            const uint64_t th = gibbs_threshold(P, gtab, h);
            // u < 1 always: T == 2^53 needs no draw, nor T == 0
            const bool one = th >= kOne ? true
                             : (th == 0 ? false : (chacha8_draw(key.k, draw0 + (uint64_t)p * D.r + rep) >> 11) < th);
            flip = one != x;
        }
        const uint32_t mask = __ballot_sync(0xffffffffu, flip);
        if (lane == 0) {
            own[(size_t)site * D.w2 + g] = ownw ^ mask;
            acc_count += __popc(mask);
        }
        if (flip) eacc += x ? -h : h;
    }
    if (valid && eacc) atomicAdd(D.energies + rep, (unsigned long long)eacc);
    if (lane == 0 && acc_count) atomicAdd(D.counter, acc_count);
}

// Host tables for v2_gibbs_color. For t > 0 the fields |h| <= 40 t + 1 are
// tabulated with libm exp (the reference's function); beyond, exp(h / t) is
// below 2^-54 (P rounds to 1, T = 2^53) or above 2^57 (0 < P < 2^-53, T = 1)
// until exp overflows (P = 0). t <= 0 or NaN: bh = sign(h) * inf, the
// reference's greedy limit (P = 0, 1/2, 1); t = +inf: bh = 0, P = 1/2.
ie_status gibbs_tables(const double* temps, uint32_t nt, int64_t hb, std::vector<GParam>& P,
                       std::vector<uint64_t>& tab) {
    constexpr uint64_t kOne = 1ull << 53;
    P.assign(nt, GParam{});
    tab.clear();
    for (uint32_t ti = 0; ti < nt; ti++) {
        const double t = temps[ti];
        GParam& g = P[ti];
        g.off = tab.size();
        if (!(t > 0.0)) {
            g.lo = 0;
            g.len = 1;
            tab.push_back(kOne / 2);
            g.below = kOne;
            g.above = 0;
            g.und = 0;
            continue;
        }
        if (std::isinf(t)) {
            g.lo = hb + 1;
            g.len = 0;
            g.below = kOne / 2;
            g.above = 0;
            g.und = hb;
            continue;
        }
        const double m = std::ceil(40.0 * t) + 1.0;
        const int64_t hi = m >= (double)hb ? hb : (int64_t)m;
        g.lo = -hi;
        g.len = (uint64_t)(2 * hi + 1);
        if (tab.size() + g.len > (1u << 24)) return fail(IE_ERR_UNSUPPORTED, "temperatures too high for the threshold tables");
        for (int64_t h = -hi; h <= hi; h++)
            tab.push_back((uint64_t)std::ceil(std::ldexp(1.0 / (1.0 + std::exp((double)h / t)), 53)));
        g.below = kOne;
        g.above = 1;
        int64_t a = hi, b = hb + 1;  // largest h <= hb with exp(h / t) finite
        if (std::isinf(std::exp((double)hi / t))) b = hi + 1;
        while (b - a > 1) {
            const int64_t mid = a + (b - a) / 2;
            if (std::isfinite(std::exp((double)mid / t))) a = mid;
            else b = mid;
        }
        g.und = a;
    }
    return IE_OK;
}

// One exchange round's decisions: pairs (k, k+1), k = start, start + 2, ...;
// pair p takes draw draw0 + p. Energies of swapped pairs are exchanged and
// the pair's bit set in pmask for v2_swap_pairs.
__global__ void __launch_bounds__(256) v2_exchange_round(V2Dev D, Key key, uint32_t start, uint64_t draw0) {
    for (uint32_t q = threadIdx.x; q < D.w; q += blockDim.x) D.pmask[q] = 0;
    __syncthreads();
    const uint32_t np = (D.r - start) / 2;
    unsigned long long acc_count = 0;
    long long* E = reinterpret_cast<long long*>(D.energies);
    for (uint32_t p = threadIdx.x; p < np; p += blockDim.x) {
        const uint32_t k = start + 2 * p;
        const double de = __dsub_rn((double)E[k], (double)E[k + 1]);
        const double ex = __dmul_rn(D.dbeta[k], de);
        bool accept = ex >= 0.0;
        if (!accept) {
            const uint64_t ad = (uint64_t)fabs(de);
            const uint64_t th = ad <= D.xdmax[k] ? D.xtab[D.xoff[k] + ad - 1] : (ad <= D.xdund[k] ? 1ull : 0ull);
            accept = th && (chacha8_draw(key.k, draw0 + p) >> 11) < th;
        }
        if (accept) {
            const long long t = E[k];
            E[k] = E[k + 1];
            E[k + 1] = t;
            atomicOr(reinterpret_cast<unsigned long long*>(D.pmask + k / 64), 1ull << (k % 64));
            acc_count++;
        }
    }
    if (acc_count) atomicAdd(D.counter, acc_count);
}

// swap_replicas (state.rs:126-140) for every swapped pair at every site: the
// two replicas' bits exchange.
__global__ void v2_swap_pairs(V2Dev D) {
    for (size_t site = (size_t)blockIdx.x * blockDim.x + threadIdx.x; site < D.n; site += (size_t)gridDim.x * blockDim.x) {
        uint64_t* s = D.spins + site * D.w;
        for (uint32_t q = 0; q < D.w; q++) {
            const uint64_t m = D.pmask[q] & 0x7FFFFFFFFFFFFFFFull;  // pairs inside word q
            if (!m) continue;
            const uint64_t x = s[q];
            const uint64_t d = ((x >> 1) ^ x) & m;
            s[q] = x ^ (d | (d << 1));
        }
        for (uint32_t q = 0; q + 1 < D.w; q++) {
            if (!(D.pmask[q] >> 63)) continue;  // pair (64q + 63, 64q + 64) across words
            const uint64_t x = s[q], y = s[q + 1];
            if (((x >> 63) ^ y) & 1u) {
                s[q] = x ^ (1ull << 63);
                s[q + 1] = y ^ 1ull;
            }
        }
    }
}

// ProblemIR::greedy_coloring (src/engine_v2/ir.rs:114-139): site i takes the
// smallest colour not used by an already-coloured neighbour.
std::vector<uint32_t> greedy_coloring(uint32_t n, const std::vector<uint32_t>& row, const std::vector<uint32_t>& col) {
    std::vector<uint32_t> colors(n, 0xFFFFFFFFu), used;
    for (uint32_t i = 0; i < n; i++) {
        used.clear();
        for (uint32_t e = row[i]; e < row[i + 1]; e++)
            if (colors[col[e]] != 0xFFFFFFFFu) used.push_back(colors[col[e]]);
        std::sort(used.begin(), used.end());
        uint32_t c = 0;
        for (uint32_t u : used) {
            if (u == c) c++;
            else if (u > c) break;
        }
        colors[i] = c;
    }
    return colors;
}

}  // namespace

struct ie_v2 {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t n = 0, r = 0, w = 0;
    int64_t offset = 0;
    int64_t hbound = 0;
    std::vector<uint32_t> row, col, order, color_off;
    std::vector<int32_t> wt, lin;
    DevBuf<uint32_t> d_row, d_col, d_order;
    DevBuf<int32_t> d_wt, d_lin;
    DevBuf<uint64_t> d_spins, d_thr, d_thr_off, d_thr_max, d_thr_und, d_xtab, d_xoff, d_xdmax, d_xdund, d_pmask;
    DevBuf<double> d_dbeta;
    DevBuf<GParam> d_gp;
    DevBuf<uint64_t> d_gtab;
    DevBuf<unsigned long long> d_E, d_cnt;

    ~ie_v2() {
        if (stream) cudaStreamDestroy(stream);
    }

    V2Dev dev() const {
        V2Dev D{};
        D.n = n;
        D.r = r;
        D.w = w;
        D.w2 = 2 * w;
        D.row = d_row.p;
        D.col = d_col.p;
        D.wt = d_wt.p;
        D.lin = d_lin.p;
        D.order = d_order.p;
        D.spins = d_spins.p;
        D.energies = d_E.p;
        D.counter = d_cnt.p;
        D.thr = d_thr.p;
        D.thr_off = d_thr_off.p;
        D.thr_max = d_thr_max.p;
        D.thr_und = d_thr_und.p;
        D.xtab = d_xtab.p;
        D.xoff = d_xoff.p;
        D.xdmax = d_xdmax.p;
        D.xdund = d_xdund.p;
        D.dbeta = d_dbeta.p;
        D.pmask = d_pmask.p;
        return D;
    }

    // SparseBitSlice::energy_of (sparse_bitslice.rs:116-137) from the host copy of the planes.
    std::vector<int64_t> energies_from(const std::vector<uint64_t>& s) const {
        std::vector<int64_t> E(r, 0);
        for (uint32_t rep = 0; rep < r; rep++) {
            int64_t l = 0, q = 0;
            auto bit = [&](uint32_t site) { return (s[(size_t)site * w + rep / 64] >> (rep % 64)) & 1u; };
            for (uint32_t i = 0; i < n; i++) {
                if (!bit(i)) continue;
                l += lin[i];
                for (uint32_t e = row[i]; e < row[i + 1]; e++)
                    if (bit(col[e])) q += wt[e];
            }
            E[rep] = offset + l + q / 2;
        }
        return E;
    }

    ie_status create(const ie_problem* p, uint32_t num_replicas, const uint8_t* init, int32_t dev) {
        if (!p || !init) return fail(IE_ERR_INVALID, "NULL argument");
        if (num_replicas == 0) return fail(IE_ERR_INVALID, "num_replicas must be >= 1");
        if (p->num_vars == 0 || p->num_vars >= (1ull << 31)) return fail(IE_ERR_INVALID, "num_vars out of range");
        if (!p->linear || !p->row_offsets) return fail(IE_ERR_INVALID, "linear/row_offsets must be non-NULL");
        n = (uint32_t)p->num_vars;
        r = num_replicas;
        w = (r + 63) / 64;
        const uint64_t nnz = p->row_offsets[n];
        if (nnz && (!p->col_indices || !p->values)) return fail(IE_ERR_INVALID, "col_indices/values must be non-NULL");
        if (nnz >= (1ull << 32)) return fail(IE_ERR_INVALID, "too many couplings");
        // SparseBitSlice::new: integral instances only (is_integral, ir.rs:143-148)
        auto intish = [](double v) { return std::isfinite(v) && v == std::trunc(v); };
        if (!intish(p->energy_offset)) return fail(IE_ERR_INVALID, "the bit-sliced state requires integral couplings");
        offset = (int64_t)p->energy_offset;
        row.resize(n + 1);
        col.resize(nnz);
        wt.resize(nnz);
        lin.resize(n);
        hbound = 0;
        for (uint32_t i = 0; i <= n; i++) row[i] = (uint32_t)p->row_offsets[i];
        for (uint32_t i = 0; i < n; i++) {
            if (!intish(p->linear[i])) return fail(IE_ERR_INVALID, "the bit-sliced state requires integral couplings");
            if (row[i + 1] < row[i]) return fail(IE_ERR_INVALID, "row_offsets must be non-decreasing");
            double b = std::fabs(p->linear[i]);
            for (uint32_t e = row[i]; e < row[i + 1]; e++) {
                const double v = p->values[e];
                if (!intish(v)) return fail(IE_ERR_INVALID, "the bit-sliced state requires integral couplings");
                if (p->col_indices[e] >= n) return fail(IE_ERR_INVALID, "column index out of range");
                b += std::fabs(v);
            }
            if (b >= 2147483647.0) return fail(IE_ERR_UNSUPPORTED, "local fields exceed 32 bits");
            hbound = std::max<int64_t>(hbound, (int64_t)b);
            lin[i] = (int32_t)p->linear[i];
        }
        for (uint64_t e = 0; e < nnz; e++) {
            col[e] = (uint32_t)p->col_indices[e];
            wt[e] = (int32_t)p->values[e];
        }
        const std::vector<uint32_t> colors = greedy_coloring(n, row, col);
        uint32_t ncol = 0;
        for (uint32_t c : colors) ncol = std::max(ncol, c + 1);
        color_off.assign(ncol + 1, 0);
        order.clear();
        for (uint32_t c = 0; c < ncol; c++) {
            color_off[c] = (uint32_t)order.size();
            for (uint32_t i = 0; i < n; i++)
                if (colors[i] == c) order.push_back(i);
        }
        color_off[ncol] = (uint32_t)order.size();
        // planes: every replica starts from init (sparse_bitslice.rs:52-66)
        std::vector<uint64_t> s((size_t)n * w, 0);
        for (uint32_t i = 0; i < n; i++)
            if (init[i] & 1u)
                for (uint32_t q = 0; q < w; q++) {
                    const uint32_t valid = std::min<uint32_t>(r - 64 * q, 64);
                    s[(size_t)i * w + q] = valid == 64 ? ~0ull : ((1ull << valid) - 1);
                }
        const std::vector<int64_t> E = energies_from(s);
        std::vector<unsigned long long> Eu(E.begin(), E.end());
        device = dev;
        int ndev = 0;
        IE_CUDA(cudaGetDeviceCount(&ndev));
        if (dev < 0 || dev >= ndev) return fail(IE_ERR_INVALID, "invalid CUDA device ordinal");
        IE_CUDA(cudaSetDevice(dev));
        IE_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        IE_TRY(d_row.upload(row, stream));
        IE_TRY(d_col.upload(col.empty() ? std::vector<uint32_t>(1, 0) : col, stream));
        IE_TRY(d_wt.upload(wt.empty() ? std::vector<int32_t>(1, 0) : wt, stream));
        IE_TRY(d_lin.upload(lin, stream));
        IE_TRY(d_order.upload(order, stream));
        IE_TRY(d_spins.upload(s, stream));
        IE_TRY(d_E.upload(Eu, stream));
        IE_TRY(d_cnt.alloc(1));
        IE_TRY(d_pmask.alloc(w));
        IE_CUDA(cudaStreamSynchronize(stream));
        return IE_OK;
    }

    ie_status metropolis(const double* temps, uint32_t nt, uint64_t sweeps, uint64_t seed, uint64_t draw_offset,
                         uint64_t* proposed, uint64_t* accepted) {
        if (!temps || nt == 0) return fail(IE_ERR_INVALID, "MetropolisSweep needs a temperature");
        // thresholds per temperature: ceil(exp(-d / t) * 2^53) for d = 1..
        std::vector<uint64_t> thr, off(nt), dmax(nt), dund(nt);
        for (uint32_t ti = 0; ti < nt; ti++) {
            const double t = temps[ti];
            if (std::isnan(t)) return fail(IE_ERR_INVALID, "temperature is NaN");
            off[ti] = thr.size();
            if (!(t > 0.0)) {  // T <= 0: pure descent, uphill never accepted
                dmax[ti] = dund[ti] = 0;
                continue;
            }
            uint64_t d = 1;
            for (; d <= (uint64_t)hbound; d++) {
                const double T = std::ceil(std::ldexp(std::exp(-(double)d / t), 53));
                if (T <= 1.0) break;
                thr.push_back((uint64_t)T);
                if (thr.size() > (1u << 24)) return fail(IE_ERR_UNSUPPORTED, "temperatures too high for the threshold tables");
            }
            dmax[ti] = d - 1;
            uint64_t lo = d - 1, hi = (uint64_t)hbound + 1;
            while (hi - lo > 1) {  // largest d <= hbound with exp(-d/t) > 0
                const uint64_t mid = lo + (hi - lo) / 2;
                if (std::exp(-(double)mid / t) > 0.0) lo = mid;
                else hi = mid;
            }
            dund[ti] = lo;
        }
        IE_CUDA(cudaSetDevice(device));
        IE_TRY(d_thr.upload(thr.empty() ? std::vector<uint64_t>(1, 0) : thr, stream));
        IE_TRY(d_thr_off.upload(off, stream));
        IE_TRY(d_thr_max.upload(dmax, stream));
        IE_TRY(d_thr_und.upload(dund, stream));
        IE_CUDA(cudaMemsetAsync(d_cnt.p, 0, sizeof(unsigned long long), stream));
        Key key;
        chacha_key_from_u64(seed, key.k);
        V2Dev D = dev();
        D.n_temps = nt;
        const uint32_t ng = (r + 31) / 32;
        if (ng > 65535) return fail(IE_ERR_UNSUPPORTED, "too many replicas");
        for (uint64_t sw = 0; sw < sweeps; sw++) {
            const uint64_t draw0 = draw_offset + sw * (uint64_t)n * r;
            for (size_t c = 0; c + 1 < color_off.size(); c++) {
                const uint32_t cnt = color_off[c + 1] - color_off[c];
                const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>((cnt + 3) / 4, 1184 / ng + 1));
                v2_metropolis_color<<<dim3(blocks, ng), 128, 0, stream>>>(D, key, color_off[c], color_off[c + 1], draw0);
                IE_CUDA(cudaGetLastError());
            }
        }
        unsigned long long a = 0;
        IE_CUDA(cudaMemcpyAsync(&a, d_cnt.p, sizeof(a), cudaMemcpyDeviceToHost, stream));
        IE_CUDA(cudaStreamSynchronize(stream));
        if (proposed) *proposed = sweeps * (uint64_t)n * r;
        if (accepted) *accepted = a;
        return IE_OK;
    }

    ie_status gibbs(const double* temps, uint32_t nt, uint64_t sweeps, uint64_t seed, uint64_t draw_offset,
                    uint64_t* proposed, uint64_t* accepted) {
        if (!temps || nt == 0) return fail(IE_ERR_INVALID, "GibbsColorSweep needs a temperature");
        std::vector<GParam> gp;
        std::vector<uint64_t> gtab;
        IE_TRY(gibbs_tables(temps, nt, hbound, gp, gtab));
        IE_CUDA(cudaSetDevice(device));
        IE_TRY(d_gp.upload(gp, stream));
        IE_TRY(d_gtab.upload(gtab.empty() ? std::vector<uint64_t>(1, 0) : gtab, stream));
        IE_CUDA(cudaMemsetAsync(d_cnt.p, 0, sizeof(unsigned long long), stream));
        Key key;
        chacha_key_from_u64(seed, key.k);
        V2Dev D = dev();
        D.n_temps = nt;
        const uint32_t ng = (r + 31) / 32;
        if (ng > 65535) return fail(IE_ERR_UNSUPPORTED, "too many replicas");
        for (uint64_t sw = 0; sw < sweeps; sw++) {
            const uint64_t draw0 = draw_offset + sw * (uint64_t)n * r;
            for (size_t c = 0; c + 1 < color_off.size(); c++) {
                const uint32_t cnt = color_off[c + 1] - color_off[c];
                const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>((cnt + 3) / 4, 1184 / ng + 1));
                v2_gibbs_color<<<dim3(blocks, ng), 128, 0, stream>>>(D, d_gp.p, d_gtab.p, key, color_off[c],
                                                                    color_off[c + 1], draw0);
                IE_CUDA(cudaGetLastError());
            }
        }
        unsigned long long a = 0;
        IE_CUDA(cudaMemcpyAsync(&a, d_cnt.p, sizeof(a), cudaMemcpyDeviceToHost, stream));
        IE_CUDA(cudaStreamSynchronize(stream));
        if (proposed) *proposed = sweeps * (uint64_t)n * r;
        if (accepted) *accepted = a;
        return IE_OK;
    }

    ie_status exchange(const double* temps, uint32_t nt, uint64_t rounds, uint64_t seed, uint64_t draw_offset,
                       uint64_t* proposed, uint64_t* accepted) {
        if (proposed) *proposed = 0;
        if (accepted) *accepted = 0;
        if (r < 2 || nt == 0 || !temps) return IE_OK;  // replica_exchange.rs:69-71
        std::vector<double> ladder(r);
        for (uint32_t k = 0; k < r; k++) {
            ladder[k] = temps[k % nt];
            if (!(ladder[k] > 0.0) || !std::isfinite(ladder[k]))
                return fail(IE_ERR_INVALID, "exchange temperatures must be positive and finite");
        }
        XTables X;
        IE_TRY(build_xtables(ladder.data(), r, X));
        IE_CUDA(cudaSetDevice(device));
        IE_TRY(d_xtab.upload(X.tab.empty() ? std::vector<uint64_t>(1, 0) : X.tab, stream));
        IE_TRY(d_xoff.upload(X.off, stream));
        IE_TRY(d_xdmax.upload(X.dmax, stream));
        IE_TRY(d_xdund.upload(X.dund, stream));
        IE_TRY(d_dbeta.upload(X.dbeta, stream));
        IE_CUDA(cudaMemsetAsync(d_cnt.p, 0, sizeof(unsigned long long), stream));
        Key key;
        chacha_key_from_u64(seed, key.k);
        const V2Dev D = dev();
        uint64_t draws = 0;
        const int sgrid = (int)std::min<uint32_t>((n + 255) / 256, 1184);
        for (uint64_t round = 0; round < rounds; round++) {
            const uint32_t start = (uint32_t)(round & 1);
            v2_exchange_round<<<1, 256, 0, stream>>>(D, key, start, draw_offset + draws);
            IE_CUDA(cudaGetLastError());
            v2_swap_pairs<<<std::max(sgrid, 1), 256, 0, stream>>>(D);
            IE_CUDA(cudaGetLastError());
            draws += (r - start) / 2;
        }
        unsigned long long a = 0;
        IE_CUDA(cudaMemcpyAsync(&a, d_cnt.p, sizeof(a), cudaMemcpyDeviceToHost, stream));
        IE_CUDA(cudaStreamSynchronize(stream));
        if (proposed) *proposed = draws;
        if (accepted) *accepted = a;
        return IE_OK;
    }

    ie_status read(uint64_t* planes, double* energies) {
        IE_CUDA(cudaSetDevice(device));
        std::vector<unsigned long long> E(r);
        if (planes)
            IE_CUDA(cudaMemcpyAsync(planes, d_spins.p, (size_t)n * w * 8, cudaMemcpyDeviceToHost, stream));
        IE_CUDA(cudaMemcpyAsync(E.data(), d_E.p, (size_t)r * 8, cudaMemcpyDeviceToHost, stream));
        IE_CUDA(cudaStreamSynchronize(stream));
        if (energies)
            for (uint32_t k = 0; k < r; k++) energies[k] = (double)(long long)E[k];
        return IE_OK;
    }

    // SparseBitSlice::audit (sparse_bitslice.rs:317-346): largest |ledger -
    // recomputed| energy (the gathered fields have no ledger to drift).
    ie_status audit(double* drift) {
        std::vector<uint64_t> s((size_t)n * w);
        std::vector<double> E(r);
        IE_TRY(read(s.data(), E.data()));
        const std::vector<int64_t> F = energies_from(s);
        int64_t dmax = 0;
        for (uint32_t k = 0; k < r; k++) dmax = std::max<int64_t>(dmax, std::llabs((long long)E[k] - F[k]));
        *drift = (double)dmax;
        return IE_OK;
    }
};

extern "C" {

ie_status ie_v2_create(const ie_problem* ir, uint32_t num_replicas, const uint8_t* init, int32_t device,
                       ie_v2** out) {
    if (!out) return fail(IE_ERR_INVALID, "out is NULL");
    *out = nullptr;
    std::unique_ptr<ie_v2> h(new ie_v2());
    IE_TRY(h->create(ir, num_replicas, init, device));
    *out = h.release();
    return IE_OK;
}

ie_status ie_v2_destroy(ie_v2* h) {
    delete h;
    return IE_OK;
}

ie_status ie_v2_metropolis(ie_v2* h, const double* temps, uint32_t n_temps, uint64_t sweeps, uint64_t seed,
                           uint64_t draw_offset, uint64_t* proposed, uint64_t* accepted) {
    if (!h) return fail(IE_ERR_INVALID, "handle is NULL");
    return h->metropolis(temps, n_temps, sweeps, seed, draw_offset, proposed, accepted);
}

ie_status ie_v2_gibbs(ie_v2* h, const double* temps, uint32_t n_temps, uint64_t sweeps, uint64_t seed,
                      uint64_t draw_offset, uint64_t* proposed, uint64_t* accepted) {
    if (!h) return fail(IE_ERR_INVALID, "handle is NULL");
    return h->gibbs(temps, n_temps, sweeps, seed, draw_offset, proposed, accepted);
}

ie_status ie_v2_exchange(ie_v2* h, const double* temps, uint32_t n_temps, uint64_t rounds, uint64_t seed,
                         uint64_t draw_offset, uint64_t* proposed, uint64_t* accepted) {
    if (!h) return fail(IE_ERR_INVALID, "handle is NULL");
    return h->exchange(temps, n_temps, rounds, seed, draw_offset, proposed, accepted);
}

ie_status ie_v2_read(ie_v2* h, uint64_t* planes, double* energies) {
    if (!h) return fail(IE_ERR_INVALID, "handle is NULL");
    return h->read(planes, energies);
}

ie_status ie_v2_audit(ie_v2* h, double* drift) {
    if (!h || !drift) return fail(IE_ERR_INVALID, "NULL argument");
    return h->audit(drift);
}

ie_status ie_v2_coloring(const ie_problem* ir, uint32_t* colors) {
    if (!ir || !colors || !ir->row_offsets) return fail(IE_ERR_INVALID, "NULL argument");
    const uint32_t n = (uint32_t)ir->num_vars;
    std::vector<uint32_t> row(n + 1), col(n ? ir->row_offsets[n] : 0);
    for (uint32_t i = 0; i <= n; i++) row[i] = (uint32_t)ir->row_offsets[i];
    for (size_t e = 0; e < col.size(); e++) col[e] = (uint32_t)ir->col_indices[e];
    const std::vector<uint32_t> c = greedy_coloring(n, row, col);
    std::copy(c.begin(), c.end(), colors);
    return IE_OK;
}

}  // extern "C"
