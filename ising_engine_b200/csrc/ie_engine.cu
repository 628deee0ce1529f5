// Host side of the B200 engine: problem ingestion, device memory, launch
// orchestration and the C ABI declared in include/ising_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/ising_b200.h"
#include "ie_device.cuh"
#include "ie_host.h"
#include "ie_launch.h"
#include "ie_level_host.h"

using namespace ie;

namespace ie {

thread_local std::string g_err;

ie_status fail(ie_status s, const std::string& msg) {
    g_err = msg;
    return s;
}

// rand_core 0.6.4 SeedableRng::seed_from_u64: PCG32 outputs fill the 32-byte
// ChaCha8 key (little-endian), as ChaCha8Rng::seed_from_u64 (ultimate.rs:152).
void chacha_key_from_u64(uint64_t state, uint32_t key[8]) {
    const uint64_t mul = 6364136223846793005ULL, inc = 11634580027462260723ULL;
    for (int i = 0; i < 8; i++) {
        state = state * mul + inc;
        const uint32_t xs = (uint32_t)(((state >> 18) ^ state) >> 27);
        const uint32_t rot = (uint32_t)(state >> 59);
        key[i] = (xs >> rot) | (xs << ((32 - rot) & 31));
    }
}

// Exchange thresholds for the integer mode (engine.rs:725-727): for the pair
// (t, t+1) with db = 1/T_t - 1/T_{t+1}, a swap with exponent db*de < 0 is
// accepted iff gen::<f64>() < exp(db*de), i.e. iff (draw >> 11) <
// ceil(exp(db*de) * 2^53), which depends only on |de|. Built with the host
// libm exp, the same function the reference calls.
ie_status build_xtables(const double* temps, uint32_t nt, XTables& X) {
    X = XTables();
    const uint32_t np = nt > 1 ? nt - 1 : 0;
    X.off.resize(std::max<uint32_t>(np, 1));
    X.dmax.resize(std::max<uint32_t>(np, 1));
    X.dund.resize(std::max<uint32_t>(np, 1));
    X.dbeta.resize(std::max<uint32_t>(np, 1));
    for (uint32_t t = 0; t < np; t++) {
        const double b1 = 1.0 / temps[t], b2 = 1.0 / temps[t + 1];
        const double db = b1 - b2;
        X.dbeta[t] = db;
        X.off[t] = X.tab.size();
        const double adb = std::fabs(db);
        if (!(adb > 0.0) || !std::isfinite(adb)) {
            X.dmax[t] = 0;
            X.dund[t] = 0;
            continue;
        }
        uint64_t a = 1;
        for (;; a++) {
            const double ex = -(adb * (double)a);
            const double T = std::ceil(std::ldexp(std::exp(ex), 53));
            if (T <= 1.0) break;
            X.tab.push_back((uint64_t)T);
            if (X.tab.size() > (1u << 24))
                return fail(IE_ERR_UNSUPPORTED, "temperature ladder too fine for the integer exchange tables");
        }
        X.dmax[t] = a - 1;
        // largest |de| with exp(-adb*|de|) > 0 (monotone), by bisection
        uint64_t lo = a - 1, hi = (uint64_t)std::min(1e18, std::ceil(800.0 / adb) + 2.0);
        while (hi - lo > 1) {
            const uint64_t mid = lo + (hi - lo) / 2;
            if (std::exp(-(adb * (double)mid)) > 0.0) lo = mid;
            else hi = mid;
        }
        X.dund[t] = lo;
    }
    return IE_OK;
}

}  // namespace ie

namespace {

// Runs fn(i) for every i in [0, count) on up to 32 host threads, in chunks of
// 16 indices handed out in order.
template <typename F>
void parallel_for(uint32_t count, F&& fn) {
    const unsigned nth = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
    if (count < 64 || nth == 1) {
        for (uint32_t i = 0; i < count; i++) fn(i);
        return;
    }
    std::atomic<uint32_t> next{0};
    auto work = [&]() {
        for (;;) {
            const uint32_t i0 = next.fetch_add(16);
            if (i0 >= count) break;
            for (uint32_t i = i0; i < std::min(i0 + 16, count); i++) fn(i);
        }
    };
    std::vector<std::thread> ts;
    for (unsigned k = 1; k < nth; k++) ts.emplace_back(work);
    work();
    for (auto& t : ts) t.join();
}

// f64::powi for a runtime exponent lowers to compiler-rt's __powidf2.
double powi_rt(double a, int b) {
    const bool recip = b < 0;
    double r = 1.0;
    for (;;) {
        if (b & 1) r *= a;
        b /= 2;
        if (b == 0) break;
        a *= a;
    }
    return recip ? 1.0 / r : r;
}

// One ingested problem (both triangles, reference row order).
struct HostInst {
    uint32_t n = 0;
    int32_t H = 0;
    uint32_t mode = kModeF64;
    double offset = 0.0;
    std::vector<uint32_t> rows;   // n + 1
    std::vector<uint32_t> ents;   // integer mode packed entries
    std::vector<int32_t> linp;
    std::vector<uint32_t> cols;
    std::vector<double> vals;
    std::vector<double> lin;
    std::vector<uint32_t> recpos, reclen;  // first record of each site: word offset and length in its stream
    uint32_t pmj = 0;                      // +-J form for the level kernel: c | D << 16 (0: not)
    bool windowed_ok = false;              // the windowed kernel is preferred (parallel windows)
    bool has_wtab = false;                 // has a window table (the windowed kernel can run it)
    uint64_t nnz = 0;
};

ie_status ingest(const ie_problem* p, bool force_f64, HostInst& out) {
    if (!p) return fail(IE_ERR_INVALID, "problem is NULL");
    const uint64_t n = p->num_vars;
    if (n >= (1ULL << 31)) return fail(IE_ERR_INVALID, "num_vars too large");
    if (n > 0 && (!p->linear || !p->row_offsets))
        return fail(IE_ERR_INVALID, "linear/row_offsets must be non-NULL");
    const uint64_t nnz = n ? p->row_offsets[n] : 0;
    if (n && p->row_offsets[0] != 0) return fail(IE_ERR_INVALID, "row_offsets[0] must be 0");
    if (nnz >= (1ULL << 32)) return fail(IE_ERR_INVALID, "too many couplings");
    if (nnz && (!p->col_indices || !p->values)) return fail(IE_ERR_INVALID, "col_indices/values must be non-NULL");
    out.n = (uint32_t)n;
    out.nnz = nnz;
    out.offset = p->energy_offset;
    out.rows.resize(n + 1);
    out.lin.assign(p->linear, p->linear + n);
    out.cols.resize(nnz);
    out.vals.assign(p->values, p->values + nnz);
    for (uint64_t i = 0; i <= n; i++) {
        if (i && p->row_offsets[i] < p->row_offsets[i - 1])
            return fail(IE_ERR_INVALID, "row_offsets must be non-decreasing");
        out.rows[i] = (uint32_t)p->row_offsets[i];
    }
    for (uint64_t k = 0; k < nnz; k++) {
        if (p->col_indices[k] >= n) return fail(IE_ERR_INVALID, "column index out of range");
        if (!std::isfinite(p->values[k])) return fail(IE_ERR_INVALID, "non-finite coupling");
        out.cols[k] = (uint32_t)p->col_indices[k];
    }
    for (uint64_t i = 0; i < n; i++)
        if (!std::isfinite(p->linear[i])) return fail(IE_ERR_INVALID, "non-finite linear term");

    // Integer mode: integral values, |w| <= 127, |local field| <= 127 at every
    // site, tracked energies within int32 and columns within 24 bits.
    bool integral = !force_f64 && n < (1u << 24);
    double ebound = 0.0;
    int32_t H = 0;
    std::vector<int32_t> linp(n);
    for (uint64_t i = 0; integral && i < n; i++) {
        const double l = p->linear[i];
        if (l != std::trunc(l) || std::fabs(l) > 127.0) {
            integral = false;
            break;
        }
        double neg = 0.0, pos = 0.0;
        for (uint64_t k = p->row_offsets[i]; k < p->row_offsets[i + 1]; k++) {
            const double w = p->values[k];
            if (w != std::trunc(w) || std::fabs(w) > 127.0) {
                integral = false;
                break;
            }
            if (w < 0) neg += w;
            else pos += w;
            if (p->col_indices[k] > i) ebound += std::fabs(w);
        }
        if (!integral) break;
        const double hlo = l + neg, hhi = l + pos;
        const double hv = std::max(std::fabs(hlo), std::fabs(hhi));
        if (hv > (double)kMaxH) {
            integral = false;
            break;
        }
        H = std::max(H, (int32_t)hv);
        linp[i] = (int32_t)hlo;
        ebound += std::fabs(l);
    }
    if (integral && ebound >= 2147483647.0) integral = false;
    if (integral) {
        out.mode = kModeInt;
        out.H = H;
        out.linp = std::move(linp);
        // +-J form: one coupling magnitude c, lin_v = -sum_j w_vj / 2 and one
        // degree D <= 8 at every site (the Ising lowering of a +-J lattice)
        bool pm = n > 0 && nnz > 0;
        const double c = pm ? std::fabs(p->values[0]) : 0.0;
        const uint64_t D = pm ? p->row_offsets[1] - p->row_offsets[0] : 0;
        pm = pm && D >= 1 && D <= 8 && c >= 1.0;
        for (uint64_t i = 0; pm && i < n; i++) {
            if (p->row_offsets[i + 1] - p->row_offsets[i] != D) pm = false;
            double sw = 0.0;
            for (uint64_t k = p->row_offsets[i]; pm && k < p->row_offsets[i + 1]; k++) {
                if (std::fabs(p->values[k]) != c) pm = false;
                sw += p->values[k];
            }
            if (pm && 2.0 * p->linear[i] != -sw) pm = false;
        }
        out.pmj = pm ? ((uint32_t)c | (uint32_t)D << 16) : 0u;
        out.ents.resize(nnz);
        for (uint64_t k = 0; k < nnz; k++) {
            const double w = p->values[k];
            const uint32_t aw = (uint32_t)std::fabs(w);
            out.ents[k] = (uint32_t)p->col_indices[k] | (aw << 24) | (w < 0 ? 0x80000000u : 0u);
        }
    } else {
        out.mode = kModeF64;
        out.H = 0;
    }
    return IE_OK;
}

// Appends the chunk-packed site-record stream of one instance (layout in
// ie_kernels.cuh); the stream starts and ends on a chunk boundary.
ie_status build_records(HostInst& h, const std::vector<uint8_t>& clampf, size_t site0,
                        std::vector<uint32_t>& out, uint64_t& off, uint64_t& len, uint32_t max_deg = kRecMaxDeg) {
    off = out.size();
    h.recpos.assign(h.n, 0);
    h.reclen.assign(h.n, 0);
    bool first_of_site = true;
    uint32_t cur_site = 0;
    uint32_t c = 0;
    std::vector<uint32_t> rec;
    auto emit = [&](const std::vector<uint32_t>& r) {
        if (c + r.size() > kChunk) {
            out.push_back(kRecPad);
            while (out.size() % kChunk) out.push_back(0);
            c = 0;
        }
        if (first_of_site) {
            h.recpos[cur_site] = (uint32_t)(out.size() - off);
            h.reclen[cur_site] = (uint32_t)r.size();
            first_of_site = false;
        }
        out.insert(out.end(), r.begin(), r.end());
        c = (uint32_t)((c + r.size()) % kChunk);
    };
    for (uint32_t v = 0; v < h.n; v++) {
        const uint32_t beg = h.rows[v], end = h.rows[v + 1];
        const bool clamp = clampf[site0 + v] != 0;
        cur_site = v;
        first_of_site = true;
        if (clamp) {
            emit({kRecClamp, 0, 0, 0});
            continue;
        }
        uint32_t e0 = beg;
        do {
            const uint32_t deg = std::min<uint32_t>(end - e0, max_deg);
            const uint32_t deg4 = (deg + 3u) & ~3u;
            const uint32_t cont = (e0 + deg < end) ? kRecCont : 0u;
            rec.clear();
            if (h.mode == kModeInt) {
                rec.push_back(deg | cont | ((uint32_t)(h.linp[v] + 128) << 16));
                rec.push_back(0);
                rec.push_back(0);
                rec.push_back(0);
                for (uint32_t e = 0; e < deg4; e++) rec.push_back(e < deg ? h.ents[e0 + e] : 0u);
            } else {
                uint32_t w2[2];
                rec.push_back(deg | cont);
                rec.push_back(0);
                std::memcpy(w2, &h.lin[v], 8);
                rec.push_back(w2[0]);
                rec.push_back(w2[1]);
                for (uint32_t e = 0; e < deg4; e++) rec.push_back(e < deg ? h.cols[e0 + e] : 0u);
                for (uint32_t e = 0; e < deg4; e++) {
                    const double w = e < deg ? h.vals[e0 + e] : 0.0;
                    std::memcpy(w2, &w, 8);
                    rec.push_back(w2[0]);
                    rec.push_back(w2[1]);
                }
            }
            emit(rec);
            e0 += deg;
        } while (e0 < end);
    }
    if (c != 0 || out.size() == off) {
        if (c != 0) out.push_back(kRecPad);
        while (out.size() % kChunk || out.size() == off) out.push_back(0);
    }
    len = out.size() - off;
    return IE_OK;
}

// Window table of the windowed kernel (layout in ie_kernels.cu), 16 words per
// window of 8 sites, built when every site has at most 32 couplings (sets
// h.has_wtab). The windowed kernel is preferred (h.windowed_ok) when the
// windows have on average at least 2 sites per dependency level; it is the
// only form for instances whose spins do not fit shared memory. Needs
// h.recpos / h.reclen of a stream with one record per site (window_records).
bool window_table(HostInst& h, std::vector<uint32_t>& tab) {
    h.windowed_ok = false;
    h.has_wtab = false;
    tab.clear();
    if (h.n < (uint32_t)kWin) return false;
    for (uint32_t v = 0; v < h.n; v++)
        if (h.rows[v + 1] - h.rows[v] > kWinMaxDeg) return false;
    const uint32_t nwin = (h.n + kWin - 1) / kWin;
    tab.assign((size_t)nwin * kWT, 0);
    double par = 0;
    for (uint32_t w = 0; w < nwin; w++) {
        uint32_t lvl[kWin] = {}, maxl = 0;
        uint32_t* e = &tab[(size_t)kWT * w];
        for (uint32_t k = 0; k < (uint32_t)kWin; k++) {
            const uint32_t v = kWin * w + k;
            if (v >= h.n) break;
            uint32_t l = 0;
            for (uint32_t q = h.rows[v]; q < h.rows[v + 1]; q++) {
                const uint32_t j = h.cols[q];
                if (j >= kWin * w && j < v) l = std::max(l, lvl[j - kWin * w] + 1);
            }
            lvl[k] = l;
            maxl = std::max(maxl, l);
            e[kWin + k / 8] |= l << (4 * (k % 8));
            e[k] = (h.recpos[v] / 4) | ((h.reclen[v] / 4) << 24);
        }
        e[kWin + 2] = maxl;
        par += (double)kWin / (maxl + 1);
    }
    h.has_wtab = true;
    h.windowed_ok = par / nwin >= 2.0;
    return true;
}

// Appends the windowed kernel's record stream when the batched stream (at
// off, records of at most 16 couplings) does not already have one record per
// site, i.e. when some site has 17..32 couplings; returns the stream's offset
// in wrec and leaves h.recpos / h.reclen describing it.
ie_status window_records(HostInst& h, const std::vector<uint8_t>& clampf, size_t site0,
                         std::vector<uint32_t>& out, uint64_t off, uint64_t& wrec) {
    wrec = off;
    uint32_t maxdeg = 0;
    for (uint32_t v = 0; v < h.n; v++) maxdeg = std::max(maxdeg, h.rows[v + 1] - h.rows[v]);
    if (maxdeg <= kRecMaxDeg || maxdeg > kWinMaxDeg) return IE_OK;
    uint64_t len = 0;
    return build_records(h, clampf, site0, out, wrec, len, kWinMaxDeg);
}

int g_sm_count = -1;

struct Engine {
    int device = 0;
    cudaStream_t stream = nullptr, stream2 = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    uint32_t count = 0;
    uint32_t nt = 1;
    std::vector<InstDesc> desc;
    std::vector<HostInst> insts;
    std::vector<uint8_t> clampf;
    std::vector<int8_t> clampv;
    std::vector<uint32_t> keys;
    size_t total_sites = 0, total_nnz = 0, total_words = 0, total_energy = 0;
    int32_t maxH = 0;

    DevBuf<InstDesc> d_desc;
    DevBuf<uint32_t> d_rows, d_ents, d_cols, d_keys, d_queue, d_draw_idx, d_unclamped, d_recs, d_wtab;
    DevBuf<int32_t> d_linp, d_Ei, d_deo, d_err;
    DevBuf<double> d_vals, d_lin, d_Ef, d_temps, d_dbeta, d_scratch;
    DevBuf<uint8_t> d_clampf;
    DevBuf<int8_t> d_clampv;
    DevBuf<uint64_t> d_spins, d_pos, d_att, d_acc, d_xtab, d_xoff, d_xdmax, d_xdund, d_done;

    uint64_t steps_done = 0;
    bool quads_built = false;
    bool recs_dirty = true;
    double last_ms = 0.0;
    uint64_t last_launches = 0;
    uint32_t threads_per_block = 0, blocks_per_sm = 0;
    std::vector<double> xtemps;  // ladder the exchange tables were built for
    bool initialized = false;
    // populations: the instance's nt cells are nt / pop_len populations of
    // pop_len cells (0: one ladder of nt cells); the population driver
    // re-syncs energies itself, so the PT loop's periodic re-sync is off
    uint32_t pop_len = 0;
    bool periodic_resync = true;
    // round-trip tracking of the exchange (feedback-optimized ladder tuning)
    bool track_roundtrips = false;
    DevBuf<int8_t> d_labels;
    DevBuf<unsigned long long> d_rt;
    DevBuf<uint32_t> d_icm_count, d_icm_rank, d_icm_stack;
    DevBuf<uint8_t> d_icm_flags;

    // icm_sweep (src/solver/icm.rs:161-185) on instance 0: up to 256 MiB of
    // scratch (9 bytes per site per concurrent pair)
    ie_status icm_sweep() {
        const InstDesc& d = desc[0];
        if (d.n == 0) return IE_OK;
        const uint32_t pairs = nt * 32u;
        const uint64_t per = 9ull * d.n;
        const uint32_t slots = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(pairs, (256ull << 20) / per));
        IE_TRY(d_icm_count.alloc(pairs));
        IE_TRY(d_icm_rank.alloc(pairs));
        IE_TRY(d_icm_flags.alloc((size_t)slots * d.n));
        IE_TRY(d_icm_stack.alloc((size_t)slots * 2 * d.n));
        IE_CUDA(launch_icm(arrays(), 0, d.mode, nt, d_icm_count.p, d_icm_rank.p, d_icm_flags.p, d_icm_stack.p, slots,
                           stream));
        return IE_OK;
    }

    ~Engine() {
        if (device >= 0) cudaSetDevice(device);
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        if (evfork) cudaEventDestroy(evfork);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (ev2) cudaEventDestroy(ev2);
        if (stream) cudaStreamDestroy(stream);
        if (stream2) cudaStreamDestroy(stream2);
        for (cudaStream_t st : cstreams) cudaStreamDestroy(st);
        for (cudaEvent_t ev : cevents) cudaEventDestroy(ev);
        for (cudaEvent_t ev : cstart) cudaEventDestroy(ev);
        for (cudaEvent_t ev : cjoin) cudaEventDestroy(ev);
    }

    DevArrays arrays() const {
        DevArrays A{};
        A.desc = d_desc.p;
        A.rows = d_rows.p;
        A.ents = d_ents.p;
        A.linp = d_linp.p;
        A.cols = d_cols.p;
        A.vals = d_vals.p;
        A.lin = d_lin.p;
        A.clampf = d_clampf.p;
        A.clampv = d_clampv.p;
        A.recs = d_recs.p;
        A.wtab = d_wtab.p;
        A.keys = d_keys.p;
        A.spins = d_spins.p;
        A.Ei = d_Ei.p;
        A.Ef = d_Ef.p;
        A.pos = d_pos.p;
        A.deo = d_deo.p;
        A.att = d_att.p;
        A.acc = d_acc.p;
        A.err = d_err.p;
        A.done = d_done.p;
        return A;
    }

    ie_status setup_device(int dev) {
        device = dev;
        int ndev = 0;
        IE_CUDA(cudaGetDeviceCount(&ndev));
        if (dev < 0 || dev >= ndev) return fail(IE_ERR_INVALID, "invalid CUDA device ordinal");
        IE_CUDA(cudaSetDevice(dev));
        IE_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        IE_CUDA(cudaStreamCreateWithFlags(&stream2, cudaStreamNonBlocking));
        IE_CUDA(cudaEventCreate(&ev0));
        IE_CUDA(cudaEventCreate(&ev1));
        IE_CUDA(cudaEventCreate(&ev2));
        if (g_sm_count < 0) IE_CUDA(cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev));
        return IE_OK;
    }

    // Lays out `problems` (each with `cells` temperature cells) and uploads.
    ie_status build(const ie_problem* problems, uint32_t n_problems, uint32_t cells, const uint64_t* seeds,
                    bool force_f64) {
        count = n_problems;
        nt = cells;
        insts.resize(count);
        desc.resize(count);
        keys.resize((size_t)count * 8);
        {
            // per-instance ingestion on host threads; an error is raised again
            // on this thread with its message
            std::vector<ie_status> st(count, IE_OK);
            std::vector<std::string> msg(count);
            parallel_for(count, [&](uint32_t i) {
                st[i] = ingest(&problems[i], force_f64, insts[i]);
                if (st[i] != IE_OK) msg[i] = g_err;
                chacha_key_from_u64(seeds[i], &keys[(size_t)8 * i]);
            });
            for (uint32_t i = 0; i < count; i++)
                if (st[i] != IE_OK) return fail(st[i], msg[i]);
        }
        size_t site = 0, ent = 0, spin = 0, energy = 0, stat = 0;
        for (uint32_t i = 0; i < count; i++) {
            const HostInst& h = insts[i];
            InstDesc& d = desc[i];
            d.n = h.n;
            d.H = h.H;
            d.mode = h.mode;
            d.nt = nt;
            d.owner = i;
            d.cell = 0;
            d.row = site + i;  // rows are n+1 per instance
            d.ent = ent;
            d.site = site;
            d.spin = spin;
            d.energy = energy;
            d.stat = stat;
            site += h.n;
            ent += h.cols.size();
            spin += (size_t)nt * h.n;
            energy += (size_t)nt * kReplicas;
            stat += nt > 1 ? nt - 1 : 1;
            maxH = std::max(maxH, h.H);
        }
        total_sites = site;
        total_nnz = ent;
        total_words = spin;
        total_energy = energy;
        std::vector<uint32_t> rows(site + count), ents(ent), cols(ent);
        std::vector<int32_t> linp(site, 0);
        std::vector<double> vals(ent), lin(site);
        parallel_for(count, [&](uint32_t i) {
            const HostInst& h = insts[i];
            const InstDesc& d = desc[i];
            std::copy(h.rows.begin(), h.rows.end(), rows.begin() + d.row);
            std::copy(h.cols.begin(), h.cols.end(), cols.begin() + d.ent);
            std::copy(h.vals.begin(), h.vals.end(), vals.begin() + d.ent);
            std::copy(h.lin.begin(), h.lin.end(), lin.begin() + d.site);
            if (h.mode == kModeInt) {
                std::copy(h.ents.begin(), h.ents.end(), ents.begin() + d.ent);
                std::copy(h.linp.begin(), h.linp.end(), linp.begin() + d.site);
            }
        });
        clampf.assign(site, 0);
        clampv.assign(site, 0);
        IE_TRY(d_desc.upload(desc, stream));
        IE_TRY(d_rows.upload(rows, stream));
        IE_TRY(d_ents.upload(ents, stream));
        IE_TRY(d_linp.upload(linp, stream));
        IE_TRY(d_cols.upload(cols, stream));
        IE_TRY(d_vals.upload(vals, stream));
        IE_TRY(d_lin.upload(lin, stream));
        IE_TRY(d_keys.upload(keys, stream));
        IE_TRY(d_clampf.upload(clampf, stream));
        IE_TRY(d_clampv.upload(clampv, stream));
        IE_TRY(d_spins.alloc(std::max<size_t>(spin, 1)));
        IE_CUDA(cudaMemsetAsync(d_spins.p, 0, std::max<size_t>(spin, 1) * sizeof(uint64_t), stream));
        IE_TRY(d_Ei.alloc(std::max<size_t>(energy, 1)));
        IE_TRY(d_Ef.alloc(std::max<size_t>(energy, 1)));
        IE_CUDA(cudaMemsetAsync(d_Ei.p, 0, std::max<size_t>(energy, 1) * sizeof(int32_t), stream));
        IE_CUDA(cudaMemsetAsync(d_Ef.p, 0, std::max<size_t>(energy, 1) * sizeof(double), stream));
        std::vector<uint64_t> zeros64(count, 0);
        std::vector<int32_t> zeros32(count, 0);
        IE_TRY(d_pos.upload(zeros64, stream));
        IE_TRY(d_deo.upload(zeros32, stream));
        std::vector<uint64_t> zstat(std::max<size_t>(stat, 1), 0);
        IE_TRY(d_att.upload(zstat, stream));
        IE_TRY(d_acc.upload(zstat, stream));
        IE_TRY(d_err.upload(std::vector<int32_t>(1, 0), stream));
        IE_TRY(d_queue.alloc(1));
        IE_TRY(d_scratch.alloc(std::max<size_t>((size_t)nt * kReplicas, 1)));
        IE_TRY(upload_draw_idx());
        IE_CUDA(cudaStreamSynchronize(stream));
        return IE_OK;
    }

    ie_status upload_draw_idx() {
        std::vector<uint32_t> idx(std::max<size_t>(total_sites, 1), 0), unc(count, 0);
        for (uint32_t i = 0; i < count; i++) {
            uint32_t c = 0;
            for (uint32_t v = 0; v < desc[i].n; v++) {
                idx[desc[i].site + v] = c;
                if (!clampf[desc[i].site + v]) c++;
            }
            unc[i] = c;
        }
        IE_TRY(d_draw_idx.upload(idx, stream));
        IE_TRY(d_unclamped.upload(unc, stream));
        return IE_OK;
    }

    ie_status set_clamps(uint32_t inst, const uint8_t* f, const int8_t* v) {
        const InstDesc& d = desc[inst];
        for (uint32_t i = 0; i < d.n; i++) {
            clampf[d.site + i] = f ? (f[i] ? 1 : 0) : 0;
            clampv[d.site + i] = (f && f[i] && v) ? (v[i] == 1 ? 1 : 0) : 0;
        }
        IE_CUDA(cudaMemcpyAsync(d_clampf.p, clampf.data(), clampf.size(), cudaMemcpyHostToDevice, stream));
        IE_CUDA(cudaMemcpyAsync(d_clampv.p, clampv.data(), clampv.size(), cudaMemcpyHostToDevice, stream));
        IE_TRY(upload_draw_idx());
        IE_CUDA(cudaStreamSynchronize(stream));
        recs_dirty = true;
        return IE_OK;
    }

    void build_window_table(uint32_t i, std::vector<uint32_t>& wt) {
        desc[i].win = 0;
        std::vector<uint32_t> tab;
        if (!window_table(insts[i], tab)) return;
        desc[i].win = wt.size();
        wt.insert(wt.end(), tab.begin(), tab.end());
    }

    // Record streams and window tables, built per instance on host threads
    // (each stream a whole number of chunks) and concatenated.
    ie_status build_record_streams() {
        // the per-lane kernels' streams: needed unless every instance runs on
        // the level kernel (a batch on kernel_form 0; handles keep them for
        // f64 cells)
        bool old_needed = kernel_form != 0;
        for (uint32_t i = 0; i < count && !old_needed; i++) old_needed = !is_batch && desc[i].mode == kModeF64;
        std::vector<std::vector<uint32_t>> lrec(count), lwt(count);
        std::vector<ie_status> st(count, IE_OK);
        std::vector<std::string> msg(count);
        parallel_for(old_needed ? count : 0u, [&](uint32_t i) {
            st[i] = build_records(insts[i], clampf, desc[i].site, lrec[i], desc[i].rec, desc[i].rec_len);
            if (st[i] == IE_OK) st[i] = window_records(insts[i], clampf, desc[i].site, lrec[i], desc[i].rec, desc[i].wrec);
            if (st[i] != IE_OK) {
                msg[i] = g_err;
                return;
            }
            build_window_table(i, lwt[i]);
        });
        for (uint32_t i = 0; i < count; i++)
            if (st[i] != IE_OK) return fail(st[i], msg[i]);
        std::vector<uint64_t> roff(count + 1, 0), woff(count + 1, 0);
        for (uint32_t i = 0; i < count; i++) {
            roff[i + 1] = roff[i] + lrec[i].size();
            woff[i + 1] = woff[i] + lwt[i].size();
        }
        std::vector<uint32_t> recs(roff[count] + kChunk, 0), wt(std::max<uint64_t>(woff[count], kWT), 0);
        parallel_for(count, [&](uint32_t i) {
            std::copy(lrec[i].begin(), lrec[i].end(), recs.begin() + roff[i]);
            std::copy(lwt[i].begin(), lwt[i].end(), wt.begin() + woff[i]);
            desc[i].rec += roff[i];
            desc[i].wrec += roff[i];
            desc[i].win += woff[i];
        });
        IE_TRY(d_recs.upload(recs, stream));
        IE_TRY(d_wtab.upload(wt, stream));
        quads_built = false;
        IE_CUDA(cudaMemcpyAsync(d_desc.p, desc.data(), desc.size() * sizeof(InstDesc), cudaMemcpyHostToDevice, stream));
        if (kernel_form == 0) IE_TRY(build_level_data());
        IE_CUDA(cudaStreamSynchronize(stream));
        recs_dirty = false;
        return IE_OK;
    }

    // warm-start probabilities per site (single-instance handles); empty:
    // the random init
    std::vector<double> init_probs;

    ie_status init_random() {
        if (!init_probs.empty()) {
            // the warm start is drawn on the host at the stream's position
            // and uploaded like ie_set_spins; the position advances past it
            const InstDesc& d = desc[0];
            HostStream rng{};
            std::copy(keys.begin(), keys.begin() + 8, rng.key);
            IE_CUDA(cudaMemcpyAsync(&rng.pos, d_pos.p, sizeof(uint64_t), cudaMemcpyDeviceToHost, stream));
            IE_CUDA(cudaStreamSynchronize(stream));
            std::vector<uint64_t> w((size_t)d.nt * d.n);
            warm_start_words(rng, init_probs.data(), clampf.data() + d.site, clampv.data() + d.site, d.n, d.nt,
                             w.data());
            IE_TRY(write_words(0, w.data()));
            IE_CUDA(cudaMemcpyAsync(d_pos.p, &rng.pos, sizeof(uint64_t), cudaMemcpyHostToDevice, stream));
            IE_CUDA(cudaStreamSynchronize(stream));
            return IE_OK;
        }
        const DevArrays A = arrays();
        IE_CUDA(launch_init(A, 0, count, d_draw_idx.p, d_unclamped.p, stream));
        IE_CUDA(launch_energy(A, 0, count, stream));
        IE_CUDA(cudaStreamSynchronize(stream));
        initialized = true;
        return IE_OK;
    }

    static double inst_work(const HostInst& h) {
        const double deg = h.n ? (double)h.nnz / h.n : 0.0;
        return (double)h.n * (deg + 12.0) * (h.mode == kModeF64 ? 2.5 : 1.0);
    }

    // Work classes (mode, TPL, spin capacity): TPL threads per Xoshiro lane,
    // so the largest instances, whose sequential site chain sets the
    // makespan, get the most threads; the shared-memory capacity of a class
    // is the smallest of kCaps that holds its instances.
    static constexpr uint32_t kCaps[10] = {256, 512, 768, 1024, 1536, 2048, 3072, 4096, 8192, 16384};
    // size thresholds per mode (see tpl_of); defaults are the autotuner's
    // usual choice on uneven random-graph batches
    uint32_t tune_n4[2] = {256, 768}, tune_n2[2] = {128, 256};
    struct WorkClass {
        uint32_t mode = 0;
        int tpl = 1;
        uint32_t cap = 64;
        uint32_t nitems = 0;
        double work = 0;       // longest item
        double site_steps = 0; // sites summed over the class (per sweep)
        DevBuf<uint32_t> items;
        DevBuf<int32_t> itemh;
        // level-kernel class: items of the shared item arrays in launch order
        bool level = false;
        bool gsp = false;
        uint32_t split = 1;  // CTAs per cluster (one item per cluster)
        uint32_t ntab = 1;
        int grid = 0;
        uint64_t keystride = 0, keyoff = 0;
        uint32_t ov = 0;  // > 0: sweeps overlapped, a generator group of ov threads per CTA
        DevBuf<uint32_t> order;
    };
    static constexpr int kLevelForm = 32;  // tpl tag of a level-kernel class
    std::vector<std::unique_ptr<WorkClass>> classes;
    std::vector<cudaStream_t> cstreams;
    std::vector<cudaEvent_t> cevents, cstart, cjoin;
    std::vector<double> class_ms;  // device time of each class launch in the last run

    ie_status ensure_class_streams(size_t k) {
        while (cstreams.size() < k) {
            cudaStream_t st;
            cudaEvent_t ev, ev0, ej;
            IE_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            IE_CUDA(cudaEventCreate(&ev));
            IE_CUDA(cudaEventCreate(&ev0));
            IE_CUDA(cudaEventCreateWithFlags(&ej, cudaEventDisableTiming));
            cstreams.push_back(st);
            cevents.push_back(ev);
            cstart.push_back(ev0);
            cjoin.push_back(ej);
        }
        return IE_OK;
    }

    // Kernel form of an instance: 1, 2, 4 threads per lane (batch_kernel), 8:
    // the windowed kernel, 16: the chain kernel (one CTA per instance). Above
    // n4, instances whose windows are parallel take the windowed kernel; other
    // instances above n2 (sequential site chains: lattices) the chain kernel;
    // the rest run 2 to a warp above n2 and 4 to a warp below. Spins beyond
    // shared memory stay in global memory. Without windows (use_windows
    // false) the one-warp forms 4 / 2 / 1 only.
    static constexpr uint32_t kSmemSpinCap = 24576;
    static constexpr int kChain = 16;
    int tpl_of(const InstDesc& d, const HostInst& h) const {
        const uint32_t n = d.n, m = d.mode;
        if (cap_of(n) > kSmemSpinCap) return h.windowed_ok && use_windows ? 8 : kChain;
        if (!use_windows) return n > tune_n4[m] ? 4 : (n > tune_n2[m] ? 2 : 1);
        if (n > tune_n4[m]) return h.windowed_ok ? 8 : kChain;
        if (n > tune_n2[m] && !h.windowed_ok) return kChain;
        return n > tune_n2[m] ? 2 : 1;
    }
    // shared-memory spin capacity of the instance's class; 0: spins in global memory
    static uint32_t class_cap(const InstDesc& d) { return cap_of(d.n) > kSmemSpinCap ? 0u : cap_of(d.n); }
    bool use_windows = true;
    bool is_batch = false;        // ie_batch: single-cell instances, no PT cells
    std::vector<uint8_t> active;  // instances in the work classes (empty: all)

    // Level kernel (ie_level.cu): kernel_form 0 runs batched instances and
    // integer-mode PT cells on it; 1 keeps the per-lane kernels.
    int kernel_form = 0;
    uint32_t lvl_cap = 4096;  // spin words per item (shared memory)
    int lvl_threads = 256;
    uint32_t lvl_tie_shift = 0;
    bool lvl_split = true;    // large single-member items on thread block clusters
    bool lvl_overlap = true;  // latency-bound launches overlap the generator and decision phases
    // per class mode (int, f64, +-J): spin words an item is packed to (0: lvl_cap);
    // integer items at 2048 measured 1.5-2 % faster on the uneven batch (f64 at 2048: slower)
    uint32_t lvl_pack[3] = {2048, 0, 0};
    bool bulk_ring = false;   // per-lane kernels: record chunks by bulk copies (cp.async measured faster)
    uint32_t lvl_cluster_max = 0;  // most CTAs per cluster (0: 16)
    int32_t pmj_policy = 0;   // +-J instances on the bit-sliced form: 0 auto, 1 always, -1 never
    bool serving = false;     // serving launches: one threshold table per member
    std::vector<std::vector<uint32_t>> lv_sites, lv_off;  // per instance: sites by level, level starts
    std::vector<uint32_t> h_recoff;                       // level-record offset per site
    DevBuf<uint32_t> d_lrecs, d_recoff, d_llvl, d_lseg, d_keybuf;
    DevBuf<LvlEntry> d_lent;
    DevBuf<LvlItem> d_litems;
    DevBuf<LvlMember> d_lmem;
    DevBuf<uint64_t> d_jpoly;
    DevBuf<int32_t> d_exact;
    DevBuf<uint32_t> d_plainq;  // queue counters of the one-launch-per-cell path
    uint32_t jpoly_count = 0;
    LvlHost lvh;

    bool level_ok(const InstDesc& d, bool cells_view) const {
        if (kernel_form != 0) return false;
        return !cells_view || d.mode == kModeInt;
    }

    static LvlSource lvl_source(const HostInst& h, const uint8_t* clampf) {
        LvlSource s;
        s.n = h.n;
        s.mode = h.mode;
        s.rows = h.rows.data();
        s.cols = h.cols.data();
        s.vals = h.vals.data();
        s.lin = h.lin.data();
        s.ents = h.ents.data();
        s.linp = h.linp.data();
        s.clampf = clampf;
        return s;
    }

    // Level records (recoff indexed by InstDesc::site + v) and dependency
    // levels of every instance, built on host threads.
    ie_status build_level_data() {
        std::vector<std::vector<uint32_t>> lrec(count);
        std::vector<uint32_t> recoff(std::max<size_t>(total_sites, 1), 0);
        lv_sites.assign(count, {});
        lv_off.assign(count, {});
        parallel_for(count, [&](uint32_t i) {
            const LvlSource src = lvl_source(insts[i], clampf.data() + desc[i].site);
            level_records(src, lrec[i], recoff.data() + desc[i].site);
            site_levels(src, lv_sites[i], lv_off[i]);
        });
        std::vector<uint64_t> base(count + 1, 0);
        for (uint32_t i = 0; i < count; i++) base[i + 1] = base[i] + lrec[i].size();
        if (base[count] / 4 >= (1ull << 32)) return fail(IE_ERR_UNSUPPORTED, "level records exceed 64 GiB");
        std::vector<uint32_t> recs(std::max<uint64_t>(base[count], 4), 0);
        parallel_for(count, [&](uint32_t i) {
            std::copy(lrec[i].begin(), lrec[i].end(), recs.begin() + base[i]);
            const uint32_t b16 = (uint32_t)(base[i] / 4);
            for (uint32_t v = 0; v < desc[i].n; v++) recoff[desc[i].site + v] += b16;
        });
        IE_TRY(d_lrecs.upload(recs, stream));
        IE_TRY(d_recoff.upload(recoff, stream));
        h_recoff = std::move(recoff);
        return IE_OK;
    }

    // CUDA graph of one batched run (use_graph): valid for the classes it was
    // captured with and for runs of g_steps steps; the step base is read from
    // d_stepbase so replays continue the trajectory.
    bool use_graph = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaEvent_t evfork = nullptr;
    bool graph_valid = false;
    uint64_t g_steps = 0;
    DevBuf<uint64_t> d_stepbase;

    // PT cells as work items: 0 chooses by size, 1 runs one CTA per instance
    // (pt_kernel), 2 runs every cell as its own work item of the batched /
    // windowed kernels with the exchange in exchange_kernel
    int pt_path = 0;
    std::vector<InstDesc> cdesc;
    std::vector<HostInst> cinsts;
    DevBuf<InstDesc> d_cdesc;
    DevBuf<uint64_t> d_xmask;
    bool cells_built = false;
    static uint32_t cap_of(uint32_t n) {
        for (uint32_t c : kCaps)
            if (n <= c) return c;
        return (n + 63u) & ~63u;
    }

    // Level-kernel classes over an instance view: one class per (mode,
    // spins in shared / global memory); items of up to lvl_cap spin words
    // (a PT cell of 512 sites or more is an item of its own, so a ladder
    // spreads over as many CTAs as it has cells). Each class's grid and
    // per-CTA output buffer are fixed here.
    template <typename Live>
    ie_status build_level_classes(const std::vector<InstDesc>& D, const std::vector<HostInst>& HI, bool cells_view,
                                  Live live, bool one_per_item = false) {
        lvh.clear();
        std::vector<uint64_t> nnz_of(D.size());
        std::vector<uint32_t> pmj_of(D.size()), dmax_of(D.size(), 0);
        for (size_t i = 0; i < D.size(); i++) {
            nnz_of[i] = HI[i].nnz;
            if (!live(i)) continue;
            const std::vector<uint32_t>& rw = HI[i].rows;
            for (size_t v = 0; v + 1 < rw.size(); v++) dmax_of[i] = std::max(dmax_of[i], rw[v + 1] - rw[v]);
        }
        const bool own = cells_view || serving;
        // classes: integer, f64, +-J form (one magnitude c per launch)
        std::vector<uint32_t> mem[3][2];
        uint64_t live_count = 0, pm_count = 0;
        uint32_t c0 = 0;
        for (uint32_t i = 0; i < (uint32_t)D.size(); i++)
            if (live(i) && level_ok(D[i], cells_view) && HI[i].pmj) pm_count++;
        for (uint32_t i = 0; i < (uint32_t)D.size(); i++) {
            if (!live(i) || !level_ok(D[i], cells_view)) continue;
            live_count++;
            const bool gsp = D[i].n > lvl_cap;
            // the +-J form trades a dearer generator (exact masks per level) for
            // far cheaper decisions: taken for large instances and for enough
            // instances to fill the GPU, not for a few small latency-bound ones
            const bool want = pmj_policy > 0 || (pmj_policy == 0 && (gsp || pm_count >= (uint64_t)g_sm_count));
            const uint32_t pm = want ? HI[i].pmj : 0u;
            if (pm && !c0) c0 = pm & 0xFFFFu;
            const bool as_pmj = pm && (pm & 0xFFFFu) == c0;
            pmj_of[i] = as_pmj ? pm : 0u;
            mem[as_pmj ? 2 : D[i].mode == kModeF64 ? 1 : 0][gsp ? 1 : 0].push_back(i);
        }
        uint64_t keytotal = 0;
        for (int m = 0; m < 3; m++)
            for (int g = 0; g < 2; g++) {
                if (mem[m][g].empty()) continue;
                // spins in global memory: few large items spread over clusters
                // of up to 16 CTAs while that keeps every SM busy
                uint32_t split = 1;
                const uint32_t kmode = m == 2 ? kModePmJ : m ? kModeF64 : kModeInt;
                const size_t smem0 = level_smem(kmode, own ? (one_per_item ? 1u : kLvlMaxOwnTables) : 1u, 0);
                if (g && !one_per_item && lvl_split && !(cells_view && pt_path == 3)) {
                    const int occ1 = level_occupancy(kmode, true, lvl_threads, smem0);
                    const uint32_t cmax = lvl_cluster_max ? lvl_cluster_max : 16u;
                    while (split < cmax && (uint64_t)mem[m][g].size() * split * 2 <= (uint64_t)occ1 * g_sm_count)
                        split *= 2;
                    if (serving) split = std::min<uint32_t>(cmax, split * 2);
                    while (split > 1 && level_clusters(kmode, lvl_threads, smem0, split) <= 0)
                        split /= 2;
                }
                std::unique_ptr<WorkClass> wc(new WorkClass());
                wc->level = true;
                wc->mode = kmode;
                wc->gsp = g != 0;
                wc->tpl = kLevelForm;
                wc->cap = g ? 0u : lvl_cap;
                uint32_t cap = lvl_cap, maxn = 0;
                for (uint32_t i : mem[m][g]) maxn = std::max(maxn, D[i].n);
                if (cells_view && maxn >= 512) cap = std::min(cap, maxn);
                // items packed to fewer sites than the shared-memory capacity:
                // shorter items, a shorter tail of the class's last ones
                if (lvl_pack[m] && !g) cap = std::min(cap, lvl_pack[m]);
                // serving: one request per CTA while the requests fit the GPU's
                // CTA slots (a packed item advances all its requests at the rate of one)
                const bool alone = one_per_item || (serving && live_count <= (uint64_t)4 * g_sm_count);
                const uint32_t maxmem = alone ? 1u : own ? kLvlMaxOwnTables : kLvlMaxMembers;
                std::vector<uint32_t> order;
                double longest = 0;
                const size_t item_begin = lvh.items.size();
                build_level_items(D, nnz_of, dmax_of, pmj_of, lv_sites, lv_off, h_recoff, mem[m][g], g != 0, cap, maxmem,
                                  split, lvh, order, longest);
                wc->nitems = (uint32_t)order.size();
                wc->work = longest;
                for (uint32_t i : mem[m][g]) wc->site_steps += (double)D[i].n;
                wc->ntab = own ? std::max<uint32_t>(maxmem, 1u) : 1u;
                // latency-bound launches (an item per CTA, narrow levels): the
                // generator half of each CTA runs one sweep ahead of the decider half
                {
                    double sites = 0, levels = 0;
                    for (size_t q = item_begin; q < lvh.items.size(); q++) {
                        sites += (double)lvh.items[q].sites;
                        levels += (double)std::max<uint32_t>(lvh.items[q].nlvl, 1);
                    }
                    const double width = (kmode == kModePmJ ? 1.0 : 8.0) * sites / std::max(levels, 1.0);
                    const uint32_t gen = kLvlOverlapGen;
                    const int occ0 = level_occupancy(wc->mode, g != 0, lvl_threads + (int)gen,
                                                     level_smem(wc->mode, wc->ntab, g ? 0 : lvl_cap, true));
                    wc->ov = lvl_overlap && split == 1 && occ0 > 0 && wc->nitems <= (uint32_t)(occ0 * g_sm_count) &&
                                     width <= lvl_threads
                                 ? gen
                                 : 0u;
                }
                const size_t smem = level_smem(wc->mode, wc->ntab, g ? 0 : lvl_cap, wc->ov != 0);
                int occ = level_occupancy(wc->mode, g != 0, lvl_threads + (int)wc->ov, smem);
                if (occ <= 0) return fail(IE_ERR_UNSUPPORTED, "level kernel does not fit on an SM");
                if (blocks_per_sm) occ = std::min<int>(occ, (int)blocks_per_sm);
                wc->split = split;
                if (split > 1) {
                    const int nc = level_clusters(wc->mode, lvl_threads, smem, split);
                    wc->grid = (int)split * std::max(1, std::min<int>((int)wc->nitems, nc));
                } else {
                    wc->grid = std::max(1, std::min<int>((int)wc->nitems, occ * g_sm_count));
                }
                wc->keystride = 64ull * (g ? maxn : lvl_cap) * (wc->ov ? 2 : 1);
                wc->keyoff = keytotal;
                keytotal += wc->keystride * (uint64_t)(wc->grid / split);
                IE_TRY(wc->order.upload(order, stream));
                classes.push_back(std::move(wc));
            }
        if (lvh.items.empty()) return IE_OK;
        IE_TRY(d_litems.upload(lvh.items, stream));
        IE_TRY(d_lmem.upload(lvh.members, stream));
        IE_TRY(d_lent.upload(lvh.entries.empty() ? std::vector<LvlEntry>(1, LvlEntry{0, 0}) : lvh.entries, stream));
        IE_TRY(d_llvl.upload(lvh.lvloff, stream));
        IE_TRY(d_lseg.upload(lvh.segs, stream));
        IE_TRY(d_keybuf.alloc(std::max<uint64_t>(keytotal, 1)));
        if (lvh.max_segs > jpoly_count) {
            std::vector<uint64_t> tab;
            if (!xoshiro_segment_polys(lvh.max_segs, tab))
                return fail(IE_ERR_DEVICE, "Xoshiro jump polynomial could not be derived");
            IE_TRY(d_jpoly.upload(tab, stream));
            jpoly_count = lvh.max_segs;
        }
        if (!d_exact.p) IE_TRY(d_exact.upload(std::vector<int32_t>(1, 0), stream));
        return IE_OK;
    }

    LvlArgs level_args(const WorkClass& wc, uint32_t* queue) const {
        LvlArgs L{};
        L.items = d_litems.p;
        L.order = wc.order.p;
        L.nitems = wc.nitems;
        L.queue = queue;
        L.members = d_lmem.p;
        L.entries = d_lent.p;
        L.lvloff = d_llvl.p;
        L.segs = d_lseg.p;
        L.jpoly = d_jpoly.p;
        L.recoff = d_recoff.p;
        L.lrecs = d_lrecs.p;
        L.keybuf = d_keybuf.p + wc.keyoff;
        L.keystride = wc.keystride;
        L.ov = wc.ov;
        L.keyhalf = wc.ov ? wc.keystride / 2 : 0;
        L.spin_cap = wc.gsp ? 0u : lvl_cap;
        L.ntab = wc.ntab;
        L.tie_shift = lvl_tie_shift;
        L.exact_count = d_exact.p;
        return L;
    }

    // Per class: instances ordered by degree then size into items of 4/TPL
    // (the groups of a warp stay in step sweep by sweep), items ordered by
    // work, longest first; classes ordered by their longest item.
    // Work classes over an instance view (D, HI): the engine's instances, or
    // the cells of its PT instances.
    ie_status build_quads(const std::vector<InstDesc>* Dp = nullptr, const std::vector<HostInst>* Hp = nullptr) {
        const std::vector<InstDesc>& D = Dp ? *Dp : desc;
        const std::vector<HostInst>& HI = Hp ? *Hp : insts;
        const uint32_t N = (uint32_t)D.size();
        classes.clear();
        cells_built = false;
        graph_valid = false;
        std::vector<std::tuple<uint32_t, int, uint32_t>> keys;
        auto live0 = [&](uint32_t i) { return Dp || active.empty() || active[i] != 0; };
        IE_TRY(build_level_classes(D, HI, Dp != nullptr, live0));
        auto live = [&](uint32_t i) { return live0(i) && !level_ok(D[i], Dp != nullptr); };
        for (uint32_t i = 0; i < N; i++) {
            if (!live(i)) continue;
            auto k = std::make_tuple(D[i].mode, tpl_of(D[i], HI[i]), class_cap(D[i]));
            if (std::find(keys.begin(), keys.end(), k) == keys.end()) keys.push_back(k);
        }
        auto degree = [&](uint32_t i) {
            return HI[i].n ? (uint32_t)((HI[i].nnz + HI[i].n / 2) / HI[i].n) : 0u;
        };
        for (auto& k : keys) {
            std::unique_ptr<WorkClass> wc(new WorkClass());
            wc->mode = std::get<0>(k);
            wc->tpl = std::get<1>(k);
            wc->cap = std::get<2>(k);
            const int ng = wc->tpl >= 8 ? 1 : 4 / wc->tpl;
            std::vector<uint32_t> order;
            for (uint32_t i = 0; i < N; i++)
                if (live(i) && D[i].mode == wc->mode && tpl_of(D[i], HI[i]) == wc->tpl && class_cap(D[i]) == wc->cap)
                    order.push_back(i);
            std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
                if (degree(a) != degree(b)) return degree(a) > degree(b);
                return D[a].n > D[b].n;
            });
            std::vector<std::vector<uint32_t>> items;
            for (size_t i = 0; i < order.size();) {
                std::vector<uint32_t> q;
                const uint32_t dg = degree(order[i]);
                while ((int)q.size() < ng && i < order.size() && degree(order[i]) == dg) q.push_back(order[i++]);
                items.push_back(q);
            }
            auto work = [&](const std::vector<uint32_t>& q) {
                double w = 0;
                for (uint32_t i : q) w = std::max(w, inst_work(HI[i]) / (wc->tpl == 8 ? 5 : wc->tpl == kChain ? 6 : wc->tpl));
                return w;
            };
            std::stable_sort(items.begin(), items.end(), [&](const std::vector<uint32_t>& a,
                                                             const std::vector<uint32_t>& b) { return work(a) > work(b); });
            std::vector<uint32_t> flat;
            std::vector<int32_t> qh;
            for (auto& q : items) {
                int32_t hh = 0;
                for (int j = 0; j < 4; j++) {
                    flat.push_back(j < (int)q.size() ? q[j] : 0xffffffffu);
                    if (j < (int)q.size()) {
                        hh = std::max(hh, D[q[j]].H);
                        wc->site_steps += (double)D[q[j]].n;
                    }
                }
                qh.push_back(hh);
                wc->work = std::max(wc->work, work(q));
            }
            wc->nitems = (uint32_t)items.size();
            IE_TRY(wc->items.upload(flat, stream));
            IE_TRY(wc->itemh.upload(qh, stream));
            classes.push_back(std::move(wc));
        }
        std::stable_sort(classes.begin(), classes.end(),
                         [](const std::unique_ptr<WorkClass>& a, const std::unique_ptr<WorkClass>& b) {
                             return a->work > b->work;
                         });
        IE_TRY(d_queue.alloc(std::max<size_t>(classes.size(), 1)));
        quads_built = true;
        return IE_OK;
    }

    bool use_cells() const {
        if (pop_len) return true;
        if (pt_path == 1) return false;
        if (pt_path >= 2) return true;
        return desc[0].n >= 256;
    }

    // Cell view: cell c of instance i as its own entry (spins and energies of
    // the cell, records and window table of the instance, owner i).
    ie_status build_cells() {
        if (recs_dirty) IE_TRY(build_record_streams());
        cdesc.clear();
        cinsts.clear();
        for (uint32_t i = 0; i < count; i++)
            for (uint32_t c = 0; c < desc[i].nt; c++) {
                InstDesc e = desc[i];
                e.nt = 1;
                e.spin = desc[i].spin + (uint64_t)c * desc[i].n;
                e.energy = desc[i].energy + (uint64_t)c * kReplicas;
                e.owner = i;
                e.cell = c;
                cdesc.push_back(e);
                HostInst l;
                l.n = insts[i].n;
                l.H = insts[i].H;
                l.mode = insts[i].mode;
                l.nnz = insts[i].nnz;
                l.windowed_ok = insts[i].windowed_ok;
                l.has_wtab = insts[i].has_wtab;
                l.pmj = insts[i].pmj;
                cinsts.push_back(l);
            }
        IE_TRY(d_cdesc.upload(cdesc, stream));
        IE_TRY(d_xmask.alloc(std::max<size_t>(d_att.n, 1)));
        IE_TRY(build_quads(&cdesc, &cinsts));
        quads_built = false;
        cells_built = true;
        return IE_OK;
    }

    // PT steps with the cells as work items: launches of the cells' sweeps
    // end at every exchange step (and f64 resync step); after each, the
    // exchange kernel decides the DEO pairs and advances the stream, the swap
    // kernel exchanges configurations, and on resync steps the energies are
    // recomputed (ultimate.rs:316-324: after the step's exchange).
    ie_status run_pt_cells(uint64_t steps, bool per_step, const RunArgs& X) {
        if (recs_dirty || !cells_built) IE_TRY(build_cells());
        const uint32_t mode = desc[0].mode;
        DevArrays A = arrays();
        A.xmask = d_xmask.p;
        DevArrays AC = A;
        AC.desc = d_cdesc.p;
        RunArgs R = X;
        R.cells = 1;
        R.ladder = nt;
        R.temps_per_step = per_step ? 1 : 0;
        const uint64_t kx = R.exchange_interval;
        IE_CUDA(cudaEventRecord(ev2, stream));
        uint64_t done = 0, launches = 0;
        while (done < steps) {
            const uint64_t g0 = steps_done + done;
            uint64_t k = kx - g0 % kx;
            // a single cell has no exchange pairs: its exchange steps only
            // toggle the DEO phase, so one launch runs every step
            if (nt == 1) k = std::min<uint64_t>(steps - done, 1u << 20);
            if (mode == kModeF64 && periodic_resync) k = std::min<uint64_t>(k, kResyncEvery - g0 % kResyncEvery);
            k = std::min<uint64_t>(k, steps - done);
            R.steps = (uint32_t)k;
            R.step_base = g0;
            R.temps = d_temps.p + (per_step ? done * nt : 0);
            IE_TRY(launch_classes(R, AC));
            launches += last_launches;
            const bool ex = nt == 1 ? (((g0 + k) / kx - g0 / kx) & 1u) != 0 : (g0 + k) % kx == 0;
            IE_CUDA(launch_exchange(A, R, count, mode, (uint32_t)k, ex, stream));
            launches++;
            if (ex && nt > 1)
                for (uint32_t i = 0; i < count; i++) {
                    IE_CUDA(launch_swap(A, i, desc[i].n, g_sm_count, stream));
                    launches++;
                }
            if (mode == kModeF64 && periodic_resync && (g0 + k) % kResyncEvery == 0) {
                IE_CUDA(launch_energy(A, 0, count, stream));
                launches++;
            }
            done += k;
        }
        IE_CUDA(cudaEventRecord(ev1, stream));
        IE_CUDA(cudaEventSynchronize(ev1));
        float ms = 0;
        IE_CUDA(cudaEventElapsedTime(&ms, ev2, ev1));
        last_ms = ms;
        last_launches = launches;
        steps_done += steps;
        return IE_OK;
    }

    RunArgs sa_args(uint64_t steps) const {
        RunArgs R{};
        R.temps = d_temps.p;
        R.temps_per_step = 1;
        R.steps = (uint32_t)steps;
        R.step_base = steps_done;
        R.exchange_interval = 1;
        return R;
    }

    // Runs temps[steps] on every single-cell instance: one persistent launch
    // per work class, all in flight together on their own streams.
    ie_status run_batch(const double* temps, uint64_t steps) {
        if (nt != 1) return fail(IE_ERR_INVALID, "batched runs need single-cell instances");
        if (!initialized) return fail(IE_ERR_INVALID, "call init_random before running");
        if (steps == 0) return IE_OK;
        if (steps > 0xffffffffULL) return fail(IE_ERR_INVALID, "too many steps in one call");
        if (recs_dirty) IE_TRY(build_record_streams());
        if (!quads_built) IE_TRY(build_quads());
        IE_TRY(ensure_class_streams(classes.size()));
        std::vector<double> t(temps, temps + steps);
        for (double x : t)
            if (!(x > 0.0) || !std::isfinite(x)) return fail(IE_ERR_INVALID, "temperatures must be positive");
        IE_TRY(d_temps.upload(t, stream));
        RunArgs R = sa_args(steps);
        if (use_graph) {
            IE_TRY(d_stepbase.alloc(1));
            IE_CUDA(cudaMemcpyAsync(d_stepbase.p, &steps_done, sizeof(uint64_t), cudaMemcpyHostToDevice, stream));
            R.step_base_dev = d_stepbase.p;
            IE_TRY(launch_classes(R, arrays(), true));
        } else {
            IE_TRY(launch_classes(R));
        }
        steps_done += steps;
        return IE_OK;
    }

    // One persistent launch per work class, all in flight together on their
    // own streams, largest classes first (their CTAs are dispatched first and
    // the smaller classes fill the remaining room), forked from and joined
    // back into the engine's stream. Only stream operations, so the sequence
    // can be captured into a CUDA graph; grids are computed beforehand.
    ie_status class_grids(const RunArgs& base, std::vector<int>& grids) {
        grids.assign(classes.size(), 0);
        for (size_t k = 0; k < classes.size(); k++) {
            WorkClass& wc = *classes[k];
            if (!wc.nitems) continue;
            if (wc.level) {
                grids[k] = wc.grid;
                continue;
            }
            int occ = wc.tpl == 8       ? window_occupancy(wc.mode, wc.cap)
                      : wc.tpl == kChain ? chain_occupancy(wc.mode, wc.cap)
                                         : batch_occupancy(wc.mode, wc.tpl, wc.cap, base.serve != 0 || base.cells != 0);
            if (occ <= 0) return fail(IE_ERR_UNSUPPORTED, "batched kernel does not fit on an SM");
            if (blocks_per_sm) occ = std::min<int>(occ, (int)blocks_per_sm);
            grids[k] = std::max(1, std::min<int>((int)wc.nitems, occ * g_sm_count));
        }
        return IE_OK;
    }

    // capturing: the timing events become event-record nodes of the graph
    // (cudaEventRecordExternal); the joins use their own events.
    ie_status enqueue_classes(const RunArgs& base, const DevArrays& A, const std::vector<int>& grids,
                              uint64_t& launches, bool capturing = false) {
        const unsigned rec = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
        launches = 0;
        IE_CUDA(cudaMemsetAsync(d_queue.p, 0, classes.size() * sizeof(uint32_t), stream));
        uint32_t plain_base = 0;
        if (pt_path == 3 && base.cells) {
            uint32_t total = 0;
            for (auto& c : classes) total += c->level ? c->nitems : 0u;
            IE_TRY(d_plainq.alloc(std::max<uint32_t>(total, 1)));
            IE_CUDA(cudaMemsetAsync(d_plainq.p, 0, d_plainq.n * sizeof(uint32_t), stream));
        }
        IE_CUDA(cudaEventRecord(evfork, stream));
        for (size_t k = 0; k < classes.size(); k++) {
            WorkClass& wc = *classes[k];
            if (!wc.nitems) continue;
            IE_CUDA(cudaStreamWaitEvent(cstreams[k], evfork, 0));
            RunArgs R = base;
            R.bulk_ring = bulk_ring ? 1u : 0u;
            R.quads = wc.items.p;
            R.quad_h = wc.itemh.p;
            R.nquads = wc.nitems;
            R.queue = d_queue.p + k;
            IE_CUDA(cudaEventRecordWithFlags(cstart[k], cstreams[k], rec));
            if (wc.level && pt_path == 3 && base.cells) {
                // the plain per-temperature method: one launch (one CTA) per
                // cell, one after another
                for (uint32_t it = 0; it < wc.nitems; it++) {
                    LvlArgs L = level_args(wc, d_plainq.p + plain_base + it);
                    L.order = wc.order.p + it;
                    L.nitems = 1;
                    IE_CUDA(launch_level(A, R, L, wc.mode, wc.gsp, lvl_threads, 1, cstreams[k]));
                    launches++;
                }
                plain_base += wc.nitems;
                launches--;
            } else if (wc.level)
                IE_CUDA(launch_level(A, R, level_args(wc, d_queue.p + k), wc.mode, wc.gsp, lvl_threads, grids[k],
                                     cstreams[k], wc.split));
            else if (wc.tpl == 8) IE_CUDA(launch_window(A, R, wc.mode, wc.cap, grids[k], cstreams[k]));
            else if (wc.tpl == kChain) IE_CUDA(launch_chain(A, R, wc.mode, wc.cap, grids[k], cstreams[k]));
            else IE_CUDA(launch_batch(A, R, wc.mode, wc.tpl, wc.cap, grids[k], cstreams[k]));
            IE_CUDA(cudaEventRecordWithFlags(cevents[k], cstreams[k], rec));
            IE_CUDA(cudaEventRecord(cjoin[k], cstreams[k]));
            IE_CUDA(cudaStreamWaitEvent(stream, cjoin[k], 0));
            launches++;
        }
        return IE_OK;
    }

    // Runs the class launches (directly, or by replaying the captured graph)
    // and waits for them; records the device time of the run and of each class.
    ie_status launch_classes(const RunArgs& base) { return launch_classes(base, arrays()); }
    ie_status launch_classes(const RunArgs& base, const DevArrays& A, bool graphed = false) {
        IE_TRY(ensure_class_streams(classes.size()));
        if (!evfork) IE_CUDA(cudaEventCreateWithFlags(&evfork, cudaEventDisableTiming));
        std::vector<int> grids;
        IE_TRY(class_grids(base, grids));
        uint64_t launches = 0;
        if (graphed) {
            if (!graph_valid || g_steps != base.steps) {
                if (gexec) IE_CUDA(cudaGraphExecDestroy(gexec));
                if (graph) IE_CUDA(cudaGraphDestroy(graph));
                gexec = nullptr;
                graph = nullptr;
                IE_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
                uint64_t n = 0;
                const ie_status st = enqueue_classes(base, A, grids, n, true);
                cudaGraph_t g = nullptr;
                const cudaError_t ce = cudaStreamEndCapture(stream, &g);
                if (st != IE_OK) {
                    if (g) cudaGraphDestroy(g);
                    return st;
                }
                IE_CUDA(ce);
                graph = g;
                IE_CUDA(cudaGraphInstantiate(&gexec, graph, 0));
                graph_valid = true;
                g_steps = base.steps;
            }
            IE_CUDA(cudaEventRecord(ev0, stream));
            IE_CUDA(cudaGraphLaunch(gexec, stream));
            for (size_t k = 0; k < classes.size(); k++) launches += classes[k]->nitems ? 1 : 0;
        } else {
            IE_CUDA(cudaEventRecord(ev0, stream));
            IE_TRY(enqueue_classes(base, A, grids, launches));
        }
        IE_CUDA(cudaEventRecord(ev1, stream));
        IE_CUDA(cudaEventSynchronize(ev1));
        float ms = 0;
        IE_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        last_ms = ms;
        last_launches = launches;
        class_ms.assign(classes.size(), 0.0);
        for (size_t k = 0; k < classes.size(); k++) {
            if (!classes[k]->nitems) continue;
            float cm = 0;
            IE_CUDA(cudaEventElapsedTime(&cm, cstart[k], cevents[k]));
            class_ms[k] = cm;
        }
        return IE_OK;
    }

    // Autotuner: times a short trial of the schedule for a grid of thread-class
    // thresholds (the device state is saved before and restored after every
    // trial) and keeps the fastest. Returns the chosen thresholds.
    ie_status autotune(const double* temps, uint64_t trial_steps, uint32_t out[4]) {
        if (!initialized) return fail(IE_ERR_INVALID, "call init_random before autotuning");
        if (trial_steps == 0) return fail(IE_ERR_INVALID, "trial_steps must be >= 1");
        if (recs_dirty) IE_TRY(build_record_streams());
        DevBuf<uint64_t> s_spins, s_pos;
        DevBuf<int32_t> s_ei, s_deo;
        DevBuf<double> s_ef;
        IE_TRY(s_spins.alloc(std::max<size_t>(total_words, 1)));
        IE_TRY(s_pos.alloc(count));
        IE_TRY(s_ei.alloc(std::max<size_t>(total_energy, 1)));
        IE_TRY(s_deo.alloc(count));
        IE_TRY(s_ef.alloc(std::max<size_t>(total_energy, 1)));
        auto copy_all = [&](bool save) -> ie_status {
            auto cp = [&](void* dst, const void* src, size_t bytes) -> ie_status {
                IE_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream));
                return IE_OK;
            };
            const size_t w = std::max<size_t>(total_words, 1) * 8, e = std::max<size_t>(total_energy, 1);
            if (save) {
                IE_TRY(cp(s_spins.p, d_spins.p, w));
                IE_TRY(cp(s_pos.p, d_pos.p, count * 8));
                IE_TRY(cp(s_ei.p, d_Ei.p, e * 4));
                IE_TRY(cp(s_deo.p, d_deo.p, count * 4));
                IE_TRY(cp(s_ef.p, d_Ef.p, e * 8));
            } else {
                IE_TRY(cp(d_spins.p, s_spins.p, w));
                IE_TRY(cp(d_pos.p, s_pos.p, count * 8));
                IE_TRY(cp(d_Ei.p, s_ei.p, e * 4));
                IE_TRY(cp(d_deo.p, s_deo.p, count * 4));
                IE_TRY(cp(d_Ef.p, s_ef.p, e * 8));
            }
            IE_CUDA(cudaStreamSynchronize(stream));
            return IE_OK;
        };
        IE_TRY(copy_all(true));
        const uint64_t saved_steps = steps_done;
        if (kernel_form == 0) {
            // Level kernel: the CTA work tile (spin words per item, i.e. 64
            // replica bytes per word) and the CTA size; the fastest of each
            // pair on the best of two trials wins.
            const uint32_t caps[4] = {1024, 2048, 4096, 8192};
            const int thrs[2] = {128, 256};
            double best = 1e300;
            uint32_t bc = lvl_cap;
            int bt = lvl_threads;
            for (uint32_t c : caps)
                for (int t : thrs) {
                    lvl_cap = c;
                    lvl_threads = t;
                    quads_built = false;
                    double ms_best = 1e300;
                    for (int rep = 0; rep < 2; rep++) {
                        IE_TRY(run_batch(temps, trial_steps));
                        IE_TRY(copy_all(false));
                        steps_done = saved_steps;
                        ms_best = std::min(ms_best, last_ms);
                    }
                    if (ms_best < best) {
                        best = ms_best;
                        bc = c;
                        bt = t;
                    }
                }
            lvl_cap = bc;
            lvl_threads = bt;
            quads_built = false;
            IE_TRY(build_quads());
            if (out) {
                out[0] = bc;
                out[1] = (uint32_t)bt;
                out[2] = out[3] = 0;
            }
            return IE_OK;
        }
        // Coordinate search: the (n4, n2) pair of one mode over its grid with
        // the other mode's pair held, integer then f64, two passes; each trial
        // is timed on the same state (restored after it).
        const uint32_t n4s[5] = {256, 512, 768, 1536, 3072}, n2s[3] = {128, 256, 512};
        uint32_t bi[4] = {tune_n4[0], tune_n2[0], tune_n4[1], tune_n2[1]};
        const uint32_t start[4] = {bi[0], bi[1], bi[2], bi[3]};
        auto trial = [&](double& ms) -> ie_status {
            tune_n4[0] = bi[0];
            tune_n2[0] = bi[1];
            tune_n4[1] = bi[2];
            tune_n2[1] = bi[3];
            quads_built = false;
            IE_TRY(run_batch(temps, trial_steps));
            IE_TRY(copy_all(false));
            steps_done = saved_steps;
            ms = last_ms;
            return IE_OK;
        };
        for (int pass = 0; pass < 2; pass++)
            for (int m = 0; m < 2; m++) {
                double best = 1e300;
                uint32_t b4 = bi[2 * m], b2 = bi[2 * m + 1];
                for (uint32_t a4 : n4s)
                    for (uint32_t a2 : n2s) {
                        if (a2 >= a4) continue;
                        bi[2 * m] = a4;
                        bi[2 * m + 1] = a2;
                        double ms = 0;
                        IE_TRY(trial(ms));
                        if (ms < best) {
                            best = ms;
                            b4 = a4;
                            b2 = a2;
                        }
                    }
                bi[2 * m] = b4;
                bi[2 * m + 1] = b2;
            }
        // Single short trials are noisy: the search's choice replaces the
        // starting thresholds only if it is faster on the best of three
        // repeated trials each.
        if (!std::equal(bi, bi + 4, start)) {
            const uint32_t found[4] = {bi[0], bi[1], bi[2], bi[3]};
            double t_found = 1e300, t_start = 1e300;
            for (int rep = 0; rep < 3; rep++) {
                double ms = 0;
                std::copy(found, found + 4, bi);
                IE_TRY(trial(ms));
                t_found = std::min(t_found, ms);
                std::copy(start, start + 4, bi);
                IE_TRY(trial(ms));
                t_start = std::min(t_start, ms);
            }
            std::copy(t_found < t_start ? found : start, (t_found < t_start ? found : start) + 4, bi);
        }
        tune_n4[0] = bi[0];
        tune_n2[0] = bi[1];
        tune_n4[1] = bi[2];
        tune_n2[1] = bi[3];
        quads_built = false;
        IE_TRY(build_quads());
        if (out) std::copy(bi, bi + 4, out);
        return IE_OK;
    }

    // The plain method: one launch per instance, in sequence, on one stream
    // (eight threads per instance, the reference's lane count).
    ie_status run_plain(const double* temps, uint64_t steps, uint32_t first, uint32_t n_inst) {
        if (nt != 1) return fail(IE_ERR_INVALID, "plain runs need single-cell instances");
        if (!initialized) return fail(IE_ERR_INVALID, "call init_random before running");
        if ((uint64_t)first + n_inst > count) return fail(IE_ERR_INVALID, "instance range out of bounds");
        if (steps == 0 || n_inst == 0) return IE_OK;
        if (recs_dirty) IE_TRY(build_record_streams());
        std::vector<double> t(temps, temps + steps);
        IE_TRY(d_temps.upload(t, stream));
        if (kernel_form == 0) {
            // the level kernel, one launch (one CTA) per instance in sequence
            quads_built = false;
            graph_valid = false;
            classes.clear();
            IE_TRY(build_level_classes(desc, insts, false,
                                       [&](uint32_t j) { return j >= first && j < first + n_inst; }, true));
            DevBuf<uint32_t> counters;
            IE_TRY(counters.upload(std::vector<uint32_t>(n_inst, 0), stream));
            IE_CUDA(cudaEventRecord(ev0, stream));
            uint32_t launched = 0;
            for (auto& wcp : classes) {
                const WorkClass& wc = *wcp;
                for (uint32_t k = 0; k < wc.nitems; k++) {
                    RunArgs R = sa_args(steps);
                    LvlArgs L = level_args(wc, counters.p + launched);
                    L.order = wc.order.p + k;
                    L.nitems = 1;
                    IE_CUDA(launch_level(arrays(), R, L, wc.mode, wc.gsp, lvl_threads, 1, stream));
                    launched++;
                }
            }
            IE_CUDA(cudaEventRecord(ev1, stream));
            IE_CUDA(cudaEventSynchronize(ev1));
            float ms = 0;
            IE_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
            last_ms = ms;
            last_launches = launched;
            classes.clear();
            return IE_OK;
        }
        std::vector<uint32_t> quads((size_t)4 * n_inst, 0xffffffffu);
        std::vector<int32_t> qh(n_inst);
        for (uint32_t i = 0; i < n_inst; i++) {
            quads[4 * (size_t)i] = first + i;
            qh[i] = desc[first + i].H;
        }
        DevBuf<uint32_t> dq;
        DevBuf<int32_t> dh;
        IE_TRY(dq.upload(quads, stream));
        IE_TRY(dh.upload(qh, stream));
        std::vector<uint32_t> zeros(n_inst, 0);
        DevBuf<uint32_t> counters;
        IE_TRY(counters.upload(zeros, stream));
        IE_CUDA(cudaEventRecord(ev0, stream));
        for (uint32_t i = 0; i < n_inst; i++) {
            RunArgs R = sa_args(steps);
            R.bulk_ring = bulk_ring ? 1u : 0u;
            R.quads = dq.p + 4 * (size_t)i;
            R.quad_h = dh.p + i;
            R.nquads = 1;
            R.queue = counters.p + i;
            const uint32_t cap = std::max(64u, (desc[first + i].n + 63u) & ~63u);
            if (batch_occupancy(desc[first + i].mode, 1, cap, false) <= 0)
                return fail(IE_ERR_UNSUPPORTED, "instance too large for the plain kernel's shared memory");
            IE_CUDA(launch_batch(arrays(), R, desc[first + i].mode, 1, cap, 1, stream));
        }
        IE_CUDA(cudaEventRecord(ev1, stream));
        IE_CUDA(cudaEventSynchronize(ev1));
        float ms = 0;
        IE_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        last_ms = ms;
        last_launches = n_inst;
        return IE_OK;
    }

    size_t pt_smem(uint32_t cells, int32_t H, uint32_t mode) const {
        const size_t tab = mode == kModeInt ? (size_t)cells * (2 * H + 1) : 0;
        return (tab + (size_t)cells * kReplicas + cells + 2) * sizeof(uint64_t);
    }

    // engine::step n_steps times on instance 0 (all nt cells) with a constant
    // ladder (temps_per_step = 0) or a per-step ladder.
    ie_status run_pt(const double* temps, uint64_t steps, bool per_step, uint32_t exchange_interval) {
        if (!initialized) return fail(IE_ERR_INVALID, "call init_random or set_spins before stepping");
        if (steps == 0) return IE_OK;
        const uint32_t rows = per_step ? (uint32_t)steps : 1u;
        std::vector<double> t(temps, temps + (size_t)rows * nt);
        for (double x : t)
            if (!(x > 0.0) || !std::isfinite(x)) return fail(IE_ERR_INVALID, "temperatures must be positive");
        const InstDesc& d = desc[0];
        const uint32_t L = pop_len ? pop_len : nt;  // one population's ladder
        if (per_step && nt > 1 && d.mode == kModeInt) {
            // exchange tables are per ladder: one launch per step
            for (uint64_t s = 0; s < steps; s++) IE_TRY(run_pt(temps + s * nt, 1, false, exchange_interval));
            return IE_OK;
        }
        if (nt > 1 && d.mode == kModeInt && (xtemps.size() != L || !std::equal(xtemps.begin(), xtemps.end(), t.begin()))) {
            XTables X;
            IE_TRY(build_xtables(t.data(), L, X));
            IE_TRY(d_xtab.upload(X.tab.empty() ? std::vector<uint64_t>(1, 0) : X.tab, stream));
            IE_TRY(d_xoff.upload(X.off, stream));
            IE_TRY(d_xdmax.upload(X.dmax, stream));
            IE_TRY(d_xdund.upload(X.dund, stream));
            IE_TRY(d_dbeta.upload(X.dbeta, stream));
            xtemps.assign(t.begin(), t.begin() + L);
        } else if (nt > 1 && d.mode == kModeF64) {
            std::vector<double> db(std::max<uint32_t>(L, 2) - 1);
            for (uint32_t k = 0; k + 1 < L; k++) db[k] = 1.0 / t[k] - 1.0 / t[k + 1];
            if (per_step) {
                // f64 exchange reads dbeta of the current ladder: one launch per step
                for (uint64_t s = 0; s < steps; s++) IE_TRY(run_pt(temps + s * nt, 1, false, exchange_interval));
                return IE_OK;
            }
            IE_TRY(d_dbeta.upload(db, stream));
        }
        IE_TRY(d_temps.upload(t, stream));
        if (use_cells()) {
            RunArgs X{};
            X.exchange_interval = exchange_interval ? exchange_interval : 1;
            X.xtab = d_xtab.p;
            X.xoff = d_xoff.p;
            X.xdmax = d_xdmax.p;
            X.xdund = d_xdund.p;
            X.dbeta = d_dbeta.p;
            X.pop_len = pop_len;
            if (track_roundtrips) {
                X.labels = d_labels.p;
                X.rt = d_rt.p;
            }
            return run_pt_cells(steps, per_step, X);
        }
        const int block = (int)(((nt * 8) + 31) / 32 * 32);
        if (block > 1024) return fail(IE_ERR_UNSUPPORTED, "at most 128 temperatures per instance");
        const size_t smem = pt_smem(nt, d.H, d.mode);
        if (smem > 227 * 1024) return fail(IE_ERR_UNSUPPORTED, "temperature ladder too large for shared memory");
        IE_CUDA(set_smem_limits(std::max<size_t>(smem, 48 * 1024)));
        RunArgs R{};
        R.temps = d_temps.p;
        R.temps_per_step = per_step ? 1 : 0;
        R.step_base = steps_done;
        R.exchange_interval = exchange_interval ? exchange_interval : 1;
        R.xtab = d_xtab.p;
        R.xoff = d_xoff.p;
        R.xdmax = d_xdmax.p;
        R.xdund = d_xdund.p;
        R.dbeta = d_dbeta.p;
        IE_CUDA(cudaEventRecord(ev0, stream));
        uint64_t launches = 0;
        // f64 resync points and very long runs split into launches of at most
        // 2^30 steps; each launch continues the same trajectory.
        uint64_t done = 0;
        while (done < steps) {
            const uint64_t chunk = std::min<uint64_t>(steps - done, 1ULL << 30);
            R.steps = (uint32_t)chunk;
            R.step_base = steps_done + done;
            R.temps = d_temps.p + (per_step ? done * nt : 0);
            IE_CUDA(launch_pt(arrays(), R, 0, 1, d.mode, block, d.mode == kModeInt ? 2 * d.H + 1 : 0, smem, stream));
            launches++;
            done += chunk;
        }
        IE_CUDA(cudaEventRecord(ev1, stream));
        IE_CUDA(cudaEventSynchronize(ev1));
        float ms = 0;
        IE_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        last_ms = ms;
        last_launches = launches;
        steps_done += steps;
        class_ms.assign(classes.size(), 0.0);
        for (size_t k = 0; k < classes.size(); k++) {
            if (!classes[k]->nitems) continue;
            float cm = 0;
            IE_CUDA(cudaEventElapsedTime(&cm, cstart[k], cevents[k]));
            class_ms[k] = cm;
        }
        return IE_OK;
    }

    ie_status read_words(uint32_t inst0, uint32_t ninst, uint64_t* out) {
        const size_t w0 = desc[inst0].spin;
        const size_t w1 = (inst0 + ninst < count) ? desc[inst0 + ninst].spin : total_words;
        std::vector<uint64_t> h(w1 - w0);
        if (!h.empty())
            IE_CUDA(cudaMemcpyAsync(h.data(), d_spins.p + w0, h.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream));
        IE_CUDA(cudaStreamSynchronize(stream));
        for (size_t i = 0; i < h.size(); i++) out[i] = transpose8x8(h[i]);
        return IE_OK;
    }

    ie_status write_words(uint32_t inst, const uint64_t* in) {
        const InstDesc& d = desc[inst];
        std::vector<uint64_t> h((size_t)d.nt * d.n);
        for (size_t i = 0; i < h.size(); i++) h[i] = transpose8x8(in[i]);
        if (!h.empty())
            IE_CUDA(cudaMemcpyAsync(d_spins.p + d.spin, h.data(), h.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, stream));
        IE_CUDA(launch_energy(arrays(), inst, 1, stream));
        IE_CUDA(cudaStreamSynchronize(stream));
        initialized = true;
        return IE_OK;
    }

    ie_status read_energies(double* out) {
        std::vector<int32_t> ei(total_energy);
        std::vector<double> ef(total_energy);
        IE_CUDA(cudaMemcpyAsync(ei.data(), d_Ei.p, total_energy * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
        IE_CUDA(cudaMemcpyAsync(ef.data(), d_Ef.p, total_energy * sizeof(double), cudaMemcpyDeviceToHost, stream));
        IE_CUDA(cudaStreamSynchronize(stream));
        for (uint32_t i = 0; i < count; i++) {
            const InstDesc& d = desc[i];
            for (size_t k = 0; k < (size_t)d.nt * kReplicas; k++)
                out[d.energy + k] = d.mode == kModeInt ? (double)ei[d.energy + k] : ef[d.energy + k];
        }
        return IE_OK;
    }

    ie_status recompute_energies(double* out) {
        DevBuf<double> tmp;
        IE_TRY(tmp.alloc(std::max<size_t>(total_energy, 1)));
        IE_CUDA(launch_energy_check(arrays(), 0, count, tmp.p, stream));
        IE_CUDA(cudaMemcpyAsync(out, tmp.p, total_energy * sizeof(double), cudaMemcpyDeviceToHost, stream));
        IE_CUDA(cudaStreamSynchronize(stream));
        return IE_OK;
    }

    ie_status check_err() {
        int32_t e = 0;
        IE_CUDA(cudaMemcpy(&e, d_err.p, sizeof(e), cudaMemcpyDeviceToHost));
        if (e) return fail(IE_ERR_DEVICE, "device-side check failed (code " + std::to_string(e) + ")");
        return IE_OK;
    }
};

// First-fit range allocator over [0, cap) in elements of one device pool;
// freed ranges coalesce with their neighbours.
struct RangeAlloc {
    uint64_t cap = 0, used = 0;
    std::map<uint64_t, uint64_t> fr;  // free ranges: offset -> length
    void reset(uint64_t c) {
        cap = c;
        used = 0;
        fr.clear();
        if (c) fr[0] = c;
    }
    bool alloc(uint64_t n, uint64_t align, uint64_t& off) {
        off = 0;
        if (n == 0) return true;
        for (auto it = fr.begin(); it != fr.end(); ++it) {
            const uint64_t b = it->first, e = it->first + it->second;
            const uint64_t a = (b + align - 1) / align * align;
            if (a + n > e) continue;
            fr.erase(it);
            if (a > b) fr[b] = a - b;
            if (a + n < e) fr[a + n] = e - (a + n);
            off = a;
            used += n;
            return true;
        }
        return false;
    }
    void release(uint64_t off, uint64_t n) {
        if (n == 0) return;
        used -= n;
        auto it = fr.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != fr.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            fr.erase(nx);
        }
        if (it != fr.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                fr.erase(it);
            }
        }
    }
};

// One serving request: the host-side layout prepared at submission, its
// placement in the device pools while resident, and its result.
struct ServeReq {
    uint64_t id = 0;
    HostInst h;
    std::vector<uint8_t> clampf;
    std::vector<int8_t> clampv;
    std::vector<uint32_t> recs, wtab, draw_idx;
    std::vector<uint32_t> lrecs, lrecoff, lv_sites, lv_off;  // level kernel: records, offsets, levels
    uint32_t unclamped = 0;
    uint64_t wrec = 0;  // offset of the windowed record stream within recs
    std::vector<double> temps;
    uint32_t key[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint64_t slot = 0, o_row = 0, o_site = 0, o_ent = 0, o_rec = 0, o_win = 0, o_sched = 0, o_lrec = 0;
    uint64_t done = 0;  // steps executed (host mirror of DevArrays::done)
    std::vector<uint64_t> words;
    std::vector<double> energies;
};

// Serving engine: an Engine whose device arrays are pools sized at creation;
// each resident request owns ranges of them (slot: descriptor, key, generator
// position, energies; rows; sites: linear terms, clamps, draw indices and spin
// words; couplings; site records; window table; schedule).
struct ServeEngine {
    Engine eng;
    ie_serve_config cfg{};
    RangeAlloc a_slot, a_row, a_site, a_ent, a_rec, a_win, a_sched, a_lrec;
    std::mutex mu;  // guards pending, finished, next_id
    std::deque<std::unique_ptr<ServeReq>> pending;
    std::vector<std::unique_ptr<ServeReq>> slots;
    std::map<uint64_t, std::unique_ptr<ServeReq>> finished;
    uint64_t next_id = 1;
    uint32_t n_active = 0;
    bool set_changed = true;     // a request was admitted or retired since the work items were built
    std::vector<uint32_t> unit;  // per slot: sites one unit of the site budget covers
    // level kernel: per slot the steps of this tick, and the device cycles per
    // step its work item measured in the last tick (0: not yet run)
    std::vector<uint32_t> plan;
    std::vector<float> cost;
    DevBuf<uint32_t> d_plan;
    DevBuf<float> d_cost;
    double tick_cycles = 0;
    static constexpr uint32_t kProbeSteps = 64;  // a request's first tick on the level kernel

    bool level() const { return cfg.kernel_form == 0; }
    uint64_t rec_cap() const { return level() ? 0 : 8 * cfg.max_sites + 4 * cfg.max_couplings + kChunk; }
    // level records: 4 header words per site, then per coupling one word
    // (integer) or three (f64), rows padded to 4
    uint64_t lrec_cap() const { return level() ? 13 * cfg.max_sites + 3 * cfg.max_couplings + 4 : 0; }
    uint64_t win_cap() const { return (uint64_t)kWT * ((cfg.max_sites + kWin - 1) / kWin + cfg.max_requests); }

    ie_status create(const ie_serve_config* c) {
        if (c) cfg = *c;
        if (!cfg.max_requests) cfg.max_requests = 4096;
        if (!cfg.site_budget) cfg.site_budget = 65536;
        if (!cfg.max_sites) cfg.max_sites = 1ull << 24;
        if (!cfg.max_couplings) cfg.max_couplings = 1ull << 27;
        if (!cfg.max_schedule_steps) cfg.max_schedule_steps = 1ull << 25;
        if (!cfg.tick_us) cfg.tick_us = 200000;
        if (cfg.max_sites >= (1ull << 32) || cfg.max_couplings >= (1ull << 32))
            return fail(IE_ERR_INVALID, "max_sites and max_couplings must be below 2^32");
        IE_TRY(eng.setup_device(cfg.device));
        if (cfg.kernel_form < 0 || cfg.kernel_form > 1) return fail(IE_ERR_INVALID, "kernel_form must be 0 or 1");
        eng.kernel_form = cfg.kernel_form;
        eng.serving = true;
        // requests above 1024 sites keep their spins in global memory, so a
        // request can run on a cluster of CTAs
        eng.lvl_cap = 1024;
        const uint32_t S = cfg.max_requests;
        eng.nt = 1;
        eng.count = S;
        eng.desc.assign(S, InstDesc{});
        eng.insts.assign(S, HostInst{});
        eng.active.assign(S, 0);
        IE_TRY(eng.d_desc.alloc(S));
        IE_TRY(eng.d_keys.alloc(8 * (size_t)S));
        IE_TRY(eng.d_pos.alloc(S));
        IE_TRY(eng.d_deo.alloc(S));
        IE_TRY(eng.d_done.alloc(S));
        IE_TRY(d_plan.alloc(S));
        IE_TRY(d_cost.upload(std::vector<float>(S, 0.0f), eng.stream));
        plan.assign(S, 0);
        cost.assign(S, 0.0f);
        {
            int khz = 0;
            IE_CUDA(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, eng.device));
            tick_cycles = (double)cfg.tick_us * (double)khz / 1000.0;
        }
        IE_TRY(eng.d_unclamped.alloc(S));
        IE_TRY(eng.d_Ei.alloc((size_t)kReplicas * S));
        IE_TRY(eng.d_Ef.alloc((size_t)kReplicas * S));
        IE_TRY(eng.d_rows.alloc(cfg.max_sites + S));
        IE_TRY(eng.d_lin.alloc(cfg.max_sites));
        IE_TRY(eng.d_linp.alloc(cfg.max_sites));
        IE_TRY(eng.d_clampf.alloc(cfg.max_sites));
        IE_TRY(eng.d_clampv.alloc(cfg.max_sites));
        IE_TRY(eng.d_draw_idx.alloc(cfg.max_sites));
        IE_TRY(eng.d_spins.alloc(cfg.max_sites));
        IE_TRY(eng.d_ents.alloc(std::max<uint64_t>(cfg.max_couplings, 1)));
        IE_TRY(eng.d_cols.alloc(std::max<uint64_t>(cfg.max_couplings, 1)));
        IE_TRY(eng.d_vals.alloc(std::max<uint64_t>(cfg.max_couplings, 1)));
        IE_TRY(eng.d_recs.alloc(rec_cap() + kChunk));
        IE_TRY(eng.d_wtab.alloc(level() ? 1 : win_cap()));
        if (level()) {
            IE_TRY(eng.d_lrecs.alloc(lrec_cap()));
            IE_TRY(eng.d_recoff.alloc(cfg.max_sites));
            eng.h_recoff.assign(cfg.max_sites, 0);
            eng.lv_sites.assign(S, {});
            eng.lv_off.assign(S, {});
        }
        IE_TRY(eng.d_temps.alloc(cfg.max_schedule_steps));
        IE_TRY(eng.d_att.alloc(1));
        IE_TRY(eng.d_acc.alloc(1));
        IE_TRY(eng.d_err.upload(std::vector<int32_t>(1, 0), eng.stream));
        IE_TRY(eng.d_queue.alloc(64));
        IE_CUDA(cudaMemsetAsync(eng.d_recs.p, 0, eng.d_recs.n * sizeof(uint32_t), eng.stream));
        IE_CUDA(cudaStreamSynchronize(eng.stream));
        a_slot.reset(S);
        a_row.reset(cfg.max_sites + S);
        a_site.reset(cfg.max_sites);
        a_ent.reset(cfg.max_couplings);
        a_rec.reset(rec_cap());
        a_win.reset(level() ? 0 : win_cap());
        a_sched.reset(cfg.max_schedule_steps);
        a_lrec.reset(lrec_cap());
        slots.resize(S);
        eng.initialized = true;
        eng.recs_dirty = false;
        return IE_OK;
    }

    // Host-side preparation of one request (any thread; touches no shared state).
    ie_status prepare(const ie_problem* p, uint64_t seed, const double* temps, uint64_t n_steps,
                      const uint8_t* is_clamped, const int8_t* clamp_val, ServeReq& r) const {
        if (!p || !temps) return fail(IE_ERR_INVALID, "NULL argument");
        if (p->num_vars == 0) return fail(IE_ERR_INVALID, "num_vars must be > 0");
        if (n_steps == 0) return fail(IE_ERR_INVALID, "n_steps must be >= 1");
        IE_TRY(ingest(p, cfg.force_f64 != 0, r.h));
        const uint32_t n = r.h.n;
        r.temps.assign(temps, temps + n_steps);
        for (double x : r.temps)
            if (!(x > 0.0) || !std::isfinite(x)) return fail(IE_ERR_INVALID, "temperatures must be positive");
        r.clampf.assign(n, 0);
        r.clampv.assign(n, 0);
        if (is_clamped)
            for (uint32_t i = 0; i < n; i++) {
                r.clampf[i] = is_clamped[i] ? 1 : 0;
                r.clampv[i] = (is_clamped[i] && clamp_val && clamp_val[i] == 1) ? 1 : 0;
            }
        r.draw_idx.assign(n, 0);
        uint32_t c = 0;
        for (uint32_t v = 0; v < n; v++) {
            r.draw_idx[v] = c;
            if (!r.clampf[v]) c++;
        }
        r.unclamped = c;
        if (level()) {
            const LvlSource src = Engine::lvl_source(r.h, r.clampf.data());
            r.lrecoff.assign(n, 0);
            level_records(src, r.lrecs, r.lrecoff.data());
            site_levels(src, r.lv_sites, r.lv_off);
        } else {
            uint64_t off = 0, len = 0;
            IE_TRY(build_records(r.h, r.clampf, 0, r.recs, off, len));
            IE_TRY(window_records(r.h, r.clampf, 0, r.recs, 0, r.wrec));
            window_table(r.h, r.wtab);
        }
        chacha_key_from_u64(seed, r.key);
        // capacity checks: the request alone must fit every pool and the
        // shared memory of the kernels that can run it
        if (n + 1 > a_row.cap || n > a_site.cap || r.h.nnz > a_ent.cap || r.recs.size() > a_rec.cap ||
            r.lrecs.size() > a_lrec.cap ||
            r.wtab.size() > a_win.cap || n_steps > a_sched.cap)
            return fail(IE_ERR_OOM, "request exceeds the serving engine's capacity");
        return IE_OK;
    }

    static uint64_t bytes_of(const ServeReq& r) {
        const uint64_t n = r.h.n;
        return (n + 1) * 4 + n * (8 + 4 + 1 + 1 + 4 + 8 + 4) + r.h.nnz * (4 + 4 + 8) + r.recs.size() * 4 +
               r.lrecs.size() * 4 +
               r.wtab.size() * 4 + r.temps.size() * 8 + sizeof(InstDesc) + 32 + 8 + 4 + 8 + 4 +
               kReplicas * (4 + 8);
    }

    // Reserves every pool range of r; all or nothing.
    bool place(ServeReq& r) {
        const uint64_t n = r.h.n;
        uint64_t o[8];
        RangeAlloc* al[8] = {&a_slot, &a_row, &a_site, &a_ent, &a_rec, &a_win, &a_sched, &a_lrec};
        const uint64_t len[8] = {1, n + 1, n, r.h.nnz, r.recs.size(), r.wtab.size(), r.temps.size(), r.lrecs.size()};
        const uint64_t align[8] = {1, 4, 4, 4, kChunk, 4, 2, 4};
        int k = 0;
        for (; k < 8; k++)
            if (!al[k]->alloc(len[k], align[k], o[k])) break;
        if (k < 8) {
            for (int j = 0; j < k; j++) al[j]->release(o[j], len[j]);
            return false;
        }
        r.slot = o[0];
        r.o_row = o[1];
        r.o_site = o[2];
        r.o_ent = o[3];
        r.o_rec = o[4];
        r.o_win = o[5];
        r.o_sched = o[6];
        r.o_lrec = o[7];
        return true;
    }

    void unplace(const ServeReq& r) {
        const uint64_t n = r.h.n;
        a_slot.release(r.slot, 1);
        a_row.release(r.o_row, n + 1);
        a_site.release(r.o_site, n);
        a_ent.release(r.o_ent, r.h.nnz);
        a_rec.release(r.o_rec, r.recs.size());
        a_win.release(r.o_win, r.wtab.size());
        a_sched.release(r.o_sched, r.temps.size());
        a_lrec.release(r.o_lrec, r.lrecs.size());
    }

    template <typename T>
    ie_status put(T* base, uint64_t off, const T* src, size_t count) {
        if (count) IE_CUDA(cudaMemcpyAsync(base + off, src, count * sizeof(T), cudaMemcpyHostToDevice, eng.stream));
        return IE_OK;
    }

    // Uploads an admitted request and draws its initial state (ultimate.rs:248-290).
    ie_status upload(ServeReq& r) {
        const HostInst& h = r.h;
        const uint32_t s = (uint32_t)r.slot;
        InstDesc& d = eng.desc[s];
        d = InstDesc{};
        d.n = h.n;
        d.H = h.H;
        d.mode = h.mode;
        d.nt = 1;
        d.row = r.o_row;
        d.ent = r.o_ent;
        d.site = r.o_site;
        d.spin = r.o_site;
        d.energy = (uint64_t)s * kReplicas;
        d.stat = 0;
        d.rec = r.o_rec;
        d.wrec = r.o_rec + r.wrec;
        d.owner = s;
        d.rec_len = r.recs.size();
        d.win = r.o_win;
        d.sched = r.o_sched;
        d.sched_len = r.temps.size();
        HostInst& e = eng.insts[s];
        e = HostInst();
        e.n = h.n;
        e.H = h.H;
        e.mode = h.mode;
        e.nnz = h.nnz;
        e.windowed_ok = h.windowed_ok;
        e.has_wtab = h.has_wtab;
        IE_TRY(put(eng.d_rows.p, r.o_row, h.rows.data(), h.rows.size()));
        IE_TRY(put(eng.d_lin.p, r.o_site, h.lin.data(), h.n));
        if (h.mode == kModeInt) {
            IE_TRY(put(eng.d_linp.p, r.o_site, h.linp.data(), h.n));
            IE_TRY(put(eng.d_ents.p, r.o_ent, h.ents.data(), h.nnz));
        }
        IE_TRY(put(eng.d_cols.p, r.o_ent, h.cols.data(), h.nnz));
        IE_TRY(put(eng.d_vals.p, r.o_ent, h.vals.data(), h.nnz));
        IE_TRY(put(eng.d_clampf.p, r.o_site, r.clampf.data(), h.n));
        IE_TRY(put(eng.d_clampv.p, r.o_site, r.clampv.data(), h.n));
        IE_TRY(put(eng.d_draw_idx.p, r.o_site, r.draw_idx.data(), h.n));
        IE_TRY(put(eng.d_recs.p, r.o_rec, r.recs.data(), r.recs.size()));
        IE_TRY(put(eng.d_wtab.p, r.o_win, r.wtab.data(), r.wtab.size()));
        IE_TRY(put(eng.d_temps.p, r.o_sched, r.temps.data(), r.temps.size()));
        if (level()) {
            IE_TRY(put(eng.d_lrecs.p, r.o_lrec, r.lrecs.data(), r.lrecs.size()));
            const uint32_t b16 = (uint32_t)(r.o_lrec / 4);
            for (uint32_t v = 0; v < h.n; v++) eng.h_recoff[r.o_site + v] = r.lrecoff[v] + b16;
            IE_TRY(put(eng.d_recoff.p, r.o_site, eng.h_recoff.data() + r.o_site, h.n));
            eng.lv_sites[s] = r.lv_sites;
            eng.lv_off[s] = r.lv_off;
        }
        IE_TRY(put(eng.d_keys.p, 8 * (uint64_t)s, r.key, 8));
        IE_TRY(put(eng.d_unclamped.p, s, &r.unclamped, 1));
        IE_TRY(put(eng.d_desc.p, s, &d, 1));
        IE_CUDA(cudaMemsetAsync(eng.d_pos.p + s, 0, sizeof(uint64_t), eng.stream));
        IE_CUDA(cudaMemsetAsync(eng.d_deo.p + s, 0, sizeof(int32_t), eng.stream));
        IE_CUDA(cudaMemsetAsync(eng.d_done.p + s, 0, sizeof(uint64_t), eng.stream));
        IE_CUDA(cudaMemsetAsync(d_cost.p + s, 0, sizeof(float), eng.stream));
        cost[s] = 0.0f;
        const DevArrays A = eng.arrays();
        IE_CUDA(launch_init(A, s, 1, eng.d_draw_idx.p, eng.d_unclamped.p, eng.stream));
        IE_CUDA(launch_energy(A, s, 1, eng.stream));
        eng.active[s] = 1;
        r.done = 0;
        return IE_OK;
    }

    // Copies a finished request's result to the host and frees its ranges.
    ie_status retire(std::unique_ptr<ServeReq>& rp) {
        ServeReq& r = *rp;
        const uint32_t s = (uint32_t)r.slot;
        const InstDesc& d = eng.desc[s];
        std::vector<uint64_t> w(r.h.n);
        std::vector<int32_t> ei(kReplicas);
        r.energies.assign(kReplicas, 0.0);
        IE_CUDA(cudaMemcpyAsync(w.data(), eng.d_spins.p + d.spin, w.size() * 8, cudaMemcpyDeviceToHost, eng.stream));
        if (d.mode == kModeInt)
            IE_CUDA(cudaMemcpyAsync(ei.data(), eng.d_Ei.p + d.energy, kReplicas * 4, cudaMemcpyDeviceToHost, eng.stream));
        else
            IE_CUDA(cudaMemcpyAsync(r.energies.data(), eng.d_Ef.p + d.energy, kReplicas * 8, cudaMemcpyDeviceToHost,
                                    eng.stream));
        IE_CUDA(cudaStreamSynchronize(eng.stream));
        if (d.mode == kModeInt)
            for (int k = 0; k < kReplicas; k++) r.energies[k] = (double)ei[k];
        r.words.resize(w.size());
        for (size_t i = 0; i < w.size(); i++) r.words[i] = transpose8x8(w[i]);
        eng.active[s] = 0;
        unplace(r);
        // the host layout is no longer needed
        r.h = HostInst();
        r.recs.clear();
        r.wtab.clear();
        r.lrecs.clear();
        r.lrecoff.clear();
        r.lv_sites.clear();
        r.lv_off.clear();
        r.temps.clear();
        r.clampf.clear();
        r.clampv.clear();
        r.draw_idx.clear();
        std::lock_guard<std::mutex> lk(mu);
        finished[r.id] = std::move(rp);
        return IE_OK;
    }

    ie_status tick(uint32_t* na, uint32_t* np, uint32_t* nf) {
        // admission, first come first served: stop at the first request that
        // does not fit, so a large request is not overtaken indefinitely
        std::vector<ServeReq*> admitted;
        {
            std::lock_guard<std::mutex> lk(mu);
            while (!pending.empty()) {
                ServeReq& r = *pending.front();
                if (!place(r)) break;
                const uint64_t s = r.slot;
                slots[s] = std::move(pending.front());
                pending.pop_front();
                admitted.push_back(slots[s].get());
            }
        }
        for (ServeReq* r : admitted) {
            IE_TRY(upload(*r));
            n_active++;
            set_changed = true;
        }
        eng.last_ms = 0.0;
        eng.last_launches = 0;
        if (n_active) {
            if (set_changed || !eng.quads_built) {
                // the resident set changed: new work items, and per slot the
                // sites one budget unit covers (its item's sites on the level
                // kernel, its own on the per-lane kernels)
                IE_TRY(eng.build_quads());
                unit.assign(cfg.max_requests, 0);
                for (const LvlItem& it : eng.lvh.items)
                    for (uint32_t k = 0; k < it.nmem; k++)
                        unit[eng.lvh.members[it.mem0 + k].inst] = (it.sites + it.split - 1) / it.split;
                set_changed = false;
            }
            RunArgs R{};
            R.temps = eng.d_temps.p;
            R.temps_per_step = 1;
            R.exchange_interval = 1;
            R.serve = 1;
            R.site_budget = cfg.site_budget;
            // the tick's plan: about tick_us of device time per work item
            for (uint32_t s = 0; s < cfg.max_requests; s++) {
                plan[s] = 0;
                if (!slots[s] || !eng.active[s]) continue;
                const ServeReq& r = *slots[s];
                const uint64_t left = r.temps.size() - r.done;
                const uint32_t u = unit[s] ? unit[s] : r.h.n;
                uint64_t want = std::max<uint64_t>(1, cfg.site_budget / std::max<uint32_t>(u, 1));
                if (level()) {
                    want = cost[s] > 0.0f ? std::max<uint64_t>(1, (uint64_t)(tick_cycles / (double)cost[s]))
                                          : std::min<uint64_t>(want, kProbeSteps);
                }
                plan[s] = (uint32_t)std::min<uint64_t>({left, want, 0xFFFFFFFFull});
            }
            IE_CUDA(cudaMemcpyAsync(d_plan.p, plan.data(), plan.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                    eng.stream));
            R.plan = d_plan.p;
            R.cost = level() ? d_cost.p : nullptr;
            IE_TRY(eng.launch_classes(R));
            IE_TRY(eng.check_err());
            if (level())
                IE_CUDA(cudaMemcpy(cost.data(), d_cost.p, cost.size() * sizeof(float), cudaMemcpyDeviceToHost));
            for (uint32_t s = 0; s < cfg.max_requests; s++) {
                if (!slots[s] || !eng.active[s]) continue;
                ServeReq& r = *slots[s];
                r.done += plan[s];
                if (r.done == r.temps.size()) {
                    IE_TRY(retire(slots[s]));
                    slots[s].reset();
                    n_active--;
                    set_changed = true;
                }
            }
        }
        std::lock_guard<std::mutex> lk(mu);
        if (na) *na = n_active;
        if (np) *np = (uint32_t)pending.size();
        if (nf) *nf = (uint32_t)finished.size();
        return IE_OK;
    }
};

bool cfg_valid(const ie_config* c, std::string& why) {
    if (!c) {
        why = "config is NULL";
        return false;
    }
    if (c->num_pops > 64) {
        why = "at most 64 populations";
        return false;
    }
    if (c->num_slices != 0 && c->num_slices != 1) {
        why = "num_slices must be 1 (the Trotter branch is not on this path)";
        return false;
    }
    return true;
}

}  // namespace

struct ie_handle {
    Engine eng;
    ie_config cfg{};
    double offset = 0.0;
    DevBuf<double> d_inc_e;
    DevBuf<uint64_t> d_inc_state;
    bool have_incumbent = false;
};

struct ie_batch {
    Engine eng;
};

struct ie_serve {
    ServeEngine s;
};

namespace ie {
void set_last_error(const char* msg) { g_err = msg; }
}  // namespace ie

extern "C" {

const char* ie_last_error(void) { return g_err.c_str(); }
int ie_abi_version(void) { return 1; }

ie_status ie_geometric_temps(double temp_max, double temp_min, uint32_t num_temps, double* out) {
    if (!out || num_temps == 0) return fail(IE_ERR_INVALID, "num_temps must be >= 1");
    const double f = num_temps > 1 ? std::pow(temp_min / temp_max, 1.0 / (double)(num_temps - 1)) : 1.0;
    for (uint32_t i = 0; i < num_temps; i++) out[i] = temp_max * powi_rt(f, (int)i);
    return IE_OK;
}

ie_status ie_suggested_temp_range(const ie_problem* p, double* tmax, double* tmin) {
    if (!p || !tmax || !tmin) return fail(IE_ERR_INVALID, "NULL argument");
    double max_local = 0.0, min_nz = std::numeric_limits<double>::infinity();
    for (uint64_t i = 0; i < p->num_vars; i++) {
        double local = std::fabs(p->linear[i]);
        if (p->linear[i] != 0.0) min_nz = std::min(min_nz, std::fabs(p->linear[i]));
        for (uint64_t k = p->row_offsets[i]; k < p->row_offsets[i + 1]; k++) {
            const double w = p->values[k];
            local += std::fabs(w);
            if (w != 0.0) min_nz = std::min(min_nz, std::fabs(w));
        }
        max_local = std::max(max_local, local);
    }
    if (max_local == 0.0 || !std::isfinite(min_nz)) {
        *tmax = 1.0;
        *tmin = 0.1;
        return IE_OK;
    }
    const double t_max = max_local / 0.693147180559945309417232121458176568;  // LN_2
    const double t_min = std::min(min_nz / std::log(100.0), t_max * 0.5);
    *tmax = t_max;
    *tmin = t_min;
    return IE_OK;
}

ie_status ie_create(const ie_problem* problem, const ie_config* config, ie_handle** out) {
    if (!out) return fail(IE_ERR_INVALID, "out is NULL");
    *out = nullptr;
    std::string why;
    if (!cfg_valid(config, why)) return fail(config ? IE_ERR_UNSUPPORTED : IE_ERR_INVALID, why);
    std::unique_ptr<ie_handle> h(new ie_handle());
    h->cfg = *config;
    if (h->cfg.num_temps == 0) h->cfg.num_temps = 10;
    if (h->cfg.exchange_interval == 0) h->cfg.exchange_interval = 1;
    if (h->cfg.num_temps > 128) return fail(IE_ERR_UNSUPPORTED, "at most 128 temperatures");
    if (h->cfg.pt_path < 0 || h->cfg.pt_path > 3) return fail(IE_ERR_INVALID, "pt_path must be 0, 1, 2 or 3");
    if (h->cfg.kernel_form < 0 || h->cfg.kernel_form > 1) return fail(IE_ERR_INVALID, "kernel_form must be 0 or 1");
    if (h->cfg.pt_path == 3 && h->cfg.kernel_form != 0)
        return fail(IE_ERR_INVALID, "pt_path 3 (one launch per cell) runs on the level kernel (kernel_form 0)");
    IE_TRY(h->eng.setup_device(config->device));
    h->eng.pt_path = h->cfg.pt_path;
    h->eng.kernel_form = h->cfg.kernel_form;
    if (h->cfg.max_cluster > 16 || (h->cfg.max_cluster & (h->cfg.max_cluster - 1)))
        return fail(IE_ERR_INVALID, "max_cluster must be 0, 1, 2, 4, 8 or 16");
    h->eng.lvl_cluster_max = h->cfg.max_cluster;
    if (h->cfg.bit_sliced < -1 || h->cfg.bit_sliced > 1) return fail(IE_ERR_INVALID, "bit_sliced must be -1, 0 or 1");
    h->eng.pmj_policy = h->cfg.bit_sliced;
    const uint32_t pops = std::max<uint32_t>(h->cfg.num_pops, 1);
    if (pops > 1) {
        // QuantumField::new(n, 1, num_temps, num_pops): cell t + num_temps * p,
        // each a work item of the batched kernels
        h->eng.pop_len = h->cfg.num_temps;
        h->eng.periodic_resync = false;
    }
    IE_TRY(h->eng.build(problem, 1, h->cfg.num_temps * pops, &config->seed, config->force_f64 != 0));
    h->offset = problem->energy_offset;
    IE_TRY(h->d_inc_e.upload(std::vector<double>(1, std::numeric_limits<double>::infinity()), h->eng.stream));
    IE_TRY(h->d_inc_state.alloc(std::max<uint64_t>((problem->num_vars + 63) / 64, 1)));
    IE_CUDA(cudaMemsetAsync(h->d_inc_state.p, 0, h->d_inc_state.n * sizeof(uint64_t), h->eng.stream));
    IE_CUDA(cudaStreamSynchronize(h->eng.stream));
    *out = h.release();
    return IE_OK;
}

ie_status ie_destroy(ie_handle* h) {
    delete h;
    return IE_OK;
}

ie_status ie_set_clamps(ie_handle* h, const uint8_t* is_clamped, const int8_t* clamp_val) {
    if (!h) return fail(IE_ERR_INVALID, "handle is NULL");
    IE_CUDA(cudaSetDevice(h->eng.device));
    return h->eng.set_clamps(0, is_clamped, clamp_val);
}

ie_status ie_set_init_probs(ie_handle* h, const double* probs) {
    if (!h) return fail(IE_ERR_INVALID, "handle is NULL");
    if (!probs) {
        h->eng.init_probs.clear();
        return IE_OK;
    }
    h->eng.init_probs.assign(probs, probs + h->eng.desc[0].n);
    return IE_OK;
}

ie_status ie_init_random(ie_handle* h) {
    if (!h) return fail(IE_ERR_INVALID, "handle is NULL");
    IE_CUDA(cudaSetDevice(h->eng.device));
    return h->eng.init_random();
}

ie_status ie_set_spins(ie_handle* h, const uint64_t* words) {
    if (!h || !words) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(h->eng.device));
    return h->eng.write_words(0, words);
}

// A population handle's cells take temps[t % num_temps]: the ladder rows are
// repeated once per population.
static std::vector<double> ladder_rows(const Engine& E, const double* temps, uint64_t rows) {
    const uint32_t L = E.pop_len ? E.pop_len : E.nt;
    std::vector<double> out((size_t)rows * E.nt);
    for (uint64_t s = 0; s < rows; s++)
        for (uint32_t c = 0; c < E.nt; c++) out[(size_t)s * E.nt + c] = temps[(size_t)s * L + c % L];
    return out;
}

ie_status ie_step(ie_handle* h, const double* temps, uint32_t n_temps, uint64_t n_steps) {
    if (!h || !temps) return fail(IE_ERR_INVALID, "NULL argument");
    if (n_temps != h->cfg.num_temps) return fail(IE_ERR_INVALID, "n_temps must equal the handle's num_temps");
    IE_CUDA(cudaSetDevice(h->eng.device));
    if (!h->eng.pop_len) IE_TRY(h->eng.run_pt(temps, n_steps, false, h->cfg.exchange_interval));
    else IE_TRY(h->eng.run_pt(ladder_rows(h->eng, temps, 1).data(), n_steps, false, h->cfg.exchange_interval));
    return h->eng.check_err();
}

ie_status ie_run_schedule(ie_handle* h, const double* temps, uint32_t n_temps, uint64_t n_steps) {
    if (!h || !temps) return fail(IE_ERR_INVALID, "NULL argument");
    if (n_temps != h->cfg.num_temps) return fail(IE_ERR_INVALID, "n_temps must equal the handle's num_temps");
    IE_CUDA(cudaSetDevice(h->eng.device));
    if (!h->eng.pop_len) IE_TRY(h->eng.run_pt(temps, n_steps, true, h->cfg.exchange_interval));
    else IE_TRY(h->eng.run_pt(ladder_rows(h->eng, temps, n_steps).data(), n_steps, true, h->cfg.exchange_interval));
    return h->eng.check_err();
}

ie_status ie_run_pt(ie_handle* h) {
    if (!h) return fail(IE_ERR_INVALID, "handle is NULL");
    if (h->eng.pop_len) return fail(IE_ERR_INVALID, "a handle with num_pops > 1 runs ie_run_pa");
    IE_CUDA(cudaSetDevice(h->eng.device));
    std::vector<double> temps(h->eng.nt);
    IE_TRY(ie_geometric_temps(h->cfg.temp_max, h->cfg.temp_min, h->eng.nt, temps.data()));
    const uint32_t n_words = (uint32_t)h->d_inc_state.n;
    for (uint64_t ex = 0; ex < h->cfg.total_exchanges; ex++) {
        IE_TRY(h->eng.run_pt(temps.data(), h->cfg.sweeps_per_exchange, false, h->cfg.exchange_interval));
        if (h->cfg.use_icm) IE_TRY(h->eng.icm_sweep());  // ultimate.rs:326-328
        IE_CUDA(launch_incumbent(h->eng.arrays(), 0, h->offset, h->d_inc_e.p, h->d_inc_state.p, n_words,
                                 h->eng.stream));
    }
    IE_CUDA(cudaStreamSynchronize(h->eng.stream));
    h->have_incumbent = true;
    return h->eng.check_err();
}

// UltimateSolver::solve_population_annealing_diag (ultimate.rs:576-852) with
// either ladder mode and optional ICM. The steps, energies and
// resampled configurations stay on the device; per stage the host reads the
// cold-level energies (64 per population) for the weights and, on a
// resampling event, takes the offset and shuffle draws from the master
// stream at the device's position and advances it.
ie_status ie_run_pa(ie_handle* h, const ie_pa_config* pc, ie_pa_report* rep) {
    if (!h || !pc) return fail(IE_ERR_INVALID, "NULL argument");
    Engine& E = h->eng;
    if (!E.pop_len) return fail(IE_ERR_INVALID, "ie_run_pa needs a handle created with num_pops > 1");
    if (pc->ladder_mode != 0 && pc->ladder_mode != 1) return fail(IE_ERR_INVALID, "ladder_mode must be 0 or 1");
    if (std::isnan(pc->ess_threshold)) return fail(IE_ERR_INVALID, "ess_threshold is NaN");
    IE_CUDA(cudaSetDevice(E.device));
    const uint32_t L = E.pop_len, pops = E.nt / L, R = pops * (uint32_t)kReplicas;
    const double tmax = h->cfg.temp_max, tmin = h->cfg.temp_min;
    const uint32_t mode = E.desc[0].mode;
    const uint64_t n = E.desc[0].n;
    const size_t words = (size_t)E.nt * n;
    cudaStream_t st = E.stream;
    HostStream rng{};
    std::copy(E.keys.begin(), E.keys.begin() + 8, rng.key);
    auto run_steps = [&](const std::vector<double>& temps, uint64_t k) -> ie_status {
        if (k == 0) return IE_OK;
        return E.run_pt(ladder_rows(E, temps.data(), 1).data(), k, false, 1);
    };
    // StepScratch::for_field: a fresh scratch starts in the even DEO phase
    auto fresh_scratch = [&]() -> ie_status {
        IE_CUDA(cudaMemsetAsync(E.d_deo.p, 0, sizeof(int32_t), st));
        return IE_OK;
    };

    // ladder shape alpha_t in log-temperature space, tuned on a throwaway field
    const double denom = (double)std::max<uint32_t>(L - 1, 1);
    std::vector<double> alphas(L), temps(L);
    for (uint32_t t = 0; t < L; t++) alphas[t] = (double)t / denom;
    if (L >= 3 && pc->ladder_tuning_iters > 0 && pc->ladder_tuning_steps > 0) {
        IE_TRY(E.init_random());
        IE_TRY(fresh_scratch());
        std::vector<uint64_t> att(L - 1), acc(L - 1);
        std::vector<double> rates(L - 1), sp(L - 1);
        const bool feedback = pc->ladder_mode == 1;
        std::vector<unsigned long long> rt(1 + 2 * (size_t)L);
        // tracking belongs to the throwaway tuning field only: off again on
        // every way out of this block
        struct TrackingOff {
            Engine& e;
            ~TrackingOff() { e.track_roundtrips = false; }
        } tracking_off{E};
        if (feedback) {
            IE_TRY(E.d_labels.alloc(E.total_energy));
            IE_TRY(E.d_rt.alloc(rt.size()));
            E.track_roundtrips = true;
        }
        for (uint32_t it = 0; it < pc->ladder_tuning_iters; it++) {
            for (uint32_t t = 0; t < L; t++) temps[t] = tmax * std::pow(tmin / tmax, alphas[t]);
            if (feedback) {
                // reset_roundtrip_stats (engine.rs:529-536): counts and labels to zero
                IE_CUDA(cudaMemsetAsync(E.d_labels.p, 0, E.total_energy, st));
                IE_CUDA(cudaMemsetAsync(E.d_rt.p, 0, rt.size() * sizeof(unsigned long long), st));
                IE_TRY(run_steps(temps, pc->ladder_tuning_steps));
                IE_CUDA(cudaMemcpyAsync(rt.data(), E.d_rt.p, rt.size() * sizeof(unsigned long long),
                                        cudaMemcpyDeviceToHost, st));
                IE_CUDA(cudaStreamSynchronize(st));
                // KTHT redistribution only with enough round trips (ultimate.rs:662-677)
                if (rt[0] >= (unsigned long long)L) {
                    std::vector<double> flow(L);
                    for (uint32_t t = 0; t < L; t++) {
                        const unsigned long long u = rt[1 + t], dn = rt[1 + L + t];
                        flow[t] = u + dn == 0 ? 0.0 : (double)u / (double)(u + dn);
                    }
                    alphas = pa::feedback_optimized_alphas(alphas, flow, 0.5);
                    alphas[0] = 0.0;
                    alphas[L - 1] = 1.0;
                }
                continue;
            }
            IE_CUDA(cudaMemsetAsync(E.d_att.p, 0, (L - 1) * sizeof(uint64_t), st));
            IE_CUDA(cudaMemsetAsync(E.d_acc.p, 0, (L - 1) * sizeof(uint64_t), st));
            IE_TRY(run_steps(temps, pc->ladder_tuning_steps));
            IE_CUDA(cudaMemcpyAsync(att.data(), E.d_att.p, (L - 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
            IE_CUDA(cudaMemcpyAsync(acc.data(), E.d_acc.p, (L - 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
            IE_CUDA(cudaStreamSynchronize(st));
            for (uint32_t t = 0; t + 1 < L; t++) {
                rates[t] = att[t] == 0 ? 0.0 : (double)acc[t] / (double)att[t];
                sp[t] = alphas[t + 1] - alphas[t];
            }
            const std::vector<double> ns = pa::adapt_spacings(sp.data(), rates.data(), L - 1);
            double a = 0.0;
            for (uint32_t t = 0; t + 1 < L; t++) {
                a += ns[t];
                alphas[t + 1] = a;
            }
            alphas[L - 1] = 1.0;
        }
    }

    // production population (a fresh scratch: no round-trip tracking)
    IE_TRY(E.init_random());
    IE_TRY(fresh_scratch());
    IE_TRY(h->d_inc_e.upload(std::vector<double>(1, std::numeric_limits<double>::infinity()), st));
    const uint32_t n_words = (uint32_t)h->d_inc_state.n;
    const uint64_t K = std::max<uint64_t>(h->cfg.total_exchanges, 1);
    const double cold_factor = K > 1 ? std::pow(tmin / tmax, 1.0 / (double)(K - 1)) : 1.0;
    std::vector<double> log_w(R, 0.0), en(E.total_energy), ess_hist, rho_hist;
    std::vector<uint64_t> family(R), fam_hist;
    for (uint32_t i = 0; i < R; i++) family[i] = i;
    double free_energy = 0.0;
    uint64_t resamples = 0;
    bool have_prev = false;
    double beta_prev = 0.0;
    DevBuf<uint64_t> old_spins;
    DevBuf<int32_t> old_ei;
    DevBuf<double> old_ef;
    DevBuf<uint32_t> d_parents;
    for (uint64_t k = 0; k < K; k++) {
        const double t_cold = K > 1 ? tmax * powi_rt(cold_factor, (int)k) : tmin;
        const double span = t_cold / tmax;
        for (uint32_t t = 0; t < L; t++) temps[t] = tmax * std::pow(span, alphas[t]);
        const double beta_cold = 1.0 / t_cold;
        if (have_prev) {
            IE_TRY(E.read_energies(en.data()));
            const double db = beta_cold - beta_prev;
            for (uint32_t p = 0; p < pops; p++)
                for (uint32_t r = 0; r < (uint32_t)kReplicas; r++)
                    log_w[p * kReplicas + r] -= db * en[((size_t)(L - 1) + (size_t)L * p) * kReplicas + r];
            const std::vector<double> w = pa::normalized_weights(log_w.data(), R);
            const double ess = pa::effective_sample_size(w.data(), R);
            ess_hist.push_back(ess);
            if (ess < pc->ess_threshold * (double)R) {
                free_energy += pa::free_energy_increment(log_w.data(), R);
                IE_CUDA(cudaMemcpyAsync(&rng.pos, E.d_pos.p, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
                IE_CUDA(cudaStreamSynchronize(st));
                const double u = rng.unit_f64();
                const std::vector<uint64_t> counts = pa::systematic_resample(w.data(), R, u);
                const std::vector<uint32_t> parents = pa::shuffled_parents(counts, rng);
                IE_CUDA(cudaMemcpyAsync(E.d_pos.p, &rng.pos, sizeof(uint64_t), cudaMemcpyHostToDevice, st));
                IE_TRY(old_spins.alloc(words));
                IE_CUDA(cudaMemcpyAsync(old_spins.p, E.d_spins.p, words * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
                if (mode == kModeInt) {
                    IE_TRY(old_ei.alloc(E.total_energy));
                    IE_CUDA(cudaMemcpyAsync(old_ei.p, E.d_Ei.p, E.total_energy * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
                } else {
                    IE_TRY(old_ef.alloc(E.total_energy));
                    IE_CUDA(cudaMemcpyAsync(old_ef.p, E.d_Ef.p, E.total_energy * sizeof(double), cudaMemcpyDeviceToDevice, st));
                }
                IE_TRY(d_parents.upload(parents, st));
                IE_CUDA(launch_resample(E.arrays(), 0, mode, (uint32_t)words, L, d_parents.p, old_spins.p, old_ei.p,
                                        old_ef.p, g_sm_count, st));
                const std::vector<uint64_t> before = family;
                for (uint32_t d = 0; d < R; d++) family[d] = before[parents[d]];
                double rho = 0.0;
                uint64_t nf = 0;
                pa::family_entropy(family.data(), R, rho, nf);
                rho_hist.push_back(rho);
                fam_hist.push_back(nf);
                resamples++;
                std::fill(log_w.begin(), log_w.end(), 0.0);
                IE_TRY(run_steps(temps, pc->post_resample_relaxation));
            }
        }
        have_prev = true;
        beta_prev = beta_cold;
        IE_TRY(run_steps(temps, h->cfg.sweeps_per_exchange));
        // exact re-sync of every level (again after ICM), then the stage's incumbent
        IE_CUDA(launch_energy(E.arrays(), 0, 1, st));
        if (pc->use_icm) {
            IE_TRY(E.icm_sweep());
            IE_CUDA(launch_energy(E.arrays(), 0, 1, st));
        }
        IE_CUDA(launch_incumbent(E.arrays(), 0, h->offset, h->d_inc_e.p, h->d_inc_state.p, n_words, st));
    }
    IE_CUDA(cudaStreamSynchronize(st));
    h->have_incumbent = true;
    if (rep) {
        rep->free_energy = free_energy;
        rep->resample_events = resamples;
        rep->n_ess = ess_hist.size();
        const uint64_t ne = std::min<uint64_t>(rep->capacity, ess_hist.size());
        const uint64_t nr = std::min<uint64_t>(rep->capacity, rho_hist.size());
        if (rep->ess_history) std::copy(ess_hist.begin(), ess_hist.begin() + ne, rep->ess_history);
        if (rep->family_rho) std::copy(rho_hist.begin(), rho_hist.begin() + nr, rep->family_rho);
        if (rep->family_count) std::copy(fam_hist.begin(), fam_hist.begin() + nr, rep->family_count);
        if (rep->alphas) std::copy(alphas.begin(), alphas.end(), rep->alphas);
    }
    return IE_OK;
}

ie_status ie_read_spins(ie_handle* h, uint64_t* words) {
    if (!h || !words) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(h->eng.device));
    return h->eng.read_words(0, 1, words);
}

ie_status ie_read_energies(ie_handle* h, double* energies) {
    if (!h || !energies) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(h->eng.device));
    return h->eng.read_energies(energies);
}

ie_status ie_read_swap_stats(ie_handle* h, uint64_t* attempts, uint64_t* accepts) {
    if (!h || !attempts || !accepts) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(h->eng.device));
    const uint32_t L = h->eng.pop_len ? h->eng.pop_len : h->eng.nt;
    const uint32_t np = L > 1 ? L - 1 : 0;
    if (np) {
        IE_CUDA(cudaMemcpy(attempts, h->eng.d_att.p, np * sizeof(uint64_t), cudaMemcpyDeviceToHost));
        IE_CUDA(cudaMemcpy(accepts, h->eng.d_acc.p, np * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    }
    return IE_OK;
}

ie_status ie_read_rng_state(ie_handle* h, uint64_t* draws, int32_t* deo) {
    if (!h || !draws || !deo) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(h->eng.device));
    IE_CUDA(cudaMemcpy(draws, h->eng.d_pos.p, sizeof(uint64_t), cudaMemcpyDeviceToHost));
    IE_CUDA(cudaMemcpy(deo, h->eng.d_deo.p, sizeof(int32_t), cudaMemcpyDeviceToHost));
    return IE_OK;
}

// ---- checkpoint ----
namespace {
constexpr uint64_t kStateMagic = 0x3154534232424549ull;  // "IEB2BST1"

struct StateHeader {
    uint64_t magic;
    uint32_t version, mode;
    uint64_t n, cells, npairs, steps_done, draws;
    int32_t deo, have_inc;
    double inc_e;
    uint64_t digest, inc_words;
};

uint64_t fnv1a_bytes(const uint8_t* b, uint64_t n, uint64_t h = 0xcbf29ce484222325ull) {
    for (uint64_t i = 0; i < n; i++) {
        h ^= b[i];
        h *= 0x100000001b3ull;
    }
    return h;
}

// FNV-1a over the reference-layout words of lane-major device words (little-endian bytes)
uint64_t spin_digest(const std::vector<uint64_t>& lane_major) {
    uint64_t h = 0xcbf29ce484222325ull;
    for (uint64_t w : lane_major) {
        const uint64_t r = transpose8x8(w);
        uint8_t b[8];
        for (int i = 0; i < 8; i++) b[i] = (uint8_t)(r >> (8 * i));
        h = fnv1a_bytes(b, 8, h);
    }
    return h;
}

uint64_t state_bytes(const Engine& E, uint64_t inc_words) {
    const InstDesc& d = E.desc[0];
    const uint32_t L = E.nt;
    const uint64_t np = L > 1 ? L - 1 : 0;
    return sizeof(StateHeader) + 8ull * d.nt * d.n + (d.mode == kModeInt ? 4ull : 8ull) * d.nt * kReplicas +
           16ull * np + 8ull * inc_words;
}
}  // namespace

ie_status ie_state_size(ie_handle* h, uint64_t* bytes) {
    if (!h || !bytes) return fail(IE_ERR_INVALID, "NULL argument");
    if (h->eng.pop_len) return fail(IE_ERR_UNSUPPORTED, "checkpoints cover handles with num_pops = 1");
    *bytes = state_bytes(h->eng, h->d_inc_state.n);
    return IE_OK;
}

ie_status ie_state_digest(ie_handle* h, uint64_t* digest) {
    if (!h || !digest) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(h->eng.device));
    const InstDesc& d = h->eng.desc[0];
    std::vector<uint64_t> w((size_t)d.nt * d.n);
    if (!w.empty())
        IE_CUDA(cudaMemcpy(w.data(), h->eng.d_spins.p + d.spin, w.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    *digest = spin_digest(w);
    return IE_OK;
}

ie_status ie_fnv1a(const void* bytes, uint64_t n, uint64_t* digest) {
    if ((!bytes && n) || !digest) return fail(IE_ERR_INVALID, "NULL argument");
    *digest = fnv1a_bytes(static_cast<const uint8_t*>(bytes), n);
    return IE_OK;
}

ie_status ie_save_state(ie_handle* h, void* blob, uint64_t bytes) {
    if (!h || !blob) return fail(IE_ERR_INVALID, "NULL argument");
    Engine& E = h->eng;
    if (E.pop_len) return fail(IE_ERR_UNSUPPORTED, "checkpoints cover handles with num_pops = 1");
    if (!E.initialized) return fail(IE_ERR_INVALID, "the handle's state is not initialised");
    const uint64_t iw = h->d_inc_state.n;
    if (bytes < state_bytes(E, iw)) return fail(IE_ERR_INVALID, "blob smaller than ie_state_size");
    IE_CUDA(cudaSetDevice(E.device));
    IE_CUDA(cudaStreamSynchronize(E.stream));
    const InstDesc& d = E.desc[0];
    const uint64_t nw = (uint64_t)d.nt * d.n, ne = (uint64_t)d.nt * kReplicas, np = E.nt > 1 ? E.nt - 1 : 0;
    uint8_t* p = static_cast<uint8_t*>(blob);
    StateHeader hd{};
    hd.magic = kStateMagic;
    hd.version = 1;
    hd.mode = d.mode;
    hd.n = d.n;
    hd.cells = d.nt;
    hd.npairs = np;
    hd.steps_done = E.steps_done;
    hd.have_inc = h->have_incumbent ? 1 : 0;
    hd.inc_words = iw;
    IE_CUDA(cudaMemcpy(&hd.draws, E.d_pos.p, sizeof(uint64_t), cudaMemcpyDeviceToHost));
    IE_CUDA(cudaMemcpy(&hd.deo, E.d_deo.p, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (h->d_inc_e.p) IE_CUDA(cudaMemcpy(&hd.inc_e, h->d_inc_e.p, sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<uint64_t> w(nw);
    if (nw) IE_CUDA(cudaMemcpy(w.data(), E.d_spins.p + d.spin, nw * 8, cudaMemcpyDeviceToHost));
    hd.digest = spin_digest(w);
    std::memcpy(p, &hd, sizeof(hd));
    p += sizeof(hd);
    std::memcpy(p, w.data(), nw * 8);
    p += nw * 8;
    if (d.mode == kModeInt) {
        IE_CUDA(cudaMemcpy(p, E.d_Ei.p + d.energy, ne * 4, cudaMemcpyDeviceToHost));
        p += ne * 4;
    } else {
        IE_CUDA(cudaMemcpy(p, E.d_Ef.p + d.energy, ne * 8, cudaMemcpyDeviceToHost));
        p += ne * 8;
    }
    if (np) {
        IE_CUDA(cudaMemcpy(p, E.d_att.p, np * 8, cudaMemcpyDeviceToHost));
        IE_CUDA(cudaMemcpy(p + np * 8, E.d_acc.p, np * 8, cudaMemcpyDeviceToHost));
        p += 16 * np;
    }
    if (iw) IE_CUDA(cudaMemcpy(p, h->d_inc_state.p, iw * 8, cudaMemcpyDeviceToHost));
    return IE_OK;
}

ie_status ie_load_state(ie_handle* h, const void* blob, uint64_t bytes) {
    if (!h || !blob) return fail(IE_ERR_INVALID, "NULL argument");
    Engine& E = h->eng;
    if (E.pop_len) return fail(IE_ERR_UNSUPPORTED, "checkpoints cover handles with num_pops = 1");
    if (bytes < sizeof(StateHeader)) return fail(IE_ERR_INVALID, "blob too small");
    StateHeader hd;
    std::memcpy(&hd, blob, sizeof(hd));
    const InstDesc& d = E.desc[0];
    const uint64_t nw = (uint64_t)d.nt * d.n, ne = (uint64_t)d.nt * kReplicas, np = E.nt > 1 ? E.nt - 1 : 0;
    if (hd.magic != kStateMagic || hd.version != 1) return fail(IE_ERR_INVALID, "not a state blob of this version");
    if (hd.n != d.n || hd.cells != d.nt || hd.mode != d.mode || hd.npairs != np || hd.inc_words != h->d_inc_state.n)
        return fail(IE_ERR_INVALID, "state blob of another problem or config (sites, cells, mode)");
    if (bytes < state_bytes(E, hd.inc_words)) return fail(IE_ERR_INVALID, "blob truncated");
    const uint8_t* p = static_cast<const uint8_t*>(blob) + sizeof(hd);
    std::vector<uint64_t> w(nw);
    std::memcpy(w.data(), p, nw * 8);
    p += nw * 8;
    if (spin_digest(w) != hd.digest) return fail(IE_ERR_INVALID, "state blob digest mismatch");
    IE_CUDA(cudaSetDevice(E.device));
    IE_CUDA(cudaStreamSynchronize(E.stream));
    if (nw) IE_CUDA(cudaMemcpy(E.d_spins.p + d.spin, w.data(), nw * 8, cudaMemcpyHostToDevice));
    if (d.mode == kModeInt) {
        IE_CUDA(cudaMemcpy(E.d_Ei.p + d.energy, p, ne * 4, cudaMemcpyHostToDevice));
        p += ne * 4;
    } else {
        IE_CUDA(cudaMemcpy(E.d_Ef.p + d.energy, p, ne * 8, cudaMemcpyHostToDevice));
        p += ne * 8;
    }
    if (np) {
        IE_CUDA(cudaMemcpy(E.d_att.p, p, np * 8, cudaMemcpyHostToDevice));
        IE_CUDA(cudaMemcpy(E.d_acc.p, p + np * 8, np * 8, cudaMemcpyHostToDevice));
        p += 16 * np;
    }
    if (hd.inc_words) IE_CUDA(cudaMemcpy(h->d_inc_state.p, p, hd.inc_words * 8, cudaMemcpyHostToDevice));
    if (h->d_inc_e.p) IE_CUDA(cudaMemcpy(h->d_inc_e.p, &hd.inc_e, sizeof(double), cudaMemcpyHostToDevice));
    IE_CUDA(cudaMemcpy(E.d_pos.p, &hd.draws, sizeof(uint64_t), cudaMemcpyHostToDevice));
    IE_CUDA(cudaMemcpy(E.d_deo.p, &hd.deo, sizeof(int32_t), cudaMemcpyHostToDevice));
    E.steps_done = hd.steps_done;
    E.initialized = true;
    h->have_incumbent = hd.have_inc != 0;
    return IE_OK;
}

ie_status ie_read_incumbent(ie_handle* h, double* energy, int8_t* state) {
    if (!h || !energy || !state) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(h->eng.device));
    const uint64_t n = h->eng.desc[0].n;
    std::vector<uint64_t> w(h->d_inc_state.n);
    IE_CUDA(cudaMemcpy(energy, h->d_inc_e.p, sizeof(double), cudaMemcpyDeviceToHost));
    IE_CUDA(cudaMemcpy(w.data(), h->d_inc_state.p, w.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    for (uint64_t i = 0; i < n; i++) state[i] = (int8_t)((w[i / 64] >> (i % 64)) & 1);
    return IE_OK;
}

ie_status ie_read_best(ie_handle* h, double* energy, int8_t* state) {
    if (!h || !energy || !state) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(h->eng.device));
    Engine& E = h->eng;
    const uint32_t nt = E.nt;
    const uint64_t n = E.desc[0].n;
    // model energies of every (cell, replica), argmin and the replica's
    // configuration on the device (ultimate.rs:345-368)
    DevBuf<double> es, be;
    DevBuf<int8_t> st;
    DevBuf<int32_t> fd;
    IE_TRY(es.alloc((size_t)nt * kReplicas));
    IE_TRY(be.alloc(1));
    IE_TRY(st.alloc(std::max<uint64_t>(n, 1)));
    IE_TRY(fd.alloc(1));
    IE_CUDA(launch_model_energy(E.arrays(), 0, nt, h->offset, es.p, E.stream));
    IE_CUDA(launch_best_extract(E.arrays(), 0, es.p, nt * kReplicas, st.p, be.p, fd.p, E.stream));
    double best = 0;
    IE_CUDA(cudaMemcpyAsync(&best, be.p, sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    if (n) IE_CUDA(cudaMemcpyAsync(state, st.p, n, cudaMemcpyDeviceToHost, E.stream));
    IE_CUDA(cudaStreamSynchronize(E.stream));
    *energy = best;
    if (h->have_incumbent) {
        double ie_ = 0;
        std::vector<int8_t> inc(n);
        IE_TRY(ie_read_incumbent(h, &ie_, inc.data()));
        if (ie_ < best) {
            *energy = ie_;
            std::copy(inc.begin(), inc.end(), state);
        }
    }
    return IE_OK;
}

ie_status ie_one_opt(ie_handle* h, int8_t* state, const uint8_t* is_clamped, double* improvement) {
    if (!h || !state) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(h->eng.device));
    Engine& E = h->eng;
    const uint64_t n = E.desc[0].n;
    if (n == 0) {
        if (improvement) *improvement = 0.0;
        return IE_OK;
    }
    for (uint64_t v = 0; v < n; v++)
        if (state[v] != 0 && state[v] != 1) return fail(IE_ERR_INVALID, "state must be 0/1");
    DevBuf<int8_t> st;
    DevBuf<uint8_t> cl;
    DevBuf<double> g, imp;
    DevBuf<uint64_t> fl;
    IE_TRY(st.alloc(n));
    IE_TRY(g.alloc(n));
    IE_TRY(imp.alloc(1));
    IE_TRY(fl.alloc(1));
    IE_CUDA(cudaMemcpyAsync(st.p, state, n, cudaMemcpyHostToDevice, E.stream));
    if (is_clamped) {
        IE_TRY(cl.alloc(n));
        IE_CUDA(cudaMemcpyAsync(cl.p, is_clamped, n, cudaMemcpyHostToDevice, E.stream));
    }
    // every flip lowers the energy by more than 1e-12, so the descent ends;
    // the bound only guards against non-finite input
    IE_CUDA(launch_one_opt(E.arrays(), 0, st.p, is_clamped ? cl.p : nullptr, g.p, imp.p, fl.p, 64 * n + 1024,
                           E.stream));
    double total = 0;
    IE_CUDA(cudaMemcpyAsync(state, st.p, n, cudaMemcpyDeviceToHost, E.stream));
    IE_CUDA(cudaMemcpyAsync(&total, imp.p, sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    IE_CUDA(cudaStreamSynchronize(E.stream));
    if (improvement) *improvement = total;
    return IE_OK;
}

// ---- batch ----

ie_status ie_batch_create(const ie_problem* problems, uint32_t count, const uint64_t* seeds,
                          const ie_batch_config* config, ie_batch** out) {
    if (!out || !problems || !seeds) return fail(IE_ERR_INVALID, "NULL argument");
    *out = nullptr;
    if (count == 0) return fail(IE_ERR_INVALID, "count must be >= 1");
    std::unique_ptr<ie_batch> b(new ie_batch());
    ie_batch_config cfg{};
    if (config) cfg = *config;
    IE_TRY(b->eng.setup_device(cfg.device));
    b->eng.threads_per_block = cfg.threads_per_block;
    b->eng.blocks_per_sm = cfg.blocks_per_sm;
    b->eng.use_windows = cfg.disable_windows == 0;
    b->eng.use_graph = cfg.use_graph != 0;
    b->eng.is_batch = true;
    if (cfg.kernel_form < 0 || cfg.kernel_form > 1) return fail(IE_ERR_INVALID, "kernel_form must be 0 or 1");
    b->eng.kernel_form = cfg.kernel_form;
    if (cfg.item_sites) {
        if (cfg.item_sites < 64 || cfg.item_sites > 16384)
            return fail(IE_ERR_INVALID, "item_sites must be in [64, 16384]");
        b->eng.lvl_cap = cfg.item_sites;
    }
    if (cfg.tie_shift > 31) return fail(IE_ERR_INVALID, "tie_shift must be below 32");
    b->eng.lvl_tie_shift = cfg.tie_shift;
    if (cfg.bit_sliced < -1 || cfg.bit_sliced > 1) return fail(IE_ERR_INVALID, "bit_sliced must be -1, 0 or 1");
    b->eng.pmj_policy = cfg.bit_sliced;
    b->eng.bulk_ring = cfg.bulk_ring != 0;
    if (cfg.threads_per_block && (cfg.threads_per_block % 32 || cfg.threads_per_block > 256))
        return fail(IE_ERR_INVALID, "threads_per_block must be a multiple of 32, at most 256");
    if (cfg.threads_per_block) b->eng.lvl_threads = (int)cfg.threads_per_block;
    IE_TRY(b->eng.build(problems, count, 1, seeds, cfg.force_f64 != 0));
    *out = b.release();
    return IE_OK;
}

ie_status ie_batch_destroy(ie_batch* b) {
    delete b;
    return IE_OK;
}

ie_status ie_batch_init_random(ie_batch* b) {
    if (!b) return fail(IE_ERR_INVALID, "batch is NULL");
    IE_CUDA(cudaSetDevice(b->eng.device));
    return b->eng.init_random();
}

ie_status ie_batch_run_schedule(ie_batch* b, const double* temps, uint64_t n_steps) {
    if (!b || !temps) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(b->eng.device));
    IE_TRY(b->eng.run_batch(temps, n_steps));
    return b->eng.check_err();
}

ie_status ie_batch_run_schedule_plain(ie_batch* b, const double* temps, uint64_t n_steps, uint32_t first,
                                      uint32_t count) {
    if (!b || !temps) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(b->eng.device));
    return b->eng.run_plain(temps, n_steps, first, count);
}

ie_status ie_batch_read_spins(ie_batch* b, uint64_t* words) {
    if (!b || !words) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(b->eng.device));
    return b->eng.read_words(0, b->eng.count, words);
}

ie_status ie_batch_read_energies(ie_batch* b, double* energies) {
    if (!b || !energies) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(b->eng.device));
    return b->eng.read_energies(energies);
}

ie_status ie_batch_read_draws(ie_batch* b, uint64_t* draws) {
    if (!b || !draws) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(b->eng.device));
    IE_CUDA(cudaMemcpy(draws, b->eng.d_pos.p, b->eng.count * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    return IE_OK;
}

ie_status ie_batch_recompute_energies(ie_batch* b, double* energies) {
    if (!b || !energies) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(b->eng.device));
    return b->eng.recompute_energies(energies);
}

ie_status ie_batch_autotune(ie_batch* b, const double* temps, uint64_t trial_steps, uint32_t* chosen) {
    if (!b || !temps) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(b->eng.device));
    return b->eng.autotune(temps, trial_steps, chosen);
}

ie_status ie_batch_last_run_ms(ie_batch* b, double* ms) {
    if (!b || !ms) return fail(IE_ERR_INVALID, "NULL argument");
    *ms = b->eng.last_ms;
    return IE_OK;
}

ie_status ie_batch_class_report(ie_batch* b, uint32_t max_classes, uint32_t* n_classes, uint32_t* info,
                                double* ms) {
    if (!b || !n_classes) return fail(IE_ERR_INVALID, "NULL argument");
    Engine& E = b->eng;
    *n_classes = (uint32_t)E.classes.size();
    for (uint32_t k = 0; k < std::min<uint32_t>(max_classes, *n_classes); k++) {
        if (info) {
            info[5 * k + 0] = E.classes[k]->mode;
            info[5 * k + 1] = (uint32_t)E.classes[k]->tpl;
            info[5 * k + 2] = E.classes[k]->cap;
            info[5 * k + 3] = E.classes[k]->nitems;
            info[5 * k + 4] = k < E.class_ms.size() ? 1u : 0u;
        }
        if (ms) ms[k] = k < E.class_ms.size() ? E.class_ms[k] : 0.0;
    }
    return IE_OK;
}

ie_status ie_batch_exact_decisions(ie_batch* b, uint64_t* count) {
    if (!b || !count) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(b->eng.device));
    int32_t c = 0;
    if (b->eng.d_exact.p) IE_CUDA(cudaMemcpy(&c, b->eng.d_exact.p, sizeof(c), cudaMemcpyDeviceToHost));
    *count = (uint64_t)(uint32_t)c;
    return IE_OK;
}

ie_status ie_batch_last_launches(ie_batch* b, uint64_t* launches) {
    if (!b || !launches) return fail(IE_ERR_INVALID, "NULL argument");
    *launches = b->eng.last_launches;
    return IE_OK;
}

// ---- serving ----

ie_status ie_serve_create(const ie_serve_config* config, ie_serve** out) {
    if (!out) return fail(IE_ERR_INVALID, "NULL argument");
    *out = nullptr;
    std::unique_ptr<ie_serve> s(new ie_serve());
    IE_TRY(s->s.create(config));
    *out = s.release();
    return IE_OK;
}

ie_status ie_serve_destroy(ie_serve* s) {
    delete s;
    return IE_OK;
}

ie_status ie_serve_submit(ie_serve* s, const ie_problem* problem, uint64_t seed, const double* temps,
                          uint64_t n_steps, const uint8_t* is_clamped, const int8_t* clamp_val, uint64_t* id) {
    if (!s || !id) return fail(IE_ERR_INVALID, "NULL argument");
    std::unique_ptr<ServeReq> r(new ServeReq());
    IE_TRY(s->s.prepare(problem, seed, temps, n_steps, is_clamped, clamp_val, *r));
    std::lock_guard<std::mutex> lk(s->s.mu);
    r->id = s->s.next_id++;
    *id = r->id;
    s->s.pending.push_back(std::move(r));
    return IE_OK;
}

ie_status ie_serve_tick(ie_serve* s, uint32_t* n_active, uint32_t* n_pending, uint32_t* n_finished) {
    if (!s) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(s->s.eng.device));
    return s->s.tick(n_active, n_pending, n_finished);
}

ie_status ie_serve_poll(ie_serve* s, uint64_t* ids, uint32_t max_ids, uint32_t* n_ids) {
    if (!s || !n_ids || (max_ids && !ids)) return fail(IE_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(s->s.mu);
    uint32_t k = 0;
    for (auto it = s->s.finished.begin(); it != s->s.finished.end() && k < max_ids; ++it) ids[k++] = it->first;
    *n_ids = k;
    return IE_OK;
}

ie_status ie_serve_result(ie_serve* s, uint64_t id, uint64_t* words, double* energies) {
    if (!s || !words || !energies) return fail(IE_ERR_INVALID, "NULL argument");
    std::unique_ptr<ServeReq> r;
    {
        std::lock_guard<std::mutex> lk(s->s.mu);
        auto it = s->s.finished.find(id);
        if (it == s->s.finished.end()) return fail(IE_ERR_INVALID, "no finished request with this id");
        r = std::move(it->second);
        s->s.finished.erase(it);
    }
    std::copy(r->words.begin(), r->words.end(), words);
    std::copy(r->energies.begin(), r->energies.end(), energies);
    return IE_OK;
}

ie_status ie_serve_footprint(ie_serve* s, const ie_problem* problem, uint64_t n_steps, uint64_t* bytes) {
    if (!s || !bytes || !problem) return fail(IE_ERR_INVALID, "NULL argument");
    ServeReq r;
    std::vector<double> t(std::max<uint64_t>(n_steps, 1), 1.0);
    IE_TRY(s->s.prepare(problem, 0, t.data(), n_steps, nullptr, nullptr, r));
    *bytes = ServeEngine::bytes_of(r);
    return IE_OK;
}

ie_status ie_serve_last_tick(ie_serve* s, double* ms, uint64_t* launches) {
    if (!s || !ms || !launches) return fail(IE_ERR_INVALID, "NULL argument");
    *ms = s->s.eng.last_ms;
    *launches = s->s.eng.last_launches;
    return IE_OK;
}

ie_status ie_probe_peaks(int32_t device, double* int_ops_per_s, double* xoshiro_per_s) {
    if (!int_ops_per_s || !xoshiro_per_s) return fail(IE_ERR_INVALID, "NULL argument");
    IE_CUDA(cudaSetDevice(device));
    int sms = 0;
    IE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    IE_CUDA(probe_peaks(sms, int_ops_per_s, xoshiro_per_s));
    return IE_OK;
}

}  // extern "C"
