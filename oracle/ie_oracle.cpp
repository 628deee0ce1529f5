// CPU oracle: a plain C++ restatement of the reference's S1 Metropolis/PT path.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product (the ising_engine_b200 package
// and its CUDA library) links, imports or calls this file. It is used by tests/,
// by __graft_entry__.smoke() as the checker, and by bench.py's cpu_baseline /
// --impl reference leg as the timed CPU restatement of the reference's Rayon path.
//
// Parity pin: the end-to-end golden of tests/test_regression_golden.rs:87-111
// (UltimateSolver::new(50,0.05,30,40,Some(2024)) on the seeded n=32 instance)
// is reproduced by or_solve(); tests/test_oracle_golden.py asserts it.
//
// Every function cites the reference file:line it restates. Compile with
// -ffp-contract=off and no fast-math: the reference's f64 arithmetic is
// uncontracted (Rust never fuses a*b+c on its own).
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <functional>
#include <limits>
#include <map>
#include <thread>
#include <vector>

namespace {

constexpr int NR = 64;  // NUM_REPLICAS, src/solver/types.rs:17

// ---------------------------------------------------------------------------
// Master RNG: rand_chacha 0.3.1 ChaCha8Rng, seeded by rand_core 0.6.4
// SeedableRng::seed_from_u64, drawn through rand 0.8.5 (gen::<u64>, gen::<f64>,
// gen_range::<f64>). Third-party crates (Cargo.lock:2656-2705), restated from
// their published algorithms; call sites ultimate.rs:151-152,272 and
// engine.rs:596,727.
// ---------------------------------------------------------------------------
static inline uint32_t rotl32(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }

// One ChaCha block with 8 rounds (4 double rounds). Input layout: constants,
// 8 key words, 64-bit block counter (words 12-13), 64-bit stream id (14-15).
static void chacha8_block(const uint32_t key[8], uint64_t counter, uint32_t out[16]) {
    uint32_t in[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                       key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                       (uint32_t)counter, (uint32_t)(counter >> 32), 0u, 0u};
    uint32_t x[16];
    std::memcpy(x, in, sizeof(x));
#define QR(a, b, c, d)                      \
    x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl32(x[d], 16); \
    x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl32(x[b], 12); \
    x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl32(x[d], 8);  \
    x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl32(x[b], 7);
    for (int i = 0; i < 4; i++) {
        QR(0, 4, 8, 12) QR(1, 5, 9, 13) QR(2, 6, 10, 14) QR(3, 7, 11, 15)
        QR(0, 5, 10, 15) QR(1, 6, 11, 12) QR(2, 7, 8, 13) QR(3, 4, 9, 14)
    }
#undef QR
    for (int i = 0; i < 16; i++) out[i] = x[i] + in[i];
}

struct ChaCha8Rng {
    uint32_t key[8];
    uint64_t counter = 0;  // next block to generate
    uint32_t buf[64];      // rand_chacha buffers 4 blocks
    int idx = 64;
    uint64_t draws = 0;    // number of u64 draws so far (stream position)

    // rand_core 0.6.4 seed_from_u64: PCG32 output fills the 32-byte seed.
    explicit ChaCha8Rng(uint64_t state) {
        const uint64_t MUL = 6364136223846793005ULL, INC = 11634580027462260723ULL;
        for (int i = 0; i < 8; i++) {
            state = state * MUL + INC;
            uint32_t xs = (uint32_t)(((state >> 18) ^ state) >> 27);
            uint32_t rot = (uint32_t)(state >> 59);
            key[i] = (xs >> rot) | (xs << ((32 - rot) & 31));  // little-endian bytes = word
        }
    }
    void refill() {
        for (int b = 0; b < 4; b++) chacha8_block(key, counter + b, buf + 16 * b);
        counter += 4;
        idx = 0;
    }
    // BlockRng::next_u64: two consecutive u32 words, low first. Every draw on
    // this path is 64-bit, so the index is always even.
    uint64_t next_u64() {
        if (idx >= 64) refill();
        uint64_t v = (uint64_t)buf[idx] | ((uint64_t)buf[idx + 1] << 32);
        idx += 2;
        draws++;
        return v;
    }
    // rand 0.8.5 Standard for f64: 53 high bits times 2^-53.
    double gen_f64() { return (double)(next_u64() >> 11) * (1.0 / 9007199254740992.0); }
    // rand 0.8.5 UniformFloat::<f64>::sample_single (gen_range(low..high)).
    double gen_range(double low, double high) {
        double scale = high - low;
        for (;;) {
            uint64_t bits = (next_u64() >> 12) | 0x3FF0000000000000ULL;
            double v12;
            std::memcpy(&v12, &bits, 8);
            double v01 = v12 - 1.0;
            double res = v01 * scale + low;
            if (res < high) return res;
            uint64_t sb;
            std::memcpy(&sb, &scale, 8);
            sb -= 1;
            std::memcpy(&scale, &sb, 8);
        }
    }
};

// ---------------------------------------------------------------------------
// Xoshiro256PlusPlusX8, src/solver/engine.rs:81-172.
// ---------------------------------------------------------------------------
static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

struct XoshiroX8 {
    uint64_t s[4][8];
    // engine.rs:87-103: SplitMix64 sequence, lane-major fill.
    explicit XoshiroX8(uint64_t seed) {
        uint64_t state = seed;
        auto next = [&]() {
            state += 0x9e3779b97f4a7c15ULL;
            uint64_t z = state;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
            return z ^ (z >> 31);
        };
        for (int lane = 0; lane < 8; lane++)
            for (int w = 0; w < 4; w++) s[w][lane] = next();
    }
    inline void advance() {
        for (int l = 0; l < 8; l++) {
            uint64_t t = s[1][l] << 17;
            s[2][l] ^= s[0][l];
            s[3][l] ^= s[1][l];
            s[1][l] ^= s[2][l];
            s[0][l] ^= s[3][l];
            s[2][l] ^= t;
            s[3][l] = rotl64(s[3][l], 45);
        }
    }
    // engine.rs:107-125: uniform = (result >> 12) * 2^-52 via the mantissa trick.
    inline void next_f64x8(double* out) {
        for (int l = 0; l < 8; l++) {
            uint64_t result = rotl64(s[0][l] + s[3][l], 23) + s[0][l];
            uint64_t bits = 0x3FF0000000000000ULL | (result >> 12);
            double d;
            std::memcpy(&d, &bits, 8);
            out[l] = d - 1.0;
        }
        advance();
    }
    // engine.rs:145-151: 64 uniforms, replica r = 8*call + lane.
    inline void next_f64x64(double* out) {
        for (int c = 0; c < 8; c++) next_f64x8(out + 8 * c);
    }
    // engine.rs:159-171
    inline void skip_f64x64() {
        for (int c = 0; c < 8; c++) advance();
    }
};

// engine.rs:181-205 (f64::clamp semantics, left-to-right sums, no contraction).
static inline double fast_exp(double x) {
    if (x < -20.0) x = -20.0;
    if (x > 0.0) x = 0.0;
    double r = x * 0.0625;
    double r2 = r * r;
    double r3 = r2 * r;
    double p = 1.0 + r + 0.5 * r2 + (1.0 / 6.0) * r3 + (1.0 / 24.0) * r2 * r2 +
               (1.0 / 120.0) * r2 * r3 + (1.0 / 720.0) * r3 * r3;
    double p2 = p * p;
    double p4 = p2 * p2;
    double p8 = p4 * p4;
    return p8 * p8;
}

// compiler-rt __powidf2, which Rust's f64::powi lowers to for a runtime exponent.
static double powi(double a, int b) {
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

// ---------------------------------------------------------------------------
// Problem: QuboModel + CsrMatrix (src/core/hubo.rs:165-189, csr_matrix.rs:6-30).
// Both triangles stored; E = offset + sum lin*x + 1/2 sum_csr w x_i x_j.
// FlatHuboModel::from_hubo (hubo.rs:94-158) keeps the rows in the same order, so
// the edge2 CSR equals the quadratic CSR (ultimate.rs:140-148).
// ---------------------------------------------------------------------------
struct Qubo {
    int64_t n = 0;
    std::vector<double> linear;
    std::vector<int64_t> row;
    std::vector<int64_t> col;
    std::vector<double> val;
    double offset = 0.0;
};

static Qubo make_qubo(int64_t n, const double* lin, const int64_t* row, const int64_t* col,
                      const double* val, double offset) {
    Qubo q;
    q.n = n;
    q.linear.assign(lin, lin + n);
    q.row.assign(row, row + n + 1);
    int64_t nnz = q.row[n];
    q.col.assign(col, col + nnz);
    q.val.assign(val, val + nnz);
    q.offset = offset;
    return q;
}

// hubo.rs:176-189
static double total_energy(const Qubo& m, const int8_t* state) {
    double e = m.offset;
    for (int64_t i = 0; i < m.n; i++) {
        if (state[i] == 1) {
            e += m.linear[i];
            for (int64_t k = m.row[i]; k < m.row[i + 1]; k++)
                if (state[m.col[k]] == 1) e += m.val[k] * 0.5;
        }
    }
    return e;
}

// ---------------------------------------------------------------------------
// QuantumField with num_slices = 1 (src/solver/types.rs:17-58). Spins are one
// byte per replica: spins[(v + n*cell)*64 + r], cell = t + nt*p.
// ---------------------------------------------------------------------------
struct Field {
    int64_t n;
    int nt, np;
    std::vector<int8_t> spins;
    std::vector<std::array<double, NR>> energies;
    Field(int64_t n_, int nt_, int np_) : n(n_), nt(nt_), np(np_),
        spins((size_t)n_ * nt_ * np_ * NR, 0), energies((size_t)nt_ * np_) {
        for (auto& e : energies) e.fill(0.0);
    }
    int8_t* cell(int c) { return spins.data() + (size_t)c * n * NR; }
};

// engine.rs:218-271 (edge2 only: QUBO input has no edge3/edge4 terms).
static inline void delta_e_local(const Qubo& m, const int8_t* spins, int64_t v, double* delta) {
    const int8_t* xv = spins + v * NR;
    int8_t sign[NR];
    for (int r = 0; r < NR; r++) sign[r] = (int8_t)(1 - 2 * xv[r]);
    const double wl = m.linear[v];
    for (int r = 0; r < NR; r++) delta[r] = wl * (double)sign[r];
    for (int64_t k = m.row[v]; k < m.row[v + 1]; k++) {
        const int8_t* xj = spins + m.col[k] * NR;
        const double w = m.val[k];
        for (int r = 0; r < NR; r++) {
            int8_t t = (int8_t)((xj[r] ^ xv[r]) - xv[r]);
            delta[r] += w * (double)t;
        }
    }
}

// engine.rs:333-368 (num_slices = 1: the Trotter term is j_tau = 0 and adds 0).
static void replica_energies(const Qubo& m, const int8_t* spins, double* en) {
    for (int r = 0; r < NR; r++) en[r] = 0.0;
    for (int64_t v = 0; v < m.n; v++) {
        const int8_t* xv = spins + v * NR;
        const double wl = m.linear[v];
        for (int r = 0; r < NR; r++) en[r] += wl * (double)xv[r];
        for (int64_t k = m.row[v]; k < m.row[v + 1]; k++) {
            int64_t j = m.col[k];
            if (v < j) {
                const double w = m.val[k];
                const int8_t* xj = spins + j * NR;
                for (int r = 0; r < NR; r++) en[r] += w * (double)(xv[r] & xj[r]);
            }
        }
    }
}

struct StepScratch {
    std::vector<uint64_t> attempts, accepts;
    bool deo_odd = false;
    // round-trip tracking (engine.rs:454-536, opt-in): direction label per
    // (cell, replica) (+1 up, -1 down, 0 none), up/down histograms per
    // temperature, completed round trips
    bool track = false;
    std::vector<std::array<int8_t, NR>> labels;
    std::vector<uint64_t> n_up, n_down;
    uint64_t rt = 0;
};

// A tiny fork/join pool standing in for Rayon's par_chunks_mut (engine.rs:603-608).
static void parallel_for(int count, int threads, const std::function<void(int)>& fn) {
    if (threads <= 1 || count <= 1) {
        for (int i = 0; i < count; i++) fn(i);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    int nthr = std::min(threads, count);
    for (int t = 0; t < nthr; t++)
        pool.emplace_back([&]() {
            for (int i; (i = next.fetch_add(1)) < count;) fn(i);
        });
    for (auto& th : pool) th.join();
}

// Phase 1 of engine.rs:573-703 for one cell: index-order Metropolis sweep.
static void sweep_cell(const Qubo& m, int8_t* spins, double* es, double beta, uint64_t seed,
                       const std::vector<uint8_t>& clamped) {
    XoshiroX8 rng(seed);
    double u[NR], d[NR];
    for (int64_t v = 0; v < m.n; v++) {
        if (clamped[v]) {
            rng.skip_f64x64();
            continue;
        }
        rng.next_f64x64(u);
        delta_e_local(m, spins, v, d);
        int8_t* xv = spins + v * NR;
        for (int r = 0; r < NR; r++) {
            double td = d[r];
            double ev = fast_exp(-td * beta);
            bool accept = (td <= 0.0) | (u[r] < ev);
            int8_t flip = (int8_t)accept;
            xv[r] ^= flip;
            es[r] += td * (double)flip;
        }
    }
}

// Phase 2 of engine.rs:713-789: DEO replica exchange on the master RNG.
static void exchange(Field& f, const double* temps, StepScratch& sc, ChaCha8Rng& rng,
                     bool stats) {
    const int nt = f.nt;
    const int parity = sc.deo_odd ? 1 : 0;
    for (int p = 0; p < f.np; p++) {
        for (int t = parity; t + 1 < nt; t += 2) {
            auto& e1 = f.energies[t + nt * p];
            auto& e2 = f.energies[t + 1 + nt * p];
            double b1 = 1.0 / temps[t], b2 = 1.0 / temps[t + 1];
            double db = b1 - b2;
            bool mask[NR];
            bool any = false;
            int acc = 0;
            for (int r = 0; r < NR; r++) {
                double de = e1[r] - e2[r];
                double ex = db * de;
                mask[r] = ex >= 0.0 || rng.gen_f64() < std::exp(ex);
                any |= mask[r];
                acc += mask[r];
            }
            if (stats) {
                sc.attempts[t] += NR;
                sc.accepts[t] += (uint64_t)acc;
            }
            if (any) {
                int8_t* c1 = f.cell(t + nt * p);
                int8_t* c2 = f.cell(t + 1 + nt * p);
                int8_t lm[NR];
                for (int r = 0; r < NR; r++) lm[r] = (int8_t)(-(int8_t)mask[r]);
                for (int64_t v = 0; v < f.n; v++)
                    for (int r = 0; r < NR; r++) {
                        int8_t dd = (int8_t)((c1[v * NR + r] ^ c2[v * NR + r]) & lm[r]);
                        c1[v * NR + r] ^= dd;
                        c2[v * NR + r] ^= dd;
                    }
                for (int r = 0; r < NR; r++)
                    if (mask[r]) {
                        std::swap(e1[r], e2[r]);
                        if (sc.track) std::swap(sc.labels[t + nt * p][r], sc.labels[t + 1 + nt * p][r]);
                    }
            }
        }
    }
}

// engine::step (engine.rs:573-819) with an optional exchange skip: the
// exchange-interval extension runs phase 2 only when do_exchange is set, and
// the DEO phase toggles per executed exchange (interval 1 is the reference).
static void step(Field& f, const Qubo& m, const double* temps, const std::vector<uint8_t>& clamped,
                 StepScratch& sc, ChaCha8Rng& rng, bool do_exchange, bool stats, int threads,
                 uint64_t* base_seed_out) {
    const uint64_t base_seed = rng.next_u64();
    if (base_seed_out) *base_seed_out = base_seed;
    const int cells = f.nt * f.np;
    parallel_for(cells, threads, [&](int c) {
        int t = c % f.nt;
        double beta = 1.0 / temps[t];
        sweep_cell(m, f.cell(c), f.energies[c].data(), beta, base_seed + (uint64_t)c, clamped);
    });
    if (do_exchange) {
        exchange(f, temps, sc, rng, stats);
        // engine.rs:794-816: relabel the ends, count round trips, histogram
        if (sc.track && f.nt >= 2)
            for (int p = 0; p < f.np; p++) {
                const int hot = f.nt * p, cold = f.nt - 1 + f.nt * p;
                for (int r = 0; r < NR; r++) {
                    if (sc.labels[hot][r] == 1) sc.rt++;
                    sc.labels[hot][r] = -1;
                    sc.labels[cold][r] = 1;
                }
                for (int t = 0; t < f.nt; t++)
                    for (int r = 0; r < NR; r++) {
                        if (sc.labels[t + f.nt * p][r] == 1) sc.n_up[t]++;
                        else if (sc.labels[t + f.nt * p][r] == -1) sc.n_down[t]++;
                    }
            }
        sc.deo_odd = !sc.deo_odd;
    }
}

// ultimate.rs:248-280: clamped sites take their value; with warm-start
// probabilities (with_gnn_heuristic) each replica is one when its
// gen_range(0.0..1.0) draw is below probs[v]; otherwise one gen::<u64>()
// word per site.
static void init_field(Field& f, const std::vector<uint8_t>& clamped,
                       const std::vector<int8_t>& cval, ChaCha8Rng& rng, const double* probs = nullptr) {
    for (int p = 0; p < f.np; p++)
        for (int t = 0; t < f.nt; t++) {
            int8_t* s = f.cell(t + f.nt * p);
            for (int64_t v = 0; v < f.n; v++) {
                if (clamped[v]) {
                    int8_t val = cval[v] == 1 ? 1 : 0;
                    for (int r = 0; r < NR; r++) s[v * NR + r] = val;
                } else if (probs) {
                    for (int r = 0; r < NR; r++) s[v * NR + r] = rng.gen_range(0.0, 1.0) < probs[v] ? 1 : 0;
                } else {
                    uint64_t w = rng.next_u64();
                    for (int r = 0; r < NR; r++) s[v * NR + r] = (int8_t)((w >> r) & 1);
                }
            }
        }
}

// ultimate.rs:237-246
static std::vector<double> geometric_temps(double tmax, double tmin, int nt) {
    double f = nt > 1 ? std::pow(tmin / tmax, 1.0 / (double)(nt - 1)) : 1.0;
    std::vector<double> t(nt);
    for (int i = 0; i < nt; i++) t[i] = tmax * powi(f, i);
    return t;
}

// ultimate.rs:397-430 (num_slices = 1)
static void update_incumbent(const Qubo& m, Field& f, double& best_e, std::vector<int8_t>& best,
                             std::vector<int8_t>& buf) {
    int arg_c = 0, arg_r = 0;
    double mn = std::numeric_limits<double>::infinity();
    for (size_t c = 0; c < f.energies.size(); c++)
        for (int r = 0; r < NR; r++)
            if (f.energies[c][r] < mn) {
                mn = f.energies[c][r];
                arg_c = (int)c;
                arg_r = r;
            }
    if (!std::isfinite(mn)) return;
    const int8_t* s = f.cell(arg_c);
    for (int64_t v = 0; v < f.n; v++) buf[v] = s[v * NR + arg_r];
    double e = total_energy(m, buf.data());
    if (e < best_e) {
        best_e = e;
        best = buf;
    }
}

// rand 0.8.5 UniformInt<usize>::sample_single_inclusive (gen_range(0..=hi) on
// a 64-bit target): range = hi + 1, zone = (range << lz(range)) - 1; draws
// u64 v until the low half of the 128-bit v * range is <= zone and returns
// the high half. gen_range(0..len) is the same with hi = len - 1.
static uint64_t gen_index_inclusive(ChaCha8Rng& rng, uint64_t hi) {
    const uint64_t range = hi + 1;
    if (range == 0) return rng.next_u64();
    const uint64_t zone = (range << __builtin_clzll(range)) - 1;
    for (;;) {
        const unsigned __int128 m = (unsigned __int128)rng.next_u64() * range;
        if ((uint64_t)m <= zone) return (uint64_t)(m >> 64);
    }
}

// Houdayer / ICM move on lanes (a, b) of cell c (src/solver/icm.rs:91-158):
// the disagreement sites, a seed among them by gen_range(0..len), the
// connected disagreement cluster grown depth-first along the CSR rows,
// delta_a in cluster order (icm.rs:55-89), the cluster flipped in both lanes,
// the tracked energies moved by +-delta_a.
static void icm_pair_move(Field& f, const Qubo& m, int c, int a, int b, ChaCha8Rng& rng) {
    const int64_t n = f.n;
    int8_t* s = f.cell(c);
    std::vector<char> vis(n), in_c(n, 0);
    std::vector<int64_t> dis;
    for (int64_t v = 0; v < n; v++) {
        vis[v] = (s[v * NR + a] ^ s[v * NR + b]) == 0;
        if (!vis[v]) dis.push_back(v);
    }
    if (dis.empty()) return;
    const int64_t seed = dis[gen_index_inclusive(rng, dis.size() - 1)];
    std::vector<int64_t> stack{seed}, cluster;
    vis[seed] = 1;
    in_c[seed] = 1;
    while (!stack.empty()) {
        const int64_t i = stack.back();
        stack.pop_back();
        cluster.push_back(i);
        for (int64_t e = m.row[i]; e < m.row[i + 1]; e++) {
            const int64_t j = m.col[e];
            if (!vis[j]) {
                vis[j] = 1;
                in_c[j] = 1;
                stack.push_back(j);
            }
        }
    }
    double delta = 0.0;
    for (int64_t i : cluster) {
        const double xi = (double)s[i * NR + a];
        delta += m.linear[i] * (1.0 - 2.0 * xi);
        for (int64_t e = m.row[i]; e < m.row[i + 1]; e++) {
            const int64_t j = m.col[e];
            const double w = m.val[e];
            if (in_c[j]) {
                if (i < j) {
                    const double xj = (double)s[j * NR + a];
                    delta += w * ((1.0 - xi) * (1.0 - xj) - xi * xj);
                }
            } else {
                const double xj = (double)s[j * NR + a];
                delta += w * xj * (1.0 - 2.0 * xi);
            }
        }
    }
    for (int64_t i : cluster) {
        s[i * NR + a] ^= 1;
        s[i * NR + b] ^= 1;
    }
    f.energies[c][a] += delta;
    f.energies[c][b] -= delta;
}

// icm.rs:161-185: lanes (r, r + 32) of every cell, p then t then r.
static void icm_sweep(Field& f, const Qubo& m, ChaCha8Rng& rng) {
    for (int p = 0; p < f.np; p++)
        for (int t = 0; t < f.nt; t++)
            for (int r = 0; r < NR / 2; r++) icm_pair_move(f, m, t + f.nt * p, r, r + NR / 2, rng);
}

// ---------------------------------------------------------------------------
// Presolve (src/presolve/mod.rs, src/presolve/qpbo.rs) and 1-opt polish
// (src/solver/local_search.rs:19-57): needed only to reproduce the end-to-end
// golden through UltimateSolver::solve.
// ---------------------------------------------------------------------------
using Assign = std::vector<std::pair<int64_t, int8_t>>;

// presolve/mod.rs:54-105
static std::vector<int8_t> first_order_fixpoint(const Qubo& m, const Assign& assumptions) {
    const int64_t n = m.n;
    std::vector<double> h = m.linear;
    std::vector<int8_t> status(n, -1);
    for (auto& a : assumptions) status[a.first] = a.second;
    for (auto& a : assumptions)
        if (a.second == 1)
            for (int64_t k = m.row[a.first]; k < m.row[a.first + 1]; k++) h[m.col[k]] += m.val[k];
    for (;;) {
        bool changed = false;
        for (int64_t i = 0; i < n; i++) {
            if (status[i] >= 0) continue;
            double lo = h[i], hi = h[i];
            for (int64_t k = m.row[i]; k < m.row[i + 1]; k++)
                if (status[m.col[k]] < 0) {
                    double w = m.val[k];
                    if (w < 0.0) lo += w;
                    else hi += w;
                }
            if (lo >= 0.0) {
                status[i] = 0;
                changed = true;
            } else if (hi <= 0.0) {
                status[i] = 1;
                for (int64_t k = m.row[i]; k < m.row[i + 1]; k++) h[m.col[k]] += m.val[k];
                changed = true;
            }
        }
        if (!changed) break;
    }
    return status;
}

static bool has_index(const Assign& a, int64_t i) {
    for (auto& x : a)
        if (x.first == i) return true;
    return false;
}

// presolve/mod.rs:126-183
static Assign probing(const Qubo& m, const Assign& clamped) {
    const int64_t n = m.n;
    std::vector<uint8_t> user(n, 0);
    Assign assumptions = clamped;
    for (auto& c : clamped) user[c.first] = 1;
    for (;;) {
        auto base = first_order_fixpoint(m, assumptions);
        Assign newly;
        Assign assumed;
        for (int64_t i = 0; i < n; i++)
            if (base[i] >= 0) assumed.push_back({i, base[i]});
        for (int64_t i = 0; i < n; i++) {
            if (base[i] >= 0) continue;
            Assign a0 = assumed;
            a0.push_back({i, 0});
            auto b0 = first_order_fixpoint(m, a0);
            Assign a1 = assumed;
            a1.push_back({i, 1});
            auto b1 = first_order_fixpoint(m, a1);
            for (int64_t j = 0; j < n; j++) {
                if (j == i || base[j] >= 0) continue;
                if (b0[j] >= 0 && b1[j] >= 0 && b0[j] == b1[j] && !has_index(newly, j))
                    newly.push_back({j, b0[j]});
            }
        }
        size_t before = assumptions.size();
        for (auto& x : assumed)
            if (!has_index(assumptions, x.first)) assumptions.push_back(x);
        for (auto& x : newly)
            if (!has_index(assumptions, x.first)) assumptions.push_back(x);
        if (assumptions.size() == before) break;
    }
    Assign out;
    for (auto& x : assumptions)
        if (!user[x.first]) out.push_back(x);
    return out;
}

// qpbo.rs:43-140: Dinic max-flow on f64 capacities.
struct Dinic {
    int n;
    std::vector<std::vector<int>> head;
    std::vector<int> to;
    std::vector<double> cap;
    std::vector<int> level, it;
    static constexpr double EPS = 1e-9;
    explicit Dinic(int n_) : n(n_), head(n_), level(n_, 0), it(n_, 0) {}
    void add_edge(int u, int v, double c) {
        int e = (int)to.size();
        to.push_back(v);
        cap.push_back(c);
        head[u].push_back(e);
        to.push_back(u);
        cap.push_back(0.0);
        head[v].push_back(e + 1);
    }
    bool bfs(int s, int t) {
        std::fill(level.begin(), level.end(), -1);
        std::deque<int> q;
        level[s] = 0;
        q.push_back(s);
        while (!q.empty()) {
            int u = q.front();
            q.pop_front();
            for (int e : head[u])
                if (cap[e] > EPS && level[to[e]] < 0) {
                    level[to[e]] = level[u] + 1;
                    q.push_back(to[e]);
                }
        }
        return level[t] >= 0;
    }
    double dfs(int u, int t, double f) {
        if (u == t) return f;
        while (it[u] < (int)head[u].size()) {
            int e = head[u][it[u]];
            int v = to[e];
            if (cap[e] > EPS && level[v] == level[u] + 1) {
                double d = dfs(v, t, std::min(f, cap[e]));
                if (d > EPS) {
                    cap[e] -= d;
                    cap[e ^ 1] += d;
                    return d;
                }
            }
            it[u]++;
        }
        return 0.0;
    }
    double max_flow(int s, int t) {
        double flow = 0.0;
        while (bfs(s, t)) {
            std::fill(it.begin(), it.end(), 0);
            for (;;) {
                double f = dfs(s, t, std::numeric_limits<double>::infinity());
                if (f <= EPS) break;
                flow += f;
            }
        }
        return flow;
    }
};

static std::vector<uint8_t> bfs_reach(const std::vector<std::vector<int>>& adj, int s) {
    std::vector<uint8_t> seen(adj.size(), 0);
    std::deque<int> q;
    seen[s] = 1;
    q.push_back(s);
    while (!q.empty()) {
        int u = q.front();
        q.pop_front();
        for (int v : adj[u])
            if (!seen[v]) {
                seen[v] = 1;
                q.push_back(v);
            }
    }
    return seen;
}

// qpbo.rs:160-266
static std::vector<int8_t> roof_duality(const Qubo& m) {
    const int64_t n = m.n;
    if (n == 0) return {};
    const int src = (int)(2 * n), sink = (int)(2 * n + 1);
    auto node_comp = [&](int lit) { return lit == src ? sink : (lit == sink ? src : (lit ^ 1)); };
    Dinic g((int)(2 * n + 2));
    double scale = 0.0;
    for (int64_t i = 0; i < n; i++) {
        scale = std::max(scale, std::fabs(m.linear[i]));
        for (int64_t k = m.row[i]; k < m.row[i + 1]; k++) scale = std::max(scale, std::fabs(m.val[k]));
    }
    if (!(scale > 0.0)) scale = 1.0;
    const double EPS = Dinic::EPS;
    auto add_quad = [&](int u, int v, double c) {
        if (c > EPS) {
            g.add_edge(u, node_comp(v), c);
            g.add_edge(v, node_comp(u), c);
        }
    };
    auto add_linear = [&](int u, double c) {
        if (c >= 0.0) {
            if (c > EPS) {
                g.add_edge(u, sink, c);
                g.add_edge(src, node_comp(u), c);
            }
        } else {
            double cc = -c;
            int ubar = node_comp(u);
            g.add_edge(ubar, sink, cc);
            g.add_edge(src, u, cc);
        }
    };
    for (int64_t i = 0; i < n; i++) add_linear((int)(2 * i), m.linear[i] / scale);
    for (int64_t i = 0; i < n; i++)
        for (int64_t k = m.row[i]; k < m.row[i + 1]; k++) {
            int64_t j = m.col[k];
            if (i < j) {
                double w = m.val[k] / scale;
                if (w >= 0.0) {
                    add_quad((int)(2 * i), (int)(2 * j), w);
                } else {
                    add_linear((int)(2 * i), w);
                    add_quad((int)(2 * i), (int)(2 * j + 1), -w);
                }
            }
        }
    g.max_flow(src, sink);
    std::vector<std::vector<int>> adj(g.n), radj(g.n);
    for (int u = 0; u < g.n; u++)
        for (int e : g.head[u])
            if (g.cap[e] > EPS) adj[u].push_back(g.to[e]);
    for (int u = 0; u < g.n; u++)
        for (int v : adj[u]) radj[v].push_back(u);
    auto in_s = bfs_reach(adj, src);
    auto in_t = bfs_reach(radj, sink);
    std::vector<int8_t> out(n, -1);
    for (int64_t i = 0; i < n; i++) {
        int p = (int)(2 * i), q = (int)(2 * i + 1);
        if (in_s[p] && in_t[q]) out[i] = 1;
        else if (in_t[p] && in_s[q]) out[i] = 0;
    }
    return out;
}

// presolve/mod.rs:328-381
static Qubo reduce_by_clamps(const Qubo& m, const Assign& clamped, std::vector<int64_t>& free_map) {
    const int64_t n = m.n;
    std::vector<int8_t> cv(n, -1);
    for (auto& c : clamped) cv[c.first] = c.second;
    free_map.clear();
    for (int64_t i = 0; i < n; i++)
        if (cv[i] < 0) free_map.push_back(i);
    std::vector<int64_t> g2l(n, -1);
    for (size_t li = 0; li < free_map.size(); li++) g2l[free_map[li]] = (int64_t)li;
    const int64_t mm = (int64_t)free_map.size();
    Qubo r;
    r.n = mm;
    r.linear.assign(mm, 0.0);
    std::vector<std::vector<std::pair<int64_t, double>>> rows(mm);
    for (int64_t li = 0; li < mm; li++) {
        int64_t gi = free_map[li];
        double h = m.linear[gi];
        for (int64_t k = m.row[gi]; k < m.row[gi + 1]; k++) {
            int64_t j = m.col[k];
            if (cv[j] < 0) {
                if (g2l[j] >= 0) rows[li].push_back({g2l[j], m.val[k]});
            } else if (cv[j] == 1) {
                h += m.val[k];
            }
        }
        r.linear[li] = h;
    }
    r.row.push_back(0);
    for (auto& rw : rows) {
        std::stable_sort(rw.begin(), rw.end(),
                         [](const std::pair<int64_t, double>& a, const std::pair<int64_t, double>& b) {
                             return a.first < b.first;
                         });
        for (auto& e : rw) {
            r.col.push_back(e.first);
            r.val.push_back(e.second);
        }
        r.row.push_back((int64_t)r.col.size());
    }
    return r;
}

// presolve/mod.rs:283-321
static Assign full_presolve(const Qubo& m, const Assign& clamped) {
    const int64_t n = m.n;
    std::vector<uint8_t> user(n, 0);
    for (auto& c : clamped) user[c.first] = 1;
    Assign assumptions = clamped;
    std::vector<int64_t> free_map;
    Qubo red = reduce_by_clamps(m, clamped, free_map);
    auto rd = roof_duality(red);
    for (size_t li = 0; li < rd.size(); li++) {
        if (rd[li] < 0) continue;
        int64_t gi = free_map[li];
        if (!user[gi] && !has_index(assumptions, gi)) assumptions.push_back({gi, rd[li]});
    }
    auto probed = probing(m, assumptions);
    for (auto& x : probed)
        if (!user[x.first] && !has_index(assumptions, x.first)) assumptions.push_back(x);
    Assign out;
    for (auto& x : assumptions)
        if (!user[x.first]) out.push_back(x);
    return out;
}

// presolve/mod.rs:194-219
static std::vector<std::vector<int64_t>> connected_components(const Qubo& m,
                                                              const std::vector<uint8_t>& active) {
    const int64_t n = m.n;
    std::vector<uint8_t> visited(n, 0);
    std::vector<std::vector<int64_t>> comps;
    std::vector<int64_t> stack;
    for (int64_t s = 0; s < n; s++) {
        if (!active[s] || visited[s]) continue;
        std::vector<int64_t> comp;
        visited[s] = 1;
        stack.push_back(s);
        while (!stack.empty()) {
            int64_t v = stack.back();
            stack.pop_back();
            comp.push_back(v);
            for (int64_t k = m.row[v]; k < m.row[v + 1]; k++) {
                int64_t j = m.col[k];
                if (m.val[k] != 0.0 && active[j] && !visited[j]) {
                    visited[j] = 1;
                    stack.push_back(j);
                }
            }
        }
        std::sort(comp.begin(), comp.end());
        comps.push_back(comp);
    }
    return comps;
}

// presolve/mod.rs:228-270
static Qubo extract_component(const Qubo& m, const std::vector<int64_t>& comp,
                              const std::vector<uint8_t>& fixed_one) {
    std::vector<int64_t> g2l(m.n, -1);
    for (size_t li = 0; li < comp.size(); li++) g2l[comp[li]] = (int64_t)li;
    Qubo r;
    r.n = (int64_t)comp.size();
    r.row.push_back(0);
    for (int64_t gi : comp) {
        double h = m.linear[gi];
        for (int64_t k = m.row[gi]; k < m.row[gi + 1]; k++) {
            int64_t j = m.col[k];
            if (g2l[j] >= 0) {
                r.col.push_back(g2l[j]);
                r.val.push_back(m.val[k]);
            } else if (fixed_one[j]) {
                h += m.val[k];
            }
        }
        r.linear.push_back(h);
        r.row.push_back((int64_t)r.col.size());
    }
    r.offset = 0.0;
    return r;
}

// local_search.rs:19-57
static double one_opt(const Qubo& m, int8_t* state, const std::vector<uint8_t>& clamped) {
    const int64_t n = m.n;
    std::vector<double> gains(n);
    for (int64_t i = 0; i < n; i++) {
        double field = m.linear[i];
        for (int64_t k = m.row[i]; k < m.row[i + 1]; k++) field += m.val[k] * (double)state[m.col[k]];
        gains[i] = (1.0 - 2.0 * (double)state[i]) * field;
    }
    double total = 0.0;
    for (;;) {
        int64_t bi = -1;
        double bg = -1e-12;
        for (int64_t i = 0; i < n; i++)
            if (!clamped[i] && gains[i] < bg) {
                bi = i;
                bg = gains[i];
            }
        if (bi < 0) return total;
        total -= bg;
        double dir = 1.0 - 2.0 * (double)state[bi];
        state[bi] = (int8_t)(1 - state[bi]);
        gains[bi] = -bg;
        for (int64_t k = m.row[bi]; k < m.row[bi + 1]; k++) {
            int64_t j = m.col[k];
            gains[j] += (1.0 - 2.0 * (double)state[j]) * m.val[k] * dir;
        }
    }
}

// local_search.rs:123-143 with find_steepest_2opt_edge_flip (:83-121):
// 1-opt, fresh gains, the steepest improving edge 2-flip (strict <, first
// found on ties), repeated; returns max(0, E_before - E_after).
static double two_opt(const Qubo& m, int8_t* state, const std::vector<uint8_t>& clamped) {
    const int64_t n = m.n;
    const double e0 = total_energy(m, state);
    std::vector<double> g(n);
    for (;;) {
        one_opt(m, state, clamped);
        for (int64_t i = 0; i < n; i++) {
            double field = m.linear[i];
            for (int64_t k = m.row[i]; k < m.row[i + 1]; k++) field += m.val[k] * (double)state[m.col[k]];
            g[i] = (1.0 - 2.0 * (double)state[i]) * field;
        }
        int64_t bu = -1, bv = -1;
        double bd = 0.0;
        for (int64_t u = 0; u < n; u++) {
            if (clamped[u]) continue;
            const double su = 1.0 - 2.0 * (double)state[u];
            for (int64_t k = m.row[u]; k < m.row[u + 1]; k++) {
                const int64_t v = m.col[k];
                if (v > u && !clamped[v]) {
                    const double sv = 1.0 - 2.0 * (double)state[v];
                    const double d = g[u] + g[v] + m.val[k] * su * sv;
                    if (d < -1e-12 && (bu < 0 || d < bd)) {
                        bu = u;
                        bv = v;
                        bd = d;
                    }
                }
            }
        }
        if (bu < 0) break;
        state[bu] = (int8_t)(1 - state[bu]);
        state[bv] = (int8_t)(1 - state[bv]);
    }
    return std::max(0.0, e0 - total_energy(m, state));
}

// src/solver/elite.rs:21-123 (EliteArchive) and :133-181 (path_relink), and
// the finisher of ultimate.rs:436-479.
struct EliteArchive {
    size_t cap, min_h;
    std::vector<std::pair<double, std::vector<int8_t>>> entries;

    static size_t hamming(const std::vector<int8_t>& a, const std::vector<int8_t>& b) {
        size_t d = 0;
        for (size_t i = 0; i < a.size(); i++) d += a[i] != b[i];
        return d;
    }
    void sort_and_trim() {
        std::stable_sort(entries.begin(), entries.end(),
                         [](const auto& a, const auto& b) { return a.first < b.first; });
        if (entries.size() > cap) entries.resize(cap);
    }
    void insert(const std::vector<int8_t>& x, double e) {
        for (size_t i = 0; i < entries.size(); i++)
            if (hamming(entries[i].second, x) < std::max<size_t>(min_h, 1)) {
                if (e < entries[i].first - 1e-12) {
                    entries[i] = {e, x};
                    sort_and_trim();
                }
                return;
            }
        if (entries.size() < cap) {
            entries.push_back({e, x});
            sort_and_trim();
            return;
        }
        const double worst = entries.empty() ? std::numeric_limits<double>::infinity() : entries.back().first;
        if (e < worst - 1e-12) {
            entries.push_back({e, x});
            sort_and_trim();
        }
    }
};

static std::vector<int8_t> path_relink(const Qubo& m, const std::vector<int8_t>& source,
                                       const std::vector<int8_t>& target) {
    const int64_t n = m.n;
    std::vector<int8_t> x = source, best = source;
    double e = total_energy(m, x.data()), be = e;
    std::vector<double> g(n);
    for (int64_t i = 0; i < n; i++) {
        double field = m.linear[i];
        for (int64_t k = m.row[i]; k < m.row[i + 1]; k++) field += m.val[k] * (double)x[m.col[k]];
        g[i] = (1.0 - 2.0 * (double)x[i]) * field;
    }
    std::vector<int64_t> differing;
    for (int64_t i = 0; i < n; i++)
        if (source[i] != target[i]) differing.push_back(i);
    while (!differing.empty()) {
        size_t pick = 0;
        double bg = std::numeric_limits<double>::infinity();
        for (size_t k = 0; k < differing.size(); k++)
            if (g[differing[k]] < bg - 1e-15) {
                bg = g[differing[k]];
                pick = k;
            }
        const int64_t i = differing[pick];
        differing[pick] = differing.back();
        differing.pop_back();
        const double dir = 1.0 - 2.0 * (double)x[i];
        e += g[i];
        x[i] = (int8_t)(1 - x[i]);
        g[i] = -g[i];
        for (int64_t k = m.row[i]; k < m.row[i + 1]; k++) {
            const int64_t j = m.col[k];
            g[j] += (1.0 - 2.0 * (double)x[j]) * m.val[k] * dir;
        }
        if (e < be) {
            be = e;
            best = x;
        }
    }
    return best;
}

static std::vector<int8_t> path_relink_finish(const Qubo& m, const std::vector<uint64_t>& words, int64_t cells,
                                              const std::vector<uint8_t>& clamped, std::vector<int8_t> current,
                                              double current_e, double& best_e_out) {
    const int64_t n = m.n;
    EliteArchive arch{8, (size_t)std::max<int64_t>(n / 10, 1), {}};
    arch.insert(current, current_e);
    std::vector<int8_t> buf(n);
    for (int64_t c = 0; c < cells; c++)
        for (int r = 0; r < NR; r++) {
            for (int64_t v = 0; v < n; v++) buf[v] = (int8_t)((words[c * n + v] >> r) & 1);
            arch.insert(buf, total_energy(m, buf.data()));
        }
    std::vector<int8_t> best = current;
    double be = current_e;
    for (size_t i = 0; i < arch.entries.size(); i++)
        for (size_t j = i + 1; j < arch.entries.size(); j++) {
            std::vector<int8_t> x = path_relink(m, arch.entries[i].second, arch.entries[j].second);
            one_opt(m, x.data(), clamped);
            const double e = total_energy(m, x.data());
            if (e < be) {
                be = e;
                best = x;
            }
        }
    best_e_out = be;
    return best;
}

struct SolverCfg {
    double tmax, tmin;
    int64_t sweeps, exchanges;
    uint64_t seed;
    int nt;
    int threads;
    bool icm = false;  // UltimateSolver::use_icm (pairwise QUBO input: always applicable)
};

// UltimateSolver::solve, ultimate.rs:138-387, PT path (num_pops = 1,
// num_slices = 1, no GNN warm start, ICM / 2-opt / path relinking off as in
// UltimateSolver::new).
static std::vector<int8_t> solve(const Qubo& m, const Assign& clamped, const SolverCfg& cfg) {
    const int64_t n = m.n;
    ChaCha8Rng rng(cfg.seed);
    std::vector<uint8_t> is_clamped(n, 0);
    std::vector<int8_t> cval(n, 0);
    for (auto& c : clamped) {
        is_clamped[c.first] = 1;
        cval[c.first] = c.second;
    }
    auto derived = full_presolve(m, clamped);
    for (auto& d : derived) {
        is_clamped[d.first] = 1;
        cval[d.first] = d.second;
    }
    std::vector<uint8_t> free(n);
    for (int64_t i = 0; i < n; i++) free[i] = !is_clamped[i];
    auto comps = connected_components(m, free);
    if (comps.size() > 1) {
        std::vector<uint8_t> fixed_one(n, 0);
        std::vector<int8_t> result(n, 0);
        for (int64_t v = 0; v < n; v++)
            if (is_clamped[v]) {
                result[v] = cval[v];
                fixed_one[v] = cval[v] == 1;
            }
        for (size_t ci = 0; ci < comps.size(); ci++) {
            Qubo sub = extract_component(m, comps[ci], fixed_one);
            SolverCfg sc = cfg;
            sc.seed = cfg.seed + (uint64_t)ci + 1;
            auto ss = solve(sub, {}, sc);
            for (size_t li = 0; li < comps[ci].size(); li++) result[comps[ci][li]] = ss[li];
        }
        return result;
    }
    Field f(n, cfg.nt, 1);
    auto temps = geometric_temps(cfg.tmax, cfg.tmin, cfg.nt);
    init_field(f, is_clamped, cval, rng);
    for (int t = 0; t < cfg.nt; t++) replica_energies(m, f.cell(t), f.energies[t].data());
    StepScratch sc;
    sc.attempts.assign(std::max(cfg.nt - 1, 0), 0);
    sc.accepts.assign(std::max(cfg.nt - 1, 0), 0);
    double inc_e = std::numeric_limits<double>::infinity();
    std::vector<int8_t> inc(n, 0), buf(n, 0);
    uint64_t counter = 0;
    for (int64_t ex = 0; ex < cfg.exchanges; ex++) {
        for (int64_t sw = 0; sw < cfg.sweeps; sw++) {
            step(f, m, temps.data(), is_clamped, sc, rng, true, false, cfg.threads, nullptr);
            counter++;
            if (counter % 1000 == 0)
                for (int t = 0; t < cfg.nt; t++) replica_energies(m, f.cell(t), f.energies[t].data());
        }
        if (cfg.icm) icm_sweep(f, m, rng);  // ultimate.rs:326-328
        update_incumbent(m, f, inc_e, inc, buf);
    }
    std::vector<int8_t> best(n, 0), rb((size_t)NR * n);
    double best_e = std::numeric_limits<double>::infinity();
    for (int t = 0; t < cfg.nt; t++) {
        const int8_t* s = f.cell(t);
        for (int64_t v = 0; v < n; v++)
            for (int r = 0; r < NR; r++) rb[(size_t)r * n + v] = s[v * NR + r];
        for (int r = 0; r < NR; r++) {
            double e = total_energy(m, rb.data() + (size_t)r * n);
            if (e < best_e) {
                best_e = e;
                std::copy(rb.begin() + (size_t)r * n, rb.begin() + (size_t)(r + 1) * n, best.begin());
            }
        }
    }
    if (inc_e < best_e) best = inc;
    one_opt(m, best.data(), is_clamped);
    return best;
}

// ---------------------------------------------------------------------------
// Population annealing with PT equilibration (num_pops > 1):
// src/solver/population_annealing.rs:51-287 (weights, ESS, free energy,
// family entropy, systematic resampling, spacing adaptation, apply_resample)
// and UltimateSolver::solve_population_annealing_diag (ultimate.rs:576-852)
// with either ladder mode (acceptance-uniform, the default, or feedback-
// optimized with round-trip tracking) and optional ICM; GNN warm start and
// 2-opt off. Entered as solve_with_pa_diagnostics does (ultimate.rs:858-890):
// no presolve or decomposition.
// ---------------------------------------------------------------------------

// population_annealing.rs:51-56
static std::vector<double> pa_normalized_weights(const std::vector<double>& lw) {
    double m = -std::numeric_limits<double>::infinity();
    for (double x : lw) m = std::max(m, x);
    std::vector<double> e(lw.size());
    double z = 0.0;
    for (size_t i = 0; i < lw.size(); i++) {
        e[i] = std::exp(lw[i] - m);
        z += e[i];
    }
    for (double& x : e) x /= z;
    return e;
}

// population_annealing.rs:60-63
static double pa_ess(const std::vector<double>& w) {
    double s2 = 0.0;
    for (double x : w) s2 += x * x;
    return 1.0 / s2;
}

// population_annealing.rs:70-78
static double pa_free_energy_increment(const std::vector<double>& lw) {
    const double r = (double)lw.size();
    double m = -std::numeric_limits<double>::infinity();
    for (double x : lw) m = std::max(m, x);
    if (!std::isfinite(m)) return 0.0;
    double s = 0.0;
    for (double x : lw) s += std::exp(x - m);
    return m + std::log(s) - std::log(r);
}

// population_annealing.rs:84-101; families summed in ascending id order (the
// reference sums in its hash map's order, which is unspecified).
static std::pair<double, int64_t> pa_family_entropy(const std::vector<int64_t>& ids) {
    if (ids.empty()) return {0.0, 0};
    std::map<int64_t, int64_t> cnt;
    for (int64_t f : ids) cnt[f]++;
    const double r = (double)ids.size();
    double rho = 0.0;
    for (auto& kv : cnt) {
        const double frac = (double)kv.second / r;
        rho += frac * frac;
    }
    return {rho * r, (int64_t)cnt.size()};
}

// population_annealing.rs:106-127
static std::vector<int64_t> pa_systematic_resample(const std::vector<double>& w, double u) {
    const size_t R = w.size();
    std::vector<int64_t> counts(R, 0);
    double cum = 0.0;
    size_t j = 0;
    for (size_t i = 0; i < R; i++) {
        cum += w[i];
        while (j < R && (((double)j + u) / (double)R) < cum) {
            counts[i]++;
            j++;
        }
    }
    if (j < R) counts[R - 1] += (int64_t)(R - j);
    return counts;
}

// population_annealing.rs:141-152
static std::vector<double> pa_adapt_spacings(const std::vector<double>& d, const std::vector<double>& a) {
    std::vector<double> raw(d.size());
    double old_total = 0.0, new_total = 0.0;
    for (size_t k = 0; k < d.size(); k++) raw[k] = d[k] * std::sqrt(std::max(a[k], 0.02));
    for (double x : d) old_total += x;
    for (double x : raw) new_total += x;
    for (double& x : raw) x = x * old_total / new_total;
    return raw;
}

// population_annealing.rs:240-287: parents per offspring slot, Fisher-Yates
// shuffled with gen_range(0..=k), then every level's configuration and
// tracked energies of member dst = parent member src.
static std::vector<int64_t> pa_apply_resample(Field& f, const std::vector<int64_t>& counts, ChaCha8Rng& rng) {
    const int64_t R = (int64_t)f.np * NR;
    std::vector<int64_t> parents;
    for (int64_t i = 0; i < R; i++)
        for (int64_t c = 0; c < counts[i]; c++) parents.push_back(i);
    for (int64_t k = (int64_t)parents.size() - 1; k >= 1; k--) {
        const int64_t j = (int64_t)gen_index_inclusive(rng, (uint64_t)k);
        std::swap(parents[k], parents[j]);
    }
    const std::vector<int8_t> old = f.spins;
    const auto old_e = f.energies;
    for (int64_t dst = 0; dst < R; dst++) {
        const int64_t src = parents[dst];
        if (dst == src) continue;
        const int64_t dp = dst / NR, dr = dst % NR, sp = src / NR, sr = src % NR;
        for (int t = 0; t < f.nt; t++) {
            const size_t dc = (size_t)(t + f.nt * dp) * f.n, sc = (size_t)(t + f.nt * sp) * f.n;
            for (int64_t v = 0; v < f.n; v++) f.spins[(dc + v) * NR + dr] = old[(sc + v) * NR + sr];
            f.energies[t + f.nt * dp][dr] = old_e[t + f.nt * sp][sr];
        }
    }
    return parents;
}

// population_annealing.rs:172-232: monotone flow, interval masses
// sqrt(max(|df|, 1e-6) * max(|da|, 1e-6)), interior points equidistributed
// in cumulative mass (damped), strict order enforced, endpoints rescaled.
static std::vector<double> pa_feedback_alphas(const std::vector<double>& alphas, const std::vector<double>& flow,
                                              double damping) {
    const size_t nt = alphas.size();
    if (nt < 3) return alphas;
    std::vector<double> f = flow;
    for (size_t k = 1; k < nt; k++)
        if (f[k] < f[k - 1]) f[k] = f[k - 1];
    const double eps = 1e-6;
    std::vector<double> mass(nt - 1);
    for (size_t k = 0; k + 1 < nt; k++)
        mass[k] = std::sqrt(std::max(std::fabs(f[k + 1] - f[k]), eps) * std::max(std::fabs(alphas[k + 1] - alphas[k]), eps));
    double total = 0.0;
    for (double x : mass) total += x;
    if (total <= 0.0 || !std::isfinite(total)) return alphas;
    std::vector<double> cum(nt, 0.0);
    for (size_t k = 0; k + 1 < nt; k++) cum[k + 1] = cum[k] + mass[k];
    std::vector<double> na(nt, 0.0);
    na[0] = alphas[0];
    na[nt - 1] = alphas[nt - 1];
    for (size_t i = 1; i + 1 < nt; i++) {
        const double target = (double)i / (double)(nt - 1) * total;
        size_t k = 0;
        while (k < nt - 2 && cum[k + 1] < target) k++;
        const double frac = mass[k] > 0.0 ? (target - cum[k]) / mass[k] : 0.0;
        const double interp = alphas[k] + frac * (alphas[k + 1] - alphas[k]);
        na[i] = damping * interp + (1.0 - damping) * alphas[i];
    }
    for (size_t i = 1; i < nt; i++)
        if (na[i] <= na[i - 1]) na[i] = na[i - 1] + eps;
    const double base = na[0], span = na[nt - 1] - na[0], old_span = alphas[nt - 1] - alphas[0];
    if (span > 0.0)
        for (double& a : na) a = alphas[0] + (a - base) / span * old_span;
    return na;
}

struct PaCfg {
    double tmax, tmin;
    int64_t sweeps, exchanges;
    uint64_t seed;
    int nt, pops;
    double ess_threshold;
    int64_t tuning_iters, tuning_steps, relax;
    int threads;
    int ladder_mode;  // 0 acceptance-uniform, 1 feedback-optimized
    bool icm = false;
};

struct PaOut {
    std::vector<double> alphas, ess, rho;
    std::vector<int64_t> families;
    double free_energy = 0.0;
    int64_t resamples = 0;
    std::vector<int8_t> best_pre, best;
    double incumbent_e = 0.0;
};

static void all_energies(const Qubo& m, Field& f) {
    for (int c = 0; c < f.nt * f.np; c++) replica_energies(m, f.cell(c), f.energies[c].data());
}

// ultimate.rs:576-852 (defaults as above; num_slices = 1)
static Field pa_run(const Qubo& m, const std::vector<uint8_t>& is_clamped, const std::vector<int8_t>& cval,
                    const PaCfg& cfg, PaOut& out, ChaCha8Rng& rng) {
    const int64_t n = m.n;
    const int nt = std::max(cfg.nt, 1), pops = cfg.pops;
    const int64_t R = (int64_t)pops * NR;
    std::vector<int64_t> family(R);
    for (int64_t i = 0; i < R; i++) family[i] = i;
    const double denom = (double)std::max(nt - 1, 1);
    std::vector<double> alphas(nt);
    for (int t = 0; t < nt; t++) alphas[t] = (double)t / denom;
    std::vector<double> temps(nt);
    if (nt >= 3 && cfg.tuning_iters > 0 && cfg.tuning_steps > 0) {
        Field tf(n, nt, pops);
        init_field(tf, is_clamped, cval, rng);
        all_energies(m, tf);
        StepScratch sc;
        sc.attempts.assign(nt - 1, 0);
        sc.accepts.assign(nt - 1, 0);
        const bool feedback = cfg.ladder_mode == 1;
        sc.track = feedback;
        sc.labels.assign((size_t)nt * pops, {});
        sc.n_up.assign(nt, 0);
        sc.n_down.assign(nt, 0);
        for (int64_t it = 0; it < cfg.tuning_iters; it++) {
            for (int t = 0; t < nt; t++) temps[t] = cfg.tmax * std::pow(cfg.tmin / cfg.tmax, alphas[t]);
            if (feedback) {
                std::fill(sc.n_up.begin(), sc.n_up.end(), 0);
                std::fill(sc.n_down.begin(), sc.n_down.end(), 0);
                sc.rt = 0;
                for (auto& l : sc.labels) l.fill(0);
            } else {
                std::fill(sc.attempts.begin(), sc.attempts.end(), 0);
                std::fill(sc.accepts.begin(), sc.accepts.end(), 0);
            }
            for (int64_t s = 0; s < cfg.tuning_steps; s++)
                step(tf, m, temps.data(), is_clamped, sc, rng, true, !feedback, cfg.threads, nullptr);
            if (feedback) {
                if (sc.rt >= (uint64_t)nt) {
                    std::vector<double> flow(nt);
                    for (int t = 0; t < nt; t++) {
                        const uint64_t u = sc.n_up[t], d = sc.n_down[t];
                        flow[t] = u + d == 0 ? 0.0 : (double)u / (double)(u + d);
                    }
                    alphas = pa_feedback_alphas(alphas, flow, 0.5);
                    alphas[0] = 0.0;
                    alphas[nt - 1] = 1.0;
                }
                continue;
            }
            std::vector<double> rates(nt - 1), sp(nt - 1);
            for (int t = 0; t + 1 < nt; t++) {
                rates[t] = sc.attempts[t] == 0 ? 0.0 : (double)sc.accepts[t] / (double)sc.attempts[t];
                sp[t] = alphas[t + 1] - alphas[t];
            }
            const std::vector<double> ns = pa_adapt_spacings(sp, rates);
            double acc = 0.0;
            for (int t = 0; t + 1 < nt; t++) {
                acc += ns[t];
                alphas[t + 1] = acc;
            }
            alphas[nt - 1] = 1.0;
        }
    }
    out.alphas = alphas;
    Field f(n, nt, pops);
    init_field(f, is_clamped, cval, rng);
    all_energies(m, f);
    const int64_t K = std::max<int64_t>(cfg.exchanges, 1);
    const double cold_factor = K > 1 ? std::pow(cfg.tmin / cfg.tmax, 1.0 / (double)(K - 1)) : 1.0;
    StepScratch sc;
    sc.attempts.assign(std::max(nt - 1, 0), 0);
    sc.accepts.assign(std::max(nt - 1, 0), 0);
    std::vector<double> log_w(R, 0.0);
    bool have_prev = false;
    double beta_prev = 0.0;
    double inc_e = std::numeric_limits<double>::infinity();
    std::vector<int8_t> inc(n, 0), buf(n, 0);
    for (int64_t k = 0; k < K; k++) {
        const double t_cold = K > 1 ? cfg.tmax * powi(cold_factor, (int)k) : cfg.tmin;
        const double span = t_cold / cfg.tmax;
        for (int t = 0; t < nt; t++) temps[t] = cfg.tmax * std::pow(span, alphas[t]);
        const double beta_cold = 1.0 / t_cold;
        if (have_prev) {
            const double db = beta_cold - beta_prev;
            const int cold = nt - 1;
            for (int p = 0; p < pops; p++)
                for (int r = 0; r < NR; r++) log_w[p * NR + r] -= db * f.energies[cold + nt * p][r];
            const std::vector<double> w = pa_normalized_weights(log_w);
            const double ess = pa_ess(w);
            out.ess.push_back(ess);
            if (ess < cfg.ess_threshold * (double)R) {
                out.free_energy += pa_free_energy_increment(log_w);
                const double u = rng.gen_range(0.0, 1.0);
                const std::vector<int64_t> counts = pa_systematic_resample(w, u);
                const std::vector<int64_t> parents = pa_apply_resample(f, counts, rng);
                const std::vector<int64_t> old = family;
                for (int64_t d = 0; d < R; d++) family[d] = old[parents[d]];
                const auto fe = pa_family_entropy(family);
                out.rho.push_back(fe.first);
                out.families.push_back(fe.second);
                out.resamples++;
                std::fill(log_w.begin(), log_w.end(), 0.0);
                for (int64_t s = 0; s < cfg.relax; s++)
                    step(f, m, temps.data(), is_clamped, sc, rng, true, false, cfg.threads, nullptr);
            }
        }
        have_prev = true;
        beta_prev = beta_cold;
        for (int64_t s = 0; s < cfg.sweeps; s++)
            step(f, m, temps.data(), is_clamped, sc, rng, true, false, cfg.threads, nullptr);
        all_energies(m, f);
        if (cfg.icm) {  // ultimate.rs:800-808
            icm_sweep(f, m, rng);
            all_energies(m, f);
        }
        update_incumbent(m, f, inc_e, inc, buf);
    }
    // best member by true model energy (p, t, r order), then the incumbent
    std::vector<int8_t> best(n, 0), rb((size_t)NR * n);
    double best_e = std::numeric_limits<double>::infinity();
    for (int c = 0; c < nt * pops; c++) {
        const int8_t* s = f.cell(c);
        for (int64_t v = 0; v < n; v++)
            for (int r = 0; r < NR; r++) rb[(size_t)r * n + v] = s[v * NR + r];
        for (int r = 0; r < NR; r++) {
            const double e = total_energy(m, rb.data() + (size_t)r * n);
            if (e < best_e) {
                best_e = e;
                std::copy(rb.begin() + (size_t)r * n, rb.begin() + (size_t)(r + 1) * n, best.begin());
            }
        }
    }
    if (inc_e < best_e) best = inc;
    out.incumbent_e = inc_e;
    out.best_pre = best;
    one_opt(m, best.data(), is_clamped);
    out.best = best;
    return f;
}

static void pack_words(const Field& f, uint64_t* words) {
    const int cells = f.nt * f.np;
    for (int c = 0; c < cells; c++)
        for (int64_t v = 0; v < f.n; v++) {
            uint64_t w = 0;
            const int8_t* s = f.spins.data() + ((size_t)c * f.n + v) * NR;
            for (int r = 0; r < NR; r++) w |= (uint64_t)(s[r] & 1) << r;
            words[(size_t)c * f.n + v] = w;
        }
}

static void unpack_words(Field& f, const uint64_t* words) {
    const int cells = f.nt * f.np;
    for (int c = 0; c < cells; c++)
        for (int64_t v = 0; v < f.n; v++) {
            uint64_t w = words[(size_t)c * f.n + v];
            int8_t* s = f.spins.data() + ((size_t)c * f.n + v) * NR;
            for (int r = 0; r < NR; r++) s[r] = (int8_t)((w >> r) & 1);
        }
}

}  // namespace

// ===========================================================================
// C API (ctypes). Problems are passed as (n, linear, row_offsets, cols, vals,
// offset) with int64 CSR indices, mirroring QuboModel/CsrMatrix.
// ===========================================================================
namespace {

// ---------------------------------------------------------------------------
// engine_v2 (S2): the integral bit-sliced state with its i64 field ledger
// (src/engine_v2/backends/sparse_bitslice.rs:19-346), the default
// swap_replicas of the SpinState trait (src/engine_v2/state.rs:126-140),
// ProblemIR::greedy_coloring (src/engine_v2/ir.rs:114-139), MetropolisSweep
// (src/engine_v2/operators/metropolis_sweep.rs:40-146), GibbsColorSweep
// (src/engine_v2/operators/gibbs_color_sweep.rs:55-165) and ReplicaExchange
// (src/engine_v2/operators/replica_exchange.rs:61-110).
// ---------------------------------------------------------------------------
struct V2State {
    int64_t n = 0, r = 0, w = 0;
    std::vector<int64_t> row, col, ilin, iw;
    int64_t offset = 0;
    std::vector<uint64_t> spins;      // spins[site * w + word], bit b = replica 64 word + b
    std::vector<int64_t> fields;      // fields[site * r + rep]
    std::vector<int64_t> energies;    // [r]

    uint64_t bit(int64_t site, int64_t rep) const { return (spins[site * w + rep / 64] >> (rep % 64)) & 1; }

    // sparse_bitslice.rs:88-112
    void rebuild() {
        for (int64_t s = 0; s < n; s++)
            for (int64_t k = 0; k < r; k++) fields[s * r + k] = ilin[s];
        for (int64_t s = 0; s < n; s++)
            for (int64_t e = row[s]; e < row[s + 1]; e++)
                for (int64_t k = 0; k < r; k++)
                    if (bit(s, k)) fields[col[e] * r + k] += iw[e];
        for (int64_t k = 0; k < r; k++) energies[k] = energy_of(k);
    }
    // sparse_bitslice.rs:116-137
    int64_t energy_of(int64_t rep) const {
        int64_t l = 0, q = 0;
        for (int64_t s = 0; s < n; s++) {
            if (!bit(s, rep)) continue;
            l += ilin[s];
            for (int64_t e = row[s]; e < row[s + 1]; e++)
                if (bit(col[e], rep)) q += iw[e];
        }
        return offset + l + q / 2;
    }
    // sparse_bitslice.rs:247-255
    void delta_e_into(int64_t site, std::vector<double>& out) const {
        for (int64_t k = 0; k < r; k++) {
            const int64_t h = fields[site * r + k];
            out[k] = (double)(bit(site, k) == 0 ? h : -h);
        }
    }
    // sparse_bitslice.rs:145-174 (the dense form at :184-235 is bit-identical)
    void apply_flips(int64_t site, const std::vector<uint64_t>& mask) {
        for (int64_t q = 0; q < w; q++) {
            const uint64_t mb = mask[q];
            if (!mb) continue;
            const uint64_t sw = spins[site * w + q];
            uint64_t b = mb;
            while (b) {
                const int bp = __builtin_ctzll(b);
                const int64_t rep = q * 64 + bp;
                const uint64_t x = (sw >> bp) & 1;
                const int64_t h = fields[site * r + rep];
                energies[rep] += x == 0 ? h : -h;
                const int64_t sign = x == 0 ? 1 : -1;
                for (int64_t e = row[site]; e < row[site + 1]; e++) fields[col[e] * r + rep] += sign * iw[e];
                b &= b - 1;
            }
            spins[site * w + q] ^= mb;
        }
    }
    // state.rs:126-140
    void swap_replicas(int64_t a, int64_t b) {
        if (a == b) return;
        std::vector<uint64_t> mask(w);
        for (int64_t s = 0; s < n; s++) {
            if (bit(s, a) != bit(s, b)) {
                std::fill(mask.begin(), mask.end(), 0);
                mask[a / 64] |= 1ull << (a % 64);
                mask[b / 64] |= 1ull << (b % 64);
                apply_flips(s, mask);
            }
        }
    }
};

// ir.rs:114-139
static std::vector<uint32_t> v2_greedy_coloring(const V2State& s) {
    std::vector<uint32_t> colors(s.n, 0xFFFFFFFFu), used;
    for (int64_t i = 0; i < s.n; i++) {
        used.clear();
        for (int64_t e = s.row[i]; e < s.row[i + 1]; e++)
            if (colors[s.col[e]] != 0xFFFFFFFFu) used.push_back(colors[s.col[e]]);
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

// metropolis_sweep.rs:40-58 (order) and :95-146 (apply)
static void v2_metropolis(V2State& s, const double* temps, int nt, int64_t sweeps, ChaCha8Rng& rng,
                          int64_t& proposed, int64_t& accepted) {
    const std::vector<uint32_t> colors = v2_greedy_coloring(s);
    uint32_t ncol = 0;
    for (uint32_t c : colors) ncol = std::max(ncol, c + 1);
    std::vector<int64_t> order;
    for (uint32_t c = 0; c < ncol; c++)
        for (int64_t i = 0; i < s.n; i++)
            if (colors[i] == c) order.push_back(i);
    std::vector<double> de(s.r);
    std::vector<uint64_t> mask(s.w);
    for (int64_t sw = 0; sw < sweeps; sw++)
        for (int64_t site : order) {
            s.delta_e_into(site, de);
            std::fill(mask.begin(), mask.end(), 0);
            bool any = false;
            for (int64_t rep = 0; rep < s.r; rep++) {
                const double d = de[rep];
                const double t = temps[rep % nt];
                bool acc;
                if (d <= 0.0) {
                    (void)rng.gen_f64();
                    acc = true;
                } else {
                    const double p = t > 0.0 ? std::exp(-d / t) : 0.0;
                    const double u = rng.gen_f64();
                    acc = u < p;
                }
                proposed++;
                if (acc) {
                    mask[rep / 64] |= 1ull << (rep % 64);
                    accepted++;
                    any = true;
                }
            }
            if (any) s.apply_flips(site, mask);
        }
}

// gibbs_color_sweep.rs:55-74 (order) and :119-165 (apply): heat-bath
// resampling P(x = 1) = 1 / (1 + exp(h / t)), the greedy limit for t <= 0,
// one draw per (site, replica) in chromatic order.
static void v2_gibbs(V2State& s, const double* temps, int nt, int64_t sweeps, ChaCha8Rng& rng, int64_t& proposed,
                     int64_t& accepted) {
    const std::vector<uint32_t> colors = v2_greedy_coloring(s);
    uint32_t ncol = 0;
    for (uint32_t c : colors) ncol = std::max(ncol, c + 1);
    std::vector<int64_t> order;
    for (uint32_t c = 0; c < ncol; c++)
        for (int64_t i = 0; i < s.n; i++)
            if (colors[i] == c) order.push_back(i);
    std::vector<double> de(s.r);
    std::vector<uint64_t> mask(s.w);
    const double inf = std::numeric_limits<double>::infinity();
    for (int64_t sw = 0; sw < sweeps; sw++)
        for (int64_t site : order) {
            s.delta_e_into(site, de);
            std::fill(mask.begin(), mask.end(), 0);
            bool any = false;
            for (int64_t rep = 0; rep < s.r; rep++) {
                const bool x = s.bit(site, rep) != 0;
                const double h = x ? -de[rep] : de[rep];
                const double t = temps[rep % nt];
                const double bh = t > 0.0 ? h / t : (h > 0.0 ? inf : (h < 0.0 ? -inf : 0.0));
                const double p1 = 1.0 / (1.0 + std::exp(bh));
                const bool one = rng.gen_f64() < p1;
                proposed++;
                if (one != x) {
                    mask[rep / 64] |= 1ull << (rep % 64);
                    accepted++;
                    any = true;
                }
            }
            if (any) s.apply_flips(site, mask);
        }
}

// replica_exchange.rs:61-110
static void v2_exchange(V2State& s, const double* temps, int nt, int64_t rounds, ChaCha8Rng& rng,
                        int64_t& proposed, int64_t& accepted) {
    if (s.r < 2 || nt == 0) return;
    auto beta = [&](int64_t rep) {
        const double t = temps[rep % nt];
        return t > 0.0 ? 1.0 / t : std::numeric_limits<double>::infinity();
    };
    std::vector<double> e(s.r);
    for (int64_t round = 0; round < rounds; round++) {
        for (int64_t k = 0; k < s.r; k++) e[k] = (double)s.energies[k];
        for (int64_t k = round & 1; k + 1 < s.r; k += 2) {
            const double delta = (beta(k) - beta(k + 1)) * (e[k] - e[k + 1]);
            proposed++;
            const double u = rng.gen_f64();
            if (delta >= 0.0 || u < std::exp(delta)) {
                s.swap_replicas(k, k + 1);
                std::swap(e[k], e[k + 1]);
                accepted++;
            }
        }
    }
}

}  // namespace

extern "C" {

int or_abi_version() { return 3; }

void or_chacha8_u64(uint64_t seed, uint64_t skip, uint64_t count, uint64_t* out) {
    ChaCha8Rng r(seed);
    for (uint64_t i = 0; i < skip; i++) r.next_u64();
    for (uint64_t i = 0; i < count; i++) out[i] = r.next_u64();
}

void or_chacha8_block(const uint32_t* key, uint64_t counter, uint32_t* out) {
    chacha8_block(key, counter, out);
}

void or_xoshiro_x8_f64(uint64_t seed, uint64_t calls, double* out) {
    XoshiroX8 r(seed);
    for (uint64_t c = 0; c < calls; c++) r.next_f64x8(out + 8 * c);
}

double or_fast_exp(double x) { return fast_exp(x); }

void or_geometric_temps(double tmax, double tmin, int nt, double* out) {
    auto t = geometric_temps(tmax, tmin, nt);
    std::copy(t.begin(), t.end(), out);
}

// The seeded n=32 dense instance of tests/test_regression_golden.rs:25-57.
// Writes 992 CSR entries (rows of 31) and 32 linear terms.
void or_golden_instance(int64_t* row, int64_t* col, double* val, double* lin) {
    const int n = 32;
    ChaCha8Rng rng(0xC0FFEEULL);
    std::vector<double> upper((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) upper[(size_t)i * n + j] = rng.gen_range(-1.0, 1.0);
    int64_t k = 0;
    row[0] = 0;
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < n; j++)
            if (i != j) {
                col[k] = j;
                val[k] = i < j ? upper[(size_t)i * n + j] : upper[(size_t)j * n + i];
                k++;
            }
        row[i + 1] = k;
    }
    for (int i = 0; i < n; i++) lin[i] = rng.gen_range(-1.0, 1.0);
}

double or_total_energy(int64_t n, const double* lin, const int64_t* row, const int64_t* col,
                       const double* val, double offset, const int8_t* state) {
    Qubo m = make_qubo(n, lin, row, col, val, offset);
    return total_energy(m, state);
}

// UltimateSolver::new(tmax, tmin, sweeps, exchanges, Some(seed)) with num_temps
// = nt, then .solve(model, clamped). Writes n states; returns 0.
int or_solve(int64_t n, const double* lin, const int64_t* row, const int64_t* col,
             const double* val, double offset, double tmax, double tmin, int64_t sweeps,
             int64_t exchanges, uint64_t seed, int nt, const int64_t* clamp_idx,
             const int8_t* clamp_val, int64_t n_clamps, int threads, int8_t* state_out, int use_icm) {
    Qubo m = make_qubo(n, lin, row, col, val, offset);
    Assign cl;
    for (int64_t i = 0; i < n_clamps; i++) cl.push_back({clamp_idx[i], clamp_val[i]});
    SolverCfg cfg{tmax, tmin, sweeps, exchanges, seed, nt, threads, use_icm != 0};
    auto s = solve(m, cl, cfg);
    std::copy(s.begin(), s.end(), state_out);
    return 0;
}

// full_presolve: writes derived (idx, val) fixings; returns their count.
int64_t or_full_presolve(int64_t n, const double* lin, const int64_t* row, const int64_t* col,
                         const double* val, const int64_t* clamp_idx, const int8_t* clamp_val,
                         int64_t n_clamps, int64_t* out_idx, int8_t* out_val) {
    Qubo m = make_qubo(n, lin, row, col, val, 0.0);
    Assign cl;
    for (int64_t i = 0; i < n_clamps; i++) cl.push_back({clamp_idx[i], clamp_val[i]});
    auto d = full_presolve(m, cl);
    for (size_t i = 0; i < d.size(); i++) {
        out_idx[i] = d[i].first;
        out_val[i] = d[i].second;
    }
    return (int64_t)d.size();
}

double or_path_relink(int64_t n, const double* lin, const int64_t* row, const int64_t* col, const double* val,
                      double offset, const uint64_t* words, int64_t cells, const uint8_t* clamped, int8_t* state) {
    Qubo m = make_qubo(n, lin, row, col, val, offset);
    std::vector<uint8_t> cl(clamped, clamped + n);
    std::vector<int8_t> cur(state, state + n);
    double be = 0.0;
    const std::vector<int8_t> best = path_relink_finish(m, std::vector<uint64_t>(words, words + cells * n), cells, cl,
                                                        cur, total_energy(m, state), be);
    std::copy(best.begin(), best.end(), state);
    return be;
}

// Warm-start words of `cells` cells (ultimate.rs:256-263) from
// seed_from_u64(seed) after `skip` draws; returns the position after them.
uint64_t or_warm_start_words(uint64_t seed, uint64_t skip, const double* probs, const uint8_t* clamped,
                             const int8_t* clamp_val, int64_t n, int cells, uint64_t* words_out) {
    ChaCha8Rng rng(seed);
    for (uint64_t k = 0; k < skip; k++) rng.next_u64();
    Field f(n, cells, 1);
    std::vector<uint8_t> cl(clamped, clamped + n);
    std::vector<int8_t> cv(clamp_val, clamp_val + n);
    init_field(f, cl, cv, rng, probs);
    pack_words(f, words_out);
    return rng.draws;
}

double or_two_opt(int64_t n, const double* lin, const int64_t* row, const int64_t* col, const double* val,
                  double offset, int8_t* state, const uint8_t* clamped) {
    Qubo m = make_qubo(n, lin, row, col, val, offset);
    std::vector<uint8_t> cl(clamped, clamped + n);
    return two_opt(m, state, cl);
}

double or_one_opt(int64_t n, const double* lin, const int64_t* row, const int64_t* col,
                  const double* val, int8_t* state, const uint8_t* clamped) {
    Qubo m = make_qubo(n, lin, row, col, val, 0.0);
    std::vector<uint8_t> cl(clamped, clamped + n);
    return one_opt(m, state, cl);
}

// The PT/SA step loop of ultimate.rs:248-336 under a caller-given per-step
// temperature schedule temps[step][nt] (a constant ladder repeated = the
// reference's PT run; one temperature per step = an SA schedule).
//   init_words: if non-null, [nt][n] u64 spin words used instead of the random
//               init (the master stream then draws nothing for the init).
//   exchange_interval: phase 2 runs after every k-th step (k = 1 is the reference).
//   incumbent_every: if > 0, update_incumbent after every that many steps.
//   icm_every: if > 0, icm_sweep after every that many steps (before the
//              incumbent, as the PT loop orders them).
// Outputs: words [nt][n], energies [nt][64] (tracked), swap attempts/accepts
// [nt-1], draws = master-stream u64 position, base_seeds [steps] (optional),
// incumbent energy and state (optional).
int or_run_schedule(int64_t n, const double* lin, const int64_t* row, const int64_t* col,
                    const double* val, int nt, const double* temps, int64_t steps, uint64_t seed,
                    const uint64_t* init_words, const uint8_t* clamped, const int8_t* clamp_val,
                    int64_t exchange_interval, int collect_stats, int64_t incumbent_every,
                    int threads, uint64_t* words_out, double* energies_out, uint64_t* attempts_out,
                    uint64_t* accepts_out, uint64_t* draws_out, uint64_t* base_seeds_out,
                    double* inc_energy_out, int8_t* inc_state_out, int64_t icm_every) {
    Qubo m = make_qubo(n, lin, row, col, val, 0.0);
    std::vector<uint8_t> isc(n, 0);
    std::vector<int8_t> cv(n, 0);
    if (clamped) {
        for (int64_t i = 0; i < n; i++) {
            isc[i] = clamped[i];
            cv[i] = clamp_val ? clamp_val[i] : 0;
        }
    }
    ChaCha8Rng rng(seed);
    Field f(n, nt, 1);
    if (init_words) unpack_words(f, init_words);
    else init_field(f, isc, cv, rng);
    for (int t = 0; t < nt; t++) replica_energies(m, f.cell(t), f.energies[t].data());
    StepScratch sc;
    sc.attempts.assign(std::max(nt - 1, 0), 0);
    sc.accepts.assign(std::max(nt - 1, 0), 0);
    if (exchange_interval < 1) exchange_interval = 1;
    double inc_e = std::numeric_limits<double>::infinity();
    std::vector<int8_t> inc(n, 0), buf(n, 0);
    for (int64_t s = 0; s < steps; s++) {
        bool ex = ((s + 1) % exchange_interval) == 0;
        step(f, m, temps + (size_t)s * nt, isc, sc, rng, ex, collect_stats != 0, threads,
             base_seeds_out ? base_seeds_out + s : nullptr);
        if ((uint64_t)(s + 1) % 1000 == 0)
            for (int t = 0; t < nt; t++) replica_energies(m, f.cell(t), f.energies[t].data());
        if (icm_every > 0 && (s + 1) % icm_every == 0) icm_sweep(f, m, rng);
        if (incumbent_every > 0 && (s + 1) % incumbent_every == 0) update_incumbent(m, f, inc_e, inc, buf);
    }
    if (words_out) pack_words(f, words_out);
    if (energies_out)
        for (int t = 0; t < nt; t++)
            for (int r = 0; r < NR; r++) energies_out[(size_t)t * NR + r] = f.energies[t][r];
    if (attempts_out)
        for (int t = 0; t + 1 < nt; t++) {
            attempts_out[t] = sc.attempts[t];
            accepts_out[t] = sc.accepts[t];
        }
    if (draws_out) *draws_out = rng.draws;
    if (inc_energy_out) *inc_energy_out = inc_e;
    if (inc_state_out) std::copy(inc.begin(), inc.end(), inc_state_out);
    return 0;
}

// Recomputes per-replica energies of spin words [cells][n] (engine.rs:333-418).
void or_replica_energies(int64_t n, const double* lin, const int64_t* row, const int64_t* col,
                         const double* val, int cells, const uint64_t* words, double* out) {
    Qubo m = make_qubo(n, lin, row, col, val, 0.0);
    Field f(n, cells, 1);
    unpack_words(f, words);
    for (int c = 0; c < cells; c++) replica_energies(m, f.cell(c), out + (size_t)c * NR);
}

// Many independent single-cell SA runs in parallel over instances (the CPU
// baseline for the batched configuration). Instance i has its CSR at
// row_ptrs[i] etc. All share the temps schedule temps[steps]. Words out at
// words_out + word_off[i]; energies at energies_out + 64*i.
int or_run_sa_batch(int64_t count, const int64_t* ns, const double* const* lins,
                    const int64_t* const* rows, const int64_t* const* cols,
                    const double* const* vals, const uint64_t* seeds, const double* temps,
                    int64_t steps, int threads, uint64_t* words_out, const int64_t* word_off,
                    double* energies_out) {
    parallel_for((int)count, threads, [&](int i) {
        Qubo m = make_qubo(ns[i], lins[i], rows[i], cols[i], vals[i], 0.0);
        std::vector<uint8_t> isc(m.n, 0);
        std::vector<int8_t> cv(m.n, 0);
        ChaCha8Rng rng(seeds[i]);
        Field f(m.n, 1, 1);
        init_field(f, isc, cv, rng);
        replica_energies(m, f.cell(0), f.energies[0].data());
        StepScratch sc;
        for (int64_t s = 0; s < steps; s++) {
            step(f, m, temps + s, isc, sc, rng, true, false, 1, nullptr);
            if ((uint64_t)(s + 1) % 1000 == 0) replica_energies(m, f.cell(0), f.energies[0].data());
        }
        if (words_out) pack_words(f, words_out + word_off[i]);
        if (energies_out)
            for (int r = 0; r < NR; r++) energies_out[(size_t)i * NR + r] = f.energies[0][r];
    });
    return 0;
}

// UltimateSolver with num_temps = nt, num_pops = pops >= 2 and the PA knobs,
// run through solve_with_pa_diagnostics(model, clamped). Outputs: final
// words [nt * pops][n] (cell t + nt p), tracked energies [nt * pops][64],
// master-stream position, tuned alphas [nt], ESS per stage [exchanges - 1],
// family (rho, count) per resampling event, free energy, resampling events,
// the best member before 1-opt, the incumbent energy and the solution.
int or_pa_run(int64_t n, const double* lin, const int64_t* row, const int64_t* col, const double* val,
              double offset, double tmax, double tmin, int64_t sweeps, int64_t exchanges, uint64_t seed, int nt,
              int pops, double ess_threshold, int64_t tuning_iters, int64_t tuning_steps, int64_t relax,
              int ladder_mode, int use_icm, const uint8_t* clamped, const int8_t* clamp_val, int threads,
              uint64_t* words_out,
              double* energies_out, uint64_t* draws_out, double* alphas_out, double* ess_out, int64_t* n_ess,
              double* rho_out, int64_t* fam_out, int64_t* n_res, double* free_energy_out, int8_t* best_pre_out,
              double* incumbent_out, int8_t* state_out) {
    Qubo m = make_qubo(n, lin, row, col, val, offset);
    std::vector<uint8_t> cl(n, 0);
    std::vector<int8_t> cv(n, 0);
    for (int64_t i = 0; i < n; i++) {
        cl[i] = clamped ? clamped[i] : 0;
        cv[i] = clamp_val ? clamp_val[i] : 0;
    }
    PaCfg cfg{tmax, tmin, sweeps, exchanges, seed, nt, pops, ess_threshold, tuning_iters, tuning_steps, relax, threads,
              ladder_mode, use_icm != 0};
    ChaCha8Rng rng(seed);
    PaOut o;
    Field f = pa_run(m, cl, cv, cfg, o, rng);
    pack_words(f, words_out);
    for (size_t c = 0; c < f.energies.size(); c++)
        for (int r = 0; r < NR; r++) energies_out[c * NR + r] = f.energies[c][r];
    *draws_out = rng.draws;
    std::copy(o.alphas.begin(), o.alphas.end(), alphas_out);
    std::copy(o.ess.begin(), o.ess.end(), ess_out);
    *n_ess = (int64_t)o.ess.size();
    std::copy(o.rho.begin(), o.rho.end(), rho_out);
    std::copy(o.families.begin(), o.families.end(), fam_out);
    *n_res = o.resamples;
    *free_energy_out = o.free_energy;
    std::copy(o.best_pre.begin(), o.best_pre.end(), best_pre_out);
    *incumbent_out = o.incumbent_e;
    std::copy(o.best.begin(), o.best.end(), state_out);
    return 0;
}

// population_annealing.rs primitives for the host tests.
void or_pa_normalized_weights(const double* lw, int64_t r, double* out) {
    const auto w = pa_normalized_weights(std::vector<double>(lw, lw + r));
    std::copy(w.begin(), w.end(), out);
}
void or_pa_systematic_resample(const double* w, int64_t r, double u, int64_t* counts) {
    const auto c = pa_systematic_resample(std::vector<double>(w, w + r), u);
    std::copy(c.begin(), c.end(), counts);
}
void or_pa_feedback_alphas(const double* alphas, const double* flow, int64_t nt, double damping, double* out) {
    const auto a = pa_feedback_alphas(std::vector<double>(alphas, alphas + nt), std::vector<double>(flow, flow + nt),
                                      damping);
    std::copy(a.begin(), a.end(), out);
}
// gen_range(0..=hi[i]) in sequence on ChaCha8Rng::seed_from_u64(seed).
void or_gen_index_inclusive(uint64_t seed, const uint64_t* hi, int64_t count, uint64_t* out, uint64_t* draws) {
    ChaCha8Rng rng(seed);
    for (int64_t i = 0; i < count; i++) out[i] = gen_index_inclusive(rng, hi[i]);
    *draws = rng.draws;
}

// A program of S2 operator applications on one state with one master stream
// (ChaCha8Rng::seed_from_u64(seed) after skip_draws draws): op i is
// MetropolisSweep (kinds[i] == 0) for counts[i] sweeps, ReplicaExchange
// (kinds[i] == 1) for counts[i] rounds or GibbsColorSweep (kinds[i] == 2) for
// counts[i] sweeps, all at temps[nt]. Outputs the planes
// [n * ceil(r/64)], the ledger energies [r], (proposed, accepted) per op, the
// largest ledger drift against a rebuild and the stream position.
int or_v2_program(int64_t n, const double* lin, const int64_t* row, const int64_t* col, const double* val,
                  double offset, int64_t r, const uint8_t* init, uint64_t seed, uint64_t skip_draws, int64_t nops,
                  const int32_t* kinds, const int64_t* counts, const double* temps, int32_t nt,
                  uint64_t* planes_out, double* energies_out, int64_t* stats_out, double* drift_out,
                  uint64_t* draws_out) {
    V2State s;
    s.n = n;
    s.r = r;
    s.w = (r + 63) / 64;
    s.row.assign(row, row + n + 1);
    s.col.assign(col, col + row[n]);
    s.offset = (int64_t)offset;
    s.ilin.resize(n);
    for (int64_t i = 0; i < n; i++) s.ilin[i] = (int64_t)lin[i];
    s.iw.resize(row[n]);
    for (int64_t e = 0; e < row[n]; e++) s.iw[e] = (int64_t)val[e];
    s.spins.assign(n * s.w, 0);
    for (int64_t i = 0; i < n; i++)
        if (init[i] & 1)
            for (int64_t q = 0; q < s.w; q++) {
                const int64_t valid = std::min<int64_t>(r - 64 * q, 64);
                s.spins[i * s.w + q] = valid == 64 ? ~0ull : ((1ull << valid) - 1);
            }
    s.fields.assign(n * r, 0);
    s.energies.assign(r, 0);
    s.rebuild();
    ChaCha8Rng rng(seed);
    for (uint64_t k = 0; k < skip_draws; k++) rng.next_u64();
    for (int64_t i = 0; i < nops; i++) {
        int64_t p = 0, a = 0;
        if (kinds[i] == 0) v2_metropolis(s, temps, nt, counts[i], rng, p, a);
        else if (kinds[i] == 1) v2_exchange(s, temps, nt, counts[i], rng, p, a);
        else v2_gibbs(s, temps, nt, counts[i], rng, p, a);
        stats_out[2 * i] = p;
        stats_out[2 * i + 1] = a;
    }
    std::copy(s.spins.begin(), s.spins.end(), planes_out);
    for (int64_t k = 0; k < r; k++) energies_out[k] = (double)s.energies[k];
    // audit (sparse_bitslice.rs:317-346)
    V2State fresh = s;
    fresh.rebuild();
    int64_t drift = 0;
    for (size_t i = 0; i < s.fields.size(); i++) drift = std::max<int64_t>(drift, std::llabs(s.fields[i] - fresh.fields[i]));
    for (int64_t k = 0; k < r; k++) drift = std::max<int64_t>(drift, std::llabs(s.energies[k] - fresh.energies[k]));
    *drift_out = (double)drift;
    *draws_out = rng.draws;
    return 0;
}

}  // extern "C"
