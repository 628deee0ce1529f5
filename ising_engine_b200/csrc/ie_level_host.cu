// Host-side builders of the level kernel's data (see ie_level_host.h).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "../../include/ising_b200.h"
#include "ie_level_host.h"

namespace ie {

namespace {

// ---------------------------------------------------------------------------
// Xoshiro256 state transition over GF(2) (engine.rs:115-121) on the host.
// ---------------------------------------------------------------------------
struct Xo4 {
    uint64_t s[4];
    void step() {
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = (s[3] << 45) | (s[3] >> 19);
    }
};

// Polynomials over GF(2) of degree < 256 as 4 words (bit i = x^i); the
// modulus P(x) = x^256 + low(x).
struct Poly {
    uint64_t w[4] = {0, 0, 0, 0};
    bool bit(int i) const { return (w[i >> 6] >> (i & 63)) & 1u; }
};

// a * b mod P by shift-and-add: 512-bit product, then reduction from the top
// (x^k = x^(k - 256) low(x) for k >= 256).
Poly mulmod(const Poly& a, const Poly& b, const Poly& low) {
    uint64_t r[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 256; i++) {
        if (!a.bit(i)) continue;
        const int ws = i >> 6, bs = i & 63;
        for (int k = 0; k < 4; k++) {
            r[k + ws] ^= b.w[k] << bs;
            if (bs) r[k + ws + 1] ^= b.w[k] >> (64 - bs);
        }
    }
    for (int k = 511; k >= 256; k--) {
        if (!((r[k >> 6] >> (k & 63)) & 1u)) continue;
        r[k >> 6] ^= 1ull << (k & 63);
        const int sh = k - 256, ws = sh >> 6, bs = sh & 63;
        for (int j = 0; j < 4; j++) {
            r[j + ws] ^= low.w[j] << bs;
            if (bs) r[j + ws + 1] ^= low.w[j] >> (64 - bs);
        }
    }
    Poly out;
    for (int k = 0; k < 4; k++) out.w[k] = r[k];
    return out;
}

std::mutex g_poly_mu;
bool g_poly_ok = false;
Poly g_low;

void jump_state(const Poly& r, Xo4& x) {
    Xo4 acc{{0, 0, 0, 0}};
    for (int i = 0; i < 256; i++) {
        if (r.bit(i))
            for (int k = 0; k < 4; k++) acc.s[k] ^= x.s[k];
        x.step();
    }
    x = acc;
}

Poly xpow(uint64_t e, const Poly& low) {
    Poly result;
    result.w[0] = 1;
    Poly base;
    base.w[0] = 2;  // x
    while (e) {
        if (e & 1) result = mulmod(result, base, low);
        base = mulmod(base, base, low);
        e >>= 1;
    }
    return result;
}

// The characteristic polynomial of the transition, as the minimal polynomial
// (Berlekamp-Massey) of one state bit's sequence; the transition has full
// period, so it has degree 256. Checked by jumps against plain stepping.
bool derive_poly() {
    if (g_poly_ok) return true;
    const int N = 1024;
    std::vector<uint8_t> seq(N);
    Xo4 x{{0x9e3779b97f4a7c15ULL, 0xbf58476d1ce4e5b9ULL, 0x94d049bb133111ebULL, 0x2545f4914f6cdd1dULL}};
    for (int i = 0; i < N; i++) {
        seq[i] = (uint8_t)(x.s[0] & 1u);
        x.step();
    }
    // Berlekamp-Massey over GF(2): C(x) = 1 + c_1 x + ... + c_L x^L with
    // s_n = sum c_i s_{n-i}
    std::vector<uint8_t> C(N + 1, 0), B(N + 1, 0), Tmp;
    C[0] = B[0] = 1;
    int L = 0, m = 1;
    for (int n = 0; n < N; n++) {
        uint8_t d = seq[n];
        for (int i = 1; i <= L; i++) d ^= (uint8_t)(C[i] & seq[n - i]);
        if (!d) {
            m++;
            continue;
        }
        Tmp = C;
        for (int i = 0; i + m <= N; i++) C[i + m] ^= B[i];
        if (2 * L <= n) {
            L = n + 1 - L;
            B = Tmp;
            m = 1;
        } else {
            m++;
        }
    }
    if (L != 256) return false;
    // P(x) = x^256 + sum_{i=1..256} c_i x^(256 - i)
    Poly low;
    for (int i = 1; i <= 256; i++)
        if (C[i]) low.w[(256 - i) >> 6] |= 1ull << ((256 - i) & 63);
    for (uint64_t D : {5ull, 1000ull, 4096ull}) {
        Xo4 a{{0x0123456789abcdefULL, 0xfedcba9876543210ULL, 0x0f1e2d3c4b5a6978ULL, 0x8796a5b4c3d2e1f0ULL}};
        Xo4 b = a;
        jump_state(xpow(D, low), a);
        for (uint64_t i = 0; i < D; i++) b.step();
        if (std::memcmp(a.s, b.s, sizeof(a.s)) != 0) return false;
    }
    g_low = low;
    g_poly_ok = true;
    return true;
}

}  // namespace

bool xoshiro_jump_poly(uint64_t steps, uint64_t out[4]) {
    std::lock_guard<std::mutex> lk(g_poly_mu);
    if (!derive_poly()) return false;
    const Poly r = xpow(steps, g_low);
    std::memcpy(out, r.w, sizeof(r.w));
    return true;
}

bool xoshiro_segment_polys(uint32_t count, std::vector<uint64_t>& table) {
    std::lock_guard<std::mutex> lk(g_poly_mu);
    if (!derive_poly()) return false;
    table.assign(4ull * std::max<uint32_t>(count, 1), 0);
    Poly cur;
    cur.w[0] = 1;
    const Poly step = xpow(8ull * kLvlSeg, g_low);
    for (uint32_t j = 0; j < count; j++) {
        std::memcpy(&table[4ull * j], cur.w, sizeof(cur.w));
        cur = mulmod(cur, step, g_low);
    }
    return true;
}

void level_records(const LvlSource& s, std::vector<uint32_t>& recs, uint32_t* off16) {
    for (uint32_t v = 0; v < s.n; v++) {
        off16[v] = (uint32_t)(recs.size() / 4);
        const uint32_t beg = s.rows[v], end = s.rows[v + 1];
        const uint32_t deg = end - beg, deg4 = (deg + 3u) & ~3u;
        const uint32_t hdr = deg | (s.clampf && s.clampf[v] ? 0x80000000u : 0u);
        if (s.mode == kModeInt) {
            recs.push_back(hdr);
            recs.push_back((uint32_t)s.linp[v]);
            recs.push_back((uint32_t)(int32_t)s.lin[v]);
            recs.push_back(0);
            for (uint32_t e = 0; e < deg4; e++) recs.push_back(e < deg ? s.ents[beg + e] : 0u);
        } else {
            uint32_t w2[2];
            recs.push_back(hdr);
            recs.push_back(0);
            std::memcpy(w2, &s.lin[v], 8);
            recs.push_back(w2[0]);
            recs.push_back(w2[1]);
            for (uint32_t e = 0; e < deg4; e++) recs.push_back(e < deg ? s.cols[beg + e] : 0u);
            for (uint32_t e = 0; e < deg4; e++) {
                const double w = e < deg ? s.vals[beg + e] : 0.0;
                std::memcpy(w2, &w, 8);
                recs.push_back(w2[0]);
                recs.push_back(w2[1]);
            }
        }
    }
}

void site_levels(const LvlSource& s, std::vector<uint32_t>& sites, std::vector<uint32_t>& off) {
    std::vector<uint32_t> lvl(s.n, 0);
    uint32_t depth = 0;
    size_t live = 0;
    for (uint32_t v = 0; v < s.n; v++) {
        if (s.clampf && s.clampf[v]) continue;
        uint32_t l = 0;
        for (uint32_t e = s.rows[v]; e < s.rows[v + 1]; e++) {
            const uint32_t u = s.cols[e];
            if (u < v && !(s.clampf && s.clampf[u])) l = std::max(l, lvl[u] + 1);
        }
        lvl[v] = l;
        depth = std::max(depth, l + 1);
        live++;
    }
    off.assign(depth + 1, 0);
    for (uint32_t v = 0; v < s.n; v++)
        if (!(s.clampf && s.clampf[v])) off[lvl[v] + 1]++;
    for (uint32_t l = 0; l < depth; l++) off[l + 1] += off[l];
    sites.assign(live, 0);
    std::vector<uint32_t> pos(off.begin(), off.end() - 1);
    for (uint32_t v = 0; v < s.n; v++)
        if (!(s.clampf && s.clampf[v])) sites[pos[lvl[v]]++] = v;
}

void build_level_items(const std::vector<InstDesc>& D, const std::vector<uint64_t>& nnz_of,
                       const std::vector<uint32_t>& dmax_of, const std::vector<uint32_t>& pmj_of,
                       const std::vector<std::vector<uint32_t>>& lv_sites,
                       const std::vector<std::vector<uint32_t>>& lv_off, const std::vector<uint32_t>& recoff,
                       const std::vector<uint32_t>& mem,
                       bool gsp, uint32_t cap, uint32_t max_mem, uint32_t split, LvlHost& out,
                       std::vector<uint32_t>& order, double& longest) {
    if (!gsp || split < 1) split = 1;
    std::vector<uint32_t> m = mem;
    std::stable_sort(m.begin(), m.end(), [&](uint32_t a, uint32_t b) { return D[a].n > D[b].n; });
    std::vector<std::vector<uint32_t>> groups;
    if (gsp) {
        for (uint32_t i : m) groups.push_back({i});
    } else {
        std::vector<uint32_t> cur;
        uint64_t sites = 0;
        for (uint32_t i : m) {
            if (!cur.empty() && (sites + D[i].n > cap || cur.size() >= max_mem)) {
                groups.push_back(cur);
                cur.clear();
                sites = 0;
            }
            cur.push_back(i);
            sites += D[i].n;
        }
        if (!cur.empty()) groups.push_back(cur);
    }
    std::vector<std::pair<double, uint32_t>> work;
    for (const auto& g : groups) {
        LvlItem it{};
        it.mem0 = (uint32_t)out.members.size();
        it.nmem = (uint32_t)g.size();
        it.ent0 = (uint32_t)out.entries.size();
        it.lvl0 = (uint32_t)out.lvloff.size();
        it.seg0 = (uint32_t)out.segs.size();
        it.gsp = gsp ? 1u : 0u;
        it.split = split;
        uint32_t flat = 0, depth = 0;
        double w = 0;
        for (uint32_t slot = 0; slot < g.size(); slot++) {
            const InstDesc& d = D[g[slot]];
            out.members.push_back(LvlMember{g[slot], flat, pmj_of[g[slot]]});
            const uint32_t ns = (d.n + kLvlSeg - 1) / kLvlSeg;
            for (uint32_t sg = 0; sg < ns; sg++) out.segs.push_back(slot << 24 | sg);
            out.max_segs = std::max(out.max_segs, ns);
            it.nseg += ns;
            it.H = std::max(it.H, d.H);
            it.dmax = std::max(it.dmax, dmax_of[g[slot]]);
            depth = std::max(depth, (uint32_t)lv_off[d.owner].size() - 1);
            const double deg = d.n ? (double)nnz_of[g[slot]] / d.n : 0.0;
            w += (double)d.n * (deg + 12.0) * (d.mode == kModeF64 ? 2.5 : 1.0);
            flat += d.n;
        }
        it.sites = flat;
        it.nlvl = depth;
        for (uint32_t l = 0; l < depth; l++)
            for (uint32_t r = 0; r < split; r++) {
                out.lvloff.push_back((uint32_t)(out.entries.size() - it.ent0));
                for (uint32_t slot = 0; slot < g.size(); slot++) {
                    const InstDesc& d = D[g[slot]];
                    const std::vector<uint32_t>& off = lv_off[d.owner];
                    if (l + 1 >= off.size()) continue;
                    const std::vector<uint32_t>& st = lv_sites[d.owner];
                    const uint32_t f0 = out.members[it.mem0 + slot].flat;
                    for (uint32_t q = off[l]; q < off[l + 1]; q++)
                        if (split == 1 || (st[q] / kLvlSeg) % split == r)
                            out.entries.push_back(
                                LvlEntry{slot << kLvlFlatBits | (f0 + st[q]), recoff[d.site + st[q]]});
                }
            }
        out.lvloff.push_back((uint32_t)(out.entries.size() - it.ent0));
        // per-level barrier and latency, in site-work units
        w += (double)depth * 400.0;
        work.push_back({w, (uint32_t)out.items.size()});
        longest = std::max(longest, w);
        out.items.push_back(it);
    }
    std::stable_sort(work.begin(), work.end(),
                     [](const std::pair<double, uint32_t>& a, const std::pair<double, uint32_t>& b) {
                         return a.first > b.first;
                     });
    order.clear();
    for (auto& p : work) order.push_back(p.second);
}

}  // namespace ie

extern "C" ie_status ie_xoshiro_jump_poly(uint64_t steps, uint64_t* out) {
    if (!out) return IE_ERR_INVALID;
    return ie::xoshiro_jump_poly(steps, out) ? IE_OK : IE_ERR_DEVICE;
}
