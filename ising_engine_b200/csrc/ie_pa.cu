// Population-annealing primitives on the host (src/solver/population_annealing.rs:
// normalized_weights :51-56, effective_sample_size :60-63,
// free_energy_increment :70-78, family_entropy :84-101, systematic_resample
// :106-127, adapt_spacings :141-152, feedback_optimized_alphas :172-232, the
// shuffle of apply_resample :240-260)
// and the master-stream draws they take: rand 0.8.5's gen_range on
// rand_chacha 0.3.1's ChaCha8Rng, addressed by draw index like the device's
// chacha8_draw.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <vector>

#include "ie_host.h"

namespace ie {

namespace {

inline uint32_t rl(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }

inline void quarter(uint32_t* x, int a, int b, int c, int d) {
    x[a] += x[b]; x[d] = rl(x[d] ^ x[a], 16);
    x[c] += x[d]; x[b] = rl(x[b] ^ x[c], 12);
    x[a] += x[b]; x[d] = rl(x[d] ^ x[a], 8);
    x[c] += x[d]; x[b] = rl(x[b] ^ x[c], 7);
}

}  // namespace

// Draw k of the stream: words (2(k % 8), 2(k % 8) + 1) of block k / 8 (8
// rounds, 64-bit block counter in words 12-13, stream id 0), low word first.
uint64_t chacha8_draw_host(const uint32_t key[8], uint64_t k) {
    const uint64_t blk = k >> 3;
    uint32_t in[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                       key[4], key[5], key[6], key[7], (uint32_t)blk, (uint32_t)(blk >> 32), 0u, 0u};
    uint32_t x[16];
    std::copy(in, in + 16, x);
    for (int i = 0; i < 4; i++) {
        quarter(x, 0, 4, 8, 12); quarter(x, 1, 5, 9, 13); quarter(x, 2, 6, 10, 14); quarter(x, 3, 7, 11, 15);
        quarter(x, 0, 5, 10, 15); quarter(x, 1, 6, 11, 12); quarter(x, 2, 7, 8, 13); quarter(x, 3, 4, 9, 14);
    }
    const int w = (int)(k & 7) * 2;
    return (uint64_t)(x[w] + in[w]) | ((uint64_t)(x[w + 1] + in[w + 1]) << 32);
}

uint64_t HostStream::next_u64() { return chacha8_draw_host(key, pos++); }

// rand 0.8.5 UniformFloat<f64>::sample_single(0.0, 1.0): the 52 high bits of
// a draw as the mantissa of a number in [1, 2), minus 1; times the scale 1
// plus 0 it stays below 1, so one draw always suffices.
double HostStream::unit_f64() {
    const uint64_t bits = (next_u64() >> 12) | 0x3FF0000000000000ull;
    double v;
    std::memcpy(&v, &bits, sizeof v);
    return (v - 1.0) * 1.0 + 0.0;
}

// rand 0.8.5 UniformInt<usize>::sample_single_inclusive(0, hi) on a 64-bit
// target: with range = hi + 1 and zone = (range << leading_zeros(range)) - 1,
// a draw v is accepted when the low 64 bits of v * range are <= zone, and the
// high 64 bits are the result.
uint64_t HostStream::index_inclusive(uint64_t hi) {
    const uint64_t range = hi + 1;
    if (range == 0) return next_u64();
    const uint64_t zone = (range << __builtin_clzll(range)) - 1;
    for (;;) {
        const unsigned __int128 prod = (unsigned __int128)next_u64() * range;
        if ((uint64_t)prod <= zone) return (uint64_t)(prod >> 64);
    }
}

// UltimateSolver's warm start (ultimate.rs:256-263, the same policy for every
// field geometry at :481-518): for cell c (cell-major) and site v, a clamped
// site takes its value in every replica and draws nothing; otherwise replica
// r is one when its gen_range(0.0..1.0) draw is below probs[v], 64 draws per
// site in replica order. Words in the reference layout (bit r = replica r).
void warm_start_words(HostStream& rng, const double* probs, const uint8_t* clampf, const int8_t* clampv, uint64_t n,
                      uint64_t cells, uint64_t* words) {
    for (uint64_t c = 0; c < cells; c++)
        for (uint64_t v = 0; v < n; v++) {
            uint64_t w = 0;
            if (clampf && clampf[v]) {
                w = clampv && clampv[v] == 1 ? ~0ull : 0ull;
            } else {
                for (int r = 0; r < 64; r++)
                    if (rng.unit_f64() < probs[v]) w |= 1ull << r;
            }
            words[c * n + v] = w;
        }
}

namespace pa {

std::vector<double> normalized_weights(const double* lw, size_t r) {
    double m = -std::numeric_limits<double>::infinity();
    for (size_t i = 0; i < r; i++) m = std::max(m, lw[i]);
    std::vector<double> w(r);
    double z = 0.0;
    for (size_t i = 0; i < r; i++) {
        w[i] = std::exp(lw[i] - m);
        z += w[i];
    }
    for (double& x : w) x = x / z;
    return w;
}

double effective_sample_size(const double* w, size_t r) {
    double s2 = 0.0;
    for (size_t i = 0; i < r; i++) s2 += w[i] * w[i];
    return 1.0 / s2;
}

double free_energy_increment(const double* lw, size_t r) {
    double m = -std::numeric_limits<double>::infinity();
    for (size_t i = 0; i < r; i++) m = std::max(m, lw[i]);
    if (!std::isfinite(m)) return 0.0;
    double s = 0.0;
    for (size_t i = 0; i < r; i++) s += std::exp(lw[i] - m);
    return m + std::log(s) - std::log((double)r);
}

void family_entropy(const uint64_t* ids, size_t r, double& rho, uint64_t& families) {
    rho = 0.0;
    families = 0;
    if (r == 0) return;
    std::map<uint64_t, uint64_t> sizes;
    for (size_t i = 0; i < r; i++) sizes[ids[i]]++;
    double s = 0.0;
    for (const auto& kv : sizes) {
        const double frac = (double)kv.second / (double)r;
        s += frac * frac;
    }
    rho = s * (double)r;
    families = sizes.size();
}

std::vector<uint64_t> systematic_resample(const double* w, size_t r, double u) {
    std::vector<uint64_t> counts(r, 0);
    double cum = 0.0;
    size_t j = 0;
    for (size_t i = 0; i < r; i++) {
        cum += w[i];
        for (; j < r && ((double)j + u) / (double)r < cum; j++) counts[i]++;
    }
    if (j < r) counts[r - 1] += r - j;
    return counts;
}

std::vector<double> adapt_spacings(const double* d, const double* acc, size_t k) {
    std::vector<double> out(k);
    double old_total = 0.0, new_total = 0.0;
    for (size_t i = 0; i < k; i++) out[i] = d[i] * std::sqrt(std::max(acc[i], 0.02));
    for (size_t i = 0; i < k; i++) old_total += d[i];
    for (size_t i = 0; i < k; i++) new_total += out[i];
    for (double& x : out) x = x * old_total / new_total;
    return out;
}

std::vector<double> feedback_optimized_alphas(const std::vector<double>& alphas, const std::vector<double>& flow,
                                              double damping) {
    const size_t nt = alphas.size();
    if (nt < 3) return alphas;
    constexpr double kEps = 1e-6;
    std::vector<double> f(flow);  // cumulative max from the hot end
    for (size_t k = 1; k < nt; k++) f[k] = f[k] < f[k - 1] ? f[k - 1] : f[k];
    std::vector<double> mass(nt - 1), cum(nt, 0.0);
    double total = 0.0;
    for (size_t k = 0; k + 1 < nt; k++) {
        mass[k] = std::sqrt(std::max(std::fabs(f[k + 1] - f[k]), kEps) *
                            std::max(std::fabs(alphas[k + 1] - alphas[k]), kEps));
        total += mass[k];
    }
    if (total <= 0.0 || !std::isfinite(total)) return alphas;
    for (size_t k = 0; k + 1 < nt; k++) cum[k + 1] = cum[k] + mass[k];
    std::vector<double> out(nt, 0.0);
    out[0] = alphas[0];
    out[nt - 1] = alphas[nt - 1];
    size_t k = 0;
    for (size_t i = 1; i + 1 < nt; i++) {
        const double target = (double)i / (double)(nt - 1) * total;
        k = 0;
        while (k < nt - 2 && cum[k + 1] < target) k++;
        const double frac = mass[k] > 0.0 ? (target - cum[k]) / mass[k] : 0.0;
        out[i] = damping * (alphas[k] + frac * (alphas[k + 1] - alphas[k])) + (1.0 - damping) * alphas[i];
    }
    for (size_t i = 1; i < nt; i++)
        if (out[i] <= out[i - 1]) out[i] = out[i - 1] + kEps;
    const double base = out[0], span = out[nt - 1] - out[0], old_span = alphas[nt - 1] - alphas[0];
    if (span > 0.0)
        for (double& a : out) a = alphas[0] + (a - base) / span * old_span;
    return out;
}

std::vector<uint32_t> shuffled_parents(const std::vector<uint64_t>& counts, HostStream& rng) {
    std::vector<uint32_t> parents;
    parents.reserve(counts.size());
    for (size_t i = 0; i < counts.size(); i++) parents.insert(parents.end(), counts[i], (uint32_t)i);
    for (size_t k = parents.size(); k-- > 1;) std::swap(parents[k], parents[rng.index_inclusive(k)]);
    return parents;
}

}  // namespace pa
}  // namespace ie

using namespace ie;

extern "C" {

ie_status ie_warm_start_words(uint64_t seed, uint64_t draw_offset, const double* probs, const uint8_t* is_clamped,
                              const int8_t* clamp_val, uint64_t n, uint64_t cells, uint64_t* words, uint64_t* draws) {
    if ((n && (!probs || !words)) || !draws) return fail(IE_ERR_INVALID, "NULL argument");
    HostStream rng{};
    chacha_key_from_u64(seed, rng.key);
    rng.pos = draw_offset;
    warm_start_words(rng, probs, is_clamped, clamp_val, n, cells, words);
    *draws = rng.pos;
    return IE_OK;
}

ie_status ie_pa_normalized_weights(const double* log_w, uint64_t r, double* w_out) {
    if ((!log_w || !w_out) && r) return fail(IE_ERR_INVALID, "NULL argument");
    const std::vector<double> w = pa::normalized_weights(log_w, r);
    std::copy(w.begin(), w.end(), w_out);
    return IE_OK;
}

ie_status ie_pa_effective_sample_size(const double* w, uint64_t r, double* ess) {
    if ((!w && r) || !ess) return fail(IE_ERR_INVALID, "NULL argument");
    *ess = pa::effective_sample_size(w, r);
    return IE_OK;
}

ie_status ie_pa_free_energy_increment(const double* log_w, uint64_t r, double* out) {
    if ((!log_w && r) || !out) return fail(IE_ERR_INVALID, "NULL argument");
    *out = pa::free_energy_increment(log_w, r);
    return IE_OK;
}

ie_status ie_pa_family_entropy(const uint64_t* family_ids, uint64_t r, double* rho, uint64_t* families) {
    if ((!family_ids && r) || !rho || !families) return fail(IE_ERR_INVALID, "NULL argument");
    pa::family_entropy(family_ids, r, *rho, *families);
    return IE_OK;
}

ie_status ie_pa_systematic_resample(const double* w, uint64_t r, double u, uint64_t* counts) {
    if ((!w || !counts) && r) return fail(IE_ERR_INVALID, "NULL argument");
    const std::vector<uint64_t> c = pa::systematic_resample(w, r, u);
    std::copy(c.begin(), c.end(), counts);
    return IE_OK;
}

ie_status ie_pa_feedback_optimized_alphas(const double* alphas, const double* flow, uint64_t nt, double damping,
                                          double* out) {
    if ((!alphas || !flow || !out) && nt) return fail(IE_ERR_INVALID, "NULL argument");
    const std::vector<double> a = pa::feedback_optimized_alphas(std::vector<double>(alphas, alphas + nt),
                                                                std::vector<double>(flow, flow + nt), damping);
    std::copy(a.begin(), a.end(), out);
    return IE_OK;
}

ie_status ie_pa_adapt_spacings(const double* spacings, const double* acceptance, uint64_t k, double* out) {
    if ((!spacings || !acceptance || !out) && k) return fail(IE_ERR_INVALID, "NULL argument");
    const std::vector<double> d = pa::adapt_spacings(spacings, acceptance, k);
    std::copy(d.begin(), d.end(), out);
    return IE_OK;
}

}  // extern "C"
