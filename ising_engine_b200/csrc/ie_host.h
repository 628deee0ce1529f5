// Host-side helpers shared by the library's translation units: status and
// error message, CUDA/IE status propagation, device arrays, the master-stream
// key expansion.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ising_b200.h"

namespace ie {

// Records msg as this thread's last error (ie_last_error) and returns s.
ie_status fail(ie_status s, const std::string& msg);

// rand_core 0.6.4 SeedableRng::seed_from_u64: PCG32 outputs fill the 32-byte
// ChaCha8 key (little-endian), as ChaCha8Rng::seed_from_u64 (ultimate.rs:152).
void chacha_key_from_u64(uint64_t state, uint32_t key[8]);

// Exchange thresholds of a ladder temps[nt] (engine.rs:725-727): for the pair
// (t, t+1) with db = 1/T_t - 1/T_{t+1}, a swap whose exponent db*de is
// negative is accepted iff gen::<f64>() < exp(db*de), i.e. iff (draw >> 11) <
// ceil(exp(db*de) * 2^53), which depends only on |de|: tab[off[t] + |de| - 1]
// for |de| <= dmax[t], 1 up to dund[t] (the largest |de| with exp > 0), then 0.
// Built with the host libm exp, the function the reference calls.
struct XTables {
    std::vector<uint64_t> tab, off, dmax, dund;
    std::vector<double> dbeta;
};
ie_status build_xtables(const double* temps, uint32_t nt, XTables& X);

// The master stream on the host, addressed by draw index (same draws as the
// device's chacha8_draw), with rand 0.8.5's gen_range forms the population
// annealing driver takes.
uint64_t chacha8_draw_host(const uint32_t key[8], uint64_t k);
struct HostStream {
    uint32_t key[8];
    uint64_t pos;
    uint64_t next_u64();
    double unit_f64();                    // gen_range(0.0..1.0)
    uint64_t index_inclusive(uint64_t hi);  // gen_range(0..=hi) for usize
};

// The warm-start initial words (reference layout, bit r = replica r) of
// `cells` cells of n sites from the stream at rng.pos; rng.pos advances.
void warm_start_words(HostStream& rng, const double* probs, const uint8_t* clampf, const int8_t* clampv, uint64_t n,
                      uint64_t cells, uint64_t* words);

namespace pa {
std::vector<double> normalized_weights(const double* lw, size_t r);
double effective_sample_size(const double* w, size_t r);
double free_energy_increment(const double* lw, size_t r);
void family_entropy(const uint64_t* ids, size_t r, double& rho, uint64_t& families);
std::vector<uint64_t> systematic_resample(const double* w, size_t r, double u);
std::vector<double> adapt_spacings(const double* d, const double* acc, size_t k);
std::vector<double> feedback_optimized_alphas(const std::vector<double>& alphas, const std::vector<double>& flow,
                                              double damping);
// apply_resample's parent list: parent i repeated counts[i] times, then the
// Fisher-Yates shuffle with gen_range(0..=k) for k = len - 1 down to 1.
std::vector<uint32_t> shuffled_parents(const std::vector<uint64_t>& counts, HostStream& rng);
}  // namespace pa

}  // namespace ie

#define IE_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(e_ == cudaErrorMemoryAllocation ? IE_ERR_OOM : IE_ERR_CUDA,        \
                        std::string(#call) + ": " + cudaGetErrorString(e_));               \
    } while (0)

#define IE_TRY(expr)                   \
    do {                               \
        ie_status s_ = (expr);         \
        if (s_ != IE_OK) return s_;    \
    } while (0)

namespace ie {

// Device array; alloc() keeps the allocation when it is large enough (the
// contents are not preserved either way).
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0, cap = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    ie_status alloc(size_t count) {
        n = count;
        if (count == 0 || (p && count <= cap)) return IE_OK;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        IE_CUDA(cudaMalloc(&p, count * sizeof(T)));
        cap = count;
        return IE_OK;
    }
    ie_status upload(const std::vector<T>& h, cudaStream_t st) {
        IE_TRY(alloc(h.size()));
        if (!h.empty()) IE_CUDA(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
        return IE_OK;
    }
};

}  // namespace ie
