// CUDA kernels of the B200 Metropolis / PT engine (sm_100a).
//
// Work decomposition. The reference sweeps each cell (temperature) in site
// order v = 0..n-1 and draws the 64 uniforms of site v from an 8-lane
// Xoshiro256++ generator: lane l produces the uniforms of replicas
// l, l+8, ..., l+56 (engine.rs:145-151). Replicas are independent Markov
// chains, so the natural unit of parallel work is (cell, lane): one thread
// runs one lane's generator and owns exactly the 8 replicas it drives. The 8
// threads of a cell never communicate during a sweep. Spin words are stored
// lane-major: byte l of word [cell][v] holds replicas l+8k at bit k, so a
// thread reads and writes only its own byte and no two threads ever write the
// same byte.
//
// Integer mode (bit-exact): the local field of the thread's 8 replicas is
// accumulated SWAR-style, one byte per replica, from non-negative weight
// magnitudes (negative couplings contribute |w| * (1 - x_j) and are folded
// into a per-site constant). The Metropolis decision is one 64-bit compare of
// the raw Xoshiro output against a per-temperature threshold table indexed by
// dE (metropolis_threshold), which reproduces u < fast_exp(-dE*beta) exactly.
//
// f64 mode: the reference's f64 arithmetic in the reference's order
// (engine.rs:218-271, 663-670) with every operation explicitly rounded.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "ie_device.cuh"
#include "ie_kernels.cuh"
#include "ie_sweep.cuh"

namespace ie {

// ---------------------------------------------------------------------------
// One cell sweep by one (cell, lane) thread, integer mode.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void sweep_int(const DevArrays& A, const InstDesc& d, uint64_t* words,
                                          int lane, const uint64_t* __restrict__ tab,
                                          uint64_t cell_seed, int32_t (&E)[8]) {
    Xoshiro x;
    x.seed_lane(cell_seed, lane);
    uint8_t* sp = reinterpret_cast<uint8_t*>(words) + lane;
    const uint32_t* __restrict__ rows = A.rows + d.row;
    const uint32_t* __restrict__ ents = A.ents + d.ent;
    const int32_t* __restrict__ linp = A.linp + d.site;
    const uint8_t* __restrict__ clampf = A.clampf + d.site;
    const int H = d.H;
    uint32_t beg = __ldg(rows);
    for (uint32_t v = 0; v < d.n; v++) {
        const uint32_t end = __ldg(rows + v + 1);
        if (__ldg(clampf + v)) {
#pragma unroll
            for (int k = 0; k < 8; k++) x.advance();
            beg = end;
            continue;
        }
        uint64_t res[8];
#pragma unroll
        for (int k = 0; k < 8; k++) res[k] = x.next();
        uint32_t aL = 0, aH = 0;
        for (uint32_t e = beg; e < end; e++) {
            const uint32_t en = __ldg(ents + e);
            const uint32_t b = sp[8u * (en & 0xFFFFFFu)];
            const uint32_t w = (en >> 24) & 0x7Fu;
            const uint32_t nm = (0u - (en >> 31)) & 0x01010101u;
            aL += w * (spread4(b) ^ nm);
            aH += w * (spread4(b >> 4) ^ nm);
        }
        beg = end;
        const uint32_t xb = sp[8u * v];
        const int lp = __ldg(linp + v);
        const uint32_t cA = (uint32_t)(H + lp) * 0x01010101u;
        const uint32_t cB = (uint32_t)(H - lp) * 0x01010101u;
        const uint32_t xL = spread4(xb) * 0xFFu;
        const uint32_t xH = spread4(xb >> 4) * 0xFFu;
        // byte k of iL/iH = dE_k + H for replica lane + 8k
        const uint32_t iL = ((aL + cA) & ~xL) | ((cB - aL) & xL);
        const uint32_t iH = ((aH + cA) & ~xH) | ((cB - aH) & xH);
        uint32_t flips = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const uint32_t idx = ((k < 4 ? iL : iH) >> (8 * (k & 3))) & 0xFFu;
            if (res[k] <= tab[idx]) {
                flips |= 1u << k;
                E[k] += (int32_t)idx - H;
            }
        }
        sp[8u * v] = (uint8_t)(xb ^ flips);
    }
}

// ---------------------------------------------------------------------------
// One cell sweep by one (cell, lane) thread, f64 mode (engine.rs:218-271 and
// 663-670 in order; adding w * 0.0 is skipped, which changes no value).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void sweep_f64(const DevArrays& A, const InstDesc& d, uint64_t* words,
                                          int lane, double beta, uint64_t cell_seed,
                                          double (&E)[8]) {
    Xoshiro x;
    x.seed_lane(cell_seed, lane);
    uint8_t* sp = reinterpret_cast<uint8_t*>(words) + lane;
    const uint32_t* __restrict__ rows = A.rows + d.row;
    const uint32_t* __restrict__ cols = A.cols + d.ent;
    const double* __restrict__ vals = A.vals + d.ent;
    const double* __restrict__ lin = A.lin + d.site;
    const uint8_t* __restrict__ clampf = A.clampf + d.site;
    uint32_t beg = __ldg(rows);
    for (uint32_t v = 0; v < d.n; v++) {
        const uint32_t end = __ldg(rows + v + 1);
        if (__ldg(clampf + v)) {
#pragma unroll
            for (int k = 0; k < 8; k++) x.advance();
            beg = end;
            continue;
        }
        uint64_t res[8];
#pragma unroll
        for (int k = 0; k < 8; k++) res[k] = x.next();
        const uint32_t xb = sp[8u * v];
        const double wl = __ldg(lin + v);
        double dl[8];
#pragma unroll
        for (int k = 0; k < 8; k++) dl[k] = ((xb >> k) & 1u) ? -wl : wl;
        for (uint32_t e = beg; e < end; e++) {
            const uint32_t j = __ldg(cols + e);
            const double w = __ldg(vals + e);
            const uint32_t bj = sp[8u * j];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                if ((bj >> k) & 1u) dl[k] = __dadd_rn(dl[k], ((xb >> k) & 1u) ? -w : w);
            }
        }
        beg = end;
        uint32_t flips = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const double ev = fast_exp_rn(__dmul_rn(-dl[k], beta));
            const double u = __dmul_rn((double)(res[k] >> 12), 2.220446049250313e-16);  // 2^-52
            if (dl[k] <= 0.0 || u < ev) {
                flips |= 1u << k;
                E[k] = __dadd_rn(E[k], dl[k]);
            }
        }
        sp[8u * v] = (uint8_t)(xb ^ flips);
    }
}

// calculate_replica_energies_local (engine.rs:333-368) for the thread's 8
// replicas, f64 in reference order (site order, CSR order, v < j edges).
__device__ void energies_f64_sp(const DevArrays& A, const InstDesc& d, const uint8_t* sp, double (&E)[8]) {
    const uint32_t* rows = A.rows + d.row;
    const uint32_t* cols = A.cols + d.ent;
    const double* vals = A.vals + d.ent;
    const double* lin = A.lin + d.site;
#pragma unroll
    for (int k = 0; k < 8; k++) E[k] = 0.0;
    for (uint32_t v = 0; v < d.n; v++) {
        const uint32_t xb = sp[8u * v];
        const double wl = lin[v];
#pragma unroll
        for (int k = 0; k < 8; k++)
            if ((xb >> k) & 1u) E[k] = __dadd_rn(E[k], wl);
        for (uint32_t e = rows[v]; e < rows[v + 1]; e++) {
            const uint32_t j = cols[e];
            if (v < j) {
                const uint32_t m = xb & sp[8u * j];
                if (m) {
                    const double w = vals[e];
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        if ((m >> k) & 1u) E[k] = __dadd_rn(E[k], w);
                }
            }
        }
    }
}

__device__ __forceinline__ void energies_f64(const DevArrays& A, const InstDesc& d, const uint64_t* words, int lane,
                                             double (&E)[8]) {
    energies_f64_sp(A, d, reinterpret_cast<const uint8_t*>(words) + lane, E);
}

__device__ __forceinline__ unsigned group_mask(int tid) { return 0xFFu << (8 * ((tid >> 3) & 3)); }

// ---------------------------------------------------------------------------
// Batched single-cell kernel.
//
// Persistent one-warp CTAs pull work items from a global queue ordered
// longest-first. An instance is run by a group of 8*TPL threads: TPL threads
// per Xoshiro lane, each running the lane's generator and owning the
// decisions of the calls k = h, h+TPL, ... (h = its index within the lane).
// Integer mode splits each site's neighbour sum across the TPL threads
// (SWAR partial sums, reduced with two shuffles per level); f64 mode splits the
// replicas. A warp holds 4/TPL instances; in a batched run they run the same
// schedule in step and share one threshold table per sweep, in a serving or
// PT-cells run each has its own schedule and table. Each instance streams its
// site records through a 3-slot shared-memory ring (two 512-byte chunks in
// flight ahead of the sweep: 16-byte cp.async copies spread over the group, or
// with RunArgs::bulk_ring one 1D bulk copy by the group's first thread
// completing on the slot's mbarrier); its spin words stay in shared memory
// for the whole run. Every thread of a lane writes the same combined byte, so
// each thread's later reads see the update in program order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(uint32_t* smem_dst, const uint32_t* gsrc) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait2() { asm volatile("cp.async.wait_group 2;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }

// Record ring of the per-lane kernels, two forms. cp.async: the group's
// threads copy a chunk 16 bytes each and commit one group per chunk (an empty
// one beyond the stream end); chunk k is complete once at most two newer
// groups are pending. Bulk: slot s has its own mbarrier bar[s] (arrival count
// 1); the group's first thread arms it with the chunk's 512 bytes and issues
// the 1D bulk copy (cp.async.bulk, no multicast), every thread of the group
// waits for the slot's phase. Every fetched chunk is waited for exactly once
// and in order, so the phase parity of slot s is bit s of ph. Bulk waits give
// up after kRingWaitCycles, set the error word and stop waiting (the results
// are void, the launch still ends).
constexpr long long kRingWaitCycles = 1ll << 31;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ring_init(uint64_t* bar) {
    for (uint32_t s = 0; s < kSlots; s++)
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar + s)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Chunk k of a stream into its ring slot (beyond the stream end: no copy).
template <int G>
__device__ __forceinline__ void ring_fetch(bool bulk, uint32_t* ring, uint64_t* bar, const uint32_t* stream,
                                           uint32_t nchunks, uint32_t k, int t) {
    if (!bulk) {
        if (k < nchunks) {
            uint32_t* dst = ring + (k % kSlots) * kChunk;
            const uint32_t* src = stream + (size_t)k * kChunk;
#pragma unroll
            for (int i = 0; i < 32 / G; i++) cp_async16(dst + 4 * (t + G * i), src + 4 * (t + G * i));
        }
        cp_async_commit();
        return;
    }
    if (k < nchunks && t == 0) {
        const uint32_t b = smem_u32(bar + k % kSlots);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(kChunk * 4u) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_u32(ring + (k % kSlots) * kChunk)),
                     "l"(stream + (size_t)k * kChunk), "r"(kChunk * 4u), "r"(b)
                     : "memory");
    }
}

// Waits for chunk k (fetched, two newer fetches issued, not yet waited for).
__device__ __forceinline__ void ring_wait(bool bulk, uint64_t* bar, uint32_t k, uint32_t& ph, bool& bad, int32_t* err) {
    if (!bulk) {
        cp_async_wait2();
        return;
    }
    const uint32_t s = k % kSlots, b = smem_u32(bar + s), parity = (ph >> s) & 1u;
    ph ^= 1u << s;
    if (bad) return;
    uint32_t ok = 0;
    long long t0 = 0;
    for (bool first = true;; first = false) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(b), "r"(parity)
            : "memory");
        if (ok) return;
        if (first) t0 = clock64();
        else if (clock64() - t0 > kRingWaitCycles) break;
    }
    bad = true;
    atomicExch(err, 5);
}

// The reference decision dE <= 0 || u < fast_exp(-dE * beta) (engine.rs:665-666),
// u = (res >> 12) * 2^-52: decided in f32 when the f32 value is clear of the
// band, otherwise in f64 exactly.
__device__ __forceinline__ bool metropolis_accept_f64(double de, double beta, uint64_t res) {
    const double x = __dmul_rn(-de, beta);
    const uint64_t m = res >> 12;
    const float f = fast_exp_f32((float)x);
    const float u = __fmul_rn(__ull2float_rn(m), 2.220446049250313e-16f);
    const bool sure_yes = u < __fmul_rn(f, 0.9990234375f);
    const bool sure_no = u > __fmul_rn(f, 1.0009765625f);
    bool acc = sure_yes;
    if (!sure_yes && !sure_no && de > 0.0) acc = metropolis_exact_f64(x, m);
    return de <= 0.0 || acc;
}

template <int TPL>
__device__ __forceinline__ uint32_t lane_or(uint32_t v, unsigned gmask) {
    if constexpr (TPL >= 2) v |= __shfl_xor_sync(gmask, v, 1);
    if constexpr (TPL >= 4) v |= __shfl_xor_sync(gmask, v, 2);
    return v;
}
template <int TPL>
__device__ __forceinline__ uint32_t lane_add(uint32_t v, unsigned gmask) {
    if constexpr (TPL >= 2) v += __shfl_xor_sync(gmask, v, 1);
    if constexpr (TPL >= 4) v += __shfl_xor_sync(gmask, v, 2);
    return v;
}

// Hand-over between a generator warp and decider warps: two output buffers of
// one window of kWin sites each (row (site, lane) holds the lane's 8 calls),
// guarded by named barriers: bar.arrive by the producing side, bar.sync by the
// waiting side, with the exact thread count of the two sides.
constexpr int kRS = 10;  // u64 per (site, lane) row of the output / dE buffers (8 calls + padding against bank conflicts)
constexpr int kBarFull0 = 1, kBarEmpty0 = 3, kBarCons = 5;

__device__ __forceinline__ void bar_sync(int id, int count) { asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(count) : "memory"); }
__device__ __forceinline__ void bar_arrive(int id, int count) { asm volatile("bar.arrive %0, %1;\n" ::"r"(id), "r"(count) : "memory"); }

// Generator of the windowed and chain kernels: thread (lane rl = t / 4, offset
// rh = t % 4) runs lane rl's Xoshiro chain (engine.rs:87-123) over the sweep
// and stores the calls it owns (rh, rh + 4) of every site into the window's
// buffer; nthreads is the barrier count of the whole hand-over.
__device__ __forceinline__ void produce_windows(uint64_t base, uint32_t n, uint64_t* rngb, int t, int nthreads) {
    const int rl = t >> 2, rh = t & 3;
    Xoshiro x;
    x.seed_lane(base, rl);
    for (int i = 0; i < rh; i++) x.advance();
    const uint32_t nwin = (n + kWin - 1) / kWin;
    for (uint32_t w = 0; w < nwin; w++) {
        const int b = w & 1;
        if (w >= 2) bar_sync(kBarEmpty0 + b, nthreads);
        uint64_t* ob = rngb + b * (8 * kWin) * kRS;
#pragma unroll
        for (int i = 0; i < kWin; i++) {
#pragma unroll
            for (int kk = 0; kk < 8; kk++) {
                if (kk % 4 == 0) ob[(i * 8 + rl) * kRS + rh + kk] = x.next();
                else x.advance();
            }
        }
        bar_arrive(kBarFull0 + b, nthreads);
    }
    for (uint32_t w = nwin >= 2 ? nwin - 2 : 0; w < nwin; w++) bar_sync(kBarEmpty0 + (w & 1), nthreads);
}

template <uint32_t MODE, int TPL>
using ETypeT = typename std::conditional<MODE == kModeInt, int32_t, double>::type;

// PROD: the uniforms come from a generator warp through rngb (produce_windows;
// barrier count 64), window by window, instead of the thread's own generator.
template <uint32_t MODE, int TPL, bool PROD = false>
__device__ __forceinline__ void sweep_stream(const DevArrays& A, const InstDesc& d, bool bulk, uint32_t* ring,
                                             uint64_t* bar, uint32_t& ph, bool& bad, uint8_t* sp,
                                             const uint2* __restrict__ lut, int lane, int h, unsigned gmask,
                                             const uint64_t* __restrict__ tab,
                                             int H, double beta, uint64_t cell_seed,
                                             ETypeT<MODE, TPL> (&E)[8 / TPL], const uint64_t* rngb = nullptr) {
    constexpr int G = 8 * TPL;
    constexpr int KP = 8 / TPL;    // calls owned by this thread: k = j*TPL + h
    constexpr int EP = 16 / TPL;   // integer mode: record entries summed by this thread
    const int t = lane * TPL + h;
    // Thread h of a lane runs the lane's generator h steps ahead, so the calls
    // it owns (k = j*TPL + h) fall on its local steps j*TPL.
    Xoshiro x;
    if (!PROD) {
        x.seed_lane(cell_seed, lane);
        for (int i = 0; i < h; i++) x.advance();
    }
    const uint32_t* stream = A.recs + d.rec;
    const uint32_t nchunks = (uint32_t)(d.rec_len / kChunk);
    ring_fetch<G>(bulk, ring, bar, stream, nchunks, 0, t);
    ring_fetch<G>(bulk, ring, bar, stream, nchunks, 1, t);
    ring_fetch<G>(bulk, ring, bar, stream, nchunks, 2, t);
    if (nchunks) ring_wait(bulk, bar, 0, ph, bad, A.err);
    __syncwarp(gmask);
    uint32_t k = 0, c = 0;
    const uint32_t* chunk = ring;
    bool open = false;
    uint64_t res[KP];
    uint32_t xb = 0, aL = 0, aH = 0;
    int lp = 0;
    double dl[KP], tp[KP];
    for (uint32_t v = 0; v < d.n;) {
        const uint32_t hdr = (c < kChunk) ? chunk[c] : kRecPad;
        if (hdr == kRecPad) {
            __syncwarp(gmask);
            k++;
            c = 0;
            ring_fetch<G>(bulk, ring, bar, stream, nchunks, k + 2, t);
            ring_wait(bulk, bar, k, ph, bad, A.err);
            __syncwarp(gmask);
            chunk = ring + (k % kSlots) * kChunk;
            continue;
        }
        const uint32_t* rec = chunk + c;
        const uint32_t deg = hdr & 0x1Fu;
        const uint32_t deg4 = (deg + 3u) & ~3u;
        if (!open) {
            // first record of site v: this site's uniforms and current spins
            if constexpr (PROD) {
                const uint32_t vw = v % kWin, b = (v / kWin) & 1u;
                if (vw == 0) bar_sync(kBarFull0 + b, 64);
                const uint64_t* rr = rngb + b * (8 * kWin) * kRS + (vw * 8 + lane) * kRS + h;
#pragma unroll
                for (int j = 0; j < KP; j++) res[j] = rr[j * TPL];
            } else {
#pragma unroll
                for (int kk = 0; kk < 8; kk++) {
                    if (kk % TPL == 0) res[kk / TPL] = x.next();
                    else x.advance();
                }
            }
            xb = sp[8u * v];
            if constexpr (MODE == kModeInt) {
                aL = aH = 0;
                lp = (int)(hdr >> 16) - 128;
            } else {
                const double wl = *reinterpret_cast<const double*>(rec + 2);
#pragma unroll
                for (int j = 0; j < KP; j++) {
                    const bool xv = (xb >> (j * TPL + h)) & 1u;
                    tp[j] = xv ? -1.0 : 1.0;
                    dl[j] = xv ? -wl : wl;
                }
            }
        }
        const bool clamped = hdr & kRecClamp;
        if constexpr (MODE == kModeInt) {
            c += 4 + deg4;
            const uint32_t* ent = rec + 4 + EP * h;
#pragma unroll
            for (int qd = 0; qd < EP / 4; qd++) {
                if ((uint32_t)(EP * h + 4 * qd) < deg) {
                    const uint4 e4 = *reinterpret_cast<const uint4*>(ent + 4 * qd);
                    const uint32_t en[4] = {e4.x, e4.y, e4.z, e4.w};
                    uint32_t li[4];
#pragma unroll
                    for (int e = 0; e < 4; e++) li[e] = sp[8u * (en[e] & 0xFFFFFFu)] | ((en[e] >> 23) & 0x100u);
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const uint2 sv = lut[li[e]];
                        const uint32_t w = (en[e] >> 24) & 0x7Fu;
                        aL += w * sv.x;
                        aH += w * sv.y;
                    }
                }
            }
        } else {
            const uint32_t* cols = rec + 4;
            const double* vals = reinterpret_cast<const double*>(rec + 4 + deg4);
            c += 4 + 3 * deg4;
#pragma unroll
            for (int qd = 0; qd < 4; qd++) {
                if ((uint32_t)(4 * qd) < deg) {
                    const uint4 c4 = *reinterpret_cast<const uint4*>(cols + 4 * qd);
                    const uint32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
                    const double2 w01 = *reinterpret_cast<const double2*>(vals + 4 * qd);
                    const double2 w23 = *reinterpret_cast<const double2*>(vals + 4 * qd + 2);
                    const double ww[4] = {w01.x, w01.y, w23.x, w23.y};
                    uint32_t bj[4];
#pragma unroll
                    for (int e = 0; e < 4; e++) bj[e] = sp[8u * cc[e]];
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        if ((uint32_t)(4 * qd + e) < deg) {
#pragma unroll
                            for (int j = 0; j < KP; j++) {
                                // t = (x_j ^ x_v) - x_v = x_j ? (x_v ? -1 : 1) : 0; w * t is
                                // exact, so fma(w, t, dE) equals the reference's dE + w * t.
                                const double tt = ((bj[e] >> (j * TPL + h)) & 1u) ? tp[j] : 0.0;
                                dl[j] = __fma_rn(ww[e], tt, dl[j]);
                            }
                        }
                    }
                }
            }
        }
        if (hdr & kRecCont) {
            open = true;
            continue;
        }
        open = false;
        if (!clamped) {
            uint32_t flips = 0;
            if constexpr (MODE == kModeInt) {
                aL = lane_add<TPL>(aL, gmask);
                aH = lane_add<TPL>(aH, gmask);
                const uint32_t cA = (uint32_t)(H + lp) * 0x01010101u;
                const uint32_t cB = (uint32_t)(H - lp) * 0x01010101u;
                const uint32_t xL = spread4(xb) * 0xFFu;
                const uint32_t xH = spread4(xb >> 4) * 0xFFu;
                const uint32_t iL = ((aL + cA) & ~xL) | ((cB - aL) & xL);
                const uint32_t iH = ((aH + cA) & ~xH) | ((cB - aH) & xH);
#pragma unroll
                for (int j = 0; j < KP; j++) {
                    const int kk = j * TPL + h;
                    const uint32_t idx = ((kk < 4 ? iL : iH) >> (8 * (kk & 3))) & 0xFFu;
                    if (res[j] <= tab[idx]) {
                        flips |= 1u << kk;
                        E[j] += (int32_t)idx - H;
                    }
                }
            } else {
#pragma unroll
                for (int j = 0; j < KP; j++) {
                    if (metropolis_accept_f64(dl[j], beta, res[j])) {
                        flips |= 1u << (j * TPL + h);
                        E[j] = __dadd_rn(E[j], dl[j]);
                    }
                }
            }
            flips = lane_or<TPL>(flips, gmask);
            sp[8u * v] = (uint8_t)(xb ^ flips);
        }
        if constexpr (PROD) {
            if (v % kWin == kWin - 1 || v + 1 == d.n) bar_arrive(kBarEmpty0 + ((v / kWin) & 1u), 64);
        }
        v++;
    }
    if (!bulk) cp_async_wait0();
    __syncwarp(gmask);
}

// f64 recompute of the energies of the calls this thread owns (engine.rs:333-368).
template <int TPL>
__device__ void energies_f64_calls(const DevArrays& A, const InstDesc& d, const uint8_t* sp, int h,
                                   double (&E)[8 / TPL]) {
    double e8[8];
    energies_f64_sp(A, d, sp, e8);
#pragma unroll
    for (int j = 0; j < 8 / TPL; j++) {
        double v = e8[0];
#pragma unroll
        for (int kk = 0; kk < 8; kk++)
            if (kk == j * TPL + h) v = e8[kk];
        E[j] = v;
    }
}

// Dynamic shared memory of a batched CTA: threshold tables (2 KB each: one
// shared by the warp, or in a serving launch one per instance, whose
// temperatures differ) | spread table (4 KB) | NG rings | NG spin arrays of
// spin_cap words each (the instance's spins stay resident in shared memory
// for the whole schedule).
__host__ __device__ constexpr size_t batch_smem_bytes(int ng, uint32_t spin_cap, bool own_tables) {
    return 2048 * (size_t)(own_tables ? ng : 1) + 4096 + (size_t)ng * kSlots * kChunk * 4 + (size_t)ng * spin_cap * 8;
}

template <uint32_t MODE, int TPL>
__global__ void __launch_bounds__(32) batch_kernel(DevArrays A, RunArgs R, uint32_t spin_cap) {
    constexpr int G = 8 * TPL;
    constexpr int NG = 4 / TPL;  // instances per warp
    constexpr int KP = 8 / TPL;
    extern __shared__ __align__(16) uint64_t dsm[];
    const int tid = threadIdx.x;
    const int g = tid / G;
    const int t = tid % G;
    const int lane = t / TPL;
    const int h = t % TPL;
    // per-instance threshold tables when the instances of a warp run at
    // different temperatures (serving, PT cells)
    const bool own_tab = R.serve != 0 || R.cells != 0;
    const int ntab = own_tab ? NG : 1;
    uint64_t* tab = dsm + (own_tab ? 256 * g : 0);
    uint2* lut = reinterpret_cast<uint2*>(dsm + 256 * ntab);
    uint32_t* ring = reinterpret_cast<uint32_t*>(dsm + 256 * ntab + 512) + (size_t)g * kSlots * kChunk;
    uint64_t* sw = reinterpret_cast<uint64_t*>(reinterpret_cast<uint32_t*>(dsm + 256 * ntab + 512) +
                                               (size_t)NG * kSlots * kChunk) +
                   (size_t)g * spin_cap;
    // spread table: entry b (and 256 + b for a negative coupling, which
    // contributes |w| (1 - x_j)) holds bit k of b (resp. ~b) in byte k of
    // (lo word: k < 4, hi word: k >= 4)
    if constexpr (MODE == kModeInt) {
        for (int i = tid; i < 512; i += 32) {
            const uint32_t b = (i < 256 ? (uint32_t)i : (uint32_t)(i - 256) ^ 0xFFu);
            lut[i] = make_uint2(spread4(b), spread4(b >> 4));
        }
        __syncwarp();
    }
    uint8_t* sp = reinterpret_cast<uint8_t*>(sw) + lane;
    const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (G * g));
    __shared__ __align__(8) uint64_t s_bar[NG][kSlots];
    if (t == 0) ring_init(s_bar[g]);
    __syncwarp();
    uint32_t ph = 0;
    bool bad = false;
    typedef ETypeT<MODE, TPL> EType;
    for (;;) {
        uint32_t q = 0;
        if (tid == 0) q = atomicAdd(R.queue, 1u);
        q = __shfl_sync(0xffffffffu, q, 0);
        if (q >= R.nquads) break;
        const uint32_t inst = R.quads[4 * q + g];
        const bool active = inst != 0xffffffffu;
        const int H = MODE == kModeInt ? R.quad_h[q] : 0;
        InstDesc d{};
        uint32_t key[8];
        uint64_t pos0 = 0;
        EType E[KP];
        StepPlan P{R.step_base, own_tab ? 0u : R.steps, R.temps_per_step, R.temps};
        if (active) {
            d = A.desc[inst];
            if (d.n > spin_cap) {  // host sizing error: report and skip the instance
                if (t == 0) atomicExch(A.err, 2);
                continue;
            }
            P = step_plan(A, R, d, inst);
#pragma unroll
            for (int i = 0; i < 8; i++) key[i] = A.keys[8 * (size_t)d.owner + i];
            pos0 = A.pos[d.owner];
#pragma unroll
            for (int j = 0; j < KP; j++) {
                const size_t o = d.energy + lane + 8 * (j * TPL + h);
                if constexpr (MODE == kModeInt) E[j] = A.Ei[o];
                else E[j] = A.Ef[o];
            }
            const uint64_t* gw = A.spins + d.spin;
            for (uint32_t i = t; i < d.n; i += G) sw[i] = gw[i];
            __syncwarp(gmask);
        }
        // Shared table: every group (active or not) runs the launch's steps in
        // step and the warp fills the table. Own tables: each active group runs
        // its own steps and fills its own table.
        for (uint32_t s = 0; s < P.steps; s++) {
            const double beta = __ddiv_rn(1.0, P.temps[(size_t)P.tstride * s]);
            if constexpr (MODE == kModeInt) {
                if (own_tab) {
                    __syncwarp(gmask);
                    for (int i = t; i < 2 * H + 1; i += G) tab[i] = metropolis_threshold(i - H, beta);
                    __syncwarp(gmask);
                } else {
                    __syncwarp();
                    for (int i = tid; i < 2 * H + 1; i += 32) tab[i] = metropolis_threshold(i - H, beta);
                    __syncwarp();
                }
            }
            if (active) {
                const uint64_t base = chacha8_draw(key, pos0 + s) + d.cell;
                sweep_stream<MODE, TPL>(A, d, R.bulk_ring != 0, ring, s_bar[g], ph, bad, sp, lut, lane, h, gmask, tab, H, beta, base, E);
                if constexpr (MODE == kModeF64) {
                    if (!R.cells && (P.base + s + 1) % kResyncEvery == 0) {
                        __syncwarp(gmask);
                        energies_f64_calls<TPL>(A, d, sp, h, E);
                    }
                }
            }
        }
        if (active) {
            __syncwarp(gmask);
            uint64_t* gw = A.spins + d.spin;
            for (uint32_t i = t; i < d.n; i += G) gw[i] = sw[i];
#pragma unroll
            for (int j = 0; j < KP; j++) {
                const size_t o = d.energy + lane + 8 * (j * TPL + h);
                if constexpr (MODE == kModeInt) A.Ei[o] = E[j];
                else A.Ef[o] = E[j];
            }
            __syncwarp(gmask);
            if (t == 0 && !R.cells) {
                A.pos[d.owner] = pos0 + P.steps;
                A.deo[d.owner] ^= (int32_t)(exchanges_in(P.base, P.steps, R.exchange_interval) & 1u);
                if (R.serve) A.done[d.owner] = P.base + P.steps;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Chain kernel: the per-lane sweep of batch_kernel<MODE, 4> (one instance per
// CTA, 4 threads per Xoshiro lane) with the uniforms made ahead by a generator
// warp (produce_windows), so the site chain carries no generator steps. For
// instances whose consecutive sites are coupled (lattices), where the
// windowed kernel has one site per level. GSP: spins stay in global memory.
// Dynamic shared memory: threshold table | spread table | record ring |
// generator buffers | spins (spin_cap words; none when GSP).
// ---------------------------------------------------------------------------
__host__ __device__ constexpr size_t chain_smem_bytes(uint32_t spin_cap) {
    return 2048 + 4096 + (size_t)kSlots * kChunk * 4 + 2 * (8 * kWin) * kRS * 8 + (size_t)spin_cap * 8;
}

template <uint32_t MODE, bool GSP>
__global__ void __launch_bounds__(64, 1) chain_kernel(DevArrays A, RunArgs R, uint32_t spin_cap) {
    extern __shared__ __align__(16) uint64_t dsm[];
    __shared__ uint32_t s_item;
    uint64_t* tab = dsm;
    uint2* lut = reinterpret_cast<uint2*>(dsm + 256);
    uint32_t* ring = reinterpret_cast<uint32_t*>(dsm + 768);
    uint64_t* rngb = reinterpret_cast<uint64_t*>(ring + kSlots * kChunk);
    uint64_t* const ssw = rngb + 2 * (8 * kWin) * kRS;
    const int tid = threadIdx.x;
    const bool producer = tid < 32;
    const int t = tid & 31;
    const int lane = t >> 2, h = t & 3;
    __shared__ __align__(8) uint64_t s_bar[kSlots];
    if (tid == 32) ring_init(s_bar);
    uint32_t ph = 0;
    bool bad = false;
    typedef ETypeT<MODE, 4> EType;
    if constexpr (MODE == kModeInt) {
        for (int i = tid; i < 512; i += 64) {
            const uint32_t b = (i < 256 ? (uint32_t)i : (uint32_t)(i - 256) ^ 0xFFu);
            lut[i] = make_uint2(spread4(b), spread4(b >> 4));
        }
    }
    __syncthreads();
    for (;;) {
        if (tid == 0) s_item = atomicAdd(R.queue, 1u);
        __syncthreads();
        const uint32_t q = s_item;
        __syncthreads();
        if (q >= R.nquads) break;
        const uint32_t inst = R.quads[4 * q];
        if (inst == 0xffffffffu) continue;
        const int H = MODE == kModeInt ? R.quad_h[q] : 0;
        const InstDesc d = A.desc[inst];
        if (!GSP && d.n > spin_cap) {
            if (tid == 0) atomicExch(A.err, 2);
            continue;
        }
        uint64_t* const sw = GSP ? A.spins + d.spin : ssw;
        uint8_t* const sp = reinterpret_cast<uint8_t*>(sw) + lane;
        const StepPlan P = step_plan(A, R, d, inst);
        uint32_t key[8];
#pragma unroll
        for (int i = 0; i < 8; i++) key[i] = A.keys[8 * (size_t)d.owner + i];
        const uint64_t pos0 = A.pos[d.owner];
        EType E[2] = {0, 0};
        if (!producer) {
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const size_t o = d.energy + lane + 8 * (j * 4 + h);
                if constexpr (MODE == kModeInt) E[j] = A.Ei[o];
                else E[j] = A.Ef[o];
            }
        }
        if (!GSP) {
            const uint64_t* gw = A.spins + d.spin;
            for (uint32_t i = tid; i < d.n; i += 64) sw[i] = gw[i];
        }
        __syncthreads();
        for (uint32_t s = 0; s < P.steps; s++) {
            const double beta = __ddiv_rn(1.0, P.temps[(size_t)P.tstride * s]);
            const uint64_t base = chacha8_draw(key, pos0 + s) + d.cell;
            if (producer) {
                produce_windows(base, d.n, rngb, t, 64);
            } else {
                if constexpr (MODE == kModeInt) {
                    __syncwarp();
                    for (int i = t; i < 2 * H + 1; i += 32) tab[i] = metropolis_threshold(i - H, beta);
                    __syncwarp();
                }
                sweep_stream<MODE, 4, true>(A, d, R.bulk_ring != 0, ring, s_bar, ph, bad, sp, lut, lane, h, 0xffffffffu, tab, H, beta, base,
                                            E, rngb);
                if constexpr (MODE == kModeF64) {
                    if (!R.cells && (P.base + s + 1) % kResyncEvery == 0) {
                        __syncwarp();
                        energies_f64_calls<4>(A, d, sp, h, E);
                    }
                }
            }
        }
        __syncthreads();
        if (!GSP) {
            uint64_t* gwo = A.spins + d.spin;
            for (uint32_t i = tid; i < d.n; i += 64) gwo[i] = sw[i];
        }
        if (!producer) {
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const size_t o = d.energy + lane + 8 * (j * 4 + h);
                if constexpr (MODE == kModeInt) A.Ei[o] = E[j];
                else A.Ef[o] = E[j];
            }
        }
        if (tid == 0 && !R.cells) {
            A.pos[d.owner] = pos0 + P.steps;
            A.deo[d.owner] ^= (int32_t)(exchanges_in(P.base, P.steps, R.exchange_interval) & 1u);
            if (R.serve) A.done[d.owner] = P.base + P.steps;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Windowed kernel for large instances whose consecutive sites are rarely
// coupled (random graphs). One CTA runs one instance through windows of kWin
// consecutive sites, warp-specialised:
//  1. warp 0 is the generator (produce_windows): thread (lane rl, offset rh)
//     runs lane rl's Xoshiro chain and stores the calls it owns (rh, rh + 4)
//     of every site of window w + 1 while the deciders work on window w;
//  2. NC decider warps take the window's 8 kWin (site, lane) tasks (SPLIT
//     threads each) level by level (a site waits only for lower-indexed
//     neighbours in the same window; the levels come from a host-built window
//     table), so the outcome equals the reference's site order exactly;
//  3. each accepted dE goes to shared memory and every replica's energy is
//     accumulated in site order, the reference's f64 summation order.
// The records of window w + 2 stream into one of three shared buffers with
// cp.async while window w is processed. Spins stay in shared memory, or in
// global memory (GSP) for instances beyond it.
// Window table layout: kWin / kWT in ie_kernels.cuh.
// ---------------------------------------------------------------------------
constexpr uint32_t kWinRecWords = kWin * (4 + 3 * kWinMaxDeg);  // kWin f64 records of degree <= 32
constexpr uint32_t kWinBufs = 3;  // record buffers: window w in use, w+1 landed, w+2 in flight


// Copies the records of one window (positions from its table entry) into buf.
__device__ __forceinline__ void window_fetch(const uint32_t* ent, const uint32_t* stream, uint32_t* buf, int tid,
                                             int nthreads) {
    uint32_t pos[kWin], off[kWin + 1];
    off[0] = 0;
#pragma unroll
    for (int i = 0; i < kWin; i++) {
        const uint32_t e = ent[i];
        pos[i] = e & 0xFFFFFFu;
        off[i + 1] = off[i] + (e >> 24);
    }
    for (uint32_t j = tid; j < off[kWin]; j += nthreads) {
        uint32_t src = 0;
#pragma unroll
        for (int i = 0; i < kWin; i++)
            if (j >= off[i] && j < off[i + 1]) src = pos[i] + (j - off[i]);
        cp_async16(buf + 4 * j, stream + 4 * (size_t)src);
    }
}

__host__ __device__ constexpr size_t ws_smem_bytes(uint32_t spin_cap) {
    // tab 2 KB | spread table 4 KB | outputs 2 x 8 kWin rows | dE 8 kWin rows | records | spins
    return 2048 + 4096 + 2 * (8 * kWin) * kRS * 8 + (8 * kWin) * kRS * 8 + kWinBufs * kWinRecWords * 4 +
           (size_t)spin_cap * 8;
}

template <uint32_t MODE>
struct WsCfg {
    static constexpr int SPLIT = MODE == kModeInt ? 1 : 2;  // decider threads per (site, lane) task
    static constexpr int NC = kWin * 8 * SPLIT / 32;        // decider warps: one thread per task share
    static constexpr int THREADS = 32 * (1 + NC);
    static constexpr int KPT = 8 / SPLIT;                  // calls decided per thread
};

// One (site, lane) decision task (or one half of it in f64 mode): dE of the
// thread's calls, Metropolis decisions, the accepted dE into deb, and the new
// spin byte. Returns the flip bits of the thread's calls.
template <uint32_t MODE>
__device__ __forceinline__ uint32_t ws_task(const uint32_t* rec, uint8_t* spc, uint32_t v, const uint64_t* rp,
                                            void* debrow, const uint2* __restrict__ lut,
                                            const uint64_t* __restrict__ tab, int H, double beta, int half) {
    constexpr int KPT = WsCfg<MODE>::KPT;
    const uint32_t hdr = rec[0];
    const uint32_t deg = hdr & 0x3Fu;
    const uint32_t deg4 = (deg + 3u) & ~3u;
    const uint32_t xb = spc[8u * v];
    uint32_t flips = 0;
    if constexpr (MODE == kModeInt) {
        int64_t* deb = reinterpret_cast<int64_t*>(debrow);
        if (hdr & kRecClamp) {
#pragma unroll
            for (int k = 0; k < 8; k++) deb[k] = 0;
            return 0;
        }
        uint64_t res[8];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const ulonglong2 r2 = *reinterpret_cast<const ulonglong2*>(rp + 2 * q);
            res[2 * q] = r2.x;
            res[2 * q + 1] = r2.y;
        }
        uint32_t aL = 0, aH = 0;
#pragma unroll
        for (int qd = 0; qd < (int)kWinMaxDeg / 4; qd++) {
            if ((uint32_t)(4 * qd) < deg) {
                const uint4 e4 = *reinterpret_cast<const uint4*>(rec + 4 + 4 * qd);
                const uint32_t en[4] = {e4.x, e4.y, e4.z, e4.w};
                uint32_t li[4];
#pragma unroll
                for (int e = 0; e < 4; e++) li[e] = spc[8u * (en[e] & 0xFFFFFFu)] | ((en[e] >> 23) & 0x100u);
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const uint2 sv = lut[li[e]];
                    const uint32_t ww = (en[e] >> 24) & 0x7Fu;
                    aL += ww * sv.x;
                    aH += ww * sv.y;
                }
            }
        }
        const int lp = (int)(hdr >> 16) - 128;
        const uint32_t cA = (uint32_t)(H + lp) * 0x01010101u;
        const uint32_t cB = (uint32_t)(H - lp) * 0x01010101u;
        const uint32_t xL = spread4(xb) * 0xFFu;
        const uint32_t xH = spread4(xb >> 4) * 0xFFu;
        const uint32_t iL = ((aL + cA) & ~xL) | ((cB - aL) & xL);
        const uint32_t iH = ((aH + cA) & ~xH) | ((cB - aH) & xH);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const uint32_t idx = ((k < 4 ? iL : iH) >> (8 * (k & 3))) & 0xFFu;
            const bool acc = res[k] <= tab[idx];
            flips |= (uint32_t)acc << k;
            deb[k] = acc ? (int64_t)((int32_t)idx - H) : 0;
        }
    } else {
        double* deb = reinterpret_cast<double*>(debrow) + KPT * half;
        if (hdr & kRecClamp) {
#pragma unroll
            for (int j = 0; j < KPT; j++) deb[j] = 0.0;
            return 0;
        }
        uint64_t res[KPT];
#pragma unroll
        for (int q = 0; q < KPT / 2; q++) {
            const ulonglong2 r2 = *reinterpret_cast<const ulonglong2*>(rp + KPT * half + 2 * q);
            res[2 * q] = r2.x;
            res[2 * q + 1] = r2.y;
        }
        const double wl = *reinterpret_cast<const double*>(rec + 2);
        const uint32_t* cols = rec + 4;
        const double* vals = reinterpret_cast<const double*>(rec + 4 + deg4);
        const uint32_t xs = xb >> (KPT * half);
        double dl[KPT], tp[KPT];
#pragma unroll
        for (int j = 0; j < KPT; j++) {
            const bool xv = (xs >> j) & 1u;
            tp[j] = xv ? -1.0 : 1.0;
            dl[j] = xv ? -wl : wl;
        }
#pragma unroll
        for (int qd = 0; qd < (int)kWinMaxDeg / 4; qd++) {
            if ((uint32_t)(4 * qd) < deg) {
                const uint4 c4 = *reinterpret_cast<const uint4*>(cols + 4 * qd);
                const uint32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
                const double2 w01 = *reinterpret_cast<const double2*>(vals + 4 * qd);
                const double2 w23 = *reinterpret_cast<const double2*>(vals + 4 * qd + 2);
                const double wv[4] = {w01.x, w01.y, w23.x, w23.y};
                uint32_t bj[4];
#pragma unroll
                for (int e = 0; e < 4; e++) bj[e] = spc[8u * cc[e]] >> (KPT * half);
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    if ((uint32_t)(4 * qd + e) < deg) {
#pragma unroll
                        for (int j = 0; j < KPT; j++) dl[j] = __fma_rn(wv[e], ((bj[e] >> j) & 1u) ? tp[j] : 0.0, dl[j]);
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < KPT; j++) {
            const bool acc = metropolis_accept_f64(dl[j], beta, res[j]);
            flips |= (uint32_t)acc << (KPT * half + j);
            deb[j] = acc ? dl[j] : 0.0;
        }
    }
    return flips;
}

// GSP: the instance's spin words stay in global memory (instances too large
// for shared memory); otherwise they are copied into shared memory per item.
template <uint32_t MODE, bool GSP>
__global__ void __launch_bounds__(WsCfg<MODE>::THREADS, 1) window_kernel(DevArrays A, RunArgs R, uint32_t spin_cap) {
    constexpr int NC = WsCfg<MODE>::NC;
    constexpr int NT = WsCfg<MODE>::THREADS;
    constexpr int SPLIT = WsCfg<MODE>::SPLIT;
    extern __shared__ __align__(16) uint64_t dsm[];
    __shared__ uint32_t s_item;
    uint64_t* tab = dsm;
    uint2* lut = reinterpret_cast<uint2*>(dsm + 256);
    uint64_t* rngb = dsm + 768;                            // 2 x 8 kWin rows of kRS
    uint64_t* deb = rngb + 2 * (8 * kWin) * kRS;           // 8 kWin rows of kRS
    uint32_t* recb = reinterpret_cast<uint32_t*>(deb + (8 * kWin) * kRS);
    uint64_t* const ssw = reinterpret_cast<uint64_t*>(recb + kWinBufs * kWinRecWords);
    const int tid = threadIdx.x;
    const bool producer = tid < 32;
    const int c = tid - 32;  // decider index
    // decider task: site ti (0 .. kWin - 1), lane tl, half th
    const int ti = producer ? 0 : c / (8 * SPLIT);
    const int tl = producer ? 0 : (c / SPLIT) & 7;
    const int th = producer ? 0 : c % SPLIT;
    typedef typename std::conditional<MODE == kModeInt, int32_t, double>::type EType;
    if constexpr (MODE == kModeInt) {
        for (int i = tid; i < 512; i += NT) {
            const uint32_t b = (i < 256 ? (uint32_t)i : (uint32_t)(i - 256) ^ 0xFFu);
            lut[i] = make_uint2(spread4(b), spread4(b >> 4));
        }
    }
    __syncthreads();
    for (;;) {
        if (tid == 0) s_item = atomicAdd(R.queue, 1u);
        __syncthreads();
        const uint32_t q = s_item;
        __syncthreads();
        if (q >= R.nquads) break;
        const uint32_t inst = R.quads[4 * q];
        if (inst == 0xffffffffu) continue;
        const int H = MODE == kModeInt ? R.quad_h[q] : 0;
        const InstDesc d = A.desc[inst];
        if (!GSP && d.n > spin_cap) {
            if (tid == 0) atomicExch(A.err, 2);
            continue;
        }
        uint64_t* const sw = GSP ? A.spins + d.spin : ssw;
        uint8_t* const spc = reinterpret_cast<uint8_t*>(sw) + tl;
        const StepPlan P = step_plan(A, R, d, inst);
        uint32_t key[8];
#pragma unroll
        for (int i = 0; i < 8; i++) key[i] = A.keys[8 * (size_t)d.owner + i];
        const uint64_t pos0 = A.pos[d.owner];
        // energies: decider c < 64 owns replica (lane c / 8, call c % 8)
        const int el = c >> 3, ek = c & 7;
        const bool eown = !producer && c < 64;
        EType E = 0;
        if (eown) {
            const size_t o = d.energy + el + 8 * ek;
            if constexpr (MODE == kModeInt) E = A.Ei[o];
            else E = A.Ef[o];
        }
        if (!GSP) {
            const uint64_t* gw = A.spins + d.spin;
            for (uint32_t i = tid; i < d.n; i += NT) sw[i] = gw[i];
        }
        const uint32_t nwin = (d.n + kWin - 1) / kWin;
        const uint32_t* wt = A.wtab + d.win;
        const uint32_t* stream = A.recs + d.wrec;
        for (uint32_t s = 0; s < P.steps; s++) {
            __syncthreads();
            const double beta = __ddiv_rn(1.0, P.temps[(size_t)P.tstride * s]);
            if constexpr (MODE == kModeInt) {
                for (int i = tid; i < 2 * H + 1; i += NT) tab[i] = metropolis_threshold(i - H, beta);
                __syncthreads();
            }
            const uint64_t base = chacha8_draw(key, pos0 + s) + d.cell;
            if (producer) {
                produce_windows(base, d.n, rngb, tid, NT);
            } else {
                // records of window w + 2 are fetched while window w runs
                window_fetch(wt, stream, recb, c, 32 * NC);
                cp_async_commit();
                if (nwin > 1) window_fetch(wt + kWT, stream, recb + kWinRecWords, c, 32 * NC);
                cp_async_commit();
                for (uint32_t w = 0; w < nwin; w++) {
                    const int b = w & 1;
                    uint32_t cur[kWin + 3];
#pragma unroll
                    for (int i = 0; i < kWin + 3; i++) cur[i] = wt[kWT * (size_t)w + i];
                    if (w + 2 < nwin)
                        window_fetch(wt + kWT * (size_t)(w + 2), stream, recb + ((w + 2) % kWinBufs) * kWinRecWords, c,
                                     32 * NC);
                    cp_async_commit();
                    cp_async_wait1();
                    bar_sync(kBarFull0 + b, NT);  // outputs of window w are ready; records of w, w+1 visible
                    const uint32_t* rb = recb + (w % kWinBufs) * kWinRecWords;
                    uint32_t off = 0;
#pragma unroll
                    for (int i = 0; i < kWin; i++)
                        if (i < ti) off += cur[i] >> 24;
                    const uint32_t v = w * kWin + ti;
                    const uint32_t lev = ((ti < 8 ? cur[kWin] : cur[kWin + 1]) >> (4 * (ti % 8))) & 15u;
                    const uint64_t* rp = rngb + b * (8 * kWin) * kRS + (ti * 8 + tl) * kRS;
                    uint64_t* drow = deb + (ti * 8 + tl) * kRS;
                    for (uint32_t L = 0; L <= cur[kWin + 2]; L++) {
                        if (v < d.n && lev == L) {
                            // the SPLIT threads of a task read the byte before any of
                            // them writes (the shuffles order them), then all write
                            // the same combined value
                            const uint32_t xb0 = spc[8u * v];
                            uint32_t f = ws_task<MODE>(rb + 4 * off, spc, v, rp, drow, lut, tab, H, beta, th);
                            if constexpr (SPLIT >= 2) {
                                const unsigned pm = ((1u << SPLIT) - 1u) << (tid & 31 & ~(SPLIT - 1));
                                f |= __shfl_xor_sync(pm, f, 1);
                                if constexpr (SPLIT >= 4) f |= __shfl_xor_sync(pm, f, 2);
                            }
                            spc[8u * v] = (uint8_t)(xb0 ^ f);
                        }
                        bar_sync(kBarCons, 32 * NC);
                    }
                    bar_arrive(kBarEmpty0 + b, NT);
                    if (eown) {
#pragma unroll
                        for (int i = 0; i < kWin; i++) {
                            if (w * kWin + i < d.n) {
                                const uint64_t* dr = deb + (i * 8 + el) * kRS;
                                if constexpr (MODE == kModeInt) E += (int32_t) reinterpret_cast<const int64_t*>(dr)[ek];
                                else E = __dadd_rn(E, reinterpret_cast<const double*>(dr)[ek]);
                            }
                        }
                    }
                    bar_sync(kBarCons, 32 * NC);
                }
                cp_async_wait0();
                if constexpr (MODE == kModeF64) {
                    if (!R.cells && (P.base + s + 1) % kResyncEvery == 0) {
                        bar_sync(kBarCons, 32 * NC);
                        if (eown) {
                            double e8[8];
                            energies_f64_sp(A, d, reinterpret_cast<const uint8_t*>(sw) + el, e8);
                            double vv = e8[0];
#pragma unroll
                            for (int k = 0; k < 8; k++)
                                if (k == ek) vv = e8[k];
                            E = vv;
                        }
                    }
                }
            }
        }
        __syncthreads();
        if (!GSP) {
            uint64_t* gwo = A.spins + d.spin;
            for (uint32_t i = tid; i < d.n; i += NT) gwo[i] = sw[i];
        }
        if (eown) {
            const size_t o = d.energy + el + 8 * ek;
            if constexpr (MODE == kModeInt) A.Ei[o] = E;
            else A.Ef[o] = E;
        }
        if (tid == 0 && !R.cells) {
            A.pos[d.owner] = pos0 + P.steps;
            A.deo[d.owner] ^= (int32_t)(exchanges_in(P.base, P.steps, R.exchange_interval) & 1u);
            if (R.serve) A.done[d.owner] = P.base + P.steps;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// PT kernel: one CTA per instance, thread (cell c, lane l) = threadIdx.x.
// Runs R.steps steps of engine::step: base_seed draw, sweep of every cell,
// and every exchange_interval-th step the DEO exchange (engine.rs:713-789)
// decided by warp 0 with ballots for the draw positions and applied as a
// masked XOR swap of whole configurations by the whole CTA.
// Shared memory: [nt][tab_stride] thresholds | [nt][64] energies (f64) |
// [nt] swap masks | master position.
// ---------------------------------------------------------------------------
template <uint32_t MODE>
__global__ void __launch_bounds__(1024) pt_kernel(DevArrays A, RunArgs R, uint32_t inst0, int tab_stride) {
    extern __shared__ uint64_t smem[];
    const uint32_t inst = inst0 + blockIdx.x;
    const InstDesc d = A.desc[inst];
    const int nt = (int)d.nt;
    const int tid = threadIdx.x;
    const int lane = tid & 7;
    const int c = tid >> 3;
    const bool active = c < nt;
    const unsigned gmask = group_mask(tid);
    uint64_t* tab = smem + (size_t)c * tab_stride;
    double* Es = reinterpret_cast<double*>(smem + (size_t)nt * tab_stride);
    uint64_t* masks = reinterpret_cast<uint64_t*>(Es + (size_t)nt * kReplicas);
    uint64_t* spos = masks + nt;
    uint64_t* words = A.spins + d.spin;
    uint32_t key[8];
#pragma unroll
    for (int i = 0; i < 8; i++) key[i] = A.keys[8 * (size_t)inst + i];
    uint64_t pos = A.pos[inst];
    int deo = A.deo[inst];
    typedef typename std::conditional<MODE == kModeInt, int32_t, double>::type EType;
    EType E[8];
    if (active) {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            if constexpr (MODE == kModeInt) E[k] = A.Ei[d.energy + (size_t)c * kReplicas + lane + 8 * k];
            else E[k] = A.Ef[d.energy + (size_t)c * kReplicas + lane + 8 * k];
        }
    }
    const int ts = 2 * d.H + 1;
    for (uint32_t s = 0; s < R.steps; s++) {
        const double* T = R.temps + (R.temps_per_step ? (size_t)s * nt : 0);
        const uint64_t base = chacha8_draw(key, pos);
        pos += 1;
        if (active) {
            const double beta = __ddiv_rn(1.0, T[c]);
            uint64_t* cw = words + (size_t)c * d.n;
            if constexpr (MODE == kModeInt) {
                __syncwarp(gmask);
                for (int i = lane; i < ts; i += 8) tab[i] = metropolis_threshold(i - d.H, beta);
                __syncwarp(gmask);
                sweep_int(A, d, cw, lane, tab, base + (uint64_t)c, E);
            } else {
                sweep_f64(A, d, cw, lane, beta, base + (uint64_t)c, E);
            }
        }
        const uint64_t g = R.step_base + s + 1;
        if (g % R.exchange_interval == 0) {
            if (nt > 1) {
                __syncthreads();
                if (active) {
#pragma unroll
                    for (int k = 0; k < 8; k++) Es[c * kReplicas + lane + 8 * k] = (double)E[k];
                }
                for (int t = tid; t < nt; t += blockDim.x) masks[t] = 0;
                __syncthreads();
                if (tid < 32) {
                    uint64_t p = pos;
                    const unsigned lt = (1u << tid) - 1u;
                    for (int t = deo; t + 1 < nt; t += 2) {
                        const double db = R.dbeta[t];
                        const double dea = __dsub_rn(Es[t * kReplicas + tid], Es[(t + 1) * kReplicas + tid]);
                        const double deb = __dsub_rn(Es[t * kReplicas + tid + 32], Es[(t + 1) * kReplicas + tid + 32]);
                        const double exa = __dmul_rn(db, dea);
                        const double exb = __dmul_rn(db, deb);
                        const bool na = exa < 0.0, nb = exb < 0.0;
                        const unsigned ma = __ballot_sync(0xffffffffu, na);
                        const unsigned mb = __ballot_sync(0xffffffffu, nb);
                        bool aa = !na, ab = !nb;
                        if (na) {
                            const uint64_t m = chacha8_draw(key, p + __popc(ma & lt)) >> 11;
                            if constexpr (MODE == kModeInt) {
                                const uint64_t ad = (uint64_t)fabs(dea);
                                const uint64_t th = ad <= R.xdmax[t] ? R.xtab[R.xoff[t] + ad - 1]
                                                                     : (ad <= R.xdund[t] ? 1ULL : 0ULL);
                                aa = m < th;
                            } else {
                                aa = __dmul_rn((double)m, 1.1102230246251565e-16) < exp(exa);
                            }
                        }
                        if (nb) {
                            const uint64_t m = chacha8_draw(key, p + __popc(ma) + __popc(mb & lt)) >> 11;
                            if constexpr (MODE == kModeInt) {
                                const uint64_t ad = (uint64_t)fabs(deb);
                                const uint64_t th = ad <= R.xdmax[t] ? R.xtab[R.xoff[t] + ad - 1]
                                                                     : (ad <= R.xdund[t] ? 1ULL : 0ULL);
                                ab = m < th;
                            } else {
                                ab = __dmul_rn((double)m, 1.1102230246251565e-16) < exp(exb);
                            }
                        }
                        p += (uint64_t)(__popc(ma) + __popc(mb));
                        const unsigned Aa = __ballot_sync(0xffffffffu, aa);
                        const unsigned Ab = __ballot_sync(0xffffffffu, ab);
                        if (aa) {
                            const double tmp = Es[t * kReplicas + tid];
                            Es[t * kReplicas + tid] = Es[(t + 1) * kReplicas + tid];
                            Es[(t + 1) * kReplicas + tid] = tmp;
                        }
                        if (ab) {
                            const double tmp = Es[t * kReplicas + tid + 32];
                            Es[t * kReplicas + tid + 32] = Es[(t + 1) * kReplicas + tid + 32];
                            Es[(t + 1) * kReplicas + tid + 32] = tmp;
                        }
                        if (tid == 0) {
                            masks[t] = (uint64_t)Aa | ((uint64_t)Ab << 32);
                            A.att[d.stat + t] += kReplicas;
                            A.acc[d.stat + t] += (uint64_t)(__popc(Aa) + __popc(Ab));
                        }
                    }
                    if (tid == 0) *spos = p;
                }
                __syncthreads();
                pos = *spos;
                for (int t = deo; t + 1 < nt; t += 2) {
                    const uint64_t M = masks[t];
                    if (M == 0) continue;
                    const uint64_t LM = transpose8x8(M);
                    uint64_t* w1 = words + (size_t)t * d.n;
                    uint64_t* w2 = words + (size_t)(t + 1) * d.n;
                    for (uint32_t v = tid; v < d.n; v += blockDim.x) {
                        const uint64_t a = w1[v], b = w2[v];
                        const uint64_t dd = (a ^ b) & LM;
                        w1[v] = a ^ dd;
                        w2[v] = b ^ dd;
                    }
                }
                __syncthreads();
                if (active) {
#pragma unroll
                    for (int k = 0; k < 8; k++) E[k] = (EType)Es[c * kReplicas + lane + 8 * k];
                }
            }
            deo ^= 1;
        }
        if constexpr (MODE == kModeF64) {
            if (g % kResyncEvery == 0) {
                if (nt > 1) __syncthreads();  // swaps by other threads are visible
                if (active) energies_f64(A, d, words + (size_t)c * d.n, lane, E);
            }
        }
    }
    if (active) {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            if constexpr (MODE == kModeInt) A.Ei[d.energy + (size_t)c * kReplicas + lane + 8 * k] = E[k];
            else A.Ef[d.energy + (size_t)c * kReplicas + lane + 8 * k] = E[k];
        }
    }
    if (tid == 0) {
        A.pos[inst] = pos;
        A.deo[inst] = deo;
    }
}

template __global__ void pt_kernel<kModeInt>(DevArrays, RunArgs, uint32_t, int);
template __global__ void pt_kernel<kModeF64>(DevArrays, RunArgs, uint32_t, int);

// ---------------------------------------------------------------------------
// Exchange step of PT cells run as separate work items (engine.rs:713-789),
// one warp per instance. The sweep launch before it ran `steps` steps whose
// base seeds were draws pos .. pos + steps - 1. On an exchange step the DEO
// pairs of the current parity are decided from the cells' tracked energies
// with draws from pos + steps on (ballots give each replica's draw position),
// energies are swapped in place and each pair's swap mask (0 for pairs not
// exchanged) goes to A.xmask for swap_kernel; the phase toggles. Otherwise
// only the stream position advances. With populations (RunArgs::pop_len) the
// populations' pairs are decided in population order (engine.rs:714-716).
// ---------------------------------------------------------------------------
template <uint32_t MODE>
__global__ void __launch_bounds__(32) exchange_kernel(DevArrays A, RunArgs R, uint32_t steps, uint32_t exchange) {
    const uint32_t inst = blockIdx.x;
    const InstDesc d = A.desc[inst];
    const int nt = (int)d.nt;
    const int tid = threadIdx.x;
    uint32_t key[8];
#pragma unroll
    for (int i = 0; i < 8; i++) key[i] = A.keys[8 * (size_t)inst + i];
    uint64_t p = A.pos[inst] + steps;
    int deo = A.deo[inst];
    auto energy = [&](int t, int r) -> double {
        if constexpr (MODE == kModeInt) return (double)A.Ei[d.energy + (size_t)t * kReplicas + r];
        else return A.Ef[d.energy + (size_t)t * kReplicas + r];
    };
    auto swap_energy = [&](int t, int r) {
        const size_t a = d.energy + (size_t)t * kReplicas + r, b = a + kReplicas;
        if constexpr (MODE == kModeInt) {
            const int32_t x = A.Ei[a];
            A.Ei[a] = A.Ei[b];
            A.Ei[b] = x;
        } else {
            const double x = A.Ef[a];
            A.Ef[a] = A.Ef[b];
            A.Ef[b] = x;
        }
    };
    if (exchange) {
        if (nt > 1) {
            // L cells per population; pairs (c, c + 1) with c = t + L * q
            const int L = R.pop_len ? (int)R.pop_len : nt;
            const int pops = nt / L;
            for (int c = tid; c + 1 < nt; c += 32) {
                const int t = c % L;
                if ((t & 1) != deo || t + 1 >= L) A.xmask[d.stat + c] = 0;
            }
            const unsigned lt = (1u << tid) - 1u;
            for (int q = 0; q < pops; q++)
                for (int t = deo; t + 1 < L; t += 2) {
                    const int c = t + L * q;
                    const double db = R.dbeta[t];
                    const double dea = __dsub_rn(energy(c, tid), energy(c + 1, tid));
                    const double deb = __dsub_rn(energy(c, tid + 32), energy(c + 1, tid + 32));
                    const double exa = __dmul_rn(db, dea);
                    const double exb = __dmul_rn(db, deb);
                    const bool na = exa < 0.0, nb = exb < 0.0;
                    const unsigned ma = __ballot_sync(0xffffffffu, na);
                    const unsigned mb = __ballot_sync(0xffffffffu, nb);
                    bool aa = !na, ab = !nb;
                    if (na) {
                        const uint64_t m = chacha8_draw(key, p + __popc(ma & lt)) >> 11;
                        if constexpr (MODE == kModeInt) {
                            const uint64_t ad = (uint64_t)fabs(dea);
                            const uint64_t th = ad <= R.xdmax[t] ? R.xtab[R.xoff[t] + ad - 1]
                                                                 : (ad <= R.xdund[t] ? 1ULL : 0ULL);
                            aa = m < th;
                        } else {
                            aa = __dmul_rn((double)m, 1.1102230246251565e-16) < exp(exa);
                        }
                    }
                    if (nb) {
                        const uint64_t m = chacha8_draw(key, p + __popc(ma) + __popc(mb & lt)) >> 11;
                        if constexpr (MODE == kModeInt) {
                            const uint64_t ad = (uint64_t)fabs(deb);
                            const uint64_t th = ad <= R.xdmax[t] ? R.xtab[R.xoff[t] + ad - 1]
                                                                 : (ad <= R.xdund[t] ? 1ULL : 0ULL);
                            ab = m < th;
                        } else {
                            ab = __dmul_rn((double)m, 1.1102230246251565e-16) < exp(exb);
                        }
                    }
                    p += (uint64_t)(__popc(ma) + __popc(mb));
                    const unsigned Aa = __ballot_sync(0xffffffffu, aa);
                    const unsigned Ab = __ballot_sync(0xffffffffu, ab);
                    if (aa) swap_energy(c, tid);
                    if (ab) swap_energy(c, tid + 32);
                    if (R.labels) {
                        int8_t* lab = R.labels + d.energy + (size_t)c * kReplicas;
                        if (aa) {
                            const int8_t x = lab[tid];
                            lab[tid] = lab[kReplicas + tid];
                            lab[kReplicas + tid] = x;
                        }
                        if (ab) {
                            const int8_t x = lab[tid + 32];
                            lab[tid + 32] = lab[kReplicas + tid + 32];
                            lab[kReplicas + tid + 32] = x;
                        }
                    }
                    if (tid == 0) {
                        A.xmask[d.stat + c] = (uint64_t)Aa | ((uint64_t)Ab << 32);
                        A.att[d.stat + t] += kReplicas;
                        A.acc[d.stat + t] += (uint64_t)(__popc(Aa) + __popc(Ab));
                    }
                }
            if (R.labels && L >= 2) {
                // the hot end's up-labels complete round trips; relabel both
                // ends, then count labels per ladder position
                for (int q = 0; q < pops; q++) {
                    int8_t* hot = R.labels + d.energy + (size_t)(L * q) * kReplicas;
                    int8_t* cold = R.labels + d.energy + (size_t)(L - 1 + L * q) * kReplicas;
                    const unsigned done = __ballot_sync(0xffffffffu, hot[tid] == 1);
                    const unsigned done2 = __ballot_sync(0xffffffffu, hot[tid + 32] == 1);
                    hot[tid] = -1;
                    hot[tid + 32] = -1;
                    cold[tid] = 1;
                    cold[tid + 32] = 1;
                    __syncwarp();
                    if (tid == 0) R.rt[0] += (unsigned long long)(__popc(done) + __popc(done2));
                    for (int t = 0; t < L; t++) {
                        const int8_t* lab = R.labels + d.energy + (size_t)(t + L * q) * kReplicas;
                        const unsigned up = __ballot_sync(0xffffffffu, lab[tid] == 1);
                        const unsigned up2 = __ballot_sync(0xffffffffu, lab[tid + 32] == 1);
                        const unsigned dn = __ballot_sync(0xffffffffu, lab[tid] == -1);
                        const unsigned dn2 = __ballot_sync(0xffffffffu, lab[tid + 32] == -1);
                        if (tid == 0) {
                            R.rt[1 + t] += (unsigned long long)(__popc(up) + __popc(up2));
                            R.rt[1 + L + t] += (unsigned long long)(__popc(dn) + __popc(dn2));
                        }
                    }
                    __syncwarp();
                }
            }
        }
        deo ^= 1;
    }
    if (tid == 0) {
        A.pos[inst] = p;
        A.deo[inst] = deo;
    }
}

template __global__ void exchange_kernel<kModeInt>(DevArrays, RunArgs, uint32_t, uint32_t);
template __global__ void exchange_kernel<kModeF64>(DevArrays, RunArgs, uint32_t, uint32_t);

// Masked swap of whole configurations for the pairs exchange_kernel decided
// (engine.rs:751-769): words of cells t and t+1 exchange the bits of the
// swapped replicas.
__global__ void swap_kernel(DevArrays A, uint32_t inst) {
    const InstDesc d = A.desc[inst];
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (uint32_t t = 0; t + 1 < d.nt; t++) {
        const uint64_t M = A.xmask[d.stat + t];
        if (M == 0) continue;
        const uint64_t LM = transpose8x8(M);
        uint64_t* w1 = A.spins + d.spin + (size_t)t * d.n;
        uint64_t* w2 = w1 + d.n;
        for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < d.n; v += stride) {
            const uint64_t a = w1[v], b = w2[v];
            const uint64_t dd = (a ^ b) & LM;
            w1[v] = a ^ dd;
            w2[v] = b ^ dd;
        }
    }
}

// apply_resample (population_annealing.rs:240-287) on the device: member
// (population q, replica r) of every level takes the configuration and tracked
// energies of member parents[64 q + r], read from copies taken before.
// Replica r sits at bit 8 (r % 8) + r / 8 of a lane-major spin word.
template <uint32_t MODE>
__global__ void resample_kernel(DevArrays A, uint32_t inst, uint32_t pop_len, const uint32_t* parents,
                                const uint64_t* old_spins, const int32_t* old_ei, const double* old_ef) {
    const InstDesc d = A.desc[inst];
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t words = (size_t)d.nt * d.n;
    auto bitpos = [](uint32_t r) { return ((r & 7u) << 3) | (r >> 3); };
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) {
        const uint32_t c = (uint32_t)(i / d.n), v = (uint32_t)(i % d.n);
        const uint32_t t = c % pop_len, q = c / pop_len;
        uint64_t w = 0;
        for (uint32_t r = 0; r < (uint32_t)kReplicas; r++) {
            const uint32_t src = parents[q * kReplicas + r];
            const uint32_t sq = src / kReplicas, sr = src % kReplicas;
            const uint64_t sw = old_spins[(size_t)(t + pop_len * sq) * d.n + v];
            w |= ((sw >> bitpos(sr)) & 1ull) << bitpos(r);
        }
        A.spins[d.spin + i] = w;
    }
    const size_t ne = (size_t)d.nt * kReplicas;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += stride) {
        const uint32_t c = (uint32_t)(i / kReplicas), r = (uint32_t)(i % kReplicas);
        const uint32_t t = c % pop_len, q = c / pop_len;
        const uint32_t src = parents[q * kReplicas + r];
        const size_t o = (size_t)(t + pop_len * (src / kReplicas)) * kReplicas + src % kReplicas;
        if constexpr (MODE == kModeInt) A.Ei[d.energy + i] = old_ei[o];
        else A.Ef[d.energy + i] = old_ef[o];
    }
}

// ---------------------------------------------------------------------------
// Isoenergetic cluster moves (src/solver/icm.rs:91-185) on lane pairs
// (r, r + 32) of every cell of instance `inst`, pair k = 32 * cell + r.
// Pairs touch disjoint lanes, so they are independent except for the
// master-stream draws of their seeds, which follow pair order:
//  icm_count_kernel  one warp per cell, lane r counts pair r's disagreements
//                    (the cell's words are read once, broadcast);
//  icm_draw_kernel   one thread walks the pairs in order and takes each
//                    seed rank with rand's gen_range(0..count) from the
//                    stream (no draw when the replicas agree everywhere);
//  icm_move_kernel   one thread per pair: the rank-th disagreeing site,
//                    the depth-first cluster along the CSR rows, delta_a in
//                    cluster order, the cluster flipped in both lanes
//                    (atomic XOR: other pairs flip other bits of the same
//                    words) and the tracked energies moved by +-delta_a.
// Scratch per concurrent pair: n flag bytes and 2n u32 (stack, cluster).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t lane_bit(uint32_t r) { return ((r & 7u) << 3) | (r >> 3); }

__global__ void __launch_bounds__(32) icm_count_kernel(DevArrays A, uint32_t inst, uint32_t* count) {
    const InstDesc d = A.desc[inst];
    const uint32_t c = blockIdx.x, r = threadIdx.x;
    const uint64_t* w = A.spins + d.spin + (size_t)c * d.n;
    const uint32_t pa = lane_bit(r), pb = lane_bit(r + 32);
    uint32_t k = 0;
    for (uint32_t v = 0; v < d.n; v++) {
        const uint64_t x = w[v];
        k += (uint32_t)(((x >> pa) ^ (x >> pb)) & 1ull);
    }
    count[(size_t)c * 32 + r] = k;
}

__global__ void icm_draw_kernel(DevArrays A, uint32_t inst, const uint32_t* count, uint32_t* rank) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const InstDesc d = A.desc[inst];
    uint32_t key[8];
#pragma unroll
    for (int i = 0; i < 8; i++) key[i] = A.keys[8 * (size_t)inst + i];
    uint64_t pos = A.pos[inst];
    const uint32_t pairs = d.nt * 32u;
    for (uint32_t k = 0; k < pairs; k++) {
        const uint32_t m = count[k];
        if (m == 0) {
            rank[k] = 0xFFFFFFFFu;
            continue;
        }
        // rand 0.8.5 sample_single_inclusive(0, m - 1): zone = (m << lz(m)) - 1
        const uint64_t range = m;
        const uint64_t zone = (range << __clzll((long long)range)) - 1;
        for (;;) {
            const uint64_t v = chacha8_draw(key, pos++);
            if (v * range <= zone) {
                rank[k] = (uint32_t)__umul64hi(v, range);
                break;
            }
        }
    }
    A.pos[inst] = pos;
}

template <uint32_t MODE>
__global__ void __launch_bounds__(64) icm_move_kernel(DevArrays A, uint32_t inst, const uint32_t* rank, uint8_t* flags,
                                                      uint32_t* stack, uint32_t slots) {
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= slots) return;
    const InstDesc d = A.desc[inst];
    const uint32_t n = d.n;
    const uint32_t* rows = A.rows + d.row;
    const uint32_t* cols = A.cols + d.ent;
    const double* vals = A.vals + d.ent;
    const double* lin = A.lin + d.site;
    uint8_t* fl = flags + (size_t)slot * n;       // bit 0 visited, bit 1 in cluster
    uint32_t* st = stack + (size_t)slot * 2 * n;  // [0, n) stack, [n, 2n) cluster
    uint32_t* cl = st + n;
    for (uint32_t k = slot; k < d.nt * 32u; k += slots) {
        const uint32_t seed_rank = rank[k];
        if (seed_rank == 0xFFFFFFFFu) continue;
        const uint32_t c = k / 32, a = k % 32, b = a + 32;
        const uint32_t pa = lane_bit(a), pb = lane_bit(b);
        unsigned long long* w = reinterpret_cast<unsigned long long*>(A.spins + d.spin + (size_t)c * n);
        uint32_t seed = 0, seen = 0;
        for (uint32_t v = 0; v < n; v++) {
            const uint64_t x = w[v];
            const bool dis = ((x >> pa) ^ (x >> pb)) & 1ull;
            fl[v] = dis ? 0 : 1;
            if (dis) {
                if (seen == seed_rank) seed = v;
                seen++;
            }
        }
        uint32_t sp = 0, nc = 0;
        st[sp++] = seed;
        fl[seed] = 3;
        while (sp) {
            const uint32_t i = st[--sp];
            cl[nc++] = i;
            for (uint32_t e = rows[i]; e < rows[i + 1]; e++) {
                const uint32_t j = cols[e];
                if (!(fl[j] & 1)) {
                    fl[j] = 3;
                    st[sp++] = j;
                }
            }
        }
        // icm.rs:55-89 in cluster order; every product is by 0 or +-1 (exact)
        double delta = 0.0;
        for (uint32_t q = 0; q < nc; q++) {
            const uint32_t i = cl[q];
            const double xi = (double)((w[i] >> pa) & 1ull);
            delta = __dadd_rn(delta, __dmul_rn(lin[i], 1.0 - 2.0 * xi));
            for (uint32_t e = rows[i]; e < rows[i + 1]; e++) {
                const uint32_t j = cols[e];
                const double xj = (double)((w[j] >> pa) & 1ull);
                if (fl[j] & 2) {
                    if (i < j) delta = __dadd_rn(delta, __dmul_rn(vals[e], (1.0 - xi) * (1.0 - xj) - xi * xj));
                } else {
                    delta = __dadd_rn(delta, __dmul_rn(__dmul_rn(vals[e], xj), 1.0 - 2.0 * xi));
                }
            }
        }
        const unsigned long long m = (1ull << pa) | (1ull << pb);
        for (uint32_t q = 0; q < nc; q++) atomicXor(w + cl[q], m);
        const size_t ea = d.energy + (size_t)c * kReplicas + a, eb = ea + 32;
        if constexpr (MODE == kModeInt) {
            A.Ei[ea] += (int32_t)delta;
            A.Ei[eb] -= (int32_t)delta;
        } else {
            A.Ef[ea] = __dadd_rn(A.Ef[ea], delta);
            A.Ef[eb] = __dsub_rn(A.Ef[eb], delta);
        }
    }
}

// ---------------------------------------------------------------------------
// Random init (ultimate.rs:248-280): one gen::<u64>() word per unclamped
// (cell, site) in cell-major, site-minor order; clamped sites take their value
// in every replica. One CTA per instance. draw_idx[site] = number of unclamped
// sites before it; unclamped = their total.
// ---------------------------------------------------------------------------
__global__ void init_spins_kernel(DevArrays A, uint32_t inst0, const uint32_t* draw_idx,
                                  const uint32_t* unclamped) {
    const uint32_t inst = inst0 + blockIdx.x;
    const InstDesc d = A.desc[inst];
    uint32_t key[8];
#pragma unroll
    for (int i = 0; i < 8; i++) key[i] = A.keys[8 * (size_t)inst + i];
    const uint64_t pos0 = A.pos[inst];
    const uint64_t U = unclamped[inst];
    const uint64_t total = (uint64_t)d.nt * d.n;
    for (uint64_t i = threadIdx.x; i < total; i += blockDim.x) {
        const uint32_t c = (uint32_t)(i / d.n);
        const uint32_t v = (uint32_t)(i % d.n);
        uint64_t w;
        if (A.clampf[d.site + v]) {
            w = A.clampv[d.site + v] == 1 ? ~0ULL : 0ULL;
        } else {
            w = transpose8x8(chacha8_draw(key, pos0 + (uint64_t)c * U + draw_idx[d.site + v]));
        }
        A.spins[d.spin + i] = w;
    }
    __syncthreads();
    if (threadIdx.x == 0) A.pos[inst] = pos0 + (uint64_t)d.nt * U;
}

// Tracked energies from scratch: one (cell, lane) thread per 8 replicas,
// reference order. Integer mode stores the exact integer value.
__global__ void energy_kernel(DevArrays A, uint32_t inst0) {
    const uint32_t inst = inst0 + blockIdx.x;
    const InstDesc d = A.desc[inst];
    for (uint32_t t = threadIdx.x; t < d.nt * 8u; t += blockDim.x) {
        const uint32_t c = t >> 3, lane = t & 7;
        double E[8];
        energies_f64(A, d, A.spins + d.spin + (size_t)c * d.n, (int)lane, E);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const size_t o = d.energy + (size_t)c * kReplicas + lane + 8 * k;
            if (d.mode == kModeInt) A.Ei[o] = (int32_t)E[k];
            else A.Ef[o] = E[k];
        }
    }
}

// Same recompute into a separate f64 buffer [inst][cell][64] without touching
// the tracked energies (FP64 verification of any mode).
__global__ void energy_check_kernel(DevArrays A, uint32_t inst0, double* out) {
    const uint32_t inst = inst0 + blockIdx.x;
    const InstDesc d = A.desc[inst];
    for (uint32_t t = threadIdx.x; t < d.nt * 8u; t += blockDim.x) {
        const uint32_t c = t >> 3, lane = t & 7;
        double E[8];
        energies_f64(A, d, A.spins + d.spin + (size_t)c * d.n, (int)lane, E);
#pragma unroll
        for (int k = 0; k < 8; k++) out[d.energy + (size_t)c * kReplicas + lane + 8 * k] = E[k];
    }
}

// Model energy (hubo.rs:176-189: offset, then per set variable its linear
// term and half of each set neighbour's coupling, CSR order) of one replica's
// configuration. One thread per (cell, replica); used for the incumbent and
// the final best-replica extraction (ultimate.rs:345-368, 397-430).
__global__ void model_energy_kernel(DevArrays A, uint32_t inst, double offset, double* out) {
    const InstDesc d = A.desc[inst];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.nt * (uint32_t)kReplicas) return;
    const uint32_t c = t >> 6, r = t & 63;
    const uint8_t* sp = reinterpret_cast<const uint8_t*>(A.spins + d.spin + (size_t)c * d.n) + (r & 7);
    const uint32_t bit = r >> 3;
    const uint32_t* rows = A.rows + d.row;
    const uint32_t* cols = A.cols + d.ent;
    const double* vals = A.vals + d.ent;
    const double* lin = A.lin + d.site;
    double e = offset;
    for (uint32_t i = 0; i < d.n; i++) {
        if ((sp[8u * i] >> bit) & 1u) {
            e = __dadd_rn(e, lin[i]);
            for (uint32_t k = rows[i]; k < rows[i + 1]; k++)
                if ((sp[8u * cols[k]] >> bit) & 1u) e = __dadd_rn(e, __dmul_rn(vals[k], 0.5));
        }
    }
    out[t] = e;
}

// Best replica (ultimate.rs:345-368): argmin of the model energies es[count]
// in (cell, replica) order with strict < (lowest index on ties), and that
// replica's configuration as 0/1 bytes. Single CTA.
__global__ void __launch_bounds__(1024) best_extract_kernel(DevArrays A, uint32_t inst, const double* es,
                                                           uint32_t count, int8_t* state, double* best_out,
                                                           int32_t* found_out) {
    __shared__ double sv[32];
    __shared__ uint32_t si[32];
    const InstDesc d = A.desc[inst];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    double bv = inf;
    uint32_t bi = 0xFFFFFFFFu;
    for (uint32_t i = tid; i < count; i += blockDim.x)
        if (es[i] < bv) {
            bv = es[i];
            bi = i;
        }
    for (int o = 16; o; o >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, bv, o);
        const uint32_t oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ov < bv || (ov == bv && oi < bi)) {
            bv = ov;
            bi = oi;
        }
    }
    if (lane == 0) {
        sv[wid] = bv;
        si[wid] = bi;
    }
    __syncthreads();
    if (tid == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); k++)
            if (sv[k] < sv[0] || (sv[k] == sv[0] && si[k] < si[0])) {
                sv[0] = sv[k];
                si[0] = si[k];
            }
        *best_out = sv[0];
        *found_out = sv[0] < inf ? 1 : 0;
    }
    __syncthreads();
    const bool found = sv[0] < inf;
    const uint32_t arg = si[0];
    const uint32_t c = found ? arg >> 6 : 0, r = found ? arg & 63 : 0;
    const uint8_t* sp = reinterpret_cast<const uint8_t*>(A.spins + d.spin + (size_t)c * d.n) + (r & 7);
    for (uint32_t v = tid; v < d.n; v += blockDim.x) state[v] = found ? (int8_t)((sp[8u * v] >> (r >> 3)) & 1u) : 0;
}

// steepest_descent_1opt (local_search.rs:19-57) on one configuration: gains
// g_i = (1 - 2 x_i)(lin_i + sum_j w_ij x_j) in CSR order, then repeatedly the
// steepest improving flip among free variables (g < -1e-12, lowest index on
// ties) with the neighbours' gains updated in CSR order, all in the
// reference's f64 operation order. Single CTA: a block-wide argmin per flip.
__global__ void __launch_bounds__(1024) one_opt_kernel(DevArrays A, uint32_t inst, int8_t* state,
                                                       const uint8_t* clamped, double* gains, double* improvement,
                                                       uint64_t* flips_out, uint64_t max_flips) {
    __shared__ double sv[32];
    __shared__ uint32_t si[32];
    const InstDesc d = A.desc[inst];
    const uint32_t* rows = A.rows + d.row;
    const uint32_t* cols = A.cols + d.ent;
    const double* vals = A.vals + d.ent;
    const double* lin = A.lin + d.site;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    for (uint32_t v = tid; v < d.n; v += blockDim.x) {
        double field = lin[v];
        for (uint32_t e = rows[v]; e < rows[v + 1]; e++) field = __dadd_rn(field, __dmul_rn(vals[e], (double)state[cols[e]]));
        gains[v] = __dmul_rn(1.0 - 2.0 * (double)state[v], field);
    }
    __syncthreads();
    double total = 0.0;
    uint64_t flips = 0;
    for (; flips < max_flips; flips++) {
        double bv = -1e-12;
        uint32_t bi = 0xFFFFFFFFu;
        for (uint32_t v = tid; v < d.n; v += blockDim.x)
            if (!(clamped && clamped[v]) && gains[v] < bv) {
                bv = gains[v];
                bi = v;
            }
        for (int o = 16; o; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, bv, o);
            const uint32_t oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov < bv || (ov == bv && oi < bi)) {
                bv = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            sv[wid] = bv;
            si[wid] = bi;
        }
        __syncthreads();
        if (tid == 0) {
            for (int k = 1; k < nw; k++)
                if (sv[k] < sv[0] || (sv[k] == sv[0] && si[k] < si[0])) {
                    sv[0] = sv[k];
                    si[0] = si[k];
                }
            const uint32_t i = si[0];
            if (i != 0xFFFFFFFFu) {
                const double g = sv[0];
                total = __dsub_rn(total, g);
                const double dir = 1.0 - 2.0 * (double)state[i];
                state[i] = (int8_t)(1 - state[i]);
                gains[i] = -g;
                for (uint32_t e = rows[i]; e < rows[i + 1]; e++) {
                    const uint32_t j = cols[e];
                    gains[j] = __dadd_rn(gains[j], __dmul_rn(__dmul_rn(1.0 - 2.0 * (double)state[j], vals[e]), dir));
                }
            }
        }
        __syncthreads();
        const bool done = si[0] == 0xFFFFFFFFu;
        __syncthreads();
        if (done) break;
    }
    if (tid == 0) {
        *improvement = total;
        *flips_out = flips;
    }
}

// update_incumbent (ultimate.rs:397-430): argmin of the tracked energies in
// (cell, replica) order with strict <, re-scored with the model energy; the
// incumbent changes only on a strict improvement. Single CTA of 64 threads.
__global__ void incumbent_kernel(DevArrays A, uint32_t inst, double offset, double* inc_e,
                                 uint64_t* inc_state, uint32_t n_words) {
    __shared__ double sv[64];
    __shared__ int si[64];
    __shared__ double score;
    __shared__ int argc, argr;
    const InstDesc d = A.desc[inst];
    const int tid = threadIdx.x;
    double best = __longlong_as_double(0x7ff0000000000000LL);
    int bi = 0x7fffffff;
    for (uint32_t t = tid; t < d.nt * (uint32_t)kReplicas; t += 64) {
        const double e = d.mode == kModeInt ? (double)A.Ei[d.energy + t] : A.Ef[d.energy + t];
        if (e < best) {
            best = e;
            bi = (int)t;
        }
    }
    sv[tid] = best;
    si[tid] = bi;
    __syncthreads();
    if (tid == 0) {
        double b = sv[0];
        int i0 = si[0];
        for (int i = 1; i < 64; i++)
            if (sv[i] < b || (sv[i] == b && si[i] < i0)) {
                b = sv[i];
                i0 = si[i];
            }
        argc = -1;
        if (b < __longlong_as_double(0x7ff0000000000000LL)) {
            argc = i0 >> 6;
            argr = i0 & 63;
        }
    }
    __syncthreads();
    if (argc < 0) return;
    const uint8_t* sp = reinterpret_cast<const uint8_t*>(A.spins + d.spin + (size_t)argc * d.n) + (argr & 7);
    const uint32_t bit = argr >> 3;
    if (tid == 0) {
        const uint32_t* rows = A.rows + d.row;
        const uint32_t* cols = A.cols + d.ent;
        const double* vals = A.vals + d.ent;
        const double* lin = A.lin + d.site;
        double e = offset;
        for (uint32_t i = 0; i < d.n; i++) {
            if ((sp[8u * i] >> bit) & 1u) {
                e = __dadd_rn(e, lin[i]);
                for (uint32_t k = rows[i]; k < rows[i + 1]; k++)
                    if ((sp[8u * cols[k]] >> bit) & 1u) e = __dadd_rn(e, __dmul_rn(vals[k], 0.5));
            }
        }
        score = e;
    }
    __syncthreads();
    if (score < *inc_e) {
        // packed incumbent state: bit i%64 of word i/64
        for (uint32_t w = tid; w < n_words; w += 64) {
            uint64_t acc = 0;
            for (uint32_t b = 0; b < 64 && 64 * w + b < d.n; b++)
                acc |= (uint64_t)((sp[8u * (64 * w + b)] >> bit) & 1u) << b;
            inc_state[w] = acc;
        }
        __syncthreads();
        if (tid == 0) *inc_e = score;
    }
}

// ---------------------------------------------------------------------------
// Peak probes for the roofline denominators (measured, not part of the path).
// alu_probe: independent chains of 3-input LOP3 / IADD3 on 32-bit registers,
// 16 ops per chain per iteration (8 chains per thread).
// xoshiro_probe: 4 independent Xoshiro256++ lanes per thread, each output
// compared against a threshold (the per-attempt work the sweep cannot avoid).
// ---------------------------------------------------------------------------
__global__ void alu_probe_kernel(uint32_t seed, int iters, uint32_t* out) {
    uint32_t a[8], b = seed ^ threadIdx.x, c = seed * 7u + blockIdx.x;
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] = seed + i * 0x9E3779B9u + threadIdx.x;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int r = 0; r < 8; r++) {
#pragma unroll
            for (int i = 0; i < 8; i++) {
                asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(a[i]) : "r"(b), "r"(c));
                asm volatile("add.u32 %0, %0, %1;" : "+r"(a[i]) : "r"(c));
            }
        }
    }
    uint32_t x = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) x ^= a[i];
    if (x == 0x12345678u) out[0] = x;
}

__global__ void xoshiro_probe_kernel(uint64_t seed, int iters, uint64_t thr, uint32_t* out) {
    Xoshiro x[4];
#pragma unroll
    for (int i = 0; i < 4; i++) x[i].seed_lane(seed + blockIdx.x * 1024 + threadIdx.x, i);
    uint32_t acc = 0;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 4; i++) acc += x[i].next() <= thr;
    }
    if (acc == 0xFFFFFFFFu) out[0] = acc;
}

cudaError_t probe_peaks(int sm_count, double* int_ops_per_s, double* xoshiro_per_s) {
    uint32_t* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(uint32_t));
    if (e != cudaSuccess) return e;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = sm_count * 8, threads = 256;
    float best_alu = 1e30f, best_xo = 1e30f;
    const int it_alu = 4096, it_xo = 8192;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(a);
        alu_probe_kernel<<<blocks, threads>>>(1u + rep, it_alu, d);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms;
        cudaEventElapsedTime(&ms, a, b);
        best_alu = ms < best_alu ? ms : best_alu;
        cudaEventRecord(a);
        xoshiro_probe_kernel<<<blocks, threads>>>(7ULL + rep, it_xo, 0x8000000000000000ULL, d);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&ms, a, b);
        best_xo = ms < best_xo ? ms : best_xo;
    }
    e = cudaGetLastError();
    *int_ops_per_s = (double)blocks * threads * it_alu * 8.0 * 16.0 / (best_alu * 1e-3);
    *xoshiro_per_s = (double)blocks * threads * it_xo * 4.0 / (best_xo * 1e-3);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    return e;
}

// ---------------------------------------------------------------------------
// Host-side launch wrappers (declared in ie_launch.h).
// ---------------------------------------------------------------------------
cudaError_t set_smem_limits(size_t pt_bytes) {
    cudaError_t e = cudaFuncSetAttribute(pt_kernel<kModeInt>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pt_bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(pt_kernel<kModeF64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pt_bytes);
}

// The dynamic shared-memory limit of the batched and windowed kernels is set
// to the per-CTA maximum, so occupancy queries for one class never lower the
// limit below another class's launch of the same kernel.
constexpr int kMaxDynSmem = 226 * 1024;  // 227 KB per CTA less room for static shared memory

template <uint32_t MODE, int TPL>
static int occ_of(size_t smem) {
    int n = 0;
    if (smem > (size_t)kMaxDynSmem ||
        cudaFuncSetAttribute(batch_kernel<MODE, TPL>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem) !=
            cudaSuccess)
        return 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<MODE, TPL>, 32, smem) == cudaSuccess ? n : 0;
}

size_t batch_smem(int tpl, uint32_t spin_cap, bool serve) { return batch_smem_bytes(4 / tpl, spin_cap, serve); }

int batch_occupancy(uint32_t mode, int tpl, uint32_t spin_cap, bool serve) {
    const size_t sm = batch_smem(tpl, spin_cap, serve);
    if (mode == kModeInt)
        return tpl == 1 ? occ_of<kModeInt, 1>(sm) : tpl == 2 ? occ_of<kModeInt, 2>(sm) : occ_of<kModeInt, 4>(sm);
    return tpl == 1 ? occ_of<kModeF64, 1>(sm) : tpl == 2 ? occ_of<kModeF64, 2>(sm) : occ_of<kModeF64, 4>(sm);
}

cudaError_t launch_batch(const DevArrays& A, const RunArgs& R, uint32_t mode, int tpl, uint32_t spin_cap, int grid,
                         cudaStream_t st) {
    const size_t sm = batch_smem(tpl, spin_cap, R.serve != 0 || R.cells != 0);
    if (mode == kModeInt) {
        if (tpl == 1) batch_kernel<kModeInt, 1><<<grid, 32, sm, st>>>(A, R, spin_cap);
        else if (tpl == 2) batch_kernel<kModeInt, 2><<<grid, 32, sm, st>>>(A, R, spin_cap);
        else batch_kernel<kModeInt, 4><<<grid, 32, sm, st>>>(A, R, spin_cap);
    } else {
        if (tpl == 1) batch_kernel<kModeF64, 1><<<grid, 32, sm, st>>>(A, R, spin_cap);
        else if (tpl == 2) batch_kernel<kModeF64, 2><<<grid, 32, sm, st>>>(A, R, spin_cap);
        else batch_kernel<kModeF64, 4><<<grid, 32, sm, st>>>(A, R, spin_cap);
    }
    return cudaGetLastError();
}

template <uint32_t MODE, bool GSP>
static int occ_win(size_t smem) {
    int n = 0;
    if (smem > (size_t)kMaxDynSmem ||
        cudaFuncSetAttribute(window_kernel<MODE, GSP>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem) !=
            cudaSuccess)
        return 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, window_kernel<MODE, GSP>, WsCfg<MODE>::THREADS, smem) ==
                   cudaSuccess
               ? n
               : 0;
}

// spin_cap 0: spins stay in global memory
int window_occupancy(uint32_t mode, uint32_t spin_cap) {
    const size_t sm = ws_smem_bytes(spin_cap);
    if (spin_cap == 0) return mode == kModeInt ? occ_win<kModeInt, true>(sm) : occ_win<kModeF64, true>(sm);
    return mode == kModeInt ? occ_win<kModeInt, false>(sm) : occ_win<kModeF64, false>(sm);
}

cudaError_t launch_window(const DevArrays& A, const RunArgs& R, uint32_t mode, uint32_t spin_cap, int grid,
                          cudaStream_t st) {
    const size_t sm = ws_smem_bytes(spin_cap);
    if (spin_cap == 0) {
        if (mode == kModeInt) window_kernel<kModeInt, true><<<grid, WsCfg<kModeInt>::THREADS, sm, st>>>(A, R, 0);
        else window_kernel<kModeF64, true><<<grid, WsCfg<kModeF64>::THREADS, sm, st>>>(A, R, 0);
    } else {
        if (mode == kModeInt) window_kernel<kModeInt, false><<<grid, WsCfg<kModeInt>::THREADS, sm, st>>>(A, R, spin_cap);
        else window_kernel<kModeF64, false><<<grid, WsCfg<kModeF64>::THREADS, sm, st>>>(A, R, spin_cap);
    }
    return cudaGetLastError();
}

template <uint32_t MODE, bool GSP>
static int occ_chain(size_t smem) {
    int n = 0;
    if (smem > (size_t)kMaxDynSmem ||
        cudaFuncSetAttribute(chain_kernel<MODE, GSP>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem) !=
            cudaSuccess)
        return 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, chain_kernel<MODE, GSP>, 64, smem) == cudaSuccess ? n : 0;
}

// spin_cap 0: spins stay in global memory
int chain_occupancy(uint32_t mode, uint32_t spin_cap) {
    const size_t sm = chain_smem_bytes(spin_cap);
    if (spin_cap == 0) return mode == kModeInt ? occ_chain<kModeInt, true>(sm) : occ_chain<kModeF64, true>(sm);
    return mode == kModeInt ? occ_chain<kModeInt, false>(sm) : occ_chain<kModeF64, false>(sm);
}

cudaError_t launch_chain(const DevArrays& A, const RunArgs& R, uint32_t mode, uint32_t spin_cap, int grid,
                         cudaStream_t st) {
    const size_t sm = chain_smem_bytes(spin_cap);
    if (spin_cap == 0) {
        if (mode == kModeInt) chain_kernel<kModeInt, true><<<grid, 64, sm, st>>>(A, R, 0);
        else chain_kernel<kModeF64, true><<<grid, 64, sm, st>>>(A, R, 0);
    } else {
        if (mode == kModeInt) chain_kernel<kModeInt, false><<<grid, 64, sm, st>>>(A, R, spin_cap);
        else chain_kernel<kModeF64, false><<<grid, 64, sm, st>>>(A, R, spin_cap);
    }
    return cudaGetLastError();
}

cudaError_t launch_exchange(const DevArrays& A, const RunArgs& R, uint32_t ninst, uint32_t mode, uint32_t steps,
                            bool exchange, cudaStream_t st) {
    if (mode == kModeInt) exchange_kernel<kModeInt><<<ninst, 32, 0, st>>>(A, R, steps, exchange ? 1u : 0u);
    else exchange_kernel<kModeF64><<<ninst, 32, 0, st>>>(A, R, steps, exchange ? 1u : 0u);
    return cudaGetLastError();
}

cudaError_t launch_swap(const DevArrays& A, uint32_t inst, uint32_t n_words, int sm_count, cudaStream_t st) {
    const int grid = (int)std::min<uint32_t>((n_words + 255) / 256, (uint32_t)(4 * sm_count));
    swap_kernel<<<std::max(grid, 1), 256, 0, st>>>(A, inst);
    return cudaGetLastError();
}

cudaError_t launch_resample(const DevArrays& A, uint32_t inst, uint32_t mode, uint32_t n_words, uint32_t pop_len,
                            const uint32_t* parents, const uint64_t* old_spins, const int32_t* old_ei,
                            const double* old_ef, int sm_count, cudaStream_t st) {
    const int grid = std::max(1, (int)std::min<uint32_t>((n_words + 255) / 256, (uint32_t)(4 * sm_count)));
    if (mode == kModeInt) resample_kernel<kModeInt><<<grid, 256, 0, st>>>(A, inst, pop_len, parents, old_spins, old_ei, old_ef);
    else resample_kernel<kModeF64><<<grid, 256, 0, st>>>(A, inst, pop_len, parents, old_spins, old_ei, old_ef);
    return cudaGetLastError();
}

cudaError_t launch_icm(const DevArrays& A, uint32_t inst, uint32_t mode, uint32_t cells, uint32_t* count,
                       uint32_t* rank, uint8_t* flags, uint32_t* stack, uint32_t slots, cudaStream_t st) {
    icm_count_kernel<<<cells, 32, 0, st>>>(A, inst, count);
    icm_draw_kernel<<<1, 32, 0, st>>>(A, inst, count, rank);
    const int grid = (int)((slots + 63) / 64);
    if (mode == kModeInt) icm_move_kernel<kModeInt><<<grid, 64, 0, st>>>(A, inst, rank, flags, stack, slots);
    else icm_move_kernel<kModeF64><<<grid, 64, 0, st>>>(A, inst, rank, flags, stack, slots);
    return cudaGetLastError();
}

cudaError_t launch_pt(const DevArrays& A, const RunArgs& R, uint32_t inst0, uint32_t ninst, uint32_t mode,
                      int block, int tab_stride, size_t smem, cudaStream_t st) {
    if (mode == kModeInt) pt_kernel<kModeInt><<<ninst, block, smem, st>>>(A, R, inst0, tab_stride);
    else pt_kernel<kModeF64><<<ninst, block, smem, st>>>(A, R, inst0, tab_stride);
    return cudaGetLastError();
}

cudaError_t launch_init(const DevArrays& A, uint32_t inst0, uint32_t ninst, const uint32_t* draw_idx,
                        const uint32_t* unclamped, cudaStream_t st) {
    init_spins_kernel<<<ninst, 256, 0, st>>>(A, inst0, draw_idx, unclamped);
    return cudaGetLastError();
}

cudaError_t launch_energy(const DevArrays& A, uint32_t inst0, uint32_t ninst, cudaStream_t st) {
    energy_kernel<<<ninst, 128, 0, st>>>(A, inst0);
    return cudaGetLastError();
}

cudaError_t launch_energy_check(const DevArrays& A, uint32_t inst0, uint32_t ninst, double* out, cudaStream_t st) {
    energy_check_kernel<<<ninst, 128, 0, st>>>(A, inst0, out);
    return cudaGetLastError();
}

cudaError_t launch_model_energy(const DevArrays& A, uint32_t inst, uint32_t nt, double offset, double* out,
                                cudaStream_t st) {
    const uint32_t total = nt * (uint32_t)kReplicas;
    model_energy_kernel<<<(total + 127) / 128, 128, 0, st>>>(A, inst, offset, out);
    return cudaGetLastError();
}

cudaError_t launch_incumbent(const DevArrays& A, uint32_t inst, double offset, double* inc_e, uint64_t* inc_state,
                             uint32_t n_words, cudaStream_t st) {
    incumbent_kernel<<<1, 64, 0, st>>>(A, inst, offset, inc_e, inc_state, n_words);
    return cudaGetLastError();
}

cudaError_t launch_best_extract(const DevArrays& A, uint32_t inst, const double* es, uint32_t count, int8_t* state,
                                double* best, int32_t* found, cudaStream_t st) {
    best_extract_kernel<<<1, 1024, 0, st>>>(A, inst, es, count, state, best, found);
    return cudaGetLastError();
}

cudaError_t launch_one_opt(const DevArrays& A, uint32_t inst, int8_t* state, const uint8_t* clamped, double* gains,
                           double* improvement, uint64_t* flips, uint64_t max_flips, cudaStream_t st) {
    one_opt_kernel<<<1, 1024, 0, st>>>(A, inst, state, clamped, gains, improvement, flips, max_flips);
    return cudaGetLastError();
}

}  // namespace ie
