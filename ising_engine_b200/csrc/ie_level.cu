// Level kernel: the sweep of a group of instances ("item") by a whole CTA,
// generator phase then decision phase (data model in ie_level.cuh).
//
// Why: the reference's sweep is a chain over sites, and each of a cell's 8
// Xoshiro lanes is a chain over its 8n calls per sweep. Run as such, a few
// threads per instance do dependent work and the SMs idle. Here both chains
// are cut: the lane streams by GF(2) jumps into segments that threads
// generate side by side, the site chain by dependency levels whose sites the
// CTA decides side by side. The values are the reference's, bit for bit: the
// same Xoshiro outputs at the same stream positions, the same neighbour
// values at every decision.
//
// Generator phase: thread (segment, lane) seeds its lane (engine.rs:87-103),
// jumps to the segment's first call and stores the top 32 bits of each output
// at keys[site][lane][call] (lane l's call k at site v is replica l + 8k,
// engine.rs:145-151, 617-621). Decision phase: level by level, thread (site,
// lane) computes dE of its 8 replicas and decides with those 32 bits; the
// decision is certain unless the 32 bits equal the threshold's (probability
// 2^-32 per attempt), in which case the full output is recomputed from the
// lane's seed (lane_output) and decided exactly.
//
// Integer mode: dE by SWAR byte sums (as the batched kernel) and a table of
// the top 32 bits of the thresholds m < ceil(fast_exp(-dE beta) 2^52), m the
// output's 52-bit mantissa (engine.rs:665-666). f64 mode: dE in the
// reference's f64 order (engine.rs:218-271), then u < fast_exp(x) decided by
// an ex2 estimate, the f32 form, or exactly in f64.
//
// Energies are not tracked through the sweep: at the end of a launch (or of a
// request's schedule) they are computed from the spins, integer exactly and
// f64 in the reference's summation order (engine.rs:333-368), which is the
// value the reference's periodic re-sync (ultimate.rs:316-324) takes.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "ie_device.cuh"
#include "ie_kernels.cuh"
#include "ie_level.cuh"
#include "ie_sweep.cuh"

namespace cg = cooperative_groups;

namespace ie {

struct LvlMem {
    const double* temps;
    uint64_t site, spin, energy, pos0, step0;
    uint64_t base[2];  // lane seed base of the sweep in buffer b (two sweeps in flight when overlapped)
    double beta[2];
    uint32_t key[8];
    uint32_t inst, flat, n, steps, tstride, cell, owner, fin;
    uint32_t pmj;  // +-J form: c | degree << 16
};

// Top 32 bits of the integer threshold: accept iff m < T with T =
// ceil(fast_exp(-de beta) 2^52) (metropolis_threshold returns (T << 12) - 1);
// every m whose top 32 bits are below Q = T >> 20 accepts, above it rejects.
// 0xffffffff: every m accepts (dE <= 0, or T = 2^52).
__device__ __forceinline__ uint32_t q_threshold(int de, double beta) {
    if (de <= 0) return 0xFFFFFFFFu;
    const uint64_t U = metropolis_threshold(de, beta);
    if (U == ~0ULL) return 0xFFFFFFFFu;
    return (uint32_t)(((U + 1) >> 12) >> 20);
}

// Output `8 (v - segment start) + k` of the segment of lane `lane` that holds
// site v, recomputed from the lane's seed and the segment's jump.
__device__ __noinline__ uint64_t lane_output(uint64_t base, int lane, uint32_t v, int k, const uint64_t* jpoly) {
    Xoshiro x;
    x.seed_lane(base, lane);
    const uint32_t seg = v / kLvlSeg;
    if (seg) x.jump(jpoly + 4ull * seg);
    const uint32_t skip = 8u * (v - seg * kLvlSeg) + (uint32_t)k;
    for (uint32_t i = 0; i < skip; i++) x.advance();
    return x.next();
}

__device__ __forceinline__ LvlEntry load_entry(const LvlEntry* p) {
    const uint2 u = __ldg(reinterpret_cast<const uint2*>(p));
    return LvlEntry{u.x, u.y};
}

__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// A spin word (+-J form); CG: from L2.
template <bool CG>
__device__ __forceinline__ uint64_t ld_word(const uint64_t* p) {
    if constexpr (CG) return __ldcg(reinterpret_cast<const unsigned long long*>(p));
    else return *p;
}

// A spin byte; CG: from L2 (another CTA of the cluster may have written it).
template <bool CG>
__device__ __forceinline__ uint32_t ld_spin(const uint8_t* p) {
    if constexpr (CG) return __ldcg(p);
    else return *p;
}

__device__ __forceinline__ float ex2_approx(float a) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}

// f64 decision for dE > 0 knowing the top bits of the output: 1 accept,
// -1 reject, 0 undecided (the bits equal the threshold's). The uniform u =
// m 2^-52 lies in [lo 2^-32, (lo + 2^sh) 2^-32), lo = mh with its low sh bits
// cleared. fast_exp(x) >= exp(x) (the alternating Taylor tail is negative) and
// <= 1.054 exp(x) on [-20, 0]; ex2.approx is within 3e-6 of exp here.
// Out of line (the rare case: u within the ex2 bracket): the f32 form of
// fast_exp with its 2^-10 band, then the exact f64 value.
__device__ __noinline__ int f64_decide_slow(double x, uint32_t lo, uint32_t sh, float ulo, float uhi) {
    const float f = fast_exp_f32(__double2float_rn(x));
    if (uhi < __fmul_rn(f, 0.9990234375f)) return 1;
    if (ulo > __fmul_rn(f, 1.0009765625f)) return -1;
    const uint64_t T = (uint64_t)ceil(__dmul_rn(fast_exp_rn(x), 4503599627370496.0));
    const uint64_t mlo = (uint64_t)lo << 20, mhi = ((uint64_t)lo + (1ull << sh)) << 20;
    if (mhi <= T) return 1;
    if (mlo >= T) return -1;
    return 0;
}

__device__ __forceinline__ int f64_decide(double de, double beta, uint32_t mh, uint32_t sh) {
    const double x = __dmul_rn(-de, beta);
    const uint32_t lo = (mh >> sh) << sh;
    const float s32 = 2.3283064365386963e-10f;  // 2^-32
    const float ulo = __fmul_rn(__uint2float_rd(lo), s32);
    const float uhi = __fmul_rn(__fadd_ru(__uint2float_ru(lo), (float)(1u << sh)), s32);
    const float xf = __double2float_rn(fmax(x, -20.0));
    const float ex = ex2_approx(__fmul_rn(xf, 1.4426950408889634f));
    if (uhi <= __fmul_rn(ex, 0.99998f)) return 1;
    if (ulo >= __fmul_rn(ex, 1.0625f)) return -1;
    return f64_decide_slow(x, lo, sh, ulo, uhi);
}

// Exact decisions of the undecided calls (bit k of `ties`): the outputs are
// recomputed and decided as the reference does.
__device__ __noinline__ uint32_t exact_flips_int(uint32_t ties, uint64_t base, int lane, uint32_t v, uint32_t iL,
                                                 uint32_t iH, int H, double beta, const uint64_t* jpoly) {
    uint32_t f = 0;
    for (int k = 0; k < 8; k++) {
        if (!((ties >> k) & 1u)) continue;
        const int idx = (int)(((k < 4 ? iL : iH) >> (8 * (k & 3))) & 0xFFu);
        const uint64_t res = lane_output(base, lane, v, k, jpoly);
        if (res <= metropolis_threshold(idx - H, beta)) f |= 1u << k;
    }
    return f;
}

// x = -dE beta of one undecided call k
__device__ __noinline__ uint32_t exact_flip_f64(uint64_t base, int lane, uint32_t v, int k, double x,
                                                const uint64_t* jpoly) {
    const uint64_t res = lane_output(base, lane, v, k, jpoly);
    return metropolis_exact_f64(x, res >> 12) ? 1u : 0u;
}

// Integer energies of one member (hubo.rs:176-189 restricted to QUBO, each
// edge once from its lower end): thread (site, lane) adds x_v (lin_v +
// sum_{j > v} w x_j) for its 8 replicas, by SWAR byte sums as in the sweep.
template <bool CG>
__device__ __forceinline__ void member_energy_int(const LvlArgs& L, const LvlMem& m, const uint8_t* spb,
                                                  const uint2* lut, int tid, int T, int32_t* sE) {
    int32_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t i = tid; i < 8u * m.n; i += T) {
        const uint32_t v = i >> 3;
        const uint32_t f = m.flat + v;
        const uint32_t xb = ld_spin<CG>(spb + 8u * f);
        if (!xb) continue;
        const uint32_t* rec = L.lrecs + 4ull * __ldg(L.recoff + m.site + v);
        const uint4 hd = __ldg(reinterpret_cast<const uint4*>(rec));
        const uint32_t deg = hd.x & 0x7FFFFFFFu;
        const int lin = (int)hd.z;
        uint32_t aL = 0, aH = 0;
        int nsum = 0;
        const uint4* e4p = reinterpret_cast<const uint4*>(rec + 4);
        for (uint32_t q = 0; q < deg; q += 4) {
            const uint4 e4 = __ldg(e4p + (q >> 2));
            const uint32_t en[4] = {e4.x, e4.y, e4.z, e4.w};
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const uint32_t col = en[e] & 0xFFFFFFu;
                const uint32_t w = (en[e] >> 24) & 0x7Fu;
                if (col > v && w) {
                    const uint2 sv = lut[ld_spin<CG>(spb + 8u * (m.flat + col)) | ((en[e] >> 23) & 0x100u)];
                    aL += w * sv.x;
                    aH += w * sv.y;
                    if (en[e] >> 31) nsum += (int)w;
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 8; k++)
            if ((xb >> k) & 1u) acc[k] += lin + (int)(((k < 4 ? aL : aH) >> (8 * (k & 3))) & 0xFFu) - nsum;
    }
    const int lane = tid & 7;
#pragma unroll
    for (int k = 0; k < 8; k++)
        if (acc[k]) atomicAdd(sE + lane + 8 * k, acc[k]);
}

// f64 energies of one (member, lane): calculate_replica_energies_local
// (engine.rs:333-368) in its order: site order, lin then the CSR entries with
// v < j, each added with one rounding.
template <bool CG>
__device__ void member_energy_f64(const DevArrays& A, const LvlMem& m, const uint8_t* spb, double* out) {
    const InstDesc d = A.desc[m.inst];
    const uint32_t* rows = A.rows + d.row;
    const uint32_t* cols = A.cols + d.ent;
    const double* vals = A.vals + d.ent;
    const double* lin = A.lin + d.site;
    double E[8];
#pragma unroll
    for (int k = 0; k < 8; k++) E[k] = 0.0;
    for (uint32_t v = 0; v < d.n; v++) {
        const uint32_t xb = ld_spin<CG>(spb + 8u * (m.flat + v));
        if (!xb) continue;
        const double wl = lin[v];
#pragma unroll
        for (int k = 0; k < 8; k++)
            if ((xb >> k) & 1u) E[k] = __dadd_rn(E[k], wl);
        for (uint32_t e = rows[v]; e < rows[v + 1]; e++) {
            const uint32_t j = cols[e];
            if (v < j) {
                const uint32_t mk = xb & ld_spin<CG>(spb + 8u * (m.flat + j));
                if (mk) {
                    const double w = vals[e];
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        if ((mk >> k) & 1u) E[k] = __dadd_rn(E[k], w);
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 8; k++) out[8 * k] = E[k];
}

// SPLIT: the item (one member, spins in global memory) is run by a thread
// block cluster; CTA r of C generates and decides the sites of segments s
// with s % C == r, reads spins from L2 and meets the other CTAs at a cluster
// barrier (release / acquire) after every level.
template <uint32_t MODE, bool GSP, bool SPLIT>
// 64 registers: four CTAs of 256 threads per SM; overlapped launches add a
// generator group to the 256 decider threads (at most 384 threads)
__global__ void __maxnreg__(64) level_kernel(DevArrays A, RunArgs R, LvlArgs L) {
    extern __shared__ __align__(16) uint64_t dsm[];
    __shared__ LvlMem ms[kLvlMaxMembers];
    __shared__ uint32_t s_item, s_steps;
    __shared__ int32_t sE[kReplicas];
    const int tid = threadIdx.x;
    const int T = blockDim.x;  // a multiple of 8: thread tid always serves lane tid % 8
    const int lane = tid & 7;
    const bool own_tab = R.serve != 0 || R.cells != 0;
    uint32_t* const tabs = reinterpret_cast<uint32_t*>(dsm);
    uint2* const lut = reinterpret_cast<uint2*>(tabs + (size_t)L.ntab * kLvlTab * (L.ov ? 2u : 1u));
    uint64_t* const ssw = reinterpret_cast<uint64_t*>(lut + (MODE != kModeF64 ? 512 : 0));
    uint64_t* const tabs64 = reinterpret_cast<uint64_t*>(tabs);  // +-J form: thresholds per level
    uint32_t crank = 0, csize = 1;
    if constexpr (SPLIT) {
        crank = cg::this_cluster().block_rank();
        csize = cg::this_cluster().num_blocks();
    }
    // one output buffer per CTA, or per cluster (its CTAs write disjoint segments)
    uint32_t* const kb = L.keybuf + (size_t)(blockIdx.x / csize) * L.keystride;
    if constexpr (MODE != kModeF64) {
        // spread table: entry b (256 + b for a negative coupling, which
        // contributes |w| (1 - x_j)) holds bit k of b (~b) in byte k
        for (int i = tid; i < 512; i += T) {
            const uint32_t b = (i < 256 ? (uint32_t)i : (uint32_t)(i - 256) ^ 0xFFu);
            lut[i] = make_uint2(spread4(b), spread4(b >> 4));
        }
    }
    for (;;) {
        uint32_t it;
        if constexpr (SPLIT) {
            // the cluster's first CTA takes the item, the others read it from
            // its shared memory
            cg::this_cluster().sync();
            if (crank == 0 && tid == 0) {
                const uint32_t q = atomicAdd(L.queue, 1u);
                s_item = q < L.nitems ? L.order[q] : 0xffffffffu;
            }
            cg::this_cluster().sync();
            it = *cg::this_cluster().map_shared_rank(&s_item, 0);
            // every CTA has read the leader's shared memory before the leader
            // can overwrite it or exit
            cg::this_cluster().sync();
        } else {
            __syncthreads();
            if (tid == 0) {
                const uint32_t q = atomicAdd(L.queue, 1u);
                s_item = q < L.nitems ? L.order[q] : 0xffffffffu;
            }
            __syncthreads();
            it = s_item;
        }
        if (it == 0xffffffffu) break;
        const LvlItem I = L.items[it];
        if ((!GSP && I.sites > L.spin_cap) || I.nmem > kLvlMaxMembers || I.nmem == 0 ||
            (own_tab && I.nmem > L.ntab) || (uint64_t)I.sites * 64 > (L.ov ? L.keyhalf : L.keystride) ||
            (GSP && I.nmem != 1) || I.split != csize || (L.ov && !SPLIT && (L.ov % 32 || L.ov >= (uint32_t)T))) {
            if (tid == 0) atomicExch(A.err, 2);  // host sizing error: report, skip the item
            continue;
        }
        if (tid == 0) s_steps = 0;
        __syncthreads();
        for (uint32_t k = tid; k < I.nmem; k += T) {
            const LvlMember mb = L.members[I.mem0 + k];
            const InstDesc d = A.desc[mb.inst];
            // serving: the site budget is per CTA, so a cluster's item gets split times as many steps
            const StepPlan P = step_plan(A, R, d, mb.inst, (I.sites + I.split - 1) / I.split);
            LvlMem& m = ms[k];
            m.temps = P.temps;
            m.tstride = P.tstride;
            m.steps = P.steps;
            m.step0 = P.base;
            m.site = d.site;
            m.spin = d.spin;
            m.energy = d.energy;
            m.n = d.n;
            m.flat = mb.flat;
            m.inst = mb.inst;
            m.pmj = mb.pmj;
            m.cell = d.cell;
            m.owner = d.owner;
            m.pos0 = A.pos[d.owner];
            // energies at the end: every batched / PT launch, a request when
            // its schedule is done
            m.fin = !R.serve || P.base + P.steps >= d.sched_len;
#pragma unroll
            for (int i = 0; i < 8; i++) m.key[i] = A.keys[8 * (size_t)d.owner + i];
            atomicMax(&s_steps, P.steps);
        }
        __syncthreads();
        const uint32_t nsteps = s_steps;
        uint64_t* const sw = GSP ? A.spins + ms[0].spin : ssw;
        uint8_t* const spb = reinterpret_cast<uint8_t*>(sw) + lane;
        if (!GSP) {
            for (uint32_t k = 0; k < I.nmem; k++) {
                const uint64_t* gw = A.spins + ms[k].spin;
                for (uint32_t i = tid; i < ms[k].n; i += T) ssw[ms[k].flat + i] = gw[i];
            }
        }
        // Sweep s uses buffer b = s & 1 when overlapped (L.ov: the generator
        // warps produce sweep s + 1 while the decider warps decide sweep s),
        // else buffer 0. prep: seed bases and betas; tables: thresholds.
        auto prep = [&](uint32_t s, uint32_t b, uint32_t t0, uint32_t TT) {
            for (uint32_t k = t0; k < I.nmem; k += TT) {
                LvlMem& m = ms[k];
                if (s < m.steps) {
                    m.base[b] = chacha8_draw(m.key, m.pos0 + s) + m.cell;
                    m.beta[b] = __ddiv_rn(1.0, m.temps[(size_t)m.tstride * s]);
                }
            }
        };
        auto tables = [&](uint32_t s, uint32_t b, uint32_t t0, uint32_t TT) {
            if constexpr (MODE == kModeInt) {
                const int H = I.H, W = 2 * H + 1;
                const uint32_t nt = own_tab ? I.nmem : 1u;
                uint32_t* const tb = tabs + (size_t)b * L.ntab * kLvlTab;
                for (uint32_t i = t0; i < nt * (uint32_t)W; i += TT) {
                    const uint32_t k = i / (uint32_t)W, idx = i % (uint32_t)W;
                    if (s < ms[k].steps) tb[k * kLvlTab + idx] = q_threshold((int)idx - H, ms[k].beta[b]);
                }
            }
            if constexpr (MODE == kModePmJ) {
                // threshold of dE = c e / 2 for e = 1..15 (the odd e only occur
                // for even c); the full 64-bit form, decided exactly in the generator
                const uint32_t nt = own_tab ? I.nmem : 1u;
                uint64_t* const tb = tabs64 + (size_t)b * L.ntab * (kLvlTab / 2);
                for (uint32_t i = t0; i < nt * 16u; i += TT) {
                    const uint32_t k = i >> 4, e = i & 15u, c = ms[k].pmj & 0xFFFFu;
                    if (s < ms[k].steps && e && (c * e) % 2 == 0)
                        tb[k * (kLvlTab / 2) + e] = metropolis_threshold((int)(c * e / 2), ms[k].beta[b]);
                }
            }
        };
        // generator phase of sweep s into buffer b by threads t0 .. t0 + TT:
        // chain j = (this CTA's segment j / 8, lane j % 8)
        auto generate = [&](uint32_t s, uint32_t b, uint32_t t0, uint32_t TT) {
            uint32_t* const kbb = kb + (size_t)b * L.keyhalf;
            const uint64_t* const tb64 = tabs64 + (size_t)b * L.ntab * (kLvlTab / 2);
            for (uint32_t j = t0;; j += TT) {
                const uint32_t sg = crank + csize * (j >> 3);
                if (sg >= I.nseg) break;
                const uint32_t sd = __ldg(L.segs + I.seg0 + sg);
                const uint32_t slot = sd >> 24, seg = sd & 0xFFFFFFu;
                const LvlMem& m = ms[slot];
                if (s >= m.steps) continue;
                Xoshiro x;
                x.seed_lane(m.base[b], lane);
                if (seg) x.jump(L.jpoly + 4ull * seg);
                const uint32_t v0 = seg * kLvlSeg, v1 = min(m.n, v0 + kLvlSeg);
                if constexpr (MODE == kModePmJ) {
                    // acceptance masks: byte `lane` of word i of the site's row
                    // holds [output <= U(dE of uphill level i + 1)] for the lane's
                    // 8 calls, exactly (engine.rs:665-666)
                    const uint32_t D = m.pmj >> 16, odd = D & 1u, nl = (D + 1) >> 1;
                    const uint64_t* U = tb64 + (own_tab ? slot * (kLvlTab / 2) : 0u);
                    uint64_t ul[4];
#pragma unroll
                    for (int i = 0; i < 4; i++) ul[i] = (uint32_t)i < nl ? U[2 * (i + 1) - odd] : 0ull;
                    uint8_t* out8 = reinterpret_cast<uint8_t*>(kbb + (size_t)(m.flat + v0) * 64) + lane;
                    for (uint32_t v = v0; v < v1; v++) {
                        uint32_t a[4] = {0, 0, 0, 0};
#pragma unroll
                        for (int k = 0; k < 8; k++) {
                            const uint64_t res = x.next();
#pragma unroll
                            for (int i = 0; i < 4; i++) a[i] |= (uint32_t)(res <= ul[i]) << k;
                        }
#pragma unroll
                        for (int i = 0; i < 4; i++)
                            if ((uint32_t)i < nl) out8[8 * i] = (uint8_t)a[i];
                        out8 += 256;
                    }
                } else {
                    uint4* out = reinterpret_cast<uint4*>(kbb + (size_t)(m.flat + v0) * 64 + lane * 8);
                    for (uint32_t v = v0; v < v1; v++) {
                        uint32_t h[8];
#pragma unroll
                        for (int k = 0; k < 8; k++) h[k] = x.next_hi();
                        out[0] = make_uint4(h[0], h[1], h[2], h[3]);
                        out[1] = make_uint4(h[4], h[5], h[6], h[7]);
                        out += 16;
                    }
                }
            }
        };
        // decision phase of sweep s from buffer b by threads t0 .. t0 + TT
        // (thread t0 + i serves lane i % 8), level by level; before each level
        // barrier a thread loads its first entry of the next level and
        // prefetches that site's record and outputs (read-only during the phase)
        auto decide = [&](uint32_t s, uint32_t b, uint32_t t0, uint32_t TT) {
            const uint32_t* const kbb = kb + (size_t)b * L.keyhalf;
            const uint32_t* const tabb = tabs + (size_t)b * L.ntab * kLvlTab;
            const uint32_t dt = (uint32_t)tid - t0;
            const uint32_t sh = L.tie_shift;
            // this CTA's entries of level l: lvloff[lvl0 + l C + r .. + 1]
            const uint32_t* const lo = L.lvloff + I.lvl0 + crank;
            uint32_t e0 = I.nlvl ? __ldg(lo) : 0u, e1 = I.nlvl ? __ldg(lo + 1) : 0u;
            LvlEntry nxt{0, 0};
            for (uint32_t l = 0; l < I.nlvl; l++) {
                // items of high degree (records of several lines): threads
                // without a task on this level bring into L1 the entries of
                // level l + 3 and the records and output rows of level l + 2
                // (whose entries came a level earlier); all are read-only
                // during the phase. (With short records the first task's
                // prefetch before each barrier covers them, and this would only
                // take issue slots from the level's chains.)
                if (I.dmax > 8) {
                    const uint32_t busy = (MODE == kModePmJ ? 1u : 8u) * (e1 - e0);
                    if (dt >= busy && l + 2 < I.nlvl) {
                        const uint32_t stride = TT - busy, q0 = dt - busy;
                        if (l + 3 < I.nlvl) {
                            const uint32_t b0 = __ldg(lo + (l + 3) * csize), b1 = __ldg(lo + (l + 3) * csize + 1);
                            for (uint32_t j = 16u * q0; j < b1 - b0; j += 16u * stride)
                                prefetch_l1(L.entries + I.ent0 + b0 + j);
                        }
                        const uint32_t a0 = __ldg(lo + (l + 2) * csize), a1 = __ldg(lo + (l + 2) * csize + 1);
                        for (uint32_t j = q0; j < a1 - a0; j += stride) {
                            const LvlEntry en = load_entry(L.entries + I.ent0 + a0 + j);
                            prefetch_l1(L.lrecs + 4ull * en.rec);
                            prefetch_l1(L.lrecs + 4ull * en.rec + 32);
                            const uint32_t* kr = kbb + (size_t)(en.site & ((1u << kLvlFlatBits) - 1u)) * 64;
                            prefetch_l1(kr);
                            if (MODE != kModePmJ) prefetch_l1(kr + 32);
                        }
                    }
                }
                if constexpr (MODE == kModePmJ) {
                    // one thread per site, all 64 replicas at once: cnt = number of
                    // neighbours j with x_j ^ (w_j < 0) = 1, kept as 4 bit planes;
                    // dE = (c/2)(2 cnt - D) for x_v = 0 and (c/2)(D - 2 cnt) for
                    // x_v = 1 (|w| = c, lin = -sum w / 2), uphill level i at cnt =
                    // floor(D/2) + i resp. ceil(D/2) - i; flip unless an uphill
                    // level's acceptance bit is clear
                    for (uint32_t i = dt; i < e1 - e0; i += TT) {
                        const LvlEntry en = (i == dt && l) ? nxt : load_entry(L.entries + I.ent0 + e0 + i);
                        const uint32_t slot = en.site >> kLvlFlatBits, f = en.site & ((1u << kLvlFlatBits) - 1u);
                        const LvlMem& m = ms[slot];
                        if (s >= m.steps) continue;
                        const uint32_t* rec = L.lrecs + 4ull * en.rec;
                        const uint32_t D = __ldg(rec) & 0x7FFFFFFFu;
                        const uint64_t xw = ld_word<SPLIT>(sw + f);
                        uint64_t p0 = 0, p1 = 0, p2 = 0, p3 = 0;
                        const uint4* e4p = reinterpret_cast<const uint4*>(rec + 4);
                        for (uint32_t q = 0; q < D; q += 4) {
                            const uint4 e4 = __ldg(e4p + (q >> 2));
                            const uint32_t ev[4] = {e4.x, e4.y, e4.z, e4.w};
#pragma unroll
                            for (int e = 0; e < 4; e++) {
                                if (q + e < D) {
                                    uint64_t b = ld_word<SPLIT>(sw + m.flat + (ev[e] & 0xFFFFFFu));
                                    if (ev[e] >> 31) b = ~b;
                                    uint64_t c = p0 & b;
                                    p0 ^= b;
                                    const uint64_t c1 = p1 & c;
                                    p1 ^= c;
                                    c = p2 & c1;
                                    p2 ^= c1;
                                    p3 ^= c;
                                }
                            }
                        }
                        const uint64_t* A = reinterpret_cast<const uint64_t*>(kbb + (size_t)f * 64);
                        const uint32_t nl = (D + 1) >> 1, hD = D >> 1, cD = (D + 1) >> 1;
                        uint64_t bad = 0;
                        for (uint32_t lv = 1; lv <= nl; lv++) {
                            const uint32_t K0 = hD + lv, K1 = cD - lv;
                            uint64_t eq = ~0ull;
                            const uint64_t pl[4] = {p0, p1, p2, p3};
#pragma unroll
                            for (int b = 0; b < 4; b++) {
                                const uint64_t t = (((K1 >> b) & 1u) ? xw : 0ull) | (((K0 >> b) & 1u) ? ~xw : 0ull);
                                eq &= ~(pl[b] ^ t);
                            }
                            bad |= eq & ~A[lv - 1];
                        }
                        sw[f] = xw ^ ~bad;
                    }
                } else {
                    for (uint32_t i = dt; i < 8u * (e1 - e0); i += TT) {
                        const LvlEntry en = (i == dt && l) ? nxt : load_entry(L.entries + I.ent0 + e0 + (i >> 3));
                        const uint32_t slot = en.site >> kLvlFlatBits, f = en.site & ((1u << kLvlFlatBits) - 1u);
                        const LvlMem& m = ms[slot];
                        if (s >= m.steps) continue;
                        const uint32_t v = f - m.flat;
                        const uint32_t* rec = L.lrecs + 4ull * en.rec;
                        const uint4 hd = __ldg(reinterpret_cast<const uint4*>(rec));
                        const uint32_t deg = hd.x & 0x7FFFFFFFu;
                        const uint32_t fb = m.flat;
                        const uint32_t xb = ld_spin<SPLIT>(spb + 8u * f);
                        const uint4* kp = reinterpret_cast<const uint4*>(kbb + (size_t)f * 64 + lane * 8);
                        uint32_t flips = 0, ties = 0;
                        if constexpr (MODE == kModeInt) {
                            const uint4 k0 = kp[0], k1 = kp[1];
                            const uint32_t mh[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
                            const int lp = (int)hd.y;
                            uint32_t aL = 0, aH = 0;
                            const uint4* e4p = reinterpret_cast<const uint4*>(rec + 4);
                            for (uint32_t q = 0; q < deg; q += 4) {
                                const uint4 e4 = __ldg(e4p + (q >> 2));
                                const uint32_t en[4] = {e4.x, e4.y, e4.z, e4.w};
                                uint32_t li[4];
#pragma unroll
                                for (int e = 0; e < 4; e++)
                                    li[e] = ld_spin<SPLIT>(spb + 8u * (fb + (en[e] & 0xFFFFFFu))) |
                                            ((en[e] >> 23) & 0x100u);
#pragma unroll
                                for (int e = 0; e < 4; e++) {
                                    const uint2 sv = lut[li[e]];
                                    const uint32_t w = (en[e] >> 24) & 0x7Fu;
                                    aL += w * sv.x;
                                    aH += w * sv.y;
                                }
                            }
                            const int H = I.H;
                            const uint32_t cA = (uint32_t)(H + lp) * 0x01010101u;
                            const uint32_t cB = (uint32_t)(H - lp) * 0x01010101u;
                            const uint32_t xL = spread4(xb) * 0xFFu;
                            const uint32_t xH = spread4(xb >> 4) * 0xFFu;
                            // byte k of iL / iH = dE_k + H for replica lane + 8k
                            const uint32_t iL = ((aL + cA) & ~xL) | ((cB - aL) & xL);
                            const uint32_t iH = ((aH + cA) & ~xH) | ((cB - aH) & xH);
                            const uint32_t* tb = tabb + (own_tab ? slot * kLvlTab : 0u);
                            if (sh == 0) {
#pragma unroll
                                for (int k = 0; k < 8; k++) {
                                    const uint32_t qa = mh[k], qb = tb[((k < 4 ? iL : iH) >> (8 * (k & 3))) & 0xFFu];
                                    flips |= (uint32_t)(qa < qb) << k;
                                    ties |= (uint32_t)(qa == qb) << k;
                                }
                            } else {
#pragma unroll
                                for (int k = 0; k < 8; k++) {
                                    const uint32_t idx = ((k < 4 ? iL : iH) >> (8 * (k & 3))) & 0xFFu;
                                    const uint32_t qa = mh[k] >> sh, qb = tb[idx] >> sh;
                                    flips |= (uint32_t)(qa < qb) << k;
                                    ties |= (uint32_t)(qa == qb) << k;
                                }
                            }
                            if (ties) {
                                flips |= exact_flips_int(ties, m.base[b], lane, v, iL, iH, H, m.beta[b], L.jpoly);
                                if (L.exact_count) atomicAdd(L.exact_count, __popc(ties));
                            }
                        } else {
                            const double wl = __hiloint2double((int)hd.w, (int)hd.z);
                            const uint32_t deg4 = (deg + 3u) & ~3u;
                            const uint4* c4p = reinterpret_cast<const uint4*>(rec + 4);
                            const double2* w2p = reinterpret_cast<const double2*>(rec + 4 + deg4);
                            // dE_k = s_k (lin + sum of w over the neighbours with x_j = 1, in
                            // CSR order), s_k = 1 - 2 x_v: the reference adds w ((x_j ^ x_v) -
                            // x_v) = s_k w or a zero term, and round-to-nearest is symmetric
                            // (fl(-a - b) = -fl(a + b)), so the sum of signed terms is s_k
                            // times the sum of the weights; zero terms change no nonzero sum.
                            // the outputs are read after the sum (fewer live registers), from L1
                            prefetch_l1(kp);
                            double dl[8];
#pragma unroll
                            for (int k = 0; k < 8; k++) dl[k] = wl;
                            for (uint32_t q = 0; q < deg; q += 4) {
                                const uint4 c4 = __ldg(c4p + (q >> 2));
                                const double2 w01 = __ldg(w2p + (q >> 1));
                                const double2 w23 = __ldg(w2p + (q >> 1) + 1);
                                const uint32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
                                const double ww[4] = {w01.x, w01.y, w23.x, w23.y};
                                uint32_t bj[4];
#pragma unroll
                                for (int e = 0; e < 4; e++) bj[e] = ld_spin<SPLIT>(spb + 8u * (fb + cc[e]));
                                // branch-free: a clear bit (or a padding entry, w = 0) adds +0.0,
                                // which leaves every sum but -0.0 unchanged, and -0.0 and +0.0
                                // take the same decision (dE <= 0 accepts)
#pragma unroll
                                for (int e = 0; e < 4; e++) {
#pragma unroll
                                    for (int k = 0; k < 8; k++)
                                        dl[k] = __dadd_rn(dl[k], ((bj[e] >> k) & 1u) ? ww[e] : 0.0);
                                }
                            }
                            const uint4 k0 = kp[0], k1 = kp[1];
                            const uint32_t mh[8] = {k0.x, k0.y, k0.z, k0.w, k1.x, k1.y, k1.z, k1.w};
#pragma unroll
                            for (int k = 0; k < 8; k++) {
                                if ((xb >> k) & 1u) dl[k] = -dl[k];
                                if (dl[k] <= 0.0) {
                                    flips |= 1u << k;
                                    continue;
                                }
                                const int r = f64_decide(dl[k], m.beta[b], mh[k], sh);
                                flips |= (uint32_t)(r > 0) << k;
                                ties |= (uint32_t)(r == 0) << k;
                            }
                            if (ties) {
#pragma unroll
                                for (int k = 0; k < 8; k++)
                                    if ((ties >> k) & 1u)
                                        flips |= exact_flip_f64(m.base[b], lane, v, k, __dmul_rn(-dl[k], m.beta[b]),
                                                                L.jpoly)
                                                 << k;
                                if (L.exact_count) atomicAdd(L.exact_count, __popc(ties));
                            }
                        }
                        spb[8u * f] = (uint8_t)(xb ^ flips);
                    }
                }
                if (l + 1 < I.nlvl) {
                    e0 = __ldg(lo + (l + 1) * csize);
                    e1 = __ldg(lo + (l + 1) * csize + 1);
                    if (MODE != kModePmJ && dt < 8u * (e1 - e0)) {
                        nxt = load_entry(L.entries + I.ent0 + e0 + (dt >> 3));
                        prefetch_l1(L.lrecs + 4ull * nxt.rec);
                        prefetch_l1(kbb + (size_t)(nxt.site & ((1u << kLvlFlatBits) - 1u)) * 64 + lane * 8);
                    }
                    if (MODE == kModePmJ && dt < e1 - e0) {
                        nxt = load_entry(L.entries + I.ent0 + e0 + dt);
                        prefetch_l1(L.lrecs + 4ull * nxt.rec);
                        prefetch_l1(kbb + (size_t)(nxt.site & ((1u << kLvlFlatBits) - 1u)) * 64);
                    }
                }
                if constexpr (SPLIT) {
                    cg::this_cluster().sync();
                } else {
                    if (TT == (uint32_t)T) __syncthreads();
                    else asm volatile("bar.sync 1, %0;" ::"r"(TT) : "memory");
                }
            }
        };
        // the sweeps: overlapped (generator warps t < L.ov one sweep ahead of
        // the decider warps t >= L.ov) or in sequence with every thread on each phase
        const bool ov = L.ov && !SPLIT;
        const long long t_item = clock64();
        if (!ov) {
            for (uint32_t s = 0; s < nsteps; s++) {
                __syncthreads();
                prep(s, 0, tid, T);
                __syncthreads();
                tables(s, 0, tid, T);
                __syncthreads();
                generate(s, 0, tid, T);
                __syncthreads();
                decide(s, 0, 0, T);
            }
        } else if (nsteps) {
            const uint32_t gn = L.ov, dn = (uint32_t)T - L.ov;
            __syncthreads();
            prep(0, 0, tid, T);
            __syncthreads();
            tables(0, 0, tid, T);
            __syncthreads();
            generate(0, 0, tid, T);
            for (uint32_t s = 0; s < nsteps; s++) {
                // sweep s's outputs, tables and bases are complete; buffer
                // (s + 1) & 1 is free (sweep s - 1 is decided)
                __syncthreads();
                const uint32_t nb = (s + 1) & 1u;
                if ((uint32_t)tid < gn) {
                    if (s + 1 < nsteps) {
                        prep(s + 1, nb, tid, gn);
                        asm volatile("bar.sync 2, %0;" ::"r"(gn) : "memory");
                        tables(s + 1, nb, tid, gn);
                        asm volatile("bar.sync 2, %0;" ::"r"(gn) : "memory");
                        generate(s + 1, nb, tid, gn);
                    }
                } else {
                    decide(s, s & 1u, gn, dn);
                }
            }
        }
        if constexpr (SPLIT) {
            // every CTA's last level is done; the first CTA finishes the item
            cg::this_cluster().sync();
            if (crank != 0) continue;
        }
        // serving: the item's cycles per step, for the host's next plan
        if (R.serve && R.cost && tid == 0 && nsteps) {
            const float c = (float)(clock64() - t_item) / (float)nsteps;
            for (uint32_t k = 0; k < I.nmem; k++) R.cost[ms[k].inst] = c;
        }
        __syncthreads();
        // energies, spins and stream state of every member
        for (uint32_t k = 0; k < I.nmem; k++) {
            const LvlMem& m = ms[k];
            if (!m.fin || m.steps == 0) continue;
            if constexpr (MODE != kModeF64) {
                if (tid < kReplicas) sE[tid] = 0;
                __syncthreads();
                member_energy_int<SPLIT>(L, m, spb, lut, tid, T, sE);
                __syncthreads();
                if (tid < kReplicas) A.Ei[m.energy + tid] = sE[tid];
            }
        }
        if constexpr (MODE == kModeF64) {
            for (uint32_t p = tid; p < 8u * I.nmem; p += T) {
                const LvlMem& m = ms[p >> 3];
                if (!m.fin || m.steps == 0) continue;
                member_energy_f64<SPLIT>(A, m, reinterpret_cast<const uint8_t*>(sw) + (p & 7),
                                         A.Ef + m.energy + (p & 7));
            }
        }
        if (!GSP) {
            for (uint32_t k = 0; k < I.nmem; k++) {
                uint64_t* gw = A.spins + ms[k].spin;
                for (uint32_t i = tid; i < ms[k].n; i += T) gw[i] = ssw[ms[k].flat + i];
            }
        }
        if (!R.cells) {
            for (uint32_t k = tid; k < I.nmem; k += T) {
                const LvlMem& m = ms[k];
                A.pos[m.owner] = m.pos0 + m.steps;
                A.deo[m.owner] ^= (int32_t)(exchanges_in(m.step0, m.steps, R.exchange_interval) & 1u);
                if (R.serve) A.done[m.owner] = m.step0 + m.steps;
            }
        }
    }
}

template __global__ void level_kernel<kModeInt, false, false>(DevArrays, RunArgs, LvlArgs);
template __global__ void level_kernel<kModeInt, true, false>(DevArrays, RunArgs, LvlArgs);
template __global__ void level_kernel<kModeInt, true, true>(DevArrays, RunArgs, LvlArgs);
template __global__ void level_kernel<kModeF64, false, false>(DevArrays, RunArgs, LvlArgs);
template __global__ void level_kernel<kModeF64, true, false>(DevArrays, RunArgs, LvlArgs);
template __global__ void level_kernel<kModeF64, true, true>(DevArrays, RunArgs, LvlArgs);
template __global__ void level_kernel<kModePmJ, false, false>(DevArrays, RunArgs, LvlArgs);
template __global__ void level_kernel<kModePmJ, true, false>(DevArrays, RunArgs, LvlArgs);
template __global__ void level_kernel<kModePmJ, true, true>(DevArrays, RunArgs, LvlArgs);

size_t level_smem(uint32_t mode, uint32_t ntab, uint32_t spin_cap, bool ov) {
    return (size_t)ntab * kLvlTab * 4 * (ov ? 2 : 1) + (mode != kModeF64 ? 512 * 8 : 0) + (size_t)spin_cap * 8;
}

template <uint32_t MODE, bool GSP, bool SPLIT>
static void* level_fn() {
    return reinterpret_cast<void*>(level_kernel<MODE, GSP, SPLIT>);
}

static void* level_fn_of(uint32_t mode, bool gsp, bool split) {
    if (mode == kModePmJ)
        return split ? level_fn<kModePmJ, true, true>() : gsp ? level_fn<kModePmJ, true, false>()
                                                              : level_fn<kModePmJ, false, false>();
    if (mode == kModeInt)
        return split ? level_fn<kModeInt, true, true>() : gsp ? level_fn<kModeInt, true, false>()
                                                              : level_fn<kModeInt, false, false>();
    return split ? level_fn<kModeF64, true, true>() : gsp ? level_fn<kModeF64, true, false>()
                                                          : level_fn<kModeF64, false, false>();
}

static cudaLaunchConfig_t level_config(int grid, int threads, size_t smem, cudaStream_t st, uint32_t split,
                                       cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    attr->id = cudaLaunchAttributeClusterDimension;
    attr->val.clusterDim.x = split;
    attr->val.clusterDim.y = 1;
    attr->val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

int level_occupancy(uint32_t mode, bool gsp, int threads, size_t smem) {
    const void* k = level_fn_of(mode, gsp, false);
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess) return 0;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, threads, smem) != cudaSuccess) return 0;
    return occ;
}

int level_clusters(uint32_t mode, int threads, size_t smem, uint32_t split) {
    const void* k = level_fn_of(mode, true, true);
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess) return 0;
    // clusters of 16 CTAs are beyond the portable 8
    if (split > 8 && cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cudaLaunchAttribute attr;
    cudaLaunchConfig_t cfg = level_config((int)split, threads, smem, nullptr, split, &attr);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) != cudaSuccess) return 0;
    return n;
}

cudaError_t launch_level(const DevArrays& A, const RunArgs& R, const LvlArgs& L, uint32_t mode, bool gsp, int threads,
                         int grid, cudaStream_t st, uint32_t split) {
    if (L.ov && split <= 1) threads += (int)L.ov;  // the generator group of an overlapped launch
    const size_t smem = level_smem(mode, L.ntab, gsp ? 0 : L.spin_cap, L.ov != 0);
    if (split > 1) {
        cudaLaunchAttribute attr;
        const cudaLaunchConfig_t cfg = level_config(grid, threads, smem, st, split, &attr);
        if (mode == kModeInt) return cudaLaunchKernelEx(&cfg, level_kernel<kModeInt, true, true>, A, R, L);
        if (mode == kModePmJ) return cudaLaunchKernelEx(&cfg, level_kernel<kModePmJ, true, true>, A, R, L);
        return cudaLaunchKernelEx(&cfg, level_kernel<kModeF64, true, true>, A, R, L);
    }
    if (mode == kModePmJ) {
        if (gsp) level_kernel<kModePmJ, true, false><<<grid, threads, smem, st>>>(A, R, L);
        else level_kernel<kModePmJ, false, false><<<grid, threads, smem, st>>>(A, R, L);
    } else if (mode == kModeInt) {
        if (gsp) level_kernel<kModeInt, true, false><<<grid, threads, smem, st>>>(A, R, L);
        else level_kernel<kModeInt, false, false><<<grid, threads, smem, st>>>(A, R, L);
    } else {
        if (gsp) level_kernel<kModeF64, true, false><<<grid, threads, smem, st>>>(A, R, L);
        else level_kernel<kModeF64, false, false><<<grid, threads, smem, st>>>(A, R, L);
    }
    return cudaGetLastError();
}

}  // namespace ie
