// Kernel-side data model shared by the host code (ie_engine.cu) and kernels.
#pragma once
#include <cstdint>

namespace ie {

constexpr int kReplicas = 64;
constexpr int kLanes = 8;     // Xoshiro lanes per cell; thread (cell, lane) owns 8 replicas
constexpr int kMaxH = 127;    // integer mode: local fields within [-127, 127]
constexpr int kTabMax = 2 * kMaxH + 1;
constexpr int kResyncEvery = 1000;  // ultimate.rs:316-324

enum Mode : uint32_t { kModeInt = 0, kModeF64 = 1 };

// One instance (problem + its cells). All offsets index the engine-wide arrays.
struct InstDesc {
    uint32_t n;      // sites
    int32_t H;       // integer-mode bound on |local field|
    uint32_t mode;   // Mode
    uint32_t nt;     // cells (temperatures); num_pops = 1
    uint64_t row;    // rows[row .. row+n]: entry offsets relative to `ent`
    uint64_t ent;    // ents[] (int mode) and cols[]/vals[] base
    uint64_t site;   // linp[], lin[], clampf[] base
    uint64_t spin;   // spins[]: cell c word v at spin + c*n + v (lane-major bytes)
    uint64_t energy; // Ei[] / Ef[]: cell c replica r at energy + c*64 + r
    uint64_t stat;   // swap stats base ([nt-1] per instance)
    uint64_t rec;    // site-record stream (batched kernel): recs[rec .. rec + rec_len)
    uint64_t rec_len;
    uint64_t win;    // window table (windowed kernel): wtab[win .. win + kWT * ceil(n / kWin))
    uint64_t wrec;   // windowed kernel's record stream (one record per site): recs[wrec ..)
    uint64_t sched;  // serving: the instance's per-step temperatures at temps[sched .. sched + sched_len)
    uint64_t sched_len;
    uint32_t owner;  // instance whose master key, stream position and DEO phase this entry uses
    uint32_t cell;   // PT cell run as its own work item: Xoshiro seed offset and ladder column
};

// Site-record streams of the batched kernel. Each instance's stream is a
// sequence of chunks of kChunk words (16-byte aligned); records are 16-byte
// aligned, never straddle a chunk, and kRecPad marks "continue at the next
// chunk". A site with more than 16 couplings spans several records, all but
// the last flagged kRecCont; a clamped site is a bare header.
//  integer record: [hdr, 0, 0, 0, e_0 .. e_{d-1}, 0-padding to 4 words],
//                  hdr = d | cont << 14 | clamp << 15 | (linp + 128) << 16,
//                  e = col | |w| << 24 | (w < 0) << 31
//  f64 record:     [hdr, 0, lin (2 words), col_0 .. (padded to a multiple of 4),
//                   w_0 .. (f64, padded to a multiple of 4)], hdr = d | cont << 14 | clamp << 15
constexpr uint32_t kChunk = 128;
constexpr uint32_t kSlots = 3;
constexpr uint32_t kRecPad = 0xFFFFFFFFu;
constexpr uint32_t kRecCont = 1u << 14;
constexpr uint32_t kRecClamp = 1u << 15;
constexpr uint32_t kRecMaxDeg = 16;
constexpr uint32_t kWinMaxDeg = 32;  // windowed kernel: one record of up to 32 couplings per site
// Windowed kernel: windows of kWin consecutive sites; window table entry of
// kWT words: word i < kWin = record position | length << 24 of site i (16-byte
// units in the instance's windowed record stream), words kWin, kWin + 1 = level
// of site i in nibble i % 8 of word kWin + i / 8, word kWin + 2 = largest level.
// kWin may be 8 or 16 (levels fit the nibbles; kWT >= kWin + 3).
constexpr int kWin = 8;
constexpr int kWT = 16;

struct DevArrays {
    const InstDesc* desc;
    const uint32_t* rows;
    const uint32_t* ents;    // int mode: col | (|w| << 24) | (w < 0) << 31
    const int32_t* linp;     // int mode: lin + sum of negative weights of the row
    const uint32_t* cols;    // original CSR (both modes), reference order
    const double* vals;
    const double* lin;
    const uint8_t* clampf;   // 1 = clamped site
    const int8_t* clampv;    // clamp value (0/1)
    const uint32_t* recs;    // site-record streams
    const uint32_t* wtab;    // window tables of the windowed kernel
    const uint32_t* keys;    // master ChaCha8 key [inst][8]
    uint64_t* spins;
    int32_t* Ei;
    double* Ef;
    uint64_t* pos;           // master-stream position (u64 draws) [inst]
    int32_t* deo;            // DEO phase [inst]
    uint64_t* att;           // swap attempts [stat + pair]
    uint64_t* acc;           // swap accepts
    int32_t* err;            // device error word
    uint64_t* done;          // serving: steps of its schedule each instance has executed
    uint64_t* xmask;         // PT cells: swap mask of each pair in the last exchange [stat + pair]
};

// Run parameters of one launch.
struct RunArgs {
    const double* temps;      // [steps][nt] temperatures, or [nt] when temps_per_step == 0
    uint32_t temps_per_step;  // 1: temps advance with the step, 0: constant ladder
    uint32_t steps;
    uint64_t step_base;       // steps already executed (resync and exchange cadence)
    uint32_t exchange_interval;
    // exchange thresholds (int mode): per pair t of the ladder
    const uint64_t* xtab;     // thresholds ceil(exp(db*de) * 2^53) for |de| = 1..dmax[t]
    const uint64_t* xoff;     // [nt-1] offsets into xtab
    const uint64_t* xdmax;    // [nt-1]
    const uint64_t* xdund;    // [nt-1] largest |de| with exp > 0
    const double* dbeta;      // [nt-1] 1/T_t - 1/T_{t+1}
    // batched work queue
    const uint32_t* quads;    // [nquads][4] instance ids (0xffffffff = empty)
    const int32_t* quad_h;    // [nquads] largest H of the quad (integer mode)
    uint32_t nquads;
    uint32_t* queue;          // atomic counter
    // serving: every instance runs its own schedule (InstDesc::sched) from
    // its next unexecuted step (DevArrays::done) for plan[inst] steps in this
    // launch (without a plan: up to max(1, site_budget / n)); the level kernel
    // writes each instance's device cycles per step of its item to cost[inst]
    uint32_t serve;
    uint32_t site_budget;
    const uint32_t* plan;
    float* cost;
    // per-lane kernels: record chunks by 1D bulk copies on mbarriers (else cp.async)
    uint32_t bulk_ring;
    // PT cells: every work item is one cell (InstDesc::owner, ::cell) of a
    // ladder of `ladder` temperatures; the launch runs steps that end at an
    // exchange or resync step at the latest, and leaves the stream position,
    // DEO phase and f64 resync to the exchange step (exchange_kernel)
    uint32_t cells;
    uint32_t ladder;
    // populations (PA-PT): when nonzero, an instance's cells are populations
    // of pop_len consecutive cells (cell t + pop_len * p); the exchange pairs
    // stay inside a population and the exchange tables, dbeta and swap
    // statistics are indexed by the pair t within it
    uint32_t pop_len;
    // round-trip tracking (engine.rs:794-816), on when labels is set: a
    // direction label per (cell, replica) at the energy index, swapped with
    // the replicas; rt[0] completed round trips, rt[1 + t] up-labels and
    // rt[1 + L + t] down-labels counted at ladder position t after each exchange
    int8_t* labels;
    unsigned long long* rt;
    // when set, the launch's step_base is read from device memory (so a
    // captured CUDA graph of the launch stays valid across runs)
    const uint64_t* step_base_dev;
};

}  // namespace ie
