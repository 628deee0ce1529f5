// Data model of the level kernel (ie_level.cu), shared with the host code.
//
// The level kernel runs one sweep of a group of instances ("item") in two
// phases. Generator phase: every Xoshiro lane's stream of the sweep is cut
// into segments of kLvlSeg sites (8 * kLvlSeg calls); each segment is one
// thread's chain, started by a GF(2) jump of the lane's seeded state
// (x^(8 kLvlSeg j) mod P(x), P the characteristic polynomial of the
// Xoshiro256 state transition), and the top 32 bits of every output go to a
// per-CTA buffer, row [site][lane][call]. Decision phase: the sites are taken
// level by level, where level(v) = 1 + max level(u) over the unclamped
// neighbours u < v (0 without one). Sites of one level are never neighbours,
// a site's lower neighbours are all on lower levels and its higher
// neighbours on higher ones, so deciding a level's sites in parallel reads
// exactly the spin values the reference's site order reads.
#pragma once
#include <cstdint>

namespace ie {

constexpr uint32_t kLvlSeg = 128;          // sites per generator segment
// Kernel mode of the +-J form (integer couplings of one magnitude c, lin_v =
// -sum_j w_vj / 2, every site of degree D <= 8): bit-sliced decisions, one
// thread per site (the instances' InstDesc mode stays the integer mode).
constexpr uint32_t kModePmJ = 2;
constexpr uint32_t kLvlMaxMembers = 64;    // instances per item
constexpr uint32_t kLvlMaxOwnTables = 16;  // members per item when each has its own threshold table
constexpr uint32_t kLvlFlatBits = 26;      // entry = slot << 26 | flat site index within the item
constexpr uint32_t kLvlTab = 256;          // u32 per threshold table (indices 0 .. 2H <= 254)
constexpr uint32_t kLvlOverlapGen = 128;   // generator threads of an overlapped launch

// One item: members[mem0 .. mem0 + nmem) share a CTA; their spin words are
// laid out one after another (member slot s at flat offset members[s].flat).
struct LvlItem {
    uint32_t mem0, nmem;
    uint32_t ent0;   // entries[ent0 ..]: sites of every level, level-major
    uint32_t lvl0;   // lvloff[lvl0 .. lvl0 + nlvl]: level starts relative to ent0
    uint32_t nlvl;
    uint32_t seg0;   // segs[seg0 .. seg0 + nseg): slot << 24 | segment
    uint32_t nseg;
    uint32_t sites;  // flat spin words of the item
    int32_t H;       // integer mode: largest H of the members
    uint32_t gsp;    // 1: one member whose spins stay in global memory
    uint32_t split;  // CTAs (a cluster) running the item; lvloff holds nlvl * split + 1 offsets,
                     // level l's sites for CTA r (segment % split == r) at [l split + r]
    uint32_t dmax;   // largest site degree of the members
};

struct LvlMember {
    uint32_t inst;  // index into the launch's InstDesc array
    uint32_t flat;  // first flat spin word of the member
    uint32_t pmj;   // +-J form: c | D << 16 (0: not)
};

// One site of a level: slot << 26 | flat site index, and its level record's
// offset in 16-byte units (one load gives both).
struct alignas(8) LvlEntry {
    uint32_t site;
    uint32_t rec;
};

// Level-record stream: one record per site, 16-byte aligned.
//  integer: [deg | clamp << 31, linp, lin, 0, e_0 .. e_{deg-1}, 0-padding to 4],
//           e = col | |w| << 24 | (w < 0) << 31 (padding entries are 0: no effect)
//  f64:     [deg | clamp << 31, 0, lin (2 words), col_0 .. (padded to 4), w_0 .. (f64, padded to 4)]
struct LvlArgs {
    const LvlItem* items;
    const uint32_t* order;     // item ids of this launch, longest first
    uint32_t nitems;
    uint32_t* queue;
    const LvlMember* members;
    const LvlEntry* entries;
    const uint32_t* lvloff;
    const uint32_t* segs;
    const uint64_t* jpoly;     // [j][4]: x^(8 kLvlSeg j) mod P(x), bit i = coefficient of x^i
    const uint32_t* recoff;    // per site (InstDesc::site + v): record offset in 16-byte units
    const uint32_t* lrecs;
    uint32_t* keybuf;          // per CTA: keystride u32 (64 per flat site, twice when overlapped)
    uint64_t keystride;
    // > 0: each CTA overlaps sweeps, its first ov threads generating sweep
    // s + 1 while the others decide sweep s; outputs, thresholds and seeds
    // double-buffered (second output buffer at keyhalf)
    uint32_t ov;
    uint64_t keyhalf;
    uint32_t spin_cap;         // shared-memory spin words per CTA (0: global spins)
    uint32_t ntab;             // threshold tables per CTA (own tables: one per member)
    // Test hook: decisions compare only the top 32 - tie_shift bits of the
    // stored outputs, so the exact path (output recomputed from the lane's
    // seed) runs often; 0 in normal runs.
    uint32_t tie_shift;
    int32_t* exact_count;      // when set: number of decisions taken on the exact path
};

}  // namespace ie
