// Host-side builders of the level kernel's data (ie_level.cuh): the Xoshiro
// jump polynomials, the per-site level records, the dependency levels of an
// instance's sites and the items (groups of instances sharing a CTA).
#pragma once
#include <cstdint>
#include <vector>

#include "ie_kernels.cuh"
#include "ie_level.cuh"

namespace ie {

// x^D mod P(x) for the Xoshiro256 state transition (bit i of out[i / 64] is
// the coefficient of x^i); false if P could not be derived.
bool xoshiro_jump_poly(uint64_t steps, uint64_t out[4]);

// Table of x^(8 kLvlSeg j) mod P(x) for j = 0 .. count - 1 (j = 0: 1), 4 words each.
bool xoshiro_segment_polys(uint32_t count, std::vector<uint64_t>& table);

// One instance's CSR as the level kernel reads it.
struct LvlSource {
    uint32_t n = 0;
    uint32_t mode = kModeF64;
    const uint32_t* rows = nullptr;  // n + 1
    const uint32_t* cols = nullptr;
    const double* vals = nullptr;
    const double* lin = nullptr;
    const uint32_t* ents = nullptr;  // integer mode packed entries
    const int32_t* linp = nullptr;   // integer mode
    const uint8_t* clampf = nullptr; // n
};

// Appends the instance's level records (layout in ie_level.cuh) to `recs`
// and writes each site's record offset in 16-byte units (from the start of
// `recs`) to off16[v].
void level_records(const LvlSource& s, std::vector<uint32_t>& recs, uint32_t* off16);

// Dependency levels of the unclamped sites: level(v) = 1 + max level(u) over
// unclamped neighbours u < v (0 without one). sites: the unclamped sites
// ordered by (level, index); off: start of each level in `sites` (depth + 1).
void site_levels(const LvlSource& s, std::vector<uint32_t>& sites, std::vector<uint32_t>& off);

// Items of one launch class: members (indices into the view of InstDesc `D`)
// grouped into items of at most cap spin words and max_mem members (gsp: one
// member per item, spins in global memory). Level lists of member i are
// lv_sites / lv_off of instance D[i].owner; recoff[D[i].site + v] is site v's
// level-record offset. split > 1 (gsp only): each item runs on a cluster of
// split CTAs, CTA r taking the sites of segments s with s % split == r.
// Appends to the item arrays and
// returns the class's item ids ordered longest first.
struct LvlHost {
    std::vector<LvlItem> items;
    std::vector<LvlMember> members;
    std::vector<LvlEntry> entries;
    std::vector<uint32_t> lvloff, segs;
    uint32_t max_segs = 1;  // largest segment count of any member
    void clear() {
        items.clear();
        members.clear();
        entries.clear();
        lvloff.clear();
        segs.clear();
        max_segs = 1;
    }
};
void build_level_items(const std::vector<InstDesc>& D, const std::vector<uint64_t>& nnz_of,
                       const std::vector<uint32_t>& dmax_of, const std::vector<uint32_t>& pmj_of,
                       const std::vector<std::vector<uint32_t>>& lv_sites,
                       const std::vector<std::vector<uint32_t>>& lv_off, const std::vector<uint32_t>& recoff,
                       const std::vector<uint32_t>& mem,
                       bool gsp, uint32_t cap, uint32_t max_mem, uint32_t split, LvlHost& out,
                       std::vector<uint32_t>& order, double& longest);

}  // namespace ie
