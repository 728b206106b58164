// bph_noalloc_plan.h -- sizing of the allocation-free boundary contraction.
//
// bph_green_contract_noalloc keeps its scratch in a fixed file-scope device
// array: per-tile arrival counters first, then the split-K partial sums
// partials[split][m][b][cos|sin].  This header decides, from the grid alone,
// whether a grid fits and how many splits of the interior the kernel uses.
// Plain C++ with no CUDA dependence, so that the limits are testable on a
// machine without a GPU (tests/test_host_logic_cpp.py).
#pragma once

#include <cstddef>

namespace bph {
namespace noalloc {

constexpr size_t kScratchBytes = size_t(8) << 20;  // the whole array, per device
constexpr size_t kCounterBytes = 64 * 1024;        // up to 16384 (mode, row-group) tiles
constexpr int kRows = 8;                           // boundary rows per CTA
constexpr int kMaxSplits = 16;                     // interior slices reduced in parallel

struct Plan {
    int groups = 0;      // row groups of kRows boundary rows
    size_t tiles = 0;    // (mode, row group) pairs, one arrival counter each
    int nsplit = 0;      // slices of the interior, one partial-sum block each
};

// Partial sums one split needs: mmax * nb * (cos, sin).
inline size_t split_doubles(int mmax, int nb) { return (size_t)mmax * (size_t)nb * 2; }

// Doubles available for partial sums after the counters.
inline size_t partial_capacity() { return (kScratchBytes - kCounterBytes) / sizeof(double); }

// Fills *out and returns true when the grid fits the scratch; false (and
// *out untouched) when its counters or one split's partial sums do not.
inline bool plan(int mmax, int nb, long long np, Plan *out) {
    if (mmax < 1 || nb < 1 || np < 1) return false;
    const int groups = (nb + kRows - 1) / kRows;
    const size_t tiles = (size_t)mmax * (size_t)groups;
    const size_t per_split = split_doubles(mmax, nb);
    if (tiles * sizeof(unsigned int) > kCounterBytes || per_split > partial_capacity()) return false;
    size_t nsplit = partial_capacity() / per_split;
    if (nsplit > (size_t)kMaxSplits) nsplit = kMaxSplits;
    if ((long long)nsplit > np) nsplit = (size_t)np;  // every split owns at least one zone
    out->groups = groups;
    out->tiles = tiles;
    out->nsplit = (int)nsplit;
    return true;
}

}  // namespace noalloc
}  // namespace bph
