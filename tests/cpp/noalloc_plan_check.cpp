// Checks the scratch sizing of the allocation-free contraction
// (bipoly_hydro_b200/csrc/bph_noalloc_plan.h): grids beyond the counter or
// partial-sum capacity are rejected without touching the plan, and the
// split count is clamped to kMaxSplits and to the number of interior zones.
#include <cstdio>

#include "bph_noalloc_plan.h"

namespace {
int failures = 0;
void expect(bool ok, const char *what) {
    if (!ok) {
        std::printf("FAIL: %s\n", what);
        ++failures;
    }
}
}  // namespace

int main() {
    using namespace bph::noalloc;
    Plan p;
    // 130x98x256, isym 2, mmax 30: nb = 224, np = 12288
    expect(plan(30, 224, 12288, &p), "production grid fits");
    expect(p.groups == 28 && p.tiles == 840u, "production grid tiles");
    expect(p.nsplit == kMaxSplits, "split count clamped to kMaxSplits");
    // 5x5 grid: 3x3 = 9 interior zones (odd), nb = 6, mmax 2: nsplit clamped to np
    expect(plan(2, 6, 9, &p), "tiny grid fits");
    expect(p.nsplit == 9, "split count clamped to the interior zone count");
    expect(p.groups == 1 && p.tiles == 2u, "tiny grid tiles");
    // counters: 64 KiB hold 16384 tiles; mmax 64 allows 256 row groups (nb <= 2048)
    expect(plan(64, 2048, 1 << 20, &p), "largest row count within the counters");
    Plan keep;
    keep.groups = -7;
    keep.tiles = 12345;
    keep.nsplit = -3;
    Plan q = keep;
    expect(!plan(64, 2049, 1 << 20, &q), "one row group beyond the counters rejected");
    expect(q.groups == -7 && q.tiles == 12345u && q.nsplit == -3, "rejected plan left untouched");
    // partial sums: one split needs mmax*nb*2 doubles of (8 MiB - 64 KiB)/8 = 1040384
    expect(partial_capacity() == (kScratchBytes - kCounterBytes) / 8, "partial capacity");
    // nb = 8128 at mmax 64: 1040384 doubles exactly, but its 1016 row groups exceed the counters
    expect(!plan(64, 8128, 1 << 20, &q), "rows beyond the counter limit rejected");
    // mmax 2: 16384 tiles allow 8192 row groups (nb <= 65536); one split then
    // needs 262144 doubles, a quarter of the partial capacity (4 splits fit)
    expect(plan(2, 65536, 1 << 24, &p) && p.nsplit == 3, "largest two-mode grid: three splits");
    expect(!plan(2, 65537, 1 << 24, &q), "two-mode grid beyond the counters rejected");
    // whenever the counters fit, one split's partial sums fit too
    for (int mmax = 1; mmax <= 64; ++mmax) {
        const int nb = (int)(kCounterBytes / sizeof(unsigned int) / mmax) * kRows;
        expect(split_doubles(mmax, nb) <= partial_capacity(), "counters bind before the partial sums");
    }
    // degenerate inputs
    expect(!plan(0, 10, 10, &q) && !plan(2, 0, 10, &q) && !plan(2, 10, 0, &q), "empty grid rejected");
    if (failures == 0) std::printf("noalloc plan: all checks passed\n");
    return failures == 0 ? 0 : 1;
}
