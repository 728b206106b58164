// Host check of bph_slices.h: the slices of the split-K tensor-core
// contraction cover every zone exactly once, each slice is a whole number of
// chunks, and the chunks of a slice read no zone of another slice.
#include <cstdio>
#include <vector>

#include "bph_slices.h"

static int fails = 0;
#define CHECK(cond, ...)                  \
    do {                                  \
        if (!(cond)) {                    \
            std::printf(__VA_ARGS__);     \
            std::printf("\n");            \
            ++fails;                      \
        }                                 \
    } while (0)

int main() {
    const long long nps[] = {1, 7, 8, 9, 63, 64, 65, 825, 1024, 2999, 4096, 12288, 30000, 49152, 30001, 130 * 98 + 3};
    for (long long np : nps)
        for (int nsplit = 1; nsplit <= 16; ++nsplit)
            for (int chunk : {1, 2, 4, 8}) {
                std::vector<int> seen((size_t)np, 0);
                long long prev_end = 0;
                for (int sp = 0; sp < nsplit; ++sp) {
                    const bph::ZoneSlice s = bph::zone_slice(np, nsplit, sp, chunk);
                    CHECK(s.k_end >= s.k_begin, "np %lld nsplit %d: slice %d reversed", np, nsplit, sp);
                    CHECK(s.z_end <= np, "np %lld: z_end past np", np);
                    if (s.k_end > s.k_begin) {
                        CHECK(s.k_begin % chunk == 0, "np %lld nsplit %d chunk %d: slice %d starts mid-chunk", np,
                              nsplit, chunk, sp);
                        CHECK(8 * s.k_begin == prev_end, "np %lld nsplit %d: gap before slice %d", np, nsplit, sp);
                        prev_end = s.z_end;
                    }
                    // the chunks the kernel issues: zones [8 (k_begin + chunk ch), + 8 chunk), masked by z_end
                    const long long nchunk = (s.k_end - s.k_begin + chunk - 1) / chunk;
                    for (long long ch = 0; ch < nchunk; ++ch)
                        for (long long z = 8 * (s.k_begin + chunk * ch); z < 8 * (s.k_begin + chunk * (ch + 1)); ++z)
                            if (z < s.z_end) ++seen[(size_t)z];
                }
                CHECK(prev_end == np, "np %lld nsplit %d chunk %d: zones end at %lld", np, nsplit, chunk, prev_end);
                for (long long z = 0; z < np; ++z)
                    CHECK(seen[(size_t)z] == 1, "np %lld nsplit %d chunk %d: zone %lld read %d times", np, nsplit,
                          chunk, z, seen[(size_t)z]);
            }
    if (fails) {
        std::printf("%d checks failed\n", fails);
        return 1;
    }
    std::printf("all checks passed\n");
    return 0;
}
