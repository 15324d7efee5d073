// CPU check of the record staging plan (peridyn_b200/csrc/pd_stage_plan.h):
// for random stencil slices, simulate the staging copies and verify that
// every lane whose record is in range reads exactly record p0 + off + lane
// from the staged array, inside [0, T).  Prints "ok <cases>" or the first
// failure; exit status 0 on success.
#include <cstdio>
#include <random>
#include <set>

#include "../../peridyn_b200/csrc/pd_stage_plan.h"

int main() {
    std::mt19937_64 rng(12345);
    int cases = 0;
    for (int it = 0; it < 20000; ++it) {
        const int64_t n = 32 * (1 + (int64_t)(rng() % 400));
        const int64_t S = n / 32, s = (int64_t)(rng() % S), p0 = 32 * s;
        // offsets: a lattice-like stencil (row stride R, plane stride P) or random
        std::set<int32_t, std::greater<int32_t>> offs;
        const int kind = (int)(rng() % 3);
        const int32_t R = 5 + (int32_t)(rng() % 60), P = R * (3 + (int32_t)(rng() % 40));
        const int h = 1 + (int)(rng() % 3);
        if (kind < 2) {
            for (int dz = -h; dz <= h; ++dz)
                for (int dy = -h; dy <= h; ++dy)
                    for (int dx = -h; dx <= h; ++dx)
                        if ((dx || dy || dz) && dx * dx + dy * dy + dz * dz <= h * h + (kind ? 1 : 0))
                            offs.insert(dx + R * dy + P * dz);
        } else {
            const int m = 1 + (int)(rng() % 120);
            for (int k = 0; k < m; ++k) offs.insert((int32_t)((int64_t)(rng() % (2 * n)) - n));
        }
        std::vector<int32_t> off(offs.begin(), offs.end());
        std::vector<int32_t> ranges, pos;
        const int64_t T = pd::stage_plan(p0, n, off, ranges, pos);
        // simulate the copies
        std::vector<int64_t> staged;
        for (size_t m = 0; m < ranges.size(); m += 2) {
            if (m > 0 && ranges[m] <= ranges[m - 2] + ranges[m - 1]) {
                std::printf("ranges not disjoint ascending at case %d\n", it);
                return 1;
            }
            for (int32_t i = 0; i < ranges[m + 1]; ++i) staged.push_back(ranges[m] + i);
        }
        if ((int64_t)staged.size() != T || pos.size() != off.size()) {
            std::printf("size mismatch at case %d\n", it);
            return 1;
        }
        for (size_t j = 0; j < off.size(); ++j)
            for (int l = 0; l < 32; ++l) {
                const int64_t rec = p0 + off[j] + l;
                if (rec < 0 || rec >= n) continue;  // such a lane never reads this slot
                const int64_t at = (int64_t)pos[j] + l;
                if (at < 0 || at >= T || staged[at] != rec) {
                    std::printf("case %d slot %zu lane %d: staged[%lld] != %lld\n", it, j, l, (long long)at,
                                (long long)rec);
                    return 1;
                }
            }
        ++cases;
    }
    std::printf("ok %d\n", cases);
    return 0;
}
