// Record staging plan of one stencil slice (host code, shared by the
// runtime layout builder and its CPU test).
//
// The 32 particles p0 .. p0+31 of a stencil slice read, for slot j, the
// records p0 + off[j] + lane.  The plan merges the windows
// [p0 + off[j], p0 + off[j] + 32) (clipped to [0, n)) into ranges of
// consecutive records; staging copies range m to positions base_m ..
// base_m + len_m - 1 of the block's shared array, and pos[j] is the staged
// position of lane 0's record of slot j (lane l reads pos[j] + l).
#pragma once
#include <algorithm>
#include <cstdint>
#include <vector>

namespace pd {

// off: the slice's offsets in descending order (one per slot).  Returns
// the number of staged records T (0 when no window is in range); ranges
// receives (first record, count) pairs and pos one entry per slot.
inline int64_t stage_plan(int64_t p0, int64_t n, const std::vector<int32_t> &off, std::vector<int32_t> &ranges,
                          std::vector<int32_t> &pos) {
    const int64_t W = 32;
    ranges.clear();
    pos.assign(off.size(), 0);
    int64_t cs = 0, ce = 0, T = 0;
    bool open = false;
    for (size_t jj = off.size(); jj-- > 0;) {  // ascending offsets
        // only lanes whose record is in range read the window
        const int64_t a = std::max<int64_t>(0, p0 + off[jj]), b = std::min<int64_t>(n, p0 + off[jj] + W);
        if (b <= a) continue;
        if (open && a <= ce) {
            ce = std::max(ce, b);
            continue;
        }
        if (open) {
            ranges.push_back((int32_t)cs);
            ranges.push_back((int32_t)(ce - cs));
            T += ce - cs;
        }
        cs = a;
        ce = b;
        open = true;
    }
    if (!open) return 0;
    ranges.push_back((int32_t)cs);
    ranges.push_back((int32_t)(ce - cs));
    T += ce - cs;
    // staged position of each slot's lane-0 record (ranges ascend)
    int64_t base = 0;
    size_t m = 0;
    const size_t nr = ranges.size() / 2;
    for (size_t jj = off.size(); jj-- > 0;) {
        const int64_t r0 = p0 + off[jj];
        while (m + 1 < nr && r0 >= (int64_t)ranges[2 * m] + ranges[2 * m + 1]) base += ranges[2 * m + 1], ++m;
        pos[jj] = (int32_t)(base + r0 - ranges[2 * m]);
    }
    return T;
}

}  // namespace pd
