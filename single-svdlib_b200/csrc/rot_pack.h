// Packing of imtql2's plane rotations for the device (rot_apply): host code
// only, so that the CPU tests compile the same lines.
#pragma once

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "svdb_internal.h"

namespace svdb {

// Rotations are staged in chunks of kRotChunk; a rotation takes 24 bytes of a
// stage: (c, s) and (index, segment length).
constexpr int kRotChunk = 512;
constexpr int kRotStageBytes = 24;
inline int64_t rot_padded(int64_t nrot) { return std::max<int64_t>(4, (nrot + 3) / 4 * 4); }
// Packs the recorded rotations for rot_apply: cs[2t], cs[2t+1] = c, s of
// rotation t; il[2t] = its index; il[2t+1] = the length of the segment that
// starts at t (0 inside one).  Segments are runs whose index falls by one
// from rotation to rotation, cut at multiples of kRotChunk.  Both lists hold
// 2 * rot_padded(nrot) entries.  Throws SVDB_ERR_LAS2 for an index outside
// [0, js - 2].
inline void rot_pack(const int32_t* ri, const double* rc, const double* rs, int64_t nrot, int64_t js, double* cs,
                     int32_t* il) {
    const int64_t npad = rot_padded(nrot);
    std::fill(cs, cs + 2 * npad, 0.0);
    std::fill(il, il + 2 * npad, 0);
    int64_t start = 0;
    for (int64_t t = 0; t <= nrot; ++t) {
        if (t < nrot) {
            if (ri[t] < 0 || ri[t] > js - 2)
                throw Error(SVDB_ERR_LAS2, "rotation " + std::to_string(t) + " has index " + std::to_string(ri[t]) +
                                               " outside [0, " + std::to_string(js - 2) + "]");
            cs[2 * t] = rc[t];
            cs[2 * t + 1] = rs[t];
            il[2 * t] = ri[t];
        }
        const bool cut = t == nrot || (t > start && (t % kRotChunk == 0 || ri[t] != ri[t - 1] - 1));
        if (cut) {
            il[2 * start + 1] = (int32_t)(t - start);
            start = t;
        }
    }
}

inline void rot_pack(const int32_t* ri, const double* rc, const double* rs, int64_t nrot, int64_t js,
                     std::vector<double>& cs, std::vector<int32_t>& il) {
    cs.resize((size_t)(2 * rot_padded(nrot)));
    il.resize((size_t)(2 * rot_padded(nrot)));
    rot_pack(ri, rc, rs, nrot, js, cs.data(), il.data());
}

}  // namespace svdb
