// Device half of ritvec: launchers (ritvec.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
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
void rot_pack(const int32_t* ri, const double* rc, const double* rs, int64_t nrot, int64_t js, double* cs,
              int32_t* il);
void rot_pack(const int32_t* ri, const double* rc, const double* rs, int64_t nrot, int64_t js,
              std::vector<double>& cs, std::vector<int32_t>& il);
// Z (js x js, column-major) = Z0 rotated by the packed rotations, where Z0 is
// I (first) or Z itself: a list may be applied in consecutive pieces (a cut
// between two rotations is exact).
void rot_apply(double* z, int64_t js, const double* cs, const int32_t* il, int64_t nrot, bool first, cudaStream_t s);
// Coefficients of the back-transform for output rows rowk[0..d).
void build_coef(const double* z, int64_t js, const int32_t* perm, const int32_t* rowk, int64_t d, bool legacy,
                double eps_a, double* C, cudaStream_t s);
// Vt (d x n) = C (d x js) Q (js x n), ascending-i unfused accumulation.
void backtransform(const double* C, const double* Q, int64_t js, int64_t n, int64_t d, double* Vt, cudaStream_t s);
// S[r] = sqrt(v_r^T B v_r), Ut[r] = (A v_r) / S[r]  (op1 = A, op2 = A^T in the internal orientation)
void sigma_and_u(const DevCompressed& op1, const DevCompressed& op2, bool fp32, const double* Vt, int64_t d,
                 int64_t n, int64_t m, bool legacy, double eps_a, double* S, double* Ut, cudaStream_t s);

}  // namespace svdb
