// Device half of ritvec: launchers (ritvec.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "rot_pack.h"
#include "svdb_internal.h"

namespace svdb {

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
