// Host-side launchers of the standalone device operators (ops.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "svdb_internal.h"

namespace svdb {

// lanes per row for a row gather with `avg` entries per row (power of two, 2..32)
int group_for(double avg);

// Y (nmajor x l) = M X with X (nminor x l), row-major (spmm.cu); values FP32
// when fp32 and the FP32 copy exists; accumulation in FP64.
// Instantiated for (double, double), (float, float) and (float, double).
template <typename XT, typename OT>
void spmm_dev(const DevCompressed& m, bool fp32, const XT* X, int l, OT* Y, cudaStream_t s);
// FP32 values and operand, the operand's rows ldx floats apart (a multiple of 32), FP64 output
bool spmm_f32_strided_ok(const DevCompressed& m, int l, int64_t ldx);
void spmm_f32_strided(const DevCompressed& m, const float* X, int l, int64_t ldx, double* Y, cudaStream_t s);
// Raises the error a TMA gather wait of an earlier SpMM recorded (synchronises).
void spmm_tma_check();
// FP32 SpMM by panels of X in shared memory (spmm_panel.cu); the plan is
// built on the first call for a structure.  spmm_panel returns false when the
// plan does not suit the matrix; spmm_panel_check raises a recorded timeout.
bool spmm_panel_eligible(const DevCompressed& m, int l, const void* X);
bool spmm_panel(DevCompressed& m, const float* X, int l, double* Y, cudaStream_t s,
                void (*heavy_segments)(const DevCompressed&, const int32_t*, const int64_t*, const int64_t*, int64_t,
                                       const float*, int, double*, double*, cudaStream_t));
void spmm_panel_check();
// X^T X on the tensor cores (gram_tc.cu): part gets one c x c FP64 partial per
// block (gram_tc_blocks(rows) of them); gram_tc_check raises a recorded timeout.
int gram_tc_launch(const double* X, int64_t rows, int c, double* part, int64_t part_cap, const int* cond,
                   cudaStream_t s);
int gram_tc_blocks(int64_t rows);
void gram_tc_check();

// Centred products (randomized.cu).  mu (csc.nmajor) = the column sums of A
// over its `rows` rows, divided by rows.  center_product turns Out = A X
// (out_is_rows, X: xrows = ncols rows) into A X - 1 (mu^T X), or Out = A^T X
// (X: xrows = nrows rows) into A^T X - mu (1^T X).  X and Out are row-major
// with c columns.
void column_means_dev(const DevCompressed& csc, int64_t rows, double* mu, cudaStream_t s);
void center_product(const double* X, int64_t xrows, int c, const double* mu, double* Out, int64_t orows,
                    bool out_is_rows, cudaStream_t s);

void datx(double a, const double* x, double* y, int64_t n, cudaStream_t s);  // y = a * x

void gemv_t(const double* Q, int64_t n, int64_t i0, int64_t cnt, const double* x, double* t, double* scratch,
            int64_t scratch_cap, cudaStream_t s);

template <typename T>
void transpose_dense(const T* in, T* out, int64_t rows, int64_t cols, cudaStream_t s);

void transpose(const DevCompressed& in, DevCompressed& out, cudaStream_t s);

}  // namespace svdb
