// Shared declarations of the cooperative Lanczos-block kernel.
#pragma once

#include <cstdint>

#include "device_common.cuh"
#include "spmv.cuh"
#include "svdb_internal.h"

namespace svdb {

// Scalar state of a Lanczos run, shared by the host driver and the kernel.
struct LzState {
    double rnm, tol;
    int64_t j;        // on exit: the step the loop stopped at
    int64_t ll;
    int32_t perm[8];  // work vector k lives in buffer W[perm[k]] (k = 0..6)
    int32_t eta_sel;  // 0: eta = etaA / oldeta = etaB, 1: swapped
    int32_t status;   // 0: reached `last`; 1: restart (startv) needed at step j
    int32_t purge_flag;
    int32_t pad;
    int64_t npurge;
};

struct LzOperand {
    const int64_t* rp;
    const int32_t* ci;
    const double* v;
    const float* vf;  // FP32 values (mixed precision) or null
    int64_t rows;
    const int32_t* long_rows;  // rows of more than kSegNnz entries, one block each
    int64_t nlong;
    SpmvBins bins;             // the other rows, by length
    // the column-sliced copy (sliced launches only, spmv.cuh): its values
    SlicedOp sl;
    const double* sv;
    const float* svf;
};

struct LzArgs {
    LzOperand op1;     // temp = op1 x  (rows: internal nrows)
    LzOperand op2;     // y = op2 temp  (rows: n)
    int64_t n;
    double* W[7];
    double* temp;
    double* Q;         // store: q_i = Q + i * n
    double* P;         // p_0, p_1
    double* alf;
    double* bet;
    double* etaA;
    double* etaB;
    double* part;      // per-block / per-task partial sums
    int64_t part_cap;  // doubles available in part
    double* tq;        // purge coefficients (step-indexed)
    double* tr;
    LzState* st;
    GridBarrier* bar;
    int64_t first, last;
    int32_t resume;    // 1: the host performed startv for step `first`
    double eps1;       // eps * sqrt(n), lanczos_step / purge (mod.rs:685,774)
    double sqrt_eps;   // sqrt(eps): lanczos_step's tol and purge's reps (mod.rs:745,773)
};

// blocks: a cooperative grid; cluster > 0: one thread-block cluster of that many blocks instead.
// sliced: both operands carry their column-sliced copy (op.sl), and the grid
// (one block per SM) stages x slices in kSlSmem bytes of dynamic shared memory.
void launch_lanczos_block(const LzArgs& a, int blocks, int threads, int cluster, cudaStream_t s, bool sliced = false);
int lanczos_sliced_blocks(int threads);
// The column-sliced copy of m (spmv_sliced.cu): built on first use, and its
// FP32 values when fp32; false when m gets none.  sliced_view: its arrays.
bool sliced_prepare(const DevCompressed& m, bool fp32, cudaStream_t s);
SlicedOp sliced_view(const DevCompressed& m);
int lanczos_max_blocks(int threads);
bool lanczos_cluster_ok(int cluster, int threads);

}  // namespace svdb
