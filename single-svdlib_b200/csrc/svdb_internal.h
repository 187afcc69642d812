// Internal declarations shared by the CUDA sources of libsvdb200.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/svdb200.h"

namespace svdb {

// ---------------------------------------------------------------- errors ----
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);

#define SVDB_CUDA(call)                                                                        \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            throw ::svdb::Error(e_ == cudaErrorMemoryAllocation ? SVDB_ERR_OOM : SVDB_ERR_CUDA, \
                                std::string(#call) + ": " + cudaGetErrorString(e_));            \
    } while (0)

// Every kernel launch site is followed by SVDB_CHECK_LAUNCH(n), n being the
// number of kernels launched since the previous check; the count feeds
// svdb_kernel_launches().
void count_launches(uint64_t n);
void discount_launches(uint64_t n);  // launches recorded into a graph, counted when it runs
#define SVDB_CHECK_LAUNCH_N(n)             \
    do {                                   \
        ::svdb::count_launches(n);         \
        SVDB_CUDA(cudaGetLastError());     \
    } while (0)
#define SVDB_CHECK_LAUNCH() SVDB_CHECK_LAUNCH_N(1)

// --------------------------------------------------------- device memory ----
// Owning device buffer, stream-ordered (cudaMallocAsync pool).
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    DevBuf() {}
    DevBuf(size_t count, cudaStream_t st) { alloc(count, st); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; s = o.s; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t count, cudaStream_t st) {
        release();
        s = st;
        n = count;
        if (count) SVDB_CUDA(cudaMallocAsync((void**)&p, count * sizeof(T), st));
    }
    void release() {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    T* detach() { T* q = p; p = nullptr; n = 0; return q; }
    size_t bytes() const { return n * sizeof(T); }
};

// ------------------------------------------------------------ matrices ------
// A compressed sparse structure in HBM: `nmajor` rows of a CSR (or columns of
// a CSC, i.e. rows of the transpose).  Column indices are int32 (minor
// dimension < 2^31), offsets int64.
// Load-balancing plan for the row gathers of SpMM: every row is cut into
// segments of at most kSegNnz entries; seg_first[r] .. seg_first[r+1] are the
// segments of row r; segment s covers entries [seg_beg[s], seg_end[s]) of row
// seg_row[s], stored as -(row + 1) when the row has several segments; those
// rows are listed in multi_rows and merged by a second, ordered pass.
constexpr int64_t kSegNnz = 2048;
// SpMV row bins: bin b (< kSpmvBins) holds the rows of at most
// kSpmvBinLen[b] entries (and more than kSpmvBinLen[b-1]), ascending, taken
// by groups of (2 << b) lanes; rows of more than kSegNnz entries are the
// multi rows, one block each.
constexpr int kSpmvBins = 5;
constexpr int64_t kSpmvBinLen[kSpmvBins] = {8, 16, 32, 64, kSegNnz};
struct SpmvBins {
    const int32_t* rows;             // bin_rows
    int64_t off[kSpmvBins + 1];      // bin b: rows[off[b] .. off[b+1])
    int64_t items[kSpmvBins + 1];    // warp items before bin b (32 / (2 << b) rows per item)
};
struct SegPlan {
    int64_t nseg = 0, nmulti = 0;
    DevBuf<int32_t> bin_rows;
    SpmvBins bins{};
    DevBuf<int64_t> seg_first;
    DevBuf<int32_t> seg_row;
    DevBuf<int64_t> seg_beg, seg_end;
    DevBuf<int32_t> multi_rows;
};

// Panel plan of the FP32 SpMM (spmm_panel.cu), built on first use.  Rows
// up to `heavy` nonzeros are dealt to (virtual CTA, warp, slot); their entries
// are copied grouped by (virtual CTA, panel of the dense operand) -- a "CTA
// panel", padded to an even count -- and inside it by (warp, slot).  Longer
// rows keep the segment kernel: their segments of `plan`, compacted into
// hseg_*, and hmulti rows merged from partials.
struct PanelPlan {
    bool tried = false, usable = false;
    int rw = 0, vctas = 0, npanels = 0, sstride = 0;
    int64_t heavy = 0, nlight = 0, ecap = 0;
    DevBuf<uint64_t> ent;      // row within the panel (low 32 bits) | FP32 value bits (high 32)
    DevBuf<int64_t> cbase;     // vctas * npanels + 1: first entry of each CTA panel
    DevBuf<int32_t> soff;      // per CTA panel, stride sstride: warps * rw + 1 slot offsets in it
    DevBuf<int32_t> slot_row;  // vctas * warps * rw rows, -1 for an empty slot
    int64_t nhseg = 0, nhmulti = 0;
    DevBuf<int32_t> hseg_row;  // negative: a partial at the list position; else the row
    DevBuf<int64_t> hseg_beg, hseg_end;
    DevBuf<int32_t> hmulti_row;
    DevBuf<int64_t> hmulti_first, hmulti_count;
};

// Column-sliced copy of a structure for the SpMV (spmv_sliced.cu), built on
// the first product of a large operator: per slice of columns, a CSR over
// all rows with 16-bit column offsets, and the rows cut into ranges for the
// CTAs.
struct SlicedPlan {
    bool tried = false, usable = false;
    int32_t nslices = 0, nranges = 0;
    DevBuf<int64_t> sbase;   // nslices + 1: first entry of each slice
    DevBuf<int32_t> sptr;    // nslices x (nmajor + 1): row offsets from sbase[s]
    DevBuf<uint16_t> sidx;   // column minus the slice's first column
    DevBuf<double> sval;
    DevBuf<float> sval32;    // made on the first FP32 product
    DevBuf<int64_t> rstart;  // nranges + 1 row boundaries
};

struct DevCompressed {
    int64_t nmajor = 0, nminor = 0, nnz = 0;
    DevBuf<int64_t> ptr;
    DevBuf<int32_t> idx;
    DevBuf<double> val;
    DevBuf<float> val32;  // FP32 copy of val, made on first mixed-precision use
    SegPlan plan;         // built when the handle is created
    PanelPlan panel;      // built on the first panel SpMM
    SlicedPlan sliced;    // built on the first SpMV of a large operator
    // stream of the handle that owns this structure: buffers made after
    // creation (the panel plan) are allocated, and so freed, on it
    cudaStream_t owner_stream = nullptr;
    double avg_per_major() const { return nmajor ? double(nnz) / double(nmajor) : 0.0; }
};

// Builds m.plan on stream s (called once per structure, at creation).
void build_seg_plan(DevCompressed& m, cudaStream_t s);

// Dense-column split of a matrix for the FP32 SpMM (dense_split.cu): the
// columns J of density above a threshold as a dense block D = A[:, J]
// (m x ndp FP32, row-major) and its transpose Dt (ndp x mp), and the rest
// of A without them as a CSR (rest_csr) and a CSR of its transpose with the
// rows J emptied (rest_csc), each with FP32 values and a segment plan.
struct DenseSplit {
    int64_t nd = 0, ndp = 0, mp = 0;  // dense columns; padded to 128; rows padded to 32
    int64_t dense_nnz = 0;
    DevBuf<int32_t> cols;             // ndp original column ids, -1 for padding
    DevBuf<float> D, Dl, Dt, Dtl;     // A[:, J] and its transpose: TF32 heads and remainders
    DevCompressed rest_csr, rest_csc;
};

enum MatKind { KIND_CSR = 0, KIND_CSC = 1, KIND_COO = 2, KIND_MASKED = 3 };

}  // namespace svdb

struct svdb_matrix {
    int kind = svdb::KIND_CSR;
    int device = 0;
    int64_t nrows = 0, ncols = 0;  // logical shape (masked: masked column count)
    int64_t nnz = 0;               // SMat::nnz (masked: entries in the mask)
    cudaStream_t stream = nullptr;
    svdb::DevCompressed csr;  // A, rows
    svdb::DevCompressed csc;  // A^T, rows = columns of A
    // masked view data
    const svdb_matrix* parent = nullptr;
    bool all_columns = false;
    svdb::DevBuf<int64_t> m2o, o2m;
    std::mutex mu;  // serialises calls on one handle
    // dense-column split of csr/csc for the FP32 SpMM, built on first use
    std::unique_ptr<svdb::DenseSplit> dense;
    bool dense_tried = false;
};

namespace svdb {

const DevCompressed& csr_of(const svdb_matrix* a);
const DevCompressed& csc_of(const svdb_matrix* a);
void ensure_fp32(const svdb_matrix* a);
// FP32 SpMM through the dense-column split (dense_split.cu): usable when the
// matrix has enough dense columns and l <= 64 (builds the split on first use).
bool dense_split_usable(const svdb_matrix* a, int l);
template <typename XT, typename OT>
void dense_split_spmm(const svdb_matrix* a, bool transpose, const XT* X, const float* x32, int l, OT* Y,
                      cudaStream_t s);
void dense_split_check();  // raises a wait timeout an earlier split SpMM recorded (synchronises)
void dense_split_info(const svdb_matrix* a, uint64_t* nd, uint64_t* dense_nnz);
// Batches of column subsets through the split (dense_split.cu): the split of
// a (built on first use; null without one), the device workspace the two
// products need for count subsets of l columns (the B operands of both GEMMs
// and the partial tiles), and the products' dense parts: Y (count x m x l)
// += the dense columns' share of A_b X_b (X_b at X + coff[b] l), and
// Z_b rows of the dense columns = A_b^T Y_b there.
const DenseSplit* dense_split_get(const svdb_matrix* a);
size_t dense_batch_workspace(const DenseSplit& ds, int64_t count, int l);
void dense_batch_rows(const svdb_matrix* a, const float* X, const int64_t* coff, const int32_t* o2m, int64_t count,
                      int l, float* Y, float* bh, float* bl, cudaStream_t s);
template <typename OT>
void dense_batch_cols(const svdb_matrix* a, const float* Y, const int64_t* coff, const int32_t* o2m, int64_t count,
                      int l, OT* Z, float* bh, float* bl, double* part, cudaStream_t s);

struct DeviceProps {
    int sms = 148;
    int coop = 1;
    size_t l2 = 0;
    size_t smem_optin = 0;  // dynamic shared memory a block may opt into (less 1 KB for static use)
};
const DeviceProps& device_props();
// Looks up (once per device) the address of svdb_opb_device_noalloc's
// scratch array on the current device, which places the array in device
// memory; called by every matrix handle's creation (csrc/noalloc.cu).
void noalloc_reserve();
// Limit of the bounded device waits on the default path (the Lanczos grid
// barrier, the tensor-core Gram's commit waits): SVDB_WAIT_LIMIT_NS from the
// environment (read at each launch, at least 1), else 2 s.
uint64_t wait_limit_ns();

// ------------------------------------------------------- kernel entries ----
// y[r] = sum_k val[k] * x[idx[k]] over the rows of `m` (group-per-row).
// allow_sliced = false keeps the gather kernel (no plan is built: nothing allocated).
void spmv(const DevCompressed& m, bool fp32, const double* x, double* y, cudaStream_t s, bool allow_sliced = true);
// The column-sliced SpMV (spmv_sliced.cu); false when m has no sliced plan
// (small, unsorted within rows, or not enough memory), nothing launched.
bool spmv_sliced(const DevCompressed& m, bool fp32, const double* x, double* y, cudaStream_t s);
void sliced_info(const DevCompressed& m, int* nslices, int* nranges);  // 0, 0 without a plan

// Reductions and BLAS-1 (deterministic two-level reductions).
void dot(const double* x, const double* y, int64_t n, double* d_out, double* scratch, cudaStream_t s);
double dot_host(const double* x, const double* y, int64_t n, double* scratch, cudaStream_t s);
void axpy(double a, const double* x, double* y, int64_t n, cudaStream_t s);   // y += a*x (unfused mul then add)
void scal(double a, double* x, int64_t n, cudaStream_t s);                    // x *= a
void copy(const double* x, double* y, int64_t n, cudaStream_t s);
void narrow(const double* x, float* y, int64_t n, cudaStream_t s);  // y = (float)x, round to nearest
void widen(const float* x, double* y, int64_t n, cudaStream_t s);   // y = (double)x
void round_f32(double* x, int64_t n, cudaStream_t s);               // x = (double)(float)x
size_t reduce_scratch_doubles();

// Host result buffers (hostmem.cu): page-locked and reused from 64 KB up,
// malloc below; host_result_free takes either kind, host_result_release
// returns the idle page-locked buffers to the driver.
void* host_result_alloc(size_t bytes);
void host_result_free(void* p);
void host_result_release();

// Start vector: rand 0.9 StdRng::from_seed(seed bytes) + random_range(-1.0..1.0),
// rounded to f32 when round_f32 (T = f32).
void start_vector(uint32_t seed, double* w, int64_t n, cudaStream_t s, bool round_f32 = false);

// y[e] = y[e] - t[i] * Q[i0+i][e], sequentially over i (the crate's axpy order)
void gemv_sub(const double* Q, int64_t n, int64_t i0, int64_t cnt, const double* t, double* y, cudaStream_t s);

}  // namespace svdb
