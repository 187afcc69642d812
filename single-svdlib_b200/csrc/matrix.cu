// Sparse operator handles in HBM: upload + validation, CSR <-> CSC transpose,
// COO ingestion, and the MaskedCSRMatrix column remap / compaction.
//
// Layout: every handle keeps A twice, as CSR (rows of A) and as CSC (rows of
// A^T), so both products of SMat::svd_opa (src/utils.rs:26) are row gathers
// with coalesced index/value streams and no atomics.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>

#include "device_common.cuh"
#include "svdb_internal.h"

namespace svdb {

uint64_t wait_limit_ns() {
    const char* e = getenv("SVDB_WAIT_LIMIT_NS");
    if (!e || !*e) return 2000000000ull;
    const unsigned long long v = strtoull(e, nullptr, 10);
    return v ? v : 1;
}

const DeviceProps& device_props() {
    static thread_local int cached_dev = -1;
    static thread_local DeviceProps props;
    int dev = 0;
    SVDB_CUDA(cudaGetDevice(&dev));
    if (dev != cached_dev) {
        cudaDeviceProp p;
        SVDB_CUDA(cudaGetDeviceProperties(&p, dev));
        props.sms = p.multiProcessorCount;
        props.coop = p.cooperativeLaunch;
        props.l2 = p.l2CacheSize;
        props.smem_optin = p.sharedMemPerBlockOptin > 1024 ? p.sharedMemPerBlockOptin - 1024 : 0;
        cached_dev = dev;
    }
    return props;
}

// ------------------------------------------------------------------ kernels
__global__ void k_check_convert_ptr(const uint64_t* in, int64_t* out, int64_t nmajor, uint64_t nnz, int* bad) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i <= nmajor; i += stride) {
        uint64_t v = in[i];
        out[i] = (int64_t)v;
        if (i == 0 && v != 0) atomicOr(bad, 1);
        if (i == nmajor && v != nnz) atomicOr(bad, 2);
        if (i < nmajor && in[i + 1] < v) atomicOr(bad, 4);
    }
}

__global__ void k_check_convert_idx(const uint64_t* in, int32_t* out, uint64_t nnz, uint64_t bound, int* bad) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < nnz; i += stride) {
        uint64_t v = in[i];
        if (v >= bound) { atomicOr(bad, 8); v = 0; }
        out[i] = (int32_t)v;
    }
}

template <typename IT>
__global__ void k_iota(IT* v, int64_t n) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; k < n; k += stride) v[k] = (IT)k;
}

// row id of every entry, one warp per row (writes stay inside [0, nnz) for any offsets)
__global__ void k_fill_major(const int64_t* __restrict__ ptr, int64_t nmajor, int64_t nnz,
                             int32_t* __restrict__ major_of) {
    const int lane = threadIdx.x & 31;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = gwarp; r < nmajor; r += nwarps) {
        const int64_t b = ptr[r] < 0 ? 0 : ptr[r], e = ptr[r + 1] > nnz ? nnz : ptr[r + 1];
        for (int64_t k = b + lane; k < e; k += 32) major_of[k] = (int32_t)r;
    }
}

template <typename IT>
__global__ void k_gather_idx(const IT* perm, const int32_t* major_of, int32_t* out_idx, int64_t nnz) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; k < nnz; k += stride) out_idx[k] = major_of[perm[k]];
}
template <typename IT>
__global__ void k_gather_val(const IT* perm, const double* val, double* out_val, int64_t nnz) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; k < nnz; k += stride) out_val[k] = val[perm[k]];
}

// out_ptr[c] = first position with key >= c (keys sorted ascending), c in [0, nminor]
__global__ void k_offsets_from_sorted(const int32_t* keys, int64_t nnz, int64_t nminor, int64_t* out_ptr) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; c <= nminor; c += stride) {
        int64_t lo = 0, hi = nnz;
        while (lo < hi) {
            int64_t mid = (lo + hi) >> 1;
            if ((int64_t)keys[mid] < c) lo = mid + 1; else hi = mid;
        }
        out_ptr[c] = lo;
    }
}

__global__ void k_to_f32(const double* in, float* out, int64_t n) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; k < n; k += stride) out[k] = (float)in[k];
}

static int grid_for(int64_t n, int threads = 256) {
    int64_t b = (n + threads - 1) / threads;
    int64_t cap = (int64_t)device_props().sms * 32;
    return (int)std::max<int64_t>(1, std::min(b, cap));
}

static int bits_for(int64_t n) {
    int b = 1;
    while (b < 31 && (int64_t(1) << b) < n) ++b;
    return b;
}

// Stable sort of entry positions by minor index: the transpose keeps majors
// ascending inside every minor slice (CSR rows ascending inside each column).
// The structure (offsets, indices) needs only in.ptr and in.idx; the values
// follow through the returned permutation, so an upload can still be copying
// in.val while the structure is built.
template <typename IT>
static DevBuf<IT> transpose_structure(const DevCompressed& in, DevCompressed& out, cudaStream_t s) {
    const int64_t nnz = in.nnz;
    out.nmajor = in.nminor;
    out.nminor = in.nmajor;
    out.nnz = nnz;
    out.ptr.alloc(out.nmajor + 1, s);
    out.idx.alloc(std::max<int64_t>(nnz, 1), s);
    out.val.alloc(std::max<int64_t>(nnz, 1), s);
    DevBuf<IT> perm(std::max<int64_t>(nnz, 1), s);
    if (nnz == 0) {
        SVDB_CUDA(cudaMemsetAsync(out.ptr.p, 0, (out.nmajor + 1) * sizeof(int64_t), s));
        return perm;
    }
    DevBuf<int32_t> major_of(nnz, s), keys_out(nnz, s);
    DevBuf<IT> vals_in(nnz, s);
    k_fill_major<<<grid_for(in.nmajor * 32), 256, 0, s>>>(in.ptr.p, in.nmajor, nnz, major_of.p);
    k_iota<IT><<<grid_for(nnz), 256, 0, s>>>(vals_in.p, nnz);
    SVDB_CHECK_LAUNCH_N(2);
    size_t tmp_bytes = 0;
    int end_bit = bits_for(std::max<int64_t>(in.nminor, 2));
    SVDB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, in.idx.p, keys_out.p, vals_in.p, perm.p,
                                              nnz, 0, end_bit, s));
    DevBuf<uint8_t> tmp(std::max<size_t>(tmp_bytes, 1), s);
    SVDB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, in.idx.p, keys_out.p, vals_in.p, perm.p, nnz,
                                              0, end_bit, s));
    k_gather_idx<IT><<<grid_for(nnz), 256, 0, s>>>(perm.p, major_of.p, out.idx.p, nnz);
    k_offsets_from_sorted<<<grid_for(out.nmajor + 1), 256, 0, s>>>(keys_out.p, nnz, out.nmajor, out.ptr.p);
    SVDB_CHECK_LAUNCH_N(2);
    return perm;
}
template <typename IT>
static void transpose_values(const DevCompressed& in, DevCompressed& out, const DevBuf<IT>& perm, cudaStream_t s) {
    if (in.nnz == 0) return;
    k_gather_val<IT><<<grid_for(in.nnz), 256, 0, s>>>(perm.p, in.val.p, out.val.p, in.nnz);
    SVDB_CHECK_LAUNCH();
}

void transpose(const DevCompressed& in, DevCompressed& out, cudaStream_t s) {
    if (in.nnz <= INT32_MAX) {
        DevBuf<int32_t> perm = transpose_structure<int32_t>(in, out, s);
        transpose_values(in, out, perm, s);
    } else {
        DevBuf<int64_t> perm = transpose_structure<int64_t>(in, out, s);
        transpose_values(in, out, perm, s);
    }
}

// The FP32 copies belong to the handle that owns the arrays (the parent of an
// all-columns masked view), so they are allocated, filled and later freed on
// that handle's stream, which lives as long as they do.
void ensure_fp32(const svdb_matrix* a) {
    const svdb_matrix* owner = (a->kind == KIND_MASKED && a->all_columns) ? a->parent : a;
    bool launched = false;
    for (const DevCompressed* c : {&csr_of(a), &csc_of(a)}) {
        DevCompressed* m = const_cast<DevCompressed*>(c);
        if (m->val32.p || m->nnz == 0) continue;
        m->val32.alloc(m->nnz, owner->stream);
        k_to_f32<<<grid_for(m->nnz), 256, 0, owner->stream>>>(m->val.p, m->val32.p, m->nnz);
        SVDB_CHECK_LAUNCH();
        launched = true;
    }
    if (launched) SVDB_CUDA(cudaStreamSynchronize(owner->stream));
}

// SpMM load-balancing plans for both orientations (spmm.cu)
static void build_plans(svdb_matrix* a, cudaStream_t s) {
    a->csr.owner_stream = a->stream;
    a->csc.owner_stream = a->stream;
    build_seg_plan(a->csr, s);
    build_seg_plan(a->csc, s);
}

const DevCompressed& csr_of(const svdb_matrix* a) {
    if (a->kind == KIND_MASKED && a->all_columns) return a->parent->csr;
    return a->csr;
}
const DevCompressed& csc_of(const svdb_matrix* a) {
    if (a->kind == KIND_MASKED && a->all_columns) return a->parent->csc;
    return a->csc;
}

// A second stream for the value upload of a new handle, synchronised and
// destroyed on every exit (so no buffer it writes is freed under it).
struct SideStream {
    cudaStream_t s = nullptr;
    cudaEvent_t e = nullptr;
    SideStream() {
        SVDB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        SVDB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    ~SideStream() {
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
        if (e) cudaEventDestroy(e);
    }
};

static void build_plans(svdb_matrix* a, cudaStream_t s);

// Uploads a compressed structure `c` given with usize offsets / indices and f64
// values, or f32 values (val32, kept as the FP32 copy and widened exactly),
// builds its transpose `t` and both segment plans.  The offsets are checked
// first (the plans size their buffers from them).  The values then travel on a
// second stream after the indices, while this stream converts the indices,
// sorts the transpose's structure and builds the plans: only the last step,
// placing the values in the transpose, waits for them.  Out-of-range indices
// are read as 0 on the device (every step stays in bounds) and reported at
// the end.
static void upload_and_transpose(svdb_matrix* a, DevCompressed& c, DevCompressed& t, int64_t nmajor, int64_t nminor,
                                 uint64_t nnz, const uint64_t* ptr, const uint64_t* idx, const double* val,
                                 const float* val32) {
    cudaStream_t s = a->stream;
    if (!ptr || (nnz && (!idx || (!val && !val32)))) throw Error(SVDB_ERR_ARG, "null array");
    if (nminor > INT32_MAX) throw Error(SVDB_ERR_UNSUPPORTED, "minor dimension above 2^31-1");
    c.nmajor = nmajor;
    c.nminor = nminor;
    c.nnz = (int64_t)nnz;
    DevBuf<uint64_t> tptr(nmajor + 1, s), tidx(std::max<uint64_t>(nnz, 1), s);
    DevBuf<int> bad(1, s);
    c.ptr.alloc(nmajor + 1, s);
    c.idx.alloc(std::max<uint64_t>(nnz, 1), s);
    c.val.alloc(std::max<uint64_t>(nnz, 1), s);
    if (val32 && nnz) c.val32.alloc(nnz, s);
    SVDB_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    SVDB_CUDA(cudaMemcpyAsync(tptr.p, ptr, (nmajor + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    k_check_convert_ptr<<<grid_for(nmajor + 1), 256, 0, s>>>(tptr.p, c.ptr.p, nmajor, nnz, bad.p);
    SVDB_CHECK_LAUNCH();
    int hbad = 0;
    SVDB_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaStreamSynchronize(s));
    auto report = [&](int b) {
        std::string m = "invalid compressed sparse input:";
        if (b & 1) m += " offsets[0] != 0;";
        if (b & 2) m += " offsets[last] != nnz;";
        if (b & 4) m += " offsets not monotone;";
        if (b & 8) m += " index out of bounds;";
        throw Error(SVDB_ERR_SHAPE, m);
    };
    if (hbad) report(hbad);
    SideStream side;
    if (nnz) {
        SVDB_CUDA(cudaMemcpyAsync(tidx.p, idx, nnz * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
        // the values follow the indices on the link, on the side stream
        SVDB_CUDA(cudaEventRecord(side.e, s));
        SVDB_CUDA(cudaStreamWaitEvent(side.s, side.e, 0));
        if (val32) {
            SVDB_CUDA(cudaMemcpyAsync(c.val32.p, val32, nnz * sizeof(float), cudaMemcpyHostToDevice, side.s));
            widen(c.val32.p, c.val.p, (int64_t)nnz, side.s);
        } else {
            SVDB_CUDA(cudaMemcpyAsync(c.val.p, val, nnz * sizeof(double), cudaMemcpyHostToDevice, side.s));
        }
        SVDB_CUDA(cudaEventRecord(side.e, side.s));
        k_check_convert_idx<<<grid_for(nnz), 256, 0, s>>>(tidx.p, c.idx.p, nnz, (uint64_t)nminor, bad.p);
        SVDB_CHECK_LAUNCH();
    }
    auto finish = [&](auto perm) {
        build_plans(a, s);
        if (nnz) SVDB_CUDA(cudaStreamWaitEvent(s, side.e, 0));
        transpose_values(c, t, perm, s);
    };
    if (c.nnz <= INT32_MAX) finish(transpose_structure<int32_t>(c, t, s));
    else finish(transpose_structure<int64_t>(c, t, s));
    SVDB_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaStreamSynchronize(s));
    if (hbad) report(hbad);
}

// Device buffers come from the device's default stream-ordered pool.  With
// its default release threshold of 0 the pool hands memory back to the driver
// at every synchronisation, and the next call pays for fresh allocations;
// the library keeps what it freed cached instead (svdb_release_cached_memory
// trims it).
static void keep_pool_cached(int dev) {
    static std::mutex mu;
    static bool done[64] = {};
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 0 || dev >= 64 || done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    done[dev] = true;
}

void release_cached_memory() {
    int dev = 0;
    SVDB_CUDA(cudaGetDevice(&dev));
    cudaMemPool_t pool;
    SVDB_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    SVDB_CUDA(cudaDeviceSynchronize());
    SVDB_CUDA(cudaMemPoolTrimTo(pool, 0));
    host_result_release();
}

static svdb_matrix* new_handle() {
    noalloc_reserve();  // svdb_opb_device_noalloc's scratch on the current device
    svdb_matrix* a = new svdb_matrix();
    SVDB_CUDA(cudaGetDevice(&a->device));
    keep_pool_cached(a->device);
    SVDB_CUDA(cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking));
    return a;
}

svdb_matrix* create_csr(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* indptr,
                        const uint64_t* indices, const double* values, const float* values32) {
    svdb_matrix* a = new_handle();
    try {
        a->kind = KIND_CSR;
        a->nrows = nrows; a->ncols = ncols; a->nnz = nnz;
        upload_and_transpose(a, a->csr, a->csc, nrows, ncols, nnz, indptr, indices, values, values32);
    } catch (...) {
        cudaStreamSynchronize(a->stream);
        delete a;
        throw;
    }
    return a;
}

svdb_matrix* create_csc(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* colptr,
                        const uint64_t* rowidx, const double* values, const float* values32) {
    svdb_matrix* a = new_handle();
    try {
        a->kind = KIND_CSC;
        a->nrows = nrows; a->ncols = ncols; a->nnz = nnz;
        if (nrows > INT32_MAX) throw Error(SVDB_ERR_UNSUPPORTED, "nrows above 2^31-1");
        upload_and_transpose(a, a->csc, a->csr, ncols, nrows, nnz, colptr, rowidx, values, values32);
    } catch (...) {
        cudaStreamSynchronize(a->stream);
        delete a;
        throw;
    }
    return a;
}

// COO: entries stay in push order inside each row (stable sort by row), and
// duplicates remain separate entries, as the crate's triplet loops use them.
svdb_matrix* create_coo(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* rows, const uint64_t* cols,
                        const double* values, const float* values32) {
    svdb_matrix* a = new_handle();
    try {
        a->kind = KIND_COO;
        a->nrows = nrows; a->ncols = ncols; a->nnz = nnz;
        if (nrows > INT32_MAX || ncols > INT32_MAX) throw Error(SVDB_ERR_UNSUPPORTED, "dimension above 2^31-1");
        cudaStream_t s = a->stream;
        // Treat (row ids, col ids) as a "CSC-like" structure keyed by row:
        // sort entry positions by row, stable.
        DevCompressed tmp;
        tmp.nmajor = 1; tmp.nminor = nrows; tmp.nnz = nnz;
        DevBuf<uint64_t> tr(std::max<uint64_t>(nnz, 1), s), tc(std::max<uint64_t>(nnz, 1), s);
        DevBuf<int32_t> r32(std::max<uint64_t>(nnz, 1), s), c32(std::max<uint64_t>(nnz, 1), s);
        DevBuf<double> v(std::max<uint64_t>(nnz, 1), s);
        DevBuf<int> bad(1, s);
        SVDB_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
        if (nnz) {
            if (!rows || !cols || (!values && !values32)) throw Error(SVDB_ERR_ARG, "null array");
            SVDB_CUDA(cudaMemcpyAsync(tr.p, rows, nnz * 8, cudaMemcpyHostToDevice, s));
            SVDB_CUDA(cudaMemcpyAsync(tc.p, cols, nnz * 8, cudaMemcpyHostToDevice, s));
            if (values32) {
                DevBuf<float> v32(nnz, s);
                SVDB_CUDA(cudaMemcpyAsync(v32.p, values32, nnz * 4, cudaMemcpyHostToDevice, s));
                widen(v32.p, v.p, (int64_t)nnz, s);
            } else {
                SVDB_CUDA(cudaMemcpyAsync(v.p, values, nnz * 8, cudaMemcpyHostToDevice, s));
            }
            k_check_convert_idx<<<grid_for(nnz), 256, 0, s>>>(tr.p, r32.p, nnz, nrows, bad.p);
            k_check_convert_idx<<<grid_for(nnz), 256, 0, s>>>(tc.p, c32.p, nnz, ncols, bad.p);
            SVDB_CHECK_LAUNCH_N(2);
        }
        int hbad = 0;
        SVDB_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
        if (hbad) throw Error(SVDB_ERR_SHAPE, "COO index out of bounds");
        a->csr.nmajor = nrows; a->csr.nminor = ncols; a->csr.nnz = nnz;
        a->csr.ptr.alloc(nrows + 1, s);
        a->csr.idx.alloc(std::max<uint64_t>(nnz, 1), s);
        a->csr.val.alloc(std::max<uint64_t>(nnz, 1), s);
        if (nnz == 0) {
            SVDB_CUDA(cudaMemsetAsync(a->csr.ptr.p, 0, (nrows + 1) * 8, s));
        } else {
            DevBuf<int32_t> keys_out(nnz, s);
            DevBuf<int64_t> pin(nnz, s), pout(nnz, s);
            k_iota<int64_t><<<grid_for(nnz), 256, 0, s>>>(pin.p, nnz);
            size_t tb = 0;
            int eb = bits_for(std::max<int64_t>(nrows, 2));
            SVDB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, r32.p, keys_out.p, pin.p, pout.p, nnz, 0, eb, s));
            DevBuf<uint8_t> t(std::max<size_t>(tb, 1), s);
            SVDB_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tb, r32.p, keys_out.p, pin.p, pout.p, nnz, 0, eb, s));
            k_gather_idx<int64_t><<<grid_for(nnz), 256, 0, s>>>(pout.p, c32.p, a->csr.idx.p, nnz);
            k_gather_val<int64_t><<<grid_for(nnz), 256, 0, s>>>(pout.p, v.p, a->csr.val.p, nnz);
            k_offsets_from_sorted<<<grid_for(nrows + 1), 256, 0, s>>>(keys_out.p, nnz, nrows, a->csr.ptr.p);
            SVDB_CHECK_LAUNCH_N(4);
        }
        transpose(a->csr, a->csc, s);
        build_plans(a, s);
        SVDB_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        cudaStreamSynchronize(a->stream);
        delete a;
        throw;
    }
    return a;
}

__global__ void k_copy_i64(const int64_t* in, int64_t* out, int64_t n, int64_t bound, int* bad, int check_mono,
                           int64_t nnz) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        int64_t v = in[i];
        out[i] = v;
        if (check_mono) {
            if (i == 0 && v != 0) atomicOr(bad, 1);
            if (i == n - 1 && v != nnz) atomicOr(bad, 2);
            if (i + 1 < n && in[i + 1] < v) atomicOr(bad, 4);
        }
    }
}
__global__ void k_copy_i32_checked(const int32_t* in, int32_t* out, int64_t n, int64_t bound, int* bad) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        int32_t v = in[i];
        if (v < 0 || v >= bound) { atomicOr(bad, 8); v = 0; }
        out[i] = v;
    }
}

svdb_matrix* create_csr_device(uint64_t nrows, uint64_t ncols, uint64_t nnz, const int64_t* d_indptr,
                               const int32_t* d_indices, const double* d_values) {
    svdb_matrix* a = new_handle();
    try {
        if (ncols > INT32_MAX) throw Error(SVDB_ERR_UNSUPPORTED, "ncols above 2^31-1");
        cudaStream_t s = a->stream;
        a->kind = KIND_CSR;
        a->nrows = nrows; a->ncols = ncols; a->nnz = nnz;
        DevCompressed& c = a->csr;
        c.nmajor = nrows; c.nminor = ncols; c.nnz = nnz;
        c.ptr.alloc(nrows + 1, s);
        c.idx.alloc(std::max<uint64_t>(nnz, 1), s);
        c.val.alloc(std::max<uint64_t>(nnz, 1), s);
        DevBuf<int> bad(1, s);
        SVDB_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
        k_copy_i64<<<grid_for(nrows + 1), 256, 0, s>>>(d_indptr, c.ptr.p, nrows + 1, 0, bad.p, 1, nnz);
        if (nnz) {
            k_copy_i32_checked<<<grid_for(nnz), 256, 0, s>>>(d_indices, c.idx.p, nnz, ncols, bad.p);
            SVDB_CUDA(cudaMemcpyAsync(c.val.p, d_values, nnz * 8, cudaMemcpyDeviceToDevice, s));
        }
        SVDB_CHECK_LAUNCH_N(nnz ? 2 : 1);
        int hbad = 0;
        SVDB_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
        if (hbad) throw Error(SVDB_ERR_SHAPE, "invalid compressed sparse input");
        transpose(a->csr, a->csc, s);
        build_plans(a, s);
        SVDB_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        cudaStreamSynchronize(a->stream);
        delete a;
        throw;
    }
    return a;
}

// ----------------------------------------------------------- masked view --
// original_to_masked[c] = rank of c among included columns (-1 = None),
// masked_to_original[rank] = c; the ranks come from an exclusive scan of the
// mask, so masked column j is the j-th included column in ascending order
// (masked.rs:32-38).
__global__ void k_mask_maps(const uint8_t* mask, const int64_t* scan, int64_t n, int64_t* o2m, int64_t* m2o) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; c < n; c += stride) {
        if (mask[c]) { o2m[c] = scan[c]; m2o[scan[c]] = c; }
        else o2m[c] = -1;
    }
}

__global__ void k_mask_to_i64(const uint8_t* mask, int64_t* out, int64_t n) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; c < n; c += stride) out[c] = mask[c] ? 1 : 0;
}

__global__ void k_mask_flags(const int32_t* idx, const uint8_t* mask, int64_t nnz, int64_t* flags) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; k < nnz; k += stride) flags[k] = mask[idx[k]] ? 1 : 0;
}

// Kept entries keep their order (scan positions); columns are remapped.
__global__ void k_mask_compact(const int32_t* idx, const double* val, const int64_t* pos, const int64_t* o2m,
                               int64_t nnz, int32_t* out_idx, double* out_val) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; k < nnz; k += stride) {
        int64_t mc = o2m[idx[k]];
        if (mc >= 0) {
            int64_t p = pos[k];
            out_idx[p] = (int32_t)mc;
            out_val[p] = val[k];
        }
    }
}

__global__ void k_mask_rowptr(const int64_t* ptr, const int64_t* pos, int64_t nrows, int64_t* out_ptr) {
    int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; r <= nrows; r += stride) out_ptr[r] = pos[ptr[r]];
}

svdb_matrix* masked_new(const svdb_matrix* parent, const uint8_t* hmask, uint64_t mask_len) {
    if (!parent || !hmask) throw Error(SVDB_ERR_ARG, "null argument");
    if (parent->kind == KIND_MASKED) throw Error(SVDB_ERR_ARG, "MaskedCSRMatrix borrows a CsrMatrix, not a view");
    if ((int64_t)mask_len != parent->ncols)
        throw Error(SVDB_ERR_SHAPE, "Column mask must have the same length as the number of columns in the matrix");
    svdb_matrix* a = new_handle();
    try {
        cudaStream_t s = a->stream;
        // The parent may be in use on its own stream; order after it.
        SVDB_CUDA(cudaStreamSynchronize(parent->stream));
        a->kind = KIND_MASKED;
        a->parent = parent;
        a->nrows = parent->nrows;
        const int64_t n = parent->ncols;
        const DevCompressed& P = parent->csr;
        const int64_t nnz = P.nnz;
        DevBuf<uint8_t> mask(std::max<int64_t>(n, 1), s);
        DevBuf<int64_t> mask64(n + 1, s), scan(n + 1, s);
        a->o2m.alloc(std::max<int64_t>(n, 1), s);
        a->m2o.alloc(std::max<int64_t>(n, 1), s);
        if (n) SVDB_CUDA(cudaMemcpyAsync(mask.p, hmask, n, cudaMemcpyHostToDevice, s));
        // exclusive scan of the mask (as int64, one trailing zero) -> ranks;
        // the last element is the masked column count
        DevBuf<uint8_t> mask_pad(n + 1, s);
        SVDB_CUDA(cudaMemsetAsync(mask_pad.p, 0, n + 1, s));
        if (n) SVDB_CUDA(cudaMemcpyAsync(mask_pad.p, mask.p, n, cudaMemcpyDeviceToDevice, s));
        k_mask_to_i64<<<grid_for(n + 1), 256, 0, s>>>(mask_pad.p, mask64.p, n + 1);
        size_t tb = 0;
        SVDB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, mask64.p, scan.p, n + 1, s));
        DevBuf<uint8_t> tmp(std::max<size_t>(tb, 1), s);
        SVDB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, mask64.p, scan.p, n + 1, s));
        k_mask_maps<<<grid_for(std::max<int64_t>(n, 1)), 256, 0, s>>>(mask_pad.p, scan.p, n, a->o2m.p, a->m2o.p);
        SVDB_CHECK_LAUNCH_N(2);
        int64_t nm = 0;
        SVDB_CUDA(cudaMemcpyAsync(&nm, scan.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
        a->ncols = nm;
        bool all = (nm == n);
        a->all_columns = all;
        if (all) {
            a->nnz = nnz;  // uses_all_columns: the view is the parent operator
            return a;
        }
        // Compaction: flags -> exclusive scan -> scatter, order preserved.
        DevBuf<int64_t> flags(nnz + 1, s), pos(nnz + 1, s);
        SVDB_CUDA(cudaMemsetAsync(flags.p, 0, (nnz + 1) * sizeof(int64_t), s));
        if (nnz) k_mask_flags<<<grid_for(nnz), 256, 0, s>>>(P.idx.p, mask_pad.p, nnz, flags.p);
        size_t tb2 = 0;
        SVDB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb2, flags.p, pos.p, nnz + 1, s));
        DevBuf<uint8_t> tmp2(std::max<size_t>(tb2, 1), s);
        SVDB_CUDA(cub::DeviceScan::ExclusiveSum(tmp2.p, tb2, flags.p, pos.p, nnz + 1, s));
        int64_t mnnz = 0;
        SVDB_CUDA(cudaMemcpyAsync(&mnnz, pos.p + nnz, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
        a->nnz = mnnz;
        DevCompressed& C = a->csr;
        C.nmajor = parent->nrows; C.nminor = nm; C.nnz = mnnz;
        C.ptr.alloc(C.nmajor + 1, s);
        C.idx.alloc(std::max<int64_t>(mnnz, 1), s);
        C.val.alloc(std::max<int64_t>(mnnz, 1), s);
        if (nnz) k_mask_compact<<<grid_for(nnz), 256, 0, s>>>(P.idx.p, P.val.p, pos.p, a->o2m.p, nnz, C.idx.p,
                                                              C.val.p);
        k_mask_rowptr<<<grid_for(C.nmajor + 1), 256, 0, s>>>(P.ptr.p, pos.p, C.nmajor, C.ptr.p);
        SVDB_CHECK_LAUNCH_N(nnz ? 3 : 1);
        transpose(a->csr, a->csc, s);
        build_plans(a, s);
        SVDB_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        cudaStreamSynchronize(a->stream);
        delete a;
        throw;
    }
    return a;
}

void masked_maps(const svdb_matrix* a, int64_t* m2o, int64_t* o2m) {
    if (a->kind != KIND_MASKED) throw Error(SVDB_ERR_ARG, "not a MaskedCSRMatrix handle");
    if (a->ncols) SVDB_CUDA(cudaMemcpyAsync(m2o, a->m2o.p, a->ncols * 8, cudaMemcpyDeviceToHost, a->stream));
    if (a->parent->ncols)
        SVDB_CUDA(cudaMemcpyAsync(o2m, a->o2m.p, a->parent->ncols * 8, cudaMemcpyDeviceToHost, a->stream));
    SVDB_CUDA(cudaStreamSynchronize(a->stream));
}

void destroy(svdb_matrix* a) {
    if (!a) return;
    cudaStreamSynchronize(a->stream);
    // buffers free themselves on a->stream
    cudaStream_t s = a->stream;
    delete a;
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
}

}  // namespace svdb
