// Column-sliced SpMV for large operators (svd_opa, src/lanczos/mod.rs:1551-1602):
// y = M x with x staged in shared memory one slice of columns at a time.
//
// The gather SpMV (k_spmv) reads x at every nonzero: on the 1M x 200k LAS2
// matrix that is 200 M random 8-byte reads, each moving a 32-byte sector
// through L2, and the kernel sits near a quarter of HBM bandwidth however
// narrow the values are.  Here the columns are cut into slices of W (18,432)
// and the entries regrouped slice-major: per slice, a CSR over all rows
// whose column indices are 16-bit offsets into the slice.  A CTA owns a
// contiguous range of rows (balanced by nonzeros, at most kSlRowCap rows);
// for each slice it copies x[sW, sW + W) into shared memory with coalesced
// loads, then sums its rows' entries of that slice (a thread per row, a warp
// per long piece; spmv.cuh), reading x from shared memory and adding each
// row's slice sum to an FP64 accumulator in shared memory.  The matrix is read once, 2 + value bytes per nonzero, plus 4
// bytes per (row, slice) of offsets.  Sums run over slices in order and, in
// a slice, over 8-lane groups in a fixed tree: deterministic.
//
// The plan needs column indices non-decreasing within every row (the crate's
// CSR invariant, and what the device transpose produces); otherwise it is
// not built and the gather SpMV stays.
#include <cub/cub.cuh>

#include <algorithm>
#include <mutex>
#include <vector>

#include "device_common.cuh"
#include "ops.cuh"
#include "spmv.cuh"
#include "svdb_internal.h"

namespace svdb {

constexpr int kSlThreads = 1024;
constexpr int64_t kSlMinNnz = int64_t(1) << 22;

template <typename VT>
__global__ void __launch_bounds__(kSlThreads, 1)
    k_spmv_sliced(const __grid_constant__ SlicedOp a, const VT* __restrict__ val, const double* __restrict__ x,
                  double* __restrict__ y) {
    extern __shared__ double sl_sm[];
    sliced_rows<VT, false>(a, val, x, 1.0, sl_sm, [&](int64_t r, double acc) { y[r] = acc; });
}

// ------------------------------------------------------------- plan --
__device__ __forceinline__ int64_t sl_lower_bound(const int32_t* idx, int64_t b, int64_t e, int64_t v) {
    while (b < e) {
        const int64_t mid = (b + e) >> 1;
        if ((int64_t)idx[mid] < v) b = mid + 1;
        else e = mid;
    }
    return b;
}

// flags a row whose column indices fall
__global__ void k_sl_sorted(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci, int64_t rows,
                            int* __restrict__ bad) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = gw; r < rows; r += nw)
        for (int64_t k = rp[r] + 1 + lane; k < rp[r + 1]; k += 32)
            if (ci[k - 1] > ci[k]) *bad = 1;
}

// cnt[s * (rows + 1) + r] = entries of row r in slice s: written by the lane
// holding the row's first entry of that slice
__global__ void k_sl_count(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci, int64_t rows,
                           int64_t* __restrict__ cnt) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = gw; r < rows; r += nw) {
        const int64_t b = rp[r], e = rp[r + 1];
        for (int64_t k = b + lane; k < e; k += 32) {
            const int64_t s = ci[k] / kSlW;
            if (k == b || ci[k - 1] / kSlW != s) {
                const int64_t end = sl_lower_bound(ci, k, e, (s + 1) * kSlW);
                cnt[s * (rows + 1) + r] = end - k;
            }
        }
    }
}

__global__ void k_sl_ptr(const int64_t* __restrict__ off, int64_t rows, int nslices, int64_t* __restrict__ sbase,
                         int32_t* __restrict__ sptr) {
    const int64_t total = (int64_t)nslices * (rows + 1);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = i / (rows + 1);
        const int64_t b = off[s * (rows + 1)];
        sptr[i] = (int32_t)(off[i] - b);
        if (i == s * (rows + 1)) sbase[s] = b;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) sbase[nslices] = off[total - 1];
}

// entry k of row r, in slice s, goes to off[s][r] + (k - first entry of the row in slice s)
__global__ void k_sl_fill(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                          const double* __restrict__ v, int64_t rows, const int64_t* __restrict__ off,
                          uint16_t* __restrict__ sidx, double* __restrict__ sval) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = gw; r < rows; r += nw) {
        const int64_t b = rp[r], e = rp[r + 1];
        for (int64_t k = b + lane; k < e; k += 32) {
            const int64_t c = ci[k], s = c / kSlW;
            const int64_t first = sl_lower_bound(ci, b, k, s * kSlW);
            const int64_t pos = off[s * (rows + 1) + r] + (k - first);
            sidx[pos] = (uint16_t)(c - s * kSlW);
            sval[pos] = v[k];
        }
    }
}

static int sl_blocks(int64_t work, int threads) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((work + threads - 1) / threads, (int64_t)device_props().sms * 8));
}

static std::mutex g_sl_mu;

// Builds m.sliced on first use (operators of at least kSlMinNnz nonzeros and
// more than one slice of columns); false when the plan is not used.
static bool sliced_ready(const DevCompressed& mc, cudaStream_t s) {
    DevCompressed& m = const_cast<DevCompressed&>(mc);
    std::lock_guard<std::mutex> lk(g_sl_mu);
    SlicedPlan& p = m.sliced;
    if (p.tried) return p.usable;
    p.tried = true;
    if (m.nnz < kSlMinNnz || m.nnz > (int64_t)INT32_MAX || m.nminor <= kSlW || m.nminor > (int64_t)INT32_MAX)
        return false;
    const int64_t rows = m.nmajor;
    const int nslices = (int)((m.nminor + kSlW - 1) / kSlW);
    if ((int64_t)nslices * (rows + 1) > (int64_t)1 << 31) return false;
    cudaStream_t os = m.owner_stream ? m.owner_stream : s;
    SVDB_CUDA(cudaStreamSynchronize(s));  // the structure's arrays are complete
    {
        DevBuf<int> bad(1, os);
        SVDB_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), os));
        k_sl_sorted<<<sl_blocks(rows * 32, 256), 256, 0, os>>>(m.ptr.p, m.idx.p, rows, bad.p);
        SVDB_CHECK_LAUNCH();
        int hb = 0;
        SVDB_CUDA(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, os));
        SVDB_CUDA(cudaStreamSynchronize(os));
        if (hb) return false;
    }
    // memory: 2 + 8 (+ 4) bytes per nonzero and 4 per (row, slice); a quarter of the free memory at most
    size_t free_b = 0, total_b = 0;
    SVDB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const double need = (double)m.nnz * 14.0 + (double)nslices * (rows + 1) * 12.0;
    if (need > 0.25 * (double)free_b) return false;
    const int64_t tot = (int64_t)nslices * (rows + 1);
    DevBuf<int64_t> cnt(tot, os), off(tot, os);
    SVDB_CUDA(cudaMemsetAsync(cnt.p, 0, tot * sizeof(int64_t), os));
    k_sl_count<<<sl_blocks(rows * 32, 256), 256, 0, os>>>(m.ptr.p, m.idx.p, rows, cnt.p);
    SVDB_CHECK_LAUNCH();
    size_t tb = 0;
    SVDB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.p, off.p, tot, os));
    DevBuf<uint8_t> tmp(std::max<size_t>(tb, 1), os);
    SVDB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.p, off.p, tot, os));
    p.sbase.alloc(nslices + 1, os);
    p.sptr.alloc(tot, os);
    k_sl_ptr<<<sl_blocks(tot, 256), 256, 0, os>>>(off.p, rows, nslices, p.sbase.p, p.sptr.p);
    SVDB_CHECK_LAUNCH();
    p.sidx.alloc(std::max<int64_t>(m.nnz, 1), os);
    p.sval.alloc(std::max<int64_t>(m.nnz, 1), os);
    k_sl_fill<<<sl_blocks(rows * 32, 256), 256, 0, os>>>(m.ptr.p, m.idx.p, m.val.p, rows, off.p, p.sidx.p, p.sval.p);
    SVDB_CHECK_LAUNCH();
    // row ranges: about nnz / sms nonzeros and at most kSlRowCap rows each
    std::vector<int64_t> hp(rows + 1);
    SVDB_CUDA(cudaMemcpyAsync(hp.data(), m.ptr.p, (rows + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, os));
    SVDB_CUDA(cudaStreamSynchronize(os));
    const int64_t target = std::max<int64_t>(1, (m.nnz + device_props().sms - 1) / device_props().sms);
    std::vector<int64_t> rs{0};
    int64_t r0 = 0;
    for (int64_t r = 1; r <= rows; ++r)
        if (r == rows || r - r0 >= kSlRowCap || hp[r] - hp[r0] >= target) {
            rs.push_back(r);
            r0 = r;
        }
    if (rs.back() != rows) rs.push_back(rows);
    p.nranges = (int)rs.size() - 1;
    p.rstart.alloc(rs.size(), os);
    SVDB_CUDA(cudaMemcpyAsync(p.rstart.p, rs.data(), rs.size() * sizeof(int64_t), cudaMemcpyHostToDevice, os));
    p.nslices = nslices;
    SVDB_CUDA(cudaStreamSynchronize(os));
    static std::once_flag attr;
    std::call_once(attr, [] {
        SVDB_CUDA(cudaFuncSetAttribute(k_spmv_sliced<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSlSmem));
        SVDB_CUDA(cudaFuncSetAttribute(k_spmv_sliced<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSlSmem));
    });
    p.usable = true;
    return true;
}

// FP32 values of the plan, (float) of its FP64 values as val32 is of val
__global__ void k_sl_narrow(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

void sliced_info(const DevCompressed& m, int* nslices, int* nranges) {
    std::lock_guard<std::mutex> lk(g_sl_mu);
    *nslices = m.sliced.usable ? m.sliced.nslices : 0;
    *nranges = m.sliced.usable ? m.sliced.nranges : 0;
}

bool sliced_prepare(const DevCompressed& mc, bool fp32, cudaStream_t s) {
    if (!sliced_ready(mc, s)) return false;
    DevCompressed& m = const_cast<DevCompressed&>(mc);
    SlicedPlan& p = m.sliced;
    if (fp32 && !p.sval32.p) {
        std::lock_guard<std::mutex> lk(g_sl_mu);
        if (!p.sval32.p) {
            cudaStream_t os = m.owner_stream ? m.owner_stream : s;
            p.sval32.alloc(std::max<int64_t>(m.nnz, 1), os);
            k_sl_narrow<<<sl_blocks(m.nnz, 256), 256, 0, os>>>(p.sval.p, p.sval32.p, m.nnz);
            SVDB_CHECK_LAUNCH();
            SVDB_CUDA(cudaStreamSynchronize(os));
        }
    }
    return true;
}

SlicedOp sliced_view(const DevCompressed& m) {
    const SlicedPlan& p = m.sliced;
    SlicedOp a;
    a.nmajor = m.nmajor;
    a.nminor = m.nminor;
    a.nslices = p.nslices;
    a.nranges = p.nranges;
    a.sbase = p.sbase.p;
    a.sptr = p.sptr.p;
    a.sidx = p.sidx.p;
    a.rstart = p.rstart.p;
    return a;
}

bool spmv_sliced(const DevCompressed& mc, bool fp32, const double* x, double* y, cudaStream_t s) {
    if (!sliced_prepare(mc, fp32, s)) return false;
    const DevCompressed& m = mc;
    const SlicedPlan& p = m.sliced;
    const SlicedOp a = sliced_view(m);
    const int grid = std::min(p.nranges, device_props().sms);
    if (fp32) k_spmv_sliced<float><<<grid, kSlThreads, kSlSmem, s>>>(a, p.sval32.p, x, y);
    else k_spmv_sliced<double><<<grid, kSlThreads, kSlSmem, s>>>(a, p.sval.p, x, y);
    SVDB_CHECK_LAUNCH();
    return true;
}

}  // namespace svdb
