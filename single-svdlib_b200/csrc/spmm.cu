// SpMM row gather: Y (rows x l) = M X, X (minor x l), both row-major, for the
// dense products of randomized_svd (masked.rs:265-733) and the sigma/u step
// of ritvec (mod.rs:1197-1210).
//
// Work unit: a row segment of at most kSegNnz entries (SegPlan), so rows of
// any length spread over warps evenly; rows cut into several segments write
// per-segment partials that a second kernel adds in segment order, keeping
// the result deterministic.  Inside a warp, H groups of 32/H lanes each take
// every H-th entry of the segment; a lane owns CPL consecutive columns and
// reads them with one vector load, and each group keeps U gathers in flight.
// Accumulation is FP64 (for FP32 operands: FP32 within a 32-entry chunk,
// FP64 across chunks).  Register caps: 64 per thread for FP32 operands, 85 for
// FP64 operands (no spills at 4 gathers in flight per group).
#include <cub/cub.cuh>

#include <algorithm>

#include "device_common.cuh"
#include "ops.cuh"
#include "svdb_internal.h"

namespace svdb {

namespace {

template <typename T, int N>
struct Vec;
template <>
struct alignas(8) Vec<float, 2> { float v[2]; };
template <>
struct alignas(16) Vec<float, 4> { float v[4]; };
template <>
struct alignas(16) Vec<double, 2> { double v[2]; };
template <>
struct alignas(16) Vec<double, 4> { double v[4]; };  // two 16-byte loads
template <typename T>
struct alignas(sizeof(T)) Vec<T, 1> { T v[1]; };

template <typename T, int N>
__device__ __forceinline__ void load_cols(const T* __restrict__ p, bool vec, int ncols_here, double (&out)[N]) {
    if (vec && ncols_here == N) {
        if constexpr (sizeof(T) * N <= 16) {
            Vec<T, N> t = *reinterpret_cast<const Vec<T, N>*>(p);
#pragma unroll
            for (int j = 0; j < N; ++j) out[j] = (double)t.v[j];
        } else {
            const Vec<T, 2>* q = reinterpret_cast<const Vec<T, 2>*>(p);
#pragma unroll
            for (int h = 0; h < N / 2; ++h) {
                Vec<T, 2> t = q[h];
                out[2 * h] = (double)t.v[0];
                out[2 * h + 1] = (double)t.v[1];
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < N; ++j) out[j] = j < ncols_here ? (double)p[j] : 0.0;
    }
}

template <typename T, int N>
__device__ __forceinline__ void store_cols(T* __restrict__ p, int ncols_here, const double (&a)[N]) {
#pragma unroll
    for (int j = 0; j < N; ++j)
        if (j < ncols_here) p[j] = (T)a[j];
}

}  // namespace

// Work per lane group and round: U gathers are issued before any of them is
// used.  The (index, value) pairs of the next 32 entries are loaded while the
// current ones are consumed.  With FP32 operands the products of one 32-entry
// chunk are summed in FP32 and the chunk sum is added to an FP64 accumulator.
template <typename T>
struct AccOf { using type = double; };
template <>
struct AccOf<float> { using type = float; };

template <typename VT, typename XT, typename OT, int CPL, int H, int U>
__global__ void __launch_bounds__(256, sizeof(XT) == 4 ? 4 : 3) k_spmm_seg(const int32_t* __restrict__ ci, const VT* __restrict__ val,
                                                     const int32_t* __restrict__ seg_row,
                                                     const int64_t* __restrict__ seg_beg,
                                                     const int64_t* __restrict__ seg_end, int64_t nseg,
                                                     const XT* __restrict__ X, int64_t ldx, int l, bool vec,
                                                     OT* __restrict__ Y, int64_t ldy, double* __restrict__ part) {
    using CT = typename AccOf<XT>::type;  // chunk accumulator: FP32 for FP32 operands
    constexpr int GL = 32 / H;
    const int lane = threadIdx.x & 31;
    const int g = lane / GL, gl = lane % GL;
    const int col0 = gl * CPL;
    const int ncols_here = (l - col0) < CPL ? (l - col0) : CPL;
    const bool active = ncols_here > 0;
    const bool full = vec && ncols_here == CPL;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s = gwarp; s < nseg; s += nwarps) {
        const int32_t rr = __ldg(seg_row + s);
        const int64_t a = __ldg(seg_beg + s), b = __ldg(seg_end + s);
        double acc[CPL];
#pragma unroll
        for (int j = 0; j < CPL; ++j) acc[j] = 0.0;
        int32_t myc = 0;
        VT myv = VT(0);
        if (a + lane < b) { myc = __ldg(ci + a + lane); myv = __ldg(val + a + lane); }
        for (int64_t k0 = a; k0 < b; k0 += 32) {
            const int cnt = (b - k0) < 32 ? (int)(b - k0) : 32;
            // prefetch the next 32 pairs
            int32_t nc = 0;
            VT nv = VT(0);
            if (k0 + 32 + lane < b) { nc = __ldg(ci + k0 + 32 + lane); nv = __ldg(val + k0 + 32 + lane); }
            CT cacc[CPL];
#pragma unroll
            for (int j = 0; j < CPL; ++j) cacc[j] = CT(0);
            for (int qb = 0; qb < cnt; qb += H * U) {
                XT xv[U][CPL];
                CT vq[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int q = qb + u * H + g;
                    const int32_t c = __shfl_sync(0xffffffffu, myc, q & 31);
                    const VT v = __shfl_sync(0xffffffffu, myv, q & 31);
                    const bool ok = q < cnt && active;
                    vq[u] = ok ? (CT)v : CT(0);
                    const XT* p = X + (int64_t)c * ldx + col0;
                    if (ok && full) {
                        if constexpr (sizeof(XT) * CPL <= 16) {
                            const Vec<XT, CPL> t = *reinterpret_cast<const Vec<XT, CPL>*>(p);
#pragma unroll
                            for (int j = 0; j < CPL; ++j) xv[u][j] = t.v[j];
                        } else {
#pragma unroll
                            for (int h = 0; h < CPL / 2; ++h) {
                                const Vec<XT, 2> t = reinterpret_cast<const Vec<XT, 2>*>(p)[h];
                                xv[u][2 * h] = t.v[0];
                                xv[u][2 * h + 1] = t.v[1];
                            }
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < CPL; ++j) xv[u][j] = (ok && j < ncols_here) ? p[j] : XT(0);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int j = 0; j < CPL; ++j) cacc[j] = fma(vq[u], (CT)xv[u][j], cacc[j]);
            }
#pragma unroll
            for (int j = 0; j < CPL; ++j) acc[j] += (double)cacc[j];
            myc = nc;
            myv = nv;
        }
        if (H == 2) {
#pragma unroll
            for (int j = 0; j < CPL; ++j) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], 16);
        }
        if (g == 0 && active) {
            if (rr >= 0) store_cols<OT, CPL>(Y + (int64_t)rr * ldy + col0, ncols_here, acc);
            else store_cols<double, CPL>(part + s * (int64_t)l + col0, ncols_here, acc);
        }
    }
}

// rows split into several segments: add their partials in segment order
template <typename OT>
__global__ void k_spmm_merge(const int64_t* __restrict__ seg_first, const int32_t* __restrict__ multi_rows,
                             int64_t nmulti, const double* __restrict__ part, int l, OT* __restrict__ Y,
                             int64_t ldy) {
    const int lane = threadIdx.x & 31;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t t = gwarp; t < nmulti; t += nwarps) {
        const int64_t r = multi_rows[t];
        const int64_t f = seg_first[r], f1 = seg_first[r + 1];
        for (int c = lane; c < l; c += 32) {
            double acc = 0.0;
            for (int64_t s = f; s < f1; ++s) acc += part[s * (int64_t)l + c];
            Y[r * ldy + c] = (OT)acc;
        }
    }
}

// ------------------------------------------------------------- the plan --
__global__ void k_seg_count(const int64_t* __restrict__ rp, int64_t rows, int64_t* __restrict__ cnt) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r <= rows; r += (int64_t)gridDim.x * blockDim.x) {
        if (r == rows) { cnt[r] = 0; continue; }
        const int64_t len = rp[r + 1] - rp[r];
        cnt[r] = len <= kSegNnz ? 1 : (len + kSegNnz - 1) / kSegNnz;
    }
}
__global__ void k_seg_fill(const int64_t* __restrict__ rp, const int64_t* __restrict__ first, int64_t rows,
                           int32_t* __restrict__ seg_row, int64_t* __restrict__ seg_beg, int64_t* __restrict__ seg_end,
                           int32_t* __restrict__ multi_rows, unsigned long long* __restrict__ nmulti) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t f = first[r], f1 = first[r + 1], e = rp[r + 1];
        const bool multi = f1 - f > 1;
        for (int64_t s = f; s < f1; ++s) {
            const int64_t a = rp[r] + (s - f) * kSegNnz;
            seg_row[s] = multi ? -(int32_t)r - 1 : (int32_t)r;
            seg_beg[s] = a;
            seg_end[s] = (a + kSegNnz < e) ? a + kSegNnz : e;
        }
        if (multi) multi_rows[atomicAdd(nmulti, 1ull)] = (int32_t)r;  // order is irrelevant to the sums
    }
}

__global__ void k_bin_flags(const int64_t* __restrict__ rp, int64_t rows, int64_t lo, int64_t hi,
                            uint8_t* __restrict__ flag, int32_t* __restrict__ ids) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t len = rp[r + 1] - rp[r];
        flag[r] = (len > lo && len <= hi) ? 1 : 0;
        ids[r] = (int32_t)r;
    }
}

static int nblk(int64_t work, int threads, int per_sm) {
    int64_t b = (work + threads - 1) / threads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)device_props().sms * per_sm));
}

void build_seg_plan(DevCompressed& m, cudaStream_t s) {
    SegPlan& p = m.plan;
    const int64_t rows = m.nmajor;
    p.seg_first.alloc(rows + 1, s);
    if (rows == 0) {
        SVDB_CUDA(cudaMemsetAsync(p.seg_first.p, 0, sizeof(int64_t), s));
        p.nseg = p.nmulti = 0;
        return;
    }
    DevBuf<int64_t> cnt(rows + 1, s);
    k_seg_count<<<nblk(rows + 1, 256, 16), 256, 0, s>>>(m.ptr.p, rows, cnt.p);
    SVDB_CHECK_LAUNCH();
    size_t tb = 0;
    SVDB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.p, p.seg_first.p, rows + 1, s));
    DevBuf<uint8_t> tmp(std::max<size_t>(tb, 1), s);
    SVDB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.p, p.seg_first.p, rows + 1, s));
    int64_t nseg = 0;
    SVDB_CUDA(cudaMemcpyAsync(&nseg, p.seg_first.p + rows, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaStreamSynchronize(s));
    p.nseg = nseg;
    p.seg_row.alloc(std::max<int64_t>(nseg, 1), s);
    p.seg_beg.alloc(std::max<int64_t>(nseg, 1), s);
    p.seg_end.alloc(std::max<int64_t>(nseg, 1), s);
    p.multi_rows.alloc(std::max<int64_t>(rows, 1), s);
    DevBuf<unsigned long long> nm(1, s);
    SVDB_CUDA(cudaMemsetAsync(nm.p, 0, sizeof(unsigned long long), s));
    k_seg_fill<<<nblk(rows, 256, 16), 256, 0, s>>>(m.ptr.p, p.seg_first.p, rows, p.seg_row.p, p.seg_beg.p,
                                                   p.seg_end.p, p.multi_rows.p, nm.p);
    SVDB_CHECK_LAUNCH();
    unsigned long long hm = 0;
    SVDB_CUDA(cudaMemcpyAsync(&hm, nm.p, sizeof(hm), cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaStreamSynchronize(s));
    p.nmulti = (int64_t)hm;

    // SpMV bins: a stable partition of the rows by length
    p.bin_rows.alloc(std::max<int64_t>(rows, 1), s);
    DevBuf<uint8_t> flag(rows, s);
    DevBuf<int32_t> ids(rows, s);
    DevBuf<int64_t> nsel(1, s);
    size_t tb2 = 0;
    SVDB_CUDA(cub::DeviceSelect::Flagged(nullptr, tb2, ids.p, flag.p, p.bin_rows.p, nsel.p, rows, s));
    DevBuf<uint8_t> tmp2(std::max<size_t>(tb2, 1), s);
    int64_t off = 0, items = 0;
    for (int b = 0; b < kSpmvBins; ++b) {
        const int64_t lo = b ? kSpmvBinLen[b - 1] : -1, hi = kSpmvBinLen[b];
        k_bin_flags<<<nblk(rows, 256, 16), 256, 0, s>>>(m.ptr.p, rows, lo, hi, flag.p, ids.p);
        SVDB_CHECK_LAUNCH();
        SVDB_CUDA(cub::DeviceSelect::Flagged(tmp2.p, tb2, ids.p, flag.p, p.bin_rows.p + off, nsel.p, rows, s));
        int64_t cnt = 0;
        SVDB_CUDA(cudaMemcpyAsync(&cnt, nsel.p, sizeof(cnt), cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
        p.bins.off[b] = off;
        p.bins.items[b] = items;
        const int64_t rpw = 32 / (2 << b);
        off += cnt;
        items += (cnt + rpw - 1) / rpw;
    }
    p.bins.off[kSpmvBins] = off;
    p.bins.items[kSpmvBins] = items;
    p.bins.rows = p.bin_rows.p;
}

// ------------------------------------------------------------- launcher --
template <typename VT, typename XT, typename OT, int CPL, int H>
static void launch_seg(const DevCompressed& m, const VT* v, const XT* X, int64_t ldx, int lc, OT* Y, int64_t ldy,
                       double* part, cudaStream_t s) {
    const uintptr_t align = std::min<uintptr_t>(16, sizeof(XT) * CPL);
    const bool vec = (CPL > 1) && (ldx % CPL == 0) && ((reinterpret_cast<uintptr_t>(X) % align) == 0);
    const int blocks = nblk(m.plan.nseg * 32, 256, 16);
    constexpr int U = 4;
    k_spmm_seg<VT, XT, OT, CPL, H, U><<<blocks, 256, 0, s>>>(m.idx.p, v, m.plan.seg_row.p, m.plan.seg_beg.p,
                                                             m.plan.seg_end.p, m.plan.nseg, X, ldx, lc, vec, Y,
                                                             ldy, part);
    SVDB_CHECK_LAUNCH();
}

template <typename VT, typename XT, typename OT>
static void spmm_impl(const DevCompressed& m, const VT* v, const XT* X, int l, OT* Y, cudaStream_t s) {
    DevBuf<double> part;
    if (m.plan.nmulti) part.alloc(m.plan.nseg * (int64_t)std::min(l, 128), s);
    for (int c0 = 0; c0 < l; c0 += 128) {
        const int lc = std::min(128, l - c0);
        const XT* Xc = X + c0;
        OT* Yc = Y + c0;
        if (lc <= 32) launch_seg<VT, XT, OT, 2, 2>(m, v, Xc, l, lc, Yc, l, part.p, s);
        else if (lc <= 64) launch_seg<VT, XT, OT, 4, 2>(m, v, Xc, l, lc, Yc, l, part.p, s);
        else launch_seg<VT, XT, OT, 4, 1>(m, v, Xc, l, lc, Yc, l, part.p, s);
        if (m.plan.nmulti) {
            k_spmm_merge<OT><<<nblk(m.plan.nmulti * 32, 256, 16), 256, 0, s>>>(
                m.plan.seg_first.p, m.plan.multi_rows.p, m.plan.nmulti, part.p, lc, Yc, l);
            SVDB_CHECK_LAUNCH();
        }
    }
}

template <typename XT, typename OT>
void spmm_dev(const DevCompressed& m, bool fp32, const XT* X, int l, OT* Y, cudaStream_t s) {
    if (m.nmajor == 0 || l == 0) return;
    if (fp32 && m.val32.p) spmm_impl<float, XT, OT>(m, m.val32.p, X, l, Y, s);
    else spmm_impl<double, XT, OT>(m, m.val.p, X, l, Y, s);
}

template void spmm_dev<double, double>(const DevCompressed&, bool, const double*, int, double*, cudaStream_t);
template void spmm_dev<float, float>(const DevCompressed&, bool, const float*, int, float*, cudaStream_t);
template void spmm_dev<float, double>(const DevCompressed&, bool, const float*, int, double*, cudaStream_t);

}  // namespace svdb
