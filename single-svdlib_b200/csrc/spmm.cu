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
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <string>
#include <type_traits>

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

// Lean gather kernel: values and dense operand of one type T (float or
// double), l <= 64 (H = 2) or <= 32 (H = 4), rows of X 16-byte aligned: the
// same segments, lane groups and summation order as k_spmm_seg (group g takes
// entries g, g + H, ... of a 32-entry chunk; FP32 sums within a chunk and
// FP64 across chunks for float, FP64 throughout for double), with fewer
// instructions per entry.  k_spmm_seg spent about 21 warp instructions per
// nonzero at FP32 (its shuffles, 64-bit address arithmetic and per-entry
// bounds tests), and with X resident in L1 it was bound by instruction issue,
// not by memory.  Here a chunk's (row offset, value) pairs are written once to
// a per-warp shared buffer and read back by broadcast, offsets are 32-bit, and
// full chunks run without bounds tests with U gathers in flight per lane.
constexpr int kF32Warps = 8;
template <typename T>
struct LeanEntry;
template <>
struct alignas(8) LeanEntry<float> { int32_t off; float v; };
template <>
struct alignas(16) LeanEntry<double> { int32_t off; int32_t pad; double v; };

// four consecutive elements of a row (16-byte aligned)
__device__ __forceinline__ void load4(const float* p, float (&x)[4]) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    x[0] = t.x; x[1] = t.y; x[2] = t.z; x[3] = t.w;
}
__device__ __forceinline__ void load4(const double* p, double (&x)[4]) {
    const double2 t0 = reinterpret_cast<const double2*>(p)[0], t1 = reinterpret_cast<const double2*>(p)[1];
    x[0] = t0.x; x[1] = t0.y; x[2] = t1.x; x[3] = t1.y;
}

template <typename T, typename OT, int H, int U, int MINB>
__global__ void __launch_bounds__(kF32Warps * 32, MINB)
    k_spmm_lean(const int32_t* __restrict__ ci, const T* __restrict__ val, const int32_t* __restrict__ seg_row,
                const int64_t* __restrict__ seg_beg, const int64_t* __restrict__ seg_end, int64_t nseg,
                const T* __restrict__ X, int32_t ldx, int l, OT* __restrict__ Y, int64_t ldy,
                double* __restrict__ part) {
    using CT = typename AccOf<T>::type;  // chunk sums: FP32 for float, FP64 for double
    constexpr int GL = 32 / H;           // lanes per group
    constexpr int PER = 32 / H;          // entries of a chunk per group
    __shared__ LeanEntry<T> s_ent[kF32Warps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane / GL, gl = lane % GL;
    const int col0 = gl * 4;
    const int ncols_here = (l - col0) < 4 ? (l - col0) : 4;
    const bool active = ncols_here > 0;
    const uint32_t c0a = active ? (uint32_t)col0 : 0u;  // gathers at X + a 32-bit offset
    LeanEntry<T>* E = s_ent[w];
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t sg = gwarp; sg < nseg; sg += nwarps) {
        const int32_t rr = __ldg(seg_row + sg);
        const int64_t a = __ldg(seg_beg + sg), b = __ldg(seg_end + sg);
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        int32_t myc = 0;
        T myv = T(0);
        if (a + lane < b) { myc = __ldg(ci + a + lane); myv = __ldg(val + a + lane); }
        for (int64_t k0 = a; k0 < b; k0 += 32) {
            const int cnt = (b - k0) < 32 ? (int)(b - k0) : 32;
            __syncwarp();  // the previous chunk's entries have been read
            LeanEntry<T> en;
            en.off = myc * ldx;
            en.v = myv;
            E[lane] = en;
            __syncwarp();
            if (k0 + 32 + lane < b) {  // the next chunk's pairs, while this one is used
                myc = __ldg(ci + k0 + 32 + lane);
                myv = __ldg(val + k0 + 32 + lane);
            }
            CT c4[4] = {CT(0), CT(0), CT(0), CT(0)};
            if (cnt == 32) {
#pragma unroll 1
                for (int qb = 0; qb < PER; qb += U) {  // batches of U gathers, one batch live at a time
                    T xv[U][4];
                    T vv[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const LeanEntry<T> e = E[(qb + u) * H + g];
                        vv[u] = e.v;
                        if (active) load4(X + ((uint32_t)e.off + c0a), xv[u]);
                        else xv[u][0] = xv[u][1] = xv[u][2] = xv[u][3] = T(0);
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u)
#pragma unroll
                        for (int j = 0; j < 4; ++j) c4[j] = fma((CT)vv[u], (CT)xv[u][j], c4[j]);
                }
            } else {
                for (int q = g; q < cnt; q += H) {
                    const LeanEntry<T> e = E[q];
                    T x[4] = {T(0), T(0), T(0), T(0)};
                    if (active) load4(X + ((uint32_t)e.off + c0a), x);
#pragma unroll
                    for (int j = 0; j < 4; ++j) c4[j] = fma((CT)e.v, (CT)x[j], c4[j]);
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[j] += (double)c4[j];
        }
#pragma unroll
        for (int o = GL; o < 32; o <<= 1)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
        if (g == 0 && active) {
            if (rr >= 0) store_cols<OT, 4>(Y + (int64_t)rr * ldy + col0, ncols_here, acc);
            else store_cols<double, 4>(part + sg * (int64_t)l + col0, ncols_here, acc);
        }
    }
}

// The FP32 form, kept apart from the template: its own instruction schedule
// measured 7 % faster than k_spmm_lean<float> on the 100k x 30k workload.
template <typename OT, int H>
__global__ void __launch_bounds__(kF32Warps * 32, 4)
    k_spmm_f32(const int32_t* __restrict__ ci, const float* __restrict__ val, const int32_t* __restrict__ seg_row,
               const int64_t* __restrict__ seg_beg, const int64_t* __restrict__ seg_end, int64_t nseg,
               const float* __restrict__ X, int32_t ldx, int l, OT* __restrict__ Y, int64_t ldy,
               double* __restrict__ part) {
    constexpr int GL = 32 / H;        // lanes per group
    constexpr int PER = 32 / H;       // entries of a chunk per group
    constexpr int U = 8;              // gathers in flight per lane
    __shared__ int2 s_ent[kF32Warps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane / GL, gl = lane % GL;
    const int col0 = gl * 4;
    const int ncols_here = (l - col0) < 4 ? (l - col0) : 4;
    const bool active = ncols_here > 0;
    // gathers address X + (32-bit offset): the base is the same for every
    // lane, which saves the 64-bit per-lane address arithmetic (4 % per pass)
    const uint32_t c0a = active ? (uint32_t)col0 : 0u;
    int2* E = s_ent[w];
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t sg = gwarp; sg < nseg; sg += nwarps) {
        const int32_t rr = __ldg(seg_row + sg);
        const int64_t a = __ldg(seg_beg + sg), b = __ldg(seg_end + sg);
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        int32_t myc = 0;
        float myv = 0.f;
        if (a + lane < b) { myc = __ldg(ci + a + lane); myv = __ldg(val + a + lane); }
        for (int64_t k0 = a; k0 < b; k0 += 32) {
            const int cnt = (b - k0) < 32 ? (int)(b - k0) : 32;
            __syncwarp();  // the previous chunk's entries have been read
            E[lane] = make_int2(myc * ldx, __float_as_int(myv));
            __syncwarp();
            if (k0 + 32 + lane < b) {  // the next chunk's pairs, while this one is used
                myc = __ldg(ci + k0 + 32 + lane);
                myv = __ldg(val + k0 + 32 + lane);
            }
            float c4[4] = {0.f, 0.f, 0.f, 0.f};
            if (cnt == 32) {
#pragma unroll 1
                for (int qb = 0; qb < PER; qb += U) {  // batches of U gathers, one batch live at a time
                    float4 xv[U];
                    float vv[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int2 e = E[(qb + u) * H + g];
                        vv[u] = __int_as_float(e.y);
                        xv[u] = active ? *reinterpret_cast<const float4*>(X + ((uint32_t)e.x + c0a))
                                       : make_float4(0.f, 0.f, 0.f, 0.f);
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        c4[0] = fmaf(vv[u], xv[u].x, c4[0]);
                        c4[1] = fmaf(vv[u], xv[u].y, c4[1]);
                        c4[2] = fmaf(vv[u], xv[u].z, c4[2]);
                        c4[3] = fmaf(vv[u], xv[u].w, c4[3]);
                    }
                }
            } else {
                for (int q = g; q < cnt; q += H) {
                    const int2 e = E[q];
                    const float v = __int_as_float(e.y);
                    const float4 x = active ? *reinterpret_cast<const float4*>(X + ((uint32_t)e.x + c0a))
                                            : make_float4(0.f, 0.f, 0.f, 0.f);
                    c4[0] = fmaf(v, x.x, c4[0]);
                    c4[1] = fmaf(v, x.y, c4[1]);
                    c4[2] = fmaf(v, x.z, c4[2]);
                    c4[3] = fmaf(v, x.w, c4[3]);
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[j] += (double)c4[j];
        }
#pragma unroll
        for (int o = GL; o < 32; o <<= 1)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
        if (g == 0 && active) {
            if (rr >= 0) store_cols<OT, 4>(Y + (int64_t)rr * ldy + col0, ncols_here, acc);
            else store_cols<double, 4>(part + sg * (int64_t)l + col0, ncols_here, acc);
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
                       double* part, cudaStream_t s, int64_t lo = 0, int64_t hi = -1) {
    if (hi < 0) hi = m.plan.nseg;
    if (hi <= lo) return;
    const uintptr_t align = std::min<uintptr_t>(16, sizeof(XT) * CPL);
    const bool vec = (CPL > 1) && (ldx % CPL == 0) && ((reinterpret_cast<uintptr_t>(X) % align) == 0);
    const int blocks = nblk((hi - lo) * 32, 256, 16);
    constexpr int U = 4;
    // segment s of the range is segment lo + s of the plan; its partial row lives at part[(lo + s) * lc]
    k_spmm_seg<VT, XT, OT, CPL, H, U><<<blocks, 256, 0, s>>>(m.idx.p, v, m.plan.seg_row.p + lo, m.plan.seg_beg.p + lo,
                                                             m.plan.seg_end.p + lo, hi - lo, X, ldx, lc, vec, Y,
                                                             ldy, part ? part + lo * (int64_t)lc : nullptr);
    SVDB_CHECK_LAUNCH();
}

// k_spmm_lean applies: values and operand of one type, l <= 64 and a
// multiple of 4, a 16-byte aligned operand with rows of a 16-byte multiple,
// 32-bit element offsets (nminor * ldx < 2^31), and SVDB_SPMM=seg not set
// (that keeps k_spmm_seg, for comparisons)
template <typename VT, typename XT>
static bool lean_eligible(const DevCompressed& m, const XT* X, int l, int64_t ldx) {
    if constexpr (!std::is_same<VT, XT>::value) {
        return false;
    } else {
        const char* e = getenv("SVDB_SPMM");
        if (e && std::string(e) == "seg") return false;
        return l >= 1 && l <= 64 && l % 4 == 0 && ldx >= l && (ldx * (int64_t)sizeof(XT)) % 16 == 0 &&
               (reinterpret_cast<uintptr_t>(X) % 16) == 0 && m.nminor * ldx < ((int64_t)1 << 31);
    }
}

// FP32: 64 registers and four blocks per SM with eight gathers in flight per
// lane (1.10 ms for A X of the 100k x 30k workload, against 1.64 ms at two
// blocks and 1.33-1.36 ms at three); FP64: four gathers in flight, three blocks.
template <typename T, typename OT>
static void launch_lean(const DevCompressed& m, const T* v, const T* X, int l, OT* Y, double* part,
                        cudaStream_t s, int64_t ldx = 0) {
    if (ldx == 0) ldx = l;
    const int64_t ns = m.plan.nseg;
    if (ns <= 0) return;
    constexpr bool f32 = std::is_same<T, float>::value;
    constexpr int U = f32 ? 8 : 4, MINB = f32 ? 4 : 3;
    // 8x the resident blocks: timed against the resident blocks only, 1.10
    // against 1.20 ms for A X of the 100k x 30k workload
    const int blocks = nblk(ns * 32, kF32Warps * 32, MINB * 8);
    if constexpr (f32) {
        if (l <= 32)
            k_spmm_f32<OT, 4><<<blocks, kF32Warps * 32, 0, s>>>(m.idx.p, v, m.plan.seg_row.p, m.plan.seg_beg.p,
                                                                m.plan.seg_end.p, ns, X, (int32_t)ldx, l, Y, l, part);
        else
            k_spmm_f32<OT, 2><<<blocks, kF32Warps * 32, 0, s>>>(m.idx.p, v, m.plan.seg_row.p, m.plan.seg_beg.p,
                                                                m.plan.seg_end.p, ns, X, (int32_t)ldx, l, Y, l, part);
    } else {
        if (l <= 32)
            k_spmm_lean<T, OT, 4, U, MINB><<<blocks, kF32Warps * 32, 0, s>>>(
                m.idx.p, v, m.plan.seg_row.p, m.plan.seg_beg.p, m.plan.seg_end.p, ns, X, (int32_t)ldx, l, Y, l, part);
        else
            k_spmm_lean<T, OT, 2, U, MINB><<<blocks, kF32Warps * 32, 0, s>>>(
                m.idx.p, v, m.plan.seg_row.p, m.plan.seg_beg.p, m.plan.seg_end.p, ns, X, (int32_t)ldx, l, Y, l, part);
    }
    SVDB_CHECK_LAUNCH();
}

template <typename VT, typename XT, typename OT>
static void spmm_impl(const DevCompressed& m, const VT* v, const XT* X, int l, OT* Y, cudaStream_t s) {
    DevBuf<double> part;
    if (m.plan.nmulti) part.alloc(m.plan.nseg * (int64_t)std::min(l, 128), s);
    if constexpr (std::is_same<VT, XT>::value) {
        if (lean_eligible<VT, XT>(m, X, l, l)) {
            launch_lean<VT, OT>(m, v, X, l, Y, part.p, s);
            if (m.plan.nmulti) {
                k_spmm_merge<OT><<<nblk(m.plan.nmulti * 32, 256, 16), 256, 0, s>>>(
                    m.plan.seg_first.p, m.plan.multi_rows.p, m.plan.nmulti, part.p, l, Y, l);
                SVDB_CHECK_LAUNCH();
            }
            return;
        }
    }
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


// ------------------------------------------------------ TMA row gathers --
// FP32 dense operand, FP32 matrix values: the rows X[c] of a chunk of 32
// entries are fetched by the tensor memory accelerator (tile::gather4: four
// rows of one box each, the box one row high and BOXW columns wide; columns
// past l read as zero) into a per-warp shared-memory ring of kTS chunks, so
// the bytes in flight cost no registers.  Each warp owns whole segments of
// the plan; a chunk's sums are FP32, chunks are added in FP64 as in
// k_spmm_seg.  Waits on the ring's mbarriers give up after 2 s of
// %globaltimer and raise g_tma_err (read by spmm_tma_check).
constexpr int kTW = 8;   // warps per CTA
constexpr int kTS = 3;   // chunks in flight per warp
constexpr int kTE = 32;  // entries per chunk
__device__ int g_tma_err;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = gtimer();
    while (!mbar_try_wait(bar, parity))
        if (gtimer() - t0 > limit_ns) return false;
    return true;
}

template <typename OT, int BOXW>
__global__ void __launch_bounds__(kTW * 32, 1) k_spmm_tma(const __grid_constant__ CUtensorMap xmap,
                                                           const int32_t* __restrict__ ci,
                                                           const float* __restrict__ val,
                                                           const int32_t* __restrict__ seg_row,
                                                           const int64_t* __restrict__ seg_beg,
                                                           const int64_t* __restrict__ seg_end, int64_t nseg, int l,
                                                           OT* __restrict__ Y, int64_t ldy,
                                                           double* __restrict__ part) {
    constexpr int ROWB = BOXW * 4;            // bytes of one gathered row
    constexpr int CHUNKB = kTE * ROWB;        // bytes of one chunk
    constexpr int CPL = BOXW / 32;            // columns per lane
    const unsigned full = 0xffffffffu;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[kTW][kTS];
    __shared__ float svals[kTW][kTS][kTE];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (smem_u32(smem) & 127) {  // TMA destinations need 128-byte alignment
        if (threadIdx.x == 0) atomicOr(&g_tma_err, 2);
        return;
    }
    unsigned char* ring = smem + (size_t)w * kTS * CHUNKB;
    if (lane == 0) {
        for (int st = 0; st < kTS; ++st)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[w][st])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    const int64_t nw = (int64_t)gridDim.x * kTW;
    int64_t i_sg = blockIdx.x * (int64_t)kTW + w, i_k0 = i_sg < nseg ? seg_beg[i_sg] : 0;
    int64_t c_sg = i_sg, c_k0 = i_k0;
    int issued = 0, consumed = 0;

    auto issue = [&]() {
        if (i_sg >= nseg) return;
        const int64_t e = seg_end[i_sg];
        const int cnt = (int)min((int64_t)kTE, e - i_k0);
        const int st = issued % kTS;
        const int32_t cm = lane < cnt ? __ldg(ci + i_k0 + lane) : 0;
        svals[w][st][lane] = lane < cnt ? __ldg(val + i_k0 + lane) : 0.f;
        const int ng = (cnt + 3) >> 2;
        int32_t r[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int32_t cu = __shfl_sync(full, cm, (4 * lane + u) & 31);
            const int32_t cb = __shfl_sync(full, cm, (4 * lane) & 31);
            r[u] = (4 * lane + u < cnt) ? cu : cb;  // pad a short group with its first row
        }
        const uint32_t bar = smem_u32(&bars[w][st]);
        if (lane == 0)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(ng * 4 * ROWB)
                         : "memory");
        __syncwarp();
        if (lane < ng) {
            const uint32_t dst = smem_u32(ring + st * CHUNKB + lane * 4 * ROWB);
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
                " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
                "l"(reinterpret_cast<uint64_t>(&xmap)), "r"(0), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(bar)
                : "memory");
        }
        ++issued;
        i_k0 += kTE;
        if (i_k0 >= e) {
            i_sg += nw;
            if (i_sg < nseg) i_k0 = seg_beg[i_sg];
        }
    };

#pragma unroll
    for (int p = 0; p < kTS; ++p) issue();
    double acc[CPL];
#pragma unroll
    for (int u = 0; u < CPL; ++u) acc[u] = 0.0;
    bool failed = false;
    while (consumed < issued) {
        const int st = consumed % kTS;
        if (!mbar_wait_bounded(smem_u32(&bars[w][st]), (uint32_t)((consumed / kTS) & 1), 2000000000ull)) {
            failed = true;
            break;
        }
        const int64_t e = seg_end[c_sg];
        const int cnt = (int)min((int64_t)kTE, e - c_k0);
        const float v = svals[w][st][lane];
        const float* xs = reinterpret_cast<const float*>(ring + st * CHUNKB) + CPL * lane;
        float sum[CPL];
#pragma unroll
        for (int u = 0; u < CPL; ++u) sum[u] = 0.f;
#pragma unroll 4
        for (int q = 0; q < cnt; ++q) {
            const float vq = __shfl_sync(full, v, q);
            if (CPL == 2) {
                const float2 x = *reinterpret_cast<const float2*>(xs + q * BOXW);
                sum[0] = fmaf(vq, x.x, sum[0]);
                sum[CPL - 1] = fmaf(vq, x.y, sum[CPL - 1]);
            } else {
                sum[0] = fmaf(vq, xs[q * BOXW], sum[0]);
            }
        }
#pragma unroll
        for (int u = 0; u < CPL; ++u) acc[u] += (double)sum[u];
        __syncwarp();
        ++consumed;
        c_k0 += kTE;
        if (c_k0 >= e) {
            const int32_t rr = seg_row[c_sg];
#pragma unroll
            for (int u = 0; u < CPL; ++u) {
                const int col = CPL * lane + u;
                if (col < l) {
                    if (rr >= 0) Y[(int64_t)rr * ldy + col] = (OT)acc[u];
                    else part[c_sg * (int64_t)l + col] = acc[u];
                }
                acc[u] = 0.0;
            }
            c_sg += nw;
            if (c_sg < nseg) c_k0 = seg_beg[c_sg];
        }
        issue();
    }
    if (failed) {
        if (lane == 0) atomicOr(&g_tma_err, 1);
        // let the copies already issued land before the ring goes away (bounded)
        for (; consumed < issued; ++consumed)
            mbar_wait_bounded(smem_u32(&bars[w][consumed % kTS]), (uint32_t)((consumed / kTS) & 1), 100000000ull);
    }
}

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// TMA path (opt-in, SVDB_SPMM=tma): FP32 operand with contiguous rows of l
// (a multiple of 4, at most 64) on a 16-byte aligned base.  On B200 it moved
// about 4.9 TB/s of 256-byte rows against 7.4 TB/s for the register gathers
// of k_spmm_seg (100,000 x 30,000, 65 M nonzeros, l = 60), and splitting the
// segments between the two kernels on two streams was no faster than
// k_spmm_seg alone: both are held by the same L2 gather traffic.  So it is
// not the default; the variable is read on every call.
static bool tma_eligible(const void* X, int l, int64_t ldx) {
    const char* e = getenv("SVDB_SPMM");
    const bool on = e && std::string(e) == "tma";
    return on && ldx == l && l % 4 == 0 && l <= 64 && (reinterpret_cast<uintptr_t>(X) % 16) == 0 && encode_fn();
}

template <typename OT>
static void launch_tma(const DevCompressed& m, const float* v, const float* X, int l, OT* Y, double* part,
                       cudaStream_t s, int64_t lo = 0, int64_t hi = -1, bool merge = true) {
    if (hi < 0) hi = m.plan.nseg;
    const int boxw = l <= 32 ? 32 : 64;
    CUtensorMap map;
    cuuint64_t gdim[2] = {(cuuint64_t)l, (cuuint64_t)m.nminor};
    cuuint64_t gstr[1] = {(cuuint64_t)l * 4};
    cuuint32_t box[2] = {(cuuint32_t)boxw, 1};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(X), gdim, gstr, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(SVDB_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    const size_t smem = (size_t)kTW * kTS * kTE * boxw * 4;
    const int64_t ns = hi - lo;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((ns + kTW - 1) / kTW, (int64_t)device_props().sms));
    double* pp = part ? part + lo * (int64_t)l : nullptr;
    if (ns > 0) {
        if (boxw == 32) {
            SVDB_CUDA(cudaFuncSetAttribute(k_spmm_tma<OT, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_spmm_tma<OT, 32><<<blocks, kTW * 32, smem, s>>>(map, m.idx.p, v, m.plan.seg_row.p + lo,
                                                              m.plan.seg_beg.p + lo, m.plan.seg_end.p + lo, ns, l, Y,
                                                              l, pp);
        } else {
            SVDB_CUDA(cudaFuncSetAttribute(k_spmm_tma<OT, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_spmm_tma<OT, 64><<<blocks, kTW * 32, smem, s>>>(map, m.idx.p, v, m.plan.seg_row.p + lo,
                                                              m.plan.seg_beg.p + lo, m.plan.seg_end.p + lo, ns, l, Y,
                                                              l, pp);
        }
        SVDB_CHECK_LAUNCH();
    }
    if (merge && m.plan.nmulti) {
        k_spmm_merge<OT><<<nblk(m.plan.nmulti * 32, 256, 16), 256, 0, s>>>(m.plan.seg_first.p, m.plan.multi_rows.p,
                                                                          m.plan.nmulti, part, l, Y, l);
        SVDB_CHECK_LAUNCH();
    }
}

void spmm_tma_check() {
    int e = 0;
    SVDB_CUDA(cudaMemcpyFromSymbol(&e, g_tma_err, sizeof(int)));
    if (e) {
        const int z = 0;
        SVDB_CUDA(cudaMemcpyToSymbol(g_tma_err, &z, sizeof(int)));
        if (e & 2) throw Error(SVDB_ERR_CUDA, "SpMM: shared-memory ring not 128-byte aligned; no gather was issued");
        throw Error(SVDB_ERR_TIMEOUT, "SpMM: a tensor-memory gather did not complete within 2 s");
    }
}

// The rows the panel kernel leaves to the segment kernel: an explicit list
// of segments (row < 0: partial k of the list, at part[k * l]).
static void heavy_segments_f32(const DevCompressed& m, const int32_t* row, const int64_t* beg, const int64_t* end,
                               int64_t n, const float* X, int l, double* Y, double* part, cudaStream_t s) {
    if (n <= 0) return;
    const uintptr_t align = 16;
    const bool vec = (l % 4 == 0) && ((reinterpret_cast<uintptr_t>(X) % align) == 0);
    const int blocks = nblk(n * 32, 256, 16);
    if (l <= 32)
        k_spmm_seg<float, float, double, 2, 2, 4><<<blocks, 256, 0, s>>>(m.idx.p, m.val32.p, row, beg, end, n, X, l,
                                                                         l, vec, Y, l, part);
    else
        k_spmm_seg<float, float, double, 4, 2, 4><<<blocks, 256, 0, s>>>(m.idx.p, m.val32.p, row, beg, end, n, X, l,
                                                                         l, vec, Y, l, part);
    SVDB_CHECK_LAUNCH();
}

// FP32 products with the dense operand's rows ldx floats apart (ldx >= l, a
// multiple of 32: every row starts on a 128-byte line, so a gathered row of
// l <= 64 floats touches whole lines only).  False when k_spmm_lean does not
// apply (the caller then keeps the unpadded path).
bool spmm_f32_strided_ok(const DevCompressed& m, int l, int64_t ldx) {
    const char* e = getenv("SVDB_SPMM");
    if (e && *e) return false;  // an explicit kernel choice keeps the unpadded path
    return m.val32.p && m.nnz > 0 && l >= 1 && l <= 64 && l % 4 == 0 && ldx >= l && ldx % 32 == 0 &&
           m.nminor * ldx < ((int64_t)1 << 31);
}

void spmm_f32_strided(const DevCompressed& m, const float* X, int l, int64_t ldx, double* Y, cudaStream_t s) {
    if (m.nmajor == 0) return;
    if (!spmm_f32_strided_ok(m, l, ldx) || (reinterpret_cast<uintptr_t>(X) % 16))
        throw Error(SVDB_ERR_ARG, "spmm_f32_strided: operand layout not supported");
    DevBuf<double> part;
    if (m.plan.nmulti) part.alloc(m.plan.nseg * (int64_t)l, s);
    launch_lean<float, double>(m, m.val32.p, X, l, Y, part.p, s, ldx);
    if (m.plan.nmulti) {
        k_spmm_merge<double><<<nblk(m.plan.nmulti * 32, 256, 16), 256, 0, s>>>(m.plan.seg_first.p, m.plan.multi_rows.p,
                                                                              m.plan.nmulti, part.p, l, Y, l);
        SVDB_CHECK_LAUNCH();
    }
}

template <typename XT, typename OT>
void spmm_dev(const DevCompressed& m, bool fp32, const XT* X, int l, OT* Y, cudaStream_t s) {
    if (m.nmajor == 0 || l == 0) return;
    if constexpr (std::is_same<XT, float>::value && std::is_same<OT, double>::value) {
        if (fp32 && spmm_panel_eligible(m, l, X) &&
            spmm_panel(const_cast<DevCompressed&>(m), X, l, Y, s, heavy_segments_f32))
            return;
    }
    if constexpr (std::is_same<XT, float>::value) {
        if (fp32 && m.val32.p && m.nnz > 0 && tma_eligible(X, l, l)) {
            DevBuf<double> part;
            if (m.plan.nmulti) part.alloc(m.plan.nseg * (int64_t)l, s);
            launch_tma<OT>(m, m.val32.p, X, l, Y, part.p, s);
            return;
        }
    }
    if (fp32 && m.val32.p) spmm_impl<float, XT, OT>(m, m.val32.p, X, l, Y, s);
    else spmm_impl<double, XT, OT>(m, m.val.p, X, l, Y, s);
}

template void spmm_dev<double, double>(const DevCompressed&, bool, const double*, int, double*, cudaStream_t);
template void spmm_dev<float, float>(const DevCompressed&, bool, const float*, int, float*, cudaStream_t);
template void spmm_dev<float, double>(const DevCompressed&, bool, const float*, int, double*, cudaStream_t);

}  // namespace svdb
