// Device side of the sparse matrix-vector product, shared by the standalone
// kernels (ops.cu) and the cooperative Lanczos kernel.
//
// Rows of at most kSegNnz entries are taken by groups of G lanes; longer rows
// (the segment plan's multi-segment rows) by a whole block each, so that a
// 20,000-entry row does not hold one warp while the rest of the grid idles.
// Each lane keeps kSpmvUnroll independent (index, value, gather) chains in
// flight and sums them in a fixed order, so the result does not depend on
// the grid size.
#pragma once

#include <cstdint>

#include "device_common.cuh"
#include "svdb_internal.h"

namespace svdb {

constexpr int kSpmvUnroll = 4;

// sum of v[k] * xload(ci[k]) over the entries k = s + sub + G (kSpmvUnroll t + u)
// of [s, e) owned by lane `sub` of a G-lane group
template <typename VT, typename XL>
__device__ __forceinline__ double row_dot(const int32_t* __restrict__ ci, const VT* __restrict__ v, int64_t s,
                                          int64_t e, int sub, int G, XL xload) {
    double acc = 0.0;
    for (int64_t k = s + sub; k < e; k += (int64_t)kSpmvUnroll * G) {
        double vv[kSpmvUnroll], xv[kSpmvUnroll];
#pragma unroll
        for (int u = 0; u < kSpmvUnroll; ++u) {
            const int64_t kk = k + (int64_t)u * G;
            if (kk < e) {
                vv[u] = (double)__ldg(v + kk);
                xv[u] = xload(__ldg(ci + kk));
            } else {
                vv[u] = 0.0;
                xv[u] = 0.0;
            }
        }
#pragma unroll
        for (int u = 0; u < kSpmvUnroll; ++u) acc = fma(vv[u], xv[u], acc);
    }
    return acc;
}

// Rows of at most kSegNnz entries through the length bins: warp item i of
// bin b covers 32 / G rows (G = 2 << b lanes each).  FIN(r, sum) is called
// once per row by the row's first lane.
template <typename VT, typename XL, typename FIN>
__device__ __forceinline__ void spmv_binned(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                            const VT* __restrict__ v, const SpmvBins& bins, int64_t warp0,
                                            int64_t nwarps, XL xload, FIN fin) {
    const int lane = threadIdx.x & 31;
    const int64_t total = bins.items[kSpmvBins];
    for (int64_t it = warp0; it < total; it += nwarps) {
        int b = 0;
        while (b + 1 < kSpmvBins && it >= bins.items[b + 1]) ++b;
        const int G = 2 << b;
        const int sub = lane & (G - 1);
        const int64_t p = bins.off[b] + (it - bins.items[b]) * (32 / G) + lane / G;
        const bool valid = p < bins.off[b + 1];
        double acc = 0.0;
        int64_t r = 0;
        if (valid) {
            r = __ldg(bins.rows + p);
            acc = row_dot(ci, v, __ldg(rp + r), __ldg(rp + r + 1), sub, G, xload);
        }
        for (int o = G >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (valid && sub == 0) fin(r, acc);
    }
}

// ------------------------------------------------- column-sliced SpMV ----
// Shared by the standalone kernel (spmv_sliced.cu) and the cooperative
// Lanczos block.  A CTA takes row ranges rg = blockIdx.x, += gridDim.x; for
// each, every slice of x (scaled by rinv when SCALE) is copied into shared
// memory and the range's entries of that slice are summed into FP64
// accumulators in shared memory; FIN(r, sum) is then called once per row (by
// some thread of the CTA).  In a slice a row's piece is short (tens of
// entries), so each thread takes whole rows and keeps four loads in flight;
// pieces longer than kSlLong entries are listed in shared memory (room for
// every row of the range, so the choice never depends on timing) and taken by
// whole warps afterwards.  Which path a piece takes depends only on its
// length, and every accumulator gets one sum per slice in slice order, so the
// product is deterministic.  `dyn` holds kSlSmem bytes.
constexpr int kSlW = 18432;        // columns per slice: 144 KB of FP64 x
constexpr int kSlRowCap = 8192;    // rows per CTA range: 64 KB of FP64 accumulators
constexpr int kSlLong = 128;       // a longer piece of a row is summed by a warp
constexpr int kSlUnroll = 4;
constexpr int kSlSmem = (kSlW + kSlRowCap) * 8 + kSlRowCap * 2 + 16;  // + the long-piece list

struct SlicedOp {
    int64_t nmajor, nminor;
    int32_t nslices, nranges;
    const int64_t* sbase;   // nslices + 1
    const int32_t* sptr;    // nslices x (nmajor + 1), relative to sbase[s]
    const uint16_t* sidx;   // column - s * kSlW
    const int64_t* rstart;  // nranges + 1
};

// sum of val[k] * xs[idx[k]] over k = k0, k0 + step, ... < e, four chains
template <typename VT>
__device__ __forceinline__ double sliced_piece(const VT* __restrict__ val, const uint16_t* __restrict__ idx,
                                               const double* xs, int64_t k0, int64_t e, int step) {
    double acc = 0.0;
    for (int64_t k = k0; k < e; k += (int64_t)step * kSlUnroll) {
        double vv[kSlUnroll], xv[kSlUnroll];
#pragma unroll
        for (int u = 0; u < kSlUnroll; ++u) {
            const int64_t kk = k + (int64_t)u * step;
            if (kk < e) {
                vv[u] = (double)__ldg(val + kk);
                xv[u] = xs[__ldg(idx + kk)];
            } else {
                vv[u] = 0.0;
                xv[u] = 0.0;
            }
        }
#pragma unroll
        for (int u = 0; u < kSlUnroll; ++u) acc = fma(vv[u], xv[u], acc);
    }
    return acc;
}

template <typename VT, bool SCALE, typename FIN>
__device__ __forceinline__ void sliced_rows(const SlicedOp& a, const VT* __restrict__ val, const double* x,
                                            double rinv, double* dyn, FIN fin) {
    double* xs = dyn;
    double* yacc = dyn + kSlW;
    uint16_t* longs = reinterpret_cast<uint16_t*>(dyn + kSlW + kSlRowCap);  // rows of the range, < kSlRowCap
    int* nlong = reinterpret_cast<int*>(longs + kSlRowCap);
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarp = nthr >> 5;
    for (int64_t rg = blockIdx.x; rg < a.nranges; rg += gridDim.x) {
        const int64_t r0 = a.rstart[rg], r1 = a.rstart[rg + 1];
        const int nr = (int)(r1 - r0);
        for (int i = tid; i < nr; i += nthr) yacc[i] = 0.0;
        for (int s = 0; s < a.nslices; ++s) {
            const int64_t c0 = (int64_t)s * kSlW;
            const int cw = (int)(a.nminor - c0 < kSlW ? a.nminor - c0 : kSlW);
            __syncthreads();  // every thread is done with the previous slice
            if (tid == 0) *nlong = 0;
            for (int i = tid; i < cw; i += nthr) xs[i] = SCALE ? mul_rn(x[c0 + i], rinv) : x[c0 + i];
            __syncthreads();
            const int32_t* pp = a.sptr + (int64_t)s * (a.nmajor + 1);
            const int64_t base = __ldg(a.sbase + s);
            for (int64_t r = r0 + tid; r < r1; r += nthr) {
                const int64_t b = base + __ldg(pp + r), e = base + __ldg(pp + r + 1);
                if (e - b > kSlLong) longs[atomicAdd(nlong, 1)] = (uint16_t)(r - r0);
                else yacc[r - r0] += sliced_piece(val, a.sidx, xs, b, e, 1);
            }
            __syncthreads();
            const int nl = *nlong;
            for (int li = warp; li < nl; li += nwarp) {  // uniform over the warp
                const int64_t r = r0 + longs[li];
                const int64_t b = base + __ldg(pp + r), e = base + __ldg(pp + r + 1);
                double acc = sliced_piece(val, a.sidx, xs, b + lane, e, 32);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                if (lane == 0) yacc[r - r0] += acc;
            }
        }
        __syncthreads();
        for (int i = tid; i < nr; i += nthr) fin(r0 + i, yacc[i]);
        __syncthreads();
    }
}

}  // namespace svdb
