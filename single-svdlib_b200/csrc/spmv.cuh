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
// memory and the range's entries of that slice are summed by 8-lane groups
// into FP64 accumulators in shared memory; FIN(r, sum) is then called once
// per row (by some thread of the CTA).  `dyn` holds kSlW + kSlRowCap doubles.
constexpr int kSlW = 20480;       // columns per slice: 160 KB of FP64 x
constexpr int kSlRowCap = 8192;   // rows per CTA range: 64 KB of FP64 accumulators
constexpr int kSlG = 8;           // lanes per row
constexpr int kSlUnroll = 4;
constexpr int kSlSmem = (kSlW + kSlRowCap) * 8;

struct SlicedOp {
    int64_t nmajor, nminor;
    int32_t nslices, nranges;
    const int64_t* sbase;   // nslices + 1
    const int32_t* sptr;    // nslices x (nmajor + 1), relative to sbase[s]
    const uint16_t* sidx;   // column - s * kSlW
    const int64_t* rstart;  // nranges + 1
};

template <typename VT, bool SCALE, typename FIN>
__device__ __forceinline__ void sliced_rows(const SlicedOp& a, const VT* __restrict__ val, const double* x,
                                            double rinv, double* dyn, FIN fin) {
    double* xs = dyn;
    double* yacc = dyn + kSlW;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int warp = tid >> 5, sub = tid % kSlG;
    const int wrow = (tid & 31) / kSlG;  // the warp's rows: 32 / kSlG at a time
    constexpr int kRowsPerWarp = 32 / kSlG;
    const int nwarp = nthr >> 5;
    for (int64_t rg = blockIdx.x; rg < a.nranges; rg += gridDim.x) {
        const int64_t r0 = a.rstart[rg], r1 = a.rstart[rg + 1];
        const int nr = (int)(r1 - r0);
        for (int i = tid; i < nr; i += nthr) yacc[i] = 0.0;
        for (int s = 0; s < a.nslices; ++s) {
            const int64_t c0 = (int64_t)s * kSlW;
            const int cw = (int)(a.nminor - c0 < kSlW ? a.nminor - c0 : kSlW);
            __syncthreads();  // every group is done with the previous slice
            for (int i = tid; i < cw; i += nthr) xs[i] = SCALE ? mul_rn(x[c0 + i], rinv) : x[c0 + i];
            __syncthreads();
            const int32_t* pp = a.sptr + (int64_t)s * (a.nmajor + 1);
            const int64_t base = __ldg(a.sbase + s);
            // the loop is uniform over the warp (every lane takes every trip), so
            // the full-mask shuffles below always see all 32 lanes
            for (int64_t rb = r0 + (int64_t)warp * kRowsPerWarp; rb < r1; rb += (int64_t)nwarp * kRowsPerWarp) {
                const int64_t r = rb + wrow;
                const bool valid = r < r1;
                const int64_t b = valid ? base + __ldg(pp + r) : 0, e = valid ? base + __ldg(pp + r + 1) : 0;
                double acc = 0.0;
                for (int64_t k = b + sub; k < e; k += (int64_t)kSlG * kSlUnroll) {
                    double vv[kSlUnroll], xv[kSlUnroll];
#pragma unroll
                    for (int u = 0; u < kSlUnroll; ++u) {
                        const int64_t kk = k + (int64_t)u * kSlG;
                        if (kk < e) {
                            vv[u] = (double)__ldg(val + kk);
                            xv[u] = xs[__ldg(a.sidx + kk)];
                        } else {
                            vv[u] = 0.0;
                            xv[u] = 0.0;
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kSlUnroll; ++u) acc = fma(vv[u], xv[u], acc);
                }
#pragma unroll
                for (int o = kSlG / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                if (valid && sub == 0) yacc[r - r0] += acc;
            }
        }
        __syncthreads();
        for (int i = tid; i < nr; i += nthr) fin(r0 + i, yacc[i]);
        __syncthreads();
    }
}

}  // namespace svdb
