// Batches of masked column subsets: randomized_svd (src/randomized/mod.rs:
// 24-199) on many MaskedCSRMatrix::with_columns views (src/lanczos/masked.rs:
// 48-55) of one matrix, solved together.
//
// Nothing is compacted per subset.  The products read A's CSR and CSC and
// remap columns through per-subset maps (o2m: original -> masked column or
// -1, m2o: masked -> original, ascending as the crate numbers them):
//   Y_b = A_b X_b  rows of A; entry (c, v) counts for b when o2m_b[c] >= 0.
//                  A group of subsets shares one read of each row of A.
//   Z_b = A_b^T Y  column m2o_b[j] of A (a row of the CSC) for masked j.
// Every kernel below covers all subsets in one launch (blockIdx.y or a
// subset-major item space), and the whole solve -- Omega, the power
// iterations with their CholeskyQR2 passes, B^T = A^T Q, the small SVDs and
// U, V^T -- is captured once into a CUDA graph that svdb_batch_run replays.
// The group size of the row products (subsets per read of a row) is picked
// by timing the candidates on the first batch of a shape class.
//
// Arithmetic follows the single-matrix path (randomized.cu): the same Omega
// stream per subset (its seed, indexed like a single call), CholeskyQR2 with
// the shifted retry and conditional third pass, one-sided Jacobi on R of B^T.
// SVDB_MIXED keeps the dense operands in FP32 (products summed in FP32 over
// 32-entry chunks, FP64 across chunks); Gram matrices, Cholesky, R^-1, the
// final QR of B^T and the Jacobi SVD are FP64.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <tuple>
#include <type_traits>
#include <vector>

#include "dense_small.cuh"
#include "device_common.cuh"
#include "ops.cuh"
#include "svdb_internal.h"

namespace svdb {

constexpr int kBatchMaxL = 64;      // sample columns per subset
constexpr int kGramChunks = 16;     // Gram partials per subset
constexpr int kBTileRows = 32;

// Per-subset dense matrices.  ROWS_M: subset b at p + b * m * cols, m rows;
// otherwise at p + coff[b] * cols with coff[b+1] - coff[b] rows.
struct SubLayout {
    int by_coff;
    int64_t m;
};
__device__ __forceinline__ int64_t sub_rows(const SubLayout& L, const int64_t* coff, int64_t b) {
    return L.by_coff ? coff[b + 1] - coff[b] : L.m;
}
__device__ __forceinline__ int64_t sub_row0(const SubLayout& L, const int64_t* coff, int64_t b) {
    return L.by_coff ? coff[b] : b * L.m;
}

// ------------------------------------------------------------ the maps ----
__global__ void k_b_o2m(const int32_t* __restrict__ m2o, const int64_t* __restrict__ coff, int64_t n,
                        int32_t* __restrict__ o2m) {
    const int64_t b = blockIdx.y;
    const int64_t c0 = coff[b], nb = coff[b + 1] - c0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nb; j += (int64_t)gridDim.x * blockDim.x)
        o2m[b * n + m2o[c0 + j]] = (int32_t)j;
}

// Omega_b (nb x l): entries 0 .. nb*l of the seed's stream, as a single call draws it
template <typename T>
__global__ void k_b_omega(uint64_t seed, const int64_t* __restrict__ coff, int l, T* __restrict__ Om) {
    const int64_t b = blockIdx.y;
    const int64_t base = coff[b] * l, tot = (coff[b + 1] - coff[b]) * l;
    const uint64_t key = omega_key(seed);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x)
        Om[base + i] = (T)omega_value(key, i);
}

// ------------------------------------------------------------ products ----
template <typename XT>
struct ChunkType {
    using type = typename std::conditional<sizeof(XT) == 4, float, double>::type;
};

// Y_b = A_b X_b for the subsets b = g*GS + t (t < GS) of group g; item
// (g, r), group-major, one warp each.  X_b: nb x l at X + coff[b]*l; Y_b:
// m x l at Y + b*m*l.  Lane owns dense columns lane*CPL .. +CPL.
template <typename VT, typename XT, int GS, int CPL>
__global__ void __launch_bounds__(256) k_b_spmm_rows(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                     const VT* __restrict__ val, int64_t m,
                                                     const int32_t* __restrict__ o2m, int64_t n,
                                                     const int64_t* __restrict__ coff, int64_t count, int l,
                                                     const XT* __restrict__ X, XT* __restrict__ Y) {
    using CT = typename ChunkType<XT>::type;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t ngroups = (count + GS - 1) / GS;
    const int64_t items = ngroups * m;
    const int c0 = lane * CPL;
    for (int64_t it = warp0; it < items; it += nw) {
        const int64_t g = it / m, r = it - g * m;
        const XT* xb[GS];
        int64_t bb[GS];
#pragma unroll
        for (int t = 0; t < GS; ++t) {
            bb[t] = g * GS + t;
            xb[t] = bb[t] < count ? X + coff[bb[t]] * l : X;
        }
        double acc[GS][CPL];
#pragma unroll
        for (int t = 0; t < GS; ++t)
#pragma unroll
            for (int u = 0; u < CPL; ++u) acc[t][u] = 0.0;
        const int64_t s = rp[r], e = rp[r + 1];
        for (int64_t k0 = s; k0 < e; k0 += 32) {
            const int cnt = (int)min((int64_t)32, e - k0);
            int32_t cm = 0;
            CT vm = CT(0);
            if (lane < cnt) {
                cm = __ldg(ci + k0 + lane);
                vm = (CT)__ldg(val + k0 + lane);
            }
            int32_t jm[GS];
#pragma unroll
            for (int t = 0; t < GS; ++t) jm[t] = (lane < cnt && bb[t] < count) ? __ldg(o2m + bb[t] * n + cm) : -1;
            CT ch[GS][CPL];
#pragma unroll
            for (int t = 0; t < GS; ++t)
#pragma unroll
                for (int u = 0; u < CPL; ++u) ch[t][u] = CT(0);
            for (int q = 0; q < cnt; ++q) {
                const CT vq = __shfl_sync(full, vm, q);
#pragma unroll
                for (int t = 0; t < GS; ++t) {
                    const int32_t jq = __shfl_sync(full, jm[t], q);
                    if (jq >= 0) {
                        const XT* xr = xb[t] + (int64_t)jq * l + c0;
#pragma unroll
                        for (int u = 0; u < CPL; ++u)
                            if (c0 + u < l) ch[t][u] = fma(vq, (CT)__ldg(xr + u), ch[t][u]);
                    }
                }
            }
#pragma unroll
            for (int t = 0; t < GS; ++t)
#pragma unroll
                for (int u = 0; u < CPL; ++u) acc[t][u] += (double)ch[t][u];
        }
#pragma unroll
        for (int t = 0; t < GS; ++t) {
            if (bb[t] >= count) continue;
            XT* yr = Y + (bb[t] * m + r) * l + c0;
#pragma unroll
            for (int u = 0; u < CPL; ++u)
                if (c0 + u < l) yr[u] = (XT)acc[t][u];
        }
    }
}

// Z_b[j] = sum over the entries (r, v) of column m2o_b[j] of A of v * Y_b[r];
// item j of the concatenated masked columns (subset-major), one warp each.
template <typename VT, typename XT, typename OT, int CPL>
__global__ void __launch_bounds__(256) k_b_spmm_cols(const int64_t* __restrict__ cp, const int32_t* __restrict__ ri,
                                                     const VT* __restrict__ cv, int64_t m,
                                                     const int32_t* __restrict__ m2o, const int64_t* __restrict__ coff,
                                                     int64_t count, int l, const XT* __restrict__ Y,
                                                     OT* __restrict__ Z) {
    using CT = typename ChunkType<XT>::type;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t total = coff[count];
    const int c0 = lane * CPL;
    int64_t b = 0;
    for (int64_t it = warp0; it < total; it += nw) {
        while (coff[b + 1] <= it) ++b;  // items rise, so b only moves forward
        const XT* yb = Y + b * m * l;
        const int32_t c = m2o[it];
        const int64_t s = cp[c], e = cp[c + 1];
        double acc[CPL];
#pragma unroll
        for (int u = 0; u < CPL; ++u) acc[u] = 0.0;
        for (int64_t k0 = s; k0 < e; k0 += 32) {
            const int cnt = (int)min((int64_t)32, e - k0);
            int32_t rm = 0;
            CT vm = CT(0);
            if (lane < cnt) {
                rm = __ldg(ri + k0 + lane);
                vm = (CT)__ldg(cv + k0 + lane);
            }
            CT ch[CPL];
#pragma unroll
            for (int u = 0; u < CPL; ++u) ch[u] = CT(0);
#pragma unroll 4
            for (int q = 0; q < cnt; ++q) {
                const CT vq = __shfl_sync(full, vm, q);
                const int32_t rq = __shfl_sync(full, rm, q);
                const XT* yr = yb + (int64_t)rq * l + c0;
#pragma unroll
                for (int u = 0; u < CPL; ++u)
                    if (c0 + u < l) ch[u] = fma(vq, (CT)__ldg(yr + u), ch[u]);
            }
#pragma unroll
            for (int u = 0; u < CPL; ++u) acc[u] += (double)ch[u];
        }
        OT* zr = Z + it * l + c0;
#pragma unroll
        for (int u = 0; u < CPL; ++u)
            if (c0 + u < l) zr[u] = (OT)acc[u];
    }
}

// ------------------------------------------------- lean batch products ----
// The products of an SVDB_MIXED batch (FP32 values and dense operands, l a
// multiple of 4 up to 64) with the instruction stream of k_spmm_f32: a
// chunk's 32 entries are loaded by the warp one chunk ahead, the entries
// that count are staged once in a per-warp shared buffer as (row offset,
// value) and read back by broadcast, lane groups of 32 / H lanes take every
// H-th staged entry with one 16-byte gather of four columns each (FP32 sums
// per chunk, FP64 across chunks, groups combined in a fixed xor tree).  The
// kernels above spend a warp instruction per entry and subset (a shuffle, a
// membership test and scalar gathers per entry).
constexpr int kBLeanWarps = 8;
constexpr int kBLeanU = 8;  // gathers in flight per lane

// sum over staged entries q = g, g + H, ... < cnt of v_q X[off_q + c0 ..
// c0 + 3]: batches of kBLeanU gathers issued before their FMAs; a full chunk
// (cnt == 32) needs no bounds tests.  X is the same for the whole warp and
// the offsets are 32-bit (no 64-bit per-lane address arithmetic).
template <int H>
__device__ __forceinline__ void lean_chunk(const int2* __restrict__ E, int cnt, int g, bool active,
                                           const float* __restrict__ X, uint32_t c0, float (&c4)[4]) {
    constexpr int PER = 32 / H;
    if (cnt == 32) {
#pragma unroll 1
        for (int qb = 0; qb < PER; qb += kBLeanU) {
            float4 xv[kBLeanU];
            float vv[kBLeanU];
#pragma unroll
            for (int u = 0; u < kBLeanU; ++u) {
                const int2 en = E[(qb + u) * H + g];
                vv[u] = __int_as_float(en.y);
                xv[u] = active ? *reinterpret_cast<const float4*>(X + ((uint32_t)en.x + c0))
                               : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < kBLeanU; ++u) {
                c4[0] = fmaf(vv[u], xv[u].x, c4[0]);
                c4[1] = fmaf(vv[u], xv[u].y, c4[1]);
                c4[2] = fmaf(vv[u], xv[u].z, c4[2]);
                c4[3] = fmaf(vv[u], xv[u].w, c4[3]);
            }
        }
    } else {
#pragma unroll 1
        for (int qb = g; qb < cnt; qb += H * kBLeanU) {
            float4 xv[kBLeanU];
            float vv[kBLeanU];
#pragma unroll
            for (int u = 0; u < kBLeanU; ++u) {
                const int q = qb + u * H;
                const bool ok = q < cnt && active;
                const int2 en = E[q < cnt ? q : 0];
                vv[u] = ok ? __int_as_float(en.y) : 0.f;
                xv[u] = ok ? *reinterpret_cast<const float4*>(X + ((uint32_t)en.x + c0)) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < kBLeanU; ++u) {
                c4[0] = fmaf(vv[u], xv[u].x, c4[0]);
                c4[1] = fmaf(vv[u], xv[u].y, c4[1]);
                c4[2] = fmaf(vv[u], xv[u].z, c4[2]);
                c4[3] = fmaf(vv[u], xv[u].w, c4[3]);
            }
        }
    }
}

// Items are taken in order from a counter (*next, zero at launch), one per
// warp at a time: the items in flight stay one contiguous window of the
// subset-major order, so only a few subsets' dense operands are in use at
// once (with a static grid stride, warps held by long columns fall behind
// and the window spreads over many subsets, whose operands then compete for
// L2).  An item's sums do not depend on which warp takes it.
__device__ __forceinline__ int64_t lean_next(unsigned long long* next, int lane) {
    unsigned long long it = 0;
    if (lane == 0) it = atomicAdd(next, 1ull);
    return (int64_t)__shfl_sync(0xffffffffu, it, 0);
}

// Y_b = A_b X_b, one warp per (subset, row) item, subset-major; an entry
// (c, v) of row r counts for subset b when o2m_b[c] >= 0.  The members of
// each scanned chunk are appended (ballot compaction, in entry order) to a
// 64-entry per-warp buffer, and the gathers run 32 members at a time without
// bounds tests; the last members of the row go through the guarded path.
// (Gathering each chunk's members as they came, about a third of a chunk on
// this workload, spent most gather slots on padding and ran issue-bound at
// about 10 warp instructions per scanned entry.)
template <int H>
__global__ void __launch_bounds__(kBLeanWarps * 32, 4)
    k_b_rows_lean(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci, const float* __restrict__ val,
                  int64_t m, const int32_t* __restrict__ o2m, int64_t n, const int64_t* __restrict__ coff,
                  int64_t count, int l, const float* __restrict__ X, float* __restrict__ Y,
                  unsigned long long* __restrict__ next) {
    constexpr int GL = 32 / H;
    __shared__ int2 s_ent[kBLeanWarps][64];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane / GL, gl = lane % GL;
    const int col0 = gl * 4;
    const int ncols_here = (l - col0) < 4 ? (l - col0) : 4;
    const bool active = ncols_here > 0;
    int2* E = s_ent[w];
    const int64_t items = count * m;
    for (int64_t it = lean_next(next, lane); it < items; it = lean_next(next, lane)) {
        const int64_t b = it / m, r = it - b * m;
        const float* Xb = X + coff[b] * l;
        const uint32_t c0a = active ? (uint32_t)col0 : 0u;
        const int32_t* om = o2m + b * n;
        const int64_t s = __ldg(rp + r), e = __ldg(rp + r + 1);
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        // chunk k's membership (jm) and value, and chunk k + 1's column, are
        // loaded before chunk k is used, so a lookup overlaps a chunk's gathers
        int32_t jm = -1, nxc = 0;
        float myv = 0.f, nxv = 0.f;
        if (s + lane < e) { myv = __ldg(val + s + lane); jm = __ldg(om + __ldg(ci + s + lane)); }
        if (s + 32 + lane < e) { nxc = __ldg(ci + s + 32 + lane); nxv = __ldg(val + s + 32 + lane); }
        int fill = 0;  // members waiting in E[0 .. fill)
        for (int64_t k0 = s; k0 < e; k0 += 32) {
            const unsigned mask = __ballot_sync(full, jm >= 0);
            if (jm >= 0) E[fill + __popc(mask & ((1u << lane) - 1u))] = make_int2(jm * l, __float_as_int(myv));
            fill += __popc(mask);
            jm = (k0 + 32 + lane < e) ? __ldg(om + nxc) : -1;
            myv = nxv;
            if (k0 + 64 + lane < e) {
                nxc = __ldg(ci + k0 + 64 + lane);
                nxv = __ldg(val + k0 + 64 + lane);
            }
            if (fill >= 32) {
                __syncwarp();
                float c4[4] = {0.f, 0.f, 0.f, 0.f};
                lean_chunk<H>(E, 32, g, active, Xb, c0a, c4);
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[j] += (double)c4[j];
                __syncwarp();  // every lane has read E[0 .. 32)
                const int2 keep = E[32 + lane];
                __syncwarp();
                if (lane < fill - 32) E[lane] = keep;
                fill -= 32;
                __syncwarp();
            }
        }
        if (fill > 0) {
            __syncwarp();
            float c4[4] = {0.f, 0.f, 0.f, 0.f};
            lean_chunk<H>(E, fill, g, active, Xb, c0a, c4);
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[j] += (double)c4[j];
        }
        __syncwarp();  // E is free for the next item
#pragma unroll
        for (int o = GL; o < 32; o <<= 1)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[j] += __shfl_xor_sync(full, acc[j], o);
        if (g == 0 && active) {
            float* yr = Y + (b * m + r) * l + col0;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (j < ncols_here) yr[j] = (float)acc[j];
        }
    }
}

// Z_b[j] = sum over the entries (r, v) of column m2o_b[j] of A of v Y_b[r],
// one warp per (subset, masked column) item, subset-major.
template <typename OT, int H>
__global__ void __launch_bounds__(kBLeanWarps * 32, 4)
    k_b_cols_lean(const int64_t* __restrict__ cp, const int32_t* __restrict__ ri, const float* __restrict__ cv,
                  int64_t m, const int32_t* __restrict__ m2o, const int64_t* __restrict__ coff, int64_t count, int l,
                  const float* __restrict__ Y, OT* __restrict__ Z, unsigned long long* __restrict__ next) {
    constexpr int GL = 32 / H;
    __shared__ int2 s_ent[kBLeanWarps][32];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane / GL, gl = lane % GL;
    const int col0 = gl * 4;
    const int ncols_here = (l - col0) < 4 ? (l - col0) : 4;
    const bool active = ncols_here > 0;
    int2* E = s_ent[w];
    const int64_t total = coff[count];
    int64_t b = 0;
    for (int64_t it = lean_next(next, lane); it < total; it = lean_next(next, lane)) {
        while (coff[b + 1] <= it) ++b;  // a warp's items rise, so b only moves forward
        const float* Yb = Y + b * m * l;
        const uint32_t c0a = active ? (uint32_t)col0 : 0u;
        const int32_t c = m2o[it];
        const int64_t s = __ldg(cp + c), e = __ldg(cp + c + 1);
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        int32_t myr = 0;
        float myv = 0.f;
        if (s + lane < e) { myr = __ldg(ri + s + lane); myv = __ldg(cv + s + lane); }
        for (int64_t k0 = s; k0 < e; k0 += 32) {
            const int cnt = (e - k0) < 32 ? (int)(e - k0) : 32;
            __syncwarp();
            E[lane] = make_int2(myr * l, __float_as_int(myv));
            __syncwarp();
            if (k0 + 32 + lane < e) {
                myr = __ldg(ri + k0 + 32 + lane);
                myv = __ldg(cv + k0 + 32 + lane);
            }
            float c4[4] = {0.f, 0.f, 0.f, 0.f};
            lean_chunk<H>(E, cnt, g, active, Yb, c0a, c4);
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[j] += (double)c4[j];
        }
#pragma unroll
        for (int o = GL; o < 32; o <<= 1)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[j] += __shfl_xor_sync(full, acc[j], o);
        if (g == 0 && active) {
            OT* zr = Z + it * l + col0;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (j < ncols_here) zr[j] = (OT)acc[j];
        }
    }
}


// --------------------------------------------------------- CholeskyQR2 ----
// Gram partials: block (chunk, b) sums X_b^T X_b over its rows (32-row tiles
// staged in shared memory; a 16 x 16 thread grid holds an NC x NC tile).
template <typename T, int NC>
__global__ void __launch_bounds__(256) k_b_gram_part(const T* __restrict__ X, SubLayout L,
                                                     const int64_t* __restrict__ coff, int c,
                                                     double* __restrict__ part, const int* __restrict__ cond) {
    const int64_t b = blockIdx.y;
    if (cond && cond[b] == 0) return;
    extern __shared__ double xs[];  // kBTileRows x c
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int64_t rows = sub_rows(L, coff, b);
    const T* xb = X + sub_row0(L, coff, b) * c;
    const int64_t chunk = (rows + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = blockIdx.x * chunk, r1 = min(rows, r0 + chunk);
    double acc[NC][NC];
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int j = 0; j < NC; ++j) acc[i][j] = 0.0;
    for (int64_t rb = r0; rb < r1; rb += kBTileRows) {
        const int nr = (int)min((int64_t)kBTileRows, r1 - rb);
        __syncthreads();
        for (int t = threadIdx.x; t < nr * c; t += blockDim.x) xs[t] = (double)xb[rb * c + t];
        __syncthreads();
        for (int r = 0; r < nr; ++r) {
            double xa[NC], xc[NC];
#pragma unroll
            for (int i = 0; i < NC; ++i) {
                const int a = ty + 16 * i, bq = tx + 16 * i;
                xa[i] = a < c ? xs[r * c + a] : 0.0;
                xc[i] = bq < c ? xs[r * c + bq] : 0.0;
            }
#pragma unroll
            for (int i = 0; i < NC; ++i)
#pragma unroll
                for (int j = 0; j < NC; ++j) acc[i][j] = fma(xa[i], xc[j], acc[i][j]);
        }
    }
    double* out = part + (b * gridDim.x + blockIdx.x) * (int64_t)c * c;
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int j = 0; j < NC; ++j) {
            const int a = ty + 16 * i, bq = tx + 16 * j;
            if (a < c && bq < c) out[a * c + bq] = acc[i][j];
        }
}

// G_b = sum of the subset's partials in chunk order
__global__ void k_b_gram_reduce(const double* __restrict__ part, int nchunk, int c, double* __restrict__ G,
                                const int* __restrict__ cond) {
    const int64_t b = blockIdx.y;
    if (cond && cond[b] == 0) return;
    const int cc = c * c;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < cc; p += gridDim.x * blockDim.x) {
        double s0 = 0.0, s1 = 0.0;
        int k = 0;
        for (; k + 2 <= nchunk; k += 2) {
            s0 += part[(b * nchunk + k) * cc + p];
            s1 += part[(b * nchunk + k + 1) * cc + p];
        }
        if (k < nchunk) s0 += part[(b * nchunk + k) * cc + p];
        G[b * cc + p] = s0 + s1;
    }
}

__global__ void k_b_chol_inv(const double* __restrict__ G, int c, SubLayout L, const int64_t* __restrict__ coff,
                             double* __restrict__ R, double* __restrict__ Ri, int* __restrict__ flags,
                             int* __restrict__ shifted, const int* __restrict__ cond) {
    const int64_t b = blockIdx.x;
    if (cond && cond[b] == 0) return;
    extern __shared__ double sm[];
    const int64_t rows = sub_rows(L, coff, b);
    const double shift_scale = 11.0 * ((double)rows * c + (double)c * (c + 1)) * 1.1102230246251565e-16;
    const int64_t cc = (int64_t)c * c;
    chol_inv_body(G + b * cc, c, shift_scale, R + b * cc, Ri + b * cc, flags + b, shifted + b, 1, sm);
}

// Out_b (rows x cout) = X_b (rows x c) S_b (c x lds, first cout columns),
// S_b = S + b*c*lds.  X and Out may be the same array (each tile is staged
// before it is written).  TRANS: Out_b is stored cout x rows.
template <typename TI, typename TO, bool TRANS>
__global__ void __launch_bounds__(256) k_b_right_mul(const TI* X, SubLayout LX, const int64_t* __restrict__ coff,
                                                     int c, const double* __restrict__ S, int lds, int cout, TO* Out,
                                                     const int* __restrict__ cond) {
    const int64_t b = blockIdx.y;
    if (cond && cond[b] == 0) return;
    extern __shared__ double sm[];
    double* ss = sm;                // c x cout
    double* xs = sm + c * cout;     // kBTileRows x c
    const double* sb = S + b * (int64_t)c * lds;
    for (int t = threadIdx.x; t < c * cout; t += blockDim.x) ss[t] = sb[(t / cout) * lds + t % cout];
    const int64_t rows = sub_rows(LX, coff, b), row0 = sub_row0(LX, coff, b);
    const TI* xb = X + row0 * c;
    TO* ob = Out + row0 * cout;
    for (int64_t r0 = (int64_t)blockIdx.x * kBTileRows; r0 < rows; r0 += (int64_t)gridDim.x * kBTileRows) {
        const int nr = (int)min((int64_t)kBTileRows, rows - r0);
        __syncthreads();
        for (int t = threadIdx.x; t < nr * c; t += blockDim.x) xs[t] = (double)xb[r0 * c + t];
        __syncthreads();
        for (int t = threadIdx.x; t < nr * cout; t += blockDim.x) {
            const int rr = TRANS ? t % nr : t / cout, j = TRANS ? t / nr : t % cout;
            const double* xr = xs + rr * c;
            double s = 0.0;
            for (int k = 0; k < c; ++k) s = fma(xr[k], ss[k * cout + j], s);
            if (TRANS) ob[(int64_t)j * rows + r0 + rr] = (TO)s;
            else ob[(r0 + rr) * cout + j] = (TO)s;
        }
    }
}

// C_b = A_b B_b (c x c), one block per subset
__global__ void k_b_small_gemm(const double* __restrict__ A, const double* __restrict__ B, int c,
                               double* __restrict__ C, const int* __restrict__ cond) {
    const int64_t b = blockIdx.x;
    if (cond && cond[b] == 0) return;
    const int64_t cc = (int64_t)c * c;
    for (int t = threadIdx.x; t < c * c; t += blockDim.x) {
        const int i = t / c, j = t % c;
        double s = 0.0;
        for (int k = 0; k < c; ++k) s = fma(A[b * cc + i * c + k], B[b * cc + k * c + j], s);
        C[b * cc + t] = s;
    }
}
__global__ void k_b_copy_cond(const double* __restrict__ src, double* __restrict__ dst, int64_t per,
                              const int* __restrict__ cond) {
    const int64_t b = blockIdx.y;
    if (cond && cond[b] == 0) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < per; i += (int64_t)gridDim.x * blockDim.x)
        dst[b * per + i] = src[b * per + i];
}

// LU normaliser (mod.rs:239-293): column j of X_b scaled to unit norm unless its norm is <= 1e-10
template <typename T>
__global__ void k_b_colnorm(T* __restrict__ X, SubLayout L, const int64_t* __restrict__ coff, int c) {
    __shared__ double sh[32];
    __shared__ double scale;
    const int j = blockIdx.x;
    const int64_t b = blockIdx.y;
    const int64_t rows = sub_rows(L, coff, b);
    T* xb = X + sub_row0(L, coff, b) * c;
    double acc = 0.0;
    for (int64_t r = threadIdx.x; r < rows; r += blockDim.x) {
        const double v = (double)xb[r * c + j];
        acc = fma(v, v, acc);
    }
    const double nrm = sqrt(block_sum(acc, sh));
    if (threadIdx.x == 0) scale = nrm > 1e-10 ? 1.0 / nrm : 1.0;
    __syncthreads();
    if (nrm > 1e-10)
        for (int64_t r = threadIdx.x; r < rows; r += blockDim.x) xb[r * c + j] = (T)((double)xb[r * c + j] * scale);
}

__global__ void __launch_bounds__(512) k_b_jacobi(const double* __restrict__ R, int c, double* __restrict__ U,
                                                  double* __restrict__ V, double* __restrict__ sig,
                                                  int* __restrict__ status) {
    extern __shared__ double sm[];
    const int64_t b = blockIdx.x;
    const int64_t cc = (int64_t)c * c;
    jacobi_svd_body(R + b * cc, c, U + b * cc, V + b * cc, sig + b * c, status + b, sm);
}

// ------------------------------------------------------------ the batch ----
struct TuneKey {
    int64_t m, n, nnz, count;
    int l, prec;
    bool operator<(const TuneKey& o) const {
        return std::tie(m, n, nnz, count, l, prec) < std::tie(o.m, o.n, o.nnz, o.count, o.l, o.prec);
    }
};
static std::mutex g_tune_mu;
static std::map<TuneKey, int> g_tuned;  // -> subsets per row item

}  // namespace svdb

struct svdb_batch {
    const svdb_matrix* A = nullptr;
    cudaStream_t s = nullptr;
    bool mixed = false, on_device = false, use_graph = true;
    int64_t m = 0, n = 0, count = 0, rank = 0, l = 0, q = 0, total_cols = 0;
    int normalizer = 0;
    uint64_t seed = 0;
    int gs = 4, cpl = 2;
    std::vector<int64_t> coff_h;
    svdb::DevBuf<int64_t> coff;
    svdb::DevBuf<int32_t> m2o, o2m;
    // dense operands: float (mixed) or double, addressed through void*
    svdb::DevBuf<float> Om32, Y32, Z32;
    svdb::DevBuf<double> Om64, Y64, Z64, Bt;
    svdb::DevBuf<double> part, G, R1, R2, R3, Ri, Rout, Rtmp, Ur, Vr, sig, U, Vt;
    svdb::DevBuf<int> flags, shifted, jstat;
    svdb::DevBuf<unsigned long long> next;  // the lean product kernels' item counter
    // SVDB_MIXED with a dense-column split of A: the dense columns' share of
    // every product as one GEMM over all subsets (dense_split.cu); the B
    // operands of the row and column GEMMs and the column GEMM's tiles
    const svdb::DenseSplit* dsplit = nullptr;
    svdb::DevBuf<float> dbh_r, dbl_r, dbh_c, dbl_c;
    svdb::DevBuf<double> dpart;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    size_t graph_nodes = 0;
    uint64_t kernels_per_run = 0;
    double tune_ms = 0.0, last_ms = 0.0;
    uint64_t total_nnz = 0;
    ~svdb_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (s) cudaStreamSynchronize(s);
    }
};

namespace svdb {

static int grid_cap(int per_sm) { return device_props().sms * per_sm; }

template <typename T>
static T* dense_ptr(svdb_batch& B, DevBuf<float>& f, DevBuf<double>& d) {
    if constexpr (std::is_same<T, float>::value) return f.p;
    else return d.p;
}

// the lean kernels apply to SVDB_MIXED batches with l a multiple of 4
// (16-byte rows), 32-bit offsets, and SVDB_BATCH_SPMM=warp not set
static bool lean_batch(const svdb_batch& B, int64_t rows_per_item_operand) {
    const char* e = getenv("SVDB_BATCH_SPMM");
    if (e && std::string(e) == "warp") return false;
    return B.mixed && B.l % 4 == 0 && B.l <= 64 && rows_per_item_operand * B.l < ((int64_t)1 << 31);
}

// Y_b = A_b X_b with `gs` subsets per row item
template <typename T>
static void rows_product(svdb_batch& B, const T* X, T* Y, int gs) {
    // with the split: the rest of A here, the dense columns below
    const DevCompressed& A = B.dsplit ? B.dsplit->rest_csr : csr_of(B.A);
    if constexpr (std::is_same<T, float>::value) {
        if (lean_batch(B, B.n)) {
            const int blocks = grid_cap(4);  // the resident blocks; items come from the counter
            SVDB_CUDA(cudaMemsetAsync(B.next.p, 0, sizeof(unsigned long long), B.s));
            if (B.l <= 32)
                k_b_rows_lean<4><<<blocks, kBLeanWarps * 32, 0, B.s>>>(A.ptr.p, A.idx.p, A.val32.p, B.m, B.o2m.p,
                                                                       B.n, B.coff.p, B.count, (int)B.l, X, Y,
                                                                       B.next.p);
            else
                k_b_rows_lean<2><<<blocks, kBLeanWarps * 32, 0, B.s>>>(A.ptr.p, A.idx.p, A.val32.p, B.m, B.o2m.p,
                                                                       B.n, B.coff.p, B.count, (int)B.l, X, Y,
                                                                       B.next.p);
            SVDB_CHECK_LAUNCH();
            if (B.dsplit)
                dense_batch_rows(B.A, X, B.coff.p, B.o2m.p, B.count, (int)B.l, Y, B.dbh_r.p, B.dbl_r.p, B.s);
            return;
        }
    }
    const int blocks = grid_cap(6);
#define SVDB_ROWS(GS)                                                                                             \
    case GS:                                                                                                      \
        if (B.mixed)                                                                                              \
            k_b_spmm_rows<float, T, GS, 2><<<blocks, 256, 0, B.s>>>(A.ptr.p, A.idx.p, A.val32.p, B.m, B.o2m.p,     \
                                                                    B.n, B.coff.p, B.count, (int)B.l, X, Y);      \
        else                                                                                                      \
            k_b_spmm_rows<double, T, GS, 2><<<blocks, 256, 0, B.s>>>(A.ptr.p, A.idx.p, A.val.p, B.m, B.o2m.p,      \
                                                                     B.n, B.coff.p, B.count, (int)B.l, X, Y);     \
        break;
    switch (gs) {
        SVDB_ROWS(1)
        SVDB_ROWS(2)
        SVDB_ROWS(4)
        SVDB_ROWS(8)
        default: throw Error(SVDB_ERR_ARG, "batch: bad group size");
    }
#undef SVDB_ROWS
    SVDB_CHECK_LAUNCH();
    if constexpr (std::is_same<T, float>::value) {
        if (B.dsplit) dense_batch_rows(B.A, X, B.coff.p, B.o2m.p, B.count, (int)B.l, Y, B.dbh_r.p, B.dbl_r.p, B.s);
    }
}

// Z_b = A_b^T Y_b
template <typename T, typename OT>
static void cols_product(svdb_batch& B, const T* Y, OT* Z) {
    // with the split: the rest of A^T here (rows of the dense columns empty,
    // so their Z rows are written as 0), the dense columns below
    const DevCompressed& At = B.dsplit ? B.dsplit->rest_csc : csc_of(B.A);
    if constexpr (std::is_same<T, float>::value) {
        if (lean_batch(B, B.m)) {
            const int blocks = grid_cap(4);  // the resident blocks; items come from the counter
            SVDB_CUDA(cudaMemsetAsync(B.next.p, 0, sizeof(unsigned long long), B.s));
            if (B.l <= 32)
                k_b_cols_lean<OT, 4><<<blocks, kBLeanWarps * 32, 0, B.s>>>(At.ptr.p, At.idx.p, At.val32.p, B.m,
                                                                           B.m2o.p, B.coff.p, B.count, (int)B.l, Y, Z,
                                                                           B.next.p);
            else
                k_b_cols_lean<OT, 2><<<blocks, kBLeanWarps * 32, 0, B.s>>>(At.ptr.p, At.idx.p, At.val32.p, B.m,
                                                                           B.m2o.p, B.coff.p, B.count, (int)B.l, Y, Z,
                                                                           B.next.p);
            SVDB_CHECK_LAUNCH();
            if (B.dsplit)
                dense_batch_cols<OT>(B.A, Y, B.coff.p, B.o2m.p, B.count, (int)B.l, Z, B.dbh_c.p, B.dbl_c.p,
                                     B.dpart.p, B.s);
            return;
        }
    }
    const int blocks = grid_cap(8);
    if (B.mixed)
        k_b_spmm_cols<float, T, OT, 2><<<blocks, 256, 0, B.s>>>(At.ptr.p, At.idx.p, At.val32.p, B.m, B.m2o.p,
                                                                B.coff.p, B.count, (int)B.l, Y, Z);
    else
        k_b_spmm_cols<double, T, OT, 2><<<blocks, 256, 0, B.s>>>(At.ptr.p, At.idx.p, At.val.p, B.m, B.m2o.p,
                                                                 B.coff.p, B.count, (int)B.l, Y, Z);
    SVDB_CHECK_LAUNCH();
    if constexpr (std::is_same<T, float>::value) {
        if (B.dsplit)
            dense_batch_cols<OT>(B.A, Y, B.coff.p, B.o2m.p, B.count, (int)B.l, Z, B.dbh_c.p, B.dbl_c.p, B.dpart.p,
                                 B.s);
    }
}

template <typename T>
static void gram(svdb_batch& B, const T* X, SubLayout L, const int* cond) {
    const int c = (int)B.l;
    const size_t smem = (size_t)kBTileRows * c * sizeof(double);
    dim3 grid(kGramChunks, (unsigned)B.count);
    const int nc = (c + 15) / 16;
    switch (nc) {
        case 1: k_b_gram_part<T, 1><<<grid, 256, smem, B.s>>>(X, L, B.coff.p, c, B.part.p, cond); break;
        case 2: k_b_gram_part<T, 2><<<grid, 256, smem, B.s>>>(X, L, B.coff.p, c, B.part.p, cond); break;
        case 3: k_b_gram_part<T, 3><<<grid, 256, smem, B.s>>>(X, L, B.coff.p, c, B.part.p, cond); break;
        default: k_b_gram_part<T, 4><<<grid, 256, smem, B.s>>>(X, L, B.coff.p, c, B.part.p, cond); break;
    }
    k_b_gram_reduce<<<dim3((c * c + 127) / 128, (unsigned)B.count), 128, 0, B.s>>>(B.part.p, kGramChunks, c, B.G.p,
                                                                                   cond);
    SVDB_CHECK_LAUNCH_N(2);
}

template <typename TI, typename TO, bool TRANS>
static void right_mul(svdb_batch& B, const TI* X, SubLayout L, const double* S, int lds, int cout, TO* Out,
                      const int* cond) {
    const int c = (int)B.l;
    const size_t smem = ((size_t)c * cout + (size_t)kBTileRows * c) * sizeof(double);
    if (smem > 48 * 1024)
        SVDB_CUDA(cudaFuncSetAttribute(k_b_right_mul<TI, TO, TRANS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    int64_t rows = L.by_coff ? 0 : L.m;
    if (L.by_coff)
        for (int64_t b = 0; b < B.count; ++b) rows = std::max(rows, B.coff_h[b + 1] - B.coff_h[b]);
    // about 8 blocks per SM over all subsets
    const int64_t per_subset = std::max<int64_t>(1, (int64_t)device_props().sms * 8 / B.count);
    const unsigned tiles =
        (unsigned)std::max<int64_t>(1, std::min<int64_t>((rows + kBTileRows - 1) / kBTileRows, per_subset));
    k_b_right_mul<TI, TO, TRANS><<<dim3(tiles, (unsigned)B.count), 256, smem, B.s>>>(X, L, B.coff.p, c, S, lds, cout,
                                                                                     Out, cond);
    SVDB_CHECK_LAUNCH();
}

static void chol(svdb_batch& B, SubLayout L, double* R, const int* cond) {
    const int c = (int)B.l;
    const size_t smem = 2 * (size_t)c * c * sizeof(double);
    // chol_inv_body also holds about 1 KB of static shared memory
    if (smem > 40 * 1024)
        SVDB_CUDA(cudaFuncSetAttribute(k_b_chol_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_b_chol_inv<<<(unsigned)B.count, 256, smem, B.s>>>(B.G.p, c, L, B.coff.p, R, B.Ri.p, B.flags.p, B.shifted.p,
                                                         cond);
    SVDB_CHECK_LAUNCH();
}

// CholeskyQR2 of every X_b in place (shifted retry, conditional third pass);
// Rout_b = R3 R2 R1 when requested
template <typename T>
static void cholesky_qr(svdb_batch& B, T* X, SubLayout L, bool want_r) {
    const int c = (int)B.l;
    SVDB_CUDA(cudaMemsetAsync(B.shifted.p, 0, B.count * sizeof(int), B.s));
    gram<T>(B, X, L, nullptr);
    chol(B, L, B.R1.p, nullptr);
    right_mul<T, T, false>(B, X, L, B.Ri.p, c, c, X, nullptr);
    gram<T>(B, X, L, nullptr);
    chol(B, L, B.R2.p, nullptr);
    right_mul<T, T, false>(B, X, L, B.Ri.p, c, c, X, nullptr);
    const int* cond = B.shifted.p;
    gram<T>(B, X, L, cond);
    chol(B, L, B.R3.p, cond);
    right_mul<T, T, false>(B, X, L, B.Ri.p, c, c, X, cond);
    if (want_r) {
        k_b_small_gemm<<<(unsigned)B.count, 256, 0, B.s>>>(B.R2.p, B.R1.p, c, B.Rout.p, nullptr);
        k_b_small_gemm<<<(unsigned)B.count, 256, 0, B.s>>>(B.R3.p, B.Rout.p, c, B.Rtmp.p, cond);
        k_b_copy_cond<<<dim3(1, (unsigned)B.count), 256, 0, B.s>>>(B.Rtmp.p, B.Rout.p, (int64_t)c * c, cond);
        SVDB_CHECK_LAUNCH_N(3);
    }
}

template <typename T>
static void normalize(svdb_batch& B, T* X, SubLayout L) {
    if (B.normalizer == SVDB_NORM_QR) {
        cholesky_qr<T>(B, X, L, false);
    } else if (B.normalizer == SVDB_NORM_LU) {
        k_b_colnorm<T><<<dim3((unsigned)B.l, (unsigned)B.count), 256, 0, B.s>>>(X, L, B.coff.p, (int)B.l);
        SVDB_CHECK_LAUNCH();
    }
}

// the whole solve, enqueued on B.s (captured into the graph)
template <typename T>
static void enqueue(svdb_batch& B) {
    const SubLayout LY{0, B.m}, LZ{1, 0};
    T* Om = dense_ptr<T>(B, B.Om32, B.Om64);
    T* Y = dense_ptr<T>(B, B.Y32, B.Y64);
    T* Z = dense_ptr<T>(B, B.Z32, B.Z64);
    const int c = (int)B.l;
    SVDB_CUDA(cudaMemsetAsync(B.flags.p, 0, B.count * sizeof(int), B.s));
    SVDB_CUDA(cudaMemsetAsync(B.jstat.p, 0, B.count * sizeof(int), B.s));
    k_b_omega<T><<<dim3(64, (unsigned)B.count), 256, 0, B.s>>>(B.seed, B.coff.p, c, Om);
    SVDB_CHECK_LAUNCH();
    rows_product<T>(B, Om, Y, B.gs);
    for (int64_t it = 0; it < B.q; ++it) {
        cols_product<T, T>(B, Y, Z);
        normalize<T>(B, Z, LZ);
        rows_product<T>(B, Z, Y, B.gs);
        normalize<T>(B, Y, LY);
    }
    cholesky_qr<T>(B, Y, LY, false);   // Q = qr(y).q()
    cols_product<T, double>(B, Y, B.Bt.p);  // B^T = A^T Q (FP64)
    cholesky_qr<double>(B, B.Bt.p, LZ, true);
    const size_t smem = ((size_t)c * (c + 1) + (size_t)(c + 1) * (c + 1) + (c + 1)) * sizeof(double);
    if (smem > 40 * 1024)  // jacobi_svd_body keeps a little static shared memory too
        SVDB_CUDA(cudaFuncSetAttribute(k_b_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_b_jacobi<<<(unsigned)B.count, jacobi_threads(c, 512), smem, B.s>>>(B.Rout.p, c, B.Ur.p, B.Vr.p, B.sig.p, B.jstat.p);
    SVDB_CHECK_LAUNCH();
    // U_b = Q_b V_J[:, :rank] (m x rank);  V_b^T = (Q_Bt U_J[:, :rank])^T (rank x nb)
    right_mul<T, double, false>(B, Y, LY, B.Vr.p, c, (int)B.rank, B.U.p, nullptr);
    right_mul<double, double, true>(B, B.Bt.p, LZ, B.Ur.p, c, (int)B.rank, B.Vt.p, nullptr);
}

static void enqueue_any(svdb_batch& B) {
    if (B.mixed) enqueue<float>(B);
    else enqueue<double>(B);
}

void batch_create(const svdb_matrix* A, const uint64_t* col_off, const uint64_t* cols, uint64_t count,
                  uint64_t target_rank, uint64_t n_over, uint64_t q, int normalizer, int has_seed, uint64_t seed,
                  const svdb_batch_options& o, svdb_batch** out) {
    if (A->kind == KIND_MASKED) throw Error(SVDB_ERR_UNSUPPORTED, "batch: give the parent matrix, not a masked view");
    if (count == 0 || count > 65535) throw Error(SVDB_ERR_UNSUPPORTED, "batch: between 1 and 65535 subsets");
    if (!col_off || !cols) throw Error(SVDB_ERR_ARG, "null argument");
    if (normalizer < 0 || normalizer > 2) throw Error(SVDB_ERR_ARG, "bad normalizer");
    const int64_t m = A->nrows, n = A->ncols;
    const int64_t l = (int64_t)target_rank + (int64_t)n_over;
    if (target_rank == 0 || l > kBatchMaxL)
        throw Error(SVDB_ERR_UNSUPPORTED, "batch: target_rank >= 1 and target_rank + n_oversamples <= 64");
    if (m < l) throw Error(SVDB_ERR_UNSUPPORTED, "batch: fewer rows than sample columns");
    std::unique_ptr<svdb_batch> B(new svdb_batch());
    B->A = A;
    B->s = o.stream ? (cudaStream_t)o.stream : A->stream;
    B->mixed = o.precision == SVDB_MIXED;
    B->on_device = o.result_on_device != 0;
    B->use_graph = o.use_graph != 0;
    B->m = m; B->n = n; B->count = (int64_t)count; B->rank = (int64_t)target_rank; B->l = l; B->q = (int64_t)q;
    B->normalizer = normalizer;
    B->seed = has_seed ? seed : 0;
    // with_columns per subset: ascending, duplicates dropped, bounds checked (masked.rs:48-55)
    std::vector<int32_t> m2o;
    B->coff_h.assign(count + 1, 0);
    std::vector<int64_t> tmp;
    for (uint64_t b = 0; b < count; ++b) {
        if (col_off[b + 1] < col_off[b]) throw Error(SVDB_ERR_ARG, "batch: column offsets not monotone");
        tmp.assign(cols + col_off[b], cols + col_off[b + 1]);
        for (int64_t c : tmp)
            if (c < 0 || c >= n) throw Error(SVDB_ERR_SHAPE, "Column index out of bounds");
        std::sort(tmp.begin(), tmp.end());
        tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
        if ((int64_t)tmp.size() < l)
            throw Error(SVDB_ERR_UNSUPPORTED, "batch: subset " + std::to_string(b) + " keeps " +
                                                  std::to_string(tmp.size()) + " columns, fewer than the " +
                                                  std::to_string(l) + " sample columns");
        for (int64_t c : tmp) m2o.push_back((int32_t)c);
        B->coff_h[b + 1] = B->coff_h[b] + (int64_t)tmp.size();
    }
    B->total_cols = B->coff_h[count];
    cudaStream_t s = B->s;
    B->coff.alloc(count + 1, s);
    B->m2o.alloc(B->total_cols, s);
    B->o2m.alloc(count * n, s);
    SVDB_CUDA(cudaMemcpyAsync(B->coff.p, B->coff_h.data(), (count + 1) * 8, cudaMemcpyHostToDevice, s));
    SVDB_CUDA(cudaMemcpyAsync(B->m2o.p, m2o.data(), m2o.size() * 4, cudaMemcpyHostToDevice, s));
    SVDB_CUDA(cudaMemsetAsync(B->o2m.p, 0xff, count * n * 4, s));
    k_b_o2m<<<dim3(16, (unsigned)count), 256, 0, s>>>(B->m2o.p, B->coff.p, n, B->o2m.p);
    SVDB_CHECK_LAUNCH();
    if (B->mixed) ensure_fp32(A);
    if (B->mixed && dense_split_usable(A, (int)l)) {
        const DenseSplit* ds = dense_split_get(A);
        const size_t ws = dense_batch_workspace(*ds, (int64_t)count, (int)l);
        size_t free_b = 0, total_b = 0;
        SVDB_CUDA(cudaMemGetInfo(&free_b, &total_b));
        if (ws < free_b / 2) {
            const int64_t npad = ((int64_t)count * l + 63) / 64 * 64;
            B->dbh_r.alloc(npad * ds->ndp, s);
            B->dbl_r.alloc(npad * ds->ndp, s);
            B->dbh_c.alloc(npad * ds->mp, s);
            B->dbl_c.alloc(npad * ds->mp, s);
            B->dpart.alloc(npad * ds->ndp, s);
            // the column GEMM's B rows past count * l are never written: zero once
            SVDB_CUDA(cudaMemsetAsync(B->dbh_c.p, 0, (size_t)npad * ds->mp * sizeof(float), s));
            SVDB_CUDA(cudaMemsetAsync(B->dbl_c.p, 0, (size_t)npad * ds->mp * sizeof(float), s));
            B->dsplit = ds;
        }
    }
    const int64_t tc = B->total_cols;
    if (B->mixed) {
        B->Om32.alloc(tc * l, s); B->Y32.alloc(count * m * l, s); B->Z32.alloc(tc * l, s);
    } else {
        B->Om64.alloc(tc * l, s); B->Y64.alloc(count * m * l, s); B->Z64.alloc(tc * l, s);
    }
    B->Bt.alloc(tc * l, s);
    B->part.alloc(count * kGramChunks * l * l, s);
    for (DevBuf<double>* p : {&B->G, &B->R1, &B->R2, &B->R3, &B->Ri, &B->Rout, &B->Rtmp, &B->Ur, &B->Vr})
        p->alloc(count * l * l, s);
    B->sig.alloc(count * l, s);
    B->U.alloc(count * m * (int64_t)target_rank, s);
    B->Vt.alloc(tc * (int64_t)target_rank, s);
    B->flags.alloc(count, s);
    B->next.alloc(1, s);
    B->shifted.alloc(count, s);
    B->jstat.alloc(count, s);
    {
        // nonzeros per subset (reported): host pass over column counts
        std::vector<int64_t> cp(n + 1);
        const DevCompressed& At = csc_of(A);
        SVDB_CUDA(cudaMemcpyAsync(cp.data(), At.ptr.p, (n + 1) * 8, cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
        uint64_t tot = 0;
        for (int32_t c : m2o) tot += (uint64_t)(cp[c + 1] - cp[c]);
        B->total_nnz = tot;
    }

    // autotune the rows product: subsets per row item
    const TuneKey key{m, n, A->nnz, (int64_t)count, (int)l, (int)B->mixed};
    int gs = 4;
    bool cached = false;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) { gs = it->second; cached = true; }
    }
    // the lean row kernel (SVDB_MIXED) takes one subset per item: nothing to tune
    if (!cached && lean_batch(*B, n)) {
        gs = 1;
        cached = true;
    }
    if (!cached && o.autotune) {
        auto t0 = std::chrono::steady_clock::now();
        cudaEvent_t e0, e1;
        SVDB_CUDA(cudaEventCreate(&e0));
        SVDB_CUDA(cudaEventCreate(&e1));
        float best = 1e30f;
        for (int cand : {1, 2, 4, 8}) {
            if (cand > 1 && (int64_t)count < cand) continue;
            float ms = 0.f;
            auto run = [&]() {
                if (B->mixed) {
                    k_b_omega<float><<<dim3(64, (unsigned)count), 256, 0, s>>>(B->seed, B->coff.p, (int)l, B->Om32.p);
                    SVDB_CHECK_LAUNCH();
                    SVDB_CUDA(cudaEventRecord(e0, s));
                    rows_product<float>(*B, B->Om32.p, B->Y32.p, cand);
                } else {
                    k_b_omega<double><<<dim3(64, (unsigned)count), 256, 0, s>>>(B->seed, B->coff.p, (int)l, B->Om64.p);
                    SVDB_CHECK_LAUNCH();
                    SVDB_CUDA(cudaEventRecord(e0, s));
                    rows_product<double>(*B, B->Om64.p, B->Y64.p, cand);
                }
                SVDB_CUDA(cudaEventRecord(e1, s));
                SVDB_CUDA(cudaEventSynchronize(e1));
                SVDB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            };
            run();  // warm
            run();
            if (ms < best) { best = ms; gs = cand; }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        B->tune_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned[key] = gs;
    }
    B->gs = gs;

    // capture the solve
    SVDB_CUDA(cudaStreamSynchronize(s));
    const uint64_t l0 = svdb_kernel_launches();
    if (B->use_graph) {
        SVDB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue_any(*B);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(s, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        SVDB_CUDA(cudaStreamEndCapture(s, &B->graph));
        SVDB_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
        SVDB_CUDA(cudaGraphGetNodes(B->graph, nullptr, &B->graph_nodes));
        // the capture counted its launches; they run with each svdb_batch_run
        B->kernels_per_run = svdb_kernel_launches() - l0;
        discount_launches(B->kernels_per_run);
    }
    *out = B.release();
}

void batch_run(svdb_batch* B, svdb_rec* outs) {
    cudaStream_t s = B->s;
    cudaEvent_t e0, e1;
    SVDB_CUDA(cudaEventCreate(&e0));
    SVDB_CUDA(cudaEventCreate(&e1));
    SVDB_CUDA(cudaEventRecord(e0, s));
    if (B->use_graph) {
        SVDB_CUDA(cudaGraphLaunch(B->exec, s));
        count_launches(B->kernels_per_run);
    } else {
        const uint64_t l0 = svdb_kernel_launches();
        enqueue_any(*B);
        B->kernels_per_run = svdb_kernel_launches() - l0;
    }
    SVDB_CUDA(cudaEventRecord(e1, s));
    std::vector<int> flags(B->count), jst(B->count);
    SVDB_CUDA(cudaMemcpyAsync(flags.data(), B->flags.p, B->count * sizeof(int), cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaMemcpyAsync(jst.data(), B->jstat.p, B->count * sizeof(int), cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    B->last_ms = ms;
    if (B->dsplit) dense_split_check();
    for (int64_t b = 0; b < B->count; ++b)
        if (flags[b] & 2)
            throw Error(SVDB_ERR_LAS2, "randomized_svd batch: CholeskyQR broke down even with a shift in subset " +
                                           std::to_string(b));
    if (!outs) return;
    const int64_t m = B->m, d = B->rank;
    std::vector<double> sig((size_t)B->count * B->l);
    SVDB_CUDA(cudaMemcpyAsync(sig.data(), B->sig.p, sig.size() * 8, cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaStreamSynchronize(s));
    for (int64_t b = 0; b < B->count; ++b) {
        svdb_rec* r = outs + b;
        std::memset(r, 0, sizeof(*r));
        const int64_t nb = B->coff_h[b + 1] - B->coff_h[b];
        r->d = d;
        r->u_rows = m; r->u_cols = d;
        r->vt_rows = d; r->vt_cols = nb;
        const double* du = B->U.p + b * m * d;
        const double* dvt = B->Vt.p + B->coff_h[b] * d;
        if (B->on_device) {
            SVDB_CUDA(cudaMalloc(&r->u, std::max<int64_t>(m * d, 1) * 8));
            SVDB_CUDA(cudaMalloc(&r->s, std::max<int64_t>(d, 1) * 8));
            SVDB_CUDA(cudaMalloc(&r->vt, std::max<int64_t>(d * nb, 1) * 8));
            SVDB_CUDA(cudaMemcpyAsync(r->u, du, m * d * 8, cudaMemcpyDeviceToDevice, s));
            SVDB_CUDA(cudaMemcpyAsync(r->s, sig.data() + b * B->l, d * 8, cudaMemcpyHostToDevice, s));
            SVDB_CUDA(cudaMemcpyAsync(r->vt, dvt, d * nb * 8, cudaMemcpyDeviceToDevice, s));
            r->on_device = 1;
        } else {
            r->u = (double*)host_result_alloc(std::max<int64_t>(m * d, 1) * 8);
            r->s = (double*)host_result_alloc(std::max<int64_t>(d, 1) * 8);
            r->vt = (double*)host_result_alloc(std::max<int64_t>(d * nb, 1) * 8);
            if (!r->u || !r->s || !r->vt) throw std::bad_alloc();
            SVDB_CUDA(cudaMemcpyAsync(r->u, du, m * d * 8, cudaMemcpyDeviceToHost, s));
            std::memcpy(r->s, sig.data() + b * B->l, d * 8);
            SVDB_CUDA(cudaMemcpyAsync(r->vt, dvt, d * nb * 8, cudaMemcpyDeviceToHost, s));
        }
        r->origin = SVDB_REC_RANDOMIZED;
        svdb_diagnostics& dg = r->diagnostics;
        dg.non_zero = 0;
        dg.dimensions = B->rank;
        dg.iterations = B->q;
        dg.ritz_values_stabilized = d;
        dg.significant_values = d;
        dg.singular_values = d;
        dg.end_interval[0] = -1e-30;
        dg.end_interval[1] = 1e-30;
        dg.kappa = 1e-6;
        dg.random_seed = (uint32_t)B->seed;
        r->time_ms_total = ms;
    }
    SVDB_CUDA(cudaStreamSynchronize(s));
}

const svdb_matrix* batch_matrix(const svdb_batch* B) { return B->A; }
void batch_destroy(svdb_batch* B) { delete B; }

void batch_info(const svdb_batch* B, svdb_batch_info* info) {
    std::memset(info, 0, sizeof(*info));
    info->count = B->count;
    info->subsets_per_row_item = B->gs;
    info->columns_per_lane = B->cpl;
    info->graph_nodes = B->graph_nodes;
    info->kernels_per_run = B->kernels_per_run;
    info->time_ms_tune = B->tune_ms;
    info->time_ms_last_run = B->last_ms;
    info->total_subset_nnz = B->total_nnz;
}

}  // namespace svdb
