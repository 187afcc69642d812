// Dense-column split of the FP32 SpMM (SVDB_MIXED), for A X and A^T Y with
// at most 64 dense columns, the products of randomized_svd
// (src/lanczos/masked.rs:265-471,616-733).
//
// The columns of A whose density is at least a threshold (3 % by default)
// are copied, once per matrix, into a dense block D = A[:, J] (m x nd, FP32,
// row-major) and its transpose Dt (nd x m).  Their share of every product
// then runs on the tensor cores as a streamed GEMM instead of a row gather
// per nonzero:
//
//   A X   = A_rest X          + D  X[J, :]      (every row gets both parts)
//   A^T Y = A_rest^T Y        ; rows J: Dt Y     (disjoint rows)
//
// A_rest is A without the columns J; it keeps the segment-gather kernel.
// On the count-like randomized workload (Gamma(0.5)-weighted columns) the
// columns of density >= 3 % hold about 60 % of the nonzeros, and their
// gathers of 240-byte dense rows through L2 were most of the SpMM's time.
//
// k_dense_tc computes C (128 x 64 tile) = A_tile (128 x K) . B (64 x K)^T in
// 3xTF32 (A = Ah + Al, B = Bh + Bl, C = Ah Bh + Ah Bl + Al Bh, each term
// with FP32 accumulation in tensor memory), draining the accumulator into
// FP64 every `chunk` stages of 32 columns of K.  Warp roles, one CTA per SM:
//   warp 0      TMA producer: A stage (128 x 32 FP32, 128-byte swizzle) and
//               the Bh, Bl stages (64 x 32) into a 4-deep shared-memory ring;
//   warp 1      tensor-memory owner and MMA issuer (one thread): A from tensor
//               memory (tcgen05.mma ... [a_tmem]), B from shared memory;
//   warps 2..5  read the A stage (one row per thread), split it into its TF32
//               head and remainder, store both into tensor memory
//               (tcgen05.st), and drain the accumulators into FP64.
// Keeping A out of shared memory after the TMA copy (its split goes to tensor
// memory) leaves shared memory 2 bytes of traffic per byte of A instead of 7.
// Every mbarrier wait is bounded (SVDB_WAIT_LIMIT_NS, 2 s by default); on a
// timeout the kernel raises g_dense_err, every role leaves its loop, the
// copies and MMAs in flight are waited for (bounded) and tensor memory is
// freed.  No TMA load uses multicast; every tensor map covers this GPU's own
// memory.
#include <cub/cub.cuh>
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <type_traits>
#include <vector>

#include "device_common.cuh"
#include "ops.cuh"
#include "svdb_internal.h"

#ifndef SVDB_DT_CHUNK
#define SVDB_DT_CHUNK 1
#endif

namespace svdb {

constexpr int kDtM = 128;                                  // rows per tile (tensor-memory lanes)
constexpr int kDtN = 64;                                   // output columns per tile (l <= 64)
constexpr int kDtK = 32;                                   // K per stage: one 128-byte swizzle row
constexpr int kDtStages = 4;                               // shared-memory ring
constexpr int kDtAccs = 4;                                 // accumulators in tensor memory
constexpr int kDtAbytes = kDtM * kDtK * 4;                 // 16 KB (head or remainder)
constexpr int kDtBbytes = kDtN * kDtK * 4;                 // 8 KB (head or remainder)
constexpr int kDtStageBytes = 2 * kDtAbytes + 2 * kDtBbytes;  // 48 KB
constexpr int kDtSmem = kDtStages * kDtStageBytes + 1024;
constexpr int kDtThreads = 320;                            // producer, MMA and 8 drain warps
// Stages per FP64 drain.  The tensor cores add each MMA's products into the
// FP32 accumulator with truncation, a bias toward zero that grows with the
// number of MMAs summed in one accumulator: drained every 32 stages (1,024
// columns of K) it shrank the randomized solve's singular values by 4-6e-6
// relative; drained every stage (12 MMAs) by 2e-7.
constexpr int kDtChunk = SVDB_DT_CHUNK;
// F32 accumulator, TF32 A and B, both K-major, N = 64, M = 128
constexpr uint32_t kDtIdesc =
    (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kDtN >> 3) << 17) | ((uint32_t)(kDtM >> 4) << 24);
// tensor memory: four accumulators of 64 columns
constexpr uint32_t kDtTmemCols = kDtAccs * kDtN;

__device__ int g_dense_err;

// Work items: (K split ks, N tile nt, M tile mt).  In a K split the M tiles
// go in groups of kDtGroup, and a group runs through every N tile before the
// next group starts, so the group's A tiles and the N tiles in flight stay
// in L2.  Column g of the product is column g - 64 nt of N tile nt.
constexpr int kDtGroup = 16;
struct DtArgs {
    int64_t rows;     // valid rows of A (output rows in modes 0 and 2)
    int64_t k_total;  // K extent of A and B
    int64_t k_per;    // K per work item (a multiple of kDtK)
    int64_t kst;      // K stages of A and B (k_total / kDtK): tiles per tile row of the pre-tiled operands
    int32_t m_tiles, k_splits, n_tiles;
    int32_t l;        // mode 0: output columns; mode 2: columns per subset
    int32_t mode;     // 0: out[row * ldo + g] += C (g < l)
                      // 1: out[(((ks * n_tiles + nt) * m_tiles * 128) + row) * 64 + j] = C
                      // 2: out[(b * bm + row) * l + c] += C, g = b l + c (b < bcount): a batch of products
    int32_t out_f32;  // modes 0 and 2: out holds floats (else doubles)
    void* out;
    int64_t ldo;
    int64_t bm, bcount;  // mode 2: rows per product block, products
    unsigned long long limit_ns;
};

__device__ __forceinline__ uint32_t dt_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// The GEMM operands are stored pre-tiled: tiles of R rows x 32 K (R = 128
// for A, 64 for B), each tile one contiguous R x 128-byte block, tiles in
// row-of-tiles order (kst tiles per row of tiles).  A stage's TMA copy then
// reads one contiguous block instead of R pieces of 128 bytes spread over R
// rows.  Offset of element (r, k):
__host__ __device__ __forceinline__ int64_t dt_tiled(int64_t r, int64_t k, int64_t kst, int R) {
    return (((r / R) * kst + (k >> 5)) * R + (r % R)) * 32 + (k & 31);
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart
__device__ __forceinline__ uint64_t dt_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           (1ull << 46) | (2ull << 61);
}

// bounded wait that also gives up when another role has aborted
__device__ __forceinline__ bool dt_wait(uint32_t bar, uint32_t parity, unsigned long long limit,
                                        volatile int* abort) {
    const unsigned long long t0 = global_ns();
    uint32_t ok = 0, spins = 0;
    while (true) {
        // the thread sleeps in the wait (up to the hint, 20 us) instead of spinning
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(bar), "r"(parity), "r"(20000u)
            : "memory");
        if (ok) return true;
        if ((++spins & 3u) == 0) {
            if (*abort) return false;
            if (global_ns() - t0 > limit) {
                *abort = 1;
                atomicOr(&g_dense_err, 1);
                return false;
            }
        }
    }
}

__device__ __forceinline__ void dt_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void dt_tma(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void dt_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::"r"(d),
        "l"(a), "l"(b), "r"(kDtIdesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void dt_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

#define DT_LD32(v, taddr)                                                                                          \
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, " \
                 "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, " \
                 "[%32];"                                                                                          \
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),  \
                   "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),         \
                   "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),       \
                   "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),       \
                   "=r"(v[29]), "=r"(v[30]), "=r"(v[31])                                                            \
                 : "r"(taddr)                                                                                      \
                 : "memory")

// TF32 head of x, rounded to nearest (the remainder x - head is exact in FP32)
__device__ __forceinline__ float tf32_head(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}
// The remainder of a 3xTF32 split, itself rounded to TF32.  The tensor cores
// read an FP32 operand as TF32 by dropping its low 13 bits; left to them the
// remainder would be truncated, an error of one sign that does not cancel
// in long sums of terms of both signs (it cost a factor of about 100 in the
// singular values of a randomized solve).  Rounded here, the operand is
// exactly TF32 and the error is a rounding error.
__device__ __forceinline__ float tf32_tail(double x, float head) { return tf32_head((float)(x - (double)head)); }

// hi + lo += v with Knuth's TwoSum: the rounding error of hi + v, recovered
// exactly, goes into lo (explicit round-to-nearest additions, no contraction)
__device__ __forceinline__ void two_sum(float& hi, float& lo, float v) {
    const float s = __fadd_rn(hi, v);
    const float bv = __fsub_rn(s, hi);
    const float e = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bv)), __fsub_rn(v, bv));
    hi = s;
    lo = __fadd_rn(lo, e);
}

// C = (Ah + Al)(Bh + Bl)^T less the Al Bl term: three TF32 MMAs per K step
// into an FP32 accumulator in tensor memory, drained into FP64 registers
// every kDtChunk stages.  Warp 0: TMA producer (one thread); warp 1: tensor
// memory owner and MMA issuer (one thread); warps 2-9: drains, warp w reading
// tensor-memory lanes 32 (w % 4) to 32 (w % 4) + 31 (one output row a
// thread) and accumulator columns 32 (w - 2) / 4 to that + 31.
__global__ void __launch_bounds__(kDtThreads, 1)
    k_dense_tc(const __grid_constant__ CUtensorMap ahmap, const __grid_constant__ CUtensorMap almap,
               const __grid_constant__ CUtensorMap bhmap, const __grid_constant__ CUtensorMap blmap,
               const DtArgs a) {
    extern __shared__ unsigned char dyn[];
    __shared__ __align__(8) uint64_t bar_full[kDtStages], bar_empty[kDtStages], bar_accf[kDtAccs],
        bar_acce[kDtAccs], bar_fin;
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(dyn) + 1023) & ~uintptr_t(1023));
    volatile int* abort = &s_abort;

    if (tid == 0) {
        for (int s = 0; s < kDtStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(dt_smem(&bar_full[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(dt_smem(&bar_empty[s])) : "memory");
        }
        for (int b = 0; b < kDtAccs; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(dt_smem(&bar_accf[b])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 8;" ::"r"(dt_smem(&bar_acce[b])) : "memory");
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(dt_smem(&bar_fin)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dt_smem(&s_tmem)),
                     "r"(kDtTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const int64_t per_k = (int64_t)a.m_tiles * a.n_tiles;
    const int64_t items = per_k * a.k_splits;
    auto item_geom = [&](int64_t it, int64_t& m0, int64_t& kb, int& nst, int& ks, int& nt) {
        ks = (int)(it / per_k);
        const int64_t rem = it - (int64_t)ks * per_k;
        const int64_t grp = rem / ((int64_t)kDtGroup * a.n_tiles);
        const int64_t within = rem - grp * kDtGroup * a.n_tiles;
        const int64_t gsize = min((int64_t)kDtGroup, (int64_t)a.m_tiles - grp * kDtGroup);
        nt = (int)(within / gsize);
        m0 = (grp * kDtGroup + (within - (int64_t)nt * gsize)) * kDtM;
        kb = (int64_t)ks * a.k_per;
        const int64_t ke = min(a.k_total, kb + a.k_per);
        nst = (int)((ke - kb + kDtK - 1) / kDtK);
    };

    if (warp == 0 && lane == 0) {
        // ------------------------------------------------------- producer --
        uint32_t issued = 0;
        for (int64_t it = blockIdx.x; it < items && !*abort; it += gridDim.x) {
            int64_t m0, kb;
            int nst, ks, nt;
            item_geom(it, m0, kb, nst, ks, nt);
            bool ok = true;
            for (int st = 0; st < nst; ++st, ++issued) {
                const int s = issued % kDtStages;
                if (!dt_wait(dt_smem(&bar_empty[s]), ((issued / kDtStages) & 1) ^ 1, a.limit_ns, abort)) {
                    ok = false;
                    break;
                }
                unsigned char* base = sm + s * kDtStageBytes;
                const uint32_t fb = dt_smem(&bar_full[s]);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(kDtStageBytes)
                             : "memory");
                const int64_t kt = kb / kDtK + st;  // K tile
                const int ya = (int)(((m0 / kDtM) * a.kst + kt) * kDtM);
                const int yb = (int)(((int64_t)nt * a.kst + kt) * kDtN);
                dt_tma(dt_smem(base), &ahmap, 0, ya, fb);
                dt_tma(dt_smem(base + kDtAbytes), &almap, 0, ya, fb);
                dt_tma(dt_smem(base + 2 * kDtAbytes), &bhmap, 0, yb, fb);
                dt_tma(dt_smem(base + 2 * kDtAbytes + kDtBbytes), &blmap, 0, yb, fb);
            }
            if (!ok) break;
        }
        // every copy issued must land before the CTA may exit
        for (uint32_t q = 0; q < kDtStages && q < issued; ++q) {
            const uint32_t last = issued - 1 - q;  // the last issue into slot last % kDtStages
            volatile int never = 0;
            dt_wait(dt_smem(&bar_full[last % kDtStages]), (last / kDtStages) & 1, 2000000000ull, &never);
        }
    } else if (warp == 1 && lane == 0) {
        // ------------------------------------------------------------ MMA --
        uint32_t issued = 0, ch = 0;
        bool any = false;
        for (int64_t it = blockIdx.x; it < items && !*abort; it += gridDim.x) {
            int64_t m0, kb;
            int nst, ks, nt;
            item_geom(it, m0, kb, nst, ks, nt);
            bool ok = true;
            for (int st = 0; st < nst; ++st, ++issued) {
                const int s = issued % kDtStages, b = ch % kDtAccs;
                const bool first = (st % kDtChunk) == 0, last = (st % kDtChunk) == kDtChunk - 1 || st == nst - 1;
                if (first && !dt_wait(dt_smem(&bar_acce[b]), ((ch / kDtAccs) & 1) ^ 1, a.limit_ns, abort)) {
                    ok = false;
                    break;
                }
                if (!dt_wait(dt_smem(&bar_full[s]), (issued / kDtStages) & 1, a.limit_ns, abort)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const unsigned char* base = sm + s * kDtStageBytes;
                const uint64_t ah = dt_desc(dt_smem(base));
                const uint64_t al = dt_desc(dt_smem(base + kDtAbytes));
                const uint64_t bh = dt_desc(dt_smem(base + 2 * kDtAbytes));
                const uint64_t bl = dt_desc(dt_smem(base + 2 * kDtAbytes + kDtBbytes));
                const uint32_t d = tmem + (uint32_t)b * kDtN;
#pragma unroll
                for (int kk = 0; kk < kDtK / 8; ++kk) {
                    const uint64_t koff = (uint64_t)((kk * 32) >> 4);  // 8 TF32 = 32 bytes along the swizzled row
                    dt_mma(d, ah + koff, bh + koff, (first && kk == 0) ? 0u : 1u);
                    dt_mma(d, ah + koff, bl + koff, 1u);
                    dt_mma(d, al + koff, bh + koff, 1u);
                }
                any = true;
                dt_commit(dt_smem(&bar_empty[s]));
                if (last) {
                    dt_commit(dt_smem(&bar_accf[b]));
                    ++ch;
                }
            }
            if (!ok) break;
        }
        if (any) {  // the last MMAs must complete before tensor memory is freed
            dt_commit(dt_smem(&bar_fin));
            volatile int never = 0;
            dt_wait(dt_smem(&bar_fin), 0, 2000000000ull, &never);
        }
    } else if (warp >= 2) {
        // ------------------------------- drain into FP32 pairs, write FP64 --
        // Each output is kept as an unevaluated sum hi + lo of two floats;
        // a drained value v is added with the error-free TwoSum (Knuth):
        // s = hi + v exactly equals s + e, e from five more additions, and e
        // goes into lo.  FP32 additions run at four times the rate of the
        // FP32-to-FP64 conversions an FP64 sum would take per value.
        constexpr int kH = kDtN / 2;             // accumulator columns per drain warp
        const int g = warp & 3;                  // tensor-memory lane group of this warp
        const int c0 = ((warp - 2) >> 2) * kH;   // first accumulator column of this warp
        const int r = g * 32 + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(g * 32) << 16) + (uint32_t)c0;
        float hi[kH], lo[kH];
#pragma unroll
        for (int j = 0; j < kH; ++j) hi[j] = lo[j] = 0.f;
        uint32_t ch = 0;
        bool ok = true;
        for (int64_t it = blockIdx.x; it < items && ok && !*abort; it += gridDim.x) {
            int64_t m0, kb;
            int nst, ks, nt;
            item_geom(it, m0, kb, nst, ks, nt);
            const int nch = (nst + kDtChunk - 1) / kDtChunk;
            for (int c = 0; c < nch; ++c, ++ch) {
                const int b = ch % kDtAccs;
                if (!dt_wait(dt_smem(&bar_accf[b]), (ch / kDtAccs) & 1, a.limit_ns, abort)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                uint32_t v[32];
                DT_LD32(v, lane_base + (uint32_t)b * kDtN);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0) dt_arrive(dt_smem(&bar_acce[b]));
#pragma unroll
                for (int j = 0; j < kH; ++j) two_sum(hi[j], lo[j], __uint_as_float(v[j]));
            }
            if (!ok) break;
#define DT_ACC(j) ((double)hi[j] + (double)lo[j])
            const int64_t row = m0 + r;
            const int64_t g0 = (int64_t)nt * kDtN + c0;  // product column of this thread's first value
            if (a.mode == 0) {
                if (row < a.rows) {
                    const int jn = (int)min((int64_t)kH, (int64_t)a.l - g0);
                    if (a.out_f32) {
                        float* o = static_cast<float*>(a.out) + row * a.ldo + g0;
#pragma unroll
                        for (int j = 0; j < kH; ++j)
                            if (j < jn) o[j] = (float)((double)o[j] + DT_ACC(j));
                    } else {
                        double* o = static_cast<double*>(a.out) + row * a.ldo + g0;
#pragma unroll
                        for (int j = 0; j < kH; ++j)
                            if (j < jn) o[j] += DT_ACC(j);
                    }
                }
            } else if (a.mode == 2) {
                if (row < a.rows) {
                    // column g0 + j is column c of product bb; step (bb, c) along j
                    int64_t bb = g0 / a.l, cc = g0 - bb * a.l;
#pragma unroll
                    for (int j = 0; j < kH; ++j) {
                        if (bb < a.bcount) {
                            const int64_t at = (bb * a.bm + row) * a.l + cc;
                            if (a.out_f32) {
                                float* o = static_cast<float*>(a.out);
                                o[at] = (float)((double)o[at] + DT_ACC(j));
                            } else {
                                static_cast<double*>(a.out)[at] += DT_ACC(j);
                            }
                        }
                        if (++cc == a.l) {
                            cc = 0;
                            ++bb;
                        }
                    }
                }
            } else {
                double2* o = reinterpret_cast<double2*>(static_cast<double*>(a.out) +
                                                        ((((int64_t)ks * a.n_tiles + nt) * a.m_tiles * kDtM) + row) *
                                                            kDtN +
                                                        c0);
#pragma unroll
                for (int j = 0; j < kH / 2; ++j) o[j] = make_double2(DT_ACC(2 * j), DT_ACC(2 * j + 1));
            }
#undef DT_ACC
#pragma unroll
            for (int j = 0; j < kH; ++j) hi[j] = lo[j] = 0.f;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kDtTmemCols) : "memory");
    }
}

// ------------------------------------------------------- operand prep --
// B of A X: Bh/Bl (64 x kp, pre-tiled) = TF32 head / remainder of
// X[cols[k], j] (zero past l and for padding columns cols[k] < 0).  Thread i
// writes element i of the tiled buffer: tile i / 2048 is K tile k / 32.
template <typename XT>
__global__ void k_dense_b_gather(const XT* __restrict__ X, int l, const int32_t* __restrict__ cols, int64_t kp,
                                 float* __restrict__ bh, float* __restrict__ bl) {
    const int64_t total = (int64_t)kDtN * kp;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)((i >> 5) & (kDtN - 1));
        const int64_t k = (i / (kDtN * 32)) * 32 + (i & 31);
        const int32_t c = cols[k];
        const double x = (j < l && c >= 0) ? (double)X[(int64_t)c * l + j] : 0.0;
        const float h = tf32_head((float)x);
        bh[i] = h;
        bl[i] = tf32_tail(x, h);
    }
}

// B of A^T Y: Bh/Bl (64 x kp, pre-tiled) = head / remainder of Y^T (Y: rows
// x l), zero past rows and l.  32 x 32 tiles through shared memory.
template <typename XT>
__global__ void k_dense_b_transpose(const XT* __restrict__ Y, int64_t rows, int l, int64_t kp,
                                    float* __restrict__ bh, float* __restrict__ bl) {
    __shared__ double tile[32][33];
    const int64_t k0 = (int64_t)blockIdx.x * 32;
    const int j0 = blockIdx.y * 32;
    for (int rr = threadIdx.y; rr < 32; rr += blockDim.y) {
        const int64_t k = k0 + rr;
        const int j = j0 + threadIdx.x;
        tile[rr][threadIdx.x] = (k < rows && j < l) ? (double)Y[k * l + j] : 0.0;
    }
    __syncthreads();
    for (int jj = threadIdx.y; jj < 32; jj += blockDim.y) {
        const int j = j0 + jj;
        const int64_t k = k0 + threadIdx.x;
        if (k < kp) {
            const double x = tile[threadIdx.x][jj];
            const float h = tf32_head((float)x);
            const int64_t at = dt_tiled(j, k, kp / kDtK, kDtN);
            bh[at] = h;
            bl[at] = tf32_tail(x, h);
        }
    }
}

// Z[cols[r], j] = sum over the K splits of the partial tiles (fixed order)
template <typename OT>
__global__ void k_dense_reduce(const double* __restrict__ part, int ksplits, int64_t mrows, int64_t nd,
                               const int32_t* __restrict__ cols, int l, OT* __restrict__ Z) {
    const int64_t total = nd * l;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / l;
        const int j = (int)(i - r * l);
        double acc = 0.0;
        for (int k = 0; k < ksplits; ++k) acc += part[((int64_t)k * mrows + r) * kDtN + j];
        Z[(int64_t)cols[r] * l + j] = (OT)acc;
    }
}

// --------------------------------------------------------------- build --
// D[r, k] and Dt[k, r] from column cols[k] of the CSC (one warp per column),
// as TF32 heads (D, Dt) and TF32-rounded remainders (Dl, Dtl), pre-tiled
// (128-row tiles; D: ndp / 32 K tiles a row of tiles, Dt: mp / 32).
__global__ void k_dense_scatter(const int64_t* __restrict__ cp, const int32_t* __restrict__ ri,
                                const float* __restrict__ v, const int32_t* __restrict__ cols, int64_t nd,
                                int64_t ndp, int64_t mp, float* __restrict__ D, float* __restrict__ Dl,
                                float* __restrict__ Dt, float* __restrict__ Dtl) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t k = gw; k < nd; k += nw) {
        const int32_t c = cols[k];
        for (int64_t e = cp[c] + lane; e < cp[c + 1]; e += 32) {
            const int64_t r = ri[e];
            const float h = tf32_head(v[e]), t = tf32_head(v[e] - h);  // v - h is exact
            const int64_t od = dt_tiled(r, k, ndp / kDtK, kDtM), ot = dt_tiled(k, r, mp / kDtK, kDtM);
            D[od] = h;
            Dl[od] = t;
            Dt[ot] = h;
            Dtl[ot] = t;
        }
    }
}

// entries of each major slice kept when keep(minor) (drop_major: the whole
// slice is dropped when the major index is flagged instead); counts first
__global__ void k_rest_count(const int64_t* __restrict__ p, const int32_t* __restrict__ idx, int64_t nmajor,
                             const uint8_t* __restrict__ dense, bool by_major, int64_t* __restrict__ cnt) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = gw; r <= nmajor; r += nw) {
        if (r == nmajor) {
            if (lane == 0) cnt[r] = 0;
            continue;
        }
        int64_t c = 0;
        if (by_major) {
            c = dense[r] ? 0 : p[r + 1] - p[r];
        } else {
            for (int64_t e = p[r] + lane; e < p[r + 1]; e += 32) c += dense[idx[e]] ? 0 : 1;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        }
        if (lane == 0) cnt[r] = c;
    }
}

__global__ void k_rest_fill(const int64_t* __restrict__ p, const int32_t* __restrict__ idx,
                            const float* __restrict__ v, int64_t nmajor, const uint8_t* __restrict__ dense,
                            bool by_major, const int64_t* __restrict__ np, int32_t* __restrict__ nidx,
                            float* __restrict__ nv) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = gw; r < nmajor; r += nw) {
        if (by_major && dense[r]) continue;
        int64_t out = np[r];
        for (int64_t e0 = p[r]; e0 < p[r + 1]; e0 += 32) {
            const int64_t e = e0 + lane;
            const bool in = e < p[r + 1];
            const int32_t c = in ? idx[e] : 0;
            const bool keep = in && (by_major || !dense[c]);
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const int64_t o = out + __popc(m & ((1u << lane) - 1u));
                nidx[o] = c;
                nv[o] = v[e];
            }
            out += __popc(m);
        }
    }
}

static PFN_cuTensorMapEncodeTiled_v12000 dt_encode() {
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

// A pre-tiled FP32 operand seen as rows of 32 floats (128 bytes), `rows`
// of them, copied in boxes of box_rows x 32 with the 128-byte swizzle
static CUtensorMap dt_map(const float* base, int64_t rows, int box_rows) {
    CUtensorMap m;
    const cuuint64_t gdim[2] = {(cuuint64_t)kDtK, (cuuint64_t)rows};
    const cuuint64_t gstr[1] = {(cuuint64_t)kDtK * 4};
    const cuuint32_t box[2] = {(cuuint32_t)kDtK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    if ((reinterpret_cast<uintptr_t>(base) & 15) || rows % box_rows || rows >= ((int64_t)1 << 31))
        throw Error(SVDB_ERR_CUDA, "dense split: operand not laid out for the tensor memory accelerator");
    CUresult r = dt_encode()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), gdim, gstr, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(SVDB_ERR_CUDA, "dense split: cuTensorMapEncodeTiled failed");
    return m;
}

static int dt_grid(int64_t items) {
    return (int)std::max<int64_t>(1, std::min<int64_t>(items, device_props().sms));
}

// C = A (a_rows x a_cols) . B^T with A given as its TF32 head ah and
// remainder al (pre-tiled, rows padded to 128), B (n_tiles * 64 rows x
// a_cols, pre-tiled) as bh and bl; a_cols a multiple of 32; see DtArgs for
// the modes.
struct DtLaunch {
    const float *ah, *al;
    int64_t a_rows, a_cols;
    const float *bh, *bl;
    int n_tiles = 1;
    int64_t k_per = 0;
    int ksplits = 1;
    int l = 0, mode = 0;
    bool out_f32 = false;
    void* out = nullptr;
    int64_t ldo = 0, bm = 0, bcount = 0;
};

static void dt_launch(const DtLaunch& p, cudaStream_t s) {
    static std::once_flag attr;
    std::call_once(attr, [] {
        SVDB_CUDA(cudaFuncSetAttribute(k_dense_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kDtSmem));
    });
    if (p.a_cols % kDtK) throw Error(SVDB_ERR_CUDA, "dense split: K not a multiple of 32");
    const int64_t kst = p.a_cols / kDtK;
    const int64_t a_tiles = (p.a_rows + kDtM - 1) / kDtM;
    const CUtensorMap ahm = dt_map(p.ah, a_tiles * kst * kDtM, kDtM);
    const CUtensorMap alm = dt_map(p.al, a_tiles * kst * kDtM, kDtM);
    const CUtensorMap hm = dt_map(p.bh, (int64_t)p.n_tiles * kst * kDtN, kDtN);
    const CUtensorMap lm = dt_map(p.bl, (int64_t)p.n_tiles * kst * kDtN, kDtN);
    DtArgs g;
    g.rows = p.a_rows;
    g.k_total = p.a_cols;
    g.k_per = p.k_per ? p.k_per : p.a_cols;
    g.kst = kst;
    g.m_tiles = (int)((p.a_rows + kDtM - 1) / kDtM);
    g.k_splits = p.ksplits;
    g.n_tiles = p.n_tiles;
    g.l = p.l;
    g.mode = p.mode;
    g.out_f32 = p.out_f32 ? 1 : 0;
    g.out = p.out;
    g.ldo = p.ldo;
    g.bm = p.bm;
    g.bcount = p.bcount;
    g.limit_ns = wait_limit_ns();
    const int64_t items = (int64_t)g.m_tiles * p.ksplits * p.n_tiles;
    k_dense_tc<<<dt_grid(items), kDtThreads, kDtSmem, s>>>(ahm, alm, hm, lm, g);
    SVDB_CHECK_LAUNCH();
}

void dense_split_check() {
    int e = 0;
    SVDB_CUDA(cudaMemcpyFromSymbol(&e, g_dense_err, sizeof(int)));
    if (e) {
        const int z = 0;
        SVDB_CUDA(cudaMemcpyToSymbol(g_dense_err, &z, sizeof(int)));
        throw Error(SVDB_ERR_TIMEOUT, "dense split: a tensor-core pipeline wait exceeded its limit");
    }
}

static int64_t nblocks(int64_t work, int threads) {
    return std::max<int64_t>(1, std::min<int64_t>((work + threads - 1) / threads, (int64_t)device_props().sms * 16));
}

// Compacted copy of `src` keeping the entries whose minor index is not dense
// (by_major = false) or the major slices that are not dense (by_major = true).
static void build_rest(const DevCompressed& src, const uint8_t* dense, bool by_major, DevCompressed& out,
                       cudaStream_t s) {
    out.nmajor = src.nmajor;
    out.nminor = src.nminor;
    out.owner_stream = s;
    out.ptr.alloc(src.nmajor + 1, s);
    DevBuf<int64_t> cnt(src.nmajor + 1, s);
    k_rest_count<<<(int)nblocks((src.nmajor + 1) * 32, 256), 256, 0, s>>>(src.ptr.p, src.idx.p, src.nmajor, dense,
                                                                           by_major, cnt.p);
    SVDB_CHECK_LAUNCH();
    size_t tb = 0;
    SVDB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.p, out.ptr.p, src.nmajor + 1, s));
    DevBuf<uint8_t> tmp(std::max<size_t>(tb, 1), s);
    SVDB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.p, out.ptr.p, src.nmajor + 1, s));
    int64_t nnz = 0;
    SVDB_CUDA(cudaMemcpyAsync(&nnz, out.ptr.p + src.nmajor, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaStreamSynchronize(s));
    out.nnz = nnz;
    out.idx.alloc(std::max<int64_t>(nnz, 1), s);
    out.val32.alloc(std::max<int64_t>(nnz, 1), s);
    k_rest_fill<<<(int)nblocks(src.nmajor * 32, 256), 256, 0, s>>>(src.ptr.p, src.idx.p, src.val32.p, src.nmajor,
                                                                   dense, by_major, out.ptr.p, out.idx.p, out.val32.p);
    SVDB_CHECK_LAUNCH();
    build_seg_plan(out, s);
}

static double dense_min_density() {
    const char* e = getenv("SVDB_DENSE_MIN_DENSITY");
    if (e && *e) return atof(e);
    return 0.08;
}

// Opt-in (SVDB_DENSE_SPLIT=1): with the lean gather kernel (k_spmm_lean) the
// split no longer shortens the randomized solve of the count-like workload
// (17.66 against 17.68 ms) and its sigma moves from 1e-8 to 2e-7 of the FP64
// solve, so the row gathers are the default.
static bool dense_enabled() {
    const char* e = getenv("SVDB_DENSE_SPLIT");
    return e && std::string(e) == "1";
}

static std::mutex g_dense_mu;

// The split of the structures `a` computes with, built on first use (under
// SVDB_MIXED, with FP32 values present).  Null when no column is dense
// enough, the matrix is small, or the split is switched off.
static DenseSplit* dense_split_for(const svdb_matrix* a) {
    const svdb_matrix* owner = (a->kind == KIND_MASKED && a->all_columns) ? a->parent : a;
    svdb_matrix* w = const_cast<svdb_matrix*>(owner);
    std::lock_guard<std::mutex> lk(g_dense_mu);
    if (w->dense_tried) return w->dense.get();
    w->dense_tried = true;
    const DevCompressed& csr = w->csr;
    const DevCompressed& csc = w->csc;
    const int64_t m = csr.nmajor, n = csr.nminor;
    if (m < 4 * kDtM || n < kDtM || !csr.val32.p || !csc.val32.p) return nullptr;
    cudaStream_t s = w->stream;
    // column counts from the CSC offsets; the densest columns first
    std::vector<int64_t> cp(n + 1);
    SVDB_CUDA(cudaMemcpyAsync(cp.data(), csc.ptr.p, (n + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaStreamSynchronize(s));
    const double thr = dense_min_density() * (double)m;
    std::vector<int32_t> order;
    for (int64_t j = 0; j < n; ++j)
        if ((double)(cp[j + 1] - cp[j]) >= thr) order.push_back((int32_t)j);
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t x, int32_t y) { return cp[x + 1] - cp[x] > cp[y + 1] - cp[y]; });
    // memory: D, Dt and their remainders take 16 m nd bytes; keep them under a quarter of the free memory and 16 GB
    size_t free_b = 0, total_b = 0;
    SVDB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const double cap = std::min<double>(16e9, 0.25 * (double)free_b);
    const int64_t mp = (m + kDtK - 1) / kDtK * kDtK;
    int64_t nd_max = (int64_t)(cap / (16.0 * (double)mp)) / kDtM * kDtM;
    int64_t nd = std::min<int64_t>((int64_t)order.size(), nd_max);
    if (nd < kDtM) return nullptr;
    order.resize(nd);
    std::sort(order.begin(), order.end());  // ascending columns: the operand gather reads X in order
    const int64_t ndp = (nd + kDtM - 1) / kDtM * kDtM;
    auto ds = std::make_unique<DenseSplit>();
    ds->nd = nd;
    ds->ndp = ndp;
    ds->mp = mp;
    std::vector<int32_t> cols(ndp, -1);
    std::copy(order.begin(), order.end(), cols.begin());
    std::vector<uint8_t> flag(n, 0);
    for (int32_t c : order) flag[c] = 1;
    ds->cols.alloc(ndp, s);
    DevBuf<uint8_t> dflag(n, s);
    SVDB_CUDA(cudaMemcpyAsync(ds->cols.p, cols.data(), ndp * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    SVDB_CUDA(cudaMemcpyAsync(dflag.p, flag.data(), n, cudaMemcpyHostToDevice, s));
    const int64_t m128 = (m + kDtM - 1) / kDtM * kDtM;  // D's rows, padded to whole tiles
    for (DevBuf<float>* b : {&ds->D, &ds->Dl}) {
        b->alloc((size_t)m128 * ndp, s);
        SVDB_CUDA(cudaMemsetAsync(b->p, 0, (size_t)m128 * ndp * sizeof(float), s));
    }
    for (DevBuf<float>* b : {&ds->Dt, &ds->Dtl}) {
        b->alloc((size_t)ndp * mp, s);
        SVDB_CUDA(cudaMemsetAsync(b->p, 0, (size_t)ndp * mp * sizeof(float), s));
    }
    k_dense_scatter<<<(int)nblocks(nd * 32, 256), 256, 0, s>>>(csc.ptr.p, csc.idx.p, csc.val32.p, ds->cols.p, nd, ndp,
                                                              mp, ds->D.p, ds->Dl.p, ds->Dt.p, ds->Dtl.p);
    SVDB_CHECK_LAUNCH();
    build_rest(csr, dflag.p, false, ds->rest_csr, s);
    build_rest(csc, dflag.p, true, ds->rest_csc, s);
    ds->dense_nnz = csr.nnz - ds->rest_csr.nnz;
    SVDB_CUDA(cudaStreamSynchronize(s));
    w->dense = std::move(ds);
    return w->dense.get();
}

// nd and the nonzeros in the dense block (0, 0 when the matrix has no split)
void dense_split_info(const svdb_matrix* a, uint64_t* nd, uint64_t* dense_nnz) {
    const svdb_matrix* owner = (a->kind == KIND_MASKED && a->all_columns) ? a->parent : a;
    std::lock_guard<std::mutex> lk(g_dense_mu);
    *nd = owner->dense ? (uint64_t)owner->dense->nd : 0;
    *dense_nnz = owner->dense ? (uint64_t)owner->dense->dense_nnz : 0;
}

bool dense_split_usable(const svdb_matrix* a, int l) {
    if (l < 1 || l > kDtN || !dense_enabled()) return false;
    return dense_split_for(a) != nullptr;
}

// Y (m x l) = A X (transpose = false; X: n x l) or Z (n x l) = A^T Y
// (transpose = true; Y: m x l), FP32 products; x32 is the FP32 copy of the
// dense operand (minor x l) that the sparse remainder gathers (X itself when
// XT is float).  Everything runs on stream s in order: the remainder writes
// every output row, then the dense part adds its share (A X) or writes the
// dense rows (A^T Y).
template <typename XT, typename OT>
void dense_split_spmm(const svdb_matrix* a, bool transpose, const XT* X, const float* x32, int l, OT* Y,
                      cudaStream_t s) {
    DenseSplit* ds = dense_split_for(a);
    if (!ds) throw Error(SVDB_ERR_ARG, "dense split: not available for this matrix");
    if (l < 1 || l > kDtN) throw Error(SVDB_ERR_ARG, "dense split: 1 to 64 dense columns");
    const int64_t m = ds->rest_csr.nmajor;
    constexpr bool of32 = std::is_same<OT, float>::value;
    if (!transpose) {
        spmm_dev<float, OT>(ds->rest_csr, true, x32, l, Y, s);  // every row written
        DevBuf<float> bh((size_t)kDtN * ds->ndp, s), bl((size_t)kDtN * ds->ndp, s);
        k_dense_b_gather<XT><<<(int)nblocks(kDtN * ds->ndp, 256), 256, 0, s>>>(X, l, ds->cols.p, ds->ndp, bh.p,
                                                                               bl.p);
        SVDB_CHECK_LAUNCH();
        DtLaunch p{ds->D.p, ds->Dl.p, m, ds->ndp, bh.p, bl.p};
        p.l = l;
        p.mode = 0;
        p.out_f32 = of32;
        p.out = Y;
        p.ldo = l;
        dt_launch(p, s);
    } else {
        spmm_dev<float, OT>(ds->rest_csc, true, x32, l, Y, s);  // dense rows written as 0
        DevBuf<float> bh((size_t)kDtN * ds->mp, s), bl((size_t)kDtN * ds->mp, s);
        dim3 tb(32, 8), tg((unsigned)(ds->mp / 32), (unsigned)(kDtN / 32));
        k_dense_b_transpose<XT><<<tg, tb, 0, s>>>(X, m, l, ds->mp, bh.p, bl.p);
        SVDB_CHECK_LAUNCH();
        const int64_t m_tiles = ds->ndp / kDtM;
        int ks = (int)std::max<int64_t>(1, (4 * (int64_t)device_props().sms + m_tiles - 1) / m_tiles);
        const int64_t k_per = ((ds->mp + ks - 1) / ks + kDtK - 1) / kDtK * kDtK;
        ks = (int)((ds->mp + k_per - 1) / k_per);
        DevBuf<double> part((size_t)ks * ds->ndp * kDtN, s);
        DtLaunch p{ds->Dt.p, ds->Dtl.p, ds->ndp, ds->mp, bh.p, bl.p};
        p.k_per = k_per;
        p.ksplits = ks;
        p.l = l;
        p.mode = 1;
        p.out = part.p;
        dt_launch(p, s);
        k_dense_reduce<OT><<<(int)nblocks(ds->nd * l, 256), 256, 0, s>>>(part.p, ks, ds->ndp, ds->nd, ds->cols.p, l,
                                                                          Y);
        SVDB_CHECK_LAUNCH();
    }
}

template void dense_split_spmm<double, double>(const svdb_matrix*, bool, const double*, const float*, int, double*,
                                               cudaStream_t);
template void dense_split_spmm<float, float>(const svdb_matrix*, bool, const float*, const float*, int, float*,
                                             cudaStream_t);

// ------------------------------------------------ batches of subsets --
// The products of a batch of column subsets (batch.cu) through the split:
// every subset's share of the dense columns in one GEMM whose N dimension is
// all subsets' sample columns side by side (g = b l + c).  The sparse rest
// runs through the batch's own gather kernels on split->rest_csr/rest_csc.

// B of the row products (npad x ndp, pre-tiled): head / remainder of
// X_b[o2m_b(J[k]), c] for row g = b l + c (zero when column J[k] is not in
// subset b, for padding columns, and for g >= count l); X_b sits at
// X + coff[b] l.  Thread i writes element i of the tiled buffer.
__global__ void k_bd_rows_b(const float* __restrict__ X, const int64_t* __restrict__ coff,
                            const int32_t* __restrict__ o2m, const int32_t* __restrict__ cols, int64_t n,
                            int64_t count, int l, int64_t ndp, int64_t npad, float* __restrict__ bh,
                            float* __restrict__ bl) {
    const int64_t total = npad * ndp;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = i / (kDtN * 32), kst = ndp / kDtK;  // tile t = (g / 64, k / 32)
        const int64_t g = (t / kst) * kDtN + ((i >> 5) & (kDtN - 1));
        const int64_t k = (t % kst) * 32 + (i & 31);
        const int64_t b = g / l, c = g - b * l;
        double x = 0.0;
        if (b < count && cols[k] >= 0) {
            const int32_t o = o2m[b * n + cols[k]];
            if (o >= 0) x = (double)X[(coff[b] + o) * l + c];
        }
        const float h = tf32_head((float)x);
        bh[i] = h;
        bl[i] = tf32_tail(x, h);
    }
}

// B of the column products (pre-tiled): head / remainder of Y_b[k, c] (Y_b
// at Y + b m l) for row g = b l + c, zero past m; 32 x 32 tiles per subset.
__global__ void k_bd_cols_b(const float* __restrict__ Y, int64_t m, int l, int64_t mp, float* __restrict__ bh,
                            float* __restrict__ bl) {
    __shared__ float tile[32][33];
    const int64_t b = blockIdx.z;
    const int64_t k0 = (int64_t)blockIdx.x * 32;
    const int c0 = blockIdx.y * 32;
    const float* Yb = Y + b * m * l;
    for (int rr = threadIdx.y; rr < 32; rr += blockDim.y) {
        const int64_t k = k0 + rr;
        const int c = c0 + threadIdx.x;
        tile[rr][threadIdx.x] = (k < m && c < l) ? Yb[k * l + c] : 0.f;
    }
    __syncthreads();
    for (int cc = threadIdx.y; cc < 32; cc += blockDim.y) {
        const int c = c0 + cc;
        const int64_t k = k0 + threadIdx.x;
        if (c < l && k < mp) {
            const double x = (double)tile[threadIdx.x][cc];
            const float h = tf32_head((float)x);
            const int64_t at = dt_tiled(b * l + c, k, mp / kDtK, kDtN);
            bh[at] = h;
            bl[at] = tf32_tail(x, h);
        }
    }
}

// Z_b[o2m_b(J[k]), c] = the GEMM's tile value for (row k, column b l + c)
template <typename OT>
__global__ void k_bd_reduce(const double* __restrict__ part, int64_t ndp, const int32_t* __restrict__ cols,
                            int64_t nd, const int32_t* __restrict__ o2m, const int64_t* __restrict__ coff, int64_t n,
                            int64_t count, int l, OT* __restrict__ Z) {
    const int64_t total = count * nd * l;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = i / (nd * l);
        const int64_t rem = i - b * nd * l;
        const int64_t k = rem / l, c = rem - k * l;
        const int32_t o = o2m[b * n + cols[k]];
        if (o < 0) continue;
        const int64_t g = b * l + c, nt = g / kDtN, j = g - nt * kDtN;
        Z[(coff[b] + o) * l + c] = (OT)part[(nt * ndp + k) * kDtN + j];
    }
}

const DenseSplit* dense_split_get(const svdb_matrix* a) { return dense_split_for(a); }

size_t dense_batch_workspace(const DenseSplit& ds, int64_t count, int l) {
    const int64_t npad = (count * l + kDtN - 1) / kDtN * kDtN;
    return (size_t)npad * (size_t)(ds.ndp + ds.mp) * 2 * sizeof(float) + (size_t)npad * ds.ndp * sizeof(double);
}

void dense_batch_rows(const svdb_matrix* a, const float* X, const int64_t* coff, const int32_t* o2m, int64_t count,
                      int l, float* Y, float* bh, float* bl, cudaStream_t s) {
    const DenseSplit* ds = dense_split_for(a);
    if (!ds) throw Error(SVDB_ERR_ARG, "dense split: not available for this matrix");
    const int64_t m = ds->rest_csr.nmajor, n = ds->rest_csr.nminor;
    const int64_t npad = (count * l + kDtN - 1) / kDtN * kDtN;
    k_bd_rows_b<<<(int)nblocks(npad * ds->ndp, 256), 256, 0, s>>>(X, coff, o2m, ds->cols.p, n, count, l, ds->ndp,
                                                                   npad, bh, bl);
    SVDB_CHECK_LAUNCH();
    DtLaunch p{ds->D.p, ds->Dl.p, m, ds->ndp, bh, bl};
    p.n_tiles = (int)(npad / kDtN);
    p.l = l;
    p.mode = 2;
    p.out_f32 = true;
    p.out = Y;
    p.bm = m;
    p.bcount = count;
    dt_launch(p, s);
}

template <typename OT>
void dense_batch_cols(const svdb_matrix* a, const float* Y, const int64_t* coff, const int32_t* o2m, int64_t count,
                      int l, OT* Z, float* bh, float* bl, double* part, cudaStream_t s) {
    const DenseSplit* ds = dense_split_for(a);
    if (!ds) throw Error(SVDB_ERR_ARG, "dense split: not available for this matrix");
    const int64_t m = ds->rest_csr.nmajor, n = ds->rest_csr.nminor;
    const int64_t npad = (count * l + kDtN - 1) / kDtN * kDtN;
    dim3 tb(32, 8), tg((unsigned)(ds->mp / 32), (unsigned)((l + 31) / 32), (unsigned)count);
    k_bd_cols_b<<<tg, tb, 0, s>>>(Y, m, l, ds->mp, bh, bl);
    SVDB_CHECK_LAUNCH();
    DtLaunch p{ds->Dt.p, ds->Dtl.p, ds->ndp, ds->mp, bh, bl};
    p.n_tiles = (int)(npad / kDtN);
    p.l = l;
    p.mode = 1;
    p.out = part;
    dt_launch(p, s);
    k_bd_reduce<OT><<<(int)nblocks(count * ds->nd * l, 256), 256, 0, s>>>(part, ds->ndp, ds->cols.p, ds->nd, o2m, coff,
                                                                          n, count, l, Z);
    SVDB_CHECK_LAUNCH();
}

template void dense_batch_cols<float>(const svdb_matrix*, const float*, const int64_t*, const int32_t*, int64_t, int,
                                      float*, float*, float*, double*, cudaStream_t);
template void dense_batch_cols<double>(const svdb_matrix*, const float*, const int64_t*, const int32_t*, int64_t, int,
                                       double*, float*, float*, double*, cudaStream_t);

}  // namespace svdb
