// Gram matrix X^T X of a tall FP64 X (rows x c, c <= 64) on the tensor
// cores (tcgen05.mma kind::tf32, FP32 accumulation in tensor memory), for
// the first pass of CholeskyQR2 under SVDB_MIXED.
//
// X is split per element into its TF32 head h (the top 10 mantissa bits,
// which is what the tensor core reads) and the FP32 remainder l = x - h, and
// G = H^T H + L^T H + H^T L (3xTF32), about FP32 accuracy.  The first pass
// only has to make Q1 = X R1^-1 well conditioned; the FP64 second pass
// restores orthogonality, and a breakdown still falls back to the shifted
// pass.
//
// One CTA of 128 threads takes a chunk of rows (48 KB of shared memory and 128
// TMEM columns, so four CTAs fit an SM).  A stage of 32 rows is
// written to shared memory as the 128 x 32 K-major operand A = [H^T ; L^T]
// (core matrices of 8 rows x 16 bytes, no swizzle: 128 bytes between the
// core matrices along K, 1024 bytes between groups of 8 rows).  Per 8 rows of
// K one thread issues two MMAs (M = 128, N = 64): D += A H and D2 += A L, so
// D = [H^T H ; L^T H] and D2 = [H^T L ; L^T L] in 128 TMEM columns.  The
// commit arrives on the stage's mbarrier; with two stages, the global loads of
// the next 32 rows run while the previous MMAs execute.  At the end each warp
// reads its 32 TMEM lanes (tcgen05.ld 32x32b), warps 2-3 hand D's rows 64..127
// over through shared memory, and warps 0-1 write the CTA's FP64 partial
// D[i][j] + D[64+i][j] + D2[i][j]; the partials are summed in block order by
// k_gram_reduce.  Waits give up after 2 s (g_gram_tc_err).
#include <algorithm>

#include "device_common.cuh"
#include "ops.cuh"
#include "svdb_internal.h"

namespace svdb {

constexpr int kGtK = 32;                 // rows of X per stage (the MMA K dimension)
constexpr int kGtThreads = 128;
constexpr int64_t kGtChunk = 256;        // rows per CTA
constexpr int kGtTileBytes = 128 * kGtK * 4;
constexpr int kGtSmem = 2 * kGtTileBytes + 64 * 64 * 4;  // two stages + the epilogue exchange
// instruction descriptor: F32 accumulator, TF32 A and B, both K-major, N = 64, M = 128
constexpr uint32_t kGtIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
__device__ int g_gram_tc_err;

__device__ __forceinline__ uint32_t gt_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
// shared-memory matrix descriptor: K-major, no swizzle, LBO 128 B, SBO 1024 B
__device__ __forceinline__ uint64_t gt_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
           (1ull << 46);
}
// byte offset of element (row, k) of a stage
__device__ __forceinline__ int gt_off(int row, int k) {
    return (row >> 3) * 1024 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4;
}
__device__ __forceinline__ bool gt_wait(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
    return mbar_wait_bounded(bar, parity, limit_ns);
}

#define SVDB_LD32(v, taddr)                                                                                        \
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, " \
                 "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, " \
                 "[%32];"                                                                                          \
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),  \
                   "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),         \
                   "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),       \
                   "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),       \
                   "=r"(v[29]), "=r"(v[30]), "=r"(v[31])                                                            \
                 : "r"(taddr))

__global__ void __launch_bounds__(kGtThreads) k_gram_tc(const double* __restrict__ X, int64_t rows, int c,
                                                        int64_t chunk, double* __restrict__ part,
                                                        const int* __restrict__ cond, uint64_t limit_ns) {
    if (cond && *cond == 0) return;
    extern __shared__ __align__(1024) unsigned char sm[];
    float* xch = reinterpret_cast<float*>(sm + 2 * kGtTileBytes);  // 64 x 64: rows 64..127 of D
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ int s_failed;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t r0 = blockIdx.x * chunk, r1 = min(rows, r0 + chunk);
    if (gt_smem(sm) & 1023) {  // descriptors address 16-byte units; keep the stages on a 1 KB boundary
        if (tid == 0) atomicOr(&g_gram_tc_err, 2);
        return;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(gt_smem(&s_tmem))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(gt_smem(&s_bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(gt_smem(&s_bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_failed = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    // Two stages: stage s lives in buffer s & 1; before it is rewritten, thread 0
    // waits for the commit of stage s - 2 (the MMAs of stage s - 1 may still run).
    const int nstage = (int)((r1 - r0 + kGtK - 1) / kGtK);
    uint32_t uses[2] = {0, 0};  // commits per buffer so far (its phase parity)
    for (int st = 0; st < nstage; ++st) {
        const int buf = st & 1;
        unsigned char* tile = sm + buf * kGtTileBytes;
        const int64_t kb = r0 + (int64_t)st * kGtK;
        const int nk = (int)min((int64_t)kGtK, r1 - kb);
        double xv[kGtK * 64 / kGtThreads];
#pragma unroll
        for (int u = 0; u < kGtK * 64 / kGtThreads; ++u) {  // global loads first: they overlap the wait below
            const int t = tid + u * kGtThreads, k = t >> 6, col = t & 63;
            xv[u] = (k < nk && col < c) ? X[(kb + k) * c + col] : 0.0;
        }
        if (st >= 2) {
            if (tid == 0 && !gt_wait(gt_smem(&s_bar[buf]), (uses[buf] - 1) & 1, limit_ns)) s_failed = 1;
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (s_failed) break;
        }
#pragma unroll
        for (int u = 0; u < kGtK * 64 / kGtThreads; ++u) {
            const int t = tid + u * kGtThreads, k = t >> 6, col = t & 63;
            const float x = (float)xv[u];
            const float h = __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
            *reinterpret_cast<float*>(tile + gt_off(col, k)) = h;
            *reinterpret_cast<float*>(tile + gt_off(64 + col, k)) = x - h;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            const uint32_t ta = gt_smem(tile);
#pragma unroll
            for (int kk = 0; kk < kGtK / 8; ++kk) {
                const uint64_t a = gt_desc(ta + kk * 256);             // rows 0..127, K 8kk .. 8kk+7
                const uint64_t bl = gt_desc(ta + 8 * 1024 + kk * 256);  // rows 64..127 (the L part)
                const uint32_t acc = (st == 0 && kk == 0) ? 0u : 1u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::"r"(tmem),
                    "l"(a), "l"(a), "r"(kGtIdesc), "r"(acc)
                    : "memory");
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::"r"(tmem + 64),
                    "l"(a), "l"(bl), "r"(kGtIdesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             gt_smem(&s_bar[buf]))
                         : "memory");
        }
        ++uses[buf];
    }
    // the last commit covers every MMA issued before it
    if (tid == 0 && !s_failed && nstage > 0) {
        const int lb = (nstage - 1) & 1;
        if (!gt_wait(gt_smem(&s_bar[lb]), (uses[lb] - 1) & 1, limit_ns)) s_failed = 1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    double* out = part + (int64_t)blockIdx.x * c * c;
    if (!s_failed && nstage > 0) {
        // warp w holds TMEM lanes 32w .. 32w+31: D rows; warps 0-1 also D2 rows 0..63
        const uint32_t lanes = (uint32_t)(warp * 32) << 16;
        const int row = warp * 32 + lane;
        uint32_t d[64];
        SVDB_LD32(d, tmem + lanes + 0);
        SVDB_LD32((d + 32), tmem + lanes + 32);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (warp >= 2) {
#pragma unroll
            for (int j = 0; j < 64; ++j) xch[(row - 64) * 64 + j] = __uint_as_float(d[j]);
        }
        __syncthreads();
        if (warp < 2) {  // tcgen05.ld is warp-collective: every lane of warps 0-1 loads, rows < c write
            uint32_t e[64];
            SVDB_LD32(e, tmem + lanes + 64);
            SVDB_LD32((e + 32), tmem + lanes + 96);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < c) {
#pragma unroll
                for (int j = 0; j < 64; ++j)
                    if (j < c)
                        out[row * c + j] = (double)__uint_as_float(d[j]) + (double)xch[row * 64 + j] +
                                           (double)__uint_as_float(e[j]);
            }
        }
    } else if (!s_failed) {
        for (int t = tid; t < c * c; t += kGtThreads) out[t] = 0.0;
    }
    if (s_failed && tid == 0) {
        atomicOr(&g_gram_tc_err, 1);
        for (int bq = 0; bq < 2; ++bq)  // the MMAs in flight must land before TMEM is freed (2 s at most)
            if (uses[bq]) gt_wait(gt_smem(&s_bar[bq]), (uses[bq] - 1) & 1, 2000000000ull);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(tmem) : "memory");
}

// A CTA sums at most kGtChunk rows in FP32 in tensor memory; the partials
// of the CTAs are added in FP64.
int gram_tc_blocks(int64_t rows) { return (int)std::max<int64_t>(1, (rows + kGtChunk - 1) / kGtChunk); }

// part must hold gram_tc_blocks(rows) * c * c doubles; returns that count
int gram_tc_launch(const double* X, int64_t rows, int c, double* part, int64_t part_cap, const int* cond,
                   cudaStream_t s) {
    if (c > 64 || c < 1) throw Error(SVDB_ERR_UNSUPPORTED, "tensor-core Gram: 1..64 columns");
    const int64_t chunk = kGtChunk;
    const int nblk = gram_tc_blocks(rows);
    if ((int64_t)nblk * c * c > part_cap) throw Error(SVDB_ERR_ARG, "tensor-core Gram: partial buffer too small");
    static bool attr = false;
    if (!attr) {
        SVDB_CUDA(cudaFuncSetAttribute(k_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kGtSmem));
        attr = true;
    }
    k_gram_tc<<<nblk, kGtThreads, kGtSmem, s>>>(X, rows, c, chunk, part, cond, wait_limit_ns());
    SVDB_CHECK_LAUNCH();
    return nblk;
}



void gram_tc_check() {
    int e = 0;
    SVDB_CUDA(cudaMemcpyFromSymbol(&e, g_gram_tc_err, sizeof(int)));
    if (e) {
        const int z = 0;
        SVDB_CUDA(cudaMemcpyToSymbol(g_gram_tc_err, &z, sizeof(int)));
        if (e & 2) throw Error(SVDB_ERR_CUDA, "tensor-core Gram: shared memory not 1 KB aligned; no MMA was issued");
        throw Error(SVDB_ERR_TIMEOUT, "tensor-core Gram: an MMA commit did not arrive within the wait limit");
    }
}

}  // namespace svdb
