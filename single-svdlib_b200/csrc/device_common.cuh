// Device helpers: bounded grid barrier, deterministic block reductions,
// IEEE-exact unfused arithmetic and the ChaCha block function.
#pragma once

#include <cuda/atomic>
#include <cstdint>

namespace svdb {

// Unfused multiply / add, matching the crate's `y += a * x` (Rust never
// contracts a*b+c into an FMA).
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// ------------------------------------------------------------------------
// Grid barrier for cooperative launches.  Every spin is bounded: after
// limit_ns of waiting (the host writes it with the zeroed counters before
// each launch: 2 s unless SVDB_WAIT_LIMIT_NS says otherwise) the block
// records SVDB_ERR_TIMEOUT in err and leaves the barrier; all blocks then
// return at their next check.
// ------------------------------------------------------------------------
struct GridBarrier {
    unsigned int count;
    unsigned int gen;
    int err;
    int pad;
    unsigned long long limit_ns;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for phase `parity` of the shared-memory mbarrier at shared address
// `bar` to complete; gives up after limit_ns of %globaltimer (false).
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, unsigned long long limit_ns) {
    uint32_t ok = 0;
    const unsigned long long t0 = global_ns();
    while (true) {
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(ok)
                     : "r"(bar), "r"(parity)
                     : "memory");
        if (ok) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

// Returns false (uniformly within the block) when the barrier failed.
// `expected` is the number of blocks that must arrive (0: the whole grid).
__device__ __forceinline__ bool grid_sync(GridBarrier* bar, unsigned int expected = 0) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(bar->gen);
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(bar->count);
        cuda::atomic_ref<int, cuda::thread_scope_device> err(bar->err);
        unsigned int g = gen.load(cuda::memory_order_relaxed);
        __threadfence();
        unsigned int arrived = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
        const unsigned long long limit = bar->limit_ns;
        int ok = 1;
        if (arrived == (expected ? expected : gridDim.x) - 1) {
            cnt.store(0u, cuda::memory_order_relaxed);
            gen.fetch_add(1u, cuda::memory_order_release);
        } else {
            unsigned long long t0 = global_ns();
            unsigned int spins = 0;
            while (gen.load(cuda::memory_order_acquire) == g) {
                if (err.load(cuda::memory_order_relaxed) != 0) { ok = 0; break; }
                if ((++spins & 15u) == 0 && global_ns() - t0 > limit) {
                    err.store(8 /* SVDB_ERR_TIMEOUT */, cuda::memory_order_relaxed);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        if (err.load(cuda::memory_order_relaxed) != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// ------------------------------------------------------------------------
// Block reductions in a fixed order (deterministic for a fixed block size).
// `sh` needs blockDim.x / 32 doubles.
// ------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Sum over the block; result valid in every thread.
__device__ __forceinline__ double block_sum(double v, double* sh) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = (threadIdx.x < (unsigned)nw) ? sh[threadIdx.x] : 0.0;
    if (w == 0) t = warp_sum(t);
    if (threadIdx.x == 0) sh[0] = t;
    __syncthreads();
    double r = sh[0];
    __syncthreads();
    return r;
}

// Sum of partials[0..np) in a fixed tree order; valid in every thread.
__device__ __forceinline__ double reduce_partials(const double* partials, int np, double* sh) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) acc += partials[i];
    return block_sum(acc, sh);
}

// ------------------------------------------------------------------------
// ChaCha block (RFC 8439 section 2.3), 64-bit counter / 64-bit stream words.
// ------------------------------------------------------------------------
__device__ __forceinline__ uint32_t rotl32(uint32_t v, int c) { return __funnelshift_l(v, v, c); }

__device__ __forceinline__ void chacha_block_dev(const uint32_t key[8], uint64_t counter, int rounds,
                                                 uint32_t out[16]) {
    uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                      key[4],      key[5],      key[6],      key[7],      (uint32_t)counter,
                      (uint32_t)(counter >> 32), 0u, 0u};
    uint32_t x[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = s[i];
#define SVDB_QR(a, b, c, d)                               \
    x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 16);         \
    x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 12);         \
    x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 8);          \
    x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 7);
    for (int r = 0; r < rounds; r += 2) {
        SVDB_QR(0, 4, 8, 12) SVDB_QR(1, 5, 9, 13) SVDB_QR(2, 6, 10, 14) SVDB_QR(3, 7, 11, 15)
        SVDB_QR(0, 5, 10, 15) SVDB_QR(1, 6, 11, 12) SVDB_QR(2, 7, 8, 13) SVDB_QR(3, 4, 9, 14)
    }
#undef SVDB_QR
#pragma unroll
    for (int i = 0; i < 16; ++i) out[i] = x[i] + s[i];
}

// rand's UniformFloat<f64>::sample_single(-1.0, 1.0) on one u64 draw; the
// result (2k - 2^52) / 2^52 is exact, so no rounding mode matters.
__device__ __forceinline__ double uniform_pm1_dev(uint64_t u) {
    double v12 = __longlong_as_double((long long)((u >> 12) | 0x3FF0000000000000ull));
    double v01 = v12 - 1.0;
    return __dadd_rn(__dmul_rn(v01, 2.0), -1.0);
}

}  // namespace svdb
