// randomized_svd (src/randomized/mod.rs:24-199) on the device.
//
//   Y = A Omega; q x [Z = A^T Y, normalise Z; Y = A Z, normalise Y];
//   Q = qr(Y).q; B^T = A^T Q; SVD(B); U = Q U_B.
//
// nalgebra's Householder qr().q() (third-party) is replaced by CholeskyQR2:
// the Gram X^T X in FP64, a one-block Cholesky, X R^-1, twice; if a Cholesky
// pivot breaks down the pass is redone with a shift (shifted CholeskyQR3).
// The column spaces are those of Householder QR; column signs may differ.
// nalgebra's svd(B) is replaced by: QR of B^T = Q_b R (CholeskyQR2), then a
// one-sided Jacobi SVD of the small R in one block, so that
// B = V_R S (Q_b U_R)^T, singular values in descending order.
//
// SVDB_MIXED runs the sparse products on FP32 matrix values and an FP32 copy
// of the dense operand (half the gathered bytes) with FP64 sums; the Gram
// products, Cholesky, both CholeskyQR passes and the small SVD stay FP64.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "dense_small.cuh"
#include "device_common.cuh"
#include "ops.cuh"
#include "svdb_internal.h"

namespace svdb {

static bool getenv_is(const char* name, const char* value) {
    const char* e = getenv(name);
    return e && std::strcmp(e, value) == 0;
}

static int nb(int64_t work, int threads, int per_sm = 16) {
    int64_t b = (work + threads - 1) / threads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)device_props().sms * per_sm));
}

// --------------------------------------------------------------- Omega ----
template <typename T>
__global__ void k_omega(uint64_t seed, int64_t total, T* __restrict__ out) {
    const uint64_t key = omega_key(seed);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (T)omega_value(key, i);
}

// ---------------------------------------------------------------- Gram ----
// G (c x c) = X^T X for X (rows x c) row-major.  Blocks take row chunks
// (staged through shared memory); a 16 x 16 thread grid holds an NC x NC
// register tile of G per thread (entries (ty + 16 i, tx + 16 j)).  G[a][b]
// and G[b][a] see the same products in the same order, so G is exactly
// symmetric.  Block partials are reduced in block order.  Every kernel of a
// CholeskyQR pass takes `cond`: when it points to 0 the kernel returns at
// once (the conditional third pass of shifted CholeskyQR).
constexpr int kGramRows = 32;
template <typename T, int NC>
__global__ void __launch_bounds__(256) k_gram_part(const T* __restrict__ X, int64_t rows, int c, int64_t chunk,
                                                   double* __restrict__ part, const int* __restrict__ cond) {
    if (cond && *cond == 0) return;
    extern __shared__ double xs[];  // kGramRows x c
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int64_t r0 = blockIdx.x * chunk, r1 = std::min<int64_t>(rows, r0 + chunk);
    double acc[NC][NC];
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int j = 0; j < NC; ++j) acc[i][j] = 0.0;
    for (int64_t rb = r0; rb < r1; rb += kGramRows) {
        const int nr = (int)std::min<int64_t>(kGramRows, r1 - rb);
        __syncthreads();
        for (int t = threadIdx.x; t < nr * c; t += blockDim.x) xs[t] = (double)X[(rb + t / c) * c + t % c];
        __syncthreads();
        for (int r = 0; r < nr; ++r) {
            double xa[NC], xb[NC];
#pragma unroll
            for (int i = 0; i < NC; ++i) {
                const int a = ty + 16 * i, b = tx + 16 * i;
                xa[i] = a < c ? xs[r * c + a] : 0.0;
                xb[i] = b < c ? xs[r * c + b] : 0.0;
            }
#pragma unroll
            for (int i = 0; i < NC; ++i)
#pragma unroll
                for (int j = 0; j < NC; ++j) acc[i][j] = fma(xa[i], xb[j], acc[i][j]);
        }
    }
    double* out = part + (int64_t)blockIdx.x * c * c;
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int j = 0; j < NC; ++j) {
            const int a = ty + 16 * i, b = tx + 16 * j;
            if (a < c && b < c) out[a * c + b] = acc[i][j];
        }
}
// G[p] = sum over blocks of part[b][p].  A block covers 32 elements; its 8
// warps sum fixed slices of the blocks, and the slices are added in slice
// order, so G[a][b] and G[b][a] still see the same operations (G symmetric).
constexpr int kRedSlices = 8;
__global__ void __launch_bounds__(256) k_gram_reduce(const double* __restrict__ part, int nblocks, int c,
                                                     double* __restrict__ G, const int* __restrict__ cond) {
    if (cond && *cond == 0) return;
    __shared__ double sh[kRedSlices][32];
    const int cc = c * c;
    const int e = blockIdx.x * 32 + (threadIdx.x & 31);
    const int sl = threadIdx.x >> 5;
    double acc = 0.0;
    if (e < cc) {
        const int per = (nblocks + kRedSlices - 1) / kRedSlices;
        const int b0 = sl * per, b1 = min(nblocks, b0 + per);
        for (int bq = b0; bq < b1; ++bq) acc += part[(int64_t)bq * cc + e];
    }
    sh[sl][threadIdx.x & 31] = acc;
    __syncthreads();
    if (sl == 0 && e < cc) {
        double t = 0.0;
#pragma unroll
        for (int k = 0; k < kRedSlices; ++k) t += sh[k][threadIdx.x];
        G[e] = t;
    }
}

// ------------------------------------------------------ small dense ops ----
__global__ void __launch_bounds__(1024) k_chol_inv(const double* __restrict__ G, int c, double shift_scale,
                                                   double* __restrict__ R, double* __restrict__ Ri,
                                                   int* __restrict__ flags, int* __restrict__ shifted,
                                                   const int* __restrict__ cond, int ri_in_smem) {
    if (cond && *cond == 0) return;
    extern __shared__ double sm[];  // R work (c*c) | R^-1 (c*c) when ri_in_smem
    chol_inv_body(G, c, shift_scale, R, Ri, flags, shifted, ri_in_smem, sm);
}

// C (c x c) = A (c x c) B (c x c), one block
__global__ void k_small_gemm(const double* __restrict__ A, const double* __restrict__ B, int c,
                             double* __restrict__ C, const int* __restrict__ cond) {
    if (cond && *cond == 0) return;
    for (int t = threadIdx.x; t < c * c; t += blockDim.x) {
        const int i = t / c, j = t % c;
        double s = 0.0;
        for (int k = 0; k < c; ++k) s = fma(A[i * c + k], B[k * c + j], s);
        C[t] = s;
    }
}

// Out (rows x cout) = X (rows x c) S (c x lds, first cout columns).  S and
// 64-row tiles of X are staged in shared memory; a 16 x 16 thread grid gives
// every thread a 4 x NJ register tile (rows ty + 16 i, columns tx + 16 j).
// With nbuf = 2 the next tile of X is copied (cp.async) while the current one
// is multiplied; nbuf = 1 when two tiles do not fit.
constexpr int kRmRows = 64;
__device__ __forceinline__ void rm_cp_async(void* dst, const void* src, int bytes) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
template <typename TI, typename TO, int NJ>
__global__ void __launch_bounds__(256) k_right_mul(const TI* __restrict__ X, int64_t rows, int c,
                                                   const double* __restrict__ S, int lds, int cout,
                                                   TO* __restrict__ Out, const int* __restrict__ cond, int nbuf) {
    if (cond && *cond == 0) return;
    extern __shared__ double sm[];  // S: c*cout doubles | nbuf X tiles of kRmRows*c TI
    double* ss = sm;
    TI* xbuf = reinterpret_cast<TI*>(sm + c * cout);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    for (int t = threadIdx.x; t < c * cout; t += blockDim.x) ss[t] = S[(t / cout) * lds + t % cout];
    auto load = [&](int64_t r0, int b) {  // tile at row r0 into buffer b (asynchronous)
        const int nr = (int)std::min<int64_t>(kRmRows, rows - r0);
        TI* xs = xbuf + (size_t)b * kRmRows * c;
        for (int t = threadIdx.x; t < nr * c; t += blockDim.x) rm_cp_async(xs + t, X + r0 * c + t, (int)sizeof(TI));
    };
    const int64_t step = (int64_t)gridDim.x * kRmRows;
    int64_t r0 = (int64_t)blockIdx.x * kRmRows;
    if (r0 < rows) load(r0, 0);
    asm volatile("cp.async.commit_group;" ::: "memory");
    for (int it = 0; r0 < rows; r0 += step, ++it) {
        const int b = nbuf == 2 ? (it & 1) : 0;
        if (nbuf == 2 && r0 + step < rows) load(r0 + step, b ^ 1);
        asm volatile("cp.async.commit_group;" ::: "memory");  // possibly empty: one group per iteration
        asm volatile("cp.async.wait_group 1;" ::: "memory");  // this tile's group has landed
        __syncthreads();
        const TI* xs = xbuf + (size_t)b * kRmRows * c;
        const int nr = (int)std::min<int64_t>(kRmRows, rows - r0);
        double acc[4][NJ];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < NJ; ++j) acc[i][j] = 0.0;
        for (int k = 0; k < c; ++k) {
            double xv[4], sv[NJ];
#pragma unroll
            for (int i = 0; i < 4; ++i) xv[i] = (ty + 16 * i < nr) ? (double)xs[(ty + 16 * i) * c + k] : 0.0;
#pragma unroll
            for (int j = 0; j < NJ; ++j) sv[j] = (tx + 16 * j < cout) ? ss[k * cout + tx + 16 * j] : 0.0;
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < NJ; ++j) acc[i][j] = fma(xv[i], sv[j], acc[i][j]);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int rr = ty + 16 * i;
            if (rr >= nr) continue;
#pragma unroll
            for (int j = 0; j < NJ; ++j) {
                const int col = tx + 16 * j;
                if (col < cout) Out[(r0 + rr) * cout + col] = (TO)acc[i][j];
            }
        }
        __syncthreads();  // this buffer is read; it may be refilled
        if (nbuf == 1 && r0 + step < rows) {
            load(r0 + step, 0);
            asm volatile("cp.async.commit_group;" ::: "memory");  // older than the next iteration's group
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

__global__ void k_copy_cond(const double* __restrict__ src, double* __restrict__ dst, int64_t n,
                            const int* __restrict__ cond) {
    if (cond && *cond == 0) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

template <typename T>
__global__ void k_colnorm(T* __restrict__ X, int64_t rows, int c) {
    __shared__ double sh[32];
    __shared__ double scale;
    const int j = blockIdx.x;
    double acc = 0.0;
    for (int64_t r = threadIdx.x; r < rows; r += blockDim.x) {
        const double v = (double)X[r * c + j];
        acc = fma(v, v, acc);
    }
    const double nrm = sqrt(block_sum(acc, sh));
    if (threadIdx.x == 0) scale = nrm > 1e-10 ? 1.0 / nrm : 1.0;
    __syncthreads();
    if (nrm > 1e-10)
        for (int64_t r = threadIdx.x; r < rows; r += blockDim.x) X[r * c + j] = (T)((double)X[r * c + j] * scale);
}

// One-sided Jacobi SVD of the c x c R in one block (jacobi_svd_body).
__global__ void __launch_bounds__(1024) k_jacobi_svd(const double* __restrict__ R, int c, double* __restrict__ U,
                                                     double* __restrict__ V, double* __restrict__ sig,
                                                     int* __restrict__ status) {
    extern __shared__ double sm[];
    jacobi_svd_body(R, c, U, V, sig, status, sm);
}

__global__ void k_to_float(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// out (rows x ldx) = in (rows x c), rounded to FP32; columns c .. ldx-1 are not written
__global__ void k_to_float_ld(const double* __restrict__ in, float* __restrict__ out, int64_t rows, int c,
                              int64_t ldx) {
    const int64_t n = rows * c;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / c;
        out[r * ldx + (i - r * c)] = (float)in[i];
    }
}
// copy the first `cout` columns of X (rows x c) into Out (rows x cout)
__global__ void k_take_cols(const double* __restrict__ X, int64_t rows, int c, int cout, double* __restrict__ Out) {
    const int64_t total = rows * cout;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x)
        Out[t] = X[(t / cout) * c + t % cout];
}

// ------------------------------------------------------------ centring ----
// Products of the centred matrix A - 1 mu^T, mu the column means
// (compute_column_means, masked.rs:240-263), as A X - 1 (mu^T X) and
// A^T Y - mu (1^T Y).  mu comes from the column-major copy, one warp per
// column with a fixed lane order.
__global__ void k_major_means(const int64_t* __restrict__ ptr, const double* __restrict__ val, int64_t nmajor,
                              double inv, double* __restrict__ mu) {
    const int lane = threadIdx.x & 31;
    const int64_t w0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t j = w0; j < nmajor; j += nw) {
        double acc = 0.0;
        for (int64_t k = ptr[j] + lane; k < ptr[j + 1]; k += 32) acc += val[k];
#pragma unroll
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) mu[j] = acc * inv;
    }
}
// part[b][j] = sum over the rows of chunk b of w[r] X[r][j] (w = 1 when null),
// for the c <= 128 columns of X starting at X (row stride ld).  32 x 8
// threads: x walks the columns, y the rows; the y partials are added in y order.
constexpr int kCsCols = 128;
__global__ void __launch_bounds__(256) k_wcolsum_part(const double* __restrict__ X, int64_t rows, int64_t ld, int c,
                                                      const double* __restrict__ w, int64_t chunk,
                                                      double* __restrict__ part) {
    __shared__ double sh[8][kCsCols];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int64_t r0 = blockIdx.x * chunk, r1 = std::min<int64_t>(rows, r0 + chunk);
    double acc[kCsCols / 32];
#pragma unroll
    for (int q = 0; q < kCsCols / 32; ++q) acc[q] = 0.0;
    for (int64_t r = r0 + ty; r < r1; r += 8) {
        const double wr = w ? w[r] : 1.0;
#pragma unroll
        for (int q = 0; q < kCsCols / 32; ++q) {
            const int j = tx + 32 * q;
            if (j < c) acc[q] = fma(wr, X[r * ld + j], acc[q]);
        }
    }
#pragma unroll
    for (int q = 0; q < kCsCols / 32; ++q) sh[ty][tx + 32 * q] = acc[q];
    __syncthreads();
    for (int j = threadIdx.x; j < c; j += blockDim.x) {
        double t = 0.0;
#pragma unroll
        for (int y = 0; y < 8; ++y) t += sh[y][j];
        part[(int64_t)blockIdx.x * c + j] = t;
    }
}
// t[j] = sum of part[b][j] in block order
__global__ void k_colsum_total(const double* __restrict__ part, int nblocks, int c, double* __restrict__ t) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < c; j += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int b = 0; b < nblocks; ++b) acc += part[(int64_t)b * c + j];
        t[j] = acc;
    }
}
// Y[r][j] -= a[r] t[j] (a = 1 when null), Y rows x c
__global__ void k_rank1_sub(double* __restrict__ Y, int64_t rows, int c, const double* __restrict__ a,
                            const double* __restrict__ t) {
    const int64_t total = rows * c;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / c;
        Y[i] -= (a ? a[r] : 1.0) * t[i - r * c];
    }
}

void column_means_dev(const DevCompressed& csc, int64_t rows, double* mu, cudaStream_t s) {
    if (csc.nmajor == 0) return;
    k_major_means<<<nb(csc.nmajor * 32, 256), 256, 0, s>>>(csc.ptr.p, csc.val.p, csc.nmajor,
                                                          rows > 0 ? 1.0 / (double)rows : 0.0, mu);
    SVDB_CHECK_LAUNCH();
}

void center_product(const double* X, int64_t xrows, int c, const double* mu, double* Out, int64_t orows,
                    bool out_is_rows, cudaStream_t s) {
    if (c <= 0 || orows <= 0) return;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((xrows + 255) / 256, (int64_t)device_props().sms * 4));
    const int64_t chunk = (xrows + blocks - 1) / blocks;
    DevBuf<double> part((size_t)blocks * kCsCols, s), tot(c, s);
    for (int j0 = 0; j0 < c; j0 += kCsCols) {
        const int w = std::min(kCsCols, c - j0);
        k_wcolsum_part<<<blocks, 256, 0, s>>>(X + j0, xrows, c, w, out_is_rows ? mu : nullptr, chunk, part.p);
        SVDB_CHECK_LAUNCH();
        k_colsum_total<<<1, 128, 0, s>>>(part.p, blocks, w, tot.p + j0);
        SVDB_CHECK_LAUNCH();
    }
    k_rank1_sub<<<nb(orows * c, 256), 256, 0, s>>>(Out, orows, c, out_is_rows ? nullptr : mu, tot.p);
    SVDB_CHECK_LAUNCH();
}

// ------------------------------------------------------ host helpers ----
struct RandCtx {
    cudaStream_t s;
    bool tensor_gram = false;  // first CholeskyQR pass on the tensor cores (SVDB_MIXED)
    int cmax = 0;
    DevBuf<double> part, G, R1, R2, R3, Ri, Rtmp, T;
    DevBuf<int> flags, shifted;
    int64_t part_cap = 0;
};

// G = X^T X on the tensor cores (3xTF32, FP32 accumulation; gram_tc.cu), the
// CTA partials summed in FP64 in block order
static void gram_tensor(RandCtx& cx, const double* X, int64_t rows, int c, double* G, const int* cond) {
    const int nblk = gram_tc_blocks(rows);
    if ((int64_t)nblk * c * c > cx.part_cap) {
        cx.part_cap = (int64_t)nblk * c * c;
        cx.part.alloc(cx.part_cap, cx.s);
    }
    gram_tc_launch(X, rows, c, cx.part.p, cx.part_cap, cond, cx.s);
    k_gram_reduce<<<(c * c + 31) / 32, 32 * kRedSlices, 0, cx.s>>>(cx.part.p, nblk, c, G, cond);
    SVDB_CHECK_LAUNCH();
}

static void gram(RandCtx& cx, const double* X, int64_t rows, int c, double* G, const int* cond) {
    if (c > 128) throw Error(SVDB_ERR_UNSUPPORTED, "randomized_svd: more than 128 sample columns");
    const int sms = device_props().sms;
    int64_t chunk = std::max<int64_t>(kGramRows * 4, (rows + sms * 2 - 1) / (sms * 2));
    int nblk = (int)std::max<int64_t>(1, (rows + chunk - 1) / chunk);
    if ((int64_t)nblk * c * c > cx.part_cap) {
        cx.part_cap = (int64_t)nblk * c * c;
        cx.part.alloc(cx.part_cap, cx.s);
    }
    const size_t smem = kGramRows * c * sizeof(double);
    const int nc = (c + 15) / 16;
    switch (nc) {
        case 1: k_gram_part<double, 1><<<nblk, 256, smem, cx.s>>>(X, rows, c, chunk, cx.part.p, cond); break;
        case 2: k_gram_part<double, 2><<<nblk, 256, smem, cx.s>>>(X, rows, c, chunk, cx.part.p, cond); break;
        case 3: k_gram_part<double, 3><<<nblk, 256, smem, cx.s>>>(X, rows, c, chunk, cx.part.p, cond); break;
        case 4: k_gram_part<double, 4><<<nblk, 256, smem, cx.s>>>(X, rows, c, chunk, cx.part.p, cond); break;
        case 5: k_gram_part<double, 5><<<nblk, 256, smem, cx.s>>>(X, rows, c, chunk, cx.part.p, cond); break;
        case 6: k_gram_part<double, 6><<<nblk, 256, smem, cx.s>>>(X, rows, c, chunk, cx.part.p, cond); break;
        case 7: k_gram_part<double, 7><<<nblk, 256, smem, cx.s>>>(X, rows, c, chunk, cx.part.p, cond); break;
        default: k_gram_part<double, 8><<<nblk, 256, smem, cx.s>>>(X, rows, c, chunk, cx.part.p, cond); break;
    }
    k_gram_reduce<<<(c * c + 31) / 32, 32 * kRedSlices, 0, cx.s>>>(cx.part.p, nblk, c, G, cond);
    SVDB_CHECK_LAUNCH_N(2);
}

static void right_mul(const double* X, int64_t rows, int c, const double* S, int lds, int cout, double* Out,
                      cudaStream_t s, const int* cond = nullptr) {
    const size_t s_bytes = (size_t)c * cout * sizeof(double), tile = (size_t)kRmRows * c * sizeof(double);
    if (s_bytes + tile > 220 * 1024 || cout > 128)
        throw Error(SVDB_ERR_UNSUPPORTED, "dense factor wider than the shared-memory tile");
    // one X tile buffer: at c = 60 that is 59 KB of shared memory and three
    // blocks per SM instead of two with a second buffer, 908 against 956 us
    // of k_right_mul per randomized solve (100k x 30k)
    const int nbuf = 1;
    const size_t smem = s_bytes + nbuf * tile;
    const int64_t tiles = (rows + kRmRows - 1) / kRmRows;
    auto go = [&](auto kern) {
        if (smem > 48 * 1024)
            SVDB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;  // one wave of resident blocks, each looping over tiles
        SVDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem));
        const int blocks = (int)std::max<int64_t>(
            1, std::min<int64_t>(tiles, (int64_t)device_props().sms * std::max(per_sm, 1)));
        kern<<<blocks, 256, smem, s>>>(X, rows, c, S, lds, cout, Out, cond, nbuf);
    };
    if (cout <= 16) go(k_right_mul<double, double, 1>);
    else if (cout <= 32) go(k_right_mul<double, double, 2>);
    else if (cout <= 64) go(k_right_mul<double, double, 4>);
    else go(k_right_mul<double, double, 8>);
    SVDB_CHECK_LAUNCH();
}

static void chol_inv(RandCtx& cx, const double* G, int c, int64_t rows, double* R, const int* cond) {
    const bool two = 2 * (size_t)c * c * sizeof(double) <= 200 * 1024;
    const size_t smem = (two ? 2 : 1) * (size_t)c * c * sizeof(double);
    // chol_inv_body also holds about 1 KB of static shared memory
    if (smem > 40 * 1024)
        SVDB_CUDA(cudaFuncSetAttribute(k_chol_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // shifted CholeskyQR: shift = 11 (rows c + c (c + 1)) u ||X||_F^2, ||X||_F^2 = trace(G)
    const double shift_scale = 11.0 * ((double)rows * c + (double)c * (c + 1)) * 1.1102230246251565e-16;
    k_chol_inv<<<1, 1024, smem, cx.s>>>(G, c, shift_scale, R, cx.Ri.p, cx.flags.p, cx.shifted.p, cond, two);
    SVDB_CHECK_LAUNCH();
}

// Thin Q of X (rows x c, rows >= c) in place; Rout (c x c) = R_last ... R_first
// when requested.  CholeskyQR2; a pass whose Cholesky broke down is redone with
// a shift and a third pass follows.  Nothing here waits for the device: the
// third pass's kernels read the device flag and return when it is 0.
static void cholesky_qr(RandCtx& cx, double* X, int64_t rows, int c, double* Rout) {
    cudaStream_t s = cx.s;
    if ((int64_t)cx.T.n < rows * c) cx.T.alloc(rows * c, s);
    double* T = cx.T.p;
    SVDB_CUDA(cudaMemsetAsync(cx.shifted.p, 0, sizeof(int), s));
    // pass 1: X -> T (its Gram on the tensor cores under SVDB_MIXED: only its R1
    // has to be good enough for pass 2, which is FP64)
    if (cx.tensor_gram && c <= 64) gram_tensor(cx, X, rows, c, cx.G.p, nullptr);
    else gram(cx, X, rows, c, cx.G.p, nullptr);
    chol_inv(cx, cx.G.p, c, rows, cx.R1.p, nullptr);
    right_mul(X, rows, c, cx.Ri.p, c, c, T, s);
    // pass 2: T -> X
    gram(cx, T, rows, c, cx.G.p, nullptr);
    chol_inv(cx, cx.G.p, c, rows, cx.R2.p, nullptr);
    right_mul(T, rows, c, cx.Ri.p, c, c, X, s);
    // pass 3 only after a shifted pass: X -> T -> X
    const int* cond = cx.shifted.p;
    gram(cx, X, rows, c, cx.G.p, cond);
    chol_inv(cx, cx.G.p, c, rows, cx.R3.p, cond);
    right_mul(X, rows, c, cx.Ri.p, c, c, T, s, cond);
    k_copy_cond<<<nb(rows * c, 256), 256, 0, s>>>(T, X, rows * c, cond);
    SVDB_CHECK_LAUNCH();
    if (Rout) {
        k_small_gemm<<<1, 256, 0, s>>>(cx.R2.p, cx.R1.p, c, Rout, nullptr);
        k_small_gemm<<<1, 256, 0, s>>>(cx.R3.p, Rout, c, cx.Rtmp.p, cond);
        k_copy_cond<<<1, 256, 0, s>>>(cx.Rtmp.p, Rout, (int64_t)c * c, cond);
        SVDB_CHECK_LAUNCH_N(3);
    }
}

// qr(X).q() for X (rows x c): returns the column count of Q; X is replaced by
// Q (rows x k, k = min(rows, c)) stored with row stride k.
static int thin_q(RandCtx& cx, DevBuf<double>& X, int64_t rows, int c) {
    if (rows >= c) {
        cholesky_qr(cx, X.p, rows, c, nullptr);
        return c;
    }
    // wide: Q spans R^rows; take the leading rows x rows block's Q
    const int k = (int)rows;
    DevBuf<double> Xk((int64_t)rows * k, cx.s);
    k_take_cols<<<nb(rows * k, 256), 256, 0, cx.s>>>(X.p, rows, c, k, Xk.p);
    SVDB_CHECK_LAUNCH();
    cholesky_qr(cx, Xk.p, rows, k, nullptr);
    X = std::move(Xk);
    return k;
}

static double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// svdb_gram_device: G (c x c) = X^T X for a device X (rows x c, FP64)
void gram_device(const double* X, int64_t rows, int c, double* G, int precision, cudaStream_t s) {
    if (c < 1 || c > 128) throw Error(SVDB_ERR_UNSUPPORTED, "gram: 1..128 columns");
    RandCtx cx;
    cx.s = s;
    if (precision == SVDB_MIXED) {
        if (c > 64) throw Error(SVDB_ERR_UNSUPPORTED, "gram: the tensor-core form takes at most 64 columns");
        gram_tensor(cx, X, rows, c, G, nullptr);
    } else {
        gram(cx, X, rows, c, G, nullptr);
    }
    SVDB_CUDA(cudaStreamSynchronize(s));
    gram_tc_check();
}

void randomized(const svdb_matrix* A, uint64_t target_rank, uint64_t n_oversamples, uint64_t n_power_iters,
                int normalizer, int mean_center, int has_seed, uint64_t seed, int verbose, const svdb_options& o,
                svdb_rec* rec, bool f32) {
    cudaStream_t s = o.stream ? (cudaStream_t)o.stream : A->stream;
    // f32: the crate's T = f32 run: Omega's f64 draws rounded to f32
    // (T::from_f64, randomized/mod.rs:299-313) and FP32 operands
    const bool mixed = f32 || o.precision == SVDB_MIXED;
    const int64_t m = A->nrows, n = A->ncols;
    const int64_t rank = std::min<int64_t>((int64_t)target_rank, std::min(m, n));
    int l = (int)(rank + (int64_t)n_oversamples);
    if (l <= 0) throw Error(SVDB_ERR_SHAPE, "randomized_svd: zero sample columns");
    const DevCompressed& Acsr = csr_of(A);
    const DevCompressed& Acsc = csc_of(A);
    if (mixed) ensure_fp32(A);
    auto t0 = std::chrono::steady_clock::now();
    cudaEvent_t e0, e1;
    SVDB_CUDA(cudaEventCreate(&e0));
    SVDB_CUDA(cudaEventCreate(&e1));
    SVDB_CUDA(cudaEventRecord(e0, s));
    float spmm_ms = 0.f;

    RandCtx cx;
    cx.s = s;
    cx.tensor_gram = mixed && !getenv_is("SVDB_GRAM", "fp64");
    const int cmax = l;
    for (DevBuf<double>* b : {&cx.G, &cx.R1, &cx.R2, &cx.R3, &cx.Ri, &cx.Rtmp}) b->alloc((size_t)cmax * cmax, s);
    cx.flags.alloc(1, s);
    cx.shifted.alloc(1, s);
    DevBuf<int> jac_status(1, s);
    SVDB_CUDA(cudaMemsetAsync(cx.flags.p, 0, sizeof(int), s));
    SVDB_CUDA(cudaMemsetAsync(jac_status.p, 0, sizeof(int), s));

    // Omega (n x l)
    DevBuf<double> Om(std::max<int64_t>(n * l, 1), s);
    if (o.omega) {
        SVDB_CUDA(cudaMemcpyAsync(Om.p, o.omega, n * l * 8, cudaMemcpyHostToDevice, s));
    } else {
        k_omega<double><<<nb(n * l, 256), 256, 0, s>>>(has_seed ? seed : 0, n * l, Om.p);
        SVDB_CHECK_LAUNCH();
    }
    if (f32) round_f32(Om.p, n * l, s);

    // Sparse products: FP64 operands, or under SVDB_MIXED FP32 values and an
    // FP32 copy of the dense operand (half the gathered bytes), FP64 sums and output.
    DevBuf<float> f_in;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> spmm_events;  // read once, at the end
    // SVDB_MIXED with dense columns: their share of each product on the tensor cores
    const bool split = mixed && !f32 && dense_split_usable(A, l);
    auto spmm = [&](const DevCompressed& M, const double* X, int c, double* Y) {
        cudaEvent_t a, b;
        SVDB_CUDA(cudaEventCreate(&a));
        SVDB_CUDA(cudaEventCreate(&b));
        SVDB_CUDA(cudaEventRecord(a, s));
        if (!mixed) {
            spmm_dev<double, double>(M, false, X, c, Y, s);
        } else {
            const int64_t ldp = ((int64_t)c + 31) / 32 * 32;  // rows on whole 128-byte lines
            if (!split && spmm_f32_strided_ok(M, c, ldp)) {
                if ((int64_t)f_in.n < M.nminor * ldp) f_in.alloc(M.nminor * ldp, s);
                k_to_float_ld<<<nb(M.nminor * c, 256), 256, 0, s>>>(X, f_in.p, M.nminor, c, ldp);
                SVDB_CHECK_LAUNCH();
                spmm_f32_strided(M, f_in.p, c, ldp, Y, s);
            } else {
                if ((int64_t)f_in.n < M.nminor * c) f_in.alloc(M.nminor * c, s);
                k_to_float<<<nb(M.nminor * c, 256), 256, 0, s>>>(X, f_in.p, M.nminor * c);
                SVDB_CHECK_LAUNCH();
                if (split) dense_split_spmm<double, double>(A, &M == &Acsc, X, f_in.p, c, Y, s);
                else spmm_dev<float, double>(M, true, f_in.p, c, Y, s);
            }
        }
        SVDB_CUDA(cudaEventRecord(b, s));
        spmm_events.emplace_back(a, b);
    };
    auto normalize = [&](DevBuf<double>& X, int64_t rows, int c) -> int {
        if (normalizer == SVDB_NORM_QR) return thin_q(cx, X, rows, c);
        if (normalizer == SVDB_NORM_LU) {
            k_colnorm<double><<<c, 256, 0, s>>>(X.p, rows, c);
            SVDB_CHECK_LAUNCH();
        }
        return c;
    };

    // mean_center: the products of A - 1 mu^T
    DevBuf<double> mu;
    if (mean_center) {
        mu.alloc(std::max<int64_t>(n, 1), s);
        column_means_dev(Acsc, m, mu.p, s);
    }
    auto center = [&](const double* X, int64_t xrows, int c, double* Out, int64_t orows, bool out_is_rows) {
        if (mean_center) center_product(X, xrows, c, mu.p, Out, orows, out_is_rows, s);
    };

    if (verbose) printf("SVD | Randomized | Multiplying m with omega matrix....\n");
    DevBuf<double> Y(std::max<int64_t>(m * l, 1), s);
    spmm(Acsr, Om.p, l, Y.p);
    center(Om.p, n, l, Y.p, m, true);
    int c = l;
    if (verbose) printf("SVD | Randomized | Multiplication done, took: %.3f ms of total running time\n", ms_since(t0));
    if (verbose) printf("SVD | Randomized | Starting power iterations....\n");
    for (uint64_t it = 0; it < n_power_iters; ++it) {
        if (verbose)
            printf("SVD | Randomized | Running power-iteration: %llu, current time: %.3f ms\n",
                   (unsigned long long)it, ms_since(t0));
        DevBuf<double> Z(std::max<int64_t>(n * c, 1), s);
        spmm(Acsc, Y.p, c, Z.p);
        center(Y.p, m, c, Z.p, n, false);
        c = normalize(Z, n, c);
        DevBuf<double> Y2(std::max<int64_t>(m * c, 1), s);
        spmm(Acsr, Z.p, c, Y2.p);
        center(Z.p, n, c, Y2.p, m, true);
        Y = std::move(Y2);
        c = normalize(Y, m, c);
        if (verbose)
            printf("SVD | Randomized | Power Iteration Normalization Backward-Step %.3f ms\n", ms_since(t0));
    }
    if (verbose) printf("SVD | Randomized | Running QR-Normalization after Power-Iterations %.3f ms\n", ms_since(t0));
    c = thin_q(cx, Y, m, c);  // Q = qr(y).q()
    // B^T = A^T Q (n x c)
    DevBuf<double> Bt(std::max<int64_t>(n * c, 1), s);
    spmm(Acsc, Y.p, c, Bt.p);
    center(Y.p, m, c, Bt.p, n, false);
    if (verbose) printf("SVD | Randomized | Transposed Matrix Multiplication %.3f ms\n", ms_since(t0));

    // SVD(B), B = Bt^T (c x n).  r = min(c, n).
    const int r = (int)std::min<int64_t>(c, n);
    DevBuf<double> UB((size_t)c * r, s), sig(r, s), VtB((size_t)r * n, s);
    {
        DevBuf<double> Ur((size_t)r * r, s), Vr((size_t)r * r, s), R((size_t)r * r, s);
        const size_t smem = ((size_t)r * (r + 1) + (size_t)(r + 1) * (r + 1) + (r + 1)) * sizeof(double);
        if (smem > 220 * 1024) throw Error(SVDB_ERR_UNSUPPORTED, "randomized_svd: sample width above the Jacobi tile");
        SVDB_CUDA(cudaFuncSetAttribute(k_jacobi_svd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        if (n >= c) {
            // B^T = Q_b R;  R = U_J S V_J^T  ->  B = V_J S (Q_b U_J)^T.  The one-sided
            // Jacobi runs on R^T = V_J S U_J^T, whose columns (the rows of the QR
            // factor) are graded, which takes fewer sweeps than R itself.
            cholesky_qr(cx, Bt.p, n, c, R.p);
            DevBuf<double> Rt((size_t)r * r, s);
            transpose_dense<double>(R.p, Rt.p, r, r, s);
            k_jacobi_svd<<<1, jacobi_threads(r, 1024), smem, s>>>(Rt.p, r, Vr.p, Ur.p, sig.p, jac_status.p);
            // U_B = V_J (c x r); V_B = Q_b U_J (n x r)
            SVDB_CUDA(cudaMemcpyAsync(UB.p, Vr.p, (size_t)r * r * 8, cudaMemcpyDeviceToDevice, s));
            DevBuf<double> VB((size_t)n * r, s);
            right_mul(Bt.p, n, c, Ur.p, r, r, VB.p, s);
            transpose_dense<double>(VB.p, VtB.p, n, r, s);
        } else {
            // B (c x n) is tall: B = Q_b R (R: n x n), R = U_J S V_J^T -> B = (Q_b U_J) S V_J^T
            DevBuf<double> B((size_t)c * n, s);
            transpose_dense<double>(Bt.p, B.p, n, c, s);
            cholesky_qr(cx, B.p, c, (int)n, R.p);
            DevBuf<double> Rt((size_t)r * r, s);
            transpose_dense<double>(R.p, Rt.p, r, r, s);
            k_jacobi_svd<<<1, jacobi_threads(r, 1024), smem, s>>>(Rt.p, r, Vr.p, Ur.p, sig.p, jac_status.p);
            right_mul(B.p, c, (int)n, Ur.p, r, r, UB.p, s);
            transpose_dense<double>(Vr.p, VtB.p, r, r, s);
        }
        SVDB_CHECK_LAUNCH();
    }
    if (verbose) printf("SVD | Randomized | Running Singular Value Decomposition, took %.3f ms\n", ms_since(t0));
    // U = Q U_B (m x r), truncated to actual_rank columns
    const int64_t actual = std::min<int64_t>((int64_t)target_rank, r);
    DevBuf<double> U(std::max<int64_t>(m * actual, 1), s), Vt(std::max<int64_t>(actual * n, 1), s),
        S(std::max<int64_t>(actual, 1), s);
    if (actual > 0) {
        right_mul(Y.p, m, c, UB.p, r, (int)actual, U.p, s);
        SVDB_CUDA(cudaMemcpyAsync(Vt.p, VtB.p, actual * n * 8, cudaMemcpyDeviceToDevice, s));
        SVDB_CUDA(cudaMemcpyAsync(S.p, sig.p, actual * 8, cudaMemcpyDeviceToDevice, s));
    }
    SVDB_CUDA(cudaEventRecord(e1, s));
    int hflags = 0, hjac = 0;
    SVDB_CUDA(cudaMemcpyAsync(&hflags, cx.flags.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaMemcpyAsync(&hjac, jac_status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaStreamSynchronize(s));
    float tot = 0.f;
    cudaEventElapsedTime(&tot, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (auto& ev : spmm_events) {
        float t = 0.f;
        cudaEventElapsedTime(&t, ev.first, ev.second);
        spmm_ms += t;
        cudaEventDestroy(ev.first);
        cudaEventDestroy(ev.second);
    }
    spmm_tma_check();
    spmm_panel_check();
    gram_tc_check();
    if (split) dense_split_check();
    if (verbose) printf("SVD | Randomized | Jacobi sweeps on R: %d%s\n", hjac >> 8, (hjac & 2) ? " (limit)" : "");
    if (hflags & 2) throw Error(SVDB_ERR_LAS2, "randomized_svd: CholeskyQR broke down even with a shift");

    std::memset(rec, 0, sizeof(*rec));
    rec->d = actual;
    rec->u_rows = m; rec->u_cols = actual;
    rec->vt_rows = actual; rec->vt_cols = n;
    if (o.result_on_device) {
        rec->u = U.detach(); rec->s = S.detach(); rec->vt = Vt.detach();
        rec->on_device = 1;
    } else {
        rec->u = (double*)host_result_alloc(std::max<int64_t>(m * actual, 1) * 8);
        rec->s = (double*)host_result_alloc(std::max<int64_t>(actual, 1) * 8);
        rec->vt = (double*)host_result_alloc(std::max<int64_t>(actual * n, 1) * 8);
        if (actual) {
            SVDB_CUDA(cudaMemcpyAsync(rec->u, U.p, m * actual * 8, cudaMemcpyDeviceToHost, s));
            SVDB_CUDA(cudaMemcpyAsync(rec->s, S.p, actual * 8, cudaMemcpyDeviceToHost, s));
            SVDB_CUDA(cudaMemcpyAsync(rec->vt, Vt.p, actual * n * 8, cudaMemcpyDeviceToHost, s));
        }
        SVDB_CUDA(cudaStreamSynchronize(s));
    }
    rec->origin = SVDB_REC_RANDOMIZED;
    // create_diagnostics (mod.rs:214-237)
    svdb_diagnostics& dg = rec->diagnostics;
    dg.non_zero = A->nnz;
    dg.dimensions = target_rank;
    dg.iterations = n_power_iters;
    dg.transposed = 0;
    dg.lanczos_steps = 0;
    dg.ritz_values_stabilized = actual;
    dg.significant_values = actual;
    dg.singular_values = actual;
    dg.end_interval[0] = -1e-30;
    dg.end_interval[1] = 1e-30;
    dg.kappa = 1e-6;
    dg.random_seed = (uint32_t)(has_seed ? seed : 0);
    rec->time_ms_total = tot;
    rec->time_ms_spmv = spmm_ms;
    rec->time_ms_ortho = tot - spmm_ms;
}

}  // namespace svdb
