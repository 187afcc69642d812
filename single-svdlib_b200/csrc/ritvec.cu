// Device half of ritvec (src/lanczos/mod.rs:1056-1259, src/legacy.rs:1766-1850).
//
// imtql2's eigenvector accumulation is the O(js^3) part: the host runs the
// scalar QL recurrence (which never reads z) and records every plane
// rotation (i, c, s) in order; here each thread owns one row of Z and applies
// the whole rotation list to it.  Rows are independent, and every element
// sees the crate's exact operation sequence (s*z[i] + c*f, c*z[i] - s*f,
// unfused), so Z is bit-identical to the sequential loop's.
#include <algorithm>
#include <string>

#include "device_common.cuh"
#include "ops.cuh"
#include "ritvec.cuh"
#include "svdb_internal.h"

namespace svdb {

// Z is column-major: Z(row k, col i) at z[i * js + k]; thread k walks row k.
__global__ void __launch_bounds__(128) k_rot_apply(double* __restrict__ z, int64_t js,
                                                   const int32_t* __restrict__ ri, const double* __restrict__ rc,
                                                   const double* __restrict__ rs, int64_t nrot) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= js) return;
    for (int64_t i = 0; i < js; ++i) z[i * js + k] = (i == k) ? 1.0 : 0.0;
    for (int64_t t = 0; t < nrot; ++t) {
        const int64_t i = ri[t];
        const double c = rc[t], s = rs[t];
        double* zi = z + i * js + k;
        double* zi1 = z + (i + 1) * js + k;
        const double f = *zi1;
        const double a = *zi;
        *zi1 = add_rn(mul_rn(s, a), mul_rn(c, f));
        *zi = sub_rn(mul_rn(c, a), mul_rn(s, f));
    }
}

// The same in shared memory: block b owns rows b*ROWS .. +ROWS of Z, stored
// as zs[i * ROWS + local row]; the rotation list is staged in chunks that
// every thread reads (a broadcast).  Within a QL sweep the rotations walk i
// downwards, and rotation i - 1 reads as f the z[i] that rotation i has just
// written: it is handed over in a register.  Each element still sees the
// crate's operations in order (unfused), so Z is bit-identical.
constexpr int kRotChunk = 1024;
__global__ void __launch_bounds__(64) k_rot_apply_smem(double* __restrict__ z, int64_t js,
                                                       const int32_t* __restrict__ ri,
                                                       const double* __restrict__ rc,
                                                       const double* __restrict__ rs, int64_t nrot) {
    extern __shared__ double zs[];  // js x blockDim.x
    __shared__ int32_t sri[kRotChunk];
    __shared__ double src_[kRotChunk], srs[kRotChunk];
    const int rows = blockDim.x, tid = threadIdx.x;
    const int64_t k = blockIdx.x * (int64_t)rows + tid;
    for (int64_t i = 0; i < js; ++i) zs[i * rows + tid] = (i == k) ? 1.0 : 0.0;
    int64_t prev = -2;
    double carry = 0.0;
    for (int64_t t0 = 0; t0 < nrot; t0 += kRotChunk) {
        const int cnt = (int)min((int64_t)kRotChunk, nrot - t0);
        __syncthreads();
        for (int u = tid; u < cnt; u += rows) {
            sri[u] = ri[t0 + u];
            src_[u] = rc[t0 + u];
            srs[u] = rs[t0 + u];
        }
        __syncthreads();
        for (int u = 0; u < cnt; ++u) {
            const int64_t i = sri[u];
            const double c = src_[u], s = srs[u];
            const double f = (i + 1 == prev) ? carry : zs[(i + 1) * rows + tid];
            const double a = zs[i * rows + tid];
            const double hi = add_rn(mul_rn(s, a), mul_rn(c, f));
            const double lo = sub_rn(mul_rn(c, a), mul_rn(s, f));
            zs[(i + 1) * rows + tid] = hi;
            zs[i * rows + tid] = lo;
            carry = lo;
            prev = i;
        }
    }
    __syncthreads();
    if (k < js)
        for (int64_t i = 0; i < js; ++i) z[i * js + k] = zs[i * rows + tid];
}

// C (d x js) row-major.  The final Z after imtql2's column sort is
// Zf(row, col) = Zrot(row, perm[col]).
//   lanczos (mod.rs:1150-1161): C[r][i] = Zf(k_r, i) if |.| > eps_a else 0
//   legacy (legacy.rs:1796-1806): C[r][i] = Zf(js-1-i, k_r) (zero terms skipped)
__global__ void k_build_coef(const double* __restrict__ z, int64_t js, const int32_t* __restrict__ perm,
                             const int32_t* __restrict__ rowk, int64_t d, int legacy, double eps_a,
                             double* __restrict__ C) {
    const int64_t total = d * js;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = t / js, i = t % js;
        const int64_t k = rowk[r];
        double v;
        if (!legacy) {
            v = z[(int64_t)perm[i] * js + k];
            if (!(fabs(v) > eps_a)) v = 0.0;
        } else {
            v = z[(int64_t)perm[k] * js + (js - 1 - i)];
        }
        C[t] = v;
    }
}

// Vt (d x n) = C (d x js) Q (js x n): every output element accumulates its
// terms in ascending i, skipping zero coefficients, unfused (the crate's
// `vec[j] += s * item`).  Block: 256 columns x RT rows of output.
constexpr int kRT = 16;
constexpr int kIC = 256;
__global__ void __launch_bounds__(256) k_backtransform(const double* __restrict__ C, const double* __restrict__ Q,
                                                       int64_t js, int64_t n, int64_t d, double* __restrict__ Vt) {
    __shared__ double sc[kRT][kIC];
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t r0 = blockIdx.y * (int64_t)kRT;
    double acc[kRT];
#pragma unroll
    for (int r = 0; r < kRT; ++r) acc[r] = 0.0;
    for (int64_t i0 = 0; i0 < js; i0 += kIC) {
        const int ic = (int)std::min<int64_t>(kIC, js - i0);
        __syncthreads();
        for (int t = threadIdx.x; t < kRT * kIC; t += blockDim.x) {
            const int r = t / kIC, ii = t % kIC;
            sc[r][ii] = (r0 + r < d && ii < ic) ? C[(r0 + r) * js + i0 + ii] : 0.0;
        }
        __syncthreads();
        if (e < n) {
            for (int ii = 0; ii < ic; ++ii) {
                const double q = Q[(i0 + ii) * n + e];
#pragma unroll
                for (int r = 0; r < kRT; ++r) {
                    const double c = sc[r][ii];
                    if (c != 0.0) acc[r] = add_rn(acc[r], mul_rn(c, q));
                }
            }
        }
    }
    if (e < n) {
#pragma unroll
        for (int r = 0; r < kRT; ++r)
            if (r0 + r < d) Vt[(r0 + r) * n + e] = acc[r];
    }
}

// t[r] = sum_e Vt[r][e] * T[e][r]  (T: n x d row-major)
__global__ void __launch_bounds__(256) k_col_dots(const double* __restrict__ Vt, const double* __restrict__ T,
                                                  int64_t n, int64_t d, double* __restrict__ t) {
    __shared__ double sh[32];
    const int64_t r = blockIdx.x;
    double acc = 0.0;
    for (int64_t e = threadIdx.x; e < n; e += blockDim.x) acc = fma(Vt[r * n + e], T[e * d + r], acc);
    double s = block_sum(acc, sh);
    if (threadIdx.x == 0) t[r] = s;
}

// sigma and the scale of u (mod.rs:1212-1243 / legacy.rs:1834-1848)
__global__ void k_sigma(const double* __restrict__ t, int64_t d, int legacy, double eps_a, double* __restrict__ S,
                        double* __restrict__ scale) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= d) return;
    if (!legacy) {
        const double sv = sqrt(fmax(t[r], 0.0));
        S[r] = sv;
        scale[r] = (sv > eps_a) ? 1.0 / sv : 1.0 / fmax(sv, eps_a);
    } else {
        const double sv = sqrt(t[r]);
        S[r] = sv;
        scale[r] = 1.0 / sv;
    }
}

// Ut (d x m) = (Y (m x d))^T with row r scaled by scale[r]
__global__ void k_scale_rows(double* __restrict__ Ut, int64_t d, int64_t m, const double* __restrict__ scale) {
    const int64_t total = d * m;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x)
        Ut[t] = mul_rn(Ut[t], scale[t / m]);
}

static int nblk(int64_t work, int threads) {
    int64_t b = (work + threads - 1) / threads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)device_props().sms * 16));
}

void rot_apply(double* z, int64_t js, const int32_t* ri, const double* rc, const double* rs, int64_t nrot,
               cudaStream_t s) {
    // rows per block in shared memory: as many as fit next to the staged rotations
    const size_t avail = 200 * 1024;
    int rows = 64;
    while (rows >= 16 && (size_t)js * rows * sizeof(double) > avail) rows >>= 1;
    if (rows >= 16) {
        const size_t smem = (size_t)js * rows * sizeof(double);
        // the kernel also holds 20 KB of static shared memory: always raise the dynamic limit
        SVDB_CUDA(cudaFuncSetAttribute(k_rot_apply_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_rot_apply_smem<<<(unsigned)((js + rows - 1) / rows), rows, smem, s>>>(z, js, ri, rc, rs, nrot);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            throw Error(SVDB_ERR_CUDA, "k_rot_apply_smem(js=" + std::to_string(js) + ", rows=" + std::to_string(rows) +
                                           ", smem=" + std::to_string(smem) + "): " + cudaGetErrorString(e));
    } else {
        k_rot_apply<<<(unsigned)((js + 127) / 128), 128, 0, s>>>(z, js, ri, rc, rs, nrot);
    }
    SVDB_CHECK_LAUNCH();
}

void build_coef(const double* z, int64_t js, const int32_t* perm, const int32_t* rowk, int64_t d, bool legacy,
                double eps_a, double* C, cudaStream_t s) {
    if (d == 0) return;
    k_build_coef<<<nblk(d * js, 256), 256, 0, s>>>(z, js, perm, rowk, d, legacy, eps_a, C);
    SVDB_CHECK_LAUNCH();
}

void backtransform(const double* C, const double* Q, int64_t js, int64_t n, int64_t d, double* Vt, cudaStream_t s) {
    if (d == 0 || n == 0) return;
    dim3 grid((unsigned)((n + 255) / 256), (unsigned)((d + kRT - 1) / kRT));
    k_backtransform<<<grid, 256, 0, s>>>(C, Q, js, n, d, Vt);
    SVDB_CHECK_LAUNCH();
}

void sigma_and_u(const DevCompressed& op1, const DevCompressed& op2, bool fp32, const double* Vt, int64_t d,
                 int64_t n, int64_t m, bool legacy, double eps_a, double* S, double* Ut, cudaStream_t s) {
    if (d == 0) return;
    DevBuf<double> V(n * d, s), Y(m * d, s), T(n * d, s), t(d, s), scale(d, s);
    transpose_dense<double>(Vt, V.p, d, n, s);       // V (n x d)
    spmm_dev<double, double>(op1, fp32, V.p, (int)d, Y.p, s);  // Y = A v   (m x d)
    spmm_dev<double, double>(op2, fp32, Y.p, (int)d, T.p, s);  // T = A^T A v (n x d)
    k_col_dots<<<(unsigned)d, 256, 0, s>>>(Vt, T.p, n, d, t.p);
    k_sigma<<<(unsigned)((d + 127) / 128), 128, 0, s>>>(t.p, d, legacy, eps_a, S, scale.p);
    transpose_dense<double>(Y.p, Ut, m, d, s);       // Ut (d x m)
    k_scale_rows<<<nblk(d * m, 256), 256, 0, s>>>(Ut, d, m, scale.p);
    SVDB_CHECK_LAUNCH_N(3);
}

}  // namespace svdb
