// Adjoint of the truncated SVD with respect to A's stored values, evaluated
// only at A's nonzeros (an SDDMM), and svd_flip.  The crate has no adjoint;
// svd_flip follows src/randomized/mod.rs:332-438.
//
// For A V = U S, A^T U = V S (k leading triplets) and a loss L(U, s, V):
//   dL/dA = U M V^T + Gamma V^T + U Delta^T
//   M = diag(g_s) + (F o (J_U - J_U^T)) S + S (F o (J_V - J_V^T)),
//   J_U = U^T g_U, J_V = V^T g_V, F_ij = 1/(s_j^2 - s_i^2) off the diagonal.
// The complement parts X = (I - UU^T) dU, Y = (I - VV^T) dV satisfy
//   X S - A_p Y = (I - UU^T) dA V,   Y S - A_p^T X = (I - VV^T) dA^T U
// with A_p = A - U S V^T, so their adjoint solves, column i, the same
// symmetric system with right-hand side (a_i, b_i) = ((I-UU^T) g_U e_i,
// (I-VV^T) g_V e_i):  (s_i^2 I - A_p^T A_p) delta_i = s_i b_i + A_p^T a_i,
// gamma_i = (a_i + A_p delta_i) / s_i.  s_i above the (k+1)-th singular
// value makes the matrix SPD, so the k systems run as one block CG that
// shares its sparse products.  dL/dA is then the product of the rank-2k
// factors [U M + Gamma, U] and [V, Delta], evaluated at the nonzeros.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "device_common.cuh"
#include "ops.cuh"
#include "svdb_internal.h"

namespace svdb {

static int grid_for_work(int64_t work, int threads, int per_sm = 8) {
    int64_t b = (work + threads - 1) / threads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)device_props().sms * per_sm));
}

// ------------------------------------------------------------------ SDDMM ----
// One warp per segment of the load-balancing plan (at most kSegNnz entries of
// one row).  Lane t keeps left[r][t + 32 j] (j < SLOTS) in registers.  The
// segment is taken 32 entries at a time: for entry q every lane forms its
// partial product with right[c_q] (coalesced row reads), and a butterfly
// transpose reduction (16 + 8 + 4 + 2 + 1 shuffles for all 32 entries) leaves
// lane q holding the dot product of entry q, in a fixed order.
template <typename T, int SLOTS>
__global__ void __launch_bounds__(256) k_sddmm(const int32_t* __restrict__ idx, const int32_t* __restrict__ seg_row,
                                               const int64_t* __restrict__ seg_beg,
                                               const int64_t* __restrict__ seg_end, int64_t nseg,
                                               const T* __restrict__ left, const T* __restrict__ right, int rank,
                                               T* __restrict__ out) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t sg = warp0; sg < nseg; sg += nwarps) {
        int32_t r = seg_row[sg];
        if (r < 0) r = -r - 1;
        const int64_t beg = seg_beg[sg], end = seg_end[sg];
        T lv[SLOTS];
#pragma unroll
        for (int j = 0; j < SLOTS; ++j) {
            const int t = lane + 32 * j;
            lv[j] = t < rank ? left[(int64_t)r * rank + t] : T(0);
        }
        for (int64_t p0 = beg; p0 < end; p0 += 32) {
            const int cnt = (int)min((int64_t)32, end - p0);
            const int cmine = lane < cnt ? idx[p0 + lane] : 0;
            T p[32];
#pragma unroll
            for (int q = 0; q < 32; ++q) {
                const int c = __shfl_sync(full, cmine, q);
                T acc = T(0);
                if (q < cnt) {
                    const T* rr = right + (int64_t)c * rank;
#pragma unroll
                    for (int j = 0; j < SLOTS; ++j) {
                        const int t = lane + 32 * j;
                        if (t < rank) acc = fma(lv[j], __ldg(rr + t), acc);
                    }
                }
                p[q] = acc;
            }
#pragma unroll
            for (int w = 16; w >= 1; w >>= 1) {
                const bool upper = (lane & w) != 0;
#pragma unroll
                for (int i = 0; i < w; ++i) {
                    const T send = upper ? p[i] : p[i + w];
                    const T keep = upper ? p[i + w] : p[i];
                    p[i] = keep + __shfl_xor_sync(full, send, w);
                }
            }
            if (lane < cnt) out[p0 + lane] = p[0];
        }
    }
}

template <typename T>
static void sddmm_launch(const DevCompressed& m, const T* left, const T* right, int rank, T* out, cudaStream_t s) {
    if (m.nnz == 0) return;
    const SegPlan& pl = m.plan;
    const int blocks = grid_for_work(pl.nseg * 32, 256, 8);
    const int slots = (rank + 31) / 32;
#define SVDB_SDDMM_CASE(S)                                                                                  \
    case S:                                                                                                 \
        k_sddmm<T, S><<<blocks, 256, 0, s>>>(m.idx.p, pl.seg_row.p, pl.seg_beg.p, pl.seg_end.p, pl.nseg, left, \
                                             right, rank, out);                                             \
        break;
    switch (slots) {
        SVDB_SDDMM_CASE(1)
        SVDB_SDDMM_CASE(2)
        SVDB_SDDMM_CASE(3)
        SVDB_SDDMM_CASE(4)
        SVDB_SDDMM_CASE(6)
        SVDB_SDDMM_CASE(8)
        case 5: k_sddmm<T, 6><<<blocks, 256, 0, s>>>(m.idx.p, pl.seg_row.p, pl.seg_beg.p, pl.seg_end.p, pl.nseg,
                                                     left, right, rank, out); break;
        case 7: k_sddmm<T, 8><<<blocks, 256, 0, s>>>(m.idx.p, pl.seg_row.p, pl.seg_beg.p, pl.seg_end.p, pl.nseg,
                                                     left, right, rank, out); break;
        default: throw Error(SVDB_ERR_UNSUPPORTED, "sddmm: rank above 256");
    }
#undef SVDB_SDDMM_CASE
    SVDB_CHECK_LAUNCH();
}

// The handle's own entry order: CSR handles use the CSR (rows of A, factors
// left = row side), CSC handles their CSC (rows of A^T, factors swapped).
static const DevCompressed& pattern_of(const svdb_matrix* a, bool& swapped) {
    if (a->kind == KIND_CSR) { swapped = false; return a->csr; }
    if (a->kind == KIND_CSC) { swapped = true; return a->csc; }
    throw Error(SVDB_ERR_UNSUPPORTED, "adjoint: COO handles and masked views have no stored entry order to return");
}

// ------------------------------------------------------- tall-skinny dense ----
// C (p x q) = X^T Y for X (rows x p, ld ldx), Y (rows x q, ld ldy): blocks
// take row chunks staged through shared memory; a 16 x 16 thread grid keeps
// an NC x NC tile of C.  Block partials are summed in block order.
constexpr int kAtbRows = 32;
template <int NC>
__global__ void __launch_bounds__(256) k_atb_part(const double* __restrict__ X, int64_t ldx,
                                                  const double* __restrict__ Y, int64_t ldy, int64_t rows, int p,
                                                  int q, int64_t chunk, double* __restrict__ part) {
    extern __shared__ double sm[];
    double* xs = sm;                 // kAtbRows x p
    double* ys = sm + kAtbRows * p;  // kAtbRows x q
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int64_t r0 = blockIdx.x * chunk, r1 = min(rows, r0 + chunk);
    double acc[NC][NC];
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int j = 0; j < NC; ++j) acc[i][j] = 0.0;
    for (int64_t rb = r0; rb < r1; rb += kAtbRows) {
        const int nr = (int)min((int64_t)kAtbRows, r1 - rb);
        __syncthreads();
        for (int t = threadIdx.x; t < nr * p; t += blockDim.x) xs[t] = X[(rb + t / p) * ldx + t % p];
        for (int t = threadIdx.x; t < nr * q; t += blockDim.x) ys[t] = Y[(rb + t / q) * ldy + t % q];
        __syncthreads();
        for (int r = 0; r < nr; ++r) {
            double xa[NC], yb[NC];
#pragma unroll
            for (int i = 0; i < NC; ++i) {
                const int a = ty + 16 * i, b = tx + 16 * i;
                xa[i] = a < p ? xs[r * p + a] : 0.0;
                yb[i] = b < q ? ys[r * q + b] : 0.0;
            }
#pragma unroll
            for (int i = 0; i < NC; ++i)
#pragma unroll
                for (int j = 0; j < NC; ++j) acc[i][j] = fma(xa[i], yb[j], acc[i][j]);
        }
    }
    double* o = part + (int64_t)blockIdx.x * p * q;
#pragma unroll
    for (int i = 0; i < NC; ++i)
#pragma unroll
        for (int j = 0; j < NC; ++j) {
            const int a = ty + 16 * i, b = tx + 16 * j;
            if (a < p && b < q) o[a * q + b] = acc[i][j];
        }
}

__global__ void k_sum_parts(const double* __restrict__ part, int nblocks, int count, double* __restrict__ out) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x) {
        double s0 = 0.0, s1 = 0.0;
        int b = 0;
        for (; b + 2 <= nblocks; b += 2) {
            s0 += part[(int64_t)b * count + e];
            s1 += part[(int64_t)(b + 1) * count + e];
        }
        if (b < nblocks) s0 += part[(int64_t)b * count + e];
        out[e] = s0 + s1;
    }
}

// Out (rows x q, ld ldo) = beta * Y + alpha * X diag(d) C, X: rows x p (ld
// ldx), C: p x q row-major, d: p values or null (= 1), Y null when beta = 0.
// Out may be Y (each element is read, then written, by one thread).
constexpr int kGtRows = 32;
__global__ void __launch_bounds__(256) k_gemm_tall(const double* __restrict__ X, int64_t ldx, int64_t rows, int p,
                                                   const double* __restrict__ C, const double* __restrict__ d, int q,
                                                   double alpha, const double* Y, int64_t ldy, double beta,
                                                   double* Out, int64_t ldo) {
    extern __shared__ double sm[];
    double* cs = sm;          // p x q, rows scaled by d
    double* xs = sm + p * q;  // kGtRows x p
    for (int t = threadIdx.x; t < p * q; t += blockDim.x) cs[t] = d ? d[t / q] * C[t] : C[t];
    for (int64_t r0 = (int64_t)blockIdx.x * kGtRows; r0 < rows; r0 += (int64_t)gridDim.x * kGtRows) {
        const int nr = (int)min((int64_t)kGtRows, rows - r0);
        __syncthreads();
        for (int t = threadIdx.x; t < nr * p; t += blockDim.x) xs[t] = X[(r0 + t / p) * ldx + t % p];
        __syncthreads();
        for (int t = threadIdx.x; t < nr * q; t += blockDim.x) {
            const int rr = t / q, j = t % q;
            double s = 0.0;
            for (int k = 0; k < p; ++k) s = fma(xs[rr * p + k], cs[k * q + j], s);
            const int64_t row = r0 + rr;
            const double y = (beta != 0.0) ? beta * Y[row * ldy + j] : 0.0;
            Out[row * ldo + j] = y + alpha * s;
        }
    }
}

// Out[r][j] = ca[j] A[r][j] + sb cb[j] B[r][j]; ca / cb null mean 1, B null
// drops the second term.  Out may alias A or B.
__global__ void k_axpby_cols(int64_t rows, int k, double* Out, int64_t ldo, const double* A, int64_t lda,
                             const double* __restrict__ ca, const double* B, int64_t ldb,
                             const double* __restrict__ cb, double sb) {
    const int64_t total = rows * k;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = t / k;
        const int j = (int)(t % k);
        double v = A[r * lda + j] * (ca ? ca[j] : 1.0);
        if (B) v += sb * (cb ? cb[j] : 1.0) * B[r * ldb + j];
        Out[r * ldo + j] = v;
    }
}

__global__ void k_diag(const double* __restrict__ C, int k, double* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < k) out[j] = C[j * k + j];
}

// CG scalars per column.  A column is frozen (alpha = beta = 0) once its
// residual norm is below freeze * ||rhs||, or when a denominator is not positive.
__global__ void k_cg_alpha(const double* __restrict__ rr, const double* __restrict__ pw,
                           const double* __restrict__ rhs_norm, double freeze, int k, double* __restrict__ alpha) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    const bool live = rr[j] > 0.0 && pw[j] > 0.0 && sqrt(rr[j]) > freeze * rhs_norm[j];
    alpha[j] = live ? rr[j] / pw[j] : 0.0;
}
__global__ void k_cg_beta(const double* __restrict__ rr_new, double* __restrict__ rr, const double* __restrict__ alpha,
                          int k, double* __restrict__ beta) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    beta[j] = (alpha[j] != 0.0 && rr[j] > 0.0) ? rr_new[j] / rr[j] : 0.0;
    rr[j] = rr_new[j];
}

struct TallCtx {
    cudaStream_t s;
    DevBuf<double> part;
};

static void atb(TallCtx& cx, const double* X, int64_t ldx, const double* Y, int64_t ldy, int64_t rows, int p, int q,
                double* C) {
    const int nc = (std::max(p, q) + 15) / 16;
    if (nc > 8) throw Error(SVDB_ERR_UNSUPPORTED, "adjoint: more than 128 triplets");
    const int sms = device_props().sms;
    const int64_t chunk = std::max<int64_t>(kAtbRows * 4, (rows + sms * 2 - 1) / (sms * 2));
    const int nblk = (int)std::max<int64_t>(1, (rows + chunk - 1) / chunk);
    if ((int64_t)cx.part.n < (int64_t)nblk * p * q) cx.part.alloc((size_t)nblk * p * q, cx.s);
    const size_t smem = (size_t)kAtbRows * (p + q) * sizeof(double);
#define SVDB_ATB_CASE(N)                                                                                     \
    case N:                                                                                                  \
        if (smem > 48 * 1024)                                                                                \
            SVDB_CUDA(cudaFuncSetAttribute(k_atb_part<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                           (int)smem));                                                      \
        k_atb_part<N><<<nblk, 256, smem, cx.s>>>(X, ldx, Y, ldy, rows, p, q, chunk, cx.part.p);               \
        break;
    switch (nc) {
        SVDB_ATB_CASE(1)
        SVDB_ATB_CASE(2)
        SVDB_ATB_CASE(3)
        SVDB_ATB_CASE(4)
        SVDB_ATB_CASE(5)
        SVDB_ATB_CASE(6)
        SVDB_ATB_CASE(7)
        SVDB_ATB_CASE(8)
    }
#undef SVDB_ATB_CASE
    k_sum_parts<<<grid_for_work((int64_t)p * q, 128), 128, 0, cx.s>>>(cx.part.p, nblk, p * q, C);
    SVDB_CHECK_LAUNCH_N(2);
}

static void gemm_tall(const double* X, int64_t ldx, int64_t rows, int p, const double* C, const double* d, int q,
                      double alpha, const double* Y, int64_t ldy, double beta, double* Out, int64_t ldo,
                      cudaStream_t s) {
    if (rows == 0) return;
    const size_t smem = ((size_t)p * q + (size_t)kGtRows * p) * sizeof(double);
    if (smem > 200 * 1024) throw Error(SVDB_ERR_UNSUPPORTED, "adjoint: factor wider than the shared-memory tile");
    if (smem > 48 * 1024)
        SVDB_CUDA(cudaFuncSetAttribute(k_gemm_tall, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int blocks = (int)std::max<int64_t>(
        1, std::min<int64_t>((rows + kGtRows - 1) / kGtRows, (int64_t)device_props().sms * 4));
    k_gemm_tall<<<blocks, 256, smem, s>>>(X, ldx, rows, p, C, d, q, alpha, Y, ldy, beta, Out, ldo);
    SVDB_CHECK_LAUNCH();
}

static void axpby_cols(int64_t rows, int k, double* Out, int64_t ldo, const double* A, int64_t lda, const double* ca,
                       const double* B, int64_t ldb, const double* cb, double sb, cudaStream_t s) {
    if (rows * k == 0) return;
    k_axpby_cols<<<grid_for_work(rows * k, 256), 256, 0, s>>>(rows, k, Out, ldo, A, lda, ca, B, ldb, cb, sb);
    SVDB_CHECK_LAUNCH();
}

__global__ void k_to_f32_adj(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}
__global__ void k_to_f64_adj(const float* __restrict__ in, double* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

// ---------------------------------------------------------------- adjoint ----
void svd_adjoint(const svdb_matrix* A, int64_t k, const double* u, const double* s_in, const double* v,
                 const double* g_u, const double* g_s, const double* g_v, svdb_adjoint_options& o,
                 double* grad_values) {
    bool swapped = false;
    const DevCompressed& pat = pattern_of(A, swapped);
    cudaStream_t s = o.stream ? (cudaStream_t)o.stream : A->stream;
    const int64_t m = A->nrows, n = A->ncols, nnz = pat.nnz;
    const bool dev = o.inputs_on_device != 0;
    if (k < 0 || k > std::min<int64_t>(128, std::min(m, n)))
        throw Error(SVDB_ERR_UNSUPPORTED, "adjoint: k must be at most min(nrows, ncols, 128)");
    if (!grad_values || (k > 0 && (!u || !s_in || !v))) throw Error(SVDB_ERR_ARG, "null argument");
    o.cg_iterations = 0;
    o.cg_residual = 0.0;
    o.time_ms_solve = o.time_ms_sddmm = 0.0;
    if (k == 0 || nnz == 0) {
        if (dev) SVDB_CUDA(cudaMemsetAsync(grad_values, 0, std::max<int64_t>(nnz, 0) * 8, s));
        else std::memset(grad_values, 0, std::max<int64_t>(nnz, 0) * 8);
        if (dev) SVDB_CUDA(cudaStreamSynchronize(s));
        return;
    }
    const int kk = (int)k;
    // host copies of s and g_s (the k x k algebra runs on the host)
    std::vector<double> sv(k), gs(k, 0.0);
    if (dev) {
        SVDB_CUDA(cudaMemcpyAsync(sv.data(), s_in, k * 8, cudaMemcpyDeviceToHost, s));
        if (g_s) SVDB_CUDA(cudaMemcpyAsync(gs.data(), g_s, k * 8, cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
    } else {
        std::memcpy(sv.data(), s_in, k * 8);
        if (g_s) std::memcpy(gs.data(), g_s, k * 8);
    }
    for (int i = 0; i < kk; ++i)
        if (!(sv[i] > 0.0) || !std::isfinite(sv[i]))
            throw Error(SVDB_ERR_ARG, "adjoint: singular values must be positive and finite");

    cudaEvent_t e0, e1, e2;
    SVDB_CUDA(cudaEventCreate(&e0));
    SVDB_CUDA(cudaEventCreate(&e1));
    SVDB_CUDA(cudaEventCreate(&e2));
    SVDB_CUDA(cudaEventRecord(e0, s));

    DevBuf<double> U(m * k, s), V(n * k, s), GU(m * k, s), GV(n * k, s);
    auto load = [&](DevBuf<double>& dst, const double* src, int64_t cnt) {
        if (!src) { SVDB_CUDA(cudaMemsetAsync(dst.p, 0, cnt * 8, s)); return; }
        SVDB_CUDA(cudaMemcpyAsync(dst.p, src, cnt * 8, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    };
    load(U, u, m * k);
    load(V, v, n * k);
    load(GU, g_u, m * k);
    load(GV, g_v, n * k);

    TallCtx cx;
    cx.s = s;
    DevBuf<double> kkbuf(4 * k * k, s);
    double* JU = kkbuf.p;
    double* JV = kkbuf.p + k * k;
    double* C1 = kkbuf.p + 2 * k * k;
    double* C2 = kkbuf.p + 3 * k * k;
    atb(cx, U.p, k, GU.p, k, m, kk, kk, JU);
    atb(cx, V.p, k, GV.p, k, n, kk, kk, JV);
    std::vector<double> hJ(2 * k * k);
    SVDB_CUDA(cudaMemcpyAsync(hJ.data(), JU, 2 * k * k * 8, cudaMemcpyDeviceToHost, s));

    // per-column vectors on the device: s, s^2, 1/s and CG scalars
    DevBuf<double> colv(9 * k, s);
    double* d_s = colv.p;
    double* d_s2 = colv.p + k;
    double* d_si = colv.p + 2 * k;
    double* d_rr = colv.p + 3 * k;
    double* d_rrn = colv.p + 4 * k;
    double* d_pw = colv.p + 5 * k;
    double* d_al = colv.p + 6 * k;
    double* d_be = colv.p + 7 * k;
    double* d_rhsn = colv.p + 8 * k;
    std::vector<double> hcol(3 * k);
    for (int i = 0; i < kk; ++i) {
        hcol[i] = sv[i];
        hcol[k + i] = sv[i] * sv[i];
        hcol[2 * k + i] = 1.0 / sv[i];
    }
    SVDB_CUDA(cudaMemcpyAsync(colv.p, hcol.data(), 3 * k * 8, cudaMemcpyHostToDevice, s));

    // a = (I - U U^T) g_U,  b = (I - V V^T) g_V
    DevBuf<double> Aa(m * k, s), Bb(n * k, s);
    gemm_tall(U.p, k, m, kk, JU, nullptr, kk, -1.0, GU.p, k, 1.0, Aa.p, k, s);
    gemm_tall(V.p, k, n, kk, JV, nullptr, kk, -1.0, GV.p, k, 1.0, Bb.p, k, s);

    const DevCompressed& Ar = csr_of(A);  // rows of A
    const DevCompressed& Ac = csc_of(A);  // rows of A^T
    // rhs = b diag(s) + (I - V V^T) A^T a
    DevBuf<double> Rhs(n * k, s), Z(n * k, s), T(m * k, s);
    spmm_dev<double, double>(Ac, false, Aa.p, kk, Z.p, s);
    atb(cx, V.p, k, Z.p, k, n, kk, kk, C1);
    gemm_tall(V.p, k, n, kk, C1, nullptr, kk, -1.0, Z.p, k, 1.0, Z.p, k, s);
    axpby_cols(n, kk, Rhs.p, k, Bb.p, k, d_s, Z.p, k, nullptr, 1.0, s);

    // W = (S^2 - A_p^T A_p) P
    auto apply_op = [&](const double* P, double* W) {
        spmm_dev<double, double>(Ar, false, P, kk, T.p, s);                        // T = A P
        atb(cx, V.p, k, P, k, n, kk, kk, C1);                                       // C1 = V^T P
        gemm_tall(U.p, k, m, kk, C1, d_s, kk, -1.0, T.p, k, 1.0, T.p, k, s);        // T -= U S C1
        spmm_dev<double, double>(Ac, false, T.p, kk, Z.p, s);                       // Z = A^T T
        atb(cx, U.p, k, T.p, k, m, kk, kk, C2);                                     // C2 = U^T T
        gemm_tall(V.p, k, n, kk, C2, d_s, kk, -1.0, Z.p, k, 1.0, Z.p, k, s);        // Z -= V S C2
        axpby_cols(n, kk, W, k, P, k, d_s2, Z.p, k, nullptr, -1.0, s);              // W = P S^2 - Z
    };

    // block CG, X = 0, R = P = rhs
    DevBuf<double> X(n * k, s), R(n * k, s), P(n * k, s), W(n * k, s);
    SVDB_CUDA(cudaMemsetAsync(X.p, 0, n * k * 8, s));
    SVDB_CUDA(cudaMemcpyAsync(R.p, Rhs.p, n * k * 8, cudaMemcpyDeviceToDevice, s));
    SVDB_CUDA(cudaMemcpyAsync(P.p, Rhs.p, n * k * 8, cudaMemcpyDeviceToDevice, s));
    atb(cx, R.p, k, R.p, k, n, kk, kk, C1);
    k_diag<<<(kk + 127) / 128, 128, 0, s>>>(C1, kk, d_rr);
    SVDB_CHECK_LAUNCH();
    std::vector<double> rhs_norm(k), rr(k);
    SVDB_CUDA(cudaMemcpyAsync(rr.data(), d_rr, k * 8, cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaStreamSynchronize(s));
    for (int j = 0; j < kk; ++j) rhs_norm[j] = std::sqrt(rr[j]);
    SVDB_CUDA(cudaMemcpyAsync(d_rhsn, rhs_norm.data(), k * 8, cudaMemcpyHostToDevice, s));
    const double tol = o.cg_tol > 0.0 ? o.cg_tol : 1e-12;
    const uint64_t max_it = o.cg_max_iters ? o.cg_max_iters : 5000;
    auto residual = [&]() {
        double worst = 0.0;
        for (int j = 0; j < kk; ++j)
            if (rhs_norm[j] > 0.0) worst = std::max(worst, std::sqrt(std::max(rr[j], 0.0)) / rhs_norm[j]);
        return worst;
    };
    double res = residual();
    uint64_t it = 0;
    while (res > tol && it < max_it) {
        apply_op(P.p, W.p);
        atb(cx, P.p, k, W.p, k, n, kk, kk, C1);
        k_diag<<<(kk + 127) / 128, 128, 0, s>>>(C1, kk, d_pw);
        k_cg_alpha<<<(kk + 127) / 128, 128, 0, s>>>(d_rr, d_pw, d_rhsn, 0.25 * tol, kk, d_al);
        SVDB_CHECK_LAUNCH_N(2);
        axpby_cols(n, kk, X.p, k, X.p, k, nullptr, P.p, k, d_al, 1.0, s);   // X += P alpha
        axpby_cols(n, kk, R.p, k, R.p, k, nullptr, W.p, k, d_al, -1.0, s);  // R -= W alpha
        atb(cx, V.p, k, R.p, k, n, kk, kk, C2);                               // keep R off span(V)
        gemm_tall(V.p, k, n, kk, C2, nullptr, kk, -1.0, R.p, k, 1.0, R.p, k, s);
        atb(cx, R.p, k, R.p, k, n, kk, kk, C1);
        k_diag<<<(kk + 127) / 128, 128, 0, s>>>(C1, kk, d_rrn);
        k_cg_beta<<<(kk + 127) / 128, 128, 0, s>>>(d_rrn, d_rr, d_al, kk, d_be);
        SVDB_CHECK_LAUNCH_N(2);
        axpby_cols(n, kk, P.p, k, R.p, k, nullptr, P.p, k, d_be, 1.0, s);   // P = R + P beta
        SVDB_CUDA(cudaMemcpyAsync(rr.data(), d_rr, k * 8, cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
        ++it;
        res = residual();
    }
    o.cg_iterations = it;
    o.cg_residual = res;

    // Gamma = (a + A_p Delta) diag(1/s), Delta = X
    DevBuf<double> Gm(m * k, s);
    spmm_dev<double, double>(Ar, false, X.p, kk, T.p, s);
    atb(cx, V.p, k, X.p, k, n, kk, kk, C1);
    gemm_tall(U.p, k, m, kk, C1, d_s, kk, -1.0, T.p, k, 1.0, T.p, k, s);
    atb(cx, U.p, k, T.p, k, m, kk, kk, C2);  // A_p Delta lies off span(U): drop the rounding residue
    gemm_tall(U.p, k, m, kk, C2, nullptr, kk, -1.0, T.p, k, 1.0, T.p, k, s);
    axpby_cols(m, kk, Gm.p, k, Aa.p, k, d_si, T.p, k, d_si, 1.0, s);

    // M on the host
    std::vector<double> M(k * k, 0.0);
    {
        const double* hJU = hJ.data();
        const double* hJV = hJ.data() + k * k;
        double smax2 = 0.0;
        for (int i = 0; i < kk; ++i) smax2 = std::max(smax2, sv[i] * sv[i]);
        for (int i = 0; i < kk; ++i)
            for (int j = 0; j < kk; ++j) {
                if (i == j) { M[i * k + j] = gs[i]; continue; }
                const double den = sv[j] * sv[j] - sv[i] * sv[i];
                const double f = std::fabs(den) > 1e-300 ? 1.0 / den : 0.0;
                const double au = hJU[i * k + j] - hJU[j * k + i];
                const double avv = hJV[i * k + j] - hJV[j * k + i];
                M[i * k + j] = f * au * sv[j] + sv[i] * f * avv;
            }
        (void)smax2;
    }
    DevBuf<double> dM(k * k, s);
    SVDB_CUDA(cudaMemcpyAsync(dM.p, M.data(), k * k * 8, cudaMemcpyHostToDevice, s));

    // factors: Lf = [U M + Gamma | U] (m x 2k), Rf = [V | Delta] (n x 2k)
    const int rank = 2 * kk;
    DevBuf<double> Lf(m * rank, s), Rf(n * rank, s);
    gemm_tall(U.p, k, m, kk, dM.p, nullptr, kk, 1.0, Gm.p, k, 1.0, Lf.p, rank, s);
    axpby_cols(m, kk, Lf.p + k, rank, U.p, k, nullptr, nullptr, 0, nullptr, 0.0, s);
    axpby_cols(n, kk, Rf.p, rank, V.p, k, nullptr, nullptr, 0, nullptr, 0.0, s);
    axpby_cols(n, kk, Rf.p + k, rank, X.p, k, nullptr, nullptr, 0, nullptr, 0.0, s);
    SVDB_CUDA(cudaEventRecord(e1, s));

    const double* left = swapped ? Rf.p : Lf.p;
    const double* right = swapped ? Lf.p : Rf.p;
    DevBuf<double> out_dev;
    double* out = grad_values;
    if (!dev) {
        out_dev.alloc(nnz, s);
        out = out_dev.p;
    }
    if (o.precision == SVDB_MIXED) {
        const int64_t nl = (swapped ? n : m) * rank, nr = (swapped ? m : n) * rank;
        DevBuf<float> l32(nl, s), r32(nr, s), o32(nnz, s);
        k_to_f32_adj<<<grid_for_work(nl, 256), 256, 0, s>>>(left, l32.p, nl);
        k_to_f32_adj<<<grid_for_work(nr, 256), 256, 0, s>>>(right, r32.p, nr);
        SVDB_CHECK_LAUNCH_N(2);
        sddmm_launch<float>(pat, l32.p, r32.p, rank, o32.p, s);
        k_to_f64_adj<<<grid_for_work(nnz, 256), 256, 0, s>>>(o32.p, out, nnz);
        SVDB_CHECK_LAUNCH();
    } else {
        sddmm_launch<double>(pat, left, right, rank, out, s);
    }
    SVDB_CUDA(cudaEventRecord(e2, s));
    if (!dev) SVDB_CUDA(cudaMemcpyAsync(grad_values, out, nnz * 8, cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaStreamSynchronize(s));
    float t1 = 0.f, t2 = 0.f;
    cudaEventElapsedTime(&t1, e0, e1);
    cudaEventElapsedTime(&t2, e1, e2);
    o.time_ms_solve = t1;
    o.time_ms_sddmm = t2;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    if (res > tol)
        throw Error(SVDB_ERR_NOCONV, "adjoint: block CG stopped at relative residual " + std::to_string(res) +
                                         " after " + std::to_string(it) + " iterations");
}

void sddmm_device(const svdb_matrix* A, const void* left, const void* right, int64_t rank, void* out, int precision,
                  cudaStream_t s) {
    bool swapped = false;
    const DevCompressed& pat = pattern_of(A, swapped);
    if (rank <= 0 || rank > 256) throw Error(SVDB_ERR_UNSUPPORTED, "sddmm: rank must be in 1..256");
    const void* l = swapped ? right : left;
    const void* r = swapped ? left : right;
    if (precision == SVDB_MIXED)
        sddmm_launch<float>(pat, (const float*)l, (const float*)r, (int)rank, (float*)out, s);
    else
        sddmm_launch<double>(pat, (const double*)l, (const double*)r, (int)rank, (double*)out, s);
}

// --------------------------------------------------------------- svd_flip ----
// sign[v] for vector v of X (rows x cols row-major): column v (by_row = 0) or
// row v (by_row = 1).  The deciding entry is the first one of largest
// magnitude (a strict > scan, as mod.rs:357-365 / :405-413); an all-zero
// vector decides by its entry 0.
__global__ void k_flip_signs(const double* __restrict__ X, int64_t rows, int64_t cols, int by_row,
                             double* __restrict__ sign) {
    __shared__ double sa[256];
    __shared__ int64_t si[256];
    const int64_t v = blockIdx.x;
    const int64_t len = by_row ? cols : rows;
    double best = 0.0;
    int64_t bi = INT64_MAX;
    for (int64_t i = threadIdx.x; i < len; i += blockDim.x) {
        const double a = fabs(by_row ? X[v * cols + i] : X[i * cols + v]);
        if (a > best) { best = a; bi = i; }
    }
    sa[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            const double a2 = sa[threadIdx.x + w];
            const int64_t i2 = si[threadIdx.x + w];
            if (a2 > sa[threadIdx.x] || (a2 == sa[threadIdx.x] && i2 < si[threadIdx.x])) {
                sa[threadIdx.x] = a2;
                si[threadIdx.x] = i2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const int64_t i = si[0] == INT64_MAX ? 0 : si[0];
        const double x = len ? (by_row ? X[v * cols + i] : X[i * cols + v]) : 0.0;
        sign[v] = x < 0.0 ? -1.0 : 1.0;
    }
}
// X (rows x cols): by_row = 0 scales column j by sign[j] (j < nsign), 1 scales row i.
__global__ void k_apply_signs(double* __restrict__ X, int64_t rows, int64_t cols, int by_row,
                              const double* __restrict__ sign, int64_t nsign) {
    const int64_t total = rows * cols;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t which = by_row ? t / cols : t % cols;
        if (which < nsign) X[t] *= sign[which];
    }
}

void svd_flip(double* u, int64_t u_rows, int64_t u_cols, double* v, int64_t v_rows, int64_t v_cols, bool u_based,
              bool on_device) {
    if (!u && !v) throw Error(SVDB_ERR_LAS2, "Both u and v cannot be None");
    if (u_based && !u) throw Error(SVDB_ERR_LAS2, "u cannot be None when u_based_decision is true");
    if (!u_based && !v) throw Error(SVDB_ERR_LAS2, "v cannot be None when u_based_decision is false");
    cudaStream_t s = 0;
    const int64_t nu = u ? u_rows * u_cols : 0, nv = v ? v_rows * v_cols : 0;
    DevBuf<double> du, dv;
    double* pu = u;
    double* pv = v;
    if (!on_device) {
        if (u) {
            du.alloc(std::max<int64_t>(nu, 1), s);
            if (nu) SVDB_CUDA(cudaMemcpyAsync(du.p, u, nu * 8, cudaMemcpyHostToDevice, s));
            pu = du.p;
        }
        if (v) {
            dv.alloc(std::max<int64_t>(nv, 1), s);
            if (nv) SVDB_CUDA(cudaMemcpyAsync(dv.p, v, nv * 8, cudaMemcpyHostToDevice, s));
            pv = dv.p;
        }
    }
    const int64_t nsign = u_based ? u_cols : v_rows;
    DevBuf<double> sign(std::max<int64_t>(nsign, 1), s);
    if (nsign > 0) {
        if (u_based) k_flip_signs<<<(unsigned)nsign, 256, 0, s>>>(pu, u_rows, u_cols, 0, sign.p);
        else k_flip_signs<<<(unsigned)nsign, 256, 0, s>>>(pv, v_rows, v_cols, 1, sign.p);
        SVDB_CHECK_LAUNCH();
        if (pu && nu) {
            k_apply_signs<<<grid_for_work(nu, 256), 256, 0, s>>>(pu, u_rows, u_cols, 0, sign.p,
                                                                 u_based ? u_cols : std::min(u_cols, v_rows));
            SVDB_CHECK_LAUNCH();
        }
        if (pv && nv) {
            k_apply_signs<<<grid_for_work(nv, 256), 256, 0, s>>>(pv, v_rows, v_cols, 1, sign.p,
                                                                 u_based ? std::min(v_rows, u_cols) : v_rows);
            SVDB_CHECK_LAUNCH();
        }
    }
    if (!on_device) {
        if (u && nu) SVDB_CUDA(cudaMemcpyAsync(u, du.p, nu * 8, cudaMemcpyDeviceToHost, s));
        if (v && nv) SVDB_CUDA(cudaMemcpyAsync(v, dv.p, nv * 8, cudaMemcpyDeviceToHost, s));
    }
    SVDB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace svdb
