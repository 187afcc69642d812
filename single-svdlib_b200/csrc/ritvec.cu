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
// Rotation t is (c, s) = cs[t] and index il[t].x (rot_pack).
__global__ void __launch_bounds__(128) k_rot_apply(double* __restrict__ z, int64_t js, const double2* __restrict__ cs,
                                                   const int2* __restrict__ il, int64_t nrot, int first) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= js) return;
    if (first)
        for (int64_t i = 0; i < js; ++i) z[i * js + k] = (i == k) ? 1.0 : 0.0;
    for (int64_t t = 0; t < nrot; ++t) {
        const int64_t i = il[t].x;
        const double c = cs[t].x, s = cs[t].y;
        double* zi = z + i * js + k;
        double* zi1 = z + (i + 1) * js + k;
        const double f = *zi1;
        const double a = *zi;
        *zi1 = add_rn(mul_rn(s, a), mul_rn(c, f));
        *zi = sub_rn(mul_rn(c, a), mul_rn(s, f));
    }
}

// The same in shared memory: block b owns rows b*ROWS .. +ROWS of Z, stored
// as zs[i * ROWS + local row].  The rotation list arrives in segments
// (rot_pack): runs of consecutive rotations whose index falls by one, as a
// QL sweep makes them.  Inside a segment every z[i] is read (as a) before it
// is written (as the hi of rotation i - 1), and rotation i - 1 reads as f the
// lo that rotation i has just made, which stays in a register and is stored
// once, at the segment's end.  So the a values and (c, s) of the next group
// of kRotGroup rotations are read while the current group computes (two
// register sets in turn), and what remains in sequence is f <- c*a - s*f.
// With ROWS a compile-time constant every z access is an immediate offset
// from the group's base, and (c, s) is one 16-byte broadcast read: about ten
// instructions per rotation, against a 16-cycle chain.  Each element still
// sees the crate's operations in order (unfused), so Z is bit-identical.  The
// lists are staged by chunks of kRotChunk in two shared-memory buffers: the
// next chunk is copied (cp.async) while the current one is applied.
constexpr int kRotGroup = 8;

__device__ __forceinline__ void rot_cp16(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

struct RotStage {
    double2* cs;
    int2* il;
};

__device__ __forceinline__ RotStage rot_stage(unsigned char* base, int b) {
    unsigned char* p = base + (size_t)b * kRotChunk * kRotStageBytes;
    return RotStage{reinterpret_cast<double2*>(p), reinterpret_cast<int2*>(p + kRotChunk * 16)};
}

// Copies rotations t0 .. t0 + cnt (cnt rounded up to 4: the device lists are
// padded to a multiple of 4 entries) into stage st.
__device__ __forceinline__ void rot_stage_load(const RotStage& st, const double2* cs, const int2* il, int64_t t0,
                                               int cnt) {
    const int c4 = (cnt + 3) & ~3;
    const int ni = c4 / 2;  // 16-byte units of il (cs has c4)
    for (int u = threadIdx.x; u < c4 + ni; u += blockDim.x) {
        if (u < c4) rot_cp16(st.cs + u, cs + t0 + u);
        else rot_cp16(st.il + 2 * (u - c4), il + t0 + 2 * (u - c4));
    }
}

// Group of kRotGroup rotations at indices top', top' - 1, ...: zg points at
// z[top'] of this thread's row, pg at the group's (c, s).
template <int ROWS>
__device__ __forceinline__ void rot_group_load(const double* zg, const double2* pg, double (&A)[kRotGroup],
                                               double2 (&C)[kRotGroup]) {
#pragma unroll
    for (int q = 0; q < kRotGroup; ++q) {
        A[q] = zg[-q * ROWS];
        C[q] = pg[q];
    }
}

template <int ROWS>
__device__ __forceinline__ void rot_group_apply(double* zg, const double (&A)[kRotGroup],
                                                const double2 (&C)[kRotGroup], double& f) {
#pragma unroll
    for (int q = 0; q < kRotGroup; ++q) {
        const double hi = add_rn(mul_rn(C[q].y, A[q]), mul_rn(C[q].x, f));
        f = sub_rn(mul_rn(C[q].x, A[q]), mul_rn(C[q].y, f));
        zg[-(q - 1) * ROWS] = hi;  // z[i + 1]
    }
}

template <int ROWS>
__global__ void __launch_bounds__(ROWS) k_rot_apply_smem(double* __restrict__ z, int64_t js,
                                                         const double2* __restrict__ cs,
                                                         const int2* __restrict__ il, int64_t nrot, int first) {
    extern __shared__ __align__(16) unsigned char rot_smem[];
    double* zs = reinterpret_cast<double*>(rot_smem + 2 * kRotChunk * kRotStageBytes);  // js x ROWS
    const int tid = threadIdx.x;
    const int64_t k = blockIdx.x * (int64_t)ROWS + tid;
    for (int64_t i = 0; i < js; ++i)  // I, or the Z that earlier pieces of the list made
        zs[i * ROWS + tid] = first ? ((i == k) ? 1.0 : 0.0) : (k < js ? z[i * js + k] : 0.0);
    constexpr int G = kRotGroup;
    const int64_t nchunk = (nrot + kRotChunk - 1) / kRotChunk;
    if (nchunk > 0) rot_stage_load(rot_stage(rot_smem, 0), cs, il, 0, (int)(nrot < kRotChunk ? nrot : kRotChunk));
    asm volatile("cp.async.commit_group;" ::: "memory");
    for (int64_t ch = 0; ch < nchunk; ++ch) {
        const int64_t t1 = (ch + 1) * kRotChunk;
        if (t1 < nrot)
            rot_stage_load(rot_stage(rot_smem, (int)((ch + 1) & 1)), cs, il, t1,
                           (int)(nrot - t1 < kRotChunk ? nrot - t1 : kRotChunk));
        asm volatile("cp.async.commit_group;" ::: "memory");  // possibly empty: one group per chunk
        asm volatile("cp.async.wait_group 1;" ::: "memory");  // this chunk's copies have landed
        __syncthreads();
        const RotStage st = rot_stage(rot_smem, (int)(ch & 1));
        const int cnt = (int)(nrot - ch * kRotChunk < kRotChunk ? nrot - ch * kRotChunk : kRotChunk);
        for (int u = 0; u < cnt;) {
            const int2 h = st.il[u];  // (top index, segment length)
            const int len = h.y;
            double* zp = zs + h.x * ROWS + tid;  // z[top]
            const double2* p = st.cs + u;
            double f = zp[ROWS];
            const int nfull = len / G, rem = len - nfull * G;
            double A0[G], A1[G];
            double2 C0[G], C1[G];
            int g = 0;
            if (nfull > 0) rot_group_load<ROWS>(zp, p, A0, C0);
            for (; g + 2 <= nfull; g += 2) {  // the next group is untouched by this one
                rot_group_load<ROWS>(zp - (g + 1) * G * ROWS, p + (g + 1) * G, A1, C1);
                rot_group_apply<ROWS>(zp - g * G * ROWS, A0, C0, f);
                if (g + 2 < nfull) rot_group_load<ROWS>(zp - (g + 2) * G * ROWS, p + (g + 2) * G, A0, C0);
                rot_group_apply<ROWS>(zp - (g + 1) * G * ROWS, A1, C1, f);
            }
            if (g < nfull) {
                rot_group_apply<ROWS>(zp - g * G * ROWS, A0, C0, f);
                ++g;
            }
            if (rem) {
                double* zt = zp - nfull * G * ROWS;
                const double2* pt = p + nfull * G;
#pragma unroll
                for (int q = 0; q < G; ++q)
                    if (q < rem) {
                        A1[q] = zt[-q * ROWS];
                        C1[q] = pt[q];
                    }
#pragma unroll
                for (int q = 0; q < G; ++q)
                    if (q < rem) {
                        const double hi = add_rn(mul_rn(C1[q].y, A1[q]), mul_rn(C1[q].x, f));
                        f = sub_rn(mul_rn(C1[q].x, A1[q]), mul_rn(C1[q].y, f));
                        zt[-(q - 1) * ROWS] = hi;
                    }
            }
            zp[-(len - 1) * ROWS] = f;  // z[bottom] = the last lo
            u += len;
        }
        __syncthreads();  // this stage is refilled by the next iteration's copy
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    if (k < js)
        for (int64_t i = 0; i < js; ++i) z[i * js + k] = zs[i * ROWS + tid];
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

template <int ROWS>
static void launch_rot_smem(double* z, int64_t js, const double2* cs, const int2* il, int64_t nrot, int first,
                            cudaStream_t s) {
    const size_t smem = 2 * (size_t)kRotChunk * kRotStageBytes + (size_t)js * ROWS * sizeof(double);
    SVDB_CUDA(cudaFuncSetAttribute(k_rot_apply_smem<ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_rot_apply_smem<ROWS><<<(unsigned)((js + ROWS - 1) / ROWS), ROWS, smem, s>>>(z, js, cs, il, nrot, first);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        throw Error(SVDB_ERR_CUDA, "k_rot_apply_smem(js=" + std::to_string(js) + ", rows=" + std::to_string(ROWS) +
                                       ", smem=" + std::to_string(smem) + "): " + cudaGetErrorString(e));
}

void rot_apply(double* z, int64_t js, const double* cs, const int32_t* il, int64_t nrot, bool first, cudaStream_t s) {
    // rows per block in shared memory: as many as fit next to the two stages
    const size_t stage = 2 * (size_t)kRotChunk * kRotStageBytes;
    const size_t avail = (size_t)device_props().smem_optin - stage;
    const double2* cs2 = reinterpret_cast<const double2*>(cs);
    const int2* il2 = reinterpret_cast<const int2*>(il);
    const size_t row_bytes = (size_t)js * sizeof(double);
    const int f = first ? 1 : 0;
    if (row_bytes * 64 <= avail) launch_rot_smem<64>(z, js, cs2, il2, nrot, f, s);
    else if (row_bytes * 32 <= avail) launch_rot_smem<32>(z, js, cs2, il2, nrot, f, s);
    else if (row_bytes * 16 <= avail) launch_rot_smem<16>(z, js, cs2, il2, nrot, f, s);
    else k_rot_apply<<<(unsigned)((js + 127) / 128), 128, 0, s>>>(z, js, cs2, il2, nrot, f);
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
