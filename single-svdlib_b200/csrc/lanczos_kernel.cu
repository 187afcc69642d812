// Cooperative Lanczos-block kernel: runs lanczos_step for j in [first, last)
// (src/lanczos/mod.rs:674-758) entirely on the device, including the
// ortbnd recurrence (mod.rs:815-838) and purge (mod.rs:760-813), with one
// launch per lanso block.  All blocks advance in lockstep through bounded grid
// barriers; scalar results of reductions are recomputed identically by every
// block from the same partials, so no extra broadcast round is needed.
//
// Arithmetic: sparse products and dot products use FMA and a fixed-order
// tree; the element-wise updates (datx, dscal, daxpy) use unfused IEEE
// multiply-then-add, which is what the crate's `y += a * x` computes.
#include <cooperative_groups.h>

#include <mutex>

#include "lanczos_kernel.cuh"
#include "spmv.cuh"
#include "svdb_internal.h"

namespace svdb {

constexpr double kEps = 2.220446049250313e-16;
constexpr int kThreads = 512;

__device__ __forceinline__ bool cmp_eq(double a, double b) { return fabs(b - a) < kEps; }

// Row-gather SpMV over the rows of `op`: rows of more than kSegNnz entries
// (op.long_rows) one block each, the others through the length bins
// (spmv_binned, spmv.cuh).  SCALE: x is read as x * rinv (the dscal
// of w3 folded in).  EPI: y = acc + (-rnm) * w2, and returns this thread's
// share of dot(y, w3).  Only the matrix arrays are read through the
// non-coherent path: the vectors change between phases of the same launch.
template <bool FP32, bool SCALE, bool EPI, bool SL>
__device__ __forceinline__ double spmv_rows(const LzOperand& op, const double* x, double rinv, double* y,
                                            double neg_rnm, const double* w2, const double* w3, double* sh,
                                            double* dyn) {
    auto xl = [&](int32_t c) {
        double xv = x[c];
        if (SCALE) xv = mul_rn(xv, rinv);
        return xv;
    };
    double dotacc = 0.0;
    auto finish = [&](int64_t r, double acc) {
        if (EPI) {
            const double w0 = add_rn(acc, mul_rn(neg_rnm, w2[r]));
            y[r] = w0;
            dotacc = fma(w0, w3[r], dotacc);
        } else {
            y[r] = acc;
        }
    };
    if constexpr (SL) {  // x slices in shared memory (spmv.cuh)
        if (FP32) sliced_rows<float, SCALE>(op.sl, op.svf, x, rinv, dyn, finish);
        else sliced_rows<double, SCALE>(op.sl, op.sv, x, rinv, dyn, finish);
        return dotacc;
    }
    for (int64_t i = blockIdx.x; i < op.nlong; i += gridDim.x) {
        const int64_t r = __ldg(op.long_rows + i);
        const int64_t s = __ldg(op.rp + r), e = __ldg(op.rp + r + 1);
        double acc = FP32 ? row_dot(op.ci, op.vf, s, e, (int)threadIdx.x, (int)blockDim.x, xl)
                          : row_dot(op.ci, op.v, s, e, (int)threadIdx.x, (int)blockDim.x, xl);
        acc = block_sum(acc, sh);
        if (threadIdx.x == 0) finish(r, acc);
    }
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    if (FP32) spmv_binned(op.rp, op.ci, op.vf, op.bins, gwarp, nwarps, xl, finish);
    else spmv_binned(op.rp, op.ci, op.v, op.bins, gwarp, nwarps, xl, finish);
    return dotacc;
}

namespace cg = cooperative_groups;

// Barrier over all blocks: the bounded grid barrier of a cooperative launch,
// or (CL) the hardware barrier of a thread-block cluster that holds the whole
// grid.  Cluster mode needs control flow uniform over the blocks, which holds
// here: every branch depends on values all blocks compute identically.
template <bool CL>
__device__ __forceinline__ bool lz_sync(GridBarrier* bar) {
    if constexpr (CL) {
        cg::this_cluster().sync();
        return true;
    } else {
        return grid_sync(bar);
    }
}

// Sum over all blocks of one value per thread: block partial -> barrier ->
// every block adds the partials in the same order.  `par` alternates between
// two sets of partial slots, so a block that starts the next sum never
// overwrites a partial another block is still reading.  Cluster mode keeps
// the partials in each block's shared memory (cl_slot) and reads them across
// the cluster.
template <bool CL>
__device__ __forceinline__ bool lz_sum(double v, double* part, GridBarrier* bar, double* sh, double* cl_slot,
                                       double* cl_out, int& par, double& out) {
    const double b = block_sum(v, sh);
    const int p = par;
    par ^= 1;
    if constexpr (CL) {
        cg::cluster_group cl = cg::this_cluster();
        if (threadIdx.x == 0) cl_slot[p] = b;
        cl.sync();
        if (threadIdx.x < 32) {  // lane r reads rank r's partial; a fixed shuffle tree adds them
            const unsigned nb = cl.num_blocks();
            double acc = threadIdx.x < nb ? *cl.map_shared_rank(cl_slot + p, threadIdx.x) : 0.0;
            acc = warp_sum(acc);
            if (threadIdx.x == 0) *cl_out = acc;
        }
        __syncthreads();
        out = *cl_out;
        __syncthreads();
        return true;
    } else {
        double* pp = part + (size_t)p * gridDim.x;
        if (threadIdx.x == 0) pp[blockIdx.x] = b;
        if (!grid_sync(bar)) return false;
        out = reduce_partials(pp, gridDim.x, sh);
        return true;
    }
}

template <bool FP32, bool CL, bool SL = false>
__global__ void __launch_bounds__(kThreads, (CL || SL) ? 1 : 2) k_lanczos_block(const __grid_constant__ LzArgs a) {
    extern __shared__ double lz_dyn[];  // SL: the x slice and the row accumulators
    __shared__ double sh[32];
    __shared__ double cl_slot[2], cl_out;
    int par = 0;
    const int64_t n = a.n;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    const bool leader = (blockIdx.x == 0 && threadIdx.x == 0);

    // Every block starts from the state the host wrote.
    double rnm = a.st->rnm, tol = a.st->tol;
    int64_t ll = a.st->ll;
    int perm[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) perm[k] = a.st->perm[k];
    int eta_sel = a.st->eta_sel;
    int64_t npurge = a.st->npurge;
    bool resume = a.resume != 0;
    int64_t j = a.first;
    const double eps1 = a.eps1;
    const double sqrt_eps = a.sqrt_eps;  // of the run's scalar T

#define WV(k) (a.W[perm[k]])

    while (j < a.last) {
        double bet_j;
        if (!resume) {
            // mem::swap(w1, w2); mem::swap(w3, w4)
            int t = perm[1]; perm[1] = perm[2]; perm[2] = t;
            t = perm[3]; perm[3] = perm[4]; perm[4] = t;
            bet_j = rnm;  // wrk.bet[j] = rnm
            if (leader) a.bet[j] = bet_j;
            if (cmp_eq(rnm, 0.0)) {
                // invariant subspace: store q_{j-1}, p_{j-1} and hand over to the host's startv
                double* w2 = WV(2);
                double* w4 = WV(4);
                for (int64_t e = tid; e < n; e += nth) {
                    a.Q[(j - 1) * n + e] = w2[e];
                    if (j - 1 < 2) a.P[(j - 1) * n + e] = w4[e];
                }
                if (leader) {
                    a.st->status = 1;
                    a.st->j = j;
                    for (int k = 0; k < 7; ++k) a.st->perm[k] = perm[k];
                    a.st->rnm = rnm; a.st->tol = tol; a.st->ll = ll;
                    a.st->eta_sel = eta_sel; a.st->npurge = npurge;
                }
                if constexpr (CL) cg::this_cluster().sync();  // no block leaves while others may read its slots
                return;
            }
        } else {
            bet_j = a.bet[j];  // set before the host restart
        }

        // ---- phase 1: temp = op1 (w3 / rnm); w1 = w0 / rnm; w3' = w3 / rnm; store copies
        const double rinv = 1.0 / rnm;
        {
            const double* w0 = WV(0);
            const double* w2 = WV(2);
            const double* w3 = WV(3);
            const double* w4 = WV(4);
            double* w1 = WV(1);
            double* w3s = WV(6);
            spmv_rows<FP32, true, false, SL>(a.op1, w3, rinv, a.temp, 0.0, nullptr, nullptr, sh, lz_dyn);
            for (int64_t e = tid; e < n; e += nth) {
                w1[e] = mul_rn(rinv, w0[e]);
                w3s[e] = mul_rn(w3[e], rinv);
                if (!resume) {
                    a.Q[(j - 1) * n + e] = w2[e];
                    if (j - 1 < 2) a.P[(j - 1) * n + e] = w4[e];
                }
            }
            int t = perm[3]; perm[3] = perm[6]; perm[6] = t;
        }
        resume = false;
        if (!lz_sync<CL>(a.bar)) return;

        // ---- phase 2: w0 = op2 temp - rnm w2; alf[j] = w0 . w3
        double alf_j;
        {
            double part = spmv_rows<FP32, false, true, SL>(a.op2, a.temp, 1.0, WV(0), -rnm, WV(2), WV(3), sh, lz_dyn);
            if (!lz_sum<CL>(part, a.part, a.bar, sh, cl_slot, &cl_out, par, alf_j)) return;
        }

        // orthogonalise against the initial Lanczos vectors (mod.rs:722-731)
        if (j <= 2 && fabs(a.alf[j - 1]) > 4.0 * fabs(alf_j)) ll = j;
        const int64_t nloc = (j - 1 < ll) ? (j - 1) : ll;
        double* etaC = eta_sel ? a.etaB : a.etaA;  // eta
        double* etaO = eta_sel ? a.etaA : a.etaB;  // oldeta

        // ---- chain of (t = dot(w0, d); w0 -= t * u), fused pairwise
        double coef = alf_j;
        const double* axv = WV(1);
        for (int64_t step = 0; step < nloc + 2; ++step) {
            const double* dv = (step < nloc) ? (a.P + step * n) : (step == nloc ? WV(4) : WV(3));
            double* w0 = WV(0);
            double acc = 0.0;
            for (int64_t e = tid; e < n; e += nth) {
                const double v = add_rn(w0[e], mul_rn(-coef, axv[e]));
                w0[e] = v;
                acc = fma(v, dv[e], acc);
            }
            double t;
            if (!lz_sum<CL>(acc, a.part, a.bar, sh, cl_slot, &cl_out, par, t)) return;
            if (step < nloc) {
                if (leader) { etaC[step] = eps1; etaO[step] = eps1; }
                axv = a.Q + step * n;
            } else if (step == nloc) {
                if (bet_j > 0.0) bet_j += t;
                axv = WV(2);
            } else {
                alf_j += t;
                axv = WV(1);
            }
            coef = t;
        }
        {
            double* w0 = WV(0);
            double* w4 = WV(4);
            double acc = 0.0;
            for (int64_t e = tid; e < n; e += nth) {
                const double v = add_rn(w0[e], mul_rn(-coef, axv[e]));
                w0[e] = v;
                w4[e] = v;
                acc = fma(v, v, acc);
            }
            double s2;
            if (!lz_sum<CL>(acc, a.part, a.bar, sh, cl_slot, &cl_out, par, s2)) return;
            rnm = sqrt(s2);
        }
        if (leader) { a.alf[j] = alf_j; a.bet[j] = bet_j; }
        tol = sqrt_eps * (bet_j + fabs(alf_j) + rnm);

        // ---- ortbnd (mod.rs:815-838) and the purge test (mod.rs:768-770) in block 0
        if (blockIdx.x == 0) {
            __syncthreads();  // alf[j], bet[j] written by the leader
            if (!cmp_eq(rnm, 0.0) && j > 1) {
                for (int64_t i = threadIdx.x; i <= j - 2; i += blockDim.x) {
                    double v;
                    if (i == 0) {
                        v = sub_rn(add_rn(mul_rn(a.bet[1], etaC[1]), mul_rn(sub_rn(a.alf[0], a.alf[j]), etaC[0])),
                                   mul_rn(a.bet[j], etaO[0]));
                    } else {
                        v = sub_rn(add_rn(add_rn(mul_rn(a.bet[i + 1], etaC[i + 1]),
                                                 mul_rn(sub_rn(a.alf[i], a.alf[j]), etaC[i])),
                                          mul_rn(a.bet[i], etaC[i - 1])),
                                   mul_rn(a.bet[j], etaO[i]));
                    }
                    etaO[i] = add_rn(__ddiv_rn(v, rnm), eps1);
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) etaO[j - 1] = eps1;
            __syncthreads();
            // swap(oldeta, eta); eta[j] = eps1
            double* t = etaC; etaC = etaO; etaO = t;
            if (threadIdx.x == 0) etaC[j] = eps1;
            __syncthreads();
            if (j >= ll + 2) {
                // k = svd_idamax(step - (ll + 1), eta) + ll; purge if |eta[k]| > sqrt(eps).
                // idamax keeps the first index of the largest |eta[i]|, i in [0, cnt).
                const int64_t cnt = j - ll - 1;
                double best = -1.0;
                int64_t bi = 0;
                for (int64_t i = threadIdx.x; i < cnt; i += blockDim.x) {
                    const double v = fabs(etaC[i]);
                    if (v > best) { best = v; bi = i; }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                    const int64_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
                    if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
                }
                __shared__ double shb[32];
                __shared__ int64_t shi[32];
                if ((threadIdx.x & 31) == 0) { shb[threadIdx.x >> 5] = best; shi[threadIdx.x >> 5] = bi; }
                __syncthreads();
                if (threadIdx.x == 0) {
                    double b2 = shb[0];
                    int64_t i2 = shi[0];
                    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
                        if (shb[w] > b2 || (shb[w] == b2 && shi[w] < i2)) { b2 = shb[w]; i2 = shi[w]; }
                    a.st->purge_flag = fabs(etaC[i2 + ll]) > sqrt_eps;
                }
            } else if (threadIdx.x == 0) {
                a.st->purge_flag = 0;
            }
        } else {
            double* t = etaC; etaC = etaO; etaO = t;
        }
        eta_sel ^= 1;
        if (!lz_sync<CL>(a.bar)) return;
        const int do_purge = *(volatile int*)&a.st->purge_flag;

        if (do_purge) {
            // ---- purge (mod.rs:760-813): <= 2 sweeps of classical Gram-Schmidt
            // of q (w1, via w3) and r (w0, via w4) against q_ll .. q_{j-1}.
            ++npurge;
            const double reps1 = eps1 / sqrt_eps;
            const int64_t cnt = j - ll;
            int64_t nsplit = (n + 2047) / 2048;
            int64_t maxsplit = a.part_cap / (2 * cnt);
            if (nsplit > maxsplit) nsplit = maxsplit < 1 ? 1 : maxsplit;
            const int64_t chunk = (n + nsplit - 1) / nsplit;
            const int lane = threadIdx.x & 31;
            const int64_t gwarp = tid >> 5, nwarps = nth >> 5;
            for (int it = 0; it < 2; ++it) {
                if (!(rnm > tol)) continue;
                const double* w3 = WV(3);
                const double* w4 = WV(4);
                // dots Q[i] . w3 and Q[i] . w4 (the crate computes them before each
                // axpy, but w3 and w4 are not modified inside the loop)
                for (int64_t task = gwarp; task < cnt * nsplit; task += nwarps) {
                    const int64_t i = ll + task / nsplit, c = task % nsplit;
                    const int64_t e0 = c * chunk, e1 = (e0 + chunk < n) ? e0 + chunk : n;
                    const double* q = a.Q + i * n;
                    double sq = 0.0, sr = 0.0;
#pragma unroll 4
                    for (int64_t e = e0 + lane; e < e1; e += 32) {
                        const double qv = q[e];
                        sq = fma(qv, w3[e], sq);
                        sr = fma(qv, w4[e], sr);
                    }
                    sq = warp_sum(sq);
                    sr = warp_sum(sr);
                    if (lane == 0) { a.part[2 * task] = sq; a.part[2 * task + 1] = sr; }
                }
                if (!lz_sync<CL>(a.bar)) return;
                for (int64_t i = gwarp; i < cnt; i += nwarps) {
                    double sq = 0.0, sr = 0.0;
                    for (int64_t c = lane; c < nsplit; c += 32) {
                        sq += a.part[2 * (i * nsplit + c)];
                        sr += a.part[2 * (i * nsplit + c) + 1];
                    }
                    sq = warp_sum(sq);
                    sr = warp_sum(sr);
                    if (lane == 0) { a.tq[ll + i] = sq; a.tr[ll + i] = sr; }
                }
                if (!lz_sync<CL>(a.bar)) return;
                // tq = sum |t_q|, tr = sum |t_r|
                double aq = 0.0, ar = 0.0;
                for (int64_t i = threadIdx.x; i < cnt; i += blockDim.x) {
                    aq += fabs(a.tq[ll + i]);
                    ar += fabs(a.tr[ll + i]);
                }
                const double tq_sum = block_sum(aq, sh);
                double tr_sum = block_sum(ar, sh);
                // w1 -= sum_i tq_i q_i ; w0 -= sum_i tr_i q_i (in i order); w3 = w1
                double* w1 = WV(1);
                double* w0 = WV(0);
                double* w3w = WV(3);
                double acc = 0.0;
                for (int64_t e = tid; e < n; e += nth) {
                    double v1 = w1[e], v0 = w0[e];
                    // the crate's order over i (unfused multiply, then add); the
                    // loads of eight vectors are issued before their updates
                    int64_t i = ll;
                    for (; i + 8 <= j; i += 8) {
                        double qv[8], t1[8], t0[8];
#pragma unroll
                        for (int u = 0; u < 8; ++u) {
                            qv[u] = a.Q[(i + u) * n + e];
                            t1[u] = a.tq[i + u];
                            t0[u] = a.tr[i + u];
                        }
#pragma unroll
                        for (int u = 0; u < 8; ++u) {
                            v1 = add_rn(v1, mul_rn(-t1[u], qv[u]));
                            v0 = add_rn(v0, mul_rn(-t0[u], qv[u]));
                        }
                    }
                    for (; i < j; ++i) {
                        const double qv = a.Q[i * n + e];
                        v1 = add_rn(v1, mul_rn(-a.tq[i], qv));
                        v0 = add_rn(v0, mul_rn(-a.tr[i], qv));
                    }
                    w1[e] = v1;
                    w3w[e] = v1;
                    w0[e] = v0;
                    acc = fma(v0, v1, acc);
                }
                double t;
                if (!lz_sum<CL>(acc, a.part, a.bar, sh, cl_slot, &cl_out, par, t)) return;
                tr_sum += fabs(t);
                double* w4w = WV(4);
                double acc2 = 0.0;
                for (int64_t e = tid; e < n; e += nth) {
                    const double v = add_rn(w0[e], mul_rn(-t, w1[e]));
                    w0[e] = v;
                    w4w[e] = v;
                    acc2 = fma(v, v, acc2);
                }
                double s2;
                if (!lz_sum<CL>(acc2, a.part, a.bar, sh, cl_slot, &cl_out, par, s2)) return;
                rnm = sqrt(s2);
                if (tq_sum <= reps1 && tr_sum <= rnm * reps1) break;
            }
            if (blockIdx.x == 0) {
                for (int64_t i = ll + threadIdx.x; i <= j; i += blockDim.x) { etaC[i] = eps1; etaO[i] = eps1; }
            }
        }
        if (rnm <= tol) rnm = 0.0;
        ++j;
    }
    if (leader) {
        a.st->status = 0;
        a.st->j = j;
        for (int k = 0; k < 7; ++k) a.st->perm[k] = perm[k];
        a.st->rnm = rnm; a.st->tol = tol; a.st->ll = ll;
        a.st->eta_sel = eta_sel; a.st->npurge = npurge;
    }
    if constexpr (CL) cg::this_cluster().sync();  // no block leaves while others may read its slots
#undef WV
}

int lanczos_max_blocks(int threads) {
    int per_sm = 0;
    SVDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lanczos_block<false, false>, threads, 0));
    int per_sm32 = 0;
    SVDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm32, k_lanczos_block<true, false>, threads, 0));
    per_sm = per_sm < per_sm32 ? per_sm : per_sm32;
    if (per_sm < 1) per_sm = 1;
    return per_sm * device_props().sms;
}

// Blocks of the sliced cooperative grid: one per SM (the x slice takes most
// of the SM's shared memory).
int lanczos_sliced_blocks(int threads) {
    static std::once_flag attr;
    std::call_once(attr, [] {
        SVDB_CUDA(cudaFuncSetAttribute(k_lanczos_block<false, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kSlSmem));
        SVDB_CUDA(cudaFuncSetAttribute(k_lanczos_block<true, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kSlSmem));
    });
    int per_sm = 0, per_sm32 = 0;
    SVDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lanczos_block<false, false, true>, threads,
                                                            kSlSmem));
    SVDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm32, k_lanczos_block<true, false, true>, threads,
                                                            kSlSmem));
    per_sm = per_sm < per_sm32 ? per_sm : per_sm32;
    return per_sm >= 1 ? per_sm * device_props().sms : 0;
}

void launch_lanczos_block(const LzArgs& a, int blocks, int threads, int cluster, cudaStream_t s, bool sliced) {
    const bool fp32 = a.op1.vf != nullptr;
    if (sliced) {
        void* args[] = {(void*)&a};
        const void* fn = fp32 ? (const void*)k_lanczos_block<true, false, true>
                              : (const void*)k_lanczos_block<false, false, true>;
        SVDB_CUDA(cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(threads), args, kSlSmem, s));
        count_launches(1);
        return;
    }
    if (cluster > 0) {  // the whole grid is one cluster of `cluster` blocks
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(cluster);
        cfg.blockDim = dim3(threads);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if (fp32) SVDB_CUDA(cudaLaunchKernelEx(&cfg, k_lanczos_block<true, true>, a));
        else SVDB_CUDA(cudaLaunchKernelEx(&cfg, k_lanczos_block<false, true>, a));
    } else {
        void* args[] = {(void*)&a};
        const void* fn = fp32 ? (const void*)k_lanczos_block<true, false> : (const void*)k_lanczos_block<false, false>;
        SVDB_CUDA(cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(threads), args, 0, s));
    }
    count_launches(1);
}

// Whether a cluster of `cluster` blocks of `threads` threads can be resident
// (sizes above 8 are opted into per kernel).
bool lanczos_cluster_ok(int cluster, int threads) {
    if (cluster > 8) {
        if (cudaFuncSetAttribute(k_lanczos_block<false, true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                cudaSuccess ||
            cudaFuncSetAttribute(k_lanczos_block<true, true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                cudaSuccess) {
            cudaGetLastError();
            return false;
        }
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster);
    cfg.blockDim = dim3(threads);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0, n32 = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_lanczos_block<false, true>, &cfg) != cudaSuccess ||
        cudaOccupancyMaxActiveClusters(&n32, k_lanczos_block<true, true>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return n >= 1 && n32 >= 1;
}

}  // namespace svdb
