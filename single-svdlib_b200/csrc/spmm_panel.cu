// FP32 SpMM by panels of the dense operand: Y (rows x l, FP64) = M X, X
// (nminor x l, FP32, row-major), FP32 matrix values, l a multiple of 4 up to 64.
// The products of randomized_svd (masked.rs:265-733) under SVDB_MIXED.
//
// The row-gather kernel (spmm.cu) reads a 240-byte row of X from L2 for every
// nonzero: 65 M nonzeros move 15.6 GB per product although X is 7-24 MB.
// Here each CTA streams X once through shared memory instead, in panels of
// kPanelRows rows, and applies its rows' nonzeros to the panel there:
//   - a warp owns up to RW rows (slots) with FP32 accumulators in registers;
//     its four quarter-warps work on four slots at once, lane ql of a
//     quarter holding float4 columns ql and 8 + ql (two conflict-free 16-byte
//     shared-memory reads and eight FMAs per nonzero);
//   - the plan dealt rows to (virtual CTA, warp, slot) in snake order of
//     their lengths, so every warp gets about the same number of nonzeros, and
//     copied the nonzeros grouped by (virtual CTA, panel) -- a CTA panel --
//     and inside it by (warp, slot), with a table of slot offsets;
//   - per panel, one mbarrier covers three bulk asynchronous copies into one
//     of two shared-memory stages: the X panel, the CTA panel's entries and
//     its slot offsets, so the loop over a slot's entries reads shared memory
//     only; slots are visited in a fixed (unrolled) order;
//   - a slot's FP32 sum is added into its FP64 row of Y after at most
//     kPanelFlush terms and at the end;
//   - rows longer than a warp's share (`heavy`) keep the segment kernel.
// Waits on the stage mbarriers give up after 2 s of %globaltimer and raise
// g_panel_err (read by spmm_panel_check); the CTA then leaves its loop.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <string>

#include "device_common.cuh"
#include "ops.cuh"
#include "svdb_internal.h"

namespace svdb {

constexpr int kPanelRows = 256;   // rows of X per panel
constexpr int kPanelWarps = 16;   // warps per CTA
constexpr int kPanelMaxRw = 24;   // slots per warp: 6 per quarter-warp, 8 FP32 accumulators each per lane
constexpr int kPanelFlush = 512;  // FP32 terms of a slot before it is added into Y
constexpr uint64_t kPanelWaitNs = 2000000000ull;

__device__ int g_panel_err;

namespace {

__device__ __forceinline__ uint32_t pn_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint64_t pn_timer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool pn_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok = 0;
    const uint64_t t0 = pn_timer();
    while (true) {
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(ok)
                     : "r"(bar), "r"(parity)
                     : "memory");
        if (ok) return true;
        if (pn_timer() - t0 > kPanelWaitNs) return false;
    }
}
__device__ __forceinline__ void pn_bulk(void* dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     pn_smem(dst)),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

struct PanelArgs {
    const float* X;
    int64_t nx;  // rows of X
    int l;
    const uint64_t* ent;
    const int64_t* cbase;
    const int32_t* soff;
    int sstride;
    int64_t ecap;  // entries per stage
    const int32_t* slot_row;
    int vctas, npanels;
    double* Y;
};

// Shared memory: X panels [2] | entries [2] | slot offsets [2] | mbarriers [2]
struct PanelStage {
    unsigned char* base;
    uint32_t xsz, esz, osz;
    __device__ float* x(int b) const { return reinterpret_cast<float*>(base + b * xsz); }
    __device__ uint2* e(int b) const { return reinterpret_cast<uint2*>(base + 2 * xsz + b * esz); }
    __device__ int32_t* o(int b) const { return reinterpret_cast<int32_t*>(base + 2 * (xsz + esz) + b * osz); }
    __device__ uint64_t* bar() const { return reinterpret_cast<uint64_t*>(base + 2 * (xsz + esz + osz)); }
};

// Stage `it & 1` gets CTA panel `it` of this CTA: the X panel, its entries
// and its slot offsets (one thread).
__device__ __forceinline__ void pn_issue(const PanelArgs& a, const PanelStage& st, int it) {
    const int b = it & 1;
    const int p = it % a.npanels;
    const int64_t vc = (int64_t)blockIdx.x + (int64_t)(it / a.npanels) * gridDim.x;
    const int64_t cp = vc * a.npanels + p;
    const int64_t r0 = (int64_t)p * kPanelRows;
    const uint32_t xb = (uint32_t)(min((int64_t)kPanelRows, a.nx - r0) * a.l * 4);  // 16 | bytes: l % 4 == 0
    const int64_t e0 = __ldg(a.cbase + cp);
    int64_t ne = __ldg(a.cbase + cp + 1) - e0;  // even: CTA panels are padded
    if (ne > a.ecap || ne < 0) {                // the plan sized the stages; a mismatch is an error, not a copy
        atomicOr(&g_panel_err, 2);
        ne = 0;
    }
    const uint32_t eb = (uint32_t)(ne * 8), ob = (uint32_t)(a.sstride * 4);
    const uint32_t bar = pn_smem(st.bar() + b);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(xb + eb + ob) : "memory");
    pn_bulk(st.x(b), a.X + r0 * a.l, xb, bar);
    if (eb) pn_bulk(st.e(b), a.ent + e0, eb, bar);
    pn_bulk(st.o(b), a.soff + cp * a.sstride, ob, bar);
}

// Writes (first) or adds a slot's columns 4 ql .. 4 ql + 3 and 32 + 4 ql ..
// 32 + 4 ql + 3 (those below l) into its FP64 row of Y.
__device__ __forceinline__ void pn_store4(double* Y, int l, int row, bool first, int c, const float4& v) {
    if (c >= l) return;  // l % 4 == 0: a float4 column is wholly inside or outside
    double2* y = reinterpret_cast<double2*>(Y + (int64_t)row * l + c);
    double2 u = first ? make_double2(0.0, 0.0) : y[0];
    double2 w = first ? make_double2(0.0, 0.0) : y[1];
    u.x += (double)v.x;
    u.y += (double)v.y;
    w.x += (double)v.z;
    w.y += (double)v.w;
    y[0] = u;
    y[1] = w;
}
__device__ __forceinline__ void pn_store8(double* Y, int l, int row, bool first, int ql, const float4& c0,
                                          const float4& c1) {
    if (row < 0) return;
    pn_store4(Y, l, row, first, 4 * ql, c0);
    pn_store4(Y, l, row, first, 32 + 4 * ql, c1);
}

__device__ __forceinline__ void pn_fma(float4& ac, float v, const float4& x) {
    ac.x = fmaf(v, x.x, ac.x);
    ac.y = fmaf(v, x.y, ac.y);
    ac.z = fmaf(v, x.z, ac.z);
    ac.w = fmaf(v, x.w, ac.w);
}

template <int RQ>
__global__ void __launch_bounds__(kPanelWarps * 32, 1) k_spmm_panel(const __grid_constant__ PanelArgs a) {
    constexpr int RW = 4 * RQ;  // slots per warp
    extern __shared__ __align__(128) unsigned char sm_raw[];
    __shared__ int s_abort;
    PanelStage st;
    st.base = sm_raw;
    st.xsz = (uint32_t)kPanelRows * a.l * 4;
    st.esz = (uint32_t)a.ecap * 8;
    st.osz = (uint32_t)a.sstride * 4;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int qt = lane >> 3, ql = lane & 7;  // quarter of the warp, lane in it
    const int hq = a.l >> 2;                  // float4 columns of a row of X
    // float4 columns ql and 8 + ql of a row, kept inside the row (lanes past l read and discard)
    const int cq0 = min(ql, hq - 1), cq1 = min(8 + ql, hq - 1);
    const int nmine = (a.vctas - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
    const int total = nmine * a.npanels;
    if (total <= 0) return;
    if (tid == 0) {
        s_abort = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pn_smem(st.bar())) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pn_smem(st.bar() + 1)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int issued = 0, landed = 0;  // thread 0: stages issued and waited for
    if (tid == 0) {
        pn_issue(a, st, 0);
        issued = 1;
        if (total > 1) {
            pn_issue(a, st, 1);
            issued = 2;
        }
        if (pn_wait(pn_smem(st.bar()), 0)) {
            landed = 1;
        } else {
            s_abort = 1;
            atomicOr(&g_panel_err, 1);
        }
    }
    __syncthreads();

    // slot s = 4 t + q belongs to quarter q (lanes 8q .. 8q+7); lane ql of a
    // quarter holds float4 columns ql and 8 + ql of its RQ slots (each quarter
    // reads 128 contiguous bytes of a row per instruction: no bank conflicts)
    float4 acc[RQ][2];
    int row[RQ], cnt[RQ];
    unsigned flushed = 0;  // bit t: slot 4 t + q was written to Y before
    for (int it = 0; it < total; ++it) {
        if (s_abort) break;
        const int p = it % a.npanels;
        if (p == 0) {
            const int64_t vc = (int64_t)blockIdx.x + (int64_t)(it / a.npanels) * gridDim.x;
#pragma unroll
            for (int t = 0; t < RQ; ++t) {
                acc[t][0] = acc[t][1] = make_float4(0.f, 0.f, 0.f, 0.f);
                row[t] = __ldg(a.slot_row + (vc * kPanelWarps + w) * RW + 4 * t + qt);
                cnt[t] = 0;
            }
            flushed = 0;
        }
        const int b = it & 1;
        // every thread acquires the stage the barrier announced as complete
        if (!pn_wait(pn_smem(st.bar() + b), (it >> 1) & 1)) {
            s_abort = 1;
            atomicOr(&g_panel_err, 1);
        }
        const float4* X4 = reinterpret_cast<const float4*>(st.x(b));
        const uint2* E = st.e(b);
        const int32_t* O = st.o(b) + w * RW + qt;
#pragma unroll
        for (int t = 0; t < RQ; ++t) {
            const int o = O[4 * t], o1 = O[4 * t + 1];
            float4 c0 = acc[t][0], c1 = acc[t][1];
            int j = o;
            for (; j + 1 < o1; j += 2) {
                const uint2 e0 = E[j], e1 = E[j + 1];
                const float4* x0 = X4 + (int)e0.x * hq;
                const float4* x1 = X4 + (int)e1.x * hq;
                const float4 x00 = x0[cq0], x01 = x0[cq1], x10 = x1[cq0], x11 = x1[cq1];
                const float v0 = __uint_as_float(e0.y), v1 = __uint_as_float(e1.y);
                pn_fma(c0, v0, x00);
                pn_fma(c1, v0, x01);
                pn_fma(c0, v1, x10);
                pn_fma(c1, v1, x11);
            }
            if (j < o1) {
                const uint2 e0 = E[j];
                const float4* x0 = X4 + (int)e0.x * hq;
                const float v0 = __uint_as_float(e0.y);
                pn_fma(c0, v0, x0[cq0]);
                pn_fma(c1, v0, x0[cq1]);
            }
            cnt[t] += o1 - o;
            if (cnt[t] >= kPanelFlush) {  // this quarter only
                pn_store8(a.Y, a.l, row[t], !(flushed >> t & 1u), ql, c0, c1);
                c0 = c1 = make_float4(0.f, 0.f, 0.f, 0.f);
                cnt[t] = 0;
                flushed |= 1u << t;
            }
            acc[t][0] = c0;
            acc[t][1] = c1;
        }
        if (p == a.npanels - 1) {  // the virtual CTA's last panel: write every slot
#pragma unroll
            for (int t = 0; t < RQ; ++t) {
                const bool first = !(flushed >> t & 1u);
                if (first || cnt[t] > 0) pn_store8(a.Y, a.l, row[t], first, ql, acc[t][0], acc[t][1]);
            }
        }
        if (tid == 0 && it + 1 < total && !s_abort) {
            if (pn_wait(pn_smem(st.bar() + ((it + 1) & 1)), ((it + 1) >> 1) & 1)) {
                landed = it + 2;
            } else {
                s_abort = 1;
                atomicOr(&g_panel_err, 1);
            }
        }
        __syncthreads();  // stage it & 1 is free; stage (it + 1) & 1 is complete (or the CTA aborts)
        if (tid == 0 && it + 2 < total && !s_abort) {
            pn_issue(a, st, it + 2);
            issued = it + 3;
        }
    }
    if (tid == 0) {  // after an abort: let the copies still in flight land (bounded) before leaving
        for (int q2 = landed; q2 < issued; ++q2) pn_wait(pn_smem(st.bar() + (q2 & 1)), (q2 >> 1) & 1);
    }
}

// ------------------------------------------------------------- the plan --
__global__ void k_pn_lengths(const int64_t* __restrict__ rp, int64_t rows, int32_t* __restrict__ len,
                             int32_t* __restrict__ ids, int32_t* __restrict__ rinfo) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = rp[r + 1] - rp[r];
        len[r] = (int32_t)min(n, (int64_t)INT32_MAX);
        ids[r] = (int32_t)r;
        rinfo[r] = -1;
    }
}
__global__ void k_pn_count_heavy(const int32_t* __restrict__ len, int64_t rows, int64_t heavy,
                                 unsigned long long* __restrict__ n) {
    unsigned long long c = 0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x)
        c += (int64_t)len[r] > heavy ? 1 : 0;
    c = __reduce_add_sync(0xffffffffu, (unsigned)c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(n, c);
}
// sorted position q of the light rows (longest first) -> snake over the G warps
__global__ void k_pn_assign(const int32_t* __restrict__ sorted_rows, int64_t nheavy, int64_t nlight, int64_t G,
                            int rw, int32_t* __restrict__ slot_row, int32_t* __restrict__ rinfo) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nlight;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int32_t row = sorted_rows[nheavy + q];
        const int64_t round = q / G, pos = q % G;
        const int64_t gw = (round & 1) ? G - 1 - pos : pos;
        const int64_t slot = gw * rw + round;
        slot_row[slot] = row;
        rinfo[row] = (int32_t)slot;
    }
}
// One warp per light row: entries counted per (virtual CTA, panel, warp, slot)
// bucket (count pass), or copied to their place (fill pass): the CTA panel's
// base, the bucket's offset in it, and the rank among the bucket's entries.
// Lanes of a 32-entry chunk that share a bucket take consecutive places in
// lane order, chunks in order, so the copy is deterministic.
template <bool FILL>
__global__ void k_pn_bucket(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                            const float* __restrict__ v32, int64_t rows, const int32_t* __restrict__ rinfo, int rw,
                            int npanels, int32_t* __restrict__ cursor, const int64_t* __restrict__ cbase,
                            const int32_t* __restrict__ soff, int sstride, uint64_t* __restrict__ ent) {
    const int lane = threadIdx.x & 31;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t per_cp = (int64_t)kPanelWarps * rw;
    for (int64_t r = gwarp; r < rows; r += nwarps) {
        const int32_t info = rinfo[r];
        if (info < 0) continue;
        const int64_t gw = info / rw, slot = info % rw;
        const int64_t vc = gw / kPanelWarps, w = gw % kPanelWarps;
        const int64_t k_in_cp = w * rw + slot;
        for (int64_t k0 = rp[r]; k0 < rp[r + 1]; k0 += 32) {
            const int64_t k = k0 + lane;
            const bool ok = k < rp[r + 1];
            const unsigned act = __ballot_sync(0xffffffffu, ok);
            if (!ok) continue;
            const int c = ci[k];
            const int p = c / kPanelRows;
            const int64_t cp = vc * npanels + p;
            const int64_t b = cp * per_cp + k_in_cp;
            const unsigned peers = __match_any_sync(act, b);
            const int leader = __ffs(peers) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(cursor + b, __popc(peers));
            base = __shfl_sync(peers, base, leader);
            if (FILL) {
                const int64_t pos = cbase[cp] + soff[cp * sstride + k_in_cp] + base +
                                    __popc(peers & ((1u << lane) - 1u));
                ent[pos] = (uint64_t)(uint32_t)(c - p * kPanelRows) | ((uint64_t)__float_as_uint(v32[k]) << 32);
            }
        }
    }
}
// One warp per CTA panel: exclusive scan of its W * rw bucket counts into
// the slot offsets (plus the total at index W * rw); the padded total, even,
// goes to cpt for the scan of the CTA panel bases.
__global__ void k_pn_cp_scan(const int32_t* __restrict__ cnt, int64_t ncp, int per_cp, int sstride,
                             int32_t* __restrict__ soff, int64_t* __restrict__ cpt) {
    const int lane = threadIdx.x & 31;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t cp = gwarp; cp < ncp; cp += nwarps) {
        int carry = 0;
        for (int i0 = 0; i0 < per_cp; i0 += 32) {
            const int i = i0 + lane;
            const int v = i < per_cp ? cnt[cp * per_cp + i] : 0;
            int x = v;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, d);
                if (lane >= d) x += y;
            }
            if (i < per_cp) soff[cp * sstride + i] = carry + x - v;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
        if (lane == 0) {
            soff[cp * sstride + per_cp] = carry;
            cpt[cp] = (carry + 1) & ~1;
        }
    }
}
__global__ void k_pn_max(const int64_t* __restrict__ v, int64_t n, unsigned long long* __restrict__ mx) {
    unsigned long long m = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = max(m, (unsigned long long)v[i]);
    m = __reduce_max_sync(0xffffffffu, (unsigned)min(m, (unsigned long long)0xffffffffu));
    if ((threadIdx.x & 31) == 0) atomicMax(mx, m);
}
// heavy rows: their segments of the segment plan
__global__ void k_pn_heavy_flags(const int32_t* __restrict__ seg_row, int64_t nseg, const int64_t* __restrict__ rp,
                                 int64_t heavy, uint8_t* __restrict__ flag, int64_t* __restrict__ iota) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < nseg; s += (int64_t)gridDim.x * blockDim.x) {
        const int32_t rr = seg_row[s];
        const int64_t r = rr >= 0 ? rr : -(int64_t)rr - 1;
        flag[s] = (rp[r + 1] - rp[r]) > heavy ? 1 : 0;
        iota[s] = s;
    }
}
__global__ void k_pn_heavy_gather(const int64_t* __restrict__ sel, int64_t nh, const int32_t* __restrict__ seg_row,
                                  const int64_t* __restrict__ seg_beg, const int64_t* __restrict__ seg_end,
                                  int32_t* __restrict__ hrow, int64_t* __restrict__ hbeg, int64_t* __restrict__ hend) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nh; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = sel[t];
        const int32_t rr = seg_row[s];
        hrow[t] = rr >= 0 ? rr : -1;  // negative: a partial at t
        hbeg[t] = seg_beg[s];
        hend[t] = seg_end[s];
    }
}
// multi-segment heavy rows: first compact segment and count
__global__ void k_pn_heavy_multi(const int32_t* __restrict__ multi_rows, int64_t nmulti,
                                 const int64_t* __restrict__ seg_first, const int64_t* __restrict__ rp, int64_t heavy,
                                 const int64_t* __restrict__ cpos, int32_t* __restrict__ hm_row,
                                 int64_t* __restrict__ hm_first, int64_t* __restrict__ hm_count,
                                 unsigned long long* __restrict__ nh) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nmulti;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = multi_rows[t];
        if (rp[r + 1] - rp[r] <= heavy) continue;
        const unsigned long long q = atomicAdd(nh, 1ull);
        hm_row[q] = r;
        hm_first[q] = cpos[seg_first[r]];
        hm_count[q] = seg_first[r + 1] - seg_first[r];
    }
}
__global__ void k_pn_heavy_merge(const int32_t* __restrict__ hm_row, const int64_t* __restrict__ hm_first,
                                 const int64_t* __restrict__ hm_count, int64_t n, const double* __restrict__ part,
                                 int l, double* __restrict__ Y) {
    const int lane = threadIdx.x & 31;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t t = gwarp; t < n; t += nwarps) {
        const int64_t r = hm_row[t], f = hm_first[t], c = hm_count[t];
        for (int col = lane; col < l; col += 32) {
            double s = 0.0;
            for (int64_t q = 0; q < c; ++q) s += part[(f + q) * l + col];
            Y[r * l + col] = s;
        }
    }
}

int pn_blocks(int64_t work, int threads) {
    const int64_t b = (work + threads - 1) / threads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)device_props().sms * 16));
}

int pn_rw_template(int64_t rw) { return rw <= 8 ? 8 : rw <= 16 ? 16 : 24; }

}  // namespace

// Builds m.panel for the FP32 panel SpMM.  Needs the FP32 values and the
// segment plan; leaves usable = false when the shape does not suit it.
void build_panel_plan(DevCompressed& m, cudaStream_t s) {
    PanelPlan& pp = m.panel;
    pp.tried = true;
    pp.usable = false;
    const int64_t rows = m.nmajor, nnz = m.nnz;
    if (rows == 0 || nnz == 0 || !m.val32.p || m.nminor == 0 || m.nminor > (int64_t)INT32_MAX) return;
    const int sms = device_props().sms;
    const int64_t perv = (int64_t)kPanelWarps * kPanelMaxRw;
    const int64_t waves = std::max<int64_t>(1, (rows + (int64_t)sms * perv - 1) / ((int64_t)sms * perv));
    const int64_t vctas = (int64_t)sms * waves;
    const int64_t G = vctas * kPanelWarps;
    const int64_t heavy = std::max<int64_t>(kSegNnz, (nnz + G - 1) / G);
    const int64_t npanels = (m.nminor + kPanelRows - 1) / kPanelRows;
    // the plan lives as long as the structure: its buffers belong to the
    // owner's stream (the caller's stream may end first); each group is
    // allocated there and that stream synchronised before `s` uses it
    cudaStream_t os = m.owner_stream ? m.owner_stream : s;

    DevBuf<int32_t> len(rows, s), ids(rows, s), slen(rows, s), sids(rows, s), rinfo(rows, s);
    k_pn_lengths<<<pn_blocks(rows, 256), 256, 0, s>>>(m.ptr.p, rows, len.p, ids.p, rinfo.p);
    SVDB_CHECK_LAUNCH();
    size_t tb = 0;
    SVDB_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, len.p, slen.p, ids.p, sids.p, rows, 0, 32, s));
    DevBuf<uint8_t> tmp(std::max<size_t>(tb, 1), s);
    SVDB_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.p, tb, len.p, slen.p, ids.p, sids.p, rows, 0, 32, s));
    // heavy rows lead the descending order
    DevBuf<unsigned long long> nheavy_d(1, s);
    SVDB_CUDA(cudaMemsetAsync(nheavy_d.p, 0, sizeof(unsigned long long), s));
    k_pn_count_heavy<<<pn_blocks(rows, 256), 256, 0, s>>>(len.p, rows, heavy, nheavy_d.p);
    SVDB_CHECK_LAUNCH();
    unsigned long long nheavy_h = 0;
    SVDB_CUDA(cudaMemcpyAsync(&nheavy_h, nheavy_d.p, sizeof(nheavy_h), cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaStreamSynchronize(s));
    const int64_t nheavy = (int64_t)nheavy_h;
    pp.nlight = rows - nheavy;
    const int64_t rw_need = std::max<int64_t>(1, (pp.nlight + G - 1) / G);
    if (rw_need > kPanelMaxRw) return;
    const int rw = pn_rw_template(rw_need);
    const int64_t ncp = vctas * npanels, per_cp = (int64_t)kPanelWarps * rw;
    const int64_t nb = ncp * per_cp;
    if (nb > ((int64_t)1 << 31) || nnz > ((int64_t)1 << 31)) return;
    const int sstride = (int)((per_cp + 1 + 3) & ~(int64_t)3);  // 16-byte rows of slot offsets

    pp.slot_row.alloc(vctas * kPanelWarps * rw, os);
    pp.soff.alloc(ncp * sstride, os);
    pp.cbase.alloc(ncp + 1, os);
    SVDB_CUDA(cudaStreamSynchronize(os));
    SVDB_CUDA(cudaMemsetAsync(pp.slot_row.p, 0xFF, vctas * kPanelWarps * rw * sizeof(int32_t), s));
    SVDB_CUDA(cudaMemsetAsync(pp.soff.p, 0, ncp * sstride * sizeof(int32_t), s));
    if (pp.nlight > 0) {
        k_pn_assign<<<pn_blocks(pp.nlight, 256), 256, 0, s>>>(sids.p, nheavy, pp.nlight, G, rw, pp.slot_row.p,
                                                              rinfo.p);
        SVDB_CHECK_LAUNCH();
    }
    DevBuf<int32_t> cursor(nb, s);
    SVDB_CUDA(cudaMemsetAsync(cursor.p, 0, nb * sizeof(int32_t), s));
    k_pn_bucket<false><<<pn_blocks(rows * 32, 256), 256, 0, s>>>(m.ptr.p, m.idx.p, m.val32.p, rows, rinfo.p, rw,
                                                                  (int)npanels, cursor.p, nullptr, nullptr, 0,
                                                                  nullptr);
    SVDB_CHECK_LAUNCH();
    DevBuf<int64_t> cpt(ncp + 1, s);
    SVDB_CUDA(cudaMemsetAsync(cpt.p + ncp, 0, sizeof(int64_t), s));
    k_pn_cp_scan<<<pn_blocks(ncp * 32, 256), 256, 0, s>>>(cursor.p, ncp, (int)per_cp, sstride, pp.soff.p, cpt.p);
    SVDB_CHECK_LAUNCH();
    size_t tb2 = 0;
    SVDB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb2, cpt.p, pp.cbase.p, ncp + 1, s));
    DevBuf<uint8_t> tmp2(std::max<size_t>(tb2, 1), s);
    SVDB_CUDA(cub::DeviceScan::ExclusiveSum(tmp2.p, tb2, cpt.p, pp.cbase.p, ncp + 1, s));
    DevBuf<unsigned long long> mx(1, s);
    SVDB_CUDA(cudaMemsetAsync(mx.p, 0, sizeof(unsigned long long), s));
    k_pn_max<<<pn_blocks(ncp, 256), 256, 0, s>>>(cpt.p, ncp, mx.p);
    SVDB_CHECK_LAUNCH();
    int64_t nent = 0;
    unsigned long long emax = 0;
    SVDB_CUDA(cudaMemcpyAsync(&nent, pp.cbase.p + ncp, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaMemcpyAsync(&emax, mx.p, sizeof(emax), cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaMemsetAsync(cursor.p, 0, nb * sizeof(int32_t), s));
    SVDB_CUDA(cudaStreamSynchronize(s));
    pp.ecap = std::max<int64_t>(2, (int64_t)emax);
    pp.ent.alloc(std::max<int64_t>(nent, 2), os);
    SVDB_CUDA(cudaStreamSynchronize(os));
    k_pn_bucket<true><<<pn_blocks(rows * 32, 256), 256, 0, s>>>(m.ptr.p, m.idx.p, m.val32.p, rows, rinfo.p, rw,
                                                                 (int)npanels, cursor.p, pp.cbase.p, pp.soff.p,
                                                                 sstride, pp.ent.p);
    SVDB_CHECK_LAUNCH();
    pp.sstride = sstride;

    // heavy rows: their segments, compacted, and the rows to merge
    pp.nhseg = pp.nhmulti = 0;
    if (nheavy > 0) {
        const int64_t nseg = m.plan.nseg;
        DevBuf<uint8_t> flag(nseg, s);
        DevBuf<int64_t> iota(nseg, s), sel(nseg, s), cpos(nseg, s), nsel(1, s);
        k_pn_heavy_flags<<<pn_blocks(nseg, 256), 256, 0, s>>>(m.plan.seg_row.p, nseg, m.ptr.p, heavy, flag.p,
                                                             iota.p);
        SVDB_CHECK_LAUNCH();
        size_t tb3 = 0;
        SVDB_CUDA(cub::DeviceSelect::Flagged(nullptr, tb3, iota.p, flag.p, sel.p, nsel.p, nseg, s));
        size_t tb4 = 0;
        SVDB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb4, flag.p, cpos.p, nseg, s));
        DevBuf<uint8_t> tmp3(std::max<size_t>(std::max(tb3, tb4), 1), s);
        SVDB_CUDA(cub::DeviceSelect::Flagged(tmp3.p, tb3, iota.p, flag.p, sel.p, nsel.p, nseg, s));
        SVDB_CUDA(cub::DeviceScan::ExclusiveSum(tmp3.p, tb4, flag.p, cpos.p, nseg, s));
        SVDB_CUDA(cudaMemcpyAsync(&pp.nhseg, nsel.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
        pp.hseg_row.alloc(std::max<int64_t>(pp.nhseg, 1), os);
        pp.hseg_beg.alloc(std::max<int64_t>(pp.nhseg, 1), os);
        pp.hseg_end.alloc(std::max<int64_t>(pp.nhseg, 1), os);
        SVDB_CUDA(cudaStreamSynchronize(os));
        k_pn_heavy_gather<<<pn_blocks(pp.nhseg, 256), 256, 0, s>>>(sel.p, pp.nhseg, m.plan.seg_row.p,
                                                                   m.plan.seg_beg.p, m.plan.seg_end.p,
                                                                   pp.hseg_row.p, pp.hseg_beg.p, pp.hseg_end.p);
        SVDB_CHECK_LAUNCH();
        const int64_t nm = m.plan.nmulti;
        pp.hmulti_row.alloc(std::max<int64_t>(nm, 1), os);
        pp.hmulti_first.alloc(std::max<int64_t>(nm, 1), os);
        pp.hmulti_count.alloc(std::max<int64_t>(nm, 1), os);
        SVDB_CUDA(cudaStreamSynchronize(os));
        DevBuf<unsigned long long> nh(1, s);
        SVDB_CUDA(cudaMemsetAsync(nh.p, 0, sizeof(unsigned long long), s));
        if (nm > 0) {
            k_pn_heavy_multi<<<pn_blocks(nm, 256), 256, 0, s>>>(m.plan.multi_rows.p, nm, m.plan.seg_first.p, m.ptr.p,
                                                               heavy, cpos.p, pp.hmulti_row.p, pp.hmulti_first.p,
                                                               pp.hmulti_count.p, nh.p);
            SVDB_CHECK_LAUNCH();
        }
        unsigned long long hn = 0;
        SVDB_CUDA(cudaMemcpyAsync(&hn, nh.p, sizeof(hn), cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
        pp.nhmulti = (int64_t)hn;
    }
    SVDB_CUDA(cudaStreamSynchronize(s));
    pp.rw = rw;
    pp.vctas = (int)vctas;
    pp.npanels = (int)npanels;
    pp.heavy = heavy;
    pp.usable = true;
}

// Opt-in (SVDB_SPMM=panel, read on every call).  On B200, for the 100,000 x
// 30,000 count-like matrix (65 M nonzeros, l = 60), one product took 1.47 ms
// for A Z and 2.77 ms for A^T Y, against 2.25 ms with the segment kernel.
// The staging alone (copies and barriers, compute left out) took 0.35 and
// 0.54 ms.  A^T Y is held by per-panel imbalance: its rows (columns of A)
// have very skewed lengths, and a panel step waits for the warp whose long
// row occupies one quarter.  Building the plan takes about 4 ms per
// structure, which a call on a new handle pays.
bool spmm_panel_eligible(const DevCompressed& m, int l, const void* X) {
    const char* e = getenv("SVDB_SPMM");
    if (!e || std::string(e) != "panel") return false;
    if (l < 4 || l > 64 || l % 4 != 0 || (reinterpret_cast<uintptr_t>(X) % 16) != 0) return false;
    return m.val32.p && m.nnz > 0 && m.nmajor > 0;
}

// Y (FP64) = M X through the panel plan (built on first use).  Returns false
// when the plan is not usable for M; the caller then takes the segment kernel.
bool spmm_panel(DevCompressed& m, const float* X, int l, double* Y, cudaStream_t s,
                void (*heavy_segments)(const DevCompressed&, const int32_t*, const int64_t*, const int64_t*, int64_t,
                                       const float*, int, double*, double*, cudaStream_t)) {
    if (!m.panel.tried) build_panel_plan(m, s);
    const PanelPlan& pp = m.panel;
    if (!pp.usable) return false;
    const size_t smem =
        2 * ((size_t)kPanelRows * l * 4 + (size_t)pp.ecap * 8 + (size_t)pp.sstride * 4) + 2 * sizeof(uint64_t);
    if (smem > device_props().smem_optin) return false;  // a CTA panel too large for two stages
    PanelArgs a;
    a.X = X;
    a.nx = m.nminor;
    a.l = l;
    a.ent = pp.ent.p;
    a.cbase = pp.cbase.p;
    a.soff = pp.soff.p;
    a.sstride = pp.sstride;
    a.ecap = pp.ecap;
    a.slot_row = pp.slot_row.p;
    a.vctas = pp.vctas;
    a.npanels = pp.npanels;
    a.Y = Y;
    const int grid = std::min(pp.vctas, device_props().sms);
    switch (pp.rw) {
#define SVDB_PANEL_LAUNCH(RQ)                                                                                   \
    case 4 * RQ:                                                                                                \
        SVDB_CUDA(cudaFuncSetAttribute(k_spmm_panel<RQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
        k_spmm_panel<RQ><<<grid, kPanelWarps * 32, smem, s>>>(a);                                               \
        break;
        SVDB_PANEL_LAUNCH(2)
        SVDB_PANEL_LAUNCH(4)
        SVDB_PANEL_LAUNCH(6)
#undef SVDB_PANEL_LAUNCH
        default:
            throw Error(SVDB_ERR_CUDA, "panel SpMM: unexpected slot count");
    }
    SVDB_CHECK_LAUNCH();
    if (pp.nhseg > 0) {
        DevBuf<double> part(std::max<int64_t>(pp.nhseg * l, 1), s);
        heavy_segments(m, pp.hseg_row.p, pp.hseg_beg.p, pp.hseg_end.p, pp.nhseg, X, l, Y, part.p, s);
        if (pp.nhmulti > 0) {
            k_pn_heavy_merge<<<pn_blocks(pp.nhmulti * 32, 256), 256, 0, s>>>(
                pp.hmulti_row.p, pp.hmulti_first.p, pp.hmulti_count.p, pp.nhmulti, part.p, l, Y);
            SVDB_CHECK_LAUNCH();
        }
    }
    return true;
}

void spmm_panel_check() {
    int e = 0;
    SVDB_CUDA(cudaMemcpyFromSymbol(&e, g_panel_err, sizeof(int)));
    if (e) {
        const int z = 0;
        SVDB_CUDA(cudaMemcpyToSymbol(g_panel_err, &z, sizeof(int)));
        if (e & 2) throw Error(SVDB_ERR_CUDA, "SpMM: a CTA panel larger than its shared-memory stage");
        throw Error(SVDB_ERR_TIMEOUT, "SpMM: a panel copy did not complete within 2 s");
    }
}

}  // namespace svdb
