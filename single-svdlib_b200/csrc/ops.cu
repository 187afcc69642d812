// Standalone device operators: SpMV row gathers, deterministic
// reductions, element-wise BLAS-1 (src/lanczos/mod.rs:311-424), classical
// Gram-Schmidt GEMV pairs for startv (mod.rs:624-628), the ChaCha12 start
// vector (mod.rs:598-605) and dense transposes.
#include <algorithm>
#include <cstdlib>
#include <string>

#include "device_common.cuh"
#include "ops.cuh"
#include "spmv.cuh"
#include "svdb_internal.h"

namespace svdb {

static int blocks_for(int64_t work, int threads, int per_sm = 8) {
    int64_t b = (work + threads - 1) / threads;
    int64_t cap = (int64_t)device_props().sms * per_sm;
    return (int)std::max<int64_t>(1, std::min(b, cap));
}

int group_for(double avg) {
    int g = 1;
    while (g < 32 && g < avg) g <<= 1;
    return g < 2 ? 2 : g;
}

// --------------------------------------------------------------- SpMV ----
// One launch: every block first takes its share of the rows of more than
// kSegNnz entries (one block per row, the plan's multi rows), then its warps
// take the other rows through the length bins.  The grid is one wave of
// resident blocks, so the two parts overlap and no partial wave trails.
template <typename VT>
__global__ void __launch_bounds__(256) k_spmv(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                              const VT* __restrict__ v, const __grid_constant__ SpmvBins bins,
                                              const int32_t* __restrict__ long_rows, int64_t nlong,
                                              const double* __restrict__ x, double* __restrict__ y) {
    __shared__ double sh[32];
    auto xl = [&](int32_t c) { return __ldg(x + c); };
    for (int64_t i = blockIdx.x; i < nlong; i += gridDim.x) {
        const int64_t r = long_rows[i];
        const double acc = row_dot(ci, v, rp[r], rp[r + 1], (int)threadIdx.x, (int)blockDim.x, xl);
        const double tot = block_sum(acc, sh);
        if (threadIdx.x == 0) y[r] = tot;
    }
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    spmv_binned(rp, ci, v, bins, gwarp, nwarps, xl, [&](int64_t r, double acc) { y[r] = acc; });
}

// The column-sliced kernel is opt-in (SVDB_SPMV=sliced): on the 1M x 200k
// LAS2 matrix its short per-slice row pieces left it slower than the gather
// kernel (2.2 against 0.94 ms for A x).
static bool sliced_off() {
    const char* e = getenv("SVDB_SPMV");
    return !(e && std::string(e) == "sliced");
}

// One resident wave of k_spmv<VT> on the current device.  The occupancy is
// cached per thread and device, like device_props().
template <typename VT>
static int spmv_grid() {
    static thread_local int cached_dev = -1;
    static thread_local int per_sm = 0;
    int dev = 0;
    SVDB_CUDA(cudaGetDevice(&dev));
    if (dev != cached_dev) {
        SVDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spmv<VT>, 256, 0));
        if (per_sm < 1) per_sm = 1;
        cached_dev = dev;
    }
    return per_sm * device_props().sms;
}

void spmv(const DevCompressed& m, bool fp32, const double* x, double* y, cudaStream_t s, bool allow_sliced) {
    if (m.nmajor == 0) return;
    const bool f = fp32 && m.val32.p;
    if (allow_sliced && !sliced_off() && spmv_sliced(m, f, x, y, s)) return;
    const int64_t work = std::max<int64_t>(m.plan.bins.items[kSpmvBins] / 8, m.plan.nmulti);
    if (f) {
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(work, spmv_grid<float>()));
        k_spmv<float><<<blocks, 256, 0, s>>>(m.ptr.p, m.idx.p, m.val32.p, m.plan.bins, m.plan.multi_rows.p,
                                             m.plan.nmulti, x, y);
    } else {
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(work, spmv_grid<double>()));
        k_spmv<double><<<blocks, 256, 0, s>>>(m.ptr.p, m.idx.p, m.val.p, m.plan.bins, m.plan.multi_rows.p,
                                              m.plan.nmulti, x, y);
    }
    SVDB_CHECK_LAUNCH();
}

// --------------------------------------------------------- reductions ----
constexpr int kRedBlocks = 256;
constexpr int kRedThreads = 256;

size_t reduce_scratch_doubles() { return kRedBlocks + 8; }

__global__ void __launch_bounds__(kRedThreads) k_dot_part(const double* __restrict__ x, const double* __restrict__ y,
                                                          int64_t n, double* __restrict__ part) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc = fma(x[i], y[i], acc);
    double b = block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = b;
}

__global__ void __launch_bounds__(kRedThreads) k_reduce(const double* __restrict__ part, int np, double* out) {
    __shared__ double sh[32];
    double r = reduce_partials(part, np, sh);
    if (threadIdx.x == 0) *out = r;
}

void dot(const double* x, const double* y, int64_t n, double* d_out, double* scratch, cudaStream_t s) {
    // fixed grid: the summation order does not depend on the device
    k_dot_part<<<kRedBlocks, kRedThreads, 0, s>>>(x, y, n, scratch);
    k_reduce<<<1, kRedThreads, 0, s>>>(scratch, kRedBlocks, d_out);
    SVDB_CHECK_LAUNCH_N(2);
}

double dot_host(const double* x, const double* y, int64_t n, double* scratch, cudaStream_t s) {
    dot(x, y, n, scratch + kRedBlocks, scratch, s);
    double h = 0.0;
    SVDB_CUDA(cudaMemcpyAsync(&h, scratch + kRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, s));
    SVDB_CUDA(cudaStreamSynchronize(s));
    return h;
}

// ------------------------------------------------------------ BLAS-1 ----
__global__ void k_axpy(double a, const double* __restrict__ x, double* __restrict__ y, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = add_rn(y[i], mul_rn(a, x[i]));
}
__global__ void k_scal(double a, double* __restrict__ x, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = mul_rn(x[i], a);
}
__global__ void k_datx(double a, const double* __restrict__ x, double* __restrict__ y, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = mul_rn(a, x[i]);
}

void axpy(double a, const double* x, double* y, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_axpy<<<blocks_for(n, 256), 256, 0, s>>>(a, x, y, n);
    SVDB_CHECK_LAUNCH();
}
void scal(double a, double* x, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_scal<<<blocks_for(n, 256), 256, 0, s>>>(a, x, n);
    SVDB_CHECK_LAUNCH();
}
void datx(double a, const double* x, double* y, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_datx<<<blocks_for(n, 256), 256, 0, s>>>(a, x, y, n);
    SVDB_CHECK_LAUNCH();
}
void copy(const double* x, double* y, int64_t n, cudaStream_t s) {
    if (n <= 0 || x == y) return;
    SVDB_CUDA(cudaMemcpyAsync(y, x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
}

__global__ void k_narrow(const double* __restrict__ x, float* __restrict__ y, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = __double2float_rn(x[i]);
}
__global__ void k_widen(const float* __restrict__ x, double* __restrict__ y, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = (double)x[i];
}
__global__ void k_round_f32(double* __restrict__ x, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = (double)__double2float_rn(x[i]);
}
void narrow(const double* x, float* y, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_narrow<<<blocks_for(n, 256), 256, 0, s>>>(x, y, n);
    SVDB_CHECK_LAUNCH();
}
void widen(const float* x, double* y, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_widen<<<blocks_for(n, 256), 256, 0, s>>>(x, y, n);
    SVDB_CHECK_LAUNCH();
}
void round_f32(double* x, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_round_f32<<<blocks_for(n, 256), 256, 0, s>>>(x, n);
    SVDB_CHECK_LAUNCH();
}

// ------------------------------------------------------- CGS helpers ----
// t[i] = Q[i0+i] . x; block (split, i) partials then an ordered reduction.
__global__ void __launch_bounds__(256) k_gemv_t_part(const double* __restrict__ Q, int64_t n, int64_t i0,
                                                     const double* __restrict__ x, int64_t chunk,
                                                     double* __restrict__ part, int nsplit) {
    __shared__ double sh[32];
    const int64_t i = blockIdx.y;
    const int64_t e0 = blockIdx.x * chunk, e1 = std::min<int64_t>(n, e0 + chunk);
    const double* q = Q + (i0 + i) * n;
    double acc = 0.0;
    for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) acc = fma(q[e], x[e], acc);
    double b = block_sum(acc, sh);
    if (threadIdx.x == 0) part[i * nsplit + blockIdx.x] = b;
}
__global__ void __launch_bounds__(32) k_gemv_t_red(const double* __restrict__ part, int nsplit, int64_t cnt,
                                                   double* __restrict__ t) {
    const int64_t i = blockIdx.x;
    double acc = 0.0;
    for (int c = threadIdx.x; c < nsplit; c += 32) acc += part[i * nsplit + c];
    acc = warp_sum(acc);
    if (threadIdx.x == 0) t[i] = acc;
}

void gemv_t(const double* Q, int64_t n, int64_t i0, int64_t cnt, const double* x, double* t, double* scratch,
            int64_t scratch_cap, cudaStream_t s) {
    if (cnt <= 0) return;
    int nsplit = (int)std::max<int64_t>(1, std::min<int64_t>((n + 8191) / 8192, scratch_cap / cnt));
    int64_t chunk = (n + nsplit - 1) / nsplit;
    int64_t y0 = 0;
    while (y0 < cnt) {  // gridDim.y <= 65535
        int64_t cy = std::min<int64_t>(cnt - y0, 65535);
        k_gemv_t_part<<<dim3(nsplit, (unsigned)cy), 256, 0, s>>>(Q, n, i0 + y0, x, chunk, scratch, nsplit);
        k_gemv_t_red<<<(unsigned)cy, 32, 0, s>>>(scratch, nsplit, cy, t + y0);
        SVDB_CHECK_LAUNCH_N(2);
        y0 += cy;
    }
}

// y[e] = y[e] + (-t[i]) * Q[i0+i][e], i ascending (the crate's axpy sequence)
__global__ void k_gemv_sub(const double* __restrict__ Q, int64_t n, int64_t i0, int64_t cnt,
                           const double* __restrict__ t, double* __restrict__ y) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        double v = y[e];
        for (int64_t i = 0; i < cnt; ++i) v = add_rn(v, mul_rn(-t[i], Q[(i0 + i) * n + e]));
        y[e] = v;
    }
}

void gemv_sub(const double* Q, int64_t n, int64_t i0, int64_t cnt, const double* t, double* y, cudaStream_t s) {
    if (cnt <= 0 || n <= 0) return;
    k_gemv_sub<<<blocks_for(n, 256), 256, 0, s>>>(Q, n, i0, cnt, t, y);
    SVDB_CHECK_LAUNCH();
}

// ------------------------------------------------------ start vector ----
// Value v uses u64 draw v = words (2v, 2v+1) of the ChaCha12 keystream with
// key = seed bytes (u32 little endian, rest zero), counter from 0, stream 0:
// one thread per 64-byte block, 8 values each.  round_f32: each value is
// rounded to f32, as T::from_f64 does for T = f32 (src/lanczos/mod.rs:604-606).
__global__ void k_start_vector(uint32_t seed, double* __restrict__ w, int64_t n, int round_f32) {
    const int64_t nblk = (n + 7) / 8;
    uint32_t key[8] = {seed, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nblk; b += (int64_t)gridDim.x * blockDim.x) {
        uint32_t out[16];
        chacha_block_dev(key, (uint64_t)b, 12, out);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int64_t i = b * 8 + q;
            if (i < n) {
                const uint64_t u = (uint64_t)out[2 * q] | ((uint64_t)out[2 * q + 1] << 32);
                const double v = uniform_pm1_dev(u);
                w[i] = round_f32 ? (double)__double2float_rn(v) : v;
            }
        }
    }
}

void start_vector(uint32_t seed, double* w, int64_t n, cudaStream_t s, bool round_f32) {
    if (n <= 0) return;
    k_start_vector<<<blocks_for((n + 7) / 8, 128), 128, 0, s>>>(seed, w, n, round_f32 ? 1 : 0);
    SVDB_CHECK_LAUNCH();
}

// ------------------------------------------------------ dense helpers ----
// out (cols x rows) = in (rows x cols)^T, both row-major
template <typename T>
__global__ void k_transpose(const T* __restrict__ in, T* __restrict__ out, int64_t rows, int64_t cols) {
    __shared__ T tile[32][33];
    const int64_t tcols = (cols + 31) / 32, tiles = ((rows + 31) / 32) * tcols;
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int64_t bx = (t % tcols) * 32, by = (t / tcols) * 32;
        __syncthreads();
        for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
            const int64_t r = by + yy, c = bx + threadIdx.x;
            if (r < rows && c < cols) tile[yy][threadIdx.x] = in[r * cols + c];
        }
        __syncthreads();
        for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
            const int64_t c = bx + yy, r = by + threadIdx.x;
            if (r < rows && c < cols) out[c * rows + r] = tile[threadIdx.x][yy];
        }
    }
}

template <typename T>
void transpose_dense(const T* in, T* out, int64_t rows, int64_t cols, cudaStream_t s) {
    if (rows <= 0 || cols <= 0) return;
    const int64_t tiles = ((rows + 31) / 32) * ((cols + 31) / 32);
    const int blocks = (int)std::min<int64_t>(tiles, (int64_t)device_props().sms * 16);
    k_transpose<T><<<blocks, dim3(32, 8), 0, s>>>(in, out, rows, cols);
    SVDB_CHECK_LAUNCH();
}
template void transpose_dense<double>(const double*, double*, int64_t, int64_t, cudaStream_t);
template void transpose_dense<float>(const float*, float*, int64_t, int64_t, cudaStream_t);

}  // namespace svdb
