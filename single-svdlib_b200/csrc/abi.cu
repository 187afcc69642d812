// extern "C" entry points of libsvdb200 (include/svdb200.h).
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <string>

#include "ops.cuh"
#include "svdb_internal.h"

namespace svdb {
svdb_matrix* create_csr(uint64_t, uint64_t, uint64_t, const uint64_t*, const uint64_t*, const double*, const float*);
svdb_matrix* create_csc(uint64_t, uint64_t, uint64_t, const uint64_t*, const uint64_t*, const double*, const float*);
svdb_matrix* create_coo(uint64_t, uint64_t, uint64_t, const uint64_t*, const uint64_t*, const double*, const float*);
svdb_matrix* create_csr_device(uint64_t, uint64_t, uint64_t, const int64_t*, const int32_t*, const double*);
svdb_matrix* masked_new(const svdb_matrix*, const uint8_t*, uint64_t);
void masked_maps(const svdb_matrix*, int64_t*, int64_t*);
void destroy(svdb_matrix*);
void las2(const svdb_matrix*, uint64_t, uint64_t, const double[2], double, uint32_t, bool, const svdb_options&,
          svdb_rec*, bool);
int las2_plan(uint64_t, uint64_t, uint64_t, uint64_t, uint64_t, uint64_t*, uint64_t*, int32_t*, int32_t*);
void randomized(const svdb_matrix*, uint64_t, uint64_t, uint64_t, int, int, int, uint64_t, int,
                const svdb_options&, svdb_rec*, bool);
void svd_adjoint(const svdb_matrix*, int64_t, const double*, const double*, const double*, const double*,
                 const double*, const double*, svdb_adjoint_options&, double*);
void sddmm_device(const svdb_matrix*, const void*, const void*, int64_t, void*, int, cudaStream_t);
void svd_flip(double*, int64_t, int64_t, double*, int64_t, int64_t, bool, bool);
void release_cached_memory();
void gram_device(const double*, int64_t, int, double*, int, cudaStream_t);
void batch_create(const svdb_matrix*, const uint64_t*, const uint64_t*, uint64_t, uint64_t, uint64_t, uint64_t, int, int,
                  uint64_t, const svdb_batch_options&, svdb_batch**);
void batch_run(svdb_batch*, svdb_rec*);
void batch_info(const svdb_batch*, svdb_batch_info*);
const svdb_matrix* batch_matrix(const svdb_batch*);
void batch_destroy(svdb_batch*);

static thread_local std::string g_last_error;
void set_last_error(const std::string& m) { g_last_error = m; }

static std::atomic<uint64_t> g_launches{0};
void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void discount_launches(uint64_t n) { g_launches.fetch_sub(n, std::memory_order_relaxed); }

// Runs `f`, mapping exceptions to status codes and the thread's last error.
template <typename F>
static int guarded(F&& f) {
    try {
        f();
        return SVDB_OK;
    } catch (Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return SVDB_ERR_OOM;
    } catch (std::exception& e) {
        g_last_error = e.what();
        return SVDB_ERR_ARG;
    }
}

struct DeviceGuard {  // runs a call on the handle's device
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) SVDB_CUDA(cudaSetDevice(dev));
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

static svdb_options opts_or_default(const svdb_options* o) {
    svdb_options d;
    svdb_options_default(&d);
    return o ? *o : d;
}

static void check_handle(const svdb_matrix* a) {
    if (!a) throw Error(SVDB_ERR_ARG, "null matrix handle");
}

}  // namespace svdb

using namespace svdb;

extern "C" {

void svdb_options_default(svdb_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->precision = SVDB_F64;
    o->algorithm = SVDB_LANCZOS;
}

const char* svdb_last_error_message(void) { return g_last_error.c_str(); }
int svdb_version(void) { return 10009; }

int svdb_matrix_create_csr(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* indptr,
                           const uint64_t* indices, const double* values, svdb_matrix** out) {
    return guarded([&] {
        if (!out) throw Error(SVDB_ERR_ARG, "null out");
        *out = create_csr(nrows, ncols, nnz, indptr, indices, values, nullptr);
    });
}
int svdb_matrix_create_csr_f32(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* indptr,
                               const uint64_t* indices, const float* values,
                               svdb_matrix** out) {
    return guarded([&] {
        if (!out) throw Error(SVDB_ERR_ARG, "null out");
        *out = create_csr(nrows, ncols, nnz, indptr, indices, nullptr, values);
    });
}
int svdb_matrix_create_csc(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* colptr,
                           const uint64_t* rowidx, const double* values, svdb_matrix** out) {
    return guarded([&] {
        if (!out) throw Error(SVDB_ERR_ARG, "null out");
        *out = create_csc(nrows, ncols, nnz, colptr, rowidx, values, nullptr);
    });
}
int svdb_matrix_create_csc_f32(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* colptr,
                               const uint64_t* rowidx, const float* values,
                               svdb_matrix** out) {
    return guarded([&] {
        if (!out) throw Error(SVDB_ERR_ARG, "null out");
        *out = create_csc(nrows, ncols, nnz, colptr, rowidx, nullptr, values);
    });
}
int svdb_matrix_create_coo(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* rows, const uint64_t* cols,
                           const double* values, svdb_matrix** out) {
    return guarded([&] {
        if (!out) throw Error(SVDB_ERR_ARG, "null out");
        *out = create_coo(nrows, ncols, nnz, rows, cols, values, nullptr);
    });
}
int svdb_matrix_create_coo_f32(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* rows,
                               const uint64_t* cols, const float* values,
                               svdb_matrix** out) {
    return guarded([&] {
        if (!out) throw Error(SVDB_ERR_ARG, "null out");
        *out = create_coo(nrows, ncols, nnz, rows, cols, nullptr, values);
    });
}
int svdb_matrix_create_csr_device(uint64_t nrows, uint64_t ncols, uint64_t nnz, const int64_t* d_indptr,
                                  const int32_t* d_indices, const double* d_values, svdb_matrix** out) {
    return guarded([&] {
        if (!out || !d_indptr || (nnz && (!d_indices || !d_values))) throw Error(SVDB_ERR_ARG, "null argument");
        *out = create_csr_device(nrows, ncols, nnz, d_indptr, d_indices, d_values);
    });
}
void svdb_matrix_destroy(svdb_matrix* a) {
    if (!a) return;
    guarded([&] {
        DeviceGuard g(a->device);
        destroy(a);
    });
}
uint64_t svdb_matrix_nrows(const svdb_matrix* a) { return a ? a->nrows : 0; }
uint64_t svdb_matrix_ncols(const svdb_matrix* a) { return a ? a->ncols : 0; }
uint64_t svdb_matrix_nnz(const svdb_matrix* a) { return a ? a->nnz : 0; }

int svdb_masked_new(const svdb_matrix* csr, const uint8_t* column_mask, uint64_t mask_len, svdb_matrix** out) {
    return guarded([&] {
        check_handle(csr);
        if (!out) throw Error(SVDB_ERR_ARG, "null out");
        DeviceGuard g(csr->device);
        *out = masked_new(csr, column_mask, mask_len);
    });
}
int svdb_masked_with_columns(const svdb_matrix* csr, const uint64_t* columns, uint64_t ncolumns,
                             svdb_matrix** out) {
    return guarded([&] {
        check_handle(csr);
        if (!out || (ncolumns && !columns)) throw Error(SVDB_ERR_ARG, "null argument");
        std::vector<uint8_t> mask((size_t)csr->ncols, 0);  // masked.rs:48-55
        for (uint64_t k = 0; k < ncolumns; ++k) {
            if (columns[k] >= (uint64_t)csr->ncols) throw Error(SVDB_ERR_SHAPE, "Column index out of bounds");
            mask[columns[k]] = 1;
        }
        DeviceGuard g(csr->device);
        *out = masked_new(csr, mask.data(), mask.size());
    });
}
int svdb_masked_maps(const svdb_matrix* m, int64_t* m2o, int64_t* o2m) {
    return guarded([&] {
        check_handle(m);
        if (!m2o || !o2m) throw Error(SVDB_ERR_ARG, "null argument");
        DeviceGuard g(m->device);
        masked_maps(m, m2o, o2m);
    });
}
int svdb_masked_uses_all_columns(const svdb_matrix* m) {
    if (!m || m->kind != KIND_MASKED) return -1;
    return m->all_columns ? 1 : 0;
}

int svdb_opa(const svdb_matrix* a, const double* x, double* y, int transposed) {
    return guarded([&] {
        check_handle(a);
        if (!x || !y) throw Error(SVDB_ERR_ARG, "null argument");
        svdb_matrix* am = const_cast<svdb_matrix*>(a);
        std::lock_guard<std::mutex> lk(am->mu);
        DeviceGuard g(a->device);
        cudaStream_t s = a->stream;
        const DevCompressed& op = transposed ? csc_of(a) : csr_of(a);
        DevBuf<double> dx(std::max<int64_t>(op.nminor, 1), s), dy(std::max<int64_t>(op.nmajor, 1), s);
        SVDB_CUDA(cudaMemcpyAsync(dx.p, x, op.nminor * 8, cudaMemcpyHostToDevice, s));
        spmv(op, false, dx.p, dy.p, s);
        SVDB_CUDA(cudaMemcpyAsync(y, dy.p, op.nmajor * 8, cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
    });
}
int svdb_opb(const svdb_matrix* a, const double* x, double* y, int transposed) {
    return guarded([&] {
        check_handle(a);
        if (!x || !y) throw Error(SVDB_ERR_ARG, "null argument");
        svdb_matrix* am = const_cast<svdb_matrix*>(a);
        std::lock_guard<std::mutex> lk(am->mu);
        DeviceGuard g(a->device);
        cudaStream_t s = a->stream;
        const DevCompressed& o1 = transposed ? csc_of(a) : csr_of(a);
        const DevCompressed& o2 = transposed ? csr_of(a) : csc_of(a);
        DevBuf<double> dx(std::max<int64_t>(o1.nminor, 1), s), dt(std::max<int64_t>(o1.nmajor, 1), s),
            dy(std::max<int64_t>(o2.nmajor, 1), s);
        SVDB_CUDA(cudaMemcpyAsync(dx.p, x, o1.nminor * 8, cudaMemcpyHostToDevice, s));
        spmv(o1, false, dx.p, dt.p, s);
        spmv(o2, false, dt.p, dy.p, s);
        SVDB_CUDA(cudaMemcpyAsync(y, dy.p, o2.nmajor * 8, cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
    });
}
int svdb_multiply_with_dense(const svdb_matrix* a, const double* dense, uint64_t l, double* result,
                             int transpose_self) {
    return guarded([&] {
        check_handle(a);
        if (!dense || !result) throw Error(SVDB_ERR_ARG, "null argument");
        svdb_matrix* am = const_cast<svdb_matrix*>(a);
        std::lock_guard<std::mutex> lk(am->mu);
        DeviceGuard g(a->device);
        cudaStream_t s = a->stream;
        const DevCompressed& op = transpose_self ? csc_of(a) : csr_of(a);
        DevBuf<double> dx(std::max<int64_t>(op.nminor * l, 1), s), dy(std::max<int64_t>(op.nmajor * l, 1), s);
        SVDB_CUDA(cudaMemcpyAsync(dx.p, dense, op.nminor * l * 8, cudaMemcpyHostToDevice, s));
        spmm_dev<double, double>(op, false, dx.p, (int)l, dy.p, s);
        SVDB_CUDA(cudaMemcpyAsync(result, dy.p, op.nmajor * l * 8, cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
    });
}
int svdb_opa_device(const svdb_matrix* a, const double* d_x, double* d_y, int transposed, int precision,
                    void* stream) {
    return guarded([&] {
        check_handle(a);
        if (!d_x || !d_y) throw Error(SVDB_ERR_ARG, "null argument");
        if (precision != SVDB_F64 && precision != SVDB_MIXED) throw Error(SVDB_ERR_ARG, "bad precision");
        DeviceGuard g(a->device);
        const DevCompressed& op = transposed ? csc_of(a) : csr_of(a);
        if (precision == SVDB_MIXED && !op.val32.p) {
            svdb_matrix* am = const_cast<svdb_matrix*>(a);
            std::lock_guard<std::mutex> lk(am->mu);
            ensure_fp32(a);
        }
        spmv(op, precision == SVDB_MIXED, d_x, d_y, stream ? (cudaStream_t)stream : a->stream);
    });
}

int svdb_multiply_with_dense_device(const svdb_matrix* a, const void* d_dense, uint64_t l, void* d_result,
                                    int transpose_self, int precision, void* stream) {
    return guarded([&] {
        check_handle(a);
        if (!d_dense || !d_result) throw Error(SVDB_ERR_ARG, "null argument");
        if (precision != SVDB_F64 && precision != SVDB_MIXED) throw Error(SVDB_ERR_ARG, "bad precision");
        DeviceGuard g(a->device);
        cudaStream_t s = stream ? (cudaStream_t)stream : a->stream;
        const DevCompressed& op = transpose_self ? csc_of(a) : csr_of(a);
        if (precision == SVDB_F64) {
            spmm_dev<double, double>(op, false, (const double*)d_dense, (int)l, (double*)d_result, s);
        } else {
            if (!op.val32.p) {
                svdb_matrix* am = const_cast<svdb_matrix*>(a);
                std::lock_guard<std::mutex> lk(am->mu);
                ensure_fp32(a);
                SVDB_CUDA(cudaStreamSynchronize(a->stream));
            }
            if (dense_split_usable(a, (int)l)) {
                dense_split_spmm<float, float>(a, transpose_self != 0, (const float*)d_dense, (const float*)d_dense,
                                               (int)l, (float*)d_result, s);
                dense_split_check();
            } else {
                spmm_dev<float, float>(op, true, (const float*)d_dense, (int)l, (float*)d_result, s);
            }
        }
    });
}

uint64_t svdb_kernel_launches(void) { return g_launches.load(); }

int svdb_sliced_spmv_info(const svdb_matrix* a, int transposed, int32_t* nslices, int32_t* nranges) {
    return guarded([&] {
        check_handle(a);
        if (!nslices || !nranges) throw Error(SVDB_ERR_ARG, "null argument");
        sliced_info(transposed ? csc_of(a) : csr_of(a), nslices, nranges);
    });
}

int svdb_dense_split_info(const svdb_matrix* a, uint64_t* dense_cols, uint64_t* dense_nnz) {
    return guarded([&] {
        check_handle(a);
        if (!dense_cols || !dense_nnz) throw Error(SVDB_ERR_ARG, "null argument");
        dense_split_info(a, dense_cols, dense_nnz);
    });
}

int svdb_multiply_transposed_by_dense(const svdb_matrix* a, const double* q, uint64_t l, double* result) {
    return guarded([&] {
        check_handle(a);
        if (!q || !result) throw Error(SVDB_ERR_ARG, "null argument");
        svdb_matrix* am = const_cast<svdb_matrix*>(a);
        std::lock_guard<std::mutex> lk(am->mu);
        DeviceGuard g(a->device);
        cudaStream_t s = a->stream;
        const DevCompressed& op = csc_of(a);  // (Q^T A)^T = A^T Q
        DevBuf<double> dq(std::max<int64_t>(op.nminor * l, 1), s), dz(std::max<int64_t>(op.nmajor * l, 1), s),
            dr(std::max<int64_t>(op.nmajor * l, 1), s);
        SVDB_CUDA(cudaMemcpyAsync(dq.p, q, op.nminor * l * 8, cudaMemcpyHostToDevice, s));
        spmm_dev<double, double>(op, false, dq.p, (int)l, dz.p, s);
        transpose_dense<double>(dz.p, dr.p, op.nmajor, (int64_t)l, s);
        SVDB_CUDA(cudaMemcpyAsync(result, dr.p, op.nmajor * l * 8, cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
    });
}

int svdb_column_means(const svdb_matrix* a, double* means) {
    return guarded([&] {
        check_handle(a);
        if (!means) throw Error(SVDB_ERR_ARG, "null argument");
        svdb_matrix* am = const_cast<svdb_matrix*>(a);
        std::lock_guard<std::mutex> lk(am->mu);
        DeviceGuard g(a->device);
        cudaStream_t s = a->stream;
        const DevCompressed& t = csc_of(a);
        DevBuf<double> mu(std::max<int64_t>(t.nmajor, 1), s);
        column_means_dev(t, a->nrows, mu.p, s);
        if (t.nmajor) SVDB_CUDA(cudaMemcpyAsync(means, mu.p, t.nmajor * 8, cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
    });
}

int svdb_multiply_with_dense_centered(const svdb_matrix* a, const double* dense, uint64_t l, const double* means,
                                      double* result, int transpose_self) {
    return guarded([&] {
        check_handle(a);
        if (!dense || !result || !means) throw Error(SVDB_ERR_ARG, "null argument");
        svdb_matrix* am = const_cast<svdb_matrix*>(a);
        std::lock_guard<std::mutex> lk(am->mu);
        DeviceGuard g(a->device);
        cudaStream_t s = a->stream;
        const DevCompressed& op = transpose_self ? csc_of(a) : csr_of(a);
        DevBuf<double> dx(std::max<int64_t>(op.nminor * l, 1), s), dy(std::max<int64_t>(op.nmajor * l, 1), s),
            mu(std::max<int64_t>(a->ncols, 1), s);
        SVDB_CUDA(cudaMemcpyAsync(dx.p, dense, op.nminor * l * 8, cudaMemcpyHostToDevice, s));
        SVDB_CUDA(cudaMemcpyAsync(mu.p, means, a->ncols * 8, cudaMemcpyHostToDevice, s));
        spmm_dev<double, double>(op, false, dx.p, (int)l, dy.p, s);
        center_product(dx.p, op.nminor, (int)l, mu.p, dy.p, op.nmajor, !transpose_self, s);
        SVDB_CUDA(cudaMemcpyAsync(result, dy.p, op.nmajor * l * 8, cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
    });
}

int svdb_multiply_transposed_by_dense_centered(const svdb_matrix* a, const double* q, uint64_t l, const double* means,
                                               double* result) {
    return guarded([&] {
        check_handle(a);
        if (!q || !result || !means) throw Error(SVDB_ERR_ARG, "null argument");
        svdb_matrix* am = const_cast<svdb_matrix*>(a);
        std::lock_guard<std::mutex> lk(am->mu);
        DeviceGuard g(a->device);
        cudaStream_t s = a->stream;
        const DevCompressed& op = csc_of(a);  // (Q^T (A - 1 mu^T))^T = A^T Q - mu (1^T Q)
        DevBuf<double> dq(std::max<int64_t>(op.nminor * l, 1), s), dz(std::max<int64_t>(op.nmajor * l, 1), s),
            dr(std::max<int64_t>(op.nmajor * l, 1), s), mu(std::max<int64_t>(a->ncols, 1), s);
        SVDB_CUDA(cudaMemcpyAsync(dq.p, q, op.nminor * l * 8, cudaMemcpyHostToDevice, s));
        SVDB_CUDA(cudaMemcpyAsync(mu.p, means, a->ncols * 8, cudaMemcpyHostToDevice, s));
        spmm_dev<double, double>(op, false, dq.p, (int)l, dz.p, s);
        center_product(dq.p, op.nminor, (int)l, mu.p, dz.p, op.nmajor, false, s);
        transpose_dense<double>(dz.p, dr.p, op.nmajor, (int64_t)l, s);
        SVDB_CUDA(cudaMemcpyAsync(result, dr.p, op.nmajor * l * 8, cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
    });
}

static int las2_common(const svdb_matrix* a, uint64_t dimensions, uint64_t iterations, const double end_interval[2],
                       double kappa, uint32_t seed, const svdb_options* opts, svdb_rec* out, int force_legacy) {
    return guarded([&] {
        check_handle(a);
        if (!out) throw Error(SVDB_ERR_ARG, "null out");
        const double ei_default[2] = {-1.0e-30, 1.0e-30};
        const double* ei = end_interval ? end_interval : ei_default;
        svdb_options o = opts_or_default(opts);
        bool legacy = force_legacy || o.algorithm == SVDB_LEGACY;
        svdb_matrix* am = const_cast<svdb_matrix*>(a);
        std::lock_guard<std::mutex> lk(am->mu);
        DeviceGuard g(a->device);
        las2(a, dimensions, iterations, ei, kappa, seed, legacy, o, out, false);
    });
}

int svdb_las2(const svdb_matrix* a, uint64_t dimensions, uint64_t iterations, const double end_interval[2],
              double kappa, uint32_t random_seed, const svdb_options* opts, svdb_rec* out) {
    return las2_common(a, dimensions, iterations, end_interval, kappa, random_seed, opts, out, 0);
}
int svdb_svd(const svdb_matrix* a, svdb_rec* out) {
    return las2_common(a, 0, 0, nullptr, 1.0e-6, 0, nullptr, out, 0);
}
int svdb_svd_dim(const svdb_matrix* a, uint64_t dimensions, svdb_rec* out) {
    return las2_common(a, dimensions, 0, nullptr, 1.0e-6, 0, nullptr, out, 0);
}
int svdb_svd_dim_seed(const svdb_matrix* a, uint64_t dimensions, uint32_t random_seed, svdb_rec* out) {
    return las2_common(a, dimensions, 0, nullptr, 1.0e-6, random_seed, nullptr, out, 0);
}
int svdb_legacy_svd_las2(const svdb_matrix* a, uint64_t dimensions, uint64_t iterations,
                         const double end_interval[2], double kappa, uint32_t random_seed,
                         const svdb_options* opts, svdb_rec* out) {
    return las2_common(a, dimensions, iterations, end_interval, kappa, random_seed, opts, out, 1);
}

int svdb_start_vector(uint32_t seed, double* out, uint64_t n) {
    return guarded([&] {
        if (!out && n) throw Error(SVDB_ERR_ARG, "null out");
        cudaStream_t s = nullptr;
        SVDB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            DevBuf<double> w(std::max<uint64_t>(n, 1), s);
            start_vector(seed, w.p, (int64_t)n, s);
            if (n) SVDB_CUDA(cudaMemcpyAsync(out, w.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
            SVDB_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        cudaStreamDestroy(s);
    });
}

int svdb_las2_plan(uint64_t nrows, uint64_t ncols, uint64_t nnz, uint64_t dimensions, uint64_t iterations,
                   uint64_t* dimensions_out, uint64_t* iterations_out, int32_t* transposed_out,
                   int32_t* sparsity_branch_out) {
    return guarded([&] {
        las2_plan(nrows, ncols, nnz, dimensions, iterations, dimensions_out, iterations_out, transposed_out,
                  sparsity_branch_out);
    });
}

int svdb_randomized_svd(const svdb_matrix* a, uint64_t target_rank, uint64_t n_oversamples, uint64_t n_power_iters,
                        int normalizer, int mean_center, int has_seed, uint64_t seed, int verbose,
                        const svdb_options* opts, svdb_rec* out) {
    return guarded([&] {
        check_handle(a);
        if (!out) throw Error(SVDB_ERR_ARG, "null out");
        if (normalizer < 0 || normalizer > 2) throw Error(SVDB_ERR_ARG, "bad normalizer");
        svdb_options o = opts_or_default(opts);
        svdb_matrix* am = const_cast<svdb_matrix*>(a);
        std::lock_guard<std::mutex> lk(am->mu);
        DeviceGuard g(a->device);
        randomized(a, target_rank, n_oversamples, n_power_iters, normalizer, mean_center, has_seed, seed, verbose,
                   o, out, false);
    });
}

// ---- T = f32 entry points: the solver runs with its results in HBM, which
// are then narrowed to f32 (round to nearest) into the caller's record.
extern "C++" {
template <typename Solve>
static int solve_f32(const svdb_matrix* a, const svdb_options* opts, svdb_rec_f32* out, Solve&& solve) {
    return guarded([&] {
        check_handle(a);
        if (!out) throw Error(SVDB_ERR_ARG, "null out");
        svdb_options o = opts_or_default(opts);
        const bool host = !o.result_on_device;
        o.result_on_device = 1;
        cudaStream_t s = o.stream ? (cudaStream_t)o.stream : a->stream;
        svdb_rec r;
        std::memset(&r, 0, sizeof r);
        std::memset(out, 0, sizeof(*out));
        svdb_matrix* am = const_cast<svdb_matrix*>(a);
        std::lock_guard<std::mutex> lk(am->mu);
        DeviceGuard g(a->device);
        solve(o, &r);
        struct Owned {  // the f64 device record, released stream-ordered on every path
            svdb_rec* r;
            cudaStream_t s;
            ~Owned() {
                for (double* q : {r->u, r->s, r->vt})
                    if (q) cudaFreeAsync(q, s);
            }
        } owned{&r, s};
        const int64_t nu = (int64_t)(r.u_rows * r.u_cols), nv = (int64_t)(r.vt_rows * r.vt_cols), ns = (int64_t)r.d;
        DevBuf<float> u(std::max<int64_t>(nu, 1), s), sv(std::max<int64_t>(ns, 1), s), vt(std::max<int64_t>(nv, 1), s);
        narrow(r.u, u.p, nu, s);
        narrow(r.s, sv.p, ns, s);
        narrow(r.vt, vt.p, nv, s);
        out->d = r.d;
        out->u_rows = r.u_rows; out->u_cols = r.u_cols;
        out->vt_rows = r.vt_rows; out->vt_cols = r.vt_cols;
        out->diagnostics = r.diagnostics;
        out->origin = r.origin;
        out->time_ms_total = r.time_ms_total;
        out->time_ms_spmv = r.time_ms_spmv;
        out->time_ms_ortho = r.time_ms_ortho;
        out->time_ms_tridiag = r.time_ms_tridiag;
        out->time_ms_ritvec = r.time_ms_ritvec;
        if (!host) {
            SVDB_CUDA(cudaStreamSynchronize(s));
            out->u = u.detach(); out->s = sv.detach(); out->vt = vt.detach();
            out->on_device = 1;
            return;
        }
        out->u = (float*)host_result_alloc(std::max<int64_t>(nu, 1) * sizeof(float));
        out->s = (float*)host_result_alloc(std::max<int64_t>(ns, 1) * sizeof(float));
        out->vt = (float*)host_result_alloc(std::max<int64_t>(nv, 1) * sizeof(float));
        if (nu) SVDB_CUDA(cudaMemcpyAsync(out->u, u.p, nu * sizeof(float), cudaMemcpyDeviceToHost, s));
        if (ns) SVDB_CUDA(cudaMemcpyAsync(out->s, sv.p, ns * sizeof(float), cudaMemcpyDeviceToHost, s));
        if (nv) SVDB_CUDA(cudaMemcpyAsync(out->vt, vt.p, nv * sizeof(float), cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
        out->on_device = 0;
    });
}
}  // extern "C++"

int svdb_las2_f32(const svdb_matrix* a, uint64_t dimensions, uint64_t iterations, const float end_interval[2],
                  float kappa, uint32_t random_seed, const svdb_options* opts, svdb_rec_f32* out) {
    return solve_f32(a, opts, out, [&](const svdb_options& o, svdb_rec* r) {
        if (o.algorithm == SVDB_LEGACY) throw Error(SVDB_ERR_UNSUPPORTED, "legacy::svdLAS2 is f64-only");
        const double ei[2] = {end_interval ? (double)end_interval[0] : (double)-1.0e-30f,
                              end_interval ? (double)end_interval[1] : (double)1.0e-30f};
        las2(a, dimensions, iterations, ei, (double)kappa, random_seed, false, o, r, true);
    });
}
int svdb_svd_f32(const svdb_matrix* a, svdb_rec_f32* out) {
    return svdb_las2_f32(a, 0, 0, nullptr, 1.0e-6f, 0, nullptr, out);
}
int svdb_svd_dim_f32(const svdb_matrix* a, uint64_t dimensions, svdb_rec_f32* out) {
    return svdb_las2_f32(a, dimensions, 0, nullptr, 1.0e-6f, 0, nullptr, out);
}
int svdb_svd_dim_seed_f32(const svdb_matrix* a, uint64_t dimensions, uint32_t random_seed, svdb_rec_f32* out) {
    return svdb_las2_f32(a, dimensions, 0, nullptr, 1.0e-6f, random_seed, nullptr, out);
}
int svdb_randomized_svd_f32(const svdb_matrix* a, uint64_t target_rank, uint64_t n_oversamples,
                            uint64_t n_power_iters, int normalizer, int mean_center, int has_seed, uint64_t seed,
                            int verbose, const svdb_options* opts, svdb_rec_f32* out) {
    return solve_f32(a, opts, out, [&](const svdb_options& o, svdb_rec* r) {
        if (normalizer < 0 || normalizer > 2) throw Error(SVDB_ERR_ARG, "bad normalizer");
        randomized(a, target_rank, n_oversamples, n_power_iters, normalizer, mean_center, has_seed, seed, verbose,
                   o, r, true);
    });
}

void svdb_rec_f32_free(svdb_rec_f32* r) {
    if (!r) return;
    if (r->on_device) {
        cudaFree(r->u);
        cudaFree(r->s);
        cudaFree(r->vt);
    } else {
        host_result_free(r->u);
        host_result_free(r->s);
        host_result_free(r->vt);
    }
    std::memset(r, 0, sizeof(*r));
}

void svdb_rec_free(svdb_rec* r) {
    if (!r) return;
    if (r->on_device) {
        cudaFree(r->u);
        cudaFree(r->s);
        cudaFree(r->vt);
    } else {
        host_result_free(r->u);
        host_result_free(r->s);
        host_result_free(r->vt);
    }
    std::memset(r, 0, sizeof(*r));
}

int svdb_rec_recompose(const svdb_rec* r, double* out) {
    return guarded([&] {
        if (!r || !out) throw Error(SVDB_ERR_ARG, "null argument");
        if (r->on_device) throw Error(SVDB_ERR_UNSUPPORTED, "recompose of a device-resident record");
        const uint64_t n = r->vt_cols, d = r->d;
        if (r->origin == SVDB_REC_LEGACY) {  // ut.t() . diag(s) . vt
            const uint64_t m = r->u_cols;
            for (uint64_t i = 0; i < m; ++i)
                for (uint64_t j = 0; j < n; ++j) {
                    double acc = 0.0;
                    for (uint64_t k = 0; k < d; ++k) acc += r->u[k * m + i] * r->s[k] * r->vt[k * n + j];
                    out[i * n + j] = acc;
                }
            return;
        }
        // u . diag(s) . vt exactly as written; ndarray requires u_cols == len(s)
        if (r->u_cols != d)
            throw Error(SVDB_ERR_SHAPE, "ndarray: inputs " + std::to_string(r->u_rows) + " x " +
                                            std::to_string(r->u_cols) + " and " + std::to_string(d) + " x " +
                                            std::to_string(d) + " are not compatible for matrix multiplication");
        const uint64_t m = r->u_rows;
        for (uint64_t i = 0; i < m; ++i)
            for (uint64_t j = 0; j < n; ++j) {
                double acc = 0.0;
                for (uint64_t k = 0; k < d; ++k) acc += r->u[i * d + k] * r->s[k] * r->vt[k * n + j];
                out[i * n + j] = acc;
            }
    });
}

void svdb_adjoint_options_default(svdb_adjoint_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->precision = SVDB_F64;
    o->cg_tol = 1e-12;
    o->cg_max_iters = 5000;
}

int svdb_svd_adjoint(const svdb_matrix* a, uint64_t k, const double* u, const double* s, const double* v,
                     const double* g_u, const double* g_s, const double* g_v, svdb_adjoint_options* opts,
                     double* grad_values) {
    return guarded([&] {
        check_handle(a);
        svdb_adjoint_options d;
        svdb_adjoint_options_default(&d);
        svdb_adjoint_options& o = opts ? *opts : d;
        if (o.precision != SVDB_F64 && o.precision != SVDB_MIXED) throw Error(SVDB_ERR_ARG, "bad precision");
        svdb_matrix* am = const_cast<svdb_matrix*>(a);
        std::lock_guard<std::mutex> lk(am->mu);
        DeviceGuard g(a->device);
        svd_adjoint(a, (int64_t)k, u, s, v, g_u, g_s, g_v, o, grad_values);
    });
}

int svdb_sddmm_device(const svdb_matrix* a, const void* d_left, const void* d_right, uint64_t rank, void* d_out,
                      int precision, void* stream) {
    return guarded([&] {
        check_handle(a);
        if (!d_left || !d_right || !d_out) throw Error(SVDB_ERR_ARG, "null argument");
        if (precision != SVDB_F64 && precision != SVDB_MIXED) throw Error(SVDB_ERR_ARG, "bad precision");
        DeviceGuard g(a->device);
        sddmm_device(a, d_left, d_right, (int64_t)rank, d_out, precision, stream ? (cudaStream_t)stream : a->stream);
    });
}

void svdb_batch_options_default(svdb_batch_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->precision = SVDB_MIXED;
    o->autotune = 1;
    o->use_graph = 1;
}

int svdb_batch_create(const svdb_matrix* a, const uint64_t* col_offsets, const uint64_t* columns, uint64_t count,
                      uint64_t target_rank, uint64_t n_oversamples, uint64_t n_power_iters, int normalizer,
                      int has_seed, uint64_t seed, const svdb_batch_options* opts, svdb_batch** out) {
    return guarded([&] {
        check_handle(a);
        if (!out) throw Error(SVDB_ERR_ARG, "null out");
        svdb_batch_options o;
        svdb_batch_options_default(&o);
        if (opts) o = *opts;
        if (o.precision != SVDB_F64 && o.precision != SVDB_MIXED) throw Error(SVDB_ERR_ARG, "bad precision");
        svdb_matrix* am = const_cast<svdb_matrix*>(a);
        std::lock_guard<std::mutex> lk(am->mu);
        DeviceGuard g(a->device);
        batch_create(a, col_offsets, columns, count, target_rank, n_oversamples, n_power_iters, normalizer, has_seed,
                     seed, o, out);
    });
}

int svdb_batch_run(svdb_batch* b, svdb_rec* outs) {
    return guarded([&] {
        if (!b) throw Error(SVDB_ERR_ARG, "null batch");
        svdb_matrix* am = const_cast<svdb_matrix*>(batch_matrix(b));
        std::lock_guard<std::mutex> lk(am->mu);
        DeviceGuard g(am->device);
        batch_run(b, outs);
    });
}

int svdb_batch_get_info(const svdb_batch* b, svdb_batch_info* info) {
    return guarded([&] {
        if (!b || !info) throw Error(SVDB_ERR_ARG, "null argument");
        batch_info(b, info);
    });
}

void svdb_batch_destroy(svdb_batch* b) {
    if (!b) return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(batch_matrix(b)->device);
    batch_destroy(b);
    if (prev >= 0) cudaSetDevice(prev);
}

int svdb_randomized_svd_batch(const svdb_matrix* a, const uint64_t* col_offsets, const uint64_t* columns,
                              uint64_t count, uint64_t target_rank, uint64_t n_oversamples, uint64_t n_power_iters,
                              int normalizer, int has_seed, uint64_t seed, const svdb_batch_options* opts,
                              svdb_rec* outs) {
    svdb_batch* b = nullptr;
    int st = svdb_batch_create(a, col_offsets, columns, count, target_rank, n_oversamples, n_power_iters, normalizer,
                               has_seed, seed, opts, &b);
    if (st != SVDB_OK) return st;
    st = svdb_batch_run(b, outs);
    svdb_batch_destroy(b);
    return st;
}

int svdb_gram_device(const double* d_x, uint64_t rows, uint64_t c, double* d_g, int precision, void* stream) {
    return guarded([&] {
        if (!d_x || !d_g) throw Error(SVDB_ERR_ARG, "null argument");
        if (precision != SVDB_F64 && precision != SVDB_MIXED) throw Error(SVDB_ERR_ARG, "bad precision");
        gram_device(d_x, (int64_t)rows, (int)c, d_g, precision, (cudaStream_t)stream);
    });
}

int svdb_release_cached_memory(void) {
    return guarded([&] { release_cached_memory(); });
}

int svdb_svd_flip(double* u, uint64_t u_rows, uint64_t u_cols, double* v, uint64_t v_rows, uint64_t v_cols,
                  int u_based_decision, int on_device) {
    return guarded([&] {
        svd_flip(u, (int64_t)u_rows, (int64_t)u_cols, v, (int64_t)v_rows, (int64_t)v_cols, u_based_decision != 0,
                 on_device != 0);
    });
}

}  // extern "C"
