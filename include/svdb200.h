/*
 * svdb200.h -- C ABI of the B200 implementation of single-svdlib's hot path.
 *
 * The boundary is the reference crate's public API (single-svdlib 1.0.9):
 * one call here per Rust entry point, with plain pointers and sizes.  Each
 * declaration names the reference item it replaces (paths relative to the
 * crate root).  All dense arrays are row-major.  Host arrays passed in are
 * borrowed for the duration of the call only (the crate's &CsrMatrix borrow);
 * results are allocated by the library and released with svdb_rec_free.
 *
 * Errors: every entry point returns an svdb_status.  SvdLibError variants map
 * one to one (src/error.rs:4-21); conditions the crate reports by panicking
 * (assert!, todo!) return SVDB_ERR_SHAPE / SVDB_ERR_UNSUPPORTED.  The message
 * of the last error on the calling thread is svdb_last_error_message().
 *
 * Threading: a matrix handle is bound to the CUDA device that was current when
 * it was created.  Calls on different handles may run concurrently from
 * different host threads; calls on one handle are serialised internally.
 */
#ifndef SVDB200_H
#define SVDB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  1..5 are SvdLibError (src/error.rs:4-21). */
typedef enum svdb_status {
    SVDB_OK = 0,
    SVDB_ERR_IMTQLB = 1,      /* SvdLibError::ImtqlbError  (src/error.rs:6) */
    SVDB_ERR_STARTV = 2,      /* SvdLibError::StartvError  (src/error.rs:9) */
    SVDB_ERR_STPONE = 3,      /* SvdLibError::StponeError  (src/error.rs:12) */
    SVDB_ERR_IMTQL2 = 4,      /* SvdLibError::Imtql2Error  (src/error.rs:15) */
    SVDB_ERR_LAS2 = 5,        /* SvdLibError::Las2Error    (src/error.rs:18) */
    SVDB_ERR_SHAPE = 6,       /* the crate panics: assert! on shapes / bounds */
    SVDB_ERR_CUDA = 7,        /* a CUDA runtime call failed */
    SVDB_ERR_TIMEOUT = 8,     /* a device-side wait hit its iteration limit */
    SVDB_ERR_UNSUPPORTED = 9, /* the crate has todo!() here, or an option not provided */
    SVDB_ERR_ARG = 10,        /* null pointer, bad enum value */
    SVDB_ERR_OOM = 11,        /* device allocation failed */
    SVDB_ERR_NOCONV = 12      /* an iterative solve stopped above its tolerance */
} svdb_status;

/* Arithmetic of the sparse products.  SVDB_F64 is the drop-in (the crate's
 * f64 path).  SVDB_MIXED stores matrix values in FP32 (SpMV accumulates in
 * FP64; SpMM and Gram products in FP32), while the Lanczos scalars,
 * reorthogonalisation, tridiagonal solves and the second CholeskyQR pass stay
 * FP64. */
typedef enum svdb_precision { SVDB_F64 = 0, SVDB_MIXED = 1 } svdb_precision;

/* Which LAS2 restatement runs.  SVDB_LANCZOS follows lanczos::svd_las2 as
 * written (src/lanczos/mod.rs:104-1406); SVDB_LEGACY follows legacy::svdLAS2
 * (src/legacy.rs:569-2016, SVDLIBC semantics). */
typedef enum svdb_las2_algorithm { SVDB_LANCZOS = 0, SVDB_LEGACY = 1 } svdb_las2_algorithm;

/* PowerIterationNormalizer (src/randomized/mod.rs:14-19). */
typedef enum svdb_normalizer { SVDB_NORM_QR = 0, SVDB_NORM_LU = 1, SVDB_NORM_NONE = 2 } svdb_normalizer;

/* Opaque device-resident sparse operator: the SMat<T> trait object
 * (src/utils.rs:22-33).  Holds A in CSR and in CSC (= CSR of A^T) in HBM. */
typedef struct svdb_matrix svdb_matrix;

/* Diagnostics<T> (src/utils.rs:67-79). */
typedef struct svdb_diagnostics {
    uint64_t non_zero;
    uint64_t dimensions;
    uint64_t iterations;
    int32_t transposed;
    uint64_t lanczos_steps;
    uint64_t ritz_values_stabilized;
    uint64_t significant_values;
    uint64_t singular_values;
    double end_interval[2];
    double kappa;
    uint32_t random_seed;
} svdb_diagnostics;

/* Producer of an svdb_rec; decides svdb_rec_recompose's formula. */
typedef enum svdb_rec_origin { SVDB_REC_LANCZOS = 0, SVDB_REC_LEGACY = 1, SVDB_REC_RANDOMIZED = 2 } svdb_rec_origin;

/* SvdRec<T> (src/utils.rs:44-50).  u is u_rows x u_cols row-major: d x m for
 * LAS2 (src/lanczos/mod.rs:172), m x d for randomized_svd
 * (src/randomized/mod.rs:175-184), as the crate returns them.  When the call
 * asked for device results (svdb_options.result_on_device), u/s/vt are device
 * pointers. */
typedef struct svdb_rec {
    uint64_t d;
    uint64_t u_rows, u_cols;
    double* u;
    double* s;
    uint64_t vt_rows, vt_cols;
    double* vt;
    svdb_diagnostics diagnostics;
    int32_t on_device;
    int32_t origin;           /* svdb_rec_origin: which entry point produced it */
    /* Per-phase device times of the call in milliseconds (CUDA events);
     * the verbose timers of randomized_svd (src/randomized/mod.rs:39-166). */
    double time_ms_total;
    double time_ms_spmv;
    double time_ms_ortho;
    double time_ms_tridiag;
    double time_ms_ritvec;
} svdb_rec;

/* SvdRec<f32> (T = f32, src/utils.rs:44-99): svdb_rec with f32 buffers.
 * diagnostics.end_interval and kappa hold the f32 values, widened. */
typedef struct svdb_rec_f32 {
    uint64_t d;
    uint64_t u_rows, u_cols;
    float* u;
    float* s;
    uint64_t vt_rows, vt_cols;
    float* vt;
    svdb_diagnostics diagnostics;
    int32_t on_device;
    int32_t origin;
    double time_ms_total;
    double time_ms_spmv;
    double time_ms_ortho;
    double time_ms_tridiag;
    double time_ms_ritvec;
} svdb_rec_f32;

/* Internals of one LAS2 run, filled when svdb_options.trace is set: the
 * tridiagonal T (alf: steps+1 values, bet: steps+2 values) and the Ritz values
 * and bounds of the last lanso analysis (steps+1 values each), copied into
 * caller arrays of `cap` doubles (truncated to cap). */
typedef struct svdb_trace {
    double* alf;
    double* bet;
    double* ritz;
    double* bnd;
    uint64_t cap;
    uint64_t steps;      /* out: j of lanso */
    uint64_t purges;     /* out: number of purge sweeps that ran */
    int32_t sparsity_branch; /* out: 0 <= 0.9 < 1 <= 0.99 < 2 <= 0.999 < 3 */
    int32_t lanczos_blocks;  /* out: cooperative grid size used */
} svdb_trace;

/* Options beyond the crate's arguments.  svdb_options_default fills the
 * drop-in behaviour (f64, lanczos::*, results on the host). */
typedef struct svdb_options {
    int32_t precision;        /* svdb_precision */
    int32_t algorithm;        /* svdb_las2_algorithm */
    int32_t result_on_device; /* 1: leave u/s/vt in HBM */
    int32_t verbose;          /* randomized_svd's verbose flag */
    const double* omega;      /* randomized: explicit Omega (ncols x l row-major, host) or NULL */
    void* stream;             /* cudaStream_t to run on, or NULL for the handle's stream */
    svdb_trace* trace;        /* LAS2: optional run internals, or NULL */
} svdb_options;

void svdb_options_default(svdb_options* opts);

/* ---- matrices (nalgebra_sparse storage the crate takes by reference) ---- */

/* CsrMatrix<f64>: indptr[nrows+1], indices[nnz] (usize), values[nnz].
 * Replaces `impl SMat<T> for CsrMatrix<T>` (src/lanczos/mod.rs:1506-1655). */
int svdb_matrix_create_csr(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* indptr,
                           const uint64_t* indices, const double* values, svdb_matrix** out);
/* CscMatrix<f64>: colptr[ncols+1], row indices[nnz].
 * Replaces `impl SMat<T> for CscMatrix<T>` (src/lanczos/mod.rs:1415-1504). */
int svdb_matrix_create_csc(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* colptr,
                           const uint64_t* rowidx, const double* values, svdb_matrix** out);
/* CooMatrix<f64>: triplets in push order; duplicates are kept and summed by
 * the products, as the crate's triplet loop does.
 * Replaces `impl SMat<T> for CooMatrix<T>` (src/lanczos/mod.rs:1657-1740). */
int svdb_matrix_create_coo(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* rows,
                           const uint64_t* cols, const double* values, svdb_matrix** out);
/* The same matrices with f32 values (CsrMatrix<f32>, CscMatrix<f32>,
 * CooMatrix<f32>): the values travel and stay as f32, widened exactly to f64
 * on the device.  Any solver runs on them; the *_f32 entry points give the
 * crate's T = f32 semantics. */
int svdb_matrix_create_csr_f32(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* indptr,
                               const uint64_t* indices, const float* values, svdb_matrix** out);
int svdb_matrix_create_csc_f32(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* colptr,
                               const uint64_t* rowidx, const float* values, svdb_matrix** out);
int svdb_matrix_create_coo_f32(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* rows,
                               const uint64_t* cols, const float* values, svdb_matrix** out);
/* CSR whose arrays are already in device memory (int64 indptr, int32 column
 * indices); the library copies them.  Same contract as svdb_matrix_create_csr. */
int svdb_matrix_create_csr_device(uint64_t nrows, uint64_t ncols, uint64_t nnz, const int64_t* d_indptr,
                                  const int32_t* d_indices, const double* d_values, svdb_matrix** out);
void svdb_matrix_destroy(svdb_matrix* a);
/* SMat::nrows / ncols / nnz (src/utils.rs:23-25). */
uint64_t svdb_matrix_nrows(const svdb_matrix* a);
uint64_t svdb_matrix_ncols(const svdb_matrix* a);
uint64_t svdb_matrix_nnz(const svdb_matrix* a);

/* ---- MaskedCSRMatrix (src/lanczos/masked.rs) ---- */

/* MaskedCSRMatrix::new (masked.rs:21-46): mask_len must equal ncols
 * (the crate's assert_eq!, masked.rs:22-26 -> SVDB_ERR_SHAPE).  The view is
 * built on the device and is independent of later changes to `csr`; `csr`
 * must outlive it (the crate's 'a lifetime). */
int svdb_masked_new(const svdb_matrix* csr, const uint8_t* column_mask, uint64_t mask_len, svdb_matrix** out);
/* MaskedCSRMatrix::with_columns (masked.rs:48-55): duplicates and order are
 * ignored; an index >= ncols returns SVDB_ERR_SHAPE ("Column index out of
 * bounds", masked.rs:51). */
int svdb_masked_with_columns(const svdb_matrix* csr, const uint64_t* columns, uint64_t ncolumns,
                             svdb_matrix** out);
/* masked_to_original[ncols(masked)] (ascending) and original_to_masked[ncols(parent)]
 * with -1 for None (masked.rs:15-17, 32-38); bit-exact. */
int svdb_masked_maps(const svdb_matrix* masked, int64_t* masked_to_original, int64_t* original_to_masked);
/* MaskedCSRMatrix::uses_all_columns (masked.rs:57-59); 1 / 0, -1 if not a masked view. */
int svdb_masked_uses_all_columns(const svdb_matrix* masked);

/* ---- SMat operator entry points (host buffers) ---- */

/* SMat::svd_opa (src/utils.rs:26): y = A x, or A^T x when transposed. */
int svdb_opa(const svdb_matrix* a, const double* x, double* y, int transposed);
/* svd_opb (src/lanczos/mod.rs:311-319): y = A^T (A x), or A (A^T x) when transposed. */
int svdb_opb(const svdb_matrix* a, const double* x, double* y, int transposed);
/* SMat::multiply_with_dense (masked.rs:265-471): result = A X (X: ncols x l)
 * or A^T X (X: nrows x l) when transpose_self.  The crate implements it only
 * for MaskedCSRMatrix (todo!() for CSR/CSC/COO, src/lanczos/mod.rs:1629-1654);
 * here it is defined for every handle.  The transposed product is the
 * mathematical A^T X (masked.rs:388-393 indexes X as if row-major). */
int svdb_multiply_with_dense(const svdb_matrix* a, const double* dense, uint64_t dense_cols, double* result,
                             int transpose_self);
/* SMat::multiply_transposed_by_dense (masked.rs:616-733): result (l x ncols) = Q^T A, Q: nrows x l. */
int svdb_multiply_transposed_by_dense(const svdb_matrix* a, const double* q, uint64_t q_cols, double* result);

/* The column means of the (masked) matrix, ncols values: column sums over
 * the rows times 1/nrows (masked.rs:240-263, compute_column_means). */
int svdb_column_means(const svdb_matrix* a, double* means);
/* SMat::multiply_with_dense_centered (src/utils.rs:29): products of the
 * centred matrix A - 1 means^T (means: ncols values), result = A X - 1 (means^T X)
 * or, when transpose_self, A^T X - means (1^T X).  The crate's masked version
 * (masked.rs:473-614) subtracts other terms; this is the exact product. */
int svdb_multiply_with_dense_centered(const svdb_matrix* a, const double* dense, uint64_t dense_cols,
                                      const double* means, double* result, int transpose_self);
/* SMat::multiply_transposed_by_dense_centered (src/utils.rs:32): result
 * (l x ncols) = Q^T (A - 1 means^T); the crate's masked version is
 * masked.rs:735-874. */
int svdb_multiply_transposed_by_dense_centered(const svdb_matrix* a, const double* q, uint64_t q_cols,
                                               const double* means, double* result);

/* multiply_with_dense on device buffers: d_result = A d_dense (transpose_self
 * = 0, d_dense ncols x l) or A^T d_dense (nrows x l), row-major, enqueued on
 * `stream` (cudaStream_t, NULL = the handle's stream) without synchronising.
 * precision SVDB_F64: double operands; SVDB_MIXED: float operands and FP32
 * matrix values. */
int svdb_multiply_with_dense_device(const svdb_matrix* a, const void* d_dense, uint64_t dense_cols, void* d_result,
                                    int transpose_self, int precision, void* stream);

/* svd_opb on device buffers without allocating: d_y = A^T (A d_x), or
 * A (A^T d_x) when transposed, enqueued on `stream` (NULL = the handle's
 * stream).  No counterpart in the reference: it serves callers that cannot
 * allocate device memory where they apply the operator (their own allocator
 * holds the GPU's memory, or an allocation's synchronisation is not
 * acceptable there).  The intermediate vector lives in a fixed 2^20-double
 * (8 MiB) device array.  It is placed in a GPU's memory, and its address looked
 * up, when the first matrix handle is created on that GPU (an allocating call),
 * and it stays there until exit; this call itself loads and allocates nothing.
 * The handle's device must be the current device (SVDB_ERR_ARG otherwise).
 * A larger intermediate (rows of A, or columns when transposed) returns
 * SVDB_ERR_UNSUPPORTED.  All calls share the array: calls that overlap on the
 * GPU race and must be serialised. */
int svdb_opb_device_noalloc(const svdb_matrix* a, const double* d_x, double* d_y, int transposed, void* stream);

/* svd_opa on device buffers: d_y = A d_x, or A^T d_x when transposed (double
 * vectors), enqueued on `stream` (NULL = the handle's stream) without
 * synchronising.  precision SVDB_MIXED reads the FP32 copy of the matrix
 * values (made on first use) and still sums in FP64. */
int svdb_opa_device(const svdb_matrix* a, const double* d_x, double* d_y, int transposed, int precision,
                    void* stream);

/* Gram matrix of a tall dense matrix on device buffers: d_g (c x c) =
 * X^T X for d_x (rows x c, row-major FP64).  SVDB_F64 sums in FP64 on the
 * CUDA cores; SVDB_MIXED uses the tensor cores (3xTF32 products, FP32
 * accumulation per block, FP64 across blocks; c <= 64), the form the first
 * CholeskyQR pass of randomized_svd takes under SVDB_MIXED.  Synchronises
 * `stream`.  No counterpart in the reference (its QR is nalgebra's). */
int svdb_gram_device(const double* d_x, uint64_t rows, uint64_t c, double* d_g, int precision, void* stream);

/* Device buffers come from the device's stream-ordered pool, which the
 * library keeps cached between calls, and host results of 64 KB and more
 * are page-locked buffers that svdb_rec_free keeps for reuse; this returns
 * both caches (of the current device) to the driver, after a device
 * synchronisation. */
int svdb_release_cached_memory(void);

/* The tridiagonal QL recurrences on the device, one GPU thread in FP64 with
 * the crate's unfused operation order: routine 0 = imtqlb of SVDLIBC
 * (src/legacy.rs:955-1070), 1 = imtqlb as written (src/lanczos/mod.rs:428-584,
 * max_it its iteration cap, *warned its soft failure), 2/3 = imtql2's scalar
 * chain with SVDLIBC's / the current pythag (src/legacy.rs:1590-1700,
 * src/lanczos/mod.rs:901-1028), max_it its cap.  d and e (order n, e[0]
 * unused) are host arrays, overwritten with the results as the host routines
 * leave them; bnd (routines 0-1, in and out: order 1 leaves it as given)
 * gets the bounds row, perm (2-3) imtql2's
 * column order; the first rot_cap plane rotations (i, c, s) are returned and
 * *n_rot counts them all (routine 1 records none).  *device_ms is the kernel's
 * time.  Errors: SVDB_ERR_IMTQLB / SVDB_ERR_IMTQL2 as the crate raises them.
 * The solver runs these recurrences on the host, where the chain of
 * divisions is faster; this entry point exists to measure and test the device
 * form. */
int svdb_tridiag_device(int routine, uint64_t n, double* d, double* e, double* bnd, int32_t* rot_i, double* rot_c,
                        double* rot_s, uint64_t rot_cap, uint64_t* n_rot, int32_t* perm, uint64_t max_it,
                        int* warned, double* device_ms);

/* Self-test of the bounded device waits, with no counterpart in the
 * reference: makes one wait run out on purpose -- which = 0 the grid barrier
 * of the cooperative Lanczos block (a one-block grid that expects a second
 * arrival), which = 1 the mbarrier wait of the tensor-core Gram (a barrier
 * nothing arrives on) -- with a limit of limit_ns (1 .. 2e9).  Returns
 * SVDB_ERR_TIMEOUT when the wait gave up as designed; the context stays
 * usable.  The limit of the real waits (2 s) can be lowered for a process with
 * the environment variable SVDB_WAIT_LIMIT_NS, read at each launch. */
int svdb_wait_selftest(int which, uint64_t limit_ns);

/* The column-sliced SpMV of one orientation of this matrix (transposed = 1:
 * A^T x), with no counterpart in the reference.  Opt-in: with the environment
 * variable SVDB_SPMV=sliced, operators of at least 2^22 nonzeros and more
 * than 18,432 columns whose column indices do not fall within a row get, on
 * their first SpMV (svdb_opa, svdb_opb, LAS2's products), a copy of their
 * entries grouped by slices of 18,432 columns, and the product stages each
 * slice of x in shared memory instead of gathering it from L2 at every
 * nonzero.  Reports the slices and the CTA row ranges, 0 and 0 when the
 * operator has no such plan. */
int svdb_sliced_spmv_info(const svdb_matrix* a, int transposed, int32_t* nslices, int32_t* nranges);

/* The dense-column split the FP32 products (SVDB_MIXED) of this matrix use,
 * with no counterpart in the reference: the number of columns whose density
 * is at least SVDB_DENSE_MIN_DENSITY (0.08 by default) that are multiplied as
 * a dense block on the tensor cores (3xTF32, FP64 drains), and the nonzeros
 * they hold; both 0 before the first FP32 product or when no split is used
 * (too few dense columns, more than 64 dense operand columns, or
 * SVDB_DENSE_SPLIT is not 1: the split is opt-in). */
int svdb_dense_split_info(const svdb_matrix* a, uint64_t* dense_cols, uint64_t* dense_nnz);

/* Number of kernels this library has launched in the process so far. */
uint64_t svdb_kernel_launches(void);

/* ---- LAS2 (src/lanczos/mod.rs) ---- */

/* lanczos::svd_las2 (src/lanczos/mod.rs:104-189); opts may be NULL. */
int svdb_las2(const svdb_matrix* a, uint64_t dimensions, uint64_t iterations, const double end_interval[2],
              double kappa, uint32_t random_seed, const svdb_options* opts, svdb_rec* out);
/* lanczos::svd (src/lanczos/mod.rs:27-36) */
int svdb_svd(const svdb_matrix* a, svdb_rec* out);
/* lanczos::svd_dim (src/lanczos/mod.rs:45-55) */
int svdb_svd_dim(const svdb_matrix* a, uint64_t dimensions, svdb_rec* out);
/* lanczos::svd_dim_seed (src/lanczos/mod.rs:65-86) */
int svdb_svd_dim_seed(const svdb_matrix* a, uint64_t dimensions, uint32_t random_seed, svdb_rec* out);
/* legacy::svdLAS2 (src/legacy.rs:569-654): the SVDLIBC semantics. */
int svdb_legacy_svd_las2(const svdb_matrix* a, uint64_t dimensions, uint64_t iterations,
                         const double end_interval[2], double kappa, uint32_t random_seed,
                         const svdb_options* opts, svdb_rec* out);

/* The LAS2 start vector on the current device: n draws of
 * StdRng::from_seed([seed as u32 LE, 0, ...]).random_range(-1.0..1.0)
 * (src/lanczos/mod.rs:598-605; rand 0.9 ChaCha12).  out: host array of n. */
int svdb_start_vector(uint32_t seed, double* out, uint64_t n);

/* The host-side argument handling of svd_las2 (src/lanczos/mod.rs:116-145):
 * clamped dimensions / iterations, the transpose decision and the sparsity
 * branch (0: <=0.9, 1: >0.9, 2: >0.99, 3: >0.999).  Needs no device. */
int svdb_las2_plan(uint64_t nrows, uint64_t ncols, uint64_t nnz, uint64_t dimensions, uint64_t iterations,
                   uint64_t* dimensions_out, uint64_t* iterations_out, int32_t* transposed_out,
                   int32_t* sparsity_branch_out);

/* ---- randomized SVD (src/randomized/mod.rs) ---- */

/* randomized::randomized_svd (src/randomized/mod.rs:24-199).  has_seed = 0
 * means seed None (the crate then seeds with 0, :304-307).  Omega is drawn on
 * the device from a counter-based generator keyed by the seed, or taken from
 * opts->omega.  mean_center = 1 factorises the centred matrix A - 1 mu^T,
 * mu the column means of the (masked) matrix (src/lanczos/masked.rs:240-263),
 * through the exact products A X - 1 (mu^T X) and A^T Y - mu (1^T Y); the
 * crate's own adjusted products (masked.rs:496-509, 793-809) do not equal
 * these. */
int svdb_randomized_svd(const svdb_matrix* a, uint64_t target_rank, uint64_t n_oversamples,
                        uint64_t n_power_iters, int normalizer, int mean_center, int has_seed, uint64_t seed,
                        int verbose, const svdb_options* opts, svdb_rec* out);

/* ---- T = f32 (impl SvdFloat for f32, src/utils.rs:87-99) ---- */

/* lanczos::svd_las2 / svd / svd_dim / svd_dim_seed monomorphised at T = f32
 * (src/lanczos/mod.rs:27-189): every tolerance takes f32::EPSILON (eps,
 * eps34, sqrt(eps), compare), kappa is clamped to f32 eps34, and the start
 * vector's f64 draws are rounded to f32.  The products use the FP32 values
 * and FP32 operand vectors; sums and the recurrences stay FP64, and u/s/vt
 * are rounded to f32 at the end.  opts->algorithm = SVDB_LEGACY returns
 * SVDB_ERR_UNSUPPORTED (legacy::svdLAS2 is f64-only); opts->precision is
 * ignored. */
int svdb_las2_f32(const svdb_matrix* a, uint64_t dimensions, uint64_t iterations, const float end_interval[2],
                  float kappa, uint32_t random_seed, const svdb_options* opts, svdb_rec_f32* out);
int svdb_svd_f32(const svdb_matrix* a, svdb_rec_f32* out);
int svdb_svd_dim_f32(const svdb_matrix* a, uint64_t dimensions, svdb_rec_f32* out);
int svdb_svd_dim_seed_f32(const svdb_matrix* a, uint64_t dimensions, uint32_t random_seed, svdb_rec_f32* out);
/* randomized::randomized_svd at T = f32: Omega's f64 draws (or opts->omega)
 * rounded to f32, FP32 operands in the products, FP64 factorisations,
 * results rounded to f32. */
int svdb_randomized_svd_f32(const svdb_matrix* a, uint64_t target_rank, uint64_t n_oversamples,
                            uint64_t n_power_iters, int normalizer, int mean_center, int has_seed, uint64_t seed,
                            int verbose, const svdb_options* opts, svdb_rec_f32* out);
void svdb_rec_f32_free(svdb_rec_f32* r);

/* ---- batches of masked column subsets (no reference counterpart) ---- */

/* A prepared batch: randomized_svd on `count` column subsets of one matrix,
 * each equivalent to randomized_svd(MaskedCSRMatrix::with_columns(a, cols_b),
 * ...) with the same arguments and seed.  The subsets are never compacted:
 * the sparse products read A (CSR and CSC) and remap columns through
 * per-subset maps.  Every kernel covers all subsets in one launch; the whole
 * solve is captured once into a CUDA graph and replayed by svdb_batch_run. */
typedef struct svdb_batch svdb_batch;

typedef struct svdb_batch_options {
    int32_t precision;        /* SVDB_MIXED (FP32 products and dense operands, FP64 Gram,
                                 Cholesky, CholeskyQR passes and small SVD) or SVDB_F64 */
    int32_t result_on_device; /* 1: u/s/vt of each record in HBM */
    int32_t autotune;         /* 1: time the candidate product shapes on the first batch of
                                 this shape class and keep the fastest (cached per process) */
    int32_t use_graph;        /* 1: capture the solve into a CUDA graph (default) */
    void* stream;             /* cudaStream_t, NULL = the matrix handle's stream */
} svdb_batch_options;

typedef struct svdb_batch_info {
    uint64_t count;
    int32_t subsets_per_row_item; /* autotuned: subsets sharing one read of a row of A (1, untuned, under SVDB_MIXED) */
    int32_t columns_per_lane;     /* autotuned: dense columns per lane (vector width) */
    uint64_t graph_nodes;         /* kernels and copies in the captured graph (0 without) */
    uint64_t kernels_per_run;     /* kernel launches of one run */
    double time_ms_tune;          /* autotuning time at creation */
    double time_ms_last_run;      /* device time of the last svdb_batch_run */
    uint64_t total_subset_nnz;    /* sum over subsets of their nonzeros */
} svdb_batch_info;

void svdb_batch_options_default(svdb_batch_options* opts);
/* columns of subset b: columns[col_offsets[b] .. col_offsets[b+1]), as
 * MaskedCSRMatrix::with_columns takes them (duplicates and order ignored,
 * an index >= ncols is SVDB_ERR_SHAPE).  Every subset must keep at least
 * target_rank + n_oversamples columns (SVDB_ERR_UNSUPPORTED otherwise).
 * `a` is a CSR, CSC or COO handle. */
int svdb_batch_create(const svdb_matrix* a, const uint64_t* col_offsets, const uint64_t* columns, uint64_t count,
                      uint64_t target_rank, uint64_t n_oversamples, uint64_t n_power_iters, int normalizer,
                      int has_seed, uint64_t seed, const svdb_batch_options* opts, svdb_batch** out);
/* Runs the batch (one graph launch) and fills outs[0..count) like
 * svdb_randomized_svd: u m x d, s d, vt d x ncols_b. */
int svdb_batch_run(svdb_batch* batch, svdb_rec* outs);
int svdb_batch_get_info(const svdb_batch* batch, svdb_batch_info* info);
void svdb_batch_destroy(svdb_batch* batch);
/* create + run + destroy. */
int svdb_randomized_svd_batch(const svdb_matrix* a, const uint64_t* col_offsets, const uint64_t* columns,
                              uint64_t count, uint64_t target_rank, uint64_t n_oversamples, uint64_t n_power_iters,
                              int normalizer, int has_seed, uint64_t seed, const svdb_batch_options* opts,
                              svdb_rec* outs);

/* ---- adjoint of the truncated SVD (no reference counterpart) ---- */

/* Options of svdb_svd_adjoint; svdb_adjoint_options_default gives FP64,
 * host buffers, cg_tol 1e-12 and cg_max_iters 5000. */
typedef struct svdb_adjoint_options {
    int32_t precision;        /* SVDB_F64, or SVDB_MIXED: FP32 factors and sums in the SDDMM */
    int32_t inputs_on_device; /* 1: u, s, v, g_u, g_s, g_v and grad_values are device pointers */
    double cg_tol;            /* relative residual of the complement solves */
    uint64_t cg_max_iters;
    void* stream;             /* cudaStream_t, NULL = the handle's stream */
    uint64_t cg_iterations;   /* out: block-CG iterations run */
    double cg_residual;       /* out: largest relative residual at exit */
    double time_ms_solve;     /* out: device time of everything before the SDDMM */
    double time_ms_sddmm;     /* out: device time of the SDDMM */
} svdb_adjoint_options;

void svdb_adjoint_options_default(svdb_adjoint_options* opts);

/* Gradient of L(U, s, V) with respect to A's stored values, where
 * A V = U diag(s), A^T U = V diag(s) are the k leading singular triplets
 * (u: nrows x k, v: ncols x k, row-major; s descending, s_k above the next
 * singular value of A) and g_u, g_s, g_v = dL/dU, dL/ds, dL/dV (NULL = 0).
 * The dense gradient is
 *   U M V^T + Gamma V^T + U Delta^T,
 *   M = diag(g_s) + (F o (U^T g_u - g_u^T U)) S + S (F o (V^T g_v - g_v^T V)),
 *   F_ij = 1 / (s_j^2 - s_i^2) (i != j), 0 on the diagonal,
 * and (Gamma, Delta) solve, column by column, the shifted systems of the
 * residual operator A_perp = A - U S V^T that carry the complement
 * projections (I - U U^T) g_u, (I - V V^T) g_v:
 *   (s_i^2 I - A_perp^T A_perp) delta_i = s_i b_i + A_perp^T a_i,
 *   gamma_i = (a_i + A_perp delta_i) / s_i,
 * solved by block CG on the device.  The gradient is evaluated only at A's
 * nonzeros, as an SDDMM of the rank-2k factors [U M + Gamma, U] and
 * [V, Delta]: grad_values[e] = dL/dA(r_e, c_e) in the order the handle was
 * created with (CSR entry order, or CSC entry order for CSC handles).  COO
 * handles and masked views return SVDB_ERR_UNSUPPORTED; a CG that stops above
 * cg_tol returns SVDB_ERR_NOCONV with grad_values filled. */
int svdb_svd_adjoint(const svdb_matrix* a, uint64_t k, const double* u, const double* s, const double* v,
                     const double* g_u, const double* g_s, const double* g_v, svdb_adjoint_options* opts,
                     double* grad_values);

/* SDDMM on the handle's pattern with device factors:
 * d_out[e] = sum_t left[r_e][t] * right[c_e][t] (left: nrows x rank,
 * right: ncols x rank, row-major), in the entry order of svdb_svd_adjoint.
 * precision SVDB_F64: double factors and output; SVDB_MIXED: float. */
int svdb_sddmm_device(const svdb_matrix* a, const void* d_left, const void* d_right, uint64_t rank, void* d_out,
                      int precision, void* stream);

/* svd_flip(u, v, u_based_decision) (src/randomized/mod.rs:332-438), in place
 * on row-major arrays (u: u_rows x u_cols, v: v_rows x v_cols; either may be
 * NULL).  u-based: column j of u is negated when its first entry of largest
 * magnitude is negative, and so is row j of v (j < min(v_rows, u_cols)).
 * v-based: row i of v by its largest entry, and column i of u
 * (i < min(u_cols, v_rows)).  Both NULL, or the deciding matrix NULL, return
 * SVDB_ERR_LAS2 as the crate's Las2Error.  on_device = 1: device pointers
 * (the flip runs on the current device's default stream and synchronises). */
int svdb_svd_flip(double* u, uint64_t u_rows, uint64_t u_cols, double* v, uint64_t v_rows, uint64_t v_cols,
                  int u_based_decision, int on_device);

/* ---- results ---- */

/* Frees u, s, vt (host or device) and zeroes the record.  Host results are
 * library memory (page-locked from 64 KB up): release them with this call,
 * never with free(). */
void svdb_rec_free(svdb_rec* rec);
/* SvdRec::recompose: out (u_rows x vt_cols, host) = u diag(s) vt as the crate
 * writes it (src/lanczos/mod.rs:1408-1413), which needs u_cols == d
 * (otherwise SVDB_ERR_SHAPE, where ndarray panics); for legacy records
 * ut^T diag(s) vt (src/legacy.rs:2023-2028), out being u_cols x vt_cols. */
int svdb_rec_recompose(const svdb_rec* rec, double* out);

const char* svdb_last_error_message(void);
/* Library version (major * 10000 + minor * 100 + patch). */
int svdb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SVDB200_H */
