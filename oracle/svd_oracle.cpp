// ============================================================================
// svd_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A CPU FP64 restatement of single-svdlib's hot path, used as the CHECKER for
// the CUDA implementation.  Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / --impl reference legs may load this library.  The product
// (single-svdlib_b200/) never links, calls or falls back to it.
//
// Every function cites the reference file:line it restates (paths relative to
// the single-svdlib crate root).  Build: oracle/Makefile (g++ -O2
// -ffp-contract=off, no -ffast-math, so a*b+c is never fused, matching Rust).
//
// What is restated:
//   * rand 0.9 StdRng (= rand_chacha 0.9 ChaCha12Rng, rand_core 0.9 BlockRng)
//     and rand's UniformFloat<f64>::sample_single, for the LAS2 start vector
//     (src/lanczos/mod.rs:598-605).  ChaCha follows Bernstein's specification
//     (RFC 8439 block function, 64-bit counter / 64-bit stream variant).
//   * SMat operators for CSR / CSC / COO (src/lanczos/mod.rs:1415-1700) and
//     MaskedCSRMatrix (src/lanczos/masked.rs:21-733), including the chunked
//     Rayon decomposition of A^T x (src/utils.rs:10-20) for a given thread count.
//   * lanczos::svd_las2 as written (src/lanczos/mod.rs:104-1406), with its
//     modified tolerances and its svd_pythag / imtqlb / ritvec behaviour.
//   * legacy::svdLAS2 (src/legacy.rs:569-2016), the SVDLIBC semantics.
//   * randomized::randomized_svd (src/randomized/mod.rs:24-199) with an
//     explicit Omega, Householder thin QR and a one-sided Jacobi SVD standing
//     in for nalgebra's qr()/svd() (third-party, nalgebra 0.34.1), plus a
//     switch reproducing the masked A^T*Y indexing of masked.rs:388-393.
// ============================================================================
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// The scalar T of the crate's generic solvers (SvdFloat): f64, or f32 when
// built with -DORC_F32 (lanczos and randomized only; legacy is f64-only).
#ifdef ORC_F32
using real = float;
#else
using real = double;
#endif

static const real EPS = std::numeric_limits<real>::epsilon();  // SvdFloat::eps, src/utils.rs:87-113
static int g_threads = 1;  // stands in for rayon::current_num_threads()

static real eps34() { return std::pow(EPS, 0.75); }  // src/utils.rs:106-108

// SvdFloat::compare, src/utils.rs:110-112 (absolute epsilon)
static inline bool compare(real a, real b) { return std::fabs(b - a) < EPS; }

// Rust f64::max / f64::min ignore a NaN operand, like C fmax / fmin.
static inline real fmax_(real a, real b) { return std::fmax(a, b); }
static inline real fmin_(real a, real b) { return std::fmin(a, b); }

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
enum {
    E_OK = 0, E_IMTQLB = 1, E_STARTV = 2, E_STPONE = 3, E_IMTQL2 = 4, E_LAS2 = 5,
    E_SHAPE = 6, E_UNSUPPORTED = 9, E_PANIC = 10
};

// ---------------------------------------------------------------------------
// ChaCha block function (RFC 8439 section 2.3; 64-bit counter in words 12-13,
// 64-bit stream id in words 14-15 as rand_chacha uses it).
// ---------------------------------------------------------------------------
static inline uint32_t rotl32(uint32_t v, int c) { return (v << c) | (v >> (32 - c)); }

static void chacha_block(const uint32_t key[8], uint64_t counter, uint64_t stream, int rounds,
                         uint32_t out[16]) {
    uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                      key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                      (uint32_t)counter, (uint32_t)(counter >> 32),
                      (uint32_t)stream, (uint32_t)(stream >> 32)};
    uint32_t x[16];
    std::memcpy(x, s, sizeof(x));
#define QR(a, b, c, d)                      \
    x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 16); \
    x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 12); \
    x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 8);  \
    x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 7);
    for (int r = 0; r < rounds; r += 2) {
        QR(0, 4, 8, 12) QR(1, 5, 9, 13) QR(2, 6, 10, 14) QR(3, 7, 11, 15)
        QR(0, 5, 10, 15) QR(1, 6, 11, 12) QR(2, 7, 8, 13) QR(3, 4, 9, 14)
    }
#undef QR
    for (int i = 0; i < 16; ++i) out[i] = x[i] + s[i];
}

// rand_core 0.9 BlockRng over a 4-block (64-word) ChaCha buffer.
struct ChaChaRng {
    uint32_t key[8];
    uint64_t counter = 0;
    int rounds;
    uint32_t buf[64];
    int index = 64;
    ChaChaRng(const uint8_t seed[32], int rounds_) : rounds(rounds_) {
        for (int i = 0; i < 8; ++i)
            key[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) |
                     ((uint32_t)seed[4 * i + 2] << 16) | ((uint32_t)seed[4 * i + 3] << 24);
    }
    void refill() {
        for (int b = 0; b < 4; ++b) chacha_block(key, counter + b, 0, rounds, buf + 16 * b);
        counter += 4;
    }
    uint32_t next_u32() {
        if (index >= 64) { refill(); index = 0; }
        return buf[index++];
    }
    uint64_t next_u64() {
        uint64_t lo, hi;
        if (index < 63) { lo = buf[index]; hi = buf[index + 1]; index += 2; }
        else if (index >= 64) { refill(); lo = buf[0]; hi = buf[1]; index = 2; }
        else { lo = buf[63]; refill(); hi = buf[0]; index = 1; }
        return lo | (hi << 32);
    }
};

// UniformFloat<f64>::sample_single(-1.0, 1.0): value in [1,2) from the top 52
// bits, minus 1, times the scale (2.0) plus low (-1.0).
static inline double uniform_pm1(uint64_t u) {
    uint64_t bits = (u >> 12) | 0x3FF0000000000000ull;
    double v12;
    std::memcpy(&v12, &bits, 8);
    double v01 = v12 - 1.0;
    double scale = 2.0;
    return v01 * scale + (-1.0);
}

// startv's fill: StdRng::from_seed(seed u32 in bytes 0..3), src/lanczos/mod.rs:598-605;
// each f64 draw is rounded to T (T::from_f64)
static void start_vector(uint32_t seed, real* w, size_t n) {
    uint8_t bytes[32] = {0};
    bytes[0] = seed & 0xff; bytes[1] = (seed >> 8) & 0xff;
    bytes[2] = (seed >> 16) & 0xff; bytes[3] = (seed >> 24) & 0xff;
    ChaChaRng rng(bytes, 12);
    for (size_t i = 0; i < n; ++i) w[i] = (real)uniform_pm1(rng.next_u64());
}

// ---------------------------------------------------------------------------
// Operators (trait SMat, src/utils.rs:22-33)
// ---------------------------------------------------------------------------
// determine_chunk_size, src/utils.rs:10-20
static size_t determine_chunk_size(size_t nrows) {
    size_t target = (size_t)g_threads * 4;
    size_t c = (nrows + target - 1) / target;
    return std::max<size_t>(c, 64);
}

struct SMat {
    virtual ~SMat() {}
    virtual size_t nrows() const = 0;
    virtual size_t ncols() const = 0;
    virtual size_t nnz() const = 0;
    virtual void svd_opa(const real* x, real* y, bool transposed) const = 0;
};

struct Compressed {  // major offsets, minor indices, values
    size_t nmajor = 0, nminor = 0;
    std::vector<uint64_t> ptr, idx;
    std::vector<real> val;
};

// SMat for CsrMatrix, src/lanczos/mod.rs:1506-1603.  `legacy` selects the
// sequential operator of src/legacy.rs:2080-2104.
struct CsrOp : SMat {
    const Compressed* a;
    bool legacy;
    CsrOp(const Compressed* a_, bool legacy_) : a(a_), legacy(legacy_) {}
    size_t nrows() const override { return a->nmajor; }
    size_t ncols() const override { return a->nminor; }
    size_t nnz() const override { return a->idx.size(); }
    void svd_opa(const real* x, real* y, bool transposed) const override {
        const size_t m = a->nmajor, n = a->nminor;
        const uint64_t* p = a->ptr.data();
        const uint64_t* ci = a->idx.data();
        const real* v = a->val.data();
        if (!transposed) {
            // row gather, mod.rs:1551-1570 (per-row sequential sum, rows in parallel)
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
            for (size_t i = 0; i < m; ++i) {
                real sum = 0.0;
                for (uint64_t j = p[i]; j < p[i + 1]; ++j) sum += v[j] * x[ci[j]];
                y[i] = sum;
            }
            return;
        }
        std::fill(y, y + n, 0.0);
        if (legacy) {  // legacy.rs:2096-2101: sequential scatter
            for (size_t i = 0; i < m; ++i)
                for (uint64_t j = p[i]; j < p[i + 1]; ++j) y[ci[j]] += v[j] * x[i];
            return;
        }
        // chunk-private buffers + serial combine, mod.rs:1571-1602
        size_t cs = determine_chunk_size(m);
        size_t nch = (m + cs - 1) / cs;
        std::vector<std::vector<real>> loc(nch);
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads) if (g_threads > 1)
        for (size_t c = 0; c < nch; ++c) {
            std::vector<real> ly(n, 0.0);
            size_t s = c * cs, e = std::min(s + cs, m);
            for (size_t i = s; i < e; ++i) {
                real rv = x[i];
                for (uint64_t j = p[i]; j < p[i + 1]; ++j) ly[ci[j]] += v[j] * rv;
            }
            loc[c].swap(ly);
        }
        for (size_t c = 0; c < nch; ++c)
            for (size_t k = 0; k < n; ++k)
                if (loc[c][k] != 0.0) y[k] += loc[c][k];
    }
};

// SMat for CscMatrix, src/lanczos/mod.rs:1415-1472 (and legacy.rs:2050-2070)
struct CscOp : SMat {
    const Compressed* a;  // major = columns
    CscOp(const Compressed* a_) : a(a_) {}
    size_t nrows() const override { return a->nminor; }
    size_t ncols() const override { return a->nmajor; }
    size_t nnz() const override { return a->idx.size(); }
    void svd_opa(const real* x, real* y, bool transposed) const override {
        const uint64_t* p = a->ptr.data();
        const uint64_t* ri = a->idx.data();
        const real* v = a->val.data();
        size_t ylen = transposed ? a->nmajor : a->nminor;
        std::fill(y, y + ylen, 0.0);
        if (transposed) {
            for (size_t i = 0; i < a->nmajor; ++i)
                for (uint64_t j = p[i]; j < p[i + 1]; ++j) y[i] += v[j] * x[ri[j]];
        } else {
            for (size_t i = 0; i < a->nmajor; ++i) {
                real xv = x[i];
                for (uint64_t j = p[i]; j < p[i + 1]; ++j) y[ri[j]] += v[j] * xv;
            }
        }
    }
};

// SMat for CooMatrix, src/lanczos/mod.rs:1657-1700 (triplets in push order)
struct CooOp : SMat {
    size_t m, n;
    std::vector<uint64_t> r, c;
    std::vector<real> v;
    size_t nrows() const override { return m; }
    size_t ncols() const override { return n; }
    size_t nnz() const override { return v.size(); }
    void svd_opa(const real* x, real* y, bool transposed) const override {
        size_t ylen = transposed ? n : m;
        std::fill(y, y + ylen, 0.0);
        if (transposed) {
            for (size_t k = 0; k < v.size(); ++k) y[c[k]] += v[k] * x[r[k]];
        } else {
            for (size_t k = 0; k < v.size(); ++k) y[r[k]] += v[k] * x[c[k]];
        }
    }
};

// MaskedCSRMatrix, src/lanczos/masked.rs:13-238.
struct MaskedOp : SMat {
    const Compressed* a;
    std::vector<uint8_t> mask;
    std::vector<int64_t> m2o;  // masked_to_original (ascending)
    std::vector<int64_t> o2m;  // original_to_masked, -1 = None
    // masked.rs:133-143 delegates small matrices to the full CSR operator,
    // which asserts on the masked vector length (a panic for a real mask).
    // The checker computes the general masked product there instead and
    // records that the reference would have panicked.
    mutable bool would_panic = false;
    MaskedOp(const Compressed* a_, const uint8_t* mk) : a(a_) {
        mask.assign(mk, mk + a->nminor);
        o2m.assign(a->nminor, -1);
        int64_t mi = 0;  // masked.rs:32-38
        for (size_t i = 0; i < a->nminor; ++i)
            if (mask[i]) { m2o.push_back((int64_t)i); o2m[i] = mi++; }
    }
    bool uses_all_columns() const {  // masked.rs:57-59
        if (m2o.size() != a->nminor) return false;
        for (auto b : mask) if (!b) return false;
        return true;
    }
    size_t nrows() const override { return a->nmajor; }
    size_t ncols() const override { return m2o.size(); }
    size_t nnz() const override {  // masked.rs:89-102
        size_t cnt = 0;
        for (size_t i = 0; i < a->idx.size(); ++i) if (mask[a->idx[i]]) ++cnt;
        return cnt;
    }
    void svd_opa(const real* x, real* y, bool transposed) const override {
        const size_t m = a->nmajor;
        const uint64_t* p = a->ptr.data();
        const uint64_t* ci = a->idx.data();
        const real* v = a->val.data();
        if (uses_all_columns()) {
            CsrOp(a, false).svd_opa(x, y, transposed);
            return;
        }
        if (a->nmajor < 1000 && a->nminor < 1000) would_panic = true;
        size_t nm = ncols();
        if (!transposed) {  // masked.rs:145-196
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
            for (size_t i = 0; i < m; ++i) {
                real sum = 0.0;
                for (uint64_t j = p[i]; j < p[i + 1]; ++j) {
                    int64_t mc = o2m[ci[j]];
                    if (mc >= 0) sum += v[j] * x[mc];
                }
                y[i] = sum;
            }
            return;
        }
        // masked.rs:197-237
        std::fill(y, y + nm, 0.0);
        size_t cs = determine_chunk_size(m);
        size_t nch = (m + cs - 1) / cs;
        std::vector<std::vector<real>> loc(nch);
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads) if (g_threads > 1)
        for (size_t c = 0; c < nch; ++c) {
            std::vector<real> ly(nm, 0.0);
            size_t s = c * cs, e = std::min(s + cs, m);
            for (size_t i = s; i < e; ++i) {
                real rv = x[i];
                if (rv == 0.0) continue;
                for (uint64_t j = p[i]; j < p[i + 1]; ++j) {
                    int64_t mc = o2m[ci[j]];
                    if (mc >= 0) ly[mc] += v[j] * rv;
                }
            }
            loc[c].swap(ly);
        }
        for (size_t c = 0; c < nch; ++c)
            for (size_t k = 0; k < nm; ++k)
                if (loc[c][k] != 0.0) y[k] += loc[c][k];
    }
};

// ---------------------------------------------------------------------------
// BLAS-1, src/lanczos/mod.rs:311-424 (legacy: src/legacy.rs:845-930)
// ---------------------------------------------------------------------------
static bool g_legacy_blas = false;  // legacy BLAS-1 is always sequential

static void svd_opb(const SMat& A, const real* x, real* y, real* temp, bool transposed) {
    A.svd_opa(x, temp, transposed);
    A.svd_opa(temp, y, !transposed);
}
static void svd_daxpy(real da, const real* x, real* y, size_t n) {
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1 && n >= 1000 && !g_legacy_blas)
    for (size_t i = 0; i < n; ++i) y[i] += da * x[i];
}
static size_t svd_idamax(size_t n, const real* x) {
    if (n == 0) throw Error(E_PANIC, "svd_idamax: unexpected inputs!");
    if (n == 1) return 0;
    size_t imax = 0;
    for (size_t i = 1; i < n; ++i)
        if (std::fabs(x[i]) > std::fabs(x[imax])) imax = i;
    return imax;
}
static real svd_fsign(real a, real b) {
    return ((a >= 0.0 && b >= 0.0) || (a < 0.0 && b < 0.0)) ? a : -a;
}
// Current crate: mod.rs:361-380.  The loop sets r = (s/u)^2 (the factor r of
// the Moler-Morrison update is absent), so for comparable |a|, |b| the result
// exceeds hypot(a, b); restated as written.
static real svd_pythag_current(real a, real b) {
    real n = fmax_(std::fabs(a), std::fabs(b));
    if (!(n > 0.0)) return 0.0;
    real p = n;
    real q = fmin_(std::fabs(a), std::fabs(b)) / p;
    real r = q * q;
    real t = 4.0 + r;
    while (!compare(t, 4.0)) {
        real s = r / t;
        real u = 1.0 + 2.0 * s;
        p = p * u;
        real su = s / u;
        r = su * su;
        t = 4.0 + r;
    }
    return p;
}
// Legacy: legacy.rs:878-895 (r *= (s/u)^2)
static real svd_pythag_legacy(real a, real b) {
    real n = fmax_(std::fabs(a), std::fabs(b));
    if (!(n > 0.0)) return 0.0;
    real p = n;
    real q = fmin_(std::fabs(a), std::fabs(b)) / p;
    real r = q * q;
    real t = 4.0 + r;
    while (!compare(t, 4.0)) {
        real s = r / t;
        real u = 1.0 + 2.0 * s;
        p *= u;
        real su = s / u;
        r *= su * su;
        t = 4.0 + r;
    }
    return p;
}
static real svd_ddot(const real* x, const real* y, size_t n) {
    if (g_threads <= 1 || n < 1000 || g_legacy_blas) {
        real s = 0.0;
        for (size_t i = 0; i < n; ++i) s += x[i] * y[i];
        return s;
    }
    // Rayon's reduction tree is scheduling dependent; a fixed-chunk ordered
    // reduction stands in for it.
    int T = g_threads;
    std::vector<real> part(T, 0.0);
#pragma omp parallel for schedule(static, 1) num_threads(T)
    for (int t = 0; t < T; ++t) {
        size_t s = n * t / T, e = n * (t + 1) / T;
        real acc = 0.0;
        for (size_t i = s; i < e; ++i) acc += x[i] * y[i];
        part[t] = acc;
    }
    real s = 0.0;
    for (int t = 0; t < T; ++t) s += part[t];
    return s;
}
static real svd_norm(const real* x, size_t n) { return std::sqrt(svd_ddot(x, x, n)); }
static void svd_datx(real d, const real* x, real* y, size_t n) {
    for (size_t i = 0; i < n; ++i) y[i] = d * x[i];
}
static void svd_dscal(real d, real* x, size_t n) {
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1 && n >= 1000 && !g_legacy_blas)
    for (size_t i = 0; i < n; ++i) x[i] *= d;
}
// reversing copy, mod.rs:417-424
static void svd_dcopy(size_t n, size_t off, const real* x, real* y) {
    if (n > 0) {
        size_t start = n - 1;
        for (size_t i = 0; i < n; ++i) y[off + start - i] = x[off + i];
    }
}
// mod.rs:297-307
static void insert_sort(size_t n, real* a1, real* a2) {
    for (size_t i = 1; i < n; ++i)
        for (size_t j = i; j >= 1; --j) {
            if (a1[j - 1] <= a1[j]) break;
            std::swap(a1[j - 1], a1[j]);
            std::swap(a2[j - 1], a2[j]);
        }
}

// ---------------------------------------------------------------------------
// Work space and store, mod.rs:191-272
// ---------------------------------------------------------------------------
static const size_t MAXLL = 2;
struct Store {
    size_t n;
    std::vector<std::vector<real>> vecs;
    explicit Store(size_t n_) : n(n_) {}
    void storq(size_t idx, const real* v) {
        while (idx + MAXLL >= vecs.size()) vecs.emplace_back(n, 0.0);
        std::memcpy(vecs[idx + MAXLL].data(), v, n * sizeof(real));
    }
    void storp(size_t idx, const real* v) {
        while (idx >= vecs.size()) vecs.emplace_back(n, 0.0);
        std::memcpy(vecs[idx].data(), v, n * sizeof(real));
    }
    const real* retrq(size_t idx) const { return vecs.at(idx + MAXLL).data(); }
    const real* retrp(size_t idx) const { return vecs.at(idx).data(); }
};

struct Work {
    size_t nrows, ncols;
    bool transposed;
    std::vector<real> w0, w1, w2, w3, w4, w5, alf, eta, oldeta, bet, bnd, ritz, temp;
    Work(size_t nr, size_t nc, bool tr, size_t it)
        : nrows(nr), ncols(nc), transposed(tr), w0(nc), w1(nc), w2(nc), w3(nc), w4(nc), w5(nc),
          alf(it), eta(it), oldeta(it), bet(1 + it), bnd(1 + it, std::numeric_limits<real>::max()),
          ritz(1 + it), temp(nr) {}
};

// Per-run settings that differ between lanczos::* and legacy::*.
struct Mode {
    bool legacy = false;
    real sparsity = 0.0;
    real adaptive_eps = EPS;
    size_t max_imtqlb = 100;
    size_t max_imtql2 = 50;
    size_t extra_steps = 0;
};

// mod.rs:1068-1070 / 1273-1275
static real sparsity_of(const SMat& A) {
    return 1.0 - ((real)A.nnz() / ((real)A.nrows() * (real)A.ncols()));
}
static Mode make_mode(const SMat& A, bool legacy) {
    Mode md;
    md.legacy = legacy;
    if (legacy) { md.max_imtqlb = 30; md.max_imtql2 = 30; return md; }
    real sp = sparsity_of(A);
    md.sparsity = sp;
    md.max_imtqlb = sp > 0.999 ? 500 : sp > 0.99 ? 300 : sp > 0.9 ? 100 : 50;    // mod.rs:1276-1288
    md.adaptive_eps = sp > 0.99 ? EPS * 100.0 : sp > 0.9 ? EPS * 10.0 : EPS;     // mod.rs:1291-1300
    md.max_imtql2 = sp > 0.999 ? 500 : sp > 0.99 ? 300 : sp > 0.9 ? 200 : 50;    // mod.rs:1084-1096
    md.extra_steps = sp > 0.99 ? 5 : 0;                                           // mod.rs:1390-1394
    return md;
}

// ---------------------------------------------------------------------------
// imtqlb: current (mod.rs:428-584) and legacy (legacy.rs:955-1070)
// ---------------------------------------------------------------------------
static bool g_imtqlb_warned = false;

static void imtqlb_current(size_t n, real* d, real* e, real* bnd, size_t max_imtqlb) {
    if (n == 1) return;
    real msf = std::sqrt((real)n);
    bnd[0] = 1.0;
    size_t last = n - 1;
    for (size_t i = 1; i <= last; ++i) { bnd[i] = 0.0; e[i - 1] = e[i]; }
    e[last] = 0.0;
    size_t i = 0;
    bool had_issues = false;
    for (size_t l = 0; l <= last; ++l) {
        size_t iteration = 0;
        real p = d[l];   // set once per l (mod.rs:452-453)
        real f = bnd[l];
        while (iteration <= max_imtqlb) {
            size_t m = l;
            while (m < n) {
                if (m == last) break;
                real test = std::fabs(d[m]) + std::fabs(d[m + 1]);
                real tol = EPS * 100.0 * fmax_(test, 1.0) * msf;
                if (std::fabs(e[m]) <= tol) break;
                ++m;
            }
            if (m == l) {
                bool exchange = true;
                if (l > 0) {
                    i = l;
                    while (i >= 1 && exchange) {
                        if (p < d[i - 1]) { d[i] = d[i - 1]; bnd[i] = bnd[i - 1]; --i; }
                        else exchange = false;
                    }
                }
                if (exchange) i = 0;
                d[i] = p;
                bnd[i] = f;
                iteration = max_imtqlb + 1;
            } else {
                if (iteration == max_imtqlb) {
                    had_issues = true;
                    for (size_t idx = l; idx <= m; ++idx) bnd[idx] = fmax_(bnd[idx], 0.1);
                    e[l] = 0.0;
                    break;
                }
                ++iteration;
                real g = (d[l + 1] - p) / (2.0 * e[l]);
                real r = svd_pythag_current(g, 1.0);
                g = d[m] - p + e[l] / (g + svd_fsign(r, g));
                real s = 1.0, c = 1.0;
                p = 0.0;
                if (m == 0) throw Error(E_PANIC, "imtqlb: expected 'm' to be non-zero");
                i = m - 1;
                bool underflow = false;
                while (!underflow && i >= l) {
                    f = s * e[i];
                    real b = c * e[i];
                    r = svd_pythag_current(f, g);
                    e[i + 1] = r;
                    if (r < EPS * 1000.0 * (std::fabs(f) + std::fabs(g))) { underflow = true; break; }
                    if (std::fabs(r) < EPS * 100.0) r = EPS * 100.0 * svd_fsign(1.0, r);
                    s = f / r;
                    c = g / r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    p = s * r;
                    d[i + 1] = g + p;
                    g = c * r - b;
                    f = bnd[i + 1];
                    bnd[i + 1] = s * bnd[i] + c * f;
                    bnd[i] = c * bnd[i] - s * f;
                    if (i == 0) break;
                    --i;
                }
                if (underflow) d[i + 1] -= p;
                else { d[l] -= p; e[l] = g; }
                e[m] = 0.0;
            }
        }
    }
    if (had_issues) g_imtqlb_warned = true;
}

static void imtqlb_legacy(size_t n, real* d, real* e, real* bnd) {
    if (n == 1) return;
    bnd[0] = 1.0;
    size_t last = n - 1;
    for (size_t i = 1; i <= last; ++i) { bnd[i] = 0.0; e[i - 1] = e[i]; }
    e[last] = 0.0;
    size_t i = 0;
    for (size_t l = 0; l <= last; ++l) {
        size_t iteration = 0;
        while (iteration <= 30) {
            size_t m = l;
            while (m < n) {
                if (m == last) break;
                real test = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (compare(test, test + std::fabs(e[m]))) break;
                ++m;
            }
            real p = d[l];
            real f = bnd[l];
            if (m == l) {
                bool exchange = true;
                if (l > 0) {
                    i = l;
                    while (i >= 1 && exchange) {
                        if (p < d[i - 1]) { d[i] = d[i - 1]; bnd[i] = bnd[i - 1]; --i; }
                        else exchange = false;
                    }
                }
                if (exchange) i = 0;
                d[i] = p;
                bnd[i] = f;
                iteration = 31;
            } else {
                if (iteration == 30)
                    throw Error(E_IMTQLB, "svdlibrs/imtqlb: imtqlb no convergence to an eigenvalue after 30 iterations");
                ++iteration;
                real g = (d[l + 1] - p) / (2.0 * e[l]);
                real r = svd_pythag_legacy(g, 1.0);
                g = d[m] - p + e[l] / (g + svd_fsign(r, g));
                real s = 1.0, c = 1.0;
                p = 0.0;
                if (m == 0) throw Error(E_PANIC, "imtqlb: expected 'm' to be non-zero");
                i = m - 1;
                bool underflow = false;
                while (!underflow && i >= l) {
                    f = s * e[i];
                    real b = c * e[i];
                    r = svd_pythag_legacy(f, g);
                    e[i + 1] = r;
                    if (compare(r, 0.0)) { underflow = true; break; }
                    s = f / r;
                    c = g / r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    p = s * r;
                    d[i + 1] = g + p;
                    g = c * r - b;
                    f = bnd[i + 1];
                    bnd[i + 1] = s * bnd[i] + c * f;
                    bnd[i] = c * bnd[i] - s * f;
                    if (i == 0) break;
                    --i;
                }
                if (underflow) d[i + 1] -= p;
                else { d[l] -= p; e[l] = g; }
                e[m] = 0.0;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// startv / stpone / lanczos_step / purge / ortbnd / error_bound
// mod.rs:587-899 (identical in legacy.rs:1100-1540)
// ---------------------------------------------------------------------------
static real startv(const SMat& A, Work& w, size_t step, Store& store, uint32_t seed) {
    size_t n = w.ncols;
    real rnm2 = svd_ddot(w.w0.data(), w.w0.data(), n);
    for (int id = 0; id < 3; ++id) {
        if (id > 0 || step > 0 || compare(rnm2, 0.0)) start_vector(seed, w.w0.data(), n);
        w.w3 = w.w0;
        svd_opb(A, w.w3.data(), w.w0.data(), w.temp.data(), w.transposed);
        w.w3 = w.w0;
        rnm2 = svd_ddot(w.w3.data(), w.w3.data(), n);
        if (rnm2 > 0.0) break;
    }
    if (rnm2 <= 0.0) {
        char buf[128];
        snprintf(buf, sizeof buf, "svdlibrs/startv: rnm2 <= 0.0, rnm2 = %g", rnm2);
        throw Error(E_STARTV, buf);
    }
    if (step > 0) {
        for (size_t i = 0; i < step; ++i) {
            const real* v = store.retrq(i);
            svd_daxpy(-svd_ddot(w.w3.data(), v, n), v, w.w0.data(), n);
        }
        svd_daxpy(-svd_ddot(w.w4.data(), w.w0.data(), n), w.w2.data(), w.w0.data(), n);
        w.w3 = w.w0;
        real dot = svd_ddot(w.w3.data(), w.w3.data(), n);
        rnm2 = (dot <= EPS * rnm2) ? 0.0 : dot;
    }
    return std::sqrt(rnm2);
}

static void stpone(const SMat& A, Work& w, Store& store, uint32_t seed, real& rnm_out, real& tol_out) {
    size_t n = w.ncols;
    real rnm = startv(A, w, 0, store, seed);
    if (compare(rnm, 0.0)) throw Error(E_STPONE, "svdlibrs/stpone: rnm == 0.0");
    svd_datx(1.0 / rnm, w.w0.data(), w.w1.data(), n);
    svd_dscal(1.0 / rnm, w.w3.data(), n);
    svd_opb(A, w.w3.data(), w.w0.data(), w.temp.data(), w.transposed);
    w.alf[0] = svd_ddot(w.w0.data(), w.w3.data(), n);
    svd_daxpy(-w.alf[0], w.w1.data(), w.w0.data(), n);
    real t = svd_ddot(w.w0.data(), w.w3.data(), n);
    w.alf[0] += t;
    svd_daxpy(-t, w.w1.data(), w.w0.data(), n);
    w.w4 = w.w0;
    rnm = svd_norm(w.w4.data(), n);
    real anorm = rnm + std::fabs(w.alf[0]);
    rnm_out = rnm;
    tol_out = std::sqrt(EPS) * anorm;
}

static void ortbnd(Work& w, size_t step, real rnm, real eps1) {
    if (step < 1) return;
    if (!compare(rnm, 0.0) && step > 1) {
        w.oldeta[0] = (w.bet[1] * w.eta[1] + (w.alf[0] - w.alf[step]) * w.eta[0] -
                       w.bet[step] * w.oldeta[0]) / rnm + eps1;
        if (step > 2)
            for (size_t i = 1; i <= step - 2; ++i)
                w.oldeta[i] = (w.bet[i + 1] * w.eta[i + 1] + (w.alf[i] - w.alf[step]) * w.eta[i] +
                               w.bet[i] * w.eta[i - 1] - w.bet[step] * w.oldeta[i]) / rnm + eps1;
    }
    w.oldeta[step - 1] = eps1;
    std::swap(w.oldeta, w.eta);
    w.eta[step] = eps1;
}

static size_t g_purge_count = 0;

static void purge(size_t n, size_t ll, Work& w, size_t step, real& rnm, real tol, Store& store) {
    if (step < ll + 2) return;
    real reps = std::sqrt(EPS);
    real eps1 = EPS * std::sqrt((real)n);
    size_t k = svd_idamax(step - (ll + 1), w.eta.data()) + ll;
    if (std::fabs(w.eta[k]) > reps) {
        ++g_purge_count;
        real reps1 = eps1 / reps;
        int iteration = 0;
        bool flag = true;
        size_t nn = w.ncols;
        while (iteration < 2 && flag) {
            if (rnm > tol) {
                real tq = 0.0, tr = 0.0;
                for (size_t i = ll; i < step; ++i) {
                    const real* v = store.retrq(i);
                    real t = svd_ddot(v, w.w3.data(), nn);
                    tq += std::fabs(t);
                    svd_daxpy(-t, v, w.w1.data(), nn);
                    t = svd_ddot(v, w.w4.data(), nn);
                    tr += std::fabs(t);
                    svd_daxpy(-t, v, w.w0.data(), nn);
                }
                w.w3 = w.w1;
                real t = svd_ddot(w.w0.data(), w.w3.data(), nn);
                tr += std::fabs(t);
                svd_daxpy(-t, w.w1.data(), w.w0.data(), nn);
                w.w4 = w.w0;
                rnm = svd_norm(w.w4.data(), nn);
                if (tq <= reps1 && tr <= rnm * reps1) flag = false;
            }
            ++iteration;
        }
        for (size_t i = ll; i <= step; ++i) { w.eta[i] = eps1; w.oldeta[i] = eps1; }
    }
}

static size_t lanczos_step(const SMat& A, Work& w, size_t first, size_t last, size_t& ll, bool& enough,
                           real& rnm, real& tol, Store& store) {
    size_t n = w.ncols;
    real eps1 = EPS * std::sqrt((real)n);
    size_t j = first;
    while (j < last) {
        std::swap(w.w1, w.w2);
        std::swap(w.w3, w.w4);
        store.storq(j - 1, w.w2.data());
        if (j - 1 < MAXLL) store.storp(j - 1, w.w4.data());
        w.bet[j] = rnm;
        if (compare(rnm, 0.0)) {
            rnm = startv(A, w, j, store, 0);
            if (compare(rnm, 0.0)) enough = true;
        }
        if (enough) { std::swap(w.w1, w.w2); break; }
        svd_datx(1.0 / rnm, w.w0.data(), w.w1.data(), n);
        svd_dscal(1.0 / rnm, w.w3.data(), n);
        svd_opb(A, w.w3.data(), w.w0.data(), w.temp.data(), w.transposed);
        svd_daxpy(-rnm, w.w2.data(), w.w0.data(), n);
        w.alf[j] = svd_ddot(w.w0.data(), w.w3.data(), n);
        svd_daxpy(-w.alf[j], w.w1.data(), w.w0.data(), n);
        if (j <= MAXLL && std::fabs(w.alf[j - 1]) > 4.0 * std::fabs(w.alf[j])) ll = j;
        for (size_t i = 0; i < std::min(j - 1, ll); ++i) {
            real t = svd_ddot(store.retrp(i), w.w0.data(), n);
            svd_daxpy(-t, store.retrq(i), w.w0.data(), n);
            w.eta[i] = eps1;
            w.oldeta[i] = eps1;
        }
        real t = svd_ddot(w.w0.data(), w.w4.data(), n);
        svd_daxpy(-t, w.w2.data(), w.w0.data(), n);
        if (w.bet[j] > 0.0) w.bet[j] += t;
        t = svd_ddot(w.w0.data(), w.w3.data(), n);
        svd_daxpy(-t, w.w1.data(), w.w0.data(), n);
        w.alf[j] += t;
        w.w4 = w.w0;
        rnm = svd_norm(w.w4.data(), n);
        real anorm = w.bet[j] + std::fabs(w.alf[j]) + rnm;
        tol = std::sqrt(EPS) * anorm;
        ortbnd(w, j, rnm, eps1);
        purge(w.ncols, ll, w, j, rnm, tol, store);
        if (rnm <= tol) rnm = 0.0;
        ++j;
    }
    return j;
}

static size_t error_bound(bool& enough, real endl, real endr, real* ritz, real* bnd, size_t step,
                          real tol) {
    if (step == 0) throw Error(E_PANIC, "error_bound: expected 'step' to be non-zero");
    size_t mid = svd_idamax(step + 1, bnd);
    real e34 = eps34();
    size_t i = ((step + 1) + (step - 1)) / 2;
    while (i > mid + 1) {
        if (std::fabs(ritz[i - 1] - ritz[i]) < e34 * std::fabs(ritz[i]) && bnd[i] > tol && bnd[i - 1] > tol) {
            bnd[i - 1] = std::sqrt(bnd[i] * bnd[i] + bnd[i - 1] * bnd[i - 1]);
            bnd[i] = 0.0;
        }
        --i;
    }
    i = ((step + 1) - (step - 1)) / 2;
    while (i + 1 < mid) {
        if (std::fabs(ritz[i + 1] - ritz[i]) < e34 * std::fabs(ritz[i]) && bnd[i] > tol && bnd[i + 1] > tol) {
            bnd[i + 1] = std::sqrt(bnd[i] * bnd[i] + bnd[i + 1] * bnd[i + 1]);
            bnd[i] = 0.0;
        }
        ++i;
    }
    size_t neig = 0;
    real gapl = ritz[step] - ritz[0];
    for (size_t k = 0; k <= step; ++k) {
        real gap = gapl;
        if (k < step) gapl = ritz[k + 1] - ritz[k];
        gap = fmin_(gap, gapl);
        if (gap > bnd[k]) bnd[k] *= bnd[k] / gap;
        if (bnd[k] <= 16.0 * EPS * std::fabs(ritz[k])) {
            ++neig;
            if (!enough) enough = endl < ritz[k] && ritz[k] < endr;
        }
    }
    return neig;
}

// imtql2: current mod.rs:901-1028 (pythag as written, max iterations by
// sparsity) / legacy legacy.rs:1590-1700 (30 iterations).
static void imtql2(size_t nm, size_t n, real* d, real* e, real* z, const Mode& md) {
    size_t max_it = md.max_imtql2;
    if (n == 1) return;
    size_t last = n - 1;
    for (size_t i = 1; i < n; ++i) e[i - 1] = e[i];
    e[last] = 0.0;
    size_t nnm = n * nm;
    for (size_t l = 0; l < n; ++l) {
        size_t iteration = 0;
        while (iteration <= max_it) {
            size_t m = l;
            while (m < n) {
                if (m == last) break;
                real test = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (compare(test, test + std::fabs(e[m]))) break;
                ++m;
            }
            if (m == l) break;
            if (iteration == max_it) {
                char buf[160];
                snprintf(buf, sizeof buf,
                         "svdlibrs/imtql2: imtql2 no convergence to an eigenvalue after %zu iterations", max_it);
                throw Error(E_IMTQL2, buf);
            }
            ++iteration;
            real g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            real r = md.legacy ? svd_pythag_legacy(g, 1.0) : svd_pythag_current(g, 1.0);
            g = d[m] - d[l] + e[l] / (g + svd_fsign(r, g));
            real s = 1.0, c = 1.0, p = 0.0;
            size_t i = m - 1;
            bool underflow = false;
            while (!underflow && i >= l) {
                real f = s * e[i];
                real b = c * e[i];
                r = md.legacy ? svd_pythag_legacy(f, g) : svd_pythag_current(f, g);
                e[i + 1] = r;
                if (compare(r, 0.0)) underflow = true;
                else {
                    s = f / r;
                    c = g / r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    p = s * r;
                    d[i + 1] = g + p;
                    g = c * r - b;
                    for (size_t k = 0; k < nnm; k += n) {
                        size_t index = k + i;
                        f = z[index + 1];
                        z[index + 1] = s * z[index] + c * f;
                        z[index] = c * z[index] - s * f;
                    }
                    if (i == 0) break;
                    --i;
                }
            }
            if (underflow) d[i + 1] -= p;
            else { d[l] -= p; e[l] = g; }
            e[m] = 0.0;
        }
    }
    for (size_t l = 1; l < n; ++l) {
        size_t i = l - 1, k = i;
        real p = d[i];
        for (size_t j = l; j < n; ++j)
            if (d[j] < p) { k = j; p = d[j]; }
        if (k != i) {
            d[k] = d[i];
            d[i] = p;
            for (size_t j = 0; j < nnm; j += n) std::swap(z[j + i], z[j + k]);
        }
    }
}

// rotate_array, mod.rs:1030-1053 / legacy.rs:1702-1725
static void rotate_array(real* a, size_t n, size_t x) {
    size_t j = 0, start = 0;
    real t1 = a[0];
    for (size_t c = 0; c < n; ++c) {
        j = (j >= x) ? j - x : j + n - x;
        real t2 = a[j];
        a[j] = t1;
        if (j == start) { ++j; start = j; t1 = a[j]; }
        else t1 = t2;
    }
}

struct Trace {  // per-run internals exposed to the tests
    std::vector<real> alf, bet, ritz, bnd;
    size_t steps = 0, neig = 0, nsig = 0, purges = 0;
    real sparsity = 0.0;
    bool imtqlb_warned = false;
};

struct Raw {
    size_t d = 0, nsig = 0, ut_cols = 0, vt_cols = 0;
    std::vector<real> ut, s, vt;
};

// ritvec: current mod.rs:1056-1259; legacy legacy.rs:1766-1850
static Raw ritvec(const SMat& A, size_t dimensions, real kappa, Work& w, size_t steps, size_t neig,
                  Store& store, const Mode& md) {
    size_t js = steps + 1, jsq = js * js;
    std::vector<real> s(jsq, 0.0);
    for (size_t i = 0; i < jsq; i += js + 1) s[i] = 1.0;
    Raw R;
    size_t cols = w.ncols;
    std::vector<real> vt(cols * dimensions, 0.0);
    svd_dcopy(js, 0, w.alf.data(), vt.data());
    svd_dcopy(steps, 1, w.bet.data(), w.w5.data());
    imtql2(js, js, vt.data(), w.w5.data(), s.data(), md);

    std::vector<std::vector<real>> rows;  // selected Vt rows, in output order
    size_t nsig = 0;
    if (!md.legacy) {
        real ae = md.adaptive_eps;
        real max_eig = 0.0;
        for (real v : vt) max_eig = fmax_(max_eig, std::fabs(v));
        real akappa = md.sparsity > 0.99 ? kappa * 10.0 : kappa;
        std::vector<size_t> sig;
        for (size_t k = 0; k < js; ++k) {
            real rel = akappa * fmax_(std::fabs(w.ritz[k]), max_eig * ae);
            if (w.bnd[k] <= rel && k + 1 > js - neig) sig.push_back(k);
        }
        nsig = sig.size();
        size_t d = std::min(dimensions, nsig);
        for (size_t r = 0; r < d; ++r) {
            size_t k = sig[r];
            std::vector<real> vec(cols, 0.0);
            for (size_t i = 0; i < js; ++i) {
                real c = s[k * js + i];
                if (std::fabs(c) > ae) {
                    const real* q = store.retrq(i);
                    for (size_t j = 0; j < cols; ++j) vec[j] += c * q[j];
                }
            }
            rows.push_back(std::move(vec));
        }
    } else {
        size_t x = 0, id2 = jsq - js;
        for (size_t k = 0; k < js; ++k) {
            if (w.bnd[k] <= kappa * std::fabs(w.ritz[k]) && k + 1 > js - neig) {
                x = (x == 0) ? dimensions - 1 : x - 1;
                size_t off = x * cols;
                std::fill(vt.begin() + off, vt.begin() + off + cols, 0.0);
                size_t idx = id2 + js;
                for (size_t i = 0; i < js; ++i) {
                    idx -= js;
                    if (s[idx] != 0.0) {
                        const real* q = store.retrq(i);
                        for (size_t j = 0; j < cols; ++j) vt[j + off] += s[idx] * q[j];
                    }
                }
                ++nsig;
            }
            ++id2;
        }
        if (x > 0) rotate_array(vt.data(), vt.size(), x * cols);
        size_t d = std::min(dimensions, nsig);
        for (size_t r = 0; r < d; ++r)
            rows.emplace_back(vt.begin() + r * cols, vt.begin() + (r + 1) * cols);
    }
    size_t d = rows.size();
    R.d = d;
    R.nsig = nsig;
    R.ut_cols = w.nrows;
    R.vt_cols = cols;
    R.s.assign(d, 0.0);
    R.ut.assign(d * w.nrows, 0.0);
    R.vt.assign(d * cols, 0.0);
    std::vector<real> tmp(cols);
    for (size_t i = 0; i < d; ++i) {
        const real* v = rows[i].data();
        real* ut = R.ut.data() + i * w.nrows;
        svd_opb(A, v, tmp.data(), w.temp.data(), w.transposed);
        A.svd_opa(v, ut, w.transposed);
        real t = svd_ddot(v, tmp.data(), cols);
        if (!md.legacy) {
            real sval = std::sqrt(fmax_(t, 0.0));
            R.s[i] = sval;
            real ae = md.adaptive_eps;
            if (sval > ae) svd_dscal(1.0 / sval, ut, w.nrows);
            else svd_dscal(1.0 / fmax_(sval, ae), ut, w.nrows);
        } else {
            real sval = std::sqrt(t);
            R.s[i] = sval;
            svd_dscal(1.0 / sval, ut, w.nrows);
        }
        std::memcpy(R.vt.data() + i * cols, v, cols * sizeof(real));
    }
    return R;
}

static size_t lanso(const SMat& A, size_t dim, size_t iterations, real endl, real endr, Work& w,
                    size_t& neig, Store& store, uint32_t seed, const Mode& md, Trace* tr) {
    real rnm, tol;
    stpone(A, w, store, seed, rnm, tol);
    real eps1 = (md.legacy ? EPS : md.adaptive_eps) * std::sqrt((real)w.ncols);
    w.eta[0] = eps1;
    w.oldeta[0] = eps1;
    size_t ll = 0, first = 1;
    size_t last = std::min(iterations, std::max(dim, (size_t)8) + dim);
    bool enough = false;
    size_t j = 0, intro = 0;
    while (!enough) {
        if (rnm <= tol) rnm = 0.0;
        size_t steps = lanczos_step(A, w, first, last, ll, enough, rnm, tol, store);
        j = enough ? steps - 1 : last - 1;
        first = j + 1;
        w.bet[first] = rnm;
        size_t l = 0;
        for (size_t it = 0; it < j; ++it) {
            if (l > j) break;
            size_t i = l;
            while (i <= j) {
                bool split = md.legacy ? compare(w.bet[i + 1], 0.0) : std::fabs(w.bet[i + 1]) <= md.adaptive_eps;
                if (split) break;
                ++i;
            }
            i = std::min(i, j);
            size_t sz = i - l;
            svd_dcopy(sz + 1, l, w.alf.data(), w.ritz.data());
            svd_dcopy(sz, l + 1, w.bet.data(), w.w5.data());
            if (md.legacy) imtqlb_legacy(sz + 1, w.ritz.data() + l, w.w5.data() + l, w.bnd.data() + l);
            else imtqlb_current(sz + 1, w.ritz.data() + l, w.w5.data() + l, w.bnd.data() + l, md.max_imtqlb);
            for (size_t m = l; m <= i; ++m) w.bnd[m] = rnm * std::fabs(w.bnd[m]);
            l = i + 1;
        }
        insert_sort(j + 1, w.ritz.data(), w.bnd.data());
        neig = error_bound(enough, endl, endr, w.ritz.data(), w.bnd.data(), j, tol);
        if (neig < dim) {
            if (neig == 0) { last = first + 9; intro = first; }
            else {
                size_t ext = std::max<size_t>(3, 1 + ((j - intro) * (dim - neig)) / neig);
                last = first + ext + (md.legacy ? 0 : md.extra_steps);
            }
            last = std::min(last, iterations);
        } else enough = true;
        enough = enough || first >= iterations;
    }
    store.storq(j, w.w1.data());
    if (tr) {
        tr->alf.assign(w.alf.begin(), w.alf.begin() + j + 1);
        tr->bet.assign(w.bet.begin(), w.bet.begin() + j + 2);
        tr->ritz.assign(w.ritz.begin(), w.ritz.begin() + j + 1);
        tr->bnd.assign(w.bnd.begin(), w.bnd.begin() + j + 1);
    }
    return j;
}

struct Las2Result {
    Raw raw;
    size_t dimensions = 0, iterations = 0, nnz = 0, steps = 0, neig = 0;
    bool transposed = false;
    real kappa = 0.0;
    uint32_t seed = 0;
};

// svd_las2: mod.rs:104-189 / legacy svdLAS2 legacy.rs:569-654
static Las2Result svd_las2(const SMat& A, size_t dimensions, size_t iterations, real endl, real endr,
                           real kappa, uint32_t seed, bool legacy, Trace* tr) {
    if (seed == 0) seed = std::random_device{}();
    size_t mn = std::min(A.nrows(), A.ncols());
    if (dimensions == 0 || dimensions > mn) dimensions = mn;
    if (iterations == 0 || iterations > mn) iterations = mn;
    else if (iterations < dimensions) iterations = dimensions;
    if (dimensions < 2) {
        char buf[128];
        snprintf(buf, sizeof buf, legacy ? "svdlibrs/svdLas2: svdLAS2: insufficient dimensions: %zu"
                                         : "svdlibrs/svdLas2: svd_las2: insufficient dimensions: %zu", dimensions);
        throw Error(E_LAS2, buf);
    }
    bool transposed = (real)A.ncols() >= (real)A.nrows() * 1.2;
    size_t nrows = transposed ? A.ncols() : A.nrows();
    size_t ncols = transposed ? A.nrows() : A.ncols();
    Work w(nrows, ncols, transposed, iterations);
    Store store(ncols);
    Mode md = make_mode(A, legacy);
    g_legacy_blas = legacy;
    g_purge_count = 0;
    g_imtqlb_warned = false;
    size_t neig = 0;
    size_t steps = lanso(A, dimensions, iterations, endl, endr, w, neig, store, seed, md, tr);
    if (tr) {
        tr->steps = steps;
        tr->neig = neig;
        tr->purges = g_purge_count;
        tr->sparsity = sparsity_of(A);
    }
    real kap = fmax_(std::fabs(kappa), eps34());
    Las2Result res;
    res.raw = ritvec(A, dimensions, kap, w, steps, neig, store, md);
    if (transposed) {
        std::swap(res.raw.ut, res.raw.vt);
        std::swap(res.raw.ut_cols, res.raw.vt_cols);
    }
    res.dimensions = dimensions;
    res.iterations = iterations;
    res.nnz = A.nnz();
    res.steps = steps;
    res.neig = neig;
    res.transposed = transposed;
    res.kappa = kap;
    res.seed = seed;
    if (tr) {
        tr->steps = steps;
        tr->neig = neig;
        tr->nsig = res.raw.nsig;
        tr->purges = g_purge_count;
        tr->sparsity = sparsity_of(A);
        tr->imtqlb_warned = g_imtqlb_warned;
    }
    g_legacy_blas = false;
    return res;
}

// ---------------------------------------------------------------------------
// Randomized SVD, src/randomized/mod.rs:24-199, on a MaskedCSRMatrix
// (the only SMat type whose dense products exist, masked.rs:265-733).
// Dense matrices are column-major (nalgebra DMatrix layout).
// ---------------------------------------------------------------------------
struct DMatrix {
    size_t r = 0, c = 0;
    std::vector<real> a;  // column-major
    DMatrix() {}
    DMatrix(size_t r_, size_t c_) : r(r_), c(c_), a(r_ * c_, 0.0) {}
    real& operator()(size_t i, size_t j) { return a[i + j * r]; }
    real operator()(size_t i, size_t j) const { return a[i + j * r]; }
};

// masked multiply_with_dense, masked.rs:265-471.  compat_d3 reproduces the
// row pointer dense.as_ptr().add(i*dense_cols) of masked.rs:388-393.
static void masked_multiply_with_dense(const MaskedOp& M, const DMatrix& dense, DMatrix& result, bool transpose_self,
                                       bool compat_d3) {
    const Compressed* a = M.a;
    const uint64_t* p = a->ptr.data();
    const uint64_t* ci = a->idx.data();
    const real* v = a->val.data();
    size_t l = dense.c;
    if (!transpose_self) {
        size_t rows = a->nmajor;
        result = DMatrix(rows, l);
#pragma omp parallel for schedule(dynamic, 64) num_threads(g_threads) if (g_threads > 1)
        for (size_t row = 0; row < rows; ++row) {
            std::vector<real> acc(l, 0.0);
            for (uint64_t j = p[row]; j < p[row + 1]; ++j) {
                int64_t mc = M.o2m[ci[j]];
                if (mc < 0) continue;
                real val = v[j];
                for (size_t c = 0; c < l; ++c) acc[c] += val * dense((size_t)mc, c);
            }
            for (size_t c = 0; c < l; ++c) result(row, c) = acc[c];
        }
        return;
    }
    size_t nrows = a->nmajor, nm = M.ncols();
    result = DMatrix(nm, l);
    size_t cs = determine_chunk_size(nrows);
    size_t nch = (nrows + cs - 1) / cs;
    std::vector<std::vector<real>> loc(nch);
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads) if (g_threads > 1)
    for (size_t ch = 0; ch < nch; ++ch) {
        std::vector<real> lr(nm * l, 0.0);
        size_t s = ch * cs, e = std::min(s + cs, nrows);
        std::vector<real> drow(l);
        for (size_t i = s; i < e; ++i) {
            for (size_t c = 0; c < l; ++c) {
                if (compat_d3) {
                    size_t flat = i * l + c;  // column-major storage read as row-major
                    drow[c] = flat < dense.a.size() ? dense.a[flat] : 0.0;
                } else drow[c] = dense(i, c);
            }
            for (uint64_t j = p[i]; j < p[i + 1]; ++j) {
                int64_t mc = M.o2m[ci[j]];
                if (mc < 0) continue;
                real val = v[j];
                size_t base = (size_t)mc * l;
                for (size_t c = 0; c < l; ++c) lr[base + c] += val * drow[c];
            }
        }
        loc[ch].swap(lr);
    }
    for (size_t ch = 0; ch < nch; ++ch)
        for (size_t r = 0; r < nm; ++r)
            for (size_t c = 0; c < l; ++c) {
                real val = loc[ch][r * l + c];
                if (val != 0.0) result(r, c) += val;
            }
}

// multiply_transposed_by_dense (B = Q^T A), masked.rs:616-733
static void masked_multiply_transposed_by_dense(const MaskedOp& M, const DMatrix& q, DMatrix& result) {
    const Compressed* a = M.a;
    const uint64_t* p = a->ptr.data();
    const uint64_t* ci = a->idx.data();
    const real* v = a->val.data();
    size_t qc = q.c, nm = M.ncols(), nrows = a->nmajor;
    result = DMatrix(qc, nm);
    size_t cs = determine_chunk_size(nrows);
    size_t nch = (nrows + cs - 1) / cs;
    std::vector<std::vector<real>> loc(nch);
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads) if (g_threads > 1)
    for (size_t ch = 0; ch < nch; ++ch) {
        std::vector<real> lr(qc * nm, 0.0);  // column-major qc x nm
        size_t s = ch * cs, e = std::min(s + cs, nrows);
        for (size_t row = s; row < e; ++row)
            for (uint64_t idx = p[row]; idx < p[row + 1]; ++idx) {
                int64_t mc = M.o2m[ci[idx]];
                if (mc < 0) continue;
                real sv = v[idx];
                for (size_t c = 0; c < qc; ++c) lr[c + (size_t)mc * qc] += q(row, c) * sv;
            }
        loc[ch].swap(lr);
    }
    for (size_t ch = 0; ch < nch; ++ch)
        for (size_t cc = 0; cc < nm; ++cc)
            for (size_t r = 0; r < qc; ++r) {
                real val = loc[ch][r + cc * qc];
                if (val != 0.0) result(r, cc) += val;
            }
}

// Thin Householder QR returning Q (rows x min(rows, cols)), standing in for
// nalgebra's z.qr().q() (randomized/mod.rs:96-101,122-125,143-144).
static DMatrix thin_q(const DMatrix& X) {
    size_t m = X.r, n = X.c, k = std::min(m, n);
    DMatrix A = X;
    std::vector<std::vector<real>> vs(k);
    std::vector<real> betas(k, 0.0);
    for (size_t j = 0; j < k; ++j) {
        real norm = 0.0;
        for (size_t i = j; i < m; ++i) norm += A(i, j) * A(i, j);
        norm = std::sqrt(norm);
        std::vector<real> v(m - j, 0.0);
        if (norm == 0.0) { vs[j] = v; betas[j] = 0.0; continue; }
        real alpha = A(j, j) >= 0 ? -norm : norm;
        for (size_t i = j; i < m; ++i) v[i - j] = A(i, j);
        v[0] -= alpha;
        real vn = 0.0;
        for (real t : v) vn += t * t;
        real beta = vn > 0 ? 2.0 / vn : 0.0;
        for (size_t c = j; c < n; ++c) {
            real dot = 0.0;
            for (size_t i = j; i < m; ++i) dot += v[i - j] * A(i, c);
            dot *= beta;
            for (size_t i = j; i < m; ++i) A(i, c) -= dot * v[i - j];
        }
        vs[j] = v;
        betas[j] = beta;
    }
    DMatrix Q(m, k);
    for (size_t j = 0; j < k; ++j) Q(j, j) = 1.0;
    for (size_t jj = k; jj-- > 0;) {
        const std::vector<real>& v = vs[jj];
        real beta = betas[jj];
        if (beta == 0.0) continue;
        for (size_t c = 0; c < k; ++c) {
            real dot = 0.0;
            for (size_t i = jj; i < m; ++i) dot += v[i - jj] * Q(i, c);
            dot *= beta;
            for (size_t i = jj; i < m; ++i) Q(i, c) -= dot * v[i - jj];
        }
    }
    return Q;
}

// normalize_columns, randomized/mod.rs:239-293
static void normalize_columns(DMatrix& M) {
    for (size_t j = 0; j < M.c; ++j) {
        real norm = 0.0;
        for (size_t i = 0; i < M.r; ++i) norm += M(i, j) * M(i, j);
        norm = std::sqrt(norm);
        if (norm > 1e-10) {
            real scale = 1.0 / norm;
            for (size_t i = 0; i < M.r; ++i) M(i, j) *= scale;
        }
    }
}

// One-sided Jacobi SVD of B (l x n): columns of B^T are orthogonalised.
// Returns U_B (l x r), sigma (r, descending), V_B^T (r x n), r = min(l, n);
// stands in for nalgebra's b.svd(true, true) (randomized/mod.rs:160).
static void jacobi_svd(const DMatrix& B, DMatrix& U, std::vector<real>& sig, DMatrix& Vt) {
    size_t l = B.r, n = B.c;
    bool wide = n >= l;
    // Work on W (p x q) with p >= q: W = B^T if wide else B
    size_t p = wide ? n : l, q = wide ? l : n;
    DMatrix W(p, q), V(q, q);
    for (size_t i = 0; i < p; ++i)
        for (size_t j = 0; j < q; ++j) W(i, j) = wide ? B(j, i) : B(i, j);
    for (size_t j = 0; j < q; ++j) V(j, j) = 1.0;
    for (int sweep = 0; sweep < 80; ++sweep) {
        real off = 0.0;
        for (size_t a = 0; a + 1 < q; ++a)
            for (size_t b = a + 1; b < q; ++b) {
                real al = 0, be = 0, ga = 0;
                for (size_t i = 0; i < p; ++i) {
                    al += W(i, a) * W(i, a);
                    be += W(i, b) * W(i, b);
                    ga += W(i, a) * W(i, b);
                }
                if (ga == 0.0) continue;
                real conv = std::fabs(ga) / std::sqrt(al * be);
                if (!(conv > 1e-15)) continue;
                off = std::max(off, conv);
                real zeta = (be - al) / (2.0 * ga);
                real t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                real c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
                for (size_t i = 0; i < p; ++i) {
                    real x = W(i, a), y = W(i, b);
                    W(i, a) = c * x - s * y;
                    W(i, b) = s * x + c * y;
                }
                for (size_t i = 0; i < q; ++i) {
                    real x = V(i, a), y = V(i, b);
                    V(i, a) = c * x - s * y;
                    V(i, b) = s * x + c * y;
                }
            }
        if (off < 1e-15) break;
    }
    std::vector<real> nrm(q);
    for (size_t j = 0; j < q; ++j) {
        real s2 = 0;
        for (size_t i = 0; i < p; ++i) s2 += W(i, j) * W(i, j);
        nrm[j] = std::sqrt(s2);
    }
    std::vector<size_t> ord(q);
    for (size_t j = 0; j < q; ++j) ord[j] = j;
    std::stable_sort(ord.begin(), ord.end(), [&](size_t x, size_t y) { return nrm[x] > nrm[y]; });
    size_t r = q;
    sig.assign(r, 0.0);
    // W = Ubig * diag(nrm) (p x q), V (q x q):  M = W V^T
    DMatrix Ubig(p, r), Vs(q, r);
    for (size_t k = 0; k < r; ++k) {
        size_t j = ord[k];
        sig[k] = nrm[j];
        for (size_t i = 0; i < p; ++i) Ubig(i, k) = nrm[j] > 0 ? W(i, j) / nrm[j] : 0.0;
        for (size_t i = 0; i < q; ++i) Vs(i, k) = V(i, j);
    }
    if (wide) {  // B^T = Ubig S Vs^T  ->  B = Vs S Ubig^T
        U = Vs;  // l x r
        Vt = DMatrix(r, n);
        for (size_t k = 0; k < r; ++k)
            for (size_t i = 0; i < n; ++i) Vt(k, i) = Ubig(i, k);
    } else {  // B = Ubig S Vs^T
        U = Ubig;
        Vt = DMatrix(r, n);
        for (size_t k = 0; k < r; ++k)
            for (size_t i = 0; i < n; ++i) Vt(k, i) = Vs(i, k);
    }
}

struct RandResult {
    size_t d = 0, m = 0, n = 0;
    std::vector<real> u;   // m x d row-major
    std::vector<real> s;   // d
    std::vector<real> vt;  // d x n row-major
    // wall time by what it scales with: sparse products (nnz), work on
    // m-row dense matrices (rows), work on n-row matrices and the small SVD (fixed)
    double t_sparse = 0, t_rows = 0, t_fixed = 0;
};

static double wall() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// compute_column_means (masked.rs:240-263): sums of the masked columns over
// the rows, times 1/nrows
static std::vector<real> column_means(const MaskedOp& M) {
    const Compressed* a = M.a;
    std::vector<real> mu(M.ncols(), 0.0);
    for (size_t i = 0; i < a->nmajor; ++i)
        for (uint64_t j = a->ptr[i]; j < a->ptr[i + 1]; ++j) {
            int64_t mc = M.o2m[a->idx[j]];
            if (mc >= 0) mu[(size_t)mc] += a->val[j];
        }
    const real rc = 1.0 / (real)a->nmajor;
    for (real& v : mu) v *= rc;
    return mu;
}

// Products of the centred matrix A - 1 mu^T (mean_center, mod.rs:46-53), by
// the rank-1 corrections A X - 1 (mu^T X) and A^T Y - mu (1^T Y).  The crate's
// own adjustments (masked.rs:496-509, 793-809) differ from this algebra.
static void center_rows(DMatrix& y, const DMatrix& x, const std::vector<real>& mu) {
    for (size_t c = 0; c < y.c; ++c) {
        real t = 0.0;
        for (size_t j = 0; j < mu.size(); ++j) t += mu[j] * x(j, c);
        for (size_t i = 0; i < y.r; ++i) y(i, c) -= t;
    }
}
static void center_cols(DMatrix& z, const DMatrix& y, const std::vector<real>& mu) {
    for (size_t c = 0; c < z.c; ++c) {
        real t = 0.0;
        for (size_t i = 0; i < y.r; ++i) t += y(i, c);
        for (size_t j = 0; j < z.r; ++j) z(j, c) -= mu[j] * t;
    }
}

// normalizer: 0 = QR, 1 = LU (column normalisation), 2 = None
static RandResult randomized_svd(const MaskedOp& M, size_t target_rank, size_t n_oversamples, size_t n_power_iters,
                                 int normalizer, const double* omega_rowmajor, bool compat_d3,
                                 bool mean_center = false) {
    RandResult R;
    size_t m = M.nrows(), n = M.ncols();
    std::vector<real> mu;
    if (mean_center) mu = column_means(M);
    size_t rank = std::min(target_rank, std::min(m, n));
    size_t l = rank + n_oversamples;
    DMatrix omega(n, l);
    for (size_t i = 0; i < n; ++i)
        for (size_t c = 0; c < l; ++c) omega(i, c) = (real)omega_rowmajor[i * l + c];  // T::from_f64
    DMatrix y;
    double t = wall();
    auto lap = [&](double& acc) { double now = wall(); acc += now - t; t = now; };
    masked_multiply_with_dense(M, omega, y, false, compat_d3);
    if (mean_center) center_rows(y, omega, mu);
    lap(R.t_sparse);
    if (n_power_iters > 0) {
        DMatrix z;
        for (size_t it = 0; it < n_power_iters; ++it) {
            masked_multiply_with_dense(M, y, z, true, compat_d3);
            if (mean_center) center_cols(z, y, mu);
            lap(R.t_sparse);
            if (normalizer == 0) z = thin_q(z);
            else if (normalizer == 1) normalize_columns(z);
            lap(R.t_fixed);
            masked_multiply_with_dense(M, z, y, false, compat_d3);
            if (mean_center) center_rows(y, z, mu);
            lap(R.t_sparse);
            if (normalizer == 0) y = thin_q(y);
            else if (normalizer == 1) normalize_columns(y);
            lap(R.t_rows);
        }
    }
    DMatrix Q = thin_q(y);
    lap(R.t_rows);
    DMatrix B;
    masked_multiply_transposed_by_dense(M, Q, B);
    if (mean_center) {  // B = Q^T (A - 1 mu^T): row c of B loses (1^T Q e_c) mu^T
        for (size_t c = 0; c < B.r; ++c) {
            real t = 0.0;
            for (size_t i = 0; i < Q.r; ++i) t += Q(i, c);
            for (size_t j = 0; j < B.c; ++j) B(c, j) -= t * mu[j];
        }
    }
    lap(R.t_sparse);
    DMatrix Ub, Vt;
    std::vector<real> sig;
    jacobi_svd(B, Ub, sig, Vt);
    lap(R.t_fixed);
    size_t r = sig.size();
    size_t actual = std::min(target_rank, r);
    R.d = actual; R.m = m; R.n = n;
    R.u.assign(m * actual, 0.0);
    for (size_t i = 0; i < m; ++i)
        for (size_t k = 0; k < actual; ++k) {
            real acc = 0.0;
            for (size_t j = 0; j < Q.c; ++j) acc += Q(i, j) * Ub(j, k);
            R.u[i * actual + k] = acc;
        }
    lap(R.t_rows);
    R.s.assign(sig.begin(), sig.begin() + actual);
    R.vt.assign(actual * n, 0.0);
    for (size_t k = 0; k < actual; ++k)
        for (size_t i = 0; i < n; ++i) R.vt[k * n + i] = Vt(k, i);
    return R;
}

}  // namespace orc

// ===========================================================================
// C interface for the Python test harness (oracle/oracle.py)
// ===========================================================================
extern "C" {

static thread_local std::string g_orc_err;
static thread_local orc::Trace g_last_trace;

const char* orc_last_error() { return g_orc_err.c_str(); }

void orc_set_threads(int t) { orc::g_threads = t < 1 ? 1 : t; }

// ChaCha block for known-answer tests.
void orc_chacha_block(const uint8_t key[32], uint64_t counter, uint64_t stream, int rounds, uint32_t out[16]) {
    uint32_t k[8];
    for (int i = 0; i < 8; ++i)
        k[i] = (uint32_t)key[4 * i] | ((uint32_t)key[4 * i + 1] << 8) | ((uint32_t)key[4 * i + 2] << 16) |
               ((uint32_t)key[4 * i + 3] << 24);
    orc::chacha_block(k, counter, stream, rounds, out);
}

// sizeof(T): 8 for the f64 build, 4 for the f32 build (-DORC_F32)
int orc_real_bytes() { return (int)sizeof(orc::real); }

void orc_start_vector(uint32_t seed, double* out, size_t n) {
    std::vector<orc::real> w(n);
    orc::start_vector(seed, w.data(), n);
    for (size_t i = 0; i < n; ++i) out[i] = w[i];
}

#ifndef ORC_F32
double orc_pythag(double a, double b, int legacy) {
    return legacy ? orc::svd_pythag_legacy(a, b) : orc::svd_pythag_current(a, b);
}

// Tridiagonal eigen-solver entry points, for unit tests of the host/device
// split.  d (n), e (n, e[0] arbitrary), bnd (n); z (n*n row-major).
int orc_imtqlb(size_t n, double* d, double* e, double* bnd, int legacy, size_t max_it) {
    try {
        if (legacy) orc::imtqlb_legacy(n, d, e, bnd);
        else orc::imtqlb_current(n, d, e, bnd, max_it);
        return 0;
    } catch (orc::Error& ex) { g_orc_err = ex.what(); return ex.code; }
}
int orc_imtql2(size_t n, double* d, double* e, double* z, int legacy, size_t max_it) {
    orc::Mode md;
    md.legacy = legacy != 0;
    md.max_imtql2 = max_it;
    try { orc::imtql2(n, n, d, e, z, md); return 0; }
    catch (orc::Error& ex) { g_orc_err = ex.what(); return ex.code; }
}
#endif

struct orc_las2_out {
    uint64_t d, ut_rows, ut_cols, vt_rows, vt_cols;
    double* ut;
    double* s;
    double* vt;
    uint64_t dimensions, iterations, nnz, lanczos_steps, ritz_values_stabilized, significant_values,
        singular_values;
    int32_t transposed;
    double kappa;
    uint32_t random_seed;
    // trace
    uint64_t steps;
    double* alf;  // steps+1
    double* bet;  // steps+2
    double* ritz;
    double* bnd;
    uint64_t purges;
    double sparsity;
    int32_t imtqlb_warned;
    int32_t masked_would_panic;
};

extern "C++" {
template <typename V>
static double* dup_vec(const V& v) {
    double* p = (double*)std::malloc(std::max<size_t>(1, v.size()) * sizeof(double));
    for (size_t i = 0; i < v.size(); ++i) p[i] = (double)v[i];
    return p;
}
}

void orc_las2_free(orc_las2_out* o) {
    std::free(o->ut); std::free(o->s); std::free(o->vt);
    std::free(o->alf); std::free(o->bet); std::free(o->ritz); std::free(o->bnd);
    std::memset(o, 0, sizeof(*o));
}

// kind: 0 CSR, 1 CSC, 2 COO (ptr = row ids, idx = col ids), 3 masked CSR (mask of ncols bytes)
int orc_las2(int kind, uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* ptr, const uint64_t* idx,
             const double* val, const uint8_t* mask, uint64_t dimensions, uint64_t iterations, double endl,
             double endr, double kappa, uint32_t seed, int legacy, orc_las2_out* out) {
    std::memset(out, 0, sizeof(*out));
    try {
        orc::Compressed cm;
        std::unique_ptr<orc::SMat> op;
        orc::CooOp* coo = nullptr;
        orc::MaskedOp* msk = nullptr;
        if (kind == 0 || kind == 3) {
            cm.nmajor = nrows; cm.nminor = ncols;
            cm.ptr.assign(ptr, ptr + nrows + 1);
            cm.idx.assign(idx, idx + nnz);
            cm.val.assign(val, val + nnz);
            if (kind == 0) op.reset(new orc::CsrOp(&cm, legacy != 0));
            else { msk = new orc::MaskedOp(&cm, mask); op.reset(msk); }
        } else if (kind == 1) {
            cm.nmajor = ncols; cm.nminor = nrows;
            cm.ptr.assign(ptr, ptr + ncols + 1);
            cm.idx.assign(idx, idx + nnz);
            cm.val.assign(val, val + nnz);
            op.reset(new orc::CscOp(&cm));
        } else if (kind == 2) {
            coo = new orc::CooOp();
            coo->m = nrows; coo->n = ncols;
            coo->r.assign(ptr, ptr + nnz);
            coo->c.assign(idx, idx + nnz);
            coo->v.assign(val, val + nnz);
            op.reset(coo);
        } else { g_orc_err = "bad kind"; return orc::E_UNSUPPORTED; }
        orc::Trace& tr = g_last_trace;
        tr = orc::Trace();
        orc::Las2Result r = orc::svd_las2(*op, dimensions, iterations, endl, endr, kappa, seed, legacy != 0, &tr);
        out->d = r.raw.d;
        out->ut_rows = r.raw.d; out->ut_cols = r.raw.ut_cols;
        out->vt_rows = r.raw.d; out->vt_cols = r.raw.vt_cols;
        out->ut = dup_vec(r.raw.ut); out->s = dup_vec(r.raw.s); out->vt = dup_vec(r.raw.vt);
        out->dimensions = r.dimensions; out->iterations = r.iterations; out->nnz = r.nnz;
        out->lanczos_steps = r.steps + 1;
        out->ritz_values_stabilized = r.neig;
        out->significant_values = r.raw.d;
        out->singular_values = r.raw.nsig;
        out->transposed = r.transposed;
        out->kappa = r.kappa;
        out->random_seed = r.seed;
        out->steps = tr.steps;
        out->alf = dup_vec(tr.alf); out->bet = dup_vec(tr.bet);
        out->ritz = dup_vec(tr.ritz); out->bnd = dup_vec(tr.bnd);
        out->purges = tr.purges;
        out->sparsity = tr.sparsity;
        out->imtqlb_warned = tr.imtqlb_warned;
        out->masked_would_panic = msk ? msk->would_panic : 0;
        return 0;
    } catch (orc::Error& ex) {
        g_orc_err = ex.what();
        out->steps = g_last_trace.steps;
        out->lanczos_steps = g_last_trace.steps + 1;
        out->ritz_values_stabilized = g_last_trace.neig;
        out->purges = g_last_trace.purges;
        out->sparsity = g_last_trace.sparsity;
        return ex.code;
    } catch (std::exception& ex) {
        g_orc_err = ex.what();
        return orc::E_PANIC;
    }
}

// Operator application y = A x (or A^T x) through the SMat of `kind`.
int orc_opa(int kind, uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* ptr, const uint64_t* idx,
            const double* val, const uint8_t* mask, const double* x, double* y, int transposed, int legacy) {
    try {
        orc::Compressed cm;
        std::unique_ptr<orc::SMat> op;
        if (kind == 0 || kind == 3) {
            cm.nmajor = nrows; cm.nminor = ncols;
            cm.ptr.assign(ptr, ptr + nrows + 1);
            cm.idx.assign(idx, idx + nnz);
            cm.val.assign(val, val + nnz);
            if (kind == 0) op.reset(new orc::CsrOp(&cm, legacy != 0));
            else op.reset(new orc::MaskedOp(&cm, mask));
        } else if (kind == 1) {
            cm.nmajor = ncols; cm.nminor = nrows;
            cm.ptr.assign(ptr, ptr + ncols + 1);
            cm.idx.assign(idx, idx + nnz);
            cm.val.assign(val, val + nnz);
            op.reset(new orc::CscOp(&cm));
        } else if (kind == 2) {
            auto* coo = new orc::CooOp();
            coo->m = nrows; coo->n = ncols;
            coo->r.assign(ptr, ptr + nnz);
            coo->c.assign(idx, idx + nnz);
            coo->v.assign(val, val + nnz);
            op.reset(coo);
        } else return orc::E_UNSUPPORTED;
        const size_t nx = transposed ? nrows : (kind == 3 ? op->ncols() : ncols);
        const size_t ny = transposed ? (kind == 3 ? op->ncols() : ncols) : nrows;
        std::vector<orc::real> xr(x, x + nx), yr(ny);
        op->svd_opa(xr.data(), yr.data(), transposed != 0);
        for (size_t i = 0; i < ny; ++i) y[i] = yr[i];
        return 0;
    } catch (std::exception& ex) { g_orc_err = ex.what(); return orc::E_PANIC; }
}

// Masked maps and nnz, masked.rs:21-102.
int orc_masked_maps(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* ptr, const uint64_t* idx,
                    const uint8_t* mask, int64_t* m2o, uint64_t* n_masked, int64_t* o2m, uint64_t* masked_nnz) {
    orc::Compressed cm;
    cm.nmajor = nrows; cm.nminor = ncols;
    cm.ptr.assign(ptr, ptr + nrows + 1);
    cm.idx.assign(idx, idx + nnz);
    cm.val.assign(nnz, 0.0);
    orc::MaskedOp M(&cm, mask);
    *n_masked = M.m2o.size();
    for (size_t i = 0; i < M.m2o.size(); ++i) m2o[i] = M.m2o[i];
    for (size_t i = 0; i < ncols; ++i) o2m[i] = M.o2m[i];
    *masked_nnz = M.nnz();
    return 0;
}

// Masked dense products.  Dense inputs / outputs are row-major here.
// op 0: R (m x l) = A X (X: nmasked x l); op 1: R (nmasked x l) = A^T X (X: m x l);
// op 2: R (l x nmasked) = X^T A (X: m x l).
int orc_masked_dense(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* ptr, const uint64_t* idx,
                     const double* val, const uint8_t* mask, int op, const double* X, uint64_t l, double* R,
                     int compat_d3) {
    orc::Compressed cm;
    cm.nmajor = nrows; cm.nminor = ncols;
    cm.ptr.assign(ptr, ptr + nrows + 1);
    cm.idx.assign(idx, idx + nnz);
    cm.val.assign(val, val + nnz);
    orc::MaskedOp M(&cm, mask);
    size_t xr = (op == 0) ? M.ncols() : nrows;
    orc::DMatrix D(xr, l), out;
    for (size_t i = 0; i < xr; ++i)
        for (size_t c = 0; c < l; ++c) D(i, c) = X[i * l + c];
    if (op == 0 || op == 1) orc::masked_multiply_with_dense(M, D, out, op == 1, compat_d3 != 0);
    else orc::masked_multiply_transposed_by_dense(M, D, out);
    for (size_t i = 0; i < out.r; ++i)
        for (size_t c = 0; c < out.c; ++c) R[i * out.c + c] = out(i, c);
    return 0;
}

struct orc_rand_out {
    uint64_t d, m, n;
    double* u;
    double* s;
    double* vt;
    double t_sparse, t_rows, t_fixed;
};
void orc_rand_free(orc_rand_out* o) {
    std::free(o->u); std::free(o->s); std::free(o->vt);
    std::memset(o, 0, sizeof(*o));
}

int orc_randomized(uint64_t nrows, uint64_t ncols, uint64_t nnz, const uint64_t* ptr, const uint64_t* idx,
                   const double* val, const uint8_t* mask, uint64_t target_rank, uint64_t n_oversamples,
                   uint64_t n_power_iters, int normalizer, const double* omega, int compat_d3, int mean_center,
                   orc_rand_out* out) {
    std::memset(out, 0, sizeof(*out));
    try {
        orc::Compressed cm;
        cm.nmajor = nrows; cm.nminor = ncols;
        cm.ptr.assign(ptr, ptr + nrows + 1);
        cm.idx.assign(idx, idx + nnz);
        cm.val.assign(val, val + nnz);
        std::vector<uint8_t> mk(ncols, 1);
        if (mask) mk.assign(mask, mask + ncols);
        orc::MaskedOp M(&cm, mk.data());
        orc::RandResult r = orc::randomized_svd(M, target_rank, n_oversamples, n_power_iters, normalizer, omega,
                                                compat_d3 != 0, mean_center != 0);
        out->d = r.d; out->m = r.m; out->n = r.n;
        out->u = dup_vec(r.u); out->s = dup_vec(r.s); out->vt = dup_vec(r.vt);
        out->t_sparse = r.t_sparse; out->t_rows = r.t_rows; out->t_fixed = r.t_fixed;
        return 0;
    } catch (std::exception& ex) { g_orc_err = ex.what(); return orc::E_PANIC; }
}

}  // extern "C"
