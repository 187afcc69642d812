// The tridiagonal QL recurrences on the device: imtqlb (SVDLIBC,
// src/legacy.rs:955-1070, and as written, src/lanczos/mod.rs:428-584) and the
// scalar chain of imtql2 (src/lanczos/mod.rs:901-1028, src/legacy.rs:1590-1700)
// in one GPU thread, FP64, every product and sum rounded separately (the
// crate's unfused operation order, as csrc/ql_host.h has it), so the results
// equal the host routines' bit for bit.
//
// The recurrence is one dependent chain of divisions (SVDLIBC's pythag
// iterates s = r / t, u = 1 + 2 s, s / u per step), and one GPU thread runs
// it at FP64 division latency.  svdb_tridiag_device times it on the device;
// the solver keeps the host routines, which finish the same chain several
// times faster (the measured figures are in the design notes).  This entry
// point makes that comparison repeatable and lets the tests check the device
// restatement against the checker.
#include <cmath>

#include "svdb_internal.h"

namespace svdb {

namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ bool cmp(double a, double b, double eps) { return fabs(sub(b, a)) < eps; }
__device__ __forceinline__ double fsign(double a, double b) {
    return ((a >= 0.0 && b >= 0.0) || (a < 0.0 && b < 0.0)) ? a : -a;
}

// pythag as the crate writes it (legacy = false: r = (s/u)^2; true: r *= (s/u)^2)
__device__ double pythag(double a, double b, bool legacy, double eps) {
    const double n = fmax(fabs(a), fabs(b));
    if (!(n > 0.0)) return 0.0;
    double p = n, q = dvd(fmin(fabs(a), fabs(b)), p);
    double r = mul(q, q), t = add(4.0, r);
    // converges in a few steps for finite input; the cap only stops a NaN from spinning
    for (int it = 0; it < 64 && !cmp(t, 4.0, eps); ++it) {
        const double s = dvd(r, t), u = add(1.0, mul(2.0, s));
        p = mul(p, u);
        const double su = dvd(s, u);
        r = legacy ? mul(r, mul(su, su)) : mul(su, su);
        t = add(4.0, r);
    }
    return p;
}

struct RotOut {
    int32_t* i;
    double* c;
    double* s;
    uint64_t cap, n;
};

__device__ void rot_push(RotOut* R, int32_t i, double c, double s) {
    if (!R) return;
    if (R->n < R->cap) {
        R->i[R->n] = i;
        R->c[R->n] = c;
        R->s[R->n] = s;
    }
    ++R->n;
}

// imtqlb (SVDLIBC): status 0, or SVDB_ERR_IMTQLB after 30 iterations on one value
__device__ int imtqlb_legacy_dev(int64_t n, double* d, double* e, double* bnd, RotOut* R, double eps) {
    if (n == 1) return 0;
    bnd[0] = 1.0;
    const int64_t last = n - 1;
    for (int64_t i = 1; i <= last; ++i) { bnd[i] = 0.0; e[i - 1] = e[i]; }
    e[last] = 0.0;
    int64_t i = 0;
    for (int64_t l = 0; l <= last; ++l) {
        int64_t iteration = 0;
        while (iteration <= 30) {
            int64_t m = l;
            while (m < n) {
                if (m == last) break;
                const double test = add(fabs(d[m]), fabs(d[m + 1]));
                if (cmp(test, add(test, fabs(e[m])), eps)) break;
                ++m;
            }
            double p = d[l], f = bnd[l];
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
                if (iteration == 30) return SVDB_ERR_IMTQLB;
                ++iteration;
                double g = dvd(sub(d[l + 1], p), mul(2.0, e[l]));
                double r = pythag(g, 1.0, true, eps);
                g = add(sub(d[m], p), dvd(e[l], add(g, fsign(r, g))));
                double s = 1.0, c = 1.0;
                p = 0.0;
                i = m - 1;
                bool underflow = false;
                while (!underflow && i >= l) {
                    f = mul(s, e[i]);
                    const double b = mul(c, e[i]);
                    r = pythag(f, g, true, eps);
                    e[i + 1] = r;
                    if (cmp(r, 0.0, eps)) { underflow = true; break; }
                    s = dvd(f, r);
                    c = dvd(g, r);
                    g = sub(d[i + 1], p);
                    r = add(mul(sub(d[i], g), s), mul(mul(2.0, c), b));
                    p = mul(s, r);
                    d[i + 1] = add(g, p);
                    g = sub(mul(c, r), b);
                    f = bnd[i + 1];
                    bnd[i + 1] = add(mul(s, bnd[i]), mul(c, f));
                    bnd[i] = sub(mul(c, bnd[i]), mul(s, f));
                    rot_push(R, (int32_t)i, c, s);
                    if (i == 0) break;
                    --i;
                }
                if (underflow) d[i + 1] = sub(d[i + 1], p);
                else { d[l] = sub(d[l], p); e[l] = g; }
                e[m] = 0.0;
            }
        }
    }
    return 0;
}

// imtqlb as written (mod.rs:428-584): tolerance 100 eps max(test, 1) sqrt(n),
// the 1000 eps underflow test, and a soft failure (warned) at max_it
__device__ int imtqlb_current_dev(int64_t n, double* d, double* e, double* bnd, uint64_t max_it, int* warned,
                                  double eps) {
    if (n == 1) return 0;
    const double msf = sqrt((double)n);
    bnd[0] = 1.0;
    const int64_t last = n - 1;
    for (int64_t i = 1; i <= last; ++i) { bnd[i] = 0.0; e[i - 1] = e[i]; }
    e[last] = 0.0;
    int64_t i = 0;
    for (int64_t l = 0; l <= last; ++l) {
        uint64_t iteration = 0;
        double p = d[l], f = bnd[l];
        while (iteration <= max_it) {
            int64_t m = l;
            while (m < n) {
                if (m == last) break;
                const double test = add(fabs(d[m]), fabs(d[m + 1]));
                const double tol = mul(mul(mul(eps, 100.0), fmax(test, 1.0)), msf);
                if (fabs(e[m]) <= tol) break;
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
                iteration = max_it + 1;
            } else {
                if (iteration == max_it) {
                    *warned = 1;
                    for (int64_t idx = l; idx <= m; ++idx) bnd[idx] = fmax(bnd[idx], 0.1);
                    e[l] = 0.0;
                    break;
                }
                ++iteration;
                double g = dvd(sub(d[l + 1], p), mul(2.0, e[l]));
                double r = pythag(g, 1.0, false, eps);
                g = add(sub(d[m], p), dvd(e[l], add(g, fsign(r, g))));
                double s = 1.0, c = 1.0;
                p = 0.0;
                i = m - 1;
                bool underflow = false;
                while (!underflow && i >= l) {
                    f = mul(s, e[i]);
                    const double b = mul(c, e[i]);
                    r = pythag(f, g, false, eps);
                    e[i + 1] = r;
                    if (r < mul(mul(eps, 1000.0), add(fabs(f), fabs(g)))) { underflow = true; break; }
                    if (fabs(r) < mul(eps, 100.0)) r = mul(mul(eps, 100.0), fsign(1.0, r));
                    s = dvd(f, r);
                    c = dvd(g, r);
                    g = sub(d[i + 1], p);
                    r = add(mul(sub(d[i], g), s), mul(mul(2.0, c), b));
                    p = mul(s, r);
                    d[i + 1] = add(g, p);
                    g = sub(mul(c, r), b);
                    f = bnd[i + 1];
                    bnd[i + 1] = add(mul(s, bnd[i]), mul(c, f));
                    bnd[i] = sub(mul(c, bnd[i]), mul(s, f));
                    if (i == 0) break;
                    --i;
                }
                if (underflow) d[i + 1] = sub(d[i + 1], p);
                else { d[l] = sub(d[l], p); e[l] = g; }
                e[m] = 0.0;
            }
        }
    }
    return 0;
}

// imtql2's scalar chain, recording the rotations and the final column order
__device__ int imtql2_dev(int64_t n, double* d, double* e, bool legacy, uint64_t max_it, RotOut* R, int32_t* perm,
                          double eps) {
    for (int64_t k = 0; k < n; ++k) perm[k] = (int32_t)k;
    if (n == 1) return 0;
    const int64_t last = n - 1;
    for (int64_t i = 1; i < n; ++i) e[i - 1] = e[i];
    e[last] = 0.0;
    for (int64_t l = 0; l < n; ++l) {
        uint64_t iteration = 0;
        while (iteration <= max_it) {
            int64_t m = l;
            while (m < n) {
                if (m == last) break;
                const double test = add(fabs(d[m]), fabs(d[m + 1]));
                if (cmp(test, add(test, fabs(e[m])), eps)) break;
                ++m;
            }
            if (m == l) break;
            if (iteration == max_it) return SVDB_ERR_IMTQL2;
            ++iteration;
            double g = dvd(sub(d[l + 1], d[l]), mul(2.0, e[l]));
            double r = pythag(g, 1.0, legacy, eps);
            g = add(sub(d[m], d[l]), dvd(e[l], add(g, fsign(r, g))));
            double s = 1.0, c = 1.0, p = 0.0;
            int64_t i = m - 1;
            bool underflow = false;
            while (!underflow && i >= l) {
                const double f = mul(s, e[i]);
                const double b = mul(c, e[i]);
                r = pythag(f, g, legacy, eps);
                e[i + 1] = r;
                if (cmp(r, 0.0, eps)) underflow = true;
                else {
                    s = dvd(f, r);
                    c = dvd(g, r);
                    g = sub(d[i + 1], p);
                    r = add(mul(sub(d[i], g), s), mul(mul(2.0, c), b));
                    p = mul(s, r);
                    d[i + 1] = add(g, p);
                    g = sub(mul(c, r), b);
                    rot_push(R, (int32_t)i, c, s);
                    if (i == 0) break;
                    --i;
                }
            }
            if (underflow) d[i + 1] = sub(d[i + 1], p);
            else { d[l] = sub(d[l], p); e[l] = g; }
            e[m] = 0.0;
        }
    }
    // the closing selection sort, as a column permutation
    for (int64_t l = 1; l < n; ++l) {
        const int64_t i = l - 1;
        int64_t k = i;
        double p = d[i];
        for (int64_t j = l; j < n; ++j)
            if (d[j] < p) { k = j; p = d[j]; }
        if (k != i) {
            d[k] = d[i];
            d[i] = p;
            const int32_t t = perm[i];
            perm[i] = perm[k];
            perm[k] = t;
        }
    }
    return 0;
}

}  // namespace

__global__ void k_tridiag(int routine, int64_t n, double* d, double* e, double* bnd, int32_t* ri, double* rc,
                          double* rs, uint64_t rcap, uint64_t* nrot, int32_t* perm, uint64_t max_it, double eps,
                          int* status) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    RotOut R{ri, rc, rs, rcap, 0};
    int st = 0, warned = 0;
    switch (routine) {
        case 0: st = imtqlb_legacy_dev(n, d, e, bnd, ri ? &R : nullptr, eps); break;
        case 1: st = imtqlb_current_dev(n, d, e, bnd, max_it, &warned, eps); break;
        case 2: st = imtql2_dev(n, d, e, true, max_it, &R, perm, eps); break;
        default: st = imtql2_dev(n, d, e, false, max_it, &R, perm, eps); break;
    }
    *nrot = R.n;
    status[0] = st;
    status[1] = warned;
}

}  // namespace svdb

extern "C" int svdb_tridiag_device(int routine, uint64_t n, double* d, double* e, double* bnd, int32_t* rot_i,
                                   double* rot_c, double* rot_s, uint64_t rot_cap, uint64_t* n_rot, int32_t* perm,
                                   uint64_t max_it, int* warned, double* device_ms) {
    using namespace svdb;
    try {
        if (routine < 0 || routine > 3) throw Error(SVDB_ERR_ARG, "svdb_tridiag_device: routine 0..3");
        if (n == 0 || !d || !e || ((routine <= 1) && !bnd) || (routine >= 2 && !perm) || !n_rot)
            throw Error(SVDB_ERR_ARG, "svdb_tridiag_device: null argument");
        if (rot_cap && (!rot_i || !rot_c || !rot_s)) throw Error(SVDB_ERR_ARG, "svdb_tridiag_device: null record");
        if (n > (uint64_t)INT32_MAX) throw Error(SVDB_ERR_UNSUPPORTED, "svdb_tridiag_device: order above 2^31-1");
        if (max_it > 100000) throw Error(SVDB_ERR_ARG, "svdb_tridiag_device: max_it above 100000");
        cudaStream_t s = nullptr;
        SVDB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        int st[2] = {0, 0};
        uint64_t nr = 0;
        float ms = 0.f;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        try {
            DevBuf<double> dd(n, s), de(n, s), db(n, s), dc(std::max<uint64_t>(rot_cap, 1), s),
                dsn(std::max<uint64_t>(rot_cap, 1), s);
            DevBuf<int32_t> di(std::max<uint64_t>(rot_cap, 1), s), dp(n, s);
            DevBuf<uint64_t> dn(1, s);
            DevBuf<int> dst(2, s);
            SVDB_CUDA(cudaMemcpyAsync(dd.p, d, n * 8, cudaMemcpyHostToDevice, s));
            SVDB_CUDA(cudaMemcpyAsync(de.p, e, n * 8, cudaMemcpyHostToDevice, s));
            // bnd is in and out, as the reference's array: order 1 leaves it as given
            if (routine <= 1) SVDB_CUDA(cudaMemcpyAsync(db.p, bnd, n * 8, cudaMemcpyHostToDevice, s));
            SVDB_CUDA(cudaEventCreate(&e0));
            SVDB_CUDA(cudaEventCreate(&e1));
            SVDB_CUDA(cudaEventRecord(e0, s));
            k_tridiag<<<1, 32, 0, s>>>(routine, (int64_t)n, dd.p, de.p, db.p, rot_cap ? di.p : nullptr, dc.p, dsn.p,
                                       rot_cap, dn.p, dp.p, max_it, 2.220446049250313e-16, dst.p);
            SVDB_CHECK_LAUNCH();
            SVDB_CUDA(cudaEventRecord(e1, s));
            SVDB_CUDA(cudaMemcpyAsync(d, dd.p, n * 8, cudaMemcpyDeviceToHost, s));
            SVDB_CUDA(cudaMemcpyAsync(e, de.p, n * 8, cudaMemcpyDeviceToHost, s));
            if (routine <= 1) SVDB_CUDA(cudaMemcpyAsync(bnd, db.p, n * 8, cudaMemcpyDeviceToHost, s));
            else SVDB_CUDA(cudaMemcpyAsync(perm, dp.p, n * 4, cudaMemcpyDeviceToHost, s));
            SVDB_CUDA(cudaMemcpyAsync(&nr, dn.p, 8, cudaMemcpyDeviceToHost, s));
            SVDB_CUDA(cudaMemcpyAsync(st, dst.p, 8, cudaMemcpyDeviceToHost, s));
            SVDB_CUDA(cudaStreamSynchronize(s));
            const uint64_t keep = std::min<uint64_t>(nr, rot_cap);
            if (keep) {
                SVDB_CUDA(cudaMemcpyAsync(rot_i, di.p, keep * 4, cudaMemcpyDeviceToHost, s));
                SVDB_CUDA(cudaMemcpyAsync(rot_c, dc.p, keep * 8, cudaMemcpyDeviceToHost, s));
                SVDB_CUDA(cudaMemcpyAsync(rot_s, dsn.p, keep * 8, cudaMemcpyDeviceToHost, s));
            }
            SVDB_CUDA(cudaStreamSynchronize(s));
            cudaEventElapsedTime(&ms, e0, e1);
        } catch (...) {
            cudaStreamSynchronize(s);
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            cudaStreamDestroy(s);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        SVDB_CUDA(cudaStreamDestroy(s));
        *n_rot = nr;
        if (warned) *warned = st[1];
        if (device_ms) *device_ms = ms;
        if (st[0] == SVDB_ERR_IMTQLB) throw Error(SVDB_ERR_IMTQLB, "svdlibrs/imtqlb: imtqlb no convergence to an eigenvalue after 30 iterations");
        if (st[0] == SVDB_ERR_IMTQL2) throw Error(SVDB_ERR_IMTQL2, "svdlibrs/imtql2: imtql2 no convergence to an eigenvalue");
        return SVDB_OK;
    } catch (Error& x) {
        set_last_error(x.what());
        return x.code;
    }
}
