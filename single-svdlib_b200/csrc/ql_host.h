// The scalar recurrences of the tridiagonal QL iterations (SVDLIBC's imtqlb
// and imtql2 as src/legacy.rs and src/lanczos/mod.rs restate them), kept free
// of device code so that the host library and the CPU tests compile the same
// lines.  Every routine reproduces the crate's exact floating-point
// operation sequence.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <limits>
#include <vector>

#include "svdb_internal.h"

namespace svdb {

// SvdFloat::eps of the run's scalar T (src/utils.rs:87-113): f64::EPSILON,
// or f32::EPSILON while a T = f32 run holds a ScalarEps on this thread.  The
// tolerances, pythag's and compare's thresholds all follow it; the arithmetic
// stays FP64.
static thread_local double EPS = std::numeric_limits<double>::epsilon();
struct ScalarEps {
    double saved;
    explicit ScalarEps(bool f32) : saved(EPS) {
        EPS = f32 ? (double)std::numeric_limits<float>::epsilon() : std::numeric_limits<double>::epsilon();
    }
    ~ScalarEps() { EPS = saved; }
};
static inline double eps34() { return std::pow(EPS, 0.75); }
static inline bool compare(double a, double b) { return std::fabs(b - a) < EPS; }  // src/utils.rs:110-112

// ------------------------------------------------------ scalar helpers ----
// svd_pythag as written in the current crate (mod.rs:361-380): r = (s/u)^2.
static inline double pythag_current(double a, double b) {
    double n = std::fmax(std::fabs(a), std::fabs(b));
    if (!(n > 0.0)) return 0.0;
    double p = n, q = std::fmin(std::fabs(a), std::fabs(b)) / p;
    double r = q * q, t = 4.0 + r;
    while (!compare(t, 4.0)) {
        double s = r / t, u = 1.0 + 2.0 * s;
        p = p * u;
        double su = s / u;
        r = su * su;
        t = 4.0 + r;
    }
    return p;
}
// Moler-Morrison as in SVDLIBC / legacy.rs:878-895: r *= (s/u)^2.
static inline double pythag_legacy(double a, double b) {
    double n = std::fmax(std::fabs(a), std::fabs(b));
    if (!(n > 0.0)) return 0.0;
    double p = n, q = std::fmin(std::fabs(a), std::fabs(b)) / p;
    double r = q * q, t = 4.0 + r;
    while (!compare(t, 4.0)) {
        double s = r / t, u = 1.0 + 2.0 * s;
        p *= u;
        double su = s / u;
        r *= su * su;
        t = 4.0 + r;
    }
    return p;
}
static inline double fsign(double a, double b) { return ((a >= 0.0 && b >= 0.0) || (a < 0.0 && b < 0.0)) ? a : -a; }

// The scalar chain of imtql2 (mod.rs:901-1028 / legacy.rs:1590-1700) without
// z: every applied rotation is recorded, and the final selection sort of the
// eigenvalues becomes a column permutation.
struct Rotations {
    std::vector<int32_t> i;
    std::vector<double> c, s;
    std::vector<int32_t> perm;
    std::vector<double> d;  // eigenvalue l as it converged (before the final sort)
};

// imtqlb of SVDLIBC (legacy.rs:955-1070).  With rec, the plane rotations
// (i, c, s) of every sweep are recorded in order and rec->d[l] is eigenvalue
// l as it converged.  The shifts, sweeps and convergence tests are imtql2's
// (legacy.rs:1590-1700) on the same (d, e): imtqlb adds only the bnd row and
// an insertion sort of the converged entries below l, which no later sweep
// reads.  So for the T that ritvec passes to imtql2 the record is imtql2's.
// With flush, flush(k) is called each time the record reaches k rotations, k
// a multiple of every: rotations before k are final.
static inline void imtqlb_legacy(size_t n, double* d, double* e, double* bnd, Rotations* rec = nullptr,
                                 const std::function<void(size_t)>* flush = nullptr, size_t every = 0) {
    if (rec) {
        rec->i.clear();
        rec->c.clear();
        rec->s.clear();
        rec->d.assign(n, 0.0);
        if (n == 1) rec->d[0] = d[0];
    }
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
                double test = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (compare(test, test + std::fabs(e[m]))) break;
                ++m;
            }
            double p = d[l], f = bnd[l];
            if (m == l) {
                if (rec) rec->d[l] = p;
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
                    throw Error(SVDB_ERR_IMTQLB,
                                "svdlibrs/imtqlb: imtqlb no convergence to an eigenvalue after 30 iterations");
                ++iteration;
                double g = (d[l + 1] - p) / (2.0 * e[l]);
                double r = pythag_legacy(g, 1.0);
                g = d[m] - p + e[l] / (g + fsign(r, g));
                double s = 1.0, c = 1.0;
                p = 0.0;
                i = m - 1;
                bool underflow = false;
                while (!underflow && i >= l) {
                    f = s * e[i];
                    double b = c * e[i];
                    r = pythag_legacy(f, g);
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
                    if (rec) {
                        rec->i.push_back((int32_t)i);
                        rec->c.push_back(c);
                        rec->s.push_back(s);
                        if (flush && every && rec->i.size() % every == 0) (*flush)(rec->i.size());
                    }
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

// imtql2's closing selection sort of the eigenvalues (legacy.rs:1669-1689,
// mod.rs:1005-1025), as a permutation of Z's columns: perm must start as the
// identity.
static inline void ql_sort_perm(size_t n, double* d, std::vector<int32_t>& perm) {
    for (size_t l = 1; l < n; ++l) {
        size_t i = l - 1, k = i;
        double p = d[i];
        for (size_t j = l; j < n; ++j)
            if (d[j] < p) { k = j; p = d[j]; }
        if (k != i) {
            d[k] = d[i];
            d[i] = p;
            std::swap(perm[i], perm[k]);
        }
    }
}


static inline void imtql2_scalar(size_t n, double* d, double* e, bool legacy, size_t max_it, Rotations& R) {
    R.perm.resize(n);
    for (size_t k = 0; k < n; ++k) R.perm[k] = (int32_t)k;
    if (n == 1) return;
    size_t last = n - 1;
    for (size_t i = 1; i < n; ++i) e[i - 1] = e[i];
    e[last] = 0.0;
    for (size_t l = 0; l < n; ++l) {
        size_t iteration = 0;
        while (iteration <= max_it) {
            size_t m = l;
            while (m < n) {
                if (m == last) break;
                double test = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (compare(test, test + std::fabs(e[m]))) break;
                ++m;
            }
            if (m == l) break;
            if (iteration == max_it) {
                char buf[160];
                snprintf(buf, sizeof buf,
                         "svdlibrs/imtql2: imtql2 no convergence to an eigenvalue after %zu iterations", max_it);
                throw Error(SVDB_ERR_IMTQL2, buf);
            }
            ++iteration;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = legacy ? pythag_legacy(g, 1.0) : pythag_current(g, 1.0);
            g = d[m] - d[l] + e[l] / (g + fsign(r, g));
            double s = 1.0, c = 1.0, p = 0.0;
            size_t i = m - 1;
            bool underflow = false;
            while (!underflow && i >= l) {
                double f = s * e[i];
                double b = c * e[i];
                r = legacy ? pythag_legacy(f, g) : pythag_current(f, g);
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
                    R.i.push_back((int32_t)i);
                    R.c.push_back(c);
                    R.s.push_back(s);
                    if (i == 0) break;
                    --i;
                }
            }
            if (underflow) d[i + 1] -= p;
            else { d[l] -= p; e[l] = g; }
            e[m] = 0.0;
        }
    }
    ql_sort_perm(n, d, R.perm);
}

}  // namespace svdb
