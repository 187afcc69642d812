// Device bodies of the small dense steps of randomized_svd, shared by the
// single-problem kernels (randomized.cu) and the batched kernels (batch.cu):
// the Omega generator, the one-block Cholesky with R^-1, and the one-block
// one-sided Jacobi SVD.
#pragma once

#include <cstdint>

#include "device_common.cuh"

namespace svdb {

// --------------------------------------------------------------- Omega ----
// N(0,1) entries from a counter-based generator: splitmix64 (Steele, Lea and
// Flood 2014) of (seed, index) gives two uniforms, Box-Muller gives the
// normal.  rand_distr's ziggurat stream is not reproduced.
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
__device__ __forceinline__ uint64_t omega_key(uint64_t seed) { return splitmix64(seed ^ 0x5DEECE66Dull); }
// entry i of the row-major Omega stream of `key`
__device__ __forceinline__ double omega_value(uint64_t key, int64_t i) {
    const uint64_t a = splitmix64(key + 2 * (uint64_t)i), b = splitmix64(key + 2 * (uint64_t)i + 1);
    const double u1 = ((double)(a >> 11) + 0.5) * (1.0 / 9007199254740992.0);  // (0,1)
    const double u2 = (double)(b >> 11) * (1.0 / 9007199254740992.0);          // [0,1)
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

// One block: G = R^T R (upper R) in shared memory, then R^-1.  A non-positive
// pivot restarts the factorisation on G + shift I with shift =
// shift_scale * trace(G) (shifted CholeskyQR); that sets bit 1 of *flags and
// *shifted (which enables the third pass).  A second breakdown sets bit 2 and
// leaves R = R^-1 = I.  R and R^-1 are written to global memory.
// The factorisation runs on the first 128 threads with one named barrier per
// step: step k updates a_ij -= a_ki a_kj / a_kk with the unscaled pivot row,
// and every row is scaled by 1/sqrt(a_kk) at the end.
// sm: c*c doubles of shared memory (2*c*c when ri_in_smem); c <= 128; at
// least 128 threads.
__device__ __forceinline__ void chol_inv_body(const double* __restrict__ G, int c, double shift_scale,
                                              double* __restrict__ R, double* __restrict__ Ri,
                                              int* __restrict__ flags, int* __restrict__ shifted, int ri_in_smem,
                                              double* sm) {
    __shared__ int s_fail;
    __shared__ double s_shift;
    __shared__ double s_rd[128];  // 1 / sqrt(a_kk)
    const int cc = c * c;
    double* ri = ri_in_smem ? sm + cc : Ri;
    if (blockDim.x < 128 || c > 128) {  // the named barrier needs 128 threads; s_rd holds 128 pivots
        if (threadIdx.x == 0) atomicOr(flags, 2);
        for (int t = threadIdx.x; t < cc; t += blockDim.x) R[t] = Ri[t] = (t / c == t % c) ? 1.0 : 0.0;
        return;
    }
    for (int attempt = 0; attempt < 2; ++attempt) {
        for (int t = threadIdx.x; t < cc; t += blockDim.x)
            sm[t] = G[t] + ((attempt == 1 && t / c == t % c) ? s_shift : 0.0);
        if (threadIdx.x == 0) s_fail = 0;
        __syncthreads();
        if (threadIdx.x < 128) {
            for (int k = 0; k < c; ++k) {
                const double d = sm[k * c + k];
                if (!(d > 0.0 && isfinite(d))) {  // the same value for all 128 threads
                    if (threadIdx.x == 0) s_fail = 1;
                    break;
                }
                const double inv = 1.0 / d;
                // upper triangle i <= j of the trailing block: 8 rows x 16 columns of
                // threads, no index division
                const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
                for (int i = k + 1 + ty; i < c; i += 8) {
                    const double aki = sm[k * c + i];
                    for (int j = i + tx; j < c; j += 16) sm[i * c + j] -= aki * sm[k * c + j] * inv;
                }
                asm volatile("bar.sync 1, 128;" ::: "memory");
            }
        }
        __syncthreads();
        if (!s_fail) break;
        if (attempt == 0) {
            if (threadIdx.x == 0) {
                double tr = 0.0;
                for (int i = 0; i < c; ++i) tr += G[i * c + i];
                s_shift = shift_scale * tr > 0.0 ? shift_scale * tr : 1e-300;
                atomicOr(flags, 1);
                *shifted = 1;
            }
            __syncthreads();
        }
    }
    if (s_fail) {
        if (threadIdx.x == 0) atomicOr(flags, 2);
        for (int t = threadIdx.x; t < cc; t += blockDim.x) {
            const double v = (t / c == t % c) ? 1.0 : 0.0;
            R[t] = v;
            Ri[t] = v;
        }
        return;
    }
    for (int k = threadIdx.x; k < c; k += blockDim.x) s_rd[k] = 1.0 / sqrt(sm[k * c + k]);
    __syncthreads();
    for (int t = threadIdx.x; t < cc; t += blockDim.x) {
        const int i = t / c, j = t % c;
        double v = 0.0;
        if (i == j) v = sqrt(sm[t]);
        else if (i < j) v = sm[t] * s_rd[i];
        ri[t] = v;  // staged: sm still holds the pivots other threads read
    }
    __syncthreads();
    for (int t = threadIdx.x; t < cc; t += blockDim.x) {
        sm[t] = ri[t];
        R[t] = ri[t];
        ri[t] = 0.0;
    }
    __syncthreads();
    // R^-1 row i, one warp per row: x^T R = e_i^T by forward substitution in
    // axpy form.  Lane l holds x_l, x_{l+32}, x_{l+64}, x_{l+96}; step k scales
    // x_k by 1 / R_kk and subtracts x_k R[k, k+1..] from the later entries,
    // reading row k of R (contiguous, no bank conflicts).  No reductions: the
    // dependent path of a step is one shuffle, one multiply and one FMA.
    for (int k = threadIdx.x; k < c; k += blockDim.x) s_rd[k] = 1.0 / sm[k * c + k];
    __syncthreads();
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
        for (int i = warp; i < c; i += nwarps) {
            double x[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) x[q] = (lane + 32 * q == i) ? 1.0 : 0.0;
            for (int k = i; k < c; ++k) {
                const int ks = k >> 5, kl = k & 31;
                double own = x[0];
#pragma unroll
                for (int q = 1; q < 4; ++q)
                    if (ks == q) own = x[q];
                const double xk = __shfl_sync(0xffffffffu, own, kl) * s_rd[k];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int e = lane + 32 * q;
                    if (e == k) x[q] = xk;
                    else if (e > k && e < c) x[q] = fma(-xk, sm[k * c + e], x[q]);
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int e = lane + 32 * q;
                if (e < c) ri[i * c + e] = e >= i ? x[q] : 0.0;
            }
        }
    }
    if (ri_in_smem) {
        __syncthreads();
        for (int t = threadIdx.x; t < cc; t += blockDim.x) Ri[t] = ri[t];
    }
}

// Lanes per column pair in jacobi_svd_body (about eight elements of a column
// per lane), and the block size that gives every pair of the padded columns
// its lanes, capped at `cap` threads.
__host__ __device__ inline int jacobi_group(int c) { return c <= 64 ? 8 : (c <= 128 ? 16 : 32); }
__host__ __device__ inline int jacobi_threads(int c, int cap) {
    const int cp = c + (c & 1);
    const int t = ((cp / 2) * jacobi_group(c) + 31) / 32 * 32;
    return t < 32 ? 32 : (t > cap ? cap : t);
}

// One-sided Jacobi SVD of R (c x c, row-major) in one block: W = R V with
// orthogonal columns, sigma_j = |W_j|, U_j = W_j / sigma_j.  Round-robin pair
// ordering, jacobi_group(c) lanes per pair.  Outputs sorted by descending sigma:
// U (c x c), V (c x c), sig (c).  *status = sweeps << 8, | 2 if the sweep limit is reached.
// sm: (c * cp + cp * cp + cp) doubles, cp = c rounded up to even.  Any
// block size that is a multiple of 32.
__device__ __forceinline__ void jacobi_svd_body(const double* __restrict__ R, int c, double* __restrict__ U,
                                                double* __restrict__ V, double* __restrict__ sig,
                                                int* __restrict__ status, double* sm) {
    // W (c x cp) | Vs (c x cp) | norms (cp) ; column-major
    const int cp = c + (c & 1);     // even number of columns (zero padding column)
    double* W = sm;
    double* Vs = sm + (size_t)c * cp;
    double* nr = Vs + (size_t)cp * cp;
    __shared__ int s_rot;
    for (int t = threadIdx.x; t < c * cp; t += blockDim.x) {
        const int i = t % c, j = t / c;
        W[j * c + i] = (j < c) ? R[i * c + j] : 0.0;
    }
    for (int t = threadIdx.x; t < cp * cp; t += blockDim.x) Vs[t] = ((t % cp) == (t / cp)) ? 1.0 : 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int half = cp / 2;
    // G lanes per column pair, 32 / G pairs per warp: the pair's scalar work
    // (three sums, the rotation's sqrt, division and rsqrt) is issued once
    // per warp for 32 / G pairs.  Pairs are walked warp by warp so that the
    // shuffles see the whole warp.
    const int G = jacobi_group(c), gpw = 32 / G, sub = lane & (G - 1), gw = lane / G;
    const double tol = 2.220446049250313e-16 * (double)(c > 4 ? c : 4);
    int sweep = 0;
    for (; sweep < 60; ++sweep) {
        if (threadIdx.x == 0) s_rot = 0;
        __syncthreads();
        for (int round = 0; round < cp - 1; ++round) {
            for (int base = warp * gpw; base < half; base += nwarps * gpw) {
                const int pr = base + gw;
                const bool valid = pr < half;
                // round-robin: position 0 fixed, others rotate
                auto at = [&](int pos) { return pos == 0 ? 0 : 1 + (pos - 1 + round) % (cp - 1); };
                int p = 0, q = 0;
                if (valid) {
                    p = at(pr);
                    q = at(cp - 1 - pr);
                    if (p > q) { int t = p; p = q; q = t; }
                }
                double al = 0, be = 0, ga = 0;
                if (valid)
                    for (int i = sub; i < c; i += G) {
                        const double x = W[p * c + i], y = W[q * c + i];
                        al = fma(x, x, al);
                        be = fma(y, y, be);
                        ga = fma(x, y, ga);
                    }
                for (int o = G >> 1; o > 0; o >>= 1) {
                    al += __shfl_xor_sync(0xffffffffu, al, o);
                    be += __shfl_xor_sync(0xffffffffu, be, o);
                    ga += __shfl_xor_sync(0xffffffffu, ga, o);
                }
                // |ga| > tol sqrt(al be), compared in squares.  The rotation of the
                // usual zeta = (be - al) / (2 ga), t = sign(zeta) / (|zeta| +
                // sqrt(1 + zeta^2)), cs = 1 / sqrt(1 + t^2), with numerator and
                // denominator of t scaled by |2 ga|: one sqrt, one division, one
                // reciprocal square root on the dependent path.
                if (valid && ga != 0.0 && ga * ga > (tol * tol) * (al * be)) {
                    const double d = be - al, g2 = 2.0 * ga;
                    const bool pos = (d >= 0.0) == (ga > 0.0) || d == 0.0;  // sign(zeta) >= 0
                    const double t = (pos ? fabs(g2) : -fabs(g2)) / (fabs(d) + sqrt(fma(d, d, g2 * g2)));
                    const double cs = rsqrt(fma(t, t, 1.0)), sn = cs * t;
                    for (int i = sub; i < c; i += G) {
                        const double x = W[p * c + i], y = W[q * c + i];
                        W[p * c + i] = cs * x - sn * y;
                        W[q * c + i] = sn * x + cs * y;
                    }
                    for (int i = sub; i < cp; i += G) {
                        const double x = Vs[p * cp + i], y = Vs[q * cp + i];
                        Vs[p * cp + i] = cs * x - sn * y;
                        Vs[q * cp + i] = sn * x + cs * y;
                    }
                    if (sub == 0) s_rot = 1;
                }
            }
            __syncthreads();
        }
        if (!s_rot) break;
        __syncthreads();
    }
    if (threadIdx.x == 0) *status = (sweep << 8) | (sweep == 60 ? 2 : 0);  // sweeps, limit flag
    for (int j = warp; j < cp; j += nwarps) {
        double s = 0.0;
        for (int i = lane; i < c; i += 32) s = fma(W[j * c + i], W[j * c + i], s);
        s = warp_sum(s);
        if (lane == 0) nr[j] = sqrt(s);
    }
    __syncthreads();
    // rank of each column by descending norm (ties by index) -> output position
    for (int j = threadIdx.x; j < c; j += blockDim.x) {
        int pos = 0;
        for (int k = 0; k < c; ++k)
            if (nr[k] > nr[j] || (nr[k] == nr[j] && k < j)) ++pos;
        sig[pos] = nr[j];
        for (int i = 0; i < c; ++i) {
            U[i * c + pos] = nr[j] > 0.0 ? W[j * c + i] / nr[j] : (i == pos ? 1.0 : 0.0);
            V[i * c + pos] = Vs[j * cp + i];
        }
    }
}

}  // namespace svdb
