// Checks the packed rotation lists that the device rotation kernel relies on
// (single-svdlib_b200/csrc/rot_pack.h), on random lists shaped like QL sweeps:
//  - segments tile the list, each a run whose index falls by one, none
//    crossing a kRotChunk boundary, padding zeroed, (c, s, index) in place;
//  - applying a row segment by segment, with the lo of each rotation carried
//    in a register and stored once at the segment's end (the kernel's
//    schedule), is bit for bit the sequential loop;
//  - packing and applying the list in pieces gives the same Z;
//  - an index outside [0, js - 2] is refused.
// Prints "ok <lists> <rotations>" or the first failure.  Built and run by
// test_rot_pack.py.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "rot_pack.h"

using namespace svdb;

static double mul(double a, double b) { volatile double r = a * b; return r; }
static double add(double a, double b) { volatile double r = a + b; return r; }
static double sub(double a, double b) { volatile double r = a - b; return r; }

// the sequential loop of imtql2's vector accumulation, on one row z
static void apply_plain(std::vector<double>& z, const std::vector<int32_t>& ri, const std::vector<double>& rc,
                        const std::vector<double>& rs, size_t from, size_t to) {
    for (size_t t = from; t < to; ++t) {
        const int i = ri[t];
        const double f = z[i + 1], a = z[i];
        z[i + 1] = add(mul(rs[t], a), mul(rc[t], f));
        z[i] = sub(mul(rc[t], a), mul(rs[t], f));
    }
}

// the segment schedule on packed lists
static bool apply_packed(std::vector<double>& z, const std::vector<double>& cs, const std::vector<int32_t>& il,
                         int64_t nrot) {
    for (int64_t u = 0; u < nrot;) {
        const int len = il[2 * u + 1], top = il[2 * u];
        if (len < 1 || u + len > nrot) return false;
        double f = z[top + 1];
        for (int q = 0; q < len; ++q) {
            const double c = cs[2 * (u + q)], s = cs[2 * (u + q) + 1], a = z[top - q];
            const double hi = add(mul(s, a), mul(c, f));
            f = sub(mul(c, a), mul(s, f));
            z[top - q + 1] = hi;
        }
        z[top - len + 1] = f;
        u += len;
    }
    return true;
}

int main() {
    std::mt19937_64 g(17);
    int64_t lists = 0, total = 0;
    for (int trial = 0; trial < 200; ++trial) {
        const int js = 2 + (int)(g() % 90);
        const int64_t nrot = trial < 3 ? trial : (int64_t)(g() % 6000);
        std::vector<int32_t> ri((size_t)nrot);
        std::vector<double> rc((size_t)nrot), rs((size_t)nrot);
        int cur = (int)(g() % (js - 1));
        for (int64_t t = 0; t < nrot; ++t) {  // mostly falling runs, as sweeps make them
            const int m = (int)(g() % 10);
            if (m < 7 && cur > 0) --cur;
            else if (m == 8 && cur + 1 < js - 1) ++cur;
            else if (m == 9) cur = (int)(g() % (js - 1));
            ri[(size_t)t] = cur;
            const double th = (double)(g() % 100000) * 1e-4;
            rc[(size_t)t] = std::cos(th);
            rs[(size_t)t] = std::sin(th);
        }
        std::vector<double> cs;
        std::vector<int32_t> il;
        rot_pack(ri.data(), rc.data(), rs.data(), nrot, js, cs, il);
        if ((int64_t)cs.size() != 2 * rot_padded(nrot) || (int64_t)il.size() != 2 * rot_padded(nrot)) {
            std::printf("trial %d: list sizes\n", trial);
            return 1;
        }
        for (int64_t u = 0; u < nrot;) {
            const int len = il[2 * u + 1];
            if (len < 1 || u + len > nrot || u / kRotChunk != (u + len - 1) / kRotChunk) {
                std::printf("trial %d: bad segment at %lld (len %d)\n", trial, (long long)u, len);
                return 1;
            }
            for (int q = 0; q < len; ++q) {
                const int64_t t = u + q;
                if (il[2 * t] != ri[t] || cs[2 * t] != rc[t] || cs[2 * t + 1] != rs[t] || (q && il[2 * t + 1]) ||
                    (q && ri[t] != ri[u] - q)) {
                    std::printf("trial %d: segment contents at %lld\n", trial, (long long)t);
                    return 1;
                }
            }
            // a segment is maximal inside its chunk
            const int64_t e = u + len;
            if (e < nrot && e % kRotChunk != 0 && ri[e] == ri[e - 1] - 1) {
                std::printf("trial %d: segment at %lld stops early\n", trial, (long long)u);
                return 1;
            }
            u = e;
        }
        for (int64_t t = nrot; t < rot_padded(nrot); ++t)
            if (cs[2 * t] != 0.0 || cs[2 * t + 1] != 0.0 || il[2 * t] != 0 || il[2 * t + 1] != 0) {
                std::printf("trial %d: padding\n", trial);
                return 1;
            }
        for (int k = 0; k < js; k += 1 + js / 8) {
            std::vector<double> z0((size_t)js, 0.0);
            z0[(size_t)k] = 1.0;
            std::vector<double> za = z0, zb = z0, zc = z0;
            apply_plain(za, ri, rc, rs, 0, (size_t)nrot);
            if (!apply_packed(zb, cs, il, nrot)) return 1;
            // in pieces of 777 rotations, each packed on its own
            for (int64_t p0 = 0; p0 < nrot; p0 += 777) {
                const int64_t cnt = std::min<int64_t>(777, nrot - p0);
                std::vector<double> pcs;
                std::vector<int32_t> pil;
                rot_pack(ri.data() + p0, rc.data() + p0, rs.data() + p0, cnt, js, pcs, pil);
                if (!apply_packed(zc, pcs, pil, cnt)) return 1;
            }
            if (std::memcmp(za.data(), zb.data(), (size_t)js * 8) || std::memcmp(za.data(), zc.data(), (size_t)js * 8)) {
                std::printf("trial %d: row %d differs from the sequential loop\n", trial, k);
                return 1;
            }
        }
        ++lists;
        total += nrot;
    }
    // refused indices
    for (int bad : {-1, 9}) {
        std::vector<int32_t> ri = {3, 2, bad};
        std::vector<double> rc = {1, 1, 1}, rs = {0, 0, 0};
        std::vector<double> cs;
        std::vector<int32_t> il;
        bool threw = false;
        try {
            rot_pack(ri.data(), rc.data(), rs.data(), 3, 10, cs, il);
        } catch (const Error& x) {
            threw = x.code == SVDB_ERR_LAS2;
        }
        if (!threw) {
            std::printf("index %d was not refused\n", bad);
            return 1;
        }
    }
    std::printf("ok %lld %lld\n", (long long)lists, (long long)total);
    return 0;
}
