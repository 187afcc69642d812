// Reads tridiagonals (d, e; e[0] unused) from a binary file and checks that
// imtqlb_legacy's record (rotations, converged eigenvalues, column order) is
// bit for bit what imtql2_scalar makes on the same T in SVDLIBC mode, or that
// both fail alike.  Prints "ok <cases> <rotations>" or the first mismatch.
// Built and run by test_ql_record.py.
#include <cstdio>
#include <cstring>
#include <vector>

#include "ql_host.h"

using namespace svdb;

int main(int argc, char** argv) {
    if (argc != 2) return 2;
    FILE* fp = std::fopen(argv[1], "rb");
    if (!fp) return 2;
    int64_t cases = 0, total_rot = 0;
    int64_t n = 0;
    while (std::fread(&n, sizeof n, 1, fp) == 1) {
        std::vector<double> d((size_t)n), e((size_t)n);
        if (std::fread(d.data(), 8, (size_t)n, fp) != (size_t)n || std::fread(e.data(), 8, (size_t)n, fp) != (size_t)n)
            return 2;
        std::vector<double> d1 = d, e1 = e, bnd((size_t)n), d2 = d, e2 = e;
        Rotations rec, q2;
        int err1 = 0, err2 = 0;
        try {
            imtqlb_legacy((size_t)n, d1.data(), e1.data(), bnd.data(), &rec);
        } catch (const Error& x) {
            err1 = x.code;
        }
        try {
            imtql2_scalar((size_t)n, d2.data(), e2.data(), true, 30, q2);
        } catch (const Error& x) {
            err2 = x.code;
        }
        if ((err1 != 0) != (err2 != 0)) {
            std::printf("case %lld: imtqlb status %d, imtql2 status %d\n", (long long)cases, err1, err2);
            return 1;
        }
        if (!err1) {
            std::vector<int32_t> perm((size_t)n);
            for (int64_t k = 0; k < n; ++k) perm[(size_t)k] = (int32_t)k;
            std::vector<double> dr = rec.d;
            ql_sort_perm((size_t)n, dr.data(), perm);
            const size_t nr = rec.i.size();
            if (nr != q2.i.size() || std::memcmp(rec.i.data(), q2.i.data(), nr * 4) ||
                std::memcmp(rec.c.data(), q2.c.data(), nr * 8) || std::memcmp(rec.s.data(), q2.s.data(), nr * 8)) {
                std::printf("case %lld (n=%lld): rotation lists differ (%zu vs %zu)\n", (long long)cases,
                            (long long)n, nr, q2.i.size());
                return 1;
            }
            if (perm != q2.perm || std::memcmp(dr.data(), d2.data(), (size_t)n * 8)) {
                std::printf("case %lld (n=%lld): eigenvalue order differs\n", (long long)cases, (long long)n);
                return 1;
            }
            // imtqlb's own sorted output is the same set of values
            for (int64_t k = 0; k < n; ++k)
                if (std::memcmp(&d1[(size_t)k], &d2[(size_t)k], 8)) {
                    std::printf("case %lld: imtqlb's sorted eigenvalue %lld differs\n", (long long)cases, (long long)k);
                    return 1;
                }
            total_rot += (int64_t)nr;
        }
        ++cases;
    }
    std::fclose(fp);
    std::printf("ok %lld %lld\n", (long long)cases, (long long)total_rot);
    return 0;
}
