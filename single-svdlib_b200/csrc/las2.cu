// LAS2 driver: svd_las2 / lanso / stpone / startv / ritvec
// (src/lanczos/mod.rs:104-1406 and, with `legacy`, src/legacy.rs:569-2016).
//
// Division of labour.  Everything that touches an n-vector, the matrix or the
// Lanczos store Q runs on the GPU: the Lanczos blocks (one cooperative launch
// per lanso block, lanczos_kernel.cu), startv/stpone, the rotation
// accumulation of imtql2, the back-transform and the sigma/u products
// (ritvec.cu).  What stays here is the control flow of lanso and the
// strictly sequential O(js^2) scalar recurrences of the tridiagonal QL
// iterations (imtqlb, the shift/rotation chain of imtql2, error_bound,
// insert_sort), restated line by line so that their exact floating-point
// behaviour -- including the as-written svd_pythag and imtqlb of the current
// crate -- is reproduced.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <limits>
#include <random>

#include "lanczos_kernel.cuh"
#include "ops.cuh"
#include "ql_host.h"
#include "ritvec.cuh"
#include "svdb_internal.h"

namespace svdb {

static size_t idamax(size_t n, const double* x) {
    if (n == 0) throw Error(SVDB_ERR_SHAPE, "svd_idamax: unexpected inputs!");
    size_t imax = 0;
    for (size_t i = 1; i < n; ++i)
        if (std::fabs(x[i]) > std::fabs(x[imax])) imax = i;
    return imax;
}
static void dcopy_rev(size_t n, size_t off, const double* x, double* y) {
    if (n > 0)
        for (size_t i = 0; i < n; ++i) y[off + n - 1 - i] = x[off + i];
}
static void insert_sort(size_t n, double* a1, double* a2) {
    for (size_t i = 1; i < n; ++i)
        for (size_t j = i; j >= 1; --j) {
            if (a1[j - 1] <= a1[j]) break;
            std::swap(a1[j - 1], a1[j]);
            std::swap(a2[j - 1], a2[j]);
        }
}

// Lanczos blocks on operators of at most kLzClusterNnz nonzeros run as one
// cluster of 2 * kLzCluster blocks where the device allows it, else of
// kLzCluster (the portable size).
constexpr int kLzCluster = 8;
constexpr int64_t kLzClusterNnz = 1 << 20;

struct Mode {
    bool legacy = false;
    double sparsity = 0.0;
    double adaptive_eps = EPS;
    size_t max_imtqlb = 30, max_imtql2 = 30, extra_steps = 0;
    int branch = 0;
};

// sparsity branches of lanso / ritvec (mod.rs:1068-1096, 1273-1300, 1390-1394)
static Mode make_mode(int64_t nrows, int64_t ncols, int64_t nnz, bool legacy) {
    Mode md;
    md.legacy = legacy;
    double sp = 1.0 - ((double)nnz / ((double)nrows * (double)ncols));
    md.sparsity = sp;
    md.branch = sp > 0.999 ? 3 : sp > 0.99 ? 2 : sp > 0.9 ? 1 : 0;
    if (legacy) return md;
    md.max_imtqlb = sp > 0.999 ? 500 : sp > 0.99 ? 300 : sp > 0.9 ? 100 : 50;
    md.adaptive_eps = sp > 0.99 ? EPS * 100.0 : sp > 0.9 ? EPS * 10.0 : EPS;
    md.max_imtql2 = sp > 0.999 ? 500 : sp > 0.99 ? 300 : sp > 0.9 ? 200 : 50;
    md.extra_steps = sp > 0.99 ? 5 : 0;
    return md;
}

// imtqlb as written (mod.rs:428-584): p and f are taken once per l, the
// convergence test is |e_m| <= 100 eps max(test, 1) sqrt(n), and the
// iteration cap is soft.
static void imtqlb_current(size_t n, double* d, double* e, double* bnd, size_t max_it, bool& warned) {
    if (n == 1) return;
    double msf = std::sqrt((double)n);
    bnd[0] = 1.0;
    size_t last = n - 1;
    for (size_t i = 1; i <= last; ++i) { bnd[i] = 0.0; e[i - 1] = e[i]; }
    e[last] = 0.0;
    size_t i = 0;
    for (size_t l = 0; l <= last; ++l) {
        size_t iteration = 0;
        double p = d[l], f = bnd[l];
        while (iteration <= max_it) {
            size_t m = l;
            while (m < n) {
                if (m == last) break;
                double test = std::fabs(d[m]) + std::fabs(d[m + 1]);
                double tol = EPS * 100.0 * std::fmax(test, 1.0) * msf;
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
                iteration = max_it + 1;
            } else {
                if (iteration == max_it) {
                    warned = true;
                    for (size_t idx = l; idx <= m; ++idx) bnd[idx] = std::fmax(bnd[idx], 0.1);
                    e[l] = 0.0;
                    break;
                }
                ++iteration;
                double g = (d[l + 1] - p) / (2.0 * e[l]);
                double r = pythag_current(g, 1.0);
                g = d[m] - p + e[l] / (g + fsign(r, g));
                double s = 1.0, c = 1.0;
                p = 0.0;
                i = m - 1;
                bool underflow = false;
                while (!underflow && i >= l) {
                    f = s * e[i];
                    double b = c * e[i];
                    r = pythag_current(f, g);
                    e[i + 1] = r;
                    if (r < EPS * 1000.0 * (std::fabs(f) + std::fabs(g))) { underflow = true; break; }
                    if (std::fabs(r) < EPS * 100.0) r = EPS * 100.0 * fsign(1.0, r);
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

// error_bound (mod.rs:840-899, identical in legacy.rs)
static size_t error_bound(bool& enough, double endl, double endr, double* ritz, double* bnd, size_t step,
                          double tol) {
    if (step == 0) throw Error(SVDB_ERR_SHAPE, "error_bound: expected 'step' to be non-zero");
    size_t mid = idamax(step + 1, bnd);
    double e34 = eps34();
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
    double gapl = ritz[step] - ritz[0];
    for (size_t k = 0; k <= step; ++k) {
        double gap = gapl;
        if (k < step) gapl = ritz[k + 1] - ritz[k];
        gap = std::fmin(gap, gapl);
        if (gap > bnd[k]) bnd[k] *= bnd[k] / gap;
        if (bnd[k] <= 16.0 * EPS * std::fabs(ritz[k])) {
            ++neig;
            if (!enough) enough = endl < ritz[k] && ritz[k] < endr;
        }
    }
    return neig;
}

// ----------------------------------------------------------- the run ----
struct Las2Out {
    int64_t d = 0, nsig = 0, steps = 0, neig = 0, dimensions = 0, iterations = 0;
    bool transposed = false;
    double kappa = 0.0;
    uint32_t seed = 0;
    DevBuf<double> Ut, S, Vt;
    int64_t ut_cols = 0, vt_cols = 0;
    double ms_total = 0, ms_lanczos = 0, ms_tridiag = 0, ms_ritvec = 0;
    int64_t npurge = 0;
};

class Las2Run {
  public:
    // f32: the crate's T = f32 run (f32 tolerances and start vector; FP32
    // operands in the products).  fp32: FP32 operands only (SVDB_MIXED).
    Las2Run(const svdb_matrix* A, bool legacy, bool fp32, bool f32, cudaStream_t s)
        : A_(A), s_(s), fp32_(fp32 || f32), f32_(f32) {
        legacy_ = legacy;
    }
    ~Las2Run() {
        if (rot_cs_) cudaStreamSynchronize(rot_cs_);  // every copy out of rot_pin_ has finished
        for (int b = 0; b < 2; ++b) {
            if (rot_ev_[b]) cudaEventDestroy(rot_ev_[b]);
            if (rot_free_[b]) cudaEventDestroy(rot_free_[b]);
            host_result_free(rot_pin_[b]);
        }
        if (rot_cs_) cudaStreamDestroy(rot_cs_);
    }
    Las2Run(const Las2Run&) = delete;
    Las2Run& operator=(const Las2Run&) = delete;

    void run(int64_t dimensions, int64_t iterations, double endl, double endr, double kappa, uint32_t seed,
             Las2Out& out);
    void fill_trace(svdb_trace* t, int64_t steps) const;

  private:
    const svdb_matrix* A_;
    cudaStream_t s_;
    bool fp32_ = false, f32_ = false, legacy_ = false, transposed_ = false;
    int64_t m_ = 0, n_ = 0;  // internal nrows / ncols
    const DevCompressed* op1_ = nullptr;
    const DevCompressed* op2_ = nullptr;
    Mode md_;
    DevBuf<double> W_[7], temp_, Q_, P_, alf_, bet_, etaA_, etaB_, part_, tq_, tr_, scratch_, tbuf_;
    DevBuf<LzState> st_;
    DevBuf<GridBarrier> bar_;
    int64_t qcap_ = 0, part_cap_ = 0;
    int perm_[7] = {0, 1, 2, 3, 4, 5, 6};
    int eta_sel_ = 0;
    int64_t npurge_ = 0;
    int lz_blocks_ = 0, lz_cluster_ = 0;
    bool lz_sliced_ = false;  // grid launches use both operands' column-sliced copies
    std::vector<double> alf_h_, bet_h_, ritz_, bnd_, w5_;
    // rotations of lanso's last Ritz analysis when it ran imtqlb (SVDLIBC)
    // on the whole T: ritvec's imtql2 would make the same ones (ql_host.h)
    Rotations lz_rot_;
    int64_t lz_rot_n_ = -1;
    // Z of that T, applied on the stream piece by piece while imtqlb runs
    // (a recorded rotation is final): kRotPiece rotations a piece, packed
    // into two page-locked buffers and copied into two device slots in turn,
    // on a copy stream, so the upload of piece k + 1 overlaps the kernel of
    // piece k.  rot_ev_[b]: the copy into slot b finished (host buffer b free
    // again); rot_free_[b]: the kernel that read slot b finished.
    static constexpr size_t kRotPiece = 8192;
    DevBuf<double> zrot_, rot_dcs_;
    DevBuf<int32_t> rot_dil_;
    void* rot_pin_[2] = {nullptr, nullptr};
    cudaEvent_t rot_ev_[2] = {nullptr, nullptr};
    cudaEvent_t rot_free_[2] = {nullptr, nullptr};
    cudaStream_t rot_cs_ = nullptr;
    int rot_buf_ = 0;
    int64_t zrot_n_ = -1, zrot_js_ = 0, zrot_js_cur_ = 0;
    size_t rot_done_ = 0;
    bool rot_started_ = false;
    void rot_stream_begin(int64_t js);
    void rot_stream_flush(size_t upto);

    double* w(int k) { return W_[perm_[k]].p; }
    void opb(const double* x, double* y) {
        spmv(*op1_, fp32_, x, temp_.p, s_);
        spmv(*op2_, fp32_, temp_.p, y, s_);
    }
    double ddot(const double* x, const double* y) { return dot_host(x, y, n_, scratch_.p, s_); }
    void ensure_q(int64_t rows);
    double startv(int64_t step, uint32_t seed);
    void stpone(uint32_t seed, double& rnm, double& tol);
    int64_t lanczos_step(int64_t first, int64_t last, int64_t& ll, bool& enough, double& rnm, double& tol);
    int64_t lanso(int64_t dim, int64_t iterations, double endl, double endr, int64_t& neig, uint32_t seed);
    void ritvec(int64_t dimensions, double kappa, int64_t steps, int64_t neig, Las2Out& out);
};

void Las2Run::rot_stream_begin(int64_t js) {
    if (!rot_pin_[0]) {
        const size_t bytes = (size_t)rot_padded((int64_t)kRotPiece) * 24;  // (c, s) and (index, length)
        SVDB_CUDA(cudaStreamCreateWithFlags(&rot_cs_, cudaStreamNonBlocking));
        for (int b = 0; b < 2; ++b) {
            rot_pin_[b] = host_result_alloc(bytes);
            SVDB_CUDA(cudaEventCreateWithFlags(&rot_ev_[b], cudaEventDisableTiming));
            SVDB_CUDA(cudaEventCreateWithFlags(&rot_free_[b], cudaEventDisableTiming));
        }
        rot_dcs_.alloc(4 * rot_padded((int64_t)kRotPiece), s_);  // two slots of (c, s) pairs
        rot_dil_.alloc(4 * rot_padded((int64_t)kRotPiece), s_);  // and of (index, length) pairs
    }
    if (js * js > zrot_js_ * zrot_js_) zrot_.alloc(js * js, s_);
    zrot_js_ = std::max(zrot_js_, js);
    zrot_n_ = -1;
    rot_done_ = 0;
    rot_started_ = false;
    zrot_js_cur_ = js;
}

// Applies rotations rot_done_ .. upto of lz_rot_ to zrot_ (the first piece
// starts from I; an empty list still makes I).
void Las2Run::rot_stream_flush(size_t upto) {
    if (upto == rot_done_ && rot_started_) return;
    const int64_t cnt = (int64_t)(upto - rot_done_);
    const int b = rot_buf_;
    rot_buf_ ^= 1;
    SVDB_CUDA(cudaEventSynchronize(rot_ev_[b]));  // the copy out of this buffer has finished
    double* pcs = static_cast<double*>(rot_pin_[b]);
    int32_t* pil = reinterpret_cast<int32_t*>(pcs + 2 * rot_padded((int64_t)kRotPiece));
    rot_pack(lz_rot_.i.data() + rot_done_, lz_rot_.c.data() + rot_done_, lz_rot_.s.data() + rot_done_, cnt,
             zrot_js_cur_, pcs, pil);
    const int64_t slot = (int64_t)b * 2 * rot_padded((int64_t)kRotPiece);
    SVDB_CUDA(cudaStreamWaitEvent(rot_cs_, rot_free_[b], 0));  // the kernel of two pieces ago read slot b
    if (cnt) {
        SVDB_CUDA(cudaMemcpyAsync(rot_dcs_.p + slot, pcs, (size_t)cnt * 16, cudaMemcpyHostToDevice, rot_cs_));
        SVDB_CUDA(cudaMemcpyAsync(rot_dil_.p + slot, pil, (size_t)cnt * 8, cudaMemcpyHostToDevice, rot_cs_));
    }
    SVDB_CUDA(cudaEventRecord(rot_ev_[b], rot_cs_));
    SVDB_CUDA(cudaStreamWaitEvent(s_, rot_ev_[b], 0));
    rot_apply(zrot_.p, zrot_js_cur_, rot_dcs_.p + slot, rot_dil_.p + slot, cnt, !rot_started_, s_);
    SVDB_CUDA(cudaEventRecord(rot_free_[b], s_));
    rot_done_ = upto;
    rot_started_ = true;
}

void Las2Run::ensure_q(int64_t rows) {
    if (rows <= qcap_) return;
    int64_t cap = std::max<int64_t>(rows, std::min<int64_t>(2 * qcap_, (int64_t)alf_h_.size() + 1));
    DevBuf<double> nq(cap * n_, s_);
    if (qcap_) SVDB_CUDA(cudaMemcpyAsync(nq.p, Q_.p, qcap_ * n_ * sizeof(double), cudaMemcpyDeviceToDevice, s_));
    Q_ = std::move(nq);
    qcap_ = cap;
}

// startv, mod.rs:587-640
double Las2Run::startv(int64_t step, uint32_t seed) {
    double rnm2 = ddot(w(0), w(0));
    for (int id = 0; id < 3; ++id) {
        if (id > 0 || step > 0 || compare(rnm2, 0.0)) start_vector(seed, w(0), n_, s_, f32_);
        copy(w(0), w(3), n_, s_);
        opb(w(3), w(0));
        copy(w(0), w(3), n_, s_);
        rnm2 = ddot(w(3), w(3));
        if (rnm2 > 0.0) break;
    }
    if (rnm2 <= 0.0) {
        char buf[128];
        snprintf(buf, sizeof buf, "svdlibrs/startv: rnm2 <= 0.0, rnm2 = %.1f", rnm2);
        throw Error(SVDB_ERR_STARTV, buf);
    }
    if (step > 0) {
        // for i < step: w0 -= (w3 . q_i) q_i  -- w3 is not modified in the loop
        ensure_q(step);
        gemv_t(Q_.p, n_, 0, step, w(3), tbuf_.p, part_.p, part_cap_, s_);
        gemv_sub(Q_.p, n_, 0, step, tbuf_.p, w(0), s_);
        double t = ddot(w(4), w(0));
        axpy(-t, w(2), w(0), n_, s_);
        copy(w(0), w(3), n_, s_);
        double dd = ddot(w(3), w(3));
        rnm2 = (dd <= EPS * rnm2) ? 0.0 : dd;
    }
    return std::sqrt(rnm2);
}

// stpone, mod.rs:643-670
void Las2Run::stpone(uint32_t seed, double& rnm_out, double& tol_out) {
    double rnm = startv(0, seed);
    if (compare(rnm, 0.0)) throw Error(SVDB_ERR_STPONE, "svdlibrs/stpone: rnm == 0.0");
    datx(1.0 / rnm, w(0), w(1), n_, s_);
    scal(1.0 / rnm, w(3), n_, s_);
    opb(w(3), w(0));
    double a0 = ddot(w(0), w(3));
    axpy(-a0, w(1), w(0), n_, s_);
    double t = ddot(w(0), w(3));
    a0 += t;
    axpy(-t, w(1), w(0), n_, s_);
    copy(w(0), w(4), n_, s_);
    rnm = std::sqrt(ddot(w(4), w(4)));
    alf_h_[0] = a0;
    SVDB_CUDA(cudaMemcpyAsync(alf_.p, &alf_h_[0], sizeof(double), cudaMemcpyHostToDevice, s_));
    double anorm = rnm + std::fabs(a0);
    rnm_out = rnm;
    tol_out = std::sqrt(EPS) * anorm;
}

// lanczos_step, mod.rs:674-758: device blocks, host startv on restarts.
int64_t Las2Run::lanczos_step(int64_t first, int64_t last, int64_t& ll, bool& enough, double& rnm, double& tol) {
    ensure_q(std::max<int64_t>(last, first) + 1);
    int64_t j = first;
    bool resume = false;
    while (j < last) {
        LzState hs;
        std::memset(&hs, 0, sizeof hs);
        hs.rnm = rnm; hs.tol = tol; hs.ll = ll;
        for (int k = 0; k < 7; ++k) hs.perm[k] = perm_[k];
        hs.eta_sel = eta_sel_;
        hs.npurge = npurge_;
        hs.j = j;
        SVDB_CUDA(cudaMemcpyAsync(st_.p, &hs, sizeof hs, cudaMemcpyHostToDevice, s_));
        GridBarrier b0;
        std::memset(&b0, 0, sizeof b0);
        b0.limit_ns = wait_limit_ns();
        SVDB_CUDA(cudaMemcpyAsync(bar_.p, &b0, sizeof b0, cudaMemcpyHostToDevice, s_));
        LzArgs a;
        std::memset(&a, 0, sizeof a);
        a.op1 = {op1_->ptr.p, op1_->idx.p, op1_->val.p, fp32_ ? op1_->val32.p : nullptr, op1_->nmajor,
                 op1_->plan.multi_rows.p, op1_->plan.nmulti, op1_->plan.bins, SlicedOp{}, nullptr, nullptr};
        a.op2 = {op2_->ptr.p, op2_->idx.p, op2_->val.p, fp32_ ? op2_->val32.p : nullptr, op2_->nmajor,
                 op2_->plan.multi_rows.p, op2_->plan.nmulti, op2_->plan.bins, SlicedOp{}, nullptr, nullptr};
        if (lz_sliced_) {
            a.op1.sl = sliced_view(*op1_);
            a.op1.sv = op1_->sliced.sval.p;
            a.op1.svf = op1_->sliced.sval32.p;
            a.op2.sl = sliced_view(*op2_);
            a.op2.sv = op2_->sliced.sval.p;
            a.op2.svf = op2_->sliced.sval32.p;
        }
        a.n = n_;
        for (int k = 0; k < 7; ++k) a.W[k] = W_[k].p;
        a.temp = temp_.p;
        a.Q = Q_.p;
        a.P = P_.p;
        a.alf = alf_.p; a.bet = bet_.p; a.etaA = etaA_.p; a.etaB = etaB_.p;
        a.part = part_.p; a.part_cap = part_cap_;
        a.tq = tq_.p; a.tr = tr_.p;
        a.st = st_.p; a.bar = bar_.p;
        a.first = j; a.last = last; a.resume = resume ? 1 : 0;
        a.eps1 = EPS * std::sqrt((double)n_);
        a.sqrt_eps = std::sqrt(EPS);
        launch_lanczos_block(a, lz_blocks_, 512, lz_cluster_, s_, lz_sliced_);
        GridBarrier hb;
        SVDB_CUDA(cudaMemcpyAsync(&hs, st_.p, sizeof hs, cudaMemcpyDeviceToHost, s_));
        SVDB_CUDA(cudaMemcpyAsync(&hb, bar_.p, sizeof hb, cudaMemcpyDeviceToHost, s_));
        SVDB_CUDA(cudaStreamSynchronize(s_));
        if (hb.err) throw Error(SVDB_ERR_TIMEOUT, "lanczos block: grid barrier wait exceeded its limit");
        for (int k = 0; k < 7; ++k) perm_[k] = hs.perm[k];
        rnm = hs.rnm; tol = hs.tol; ll = hs.ll; eta_sel_ = hs.eta_sel; npurge_ = hs.npurge;
        j = hs.j;
        if (hs.status == 0) return j;
        // invariant subspace at step j: restart (mod.rs:699-710)
        rnm = startv(j, 0);
        if (compare(rnm, 0.0)) enough = true;
        if (enough) {
            std::swap(perm_[1], perm_[2]);
            return j;
        }
        resume = true;
    }
    return j;
}

// lanso, mod.rs:1263-1406 / legacy.rs:1920-2016
int64_t Las2Run::lanso(int64_t dim, int64_t iterations, double endl, double endr, int64_t& neig, uint32_t seed) {
    double rnm, tol;
    stpone(seed, rnm, tol);
    const double eps1 = (md_.legacy ? EPS : md_.adaptive_eps) * std::sqrt((double)n_);
    SVDB_CUDA(cudaMemcpyAsync(etaA_.p, &eps1, sizeof(double), cudaMemcpyHostToDevice, s_));
    SVDB_CUDA(cudaMemcpyAsync(etaB_.p, &eps1, sizeof(double), cudaMemcpyHostToDevice, s_));
    eta_sel_ = 0;
    int64_t ll = 0, first = 1;
    int64_t last = std::min<int64_t>(iterations, std::max<int64_t>(dim, 8) + dim);
    bool enough = false;
    int64_t j = 0, intro = 0;
    bool warned = false;
    while (!enough) {
        if (rnm <= tol) rnm = 0.0;
        int64_t steps = lanczos_step(first, last, ll, enough, rnm, tol);
        j = enough ? steps - 1 : last - 1;
        first = j + 1;
        bet_h_[first] = rnm;
        SVDB_CUDA(cudaMemcpyAsync(bet_.p + first, &bet_h_[first], sizeof(double), cudaMemcpyHostToDevice, s_));
        if (j > 0) {
            SVDB_CUDA(cudaMemcpyAsync(alf_h_.data(), alf_.p, (j + 1) * sizeof(double), cudaMemcpyDeviceToHost, s_));
            SVDB_CUDA(cudaMemcpyAsync(bet_h_.data(), bet_.p, (j + 1) * sizeof(double), cudaMemcpyDeviceToHost, s_));
            SVDB_CUDA(cudaStreamSynchronize(s_));
        }
        // analyse T in unreduced blocks (mod.rs:1345-1377)
        int64_t l = 0;
        lz_rot_n_ = zrot_n_ = -1;
        for (int64_t it = 0; it < j; ++it) {
            if (l > j) break;
            int64_t i = l;
            while (i <= j) {
                bool split = md_.legacy ? compare(bet_h_[i + 1], 0.0) : std::fabs(bet_h_[i + 1]) <= md_.adaptive_eps;
                if (split) break;
                ++i;
            }
            i = std::min(i, j);
            size_t sz = (size_t)(i - l);
            dcopy_rev(sz + 1, l, alf_h_.data(), ritz_.data());
            dcopy_rev(sz, l + 1, bet_h_.data(), w5_.data());
            if (md_.legacy) {
                if (l == 0 && i == j) {  // the whole T: record its rotations and apply them meanwhile
                    rot_stream_begin((int64_t)sz + 1);
                    const std::function<void(size_t)> flush = [this](size_t k) { rot_stream_flush(k); };
                    imtqlb_legacy(sz + 1, ritz_.data(), w5_.data(), bnd_.data(), &lz_rot_, &flush, kRotPiece);
                    rot_stream_flush(lz_rot_.i.size());
                    lz_rot_n_ = zrot_n_ = (int64_t)sz + 1;
                } else {
                    imtqlb_legacy(sz + 1, ritz_.data() + l, w5_.data() + l, bnd_.data() + l);
                }
            }
            else imtqlb_current(sz + 1, ritz_.data() + l, w5_.data() + l, bnd_.data() + l, md_.max_imtqlb, warned);
            for (int64_t mm = l; mm <= i; ++mm) bnd_[mm] = rnm * std::fabs(bnd_[mm]);
            l = i + 1;
        }
        insert_sort((size_t)j + 1, ritz_.data(), bnd_.data());
        neig = (int64_t)error_bound(enough, endl, endr, ritz_.data(), bnd_.data(), (size_t)j, tol);
        if (neig < dim) {
            if (neig == 0) { last = first + 9; intro = first; }
            else {
                int64_t ext = std::max<int64_t>(3, 1 + ((j - intro) * (dim - neig)) / neig);
                last = first + ext + (md_.legacy ? 0 : (int64_t)md_.extra_steps);
            }
            last = std::min(last, iterations);
        } else enough = true;
        enough = enough || first >= iterations;
    }
    if (warned)
        fprintf(stderr, "Warning: imtqlb had some convergence issues but continued with best estimates. "
                        "Results may have reduced accuracy.\n");
    // store.storq(j, w1)
    ensure_q(j + 1);
    SVDB_CUDA(cudaMemcpyAsync(Q_.p + j * n_, w(1), n_ * sizeof(double), cudaMemcpyDeviceToDevice, s_));
    return j;
}

// ritvec, mod.rs:1056-1259 / legacy.rs:1766-1850
void Las2Run::ritvec(int64_t dimensions, double kappa, int64_t steps, int64_t neig, Las2Out& out) {
    const int64_t js = steps + 1;
    std::vector<double> d(js, 0.0);
    dcopy_rev((size_t)js, 0, alf_h_.data(), d.data());
    SVDB_CUDA(cudaMemcpyAsync(bet_h_.data(), bet_.p, (js + 1) * sizeof(double), cudaMemcpyDeviceToHost, s_));
    SVDB_CUDA(cudaStreamSynchronize(s_));
    dcopy_rev((size_t)steps, 1, bet_h_.data(), w5_.data());
    Rotations R;
    const bool have_z = md_.legacy && lz_rot_n_ == js && zrot_n_ == js && md_.max_imtql2 == 30;
    if (md_.legacy && lz_rot_n_ == js && md_.max_imtql2 == 30) {
        // T is the one lanso's last imtqlb saw: its record is imtql2's
        R.i.swap(lz_rot_.i);
        R.c.swap(lz_rot_.c);
        R.s.swap(lz_rot_.s);
        d = lz_rot_.d;
        R.perm.resize((size_t)js);
        for (int64_t k = 0; k < js; ++k) R.perm[(size_t)k] = (int32_t)k;
        ql_sort_perm((size_t)js, d.data(), R.perm);
        lz_rot_n_ = -1;
    } else {
        imtql2_scalar((size_t)js, d.data(), w5_.data(), md_.legacy, md_.max_imtql2, R);
    }

    // selection of the output rows (their ritz index k, in output order)
    std::vector<int32_t> rowk;
    int64_t nsig = 0;
    const double ae = md_.adaptive_eps;
    if (!md_.legacy) {
        double max_eig = 0.0;  // fold over Vt.value: the js eigenvalues and zeros
        for (int64_t k = 0; k < js; ++k) max_eig = std::fmax(max_eig, std::fabs(d[k]));
        double akappa = md_.sparsity > 0.99 ? kappa * 10.0 : kappa;
        std::vector<int32_t> sig;
        for (int64_t k = 0; k < js; ++k) {
            double rel = akappa * std::fmax(std::fabs(ritz_[k]), max_eig * ae);
            if (bnd_[k] <= rel && k + 1 > js - neig) sig.push_back((int32_t)k);
        }
        nsig = (int64_t)sig.size();
        int64_t dd = std::min<int64_t>(dimensions, nsig);
        rowk.assign(sig.begin(), sig.begin() + dd);
    } else {
        // cyclic fill from row dimensions-1 downwards, then rotate_array by x rows
        std::vector<int32_t> slot(dimensions, -1);
        int64_t x = 0;
        for (int64_t k = 0; k < js; ++k) {
            if (bnd_[k] <= kappa * std::fabs(ritz_[k]) && k + 1 > js - neig) {
                x = (x == 0) ? dimensions - 1 : x - 1;
                slot[x] = (int32_t)k;
                ++nsig;
            }
        }
        int64_t dd = std::min<int64_t>(dimensions, nsig);
        for (int64_t r = 0; r < dd; ++r) rowk.push_back(slot[(r + x) % dimensions]);
    }
    const int64_t d_out = (int64_t)rowk.size();
    out.d = d_out;
    out.nsig = nsig;
    out.ut_cols = m_;
    out.vt_cols = n_;
    out.Ut.alloc(std::max<int64_t>(d_out * m_, 1), s_);
    out.S.alloc(std::max<int64_t>(d_out, 1), s_);
    out.Vt.alloc(std::max<int64_t>(d_out * n_, 1), s_);
    if (d_out == 0) return;

    cudaEvent_t e0, e1;
    SVDB_CUDA(cudaEventCreate(&e0));
    SVDB_CUDA(cudaEventCreate(&e1));
    SVDB_CUDA(cudaEventRecord(e0, s_));
    DevBuf<int32_t> dperm(js, s_), drowk(d_out, s_);
    DevBuf<double> Z, C(d_out * js, s_);
    const double* zp = zrot_.p;  // Z made while lanso's imtqlb ran
    if (!have_z) {
        const int64_t nrot = (int64_t)R.i.size();
        std::vector<double> hcs;
        std::vector<int32_t> hil;
        rot_pack(R.i.data(), R.c.data(), R.s.data(), nrot, js, hcs, hil);
        const int64_t npad = rot_padded(nrot);
        DevBuf<int32_t> dil(2 * npad, s_);
        DevBuf<double> dcs(2 * npad, s_);
        Z.alloc(js * js, s_);
        if (nrot) {
            SVDB_CUDA(cudaMemcpyAsync(dcs.p, hcs.data(), nrot * 16, cudaMemcpyHostToDevice, s_));
            SVDB_CUDA(cudaMemcpyAsync(dil.p, hil.data(), nrot * 8, cudaMemcpyHostToDevice, s_));
        }
        rot_apply(Z.p, js, dcs.p, dil.p, nrot, true, s_);
        zp = Z.p;
    }
    SVDB_CUDA(cudaMemcpyAsync(dperm.p, R.perm.data(), js * 4, cudaMemcpyHostToDevice, s_));
    SVDB_CUDA(cudaMemcpyAsync(drowk.p, rowk.data(), d_out * 4, cudaMemcpyHostToDevice, s_));
    build_coef(zp, js, dperm.p, drowk.p, d_out, md_.legacy, ae, C.p, s_);
    SVDB_CUDA(cudaEventRecord(e1, s_));
    backtransform(C.p, Q_.p, js, n_, d_out, out.Vt.p, s_);
    sigma_and_u(*op1_, *op2_, fp32_, out.Vt.p, d_out, n_, m_, md_.legacy, ae, out.S.p, out.Ut.p, s_);
    SVDB_CUDA(cudaStreamSynchronize(s_));
    float ms = 0.f;
    SVDB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    out.ms_tridiag += ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

void Las2Run::run(int64_t dimensions, int64_t iterations, double endl, double endr, double kappa, uint32_t seed,
                  Las2Out& out) {
    if (seed == 0) seed = std::random_device{}();
    const int64_t mn = std::min(A_->nrows, A_->ncols);
    if (dimensions == 0 || dimensions > mn) dimensions = mn;
    if (iterations == 0 || iterations > mn) iterations = mn;
    else if (iterations < dimensions) iterations = dimensions;
    if (dimensions < 2) {
        char buf[128];
        snprintf(buf, sizeof buf, legacy_ ? "svdlibrs/svdLas2: svdLAS2: insufficient dimensions: %lld"
                                          : "svdlibrs/svdLas2: svd_las2: insufficient dimensions: %lld",
                 (long long)dimensions);
        throw Error(SVDB_ERR_LAS2, buf);
    }
    transposed_ = (double)A_->ncols >= (double)A_->nrows * 1.2;
    m_ = transposed_ ? A_->ncols : A_->nrows;
    n_ = transposed_ ? A_->nrows : A_->ncols;
    op1_ = transposed_ ? &csc_of(A_) : &csr_of(A_);
    op2_ = transposed_ ? &csr_of(A_) : &csc_of(A_);
    md_ = make_mode(A_->nrows, A_->ncols, A_->nnz, legacy_);
    if (fp32_) ensure_fp32(A_);

    cudaEvent_t t0, t1, t2;
    SVDB_CUDA(cudaEventCreate(&t0));
    SVDB_CUDA(cudaEventCreate(&t1));
    SVDB_CUDA(cudaEventCreate(&t2));
    SVDB_CUDA(cudaEventRecord(t0, s_));

    for (auto& b : W_) {
        b.alloc(n_, s_);
        SVDB_CUDA(cudaMemsetAsync(b.p, 0, n_ * sizeof(double), s_));
    }
    temp_.alloc(std::max<int64_t>(m_, 1), s_);
    P_.alloc(2 * n_, s_);
    const int64_t cap = iterations + 2;
    alf_.alloc(cap, s_); bet_.alloc(cap, s_); etaA_.alloc(cap, s_); etaB_.alloc(cap, s_);
    tq_.alloc(cap, s_); tr_.alloc(cap, s_); tbuf_.alloc(cap, s_);
    SVDB_CUDA(cudaMemsetAsync(alf_.p, 0, cap * 8, s_));
    SVDB_CUDA(cudaMemsetAsync(bet_.p, 0, cap * 8, s_));
    SVDB_CUDA(cudaMemsetAsync(etaA_.p, 0, cap * 8, s_));
    SVDB_CUDA(cudaMemsetAsync(etaB_.p, 0, cap * 8, s_));
    scratch_.alloc(reduce_scratch_doubles(), s_);
    st_.alloc(1, s_);
    bar_.alloc(1, s_);
    alf_h_.assign(cap, 0.0);
    bet_h_.assign(cap, 0.0);
    ritz_.assign(cap, 0.0);
    bnd_.assign(cap, std::numeric_limits<double>::max());
    w5_.assign(cap, 0.0);
    // cooperative grid: enough blocks for the sparse products, at most the
    // co-resident maximum
    const int maxb = lanczos_max_blocks(512);
    int64_t want = std::max<int64_t>({op1_->nmajor * group_for(op1_->avg_per_major()),
                                      op2_->nmajor * group_for(op2_->avg_per_major()), n_}) / 512 + 1;
    if (const char* env = getenv("SVDB_LZ_BLOCKS")) want = atoi(env);
    lz_blocks_ = (int)std::max<int64_t>(1, std::min<int64_t>(want, maxb));
    // Small operators: one cluster of kLzCluster blocks, whose hardware barrier
    // and shared-memory partials replace the grid barrier (SVDB_LZ_CLUSTER=0
    // keeps the cooperative grid, =1 forces the cluster).
    {
        const char* env = getenv("SVDB_LZ_CLUSTER");
        const bool small = op1_->nnz <= kLzClusterNnz && op2_->nnz <= kLzClusterNnz;
        const bool want_cl = env ? atoi(env) != 0 : small;
        lz_cluster_ = 0;
        if (want_cl) {  // the widest cluster that fits: 16 blocks (non-portable), else 8
            for (int c : {2 * kLzCluster, kLzCluster})
                if (lanczos_cluster_ok(c, 512)) { lz_cluster_ = c; break; }
        }
        if (lz_cluster_) lz_blocks_ = lz_cluster_;
    }
    // Large operators in grid mode: x slices in shared memory for both
    // products (spmv_sliced.cu), one block per SM (SVDB_SPMV=gather keeps the
    // gather products).
    if (!lz_cluster_) {
        const char* env = getenv("SVDB_SPMV");
        const bool sliced = env && std::string(env) == "sliced";  // opt-in, as in spmv()
        if (sliced && sliced_prepare(*op1_, fp32_, s_) && sliced_prepare(*op2_, fp32_, s_)) {
            const int sb = lanczos_sliced_blocks(512);
            if (sb > 0) {
                lz_sliced_ = true;
                lz_blocks_ = sb;
            }
        }
    }
    const int64_t nsplit_max = (n_ + 2047) / 2048;
    part_cap_ = std::max<int64_t>({2 * (int64_t)lz_blocks_, 2 * cap * nsplit_max, 2 * cap});
    part_.alloc(part_cap_, s_);

    int64_t neig = 0;
    int64_t steps = lanso(dimensions, iterations, endl, endr, neig, seed);
    out.steps = steps;  // visible to the trace even if ritvec fails
    out.neig = neig;
    SVDB_CUDA(cudaEventRecord(t1, s_));
    double kap = std::fmax(std::fabs(kappa), eps34());
    if (f32_) kap = (double)(float)kap;  // Float::max(|kappa|, eps34) in f32 (mod.rs:162)
    ritvec(dimensions, kap, steps, neig, out);
    SVDB_CUDA(cudaEventRecord(t2, s_));
    SVDB_CUDA(cudaStreamSynchronize(s_));
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, t0, t1);
    cudaEventElapsedTime(&b, t1, t2);
    out.ms_lanczos = a;
    out.ms_ritvec = b;
    out.ms_total = a + b;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaEventDestroy(t2);
    if (transposed_) {
        std::swap(out.Ut, out.Vt);
        std::swap(out.ut_cols, out.vt_cols);
    }
    out.steps = steps;
    out.neig = neig;
    out.dimensions = dimensions;
    out.iterations = iterations;
    out.transposed = transposed_;
    out.kappa = kap;
    out.seed = seed;
    out.npurge = npurge_;
}

void Las2Run::fill_trace(svdb_trace* t, int64_t steps) const {
    if (!t) return;
    t->steps = (uint64_t)steps;
    t->purges = (uint64_t)npurge_;
    t->sparsity_branch = md_.branch;
    t->lanczos_blocks = lz_blocks_;
    auto put = [&](double* dst, const std::vector<double>& src, int64_t count) {
        if (!dst) return;
        int64_t c = std::min<int64_t>({count, (int64_t)t->cap, (int64_t)src.size()});
        if (c > 0) std::memcpy(dst, src.data(), c * sizeof(double));
    };
    put(t->alf, alf_h_, steps + 1);
    put(t->bet, bet_h_, steps + 2);
    put(t->ritz, ritz_, steps + 1);
    put(t->bnd, bnd_, steps + 1);
}

// Entry used by the C ABI.  f32: the crate's lanczos at T = f32 (f32
// epsilon in every tolerance, f32 start vector, FP32 operands).
void las2(const svdb_matrix* A, uint64_t dimensions, uint64_t iterations, const double end_interval[2],
          double kappa, uint32_t seed, bool legacy, const svdb_options& o, svdb_rec* rec, bool f32) {
    cudaStream_t s = o.stream ? (cudaStream_t)o.stream : A->stream;
    if (f32 && legacy) throw Error(SVDB_ERR_UNSUPPORTED, "legacy::svdLAS2 is f64-only");
    ScalarEps scalar_eps(f32);
    Las2Out out;
    {
        Las2Run run(A, legacy, o.precision == SVDB_MIXED, f32, s);
        try {
            run.run((int64_t)dimensions, (int64_t)iterations, end_interval[0], end_interval[1], kappa, seed, out);
        } catch (Error&) {
            run.fill_trace(o.trace, out.steps);
            throw;
        }
        run.fill_trace(o.trace, out.steps);
    }
    std::memset(rec, 0, sizeof(*rec));
    rec->d = out.d;
    rec->u_rows = out.d;
    rec->u_cols = out.ut_cols;
    rec->vt_rows = out.d;
    rec->vt_cols = out.vt_cols;
    const size_t nu = out.d * out.ut_cols, nv = out.d * out.vt_cols;
    if (o.result_on_device) {
        rec->u = out.Ut.detach();
        rec->s = out.S.detach();
        rec->vt = out.Vt.detach();
        rec->on_device = 1;
        SVDB_CUDA(cudaStreamSynchronize(s));
    } else {
        rec->u = (double*)host_result_alloc(std::max<size_t>(nu, 1) * sizeof(double));
        rec->s = (double*)host_result_alloc(std::max<size_t>(out.d, 1) * sizeof(double));
        rec->vt = (double*)host_result_alloc(std::max<size_t>(nv, 1) * sizeof(double));
        if (nu) SVDB_CUDA(cudaMemcpyAsync(rec->u, out.Ut.p, nu * 8, cudaMemcpyDeviceToHost, s));
        if (out.d) SVDB_CUDA(cudaMemcpyAsync(rec->s, out.S.p, out.d * 8, cudaMemcpyDeviceToHost, s));
        if (nv) SVDB_CUDA(cudaMemcpyAsync(rec->vt, out.Vt.p, nv * 8, cudaMemcpyDeviceToHost, s));
        SVDB_CUDA(cudaStreamSynchronize(s));
        rec->on_device = 0;
    }
    svdb_diagnostics& dg = rec->diagnostics;
    dg.non_zero = A->nnz;
    dg.dimensions = out.dimensions;
    dg.iterations = out.iterations;
    dg.transposed = out.transposed;
    dg.lanczos_steps = out.steps + 1;
    dg.ritz_values_stabilized = out.neig;
    dg.significant_values = out.d;
    dg.singular_values = out.nsig;
    dg.end_interval[0] = end_interval[0];
    dg.end_interval[1] = end_interval[1];
    dg.kappa = out.kappa;
    dg.random_seed = out.seed;
    rec->origin = legacy ? SVDB_REC_LEGACY : SVDB_REC_LANCZOS;
    rec->time_ms_total = out.ms_total;
    rec->time_ms_spmv = out.ms_lanczos;
    rec->time_ms_ortho = 0.0;
    rec->time_ms_tridiag = out.ms_tridiag;
    rec->time_ms_ritvec = out.ms_ritvec;
}

int las2_plan(uint64_t nrows, uint64_t ncols, uint64_t nnz, uint64_t dimensions, uint64_t iterations,
              uint64_t* dims_out, uint64_t* iters_out, int32_t* transposed_out, int32_t* branch_out) {
    uint64_t mn = std::min(nrows, ncols);
    if (dimensions == 0 || dimensions > mn) dimensions = mn;
    if (iterations == 0 || iterations > mn) iterations = mn;
    else if (iterations < dimensions) iterations = dimensions;
    if (dims_out) *dims_out = dimensions;
    if (iters_out) *iters_out = iterations;
    if (transposed_out) *transposed_out = (double)ncols >= (double)nrows * 1.2;
    if (branch_out) *branch_out = make_mode((int64_t)nrows, (int64_t)ncols, (int64_t)nnz, false).branch;
    if (dimensions < 2) {
        char buf[128];
        snprintf(buf, sizeof buf, "svdlibrs/svdLas2: svd_las2: insufficient dimensions: %llu",
                 (unsigned long long)dimensions);
        throw Error(SVDB_ERR_LAS2, buf);
    }
    return 0;
}

}  // namespace svdb
