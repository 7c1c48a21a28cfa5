// Host engine of the B200 TLR Cholesky: contexts, descriptors, the
// device-resident tile store, the per-panel scheduler that replaces PaRSEC's
// task graph, generation, band auto-tuning, solve and the C ABI.
//
// Scheduler.  The reference runs HiCMA_dpotrf_L_2flow.jdf as a distributed
// DAG.  On one GPU every panel k is executed as a short sequence of batched
// launches on one stream: POTRF(k) (blocked, DMMA updates) and L_kk^-1, then
// one batched launch group each for all TRSM(m,k), all SYRK(k,m) and all
// GEMM(m,n,k) of the panel.  Tasks of one class inside a panel are
// independent (JDF flows: TRSM(m,k) <- POTRF(k); SYRK/GEMM read column k and
// write disjoint tiles), so batching them preserves the reference's data
// flow.  The host reads the rank map once per panel (the sizes of the next
// panel's tasks depend on the ranks the recompressions produced).
#include "tlr_internal.h"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

using namespace tlr;

// --------------------------------------------------------------- errors ----
static thread_local std::string g_err;
static void set_err(const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}
extern "C" const char *hicma_tlr_last_error(void) { return g_err.c_str(); }
void tlr::tlr_set_error(const char *msg) { g_err = msg ? msg : ""; }

#ifdef TLR_BOUNDS_CHECK
// ------------------------------------------------------ bounds registry ----
// Live device regions, process-wide (contexts on several devices share it).
static std::mutex g_bc_mu;
static std::vector<std::pair<uintptr_t, size_t>> g_bc_regions;
void tlr::bc_add(const void *p, size_t bytes) {
    if (!p || !bytes) return;
    std::lock_guard<std::mutex> lk(g_bc_mu);
    g_bc_regions.push_back({(uintptr_t)p, bytes});
}
void tlr::bc_remove(const void *p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_bc_mu);
    for (size_t i = g_bc_regions.size(); i-- > 0;)
        if (g_bc_regions[i].first == (uintptr_t)p) {
            g_bc_regions.erase(g_bc_regions.begin() + (long)i);
            return;
        }
}
bool tlr::bc_inside(const void *p, size_t bytes) {
    if (!bytes) return true;
    const uintptr_t a = (uintptr_t)p;
    if (a + bytes < a) return false;
    std::lock_guard<std::mutex> lk(g_bc_mu);
    for (const auto &r : g_bc_regions)
        if (a >= r.first && a + bytes <= r.first + r.second) return true;
    return false;
}
#endif

// Named host range of a phase in profiler timelines (NVTX; a no-op unless a
// tool is attached).  end() closes it early; the destructor closes it otherwise.
struct NvtxRange {
    bool open = true;
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    void end() {
        if (open) {
            nvtxRangePop();
            open = false;
        }
    }
    ~NvtxRange() { end(); }
};

// Registers caller buffers for the length of a kernel-level call (bounds-checked builds).
struct BcScope {
    std::vector<const void *> ps;
    void add(const void *p, size_t bytes) {
        if (p && bytes) { bc_add(p, bytes); ps.push_back(p); }
    }
    ~BcScope() { for (const void *p : ps) bc_remove(p); }
};

#define CUDA_TRY(x)                                                                         \
    do {                                                                                    \
        cudaError_t e__ = (x);                                                              \
        if (e__ != cudaSuccess) {                                                           \
            set_err("%s:%d %s: %s", __FILE__, __LINE__, #x, cudaGetErrorString(e__));       \
            return e__ == cudaErrorMemoryAllocation ? HICMA_TLR_ERR_OOM : HICMA_TLR_ERR_CUDA; \
        }                                                                                   \
    } while (0)
#define TRY(x)                         \
    do {                               \
        int r__ = (x);                 \
        if (r__ != 0) return r__;      \
    } while (0)
#define ARG_CHECK(cond, msg)                      \
    do {                                          \
        if (!(cond)) {                            \
            set_err("invalid argument: %s", msg); \
            return HICMA_TLR_ERR_ARG;             \
        }                                         \
    } while (0)

// --------------------------------------------------------------- context ---
struct Arena {
    char *base = nullptr;
    size_t bytes = 0, off = 0;
};

struct hicma_tlr_ctx_s {
    int device = 0;
    cudaStream_t stream = nullptr;      // bulk work
    cudaStream_t stream_hi = nullptr;   // critical path (high priority): SYRK(k,k+1) + POTRF(k+1)
    cudaStream_t stream_side = nullptr; // wide recompressions (Householder chain) beside the CholeskyQR chain
    cudaStream_t stream_copy = nullptr; // copy-out of final factor columns during a factorization
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaStream_t cur = nullptr;         // stream the helpers launch on
    char *d_ws = nullptr;
    size_t ws_bytes = 0;
    Arena main_ar, hi_ar;               // workspace of `stream` / `stream_hi`
    Arena *ar = nullptr;                // arena of `cur`
    char *h_stage = nullptr, *d_stage = nullptr;
    size_t stage_bytes = 0, stage_off = 0;
    int *d_flags = nullptr;     // [0] info, [1] overflow, [2] Jacobi sweeps, [3] wait timed out, [4] FP32 updates,
                                // [5] CholeskyQR null pivots, [6] CholeskyQR passes repeated
    int nsm = 148;              // SM count of the device
    // choices the autotuner measures (defaults: the hand-picked values)
    int gemm_narrow_n = GEMM_NARROW_N;   // rank-wide outputs up to this width use 128 x 32 tiles
    int potrf_grid = 0;                  // CTAs of the persistent tile POTRF (0: one per SM)
    // QRs of the recompressions: randomized CholeskyQR on both sides for stacked
    // ranks up to rcholqr_kmax() and the generation range finder up to that many samples
    // (1), the Householder pipeline for all (0; HICMA_TLR_QR=householder)
    int cholqr = 1;
    double *d_scal = nullptr;   // device scalars
    double *d_profacc = nullptr;   // per profiling class: flops, bytes counted on the device
    int precision = HICMA_TLR_PREC_FP64;
    long long launches = 0;
    std::recursive_mutex mu;
    std::thread async_thread;
    int async_ret = 0;
    std::string async_err;   // error message of the background factorization (its own thread's)
    std::set<hicma_tlr_desc_s *> descs;   // live descriptors, orphaned by fini
    // per-kernel-class profiling (CUDA events around launches on `stream`)
    bool prof = false;
    struct ProfRec { int cls; cudaEvent_t a, b; double flops, bytes; };
    std::vector<ProfRec> prof_recs;
    std::vector<cudaEvent_t> ev_pool;
    double prof_acc[32][4] = {};   // per profiling class (P_* below)
};

struct hicma_tlr_desc_s {
    hicma_tlr_ctx *ctx = nullptr;
    int N = 0, NB = 0, NT = 0, maxrank = 0, band = 1, slot_band = 1, band_alloc = 1;
    int ndim = 0;
    double *d_pts = nullptr;
    double *d_band = nullptr;
    double *d_lr = nullptr;
    long long nslots = 0;
    int *d_rank = nullptr;
    std::vector<int> h_rank;
    // rank history of the last factorization (the reference's dcRank record,
    // HiCMA_dpotrf_L_2flow.jdf:353-361,683-691,1101-1106): per off-band tile the
    // rank it entered with and the smallest / largest rank it held; -1 elsewhere
    std::vector<int> rk_init, rk_min, rk_max;
    // copy-out armed by hicma_tlr_store_stream for the next factorization
    double *strm_buf = nullptr;
    size_t strm_cap = 0, strm_off = 0;
    bool strm_over = false;
    double *d_linv = nullptr;
    bool factored = false;
    double stats[16] = {0};
    double async_acc = 0;
    int async_fixed = 0, async_maxrank = 0;

    double *dense(int m, int n) const {
        return d_band + ((size_t)m * band_alloc + (size_t)(m - n)) * (size_t)NB * NB;
    }
    long long slot(int m, int n) const {
        const long long mm = m - slot_band;
        return mm * (mm + 1) / 2 + n;
    }
    double *U(int m, int n) const { return d_lr + (size_t)slot(m, n) * 2 * (size_t)NB * maxrank; }
    double *V(int m, int n) const { return U(m, n) + (size_t)NB * maxrank; }
    double *linv(int k) const { return d_linv + (size_t)k * NB * NB; }
    bool is_dense(int m, int n) const { return m - n < band; }
    int rank(int m, int n) const { return h_rank[(size_t)n * NT + m]; }
};

namespace {

size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

int ctx_sync(hicma_tlr_ctx *c) {
    CUDA_TRY(cudaStreamSynchronize(c->stream_hi));
    CUDA_TRY(cudaStreamSynchronize(c->stream_side));
    CUDA_TRY(cudaStreamSynchronize(c->stream_copy));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->stage_off = 0;
    return 0;
}

void ws_reset(hicma_tlr_ctx *c) { c->ar->off = 0; }

// Host <-> device transfers and clears, ordered on the context stream and
// complete on return.  (cudaMemcpy and cudaMemset run on the legacy default
// stream, which the context's non-blocking streams do not wait for, and a
// cudaMemcpy from pageable host memory may return before its data has
// landed: a kernel launched next on the context stream could then read the
// old contents, or have its results overwritten by the late copy.)
cudaError_t xfer(hicma_tlr_ctx *c, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, c->stream);
    return e == cudaSuccess ? cudaStreamSynchronize(c->stream) : e;
}
cudaError_t xclear(hicma_tlr_ctx *c, void *dst, size_t bytes) {
    cudaError_t e = cudaMemsetAsync(dst, 0, bytes, c->stream);
    return e == cudaSuccess ? cudaStreamSynchronize(c->stream) : e;
}

// After a synchronisation: report (and clear) a bounded device wait that gave up.
int check_timeout(hicma_tlr_ctx *c) {
    int f = 0;
    CUDA_TRY(xfer(c, &f, c->d_flags + 3, sizeof(int), cudaMemcpyDeviceToHost));
    if (f) {
        CUDA_TRY(xclear(c, c->d_flags + 3, sizeof(int)));
        set_err("a bounded device wait gave up (tile POTRF task queue)");
        return HICMA_TLR_ERR_TIMEOUT;
    }
    return 0;
}
template <class T>
T *ws_alloc(hicma_tlr_ctx *c, size_t n) {
    const size_t bytes = align_up(n * sizeof(T) + 1);
    if (c->ar->off + bytes > c->ar->bytes) return nullptr;
    T *p = (T *)(c->ar->base + c->ar->off);
    c->ar->off += bytes;
    return p;
}
size_t ws_free(hicma_tlr_ctx *c) { return c->ar->bytes - c->ar->off; }

// Switch the helpers to the critical-path stream/arena and back.
struct OnHi {
    hicma_tlr_ctx *c;
    explicit OnHi(hicma_tlr_ctx *ctx) : c(ctx) { c->cur = c->stream_hi; c->ar = &c->hi_ar; }
    ~OnHi() { c->cur = c->stream; c->ar = &c->main_ar; }
};

template <class T>
T *stage(hicma_tlr_ctx *c, const T *src, size_t n) {
    const size_t raw = n * sizeof(T);
    const size_t bytes = align_up(raw + 1);
    if (bytes > c->stage_bytes) return nullptr;
    if (c->stage_off + bytes > c->stage_bytes) {
        if (cudaStreamSynchronize(c->stream_hi) != cudaSuccess) return nullptr;
        if (cudaStreamSynchronize(c->stream_side) != cudaSuccess) return nullptr;
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) return nullptr;
        c->stage_off = 0;
    }
    std::memcpy(c->h_stage + c->stage_off, src, raw);
    if (cudaMemcpyAsync(c->d_stage + c->stage_off, c->h_stage + c->stage_off, raw,
                        cudaMemcpyHostToDevice, c->cur) != cudaSuccess)
        return nullptr;
    T *d = (T *)(c->d_stage + c->stage_off);
    c->stage_off += bytes;
    return d;
}

enum {
    P_GEMM = 0, P_QR, P_QAPPLY, P_CORE, P_POTRF, P_COV, P_COPY, P_OTHER, P_PROJ,
    // batched DMMA GEMMs by call site (P_GEMM: recompression outputs and the rest)
    P_GEMM_Y, P_GEMM_TRSM, P_GEMM_SYRK, P_GEMM_DENSE, P_GEMM_GEN,
    P_GRAM,   // split-K inner products B_V^T A_V of the recompressions
    P_CHOLQR,     // QR factors by randomized CholeskyQR
    P_NCLASS
};
static_assert(P_NCLASS <= 32, "two device counters per class in d_profacc");

cudaEvent_t pool_event(hicma_tlr_ctx *c) {
    if (!c->ev_pool.empty()) {
        cudaEvent_t e = c->ev_pool.back();
        c->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Records the device time of the launches issued in its scope (profiling on).
struct Prof {
    hicma_tlr_ctx *c;
    int cls;
    double flops, bytes;
    cudaEvent_t a = nullptr;
    Prof(hicma_tlr_ctx *ctx, int k, double f, double b) : c(ctx), cls(k), flops(f), bytes(b) {
        if (c->prof) {
            a = pool_event(c);
            cudaEventRecord(a, c->cur);
        }
    }
    ~Prof() {
        if (a) {
            cudaEvent_t b2 = pool_event(c);
            cudaEventRecord(b2, c->cur);
            c->prof_recs.push_back({cls, a, b2, flops, bytes});
        }
    }
};

void prof_flush(hicma_tlr_ctx *c) {
    for (auto &r : c->prof_recs) {
        float ms = 0.f;
        if (cudaEventSynchronize(r.b) == cudaSuccess && cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
            c->prof_acc[r.cls][0] += 1;
            c->prof_acc[r.cls][1] += ms * 1e-3;
            c->prof_acc[r.cls][2] += r.flops;
            c->prof_acc[r.cls][3] += r.bytes;
        }
        c->ev_pool.push_back(r.a);
        c->ev_pool.push_back(r.b);
    }
    c->prof_recs.clear();
}

int check_launch(hicma_tlr_ctx *c) {
    c->launches++;
    CUDA_TRY(cudaGetLastError());
    return 0;
}

// Operand extents of every task of a launch (bounds-checked builds; no-ops
// otherwise).  Device-side counts (rank read at run time) are bounded by the
// host-side capacities checked here.
#ifdef TLR_BOUNDS_CHECK
#define BC(ptr, bytes, what, idx)                                                                      \
    do {                                                                                               \
        if (!bc_inside((ptr), (bytes))) {                                                              \
            set_err("bounds check: %s of task %zu: [%p, +%zu B) lies outside every live allocation", \
                    (what), (size_t)(idx), (const void *)(ptr), (size_t)(bytes));                      \
            return HICMA_TLR_ERR_ARG;                                                                  \
        }                                                                                              \
    } while (0)
#endif

static int bc_gemms(const std::vector<GemmTask> &v) {
#ifdef TLR_BOUNDS_CHECK
    for (size_t i = 0; i < v.size(); ++i) {
        const GemmTask &t = v[i];
        // a device-side column count is a rank (or 0): never above the inner dimension
        const int n = t.n_dev ? std::min(t.n, std::max(t.k, 0)) : t.n;
        if (t.m <= 0 || n <= 0) continue;
        BC(t.A, t.opA ? bc_span(t.k, t.m, t.lda) : bc_span(t.m, t.k, t.lda), "gemm A", i);
        BC(t.B, t.opB ? bc_span(n, t.k, t.ldb) : bc_span(t.k, n, t.ldb), "gemm B", i);
        BC(t.C, bc_span(t.m, n, t.ldc), "gemm C", i);
        if (t.n_dev) BC(t.n_dev, sizeof(int), "gemm device count", i);
    }
#else
    (void)v;
#endif
    return 0;
}

static int bc_copies(const std::vector<CopyTask> &v) {
#ifdef TLR_BOUNDS_CHECK
    for (size_t i = 0; i < v.size(); ++i) {
        const CopyTask &t = v[i];
        BC(t.src, bc_span(t.rows, t.cols, t.lds), "copy source", i);
        BC(t.dst, bc_span(t.rows, t.cols, t.ldd), "copy destination", i);
    }
#else
    (void)v;
#endif
    return 0;
}

static int bc_qr(const std::vector<QRTask> &v, int m_max) {
#ifdef TLR_BOUNDS_CHECK
    const int pb = qr_panel_width(m_max);
    for (size_t i = 0; i < v.size(); ++i) {
        const QRTask &t = v[i];
        if (t.K <= 0) continue;
        BC(t.X, bc_span(t.m, t.K, t.ld), "qr X", i);
        BC(t.tau, bc_span(t.K, 1, t.K), "qr tau", i);
        BC(t.T, (size_t)((t.K + pb - 1) / pb) * pb * pb * sizeof(double), "qr T", i);
    }
#else
    (void)v; (void)m_max;
#endif
    return 0;
}

static int bc_qapply(const std::vector<QApplyTask> &v, int m_max) {
#ifdef TLR_BOUNDS_CHECK
    const int pb = qr_panel_width(m_max);
    for (size_t i = 0; i < v.size(); ++i) {
        const QApplyTask &t = v[i];
        // columns read and written: up to the device rank, checked up to min(r_cap, K)
        const int r = std::min(t.r_cap, t.K);
        if (r <= 0) continue;
        BC(t.X, bc_span(t.m, t.K, t.ld), "qapply X", i);
        BC(t.T, (size_t)((t.K + pb - 1) / pb) * pb * pb * sizeof(double), "qapply T", i);
        BC(t.S, bc_span(t.K, r, t.lds), "qapply S", i);
        BC(t.out, bc_span(t.m, r, t.ldo), "qapply out", i);
        if (t.r_dev) BC(t.r_dev, sizeof(int), "qapply rank", i);
    }
#else
    (void)v; (void)m_max;
#endif
    return 0;
}

static int bc_cores(const std::vector<CoreTask> &v) {
#ifdef TLR_BOUNDS_CHECK
    for (size_t i = 0; i < v.size(); ++i) {
        const CoreTask &t = v[i];
        if (t.K <= 0) continue;
        if (t.RU) BC(t.RU, bc_span(t.K, t.K, t.ldru), "core RU", i);
        BC(t.RV, bc_span(t.K, t.K, t.ldrv), "core RV", i);
        BC(t.SU, bc_span(t.K, t.K, t.K), "core SU", i);
        if (t.RUc) BC(t.RUc, bc_span(t.K, t.K, t.K), "core RU copy", i);
        if (t.work) BC(t.work, core_work_doubles(t.K) * sizeof(double), "core scratch", i);
        if (t.rank_out) BC(t.rank_out, sizeof(int), "core rank", i);
        if (t.rank_task) BC(t.rank_task, sizeof(int), "core task rank", i);
    }
#else
    (void)v;
#endif
    return 0;
}

static int bc_cov(const CovParams &p, const std::vector<CovTask> &v) {
#ifdef TLR_BOUNDS_CHECK
    BC(p.pts, bc_span(p.N, p.ndim, p.N), "points", 0);
    for (size_t i = 0; i < v.size(); ++i) {
        const CovTask &t = v[i];
        BC(t.out, bc_span(t.nr, t.nc, t.ld), "covariance tile", i);
        if (t.r0 < 0 || t.c0 < 0 || t.r0 + t.nr > p.N || t.c0 + t.nc > p.N) {
            set_err("bounds check: covariance tile %zu reads rows/cols outside 0..%d", i, p.N);
            return HICMA_TLR_ERR_ARG;
        }
    }
#else
    (void)p; (void)v;
#endif
    return 0;
}

static int bc_recompress_parts(const std::vector<SelTask> &sels, const std::vector<GramTask> &grams,
                               const std::vector<ProjTask> &projs, const std::vector<AssembleTask> &asm_) {
#ifdef TLR_BOUNDS_CHECK
    for (size_t i = 0; i < sels.size(); ++i) {
        BC(sels[i].na, sizeof(double), "precision norm a", i);
        BC(sels[i].nb, sizeof(double), "precision norm b", i);
        BC(sels[i].sel64, sizeof(int), "precision count 64", i);
        BC(sels[i].sel32, sizeof(int), "precision count 32", i);
    }
    for (size_t i = 0; i < grams.size(); ++i) {
        const GramTask &t = grams[i];
        BC(t.C, bc_span(t.nb, t.rc, t.nb), "gram C", i);
        BC(t.W, bc_span(t.nb, t.ra, t.nb), "gram W", i);
        BC(t.P, bc_span(t.rc, t.ra, t.rc), "gram P", i);
    }
    for (size_t i = 0; i < projs.size(); ++i) {
        const ProjTask &t = projs[i];
        BC(t.C, bc_span(t.nb, t.rc, t.nb), "projection C", i);
        BC(t.W, bc_span(t.nb, t.ra, t.nb), "projection W", i);
        BC(t.P, bc_span(t.rc, t.ra, t.rc), "projection P", i);
        BC(t.P2, bc_span(t.rc, t.ra, t.rc), "projection P2", i);
    }
    for (size_t i = 0; i < asm_.size(); ++i) {
        const AssembleTask &t = asm_[i];
        const int K = t.rc + t.ra;
        BC(t.Pu, bc_span(t.rc, t.ra, t.rc), "assemble Pu", i);
        BC(t.Wu, bc_span(t.ra, t.ra, t.nb), "assemble Wu", i);
        BC(t.RU, bc_span(K, K, K), "assemble RU", i);
    }
#else
    (void)sels; (void)grams; (void)projs; (void)asm_;
#endif
    return 0;
}

static int bc_norms(const std::vector<NormTask> &v) {
#ifdef TLR_BOUNDS_CHECK
    for (size_t i = 0; i < v.size(); ++i) {
        BC(v[i].X, bc_span(v[i].rows, v[i].cols, v[i].ld), "norm X", i);
        BC(v[i].out, sizeof(double), "norm out", i);
    }
#else
    (void)v;
#endif
    return 0;
}

int run_qr(hicma_tlr_ctx *c, std::vector<QRTask> &v, int m_max) {
    if (v.empty()) return 0;
    TRY(bc_qr(v, m_max));
    QRTask *d = stage(c, v.data(), v.size());
    if (!d) { set_err("staging failed"); return HICMA_TLR_ERR_CUDA; }
    double fl = 0, by = 0;
    for (auto &t : v) {
        fl += 2.0 * t.m * (double)t.K * t.K - 2.0 / 3.0 * (double)t.K * t.K * t.K;
        by += 16.0 * t.m * (double)t.K;
    }
    {
        Prof pf(c, P_QR, fl, by);
        launch_qr_batched(d, (int)v.size(), m_max, c->cur);
    }
    v.clear();
    return check_launch(c);
}

int run_rcholqr(hicma_tlr_ctx *c, std::vector<CQTask> &v, int kmax) {
    if (v.empty()) return 0;
#ifdef TLR_BOUNDS_CHECK
    for (size_t i = 0; i < v.size(); ++i) {
        const CQTask &t = v[i];
        const int K = t.k1 + t.k2;
        if (t.k1) BC(t.X1, bc_span(t.nb, t.k1, t.ld1), "cholqr X1", i);
        if (t.k2) BC(t.X2, bc_span(t.nb, t.k2, t.ld2), "cholqr X2", i);
        if (t.Q || t.Rinv) BC(t.Z, bc_span(t.nb, K, t.nb), "cholqr Y", i);
        BC(t.R, bc_span(K, K, K), "cholqr R", i);
        if (t.Q) BC(t.Q, bc_span(t.nb, K, t.nb), "cholqr Q", i);
        if (t.Rinv) BC(t.Rinv, bc_span(K, K, K), "cholqr R3 inverse", i);
    }
#endif
    (void)kmax;
    // all tasks form Q or none does (the kernel is instantiated both ways)
    const bool form_q = v[0].Q != nullptr;
    for (auto &t : v)
        if ((t.Q != nullptr) != form_q || (form_q && t.Rinv)) {
            set_err("CholeskyQR batch mixes tasks that form Q with tasks that do not");
            return HICMA_TLR_ERR_ARG;
        }
    // one launch per width bucket (the kernel is instantiated per bucket)
    std::vector<CQTask> b;
    int lo = 0;
    while (lo < rcholqr_kmax()) {
        const int hi = rcholqr_bucket(lo + 1);
        b.clear();
        for (auto &t : v)
            if (t.k1 + t.k2 > lo && t.k1 + t.k2 <= hi) b.push_back(t);
        lo = hi;
        if (b.empty()) continue;
        CQTask *d = stage(c, b.data(), b.size());
        if (!d) { set_err("staging failed"); return HICMA_TLR_ERR_CUDA; }
        double fl = 0, by = 0;
        for (auto &t : b) {
            // the sketch (nb K FMAs); shifted CholeskyQR3 of the 256 sketch rows (three Gram
            // products, K^2 m each, symmetric; two row substitutions, K^2 m / 2 FMAs each); one
            // pass over the rows (substitution and Gram product), and the Q substitution when Q
            // is formed
            const double K = t.k1 + t.k2, m = 256.0;
            fl += 2.0 * t.nb * K + 5.0 * m * K * K + (t.Q ? 3.0 : 2.0) * t.nb * K * K;
            // X read twice; Y written when kept; Y read and Q written when Q is formed
            by += 8.0 * t.nb * K * (2.0 + (t.Q || t.Rinv ? 1.0 : 0.0) + (t.Q ? 2.0 : 0.0));
        }
        {
            Prof pf(c, P_CHOLQR, fl, by);
            launch_rcholqr_batched(d, (int)b.size(), hi, form_q, c->d_flags + 5, c->cur);
        }
        TRY(check_launch(c));
    }
    v.clear();
    return 0;
}

int run_qapply(hicma_tlr_ctx *c, std::vector<QApplyTask> &v, int m_max) {
    if (v.empty()) return 0;
    TRY(bc_qapply(v, m_max));
    QApplyTask *d = stage(c, v.data(), v.size());
    if (!d) { set_err("staging failed"); return HICMA_TLR_ERR_CUDA; }
    double by = 0;
    for (auto &t : v) by += 8.0 * t.m * (double)t.K;
    {
        Prof pf(c, P_QAPPLY, 0, by);
        launch_qapply_batched(d, (int)v.size(), m_max, c->cur);
    }
    v.clear();
    return check_launch(c);
}

int run_core(hicma_tlr_ctx *c, std::vector<CoreTask> &v, int kmax, const CoreParams &cp) {
    if (v.empty()) return 0;
    TRY(bc_cores(v));
    CoreTask *d = stage(c, v.data(), v.size());
    if (!d) { set_err("staging failed"); return HICMA_TLR_ERR_CUDA; }
    {
        Prof pf(c, P_CORE, 0, 0);
        launch_core_svd_batched(d, (int)v.size(), std::max(kmax, 1), cp, c->cur);
    }
    v.clear();
    return check_launch(c);
}

int run_gemms_narrow(hicma_tlr_ctx *c, std::vector<GemmTask> &v, int cls);

// Appends the group table to the tile prefix sums `off` (ntasks + 1 entries):
// entry g names the task that holds tile GEMM_GROUP g.
void gemm_groups(std::vector<int> &off) {
    const int ntasks = (int)off.size() - 1, total = off[ntasks];
    const int ngrp = (total + GEMM_GROUP - 1) / GEMM_GROUP;
    off.reserve(off.size() + ngrp);
    int task = 0;
    for (int g = 0; g < ngrp; ++g) {
        const int tile = g * GEMM_GROUP;
        while (task + 1 < ntasks && off[task + 1] <= tile) ++task;
        off.push_back(task);
    }
}

// Algorithmic flops and bytes of a GEMM batch known on the host; tasks whose n
// is read on the device (n_dev, a rank decided by an earlier kernel) are left
// out here and counted on the device when profiling (returns whether any).
bool gemm_work(const std::vector<GemmTask> &v, double &fl, double &by) {
    bool ndev = false;
    for (auto &t : v) {
        if (t.n_dev) {
            ndev = true;
            continue;
        }
        // a triangular operand (L^-1 of a tile) holds half the products: m n k
        fl += (t.tri ? 1.0 : 2.0) * t.m * (double)t.n * t.k;
        by += 8.0 * ((double)t.m * t.k + (double)t.k * t.n + (t.beta != 0.0 ? 2.0 : 1.0) * t.m * (double)t.n);
    }
    return ndev;
}

int run_gemms(hicma_tlr_ctx *c, std::vector<GemmTask> &v, bool fp32 = false, int cls = 0) {
    if (v.empty()) return 0;
    TRY(bc_gemms(v));
    if (!fp32) {
        // outputs a rank wide go to the 128 x 32 tile variant
        std::vector<GemmTask> narrow, wide;
        for (auto &t : v) ((t.n <= c->gemm_narrow_n || t.n_dev) && !t.lower ? narrow : wide).push_back(t);
        if (!narrow.empty()) {
            TRY(run_gemms_narrow(c, narrow, cls));
            if (wide.empty()) { v.clear(); return 0; }
            v.swap(wide);
        }
    }
    std::vector<int> off(v.size() + 1);
    off[0] = 0;
    for (size_t i = 0; i < v.size(); ++i) off[i + 1] = off[i] + gemm_tiles(v[i]);
    if (off.back() == 0) { v.clear(); return 0; }
    gemm_groups(off);
    GemmTask *dt = stage(c, v.data(), v.size());
    int *doff = stage(c, off.data(), off.size());
    if (!dt || !doff) { set_err("task staging failed"); return HICMA_TLR_ERR_CUDA; }
    double fl = 0, by = 0;
    bool ndev = gemm_work(v, fl, by);
    {
        Prof pf(c, cls, fl, by);
        launch_gemm_batched(dt, doff, (int)v.size(), off[v.size()], c->cur, fp32);
    }
    if (ndev && c->prof) launch_gemm_devcount(dt, (int)v.size(), c->d_profacc + 2 * cls, c->cur);
    v.clear();
    return check_launch(c);
}

int run_gemms_narrow(hicma_tlr_ctx *c, std::vector<GemmTask> &v, int cls) {
    std::vector<int> off(v.size() + 1);
    off[0] = 0;
    for (size_t i = 0; i < v.size(); ++i) {
        GemmTask &t = v[i];
        t.tiles_m = (t.m + GEMM_NARROW_M - 1) / GEMM_NARROW_M;
        off[i + 1] = off[i] + t.tiles_m * ((t.n + GEMM_NARROW_N - 1) / GEMM_NARROW_N);
    }
    if (off.back() == 0) { v.clear(); return 0; }
    gemm_groups(off);
    GemmTask *dt = stage(c, v.data(), v.size());
    int *doff = stage(c, off.data(), off.size());
    if (!dt || !doff) { set_err("task staging failed"); return HICMA_TLR_ERR_CUDA; }
    double fl = 0, by = 0;
    bool ndev = gemm_work(v, fl, by);
    {
        Prof pf(c, cls, fl, by);
        launch_gemm_batched_narrow(dt, doff, (int)v.size(), off[v.size()], c->cur);
    }
    if (ndev && c->prof) launch_gemm_devcount(dt, (int)v.size(), c->d_profacc + 2 * cls, c->cur);
    v.clear();
    return check_launch(c);
}

// Batched inner products P = C^T W of nb-long columns (split-K DMMA, one CTA
// per product; k_gram_batched).
int run_grams(hicma_tlr_ctx *c, std::vector<GramTask> &v, int cls) {
    if (v.empty()) return 0;
#ifdef TLR_BOUNDS_CHECK
    for (size_t i = 0; i < v.size(); ++i) {
        const GramTask &t = v[i];
        BC(t.C, bc_span(t.nb, t.rc, t.nb), "gram C", i);
        BC(t.W, bc_span(t.nb, t.ra, t.nb), "gram W", i);
        BC(t.P, bc_span(t.rc, t.ra, t.rc), "gram P", i);
    }
#endif
    double fl = 0.0, by = 0.0;
    for (auto &g : v) {
        fl += 2.0 * g.nb * (double)g.rc * g.ra;
        by += 8.0 * g.nb * (double)(g.rc + g.ra);
    }
    GramTask *d = stage(c, v.data(), v.size());
    if (!d) { set_err("staging failed"); return HICMA_TLR_ERR_CUDA; }
    {
        Prof pf(c, cls, fl, by);
        launch_gram_batched(d, (int)v.size(), c->cur);
    }
    v.clear();
    return check_launch(c);
}

int run_copies(hicma_tlr_ctx *c, std::vector<CopyTask> &v) {
    if (v.empty()) return 0;
    TRY(bc_copies(v));
    int maxc = 0;
    for (auto &t : v) maxc = std::max(maxc, t.cols);
    CopyTask *dt = stage(c, v.data(), v.size());
    if (!dt) { set_err("task staging failed"); return HICMA_TLR_ERR_CUDA; }
    double by = 0;
    for (auto &t : v) by += 16.0 * t.rows * (double)t.cols;
    Prof pf(c, P_COPY, 0, by);
    launch_copy_batched(dt, (int)v.size(), maxc, c->cur);
    v.clear();
    return check_launch(c);
}

CopyTask make_copy(const double *src, int lds, double *dst, int ldd, int rows, int cols, double alpha = 1.0,
                   double beta = 0.0) {
    CopyTask t;
    t.src = src; t.dst = dst; t.lds = lds; t.ldd = ldd; t.rows = rows; t.cols = cols; t.alpha = alpha;
    t.beta = beta;
    return t;
}

// ----------------------------------------------------------- tile POTRF ----
// Blocked right-looking Cholesky of an n x n tile (64-column panels): the
// diagonal block is factored and inverted in one CTA, the panel below is
// multiplied by the block inverse, the trailing matrix gets a lower DMMA
// SYRK.  With Linv, L^-1 is then assembled block row by block row.
int potrf_tile(hicma_tlr_ctx *c, double *A, int n, int lda, double *Linv, int ldl, int *d_info,
               int info_base) {
#ifdef TLR_BOUNDS_CHECK
    BC(A, bc_span(n, n, lda), "potrf tile", 0);
    if (Linv) BC(Linv, bc_span(n, n, ldl), "potrf inverse", 0);
    BC(d_info, sizeof(int), "potrf info", 0);
#endif
    const int DBK = 64;
    cudaStream_t st = c->cur;
    const size_t mark = c->ar->off;
    Prof pf(c, P_POTRF, (double)n * n * n / 3.0 * (Linv ? 2.0 : 1.0), 8.0 * n * (double)n * (Linv ? 3.0 : 2.0));
    if (n <= potrf_tile_max_n()) {
        // one persistent launch: block Cholesky and block inverse as a task queue
        const int nblk = (n + DBK - 1) / DBK;
        int *cnt = ws_alloc<int>(c, potrf_tile_scratch_ints(n));
        double *D = Linv ? nullptr : ws_alloc<double>(c, (size_t)nblk * DBK * DBK);
        if (!cnt || (!Linv && !D)) { set_err("workspace exhausted (potrf)"); return HICMA_TLR_ERR_OOM; }
        if (Linv) CUDA_TRY(cudaMemset2DAsync(Linv, (size_t)ldl * sizeof(double), 0, sizeof(double) * n, n, st));
        const int grid = c->potrf_grid > 0 ? c->potrf_grid : c->nsm;
        if (launch_potrf_tile(A, lda, n, Linv, ldl, D, cnt, d_info, info_base, c->d_flags + 3, grid, st)) {
            set_err("tile POTRF launch failed: %s", cudaGetErrorString(cudaGetLastError()));
            return HICMA_TLR_ERR_CUDA;
        }
        TRY(check_launch(c));
        launch_zero_upper(A, n, lda, st);
        TRY(check_launch(c));
        c->ar->off = mark;
        return 0;
    }
    double *dscr = nullptr;
    if (!Linv) {
        dscr = ws_alloc<double>(c, DBK * DBK);
        if (!dscr) { set_err("workspace exhausted (potrf)"); return HICMA_TLR_ERR_OOM; }
    } else {
        CUDA_TRY(cudaMemset2DAsync(Linv, (size_t)ldl * sizeof(double), 0, sizeof(double) * n, n, st));
    }
    for (int j = 0; j < n; j += DBK) {
        const int jb = std::min(DBK, n - j);
        double *Dinv = Linv ? Linv + j + (size_t)j * ldl : dscr;
        const int ldd = Linv ? ldl : DBK;
        launch_potrf_diag(A + j + (size_t)j * lda, lda, jb, Dinv, ldd, d_info, info_base + j, st);
        TRY(check_launch(c));
        if (j + jb < n) {
            const int rows = n - j - jb;
            double *Pn = A + (j + jb) + (size_t)j * lda;
            launch_gemm_single(make_gemm(0, 1, rows, jb, jb, 1.0, Pn, lda, Dinv, ldd, 0.0, Pn, lda), st);
            TRY(check_launch(c));
            launch_gemm_single(make_gemm(0, 1, rows, rows, jb, -1.0, Pn, lda, Pn, lda, 1.0,
                                         A + (j + jb) + (size_t)(j + jb) * lda, lda, 1),
                               st);
            TRY(check_launch(c));
        }
    }
    launch_zero_upper(A, n, lda, st);
    TRY(check_launch(c));
    if (Linv && n > DBK) {
        double *tmp = ws_alloc<double>(c, (size_t)DBK * n);
        if (!tmp) { set_err("workspace exhausted (trtri)"); return HICMA_TLR_ERR_OOM; }
        for (int i0 = DBK; i0 < n; i0 += DBK) {
            const int ib = std::min(DBK, n - i0);
            launch_gemm_single(make_gemm(0, 0, ib, i0, i0, 1.0, A + i0, lda, Linv, ldl, 0.0, tmp, ib), st);
            TRY(check_launch(c));
            launch_gemm_single(make_gemm(0, 0, ib, i0, ib, -1.0, Linv + i0 + (size_t)i0 * ldl, ldl, tmp, ib,
                                         0.0, Linv + i0, ldl),
                               st);
            TRY(check_launch(c));
        }
    }
    c->ar->off = mark;
    return 0;
}

// ----------------------------------------------------- recompression -------
// One low-rank-C GEMM update (HCORE_dgemm_qr_svd{,_b_dense} + ormqr):
// C = [Cu Au] [Cv -Y]^T, Y = Bu (Bv^T Av) (B low rank) or Y = B Av (B dense).
struct RecompTask {
    const double *Cu, *Cv;
    int rc;
    const double *Au, *Av;
    int ra;
    const double *Bu, *Bv;   // Bv == nullptr: B dense in Bu (NB x NB)
    int rb;
    double *outU, *outV;
    int *rank_dst;
    // squared Frobenius norms of the A and B factor tiles (device); null: FP64
    const double *na = nullptr, *nb = nullptr;
};

// Workspace of one low-rank update (K = rc + ra).
size_t recomp_ws_bytes(int nb, const RecompTask &t) {
    const int K = t.rc + t.ra, rc = t.rc, ra = t.ra;
    const int pb = qr_panel_width(nb);
    const size_t npk = (size_t)(K + pb - 1) / pb + 1, npa = (size_t)(ra + pb - 1) / pb + 1;
    auto A = [](size_t n) { return align_up(sizeof(double) * n + 1); };
    size_t b = 0;
    b += A((size_t)nb * K) * 3;                          // Us = [Cu | Wu], Vs = [Cv | -Y], Vk
    b += A(ra) + A(K) + A(npa * pb * pb) + A(npk * pb * pb);  // tau, T factors of Wu and Vs
    b += A((size_t)rc * ra) * 2;                         // Pu, Pu2
    b += A((size_t)nb * ra) + A((size_t)ra * ra);        // Q and R of the residual (CholeskyQR form)
    b += A((size_t)K * K) * 6;                           // RU, SU, T1, RV, R3^-1 and R3^-1 U_r
    if (K > core_smem_kmax()) b += A(core_work_doubles(K));
    if (t.Bv) b += A((size_t)t.rb * t.ra);
    return b + 1024;
}

// Core-SVD launches bucketed by K so that small cores run several CTAs per SM.
int run_core_buckets(hicma_tlr_ctx *c, std::vector<CoreTask> &cores, const CoreParams &cp) {
    static const int edges[] = {32, 64, 96, 128, 160, 1 << 30};
    std::vector<CoreTask> bucket;
    int lo = -1;
    for (int e : edges) {
        int kmax = 0;
        for (auto &t : cores)
            if (t.K > lo && t.K <= e) { bucket.push_back(t); kmax = std::max(kmax, t.K); }
        if (!bucket.empty()) TRY(run_core(c, bucket, kmax, cp));
        lo = e;
    }
    cores.clear();
    return 0;
}

// Recompression of a batch of low-rank updates C = [Cu Au][Cv -Y]^T.
// The old U is orthonormal, so on that side only the new columns need an
// orthogonal factorisation: Au is projected twice against Cu (block classical
// Gram-Schmidt, DMMA GEMMs) and the residual Wu (nb x ra) gets a Householder
// QR, giving R_U = [[I, Pu], [0, R(Wu)]].  The old V = V Sigma is orthogonal
// only up to the core solver's tolerance relative to its largest singular
// value, which is not enough to project its weak columns, so [Cv, -Y] gets a
// full Householder QR for R_V.  The core M = R_U R_V^T is decomposed and
// truncated (core kernel), then new U = Cu U_top + Q(Wu) [U_bot; 0] and
// new V = [Cv, -Y] (R_U^T U_r).
// thr2 > 0 enables the precision policy: the products forming Y run in FP32
// for updates whose factor tiles satisfy ||A||_F^2 ||B||_F^2 <= thr2.
int run_recompress(hicma_tlr_ctx *c, int nb, std::vector<RecompTask> &tasks, double acc, int maxrank,
                   int fixed_rank, int *d_rank_task_base, double thr2) {
    if (tasks.empty()) return 0;
    const size_t mark = c->ar->off;
    size_t i0 = 0;
    while (i0 < tasks.size()) {
        c->ar->off = mark;
        // common prefix (Y products, V-side stacks) on the bulk stream; then the
        // CholeskyQR chain (F) there and the Householder chain of the wide
        // updates (S) on the side stream, joined at the end of the chunk
        std::vector<CopyTask> copies, copiesS, keeps;
        std::vector<GemmTask> g1, g2, g1s, g2s, gTU, gU, g3, g4, gQS, gUS, g3S, g4S;
        std::vector<CQTask> cqS;   // QRs of the wide updates' projected residuals (Q formed)
        std::vector<CoreTask> coresS;
        std::vector<ProjTask> projs;
        std::vector<SelTask> sels;
        std::vector<GramTask> grams;
        int *sel = thr2 > 0.0 ? ws_alloc<int>(c, 2 * (tasks.size() - i0) + 2) : nullptr;
        std::vector<QRTask> qrs;
        std::vector<CQTask> vrs;
        std::vector<AssembleTask> asm_;
        std::vector<CoreTask> cores;
        std::vector<QApplyTask> apps;
        size_t i = i0;
        int *rank_task = d_rank_task_base;
        for (; i < tasks.size(); ++i) {
            const RecompTask &t = tasks[i];
            if (recomp_ws_bytes(nb, t) > ws_free(c)) {
                if (i == i0) { set_err("workspace too small for one recompression (K=%d)", t.rc + t.ra); return HICMA_TLR_ERR_OOM; }
                break;
            }
            const int rc = t.rc, ra = t.ra, K = rc + ra;
            CoreTask ct{};
            ct.rank_out = t.rank_dst;
            ct.rank_task = rank_task + (i - i0);
            ct.K = K;
            if (K == 0) { cores.push_back(ct); continue; }
            // Stacks up to rcholqr_kmax() columns: both QRs by randomized
            // CholeskyQR (U side [Cu, Au] read in place, Q_U = Y Rc^-1 kept
            // factored; V side R only); wider stacks: block Gram-Schmidt +
            // Householder on the U side and a Householder QR on the V side.
            const bool cq = c->cholqr && K <= rcholqr_kmax();
            double *Vs = ws_alloc<double>(c, (size_t)nb * K);
            double *Us = ws_alloc<double>(c, (size_t)nb * K);    // CholeskyQR path: Y of the U side
            double *RU = ws_alloc<double>(c, (size_t)K * K);
            double *SU = ws_alloc<double>(c, (size_t)K * K), *T1 = ws_alloc<double>(c, (size_t)K * K);
            double *work = K > core_smem_kmax() ? ws_alloc<double>(c, core_work_doubles(K)) : nullptr;
            double *Yb = Vs + (size_t)nb * rc;
            if (rc > 0) copies.push_back(make_copy(t.Cv, nb, Vs, nb, nb, rc));
            if (ra > 0) {
                if (t.Bv) {
                    double *P = ws_alloc<double>(c, (size_t)t.rb * ra);
                    GemmTask a1 = make_gemm(1, 0, t.rb, ra, nb, 1.0, t.Bv, nb, t.Av, nb, 0.0, P, t.rb);
                    GemmTask a2 = make_gemm(0, 0, nb, ra, t.rb, -1.0, t.Bu, nb, P, t.rb, 0.0, Yb, nb);
                    if (sel && t.na && t.nb) {
                        // both precisions are queued; the selector zeroes one column count
                        int *s64 = sel + 2 * (i - i0), *s32 = s64 + 1;
                        sels.push_back(SelTask{t.na, t.nb, s64, s32, ra});
                        a1.n_dev = s64; a2.n_dev = s64;
                        g1.push_back(a1); g2.push_back(a2);
                        a1.n_dev = s32; a2.n_dev = s32;
                        g1s.push_back(a1); g2s.push_back(a2);
                    } else {
                        grams.push_back(GramTask{t.Bv, t.Av, P, nb, t.rb, ra});
                        g2.push_back(a2);
                    }
                } else {
                    g1.push_back(make_gemm(0, 0, nb, ra, nb, -1.0, t.Bu, nb, t.Av, nb, 0.0, Yb, nb));
                }
            }
            double *Vsrc = Vs;
            double *RinvU = nullptr, *TU = nullptr;
            if (cq) {
                double *RV = ws_alloc<double>(c, (size_t)K * K);
                RinvU = ws_alloc<double>(c, (size_t)K * K);
                TU = ws_alloc<double>(c, (size_t)K * K);
                CQTask u{t.Cu, t.Au, Us, RU, nullptr, nb, rc, ra, nb, nb};
                u.Rinv = RinvU;          // Q_U = Y Rc^-1 formed inside the output product
                vrs.push_back(u);
                vrs.push_back(CQTask{Vs, nullptr, nullptr, RV, nullptr, nb, K, 0, nb, nb});
                ct.RV = RV; ct.ldrv = K;
            } else {
                double *Vk = ws_alloc<double>(c, (size_t)nb * K);
                const int pbw = qr_panel_width(nb);
                const size_t npk = (size_t)(K + pbw - 1) / pbw + 1, npa = (size_t)(ra + pbw - 1) / pbw + 1;
                double *tauU = ws_alloc<double>(c, ra), *tauV = ws_alloc<double>(c, K);
                double *TU = ws_alloc<double>(c, npa * pbw * pbw), *TV = ws_alloc<double>(c, npk * pbw * pbw);
                double *Pu = ws_alloc<double>(c, (size_t)rc * ra), *Pu2 = ws_alloc<double>(c, (size_t)rc * ra);
                double *Wu = Us + (size_t)nb * rc;
                // R of the projected residual Wu, as the assembly reads it (top ra x ra, ld)
                const double *Rw = Wu;
                int ldrw = nb;
                if (rc > 0) copiesS.push_back(make_copy(t.Cu, nb, Us, nb, nb, rc));
                if (ra > 0) {
                    copiesS.push_back(make_copy(t.Au, nb, Wu, nb, nb, ra));
                    // two rounds of projection of Au against the old orthonormal U
                    if (rc > 0) projs.push_back(ProjTask{Us, Wu, Pu, Pu2, nb, rc, ra});
                    if (c->cholqr && ra <= rcholqr_kmax()) {
                        // residual up to 64 columns: randomized CholeskyQR with Q formed,
                        // and the new U's Q(Wu) U_bot as one GEMM
                        double *Qw = ws_alloc<double>(c, (size_t)nb * ra);
                        double *Rq = ws_alloc<double>(c, (size_t)ra * ra);
                        cqS.push_back(CQTask{Wu, nullptr, Qw, Rq, Qw, nb, ra, 0, nb, nb});
                        Rw = Rq;
                        ldrw = ra;
                        GemmTask q = make_gemm(0, 0, nb, std::min(K, maxrank), ra, 1.0, Qw, nb, SU + rc, K, 0.0,
                                               t.outU, nb);
                        q.n_dev = ct.rank_task;
                        gQS.push_back(q);
                    } else {
                        qrs.push_back(QRTask{Wu, tauU, TU, nb, ra, nb});
                        apps.push_back(QApplyTask{Wu, TU, SU + rc, t.outU, ct.rank_task, nb, ra, nb, K, nb, maxrank});
                    }
                }
                keeps.push_back(make_copy(Vs, nb, Vk, nb, nb, K));
                qrs.push_back(QRTask{Vs, tauV, TV, nb, K, nb});
                asm_.push_back(AssembleTask{Pu, Rw, RU, rc, ra, ldrw});
                ct.RV = Vs; ct.ldrv = nb;
                Vsrc = Vk;
            }
            ct.RU = RU; ct.ldru = K;
            ct.SU = SU; ct.RUc = nullptr; ct.work = work;
            (cq ? cores : coresS).push_back(ct);
            if (cq) {
                // new U = Q_U U_r = X2 (R3^-1 U_r)
                // (the new rank, read on the device, is at most min(K, maxrank): the grid stops there)
                const int rcap = std::min(K, maxrank);
                GemmTask tu = make_gemm(0, 0, K, rcap, K, 1.0, RinvU, K, SU, K, 0.0, TU, K);
                tu.n_dev = ct.rank_task;
                gTU.push_back(tu);
                GemmTask u = make_gemm(0, 0, nb, rcap, K, 1.0, Us, nb, TU, K, 0.0, t.outU, nb);
                u.n_dev = ct.rank_task;
                gU.push_back(u);
            } else if (rc > 0) {
                // new U = Q(Wu) [U_bot; 0] + Cu U_top (beta 1 after the Q application when ra > 0)
                GemmTask u = make_gemm(0, 0, nb, std::min(K, maxrank), rc, 1.0, Us, nb, SU, K, ra > 0 ? 1.0 : 0.0, t.outU, nb);
                u.n_dev = ct.rank_task;
                gUS.push_back(u);
            }
            // V Sigma = M^T U = R_V (R_U^T U): new V = [Cv, -Y] (R_U^T U_r)
            GemmTask a = make_gemm(1, 0, K, K, K, 1.0, RU, K, SU, K, 0.0, T1, K);
            a.n_dev = ct.rank_task;
            (cq ? g3 : g3S).push_back(a);
            GemmTask b = make_gemm(0, 0, nb, std::min(K, maxrank), K, 1.0, Vsrc, nb, T1, K, 0.0, t.outV, nb);
            b.n_dev = ct.rank_task;
            (cq ? g4 : g4S).push_back(b);
        }
        TRY(bc_recompress_parts(sels, grams, projs, asm_));
        TRY(run_copies(c, copies));
        if (!sels.empty()) {
            SelTask *d = stage(c, sels.data(), sels.size());
            if (!d) { set_err("staging failed"); return HICMA_TLR_ERR_CUDA; }
            launch_precision_select(d, (int)sels.size(), thr2, c->d_flags + 4, c->cur);
            TRY(check_launch(c));
        }
        TRY(run_grams(c, grams, P_GRAM));
        TRY(run_gemms(c, g1, false, P_GEMM_Y));
        TRY(run_gemms(c, g1s, true, P_GEMM_Y));
        TRY(run_gemms(c, g2, false, P_GEMM_Y));
        TRY(run_gemms(c, g2s, true, P_GEMM_Y));
        const bool side = !coresS.empty();
        cudaStream_t bulk = c->cur;
        if (side) {
            CUDA_TRY(cudaEventRecord(c->ev_fork, bulk));
            CUDA_TRY(cudaStreamWaitEvent(c->stream_side, c->ev_fork, 0));
            c->cur = c->stream_side;
        }
        TRY(run_copies(c, copiesS));
        TRY(run_copies(c, keeps));
        if (!projs.empty()) {
            double fl = 0.0, by = 0.0;
            for (auto &p : projs) {
                fl += 8.0 * p.nb * p.rc * p.ra;             // two rounds of C^T W and C P
                by += 8.0 * p.nb * (p.rc + 2.0 * p.ra);     // C and W read once, W written once
            }
            Prof pr(c, P_PROJ, fl, by);
            ProjTask *d = stage(c, projs.data(), projs.size());
            if (!d) { set_err("staging failed"); return HICMA_TLR_ERR_CUDA; }
            launch_bcgs2(d, (int)projs.size(), c->cur);
            TRY(check_launch(c));
        }
        TRY(run_qr(c, qrs, nb));
        TRY(run_rcholqr(c, cqS, 0));
        if (!asm_.empty()) {
            AssembleTask *d = stage(c, asm_.data(), asm_.size());
            if (!d) { set_err("staging failed"); return HICMA_TLR_ERR_CUDA; }
            launch_assemble_r(d, (int)asm_.size(), c->cur);
            TRY(check_launch(c));
        }
        CoreParams cp{0, acc, maxrank, fixed_rank, nb, c->d_flags + 1, c->d_flags + 2};
        TRY(run_core_buckets(c, coresS, cp));
        TRY(run_qapply(c, apps, nb));
        TRY(run_gemms(c, gQS));   // Q(Wu) U_bot before gUS adds Cu U_top
        TRY(run_gemms(c, gUS));
        TRY(run_gemms(c, g3S));
        TRY(run_gemms(c, g4S));
        if (side) {
            CUDA_TRY(cudaEventRecord(c->ev_join, c->stream_side));
            c->cur = bulk;
        }
        TRY(run_rcholqr(c, vrs, 0));
        TRY(run_core_buckets(c, cores, cp));
        TRY(run_gemms(c, gTU));
        TRY(run_gemms(c, gU));
        TRY(run_gemms(c, g3));
        TRY(run_gemms(c, g4));
        // the next chunk reuses the workspace: it starts after both chains
        if (side) CUDA_TRY(cudaStreamWaitEvent(bulk, c->ev_join, 0));
        i0 = i;
    }
    c->ar->off = mark;
    return 0;
}

// --------------------------------------------------------- op_counts -------
// hicma_parsec/op_counts.h:10-72 restated with its unsigned arithmetic and
// float32 casts.
unsigned long op_counts(char op, unsigned long a, unsigned long b, unsigned long cc, unsigned long d) {
    unsigned long res = 0;
    if (op == 'q') {
        const unsigned long m = a, n = b;
        res = 2 * m * n * n - (unsigned long)((float)(2 * n * n * n) / 3.0f) + 2 * m * n +
              (unsigned long)((float)(17 * n) / 3.0f);
    } else if (op == 'c') {
        const unsigned long n = a;
        res = (unsigned long)((double)(n * n * n / 3) - (double)(n * n) / 2.0 + (double)(n / 6));
    } else if (op == 't') {
        const unsigned long m = a, n = b;
        res = (cc == 1) ? n * m * m : (cc == 2 ? m * n * n : 0);   // other sides: 0 (and a message there)
    } else if (op == 'm') {
        res = a * b * cc * 2;
    } else if (op == 's') {
        res = 22 * a * a * a;
    } else if (op == 'o') {
        const unsigned long m = a, n = b, k = cc;
        if (d == 1) res = 4 * n * m * k - 2 * n * k * k + 3 * n * k;
        else if (d == 2) res = 4 * n * m * k - 2 * m * k * k + 2 * m * k + n * k - k * k / 2 + k / 2;
    } else if (op == 'r') {
        const unsigned long m = a, n = b;
        res = (cc == 1) ? m * m * n : (cc == 2 ? m * n * n : 0);
    }
    return res;
}

unsigned long gemm_lr_ops(unsigned long nb, unsigned long ra, unsigned long rb, unsigned long rc_old,
                          unsigned long rc_new, bool b_dense) {
    const unsigned long ka = rc_old + ra;
    const unsigned long qra = op_counts('q', nb, ka, 0, 0);
    unsigned long qrb;
    if (b_dense) qrb = op_counts('q', nb, ka, 0, 0) + op_counts('m', ra, nb, nb, 0);
    else qrb = op_counts('m', ra, rb, nb, 0) + op_counts('m', ra, nb, rb, 0) + op_counts('q', nb, ka, 0, 0);
    unsigned long svd = op_counts('r', ka, ka, 2, 0) + op_counts('s', ka, 0, 0, 0) + ka * rc_new;
    const unsigned long newu = op_counts('o', nb, rc_new, ka, 1);
    const unsigned long newv = op_counts('o', rc_new, nb, ka, 2);
    return qra + qrb + svd + newu + newv;
}

// ---------------------------------------------------------------- points ---
uint64_t mix64h(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

int kind_ndim(int kind) {
    switch (kind) {
        case HICMA_TLR_KIND_ED_SIN_2D: return 2;
        case HICMA_TLR_KIND_SQEXP_2D: return 2;
        case HICMA_TLR_KIND_SQEXP_3D: return 3;
        case HICMA_TLR_KIND_EXP_3D: return 3;
        case HICMA_TLR_KIND_ED_SIN_3D: return 3;
        case HICMA_TLR_KIND_MD_VIRUS: return 3;
        case HICMA_TLR_KIND_MD_CUBE: return 3;
        default: return 0;
    }
}

// Columns of the per-row data a problem's kernel reads: the point coordinates,
// or for randtlr the basis [Q | Q diag(S)] of K = min(NB, RANDTLR_KMAX) columns.
int data_ndim(int kind, int NB) {
    if (kind == HICMA_TLR_KIND_RANDTLR) return 2 * std::min(NB, RANDTLR_KMAX);
    return kind_ndim(kind);
}

int grid_side(long long n, int ndim) {
    long long s = std::max(1LL, (long long)llround(std::pow((double)n, 1.0 / ndim)));
    auto pw = [&](long long x) { long long r = 1; for (int i = 0; i < ndim; ++i) r *= x; return r; };
    while (pw(s) < n) ++s;
    while (s > 1 && pw(s - 1) >= n) --s;
    return (int)s;
}

// Arguments of the mesh kinds (6, 7): a known basis function, a positive
// radius and an ordering this build has (0 none, 1 Morton; the reference
// names Hilbert ordering, hicma_parsec.c:82, but STARS-H does not provide it).
int rbf_args(const hicma_tlr_problem *prob) {
    if (prob->kind != HICMA_TLR_KIND_MD_VIRUS && prob->kind != HICMA_TLR_KIND_MD_CUBE) return 0;
    ARG_CHECK(prob->rbf_kernel >= HICMA_TLR_RBF_GAUSSIAN && prob->rbf_kernel <= HICMA_TLR_RBF_WENDLAND,
              "rbf_kernel must be 0 to 8 (-B)");
    ARG_CHECK(prob->radius > 0.0 && std::isfinite(prob->radius), "radius must be positive (-R)");
    ARG_CHECK(prob->order == 0 || prob->order == 1, "order must be 0 (none) or 1 (Morton) (-O)");
    return 0;
}

// 63-bit Morton code of a point of [0, 1)^3 at 21 bits per axis (x in the
// lowest bit of each triple).
uint64_t morton3(const double *x) {
    uint64_t code = 0;
    for (int a = 0; a < 3; ++a) {
        long long q = (long long)std::floor(x[a] * 2097152.0);
        q = std::min<long long>(std::max<long long>(q, 0), 2097151);
        for (int b = 0; b < 21; ++b) code |= (((uint64_t)q >> b) & 1ull) << (b * 3 + a);
    }
    return code;
}

// The first N of a point set c (AoS, 3 per point) after a stable Morton sort
// (order 1) or as given (order 0), written [3][N].  Coordinates are mapped
// to [0, 1)^3 through the set's bounding box for the code only.
void order_points(const std::vector<double> &c, int order, int N, double *points) {
    const size_t total = c.size() / 3;
    std::vector<size_t> idx(total);
    for (size_t i = 0; i < total; ++i) idx[i] = i;
    if (order == 1 && total > 0) {
        double lo[3], hi[3];
        for (int a = 0; a < 3; ++a) { lo[a] = c[a]; hi[a] = c[a]; }
        for (size_t i = 0; i < total; ++i)
            for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], c[3 * i + a]); hi[a] = std::max(hi[a], c[3 * i + a]); }
        std::vector<uint64_t> code(total);
        for (size_t i = 0; i < total; ++i) {
            double u[3];
            for (int a = 0; a < 3; ++a) {
                const double w = hi[a] - lo[a];
                u[a] = w > 0.0 ? (c[3 * i + a] - lo[a]) / w * (1.0 - 0x1.0p-30) : 0.0;
            }
            code[i] = morton3(u);
        }
        std::stable_sort(idx.begin(), idx.end(), [&](size_t x, size_t y) { return code[x] < code[y]; });
    }
    for (int i = 0; i < N; ++i)
        for (int a = 0; a < 3; ++a) points[(size_t)a * N + i] = c[3 * idx[(size_t)i] + a];
}

// md-3d-cube nodes: cell centres of an s^3 grid on the unit cube, s = ceil(cbrt(N)).
int cube_points(int N, int order, double *points) {
    const int s = grid_side(N, 3);
    const size_t total = (size_t)s * s * s;
    std::vector<double> c(3 * total);
    for (size_t i = 0; i < total; ++i) {
        const size_t g[3] = {i % s, (i / s) % s, i / ((size_t)s * s)};
        for (int a = 0; a < 3; ++a) c[3 * i + a] = ((double)g[a] + 0.5) / (double)s;
    }
    order_points(c, order, N, points);
    return 0;
}

}  // namespace

// ======================================================================
//                                C ABI
// ======================================================================
extern "C" {

int hicma_tlr_points(const hicma_tlr_problem *prob, int N, double *points) {
    ARG_CHECK(prob && points && N > 0, "hicma_tlr_points");
    const int ndim = kind_ndim(prob->kind);
    ARG_CHECK(ndim > 0, "unsupported problem kind");
    ARG_CHECK(prob->kind != HICMA_TLR_KIND_MD_VIRUS, "md-3d-virus points come from a mesh file (hicma_tlr_points_mesh)");
    if (prob->kind == HICMA_TLR_KIND_MD_CUBE) {
        TRY(rbf_args(prob));
        return cube_points(N, prob->order, points);
    }
    const int side = grid_side(N, ndim);
    long long total = 1;
    for (int a = 0; a < ndim; ++a) total *= side;
    std::vector<double> c((size_t)total * ndim);
    std::vector<uint64_t> code((size_t)total, 0);
    const uint64_t base = mix64h((uint64_t)prob->seed);
    for (long long idx = 0; idx < total; ++idx) {
        long long div = 1;
        for (int a = 0; a < ndim; ++a) {
            const long long cc = (idx / div) % side;
            div *= side;
            const uint64_t z = mix64h(base + (uint64_t)(idx * ndim + a));
            const double u = (double)(z >> 11) * 0x1.0p-53;
            const double x = (((double)cc + 0.1) + 0.8 * u) / (double)side;
            c[(size_t)idx * ndim + a] = x;
            long long q = (long long)std::floor(x * 2097152.0);
            if (q < 0) q = 0;
            if (q > 2097151) q = 2097151;
            for (int b = 0; b < 21; ++b)
                code[(size_t)idx] |= (((uint64_t)q >> b) & 1ull) << (b * ndim + a);
        }
    }
    std::vector<long long> order((size_t)total);
    for (long long i = 0; i < total; ++i) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](long long x, long long y) { return code[(size_t)x] < code[(size_t)y]; });
    for (int i = 0; i < N; ++i)
        for (int a = 0; a < ndim; ++a) points[(size_t)a * N + i] = c[(size_t)order[i] * ndim + a];
    return 0;
}

int hicma_tlr_points_mesh(const hicma_tlr_problem *prob, const char *mesh_file, int N, double *points) {
    ARG_CHECK(prob && mesh_file && points && N > 0, "hicma_tlr_points_mesh");
    ARG_CHECK(prob->kind == HICMA_TLR_KIND_MD_VIRUS, "hicma_tlr_points_mesh: kind must be md-3d-virus (6)");
    TRY(rbf_args(prob));
    FILE *f = std::fopen(mesh_file, "rb");
    ARG_CHECK(f, "cannot open the mesh file");
    std::string text;
    char buf[1 << 16];
    for (size_t got; (got = std::fread(buf, 1, sizeof buf, f)) > 0;) text.append(buf, got);
    std::fclose(f);
    // whitespace-separated numbers, '#' to the end of its line a comment
    std::vector<double> mesh;
    bool bad = false;
    for (size_t pos = 0; pos < text.size() && !bad;) {
        size_t end = text.find('\n', pos);
        if (end == std::string::npos) end = text.size();
        std::string line = text.substr(pos, end - pos);
        pos = end + 1;
        const size_t h = line.find('#');
        if (h != std::string::npos) line.resize(h);
        const char *q = line.c_str();
        for (;;) {
            char *e = nullptr;
            const double v = std::strtod(q, &e);
            if (e == q) {
                while (*q == ' ' || *q == '\t' || *q == '\r' || *q == '\v' || *q == '\f') ++q;
                bad = *q != '\0';   // something that is not a number
                break;
            }
            if (!std::isfinite(v)) { bad = true; break; }
            mesh.push_back(v);
            q = e;
        }
    }
    ARG_CHECK(!bad, "mesh file: a token that is not a finite number");
    ARG_CHECK(!mesh.empty() && mesh.size() % 3 == 0, "mesh file: expected x y z triples");
    const size_t M = mesh.size() / 3;
    const int nobj = prob->numobj > 0 ? prob->numobj : 1;
    ARG_CHECK((long long)N <= (long long)nobj * (long long)M, "N exceeds numobj times the mesh's node count");
    // Centre the object on its bounding-box centre; d = the box diagonal.
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) { lo[a] = mesh[a]; hi[a] = mesh[a]; }
    for (size_t i = 0; i < M; ++i)
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], mesh[3 * i + a]); hi[a] = std::max(hi[a], mesh[3 * i + a]); }
    double d2 = 0.0;
    for (int a = 0; a < 3; ++a) d2 += (hi[a] - lo[a]) * (hi[a] - lo[a]);
    const double d = std::sqrt(d2) > 0.0 ? std::sqrt(d2) : 1.0;
    const int side = grid_side(nobj, 3);
    std::vector<double> ctr(3 * (size_t)nobj);
    if (prob->density > 0.0) {
        const double dens = std::min(prob->density, M_PI / 6.0);
        const double spacing = d * std::cbrt(M_PI / (6.0 * dens));
        for (int o = 0; o < nobj; ++o) {
            const int g[3] = {o % side, (o / side) % side, o / (side * side)};
            for (int a = 0; a < 3; ++a) ctr[3 * o + a] = spacing * (double)g[a];
        }
    } else {
        const double L = 2.0 * d * std::cbrt((double)nobj);
        const uint64_t base = mix64h((uint64_t)prob->seed ^ 0x4D45534856495255ull);
        for (int o = 0; o < nobj; ++o)
            for (int a = 0; a < 3; ++a) {
                const uint64_t z = mix64h(base + (uint64_t)(3 * o + a));
                ctr[3 * o + a] = L * ((double)(z >> 11) * 0x1.0p-53);
            }
    }
    std::vector<double> c(3 * (size_t)nobj * M);
    for (int o = 0; o < nobj; ++o)
        for (size_t i = 0; i < M; ++i)
            for (int a = 0; a < 3; ++a)
                c[3 * ((size_t)o * M + i) + a] = ctr[3 * o + a] + (mesh[3 * i + a] - 0.5 * (lo[a] + hi[a]));
    order_points(c, prob->order, N, points);
    return 0;
}

// Releases whatever a context holds (also a partly built one from init).
static void ctx_release(hicma_tlr_ctx *c) {
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->stream_hi) cudaStreamSynchronize(c->stream_hi);
    for (auto &r : c->prof_recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    bc_remove(c->d_ws);
    bc_remove(c->d_stage);
    bc_remove(c->d_flags);
    bc_remove(c->d_scal);
    if (c->d_ws) cudaFree(c->d_ws);
    if (c->d_stage) cudaFree(c->d_stage);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    if (c->d_flags) cudaFree(c->d_flags);
    if (c->d_scal) cudaFree(c->d_scal);
    if (c->d_profacc) cudaFree(c->d_profacc);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->stream_side) cudaStreamDestroy(c->stream_side);
    if (c->stream_copy) cudaStreamDestroy(c->stream_copy);
    if (c->stream_hi) cudaStreamDestroy(c->stream_hi);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int hicma_tlr_init(int device, size_t workspace_bytes, hicma_tlr_ctx **out) {
    ARG_CHECK(out, "ctx pointer");
    *out = nullptr;
    CUDA_TRY(cudaSetDevice(device));
    auto *c = new hicma_tlr_ctx_s();
    c->device = device;
    auto fail = [&](cudaError_t e, const char *what) {
        set_err("%s: %s", what, cudaGetErrorString(e));
        cudaGetLastError();
        ctx_release(c);
        return e == cudaErrorMemoryAllocation ? HICMA_TLR_ERR_OOM : HICMA_TLR_ERR_CUDA;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(e, "stream");
    int prio_lo = 0, prio_hi = 0;
    e = cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&c->stream_hi, cudaStreamNonBlocking, prio_hi);
    if (e != cudaSuccess) return fail(e, "priority stream");
    e = cudaStreamCreateWithFlags(&c->stream_side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream_copy, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) return fail(e, "side stream");
    c->cur = c->stream;
    if (const char *q = std::getenv("HICMA_TLR_QR")) c->cholqr = std::strcmp(q, "householder") != 0;
    size_t free_b = 0, total_b = 0;
    e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess) return fail(e, "memory info");
    if (workspace_bytes == 0) {
        workspace_bytes = std::min<size_t>(free_b / 8, (size_t)8 << 30);
        workspace_bytes = std::max<size_t>(workspace_bytes, (size_t)256 << 20);
    }
    c->ws_bytes = workspace_bytes;
    e = cudaMalloc(&c->d_ws, c->ws_bytes);
    if (e != cudaSuccess) {
        c->d_ws = nullptr;
        char what[96];
        snprintf(what, sizeof what, "cudaMalloc workspace of %zu bytes", c->ws_bytes);
        return fail(e, what);
    }
    {
        const size_t hi = std::min<size_t>(c->ws_bytes / 8, (size_t)512 << 20);
        c->hi_ar.base = c->d_ws;
        c->hi_ar.bytes = hi;
        c->main_ar.base = c->d_ws + hi;
        c->main_ar.bytes = c->ws_bytes - hi;
        c->ar = &c->main_ar;
    }
    c->stage_bytes = (size_t)64 << 20;
    if ((e = cudaMallocHost(&c->h_stage, c->stage_bytes)) != cudaSuccess) { c->h_stage = nullptr; return fail(e, "pinned staging"); }
    if ((e = cudaMalloc(&c->d_stage, c->stage_bytes)) != cudaSuccess) { c->d_stage = nullptr; return fail(e, "device staging"); }
    if ((e = cudaMalloc(&c->d_flags, 64 * sizeof(int))) != cudaSuccess) { c->d_flags = nullptr; return fail(e, "flags"); }
    if ((e = cudaMalloc(&c->d_scal, 64 * sizeof(double))) != cudaSuccess) { c->d_scal = nullptr; return fail(e, "scalars"); }
    if ((e = cudaMalloc(&c->d_profacc, 64 * sizeof(double))) != cudaSuccess) { c->d_profacc = nullptr; return fail(e, "profiling counters"); }
    if ((e = xclear(c, c->d_profacc, 64 * sizeof(double))) != cudaSuccess) return fail(e, "profiling counters reset");
    bc_add(c->d_ws, c->ws_bytes);
    bc_add(c->d_stage, c->stage_bytes);
    bc_add(c->d_flags, 64 * sizeof(int));
    bc_add(c->d_scal, 64 * sizeof(double));
    if ((e = xclear(c, c->d_flags, 64 * sizeof(int))) != cudaSuccess) return fail(e, "flags reset");
    if ((e = cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
        return fail(e, "SM count");
    *out = c;
    return 0;
}

// Matrix storage: zero-filled cudaMalloc regions (a region per array), so no
// result depends on what the memory held before.
static cudaError_t dev_alloc(hicma_tlr_ctx *c, void **p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return e;
    }
    bc_add(*p, bytes);
    e = cudaMemsetAsync(*p, 0, bytes, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e;
}
static void dev_free(hicma_tlr_ctx *c, void *p) {
    if (!p) return;
    if (c) {
        cudaStreamSynchronize(c->stream_hi);
        cudaStreamSynchronize(c->stream);
    }
    bc_remove(p);
    cudaFree(p);
}

static void desc_free_device(hicma_tlr_desc *A) {
    hicma_tlr_ctx *c = A->ctx;
    dev_free(c, A->d_pts);
    dev_free(c, A->d_band);
    dev_free(c, A->d_lr);
    dev_free(c, A->d_rank);
    dev_free(c, A->d_linv);
    A->d_pts = A->d_band = A->d_lr = A->d_linv = nullptr;
    A->d_rank = nullptr;
}

int hicma_tlr_fini(hicma_tlr_ctx *c) {
    if (!c) return 0;
    if (c->async_thread.joinable()) c->async_thread.join();
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (hicma_tlr_desc *A : c->descs) {   // descriptors outliving their context
        desc_free_device(A);
        A->ctx = nullptr;
    }
    c->descs.clear();
    ctx_release(c);
    return 0;
}

void *hicma_tlr_stream(hicma_tlr_ctx *c) { return c ? (void *)c->stream : nullptr; }

int hicma_tlr_set_precision(hicma_tlr_ctx *c, int precision) {
    ARG_CHECK(c && (precision == HICMA_TLR_PREC_FP64 || precision == HICMA_TLR_PREC_MIXED), "precision");
    c->precision = precision;
    return 0;
}

// ------------------------------------------------------------- autotuner ----
// Median device time (ms) of `reps` runs of `body` between events on the
// context stream.
static int time_median(hicma_tlr_ctx *c, int reps, const std::function<int()> &body, double *ms) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    std::vector<double> t;
    int rc = 0;
    for (int r = 0; r < reps && !rc; ++r) {
        cudaEventRecord(e0, c->stream);
        rc = body();
        cudaEventRecord(e1, c->stream);
        float v = 0.f;
        if (!rc && cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&v, e0, e1) == cudaSuccess)
            t.push_back(v);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (t.empty()) { set_err("autotune: timing failed"); return HICMA_TLR_ERR_CUDA; }
    std::sort(t.begin(), t.end());
    *ms = t[t.size() / 2];
    return 0;
}

int hicma_tlr_autotune(hicma_tlr_ctx *c, int NB, int maxrank, int reps, int *tuning, double *ms_out) {
    ARG_CHECK(c && NB >= 64 && maxrank >= 1 && maxrank <= NB && reps >= 1 && reps <= 50, "autotune arguments");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    CUDA_TRY(cudaSetDevice(c->device));
    c->cur = c->stream;
    c->ar = &c->main_ar;
    ws_reset(c);
    const int keep_n = c->gemm_narrow_n, keep_g = c->potrf_grid;
    auto restore = [&]() { c->gemm_narrow_n = keep_n; c->potrf_grid = keep_g; ws_reset(c); };
    double times[12];
    for (double &v : times) v = NAN;

    // ---- tile POTRF grid: an SPD tile A0 = G G^T / NB + I, factored with each grid
    double *G = ws_alloc<double>(c, (size_t)NB * NB), *A0 = ws_alloc<double>(c, (size_t)NB * NB);
    double *At = ws_alloc<double>(c, (size_t)NB * NB), *Li = ws_alloc<double>(c, (size_t)NB * NB);
    int *dinfo = ws_alloc<int>(c, 4);
    if (!G || !A0 || !At || !Li || !dinfo) { restore(); set_err("autotune: workspace too small"); return HICMA_TLR_ERR_OOM; }
    const size_t after_potrf_bufs = c->ar->off;
    launch_gaussian(G, NB, NB, NB, 0x4155544FULL, c->stream);
    launch_set_identity(A0, NB, NB, c->stream);
    {
        std::vector<GemmTask> g{make_gemm(0, 1, NB, NB, NB, 1.0 / NB, G, NB, G, NB, 1.0, A0, NB)};
        int rc = run_gemms(c, g);
        if (rc) { restore(); return rc; }
    }
    CUDA_TRY(cudaMemsetAsync(dinfo, 0, sizeof(int), c->stream));
    const int grids[3] = {std::max(1, c->nsm / 2), c->nsm, 2 * c->nsm};
    int best_g = c->nsm;
    double best_t = INFINITY;
    for (int gi = 0; gi < 3; ++gi) {
        c->potrf_grid = grids[gi];
        double ms = 0;
        int rc = time_median(c, reps, [&]() {
            std::vector<CopyTask> cp{make_copy(A0, NB, At, NB, NB, NB)};
            TRY(run_copies(c, cp));
            c->ar->off = after_potrf_bufs;
            return potrf_tile(c, At, NB, NB, Li, NB, dinfo, 0);
        }, &ms);
        if (rc) { restore(); return rc; }
        times[gi] = ms;
        if (ms < best_t) { best_t = ms; best_g = grids[gi]; }
    }
    int hinfo = 0;
    CUDA_TRY(xfer(c, &hinfo, dinfo, sizeof(int), cudaMemcpyDeviceToHost));
    if (hinfo != 0) { restore(); set_err("autotune: test tile not positive definite (info %d)", hinfo); return HICMA_TLR_ERR_STATE; }
    TRY(check_timeout(c));

    // ---- rank-wide GEMM outputs: 128 x 32 tiles against 64 x 64 tiles for
    // widths above the default, on batches shaped like the recompression
    // products (m = NB rows, inner dimension 2n, distinct outputs)
    c->ar->off = 0;
    const int widths[4] = {48, 64, 96, 128};
    const int kmax = 256;
    double *Aop = ws_alloc<double>(c, (size_t)NB * kmax), *Bop = ws_alloc<double>(c, (size_t)kmax * 128);
    if (!Aop || !Bop) { restore(); set_err("autotune: workspace too small"); return HICMA_TLR_ERR_OOM; }
    const size_t per_out = ((size_t)NB * 128 * sizeof(double) + 1023) & ~(size_t)1023;
    const int ntask = (int)std::min<size_t>(64, ws_free(c) / (per_out + 1024));
    if (ntask < 4) { restore(); set_err("autotune: workspace too small"); return HICMA_TLR_ERR_OOM; }
    std::vector<double *> outs(ntask);
    for (int i = 0; i < ntask; ++i) outs[i] = ws_alloc<double>(c, (size_t)NB * 128);
    launch_gaussian(Aop, NB, kmax, NB, 0x41555450ULL, c->stream);
    launch_gaussian(Bop, kmax, 128, kmax, 0x41555451ULL, c->stream);
    TRY(check_launch(c));
    int narrow_n = GEMM_NARROW_N;
    bool narrow_wins = true;
    for (int wi = 0; wi < 4 && widths[wi] <= maxrank; ++wi) {   // outputs are at most maxrank wide
        const int n = widths[wi], k = 2 * n;
        double tn = 0, tw = 0;
        for (int variant = 0; variant < 2; ++variant) {
            c->gemm_narrow_n = variant == 0 ? n : 0;
            double ms = 0;
            int rc = time_median(c, reps, [&]() {
                std::vector<GemmTask> g;
                for (int i = 0; i < ntask; ++i) g.push_back(make_gemm(0, 0, NB, n, k, 1.0, Aop, NB, Bop, kmax, 0.0, outs[i], NB));
                return run_gemms(c, g);
            }, &ms);
            if (rc) { restore(); return rc; }
            (variant == 0 ? tn : tw) = ms;
        }
        times[3 + 2 * wi] = tn;
        times[4 + 2 * wi] = tw;
        if (narrow_wins && tn <= tw) narrow_n = n;
        else narrow_wins = false;
    }
    c->gemm_narrow_n = narrow_n;
    c->potrf_grid = best_g;
    ws_reset(c);
    if (tuning) { tuning[0] = c->gemm_narrow_n; tuning[1] = c->potrf_grid; }
    if (ms_out) std::memcpy(ms_out, times, 11 * sizeof(double));
    return 0;
}

int hicma_tlr_tuning_get(hicma_tlr_ctx *c, int *tuning) {
    ARG_CHECK(c && tuning, "tuning_get arguments");
    tuning[0] = c->gemm_narrow_n;
    tuning[1] = c->potrf_grid;
    return 0;
}

int hicma_tlr_tuning_set(hicma_tlr_ctx *c, const int *tuning) {
    ARG_CHECK(c && tuning, "tuning_set arguments");
    ARG_CHECK(tuning[0] >= 0 && tuning[0] <= 4096, "gemm_narrow_n in [0, 4096]");
    ARG_CHECK(tuning[1] >= 0 && tuning[1] <= 16 * c->nsm, "potrf_grid in [0, 16 x SMs]");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    c->gemm_narrow_n = tuning[0];
    c->potrf_grid = tuning[1];
    return 0;
}

int hicma_tlr_desc_create(hicma_tlr_ctx *c, int N, int NB, int maxrank, int band_size, hicma_tlr_desc **out) {
    ARG_CHECK(c && out, "null");
    ARG_CHECK(N > 0 && NB > 0, "N, NB must be positive");
    if (N % NB != 0) {
        set_err("N (%d) must be a multiple of NB (%d): ragged last tiles are not supported", N, NB);
        return HICMA_TLR_ERR_NOT_SUPPORTED;
    }
    ARG_CHECK(maxrank >= 1 && maxrank <= NB, "maxrank in [1, NB]");
    ARG_CHECK(band_size >= 1, "band_size >= 1");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    CUDA_TRY(cudaSetDevice(c->device));
    auto *A = new hicma_tlr_desc_s();
    A->ctx = c;
    A->N = N; A->NB = NB; A->NT = N / NB; A->maxrank = maxrank;
    A->band = std::min(band_size, A->NT);
    A->slot_band = A->band;
    A->band_alloc = A->band;
    const int NT = A->NT;
    const long long mm = NT - A->slot_band;
    A->nslots = mm > 0 ? mm * (mm + 1) / 2 : 0;
    const size_t band_bytes = (size_t)NT * A->band_alloc * NB * (size_t)NB * sizeof(double);
    const size_t lr_bytes = (size_t)A->nslots * 2 * (size_t)NB * maxrank * sizeof(double);
    if (dev_alloc(c, (void **)&A->d_band, band_bytes) != cudaSuccess ||
        (lr_bytes && dev_alloc(c, (void **)&A->d_lr, lr_bytes) != cudaSuccess) ||
        dev_alloc(c, (void **)&A->d_rank, (size_t)NT * NT * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        set_err("descriptor allocation failed (band %zu B, low-rank slots %zu B)", band_bytes, lr_bytes);
        dev_free(c, A->d_band); dev_free(c, A->d_lr); dev_free(c, A->d_rank);
        delete A;
        return HICMA_TLR_ERR_OOM;
    }
    A->h_rank.assign((size_t)NT * NT, -1);
    for (int m = 0; m < NT; ++m)
        for (int n = 0; n <= m - A->band; ++n) A->h_rank[(size_t)n * NT + m] = 0;
    const cudaError_t e = xfer(c, A->d_rank, A->h_rank.data(), (size_t)NT * NT * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        set_err("rank map upload: %s", cudaGetErrorString(e));
        dev_free(c, A->d_band); dev_free(c, A->d_lr); dev_free(c, A->d_rank);
        delete A;
        return HICMA_TLR_ERR_CUDA;
    }
    c->descs.insert(A);
    *out = A;
    return 0;
}

int hicma_tlr_desc_destroy(hicma_tlr_desc *A) {
    if (!A) return 0;
    if (A->ctx) {
        hicma_tlr_ctx *c = A->ctx;
        std::lock_guard<std::recursive_mutex> lk(c->mu);
        cudaSetDevice(c->device);
        cudaStreamSynchronize(c->stream);
        desc_free_device(A);
        c->descs.erase(A);
    }
    delete A;
    return 0;
}

int hicma_tlr_desc_info(const hicma_tlr_desc *A, int *N, int *NB, int *NT, int *maxrank, int *band_size) {
    ARG_CHECK(A, "null desc");
    if (N) *N = A->N;
    if (NB) *NB = A->NB;
    if (NT) *NT = A->NT;
    if (maxrank) *maxrank = A->maxrank;
    if (band_size) *band_size = A->band;
    return 0;
}

int hicma_tlr_desc_copy(hicma_tlr_ctx *c, const hicma_tlr_desc *src, hicma_tlr_desc *dst) {
    ARG_CHECK(c && src && dst, "null");
    ARG_CHECK(src->N == dst->N && src->NB == dst->NB && src->maxrank == dst->maxrank &&
                  src->slot_band == dst->slot_band,
              "descriptor shapes differ (N, NB, maxrank and the band it was created with must match)");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    const size_t NB = src->NB, NT = src->NT;
    if (dst->band_alloc != src->band_alloc) {
        // the source's band was widened (band regeneration): the copy adopts it
        dev_free(c, dst->d_band);
        dst->d_band = nullptr;
        const size_t bytes = NT * src->band_alloc * NB * NB * sizeof(double);
        if (dev_alloc(c, (void **)&dst->d_band, bytes) != cudaSuccess) {
            cudaGetLastError();
            set_err("band allocation of %zu bytes failed", bytes);
            return HICMA_TLR_ERR_OOM;
        }
        dst->band_alloc = src->band_alloc;
    }
    CUDA_TRY(cudaMemcpyAsync(dst->d_band, src->d_band, NT * src->band_alloc * NB * NB * sizeof(double),
                             cudaMemcpyDeviceToDevice, c->stream));
    if (src->nslots)
        CUDA_TRY(cudaMemcpyAsync(dst->d_lr, src->d_lr, (size_t)src->nslots * 2 * NB * src->maxrank * sizeof(double),
                                 cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(dst->d_rank, src->d_rank, NT * NT * sizeof(int), cudaMemcpyDeviceToDevice, c->stream));
    dst->h_rank = src->h_rank;
    dst->band = src->band;
    dst->factored = src->factored;
    if (src->d_pts) {
        if (!dst->d_pts || dst->ndim != src->ndim) {
            dev_free(c, dst->d_pts);
            CUDA_TRY(dev_alloc(c, (void **)&dst->d_pts, (size_t)src->ndim * src->N * sizeof(double)));
        }
        dst->ndim = src->ndim;
        CUDA_TRY(cudaMemcpyAsync(dst->d_pts, src->d_pts, (size_t)src->ndim * src->N * sizeof(double),
                                 cudaMemcpyDeviceToDevice, c->stream));
    }
    if (src->factored && src->d_linv) {
        if (!dst->d_linv) CUDA_TRY(dev_alloc(c, (void **)&dst->d_linv, NT * NB * NB * sizeof(double)));
        CUDA_TRY(cudaMemcpyAsync(dst->d_linv, src->d_linv, NT * NB * NB * sizeof(double),
                                 cudaMemcpyDeviceToDevice, c->stream));
    }
    return ctx_sync(c);
}

// randtlr bases on the device (restated starsh_randtlr_generate,
// hicma_parsec/testing_dpotrf.c:315-321): per block row m a Gaussian NB x K
// matrix (counter generator, seed (seed ^ RANDTLR_SEED_XOR) + m), its
// Householder QR, Q formed from the reflectors, column signs fixed by R's
// diagonal, and Q diag(S) beside it.  Chunked over block rows to the arena.
static int build_randtlr_basis(hicma_tlr_ctx *c, hicma_tlr_desc *A, const hicma_tlr_problem *prob) {
    const int NB = A->NB, NT = A->NT, N = A->N;
    const int K = std::min(NB, RANDTLR_KMAX);
    const int pb = qr_panel_width(NB);
    const size_t npan = (size_t)(K + pb - 1) / pb + 1;
    const size_t mark = c->ar->off;
    double *ident = ws_alloc<double>(c, (size_t)K * K);
    if (!ident) { set_err("workspace too small for the randtlr bases"); return HICMA_TLR_ERR_OOM; }
    launch_set_identity(ident, K, K, c->stream);
    TRY(check_launch(c));
    const size_t per_block = 2 * align_up(sizeof(double) * (size_t)NB * K + 1) + align_up(sizeof(double) * K + 1) +
                             align_up(sizeof(double) * npan * pb * pb + 1) + 4096;
    const int chunk = (int)std::min<size_t>((size_t)NT, ws_free(c) / per_block);
    if (chunk < 1) { c->ar->off = mark; set_err("workspace too small for the randtlr bases"); return HICMA_TLR_ERR_OOM; }
    const size_t inner = c->ar->off;
    for (int m0 = 0; m0 < NT; m0 += chunk) {
        c->ar->off = inner;
        const int nblk = std::min(chunk, NT - m0);
        double *G = ws_alloc<double>(c, (size_t)nblk * NB * K);
        double *Q = ws_alloc<double>(c, (size_t)nblk * NB * K);
        double *tau = ws_alloc<double>(c, (size_t)nblk * K);
        double *T = ws_alloc<double>(c, (size_t)nblk * npan * pb * pb);
        if (!G || !Q || !tau || !T) { c->ar->off = mark; set_err("workspace too small for the randtlr bases"); return HICMA_TLR_ERR_OOM; }
        std::vector<QRTask> qr;
        std::vector<QApplyTask> ap;
        for (int b = 0; b < nblk; ++b) {
            double *Gb = G + (size_t)b * NB * K;
            double *Tb = T + (size_t)b * npan * pb * pb;
            const unsigned long long sd = ((unsigned long long)prob->seed ^ RANDTLR_SEED_XOR) + (unsigned long long)(m0 + b);
            launch_gaussian(Gb, NB, K, NB, sd, c->stream);
            qr.push_back(QRTask{Gb, tau + (size_t)b * K, Tb, NB, K, NB});
            ap.push_back(QApplyTask{Gb, Tb, ident, Q + (size_t)b * NB * K, nullptr, NB, K, NB, K, NB, K});
        }
        TRY(check_launch(c));
        TRY(run_qr(c, qr, NB));
        TRY(run_qapply(c, ap, NB));
        launch_randtlr_finish(G, Q, NB, K, nblk, m0, A->d_pts, N, RANDTLR_DECAY, c->stream);
        TRY(check_launch(c));
    }
    c->ar->off = mark;
    return 0;
}

static int set_points(hicma_tlr_ctx *c, hicma_tlr_desc *A, const hicma_tlr_problem *prob, const double *points) {
    const int ndim = data_ndim(prob->kind, A->NB);
    ARG_CHECK(ndim > 0, "unsupported problem kind (-D 0 to 7)");
    TRY(rbf_args(prob));
    ARG_CHECK(!(prob->kind == HICMA_TLR_KIND_MD_VIRUS && !points),
              "md-3d-virus needs the mesh points (hicma_tlr_points_mesh)");
    const bool randtlr = prob->kind == HICMA_TLR_KIND_RANDTLR;
    ARG_CHECK(!(randtlr && points), "randtlr takes no points (its bases are built on the device)");
    std::vector<double> h;
    if (!points && !randtlr) {
        h.resize((size_t)ndim * A->N);
        TRY(hicma_tlr_points(prob, A->N, h.data()));
        points = h.data();
    }
    if (!A->d_pts || A->ndim != ndim) {
        dev_free(c, A->d_pts);
        A->d_pts = nullptr;
        CUDA_TRY(dev_alloc(c, (void **)&A->d_pts, (size_t)ndim * A->N * sizeof(double)));
    }
    A->ndim = ndim;
    if (randtlr) {
        TRY(build_randtlr_basis(c, A, prob));
    } else {
        CUDA_TRY(cudaMemcpyAsync(A->d_pts, points, (size_t)ndim * A->N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    }
    return ctx_sync(c);
}

// The descriptor's per-row data must be that of prob's kind (band
// regeneration and the checks regenerate tiles from it).
static int check_problem_data(const hicma_tlr_desc *A, const hicma_tlr_problem *prob) {
    ARG_CHECK(A->d_pts, "no points: generate first");
    TRY(rbf_args(prob));
    ARG_CHECK(data_ndim(prob->kind, A->NB) == A->ndim && A->ndim > 0,
              "problem kind differs from the one the descriptor was generated with");
    return 0;
}

// Kernel parameters of a problem over N points.  A non-positive add_diag of
// the electrodynamics kinds means N, the reference's default
// (hicma_parsec/hicma_parsec.c:289-291).
static CovParams make_cov_params(const hicma_tlr_problem *prob, const double *d_points, int N, int ndim) {
    CovParams p;
    p.pts = d_points; p.N = N; p.ndim = ndim; p.kind = prob->kind;
    p.beta = prob->beta; p.sigma = prob->sigma; p.noise = prob->noise;
    p.wave_k = prob->wave_k;
    p.add_diag = prob->add_diag > 0.0 ? prob->add_diag : (double)N;
    p.rbf = prob->rbf_kernel;
    p.inv_radius = prob->radius > 0.0 ? 1.0 / prob->radius : 0.0;
    return p;
}

static CovParams cov_params(const hicma_tlr_desc *A, const hicma_tlr_problem *prob) {
    return make_cov_params(prob, A->d_pts, A->N, A->ndim);
}

static int gen_band_tiles(hicma_tlr_ctx *c, hicma_tlr_desc *A, const hicma_tlr_problem *prob) {
    std::vector<CovTask> tasks;
    for (int m = 0; m < A->NT; ++m)
        for (int n = std::max(m - A->band + 1, 0); n <= m; ++n)
            tasks.push_back(CovTask{A->dense(m, n), A->NB, m * A->NB, n * A->NB, A->NB, A->NB});
    TRY(bc_cov(cov_params(A, prob), tasks));
    CovTask *dt = stage(c, tasks.data(), tasks.size());
    if (!dt) { set_err("staging failed"); return HICMA_TLR_ERR_CUDA; }
    Prof pf(c, P_COV, 0, 8.0 * tasks.size() * (double)A->NB * A->NB);
    launch_cov_batched(cov_params(A, prob), dt, (int)tasks.size(), A->NB, A->NB, c->stream);
    return check_launch(c);
}

// Randomized range finder + truncated SVD of a batch of dense tiles
// (restated starsh_dense_dlrrsdd): Y = A Omega, Q = qr(Y), W = A^T Q,
// W = Q_W R_W, svd(R_W^T) = U S V^T, rank by relative Frobenius tol;
// U_tile = Q U_r, V_tile = Q_W V_r S_r.
struct CompressTask {
    const double *A;     // nb x nb dense (ld nb)
    double *outU, *outV;
    int *rank_dst;
};

static size_t compress_ws_bytes(int nb, int s) {
    const int pb = qr_panel_width(nb);
    const size_t npan = (size_t)(s + pb - 1) / pb + 1;
    size_t b = 0;
    b += align_up(sizeof(double) * (size_t)nb * s + 1) * 4;   // Y, Q, W, Wkeep
    b += align_up(sizeof(double) * (size_t)s + 1) * 2;
    b += align_up(sizeof(double) * npan * pb * pb + 1) * 2;
    b += align_up(sizeof(double) * (size_t)s * s + 1) * 3;    // SU (+ R_Y, R_W of the CholeskyQR path)
    if (s > core_smem_kmax()) b += align_up(sizeof(double) * core_work_doubles(s) + 1);
    return b + 1024;
}

// Largest entry of |Q^T Q - I| accepted from the randomized CholeskyQR range
// finder.  Healthy samples give about 1e-14; a sample of exactly lower rank
// than its width (a sparse tile, e.g. a compactly supported RBF) can leave Q
// far from orthonormal, and such a tile is compressed again on the Householder
// path.
constexpr double GEN_ORTH_THR = 1e-10;

// d_fail (optional, one int per task): the CholeskyQR path writes 1 where the
// range finder's Q fails the orthogonality check, else 0.  force_hh: take the
// Householder path whatever s is.
static int run_compress(hicma_tlr_ctx *c, int nb, int maxrank, double tol, const double *Omega, int s,
                        std::vector<CompressTask> &tasks, const double *d_identity, int *d_rank_task_base,
                        int *d_fail = nullptr, bool force_hh = false) {
    const int pb = qr_panel_width(nb);
    const size_t npan = (size_t)(s + pb - 1) / pb + 1;
    const size_t mark = c->ar->off;
    size_t i0 = 0;
    while (i0 < tasks.size()) {
        c->ar->off = mark;
        std::vector<GemmTask> gy, gw, gv;
        std::vector<CopyTask> keeps;
        std::vector<QRTask> qy, qw;
        std::vector<QApplyTask> aq, au;
        std::vector<CoreTask> cores;
        std::vector<CQTask> cqy, cqw;
        std::vector<GemmTask> gu;
        std::vector<GramTask> gq;
        // up to rcholqr_kmax() samples: both QRs by randomized CholeskyQR (Q of
        // Y formed, R of W only), U = Q_Y U_r as a GEMM
        const bool cq = c->cholqr && s <= rcholqr_kmax() && !force_hh;
        size_t i = i0;
        for (; i < tasks.size(); ++i) {
            if (compress_ws_bytes(nb, s) > ws_free(c)) {
                if (i == i0) { set_err("workspace too small for one tile compression"); return HICMA_TLR_ERR_OOM; }
                break;
            }
            const CompressTask &t = tasks[i];
            if (cq) {
                double *Y = ws_alloc<double>(c, (size_t)nb * s);
                double *Q = ws_alloc<double>(c, (size_t)nb * s);
                double *W = ws_alloc<double>(c, (size_t)nb * s);
                double *RY = ws_alloc<double>(c, (size_t)s * s), *RW = ws_alloc<double>(c, (size_t)s * s);
                double *SU = ws_alloc<double>(c, (size_t)s * s);
                int *rt = d_rank_task_base + (i - i0);
                gy.push_back(make_gemm(0, 0, nb, s, nb, 1.0, t.A, nb, Omega, nb, 0.0, Y, nb));
                cqy.push_back(CQTask{Y, nullptr, Q, RY, Q, nb, s, 0, nb, nb});
                if (d_fail) gq.push_back(GramTask{Q, Q, ws_alloc<double>(c, (size_t)s * s), nb, s, s});
                gw.push_back(make_gemm(1, 0, nb, s, nb, 1.0, t.A, nb, Q, nb, 0.0, W, nb));
                cqw.push_back(CQTask{W, nullptr, nullptr, RW, nullptr, nb, s, 0, nb, nb});
                CoreTask ct{};
                ct.RU = nullptr; ct.RV = RW; ct.ldru = s; ct.ldrv = s;
                ct.SU = SU; ct.RUc = nullptr; ct.work = nullptr;
                ct.rank_out = t.rank_dst; ct.rank_task = rt; ct.K = s;
                cores.push_back(ct);
                GemmTask gU = make_gemm(0, 0, nb, std::min(s, maxrank), s, 1.0, Q, nb, SU, s, 0.0, t.outU, nb);
                gU.n_dev = rt;
                gu.push_back(gU);
                // V Sigma = (A^T Q) U_r  (R_U = I)
                GemmTask g = make_gemm(0, 0, nb, std::min(s, maxrank), s, 1.0, W, nb, SU, s, 0.0, t.outV, nb);
                g.n_dev = rt;
                gv.push_back(g);
                continue;
            }
            double *Y = ws_alloc<double>(c, (size_t)nb * s);
            double *Q = ws_alloc<double>(c, (size_t)nb * s);
            double *W = ws_alloc<double>(c, (size_t)nb * s);
            double *Wk = ws_alloc<double>(c, (size_t)nb * s);
            double *tauY = ws_alloc<double>(c, s), *tauW = ws_alloc<double>(c, s);
            double *TY = ws_alloc<double>(c, npan * pb * pb), *TW = ws_alloc<double>(c, npan * pb * pb);
            double *SU = ws_alloc<double>(c, (size_t)s * s);
            double *work = s > core_smem_kmax() ? ws_alloc<double>(c, core_work_doubles(s)) : nullptr;
            int *rt = d_rank_task_base + (i - i0);
            gy.push_back(make_gemm(0, 0, nb, s, nb, 1.0, t.A, nb, Omega, nb, 0.0, Y, nb));
            qy.push_back(QRTask{Y, tauY, TY, nb, s, nb});
            aq.push_back(QApplyTask{Y, TY, d_identity, Q, nullptr, nb, s, nb, s, nb, s});
            gw.push_back(make_gemm(1, 0, nb, s, nb, 1.0, t.A, nb, Q, nb, 0.0, W, nb));
            keeps.push_back(make_copy(W, nb, Wk, nb, nb, s));
            qw.push_back(QRTask{W, tauW, TW, nb, s, nb});
            CoreTask ct{};
            ct.RU = nullptr; ct.RV = W; ct.ldru = nb; ct.ldrv = nb;
            ct.SU = SU; ct.RUc = nullptr; ct.work = work;
            ct.rank_out = t.rank_dst; ct.rank_task = rt; ct.K = s;
            cores.push_back(ct);
            au.push_back(QApplyTask{Y, TY, SU, t.outU, rt, nb, s, nb, s, nb, maxrank});
            // V Sigma = (A^T Q) U_r  (R_U = I)
            GemmTask g = make_gemm(0, 0, nb, std::min(s, maxrank), s, 1.0, Wk, nb, SU, s, 0.0, t.outV, nb);
            g.n_dev = rt;
            gv.push_back(g);
        }
        TRY(run_gemms(c, gy, false, P_GEMM_GEN));
        TRY(run_qr(c, qy, nb));
        TRY(run_rcholqr(c, cqy, 0));
        if (!gq.empty()) {
            // Q^T Q of every formed Q, then the orthogonality flags of this sub-batch
            GramTask *dq = stage(c, gq.data(), gq.size());
            if (!dq) { set_err("staging failed"); return HICMA_TLR_ERR_CUDA; }
            {
                Prof pf(c, P_GRAM, 2.0 * nb * (double)s * s * gq.size(), 8.0 * nb * (double)s * gq.size());
                launch_gram_batched(dq, (int)gq.size(), c->cur);
            }
            TRY(check_launch(c));
            launch_orth_check(dq, (int)gq.size(), GEN_ORTH_THR, d_fail + i0, c->cur);
            TRY(check_launch(c));
        }
        TRY(run_qapply(c, aq, nb));
        TRY(run_gemms(c, gw, false, P_GEMM_GEN));
        TRY(run_copies(c, keeps));
        TRY(run_qr(c, qw, nb));
        TRY(run_rcholqr(c, cqw, 0));
        CoreParams cp{1, tol, maxrank, 0, nb, nullptr, nullptr};
        TRY(run_core_buckets(c, cores, cp));
        TRY(run_qapply(c, au, nb));
        TRY(run_gemms(c, gu, false, P_GEMM_GEN));
        TRY(run_gemms(c, gv, false, P_GEMM_GEN));
        i0 = i;
    }
    c->ar->off = mark;
    return 0;
}

int hicma_tlr_generate(hicma_tlr_ctx *c, int uplo, hicma_tlr_desc *A, int *Ar, const hicma_tlr_problem *prob,
                       const double *points, double tol, int maxrank, int band_size, int send_full_tile,
                       int *info) {
    (void)send_full_tile;
    ARG_CHECK(c && A && prob, "null");
    if (uplo != HICMA_TLR_LOWER) { set_err("only uplo = Lower is supported"); return HICMA_TLR_ERR_NOT_SUPPORTED; }
    ARG_CHECK(band_size >= 1, "band_size should be not less than 1");
    ARG_CHECK(band_size == A->band, "band_size must equal the descriptor's band size");
    ARG_CHECK(maxrank >= 1 && maxrank <= A->maxrank, "maxrank must be in [1, descriptor maxrank]");
    ARG_CHECK(tol > 0.0, "tol > 0");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    NvtxRange nv("STARSH_gen");
    CUDA_TRY(cudaSetDevice(c->device));
    if (info) *info = 0;
    c->cur = c->stream;
    c->ar = &c->main_ar;
    ws_reset(c);
    TRY(set_points(c, A, prob, points));
    ws_reset(c);
    const int NT = A->NT, NB = A->NB;
    TRY(gen_band_tiles(c, A, prob));
    // off-band tiles: generate dense into the workspace, compress into slots.
    // The reference samples min(maxrank + 10, NB) columns for every tile
    // (STARSH_gen.jdf:262-266); the sampled singular values only matter up to
    // the rank, so tiles start with s = min(64, s_full) samples (the CholeskyQR
    // path; 160 with the Householder path) and a tile whose rank comes within
    // max(32, s/4) of s is generated again with twice the samples, up to
    // s_full.  Rejected tiles (2r >= NB) stay rejected: more samples can only
    // raise the rank.
    const int s_full = std::min(maxrank + 10, NB);
    double *Omega = ws_alloc<double>(c, (size_t)NB * s_full);
    double *Ident = ws_alloc<double>(c, (size_t)s_full * s_full);
    int *rtask = ws_alloc<int>(c, (size_t)NT * NT + 1);
    if (!Omega || !Ident || !rtask) { set_err("workspace too small"); return HICMA_TLR_ERR_OOM; }
    launch_gaussian(Omega, NB, s_full, NB, prob->seed ^ 0x5DEECE66Dull, c->stream);
    TRY(check_launch(c));
    std::vector<std::pair<int, int>> pending;
    for (int m = A->band; m < NT; ++m)
        for (int n = 0; n <= m - A->band; ++n) pending.push_back({m, n});
    const CovParams cp = cov_params(A, prob);
    int s = std::min(c->cholqr ? rcholqr_kmax() : 160, s_full);
    // force_hh: the round compresses tiles whose CholeskyQR range finder failed
    // its orthogonality check, on the Householder path at the same s
    bool force_hh = false;
    while (!pending.empty()) {
        const size_t mark_round = c->ar->off;
        const bool cq_round = c->cholqr && s <= rcholqr_kmax() && !force_hh;
        int *dfail = cq_round ? ws_alloc<int>(c, pending.size()) : nullptr;
        if (cq_round && !dfail) { set_err("workspace too small"); return HICMA_TLR_ERR_OOM; }
        launch_set_identity(Ident, s, s, c->stream);
        TRY(check_launch(c));
        const size_t per_tile = align_up(sizeof(double) * (size_t)NB * NB + 1) + compress_ws_bytes(NB, s);
        const size_t chunk = std::max<size_t>(1, ws_free(c) / (per_tile + 4096));
        for (size_t t0 = 0; t0 < pending.size(); t0 += chunk) {
            const size_t t1 = std::min(pending.size(), t0 + chunk);
            const size_t mark = c->ar->off;
            std::vector<CovTask> cov;
            std::vector<CompressTask> comp;
            for (size_t i = t0; i < t1; ++i) {
                const int m = pending[i].first, n = pending[i].second;
                double *D = ws_alloc<double>(c, (size_t)NB * NB);
                cov.push_back(CovTask{D, NB, m * NB, n * NB, NB, NB});
                comp.push_back(CompressTask{D, A->U(m, n), A->V(m, n), A->d_rank + (size_t)n * NT + m});
            }
            TRY(bc_cov(cp, cov));
            CovTask *dcov = stage(c, cov.data(), cov.size());
            if (!dcov) { set_err("staging failed"); return HICMA_TLR_ERR_CUDA; }
            {
                Prof pf(c, P_COV, 0, 8.0 * cov.size() * (double)NB * NB);
                launch_cov_batched(cp, dcov, (int)cov.size(), NB, NB, c->stream);
            }
            TRY(check_launch(c));
            TRY(run_compress(c, NB, maxrank, tol, Omega, s, comp, Ident, rtask, dfail ? dfail + t0 : nullptr,
                             force_hh));
            c->ar->off = mark;
        }
        std::vector<int> fails;
        if (dfail) {
            fails.resize(pending.size());
            CUDA_TRY(xfer(c, fails.data(), dfail, fails.size() * sizeof(int), cudaMemcpyDeviceToHost));
        }
        c->ar->off = mark_round;
        const bool any_fail = std::find(fails.begin(), fails.end(), 1) != fails.end();
        if (s >= s_full && !any_fail) break;
        TRY(ctx_sync(c));
        CUDA_TRY(xfer(c, A->h_rank.data(), A->d_rank, (size_t)NT * NT * sizeof(int), cudaMemcpyDeviceToHost));
        std::vector<std::pair<int, int>> more;
        const int margin = std::max(32, s / 4);
        bool grow = false;
        for (size_t i = 0; i < pending.size(); ++i) {
            const auto &t = pending[i];
            if (!fails.empty() && fails[i]) { more.push_back(t); continue; }
            const int r = A->rank(t.first, t.second);
            if (s < s_full && r >= 0 && r > s - margin) { more.push_back(t); grow = true; }
        }
        pending.swap(more);
        if (grow) s = std::min(2 * s, s_full);
        force_hh = any_fail;
    }
    TRY(ctx_sync(c));
    CUDA_TRY(xfer(c, A->h_rank.data(), A->d_rank, (size_t)NT * NT * sizeof(int), cudaMemcpyDeviceToHost));
    int bad = 0;
    for (int m = A->band; m < NT; ++m)
        for (int n = 0; n <= m - A->band; ++n)
            if (A->rank(m, n) < 0) {
                if (bad < 4) fprintf(stderr, "Tile(%d, %d) is dense, try increasing NB or maxrank \n", m, n);
                ++bad;
            }
    // Ar reports rejected tiles as -1, the value the reference leaves in dcAr
    // when starsh_dense_dlrrsdd returns rank -1 (STARSH_gen.jdf:169-175); the
    // descriptor stores them with rank 0 so that no kernel reads their slots.
    if (Ar) std::memcpy(Ar, A->h_rank.data(), (size_t)NT * NT * sizeof(int));
    if (bad) {
        for (int m = A->band; m < NT; ++m)
            for (int n = 0; n <= m - A->band; ++n)
                if (A->h_rank[(size_t)n * NT + m] < 0) A->h_rank[(size_t)n * NT + m] = 0;
        CUDA_TRY(xfer(c, A->d_rank, A->h_rank.data(), (size_t)NT * NT * sizeof(int), cudaMemcpyHostToDevice));
        if (info) *info = -1;
    }
    A->factored = false;
    return 0;
}

int hicma_tlr_rank_gather(hicma_tlr_ctx *c, hicma_tlr_desc *A, int *rank_array, int band_size) {
    ARG_CHECK(c && A && rank_array, "null");
    (void)band_size;
    const int NT = A->NT;
    for (int n = 0; n < NT; ++n)
        for (int m = 0; m < NT; ++m) rank_array[(size_t)n * NT + m] = A->is_dense(m, n) || m < n ? -1 : A->rank(m, n);
    return 0;
}

int hicma_tlr_rank_history(hicma_tlr_desc *A, int *initial, int *minimum, int *maximum, int *final_rank) {
    ARG_CHECK(A, "null");
    const size_t n2 = (size_t)A->NT * A->NT;
    if (A->rk_init.size() != n2) { set_err("no factorization has run on this descriptor"); return HICMA_TLR_ERR_STATE; }
    if (initial) std::memcpy(initial, A->rk_init.data(), n2 * sizeof(int));
    if (minimum) std::memcpy(minimum, A->rk_min.data(), n2 * sizeof(int));
    if (maximum) std::memcpy(maximum, A->rk_max.data(), n2 * sizeof(int));
    if (final_rank)
        for (size_t i = 0; i < n2; ++i) final_rank[i] = A->rk_init[i] < 0 ? -1 : A->h_rank[i];
    return 0;
}

int hicma_tlr_dpotrf_L_rank(hicma_tlr_ctx *c, int uplo, hicma_tlr_desc *A, int *Ar, int *Rank, double acc,
                            int fixed_rank, int maxrank, int *lookahead, int band_size, int hmb, int compmaxrank,
                            int send_full_tile, int *two_flow, unsigned long *tileopcounters,
                            unsigned long *opcounters, double *critical_path_time, int verbose) {
    const int info = hicma_tlr_dpotrf_L(c, uplo, A, Ar, acc, fixed_rank, maxrank, lookahead, band_size, hmb,
                                        compmaxrank, send_full_tile, two_flow, tileopcounters, opcounters,
                                        critical_path_time, verbose);
    if (info < 0 || !Rank) return info;
    // the dcRank record: 4 ints per tile (initial, minimum, maximum, final) at (n*NT + m)*4
    const size_t n2 = (size_t)A->NT * A->NT;
    std::vector<int> h(4 * n2);
    TRY(hicma_tlr_rank_history(A, h.data(), h.data() + n2, h.data() + 2 * n2, h.data() + 3 * n2));
    for (size_t t = 0; t < n2; ++t)
        for (int q = 0; q < 4; ++q) Rank[4 * t + q] = h[q * n2 + t];
    return info;
}

int hicma_tlr_rank_stat(const int *G, int NT, int band_size, int *minrk, int *maxrk, double *avgrk) {
    ARG_CHECK(G && NT > 0 && band_size >= 1, "rank_stat");
    int mn = 2147483647, mx = 0;
    long long sum = 0, num = 0;
    for (int i = band_size; i < NT; ++i)
        for (int j = 0; j < i - band_size + 1; ++j) {
            const int v = G[(size_t)j * NT + i];
            sum += v; ++num;
            mn = std::min(mn, v); mx = std::max(mx, v);
        }
    if (minrk) *minrk = mn;
    if (maxrk) *maxrk = mx;
    if (avgrk) *avgrk = num ? (double)sum / (double)num : NAN;
    return 0;
}

int hicma_tlr_band_autotune(const int *G, int NT, int NB, int verbose) {
    ARG_CHECK(G && NT > 0 && NB > 0, "band_autotune");
    const double FLUCTUATION = 0.66666667;   // hicma_parsec_internal.h:107
    int indicator_min = 0, opt_min = 0;
    for (int band = 2; band < NT; ++band) {
        long long t_tlr = 0, t_dense = 0, g_tlr = 0, g_dense = 0;
        for (int m = band - 1; m < NT; ++m) {
            const int k = m + 1 - band;
            const int ar = G[(size_t)k * NT + m];
            t_tlr += (long long)NB * NB * ar;
            t_dense += (long long)NB * NB * NB;
        }
        for (int k = 0; k <= NT - 3; ++k)
            for (int m = k + band; m < NT; ++m) {
                const int n = m + 1 - band;
                const int ar = G[(size_t)k * NT + m], br = G[(size_t)k * NT + n], cr = G[(size_t)n * NT + m];
                const unsigned long ca = (unsigned long)(cr + ar);
                const unsigned long qra = op_counts('q', NB, ca, 0, 0);
                unsigned long qrb = op_counts('m', ar, br, NB, 0);
                qrb += op_counts('m', ar, NB, br, 0);
                qrb += op_counts('q', NB, ca, 0, 0);
                unsigned long svd = op_counts('r', ca, ca, 2, 0);
                svd += op_counts('s', ca, 0, 0, 0);
                svd += ca * (unsigned long)cr;
                const unsigned long nu = op_counts('o', NB, cr, ca, 1);
                const unsigned long nv = op_counts('o', cr, NB, ca, 2);
                g_tlr += (long long)qra + qrb + svd + nu + nv;
                if (m - k < band) g_dense += (long long)2 * NB * NB * NB;
                else if (n - k < band && m - n < band) g_dense += (long long)4 * NB * NB * ar;
                else if (m - n < band) g_dense += (long long)2 * NB * NB * std::min(ar, br) + (long long)4 * NB * ar * br;
            }
        const long long s_tlr = t_tlr + g_tlr, s_dense = t_dense + g_dense;
        if (verbose)
            fprintf(stderr, "band_size: %d, ops_sum_tlr: %e, ops_sum_dense: %e\n", band, (double)s_tlr, (double)s_dense);
        if ((double)s_tlr * FLUCTUATION <= (double)s_dense && indicator_min == 0) {
            indicator_min = 1;
            opt_min = band - 1;
        }
        if (s_tlr <= s_dense) return opt_min;
    }
    return NT;
}

int hicma_tlr_band_regenerate(hicma_tlr_ctx *c, int uplo, hicma_tlr_desc *A, const hicma_tlr_problem *prob,
                              int band_size) {
    ARG_CHECK(c && A && prob, "null");
    if (uplo != HICMA_TLR_LOWER) { set_err("only uplo = Lower is supported"); return HICMA_TLR_ERR_NOT_SUPPORTED; }
    ARG_CHECK(band_size >= A->slot_band, "band_size cannot shrink below the slot band");
    TRY(check_problem_data(A, prob));
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    NvtxRange nv("band_regenerate");
    const int NT = A->NT, NB = A->NB;
    band_size = std::min(band_size, NT);
    TRY(ctx_sync(c));
    if (band_size > A->band_alloc) {
        dev_free(c, A->d_band);
        A->d_band = nullptr;
        const size_t bytes = (size_t)NT * band_size * NB * (size_t)NB * sizeof(double);
        if (dev_alloc(c, (void **)&A->d_band, bytes) != cudaSuccess) {
            cudaGetLastError();
            set_err("band allocation of %zu bytes failed", bytes);
            return HICMA_TLR_ERR_OOM;
        }
        A->band_alloc = band_size;
    }
    A->band = band_size;
    TRY(gen_band_tiles(c, A, prob));
    for (int m = 0; m < NT; ++m)
        for (int n = 0; n < NT; ++n)
            if (m < n || m - n < band_size) A->h_rank[(size_t)n * NT + m] = -1;
    CUDA_TRY(cudaMemcpyAsync(A->d_rank, A->h_rank.data(), (size_t)NT * NT * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    A->factored = false;
    return ctx_sync(c);
}

// ------------------------------------------------------- factorization -----
// Copy-out of factor column k (armed by hicma_tlr_store_stream) after `ready`
// on the copy stream, in the stream layout: the band tiles (m, k),
// m = k..min(NT-1, k+band-1), then the packed [U, V] of the off-band tiles
// (m, k), m = k+band..NT-1, with their final ranks.  A column that does not
// fit the buffer stops the copy-out (stats[15] = -1).
static int stream_column(hicma_tlr_ctx *c, hicma_tlr_desc *A, int k, cudaEvent_t ready) {
    if (A->strm_over) return 0;
    const size_t NB = A->NB;
    const int NT = A->NT;
    size_t need = 0;
    for (int m = k; m < NT; ++m)
        need += A->is_dense(m, k) ? NB * NB : 2 * NB * (size_t)std::max(A->rank(m, k), 0);
    if (A->strm_off + need * sizeof(double) > A->strm_cap) {
        A->strm_over = true;
        return 0;
    }
    CUDA_TRY(cudaStreamWaitEvent(c->stream_copy, ready, 0));
    double *p = A->strm_buf + A->strm_off / sizeof(double);
    for (int m = k; m < NT; ++m) {
        if (A->is_dense(m, k)) {
            CUDA_TRY(cudaMemcpyAsync(p, A->dense(m, k), NB * NB * sizeof(double), cudaMemcpyDeviceToHost,
                                     c->stream_copy));
            p += NB * NB;
        } else {
            const int r = A->rank(m, k);
            if (r > 0) {
                CUDA_TRY(cudaMemcpyAsync(p, A->U(m, k), NB * r * sizeof(double), cudaMemcpyDeviceToHost,
                                         c->stream_copy));
                CUDA_TRY(cudaMemcpyAsync(p + NB * r, A->V(m, k), NB * r * sizeof(double), cudaMemcpyDeviceToHost,
                                         c->stream_copy));
                p += 2 * NB * (size_t)r;
            }
        }
    }
    A->strm_off += need * sizeof(double);
    return 0;
}

// SYRK(k, m) for the listed m on the current stream/arena:
// dense T -= A A^T (CORE_dsyrk), low rank T -= U (V^T V) U^T (HCORE_dsyrk),
// HiCMA_dpotrf_L_2flow.jdf:503-565; rank 0 skips (:511-513).
static int run_syrk(hicma_tlr_ctx *c, hicma_tlr_desc *A, int k, const std::vector<int> &ms) {
    const int NB = A->NB;
    const size_t mark = c->ar->off;
    std::vector<GemmTask> g1, g2, g3;
    std::vector<GramTask> gw;
    for (int m : ms) {
        if (A->is_dense(m, k)) {
            g1.push_back(make_gemm(0, 1, NB, NB, NB, -1.0, A->dense(m, k), NB, A->dense(m, k), NB, 1.0,
                                   A->dense(m, m), NB));
            continue;
        }
        const int r = A->rank(m, k);
        if (r == 0) continue;
        double *W = ws_alloc<double>(c, (size_t)r * r);
        double *X = ws_alloc<double>(c, (size_t)NB * r);
        if (!W || !X) {
            TRY(run_gemms(c, g1, false, P_GEMM_SYRK)); TRY(run_grams(c, gw, P_GEMM_SYRK));
            TRY(run_gemms(c, g2, false, P_GEMM_SYRK)); TRY(run_gemms(c, g3, false, P_GEMM_SYRK));
            c->ar->off = mark;
            W = ws_alloc<double>(c, (size_t)r * r);
            X = ws_alloc<double>(c, (size_t)NB * r);
            if (!W || !X) { set_err("workspace too small (syrk)"); return HICMA_TLR_ERR_OOM; }
        }
        // V^T V: an NB-long reduction into r x r (split-K, not one long-K GEMM tile)
        gw.push_back(GramTask{A->V(m, k), A->V(m, k), W, NB, r, r});
        g2.push_back(make_gemm(0, 0, NB, r, r, 1.0, A->U(m, k), NB, W, r, 0.0, X, NB));
        g3.push_back(make_gemm(0, 1, NB, NB, r, -1.0, X, NB, A->U(m, k), NB, 1.0, A->dense(m, m), NB));
    }
    TRY(run_gemms(c, g1, false, P_GEMM_SYRK));
    TRY(run_grams(c, gw, P_GEMM_SYRK));
    TRY(run_gemms(c, g2, false, P_GEMM_SYRK));
    TRY(run_gemms(c, g3, false, P_GEMM_SYRK));
    c->ar->off = mark;
    return 0;
}

// The low-rank SYRK contributions of columns j in [j0, j1) to diagonal tile m
// at once: A_mm -= sum_j U_mj (V_mj^T V_mj) U_mj^T over the off-band tiles
// (m, j).  The factors of column j are final once panel j is done, so
// deferring is exact; applying them as one K-concatenated DMMA GEMM
// (K = sum of the ranks) reads and writes the dense tile once instead of once
// per panel.  The factorization applies columns 0..m-2 one panel early, off the
// critical path, and only column m-1 right before POTRF(m).  Chunked to the
// free workspace.
static int run_syrk_lazy(hicma_tlr_ctx *c, hicma_tlr_desc *A, int m, int j0, int j1) {
    const int NB = A->NB;
    const size_t mark = c->ar->off;
    std::vector<int> js;
    for (int j = j0; j < j1; ++j)
        if (!A->is_dense(m, j) && A->rank(m, j) > 0) js.push_back(j);
    size_t p = 0;
    while (p < js.size()) {
        c->ar->off = mark;
        // columns that fit: per tile r^2 (W) + 2 NB r (Y and U, concatenated)
        size_t q = p, sumr = 0, need = 4096;
        const size_t avail = ws_free(c);
        while (q < js.size()) {
            const size_t r = (size_t)A->rank(m, js[q]);
            const size_t add = align_up(sizeof(double) * r * r + 1) + 2 * sizeof(double) * NB * r;
            if (q > p && need + add + 2 * 256 > avail) break;
            need += add;
            sumr += r;
            ++q;
        }
        double *Yc = ws_alloc<double>(c, (size_t)NB * sumr);
        double *Uc = ws_alloc<double>(c, (size_t)NB * sumr);
        if (!Yc || !Uc) { set_err("workspace too small (syrk, K=%zu)", sumr); return HICMA_TLR_ERR_OOM; }
        std::vector<GramTask> g1;
        std::vector<GemmTask> g2;
        std::vector<CopyTask> cp;
        size_t off = 0;
        for (size_t t = p; t < q; ++t) {
            const int j = js[t], r = A->rank(m, j);
            double *W = ws_alloc<double>(c, (size_t)r * r);
            if (!W) { set_err("workspace too small (syrk)"); return HICMA_TLR_ERR_OOM; }
            g1.push_back(GramTask{A->V(m, j), A->V(m, j), W, NB, r, r});
            g2.push_back(make_gemm(0, 0, NB, r, r, 1.0, A->U(m, j), NB, W, r, 0.0, Yc + off * NB, NB));
            cp.push_back(make_copy(A->U(m, j), NB, Uc + off * NB, NB, NB, r));
            off += r;
        }
        TRY(run_grams(c, g1, P_GEMM_SYRK));
        TRY(run_gemms(c, g2, false, P_GEMM_SYRK));
        TRY(run_copies(c, cp));
        std::vector<GemmTask> g3{make_gemm(0, 1, NB, NB, (int)sumr, -1.0, Yc, NB, Uc, NB, 1.0, A->dense(m, m), NB, 1)};
        TRY(run_gemms(c, g3, false, P_GEMM_SYRK));
        p = q;
    }
    c->ar->off = mark;
    return 0;
}

static unsigned long syrk_ops(const hicma_tlr_desc *A, int k, int m) {
    const unsigned long NB = A->NB;
    if (A->is_dense(m, k)) return op_counts('m', NB, NB, NB, 0);
    const unsigned long r = A->rank(m, k);
    return op_counts('m', r, r, NB, 0) + op_counts('m', NB, r, r, 0) + op_counts('m', NB, NB, r, 0);
}

// Per-panel schedule with a one-panel lookahead: the critical chain
// TRSM(k+1,k) -> SYRK(k,k+1) -> POTRF(k+1) runs on the high-priority stream
// and overlaps the remaining SYRK/GEMM work of panel k on the bulk stream.
static int factorize(hicma_tlr_ctx *c, hicma_tlr_desc *A, double acc, int fixed_rank, int maxrank,
                     unsigned long *tileops, unsigned long *opcounters, double *cpt, int verbose,
                     bool lookahead) {
    const int NT = A->NT, NB = A->NB, band = A->band;
    const bool mixed = c->precision == HICMA_TLR_PREC_MIXED;
    if (!A->d_linv) {
        if (dev_alloc(c, (void **)&A->d_linv, (size_t)NT * NB * NB * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            set_err("allocation of the diagonal inverses failed");
            return HICMA_TLR_ERR_OOM;
        }
    }
    c->cur = c->stream;
    c->ar = &c->main_ar;
    c->main_ar.off = 0;
    c->hi_ar.off = 0;
    A->rk_init.assign((size_t)NT * NT, -1);
    // per diagonal tile: first column whose low-rank SYRK contribution is not yet applied
    std::vector<int> syrk_from(NT, 0);
    for (int n = 0; n < NT; ++n)
        for (int m = n + band; m < NT; ++m) A->rk_init[(size_t)n * NT + m] = A->rank(m, n);
    A->rk_min = A->rk_init;
    A->rk_max = A->rk_init;
    CUDA_TRY(cudaMemsetAsync(c->d_flags, 0, 7 * sizeof(int), c->stream));
    TRY(ctx_sync(c));
    int *d_info = c->d_flags;
    int *rtask = ws_alloc<int>(c, (size_t)NT * NT + 16);
    if (!rtask) { set_err("workspace too small"); return HICMA_TLR_ERR_OOM; }
    // precision policy: squared Frobenius norms of the low-rank tiles of the
    // current panel column, and the product-norm bound under which the FP32
    // rounding of a product (about sqrt(NB) 2^-24 ||A|| ||B||) stays below acc/100
    double *d_fro2 = mixed ? ws_alloc<double>(c, (size_t)NT + 16) : nullptr;
    if (mixed && !d_fro2) { set_err("workspace too small"); return HICMA_TLR_ERR_OOM; }
    const double thr = 0.01 * acc / (std::sqrt((double)NB) * 5.9604644775390625e-8);
    const double thr2 = mixed ? thr * thr : 0.0;
    const size_t base_mark = c->ar->off;
    std::vector<unsigned long> tops((size_t)NT * NT, 0);
    unsigned long op_total = 0;
    enum { P0, P1, T0, T1, S0, S1, G0, G1, NEV };
    cudaEvent_t ev[NEV], evP, evT, evEnd;
    CUDA_TRY(cudaEventCreate(&evEnd));
    double t_gap = 0.0;      // device idle between a panel's last kernel and the next panel's first
    bool have_end = false;
    for (auto &e : ev) CUDA_TRY(cudaEventCreate(&e));
    CUDA_TRY(cudaEventCreateWithFlags(&evP, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&evT, cudaEventDisableTiming));
    double t_phase[4] = {0, 0, 0, 0};
    const auto t_start = std::chrono::steady_clock::now();
    const long long launches0 = c->launches;
    int info = 0;
    // ops of the critical path POTRF(k) -> TRSM(k+1,k) -> SYRK(k,k+1) (the
    // reference's op_path, HiCMA_dpotrf_L_2flow.jdf:201,303-313,443-462)
    unsigned long op_path = 0;
    double jac_fl = 0.0, jac_n = 0.0;   // Jacobi flops per sweep summed over the cores, and their number
    long long khist[16] = {0};          // recompressions by stacked rank K = rc + ra, in steps of 16 (verbose > 2)
    double t_last = 0.0;   // wall time of the previous panel's end (verbose > 1)
    auto log_op = [&](unsigned long cnt, int i, int j, bool path = false) {
        tops[(size_t)i * NT + j] += cnt;
        op_total += cnt;
        if (path) op_path += cnt;
    };
    auto elapsed = [&](cudaEvent_t a, cudaEvent_t b) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        return ms * 1e-3;
    };
    // POTRF(0)
    {
        OnHi h(c);
        c->ar->off = 0;
        CUDA_TRY(cudaEventRecord(ev[P0], c->cur));
        TRY(potrf_tile(c, A->dense(0, 0), NB, NB, A->linv(0), NB, d_info, 0));
        CUDA_TRY(cudaEventRecord(ev[P1], c->cur));
        CUDA_TRY(cudaEventRecord(evP, c->cur));
    }
    log_op(op_counts('c', NB, 0, 0, 0), 0, 0, true);
    CUDA_TRY(cudaEventSynchronize(ev[P1]));
    t_phase[0] += elapsed(ev[P0], ev[P1]);
    for (int k = 0; k < NT; ++k) {
        NvtxRange nv_panel("panel");
        const double *Li = A->linv(k);
        CUDA_TRY(cudaStreamWaitEvent(c->stream, evP, 0));
        // ---- TRSM(m, k): dense C <- C L^-T ; low rank V <- L^-1 V (:366-401)
        CUDA_TRY(cudaEventRecord(ev[T0], c->stream));
        if (have_end) {
            // the previous panel ended (both streams) before the host returned from
            // its synchronisation, so this gap is the device idle time between panels
            CUDA_TRY(cudaEventSynchronize(ev[T0]));
            t_gap += elapsed(evEnd, ev[T0]);
        }
        {
            NvtxRange nv("TRSM");
            c->ar->off = base_mark;
            std::vector<GemmTask> g;
            std::vector<CopyTask> cp;
            // low-rank tiles below TRSM(k+1, k): their V factors are gathered side by
            // side into one NB x sum(r) block, so the solve is one wide product
            // L^-1 [V_m ...] (the triangle bounds each output tile's inner dimension)
            // instead of one skinny product per tile, then scattered back
            std::vector<std::pair<int, int>> lr;
            size_t sumr = 0;
            // arena bytes of the gathered block and its product for w columns
            auto lr_need = [&](size_t w) { return w ? 2 * align_up(sizeof(double) * NB * w + 1) : 0; };
            auto flush = [&]() -> int {
                TRY(run_gemms(c, g, false, P_GEMM_TRSM));
                TRY(run_copies(c, cp));
                if (!lr.empty()) {
                    double *Vc = ws_alloc<double>(c, (size_t)NB * sumr), *Tc = ws_alloc<double>(c, (size_t)NB * sumr);
                    if (!Vc || !Tc) { set_err("workspace too small (trsm, %zu columns)", sumr); return HICMA_TLR_ERR_OOM; }
                    std::vector<CopyTask> gat, sct;
                    size_t off = 0;
                    for (const auto &mr : lr) {
                        gat.push_back(make_copy(A->V(mr.first, k), NB, Vc + off * NB, NB, NB, mr.second));
                        sct.push_back(make_copy(Tc + off * NB, NB, A->V(mr.first, k), NB, NB, mr.second));
                        off += (size_t)mr.second;
                    }
                    TRY(run_copies(c, gat));
                    std::vector<GemmTask> one{make_gemm(0, 0, NB, (int)sumr, NB, 1.0, Li, NB, Vc, NB, 0.0, Tc, NB)};
                    one.back().tri = 1;
                    TRY(run_gemms(c, one, false, P_GEMM_TRSM));
                    TRY(run_copies(c, sct));
                    lr.clear();
                    sumr = 0;
                }
                c->ar->off = base_mark;
                return 0;
            };
            for (int m = k + 1; m < NT; ++m) {
                if (m == k + 2) {
                    // TRSM(k+1, k) is all the critical chain SYRK(k, k+1) -> POTRF(k+1)
                    // needs: it goes first, on its own, and releases the chain
                    TRY(flush());
                    CUDA_TRY(cudaEventRecord(evT, c->stream));
                }
                const bool dense = A->is_dense(m, k);
                const int r = dense ? NB : A->rank(m, k);
                log_op(op_counts('t', NB, r, 1, 0), m, k, m == k + 1);
                if (r == 0) continue;
                if (!dense && m > k + 1) {
                    // the pending block grows by r columns: flush first if it would not fit
                    if (lr_need(sumr + r) > ws_free(c)) {
                        TRY(flush());
                        if (lr_need(r) > ws_free(c)) { set_err("workspace too small (trsm)"); return HICMA_TLR_ERR_OOM; }
                    }
                    lr.push_back({m, r});
                    sumr += (size_t)r;
                    continue;
                }
                // a per-tile product: its output and the pending block must both fit
                if (align_up(sizeof(double) * NB * (size_t)r + 1) + lr_need(sumr) > ws_free(c)) TRY(flush());
                double *tmp = ws_alloc<double>(c, (size_t)NB * r);
                if (!tmp) { set_err("workspace too small (trsm)"); return HICMA_TLR_ERR_OOM; }
                // L^-1 is lower triangular with zeros above the diagonal: each output
                // tile runs its inner dimension only as far as L^-1 has entries
                if (dense) {
                    g.push_back(make_gemm(0, 1, NB, NB, NB, 1.0, A->dense(m, k), NB, Li, NB, 0.0, tmp, NB));
                    g.back().tri = 2;
                    cp.push_back(make_copy(tmp, NB, A->dense(m, k), NB, NB, NB));
                } else {
                    g.push_back(make_gemm(0, 0, NB, r, NB, 1.0, Li, NB, A->V(m, k), NB, 0.0, tmp, NB));
                    g.back().tri = 1;
                    cp.push_back(make_copy(tmp, NB, A->V(m, k), NB, NB, r));
                }
            }
            TRY(flush());
            if (mixed) {
                std::vector<NormTask> nt;
                for (int m = k + 1; m < NT; ++m)
                    if (!A->is_dense(m, k)) nt.push_back(NormTask{A->V(m, k), NB, A->rank(m, k), NB, d_fro2 + m});
                if (!nt.empty()) {
                    TRY(bc_norms(nt));
                    NormTask *d = stage(c, nt.data(), nt.size());
                    if (!d) { set_err("staging failed"); return HICMA_TLR_ERR_CUDA; }
                    launch_sumsq_batched(d, (int)nt.size(), c->stream);
                    TRY(check_launch(c));
                }
            }
        }
        CUDA_TRY(cudaEventRecord(ev[T1], c->stream));
        if (k + 2 >= NT) CUDA_TRY(cudaEventRecord(evT, c->stream));
        // column k of the factor is final (POTRF(k) and its TRSMs are done): copy it
        // out on the copy stream while the later panels run
        if (A->strm_buf) TRY(stream_column(c, A, k, ev[T1]));
        std::vector<RecompTask> rec;
        std::vector<int> rec_case;
        std::vector<std::array<int, 5>> rec_meta;
        if (k + 1 < NT) {
            // ---- critical chain: SYRK(k, k+1) + POTRF(k+1)
            log_op(syrk_ops(A, k, k + 1), k + 1, k + 1, true);
            log_op(op_counts('c', NB, 0, 0, 0), k + 1, k + 1, true);
            {
                OnHi h(c);
                NvtxRange nv("SYRK+POTRF(k+1)");
                if (!lookahead) c->cur = c->stream;
                c->ar->off = 0;
                CUDA_TRY(cudaStreamWaitEvent(c->cur, evT, 0));
                if (A->is_dense(k + 1, k)) TRY(run_syrk(c, A, k, std::vector<int>{k + 1}));
                TRY(run_syrk_lazy(c, A, k + 1, syrk_from[k + 1], k + 1));
                syrk_from[k + 1] = k + 1;
                CUDA_TRY(cudaEventRecord(ev[P0], c->cur));
                TRY(potrf_tile(c, A->dense(k + 1, k + 1), NB, NB, A->linv(k + 1), NB, d_info, (k + 1) * NB));
                CUDA_TRY(cudaEventRecord(ev[P1], c->cur));
                CUDA_TRY(cudaEventRecord(evP, c->cur));
                // the next diagonal tile's low-rank contributions of columns 0..k (all
                // final once this panel's whole TRSM is done: the chain waited only for
                // TRSM(k+1,k), so it waits for the rest, T1, here), after POTRF(k+1)
                // and behind the event the bulk stream waits on: they overlap this
                // panel's updates, and the next panel's chain adds only column k+1's.
                // (With a band of 3 or more the bulk stream's dense SYRK writes the
                // same tile: left to the chain.)
                if (k + 2 < NT && A->band <= 2) {
                    CUDA_TRY(cudaStreamWaitEvent(c->cur, ev[T1], 0));
                    c->ar->off = 0;
                    TRY(run_syrk_lazy(c, A, k + 2, syrk_from[k + 2], k + 1));
                    syrk_from[k + 2] = k + 1;
                }
            }
            // ---- SYRK(k, m), m > k+1
            NvtxRange nv_syrk("SYRK");
            CUDA_TRY(cudaEventRecord(ev[S0], c->stream));
            c->ar->off = base_mark;
            std::vector<int> ms;
            for (int m = k + 2; m < NT; ++m) {
                // low-rank contributions are applied lazily before POTRF(m)
                if (A->is_dense(m, k)) ms.push_back(m);
                log_op(syrk_ops(A, k, m), m, m);
            }
            TRY(run_syrk(c, A, k, ms));
            CUDA_TRY(cudaEventRecord(ev[S1], c->stream));
            nv_syrk.end();
            // ---- GEMM(m, n, k) (:699-1097)
            NvtxRange nv_gemm("GEMM");
            CUDA_TRY(cudaEventRecord(ev[G0], c->stream));
            c->ar->off = base_mark;
            std::vector<GemmTask> g1, g2, g3;
            for (int m = k + 2; m < NT; ++m) {
                for (int n = k + 1; n < m; ++n) {
                    if (m - k < band) {                                    // (i)
                        log_op(op_counts('m', NB, NB, NB, 0), m, n);
                        g1.push_back(make_gemm(0, 1, NB, NB, NB, -1.0, A->dense(m, k), NB, A->dense(n, k), NB, 1.0,
                                               A->dense(m, n), NB));
                    } else if (n - k < band && m - n < band) {             // (ii)
                        const int ra = A->rank(m, k);
                        log_op(op_counts('m', NB, NB, ra, 0) * 2, m, n);
                        if (ra == 0) continue;
                        double *tmp = ws_alloc<double>(c, (size_t)ra * NB);
                        if (!tmp) {
                            TRY(run_gemms(c, g1, false, P_GEMM_DENSE)); TRY(run_gemms(c, g2, false, P_GEMM_DENSE)); TRY(run_gemms(c, g3, false, P_GEMM_DENSE));
                            c->ar->off = base_mark;
                            tmp = ws_alloc<double>(c, (size_t)ra * NB);
                            if (!tmp) { set_err("workspace too small (gemm)"); return HICMA_TLR_ERR_OOM; }
                        }
                        g1.push_back(make_gemm(1, 1, ra, NB, NB, 1.0, A->V(m, k), NB, A->dense(n, k), NB, 0.0, tmp, ra));
                        g2.push_back(make_gemm(0, 0, NB, NB, ra, -1.0, A->U(m, k), NB, tmp, ra, 1.0, A->dense(m, n), NB));
                    } else if (m - n < band) {                             // (iii)
                        const int ra = A->rank(m, k), rb = A->rank(n, k);
                        log_op(op_counts('m', NB, NB, std::min(ra, rb), 0) + op_counts('m', NB, ra, rb, 0) * 2, m, n);
                        if (ra == 0 || rb == 0) continue;
                        double *rr = ws_alloc<double>(c, (size_t)ra * rb);
                        double *tmp = ws_alloc<double>(c, (size_t)NB * std::max(ra, rb));
                        if (!rr || !tmp) {
                            TRY(run_gemms(c, g1, false, P_GEMM_DENSE)); TRY(run_gemms(c, g2, false, P_GEMM_DENSE)); TRY(run_gemms(c, g3, false, P_GEMM_DENSE));
                            c->ar->off = base_mark;
                            rr = ws_alloc<double>(c, (size_t)ra * rb);
                            tmp = ws_alloc<double>(c, (size_t)NB * std::max(ra, rb));
                            if (!rr || !tmp) { set_err("workspace too small (gemm)"); return HICMA_TLR_ERR_OOM; }
                        }
                        g1.push_back(make_gemm(1, 0, ra, rb, NB, 1.0, A->V(m, k), NB, A->V(n, k), NB, 0.0, rr, ra));
                        if (ra > rb) {
                            g2.push_back(make_gemm(0, 0, NB, rb, ra, 1.0, A->U(m, k), NB, rr, ra, 0.0, tmp, NB));
                            g3.push_back(make_gemm(0, 1, NB, NB, rb, -1.0, tmp, NB, A->U(n, k), NB, 1.0, A->dense(m, n), NB));
                        } else {
                            g2.push_back(make_gemm(0, 1, ra, NB, rb, 1.0, rr, ra, A->U(n, k), NB, 0.0, tmp, ra));
                            g3.push_back(make_gemm(0, 0, NB, NB, ra, -1.0, A->U(m, k), NB, tmp, ra, 1.0, A->dense(m, n), NB));
                        }
                    } else if (n - k < band) {                             // (iv)
                        const int ra = A->rank(m, k), rc = A->rank(m, n);
                        rec.push_back(RecompTask{A->U(m, n), A->V(m, n), rc, A->U(m, k), A->V(m, k), ra,
                                                 A->dense(n, k), nullptr, NB, A->U(m, n), A->V(m, n),
                                                 A->d_rank + (size_t)n * NT + m});
                        rec_meta.push_back({m, n, ra, 0, rc});
                        rec_case.push_back(1);
                    } else {                                               // (v)
                        const int ra = A->rank(m, k), rb = A->rank(n, k), rc = A->rank(m, n);
                        if (ra == 0 || rb == 0) continue;
                        rec.push_back(RecompTask{A->U(m, n), A->V(m, n), rc, A->U(m, k), A->V(m, k), ra,
                                                 A->U(n, k), A->V(n, k), rb, A->U(m, n), A->V(m, n),
                                                 A->d_rank + (size_t)n * NT + m,
                                                 mixed ? d_fro2 + m : nullptr, mixed ? d_fro2 + n : nullptr});
                        rec_meta.push_back({m, n, ra, rb, rc});
                        rec_case.push_back(0);
                    }
                }
            }
            TRY(run_gemms(c, g1, false, P_GEMM_DENSE));
            TRY(run_gemms(c, g2, false, P_GEMM_DENSE));
            TRY(run_gemms(c, g3, false, P_GEMM_DENSE));
            c->ar->off = base_mark;
            TRY(run_recompress(c, NB, rec, acc, maxrank, fixed_rank, rtask, thr2));
            CUDA_TRY(cudaEventRecord(ev[G1], c->stream));
        }
        // ---- panel end: info, ranks, timings
        CUDA_TRY(cudaStreamWaitEvent(c->stream, evP, 0));
        CUDA_TRY(cudaEventRecord(evEnd, c->stream));
        have_end = true;
        TRY(ctx_sync(c));
        int hinfo = 0;
        CUDA_TRY(xfer(c, &hinfo, d_info, sizeof(int), cudaMemcpyDeviceToHost));
        if (!rec.empty()) {
            CUDA_TRY(xfer(c, A->h_rank.data(), A->d_rank, (size_t)NT * NT * sizeof(int), cudaMemcpyDeviceToHost));
            // each tile takes at most one update per panel, so per-panel minima
            // and maxima are the per-update ones of the reference
            for (const auto &mt : rec_meta) {
                const size_t i = (size_t)mt[1] * NT + mt[0];
                A->rk_min[i] = std::min(A->rk_min[i], A->h_rank[i]);
                A->rk_max[i] = std::max(A->rk_max[i], A->h_rank[i]);
            }
        }
        for (size_t i = 0; i < rec.size(); ++i) {
            const auto &mt = rec_meta[i];
            const int rn = A->rank(mt[0], mt[1]);
            ++khist[std::min(15, (mt[2] + mt[4]) / 16)];
            log_op(gemm_lr_ops(NB, mt[2], mt[3], mt[4], rn, rec_case[i] == 1), mt[0], mt[1]);
            if (c->prof) {
                // algorithmic flops of the kernels whose work depends on the new
                // rank (known once the panel is done): the core (M = R_U R_V^T,
                // pivoted QR stopped at the rank, Jacobi sweeps counted at the end)
                // and the Q application of the U side (ra reflectors on rn columns)
                const double K = mt[2] + mt[4], k = rn, ra = mt[2];
                c->prof_acc[P_CORE][2] += K * K * K / 3.0 + 4.0 * K * K * k - 4.0 * K * k * k + 4.0 / 3.0 * k * k * k;
                jac_fl += 6.0 * K * k * k;
                ++jac_n;
                if (ra > 0) c->prof_acc[P_QAPPLY][2] += 4.0 * NB * ra * k;
            }
        }
        t_phase[1] += elapsed(ev[T0], ev[T1]);
        if (k + 1 < NT) {
            t_phase[0] += elapsed(ev[P0], ev[P1]);
            t_phase[2] += elapsed(ev[S0], ev[S1]);
            t_phase[3] += elapsed(ev[G0], ev[G1]);
        }
        if (hinfo != 0) {
            info = hinfo;
            if (verbose) fprintf(stderr, "dpotrf failed: info = %d (panel %d)\n", info, k);
            break;
        }
        if (verbose > 1) {
            const double now = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
            fprintf(stderr, "panel %3d wall %8.3f ms trsm %7.3f syrk %7.3f gemm %7.3f potrf(k+1) %7.3f tasks %zu\n", k,
                    (now - t_last) * 1e3, elapsed(ev[T0], ev[T1]) * 1e3,
                    k + 1 < NT ? elapsed(ev[S0], ev[S1]) * 1e3 : 0.0, k + 1 < NT ? elapsed(ev[G0], ev[G1]) * 1e3 : 0.0,
                    k + 1 < NT ? elapsed(ev[P0], ev[P1]) * 1e3 : 0.0, rec.size());
            t_last = now;
        }
    }
    if (verbose > 2) {
        fprintf(stderr, "recompressions by stacked rank K (bins of 16):");
        for (int i = 0; i < 16; ++i) fprintf(stderr, " %lld", khist[i]);
        fprintf(stderr, "\n");
    }
    for (auto &e : ev) cudaEventDestroy(e);
    cudaEventDestroy(evP);
    cudaEventDestroy(evT);
    cudaEventDestroy(evEnd);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    int flags_h[7] = {0, 0, 0, 0, 0, 0, 0};
    CUDA_TRY(xfer(c, flags_h, c->d_flags, 7 * sizeof(int), cudaMemcpyDeviceToHost));
    if (flags_h[3]) {
        xclear(c, c->d_flags + 3, sizeof(int));
        set_err("a bounded device wait gave up (tile POTRF task queue)");
        return HICMA_TLR_ERR_TIMEOUT;
    }
    const int overflow = flags_h[1];
    // Jacobi work: the sweeps counted on the device times the mean work of a sweep
    if (c->prof && jac_n > 0) c->prof_acc[P_CORE][2] += (double)flags_h[2] * jac_fl / jac_n;
    A->stats[8] = flags_h[2];
    A->stats[9] = flags_h[4];
    if (tileops)
        for (size_t i = 0; i < tops.size(); ++i) tileops[i] += tops[i];
    if (opcounters) opcounters[0] += op_total;
    if (cpt) {
        cpt[0] = t_phase[0]; cpt[1] = t_phase[1]; cpt[2] = t_phase[2];
        cpt[3] = secs; cpt[4] = t_phase[1] + t_phase[2] + t_phase[3]; cpt[5] = t_phase[3];
    }
    A->stats[0] = secs;
    A->stats[1] = (double)op_total;
    A->stats[2] = overflow;
    A->stats[3] = (double)(c->launches - launches0);
    A->stats[4] = t_phase[0]; A->stats[5] = t_phase[1]; A->stats[6] = t_phase[2]; A->stats[7] = t_phase[3];
    A->stats[10] = (double)op_path;
    A->stats[11] = flags_h[5];
    A->stats[12] = t_gap;
    A->stats[13] = NT;
    A->stats[14] = flags_h[6];
    A->stats[15] = A->strm_buf ? (A->strm_over ? -1.0 : (double)A->strm_off) : 0.0;
    A->strm_buf = nullptr;   // the arming is used by one factorization
    A->factored = (info == 0);
    c->main_ar.off = 0;
    c->hi_ar.off = 0;
    return info;
}

int hicma_tlr_dpotrf_L(hicma_tlr_ctx *c, int uplo, hicma_tlr_desc *A, int *Ar, double acc, int fixed_rank,
                       int maxrank, int *lookahead, int band_size, int hmb, int compmaxrank, int send_full_tile,
                       int *two_flow, unsigned long *tileopcounters, unsigned long *opcounters,
                       double *critical_path_time, int verbose) {
    (void)hmb; (void)send_full_tile;
    ARG_CHECK(c && A, "null");
    // HiCMA_dpotrf_L_2flow_wrapper.c:219-237
    if (uplo != HICMA_TLR_LOWER) { set_err("HiCMA_dpotrf_L_2flow does not support dplasmaUpper"); return HICMA_TLR_ERR_NOT_SUPPORTED; }
    if (compmaxrank <= 0) compmaxrank = maxrank;
    ARG_CHECK(maxrank <= compmaxrank, "maxrank for storage larger than maxrank for buffers is not meaningful");
    ARG_CHECK(maxrank <= A->NB / 2, "maxrank should not be larger than half of block size");
    ARG_CHECK(maxrank <= A->maxrank, "maxrank larger than the descriptor's slot capacity");
    ARG_CHECK(band_size == A->band, "band_size must equal the descriptor's band size");
    ARG_CHECK(acc > 0.0 || fixed_rank > 0, "acc > 0 or fixed_rank > 0");
    if (lookahead) {
        ARG_CHECK(*lookahead >= -1, "lookahead >= -1");
        if (*lookahead == -1) *lookahead = band_size;   // hicma_parsec.c:489-495
    }
    // The reference runs its 3-flow graph when band_size == 1 and 2-flow is not
    // forced, leaving *two_flow at 0, and sets it to 1 otherwise
    // (hicma_parsec.c:517-573).  At band 1 the 3-flow graph computes the same
    // updates, so both are served by this path; *two_flow reports which one
    // the reference would have run.
    if (two_flow && (band_size != 1 || *two_flow)) *two_flow = 1;
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    NvtxRange nv("HiCMA_dpotrf_L");
    CUDA_TRY(cudaSetDevice(c->device));
    const bool la = !(lookahead && *lookahead == 0);
    const int info = factorize(c, A, acc, fixed_rank, maxrank, tileopcounters, opcounters, critical_path_time, verbose, la);
    if (Ar) std::memcpy(Ar, A->h_rank.data(), (size_t)A->NT * A->NT * sizeof(int));
    return info;
}

int hicma_tlr_dpotrf_L_start(hicma_tlr_ctx *c, hicma_tlr_desc *A, double acc, int fixed_rank, int maxrank) {
    ARG_CHECK(c && A, "null");
    if (c->async_thread.joinable()) { set_err("a factorization is already in flight on this context"); return HICMA_TLR_ERR_STATE; }
    c->async_thread = std::thread([=]() {
        int la = -1, tf = 0;
        c->async_ret = hicma_tlr_dpotrf_L(c, HICMA_TLR_LOWER, A, nullptr, acc, fixed_rank, maxrank, &la, A->band, A->NB,
                                          maxrank, 0, &tf, nullptr, nullptr, nullptr, 0);
        c->async_err = c->async_ret < 0 ? hicma_tlr_last_error() : "";
    });
    return 0;
}

int hicma_tlr_dpotrf_L_wait(hicma_tlr_ctx *c, hicma_tlr_desc *A, int *Ar) {
    ARG_CHECK(c && A, "null");
    if (!c->async_thread.joinable()) { set_err("no factorization in flight"); return HICMA_TLR_ERR_STATE; }
    c->async_thread.join();
    if (c->async_ret < 0) {
        set_err("%s", c->async_err.c_str());   // the message was set on the background thread
        return c->async_ret;
    }
    if (Ar) std::memcpy(Ar, A->h_rank.data(), (size_t)A->NT * A->NT * sizeof(int));
    return c->async_ret;
}

int hicma_tlr_last_stats(hicma_tlr_desc *A, double *stats, int nstats) {
    ARG_CHECK(A && stats, "null");
    for (int i = 0; i < nstats && i < 16; ++i) stats[i] = A->stats[i];
    return 0;
}

// ------------------------------------------------------------ transfers ----
int hicma_tlr_tile_get(hicma_tlr_ctx *c, hicma_tlr_desc *A, int m, int n, double *buf, int *rank) {
    ARG_CHECK(c && A, "null");
    ARG_CHECK(m >= 0 && n >= 0 && m < A->NT && n <= m, "tile index (lower triangle only)");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    const size_t NB = A->NB;
    TRY(ctx_sync(c));
    if (A->is_dense(m, n)) {
        if (rank) *rank = -1;
        if (buf) CUDA_TRY(xfer(c, buf, A->dense(m, n), NB * NB * sizeof(double), cudaMemcpyDeviceToHost));
        return 0;
    }
    const int r = A->rank(m, n);
    if (rank) *rank = r;
    if (buf && r > 0) {
        CUDA_TRY(xfer(c, buf, A->U(m, n), NB * r * sizeof(double), cudaMemcpyDeviceToHost));
        CUDA_TRY(xfer(c, buf + NB * r, A->V(m, n), NB * r * sizeof(double), cudaMemcpyDeviceToHost));
    }
    return 0;
}

int hicma_tlr_tile_set(hicma_tlr_ctx *c, hicma_tlr_desc *A, int m, int n, const double *buf, int rank) {
    ARG_CHECK(c && A && buf, "null");
    ARG_CHECK(m >= 0 && n >= 0 && m < A->NT && n <= m, "tile index (lower triangle only)");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    const size_t NB = A->NB, NT = A->NT;
    TRY(ctx_sync(c));
    if (A->is_dense(m, n)) {
        CUDA_TRY(xfer(c, A->dense(m, n), buf, NB * NB * sizeof(double), cudaMemcpyHostToDevice));
        A->factored = false;   // the held factor no longer belongs to this matrix
        return 0;
    }
    ARG_CHECK(rank >= 0 && rank <= A->maxrank, "rank in [0, maxrank]");
    if (rank > 0) {
        CUDA_TRY(xfer(c, A->U(m, n), buf, NB * rank * sizeof(double), cudaMemcpyHostToDevice));
        CUDA_TRY(xfer(c, A->V(m, n), buf + NB * rank, NB * rank * sizeof(double), cudaMemcpyHostToDevice));
    }
    A->h_rank[(size_t)n * NT + m] = rank;
    CUDA_TRY(xfer(c, A->d_rank + (size_t)n * NT + m, &rank, sizeof(int), cudaMemcpyHostToDevice));
    A->factored = false;
    return 0;
}

int hicma_tlr_store_bytes(hicma_tlr_ctx *c, hicma_tlr_desc *A, size_t *bytes) {
    ARG_CHECK(c && A && bytes, "null");
    const size_t NB = A->NB;
    size_t b = 0;
    for (int m = 0; m < A->NT; ++m)
        for (int n = 0; n <= m; ++n)
            b += A->is_dense(m, n) ? NB * NB : 2 * NB * (size_t)A->rank(m, n);
    *bytes = b * sizeof(double);
    return 0;
}

int hicma_tlr_store_get(hicma_tlr_ctx *c, hicma_tlr_desc *A, double *buf, int *Ar) {
    ARG_CHECK(c && A && buf, "null");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    const size_t NB = A->NB;
    TRY(ctx_sync(c));
    double *p = buf;
    for (int m = 0; m < A->NT; ++m)
        for (int n = std::max(0, m - A->band + 1); n <= m; ++n) {
            CUDA_TRY(cudaMemcpyAsync(p, A->dense(m, n), NB * NB * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
            p += NB * NB;
        }
    for (int m = A->band; m < A->NT; ++m)
        for (int n = 0; n <= m - A->band; ++n) {
            const int r = A->rank(m, n);
            if (r > 0) {
                CUDA_TRY(cudaMemcpyAsync(p, A->U(m, n), NB * r * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
                CUDA_TRY(cudaMemcpyAsync(p + NB * r, A->V(m, n), NB * r * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
            }
            p += 2 * NB * (size_t)r;
        }
    if (Ar) std::memcpy(Ar, A->h_rank.data(), (size_t)A->NT * A->NT * sizeof(int));
    return ctx_sync(c);
}

int hicma_tlr_store_set(hicma_tlr_ctx *c, hicma_tlr_desc *A, const double *buf, const int *Ar) {
    ARG_CHECK(c && A && buf && Ar, "null");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    const size_t NB = A->NB, NT = A->NT;
    TRY(ctx_sync(c));
    for (int m = A->band; m < A->NT; ++m)
        for (int n = 0; n <= m - A->band; ++n)
            ARG_CHECK(Ar[(size_t)n * NT + m] >= 0 && Ar[(size_t)n * NT + m] <= A->maxrank, "rank out of range");
    const double *p = buf;
    for (int m = 0; m < A->NT; ++m)
        for (int n = std::max(0, m - A->band + 1); n <= m; ++n) {
            CUDA_TRY(cudaMemcpyAsync(A->dense(m, n), p, NB * NB * sizeof(double), cudaMemcpyHostToDevice, c->stream));
            p += NB * NB;
        }
    for (int m = A->band; m < A->NT; ++m)
        for (int n = 0; n <= m - A->band; ++n) {
            const int r = Ar[(size_t)n * NT + m];
            if (r > 0) {
                CUDA_TRY(cudaMemcpyAsync(A->U(m, n), p, NB * r * sizeof(double), cudaMemcpyHostToDevice, c->stream));
                CUDA_TRY(cudaMemcpyAsync(A->V(m, n), p + NB * r, NB * r * sizeof(double), cudaMemcpyHostToDevice, c->stream));
            }
            p += 2 * NB * (size_t)r;
        }
    for (int m = 0; m < A->NT; ++m)
        for (int n = 0; n < A->NT; ++n)
            A->h_rank[(size_t)n * NT + m] = (m < n || A->is_dense(m, n)) ? -1 : Ar[(size_t)n * NT + m];
    CUDA_TRY(cudaMemcpyAsync(A->d_rank, A->h_rank.data(), NT * NT * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    A->factored = false;
    return ctx_sync(c);
}

int hicma_tlr_store_stream(hicma_tlr_ctx *c, hicma_tlr_desc *A, double *buf, size_t bytes) {
    ARG_CHECK(c && A, "null");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    A->strm_buf = buf;
    A->strm_cap = buf ? bytes : 0;
    A->strm_off = 0;
    A->strm_over = false;
    return 0;
}

int hicma_tlr_uncompress(hicma_tlr_ctx *c, hicma_tlr_desc *A, double *dense, long ld) {
    ARG_CHECK(c && A && dense && ld >= A->N, "null or ld < N");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    const int NT = A->NT, NB = A->NB;
    TRY(ctx_sync(c));
    ws_reset(c);
    double *tmp = ws_alloc<double>(c, (size_t)NB * NB);
    if (!tmp) { set_err("workspace too small"); return HICMA_TLR_ERR_OOM; }
    std::vector<double> h((size_t)NB * NB);
    for (int n = 0; n < NT; ++n)
        for (int m = 0; m < NT; ++m) {
            if (m < n) {
                for (int j = 0; j < NB; ++j)
                    std::memset(dense + (size_t)(n * NB + j) * ld + (size_t)m * NB, 0, sizeof(double) * NB);
                continue;
            }
            const double *src;
            if (A->is_dense(m, n)) {
                src = A->dense(m, n);
            } else {
                const int r = A->rank(m, n);
                launch_gemm_single(make_gemm(0, 1, NB, NB, r, 1.0, A->U(m, n), NB, A->V(m, n), NB, 0.0, tmp, NB), c->stream);
                TRY(check_launch(c));
                src = tmp;
            }
            CUDA_TRY(cudaMemcpy2DAsync(dense + (size_t)(n * NB) * ld + (size_t)m * NB, ld * sizeof(double), src,
                                       NB * sizeof(double), NB * sizeof(double), NB, cudaMemcpyDeviceToHost, c->stream));
            TRY(ctx_sync(c));
            if (m == n)
                for (int j = 0; j < NB; ++j)
                    for (int i = 0; i < j; ++i) dense[(size_t)(n * NB + j) * ld + (size_t)m * NB + i] = 0.0;
        }
    ws_reset(c);
    return 0;
}

// --------------------------------------------------- log-det and solves ----
int hicma_tlr_logdet(hicma_tlr_ctx *c, hicma_tlr_desc *A, double *logdet) {
    ARG_CHECK(c && A && logdet, "null");
    if (!A->factored) { set_err("descriptor is not factored"); return HICMA_TLR_ERR_STATE; }
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    std::vector<const double *> ptrs(A->NT);
    for (int k = 0; k < A->NT; ++k) ptrs[k] = A->dense(k, k);
    const double **dp = stage(c, ptrs.data(), ptrs.size());
    if (!dp) { set_err("staging failed"); return HICMA_TLR_ERR_CUDA; }
    launch_logdiag_sum(dp, A->NT, A->NB, A->NB, c->d_scal, c->stream);
    TRY(check_launch(c));
    CUDA_TRY(cudaMemcpyAsync(logdet, c->d_scal, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return ctx_sync(c);
}

// Forward (L z = b) then backward (L^T x = z) substitution over tiles with
// the stored L_kk^-1; off-diagonal updates of one step are batched.
static int solve_dev(hicma_tlr_ctx *c, hicma_tlr_desc *A, double *X, int nrhs) {
    const int NT = A->NT, NB = A->NB;
    const size_t N = A->N;
    double *tmp = ws_alloc<double>(c, (size_t)NB * nrhs);
    double *T2 = ws_alloc<double>(c, (size_t)NT * A->maxrank * nrhs + 1);
    if (!tmp || !T2) { set_err("workspace too small (solve)"); return HICMA_TLR_ERR_OOM; }
    std::vector<GemmTask> g1, g2;
    std::vector<CopyTask> cp;
    for (int k = 0; k < NT; ++k) {
        double *xk = X + (size_t)k * NB;
        g1.push_back(make_gemm(0, 0, NB, nrhs, NB, 1.0, A->linv(k), NB, xk, (int)N, 0.0, tmp, NB));
        g1.back().tri = 1;   // L^-1 lower triangular
        TRY(run_gemms(c, g1));
        cp.push_back(make_copy(tmp, NB, xk, (int)N, NB, nrhs));
        TRY(run_copies(c, cp));
        for (int m = k + 1; m < NT; ++m) {
            double *xm = X + (size_t)m * NB;
            if (A->is_dense(m, k)) {
                g2.push_back(make_gemm(0, 0, NB, nrhs, NB, -1.0, A->dense(m, k), NB, xk, (int)N, 1.0, xm, (int)N));
            } else {
                const int r = A->rank(m, k);
                if (r == 0) continue;
                double *t = T2 + (size_t)m * A->maxrank * nrhs;
                g1.push_back(make_gemm(1, 0, r, nrhs, NB, 1.0, A->V(m, k), NB, xk, (int)N, 0.0, t, r));
                g2.push_back(make_gemm(0, 0, NB, nrhs, r, -1.0, A->U(m, k), NB, t, r, 1.0, xm, (int)N));
            }
        }
        TRY(run_gemms(c, g1));
        TRY(run_gemms(c, g2));
    }
    for (int k = NT - 1; k >= 0; --k) {
        double *xk = X + (size_t)k * NB;
        g1.push_back(make_gemm(1, 0, NB, nrhs, NB, 1.0, A->linv(k), NB, xk, (int)N, 0.0, tmp, NB));
        TRY(run_gemms(c, g1));
        cp.push_back(make_copy(tmp, NB, xk, (int)N, NB, nrhs));
        TRY(run_copies(c, cp));
        for (int j = 0; j < k; ++j) {
            double *xj = X + (size_t)j * NB;
            if (A->is_dense(k, j)) {
                g2.push_back(make_gemm(1, 0, NB, nrhs, NB, -1.0, A->dense(k, j), NB, xk, (int)N, 1.0, xj, (int)N));
            } else {
                const int r = A->rank(k, j);
                if (r == 0) continue;
                double *t = T2 + (size_t)j * A->maxrank * nrhs;
                g1.push_back(make_gemm(1, 0, r, nrhs, NB, 1.0, A->U(k, j), NB, xk, (int)N, 0.0, t, r));
                g2.push_back(make_gemm(0, 0, NB, nrhs, r, -1.0, A->V(k, j), NB, t, r, 1.0, xj, (int)N));
            }
        }
        TRY(run_gemms(c, g1));
        TRY(run_gemms(c, g2));
    }
    return 0;
}

int hicma_tlr_solve(hicma_tlr_ctx *c, hicma_tlr_desc *A, int nrhs, double *B, long ldb) {
    ARG_CHECK(c && A && B && nrhs > 0 && ldb >= A->N, "solve arguments");
    if (!A->factored) { set_err("descriptor is not factored"); return HICMA_TLR_ERR_STATE; }
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    NvtxRange nv("solve");
    CUDA_TRY(cudaSetDevice(c->device));
    ws_reset(c);
    const size_t N = A->N;
    double *X = ws_alloc<double>(c, N * nrhs);
    if (!X) { set_err("workspace too small (solve)"); return HICMA_TLR_ERR_OOM; }
    CUDA_TRY(cudaMemcpy2DAsync(X, N * sizeof(double), B, ldb * sizeof(double), N * sizeof(double), nrhs,
                               cudaMemcpyHostToDevice, c->stream));
    TRY(solve_dev(c, A, X, nrhs));
    CUDA_TRY(cudaMemcpy2DAsync(B, ldb * sizeof(double), X, N * sizeof(double), N * sizeof(double), nrhs,
                               cudaMemcpyDeviceToHost, c->stream));
    TRY(ctx_sync(c));
    ws_reset(c);
    return 0;
}

int hicma_tlr_loglik(hicma_tlr_ctx *c, hicma_tlr_desc *A, const double *y, double *loglik, double *logdet, double *x) {
    ARG_CHECK(c && A && y, "null");
    if (!A->factored) { set_err("descriptor is not factored"); return HICMA_TLR_ERR_STATE; }
    std::vector<double> xs(y, y + A->N);
    TRY(hicma_tlr_solve(c, A, 1, xs.data(), A->N));
    double ld = 0.0;
    TRY(hicma_tlr_logdet(c, A, &ld));
    double q = 0.0;
    for (int i = 0; i < A->N; ++i) q += y[i] * xs[i];
    if (loglik) *loglik = -0.5 * (q + ld + A->N * std::log(2.0 * M_PI));
    if (logdet) *logdet = ld;
    if (x) std::memcpy(x, xs.data(), sizeof(double) * A->N);
    return 0;
}

// ------------------------------------------------------------ profiling ----
int hicma_tlr_prof_enable(hicma_tlr_ctx *c, int on) {
    ARG_CHECK(c, "null");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    prof_flush(c);
    std::memset(c->prof_acc, 0, sizeof c->prof_acc);
    TRY(ctx_sync(c));
    CUDA_TRY(xclear(c, c->d_profacc, 64 * sizeof(double)));
    c->prof = on != 0;
    return 0;
}

int hicma_tlr_prof_read(hicma_tlr_ctx *c, double *out, int nclass) {
    ARG_CHECK(c && out, "null");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    prof_flush(c);
    // work counted on the device (GEMMs whose n is a rank decided on the device)
    double dev[64];
    TRY(ctx_sync(c));
    CUDA_TRY(xfer(c, dev, c->d_profacc, sizeof dev, cudaMemcpyDeviceToHost));
    for (int k = 0; k < nclass && k < P_NCLASS; ++k)
        for (int j = 0; j < 4; ++j) out[k * 4 + j] = c->prof_acc[k][j] + (j >= 2 ? dev[2 * k + j - 2] : 0.0);
    return 0;
}

// ---------------------------------------------------------------- check ----
// Dense device copy (lower triangle, ld N) of a TLR descriptor.
static int densify(hicma_tlr_ctx *c, hicma_tlr_desc *A, double *D) {
    const int NT = A->NT, NB = A->NB;
    const size_t N = A->N;
    CUDA_TRY(cudaMemsetAsync(D, 0, N * N * sizeof(double), c->stream));
    std::vector<GemmTask> g;
    std::vector<CopyTask> cp;
    for (int n = 0; n < NT; ++n)
        for (int m = n; m < NT; ++m) {
            double *dst = D + (size_t)m * NB + (size_t)n * NB * N;
            if (A->is_dense(m, n)) {
                cp.push_back(make_copy(A->dense(m, n), NB, dst, (int)N, NB, NB));
            } else {
                const int r = A->rank(m, n);
                if (r > 0) g.push_back(make_gemm(0, 1, NB, NB, r, 1.0, A->U(m, n), NB, A->V(m, n), NB, 0.0, dst, (int)N));
            }
        }
    TRY(run_copies(c, cp));
    TRY(run_gemms(c, g));
    for (int k = 0; k < NT; ++k) {
        launch_zero_upper(D + (size_t)k * NB + (size_t)k * NB * N, NB, (int)N, c->stream);
        TRY(check_launch(c));
    }
    return 0;
}

// Full-size counterpart of check_dpotrf2 (testing_dpotrf.c:111-180): with
// Gaussian probes Z (N x p), ||(A - L L^T) Z||_F / ||A Z||_F estimates
// ||A - L L^T||_F / ||A||_F without forming an N x N matrix.  A Z uses the
// exact covariance, regenerated block-row by block-row in workspace chunks;
// L (L^T Z) uses the TLR tiles.  Partial products are summed in a fixed order.
int hicma_tlr_check_probe(hicma_tlr_ctx *c, hicma_tlr_desc *L, const hicma_tlr_problem *prob, int nprobe,
                          unsigned long long seed, double *res_est) {
    ARG_CHECK(c && L && prob && res_est && nprobe >= 1 && nprobe <= 64, "check_probe arguments");
    if (!L->factored) { set_err("descriptor is not factored"); return HICMA_TLR_ERR_STATE; }
    TRY(check_problem_data(L, prob));
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    NvtxRange nv("check_probe");
    CUDA_TRY(cudaSetDevice(c->device));
    c->cur = c->stream;
    c->ar = &c->main_ar;
    ws_reset(c);
    const int NT = L->NT, NB = L->NB, p = nprobe;
    const size_t N = L->N;
    double *Z = ws_alloc<double>(c, N * p), *AZ = ws_alloc<double>(c, N * p);
    double *W = ws_alloc<double>(c, N * p), *Y = ws_alloc<double>(c, N * p);
    double *part = ws_alloc<double>(c, 1024), *sc = ws_alloc<double>(c, 8);
    if (!Z || !AZ || !W || !Y || !part || !sc) { set_err("workspace too small (check_probe)"); return HICMA_TLR_ERR_OOM; }
    launch_gaussian(Z, (int)N, p, (int)N, seed ^ 0x9E3779B97F4A7C15ull, c->stream);
    CUDA_TRY(cudaMemsetAsync(AZ, 0, N * p * sizeof(double), c->stream));
    CUDA_TRY(cudaMemsetAsync(W, 0, N * p * sizeof(double), c->stream));
    CUDA_TRY(cudaMemsetAsync(Y, 0, N * p * sizeof(double), c->stream));
    const size_t base = c->ar->off;
    const CovParams cp = cov_params(L, prob);
    // ---- A Z: tiles (m, n <= m) in chunks; P = A_mn Z_n, P' = A_mn^T Z_m
    const size_t per_tile = align_up(sizeof(double) * (size_t)NB * NB + 1) + 2 * align_up(sizeof(double) * (size_t)NB * p + 1);
    for (int m = 0; m < NT; ++m) {
        int n0 = 0;
        while (n0 <= m) {
            c->ar->off = base;
            const size_t reserve = align_up(sizeof(double) * (size_t)NB * p + 1) + 4096;
            const size_t fit = ws_free(c) > reserve ? (ws_free(c) - reserve) / (per_tile + 1024) : 0;
            if (fit < 1) { set_err("workspace too small (check_probe tile)"); return HICMA_TLR_ERR_OOM; }
            const int n1 = std::min(m + 1, n0 + (int)std::min<size_t>(fit, 256));
            const int cnt = n1 - n0;
            double *R = ws_alloc<double>(c, (size_t)cnt * NB * NB);
            double *P = ws_alloc<double>(c, (size_t)cnt * NB * p);
            double *Pt = ws_alloc<double>(c, (size_t)cnt * NB * p);
            std::vector<CovTask> ct;
            std::vector<GemmTask> g;
            std::vector<CopyTask> cpy;
            for (int n = n0; n < n1; ++n) {
                double *tile = R + (size_t)(n - n0) * NB * NB;
                ct.push_back(CovTask{tile, NB, m * NB, n * NB, NB, NB});
                g.push_back(make_gemm(0, 0, NB, p, NB, 1.0, tile, NB, Z + (size_t)n * NB, (int)N, 0.0,
                                      P + (size_t)(n - n0) * NB * p, NB));
                if (n < m) {
                    double *pt = Pt + (size_t)(n - n0) * NB * p;
                    g.push_back(make_gemm(1, 0, NB, p, NB, 1.0, tile, NB, Z + (size_t)m * NB, (int)N, 0.0, pt, NB));
                    cpy.push_back(make_copy(pt, NB, AZ + (size_t)n * NB, (int)N, NB, p, 1.0, 1.0));
                }
            }
            TRY(bc_cov(cp, ct));
            CovTask *dct = stage(c, ct.data(), ct.size());
            if (!dct) { set_err("staging failed"); return HICMA_TLR_ERR_CUDA; }
            launch_cov_batched(cp, dct, (int)ct.size(), NB, NB, c->stream);
            TRY(check_launch(c));
            TRY(run_gemms(c, g));
            // AZ_m += sum of the chunk's P in order (AZ_m is NB x p with ld N: one column at a time)
            {
                // gather column blocks: P is [tile](NB x p) contiguous, so accumulate into a packed
                // NB x p buffer, then add it to the strided AZ_m with one copy
                double *acc = ws_alloc<double>(c, (size_t)NB * p);
                if (!acc) { set_err("workspace too small (check_probe acc)"); return HICMA_TLR_ERR_OOM; }
                CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(double) * NB * p, c->stream));
                launch_accumulate(acc, P, cnt, (long long)NB * p, c->stream);
                TRY(check_launch(c));
                std::vector<CopyTask> one{make_copy(acc, NB, AZ + (size_t)m * NB, (int)N, NB, p, 1.0, 1.0)};
                TRY(run_copies(c, one));
            }
            TRY(run_copies(c, cpy));
            n0 = n1;
        }
    }
    c->ar->off = base;
    // ---- W = L^T Z: block row m contributes L_mn^T Z_m to W_n (n <= m)
    for (int m = 0; m < NT; ++m) {
        c->ar->off = base;
        std::vector<GemmTask> g1, g2;
        const double *Zm = Z + (size_t)m * NB;
        for (int n = 0; n <= m; ++n) {
            double *Wn = W + (size_t)n * NB;
            if (L->is_dense(m, n)) {
                g2.push_back(make_gemm(1, 0, NB, p, NB, 1.0, L->dense(m, n), NB, Zm, (int)N, 1.0, Wn, (int)N));
            } else {
                const int r = L->rank(m, n);
                if (r <= 0) continue;
                double *t = ws_alloc<double>(c, (size_t)r * p);
                if (!t) { set_err("workspace too small (check_probe)"); return HICMA_TLR_ERR_OOM; }
                g1.push_back(make_gemm(1, 0, r, p, NB, 1.0, L->U(m, n), NB, Zm, (int)N, 0.0, t, r));
                g2.push_back(make_gemm(0, 0, NB, p, r, 1.0, L->V(m, n), NB, t, r, 1.0, Wn, (int)N));
            }
        }
        TRY(run_gemms(c, g1));
        TRY(run_gemms(c, g2));
    }
    // ---- Y = L W: block column n contributes L_mn W_n to Y_m (m >= n)
    for (int n = 0; n < NT; ++n) {
        c->ar->off = base;
        std::vector<GemmTask> g1, g2;
        const double *Wn = W + (size_t)n * NB;
        for (int m = n; m < NT; ++m) {
            double *Ym = Y + (size_t)m * NB;
            if (L->is_dense(m, n)) {
                g2.push_back(make_gemm(0, 0, NB, p, NB, 1.0, L->dense(m, n), NB, Wn, (int)N, 1.0, Ym, (int)N));
            } else {
                const int r = L->rank(m, n);
                if (r <= 0) continue;
                double *t = ws_alloc<double>(c, (size_t)r * p);
                if (!t) { set_err("workspace too small (check_probe)"); return HICMA_TLR_ERR_OOM; }
                g1.push_back(make_gemm(1, 0, r, p, NB, 1.0, L->V(m, n), NB, Wn, (int)N, 0.0, t, r));
                g2.push_back(make_gemm(0, 0, NB, p, r, 1.0, L->U(m, n), NB, t, r, 1.0, Ym, (int)N));
            }
        }
        TRY(run_gemms(c, g1));
        TRY(run_gemms(c, g2));
    }
    const int nblk = 1024;
    launch_sumsq(AZ, Y, (int)N, p, (long long)N, 0, part, nblk, sc + 0, c->stream);
    launch_sumsq(AZ, nullptr, (int)N, p, (long long)N, 0, part, nblk, sc + 1, c->stream);
    double h[2] = {0, 0};
    CUDA_TRY(cudaMemcpyAsync(h, sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    TRY(ctx_sync(c));
    ws_reset(c);
    *res_est = h[1] > 0.0 ? std::sqrt(h[0] / h[1]) : 0.0;
    return 0;
}

int hicma_tlr_check(hicma_tlr_ctx *c, hicma_tlr_desc *L, const hicma_tlr_problem *prob, hicma_tlr_desc *A0,
                    double *res_llt, double *res_diff) {
    ARG_CHECK(c && L && prob, "null");
    if (!L->factored) { set_err("descriptor is not factored"); return HICMA_TLR_ERR_STATE; }
    TRY(check_problem_data(L, prob));
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    NvtxRange nv("check");
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t N = L->N;
    double *DL = nullptr, *DA = nullptr, *D0 = nullptr, *part = nullptr, *sc = nullptr;
    int *dinfo = nullptr;
    auto cleanup = [&]() {
        for (void *p : {(void *)DL, (void *)DA, (void *)D0, (void *)part, (void *)sc, (void *)dinfo}) {
            bc_remove(p);
            cudaFree(p);
        }
    };
    const int nblk = 1024;
    if (cudaMalloc(&DL, N * N * sizeof(double)) != cudaSuccess || cudaMalloc(&DA, N * N * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&part, nblk * sizeof(double)) != cudaSuccess || cudaMalloc(&sc, 8 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&dinfo, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        set_err("check: allocation of dense N x N buffers failed (N = %zu)", N);
        return HICMA_TLR_ERR_OOM;
    }
    bc_add(DL, N * N * sizeof(double));
    bc_add(DA, N * N * sizeof(double));
    bc_add(part, nblk * sizeof(double));
    bc_add(sc, 8 * sizeof(double));
    bc_add(dinfo, sizeof(int));
    int rc = densify(c, L, DL);
    if (rc) { cleanup(); return rc; }
    // exact A (check_dpotrf2 uses the unapproximated matrix, testing_dpotrf.c:856-893)
    CovTask ct{DA, (int)N, 0, 0, (int)N, (int)N};
    CovTask *dct = stage(c, &ct, 1);
    launch_cov_batched(cov_params(L, prob), dct, 1, (int)N, (int)N, c->stream);
    launch_sumsq(DA, nullptr, (int)N, (int)N, (long long)N, 0, part, nblk, sc + 0, c->stream);
    // DA <- L L^T - A
    launch_gemm_single(make_gemm(0, 1, (int)N, (int)N, (int)N, 1.0, DL, (int)N, DL, (int)N, -1.0, DA, (int)N), c->stream);
    launch_sumsq(DA, nullptr, (int)N, (int)N, (long long)N, 0, part, nblk, sc + 1, c->stream);
    double h[4] = {0, 0, 0, 0};
    if (A0 && res_diff) {
        if (cudaMalloc(&D0, N * N * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            D0 = nullptr;
            cleanup();
            set_err("check: allocation failed");
            return HICMA_TLR_ERR_OOM;
        }
        bc_add(D0, N * N * sizeof(double));
        rc = densify(c, A0, D0);
        if (rc) { cleanup(); return rc; }
        cudaMemsetAsync(dinfo, 0, sizeof(int), c->stream);
        rc = potrf_tile(c, D0, (int)N, (int)N, nullptr, 0, dinfo, 0);
        if (rc) { cleanup(); return rc; }
        launch_sumsq(DL, D0, (int)N, (int)N, (long long)N, 1, part, nblk, sc + 2, c->stream);
        launch_sumsq(DL, nullptr, (int)N, (int)N, (long long)N, 1, part, nblk, sc + 3, c->stream);
    }
    cudaError_t e = cudaMemcpyAsync(h, sc, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    c->stage_off = 0;
    cleanup();
    if (e != cudaSuccess) { set_err("check: %s", cudaGetErrorString(e)); return HICMA_TLR_ERR_CUDA; }
    if (res_llt) *res_llt = std::sqrt(h[1]) / std::sqrt(h[0]);
    if (res_diff) *res_diff = (A0 ? std::sqrt(h[2]) / std::sqrt(h[3]) : NAN);
    return 0;
}

// ------------------------------------------------- kernel-level entries ----
int hicma_tlr_k_cov(const hicma_tlr_problem *prob, const double *d_points, int N, int r0, int nr, int c0, int nc,
                    double *d_out, int ld, void *stream) {
    ARG_CHECK(prob && d_points && d_out && N > 0 && nr >= 0 && nc >= 0 && ld >= nr, "k_cov arguments");
    ARG_CHECK(r0 >= 0 && c0 >= 0 && r0 + nr <= N && c0 + nc <= N, "k_cov range");
    const int ndim = kind_ndim(prob->kind);
    ARG_CHECK(ndim > 0, "kind (randtlr tiles come from hicma_tlr_generate: no points)");
    TRY(rbf_args(prob));
    const CovParams p = make_cov_params(prob, d_points, N, ndim);
    CovTask t{d_out, ld, r0, c0, nr, nc};
    CovTask *dt = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(cudaMallocAsync(&dt, sizeof(CovTask), st));
    CUDA_TRY(cudaMemcpyAsync(dt, &t, sizeof t, cudaMemcpyHostToDevice, st));
    launch_cov_batched(p, dt, 1, nr, nc, st);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaFreeAsync(dt, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return 0;
}

unsigned long hicma_tlr_op_counts(char op, unsigned long a, unsigned long b, unsigned long c, unsigned long d) {
    return op_counts(op, a, b, c, d);
}

int hicma_tlr_bounds_checked(void) {
#ifdef TLR_BOUNDS_CHECK
    return 1;
#else
    return 0;
#endif
}

int hicma_tlr_bounds_register(const void *p, size_t bytes) {
#ifdef TLR_BOUNDS_CHECK
    ARG_CHECK(p && bytes, "bounds_register arguments");
    bc_add(p, bytes);
    return 0;
#else
    (void)p; (void)bytes;
    set_err("this library was built without TLR_BOUNDS_CHECK");
    return HICMA_TLR_ERR_NOT_SUPPORTED;
#endif
}

int hicma_tlr_bounds_unregister(const void *p) {
#ifdef TLR_BOUNDS_CHECK
    bc_remove(p);
    return 0;
#else
    (void)p;
    set_err("this library was built without TLR_BOUNDS_CHECK");
    return HICMA_TLR_ERR_NOT_SUPPORTED;
#endif
}

int hicma_tlr_bounds_inside(const void *p, size_t bytes) {
#ifdef TLR_BOUNDS_CHECK
    return bc_inside(p, bytes) ? 1 : 0;
#else
    (void)p; (void)bytes;
    set_err("this library was built without TLR_BOUNDS_CHECK");
    return HICMA_TLR_ERR_NOT_SUPPORTED;
#endif
}

int hicma_tlr_k_wait_probe(long long polls0, long long polls1, int nblocks, double *elapsed_ms, void *stream) {
    ARG_CHECK(nblocks >= 1 && nblocks <= 64, "wait probe: 1..64 blocks");
    ARG_CHECK(polls0 >= 1 && polls1 >= 1 && polls0 <= (1LL << 26) && polls1 <= (1LL << 26),
              "wait probe: 1..2^26 polls");
    cudaStream_t st = (cudaStream_t)stream;
    int *buf = nullptr;   // [0] timeout flag, then cnt: [1] ticket, [2] abort, [3..] counters
    CUDA_TRY(cudaMalloc(&buf, (3 + 64) * sizeof(int)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int flags[3] = {0, 0, 0};
    float ms = 0.f;
    cudaError_t e = cudaMemsetAsync(buf, 0, (3 + 64) * sizeof(int), st);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaEventRecord(e0, st);
    if (e == cudaSuccess && launch_wait_probe(buf + 1, buf, nblocks, polls0, polls1, st) != 0) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(e1, st);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess) e = cudaMemcpyAsync(flags, buf, 3 * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(buf);
    if (e != cudaSuccess) {
        set_err("wait probe: %s", cudaGetErrorString(e));
        return HICMA_TLR_ERR_CUDA;
    }
    if (elapsed_ms) *elapsed_ms = ms;
    if (flags[0]) {
        set_err("a bounded device wait gave up (wait probe; abort flag %d)", flags[2]);
        return HICMA_TLR_ERR_TIMEOUT;
    }
    return 0;
}

int hicma_tlr_k_dgemm(int transA, int transB, int m, int n, int k, double alpha, const double *A, int lda,
                      const double *B, int ldb, double beta, double *C, int ldc, void *stream) {
    ARG_CHECK(m >= 0 && n >= 0 && k >= 0 && A && B && C, "k_dgemm arguments");
    launch_gemm_single(make_gemm(transA ? 1 : 0, transB ? 1 : 0, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc),
                       (cudaStream_t)stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    return 0;
}

int hicma_tlr_k_potrf(hicma_tlr_ctx *c, int n, double *d_A, int lda, double *d_linv, int *d_info, int info_offset) {
    ARG_CHECK(c && d_A && n > 0 && lda >= n && d_info, "k_potrf arguments");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    BcScope bc;
    bc.add(d_A, bc_span(n, n, lda));
    if (d_linv) bc.add(d_linv, bc_span(n, n, n));
    bc.add(d_info, sizeof(int));
    ws_reset(c);
    TRY(potrf_tile(c, d_A, n, lda, d_linv, n, d_info, info_offset));
    TRY(ctx_sync(c));
    return check_timeout(c);
}

int hicma_tlr_k_lr_update(hicma_tlr_ctx *c, int nb, const double *d_Au, const double *d_Av, int ra,
                          const double *d_Bu, const double *d_Bv, int rb, double *d_Cu, double *d_Cv, int *rc,
                          double acc, int maxrank, int fixed_rank) {
    ARG_CHECK(c && rc && d_Cu && d_Cv && nb > 0, "k_lr_update arguments");
    ARG_CHECK(ra >= 0 && rb >= 0 && *rc >= 0 && maxrank >= 1, "ranks");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    BcScope bc;
    bc.add(d_Au, bc_span(nb, ra, nb));
    bc.add(d_Av, bc_span(nb, ra, nb));
    bc.add(d_Bu, bc_span(nb, rb, nb));
    bc.add(d_Bv, bc_span(nb, rb, nb));
    bc.add(d_Cu, bc_span(nb, maxrank, nb));
    bc.add(d_Cv, bc_span(nb, maxrank, nb));
    ws_reset(c);
    int *d_r = ws_alloc<int>(c, 2);
    if (!d_r) { set_err("workspace too small"); return HICMA_TLR_ERR_OOM; }
    std::vector<RecompTask> v{RecompTask{d_Cu, d_Cv, *rc, d_Au, d_Av, ra, d_Bu, d_Bv, rb, d_Cu, d_Cv, d_r}};
    CUDA_TRY(cudaMemsetAsync(c->d_flags + 1, 0, sizeof(int), c->stream));
    TRY(run_recompress(c, nb, v, acc, maxrank, fixed_rank, d_r + 1, 0.0));
    int r = 0;
    CUDA_TRY(cudaMemcpyAsync(&r, d_r, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    TRY(ctx_sync(c));
    *rc = r;
    ws_reset(c);
    return 0;
}

int hicma_tlr_k_compress(hicma_tlr_ctx *c, int nb, const double *d_A, double *d_U, double *d_V, int maxrank,
                         double tol, int *rank) {
    ARG_CHECK(c && d_A && d_U && d_V && rank && nb > 0 && maxrank >= 1 && tol > 0, "k_compress arguments");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    BcScope bc;
    bc.add(d_A, bc_span(nb, nb, nb));
    bc.add(d_U, bc_span(nb, maxrank, nb));
    bc.add(d_V, bc_span(nb, maxrank, nb));
    ws_reset(c);
    const int s = std::min(maxrank + 10, nb);
    double *Omega = ws_alloc<double>(c, (size_t)nb * s);
    double *Ident = ws_alloc<double>(c, (size_t)s * s);
    int *d_r = ws_alloc<int>(c, 2);
    if (!Omega || !Ident || !d_r) { set_err("workspace too small"); return HICMA_TLR_ERR_OOM; }
    launch_gaussian(Omega, nb, s, nb, 0x5DEECE66Dull, c->stream);
    launch_set_identity(Ident, s, s, c->stream);
    std::vector<CompressTask> v{CompressTask{d_A, d_U, d_V, d_r}};
    int *d_fail = ws_alloc<int>(c, 1);
    if (!d_fail) { set_err("workspace too small"); return HICMA_TLR_ERR_OOM; }
    CUDA_TRY(cudaMemsetAsync(d_fail, 0, sizeof(int), c->stream));
    TRY(run_compress(c, nb, maxrank, tol, Omega, s, v, Ident, d_r + 1, d_fail));
    int fail = 0;
    CUDA_TRY(cudaMemcpyAsync(&fail, d_fail, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    TRY(ctx_sync(c));
    if (fail) {   // the range finder's Q failed its orthogonality check: Householder path
        v.assign(1, CompressTask{d_A, d_U, d_V, d_r});
        TRY(run_compress(c, nb, maxrank, tol, Omega, s, v, Ident, d_r + 1, nullptr, true));
    }
    int r = 0;
    CUDA_TRY(cudaMemcpyAsync(&r, d_r, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    TRY(ctx_sync(c));
    *rank = r;
    ws_reset(c);
    return 0;
}

}  // extern "C"
