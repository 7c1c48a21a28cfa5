// Dense diagonal-block Cholesky and inverse (one CTA per 64 x 64 block).
//
// The blocked tile POTRF (HCORE_dpotrf at
// hicma_parsec/HiCMA_dpotrf_L_2flow.jdf:233) and the tile inverse used for
// the TRSMs are driven from the host engine: this kernel factors the jb x jb
// diagonal block in shared memory, reports the first non-positive pivot as
// the reference's INFO (k*mb + iinfo, :241-242) and writes L_jj^{-1} for the
// panel solve; the panel and trailing updates are DMMA GEMMs.
#include "tlr_internal.h"

#include <cstdio>
#include <vector>

namespace tlr {
namespace {

constexpr int DB = 64;          // diagonal block size
constexpr int LDS = DB + 1;     // padded shared leading dimension

__global__ void __launch_bounds__(256) k_potrf_diag(double *A, int lda, int jb, double *Dinv, int ldd,
                                                    int *info, int info_base) {
    extern __shared__ double sm[];
    double *S = sm;              // S[c * LDS + r] = L(r, c)
    double *X = sm + DB * LDS;   // inverse
    __shared__ int fail;
    const int tid = threadIdx.x;
    if (tid == 0) fail = 0;
    for (int idx = tid; idx < jb * jb; idx += blockDim.x) {
        const int c = idx / jb, r = idx - c * jb;
        S[c * LDS + r] = A[(size_t)r + (size_t)c * lda];
    }
    __syncthreads();
    for (int c = 0; c < jb; ++c) {
        if (tid == 0) {
            const double d = S[c * LDS + c];
            if (!(d > 0.0)) {
                fail = 1;
                if (info) atomicCAS(info, 0, info_base + c + 1);
            } else {
                S[c * LDS + c] = sqrt(d);
            }
        }
        __syncthreads();
        if (fail) break;
        const double piv = S[c * LDS + c];
        for (int r = c + 1 + tid; r < jb; r += blockDim.x) S[c * LDS + r] /= piv;
        __syncthreads();
        const int w = jb - c - 1;
        for (int idx = tid; idx < w * w; idx += blockDim.x) {
            const int cc = c + 1 + idx / w, r = c + 1 + idx % w;
            if (r >= cc) S[cc * LDS + r] -= S[c * LDS + r] * S[c * LDS + cc];
        }
        __syncthreads();
    }
    if (fail) return;
    // inverse of the lower triangle, one column per thread (forward substitution)
    if (tid < jb) {
        const int j = tid;
        X[j * LDS + j] = 1.0 / S[j * LDS + j];
        for (int i = j + 1; i < jb; ++i) {
            double s = 0.0;
            for (int l = j; l < i; ++l) s += S[l * LDS + i] * X[j * LDS + l];
            X[j * LDS + i] = -s / S[i * LDS + i];
        }
    }
    __syncthreads();
    for (int idx = tid; idx < jb * jb; idx += blockDim.x) {
        const int c = idx / jb, r = idx - c * jb;
        A[(size_t)r + (size_t)c * lda] = (r >= c) ? S[c * LDS + r] : 0.0;
        if (Dinv) Dinv[(size_t)r + (size_t)c * ldd] = (r >= c) ? X[c * LDS + r] : 0.0;
    }
}

}  // namespace

void launch_potrf_diag(double *A, int lda, int jb, double *Dinv, int ldd, int *info, int info_base,
                       cudaStream_t st) {
    const size_t smem = 2 * DB * LDS * sizeof(double);
    // per device and thread-safe: set on every launch (a host-side call, no synchronisation)
    cudaFuncSetAttribute(k_potrf_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_potrf_diag<<<1, 256, smem, st>>>(A, lda, jb, Dinv, ldd, info, info_base);
}

}  // namespace tlr

// ---------------------------------------------------------------------------
// Allocation-free tile Cholesky.
//
// For callers that must not allocate device memory (for example code that
// runs inside a host framework owning every device buffer, or a latency-bound
// loop that cannot afford the device-wide synchronisation cudaMalloc may
// cause).  Its scratch is the file-scope array below: the 64 x 64 inverse of
// the current diagonal block followed by the 64 x n row panel used while the
// inverse of the factor is assembled.  Every GPU that loads this library
// holds the array until the process exits.
namespace tlr {
namespace {

constexpr int NOALLOC_MAX_N = 4096;
constexpr size_t NOALLOC_SCRATCH = 64 * 64 + (size_t)64 * NOALLOC_MAX_N;
__device__ __align__(256) double g_potrf_scratch[NOALLOC_SCRATCH];

int noalloc_fail(const char *what, cudaError_t e) {
    char msg[320];
    snprintf(msg, sizeof msg, "hicma_tlr_k_potrf_noalloc: %s: %s", what, cudaGetErrorString(e));
    tlr_set_error(msg);
    return HICMA_TLR_ERR_CUDA;
}

#ifdef TLR_BOUNDS_CHECK
// Extent checks of the bounds-checked build: every operand of every launch
// must lie inside one registered region (the caller's A, L^-1 and info are
// registered for the length of the call, the scratch array for the life of
// the process).
bool noalloc_inside(const void *p, size_t bytes, const char *what) {
    if (bc_inside(p, bytes)) return true;
    char msg[320];
    snprintf(msg, sizeof msg, "bounds check: %s [%p, +%zu B) lies outside every live allocation", what, p, bytes);
    tlr_set_error(msg);
    return false;
}
bool noalloc_gemm_inside(const GemmTask &t) {
    return noalloc_inside(t.A, t.opA ? bc_span(t.k, t.m, t.lda) : bc_span(t.m, t.k, t.lda), "noalloc gemm A") &&
           noalloc_inside(t.B, t.opB ? bc_span(t.n, t.k, t.ldb) : bc_span(t.k, t.n, t.ldb), "noalloc gemm B") &&
           noalloc_inside(t.C, bc_span(t.m, t.n, t.ldc), "noalloc gemm C");
}
#endif

}  // namespace
}  // namespace tlr

extern "C" int hicma_tlr_k_potrf_noalloc(int n, double *d_A, int lda, double *d_linv, int *d_info, int info_offset,
                                         void *stream) {
    using namespace tlr;
    if (n < 1 || n > NOALLOC_MAX_N || !d_A || lda < n || !d_info) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "hicma_tlr_k_potrf_noalloc: need 1 <= n <= %d (got %d), lda >= n, non-null A and info",
                 NOALLOC_MAX_N, n);
        tlr_set_error(msg);
        return HICMA_TLR_ERR_ARG;
    }
    // an error left by the caller's earlier work is reported as such, not
    // blamed on (or cleared by) this call
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) return noalloc_fail("an earlier CUDA error is pending", pending);
    // The host-side name of the array is not a device address: ask the runtime
    // for it on every call (a host-side lookup once the module is loaded; the
    // first call on a device loads it, so that call belongs before any stream
    // capture).  Looking it up each time keeps the address right after a
    // device reset or under another driver context of the same device.
    double *scratch = nullptr;
    {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_potrf_scratch);
        if (e != cudaSuccess || !p) return noalloc_fail("cudaGetSymbolAddress of the scratch array failed", e);
        scratch = (double *)p;
    }
    cudaStream_t st = (cudaStream_t)stream;
    double *dscr = scratch;              // 64 x 64 diagonal-block inverse
    double *tmp = scratch + 64 * 64;     // 64 x n row panel
    const int DBK = 64;
#ifdef TLR_BOUNDS_CHECK
    if (!bc_inside(scratch, NOALLOC_SCRATCH * sizeof(double))) bc_add(scratch, NOALLOC_SCRATCH * sizeof(double));
    struct Scope {
        std::vector<const void *> ps;
        void add(const void *p, size_t b) { if (p && b) { bc_add(p, b); ps.push_back(p); } }
        ~Scope() { for (const void *p : ps) bc_remove(p); }
    } reg;
    reg.add(d_A, bc_span(n, n, lda));
    if (d_linv) reg.add(d_linv, bc_span(n, n, n));
    reg.add(d_info, sizeof(int));
#define NOALLOC_GEMM(task)                                                     \
    do {                                                                       \
        const GemmTask t__ = (task);                                           \
        if (!noalloc_gemm_inside(t__)) return HICMA_TLR_ERR_ARG;               \
        launch_gemm_single(t__, st);                                           \
        const cudaError_t e__ = cudaGetLastError();                            \
        if (e__ != cudaSuccess) return noalloc_fail("GEMM launch failed", e__); \
    } while (0)
#else
#define NOALLOC_GEMM(task)                                                     \
    do {                                                                       \
        launch_gemm_single((task), st);                                        \
        const cudaError_t e__ = cudaGetLastError();                            \
        if (e__ != cudaSuccess) return noalloc_fail("GEMM launch failed", e__); \
    } while (0)
#endif
    if (d_linv) {
        const cudaError_t e = cudaMemset2DAsync(d_linv, (size_t)n * sizeof(double), 0, sizeof(double) * n, n, st);
        if (e != cudaSuccess) return noalloc_fail("clearing the inverse failed", e);
    }
    for (int j = 0; j < n; j += DBK) {
        const int jb = n - j < DBK ? n - j : DBK;
        double *Dinv = d_linv ? d_linv + j + (size_t)j * n : dscr;
        const int ldd = d_linv ? n : DBK;
        launch_potrf_diag(d_A + j + (size_t)j * lda, lda, jb, Dinv, ldd, d_info, info_offset + j, st);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return noalloc_fail("diagonal-block launch failed", e);
        if (j + jb < n) {
            const int rows = n - j - jb;
            double *Pn = d_A + (j + jb) + (size_t)j * lda;
            NOALLOC_GEMM(make_gemm(0, 1, rows, jb, jb, 1.0, Pn, lda, Dinv, ldd, 0.0, Pn, lda));
            NOALLOC_GEMM(make_gemm(0, 1, rows, rows, jb, -1.0, Pn, lda, Pn, lda, 1.0,
                                   d_A + (j + jb) + (size_t)(j + jb) * lda, lda, 1));
        }
    }
    launch_zero_upper(d_A, n, lda, st);
    {
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return noalloc_fail("clearing the upper triangle failed", e);
    }
    if (d_linv) {
        for (int i0 = DBK; i0 < n; i0 += DBK) {
            const int ib = n - i0 < DBK ? n - i0 : DBK;
            NOALLOC_GEMM(make_gemm(0, 0, ib, i0, i0, 1.0, d_A + i0, lda, d_linv, n, 0.0, tmp, ib));
            NOALLOC_GEMM(make_gemm(0, 0, ib, i0, ib, -1.0, d_linv + i0 + (size_t)i0 * n, n, tmp, ib, 0.0,
                                   d_linv + i0, n));
        }
    }
#undef NOALLOC_GEMM
    return 0;
}
