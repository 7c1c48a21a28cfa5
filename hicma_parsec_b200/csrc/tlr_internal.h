// Internal declarations of the B200 TLR engine: batched task descriptors and
// the host-side launchers of every kernel.  Column-major FP64 throughout.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/hicma_tlr.h"

namespace tlr {

// ------------------------------------------------------- bounds checking ----
// Builds with TLR_BOUNDS_CHECK check on the host, before every batched launch,
// that each task's operand extents lie inside one live device region (library
// allocations, the workspace, or caller buffers registered for the length of
// a kernel-level call); a launch that would leave them is refused with
// HICMA_TLR_ERR_ARG and the offending task in the error message.  Other
// builds compile the checks away.
#ifdef TLR_BOUNDS_CHECK
void bc_add(const void *p, size_t bytes);
void bc_remove(const void *p);
bool bc_inside(const void *p, size_t bytes);
#else
inline void bc_add(const void *, size_t) {}
inline void bc_remove(const void *) {}
inline bool bc_inside(const void *, size_t) { return true; }
#endif
// Bytes spanned by a rows x cols column-major block with leading dimension ld.
inline size_t bc_span(long long rows, long long cols, long long ld, size_t elt = sizeof(double)) {
    return rows <= 0 || cols <= 0 ? 0 : (size_t)((cols - 1) * ld + rows) * elt;
}

// ----------------------------------------------------------- batched DGEMM --
// One problem of a batched C = alpha op(A) op(B) + beta C.  Tiles of 64x64
// outputs are flattened over the batch with tile_off (prefix sums).
struct GemmTask {
    const double *A;
    const double *B;
    double *C;
    int m, n, k;
    int lda, ldb, ldc;
    int opA, opB;       // 0 = N, 1 = T
    int lower;          // skip output tiles strictly above the diagonal
    int tiles_m;        // ceil(m / 64)
    double alpha, beta;
    const int *n_dev;   // if set, n = min(n, *n_dev) at run time (rank known on device only)
    int tri = 0;        // 1: A lower triangular (an output row tile at i0 needs k < i0 + BM);
                        // 2: op(B) upper triangular (a column tile at j0 needs k < j0 + BN)
};

// Single-precision variant used by the mixed-precision policy: operands are
// FP64 in memory, products are formed in FP32 with FP32 accumulation and the
// result is written back in FP64.
// d_tile_off: prefix sums of the tasks' tile counts (ntasks + 1 entries),
// followed by the group table: entry g is the task that holds tile 32 g
// (ceil(total_tiles / 32) entries), so a CTA finds its task in a step or two.
constexpr int GEMM_GROUP = 32;
void launch_gemm_batched(const GemmTask *d_tasks, const int *d_tile_off, int ntasks,
                         int total_tiles, cudaStream_t st, bool fp32 = false);
void launch_gemm_single(const GemmTask &t, cudaStream_t st);
// FP64 variant with 128 x 32 output tiles for outputs a rank wide (n <= 32, or
// n capped on the device by n_dev); tiles_m of its tasks must be ceil(m / 128).
constexpr int GEMM_NARROW_M = 128, GEMM_NARROW_N = 32;
void launch_gemm_batched_narrow(const GemmTask *d_tasks, const int *d_tile_off, int ntasks, int total_tiles,
                                cudaStream_t st);
// Algorithmic work of the tasks whose n is read on the device (n_dev): adds
// 2 m n k flops and 8 (m k + k n + m n (2 with beta)) bytes with the device's
// n to acc[0], acc[1] (profiling; launched after the GEMMs on the same stream).
void launch_gemm_devcount(const GemmTask *d_tasks, int ntasks, double *acc, cudaStream_t st);

inline int gemm_tiles_m(int m) { return (m + 63) / 64; }
inline int gemm_tiles(const GemmTask &t) { return gemm_tiles_m(t.m) * gemm_tiles_m(t.n); }
inline GemmTask make_gemm(int opA, int opB, int m, int n, int k, double alpha, const double *A,
                          int lda, const double *B, int ldb, double beta, double *C, int ldc,
                          int lower = 0) {
    GemmTask t;
    t.A = A; t.B = B; t.C = C;
    t.m = m; t.n = n; t.k = k;
    t.lda = lda; t.ldb = ldb; t.ldc = ldc;
    t.opA = opA; t.opB = opB; t.lower = lower;
    t.tiles_m = gemm_tiles_m(m);
    t.alpha = alpha; t.beta = beta;
    t.n_dev = nullptr;
    return t;
}

// ------------------------------------------------------------ generation ----
struct CovTask {
    double *out;
    int ld;
    int r0, c0;     // global row / column offsets
    int nr, nc;
};
struct CovParams {
    const double *pts;  // [ndim][N]
    int N, ndim, kind;
    double beta, sigma, noise;
    double wave_k, add_diag;   // electrodynamics kinds; add_diag also the mesh kinds' regularisation
    int rbf;                   // mesh kinds: HICMA_TLR_RBF_* basis function
    double inv_radius;         // mesh kinds: 1 / radius
};
void launch_cov_batched(const CovParams &p, const CovTask *d_tasks, int ntasks, int max_nr,
                        int max_nc, cudaStream_t st);
// Gaussian N(0,1) matrix (counter based, seeded), column-major rows x cols.
void launch_gaussian(double *out, int rows, int cols, int ld, unsigned long long seed,
                     cudaStream_t st);
// randtlr bases of nblk block rows from their in-place QRs Xr and formed Q
// factors (each NB x K, ld NB, consecutive): pts[:, j] = sign(R_jj) Q[:, j],
// pts[:, K + j] = decay^j pts[:, j] at rows (m0 + b) * NB + i.  pts is N x 2K.
void launch_randtlr_finish(const double *Xr, const double *Q, int nb, int K, int nblk, int m0, double *pts, int N,
                           double decay, cudaStream_t st);
constexpr int RANDTLR_KMAX = 64;            // singular directions kept (0.5^64 is below FP64 resolution)
constexpr double RANDTLR_DECAY = 0.5;       // hicma_parsec/testing_dpotrf.c:318
constexpr unsigned long long RANDTLR_SEED_XOR = 0x52414E44544C5200ull;

// --------------------------------------------------------------- copies -----
struct CopyTask {
    const double *src;
    double *dst;
    int lds, ldd;
    int rows, cols;
    double alpha;
    double beta;        // dst = alpha src + beta dst (beta = 0: plain copy)
};
void launch_copy_batched(const CopyTask *d_tasks, int ntasks, int max_cols, cudaStream_t st);
void launch_zero_upper(double *A, int n, int lda, cudaStream_t st);
void launch_set_identity(double *A, int n, int lda, cudaStream_t st);

// ------------------------------------------------- recompression helpers ---
// Explicit K x K upper triangular factor of [Cu, Au] (K = rc + ra) after the
// projection of Au on the orthonormal Cu: RU = [[I, Pu], [0, R(Wu)]].
struct AssembleTask {
    const double *Pu;   // rc x ra (ld rc)
    const double *Wu;   // QR'd residual, R in its top ra x ra (ld nb)
    double *RU;         // K x K (ld K)
    int rc, ra, nb;
};
void launch_assemble_r(const AssembleTask *d_tasks, int ntasks, cudaStream_t st);
// Two rounds of block Gram-Schmidt of W (nb x ra, ld nb) against the
// orthonormal C (nb x rc, ld nb): W -= C (C^T W) twice, P = sum of the two
// coefficient blocks (rc x ra, ld rc); P2 is scratch of the same size.
struct ProjTask {
    const double *C;
    double *W;
    double *P, *P2;
    int nb, rc, ra;
};
void launch_bcgs2(const ProjTask *d_tasks, int ntasks, cudaStream_t st);
// P = C^T W (rc x ra, ld rc) with C nb x rc and W nb x ra (ld nb): one CTA per
// product, split-K over its warps, fixed-order reduction.
struct GramTask {
    const double *C, *W;
    double *P;
    int nb, rc, ra;
};
void launch_gram_batched(const GramTask *d_tasks, int ntasks, cudaStream_t st);
// fail[i] = 1 when the P of task i (a Q^T Q, rc == ra) is not the identity to
// within thr between nonzero columns, else 0 (one warp per task).
void launch_orth_check(const GramTask *d_tasks, int ntasks, double thr, int *fail, cudaStream_t st);

// ------------------------------------------------------ precision policy ---
// out = sum of squares of X (rows x cols, ld): one CTA per task.
struct NormTask {
    const double *X;
    int rows, cols, ld;
    double *out;
};
void launch_sumsq_batched(const NormTask *d_tasks, int ntasks, cudaStream_t st);
// out[i] += sum_k parts[k * len + i] for k = 0 .. nparts-1 in order.
void launch_accumulate(double *out, const double *parts, int nparts, long long len, cudaStream_t st);
// Per recompression: its products run in FP32 when na * nb <= thr2 (squared
// Frobenius norms of the two factor tiles); sel32 / sel64 receive n or 0 and
// serve as the device-side column counts of the two launches.
struct SelTask {
    const double *na, *nb;
    int *sel64, *sel32;
    int n;
};
void launch_precision_select(const SelTask *d_tasks, int ntasks, double thr2, int *count, cudaStream_t st);

// ---------------------------------------------------------------- POTRF -----
// Tile Cholesky (+ inverse when X is given, X zeroed by the caller) in one
// persistent launch of `grid` CTAs; n <= potrf_tile_max_n().  cnt: scratch of
// potrf_tile_scratch_ints(n) ints; D: (n/64 rounded up) * 4096 doubles when X
// is null.  *timeout is set if a bounded device wait gave up.
int potrf_tile_max_n();
// Test of the bounded dependency wait of the tile POTRF: nblocks CTAs wait on
// counters nothing sets (CTA 0 with limit0 polls, the others limit1); cnt has
// 2 + nblocks zeroed ints, timeout one zeroed int.
int launch_wait_probe(int *cnt, int *timeout, int nblocks, long long limit0, long long limit1, cudaStream_t st);
size_t potrf_tile_scratch_ints(int n);
int launch_potrf_tile(double *A, int lda, int n, double *X, int ldx, double *D, int *cnt, int *info,
                      int info_base, int *timeout, int grid, cudaStream_t st);
// Factor the jb x jb diagonal block at A (lda) in place (lower), write its
// inverse into Dinv (ldd); on failure set *info = info_base + j + 1 once.
void launch_potrf_diag(double *A, int lda, int jb, double *Dinv, int ldd, int *info,
                       int info_base, cudaStream_t st);

// --------------------------------------------------------- tall-skinny QR ---
// Blocked Householder QR of an m x K matrix X (ld), one CTA per task.  X is
// overwritten by R (upper) and the reflectors (below the diagonal); tau[K]
// and the block-reflector T factors (ceil(K/PB) blocks of PB x PB) are
// written.  PB is chosen from m by qr_panel_width().
struct QRTask {
    double *X;
    double *tau;
    double *T;
    int m, K, ld;
};
int qr_panel_width(int m);
size_t qr_smem_bytes(int m);
void launch_qr_batched(const QRTask *d_tasks, int ntasks, int m_max, cudaStream_t st);

// out (m x r, ldo) = Q [S; 0] with Q from a QRTask factorisation and S K x r
// (lds).  r is read from *r_dev (device) at run time, capped by r_cap.
struct QApplyTask {
    const double *X;
    const double *T;
    const double *S;
    double *out;
    const int *r_dev;
    int m, K, ld, lds, ldo;
    int r_cap;
};
void launch_qapply_batched(const QApplyTask *d_tasks, int ntasks, int m_max, cudaStream_t st);

// QR of an nb x K matrix X = [X1 (nb x k1, ld1), X2 (nb x k2, ld2)] by
// randomized CholeskyQR (a 256-row CountSketch factored by shifted
// CholeskyQR3, then one CholeskyQR pass over the rows; one CTA per task; X is
// read, not changed): R (upper, K x K, ld K) and, if Q is set, Q (nb x K,
// ld nb; may equal Z).  With Rinv set instead (and Q null), Z keeps
// Y = X Rs^-1 and Rinv (K x K, ld K) receives Rc^-1, so that Q = Z Rinv.  Z
// (nb x K, ld nb) is written only when Q or Rinv is set.  K = k1 + k2 <=
// rcholqr_kmax().  flags[0] counts the null pivots (columns of Y dependent on
// the ones before them, or zero) met by the passes over the rows, flags[1]
// the passes repeated because the sketch missed a direction.
struct CQTask {
    const double *X1, *X2;
    double *Z;
    double *R;
    double *Q;
    int nb, k1, k2, ld1, ld2;
    double *Rinv = nullptr;
};
int rcholqr_kmax();
int rcholqr_bucket(int K);   // width of the kernel instance that takes K
// form_q: every task of the launch sets Q (and none sets Rinv); otherwise none sets Q
void launch_rcholqr_batched(const CQTask *d_tasks, int ntasks, int kmax, bool form_q, int *flags,
                            cudaStream_t st);

// ------------------------------------------------------------- core SVD -----
// M = RU RV^T (RU, RV: K x K upper from the QRs; RU == nullptr means I),
// one-sided Jacobi SVD, truncation and outputs SU = U_r, SV = V_r Sigma_r
// (K x r each, ld K).  mode 0: absolute sigma >= tol (recompression);
// mode 1: relative Frobenius tol (generation, with reject rules).
struct CoreTask {
    const double *RU;    // K x K upper (ld ldru), nullptr = identity
    const double *RV;    // K x K upper (ld ldrv)
    double *SU;          // out: K x K, left singular vectors sorted by decreasing sigma
    double *RUc;         // out (if RU): clean copy of RU, K x K, zeros below the diagonal
    double *work;        // core_work_doubles(K) doubles when K > core_smem_kmax()
    int *rank_out;       // rank map entry (may be null)
    int *rank_task;      // per-task rank for the apply steps
    int K, ldru, ldrv;
};
struct CoreParams {
    int mode;
    double tol;
    int maxrank;
    int fixed_rank;
    int nb;              // tile size (generation reject rule r >= nb/2)
    int *overflow;       // device counter of capped recompressions
    int *sweeps;         // device counter of Jacobi sweeps (diagnostics, may be null)
};
int core_smem_kmax();
// Global scratch (doubles) of one core with K > core_smem_kmax().
size_t core_work_doubles(int K);
// All tasks of one launch should have K <= kmax; shared memory is sized from kmax.
void launch_core_svd_batched(const CoreTask *d_tasks, int ntasks, int kmax, const CoreParams &p,
                             cudaStream_t st);

// ---------------------------------------------------------------- misc ------
// sum of 2*log(diag) over n diagonal entries of ntiles tiles, into *out
void launch_logdiag_sum(const double *const *d_tiles, int ntiles, int n, int ld, double *out,
                        cudaStream_t st);

// sum of squares of X - Y (Y may be null) into *out (nblocks partials in
// `partial`); sym_lower: Frobenius^2 of the symmetric matrix in the lower part
void launch_sumsq(const double *X, const double *Y, int m, int n, long long ld, int sym_lower, double *partial,
                  int nblocks, double *out, cudaStream_t st);
// Record the message returned by hicma_tlr_last_error() for this thread.
void tlr_set_error(const char *msg);
}  // namespace tlr
