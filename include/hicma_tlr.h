/*
 * hicma_tlr.h -- C ABI of the B200 tile-low-rank (TLR) Cholesky engine.
 *
 * This is the drop-in boundary for HiCMA-PaRSEC's factorization path.  Every
 * entry point below names the reference interface it replaces (paths are
 * relative to the reference project root).  Plain C types only: opaque
 * handles, pointers and sizes.  All device work runs on the CUDA stream owned
 * by the context; calls return after the work is complete unless stated.
 *
 * Storage conventions (shared with the reference):
 *   - tiles are NB x NB, column-major, ld = NB (BLKLDD);
 *   - a tile (m, n) with m - n < band_size is dense; an off-band tile is the
 *     packed pair [U, V] (U: NB x r at offset 0, V: NB x r at offset NB*r) with
 *     A(m, n) ~= U V^T (hicma_parsec/HiCMA_dpotrf_L_2flow.jdf:386,518-519);
 *   - the rank map is an NT x NT column-major int array, entry n*NT + m for
 *     tile (m, n), -1 on the band (hicma_parsec/testing_dpotrf.c:441-453).
 *   - U has orthonormal columns; V carries the singular values.
 *
 * Return codes: 0 on success; > 0 is the reference's Cholesky INFO
 * (k*NB + i, the order of the first leading minor that is not positive
 * definite, hicma_parsec/HiCMA_dpotrf_L_2flow.jdf:241-242); < 0 is one of
 * the HICMA_TLR_ERR_* codes below.  Unlike the reference (which returns a NULL
 * taskpool and then 0, hicma_parsec/hicma_parsec.c:595), argument errors are
 * reported as HICMA_TLR_ERR_ARG.
 */
#ifndef HICMA_TLR_H
#define HICMA_TLR_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HICMA_TLR_SUCCESS              0
#define HICMA_TLR_ERR_ARG             -1  /* invalid argument                        */
#define HICMA_TLR_ERR_CUDA            -2  /* CUDA runtime error                      */
#define HICMA_TLR_ERR_OOM             -3  /* device memory exhausted                 */
#define HICMA_TLR_ERR_RANK_OVERFLOW   -4  /* a tile needs a rank above maxrank
                                             (STARS-H INFO=-1, STARSH_gen.jdf:169-171) */
#define HICMA_TLR_ERR_TIMEOUT         -5  /* a bounded device wait gave up           */
#define HICMA_TLR_ERR_STATE           -6  /* call out of order (e.g. solve before factor) */
#define HICMA_TLR_ERR_NOT_SUPPORTED   -7  /* e.g. uplo = Upper, N % NB != 0          */

/* uplo values of DPLASMA (dplasmaUpper / dplasmaLower). */
#define HICMA_TLR_UPPER 121
#define HICMA_TLR_LOWER 122

/* -D problem kinds (hicma_parsec/testing_dpotrf.c:12, :315-381). */
#define HICMA_TLR_KIND_RANDTLR   0   /* random TLR, equal ranks (testing_dpotrf.c:315-321) */
#define HICMA_TLR_KIND_ED_SIN_2D 1   /* sin(k r)/r, 2D (testing_dpotrf.c:325-334) */
#define HICMA_TLR_KIND_SQEXP_2D  2
#define HICMA_TLR_KIND_SQEXP_3D  3
#define HICMA_TLR_KIND_EXP_3D    4
#define HICMA_TLR_KIND_ED_SIN_3D 5   /* sin(k r)/r, 3D (testing_dpotrf.c:359-365) */
#define HICMA_TLR_KIND_MD_VIRUS  6   /* RBF over mesh points read from a file (testing_dpotrf.c:366-374) */
#define HICMA_TLR_KIND_MD_CUBE   7   /* RBF over the nodes of a cube (testing_dpotrf.c:375-381) */

/* Radial basis functions of the mesh kinds (-B, hicma_parsec.c:80), of
 * s = r / radius; the CTPS and Wendland functions vanish for s >= 1. */
#define HICMA_TLR_RBF_GAUSSIAN  0   /* exp(-s^2)                  */
#define HICMA_TLR_RBF_EXPON     1   /* exp(-s)                    */
#define HICMA_TLR_RBF_INVQUAD   2   /* 1 / (1 + s^2)              */
#define HICMA_TLR_RBF_INVMQUAD  3   /* 1 / sqrt(1 + s^2)          */
#define HICMA_TLR_RBF_MATERNC1  4   /* (1 + s) exp(-s)            */
#define HICMA_TLR_RBF_MATERNC2  5   /* (1 + s + s^2 / 3) exp(-s)  */
#define HICMA_TLR_RBF_TPS       6   /* s^2 log s (0 at s = 0)     */
#define HICMA_TLR_RBF_CTPS      7   /* (1 - s)^5 for s < 1        */
#define HICMA_TLR_RBF_WENDLAND  8   /* (1 - s)^4 (4 s + 1) for s < 1 */

/* Precision policy of the factorization (no reference counterpart). */
#define HICMA_TLR_PREC_FP64   0   /* everything in FP64                              */
#define HICMA_TLR_PREC_MIXED  1   /* off-band low-rank products of small-norm tiles in
                                     FP32; band, diagonal and truncation stay FP64     */

typedef struct hicma_tlr_ctx_s  hicma_tlr_ctx;   /* device, stream, workspace      */
typedef struct hicma_tlr_desc_s hicma_tlr_desc;  /* device tile store of a matrix */

/* STARS-H problem (starsh_ssdata_generate / starsh_eddata_generate /
 * starsh_randtlr_generate arguments, hicma_parsec/testing_dpotrf.c:300-365).
 * Spatial statistics (kinds 2-4): A_ij = sigma * k(|x_i - x_j|) + noise * [i == j].
 * Electrodynamics (kinds 1, 5): A_ij = sin(wave_k * r) / r with r = |x_i - x_j|,
 * and add_diag where r == 0.  randtlr (kind 0): tile (m, n) = Q_m diag(S) Q_n^T
 * + add_diag * [m == n] I, Q_m a random orthonormal basis of block row m
 * (first min(NB, 64) columns; seeded by seed), S_k = 0.5^k (decay of
 * testing_dpotrf.c:318).  randtlr has no points: hicma_tlr_points rejects it
 * and hicma_tlr_generate builds the bases on the device (points must be NULL).
 * Mesh kinds (6, 7): A_ij = phi(|x_i - x_j| / radius), phi the basis function
 * rbf_kernel, plus add_diag where i == j (the reference passes add_diag as the
 * regularisation, testing_dpotrf.c:371,379).  Kind 7's points come from
 * hicma_tlr_points; kind 6 reads a mesh (hicma_tlr_points_mesh) and the caller
 * passes the points to hicma_tlr_generate. */
typedef struct {
    int    kind;      /* HICMA_TLR_KIND_*                                   */
    double beta;      /* length scale (reference default 0.1)               */
    double nu;        /* smoothness, unused by sqexp/exp (default 0.5)      */
    double noise;     /* nugget added on the diagonal (reference 0.1)       */
    double sigma;     /* variance (default 1.0)                             */
    unsigned long long seed;  /* point placement seed (reference srand(0)) */
    double wave_k;    /* wave number of kinds 1, 5 (default 50, hicma_parsec.c:188)        */
    double add_diag;  /* diagonal of kinds 0, 1, 5, 6, 7; <= 0 means N (hicma_parsec.c:289-291) */
    int    rbf_kernel;  /* HICMA_TLR_RBF_* of kinds 6, 7 (-B)                            */
    double radius;      /* shape radius of kinds 6, 7, > 0 (-R)                          */
    int    numobj;      /* kind 6: copies of the mesh in the population (-K; <= 0 means 1) */
    int    order;       /* kinds 6, 7: 0 no reordering, 1 Morton (-O; 2 Hilbert rejected) */
    double density;     /* kind 6: packing density of the copies, -1 random (-S)        */
} hicma_tlr_problem;

/* ---------------------------------------------------------------- setup -- */

/* setup_parsec / cleanup_parsec (hicma_parsec/hicma_parsec.h:201-204).
 * workspace_bytes = 0 picks a default sized from free device memory. */
int hicma_tlr_init(int device, size_t workspace_bytes, hicma_tlr_ctx **ctx);
int hicma_tlr_fini(hicma_tlr_ctx *ctx);
/* The CUDA stream (cudaStream_t) the context launches on. */
void *hicma_tlr_stream(hicma_tlr_ctx *ctx);
/* Last error message of this thread ("" if none). */
const char *hicma_tlr_last_error(void);

/* Descriptor = dcA (band + off-band) + dcAr of hicma_parsec/testing_dpotrf.c:418-453.
 * Off-band tiles get fixed slots of capacity maxrank columns for U and V. */
int hicma_tlr_desc_create(hicma_tlr_ctx *ctx, int N, int NB, int maxrank, int band_size,
                          hicma_tlr_desc **A);
int hicma_tlr_desc_destroy(hicma_tlr_desc *A);
int hicma_tlr_desc_info(const hicma_tlr_desc *A, int *N, int *NB, int *NT, int *maxrank,
                        int *band_size);
/* Device-to-device copy of all tiles, ranks and points.  N, NB, maxrank and the
 * band size dst was created with must equal src's; a band src has since widened
 * (hicma_tlr_band_regenerate) is adopted by dst. */
int hicma_tlr_desc_copy(hicma_tlr_ctx *ctx, const hicma_tlr_desc *src, hicma_tlr_desc *dst);

/* ----------------------------------------------------------- generation -- */

/* Points of the problem (starsh_ssdata_generate, testing_dpotrf.c:305-312,
 * 336-358): jittered grid, Morton order.  points is [ndim][N] (SoA).
 * md-3d-cube (kind 7, starsh_generate_3d_rbf_mesh_coordinates_cube,
 * testing_dpotrf.c:375-381; STARS-H's generator is absent from the reference
 * tree): the cell centres ((i + 1/2) / s, (j + 1/2) / s, (k + 1/2) / s) of an
 * s x s x s grid on the unit cube, s = ceil(cbrt(N)), in Morton order when
 * prob->order == 1 and in x-fastest order when 0; the first N are returned. */
int hicma_tlr_points(const hicma_tlr_problem *prob, int N, double *points);

/* Points of the md-3d-virus problem (starsh_generate_3d_rbf_mesh_coordinates_virus,
 * testing_dpotrf.c:366-374; STARS-H's reader is absent from the reference tree):
 * the mesh file holds one object's nodes as whitespace-separated x y z triples
 * ('#' starts a comment).  prob->numobj copies of the object (centred on its
 * bounding-box centre, diameter d = the box diagonal) are placed on a cubic
 * lattice of side ceil(cbrt(numobj)), spacing d * cbrt(pi / (6 density)) (the
 * copies' bounding spheres fill the fraction density of space, at most pi/6,
 * where they touch); density <= 0 places the centres uniformly at random
 * (seeded by prob->seed) in a cube of side 2 d cbrt(numobj).  The population
 * is Morton ordered when prob->order == 1, and its first N nodes are returned
 * as [3][N]; N larger than numobj times the node count is an argument error. */
int hicma_tlr_points_mesh(const hicma_tlr_problem *prob, const char *mesh_file, int N, double *points);

/* STARSH_gen (hicma_parsec/hicma_parsec.h:187-198; STARSH_gen.jdf:342-369):
 * band tiles dense, off-band tiles compressed to tolerance tol and at most
 * maxrank columns.  points may be NULL (then hicma_tlr_points is used).
 * Ar (host, NT*NT, may be NULL) receives the rank map.  *info = -1 when a
 * tile is rejected (STARSH_gen.jdf:169-171). */
int hicma_tlr_generate(hicma_tlr_ctx *ctx, int uplo, hicma_tlr_desc *A, int *Ar,
                       const hicma_tlr_problem *prob, const double *points,
                       double tol, int maxrank, int band_size, int send_full_tile,
                       int *info);

/* parsec_rank_gather (hicma_parsec.h:124-127): device rank map -> host. */
int hicma_tlr_rank_gather(hicma_tlr_ctx *ctx, hicma_tlr_desc *A, int *rank_array, int band_size);

/* Rank history of the last factorization on A (the dcRank record gathered by
 * parsec_rank_print, hicma_parsec/rank_print.jdf:62-69, filled at
 * HiCMA_dpotrf_L_2flow.jdf:353-361,683-691,1101-1106): per off-band tile
 * (m, n) at [n*NT + m] the rank it entered the factorization with, the
 * smallest and largest rank it held, and its final rank; -1 for band and
 * upper tiles.  Any pointer may be NULL.  HICMA_TLR_ERR_STATE before the
 * first factorization of A. */
int hicma_tlr_rank_history(hicma_tlr_desc *A, int *initial, int *minimum, int *maximum, int *final_rank);

/* op_counts (hicma_parsec/op_counts.h:10-72): the reference's flop model of one
 * kernel call ('q' geqrf m=a n=b, 'c' potrf n=a, 't' trsm m=a n=b side=c,
 * 'm' gemm a*b*c, 's' svd n=a, 'o' ormqr m=a n=b k=c side=d, 'r' trmm m=a n=b
 * side=c), with its unsigned wrap-around and float32 casts; the counters of
 * hicma_tlr_dpotrf_L and the band auto-tuning use it. */
unsigned long hicma_tlr_op_counts(char op, unsigned long a, unsigned long b, unsigned long c, unsigned long d);

/* HICMA_get_stat2 (hicma_parsec/hicma_internal.c:52-71). */
int hicma_tlr_rank_stat(const int *rank_array, int NT, int band_size, int *minrk, int *maxrk,
                        double *avgrk);

/* parsec_band_size_auto_tuning (hicma_parsec.h:111-115;
 * band_size_auto_tuning.jdf:201-318).  Returns the tuned band size. */
int hicma_tlr_band_autotune(const int *rank_array, int NT, int NB, int verbose);

/* parsec_band_regenerate (hicma_parsec.h:94-100; band_regenerate.jdf:124-143):
 * switch the descriptor to band_size and regenerate the dense band tiles. */
int hicma_tlr_band_regenerate(hicma_tlr_ctx *ctx, int uplo, hicma_tlr_desc *A,
                              const hicma_tlr_problem *prob, int band_size);

/* --------------------------------------------------------- factorization -- */

/* HiCMA_dpotrf_L (hicma_parsec/hicma_parsec.h:38-56; hicma_parsec.c:463-646).
 * Lower TLR Cholesky in place.  Ar (host, may be NULL) receives the final
 * rank map.  tileopcounters (NT*NT) and opcounters (>= 1) are incremented
 * with the reference's op_counts model (hicma_parsec/op_counts.h).
 * critical_path_time[6] receives seconds spent in POTRF, TRSM and SYRK of the
 * panel critical path, then total factorization, TRSM+SYRK+GEMM of all
 * panels and the recompression share.  hmb is accepted and ignored (the
 * recursive sub-tiling of the reference is replaced by multi-CTA kernels).
 * *two_flow (may be NULL): 0 on entry with band_size 1 selects the
 * reference's 3-flow variant, which computes the same updates and is served
 * by the same path; it is left 0 then and set to 1 otherwise
 * (hicma_parsec.c:517-573).
 * Returns the reference's info (0, k*NB+i) or a negative error code. */
int hicma_tlr_dpotrf_L(hicma_tlr_ctx *ctx, int uplo, hicma_tlr_desc *A, int *Ar,
                       double acc, int fixed_rank, int maxrank, int *lookahead,
                       int band_size, int hmb, int compmaxrank, int send_full_tile,
                       int *two_flow, unsigned long *tileopcounters,
                       unsigned long *opcounters, double *critical_path_time, int verbose);

/* HiCMA_dpotrf_L with the reference's full parameter list, the Rank
 * descriptor included (hicma_parsec/hicma_parsec.h:38-56): the same call as
 * hicma_tlr_dpotrf_L, then, when Rank (host, 4*NT*NT ints) is not NULL and the
 * factorization ran (a return value >= 0), the dcRank record of every tile
 * (hicma_parsec/testing_dpotrf.c:619-635, filled at
 * HiCMA_dpotrf_L_2flow.jdf:353-361,683-691,1101-1106): tile (m, n) at
 * [(n*NT + m)*4 + q], q = 0 initial, 1 minimum, 2 maximum, 3 final rank; -1 for
 * band and upper tiles (hicma_tlr_rank_history in one array). */
int hicma_tlr_dpotrf_L_rank(hicma_tlr_ctx *ctx, int uplo, hicma_tlr_desc *A, int *Ar, int *Rank,
                            double acc, int fixed_rank, int maxrank, int *lookahead,
                            int band_size, int hmb, int compmaxrank, int send_full_tile,
                            int *two_flow, unsigned long *tileopcounters,
                            unsigned long *opcounters, double *critical_path_time, int verbose);

/* Precision policy for later hicma_tlr_dpotrf_L calls on this context. */
int hicma_tlr_set_precision(hicma_tlr_ctx *ctx, int precision);

/* Autotuner (no reference counterpart): measures on this device, for tile size
 * NB, the choices that have several valid kernels and keeps the fastest in the
 * context for later calls:
 *   tuning[0]  widest rank-wide GEMM output sent to the 128 x 32 tile variant
 *              instead of 64 x 64 tiles (candidates 32, 48, 64, 96, 128, up to
 *              maxrank; default 32), timed on batches shaped like the
 *              recompression products;
 *   tuning[1]  CTAs of the persistent tile POTRF (candidates SMs/2, SMs, 2 SMs;
 *              0 = one per SM, the default), timed on an SPD NB x NB tile.
 * Each candidate runs reps (1..50) times; medians in ms_out[11] (may be NULL):
 * [0..2] POTRF per grid, then for widths 48, 64, 96, 128 the 128 x 32 and the
 * 64 x 64 variant (NaN where not measured).  Uses the context workspace.
 * _get / _set read or restore a table (e.g. one cached from an earlier run). */
int hicma_tlr_autotune(hicma_tlr_ctx *ctx, int NB, int maxrank, int reps, int *tuning, double *ms_out);
int hicma_tlr_tuning_get(hicma_tlr_ctx *ctx, int *tuning);
int hicma_tlr_tuning_set(hicma_tlr_ctx *ctx, const int *tuning);

/* Asynchronous form (HiCMA_dpotrf_L_2flow_New / _Destruct,
 * hicma_parsec/hicma_parsec_internal.h:295-315): _start enqueues, _wait
 * completes and returns the info. */
int hicma_tlr_dpotrf_L_start(hicma_tlr_ctx *ctx, hicma_tlr_desc *A, double acc, int fixed_rank,
                             int maxrank);
int hicma_tlr_dpotrf_L_wait(hicma_tlr_ctx *ctx, hicma_tlr_desc *A, int *Ar);

/* ------------------------------------------------------ check / results -- */

/* STARSH_check (hicma_parsec.h:162-169; STARSH_check.jdf:90-143): expand the
 * lower triangle to a dense host N x N column-major matrix (leading dim ld). */
int hicma_tlr_uncompress(hicma_tlr_ctx *ctx, hicma_tlr_desc *A, double *dense, long ld);

/* Host copy of one tile.  Dense tiles: NB*NB doubles.  Low-rank tiles: the
 * reference's packed [U, V] (2*NB*rank doubles); *rank receives the rank
 * (-1 for dense tiles).  buf may be NULL to query the rank only. */
int hicma_tlr_tile_get(hicma_tlr_ctx *ctx, hicma_tlr_desc *A, int m, int n, double *buf,
                       int *rank);
int hicma_tlr_tile_set(hicma_tlr_ctx *ctx, hicma_tlr_desc *A, int m, int n, const double *buf,
                       int rank);

/* Whole-matrix host <-> device transfer in the reference's layout: all band
 * tiles (row m, then n = m-band+1..m) followed by the packed [U,V] of every
 * off-band tile (row m, then n = 0..m-band), each packed with its own rank.
 * bytes_needed returns the buffer size for the current ranks. */
int hicma_tlr_store_bytes(hicma_tlr_ctx *ctx, hicma_tlr_desc *A, size_t *bytes_needed);
int hicma_tlr_store_get(hicma_tlr_ctx *ctx, hicma_tlr_desc *A, double *buf, int *Ar);
int hicma_tlr_store_set(hicma_tlr_ctx *ctx, hicma_tlr_desc *A, const double *buf, const int *Ar);

/* Copy-out during the factorization (no reference counterpart): the next
 * hicma_tlr_dpotrf_L on A copies each tile column of the factor into buf as
 * soon as the column is final, on a copy stream that overlaps the remaining
 * panels.  Layout, column n = 0..NT-1 in order: the band tiles (m, n),
 * m = n..min(NT-1, n+band-1), NB x NB each, then the packed [U, V] of the
 * off-band tiles (m, n), m = n+band..NT-1, NB x rank each with the final ranks
 * (hicma_tlr_rank_gather).  buf should be page-locked for the copies to
 * overlap.  When the call returns, hicma_tlr_last_stats s[15] holds the bytes
 * written, or -1 if a column did not fit in `bytes` (the factor is complete on
 * the device either way; hicma_tlr_store_get still works).  One factorization
 * consumes the arming; buf = NULL disarms. */
int hicma_tlr_store_stream(hicma_tlr_ctx *ctx, hicma_tlr_desc *A, double *buf, size_t bytes);

/* Additions beyond the reference (no reference counterpart; testing_dpotrf.c stops at
 * the factor).  Require a factored descriptor. */
int hicma_tlr_logdet(hicma_tlr_ctx *ctx, hicma_tlr_desc *A, double *logdet);
/* Solve A X = B in place; B is host N x nrhs column-major (leading dim ldb). */
int hicma_tlr_solve(hicma_tlr_ctx *ctx, hicma_tlr_desc *A, int nrhs, double *B, long ldb);
/* Gaussian log-likelihood -1/2 (y^T A^-1 y + log det A + N log 2 pi). */
int hicma_tlr_loglik(hicma_tlr_ctx *ctx, hicma_tlr_desc *A, const double *y, double *loglik,
                     double *logdet, double *x);

/* One serving request (no reference counterpart): generate prob on a new
 * N x N descriptor with tile NB (STARSH_gen), widen the band over tiles the rank
 * rule rejected, else auto-tune it when autoband != 0
 * (parsec_band_size_auto_tuning, band_size_auto_tuning.jdf:201-318), regenerate
 * the band (parsec_band_regenerate), factor (HiCMA_dpotrf_L) and evaluate the
 * log-likelihood of y (host, N).  maxrank <= 0 means min(NB/2 - 1, 200).
 * Returns 0 with loglik, logdet, x (host N, may be NULL) and band (may be
 * NULL) set; a positive return is the factorization's info (not positive
 * definite); negative returns are errors.  The descriptor is released before
 * returning; the context's workspace is reused. */
int hicma_tlr_serve_loglik(hicma_tlr_ctx *ctx, const hicma_tlr_problem *prob, int N, int NB, double acc,
                           int maxrank, int autoband, const double *y, double *loglik, double *logdet,
                           double *x, int *band);

/* Statistics of the last factorization on A: [0] seconds, [1] TLR flops
 * (op_counts model), [2] recompressions capped at maxrank, [3] number of
 * launches of library kernels, [4] POTRF s, [5] TRSM s, [6] SYRK s,
 * [7] GEMM/recompression s, [8] Jacobi sweeps summed over all cores, [9] recompressions
 * whose products ran in FP32 under HICMA_TLR_PREC_MIXED, [10] op count of the
 * critical path POTRF(k) -> TRSM(k+1,k) -> SYRK(k,k+1) (the reference's op_path;
 * the rest of [1] is its op_offpath), [11] null pivots met by the passes of
 * the recompressions' randomized CholeskyQR over the rows (columns dependent on
 * the ones before them, or zero; 0 in the usual run), [12] seconds the device sat idle between panels (from the end
 * of a panel's last kernel to the start of the next panel's first, CUDA
 * events), [13] panels, [14] CholeskyQR passes over a stack's rows repeated
 * because its sketch missed a direction (0 in the usual run), [15] bytes copied
 * out by hicma_tlr_store_stream (-1: the buffer was too small; 0: not armed).
 * nstats <= 16. */
int hicma_tlr_last_stats(hicma_tlr_desc *A, double *stats, int nstats);

/* --check of the reference driver (check_dpotrf2 and check_diff,
 * hicma_parsec/testing_dpotrf.c:111-230, flow :642-903) on the device:
 * res_llt = ||L L^T - A||_F / ||A||_F against the exact (unapproximated)
 * covariance; res_diff = ||L - L0|| / ||L|| with L0 the dense Cholesky of the
 * approximate matrix held (unfactored) in A0 (A0 may be NULL).  Allocates
 * three dense N x N device buffers, so it is meant for moderate N. */
int hicma_tlr_check(hicma_tlr_ctx *ctx, hicma_tlr_desc *L, const hicma_tlr_problem *prob,
                    hicma_tlr_desc *A0, double *res_llt, double *res_diff);

/* Full-size counterpart of check_dpotrf2 (hicma_parsec/testing_dpotrf.c:111-180)
 * for N where no N x N matrix fits: with nprobe (1..64) seeded Gaussian probe
 * vectors Z, res_est = ||(A - L L^T) Z||_F / ||A Z||_F, A the exact covariance
 * (regenerated on the device tile by tile), L the TLR factor in L.  Uses the
 * context workspace (4 N nprobe doubles plus tile chunks). */
int hicma_tlr_check_probe(hicma_tlr_ctx *ctx, hicma_tlr_desc *L, const hicma_tlr_problem *prob, int nprobe,
                          unsigned long long seed, double *res_est);

/* Per-kernel-class device timing (CUDA events around launches on the context
 * stream).  Classes: 0 GEMM, 1 QR, 2 Q-apply, 3 core SVD, 4 tile POTRF,
 * 5 covariance generation, 6 copies, 7 other, 8 Gram-Schmidt projections, then the batched
 * GEMMs by call site: 0 recompression outputs and the rest, 9 recompression products (Y),
 * 10 TRSM, 11 SYRK, 12 dense band cases, 13 generation; 14 split-K inner products (Gram kernel),
 * 15 QR factors by randomized CholeskyQR (both sides of narrow recompressions, the generation
 * range finder).  out[4*k + j]: j = 0 launches,
 * 1 seconds, 2 algorithmic flops, 3 algorithmic bytes.  Enabling resets. */
int hicma_tlr_prof_enable(hicma_tlr_ctx *ctx, int on);
int hicma_tlr_prof_read(hicma_tlr_ctx *ctx, double *out, int nclass);

/* ------------------------------------------- kernel-level entry points -- */
/* Device pointers; used by the parity tests and by callers that manage their
 * own memory.  stream may be NULL for the context stream.  These replace the
 * per-tile bodies of the reference's task classes. */

/* STARS-H block kernel (call shape of STARSH_gen.jdf:70-72): out[nr x nc],
 * ld, of global rows r0.., cols c0.. from device points [ndim][N]. */
int hicma_tlr_k_cov(const hicma_tlr_problem *prob, const double *d_points, int N, int r0,
                    int nr, int c0, int nc, double *d_out, int ld, void *stream);

/* C = alpha op(A) op(B) + beta C on the FP64 tensor cores (CORE_dgemm). */
int hicma_tlr_k_dgemm(int transA, int transB, int m, int n, int k, double alpha,
                      const double *d_A, int lda, const double *d_B, int ldb, double beta,
                      double *d_C, int ldc, void *stream);

/* Lower Cholesky of an n x n tile in place (HCORE_dpotrf,
 * HiCMA_dpotrf_L_2flow.jdf:233); *d_info (device int) gets the 1-based
 * order of the first failing minor plus info_offset.  d_linv (n x n, may be
 * NULL) receives L^-1.  Uses ctx workspace. */
int hicma_tlr_k_potrf(hicma_tlr_ctx *ctx, int n, double *d_A, int lda, double *d_linv,
                      int *d_info, int info_offset);

/* Low-rank GEMM update with recompression of one tile
 * (HCORE_dgemm_qr_svd + HCORE_dgemm_ormqr, HiCMA_dpotrf_L_2flow.jdf:985-1058):
 * C = Cu Cv^T - Au (Bu (Bv^T Av))^T recompressed to absolute accuracy acc,
 * rank capped at maxrank.  If d_Bv is NULL, B is dense NB x NB in d_Bu
 * (HCORE_dgemm_qr_svd_b_dense, :830-903).  d_Cu/d_Cv have capacity maxrank
 * columns; *rc (host) is updated.  Returns 0 or an error code. */
int hicma_tlr_k_lr_update(hicma_tlr_ctx *ctx, int nb, const double *d_Au, const double *d_Av,
                          int ra, const double *d_Bu, const double *d_Bv, int rb, double *d_Cu,
                          double *d_Cv, int *rc, double acc, int maxrank, int fixed_rank);

/* Compress a dense nb x nb tile (starsh_dense_dlrrsdd, STARSH_gen.jdf:162-163):
 * randomized range finder with maxrank+10 samples, relative Frobenius
 * truncation at tol; *rank = -1 when rejected. */
int hicma_tlr_k_compress(hicma_tlr_ctx *ctx, int nb, const double *d_A, double *d_U, double *d_V,
                         int maxrank, double tol, int *rank);

/* Allocation-free variant of hicma_tlr_k_potrf.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc, such as code
 * embedded in a host framework that owns all device memory and only lends out
 * buffers, or latency-critical loops that must avoid the device-wide
 * synchronisation an allocation can trigger.  It factors the n x n tile d_A
 * (leading dimension lda) in place and, if d_linv is non-NULL, writes L^-1
 * there (n x n, leading dimension n); *d_info as for hicma_tlr_k_potrf.  No
 * context, no allocation, no freeing: its scratch is a fixed array inside the
 * library (2.1 MB of device memory on every GPU that loads the library, held
 * until the process exits), which limits n to 1..4096; larger n returns
 * HICMA_TLR_ERR_ARG with a message in hicma_tlr_last_error().  Every call
 * looks up the device address of that array for the current device and
 * context (a host-side lookup once the library's module is loaded); the first
 * call on a device loads the module, so make that first call before capturing
 * the stream into a CUDA graph.  A CUDA error already pending when the call
 * starts is reported (HICMA_TLR_ERR_CUDA) and left in place; a failed launch
 * stops the call at once.  The work is enqueued on `stream` (NULL = legacy
 * default stream) and the call returns without waiting.  All calls share the
 * one array: calls whose work overlaps on the GPU (other streams, other host
 * threads) race on it and must be ordered by the caller. */
int hicma_tlr_k_potrf_noalloc(int n, double *d_A, int lda, double *d_linv, int *d_info,
                              int info_offset, void *stream);

/* Bounds-checked builds (libhicma_tlr_checked.so, compiled with
 * TLR_BOUNDS_CHECK; no reference counterpart): before every batched launch
 * the host checks that each task's operand extents lie inside one live device
 * region and refuses the launch with HICMA_TLR_ERR_ARG otherwise.  Regions are
 * the library's own allocations, the context workspace, and caller buffers
 * passed to the kernel-level entries (registered for the length of the call).
 * _checked returns 1 in such a build, 0 otherwise; the other three manage and
 * query the region list directly (HICMA_TLR_ERR_NOT_SUPPORTED in a build
 * without the checks); _inside returns 1 when [p, p + bytes) lies in one
 * region. */
int hicma_tlr_bounds_checked(void);
int hicma_tlr_bounds_register(const void *p, size_t bytes);
int hicma_tlr_bounds_unregister(const void *p);
int hicma_tlr_bounds_inside(const void *p, size_t bytes);

/* Test of the bounded dependency wait of the tile POTRF task queue (no
 * reference counterpart): nblocks (1..64) CTAs each wait, with the queue's own
 * wait routine, on a counter that nothing sets; CTA 0 gives up after polls0
 * polls, the others after polls1 (1..2^26; a poll is about 0.25 us).  The
 * first wait to give up raises the abort flag, on which the others leave.
 * Returns HICMA_TLR_ERR_TIMEOUT (the status a factorization reports when a
 * wait gives up) with the kernel's duration in *elapsed_ms (may be NULL). */
int hicma_tlr_k_wait_probe(long long polls0, long long polls1, int nblocks, double *elapsed_ms, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* HICMA_TLR_H */
