// QR factorization of a tall-skinny matrix by randomized CholeskyQR, one CTA
// per matrix, FP64 (Gram products on the FP64 tensor cores).
//
// Replaces both QRs of HCORE_dgemm_qr_svd (call sites
// hicma_parsec/HiCMA_dpotrf_L_2flow.jdf:830-903,985-1058): the U side
// [Cu, Au] = Q_U R_U (Q_U kept as Y with Rc^-1, the new U being
// Y (Rc^-1 U_r), which replaces the Householder Q application of
// HCORE_dgemm_ormqr), and the V side [Cv, -Y] = Q_V R_V with R only (the new
// V is [Cv, -Y] R_U^T U_r).  The matrix is given as two column blocks read
// where they lie, so [Cu, Au] is never copied.  Also the range finder's QR
// of the randomized compression (Q formed).
//
// Algorithm (randomized preconditioned CholeskyQR: Fan, Guo and Lin, "A novel
// randomized XR-based preconditioned CholeskyQR algorithm", 2021; Balabanov,
// "Randomized Cholesky QR factorizations", 2022), for X with m rows and K
// columns:
//   1. sketch S = Omega X, 256 x K: row i of X, times a sign taken from a
//      32-bit hash of i, is added to row i mod 256 of S (a CountSketch); one
//      pass over the rows, S held in registers (one sketch row per thread);
//   2. Rs = R of S by shifted CholeskyQR3 (Fukaya, Kannan, Nakatsukasa,
//      Yamamoto and Yanagisawa, SIAM J. Sci. Comput. 42(1), 2020) on the
//      sketch rows, with D the column norms of S:
//        R1 = chol(D^-1 S^T S D^-1 + s I),  S1 = S D^-1 R1^-1,
//        R2 = chol(S1^T S1),  S2 = S1 R2^-1,  R3 = chol(S2^T S2),
//        Rs = R3 R2 R1 D,
//      s = 11 (256 K + K (K + 1)) u tr(G);
//   3. one pass over the rows: Y = X Rs^-1 (written out when Q is wanted),
//      G = Y^T Y, Rc = chol(G);  R = Rc Rs,  Q = Y Rc^-1.
// The sketch shrinks no vector of range(X) by more than a factor
// sqrt(ceil(m / 256)) (at most that many rows share a bucket), so the
// singular values of Y over range(X) are bounded below; a large ||G||_inf
// means the sketch missed a direction (Y has a large singular value), and step
// 3 repeats with R in place of Rs (a CholeskyQR step on Y), at most CQ_APPLY
// passes.  Directions where X itself is numerically null stay small in Y and
// need no repeat (the core SVD of R truncates them).  A pivot of a Cholesky
// factorization that is not positive (a column dependent on the ones before
// it, or zero) is set to the shift s with its column zeroed, instead of
// shifting the whole matrix, so the other columns keep their factor.  X R^-1
// is a row-wise substitution (the backward-stable triangular solve the error
// bounds assume).
//
// Layout: each thread owns the rows i = 256 c + tid.  A lane keeps its row in
// registers for the substitution (R read as broadcasts from shared memory),
// stages it into shared memory (column-major, pitch == 4 mod 16: conflict-free
// row stores and DMMA fragment loads), and the Gram product accumulates with
// mma.sync m8n8k4 f64.  Widths up to 48: each warp stages its own 32-row
// chunks and accumulates the whole lower triangle (one fragment load per
// 8-column block and row quad, reused by every tile of that block); the eight
// per-warp partials are added in warp order (deterministic).  Width 64: the
// CTA stages 256-row chunks and each warp accumulates the tiles it owns.  The
// K x K Cholesky factorizations run on the whole CTA.  Kernels are
// instantiated per width bucket (KM = 16, 32, 48, 64 columns); wider stacks
// take the Householder path.
#include "tlr_internal.h"

namespace tlr {
namespace {

constexpr int CQ_WARPS = 8;
constexpr int CQ_THREADS = CQ_WARPS * 32;
constexpr int CQ_PITCH = 36;            // per-warp staged chunk pitch (== 4 mod 16)
constexpr int CQ_CH = CQ_THREADS;       // rows of a CTA-staged chunk (one per thread); sketch rows
constexpr int CQ_LDZ = CQ_CH + 4;       // its pitch (== 4 mod 16)
constexpr int CQ_APPLY = 3;             // passes of step 3 at most
constexpr int CQ_SKB = 16;              // loads in flight per thread in the sketch pass
constexpr double CQ_GMAX = 1e4;         // ||Y^T Y||_inf above this: the sketch missed a direction
constexpr double CQ_U = 1.1102230246251565e-16;
// pivot floor when G is zero: factors of 1e-100 keep the product of the four
// factors (and its inverse) finite, and R of a zero X comes out zero
constexpr double CQ_TINY = 1e-200;

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// Sign of row i in the sketch: the low bit of a 32-bit integer hash of i
// (xor-shift / multiply rounds of the "lowbias32" mixer).
__device__ __forceinline__ double row_sign(unsigned i) {
    i ^= i >> 16;
    i *= 0x7feb352du;
    i ^= i >> 15;
    i *= 0x846ca68bu;
    i ^= i >> 16;
    return (i & 1u) ? -1.0 : 1.0;
}

// Widths up to 48: every warp stages and reduces its own 32-row chunks.
// Width 64 (CTA-staged): the row and the accumulators of all 36 tiles would
// not fit a thread's registers, so the CTA stages 256-row chunks and each
// warp accumulates the tiles it owns (no reduction); G then lives in the chunk
// buffer between passes.
template <int KM>
struct CQSmem {
    static constexpr bool STAGED = KM > 48;
    static constexpr int NT8 = KM / 8;
    static constexpr int NTILE = NT8 * (NT8 + 1) / 2;
    static constexpr int TPW = (NTILE + CQ_WARPS - 1) / CQ_WARPS;   // owned tiles per warp (staged)
    static constexpr int NACC = STAGED ? 2 * TPW : NTILE;           // accumulators per lane
    static constexpr size_t W = (size_t)KM * CQ_PITCH;    // one warp's staged chunk
    static constexpr size_t KK = (size_t)KM * KM;
    static constexpr size_t CHUNK = STAGED ? (size_t)KM * CQ_LDZ : CQ_WARPS * W;
    // chunk buffer(s) | [G, unless in the chunk buffer] | Rr | Rt | 1/diag Rr | 1/diag Rt | d
    static constexpr size_t bytes() { return sizeof(double) * (CHUNK + (STAGED ? 2 : 3) * KK + 3 * KM); }
    static_assert(!STAGED || CHUNK >= KK, "G lives in the chunk buffer");
};

// x <- x R^-1 for one row x (registers): right-looking substitution with the
// row-major upper R in shared memory.  Written as compile-time recursion so
// that every index into x is static and x stays in registers at any width.
template <int KM, int J, int C>
__device__ __forceinline__ void subst_cols(double (&x)[KM], double xj, const double *rj) {
    if constexpr (C < KM) {
        x[C] -= xj * rj[C];
        subst_cols<KM, J, C + 1>(x, xj, rj);
    }
}
template <int KM, int J>
__device__ __forceinline__ void subst_rows(double (&x)[KM], const double *Rr, const double *rdg) {
    if constexpr (J < KM) {
        x[J] *= rdg[J];
        subst_cols<KM, J, J + 1>(x, x[J], Rr + J * KM);
        subst_rows<KM, J + 1>(x, Rr, rdg);
    }
}

// Gram product of one chunk of rows (x: this thread's row, zero past K and
// for rows past the end) added to the lane's accumulators.
template <int KM>
__device__ __forceinline__ void gram_chunk(const double (&x)[KM], double (&acc)[CQSmem<KM>::NACC][2], double *sm,
                                           int tid, const int (&tmi)[CQSmem<KM>::TPW],
                                           const int (&tni)[CQSmem<KM>::TPW]) {
    using S = CQSmem<KM>;
    const int lane = tid & 31, g = lane >> 2, tig = lane & 3;
    if constexpr (S::STAGED) {
#pragma unroll
        for (int j = 0; j < KM; ++j) sm[j * CQ_LDZ + tid] = x[j];
        __syncthreads();
        // owned tiles over the 256 rows, two chains per tile (even / odd row quads)
#pragma unroll 2
        for (int s = 0; s < CQ_CH; s += 8) {
#pragma unroll
            for (int q = 0; q < S::TPW; ++q) {
                if (tmi[q] < 0) continue;
                const double *za = sm + (8 * tmi[q] + g) * CQ_LDZ + tig + s;
                const double *zb = sm + (8 * tni[q] + g) * CQ_LDZ + tig + s;
                dmma884(acc[2 * q], za[0], zb[0]);
                dmma884(acc[2 * q + 1], za[4], zb[4]);
            }
        }
        __syncthreads();
    } else {
        double *Zw = sm + (tid >> 5) * S::W;
#pragma unroll
        for (int j = 0; j < KM; ++j) Zw[j * CQ_PITCH + lane] = x[j];
        __syncwarp();
        // row quads s, one fragment per 8-column block
#pragma unroll 1
        for (int s = 0; s < 32; s += 4) {
            double a[S::NT8];
#pragma unroll
            for (int mi = 0; mi < S::NT8; ++mi) a[mi] = Zw[(8 * mi + g) * CQ_PITCH + s + tig];
            int q = 0;
#pragma unroll
            for (int mi = 0; mi < S::NT8; ++mi)
#pragma unroll
                for (int ni = 0; ni <= mi; ++ni, ++q) dmma884(acc[q], a[mi], a[ni]);
        }
        __syncwarp();
    }
}

// Accumulators -> G (column-major, ld KM, both triangles of [0, K)), visible
// to the CTA on return.
template <int KM>
__device__ __forceinline__ void gram_reduce(const double (&acc)[CQSmem<KM>::NACC][2], double *G, int tid,
                                            const int (&tmi)[CQSmem<KM>::TPW], const int (&tni)[CQSmem<KM>::TPW]) {
    using S = CQSmem<KM>;
    const int lane = tid & 31, warp = tid >> 5, g = lane >> 2, tig = lane & 3;
    if constexpr (S::STAGED) {
        // owned tiles (the chunk buffer is free after the last barrier); tiles
        // past K are not computed and stay out of everything that reads G
#pragma unroll
        for (int q = 0; q < S::TPW; ++q) {
            if (tmi[q] < 0) continue;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int i = 8 * tmi[q] + g, j = 8 * tni[q] + 2 * tig + e;
                const double v = acc[2 * q][e] + acc[2 * q + 1][e];
                G[i + j * KM] = v;
                G[j + i * KM] = v;
            }
        }
        __syncthreads();
    } else {
        // per-warp partials, added in warp order
        for (int idx = tid; idx < KM * KM; idx += CQ_THREADS) G[idx] = 0.0;
        __syncthreads();
        for (int w = 0; w < CQ_WARPS; ++w) {
            if (warp == w) {
                int q = 0;
#pragma unroll
                for (int mi = 0; mi < S::NT8; ++mi)
#pragma unroll
                    for (int ni = 0; ni <= mi; ++ni, ++q)
#pragma unroll
                        for (int e = 0; e < 2; ++e) {
                            const int i = 8 * mi + g, j = 8 * ni + 2 * tig + e;
                            G[i + j * KM] += acc[q][e];
                            if (mi != ni) G[j + i * KM] += acc[q][e];
                        }
            }
            __syncthreads();
        }
    }
}

// In-place elimination of the K x K symmetric positive semidefinite matrix G
// (column-major, ld KM, lower part) by the whole CTA: right-looking, one
// barrier per column, the trailing update with the unscaled pivot column,
// G(i,k) -= G(i,j) G(k,j) / G(j,j).  On return G(j,j) is the j-th pivot and
// G(i,j) = L(i,j) sqrt(G(j,j)), i > j.  A pivot that is not positive (column
// j depends on the columns before it, or is zero, up to rounding) is set to
// `floor` with its column below the diagonal zeroed and no trailing update:
// a perturbation of G confined to row and column j (whose Schur complement
// entries are at rounding level), which leaves the factor of every other
// column as it was.  Threads form a 16 x 16 grid: rows i by tx (consecutive
// addresses), columns k by ty.  Returns the number of such null pivots.
template <int KM>
__device__ int cta_cholesky(double *G, int K, double floor, int tid) {
    const int tx = tid & 15, ty = tid >> 4;
    int nnull = 0;
    for (int j = 0; j < K; ++j) {
        const double d = G[j + j * KM];
        if (!(d > 0.0)) {
            ++nnull;
            __syncthreads();   // every thread has read the pivot
            if (tid == 0) G[j + j * KM] = floor;
            for (int i = j + 1 + tid; i < K; i += CQ_THREADS) G[i + j * KM] = 0.0;
            __syncthreads();
            continue;
        }
        const double id = 1.0 / d;
        for (int k = j + 1 + ty; k < K; k += 16) {
            const double gkj = G[k + j * KM] * id;
            for (int i = k + ((j + 1 + tx - k) & 15); i < K; i += 16) G[i + k * KM] -= G[i + j * KM] * gkj;
        }
        __syncthreads();
    }
    return nnull;
}

// R = chol(G + shift)^T into Rr (upper, row-major, zero outside [0, K)) and
// rdg = 1/diag(Rr), with s = 11 (m K + K (K + 1)) u tr(G): the shift when
// `shifted` (none otherwise) and the floor of null pivots (CQ_TINY when
// s = 0).  G must be complete and visible; it is free on return.  Returns the
// number of null pivots.
template <int KM>
__device__ int factor(double *G, double *Rr, double *rdg, int K, double m, bool shifted, int tid) {
    double tr = 0.0;
    for (int j = 0; j < K; ++j) tr += G[j + j * KM];
    const double s0 = 11.0 * (m * K + (double)K * (K + 1)) * CQ_U * tr;
    if (shifted && s0 > 0.0) {
        __syncthreads();   // every thread has read the diagonal
        for (int j = tid; j < K; j += CQ_THREADS) G[j + j * KM] += s0;
        __syncthreads();
    }
    const int nnull = cta_cholesky<KM>(G, K, s0 > 0.0 ? s0 : CQ_TINY, tid);
    for (int idx = tid; idx < KM * KM; idx += CQ_THREADS) {
        const int j = idx / KM, k = idx % KM;
        double v = 0.0;
        if (j <= k && k < K) {
            const double p = sqrt(G[j + j * KM]);
            v = j == k ? p : G[k + j * KM] / p;
        }
        Rr[j * KM + k] = v;
    }
    __syncthreads();
    for (int j = tid; j < KM; j += CQ_THREADS) rdg[j] = j < K ? 1.0 / Rr[j * KM + j] : 0.0;
    __syncthreads();
    return nnull;
}

// Rt <- Rr Rt (upper times upper, both row-major; consecutive threads take
// consecutive columns: Rr read as a broadcast, Rt conflict-free) through the
// scratch P, and rdt = 1/diag(Rt).  Entries outside [0, K) stay zero.
template <int KM>
__device__ void accumulate(const double *Rr, double *Rt, double *P, double *rdt, int K, int tid) {
    for (int idx = tid; idx < K * K; idx += CQ_THREADS) {
        const int i = idx / K, j = idx % K;
        double s = 0.0;
        for (int k = i; k <= j; ++k) s += Rr[i * KM + k] * Rt[k * KM + j];
        P[i * KM + j] = i <= j ? s : 0.0;
    }
    __syncthreads();
    for (int idx = tid; idx < K * K; idx += CQ_THREADS) {
        const int i = idx / K, j = idx % K;
        Rt[i * KM + j] = P[i * KM + j];
    }
    for (int j = tid; j < KM; j += CQ_THREADS) rdt[j] = j < K ? 1.0 / P[j * KM + j] : 0.0;
    __syncthreads();
}

// P = R^-1 (R upper, row-major Rr with rdg = 1/diag), row-major: thread c
// solves R p = e_c by back substitution (R read as broadcasts, P
// conflict-free), four partial sums in flight.
template <int KM>
__device__ void tri_inverse(const double *Rr, const double *rdg, double *P, int K, int tid) {
    const int c = tid;
    if (c < K) {
        for (int i = K - 1; i >= 0; --i) {
            double v = 0.0;
            if (i == c) {
                v = rdg[i];
            } else if (i < c) {
                double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
                int l = i + 1;
                for (; l + 3 <= c; l += 4) {
                    a0 += Rr[i * KM + l] * P[l * KM + c];
                    a1 += Rr[i * KM + l + 1] * P[(l + 1) * KM + c];
                    a2 += Rr[i * KM + l + 2] * P[(l + 2) * KM + c];
                    a3 += Rr[i * KM + l + 3] * P[(l + 3) * KM + c];
                }
                for (; l <= c; ++l) a0 += Rr[i * KM + l] * P[l * KM + c];
                v = -((a0 + a1) + (a2 + a3)) * rdg[i];
            }
            P[i * KM + c] = v;
        }
    }
    __syncthreads();
}

// QF: the tasks form Q (the range finder); instances without it carry no Q
// pass, which keeps the recompression's register allocation free of it.
template <int KM, bool QF>
__global__ void __launch_bounds__(CQ_THREADS, KM <= 32 ? 2 : 1) k_rcholqr(const CQTask *__restrict__ tasks,
                                                                         int *flags) {
    using S = CQSmem<KM>;
    constexpr bool STAGED = S::STAGED;
    constexpr int NACC = S::NACC;
    extern __shared__ double sm[];
    __shared__ double gmax_sh;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double *G = STAGED ? sm : sm + S::CHUNK;       // K x K Gram (column-major, ld KM)
    double *Rr = STAGED ? sm + S::CHUNK : G + S::KK;    // factor of the step, row-major: Rr[j * KM + k] = R(j, k)
    double *Rt = Rr + S::KK;                       // accumulated R, row-major
    double *rdg = Rt + S::KK;                      // 1 / diag(Rr)
    double *rdt = rdg + KM;                        // 1 / diag(Rt)
    double *dsc = rdt + KM;                        // column norms of the sketch, then their inverses

    const CQTask t = tasks[blockIdx.x];
    const int k1 = t.k1, K = t.k1 + t.k2, nb = t.nb;
    if (K <= 0) return;

    // tiles owned by this warp in the CTA-staged form
    int tmi[S::TPW], tni[S::TPW];
#pragma unroll
    for (int q = 0; q < S::TPW; ++q) {
        const int tile = warp + CQ_WARPS * q;
        int mi = 0;
        while ((mi + 1) * (mi + 2) / 2 <= tile) ++mi;
        tmi[q] = (tile < S::NTILE && 8 * mi < K) ? mi : -1;
        tni[q] = tile - mi * (mi + 1) / 2;
    }
    double acc[NACC][2];

    // 1. the sketch: this thread's bucket is tid
    {
        double s[KM];
#pragma unroll
        for (int j = 0; j < KM; ++j) s[j] = 0.0;
#pragma unroll 1
        for (int row = tid; row < nb; row += CQ_THREADS) {
            const double sg = row_sign((unsigned)row);
            const double *p1 = t.X1 + row, *p2 = t.X2 + row;
            // the row in batches of CQ_SKB loads issued back to back (the sketch
            // row holds KM registers; a load consumed as it is issued would
            // leave one load in flight per thread)
#pragma unroll
            for (int j0 = 0; j0 < KM; j0 += CQ_SKB) {
                double v[CQ_SKB];
#pragma unroll
                for (int jj = 0; jj < CQ_SKB; ++jj) {
                    const int j = j0 + jj;
                    v[jj] = 0.0;
                    if (j < k1) {
                        v[jj] = *p1;
                        p1 += t.ld1;
                    } else if (j < K) {
                        v[jj] = *p2;
                        p2 += t.ld2;
                    }
                }
#pragma unroll
                for (int jj = 0; jj < CQ_SKB; ++jj) s[j0 + jj] += sg * v[jj];
            }
        }

        // 2. shifted CholeskyQR3 of the sketch rows
        for (int round = 0; round < 3; ++round) {
            if (round == 1) {
#pragma unroll
                for (int j = 0; j < KM; ++j) s[j] *= dsc[j];
            }
            if (round > 0) subst_rows<KM, 0>(s, Rr, rdg);
#pragma unroll
            for (int q = 0; q < NACC; ++q) acc[q][0] = acc[q][1] = 0.0;
            gram_chunk<KM>(s, acc, sm, tid, tmi, tni);
            gram_reduce<KM>(acc, G, tid, tmi, tni);
            if (round == 0) {
                for (int j = tid; j < KM; j += CQ_THREADS) {
                    const double d = j < K ? sqrt(G[j + j * KM]) : 1.0;
                    dsc[j] = d > 0.0 ? d : 1.0;
                }
                __syncthreads();
                for (int idx = tid; idx < K * K; idx += CQ_THREADS) {
                    const int i = idx % K, j = idx / K;
                    G[i + j * KM] /= dsc[i] * dsc[j];
                }
                __syncthreads();
            }
            factor<KM>(G, Rr, rdg, K, (double)CQ_CH, round == 0, tid);
            if (round == 0) {
                // Rt = R1 D, then the substitution of round 1 scales by 1/d first
                for (int idx = tid; idx < KM * KM; idx += CQ_THREADS) Rt[idx] = Rr[idx] * dsc[idx % KM];
                __syncthreads();
                for (int j = tid; j < KM; j += CQ_THREADS) {
                    rdt[j] = j < K ? 1.0 / Rt[j * KM + j] : 0.0;
                    dsc[j] = 1.0 / dsc[j];
                }
                __syncthreads();
            } else {
                accumulate<KM>(Rr, Rt, G, rdt, K, tid);
            }
        }
    }

    // 3. Y = X R^-1 and its Gram product; R <- chol(Y^T Y) R
    const bool keep_y = QF || t.Rinv;
    for (int pass = 0;; ++pass) {
#pragma unroll
        for (int q = 0; q < NACC; ++q) acc[q][0] = acc[q][1] = 0.0;
#pragma unroll 1
        for (int r0 = STAGED ? 0 : warp * 32; r0 < nb; r0 += CQ_THREADS) {
            const int row = r0 + (STAGED ? tid : lane);
            const bool valid = row < nb;
            double x[KM];
            {
                // two column blocks, walked with one running pointer each
                const double *p1 = t.X1 + row, *p2 = t.X2 + row;
#pragma unroll
                for (int j = 0; j < KM; ++j) {
                    double v = 0.0;
                    if (j < k1) {
                        if (valid) v = *p1;
                        p1 += t.ld1;
                    } else if (j < K) {
                        if (valid) v = *p2;
                        p2 += t.ld2;
                    }
                    x[j] = v;
                }
            }
            // rdt and Rt are zero past K, so the padding columns stay zero
            subst_rows<KM, 0>(x, Rt, rdt);
            if (valid && keep_y) {
                double *pz = t.Z + row;
#pragma unroll
                for (int j = 0; j < KM; ++j, pz += nb)
                    if (j < K) *pz = x[j];
            }
            gram_chunk<KM>(x, acc, sm, tid, tmi, tni);
        }
        gram_reduce<KM>(acc, G, tid, tmi, tni);
        if (warp == 0) {
            // ||G||_inf (rows of the symmetric G), max over lanes
            double mx = 0.0;
            for (int i = lane; i < K; i += 32) {
                double r = 0.0;
                for (int j = 0; j < K; ++j) r += fabs(G[i + j * KM]);
                mx = fmax(mx, r);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if (lane == 0) gmax_sh = mx;
        }
        const int nnull = factor<KM>(G, Rr, rdg, K, (double)nb, false, tid);   // barriers: gmax_sh visible
        if (nnull && tid == 0 && flags) atomicAdd(flags, nnull);
        const bool again = !(gmax_sh <= CQ_GMAX) && pass + 1 < CQ_APPLY;
        accumulate<KM>(Rr, Rt, G, rdt, K, tid);
        if (!again) break;
        if (tid == 0 && flags) atomicAdd(flags + 1, 1);
    }

    // outputs: R (column-major); Rc^-1 for a deferred Q; or Q = Y Rc^-1
    for (int idx = tid; idx < K * K; idx += CQ_THREADS) {
        const int i = idx % K, j = idx / K;
        t.R[i + (size_t)j * K] = Rt[i * KM + j];
    }
    if (!QF && t.Rinv) {
        tri_inverse<KM>(Rr, rdg, G, K, tid);
        for (int idx = tid; idx < K * K; idx += CQ_THREADS) {
            const int i = idx % K, c = idx / K;
            t.Rinv[i + (size_t)c * K] = i <= c ? G[i * KM + c] : 0.0;
        }
    }
    if constexpr (QF) {
#pragma unroll 1
        for (int row = tid; row < nb; row += CQ_THREADS) {
            double x[KM];
            const double *pz = t.Z + row;
#pragma unroll
            for (int j = 0; j < KM; ++j, pz += nb) x[j] = j < K ? *pz : 0.0;
            subst_rows<KM, 0>(x, Rr, rdg);
            double *pq = t.Q + row;
#pragma unroll
            for (int j = 0; j < KM; ++j, pq += nb)
                if (j < K) *pq = x[j];
        }
    }
}

template <int KM, bool QF>
void launch_cq(const CQTask *d_tasks, int ntasks, int *flags, cudaStream_t st) {
    const size_t smem = CQSmem<KM>::bytes();
    // per device and thread-safe: set on every launch (a host-side call, no synchronisation)
    cudaFuncSetAttribute(k_rcholqr<KM, QF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_rcholqr<KM, QF><<<ntasks, CQ_THREADS, smem, st>>>(d_tasks, flags);
}

template <bool QF>
void launch_bucket(const CQTask *d_tasks, int ntasks, int kmax, int *flags, cudaStream_t st) {
    switch (rcholqr_bucket(kmax)) {
        case 16: launch_cq<16, QF>(d_tasks, ntasks, flags, st); break;
        case 32: launch_cq<32, QF>(d_tasks, ntasks, flags, st); break;
        case 48: launch_cq<48, QF>(d_tasks, ntasks, flags, st); break;
        default: launch_cq<64, QF>(d_tasks, ntasks, flags, st); break;
    }
}

}  // namespace

int rcholqr_kmax() { return 64; }

int rcholqr_bucket(int K) { return K <= 16 ? 16 : K <= 32 ? 32 : K <= 48 ? 48 : 64; }

void launch_rcholqr_batched(const CQTask *d_tasks, int ntasks, int kmax, bool form_q, int *flags,
                            cudaStream_t st) {
    if (ntasks <= 0) return;
    if (form_q)
        launch_bucket<true>(d_tasks, ntasks, kmax, flags, st);
    else
        launch_bucket<false>(d_tasks, ntasks, kmax, flags, st);
}

}  // namespace tlr
