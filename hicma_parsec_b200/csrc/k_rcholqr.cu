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
    static constexpr int RLD = KM + 4;                     // row pitch of the K x K factors (== 4 mod 16)
    static constexpr size_t RR = (size_t)KM * RLD;
    static constexpr size_t CHUNK = STAGED ? (size_t)KM * CQ_LDZ : CQ_WARPS * W;
    static constexpr size_t WS = CQ_WARPS * 96;           // per-warp 8 x 8 scratch (pitch 12), end of the chunk buffer
    // chunk buffer(s) | [G / product scratch, unless in the chunk buffer] | Rr | Rt |
    // 1/diag Rr | 1/diag Rt | d | 1/pivots
    static constexpr size_t bytes() { return sizeof(double) * (CHUNK + (STAGED ? 2 : 3) * RR + 4 * KM); }
    static_assert(CHUNK >= WS && (!STAGED || CHUNK >= RR + WS), "scratch regions fit the chunk buffer");
    static_assert(RR >= KK, "G fits its region");
    static_assert(STAGED || W >= (size_t)NTILE * 64, "per-warp Gram partials fit the warp's chunk slice");
};

// x <- x R^-1 for one row x (registers): right-looking substitution with the
// row-major upper R (pitch RLD) in shared memory, read as broadcasts, two
// entries per 128-bit load (rows start 16-byte aligned: RLD is even).  Written
// as compile-time recursion so that every index into x is static and x stays
// in registers at any width.
template <int KM, int C>
__device__ __forceinline__ void subst_cols(double (&x)[KM], double xj, const double *rj) {
    if constexpr (C < KM) {
        if constexpr ((C & 1) == 0 && C + 1 < KM) {
            const double2 r = *reinterpret_cast<const double2 *>(rj + C);
            x[C] -= xj * r.x;
            x[C + 1] -= xj * r.y;
            subst_cols<KM, C + 2>(x, xj, rj);
        } else {
            x[C] -= xj * rj[C];
            subst_cols<KM, C + 1>(x, xj, rj);
        }
    }
}
template <int KM, int J>
__device__ __forceinline__ void subst_rows(double (&x)[KM], const double *R, const double *rd) {
    if constexpr (J < KM) {
        x[J] *= rd[J];
        subst_cols<KM, J + 1>(x, x[J], R + J * CQSmem<KM>::RLD);
        subst_rows<KM, J + 1>(x, R, rd);
    }
}

// Gram product of a staged 256-row chunk (CTA-staged form, after a barrier):
// each warp's owned tiles, two chains per tile (even / odd row quads).
template <int KM>
__device__ __forceinline__ void gram_tiles(double (&acc)[CQSmem<KM>::NACC][2], const double *sm, int lane,
                                           const int (&tmi)[CQSmem<KM>::TPW], const int (&tni)[CQSmem<KM>::TPW]) {
    using S = CQSmem<KM>;
    const int g = lane >> 2, tig = lane & 3;
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
}

// Gram product of a warp's staged 32-row chunk (per-warp form): row quads s,
// one fragment per 8-column block, reused by every tile of that block.
template <int KM>
__device__ __forceinline__ void gram_warp(double (&acc)[CQSmem<KM>::NACC][2], const double *Zw, int lane) {
    using S = CQSmem<KM>;
    const int g = lane >> 2, tig = lane & 3;
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
}

// Gram product of one chunk of rows held in registers (x: this thread's row,
// zero past K and for rows past the end), staged first.
template <int KM>
__device__ __forceinline__ void gram_chunk(const double (&x)[KM], double (&acc)[CQSmem<KM>::NACC][2], double *sm,
                                           int tid, const int (&tmi)[CQSmem<KM>::TPW],
                                           const int (&tni)[CQSmem<KM>::TPW]) {
    using S = CQSmem<KM>;
    const int lane = tid & 31;
    if constexpr (S::STAGED) {
#pragma unroll
        for (int j = 0; j < KM; ++j) sm[j * CQ_LDZ + tid] = x[j];
        __syncthreads();
        gram_tiles<KM>(acc, sm, lane, tmi, tni);
        __syncthreads();
    } else {
        double *Zw = sm + (tid >> 5) * S::W;
#pragma unroll
        for (int j = 0; j < KM; ++j) Zw[j * CQ_PITCH + lane] = x[j];
        __syncwarp();
        gram_warp<KM>(acc, Zw, lane);
        __syncwarp();
    }
}

// Row `row` of X = [X1, X2] into v (zero past K and for rows past the end):
// every load issued before any use.
template <int KM>
__device__ __forceinline__ void load_row(const CQTask &t, int row, int nb, int k1, int K, double (&v)[KM]) {
    const bool valid = row < nb;
    const double *p1 = t.X1 + row, *p2 = t.X2 + row;
#pragma unroll
    for (int j = 0; j < KM; ++j) {
        double x = 0.0;
        if (j < k1) {
            if (valid) x = *p1;
            p1 += t.ld1;
        } else if (j < K) {
            if (valid) x = *p2;
            p2 += t.ld2;
        }
        v[j] = x;
    }
}

// Y = X R^-1 in place for a warp's 32 staged rows (column-major, pitch P):
// 8-column blocks J = 0, 1, ...: C = sum_{I<J} Y_I R_IJ on DMMA (four 8-row
// tiles, the block of R shared), Z_J -= C, then each lane solves its row's
// 8 x 8 diagonal block by substitution (R broadcast from shared memory).  R is
// the row-major upper factor (pitch RLD) with rd = 1/diag, zero past K.
template <int KM, int P>
__device__ __forceinline__ void warp_trsm(double *zb, const double *R, const double *rd, int K, int lane) {
    constexpr int L = CQSmem<KM>::RLD;
    const int g = lane >> 2, tig = lane & 3;
    const int NK = (K + 7) >> 3;
    for (int J = 0; J < NK; ++J) {
        if (J > 0) {
            double acc[4][2];
#pragma unroll
            for (int mt = 0; mt < 4; ++mt) acc[mt][0] = acc[mt][1] = 0.0;
            for (int I = 0; I < J; ++I) {
#pragma unroll
                for (int k4 = 0; k4 < 8; k4 += 4) {
                    const double b = R[(8 * I + k4 + tig) * L + 8 * J + g];
                    const double *za = zb + (8 * I + k4 + tig) * P + g;
#pragma unroll
                    for (int mt = 0; mt < 4; ++mt) dmma884(acc[mt], za[8 * mt], b);
                }
            }
#pragma unroll
            for (int mt = 0; mt < 4; ++mt)
#pragma unroll
                for (int e = 0; e < 2; ++e) zb[(8 * J + 2 * tig + e) * P + 8 * mt + g] -= acc[mt][e];
            __syncwarp();
        }
        double z[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) z[c] = zb[(8 * J + c) * P + lane];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            z[c] *= rd[8 * J + c];
#pragma unroll
            for (int c2 = c + 1; c2 < 8; ++c2) z[c2] -= z[c] * R[(8 * J + c) * L + 8 * J + c2];
        }
#pragma unroll
        for (int c = 0; c < 8; ++c) zb[(8 * J + c) * P + lane] = z[c];
        __syncwarp();
    }
}

// Accumulators -> G (column-major, ld KM, both triangles of [0, K)), visible
// to the CTA on return.
template <int KM>
__device__ __forceinline__ void gram_reduce(const double (&acc)[CQSmem<KM>::NACC][2], double *G, double *sm, int tid,
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
        // per-warp partials into the warp's own chunk slice (free after its Gram),
        // then every entry summed over the eight slices in warp order
        double *Pw = sm + warp * S::W;
        {
            int q = 0;
#pragma unroll
            for (int mi = 0; mi < S::NT8; ++mi)
#pragma unroll
                for (int ni = 0; ni <= mi; ++ni, ++q)
#pragma unroll
                    for (int e = 0; e < 2; ++e) Pw[q * 64 + g * 8 + 2 * tig + e] = acc[q][e];
        }
        __syncthreads();
        for (int idx = tid; idx < S::NTILE * 64; idx += CQ_THREADS) {
            const int q = idx >> 6, r = idx & 63;
            int mi = 0;
            while ((mi + 1) * (mi + 2) / 2 <= q) ++mi;
            const int ni = q - mi * (mi + 1) / 2;
            double v = 0.0;
#pragma unroll
            for (int w = 0; w < CQ_WARPS; ++w) v += sm[w * S::W + idx];
            const int i = 8 * mi + (r >> 3), j = 8 * ni + (r & 7);
            G[i + j * KM] = v;
            G[j + i * KM] = v;
        }
        __syncthreads();
    }
}

// In-place elimination of the K x K symmetric positive semidefinite matrix G
// (column-major, ld KM, lower part), padded to Kp = 8 ceil(K / 8) with an
// identity block: right-looking in 8-column panels.  Warp 0 eliminates a
// panel (lanes own rows, two each; the pivot row's entries by shuffles), then
// the CTA applies the panel's rank-8 update to the trailing lower triangle,
// G(i,k) -= sum_c G(i,c) G(k,c) / G(c,c) (threads on a 16 x 16 grid of rows
// and columns, the row's panel entries in registers).  On return G(j,j) is the
// j-th pivot and G(i,j) = L(i,j) sqrt(G(j,j)), i > j.  A pivot that is not
// positive (column j depends on the columns before it, or is zero, up to
// rounding) is set to `floor` with its column below the diagonal zeroed and
// no update from it: a perturbation of G confined to row and column j (whose
// Schur complement entries are at rounding level), which leaves the factor of
// every other column as it was.  iv receives the inverse pivots.  Returns the
// number of such null pivots on thread 0.
template <int KM>
__device__ int cta_cholesky(double *G, int K, double floor, double *iv, int tid) {
    const int lane = tid & 31, warp = tid >> 5;
    const int Kp = (K + 7) & ~7;
    if (Kp > K) {
        for (int idx = tid; idx < (Kp - K) * Kp; idx += CQ_THREADS) {
            const int i = K + idx % (Kp - K), j = idx / (Kp - K);
            G[i + j * KM] = i == j ? 1.0 : 0.0;
        }
        __syncthreads();
    }
    int nnull = 0;
    for (int j0 = 0; j0 < Kp; j0 += 8) {
        if (warp == 0) {
            const int ra = j0 + lane, rb = j0 + 32 + lane;
            double a[8], b[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                a[c] = ra < Kp ? G[ra + (j0 + c) * KM] : 0.0;
                b[c] = rb < Kp ? G[rb + (j0 + c) * KM] : 0.0;
            }
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const double d = __shfl_sync(0xffffffffu, a[c], c);
                if (!(d > 0.0)) {
                    if (lane > c) a[c] = 0.0;
                    if (lane == c) a[c] = floor;
                    b[c] = 0.0;
                    ++nnull;
                    continue;
                }
                const double id = 1.0 / d;
#pragma unroll
                for (int c2 = c + 1; c2 < 8; ++c2) {
                    const double lc = __shfl_sync(0xffffffffu, a[c], c2) * id;
                    if (lane > c) a[c2] -= a[c] * lc;
                    b[c2] -= b[c] * lc;
                }
            }
            double piv = 1.0;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                if (ra < Kp && lane >= c) G[ra + (j0 + c) * KM] = a[c];
                if (rb < Kp) G[rb + (j0 + c) * KM] = b[c];
                if (lane == c) piv = a[c];
            }
            if (lane < 8) iv[j0 + lane] = 1.0 / piv;
        }
        __syncthreads();
        const int t0 = j0 + 8;
        if (t0 < Kp) {
            const int tx = tid & 15, ty = tid >> 4;
            double ivc[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) ivc[c] = iv[j0 + c];
            for (int i = t0 + tx; i < Kp; i += 16) {
                double pi[8];
#pragma unroll
                for (int c = 0; c < 8; ++c) pi[c] = G[i + (j0 + c) * KM] * ivc[c];
                for (int k = t0 + ty; k <= i; k += 16) {
                    double v = G[i + k * KM];
#pragma unroll
                    for (int c = 0; c < 8; ++c) v -= pi[c] * G[k + (j0 + c) * KM];
                    G[i + k * KM] = v;
                }
            }
            __syncthreads();
        }
    }
    return nnull;
}

// R = chol(G + shift)^T into Rr (upper, row-major, pitch RLD, zero outside
// [0, K)) and rdg = 1/diag(Rr), with s = 11 (m K + K (K + 1)) u tr(G): the
// shift when `shifted` (none otherwise) and the floor of null pivots (CQ_TINY
// when s = 0).  G must be complete and visible; it is free on return.
// Returns the number of null pivots (on thread 0).
template <int KM>
__device__ int factor(double *G, double *Rr, double *rdg, double *iv, int K, double m, bool shifted, int tid) {
    constexpr int L = CQSmem<KM>::RLD;
    const int lane = tid & 31;
    // trace: every warp reduces the diagonal the same way (same value everywhere)
    double tr = 0.0;
    for (int j = lane; j < K; j += 32) tr += G[j + j * KM];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tr += __shfl_xor_sync(0xffffffffu, tr, o);
    const double s0 = 11.0 * (m * K + (double)K * (K + 1)) * CQ_U * tr;
    __syncthreads();   // every thread has read the diagonal
    if (shifted && s0 > 0.0) {
        for (int j = tid; j < K; j += CQ_THREADS) G[j + j * KM] += s0;
        __syncthreads();
    }
    const int nnull = cta_cholesky<KM>(G, K, s0 > 0.0 ? s0 : CQ_TINY, iv, tid);
    for (int j = tid; j < KM; j += CQ_THREADS) {
        const double p = j < K ? sqrt(G[j + j * KM]) : 0.0;
        rdg[j] = j < K ? 1.0 / p : 0.0;
        Rr[j * L + j] = p;
    }
    __syncthreads();
    for (int idx = tid; idx < KM * KM; idx += CQ_THREADS) {
        const int j = idx / KM, k = idx % KM;
        if (j != k) Rr[j * L + k] = (j < k && k < K) ? G[k + j * KM] * rdg[j] : 0.0;
    }
    __syncthreads();
    return nnull;
}

// Rt <- Rr Rt (upper times upper, row-major, pitch RLD) on DMMA: warp w takes
// the upper 8 x 8 output tiles q = w, w + 8, ... (NK = ceil(K / 8) tiles a
// side), each the sum over M = I..J of Rr_IM Rt_MJ (the blocks of the two
// factors are triangular with exact zeros below the diagonal, and zero past
// K), into the scratch P, copied back after a barrier; rdt = 1/diag(Rt).
template <int KM>
__device__ void accumulate(const double *Rr, double *Rt, double *P, double *rdt, int K, int tid) {
    constexpr int L = CQSmem<KM>::RLD;
    const int lane = tid & 31, warp = tid >> 5, g = lane >> 2, tig = lane & 3;
    const int NK = (K + 7) >> 3, NQ = NK * (NK + 1) / 2;
    for (int q = warp; q < NQ; q += CQ_WARPS) {
        int I = 0, rem = q;
        while (rem >= NK - I) {
            rem -= NK - I;
            ++I;
        }
        const int J = I + rem;
        double acc[2] = {0.0, 0.0};
        for (int M = I; M <= J; ++M) {
#pragma unroll
            for (int k4 = 0; k4 < 8; k4 += 4)
                dmma884(acc, Rr[(8 * I + g) * L + 8 * M + k4 + tig], Rt[(8 * M + k4 + tig) * L + 8 * J + g]);
        }
        P[(8 * I + g) * L + 8 * J + 2 * tig] = acc[0];
        P[(8 * I + g) * L + 8 * J + 2 * tig + 1] = acc[1];
    }
    __syncthreads();
    const int n8 = 8 * NK;
    for (int idx = tid; idx < n8 * n8; idx += CQ_THREADS) {
        const int i = idx / n8, j = idx % n8;
        if ((i >> 3) <= (j >> 3)) Rt[i * L + j] = P[i * L + j];
    }
    for (int j = tid; j < KM; j += CQ_THREADS) rdt[j] = j < K ? 1.0 / P[j * L + j] : 0.0;
    __syncthreads();
}

// P = R^-1 (R upper, row-major Rr with pitch RLD, rdg = 1/diag), row-major
// pitch RLD, upper tiles only: the 8 x 8 diagonal blocks by back substitution
// (warp I, lanes over columns), then the blocks at distance dlt = 1, 2, ...
// from the diagonal, X_IJ = -X_II (sum_{M=I+1..J} R_IM X_MJ) on DMMA, one
// barrier per distance; the inner sum passes through the warp's 8 x 8 scratch
// in W to become an operand.
template <int KM>
__device__ void tri_inverse(const double *Rr, const double *rdg, double *P, double *W, int K, int tid) {
    constexpr int L = CQSmem<KM>::RLD;
    const int lane = tid & 31, warp = tid >> 5, g = lane >> 2, tig = lane & 3;
    const int NK = (K + 7) >> 3;
    if (warp < NK && lane < 8) {
        const int b0 = 8 * warp, c = lane;
        double x[8];
#pragma unroll
        for (int i = 7; i >= 0; --i) {
            double v = i == c ? 1.0 : 0.0;
#pragma unroll
            for (int m = i + 1; m < 8; ++m) v -= Rr[(b0 + i) * L + b0 + m] * x[m];
            x[i] = i <= c ? v * rdg[b0 + i] : 0.0;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) P[(b0 + i) * L + b0 + c] = x[i];
    }
    __syncthreads();
    double *w = W + warp * 96;
    for (int dlt = 1; dlt < NK; ++dlt) {
        const int I = warp, J = warp + dlt;
        if (J < NK) {
            double tacc[2] = {0.0, 0.0};
            for (int M = I + 1; M <= J; ++M) {
#pragma unroll
                for (int k4 = 0; k4 < 8; k4 += 4)
                    dmma884(tacc, Rr[(8 * I + g) * L + 8 * M + k4 + tig], P[(8 * M + k4 + tig) * L + 8 * J + g]);
            }
            w[g * 12 + 2 * tig] = tacc[0];
            w[g * 12 + 2 * tig + 1] = tacc[1];
            __syncwarp();
            double xacc[2] = {0.0, 0.0};
#pragma unroll
            for (int k4 = 0; k4 < 8; k4 += 4)
                dmma884(xacc, -P[(8 * I + g) * L + 8 * I + k4 + tig], w[(k4 + tig) * 12 + g]);
            P[(8 * I + g) * L + 8 * J + 2 * tig] = xacc[0];
            P[(8 * I + g) * L + 8 * J + 2 * tig + 1] = xacc[1];
        }
        __syncthreads();
    }
}

// QF: the tasks form Q (the range finder); instances without it carry no Q
// pass, which keeps the recompression's register allocation free of it.
template <int KM, bool QF>
__global__ void __launch_bounds__(CQ_THREADS, KM <= 32 ? 2 : 1) k_rcholqr(const CQTask *__restrict__ tasks,
                                                                         int *flags) {
    using S = CQSmem<KM>;
    constexpr bool STAGED = S::STAGED;
    constexpr int NACC = S::NACC;
    extern __shared__ __align__(16) double sm[];
    __shared__ double gmax_sh[CQ_WARPS];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int L = S::RLD;
    double *G = STAGED ? sm : sm + S::CHUNK;       // K x K Gram (column-major, ld KM); product scratch (pitch L)
    double *Rr = STAGED ? sm + S::CHUNK : G + S::RR;    // factor of the step, row-major: Rr[j * L + k] = R(j, k)
    double *Rt = Rr + S::RR;                       // accumulated R, row-major
    double *rdg = Rt + S::RR;                      // 1 / diag(Rr)
    double *rdt = rdg + KM;                        // 1 / diag(Rt)
    double *dsc = rdt + KM;                        // column norms of the sketch, then their inverses
    double *ivp = dsc + KM;                        // inverse pivots of the elimination
    double *Wsc = sm + S::CHUNK - S::WS;           // per-warp 8 x 8 scratch

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
            gram_reduce<KM>(acc, G, sm, tid, tmi, tni);
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
            factor<KM>(G, Rr, rdg, ivp, K, (double)CQ_CH, round == 0, tid);
            if (round == 0) {
                // Rt = R1 D, then the substitution of round 1 scales by 1/d first
                for (int idx = tid; idx < KM * KM; idx += CQ_THREADS) {
                    const int j = idx / KM, k = idx % KM;
                    Rt[j * L + k] = Rr[j * L + k] * dsc[k];
                }
                __syncthreads();
                for (int j = tid; j < KM; j += CQ_THREADS) {
                    rdt[j] = j < K ? 1.0 / Rt[j * L + j] : 0.0;
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
        // this warp's 32 rows of each chunk, staged column-major; at widths of
        // 48 and up (one CTA per SM, registers to spare) the next chunk's row is
        // loaded into registers while this one is solved and multiplied
        constexpr int P = STAGED ? CQ_LDZ : CQ_PITCH;
        constexpr bool PREFETCH = KM >= 48;
        double *zb = STAGED ? sm + warp * 32 : sm + warp * S::W;
        double v[KM];
        if (PREFETCH) load_row<KM>(t, STAGED ? tid : warp * 32 + lane, nb, k1, K, v);
#pragma unroll 1
        for (int r0 = STAGED ? 0 : warp * 32; r0 < nb; r0 += CQ_THREADS) {
            const int row = r0 + (STAGED ? tid : lane);
            const bool valid = row < nb;
            if (!PREFETCH) load_row<KM>(t, row, nb, k1, K, v);
#pragma unroll
            for (int j = 0; j < KM; ++j) zb[j * P + lane] = v[j];
            if (PREFETCH && r0 + CQ_THREADS < nb) load_row<KM>(t, row + CQ_THREADS, nb, k1, K, v);
            __syncwarp();
            // rd and R are zero past K, so the padding columns stay zero
            warp_trsm<KM, P>(zb, Rt, rdt, K, lane);
            if (valid && keep_y) {
                double *pz = t.Z + row;
                for (int j = 0; j < K; ++j, pz += nb) *pz = zb[j * P + lane];
            }
            if constexpr (STAGED) {
                __syncthreads();
                gram_tiles<KM>(acc, sm, lane, tmi, tni);
                __syncthreads();
            } else {
                gram_warp<KM>(acc, zb, lane);
                __syncwarp();
            }
        }
        gram_reduce<KM>(acc, G, sm, tid, tmi, tni);
        {
            // ||G||_inf: warp w sums the rows i = w, w + 8, ... (column i of the
            // symmetric G, lanes over its entries), then the max over the warps
            double mx = 0.0;
            for (int i = warp; i < K; i += CQ_WARPS) {
                double r = 0.0;
                for (int j = lane; j < K; j += 32) r += fabs(G[j + i * KM]);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
                mx = fmax(mx, r);
            }
            if (lane == 0) gmax_sh[warp] = mx;
        }
        const int nnull = factor<KM>(G, Rr, rdg, ivp, K, (double)nb, false, tid);   // barriers: gmax_sh visible
        if (nnull && tid == 0 && flags) atomicAdd(flags, nnull);
        double gmax = 0.0;
#pragma unroll
        for (int w = 0; w < CQ_WARPS; ++w) gmax = fmax(gmax, gmax_sh[w]);
        const bool again = !(gmax <= CQ_GMAX) && pass + 1 < CQ_APPLY;
        accumulate<KM>(Rr, Rt, G, rdt, K, tid);
        if (!again) break;
        if (tid == 0 && flags) atomicAdd(flags + 1, 1);
    }

    // outputs: R (column-major); Rc^-1 for a deferred Q; or Q = Y Rc^-1
    for (int idx = tid; idx < K * K; idx += CQ_THREADS) {
        const int i = idx % K, j = idx / K;
        t.R[i + (size_t)j * K] = Rt[i * L + j];
    }
    if (!QF && t.Rinv) {
        tri_inverse<KM>(Rr, rdg, G, Wsc, K, tid);
        for (int idx = tid; idx < K * K; idx += CQ_THREADS) {
            const int i = idx % K, c = idx / K;
            t.Rinv[i + (size_t)c * K] = i <= c ? G[i * L + c] : 0.0;
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
