// Tile Cholesky and tile inverse in one persistent launch.
//
// Replaces HCORE_dpotrf on a diagonal tile (hicma_parsec/HiCMA_dpotrf_L_2flow.jdf
// :233-242) together with the inverse L^-1 that the panel solves of this
// engine apply as a GEMM.  The tile is split into 64 x 64 blocks and the
// blocked right-looking algorithm becomes a list of block tasks:
//   CHAIN        the critical path, run by one CTA from start to end: for each
//                block column j, Cholesky of A_jj and D_j = L_jj^-1, then
//                L_j+1,j = A_j+1,j D_j^T and A_j+1,j+1 -= L_j+1,j L_j+1,j^T,
//                the next diagonal block staying in shared memory
//   PANEL(j,i)   L_ij = A_ij D_j^T                        (i >= j + 2)
//   UPD(j,i,k)   A_ik -= L_ij L_kj^T         (j < k <= i, (i,k) != (j+1,j+1))
//   XDIAG(j,k)   X_jk = D_j B_jk                           (k < j)
//   XUPD(j,i,k)  B_ik -= L_ij X_jk                         (k <= j < i)
// where X = L^-1 is produced by block forward substitution on the identity
// (B starts as zero off the diagonal).  The chain is the first task; the rest
// of the list is in a topological order and CTAs take tasks from it with an
// atomic ticket, so every task waits only on the chain or on tasks already
// held by running CTAs, and the chain waits only on tasks of earlier block
// columns, which the other CTAs take in list order: the kernel makes progress
// with two or more CTAs, whether or not they are resident together, and needs
// no cooperative launch.  Dependencies are per-block counters released
// with a fence after the block is written and acquired by one thread before
// the CTA reads (through L2: ld.global.cg).  Every wait is bounded; a wait
// that gives up sets the timeout flag and the abort flag, and every CTA leaves
// at its next task.  A non-positive pivot sets the reference's INFO
// (k*NB + iinfo) and aborts the same way.  The block products run on the FP64
// tensor cores (mma.sync m8n8k4 f64).
#include "tlr_internal.h"

#include <map>
#include <mutex>
#include <vector>

namespace tlr {
namespace {

constexpr int TB = 64;          // block edge
constexpr int TPITCH = 72;      // shared pitch of DMMA operand tiles
constexpr int CP = TB + 4;      // shared pitch of the chain CTA's blocks (conflict-free DMMA fragments)
constexpr int NTH = 256;
constexpr long long SPIN_LIMIT = 1LL << 24;

enum { IT_CHAIN = 0, IT_PANEL, IT_UPD, IT_XDIAG, IT_XUPD };
struct PItem {
    unsigned short type, j, i, k;
};

struct PotrfParams {
    double *A;
    int lda, n, nblk;
    double *X;          // L^-1 (zeroed), or null
    int ldx;
    double *D;          // nblk x (64 x 64) block inverses when X is null
    const PItem *items;
    int nitems;
    int *cnt;           // [0] ticket [1] abort, then ver, pdone, xver, xdone (nblk^2 each), ddone (nblk)
    int *info;
    int info_base;
    int *timeout;
    long long spin_limit;   // polls before a wait gives up (SPIN_LIMIT in production)
};

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ int ld_volatile(const int *p) { return *(const volatile int *)p; }

// thread 0 only: wait until *p >= v
__device__ bool wait_ge(const int *p, int v, const PotrfParams &P) {
    for (long long it = 0; it < P.spin_limit; ++it) {
        if (ld_volatile(p) >= v) {
            __threadfence();
            return true;
        }
        if (ld_volatile(P.cnt + 1)) return false;
        __nanosleep(it < 256 ? 32 : 256);
    }
    atomicExch(P.timeout, 1);
    atomicExch(P.cnt + 1, 1);
    return false;
}

__device__ __forceinline__ int bsz(int b, int n) { return min(TB, n - b * TB); }

// C (m x nn, ldc) = beta C + alpha opA(A) opB(B), inner dimension kk <= 64.
// Operands are staged in shared memory before C is written, so C may alias
// A or B when beta = 0 (with beta != 0, C is read before the products and
// must not alias them).  The operand loads go out in two rounds of 16 per
// thread, and C's entries are fetched ahead of the products.
__device__ void blk_gemm(double *sm, double *C, int ldc, int m, int nn, int kk, double alpha, double beta,
                         const double *A, int lda, int opA, const double *B, int ldb, int opB) {
    double *As = sm;                 // As[k][i]
    double *Bs = sm + TB * TPITCH;   // Bs[k][j]
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int wm = warp & 1, wn = warp >> 1;   // 2 x 4 warps, 32 x 16 each
    constexpr int HALF = (TB * TB) / NTH / 2;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        double va[HALF], vb[HALF];
#pragma unroll
        for (int q = 0; q < HALF; ++q) {
            const int e = tid + (h * HALF + q) * NTH;
            int i, k;
            if (opA == 0) { i = e & (TB - 1); k = e >> 6; } else { k = e & (TB - 1); i = e >> 6; }
            va[q] = (i < m && k < kk) ? __ldcg(opA == 0 ? A + i + (size_t)k * lda : A + k + (size_t)i * lda) : 0.0;
            int j;
            if (opB == 0) { k = e & (TB - 1); j = e >> 6; } else { j = e & (TB - 1); k = e >> 6; }
            vb[q] = (j < nn && k < kk) ? __ldcg(opB == 0 ? B + k + (size_t)j * ldb : B + j + (size_t)k * ldb) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < HALF; ++q) {
            const int e = tid + (h * HALF + q) * NTH;
            int i, k, j;
            if (opA == 0) { i = e & (TB - 1); k = e >> 6; } else { k = e & (TB - 1); i = e >> 6; }
            As[k * TPITCH + i] = va[q];
            if (opB == 0) { k = e & (TB - 1); j = e >> 6; } else { j = e & (TB - 1); k = e >> 6; }
            Bs[k * TPITCH + j] = vb[q];
        }
    }
    double cv[4][2][2];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 2; ++ni)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int row = wm * 32 + mi * 8 + g, col = wn * 16 + ni * 8 + 2 * tig + e;
                cv[mi][ni][e] = (beta != 0.0 && row < m && col < nn) ? __ldcg(C + row + (size_t)col * ldc) : 0.0;
            }
    __syncthreads();
    double acc[4][2][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    const int k4end = (kk + 3) & ~3;
    for (int k4 = 0; k4 < k4end; k4 += 4) {
        double a[4], b[2];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) a[mi] = As[(k4 + tig) * TPITCH + wm * 32 + mi * 8 + g];
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) b[ni] = Bs[(k4 + tig) * TPITCH + wn * 16 + ni * 8 + g];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 2; ++ni) dmma884(acc[mi][ni], a[mi], b[ni]);
    }
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
        const int row = wm * 32 + mi * 8 + g;
        if (row >= m) continue;
#pragma unroll
        for (int ni = 0; ni < 2; ++ni)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int col = wn * 16 + ni * 8 + 2 * tig + e;
                if (col >= nn) continue;
                C[row + (size_t)col * ldc] = alpha * acc[mi][ni][e] + beta * cv[mi][ni][e];
            }
    }
}

// ------------------------------------------------------------ the chain ----
// The chain CTA keeps three 64 x 64 column-major blocks in shared memory
// (pitch CP): S (the diagonal block being factored), Xs (its inverse) and Pn
// (the panel block below it, and scratch of the inverse).  Blocks smaller
// than 64 are padded: with the identity on the diagonal of S, with zeros in
// Pn, so the padded parts factor to the identity and never reach the tile.
constexpr int CHAIN_SMEM_DOUBLES = 3 * TB * CP;

// M(r, c) = G(r, c) for r < rows, c < cols, else (r == c && pad_id); all of a
// thread's loads are issued before its shared stores.
__device__ __forceinline__ void load_frame(double *M, const double *G, int ld, int rows, int cols, bool pad_id) {
    const int tid = threadIdx.x;
    double v[(TB * TB) / NTH];
#pragma unroll
    for (int q = 0; q < (TB * TB) / NTH; ++q) {
        const int e = tid + q * NTH, r = e & (TB - 1), c = e >> 6;
        v[q] = (r < rows && c < cols) ? __ldcg(G + r + (size_t)c * ld) : ((pad_id && r == c) ? 1.0 : 0.0);
    }
#pragma unroll
    for (int q = 0; q < (TB * TB) / NTH; ++q) {
        const int e = tid + q * NTH;
        M[(e >> 6) * CP + (e & (TB - 1))] = v[q];
    }
}

// The 8-column panel p0..p0+7 of S on warps 0-2.  Every lane of the three
// warps factors the panel's 8 x 8 diagonal block itself, its lower part in
// registers, so the pivot chain has no shuffles (rsqrt(d) scales the column;
// the pivot is d * rsqrt(d), and the diagonal register keeps the reciprocal).
// The three warps meet once all of them have read the block; then lane 0 of
// warp 0 stores the factored block, warps 0 and 1 solve the rows below it (row p0+8+lane, row p0+40+lane), and lanes
// 0-7 of warp 2 write column `lane` of the block's inverse into Xs by forward
// substitution.  Returns the panel column of a non-positive pivot, or -1.
__device__ int chain_panel(double *S, double *Xs, int p0, int warp, int lane) {
    double d[8][8];   // d[r][c], c <= r
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c <= r; ++c) d[r][c] = S[(p0 + c) * CP + p0 + r];
    asm volatile("bar.sync 1, 96;" ::: "memory");   // warps 0-2: the block is read before it is rewritten
    const bool store = warp == 0 && lane == 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const double dc = d[c][c];
        if (!(dc > 0.0)) return c;          // the same on every lane
        const double inv = rsqrt(dc);
        d[c][c] = inv;
        if (store) S[(p0 + c) * CP + p0 + c] = dc * inv;
#pragma unroll
        for (int r = c + 1; r < 8; ++r) d[r][c] *= inv;
#pragma unroll
        for (int cc = c + 1; cc < 8; ++cc)
#pragma unroll
            for (int r = cc; r < 8; ++r) d[r][cc] = fma(-d[r][c], d[cc][c], d[r][cc]);
    }
    if (store) {
#pragma unroll
        for (int c = 0; c < 8; ++c)
#pragma unroll
            for (int r = c + 1; r < 8; ++r) S[(p0 + c) * CP + p0 + r] = d[r][c];
    }
    if (warp < 2) {
        const int row = p0 + 8 + 32 * warp + lane;
        if (row < TB) {
            double a[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) a[c] = S[(p0 + c) * CP + row];
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                a[c] *= d[c][c];
#pragma unroll
                for (int cc = c + 1; cc < 8; ++cc) a[cc] = fma(-a[c], d[cc][c], a[cc]);
            }
#pragma unroll
            for (int c = 0; c < 8; ++c) S[(p0 + c) * CP + row] = a[c];
        }
    } else if (lane < 8) {
        const int c = lane;
        double x[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            double s = 0.0;
#pragma unroll
            for (int l = 0; l < r; ++l)
                if (l >= c) s = fma(d[r][l], x[l], s);
            x[r] = r < c ? 0.0 : (r == c ? d[r][r] : -s * d[r][r]);
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) Xs[(p0 + c) * CP + p0 + r] = x[r];
    }
    return -1;
}

// Cholesky of S in place and its inverse in Xs (Pn is scratch).  Blocked by
// 8-column panels (chain_panel, which also inverts the panel's diagonal
// block), then every warp applies the panel's rank-8 update to the lower 8 x 8
// tiles of the trailing block on the tensor cores.  The inverse's diagonal
// blocks are then merged in pairs as X21 = -X22 (L21 X11) at widths 8, 16, 32.
// Returns the column (0..63) of a non-positive pivot, or -1.
__device__ int chain_diag(double *S, double *Xs, double *Pn) {
    __shared__ int bad_sh;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tig = lane & 3;
    for (int e = tid; e < TB * CP; e += NTH) Xs[e] = 0.0;
    __syncthreads();
    for (int p0 = 0; p0 < TB; p0 += 8) {
        if (warp < 3) {
            const int b = chain_panel(S, Xs, p0, warp, lane);
            if (warp == 0 && lane == 0) bad_sh = b < 0 ? -1 : p0 + b;
        }
        __syncthreads();
        if (bad_sh >= 0) return bad_sh;
        const int nbt = (TB - p0 - 8) / 8;   // trailing 8 x 8 block rows
        for (int t = warp; t < nbt * (nbt + 1) / 2; t += NTH / 32) {
            int bi = 0;
            while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
            const int bj = t - bi * (bi + 1) / 2;
            const int m0 = p0 + 8 + 8 * bi, n0 = p0 + 8 + 8 * bj;
            double acc[2] = {S[(n0 + 2 * tig) * CP + m0 + g], S[(n0 + 2 * tig + 1) * CP + m0 + g]};
#pragma unroll
            for (int k = 0; k < 8; k += 4)
                dmma884(acc, -S[(p0 + k + tig) * CP + m0 + g], S[(p0 + k + tig) * CP + n0 + g]);
            S[(n0 + 2 * tig) * CP + m0 + g] = acc[0];
            S[(n0 + 2 * tig + 1) * CP + m0 + g] = acc[1];
        }
        __syncthreads();
    }
    for (int h = 8; h < TB; h *= 2) {
        const int hb = h / 8, tpp = hb * hb, nt = (TB / (2 * h)) * tpp;
        // T = L21 X11 into the frame position of X21 in Pn (X11 lower: k >= the column block)
        for (int t = warp; t < nt; t += NTH / 32) {
            const int s0 = (t / tpp) * 2 * h, ti = (t % tpp) % hb, tj = (t % tpp) / hb;
            const int m0 = s0 + h + 8 * ti, n0 = s0 + 8 * tj;
            // two accumulators: the trip count is even, and the chains interleave
            double acc[2] = {0.0, 0.0}, acd[2] = {0.0, 0.0};
            for (int k = s0 + 8 * tj; k < s0 + h; k += 8) {
                dmma884(acc, S[(k + tig) * CP + m0 + g], Xs[(n0 + g) * CP + k + tig]);
                dmma884(acd, S[(k + 4 + tig) * CP + m0 + g], Xs[(n0 + g) * CP + k + 4 + tig]);
            }
            Pn[(n0 + 2 * tig) * CP + m0 + g] = acc[0] + acd[0];
            Pn[(n0 + 2 * tig + 1) * CP + m0 + g] = acc[1] + acd[1];
        }
        __syncthreads();
        // X21 = -X22 T (X22 lower: k up to the row block)
        for (int t = warp; t < nt; t += NTH / 32) {
            const int s0 = (t / tpp) * 2 * h, ti = (t % tpp) % hb, tj = (t % tpp) / hb;
            const int m0 = s0 + h + 8 * ti, n0 = s0 + 8 * tj;
            double acc[2] = {0.0, 0.0}, acd[2] = {0.0, 0.0};
            for (int k = s0 + h; k < m0 + 8; k += 8) {
                dmma884(acc, -Xs[(k + tig) * CP + m0 + g], Pn[(n0 + g) * CP + k + tig]);
                dmma884(acd, -Xs[(k + 4 + tig) * CP + m0 + g], Pn[(n0 + g) * CP + k + 4 + tig]);
            }
            Xs[(n0 + 2 * tig) * CP + m0 + g] = acc[0] + acd[0];
            Xs[(n0 + 2 * tig + 1) * CP + m0 + g] = acc[1] + acd[1];
        }
        __syncthreads();
    }
    return -1;
}

// One warp's 32 x 16 tile (rows wm*32.., cols wn*16..) of C = alpha X Y^T
// over k in [0, kend), X and Y column-major in shared memory; acc holds C on
// entry (or zero).
__device__ __forceinline__ void chain_mm_nt(double (&acc)[4][2][2], const double *X, const double *Y, double alpha,
                                            int kend, int wm, int wn, int g, int tig) {
    for (int k = 0; k < kend; k += 4) {
        double a[4], b[2];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) a[mi] = alpha * X[(k + tig) * CP + wm * 32 + mi * 8 + g];
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) b[ni] = Y[(k + tig) * CP + wn * 16 + ni * 8 + g];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 2; ++ni) dmma884(acc[mi][ni], a[mi], b[ni]);
    }
}

// The critical path of the tile: for j = 0, 1, ...: factor the diagonal block
// held in S, write L_jj and D_j, release ddone(j); then L_j+1,j = A_j+1,j D_j^T
// (written, released as pdone(j+1, j)) and S = A_j+1,j+1 - L_j+1,j L_j+1,j^T,
// each after the block's updates from the earlier columns are in.  Returns
// false if a wait gave up or a pivot failed (the abort flag is then set).
__device__ bool run_chain(double *sm, const PotrfParams &P) {
    __shared__ int ok_c;
    double *S = sm, *Xs = sm + TB * CP, *Pn = sm + 2 * TB * CP;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tig = lane & 3, wm = warp & 1, wn = warp >> 1;
    const int nb = P.nblk, n = P.n, lda = P.lda;
    int *ver = P.cnt + 8, *pdone = ver + nb * nb, *ddone = pdone + 3 * nb * nb;
    auto Ablk = [&](int r, int c) { return P.A + (size_t)r * TB + (size_t)c * TB * lda; };
    auto wait_all = [&](const int *p, int v) {
        if (tid == 0) ok_c = wait_ge(p, v, P);
        __syncthreads();
        return ok_c != 0;
    };
    load_frame(S, Ablk(0, 0), lda, bsz(0, n), bsz(0, n), true);
    __syncthreads();
    for (int j = 0; j < nb; ++j) {
        const int jb = bsz(j, n);
        const int bad = chain_diag(S, Xs, Pn);
        if (bad >= 0) {
            if (tid == 0) {
                // a pivot of the padding is 1: bad < jb
                if (P.info) atomicCAS(P.info, 0, P.info_base + j * TB + bad + 1);
                atomicExch(P.cnt + 1, 1);
            }
            return false;
        }
        double *Dj = P.X ? P.X + (size_t)j * TB + (size_t)j * TB * P.ldx : P.D + (size_t)j * TB * TB;
        const int ldd = P.X ? P.ldx : TB;
        double *Ajj = Ablk(j, j);
#pragma unroll 4
        for (int q = 0; q < (TB * TB) / NTH; ++q) {
            const int e = tid + q * NTH, r = e & (TB - 1), c = e >> 6;
            if (r < jb && c < jb) {
                Ajj[r + (size_t)c * lda] = r >= c ? S[c * CP + r] : 0.0;
                Dj[r + (size_t)c * ldd] = r >= c ? Xs[c * CP + r] : 0.0;
            }
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicExch(ddone + j, 1);
        }
        const int i = j + 1;
        if (i >= nb) break;
        const int ib = bsz(i, n);
        // L_ij = A_ij D_j^T (D_j^T upper: k stops at the warp's last column)
        if (!wait_all(ver + i * nb + j, j)) return false;
        load_frame(Pn, Ablk(i, j), lda, ib, TB, false);
        __syncthreads();
        double acc[4][2][2];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
        chain_mm_nt(acc, Pn, Xs, 1.0, wn * 16 + 16, wm, wn, g, tig);
        __syncthreads();
        double *Aij = Ablk(i, j);
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) {
            const int row = wm * 32 + mi * 8 + g;
#pragma unroll
            for (int ni = 0; ni < 2; ++ni)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int col = wn * 16 + ni * 8 + 2 * tig + e;
                    Pn[col * CP + row] = acc[mi][ni][e];
                    if (row < ib) Aij[row + (size_t)col * lda] = acc[mi][ni][e];
                }
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicExch(pdone + i * nb + j, 1);
        }
        // S = A_ii - L_ij L_ij^T (lower tiles; the warps above the diagonal skip)
        if (!wait_all(ver + i * nb + i, j)) return false;
        load_frame(S, Ablk(i, i), lda, ib, ib, true);
        __syncthreads();
        if (wm * 32 + 31 >= wn * 16) {
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 2; ++ni)
#pragma unroll
                    for (int e = 0; e < 2; ++e)
                        acc[mi][ni][e] = S[(wn * 16 + ni * 8 + 2 * tig + e) * CP + wm * 32 + mi * 8 + g];
            chain_mm_nt(acc, Pn, Pn, -1.0, TB, wm, wn, g, tig);
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 2; ++ni)
#pragma unroll
                    for (int e = 0; e < 2; ++e)
                        S[(wn * 16 + ni * 8 + 2 * tig + e) * CP + wm * 32 + mi * 8 + g] = acc[mi][ni][e];
        }
        __syncthreads();
    }
    return true;
}

__global__ void __launch_bounds__(NTH, 2) k_potrf_tile(PotrfParams P) {
    extern __shared__ double sm[];
    __shared__ int item_sh, ok_sh;
    const int tid = threadIdx.x;
    const int nb2 = P.nblk * P.nblk;
    int *ver = P.cnt + 8, *pdone = ver + nb2, *xver = pdone + nb2, *xdone = xver + nb2, *ddone = xdone + nb2;
    for (;;) {
        if (tid == 0) {
            int t = -1;
            if (!ld_volatile(P.cnt + 1)) {
                t = atomicAdd(P.cnt, 1);
                if (t >= P.nitems) t = -1;
            }
            item_sh = t;
        }
        __syncthreads();
        const int t = item_sh;
        if (t < 0) break;
        const PItem it = P.items[t];
        if (it.type == IT_CHAIN) {
            if (!run_chain(sm, P)) break;
            __syncthreads();
            continue;
        }
        const int j = it.j, i = it.i, k = it.k, n = P.n, nb = P.nblk;
        if (tid == 0) {
            bool ok = true;
            switch (it.type) {
                case IT_PANEL: ok = wait_ge(ddone + j, 1, P) && wait_ge(ver + i * nb + j, j, P); break;
                case IT_UPD:
                    ok = wait_ge(pdone + i * nb + j, 1, P) && wait_ge(pdone + k * nb + j, 1, P) &&
                         wait_ge(ver + i * nb + k, j, P);
                    break;
                case IT_XDIAG: ok = wait_ge(ddone + j, 1, P) && wait_ge(xver + j * nb + k, j - k, P); break;
                default:
                    ok = wait_ge(pdone + i * nb + j, 1, P) &&
                         (k == j ? wait_ge(ddone + j, 1, P) : wait_ge(xdone + j * nb + k, 1, P)) &&
                         wait_ge(xver + i * nb + k, j - k, P);
                    break;
            }
            ok_sh = ok;
        }
        __syncthreads();
        if (!ok_sh) break;
        const int lda = P.lda;
        auto Ablk = [&](int r, int c) { return P.A + (size_t)r * TB + (size_t)c * TB * lda; };
        auto Xblk = [&](int r, int c) { return P.X + (size_t)r * TB + (size_t)c * TB * P.ldx; };
        double *Dj = P.X ? Xblk(j, j) : P.D + (size_t)j * TB * TB;
        const int ldd = P.X ? P.ldx : TB;
        switch (it.type) {
            case IT_PANEL:
                blk_gemm(sm, Ablk(i, j), lda, bsz(i, n), bsz(j, n), bsz(j, n), 1.0, 0.0, Ablk(i, j), lda, 0, Dj, ldd, 1);
                break;
            case IT_UPD:
                blk_gemm(sm, Ablk(i, k), lda, bsz(i, n), bsz(k, n), bsz(j, n), -1.0, 1.0, Ablk(i, j), lda, 0,
                         Ablk(k, j), lda, 1);
                break;
            case IT_XDIAG:
                blk_gemm(sm, Xblk(j, k), P.ldx, bsz(j, n), bsz(k, n), bsz(j, n), 1.0, 0.0, Dj, ldd, 0, Xblk(j, k),
                         P.ldx, 0);
                break;
            default:
                blk_gemm(sm, Xblk(i, k), P.ldx, bsz(i, n), bsz(k, n), bsz(j, n), -1.0, 1.0, Ablk(i, j), lda, 0,
                         Xblk(j, k), P.ldx, 0);
                break;
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            switch (it.type) {
                case IT_PANEL: atomicExch(pdone + i * nb + j, 1); break;
                case IT_UPD: atomicExch(ver + i * nb + k, j + 1); break;
                case IT_XDIAG: atomicExch(xdone + j * nb + k, 1); break;
                default: atomicExch(xver + i * nb + k, j - k + 1); break;
            }
        }
    }
}

// The bulk tasks column by column (right-looking order: the updates of one
// block come from different columns, so they never queue behind each other).
// Each column starts with the three tasks the chain's step after next waits
// on: PANEL(j, j+2), UPD(j, j+2, j+1) and UPD(j, j+2, j+2).
std::vector<PItem> build_items(int nblk, bool inv) {
    std::vector<PItem> v;
    auto add = [&](int t, int j, int i, int k) {
        v.push_back(PItem{(unsigned short)t, (unsigned short)j, (unsigned short)i, (unsigned short)k});
    };
    add(IT_CHAIN, 0, 0, 0);
    for (int j = 0; j < nblk; ++j) {
        // the chain does PANEL(j, j+1) and UPD(j, j+1, j+1)
        if (j + 2 < nblk) {
            add(IT_PANEL, j, j + 2, 0);
            add(IT_UPD, j, j + 2, j + 1);
            add(IT_UPD, j, j + 2, j + 2);
        }
        for (int i = j + 3; i < nblk; ++i) add(IT_PANEL, j, i, 0);
        for (int i = j + 3; i < nblk; ++i) add(IT_UPD, j, i, j + 1);
        for (int k = j + 2; k < nblk; ++k)
            for (int i = k; i < nblk; ++i)
                if (i != j + 2 || k != j + 2) add(IT_UPD, j, i, k);
        if (inv) {
            for (int k = 0; k < j; ++k) add(IT_XDIAG, j, 0, k);
            for (int i = j + 1; i < nblk; ++i)
                for (int k = 0; k <= j; ++k) add(IT_XUPD, j, i, k);
        }
    }
    return v;
}

struct ItemList {
    PItem *d = nullptr;
    int n = 0;
};
std::mutex g_items_mu;
std::map<std::pair<int, long long>, ItemList> g_items;   // (device, nblk*2 + inv)

const ItemList *get_items(int nblk, bool inv, cudaStream_t st) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_items_mu);
    auto key = std::make_pair(dev, (long long)nblk * 2 + (inv ? 1 : 0));
    auto f = g_items.find(key);
    if (f != g_items.end()) return &f->second;
    std::vector<PItem> h = build_items(nblk, inv);
    ItemList L;
    if (cudaMalloc(&L.d, h.size() * sizeof(PItem)) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    // ordered on the launch stream and complete before the list is used (a
    // legacy-stream copy from pageable memory may land after the kernel reads it)
    if (cudaMemcpyAsync(L.d, h.data(), h.size() * sizeof(PItem), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaFree(L.d);
        return nullptr;
    }
    L.n = (int)h.size();
    return &(g_items[key] = L);
}

// Exercise of the bounded wait above, for tests: thread 0 of CTA b waits
// with wait_ge on the counter cnt[2 + b], which nothing sets, with limit
// limit0 (CTA 0) or limit1 (the others).  The first wait to run out sets the
// timeout and abort flags; the others then leave at their next poll.
__global__ void k_wait_probe(PotrfParams P, long long limit0, long long limit1) {
    if (threadIdx.x != 0) return;
    P.spin_limit = blockIdx.x == 0 ? limit0 : limit1;
    wait_ge(P.cnt + 2 + blockIdx.x, 1, P);
}

}  // namespace

int potrf_tile_max_n() { return 128 * TB; }

size_t potrf_tile_scratch_ints(int n) {
    const size_t nb = (size_t)(n + TB - 1) / TB;
    return 8 + 4 * nb * nb + nb;
}

// The caller provides cnt (potrf_tile_scratch_ints(n) ints, any content) and,
// when X is null, D (nblk * 64 * 64 doubles); X, when given, must be zeroed.
int launch_potrf_tile(double *A, int lda, int n, double *X, int ldx, double *D, int *cnt, int *info,
                      int info_base, int *timeout, int grid, cudaStream_t st) {
    const int nblk = (n + TB - 1) / TB;
    const ItemList *L = get_items(nblk, X != nullptr, st);
    if (!L) return -1;
    if (cudaMemsetAsync(cnt, 0, potrf_tile_scratch_ints(n) * sizeof(int), st) != cudaSuccess) return -1;
    const int smem = (int)sizeof(double) * (2 * TB * TPITCH > CHAIN_SMEM_DOUBLES ? 2 * TB * TPITCH : CHAIN_SMEM_DOUBLES);
    // per device and thread-safe: set on every launch (a host-side call, no synchronisation)
    cudaFuncSetAttribute(k_potrf_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    PotrfParams P{A, lda, n, nblk, X, ldx, D, L->d, L->n, cnt, info, info_base, timeout, SPIN_LIMIT};
    // the chain waits on bulk tasks of earlier block columns, which only the
    // other CTAs take: with any bulk task in the list the launch has two CTAs
    // or more (they need not be resident at the same time)
    if (grid > L->n) grid = L->n;
    if (grid < 2) grid = L->n > 1 ? 2 : 1;
    k_potrf_tile<<<grid, NTH, smem, st>>>(P);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// cnt: 2 + nblocks zeroed ints (abort flag at [1]); timeout: one zeroed int.
int launch_wait_probe(int *cnt, int *timeout, int nblocks, long long limit0, long long limit1, cudaStream_t st) {
    if (nblocks < 1 || nblocks > 64 || limit0 < 1 || limit1 < 1) return -1;
    PotrfParams P{};
    P.cnt = cnt;
    P.timeout = timeout;
    k_wait_probe<<<nblocks, 32, 0, st>>>(P, limit0, limit1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace tlr
