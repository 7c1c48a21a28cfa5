// QR factorization of a tall-skinny matrix by shifted CholeskyQR3, one CTA
// per matrix, FP64 (Gram products on the FP64 tensor cores).
//
// Replaces both QRs of HCORE_dgemm_qr_svd (call sites
// hicma_parsec/HiCMA_dpotrf_L_2flow.jdf:830-903,985-1058): the U side
// [Cu, Au] = Q_U R_U with Q_U formed (the new U is Q_U U_r, which replaces
// the Householder Q application of HCORE_dgemm_ormqr), and the V side
// [Cv, -Y] = Q_V R_V with R only (the new V is [Cv, -Y] R_U^T U_r).  The
// matrix is given as two column blocks read where they lie, so [Cu, Au] is
// never copied.
//
// Algorithm (Fukaya, Kannan, Nakatsukasa, Yamamoto, Yanagisawa, "Shifted
// Cholesky QR for computing the QR factorization of ill-conditioned
// matrices", SIAM J. Sci. Comput. 42(1), 2020): with D the column norms,
//   pass 0: G = D^-1 X^T X D^-1 + s I,  R1 = chol(G)
//   pass 1: X1 = X D^-1 R1^-1 (written to scratch), G = X1^T X1, R2 = chol(G)
//   pass 2: X2 = X1 R2^-1 (stored when Q is wanted), G = X2^T X2, R3 = chol(G)
//   pass 3: Q = X2 R3^-1 (only when Q is wanted; or X2 kept with R3^-1 out)
//   R = R3 R2 R1 D,
// s = 11 (m K + K (K + 1)) u tr(G); passes 1 and 2 add the same shift only if
// the plain Cholesky breaks down.  X R^-1 is a row-wise substitution (the
// backward-stable triangular solve the method's error bounds assume; an
// explicit inverse of R1 would add an error of order u cond(R1) ||X||).
//
// Layout: 8 warps, each working on its own 32-row chunks (rows warp*32 +
// 256 i + lane) with no CTA barrier inside a pass.  A lane keeps its row in
// registers for the substitution (R read as broadcasts from shared memory),
// stages the row into its warp's slice of shared memory (column-major, pitch
// 36: conflict-free for the row stores and for the DMMA fragment loads), and
// the warp accumulates the whole lower triangle of the chunk's Gram product
// with mma.sync m8n8k4 f64 (one fragment load per 8-column block and row
// quad, reused by every tile of that block).  The eight per-warp Gram
// partials are added in warp order at the end of a pass (deterministic), and
// one warp factors G in shared memory.  Kernels are instantiated per width
// bucket (KM = 16, 32, 48, 64 columns) so that unrolled loops do not run far
// past the actual K; at width 64 the CTA stages 256-row chunks instead (see
// CQSmem).  Wider stacks take the Householder path.
#include "tlr_internal.h"

namespace tlr {
namespace {

constexpr int CQ_WARPS = 8;
constexpr int CQ_THREADS = CQ_WARPS * 32;
constexpr int CQ_PITCH = 36;            // per-warp staged chunk pitch (== 4 mod 16)

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

constexpr int CQ_CH = CQ_THREADS;       // rows of a CTA-staged chunk (one per thread)
constexpr int CQ_LDZ = CQ_CH + 4;       // its pitch (== 4 mod 16)

// Widths up to 48: every warp stages and reduces its own 32-row chunks.
// Width 64 (CTA-staged): the row and the accumulators of all 36 tiles would
// not fit a thread's registers, so the CTA stages 256-row chunks and each
// warp accumulates the tiles it owns (no reduction); G and the scratch then
// live in the chunk buffer between passes.
template <int KM>
struct CQSmem {
    static constexpr bool STAGED = KM > 48;
    static constexpr int NT8 = KM / 8;
    static constexpr int NTILE = NT8 * (NT8 + 1) / 2;
    static constexpr int TPW = (NTILE + CQ_WARPS - 1) / CQ_WARPS;   // owned tiles per warp (staged)
    static constexpr size_t W = (size_t)KM * CQ_PITCH;    // one warp's staged chunk
    static constexpr size_t KK = (size_t)KM * KM;
    static constexpr size_t CHUNK = STAGED ? (size_t)KM * CQ_LDZ : CQ_WARPS * W;
    // chunk buffer(s) | [G | G copy / product scratch, unless in the chunk buffer] | Rr | Rt | d | 1/diag
    static constexpr size_t bytes() { return sizeof(double) * (CHUNK + (STAGED ? 2 : 4) * KK + 2 * KM); }
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

// In-place lower Cholesky of the K x K matrix G (column-major, ld KM) by one
// warp (lanes own rows); returns false on a non-positive pivot.
template <int KM>
__device__ bool warp_cholesky(double *G, int K, int lane) {
    for (int j = 0; j < K; ++j) {
        const double d = G[j + j * KM];
        if (!(d > 0.0)) return false;
        const double l = sqrt(d);
        const double il = 1.0 / l;
        __syncwarp();
        for (int i = j + 1 + lane; i < K; i += 32) G[i + j * KM] *= il;
        if (lane == 0) G[j + j * KM] = l;
        __syncwarp();
        // trailing update of the lower part: G[i][k] -= G[i][j] G[k][j], j < k <= i
        for (int i = j + 1 + lane; i < K; i += 32) {
            const double gij = G[i + j * KM];
            for (int k = j + 1; k <= i; ++k) G[i + k * KM] -= gij * G[k + j * KM];
        }
        __syncwarp();
    }
    return true;
}

template <int KM>
__global__ void __launch_bounds__(CQ_THREADS, KM <= 32 ? 2 : 1) k_cholqr3(const CQTask *__restrict__ tasks, int *fail) {
    using S = CQSmem<KM>;
    constexpr int NT8 = S::NT8, NTILE = S::NTILE;
    extern __shared__ double sm[];
    __shared__ int ok_sh;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tig = lane & 3;
    constexpr bool STAGED = S::STAGED;
    double *Zw = sm + warp * S::W;                 // this warp's staged chunk (widths up to 48)
    double *G = STAGED ? sm : sm + S::CHUNK;       // K x K Gram (column-major, ld KM)
    double *Gc = G + S::KK;                        // copy for a retry; product scratch
    double *Rr = STAGED ? sm + S::CHUNK : Gc + S::KK;   // R of the pass, row-major: Rr[j * KM + k] = R(j, k)
    double *Rt = Rr + S::KK;                       // accumulated R (column-major)
    double *dsc = Rt + S::KK;                      // column norms d_j (1 / d_j from pass 1 on)
    double *rdg = dsc + KM;                        // 1 / diag(R)

    const CQTask t = tasks[blockIdx.x];
    const int k1 = t.k1, K = t.k1 + t.k2, nb = t.nb;
    if (K <= 0) return;
    const double u = 1.1102230246251565e-16;
    const int npass = t.Q ? 4 : 3;

    // tiles owned by this warp in the CTA-staged form
    int tmi[S::TPW], tni[S::TPW];
#pragma unroll
    for (int q = 0; q < S::TPW; ++q) {
        const int tile = warp + CQ_WARPS * q;
        int mi = 0;
        while ((mi + 1) * (mi + 2) / 2 <= tile) ++mi;
        tmi[q] = (tile < NTILE && 8 * mi < K) ? mi : -1;
        tni[q] = tile - mi * (mi + 1) / 2;
    }

    for (int pass = 0; pass < npass; ++pass) {
        constexpr int NACC = STAGED ? 2 * S::TPW : NTILE;
        double acc[NACC][2];
#pragma unroll
        for (int q = 0; q < NACC; ++q) acc[q][0] = acc[q][1] = 0.0;
        const bool gram = pass < 3;

        for (int r0 = STAGED ? 0 : warp * 32; r0 < nb; r0 += CQ_THREADS) {
            const int row = r0 + (STAGED ? tid : lane);
            const bool valid = row < nb;
            double x[KM];
            if (pass < 2) {
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
            } else {
#pragma unroll
                for (int j = 0; j < KM; ++j) x[j] = (valid && j < K) ? t.Z[(size_t)row + (size_t)j * nb] : 0.0;
            }
            if (pass > 0) {
                if (pass == 1) {
#pragma unroll
                    for (int j = 0; j < KM; ++j) x[j] *= dsc[j];
                }
                // x <- x R^-1 (right-looking row substitution; R and 1/diag are
                // zero past K, so the padding columns stay zero)
                subst_rows<KM, 0>(x, Rr, rdg);
                // pass 1 stores X1, pass 2 X2 (when Q is wanted), pass 3 Q: each
                // lane rewrites only the row it read
                double *dst = pass == 3 ? t.Q : t.Z;
                if (valid && (pass == 1 || pass == 3 || (pass == 2 && (t.Q || t.Rinv)))) {
#pragma unroll
                    for (int j = 0; j < KM; ++j)
                        if (j < K) dst[(size_t)row + (size_t)j * nb] = x[j];
                }
            }
            if (!gram) continue;
            if constexpr (STAGED) {
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
                continue;
            }
#pragma unroll
            for (int j = 0; j < KM; ++j) Zw[j * CQ_PITCH + lane] = x[j];
            __syncwarp();
            // Gram of the chunk: row quads s, one fragment per 8-column block
            if constexpr (!STAGED) {
#pragma unroll 1
                for (int s = 0; s < 32; s += 4) {
                    double a[NT8];
#pragma unroll
                    for (int mi = 0; mi < NT8; ++mi) a[mi] = Zw[(8 * mi + g) * CQ_PITCH + s + tig];
                    int q = 0;
#pragma unroll
                    for (int mi = 0; mi < NT8; ++mi)
#pragma unroll
                        for (int ni = 0; ni <= mi; ++ni, ++q) dmma884(acc[q], a[mi], a[ni]);
                }
            }
            __syncwarp();
        }
        if (!gram) break;
        if constexpr (STAGED) {
            // owned tiles -> G (both triangles; the chunk buffer is free after the last barrier)
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
            // tiles past K (not computed) stay out of the factorization, which reads [0, K)
            __syncthreads();
        } else {
            // per-warp partials -> G in warp order (both triangles)
            for (int idx = tid; idx < KM * KM; idx += CQ_THREADS) G[idx] = 0.0;
            __syncthreads();
            for (int w = 0; w < CQ_WARPS; ++w) {
                if (warp == w) {
                    int q = 0;
#pragma unroll
                    for (int mi = 0; mi < NT8; ++mi)
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
        if (pass == 0) {
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
        // shift from the trace of G; Cholesky on warp 0
        if (warp == 0) {
            double tr = 0.0;
            for (int j = lane; j < K; j += 32) tr += G[j + j * KM];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) tr += __shfl_xor_sync(0xffffffffu, tr, o);
            const double shift = 11.0 * ((double)nb * K + (double)K * (K + 1)) * u * tr;
            for (int idx = lane; idx < K * K; idx += 32) {
                const int i = idx % K, j = idx / K;
                Gc[i + j * KM] = G[i + j * KM];
            }
            __syncwarp();
            // pass 0 always shifted; later passes shifted only after a breakdown,
            // and larger shifts (x100 each) should that still break down
            double sh = pass == 0 ? shift : 0.0;
            if (sh != 0.0) {
                for (int j = lane; j < K; j += 32) G[j + j * KM] += sh;
                __syncwarp();
            }
            bool good = warp_cholesky<KM>(G, K, lane);
            sh = pass == 0 ? shift * 100.0 : shift;
            for (int attempt = 0; !good && attempt < 4; ++attempt) {
                __syncwarp();
                for (int idx = lane; idx < K * K; idx += 32) {
                    const int i = idx % K, j = idx / K;
                    G[i + j * KM] = Gc[i + j * KM];
                }
                __syncwarp();
                for (int j = lane; j < K; j += 32) G[j + j * KM] += sh;
                __syncwarp();
                good = warp_cholesky<KM>(G, K, lane);
                sh = sh > 0.0 ? sh * 100.0 : 1e-300;
            }
            if (lane == 0) {
                ok_sh = good;
                if (!good && fail) atomicAdd(fail, 1);
            }
        }
        __syncthreads();
        // R of the pass, row-major (upper): Rr[j][k] = L(k, j); zero outside K
        for (int idx = tid; idx < KM * KM; idx += CQ_THREADS) {
            const int j = idx / KM, k = idx % KM;
            double v = 0.0;
            if (j <= k && k < K) v = ok_sh ? G[k + j * KM] : (j == k ? 1.0 : 0.0);
            Rr[j * KM + k] = v;
        }
        __syncthreads();
        for (int j = tid; j < KM; j += CQ_THREADS) rdg[j] = j < K ? 1.0 / Rr[j * KM + j] : 0.0;
        if (pass == 0) {
            for (int idx = tid; idx < KM * KM; idx += CQ_THREADS) Rt[idx] = Rr[idx];
        } else {
            // Rt <- R Rt (upper times upper, both row-major; consecutive threads
            // take consecutive columns: R read as a broadcast, Rt conflict-free)
            for (int idx = tid; idx < K * K; idx += CQ_THREADS) {
                const int i = idx / K, j = idx % K;
                double s = 0.0;
                for (int k = i; k <= j; ++k) s += Rr[i * KM + k] * Rt[k * KM + j];
                Gc[i * KM + j] = i <= j ? s : 0.0;
            }
            __syncthreads();
            for (int idx = tid; idx < K * K; idx += CQ_THREADS) {
                const int i = idx / K, j = idx % K;
                Rt[i * KM + j] = Gc[i * KM + j];
            }
        }
        __syncthreads();
        if (pass == 0) {
            // the substitution of pass 1 scales by 1/d first
            for (int j = tid; j < KM; j += CQ_THREADS) dsc[j] = 1.0 / dsc[j];
            __syncthreads();
        }
    }
    // R = Rt D (dsc holds 1/d)
    for (int idx = tid; idx < K * K; idx += CQ_THREADS) {
        const int i = idx % K, j = idx / K;
        t.R[i + (size_t)j * K] = i <= j ? Rt[i * KM + j] / dsc[j] : 0.0;
    }
    // Q deferred: X2 stays in Z and R3^-1 (R3 is the last pass's factor, still
    // in Rr, close to the identity) goes out, so the caller forms Q times a
    // small matrix as X2 (R3^-1 S) instead of a fourth pass over the rows.
    // One warp, rows of the inverse from the bottom up (lanes over columns),
    // built row-major in the scratch and written out column-major.
    if (t.Rinv && !t.Q) {
        if (warp == 0) {
            for (int i = K - 1; i >= 0; --i) {
                for (int c = lane; c < K; c += 32) {
                    double v = 0.0;
                    if (c == i) {
                        v = rdg[i];
                    } else if (c > i) {
                        double acc = 0.0;
                        for (int l = i + 1; l <= c; ++l) acc += Rr[i * KM + l] * Gc[l * KM + c];
                        v = -acc * rdg[i];
                    }
                    Gc[i * KM + c] = v;
                }
                __syncwarp();
            }
        }
        __syncthreads();
        for (int idx = tid; idx < K * K; idx += CQ_THREADS) {
            const int i = idx % K, c = idx / K;
            t.Rinv[i + (size_t)c * K] = Gc[i * KM + c];
        }
    }
}

template <int KM>
void launch_cq(const CQTask *d_tasks, int ntasks, int *fail, cudaStream_t st) {
    const size_t smem = CQSmem<KM>::bytes();
    // per device and thread-safe: set on every launch (a host-side call, no synchronisation)
    cudaFuncSetAttribute(k_cholqr3<KM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_cholqr3<KM><<<ntasks, CQ_THREADS, smem, st>>>(d_tasks, fail);
}

}  // namespace

int cholqr3_kmax() { return 64; }

int cholqr3_bucket(int K) { return K <= 16 ? 16 : K <= 32 ? 32 : K <= 48 ? 48 : 64; }

void launch_cholqr3_batched(const CQTask *d_tasks, int ntasks, int kmax, int *fail, cudaStream_t st) {
    if (ntasks <= 0) return;
    switch (cholqr3_bucket(kmax)) {
        case 16: launch_cq<16>(d_tasks, ntasks, fail, st); break;
        case 32: launch_cq<32>(d_tasks, ntasks, fail, st); break;
        case 48: launch_cq<48>(d_tasks, ntasks, fail, st); break;
        default: launch_cq<64>(d_tasks, ntasks, fail, st); break;
    }
}

}  // namespace tlr
