// R factor of a tall-skinny matrix by shifted CholeskyQR3, one CTA per
// matrix, FP64 (Gram products on the FP64 tensor cores).
//
// Replaces the V-side QR of HCORE_dgemm_qr_svd (call sites
// hicma_parsec/HiCMA_dpotrf_L_2flow.jdf:830-903,985-1058): only R_V of
// [Cv, -Y] = Q_V R_V is needed there (the new V is formed as
// [Cv, -Y] R_U^T U_r), so no Q is kept.
//
// Algorithm (Fukaya, Kannan, Nakatsukasa, Yamamoto, Yanagisawa, "Shifted
// Cholesky QR for computing the QR factorization of ill-conditioned
// matrices", SIAM J. Sci. Comput. 42(1), 2020): with D the column norms,
//   pass 0: G = D^-1 X^T X D^-1 + s I,  R1 = chol(G)
//   pass 1: X1 = X D^-1 R1^-1 (written to scratch), G = X1^T X1, R2 = chol(G)
//   pass 2: X2 = X1 R2^-1 (not stored),             G = X2^T X2, R3 = chol(G)
//   R = R3 R2 R1 D,
// s = 11 (m K + K (K + 1)) u tr(G); passes 1 and 2 add the same shift only if
// the plain Cholesky breaks down.  X R^-1 is a row-wise substitution (the
// backward-stable triangular solve the method's error bounds assume; an
// explicit inverse of R1 would add an error of order u cond(R1) ||X||).
//
// Layout: 256 threads, one row per thread in chunks of 256 rows; a thread
// keeps its row in registers for the substitution, then the chunk is staged
// column-major in shared memory (leading dimension 260: conflict-free both
// for the row-per-thread stores and for the DMMA fragment loads) and each
// warp accumulates its own 8 x 8 tiles of the lower triangle of G with
// mma.sync m8n8k4 f64 over the chunk.  Tiles are owned, so no cross-warp
// reduction is needed.  The K x K Cholesky runs in shared memory on one warp.
#include "tlr_internal.h"

namespace tlr {
namespace {

constexpr int VR_THREADS = 256;
constexpr int VR_CH = 256;              // rows per chunk (one per thread)
constexpr int VR_LDZ = VR_CH + 4;       // staged chunk leading dimension (== 4 mod 16)

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

template <int KM>
struct VRSmem {
    static constexpr int NT8 = KM / 8;
    static constexpr int NTILE = NT8 * (NT8 + 1) / 2;
    static constexpr int TPW = (NTILE + 7) / 8;     // tiles per warp (at most)
    static constexpr size_t Z = (size_t)KM * VR_LDZ; // staged chunk; also G and scratch between passes
    static constexpr size_t bytes() { return sizeof(double) * (Z + 2 * (size_t)KM * KM + 2 * KM); }
};

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
__global__ void __launch_bounds__(VR_THREADS, KM <= 32 ? 2 : 1) k_vside_r(const VRTask *__restrict__ tasks, int *fail) {
    using S = VRSmem<KM>;
    extern __shared__ double sm[];
    double *Zs = sm;                          // KM x VR_LDZ staged chunk (column j at j * VR_LDZ)
    double *Rp = Zs + S::Z;                   // this pass's R (upper, column-major, ld KM)
    double *Rt = Rp + (size_t)KM * KM;        // accumulated R
    double *dsc = Rt + (size_t)KM * KM;       // column norms d_j
    double *rdg = dsc + KM;                   // 1 / diag(Rp)
    __shared__ int ok_sh;

    const VRTask t = tasks[blockIdx.x];
    const int K = t.K, nb = t.nb, ldx = t.ldx;
    if (K <= 0) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int nt8 = (K + 7) / 8;
    const double u = 1.1102230246251565e-16;

    // this warp's tiles of the lower triangle of G (8 x 8 blocks (mi, ni), mi >= ni)
    int tmi[S::TPW], tni[S::TPW];
#pragma unroll
    for (int q = 0; q < S::TPW; ++q) {
        const int tile = warp + 8 * q;
        int mi = 0;
        while ((mi + 1) * (mi + 2) / 2 <= tile) ++mi;
        tmi[q] = (tile < S::NTILE && mi < nt8) ? mi : -1;
        tni[q] = tile - mi * (mi + 1) / 2;
    }

    for (int pass = 0; pass < 3; ++pass) {
        // two accumulators per tile (even and odd row quads): independent DMMA chains
        double acc[S::TPW][2][2];
#pragma unroll
        for (int q = 0; q < S::TPW; ++q) acc[q][0][0] = acc[q][0][1] = acc[q][1][0] = acc[q][1][1] = 0.0;

        for (int c0 = 0; c0 < nb; c0 += VR_CH) {
            const int row = c0 + tid;
            const bool valid = row < nb;
            double x[KM];
            const double *src = pass == 2 ? t.Z : t.X;
            const int lds = pass == 2 ? nb : ldx;
#pragma unroll
            for (int j = 0; j < KM; ++j) x[j] = (valid && j < K) ? src[(size_t)row + (size_t)j * lds] : 0.0;
            if (pass > 0) {
                if (pass == 1) {
#pragma unroll
                    for (int j = 0; j < KM; ++j)
                        if (j < K) x[j] /= dsc[j];
                }
                // x <- x Rp^-1 (right-looking row substitution)
#pragma unroll
                for (int j = 0; j < KM; ++j) {
                    if (j < K) {
                        x[j] *= rdg[j];
                        const double xj = x[j];
#pragma unroll
                        for (int k = j + 1; k < KM; ++k)
                            if (k < K) x[k] -= xj * Rp[j + k * KM];
                    }
                }
                if (pass == 1 && valid) {
#pragma unroll
                    for (int j = 0; j < KM; ++j)
                        if (j < K) t.Z[(size_t)row + (size_t)j * nb] = x[j];
                }
            }
#pragma unroll
            for (int j = 0; j < KM; ++j) Zs[j * VR_LDZ + tid] = x[j];
            __syncthreads();
            // G += Zc^T Zc over this chunk, all of this warp's tiles per row quad
#pragma unroll 2
            for (int r = 0; r < VR_CH; r += 8) {
#pragma unroll
                for (int q = 0; q < S::TPW; ++q) {
                    if (tmi[q] < 0) continue;
                    const double *za = Zs + (8 * tmi[q] + g) * VR_LDZ + tig + r;
                    const double *zb = Zs + (8 * tni[q] + g) * VR_LDZ + tig + r;
                    dmma884(acc[q][0], za[0], zb[0]);
                    dmma884(acc[q][1], za[4], zb[4]);
                }
            }
            __syncthreads();
        }
        // accumulators -> G (column-major KM x KM in the chunk buffer), both triangles
        double *G = Zs;
        double *Gc = Zs + (size_t)KM * KM;    // copy for a retry
#pragma unroll
        for (int q = 0; q < S::TPW; ++q) {
            if (tmi[q] < 0) continue;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int i = 8 * tmi[q] + g, j = 8 * tni[q] + 2 * tig + e;
                const double v = acc[q][0][e] + acc[q][1][e];
                G[i + j * KM] = v;
                G[j + i * KM] = v;
            }
        }
        __syncthreads();
        if (pass == 0) {
            for (int j = tid; j < K; j += VR_THREADS) {
                const double d = sqrt(G[j + j * KM]);
                dsc[j] = d > 0.0 ? d : 1.0;
            }
            __syncthreads();
            for (int idx = tid; idx < K * K; idx += VR_THREADS) {
                const int i = idx % K, j = idx / K;
                G[i + j * KM] /= dsc[i] * dsc[j];
            }
            __syncthreads();
        }
        // shift from the trace of G
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
        // Rp = L^T (upper), 1 / diag
        for (int idx = tid; idx < KM * KM; idx += VR_THREADS) {
            const int i = idx % KM, j = idx / KM;
            double v = 0.0;
            if (i <= j && j < K) v = ok_sh ? G[j + i * KM] : (i == j ? 1.0 : 0.0);
            Rp[i + j * KM] = v;
        }
        __syncthreads();
        for (int j = tid; j < K; j += VR_THREADS) rdg[j] = 1.0 / Rp[j + j * KM];
        // Rt <- Rp Rt (pass 0: Rt = Rp); upper times upper, via the G buffer
        if (pass == 0) {
            for (int idx = tid; idx < KM * KM; idx += VR_THREADS) Rt[idx] = Rp[idx];
        } else {
            double *T = Zs + 2 * (size_t)KM * KM;
            for (int idx = tid; idx < K * K; idx += VR_THREADS) {
                const int i = idx % K, j = idx / K;
                double s = 0.0;
                for (int k = i; k <= j; ++k) s += Rp[i + k * KM] * Rt[k + j * KM];
                T[i + j * KM] = i <= j ? s : 0.0;
            }
            __syncthreads();
            for (int idx = tid; idx < K * K; idx += VR_THREADS) {
                const int i = idx % K, j = idx / K;
                Rt[i + j * KM] = T[i + j * KM];
            }
        }
        __syncthreads();
    }
    // R = Rt D
    for (int idx = tid; idx < K * K; idx += VR_THREADS) {
        const int i = idx % K, j = idx / K;
        t.R[i + (size_t)j * K] = i <= j ? Rt[i + j * KM] * dsc[j] : 0.0;
    }
}

template <int KM>
void launch_vr(const VRTask *d_tasks, int ntasks, int *fail, cudaStream_t st) {
    const size_t smem = VRSmem<KM>::bytes();
    // per device and thread-safe: set on every launch (a host-side call, no synchronisation)
    cudaFuncSetAttribute(k_vside_r<KM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_vside_r<KM><<<ntasks, VR_THREADS, smem, st>>>(d_tasks, fail);
}

}  // namespace

int vside_r_kmax() { return 64; }

void launch_vside_r_batched(const VRTask *d_tasks, int ntasks, int kmax, int *fail, cudaStream_t st) {
    if (ntasks <= 0) return;
    if (kmax <= 32) launch_vr<32>(d_tasks, ntasks, fail, st);
    else launch_vr<64>(d_tasks, ntasks, fail, st);
}

}  // namespace tlr
