// Dense diagonal-block Cholesky and inverse (one CTA per 64 x 64 block).
//
// The blocked tile POTRF (HCORE_dpotrf at
// hicma_parsec/HiCMA_dpotrf_L_2flow.jdf:233) and the tile inverse used for
// the TRSMs are driven from the host engine: this kernel factors the jb x jb
// diagonal block in shared memory, reports the first non-positive pivot as
// the reference's INFO (k*mb + iinfo, :241-242) and writes L_jj^{-1} for the
// panel solve; the panel and trailing updates are DMMA GEMMs.
#include "tlr_internal.h"

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
    static bool configured = false;
    const size_t smem = 2 * DB * LDS * sizeof(double);
    if (!configured) {
        cudaFuncSetAttribute(k_potrf_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        configured = true;
    }
    k_potrf_diag<<<1, 256, smem, st>>>(A, lda, jb, Dinv, ldd, info, info_base);
}

}  // namespace tlr
