// Tile generation (STARS-H covariance kernels), Gaussian sketch matrices,
// batched copies and small reductions.
//
// The covariance kernel restates starsh_ssdata_block_{sqrexp_kernel_2d,
// sqrexp_kernel_3d,exp_kernel_3d} (kernel pointers chosen at
// hicma_parsec/testing_dpotrf.c:338,346,354; call shape of
// hicma_parsec/STARSH_gen.jdf:70-72): A_ij = sigma * k(|x_i - x_j|) with the
// nugget added where the global row and column indices coincide.  The
// electrodynamics kinds restate starsh_eddata_block_sin_kernel_{2d,3d}
// (hicma_parsec/testing_dpotrf.c:330,361): A_ij = sin(k r) / r, and add_diag
// where r == 0.  randtlr (hicma_parsec/testing_dpotrf.c:315-321) reads a
// basis instead of points: pts holds [Q | Q diag(S)] (N x 2K, column-major)
// and A_ij = sum_k Q[i][k] (Q S)[j][k], plus add_diag where i == j.  The
// mesh-deformation kinds (md-3d-virus, md-3d-cube;
// hicma_parsec/testing_dpotrf.c:366-381, kernels starsh_generate_3d_virus /
// starsh_generate_3d_cube of the absent STARS-H) evaluate a radial basis
// function phi(r / radius) (-B, hicma_parsec/hicma_parsec.c:80) and add
// add_diag where i == j.
// Distances are accumulated with explicitly rounded operations
// (no FMA contraction) so that they match the CPU restatement bit for bit;
// exp/sin/sqrt are CUDA's.
#include "tlr_internal.h"

#include <algorithm>

namespace tlr {
namespace {

constexpr int COV_ROWS = 256;   // threads per block = rows per block
constexpr int COV_COLS = 8;     // columns per block

// Kernel families: the point kernels of the statistics problems, the
// electrodynamics sin(k r)/r kernels, and the randtlr basis products.  One
// instantiation each, so the families that need sin or the K-term loop do not
// add registers or stack to the others.
enum CovFamily { COV_STATS = 0, COV_ED = 1, COV_RANDTLR = 2, COV_RBF = 3 };

// Radial basis functions of s = r / radius (HICMA_TLR_RBF_*), polynomials
// with explicitly rounded operations (no FMA contraction).
__device__ __forceinline__ double rbf_phi(int f, double s) {
    switch (f) {
        case HICMA_TLR_RBF_GAUSSIAN: return exp(-__dmul_rn(s, s));
        case HICMA_TLR_RBF_EXPON: return exp(-s);
        case HICMA_TLR_RBF_INVQUAD: return __ddiv_rn(1.0, __dadd_rn(1.0, __dmul_rn(s, s)));
        case HICMA_TLR_RBF_INVMQUAD: return __ddiv_rn(1.0, __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(s, s))));
        case HICMA_TLR_RBF_MATERNC1: return __dmul_rn(__dadd_rn(1.0, s), exp(-s));
        case HICMA_TLR_RBF_MATERNC2:
            return __dmul_rn(__dadd_rn(__dadd_rn(1.0, s), __ddiv_rn(__dmul_rn(s, s), 3.0)), exp(-s));
        case HICMA_TLR_RBF_TPS: return s > 0.0 ? __dmul_rn(__dmul_rn(s, s), log(s)) : 0.0;
        case HICMA_TLR_RBF_CTPS: {
            if (s >= 1.0) return 0.0;
            const double t = __dsub_rn(1.0, s), t2 = __dmul_rn(t, t);
            return __dmul_rn(__dmul_rn(t2, t2), t);
        }
        default: {  // Wendland
            if (s >= 1.0) return 0.0;
            const double t = __dsub_rn(1.0, s), t2 = __dmul_rn(t, t);
            return __dmul_rn(__dmul_rn(t2, t2), __dadd_rn(__dmul_rn(4.0, s), 1.0));
        }
    }
}

template <int FAM>
__global__ void __launch_bounds__(COV_ROWS) k_cov_batched(CovParams p, const CovTask *__restrict__ tasks) {
    const CovTask t = tasks[blockIdx.z];
    const int r = blockIdx.x * COV_ROWS + threadIdx.x;
    const int c0 = blockIdx.y * COV_COLS;
    if (r >= t.nr || c0 >= t.nc) return;
    const int gr = t.r0 + r;
    const int cend = min(c0 + COV_COLS, t.nc);
    if (FAM == COV_RANDTLR) {
        const int K = p.ndim / 2;
        for (int c = c0; c < cend; ++c) {
            const int gc = t.c0 + c;
            double acc = 0.0;
            for (int k = 0; k < K; ++k)
                acc = fma(p.pts[(size_t)k * p.N + gr], p.pts[(size_t)(K + k) * p.N + gc], acc);
            if (gr == gc) acc += p.add_diag;
            t.out[(size_t)r + (size_t)c * t.ld] = acc;
        }
        return;
    }
    double xr[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) xr[a] = a < p.ndim ? p.pts[(size_t)a * p.N + gr] : 0.0;
    const double den = __dmul_rn(__dmul_rn(2.0, p.beta), p.beta);
    for (int c = c0; c < cend; ++c) {
        const int gc = t.c0 + c;
        double r2 = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (a < p.ndim) {
                const double d = __dsub_rn(xr[a], p.pts[(size_t)a * p.N + gc]);
                r2 = __dadd_rn(r2, __dmul_rn(d, d));
            }
        }
        double v;
        if (FAM == COV_RBF) {
            v = rbf_phi(p.rbf, __dmul_rn(__dsqrt_rn(r2), p.inv_radius));
            if (gr == gc) v = __dadd_rn(v, p.add_diag);
        } else if (FAM == COV_ED) {
            const double rr = __dsqrt_rn(r2);
            v = r2 == 0.0 ? p.add_diag : __ddiv_rn(sin(__dmul_rn(p.wave_k, rr)), rr);
        } else {
            if (p.kind == HICMA_TLR_KIND_EXP_3D)
                v = __dmul_rn(p.sigma, exp(-__ddiv_rn(__dsqrt_rn(r2), p.beta)));
            else
                v = __dmul_rn(p.sigma, exp(-__ddiv_rn(r2, den)));
            if (gr == gc) v = __dadd_rn(v, p.noise);
        }
        t.out[(size_t)r + (size_t)c * t.ld] = v;
    }
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    unsigned long long z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Box-Muller on two counter-based uniforms (u1 in (0,1], u2 in [0,1)).
__global__ void k_gaussian(double *out, int rows, int cols, int ld, unsigned long long seed) {
    const long long n = (long long)rows * cols;
    const unsigned long long base = mix64(seed);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long z1 = mix64(base + 2ull * (unsigned long long)i);
        const unsigned long long z2 = mix64(base + 2ull * (unsigned long long)i + 1ull);
        const double u1 = ((double)(z1 >> 11) + 1.0) * 0x1.0p-53;
        const double u2 = (double)(z2 >> 11) * 0x1.0p-53;
        const double g = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
        const int r = (int)(i % rows), c = (int)(i / rows);
        out[(size_t)r + (size_t)c * ld] = g;
    }
}

// randtlr bases: block b of a chunk was factored in place (R on and above
// the diagonal of Xr_b, NB x K, ld NB) and Q_b (NB x K) formed from its
// reflectors.  Column j is flipped where R_jj < 0 (the unique thin QR with a
// positive diagonal) and written to pts column j, and times decay^j to pts
// column K + j, at global row (m0 + b) * NB + i.
__global__ void k_randtlr_finish(const double *__restrict__ Xr, const double *__restrict__ Q, int nb, int K,
                                 int m0, double *__restrict__ pts, int N, double decay) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, b = blockIdx.z;
    if (i >= nb || j >= K) return;
    const size_t blk = (size_t)b * nb * K;
    const double sg = Xr[blk + (size_t)j + (size_t)j * nb] < 0.0 ? -1.0 : 1.0;
    double sj = 1.0;
    for (int t = 0; t < j; ++t) sj *= decay;
    const double q = Q[blk + (size_t)i + (size_t)j * nb] * sg;
    const size_t row = (size_t)(m0 + b) * nb + i;
    pts[(size_t)j * N + row] = q;
    pts[(size_t)(K + j) * N + row] = q * sj;
}

constexpr int CP_COLS = 4;
constexpr int CP_ROWS = 4;   // row iterations whose loads are issued together
// Copies (or scales, or adds into) CP_COLS columns of one task per CTA.  Source
// and destination never overlap (__restrict__), so every thread issues the
// loads of CP_COLS x CP_ROWS entries before its first store.
__global__ void __launch_bounds__(256) k_copy_batched(const CopyTask *__restrict__ tasks) {
    const CopyTask t = tasks[blockIdx.y];
    const int c0 = blockIdx.x * CP_COLS;
    if (c0 >= t.cols) return;
    const int nc = min(CP_COLS, t.cols - c0);
    const double *__restrict__ src = t.src + (size_t)c0 * t.lds;
    double *__restrict__ dst = t.dst + (size_t)c0 * t.ldd;
    const double alpha = t.alpha, beta = t.beta;
    for (int r0 = threadIdx.x; r0 < t.rows; r0 += CP_ROWS * blockDim.x) {
        double v[CP_COLS][CP_ROWS], w[CP_COLS][CP_ROWS];
#pragma unroll
        for (int c = 0; c < CP_COLS; ++c)
#pragma unroll
            for (int q = 0; q < CP_ROWS; ++q) {
                const int r = r0 + q * blockDim.x;
                const bool in = c < nc && r < t.rows;
                v[c][q] = in ? src[(size_t)c * t.lds + r] : 0.0;
                w[c][q] = (in && beta != 0.0) ? dst[(size_t)c * t.ldd + r] : 0.0;
            }
#pragma unroll
        for (int c = 0; c < CP_COLS; ++c)
#pragma unroll
            for (int q = 0; q < CP_ROWS; ++q) {
                const int r = r0 + q * blockDim.x;
                if (c < nc && r < t.rows)
                    dst[(size_t)c * t.ldd + r] = beta != 0.0 ? alpha * v[c][q] + beta * w[c][q]
                                                             : (alpha == 1.0 ? v[c][q] : alpha * v[c][q]);
            }
    }
}

__global__ void k_zero_upper(double *A, int n, int lda) {
    const int c = blockIdx.x;
    for (int r = threadIdx.x; r < c && r < n; r += blockDim.x) A[(size_t)r + (size_t)c * lda] = 0.0;
}

__global__ void k_set_identity(double *A, int n, int lda) {
    const int c = blockIdx.x;
    for (int r = threadIdx.x; r < n; r += blockDim.x) A[(size_t)r + (size_t)c * lda] = (r == c) ? 1.0 : 0.0;
}

// Deterministic single-block reduction of 2*log(diag).
__global__ void __launch_bounds__(1024) k_logdiag_sum(const double *const *tiles, int ntiles, int n,
                                                      int ld, double *out) {
    __shared__ double red[1024];
    double s = 0.0;
    const long long total = (long long)ntiles * n;
    for (long long i = threadIdx.x; i < total; i += blockDim.x) {
        const int t = (int)(i / n), j = (int)(i % n);
        s += 2.0 * log(tiles[t][(size_t)j + (size_t)j * ld]);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// Sum of squares of (X - Y) (Y may be null) over an m x n column-major
// matrix; sym_lower counts only the lower triangle with off-diagonal
// entries twice (Frobenius norm of the symmetric matrix stored in the lower
// triangle, as dplasma_dlansy(Frobenius, Lower)).  Per-block partials.
__global__ void __launch_bounds__(256) k_sumsq(const double *X, const double *Y, int m, int n, long long ld,
                                               int sym_lower, double *partial) {
    __shared__ double red[256];
    double s = 0.0;
    const long long total = (long long)m * n;
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < total; i += (long long)gridDim.x * 256) {
        const int r = (int)(i % m), c = (int)(i / m);
        if (sym_lower && r < c) continue;
        double v = X[(size_t)r + (size_t)c * ld];
        if (Y) v -= Y[(size_t)r + (size_t)c * ld];
        v *= v;
        s += (sym_lower && r > c) ? 2.0 * v : v;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void k_sum_final(const double *partial, int n, double *out) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) s += partial[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

__global__ void __launch_bounds__(256) k_assemble_r(const AssembleTask *__restrict__ tasks) {
    const AssembleTask t = tasks[blockIdx.x];
    const int rc = t.rc, ra = t.ra, K = rc + ra;
    for (int idx = threadIdx.x; idx < K * K; idx += blockDim.x) {
        const int i = idx % K, j = idx / K;
        double u = 0.0;
        if (i < rc) {
            if (j < rc) u = (i == j) ? 1.0 : 0.0;
            else u = t.Pu[(size_t)i + (size_t)(j - rc) * rc];
        } else if (j >= i) {
            u = t.Wu[(size_t)(i - rc) + (size_t)(j - rc) * t.nb];
        }
        t.RU[idx] = u;
    }
}

__global__ void __launch_bounds__(256) k_sumsq_batched(const NormTask *__restrict__ tasks) {
    const NormTask t = tasks[blockIdx.x];
    __shared__ double red[8];
    double s = 0.0;
    for (long long idx = threadIdx.x; idx < (long long)t.rows * t.cols; idx += blockDim.x) {
        const int r = (int)(idx % t.rows), c = (int)(idx / t.rows);
        const double x = t.X[(size_t)r + (size_t)c * t.ld];
        s += x * x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < 8; ++w) tot += red[w];
        *t.out = tot;
    }
}

__global__ void k_precision_select(const SelTask *__restrict__ tasks, int ntasks, double thr2, int *count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntasks) return;
    const SelTask t = tasks[i];
    const bool low = (*t.na) * (*t.nb) <= thr2;
    *t.sel32 = low ? t.n : 0;
    *t.sel64 = low ? 0 : t.n;
    if (low && count) atomicAdd(count, 1);
}

// out[i] += sum_k parts[k * len + i], k in increasing order (deterministic).
__global__ void k_accumulate(double *out, const double *parts, int nparts, long long len) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x) {
        double s = out[i];
        for (int k = 0; k < nparts; ++k) s += parts[(size_t)k * len + i];
        out[i] = s;
    }
}

}  // namespace

void launch_assemble_r(const AssembleTask *d_tasks, int ntasks, cudaStream_t st) {
    if (ntasks > 0) k_assemble_r<<<ntasks, 256, 0, st>>>(d_tasks);
}

void launch_sumsq_batched(const NormTask *d_tasks, int ntasks, cudaStream_t st) {
    if (ntasks > 0) k_sumsq_batched<<<ntasks, 256, 0, st>>>(d_tasks);
}
void launch_precision_select(const SelTask *d_tasks, int ntasks, double thr2, int *count, cudaStream_t st) {
    if (ntasks > 0) k_precision_select<<<(ntasks + 127) / 128, 128, 0, st>>>(d_tasks, ntasks, thr2, count);
}

void launch_accumulate(double *out, const double *parts, int nparts, long long len, cudaStream_t st) {
    if (len <= 0 || nparts <= 0) return;
    const long long blocks = std::min<long long>((len + 255) / 256, 4096);
    k_accumulate<<<(int)blocks, 256, 0, st>>>(out, parts, nparts, len);
}

void launch_sumsq(const double *X, const double *Y, int m, int n, long long ld, int sym_lower, double *partial,
                  int nblocks, double *out, cudaStream_t st) {
    k_sumsq<<<nblocks, 256, 0, st>>>(X, Y, m, n, ld, sym_lower, partial);
    k_sum_final<<<1, 256, 0, st>>>(partial, nblocks, out);
}

void launch_cov_batched(const CovParams &p, const CovTask *d_tasks, int ntasks, int max_nr, int max_nc,
                        cudaStream_t st) {
    if (ntasks <= 0) return;
    dim3 grid((max_nr + COV_ROWS - 1) / COV_ROWS, (max_nc + COV_COLS - 1) / COV_COLS, ntasks);
    if (p.kind == HICMA_TLR_KIND_RANDTLR)
        k_cov_batched<COV_RANDTLR><<<grid, COV_ROWS, 0, st>>>(p, d_tasks);
    else if (p.kind == HICMA_TLR_KIND_ED_SIN_2D || p.kind == HICMA_TLR_KIND_ED_SIN_3D)
        k_cov_batched<COV_ED><<<grid, COV_ROWS, 0, st>>>(p, d_tasks);
    else if (p.kind == HICMA_TLR_KIND_MD_VIRUS || p.kind == HICMA_TLR_KIND_MD_CUBE)
        k_cov_batched<COV_RBF><<<grid, COV_ROWS, 0, st>>>(p, d_tasks);
    else
        k_cov_batched<COV_STATS><<<grid, COV_ROWS, 0, st>>>(p, d_tasks);
}

void launch_gaussian(double *out, int rows, int cols, int ld, unsigned long long seed, cudaStream_t st) {
    const long long n = (long long)rows * cols;
    if (n <= 0) return;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_gaussian<<<blocks, 256, 0, st>>>(out, rows, cols, ld, seed);
}

void launch_randtlr_finish(const double *Xr, const double *Q, int nb, int K, int nblk, int m0, double *pts, int N,
                           double decay, cudaStream_t st) {
    if (nb <= 0 || K <= 0 || nblk <= 0) return;
    dim3 grid((nb + 255) / 256, K, nblk);
    k_randtlr_finish<<<grid, 256, 0, st>>>(Xr, Q, nb, K, m0, pts, N, decay);
}

void launch_copy_batched(const CopyTask *d_tasks, int ntasks, int max_cols, cudaStream_t st) {
    if (ntasks <= 0 || max_cols <= 0) return;
    dim3 grid((max_cols + CP_COLS - 1) / CP_COLS, ntasks);
    k_copy_batched<<<grid, 256, 0, st>>>(d_tasks);
}

void launch_zero_upper(double *A, int n, int lda, cudaStream_t st) {
    if (n <= 1) return;
    k_zero_upper<<<n, 256, 0, st>>>(A, n, lda);
}

void launch_set_identity(double *A, int n, int lda, cudaStream_t st) {
    if (n <= 0) return;
    k_set_identity<<<n, 256, 0, st>>>(A, n, lda);
}

void launch_logdiag_sum(const double *const *d_tiles, int ntiles, int n, int ld, double *out,
                        cudaStream_t st) {
    k_logdiag_sum<<<1, 1024, 0, st>>>(d_tiles, ntiles, n, ld, out);
}

}  // namespace tlr
