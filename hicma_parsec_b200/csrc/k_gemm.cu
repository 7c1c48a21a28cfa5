// Batched variable-size FP64 GEMM on the FP64 tensor cores (DMMA,
// mma.sync m8n8k4 f64) for sm_100a.  tcgen05 has no f64 kind, so FP64
// tensor-core work on Blackwell goes through DMMA.
//
// Replaces the CORE_dgemm / cblas_dgemm bodies of the reference task classes
// (hicma_parsec/HiCMA_dpotrf_L_2flow.jdf:704-708,717-728,745-778) and the
// products inside HCORE (low-rank SYRK/GEMM, QR/SVD recompression).
//
// CTA tile 64 x 64 x 16 (or 128 x 32 x 16 for outputs a rank wide), 4 warps
// (2 x 2 or 4 x 1, 32 x 32 each = 4 x 4 DMMA tiles),
// operands staged in shared memory by cp.async (2 stages, zero-filled at the
// edges).  op(A)/op(B) transposes are handled by the load mapping so every
// global load walks the contiguous dimension.  A batch is a list of tasks
// whose output tiles are flattened into one grid (prefix sums in tile_off).
#include "tlr_internal.h"

namespace tlr {
namespace {

constexpr int BM = 64, BN = 64, BK = 16, PAD = 8, NT = 128;

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async8(void *smem, const double *gmem, bool pred) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int sz = pred ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

template <int BM_, int BN_>
struct Smem {
    double A[2][BK][BM_ + PAD];
    double B[2][BK][BN_ + PAD];
};

template <int BM_, int BN_>
__device__ __forceinline__ void load_stage(Smem<BM_, BN_> &sm, int s, const GemmTask &t, int i0, int j0,
                                           int k0) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int q = 0; q < (BM_ * BK) / NT; ++q) {
        const int e = tid + q * NT;
        int i, kk;
        if (t.opA == 0) { i = e & (BM_ - 1); kk = e / BM_; }
        else            { kk = e & (BK - 1); i = e / BK; }
        const int gi = i0 + i, gk = k0 + kk;
        const bool p = gi < t.m && gk < t.k;
        const double *src = t.A;
        if (p) src += (t.opA == 0) ? ((size_t)gi + (size_t)gk * t.lda) : ((size_t)gk + (size_t)gi * t.lda);
        cp_async8(&sm.A[s][kk][i], src, p);
    }
#pragma unroll
    for (int q = 0; q < (BN_ * BK) / NT; ++q) {
        const int e = tid + q * NT;
        int j, kk;
        if (t.opB == 0) { kk = e & (BK - 1); j = e / BK; }
        else            { j = e & (BN_ - 1); kk = e / BN_; }
        const int gj = j0 + j, gk = k0 + kk;
        const bool p = gj < t.n && gk < t.k;
        const double *src = t.B;
        if (p) src += (t.opB == 0) ? ((size_t)gk + (size_t)gj * t.ldb) : ((size_t)gj + (size_t)gk * t.ldb);
        cp_async8(&sm.B[s][kk][j], src, p);
    }
    cp_async_commit();
}

// One BM_ x BN_ output tile; four warps of 32 x 32 (2 x 2 for 64 x 64,
// 4 x 1 for the narrow 128 x 32 tile used when n is a rank).
template <int BM_, int BN_>
__device__ __forceinline__ void gemm_tile(Smem<BM_, BN_> &sm, GemmTask t, int tm, int tn) {
    constexpr int WM = BM_ / 32;
    const int i0 = tm * BM_, j0 = tn * BN_;
    if (t.lower && j0 >= i0 + BM_) return;
    if (t.n_dev) {
        const int nd = *t.n_dev;
        t.n = nd < t.n ? nd : t.n;
    }
    if (j0 >= t.n) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int wm = warp % WM, wn = warp / WM;

    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

    // a triangular operand leaves the rest of the inner dimension zero for this tile
    int kend = t.k;
    if (t.tri == 1) kend = min(kend, i0 + BM_);
    else if (t.tri == 2) kend = min(kend, j0 + BN_);
    const int ktiles = (kend + BK - 1) / BK;
    if (ktiles > 0) load_stage<BM_, BN_>(sm, 0, t, i0, j0, 0);
    for (int kt = 0; kt < ktiles; ++kt) {
        const int s = kt & 1;
        if (kt + 1 < ktiles) {
            load_stage<BM_, BN_>(sm, s ^ 1, t, i0, j0, (kt + 1) * BK);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int k4 = 0; k4 < BK; k4 += 4) {
            double a[4], b[4];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi) a[mi] = sm.A[s][k4 + tig][wm * 32 + mi * 8 + g];
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) b[ni] = sm.B[s][k4 + tig][wn * 32 + ni * 8 + g];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) dmma884(acc[mi][ni], a[mi], b[ni]);
        }
        __syncthreads();
    }

    const double alpha = t.alpha, beta = t.beta;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
        const int row = i0 + wm * 32 + mi * 8 + g;
        if (row >= t.m) continue;
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int col = j0 + wn * 32 + ni * 8 + tig * 2 + e;
                if (col >= t.n) continue;
                double *c = t.C + (size_t)row + (size_t)col * t.ldc;
                double v = alpha * acc[mi][ni][e];
                if (beta != 0.0) v += beta * (*c);
                *c = v;
            }
        }
    }
}

// Task of output tile `bid`: the group table (after the ntasks + 1 prefix
// sums) names the task of the group's first tile; step forward from there.
__device__ __forceinline__ int task_of(const int *__restrict__ tile_off, int ntasks, int bid) {
    int lo = tile_off[ntasks + 1 + bid / GEMM_GROUP];
    while (lo + 1 < ntasks && tile_off[lo + 1] <= bid) ++lo;
    return lo;
}

template <int BM_, int BN_>
__global__ void __launch_bounds__(NT, 3) k_gemm_batched(const GemmTask *__restrict__ tasks,
                                                     const int *__restrict__ tile_off, int ntasks) {
    __shared__ __align__(16) Smem<BM_, BN_> sm;
    const int bid = blockIdx.x;
    const int lo = task_of(tile_off, ntasks, bid);
    const GemmTask t = tasks[lo];
    const int local = bid - tile_off[lo];
    gemm_tile<BM_, BN_>(sm, t, local % t.tiles_m, local / t.tiles_m);
}

__global__ void __launch_bounds__(NT) k_gemm_single(GemmTask t) {
    __shared__ __align__(16) Smem<BM, BN> sm;
    gemm_tile<BM, BN>(sm, t, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// FP32 product path of the mixed-precision policy: operands are read in FP64,
// rounded to FP32 in shared memory and multiplied with FP32 FMAs (FP32
// accumulation); the result is scaled and written back in FP64.
constexpr int FB = 64, FK = 16;
__global__ void __launch_bounds__(256) k_sgemm_batched(const GemmTask *__restrict__ tasks,
                                                       const int *__restrict__ tile_off, int ntasks) {
    __shared__ float As[FK][FB + 4];
    __shared__ float Bs[FK][FB + 4];
    const int bid = blockIdx.x;
    const int lo = task_of(tile_off, ntasks, bid);
    GemmTask t = tasks[lo];
    const int local = bid - tile_off[lo];
    const int i0 = (local % t.tiles_m) * FB, j0 = (local / t.tiles_m) * FB;
    if (t.lower && j0 >= i0 + FB) return;
    if (t.n_dev) {
        const int nd = *t.n_dev;
        t.n = nd < t.n ? nd : t.n;
    }
    if (j0 >= t.n) return;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    float acc[4][4] = {};
    int kend = t.k;
    if (t.tri == 1) kend = min(kend, i0 + FB);
    else if (t.tri == 2) kend = min(kend, j0 + FB);
    for (int k0 = 0; k0 < kend; k0 += FK) {
        for (int e = tid; e < FB * FK; e += 256) {
            int i, kk;
            if (t.opA == 0) { i = e & (FB - 1); kk = e / FB; } else { kk = e & (FK - 1); i = e / FK; }
            const int gi = i0 + i, gk = k0 + kk;
            float v = 0.f;
            if (gi < t.m && gk < t.k)
                v = (float)((t.opA == 0) ? t.A[(size_t)gi + (size_t)gk * t.lda] : t.A[(size_t)gk + (size_t)gi * t.lda]);
            As[kk][i] = v;
            int j;
            if (t.opB == 0) { kk = e & (FK - 1); j = e / FK; } else { j = e & (FB - 1); kk = e / FB; }
            const int gj = j0 + j, gk2 = k0 + kk;
            float w = 0.f;
            if (gj < t.n && gk2 < t.k)
                w = (float)((t.opB == 0) ? t.B[(size_t)gk2 + (size_t)gj * t.ldb] : t.B[(size_t)gj + (size_t)gk2 * t.ldb]);
            Bs[kk][j] = w;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < FK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) { a[q] = As[kk][tx + 16 * q]; b[q] = Bs[kk][ty + 16 * q]; }
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[p][q] = fmaf(a[p], b[q], acc[p][q]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int row = i0 + tx + 16 * p;
        if (row >= t.m) continue;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int col = j0 + ty + 16 * q;
            if (col >= t.n) continue;
            double *c = t.C + (size_t)row + (size_t)col * t.ldc;
            double v = t.alpha * (double)acc[p][q];
            if (t.beta != 0.0) v += t.beta * (*c);
            *c = v;
        }
    }
}

__global__ void k_gemm_devcount(const GemmTask *__restrict__ tasks, int ntasks, double *acc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntasks) return;
    const GemmTask t = tasks[i];
    if (!t.n_dev) return;
    const int nd = *t.n_dev;
    const double n = nd < t.n ? nd : t.n;
    if (n <= 0) return;
    atomicAdd(acc, 2.0 * t.m * n * t.k);
    atomicAdd(acc + 1, 8.0 * ((double)t.m * t.k + (double)t.k * n + (t.beta != 0.0 ? 2.0 : 1.0) * t.m * n));
}

}  // namespace

void launch_gemm_devcount(const GemmTask *d_tasks, int ntasks, double *acc, cudaStream_t st) {
    if (ntasks <= 0) return;
    k_gemm_devcount<<<(ntasks + 255) / 256, 256, 0, st>>>(d_tasks, ntasks, acc);
}

void launch_gemm_batched(const GemmTask *d_tasks, const int *d_tile_off, int ntasks, int total_tiles,
                         cudaStream_t st, bool fp32) {
    if (ntasks <= 0 || total_tiles <= 0) return;
    if (fp32)
        k_sgemm_batched<<<total_tiles, 256, 0, st>>>(d_tasks, d_tile_off, ntasks);
    else
        k_gemm_batched<BM, BN><<<total_tiles, NT, 0, st>>>(d_tasks, d_tile_off, ntasks);
}

void launch_gemm_batched_narrow(const GemmTask *d_tasks, const int *d_tile_off, int ntasks, int total_tiles,
                                cudaStream_t st) {
    if (ntasks <= 0 || total_tiles <= 0) return;
    k_gemm_batched<GEMM_NARROW_M, GEMM_NARROW_N><<<total_tiles, NT, 0, st>>>(d_tasks, d_tile_off, ntasks);
}

void launch_gemm_single(const GemmTask &t, cudaStream_t st) {
    if (t.m <= 0 || t.n <= 0) return;
    dim3 grid((t.m + BM - 1) / BM, (t.n + BN - 1) / BN);
    k_gemm_single<<<grid, NT, 0, st>>>(t);
}

}  // namespace tlr
