// Block Gram-Schmidt projection of new columns against an orthonormal basis
// (two rounds, "BCGS2"): W <- (I - C C^T)^2 W and P = C^T W_in accumulated,
// so that [C, W_in] = [C, W_out] [[I, P], [0, I]].
//
// Part of the recompression of a low-rank GEMM update (the QR of [U_C, U_A]
// inside HCORE_dgemm_qr_svd, called from hicma_parsec/HiCMA_dpotrf_L_2flow.jdf
// :745-778): the old U_C is orthonormal, so only the new columns need work.
//
// One CTA (8 warps) per update.  C^T W is an nb-long reduction into a small
// rc x ra block: each warp accumulates a 32 x 32 block of it over its own row
// slice with DMMA (mma.sync m8n8k4 f64), the slices are summed in a fixed
// order in shared memory (deterministic), and the CTA then forms
// W -= C P with DMMA, 32 x 32 output blocks per warp.  The update's data is
// read straight from global memory; between the passes it stays hot in L2.
#include "tlr_internal.h"

namespace tlr {
namespace {

constexpr int PW = 8;            // warps per CTA
constexpr int PT = PW * 32;
constexpr int PB = 32;           // output block edge

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// Pr = C^T W (rc x ra, ld rc)
__device__ void proj_gram(const double *__restrict__ C, const double *W, double *Pr, int nb, int rc, int ra,
                          double *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, tig = lane & 3;
    int chunk = (nb + PW - 1) / PW;
    chunk = (chunk + 3) & ~3;
    const int r0 = warp * chunk, r1 = min(nb, r0 + chunk);
    for (int bi = 0; bi < rc; bi += PB) {
        for (int bj = 0; bj < ra; bj += PB) {
            double acc[4][4][2];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
            // column offsets of this lane's C and W columns (-1: outside)
            int co[4], wo[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int ci = bi + 8 * q + g, cj = bj + 8 * q + g;
                co[q] = ci < rc ? ci * nb : -1;
                wo[q] = cj < ra ? cj * nb : -1;
            }
#pragma unroll 2
            for (int k = r0; k < r1; k += 4) {
                const int row = k + tig;
                const bool rv = row < r1;
                double a[4], b[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    a[q] = (rv && co[q] >= 0) ? __ldg(C + co[q] + row) : 0.0;
                    b[q] = (rv && wo[q] >= 0) ? W[wo[q] + row] : 0.0;
                }
#pragma unroll
                for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni) dmma884(acc[mi][ni], a[mi], b[ni]);
            }
            double *my = red + warp * PB * PB;
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                    for (int e = 0; e < 2; ++e) my[(8 * mi + g) * PB + 8 * ni + 2 * tig + e] = acc[mi][ni][e];
            __syncthreads();
            for (int idx = threadIdx.x; idx < PB * PB; idx += PT) {
                const int i = idx / PB, j = idx % PB;
                double s = 0.0;
#pragma unroll
                for (int w = 0; w < PW; ++w) s += red[w * PB * PB + idx];
                if (bi + i < rc && bj + j < ra) Pr[(size_t)(bi + i) + (size_t)(bj + j) * rc] = s;
            }
            __syncthreads();
        }
    }
}

// W -= C Pr
__device__ void proj_update(const double *__restrict__ C, double *W, const double *Pr, int nb, int rc, int ra) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int nrt = (nb + PB - 1) / PB, nbj = (ra + PB - 1) / PB;
    for (int item = warp; item < nrt * nbj; item += PW) {
        const int i0 = (item % nrt) * PB, j0 = (item / nrt) * PB;
        double acc[4][4][2];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
        for (int k = 0; k < rc; k += 4) {
            const int kk = k + tig;
            const bool kv = kk < rc;
            double a[4], b[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int row = i0 + 8 * q + g, col = j0 + 8 * q + g;
                a[q] = (kv && row < nb) ? __ldg(C + (size_t)row + (size_t)kk * nb) : 0.0;
                b[q] = (kv && col < ra) ? Pr[(size_t)kk + (size_t)col * rc] : 0.0;
            }
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) dmma884(acc[mi][ni], a[mi], b[ni]);
        }
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) {
            const int row = i0 + 8 * mi + g;
            if (row >= nb) continue;
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int col = j0 + 8 * ni + 2 * tig + e;
                    if (col < ra) W[(size_t)row + (size_t)col * nb] -= acc[mi][ni][e];
                }
        }
    }
}

__global__ void __launch_bounds__(PT, 2) k_bcgs2(const ProjTask *__restrict__ tasks) {
    extern __shared__ double red[];
    const ProjTask t = tasks[blockIdx.x];
    if (t.rc <= 0 || t.ra <= 0) return;
    proj_gram(t.C, t.W, t.P, t.nb, t.rc, t.ra, red);
    proj_update(t.C, t.W, t.P, t.nb, t.rc, t.ra);
    __syncthreads();
    proj_gram(t.C, t.W, t.P2, t.nb, t.rc, t.ra, red);
    proj_update(t.C, t.W, t.P2, t.nb, t.rc, t.ra);
    __syncthreads();
    for (int idx = threadIdx.x; idx < t.rc * t.ra; idx += PT) t.P[idx] += t.P2[idx];
}

// P = C^T W for a batch (the inner product B_V^T A_V of a recompression):
// the split-K DMMA reduction of the projection, one CTA per product.
__global__ void __launch_bounds__(PT, 2) k_gram_batched(const GramTask *__restrict__ tasks) {
    extern __shared__ double red[];
    const GramTask t = tasks[blockIdx.x];
    if (t.rc <= 0 || t.ra <= 0) return;
    proj_gram(t.C, t.W, t.P, t.nb, t.rc, t.ra, red);
}

// Orthogonality check of formed Q factors (the generation range finder):
// fail[i] = 1 when P = Q^T Q of task i (rc x rc, ld rc) differs from the
// identity by more than thr in an entry between nonzero columns, else 0.  A
// column of Q that is exactly zero (the sample had no component there) is
// harmless and skipped; NaN fails.  One warp per task.
__global__ void k_orth_check(const GramTask *__restrict__ tasks, int n, double thr, int *__restrict__ fail) {
    const int w = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (w >= n) return;
    const GramTask t = tasks[w];
    const int K = t.rc;
    int bad = 0;
    for (int idx = lane; idx < K * K; idx += 32) {
        const int i = idx % K, j = idx / K;
        const double gii = t.P[i + (size_t)i * K], gjj = t.P[j + (size_t)j * K];
        if (gii == 0.0 || gjj == 0.0) continue;
        const double e = t.P[idx] - (i == j ? 1.0 : 0.0);
        if (!(fabs(e) <= thr)) bad = 1;
    }
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) fail[w] = bad;
}

}  // namespace

void launch_orth_check(const GramTask *d_tasks, int ntasks, double thr, int *fail, cudaStream_t st) {
    if (ntasks <= 0) return;
    k_orth_check<<<(ntasks + 7) / 8, 256, 0, st>>>(d_tasks, ntasks, thr, fail);
}

void launch_gram_batched(const GramTask *d_tasks, int ntasks, cudaStream_t st) {
    if (ntasks <= 0) return;
    const int smem = PW * PB * PB * (int)sizeof(double);
    // per device and thread-safe: set on every launch (a host-side call, no synchronisation)
    cudaFuncSetAttribute(k_gram_batched, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_gram_batched<<<ntasks, PT, smem, st>>>(d_tasks);
}

void launch_bcgs2(const ProjTask *d_tasks, int ntasks, cudaStream_t st) {
    if (ntasks <= 0) return;
    const int smem = PW * PB * PB * (int)sizeof(double);
    // per device and thread-safe: set on every launch (a host-side call, no synchronisation)
    cudaFuncSetAttribute(k_bcgs2, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_bcgs2<<<ntasks, PT, smem, st>>>(d_tasks);
}

}  // namespace tlr
