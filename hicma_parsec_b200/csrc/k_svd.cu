// Batched small-core SVD and rank truncation, FP64.
//
// Replaces the SVD + truncation step inside HCORE_dgemm_qr_svd (the r x r
// core R_U R_V^T of a recompression, call sites
// hicma_parsec/HiCMA_dpotrf_L_2flow.jdf:830-903,985-1058) and the rank rule of
// starsh_dense_dlrrsdd (STARSH_gen.jdf:162-171).
//
// One CTA per core.  M = R_U R_V^T is formed in shared memory (global scratch
// when K is too large), then a one-sided (Hestenes) Jacobi SVD orthogonalises
// its columns with a round-robin tournament ordering: every round K/2
// disjoint column pairs are rotated in parallel, one warp per pair, the three
// dot products of a pair reduced with warp shuffles.  One-sided Jacobi gives
// small singular values to high relative accuracy, which is what the
// absolute truncation threshold needs.  The truncation decision is FP64.
#include "tlr_internal.h"

namespace tlr {
namespace {

constexpr int CT = 512;
constexpr int CW = CT / 32;
constexpr int KMAX_SMEM = 112;
constexpr int MAX_SWEEPS = 40;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int tourney(int slot, int round, int Kp) {
    return slot == 0 ? 0 : 1 + ((slot - 1 + round) % (Kp - 1));
}

__global__ void __launch_bounds__(CT) k_core_svd(const CoreTask *__restrict__ tasks, CoreParams p) {
    extern __shared__ double sm[];
    __shared__ int rotated;
    __shared__ int rank_sh;
    const CoreTask t = tasks[blockIdx.x];
    const int K = t.K;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (K <= 0) {
        if (tid == 0) {
            if (t.rank_out) *t.rank_out = 0;
            if (t.rank_task) *t.rank_task = 0;
        }
        return;
    }
    const bool in_smem = K <= KMAX_SMEM;
    double *M = in_smem ? sm : t.work;
    double *V = in_smem ? sm + (size_t)K * K : t.work + (size_t)K * K;
    double *sig = in_smem ? sm + 2 * (size_t)K * K : sm;
    int *order = (int *)(sig + K);

    // M = RU RV^T with RU, RV upper triangular (RU null: identity)
    for (long long idx = tid; idx < (long long)K * K; idx += CT) {
        const int i = (int)(idx % K), j = (int)(idx / K);
        double s = 0.0;
        if (t.RU) {
            const int l0 = i > j ? i : j;
            for (int l = l0; l < K; ++l)
                s += t.RU[(size_t)i + (size_t)l * t.ldru] * t.RV[(size_t)j + (size_t)l * t.ldrv];
        } else {
            s = (j <= i) ? t.RV[(size_t)j + (size_t)i * t.ldrv] : 0.0;
        }
        M[idx] = s;
        V[idx] = (i == j) ? 1.0 : 0.0;
    }
    __syncthreads();

    const int Kp = K + (K & 1);
    const double tolj = 2.3e-16 * sqrt((double)K);
    if (K > 1) {
        for (int sweep = 0; sweep < MAX_SWEEPS; ++sweep) {
            if (tid == 0) rotated = 0;
            __syncthreads();
            for (int round = 0; round < Kp - 1; ++round) {
                for (int pr = warp; pr < Kp / 2; pr += CW) {
                    int a = tourney(pr, round, Kp), b = tourney(Kp - 1 - pr, round, Kp);
                    if (a >= K || b >= K) continue;
                    if (a > b) { const int tmp = a; a = b; b = tmp; }
                    double *mp = M + (size_t)a * K, *mq = M + (size_t)b * K;
                    double aa = 0.0, bb = 0.0, cc = 0.0;
                    for (int r = lane; r < K; r += 32) {
                        const double x = mp[r], y = mq[r];
                        aa += x * x; bb += y * y; cc += x * y;
                    }
                    aa = warp_sum(aa); bb = warp_sum(bb); cc = warp_sum(cc);
                    if (cc == 0.0 || aa < 1e-290 || bb < 1e-290) continue;
                    if (fabs(cc) <= tolj * sqrt(aa) * sqrt(bb)) continue;
                    const double zeta = (bb - aa) / (2.0 * cc);
                    double tt;
                    if (fabs(zeta) > 1e150) tt = 0.5 / zeta;
                    else tt = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                    const double cs = 1.0 / sqrt(1.0 + tt * tt), sn = cs * tt;
                    for (int r = lane; r < K; r += 32) {
                        const double x = mp[r], y = mq[r];
                        mp[r] = cs * x - sn * y;
                        mq[r] = sn * x + cs * y;
                    }
                    double *vp = V + (size_t)a * K, *vq = V + (size_t)b * K;
                    for (int r = lane; r < K; r += 32) {
                        const double x = vp[r], y = vq[r];
                        vp[r] = cs * x - sn * y;
                        vq[r] = sn * x + cs * y;
                    }
                    if (lane == 0) rotated = 1;
                }
                __syncthreads();
            }
            if (!rotated) break;
            __syncthreads();
        }
    }

    // singular values and descending order
    for (int c = warp; c < K; c += CW) {
        double s = 0.0;
        for (int r = lane; r < K; r += 32) s += M[(size_t)c * K + r] * M[(size_t)c * K + r];
        s = warp_sum(s);
        if (lane == 0) sig[c] = sqrt(s);
    }
    __syncthreads();
    for (int c = tid; c < K; c += CT) {
        const double sc = sig[c];
        int pos = 0;
        for (int l = 0; l < K; ++l) {
            const double sl = sig[l];
            pos += (sl > sc) || (sl == sc && l < c);
        }
        order[pos] = c;
    }
    __syncthreads();
    if (tid == 0) {
        int r;
        if (p.mode == 0) {
            if (p.fixed_rank > 0) {
                r = p.fixed_rank < K ? p.fixed_rank : K;
            } else {
                r = 0;
                while (r < K && sig[order[r]] >= p.tol) ++r;
            }
            if (r > p.maxrank) {
                r = p.maxrank;
                if (p.overflow) atomicAdd(p.overflow, 1);
            }
        } else {
            double total = 0.0;
            for (int l = 0; l < K; ++l) total += sig[l] * sig[l];
            if (total == 0.0) {
                r = 0;
            } else {
                const double thr = p.tol * p.tol * total;
                double tail = 0.0;
                r = K;
                while (r > 0) {
                    const double s2 = sig[order[r - 1]] * sig[order[r - 1]];
                    if (tail + s2 > thr) break;
                    tail += s2;
                    --r;
                }
            }
            if (!(2 * r < p.nb && r <= p.maxrank)) r = -1;
        }
        rank_sh = r;
        if (t.rank_out) *t.rank_out = r;
        if (t.rank_task) *t.rank_task = r;
    }
    __syncthreads();
    const int r = rank_sh;
    for (long long idx = tid; idx < (long long)K * (r > 0 ? r : 0); idx += CT) {
        const int row = (int)(idx % K), i = (int)(idx / K);
        const int c = order[i];
        const double s = sig[c];
        t.SU[(size_t)row + (size_t)i * K] = s > 0.0 ? M[(size_t)c * K + row] / s : 0.0;
        t.SV[(size_t)row + (size_t)i * K] = V[(size_t)c * K + row] * s;
    }
}

}  // namespace

int core_smem_kmax() { return KMAX_SMEM; }

void launch_core_svd_batched(const CoreTask *d_tasks, int ntasks, int kmax, const CoreParams &p,
                             cudaStream_t st) {
    if (ntasks <= 0) return;
    size_t smem;
    if (kmax <= KMAX_SMEM)
        smem = sizeof(double) * (2 * (size_t)kmax * kmax + (size_t)kmax) + sizeof(int) * kmax;
    else
        smem = sizeof(double) * (size_t)kmax + sizeof(int) * kmax;
    // tasks with K <= KMAX_SMEM keep M and V in shared memory
    const size_t smem_small = sizeof(double) * (2 * (size_t)KMAX_SMEM * KMAX_SMEM + KMAX_SMEM) +
                              sizeof(int) * KMAX_SMEM;
    if (smem < smem_small && kmax > KMAX_SMEM) smem = smem_small;
    if (kmax > KMAX_SMEM) smem = smem > smem_small ? smem : smem_small;
    cudaFuncSetAttribute(k_core_svd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_core_svd<<<ntasks, CT, smem, st>>>(d_tasks, p);
}

}  // namespace tlr
