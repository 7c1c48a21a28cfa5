// Batched small-core SVD and rank truncation, FP64.
//
// Replaces the SVD + truncation step inside HCORE_dgemm_qr_svd (the core
// R_U R_V^T of a recompression, call sites
// hicma_parsec/HiCMA_dpotrf_L_2flow.jdf:830-903,985-1058) and the rank rule of
// starsh_dense_dlrrsdd (STARSH_gen.jdf:162-171).
//
// One CTA per core.  M = R_U R_V^T is formed in shared memory (global
// scratch when K is large) and a one-sided (Hestenes) Jacobi SVD
// orthogonalises its columns, W = M J = U Sigma, with a round-robin
// tournament ordering: each round rotates K/2 disjoint column pairs in
// parallel, LP lanes per pair, the three dot products of a pair reduced with
// warp shuffles.  The rotations are not accumulated: the caller recovers
// V Sigma = M^T U = R_V (R_U^T U) with two GEMMs, so only W lives on chip.
// One-sided Jacobi resolves small singular values to high relative accuracy,
// which the absolute truncation threshold needs; the decision is FP64.
#include "tlr_internal.h"

namespace tlr {
namespace {

constexpr int KMAX_SMEM = 160;
constexpr int MAX_SWEEPS = 40;

__device__ __forceinline__ int tourney(int slot, int round, int Kp) {
    return slot == 0 ? 0 : 1 + ((slot - 1 + round) % (Kp - 1));
}

template <int LP>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
    for (int o = LP / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int LP, int CT>
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
    double *W = in_smem ? sm : t.work;
    double *sig = in_smem ? sm + (size_t)K * K : sm;
    int *order = (int *)(sig + K);

    // M = RU RV^T (RU, RV upper triangular; RU null: identity); clean copy of RU
    for (long long idx = tid; idx < (long long)K * K; idx += CT) {
        const int i = (int)(idx % K), j = (int)(idx / K);
        double s = 0.0;
        if (t.RU) {
            const int l0 = i > j ? i : j;
            for (int l = l0; l < K; ++l)
                s += t.RU[(size_t)i + (size_t)l * t.ldru] * t.RV[(size_t)j + (size_t)l * t.ldrv];
            if (t.RUc) t.RUc[idx] = (i <= j) ? t.RU[(size_t)i + (size_t)j * t.ldru] : 0.0;
        } else {
            s = (j <= i) ? t.RV[(size_t)j + (size_t)i * t.ldrv] : 0.0;
        }
        W[idx] = s;
    }
    __syncthreads();

    // Columns whose norm is below tau can only move the result by O(tau) and
    // are truncated anyway: pairs involving them are not rotated.  tau is
    // 1e-3 of the absolute threshold (recompression) or of tol * ||M||_F
    // (generation); fixed-rank mode keeps every rotation.
    __shared__ double tau2_sh;
    if (tid == 0) {
        double tau = 0.0;
        if (p.mode == 0 && p.fixed_rank <= 0) tau = 1e-3 * p.tol;
        tau2_sh = tau * tau;
    }
    if (p.mode == 1) {
        double s2 = 0.0;
        for (long long idx = tid; idx < (long long)K * K; idx += CT) s2 += W[idx] * W[idx];
        s2 = group_sum<32>(s2);
        __shared__ double red[CT / 32];
        if (lane == 0) red[warp] = s2;
        __syncthreads();
        if (tid == 0) {
            double tot = 0.0;
            for (int w = 0; w < CT / 32; ++w) tot += red[w];
            tau2_sh = 1e-6 * p.tol * p.tol * tot;
        }
    }
    __syncthreads();
    const double tau2 = tau2_sh;

    constexpr int GPW = 32 / LP;                 // pair groups per warp
    const int groups = (CT / 32) * GPW;          // pair groups per CTA
    const int gsub = lane / LP, gl = lane % LP;
    const int Kp = K + (K & 1);
    // A pair counts as orthogonal when |c| <= tolj sqrt(a b).  The computed dot
    // products of K-term columns carry a rounding error of about K eps, so a
    // tighter threshold would keep rotating noise and never converge.
    const double tolj = 4.4e-16 * (double)(K > 16 ? K : 16);
    int sweeps = 0;
    if (K > 1) {
        for (int sweep = 0; sweep < MAX_SWEEPS; ++sweep) {
            if (tid == 0) rotated = 0;
            // exact squared column norms at the start of every sweep (sig is
            // free until the sweeps end); rotations keep them up to date
            for (int c = warp; c < K; c += CT / 32) {
                double s2 = 0.0;
                for (int r = lane; r < K; r += 32) s2 += W[(size_t)c * K + r] * W[(size_t)c * K + r];
                s2 = group_sum<32>(s2);
                if (lane == 0) sig[c] = s2;
            }
            __syncthreads();
            ++sweeps;
            for (int round = 0; round < Kp - 1; ++round) {
                // uniform trip count per warp: every lane reaches the shuffles
                for (int base = warp * GPW; base < Kp / 2; base += groups) {
                    const int pr = base + gsub;
                    int a = 0, b = 0;
                    bool valid = pr < Kp / 2;
                    if (valid) {
                        a = tourney(pr, round, Kp);
                        b = tourney(Kp - 1 - pr, round, Kp);
                        if (a > b) { const int tmp = a; a = b; b = tmp; }
                        valid = b < K && sig[a] > tau2 && sig[b] > tau2;
                    }
                    double aa = 0.0, bb = 0.0, cc = 0.0;
                    double *mp = W + (size_t)a * K, *mq = W + (size_t)b * K;
                    if (valid) {
                        for (int r = gl; r < K; r += LP) {
                            const double x = mp[r], y = mq[r];
                            aa += x * x; bb += y * y; cc += x * y;
                        }
                    }
                    aa = group_sum<LP>(aa);
                    bb = group_sum<LP>(bb);
                    cc = group_sum<LP>(cc);
                    if (!valid || cc == 0.0 || aa <= tau2 || bb <= tau2 || aa < 1e-290 || bb < 1e-290) continue;
                    if (fabs(cc) <= tolj * sqrt(aa) * sqrt(bb)) continue;
                    const double zeta = (bb - aa) / (2.0 * cc);
                    double tt;
                    if (fabs(zeta) > 1e150) tt = 0.5 / zeta;
                    else tt = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                    const double cs = 1.0 / sqrt(1.0 + tt * tt), sn = cs * tt;
                    for (int r = gl; r < K; r += LP) {
                        const double x = mp[r], y = mq[r];
                        mp[r] = cs * x - sn * y;
                        mq[r] = sn * x + cs * y;
                    }
                    if (gl == 0) {
                        rotated = 1;
                        sig[a] = aa - tt * cc;
                        sig[b] = bb + tt * cc;
                    }
                }
                __syncthreads();
            }
            if (!rotated) break;
            __syncthreads();
        }
    }

    // singular values and descending order
    for (int c = warp; c < K; c += CT / 32) {
        double s = 0.0;
        for (int r = lane; r < K; r += 32) s += W[(size_t)c * K + r] * W[(size_t)c * K + r];
        s = group_sum<32>(s);
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
        if (p.sweeps) atomicAdd(p.sweeps, sweeps);
    }
    __syncthreads();
    // left singular vectors, all K columns in decreasing sigma order
    for (long long idx = tid; idx < (long long)K * K; idx += CT) {
        const int row = (int)(idx % K), i = (int)(idx / K);
        const int c = order[i];
        const double s = sig[c];
        t.SU[idx] = s > 0.0 ? W[(size_t)c * K + row] / s : 0.0;
    }
}

template <int LP, int CT>
void launch_lp(const CoreTask *d, int n, size_t smem, const CoreParams &p, cudaStream_t st) {
    cudaFuncSetAttribute(k_core_svd<LP, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_core_svd<LP, CT><<<n, CT, smem, st>>>(d, p);
}

}  // namespace

int core_smem_kmax() { return KMAX_SMEM; }

void launch_core_svd_batched(const CoreTask *d_tasks, int ntasks, int kmax, const CoreParams &p,
                             cudaStream_t st) {
    if (ntasks <= 0) return;
    if (kmax < 1) kmax = 1;
    size_t smem;
    if (kmax <= KMAX_SMEM)
        smem = sizeof(double) * ((size_t)kmax * kmax + kmax) + sizeof(int) * kmax;
    else
        smem = sizeof(double) * (size_t)kmax + sizeof(int) * kmax;
    smem = (smem + 15) / 16 * 16;
    // lanes per pair ~ K/8 elements each; more pair groups per CTA for large K
    if (kmax <= 64) launch_lp<8, 256>(d_tasks, ntasks, smem, p, st);
    else if (kmax <= 96) launch_lp<16, 256>(d_tasks, ntasks, smem, p, st);
    else if (kmax <= KMAX_SMEM) launch_lp<16, 512>(d_tasks, ntasks, smem, p, st);
    else launch_lp<32, 512>(d_tasks, ntasks, smem, p, st);
}

}  // namespace tlr
