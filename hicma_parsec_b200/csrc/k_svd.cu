// Batched small-core SVD and rank truncation, FP64.
//
// Replaces the SVD + truncation step inside HCORE_dgemm_qr_svd (the core
// R_U R_V^T of a recompression, call sites
// hicma_parsec/HiCMA_dpotrf_L_2flow.jdf:830-903,985-1058) and the rank rule of
// starsh_dense_dlrrsdd (STARSH_gen.jdf:162-171).
//
// One CTA per core, QR-preconditioned one-sided Jacobi (Drmac and Veselic,
// "New fast and accurate Jacobi SVD algorithm", SIMAX 2008):
//   1. T = M^T with M = R_U R_V^T is formed in shared memory (global scratch
//      when K is large).
//   2. Householder QR with column pivoting, T P = Q R, one warp choosing the
//      pivot and building the reflector, all warps applying it (one column
//      per warp, exact partial column norms recomputed in the same pass).  It
//      stops at step k once the trailing block's Frobenius norm is below the
//      truncation floor, so only the leading k rows of R survive; k is about
//      the numerical rank, not K.
//   3. R^T (K x k, in place) is orthogonalised by one-sided (Hestenes) Jacobi,
//      X J = W Sigma, with a round-robin tournament ordering: each round
//      rotates k/2 disjoint column pairs in parallel, LP lanes per pair, dot
//      products reduced with warp shuffles.  The rows of a pivoted R are
//      graded, so the columns of R^T are nearly orthogonal and few sweeps are
//      needed.
//   4. P^T M = R^T Q^T, so the left singular vectors of M are the rows of W
//      permuted back: U[piv[q], :] = W[q, :] / sigma.  Neither Q nor J is
//      formed; the caller recovers V Sigma = M^T U = R_V (R_U^T U) with GEMMs.
// One-sided Jacobi resolves small singular values to high relative accuracy,
// which the absolute truncation threshold needs; the decision is FP64.
#include "tlr_internal.h"

#include <cooperative_groups.h>

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
    __shared__ int rotated, rank_sh, stop_sh;
    __shared__ double tau_sh, tail_sh, tau2_sh;
    constexpr int NW = CT / 32;
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
    double *sig = in_smem ? sm + (size_t)K * K : sm;   // partial norms^2, then sigma
    double *hv = sig + K;                               // Householder vector
    int *order = (int *)(hv + K);
    int *piv = order + K;

    // 1. T = M^T: T(i, c) = M(c, i) = sum_{l >= max(i, c)} RU(c, l) RV(i, l)
    //    (RU null: M = RV^T, T = RV); clean copy of RU on request
    for (long long idx = tid; idx < (long long)K * K; idx += CT) {
        const int i = (int)(idx % K), c = (int)(idx / K);
        double s = 0.0;
        if (t.RU) {
            const int l0 = i > c ? i : c;
            for (int l = l0; l < K; ++l)
                s += t.RU[(size_t)c + (size_t)l * t.ldru] * t.RV[(size_t)i + (size_t)l * t.ldrv];
            if (t.RUc) t.RUc[idx] = (i <= c) ? t.RU[(size_t)i + (size_t)c * t.ldru] : 0.0;
        } else {
            s = (i <= c) ? t.RV[(size_t)i + (size_t)c * t.ldrv] : 0.0;
        }
        W[idx] = s;
    }
    __syncthreads();
    // column norms^2 and the identity pivot
    for (int c = warp; c < K; c += NW) {
        double s2 = 0.0;
        for (int r = lane; r < K; r += 32) s2 += W[(size_t)c * K + r] * W[(size_t)c * K + r];
        s2 = group_sum<32>(s2);
        if (lane == 0) { sig[c] = s2; piv[c] = c; }
    }
    __syncthreads();
    // Truncation floor tau2 on squared norms: 1e-3 of the absolute threshold
    // (recompression) or of tol * ||M||_F (generation); zero in fixed-rank mode.
    if (tid == 0) {
        double tau = 0.0;
        if (p.mode == 0 && p.fixed_rank <= 0) tau = 1e-3 * p.tol;
        double tau2 = tau * tau;
        if (p.mode == 1) {
            double tot = 0.0;
            for (int c = 0; c < K; ++c) tot += sig[c];
            tau2 = 1e-6 * p.tol * p.tol * tot;
        }
        tau2_sh = tau2;
        tail_sh = 0.0;
    }
    __syncthreads();
    const double tau2 = tau2_sh;

    // 2. pivoted Householder QR of T, stopped when the trailing mass <= tau2
    int k = K;
    for (int j = 0; j < K; ++j) {
        if (warp == 0) {
            double tr = 0.0, best = -1.0;
            int bi = j;
            for (int c = j + lane; c < K; c += 32) {
                const double v = sig[c];
                tr += v;
                if (v > best) { best = v; bi = c; }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                tr += __shfl_xor_sync(0xffffffffu, tr, o);
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            const bool stop = !(tr > tau2);
            if (lane == 0) {
                stop_sh = stop;
                if (stop) tail_sh = tr;
            }
            if (!stop) {
                double *cj = W + (size_t)j * K;
                if (bi != j) {
                    double *cb = W + (size_t)bi * K;
                    for (int r = lane; r < K; r += 32) {
                        const double x = cj[r];
                        cj[r] = cb[r];
                        cb[r] = x;
                    }
                    if (lane == 0) {
                        const double sx = sig[j]; sig[j] = sig[bi]; sig[bi] = sx;
                        const int px = piv[j]; piv[j] = piv[bi]; piv[bi] = px;
                    }
                    __syncwarp();
                }
                const double alpha = cj[j];
                double s2 = 0.0;
                for (int r = j + 1 + lane; r < K; r += 32) s2 += cj[r] * cj[r];
                s2 = group_sum<32>(s2);
                double th = 0.0, scl = 0.0, beta = alpha;
                if (s2 > 0.0) {
                    beta = -copysign(sqrt(alpha * alpha + s2), alpha);
                    th = (beta - alpha) / beta;
                    scl = 1.0 / (alpha - beta);
                }
                for (int r = j + 1 + lane; r < K; r += 32) {
                    hv[r] = cj[r] * scl;
                    cj[r] = 0.0;
                }
                if (lane == 0) {
                    hv[j] = 1.0;
                    cj[j] = beta;
                    tau_sh = th;
                }
            }
        }
        __syncthreads();
        if (stop_sh) { k = j; break; }
        const double th = tau_sh;
        for (int c = j + 1 + warp; c < K; c += NW) {
            double *col = W + (size_t)c * K;
            double w = 0.0;
            for (int r = j + lane; r < K; r += 32) w += hv[r] * col[r];
            w = group_sum<32>(w) * th;
            double s2 = 0.0;
            for (int r = j + lane; r < K; r += 32) {
                const double x = col[r] - w * hv[r];
                col[r] = x;
                if (r > j) s2 += x * x;
            }
            s2 = group_sum<32>(s2);
            if (lane == 0) sig[c] = s2;
        }
        __syncthreads();
    }
    // R^T in place: swap the upper and lower triangles of the rows that stay
    for (long long idx = tid; idx < (long long)K * K; idx += CT) {
        const int i = (int)(idx % K), c = (int)(idx / K);
        if (i < c && i < k) {
            const double x = W[(size_t)i + (size_t)c * K];
            W[(size_t)i + (size_t)c * K] = W[(size_t)c + (size_t)i * K];
            W[(size_t)c + (size_t)i * K] = x;
        }
    }
    __syncthreads();

    // 3. one-sided Jacobi on the k columns (length K) of R^T
    constexpr int GPW = 32 / LP;                 // pair groups per warp
    const int groups = NW * GPW;                 // pair groups per CTA
    const int gsub = lane / LP, gl = lane % LP;
    const int kp = k + (k & 1);
    // A pair counts as orthogonal when |c| <= tolj sqrt(a b).  The computed dot
    // products of K-term columns carry a rounding error of about K eps, so a
    // tighter threshold would keep rotating noise and never converge.
    const double tolj = 4.4e-16 * (double)(K > 16 ? K : 16);
    int sweeps = 0;
    if (k > 1) {
        for (int sweep = 0; sweep < MAX_SWEEPS; ++sweep) {
            if (tid == 0) rotated = 0;
            // exact squared column norms at the start of every sweep; rotations
            // keep them up to date
            for (int c = warp; c < k; c += NW) {
                double s2 = 0.0;
                for (int r = lane; r < K; r += 32) s2 += W[(size_t)c * K + r] * W[(size_t)c * K + r];
                s2 = group_sum<32>(s2);
                if (lane == 0) sig[c] = s2;
            }
            __syncthreads();
            ++sweeps;
            for (int round = 0; round < kp - 1; ++round) {
                // uniform trip count per warp: every lane reaches the shuffles
                for (int base = warp * GPW; base < kp / 2; base += groups) {
                    const int pr = base + gsub;
                    int a = 0, b = 0;
                    bool valid = pr < kp / 2;
                    if (valid) {
                        a = tourney(pr, round, kp);
                        b = tourney(kp - 1 - pr, round, kp);
                        if (a > b) { const int tmp = a; a = b; b = tmp; }
                        valid = b < k && sig[a] > tau2 && sig[b] > tau2;
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

    // 4. singular values and descending order
    for (int c = warp; c < k; c += NW) {
        double s = 0.0;
        for (int r = lane; r < K; r += 32) s += W[(size_t)c * K + r] * W[(size_t)c * K + r];
        s = group_sum<32>(s);
        if (lane == 0) sig[c] = sqrt(s);
    }
    __syncthreads();
    for (int c = tid; c < k; c += CT) {
        const double sc = sig[c];
        int pos = 0;
        for (int l = 0; l < k; ++l) {
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
                while (r < k && sig[order[r]] >= p.tol) ++r;
            }
            if (r > p.maxrank) {
                r = p.maxrank;
                if (p.overflow) atomicAdd(p.overflow, 1);
            }
        } else {
            // the truncated trailing mass belongs to the tail of the spectrum
            const double dropped = tail_sh;
            double total = dropped;
            for (int l = 0; l < k; ++l) total += sig[l] * sig[l];
            if (total == 0.0) {
                r = 0;
            } else {
                const double thr = p.tol * p.tol * total;
                double tail = dropped;
                r = k;
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
    // left singular vectors of M in decreasing sigma order: U(piv[q], i) = W(q, order[i]) / sigma;
    // columns past k (zero singular values) are zero
    for (long long idx = tid; idx < (long long)K * K; idx += CT) {
        const int q = (int)(idx % K), i = (int)(idx / K);
        if (i < k) {
            const int c = order[i];
            const double s = sig[c];
            t.SU[(size_t)piv[q] + (size_t)i * K] = s > 0.0 ? W[(size_t)c * K + q] / s : 0.0;
        } else {
            t.SU[idx] = 0.0;
        }
    }
}

// Large cores (K > KMAX_SMEM): the same algorithm on an 8-CTA thread-block
// cluster per core.  T, the partial norms, the reflector and the pivots live
// in the task's global scratch (read through L2 with ld.global.cg, since other
// CTAs of the cluster write them); the steps are separated by hardware cluster
// barriers, and the column work of each step (reflector application, Jacobi
// pairs, output) is spread over the cluster's 64 warps.
constexpr int CL_CS = 8;
constexpr int CL_CT = 256;

__device__ __forceinline__ double ldg2(const double *p) { return __ldcg(p); }
__device__ __forceinline__ int ldg2(const int *p) { return __ldcg(p); }

__global__ void __launch_bounds__(CL_CT) k_core_svd_cl(const CoreTask *__restrict__ tasks, CoreParams p) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    constexpr int NW = CL_CT / 32;
    const int crank = (int)cl.block_rank();
    const CoreTask t = tasks[blockIdx.x / CL_CS];
    const int K = t.K;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gw = crank * NW + warp, GW = CL_CS * NW;
    const long long gt = (long long)crank * CL_CT + tid, GT = (long long)CL_CS * CL_CT;
    if (K <= 0) {
        if (crank == 0 && tid == 0) {
            if (t.rank_out) *t.rank_out = 0;
            if (t.rank_task) *t.rank_task = 0;
        }
        return;
    }
    double *W = t.work;
    double *sig = W + (size_t)K * K;
    double *hv = sig + K;
    int *piv = (int *)(hv + K);
    int *order = piv + K;
    double *misc = (double *)(piv + 2 * K);           // [0] tau2 [1] tail [2] stop [3] tau [4] rotated
    enum { M_TAU2 = 0, M_TAIL, M_STOP, M_TH, M_ROT };

    for (long long idx = gt; idx < (long long)K * K; idx += GT) {
        const int i = (int)(idx % K), c = (int)(idx / K);
        double s = 0.0;
        if (t.RU) {
            const int l0 = i > c ? i : c;
            for (int l = l0; l < K; ++l)
                s += t.RU[(size_t)c + (size_t)l * t.ldru] * t.RV[(size_t)i + (size_t)l * t.ldrv];
            if (t.RUc) t.RUc[idx] = (i <= c) ? t.RU[(size_t)i + (size_t)c * t.ldru] : 0.0;
        } else {
            s = (i <= c) ? t.RV[(size_t)i + (size_t)c * t.ldrv] : 0.0;
        }
        W[idx] = s;
    }
    cl.sync();
    for (int c = gw; c < K; c += GW) {
        double s2 = 0.0;
        for (int r = lane; r < K; r += 32) { const double x = ldg2(W + (size_t)c * K + r); s2 += x * x; }
        s2 = group_sum<32>(s2);
        if (lane == 0) { sig[c] = s2; piv[c] = c; }
    }
    cl.sync();
    if (crank == 0 && tid == 0) {
        double tau = 0.0;
        if (p.mode == 0 && p.fixed_rank <= 0) tau = 1e-3 * p.tol;
        double tau2 = tau * tau;
        if (p.mode == 1) {
            double tot = 0.0;
            for (int c = 0; c < K; ++c) tot += ldg2(sig + c);
            tau2 = 1e-6 * p.tol * p.tol * tot;
        }
        misc[M_TAU2] = tau2;
        misc[M_TAIL] = 0.0;
        misc[M_STOP] = 0.0;
    }
    cl.sync();
    const double tau2 = ldg2(misc + M_TAU2);

    // pivoted Householder QR of T, stopped when the trailing mass <= tau2
    int k = K;
    for (int j = 0; j < K; ++j) {
        if (crank == 0 && warp == 0) {
            double tr = 0.0, best = -1.0;
            int bi = j;
            for (int c = j + lane; c < K; c += 32) {
                const double v = ldg2(sig + c);
                tr += v;
                if (v > best) { best = v; bi = c; }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                tr += __shfl_xor_sync(0xffffffffu, tr, o);
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            const bool stop = !(tr > tau2);
            if (lane == 0) {
                misc[M_STOP] = stop ? 1.0 : 0.0;
                if (stop) misc[M_TAIL] = tr;
            }
            if (!stop) {
                double *cj = W + (size_t)j * K;
                if (bi != j) {
                    double *cb = W + (size_t)bi * K;
                    for (int r = lane; r < K; r += 32) {
                        const double x = ldg2(cj + r);
                        cj[r] = ldg2(cb + r);
                        cb[r] = x;
                    }
                    if (lane == 0) {
                        const double sx = ldg2(sig + j); sig[j] = ldg2(sig + bi); sig[bi] = sx;
                        const int px = ldg2(piv + j); piv[j] = ldg2(piv + bi); piv[bi] = px;
                    }
                    __syncwarp();
                }
                const double alpha = ldg2(cj + j);
                double s2 = 0.0;
                for (int r = j + 1 + lane; r < K; r += 32) { const double x = ldg2(cj + r); s2 += x * x; }
                s2 = group_sum<32>(s2);
                double th = 0.0, scl = 0.0, beta = alpha;
                if (s2 > 0.0) {
                    beta = -copysign(sqrt(alpha * alpha + s2), alpha);
                    th = (beta - alpha) / beta;
                    scl = 1.0 / (alpha - beta);
                }
                for (int r = j + 1 + lane; r < K; r += 32) {
                    hv[r] = ldg2(cj + r) * scl;
                    cj[r] = 0.0;
                }
                if (lane == 0) {
                    hv[j] = 1.0;
                    cj[j] = beta;
                    misc[M_TH] = th;
                }
            }
        }
        cl.sync();
        if (ldg2(misc + M_STOP) != 0.0) { k = j; break; }
        const double th = ldg2(misc + M_TH);
        for (int c = j + 1 + gw; c < K; c += GW) {
            double *col = W + (size_t)c * K;
            double w = 0.0;
            for (int r = j + lane; r < K; r += 32) w += ldg2(hv + r) * ldg2(col + r);
            w = group_sum<32>(w) * th;
            double s2 = 0.0;
            for (int r = j + lane; r < K; r += 32) {
                const double x = ldg2(col + r) - w * ldg2(hv + r);
                col[r] = x;
                if (r > j) s2 += x * x;
            }
            s2 = group_sum<32>(s2);
            if (lane == 0) sig[c] = s2;
        }
        cl.sync();
    }
    // R^T in place for the rows that stay
    for (long long idx = gt; idx < (long long)K * K; idx += GT) {
        const int i = (int)(idx % K), c = (int)(idx / K);
        if (i < c && i < k) {
            const double x = ldg2(W + (size_t)i + (size_t)c * K);
            W[(size_t)i + (size_t)c * K] = ldg2(W + (size_t)c + (size_t)i * K);
            W[(size_t)c + (size_t)i * K] = x;
        }
    }
    cl.sync();

    // one-sided Jacobi on the k columns of R^T, one warp per pair
    const int kp = k + (k & 1);
    const double tolj = 4.4e-16 * (double)(K > 16 ? K : 16);
    int sweeps = 0;
    if (k > 1) {
        for (int sweep = 0; sweep < MAX_SWEEPS; ++sweep) {
            for (int c = gw; c < k; c += GW) {
                double s2 = 0.0;
                for (int r = lane; r < K; r += 32) { const double x = ldg2(W + (size_t)c * K + r); s2 += x * x; }
                s2 = group_sum<32>(s2);
                if (lane == 0) sig[c] = s2;
            }
            if (crank == 0 && tid == 0) misc[M_ROT] = 0.0;
            cl.sync();
            ++sweeps;
            for (int round = 0; round < kp - 1; ++round) {
                for (int pr = gw; pr < kp / 2; pr += GW) {
                    int a = tourney(pr, round, kp), b = tourney(kp - 1 - pr, round, kp);
                    if (a > b) { const int tmp = a; a = b; b = tmp; }
                    if (b >= k) continue;
                    const double sa = ldg2(sig + a), sb = ldg2(sig + b);
                    if (!(sa > tau2 && sb > tau2)) continue;
                    double *mp = W + (size_t)a * K, *mq = W + (size_t)b * K;
                    double aa = 0.0, bb = 0.0, cc = 0.0;
                    for (int r = lane; r < K; r += 32) {
                        const double x = ldg2(mp + r), y = ldg2(mq + r);
                        aa += x * x; bb += y * y; cc += x * y;
                    }
                    aa = group_sum<32>(aa);
                    bb = group_sum<32>(bb);
                    cc = group_sum<32>(cc);
                    if (cc == 0.0 || aa <= tau2 || bb <= tau2 || aa < 1e-290 || bb < 1e-290) continue;
                    if (fabs(cc) <= tolj * sqrt(aa) * sqrt(bb)) continue;
                    const double zeta = (bb - aa) / (2.0 * cc);
                    double tt;
                    if (fabs(zeta) > 1e150) tt = 0.5 / zeta;
                    else tt = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                    const double cs = 1.0 / sqrt(1.0 + tt * tt), sn = cs * tt;
                    for (int r = lane; r < K; r += 32) {
                        const double x = ldg2(mp + r), y = ldg2(mq + r);
                        mp[r] = cs * x - sn * y;
                        mq[r] = sn * x + cs * y;
                    }
                    if (lane == 0) {
                        misc[M_ROT] = 1.0;
                        sig[a] = aa - tt * cc;
                        sig[b] = bb + tt * cc;
                    }
                }
                cl.sync();
            }
            const bool rot = ldg2(misc + M_ROT) != 0.0;
            cl.sync();
            if (!rot) break;
        }
    }
    for (int c = gw; c < k; c += GW) {
        double s = 0.0;
        for (int r = lane; r < K; r += 32) { const double x = ldg2(W + (size_t)c * K + r); s += x * x; }
        s = group_sum<32>(s);
        if (lane == 0) sig[c] = sqrt(s);
    }
    cl.sync();
    for (long long c = gt; c < k; c += GT) {
        const double sc = ldg2(sig + c);
        int pos = 0;
        for (int l = 0; l < k; ++l) {
            const double sl = ldg2(sig + l);
            pos += (sl > sc) || (sl == sc && l < c);
        }
        order[pos] = (int)c;
    }
    cl.sync();
    if (crank == 0 && tid == 0) {
        int r;
        if (p.mode == 0) {
            if (p.fixed_rank > 0) {
                r = p.fixed_rank < K ? p.fixed_rank : K;
            } else {
                r = 0;
                while (r < k && ldg2(sig + ldg2(order + r)) >= p.tol) ++r;
            }
            if (r > p.maxrank) {
                r = p.maxrank;
                if (p.overflow) atomicAdd(p.overflow, 1);
            }
        } else {
            const double dropped = ldg2(misc + M_TAIL);
            double total = dropped;
            for (int l = 0; l < k; ++l) { const double x = ldg2(sig + l); total += x * x; }
            if (total == 0.0) {
                r = 0;
            } else {
                const double thr = p.tol * p.tol * total;
                double tail = dropped;
                r = k;
                while (r > 0) {
                    const double x = ldg2(sig + ldg2(order + r - 1));
                    if (tail + x * x > thr) break;
                    tail += x * x;
                    --r;
                }
            }
            if (!(2 * r < p.nb && r <= p.maxrank)) r = -1;
        }
        if (t.rank_out) *t.rank_out = r;
        if (t.rank_task) *t.rank_task = r;
        if (p.sweeps) atomicAdd(p.sweeps, sweeps);
    }
    for (long long idx = gt; idx < (long long)K * K; idx += GT) {
        const int q = (int)(idx % K), i = (int)(idx / K);
        if (i < k) {
            const int c = ldg2(order + i);
            const double sv = ldg2(sig + c);
            t.SU[(size_t)ldg2(piv + q) + (size_t)i * K] = sv > 0.0 ? ldg2(W + (size_t)c * K + q) / sv : 0.0;
        } else {
            t.SU[idx] = 0.0;
        }
    }
}

template <int LP, int CT>
void launch_lp(const CoreTask *d, int n, size_t smem, const CoreParams &p, cudaStream_t st) {
    cudaFuncSetAttribute(k_core_svd<LP, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_core_svd<LP, CT><<<n, CT, smem, st>>>(d, p);
}

}  // namespace

int core_smem_kmax() { return KMAX_SMEM; }

size_t core_work_doubles(int K) { return (size_t)K * K + 4 * (size_t)K + 16; }

void launch_core_svd_batched(const CoreTask *d_tasks, int ntasks, int kmax, const CoreParams &p,
                             cudaStream_t st) {
    if (ntasks <= 0) return;
    if (kmax < 1) kmax = 1;
    size_t smem;
    // W (K x K, on chip when small), partial norms / sigma, Householder vector,
    // order and pivot
    if (kmax <= KMAX_SMEM)
        smem = sizeof(double) * ((size_t)kmax * kmax + 2 * (size_t)kmax) + 2 * sizeof(int) * kmax;
    else
        smem = 2 * sizeof(double) * (size_t)kmax + 2 * sizeof(int) * kmax;
    smem = (smem + 15) / 16 * 16;
    // lanes per pair ~ K/8 elements each; more pair groups per CTA for large K
    if (kmax <= 64) launch_lp<8, 256>(d_tasks, ntasks, smem, p, st);
    else if (kmax <= 96) launch_lp<16, 256>(d_tasks, ntasks, smem, p, st);
    else if (kmax <= KMAX_SMEM) launch_lp<16, 512>(d_tasks, ntasks, smem, p, st);
    else {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)ntasks * CL_CS);
        cfg.blockDim = dim3(CL_CT);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = CL_CS;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, k_core_svd_cl, d_tasks, p);
    }
}

}  // namespace tlr
