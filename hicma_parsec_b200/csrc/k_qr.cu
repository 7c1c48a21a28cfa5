// Batched tall-skinny Householder QR and application of Q, FP64.
//
// Replaces the QR halves of HCORE_dgemm_qr_svd / HCORE_dgemm_ormqr (call sites
// hicma_parsec/HiCMA_dpotrf_L_2flow.jdf:830-903,985-1058) and the range
// finder QR of starsh_dense_dlrrsdd (STARSH_gen.jdf:162-163).
//
// One CTA per m x K matrix (m = NB up to a few thousand, K = stacked rank).
// Panels of PB columns are factored in shared memory (PB chosen so that an
// m x PB panel fits); each column's norm and the dots against the remaining
// panel columns are one block reduction (warp shuffles, then shared memory).
// The block reflector I - V T V^T of each panel (LAPACK dlarft, forward,
// columnwise) is applied to the trailing columns one warp per column:
// w = V^T x (warp-shuffle reduction), w = T^T w, x -= V w.  The T factors are
// kept so that Q [S; 0] can be formed later without re-deriving them.
#include "tlr_internal.h"

namespace tlr {
namespace {

constexpr int QW_MAX = 16;         // warps of the largest CTA (reduction scratch)

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Element r (panel-relative row) of reflector i of a panel stored in P
// (column-major, mr rows): 0 above, 1 on the diagonal, stored value below.
__device__ __forceinline__ double vref(const double *P, int mr, int i, int r) {
    return r > i ? P[i * mr + r] : (r == i ? 1.0 : 0.0);
}

// w[i] = sum_r v_i(r) y[r] over the panel rows (warp-wide, 4 rows in flight per lane)
template <int PB>
__device__ __forceinline__ void panel_dots(const double *P, int mr, int jb, const double *y, int lane, double (&w)[PB]) {
#pragma unroll
    for (int i = 0; i < PB; ++i) w[i] = 0.0;
    int r = lane;
    for (; r + 96 < mr; r += 128) {
        const double x0 = y[r], x1 = y[r + 32], x2 = y[r + 64], x3 = y[r + 96];
#pragma unroll
        for (int i = 0; i < PB; ++i)
            if (i < jb)
                w[i] += vref(P, mr, i, r) * x0 + vref(P, mr, i, r + 32) * x1 + vref(P, mr, i, r + 64) * x2 +
                        vref(P, mr, i, r + 96) * x3;
    }
    for (; r < mr; r += 32) {
        const double x = y[r];
#pragma unroll
        for (int i = 0; i < PB; ++i)
            if (i < jb) w[i] += vref(P, mr, i, r) * x;
    }
#pragma unroll
    for (int i = 0; i < PB; ++i) w[i] = warp_sum(w[i]);
}

// y[r] -= sum_i v_i(r) w2[i]
template <int PB>
__device__ __forceinline__ void panel_update(const double *P, int mr, int jb, double *y, int lane, const double (&w2)[PB]) {
    int r = lane;
    for (; r + 96 < mr; r += 128) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
        for (int i = 0; i < PB; ++i)
            if (i < jb) {
                a0 += vref(P, mr, i, r) * w2[i];
                a1 += vref(P, mr, i, r + 32) * w2[i];
                a2 += vref(P, mr, i, r + 64) * w2[i];
                a3 += vref(P, mr, i, r + 96) * w2[i];
            }
        y[r] -= a0; y[r + 32] -= a1; y[r + 64] -= a2; y[r + 96] -= a3;
    }
    for (; r < mr; r += 32) {
        double a = 0.0;
#pragma unroll
        for (int i = 0; i < PB; ++i)
            if (i < jb) a += vref(P, mr, i, r) * w2[i];
        y[r] -= a;
    }
}

template <int PB, int QT>
__global__ void __launch_bounds__(QT) k_qr(const QRTask *__restrict__ tasks) {
    constexpr int QW = QT / 32;
    extern __shared__ double sm[];
    const QRTask t = tasks[blockIdx.x];
    const int m = t.m, K = t.K, ld = t.ld;
    if (K <= 0) return;
    double *X = t.X;
    double *P = sm;                       // PB * m
    double *red = P + PB * m;             // QW_MAX * PB
    double *Ts = red + QW_MAX * PB;       // PB * PB
    double *wsm = Ts + PB * PB;           // PB
    double *sc = wsm + PB;                // 4 scalars
    double *G = sc + 4;                   // PB * PB gram of the panel reflectors
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    for (int j0 = 0; j0 < K; j0 += PB) {
        const int jb = min(PB, K - j0);
        const int mr = m - j0;
        for (int idx = tid; idx < jb * mr; idx += QT) {
            const int c = idx / mr, r = idx - c * mr;
            P[c * mr + r] = X[(size_t)(j0 + r) + (size_t)(j0 + c) * ld];
        }
        __syncthreads();

        // Column c: norm of P[c][c+1:] and dots with the later panel columns
        // (reduced across the CTA), reflector from warp 0, then one fused pass
        // that applies H_c to the later columns and accumulates the sums of
        // column c+1 for the next step.
        double s[PB];
#pragma unroll
        for (int i = 0; i < PB; ++i) s[i] = 0.0;
        for (int r = 1 + tid; r < mr; r += QT) {
            const double x = P[r];
            s[0] += x * x;
#pragma unroll
            for (int cc = 1; cc < PB; ++cc)
                if (cc < jb) s[cc] += x * P[cc * mr + r];
        }
        for (int c = 0; c < jb; ++c) {
#pragma unroll
            for (int i = 0; i < PB; ++i) {
                const double v = warp_sum(s[i]);
                if (lane == 0) red[warp * PB + i] = v;
            }
            __syncthreads();
            if (warp == 0) {
                // lane i sums entry i over the warps
                double acc = 0.0;
                if (lane < PB)
                    for (int w = 0; w < QW; ++w) acc += red[w * PB + lane];
                const double norm2 = __shfl_sync(0xffffffffu, acc, 0);
                const double alpha = P[c * mr + c];
                double tau, beta, scale;
                if (norm2 == 0.0) {
                    tau = 0.0; beta = alpha; scale = 0.0;
                } else {
                    beta = -copysign(sqrt(alpha * alpha + norm2), alpha);
                    tau = (beta - alpha) / beta;
                    scale = 1.0 / (alpha - beta);
                }
                if (lane > c && lane < jb) wsm[lane] = P[lane * mr + c] + scale * acc;
                if (lane == 0) {
                    sc[0] = tau; sc[1] = beta; sc[2] = scale;
                    t.tau[j0 + c] = tau;
                }
            }
            __syncthreads();
            const double tau = sc[0], beta = sc[1], scale = sc[2];
            const int c1 = c + 1;
#pragma unroll
            for (int i = 0; i < PB; ++i) s[i] = 0.0;
            for (int r = c + tid; r < mr; r += QT) {
                double v;
                if (r == c) { v = 1.0; P[c * mr + c] = beta; }
                else        { v = P[c * mr + r] * scale; P[c * mr + r] = v; }
                const double tv = tau * v;
                double xn = 0.0;
#pragma unroll
                for (int cc = 1; cc < PB; ++cc) {
                    if (cc > c && cc < jb) {
                        const double y = P[cc * mr + r] - tv * wsm[cc];
                        P[cc * mr + r] = y;
                        if (cc == c1) xn = y;
                        else if (cc > c1 && r > c1) s[cc] += xn * y;
                    }
                }
                if (r > c1 && c1 < jb) s[0] += xn * xn;
            }
        }
        __syncthreads();

        // Gram of the panel reflectors: G[l][i] = v_l . v_i for l < i.
        const int npairs = jb * (jb - 1) / 2;
        for (int pidx = warp; pidx < npairs; pidx += QW) {
            int i = 1, acc = 0;
            while (acc + i <= pidx) { acc += i; ++i; }
            const int l = pidx - acc;     // 0 <= l < i
            double s = 0.0;
            for (int r = i + 1 + lane; r < mr; r += 32) s += P[l * mr + r] * P[i * mr + r];
            s = warp_sum(s);
            if (lane == 0) G[l + i * PB] = s + P[l * mr + i];
        }
        __syncthreads();
        if (tid == 0) {
            // T (upper): T[i][i] = tau_i, T[0:i, i] = -tau_i T[0:i,0:i] G[0:i, i]
            for (int i = 0; i < jb; ++i) {
                const double ti = t.tau[j0 + i];
                for (int l = 0; l < i; ++l) {
                    double z = 0.0;
                    for (int q = l; q < i; ++q) z += Ts[l + q * PB] * G[q + i * PB];
                    Ts[l + i * PB] = -ti * z;
                }
                Ts[i + i * PB] = ti;
                for (int l = i + 1; l < PB; ++l) Ts[l + i * PB] = 0.0;
            }
            for (int i = jb; i < PB; ++i)
                for (int l = 0; l < PB; ++l) Ts[l + i * PB] = 0.0;
        }
        __syncthreads();
        double *Tg = t.T + (size_t)(j0 / PB) * PB * PB;
        for (int idx = tid; idx < PB * PB; idx += QT) Tg[idx] = Ts[idx];
        for (int idx = tid; idx < jb * mr; idx += QT) {
            const int c = idx / mr, r = idx - c * mr;
            X[(size_t)(j0 + r) + (size_t)(j0 + c) * ld] = P[c * mr + r];
        }

        // trailing update: x <- x - V T^T V^T x, one warp per column
        for (int col = j0 + jb + warp; col < K; col += QW) {
            double *xcol = X + (size_t)col * ld + j0;
            double w[PB];
            panel_dots<PB>(P, mr, jb, xcol, lane, w);
            double w2[PB];
#pragma unroll
            for (int i = 0; i < PB; ++i) {
                double z = 0.0;
#pragma unroll
                for (int l = 0; l < PB; ++l)
                    if (l <= i) z += Ts[l + i * PB] * w[l];
                w2[i] = z;
            }
            panel_update<PB>(P, mr, jb, xcol, lane, w2);
        }
        __syncthreads();
    }
}

template <int PB, int QT>
__global__ void __launch_bounds__(QT) k_qapply(const QApplyTask *__restrict__ tasks) {
    constexpr int QW = QT / 32;
    extern __shared__ double sm[];
    const QApplyTask t = tasks[blockIdx.x];
    int r = t.r_dev ? *t.r_dev : t.r_cap;
    if (r > t.r_cap) r = t.r_cap;
    if (r <= 0) return;
    const int m = t.m, K = t.K;
    double *P = sm;
    double *Ts = P + PB * m;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (long long idx = tid; idx < (long long)m * r; idx += QT) {
        const int c = (int)(idx / m), row = (int)(idx - (long long)c * m);
        t.out[(size_t)row + (size_t)c * t.ldo] = row < K ? t.S[(size_t)row + (size_t)c * t.lds] : 0.0;
    }
    __syncthreads();
    const int npan = (K + PB - 1) / PB;
    for (int p = npan - 1; p >= 0; --p) {
        const int j0 = p * PB;
        const int jb = min(PB, K - j0);
        const int mr = m - j0;
        for (int idx = tid; idx < jb * mr; idx += QT) {
            const int c = idx / mr, rr = idx - c * mr;
            P[c * mr + rr] = t.X[(size_t)(j0 + rr) + (size_t)(j0 + c) * t.ld];
        }
        for (int idx = tid; idx < PB * PB; idx += QT) Ts[idx] = t.T[(size_t)p * PB * PB + idx];
        __syncthreads();
        for (int col = warp; col < r; col += QW) {
            double *y = t.out + (size_t)col * t.ldo + j0;
            double w[PB];
            panel_dots<PB>(P, mr, jb, y, lane, w);
            double w2[PB];
#pragma unroll
            for (int i = 0; i < PB; ++i) {
                double z = 0.0;
#pragma unroll
                for (int l = 0; l < PB; ++l)
                    if (l >= i) z += Ts[i + l * PB] * w[l];
                w2[i] = z;
            }
            panel_update<PB>(P, mr, jb, y, lane, w2);
        }
        __syncthreads();
    }
}

template <int PB>
size_t qr_smem(int m) { return sizeof(double) * ((size_t)PB * m + QW_MAX * PB + 2 * PB * PB + PB + 4); }

// 512 threads where the register budget allows it (PB <= 16), else 256
template <int PB>
constexpr int qr_threads() { return PB <= 16 ? 512 : 256; }

template <int PB>
void launch_qr_pb(const QRTask *d_tasks, int ntasks, int m_max, cudaStream_t st) {
    const size_t smem = qr_smem<PB>(m_max);
    constexpr int T = qr_threads<PB>();
    cudaFuncSetAttribute(k_qr<PB, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_qr<PB, T><<<ntasks, T, smem, st>>>(d_tasks);
}

template <int PB>
void launch_qapply_pb(const QApplyTask *d_tasks, int ntasks, int m_max, cudaStream_t st) {
    const size_t smem = sizeof(double) * ((size_t)PB * m_max + PB * PB);
    constexpr int T = qr_threads<PB>();
    cudaFuncSetAttribute(k_qapply<PB, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_qapply<PB, T><<<ntasks, T, smem, st>>>(d_tasks);
}

}  // namespace

int qr_panel_width(int m) {
    const long long budget = 200 * 1024;
    const long long pb = budget / ((long long)m * 8 + 1);
    if (pb >= 32) return 32;
    if (pb >= 16) return 16;
    if (pb >= 8) return 8;
    if (pb >= 4) return 4;
    return 2;
}

size_t qr_smem_bytes(int m) {
    switch (qr_panel_width(m)) {
        case 32: return qr_smem<32>(m);
        case 16: return qr_smem<16>(m);
        case 8: return qr_smem<8>(m);
        case 4: return qr_smem<4>(m);
        default: return qr_smem<2>(m);
    }
}

void launch_qr_batched(const QRTask *d_tasks, int ntasks, int m_max, cudaStream_t st) {
    if (ntasks <= 0) return;
    switch (qr_panel_width(m_max)) {
        case 32: launch_qr_pb<32>(d_tasks, ntasks, m_max, st); break;
        case 16: launch_qr_pb<16>(d_tasks, ntasks, m_max, st); break;
        case 8: launch_qr_pb<8>(d_tasks, ntasks, m_max, st); break;
        case 4: launch_qr_pb<4>(d_tasks, ntasks, m_max, st); break;
        default: launch_qr_pb<2>(d_tasks, ntasks, m_max, st); break;
    }
}

void launch_qapply_batched(const QApplyTask *d_tasks, int ntasks, int m_max, cudaStream_t st) {
    if (ntasks <= 0) return;
    switch (qr_panel_width(m_max)) {
        case 32: launch_qapply_pb<32>(d_tasks, ntasks, m_max, st); break;
        case 16: launch_qapply_pb<16>(d_tasks, ntasks, m_max, st); break;
        case 8: launch_qapply_pb<8>(d_tasks, ntasks, m_max, st); break;
        case 4: launch_qapply_pb<4>(d_tasks, ntasks, m_max, st); break;
        default: launch_qapply_pb<2>(d_tasks, ntasks, m_max, st); break;
    }
}

}  // namespace tlr
