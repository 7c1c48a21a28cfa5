// Tile Cholesky and tile inverse in one persistent launch.
//
// Replaces HCORE_dpotrf on a diagonal tile (hicma_parsec/HiCMA_dpotrf_L_2flow.jdf
// :233-242) together with the inverse L^-1 that the panel solves of this
// engine apply as a GEMM.  The tile is split into 64 x 64 blocks and the
// blocked right-looking algorithm becomes a list of block tasks:
//   DIAG(j)      Cholesky of A_jj and D_j = L_jj^-1 (one CTA, shared memory,
//                8-column panels factored by one warp)
//   PANEL(j,i)   L_ij = A_ij D_j^T
//   UPD(j,i,k)   A_ik -= L_ij L_kj^T                       (j < k <= i)
//   XDIAG(j,k)   X_jk = D_j B_jk                           (k < j)
//   XUPD(j,i,k)  B_ik -= L_ij X_jk                         (k <= j < i)
// where X = L^-1 is produced by block forward substitution on the identity
// (B starts as zero off the diagonal).  The list is in a topological order
// and CTAs take tasks from it with an atomic ticket, so every task waits only
// on tasks already held by running CTAs: the kernel makes progress with any
// number of resident CTAs and needs no cooperative launch.  Dependencies are
// per-block counters released with a fence after the block is written and
// acquired by one thread before the CTA reads (through L2: ld.global.cg).
// Every wait is bounded; a wait that gives up sets the timeout flag and the
// abort flag, and every CTA leaves at its next task.  A non-positive pivot
// sets the reference's INFO (k*NB + iinfo) and aborts the same way.
// The 64 x 64 products run on the FP64 tensor cores (mma.sync m8n8k4 f64).
#include "tlr_internal.h"

#include <map>
#include <mutex>
#include <vector>

namespace tlr {
namespace {

constexpr int TB = 64;          // block edge
constexpr int TPITCH = 72;      // shared pitch of DMMA operand tiles
constexpr int LDS = TB + 1;     // shared pitch of the diagonal block
constexpr int NTH = 256;
constexpr long long SPIN_LIMIT = 1LL << 24;

enum { IT_DIAG = 0, IT_PANEL, IT_UPD, IT_XDIAG, IT_XUPD };
struct PItem {
    unsigned short type, j, i, k;
};

struct PotrfParams {
    double *A;
    int lda, n, nblk;
    double *X;          // L^-1 (zeroed), or null
    int ldx;
    double *D;          // nblk x (64 x 64) block inverses when X is null
    const PItem *items;
    int nitems;
    int *cnt;           // [0] ticket [1] abort, then ver, pdone, xver, xdone (nblk^2 each), ddone (nblk)
    int *info;
    int info_base;
    int *timeout;
    long long spin_limit;   // polls before a wait gives up (SPIN_LIMIT in production)
};

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ int ld_volatile(const int *p) { return *(const volatile int *)p; }

// thread 0 only: wait until *p >= v
__device__ bool wait_ge(const int *p, int v, const PotrfParams &P) {
    for (long long it = 0; it < P.spin_limit; ++it) {
        if (ld_volatile(p) >= v) {
            __threadfence();
            return true;
        }
        if (ld_volatile(P.cnt + 1)) return false;
        __nanosleep(it < 256 ? 32 : 256);
    }
    atomicExch(P.timeout, 1);
    atomicExch(P.cnt + 1, 1);
    return false;
}

__device__ __forceinline__ int bsz(int b, int n) { return min(TB, n - b * TB); }

// C (m x nn, ldc) = beta C + alpha opA(A) opB(B), inner dimension kk <= 64.
// Operands are staged in shared memory before C is written, so C may alias
// A or B when beta = 0.
__device__ void blk_gemm(double *sm, double *C, int ldc, int m, int nn, int kk, double alpha, double beta,
                         const double *A, int lda, int opA, const double *B, int ldb, int opB) {
    double *As = sm;                 // As[k][i]
    double *Bs = sm + TB * TPITCH;   // Bs[k][j]
    const int tid = threadIdx.x;
#pragma unroll 4
    for (int q = 0; q < (TB * TB) / NTH; ++q) {
        const int e = tid + q * NTH;
        int i, k;
        if (opA == 0) { i = e & (TB - 1); k = e >> 6; } else { k = e & (TB - 1); i = e >> 6; }
        double v = 0.0;
        if (i < m && k < kk) v = __ldcg(opA == 0 ? A + i + (size_t)k * lda : A + k + (size_t)i * lda);
        As[k * TPITCH + i] = v;
        int j;
        if (opB == 0) { k = e & (TB - 1); j = e >> 6; } else { j = e & (TB - 1); k = e >> 6; }
        double w = 0.0;
        if (j < nn && k < kk) w = __ldcg(opB == 0 ? B + k + (size_t)j * ldb : B + j + (size_t)k * ldb);
        Bs[k * TPITCH + j] = w;
    }
    __syncthreads();
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int wm = warp & 1, wn = warp >> 1;   // 2 x 4 warps, 32 x 16 each
    double acc[4][2][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    const int k4end = (kk + 3) & ~3;
    for (int k4 = 0; k4 < k4end; k4 += 4) {
        double a[4], b[2];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) a[mi] = As[(k4 + tig) * TPITCH + wm * 32 + mi * 8 + g];
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) b[ni] = Bs[(k4 + tig) * TPITCH + wn * 16 + ni * 8 + g];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 2; ++ni) dmma884(acc[mi][ni], a[mi], b[ni]);
    }
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
        const int row = wm * 32 + mi * 8 + g;
        if (row >= m) continue;
#pragma unroll
        for (int ni = 0; ni < 2; ++ni)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int col = wn * 16 + ni * 8 + 2 * tig + e;
                if (col >= nn) continue;
                double *cp = C + row + (size_t)col * ldc;
                double v = alpha * acc[mi][ni][e];
                if (beta != 0.0) v += beta * __ldcg(cp);
                *cp = v;
            }
    }
}

// Cholesky of the jb x jb block at Ajj (lda) and its inverse, written to Ajj
// (lower, zero upper) and Dj (ldd).  Returns false on a non-positive pivot.
__device__ bool diag_block(double *sm, double *Ajj, int lda, int jb, double *Dj, int ldd, int *info, int info_col0) {
    double *S = sm;                  // S[c * LDS + r] = L(r, c)
    double *Xs = sm + TB * LDS;      // inverse
    double *Ts = sm + 2 * TB * LDS;  // 32 x 32 scratch
    double *invd = Ts + 32 * 32;
    __shared__ int fail;
    const int tid = threadIdx.x;
    if (tid == 0) fail = 0;
    for (int idx = tid; idx < TB * LDS; idx += NTH) Xs[idx] = 0.0;
    for (int idx = tid; idx < jb * jb; idx += NTH) {
        const int c = idx / jb, r = idx - c * jb;
        S[c * LDS + r] = __ldcg(Ajj + r + (size_t)c * lda);
    }
    __syncthreads();
    // blocked right-looking Cholesky: warp 0 factors each 8-column panel with
    // warp-level synchronisation only, then all threads apply the panel's
    // rank-8 update to the trailing block (two CTA barriers per panel)
    for (int p0 = 0; p0 < jb; p0 += 8) {
        const int pe = min(jb, p0 + 8);
        if (tid < 32) {
            const int lane = tid;
            for (int c = p0; c < pe; ++c) {
                const double d = S[c * LDS + c];
                if (!(d > 0.0)) {
                    if (lane == 0) {
                        fail = 1;
                        if (info) atomicCAS(info, 0, info_col0 + c + 1);
                    }
                    break;
                }
                const double piv = sqrt(d), inv = 1.0 / piv;
                __syncwarp();
                if (lane == 0) { S[c * LDS + c] = piv; invd[c] = inv; }
                for (int r = c + 1 + lane; r < jb; r += 32) S[c * LDS + r] *= inv;
                __syncwarp();
                for (int cc = c + 1; cc < pe; ++cc) {
                    const double lc = S[c * LDS + cc];
                    for (int r = cc + lane; r < jb; r += 32) S[cc * LDS + r] -= S[c * LDS + r] * lc;
                }
                __syncwarp();
            }
        }
        __syncthreads();
        if (fail) return false;
        const int w = jb - pe;
        for (int idx = tid; idx < w * w; idx += NTH) {
            const int cc = pe + idx / w, r = pe + idx % w;
            if (r < cc) continue;
            double acc = S[cc * LDS + r];
            for (int l = p0; l < pe; ++l) acc -= S[l * LDS + r] * S[l * LDS + cc];
            S[cc * LDS + r] = acc;
        }
        __syncthreads();
    }
    // (the last column has nothing below its diagonal)
    // inverse: 8 x 8 diagonal blocks by forward substitution, then pairs of
    // blocks merged with X21 = -X22 (L21 X11) at widths 8, 16, 32
    {
        const int c = tid;
        if (c < jb) {
            const int e = min(jb, (c / 8) * 8 + 8);
            Xs[c * LDS + c] = invd[c];
            for (int r = c + 1; r < e; ++r) {
                double s = 0.0;
                for (int l = c; l < r; ++l) s += S[l * LDS + r] * Xs[c * LDS + l];
                Xs[c * LDS + r] = -s * invd[r];
            }
        }
    }
    __syncthreads();
    for (int h = 8; h < TB; h *= 2) {
        const int npair = (jb + 2 * h - 1) / (2 * h);
        // T = L21 X11 (rows s0+h .. e, cols s0 .. s0+h)
        for (int idx = tid; idx < npair * h * h; idx += NTH) {
            const int pr = idx / (h * h), rem = idx % (h * h);
            const int rr = rem % h, cc = rem / h;
            const int s0 = pr * 2 * h, r = s0 + h + rr, c = s0 + cc;
            if (r >= jb) continue;
            double s = 0.0;
            for (int l = c; l < s0 + h; ++l) s += S[l * LDS + r] * Xs[c * LDS + l];
            Ts[pr * h * h + cc * h + rr] = s;
        }
        __syncthreads();
        // X21 = -X22 T
        for (int idx = tid; idx < npair * h * h; idx += NTH) {
            const int pr = idx / (h * h), rem = idx % (h * h);
            const int rr = rem % h, cc = rem / h;
            const int s0 = pr * 2 * h, r = s0 + h + rr, c = s0 + cc;
            if (r >= jb) continue;
            double s = 0.0;
            for (int m = s0 + h; m <= r; ++m) s += Xs[m * LDS + r] * Ts[pr * h * h + cc * h + (m - s0 - h)];
            Xs[c * LDS + r] = -s;
        }
        __syncthreads();
    }
    for (int idx = tid; idx < jb * jb; idx += NTH) {
        const int c = idx / jb, r = idx - c * jb;
        Ajj[r + (size_t)c * lda] = (r >= c) ? S[c * LDS + r] : 0.0;
        Dj[r + (size_t)c * ldd] = (r >= c) ? Xs[c * LDS + r] : 0.0;
    }
    return true;
}

__global__ void __launch_bounds__(NTH, 2) k_potrf_tile(PotrfParams P) {
    extern __shared__ double sm[];
    __shared__ int item_sh, ok_sh;
    const int tid = threadIdx.x;
    const int nb2 = P.nblk * P.nblk;
    int *ver = P.cnt + 8, *pdone = ver + nb2, *xver = pdone + nb2, *xdone = xver + nb2, *ddone = xdone + nb2;
    for (;;) {
        if (tid == 0) {
            int t = -1;
            if (!ld_volatile(P.cnt + 1)) {
                t = atomicAdd(P.cnt, 1);
                if (t >= P.nitems) t = -1;
            }
            item_sh = t;
        }
        __syncthreads();
        const int t = item_sh;
        if (t < 0) break;
        const PItem it = P.items[t];
        const int j = it.j, i = it.i, k = it.k, n = P.n, nb = P.nblk;
        if (tid == 0) {
            bool ok = true;
            switch (it.type) {
                case IT_DIAG: ok = wait_ge(ver + j * nb + j, j, P); break;
                case IT_PANEL: ok = wait_ge(ddone + j, 1, P) && wait_ge(ver + i * nb + j, j, P); break;
                case IT_UPD:
                    ok = wait_ge(pdone + i * nb + j, 1, P) && wait_ge(pdone + k * nb + j, 1, P) &&
                         wait_ge(ver + i * nb + k, j, P);
                    break;
                case IT_XDIAG: ok = wait_ge(ddone + j, 1, P) && wait_ge(xver + j * nb + k, j - k, P); break;
                default:
                    ok = wait_ge(pdone + i * nb + j, 1, P) &&
                         (k == j ? wait_ge(ddone + j, 1, P) : wait_ge(xdone + j * nb + k, 1, P)) &&
                         wait_ge(xver + i * nb + k, j - k, P);
                    break;
            }
            ok_sh = ok;
        }
        __syncthreads();
        if (!ok_sh) break;
        const int lda = P.lda;
        auto Ablk = [&](int r, int c) { return P.A + (size_t)r * TB + (size_t)c * TB * lda; };
        auto Xblk = [&](int r, int c) { return P.X + (size_t)r * TB + (size_t)c * TB * P.ldx; };
        double *Dj = P.X ? Xblk(j, j) : P.D + (size_t)j * TB * TB;
        const int ldd = P.X ? P.ldx : TB;
        bool good = true;
        switch (it.type) {
            case IT_DIAG:
                good = diag_block(sm, Ablk(j, j), lda, bsz(j, n), Dj, ldd, P.info, P.info_base + j * TB);
                break;
            case IT_PANEL:
                blk_gemm(sm, Ablk(i, j), lda, bsz(i, n), bsz(j, n), bsz(j, n), 1.0, 0.0, Ablk(i, j), lda, 0, Dj, ldd, 1);
                break;
            case IT_UPD:
                blk_gemm(sm, Ablk(i, k), lda, bsz(i, n), bsz(k, n), bsz(j, n), -1.0, 1.0, Ablk(i, j), lda, 0,
                         Ablk(k, j), lda, 1);
                break;
            case IT_XDIAG:
                blk_gemm(sm, Xblk(j, k), P.ldx, bsz(j, n), bsz(k, n), bsz(j, n), 1.0, 0.0, Dj, ldd, 0, Xblk(j, k),
                         P.ldx, 0);
                break;
            default:
                blk_gemm(sm, Xblk(i, k), P.ldx, bsz(i, n), bsz(k, n), bsz(j, n), -1.0, 1.0, Ablk(i, j), lda, 0,
                         Xblk(j, k), P.ldx, 0);
                break;
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            if (!good) {
                atomicExch(P.cnt + 1, 1);
            } else {
                switch (it.type) {
                    case IT_DIAG: atomicExch(ddone + j, 1); break;
                    case IT_PANEL: atomicExch(pdone + i * nb + j, 1); break;
                    case IT_UPD: atomicExch(ver + i * nb + k, j + 1); break;
                    case IT_XDIAG: atomicExch(xdone + j * nb + k, 1); break;
                    default: atomicExch(xver + i * nb + k, j - k + 1); break;
                }
            }
        }
    }
}

std::vector<PItem> build_items(int nblk, bool inv) {
    std::vector<PItem> v;
    auto add = [&](int t, int j, int i, int k) {
        v.push_back(PItem{(unsigned short)t, (unsigned short)j, (unsigned short)i, (unsigned short)k});
    };
    add(IT_DIAG, 0, 0, 0);
    for (int j = 0; j < nblk; ++j) {
        for (int i = j + 1; i < nblk; ++i) add(IT_PANEL, j, i, 0);
        if (j + 1 < nblk) {
            add(IT_UPD, j, j + 1, j + 1);
            add(IT_DIAG, j + 1, 0, 0);
            for (int i = j + 2; i < nblk; ++i) add(IT_UPD, j, i, j + 1);
            for (int k = j + 2; k < nblk; ++k)
                for (int i = k; i < nblk; ++i) add(IT_UPD, j, i, k);
        }
        if (inv) {
            for (int k = 0; k < j; ++k) add(IT_XDIAG, j, 0, k);
            for (int i = j + 1; i < nblk; ++i)
                for (int k = 0; k <= j; ++k) add(IT_XUPD, j, i, k);
        }
    }
    return v;
}

struct ItemList {
    PItem *d = nullptr;
    int n = 0;
};
std::mutex g_items_mu;
std::map<std::pair<int, long long>, ItemList> g_items;   // (device, nblk*2 + inv)

const ItemList *get_items(int nblk, bool inv, cudaStream_t st) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_items_mu);
    auto key = std::make_pair(dev, (long long)nblk * 2 + (inv ? 1 : 0));
    auto f = g_items.find(key);
    if (f != g_items.end()) return &f->second;
    std::vector<PItem> h = build_items(nblk, inv);
    ItemList L;
    if (cudaMalloc(&L.d, h.size() * sizeof(PItem)) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    // ordered on the launch stream and complete before the list is used (a
    // legacy-stream copy from pageable memory may land after the kernel reads it)
    if (cudaMemcpyAsync(L.d, h.data(), h.size() * sizeof(PItem), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaFree(L.d);
        return nullptr;
    }
    L.n = (int)h.size();
    return &(g_items[key] = L);
}

// Exercise of the bounded wait above, for tests: thread 0 of CTA b waits
// with wait_ge on the counter cnt[2 + b], which nothing sets, with limit
// limit0 (CTA 0) or limit1 (the others).  The first wait to run out sets the
// timeout and abort flags; the others then leave at their next poll.
__global__ void k_wait_probe(PotrfParams P, long long limit0, long long limit1) {
    if (threadIdx.x != 0) return;
    P.spin_limit = blockIdx.x == 0 ? limit0 : limit1;
    wait_ge(P.cnt + 2 + blockIdx.x, 1, P);
}

}  // namespace

int potrf_tile_max_n() { return 128 * TB; }

size_t potrf_tile_scratch_ints(int n) {
    const size_t nb = (size_t)(n + TB - 1) / TB;
    return 8 + 4 * nb * nb + nb;
}

// The caller provides cnt (potrf_tile_scratch_ints(n) ints, any content) and,
// when X is null, D (nblk * 64 * 64 doubles); X, when given, must be zeroed.
int launch_potrf_tile(double *A, int lda, int n, double *X, int ldx, double *D, int *cnt, int *info,
                      int info_base, int *timeout, int grid, cudaStream_t st) {
    const int nblk = (n + TB - 1) / TB;
    const ItemList *L = get_items(nblk, X != nullptr, st);
    if (!L) return -1;
    if (cudaMemsetAsync(cnt, 0, potrf_tile_scratch_ints(n) * sizeof(int), st) != cudaSuccess) return -1;
    const int smem = (int)sizeof(double) * (2 * TB * TPITCH > 2 * TB * LDS + 32 * 32 + TB ? 2 * TB * TPITCH
                                                                                        : 2 * TB * LDS + 32 * 32 + TB);
    // per device and thread-safe: set on every launch (a host-side call, no synchronisation)
    cudaFuncSetAttribute(k_potrf_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    PotrfParams P{A, lda, n, nblk, X, ldx, D, L->d, L->n, cnt, info, info_base, timeout, SPIN_LIMIT};
    if (grid > L->n) grid = L->n;
    if (grid < 1) grid = 1;
    k_potrf_tile<<<grid, NTH, smem, st>>>(P);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// cnt: 2 + nblocks zeroed ints (abort flag at [1]); timeout: one zeroed int.
int launch_wait_probe(int *cnt, int *timeout, int nblocks, long long limit0, long long limit1, cudaStream_t st) {
    if (nblocks < 1 || nblocks > 64 || limit0 < 1 || limit1 < 1) return -1;
    PotrfParams P{};
    P.cnt = cnt;
    P.timeout = timeout;
    k_wait_probe<<<nblocks, 32, 0, st>>>(P, limit0, limit1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace tlr
