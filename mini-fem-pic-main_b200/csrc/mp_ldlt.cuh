// Dense symmetric factorization J = L D L^T of the Newton Jacobian and the
// solve J y = G, replacing the reference's LAPACK dsysv_ call
// (FESolver::solveLinearLapack, src/FESolver.cpp:528-558).
//
// Blocked right-looking LDL^T without pivoting on the lower triangle (row-major
// storage, leading dimension padded to 32).  Per block column k of width NB:
//   diag   : L_kk D_k L_kk^T = A_kk in shared memory (one CTA); z_k = L_kk^-1 b_k
//   panel  : W_ik = A_ik L_kk^-T,  L_ik = W_ik D_k^-1, b_i -= L_ik z_k  (rows below)
//   update : A_ij -= L_ik W_jk^T on the lower tiles of the trailing matrix
// The forward substitution rides on the panel pass; the backward substitution
// L^T y = D^-1 z runs block column by block column afterwards.
//
// J is symmetric (K is assembled symmetric, FP only touches the diagonal) and
// in these problems sign-definite, the case where LDL^T needs no pivoting.  A
// zero or non-finite pivot sets FLAG_SINGULAR and the call returns
// MP_ERR_SINGULAR; the solve's residual ||G - J y|| is reported either way.
//
// The FP32 instantiation is the factorization of the mixed form; its solve is
// wrapped in FP64 iterative refinement (residual from the FP64 K and FP).
#include <cmath>

#include "mp_internal.h"
#include "mp_tc.cuh"

namespace mp {

constexpr int NB = 64;

template <typename T>
__device__ __forceinline__ bool bad_pivot(T d) {
    return !(fabs((double)d) > 0.0) || !isfinite((double)d);
}

// Factor the kb x kb diagonal block at (k0,k0) in shared memory: L (strict
// lower) and D written back, and Linv = L_kk^-1 (unit lower, row-major, leading
// dimension NB) for the panel, built during the elimination by applying each
// step's row operations to an identity.  If b is non-null, z_k = L_kk^-1 b_k
// (the forward substitution riding on the factorization).  256 threads; the
// only serial dimension is the kb elimination steps, two barriers each.
// Dynamic smem: s, si [NB][NB+1], sl [2][NB], sb [NB].
template <typename T>
__global__ void __launch_bounds__(256) k_ldlt_diag(int n, long long ld, T *A, int k0, int kb, T *dvec, T *Linv,
                                                   T *b, unsigned long long *flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T(*s)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(smem_raw);
    T(*si)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(smem_raw + sizeof(T) * NB * (NB + 1));
    T *slbuf = reinterpret_cast<T *>(smem_raw + sizeof(T) * 2 * NB * (NB + 1));  // [2][NB]
    T *sb = slbuf + 2 * NB;
    const int t = threadIdx.x;
    {
        T v[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
            int idx = q * 256 + t;
            int r = idx >> 6, c = idx & 63;
            v[q] = (r < kb && c <= r) ? A[(long long)(k0 + r) * ld + k0 + c] : T(0);
        }
#pragma unroll
        for (int q = 0; q < 16; q++) {
            int idx = q * 256 + t;
            int r = idx >> 6, c = idx & 63;
            s[r][c] = v[q];
            si[r][c] = r == c ? T(1) : T(0);
        }
    }
    if (b && t < kb) sb[t] = b[k0 + t];
    __syncthreads();
    for (int j = 0; j < kb; j++) {
        T *sl = slbuf + (j & 1) * NB;
        T d = s[j][j];
        if (bad_pivot(d)) {
            if (t == 0) atomicOr(flags, FLAG_SINGULAR);
            d = T(1);
        }
        const int m = kb - j - 1;
        if (t < m) sl[j + 1 + t] = s[j + 1 + t][j] / d;
        __syncthreads();
        // trailing rank-1 update with the unscaled column w_l = s[l][j]: thread
        // (column l, row phase) walks rows i >= l of its phase
        {
            const int l = j + 1 + (t & 63), ph = t >> 6;
            if (l < kb) {
                const T wl = s[l][j];
                for (int i = l + ((j + 1 + ph - l) & 3); i < kb; i += 4) s[i][l] -= sl[i] * wl;
            }
            // the same row operation on the identity: row_i -= l_ij row_j (columns <= j)
            const int c = t & 63;
            if (c <= j) {
                const T rj = si[j][c];
                for (int i = j + 1 + ph; i < kb; i += 4) si[i][c] -= sl[i] * rj;
            }
        }
        __syncthreads();
        if (t < m) s[j + 1 + t][j] = sl[j + 1 + t];
    }
    __syncthreads();
    {
#pragma unroll
        for (int q = 0; q < 16; q++) {
            int idx = q * 256 + t;
            int r = idx >> 6, c = idx & 63;
            if (r < kb && c < kb) {
                if (c <= r) A[(long long)(k0 + r) * ld + k0 + c] = s[r][c];
                Linv[r * NB + c] = si[r][c];
            }
        }
    }
    if (t < kb) {
        dvec[k0 + t] = s[t][t];
        if (b) {
            T z = 0;
            for (int pp = 0; pp <= t; pp++) z += si[t][pp] * sb[pp];
            b[k0 + t] = z;
        }
    }
}

// Panel: rows [r0, r0+64) below the diagonal block.  W = A_ik L_kk^-T (a small
// product with Linv), L_ik = W D^-1, and b_i -= L_ik z_k.  Dynamic smem: the
// rows' panel [64][NB+1] and Linv [NB][NB+1].
template <typename T>
__global__ void __launch_bounds__(256) k_ldlt_panel(int n, long long ld, T *A, int k0, int kb, const T *dvec,
                                                    const T *Linv, T *W, int ldw, T *b) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T(*sA)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(smem_raw);
    T(*sI)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(smem_raw + sizeof(T) * 64 * (NB + 1));
    T *sd = reinterpret_cast<T *>(smem_raw + sizeof(T) * 2 * 64 * (NB + 1));
    T *sz = sd + NB;
    const int r0 = k0 + kb + blockIdx.x * 64;
    {
        T va[16], vi[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
            int idx = q * 256 + threadIdx.x;
            int r = idx >> 6, c = idx & 63;
            int row = r0 + r;
            va[q] = (row < n && c < kb) ? A[(long long)row * ld + k0 + c] : T(0);
            vi[q] = (r < kb && c < kb) ? __ldg(&Linv[r * NB + c]) : T(0);
        }
#pragma unroll
        for (int q = 0; q < 16; q++) {
            int idx = q * 256 + threadIdx.x;
            sA[idx >> 6][idx & 63] = va[q];
            sI[idx >> 6][idx & 63] = vi[q];
        }
    }
    if (threadIdx.x < kb) {
        sd[threadIdx.x] = dvec[k0 + threadIdx.x];
        if (b) sz[threadIdx.x] = b[k0 + threadIdx.x];
    }
    __syncthreads();
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // 4 rows x 4 cols each
    T acc[4][4] = {};
    for (int pp = 0; pp < kb; pp++) {
        T a[4], w[4];
#pragma unroll
        for (int u = 0; u < 4; u++) a[u] = sA[ty * 4 + u][pp];
#pragma unroll
        for (int v = 0; v < 4; v++) {
            int c = tx * 4 + v;
            w[v] = (c < kb && pp <= c) ? sI[c][pp] : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int v = 0; v < 4; v++) acc[u][v] = fma(a[u], w[v], acc[u][v]);
    }
    T bsum[4] = {0, 0, 0, 0};
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int row = r0 + ty * 4 + u;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int c = tx * 4 + v;
            if (row < n && c < kb) {
                const T wv = acc[u][v];
                const T lv = wv / sd[c];
                W[(long long)row * ldw + c] = wv;
                A[(long long)row * ld + k0 + c] = lv;
                if (b) bsum[u] += lv * sz[c];
            }
        }
    }
    if (b) {
#pragma unroll
        for (int u = 0; u < 4; u++) {
            T v = bsum[u];
            for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            const int row = r0 + ty * 4 + u;
            if (tx == 0 && row < n) b[row] -= v;
        }
    }
}

// Trailing update of the lower 64x64 tiles: A_ij -= L_i W_j^T over p < kb.
template <typename T>
__global__ void __launch_bounds__(256) k_ldlt_update(int n, long long ld, T *A, int k0, int kb, const T *W, int ldw,
                                                     int k1) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *sLt = reinterpret_cast<T *>(smem_raw);   // [NB][64+pad] transposed: sLt[p][r]
    T *sWt = sLt + NB * 68;                      // [NB][68]
    long long bidx = blockIdx.x;
    int bi = (int)((sqrt(8.0 * (double)bidx + 1.0) - 1.0) * 0.5);
    while ((long long)(bi + 1) * (bi + 2) / 2 <= bidx) bi++;
    while ((long long)bi * (bi + 1) / 2 > bidx) bi--;
    int bj = (int)(bidx - (long long)bi * (bi + 1) / 2);
    const int i0 = k1 + bi * 64, j0 = k1 + bj * 64;
    {
        // 64 x NB elements of each operand, 16 per thread: issue all loads first
        T la[16], wa[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
            int idx = q * 256 + threadIdx.x;
            int r = idx / NB, p = idx % NB;
            int ri = i0 + r, rj = j0 + r;
            la[q] = (p < kb && ri < n) ? A[(long long)ri * ld + k0 + p] : T(0);
            wa[q] = (p < kb && rj < n) ? __ldg(&W[(long long)rj * ldw + p]) : T(0);
        }
#pragma unroll
        for (int q = 0; q < 16; q++) {
            int idx = q * 256 + threadIdx.x;
            int r = idx / NB, p = idx % NB;
            sLt[p * 68 + r] = la[q];
            sWt[p * 68 + r] = wa[q];
        }
    }
    __syncthreads();
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    T acc[4][4] = {};
    for (int p = 0; p < kb; p++) {
        T a[4], w[4];
#pragma unroll
        for (int u = 0; u < 4; u++) a[u] = sLt[p * 68 + ty * 4 + u];
#pragma unroll
        for (int v = 0; v < 4; v++) w[v] = sWt[p * 68 + tx * 4 + v];
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int v = 0; v < 4; v++) acc[u][v] = fma(a[u], w[v], acc[u][v]);
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
        int i = i0 + ty * 4 + u;
        if (i >= n) continue;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            int j = j0 + tx * 4 + v;
            if (j < n && j <= i) A[(long long)i * ld + j] -= acc[u][v];
        }
    }
}

// Update restricted to the columns [k1, jend) of the current outer panel:
// A_ij -= L_i W_j^T for rows i in [k1, n), 64x64 tiles, grid (col tile, row tile).
template <typename T>
__global__ void __launch_bounds__(256) k_ldlt_update_cols(int n, long long ld, T *A, int k0, int kb, const T *W,
                                                          int ldw, int k1, int jend) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *sLt = reinterpret_cast<T *>(smem_raw);
    T *sWt = sLt + NB * 68;
    const int i0 = k1 + blockIdx.y * 64, j0 = k1 + blockIdx.x * 64;
    if (j0 > i0 + 63 || j0 >= jend) return;  // tile entirely above the diagonal or outside the panel
    {
        T la[16], wa[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
            int idx = q * 256 + threadIdx.x;
            int r = idx / NB, p = idx % NB;
            int ri = i0 + r, rj = j0 + r;
            la[q] = (p < kb && ri < n) ? A[(long long)ri * ld + k0 + p] : T(0);
            wa[q] = (p < kb && rj < jend) ? __ldg(&W[(long long)rj * ldw + p]) : T(0);
        }
#pragma unroll
        for (int q = 0; q < 16; q++) {
            int idx = q * 256 + threadIdx.x;
            int r = idx / NB, p = idx % NB;
            sLt[p * 68 + r] = la[q];
            sWt[p * 68 + r] = wa[q];
        }
    }
    __syncthreads();
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    T acc[4][4] = {};
    for (int p = 0; p < kb; p++) {
        T a[4], w[4];
#pragma unroll
        for (int u = 0; u < 4; u++) a[u] = sLt[p * 68 + ty * 4 + u];
#pragma unroll
        for (int v = 0; v < 4; v++) w[v] = sWt[p * 68 + tx * 4 + v];
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int v = 0; v < 4; v++) acc[u][v] = fma(a[u], w[v], acc[u][v]);
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
        int i = i0 + ty * 4 + u;
        if (i >= n) continue;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            int j = j0 + tx * 4 + v;
            if (j < jend && j <= i) A[(long long)i * ld + j] -= acc[u][v];
        }
    }
}

// ---- triangular solves with an existing factor --------------------------------------
// One persistent launch per direction.  CTA g takes row blocks g, g+G, ... (in
// solve order); a block first subtracts the contributions of the blocks already
// solved (each published by a per-block ready word holding the solve's epoch),
// then solves its unit-triangular diagonal block with one warp.  Each poll takes
// every block already published (up to 256) at once, so a block's wait ends one
// block behind the wavefront.  The grid never exceeds the resident capacity, so
// the lowest unsolved block always runs.  Waits are bounded (TRSV_SPIN_LIMIT
// empty polls); a timeout sets the error flag.
constexpr long long TRSV_SPIN_LIMIT = 1ll << 20;

// Number of leading blocks (from `from`) known solved, up to `to`: a block is
// published only after all blocks before it (it waited for them), so the ready
// words form a prefix.  All threads call it; one round trip per call.
__device__ __forceinline__ int ready_prefix(const int *ready, int from, int to, int step, int epoch, int *s_cnt) {
    const int t = threadIdx.x;
    const int span = (to - from) * step;  // number of candidate blocks (step = +1 or -1)
    int k = from + step * t;
    bool ok = t < span && *(volatile const int *)&ready[k] == epoch;
    unsigned bal = __ballot_sync(0xffffffffu, ok);
    if (ok) __threadfence();  // acquire: the block's x values are read after this
    if ((t & 31) == 0) s_cnt[t >> 5] = bal == 0xffffffffu ? 32 : __ffs(~bal) - 1;
    __syncthreads();
    int cnt = 0;
    for (int w = 0; w < 8; w++) {
        int c = s_cnt[w];
        cnt += c;
        if (c < 32) break;
    }
    __syncthreads();
    return cnt < span ? cnt : span;
}

// L z = b (unit lower, in place on x)
template <typename T>
__global__ void __launch_bounds__(256) k_trsv_fwd(int n, long long ld, const T *A, T *x, int *ready, int epoch,
                                                  unsigned long long *flags) {
    __shared__ T sL[NB][NB + 1];
    __shared__ T srhs[NB];
    __shared__ int s_cnt[8];
    const int nblk = (n + NB - 1) / NB;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        const int r0 = blk * NB, kb = n - r0 < NB ? n - r0 : NB;
        const int r = t >> 2, q = t & 3;  // row, quarter of each 64-column block
        for (int idx = t; idx < kb * kb; idx += blockDim.x) {
            int i = idx / kb, j = idx % kb;
            sL[i][j] = j < i ? A[(long long)(r0 + i) * ld + r0 + j] : T(0);
        }
        T acc = 0;
        int done = 0;  // columns blocks [0, done) accumulated
        long long spins = 0;
        while (done < blk) {
            int avail = done + ready_prefix(ready, done, blk < done + 256 ? blk : done + 256, 1, epoch, s_cnt);
            if (avail == done) {
                if (++spins > TRSV_SPIN_LIMIT) {
                    if (t == 0) atomicOr(flags, FLAG_LOOKBACK_TIMEOUT);
                    break;
                }
                __nanosleep(32);
                continue;
            }
            __threadfence();
            if (r < kb) {
                const T *row = A + (long long)(r0 + r) * ld;
                for (int c = done; c < avail; c++) {
                    const int cb = c * NB + q * 16;
#pragma unroll
                    for (int k = 0; k < 16; k++) acc += __ldg(&row[cb + k]) * __ldcg(&x[cb + k]);
                }
            }
            done = avail;
        }
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        acc += __shfl_xor_sync(0xffffffffu, acc, 2);
        if (q == 0 && r < kb) srhs[r] = x[r0 + r] - acc;
        __syncthreads();
        if (warp == 0) {
            T v0 = lane < kb ? srhs[lane] : T(0), v1 = lane + 32 < kb ? srhs[lane + 32] : T(0);
            for (int j = 0; j < kb; j++) {
                T xj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
                if (lane > j && lane < kb) v0 -= sL[lane][j] * xj;
                if (lane + 32 > j && lane + 32 < kb) v1 -= sL[lane + 32][j] * xj;
            }
            if (lane < kb) x[r0 + lane] = v0;
            if (lane + 32 < kb) x[r0 + lane + 32] = v1;
            __threadfence();
            __syncwarp();
            if (lane == 0) *(volatile int *)&ready[blk] = epoch;
        }
        __syncthreads();
    }
}

// L^T y = D^-1 z (unit upper after scaling, in place on x), blocks from the last
template <typename T>
__global__ void __launch_bounds__(256) k_trsv_bwd(int n, long long ld, const T *A, const T *dvec, T *x, int *ready,
                                                  int epoch, unsigned long long *flags) {
    __shared__ T sL[NB][NB + 1];
    __shared__ T srhs[NB];
    __shared__ T spart[4][NB];
    __shared__ int s_cnt[8];
    const int nblk = (n + NB - 1) / NB;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    for (int g = blockIdx.x; g < nblk; g += gridDim.x) {
        const int blk = nblk - 1 - g;
        const int r0 = blk * NB, kb = n - r0 < NB ? n - r0 : NB;
        const int col = t & 63, part = t >> 6;  // column of this block, quarter of each later block's rows
        for (int idx = t; idx < kb * kb; idx += blockDim.x) {
            int i = idx / kb, j = idx % kb;
            sL[i][j] = j < i ? A[(long long)(r0 + i) * ld + r0 + j] : T(0);
        }
        T acc = 0;
        int done = nblk - 1;  // blocks (done, nblk) accumulated
        long long spins = 0;
        while (done > blk) {
            int lim = done - blk < 256 ? blk : done - 256;
            int avail = done - ready_prefix(ready, done, lim, -1, epoch, s_cnt);
            if (avail == done) {
                if (++spins > TRSV_SPIN_LIMIT) {
                    if (t == 0) atomicOr(flags, FLAG_LOOKBACK_TIMEOUT);
                    break;
                }
                __nanosleep(32);
                continue;
            }
            __threadfence();
            if (col < kb) {
                for (int c = done; c > avail; c--) {
                    const int c0 = c * NB, cb = n - c0 < NB ? n - c0 : NB;
                    for (int i = part * 16; i < part * 16 + 16 && i < cb; i++)
                        acc += __ldg(&A[(long long)(c0 + i) * ld + r0 + col]) * __ldcg(&x[c0 + i]);
                }
            }
            done = avail;
        }
        spart[part][col] = acc;
        __syncthreads();
        if (t < kb) srhs[t] = x[r0 + t] / dvec[r0 + t] - (spart[0][t] + spart[1][t] + spart[2][t] + spart[3][t]);
        __syncthreads();
        if (warp == 0) {
            T v0 = lane < kb ? srhs[lane] : T(0), v1 = lane + 32 < kb ? srhs[lane + 32] : T(0);
            for (int j = kb - 1; j >= 0; j--) {
                T yj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
                if (lane < j) v0 -= sL[j][lane] * yj;
                if (lane + 32 < j) v1 -= sL[j][lane + 32] * yj;
            }
            if (lane < kb) x[r0 + lane] = v0;
            if (lane + 32 < kb) x[r0 + lane + 32] = v1;
            __threadfence();
            __syncwarp();
            if (lane == 0) *(volatile int *)&ready[blk] = epoch;
        }
        __syncthreads();
    }
}

template <typename T>
struct LdltWork {
    T *dvec, *W, *s;
    T *Linv;       // [NB][NB] inverse of the current diagonal block's L
    int *ready;    // [2][blocks] per-block ready words of the two solves
};

static int g_solve_epoch = 0;

template <typename T>
int trsv_grid(mp_ctx *ctx, const void *kernel, int nblk) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0);
    if (per_sm < 1) per_sm = 1;
    int cap = per_sm * ctx->sm_count;  // every CTA resident: the wavefront cannot stall
    return nblk < cap ? nblk : cap;
}

template <typename T>
int ldlt_factor_solve(mp_ctx *ctx, T *A, long long ld, int n, T *b, LdltWork<T> w, bool factor,
                      bool tensor_cores = false) {
    cudaStream_t st = ctx->stream;
    const size_t diag_smem = sizeof(T) * (2 * NB * (NB + 1) + 3 * NB);
    const size_t panel_smem = sizeof(T) * (64 * (NB + 1) + NB * (NB + 1) + 2 * NB);
    const size_t upd_smem = sizeof(T) * 2 * NB * 68;
    static bool attr = false;
    if (!attr) {
        const int big = 96 * 1024;
        cudaFuncSetAttribute(k_ldlt_diag<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(k_ldlt_diag<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(k_ldlt_panel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(k_ldlt_panel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(k_ldlt_update<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(k_ldlt_update<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(k_ldlt_update_cols<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(k_ldlt_update_cols<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(tc::k_update_tf32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::SMEM_BYTES);
        attr = true;
    }
    unsigned long long *flags = ctx->counters + C_FLAGS;
    auto diag_and_panel = [&](int k0, int kb, T *W, int ldw) {
        k_ldlt_diag<T><<<1, 256, diag_smem, st>>>(n, ld, A, k0, kb, w.dvec, w.Linv, b, flags), ++ctx->launches;
        int k1 = k0 + kb;
        if (k1 < n)
            k_ldlt_panel<T><<<(n - k1 + 63) / 64, 256, panel_smem, st>>>(n, ld, A, k0, kb, w.dvec, w.Linv, W, ldw, b),
                ++ctx->launches;
    };
    if (factor && tensor_cores) {
        // two-level LDL^T: 256-wide outer panels factored with the 64-wide kernels,
        // trailing update of each outer panel on the tensor cores
        const int PW = 256;
        for (int P0 = 0; P0 < n; P0 += PW) {
            const int P1 = P0 + PW < n ? P0 + PW : n;
            for (int k0 = P0; k0 < P1; k0 += NB) {
                int kb = P1 - k0 < NB ? P1 - k0 : NB;
                int k1 = k0 + kb;
                diag_and_panel(k0, kb, w.W + (k0 - P0), PW);
                if (k1 < n && k1 < P1) {
                    dim3 g((P1 - k1 + 63) / 64, (n - k1 + 63) / 64);
                    k_ldlt_update_cols<T><<<g, 256, upd_smem, st>>>(n, ld, A, k0, kb, w.W + (k0 - P0), PW, k1, P1),
                        ++ctx->launches;
                }
            }
            if (P1 < n) {
                long long tiles = (n - P1 + tc::TILE - 1) / tc::TILE;
                long long nblk = tiles * (tiles + 1) / 2;
                tc::k_update_tf32<<<(unsigned)nblk, tc::THREADS, tc::SMEM_BYTES, st>>>(
                    n, ld, reinterpret_cast<float *>(A), P0, P1 - P0, P1, reinterpret_cast<const float *>(w.W), PW,
                    flags), ++ctx->launches;
            }
        }
    } else if (factor) {
        for (int k0 = 0; k0 < n; k0 += NB) {
            int kb = n - k0 < NB ? n - k0 : NB;
            int k1 = k0 + kb;
            diag_and_panel(k0, kb, w.W, NB);
            if (k1 < n) {
                long long tiles = (n - k1 + 63) / 64;
                long long nblk = tiles * (tiles + 1) / 2;
                k_ldlt_update<T><<<(unsigned)nblk, 256, upd_smem, st>>>(n, ld, A, k0, kb, w.W, NB, k1), ++ctx->launches;
            }
        }
    }
    const int nblk = (n + NB - 1) / NB;
    const int epoch = ++g_solve_epoch;
    if (!factor) {
        int g = trsv_grid<T>(ctx, (const void *)k_trsv_fwd<T>, nblk);
        k_trsv_fwd<T><<<g, 256, 0, st>>>(n, ld, A, b, w.ready, epoch, flags), ++ctx->launches;
    }
    int g = trsv_grid<T>(ctx, (const void *)k_trsv_bwd<T>, nblk);
    k_trsv_bwd<T><<<g, 256, 0, st>>>(n, ld, A, w.dvec, b, w.ready + nblk, epoch, flags), ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

}  // namespace mp
