// Dense symmetric factorization J = L D L^T of the Newton Jacobian and the
// solve J y = G, replacing the reference's LAPACK dsysv_ call
// (FESolver::solveLinearLapack, src/FESolver.cpp:528-558).
//
// Blocked right-looking LDL^T without pivoting on the lower triangle (row-major
// storage, leading dimension padded to 32).  Per block column k of width NB:
//   diag   : L_kk D_k L_kk^T = A_kk in shared memory (one CTA); z_k = L_kk^-1 b_k
//   panel  : W_ik = A_ik L_kk^-T,  L_ik = W_ik D_k^-1, b_i -= L_ik z_k  (rows below)
//   update : A_ij -= L_ik W_jk^T on the lower tiles of the trailing matrix,
//            two-level: within each 256-wide outer panel only the panel's own
//            columns, and the rest of the trailing matrix once per outer panel
// The forward substitution rides on the panel pass; the backward substitution
// L^T y = D^-1 z runs afterwards.
//
// J is symmetric (K is assembled symmetric, FP only touches the diagonal) and
// in these problems sign-definite, the case where LDL^T needs no pivoting.  A
// zero or non-finite pivot sets FLAG_SINGULAR and the call returns
// MP_ERR_SINGULAR; the solve's residual ||G - J y|| is reported either way.
//
// The FP32 instantiation is the factorization of the mixed form; its solve is
// wrapped in FP64 iterative refinement (residual from the FP64 K and FP).
#include <algorithm>
#include <cmath>
#include <type_traits>

#include <cudaTypedefs.h>

#include "mp_internal.h"
#include "mp_tc.cuh"

namespace mp {

constexpr int NB = 64;

template <typename T>
__device__ __forceinline__ bool bad_pivot(T d) {
    return !(fabs((double)d) > 0.0) || !isfinite((double)d);
}

// Factor the kb x kb diagonal block at (k0,k0): L (strict lower) and D written
// back, and Linv = L_kk^-1 (unit lower, row-major NB x NB, zero outside kb x kb)
// for the panel and the triangular solves.  If b is non-null,
// z_k = L_kk^-1 b_k (the forward substitution riding on the factorization).
//
// 256 threads, the block in shared memory (padded to 64 x 64 with an identity).
// Four sub-panels of SUB = 16 columns:
//   factor the sub-panel (64 x 16): 16 elimination steps, one barrier each;
//     thread (row i, column quad g) updates its 4 columns from the step's
//     published column (double-buffered), and the rows of the sub-panel's
//     16 x 16 diagonal block apply the same row operation to an identity,
//     which leaves that block's inverse;
//   rank-16 update of the trailing block, 4 x 4 register tiles per thread.
// The off-diagonal blocks of Linv follow by block substitution:
//   X_qp = -X_qq sum_{r=p}^{q-1} L_qr X_rp.
// Dynamic smem: A [64][65], Linv [64][65], W [64][17], T [16][17], w [2][64], b [64].
constexpr int SUB = 16;

template <typename T>
__global__ void __launch_bounds__(256) k_ldlt_diag(int n, long long ld, T *A, int k0, int kb, T *dvec, T *Linv,
                                                   T *b, unsigned long long *flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T(*sA)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(smem_raw);
    T(*sI)[NB + 1] = sA + NB;
    T(*sW)[SUB + 1] = reinterpret_cast<T(*)[SUB + 1]>(sI + NB);
    T(*sT)[SUB + 1] = sW + NB;
    T *sw = reinterpret_cast<T *>(sT + SUB);  // [2][NB]
    T *sb = sw + 2 * NB;
    const int t = threadIdx.x;
    // load the lower triangle, pad with an identity past kb; Linv starts as the identity
    {
        T v[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int idx = q * 256 + t, r = idx >> 6, c = idx & 63;
            v[q] = (r < kb && c < kb && c <= r) ? A[(long long)(k0 + r) * ld + k0 + c] : T(0);
        }
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int idx = q * 256 + t, r = idx >> 6, c = idx & 63;
            sA[r][c] = (r >= kb && r == c) ? T(1) : v[q];
            sI[r][c] = r == c ? T(1) : T(0);
        }
    }
    if (b && t < NB) sb[t] = t < kb ? b[k0 + t] : T(0);
    __syncthreads();
    if (t < NB) sw[t] = sA[t][0];  // publish column 0
    __syncthreads();
    const int i = t >> 2, g = t & 3;  // this thread's row and column quad in the sub-panel
    bool singular = false;
    for (int p = 0; p < NB / SUB; p++) {
        const int c0 = p * SUB;
        // ---- factor the sub-panel: columns [c0, c0+16), rows [c0, 64) ----
        for (int j = c0; j < c0 + SUB; j++) {
            const T *w = sw + (j & 1) * NB;
            T d = w[j];
            if (bad_pivot(d)) {
                singular = true;
                d = T(1);
            }
            const T rd = T(1) / d;
            const T wi = w[i];
            const T li = wi * rd;  // L[i][j] for i > j
            if (i > j) {
#pragma unroll
                for (int cc = 0; cc < 4; cc++) {
                    const int col = c0 + 4 * g + cc;
                    if (col > j && col <= i) sA[i][col] -= li * w[col];
                    if (col == j) sA[i][j] = li;
                    // the sub-panel's diagonal block: the same row operation on the identity
                    if (i < c0 + SUB && col <= j) sI[i][col] -= li * sI[j][col];
                }
            }
            // publish column j+1 (final for this step once its own update above has run)
            if (j + 1 < c0 + SUB && 4 * g <= j + 1 - c0 && j + 1 - c0 < 4 * g + 4) sw[((j + 1) & 1) * NB + i] = sA[i][j + 1];
            __syncthreads();
        }
        if (p == NB / SUB - 1) break;
        // ---- rank-16 update of the trailing block [c0+16, 64)^2 ----
        const int e0 = c0 + SUB;
        if (t < NB) {
#pragma unroll
            for (int jl = 0; jl < SUB; jl++) sW[t][jl] = sA[t][c0 + jl] * sA[c0 + jl][c0 + jl];
        }
        __syncthreads();
        {
            const int ti = t >> 4, tk = t & 15;
            const int r0 = 4 * ti, q0 = 4 * tk;
            if (r0 + 3 >= e0 && q0 + 3 >= e0 && q0 <= r0 + 3) {
                T acc[4][4] = {};
#pragma unroll
                for (int jl = 0; jl < SUB; jl++) {
                    T av[4], wv[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) av[u] = sA[r0 + u][c0 + jl];
#pragma unroll
                    for (int v = 0; v < 4; v++) wv[v] = sW[q0 + v][jl];
#pragma unroll
                    for (int u = 0; u < 4; u++)
#pragma unroll
                        for (int v = 0; v < 4; v++) acc[u][v] += av[u] * wv[v];
                }
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int v = 0; v < 4; v++) {
                        const int r = r0 + u, q = q0 + v;
                        if (r >= e0 && q >= e0 && q <= r) sA[r][q] -= acc[u][v];
                    }
            }
        }
        __syncthreads();
        if (t < NB) sw[(e0 & 1) * NB + t] = sA[t][e0];  // publish the next sub-panel's first column
        __syncthreads();
    }
    if (singular && t == 0) atomicOr(flags, FLAG_SINGULAR);
    // ---- off-diagonal blocks of Linv, by block distance ----
    for (int dist = 1; dist < NB / SUB; dist++) {
        for (int p = 0; p + dist < NB / SUB; p++) {
            const int q = p + dist;
            const int a = t >> 4, c = t & 15;  // element (a, c) of the 16 x 16 block
            // T = sum_{r=p}^{q-1} L_qr X_rp
            T acc = 0;
            for (int r = p; r < q; r++)
#pragma unroll
                for (int m = 0; m < SUB; m++) acc += sA[q * SUB + a][r * SUB + m] * sI[r * SUB + m][p * SUB + c];
            sT[a][c] = acc;
            __syncthreads();
            // X_qp = -X_qq T (X_qq unit lower)
            T x = 0;
#pragma unroll
            for (int m = 0; m < SUB; m++) x += sI[q * SUB + a][q * SUB + m] * sT[m][c];
            sI[q * SUB + a][p * SUB + c] = -x;
            __syncthreads();
        }
    }
    // ---- write back L, D, Linv; z = Linv b ----
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int idx = q * 256 + t, r = idx >> 6, c = idx & 63;
        const bool in = r < kb && c < kb;
        if (in && c <= r) A[(long long)(k0 + r) * ld + k0 + c] = sA[r][c];
        Linv[r * NB + c] = in ? sI[r][c] : T(0);
    }
    if (t < kb) {
        dvec[k0 + t] = sA[t][t];
        if (b) {
            T z = 0;
            for (int pp = 0; pp <= t; pp++) z += sI[t][pp] * sb[pp];
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

// FP64 form: A[i][j] -= sum_{k<K} L[i][k] W[j][k] for rows/cols from R0, with
// L = A[i][K0 ...] and W rows of pitch ldw (K a multiple of 16).  colblocks = 0:
// the lower 128x128 tiles of [R0, n)^2 (the trailing update of a super-panel);
// colblocks > 0: every tile of rows [R0, n) x columns [R0, R0 + 128*colblocks)
// (a strip inside a super-panel), lower parts only.  256 threads, 8x8
// accumulators per thread (rows ty + 16u, columns tx + 16v), K streamed in
// 16-wide chunks through two shared-memory buffers stored k-major (the next
// chunk is loaded into registers while this one computes).
constexpr int WTILE = 128, WKC = 16;

__global__ void __launch_bounds__(256, 1) k_update_f64(int n, long long ld, double *A, int K0, int K, int R0,
                                                       const double *__restrict__ W, int ldw, int colblocks) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double(*sL)[WKC][WTILE] = reinterpret_cast<double(*)[WKC][WTILE]>(smem_raw);
    double(*sW)[WKC][WTILE] = sL + 2;
    long long bidx = blockIdx.x;
    int bi, bj;
    if (colblocks > 0) {
        bi = (int)(bidx / colblocks);
        bj = (int)(bidx % colblocks);
    } else {
        bi = (int)((sqrt(8.0 * (double)bidx + 1.0) - 1.0) * 0.5);
        while ((long long)(bi + 1) * (bi + 2) / 2 <= bidx) bi++;
        while ((long long)bi * (bi + 1) / 2 > bidx) bi--;
        bj = (int)(bidx - (long long)bi * (bi + 1) / 2);
    }
    const long long i0 = R0 + (long long)bi * WTILE, j0 = R0 + (long long)bj * WTILE;
    if (j0 > i0 + WTILE - 1) return;  // strip tile entirely above the diagonal
    const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
    // loader: row lr of the tile, k half lh (8 values)
    const int lr = t >> 1, lh = t & 1;
    const bool lrow = i0 + lr < n, wrow = j0 + lr < n;
    const double *lsrc = A + (i0 + (lrow ? lr : 0)) * ld + K0 + lh * 8;
    const double *wsrc = W + (j0 + (wrow ? lr : 0)) * (long long)ldw + lh * 8;
    double2 pl[4], pw[4];
    auto fetch = [&](int kc) {
#pragma unroll
        for (int e = 0; e < 4; e++) {
            pl[e] = lrow ? __ldg(reinterpret_cast<const double2 *>(lsrc + kc * WKC) + e) : make_double2(0.0, 0.0);
            pw[e] = wrow ? __ldg(reinterpret_cast<const double2 *>(wsrc + kc * WKC) + e) : make_double2(0.0, 0.0);
        }
    };
    auto stash = [&](int buf) {
#pragma unroll
        for (int e = 0; e < 4; e++) {
            sL[buf][lh * 8 + 2 * e][lr] = pl[e].x;
            sL[buf][lh * 8 + 2 * e + 1][lr] = pl[e].y;
            sW[buf][lh * 8 + 2 * e][lr] = pw[e].x;
            sW[buf][lh * 8 + 2 * e + 1][lr] = pw[e].y;
        }
    };
    double acc[8][8];
#pragma unroll
    for (int u = 0; u < 8; u++)
#pragma unroll
        for (int v = 0; v < 8; v++) acc[u][v] = 0.0;
    fetch(0);
    stash(0);
    __syncthreads();
    const int NKC = K / WKC;
#pragma unroll 1
    for (int kc = 0; kc < NKC; kc++) {
        const int buf = kc & 1;
        if (kc + 1 < NKC) fetch(kc + 1);
#pragma unroll
        for (int k = 0; k < WKC; k++) {
            double a[8], b[8];
#pragma unroll
            for (int u = 0; u < 8; u++) a[u] = sL[buf][k][ty + 16 * u];
#pragma unroll
            for (int v = 0; v < 8; v++) b[v] = sW[buf][k][tx + 16 * v];
#pragma unroll
            for (int u = 0; u < 8; u++)
#pragma unroll
                for (int v = 0; v < 8; v++) acc[u][v] = fma(a[u], b[v], acc[u][v]);
        }
        if (kc + 1 < NKC) stash(buf ^ 1);
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
        const long long row = i0 + ty + 16 * u;
        if (row >= n) continue;
#pragma unroll
        for (int v = 0; v < 8; v++) {
            const long long col = j0 + tx + 16 * v;
            if (col < n && col <= row) A[row * ld + col] -= acc[u][v];
        }
    }
}

// ---- triangular solves with an existing factor --------------------------------------
// One persistent launch per direction.  CTA g takes row blocks g, g+G, ... (in
// solve order); a block subtracts the contributions of the blocks already
// solved (each published by a per-block ready word holding the solve's epoch,
// stored with release semantics and polled with acquire loads), then applies
// its diagonal block's stored inverse: the block's own solve is a 64 x 64
// product, not a serial substitution.  Each poll takes every block already
// published (up to 256) at once, and the operand chunk of the next awaited block
// is loaded before the poll, so a block's wait ends one chunk behind the
// wavefront.  The grid never exceeds the resident capacity, so the lowest
// unsolved block always runs.  Waits are bounded (TRSV_SPIN_LIMIT empty polls);
// a timeout sets the error flag.
constexpr long long TRSV_SPIN_LIMIT = 1ll << 20;

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Number of consecutive published blocks from `from` in direction `step`
// (+1 or -1), at most `span`.  All threads call it; one round trip per call.
__device__ __forceinline__ int ready_prefix(const int *ready, int from, int span, int step, int epoch, int *s_cnt) {
    const int t = threadIdx.x;
    const bool ok = t < span && ld_acquire(ready + from + step * t) == epoch;
    const unsigned bal = __ballot_sync(0xffffffffu, ok);
    if ((t & 31) == 0) s_cnt[t >> 5] = bal == 0xffffffffu ? 32 : __ffs(~bal) - 1;
    __syncthreads();
    int cnt = 0;
    for (int w = 0; w < 8; w++) {
        const int c = s_cnt[w];
        cnt += c;
        if (c < 32) break;
    }
    __syncthreads();
    return cnt < span ? cnt : span;
}

// 16 consecutive values (64-byte aligned for float, 128 for double) as vector loads
template <typename T, bool CG>
__device__ __forceinline__ void load16(const T *p, T (&v)[16]) {
    if constexpr (sizeof(T) == 8) {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            double2 d = CG ? __ldcg(reinterpret_cast<const double2 *>(p) + k) : __ldg(reinterpret_cast<const double2 *>(p) + k);
            v[2 * k] = d.x;
            v[2 * k + 1] = d.y;
        }
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            float4 f = CG ? __ldcg(reinterpret_cast<const float4 *>(p) + k) : __ldg(reinterpret_cast<const float4 *>(p) + k);
            v[4 * k] = f.x;
            v[4 * k + 1] = f.y;
            v[4 * k + 2] = f.z;
            v[4 * k + 3] = f.w;
        }
    }
}

// L z = b (unit lower, in place on x)
template <typename T>
__global__ void __launch_bounds__(256) k_trsv_fwd(int n, long long ld, const T *A, const T *Linv, T *x, int *ready,
                                                  int epoch, unsigned long long *flags) {
    __shared__ T sI[NB][NB + 1];
    __shared__ T srhs[NB];
    __shared__ int s_cnt[8];
    const int nblk = (n + NB - 1) / NB;
    const int t = threadIdx.x;
    const int r = t >> 2, q = t & 3;  // row of the block, quarter of each 64-column chunk
    for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        const int r0 = blk * NB, kb = n - r0 < NB ? n - r0 : NB;
        for (int idx = t; idx < NB * NB; idx += 256) sI[idx >> 6][idx & 63] = __ldg(&Linv[(size_t)blk * NB * NB + idx]);
        // this block's right-hand side is no other block's output: read it before waiting
        const T rhs = (q == 0 && r < kb) ? __ldcg(&x[r0 + r]) : T(0);
        const T *row = A + (long long)(r0 + (r < kb ? r : 0)) * ld + q * 16;
        T acc = 0, ap[16], xv[16];
        int done = 0;  // column chunks [0, done) accumulated
        if (done < blk) load16<T, false>(row, ap);
        long long spins = 0;
        while (done < blk) {
            const int span = blk - done < 256 ? blk - done : 256;
            const int cnt = ready_prefix(ready, done, span, 1, epoch, s_cnt);
            if (cnt == 0) {
                if (++spins > TRSV_SPIN_LIMIT) {
                    if (t == 0) atomicOr(flags, FLAG_LOOKBACK_TIMEOUT);
                    break;
                }
                __nanosleep(32);
                continue;
            }
            const int avail = done + cnt;
            load16<T, true>(x + done * NB + q * 16, xv);
#pragma unroll
            for (int k = 0; k < 16; k++) acc = fma(ap[k], xv[k], acc);
            for (int c = done + 1; c < avail; c++) {
                load16<T, false>(row + c * NB, ap);
                load16<T, true>(x + c * NB + q * 16, xv);
#pragma unroll
                for (int k = 0; k < 16; k++) acc = fma(ap[k], xv[k], acc);
            }
            done = avail;
            if (done < blk) load16<T, false>(row + done * NB, ap);
        }
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        acc += __shfl_xor_sync(0xffffffffu, acc, 2);
        if (q == 0) srhs[r] = r < kb ? rhs - acc : T(0);
        __syncthreads();
        T v = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) v = fma(sI[r][q * 16 + k], srhs[q * 16 + k], v);
        v += __shfl_xor_sync(0xffffffffu, v, 1);
        v += __shfl_xor_sync(0xffffffffu, v, 2);
        if (q == 0 && r < kb) x[r0 + r] = v;
        __syncthreads();
        if (t == 0) st_release(ready + blk, epoch);
    }
}

// 4 consecutive values (16-byte aligned for float, 32 for double) as vector loads
template <typename T, bool CG>
__device__ __forceinline__ void load4(const T *p, T (&v)[4]) {
    if constexpr (sizeof(T) == 8) {
        const double2 a = CG ? __ldcg(reinterpret_cast<const double2 *>(p)) : __ldg(reinterpret_cast<const double2 *>(p));
        const double2 b = CG ? __ldcg(reinterpret_cast<const double2 *>(p) + 1)
                             : __ldg(reinterpret_cast<const double2 *>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    } else {
        const float4 a = CG ? __ldcg(reinterpret_cast<const float4 *>(p)) : __ldg(reinterpret_cast<const float4 *>(p));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
}

// L^T y = D^-1 z (unit upper after scaling, in place on x), blocks from the last.
// Thread (column quad c4, row quad part) takes a 4 x 4 piece of every later
// 64 x 64 chunk with vector loads; the 16 partial sums of each column meet in
// shared memory.
template <typename T>
__global__ void __launch_bounds__(256) k_trsv_bwd(int n, long long ld, const T *A, const T *Linv, const T *dvec, T *x,
                                                  int *ready, int epoch, unsigned long long *flags) {
    __shared__ T sI[NB][NB + 1];
    __shared__ T srhs[NB];
    __shared__ T spart[16][NB + 1];
    __shared__ int s_cnt[8];
    const int nblk = (n + NB - 1) / NB;
    const int t = threadIdx.x;
    const int c4 = t & 15, part = t >> 4;  // columns 4*c4 .. +3 of this block, rows 4*part .. +3 of each chunk
    for (int g = blockIdx.x; g < nblk; g += gridDim.x) {
        const int blk = nblk - 1 - g;
        const int r0 = blk * NB, kb = n - r0 < NB ? n - r0 : NB;
        // D^-1 z of this block: final before the kernel started, read before waiting
        const T rhs = (t < NB && t < kb) ? __ldcg(&x[r0 + t]) / dvec[r0 + t] : T(0);
        for (int idx = t; idx < NB * NB; idx += 256) sI[idx >> 6][idx & 63] = __ldg(&Linv[(size_t)blk * NB * NB + idx]);
        T acc[4] = {0, 0, 0, 0}, ap[4][4];
        // rows c*NB + 4*part + e, columns r0 + 4*c4 .. +3 (zero past n; every block before the last is full)
        auto fetch = [&](int c) {
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int i = c * NB + 4 * part + e;
                if (i < n) {
                    load4<T, false>(A + (long long)i * ld + r0 + 4 * c4, ap[e]);
                } else {
#pragma unroll
                    for (int j = 0; j < 4; j++) ap[e][j] = T(0);
                }
            }
        };
        int done = nblk - 1;  // chunks (done, nblk) accumulated
        if (done > blk) fetch(done);
        long long spins = 0;
        while (done > blk) {
            const int span = done - blk < 256 ? done - blk : 256;
            const int cnt = ready_prefix(ready, done, span, -1, epoch, s_cnt);
            if (cnt == 0) {
                if (++spins > TRSV_SPIN_LIMIT) {
                    if (t == 0) atomicOr(flags, FLAG_LOOKBACK_TIMEOUT);
                    break;
                }
                __nanosleep(32);
                continue;
            }
            const int avail = done - cnt;
            for (int c = done; c > avail; c--) {
                if (c != done) fetch(c);
                const int i0 = c * NB + 4 * part;
                T xv[4];
                if (i0 + 3 < n) {
                    load4<T, true>(x + i0, xv);
                } else {
#pragma unroll
                    for (int e = 0; e < 4; e++) xv[e] = i0 + e < n ? __ldcg(&x[i0 + e]) : T(0);
                }
#pragma unroll
                for (int e = 0; e < 4; e++)
#pragma unroll
                    for (int j = 0; j < 4; j++) acc[j] = fma(ap[e][j], xv[e], acc[j]);
            }
            done = avail;
            if (done > blk) fetch(done);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) spart[part][4 * c4 + j] = acc[j];
        __syncthreads();
        if (t < NB) {
            T sum = 0;
#pragma unroll
            for (int pp = 0; pp < 16; pp++) sum += spart[pp][t];
            srhs[t] = t < kb ? rhs - sum : T(0);
        }
        __syncthreads();
        // y = Linv^T srhs
        T v[4] = {0, 0, 0, 0};
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const T rr = srhs[4 * part + e];
#pragma unroll
            for (int j = 0; j < 4; j++) v[j] = fma(sI[4 * part + e][4 * c4 + j], rr, v[j]);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) spart[part][4 * c4 + j] = v[j];
        __syncthreads();
        if (t < kb) {
            T sum = 0;
#pragma unroll
            for (int pp = 0; pp < 16; pp++) sum += spart[pp][t];
            x[r0 + t] = sum;
        }
        __syncthreads();
        if (t == 0) st_release(ready + blk, epoch);
    }
}

template <typename T>
struct LdltWork {
    T *dvec, *W, *s;
    T *Linv;       // [blocks][NB][NB] inverses of the diagonal blocks' L (the solves use them)
    int *ready;    // [2][blocks] per-block ready words of the two solves
    float *split;  // tensor-core path: [4][n][SUPER_W] hi/lo copies of the update's L and W rows
};

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// Map of a [rows][K] FP32 operand with row pitch `pitch` elements, loaded as
// boxes of 32 (K) x box_rows rows with the 128-byte swizzle the UMMA
// descriptors use.  base must be 16-byte aligned and pitch*4 a multiple of 16.
static bool operand_map(CUtensorMap *m, const float *base, long long rows, long long pitch, int box_rows, int K) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = tensor_map_encoder();
    if (!fn || rows < 1 || (reinterpret_cast<size_t>(base) & 15) || ((pitch * 4) & 15)) return false;
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)pitch * 4};
    cuuint32_t box[2] = {(cuuint32_t)tc::KC, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Super-panel width of the two-level LDL^T: the trailing matrix is read and
// written once per SUPER_W columns (the HBM traffic that bounds the trailing
// update), the panels inside a super-panel update only its remaining columns.
constexpr int PANEL_W = 256, SUPER_W = 4 * PANEL_W;

// The wavefront kernels wait on blocks that other CTAs of the same grid
// publish, so every CTA must be resident at once: they go out as cooperative
// launches, which the runtime schedules only as a whole grid (a second
// context's kernels on the same GPU cannot hold part of it back).
template <typename... Args>
static cudaError_t launch_wavefront(void (*kernel)(Args...), int grid, cudaStream_t st, Args... args) {
    void *argv[] = {(void *)&args...};
    return cudaLaunchCooperativeKernel((const void *)kernel, dim3(grid), dim3(256), argv, 0, st);
}

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
                      int tc_terms = 0) {
    cudaStream_t st = ctx->stream;
    const size_t diag_smem = sizeof(T) * (2 * NB * (NB + 1) + NB * (SUB + 1) + SUB * (SUB + 1) + 3 * NB);
    const size_t panel_smem = sizeof(T) * (64 * (NB + 1) + NB * (NB + 1) + 2 * NB);
    const size_t upd_smem = sizeof(T) * 2 * NB * 68;
    const size_t f64_smem = sizeof(double) * 4 * WKC * WTILE;
    if (!ctx->ldlt_attr) {  // per context: the attributes belong to the context's device
        const int big = 96 * 1024;
        cudaFuncSetAttribute(k_ldlt_diag<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(k_ldlt_diag<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(k_ldlt_panel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(k_ldlt_panel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(k_update_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(k_ldlt_update_cols<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(k_ldlt_update_cols<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(tc::k_update_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tc::smem_bytes(false));
        cudaFuncSetAttribute(tc::k_update_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tc::smem_bytes(true));
        ctx->ldlt_attr = true;
    }
    unsigned long long *flags = ctx->counters + C_FLAGS;
    auto diag_and_panel = [&](int k0, int kb, T *W, int ldw) {
        T *Li = w.Linv + (size_t)(k0 / NB) * NB * NB;
        int mk = kt_begin(ctx, MP_KT_DIAG, 0);
        k_ldlt_diag<T><<<1, 256, diag_smem, st>>>(n, ld, A, k0, kb, w.dvec, Li, b, flags), ++ctx->launches;
        kt_end(ctx, mk);
        int k1 = k0 + kb;
        if (k1 < n) {
            mk = kt_begin(ctx, MP_KT_PANEL, 0);
            k_ldlt_panel<T><<<(n - k1 + 63) / 64, 256, panel_smem, st>>>(n, ld, A, k0, kb, w.dvec, Li, W, ldw, b),
                ++ctx->launches;
            kt_end(ctx, mk);
        }
    };
    // algorithmic flops of an update of rows [R0, n) x columns [R0, C1), lower part, depth K
    auto update_flops = [&](int R0, int C1, int K) {
        const double m = n - R0, wcol = C1 - R0;
        const double pairs = C1 >= n ? m * (m + 1) / 2 : wcol * (wcol + 1) / 2 + (m - wcol) * wcol;
        return 2.0 * K * pairs;
    };
    // A[i][j] -= sum_{k<K} L[i][K0+k] W[j][kofs+k] for rows [R0, n) and columns
    // [R0, C1): a strip inside a super-panel when C1 < n, else the lower
    // triangle of the trailing matrix.  W rows are global rows, pitch SUPER_W.
    auto update = [&](int R0, int C1, int K0, int K, int kofs) -> int {
        const bool strip = C1 < n;
        if (std::is_same<T, double>::value) {
            const long long rb = (n - R0 + WTILE - 1) / WTILE;
            const int cb = strip ? (C1 - R0) / WTILE : 0;
            const long long ntiles = strip ? rb * cb : rb * (rb + 1) / 2;
            const int mk = kt_begin(ctx, MP_KT_UPDATE, update_flops(R0, C1, K));
            k_update_f64<<<(unsigned)ntiles, 256, f64_smem, st>>>(n, ld, reinterpret_cast<double *>(A), K0, K, R0,
                                                                 reinterpret_cast<const double *>(w.W) + kofs,
                                                                 SUPER_W, cb),
                ++ctx->launches;
            kt_end(ctx, mk);
            return MP_OK;
        }
        const long long rb = (n - R0 + tc::TILE - 1) / tc::TILE;
        const int cb = strip ? (C1 - R0) / tc::TILE_N : 0;
        const long long ntiles = strip ? rb * cb : tc::tile_count(rb);
        const long long wrows = (strip ? C1 : n) - R0;
        const bool split = tc_terms == 3;
        float *Af = reinterpret_cast<float *>(A);
        const float *Wf = reinterpret_cast<const float *>(w.W);
        const float *Lsrc = Af + (long long)R0 * ld + K0, *Wsrc = Wf + (long long)R0 * SUPER_W + kofs;
        CUtensorMap mLh, mWh, mLl, mWl;
        bool ok;
        if (split) {
            const size_t plane = (size_t)n * SUPER_W;
            float *Lh = w.split, *Ll = w.split + plane, *Wh = w.split + 2 * plane, *Wl = w.split + 3 * plane;
            const int gl = (int)std::min<long long>(((n - R0) * (K / 4) + 255) / 256, (long long)ctx->sm_count * 8);
            const int gw = (int)std::min<long long>((wrows * (K / 4) + 255) / 256, (long long)ctx->sm_count * 8);
            const int mk = kt_begin(ctx, MP_KT_PANEL, 0);
            tc::k_split_rows<<<gl, 256, 0, st>>>(Lsrc, ld, n - R0, K, Lh, Ll), ++ctx->launches;
            tc::k_split_rows<<<gw, 256, 0, st>>>(Wsrc, SUPER_W, wrows, K, Wh, Wl), ++ctx->launches;
            kt_end(ctx, mk);
            ok = operand_map(&mLh, Lh, n - R0, K, tc::TILE, K) && operand_map(&mWh, Wh, wrows, K, tc::TILE_N, K) &&
                 operand_map(&mLl, Ll, n - R0, K, tc::TILE, K) && operand_map(&mWl, Wl, wrows, K, tc::TILE_N, K);
        } else {
            ok = operand_map(&mLh, Lsrc, n - R0, ld, tc::TILE, K) &&
                 operand_map(&mWh, Wsrc, wrows, SUPER_W, tc::TILE_N, K);
            mLl = mLh;
            mWl = mWh;
        }
        if (!ok) return fail(ctx, MP_ERR_CUDA, "cuTensorMapEncodeTiled failed for the tensor-core update");
        const int grid = (int)std::min<long long>(ntiles, (long long)ctx->sm_count);
        auto kern = split ? tc::k_update_tc<true> : tc::k_update_tc<false>;
        const int mk = kt_begin(ctx, MP_KT_UPDATE, update_flops(R0, C1, K));
        kern<<<grid, tc::THREADS, tc::smem_bytes(split), st>>>(mLh, mWh, mLl, mWl, n, ld, Af, R0, ntiles, K / tc::KC,
                                                               cb, flags),
            ++ctx->launches;
        kt_end(ctx, mk);
        return MP_OK;
    };
    if (factor) {
        // Two-level LDL^T over super-panels of SUPER_W columns, each made of
        // PANEL_W-wide panels.  A panel is factored with the 64-wide kernels
        // (diagonal block, panel, updates restricted to the panel's columns),
        // then updates the rest of its super-panel (a strip); the trailing
        // matrix gets one update per super-panel with K = SUPER_W: on the tensor
        // cores for the FP32 factor (TF32, or 3xTF32 when tc_terms == 3),
        // register-tiled FP64 for the FP64 factor.
        for (int S0 = 0; S0 < n; S0 += SUPER_W) {
            const int S1 = S0 + SUPER_W < n ? S0 + SUPER_W : n;
            for (int P0 = S0; P0 < S1; P0 += PANEL_W) {
                const int P1 = P0 + PANEL_W < S1 ? P0 + PANEL_W : S1;
                for (int k0 = P0; k0 < P1; k0 += NB) {
                    const int kb = P1 - k0 < NB ? P1 - k0 : NB;
                    const int k1 = k0 + kb;
                    diag_and_panel(k0, kb, w.W + (k0 - S0), SUPER_W);
                    if (k1 < n && k1 < P1) {
                        dim3 g((P1 - k1 + 63) / 64, (n - k1 + 63) / 64);
                        const int mk = kt_begin(ctx, MP_KT_PANEL, 0);
                        k_ldlt_update_cols<T><<<g, 256, upd_smem, st>>>(n, ld, A, k0, kb, w.W + (k0 - S0), SUPER_W,
                                                                        k1, P1),
                            ++ctx->launches;
                        kt_end(ctx, mk);
                    }
                }
                if (P1 < S1) {  // a full panel with more of its super-panel to the right
                    int rc = update(P1, S1, P0, PANEL_W, P0 - S0);
                    if (rc) return rc;
                }
            }
            if (S1 < n) {  // a full super-panel
                int rc = update(S1, n, S0, SUPER_W, 0);
                if (rc) return rc;
            }
        }
    }
    const int nblk = (n + NB - 1) / NB;
    const int epoch = ++ctx->solve_epoch;
    const int mk = kt_begin(ctx, MP_KT_TRSV, 0);
    if (!factor) {
        int g = trsv_grid<T>(ctx, (const void *)k_trsv_fwd<T>, nblk);
        MP_CUDA(ctx, launch_wavefront(k_trsv_fwd<T>, g, st, n, ld, (const T *)A, (const T *)w.Linv, b, w.ready,
                                      epoch, flags));
        ++ctx->launches;
    }
    int g = trsv_grid<T>(ctx, (const void *)k_trsv_bwd<T>, nblk);
    MP_CUDA(ctx, launch_wavefront(k_trsv_bwd<T>, g, st, n, ld, (const T *)A, (const T *)w.Linv, (const T *)w.dvec,
                                  b, w.ready + nblk, epoch, flags));
    ++ctx->launches;
    kt_end(ctx, mk);
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

}  // namespace mp
