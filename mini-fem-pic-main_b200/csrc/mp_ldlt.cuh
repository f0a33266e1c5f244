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

namespace mp {

constexpr int NB = 64;

template <typename T>
__device__ __forceinline__ bool bad_pivot(T d) {
    return !(fabs((double)d) > 0.0) || !isfinite((double)d);
}

// Factor the kb x kb diagonal block at (k0,k0); write L (strict lower) back,
// D into dvec, and z_k = L_kk^-1 b_k into b (b may be null).
template <typename T>
__global__ void k_ldlt_diag(int n, long long ld, T *A, int k0, int kb, T *dvec, T *b,
                            unsigned long long *flags) {
    __shared__ T s[NB][NB + 1];
    __shared__ T s_w[NB];
    for (int idx = threadIdx.x; idx < kb * kb; idx += blockDim.x) {
        int r = idx / kb, c = idx % kb;
        s[r][c] = c <= r ? A[(long long)(k0 + r) * ld + k0 + c] : T(0);
    }
    __syncthreads();
    for (int j = 0; j < kb; j++) {
        T d = s[j][j];
        bool bad = bad_pivot(d);
        for (int i = j + 1 + threadIdx.x; i < kb; i += blockDim.x) s_w[i] = s[i][j];
        __syncthreads();
        if (bad) {
            if (threadIdx.x == 0) atomicOr(flags, FLAG_SINGULAR);
            d = T(1);
        }
        // rank-1 update of the remaining lower triangle
        int m = kb - j - 1;
        for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
            int i = j + 1 + idx / m, l = j + 1 + idx % m;
            if (l <= i) s[i][l] -= (s_w[i] / d) * s_w[l];
        }
        __syncthreads();
        for (int i = j + 1 + threadIdx.x; i < kb; i += blockDim.x) s[i][j] = s_w[i] / d;
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < kb * kb; idx += blockDim.x) {
        int r = idx / kb, c = idx % kb;
        if (c < r) A[(long long)(k0 + r) * ld + k0 + c] = s[r][c];
        else if (c == r) A[(long long)(k0 + r) * ld + k0 + c] = s[r][r];
    }
    if (threadIdx.x < kb) dvec[k0 + threadIdx.x] = s[threadIdx.x][threadIdx.x];
    if (b && threadIdx.x == 0) {
        for (int c = 0; c < kb; c++) {
            T x = b[k0 + c];
            for (int p = 0; p < c; p++) x -= s[c][p] * b[k0 + p];
            b[k0 + c] = x;
        }
    }
}

// Panel: rows [r0, r0+64) below the diagonal block.  Dynamic smem: L_kk [NB][NB]
// plus the CTA's rows [64][NB+1].
template <typename T>
__global__ void k_ldlt_panel(int n, long long ld, T *A, int k0, int kb, const T *dvec, T *W, T *b) {
    extern __shared__ unsigned char smem_raw[];
    T *sL = reinterpret_cast<T *>(smem_raw);           // [NB][NB]
    T *sR = sL + NB * NB;                               // [64][NB+1]
    const int r0 = k0 + kb + blockIdx.x * 64;
    for (int idx = threadIdx.x; idx < kb * kb; idx += blockDim.x) {
        int r = idx / kb, c = idx % kb;
        sL[r * NB + c] = c < r ? A[(long long)(k0 + r) * ld + k0 + c] : T(0);
    }
    for (int idx = threadIdx.x; idx < 64 * kb; idx += blockDim.x) {
        int r = idx / kb, c = idx % kb;
        int row = r0 + r;
        sR[r * (NB + 1) + c] = row < n ? A[(long long)row * ld + k0 + c] : T(0);
    }
    __syncthreads();
    if (threadIdx.x < 64) {
        int r = threadIdx.x;
        T *x = sR + r * (NB + 1);
        for (int c = 0; c < kb; c++) {
            T v = x[c];
            for (int p = 0; p < c; p++) v -= x[p] * sL[c * NB + p];
            x[c] = v;
        }
    }
    __syncthreads();
    // write W (= L D) and L, and the forward-substitution update of b
    for (int idx = threadIdx.x; idx < 64 * kb; idx += blockDim.x) {
        int r = idx / kb, c = idx % kb;
        int row = r0 + r;
        if (row < n) {
            T w = sR[r * (NB + 1) + c];
            W[(long long)row * NB + c] = w;
            A[(long long)row * ld + k0 + c] = w / dvec[k0 + c];
        }
    }
    if (b && threadIdx.x < 64) {
        int r = threadIdx.x, row = r0 + r;
        if (row < n) {
            T acc = 0;
            for (int c = 0; c < kb; c++) acc += (sR[r * (NB + 1) + c] / dvec[k0 + c]) * b[k0 + c];
            b[row] -= acc;
        }
    }
}

// Trailing update of the lower 64x64 tiles: A_ij -= L_i W_j^T over p < kb.
template <typename T>
__global__ void __launch_bounds__(256) k_ldlt_update(int n, long long ld, T *A, int k0, int kb, const T *W, int k1) {
    extern __shared__ unsigned char smem_raw[];
    T *sLt = reinterpret_cast<T *>(smem_raw);   // [NB][64+pad] transposed: sLt[p][r]
    T *sWt = sLt + NB * 68;                      // [NB][68]
    long long bidx = blockIdx.x;
    int bi = (int)((sqrt(8.0 * (double)bidx + 1.0) - 1.0) * 0.5);
    while ((long long)(bi + 1) * (bi + 2) / 2 <= bidx) bi++;
    while ((long long)bi * (bi + 1) / 2 > bidx) bi--;
    int bj = (int)(bidx - (long long)bi * (bi + 1) / 2);
    const int i0 = k1 + bi * 64, j0 = k1 + bj * 64;
    for (int idx = threadIdx.x; idx < 64 * NB; idx += blockDim.x) {
        int r = idx / NB, p = idx % NB;
        int ri = i0 + r, rj = j0 + r;
        sLt[p * 68 + r] = (p < kb && ri < n) ? A[(long long)ri * ld + k0 + p] : T(0);
        sWt[p * 68 + r] = (p < kb && rj < n) ? W[(long long)rj * NB + p] : T(0);
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

// z <- D^-1 z
template <typename T>
__global__ void k_diag_scale(int n, const T *dvec, T *z) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) z[i] /= dvec[i];
}

// Backward substitution step for block column k: s[c] = sum_{i>=k1} L[i][k0+c] y[i]
template <typename T>
__global__ void k_bwd_partial(int n, long long ld, const T *A, int k0, int kb, int k1, const T *y, T *s) {
    __shared__ T red[8][NB];
    int c = threadIdx.x & 63;
    int g = threadIdx.x >> 6;  // 4 row groups of 64 threads
    T acc = 0;
    if (c < kb)
        for (int i = k1 + blockIdx.x * 4 + g; i < n; i += gridDim.x * 4) acc += A[(long long)i * ld + k0 + c] * y[i];
    red[g][c] = acc;
    __syncthreads();
    if (g == 0 && c < kb) {
        T t = red[0][c] + red[1][c] + red[2][c] + red[3][c];
        atomicAdd(&s[c], t);
    }
}

template <typename T>
__global__ void k_bwd_diag(long long ld, const T *A, int k0, int kb, T *y, T *s) {
    __shared__ T sL[NB][NB + 1];
    for (int idx = threadIdx.x; idx < kb * kb; idx += blockDim.x) {
        int r = idx / kb, c = idx % kb;
        sL[r][c] = c < r ? A[(long long)(k0 + r) * ld + k0 + c] : T(0);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int c = kb - 1; c >= 0; c--) {
            T v = y[k0 + c] - s[c];
            for (int r = c + 1; r < kb; r++) v -= sL[r][c] * y[k0 + r];
            y[k0 + c] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x < NB) s[threadIdx.x] = 0;
}

// Forward substitution with an existing factor (refinement solves).
template <typename T>
__global__ void k_fwd_diag(long long ld, const T *A, int k0, int kb, T *b) {
    if (threadIdx.x != 0) return;
    for (int c = 0; c < kb; c++) {
        T x = b[k0 + c];
        for (int p = 0; p < c; p++) x -= A[(long long)(k0 + c) * ld + k0 + p] * b[k0 + p];
        b[k0 + c] = x;
    }
}

template <typename T>
__global__ void k_fwd_rows(int n, long long ld, const T *A, int k0, int kb, int k1, T *b) {
    int i = k1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T acc = 0;
    for (int c = 0; c < kb; c++) acc += A[(long long)i * ld + k0 + c] * b[k0 + c];
    b[i] -= acc;
}

template <typename T>
struct LdltWork {
    T *dvec, *W, *s;
};

template <typename T>
int ldlt_factor_solve(mp_ctx *ctx, T *A, long long ld, int n, T *b, LdltWork<T> w, bool factor) {
    cudaStream_t st = ctx->stream;
    size_t panel_smem = sizeof(T) * (NB * NB + 64 * (NB + 1));
    size_t upd_smem = sizeof(T) * 2 * NB * 68;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_ldlt_panel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 80 * 1024);
        cudaFuncSetAttribute(k_ldlt_panel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 80 * 1024);
        cudaFuncSetAttribute(k_ldlt_update<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 80 * 1024);
        cudaFuncSetAttribute(k_ldlt_update<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 80 * 1024);
        attr = true;
    }
    if (factor) {
        for (int k0 = 0; k0 < n; k0 += NB) {
            int kb = n - k0 < NB ? n - k0 : NB;
            int k1 = k0 + kb;
            k_ldlt_diag<T><<<1, 256, 0, st>>>(n, ld, A, k0, kb, w.dvec, b, ctx->counters + C_FLAGS), ++ctx->launches;
            if (k1 < n) {
                int rows = n - k1;
                k_ldlt_panel<T><<<(rows + 63) / 64, 256, panel_smem, st>>>(n, ld, A, k0, kb, w.dvec, w.W, b), ++ctx->launches;
                long long tiles = (rows + 63) / 64;
                long long nblk = tiles * (tiles + 1) / 2;
                k_ldlt_update<T><<<(unsigned)nblk, 256, upd_smem, st>>>(n, ld, A, k0, kb, w.W, k1), ++ctx->launches;
            }
        }
    } else {
        // forward substitution with an existing factor
        for (int k0 = 0; k0 < n; k0 += NB) {
            int kb = n - k0 < NB ? n - k0 : NB;
            int k1 = k0 + kb;
            // z_k = L_kk^-1 b_k, then b_i -= L_ik z_k
            k_fwd_diag<T><<<1, 64, 0, st>>>(ld, A, k0, kb, b), ++ctx->launches;
            if (k1 < n) k_fwd_rows<T><<<(n - k1 + 255) / 256, 256, 0, st>>>(n, ld, A, k0, kb, k1, b), ++ctx->launches;
        }
    }
    k_diag_scale<T><<<(n + 255) / 256, 256, 0, st>>>(n, w.dvec, b), ++ctx->launches;
    MP_CUDA(ctx, cudaMemsetAsync(w.s, 0, sizeof(T) * NB, st));
    int last = ((n - 1) / NB) * NB;
    for (int k0 = last; k0 >= 0; k0 -= NB) {
        int kb = n - k0 < NB ? n - k0 : NB;
        int k1 = k0 + kb;
        if (k1 < n) {
            int rows = n - k1;
            int grid = (rows + 3) / 4;
            if (grid > ctx->sm_count * 4) grid = ctx->sm_count * 4;
            k_bwd_partial<T><<<grid, 256, 0, st>>>(n, ld, A, k0, kb, k1, b, w.s), ++ctx->launches;
        }
        k_bwd_diag<T><<<1, 64, 0, st>>>(ld, A, k0, kb, b, w.s), ++ctx->launches;
    }
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

}  // namespace mp
