// Dense symmetric factorization J = L D L^T of the Newton Jacobian and the
// solve J y = G, replacing the reference's LAPACK dsysv_ call
// (FESolver::solveLinearLapack, src/FESolver.cpp:528-558).
//
// Blocked right-looking LDL^T without pivoting on the lower triangle (row-major
// storage, leading dimension padded to 32).  Per block column k of width NB:
//   diag   : L_kk D_k L_kk^T = A_kk in registers (one CTA); z_k = L_kk^-1 b_k
//   panel  : W_ik = A_ik L_kk^-T,  L_ik = W_ik D_k^-1, b_i -= L_ik z_k  (rows below)
//   update : A_ij -= L_ik W_jk^T on the lower tiles of the trailing matrix,
//            two-level: within each 256-wide outer panel only the panel's own
//            columns (mma.sync tiles, the next diagonal factor riding along),
//            the rest of its 1,024-wide super-panel once per panel, and the
//            trailing matrix once per super-panel (tcgen05 for the FP32 factor,
//            FP64 mma.sync for the FP64 one)
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
constexpr int MS = NB + 4;  // row pitch of shared 64-wide blocks: a warp's quad or fragment reads hit all banks

template <typename T>
__device__ __forceinline__ bool bad_pivot(T d) {
    return !(fabs((double)d) > 0.0) || !isfinite((double)d);
}

// The factorization's 64-wide chain (diagonal factor, panel, in-panel column
// update) goes out as programmatic dependent launches: a kernel lets the next
// one be scheduled as soon as all of its own CTAs are running, and waits for
// the previous kernel's completion and memory before it touches any data, so
// the next kernel's CTAs are resident when the previous one ends.
__device__ __forceinline__ void chain_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// 4 consecutive values (16-byte aligned for float, 32 for double) as vector loads
template <typename T>
__device__ __forceinline__ void load4p(const T *p, T *v) {
    if constexpr (sizeof(T) == 8) {
        const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
        const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    } else {
        const float4 a = __ldg(reinterpret_cast<const float4 *>(p));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
}

// Factor the kb x kb diagonal block at (k0,k0): L (strict lower) and D written
// back, and Linv = L_kk^-1 (unit lower, row-major NB x NB, zero outside kb x kb)
// for the panel and the triangular solves.  If b is non-null,
// z_k = L_kk^-1 b_k (the forward substitution riding on the factorization).
// The block is padded to 64 x 64 with an identity.
//
// The block and its inverse live in registers: thread (ti, tc) of 256 holds
// the 4 x 4 tiles at rows 4ti.., columns 4tc.. of the block and of Linv (and,
// for tc == 0, b at rows 4ti..).  Step jj eliminates the four pivots j0 = 4jj
// .. j0+3 behind one barrier:
//   publish   the owners of the step's four columns (tc == jj) put them in
//             shared memory, the owners of Linv's rows j0.. (ti == jj) those
//             rows and b_j0.., and the owner of the 4 x 4 pivot block (ti ==
//             tc == jj) factors it, P = L_P D_P L_P^T, and publishes L_P, D_P
//             and 1/D_P;
//   eliminate every thread forms, for its rows i > j0+3, z_i = L_P^-1 x_i from
//             the row's four column values x_i and the multipliers
//             l_im = z_im / d_m, and for its columns c the same z_c; its
//             tile takes the rank-4 update A_ic -= sum_m l_im z_cm; the four
//             Linv rows become L_P^-1 (rows) and every later row subtracts
//             sum_m l_im (that row m); b likewise.  The owners of the step's
//             columns keep l_im there (L), the pivot owner L_P and D_P.
// The steps run as a dataflow, not in lock step: every step has its own
// shared-memory buffers and an mbarrier.  A warp holds two column tiles of all
// row tiles, so the publishers of step jj are warps 0 .. jj/2 (the columns,
// the pivot, Linv's rows and b); each of their lanes arrives on the step's
// mbarrier after its writes, and every thread waits on it before it
// eliminates.  A warp publishes step jj only after eliminating step jj-1, so
// the chain from one pivot to the next runs through the warp that owns the
// next column while the other warps' updates trail behind, instead of the
// whole CTA meeting at a barrier every step.  Waits are bounded (a wait that
// gives up raises FLAG_LOOKBACK_TIMEOUT).
template <typename T>
__device__ __forceinline__ void ld4s(const T *p, T (&v)[4]) {
    if constexpr (sizeof(T) == 8) {
        const double2 x = reinterpret_cast<const double2 *>(p)[0], y = reinterpret_cast<const double2 *>(p)[1];
        v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
    } else {
        const float4 x = *reinterpret_cast<const float4 *>(p);
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    }
}
template <typename T>
__device__ __forceinline__ void st4s(T *p, const T (&v)[4]) {
    if constexpr (sizeof(T) == 8) {
        reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
    } else {
        *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
}

// One step's published data.
template <typename T>
struct __align__(16) DiagStep {
    T col[NB][4];  // the step's four columns, every row
    T row[4][NB];  // Linv's rows j0 .. j0+3, every column
    T piv[4][4];   // the factored pivot block: L_P below the diagonal, D_P on it
    T rd[4];       // 1 / D_P
    T bp[4];       // b_j0 .. b_j0+3
};
// shared scratch of diag_block: the 16 steps' buffers, then their mbarriers
template <typename T>
__host__ __device__ constexpr size_t diag_scratch() {
    return (size_t)(NB / 4) * sizeof(DiagStep<T>) + (NB / 4) * sizeof(unsigned long long);
}
constexpr long long DIAG_SPIN_LIMIT = 1ll << 22;

// The block is read with coherent loads, or from stile (shared memory, row
// pitch MS) where the chain step that has just updated it hands it over.
// scratch: diag_scratch<T>() bytes of shared memory, 16-byte aligned.  All 256
// threads of the CTA call it.
template <typename T>
__device__ __forceinline__ void diag_block(int n, long long ld, T *A, int k0, int kb, T *dvec, T *Linv, T *b,
                                           unsigned long long *flags, unsigned char *scratch,
                                           const T *stile = nullptr) {
    DiagStep<T> *steps = reinterpret_cast<DiagStep<T> *>(scratch);
    unsigned long long *pub = reinterpret_cast<unsigned long long *>(steps + NB / 4);
    // a warp holds two column tiles (tc) of all 16 row tiles (ti), so the
    // column-dependent branches of a step (update the block, or Linv) are
    // uniform over a warp
    const int t = threadIdx.x, ti = t & 15, tc = t >> 4;
    T a[4][4], li[4][4], bb[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int r = 4 * ti + u;
        const T *row = A + (long long)(k0 + r) * ld + k0 + 4 * tc;
        T v4[4] = {T(0), T(0), T(0), T(0)};
        if (r < kb) {
#pragma unroll
            for (int v = 0; v < 4; v++)
                if (4 * tc + v < kb) v4[v] = stile ? stile[r * MS + 4 * tc + v] : __ldcg(row + v);
        }
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int c = 4 * tc + v;
            a[u][v] = r < kb ? (c <= r ? v4[v] : T(0)) : (r == c ? T(1) : T(0));
            li[u][v] = r == c ? T(1) : T(0);
        }
        bb[u] = (b && tc == 0 && r < kb) ? __ldcg(&b[k0 + r]) : T(0);
    }
    if (t == 0)
        for (int jj = 0; jj < NB / 4; jj++) mp::tc::mbar_init(&pub[jj], 32 * (jj / 2 + 1));
    __syncthreads();
    bool singular = false, stalled = false;
    for (int jj = 0; jj < NB / 4; jj++) {
        DiagStep<T> &S = steps[jj];
        // ---- publish ----
        if (tc == jj) {
#pragma unroll
            for (int u = 0; u < 4; u++) st4s<T>(S.col[4 * ti + u], a[u]);
            if (ti == jj) {
                T P[4][4], rd[4];
#pragma unroll
                for (int m = 0; m < 4; m++)
#pragma unroll
                    for (int c = 0; c < 4; c++) P[m][c] = a[m][c];
#pragma unroll
                for (int m = 0; m < 4; m++) {
                    T d = P[m][m];
                    if (bad_pivot(d)) {
                        singular = true;
                        d = T(1);
                    }
                    rd[m] = T(1) / d;
                    T w[4];
#pragma unroll
                    for (int r = 0; r < 4; r++) w[r] = P[r][m];
#pragma unroll
                    for (int r = m + 1; r < 4; r++) {
                        const T l = w[r] * rd[m];
#pragma unroll
                        for (int c = m + 1; c <= r; c++) P[r][c] = fma(-l, w[c], P[r][c]);
                        P[r][m] = l;
                    }
                }
#pragma unroll
                for (int m = 0; m < 4; m++) st4s<T>(S.piv[m], P[m]);
                st4s<T>(S.rd, rd);
            }
        }
        if (ti == jj) {
#pragma unroll
            for (int m = 0; m < 4; m++) st4s<T>(&S.row[m][4 * tc], li[m]);
            if (tc == 0) st4s<T>(S.bp, bb);
        }
        if ((t >> 5) <= jj / 2) mp::tc::mbar_arrive(&pub[jj]);  // this warp's part of step jj is written
        for (long long i = 0; !stalled && !mp::tc::mbar_try(&pub[jj], 0); i++)
            if (i > DIAG_SPIN_LIMIT) stalled = true;
        // ---- eliminate ----
        T lp[4][4], rd[4];
#pragma unroll
        for (int m = 0; m < 4; m++) ld4s<T>(S.piv[m], lp[m]);
        ld4s<T>(S.rd, rd);
        // z = L_P^-1 x (L_P unit lower, from lp's strict lower part)
        auto fwd = [&](const T (&x)[4], T (&z)[4]) {
            z[0] = x[0];
            z[1] = fma(-z[0], lp[1][0], x[1]);
            z[2] = fma(-z[1], lp[2][1], fma(-z[0], lp[2][0], x[2]));
            z[3] = fma(-z[2], lp[3][2], fma(-z[1], lp[3][1], fma(-z[0], lp[3][0], x[3])));
        };
        const bool rowact = ti > jj;
        T L[4][4];
        if (rowact) {
#pragma unroll
            for (int u = 0; u < 4; u++) {
                T x[4], z[4];
                ld4s<T>(S.col[4 * ti + u], x);
                fwd(x, z);
#pragma unroll
                for (int m = 0; m < 4; m++) L[u][m] = z[m] * rd[m];
            }
            if (tc > jj) {
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    T x[4], z[4];
                    ld4s<T>(S.col[4 * tc + v], x);
                    fwd(x, z);
#pragma unroll
                    for (int u = 0; u < 4; u++)
#pragma unroll
                        for (int m = 0; m < 4; m++) a[u][v] = fma(-L[u][m], z[m], a[u][v]);
                }
            }
        }
        if (tc <= jj) {  // Linv's rows j0.. are zero right of column j0+3
            T R[4][4];
#pragma unroll
            for (int m = 0; m < 4; m++) ld4s<T>(&S.row[m][4 * tc], R[m]);
#pragma unroll
            for (int v = 0; v < 4; v++) {
                R[1][v] = fma(-R[0][v], lp[1][0], R[1][v]);
                R[2][v] = fma(-R[1][v], lp[2][1], fma(-R[0][v], lp[2][0], R[2][v]));
                R[3][v] = fma(-R[2][v], lp[3][2], fma(-R[1][v], lp[3][1], fma(-R[0][v], lp[3][0], R[3][v])));
            }
            if (rowact) {
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int v = 0; v < 4; v++)
#pragma unroll
                        for (int m = 0; m < 4; m++) li[u][v] = fma(-L[u][m], R[m][v], li[u][v]);
            } else if (ti == jj) {
#pragma unroll
                for (int m = 0; m < 4; m++)
#pragma unroll
                    for (int v = 0; v < 4; v++) li[m][v] = R[m][v];
            }
        }
        if (tc == 0 && ti >= jj) {
            T x[4], z[4];
            ld4s<T>(S.bp, x);
            fwd(x, z);
            if (rowact) {
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int m = 0; m < 4; m++) bb[u] = fma(-L[u][m], z[m], bb[u]);
            } else {
#pragma unroll
                for (int m = 0; m < 4; m++) bb[m] = z[m];
            }
        }
        if (tc == jj) {
            if (rowact) {
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int m = 0; m < 4; m++) a[u][m] = L[u][m];
            } else if (ti == jj) {
#pragma unroll
                for (int m = 0; m < 4; m++)
#pragma unroll
                    for (int c = 0; c < 4; c++) a[m][c] = lp[m][c];
            }
        }
    }
    if (singular) atomicOr(flags, FLAG_SINGULAR);
    if (stalled) atomicOr(flags, FLAG_LOOKBACK_TIMEOUT);
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int r = 4 * ti + u;
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int c = 4 * tc + v;
            const bool in = r < kb && c < kb;
            if (in && c <= r) A[(long long)(k0 + r) * ld + k0 + c] = a[u][v];
            Linv[r * NB + c] = in ? li[u][v] : T(0);
        }
        if (r < kb) {
            if (ti == tc) dvec[k0 + r] = a[u][u];
            if (b && tc == 0) b[k0 + r] = bb[u];
        }
    }
}

// kout (or null): the first fused chain step's copy of column block k0 in rows
// [k0 + kb, jend), [rows][64] (see k_ldlt_step_tc); kb is then 64, so every
// 16-byte vector of a row is whole and aligned (ld a multiple of 32, k0 of 64).
template <typename T>
__global__ void __launch_bounds__(256) k_ldlt_diag(int n, long long ld, T *A, int k0, int kb, T *dvec, T *Linv,
                                                   T *b, unsigned long long *flags, T *kout, int jend) {
    chain_enter();
    extern __shared__ __align__(16) unsigned char smem_raw[];  // diag_scratch<T>()
    if (kout) {  // at most 3 x 64 rows of 64 values: every load issued before the stores
        const int k1 = k0 + kb, rows = jend - k1;
        constexpr int V = 16 / sizeof(T), PER = 3 * NB * NB / V / 256;  // 16-byte vectors a thread
        using Vec = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
        Vec v[PER];
#pragma unroll
        for (int i = 0; i < PER; i++) {
            const int idx = threadIdx.x + 256 * i, r = idx / (NB / V), c = (idx % (NB / V)) * V;
            if (r < rows && c < kb) v[i] = *reinterpret_cast<const Vec *>(A + (long long)(k1 + r) * ld + k0 + c);
        }
#pragma unroll
        for (int i = 0; i < PER; i++) {
            const int idx = threadIdx.x + 256 * i, r = idx / (NB / V), c = (idx % (NB / V)) * V;
            if (r < rows && c < kb) *reinterpret_cast<Vec *>(kout + (size_t)r * NB + c) = v[i];
        }
    }
    diag_block<T>(n, ld, A, k0, kb, dvec, Linv, b, flags, smem_raw);
}

// The next block's diagonal factor, run by the CTA of an in-panel column
// update that owns the next diagonal tile (grid tile (0, 0)) once that tile is
// stored: it overlaps the rest of the update and saves a launch per block.
struct NextDiag {
    int k0, kb;  // kb == 0: none
    void *dvec, *Linv, *b;
    unsigned long long *flags;
};
template <typename T>
__device__ __forceinline__ bool owns_next_diag(const NextDiag &nd) {
    return nd.kb > 0 && blockIdx.x == 0 && blockIdx.y == 0;
}
// stile: the updated tile in shared memory (row pitch MS), lower part;
// scratch: diag_scratch<T>() bytes of free shared memory
template <typename T>
__device__ __forceinline__ void fused_next_diag(int n, long long ld, T *A, const NextDiag &nd, const T *stile,
                                                unsigned char *scratch) {
    if (owns_next_diag<T>(nd)) {
        __syncthreads();  // the tile is complete in shared memory
        diag_block<T>(n, ld, A, nd.k0, nd.kb, static_cast<T *>(nd.dvec), static_cast<T *>(nd.Linv),
                      static_cast<T *>(nd.b), nd.flags, scratch, stile);
    }
}

// FP64 form: A[i][j] -= sum_{k<K} L[i][k] W[j][k] for rows/cols from R0, with
// L = A[i][K0 ...] and W rows of pitch ldw (K a multiple of 16).  colblocks = 0:
// the lower 128x128 tiles of [R0, n)^2 (the trailing update of a super-panel);
// colblocks > 0: every tile of rows [R0, n) x columns [R0, R0 + 128*colblocks)
// (a strip inside a super-panel), lower parts only.  K streams in 16-wide
// chunks through two shared-memory buffers stored k-major.
constexpr int WTILE = 128, WKC = 16;

// The update runs on the FP64 tensor cores (mma.sync m8n8k4, FP64 in and out,
// so the products and sums are FP64 operations).  Warp w
// takes rows 32(w/2) .. +31 and columns 64(w%2) .. +63 of the 128 x 128 tile:
// 4 x 8 MMA tiles of 8 x 8, 64 accumulators a thread.  Fragments of m8n8k4
// (g = lane / 4, t = lane % 4): A (row g, k t), B (k t, column g), C (row g,
// columns 2t, 2t+1).  The k-major shared operands have a pitch of WPITCH = 132
// doubles (132 = 4 mod 16), so a half-warp's fragment reads hit 16 distinct
// 8-byte banks.
constexpr int WPITCH = WTILE + 4;
__device__ __forceinline__ void dmma_8x8x4(double &c0, double &c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(256, 1) k_update_f64_mma(int n, long long ld, double *A, int K0, int K, int R0,
                                                           const double *__restrict__ W, int ldw, int colblocks) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double(*sL)[WKC][WPITCH] = reinterpret_cast<double(*)[WKC][WPITCH]>(smem_raw);
    double(*sW)[WKC][WPITCH] = sL + 2;
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
    const int t = threadIdx.x;
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
    const int w = t >> 5, lane = t & 31, g = lane >> 2, tq = lane & 3;
    const int wm0 = 32 * (w >> 1), wn0 = 64 * (w & 1);
    double acc[4][8][2];
#pragma unroll
    for (int mi = 0; mi < 4; mi++)
#pragma unroll
        for (int ni = 0; ni < 8; ni++) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
    fetch(0);
    stash(0);
    __syncthreads();
    const int NKC = K / WKC;
#pragma unroll 1
    for (int kc = 0; kc < NKC; kc++) {
        const int buf = kc & 1;
        if (kc + 1 < NKC) fetch(kc + 1);
#pragma unroll
        for (int k4 = 0; k4 < WKC; k4 += 4) {
            double a[4], b[8];
#pragma unroll
            for (int mi = 0; mi < 4; mi++) a[mi] = sL[buf][k4 + tq][wm0 + 8 * mi + g];
#pragma unroll
            for (int ni = 0; ni < 8; ni++) b[ni] = sW[buf][k4 + tq][wn0 + 8 * ni + g];
#pragma unroll
            for (int mi = 0; mi < 4; mi++)
#pragma unroll
                for (int ni = 0; ni < 8; ni++) dmma_8x8x4(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
        }
        if (kc + 1 < NKC) stash(buf ^ 1);
        __syncthreads();
    }
#pragma unroll
    for (int mi = 0; mi < 4; mi++) {
        const long long row = i0 + wm0 + 8 * mi + g;
        if (row >= n) continue;
#pragma unroll
        for (int ni = 0; ni < 8; ni++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const long long col = j0 + wn0 + 8 * ni + 2 * tq + e;
                if (col < n && col <= row) A[row * ld + col] -= acc[mi][ni][e];
            }
    }
}

// ---- triangular solves with an existing factor --------------------------------------
// One persistent cooperative launch per direction over 64-row blocks; CTA g
// takes blocks g, g+G, ... in solve order, so the lowest unsolved block always
// runs.  A solved block is published as low-latency words: each 8-byte word
// holds 32 bits of a value and the solve's epoch in its upper half, written and
// read as one relaxed gpu-scope 64-bit access (single-copy atomic), so a reader
// that sees the epoch holds the value -- one L2 round trip per block instead of
// a release flag followed by a load of the data.  One warp per CTA polls; the
// others wait at the block barrier.
//
// A block sums the contributions of every solved block except its nearest
// predecessor as they arrive (polling with a back-off that grows with its
// distance from the front), applies its diagonal block's stored inverse, and
// then waits for the predecessor alone, whose contribution is one 64 x 64
// product with a coupling block computed once per factorization:
//   forward  z_i = Linv_ii (b_i - sum_{j<i-1} L_ij z_j) - Mf_i z_{i-1},  Mf_i = Linv_ii L_{i,i-1}
//   backward y_i = Linv_ii^T (D_i^-1 z_i - sum_{j>i+1} L_ji^T y_j) - Mb_i y_{i+1},
//            Mb_i = Linv_ii^T L_{i+1,i}^T
// so a step of the chain is a poll, 16 multiply-adds a thread, two shuffles and
// a store.  Waits are bounded (TRSV_SPIN_LIMIT empty polls); a wait that gives
// up sets the error flag and the block publishes what it has, so no other
// block waits on it for long.
constexpr long long TRSV_SPIN_LIMIT = 1ll << 20;

__device__ __forceinline__ void st_ll(unsigned long long *p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_ll(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Words of block `blk`: FP32 one per value ([blk][64]); FP64 two, the low and
// high halves in two planes ([blk][2][64]).
template <typename T>
__device__ __forceinline__ void ll_put(unsigned long long *ll, int blk, int r, T v, unsigned epoch) {
    const unsigned long long e = (unsigned long long)epoch << 32;
    if constexpr (sizeof(T) == 4) {
        st_ll(ll + (size_t)blk * NB + r, e | __float_as_uint(v));
    } else {
        const unsigned long long b = (unsigned long long)__double_as_longlong(v);
        unsigned long long *p = ll + (size_t)blk * 2 * NB;
        st_ll(p + r, e | (b & 0xffffffffull));
        st_ll(p + NB + r, e | (b >> 32));
    }
}

// One poll of block c's 64 values by a whole warp; true (warp-uniform) when all
// carry `epoch`, and then they are in dst[0..63].
template <typename T>
__device__ __forceinline__ bool ll_try(const unsigned long long *ll, int c, unsigned epoch, T *dst) {
    const int lane = threadIdx.x & 31;
    if constexpr (sizeof(T) == 4) {
        const unsigned long long *p = ll + (size_t)c * NB;
        const unsigned long long w0 = ld_ll(p + lane), w1 = ld_ll(p + 32 + lane);
        const bool ok = (unsigned)(w0 >> 32) == epoch && (unsigned)(w1 >> 32) == epoch;
        if (!__all_sync(0xffffffffu, ok)) return false;
        dst[lane] = __uint_as_float((unsigned)w0);
        dst[lane + 32] = __uint_as_float((unsigned)w1);
    } else {
        const unsigned long long *p = ll + (size_t)c * 2 * NB;
        const unsigned long long l0 = ld_ll(p + lane), l1 = ld_ll(p + 32 + lane);
        const unsigned long long h0 = ld_ll(p + NB + lane), h1 = ld_ll(p + NB + 32 + lane);
        const bool ok = (unsigned)(l0 >> 32) == epoch && (unsigned)(l1 >> 32) == epoch &&
                        (unsigned)(h0 >> 32) == epoch && (unsigned)(h1 >> 32) == epoch;
        if (!__all_sync(0xffffffffu, ok)) return false;
        dst[lane] = __longlong_as_double((long long)((h0 << 32) | (l0 & 0xffffffffull)));
        dst[lane + 32] = __longlong_as_double((long long)((h1 << 32) | (l1 & 0xffffffffull)));
    }
    return true;
}

// All threads call it: warp 0 polls block c into dst (sleeping `backoff` ns
// between empty polls), then the CTA meets at a barrier.  Returns false (and
// raises the error flag) when the wait gave up.  `ok` is a shared slot that
// alternates with dst, so a slot is rewritten only after every thread has
// passed the next barrier.
template <typename T>
__device__ __forceinline__ bool wait_chunk(const unsigned long long *ll, int c, unsigned epoch, T *dst, int backoff,
                                           int *ok, unsigned long long *flags) {
    if (threadIdx.x < 32) {
        bool got = false;
        for (long long spins = 0; spins <= TRSV_SPIN_LIMIT; spins++) {
            if (ll_try<T>(ll, c, epoch, dst)) {
                got = true;
                break;
            }
            if (backoff) __nanosleep(backoff);
        }
        if (threadIdx.x == 0) {
            *ok = got ? 1 : 0;
            if (!got) atomicOr(flags, FLAG_LOOKBACK_TIMEOUT);
        }
    }
    __syncthreads();
    return *ok != 0;
}

// wait_chunk for up to gmax consecutive blocks c, c + dir, ...: warp 0 waits
// for block c, then takes the following blocks that are already published
// (one poll each) into dst + i*NB; returns how many it took (0: the wait gave
// up).  Behind the front, where the blocks were published long ago, one
// barrier then covers several blocks.
template <typename T>
__device__ __forceinline__ int wait_chunks(const unsigned long long *ll, int c, int dir, int gmax, unsigned epoch,
                                           T *dst, int backoff, int *cnt, unsigned long long *flags) {
    if (threadIdx.x < 32) {
        int got = 0;
        for (long long spins = 0; spins <= TRSV_SPIN_LIMIT; spins++) {
            if (ll_try<T>(ll, c, epoch, dst)) {
                got = 1;
                break;
            }
            if (backoff) __nanosleep(backoff);
        }
        if (got)
            while (got < gmax && ll_try<T>(ll, c + dir * got, epoch, dst + got * NB)) got++;
        if (threadIdx.x == 0) {
            *cnt = got;
            if (!got) atomicOr(flags, FLAG_LOOKBACK_TIMEOUT);
        }
    }
    __syncthreads();
    return *cnt;
}
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// The chain's critical wait: every warp polls block c's words itself, so no
// CTA barrier follows; this lane gets values lane (v0) and lane + 32 (v1).  A
// wait that gives up raises the error flag and leaves zeros (the caller's
// control flow does not depend on it, so every warp takes the same barriers).
template <typename T>
__device__ __forceinline__ void wait_warp(const unsigned long long *ll, int c, unsigned epoch, T &v0, T &v1,
                                          unsigned long long *flags) {
    const int lane = threadIdx.x & 31;
    for (long long spins = 0; spins <= TRSV_SPIN_LIMIT; spins++) {
        if constexpr (sizeof(T) == 4) {
            const unsigned long long *p = ll + (size_t)c * NB;
            const unsigned long long w0 = ld_ll(p + lane), w1 = ld_ll(p + 32 + lane);
            const bool ok = (unsigned)(w0 >> 32) == epoch && (unsigned)(w1 >> 32) == epoch;
            if (__all_sync(0xffffffffu, ok)) {
                v0 = __uint_as_float((unsigned)w0);
                v1 = __uint_as_float((unsigned)w1);
                return;
            }
        } else {
            const unsigned long long *p = ll + (size_t)c * 2 * NB;
            const unsigned long long l0 = ld_ll(p + lane), l1 = ld_ll(p + 32 + lane);
            const unsigned long long h0 = ld_ll(p + NB + lane), h1 = ld_ll(p + NB + 32 + lane);
            const bool ok = (unsigned)(l0 >> 32) == epoch && (unsigned)(l1 >> 32) == epoch &&
                            (unsigned)(h0 >> 32) == epoch && (unsigned)(h1 >> 32) == epoch;
            if (__all_sync(0xffffffffu, ok)) {
                v0 = __longlong_as_double((long long)((h0 << 32) | (l0 & 0xffffffffull)));
                v1 = __longlong_as_double((long long)((h1 << 32) | (l1 & 0xffffffffull)));
                return;
            }
        }
    }
    v0 = v1 = T(0);
    if (lane == 0) atomicOr(flags, FLAG_LOOKBACK_TIMEOUT);
}

// value 4k + q of a block held across the warp as (v0, v1) by wait_warp
template <typename T, int K>
__device__ __forceinline__ T warp_value(T v0, T v1, int q) {
    return __shfl_sync(0xffffffffu, K < 8 ? v0 : v1, (4 * K + q) & 31);
}

// sleep between empty polls for a block `dist` steps from the one it waits on
__device__ __forceinline__ int poll_backoff(int dist) { return dist > 8 ? 512 : 64 * dist; }

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


// Shared memory of k_trsv_ll: inverse and coupling blocks, partial sums, two
// poll buffers, the right-hand side, two poll results.
template <typename T>
constexpr size_t trsv_smem() {
    return sizeof(T) * (2 * NB * MS + 16 * (NB + 1) + 3 * NB) + 2 * sizeof(int);
}

// DIR = +1: L z = b (unit lower, in place on x); DIR = -1: L^T y = D^-1 z (in
// place on x).  Mc holds the direction's coupling blocks; ll its words.
template <typename T, int DIR>
__global__ void __launch_bounds__(256) k_trsv_ll(int n, long long ld, const T *__restrict__ A,
                                                 const T *__restrict__ Linv, const T *__restrict__ Mc,
                                                 const T *__restrict__ dvec, T *x, unsigned long long *ll,
                                                 unsigned epoch, unsigned long long *flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T(*sI)[MS] = reinterpret_cast<T(*)[MS]>(smem_raw);
    T(*sC)[MS] = sI + NB;
    T(*spart)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(sC + NB);
    T *sx = reinterpret_cast<T *>(spart + 16);  // [2][NB]
    T *srhs = sx + 2 * NB;
    int *sok = reinterpret_cast<int *>(srhs + NB);  // [2]
    const int nblk = (n + NB - 1) / NB;
    const int t = threadIdx.x;
    const int r = t >> 2, q = t & 3;       // forward sums and the chain step: row r, columns 4k + q / 16q + k
    const int c4 = t & 15, part = t >> 4;  // backward sums: columns 4c4 .. +3, chunk rows 4part .. +3
    int par = 0;
    for (int g = blockIdx.x; g < nblk; g += gridDim.x) {
        const int blk = DIR > 0 ? g : nblk - 1 - g;
        const int r0 = blk * NB, kb = n - r0 < NB ? n - r0 : NB;
        const int pred = blk - DIR;
        const bool has_pred = pred >= 0 && pred < nblk;
        for (int idx = t; idx < NB * NB; idx += 256) {
            sI[idx >> 6][idx & 63] = __ldg(&Linv[(size_t)blk * NB * NB + idx]);
            sC[idx >> 6][idx & 63] = has_pred ? __ldg(&Mc[(size_t)blk * NB * NB + idx]) : T(0);
        }
        // this block's right-hand side is no other block's output: read it before any wait
        if (t < NB) srhs[t] = t < kb ? (DIR > 0 ? __ldcg(&x[r0 + t]) : __ldcg(&x[r0 + t]) / dvec[r0 + t]) : T(0);
        // far blocks: forward 0 .. blk-2, backward nblk-1 .. blk+2
        const int nfar = DIR > 0 ? (blk > 1 ? blk - 1 : 0) : (nblk - 2 - blk > 0 ? nblk - 2 - blk : 0);
        T acc = 0, acc4[4] = {0, 0, 0, 0}, ap[16];
        auto fetch = [&](int j) {
            if (DIR > 0) {
                if (r < kb) {
                    load16<T, false>(A + (long long)(r0 + r) * ld + j * NB + q * 16, ap);
                } else {
#pragma unroll
                    for (int k = 0; k < 16; k++) ap[k] = T(0);
                }
            } else {
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int i = j * NB + 4 * part + e;
                    if (i < n) {
                        load4p<T>(A + (long long)i * ld + r0 + 4 * c4, ap + 4 * e);
                    } else {
#pragma unroll
                        for (int k = 0; k < 4; k++) ap[4 * e + k] = T(0);
                    }
                }
            }
        };
        bool ok = true;
        if (nfar > 0) fetch(DIR > 0 ? 0 : nblk - 1);
        for (int s = 0; s < nfar; s++) {
            const int j = DIR > 0 ? s : nblk - 1 - s;
            T *buf = sx + par * NB;
            ok = wait_chunk<T>(ll, j, epoch, buf, poll_backoff(nfar - s), sok + par, flags);
            par ^= 1;
            if (!ok) break;
            if (DIR > 0) {
#pragma unroll
                for (int k = 0; k < 16; k++) acc = fma(ap[k], buf[q * 16 + k], acc);
            } else {
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const T xe = buf[4 * part + e];
#pragma unroll
                    for (int k = 0; k < 4; k++) acc4[k] = fma(ap[4 * e + k], xe, acc4[k]);
                }
            }
            if (s + 1 < nfar) fetch(DIR > 0 ? j + 1 : j - 1);
        }
        if (DIR > 0) {
            acc += __shfl_xor_sync(0xffffffffu, acc, 1);
            acc += __shfl_xor_sync(0xffffffffu, acc, 2);
            if (q == 0) spart[0][r] = acc;
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) spart[part][4 * c4 + k] = acc4[k];
        }
        __syncthreads();
        if (t < NB) {
            T sum = 0;
            if (DIR > 0) {
                sum = spart[0][t];
            } else {
#pragma unroll
                for (int p = 0; p < 16; p++) sum += spart[p][t];
            }
            srhs[t] -= sum;
        }
        __syncthreads();
        // y = Linv srhs (forward) or Linv^T srhs (backward), row r split over the quad
        T y = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const int c = 4 * k + q;
            y = fma(DIR > 0 ? sI[r][c] : sI[c][r], srhs[c], y);
        }
        y += __shfl_xor_sync(0xffffffffu, y, 1);
        y += __shfl_xor_sync(0xffffffffu, y, 2);
        // the chain step: the nearest predecessor through the coupling block
        T xr = y;
        if (has_pred && ok) {
            T p0, p1;
            wait_warp<T>(ll, pred, epoch, p0, p1, flags);
            T v = 0;
#define MP_STEP(K) v = fma(sC[r][4 * K + q], warp_value<T, K>(p0, p1, q), v);
            MP_STEP(0) MP_STEP(1) MP_STEP(2) MP_STEP(3) MP_STEP(4) MP_STEP(5) MP_STEP(6) MP_STEP(7)
            MP_STEP(8) MP_STEP(9) MP_STEP(10) MP_STEP(11) MP_STEP(12) MP_STEP(13) MP_STEP(14) MP_STEP(15)
#undef MP_STEP
            v += __shfl_xor_sync(0xffffffffu, v, 1);
            v += __shfl_xor_sync(0xffffffffu, v, 2);
            xr = y - v;
        }
        if (q == 0) {
            ll_put<T>(ll, blk, r, r < kb ? xr : T(0), epoch);
            if (r < kb) x[r0 + r] = xr;
        }
        __syncthreads();  // shared memory is reused by this CTA's next block
    }
}

// ---- banded wavefront solves -----------------------------------------------------------
// The same solves with each CTA owning a band of two consecutive blocks in
// solve order, b1 then b2, so the step from b1 to b2 is a block barrier inside
// the CTA and only every second step of the chain crosses SMs.  With p the
// block before b1 in solve order, C1 / C2 the direction's coupling blocks at
// distance 1 and 2 (k_trsv_couplings) and y_b the block's inverse (forward
// Linv, backward Linv^T) applied to its right-hand side less the blocks before
// p, which the band sums as they are published:
//   x_b1 = y_b1 - C1_b1 x_p,    x_b2 = (y_b2 - C2_b2 x_p) - C1_b2 x_b1.
// Each band sums two blocks' rows per published chunk, so a band step asks
// twice the loads of its CTA; the banded form is used from 256 blocks on (16,384
// unknowns), where halving the chain's hops outweighs that.
// Shared memory: the two inverses, C1_b1, C2_b2, C1_b2 ([64][MS] each), the
// two blocks' partial sums, poll buffers, right-hand sides, x_b1.
constexpr int BAND_FROM_BLOCKS = 256;
// far blocks: up to BAND_GROUP published blocks a poll; L's rows of the block
// BAND_PREFETCH ahead of the one in registers are prefetched into L2 (L does not
// depend on the front, only the values do)
constexpr int BAND_GROUP = 4, BAND_PREFETCH = 4;
template <typename T>
constexpr size_t band_smem() {
    return sizeof(T) * (5 * NB * MS + 2 * 16 * (NB + 1) + (2 * BAND_GROUP + 3) * NB) + 2 * sizeof(int);
}

template <typename T, int DIR>
__global__ void __launch_bounds__(256, 2)
    k_trsv_band(int n, long long ld, const T *__restrict__ A, const T *__restrict__ Linv, const T *__restrict__ C1,
                const T *__restrict__ C2, const T *__restrict__ dvec, T *x, unsigned long long *ll, unsigned epoch,
                unsigned long long *flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T(*sI1)[MS] = reinterpret_cast<T(*)[MS]>(smem_raw);
    T(*sI2)[MS] = sI1 + NB;
    T(*sC11)[MS] = sI2 + NB;  // C1 of b1
    T(*sC22)[MS] = sC11 + NB;  // C2 of b2
    T(*sC12)[MS] = sC22 + NB;  // C1 of b2
    T(*spart)[16][NB + 1] = reinterpret_cast<T(*)[16][NB + 1]>(sC12 + NB);  // [2][16][65]
    T *sx = reinterpret_cast<T *>(spart + 2);                                // [2][BAND_GROUP][NB]
    T *srhs = sx + 2 * BAND_GROUP * NB;                                      // [2][NB]
    T *sx1 = srhs + 2 * NB;                                                  // [NB]
    int *sok = reinterpret_cast<int *>(sx1 + NB);                            // [2]
    const int nblk = (n + NB - 1) / NB, nband = (nblk + 1) / 2;
    const int t = threadIdx.x;
    const int r = t >> 2, q = t & 3;       // forward sums and the chain steps: row r
    const int c4 = t & 15, part = t >> 4;  // backward sums: columns 4c4 .. +3, chunk rows 4part .. +3
    int par = 0;
    for (int g = blockIdx.x; g < nband; g += gridDim.x) {
        const int b1 = DIR > 0 ? 2 * g : nblk - 1 - 2 * g, b2 = b1 + DIR, p = b1 - DIR;
        const bool two = b2 >= 0 && b2 < nblk, has_p = p >= 0 && p < nblk;
        const int r01 = b1 * NB, kb1 = n - r01 < NB ? n - r01 : NB;
        const int r02 = b2 * NB, kb2 = two ? (n - r02 < NB ? n - r02 : NB) : 0;
        for (int idx = t; idx < NB * NB; idx += 256) {
            const int rr = idx >> 6, cc = idx & 63;
            sI1[rr][cc] = __ldg(&Linv[(size_t)b1 * NB * NB + idx]);
            sC11[rr][cc] = has_p ? __ldg(&C1[(size_t)b1 * NB * NB + idx]) : T(0);
            sI2[rr][cc] = two ? __ldg(&Linv[(size_t)b2 * NB * NB + idx]) : T(0);
            sC22[rr][cc] = two && has_p ? __ldg(&C2[(size_t)b2 * NB * NB + idx]) : T(0);
            sC12[rr][cc] = two ? __ldg(&C1[(size_t)b2 * NB * NB + idx]) : T(0);
        }
        // the band's right-hand sides are no other block's output: read them before any wait
        if (t < 2 * NB) {
            const int h = t >> 6, rr = t & 63, kb = h ? kb2 : kb1, row = (h ? r02 : r01) + rr;
            T v = T(0);
            if (rr < kb) v = DIR > 0 ? __ldcg(&x[row]) : __ldcg(&x[row]) / dvec[row];
            srhs[t] = v;
        }
        // blocks before p: forward 0 .. b1-2, backward nblk-1 .. b1+2
        const int nfar = DIR > 0 ? (b1 > 1 ? b1 - 1 : 0) : (nblk - 2 - b1 > 0 ? nblk - 2 - b1 : 0);
        T acc1 = T(0), acc2 = T(0), a41[4] = {T(0), T(0), T(0), T(0)}, a42[4] = {T(0), T(0), T(0), T(0)};
        T ap1[16], ap2[16];
        auto fetch = [&](int j) {
            if (DIR > 0) {
                if (r < kb1) {
                    load16<T, false>(A + (long long)(r01 + r) * ld + j * NB + q * 16, ap1);
                } else {
#pragma unroll
                    for (int k = 0; k < 16; k++) ap1[k] = T(0);
                }
                if (r < kb2) {
                    load16<T, false>(A + (long long)(r02 + r) * ld + j * NB + q * 16, ap2);
                } else {
#pragma unroll
                    for (int k = 0; k < 16; k++) ap2[k] = T(0);
                }
            } else {
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int i = j * NB + 4 * part + e;
                    if (i < n) {
                        load4p<T>(A + (long long)i * ld + r01 + 4 * c4, ap1 + 4 * e);
                        if (two) {
                            load4p<T>(A + (long long)i * ld + r02 + 4 * c4, ap2 + 4 * e);
                        } else {
#pragma unroll
                            for (int k = 0; k < 4; k++) ap2[4 * e + k] = T(0);
                        }
                    } else {
#pragma unroll
                        for (int k = 0; k < 4; k++) ap1[4 * e + k] = ap2[4 * e + k] = T(0);
                    }
                }
            }
        };
        // the lines of L a thread will load for far block j, into L2
        auto prefetch = [&](int j) {
            if (DIR > 0) {
                if ((q & 1) == 0) {  // q = 0, 2: the row's two 128-byte lines
                    if (r < kb1) prefetch_l2(A + (long long)(r01 + r) * ld + j * NB + q * 16);
                    if (r < kb2) prefetch_l2(A + (long long)(r02 + r) * ld + j * NB + q * 16);
                }
            } else if ((c4 & 7) == 0) {  // c4 = 0, 8: each block's two lines of a row
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int i = j * NB + 4 * part + e;
                    if (i < n) {
                        prefetch_l2(A + (long long)i * ld + r01 + 4 * c4);
                        if (two) prefetch_l2(A + (long long)i * ld + r02 + 4 * c4);
                    }
                }
            }
        };
        bool ok = true;
        if (nfar > 0) fetch(DIR > 0 ? 0 : nblk - 1);
        for (int s = 1; s <= BAND_PREFETCH && s < nfar; s++) prefetch(DIR > 0 ? s : nblk - 1 - s);
        for (int s = 0; s < nfar;) {
            T *buf = sx + par * BAND_GROUP * NB;
            const int gmax = nfar - s < BAND_GROUP ? nfar - s : BAND_GROUP;
            const int m = wait_chunks<T>(ll, DIR > 0 ? s : nblk - 1 - s, DIR, gmax, epoch, buf,
                                         poll_backoff(nfar - s), sok + par, flags);
            par ^= 1;
            if (m == 0) {
                ok = false;
                break;
            }
            for (int u = 0; u < m; u++, s++) {
                const int j = DIR > 0 ? s : nblk - 1 - s;
                const T *xb = buf + u * NB;
                if (DIR > 0) {
#pragma unroll
                    for (int k = 0; k < 16; k++) {
                        const T xv = xb[q * 16 + k];
                        acc1 = fma(ap1[k], xv, acc1);
                        acc2 = fma(ap2[k], xv, acc2);
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const T xe = xb[4 * part + e];
#pragma unroll
                        for (int k = 0; k < 4; k++) {
                            a41[k] = fma(ap1[4 * e + k], xe, a41[k]);
                            a42[k] = fma(ap2[4 * e + k], xe, a42[k]);
                        }
                    }
                }
                if (s + 1 < nfar) fetch(DIR > 0 ? j + 1 : j - 1);
                if (s + 1 + BAND_PREFETCH < nfar) prefetch(DIR > 0 ? j + 1 + BAND_PREFETCH : j - 1 - BAND_PREFETCH);
            }
        }
        if (DIR > 0) {
            acc1 += __shfl_xor_sync(0xffffffffu, acc1, 1);
            acc1 += __shfl_xor_sync(0xffffffffu, acc1, 2);
            acc2 += __shfl_xor_sync(0xffffffffu, acc2, 1);
            acc2 += __shfl_xor_sync(0xffffffffu, acc2, 2);
            if (q == 0) {
                spart[0][0][r] = acc1;
                spart[1][0][r] = acc2;
            }
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                spart[0][part][4 * c4 + k] = a41[k];
                spart[1][part][4 * c4 + k] = a42[k];
            }
        }
        __syncthreads();
        if (t < 2 * NB) {
            const int h = t >> 6, rr = t & 63;
            T sum = T(0);
            if (DIR > 0) {
                sum = spart[h][0][rr];
            } else {
#pragma unroll
                for (int pp = 0; pp < 16; pp++) sum += spart[h][pp][rr];
            }
            srhs[t] -= sum;
        }
        __syncthreads();
        T y1 = T(0), y2 = T(0);
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const int c = 4 * k + q;
            y1 = fma(DIR > 0 ? sI1[r][c] : sI1[c][r], srhs[c], y1);
            y2 = fma(DIR > 0 ? sI2[r][c] : sI2[c][r], srhs[NB + c], y2);
        }
        y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
        y2 += __shfl_xor_sync(0xffffffffu, y2, 1);
        y2 += __shfl_xor_sync(0xffffffffu, y2, 2);
        // the chain: p crosses SMs, b1 -> b2 stays in the CTA
        T x1 = y1, t2 = y2;
        if (has_p && ok) {
            T p0, p1;
            wait_warp<T>(ll, p, epoch, p0, p1, flags);
            T v1 = T(0), v2 = T(0);
#define MP_STEP(K)                                       \
    {                                                    \
        const T xv = warp_value<T, K>(p0, p1, q);        \
        v1 = fma(sC11[r][4 * K + q], xv, v1);            \
        v2 = fma(sC22[r][4 * K + q], xv, v2);            \
    }
            MP_STEP(0) MP_STEP(1) MP_STEP(2) MP_STEP(3) MP_STEP(4) MP_STEP(5) MP_STEP(6) MP_STEP(7)
            MP_STEP(8) MP_STEP(9) MP_STEP(10) MP_STEP(11) MP_STEP(12) MP_STEP(13) MP_STEP(14) MP_STEP(15)
#undef MP_STEP
            v1 += __shfl_xor_sync(0xffffffffu, v1, 1);
            v1 += __shfl_xor_sync(0xffffffffu, v1, 2);
            v2 += __shfl_xor_sync(0xffffffffu, v2, 1);
            v2 += __shfl_xor_sync(0xffffffffu, v2, 2);
            x1 = y1 - v1;
            t2 = y2 - v2;
        }
        if (q == 0) {
            ll_put<T>(ll, b1, r, r < kb1 ? x1 : T(0), epoch);
            if (r < kb1) x[r01 + r] = x1;
            sx1[r] = r < kb1 ? x1 : T(0);
        }
        if (two) {
            __syncthreads();
            T v3 = T(0);
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const int c = 4 * k + q;
                v3 = fma(sC12[r][c], sx1[c], v3);
            }
            v3 += __shfl_xor_sync(0xffffffffu, v3, 1);
            v3 += __shfl_xor_sync(0xffffffffu, v3, 2);
            const T x2 = t2 - v3;
            if (q == 0) {
                ll_put<T>(ll, b2, r, r < kb2 ? x2 : T(0), epoch);
                if (r < kb2) x[r02 + r] = x2;
            }
        }
        __syncthreads();  // shared memory is reused by this CTA's next band
    }
}

// Coupling blocks of the wavefront solves, one CTA per block, at block
// distance d: Mf_i = Linv_ii L_{i,i-d} (i >= d) and, when Mb is given,
// Mb_i = Linv_ii^T L_{i+d,i}^T (i < nblk-d).  With skip_tiny, rows of
// L_{i,i-d} whose diagonal entry of A has magnitude below 1e-12 count as zero
// (the Gauss-Seidel sweep keeps those rows' values).  Dynamic smem: two
// [64][65] blocks.
template <typename T>
__global__ void __launch_bounds__(256) k_trsv_couplings(int n, long long ld, const T *__restrict__ A,
                                                        const T *__restrict__ Linv, T *Mf, T *Mb, int skip_tiny,
                                                        int dist) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T(*sI)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(smem_raw);
    T(*sL)[NB + 1] = sI + NB;
    const int nblk = (n + NB - 1) / NB, blk = blockIdx.x, r0 = blk * NB, t = threadIdx.x;
    const int tx = t & 15, ty = t >> 4;
    for (int idx = t; idx < NB * NB; idx += 256) sI[idx >> 6][idx & 63] = Linv[(size_t)blk * NB * NB + idx];
    if (blk >= dist) {
        for (int idx = t; idx < NB * NB; idx += 256) {
            const int rr = idx >> 6, cc = idx & 63, row = r0 + rr;
            bool keep = row < n;
            if (keep && skip_tiny) keep = fabs((double)A[(long long)row * ld + row]) >= 1e-12;
            sL[rr][cc] = keep ? A[(long long)row * ld + r0 - dist * NB + cc] : T(0);
        }
        __syncthreads();
        T acc[4][4] = {};
        for (int k = 0; k < NB; k++) {
            T a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; u++) a[u] = sI[4 * ty + u][k];
#pragma unroll
            for (int v = 0; v < 4; v++) b[v] = sL[k][4 * tx + v];
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < 4; v++) acc[u][v] = fma(a[u], b[v], acc[u][v]);
        }
        T *out = Mf + (size_t)blk * NB * NB;
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int v = 0; v < 4; v++) out[(4 * ty + u) * NB + 4 * tx + v] = acc[u][v];
        __syncthreads();
    }
    if (Mb && blk + dist < nblk) {
        for (int idx = t; idx < NB * NB; idx += 256) {
            const int rr = idx >> 6, cc = idx & 63, row = r0 + dist * NB + rr;
            sL[rr][cc] = row < n ? A[(long long)row * ld + r0 + cc] : T(0);
        }
        __syncthreads();
        T acc[4][4] = {};
        for (int k = 0; k < NB; k++) {
            T a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; u++) a[u] = sI[k][4 * ty + u];
#pragma unroll
            for (int v = 0; v < 4; v++) b[v] = sL[4 * tx + v][k];
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < 4; v++) acc[u][v] = fma(a[u], b[v], acc[u][v]);
        }
        T *out = Mb + (size_t)blk * NB * NB;
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int v = 0; v < 4; v++) out[(4 * ty + u) * NB + 4 * tx + v] = acc[u][v];
    }
}

// ---- tensor-core panels of the FP32 factor ----------------------------------------------
// The mixed form's panel products (W = A_ik Linv^T) and in-panel column updates
// (A_ij -= L_ik W_jk^T) are 64 x 64 x 64 products; they run on mma.sync
// m16n8k8 TF32 fragments with FP32 accumulation, in the same arithmetic as the
// trailing update: TERMS = 1 rounds each operand to TF32, TERMS = 3 splits it
// into hi = RN_tf32(x) and lo = RN_tf32(x - hi) and sums hi*hi + hi*lo + lo*hi.
// Operands sit in shared memory with a row pitch of MS = 68 floats, so the
// fragment reads of a warp (row 4g + t) hit 32 distinct banks.
__device__ __forceinline__ unsigned tf32_rn(float x) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void mma_m16n8k8(float (&c)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One warp: acc[nt] (16 x 8 tiles nt = 0..3, rows m0 + 0..15, columns n0 + 8nt
// + 0..7) += sum over k < 64 of sa[row][k] * sb[col][k].  Fragment layout of
// m16n8k8 (g = lane / 4, t = lane % 4): A a0 (g, t), a1 (g+8, t), a2 (g, t+4),
// a3 (g+8, t+4); B b0 (k = t, n = g), b1 (k = t+4, n = g); C c0 (g, 2t),
// c1 (g, 2t+1), c2 (g+8, 2t), c3 (g+8, 2t+1).
template <int TERMS>
__device__ __forceinline__ void warp_mma_64(const float (*sa)[MS], const float (*sb)[MS], int m0, int n0,
                                            float (&acc)[4][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll 2
    for (int k0 = 0; k0 < NB; k0 += 8) {
        const float af[4] = {sa[m0 + g][k0 + t], sa[m0 + g + 8][k0 + t], sa[m0 + g][k0 + t + 4],
                             sa[m0 + g + 8][k0 + t + 4]};
        unsigned ah[4], al[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            ah[i] = tf32_rn(af[i]);
            if (TERMS == 3) al[i] = tf32_rn(af[i] - __uint_as_float(ah[i]));
        }
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            const int c = n0 + 8 * nt + g;
            const float bf[2] = {sb[c][k0 + t], sb[c][k0 + t + 4]};
            unsigned bh[2], bl[2];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                bh[i] = tf32_rn(bf[i]);
                if (TERMS == 3) bl[i] = tf32_rn(bf[i] - __uint_as_float(bh[i]));
            }
            if (TERMS == 3) {
                mma_m16n8k8(acc[nt], al, bh);
                mma_m16n8k8(acc[nt], ah, bl);
            }
            mma_m16n8k8(acc[nt], ah, bh);
        }
    }
}

// One step of the 64-wide chain of the FP32 factor inside a 256-wide panel, in
// one launch: the panel of block k (rows [k1, n)), the in-panel column update
// of columns [k1, jend) and the diagonal factor of block k1.  CTA b takes the
// row block i0 = k1 + 64 b:
//   W_ik = A_ik Linv_k^T and L_ik = W_ik D_k^-1 (written over A_ik), b_i -= L_ik z_k;
//   A_ij -= L_ik W_jk^T for each panel column block j0 = k1 + 64 c <= i0, with
//   W_jk its own for j0 == i0 and otherwise formed again from kin, the copy of
//   A_jk taken before this launch (the CTA of row block j overwrites A_jk with
//   L_jk meanwhile); the same arithmetic gives the same W_jk bit for bit;
//   the updated tiles of column block k1 in rows [k1 + 64, jend) go to kout,
//   the next step's kin;
//   CTA 0 then factors block k1 from its updated tile (NextDiag).
// Against a panel launch followed by a column-update launch (the structure it
// replaced), the chain loses a launch and the panel's wait per block: the next
// diagonal factor starts once CTA 0's own row block is done.  Shared memory: Linv_k, A_ik (then a copied
// A_jk), L_ik (then the next diagonal tile), W_ik, W_jk, and D_k, z_k and the b
// sums.
constexpr size_t STEP_TC_SMEM = sizeof(float) * (5 * NB * MS + 4 * NB);
template <int TERMS>
__global__ void __launch_bounds__(256) k_ldlt_step_tc(int n, long long ld, float *A, int k0, int kb,
                                                      const float *dvec, const float *Linv, float *W, int ldw,
                                                      float *b, int k1, int jend, const float *kin, float *kout,
                                                      NextDiag nd) {
    chain_enter();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float(*sI)[MS] = reinterpret_cast<float(*)[MS]>(smem_raw);
    float(*sA)[MS] = sI + NB;
    float(*sL)[MS] = sA + NB;
    float(*sWo)[MS] = sL + NB;
    float(*sY)[MS] = sWo + NB;
    float *sd = reinterpret_cast<float *>(sY + NB);
    float *sz = sd + NB;
    float(*sbs)[NB] = reinterpret_cast<float(*)[NB]>(sz + NB);  // [2][64]
    const int ib = blockIdx.x, i0 = k1 + 64 * ib, t = threadIdx.x;
    {
        float va[16], vi[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int idx = q * 256 + t, r = idx >> 6, c = idx & 63, row = i0 + r;
            va[q] = (row < n && c < kb) ? A[(long long)row * ld + k0 + c] : 0.f;
            vi[q] = (r < kb && c < kb) ? __ldg(&Linv[r * NB + c]) : 0.f;
        }
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int idx = q * 256 + t;
            sA[idx >> 6][idx & 63] = va[q];
            sI[idx >> 6][idx & 63] = vi[q];
        }
    }
    if (t < NB) {
        sd[t] = t < kb ? dvec[k0 + t] : 1.f;
        sz[t] = (b && t < kb) ? b[k0 + t] : 0.f;
    }
    __syncthreads();
    const int w = t >> 5, lane = t & 31, g = lane >> 2, tq = lane & 3;
    const int m0 = 16 * (w >> 1), n0 = 32 * (w & 1);
    {
        float acc[4][4] = {};
        warp_mma_64<TERMS>(sA, sI, m0, n0, acc);
        float bsum[2] = {0.f, 0.f};  // rows m0 + g and m0 + g + 8
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int rr = m0 + g + (e >> 1) * 8, c = n0 + 8 * nt + 2 * tq + (e & 1), row = i0 + rr;
                const float wv = acc[nt][e];
                const float lv = wv / sd[c];
                sWo[rr][c] = wv;
                sL[rr][c] = lv;
                if (row < n && c < kb) {
                    W[(long long)row * ldw + c] = wv;
                    A[(long long)row * ld + k0 + c] = lv;
                    bsum[e >> 1] += lv * sz[c];
                }
            }
        if (b) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                float v = bsum[h];
                v += __shfl_xor_sync(0xffffffffu, v, 1);
                v += __shfl_xor_sync(0xffffffffu, v, 2);
                if (tq == 0) sbs[w & 1][m0 + g + 8 * h] = v;
            }
        }
    }
    __syncthreads();  // sL and sWo complete, sA free
    if (b && t < NB && i0 + t < n) b[i0 + t] -= sbs[0][t] + sbs[1][t];
    const int nj = jend > k1 ? (jend - k1 + 63) / 64 : 0;
    for (int jb = 0; jb < nj && jb <= ib; jb++) {
        const int j0 = k1 + 64 * jb;
        const float(*Wj)[MS] = sWo;
        if (jb != ib) {  // W_jk from the copy of A_jk
            float va[16];
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int idx = q * 256 + t, r = idx >> 6, c = idx & 63;
                va[q] = (j0 + r < jend && c < kb) ? kin[((size_t)jb * NB + r) * NB + c] : 0.f;
            }
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int idx = q * 256 + t;
                sA[idx >> 6][idx & 63] = va[q];
            }
            __syncthreads();
            float accw[4][4] = {};
            warp_mma_64<TERMS>(sA, sI, m0, n0, accw);
#pragma unroll
            for (int nt = 0; nt < 4; nt++)
#pragma unroll
                for (int e = 0; e < 4; e++)
                    sY[m0 + g + (e >> 1) * 8][n0 + 8 * nt + 2 * tq + (e & 1)] = accw[nt][e];
            __syncthreads();
            Wj = sY;
        }
        float acc[4][4] = {};
        warp_mma_64<TERMS>(sL, Wj, m0, n0, acc);
        const bool keep = jb == 0 && owns_next_diag<float>(nd);  // CTA 0: the next diagonal tile, into sA
        const bool tocopy = jb == 0 && ib >= 1 && i0 < jend;    // the next step's copy of column block k1
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int ii = m0 + g + (e >> 1) * 8, jj = n0 + 8 * nt + 2 * tq + (e & 1), i = i0 + ii, j = j0 + jj;
                if (i < n && j < jend && j <= i) {
                    const float v = A[(long long)i * ld + j] - acc[nt][e];
                    A[(long long)i * ld + j] = v;
                    if (keep) sA[ii][jj] = v;
                    if (tocopy) kout[((size_t)(ib - 1) * NB + ii) * NB + jj] = v;
                }
            }
        __syncthreads();  // sA and sY are reused by the next column block
    }
    // the diagonal factor's scratch: sWo and sY, free now
    static_assert(diag_scratch<float>() <= sizeof(float) * 2 * NB * MS, "diagonal scratch");
    fused_next_diag<float>(n, ld, A, nd, &sA[0][0], reinterpret_cast<unsigned char *>(&sWo[0][0]));
}

// The FP64 factor's fused chain step: k_ldlt_step_tc's structure with the
// products on the FP64 tensor cores (mma.sync m8n8k4 f64;
// warp w: rows 16(w/2) .. +15, columns 32(w%2) .. +31 as 2 x 4 tiles of 8 x 8).
__device__ __forceinline__ void warp_dmma_64(const double (*sa)[MS], const double (*sb)[MS], int m0, int n0,
                                             double (&acc)[2][4][2]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
#pragma unroll 4
    for (int kk = 0; kk < NB; kk += 4) {
        const double a0 = sa[m0 + g][kk + tq], a1 = sa[m0 + 8 + g][kk + tq];
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            const double bv = sb[n0 + 8 * nt + g][kk + tq];
            dmma_8x8x4(acc[0][nt][0], acc[0][nt][1], a0, bv);
            dmma_8x8x4(acc[1][nt][0], acc[1][nt][1], a1, bv);
        }
    }
}
constexpr size_t STEP_DMMA_SMEM = sizeof(double) * (5 * NB * MS + 4 * NB);
__global__ void __launch_bounds__(256) k_ldlt_step_dmma(int n, long long ld, double *A, int k0, int kb,
                                                        const double *dvec, const double *Linv, double *W, int ldw,
                                                        double *b, int k1, int jend, const double *kin, double *kout,
                                                        NextDiag nd) {
    chain_enter();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double(*sI)[MS] = reinterpret_cast<double(*)[MS]>(smem_raw);
    double(*sA)[MS] = sI + NB;
    double(*sL)[MS] = sA + NB;
    double(*sWo)[MS] = sL + NB;
    double(*sY)[MS] = sWo + NB;
    double *sd = reinterpret_cast<double *>(sY + NB);
    double *sz = sd + NB;
    double(*sbs)[NB] = reinterpret_cast<double(*)[NB]>(sz + NB);  // [2][64]
    const int ib = blockIdx.x, i0 = k1 + 64 * ib, t = threadIdx.x;
    for (int q = 0; q < 16; q++) {
        const int idx = q * 256 + t, r = idx >> 6, c = idx & 63, row = i0 + r;
        sA[r][c] = (row < n && c < kb) ? A[(long long)row * ld + k0 + c] : 0.0;
        sI[r][c] = (r < kb && c < kb) ? __ldg(&Linv[r * NB + c]) : 0.0;
    }
    if (t < NB) {
        sd[t] = t < kb ? dvec[k0 + t] : 1.0;
        sz[t] = (b && t < kb) ? b[k0 + t] : 0.0;
    }
    __syncthreads();
    const int w = t >> 5, lane = t & 31, g = lane >> 2, tq = lane & 3;
    const int m0 = 16 * (w >> 1), n0 = 32 * (w & 1);
    {
        double acc[2][4][2] = {};
        warp_dmma_64(sA, sI, m0, n0, acc);
        double bsum[2] = {0.0, 0.0};  // rows m0 + g and m0 + 8 + g
#pragma unroll
        for (int mi = 0; mi < 2; mi++)
#pragma unroll
            for (int nt = 0; nt < 4; nt++)
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int rr = m0 + 8 * mi + g, c = n0 + 8 * nt + 2 * tq + e, row = i0 + rr;
                    const double wv = acc[mi][nt][e];
                    const double lv = wv / sd[c];
                    sWo[rr][c] = wv;
                    sL[rr][c] = lv;
                    if (row < n && c < kb) {
                        W[(long long)row * ldw + c] = wv;
                        A[(long long)row * ld + k0 + c] = lv;
                        bsum[mi] += lv * sz[c];
                    }
                }
        if (b) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                double v = bsum[h];
                v += __shfl_xor_sync(0xffffffffu, v, 1);
                v += __shfl_xor_sync(0xffffffffu, v, 2);
                if (tq == 0) sbs[w & 1][m0 + 8 * h + g] = v;
            }
        }
    }
    __syncthreads();
    if (b && t < NB && i0 + t < n) b[i0 + t] -= sbs[0][t] + sbs[1][t];
    const int nj = jend > k1 ? (jend - k1 + 63) / 64 : 0;
    for (int jb = 0; jb < nj && jb <= ib; jb++) {
        const int j0 = k1 + 64 * jb;
        const double(*Wj)[MS] = sWo;
        if (jb != ib) {
            for (int q = 0; q < 16; q++) {
                const int idx = q * 256 + t, r = idx >> 6, c = idx & 63;
                sA[r][c] = (j0 + r < jend && c < kb) ? kin[((size_t)jb * NB + r) * NB + c] : 0.0;
            }
            __syncthreads();
            double accw[2][4][2] = {};
            warp_dmma_64(sA, sI, m0, n0, accw);
#pragma unroll
            for (int mi = 0; mi < 2; mi++)
#pragma unroll
                for (int nt = 0; nt < 4; nt++)
#pragma unroll
                    for (int e = 0; e < 2; e++) sY[m0 + 8 * mi + g][n0 + 8 * nt + 2 * tq + e] = accw[mi][nt][e];
            __syncthreads();
            Wj = sY;
        }
        double acc[2][4][2] = {};
        warp_dmma_64(sL, Wj, m0, n0, acc);
        const bool keep = jb == 0 && owns_next_diag<double>(nd);
        const bool tocopy = jb == 0 && ib >= 1 && i0 < jend;
#pragma unroll
        for (int mi = 0; mi < 2; mi++)
#pragma unroll
            for (int nt = 0; nt < 4; nt++)
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int ii = m0 + 8 * mi + g, jj = n0 + 8 * nt + 2 * tq + e, i = i0 + ii, j = j0 + jj;
                    if (i < n && j < jend && j <= i) {
                        const double v = A[(long long)i * ld + j] - acc[mi][nt][e];
                        A[(long long)i * ld + j] = v;
                        if (keep) sA[ii][jj] = v;
                        if (tocopy) kout[((size_t)(ib - 1) * NB + ii) * NB + jj] = v;
                    }
                }
        __syncthreads();
    }
    static_assert(diag_scratch<double>() <= sizeof(double) * 2 * NB * MS, "diagonal scratch");
    fused_next_diag<double>(n, ld, A, nd, &sA[0][0], reinterpret_cast<unsigned char *>(&sWo[0][0]));
}

template <typename T>
struct LdltWork {
    T *dvec, *W;
    T *s;                    // [NB]; s[0]: the inverse operand scale of an FP16 trailing update
    T *ktile;                // [2][3][NB][NB] copies of a column block's tiles in a panel (fused chain steps)
    T *Linv;                 // [blocks][NB][NB] inverses of the diagonal blocks' L (the solves use them)
    T *Mc;                   // [4][blocks][NB][NB] coupling blocks: forward, backward at distance 1, then 2
    unsigned long long *ll;  // [2][blocks][2][NB] words the two solves publish their blocks in
    float *split;            // tensor-core path: [4][n][SUPER_W] hi/lo copies of the update's L and W rows
                             // (3xTF32), or [2][n][SUPER_W] FP16 copies (FP16 operands)
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
// Boxes are one 128-byte swizzle row wide: 32 FP32 or 64 FP16 values.
static bool operand_map(CUtensorMap *m, const void *base, long long rows, long long pitch, int box_rows, int K,
                        bool half = false) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = tensor_map_encoder();
    const long long esz = half ? 2 : 4;
    if (!fn || rows < 1 || (reinterpret_cast<size_t>(base) & 15) || ((pitch * esz) & 15)) return false;
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(pitch * esz)};
    cuuint32_t box[2] = {(cuuint32_t)(128 / esz), (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, half ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base),
              dims, strides, box, estr,
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
// A chain kernel (see chain_enter) as a programmatic dependent launch.
template <typename... KArgs, typename... Args>
static cudaError_t launch_chain(void (*kernel)(KArgs...), dim3 grid, size_t smem, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

template <typename... Args>
static cudaError_t launch_wavefront(void (*kernel)(Args...), int grid, size_t smem, cudaStream_t st,
                                    Args... args) {
    void *argv[] = {(void *)&args...};
    return cudaLaunchCooperativeKernel((const void *)kernel, dim3(grid), dim3(256), argv, smem, st);
}

// CTAs of a wavefront launch over nblk blocks: at most one per block and never
// more than can be resident at once (then the lowest unsolved block always runs).
static int wavefront_grid(mp_ctx *ctx, const void *kernel, int nblk, size_t smem) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, smem);
    if (per_sm < 1) per_sm = 1;
    int cap = per_sm * ctx->sm_count;
    return nblk < cap ? nblk : cap;
}

// Words of a wavefront solve: the epoch in the upper half of every word is the
// context's solve count, so words left by earlier solves never match.  Returns
// the next epoch; before the count would wrap, the words are cleared.
static unsigned next_wavefront_epoch(mp_ctx *ctx, unsigned long long *ll, size_t words) {
    if (ctx->solve_epoch >= 0x7ffffff0) {
        cudaMemsetAsync(ll, 0, words * sizeof(unsigned long long), ctx->stream);
        ctx->solve_epoch = 0;
    }
    return (unsigned)++ctx->solve_epoch;
}

// >48 KB dynamic shared memory of the wavefront kernels, set once per context
template <typename T>
static void wavefront_attrs() {
    cudaFuncSetAttribute(k_trsv_ll<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsv_smem<T>());
    cudaFuncSetAttribute(k_trsv_ll<T, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsv_smem<T>());
    cudaFuncSetAttribute(k_trsv_couplings<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(2 * NB * (NB + 1) * sizeof(T)));
    if constexpr (std::is_same<T, float>::value) {
        cudaFuncSetAttribute(k_trsv_band<float, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)band_smem<float>());
        cudaFuncSetAttribute(k_trsv_band<float, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)band_smem<float>());
    }
}

template <typename T>
int ldlt_factor_solve(mp_ctx *ctx, T *A, long long ld, int n, T *b, LdltWork<T> w, bool factor,
                      int tc_terms = 0) {
    cudaStream_t st = ctx->stream;
    const size_t f64_smem = sizeof(double) * 4 * WKC * WPITCH;
    if (!ctx->ldlt_attr) {  // per context: the attributes belong to the context's device
        const int big = 96 * 1024;
        cudaFuncSetAttribute(k_update_f64_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(tc::k_update_tc<tc::MODE_TF32X3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tc::smem_bytes(tc::MODE_TF32X3));
        cudaFuncSetAttribute(tc::k_update_tc_tma<tc::MODE_TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tc::smem_bytes_tma());
        cudaFuncSetAttribute(tc::k_update_tc_tma<tc::MODE_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tc::smem_bytes_tma());
        wavefront_attrs<float>();
        wavefront_attrs<double>();
        cudaFuncSetAttribute(k_ldlt_step_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)STEP_DMMA_SMEM);
        cudaFuncSetAttribute(k_ldlt_diag<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)diag_scratch<double>());
        for (const void *f : {(const void *)k_ldlt_step_tc<1>, (const void *)k_ldlt_step_tc<3>})
            cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        ctx->ldlt_attr = true;
    }
    unsigned long long *flags = ctx->counters + C_FLAGS;
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
            k_update_f64_mma<<<(unsigned)ntiles, 256, f64_smem, st>>>(n, ld, reinterpret_cast<double *>(A), K0, K,
                                                                     R0, reinterpret_cast<const double *>(w.W) + kofs,
                                                                     SUPER_W, cb),
                ++ctx->launches;
            kt_end(ctx, mk);
            return MP_OK;
        }
        const long long rb = (n - R0 + tc::TILE - 1) / tc::TILE;
        const int cb = strip ? (C1 - R0) / tc::TILE_N : 0;
        const long long ntiles = strip ? rb * cb : tc::tile_count(rb);
        const long long wrows = (strip ? C1 : n) - R0;
        // the strips keep TF32 operands in the FP16 mode: their conversion
        // would cost more than their MMAs save
        const int mode = tc_terms == 3 ? tc::MODE_TF32X3 : (tc_terms == 2 && !strip ? tc::MODE_F16 : tc::MODE_TF32);
        const bool split = mode == tc::MODE_TF32X3;
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
        } else if (mode == tc::MODE_F16) {
            __half *Lh = reinterpret_cast<__half *>(w.split), *Wh = Lh + (size_t)n * SUPER_W;
            const long long groups = (n - R0 + wrows) * (K / 8);
            const int gh = (int)std::min<long long>((groups + 255) / 256, (long long)ctx->sm_count * 8);
            const int mk = kt_begin(ctx, MP_KT_PANEL, 0);
            tc::k_half_operands<<<gh, 256, 0, st>>>(Lsrc, ld, n - R0, Wsrc, SUPER_W, wrows, K,
                                                    reinterpret_cast<const float *>(w.dvec) + K0, Lh, Wh,
                                                    reinterpret_cast<float *>(w.s), flags),
                ++ctx->launches;
            kt_end(ctx, mk);
            ok = operand_map(&mLh, Lh, n - R0, K, tc::TILE, K, true) &&
                 operand_map(&mWh, Wh, wrows, K, tc::TILE_N, K, true);
            mLl = mLh;
            mWl = mWh;
        } else {
            ok = operand_map(&mLh, Lsrc, n - R0, ld, tc::TILE, K) &&
                 operand_map(&mWh, Wsrc, wrows, SUPER_W, tc::TILE_N, K);
            mLl = mLh;
            mWl = mWh;
        }
        if (!ok) return fail(ctx, MP_ERR_CUDA, "cuTensorMapEncodeTiled failed for the tensor-core update");
        const int grid = (int)std::min<long long>(ntiles, (long long)ctx->sm_count);
        if (!split) {  // single-product modes: the old values of A move by TMA
            CUtensorMap mC;
            if (!operand_map(&mC, Af, n, ld, tc::TILE, n))
                return fail(ctx, MP_ERR_CUDA, "cuTensorMapEncodeTiled failed for the tensor-core update");
            auto kt = mode == tc::MODE_F16 ? tc::k_update_tc_tma<tc::MODE_F16> : tc::k_update_tc_tma<tc::MODE_TF32>;
            const int mk = kt_begin(ctx, MP_KT_UPDATE, update_flops(R0, C1, K));
            kt<<<grid, tc::THREADS_TMA, tc::smem_bytes_tma(), st>>>(mLh, mWh, mC, n, R0, ntiles, K / tc::kc_of(mode),
                                                                     cb, reinterpret_cast<const float *>(w.s), flags),
                ++ctx->launches;
            kt_end(ctx, mk);
            return MP_OK;
        }
        auto kern = tc::k_update_tc<tc::MODE_TF32X3>;  // the single-product modes returned above
        const int mk = kt_begin(ctx, MP_KT_UPDATE, update_flops(R0, C1, K));
        kern<<<grid, tc::THREADS, tc::smem_bytes(mode), st>>>(mLh, mWh, mLl, mWl, n, ld, Af, R0, ntiles,
                                                              K / tc::kc_of(mode), cb,
                                                              reinterpret_cast<const float *>(w.s), flags),
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
        // cores for the FP32 factor (TF32; 3xTF32 when tc_terms == 3; FP16
        // operands for the trailing updates when tc_terms == 2),
        // register-tiled FP64 for the FP64 factor.
        for (int S0 = 0; S0 < n; S0 += SUPER_W) {
            const int S1 = S0 + SUPER_W < n ? S0 + SUPER_W : n;
            for (int P0 = S0; P0 < S1; P0 += PANEL_W) {
                const int P1 = P0 + PANEL_W < S1 ? P0 + PANEL_W : S1;
                bool diag_done = false;
                for (int k0 = P0, step = 0; k0 < P1; k0 += NB, step++) {
                    const int kb = P1 - k0 < NB ? P1 - k0 : NB;
                    const int k1 = k0 + kb;
                    // one launch per chain step (k_ldlt_step_tc / k_ldlt_step_dmma): the panel of
                    // block k0, the in-panel column update and the next block's diagonal factor;
                    // the first block of a panel is factored alone, which also copies its
                    // column block's panel tiles for the first step
                    T *kin = w.ktile + (size_t)(step & 1) * 3 * NB * NB;
                    T *kout = w.ktile + (size_t)((step + 1) & 1) * 3 * NB * NB;
                    T *Li = w.Linv + (size_t)(k0 / NB) * NB * NB;
                    if (!diag_done) {
                        const int mk = kt_begin(ctx, MP_KT_DIAG, 0);
                        MP_CUDA(ctx, launch_chain(k_ldlt_diag<T>, dim3(1), diag_scratch<T>(), st, n, ld, A, k0, kb,
                                                  w.dvec, Li, b, flags, k1 < P1 ? kin : (T *)nullptr, P1));
                        ++ctx->launches;
                        kt_end(ctx, mk);
                    }
                    diag_done = false;
                    if (k1 < n) {
                        const int kbn = P1 - k1 < NB ? P1 - k1 : NB;
                        const NextDiag nd{k1 < P1 ? k1 : 0, k1 < P1 ? kbn : 0, w.dvec,
                                          w.Linv + (size_t)(k1 / NB) * NB * NB, b, flags};
                        const int mk = kt_begin(ctx, MP_KT_PANEL, 0);
                        const dim3 gs((n - k1 + 63) / 64);
                        if constexpr (std::is_same<T, float>::value) {
                            MP_CUDA(ctx, launch_chain(tc_terms == 3 ? k_ldlt_step_tc<3> : k_ldlt_step_tc<1>, gs,
                                                      STEP_TC_SMEM, st, n, ld, A, k0, kb, (const float *)w.dvec,
                                                      (const float *)Li, w.W + (k0 - S0), (int)SUPER_W, b, k1, P1,
                                                      (const float *)kin, kout, nd));
                        } else {
                            MP_CUDA(ctx, launch_chain(k_ldlt_step_dmma, gs, STEP_DMMA_SMEM, st, n, ld, A, k0, kb,
                                                      (const double *)w.dvec, (const double *)Li, w.W + (k0 - S0),
                                                      (int)SUPER_W, b, k1, P1, (const double *)kin, kout, nd));
                        }
                        ++ctx->launches;
                        kt_end(ctx, mk);
                        diag_done = k1 < P1;
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
    const size_t blkw = (size_t)nblk * NB * NB, llw = (size_t)nblk * 2 * NB;
    // coupling blocks: [forward, backward] at distance 1, then (FP32: banded
    // solves) at distance 2
    T *C1f = w.Mc, *C1b = w.Mc + blkw, *C2f = w.Mc + 2 * blkw, *C2b = w.Mc + 3 * blkw;
    const bool banded = std::is_same<T, float>::value && nblk >= BAND_FROM_BLOCKS;
    if (factor) {  // the coupling blocks of the solves belong to this factor
        const int mk = kt_begin(ctx, MP_KT_TRSV, 0);
        const size_t cs = 2 * NB * (NB + 1) * sizeof(T);
        k_trsv_couplings<T><<<nblk, 256, cs, st>>>(n, ld, A, w.Linv, C1f, C1b, 0, 1), ++ctx->launches;
        if (banded) k_trsv_couplings<T><<<nblk, 256, cs, st>>>(n, ld, A, w.Linv, C2f, C2b, 0, 2), ++ctx->launches;
        kt_end(ctx, mk);
    }
    const unsigned epoch = next_wavefront_epoch(ctx, w.ll, 2 * llw);
    const int mk = kt_begin(ctx, MP_KT_TRSV, 0);
    if (banded) {
        if constexpr (std::is_same<T, float>::value) {
            const int nband = (nblk + 1) / 2;
            const size_t sm = band_smem<float>();
            if (!factor) {
                const int g = wavefront_grid(ctx, (const void *)k_trsv_band<float, 1>, nband, sm);
                MP_CUDA(ctx, launch_wavefront(k_trsv_band<float, 1>, g, sm, st, n, ld, (const float *)A,
                                                 (const float *)w.Linv, (const float *)C1f, (const float *)C2f,
                                                 (const float *)w.dvec, b, w.ll, epoch, flags));
                ++ctx->launches;
            }
            const int g = wavefront_grid(ctx, (const void *)k_trsv_band<float, -1>, nband, sm);
            MP_CUDA(ctx, launch_wavefront(k_trsv_band<float, -1>, g, sm, st, n, ld, (const float *)A,
                                             (const float *)w.Linv, (const float *)C1b, (const float *)C2b,
                                             (const float *)w.dvec, b, w.ll + llw, epoch, flags));
            ++ctx->launches;
        }
    } else {
        const size_t smem = trsv_smem<T>();
        if (!factor) {
            const int g = wavefront_grid(ctx, (const void *)k_trsv_ll<T, 1>, nblk, smem);
            MP_CUDA(ctx, launch_wavefront(k_trsv_ll<T, 1>, g, smem, st, n, ld, (const T *)A, (const T *)w.Linv,
                                          (const T *)C1f, (const T *)w.dvec, b, w.ll, epoch, flags));
            ++ctx->launches;
        }
        const int g = wavefront_grid(ctx, (const void *)k_trsv_ll<T, -1>, nblk, smem);
        MP_CUDA(ctx, launch_wavefront(k_trsv_ll<T, -1>, g, smem, st, n, ld, (const T *)A, (const T *)w.Linv,
                                      (const T *)C1b, (const T *)w.dvec, b, w.ll + llw, epoch, flags));
        ++ctx->launches;
    }
    kt_end(ctx, mk);
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

}  // namespace mp
