// Linear solves of the Newton step: the direct LDL^T path (FP64, or FP32
// factor + FP64 iterative refinement for the mixed form) and the reference's
// Gauss-Seidel iteration (FESolver::solveLinear, src/FESolver.cpp:561-601).
#include <cmath>
#include <utility>

#include "mp_internal.h"
#include "mp_ldlt.cuh"

namespace mp {

// r = b - (K y - FP .* y) = b - J y with J = K - diag(FP), in FP64; also
// accumulates ||r||^2 and ||b||^2 into sums[0], sums[1].  Optionally emits
// r in FP32 for the mixed refinement solve.
__global__ void k_resid_j(int neq, long long ld, const double *__restrict__ K, const double *__restrict__ FP,
                          const double *__restrict__ y, const double *__restrict__ b, double *r, float *r32,
                          double *sums) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= neq) return;
    const double *row = K + (long long)warp * ld;
    double s = 0;
    int n2 = neq & ~1;
    for (int j = 2 * lane; j < n2; j += 64) {
        double2 k = __ldg(reinterpret_cast<const double2 *>(row + j));
        double2 x = *reinterpret_cast<const double2 *>(y + j);
        s = fma(k.x, x.x, s);
        s = fma(k.y, x.y, s);
    }
    if ((neq & 1) && lane == 0) s = fma(row[neq - 1], y[neq - 1], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        double jy = s - FP[warp] * y[warp];
        double rr = b[warp] - jy;
        if (r) r[warp] = rr;
        if (r32) r32[warp] = (float)rr;
        atomicAdd(&sums[0], rr * rr);
        atomicAdd(&sums[1], b[warp] * b[warp]);
    }
}

__global__ void k_axpy_f32(int n, const float *__restrict__ c, double *y) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += (double)c[i];
}

// r = b - J y and the norms ||r||, ||b||: from the sparse copy of K (about 15
// nonzeros a row) when the context holds one, else from the dense K.
static int resid_norms(mp_ctx *ctx, const double *y, const double *b, double *r, float *r32, double *rn,
                       double *bn) {
    long long ld = (ctx->neq + 31) & ~31ll;
    MP_CUDA(ctx, cudaMemsetAsync(ctx->scal + 1, 0, 2 * sizeof(double), ctx->stream));
    if (ctx->sp_val) {
        int rc = fe_resid_j_sparse(ctx, y, b, r, r32, ctx->scal + 1);
        if (rc) return rc;
    } else {
        int th = 256;
        long long bl = ((long long)ctx->neq * 32 + th - 1) / th;
        k_resid_j<<<(unsigned)bl, th, 0, ctx->stream>>>(ctx->neq, ld, ctx->K, ctx->FP, y, b, r, r32, ctx->scal + 1),
            ++ctx->launches;
    }
    MP_CUDA(ctx, cudaGetLastError());
    MP_CUDA(ctx, cudaMemcpyAsync(ctx->scal_host + 1, ctx->scal + 1, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *rn = std::sqrt(ctx->scal_host[1]);
    *bn = std::sqrt(ctx->scal_host[2]);
    return MP_OK;
}

static int check_flags(mp_ctx *ctx, unsigned long long mask, unsigned long long *got) {
    MP_CUDA(ctx, cudaMemcpyAsync(ctx->counters_host + C_FLAGS, ctx->counters + C_FLAGS, sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *got = ctx->counters_host[C_FLAGS] & mask;
    if (*got) {
        unsigned long long keep = ctx->counters_host[C_FLAGS] & ~mask;
        MP_CUDA(ctx, cudaMemcpyAsync(ctx->counters + C_FLAGS, &keep, sizeof(keep), cudaMemcpyHostToDevice,
                                     ctx->stream));
        MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return MP_OK;
}

// Scratch of the dense solves, owned by the context and allocated on its
// first factorization (again when neq changes).
struct SolveScratch {
    double *dvec64 = nullptr, *W64 = nullptr, *s64 = nullptr, *r = nullptr, *Linv64 = nullptr;
    float *dvec32 = nullptr, *W32 = nullptr, *s32 = nullptr, *b32 = nullptr, *Linv32 = nullptr, *split32 = nullptr;
    float *kt32 = nullptr;              // [2][3][NB][NB] column-block copies of the fused chain steps
    double *kt64 = nullptr;
    double *Mc64 = nullptr;             // [2][blocks][NB][NB] coupling blocks (FP64 solves, Gauss-Seidel)
    float *Mc32 = nullptr;              // [4][blocks][NB][NB] coupling blocks (FP32 banded solves)
    unsigned long long *ll = nullptr;   // [2][blocks][2][NB] wavefront words
    size_t ll_words = 0;
    int neq = 0;
};

static void release(SolveScratch *s) {
    void *p[] = {s->dvec64, s->W64, s->s64, s->r, s->dvec32, s->W32, s->s32, s->b32,
                 s->Linv64, s->Linv32, s->Mc64, s->Mc32, s->ll, s->split32, s->kt32, s->kt64};
    for (void *q : p)
        if (q) cudaFree(q);
    *s = SolveScratch();
}

void solve_free(mp_ctx *ctx) {
    SolveScratch *s = static_cast<SolveScratch *>(ctx->solve_scratch);
    if (!s) return;
    release(s);
    delete s;
    ctx->solve_scratch = nullptr;
}

static int ensure_scratch(mp_ctx *ctx, SolveScratch **out) {
    if (!ctx->solve_scratch) ctx->solve_scratch = new SolveScratch();
    SolveScratch &s = *static_cast<SolveScratch *>(ctx->solve_scratch);
    *out = &s;
    if (s.neq == ctx->neq && s.dvec64) return MP_OK;
    const int n = ctx->neq;
    // the context's own stream may still read the old buffers
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    release(&s);
    MP_CUDA(ctx, cudaMalloc(&s.dvec64, sizeof(double) * (n + 64)));
    MP_CUDA(ctx, cudaMalloc(&s.W64, sizeof(double) * (size_t)(n + NB) * SUPER_W));
    MP_CUDA(ctx, cudaMalloc(&s.s64, sizeof(double) * NB));
    MP_CUDA(ctx, cudaMalloc(&s.r, sizeof(double) * (n + 64)));
    MP_CUDA(ctx, cudaMalloc(&s.dvec32, sizeof(float) * (n + 64)));
    MP_CUDA(ctx, cudaMalloc(&s.W32, sizeof(float) * (size_t)(n + NB) * SUPER_W));
    MP_CUDA(ctx, cudaMalloc(&s.s32, sizeof(float) * NB));
    MP_CUDA(ctx, cudaMalloc(&s.kt32, sizeof(float) * 2 * 3 * NB * NB));
    MP_CUDA(ctx, cudaMalloc(&s.kt64, sizeof(double) * 2 * 3 * NB * NB));
    MP_CUDA(ctx, cudaMalloc(&s.b32, sizeof(float) * (n + 64)));
    const size_t nblk = (n + NB - 1) / NB;
    MP_CUDA(ctx, cudaMalloc(&s.Linv64, sizeof(double) * nblk * NB * NB));
    MP_CUDA(ctx, cudaMalloc(&s.Linv32, sizeof(float) * nblk * NB * NB));
    MP_CUDA(ctx, cudaMalloc(&s.split32, sizeof(float) * 4 * (size_t)n * SUPER_W));
    MP_CUDA(ctx, cudaMalloc(&s.Mc64, sizeof(double) * 2 * nblk * NB * NB));
    MP_CUDA(ctx, cudaMalloc(&s.Mc32, sizeof(float) * 4 * nblk * NB * NB));
    s.ll_words = 2 * nblk * 2 * NB;
    MP_CUDA(ctx, cudaMalloc(&s.ll, sizeof(unsigned long long) * s.ll_words));
    MP_CUDA(ctx, cudaMemsetAsync(s.ll, 0, sizeof(unsigned long long) * s.ll_words, ctx->stream));
    ctx->solve_epoch = 0;  // fresh words hold epoch 0, which no solve uses
    s.neq = n;
    return MP_OK;
}

// Mixed-form refinement stop: ||G - J y|| <= REFINE_RTOL ||G|| (or the
// residual stalls above 0.7 of the previous one): the FP64 factorization's
// accuracy, so y matches dsysv_'s to the FP64 form's tolerance.
constexpr double REFINE_RTOL = 1e-14;

int fe_solve_ldlt(mp_ctx *ctx, int form, mp_newton_stats *st) {
    SolveScratch *sp = nullptr;
    int rc = ensure_scratch(ctx, &sp);
    if (rc) return rc;
    SolveScratch &sc = *sp;
    const int n = ctx->neq;
    const long long ld = (n + 31) & ~31ll;
    cudaEventRecord(ctx->t1.a, ctx->stream);
    if (form == MP_FORM_FP64) {
        if (!ctx->J || !ctx->j_current) return fail(ctx, MP_ERR_STATE, "no current FP64 J (build it first)");
        ctx->j_current = false;  // the factorization overwrites J
        MP_CUDA(ctx, cudaMemcpyAsync(ctx->y, ctx->G, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
        LdltWork<double> w{sc.dvec64, sc.W64, sc.s64, sc.kt64, sc.Linv64, sc.Mc64, sc.ll, nullptr};
        rc = ldlt_factor_solve<double>(ctx, ctx->J, ld, n, ctx->y, w, true);
        if (rc) return rc;
        cudaEventRecord(ctx->t1.b, ctx->stream);
        double rn, bn;
        rc = resid_norms(ctx, ctx->y, ctx->G, nullptr, nullptr, &rn, &bn);
        if (rc) return rc;
        if (st) {
            st->linear_iterations = 1;
            st->linear_residual = rn / n;
        }
    } else {
        // the factorization overwrites J32: it is current once per build of J;
        // otherwise it is rebuilt from K and the current FP
        if (!ctx->j32_current && (rc = fe_j32_from_k(ctx))) return rc;
        ctx->j32_current = false;
        MP_CUDA(ctx, cudaMemsetAsync(ctx->y, 0, sizeof(double) * n, ctx->stream));
        LdltWork<float> w{sc.dvec32, sc.W32, sc.s32, sc.kt32, sc.Linv32, sc.Mc32, sc.ll, sc.split32};
        double rn = 0, bn = 0;
        // r = G (y = 0), in FP32 for the first solve, which also factors J32
        rc = resid_norms(ctx, ctx->y, ctx->G, sc.r, sc.b32, &rn, &bn);
        if (rc) return rc;
        const int terms = ctx->mixed_factor != MP_MIXED_AUTO ? ctx->mixed_factor
                          : n >= MP_MIXED_FP16_FROM       ? MP_MIXED_FP16
                                                          : MP_MIXED_TF32X3;
        rc = ldlt_factor_solve<float>(ctx, ctx->J32, ld, n, sc.b32, w, true, terms);
        if (rc) return rc;
        if (terms == MP_MIXED_FP16) {
            unsigned long long range = 0;
            if ((rc = check_flags(ctx, FLAG_HALF_RANGE, &range))) return rc;
            if (range) {  // an operand did not fit FP16: factor J again with TF32 operands
                if ((rc = fe_j32_from_k(ctx))) return rc;
                ctx->j32_current = false;
                if ((rc = resid_norms(ctx, ctx->y, ctx->G, sc.r, sc.b32, &rn, &bn))) return rc;
                rc = ldlt_factor_solve<float>(ctx, ctx->J32, ld, n, sc.b32, w, true, MP_MIXED_TF32);
                if (rc) return rc;
            }
        }
        cudaEventRecord(ctx->t1.b, ctx->stream);
        k_axpy_f32<<<(n + 255) / 256, 256, 0, ctx->stream>>>(n, sc.b32, ctx->y), ++ctx->launches;
        int it = 1;
        double prev = 1e300;
        for (; it < 60; it++) {
            rc = resid_norms(ctx, ctx->y, ctx->G, sc.r, sc.b32, &rn, &bn);
            if (rc) return rc;
            if (!(rn > REFINE_RTOL * bn) || rn > 0.7 * prev) break;
            prev = rn;
            rc = ldlt_factor_solve<float>(ctx, ctx->J32, ld, n, sc.b32, w, false);
            if (rc) return rc;
            k_axpy_f32<<<(n + 255) / 256, 256, 0, ctx->stream>>>(n, sc.b32, ctx->y), ++ctx->launches;
        }
        if (st) {
            st->linear_iterations = it;
            st->linear_residual = rn / n;
        }
    }
    unsigned long long bad = 0;
    rc = check_flags(ctx, FLAG_SINGULAR | FLAG_LOOKBACK_TIMEOUT, &bad);
    if (rc) return rc;
    if (st) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->t1.a, ctx->t1.b);
        st->ms_factor = ms;
    }
    if (bad & FLAG_LOOKBACK_TIMEOUT)
        return fail(ctx, MP_ERR_TIMEOUT, "a bounded wait in the factorization or the triangular solves gave up");
    if (bad) return fail(ctx, MP_ERR_SINGULAR, "LDL^T met a zero or non-finite pivot");
    return MP_OK;
}

// ---- Gauss-Seidel ---------------------------------------------------------------------
// One sweep of the reference's row-sequential Gauss-Seidel (solveLinear,
// src/FESolver.cpp:567-578) is x_new = (D + L)^-1 (b - U x_old), with L, D, U
// the strictly lower, diagonal and strictly upper parts of J; a row with
// |J_uu| < 1e-12 keeps its value (src/FESolver.cpp:569).  The sweep runs as a
// persistent wavefront over 64-row blocks (the triangular solves' scheme):
// block k streams its rows once, summing the columns right of the diagonal
// against x_old as soon as it starts and the columns of blocks 0 .. k-2
// against x_new as those blocks publish it (wavefront words holding the
// sweep's epoch), then applies the stored inverse Minv_kk of its diagonal block
// of D + L -- a 64 x 64 product instead of 64 dependent substitutions -- and
// last takes block k-1 through the coupling block Minv_kk J~_{k,k-1} (J~: J
// without the skipped rows), so a step of the chain is one poll and one small
// product.  x_old and x_new are separate buffers (sweeps alternate them), so no
// block reads a value another block is rewriting.  The iterate is the
// reference's up to summation order.

// Inverse of each 64 x 64 diagonal block of D + L, rows with |J_uu| < 1e-12
// (and rows past n) replaced by identity rows, so the block's row keeps its
// value.  One CTA of 64 threads per block; thread j owns column j of the
// inverse X, computed row by row (X_rj = (delta_rj - sum_{c<r} M_rc X_cj) / M_rr),
// and row r of X replaces row r of M once the step has read it.
__global__ void __launch_bounds__(64) k_gs_block_inverse(int n, long long ld, const double *__restrict__ A,
                                                         double *Minv) {
    __shared__ double sM[NB][NB + 1];
    const int blk = blockIdx.x, r0 = blk * NB, j = threadIdx.x;
    for (int r = 0; r < NB; r++) {
        const int row = r0 + r;
        double v = 0.0;
        if (row < n && j <= r) v = A[(long long)row * ld + r0 + j];
        sM[r][j] = v;
    }
    __syncthreads();
    // identity rows for skipped (and padding) rows
    const bool ident = r0 + j >= n || fabs(sM[j][j]) < 1e-12;
    __syncthreads();
    if (ident)
        for (int c = 0; c < NB; c++) sM[j][c] = c == j ? 1.0 : 0.0;
    __syncthreads();
    for (int r = 0; r < NB; r++) {
        double t = r == j ? 1.0 : 0.0;
        for (int c = j; c < r; c++) t = fma(-sM[r][c], sM[c][j], t);
        const double x = r < j ? 0.0 : t / sM[r][r];
        __syncthreads();  // every thread has read row r of M
        sM[r][j] = x;
        __syncthreads();
    }
    double *out = Minv + (size_t)blk * NB * NB;
    for (int r = 0; r < NB; r++) out[r * NB + j] = sM[r][j];
}

// rup_i = b_i - sum_{j>i} J_ij x_old_j for every row: the x_old half of a sweep,
// a bandwidth-bound pass over the strict upper triangle, one warp per row.
__global__ void __launch_bounds__(256) k_gs_upper(int n, long long ld, const double *__restrict__ A,
                                                  const double *__restrict__ b, const double *__restrict__ x_old,
                                                  double *rup) {
    const int row = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (row >= n) return;
    const double *a = A + (long long)row * ld;
    double s = 0.0;
#pragma unroll 4
    for (int j = row + 1 + lane; j < n; j += 32) s = fma(__ldg(a + j), __ldg(x_old + j), s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) rup[row] = b[row] - s;
}

// Shared memory of k_gs_sweep: the block inverse and the coupling block, two
// poll buffers, the right-hand side, two poll results.
constexpr size_t gs_smem() { return sizeof(double) * (2 * NB * MS + 3 * NB) + 2 * sizeof(int); }

// The x_new half of a sweep: with rup = b - U x_old from k_gs_upper, block k
// solves (D + L)_kk x_k = rup_k - sum_{j<k} J_kj x_new_j as a wavefront.
__global__ void __launch_bounds__(256) k_gs_sweep(int n, long long ld, const double *__restrict__ A,
                                                  const double *__restrict__ rup, const double *__restrict__ Minv,
                                                  const double *__restrict__ Mc, const double *x_old, double *x_new,
                                                  unsigned long long *ll, unsigned epoch,
                                                  unsigned long long *flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double(*sI)[MS] = reinterpret_cast<double(*)[MS]>(smem_raw);
    double(*sC)[MS] = sI + NB;
    double *sx = reinterpret_cast<double *>(sC + NB);  // [2][NB]
    double *srhs = sx + 2 * NB;
    int *sok = reinterpret_cast<int *>(srhs + NB);  // [2]
    const int nblk = (n + NB - 1) / NB;
    const int t = threadIdx.x;
    const int r = t >> 2, q = t & 3;  // row of the block; quarter of each 64-column chunk / columns 4k + q
    int par = 0;
    for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        const int r0 = blk * NB, kb = n - r0 < NB ? n - r0 : NB;
        const bool has_pred = blk > 0;
        for (int idx = t; idx < NB * NB; idx += 256) {
            sI[idx >> 6][idx & 63] = __ldg(&Minv[(size_t)blk * NB * NB + idx]);
            sC[idx >> 6][idx & 63] = has_pred ? __ldg(&Mc[(size_t)blk * NB * NB + idx]) : 0.0;
        }
        const int row = r0 + (r < kb ? r : 0);
        const double *arow = A + (long long)row * ld + q * 16;
        // this row's diagonal, old value and x_old half, read before any wait
        const double d_rr = A[(long long)row * ld + row], xo_r = x_old[row], ru_r = rup[row];
        double acc = 0.0, ap[16];
        // the diagonal block's columns right of the diagonal belong to the x_old
        // half (in rup); columns of blocks 0 .. blk-2: x_new as they are published
        const int nfar = blk > 1 ? blk - 1 : 0;
        bool ok = true;
        if (nfar > 0) load16<double, false>(arow, ap);
        for (int s = 0; s < nfar; s++) {
            double *buf = sx + par * NB;
            ok = wait_chunk<double>(ll, s, epoch, buf, poll_backoff(nfar - s), sok + par, flags);
            par ^= 1;
            if (!ok) break;
#pragma unroll
            for (int k = 0; k < 16; k++) acc = fma(ap[k], buf[q * 16 + k], acc);
            if (s + 1 < nfar) load16<double, false>(arow + (s + 1) * NB, ap);
        }
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        acc += __shfl_xor_sync(0xffffffffu, acc, 2);
        if (q == 0) srhs[r] = r < kb ? (fabs(d_rr) < 1e-12 ? xo_r : ru_r - acc) : 0.0;
        __syncthreads();
        double y = 0.0;
#pragma unroll
        for (int k = 0; k < 16; k++) y = fma(sI[r][4 * k + q], srhs[4 * k + q], y);
        y += __shfl_xor_sync(0xffffffffu, y, 1);
        y += __shfl_xor_sync(0xffffffffu, y, 2);
        // block blk-1 through the coupling block Minv_kk J~_{k,k-1}
        double xr = y;
        if (has_pred && ok) {
            double p0, p1;
            wait_warp<double>(ll, blk - 1, epoch, p0, p1, flags);
            double v = 0.0;
#define MP_STEP(K) v = fma(sC[r][4 * K + q], warp_value<double, K>(p0, p1, q), v);
            MP_STEP(0) MP_STEP(1) MP_STEP(2) MP_STEP(3) MP_STEP(4) MP_STEP(5) MP_STEP(6) MP_STEP(7)
            MP_STEP(8) MP_STEP(9) MP_STEP(10) MP_STEP(11) MP_STEP(12) MP_STEP(13) MP_STEP(14) MP_STEP(15)
#undef MP_STEP
            v += __shfl_xor_sync(0xffffffffu, v, 1);
            v += __shfl_xor_sync(0xffffffffu, v, 2);
            xr = y - v;
        }
        if (q == 0) {
            ll_put<double>(ll, blk, r, r < kb ? xr : 0.0, epoch);
            if (r < kb) x_new[r0 + r] = xr;
        }
        __syncthreads();  // shared memory is reused by this CTA's next block
    }
}

// S Gauss-Seidel sweeps in one cooperative launch, one CTA per 64-row block
// (used when every block's CTA is resident).  J is symmetric and stored in
// full, so block i reads every other block j's contribution J_ij x_j as the
// 64 x 64 tile of j's row band at i's columns (J_ji, transposed): when block j
// publishes a sweep's values, all other blocks read one contiguous row band of
// J.  In sweep s, block i sums the blocks j < i-1 of sweep s as they are
// published, applies Minv_ii, takes block i-1 through the coupling block,
// publishes x_i, and then sums its own diagonal block's strictly upper part
// against x_i and the blocks j > i of sweep s, which is the x_old half of its
// sweep s+1 -- so sweep s+1 needs no separate pass and starts as soon as the
// last block of sweep s is published.  The first
// sweep's x_old half comes in rup0 = b - U x.  One word per value and sweep
// epoch suffices: a block publishes sweep s+1 only after every reader of its
// sweep-s words has moved on.  x is updated in place (only the owning block
// reads its own rows).
constexpr size_t gs_sweeps_smem() { return sizeof(double) * (2 * NB * MS + 16 * (NB + 1) + 7 * NB) + 2 * sizeof(int); }

__global__ void __launch_bounds__(256, 2) k_gs_sweeps(int n, long long ld, const double *__restrict__ A,
                                                      const double *__restrict__ b, const double *__restrict__ rup0,
                                                      const double *__restrict__ Minv, const double *__restrict__ Mc,
                                                      double *x, unsigned long long *ll, unsigned epoch0, int S,
                                                      unsigned long long *flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double(*sI)[MS] = reinterpret_cast<double(*)[MS]>(smem_raw);
    double(*sC)[MS] = sI + NB;
    double(*spart)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(sC + NB);  // [16][65]
    double *sx = reinterpret_cast<double *>(spart + 16);                     // [2][NB] poll buffers
    double *srhs = sx + 2 * NB;                                              // this sweep's right-hand side
    double *sb = srhs + NB;                                                  // b of the block's rows
    double *snext = sb + NB;                                                 // b - U x_s: the next sweep's
    double *sxo = snext + NB;                                                // the rows' current values
    double *sdu = sxo + NB;                                                  // diagonal block's upper part x x_i
    int *sok = reinterpret_cast<int *>(sdu + NB);                            // [2]
    const int nblk = (n + NB - 1) / NB, blk = blockIdx.x;
    const int r0 = blk * NB, kb = n - r0 < NB ? n - r0 : NB;
    const int t = threadIdx.x;
    const int r = t >> 2, q = t & 3;       // the chain step: row r, columns 4k + q
    const int c4 = t & 15, part = t >> 4;  // tiles: block rows 4c4 .. +3, band rows 4part .. +3
    const bool has_pred = blk > 0;
    for (int idx = t; idx < NB * NB; idx += 256) {
        sI[idx >> 6][idx & 63] = __ldg(&Minv[(size_t)blk * NB * NB + idx]);
        sC[idx >> 6][idx & 63] = has_pred ? __ldg(&Mc[(size_t)blk * NB * NB + idx]) : 0.0;
    }
    // row r's strictly upper coefficients inside the diagonal block, columns 4k + q
    double du[16];
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const int c = 4 * k + q;
        du[k] = (r < kb && c > r && c < kb) ? A[(long long)(r0 + r) * ld + r0 + c] : 0.0;
    }
    bool skip = false;  // thread t < 64: row t keeps its value (|J_tt| < 1e-12)
    if (t < NB) {
        const bool in = t < kb;
        sb[t] = in ? b[r0 + t] : 0.0;
        snext[t] = in ? rup0[r0 + t] : 0.0;
        sxo[t] = in ? x[r0 + t] : 0.0;
        skip = in && fabs(A[(long long)(r0 + t) * ld + r0 + t]) < 1e-12;
    }
    // the 4 x 4 piece of the tile of band j at this block's columns
    double ap[16];
    auto fetch = [&](int j) {
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int i = j * NB + 4 * part + e;
            if (i < n && 4 * c4 + 3 < kb) {
                load4p<double>(A + (long long)i * ld + r0 + 4 * c4, ap + 4 * e);
            } else {
#pragma unroll
                for (int k = 0; k < 4; k++) ap[4 * e + k] = (i < n && 4 * c4 + k < kb) ? A[(long long)i * ld + r0 + 4 * c4 + k] : 0.0;
            }
        }
    };
    // sums over bands j in [j0, j1) of sweep `ep` into spart; returns false if a wait gave up
    int par = 0;
    auto sum_bands = [&](int j0, int j1, unsigned ep, int crit) -> bool {
        double acc4[4] = {0.0, 0.0, 0.0, 0.0};
        bool ok = true;
        if (j0 < j1) fetch(j0);
        for (int j = j0; j < j1; j++) {
            double *buf = sx + par * NB;
            const int dist = crit > j ? crit - j : j - crit;
            ok = wait_chunk<double>(ll, j, ep, buf, poll_backoff(dist), sok + par, flags);
            par ^= 1;
            if (!ok) break;
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const double xe = buf[4 * part + e];
#pragma unroll
                for (int k = 0; k < 4; k++) acc4[k] = fma(ap[4 * e + k], xe, acc4[k]);
            }
            if (j + 1 < j1) fetch(j + 1);
        }
#pragma unroll
        for (int k = 0; k < 4; k++) spart[part][4 * c4 + k] = acc4[k];
        __syncthreads();
        return ok;
    };
    bool ok = true;
    for (int s = 0; s < S && ok; s++) {
        const unsigned ep = epoch0 + (unsigned)s;
        // blocks 0 .. blk-2 of this sweep
        ok = sum_bands(0, blk > 1 ? blk - 1 : 0, ep, blk - 1);
        if (t < NB) {
            double sum = 0.0;
#pragma unroll
            for (int p = 0; p < 16; p++) sum += spart[p][t];
            srhs[t] = t < kb ? (skip ? sxo[t] : snext[t] - sum) : 0.0;
        }
        __syncthreads();
        double y = 0.0;
#pragma unroll
        for (int k = 0; k < 16; k++) y = fma(sI[r][4 * k + q], srhs[4 * k + q], y);
        y += __shfl_xor_sync(0xffffffffu, y, 1);
        y += __shfl_xor_sync(0xffffffffu, y, 2);
        double xr = y;
        if (has_pred && ok) {
            double p0, p1;
            wait_warp<double>(ll, blk - 1, ep, p0, p1, flags);
            double v = 0.0;
#define MP_STEP(K) v = fma(sC[r][4 * K + q], warp_value<double, K>(p0, p1, q), v);
            MP_STEP(0) MP_STEP(1) MP_STEP(2) MP_STEP(3) MP_STEP(4) MP_STEP(5) MP_STEP(6) MP_STEP(7)
            MP_STEP(8) MP_STEP(9) MP_STEP(10) MP_STEP(11) MP_STEP(12) MP_STEP(13) MP_STEP(14) MP_STEP(15)
#undef MP_STEP
            v += __shfl_xor_sync(0xffffffffu, v, 1);
            v += __shfl_xor_sync(0xffffffffu, v, 2);
            xr = y - v;
        }
        if (q == 0) {
            ll_put<double>(ll, blk, r, r < kb ? xr : 0.0, ep);
            if (r < kb) {
                x[r0 + r] = xr;
                sxo[r] = xr;
            }
        }
        if (s + 1 < S && ok) {
            // the next sweep's x_old half: this block's strictly upper part
            // against x_i, then blocks blk+1 .. nblk-1 of this sweep
            __syncthreads();  // sxo holds x_i
            double v = 0.0;
#pragma unroll
            for (int k = 0; k < 16; k++) v = fma(du[k], sxo[4 * k + q], v);
            v += __shfl_xor_sync(0xffffffffu, v, 1);
            v += __shfl_xor_sync(0xffffffffu, v, 2);
            if (q == 0) sdu[r] = v;
            ok = sum_bands(blk + 1, nblk, ep, blk);
            if (t < NB) {
                double sum = 0.0;
#pragma unroll
                for (int p = 0; p < 16; p++) sum += spart[p][t];
                snext[t] = sb[t] - sdu[t] - sum;
            }
        }
        __syncthreads();
    }
}

// L2 = sqrt(sum (b - A x)^2)/neq  (src/FESolver.cpp:580-590), partial sums into sums[0]
__global__ void k_gs_resid(int neq, long long ld, const double *__restrict__ A, const double *__restrict__ b,
                           const double *__restrict__ x, double *sums) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= neq) return;
    const double *row = A + (long long)warp * ld;
    double s = 0;
    for (int j = lane; j < neq; j += 32) s = fma(row[j], x[j], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        double r = b[warp] - s;
        atomicAdd(sums, r * r);
    }
}

int fe_solve_gs(mp_ctx *ctx, mp_newton_stats *st) {
    if (!ctx->J || !ctx->j_current) return fail(ctx, MP_ERR_STATE, "no current FP64 J (build it first)");
    SolveScratch *sp = nullptr;
    int rc = ensure_scratch(ctx, &sp);
    if (rc) return rc;
    const int n = ctx->neq;
    const long long ld = (n + 31) & ~31ll;
    const int nblk = (n + NB - 1) / NB;
    const double tol = 1e-4;
    const int th = 256;
    const long long bl = ((long long)n * 32 + th - 1) / th;
    unsigned long long *flags = ctx->counters + C_FLAGS;
    // the inverses of the diagonal blocks of D + L and the coupling blocks
    // Minv_kk J~_{k,k-1}, J~ without the rows the sweep skips (J is fixed for the solve)
    k_gs_block_inverse<<<nblk, 64, 0, ctx->stream>>>(n, ld, ctx->J, sp->Linv64), ++ctx->launches;
    wavefront_attrs<double>();
    k_trsv_couplings<double><<<nblk, 256, 2 * NB * (NB + 1) * sizeof(double), ctx->stream>>>(
        n, ld, ctx->J, sp->Linv64, sp->Mc64, nullptr, 1, 1),
        ++ctx->launches;
    const size_t smem = gs_smem(), fsmem = gs_sweeps_smem();
    cudaFuncSetAttribute(k_gs_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_gs_sweeps, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsmem);
    const int grid = wavefront_grid(ctx, (const void *)k_gs_sweep, nblk, smem);
    // every block's CTA resident: the sweeps run fused, 25 a launch
    const bool fused = wavefront_grid(ctx, (const void *)k_gs_sweeps, nblk, fsmem) == nblk;
    double *xa = ctx->y, *xb = sp->r;  // per-sweep launches alternate the two
    double *rup = sp->dvec64;          // b - U x_old (the FP64 factor's D is not in use here)
    double L2 = 0;
    int it = 0, done = 0;
    bool converged = false;
    // the reference checks the residual after sweeps 1, 26, 51, ... (it % 25 == 0)
    while (done < ctx->gs_max_sweeps) {
        const int S = done == 0 ? 1 : std::min(25, ctx->gs_max_sweeps - done);
        const int mk = kt_begin(ctx, MP_KT_TRSV, 0);
        if (fused) {
            k_gs_upper<<<(unsigned)bl, th, 0, ctx->stream>>>(n, ld, ctx->J, ctx->G, xa, rup), ++ctx->launches;
            unsigned ep0 = next_wavefront_epoch(ctx, sp->ll, sp->ll_words);
            ctx->solve_epoch += S - 1;  // the launch uses epochs ep0 .. ep0 + S - 1
            MP_CUDA(ctx, launch_wavefront(k_gs_sweeps, nblk, fsmem, ctx->stream, n, ld, (const double *)ctx->J,
                                          (const double *)ctx->G, (const double *)rup, (const double *)sp->Linv64,
                                          (const double *)sp->Mc64, xa, sp->ll, ep0, S, flags));
            ++ctx->launches;
        } else {
            for (int k = 0; k < S; k++) {
                k_gs_upper<<<(unsigned)bl, th, 0, ctx->stream>>>(n, ld, ctx->J, ctx->G, xa, rup), ++ctx->launches;
                const unsigned epoch = next_wavefront_epoch(ctx, sp->ll, sp->ll_words);
                MP_CUDA(ctx, launch_wavefront(k_gs_sweep, grid, smem, ctx->stream, n, ld, (const double *)ctx->J,
                                              (const double *)rup, (const double *)sp->Linv64,
                                              (const double *)sp->Mc64, (const double *)xa, xb, sp->ll, epoch,
                                              flags));
                ++ctx->launches;
                std::swap(xa, xb);
            }
        }
        kt_end(ctx, mk);
        done += S;
        it = done - 1;
        if (it % 25 == 0) {
            MP_CUDA(ctx, cudaMemsetAsync(ctx->scal + 3, 0, sizeof(double), ctx->stream));
            k_gs_resid<<<(unsigned)bl, th, 0, ctx->stream>>>(n, ld, ctx->J, ctx->G, xa, ctx->scal + 3), ++ctx->launches;
            MP_CUDA(ctx, cudaMemcpyAsync(ctx->scal_host + 3, ctx->scal + 3, sizeof(double), cudaMemcpyDeviceToHost,
                                         ctx->stream));
            MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            L2 = std::sqrt(ctx->scal_host[3]) / n;
            if (L2 < tol) {
                converged = true;
                break;
            }
        }
    }
    if (!converged) it = ctx->gs_max_sweeps;
    if (xa != ctx->y)
        MP_CUDA(ctx, cudaMemcpyAsync(ctx->y, xa, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    MP_CUDA(ctx, cudaGetLastError());
    unsigned long long bad = 0;
    rc = check_flags(ctx, FLAG_LOOKBACK_TIMEOUT, &bad);
    if (rc) return rc;
    if (bad) return fail(ctx, MP_ERR_TIMEOUT, "a bounded wait in the Gauss-Seidel sweep gave up");
    if (st) {
        st->linear_iterations = it;
        st->linear_residual = L2;
        if (!converged) st->linear_failures++;
    }
    return MP_OK;
}

}  // namespace mp
