// Linear solves of the Newton step: the direct LDL^T path (FP64, or FP32
// factor + FP64 iterative refinement for the mixed form) and the reference's
// Gauss-Seidel iteration (FESolver::solveLinear, src/FESolver.cpp:561-601).
#include <cmath>

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

__global__ void k_j_to_f32(int neq, long long ld, const double *__restrict__ J, float *J32) {
    long long total = (long long)neq * ld;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x)
        J32[i] = (float)J[i];
}

__global__ void k_axpy_f32(int n, const float *__restrict__ c, double *y) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += (double)c[i];
}

static int resid_norms(mp_ctx *ctx, const double *y, const double *b, double *r, float *r32, double *rn,
                       double *bn) {
    long long ld = (ctx->neq + 31) & ~31ll;
    MP_CUDA(ctx, cudaMemsetAsync(ctx->scal + 1, 0, 2 * sizeof(double), ctx->stream));
    int th = 256;
    long long bl = ((long long)ctx->neq * 32 + th - 1) / th;
    k_resid_j<<<(unsigned)bl, th, 0, ctx->stream>>>(ctx->neq, ld, ctx->K, ctx->FP, y, b, r, r32, ctx->scal + 1), ++ctx->launches;
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
    int *ready = nullptr;
    int neq = 0;
};

static void release(SolveScratch *s) {
    void *p[] = {s->dvec64, s->W64, s->s64, s->r, s->dvec32, s->W32, s->s32, s->b32,
                 s->Linv64, s->Linv32, s->ready, s->split32};
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
    MP_CUDA(ctx, cudaMalloc(&s.b32, sizeof(float) * (n + 64)));
    const size_t nblk = (n + NB - 1) / NB;
    MP_CUDA(ctx, cudaMalloc(&s.Linv64, sizeof(double) * nblk * NB * NB));
    MP_CUDA(ctx, cudaMalloc(&s.Linv32, sizeof(float) * nblk * NB * NB));
    MP_CUDA(ctx, cudaMalloc(&s.split32, sizeof(float) * 4 * (size_t)n * SUPER_W));
    MP_CUDA(ctx, cudaMalloc(&s.ready, sizeof(int) * 2 * (nblk + 1)));
    MP_CUDA(ctx, cudaMemsetAsync(s.ready, 0, sizeof(int) * 2 * (nblk + 1), ctx->stream));
    ctx->solve_epoch = 0;  // fresh ready words hold epoch 0
    s.neq = n;
    return MP_OK;
}

int fe_solve_ldlt(mp_ctx *ctx, int form, mp_newton_stats *st) {
    SolveScratch *sp = nullptr;
    int rc = ensure_scratch(ctx, &sp);
    if (rc) return rc;
    SolveScratch &sc = *sp;
    const int n = ctx->neq;
    const long long ld = (n + 31) & ~31ll;
    cudaEventRecord(ctx->t1.a, ctx->stream);
    if (form == MP_FORM_FP64) {
        MP_CUDA(ctx, cudaMemcpyAsync(ctx->y, ctx->G, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
        LdltWork<double> w{sc.dvec64, sc.W64, sc.s64, sc.Linv64, sc.ready, nullptr};
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
        if (!ctx->J32) MP_CUDA(ctx, cudaMalloc(&ctx->J32, sizeof(float) * (size_t)ld * n));
        // the factorization overwrites J32: it is current once per build of J
        if (!ctx->j32_current)
            k_j_to_f32<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(n, ld, ctx->J, ctx->J32), ++ctx->launches;
        ctx->j32_current = false;
        MP_CUDA(ctx, cudaMemsetAsync(ctx->y, 0, sizeof(double) * n, ctx->stream));
        LdltWork<float> w{sc.dvec32, sc.W32, sc.s32, sc.Linv32, sc.ready, sc.split32};
        double rn = 0, bn = 0;
        // r = G (y = 0), in FP32 for the first solve, which also factors J32
        rc = resid_norms(ctx, ctx->y, ctx->G, sc.r, sc.b32, &rn, &bn);
        if (rc) return rc;
        rc = ldlt_factor_solve<float>(ctx, ctx->J32, ld, n, sc.b32, w, true, ctx->mixed_factor);
        if (rc) return rc;
        cudaEventRecord(ctx->t1.b, ctx->stream);
        k_axpy_f32<<<(n + 255) / 256, 256, 0, ctx->stream>>>(n, sc.b32, ctx->y), ++ctx->launches;
        int it = 1;
        double prev = 1e300;
        for (; it < 60; it++) {
            rc = resid_norms(ctx, ctx->y, ctx->G, sc.r, sc.b32, &rn, &bn);
            if (rc) return rc;
            if (!(rn > 1e-14 * bn) || rn > 0.7 * prev) break;
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
// One sweep of the reference's row-sequential Gauss-Seidel on the dense J, in
// one CTA: rows go in blocks of 32; the 32 warps first take each row's dot
// product with the current x over the columns outside the block (new values
// left of it, old values right of it), then one warp finishes the block's
// rows in order.  The iterate is the reference's, up to summation order.
// Rows with |J_uu| < 1e-12 keep their value (src/FESolver.cpp:569).
__global__ void __launch_bounds__(1024) k_gs_sweep(int neq, long long ld, const double *__restrict__ A,
                                                   const double *__restrict__ b, double *x) {
    __shared__ double s_t[32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int r0 = 0; r0 < neq; r0 += 32) {
        int rb = neq - r0 < 32 ? neq - r0 : 32;
        // off-block partial sums: warp w handles row r0+w
        if (warp < rb) {
            const double *row = A + (long long)(r0 + warp) * ld;
            double s = 0;
            for (int j = lane; j < neq; j += 32)
                if (j < r0 || j >= r0 + rb) s = fma(row[j], x[j], s);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) s_t[warp] = s;
        }
        __syncthreads();
        if (warp == 0) {
            int u = r0 + lane;
            double t = 0, diag = 1, xo = 0;
            bool act = lane < rb;
            if (act) {
                const double *row = A + (long long)u * ld;
                t = b[u] - s_t[lane];
                diag = row[u];
                xo = x[u];
                // within-block columns right of the diagonal use the old values
                for (int v = lane + 1; v < rb; v++) t -= row[r0 + v] * x[r0 + v];
            }
            for (int j = 0; j < rb; j++) {
                double xj = 0;
                if (lane == j) {
                    xj = fabs(diag) < 1e-12 ? xo : t / diag;
                    x[u] = xj;
                }
                xj = __shfl_sync(0xffffffffu, xj, j);
                if (act && lane > j) t -= A[(long long)u * ld + r0 + j] * xj;
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
    const int n = ctx->neq;
    const long long ld = (n + 31) & ~31ll;
    const double tol = 1e-4;
    int th = 256;
    long long bl = ((long long)n * 32 + th - 1) / th;
    double L2 = 0;
    int it;
    bool converged = false;
    for (it = 0; it < ctx->gs_max_sweeps; it++) {
        k_gs_sweep<<<1, 1024, 0, ctx->stream>>>(n, ld, ctx->J, ctx->G, ctx->y), ++ctx->launches;
        if (it % 25 == 0) {
            MP_CUDA(ctx, cudaMemsetAsync(ctx->scal + 3, 0, sizeof(double), ctx->stream));
            k_gs_resid<<<(unsigned)bl, th, 0, ctx->stream>>>(n, ld, ctx->J, ctx->G, ctx->y, ctx->scal + 3), ++ctx->launches;
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
    MP_CUDA(ctx, cudaGetLastError());
    if (st) {
        st->linear_iterations = it;
        st->linear_residual = L2;
        if (!converged) st->linear_failures++;
    }
    return MP_OK;
}

}  // namespace mp
