// Field-side bandwidth kernels of the Poisson-Boltzmann Newton step and the
// E-field gather: updateEf, the Boltzmann-electron vectors F1 and FP, the
// residual G = K d - F0 - F1, the Jacobian J = K - diag(FP), the Newton update
// and the device-side assembly of K and F0.
//
// Every per-equation sum that the reference accumulates element by element
// (addKe/addFe, src/FESolver.cpp:166-185) is a gather here over a CSR list of
// (tet, local node) pairs sorted by tet, so each entry is summed in the
// reference's element order and comes out bit-identical whenever its inputs
// are.  Only exp() (CUDA's vs the host libm's) and the dense GEMV's summation
// order can differ from the reference in the last bits.
#include <cmath>

#include "mp_internal.h"

namespace mp {

__constant__ double c_Na[4][8];

void upload_quadrature(cudaStream_t s) {
    Quadrature q = make_quadrature();
    cudaMemcpyToSymbolAsync(c_Na, q.Na, sizeof(q.Na), 0, cudaMemcpyHostToDevice, s);
}

// ---- updateEf, src/FESolver.cpp:622-636 ----------------------------------------------
__global__ void k_update_ef(int n_tets, const int *__restrict__ con, const double *__restrict__ nx,
                            const double *__restrict__ uh, double *ef, TetRec *tets, TetRec32 *tets32) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_tets) return;
    double f[3] = {0, 0, 0};
    for (int a = 0; a < 4; a++) {
        double u = uh[con[4 * e + a]];
        for (int d = 0; d < 3; d++) f[d] = __dsub_rn(f[d], __dmul_rn(nx[12 * e + 3 * a + d], u));
    }
    for (int d = 0; d < 3; d++) {
        ef[3 * e + d] = f[d];
        tets[e].ef[d] = f[d];
        if (tets32) tets32[e].ef[d] = (float)f[d];
    }
}

// ---- Boltzmann terms ---------------------------------------------------------------
// f[A] = (QE/EPS0)*(ion_den[n] + n0*exp((d[A]-phi0)/kTe))      (FESolver.cpp:493-495)
// fp[A] = -QE/EPS0*n0*exp((d[A]-phi0)/kTe)*(1/kTe)              (FESolver.cpp:374-376)
__global__ void k_node_terms(int n_nodes, const int *__restrict__ ID, const double *__restrict__ den,
                             const double *__restrict__ d, double qe_eps0, double mqe_eps0, double n0, double phi0,
                             double kTe, double inv_kTe, double *f, double *fp) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n_nodes) return;
    int A = ID[n];
    if (A < 0) return;
    double ex = exp(__ddiv_rn(__dsub_rn(d[A], phi0), kTe));
    if (f) f[A] = __dmul_rn(qe_eps0, __dadd_rn(den[n], __dmul_rn(n0, ex)));
    if (fp) fp[A] = __dmul_rn(__dmul_rn(__dmul_rn(mqe_eps0, n0), ex), inv_kTe);
}

// out[A] (+)= sum over the tets of equation A, in tet order, of
//   (sum_p term[A]*Na[a][p]*detJ[e]) * (1/8)          (FESolver.cpp:390-415, 497-523)
__global__ void k_eq_gather(int neq, const int *__restrict__ eq_ptr, const int *__restrict__ eq_tet,
                            const unsigned char *__restrict__ eq_a, const double *__restrict__ detJ,
                            const double *__restrict__ term, double *out, int accumulate) {
    int A = blockIdx.x * blockDim.x + threadIdx.x;
    if (A >= neq) return;
    double acc = accumulate ? out[A] : 0.0;
    double t = term[A];
    for (int k = eq_ptr[A]; k < eq_ptr[A + 1]; k++) {
        int e = eq_tet[k];
        int a = eq_a[k];
        double dj = detJ[e];
        double ff = 0;
#pragma unroll
        for (int p = 0; p < 8; p++) ff = __dadd_rn(ff, __dmul_rn(__dmul_rn(t, c_Na[a][p]), dj));
        ff = __dmul_rn(ff, 1.0 / 8.0);
        acc = __dadd_rn(acc, ff);
    }
    out[A] = acc;
}

int fe_build_f1(mp_ctx *ctx, const double *den_dev) {
    const double qe_eps0 = QE / EPS0;
    int th = 256;
    k_node_terms<<<(ctx->n_nodes + th - 1) / th, th, 0, ctx->stream>>>(
        ctx->n_nodes, ctx->ID, den_dev, ctx->d, qe_eps0, 0.0, ctx->n0, ctx->phi0, ctx->kTe, 1.0 / ctx->kTe,
        ctx->fvec, nullptr), ++ctx->launches;
    // F1 is accumulated, never cleared, exactly as buildF1Vector does (it only
    // adds to F1; startAssembly is the one place that zeroes it).
    k_eq_gather<<<(ctx->neq + th - 1) / th, th, 0, ctx->stream>>>(ctx->neq, ctx->eq_ptr, ctx->eq_tet, ctx->eq_a,
                                                                 ctx->detJ, ctx->fvec, ctx->F1, 1), ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

// ---- residual G = K d - F0 - F1 (FESolver.cpp:333-335): the sparse K's product,
// summed in the reference's column order (mp_sparse.cu).
int fe_residual(mp_ctx *ctx) { return fe_residual_sparse(ctx); }

// ---- J = K, J[u][u] -= FP[u] (FESolver.cpp:367-431) ----------------------------------
__global__ void k_copy_j(int neq, long long ld, const double *__restrict__ K, const double *__restrict__ FP,
                         double *J) {
    long long total = (long long)neq * ld;
    long long stride = (long long)gridDim.x * blockDim.x * 2;
    for (long long i = 2 * ((long long)blockIdx.x * blockDim.x + threadIdx.x); i < total; i += stride) {
        double2 k = *reinterpret_cast<const double2 *>(K + i);
        long long r = i / ld, c = i - r * ld;
        if (c == r) k.x = __dsub_rn(k.x, FP[r]);
        if (c + 1 == r) k.y = __dsub_rn(k.y, FP[r]);
        *reinterpret_cast<double2 *>(J + i) = k;
    }
}

// Mixed form: the FP32 Jacobian for the factorization, straight from K and FP:
// the lower triangle (all the LDL^T reads) of J = K - diag(FP), rounded to
// FP32.  One CTA per row.
__global__ void k_copy_j32(int neq, long long ld, const double *__restrict__ K, const double *__restrict__ FP,
                           float *J32) {
    for (long long r = blockIdx.x; r < neq; r += gridDim.x) {
        const double *kr = K + r * ld;
        float *jr = J32 + r * ld;
        for (long long c = 4 * threadIdx.x; c <= r; c += 4 * blockDim.x) {
            const double2 a = *reinterpret_cast<const double2 *>(kr + c);
            const double2 b = *reinterpret_cast<const double2 *>(kr + c + 2);
            double v[4] = {a.x, a.y, b.x, b.y};
            if (r >= c && r < c + 4) v[r - c] = __dsub_rn(v[r - c], FP[r]);
            *reinterpret_cast<float4 *>(jr + c) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
        }
    }
}

// K's lower triangle (in 4-wide groups, as k_copy_j32 writes J32) rounded to FP32
__global__ void k_k32_from_k(int neq, long long ld, const double *__restrict__ K, float *K32) {
    for (long long r = blockIdx.x; r < neq; r += gridDim.x) {
        const double *kr = K + r * ld;
        float *out = K32 + r * ld;
        for (long long c = 4 * threadIdx.x; c <= r; c += 4 * blockDim.x) {
            const double2 a = *reinterpret_cast<const double2 *>(kr + c);
            const double2 b = *reinterpret_cast<const double2 *>(kr + c + 2);
            *reinterpret_cast<float4 *>(out + c) = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
        }
    }
}

// J32 = K - diag(FP) from the FP32 copy of K; the diagonal from the FP64 K and
// FP, so J32 is the same as rounding the FP64 J (k_copy_j32)
__global__ void k_copy_j32_from32(int neq, long long ld, const float *__restrict__ K32,
                                  const double *__restrict__ K, const double *__restrict__ FP, float *J32) {
    for (long long r = blockIdx.x; r < neq; r += gridDim.x) {
        const float *kr = K32 + r * ld;
        float *jr = J32 + r * ld;
        for (long long c = 4 * threadIdx.x; c <= r; c += 4 * blockDim.x) {
            float4 v = *reinterpret_cast<const float4 *>(kr + c);
            if (r >= c && r < c + 4) {
                const float dg = (float)__dsub_rn(K[r * ld + r], FP[r]);
                if (r == c) v.x = dg;
                else if (r == c + 1) v.y = dg;
                else if (r == c + 2) v.z = dg;
                else v.w = dg;
            }
            *reinterpret_cast<float4 *>(jr + c) = v;
        }
    }
}

int fe_j32_from_k(mp_ctx *ctx) {
    const long long ld = (ctx->neq + 31) & ~31ll;
    if (!ctx->J32) MP_CUDA(ctx, cudaMalloc(&ctx->J32, sizeof(float) * (size_t)ld * ctx->neq));
    // K does not change between Newton steps: its FP32 copy is made once
    if (!ctx->K32) {
        if (cudaMalloc(&ctx->K32, sizeof(float) * (size_t)ld * ctx->neq) != cudaSuccess) {
            cudaGetLastError();
            ctx->K32 = nullptr;  // no room: build J32 from the FP64 K each time
        }
        ctx->k32_current = false;
    }
    if (ctx->K32) {
        if (!ctx->k32_current) {
            k_k32_from_k<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(ctx->neq, ld, ctx->K, ctx->K32),
                ++ctx->launches;
            ctx->k32_current = true;
        }
        k_copy_j32_from32<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(ctx->neq, ld, ctx->K32, ctx->K, ctx->FP,
                                                                       ctx->J32),
            ++ctx->launches;
    } else {
        k_copy_j32<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(ctx->neq, ld, ctx->K, ctx->FP, ctx->J32),
            ++ctx->launches;
    }
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

int fe_build_j(mp_ctx *ctx, int method, int form) {
    // the full symmetric J serves both dense solvers (Lapack reads only one
    // triangle); the sparse methods apply J = K - diag(FP) from K and FP
    int th = 256;
    k_node_terms<<<(ctx->n_nodes + th - 1) / th, th, 0, ctx->stream>>>(
        ctx->n_nodes, ctx->ID, nullptr, ctx->d, 0.0, -QE / EPS0, ctx->n0, ctx->phi0, ctx->kTe, 1 / ctx->kTe,
        nullptr, ctx->work), ++ctx->launches;
    k_eq_gather<<<(ctx->neq + th - 1) / th, th, 0, ctx->stream>>>(ctx->neq, ctx->eq_ptr, ctx->eq_tet, ctx->eq_a,
                                                                 ctx->detJ, ctx->work, ctx->FP, 0), ++ctx->launches;
    long long ld = (ctx->neq + 31) & ~31ll;
    if (method == MP_METHOD_SPARSE_CG || method == MP_METHOD_SPARSE_NEWTON || !ctx->K) {
        ctx->j32_current = false;
    } else if (form == MP_FORM_MIXED) {
        // the mixed form factors an FP32 copy and refines against K and FP: no FP64 J
        int rc = fe_j32_from_k(ctx);
        if (rc) return rc;
        ctx->j32_current = true;
    } else {
        // the FP64 J (neq^2 doubles) is allocated on its first use
        if (!ctx->J) MP_CUDA(ctx, cudaMalloc(&ctx->J, sizeof(double) * (size_t)ld * ctx->neq));
        k_copy_j<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(ctx->neq, ld, ctx->K, ctx->FP, ctx->J), ++ctx->launches;
        ctx->j32_current = false;
        ctx->j_current = true;
    }
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

// ---- d -= y ; L2 = sqrt(sum y^2)/neq (FESolver.cpp:341-349) ---------------------------
__global__ void k_update_d(int neq, double *d, const double *__restrict__ y, double *sumsq) {
    __shared__ double s_w[32];
    double s = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < neq; i += gridDim.x * blockDim.x) {
        double v = y[i];
        d[i] = __dsub_rn(d[i], v);
        s = fma(v, v, s);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? s_w[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) atomicAdd(sumsq, s);
    }
}

int fe_update_d(mp_ctx *ctx, double *l2_out) {
    MP_CUDA(ctx, cudaMemsetAsync(ctx->scal, 0, sizeof(double), ctx->stream));
    k_update_d<<<64, 256, 0, ctx->stream>>>(ctx->neq, ctx->d, ctx->y, ctx->scal), ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    if (l2_out) {
        MP_CUDA(ctx, cudaMemcpyAsync(ctx->scal_host, ctx->scal, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        *l2_out = std::sqrt(ctx->scal_host[0]) / ctx->neq;
    }
    return MP_OK;
}

// ---- uh = g (+ d on unknowns), FESolver.cpp:610-618 -----------------------------------
__global__ void k_uh(int n_nodes, const int *__restrict__ ID, const double *__restrict__ g,
                     const double *__restrict__ d, double *uh) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n_nodes) return;
    double u = g[n];
    int A = ID[n];
    if (A >= 0) u = __dadd_rn(u, d[A]);
    uh[n] = u;
}

int fe_uh(mp_ctx *ctx) {
    int th = 256;
    k_uh<<<(ctx->n_nodes + th - 1) / th, th, 0, ctx->stream>>>(ctx->n_nodes, ctx->ID, ctx->g, ctx->d, ctx->uh), ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

int launch_update_ef(mp_ctx *ctx) {
    int th = 256;
    k_update_ef<<<(ctx->n_tets + th - 1) / th, th, 0, ctx->stream>>>(ctx->n_tets, ctx->con, ctx->nx, ctx->uh,
                                                                     ctx->ef, ctx->tets, ctx->tets32), ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

// ---- preAssembly of K and F0 (FESolver.cpp:434-485) -----------------------------------
// One thread per equation P builds row P of K and F0[P], visiting P's tets in
// tet order, so every K[P][Q] and F0[P] is summed in the reference's order.
__global__ void k_assemble(int neq, long long ld, const int *__restrict__ eq_ptr, const int *__restrict__ eq_tet,
                           const unsigned char *__restrict__ eq_a, const int *__restrict__ LM,
                           const int *__restrict__ con, const double *__restrict__ nx,
                           const double *__restrict__ detJ, const double *__restrict__ g, double *K, double *F0) {
    int P = blockIdx.x * blockDim.x + threadIdx.x;
    if (P >= neq) return;
    double *row = K + (long long)P * ld;
    double f0 = 0;
    for (int k = eq_ptr[P]; k < eq_ptr[P + 1]; k++) {
        int e = eq_tet[k];
        int a = eq_a[k];
        double dj = detJ[e];
        double fg = 0;
        for (int b = 0; b < 4; b++) {
            double dot = 0;
            for (int dd = 0; dd < 3; dd++)
                dot = __dadd_rn(dot, __dmul_rn(nx[12 * e + 3 * a + dd], nx[12 * e + 3 * b + dd]));
            double ke = 0;
            double t = __dmul_rn(dot, dj);  // *W[i]*W[j]*W[k] with W = 1 is exact
            for (int p = 0; p < 8; p++) ke = __dadd_rn(ke, t);
            int Q = LM[4 * e + b];
            if (Q >= 0) row[Q] = __dadd_rn(row[Q], ke);
            fg = __dsub_rn(fg, __dmul_rn(ke, g[con[4 * e + b]]));
        }
        f0 = __dadd_rn(f0, __dadd_rn(0.0, fg));
    }
    F0[P] = f0;
}

int fe_assemble(mp_ctx *ctx) {
    long long ld = (ctx->neq + 31) & ~31ll;
    MP_CUDA(ctx, cudaMemsetAsync(ctx->K, 0, sizeof(double) * ld * ctx->neq, ctx->stream));
    int th = 128;
    k_assemble<<<(ctx->neq + th - 1) / th, th, 0, ctx->stream>>>(ctx->neq, ld, ctx->eq_ptr, ctx->eq_tet, ctx->eq_a,
                                                                 ctx->LM, ctx->con, ctx->nx, ctx->detJ, ctx->g,
                                                                 ctx->K, ctx->F0), ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

}  // namespace mp
