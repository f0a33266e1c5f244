// Sparse field solve: K in sliced-ELLPACK form (SELL-32), assembled on the
// device; G = K d - F0 - F1 by a sparse product in the reference's column
// order; J y = G (J = K - diag(FP)) by Jacobi-preconditioned conjugate
// gradients in FP64, one cooperative kernel per solve.
//
// K has about 15 nonzeros per row (the 14 mesh neighbours of a node and the
// node itself), so the dense neq x neq storage of FESolver (src/FESolver.cpp:
// 80-127, 434-485) is what limits the mesh size; the sparse form holds
// 12 B per nonzero and lets meshes with a few hundred thousand unknowns solve
// in one device-resident call.
//
// Layout.  Rows are grouped in slices of 32; entry k of row P (columns in
// ascending order) sits at sp_ptr[P >> 5] + 32 * k + (P & 31), so a warp
// reading entry k of its 32 rows reads 32 consecutive words.  A slice is as
// wide as its longest row; the padding has column = P and value 0.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "mp_internal.h"

namespace mp {

namespace {

constexpr int CG_THREADS = 512;
constexpr unsigned CG_SPIN_LIMIT = 1u << 22;
constexpr int CG_MAX_RESTARTS = 3;

enum CgStatus : unsigned { CG_OK = 0, CG_NOT_SPD = 1, CG_TIMEOUT = 2, CG_MAX_IT = 4 };

// Position of column Q in row P (rows are sorted), -1 if absent.
__device__ __forceinline__ long long sell_find(const int *__restrict__ col, long long base, int len, int Q) {
    int lo = 0, hi = len - 1;
    while (lo <= hi) {
        int m = (lo + hi) >> 1;
        int c = col[base + 32ll * m];
        if (c == Q) return base + 32ll * m;
        if (c < Q) lo = m + 1;
        else hi = m - 1;
    }
    return -1;
}

// preAssembly of K and F0 (src/FESolver.cpp:434-485) into the sliced layout:
// one thread per equation P visits P's tets in tet order, so every K[P][Q]
// and F0[P] is the same sum, in the same order, as the dense assembly's.
__global__ void k_assemble_sparse(int neq, const int *__restrict__ eq_ptr, const int *__restrict__ eq_tet,
                                  const unsigned char *__restrict__ eq_a, const int *__restrict__ LM,
                                  const int *__restrict__ con, const double *__restrict__ nx,
                                  const double *__restrict__ detJ, const double *__restrict__ g,
                                  const int *__restrict__ len, const long long *__restrict__ ptr,
                                  const int *__restrict__ col, double *val, double *F0, unsigned *bad) {
    int P = blockIdx.x * blockDim.x + threadIdx.x;
    if (P >= neq) return;
    const long long base = ptr[P >> 5] + (P & 31);
    const int L = len[P];
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
            if (Q >= 0) {
                long long at = sell_find(col, base, L, Q);
                if (at >= 0) val[at] = __dadd_rn(val[at], ke);
                else atomicOr(bad, 1u);
            }
            fg = __dsub_rn(fg, __dmul_rn(ke, g[con[4 * e + b]]));
        }
        f0 = __dadd_rn(f0, __dadd_rn(0.0, fg));
    }
    F0[P] = f0;
}

// Copies the nonzeros of a dense (row-major, leading dimension ld) K into the
// sliced layout.
__global__ void k_dense_to_sell(int neq, long long ld, const double *__restrict__ K, const int *__restrict__ len,
                                const long long *__restrict__ ptr, const int *__restrict__ col, double *val) {
    int P = blockIdx.x * blockDim.x + threadIdx.x;
    if (P >= neq) return;
    const long long base = ptr[P >> 5] + (P & 31);
    for (int k = 0; k < len[P]; k++) val[base + 32ll * k] = K[(long long)P * ld + col[base + 32ll * k]];
}

// G = K d - F0 - F1 (src/FESolver.cpp:333-335; matVecMultiply, src/maths.cpp:60-67):
// each row summed from zero in ascending column order with separate multiply
// and add roundings, which is the reference's dense sum with its zero
// products left out (adding a zero product leaves a sum unchanged).
__global__ void k_residual_sparse(int neq, const int *__restrict__ len, const long long *__restrict__ ptr,
                                  const int *__restrict__ col, const double *__restrict__ val,
                                  const double *__restrict__ d, const double *__restrict__ F0,
                                  const double *__restrict__ F1, double *G) {
    int P = blockIdx.x * blockDim.x + threadIdx.x;
    if (P >= neq) return;
    const long long base = ptr[P >> 5] + (P & 31);
    double s = 0;
    for (int k = 0; k < len[P]; k++) s = __dadd_rn(s, __dmul_rn(val[base + 32ll * k], d[col[base + 32ll * k]]));
    G[P] = __dsub_rn(__dsub_rn(s, F0[P]), F1[P]);
}

// ---- conjugate gradients ------------------------------------------------------------

struct CgArgs {
    int n;
    int rows_per_block;          // a multiple of 32
    const int *len;
    const long long *ptr;
    const int *col;
    const double *val;
    const double *FP;            // J = K - diag(FP)
    const double *b;
    double *x;                   // out; starts at zero; read by neighbour rows
    double *z;                   // preconditioned residual; read by neighbour rows
    double *r, *p, *q, *dinv;    // row state when it does not stay in registers
    double *ring;                // [3][2][gridDim.x] block partial sums (reduce_round)
    unsigned *sync;              // [0] abort, [1] status bits
    double *out;                 // [0] iterations, [1] ||b - J x||^2, [2] ||b||^2, [3] restarts
    double rtol2;
    int max_it;
};

// A ring slot not yet written this round: a NaN bit pattern (a block sum that
// happens to carry it is published as the canonical NaN instead).
constexpr unsigned long long EMPTY = 0xFFFFFFFFFFFFFFFFull;  // what a 0xFF byte fill writes

__device__ __forceinline__ double ld_relaxed_f64(const double *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return __longlong_as_double(v);
}
__device__ __forceinline__ void st_relaxed_f64(double *p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// One grid-wide reduction round, which is also the grid barrier (all blocks
// are resident: cooperative launch).  Each block publishes its NV block sums
// (fixed-order warp and block sums) into ring slot `round % 3` with a release
// store, after emptying its slot of ring index (round + 1) % 3: that index was
// last used by round - 2, which every block has finished reading, since every
// block has published round - 1.  Warp 0 of each block then polls all blocks'
// slots (bounded) until none is EMPTY, sums them lane-strided and by an XOR
// butterfly (each pairwise sum formed alike in both partners), so every
// thread of every block holds the same totals.  The acquire after the poll
// and the block barrier make every block's writes before its release (z, x)
// visible to all threads.  Returns false when the wait gave up or another
// block's did.
template <int NV>
__device__ bool reduce_round(const CgArgs &a, double (&v)[NV], unsigned &round, double *s_red, int *s_ok) {
    const int nb = gridDim.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; i++) {
        double t = v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) s_red[i * 32 + warp] = t;
    }
    __syncthreads();
    const int k = round % 3, kn = (round + 1) % 3;
    if (threadIdx.x == 0) {
        unsigned long long bits[NV];
#pragma unroll
        for (int i = 0; i < NV; i++) {
            double t = 0;
            for (int w = 0; w < CG_THREADS / 32; w++) t += s_red[i * 32 + w];
            bits[i] = (unsigned long long)__double_as_longlong(t);
            if (bits[i] == EMPTY) bits[i] = 0x7FF8000000000000ull;
            st_relaxed_f64(a.ring + (kn * 2 + i) * nb + blockIdx.x, EMPTY);
        }
        // release: the block's earlier writes (ordered before this thread by
        // the block barrier) and the emptied slots become visible to whoever
        // reads one of these values
        fence_acq_rel();
#pragma unroll
        for (int i = 0; i < NV; i++) st_relaxed_f64(a.ring + (k * 2 + i) * nb + blockIdx.x, bits[i]);
    }
    if (warp == 0) {
        double acc[NV];
        unsigned spins = 0;
        int ok = 1;
        while (true) {
            bool ready = true;
#pragma unroll
            for (int i = 0; i < NV; i++) {
                acc[i] = 0;
                for (int bb = lane; bb < nb; bb += 32) {
                    const double t = ld_relaxed_f64(a.ring + (k * 2 + i) * nb + bb);
                    if ((unsigned long long)__double_as_longlong(t) == EMPTY) ready = false;
                    acc[i] += t;
                }
            }
            if (__all_sync(0xffffffffu, ready)) break;
            ++spins;
            unsigned abort_seen = 0;
            if ((spins & 63) == 0 && lane == 0) abort_seen = *(volatile unsigned *)a.sync;
            abort_seen = __shfl_sync(0xffffffffu, abort_seen, 0);
            if (abort_seen) {
                ok = 0;
                break;
            }
            if (spins > CG_SPIN_LIMIT) {
                if (lane == 0) {
                    atomicExch(a.sync, 1u);
                    atomicOr(a.sync + 1, (unsigned)CG_TIMEOUT);
                }
                ok = 0;
                break;
            }
        }
        fence_acq_rel();  // acquire: the values seen were published after their blocks' writes
#pragma unroll
        for (int i = 0; i < NV; i++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
        }
        if (lane == 0) {
#pragma unroll
            for (int i = 0; i < NV; i++) s_red[64 + i] = acc[i];
            *s_ok = ok;
        }
    }
    __syncthreads();
    round++;
#pragma unroll
    for (int i = 0; i < NV; i++) v[i] = s_red[64 + i];
    const bool ok = *s_ok != 0;
    __syncthreads();  // s_red and s_ok are rewritten by the next round
    return ok;
}

// (J v)[i] = sum_k K[i][col_k] v[col_k] - FP[i] v[i]; v is read through L2
// (other blocks write it during the kernel).  The row is taken 16 entries at
// a time: all 16 column indices, then all 16 loads of v, so one row costs one
// L2 round trip (a mesh row has about 15 entries) instead of a chain of them.
__device__ __forceinline__ double j_row(const CgArgs &a, int i, long long base, int L, const double *v) {
    double s = 0;
    for (int k0 = 0; k0 < L; k0 += 16) {
        int c[16];
        double vv[16];
#pragma unroll
        for (int k = 0; k < 16; k++) c[k] = k0 + k < L ? __ldg(a.col + base + 32ll * (k0 + k)) : i;
#pragma unroll
        for (int k = 0; k < 16; k++) vv[k] = __ldcg(v + c[k]);
#pragma unroll
        for (int k = 0; k < 16; k++)
            if (k0 + k < L) s = fma(__ldg(a.val + base + 32ll * (k0 + k)), vv[k], s);
    }
    return fma(-__ldg(a.FP + i), __ldcg(v + i), s);
}

// Diagonal of J in row i.
__device__ __forceinline__ double j_diag(const CgArgs &a, int i) {
    const long long base = a.ptr[i >> 5] + (i & 31);
    double kd = 0;
    for (int k = 0; k < a.len[i]; k++)
        if (a.col[base + 32ll * k] == i) kd = a.val[base + 32ll * k];
    return kd - a.FP[i];
}

// A thread's rows r0 + threadIdx.x + j * CG_THREADS: in registers (RPT > 0
// rows a thread, loops unrolled) or, for more rows, in global memory read
// and written through L2 by the owning thread.
template <int RPT>
struct RowVec {
    double reg[RPT > 0 ? RPT : 1];
    double *g;
    __device__ __forceinline__ double get(int j, int i) const {
        if constexpr (RPT > 0) return reg[j];
        else return __ldcg(g + i);
    }
    __device__ __forceinline__ void set(int j, int i, double v) {
        if constexpr (RPT > 0) reg[j] = v;
        else __stcg(g + i, v);
    }
};

#define CG_ROWS(j, i)                                                                                   \
    for (int j = 0, i = r0 + (int)threadIdx.x; RPT > 0 ? j < RPT : i < r1; j++, i += CG_THREADS) \
        if (i < r1)

// J is definite with one sign for the whole matrix: with the reference's
// tet orientation detJ < 0, so K and the Boltzmann term -diag(FP) are both
// negative definite.  The kernel solves (sJ) x = s b with s the sign of J's
// first diagonal entry, and reports a row whose diagonal has the other sign.
//
// Jacobi-preconditioned CG with two reduction rounds per iteration, in the
// q-recurrence form: after z = D^-1 r the block sums of (r,z) and (r,r) are
// published together with z itself (round A); then w = J z, p = z + beta p,
// q = w + beta q (= J p) and the sums of (p,q) (round B).  When the
// recurrence residual meets the tolerance, the true residual b - J x is
// formed; if it misses, CG restarts from x (at most CG_MAX_RESTARTS times).
template <int RPT>
__global__ void __launch_bounds__(CG_THREADS, 1) k_cg(CgArgs a) {
    __shared__ double s_red[2 * 32 + 2];
    __shared__ int s_ok;
    const int r0 = blockIdx.x * a.rows_per_block;
    const int r1 = min(a.n, r0 + a.rows_per_block);
    unsigned round = 0;
    unsigned st = 0;
    const double sg = j_diag(a, 0) < 0 ? -1.0 : 1.0;
    RowVec<RPT> X{{}, a.x}, R{{}, a.r}, P{{}, a.p}, Q{{}, a.q}, D{{}, a.dinv}, Z{{}, a.z};
    long long base[RPT > 0 ? RPT : 1];
    int L[RPT > 0 ? RPT : 1];
#pragma unroll
    CG_ROWS(j, i) {
        double jd = sg * j_diag(a, i);
        if (!(jd > 0)) {
            st |= CG_NOT_SPD;
            jd = 1;
        }
        D.set(j, i, 1.0 / jd);
        X.set(j, i, 0.0);
        if constexpr (RPT > 0) {
            __stcg(a.x + i, 0.0);
            base[j] = a.ptr[i >> 5] + (i & 31);
            L[j] = a.len[i];
        }
    }
    if (st) atomicOr(a.sync + 1, st);
    auto row_base = [&](int j, int i) -> long long {
        if constexpr (RPT > 0) return base[j];
        else return __ldg(a.ptr + (i >> 5)) + (i & 31);
    };
    auto row_len = [&](int j, int i) -> int {
        if constexpr (RPT > 0) return L[j];
        else return __ldg(a.len + i);
    };

    double bb = 0, rz = 0, rr = 0;
    int it = 0, restarts = 0;
    bool first = true;
    while (true) {
        // residual phase: r = b - J x (x = 0 the first time)
        {
            double v[2] = {0, 0};
#pragma unroll
            CG_ROWS(j, i) {
                const double ri =
                    sg * (first ? a.b[i] : a.b[i] - j_row(a, i, row_base(j, i), row_len(j, i), a.x));
                const double zi = D.get(j, i) * ri;
                R.set(j, i, ri);
                Z.set(j, i, zi);
                if constexpr (RPT > 0) __stcg(a.z + i, zi);
                v[0] = fma(ri, zi, v[0]);
                v[1] = fma(ri, ri, v[1]);
            }
            if (!reduce_round<2>(a, v, round, s_red, &s_ok)) break;
            rz = v[0];
            rr = v[1];
            if (first) bb = rr;
        }
        if (rr <= a.rtol2 * bb) break;
        if (it >= a.max_it || (!first && restarts >= CG_MAX_RESTARTS)) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(a.sync + 1, (unsigned)CG_MAX_IT);
            break;
        }
        if (!first) restarts++;
        first = false;
        double beta = 0;
        while (true) {
            // w = J z; p = z + beta p; q = w + beta q
            double v[2] = {0, 0};
#pragma unroll
            CG_ROWS(j, i) {
                const double w = sg * j_row(a, i, row_base(j, i), row_len(j, i), a.z);
                const double zi = Z.get(j, i);
                const double pi = beta == 0 ? zi : fma(beta, P.get(j, i), zi);
                const double qi = beta == 0 ? w : fma(beta, Q.get(j, i), w);
                P.set(j, i, pi);
                Q.set(j, i, qi);
                v[0] = fma(pi, qi, v[0]);
            }
            if (!reduce_round<2>(a, v, round, s_red, &s_ok)) goto done;
            const double pq = v[0];
            if (!(pq > 0)) {
                if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(a.sync + 1, (unsigned)CG_NOT_SPD);
                goto done;
            }
            const double alpha = rz / pq;
            // x += alpha p; r -= alpha q; z = D^-1 r
            v[0] = v[1] = 0;
#pragma unroll
            CG_ROWS(j, i) {
                const double xi = fma(alpha, P.get(j, i), X.get(j, i));
                const double ri = fma(-alpha, Q.get(j, i), R.get(j, i));
                const double zi = D.get(j, i) * ri;
                X.set(j, i, xi);
                R.set(j, i, ri);
                Z.set(j, i, zi);
                if constexpr (RPT > 0) {
                    __stcg(a.x + i, xi);
                    __stcg(a.z + i, zi);
                }
                v[0] = fma(ri, zi, v[0]);
                v[1] = fma(ri, ri, v[1]);
            }
            if (!reduce_round<2>(a, v, round, s_red, &s_ok)) goto done;
            const double rz_new = v[0];
            rr = v[1];
            it++;
            if (rr <= a.rtol2 * bb || it >= a.max_it) break;
            beta = rz_new / rz;
            rz = rz_new;
        }
    }
done:
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out[0] = it;
        a.out[1] = rr;
        a.out[2] = bb;
        a.out[3] = restarts;
    }
}
#undef CG_ROWS

struct SparseScratch {
    double *vec = nullptr;       // r, z, p, q, dinv
    double *part = nullptr;
    unsigned *sync = nullptr;
    double *out = nullptr;
    double *out_host = nullptr;  // pinned [4] + status
    long long vec_len = 0;
    int part_len = 0;
};

SparseScratch *scratch_of(mp_ctx *ctx) {
    if (!ctx->sparse_scratch) ctx->sparse_scratch = new SparseScratch();
    return static_cast<SparseScratch *>(ctx->sparse_scratch);
}

}  // namespace

void sparse_free(mp_ctx *ctx) {
    void *dev[] = {ctx->sp_len, ctx->sp_ptr, ctx->sp_col, ctx->sp_val};
    for (void *p : dev)
        if (p) cudaFree(p);
    ctx->sp_len = nullptr;
    ctx->sp_ptr = nullptr;
    ctx->sp_col = nullptr;
    ctx->sp_val = nullptr;
    ctx->sp_nnz = ctx->sp_slots = 0;
    if (ctx->sparse_scratch) {
        SparseScratch *s = static_cast<SparseScratch *>(ctx->sparse_scratch);
        void *d2[] = {s->vec, s->part, s->sync, s->out};
        for (void *p : d2)
            if (p) cudaFree(p);
        if (s->out_host) cudaFreeHost(s->out_host);
        delete s;
        ctx->sparse_scratch = nullptr;
    }
}

// Column structure of K from LM: row P holds every equation that shares a
// tet with P (P included), in ascending order.
int sparse_setup(mp_ctx *ctx, const std::vector<int> &LM, const std::vector<int> &eq_ptr,
                 const std::vector<int> &eq_tet) {
    sparse_free(ctx);
    const int neq = ctx->neq;
    const int slices = (neq + 31) / 32;
    std::vector<int> len(neq), cols;
    std::vector<std::vector<int>> rows(neq);
    long long nnz = 0;
    for (int P = 0; P < neq; P++) {
        std::vector<int> &c = rows[P];
        c.reserve(4 * (eq_ptr[P + 1] - eq_ptr[P]));
        c.push_back(P);
        for (int k = eq_ptr[P]; k < eq_ptr[P + 1]; k++)
            for (int b = 0; b < 4; b++) {
                int Q = LM[4 * (size_t)eq_tet[k] + b];
                if (Q >= 0) c.push_back(Q);
            }
        std::sort(c.begin(), c.end());
        c.erase(std::unique(c.begin(), c.end()), c.end());
        len[P] = (int)c.size();
        nnz += len[P];
    }
    std::vector<long long> ptr(slices + 1, 0);
    for (int s = 0; s < slices; s++) {
        int w = 0;
        for (int P = 32 * s; P < std::min(neq, 32 * s + 32); P++) w = std::max(w, len[P]);
        ptr[s + 1] = ptr[s] + 32ll * w;
    }
    const long long slots = ptr[slices];
    std::vector<int> col(slots);
    for (int s = 0; s < slices; s++) {
        const int w = (int)((ptr[s + 1] - ptr[s]) / 32);
        for (int l = 0; l < 32; l++) {
            const int P = 32 * s + l;
            for (int k = 0; k < w; k++)
                col[ptr[s] + 32ll * k + l] = P < neq ? (k < len[P] ? rows[P][k] : P) : 0;
        }
    }
    MP_CUDA(ctx, cudaMalloc(&ctx->sp_len, sizeof(int) * std::max(1, neq)));
    MP_CUDA(ctx, cudaMalloc(&ctx->sp_ptr, sizeof(long long) * (slices + 1)));
    MP_CUDA(ctx, cudaMalloc(&ctx->sp_col, sizeof(int) * std::max(1ll, slots)));
    MP_CUDA(ctx, cudaMalloc(&ctx->sp_val, sizeof(double) * std::max(1ll, slots)));
    MP_CUDA(ctx, cudaMemcpy(ctx->sp_len, len.data(), sizeof(int) * neq, cudaMemcpyHostToDevice));
    MP_CUDA(ctx, cudaMemcpy(ctx->sp_ptr, ptr.data(), sizeof(long long) * (slices + 1), cudaMemcpyHostToDevice));
    if (slots) MP_CUDA(ctx, cudaMemcpy(ctx->sp_col, col.data(), sizeof(int) * slots, cudaMemcpyHostToDevice));
    MP_CUDA(ctx, cudaMemset(ctx->sp_val, 0, sizeof(double) * std::max(1ll, slots)));
    ctx->sp_nnz = nnz;
    ctx->sp_slots = slots;
    return MP_OK;
}

int fe_assemble_sparse(mp_ctx *ctx) {
    MP_CUDA(ctx, cudaMemsetAsync(ctx->sp_val, 0, sizeof(double) * std::max(1ll, ctx->sp_slots), ctx->stream));
    MP_CUDA(ctx, cudaMemsetAsync(ctx->scal + 4, 0, sizeof(double), ctx->stream));
    unsigned *bad = reinterpret_cast<unsigned *>(ctx->scal + 4);
    int th = 128;
    k_assemble_sparse<<<(ctx->neq + th - 1) / th, th, 0, ctx->stream>>>(
        ctx->neq, ctx->eq_ptr, ctx->eq_tet, ctx->eq_a, ctx->LM, ctx->con, ctx->nx, ctx->detJ, ctx->g, ctx->sp_len,
        ctx->sp_ptr, ctx->sp_col, ctx->sp_val, ctx->F0, bad),
        ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    unsigned h = 0;
    MP_CUDA(ctx, cudaMemcpyAsync(&h, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (h) return fail(ctx, MP_ERR_STATE, "sparse assembly: an entry outside the column structure");
    return MP_OK;
}

int fe_sparse_from_dense(mp_ctx *ctx) {
    const long long ld = (ctx->neq + 31) & ~31ll;
    int th = 128;
    k_dense_to_sell<<<(ctx->neq + th - 1) / th, th, 0, ctx->stream>>>(ctx->neq, ld, ctx->K, ctx->sp_len, ctx->sp_ptr,
                                                                      ctx->sp_col, ctx->sp_val),
        ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

// K given on the host, sparse storage only: gather the nonzeros on the host.
int fe_sparse_from_host(mp_ctx *ctx, const double *const *rows, const double *dense) {
    const int neq = ctx->neq;
    const int slices = (neq + 31) / 32;
    std::vector<int> len(neq);
    std::vector<long long> ptr(slices + 1);
    std::vector<int> col(ctx->sp_slots);
    std::vector<double> val(ctx->sp_slots, 0.0);
    MP_CUDA(ctx, cudaMemcpy(len.data(), ctx->sp_len, sizeof(int) * neq, cudaMemcpyDeviceToHost));
    MP_CUDA(ctx, cudaMemcpy(ptr.data(), ctx->sp_ptr, sizeof(long long) * (slices + 1), cudaMemcpyDeviceToHost));
    if (ctx->sp_slots)
        MP_CUDA(ctx, cudaMemcpy(col.data(), ctx->sp_col, sizeof(int) * ctx->sp_slots, cudaMemcpyDeviceToHost));
    for (int P = 0; P < neq; P++) {
        const double *row = rows ? rows[P] : dense + (size_t)P * neq;
        const long long base = ptr[P >> 5] + (P & 31);
        for (int k = 0; k < len[P]; k++) val[base + 32ll * k] = row[col[base + 32ll * k]];
    }
    if (ctx->sp_slots)
        MP_CUDA(ctx, cudaMemcpy(ctx->sp_val, val.data(), sizeof(double) * ctx->sp_slots, cudaMemcpyHostToDevice));
    return MP_OK;
}

// r = b - (K y - FP .* y) from the sparse K (a refinement residual reads 12 B
// per nonzero instead of the dense K's 8 neq^2 bytes); also emits r in FP32
// and adds ||r||^2, ||b||^2 into sums[0], sums[1] (one atomic per warp).
__global__ void k_resid_j_sparse(int neq, const int *__restrict__ len, const long long *__restrict__ ptr,
                                 const int *__restrict__ col, const double *__restrict__ val,
                                 const double *__restrict__ FP, const double *__restrict__ y,
                                 const double *__restrict__ b, double *r, float *r32, double *sums) {
    const int P = blockIdx.x * blockDim.x + threadIdx.x;
    double rr = 0.0, bb = 0.0;
    if (P < neq) {
        const long long base = ptr[P >> 5] + (P & 31);
        double sacc = 0.0;
        for (int k = 0; k < len[P]; k++) sacc = fma(val[base + 32ll * k], y[col[base + 32ll * k]], sacc);
        const double v = b[P] - (sacc - FP[P] * y[P]);
        if (r) r[P] = v;
        if (r32) r32[P] = (float)v;
        rr = v * v;
        bb = b[P] * b[P];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rr += __shfl_xor_sync(0xffffffffu, rr, o);
        bb += __shfl_xor_sync(0xffffffffu, bb, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&sums[0], rr);
        atomicAdd(&sums[1], bb);
    }
}

int fe_resid_j_sparse(mp_ctx *ctx, const double *y, const double *b, double *r, float *r32, double *sums) {
    const int th = 256;
    k_resid_j_sparse<<<(ctx->neq + th - 1) / th, th, 0, ctx->stream>>>(ctx->neq, ctx->sp_len, ctx->sp_ptr,
                                                                       ctx->sp_col, ctx->sp_val, ctx->FP, y, b,
                                                                       r, r32, sums),
        ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

int fe_residual_sparse(mp_ctx *ctx) {
    int th = 256;
    k_residual_sparse<<<(ctx->neq + th - 1) / th, th, 0, ctx->stream>>>(
        ctx->neq, ctx->sp_len, ctx->sp_ptr, ctx->sp_col, ctx->sp_val, ctx->d, ctx->F0, ctx->F1, ctx->G),
        ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

template <int RPT>
cudaError_t launch_cg(const CgArgs &a, int nb, cudaStream_t stream) {
    int occ = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cg<RPT>, CG_THREADS, 0);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorCooperativeLaunchTooLarge;
    CgArgs copy = a;
    void *args[] = {&copy};
    return cudaLaunchCooperativeKernel((const void *)k_cg<RPT>, dim3(nb), dim3(CG_THREADS), args, 0, stream);
}

// J y = G by conjugate gradients (FP must hold the current Boltzmann term).
// Rows are split in contiguous runs of rows_per_block (>= CG_THREADS) over at
// most one block per SM; a thread keeps its rows' state in registers up to 4
// rows (n <= 4 * 512 * SMs), in global memory beyond.
int fe_solve_cg(mp_ctx *ctx, mp_newton_stats *st) {
    const int n = ctx->neq;
    if (n <= 0) return MP_OK;
    SparseScratch *s = scratch_of(ctx);
    // one row a thread while the rows fit one block per SM: a thread's rows are
    // worked one after the other, which costs more than the longer grid-wide
    // rounds of more blocks (measured: 7.1 us an iteration at 8,379 unknowns
    // on 17 blocks, 10.6 us on 5 blocks of 4 rows a thread)
    const int max_blocks = ctx->sm_count;
    int rpb = (n + max_blocks - 1) / max_blocks;
    rpb = std::max(CG_THREADS, (rpb + 31) & ~31);
    const int nb = (n + rpb - 1) / rpb;
    const int rows_per_thread = (rpb + CG_THREADS - 1) / CG_THREADS;
    const long long ld = (n + 31) & ~31ll;
    if (s->vec_len < 5 * ld) {
        if (s->vec) cudaFree(s->vec);
        s->vec = nullptr;
        MP_CUDA(ctx, cudaMalloc(&s->vec, sizeof(double) * 5 * ld));
        s->vec_len = 5 * ld;
    }
    if (s->part_len < 6 * nb) {
        if (s->part) cudaFree(s->part);
        s->part = nullptr;
        MP_CUDA(ctx, cudaMalloc(&s->part, sizeof(double) * 6 * nb));
        s->part_len = 6 * nb;
    }
    if (!s->sync) {
        MP_CUDA(ctx, cudaMalloc(&s->sync, sizeof(unsigned) * 4));
        MP_CUDA(ctx, cudaMalloc(&s->out, sizeof(double) * 4));
        MP_CUDA(ctx, cudaHostAlloc(&s->out_host, sizeof(double) * 6, 0));
    }
    MP_CUDA(ctx, cudaMemsetAsync(s->sync, 0, sizeof(unsigned) * 4, ctx->stream));
    MP_CUDA(ctx, cudaMemsetAsync(s->part, 0xFF, sizeof(double) * 6 * nb, ctx->stream));  // every slot EMPTY
    CgArgs a;
    a.n = n;
    a.rows_per_block = rpb;
    a.len = ctx->sp_len;
    a.ptr = ctx->sp_ptr;
    a.col = ctx->sp_col;
    a.val = ctx->sp_val;
    a.FP = ctx->FP;
    a.b = ctx->G;
    a.x = ctx->y;
    a.r = s->vec;
    a.z = s->vec + ld;
    a.p = s->vec + 2 * ld;
    a.q = s->vec + 3 * ld;
    a.dinv = s->vec + 4 * ld;
    a.ring = s->part;
    a.sync = s->sync;
    a.out = s->out;
    a.rtol2 = ctx->cg_rtol * ctx->cg_rtol;
    a.max_it = ctx->cg_max_it;
    cudaError_t e = rows_per_thread == 1   ? launch_cg<1>(a, nb, ctx->stream)
                    : rows_per_thread == 2 ? launch_cg<2>(a, nb, ctx->stream)
                    : rows_per_thread <= 4 ? launch_cg<4>(a, nb, ctx->stream)
                                           : launch_cg<0>(a, nb, ctx->stream);
    MP_CUDA(ctx, e);
    ++ctx->launches;
    MP_CUDA(ctx, cudaMemcpyAsync(s->out_host, s->out, sizeof(double) * 4, cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaMemcpyAsync(s->out_host + 4, s->sync + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    unsigned status;
    std::memcpy(&status, s->out_host + 4, sizeof(unsigned));
    ctx->cg_last_iterations = (int)s->out_host[0];
    ctx->cg_last_restarts = (int)s->out_host[3];
    ctx->cg_last_relres = s->out_host[2] > 0 ? std::sqrt(s->out_host[1] / s->out_host[2]) : 0.0;
    if (st) {
        st->linear_iterations = (int)s->out_host[0];
        st->linear_residual = std::sqrt(s->out_host[1]) / n;
    }
    if (status & CG_TIMEOUT) return fail(ctx, MP_ERR_TIMEOUT, "conjugate gradients: a grid-wide wait gave up");
    if (status & CG_NOT_SPD) return fail(ctx, MP_ERR_SINGULAR, "conjugate gradients: J is not definite");
    if (status & CG_MAX_IT) return fail(ctx, MP_ERR_NOT_CONVERGED, "conjugate gradients: iteration limit reached");
    return MP_OK;
}

}  // namespace mp

using namespace mp;

int mp_set_fe_storage(mp_ctx *ctx, int storage) {
    if (!ctx || (storage != MP_FE_STORAGE_DENSE && storage != MP_FE_STORAGE_SPARSE)) return MP_ERR_ARG;
    if (ctx->fe_ready) return fail(ctx, MP_ERR_STATE, "storage is chosen before mp_fe_setup");
    ctx->fe_storage = storage;
    return MP_OK;
}

int mp_set_sparse_solver(mp_ctx *ctx, double rtol, int32_t max_iterations) {
    if (!ctx || !(rtol > 0) || !(rtol < 1) || max_iterations < 1) return MP_ERR_ARG;
    ctx->cg_rtol = rtol;
    ctx->cg_max_it = max_iterations;
    return MP_OK;
}

int mp_fe_sparse_matrix(mp_ctx *ctx, int64_t *nnz, int64_t *row_ptr, int32_t *col, double *val) {
    if (!ctx || !nnz) return MP_ERR_ARG;
    if (!ctx->fe_ready) return fail(ctx, MP_ERR_STATE, "no FE setup");
    *nnz = ctx->sp_nnz;
    if (!row_ptr && !col && !val) return MP_OK;
    if (!row_ptr || !col || !val) return MP_ERR_ARG;
    const int neq = ctx->neq;
    const int slices = (neq + 31) / 32;
    std::vector<int> len(neq), c(ctx->sp_slots);
    std::vector<long long> ptr(slices + 1);
    std::vector<double> v(ctx->sp_slots);
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    MP_CUDA(ctx, cudaMemcpy(len.data(), ctx->sp_len, sizeof(int) * neq, cudaMemcpyDeviceToHost));
    MP_CUDA(ctx, cudaMemcpy(ptr.data(), ctx->sp_ptr, sizeof(long long) * (slices + 1), cudaMemcpyDeviceToHost));
    if (ctx->sp_slots) {
        MP_CUDA(ctx, cudaMemcpy(c.data(), ctx->sp_col, sizeof(int) * ctx->sp_slots, cudaMemcpyDeviceToHost));
        MP_CUDA(ctx, cudaMemcpy(v.data(), ctx->sp_val, sizeof(double) * ctx->sp_slots, cudaMemcpyDeviceToHost));
    }
    long long o = 0;
    row_ptr[0] = 0;
    for (int P = 0; P < neq; P++) {
        const long long base = ptr[P >> 5] + (P & 31);
        for (int k = 0; k < len[P]; k++, o++) {
            col[o] = c[base + 32ll * k];
            val[o] = v[base + 32ll * k];
        }
        row_ptr[P + 1] = o;
    }
    return MP_OK;
}
