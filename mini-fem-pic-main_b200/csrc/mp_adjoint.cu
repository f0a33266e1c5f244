// Adjoint of K push + scatter steps with respect to the node potential phi and
// the inlet drift velocity: MoveParticles (src/mini-pic.cpp:268-320) together
// with InjectIons' velocity set-up and half-step rewind (src/mini-pic.cpp:239-257).
//
// Model.  phi is held for the K steps, so ef = updateEf(phi)
// (src/FESolver.cpp:622-636) is fixed and every particle moves on its own:
//   injected at step k0:  v = dir*v_drift + v_th - (qm*ef[c])*(0.5*dt)
//   every step k:         v += (qm*ef[c])*dt ; x += v*dt ; XtoLtet walk
// Outputs: the node density of the last step's scatter, normalised as
// MoveParticles does (den *= spwt/Vnode), and the wall energy flux
//   F = sum over particles leaving through a wall face of spwt*(0.5*m)*|v|^2
// with v after the exit step's kick; a boundary face is a wall face when its
// three nodes are wall nodes.  The walk is piecewise fixed: cells and exits do
// not move under a perturbation, so given its cells a trajectory is affine in
// (phi, v_drift) and the derivatives here are exact for that model.
//
// Layout.  A particle keeps one slot for the K steps (no compaction or
// re-sort): the initial population, then each step's injections.  One thread
// runs one slot through all of its steps, so forward, reverse and tangent are
// each one kernel over the slots.  The forward stores each slot's state at the
// checkpoint steps k = C, 2C, ...; the reverse walks the segments from the last,
// restores the segment's checkpoint, recomputes the segment's steps (their
// start cells kept in a per-thread array) and runs the adjoint recurrences back
// over them:
//   xbar constant, vbar += dt*xbar (x' = x + v'dt), Ebar[c_k] += qm*dt*vbar
// seeded by the density (xbar = sum_i gbar[n_i]*spwt/V[n_i]*grad lambda_i at the
// final cell) or the flux (vbar = Fbar*spwt*m*v' at the exit step), and closed
// at injection by vdbar += dir.vbar, Ebar[c0] -= 0.5*qm*dt*vbar.  Finally
// phibar[n] = -sum over (e,a) with con[e][a] = n of NX[e][a].Ebar[e].
// The tangent (forward mode) carries (dx, dv) along the same cells.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "mp_internal.h"
#include "mp_walk.cuh"

namespace mp {

constexpr int ADJ_MAX_SEGMENT = 32;  // checkpoint interval limit (per-thread cell array)
constexpr int ADJ_THREADS = 256;

// path codes of the recorded walk (cells >= 0 are the step's end cell)
constexpr int PATH_EXIT_OTHER = -1, PATH_EXIT_WALL = -2, PATH_HOP_LIMIT = -3;
// slot outcomes
constexpr int KIND_ALIVE = 0, KIND_WALL = 1, KIND_OTHER = 2, KIND_LIMIT = 3;

struct AdjState {
    int K = 0, C = 0, nck = 0;
    double qm = 0, mass = 0, dt = 0, spwt = 0, dir[3] = {0, 0, 0};
    int record = 0;
    long long n = 0, cap = 0;
    // slot inputs [cap]
    double *px = nullptr, *py = nullptr, *pz = nullptr, *vx = nullptr, *vy = nullptr, *vz = nullptr;
    int *cell0 = nullptr, *first = nullptr;
    unsigned char *inj = nullptr;
    // tape of the last forward
    bool tape = false;
    int mode = MP_ADJ_WALK;
    double vd = 0;
    int *exit_step = nullptr, *cell_end = nullptr;
    signed char *kind = nullptr;
    double *ck = nullptr;   // [nck][6][cap]
    int *ck_cell = nullptr; // [nck][cap]
    int *path = nullptr;    // [K][cap] (record_path)
    bool path_valid = false;
    // mesh-sized
    double *nx = nullptr;       // [n_tets][12]
    double *ef = nullptr;       // [n_tets][3] ef of the tape's phi
    double *def = nullptr;      // [n_tets][3] tangent ef / reverse Ebar
    unsigned char *wall = nullptr;  // [n_tets] bit i: face opposite vertex i is a wall face
    double *nodes_a = nullptr, *nodes_b = nullptr;  // [n_nodes] scratch
    double *scal = nullptr;     // device [4]: flux, vdbar, dflux, spare
    double *scal_host = nullptr;
};

struct Slot {
    double x, y, z, vx, vy, vz;
    int cell;
};

struct AdjArgs {
    const TetRec *tets;
    const double *ef;
    const unsigned char *wall;
    long long n, cap;
    int K, C, walk_limit, pinned, record;
    double qm, mass, dt, spwt, vd, dir0, dir1, dir2;
    const double *px, *py, *pz, *vx, *vy, *vz;
    const int *cell0, *first;
    const unsigned char *inj;
    double *ck;
    int *ck_cell;
    int *path;
    int *exit_step, *cell_end;
    signed char *kind;
    double *scal;
    unsigned long long *flags;
};

__device__ __forceinline__ Slot start_slot(const AdjArgs &a, long long p) {
    Slot s{a.px[p], a.py[p], a.pz[p], a.vx[p], a.vy[p], a.vz[p], a.cell0[p]};
    if (a.inj[p]) {
        // vel = normal*ion_velocity (+ thermal part); vel -= charge/mass*ef*(0.5*dt)
        const double *e = a.ef + 3 * s.cell;
        const double hdt = 0.5 * a.dt;
        s.vx = __dsub_rn(__dadd_rn(__dmul_rn(a.dir0, a.vd), s.vx), __dmul_rn(__dmul_rn(a.qm, e[0]), hdt));
        s.vy = __dsub_rn(__dadd_rn(__dmul_rn(a.dir1, a.vd), s.vy), __dmul_rn(__dmul_rn(a.qm, e[1]), hdt));
        s.vz = __dsub_rn(__dadd_rn(__dmul_rn(a.dir2, a.vd), s.vz), __dmul_rn(__dmul_rn(a.qm, e[2]), hdt));
    }
    return s;
}

// v += q_over_m*ef*dt ; x += v*dt  (src/mini-pic.cpp:291-295), unfused
__device__ __forceinline__ void kick_drift(Slot &s, const double *ef, double qm, double dt) {
    const double *e = ef + 3 * s.cell;
    s.vx = __dadd_rn(s.vx, __dmul_rn(__dmul_rn(qm, e[0]), dt));
    s.vy = __dadd_rn(s.vy, __dmul_rn(__dmul_rn(qm, e[1]), dt));
    s.vz = __dadd_rn(s.vz, __dmul_rn(__dmul_rn(qm, e[2]), dt));
    s.x = __dadd_rn(s.x, __dmul_rn(s.vx, dt));
    s.y = __dadd_rn(s.y, __dmul_rn(s.vy, dt));
    s.z = __dadd_rn(s.z, __dmul_rn(s.vz, dt));
}

// Cell update of step k: the reference walk, or the recorded path when pinned.
// Returns KIND_*; lc holds the end cell's coordinates when walked and inside.
__device__ __forceinline__ int move_cell(const AdjArgs &a, Slot &s, int k, long long p, double lc[4]) {
    if (a.pinned) {
        const int c = a.path[(long long)k * a.cap + p];
        if (c >= 0) {
            s.cell = c;
            return KIND_ALIVE;
        }
        return c == PATH_EXIT_WALL ? KIND_WALL : c == PATH_EXIT_OTHER ? KIND_OTHER : KIND_LIMIT;
    }
    int cell = s.cell, hops = 0, face = 0;
    const int w = walk_fp64(a.tets, cell, s.x, s.y, s.z, lc, a.walk_limit, hops, &face);
    int r;
    if (w == 1) {
        s.cell = cell;
        r = KIND_ALIVE;
    } else if (w == 0) {
        r = ((a.wall[cell] >> face) & 1) ? KIND_WALL : KIND_OTHER;
    } else {
        r = KIND_LIMIT;
    }
    if (a.record)
        a.path[(long long)k * a.cap + p] =
            r == KIND_ALIVE ? cell : r == KIND_WALL ? PATH_EXIT_WALL : r == KIND_OTHER ? PATH_EXIT_OTHER : PATH_HOP_LIMIT;
    return r;
}

__device__ __forceinline__ void store_ck(const AdjArgs &a, int j, long long p, const Slot &s) {
    double *b = a.ck + (long long)j * 6 * a.cap;
    b[p] = s.x;
    b[a.cap + p] = s.y;
    b[2 * a.cap + p] = s.z;
    b[3 * a.cap + p] = s.vx;
    b[4 * a.cap + p] = s.vy;
    b[5 * a.cap + p] = s.vz;
    a.ck_cell[(long long)j * a.cap + p] = s.cell;
}
__device__ __forceinline__ Slot load_ck(const AdjArgs &a, int j, long long p) {
    const double *b = a.ck + (long long)j * 6 * a.cap;
    return Slot{b[p], b[a.cap + p], b[2 * a.cap + p], b[3 * a.cap + p], b[4 * a.cap + p], b[5 * a.cap + p],
                a.ck_cell[(long long)j * a.cap + p]};
}

// gradient of lambda_i = (1/6)(alpha - x beta + y gamma - z delta)/V
__device__ __forceinline__ void grad_lambda(const TetRec *t, int i, double g[3]) {
    const double s = 1.0 / (6.0 * t->volume);
    g[0] = -t->beta[i] * s;
    g[1] = t->gamma[i] * s;
    g[2] = -t->delta[i] * s;
}

__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += sh[i];
    return t;  // valid in thread 0
}

__global__ void k_adj_ef(int n_tets, const int *__restrict__ con, const double *__restrict__ nx,
                         const double *__restrict__ phi, double *ef) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_tets) return;
    double f[3] = {0, 0, 0};
    for (int a = 0; a < 4; a++) {
        const double u = phi[con[4 * e + a]];
        for (int d = 0; d < 3; d++) f[d] = __dsub_rn(f[d], __dmul_rn(nx[12 * e + 3 * a + d], u));
    }
    for (int d = 0; d < 3; d++) ef[3 * e + d] = f[d];
}

__global__ void k_adj_wall(int n_tets, const TetRec *__restrict__ tets, const unsigned char *__restrict__ wall_node,
                           unsigned char *wall) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_tets) return;
    unsigned char m = 0;
    for (int i = 0; i < 4; i++) {
        if (tets[e].cell_con[i] >= 0) continue;
        bool all = true;
        for (int j = 0; j < 4; j++)
            if (j != i && !wall_node[tets[e].con[j]]) all = false;
        if (all) m |= (unsigned char)(1u << i);
    }
    wall[e] = m;
}

__global__ void __launch_bounds__(ADJ_THREADS) k_adj_forward(AdjArgs a, double *den) {
    __shared__ double sh[ADJ_THREADS / 32];
    double flux = 0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < a.n;
         p += (long long)gridDim.x * blockDim.x) {
        Slot s = start_slot(a, p);
        const int k0 = a.first[p];
        int kind = KIND_ALIVE, ek = a.K;
        double lc[4] = {0, 0, 0, 0};
        for (int k = k0; k < a.K; k++) {
            if (k > k0 && k % a.C == 0) store_ck(a, k / a.C - 1, p, s);
            kick_drift(s, a.ef, a.qm, a.dt);
            kind = move_cell(a, s, k, p, lc);
            if (kind != KIND_ALIVE) {
                ek = k;
                break;
            }
        }
        if (kind == KIND_WALL) {
            const double v2 = __dadd_rn(__dadd_rn(__dmul_rn(s.vx, s.vx), __dmul_rn(s.vy, s.vy)), __dmul_rn(s.vz, s.vz));
            flux += __dmul_rn(a.spwt, __dmul_rn(0.5 * a.mass, v2));
        } else if (kind == KIND_LIMIT) {
            atomicOr(a.flags, FLAG_WALK_LIMIT);
        } else if (kind == KIND_ALIVE) {
            const TetRec *t = a.tets + s.cell;
            if (a.pinned) lambdas_fp64(t, s.x, s.y, s.z, lc);
            for (int i = 0; i < 4; i++) atomicAdd(&den[t->con[i]], lc[i]);
        }
        a.exit_step[p] = ek;
        a.kind[p] = (signed char)kind;
        a.cell_end[p] = kind == KIND_ALIVE ? s.cell : -1;
    }
    const double t = block_sum(flux, sh);
    if (threadIdx.x == 0 && t != 0) atomicAdd(&a.scal[0], t);
}

// den_out[n] = den[n] * (spwt / Vnode[n])   (the normalisation of MoveParticles)
__global__ void k_adj_normalise(int n_nodes, const double *__restrict__ den, const double *__restrict__ vol,
                                double spwt, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_nodes) out[i] = __dmul_rn(den[i], __ddiv_rn(spwt, vol[i]));
}

__global__ void __launch_bounds__(ADJ_THREADS) k_adj_reverse(AdjArgs a, const double *__restrict__ gbar,
                                                              const double *__restrict__ vol, double fbar,
                                                              double *ebar) {
    __shared__ double sh[ADJ_THREADS / 32];
    double vdbar = 0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < a.n;
         p += (long long)gridDim.x * blockDim.x) {
        const int kind = a.kind[p];
        if (kind != KIND_ALIVE && kind != KIND_WALL) continue;  // outputs do not depend on this slot
        const int k0 = a.first[p];
        const int last = kind == KIND_WALL ? a.exit_step[p] : a.K - 1;
        double xb[3] = {0, 0, 0}, vb[3] = {0, 0, 0};
        if (kind == KIND_ALIVE) {
            const TetRec *t = a.tets + a.cell_end[p];
            for (int i = 0; i < 4; i++) {
                const int nd = t->con[i];
                const double w = gbar[nd] * (a.spwt / vol[nd]);
                double g[3];
                grad_lambda(t, i, g);
                for (int d = 0; d < 3; d++) xb[d] += w * g[d];
            }
        }
        int cs[ADJ_MAX_SEGMENT];
        for (int j = last / a.C; j >= k0 / a.C; j--) {
            const int s0 = j * a.C;
            const int kb = s0 > k0 ? s0 : k0;
            const int ke = s0 + a.C - 1 < last ? s0 + a.C - 1 : last;
            Slot s = kb == k0 ? start_slot(a, p) : load_ck(a, j - 1, p);
            double lc[4];
            for (int k = kb; k <= ke; k++) {
                cs[k - s0] = s.cell;
                kick_drift(s, a.ef, a.qm, a.dt);
                if (k == last) {
                    if (kind == KIND_WALL) {
                        const double c = fbar * a.spwt * a.mass;
                        vb[0] = c * s.vx;
                        vb[1] = c * s.vy;
                        vb[2] = c * s.vz;
                    }
                } else if (k < ke) {
                    move_cell(a, s, k, p, lc);
                }
            }
            for (int k = ke; k >= kb; k--) {
                const int c = cs[k - s0];
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    vb[d] += a.dt * xb[d];
                    atomicAdd(&ebar[3 * c + d], a.qm * a.dt * vb[d]);
                }
            }
        }
        if (a.inj[p]) {
            vdbar += a.dir0 * vb[0] + a.dir1 * vb[1] + a.dir2 * vb[2];
            const int c = a.cell0[p];
#pragma unroll
            for (int d = 0; d < 3; d++) atomicAdd(&ebar[3 * c + d], -(a.qm * (0.5 * a.dt)) * vb[d]);
        }
    }
    const double t = block_sum(vdbar, sh);
    if (threadIdx.x == 0 && t != 0) atomicAdd(&a.scal[1], t);
}

// phibar[n] = -sum_{e,a: con[e][a]=n} NX[e][a] . Ebar[e]   (transpose of updateEf)
__global__ void k_adj_phibar(int n_tets, const int *__restrict__ con, const double *__restrict__ nx,
                             const double *__restrict__ ebar, double *phibar) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_tets) return;
    const double b0 = ebar[3 * e], b1 = ebar[3 * e + 1], b2 = ebar[3 * e + 2];
    if (b0 == 0 && b1 == 0 && b2 == 0) return;
    for (int a = 0; a < 4; a++) {
        const double *g = nx + 12 * e + 3 * a;
        atomicAdd(&phibar[con[4 * e + a]], -(g[0] * b0 + g[1] * b1 + g[2] * b2));
    }
}

// Tangent: d(den raw), d(flux) along (dphi -> def, dvd), replaying the tape's cells.
__global__ void __launch_bounds__(ADJ_THREADS) k_adj_tangent(AdjArgs a, const double *__restrict__ def, double dvd,
                                                              double *dden) {
    __shared__ double sh[ADJ_THREADS / 32];
    double dflux = 0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < a.n;
         p += (long long)gridDim.x * blockDim.x) {
        if (a.kind[p] == KIND_OTHER || a.kind[p] == KIND_LIMIT) continue;
        Slot s = start_slot(a, p);
        const int k0 = a.first[p];
        double dx[3] = {0, 0, 0}, dv[3] = {0, 0, 0};
        if (a.inj[p]) {
            const double *de = def + 3 * s.cell;
            const double dir[3] = {a.dir0, a.dir1, a.dir2};
            for (int d = 0; d < 3; d++) dv[d] = dir[d] * dvd - a.qm * de[d] * (0.5 * a.dt);
        }
        int kind = KIND_ALIVE;
        double lc[4];
        for (int k = k0; k < a.K; k++) {
            const double *de = def + 3 * s.cell;
            for (int d = 0; d < 3; d++) {
                dv[d] += a.qm * de[d] * a.dt;
                dx[d] += dv[d] * a.dt;
            }
            kick_drift(s, a.ef, a.qm, a.dt);
            kind = move_cell(a, s, k, p, lc);
            if (kind != KIND_ALIVE) break;
        }
        if (kind == KIND_WALL) {
            dflux += a.spwt * a.mass * (s.vx * dv[0] + s.vy * dv[1] + s.vz * dv[2]);
        } else if (kind == KIND_ALIVE) {
            const TetRec *t = a.tets + s.cell;
            for (int i = 0; i < 4; i++) {
                double g[3];
                grad_lambda(t, i, g);
                atomicAdd(&dden[t->con[i]], g[0] * dx[0] + g[1] * dx[1] + g[2] * dx[2]);
            }
        }
    }
    const double t = block_sum(dflux, sh);
    if (threadIdx.x == 0 && t != 0) atomicAdd(&a.scal[2], t);
}

static AdjState *state(mp_ctx *ctx) { return reinterpret_cast<AdjState *>(ctx->adjoint); }

void adjoint_free(mp_ctx *ctx) {
    AdjState *s = state(ctx);
    if (!s) return;
    void *dev[] = {s->px, s->py, s->pz, s->vx, s->vy, s->vz, s->cell0, s->first, s->inj, s->exit_step,
                   s->cell_end, s->kind, s->ck, s->ck_cell, s->path, s->ef, s->def, s->wall, s->nodes_a,
                   s->nodes_b, s->scal};
    for (void *p : dev)
        if (p) cudaFree(p);
    if (s->nx && s->nx != ctx->nx) cudaFree(s->nx);
    if (s->scal_host) cudaFreeHost(s->scal_host);
    delete s;
    ctx->adjoint = nullptr;
}

static AdjArgs args_of(mp_ctx *ctx, AdjState *s, bool pinned, bool record) {
    AdjArgs a;
    a.tets = ctx->tets;
    a.ef = s->ef;
    a.wall = s->wall;
    a.n = s->n;
    a.cap = s->cap;
    a.K = s->K;
    a.C = s->C;
    a.walk_limit = ctx->walk_limit;
    a.pinned = pinned;
    a.record = record;
    a.qm = s->qm;
    a.mass = s->mass;
    a.dt = s->dt;
    a.spwt = s->spwt;
    a.vd = s->vd;
    a.dir0 = s->dir[0];
    a.dir1 = s->dir[1];
    a.dir2 = s->dir[2];
    a.px = s->px; a.py = s->py; a.pz = s->pz;
    a.vx = s->vx; a.vy = s->vy; a.vz = s->vz;
    a.cell0 = s->cell0;
    a.first = s->first;
    a.inj = s->inj;
    a.ck = s->ck;
    a.ck_cell = s->ck_cell;
    a.path = s->path;
    a.exit_step = s->exit_step;
    a.cell_end = s->cell_end;
    a.kind = s->kind;
    a.scal = s->scal;
    a.flags = ctx->counters + C_FLAGS;
    return a;
}

static int grid_of(mp_ctx *ctx, long long n) {
    long long g = (n + ADJ_THREADS - 1) / ADJ_THREADS;
    long long cap = (long long)ctx->sm_count * 8;
    return (int)std::max(1ll, std::min(g, cap));
}

// grows the slot arrays to hold `need` slots, keeping the first s->n
static int grow_slots(mp_ctx *ctx, AdjState *s, long long need) {
    if (need <= s->cap) return MP_OK;
    long long cap = std::max(need, s->cap * 2);
    cap = (cap + 255) / 256 * 256;
    auto move = [&](auto *&ptr, size_t elem) -> int {
        void *p = nullptr;
        MP_CUDA(ctx, cudaMalloc(&p, elem * cap));
        if (ptr && s->n) MP_CUDA(ctx, cudaMemcpyAsync(p, ptr, elem * s->n, cudaMemcpyDeviceToDevice, ctx->stream));
        MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (ptr) cudaFree(ptr);
        ptr = reinterpret_cast<std::remove_reference_t<decltype(ptr)>>(p);
        return MP_OK;
    };
    int rc;
    if ((rc = move(s->px, 8)) || (rc = move(s->py, 8)) || (rc = move(s->pz, 8)) || (rc = move(s->vx, 8)) ||
        (rc = move(s->vy, 8)) || (rc = move(s->vz, 8)) || (rc = move(s->cell0, 4)) || (rc = move(s->first, 4)) ||
        (rc = move(s->inj, 1)))
        return rc;
    // the tape is sized by the capacity: reallocate it empty
    void *tape[] = {s->exit_step, s->cell_end, s->kind, s->ck, s->ck_cell, s->path};
    for (void *p : tape)
        if (p) cudaFree(p);
    s->exit_step = s->cell_end = nullptr;
    s->kind = nullptr;
    s->ck = nullptr;
    s->ck_cell = s->path = nullptr;
    MP_CUDA(ctx, cudaMalloc(&s->exit_step, 4 * cap));
    MP_CUDA(ctx, cudaMalloc(&s->cell_end, 4 * cap));
    MP_CUDA(ctx, cudaMalloc(&s->kind, cap));
    if (s->nck > 0) {
        MP_CUDA(ctx, cudaMalloc(&s->ck, sizeof(double) * 6 * cap * s->nck));
        MP_CUDA(ctx, cudaMalloc(&s->ck_cell, sizeof(int) * cap * s->nck));
    }
    if (s->record) MP_CUDA(ctx, cudaMalloc(&s->path, sizeof(int) * cap * s->K));
    s->cap = cap;
    s->tape = false;
    s->path_valid = false;
    return MP_OK;
}

}  // namespace mp

using namespace mp;

extern "C" {

int mp_adjoint_setup(mp_ctx *ctx, int32_t steps, int32_t checkpoint_every, double q_over_m, double mass, double dt,
                     double spwt, const double *inlet_dir, const uint8_t *wall_nodes, const double *nx,
                     int record_path) {
    if (!ctx || steps < 1 || checkpoint_every < 1 || checkpoint_every > ADJ_MAX_SEGMENT || !inlet_dir ||
        !wall_nodes || !(mass > 0) || !(dt > 0))
        return MP_ERR_ARG;
    if (!nx && !ctx->nx) return fail(ctx, MP_ERR_STATE, "adjoint setup needs NX (pass nx or call mp_fe_setup first)");
    adjoint_free(ctx);
    AdjState *s = new AdjState();
    ctx->adjoint = s;
    s->K = steps;
    s->C = checkpoint_every;
    s->nck = (steps - 1) / checkpoint_every;  // checkpoints at k = C, 2C, ... < K
    s->qm = q_over_m;
    s->mass = mass;
    s->dt = dt;
    s->spwt = spwt;
    for (int d = 0; d < 3; d++) s->dir[d] = inlet_dir[d];
    s->record = record_path ? 1 : 0;
    const int nt = ctx->n_tets, nn = ctx->n_nodes;
    if (nx) {
        MP_CUDA(ctx, cudaMalloc(&s->nx, sizeof(double) * 12 * nt));
        MP_CUDA(ctx, cudaMemcpyAsync(s->nx, nx, sizeof(double) * 12 * nt, cudaMemcpyDefault, ctx->stream));
    } else {
        s->nx = ctx->nx;
    }
    MP_CUDA(ctx, cudaMalloc(&s->ef, sizeof(double) * 3 * nt));
    MP_CUDA(ctx, cudaMalloc(&s->def, sizeof(double) * 3 * nt));
    MP_CUDA(ctx, cudaMalloc(&s->wall, nt));
    MP_CUDA(ctx, cudaMalloc(&s->nodes_a, sizeof(double) * nn));
    MP_CUDA(ctx, cudaMalloc(&s->nodes_b, sizeof(double) * nn));
    MP_CUDA(ctx, cudaMalloc(&s->scal, sizeof(double) * 4));
    MP_CUDA(ctx, cudaMallocHost(&s->scal_host, sizeof(double) * 4));
    unsigned char *wn = nullptr;
    MP_CUDA(ctx, cudaMalloc(&wn, nn));
    MP_CUDA(ctx, cudaMemcpyAsync(wn, wall_nodes, nn, cudaMemcpyDefault, ctx->stream));
    k_adj_wall<<<(nt + 255) / 256, 256, 0, ctx->stream>>>(nt, ctx->tets, wn, s->wall), ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    cudaFree(wn);
    return MP_OK;
}

int mp_adjoint_add_particles(mp_ctx *ctx, int32_t first_step, int injected, int64_t n, const double *pos,
                             const double *vel, const int32_t *cell) {
    AdjState *s = state(ctx);
    if (!ctx || !s) return ctx ? fail(ctx, MP_ERR_STATE, "no adjoint setup") : MP_ERR_ARG;
    if (n < 0 || first_step < 0 || first_step >= s->K || (n > 0 && (!pos || !vel || !cell))) return MP_ERR_ARG;
    if (n == 0) return MP_OK;
    std::vector<double> soa(6 * (size_t)n);
    std::vector<int> c(n), f(n, first_step);
    std::vector<unsigned char> in(n, injected ? 1 : 0);
    // pos/vel may be host or device memory: stage through the host
    std::vector<double> p3(3 * (size_t)n), v3(3 * (size_t)n);
    MP_CUDA(ctx, cudaMemcpy(p3.data(), pos, sizeof(double) * 3 * n, cudaMemcpyDefault));
    MP_CUDA(ctx, cudaMemcpy(v3.data(), vel, sizeof(double) * 3 * n, cudaMemcpyDefault));
    MP_CUDA(ctx, cudaMemcpy(c.data(), cell, sizeof(int) * n, cudaMemcpyDefault));
    for (int64_t i = 0; i < n; i++) {
        if (c[i] < 0 || c[i] >= ctx->n_tets) return fail(ctx, MP_ERR_ARG, "adjoint particle cell out of range");
        for (int d = 0; d < 3; d++) {
            soa[d * n + i] = p3[3 * i + d];
            soa[(3 + d) * n + i] = v3[3 * i + d];
        }
    }
    int rc = grow_slots(ctx, s, s->n + n);
    if (rc) return rc;
    double *dst[6] = {s->px, s->py, s->pz, s->vx, s->vy, s->vz};
    for (int d = 0; d < 6; d++)
        MP_CUDA(ctx, cudaMemcpyAsync(dst[d] + s->n, soa.data() + d * n, sizeof(double) * n, cudaMemcpyHostToDevice,
                                     ctx->stream));
    MP_CUDA(ctx, cudaMemcpyAsync(s->cell0 + s->n, c.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->stream));
    MP_CUDA(ctx, cudaMemcpyAsync(s->first + s->n, f.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->stream));
    MP_CUDA(ctx, cudaMemcpyAsync(s->inj + s->n, in.data(), n, cudaMemcpyHostToDevice, ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    s->n += n;
    s->tape = false;
    s->path_valid = false;
    return MP_OK;
}

int mp_adjoint_forward(mp_ctx *ctx, const double *phi, double v_drift, int mode, double *den_out,
                       mp_adjoint_stats *st) {
    AdjState *s = state(ctx);
    if (!ctx || !s) return ctx ? fail(ctx, MP_ERR_STATE, "no adjoint setup") : MP_ERR_ARG;
    if (!phi || (mode != MP_ADJ_WALK && mode != MP_ADJ_PINNED)) return MP_ERR_ARG;
    if (mode == MP_ADJ_PINNED && !s->path_valid)
        return fail(ctx, MP_ERR_STATE, "pinned forward needs a recorded walk (record_path and a walked forward)");
    const int nt = ctx->n_tets, nn = ctx->n_nodes;
    cudaEventRecord(ctx->t0.a, ctx->stream);
    MP_CUDA(ctx, cudaMemcpyAsync(s->nodes_b, phi, sizeof(double) * nn, cudaMemcpyDefault, ctx->stream));
    k_adj_ef<<<(nt + 255) / 256, 256, 0, ctx->stream>>>(nt, ctx->con, s->nx, s->nodes_b, s->ef), ++ctx->launches;
    MP_CUDA(ctx, cudaMemsetAsync(s->nodes_a, 0, sizeof(double) * nn, ctx->stream));
    MP_CUDA(ctx, cudaMemsetAsync(s->scal, 0, sizeof(double) * 4, ctx->stream));
    s->vd = v_drift;
    const bool pinned = mode == MP_ADJ_PINNED;
    const bool record = s->record && !pinned;
    AdjArgs a = args_of(ctx, s, pinned, record);
    if (s->n > 0)
        k_adj_forward<<<grid_of(ctx, s->n), ADJ_THREADS, 0, ctx->stream>>>(a, s->nodes_a), ++ctx->launches;
    k_adj_normalise<<<(nn + 255) / 256, 256, 0, ctx->stream>>>(nn, s->nodes_a, ctx->node_volume, s->spwt,
                                                               s->nodes_b), ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    cudaEventRecord(ctx->t0.b, ctx->stream);
    if (den_out) MP_CUDA(ctx, cudaMemcpyAsync(den_out, s->nodes_b, sizeof(double) * nn, cudaMemcpyDefault, ctx->stream));
    MP_CUDA(ctx, cudaMemcpyAsync(s->scal_host, s->scal, sizeof(double) * 4, cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaMemcpyAsync(ctx->counters_host + C_FLAGS, ctx->counters + C_FLAGS, sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    s->tape = true;
    s->mode = mode;
    if (record) s->path_valid = true;
    if (st) {
        std::memset(st, 0, sizeof(*st));
        std::vector<signed char> kind(s->n);
        if (s->n) MP_CUDA(ctx, cudaMemcpy(kind.data(), s->kind, s->n, cudaMemcpyDeviceToHost));
        st->slots = s->n;
        for (signed char k : kind) {
            if (k == KIND_ALIVE) st->alive++;
            else if (k == KIND_WALL) st->wall_exits++;
            else if (k == KIND_OTHER) st->other_exits++;
        }
        st->flux = s->scal_host[0];
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->t0.a, ctx->t0.b);
        st->ms = ms;
    }
    if (ctx->counters_host[C_FLAGS] & FLAG_WALK_LIMIT) {
        unsigned long long keep = ctx->counters_host[C_FLAGS] & ~FLAG_WALK_LIMIT;
        MP_CUDA(ctx, cudaMemcpy(ctx->counters + C_FLAGS, &keep, sizeof(keep), cudaMemcpyHostToDevice));
        return fail(ctx, MP_ERR_WALK_LIMIT, "adjoint forward: a tet walk exceeded the hop limit");
    }
    return MP_OK;
}

int mp_adjoint_flux(mp_ctx *ctx, double *flux) {
    AdjState *s = state(ctx);
    if (!ctx || !s || !flux) return MP_ERR_ARG;
    if (!s->tape) return fail(ctx, MP_ERR_STATE, "no adjoint forward yet");
    *flux = s->scal_host[0];
    return MP_OK;
}

int mp_adjoint_backward(mp_ctx *ctx, const double *den_bar, double flux_bar, double *phi_bar, double *v_drift_bar) {
    AdjState *s = state(ctx);
    if (!ctx || !s) return ctx ? fail(ctx, MP_ERR_STATE, "no adjoint setup") : MP_ERR_ARG;
    if (!s->tape) return fail(ctx, MP_ERR_STATE, "no adjoint forward yet");
    const int nt = ctx->n_tets, nn = ctx->n_nodes;
    if (den_bar)
        MP_CUDA(ctx, cudaMemcpyAsync(s->nodes_a, den_bar, sizeof(double) * nn, cudaMemcpyDefault, ctx->stream));
    else
        MP_CUDA(ctx, cudaMemsetAsync(s->nodes_a, 0, sizeof(double) * nn, ctx->stream));
    MP_CUDA(ctx, cudaMemsetAsync(s->def, 0, sizeof(double) * 3 * nt, ctx->stream));
    MP_CUDA(ctx, cudaMemsetAsync(s->nodes_b, 0, sizeof(double) * nn, ctx->stream));
    MP_CUDA(ctx, cudaMemsetAsync(s->scal + 1, 0, sizeof(double), ctx->stream));
    AdjArgs a = args_of(ctx, s, s->mode == MP_ADJ_PINNED, false);
    if (s->n > 0)
        k_adj_reverse<<<grid_of(ctx, s->n), ADJ_THREADS, 0, ctx->stream>>>(a, s->nodes_a, ctx->node_volume, flux_bar,
                                                                          s->def), ++ctx->launches;
    k_adj_phibar<<<(nt + 255) / 256, 256, 0, ctx->stream>>>(nt, ctx->con, s->nx, s->def, s->nodes_b),
        ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    if (phi_bar) MP_CUDA(ctx, cudaMemcpyAsync(phi_bar, s->nodes_b, sizeof(double) * nn, cudaMemcpyDefault, ctx->stream));
    MP_CUDA(ctx, cudaMemcpyAsync(s->scal_host + 1, s->scal + 1, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (v_drift_bar) *v_drift_bar = s->scal_host[1];
    return MP_OK;
}

int mp_adjoint_tangent(mp_ctx *ctx, const double *dphi, double dv_drift, double *dden, double *dflux) {
    AdjState *s = state(ctx);
    if (!ctx || !s) return ctx ? fail(ctx, MP_ERR_STATE, "no adjoint setup") : MP_ERR_ARG;
    if (!s->tape) return fail(ctx, MP_ERR_STATE, "no adjoint forward yet");
    const int nt = ctx->n_tets, nn = ctx->n_nodes;
    if (dphi) {
        MP_CUDA(ctx, cudaMemcpyAsync(s->nodes_b, dphi, sizeof(double) * nn, cudaMemcpyDefault, ctx->stream));
        k_adj_ef<<<(nt + 255) / 256, 256, 0, ctx->stream>>>(nt, ctx->con, s->nx, s->nodes_b, s->def),
            ++ctx->launches;
    } else {
        MP_CUDA(ctx, cudaMemsetAsync(s->def, 0, sizeof(double) * 3 * nt, ctx->stream));
    }
    MP_CUDA(ctx, cudaMemsetAsync(s->nodes_a, 0, sizeof(double) * nn, ctx->stream));
    MP_CUDA(ctx, cudaMemsetAsync(s->scal + 2, 0, sizeof(double), ctx->stream));
    AdjArgs a = args_of(ctx, s, s->mode == MP_ADJ_PINNED, false);
    if (s->n > 0)
        k_adj_tangent<<<grid_of(ctx, s->n), ADJ_THREADS, 0, ctx->stream>>>(a, s->def, dv_drift, s->nodes_a),
            ++ctx->launches;
    k_adj_normalise<<<(nn + 255) / 256, 256, 0, ctx->stream>>>(nn, s->nodes_a, ctx->node_volume, s->spwt,
                                                               s->nodes_b), ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    if (dden) MP_CUDA(ctx, cudaMemcpyAsync(dden, s->nodes_b, sizeof(double) * nn, cudaMemcpyDefault, ctx->stream));
    MP_CUDA(ctx, cudaMemcpyAsync(s->scal_host + 2, s->scal + 2, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (dflux) *dflux = s->scal_host[2];
    return MP_OK;
}

}  // extern "C"
