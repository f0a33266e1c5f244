// Particle push: E gather + kick + drift + barycentric tet walk + node-density
// scatter (MoveParticles, src/mini-pic.cpp:268-320; walk XtoLtet,
// src/meshes.h:75-100), and the removal of the particles that left the domain.
//
// The push updates each particle in place, one thread per particle, with no
// block-wide synchronisation: particle data crosses HBM once per step (read
// 52 B, write 52 B in FP64; 28 + 28 B in the mixed form).  A particle that
// leaves the domain becomes a hole (cell = -1) that later pushes skip.  Holes
// are removed, keeping the survivors' order (the reference's std::erase_if
// order), by the periodic tet re-sort or by a stable compaction pass that runs
// before any download and whenever holes exceed a fraction of the slots.
// Observable results (particle list, density) are those of a per-step removal.
#include <cuda/atomic>

#include "mp_internal.h"
#include "mp_walk.cuh"

namespace mp {

constexpr int PUSH_THREADS = 256;
constexpr double FIXED_SCALE = 1099511627776.0;  // 2^40
constexpr double NEAR_FACE = 1e-5;
// Mixed form: a particle whose FP64 weights are all within ON_FACE of [0, 1]
// lies on a face of the tet and stays in it.  The reference's weight formula
// can round a point on the face shared by two tets to slightly below zero in
// both (seen: -3.4e-15 and -3.4e-14 on a Kuhn diagonal plane), and the walk
// would then hop between the two forever; FP32 offsets land exactly on such
// planes often enough to meet this within a few million particle-steps.
constexpr double ON_FACE = 1e-10;

struct PushF64Args {
    PartsF64 p;
    const TetRec *__restrict__ tets;
    double *den;
    unsigned long long *den_fixed;
    unsigned long long *counters;
    double qm, dt;
    int walk_limit;
    int absorb;  // hop limit reached: remove the particle (counted in C_LOST) instead of raising the error
    int fixed;
    int track_ids;
};

struct PushF32Args {
    PartsF32 p;
    const TetRec32 *__restrict__ tets32;
    const TetRec *__restrict__ tets;
    const double *__restrict__ x0;   // [n_tets][4]
    double *den;
    unsigned long long *den_fixed;
    unsigned long long *counters;
    float qm_dt;                     // q/m * dt
    float dt;
    int walk_limit;
    int absorb;
    int fixed;
    int track_ids;
};

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Sums v[0..3] over the lanes that share `key` (one tet), leaving the sums in
// the group's lowest lane.  All 32 lanes must call it.  Returns true for the
// lanes that hold a group sum.
//
// Pointer jumping over each group's member list: every lane starts pointing at
// the next member above it and holds the sum of the members from itself up to
// (not including) the one it points at; each round adds the pointed-to
// lane's partial sum and takes over its pointer, so ceil(log2(group size))
// rounds leave the whole group's sum in its lowest lane.  A round is one vote,
// nine shuffles and four adds, and groups need not be contiguous (particles
// that hopped since the last tet sort sit between their tet's others).  This
// replaced a tree over group ranks that located the rank r + s member with a
// bit search each round: FP64 push 0.0905 -> 0.0868 ms, mixed 0.0660 ->
// 0.0592 ms on 2M ions sorted every 10 steps.  Summing runs of adjacent equal
// keys instead (no match) was slower (0.14 ms): a tet's lanes split into
// several runs once particles hop, and every run issues its own atomics.
template <typename T>
__device__ __forceinline__ bool group_sum4(int key, T v[4]) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned peers = __match_any_sync(FULL, key);
    const unsigned above = peers & (0xfffffffeu << lane);  // members above this lane
    int nxt = above ? __ffs(above) - 1 : -1;
    while (__any_sync(FULL, nxt >= 0)) {
        const int src = nxt >= 0 ? nxt : lane;
        T t[4];
#pragma unroll
        for (int i = 0; i < 4; i++) t[i] = __shfl_sync(FULL, v[i], src);
        const int n2 = __shfl_sync(FULL, nxt, src);
        if (nxt >= 0) {
#pragma unroll
            for (int i = 0; i < 4; i++) v[i] += t[i];
            nxt = n2;
        }
    }
    return (peers & ((1u << lane) - 1u)) == 0;
}

// Asynchronous global -> shared copies (cp.async, L2 only) for staging the
// FP64 kernel's next particle chunk without holding it in registers.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// One warp's 32-particle chunk of the FP64 arrays (px, py, pz, vx, vy, vz, cell).
struct ChunkF64 {
    double d[6][32];
    int cell[32];
};

// Stages chunk c of the FP64 particle arrays into b with 16-byte copies: lanes
// 0-15 and 16-31 take alternate arrays, lanes 0-7 the cells.  The arrays start
// on 256-byte boundaries and hold whole 256-particle tiles, so every copy is
// aligned and inside the allocation, also for the last, partly filled chunk.
__device__ __forceinline__ void stage_chunk_f64(const PartsF64 &p, long long c, ChunkF64 *b) {
    const int lane = threadIdx.x & 31;
    const int h = lane >> 4, q = lane & 15;
    const long long base = c * 32 + 2 * q;
    cp_async16(&b->d[h][2 * q], (h ? p.py : p.px) + base);
    cp_async16(&b->d[2 + h][2 * q], (h ? p.vx : p.pz) + base);
    cp_async16(&b->d[4 + h][2 * q], (h ? p.vz : p.vy) + base);
    if (lane < 8) cp_async16(&b->cell[4 * lane], p.cell + c * 32 + 4 * lane);
}

// Step statistics of one thread, accumulated over all the tiles a persistent
// CTA pushes and reduced once per warp when the kernel ends: a warp reduction
// per tile costs more than the scatter itself.
struct PushStats {
    unsigned hops = 0, hmax = 0, exits = 0, near = 0, lost = 0;
    __device__ __forceinline__ void add(int state, int h, int nr, int lst) {
        hops += (unsigned)h;
        hmax = hmax > (unsigned)h ? hmax : (unsigned)h;
        exits += state == 3;
        near += (unsigned)nr;
        lost += (unsigned)lst;
    }
    // all 32 lanes call it
    __device__ __forceinline__ void flush(unsigned long long *counters) {
        const unsigned FULL = 0xffffffffu;
        const unsigned hs = __reduce_add_sync(FULL, hops), hm = __reduce_max_sync(FULL, hmax);
        const unsigned ex = __reduce_add_sync(FULL, exits), nr = __reduce_add_sync(FULL, near);
        const unsigned ls = __reduce_add_sync(FULL, lost);
        if ((threadIdx.x & 31) == 0) {
            if (hs) {
                atomicAdd(&counters[C_HOPS], (unsigned long long)hs);
                atomicMax(&counters[C_MAX_HOPS], (unsigned long long)hm);
            }
            if (ex) {
                atomicAdd(&counters[C_EXITS], (unsigned long long)ex);
                atomicAdd(&counters[C_DEAD], (unsigned long long)ex);
            }
            if (nr) atomicAdd(&counters[C_NEAR], (unsigned long long)nr);
            if (ls) atomicAdd(&counters[C_LOST], (unsigned long long)ls);
        }
    }
};

// Density scatter of one warp, aggregated over the lanes that sit in one tet.
// All 32 lanes call it; `state` 1 = inside (scatter), 2 = kept after hitting
// the hop limit, 3 = left the domain, 0 = nothing.
template <typename Lc>
__device__ __forceinline__ void scatter_warp(int state, int cell, const int con[4], Lc lcv[4], double *den,
                                             unsigned long long *den_fixed, int fixed) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    int key = state == 1 ? cell : -2 - lane;
    if (fixed) {
        unsigned long long q[4];
#pragma unroll
        for (int i = 0; i < 4; i++)
            q[i] = state == 1 ? (unsigned long long)__double2ll_rn((double)lcv[i] * FIXED_SCALE) : 0ull;
        bool leader = group_sum4<unsigned long long>(key, q);
        if (leader && state == 1) {
#pragma unroll
            for (int i = 0; i < 4; i++) atomicAdd(&den_fixed[con[i]], q[i]);
        }
    } else {
        double sv[4];
#pragma unroll
        for (int i = 0; i < 4; i++) sv[i] = state == 1 ? (double)lcv[i] : 0.0;
        bool leader = group_sum4<double>(key, sv);
        if (leader && state == 1) {
#pragma unroll
            for (int i = 0; i < 4; i++) atomicAdd(&den[con[i]], sv[i]);
        }
    }
}

// Work division of both push kernels: each CTA takes one contiguous block of
// the (tet-sorted) particle array, and its 8 warps run its 32-particle chunks
// interleaved (warp w: chunks w, w + 8, ... of the block) with no block-wide
// barrier.  The CTA's warps thus walk the mesh together through a narrow band
// of tets, whose records and hop neighbours stay in that SM's L1; striding the
// warps over the whole array instead spread every SM over the whole mesh
// (L1 hit rate 34 % FP64 / 49 % mixed; FP64 0.0839 -> 0.0762 ms, mixed
// 0.0588 -> 0.0520 ms on 2M ions sorted every 10 steps).  Each warp fetches
// its next chunk before it computes the current one, so one chunk's HBM reads
// are always in flight behind the tet-record gathers.  The particles are updated in place.  This
// replaced 3-stage TMA bulk-copy staging of 256-particle tiles with a block
// barrier per tile: the barrier was the third stall reason, and without the
// staging buffers the L1 keeps more tet records (FP64 push 0.100 -> 0.093 ms
// on 2M sorted ions).
//
// The FP64 kernel fetches the next chunk with cp.async into a per-warp shared
// slot (two slots, 26 KB per CTA) instead of registers: the 13 registers of a
// register prefetch made it spill 92 bytes per thread at the 64-register
// bound of 4 CTAs per SM (0.0868 -> 0.0837 ms on 2M sorted ions).  The mixed
// kernel's prefetch needs 7 registers and does not spill; staging it was
// slower (0.0592 -> 0.0626 ms).
template <bool EXACT_CMP>
__global__ void __launch_bounds__(PUSH_THREADS, 4) k_push_fp64(PushF64Args a) {
    const long long n = (long long)a.counters[C_N];
    const int lane = threadIdx.x & 31;
    // this CTA's contiguous block of chunks [c, n_chunks), its warps interleaved
    const long long n_all = (n + 31) >> 5;
    const long long per = (n_all + gridDim.x - 1) / gridDim.x;
    const long long cta0 = (long long)blockIdx.x * per;
    const long long n_chunks = n_all < cta0 + per ? n_all : cta0 + per;
    const long long wstride = PUSH_THREADS / 32;
    long long c = cta0 + (threadIdx.x >> 5);
    PushStats stats;
    // two staging slots per warp: the chunk being pushed and the next one
    __shared__ __align__(16) ChunkF64 stage[PUSH_THREADS / 32][2];
    ChunkF64 *ws = stage[threadIdx.x >> 5];
    if (c < n_chunks) stage_chunk_f64(a.p, c, ws);
    cp_async_commit();
    int slot = 0;
    for (; c < n_chunks; c += wstride) {
        const long long i = c * 32 + lane;
        __syncwarp();  // every lane has read the slot the next chunk overwrites
        if (c + wstride < n_chunks) stage_chunk_f64(a.p, c + wstride, ws + (slot ^ 1));
        cp_async_commit();  // possibly empty: one group per chunk keeps the count
        cp_async_wait<1>();  // this chunk's group has landed
        __syncwarp();        // ... for every lane's copies
        const ChunkF64 *cb = ws + slot;
        slot ^= 1;
        int cell = cb->cell[lane];
        double x = cb->d[0][lane], y = cb->d[1][lane], z = cb->d[2][lane];
        double vx = cb->d[3][lane], vy = cb->d[4][lane], vz = cb->d[5][lane];
        int state = 0, hops = 0, lost = 0;
        int con[4] = {0, 0, 0, 0};
        double lc[4] = {0, 0, 0, 0};
        if (i < n && cell >= 0) {
            const TetRec *t = a.tets + cell;
            // v += q_over_m*ef*dt ; x += v*dt  (src/mini-pic.cpp:291-295)
            vx = __dadd_rn(vx, __dmul_rn(__dmul_rn(a.qm, __ldg(&t->ef[0])), a.dt));
            vy = __dadd_rn(vy, __dmul_rn(__dmul_rn(a.qm, __ldg(&t->ef[1])), a.dt));
            vz = __dadd_rn(vz, __dmul_rn(__dmul_rn(a.qm, __ldg(&t->ef[2])), a.dt));
            x = __dadd_rn(x, __dmul_rn(vx, a.dt));
            y = __dadd_rn(y, __dmul_rn(vy, a.dt));
            z = __dadd_rn(z, __dmul_rn(vz, a.dt));
            int w = walk_fp64<EXACT_CMP>(a.tets, cell, x, y, z, lc, a.walk_limit, hops);
            if (w == 1) {
                state = 1;
                const int4 c4 = __ldg(reinterpret_cast<const int4 *>(a.tets[cell].con));
                con[0] = c4.x; con[1] = c4.y; con[2] = c4.z; con[3] = c4.w;
            } else if (w == -1 && a.absorb) {
                state = 3;  // the point lies outside the mesh where the walk cannot end: absorbed
                cell = -1;
                lost = 1;
            } else if (w == -1) {
                state = 2;  // kept where the walk stopped, not scattered, error raised
                atomicOr(&a.counters[C_FLAGS], FLAG_WALK_LIMIT);
            } else {
                state = 3;
                cell = -1;
            }
            a.p.px[i] = x; a.p.py[i] = y; a.p.pz[i] = z;
            a.p.vx[i] = vx; a.p.vy[i] = vy; a.p.vz[i] = vz;
            a.p.cell[i] = cell;
        }
        scatter_warp<double>(state, cell, con, lc, a.den, a.den_fixed, a.fixed);
        stats.add(state, hops, 0, lost);
    }
    stats.flush(a.counters);
}

// Mixed form.  Position is an FP32 offset r from the owning tet's vertex 0 and
// the weights are lambda_i = [i==0] + g_i . r in FP32.  When the smallest
// weight is within 1e-5 of zero the inside test and the exit face are decided
// in FP64 with the reference's formula on x = x0 + r.  Walking to a new tet
// re-bases r on that tet's vertex 0 (in FP64, rounded once to FP32).
__device__ __forceinline__ void lambdas_fp32(const TetRec32 *__restrict__ t, float rx, float ry, float rz,
                                             float lc[4]) {
    const float4 gx = __ldg(reinterpret_cast<const float4 *>(t->gx));
    const float4 gy = __ldg(reinterpret_cast<const float4 *>(t->gy));
    const float4 gz = __ldg(reinterpret_cast<const float4 *>(t->gz));
    lc[0] = 1.0f + fmaf(gx.x, rx, fmaf(gy.x, ry, gz.x * rz));
    lc[1] = fmaf(gx.y, rx, fmaf(gy.y, ry, gz.y * rz));
    lc[2] = fmaf(gx.z, rx, fmaf(gy.z, ry, gz.z * rz));
    lc[3] = fmaf(gx.w, rx, fmaf(gy.w, ry, gz.w * rz));
}

__device__ __forceinline__ void load_x0(const double *__restrict__ x0, int cell, double &x, double &y, double &z) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(x0 + 4ll * cell));
    x = a.x;
    y = a.y;
    z = __ldg(x0 + 4ll * cell + 2);
}

__global__ void __launch_bounds__(PUSH_THREADS, 4) k_push_mixed(PushF32Args a) {
    const long long n = (long long)a.counters[C_N];
    const int lane = threadIdx.x & 31;
    // this CTA's contiguous block of chunks [c, n_chunks), its warps interleaved
    const long long n_all = (n + 31) >> 5;
    const long long per = (n_all + gridDim.x - 1) / gridDim.x;
    const long long cta0 = (long long)blockIdx.x * per;
    const long long n_chunks = n_all < cta0 + per ? n_all : cta0 + per;
    const long long wstride = PUSH_THREADS / 32;
    long long c = cta0 + (threadIdx.x >> 5);
    PushStats stats;
    int cell_n = -1;
    float rxn = 0, ryn = 0, rzn = 0, vxn = 0, vyn = 0, vzn = 0;
    if (c < n_chunks && c * 32 + lane < n) {
        const long long i0 = c * 32 + lane;
        cell_n = a.p.cell[i0];
        rxn = a.p.rx[i0]; ryn = a.p.ry[i0]; rzn = a.p.rz[i0];
        vxn = a.p.vx[i0]; vyn = a.p.vy[i0]; vzn = a.p.vz[i0];
    }
    for (; c < n_chunks; c += wstride) {
        const long long i = c * 32 + lane;
        int cell = cell_n;
        float rx = rxn, ry = ryn, rz = rzn, vx = vxn, vy = vyn, vz = vzn;
        {
            const long long in = (c + wstride) * 32 + lane;
            cell_n = -1;
            if (c + wstride < n_chunks && in < n) {
                cell_n = a.p.cell[in];
                rxn = a.p.rx[in]; ryn = a.p.ry[in]; rzn = a.p.rz[in];
                vxn = a.p.vx[in]; vyn = a.p.vy[in]; vzn = a.p.vz[in];
            }
        }
        int state = 0, hops = 0, near = 0, lost = 0;
        int con[4] = {0, 0, 0, 0};
        float lc[4] = {0, 0, 0, 0};
        if (i < n && cell >= 0) {
            const TetRec32 *t = a.tets32 + cell;
            vx = fmaf(a.qm_dt, __ldg(&t->ef[0]), vx);
            vy = fmaf(a.qm_dt, __ldg(&t->ef[1]), vy);
            vz = fmaf(a.qm_dt, __ldg(&t->ef[2]), vz);
            rx = fmaf(vx, a.dt, rx);
            ry = fmaf(vy, a.dt, ry);
            rz = fmaf(vz, a.dt, rz);
            for (;;) {
                const TetRec32 *tc = a.tets32 + cell;
                lambdas_fp32(tc, rx, ry, rz, lc);
                float mn = fminf(fminf(lc[0], lc[1]), fminf(lc[2], lc[3]));
                float mx = fmaxf(fmaxf(lc[0], lc[1]), fmaxf(lc[2], lc[3]));
                // lambda > 1 implies another lambda < 0, so min alone picks the near-face cases
                bool inside;
                int min_i = 0;
                if (fabsf(mn) < (float)NEAR_FACE) {
                    // decide in FP64 on the reconstructed absolute position
                    near++;
                    double ox, oy, oz;
                    load_x0(a.x0, cell, ox, oy, oz);
                    double x = ox + (double)rx, y = oy + (double)ry, z = oz + (double)rz;
                    double l64[4];
                    lambdas_fp64(a.tets + cell, x, y, z, l64);
                    inside = true;
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        if (l64[k] < -ON_FACE || l64[k] > 1.0 + ON_FACE) inside = false;
                        lc[k] = (float)l64[k];
                    }
                    double m64 = l64[0];
#pragma unroll
                    for (int k = 1; k < 4; k++)
                        if (l64[k] < m64) {
                            m64 = l64[k];
                            min_i = k;
                        }
                } else {
                    inside = mn >= 0.0f && mx <= 1.0f;
                    float m32 = lc[0];
#pragma unroll
                    for (int k = 1; k < 4; k++)
                        if (lc[k] < m32) {
                            m32 = lc[k];
                            min_i = k;
                        }
                }
                if (inside) {
                    state = 1;
                    break;
                }
                int nb = __ldg(&tc->cell_con[min_i]);
                if (nb < 0) {
                    state = 3;
                    cell = -1;
                    break;
                }
                if (hops >= a.walk_limit) {
                    if (a.absorb) {
                        state = 3;
                        cell = -1;
                        lost = 1;
                    } else {
                        state = 2;
                        atomicOr(&a.counters[C_FLAGS], FLAG_WALK_LIMIT);
                    }
                    break;
                }
                // re-base the offset on the new tet's vertex 0
                double ax, ay, az, bx, by, bz;
                load_x0(a.x0, cell, ax, ay, az);
                load_x0(a.x0, nb, bx, by, bz);
                rx = (float)((ax - bx) + (double)rx);
                ry = (float)((ay - by) + (double)ry);
                rz = (float)((az - bz) + (double)rz);
                cell = nb;
                hops++;
            }
            if (state == 1) {
                const int4 c4 = __ldg(reinterpret_cast<const int4 *>(a.tets32[cell].con));
                con[0] = c4.x; con[1] = c4.y; con[2] = c4.z; con[3] = c4.w;
            }
            a.p.rx[i] = rx; a.p.ry[i] = ry; a.p.rz[i] = rz;
            a.p.vx[i] = vx; a.p.vy[i] = vy; a.p.vz[i] = vz;
            a.p.cell[i] = cell;
        }
        scatter_warp<float>(state, cell, con, lc, a.den, a.den_fixed, a.fixed);
        stats.add(state, hops, near, lost);
    }
    stats.flush(a.counters);
}

// den[n] *= spwt/node_volume[n] (src/mini-pic.cpp:319); fixed-point sums are
// converted first.
__global__ void k_normalise(int n_nodes, double *den, const unsigned long long *den_fixed, int fixed,
                            const double *__restrict__ vol, double spwt, unsigned long long *counters) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n_nodes) {
        double v = fixed ? (double)den_fixed[i] * (1.0 / FIXED_SCALE) : den[i];
        den[i] = __dmul_rn(v, __ddiv_rn(spwt, vol[i]));
    }
}

static int grid_for(mp_ctx *ctx, const void *kernel, int threads, size_t smem) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (per_sm < 1) per_sm = 1;
    return per_sm * ctx->sm_count;
}

int launch_push(mp_ctx *ctx, double q_over_m, double dt) {
    // per-push statistics words
    MP_CUDA(ctx, cudaMemsetAsync(ctx->counters + C_EXITS, 0, 4 * sizeof(unsigned long long), ctx->stream));
    MP_CUDA(ctx, cudaMemsetAsync(ctx->counters + C_LOST, 0, sizeof(unsigned long long), ctx->stream));
    if (ctx->scatter_mode == MP_SCATTER_FIXED64)
        MP_CUDA(ctx, cudaMemsetAsync(ctx->den_fixed, 0, ctx->n_nodes * sizeof(unsigned long long), ctx->stream));
    else
        MP_CUDA(ctx, cudaMemsetAsync(ctx->den, 0, ctx->n_nodes * sizeof(double), ctx->stream));
    long long blocks = (ctx->n_host + PUSH_THREADS - 1) / PUSH_THREADS;
    if (blocks < 1) blocks = 1;
    if (ctx->form == MP_FORM_FP64) {
        PushF64Args a;
        a.p = ctx->p64[ctx->cur];
        a.tets = ctx->tets;
        a.den = ctx->den;
        a.den_fixed = ctx->den_fixed;
        a.counters = ctx->counters;
        a.qm = q_over_m;
        a.dt = dt;
        a.walk_limit = ctx->walk_limit;
        a.absorb = ctx->walk_absorb;
        a.fixed = ctx->scatter_mode == MP_SCATTER_FIXED64;
        a.track_ids = ctx->track_ids;
        // division-free inside test when every tet volume is below 1 (see walk_fp64)
        auto kern = ctx->small_tets ? k_push_fp64<true> : k_push_fp64<false>;
        if (!ctx->push_grid[0]) ctx->push_grid[0] = grid_for(ctx, (const void *)kern, PUSH_THREADS, 0);
        long long g = blocks < ctx->push_grid[0] ? blocks : ctx->push_grid[0];
        cudaEventRecord(ctx->tp.a, ctx->stream);
        kern<<<(unsigned)g, PUSH_THREADS, 0, ctx->stream>>>(a), ++ctx->launches;
        cudaEventRecord(ctx->tp.b, ctx->stream);
    } else {
        PushF32Args a;
        a.p = ctx->p32[ctx->cur];
        a.tets32 = ctx->tets32;
        a.tets = ctx->tets;
        a.x0 = ctx->tet_x0;
        a.den = ctx->den;
        a.den_fixed = ctx->den_fixed;
        a.counters = ctx->counters;
        a.qm_dt = (float)(q_over_m * dt);
        a.dt = (float)dt;
        a.walk_limit = ctx->walk_limit;
        a.absorb = ctx->walk_absorb;
        a.fixed = ctx->scatter_mode == MP_SCATTER_FIXED64;
        a.track_ids = ctx->track_ids;
        if (!ctx->push_grid[1]) ctx->push_grid[1] = grid_for(ctx, (const void *)k_push_mixed, PUSH_THREADS, 0);
        long long g = blocks < ctx->push_grid[1] ? blocks : ctx->push_grid[1];
        cudaEventRecord(ctx->tp.a, ctx->stream);
        k_push_mixed<<<(unsigned)g, PUSH_THREADS, 0, ctx->stream>>>(a), ++ctx->launches;
        cudaEventRecord(ctx->tp.b, ctx->stream);
    }
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

// ---- stable removal of holes -----------------------------------------------------------
constexpr int COMPACT_THREADS = 256;
constexpr int COMPACT_ITEMS = 4;  // particles per thread per block
constexpr int COMPACT_TILE = COMPACT_THREADS * COMPACT_ITEMS;

__global__ void k_compact_count(long long n, const int *__restrict__ cell, int *block_count) {
    __shared__ int s_w[COMPACT_THREADS / 32];
    long long base = (long long)blockIdx.x * COMPACT_TILE;
    int c = 0;
#pragma unroll
    for (int k = 0; k < COMPACT_ITEMS; k++) {
        long long i = base + k * COMPACT_THREADS + threadIdx.x;
        c += (i < n && cell[i] >= 0) ? 1 : 0;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < COMPACT_THREADS / 32; w++) t += s_w[w];
        block_count[blockIdx.x] = t;
    }
}

// Writes the live particles of each block, in order, at the block's offset.
template <typename P>
__global__ void k_compact_scatter(long long n, P in, P out, const int *__restrict__ block_off, int track_ids) {
    __shared__ int s_w[COMPACT_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long base = (long long)blockIdx.x * COMPACT_TILE;
    int run = block_off[blockIdx.x];
#pragma unroll 1
    for (int k = 0; k < COMPACT_ITEMS; k++) {
        long long i = base + k * COMPACT_THREADS + threadIdx.x;
        bool live = i < n && in.cell[i] >= 0;
        unsigned b = __ballot_sync(0xffffffffu, live);
        if (lane == 0) s_w[warp] = __popc(b);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < COMPACT_THREADS / 32; w++) {
            int c = s_w[w];
            if (w < warp) before += c;
            total += c;
        }
        if (live) {
            long long o = run + before + __popc(b & lanemask_lt());
            if constexpr (sizeof(*in.vx) == 8) {
                out.px[o] = in.px[i]; out.py[o] = in.py[i]; out.pz[o] = in.pz[i];
            } else {
                out.rx[o] = in.rx[i]; out.ry[o] = in.ry[i]; out.rz[o] = in.rz[i];
            }
            out.vx[o] = in.vx[i]; out.vy[o] = in.vy[i]; out.vz[o] = in.vz[i];
            out.cell[o] = in.cell[i];
            if (track_ids) out.id[o] = in.id[i];
        }
        run += total;
        __syncthreads();
    }
}

__global__ void k_set_counts(unsigned long long *counters, long long live) {
    counters[C_N] = (unsigned long long)live;
    counters[C_DEAD] = 0;
}

// Exclusive scan of hist[0..m) in place, one block (defined below).
__global__ void k_scan_single(int m, int *hist);

// Requires ctx->n_host and ctx->dead_host to be exact (after a counter sync).
int launch_compact(mp_ctx *ctx) {
    long long n = ctx->n_host;
    long long live = n - ctx->dead_host;
    if (ctx->dead_host == 0) return MP_OK;
    long long blocks = (n + COMPACT_TILE - 1) / COMPACT_TILE;
    if (!ctx->compact_off || ctx->compact_len < blocks + 1) {
        if (ctx->compact_off) cudaFree(ctx->compact_off);
        ctx->compact_off = nullptr;
        MP_CUDA(ctx, cudaMalloc(&ctx->compact_off, sizeof(int) * (blocks + 1) * 2));
        ctx->compact_len = (blocks + 1) * 2;
    }
    int nxt = ctx->cur ^ 1;
    const int *cell = ctx->form == MP_FORM_FP64 ? ctx->p64[ctx->cur].cell : ctx->p32[ctx->cur].cell;
    k_compact_count<<<(unsigned)blocks, COMPACT_THREADS, 0, ctx->stream>>>(n, cell, ctx->compact_off), ++ctx->launches;
    k_scan_single<<<1, 1024, 0, ctx->stream>>>((int)blocks, ctx->compact_off), ++ctx->launches;
    if (ctx->form == MP_FORM_FP64)
        k_compact_scatter<PartsF64><<<(unsigned)blocks, COMPACT_THREADS, 0, ctx->stream>>>(
            n, ctx->p64[ctx->cur], ctx->p64[nxt], ctx->compact_off, ctx->track_ids), ++ctx->launches;
    else
        k_compact_scatter<PartsF32><<<(unsigned)blocks, COMPACT_THREADS, 0, ctx->stream>>>(
            n, ctx->p32[ctx->cur], ctx->p32[nxt], ctx->compact_off, ctx->track_ids), ++ctx->launches;
    k_set_counts<<<1, 1, 0, ctx->stream>>>(ctx->counters, live), ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    ctx->cur = nxt;
    ctx->n_host = live;
    ctx->dead_host = 0;
    return MP_OK;
}

int launch_normalise(mp_ctx *ctx, double spwt) {
    int th = 256;
    int bl = (ctx->n_nodes + th - 1) / th;
    k_normalise<<<bl, th, 0, ctx->stream>>>(ctx->n_nodes, ctx->den, ctx->den_fixed,
                                            ctx->scatter_mode == MP_SCATTER_FIXED64, ctx->node_volume, spwt,
                                            ctx->counters), ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

// ---- append / download ----------------------------------------------------------

__global__ void k_append_f64(long long n, const double *__restrict__ pos, const double *__restrict__ vel,
                             const int *__restrict__ cell, int rewind, double qm, double half_dt,
                             const TetRec *__restrict__ tets, PartsF64 p, int track_ids,
                             const unsigned long long *counters) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long base = (long long)counters[C_N];
    long long o = base + i;
    int c = cell[i];
    double v[3] = {vel[i], vel[n + i], vel[2 * n + i]};
    if (rewind) {
        // part.vel[i] -= charge/mass*ef[i]*(0.5*dt), src/mini-pic.cpp:256-257
        for (int k = 0; k < 3; k++) v[k] = __dsub_rn(v[k], __dmul_rn(__dmul_rn(qm, __ldg(&tets[c].ef[k])), half_dt));
    }
    p.px[o] = pos[i]; p.py[o] = pos[n + i]; p.pz[o] = pos[2 * n + i];
    p.vx[o] = v[0]; p.vy[o] = v[1]; p.vz[o] = v[2];
    p.cell[o] = c;
    if (track_ids) p.id[o] = (long long)counters[C_NEXT_ID] + i;
}

__global__ void k_append_f32(long long n, const double *__restrict__ pos, const double *__restrict__ vel,
                             const int *__restrict__ cell, int rewind, double qm, double half_dt,
                             const TetRec *__restrict__ tets, const double *__restrict__ x0, PartsF32 p,
                             int track_ids, const unsigned long long *counters) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long base = (long long)counters[C_N];
    long long o = base + i;
    int c = cell[i];
    double v[3] = {vel[i], vel[n + i], vel[2 * n + i]};
    if (rewind)
        for (int k = 0; k < 3; k++) v[k] = __dsub_rn(v[k], __dmul_rn(__dmul_rn(qm, __ldg(&tets[c].ef[k])), half_dt));
    p.rx[o] = (float)(pos[i] - x0[4ll * c + 0]);
    p.ry[o] = (float)(pos[n + i] - x0[4ll * c + 1]);
    p.rz[o] = (float)(pos[2 * n + i] - x0[4ll * c + 2]);
    p.vx[o] = (float)v[0]; p.vy[o] = (float)v[1]; p.vz[o] = (float)v[2];
    p.cell[o] = c;
    if (track_ids) p.id[o] = (long long)counters[C_NEXT_ID] + i;
}

__global__ void k_append_commit(long long n, unsigned long long *counters) {
    counters[C_N] += (unsigned long long)n;
    counters[C_NEXT_ID] += (unsigned long long)n;
}

int launch_append(mp_ctx *ctx, long long n, const double *pos_soa, const double *vel_soa, const int *cell,
                  int rewind, double q_over_m, double half_dt) {
    if (n <= 0) return MP_OK;
    int th = 256;
    long long bl = (n + th - 1) / th;
    if (ctx->form == MP_FORM_FP64)
        k_append_f64<<<(unsigned)bl, th, 0, ctx->stream>>>(n, pos_soa, vel_soa, cell, rewind, q_over_m, half_dt,
                                                          ctx->tets, ctx->p64[ctx->cur], ctx->track_ids,
                                                          ctx->counters), ++ctx->launches;
    else
        k_append_f32<<<(unsigned)bl, th, 0, ctx->stream>>>(n, pos_soa, vel_soa, cell, rewind, q_over_m, half_dt,
                                                          ctx->tets, ctx->tet_x0, ctx->p32[ctx->cur],
                                                          ctx->track_ids, ctx->counters), ++ctx->launches;
    k_append_commit<<<1, 1, 0, ctx->stream>>>(n, ctx->counters), ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

// Packs the live particles into SoA FP64: pos[3][n], vel[3][n], lc[4][n] (the
// walk's weights in the current tet), cell[n], id[n].
__global__ void k_pack(long long n, int form, PartsF64 p, PartsF32 q, const TetRec *__restrict__ tets,
                       const double *__restrict__ x0, double *out, int *cell_out, long long *id_out, int track_ids) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double x, y, z, vx, vy, vz;
    int c;
    long long id = i;
    if (form == MP_FORM_FP64) {
        x = p.px[i]; y = p.py[i]; z = p.pz[i];
        vx = p.vx[i]; vy = p.vy[i]; vz = p.vz[i];
        c = p.cell[i];
        if (track_ids) id = p.id[i];
    } else {
        c = q.cell[i];
        x = x0[4ll * c] + (double)q.rx[i];
        y = x0[4ll * c + 1] + (double)q.ry[i];
        z = x0[4ll * c + 2] + (double)q.rz[i];
        vx = q.vx[i]; vy = q.vy[i]; vz = q.vz[i];
        if (track_ids) id = q.id[i];
    }
    double lc[4];
    lambdas_fp64(tets + c, x, y, z, lc);
    out[i] = x; out[n + i] = y; out[2 * n + i] = z;
    out[3 * n + i] = vx; out[4 * n + i] = vy; out[5 * n + i] = vz;
    for (int k = 0; k < 4; k++) out[(6 + k) * n + i] = lc[k];
    cell_out[i] = c;
    id_out[i] = id;
}

int launch_download_pack(mp_ctx *ctx, long long n, double *out_soa, int *cell_out, long long *id_out) {
    if (n <= 0) return MP_OK;
    int th = 256;
    long long bl = (n + th - 1) / th;
    k_pack<<<(unsigned)bl, th, 0, ctx->stream>>>(n, ctx->form, ctx->p64[ctx->cur], ctx->p32[ctx->cur], ctx->tets,
                                                 ctx->tet_x0, out_soa, cell_out, id_out, ctx->track_ids), ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    return MP_OK;
}

// ---- tet sort (counting sort by cell) ---------------------------------------------

__global__ void k_hist(long long n, const int *__restrict__ cell, int *hist) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n && cell[i] >= 0) atomicAdd(&hist[cell[i]], 1);
}

// exclusive scan of hist[0..m) in place, one block
__global__ void k_scan_single(int m, int *hist) {
    __shared__ int s_part[1024];
    int t = threadIdx.x;
    int chunk = (m + blockDim.x - 1) / blockDim.x;
    int b = t * chunk, e = min(m, b + chunk);
    int s = 0;
    for (int k = b; k < e; k++) s += hist[k];
    s_part[t] = s;
    __syncthreads();
    if (t == 0) {
        int run = 0;
        for (int k = 0; k < (int)blockDim.x; k++) {
            int c = s_part[k];
            s_part[k] = run;
            run += c;
        }
    }
    __syncthreads();
    int run = s_part[t];
    for (int k = b; k < e; k++) {
        int c = hist[k];
        hist[k] = run;
        run += c;
    }
}

template <typename P>
__global__ void k_sort_scatter(long long n, P in, P out, int *cursor, int track_ids) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = in.cell[i];
    if (c < 0) return;
    int o = atomicAdd(&cursor[c], 1);
    if constexpr (sizeof(*in.vx) == 8) {
        out.px[o] = in.px[i]; out.py[o] = in.py[i]; out.pz[o] = in.pz[i];
    } else {
        out.rx[o] = in.rx[i]; out.ry[o] = in.ry[i]; out.rz[o] = in.rz[i];
    }
    out.vx[o] = in.vx[i]; out.vy[o] = in.vy[i]; out.vz[o] = in.vz[i];
    out.cell[o] = c;
    if (track_ids) out.id[o] = in.id[i];
}

int launch_sort_by_tet(mp_ctx *ctx) {
    long long n = ctx->n_host;
    if (n <= 1) return MP_OK;
    if (!ctx->sort_hist) MP_CUDA(ctx, cudaMalloc(&ctx->sort_hist, sizeof(int) * (ctx->n_tets + 1)));
    MP_CUDA(ctx, cudaMemsetAsync(ctx->sort_hist, 0, sizeof(int) * ctx->n_tets, ctx->stream));
    int th = 256;
    long long bl = (n + th - 1) / th;
    int nxt = ctx->cur ^ 1;
    const int *cell = ctx->form == MP_FORM_FP64 ? ctx->p64[ctx->cur].cell : ctx->p32[ctx->cur].cell;
    k_hist<<<(unsigned)bl, th, 0, ctx->stream>>>(n, cell, ctx->sort_hist), ++ctx->launches;
    k_scan_single<<<1, 1024, 0, ctx->stream>>>(ctx->n_tets, ctx->sort_hist), ++ctx->launches;
    if (ctx->form == MP_FORM_FP64)
        k_sort_scatter<PartsF64><<<(unsigned)bl, th, 0, ctx->stream>>>(n, ctx->p64[ctx->cur], ctx->p64[nxt],
                                                                      ctx->sort_hist, ctx->track_ids), ++ctx->launches;
    else
        k_sort_scatter<PartsF32><<<(unsigned)bl, th, 0, ctx->stream>>>(n, ctx->p32[ctx->cur], ctx->p32[nxt],
                                                                      ctx->sort_hist, ctx->track_ids), ++ctx->launches;
    long long live = n - ctx->dead_host;
    k_set_counts<<<1, 1, 0, ctx->stream>>>(ctx->counters, live), ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    ctx->cur = nxt;
    ctx->n_host = live;
    ctx->dead_host = 0;
    return MP_OK;
}

// ---- form conversion ------------------------------------------------------------

__global__ void k_f64_to_f32(long long n, PartsF64 a, PartsF32 b, const double *__restrict__ x0, int track_ids) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = a.cell[i];
    b.rx[i] = (float)(a.px[i] - x0[4ll * c]);
    b.ry[i] = (float)(a.py[i] - x0[4ll * c + 1]);
    b.rz[i] = (float)(a.pz[i] - x0[4ll * c + 2]);
    b.vx[i] = (float)a.vx[i]; b.vy[i] = (float)a.vy[i]; b.vz[i] = (float)a.vz[i];
    b.cell[i] = c;
    if (track_ids) b.id[i] = a.id[i];
}

__global__ void k_f32_to_f64(long long n, PartsF32 b, PartsF64 a, const double *__restrict__ x0, int track_ids) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = b.cell[i];
    a.px[i] = x0[4ll * c] + (double)b.rx[i];
    a.py[i] = x0[4ll * c + 1] + (double)b.ry[i];
    a.pz[i] = x0[4ll * c + 2] + (double)b.rz[i];
    a.vx[i] = b.vx[i]; a.vy[i] = b.vy[i]; a.vz[i] = b.vz[i];
    a.cell[i] = c;
    if (track_ids) a.id[i] = b.id[i];
}

int launch_convert_form(mp_ctx *ctx, int to_form) {
    long long n = ctx->n_host;
    int nxt = ctx->cur ^ 1;
    if (n > 0) {
        int th = 256;
        long long bl = (n + th - 1) / th;
        if (to_form == MP_FORM_MIXED)
            k_f64_to_f32<<<(unsigned)bl, th, 0, ctx->stream>>>(n, ctx->p64[ctx->cur], ctx->p32[nxt], ctx->tet_x0,
                                                              ctx->track_ids), ++ctx->launches;
        else
            k_f32_to_f64<<<(unsigned)bl, th, 0, ctx->stream>>>(n, ctx->p32[ctx->cur], ctx->p64[nxt], ctx->tet_x0,
                                                              ctx->track_ids), ++ctx->launches;
        MP_CUDA(ctx, cudaGetLastError());
    }
    ctx->cur = nxt;
    ctx->form = to_form;
    return MP_OK;
}

}  // namespace mp
