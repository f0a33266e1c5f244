// The C ABI (include/minipic_cuda.h): contexts, mesh and particle transfer,
// and the orchestration of MoveParticles and FESolver::computePhi on one
// stream.  There is no host compute path: every numerical step below is a
// kernel launch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "mp_internal.h"

namespace mp {

void upload_quadrature(cudaStream_t s);

int fail(mp_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->last_error = msg;
    return code;
}

int cuda_fail(mp_ctx *ctx, cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    if (ctx) ctx->last_error = m;
    return e == cudaErrorMemoryAllocation ? MP_ERR_OOM : MP_ERR_CUDA;
}

int kt_begin(mp_ctx *ctx, int cls, double work) {
    if (!(ctx->ktime_mask >> cls & 1u)) return -1;
    cudaEvent_t ev[2];
    for (int k = 0; k < 2; k++) {
        if (ctx->kevents.empty()) {
            if (cudaEventCreate(&ev[k]) != cudaSuccess) return -1;
        } else {
            ev[k] = ctx->kevents.back();
            ctx->kevents.pop_back();
        }
    }
    cudaEventRecord(ev[0], ctx->stream);
    ctx->kmarks.push_back(KernelMark{cls, work, ev[0], ev[1]});
    return (int)ctx->kmarks.size() - 1;
}

void kt_end(mp_ctx *ctx, int mark) {
    if (mark < 0 || mark >= (int)ctx->kmarks.size()) return;
    cudaEventRecord(ctx->kmarks[mark].b, ctx->stream);
}

void kt_collect(mp_ctx *ctx) {
    for (const KernelMark &m : ctx->kmarks) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, m.a, m.b) == cudaSuccess) {
            KernelClock &c = ctx->kclock[m.cls];
            c.launches++;
            c.ms += ms;
            c.work += m.work;
        }
        ctx->kevents.push_back(m.a);
        ctx->kevents.push_back(m.b);
    }
    ctx->kmarks.clear();
}

template <typename T>
static const T *strided(const void *base, int64_t stride, int64_t i) {
    return reinterpret_cast<const T *>(reinterpret_cast<const char *>(base) + stride * i);
}

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Carves the FP64 and FP32 views of one particle buffer out of one allocation.
static void carve(void *blk, long long cap, PartsF64 &a, PartsF32 &b) {
    char *p = (char *)blk;
    size_t d = align256(sizeof(double) * cap), f = align256(sizeof(float) * cap), i4 = align256(sizeof(int) * cap);
    a.px = (double *)p; a.py = (double *)(p + d); a.pz = (double *)(p + 2 * d);
    a.vx = (double *)(p + 3 * d); a.vy = (double *)(p + 4 * d); a.vz = (double *)(p + 5 * d);
    a.cell = (int *)(p + 6 * d);
    a.id = (long long *)(p + 6 * d + i4);
    b.rx = (float *)p; b.ry = (float *)(p + f); b.rz = (float *)(p + 2 * f);
    b.vx = (float *)(p + 3 * f); b.vy = (float *)(p + 4 * f); b.vz = (float *)(p + 5 * f);
    b.cell = (int *)(p + 6 * f);
    b.id = (long long *)(p + 6 * f + i4);
}

static size_t block_bytes(long long cap) {
    return 6 * align256(sizeof(double) * cap) + align256(sizeof(int) * cap) + align256(sizeof(long long) * cap);
}

static int grow_particles(mp_ctx *ctx, long long need) {
    if (need <= ctx->capacity) return MP_OK;
    long long cap = std::max<long long>(need, 2 * ctx->capacity);
    cap = std::max<long long>(cap, 1024);
    cap = (cap + 255) & ~255ll;  // whole 256-particle tiles: the push's bulk copies may round up to 16 B
    void *nb[2] = {nullptr, nullptr};
    for (int k = 0; k < 2; k++) {
        cudaError_t e = cudaMalloc(&nb[k], block_bytes(cap));
        if (e != cudaSuccess) {
            if (nb[0]) cudaFree(nb[0]);
            return cuda_fail(ctx, e, "cudaMalloc(particles)");
        }
    }
    PartsF64 a64[2];
    PartsF32 a32[2];
    carve(nb[0], cap, a64[0], a32[0]);
    carve(nb[1], cap, a64[1], a32[1]);
    long long n = ctx->n_host;
    if (n > 0 && ctx->part_block[ctx->cur]) {
        int c = ctx->cur;
        if (ctx->form == MP_FORM_FP64) {
            const PartsF64 &s = ctx->p64[c];
            double *src[6] = {s.px, s.py, s.pz, s.vx, s.vy, s.vz};
            double *dst[6] = {a64[0].px, a64[0].py, a64[0].pz, a64[0].vx, a64[0].vy, a64[0].vz};
            for (int k = 0; k < 6; k++)
                MP_CUDA(ctx, cudaMemcpyAsync(dst[k], src[k], sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
            MP_CUDA(ctx, cudaMemcpyAsync(a64[0].cell, s.cell, sizeof(int) * n, cudaMemcpyDeviceToDevice, ctx->stream));
            MP_CUDA(ctx, cudaMemcpyAsync(a64[0].id, s.id, sizeof(long long) * n, cudaMemcpyDeviceToDevice, ctx->stream));
        } else {
            const PartsF32 &s = ctx->p32[c];
            float *src[6] = {s.rx, s.ry, s.rz, s.vx, s.vy, s.vz};
            float *dst[6] = {a32[0].rx, a32[0].ry, a32[0].rz, a32[0].vx, a32[0].vy, a32[0].vz};
            for (int k = 0; k < 6; k++)
                MP_CUDA(ctx, cudaMemcpyAsync(dst[k], src[k], sizeof(float) * n, cudaMemcpyDeviceToDevice, ctx->stream));
            MP_CUDA(ctx, cudaMemcpyAsync(a32[0].cell, s.cell, sizeof(int) * n, cudaMemcpyDeviceToDevice, ctx->stream));
            MP_CUDA(ctx, cudaMemcpyAsync(a32[0].id, s.id, sizeof(long long) * n, cudaMemcpyDeviceToDevice, ctx->stream));
        }
        MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    for (int k = 0; k < 2; k++)
        if (ctx->part_block[k]) cudaFree(ctx->part_block[k]);
    for (int k = 0; k < 2; k++) {
        ctx->part_block[k] = nb[k];
        ctx->p64[k] = a64[k];
        ctx->p32[k] = a32[k];
    }
    ctx->cur = 0;
    ctx->capacity = cap;
    return MP_OK;
}

static int ensure_stage(mp_ctx *ctx, size_t bytes) {
    if (bytes <= ctx->stage_bytes) return MP_OK;
    if (ctx->stage) cudaFreeHost(ctx->stage);
    ctx->stage = nullptr;
    ctx->stage_bytes = 0;
    size_t b = std::max(bytes, ctx->stage_bytes * 2);
    MP_CUDA(ctx, cudaHostAlloc(&ctx->stage, b, cudaHostAllocDefault));
    ctx->stage_bytes = b;
    return MP_OK;
}

// Device staging of host appends and downloads, owned by the context.
static int ensure_dstage(mp_ctx *ctx, size_t bytes) {
    if (bytes <= ctx->dstage_bytes) return MP_OK;
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->dstage) cudaFree(ctx->dstage);
    ctx->dstage = nullptr;
    size_t b = std::max(bytes, ctx->dstage_bytes * 2);
    ctx->dstage_bytes = 0;
    MP_CUDA(ctx, cudaMalloc(&ctx->dstage, b));
    ctx->dstage_bytes = b;
    return MP_OK;
}

// Reads the counters back and turns error flags into a status.
static int sync_counters(mp_ctx *ctx) {
    MP_CUDA(ctx, cudaMemcpyAsync(ctx->counters_host, ctx->counters, sizeof(unsigned long long) * C_COUNT,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->n_host = (long long)ctx->counters_host[C_N];
    ctx->dead_host = (long long)ctx->counters_host[C_DEAD];
    unsigned long long flags = ctx->counters_host[C_FLAGS];
    unsigned long long part = flags & (FLAG_WALK_LIMIT | FLAG_LOOKBACK_TIMEOUT);
    if (part) {
        unsigned long long keep = flags & ~part;
        ctx->counters_host[C_FLAGS] = keep;
        MP_CUDA(ctx, cudaMemcpyAsync(ctx->counters + C_FLAGS, ctx->counters_host + C_FLAGS, sizeof(unsigned long long),
                                     cudaMemcpyHostToDevice, ctx->stream));
        MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (part & FLAG_LOOKBACK_TIMEOUT)
            return fail(ctx, MP_ERR_TIMEOUT, "a bounded device-side wait gave up");
        return fail(ctx, MP_ERR_WALK_LIMIT, "a particle's tet walk exceeded the hop limit");
    }
    return MP_OK;
}

}  // namespace mp

using namespace mp;

extern "C" {

const char *mp_error_string(int status) {
    switch (status) {
        case MP_OK: return "ok";
        case MP_ERR_ARG: return "invalid argument";
        case MP_ERR_OOM: return "out of memory";
        case MP_ERR_CUDA: return "CUDA runtime error";
        case MP_ERR_WALK_LIMIT: return "tet walk exceeded the hop limit";
        case MP_ERR_NOT_CONVERGED: return "Newton iteration did not converge";
        case MP_ERR_SINGULAR: return "singular or non-finite pivot in the factorization";
        case MP_ERR_STATE: return "call out of order";
        case MP_ERR_NO_DEVICE: return "no usable sm_100 CUDA device";
        case MP_ERR_TIMEOUT: return "bounded device wait gave up";
        case MP_ERR_LIMIT: return "size exceeds the fixed maximum of the allocation-free entry point";
    }
    return "unknown status";
}

const char *mp_last_error(const mp_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int mp_version(void) { return 10000; }

int mp_create(int device, const mp_mesh_desc *m, mp_ctx **out) {
    if (!out || !m) return MP_ERR_ARG;
    *out = nullptr;
    if (m->n_nodes <= 0 || m->n_tets <= 0 || !m->con || !m->volume || !m->alpha || !m->beta || !m->gamma ||
        !m->delta || !m->cell_con || !m->node_volume)
        return MP_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) return MP_ERR_NO_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return MP_ERR_NO_DEVICE;
    mp_ctx *ctx = new mp_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    auto bail = [&](int rc) {
        mp_destroy(ctx);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(MP_ERR_NO_DEVICE);
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(MP_ERR_CUDA);
    ctx->n_nodes = m->n_nodes;
    ctx->n_tets = m->n_tets;
    const int nt = m->n_tets, nn = m->n_nodes;
    std::vector<TetRec> rec(nt);
    std::vector<TetRec32> rec32(nt);
    std::vector<double> x0(4 * (size_t)nt, 0.0);
    std::vector<int> con(4 * (size_t)nt);
    std::vector<double> nvol(nn), npos(3 * (size_t)nn, 0.0);
    for (int n = 0; n < nn; n++) {
        nvol[n] = *strided<double>(m->node_volume, m->node_volume_stride, n);
        if (m->node_pos)
            for (int d = 0; d < 3; d++) npos[3 * n + d] = strided<double>(m->node_pos, m->node_pos_stride, n)[d];
    }
    bool small = true;  // 0 < V < 1 for every tet: the push's exact division-free inside test holds
    for (int t = 0; t < nt; t++) {
        TetRec &r = rec[t];
        std::memset(&r, 0, sizeof(r));
        const int *c = strided<int>(m->con, m->con_stride, t);
        const int *cc = strided<int>(m->cell_con, m->cell_con_stride, t);
        const double *al = strided<double>(m->alpha, m->alpha_stride, t);
        const double *be = strided<double>(m->beta, m->beta_stride, t);
        const double *ga = strided<double>(m->gamma, m->gamma_stride, t);
        const double *de = strided<double>(m->delta, m->delta_stride, t);
        r.volume = *strided<double>(m->volume, m->volume_stride, t);
        if (!(r.volume > 0.0 && r.volume < 1.0)) small = false;
        for (int i = 0; i < 4; i++) {
            if (c[i] < 0 || c[i] >= nn || cc[i] < -1 || cc[i] >= nt) {
                delete ctx;
                return MP_ERR_ARG;
            }
            r.alpha[i] = al[i]; r.beta[i] = be[i]; r.gamma[i] = ga[i]; r.delta[i] = de[i];
            r.con[i] = c[i]; r.cell_con[i] = cc[i];
            con[4 * (size_t)t + i] = c[i];
        }
        TetRec32 &q = rec32[t];
        std::memset(&q, 0, sizeof(q));
        double s = 1.0 / (6.0 * r.volume);
        for (int i = 0; i < 4; i++) {
            q.gx[i] = (float)(-r.beta[i] * s);
            q.gy[i] = (float)(r.gamma[i] * s);
            q.gz[i] = (float)(-r.delta[i] * s);
            q.con[i] = r.con[i];
            q.cell_con[i] = r.cell_con[i];
        }
        for (int d = 0; d < 3; d++) x0[4 * (size_t)t + d] = npos[3 * (size_t)c[0] + d];
    }
    ctx->small_tets = small;
#define ALLOC(ptr, bytes) if (cudaMalloc(&(ptr), (bytes)) != cudaSuccess) return bail(MP_ERR_OOM)
    ALLOC(ctx->tets, sizeof(TetRec) * nt);
    ALLOC(ctx->tets32, sizeof(TetRec32) * nt);
    ALLOC(ctx->tet_x0, sizeof(double) * 4 * nt);
    ALLOC(ctx->con, sizeof(int) * 4 * nt);
    ALLOC(ctx->ef, sizeof(double) * 3 * nt);
    ALLOC(ctx->node_volume, sizeof(double) * nn);
    ALLOC(ctx->node_pos, sizeof(double) * 3 * nn);
    ALLOC(ctx->den, sizeof(double) * nn);
    ALLOC(ctx->den_fixed, sizeof(unsigned long long) * nn);
    ALLOC(ctx->counters, sizeof(unsigned long long) * C_COUNT);
    ALLOC(ctx->scal, sizeof(double) * 8);
#undef ALLOC
    if (cudaHostAlloc(&ctx->counters_host, sizeof(unsigned long long) * C_COUNT, 0) != cudaSuccess ||
        cudaHostAlloc(&ctx->scal_host, sizeof(double) * 8, 0) != cudaSuccess)
        return bail(MP_ERR_OOM);
    cudaStream_t st = ctx->stream;
    cudaMemcpyAsync(ctx->tets, rec.data(), sizeof(TetRec) * nt, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(ctx->tets32, rec32.data(), sizeof(TetRec32) * nt, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(ctx->tet_x0, x0.data(), sizeof(double) * 4 * nt, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(ctx->con, con.data(), sizeof(int) * 4 * nt, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(ctx->node_volume, nvol.data(), sizeof(double) * nn, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(ctx->node_pos, npos.data(), sizeof(double) * 3 * nn, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(ctx->ef, 0, sizeof(double) * 3 * nt, st);
    cudaMemsetAsync(ctx->den, 0, sizeof(double) * nn, st);
    cudaMemsetAsync(ctx->counters, 0, sizeof(unsigned long long) * C_COUNT, st);
    upload_quadrature(st);
    cudaEventCreate(&ctx->t0.a); cudaEventCreate(&ctx->t0.b);
    cudaEventCreate(&ctx->t1.a); cudaEventCreate(&ctx->t1.b);
    cudaEventCreate(&ctx->tp.a); cudaEventCreate(&ctx->tp.b);
    cudaEventCreate(&ctx->ts.a); cudaEventCreate(&ctx->ts.b);
    if (cudaStreamSynchronize(st) != cudaSuccess) return bail(MP_ERR_CUDA);
    std::memset(ctx->counters_host, 0, sizeof(unsigned long long) * C_COUNT);
    int rc = grow_particles(ctx, 1024);
    if (rc) return bail(rc);
    *out = ctx;
    return MP_OK;
}

int mp_destroy(mp_ctx *ctx) {
    if (!ctx) return MP_OK;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    adjoint_free(ctx);
    solve_free(ctx);
    output_free(ctx);  // joins a writer still running
    inject_free(ctx);
    sparse_free(ctx);
    void *dev[] = {ctx->tets, ctx->tets32, ctx->tet_x0, ctx->con, ctx->ef, ctx->node_volume, ctx->node_pos,
                   ctx->den, ctx->den_fixed, ctx->counters, ctx->scal, ctx->compact_off, ctx->sort_hist,
                   ctx->part_block[0], ctx->part_block[1], ctx->ID, ctx->LM, ctx->detJ, ctx->nx, ctx->g, ctx->uh,
                   ctx->d, ctx->F0, ctx->F1, ctx->G, ctx->y, ctx->fvec, ctx->FP, ctx->work, ctx->K, ctx->J,
                   ctx->J32, ctx->K32, ctx->eq_ptr, ctx->eq_tet, ctx->eq_a, ctx->gs_minv, ctx->den_in, ctx->dstage};
    for (void *p : dev)
        if (p) cudaFree(p);
    if (ctx->counters_host) cudaFreeHost(ctx->counters_host);
    if (ctx->scal_host) cudaFreeHost(ctx->scal_host);
    if (ctx->stage) cudaFreeHost(ctx->stage);
    cudaEvent_t ev[] = {ctx->t0.a, ctx->t0.b, ctx->t1.a, ctx->t1.b, ctx->tp.a, ctx->tp.b, ctx->ts.a, ctx->ts.b};
    for (auto e : ev)
        if (e) cudaEventDestroy(e);
    for (const KernelMark &m : ctx->kmarks) {
        cudaEventDestroy(m.a);
        cudaEventDestroy(m.b);
    }
    for (cudaEvent_t e : ctx->kevents) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return MP_OK;
}

int mp_synchronize(mp_ctx *ctx) {
    if (!ctx) return MP_ERR_ARG;
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MP_OK;
}

int mp_get_stream(mp_ctx *ctx, void **s) {
    if (!ctx || !s) return MP_ERR_ARG;
    *s = (void *)ctx->stream;
    return MP_OK;
}

int mp_set_walk_limit(mp_ctx *ctx, int32_t max_hops) {
    if (!ctx || max_hops < 1) return MP_ERR_ARG;
    ctx->walk_limit = max_hops;
    return MP_OK;
}

int mp_set_walk_policy(mp_ctx *ctx, int policy) {
    if (!ctx || (policy != MP_WALK_LIMIT_ERROR && policy != MP_WALK_LIMIT_ABSORB)) return MP_ERR_ARG;
    ctx->walk_absorb = policy == MP_WALK_LIMIT_ABSORB;
    return MP_OK;
}

int mp_set_scatter_mode(mp_ctx *ctx, int mode) {
    if (!ctx || (mode != MP_SCATTER_FP64_ATOMIC && mode != MP_SCATTER_FIXED64)) return MP_ERR_ARG;
    ctx->scatter_mode = mode;
    return MP_OK;
}

int mp_set_sort_period(mp_ctx *ctx, int32_t steps) {
    if (!ctx || steps < 0) return MP_ERR_ARG;
    ctx->sort_period = steps;
    return MP_OK;
}

int mp_set_mixed_factor(mp_ctx *ctx, int mode) {
    if (!ctx || (mode != MP_MIXED_AUTO && mode != MP_MIXED_TF32 && mode != MP_MIXED_FP16 && mode != MP_MIXED_TF32X3))
        return MP_ERR_ARG;
    ctx->mixed_factor = mode;
    return MP_OK;
}

int mp_set_particle_form(mp_ctx *ctx, int form) {
    if (!ctx || (form != MP_FORM_FP64 && form != MP_FORM_MIXED)) return MP_ERR_ARG;
    if (form == ctx->form) return MP_OK;
    int rc0 = sync_counters(ctx);
    if (rc0) return rc0;
    rc0 = launch_compact(ctx);  // the conversion reads every slot's tet
    if (rc0) return rc0;
    int rc = launch_convert_form(ctx, form);
    if (rc) return rc;
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MP_OK;
}

int mp_set_track_ids(mp_ctx *ctx, int on) {
    if (!ctx) return MP_ERR_ARG;
    ctx->track_ids = on != 0;
    return MP_OK;
}

int mp_kernel_launches(mp_ctx *ctx, int64_t *n) {
    if (!ctx || !n) return MP_ERR_ARG;
    *n = ctx->launches;
    return MP_OK;
}

int mp_set_kernel_timing(mp_ctx *ctx, int on) {
    if (!ctx) return MP_ERR_ARG;
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    kt_collect(ctx);
    for (KernelClock &c : ctx->kclock) c = KernelClock();
    ctx->ktime_mask = on == 1 ? 0x1Fu : (unsigned)on & 0x1Fu;
    return MP_OK;
}

int mp_kernel_timing(mp_ctx *ctx, int cls, int64_t *launches, double *ms, double *work) {
    if (!ctx || cls < MP_KT_PUSH || cls > MP_KT_TRSV) return MP_ERR_ARG;
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    kt_collect(ctx);
    const KernelClock &c = ctx->kclock[cls];
    if (launches) *launches = c.launches;
    if (ms) *ms = c.ms;
    if (work) *work = c.work;
    return MP_OK;
}

int mp_particles_reserve(mp_ctx *ctx, int64_t capacity) {
    if (!ctx || capacity < 0) return MP_ERR_ARG;
    return grow_particles(ctx, capacity);
}

int mp_particles_count(mp_ctx *ctx, int64_t *n) {
    if (!ctx || !n) return MP_ERR_ARG;
    int rc = sync_counters(ctx);
    *n = ctx->n_host - ctx->dead_host;
    return rc;
}

int mp_particles_clear(mp_ctx *ctx) {
    if (!ctx) return MP_ERR_ARG;
    MP_CUDA(ctx, cudaMemsetAsync(ctx->counters + C_N, 0, 2 * sizeof(unsigned long long), ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->n_host = 0;
    ctx->dead_host = 0;
    return MP_OK;
}

int mp_particles_append_device(mp_ctx *ctx, int64_t n, const double *pos_soa, const double *vel_soa,
                               const int32_t *cell, int rewind, double q_over_m, double half_dt) {
    if (!ctx || n < 0 || (n > 0 && (!pos_soa || !vel_soa || !cell))) return MP_ERR_ARG;
    if (n == 0) return MP_OK;
    int rc = grow_particles(ctx, ctx->n_host + n);
    if (rc) return rc;
    rc = launch_append(ctx, n, pos_soa, vel_soa, cell, rewind, q_over_m, half_dt);
    if (rc) return rc;
    ctx->n_host += n;
    return MP_OK;
}

int mp_particles_append(mp_ctx *ctx, int64_t n, const double *pos, int64_t pos_stride, const double *vel,
                        int64_t vel_stride, const int32_t *cell, int64_t cell_stride, int rewind, double q_over_m,
                        double half_dt) {
    if (!ctx || n < 0 || (n > 0 && (!pos || !vel || !cell))) return MP_ERR_ARG;
    if (n == 0) return MP_OK;
    size_t bytes = sizeof(double) * 6 * n + sizeof(int) * n;
    int rc = ensure_stage(ctx, bytes);
    if (rc) return rc;
    rc = ensure_dstage(ctx, bytes);
    if (rc) return rc;
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // the staging buffer may still feed a copy
    double *h = (double *)ctx->stage;
    int *hc = (int *)(h + 6 * n);
    for (int64_t i = 0; i < n; i++) {
        const double *p = strided<double>(pos, pos_stride, i);
        const double *v = strided<double>(vel, vel_stride, i);
        int c = *strided<int>(cell, cell_stride, i);
        if (c < 0 || c >= ctx->n_tets) return fail(ctx, MP_ERR_ARG, "particle cell index out of range");
        h[i] = p[0]; h[n + i] = p[1]; h[2 * n + i] = p[2];
        h[3 * n + i] = v[0]; h[4 * n + i] = v[1]; h[5 * n + i] = v[2];
        hc[i] = c;
    }
    MP_CUDA(ctx, cudaMemcpyAsync(ctx->dstage, ctx->stage, bytes, cudaMemcpyHostToDevice, ctx->stream));
    double *d = (double *)ctx->dstage;
    return mp_particles_append_device(ctx, n, d, d + 3 * n, (const int32_t *)(d + 6 * n), rewind, q_over_m,
                                      half_dt);
}

int mp_particles_download(mp_ctx *ctx, int64_t n_max, double *pos, int64_t pos_stride, double *vel,
                          int64_t vel_stride, int32_t *cell, int64_t cell_stride, double *lc, int64_t lc_stride,
                          int64_t *id, int order) {
    if (!ctx) return MP_ERR_ARG;
    int rc = sync_counters(ctx);
    if (rc) return rc;
    rc = launch_compact(ctx);
    if (rc) return rc;
    long long n = ctx->n_host;
    if (n > n_max) return fail(ctx, MP_ERR_ARG, "output capacity smaller than the particle count");
    if (n == 0) return MP_OK;
    // layout: 10 FP64 arrays, cell (padded to 8 B), id
    size_t bytes = sizeof(double) * 10 * n + sizeof(int) * (n + (n & 1)) + sizeof(long long) * n;
    rc = ensure_stage(ctx, bytes);
    if (rc) return rc;
    rc = ensure_dstage(ctx, bytes);
    if (rc) return rc;
    double *d = (double *)ctx->dstage;
    int *dc = (int *)(d + 10 * n);
    long long *di = (long long *)(dc + n + (n & 1));
    rc = launch_download_pack(ctx, n, d, dc, di);
    if (rc) return rc;
    MP_CUDA(ctx, cudaMemcpyAsync(ctx->stage, ctx->dstage, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const double *h = (const double *)ctx->stage;
    const int *hc = (const int *)(h + 10 * n);
    const long long *hi = (const long long *)(hc + n + (n & 1));
    std::vector<long long> perm;
    if (order == MP_ORDER_ID && ctx->track_ids) {
        perm.resize(n);
        std::iota(perm.begin(), perm.end(), 0);
        std::sort(perm.begin(), perm.end(), [&](long long a, long long b) { return hi[a] < hi[b]; });
    }
    for (long long k = 0; k < n; k++) {
        long long i = perm.empty() ? k : perm[k];
        if (pos) {
            double *p = (double *)((char *)pos + pos_stride * k);
            p[0] = h[i]; p[1] = h[n + i]; p[2] = h[2 * n + i];
        }
        if (vel) {
            double *v = (double *)((char *)vel + vel_stride * k);
            v[0] = h[3 * n + i]; v[1] = h[4 * n + i]; v[2] = h[5 * n + i];
        }
        if (lc) {
            double *l = (double *)((char *)lc + lc_stride * k);
            for (int q = 0; q < 4; q++) l[q] = h[(6 + q) * n + i];
        }
        if (cell) *(int32_t *)((char *)cell + cell_stride * k) = hc[i];
        if (id) id[k] = hi[i];
    }
    return MP_OK;
}

int mp_push_scatter(mp_ctx *ctx, double q_over_m, double dt, double spwt, double *den_out, mp_step_stats *stats) {
    if (!ctx) return MP_ERR_ARG;
    long long n_before = ctx->n_host - ctx->dead_host;
    cudaEventRecord(ctx->ts.a, ctx->stream);
    int rc;
    if (ctx->sort_period > 0 && ++ctx->steps_since_sort >= ctx->sort_period) {
        rc = launch_sort_by_tet(ctx);
        if (rc) return rc;
        ctx->steps_since_sort = 0;
    }
    rc = launch_push(ctx, q_over_m, dt);
    if (rc) return rc;
    rc = launch_normalise(ctx, spwt);
    if (rc) return rc;
    cudaEventRecord(ctx->ts.b, ctx->stream);
    if (den_out)
        MP_CUDA(ctx, cudaMemcpyAsync(den_out, ctx->den, sizeof(double) * ctx->n_nodes, cudaMemcpyDeviceToHost,
                                     ctx->stream));
    rc = sync_counters(ctx);
    if (ctx->ktime_mask & (1u << MP_KT_PUSH)) {
        float ka = 0;
        if (cudaEventElapsedTime(&ka, ctx->tp.a, ctx->tp.b) == cudaSuccess) {
            KernelClock &c = ctx->kclock[MP_KT_PUSH];
            c.launches++;
            c.ms += ka;
            const double bpp = ctx->form == MP_FORM_FP64 ? 52.0 : 28.0;
            c.work += bpp * (double)(n_before + (ctx->n_host - ctx->dead_host));
        }
        kt_collect(ctx);
    }
    if (stats) {
        stats->n_before = n_before;
        stats->n_after = ctx->n_host - ctx->dead_host;
        stats->total_hops = (int64_t)ctx->counters_host[C_HOPS];
        stats->max_hops = (int32_t)ctx->counters_host[C_MAX_HOPS];
        stats->near_face_fp64 = (int32_t)ctx->counters_host[C_NEAR];
        stats->lost = (int64_t)ctx->counters_host[C_LOST];
        float ka = 0, kb = 0;
        cudaEventElapsedTime(&ka, ctx->tp.a, ctx->tp.b);
        cudaEventElapsedTime(&kb, ctx->ts.a, ctx->ts.b);
        stats->ms_kernel = ka;
        stats->ms_step = kb;
    }
    if (rc) return rc;
    // holes are removed by the next re-sort; without one due soon, compact once
    // they pass 1/16 of the slots
    bool sort_soon = ctx->sort_period > 0 && ctx->sort_period - ctx->steps_since_sort <= 2;
    if (!sort_soon && ctx->dead_host * 16 > ctx->n_host) rc = launch_compact(ctx);
    return rc;
}

int mp_density_download(mp_ctx *ctx, double *den) {
    if (!ctx || !den) return MP_ERR_ARG;
    MP_CUDA(ctx, cudaMemcpyAsync(den, ctx->den, sizeof(double) * ctx->n_nodes, cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MP_OK;
}

int mp_sort_by_tet(mp_ctx *ctx) {
    if (!ctx) return MP_ERR_ARG;
    int rc = sync_counters(ctx);
    if (rc) return rc;
    rc = launch_sort_by_tet(ctx);
    if (rc) return rc;
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->steps_since_sort = 0;
    return MP_OK;
}

// ---- FE -------------------------------------------------------------------------------

int mp_fe_setup(mp_ctx *ctx, const mp_fe_desc *fe) {
    if (!ctx || !fe || fe->neq <= 0 || !fe->ID || !fe->nx || !fe->detJ || !fe->g || !(fe->kTe > 0))
        return MP_ERR_ARG;
    const int nn = ctx->n_nodes, nt = ctx->n_tets, neq = fe->neq;
    // LM and the equation -> (tet, local node) lists in tet order
    std::vector<int> con(4 * (size_t)nt);
    MP_CUDA(ctx, cudaMemcpy(con.data(), ctx->con, sizeof(int) * 4 * nt, cudaMemcpyDeviceToHost));
    std::vector<int> LM(4 * (size_t)nt), cnt(neq + 1, 0);
    for (int n = 0; n < nn; n++)
        if (fe->ID[n] < -1 || fe->ID[n] >= neq) return fail(ctx, MP_ERR_ARG, "ID out of range");
    for (int e = 0; e < nt; e++)
        for (int a = 0; a < 4; a++) {
            int A = fe->ID[con[4 * (size_t)e + a]];
            LM[4 * (size_t)e + a] = A;
            if (A >= 0) cnt[A + 1]++;
        }
    for (int A = 0; A < neq; A++) cnt[A + 1] += cnt[A];
    std::vector<int> eq_tet(cnt[neq]), fillp(cnt.begin(), cnt.end() - 1);
    std::vector<unsigned char> eq_a(cnt[neq]);
    for (int e = 0; e < nt; e++)
        for (int a = 0; a < 4; a++) {
            int A = LM[4 * (size_t)e + a];
            if (A < 0) continue;
            int k = fillp[A]++;
            eq_tet[k] = e;
            eq_a[k] = (unsigned char)a;
        }
    // (re)allocate
    void *old[] = {ctx->ID, ctx->LM, ctx->detJ, ctx->nx, ctx->g, ctx->uh, ctx->d, ctx->F0, ctx->F1, ctx->G, ctx->y,
                   ctx->fvec, ctx->FP, ctx->work, ctx->K, ctx->J, ctx->J32, ctx->K32, ctx->eq_ptr, ctx->eq_tet,
                   ctx->eq_a};
    for (void *p : old)
        if (p) cudaFree(p);
    ctx->J32 = ctx->K32 = nullptr;
    ctx->k32_current = false;
    const long long ld = (neq + 31) & ~31ll;
    size_t vec = sizeof(double) * (size_t)(ld + 64);
    MP_CUDA(ctx, cudaMalloc(&ctx->ID, sizeof(int) * nn));
    MP_CUDA(ctx, cudaMalloc(&ctx->LM, sizeof(int) * 4 * nt));
    MP_CUDA(ctx, cudaMalloc(&ctx->detJ, sizeof(double) * nt));
    MP_CUDA(ctx, cudaMalloc(&ctx->nx, sizeof(double) * 12 * nt));
    MP_CUDA(ctx, cudaMalloc(&ctx->g, sizeof(double) * nn));
    MP_CUDA(ctx, cudaMalloc(&ctx->uh, sizeof(double) * nn));
    MP_CUDA(ctx, cudaMalloc(&ctx->eq_ptr, sizeof(int) * (neq + 1)));
    MP_CUDA(ctx, cudaMalloc(&ctx->eq_tet, sizeof(int) * std::max(1, cnt[neq])));
    MP_CUDA(ctx, cudaMalloc(&ctx->eq_a, std::max(1, cnt[neq])));
    double **vp[] = {&ctx->d, &ctx->F0, &ctx->F1, &ctx->G, &ctx->y, &ctx->fvec, &ctx->FP, &ctx->work};
    for (double **p : vp) {
        MP_CUDA(ctx, cudaMalloc(p, vec));
        MP_CUDA(ctx, cudaMemset(*p, 0, vec));
    }
    ctx->K = ctx->J = nullptr;  // J: allocated when an FP64 dense J is first built
    ctx->j32_current = ctx->j_current = false;
    const bool dense = ctx->fe_storage == MP_FE_STORAGE_DENSE;
    if (dense) MP_CUDA(ctx, cudaMalloc(&ctx->K, sizeof(double) * (size_t)ld * neq));
    cudaStream_t st = ctx->stream;
    MP_CUDA(ctx, cudaMemcpyAsync(ctx->ID, fe->ID, sizeof(int) * nn, cudaMemcpyHostToDevice, st));
    MP_CUDA(ctx, cudaMemcpyAsync(ctx->LM, LM.data(), sizeof(int) * 4 * nt, cudaMemcpyHostToDevice, st));
    MP_CUDA(ctx, cudaMemcpyAsync(ctx->detJ, fe->detJ, sizeof(double) * nt, cudaMemcpyHostToDevice, st));
    MP_CUDA(ctx, cudaMemcpyAsync(ctx->nx, fe->nx, sizeof(double) * 12 * nt, cudaMemcpyHostToDevice, st));
    MP_CUDA(ctx, cudaMemcpyAsync(ctx->g, fe->g, sizeof(double) * nn, cudaMemcpyHostToDevice, st));
    MP_CUDA(ctx, cudaMemcpyAsync(ctx->uh, fe->g, sizeof(double) * nn, cudaMemcpyHostToDevice, st));
    MP_CUDA(ctx, cudaMemcpyAsync(ctx->eq_ptr, cnt.data(), sizeof(int) * (neq + 1), cudaMemcpyHostToDevice, st));
    if (cnt[neq]) {
        MP_CUDA(ctx, cudaMemcpyAsync(ctx->eq_tet, eq_tet.data(), sizeof(int) * cnt[neq], cudaMemcpyHostToDevice, st));
        MP_CUDA(ctx, cudaMemcpyAsync(ctx->eq_a, eq_a.data(), cnt[neq], cudaMemcpyHostToDevice, st));
    }
    MP_CUDA(ctx, cudaStreamSynchronize(st));
    ctx->neq = neq;
    ctx->n0 = fe->n0;
    ctx->phi0 = fe->phi0;
    ctx->kTe = fe->kTe;
    int rc = sparse_setup(ctx, LM, cnt, eq_tet);
    if (rc) return rc;
    if (fe->K_rows || fe->K_dense) {
        if (!fe->F0) return fail(ctx, MP_ERR_ARG, "K given without F0");
        if (dense) {
            MP_CUDA(ctx, cudaMemset(ctx->K, 0, sizeof(double) * (size_t)ld * neq));
            for (int i = 0; i < neq; i++) {
                const double *row = fe->K_rows ? fe->K_rows[i] : fe->K_dense + (size_t)i * neq;
                MP_CUDA(ctx, cudaMemcpy(ctx->K + (size_t)i * ld, row, sizeof(double) * neq, cudaMemcpyHostToDevice));
            }
            rc = fe_sparse_from_dense(ctx);
        } else {
            rc = fe_sparse_from_host(ctx, fe->K_rows, fe->K_dense);
        }
        if (rc) return rc;
        MP_CUDA(ctx, cudaMemcpy(ctx->F0, fe->F0, sizeof(double) * neq, cudaMemcpyHostToDevice));
    } else {
        rc = dense ? fe_assemble(ctx) : fe_assemble_sparse(ctx);
        if (rc) return rc;
        if (dense && (rc = fe_sparse_from_dense(ctx))) return rc;
    }
    MP_CUDA(ctx, cudaStreamSynchronize(st));
    ctx->fe_ready = true;
    return MP_OK;
}

static double *vec_ptr(mp_ctx *ctx, int which, size_t *len) {
    switch (which) {
        case MP_VEC_F0: *len = ctx->neq; return ctx->F0;
        case MP_VEC_F1: *len = ctx->neq; return ctx->F1;
        case MP_VEC_D: *len = ctx->neq; return ctx->d;
        case MP_VEC_G: *len = ctx->n_nodes; return ctx->g;
        case MP_VEC_UH: *len = ctx->n_nodes; return ctx->uh;
        case MP_VEC_DEN: *len = ctx->n_nodes; return ctx->den;
        case MP_VEC_EF: *len = 3 * (size_t)ctx->n_tets; return ctx->ef;
        case MP_VEC_RESIDUAL: *len = ctx->neq; return ctx->G;
        case MP_VEC_Y: *len = ctx->neq; return ctx->y;
    }
    *len = 0;
    return nullptr;
}

int mp_device_buffer(mp_ctx *ctx, int which, void **ptr, int64_t *len) {
    if (!ctx || !ptr || !len) return MP_ERR_ARG;
    size_t n = 0;
    double *p = vec_ptr(ctx, which, &n);
    if (!p) return fail(ctx, MP_ERR_ARG, "no such device buffer");
    *ptr = p;
    *len = (int64_t)n;
    return MP_OK;
}

int mp_fe_download(mp_ctx *ctx, int which, double *out) {
    if (!ctx || !out) return MP_ERR_ARG;
    if (which == MP_MAT_K || which == MP_MAT_J) {
        if (!ctx->fe_ready) return fail(ctx, MP_ERR_STATE, "no FE setup");
        if (!ctx->K) return fail(ctx, MP_ERR_STATE, "sparse storage: no dense matrix (mp_fe_sparse_matrix)");
        if (which == MP_MAT_J && !ctx->J) return fail(ctx, MP_ERR_STATE, "no FP64 J built yet (mp_fe_build_j)");
        const long long ld = (ctx->neq + 31) & ~31ll;
        MP_CUDA(ctx, cudaMemcpy2DAsync(out, sizeof(double) * ctx->neq, which == MP_MAT_K ? ctx->K : ctx->J,
                                       sizeof(double) * ld, sizeof(double) * ctx->neq, ctx->neq,
                                       cudaMemcpyDeviceToHost, ctx->stream));
        MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        return MP_OK;
    }
    size_t len = 0;
    double *p = vec_ptr(ctx, which, &len);
    if (!p) return fail(ctx, which <= MP_VEC_Y ? MP_ERR_STATE : MP_ERR_ARG, "vector not available");
    MP_CUDA(ctx, cudaMemcpyAsync(out, p, sizeof(double) * len, cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MP_OK;
}

int mp_fe_upload(mp_ctx *ctx, int which, const double *values) {
    if (!ctx || !values) return MP_ERR_ARG;
    size_t len = 0;
    double *p = vec_ptr(ctx, which, &len);
    if (!p) return fail(ctx, MP_ERR_ARG, "vector not available for upload");
    MP_CUDA(ctx, cudaMemcpyAsync(p, values, sizeof(double) * len, cudaMemcpyHostToDevice, ctx->stream));
    if (which == MP_VEC_EF) {
        // keep the walk records' copy of the field in step
        MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        std::vector<double> ef(values, values + len);
        std::vector<TetRec> rec(ctx->n_tets);
        std::vector<TetRec32> rec32(ctx->n_tets);
        MP_CUDA(ctx, cudaMemcpy(rec.data(), ctx->tets, sizeof(TetRec) * ctx->n_tets, cudaMemcpyDeviceToHost));
        MP_CUDA(ctx, cudaMemcpy(rec32.data(), ctx->tets32, sizeof(TetRec32) * ctx->n_tets, cudaMemcpyDeviceToHost));
        for (int e = 0; e < ctx->n_tets; e++)
            for (int d = 0; d < 3; d++) {
                rec[e].ef[d] = ef[3 * (size_t)e + d];
                rec32[e].ef[d] = (float)ef[3 * (size_t)e + d];
            }
        MP_CUDA(ctx, cudaMemcpy(ctx->tets, rec.data(), sizeof(TetRec) * ctx->n_tets, cudaMemcpyHostToDevice));
        MP_CUDA(ctx, cudaMemcpy(ctx->tets32, rec32.data(), sizeof(TetRec32) * ctx->n_tets, cudaMemcpyHostToDevice));
    }
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MP_OK;
}

static const double *den_source(mp_ctx *ctx, const double *ion_den_host, int *rc) {
    *rc = MP_OK;
    if (!ion_den_host) return ctx->den;
    if (!ctx->den_in) {
        cudaError_t e = cudaMalloc(&ctx->den_in, sizeof(double) * ctx->n_nodes);
        if (e != cudaSuccess) {
            *rc = cuda_fail(ctx, e, "cudaMalloc(den_in)");
            return nullptr;
        }
    }
    cudaError_t e = cudaMemcpyAsync(ctx->den_in, ion_den_host, sizeof(double) * ctx->n_nodes, cudaMemcpyHostToDevice,
                                    ctx->stream);
    if (e != cudaSuccess) *rc = cuda_fail(ctx, e, "cudaMemcpyAsync(den_in)");
    return ctx->den_in;
}

int mp_fe_build_f1(mp_ctx *ctx, const double *ion_den) {
    if (!ctx) return MP_ERR_ARG;
    if (!ctx->fe_ready) return fail(ctx, MP_ERR_STATE, "no FE setup");
    int rc;
    const double *den = den_source(ctx, ion_den, &rc);
    if (rc) return rc;
    rc = fe_build_f1(ctx, den);
    if (rc) return rc;
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MP_OK;
}

int mp_fe_residual(mp_ctx *ctx) {
    if (!ctx) return MP_ERR_ARG;
    if (!ctx->fe_ready) return fail(ctx, MP_ERR_STATE, "no FE setup");
    int rc = fe_residual(ctx);
    if (rc) return rc;
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MP_OK;
}

int mp_fe_build_j(mp_ctx *ctx, int method) {
    if (!ctx) return MP_ERR_ARG;
    if (!ctx->fe_ready) return fail(ctx, MP_ERR_STATE, "no FE setup");
    if (method < MP_METHOD_NONLINEAR || method > MP_METHOD_SPARSE_NEWTON) return MP_ERR_ARG;
    if (!ctx->K && method <= MP_METHOD_LAPACK)
        return fail(ctx, MP_ERR_STATE, "sparse storage: the dense J needs MP_FE_STORAGE_DENSE");
    int rc = fe_build_j(ctx, method);
    if (rc) return rc;
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MP_OK;
}

int mp_fe_solve_linear(mp_ctx *ctx, int method, int form, const double *b, mp_newton_stats *st) {
    if (!ctx || (method != MP_METHOD_GAUSS_SEIDEL && method != MP_METHOD_LAPACK && method != MP_METHOD_SPARSE_CG))
        return MP_ERR_ARG;
    if (!ctx->fe_ready) return fail(ctx, MP_ERR_STATE, "no FE setup");
    if (!ctx->K && method != MP_METHOD_SPARSE_CG)
        return fail(ctx, MP_ERR_STATE, "sparse storage: this method needs MP_FE_STORAGE_DENSE");
    if (b) MP_CUDA(ctx, cudaMemcpyAsync(ctx->G, b, sizeof(double) * ctx->neq, cudaMemcpyHostToDevice, ctx->stream));
    MP_CUDA(ctx, cudaMemsetAsync(ctx->y, 0, sizeof(double) * ctx->neq, ctx->stream));
    mp_newton_stats local;
    if (!st) st = &local;
    std::memset(st, 0, sizeof(*st));
    int rc = method == MP_METHOD_SPARSE_CG   ? fe_solve_cg(ctx, st)
             : method == MP_METHOD_GAUSS_SEIDEL ? fe_solve_gs(ctx, st)
                                                : fe_solve_ldlt(ctx, form, st);
    if (rc) return rc;
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (st->linear_failures)
        return fail(ctx, MP_ERR_NOT_CONVERGED, "GS failed to converge");
    return MP_OK;
}

int mp_set_gs_max_sweeps(mp_ctx *ctx, int32_t sweeps) {
    if (!ctx || sweeps < 1) return MP_ERR_ARG;
    ctx->gs_max_sweeps = sweeps;
    return MP_OK;
}

int mp_compute_phi(mp_ctx *ctx, const double *ion_den, int method, int form, mp_newton_stats *st) {
    if (!ctx || method < MP_METHOD_NONLINEAR || method > MP_METHOD_SPARSE_NEWTON ||
        (form != MP_FORM_FP64 && form != MP_FORM_MIXED))
        return MP_ERR_ARG;
    if (!ctx->fe_ready) return fail(ctx, MP_ERR_STATE, "no FE setup");
    const bool sparse = method == MP_METHOD_SPARSE_CG || method == MP_METHOD_SPARSE_NEWTON;
    if (!ctx->K && !sparse) return fail(ctx, MP_ERR_STATE, "sparse storage: this method needs MP_FE_STORAGE_DENSE");
    mp_newton_stats local;
    if (!st) st = &local;
    std::memset(st, 0, sizeof(*st));
    int rc;
    const double *den = den_source(ctx, ion_den, &rc);
    if (rc) return rc;
    cudaEventRecord(ctx->t0.a, ctx->stream);
    // solve(): y starts at zero and is reused across Newton iterations
    MP_CUDA(ctx, cudaMemsetAsync(ctx->y, 0, sizeof(double) * ctx->neq, ctx->stream));
    double ms_factor = 0;
    if (method == MP_METHOD_NONLINEAR || method == MP_METHOD_SPARSE_NEWTON) {
        // solveNonLinear, src/FESolver.cpp:324-364: up to 10 Newton iterations,
        // Gauss-Seidel inner solves in the FP64 form (the mixed form uses its
        // refined LDL^T instead, SPARSE_NEWTON conjugate gradients), stop when
        // ||y||/neq < 1e-2.
        bool converged = false;
        double L2 = 0;
        int it;
        for (it = 0; it < 10; it++) {
            if ((rc = fe_build_f1(ctx, den))) return rc;
            if ((rc = fe_residual(ctx))) return rc;
            if ((rc = fe_build_j(ctx, method, form))) return rc;
            rc = sparse                    ? fe_solve_cg(ctx, st)
                 : form == MP_FORM_FP64 ? fe_solve_gs(ctx, st)
                                        : fe_solve_ldlt(ctx, form, st);
            if (rc) return rc;
            ms_factor += st->ms_factor;
            if ((rc = fe_update_d(ctx, &L2))) return rc;
            if (L2 < 1e-2) {
                converged = true;
                break;
            }
        }
        st->newton_iterations = converged ? it + 1 : it;
        st->l2 = L2;
        if ((rc = fe_uh(ctx))) return rc;
        if (!converged) {
            MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            return fail(ctx, MP_ERR_NOT_CONVERGED, "NR failed to converge");
        }
    } else {
        // one Newton step, src/FESolver.cpp:301-317
        if ((rc = fe_build_f1(ctx, den))) return rc;
        if ((rc = fe_residual(ctx))) return rc;
        if ((rc = fe_build_j(ctx, method, method == MP_METHOD_GAUSS_SEIDEL ? MP_FORM_FP64 : form))) return rc;
        rc = method == MP_METHOD_SPARSE_CG      ? fe_solve_cg(ctx, st)
             : method == MP_METHOD_GAUSS_SEIDEL ? fe_solve_gs(ctx, st)
                                                : fe_solve_ldlt(ctx, form, st);
        if (rc) return rc;
        ms_factor = st->ms_factor;
        double L2 = 0;
        if ((rc = fe_update_d(ctx, &L2))) return rc;
        st->newton_iterations = 1;
        st->l2 = L2;
        if ((rc = fe_uh(ctx))) return rc;
    }
    cudaEventRecord(ctx->t0.b, ctx->stream);
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    kt_collect(ctx);
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->t0.a, ctx->t0.b);
    st->ms_total = ms;
    st->ms_factor = ms_factor;
    return MP_OK;
}

int mp_update_ef(mp_ctx *ctx, const double *uh_host) {
    if (!ctx) return MP_ERR_ARG;
    if (!ctx->fe_ready) return fail(ctx, MP_ERR_STATE, "no FE setup");
    if (uh_host)
        MP_CUDA(ctx, cudaMemcpyAsync(ctx->uh, uh_host, sizeof(double) * ctx->n_nodes, cudaMemcpyHostToDevice,
                                     ctx->stream));
    int rc = launch_update_ef(ctx);
    if (rc) return rc;
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MP_OK;
}

int mp_field_download(mp_ctx *ctx, double *d, double *uh, double *ef) {
    if (!ctx) return MP_ERR_ARG;
    if (d) {
        if (!ctx->fe_ready) return fail(ctx, MP_ERR_STATE, "no FE setup");
        MP_CUDA(ctx, cudaMemcpyAsync(d, ctx->d, sizeof(double) * ctx->neq, cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (uh) {
        if (!ctx->fe_ready) return fail(ctx, MP_ERR_STATE, "no FE setup");
        MP_CUDA(ctx, cudaMemcpyAsync(uh, ctx->uh, sizeof(double) * ctx->n_nodes, cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (ef)
        MP_CUDA(ctx, cudaMemcpyAsync(ef, ctx->ef, sizeof(double) * 3 * ctx->n_tets, cudaMemcpyDeviceToHost, ctx->stream));
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MP_OK;
}

}  // extern "C"
