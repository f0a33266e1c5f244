// InjectIons on the device (src/mini-pic.cpp:208-265).  The per-face counts
// are the reference's, computed on the host in its arithmetic with the shared
// remainder carried across faces and calls (the injector's state, as the host
// sampler uses it); the positions and velocities are drawn on the device with
// a counter-based generator instead of the reference's sequential mt19937
// stream, so a step's injection needs no host sampling and no particle upload:
//   position  a*u + b*v + p0 with (a, b) uniform on the triangle (the
//             reference's fold of a + b > 1), in the face's tet;
//   velocity  normal*ion_velocity + a Maxwellian thermal part of standard
//             deviation thermal_sigma per component (0 = the reference's cold
//             beam), then the half-step rewind in the current field.
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC11), key = the caller's seed,
// counter = (particle index, draw, step): a run is reproducible for a given
// seed and independent of the launch shape.
#include <algorithm>
#include <cstring>
#include <vector>

#include "mp_injector.h"
#include "mp_internal.h"

namespace mp {

struct InjectState {
    const mp_injector *inj = nullptr;  // faces uploaded from this injector
    int n_faces = 0;
    double *faces = nullptr;           // [n_faces][12]: p0, u, v, normal
    int *face_cell = nullptr;          // [n_faces]
    int *prefix = nullptr;             // [n_faces + 1] first particle of each face
    int *prefix_host = nullptr;        // pinned
    double *soa = nullptr;             // [6][n] positions, velocities of a call (capacity 6 * cap)
    int *cell = nullptr;               // [cap]
    long long cap = 0;
};

struct U4 {
    unsigned x, y, z, w;
};

// Philox4x32 with 10 rounds: multipliers 0xD2511F53 / 0xCD9E8D57, key
// increments (Weyl sequence) 0x9E3779B9 / 0xBB67AE85, as published.
__device__ __forceinline__ U4 philox4x32_10(U4 c, unsigned k0, unsigned k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const unsigned lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const unsigned lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// [0, 1) with 53 random bits from two words
__device__ __forceinline__ double uniform53(unsigned hi, unsigned lo) {
    return ((double)(hi >> 5) * 67108864.0 + (double)(lo >> 6)) * (1.0 / 9007199254740992.0);
}

__global__ void k_inject(long long n, int n_faces, const int *__restrict__ prefix, const double *__restrict__ faces,
                         const int *__restrict__ face_cell, double ion_velocity, double sigma, unsigned k0,
                         unsigned k1, unsigned long long step, double *soa, int *cell) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        // the face: last f with prefix[f] <= i
        int lo = 0, hi = n_faces;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (prefix[mid] <= i) lo = mid;
            else hi = mid;
        }
        const double *f = faces + 12ll * lo;
        const unsigned s0 = (unsigned)step, s1 = (unsigned)(step >> 32);
        const U4 r0 = philox4x32_10(U4{(unsigned)i, (unsigned)(i >> 32) << 1, s0, s1}, k0, k1);
        const U4 r1 = philox4x32_10(U4{(unsigned)i, ((unsigned)(i >> 32) << 1) | 1u, s0, s1}, k0, k1);
        double a = uniform53(r0.x, r0.y), b = uniform53(r0.z, r0.w);
        if ((a + b) > 1) {
            a = 1 - a;
            b = 1 - b;
        }
        // Box-Muller: three normals from two uniform pairs
        const double u1 = 1.0 - uniform53(r1.x, r1.y), u2 = uniform53(r1.z, r1.w);
        const double rad = sqrt(-2.0 * log(u1));
        double sn, cs;
        sincospi(2.0 * u2, &sn, &cs);
        const U4 r2 = philox4x32_10(U4{(unsigned)i, ((unsigned)(i >> 32) << 1) | 1u, s0 ^ 0xA5A5A5A5u, s1}, k0, k1);
        const double u3 = 1.0 - uniform53(r2.x, r2.y), u4 = uniform53(r2.z, r2.w);
        const double n3 = sqrt(-2.0 * log(u3)) * cospi(2.0 * u4);
        const double g[3] = {rad * cs, rad * sn, n3};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            soa[d * n + i] = a * f[3 + d] + b * f[6 + d] + f[d];  // a*u + b*v + p0, the reference's order
            soa[(3 + d) * n + i] = f[9 + d] * ion_velocity + sigma * g[d];
        }
        cell[i] = face_cell[lo];
    }
}

void inject_free(mp_ctx *ctx) {
    InjectState *s = reinterpret_cast<InjectState *>(ctx->inject);
    if (!s) return;
    cudaFree(s->faces);
    cudaFree(s->face_cell);
    cudaFree(s->prefix);
    cudaFree(s->soa);
    cudaFree(s->cell);
    if (s->prefix_host) cudaFreeHost(s->prefix_host);
    delete s;
    ctx->inject = nullptr;
}

}  // namespace mp

using namespace mp;

extern "C" int mp_inject_device(mp_ctx *ctx, mp_injector *inj, double plasma_den, double ion_velocity, double dt,
                                double spwt, double thermal_sigma, double q_over_m, uint64_t seed, uint64_t step,
                                int64_t *n_out) {
    if (!ctx || !inj || !(dt > 0) || !(spwt > 0) || thermal_sigma < 0) return MP_ERR_ARG;
    InjectState *s = reinterpret_cast<InjectState *>(ctx->inject);
    if (!s) {
        s = new InjectState();
        ctx->inject = s;
    }
    const int nf = inj->n_faces;
    if (s->inj != inj || s->n_faces != nf) {
        // upload the faces of this injector (once)
        cudaFree(s->faces);
        cudaFree(s->face_cell);
        cudaFree(s->prefix);
        if (s->prefix_host) cudaFreeHost(s->prefix_host);
        s->faces = nullptr;
        s->face_cell = s->prefix = s->prefix_host = nullptr;
        std::vector<double> fh(12 * (size_t)nf);
        for (int f = 0; f < nf; f++)
            for (int d = 0; d < 3; d++) {
                fh[12 * f + d] = inj->p0[3 * f + d];
                fh[12 * f + 3 + d] = inj->u[3 * f + d];
                fh[12 * f + 6 + d] = inj->v[3 * f + d];
                fh[12 * f + 9 + d] = inj->normal[3 * f + d];
            }
        for (int f = 0; f < nf; f++)
            if (inj->cell[f] < 0 || inj->cell[f] >= ctx->n_tets) return fail(ctx, MP_ERR_ARG, "inlet face cell out of range");
        MP_CUDA(ctx, cudaMalloc(&s->faces, sizeof(double) * fh.size() + 8));
        MP_CUDA(ctx, cudaMalloc(&s->face_cell, sizeof(int) * (nf + 1)));
        MP_CUDA(ctx, cudaMalloc(&s->prefix, sizeof(int) * (nf + 1)));
        MP_CUDA(ctx, cudaMallocHost(&s->prefix_host, sizeof(int) * (nf + 1)));
        MP_CUDA(ctx, cudaMemcpy(s->faces, fh.data(), sizeof(double) * fh.size(), cudaMemcpyHostToDevice));
        MP_CUDA(ctx, cudaMemcpy(s->face_cell, inj->cell.data(), sizeof(int) * nf, cudaMemcpyHostToDevice));
        s->inj = inj;
        s->n_faces = nf;
    }
    // the reference's counts, shared remainder carried (src/mini-pic.cpp:214-227)
    MP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // the pinned prefix may still feed the last copy
    long long total = 0;
    double rem = inj->rem;
    for (int f = 0; f < nf; f++) {
        double num_per_sec = plasma_den * ion_velocity * inj->area[f];
        double num_real = num_per_sec * dt;
        double fnum_mp = num_real / spwt + rem;
        int num_mp = (int)fnum_mp;
        rem = fnum_mp - num_mp;
        s->prefix_host[f] = (int)total;
        total += num_mp;
        if (total > (1ll << 30)) return fail(ctx, MP_ERR_ARG, "more than 2^30 injected particles in one call");
    }
    s->prefix_host[nf] = (int)total;
    inj->rem = rem;
    if (n_out) *n_out = total;
    if (total == 0) return MP_OK;
    if (total > s->cap) {
        cudaFree(s->soa);
        cudaFree(s->cell);
        s->soa = nullptr;
        s->cell = nullptr;
        const long long cap = std::max<long long>(total, 2 * s->cap);
        MP_CUDA(ctx, cudaMalloc(&s->soa, sizeof(double) * 6 * cap));
        MP_CUDA(ctx, cudaMalloc(&s->cell, sizeof(int) * cap));
        s->cap = cap;
    }
    MP_CUDA(ctx, cudaMemcpyAsync(s->prefix, s->prefix_host, sizeof(int) * (nf + 1), cudaMemcpyHostToDevice,
                                 ctx->stream));
    const int th = 256;
    const int g = (int)std::min<long long>((total + th - 1) / th, (long long)ctx->sm_count * 8);
    k_inject<<<g, th, 0, ctx->stream>>>(total, nf, s->prefix, s->faces, s->face_cell, ion_velocity, thermal_sigma,
                                        (unsigned)seed, (unsigned)(seed >> 32), step, s->soa, s->cell),
        ++ctx->launches;
    MP_CUDA(ctx, cudaGetLastError());
    // positions [3][total] then velocities [3][total]
    return mp_particles_append_device(ctx, total, s->soa, s->soa + 3 * total, s->cell, 1, q_over_m, 0.5 * dt);
}
