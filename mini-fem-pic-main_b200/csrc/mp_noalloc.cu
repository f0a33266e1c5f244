// mp_push_particles_noalloc: the push + walk + scatter + stable-removal kernel
// for callers that cannot allocate device memory.
//
// Who needs it: code whose device memory belongs to someone else's allocator
// (a SYCL or framework runtime that hands out all of the GPU's memory up
// front), and code on a latency-critical path, where cudaMalloc is not allowed
// because it can synchronise the whole device and stall every other stream.
// Such a caller owns every buffer; this entry point takes the particles, mesh,
// field and density it works on, and keeps the one piece of scratch the
// kernel needs -- the per-tile words of its single-pass stable compaction and
// three counters -- in a fixed file-scope device array instead.
//
// Limits and contract:
//   * at most MP_NOALLOC_MAX_PARTICLES (8,388,608) particles per call; larger
//     calls return MP_ERR_LIMIT before touching the device;
//   * the scratch array is 262,208 bytes on every GPU that loads the library,
//     held until the process exits;
//   * every call on a device shares that array and clears it first; calls
//     that overlap on the GPU (two streams, or two host threads) race on it
//     and must be serialised by the caller;
//   * the first call on a device looks up the array's device address with that
//     device current; make that first call before any stream capture;
//   * the records are the caller's, so every index is checked before it is
//     used: a particle whose cell lies outside [0, n_tets), or whose walk meets
//     a neighbour index >= n_tets or a node index outside [0, n_nodes), stops
//     where it is, adds nothing to den, is written out unchanged from that
//     point, and the call returns MP_ERR_ARG (the reference's flagged state
//     cell_index = -1 is removed before its next push, src/mini-pic.cpp:316);
//   * after MP_ERR_TIMEOUT the contents of particles_out (and of particles_in
//     when it is the same buffer) are undefined.
#include <cuda/atomic>

#include <mutex>

#include "mp_internal.h"

namespace mp_noalloc {

constexpr int THREADS = 256;
constexpr long long MAX_PARTICLES = 8388608;  // 2^23
constexpr long long MAX_TILES = MAX_PARTICLES / THREADS;
constexpr int W_TICKET = 0, W_KEPT = 1, W_FLAGS = 2, W_TILES = 8;
constexpr long long SCRATCH_WORDS = W_TILES + MAX_TILES;
constexpr unsigned long long ST_AGG = 1ull << 62, ST_PREFIX = 2ull << 62, ST_VALUE = (1ull << 62) - 1;
constexpr long long SPIN_LIMIT = 1ll << 24;
constexpr int HOP_LIMIT = 4096;
constexpr double ONE_SIXTH = 1.0 / 6.0;
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) unsigned long long g_scratch[SCRATCH_WORDS];

// The reference's records (src/particles.h:21-26, src/meshes.h:33-43).
constexpr int P_SIZE = 88, P_POS = 0, P_VEL = 24, P_LC = 48, P_CELL = 80;
constexpr int T_SIZE = 168, T_CON = 0, T_VOL = 16, T_ALPHA = 24, T_BETA = 56, T_GAMMA = 88, T_DELTA = 120,
              T_CELLCON = 152;

__device__ __forceinline__ double ldd(const char *base, long long off) {
    return __ldg(reinterpret_cast<const double *>(base + off));
}
__device__ __forceinline__ int ldi(const char *base, long long off) {
    return __ldg(reinterpret_cast<const int *>(base + off));
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ long long lookback(unsigned long long *w, long long tile, long long count) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> mine(w[W_TILES + tile]);
    if (tile == 0) {
        mine.store(ST_PREFIX | (unsigned long long)count, cuda::memory_order_release);
        return 0;
    }
    mine.store(ST_AGG | (unsigned long long)count, cuda::memory_order_release);
    long long excl = 0, p = tile - 1, spins = 0;
    while (p >= 0) {
        cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> prev(w[W_TILES + p]);
        unsigned long long s = prev.load(cuda::memory_order_acquire);
        unsigned long long flag = s & ~ST_VALUE;
        if (flag == 0) {
            if (++spins > SPIN_LIMIT) {
                atomicOr(&w[W_FLAGS], mp::FLAG_LOOKBACK_TIMEOUT);
                break;
            }
            continue;
        }
        excl += (long long)(s & ST_VALUE);
        if (flag == ST_PREFIX) break;
        p--;
    }
    mine.store(ST_PREFIX | (unsigned long long)(excl + count), cuda::memory_order_release);
    return excl;
}

// One particle per thread, the reference's kernel body (src/mini-pic.cpp:287-308)
// with XtoLtet (src/meshes.h:75-100) in its expression order; survivors are
// written stably to `out` (which may be `in`: a tile writes only below its own
// end, after every earlier tile has read its input).
__global__ void __launch_bounds__(THREADS) k_push_aos(const char *in, char *out, long long n, const char *tetra,
                                                      int n_tets, const double *__restrict__ ef, double *den,
                                                      int n_nodes, double qm, double dt, unsigned long long *w) {
    __shared__ long long s_tile, s_base;
    __shared__ int s_wc[THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long n_tiles = (n + THREADS - 1) / THREADS;
    for (;;) {
        if (threadIdx.x == 0) s_tile = (long long)atomicAdd(&w[W_TICKET], 1ull);
        __syncthreads();
        const long long tile = s_tile;
        if (tile >= n_tiles) break;
        const long long i = tile * THREADS + threadIdx.x;
        bool keep = false;
        int cell = -1;
        double x[3] = {0, 0, 0}, v[3] = {0, 0, 0}, lc[4] = {0, 0, 0, 0};
        if (i < n) {
            const char *p = in + i * P_SIZE;
            for (int k = 0; k < 3; k++) {
                x[k] = ldd(p, P_POS + 8 * k);
                v[k] = ldd(p, P_VEL + 8 * k);
            }
            cell = ldi(p, P_CELL);
            if (cell < 0 || cell >= n_tets) {
                // not a particle of this mesh: written out as it came, nothing scattered
                keep = true;
                for (int k = 0; k < 4; k++) lc[k] = ldd(p, P_LC + 8 * k);
                atomicOr(&w[W_FLAGS], mp::FLAG_BAD_INDEX);
            }
        }
        if (i < n && !keep) {
            for (int k = 0; k < 3; k++) v[k] = __dadd_rn(v[k], __dmul_rn(__dmul_rn(qm, ef[3ll * cell + k]), dt));
            for (int k = 0; k < 3; k++) x[k] = __dadd_rn(x[k], __dmul_rn(v[k], dt));
            int hops = 0;
            for (;;) {
                const char *t = tetra + (long long)cell * T_SIZE;
                double vol = ldd(t, T_VOL);
                bool inside = true;
                for (int q = 0; q < 4; q++) {
                    double s = __dsub_rn(ldd(t, T_ALPHA + 8 * q), __dmul_rn(x[0], ldd(t, T_BETA + 8 * q)));
                    s = __dadd_rn(s, __dmul_rn(x[1], ldd(t, T_GAMMA + 8 * q)));
                    s = __dsub_rn(s, __dmul_rn(x[2], ldd(t, T_DELTA + 8 * q)));
                    lc[q] = __ddiv_rn(__dmul_rn(ONE_SIXTH, s), vol);
                    if (lc[q] < 0 || lc[q] > 1.0) inside = false;
                }
                if (inside) {
                    keep = true;
                    int nodes[4];
                    bool ok = true;
                    for (int q = 0; q < 4; q++) {
                        nodes[q] = ldi(t, T_CON + 4 * q);
                        ok = ok && nodes[q] >= 0 && nodes[q] < n_nodes;
                    }
                    if (ok) {
                        for (int q = 0; q < 4; q++) atomicAdd(&den[nodes[q]], lc[q]);
                    } else {
                        atomicOr(&w[W_FLAGS], mp::FLAG_BAD_INDEX);
                    }
                    break;
                }
                int mi = 0;
                double ml = lc[0];
                for (int q = 1; q < 4; q++)
                    if (lc[q] < ml) {
                        ml = lc[q];
                        mi = q;
                    }
                int nb = ldi(t, T_CELLCON + 4 * mi);
                if (nb < 0) break;
                if (nb >= n_tets) {
                    keep = true;  // kept in the last valid tet, not scattered
                    atomicOr(&w[W_FLAGS], mp::FLAG_BAD_INDEX);
                    break;
                }
                if (hops >= HOP_LIMIT) {
                    keep = true;  // kept where the walk stopped, not scattered
                    atomicOr(&w[W_FLAGS], mp::FLAG_WALK_LIMIT);
                    break;
                }
                cell = nb;
                hops++;
            }
        }
        __syncwarp();
        unsigned kb = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) s_wc[warp] = __popc(kb);
        __syncthreads();
        if (threadIdx.x == 0) {
            long long run = 0;
            for (int k = 0; k < THREADS / 32; k++) {
                int c = s_wc[k];
                s_wc[k] = (int)run;
                run += c;
            }
            long long excl = lookback(w, tile, run);
            s_base = excl;
            if (tile == n_tiles - 1) w[W_KEPT] = (unsigned long long)(excl + run);
        }
        __syncthreads();
        if (keep) {
            long long o = s_base + s_wc[warp] + __popc(kb & lanemask_lt());
            double *q = reinterpret_cast<double *>(out + o * P_SIZE);
            for (int k = 0; k < 3; k++) {
                q[k] = x[k];
                q[3 + k] = v[k];
            }
            for (int k = 0; k < 4; k++) q[6 + k] = lc[k];
            *reinterpret_cast<int *>(out + o * P_SIZE + P_CELL) = cell;
        }
        __syncthreads();
    }
}

static std::mutex g_mu;
static unsigned long long *g_addr[MAX_DEVICES];

static int scratch_address(int device, unsigned long long **out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[device]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) return MP_ERR_CUDA;
        g_addr[device] = reinterpret_cast<unsigned long long *>(p);
    }
    *out = g_addr[device];
    return MP_OK;
}

}  // namespace mp_noalloc

extern "C" int mp_push_particles_noalloc(const void *particles_in, void *particles_out, int64_t n,
                                         const void *tetra, int32_t n_tets, const double *ef, double *den,
                                         int32_t n_nodes, double q_over_m, double dt, void *stream,
                                         int64_t *n_out) {
    using namespace mp_noalloc;
    if (n < 0 || !n_out || n_nodes <= 0 || n_tets <= 0 || !den) return MP_ERR_ARG;
    if (n > MAX_PARTICLES) return MP_ERR_LIMIT;
    if (n > 0 && (!particles_in || !particles_out || !tetra || !ef)) return MP_ERR_ARG;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= MAX_DEVICES) return MP_ERR_NO_DEVICE;
    unsigned long long *w = nullptr;
    int rc = scratch_address(device, &w);
    if (rc) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const long long tiles = (n + THREADS - 1) / THREADS;
    // the counters and this call's tile words must start at zero
    if (cudaMemsetAsync(w, 0, sizeof(unsigned long long) * (W_TILES + tiles), st) != cudaSuccess) return MP_ERR_CUDA;
    if (cudaMemsetAsync(den, 0, sizeof(double) * n_nodes, st) != cudaSuccess) return MP_ERR_CUDA;
    if (n > 0) {
        int per_sm = 0, sms = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_push_aos, THREADS, 0);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        long long grid = (long long)(per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
        if (grid > tiles) grid = tiles;
        k_push_aos<<<(unsigned)grid, THREADS, 0, st>>>(static_cast<const char *>(particles_in),
                                                        static_cast<char *>(particles_out), n,
                                                        static_cast<const char *>(tetra), n_tets, ef, den, n_nodes,
                                                        q_over_m, dt, w);
        if (cudaGetLastError() != cudaSuccess) return MP_ERR_CUDA;
    }
    unsigned long long res[3] = {0, 0, 0};
    if (cudaMemcpyAsync(res, w, sizeof(res), cudaMemcpyDeviceToHost, st) != cudaSuccess) return MP_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return MP_ERR_CUDA;
    *n_out = (int64_t)res[W_KEPT];
    if (res[W_FLAGS] & mp::FLAG_LOOKBACK_TIMEOUT) return MP_ERR_TIMEOUT;
    if (res[W_FLAGS] & mp::FLAG_BAD_INDEX) return MP_ERR_ARG;
    if (res[W_FLAGS] & mp::FLAG_WALK_LIMIT) return MP_ERR_WALK_LIMIT;
    return MP_OK;
}
