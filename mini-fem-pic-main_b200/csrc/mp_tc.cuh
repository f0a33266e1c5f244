// Tensor-core (tcgen05, TF32 inputs, FP32 accumulators in TMEM) trailing update
// of the mixed-form LDL^T:  A[i][j] -= sum_k L[i][k] W[j][k]  on the lower
// 128x128 tiles of the trailing matrix.
//
// One CTA per output tile, 128 threads (4 warps, one per 32 TMEM lanes).  The
// K dimension streams through shared memory in 32-element chunks, two stages:
// all threads copy a chunk of L (128 rows) and of W (128 rows) into the
// K-major 128-byte-swizzled layout the UMMA descriptors describe, then one
// thread issues four 128x128x8 tcgen05.mma (kind::tf32) and commits them to the
// stage's mbarrier, which tells the loaders when the stage may be refilled.
// The epilogue reads the accumulator with tcgen05.ld and subtracts it from the
// tile in global memory.  No multicast and no cluster: each CTA loads its own
// operands.  Every mbarrier wait is bounded; a timeout sets the error bit
// FLAG_LOOKBACK_TIMEOUT, reported as MP_ERR_TIMEOUT by the caller.
//
// SPLIT (3xTF32): each FP32 operand x is split on the way into shared memory
// into hi = x rounded to TF32 (11 significant bits) and lo = x - hi (exact in
// FP32), and the product is accumulated as hi*hi + hi*lo + lo*hi, three MMAs on
// the same TMEM accumulator.  The dropped lo*lo term is ~2^-22 relative, so the
// update carries about FP32 accuracy instead of TF32's 2^-11, which is what the
// FP64 refinement of the mixed solve converges against.
#pragma once

#include "mp_internal.h"

namespace mp {
namespace tc {

constexpr int TILE = 128;         // M = N = 128
constexpr int KC = 32;            // K elements per chunk (one 128-byte swizzle atom row)
constexpr int CHUNK_BYTES = TILE * KC * 4;  // 16 KB per operand per stage
constexpr int THREADS = 128;
constexpr long long SPIN_LIMIT = 1ll << 22;

__device__ __forceinline__ unsigned saddr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr) {
    return (unsigned long long)((addr >> 4) & 0x3FFF) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor: D F32, A/B TF32, both K-major, M = 128, N = 128.
constexpr unsigned IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mbar_init(unsigned long long *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
    long long spins = 0;
    while (!mbar_try(bar, parity))
        if (++spins > SPIN_LIMIT) return false;
    return true;
}

__device__ __forceinline__ void mma_tf32(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(IDESC), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}
__device__ __forceinline__ void mma_commit(unsigned long long *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

// x rounded to the nearest TF32 value (low 13 mantissa bits cleared)
__device__ __forceinline__ float tf32_hi(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// Copies rows [r0, r0+128) x cols [k0, k0+32) of a row-major FP32 matrix into
// one swizzled chunk (and, for SPLIT, its hi part into dst and lo part into
// dst_lo); rows >= nrows and cols >= kmax are zero.
template <bool SPLIT>
__device__ __forceinline__ void load_chunk(unsigned char *dst, unsigned char *dst_lo, const float *src, long long ld,
                                           long long r0, long long nrows, int k0, int kmax) {
    // 128 rows x 8 sixteen-byte pieces = 1024 pieces, 8 per thread; all eight
    // loads are issued before any store so they are in flight together
    float4 v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        int piece = q * THREADS + threadIdx.x;
        int r = piece >> 3, c = piece & 7;
        long long row = r0 + r;
        int col = k0 + c * 4;
        v[q] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (row < nrows) {
            const float *p = src + row * ld + col;
            if (col + 3 < kmax) {
                v[q] = __ldg(reinterpret_cast<const float4 *>(p));
            } else {
                if (col < kmax) v[q].x = __ldg(p);
                if (col + 1 < kmax) v[q].y = __ldg(p + 1);
                if (col + 2 < kmax) v[q].z = __ldg(p + 2);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
        int piece = q * THREADS + threadIdx.x;
        int r = piece >> 3, c = piece & 7;
        const int off = r * 128 + ((c ^ (r & 7)) << 4);
        if constexpr (SPLIT) {
            const float4 h = make_float4(tf32_hi(v[q].x), tf32_hi(v[q].y), tf32_hi(v[q].z), tf32_hi(v[q].w));
            *reinterpret_cast<float4 *>(dst + off) = h;
            *reinterpret_cast<float4 *>(dst_lo + off) =
                make_float4(v[q].x - h.x, v[q].y - h.y, v[q].z - h.z, v[q].w - h.w);
        } else {
            *reinterpret_cast<float4 *>(dst + off) = v[q];
        }
    }
}

// A[i][j] -= sum_{k<K} L[i][k] * W[j][k] for the lower tiles of rows/cols
// [k1, n).  L = Abase + k0 (row-major, ld), W row-major with leading dim ldw.
// Each CTA takes lower tile number blockIdx.x.
template <bool SPLIT>
__global__ void __launch_bounds__(THREADS, 1) k_update_tf32(int n, long long ld, float *A, int k0, int K, int k1,
                                                           const float *W, int ldw, unsigned long long *flags) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // align the operand stages to 1024 B (swizzle atoms)
    unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<size_t>(smem_raw) + 1023) & ~size_t(1023));
    // stage s: L hi, W hi (and for SPLIT: L lo, W lo), CHUNK_BYTES each
    constexpr int PER_STAGE = SPLIT ? 4 : 2;
    __shared__ unsigned long long bars[3];
    __shared__ unsigned tmem_slot;
    __shared__ int s_bad;

    long long bidx = blockIdx.x;
    int bi = (int)((sqrt(8.0 * (double)bidx + 1.0) - 1.0) * 0.5);
    while ((long long)(bi + 1) * (bi + 2) / 2 <= bidx) bi++;
    while ((long long)bi * (bi + 1) / 2 > bidx) bi--;
    const int bj = (int)(bidx - (long long)bi * (bi + 1) / 2);
    const long long i0 = k1 + (long long)bi * TILE, j0 = k1 + (long long)bj * TILE;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        mbar_init(&bars[0]);
        mbar_init(&bars[1]);
        mbar_init(&bars[2]);
        // an earlier tile of this factorization timed out: do nothing more
        s_bad = (*(volatile unsigned long long *)flags & FLAG_LOOKBACK_TIMEOUT) ? 2 : 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (s_bad) return;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(saddr(&tmem_slot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = tmem_slot;

    const float *Lrows = A + k0;  // L[i][k] = A[i*ld + k0 + k]
    const int nchunks = (K + KC - 1) / KC;
    bool ok = true;
    for (int c = 0; c < nchunks; c++) {
        const int s = c & 1;
        if (c >= 2) {
            // the MMAs of chunk c-2 read this stage: wait for their commit
            // chunk c-2 was use number (c-2)/2 of this stage: its commit completes that phase
            if (!mbar_wait(&bars[s], (unsigned)((c >> 1) - 1) & 1u)) ok = false;
        }
        unsigned char *sa = base + s * PER_STAGE * CHUNK_BYTES, *sb = sa + CHUNK_BYTES;
        unsigned char *sal = sa + 2 * CHUNK_BYTES, *sbl = sa + 3 * CHUNK_BYTES;  // SPLIT only
        load_chunk<SPLIT>(sa, sal, Lrows, ld, i0, n, c * KC, K);
        load_chunk<SPLIT>(sb, sbl, W, ldw, j0, n, c * KC, K);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned long long da = smem_desc(saddr(sa)), db = smem_desc(saddr(sb));
            const unsigned long long dal = smem_desc(saddr(sal)), dbl = smem_desc(saddr(sbl));
#pragma unroll
            for (int kk = 0; kk < KC / 8; kk++) {  // 8 TF32 = 32 B per MMA step: +2 in the descriptor
                if constexpr (SPLIT) {
                    mma_tf32(tmem, dal + 2 * kk, db + 2 * kk, (c > 0 || kk > 0) ? 1u : 0u);
                    mma_tf32(tmem, da + 2 * kk, dbl + 2 * kk, 1u);
                    mma_tf32(tmem, da + 2 * kk, db + 2 * kk, 1u);
                } else {
                    mma_tf32(tmem, da + 2 * kk, db + 2 * kk, (c > 0 || kk > 0) ? 1u : 0u);
                }
            }
            mma_commit(&bars[s]);
        }
    }
    // all MMAs done: the last commit covers every earlier MMA of this thread
    if (threadIdx.x == 0) mma_commit(&bars[2]);
    if (!mbar_wait(&bars[2], 0)) ok = false;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) s_bad = 1;
    // epilogue, in two halves of 64 columns: TMEM -> registers -> shared
    // (row-major, padded), then each warp subtracts whole rows from the tile
    // with coalesced loads and stores (the operand stages are free now)
    float(*sD)[65] = reinterpret_cast<float(*)[65]>(base);
    const unsigned taddr = tmem + ((unsigned)(warp * 32) << 16);
#pragma unroll 1
    for (int half = 0; half < 2; half++) {
#pragma unroll 1
        for (int cb = 0; cb < 4; cb++) {
            unsigned v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(taddr + half * 64 + cb * 16));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 16; q++) sD[warp * 32 + lane][cb * 16 + q] = __uint_as_float(v[q]);
        }
        __syncthreads();
        const long long c0 = j0 + half * 64 + lane;
#pragma unroll 1
        for (int rr = 0; rr < 32; rr += 4) {
            float old[4][2];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const long long row = i0 + warp * 32 + rr + u;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const long long col = c0 + h * 32;
                    old[u][h] = (row < n && col < n) ? A[row * ld + col] : 0.f;
                }
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const long long row = i0 + warp * 32 + rr + u;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const long long col = c0 + h * 32;
                    // the strict upper part of the diagonal tiles is never read again; skip it anyway
                    if (row < n && col < n && col <= row)
                        A[row * ld + col] = old[u][h] - sD[warp * 32 + rr + u][lane + h * 32];
                }
            }
        }
        __syncthreads();
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(tmem) : "memory");
    if (threadIdx.x == 0 && s_bad) atomicOr(flags, FLAG_LOOKBACK_TIMEOUT);
}

// two stages of the operand chunks + alignment slack
constexpr size_t smem_bytes(bool split) { return (split ? 8 : 4) * (size_t)CHUNK_BYTES + 1024; }

}  // namespace tc
}  // namespace mp
