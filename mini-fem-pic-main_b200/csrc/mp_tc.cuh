// Tensor-core (tcgen05, TF32 inputs, FP32 accumulators in TMEM) trailing update
// of the mixed-form LDL^T:  A[i][j] -= sum_k L[i][k] W[j][k]  on the tiles of
// 128 rows x 256 columns that meet the lower triangle of the trailing matrix,
// K = one 256-wide outer panel.  The 256-wide tiles halve the operand bytes
// per FLOP against square 128 x 128 tiles (the operand stream from L2 is what
// bounds this kernel).
//
// Persistent, warp-specialised.  One CTA per SM walks the lower tiles
// blockIdx.x, blockIdx.x + gridDim.x, ...:
//   warp 0 (one lane)  producer: 2-D TMA tile loads (cp.async.bulk.tensor, no
//                      multicast, 128-byte swizzle) of 32-wide K chunks of the
//                      tile's L rows and W rows into STAGES shared-memory
//                      stages, each completing on its stage's "full" mbarrier;
//   warp 1 (one lane)  MMA issuer: tcgen05.mma.cta_group::1.kind::tf32 (M = 128,
//                      N = 256) from the stage into one of two 256-column TMEM
//                      accumulators (all 512 columns), then
//                      tcgen05.commit to the stage's "empty" mbarrier (frees it
//                      for the producer) and, after a tile's last chunk, to the
//                      accumulator's "full" mbarrier;
//   warps 2-17         epilogue: tcgen05.ld of their 32 TMEM lanes (= tile rows),
//                      64 columns a warp,
//                      A[row][col] -= acc for col <= row, then arrive on the
//                      accumulator's "empty" mbarrier.
// Two accumulators let the epilogue of one tile overlap the MMAs of the next.
//
// Operand modes:
//   MODE_TF32    the TMA reads L straight from the factor and W from the panel
//                scratch; one TF32 product a term (2^-11 relative).
//   MODE_TF32X3  the operands arrive pre-split by k_split_rows into hi = x
//                rounded to TF32 (11 significant bits) and lo = x - hi (exact
//                in FP32); each tile accumulates hi*hi + hi*lo + lo*hi on the
//                same TMEM accumulator.  The dropped lo*lo term is ~2^-22
//                relative: about FP32 accuracy, three times the MMAs.
//   MODE_F16     FP16 copies of the operands (k_half_operands), scaled by powers
//                of two into FP16's range, kind::f16 MMAs with FP32
//                accumulation, and the epilogue multiplies by the inverse scale.
//                FP16 keeps TF32's 11 significant bits (rounded to nearest), so
//                a term is as accurate as MODE_TF32's, while a 128-byte chunk
//                row carries 64 values instead of 32: half the operand bytes
//                from L2 per flop, at twice the tensor rate.
// Every mode's shared-memory chunk rows are 128 bytes (one swizzle row) and an
// MMA consumes 32 bytes of each row (8 TF32 or 16 FP16 values), so the
// descriptors and stage layout are the same in all three.
//
// Every mbarrier wait is bounded.  A wait that gives up raises a CTA-wide abort
// flag; every role leaves its loop, the producer and the MMA issuer wait
// (bounded) for their copies and MMAs in flight, TMEM is freed, and the kernel
// sets FLAG_LOOKBACK_TIMEOUT (reported as MP_ERR_TIMEOUT by the caller).
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>

#include "mp_internal.h"

namespace mp {
namespace tc {

constexpr int TILE = 128;                   // M: tile rows
constexpr int TILE_N = 256;                 // N: tile columns
enum { MODE_TF32 = 0, MODE_TF32X3 = 1, MODE_F16 = 2 };
constexpr int KC = 32;                      // FP32 elements per chunk row (one 128-byte swizzle row)
constexpr int CHUNK_L = TILE * 128;         // 16 KB: one L operand chunk
constexpr int CHUNK_W = TILE_N * 128;       // 32 KB: one W operand chunk
// K elements per chunk: one 128-byte row of 4-byte or 2-byte values
__host__ __device__ constexpr int kc_of(int mode) { return mode == MODE_F16 ? 64 : 32; }
__host__ __device__ constexpr int stages(int mode) { return mode == MODE_TF32X3 ? 2 : 4; }  // 192 KB of stages
constexpr int EPI_WARPS = 16;               // epilogue: 4 per TMEM lane quadrant, 64 columns each
constexpr int THREADS = 64 + 32 * EPI_WARPS; // producer warp, MMA warp, epilogue warps
constexpr long long SPIN_LIMIT = 1ll << 22;

__device__ __forceinline__ unsigned saddr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr) {
    return (unsigned long long)((addr >> 4) & 0x3FFF) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptors: D F32, A/B TF32 (format 2 of kind::tf32) or F16
// (format 0 of kind::f16), both K-major, M = 128, N = 256.
constexpr unsigned IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((256u >> 3) << 17) | ((128u >> 4) << 24);
constexpr unsigned IDESC_F16 = (1u << 4) | (0u << 7) | (0u << 10) | ((256u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
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
__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}
// Bounded wait; false when it gave up (then the abort flag is set) or another
// role already aborted.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, volatile int *abort) {
    for (long long i = 0;; i++) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 255) == 255 && *abort) return false;
        if (i > SPIN_LIMIT) {
            *abort = 1;
            return false;
        }
    }
}

// 2-D tiled TMA load of the map's box at element coordinates (x, y).
__device__ __forceinline__ void tma_load(void *dst, const CUtensorMap *map, int x, int y, unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(saddr(dst)), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(saddr(bar))
        : "memory");
}

// 2-D tiled TMA store of a shared-memory box to the map at (x, y); completes
// in this thread's bulk async-group.  Rows and columns past the map's extent
// are not written.
__device__ __forceinline__ void tma_store(const CUtensorMap *map, int x, int y, const void *src) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                     reinterpret_cast<unsigned long long>(map)),
                 "r"(x), "r"(y), "r"(saddr(src))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// generic-proxy writes to shared memory made visible to a following TMA store
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mma_tf32(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(IDESC), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}
__device__ __forceinline__ void mma_f16(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(IDESC_F16), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}
__device__ __forceinline__ void mma_commit(unsigned long long *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

// Tile number -> (bi, bj): 128-row block bi, 256-column block bj, over the
// tiles that meet the lower triangle (bj <= bi/2).  Row blocks 2M and 2M+1
// both hold M+1 tiles, so tiles before row block 2M number M(M+1) and before
// 2M+1 number (M+1)^2.
__device__ __forceinline__ void tile_coords(long long t, int &bi, int &bj) {
    long long M = (long long)((sqrt(4.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((M + 1) * (M + 2) <= t) M++;
    while (M * (M + 1) > t) M--;
    if (t < (M + 1) * (M + 1)) {
        bi = (int)(2 * M);
        bj = (int)(t - M * (M + 1));
    } else {
        bi = (int)(2 * M + 1);
        bj = (int)(t - (M + 1) * (M + 1));
    }
}
__device__ __forceinline__ void tile_of(long long t, int colblocks, int &bi, int &bj) {
    if (colblocks > 0) {
        bi = (int)(t / colblocks);
        bj = (int)(t % colblocks);
    } else {
        tile_coords(t, bi, bj);
    }
}
// number of tiles over `rb` row blocks
__host__ __device__ inline long long tile_count(long long rb) {
    const long long M = rb / 2;
    return (rb & 1) ? (M + 1) * (M + 1) : M * (M + 1);
}

// x rounded to the nearest TF32 value (low 13 mantissa bits cleared)
__device__ __forceinline__ float tf32_hi(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// Splits rows [0, nrows) x columns [0, K) of a row-major FP32 operand (pitch
// ld) into hi/lo arrays [nrows][K] for the TMA (K a multiple of 4).
__global__ void k_split_rows(const float *__restrict__ src, long long ld, long long nrows, int K, float *hi,
                             float *lo) {
    const long long total = nrows * (K / 4);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const long long r = q / (K / 4);
        const int c = (int)(q % (K / 4)) * 4;
        const float4 x = __ldg(reinterpret_cast<const float4 *>(src + r * ld + c));
        const float4 h = make_float4(tf32_hi(x.x), tf32_hi(x.y), tf32_hi(x.z), tf32_hi(x.w));
        const long long o = r * K + c;
        *reinterpret_cast<float4 *>(hi + o) = h;
        *reinterpret_cast<float4 *>(lo + o) = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
    }
}

// FP16 operands of a MODE_F16 update: rows [0, nl) of L (pitch ldl) and rows
// [0, nw) of W (pitch ldw) over K columns (a multiple of 8) into [nl][K] and
// [nw][K] arrays.  L is scaled by 2^L_EXP, W by 2^e with e set so the largest
// |d_k| of the K pivots dk lands in [2^4, 2^5) (|W_jk| = |L_jk| |d_k|), and
// *unscale = 2^-(L_EXP + e); every block finds the same e.  In the factor of a
// diagonally dominant J every |L_jk| <= 1, so both copies stay at least 2^7
// below FP16's largest value (65504); a value that would not fit sets
// FLAG_HALF_RANGE and the caller factors again with TF32 operands.  Values
// below 2^-14 of the scale lose bits as FP16 subnormals: absolute errors under
// 2^-25 2^-L_EXP for L and 2^-29 max|d_k| for W, far below the 2^-11 relative
// rounding of the larger terms.
constexpr int L_EXP = 8;
__global__ void __launch_bounds__(256) k_half_operands(const float *__restrict__ L, long long ldl, long long nl,
                                                       const float *__restrict__ W, long long ldw, long long nw,
                                                       int K, const float *__restrict__ dk, __half *Lh, __half *Wh,
                                                       float *unscale, unsigned long long *flags) {
    __shared__ float sred[8];
    float m = 0.f;
    for (int k = threadIdx.x; k < K; k += 256) m = fmaxf(m, fabsf(dk[k]));
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = m;
    __syncthreads();
    m = sred[0];
#pragma unroll
    for (int w = 1; w < 8; w++) m = fmaxf(m, sred[w]);
    // floor(log2 m) from the exponent field (m normal); e clamped so 2^e and
    // 2^-(L_EXP + e) are normal floats
    int e = 0;
    if (m >= 1.17549435e-38f && m <= 3.40282347e38f) e = 4 - (int)((__float_as_uint(m) >> 23) & 0xff) + 127;
    e = e < -100 ? -100 : (e > 100 ? 100 : e);
    const float sl = (float)(1 << L_EXP), sw = __uint_as_float((unsigned)(127 + e) << 23);
    if (blockIdx.x == 0 && threadIdx.x == 0) *unscale = __uint_as_float((unsigned)(127 - L_EXP - e) << 23);
    const int g8 = K / 8;
    const long long total = (nl + nw) * g8;
    bool bad = false;
    for (long long q = blockIdx.x * 256ll + threadIdx.x; q < total; q += (long long)gridDim.x * 256) {
        long long r = q / g8;
        const int c = (int)(q - r * g8) * 8;
        const float *src;
        __half *dst;
        float sc;
        if (r < nl) {
            src = L + r * ldl + c;
            dst = Lh + r * K + c;
            sc = sl;
        } else {
            r -= nl;
            src = W + r * ldw + c;
            dst = Wh + r * K + c;
            sc = sw;
        }
        const float4 a = __ldg(reinterpret_cast<const float4 *>(src));
        const float4 b = __ldg(reinterpret_cast<const float4 *>(src) + 1);
        const float v[8] = {a.x * sc, a.y * sc, a.z * sc, a.w * sc, b.x * sc, b.y * sc, b.z * sc, b.w * sc};
        uint4 o;
        unsigned *ow = reinterpret_cast<unsigned *>(&o);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            bad |= fabsf(v[2 * j]) >= 65520.f || fabsf(v[2 * j + 1]) >= 65520.f;
            const __half2 h = __floats2half2_rn(v[2 * j], v[2 * j + 1]);
            ow[j] = *reinterpret_cast<const unsigned *>(&h);
        }
        *reinterpret_cast<uint4 *>(dst) = o;
    }
    if (bad) atomicOr(flags, FLAG_HALF_RANGE);
}

// A[i][j] -= sum_{k<K} L[i][k] W[j][k] (K = 32*nchunk) for rows from P1 and
// columns from P1.  colblocks = 0: the 128 x 256 tiles that meet the lower
// triangle of [P1, n)^2 (the trailing update of a super-panel); colblocks > 0:
// every tile of rows [P1, n) x columns [P1, P1 + 256*colblocks) (a strip inside
// a super-panel), lower parts only.  The L maps cover the rows from P1 (rows
// past the end read as zero) and load boxes of 128 rows; the W maps cover the
// output columns' rows and load boxes of 256 rows.
template <int MODE>
__global__ void __launch_bounds__(THREADS, 1)
    k_update_tc(const __grid_constant__ CUtensorMap mLh, const __grid_constant__ CUtensorMap mWh,
                const __grid_constant__ CUtensorMap mLl, const __grid_constant__ CUtensorMap mWl, int n, long long ld,
                float *A, int P1, long long ntiles, int nchunk, int colblocks, const float *unscale,
                unsigned long long *flags) {
    constexpr bool SPLIT = MODE == MODE_TF32X3;
    constexpr int KCE = kc_of(MODE);
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<size_t>(smem_raw) + 1023) & ~size_t(1023));
    constexpr int STAGES = stages(MODE);
    // stage: L hi, W hi (, L lo, W lo)
    constexpr unsigned STAGE_BYTES = SPLIT ? 2 * (CHUNK_L + CHUNK_W) : CHUNK_L + CHUNK_W;
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(base + STAGES * STAGE_BYTES);
    unsigned long long *full = bars, *empty = bars + STAGES, *acc_full = bars + 2 * STAGES,
                       *acc_empty = bars + 2 * STAGES + 2, *drain = bars + 2 * STAGES + 4;
    unsigned *tmem_slot = reinterpret_cast<unsigned *>(bars + 2 * STAGES + 5);
    volatile int *abort = reinterpret_cast<volatile int *>(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], EPI_WARPS * 32);
        }
        mbar_init(drain, 1);
        // an earlier launch of this factorization timed out: do nothing more
        *abort = (*(volatile unsigned long long *)flags & FLAG_LOOKBACK_TIMEOUT) ? 2 : 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(saddr(tmem_slot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = *tmem_slot;

    if (*abort == 0) {
        if (warp == 0 && lane == 0) {
            // ---- producer ----
            long long it = 0;
            bool ok = true;
            for (long long t = blockIdx.x; ok && t < ntiles; t += gridDim.x) {
                int bi, bj;
                tile_of(t, colblocks, bi, bj);
                for (int kc = 0; kc < nchunk; kc++, it++) {
                    const int s = (int)(it % STAGES);
                    const long long u = it / STAGES;
                    if (u > 0 && !mbar_wait(&empty[s], (unsigned)((u - 1) & 1), abort)) {
                        ok = false;
                        break;
                    }
                    unsigned char *st = base + s * STAGE_BYTES;
                    mbar_expect_tx(&full[s], STAGE_BYTES);
                    tma_load(st, &mLh, kc * KCE, bi * TILE, &full[s]);
                    tma_load(st + CHUNK_L, &mWh, kc * KCE, bj * TILE_N, &full[s]);
                    if (SPLIT) {
                        tma_load(st + CHUNK_L + CHUNK_W, &mLl, kc * KCE, bi * TILE, &full[s]);
                        tma_load(st + 2 * CHUNK_L + CHUNK_W, &mWl, kc * KCE, bj * TILE_N, &full[s]);
                    }
                }
            }
            // the last loads of each stage have landed before the CTA may exit
            for (long long k = it - STAGES; k < it; k++) {
                if (k < 0) continue;
                const int s = (int)(k % STAGES);
                long long spins = 0;
                while (!mbar_try(&full[s], (unsigned)((k / STAGES) & 1)) && ++spins < SPIN_LIMIT) {
                }
            }
        } else if (warp == 1 && lane == 0) {
            // ---- MMA issuer ----
            long long it = 0, lt = 0;
            bool ok = true;
            for (long long t = blockIdx.x; ok && t < ntiles; t += gridDim.x, lt++) {
                const int a = (int)(lt & 1);
                const long long v = lt >> 1;
                if (v > 0 && !mbar_wait(&acc_empty[a], (unsigned)((v - 1) & 1), abort)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const unsigned d = tmem + (unsigned)(a * TILE_N);
                for (int kc = 0; kc < nchunk; kc++, it++) {
                    const int s = (int)(it % STAGES);
                    if (!mbar_wait(&full[s], (unsigned)((it / STAGES) & 1), abort)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const unsigned char *st = base + s * STAGE_BYTES;
                    const unsigned long long dl = smem_desc(saddr(st)), dw = smem_desc(saddr(st + CHUNK_L));
                    const unsigned long long dll = smem_desc(saddr(st + CHUNK_L + CHUNK_W));
                    const unsigned long long dwl = smem_desc(saddr(st + 2 * CHUNK_L + CHUNK_W));
#pragma unroll
                    for (int kk = 0; kk < 4; kk++) {  // 32 B of each row (8 TF32, 16 FP16) per MMA: +2 in the descriptor
                        const unsigned accum = (kc > 0 || kk > 0) ? 1u : 0u;
                        if (MODE == MODE_F16) {
                            mma_f16(d, dl + 2 * kk, dw + 2 * kk, accum);
                        } else if (SPLIT) {
                            mma_tf32(d, dll + 2 * kk, dw + 2 * kk, accum);
                            mma_tf32(d, dl + 2 * kk, dwl + 2 * kk, 1u);
                            mma_tf32(d, dl + 2 * kk, dw + 2 * kk, 1u);
                        } else {
                            mma_tf32(d, dl + 2 * kk, dw + 2 * kk, accum);
                        }
                    }
                    mma_commit(&empty[s]);  // the stage is free once these MMAs have read it
                }
                if (!ok) break;
                mma_commit(&acc_full[a]);  // the accumulator is complete
            }
            // every MMA this thread issued has completed once this commit arrives
            mma_commit(drain);
            long long spins = 0;
            while (!mbar_try(drain, 0) && ++spins < SPIN_LIMIT) {
            }
        } else if (warp >= 2) {
            // ---- epilogue: EPI_WARPS warps; warp w reads TMEM lanes 32*(w%4) .. +31
            // (its tile rows, the lanes a warp may access) and owns columns
            // 64*((w-2)/4) .. +63 of them.  A thread loads the old values of its
            // row's 64 columns before it waits for the accumulator (they do not
            // depend on the MMAs), so 16 loads a thread, 128 KB a CTA, are in
            // flight behind the next tile's MMAs.
            const int q = warp & 3;
            const int r = q * 32 + lane;
            const int cq = (warp - 2) >> 2;
            const float us = MODE == MODE_F16 ? *unscale : 1.0f;  // a power of two: the products stay exact
            long long lt = 0;
            for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, lt++) {
                int bi, bj;
                tile_of(t, colblocks, bi, bj);
                const long long row = P1 + (long long)bi * TILE + r;
                const long long c0 = P1 + (long long)bj * TILE_N + 64 * cq;
                const bool row_ok = row < n;
                float4 cur[16];
#pragma unroll
                for (int g = 0; g < 16; g++) {
                    const long long col = c0 + 4 * g;
                    cur[g] = (row_ok && col + 3 <= row && col + 3 < n)
                                 ? *reinterpret_cast<const float4 *>(A + row * ld + col)
                                 : make_float4(0.f, 0.f, 0.f, 0.f);
                }
                const int a = (int)(lt & 1);
                int ok = 1;
                if (lane == 0) ok = mbar_wait(&acc_full[a], (unsigned)((lt >> 1) & 1), abort);
                ok = __shfl_sync(0xffffffffu, ok, 0);
                if (!ok) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const unsigned taddr = tmem + (unsigned)(a * TILE_N + 64 * cq) + ((unsigned)(q * 32) << 16);
#pragma unroll
                for (int cb = 0; cb < 4; cb++) {
                    unsigned v[16];
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
                        "%15}, [%16];"
                        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                          "=r"(v[14]), "=r"(v[15])
                        : "r"(taddr + cb * 16));
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    const long long col = c0 + 16 * cb;
                    if (row_ok && col <= row) {
                        float *p = A + row * ld + col;
#pragma unroll
                        for (int g = 0; g < 4; g++) {
                            const long long cg = col + 4 * g;
                            if (cg + 3 <= row && cg + 3 < n) {
                                float4 o = cur[cb * 4 + g];
                                o.x -= us * __uint_as_float(v[4 * g]);
                                o.y -= us * __uint_as_float(v[4 * g + 1]);
                                o.z -= us * __uint_as_float(v[4 * g + 2]);
                                o.w -= us * __uint_as_float(v[4 * g + 3]);
                                *reinterpret_cast<float4 *>(p + 4 * g) = o;
                            } else {
#pragma unroll
                                for (int j = 0; j < 4; j++)
                                    if (cg + j <= row && cg + j < n) p[4 * g + j] -= us * __uint_as_float(v[4 * g + j]);
                            }
                        }
                    }
                }
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                mbar_arrive(&acc_empty[a]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
    if (threadIdx.x == 0 && *abort == 1) atomicOr(flags, FLAG_LOOKBACK_TIMEOUT);
}

// ---- the same update with the old values of A moved by TMA ----------------------------
// k_update_tc's epilogue reads and writes A row by row: every warp access
// touches 32 rows, so L1TEX handles 32 sectors a request and becomes the busiest
// unit of the SM, which also slows the operand TMA that passes through it.  Here
// A moves in 128-row x 32-column chunks (16 KB, one 128-byte swizzle row per
// tile row) through a ring of 4 shared-memory slots:
//   warp 2 (one lane)  C mover: TMA-loads chunk g into slot g % 4 once the slot's
//                      previous chunk is done, and TMA-stores that chunk back
//                      (bulk async-group; its shared-memory reads finish before
//                      the slot is refilled);
//   warps 3-6          epilogue: per chunk, tcgen05.ld of 32 accumulator columns
//                      of their TMEM lanes, old value from the slot (the
//                      swizzled row of the thread's tile row), new value back
//                      into the slot, proxy fence, arrive on the slot's "done".
// Chunks wholly right of column n are neither loaded nor stored.
// The store writes whole chunks: entries above the diagonal of the trailing
// matrix get (old - acc) as well.  The factorization reads only the lower
// triangle of A (diagonal factor, panels, updates, solves), so they are never
// used; rows and columns past n are neither written nor read (TMA clips them).
// Three operand stages (144 KB) and the four slots (64 KB) fit one SM.
constexpr int C_SLOTS = 4;
constexpr int C_CHUNK = TILE * 128;  // 16 KB: 128 rows x 32 FP32
constexpr int TMA_EPI_STAGES = 3;
constexpr int THREADS_TMA = 7 * 32;
template <int MODE>
__global__ void __launch_bounds__(THREADS_TMA, 1)
    k_update_tc_tma(const __grid_constant__ CUtensorMap mL, const __grid_constant__ CUtensorMap mW,
                    const __grid_constant__ CUtensorMap mC, int n, int P1, long long ntiles, int nchunk,
                    int colblocks, const float *unscale, unsigned long long *flags) {
    static_assert(MODE == MODE_TF32 || MODE == MODE_F16, "single-product modes only");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<size_t>(smem_raw) + 1023) & ~size_t(1023));
    constexpr int STAGES = TMA_EPI_STAGES;
    constexpr int KCE = kc_of(MODE);
    constexpr unsigned STAGE_BYTES = CHUNK_L + CHUNK_W;
    unsigned char *cslot = base + STAGES * STAGE_BYTES;
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(cslot + C_SLOTS * C_CHUNK);
    unsigned long long *full = bars, *empty = bars + STAGES, *acc_full = bars + 2 * STAGES,
                       *acc_empty = bars + 2 * STAGES + 2, *drain = bars + 2 * STAGES + 4,
                       *c_full = bars + 2 * STAGES + 5, *c_done = c_full + C_SLOTS;
    unsigned *tmem_slot = reinterpret_cast<unsigned *>(c_done + C_SLOTS);
    volatile int *abort = reinterpret_cast<volatile int *>(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], 4 * 32);
        }
        mbar_init(drain, 1);
        for (int s = 0; s < C_SLOTS; s++) {
            mbar_init(&c_full[s], 1);
            mbar_init(&c_done[s], 4 * 32);
        }
        *abort = (*(volatile unsigned long long *)flags & FLAG_LOOKBACK_TIMEOUT) ? 2 : 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(saddr(tmem_slot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = *tmem_slot;

    if (*abort == 0) {
        if (warp == 0 && lane == 0) {
            // ---- operand producer ----
            long long it = 0;
            bool ok = true;
            for (long long t = blockIdx.x; ok && t < ntiles; t += gridDim.x) {
                int bi, bj;
                tile_of(t, colblocks, bi, bj);
                for (int kc = 0; kc < nchunk; kc++, it++) {
                    const int s = (int)(it % STAGES);
                    const long long u = it / STAGES;
                    if (u > 0 && !mbar_wait(&empty[s], (unsigned)((u - 1) & 1), abort)) {
                        ok = false;
                        break;
                    }
                    unsigned char *st = base + s * STAGE_BYTES;
                    mbar_expect_tx(&full[s], STAGE_BYTES);
                    tma_load(st, &mL, kc * KCE, bi * TILE, &full[s]);
                    tma_load(st + CHUNK_L, &mW, kc * KCE, bj * TILE_N, &full[s]);
                }
            }
            for (long long k = it - STAGES; k < it; k++) {
                if (k < 0) continue;
                const int s = (int)(k % STAGES);
                long long spins = 0;
                while (!mbar_try(&full[s], (unsigned)((k / STAGES) & 1)) && ++spins < SPIN_LIMIT) {
                }
            }
        } else if (warp == 1 && lane == 0) {
            // ---- MMA issuer ----
            long long it = 0, lt = 0;
            bool ok = true;
            for (long long t = blockIdx.x; ok && t < ntiles; t += gridDim.x, lt++) {
                const int a = (int)(lt & 1);
                const long long v = lt >> 1;
                if (v > 0 && !mbar_wait(&acc_empty[a], (unsigned)((v - 1) & 1), abort)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const unsigned d = tmem + (unsigned)(a * TILE_N);
                for (int kc = 0; kc < nchunk; kc++, it++) {
                    const int s = (int)(it % STAGES);
                    if (!mbar_wait(&full[s], (unsigned)((it / STAGES) & 1), abort)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const unsigned char *st = base + s * STAGE_BYTES;
                    const unsigned long long dl = smem_desc(saddr(st)), dw = smem_desc(saddr(st + CHUNK_L));
#pragma unroll
                    for (int kk = 0; kk < 4; kk++) {
                        const unsigned accum = (kc > 0 || kk > 0) ? 1u : 0u;
                        if (MODE == MODE_F16)
                            mma_f16(d, dl + 2 * kk, dw + 2 * kk, accum);
                        else
                            mma_tf32(d, dl + 2 * kk, dw + 2 * kk, accum);
                    }
                    mma_commit(&empty[s]);
                }
                if (!ok) break;
                mma_commit(&acc_full[a]);
            }
            mma_commit(drain);
            long long spins = 0;
            while (!mbar_try(drain, 0) && ++spins < SPIN_LIMIT) {
            }
        } else if (warp == 2 && lane == 0) {
            // ---- C mover ----
            int xs[C_SLOTS], ys[C_SLOTS];
            long long g = 0;
            bool ok = true;
            for (long long t = blockIdx.x; ok && t < ntiles; t += gridDim.x) {
                int bi, bj;
                tile_of(t, colblocks, bi, bj);
                for (int c = 0; c < TILE_N / 32; c++, g++) {
                    const int s = (int)(g % C_SLOTS);
                    const long long u = g / C_SLOTS;
                    if (u > 0) {  // the slot's previous chunk: done by the epilogue, stored, read out
                        if (!mbar_wait(&c_done[s], (unsigned)((u - 1) & 1), abort)) {
                            ok = false;
                            break;
                        }
                        if (xs[s] < n) {
                            tma_store(&mC, xs[s], ys[s], cslot + s * C_CHUNK);
                            bulk_commit();
                            bulk_wait_read0();
                        }
                    }
                    xs[s] = P1 + bj * TILE_N + 32 * c;
                    ys[s] = P1 + bi * TILE;
                    if (xs[s] < n) {
                        mbar_expect_tx(&c_full[s], C_CHUNK);
                        tma_load(cslot + s * C_CHUNK, &mC, xs[s], ys[s], &c_full[s]);
                    } else {  // a chunk wholly right of column n: nothing to move, the epilogue runs on
                        mbar_arrive(&c_full[s]);
                    }
                }
            }
            // the ring's last chunks: stored once done; loads of an aborted run landed
            for (long long k = g - C_SLOTS; k < g; k++) {
                if (k < 0) continue;
                const int s = (int)(k % C_SLOTS);
                if (ok && mbar_wait(&c_done[s], (unsigned)((k / C_SLOTS) & 1), abort)) {
                    if (xs[s] < n) {
                        tma_store(&mC, xs[s], ys[s], cslot + s * C_CHUNK);
                        bulk_commit();
                    }
                } else {
                    ok = false;
                    long long spins = 0;
                    while (!mbar_try(&c_full[s], (unsigned)((k / C_SLOTS) & 1)) && ++spins < SPIN_LIMIT) {
                    }
                }
            }
            bulk_wait0();
        } else if (warp >= 3) {
            // ---- epilogue: TMEM lanes 32*(warp%4) .. +31 are this warp's tile rows ----
            const int q = warp & 3;
            const int r = q * 32 + lane;
            const float us = MODE == MODE_F16 ? *unscale : 1.0f;  // a power of two: the products stay exact
            long long lt = 0, g = 0;
            bool ok = true;
            for (long long t = blockIdx.x; ok && t < ntiles; t += gridDim.x, lt++) {
                const int a = (int)(lt & 1);
                int w = 1;
                if (lane == 0) w = mbar_wait(&acc_full[a], (unsigned)((lt >> 1) & 1), abort);
                if (!__shfl_sync(0xffffffffu, w, 0)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const unsigned taddr = tmem + (unsigned)(a * TILE_N) + ((unsigned)(q * 32) << 16);
                for (int c = 0; c < TILE_N / 32; c++, g++) {
                    const int s = (int)(g % C_SLOTS);
                    int wc = 1;
                    if (lane == 0) wc = mbar_wait(&c_full[s], (unsigned)((g / C_SLOTS) & 1), abort);
                    if (!__shfl_sync(0xffffffffu, wc, 0)) {
                        ok = false;
                        break;
                    }
                    unsigned v[32];
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                          "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                          "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                          "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                        : "r"(taddr + 32 * c));
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    // row r of the slot: 128 bytes, 16-byte unit j stored at j ^ (r % 8) (128-byte swizzle)
                    unsigned char *rowp = cslot + s * C_CHUNK + r * 128;
#pragma unroll
                    for (int j = 0; j < 8; j++) {
                        float4 *p = reinterpret_cast<float4 *>(rowp + ((j ^ (r & 7)) << 4));
                        float4 o = *p;
                        o.x -= us * __uint_as_float(v[4 * j]);
                        o.y -= us * __uint_as_float(v[4 * j + 1]);
                        o.z -= us * __uint_as_float(v[4 * j + 2]);
                        o.w -= us * __uint_as_float(v[4 * j + 3]);
                        *p = o;
                    }
                    fence_proxy_async();
                    mbar_arrive(&c_done[s]);
                }
                if (!ok) break;
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                mbar_arrive(&acc_empty[a]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
    if (threadIdx.x == 0 && *abort == 1) atomicOr(flags, FLAG_LOOKBACK_TIMEOUT);
}
// stages, C slots, barriers, TMEM slot, abort flag + 1024-byte alignment slack
constexpr size_t smem_bytes_tma() {
    return (size_t)TMA_EPI_STAGES * (CHUNK_L + CHUNK_W) + (size_t)C_SLOTS * C_CHUNK + 256 + 1024;
}

// operand stages + barriers, TMEM slot, abort flag + 1024-byte alignment slack
constexpr size_t smem_bytes(int mode) {
    return (size_t)stages(mode) * (mode == MODE_TF32X3 ? 2 * (CHUNK_L + CHUNK_W) : CHUNK_L + CHUNK_W) + 256 + 1024;
}

}  // namespace tc
}  // namespace mp
