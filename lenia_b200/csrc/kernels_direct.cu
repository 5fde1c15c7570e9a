// Direct convolution of the growth stage on the fifth-generation tensor cores
// (tcgen05, sm_100a): BF16 products, or split-precision BF16x3 products, with
// FP32 accumulation in tensor memory.
//
// The reference convolves every kernel with its source channel by FFT on the
// torus (lenia.cpp:435-491, init_kernel lenia.cpp:215-257):
//
//   U_k(p) = sum_r K_k(r) A_c0(p - r),  r in the kernel grid's offsets.
//
// Here the same periodic sum runs in the spatial domain.  With the taps
// T_k(dz, dy, dx) = K_k(-dx, -dy, -dz),
//
//   U_k[z, y, x] = sum_{dz, dy} sum_dx T_k(dz, dy, dx) A[z + dz, y + dy, x + dx]
//
// and each (dz, dy) term is a banded Toeplitz product along x.  One tile
// computes 128 output x (the MMA's M) by 128 output rows (its N; a row is a
// (z, y) pair of the padded grid below) for up to four kernels of one source
// channel, each kernel in its own 128-column FP32 accumulator in tensor
// memory.  For every (dz, dy) with a tap:
//   A operand  the band of T_k(dz, dy, .) over a window of Kw input x.  Output
//              x is reversed along M (row m holds x = 127 - m), so the 8x8 core
//              matrix at (m-group q, k-group j) depends on q + j only: the
//              operand is a strip of Kw/8 + 15 core matrices of 128 bytes, read
//              with leading and stride byte offsets of 128;
//   B operand  the window of the input rows y + dy of plane z + dz, taken from
//              a tile of 128 + 2R rows by Kw x that TMA loads once per dz (each
//              dy is a 16-byte row offset into it).
// BF16X3 splits both factors as hi + lo (lo = bf16(v - hi)) and sums
// T_hi A_hi + T_lo A_hi (a pass over the high input parts) + T_hi A_lo (a
// pass over the low parts).
//
// Input layout: P[part][c][zp][yp][xp] bf16, the grid padded periodically by R
// cells on each side of every axis (zp = z + R, yp = y + R, xp = x + R; the
// x extent rounded up to 8).  Output rows of a tile are consecutive padded
// rows r = zp Hp + yp, either running on across planes (rows in the y
// padding are computed and dropped) or, when that needs fewer tiles, 128
// rows y0..y0+127 of one plane.
//
// The tensor cores' accumulation adds each MMA's products into the FP32
// accumulator with a rounding bias that grows with the number of MMAs per
// output.  BF16X3 therefore drains the accumulators after every dz-run into
// U with round-to-nearest FP32 adds (each run's partial sum starts a fresh
// accumulation); BF16, whose error is set by the BF16 rounding of its
// inputs, drains once.
//
// Roles in a block of six warps: warps 0-3 drain the accumulators (warp w
// reads TMEM lanes 32w..32w+31 with tcgen05.ld) and write U; lane 0 of warp 4
// issues the copies (TMA for the input tiles, bulk copies for the strips);
// lane 0 of warp 5 issues the MMAs.  Every wait is bounded: on a timeout the
// block records LENIA's timeout bit in the error word, waits (bounded) for
// its copies in flight, frees its tensor memory and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "direct_conv.h"
#include "growth_common.cuh"
#include "tma.cuh"

namespace lenia {

namespace {

constexpr int kTileX = 128;          // output x per tile: the MMA's M
constexpr int kTileRows = 128;       // output rows per tile: the MMA's N
constexpr int kSlots = 4;            // kernels per tile: 4 accumulators of 128 columns
constexpr int kStripStagesMax = 8;   // strip pipeline depth limit
constexpr int kEpilogueWarps = 4;    // warps 0-3 drain TMEM lane quadrants 0-3
constexpr int kThreads = 32 * (kEpilogueWarps + 2);  // + the copy warp and the MMA warp
constexpr int kMaxR = 64;            // 128 + 2R rows must fit one TMA box (<= 256)
constexpr size_t kSmemLimit = 227 * 1024;
constexpr size_t kSmemHeader = 1024;  // barriers and the tensor-memory address
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s per wait
constexpr unsigned kWaitPolls = 1u << 30;

// Instruction descriptor of tcgen05.mma kind::f16: D FP32 (bits 4-5 = 1), A
// and B BF16 (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0),
// N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTileRows >> 3) << 17) |
                            ((uint32_t)(kTileX >> 4) << 24);

struct DirPair {
    short dz, dy;
    unsigned char jlo, jhi;  // K steps (16 x each) that meet the band
    unsigned char mask;      // kernels of the group with taps on this row
    unsigned char pad;
    int strip0;              // first strip of this pair in the strip tables
};

struct DirGroup {
    int src, nk;
    int kidx[kSlots];
    int pair0, npairs;
};

struct DirLaunch {
    int W, H, D, C, R, Hp, rows_s, Kw, x3, ns;
    int seg_every;        // dz-runs between accumulator drains (0: one drain)
    int nby;              // tiles per plane (0: tiles run on across planes)
    long long N;
    unsigned data_bytes;  // shared-memory bytes of one input tile slot
    unsigned data_tx;     // bytes TMA delivers into it
    unsigned strip_bytes; // bytes of one strip (S core matrices)
    unsigned stage_bytes; // bytes of one strip stage
    const DirGroup *groups;
    const DirPair *pairs;
    const unsigned char *strips_hi, *strips_lo;
    float *U;
    int *err;
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for phase `parity` of the barrier; false after kWaitNs or kWaitPolls.
__device__ bool wait_phase(uint64_t *bar, unsigned parity)
{
    const uint32_t a = smem_addr(bar);
    unsigned long long t0 = 0;
    for (unsigned i = 0; i < kWaitPolls; i++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 255u) == 0) {
            const unsigned long long t = global_ns();
            if (i == 0) t0 = t;
            else if (t - t0 > kWaitNs) return false;
        }
    }
    return false;
}

// Shared-memory matrix descriptor, no swizzle: start address, leading byte
// offset (between core matrices along K), stride byte offset (between core
// matrices along M or N), all in 16-byte units; bit 46 = descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

// The barrier completes one arrival when every MMA issued so far by this
// thread has finished.
__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// 32 consecutive accumulator columns of this warp's 32 lanes, one lane per
// thread, waited for in the same statement.
__device__ __forceinline__ void tmem_load32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ bool aborted(const int *err) { return (*(volatile const int *)err & 2) != 0; }

// Whether the accumulators are drained after dz-run `r` (counted over both
// passes) of `total` runs: every `every` runs (0: only after the last).
__device__ __forceinline__ bool seg_end(int r, int total, int every)
{
    return r == total - 1 || (every > 0 && (r + 1) % every == 0);
}

__global__ void __launch_bounds__(kThreads, 1) k_direct(DirLaunch p, const __grid_constant__ CUtensorMap tm)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t *full_d = (uint64_t *)smem;              // [2]
    uint64_t *empty_d = full_d + 2;                   // [2]
    uint64_t *full_s = empty_d + 2;                   // [kStripStagesMax]
    uint64_t *empty_s = full_s + kStripStagesMax;     // [kStripStagesMax]
    uint64_t *seg_full = empty_s + kStripStagesMax;   // accumulators ready to drain
    uint64_t *seg_empty = seg_full + 1;               // accumulators drained
    uint32_t *tmem_slot = (uint32_t *)(smem + 512);
    int *s_bad = (int *)(smem + 516);
    unsigned char *data = smem + kSmemHeader;
    unsigned char *stages = data + 2 * (size_t)p.data_bytes;

    const DirGroup g = p.groups[blockIdx.z];
    const int tile_x = blockIdx.y * kTileX;
    // padded row of the tile's first output row
    const long long row0 =
        p.nby > 0 ? (long long)(blockIdx.x / p.nby + p.R) * p.Hp + p.R + (long long)(blockIdx.x % p.nby) * kTileRows
                  : (long long)p.R * p.Hp + (long long)blockIdx.x * kTileRows;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned ncols = g.nk <= 1 ? 128u : g.nk <= 2 ? 256u : 512u;
    const int npass = p.x3 ? 2 : 1;
    const int runs = npass * (2 * p.R + 1);  // every dz in [-R, R] has a run
    const int nseg = p.seg_every > 0 ? (runs + p.seg_every - 1) / p.seg_every : 1;

    if (threadIdx.x == 0) {
        for (int i = 0; i < 2; i++) {
            mbar_init(&full_d[i], 1);
            mbar_init(&empty_d[i], 1);
        }
        for (int i = 0; i < p.ns; i++) {
            mbar_init(&full_s[i], 1);
            mbar_init(&empty_s[i], 1);
        }
        mbar_init(seg_full, 1);
        mbar_init(seg_empty, kEpilogueWarps);
        *s_bad = 0;
        mbar_init_fence();
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(tmem_slot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    int bad = 0;
    if (warp == kEpilogueWarps && lane == 0) {
        // ---------------------------------------------------------- copies
        unsigned dfill[2] = {0, 0}, sfill[kStripStagesMax];
        for (int i = 0; i < kStripStagesMax; i++) sfill[i] = 0;
        int ds = 0, ss = 0;
        for (int pass = 0; pass < npass && !bad; pass++) {
            int e = 0;
            while (e < g.npairs && !bad) {
                if (aborted(p.err)) {
                    bad = 1;
                    break;
                }
                const int dz = p.pairs[g.pair0 + e].dz;
                if (dfill[ds] && !wait_phase(&empty_d[ds], (dfill[ds] - 1) & 1u)) {
                    bad = 1;
                    break;
                }
                mbar_arrive_expect_tx(&full_d[ds], p.data_tx);
                const int y = (int)(row0 + (long long)dz * p.Hp - p.R);
                const int zc = pass * p.C + g.src;
                unsigned char *dst = data + (size_t)ds * p.data_bytes;
                for (int j = 0; j < p.Kw / 8; j++)
                    tma_load_3d(dst + (size_t)j * p.rows_s * 16, &tm, tile_x + 8 * j, y, zc, &full_d[ds]);
                dfill[ds]++;
                for (; e < g.npairs && p.pairs[g.pair0 + e].dz == dz; e++) {
                    const DirPair pr = p.pairs[g.pair0 + e];
                    if (sfill[ss] && !wait_phase(&empty_s[ss], (sfill[ss] - 1) & 1u)) {
                        bad = 1;
                        break;
                    }
                    const unsigned nb = (unsigned)g.nk * p.strip_bytes;
                    const bool two = p.x3 && pass == 0;
                    mbar_arrive_expect_tx(&full_s[ss], two ? 2 * nb : nb);
                    unsigned char *sd = stages + (size_t)ss * p.stage_bytes;
                    const size_t off = (size_t)pr.strip0 * p.strip_bytes;
                    bulk_load(sd, p.strips_hi + off, nb, &full_s[ss]);
                    if (two) bulk_load(sd + nb, p.strips_lo + off, nb, &full_s[ss]);
                    sfill[ss]++;
                    ss = ss + 1 == p.ns ? 0 : ss + 1;
                }
                ds ^= 1;
            }
        }
        if (bad) {
            // copies still in flight land before the block leaves
            for (int i = 0; i < 2; i++)
                if (dfill[i]) wait_phase(&full_d[i], (dfill[i] - 1) & 1u);
            for (int i = 0; i < p.ns; i++)
                if (sfill[i]) wait_phase(&full_s[i], (sfill[i] - 1) & 1u);
        }
    } else if (warp == kEpilogueWarps + 1 && lane == 0) {
        // ------------------------------------------------------------ MMAs
        unsigned dfill[2] = {0, 0}, sfill[kStripStagesMax];
        for (int i = 0; i < kStripStagesMax; i++) sfill[i] = 0;
        int ds = 0, ss = 0, run = 0, seg = 0;
        unsigned started = 0;  // accumulators written in the current segment
        const uint32_t data_s = smem_addr(data), stage_s = smem_addr(stages);
        const uint32_t lbo_d = (uint32_t)p.rows_s * 16;
        for (int pass = 0; pass < npass && !bad; pass++) {
            int e = 0;
            while (e < g.npairs && !bad) {
                if (aborted(p.err)) {
                    bad = 1;
                    break;
                }
                const int dz = p.pairs[g.pair0 + e].dz;
                if (started == 0 && seg > 0 && !wait_phase(seg_empty, (unsigned)(seg - 1) & 1u)) {
                    bad = 1;
                    break;
                }
                if (!wait_phase(&full_d[ds], dfill[ds] & 1u)) {
                    bad = 1;
                    break;
                }
                dfill[ds]++;
                tc_fence_after();
                for (; e < g.npairs && p.pairs[g.pair0 + e].dz == dz; e++) {
                    const DirPair pr = p.pairs[g.pair0 + e];
                    if (!wait_phase(&full_s[ss], sfill[ss] & 1u)) {
                        bad = 1;
                        break;
                    }
                    sfill[ss]++;
                    tc_fence_after();
                    const uint32_t sb = stage_s + (uint32_t)ss * p.stage_bytes;
                    const uint32_t db = data_s + (uint32_t)ds * p.data_bytes + (uint32_t)(pr.dy + p.R) * 16;
                    const uint32_t nb = (uint32_t)g.nk * p.strip_bytes;
                    for (int i = 0; i < g.nk; i++) {
                        if (!((pr.mask >> i) & 1)) continue;
                        const uint32_t td = tmem + (uint32_t)i * 128;
                        const uint32_t sa = sb + (uint32_t)i * p.strip_bytes;
                        for (int t = pr.jlo; t < pr.jhi; t++) {
                            const uint64_t bdesc = smem_desc(db + (uint32_t)t * 2 * lbo_d, lbo_d, 128);
                            mma_bf16(td, smem_desc(sa + (uint32_t)t * 256, 128, 128), bdesc, (started >> i) & 1u);
                            started |= 1u << i;
                            if (p.x3 && pass == 0)
                                mma_bf16(td, smem_desc(sa + nb + (uint32_t)t * 256, 128, 128), bdesc, 1u);
                        }
                    }
                    mma_commit(&empty_s[ss]);
                    ss = ss + 1 == p.ns ? 0 : ss + 1;
                }
                mma_commit(&empty_d[ds]);
                ds ^= 1;
                if (seg_end(run, runs, p.seg_every)) {
                    // the segment's sums are complete once its MMAs finish
                    mma_commit(seg_full);
                    seg++;
                    started = 0;
                }
                run++;
            }
        }
        if (bad) {
            atomicOr(s_bad, 1);
            mma_commit(seg_full);  // lets the drains end early
        }
    } else if (warp < kEpilogueWarps) {
        // ------------------------------------- drains: TMEM -> U, FP32 adds
        const int m = warp * 32 + lane;
        const int x = tile_x + (kTileX - 1) - m;
        for (int sgi = 0; sgi < nseg; sgi++) {
            if (!wait_phase(seg_full, (unsigned)sgi & 1u)) {
                bad = 1;
                break;
            }
            __syncwarp();
            tc_fence_after();
            if (*(volatile int *)s_bad) {
                bad = 1;
                break;
            }
            for (int i = 0; i < g.nk; i++) {
                float *Uk = p.U + (long long)g.kidx[i] * p.N;
                for (int c = 0; c < kTileRows / 32; c++) {
                    uint32_t v[32];
                    tmem_load32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(i * 128 + c * 32), v);
                    const long long row = row0 + c * 32;
                    const int zp0 = (int)(row / p.Hp);
                    const int yp0 = (int)(row - (long long)zp0 * p.Hp);
                    long long off[32];
                    int zp = zp0, yp = yp0;
#pragma unroll
                    for (int n = 0; n < 32; n++) {
                        const bool ok = x < p.W && zp < p.R + p.D && yp >= p.R && yp < p.R + p.H;
                        off[n] = ok ? ((long long)(zp - p.R) * p.H + (yp - p.R)) * p.W + x : -1;
                        if (++yp == p.Hp) {
                            yp = 0;
                            zp++;
                        }
                    }
                    if (sgi == 0) {
#pragma unroll
                        for (int n = 0; n < 32; n++)
                            if (off[n] >= 0) Uk[off[n]] = __uint_as_float(v[n]);
                    } else {
                        float old[32];
#pragma unroll
                        for (int n = 0; n < 32; n++) old[n] = off[n] >= 0 ? Uk[off[n]] : 0.0f;
#pragma unroll
                        for (int n = 0; n < 32; n++)
                            if (off[n] >= 0) Uk[off[n]] = old[n] + __uint_as_float(v[n]);
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(seg_empty);
        }
    }
    if (bad) atomicOr(s_bad, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(ncols) : "memory");
    }
    if (threadIdx.x == 0 && *s_bad) atomicOr(p.err, 2);
}

// Periodically padded BF16 copy of the grid channels, split as hi (part 0)
// and lo = bf16(v - hi) (part 1, BF16X3 only); two x per thread.
__global__ void k_pad_split(const float *__restrict__ A, __nv_bfloat16 *__restrict__ P, int W, int H, int D, int C,
                            int R, int Hp, int Dp, int Wp, int x3)
{
    const long long per_c = (long long)Dp * Hp * (Wp / 2);
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= per_c * C) return;
    const int c = (int)(i / per_c);
    long long q = i - (long long)c * per_c;
    const int xp = (int)(q % (Wp / 2)) * 2;
    q /= (Wp / 2);
    const int yp = (int)(q % Hp);
    const int zp = (int)(q / Hp);
    const int y = ((yp - R) % H + H) % H, z = ((zp - R) % D + D) % D;
    const int x0 = ((xp - R) % W + W) % W, x1 = ((xp + 1 - R) % W + W) % W;
    const float *row = A + ((long long)c * D + z) * H * W + (long long)y * W;
    const float a0 = row[x0], a1 = row[x1];
    const __nv_bfloat16 h0 = __float2bfloat16_rn(a0), h1 = __float2bfloat16_rn(a1);
    const long long o = (((long long)c * Dp + zp) * Hp + yp) * Wp + xp;
    __nv_bfloat162 hv;
    hv.x = h0;
    hv.y = h1;
    *(__nv_bfloat162 *)(P + o) = hv;
    if (x3) {
        __nv_bfloat162 lv;
        lv.x = __float2bfloat16_rn(a0 - __bfloat162float(h0));
        lv.y = __float2bfloat16_rn(a1 - __bfloat162float(h1));
        *(__nv_bfloat162 *)(P + (long long)C * Dp * Hp * Wp + o) = lv;
    }
}

// Strip of core matrices for (pair e, slot i): element (c, r, e8) at
// c*64 + r*8 + e8 holds T(dz, dy, 8c + e8 + r - (R + 127)); hi and lo parts.
// A tap exists only for offsets the kernel grid holds ([-n/2, n/2) per axis
// of extent n), so the sum equals the spectral path's circular convolution.
__global__ void k_build_strips(const float *__restrict__ grids, const DirPair *__restrict__ pairs,
                               const DirGroup *__restrict__ groups, const int *__restrict__ pair_group, int W, int H,
                               int D, long long N, int R, int S, __nv_bfloat16 *hi, __nv_bfloat16 *lo)
{
    const int e = blockIdx.x;
    const DirPair pr = pairs[e];
    const DirGroup &g = groups[pair_group[e]];
    const int slot = blockIdx.y;
    if (slot >= g.nk) return;
    const float *grid = grids + (long long)g.kidx[slot] * N;
    const long long base = ((long long)pr.strip0 + slot) * S * 64;
    for (int q = threadIdx.x; q < S * 64; q += blockDim.x) {
        const int c = q >> 6, r = (q >> 3) & 7, e8 = q & 7;
        const int dx = 8 * c + e8 + r - (R + 127);
        float v = 0.0f;
        const int ox = -dx, oy = -pr.dy, oz = -pr.dz;
        if (dx >= -R && dx <= R && ox >= -(W / 2) && ox < W - W / 2 && oy >= -(H / 2) && oy < H - H / 2 &&
            oz >= -(D / 2) && oz < D - D / 2) {
            const int gx = ox < 0 ? ox + W : ox, gy = oy < 0 ? oy + H : oy, gz = oz < 0 ? oz + D : oz;
            v = grid[((long long)gz * H + gy) * W + gx];
        }
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        hi[base + q] = h;
        lo[base + q] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
}

__global__ void k_count_taps(const float *__restrict__ grids, long long n, unsigned long long *count)
{
    unsigned long long c = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        c += grids[i] != 0.0f;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// The growth accumulation of mt_fft_step (lenia.cpp:501-538) and the early
// growth into BACK (lenia.cpp:542-592) from stored u_k, per cell, in kernel
// order (the same arithmetic as the spectral path's inverse-row epilogue).
// Four consecutive cells per thread (N is a multiple of 4), 16-byte loads
// and stores; each cell's sums still run over the kernels in order.
__device__ __forceinline__ float growth_value(const GrowthJobs &jobs, const float *__restrict__ lut_rows, int k,
                                              float u, int &bad)
{
    const int ui = (int)(u * 255);
    float l;
    if (jobs.exact_bell) {
        if (!(u == u)) bad = 1;
        l = bell_dev(u, jobs.m[k], jobs.s[k]);
    } else if (ui >= 0 && ui < 256) l = __ldg(lut_rows + k * 256 + ui);
    else {
        if (!(u == u)) bad = 1;
        l = lut_flat_dev((long long)jobs.lut_base[k] + ui);
    }
    return l;
}

// One channel at a time: its kernels' growth and u summed in kernel order
// (the additions of the all-channel form, so the fields are identical), then
// its H, U_SUM and BACK written; only one channel's sums are live.
// Five blocks of 256 per SM (48 registers, no spills).
__device__ __forceinline__ void growth_from_u_body(const Dims &d, const GrowthJobs &jobs, const ChannelOrder &ord,
                                                   const float *__restrict__ lut_rows, const float *__restrict__ U,
                                                   const float *__restrict__ A, float *__restrict__ Hout,
                                                   float *__restrict__ Uout, float *__restrict__ BACK, int *err_flag,
                                                   long long block)
{
    const long long i = (block * blockDim.x + threadIdx.x) * 4;
    if (i >= d.N) return;
    int bad = 0;
    // u of the next two kernels (in channel order) is loaded ahead of the
    // current one's growth
    const float4 *U4 = reinterpret_cast<const float4 *>(U + i);
    const long long kstride = d.N / 4;
    const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    // u_k is read once (evict-first loads), U_SUM is not read in the step
    // (evict-first store): L2 keeps H and BACK for the flow and transport
    float4 n1 = jobs.K > 0 ? __ldcs(U4 + (long long)ord.k[0] * kstride) : zero4;
    float4 n2 = jobs.K > 1 ? __ldcs(U4 + (long long)ord.k[1] * kstride) : zero4;
    int pos = 0;
    for (int c = 0; c < jobs.C; c++) {
        const long long o = (long long)c * d.N + i;
        const bool need_a = jobs.asymptotic[c] || jobs.growth_rt;
        const float4 a4 = need_a ? __ldg(reinterpret_cast<const float4 *>(A + o)) : zero4;
        float hacc[4] = {0.0f, 0.0f, 0.0f, 0.0f}, uacc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (; pos < jobs.K && jobs.c1[ord.k[pos]] == c; pos++) {
            const int k = ord.k[pos];
            const float4 u4 = n1;
            n1 = n2;
            if (pos + 2 < jobs.K) n2 = __ldcs(U4 + (long long)ord.k[pos + 2] * kstride);
            const float u[4] = {u4.x, u4.y, u4.z, u4.w};
            const float a[4] = {a4.x, a4.y, a4.z, a4.w};
            const float h = jobs.h[k];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float l = growth_value(jobs, lut_rows, k, u[j], bad);
                uacc[j] = uacc[j] + u[j];
                float g;
                if (jobs.asymptotic[c]) g = (l - a[j]) * h;
                else g = l * h;
                hacc[j] = hacc[j] + g;
            }
        }
        *reinterpret_cast<float4 *>(Hout + o) = make_float4(hacc[0], hacc[1], hacc[2], hacc[3]);
        __stcs(reinterpret_cast<float4 *>(Uout + o), make_float4(uacc[0], uacc[1], uacc[2], uacc[3]));
        // a NaN u indexes the table at 0 ((int)NaN is 0 here): test the sums
        if (!(isfinite(uacc[0]) && isfinite(uacc[1]) && isfinite(uacc[2]) && isfinite(uacc[3]))) bad = 1;
        if (jobs.growth_rt) {
            const float4 b = make_float4(early_growth(a4.x, hacc[0], jobs.timestep, jobs.soft_clip[c]),
                                         early_growth(a4.y, hacc[1], jobs.timestep, jobs.soft_clip[c]),
                                         early_growth(a4.z, hacc[2], jobs.timestep, jobs.soft_clip[c]),
                                         early_growth(a4.w, hacc[3], jobs.timestep, jobs.soft_clip[c]));
            *reinterpret_cast<float4 *>(BACK + o) = b;
        }
    }
    if (bad && err_flag) atomicOr(err_flag, 1);
}

#ifndef LENIA_GROWTH_U_MINB
#define LENIA_GROWTH_U_MINB 5
#endif
__global__ void __launch_bounds__(256, LENIA_GROWTH_U_MINB)
    k_growth_from_u(const __grid_constant__ Dims d, const __grid_constant__ GrowthJobs jobs,
                    const __grid_constant__ ChannelOrder ord, const float *__restrict__ lut_rows,
                    const float *__restrict__ U, const float *__restrict__ A, float *__restrict__ Hout,
                    float *__restrict__ Uout, float *__restrict__ BACK, int *err_flag)
{
    growth_from_u_body(d, jobs, ord, lut_rows, U, A, Hout, Uout, BACK, err_flag, blockIdx.x);
}

// The same over a batch of worlds: block b of the launch is block
// items[b].block of world items[b].world's own launch.
__global__ void __launch_bounds__(256, 5) k_growth_from_u_multi(const BatchWorldDev *__restrict__ ws,
                                                                const WorkItem *__restrict__ items)
{
    const WorkItem it = items[blockIdx.x];
    const BatchWorldDev &w = ws[it.world];
    growth_from_u_body(w.p.d, w.gj, w.ord, w.lut_rows, w.U, w.A, w.H, w.U_SUM, w.BACK, w.err, it.block);
}

int round_up(int v, int m) { return (v + m - 1) / m * m; }

}  // namespace

struct DirectConv {
    Dims d;
    int C = 0, K = 0, mode = 0;
    int R = 0, Hp = 0, Dp = 0, Wp = 0, rows_s = 0, Kw = 0, S = 0, ns = 0, nk_max = 0;
    size_t smem = 0;
    unsigned data_bytes = 0, data_tx = 0, strip_bytes = 0, stage_bytes = 0;
    int seg_every = 0;  // dz-runs per accumulator drain (0: one drain)
    int nby = 0;        // tiles per plane (0: tiles run on across planes)
    long long nb = 0;   // row tiles
    std::vector<DirGroup> groups;
    std::vector<DirPair> pairs;
    DirGroup *groups_dev = nullptr;
    DirPair *pairs_dev = nullptr;
    int *pair_group_dev = nullptr;
    __nv_bfloat16 *strips = nullptr;  // hi table, then lo table
    long long strip_count = 0;
    __nv_bfloat16 *P = nullptr;
    CUtensorMap tm;
    unsigned long long *tap_count_dev = nullptr;
    unsigned long long taps = 0;  // nonzero kernel taps over all kernels
    double issued = 0.0;          // tensor MACs per convolution (both parts counted)
};

void direct_destroy(DirectConv *dc)
{
    if (!dc) return;
    void *ps[] = {dc->groups_dev, dc->pairs_dev, dc->pair_group_dev, dc->strips, dc->P, dc->tap_count_dev};
    for (void *q : ps)
        if (q) cudaFree(q);
    delete dc;
}

// Plan for a world: tap radius, padded extents, kernel groups, the (dz, dy)
// rows each group visits (a conservative bound of the kernels' support,
// |r| < radius * r_a, with half a cell of margin; taps outside the support
// are zero in the strips) and the shared-memory split.
cudaError_t direct_create(const Dims &d, int C, const LeniaKernelParams *kernels, int K, int mode, DirectConv **out)
{
    *out = nullptr;
    if (mode != LENIA_CONV_DIRECT_BF16 && mode != LENIA_CONV_DIRECT_BF16X3) return cudaErrorInvalidValue;
    DirectConv *dc = new DirectConv();
    dc->d = d;
    dc->C = C;
    dc->K = K;
    dc->mode = mode;
    const int x3 = mode == LENIA_CONV_DIRECT_BF16X3;
    dc->seg_every = x3 ? 1 : 0;
    int R = 0;
    std::vector<float> ext(K);
    for (int k = 0; k < K; k++) {
        ext[k] = (float)kernels[k].radius * kernels[k].r_a;
        R = std::max(R, (int)ceilf(ext[k]));
    }
    R = std::min(R, std::max(d.W, std::max(d.H, d.D)) / 2);
    R = std::max(R, 1);
    if (R > kMaxR) {
        delete dc;
        return cudaErrorInvalidValue;
    }
    dc->R = R;
    dc->Hp = d.H + 2 * R;
    dc->Dp = d.D + 2 * R;
    dc->Wp = round_up(d.W + 2 * R, 8);
    dc->rows_s = round_up(kTileRows + 2 * R, 8);
    dc->Kw = round_up(kTileX + 2 * R, 16);
    dc->S = dc->Kw / 8 + kTileX / 8 - 1;
    // groups: kernels of one source channel, up to kSlots per group
    for (int c = 0; c < C; c++) {
        DirGroup g;
        memset(&g, 0, sizeof(g));
        g.src = c;
        for (int k = 0; k < K; k++) {
            if (kernels[k].c0 != c) continue;
            g.kidx[g.nk++] = k;
            if (g.nk == kSlots) {
                dc->groups.push_back(g);
                memset(&g, 0, sizeof(g));
                g.src = c;
            }
        }
        if (g.nk) dc->groups.push_back(g);
    }
    int strip0 = 0;
    const int nx = (d.W + kTileX - 1) / kTileX;
    // row tiles: across planes, or per plane when that takes fewer
    const long long nb_flat = ((long long)d.D * dc->Hp + kTileRows - 1) / kTileRows;
    const int nby = (d.H + kTileRows - 1) / kTileRows;
    dc->nby = (long long)d.D * nby < nb_flat ? nby : 0;
    dc->nb = dc->nby ? (long long)d.D * nby : nb_flat;
    const long long nb = dc->nb;
    std::vector<int> pair_group;
    for (size_t gi = 0; gi < dc->groups.size(); gi++) {
        DirGroup &g = dc->groups[gi];
        dc->nk_max = std::max(dc->nk_max, g.nk);
        g.pair0 = (int)dc->pairs.size();
        for (int dz = -R; dz <= R; dz++)
            for (int dy = -R; dy <= R; dy++) {
                int mask = 0, dxm = -1;
                for (int i = 0; i < g.nk; i++) {
                    const float lim = (ext[g.kidx[i]] + 0.5f) * (ext[g.kidx[i]] + 0.5f);
                    const float r2 = (float)(dy * dy + dz * dz);
                    // every dz has a run with every kernel of the group (its
                    // dy = 0 row), so each drain segment writes every
                    // accumulator
                    const bool centre = dy == 0;
                    if (r2 > lim && !centre) continue;
                    mask |= 1 << i;
                    const int m = r2 > lim ? 0 : std::min(R, (int)floorf(sqrtf(lim - r2)));
                    dxm = std::max(dxm, m);
                }
                if (!mask) continue;
                DirPair pr;
                pr.dz = (short)dz;
                pr.dy = (short)dy;
                pr.jlo = (unsigned char)((R - dxm) / 16);
                pr.jhi = (unsigned char)std::min(dc->Kw / 16, (kTileX - 1 + R + dxm) / 16 + 1);
                pr.mask = (unsigned char)mask;
                pr.pad = 0;
                pr.strip0 = strip0;
                strip0 += g.nk;
                dc->pairs.push_back(pr);
                pair_group.push_back((int)gi);
                int used = 0;
                for (int i = 0; i < g.nk; i++) used += (mask >> i) & 1;
                dc->issued += (double)used * (pr.jhi - pr.jlo) * kTileX * kTileRows * 16 * (x3 ? 3 : 1) * nx * nb;
            }
        g.npairs = (int)dc->pairs.size() - g.pair0;
    }
    dc->strip_count = strip0;
    dc->strip_bytes = (unsigned)dc->S * 128;
    dc->data_bytes = (unsigned)(dc->Kw / 8) * dc->rows_s * 16;
    dc->data_tx = (unsigned)(dc->Kw / 8) * (kTileRows + 2 * R) * 16;
    dc->stage_bytes = (unsigned)(x3 ? 2 : 1) * dc->nk_max * dc->strip_bytes;
    const size_t fixed = kSmemHeader + 2 * (size_t)dc->data_bytes;
    int ns = fixed < kSmemLimit && dc->stage_bytes ? (int)((kSmemLimit - fixed) / dc->stage_bytes) : 0;
    ns = std::min(ns, kStripStagesMax);
    if (ns < 2) {
        delete dc;
        return cudaErrorInvalidValue;
    }
    dc->ns = ns;
    // at least 116 KB so that one block (and one tensor-memory allocation)
    // is resident per SM
    dc->smem = std::max(fixed + (size_t)ns * dc->stage_bytes, (size_t)116 * 1024);

    cudaError_t e = cudaSuccess;
    const size_t pbytes = (size_t)2 * C * dc->Dp * dc->Hp * dc->Wp * sizeof(__nv_bfloat16);
    if ((e = cudaMalloc((void **)&dc->P, pbytes)) != cudaSuccess) goto fail;
    if ((e = cudaMemset(dc->P, 0, pbytes)) != cudaSuccess) goto fail;
    if ((e = cudaMalloc((void **)&dc->strips, (size_t)2 * dc->strip_count * dc->strip_bytes)) != cudaSuccess) goto fail;
    if ((e = cudaMalloc((void **)&dc->groups_dev, sizeof(DirGroup) * dc->groups.size())) != cudaSuccess) goto fail;
    if ((e = cudaMalloc((void **)&dc->pairs_dev, sizeof(DirPair) * dc->pairs.size())) != cudaSuccess) goto fail;
    if ((e = cudaMalloc((void **)&dc->pair_group_dev, sizeof(int) * pair_group.size())) != cudaSuccess) goto fail;
    if ((e = cudaMalloc((void **)&dc->tap_count_dev, sizeof(unsigned long long))) != cudaSuccess) goto fail;
    if ((e = cudaMemcpy(dc->groups_dev, dc->groups.data(), sizeof(DirGroup) * dc->groups.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess)
        goto fail;
    if ((e = cudaMemcpy(dc->pairs_dev, dc->pairs.data(), sizeof(DirPair) * dc->pairs.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess)
        goto fail;
    if ((e = cudaMemcpy(dc->pair_group_dev, pair_group.data(), sizeof(int) * pair_group.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess)
        goto fail;
    {
        const unsigned long long dims[3] = {(unsigned long long)dc->Wp, (unsigned long long)dc->Dp * dc->Hp,
                                            (unsigned long long)2 * C};
        const unsigned box[3] = {8u, (unsigned)(kTileRows + 2 * R), 1u};
        if ((e = encode_tensor_map_typed(&dc->tm, dc->P, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, 3, dims, box)) !=
            cudaSuccess)
            goto fail;
    }
    // the attribute is per function and shared by every plan: the limit
    // itself, so that plans of other worlds launch with their own sizes
    if ((e = cudaFuncSetAttribute(k_direct, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemLimit)) !=
        cudaSuccess)
        goto fail;
    *out = dc;
    return cudaSuccess;
fail:
    direct_destroy(dc);
    return e;
}

// Strips from the normalised kernel grids (K x N floats, the layout the
// spectral path transforms) and the count of nonzero taps.
cudaError_t direct_build(DirectConv *dc, const float *grids, cudaStream_t st)
{
    if (dc->pairs.empty()) return cudaSuccess;
    __nv_bfloat16 *hi = dc->strips, *lo = dc->strips + dc->strip_count * dc->S * 64;
    dim3 grid((unsigned)dc->pairs.size(), (unsigned)dc->nk_max);
    k_build_strips<<<grid, 256, 0, st>>>(grids, dc->pairs_dev, dc->groups_dev, dc->pair_group_dev, dc->d.W, dc->d.H,
                                         dc->d.D, dc->d.N, dc->R, dc->S, hi, lo);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(dc->tap_count_dev, 0, sizeof(unsigned long long), st)) != cudaSuccess) return e;
    k_count_taps<<<592, 256, 0, st>>>(grids, (long long)dc->K * dc->d.N, dc->tap_count_dev);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(&dc->taps, dc->tap_count_dev, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
        return e;
    return cudaStreamSynchronize(st);
}

cudaError_t direct_pad(DirectConv *dc, const float *A, cudaStream_t st)
{
    const long long n = (long long)dc->C * dc->Dp * dc->Hp * (dc->Wp / 2);
    k_pad_split<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(A, dc->P, dc->d.W, dc->d.H, dc->d.D, dc->C, dc->R, dc->Hp,
                                                              dc->Dp, dc->Wp, dc->mode == LENIA_CONV_DIRECT_BF16X3);
    return cudaGetLastError();
}

cudaError_t direct_convolve(DirectConv *dc, float *U, int *err, cudaStream_t st)
{
    if (dc->groups.empty()) return cudaSuccess;
    DirLaunch p;
    memset(&p, 0, sizeof(p));
    p.W = dc->d.W;
    p.H = dc->d.H;
    p.D = dc->d.D;
    p.C = dc->C;
    p.R = dc->R;
    p.Hp = dc->Hp;
    p.rows_s = dc->rows_s;
    p.Kw = dc->Kw;
    p.x3 = dc->mode == LENIA_CONV_DIRECT_BF16X3;
    p.ns = dc->ns;
    p.seg_every = dc->seg_every;
    p.nby = dc->nby;
    p.N = dc->d.N;
    p.data_bytes = dc->data_bytes;
    p.data_tx = dc->data_tx;
    p.strip_bytes = dc->strip_bytes;
    p.stage_bytes = dc->stage_bytes;
    p.groups = dc->groups_dev;
    p.pairs = dc->pairs_dev;
    p.strips_hi = (const unsigned char *)dc->strips;
    p.strips_lo = (const unsigned char *)(dc->strips + dc->strip_count * dc->S * 64);
    p.U = U;
    p.err = err;
    const long long nb = dc->nb;
    dim3 grid((unsigned)nb, (unsigned)((dc->d.W + kTileX - 1) / kTileX), (unsigned)dc->groups.size());
    k_direct<<<grid, kThreads, dc->smem, st>>>(p, dc->tm);
    return cudaGetLastError();
}

void direct_counts(const DirectConv *dc, double *issued_macs, double *useful_macs)
{
    const double parts = dc->mode == LENIA_CONV_DIRECT_BF16X3 ? 3.0 : 1.0;
    if (issued_macs) *issued_macs = dc->issued;
    if (useful_macs) *useful_macs = (double)dc->taps * (double)dc->d.N * parts;
}

size_t direct_smem(const DirectConv *dc) { return dc->smem; }
int direct_stages(const DirectConv *dc) { return dc->ns; }
int direct_radius(const DirectConv *dc) { return dc->R; }

// Stable grouping of the kernels by target channel; kernels aimed past the
// last channel go last and, as in the all-channel form, reach no output.
ChannelOrder channel_order(const GrowthJobs &jobs)
{
    ChannelOrder ord{};
    int n = 0;
    for (int c = 0; c <= kMaxChannels; c++)
        for (int k = 0; k < jobs.K; k++) {
            const int t = jobs.c1[k] >= 0 && jobs.c1[k] < kMaxChannels ? jobs.c1[k] : kMaxChannels;
            if (t == c) ord.k[n++] = k;
        }
    return ord;
}

// 256 threads of four cells each (N is a multiple of 4: the width is).
int growth_from_u_blocks(const Dims &d) { return (int)((d.N / 4 + 255) / 256); }

cudaError_t launch_growth_from_u(const Dims &d, const GrowthJobs &jobs, const float *lut_rows, const float *U,
                                 const float *A, float *H, float *U_SUM, float *BACK, int *err_flag, cudaStream_t st)
{
    const ChannelOrder ord = channel_order(jobs);
    k_growth_from_u<<<(unsigned)growth_from_u_blocks(d), 256, 0, st>>>(d, jobs, ord, lut_rows, U, A, H, U_SUM, BACK,
                                                                       err_flag);
    return cudaGetLastError();
}

cudaError_t launch_growth_from_u_multi(const BatchWorldDev *ws, const WorkItem *items, int n_items, cudaStream_t st)
{
    if (n_items == 0) return cudaSuccess;
    k_growth_from_u_multi<<<(unsigned)n_items, 256, 0, st>>>(ws, items);
    return cudaGetLastError();
}

}  // namespace lenia
