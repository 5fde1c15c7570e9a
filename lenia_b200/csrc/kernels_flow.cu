// Flow stage of the 3D Flow Lenia step, fused into one kernel: the events
// TSB, SOBEL_ONE, SOBEL_TWO, F, MU and TB of render.cpp:425-548.
//   gradient of SUM and of each H channel: sum_sobel / h_sobel
//     (reintegration.cpp:191-259, coefficient tables lenia.h:30-71) or
//     sum_central_diff / h_central_diff (reintegration.cpp:260-315);
//   halo faces as the border routines leave them (transposition.cpp:6-665):
//     torus copies the opposite face, wall the nearest interior cell, none
//     zero; edge and corner halo cells read 0;
//   alpha = clamp((A/theta_A)^2, 0, 1) read at the reference's offsets
//     (lenia.cpp:650-671, compute_f at lenia.cpp:700-712);
//   F = NU (1 - alpha) - NA alpha (lenia.cpp:679-719);
//   MU and V: compute_{f,velocity}_mu[_wall] (reintegration.cpp:321-602).
// Every float operation keeps the reference's order and rounding (this file
// is compiled with -fmad=false), so outputs match the CPU restatement bit for
// bit given the same inputs.
//
// A block owns a 32 x 8 x FZ tile of cells; per field (SUM, then each H
// channel) one thread copies the field's tile with its halo into shared
// memory with a TMA tensor load (zero outside the grid, which is the zero
// border and the never-written halo edges), double buffered so that field
// f+1 lands while field f is used; blocks on the grid boundary then patch the
// torus/wall halo faces.  Each thread walks its z column with the three
// planes of 3 x 3 values around it in registers.
#include <cudaTypedefs.h>

#include "lenia_internal.h"
#include "tma.cuh"

namespace lenia {

// Two cells per thread along z and four blocks per SM (64 registers)
// measured faster than four cells and three blocks (80 registers): 100.8 vs
// 106.7 us at 128^3 x 4 channels; eight cells and two blocks: 112.7 us.
#ifndef LENIA_FLOW_Z
#define LENIA_FLOW_Z 2
#endif
#ifndef LENIA_FLOW_MINB
#define LENIA_FLOW_MINB 4
#endif
// The batched form keeps four cells per thread: with the torus faces its
// many small worlds patch, deeper tiles patch fewer cells per output
// (23.7 vs 23.9 ms per step for 512 config-3 worlds).
#ifndef LENIA_FLOW_MULTI_Z
#define LENIA_FLOW_MULTI_Z 4
#endif
constexpr int kFX = 32, kFY = 8;          // output tile in x, y (one thread per column)
constexpr int kFlowZ = LENIA_FLOW_Z;      // output cells per thread along z (one world's launch)
constexpr int kFlowMultiZ = LENIA_FLOW_MULTI_Z;  // the same in the batched launch
constexpr int kTX = 40, kTY = kFY + 2;    // staged tile: x from x0 - 4 (TMA x must be 16-byte aligned), y halo

// Staged tile of a launch whose threads own FZ cells along z.
template <int FZ>
struct FlowShape {
    static constexpr int TZ = FZ + 2;
    static constexpr int TILE = kTX * kTY * TZ;  // floats per staged field
    // the second tile buffer starts TILE floats in: TMA tile destinations
    // must be 128-byte aligned
    static_assert((TILE * sizeof(float)) % 128 == 0, "a tile buffer must keep the next one 128-byte aligned");
};

__device__ __forceinline__ float smax(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float smin(float a, float b) { return a < b ? a : b; }

// Source of cell (x, y, z) under the gradient halo rules; false when the
// cell reads 0 (edges, corners, zero faces).
__device__ __forceinline__ bool gb_source(const Dims &d, int border, int &x, int &y, int &z)
{
    const int ox = (x < 0) | (x >= d.W), oy = (y < 0) | (y >= d.H), oz = (z < 0) | (z >= d.D);
    const int no = ox + oy + oz;
    if (no == 0) return true;
    if (no > 1 || border == kBorderNone) return false;
    if (border == kBorderTorus) {
        x = x < 0 ? x + d.W : (x >= d.W ? x - d.W : x);
        y = y < 0 ? y + d.H : (y >= d.H ? y - d.H : y);
        z = z < 0 ? z + d.D : (z >= d.D ? z - d.D : z);
    } else {
        x = x < 0 ? 0 : (x >= d.W ? d.W - 1 : x);
        y = y < 0 ? 0 : (y >= d.H ? d.H - 1 : y);
        z = z < 0 ? 0 : (z >= d.D ? d.D - 1 : z);
    }
    return true;
}

// Torus/wall halo faces of a staged tile (the TMA copy left zeros there).
// Only the cells the gradients read are patched: x0-1..x0+32, y0-1..y0+8,
// z0-1..z0+FZ, with exactly one coordinate one step outside the grid.
// Each grid face the staged box reaches is walked over its in-grid cells
// (edges and corners keep the copy's zeros), so a block patches at most a
// few hundred cells per field instead of testing its whole box.
template <int FZ>
__device__ void patch_faces(float *tile, const float *f, const Dims &d, int border, int x0, int y0, int z0)
{
    const int tid = threadIdx.x + threadIdx.y * kFX;
    const int lo[3] = {x0 - 1, y0 - 1, z0 - 1};
    const int hi[3] = {x0 + kFX, y0 + kFY, z0 + FZ};  // inclusive
    const int ext[3] = {d.W, d.H, d.D};
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int side = 0; side < 2; side++) {
            const int g = side == 0 ? -1 : ext[a];  // the face layer outside the grid
            if (g < lo[a] || g > hi[a]) continue;
            const int a1 = a == 0 ? 1 : 0, a2 = a == 2 ? 1 : 2;
            const int l1 = lo[a1] > 0 ? lo[a1] : 0, h1 = hi[a1] < ext[a1] - 1 ? hi[a1] : ext[a1] - 1;
            const int l2 = lo[a2] > 0 ? lo[a2] : 0, h2 = hi[a2] < ext[a2] - 1 ? hi[a2] : ext[a2] - 1;
            const int n1 = h1 - l1 + 1, n2 = h2 - l2 + 1;
            if (n1 <= 0 || n2 <= 0) continue;
            for (int e = tid; e < n1 * n2; e += kFX * kFY) {
                int c[3];
                c[a] = g;
                c[a1] = l1 + e % n1;
                c[a2] = l2 + e / n1;
                const int t = (c[0] - x0 + 4) + (c[1] - y0 + 1) * kTX + (c[2] - z0 + 1) * kTX * kTY;
                int x = c[0], y = c[1], z = c[2];
                tile[t] = gb_source(d, border, x, y, z) ? __ldg(f + x + y * d.W + z * d.W * d.H) : 0.0f;
            }
        }
}

// True when any staged value is infinite, NaN or so large that a Sobel
// product could overflow (block-wide); such blocks take the literal 27-tap
// multiply-then-add path.
template <int FZ>
__device__ __forceinline__ bool tile_unsafe(const float *tile)
{
    constexpr int kTile = FlowShape<FZ>::TILE;
    static_assert(kTile % 4 == 0 && (kTile * 4) % 16 == 0, "tiles are read as float4");
    const int tid = threadIdx.x + threadIdx.y * kFX;
    const float4 *t4 = reinterpret_cast<const float4 *>(tile);
    int bad = 0;
    for (int e = tid; e < kTile / 4; e += kFX * kFY) {
        const float4 v = t4[e];
        bad |= !(fabsf(v.x) < 1.0e30f) | !(fabsf(v.y) < 1.0e30f) | !(fabsf(v.z) < 1.0e30f) | !(fabsf(v.w) < 1.0e30f);
    }
    return __syncthreads_or(bad) != 0;
}

// A / theta_A for a theta_A without an exact reciprocal: out of line, so
// that the compiler does not evaluate the IEEE division alongside the
// multiplication that the usual power-of-two theta_A takes.
__device__ __noinline__ float div_theta(float a, float ta) { return a / ta; }

__host__ __device__ constexpr float sob_w(int dd) { return dd == 0 ? 2.0f : 1.0f; }

// The 27-tap gradient as the reference writes it, acc = acc + v * coef, in
// (dz, dy, dx) order, around tile index c (returned by value: no local
// variable of the caller has its address taken).
__device__ __noinline__ float3 sobel_literal(const float *tile, int c)
{
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                const float v = tile[c + dx + dy * kTX + dz * kTX * kTY];
                ax = ax + v * (sob_w(dx) * sob_w(dy) * (float)dz);
                ay = ay + v * ((float)dx * sob_w(dy) * sob_w(dz));
                az = az + v * (sob_w(dx) * (float)dy * sob_w(dz));
            }
    return make_float3(ax, ay, az);
}

// The same gradient from three register planes (values v[(dy+1)*3 + dx+1] of
// z-1, z, z+1).  The coefficients are 0, +-1, +-2, +-4, so for finite values
// of moderate size v * coef is exact and acc + v * coef rounds exactly like
// fma(v, coef, acc); zero taps leave acc unchanged (acc starts at +0 and
// never becomes -0): the same bits as the literal form.
__device__ __forceinline__ void sobel_window(const float (&pm)[9], const float (&p0)[9], const float (&pp)[9],
                                             float &gx, float &gy, float &gz)
{
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
#pragma unroll
    for (int dz = -1; dz <= 1; dz++)
#pragma unroll
        for (int dy = -1; dy <= 1; dy++)
#pragma unroll
            for (int dx = -1; dx <= 1; dx++) {
                const int k = (dy + 1) * 3 + dx + 1;
                const float v = dz < 0 ? pm[k] : (dz == 0 ? p0[k] : pp[k]);
                if (dz != 0) ax = __fmaf_rn(v, sob_w(dx) * sob_w(dy) * (float)dz, ax);
                if (dx != 0) ay = __fmaf_rn(v, (float)dx * sob_w(dy) * sob_w(dz), ay);
                if (dy != 0) az = __fmaf_rn(v, sob_w(dx) * (float)dy * sob_w(dz), az);
            }
    gx = ax;
    gy = ay;
    gz = az;
}

__device__ __forceinline__ void load_plane(const float *tile, int c, float (&v)[9])
{
#pragma unroll
    for (int dy = -1; dy <= 1; dy++)
#pragma unroll
        for (int dx = -1; dx <= 1; dx++) v[(dy + 1) * 3 + dx + 1] = tile[c + dx + dy * kTX];
}

// The block (bx, by) of a world's flow launch: bx over the x-y tiles, by
// over the z tiles (OWN_GRID: the launch's own blockIdx, read where used).
// FULL: every cell of the block's tile is inside the grid (decided per
// block), so no thread tests its cells' bounds.
// tm_sum / tm_h: the world's tensor maps (kernel parameters, or a batch's
// world table in global memory).
// True when tile (bx, by) of a flow launch lies inside the grid.
template <int FZ>
__device__ __forceinline__ bool flow_tile_full(const Dims &d, int bx, int by)
{
    const int tiles_x = (d.W + kFX - 1) / kFX;
    return (bx % tiles_x) * kFX + kFX <= d.W && (bx / tiles_x) * kFY + kFY <= d.H && by * FZ + FZ <= d.D;
}

template <bool OWN_GRID, bool FULL, int FZ>
__device__ __forceinline__ void flow_body(const StepParams &p, const FlowBuffers &b, const CUtensorMap *tm_sum,
                                          const CUtensorMap *tm_h, int bx_arg, int by_arg)
{
    const int bx = OWN_GRID ? (int)blockIdx.x : bx_arg, by = OWN_GRID ? (int)blockIdx.y : by_arg;
    constexpr int kTile = FlowShape<FZ>::TILE;
    extern __shared__ __align__(128) float flow_smem[];
    __shared__ __align__(8) uint64_t bars[2];
    const Dims &d = p.d;
    const int C = p.C;
    const int N = d.N;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool leader = tx == 0 && ty == 0;
    const int tiles_x = (d.W + kFX - 1) / kFX;
    const int x0 = (bx % tiles_x) * kFX;
    const int y0 = (bx / tiles_x) * kFY;
    const int z0 = by * FZ;
    const int x = x0 + tx, y = y0 + ty;
    const bool col_in = FULL || (x < d.W && y < d.H);
    const float posx = (float)x + 0.5f, posy = (float)y + 0.5f, posz0 = (float)z0 + 0.5f;
    const int sobel = p.gradient_mode == kGradSobel;
    const float ta = p.theta_a;
    const bool patch = p.sobel_border != kBorderNone &&
                       (x0 == 0 || x0 + kFX >= d.W || y0 == 0 || y0 + kFY >= d.H || z0 == 0 || z0 + FZ >= d.D);

    if (leader) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    pdl_trigger();
    pdl_wait();
    // field 0 is SUM, field 1 + c is H channel c
    auto issue = [&](int f) {
        if (!leader) return;
        const int buf = f & 1;
        fence_proxy_async();
        mbar_arrive_expect_tx(&bars[buf], kTile * 4);
        if (f == 0) tma_load_3d(flow_smem + buf * kTile, tm_sum, x0 - 4, y0 - 1, z0 - 1, &bars[buf]);
        else tma_load_4d(flow_smem + buf * kTile, tm_h, x0 - 4, y0 - 1, z0 - 1, f - 1, &bars[buf]);
    };

    // Waits for field f's tile, patches its faces and decides the path:
    // 1 when the literal (non-finite) path is needed, 0 otherwise, -1 when the
    // wait ran out (block-wide): the timeout is recorded and the copies in
    // flight (fields f and f + 1) are drained; the block then returns.
    auto land = [&](int f) -> int {
        float *tile = flow_smem + (f & 1) * kTile;
        if (!block_wait(&bars[f & 1], (unsigned)(f >> 1) & 1u, p.wait_polls)) {
            mbar_wait(&bars[f & 1], (unsigned)(f >> 1) & 1u, kDrainPolls);
            if (f + 1 <= C) mbar_wait(&bars[(f + 1) & 1], (unsigned)((f + 1) >> 1) & 1u, kDrainPolls);
            if (leader && b.err) atomicOr(b.err, 2);
            return -1;
        }
        if (patch) {
            patch_faces<FZ>(tile, f == 0 ? b.SUM : b.H + (f - 1) * N, d, p.sobel_border, x0, y0, z0);
            __syncthreads();
        }
        return (sobel && tile_unsafe<FZ>(tile)) ? 1 : 0;
    };
    // the column: tile index of (x, y, z0 + lz) is col + (lz + 1) * plane
    const int col = (tx + 4) + (ty + 1) * kTX;
    constexpr int plane = kTX * kTY;
    // Gradient of output lz of this column; win holds the Sobel planes.
    auto grad = [&](const float *tile, bool literal, int lz, float (&win)[3][9], float (&g)[3]) {
        const int cc = col + (lz + 1) * plane;
        if (sobel) {
            if (literal) {
                const float3 r = sobel_literal(tile, cc);
                g[0] = r.x;
                g[1] = r.y;
                g[2] = r.z;
            } else {
                if (lz == 0) {
                    load_plane(tile, col, win[0]);
                    load_plane(tile, col + plane, win[1]);
                }
                load_plane(tile, cc + plane, win[(lz + 2) % 3]);
                sobel_window(win[lz % 3], win[(lz + 1) % 3], win[(lz + 2) % 3], g[0], g[1], g[2]);
            }
        } else {
            g[0] = (tile[cc + 1] - tile[cc - 1]) * 0.5f;
            g[1] = (tile[cc + kTX] - tile[cc - kTX]) * 0.5f;
            g[2] = (tile[cc + plane] - tile[cc - plane]) * 0.5f;
        }
    };

    // field 0: the gradient of SUM (NA), kept in registers for every channel
    float na[FZ][3];
    issue(0);
    issue(1);
    {
        const int landed = land(0);
        if (landed < 0) return;
        const bool literal = landed != 0;
        float win[3][9];
#pragma unroll
        for (int lz = 0; lz < FZ; lz++) {
            grad(flow_smem, literal, lz, win, na[lz]);
            const int z = z0 + lz;
            if (b.NA && col_in && (FULL || z < d.D)) {
                const int i = x + y * d.W + z * d.W * d.H;
                b.NA[i] = na[lz][0];
                b.NA[N + i] = na[lz][1];
                b.NA[2 * N + i] = na[lz][2];
            }
        }
        fence_proxy_async();
        __syncthreads();
    }
    // fields 1..C: the gradient of H channel c = f - 1 and the flow epilogue
    for (int f = 1; f <= C; f++) {
        float *tile = flow_smem + (f & 1) * kTile;
        if (f < C) issue(f + 1);
        // per-cell inputs of this channel, loaded while the tile lands
        float v3[3][FZ], gal[FZ];
        unsigned gvalid = 0;  // bit lz: the alpha source of cell lz was written
        const int c = f - 1;
        if (col_in) {
#pragma unroll
            for (int lz = 0; lz < FZ; lz++) {
                const int z = z0 + lz;
                if (!FULL && z >= d.D) continue;
                const int i = x + y * d.W + z * d.W * d.H;
                const int ci = c * N + i;
#pragma unroll
                for (int q = 0; q < 3; q++) v3[q][lz] = b.V[q * C * N + ci];
                // alpha source: PREALPHA as compute_f reads it (flat c*N + i),
                // written by sobel_convolve_h from channel f / P, cell f % P (Q20)
                int src_c = c, src_i = i;
                bool valid = true;
                if (!p.alpha_index_fix) {
                    // ci < 4 N < 4 P < 2^31 (sides <= 256), so the block
                    // index is 0..3 and 32-bit arithmetic is exact
                    const int P = (int)d.P;
                    src_c = (ci >= P) + (ci >= 2 * P) + (ci >= 3 * P);
                    src_i = ci - src_c * P;
                    valid = src_c < C && src_i < N;
                }
                gal[lz] = valid ? __ldg(b.A + src_c * N + src_i) : 0.0f;
                gvalid |= (valid ? 1u : 0u) << lz;
            }
        }
        const int landed = land(f);
        if (landed < 0) return;
        const bool literal = landed != 0;
        float win[3][9];
#pragma unroll
        for (int lz = 0; lz < FZ; lz++) {
            float g[3];
            grad(tile, literal, lz, win, g);
            const int z = z0 + lz;
            if (!FULL && (!col_in || z >= d.D)) continue;
            const int i = x + y * d.W + z * d.W * d.H;
            const int ci = c * N + i;
            float alpha;
            {
                const float gv = gal[lz];
                if (!((gvalid >> lz) & 1u)) {
                    alpha = 0.0f;
                } else {
                    float pg = p.inv_theta_a != 0.0f ? gv * p.inv_theta_a : div_theta(gv, ta);
                    pg = pg * pg;
                    alpha = smin(smax(pg, 0.0f), 1.0f);
                }
            }
            if (b.PREALPHA) b.PREALPHA[ci] = alpha;
            if (b.NU) {
                b.NU[ci] = g[0];
                b.NU[C * N + ci] = g[1];
                b.NU[2LL * C * N + ci] = g[2];
            }
            if (b.ALPHA) {
                // ALPHA = |GRID - GA| with GA read at c*P + i (Q20)
                // (GA blocks past the last channel are never written: 0)
                const float ga_g = __ldg(b.A + ci);
                const int fi = p.alpha_index_fix ? ci : c * d.P + i;
                const float ga = fi < C * N ? __ldg(b.GA + fi) : 0.0f;
                b.ALPHA[ci] = fabsf(ga_g - ga);
            }
            const float a1 = 1.0f - alpha;
            float f3[3];
#pragma unroll
            for (int q = 0; q < 3; q++) f3[q] = g[q] * a1 - na[lz][q] * alpha;
            if (b.F) {
#pragma unroll
                for (int q = 0; q < 3; q++) b.F[q * C * N + ci] = f3[q];
            }
            float vv[3] = {v3[0][lz], v3[1][lz], v3[2][lz]};
            // (float)z + 0.5f, exactly: every term is a small whole or half number
            const float pos[3] = {posx, posy, posz0 + (float)lz};
            if (p.mu_vel) {
#pragma unroll
                for (int q = 0; q < 3; q++) vv[q] = (vv[q] + f3[q]) * p.v_damp;
            }
#pragma unroll
            for (int q = 0; q < 3; q++) {
                float m = (p.mu_vel ? vv[q] : f3[q]) * p.timestep;
                m = smax(m, -p.ma);
                m = smin(m, p.ma);
                m = pos[q] + m;
                if (p.border == kBorderWall) {
                    m = smax(m, p.sigma);
                    m = smin(m, q == 1 ? p.ghs : p.gws);
                }
                b.MU[q * C * N + ci] = m;
            }
            if (!p.mu_vel) {
#pragma unroll
                for (int q = 0; q < 3; q++) vv[q] = (vv[q] + f3[q]) * p.v_damp;
            }
#pragma unroll
            for (int q = 0; q < 3; q++) b.V[q * C * N + ci] = vv[q];
        }
        // every thread is done with this buffer (including its generic writes)
        // before the next TMA copy into it
        fence_proxy_async();
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kFX *kFY, LENIA_FLOW_MINB) k_flow(StepParams p, FlowBuffers b,
                                                   const __grid_constant__ CUtensorMap tm_sum,
                                                   const __grid_constant__ CUtensorMap tm_h)
{
    if (flow_tile_full<kFlowZ>(p.d, blockIdx.x, blockIdx.y))
        flow_body<true, true, kFlowZ>(p, b, &tm_sum, &tm_h, 0, 0);
    else
        flow_body<true, false, kFlowZ>(p, b, &tm_sum, &tm_h, 0, 0);
}

// Copies a world's parameter block into shared memory (whole 4-byte words).
template <typename T>
__device__ __forceinline__ void copy_to_shared(T *dst, const T *src)
{
    static_assert(sizeof(T) % 4 == 0, "copied as 4-byte words");
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int nthr = blockDim.x * blockDim.y;
    for (int i = tid; i < (int)(sizeof(T) / 4); i += nthr)
        reinterpret_cast<unsigned *>(dst)[i] = reinterpret_cast<const unsigned *>(src)[i];
}

// A tensor map written to global memory before the launch, made visible to
// the copy engine's reads of it.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap *m)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(m) : "memory");
}

// The flow of a batch of worlds: block b is block items[b].block of world
// items[b].world's own launch (x-y tile fastest); the world's parameters
// are read into shared memory first.
#ifndef LENIA_FLOW_MULTI_MINB
#define LENIA_FLOW_MULTI_MINB 3
#endif
// the batched form: four cells per thread, three blocks per SM
__global__ void __launch_bounds__(kFX *kFY, LENIA_FLOW_MULTI_MINB) k_flow_multi(const BatchWorldDev *__restrict__ ws,
                                                                         const WorkItem *__restrict__ items)
{
    __shared__ StepParams sp;
    __shared__ FlowBuffers sb;
    const WorkItem it = items[blockIdx.x];
    const BatchWorldDev *w = ws + it.world;
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        // the copy engine's descriptor reads start while the parameters load
        asm volatile("prefetch.tensormap [%0];\n" ::"l"(&w->tm_sum) : "memory");
        asm volatile("prefetch.tensormap [%0];\n" ::"l"(&w->tm_h) : "memory");
    }
    copy_to_shared(&sp, &w->p);
    copy_to_shared(&sb, &w->fb);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        tensormap_acquire(&w->tm_sum);
        tensormap_acquire(&w->tm_h);
    }
    const int gx = w->flow_gx;
    __syncthreads();
    const int bx = it.block % gx, by = it.block / gx;
    if (flow_tile_full<kFlowMultiZ>(sp.d, bx, by))
        flow_body<false, true, kFlowMultiZ>(sp, sb, &w->tm_sum, &w->tm_h, bx, by);
    else
        flow_body<false, false, kFlowMultiZ>(sp, sb, &w->tm_sum, &w->tm_h, bx, by);
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
}

cudaError_t encode_tensor_map_typed(CUtensorMap *map, const void *base, int dtype, int elem_bytes, int rank,
                                    const unsigned long long *dims, const unsigned *box)
{
    unsigned long long strides[4];
    unsigned long long stride = (unsigned long long)elem_bytes;
    for (int i = 0; i + 1 < rank && i < 4; i++) {
        stride *= dims[i];
        strides[i] = stride;
    }
    return encode_tensor_map_strided(map, base, dtype, rank, dims, strides, box);
}

cudaError_t encode_tensor_map_strided(CUtensorMap *map, const void *base, int dtype, int rank,
                                      const unsigned long long *dims, const unsigned long long *strides,
                                      const unsigned *box)
{
    if (rank < 1 || rank > 5) return cudaErrorInvalidValue;
    if (!g_encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
        g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    cuuint64_t gdim[5], gstride[4];
    cuuint32_t bdim[5], estride[5];
    for (int i = 0; i < rank; i++) {
        gdim[i] = dims[i];
        bdim[i] = box[i];
        estride[i] = 1;
        if (i > 0) gstride[i - 1] = strides[i - 1];
    }
    const CUresult r = g_encode(map, (CUtensorMapDataType)dtype, (cuuint32_t)rank, (void *)base, gdim, gstride, bdim,
                                estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t encode_tensor_map(CUtensorMap *map, const float *base, int rank, const unsigned long long *dims,
                              const unsigned *box)
{
    return encode_tensor_map_typed(map, base, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (int)sizeof(float), rank, dims, box);
}

// Blocks of a world in the batched flow launch (gx: tiles per z layer).
int flow_blocks(const Dims &d, int *gx)
{
    const int tiles_x = (d.W + kFX - 1) / kFX, tiles_y = (d.H + kFY - 1) / kFY;
    if (gx) *gx = tiles_x * tiles_y;
    return tiles_x * tiles_y * ((d.D + kFlowMultiZ - 1) / kFlowMultiZ);
}

cudaError_t launch_flow_multi(const BatchWorldDev *ws, const WorkItem *items, int n_items, cudaStream_t st)
{
    if (n_items == 0) return cudaSuccess;
    const size_t smem = 2 * FlowShape<kFlowMultiZ>::TILE * sizeof(float);
    cudaError_t e = cudaFuncSetAttribute(k_flow_multi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_flow_multi<<<(unsigned)n_items, dim3(kFX, kFY), smem, st>>>(ws, items);
    return cudaGetLastError();
}

// A flow launch's tensor maps: SUM (x, y, z) and H (x, y, z, channel), tiles
// of 40 x 10 x (fz + 2) for threads owning fz cells along z.
cudaError_t flow_maps(const StepParams &p, const FlowBuffers &b, CUtensorMap *tm_sum, CUtensorMap *tm_h, int fz)
{
    const Dims &d = p.d;
    const unsigned long long dsum[3] = {(unsigned long long)d.W, (unsigned long long)d.H, (unsigned long long)d.D};
    const unsigned long long dh[4] = {(unsigned long long)d.W, (unsigned long long)d.H, (unsigned long long)d.D,
                                      (unsigned long long)p.C};
    const unsigned box[4] = {(unsigned)kTX, (unsigned)kTY, (unsigned)(fz + 2), 1u};
    cudaError_t e = encode_tensor_map(tm_sum, b.SUM, 3, dsum, box);
    if (e == cudaSuccess) e = encode_tensor_map(tm_h, b.H, 4, dh, box);
    return e;
}

// The batched flow launch's tensor maps of a world.
cudaError_t flow_tensor_maps(const StepParams &p, const FlowBuffers &b, CUtensorMap *tm_sum, CUtensorMap *tm_h)
{
    return flow_maps(p, b, tm_sum, tm_h, kFlowMultiZ);
}

cudaError_t launch_flow(const StepParams &p, const FlowBuffers &b, cudaStream_t st)
{
    const Dims &d = p.d;
    CUtensorMap tm_sum, tm_h;
    cudaError_t e = flow_maps(p, b, &tm_sum, &tm_h, kFlowZ);
    if (e != cudaSuccess) return e;
    const int tiles_x = (d.W + kFX - 1) / kFX, tiles_y = (d.H + kFY - 1) / kFY;
    dim3 grid(tiles_x * tiles_y, (d.D + kFlowZ - 1) / kFlowZ);
    dim3 block(kFX, kFY);
    const size_t smem = 2 * FlowShape<kFlowZ>::TILE * sizeof(float);
    return launch_pdl(k_flow, grid, block, smem, st, p, b, tm_sum, tm_h);
}

}  // namespace lenia
