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
#include "lenia_internal.h"
#include "async_copy.cuh"

namespace lenia {

constexpr int kFX = 32, kFY = 8, kFZ = 4;  // output tile
constexpr int kSX = kFX + 2, kSY = kFY + 2, kSZ = kFZ + 2;

__device__ __forceinline__ float smax(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float smin(float a, float b) { return a < b ? a : b; }

// Source of tile cell (x, y, z) under the gradient halo rules; false when
// the cell reads 0 (edges, corners, zero faces).
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

// Queues the asynchronous copy of one field's tile (with its one-cell halo).
__device__ __forceinline__ void issue_tile(float *tile, const float *f, const Dims &d, int x0, int y0, int z0,
                                           int border)
{
    const int tid = threadIdx.x + threadIdx.y * kFX;
    for (int e = tid; e < kSX * kSY * kSZ; e += kFX * kFY) {
        const int lx = e % kSX, ly = (e / kSX) % kSY, lz = e / (kSX * kSY);
        int x = x0 + lx - 1, y = y0 + ly - 1, z = z0 + lz - 1;
        const bool ok = gb_source(d, border, x, y, z);
        const float *src = ok ? f + x + y * d.W + z * d.W * d.H : f;
        cp_async_f32(tile + e, src, ok);
    }
    cp_async_commit();
}

// True when any value of the tile is infinite, NaN or so large that a
// Sobel product could overflow (block-wide); such blocks take the literal
// 27-tap multiply-then-add path.
__device__ __forceinline__ bool tile_unsafe(const float *tile)
{
    const int tid = threadIdx.x + threadIdx.y * kFX;
    int bad = 0;
    for (int e = tid; e < kSX * kSY * kSZ; e += kFX * kFY) bad |= !(fabsf(tile[e]) < 1.0e30f);
    return __syncthreads_or(bad) != 0;
}

__device__ __forceinline__ float sob_w(int dd) { return dd == 0 ? 2.0f : 1.0f; }

// Gradient at tile position (lx, ly, lz) (interior coordinates).
// Literal path (`literal`): every tap as the reference writes it,
// acc = acc + v * coef.  Fast path: the coefficients are 0, +-1, +-2, +-4, so
// for finite v of moderate size v * coef is exact and acc + v * coef rounds
// exactly like fma(v, coef, acc); zero taps leave acc unchanged (acc starts at
// +0 and never becomes -0).  Both paths give the same bits.
template <bool LITERAL>
__device__ __forceinline__ void sobel_taps(const float *tile, int lx, int ly, int lz, float &gx, float &gy, float &gz)
{
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
#pragma unroll
    for (int dz = -1; dz <= 1; dz++)
#pragma unroll
        for (int dy = -1; dy <= 1; dy++)
#pragma unroll
            for (int dx = -1; dx <= 1; dx++) {
                const float v = tile[(lx + 1 + dx) + (ly + 1 + dy) * kSX + (lz + 1 + dz) * kSX * kSY];
                const float cx = sob_w(dx) * sob_w(dy) * (float)dz;
                const float cy = (float)dx * sob_w(dy) * sob_w(dz);
                const float cz = sob_w(dx) * (float)dy * sob_w(dz);
                if (LITERAL) {
                    ax = ax + v * cx;
                    ay = ay + v * cy;
                    az = az + v * cz;
                } else {
                    if (dz != 0) ax = __fmaf_rn(v, cx, ax);
                    if (dx != 0) ay = __fmaf_rn(v, cy, ay);
                    if (dy != 0) az = __fmaf_rn(v, cz, az);
                }
            }
    gx = ax;
    gy = ay;
    gz = az;
}

__device__ __noinline__ void sobel_literal(const float *tile, int lx, int ly, int lz, float &gx, float &gy, float &gz)
{
    sobel_taps<true>(tile, lx, ly, lz, gx, gy, gz);
}

__device__ __forceinline__ void gradient(const float *tile, int lx, int ly, int lz, int sobel, bool literal,
                                         float &gx, float &gy, float &gz)
{
    if (sobel) {
        if (literal) sobel_literal(tile, lx, ly, lz, gx, gy, gz);
        else sobel_taps<false>(tile, lx, ly, lz, gx, gy, gz);
    } else {
        const int c = (lx + 1) + (ly + 1) * kSX + (lz + 1) * kSX * kSY;
        gx = (tile[c + 1] - tile[c - 1]) * 0.5f;
        gy = (tile[c + kSX] - tile[c - kSX]) * 0.5f;
        gz = (tile[c + kSX * kSY] - tile[c - kSX * kSY]) * 0.5f;
    }
}

__global__ void __launch_bounds__(kFX *kFY) k_flow(StepParams p, FlowBuffers b)
{
    __shared__ float tiles[2][kSX * kSY * kSZ];
    const Dims &d = p.d;
    const int C = p.C;
    const int N = d.N;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tiles_x = (d.W + kFX - 1) / kFX;
    const int x0 = (blockIdx.x % tiles_x) * kFX;
    const int y0 = (blockIdx.x / tiles_x) * kFY;
    const int z0 = blockIdx.y * kFZ;
    const int x = x0 + tx, y = y0 + ty;
    const bool col_in = x < d.W && y < d.H;
    const int sobel = p.gradient_mode == kGradSobel;
    const float ta = p.theta_a;

    float na[kFZ][3];
    // field 0 is SUM, field 1 + c is H channel c; field f+1 loads while f computes
    issue_tile(tiles[0], b.SUM, d, x0, y0, z0, p.sobel_border);
    for (int f = 0; f <= C; f++) {
        float *tile = tiles[f & 1];
        if (f < C) issue_tile(tiles[(f + 1) & 1], b.H + f * N, d, x0, y0, z0, p.sobel_border);
        // per-cell inputs of this channel, loaded while the tile lands
        float v3[3][kFZ], gal[kFZ];
        unsigned gvalid = 0;  // bit lz: the alpha source of cell lz was written
        const int c = f - 1;
        if (f > 0 && col_in) {
#pragma unroll
            for (int lz = 0; lz < kFZ; lz++) {
                const int z = z0 + lz;
                if (z >= d.D) continue;
                const int i = x + y * d.W + z * d.W * d.H;
                const int ci = c * N + i;
#pragma unroll
                for (int q = 0; q < 3; q++) v3[q][lz] = b.V[q * C * N + ci];
                // alpha source: PREALPHA as compute_f reads it (flat c*N + i),
                // written by sobel_convolve_h from channel f / P, cell f % P (Q20)
                int src_c = c, src_i = i;
                bool valid = true;
                if (!p.alpha_index_fix) {
                    // ci < 4 N < 4 P, so the block index is 0..3
                    src_c = (ci >= d.P) + (ci >= 2 * d.P) + (ci >= 3 * d.P);
                    src_i = ci - src_c * d.P;
                    valid = src_c < C && src_i < N;
                }
                gal[lz] = valid ? __ldg(b.A + src_c * N + src_i) : 0.0f;
                gvalid |= (valid ? 1u : 0u) << lz;
            }
        }
        if (f < C) cp_async_wait<1>();
        else cp_async_wait<0>();
        __syncthreads();
        const bool literal = sobel && tile_unsafe(tile);
        if (f == 0) {
#pragma unroll
            for (int lz = 0; lz < kFZ; lz++) gradient(tile, tx, ty, lz, sobel, literal, na[lz][0], na[lz][1], na[lz][2]);
            if (b.NA && col_in) {
#pragma unroll
                for (int lz = 0; lz < kFZ; lz++) {
                    const int z = z0 + lz;
                    if (z >= d.D) continue;
                    const int i = x + y * d.W + z * d.W * d.H;
                    b.NA[i] = na[lz][0];
                    b.NA[N + i] = na[lz][1];
                    b.NA[2 * N + i] = na[lz][2];
                }
            }
        } else if (col_in) {
#pragma unroll
            for (int lz = 0; lz < kFZ; lz++) {
                const int z = z0 + lz;
                if (z >= d.D) continue;
                const int i = x + y * d.W + z * d.W * d.H;
                const int ci = c * N + i;
                float nu[3];
                gradient(tile, tx, ty, lz, sobel, literal, nu[0], nu[1], nu[2]);
                float alpha;
                {
                    const float g = gal[lz];
                    if (!((gvalid >> lz) & 1u)) {
                        alpha = 0.0f;
                    } else {
                        float pg = g / ta;
                        pg = pg * pg;
                        alpha = smin(smax(pg, 0.0f), 1.0f);
                    }
                }
                if (b.PREALPHA) b.PREALPHA[ci] = alpha;
                if (b.NU) {
                    b.NU[ci] = nu[0];
                    b.NU[C * N + ci] = nu[1];
                    b.NU[2LL * C * N + ci] = nu[2];
                }
                if (b.ALPHA) {
                    // ALPHA = |GRID - GA| with GA read at c*P + i (Q20)
                    // (GA blocks past the last channel are never written: 0)
                    const float g = __ldg(b.A + ci);
                    const int fi = p.alpha_index_fix ? ci : c * d.P + i;
                    const float ga = fi < C * N ? __ldg(b.GA + fi) : 0.0f;
                    b.ALPHA[ci] = fabsf(g - ga);
                }
                const float a1 = 1.0f - alpha;
                float f3[3];
#pragma unroll
                for (int q = 0; q < 3; q++) f3[q] = nu[q] * a1 - na[lz][q] * alpha;
                if (b.F) {
#pragma unroll
                    for (int q = 0; q < 3; q++) b.F[q * C * N + ci] = f3[q];
                }
                float vv[3] = {v3[0][lz], v3[1][lz], v3[2][lz]};
                const float pos[3] = {(float)x + 0.5f, (float)y + 0.5f, (float)z + 0.5f};
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
        }
        __syncthreads();
    }
}

cudaError_t launch_flow(const StepParams &p, const FlowBuffers &b, cudaStream_t st)
{
    const int tiles_x = (p.d.W + kFX - 1) / kFX, tiles_y = (p.d.H + kFY - 1) / kFY;
    dim3 grid(tiles_x * tiles_y, (p.d.D + kFZ - 1) / kFZ);
    dim3 block(kFX, kFY);
    k_flow<<<grid, block, 0, st>>>(p, b);
    return cudaGetLastError();
}

}  // namespace lenia
