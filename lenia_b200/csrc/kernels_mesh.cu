// Marching cubes: generate_mesh_v1/v2/v3 (mesh.cpp:34-431, 434-1109,
// 1115-2037) with the buffer reset and concatenation around them
// (render.cpp:153-212), as five launches.
//
// The reference creates vertices in a fixed order: slab (mesh thread), then
// channel, then cube (x fastest), then field (v1 meshes RBB; v2 adds U_SUM_RB,
// v3 adds H_RB, each with its own vertex map), then triangle slot; an edge's
// vertex is created by the first triangle slot that names the edge (a vertex
// map, V1_EDGES/V2_EDGES/V3_EDGES, is keyed by edge origin and axis, per
// slab), and every triangle that names the edge adds its face normal to it.
// On the GPU:
//
//   mc_count    per cube and channel: case index, triangle count, and how many
//               vertices the cube creates; per chunk of kMcThreads cubes and
//               channel the two sums (one block reduction per chunk);
//   mc_scan     exclusive scan of the chunk sums (one block, coalesced tiles);
//               emit and index skip chunk-channels without triangles, so
//               their work follows the surface, not the volume;
//   mc_emit     per cube: face normals of its triangles; position, channel and
//               source edge of the vertices it creates;
//   mc_index    per cube: the vertex of every triangle slot;
//   mc_normals  per vertex: the face normals of the triangles that name its
//               edge, summed in creation order.
//
// No atomics and no edge-keyed map: the cube that creates an edge's vertex is
// the edge's first neighbouring cube in scan order within the slab (every
// neighbour of an intersected edge has triangles on it), in the first channel
// where the edge is intersected when channels share vertices.  Each cube
// therefore knows which vertices it creates, and the creator of any edge, and
// the rank of the vertex among the creator's, follow from the stored case
// indices.  Every value is computed with the reference's operations in its
// order, so the result is bit-identical to a sequential run.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "lenia_internal.h"

namespace {

constexpr int kMcThreads = 256;          // threads per block = cubes per chunk
constexpr int kMcWarps = kMcThreads / 32;
constexpr int kMcMaxDim = 512;

// ---- cube geometry (corner order of mesh.cpp:19-32) ----------------------
// corner i: x = bit i of 0x66, y = i >= 4, z = bit i of 0xCC
__host__ __device__ constexpr int mc_cx(int i) { return (0x66 >> i) & 1; }
__host__ __device__ constexpr int mc_cy(int i) { return (i >> 2) & 1; }
__host__ __device__ constexpr int mc_cz(int i) { return (0xCC >> i) & 1; }
__host__ __device__ constexpr int mc_coord(int i, int d) { return d == 0 ? mc_cx(i) : d == 1 ? mc_cy(i) : mc_cz(i); }
// edge e joins corners p and q: e < 4: e, e+1 mod 4; e < 8: e, 4 + (e-3) mod 4;
// else e-8, e-4.  Its vertex is interpolated from the lower-numbered corner.
__host__ __device__ constexpr int mc_p(int e) { return e < 8 ? e : e - 8; }
__host__ __device__ constexpr int mc_q(int e) { return e < 4 ? ((e + 1) & 3) : e < 8 ? 4 + ((e - 3) & 3) : e - 4; }
__host__ __device__ constexpr int mc_a(int e) { return mc_p(e) < mc_q(e) ? mc_p(e) : mc_q(e); }
__host__ __device__ constexpr int mc_b(int e) { return mc_p(e) < mc_q(e) ? mc_q(e) : mc_p(e); }
__host__ __device__ constexpr int mc_axis(int e)
{
    return mc_cx(mc_a(e)) != mc_cx(mc_b(e)) ? 0 : mc_cy(mc_a(e)) != mc_cy(mc_b(e)) ? 1 : 2;
}
// origin of edge e relative to its cube, coordinate d
__host__ __device__ constexpr int mc_off(int e, int d)
{
    return mc_coord(mc_a(e), d) < mc_coord(mc_b(e), d) ? mc_coord(mc_a(e), d) : mc_coord(mc_b(e), d);
}
// The four cubes around a grid edge of axis `ax`, in scan order (z, then y,
// then x ascending): the cube that has the edge as its local edge e sits at
// the edge origin minus mc_off(e), so the order is descending (oz, oy, ox).
__host__ __device__ constexpr int mc_axis_edge(int ax, int j)
{
    for (int e = 0; e < 12; e++) {
        if (mc_axis(e) != ax) continue;
        const int key = mc_off(e, 2) * 4 + mc_off(e, 1) * 2 + mc_off(e, 0);
        int rank = 0;
        for (int f = 0; f < 12; f++)
            if (mc_axis(f) == ax && mc_off(f, 2) * 4 + mc_off(f, 1) * 2 + mc_off(f, 0) > key) rank++;
        if (rank == j) return e;
    }
    return -1;
}

// Edge descriptor: a | b << 3 | axis << 6 | ox << 8 | oy << 9 | oz << 10.
__host__ __device__ constexpr unsigned mc_edge_desc(int e)
{
    return (unsigned)(mc_a(e) | mc_b(e) << 3 | mc_axis(e) << 6 | mc_off(e, 0) << 8 | mc_off(e, 1) << 9 |
                      mc_off(e, 2) << 10);
}

__host__ __device__ __forceinline__ unsigned active_edges(int cs)
{
    unsigned m = 0;
#pragma unroll
    for (int e = 0; e < 12; e++) m |= (unsigned)(((cs >> mc_a(e)) ^ (cs >> mc_b(e))) & 1) << e;
    return m;
}

// Tables shared by the kernels (copied to shared memory per block).
struct McTables {
    // per case: edge of slot k in bits 4k..4k+3 (k < 15), triangle count in bits 60..63
    unsigned long long tri[256];
    // per boundary class (see boundary_class): the edges whose vertex this cube creates
    unsigned short owned[64];
    unsigned edge[12];              // mc_edge_desc
    unsigned char axis_edges[12];   // mc_axis_edge(ax, j) at 4 * ax + j
    unsigned short act[256];        // per case: active_edges(case)
};

constexpr int kMcMaxFields = 3;

struct McGeom {
    int W, H, D, C, F;
    int slabs, nblk;  // z slabs; chunks per slab (of the largest slab)
    long long N;
    int share;
    float iso, cell;
    float off[kMcMaxFields][3];
    const float *fld[kMcMaxFields];   // interiors
    const float *halo[kMcMaxFields];  // arrays the +1 faces copy
};

// Offset of (field f, channel c) in the per-cube arrays (cases, tri_base,
// vert_base): fields outermost.
__device__ __forceinline__ long long fc_off(const McGeom &g, int f, int c) { return (long long)(f * g.C + c) * g.N; }

__device__ __forceinline__ int slot_edge(unsigned long long t, int k) { return (int)((t >> (4 * k)) & 15); }
__device__ __forceinline__ int tri_count(unsigned long long t) { return (int)(t >> 60); }

__device__ __forceinline__ void slab_range(const McGeom &g, int s, int &z0, int &z1)
{
    z0 = (g.D / g.slabs) * s;
    z1 = s == g.slabs - 1 ? g.D : z0 + g.D / g.slabs;
}

// Which of the six slab boundaries cube (x, y, z) touches; the edges a cube
// creates depend only on this.
__device__ __forceinline__ int boundary_class(const McGeom &g, int x, int y, int z, int z0, int z1)
{
    return (x == 0) | (x == g.W - 1) << 1 | (y == 0) << 2 | (y == g.H - 1) << 3 | (z == z0) << 4 |
           (z == z1 - 1) << 5;
}

// Corner values of cube (gx, gy, gz) of one channel.  Corners on one +1 face
// read the periodic copy of `halo` (transpose_mesh_borders copies GRID into
// RBB's faces, but H and U_SUM of the current step into those of H_RB and
// U_SUM_RB, transposition.cpp:881-995); corners on two or three +1 faces
// (halo edges and corners) read 0.
__device__ __forceinline__ void load_corners(const float *f, const float *halo, const McGeom &g, int gx, int gy,
                                             int gz, float *v)
{
    const int W = g.W, WH = g.W * g.H;
    if (gx + 1 < g.W && gy + 1 < g.H && gz + 1 < g.D) {
        // cells < 2^27: 32-bit offsets
        const float *p = f + (gx + gy * W + gz * WH);
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = __ldg(p + (mc_cx(i) + mc_cy(i) * W + mc_cz(i) * WH));
        return;
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
        int x = gx + mc_cx(i), y = gy + mc_cy(i), z = gz + mc_cz(i);
        const int out = (x >= g.W) + (y >= g.H) + (z >= g.D);
        if (x >= g.W) x -= g.W;
        if (y >= g.H) y -= g.H;
        if (z >= g.D) z -= g.D;
        v[i] = out > 1 ? 0.0f : __ldg((out ? halo : f) + (x + y * W + z * WH));
    }
}

__device__ __forceinline__ float sel8(const float *v, int i)
{
    const float a = (i & 1) ? v[1] : v[0], b = (i & 1) ? v[3] : v[2];
    const float c = (i & 1) ? v[5] : v[4], d = (i & 1) ? v[7] : v[6];
    const float ab = (i & 2) ? b : a, cd = (i & 2) ? d : c;
    return (i & 4) ? cd : ab;
}

// Vertex on edge e of cube (gx, gy, gz): Pa + (Pb - Pa) * ((iso - va) / (vb - va))
// with P = (g + delta) * cell (mesh.cpp:86-196), then + the field's offset on
// each axis where it is nonzero (mesh.cpp:434-1109 shifts U_SUM_RB's mesh
// along x, mesh.cpp:1375-1397 H_RB's along z).
__device__ __forceinline__ float3 edge_vertex(const McGeom &g, int f, unsigned ed, const float *v, int gx, int gy,
                                              int gz)
{
    const int a = ed & 7, b = (ed >> 3) & 7;
    const float va = sel8(v, a), vb = sel8(v, b);
    const float T = (g.iso - va) / (vb - va);
    const float ax = ((float)gx + (float)mc_cx(a)) * g.cell, bx = ((float)gx + (float)mc_cx(b)) * g.cell;
    const float ay = ((float)gy + (float)mc_cy(a)) * g.cell, by = ((float)gy + (float)mc_cy(b)) * g.cell;
    const float az = ((float)gz + (float)mc_cz(a)) * g.cell, bz = ((float)gz + (float)mc_cz(b)) * g.cell;
    float3 r;
    r.x = ax + (bx - ax) * T;
    r.y = ay + (by - ay) * T;
    r.z = az + (bz - az) * T;
    if (g.off[f][0] != 0.0f) r.x = r.x + g.off[f][0];
    if (g.off[f][1] != 0.0f) r.y = r.y + g.off[f][1];
    if (g.off[f][2] != 0.0f) r.z = r.z + g.off[f][2];
    return r;
}

__device__ __forceinline__ void load_tables(const McTables *src, McTables &dst)
{
    const unsigned *s = (const unsigned *)src;
    unsigned *d = (unsigned *)&dst;
    for (int i = threadIdx.x; i < (int)(sizeof(McTables) / 4); i += blockDim.x) d[i] = s[i];
    __syncthreads();
}

// Exclusive scan over the block of packed counts (triangles in the low 16
// bits, created vertices in the high 16); *total receives the block sum.
__device__ __forceinline__ unsigned block_scan(unsigned v, unsigned *s_warp, unsigned *total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        unsigned w = lane < kMcWarps ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < kMcWarps; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kMcWarps) s_warp[lane] = w;
    }
    __syncthreads();
    const unsigned base = wid > 0 ? s_warp[wid - 1] : 0u;
    *total = s_warp[kMcWarps - 1];
    __syncthreads();
    return base + x - v;
}

// Cube k of chunk `chunk`: slab s, chunk b in the slab, coordinates, index.
struct CubeRef {
    int s, b, z0, z1, gx, gy, gz;
    long long p;
    bool valid;
};

__device__ __forceinline__ CubeRef cube_at(const McGeom &g, int chunk, unsigned k)
{
    CubeRef r;
    r.s = chunk / g.nblk;
    r.b = chunk - r.s * g.nblk;
    slab_range(g, r.s, r.z0, r.z1);
    // cells < 2^27 (512^3): 32-bit unsigned index arithmetic
    const unsigned WH = (unsigned)g.W * (unsigned)g.H;
    const unsigned i = (unsigned)r.b * kMcThreads + k;
    r.valid = i < WH * (unsigned)(r.z1 - r.z0);
    const unsigned p = (unsigned)r.z0 * WH + (r.valid ? i : 0u);
    r.p = p;
    const unsigned gz = p / WH, rem = p - gz * WH, gy = rem / (unsigned)g.W;
    r.gz = (int)gz;
    r.gy = (int)gy;
    r.gx = (int)(rem - gy * (unsigned)g.W);
    return r;
}

// Cube threadIdx.x of chunk `chunk` (one cube per thread of a block).
__device__ __forceinline__ CubeRef cube_of(const McGeom &g, int chunk) { return cube_at(g, chunk, threadIdx.x); }

#ifndef LENIA_MC_COUNT_MINB
#define LENIA_MC_COUNT_MINB 3
#endif
// Per chunk (kMcThreads consecutive cubes of a slab) and channel: the
// chunk's triangle and created-vertex totals, packed as tri | vert << 32.
// One warp per chunk: lane l takes cubes l, l + 32, ... of it, walks each
// cube's channels in order (a vertex shared between channels belongs to the
// first channel that intersects its edge), writes the case indices and keeps
// its counts per channel; one warp reduction per channel at the end, so no
// block barrier waits on the slowest warp.
__global__ void __launch_bounds__(kMcThreads, LENIA_MC_COUNT_MINB) k_mc_count(McGeom g, const McTables *__restrict__ tab,
                                                        unsigned char *__restrict__ cases,
                                                        unsigned long long *__restrict__ blk)
{
    __shared__ McTables s_tab;
    load_tables(tab, s_tab);
    const int nchunks = g.slabs * g.nblk;
    const unsigned lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * kMcWarps;
    for (int chunk = blockIdx.x * kMcWarps + (int)(threadIdx.x >> 5); chunk < nchunks; chunk += nwarps) {
        // nt | nn << 16 per channel: a lane's 8 cubes and the warp's 256
        // (at most 5 triangles and 12 vertices per cube and field) fit
        unsigned packed[LENIA_MAX_CHANNELS] = {0u, 0u, 0u, 0u};
#pragma unroll 1
        for (unsigned j = 0; j < kMcThreads / 32; j++) {
            const CubeRef q = cube_at(g, chunk, j * 32 + lane);
            const unsigned owned = q.valid ? s_tab.owned[boundary_class(g, q.gx, q.gy, q.gz, q.z0, q.z1)] : 0u;
#pragma unroll 1
            for (int f = 0; f < g.F; f++) {
                // every channel's corners in flight at once, then the cases
                // in channel order
                float v[LENIA_MAX_CHANNELS][8];
#pragma unroll
                for (int c = 0; c < LENIA_MAX_CHANNELS; c++)
                    if (c < g.C && q.valid)
                        load_corners(g.fld[f] + c * g.N, g.halo[f] + c * g.N, g, q.gx, q.gy, q.gz, v[c]);
                unsigned prev = 0u;
#pragma unroll
                for (int c = 0; c < LENIA_MAX_CHANNELS; c++) {
                    if (c >= g.C) break;
                    int cs = 0;
                    if (q.valid) {
#pragma unroll
                        for (int i = 0; i < 8; i++) cs |= (v[c][i] > g.iso) << i;
                        cases[fc_off(g, f, c) + q.p] = (unsigned char)cs;
                    }
                    const unsigned act = s_tab.act[cs];
                    const unsigned nn = __popc(owned & act & ~prev);
                    if (g.share) prev |= act;
                    packed[c] += (unsigned)tri_count(s_tab.tri[cs]) | nn << 16;
                }
            }
        }
        const int s = chunk / g.nblk, b = chunk - s * g.nblk;
        unsigned long long mine = 0;
#pragma unroll
        for (int c = 0; c < LENIA_MAX_CHANNELS; c++) {
            const unsigned w = __reduce_add_sync(0xffffffffu, packed[c]);
            if (lane == (unsigned)c) mine = (unsigned long long)(w & 0xffffu) | (unsigned long long)(w >> 16) << 32;
        }
        if (lane < (unsigned)g.C) blk[((long long)s * g.C + lane) * g.nblk + b] = mine;
    }
}

// Exclusive scan of the M packed chunk totals in place, and the list of
// chunk-channels with triangles in order; totals[0..2] = triangles, vertices,
// listed chunk-channels.  Packed addition is exact while the triangle total
// stays below 2^32 (the host checks it).  Two launches over tiles of
// kScanTile values (each thread scans kScanPer consecutive values):
// k_mc_scan_tiles scans every tile on its own and lists its chunk-channels
// with triangles at the tile's slot of a scratch list; k_mc_scan_add adds
// the totals of the tiles before each tile and moves its list entries to
// their final places.
constexpr int kScanThreads = 1024;
constexpr int kScanPer = 8;
constexpr int kScanTile = kScanThreads * kScanPer;

__global__ void __launch_bounds__(kScanThreads) k_mc_scan_tiles(unsigned long long *__restrict__ blk, long long M,
                                                               unsigned long long *__restrict__ tile_tot,
                                                               long long *__restrict__ tile_cnt,
                                                               long long *__restrict__ list_tmp)
{
    __shared__ unsigned long long s_warp[kScanThreads / 32];
    __shared__ unsigned s_lwarp[kScanThreads / 32];
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    const long long base = (long long)blockIdx.x * kScanTile;
    const long long i0 = base + (long long)t * kScanPer;
    unsigned long long v[kScanPer];
#pragma unroll
    for (int j = 0; j < kScanPer; j++) v[j] = i0 + j < M ? blk[i0 + j] : 0ull;
    unsigned long long sum = 0;
    unsigned nz = 0;  // chunk-channels of this thread with triangles
#pragma unroll
    for (int j = 0; j < kScanPer; j++) {
        sum += v[j];
        nz += (v[j] & 0xffffffffull) != 0;
    }
    // inclusive warp scans of the thread sums and counts, then of the warp sums
    unsigned long long x = sum;
    unsigned xn = nz;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        const unsigned yn = __shfl_up_sync(0xffffffffu, xn, o);
        if (lane >= o) {
            x += y;
            xn += yn;
        }
    }
    if (lane == 31) {
        s_warp[wid] = x;
        s_lwarp[wid] = xn;
    }
    __syncthreads();
    if (wid == 0) {
        unsigned long long w = s_warp[lane];
        unsigned wn = s_lwarp[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
            const unsigned yn = __shfl_up_sync(0xffffffffu, wn, o);
            if (lane >= o) {
                w += y;
                wn += yn;
            }
        }
        s_warp[lane] = w;
        s_lwarp[lane] = wn;
    }
    __syncthreads();
    unsigned long long run = (wid > 0 ? s_warp[wid - 1] : 0ull) + x - sum;
    long long lrun = (long long)(wid > 0 ? s_lwarp[wid - 1] : 0u) + xn - nz;
#pragma unroll
    for (int j = 0; j < kScanPer; j++) {
        if (i0 + j < M) {
            blk[i0 + j] = run;
            if ((v[j] & 0xffffffffull) != 0) list_tmp[base + lrun++] = i0 + j;
        }
        run += v[j];
    }
    if (t == kScanThreads - 1) {
        tile_tot[blockIdx.x] = run;
        tile_cnt[blockIdx.x] = lrun;
    }
}

__global__ void __launch_bounds__(kScanThreads) k_mc_scan_add(unsigned long long *__restrict__ blk, long long M,
                                                             const unsigned long long *__restrict__ tile_tot,
                                                             const long long *__restrict__ tile_cnt,
                                                             const long long *__restrict__ list_tmp,
                                                             long long *__restrict__ list, long long *totals)
{
    __shared__ unsigned long long s_off;
    __shared__ long long s_loff;
    const int t = threadIdx.x, lane = t & 31;
    const int b = blockIdx.x;
    if (t < 32) {
        // the totals of the tiles before this one, in tile order per lane
        // (integer sums: the order does not change them)
        unsigned long long off = 0;
        long long loff = 0;
        for (int k = lane; k < b; k += 32) {
            off += tile_tot[k];
            loff += tile_cnt[k];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_down_sync(0xffffffffu, off, o);
            loff += __shfl_down_sync(0xffffffffu, loff, o);
        }
        if (lane == 0) {
            s_off = off;
            s_loff = loff;
            if (b == (int)gridDim.x - 1) {
                const unsigned long long all = off + tile_tot[b];
                totals[0] = (long long)(all & 0xffffffffull);
                totals[1] = (long long)(all >> 32);
                totals[2] = loff + tile_cnt[b];
            }
        }
    }
    __syncthreads();
    const unsigned long long off = s_off;
    const long long loff = s_loff, base = (long long)b * kScanTile;
    for (int k = t; k < kScanTile; k += kScanThreads)
        if (base + k < M) blk[base + k] += off;
    const long long n = tile_cnt[b];
    for (long long k = t; k < n; k += kScanThreads) list[loff + k] = list_tmp[base + k];
}

// Chunk-channel `o` of the listed ones: its channel c and chunk index (slab
// major), from o = (slab * C + c) * nblk + chunk-in-slab.
__device__ __forceinline__ void listed_chunk(const McGeom &g, unsigned o, int &c, int &chunk)
{
    const unsigned nb = (unsigned)g.nblk, sc = o / nb;
    c = (int)(sc % (unsigned)g.C);
    chunk = (int)((sc / (unsigned)g.C) * nb + (o - sc * nb));
}

// Triangles (face normals) and created vertices of the listed chunk-channels
// (the others' cubes are all case 0 or 255: no edge is cut there).  The
// blocks walk the list, whose length the scan left in totals[2], with stride
// gridDim.x.  Writes past the output capacity (cap_t triangles, cap_v
// vertices) are skipped: the host compares the totals with the capacity
// afterwards and runs the pass again into larger buffers.
__global__ void __launch_bounds__(kMcThreads) k_mc_emit(McGeom g, const McTables *__restrict__ tab,
                                                       const unsigned char *__restrict__ cases,
                                                       const unsigned long long *__restrict__ blk,
                                                       const long long *__restrict__ list,
                                                       const long long *__restrict__ totals,
                                                       int *__restrict__ tri_base, int *__restrict__ vert_base,
                                                       float *__restrict__ fn, float *__restrict__ pos,
                                                       int *__restrict__ vch, unsigned long long *__restrict__ vsrc,
                                                       long long cap_t, long long cap_v)
{
    __shared__ McTables s_tab;
    __shared__ unsigned s_warp[kMcWarps];
    const long long nlist = totals[2];
    if (blockIdx.x >= nlist) return;
    load_tables(tab, s_tab);
    for (long long li = blockIdx.x; li < nlist; li += gridDim.x) {
        const unsigned o = (unsigned)list[li];
        int c, chunk;
        listed_chunk(g, o, c, chunk);
        const CubeRef q = cube_of(g, chunk);
        const unsigned owned = q.valid ? s_tab.owned[boundary_class(g, q.gx, q.gy, q.gz, q.z0, q.z1)] : 0u;
        int cs[kMcMaxFields] = {0, 0, 0};
        unsigned newm[kMcMaxFields] = {0u, 0u, 0u};
        unsigned nt = 0, nn = 0;
#pragma unroll
        for (int f = 0; f < kMcMaxFields; f++) {
            if (f >= g.F) break;
            cs[f] = q.valid ? cases[fc_off(g, f, c) + q.p] : 0;
            // edges the cube's earlier channels cut (they own those vertices)
            unsigned prev = 0u;
            if (g.share && q.valid)
                for (int c2 = 0; c2 < c; c2++) prev |= s_tab.act[cases[fc_off(g, f, c2) + q.p]];
            const unsigned act = s_tab.act[cs[f]];
            newm[f] = owned & act & ~prev;
            nt += tri_count(s_tab.tri[cs[f]]);
            nn += __popc(newm[f]);
        }
        unsigned total;
        const unsigned pre = block_scan(nt | nn << 16, s_warp, &total);
        if (nt == 0) continue;
        long long tb = (long long)(blk[o] & 0xffffffffull) + (pre & 0xffff);
        long long vb = (long long)(blk[o] >> 32) + (pre >> 16);
#pragma unroll
        for (int f = 0; f < kMcMaxFields; f++) {
            if (f >= g.F) break;
            const unsigned long long tl = s_tab.tri[cs[f]];
            const int ntf = tri_count(tl);
            if (ntf == 0) continue;
            tri_base[fc_off(g, f, c) + q.p] = (int)tb;
            if (newm[f]) vert_base[fc_off(g, f, c) + q.p] = (int)vb;
            float v[8];
            load_corners(g.fld[f] + c * g.N, g.halo[f] + c * g.N, g, q.gx, q.gy, q.gz, v);
            for (int t = 0; t < ntf; t++) {
                if (tb + t >= cap_t) break;
                const float3 A = edge_vertex(g, f, s_tab.edge[slot_edge(tl, 3 * t)], v, q.gx, q.gy, q.gz);
                const float3 B = edge_vertex(g, f, s_tab.edge[slot_edge(tl, 3 * t + 1)], v, q.gx, q.gy, q.gz);
                const float3 C = edge_vertex(g, f, s_tab.edge[slot_edge(tl, 3 * t + 2)], v, q.gx, q.gy, q.gz);
                const float ux = B.x - A.x, uy = B.y - A.y, uz = B.z - A.z;
                const float wx = C.x - A.x, wy = C.y - A.y, wz = C.z - A.z;
                float *fo = fn + 3 * (tb + t);
                fo[0] = uy * wz - uz * wy;
                fo[1] = uz * wx - ux * wz;
                fo[2] = ux * wy - uy * wx;
            }
            if (newm[f]) {
                unsigned seen = 0;
                for (int k = 0; k < 3 * ntf; k++) {
                    const int e = slot_edge(tl, k);
                    if ((seen >> e) & 1) continue;
                    seen |= 1u << e;
                    if (!((newm[f] >> e) & 1)) continue;
                    if (vb < cap_v) {
                        const float3 P = edge_vertex(g, f, s_tab.edge[e], v, q.gx, q.gy, q.gz);
                        pos[3 * vb] = P.x;
                        pos[3 * vb + 1] = P.y;
                        pos[3 * vb + 2] = P.z;
                        vch[vb] = c + g.C * f;
                        vsrc[vb] = (unsigned long long)(fc_off(g, f, c) + q.p) << 4 | (unsigned)e;
                    }
                    vb++;
                }
            }
            tb += ntf;
        }
    }
}

// Creator of the vertex on local edge e of cube (gx, gy, gz): the first cube
// around the edge in scan order inside the slab.  Returns the creator's
// linear index, its coordinates and its local edge.
__device__ __forceinline__ long long edge_creator(const McGeom &g, const McTables &t, int e, int gx, int gy, int gz,
                                                  int z0, int z1, int *e_out, int &ox, int &oy, int &oz)
{
    const unsigned ed = t.edge[e];
    const int ax = (ed >> 6) & 3;
    const int Gx = gx + ((ed >> 8) & 1), Gy = gy + ((ed >> 9) & 1), Gz = gz + ((ed >> 10) & 1);
    for (int j = 0; j < 4; j++) {
        const int e2 = t.axis_edges[4 * ax + j];
        const unsigned d2 = t.edge[e2];
        const int x = Gx - (int)((d2 >> 8) & 1), y = Gy - (int)((d2 >> 9) & 1), z = Gz - (int)((d2 >> 10) & 1);
        if (x >= 0 && x < g.W && y >= 0 && y < g.H && z >= z0 && z < z1) {
            *e_out = e2;
            ox = x;
            oy = y;
            oz = z;
            return x + (long long)y * g.W + (long long)z * g.W * g.H;
        }
    }
    *e_out = e;  // unreachable: the cube itself is always a candidate
    ox = gx;
    oy = gy;
    oz = gz;
    return gx + (long long)gy * g.W + (long long)gz * g.W * g.H;
}

// Vertex indices of the listed chunk-channels' triangles (the blocks walk
// the list as in k_mc_emit; triangles past cap_t are skipped).
__global__ void __launch_bounds__(kMcThreads) k_mc_index(McGeom g, const McTables *__restrict__ tab,
                                                        const unsigned char *__restrict__ cases,
                                                        const int *__restrict__ tri_base,
                                                        const int *__restrict__ vert_base,
                                                        const long long *__restrict__ list,
                                                        const long long *__restrict__ totals,
                                                        unsigned *__restrict__ idx, long long cap_t)
{
    __shared__ McTables s_tab;
    const long long nlist = totals[2];
    if (blockIdx.x >= nlist) return;
    load_tables(tab, s_tab);
    for (long long li = blockIdx.x; li < nlist; li += gridDim.x) {
        int c, chunk;
        listed_chunk(g, (unsigned)list[li], c, chunk);
        const CubeRef q = cube_of(g, chunk);
        if (!q.valid) continue;
        for (int f = 0; f < g.F; f++) {
            const int cs = cases[fc_off(g, f, c) + q.p];
            const unsigned long long tl = s_tab.tri[cs];
            const int nt = tri_count(tl);
            if (nt == 0) continue;
            const long long tb = tri_base[fc_off(g, f, c) + q.p];
            if (tb + nt > cap_t) continue;
            for (int k = 0; k < 3 * nt; k++) {
                const int e = slot_edge(tl, k);
                // channel that created the vertex
                int c0 = c;
                if (g.share)
                    for (int c2 = 0; c2 < c; c2++)
                        if ((s_tab.act[cases[fc_off(g, f, c2) + q.p]] >> e) & 1) {
                            c0 = c2;
                            break;
                        }
                int eo, ox, oy, oz;
                const long long op = edge_creator(g, s_tab, e, q.gx, q.gy, q.gz, q.z0, q.z1, &eo, ox, oy, oz);
                const int ocs = cases[fc_off(g, f, c0) + op];
                unsigned oprev = 0;
                if (g.share)
                    for (int c2 = 0; c2 < c0; c2++) oprev |= s_tab.act[cases[fc_off(g, f, c2) + op]];
                const unsigned onew =
                    s_tab.owned[boundary_class(g, ox, oy, oz, q.z0, q.z1)] & s_tab.act[ocs] & ~oprev;
                // rank of eo among the creator's new vertices, in first-slot order
                const unsigned long long otl = s_tab.tri[ocs];
                unsigned seen = 0;
                int r = 0;
                for (int k2 = 0; k2 < 3 * tri_count(otl); k2++) {
                    const int e2 = slot_edge(otl, k2);
                    if ((seen >> e2) & 1) continue;
                    seen |= 1u << e2;
                    if (e2 == eo) break;
                    r += (onew >> e2) & 1;
                }
                idx[3 * tb + k] = (unsigned)(vert_base[fc_off(g, f, c0) + op] + r);
            }
        }
    }
}

__global__ void __launch_bounds__(kMcThreads) k_mc_normals(McGeom g, const McTables *__restrict__ tab,
                                                          const unsigned char *__restrict__ cases,
                                                          const int *__restrict__ tri_base,
                                                          const unsigned long long *__restrict__ vsrc,
                                                          const float *__restrict__ fn, float *__restrict__ nrm,
                                                          const long long *__restrict__ totals, long long cap_t,
                                                          long long cap_v)
{
    __shared__ McTables s_tab;
    // the vertex count the scan left in totals[1] (vertices past cap_v skipped)
    const long long nv = totals[1] < cap_v ? totals[1] : cap_v;
    if ((long long)blockIdx.x * blockDim.x >= nv) return;
    load_tables(tab, s_tab);
    const unsigned WH = (unsigned)g.W * (unsigned)g.H;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nv;
         v += (long long)gridDim.x * blockDim.x) {
        const unsigned long long src = vsrc[v];
        const int e0 = (int)(src & 15);
        // cube slots < F C N < 2^31: 32-bit unsigned index arithmetic
        const unsigned cp = (unsigned)(src >> 4);
        const unsigned fc0 = cp / (unsigned)g.N;
        const int f = (int)fc0 / g.C, c0 = (int)fc0 - f * g.C;
        const unsigned p0 = cp - fc0 * (unsigned)g.N;
        const unsigned uz = p0 / WH, rem = p0 - uz * WH, uy = rem / (unsigned)g.W;
        const int gz = (int)uz, gy = (int)uy, gx = (int)(rem - uy * (unsigned)g.W);
        int s = gz / (g.D / g.slabs);
        if (s > g.slabs - 1) s = g.slabs - 1;
        int z0, z1;
        slab_range(g, s, z0, z1);
        const unsigned ed = s_tab.edge[e0];
        const int ax = (ed >> 6) & 3;
        const int Gx = gx + ((ed >> 8) & 1), Gy = gy + ((ed >> 9) & 1), Gz = gz + ((ed >> 10) & 1);
        float nx = 0.0f, ny = 0.0f, nz = 0.0f;
        const int c_end = g.share ? g.C : c0 + 1;
        for (int c = c0; c < c_end; c++) {
            if (c > c0 && !((s_tab.act[cases[fc_off(g, f, c) + p0]] >> e0) & 1)) continue;
            for (int j = 0; j < 4; j++) {
                const int e2 = s_tab.axis_edges[4 * ax + j];
                const unsigned d2 = s_tab.edge[e2];
                const int x = Gx - (int)((d2 >> 8) & 1), y = Gy - (int)((d2 >> 9) & 1),
                          z = Gz - (int)((d2 >> 10) & 1);
                if (x < 0 || x >= g.W || y < 0 || y >= g.H || z < z0 || z >= z1) continue;
                const long long qp = x + (long long)y * g.W + (long long)z * WH;
                const unsigned long long tl = s_tab.tri[cases[fc_off(g, f, c) + qp]];
                const int nt = tri_count(tl);
                const long long tb = tri_base[fc_off(g, f, c) + qp];
                for (int t = 0; t < nt && tb + t < cap_t; t++) {
                    if (slot_edge(tl, 3 * t) == e2 || slot_edge(tl, 3 * t + 1) == e2 ||
                        slot_edge(tl, 3 * t + 2) == e2) {
                        const float *f = fn + 3 * (tb + t);
                        nx += f[0];
                        ny += f[1];
                        nz += f[2];
                    }
                }
            }
        }
        nrm[3 * v] = nx;
        nrm[3 * v + 1] = ny;
        nrm[3 * v + 2] = nz;
    }
}

// ---- host: the triangle table --------------------------------------------
//
// Polygons of a case: on each cube face the intersected edges pair into
// segments (two intersected edges: one segment; four: the face is ambiguous
// and each of its two inside corners, value > iso, is cut off by the segment
// between its two edges); the segments link into closed loops, each walked
// from its lowest edge towards the lower of that edge's two neighbours and
// cut into a fan of triangles from its first edge.  This resolves every
// ambiguous face the same way the reference's table does (same triangle
// count in all 256 cases).
int case_triangles(int cs, int *tri)
{
    int nb[12][2], deg[12] = {0};
    for (int ax = 0; ax < 3; ax++)
        for (int side = 0; side <= 1; side++) {
            int act[4], na = 0;
            for (int e = 0; e < 12; e++) {
                const int a = mc_a(e), b = mc_b(e);
                if (mc_coord(a, ax) == side && mc_coord(b, ax) == side && (((cs >> a) ^ (cs >> b)) & 1))
                    act[na++] = e;
            }
            int seg[2][2], ns = 0;
            if (na == 2) {
                seg[0][0] = act[0];
                seg[0][1] = act[1];
                ns = 1;
            } else if (na == 4) {
                for (int k = 0; k < 8; k++) {
                    if (mc_coord(k, ax) != side || !((cs >> k) & 1)) continue;
                    int m = 0;
                    for (int i = 0; i < 4; i++)
                        if (mc_a(act[i]) == k || mc_b(act[i]) == k) seg[ns][m++] = act[i];
                    ns++;
                }
            }
            for (int i = 0; i < ns; i++) {
                const int a = seg[i][0], b = seg[i][1];
                nb[a][deg[a]++] = b;
                nb[b][deg[b]++] = a;
            }
        }
    bool visited[12] = {false};
    int nt = 0;
    for (int s = 0; s < 12; s++) {
        if (deg[s] == 0 || visited[s]) continue;
        int loop[12], n = 0, prev = -1, cur = s;
        for (;;) {
            loop[n++] = cur;
            visited[cur] = true;
            const int nx = prev < 0 ? (nb[cur][0] < nb[cur][1] ? nb[cur][0] : nb[cur][1])
                                    : (nb[cur][0] == prev ? nb[cur][1] : nb[cur][0]);
            if (nx == s) break;
            prev = cur;
            cur = nx;
        }
        for (int i = 1; i + 1 < n; i++) {
            tri[3 * nt] = loop[0];
            tri[3 * nt + 1] = loop[i];
            tri[3 * nt + 2] = loop[i + 1];
            nt++;
        }
    }
    return nt;
}

// The edges a cube creates, per boundary class: those whose first
// neighbouring cube in scan order (inside the slab) is this cube.
unsigned short owned_edges(int cls)
{
    const bool lo[3] = {(cls & 1) != 0, (cls & 4) != 0, (cls & 16) != 0};
    const bool hi[3] = {(cls & 2) != 0, (cls & 8) != 0, (cls & 32) != 0};
    unsigned short m = 0;
    for (int e = 0; e < 12; e++) {
        const int ax = mc_axis(e);
        for (int j = 0; j < 4; j++) {
            const int e2 = mc_axis_edge(ax, j);
            bool ok = true;
            for (int d = 0; d < 3; d++) {
                const int delta = mc_off(e, d) - mc_off(e2, d);  // neighbour = this cube + delta
                if ((delta < 0 && lo[d]) || (delta > 0 && hi[d])) ok = false;
            }
            if (ok) {
                if (e2 == e) m |= (unsigned short)(1u << e);
                break;
            }
        }
    }
    return m;
}

void build_tables(McTables *t)
{
    memset(t, 0, sizeof(*t));
    for (int cs = 0; cs < 256; cs++) {
        int tri[15];
        const int n = case_triangles(cs, tri);
        unsigned long long w = (unsigned long long)n << 60;
        for (int k = 0; k < 3 * n; k++) w |= (unsigned long long)tri[k] << (4 * k);
        t->tri[cs] = w;
    }
    for (int cls = 0; cls < 64; cls++) t->owned[cls] = owned_edges(cls);
    for (int cs = 0; cs < 256; cs++) t->act[cs] = (unsigned short)active_edges(cs);
    for (int e = 0; e < 12; e++) t->edge[e] = mc_edge_desc(e);
    for (int ax = 0; ax < 3; ax++)
        for (int j = 0; j < 4; j++) t->axis_edges[4 * ax + j] = (unsigned char)mc_axis_edge(ax, j);
}

}  // namespace

struct lenia_mesher {
    LeniaMeshDesc desc;
    McGeom g;
    int device = 0;
    int grid = 0;
    int list_grid = 0;
    std::string err;
    McTables *tab = nullptr;
    unsigned char *cases = nullptr;
    int *tri_base = nullptr, *vert_base = nullptr;
    unsigned long long *blk = nullptr;  // per chunk and channel: tri | vert << 32, then its exclusive scan
    long long *list = nullptr;          // chunk-channels with triangles, in order
    long long *list_tmp = nullptr;      // the same per scan tile (at the tile's first slot)
    unsigned long long *tile_tot = nullptr;  // per scan tile: its packed total
    long long *tile_cnt = nullptr;           // per scan tile: its listed chunk-channels
    long long *totals = nullptr, *h_totals = nullptr;
    float *fn = nullptr, *pos = nullptr, *nrm = nullptr;
    int *vch = nullptr;
    unsigned long long *vsrc = nullptr;
    unsigned *idx = nullptr;
    long long cap_t = 0, cap_v = 0, n_t = 0, n_v = 0;
    bool have_mesh = false;
    cudaStream_t stream = nullptr;
};

namespace {

lenia_status mfail(lenia_mesher *m, lenia_status s, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (m) m->err = buf;
    return s;
}

lenia_status mcuda(lenia_mesher *m, cudaError_t e, const char *where)
{
    return mfail(m, e == cudaErrorMemoryAllocation ? LENIA_ERR_OOM : LENIA_ERR_CUDA, "%s: %s", where,
                 cudaGetErrorString(e));
}

template <typename T>
void dfree(T *&p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

void free_outputs(lenia_mesher *m)
{
    dfree(m->fn);
    dfree(m->idx);
    dfree(m->pos);
    dfree(m->nrm);
    dfree(m->vch);
    dfree(m->vsrc);
    m->cap_t = m->cap_v = 0;
}

// Output buffers for ct triangles and cv vertices (the old ones freed).
cudaError_t alloc_outputs(lenia_mesher *m, long long ct, long long cv)
{
    free_outputs(m);
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->fn, sizeof(float) * 3 * ct);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->idx, sizeof(unsigned) * 3 * ct);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->pos, sizeof(float) * 3 * cv);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->nrm, sizeof(float) * 3 * cv);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->vch, sizeof(int) * cv);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->vsrc, sizeof(unsigned long long) * cv);
    if (e != cudaSuccess) {
        free_outputs(m);
        return e;
    }
    m->cap_t = ct;
    m->cap_v = cv;
    return cudaSuccess;
}

}  // namespace

namespace lenia {
long long mesher_field_floats(const lenia_mesher *m) { return m ? (long long)m->g.C * m->g.N : 0; }
int mesher_fields(const lenia_mesher *m) { return m ? m->g.F : 0; }
}  // namespace lenia

namespace {

// The six launches of one mesh and its one host synchronisation.
lenia_status mesher_run(lenia_mesher *m, cudaStream_t st, long long *n_vertices, long long *n_triangles)
{
    McGeom &g = m->g;
    m->stream = st;
    m->have_mesh = false;
    const long long M = (long long)g.slabs * g.nblk * g.C;
    k_mc_count<<<m->grid, kMcThreads, 0, st>>>(g, m->tab, m->cases, m->blk);
    const unsigned ntiles = (unsigned)((M + kScanTile - 1) / kScanTile);
    k_mc_scan_tiles<<<ntiles, kScanThreads, 0, st>>>(m->blk, M, m->tile_tot, m->tile_cnt, m->list_tmp);
    k_mc_scan_add<<<ntiles, kScanThreads, 0, st>>>(m->blk, M, m->tile_tot, m->tile_cnt, m->list_tmp, m->list,
                                                    m->totals);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return mcuda(m, e, "mesher count");
    // The output passes take their counts from the scan's totals on the
    // device, so they follow it without a host round trip; they write only
    // what fits the current buffers, and run again into larger ones when
    // the totals read afterwards do not fit.
    auto outputs = [&]() -> cudaError_t {
        k_mc_emit<<<m->list_grid, kMcThreads, 0, st>>>(g, m->tab, m->cases, m->blk, m->list, m->totals, m->tri_base,
                                                       m->vert_base, m->fn, m->pos, m->vch, m->vsrc, m->cap_t,
                                                       m->cap_v);
        k_mc_index<<<m->list_grid, kMcThreads, 0, st>>>(g, m->tab, m->cases, m->tri_base, m->vert_base, m->list,
                                                        m->totals, m->idx, m->cap_t);
        k_mc_normals<<<m->list_grid, kMcThreads, 0, st>>>(g, m->tab, m->cases, m->tri_base, m->vsrc, m->fn, m->nrm,
                                                          m->totals, m->cap_t, m->cap_v);
        return cudaGetLastError();
    };
    e = outputs();
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->h_totals, m->totals, 3 * sizeof(long long), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return mcuda(m, e, "mesher passes");
    const long long nt = m->h_totals[0], nv = m->h_totals[1];
    if (3 * nt > 0xffffffffLL || nv > 0x7fffffffLL)
        return mfail(m, LENIA_ERR_UNSUPPORTED, "mesh of %lld triangles exceeds 32-bit indices", nt);
    if (nt > m->cap_t || nv > m->cap_v) {
        const long long ct = nt > m->cap_t ? nt + nt / 4 + 1024 : m->cap_t;
        const long long cv = nv > m->cap_v ? nv + nv / 4 + 1024 : m->cap_v;
        if ((e = alloc_outputs(m, ct, cv)) != cudaSuccess) return mcuda(m, e, "mesher buffers");
        e = outputs();
        if (e != cudaSuccess) return mcuda(m, e, "mesher passes");
    }
    m->n_t = nt;
    m->n_v = nv;
    m->have_mesh = true;
    if (n_vertices) *n_vertices = nv;
    if (n_triangles) *n_triangles = nt;
    return LENIA_OK;
}

}  // namespace

extern "C" {

int lenia_mc_triangle_table(int *table)
{
    if (!table) return -1;
    for (int cs = 0; cs < 256; cs++) {
        int tri[15];
        const int n = case_triangles(cs, tri);
        for (int k = 0; k < 16; k++) table[cs * 16 + k] = k < 3 * n ? tri[k] : -1;
    }
    return 0;
}

lenia_status lenia_mesh_desc_for_view(int view, int width, int height, int channels, float iso_value,
                                      LeniaMeshDesc *out)
{
    if (!out || view < LENIA_VIEW_NORMAL || view > LENIA_VIEW_H) return LENIA_ERR_INVALID_ARG;
    memset(out, 0, sizeof(*out));
    out->width = width;
    out->height = height;
    out->channels = channels;
    out->fields = view + 1;
    out->iso_value = iso_value;
    out->cell_size = 3.5f;  // CELL_SIZE, render.h:26
    // GRID_WIDTH * CELL_SIZE, the shift of the second and third meshes
    const float shift = (float)width * 3.5f;
    if (view >= LENIA_VIEW_U) out->offset[1][0] = shift;
    if (view == LENIA_VIEW_H) out->offset[2][2] = shift;
    out->slabs = 2;          // MESH_THREADS, render.h:15
    out->share_channels = 1;
    return LENIA_OK;
}

lenia_status lenia_mesher_create(const LeniaMeshDesc *desc, lenia_mesher **out)
{
    if (!desc || !out) return LENIA_ERR_INVALID_ARG;
    *out = nullptr;
    const LeniaMeshDesc &d = *desc;
    if (d.width < 2 || d.width > kMcMaxDim || d.height < 2 || d.height > kMcMaxDim || d.channels < 1 ||
        d.channels > LENIA_MAX_CHANNELS || d.fields < 1 || d.fields > kMcMaxFields || d.slabs < 1 ||
        d.slabs > d.width || !(d.cell_size > 0.0f))
        return LENIA_ERR_INVALID_ARG;
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return LENIA_ERR_NO_DEVICE;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return LENIA_ERR_NO_DEVICE;
    lenia_mesher *m = new lenia_mesher();
    m->desc = d;
    m->device = dev;
    McGeom &g = m->g;
    g.W = d.width;
    g.H = d.height;
    g.D = d.width;
    g.C = d.channels;
    g.F = d.fields;
    g.N = (long long)g.W * g.H * g.D;
    g.slabs = d.slabs;
    const long long largest = (long long)g.W * g.H * (g.D - (g.D / g.slabs) * (g.slabs - 1));
    g.nblk = (int)((largest + kMcThreads - 1) / kMcThreads);
    g.share = d.share_channels != 0;
    g.iso = d.iso_value;
    g.cell = d.cell_size;
    for (int f = 0; f < kMcMaxFields; f++)
        for (int a = 0; a < 3; a++) g.off[f][a] = f < g.F ? d.offset[f][a] : 0.0f;
    const long long nchunks = (long long)g.slabs * g.nblk;
    // one warp per chunk, up to six blocks of eight warps per SM
    const long long count_blocks = (nchunks + kMcWarps - 1) / kMcWarps;
    m->grid = (int)(count_blocks < 6LL * nsm ? count_blocks : 6LL * nsm);
    const long long M = nchunks * g.C;
    // the output passes: blocks that walk the listed chunk-channels (and
    // the vertices) with a stride, eight per SM
    m->list_grid = (int)(M < 8LL * nsm ? M : 8LL * nsm);
    McTables host;
    build_tables(&host);
    cudaError_t e = cudaSuccess;
    auto alloc = [&](auto *&p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc((void **)&p, bytes);
    };
    alloc(m->tab, sizeof(McTables));
    const size_t cubes = (size_t)g.F * g.C * g.N;
    alloc(m->cases, cubes);
    alloc(m->tri_base, sizeof(int) * cubes);
    alloc(m->vert_base, sizeof(int) * cubes);
    alloc(m->blk, sizeof(unsigned long long) * (size_t)M);
    alloc(m->list, sizeof(long long) * (size_t)M);
    alloc(m->list_tmp, sizeof(long long) * (size_t)M);
    const size_t ntiles = (size_t)((M + kScanTile - 1) / kScanTile);
    alloc(m->tile_tot, sizeof(unsigned long long) * ntiles);
    alloc(m->tile_cnt, sizeof(long long) * ntiles);
    alloc(m->totals, 3 * sizeof(long long));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&m->h_totals, 3 * sizeof(long long));
    if (e == cudaSuccess) e = cudaMemcpy(m->tab, &host, sizeof(McTables), cudaMemcpyHostToDevice);
    // first output buffers: one triangle and one vertex per 32 cube slots
    // (at most 2^20 each, 60 MB), so that a first mesh rarely runs its
    // output passes twice; a larger mesh grows them
    if (e == cudaSuccess) {
        const long long first = std::min<long long>(std::max<long long>(cubes / 32, 4096), 1LL << 20);
        e = alloc_outputs(m, first, first);
    }
    if (e != cudaSuccess) {
        lenia_mesher_destroy(m);
        return e == cudaErrorMemoryAllocation ? LENIA_ERR_OOM : LENIA_ERR_CUDA;
    }
    *out = m;
    return LENIA_OK;
}

lenia_status lenia_mesher_destroy(lenia_mesher *m)
{
    if (!m) return LENIA_ERR_INVALID_ARG;
    // cudaFree waits for the device; the last run's stream may be gone already
    free_outputs(m);
    dfree(m->tab);
    dfree(m->cases);
    dfree(m->tri_base);
    dfree(m->vert_base);
    dfree(m->blk);
    dfree(m->list);
    dfree(m->list_tmp);
    dfree(m->tile_tot);
    dfree(m->tile_cnt);
    dfree(m->totals);
    if (m->h_totals) cudaFreeHost(m->h_totals);
    delete m;
    return LENIA_OK;
}

lenia_status lenia_mesher_run(lenia_mesher *m, const float *const *fields, const float *const *halos, void *stream,
                              long long *n_vertices, long long *n_triangles)
{
    if (!m || !fields) return LENIA_ERR_INVALID_ARG;
    McGeom &g = m->g;
    for (int f = 0; f < kMcMaxFields; f++) {
        if (f < g.F && !fields[f]) return mfail(m, LENIA_ERR_INVALID_ARG, "field %d is NULL", f);
        g.fld[f] = f < g.F ? fields[f] : nullptr;
        g.halo[f] = f < g.F ? (halos && halos[f] ? halos[f] : fields[f]) : nullptr;
    }
    cudaStream_t st = (cudaStream_t)stream;
    nvtxRangePushA("lenia_mesher_run");
    const lenia_status s = mesher_run(m, st, n_vertices, n_triangles);
    nvtxRangePop();
    return s;
}

lenia_status lenia_mesher_get(lenia_mesher *m, int which, void *dst, size_t count, int on_device)
{
    if (!m || !dst) return LENIA_ERR_INVALID_ARG;
    if (!m->have_mesh) return mfail(m, LENIA_ERR_INVALID_ARG, "no mesh: run the mesher first");
    const void *src = nullptr;
    size_t n = 0, elem = 4;
    switch (which) {
    case LENIA_MESH_POSITIONS: src = m->pos; n = 3 * (size_t)m->n_v; break;
    case LENIA_MESH_NORMALS: src = m->nrm; n = 3 * (size_t)m->n_v; break;
    case LENIA_MESH_VERTEX_CHANNEL: src = m->vch; n = (size_t)m->n_v; break;
    case LENIA_MESH_INDICES: src = m->idx; n = 3 * (size_t)m->n_t; break;
    case LENIA_MESH_FACE_NORMALS: src = m->fn; n = 3 * (size_t)m->n_t; break;
    case LENIA_MESH_CASES: src = m->cases; n = (size_t)m->g.F * m->g.C * m->g.N; elem = 1; break;
    default: return mfail(m, LENIA_ERR_INVALID_ARG, "unknown mesh array %d", which);
    }
    if (count != n) return mfail(m, LENIA_ERR_INVALID_ARG, "mesh array %d holds %zu elements, got %zu", which, n, count);
    if (n == 0) return LENIA_OK;
    cudaError_t e = cudaMemcpyAsync(dst, src, n * elem, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                    m->stream);
    if (e == cudaSuccess && !on_device) e = cudaStreamSynchronize(m->stream);
    if (e != cudaSuccess) return mcuda(m, e, "mesher get");
    return LENIA_OK;
}

const char *lenia_mesher_last_error(const lenia_mesher *m) { return m ? m->err.c_str() : "null mesher"; }

}  // extern "C"
