// Transport stage of the 3D Flow Lenia step, fused into one kernel: the
// events REINTEGRATION and TRM of render.cpp:550-569.
//   reintegration_step (lenia.cpp:727-918): srt, rt_border_torus,
//     rt_border_other, adv_vel, adv_f (reintegration.cpp:607-1410) written as
//     a destination gather per cell, then the oscillators;
//   halo cells as transpose_borders leaves them (transposition.cpp:671-876):
//     (int)dd periodic layers on faces, edges and corners 0;
//   transpose_to_row_major (lenia.cpp:924-1037): growth or clamp, the moving
//     averages GA and SUM, the new grid (written to a second buffer: the
//     gather reads the old one).
// Float operation order and rounding are the reference's (-fmad=false).
#include "lenia_internal.h"
#include "growth_common.cuh"
#include "tma.cuh"
#include "async_copy.cuh"

namespace lenia {

__device__ __forceinline__ float tmax(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float tmin(float a, float b) { return a < b ? a : b; }

// Value of a transported field at (x, y, z), the reference's halo rules.
__device__ __forceinline__ float tb_read(const float *f, const Dims &d, int dd, int x, int y, int z)
{
    const int ox = (x < 0) | (x >= d.W), oy = (y < 0) | (y >= d.H), oz = (z < 0) | (z >= d.D);
    const int no = ox + oy + oz;
    if (no == 0) return __ldg(f + x + (long long)y * d.W + (long long)z * d.W * d.H);
    if (no > 1) return 0.0f;
    if (x < -dd || x >= d.W + dd || y < -dd || y >= d.H + dd || z < -dd || z >= d.D + dd) return 0.0f;
    x = x < 0 ? x + d.W : (x >= d.W ? x - d.W : x);
    y = y < 0 ? y + d.H : (y >= d.H ? y - d.H : y);
    z = z < 0 ? z + d.D : (z >= d.D ? z - d.D : z);
    return __ldg(f + x + (long long)y * d.W + (long long)z * d.W * d.H);
}

__device__ __forceinline__ float torus_wrap(float m, int ext)
{
    const float half = (float)(ext / 2);
    if (m > half) m = m - (float)ext;
    if (m < -half) m = m + (float)ext;
    return m;
}

// Oscillators (lenia.cpp:803-911) and transpose_to_row_major
// (lenia.cpp:924-1037) for one destination cell; tt holds its reintegrated
// mass per channel.  ga_pre, when not null, holds the cell's GA per channel
// (stride ga_stride) already copied to shared memory; else GA is read here.
__device__ __forceinline__ void transport_epilogue(const StepParams &p, const TransportBuffers &b, float *tt, int x,
                                                   int y, int z, long long i, const float *ga_pre = nullptr,
                                                   int ga_stride = 0)
{
    const Dims &d = p.d;
    const long long N = d.N;
    const int C = p.C;
    const int dd = p.dd;
    if (p.osc_la || p.osc_flow || p.osc_div_flow) {
        const float *fl = p.osc_vel ? b.V : b.F;
#pragma unroll
        for (int c = 0; c < kMaxChannels; c++) {
            if (c >= C) continue;
            const float *g = b.A + (long long)c * N;
            const float fx1 = tb_read(g, d, dd, x + 1, y, z), fx0 = tb_read(g, d, dd, x - 1, y, z);
            const float fy1 = tb_read(g, d, dd, x, y + 1, z), fy0 = tb_read(g, d, dd, x, y - 1, z);
            const float fz1 = tb_read(g, d, dd, x, y, z + 1), fz0 = tb_read(g, d, dd, x, y, z - 1);
            const float dxv = fx1 - fx0, dyv = fy1 - fy0, dzv = fz1 - fz0;
            float t = tt[c];
            if (p.osc_la) {
                const float la = fx1 + fx0 + fy1 + fy0 + fz1 + fz0 - 6 * __ldg(g + i);
                t = t + la * p.osc_la_amt;
            }
            if (p.osc_flow) {
                const float flow = __ldg(fl + (long long)c * N + i) * dxv + __ldg(fl + (long long)(C + c) * N + i) * dyv +
                                   __ldg(fl + (long long)(2 * C + c) * N + i) * dzv;
                t = t + flow * p.osc_flow_amt;
            }
            if (p.osc_div_flow) {
                const float *fxs = fl + (long long)c * N, *fys = fl + (long long)(C + c) * N,
                            *fzs = fl + (long long)(2 * C + c) * N;
                const float *al = b.ALPHA + (long long)c * N;
                const float jx = tb_read(fxs, d, dd, x + 1, y, z) * tb_read(al, d, dd, x + 1, y, z) -
                                 tb_read(fxs, d, dd, x - 1, y, z) * tb_read(al, d, dd, x - 1, y, z);
                const float jy = tb_read(fys, d, dd, x, y + 1, z) * tb_read(al, d, dd, x, y + 1, z) -
                                 tb_read(fys, d, dd, x, y - 1, z) * tb_read(al, d, dd, x, y - 1, z);
                const float jz = tb_read(fzs, d, dd, x, y, z + 1) * tb_read(al, d, dd, x, y, z + 1) -
                                 tb_read(fzs, d, dd, x, y, z - 1) * tb_read(al, d, dd, x, y, z - 1);
                const float divj = jx + jy + jz;
                t = t + divj * p.osc_div_flow_amt;
            }
            tt[c] = t;
        }
    }
    if (b.TT)
#pragma unroll
        for (int c = 0; c < kMaxChannels; c++)
            if (c < C) b.TT[(long long)c * N + i] = tt[c];

    // transpose_to_row_major
    if (p.growth_type == kGrowthTransposition) {
#pragma unroll
        for (int c = 0; c < kMaxChannels; c++) {
            if (c >= C) continue;
            const long long ci = (long long)c * N + i;
            const float h = __ldg(b.H + ci);
            if (p.soft_clip[c]) {
                float v = __ldg(b.A + ci) + h * p.timestep;
                v = -4.0f * (v - 0.5f);
                v = fastexp_dev(v);
                v = 1.0f + v;
                v = 1.0f / v;
                b.BACK[ci] = tmin(tmax(v, 0.0f), 1.0f);
            } else {
                tt[c] = tmin(tmax(tt[c] + h * p.timestep, 0.0f), 1.0f);
            }
        }
    } else {
#pragma unroll
        for (int c = 0; c < kMaxChannels; c++)
            if (c < C) tt[c] = tmin(tmax(tt[c], 0.0f), 1.0f);
    }
    const float stam = 1.0f - p.sta, stas = p.sta, gtas = p.gta, gtam = 1.0f - p.gta;
    float ttsum = 0.0f;
#pragma unroll
    for (int c = 0; c < kMaxChannels; c++) {
        if (c >= C) continue;
        const long long ci = (long long)c * N + i;
        ttsum = ttsum + tt[c];
        const float ga = ga_pre ? ga_pre[c * ga_stride] : b.GA[ci];
        b.GA[ci] = gtam * ga + tt[c] * gtas;
        b.A_out[ci] = tt[c];
    }
    // SUM was cleared at the end of reintegration (lenia.cpp:912-915)
    b.SUM[i] = stam * 0.0f + ttsum * stas;
}

__device__ __forceinline__ void transport_cell_body(const StepParams &p, const TransportBuffers &b, long long block)
{
    const Dims &d = p.d;
    const long long N = d.N;
    const long long i = block * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int C = p.C;
    // N < 2^31 (at most 256^3 cells): the cell's coordinates by two 32-bit divisions
    const unsigned ui = (unsigned)i, plane = (unsigned)d.W * (unsigned)d.H;
    const unsigned uz = ui / plane, rem = ui - uz * plane, uy = rem / (unsigned)d.W;
    const int x = (int)(rem - uy * (unsigned)d.W), y = (int)uy, z = (int)uz;
    const float px = (float)x + 0.5f, py = (float)y + 0.5f, pz = (float)z + 0.5f;
    const int dd = p.dd;
    float tt[kMaxChannels];
#pragma unroll
    for (int c = 0; c < kMaxChannels; c++) tt[c] = 0.0f;

    if (p.mode_type == kModeSRT || p.mode_type == kModeRT) {
        const int crt = p.rt_all_channels ? C : (C < 3 ? C : 3);
        const bool torus = p.border == kBorderTorus;
        for (int c = 0; c < crt; c++) {
            const float *mux = b.MU + (long long)c * N;
            const float *muy = b.MU + (long long)(C + c) * N;
            const float *muz = b.MU + (long long)(2 * C + c) * N;
            const float *arr = b.ARR + (long long)c * N;
            float acc = 0.0f;
            if (p.mode_type == kModeSRT) {
                float mx = fabsf(px - __ldg(mux + i)), my = fabsf(py - __ldg(muy + i)), mz = fabsf(pz - __ldg(muz + i));
                mx = tmin(tmax(p.si - mx, 0.0f), p.clip);
                my = tmin(tmax(p.si - my, 0.0f), p.clip);
                mz = tmin(tmax(p.si - mz, 0.0f), p.clip);
                float w = __ldg(arr + i) * mx;
                w = w * my;
                w = w * mz;
                w = w * p.sn;
                acc = acc + w;
            } else {
                for (int oz = -dd; oz <= dd; oz++)
                    for (int oy = -dd; oy <= dd; oy++)
                        for (int ox = -dd; ox <= dd; ox++) {
                            const int sx = x + ox, sy = y + oy, sz = z + oz;
                            float mx = px - tb_read(mux, d, dd, sx, sy, sz);
                            float my = py - tb_read(muy, d, dd, sx, sy, sz);
                            float mz = pz - tb_read(muz, d, dd, sx, sy, sz);
                            if (torus) {
                                mx = torus_wrap(mx, d.W);
                                my = torus_wrap(my, d.H);
                                mz = torus_wrap(mz, d.D);
                            }
                            mx = fabsf(mx);
                            my = fabsf(my);
                            mz = fabsf(mz);
                            mx = p.si - mx;
                            my = p.si - my;
                            mz = p.si - mz;
                            mx = tmax(mx, 0.0f);
                            my = tmax(my, 0.0f);
                            mz = tmax(mz, 0.0f);
                            mx = tmin(mx, p.clip);
                            my = tmin(my, p.clip);
                            mz = tmin(mz, p.clip);
                            float w = tb_read(arr, d, dd, sx, sy, sz) * mx;
                            w = w * my;
                            w = w * mz;
                            w = w * p.sn;
                            acc = acc + w;
                        }
            }
            tt[c] = acc;
        }
    } else if (p.mode_type == kModeADV) {
        const float *vel = p.adv_vel ? b.V : b.F;
        const float ext[3] = {(float)d.W, (float)d.H, (float)d.W};
        const float pos[3] = {px, py, pz};
        // With |ma| < 1, X = (pos - 0.5) - v + ext lies in (ext - 1, 2 ext):
        // floorf(X / ext) is 1 exactly when X >= ext (a float X below ext gives
        // a quotient at most 1 - 2^-24, and X / ext < 2 - 2^-9 for ext <= 256),
        // so the comparison replaces the division with the same result.
        const bool one_wrap = fabsf(p.ma) < 1.0f;
        for (int c = 0; c < C; c++) {
            int i0[3];
            float fr[3];
#pragma unroll
            for (int q = 0; q < 3; q++) {
                float v = __ldg(vel + (long long)(q * C + c) * N + i) * p.timestep;
                v = tmin(tmax(v, -p.ma), p.ma);
                float X = (pos[q] - 0.5f) - v;
                X = X + ext[q];
                const float k = one_wrap ? (X >= ext[q] ? 1.0f : 0.0f) : floorf(X / ext[q]);
                X = X - k * ext[q];
                const float X0 = floorf(X);
                i0[q] = (int)X0;
                fr[q] = X - X0;
            }
            const float *arr = b.ARR + (long long)c * N;
            const float fx = fr[0], fy = fr[1], fz = fr[2];
            const float nfx = 1.0f - fx, nfy = 1.0f - fy, nfz = 1.0f - fz;
            const int x0 = i0[0], y0 = i0[1], z0 = i0[2];
            float a[8];
            if (x0 >= 0 && y0 >= 0 && z0 >= 0 && x0 + 1 < d.W && y0 + 1 < d.H && z0 + 1 < d.D) {
                // all eight corners inside the grid: plain loads
                const float *q0 = arr + x0 + (long long)y0 * d.W + (long long)z0 * d.W * d.H;
                const long long sy = d.W, sz = (long long)d.W * d.H;
                a[0] = __ldg(q0);
                a[1] = __ldg(q0 + 1);
                a[2] = __ldg(q0 + sy);
                a[3] = __ldg(q0 + sy + 1);
                a[4] = __ldg(q0 + sz);
                a[5] = __ldg(q0 + sz + 1);
                a[6] = __ldg(q0 + sz + sy);
                a[7] = __ldg(q0 + sz + sy + 1);
            } else {
                a[0] = tb_read(arr, d, dd, x0, y0, z0);
                a[1] = tb_read(arr, d, dd, x0 + 1, y0, z0);
                a[2] = tb_read(arr, d, dd, x0, y0 + 1, z0);
                a[3] = tb_read(arr, d, dd, x0 + 1, y0 + 1, z0);
                a[4] = tb_read(arr, d, dd, x0, y0, z0 + 1);
                a[5] = tb_read(arr, d, dd, x0 + 1, y0, z0 + 1);
                a[6] = tb_read(arr, d, dd, x0, y0 + 1, z0 + 1);
                a[7] = tb_read(arr, d, dd, x0 + 1, y0 + 1, z0 + 1);
            }
            float s = a[0] * nfx * nfy * nfz;
            s = s + a[1] * fx * nfy * nfz;
            s = s + a[2] * nfx * fy * nfz;
            s = s + a[3] * fx * fy * nfz;
            s = s + a[4] * nfx * nfy * fz;
            s = s + a[5] * fx * nfy * fz;
            s = s + a[6] * nfx * fy * fz;
            s = s + a[7] * fx * fy * fz;
            tt[c] = s;
        }
    }

    transport_epilogue(p, b, tt, x, y, z, i);
}

__global__ void __launch_bounds__(256) k_transport(const __grid_constant__ StepParams p,
                                                   const __grid_constant__ TransportBuffers b)
{
    transport_cell_body(p, b, blockIdx.x);
}

// ------------------------------------------------------------------
// RT / SRT as a tiled destination gather.  A block owns 32 x 8 x TZ cells
// (thread = one x, y column of TZ cells).  Per channel one thread copies MU
// and ARR of the block's cells plus a DD-cell halo into shared memory with
// four TMA tensor loads (zero outside the grid; double buffered across
// channels); blocks on the grid boundary then patch the DD periodic face
// layers (transpose_borders copies them whatever the border setting; edges
// and corners stay 0).  The thread walks the source layers z' upward: the x
// and y overlap factors of a source depend only on the thread's column, so
// they are computed once and reused for the (up to 2 DD + 1) destinations of
// the column that the source reaches.  Each destination still receives its
// contributions in the reference's (dz, dy, dx) order, with the reference's
// float operations, so the result is bit-identical.
constexpr int kTX = 32, kTY = 8, kTZ = 4;
constexpr int kTBoxX = 40;  // staged x range x0 - 4 .. x0 + 35 (TMA x must be 16-byte aligned)

// min(max(si - |d|, 0), clip).  With clip == 1 the clamp is a saturating
// add: identical for every input (NaN and negative values give +0 either
// way, and a -0 factor cannot change the accumulated sum).
template <bool TORUS, bool CLIP1>
__device__ __forceinline__ float overlap(float d, float si, float clip, int ext)
{
    if (TORUS) d = torus_wrap(d, ext);
    d = fabsf(d);
    if (CLIP1) return __saturatef(si - d);
    d = si - d;
    d = tmax(d, 0.0f);
    d = tmin(d, clip);
    return d;
}

// Source of a halo cell under the transported-field rules; false when the
// cell reads 0 (edges, corners, layers past dd).
__device__ __forceinline__ bool tb_source(const Dims &d, int dd, int &x, int &y, int &z)
{
    const int ox = (x < 0) | (x >= d.W), oy = (y < 0) | (y >= d.H), oz = (z < 0) | (z >= d.D);
    const int no = ox + oy + oz;
    if (no == 0) return true;
    if (no > 1) return false;
    if (x < -dd || x >= d.W + dd || y < -dd || y >= d.H + dd || z < -dd || z >= d.D + dd) return false;
    x = x < 0 ? x + d.W : (x >= d.W ? x - d.W : x);
    y = y < 0 ? y + d.H : (y >= d.H ? y - d.H : y);
    z = z < 0 ? z + d.D : (z >= d.D ? z - d.D : z);
    return true;
}

#ifndef LENIA_TRANSPORT_BUFS
#define LENIA_TRANSPORT_BUFS 1
#endif
#ifndef LENIA_TRANSPORT_MINB
#define LENIA_TRANSPORT_MINB 4
#endif
// 1 buffer and 4 blocks per SM measured faster than 2 buffers and 2 blocks
// (121 vs 157 us at 128^3 x 4 channels): other blocks cover the copy.
constexpr int kTBufs = LENIA_TRANSPORT_BUFS;  // 2: channel c + 1 lands while c is used
#ifndef LENIA_TRANSPORT_PREGA
#define LENIA_TRANSPORT_PREGA 1
#endif
constexpr bool kTransportPrefetchGA = LENIA_TRANSPORT_PREGA;
#ifndef LENIA_TRANSPORT_PREFETCH_NEXT
#define LENIA_TRANSPORT_PREFETCH_NEXT 1
#endif
constexpr bool kTransportPrefetchNext = LENIA_TRANSPORT_PREFETCH_NEXT;

template <int DD, bool TORUS, bool CLIP1>
__device__ __forceinline__ void transport_tiled_body(const StepParams &p, const TransportBuffers &b,
                                                     const CUtensorMap *tm_mu, const CUtensorMap *tm_arr, int bx,
                                                     int by)
{
    constexpr int SX = kTBoxX, SY = kTY + 2 * DD, SZ = kTZ + 2 * DD, SV = SX * SY * SZ;
    constexpr int OX = 4 - DD;  // staged x of source offset -DD from the tile's first column
    // [kTBufs buffers][MU_x, MU_y, MU_z, ARR][SV], then (DD == 1) the block's
    // GA values [channel][z][thread], copied while the gather runs
    extern __shared__ __align__(128) float tiles[];
    constexpr bool kPreGA = kTransportPrefetchGA && DD == 1;
    float *ga_s = tiles + kTBufs * 4 * SV;
    __shared__ __align__(8) uint64_t bars[2];
    const Dims &d = p.d;
    const long long N = d.N;
    const int C = p.C;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool leader = tx == 0 && ty == 0;
    const int tiles_x = (d.W + kTX - 1) / kTX;
    const int x0 = (bx % tiles_x) * kTX;
    const int y0 = (bx / tiles_x) * kTY;
    const int z0 = by * kTZ;
    const int x = x0 + tx, y = y0 + ty;
    const float px = (float)x + 0.5f, py = (float)y + 0.5f;
    const bool srt = p.mode_type == kModeSRT;
    const int crt = p.rt_all_channels ? C : (C < 3 ? C : 3);
    const int tid = tx + ty * kTX;
    const bool patch = x0 - DD < 0 || x0 + kTX + DD > d.W || y0 - DD < 0 || y0 + kTY + DD > d.H || z0 - DD < 0 ||
                       z0 + kTZ + DD > d.D;

    if (leader) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    pdl_trigger();
    pdl_wait();
    // GA of this thread's cells, read by the epilogue: copied now so that the
    // epilogue does not wait on global loads after the gather
    if (kPreGA && x < d.W && y < d.H) {
#pragma unroll
        for (int c = 0; c < kMaxChannels; c++)
#pragma unroll
            for (int j = 0; j < kTZ; j++)
                if (c < C && z0 + j < d.D)
                    cp_async_f32(ga_s + (c * kTZ + j) * (kTX * kTY) + tid,
                                 b.GA + (long long)c * N + x + (long long)y * d.W + (long long)(z0 + j) * d.W * d.H,
                                 true);
        cp_async_commit();
    }
    // queues channel c's MU and ARR tiles (cells plus a DD halo) into buffer c % kTBufs
    auto issue = [&](int c) {
        if (!leader) return;
        float *buf = tiles + (c % kTBufs) * 4 * SV;
        uint64_t *bar = &bars[c % kTBufs];
        fence_proxy_async();
        mbar_arrive_expect_tx(bar, 4 * SV * 4);
        const int gx = x0 - 4, gy = y0 - DD, gz = z0 - DD;
        tma_load_4d(buf, tm_mu, gx, gy, gz, c, bar);
        tma_load_4d(buf + SV, tm_mu, gx, gy, gz, C + c, bar);
        tma_load_4d(buf + 2 * SV, tm_mu, gx, gy, gz, 2 * C + c, bar);
        tma_load_4d(buf + 3 * SV, tm_arr, gx, gy, gz, c, bar);
        // the next channel's tiles move to L2 while this one is used, so
        // that its copy (issued once this one is done) reads L2
        if (kTransportPrefetchNext && c + 1 < crt) {
            tma_prefetch_4d(tm_mu, gx, gy, gz, c + 1);
            tma_prefetch_4d(tm_mu, gx, gy, gz, C + c + 1);
            tma_prefetch_4d(tm_mu, gx, gy, gz, 2 * C + c + 1);
            tma_prefetch_4d(tm_arr, gx, gy, gz, c + 1);
        }
    };
    // the periodic face layers of channel c's tiles: for each grid face the
    // tile crosses, the cells of its DD layers whose other coordinates are in
    // the grid (edges and corners keep the copy's zeros)
    auto patch_faces = [&](int c, float *buf) {
        const float *src[4] = {b.MU + (long long)c * N, b.MU + (long long)(C + c) * N,
                               b.MU + (long long)(2 * C + c) * N, b.ARR + (long long)c * N};
        const int lo[3] = {x0 - DD, y0 - DD, z0 - DD};
        const int hi[3] = {x0 + kTX + DD, y0 + kTY + DD, z0 + kTZ + DD};
        const int ext[3] = {d.W, d.H, d.D};
        for (int a = 0; a < 3; a++)
            for (int side = 0; side < 2; side++) {
                const int flo = side == 0 ? lo[a] : (ext[a] > lo[a] ? ext[a] : lo[a]);
                const int fhi = side == 0 ? (hi[a] < 0 ? hi[a] : 0) : hi[a];
                if (flo >= fhi) continue;
                const int a1 = (a + 1) % 3, a2 = (a + 2) % 3;
                const int l1 = lo[a1] > 0 ? lo[a1] : 0, h1 = hi[a1] < ext[a1] ? hi[a1] : ext[a1];
                const int l2 = lo[a2] > 0 ? lo[a2] : 0, h2 = hi[a2] < ext[a2] ? hi[a2] : ext[a2];
                const int nl = fhi - flo, n1 = h1 - l1, n2 = h2 - l2;
                if (n1 <= 0 || n2 <= 0) continue;
                for (int e = tid; e < nl * n1 * n2; e += kTX * kTY) {
                    int g[3];
                    g[a] = flo + e % nl;
                    g[a1] = l1 + (e / nl) % n1;
                    g[a2] = l2 + e / (nl * n1);
                    const int t = (g[0] - x0 + 4) + (g[1] - y0 + DD) * SX + (g[2] - z0 + DD) * SX * SY;
                    int gx = g[0], gy = g[1], gz = g[2];
                    const bool ok = tb_source(d, p.dd, gx, gy, gz);
                    const long long o = gx + (long long)gy * d.W + (long long)gz * d.W * d.H;
#pragma unroll
                    for (int q = 0; q < 4; q++) buf[q * SV + t] = ok ? __ldg(src[q] + o) : 0.0f;
                }
            }
    };

    float tt[kMaxChannels][kTZ];
#pragma unroll
    for (int c = 0; c < kMaxChannels; c++)
#pragma unroll
        for (int j = 0; j < kTZ; j++) tt[c][j] = 0.0f;

    if (crt > 0) issue(0);
    for (int c = 0; c < crt; c++) {
        if (kTBufs == 2 && c + 1 < crt) issue(c + 1);
        float *buf = tiles + (c % kTBufs) * 4 * SV;
        if (!block_wait(&bars[c % kTBufs], (unsigned)(c / kTBufs) & 1u, p.wait_polls)) {
            // the wait ran out: record it, drain the copies in flight, return
            mbar_wait(&bars[c % kTBufs], (unsigned)(c / kTBufs) & 1u, kDrainPolls);
            if (kTBufs == 2 && c + 1 < crt)
                mbar_wait(&bars[(c + 1) % kTBufs], (unsigned)((c + 1) / kTBufs) & 1u, kDrainPolls);
            if (kPreGA) cp_async_wait<0>();
            if (leader && b.err) atomicOr(b.err, 2);
            return;
        }
        if (patch) {
            patch_faces(c, buf);
            __syncthreads();
        }
        const float *tmx = buf, *tmy = buf + SV, *tmz = buf + 2 * SV, *tar = buf + 3 * SV;
        float acc[kTZ];
#pragma unroll
        for (int j = 0; j < kTZ; j++) acc[j] = 0.0f;
        if (srt) {
#pragma unroll
            for (int j = 0; j < kTZ; j++) {
                const int e = (tx + OX + DD) + (ty + DD) * SX + (j + DD) * SX * SY;
                const float pz = (float)(z0 + j) + 0.5f;
                float mx = fabsf(px - tmx[e]), my = fabsf(py - tmy[e]), mz = fabsf(pz - tmz[e]);
                mx = tmin(tmax(p.si - mx, 0.0f), p.clip);
                my = tmin(tmax(p.si - my, 0.0f), p.clip);
                mz = tmin(tmax(p.si - mz, 0.0f), p.clip);
                float w = tar[e] * mx;
                w = w * my;
                w = w * mz;
                w = w * p.sn;
                acc[j] = acc[j] + w;
            }
        } else {
#pragma unroll
            for (int lz = 0; lz < SZ; lz++) {          // source layer z' = z0 + lz - DD
#pragma unroll
                for (int oy = -DD; oy <= DD; oy++) {
#pragma unroll
                    for (int ox = -DD; ox <= DD; ox++) {
                        const int e = (tx + OX + DD + ox) + (ty + DD + oy) * SX + lz * SX * SY;
                        const float mx = overlap<TORUS, CLIP1>(px - tmx[e], p.si, p.clip, d.W);
                        const float my = overlap<TORUS, CLIP1>(py - tmy[e], p.si, p.clip, d.H);
                        const float am = tar[e] * mx;
                        const float amy = am * my;
                        const float smz = tmz[e];
#pragma unroll
                        for (int oz = -DD; oz <= DD; oz++) {
                            const int j = lz - DD - oz;  // destination whose offset to this source is oz
                            if (j < 0 || j >= kTZ) continue;
                            const float pz = (float)(z0 + j) + 0.5f;
                            const float mz = overlap<TORUS, CLIP1>(pz - smz, p.si, p.clip, d.D);
                            float w = amy * mz;
                            w = w * p.sn;
                            acc[j] = acc[j] + w;
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int cc = 0; cc < kMaxChannels; cc++)
            if (cc == c)
#pragma unroll
                for (int j = 0; j < kTZ; j++) tt[cc][j] = acc[j];
        // buffer c % kTBufs (and its generic patch writes) is done before it is refilled
        fence_proxy_async();
        __syncthreads();
        if (kTBufs == 1 && c + 1 < crt) issue(c + 1);
    }
    if (x >= d.W || y >= d.H) return;

    // oscillators and transpose_to_row_major, per destination cell
    if (kPreGA) cp_async_wait<0>();
#pragma unroll
    for (int j = 0; j < kTZ; j++) {
        const int z = z0 + j;
        if (z >= d.D) continue;
        const long long i = x + (long long)y * d.W + (long long)z * d.W * d.H;
        float t4[kMaxChannels];
#pragma unroll
        for (int c = 0; c < kMaxChannels; c++) t4[c] = tt[c][j];
        if (kPreGA)
            transport_epilogue(p, b, t4, x, y, z, i, ga_s + j * (kTX * kTY) + tid, kTZ * kTX * kTY);
        else
            transport_epilogue(p, b, t4, x, y, z, i);
    }
}

template <int DD, bool TORUS, bool CLIP1>
__global__ void __launch_bounds__(kTX *kTY, LENIA_TRANSPORT_MINB) k_transport_tiled(const __grid_constant__ StepParams p,
                                                              const __grid_constant__ TransportBuffers b,
                                                              const __grid_constant__ CUtensorMap tm_mu,
                                                              const __grid_constant__ CUtensorMap tm_arr)
{
    transport_tiled_body<DD, TORUS, CLIP1>(p, b, &tm_mu, &tm_arr, blockIdx.x, blockIdx.y);
}

template <typename T>
__device__ __forceinline__ void copy_words_to_shared(T *dst, const T *src)
{
    static_assert(sizeof(T) % 4 == 0, "copied as 4-byte words");
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int nthr = blockDim.x * blockDim.y;
    for (int i = tid; i < (int)(sizeof(T) / 4); i += nthr)
        reinterpret_cast<unsigned *>(dst)[i] = reinterpret_cast<const unsigned *>(src)[i];
}

// Batched transport (RT, dd = 1, the tiled gather): block b is block
// items[b].block of world items[b].world's own launch (x-y tile fastest);
// the world's parameters are read into shared memory first.
template <bool TORUS, bool CLIP1>
__global__ void __launch_bounds__(kTX *kTY, LENIA_TRANSPORT_MINB) k_transport_rt_multi(
    const BatchWorldDev *__restrict__ ws, const WorkItem *__restrict__ items)
{
    __shared__ StepParams sp;
    __shared__ TransportBuffers sb;
    const WorkItem it = items[blockIdx.x];
    const BatchWorldDev *w = ws + it.world;
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        asm volatile("prefetch.tensormap [%0];\n" ::"l"(&w->tm_mu) : "memory");
        asm volatile("prefetch.tensormap [%0];\n" ::"l"(&w->tm_arr) : "memory");
    }
    copy_words_to_shared(&sp, &w->p);
    copy_words_to_shared(&sb, &w->tb);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(&w->tm_mu) : "memory");
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(&w->tm_arr) : "memory");
    }
    const int gx = w->transport_gx;
    __syncthreads();
    transport_tiled_body<1, TORUS, CLIP1>(sp, sb, &w->tm_mu, &w->tm_arr, it.block % gx, it.block / gx);
}

// Batched per-cell transport (advection, and whatever the tiled gather does
// not take): block b is block items[b].block of world items[b].world's launch.
__global__ void __launch_bounds__(256) k_transport_cell_multi(const BatchWorldDev *__restrict__ ws,
                                                              const WorkItem *__restrict__ items)
{
    __shared__ StepParams sp;
    __shared__ TransportBuffers sb;
    const WorkItem it = items[blockIdx.x];
    const BatchWorldDev *w = ws + it.world;
    copy_words_to_shared(&sp, &w->p);
    copy_words_to_shared(&sb, &w->tb);
    __syncthreads();
    transport_cell_body(sp, sb, it.block);
}

int transport_rt_blocks(const Dims &d, int *gx)
{
    const int tiles_x = (d.W + kTX - 1) / kTX, tiles_y = (d.H + kTY - 1) / kTY;
    if (gx) *gx = tiles_x * tiles_y;
    return tiles_x * tiles_y * ((d.D + kTZ - 1) / kTZ);
}

int transport_adv_blocks(const Dims &d) { return (int)((d.N + 255) / 256); }

cudaError_t launch_transport_rt_multi(const BatchWorldDev *ws, const WorkItem *items, int n_items, bool torus,
                                      bool clip1, cudaStream_t st)
{
    if (n_items == 0) return cudaSuccess;
    auto go = [&](auto kern) -> cudaError_t {
        const int sv = kTBoxX * (kTY + 2) * (kTZ + 2);
        const size_t ga = kTransportPrefetchGA ? (size_t)kMaxChannels * kTZ * kTX * kTY : 0;
        const size_t smem = (kTBufs * 4 * (size_t)sv + ga) * sizeof(float);
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<(unsigned)n_items, dim3(kTX, kTY), smem, st>>>(ws, items);
        return cudaGetLastError();
    };
    if (torus) return clip1 ? go(k_transport_rt_multi<true, true>) : go(k_transport_rt_multi<true, false>);
    return clip1 ? go(k_transport_rt_multi<false, true>) : go(k_transport_rt_multi<false, false>);
}

cudaError_t launch_transport_adv_multi(const BatchWorldDev *ws, const WorkItem *items, int n_items, cudaStream_t st)
{
    if (n_items == 0) return cudaSuccess;
    k_transport_cell_multi<<<(unsigned)n_items, 256, 0, st>>>(ws, items);
    return cudaGetLastError();
}

// The tiled gather's tensor maps: MU (x, y, z, 3C) and ARR (x, y, z, C),
// tiles of kTBoxX x (kTY + 2 dd) x (kTZ + 2 dd).
cudaError_t transport_tensor_maps(const StepParams &p, const TransportBuffers &b, int dd, CUtensorMap *tm_mu,
                                  CUtensorMap *tm_arr)
{
    const Dims &d = p.d;
    const unsigned long long dmu[4] = {(unsigned long long)d.W, (unsigned long long)d.H, (unsigned long long)d.D,
                                       3ull * p.C};
    const unsigned long long darr[4] = {(unsigned long long)d.W, (unsigned long long)d.H, (unsigned long long)d.D,
                                        (unsigned long long)p.C};
    const unsigned box[4] = {(unsigned)kTBoxX, (unsigned)(kTY + 2 * dd), (unsigned)(kTZ + 2 * dd), 1u};
    cudaError_t e = encode_tensor_map(tm_mu, b.MU, 4, dmu, box);
    if (e == cudaSuccess) e = encode_tensor_map(tm_arr, b.ARR, 4, darr, box);
    return e;
}

// The transport kernel a world's step uses: 1 = the tiled gather with dd = 1
// (the form the batched launches take), 2 = tiled with dd = 2, 0 = per cell.
int transport_form(const StepParams &p)
{
    const int crt = p.rt_all_channels ? p.C : (p.C < 3 ? p.C : 3);
    if ((p.mode_type == kModeRT || p.mode_type == kModeSRT) && p.dd >= 1 && p.dd <= 2 && crt > 0) return p.dd;
    return 0;
}

cudaError_t launch_transport(const StepParams &p, const TransportBuffers &b, cudaStream_t st)
{
    const int crt = p.rt_all_channels ? p.C : (p.C < 3 ? p.C : 3);
    if ((p.mode_type == kModeRT || p.mode_type == kModeSRT) && p.dd >= 1 && p.dd <= 2 && crt > 0) {
        const Dims &d = p.d;
        const int tiles_x = (d.W + kTX - 1) / kTX, tiles_y = (d.H + kTY - 1) / kTY;
        dim3 grid(tiles_x * tiles_y, (d.D + kTZ - 1) / kTZ), block(kTX, kTY);
        const bool torus = p.border == kBorderTorus;
        auto go = [&](auto kern, int dd) -> cudaError_t {
            CUtensorMap tm_mu, tm_arr;
            cudaError_t e = transport_tensor_maps(p, b, dd, &tm_mu, &tm_arr);
            if (e != cudaSuccess) return e;
            const int sv = kTBoxX * (kTY + 2 * dd) * (kTZ + 2 * dd);
            const size_t ga = (kTransportPrefetchGA && dd == 1) ? (size_t)kMaxChannels * kTZ * kTX * kTY : 0;
            const size_t smem = (kTBufs * 4 * (size_t)sv + ga) * sizeof(float);
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            return launch_pdl(kern, grid, block, smem, st, p, b, tm_mu, tm_arr);
        };
        const bool c1 = p.clip == 1.0f;
        if (p.dd == 1) {
            if (c1) return torus ? go(k_transport_tiled<1, true, true>, 1) : go(k_transport_tiled<1, false, true>, 1);
            return torus ? go(k_transport_tiled<1, true, false>, 1) : go(k_transport_tiled<1, false, false>, 1);
        }
        if (c1) return torus ? go(k_transport_tiled<2, true, true>, 2) : go(k_transport_tiled<2, false, true>, 2);
        return torus ? go(k_transport_tiled<2, true, false>, 2) : go(k_transport_tiled<2, false, false>, 2);
    }
    k_transport<<<(unsigned)((p.d.N + 255) / 256), 256, 0, st>>>(p, b);
    return cudaGetLastError();
}

}  // namespace lenia
