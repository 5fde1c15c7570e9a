// Size-specialised spectral kernels for cubic grids (W = H = D in
// {24, 32, 36, 44, 48, 64, 96, 128}): the same transforms and epilogues as
// kernels_spectral.cu, with compile-time radix plans, padded conflict-free
// shared memory and the growth accumulators held in registers.  Results are
// bit-identical to the generic kernels (same float operations in the same
// order); only the schedule differs.
#include "lenia_internal.h"
#include "lfft_static.cuh"
#include "growth_common.cuh"
#include "async_copy.cuh"

namespace lenia {

namespace {

#ifndef LENIA_PLANE_THREADS
#define LENIA_PLANE_THREADS 1024
#endif
#ifndef LENIA_GROWTH_THREADS
#define LENIA_GROWTH_THREADS 256
#endif
#ifndef LENIA_GROWTH_ROWS
#define LENIA_GROWTH_ROWS 16
#endif
constexpr int kFastRowThreads = 256;
constexpr int kMaxGridY = 65535;  // the largest grid.y of a launch
constexpr int kFastPlaneThreads = LENIA_PLANE_THREADS;    // block of the plane transform
constexpr int kGrowthThreads = LENIA_GROWTH_THREADS;      // block of the growth pass
#ifndef LENIA_PLANE_PAIRED
#define LENIA_PLANE_PAIRED 1
#endif
// The plane passes (bound by instruction issue) take the paired butterflies;
// the row passes keep the scalar ones, whose fewer registers keep more blocks
// resident to cover their global-memory latency.
constexpr bool kPlanePaired = LENIA_PLANE_PAIRED;

// Rows per tile of the growth pass: at most 2048 cells, so that a thread's
// cells (prefetched spectra and growth sums in registers) stay at 8.
constexpr int growth_tile_for(int n)
{
    for (int t = LENIA_GROWTH_ROWS; t > 1; t--)
        if (n % t == 0 && t * n <= 2048) return t;
    return 1;
}

template <int W, bool GROWTH = false>
struct RowShape {
    static constexpr int TY = GROWTH ? growth_tile_for(W) : row_tile_for(W);
    static constexpr int T = TY * W;                       // cells of a tile
    static constexpr int THREADS = GROWTH ? kGrowthThreads : kFastRowThreads;
    static constexpr int NCELL = (T + THREADS - 1) / THREADS;  // cells per thread
    using PM = PadMat<W>;
};

// Job accessors: the by-value job structs of one world's launch, or the
// device job lists of a batched launch (one entry per pair / plane).
__device__ __forceinline__ const float *row_in(const FwdRowJobs &j, int p, int h) { return j.in[2 * p + h]; }
__device__ __forceinline__ float2 *row_out(const FwdRowJobs &j, int p, int h) { return j.out[2 * p + h]; }
__device__ __forceinline__ const float *row_in(const RowPairList &j, int p, int h) { return j.j[p].in[h]; }
__device__ __forceinline__ float2 *row_out(const RowPairList &j, int p, int h) { return j.j[p].out[h]; }
__device__ __forceinline__ const float2 *plane_src(const PlaneJobs &j, int i) { return j.src[i]; }
__device__ __forceinline__ float2 *plane_dst(const PlaneJobs &j, int i) { return j.dst[i]; }
__device__ __forceinline__ const float *plane_kc(const PlaneJobs &j, int i) { return j.kc[i]; }
__device__ __forceinline__ const float2 *plane_src(const PlaneJobList &j, int i) { return j.j[i].src; }
__device__ __forceinline__ float2 *plane_dst(const PlaneJobList &j, int i) { return j.j[i].dst; }
__device__ __forceinline__ const float *plane_kc(const PlaneJobList &j, int i) { return j.j[i].kc; }
// inverse rows: field h (0, 1) of pair p, null when the pair has one field
__device__ __forceinline__ const float2 *inv_spec(const BlurJobs &j, int p, int h)
{
    return 2 * p + h < j.nfields ? j.spec[2 * p + h] : nullptr;
}
__device__ __forceinline__ float *inv_out(const BlurJobs &j, int p, int h)
{
    return 2 * p + h < j.nfields ? j.out[2 * p + h] : nullptr;
}
__device__ __forceinline__ const float2 *inv_spec(const InvPairList &j, int p, int h) { return j.j[p].spec[h]; }
__device__ __forceinline__ float *inv_out(const InvPairList &j, int p, int h) { return j.j[p].out[h]; }

template <int W, typename J>
__global__ void __launch_bounds__(kFastRowThreads) k_fwd_rows_s(J jobs, const float2 *__restrict__ tw_x)
{
    using S = RowShape<W>;
    constexpr int H = W, D = W, TY = S::TY, KX = W / 2 + 1;
    extern __shared__ float2 smem[];
    float2 *tw = smem;
    float2 *buf = smem + W;
    const int z = blockIdx.x / (H / TY);
    const int y0 = (blockIdx.x % (H / TY)) * TY;
    const int pair = blockIdx.y;
    const float *fa = row_in(jobs, pair, 0);
    const float *fb = row_in(jobs, pair, 1);
    float2 *oa = row_out(jobs, pair, 0);
    float2 *ob = row_out(jobs, pair, 1);
    for (int i = threadIdx.x; i < W; i += kFastRowThreads) tw[i] = tw_x[i];
    pdl_trigger();
    pdl_wait();
    const long long base = ((long long)z * H + y0) * W;
    // all of a thread's loads are issued before its shared-memory stores
    constexpr int NE = TY * W, NI = (NE + kFastRowThreads - 1) / kFastRowThreads;
    float va[NI], vb[NI];
#pragma unroll
    for (int i = 0; i < NI; i++) {
        const int e = threadIdx.x + i * kFastRowThreads;
        if (NE % kFastRowThreads == 0 || e < NE) {
            va[i] = __ldg(fa + base + e);
            vb[i] = fb ? __ldg(fb + base + e) : 0.0f;
        }
    }
#pragma unroll
    for (int i = 0; i < NI; i++) {
        const int e = threadIdx.x + i * kFastRowThreads;
        if (NE % kFastRowThreads == 0 || e < NE) buf[S::PM::at(e / W, e % W)] = make_float2(va[i], vb[i]);
    }
    __syncthreads();
    static_fft<W, TY, false, W, kFastRowThreads>(buf, tw, -1);
    for (int e = threadIdx.x; e < TY * KX; e += kFastRowThreads) {
        const int ty = e % TY, kx = e / TY;
        const float2 p = buf[S::PM::at(ty, kx)];
        const float2 q = buf[S::PM::at(ty, (W - kx) % W)];
        const long long o = ((long long)kx * D + z) * H + y0 + ty;
        oa[o] = make_float2((p.x + q.x) * 0.5f, (p.y - q.y) * 0.5f);
        if (ob) ob[o] = make_float2((p.y + q.y) * 0.5f, (q.x - p.x) * 0.5f);
    }
}

// A plane of work: (kx, job) in the order of the former 2D grid (kx fastest),
// so that jobs reading one source spectrum run close together and share its
// planes through L2.
template <int W>
__device__ __forceinline__ void plane_unit_prefetch(const PlaneJobs &jobs, int u)
{
    constexpr int KX = W / 2 + 1, KZ = W / 2 + 1, KY = W / 2 + 1;
    const int kx = u % KX, job = u / KX;
    prefetch_l2(jobs.src[job] + (long long)kx * W * W, (size_t)W * W * sizeof(float2));
    if (jobs.kc[job]) prefetch_l2(jobs.kc[job] + (long long)kx * KZ * KY, (size_t)KZ * KY * sizeof(float));
}

// Stage 0 of the y transforms of a plane (rows z, length H along y) with its
// inputs read from global memory, times the octant kernel spectrum when kp is
// given: the butterflies of static_stage<H, 0, D, false> on the values the
// plane load would have put in buf, without that load's shared-memory pass.
template <int W>
__device__ __forceinline__ void plane_first_stage(float2 *buf, const float2 *__restrict__ src,
                                                  const float *__restrict__ kp, const float2 *tw, int sign, int tid)
{
    constexpr int H = W, D = W, R = plan_radix(H, 0), M = H / R, TOTAL = D * M, KY = H / 2 + 1;
    constexpr int NB = (TOTAL + kFastPlaneThreads - 1) / kFastPlaneThreads;
    static_assert(plan_ns(H, 0) == 1, "stage 0 takes no twiddles");
    using PM = PadMat<H>;
#pragma unroll
    for (int i = 0; i < NB; i++) {
        const int b = tid + i * kFastPlaneThreads;
        if (TOTAL % kFastPlaneThreads == 0 || b < TOTAL) {
            const int j = b % M, z = b / M;
            const int oz = z <= D - z ? z : D - z;
            float2 v[R];
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int y = j + r * M;
                const float2 t = __ldg(src + z * H + y);
                if (kp) {
                    const int oy = y <= H - y ? y : H - y;
                    const float k = __ldg(kp + oz * KY + oy);
                    v[r] = make_float2(t.x * k, t.y * k);
                } else {
                    v[r] = t;
                }
            }
            dft_small<R, kPlanePaired>(v, sign, tw, H);
#pragma unroll
            for (int r = 0; r < R; r++) buf[PM::at(z, j * R + r)] = v[r];
        }
    }
    __syncthreads();
}

// Last stage of the z transforms (columns y, length D along z) with its
// outputs written to global memory: the butterflies of
// static_stage<D, last, H, true> without the store's shared-memory pass.
template <int W>
__device__ __forceinline__ void plane_last_stage(const float2 *buf, float2 *__restrict__ dst, const float2 *tw,
                                                 int sign, int tid)
{
    constexpr int H = W, D = W, S = plan_count(D) - 1, R = plan_radix(D, S), NS = plan_ns(D, S), M = D / R;
    constexpr int TOTAL = H * M, TSTEP = D / (NS * R);
    constexpr int NB = (TOTAL + kFastPlaneThreads - 1) / kFastPlaneThreads;
    using PM = PadMat<H>;
    float2 v[NB][R];
#pragma unroll
    for (int i = 0; i < NB; i++) {
        const int b = tid + i * kFastPlaneThreads;
        if (TOTAL % kFastPlaneThreads == 0 || b < TOTAL) {
            const int l = b % H, j = b / H;
#pragma unroll
            for (int r = 0; r < R; r++) v[i][r] = buf[PM::at(j + r * M, l)];
        }
    }
#pragma unroll
    for (int i = 0; i < NB; i++) {
        const int b = tid + i * kFastPlaneThreads;
        if (TOTAL % kFastPlaneThreads == 0 || b < TOTAL) {
            const int l = b % H, j = b / H;
            const int jm = j % NS;
            if (NS > 1 && jm != 0) {
#pragma unroll
                for (int r = 1; r < R; r++) v[i][r] = cmul(v[i][r], tw[r * jm * TSTEP]);
            }
            dft_small<R, kPlanePaired>(v[i], sign, tw, D);
            const int base = (j / NS) * NS * R + jm;
#pragma unroll
            for (int r = 0; r < R; r++) dst[(base + r * NS) * H + l] = v[i][r];
        }
    }
}

template <int W, typename J>
__global__ void __launch_bounds__(kFastPlaneThreads) k_planes_s(J jobs, const float2 *__restrict__ tw_y,
                                                                const float2 *__restrict__ tw_z, int sign)
{
    constexpr int H = W, D = W;
    using PM = PadMat<H>;
    extern __shared__ float2 smem[];
    float2 *twy = smem;
    float2 *twz = smem + H;
    float2 *buf = smem + H + D;
    const int kx = blockIdx.x;
    const int job = blockIdx.y;
    const float4 *src = reinterpret_cast<const float4 *>(plane_src(jobs, job) + (long long)kx * D * H);
    float4 *dst = reinterpret_cast<float4 *>(plane_dst(jobs, job) + (long long)kx * D * H);
    const float *kc = plane_kc(jobs, job);
    for (int i = threadIdx.x; i < H; i += kFastPlaneThreads) twy[i] = tw_y[i];
    for (int i = threadIdx.x; i < D; i += kFastPlaneThreads) twz[i] = tw_z[i];
    pdl_trigger();
    pdl_wait();
    constexpr int KZ = D / 2 + 1, KY = H / 2 + 1;
    if (kc) {
        const float *kp = kc + (long long)kx * KZ * KY;
        for (int e = threadIdx.x; e < D * H / 2; e += kFastPlaneThreads) {
            const int z = (2 * e) / H, y = (2 * e) % H;
            const int oz = z <= D - z ? z : D - z;
            const int oy0 = y <= H - y ? y : H - y;
            const int oy1 = (y + 1) <= H - (y + 1) ? (y + 1) : H - (y + 1);
            const float k0 = __ldg(kp + oz * KY + oy0);
            const float k1 = __ldg(kp + oz * KY + oy1);
            const float4 t = __ldg(src + e);
            buf[PM::at(z, y)] = make_float2(t.x * k0, t.y * k0);
            buf[PM::at(z, y + 1)] = make_float2(t.z * k1, t.w * k1);
        }
    } else {
        for (int e = threadIdx.x; e < D * H / 2; e += kFastPlaneThreads) {
            const int z = (2 * e) / H, y = (2 * e) % H;
            const float4 t = __ldg(src + e);
            buf[PM::at(z, y)] = make_float2(t.x, t.y);
            buf[PM::at(z, y + 1)] = make_float2(t.z, t.w);
        }
    }
    __syncthreads();
    static_fft<H, D, false, H, kFastPlaneThreads, kPlanePaired>(buf, twy, sign);
    static_fft<D, H, true, H, kFastPlaneThreads, kPlanePaired>(buf, twz, sign);
    for (int e = threadIdx.x; e < D * H / 2; e += kFastPlaneThreads) {
        const int z = (2 * e) / H, y = (2 * e) % H;
        const float2 a = buf[PM::at(z, y)], b = buf[PM::at(z, y + 1)];
        dst[e] = make_float4(a.x, a.y, b.x, b.y);
    }
}


// At 128 the plane pass runs persistent with its first and last stages on
// global memory (k_planes_stream_s: one 1024-thread block per SM walks about
// seven planes; 136 -> 114 us for 16 inverse planes of 128^2 x 65).  Below it
// k_planes_s keeps one plane per block: a loop over planes costs registers
// there (64 instead of 32 at 64 and 48, so one block per SM instead of two;
// spills at 96 and 44), and the persistent form measured 1-4 % slower in
// batches of worlds of 24-96 cells per side.
template <int W>
constexpr bool planes_persistent() { return W >= 128; }

// Persistent: gridDim.x blocks walk the KX * njobs planes with stride
// gridDim.x; once a block has read its plane it asks L2 for its next one, so
// that load comes from L2 while this plane's transforms run.  The y
// transforms' first stage reads global memory and the z transforms' last
// stage writes it, so the plane crosses shared memory only between stages.
template <int W>
__global__ void __launch_bounds__(kFastPlaneThreads) k_planes_stream_s(PlaneJobs jobs, const float2 *__restrict__ tw_y,
                                                                const float2 *__restrict__ tw_z, int sign)
{
    constexpr int H = W, D = W, KX = W / 2 + 1, KZ = D / 2 + 1, KY = H / 2 + 1;
    static_assert(plan_count(H) >= 2, "first and last stages are separate passes");
    extern __shared__ float2 smem[];
    float2 *twy = smem;
    float2 *twz = smem + H;
    float2 *buf = smem + H + D;
    for (int i = threadIdx.x; i < H; i += kFastPlaneThreads) twy[i] = tw_y[i];
    for (int i = threadIdx.x; i < D; i += kFastPlaneThreads) twz[i] = tw_z[i];
    pdl_trigger();
    pdl_wait();
    __syncthreads();
    const int units = KX * jobs.njobs;
    const int stride = gridDim.x;
    for (int u = blockIdx.x; u < units; u += stride) {
        const int kx = u % KX;
        const int job = u / KX;
        const float2 *src = jobs.src[job] + (long long)kx * D * H;
        float2 *dst = jobs.dst[job] + (long long)kx * D * H;
        const float *kp = jobs.kc[job] ? jobs.kc[job] + (long long)kx * KZ * KY : nullptr;
        // the thread index read afresh per plane, so that the stages' index
        // arithmetic is not hoisted out of the loop into registers held
        // across it
        int tid;
        asm volatile("mov.u32 %0, %%tid.x;" : "=r"(tid));
        // its range, which the asm read hides: the stages' divisions and
        // remainders by constants then take their unsigned forms
        __builtin_assume(tid >= 0);
        __builtin_assume(tid < kFastPlaneThreads);
        plane_first_stage<W>(buf, src, kp, twy, sign, tid);
        if (tid == 0 && u + stride < units) plane_unit_prefetch<W>(jobs, u + stride);
        static_stages<H, 1, D, false, H, kFastPlaneThreads, false, plan_count(H), kPlanePaired>(buf, twy, sign, tid);
        static_stages<D, 0, H, true, H, kFastPlaneThreads, false, plan_count(D) - 1, kPlanePaired>(buf, twz, sign,
                                                                                                   tid);
        plane_last_stage<W>(buf, dst, twz, sign, tid);
        __syncthreads();  // the next plane's first stage overwrites buf
    }
}

// Split plane passes with compile-time plans, for cubic grids whose kx plane
// exceeds shared memory (256): pass y transforms kSplitLines z-lines of one
// plane (after the optional kernel product), pass z kSplitLines y-columns.
// Each line takes the same transform as in k_planes_s, so results are
// identical.
constexpr int kSplitLines = 32;
constexpr int kSplitThreads = 512;

template <int W>
__global__ void __launch_bounds__(kSplitThreads) k_plane_lines_y_s(PlaneJobs jobs, const float2 *__restrict__ tw_y,
                                                                   int sign)
{
    constexpr int H = W, D = W, TZ = kSplitLines;
    using PM = PadMat<H>;
    extern __shared__ float2 smem[];
    float2 *twy = smem;
    float2 *buf = smem + H;
    const int kx = blockIdx.x, z0 = blockIdx.y * TZ, job = blockIdx.z;
    const long long base = ((long long)kx * D + z0) * H;
    const float2 *src = jobs.src[job] + base;
    float2 *dst = jobs.dst[job] + base;
    const float *kc = jobs.kc[job];
    for (int i = threadIdx.x; i < H; i += kSplitThreads) twy[i] = tw_y[i];
    pdl_trigger();
    pdl_wait();
    constexpr int KZ = D / 2 + 1, KY = H / 2 + 1;
    for (int e = threadIdx.x; e < TZ * H; e += kSplitThreads) {
        const int t = e / H, y = e % H;
        float2 v = __ldg(src + e);
        if (kc) {
            const int z = z0 + t;
            const int oz = z <= D - z ? z : D - z;
            const int oy = y <= H - y ? y : H - y;
            const float k = __ldg(kc + (long long)kx * KZ * KY + oz * KY + oy);
            v = make_float2(v.x * k, v.y * k);
        }
        buf[PM::at(t, y)] = v;
    }
    __syncthreads();
    static_fft<H, TZ, false, H, kSplitThreads, kPlanePaired>(buf, twy, sign);
    for (int e = threadIdx.x; e < TZ * H; e += kSplitThreads) dst[e] = buf[PM::at(e / H, e % H)];
}

template <int W>
__global__ void __launch_bounds__(kSplitThreads) k_plane_lines_z_s(PlaneJobs jobs, const float2 *__restrict__ tw_z,
                                                                   int sign)
{
    constexpr int H = W, D = W, TY = kSplitLines;
    using PM = PadMat<TY>;
    extern __shared__ float2 smem[];
    float2 *twz = smem;
    float2 *buf = smem + D;
    const int kx = blockIdx.x, y0 = blockIdx.y * TY, job = blockIdx.z;
    float2 *dst = jobs.dst[job] + (long long)kx * D * H + y0;
    for (int i = threadIdx.x; i < D; i += kSplitThreads) twz[i] = tw_z[i];
    pdl_trigger();
    pdl_wait();
    for (int e = threadIdx.x; e < D * TY; e += kSplitThreads) {
        const int z = e / TY, t = e % TY;
        buf[PM::at(z, t)] = dst[(long long)z * H + t];
    }
    __syncthreads();
    static_fft<D, TY, true, TY, kSplitThreads, kPlanePaired>(buf, twz, sign);
    for (int e = threadIdx.x; e < D * TY; e += kSplitThreads) {
        const int z = e / TY, t = e % TY;
        dst[(long long)z * H + t] = buf[PM::at(z, t)];
    }
}

// Packed row spectrum of two kernels (or fields) for one tile: kx < W/2+1
// from the stored half spectra, the rest by Hermitian symmetry.
template <int W>
__device__ __forceinline__ void load_packed_rows_s(float2 *buf, const float2 *s0, const float2 *s1, int z, int y0)
{
    using S = RowShape<W>;
    constexpr int H = W, D = W, TY = S::TY, KX = W / 2 + 1;
    constexpr int NE = TY * KX, NI = (NE + kFastRowThreads - 1) / kFastRowThreads;
    // each half-spectrum value read once, for column m and its mirror W - m;
    // all of a thread's loads are issued before its shared-memory stores
    float2 a[NI], b[NI];
#pragma unroll
    for (int i = 0; i < NI; i++) {
        const int e = threadIdx.x + i * kFastRowThreads;
        if (NE % kFastRowThreads == 0 || e < NE) {
            const int ty = e % TY, m = e / TY;
            const long long o = ((long long)m * D + z) * H + y0 + ty;
            a[i] = __ldg(s0 + o);
            b[i] = s1 ? __ldg(s1 + o) : make_float2(0.0f, 0.0f);
        }
    }
#pragma unroll
    for (int i = 0; i < NI; i++) {
        const int e = threadIdx.x + i * kFastRowThreads;
        if (NE % kFastRowThreads == 0 || e < NE) {
            const int ty = e % TY, m = e / TY;
            buf[S::PM::at(ty, m)] = make_float2(a[i].x - b[i].y, a[i].y + b[i].x);
            if (m > 0 && W - m >= KX) buf[S::PM::at(ty, W - m)] = make_float2(a[i].x + b[i].y, b[i].x - a[i].y);
        }
    }
}

// EXACT: the exact-bell growth (a separate instance keeps the table path as it was)
template <int W, bool EXACT>
__global__ void __launch_bounds__(kGrowthThreads) k_growth_rows_s(GrowthJobs jobs, const float2 *__restrict__ tw_x,
                                                                   const float *__restrict__ lut_rows,
                                                                   const float *__restrict__ A,
                                                                   float *__restrict__ Hout, float *__restrict__ Uout,
                                                                   float *__restrict__ BACK, float *__restrict__ Udbg,
                                                                   int *err_flag)
{
    using S = RowShape<W, true>;
    constexpr int H = W, D = W, TY = S::TY, T = S::T, NCELL = S::NCELL, KX = W / 2 + 1;
    constexpr long long N = (long long)W * W * W;
    extern __shared__ float2 smem[];
    float2 *tw = smem;
    float2 *buf = tw + W;
    float *lut = reinterpret_cast<float *>(buf + S::PM::size(TY));
    const int C = jobs.C, K = jobs.K;
    const int z = blockIdx.x / (H / TY);
    const int y0 = (blockIdx.x % (H / TY)) * TY;
    const long long base = ((long long)z * H + y0) * W;
    const float nf = (float)N;
    for (int i = threadIdx.x; i < W; i += kGrowthThreads) tw[i] = tw_x[i];
    for (int i = threadIdx.x; i < 256 * K; i += kGrowthThreads) lut[i] = lut_rows[i];
    pdl_trigger();
    pdl_wait();

    // The packed row spectrum of a kernel pair: element e of the tile is
    // (ty = e % TY, kx = e / TY); its half-spectrum values are prefetched into
    // registers one pair ahead so the loads overlap the current transform.
    float2 pa[NCELL], pb[NCELL];
    auto prefetch = [&](int k0) {
        const float2 *s0 = jobs.spec[k0];
        const float2 *s1 = k0 + 1 < K ? jobs.spec[k0 + 1] : nullptr;
#pragma unroll
        for (int i = 0; i < NCELL; i++) {
            const int e = threadIdx.x + i * kGrowthThreads;
            if (T % kGrowthThreads != 0 && e >= T) continue;
            const int ty = e % TY, kx = e / TY;
            const int m = kx < KX ? kx : W - kx;
            const long long o = ((long long)m * D + z) * H + y0 + ty;
            pa[i] = __ldg(s0 + o);
            pb[i] = s1 ? __ldg(s1 + o) : make_float2(0.0f, 0.0f);
        }
    };

    // H accumulates in registers, U_SUM in shared memory (channel-major)
    float *uacc = lut + 256 * K;
    for (int i = threadIdx.x; i < C * T; i += kGrowthThreads) uacc[i] = 0.0f;
    float hacc[NCELL][kMaxChannels];
#pragma unroll
    for (int i = 0; i < NCELL; i++)
#pragma unroll
        for (int c = 0; c < kMaxChannels; c++) hacc[i][c] = 0.0f;
    int bad = 0;
    // u = re / N; for N a power of two the quotient is exactly re * (1/N)
    constexpr bool kPow2 = (N & (N - 1)) == 0;
    constexpr float kInvN = 1.0f / (float)N;
    if (K > 0) prefetch(0);
    for (int k0 = 0; k0 < K; k0 += 2) {
        const int k1 = k0 + 1 < K ? k0 + 1 : -1;
#pragma unroll
        for (int i = 0; i < NCELL; i++) {
            const int e = threadIdx.x + i * kGrowthThreads;
            if (T % kGrowthThreads != 0 && e >= T) continue;
            const int ty = e % TY, kx = e / TY;
            const float2 a = pa[i], b = pb[i];
            float2 r;
            if (kx < KX) r = make_float2(a.x - b.y, a.y + b.x);
            else r = make_float2(a.x + b.y, b.x - a.y);
            buf[S::PM::at(ty, kx)] = r;
        }
        __syncthreads();
        if (k0 + 2 < K) prefetch(k0 + 2);
        static_fft<W, TY, false, W, kGrowthThreads>(buf, tw, +1);
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int k = q == 0 ? k0 : k1;
            if (k < 0) continue;
            const int c1 = jobs.c1[k];
            const float h = jobs.h[k];
            const int asym = jobs.asymptotic[c1];
            float u[NCELL], g[NCELL];
#pragma unroll
            for (int i = 0; i < NCELL; i++) {
                const int e = threadIdx.x + i * kGrowthThreads;
                u[i] = 0.0f;
                g[i] = 0.0f;
                if (T % kGrowthThreads != 0 && e >= T) continue;
                const float2 zz = buf[S::PM::at(e / W, e % W)];
                const float re = q == 0 ? zz.x : zz.y;
                u[i] = kPow2 ? re * kInvN : re / nf;
                const int ui = (int)(u[i] * 255);
                float l;
                if (EXACT) {
                    if (!(u[i] == u[i])) bad = 1;
                    l = bell_dev(u[i], jobs.m[k], jobs.s[k]);
                } else if (ui >= 0 && ui < 256) l = lut[k * 256 + ui];
                else {
                    if (!(u[i] == u[i])) bad = 1;
                    l = lut_flat_dev((long long)jobs.lut_base[k] + ui);
                }
                g[i] = asym ? (l - __ldg(A + (long long)c1 * N + base + e)) * h : l * h;
                uacc[c1 * T + e] = uacc[c1 * T + e] + u[i];
                if (Udbg) Udbg[(long long)k * N + base + e] = u[i];
            }
            // uniform branch on the destination channel keeps hacc in registers
            switch (c1) {
#define LENIA_ACC(cc)                                                              \
    case cc:                                                                       \
        _Pragma("unroll") for (int i = 0; i < NCELL; i++) hacc[i][cc] = hacc[i][cc] + g[i]; \
        break;
                LENIA_ACC(0) LENIA_ACC(1) LENIA_ACC(2) LENIA_ACC(3)
#undef LENIA_ACC
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < NCELL; i++) {
        const int e = threadIdx.x + i * kGrowthThreads;
        if (T % kGrowthThreads != 0 && e >= T) continue;
#pragma unroll
        for (int c = 0; c < kMaxChannels; c++) {
            if (c >= C) continue;
            const long long o = (long long)c * N + base + e;
            const float hv = hacc[i][c];
            Hout[o] = hv;
            const float us = uacc[c * T + e];
            Uout[o] = us;
            if (!isfinite(us)) bad = 1;  // a NaN u indexes the table at 0: test the sum
            if (jobs.growth_rt) BACK[o] = early_growth(__ldg(A + o), hv, jobs.timestep, jobs.soft_clip[c]);
        }
    }
    if (bad && err_flag) atomicOr(err_flag, 1);
}

// Growth pass with warp-level transforms.  A block owns 8 warps x 2 rows of
// one z slice.  For each kernel pair the block stages the pair's half-spectrum
// rows with cp.async (double buffered, one block barrier per pair); each warp
// then builds its two packed rows, transforms them with warp-scope barriers
// only, and accumulates the growth of its 2 x W cells.  Arithmetic and order
// are those of k_growth_rows_s.
constexpr int kGwWarps = 8, kGwRows = 2, kGwRowsBlock = kGwWarps * kGwRows;

template <int W>
struct GrowthWarpShape {
    static constexpr int KX = W / 2 + 1;
    static constexpr int SP = kGwRowsBlock + 2;                   // staged row pitch (bank-conflict free)
    static constexpr int STAGE = 2 * KX * SP;                     // float2 per staged pair
    static constexpr int CELLS = kGwRows * W / 32;                // cells per lane
    using PM = PadMat<W>;
    static constexpr int ZW = PM::RP * kGwRows;                   // float2 per warp row buffer
    static size_t smem(int K, int C)
    {
        return (size_t)(W + 2 * STAGE + kGwWarps * ZW) * sizeof(float2) + (size_t)256 * K * sizeof(float) +
               (size_t)kGwWarps * C * kGwRows * W * sizeof(float);
    }
};

template <int W>
__global__ void __launch_bounds__(kGwWarps * 32) k_growth_warp(GrowthJobs jobs, const float2 *__restrict__ tw_x,
                                                               const float *__restrict__ lut_rows,
                                                               const float *__restrict__ A, float *__restrict__ Hout,
                                                               float *__restrict__ Uout, float *__restrict__ BACK,
                                                               float *__restrict__ Udbg, int *err_flag)
{
    using S = GrowthWarpShape<W>;
    constexpr int H = W, D = W, KX = S::KX, CELLS = S::CELLS, RB = kGwRowsBlock;
    constexpr int T = kGwRows * W;  // cells of a warp
    constexpr long long N = (long long)W * W * W;
    extern __shared__ float2 smem[];
    float2 *tw = smem;
    float2 *stage = tw + W;                          // [2][kernel 0/1][KX][RB]
    float2 *zrows = stage + 2 * S::STAGE;            // [warp][PadMat rows]
    float *lut = reinterpret_cast<float *>(zrows + kGwWarps * S::ZW);
    float *uall = lut + 256 * jobs.K;                // [warp][C][T]
    const int C = jobs.C, K = jobs.K;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int z = blockIdx.x / (H / RB);
    const int y0 = (blockIdx.x % (H / RB)) * RB;
    const int yw = warp * kGwRows;                   // first row of this warp within the block
    const long long base = ((long long)z * H + y0 + yw) * W;
    float2 *zb = zrows + warp * S::ZW;
    float *uacc = uall + warp * C * T;
    for (int i = threadIdx.x; i < W; i += kGwWarps * 32) tw[i] = tw_x[i];
    for (int i = threadIdx.x; i < 256 * K; i += kGwWarps * 32) lut[i] = lut_rows[i];
    for (int i = lane; i < C * T; i += 32) uacc[i] = 0.0f;

    auto issue = [&](int k0, int buf) {
        float2 *dst = stage + buf * S::STAGE;
        for (int e = threadIdx.x; e < 2 * KX * RB; e += kGwWarps * 32) {
            const int q = e / (KX * RB), rem = e % (KX * RB);
            const int kx = rem / RB, ty = rem % RB;
            const int k = k0 + q;
            const bool ok = k < K;
            const float2 *src = ok ? jobs.spec[k] + ((long long)kx * D + z) * H + y0 + ty : jobs.spec[k0];
            cp_async_f64(dst + (q * KX + kx) * S::SP + ty, src, ok);
        }
        cp_async_commit();
    };

    float hacc[CELLS][kMaxChannels];
#pragma unroll
    for (int i = 0; i < CELLS; i++)
#pragma unroll
        for (int c = 0; c < kMaxChannels; c++) hacc[i][c] = 0.0f;
    int bad = 0;
    constexpr bool kPow2 = (N & (N - 1)) == 0;
    constexpr float kInvN = 1.0f / (float)N;
    const float nf = (float)N;
    if (K > 0) issue(0, 0);
    for (int k0 = 0, it = 0; k0 < K; k0 += 2, it++) {
        const int k1 = k0 + 1 < K ? k0 + 1 : -1;
        cp_async_wait<0>();
        __syncthreads();  // staged pair visible; every warp is done with the other buffer
        if (k0 + 2 < K) issue(k0 + 2, (it + 1) & 1);
        const float2 *st = stage + (it & 1) * S::STAGE;
        // packed rows of this warp: element (r, kx), kx over the full length
#pragma unroll
        for (int i = 0; i < CELLS; i++) {
            const int e = lane + 32 * i;
            const int r = e % kGwRows, kx = e / kGwRows;
            const int m = kx < KX ? kx : W - kx;
            const float2 a = st[m * S::SP + yw + r];
            const float2 b = st[(KX + m) * S::SP + yw + r];
            float2 v;
            if (kx < KX) v = make_float2(a.x - b.y, a.y + b.x);
            else v = make_float2(a.x + b.y, b.x - a.y);
            zb[S::PM::at(r, kx)] = v;
        }
        __syncwarp();
        warp_fft_rows<W, kGwRows, W>(zb, tw, +1);
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int k = q == 0 ? k0 : k1;
            if (k < 0) continue;
            const int c1 = jobs.c1[k];
            const float h = jobs.h[k];
            const int asym = jobs.asymptotic[c1];
            float g[CELLS];
#pragma unroll
            for (int i = 0; i < CELLS; i++) {
                const int e = lane + 32 * i;
                const float2 zz = zb[S::PM::at(e / W, e % W)];
                const float re = q == 0 ? zz.x : zz.y;
                const float u = kPow2 ? re * kInvN : re / nf;
                const int ui = (int)(u * 255);
                float l;
                if (jobs.exact_bell) {
                    if (!(u == u)) bad = 1;
                    l = bell_dev(u, jobs.m[k], jobs.s[k]);
                } else if (ui >= 0 && ui < 256) l = lut[k * 256 + ui];
                else {
                    if (!(u == u)) bad = 1;
                    l = lut_flat_dev((long long)jobs.lut_base[k] + ui);
                }
                g[i] = asym ? (l - __ldg(A + (long long)c1 * N + base + e)) * h : l * h;
                uacc[c1 * T + e] = uacc[c1 * T + e] + u;
                if (Udbg) Udbg[(long long)k * N + base + e] = u;
            }
            switch (c1) {
#define LENIA_ACC(cc)                                                                       \
    case cc:                                                                                \
        _Pragma("unroll") for (int i = 0; i < CELLS; i++) hacc[i][cc] = hacc[i][cc] + g[i]; \
        break;
                LENIA_ACC(0) LENIA_ACC(1) LENIA_ACC(2) LENIA_ACC(3)
#undef LENIA_ACC
            }
        }
        __syncwarp();
    }
#pragma unroll
    for (int i = 0; i < CELLS; i++) {
        const int e = lane + 32 * i;
#pragma unroll
        for (int c = 0; c < kMaxChannels; c++) {
            if (c >= C) continue;
            const long long o = (long long)c * N + base + e;
            const float hv = hacc[i][c];
            Hout[o] = hv;
            const float us = uacc[c * T + e];
            Uout[o] = us;
            if (!isfinite(us)) bad = 1;  // a NaN u indexes the table at 0: test the sum
            if (jobs.growth_rt) BACK[o] = early_growth(__ldg(A + o), hv, jobs.timestep, jobs.soft_clip[c]);
        }
    }
    if (bad && err_flag) atomicOr(err_flag, 1);
}

template <int W, typename J>
__global__ void __launch_bounds__(kFastRowThreads) k_blur_rows_s(J jobs, const float2 *__restrict__ tw_x)
{
    using S = RowShape<W>;
    constexpr int H = W, TY = S::TY, T = S::T;
    constexpr long long N = (long long)W * W * W;
    extern __shared__ float2 smem[];
    float2 *tw = smem;
    float2 *buf = tw + W;
    const int z = blockIdx.x / (H / TY);
    const int y0 = (blockIdx.x % (H / TY)) * TY;
    const int pair = blockIdx.y;
    const long long base = ((long long)z * H + y0) * W;
    const float nf = (float)N;
    for (int i = threadIdx.x; i < W; i += kFastRowThreads) tw[i] = tw_x[i];
    pdl_trigger();
    pdl_wait();
    const float2 *s1 = inv_spec(jobs, pair, 1);
    float *o0 = inv_out(jobs, pair, 0), *o1 = inv_out(jobs, pair, 1);
    load_packed_rows_s<W>(buf, inv_spec(jobs, pair, 0), s1, z, y0);
    __syncthreads();
    static_fft<W, TY, false, W, kFastRowThreads>(buf, tw, +1);
    for (int e = threadIdx.x; e < T; e += kFastRowThreads) {
        const float2 zz = buf[S::PM::at(e / W, e % W)];
        o0[base + e] = zz.x / nf;
        if (s1) o1[base + e] = zz.y / nf;
    }
}

cudaError_t smem_attr(const void *fn, size_t bytes)
{
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int W>
cudaError_t fwd_rows_w(const Dims &d, const float2 *tw, const FwdRowJobs &jobs, cudaStream_t st)
{
    using S = RowShape<W>;
    const size_t smem = (size_t)(W + S::PM::size(S::TY)) * sizeof(float2);
    cudaError_t e = smem_attr((const void *)k_fwd_rows_s<W, FwdRowJobs>, smem);
    if (e != cudaSuccess) return e;
    return launch_pdl(k_fwd_rows_s<W, FwdRowJobs>, dim3(W * (W / S::TY), jobs.npairs), dim3(kFastRowThreads), smem, st,
                      jobs, tw);
}

template <int W>
cudaError_t planes_w(const Dims &d, const float2 *twy, const float2 *twz, const PlaneJobs &jobs, int sign,
                     cudaStream_t st)
{
    const size_t smem = (size_t)(2 * W + PadMat<W>::size(W)) * sizeof(float2);
    if constexpr (planes_persistent<W>()) {
        cudaError_t e = smem_attr((const void *)k_planes_stream_s<W>, smem);
        if (e != cudaSuccess) return e;
        // one resident wave of blocks; each walks its planes with stride grid
        static int resident = 0;
        if (resident == 0) {
            int dev = 0, nsm = 0, per_sm = 0;
            e = cudaGetDevice(&dev);
            if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            if (e == cudaSuccess)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_planes_stream_s<W>, kFastPlaneThreads,
                                                                  smem);
            if (e != cudaSuccess) return e;
            resident = nsm * (per_sm > 0 ? per_sm : 1);
        }
        const int units = (W / 2 + 1) * jobs.njobs;
        return launch_pdl(k_planes_stream_s<W>, dim3(units < resident ? units : resident), dim3(kFastPlaneThreads),
                          smem, st, jobs, twy, twz, sign);
    } else {
        cudaError_t e = smem_attr((const void *)k_planes_s<W, PlaneJobs>, smem);
        if (e != cudaSuccess) return e;
        return launch_pdl(k_planes_s<W, PlaneJobs>, dim3(W / 2 + 1, jobs.njobs), dim3(kFastPlaneThreads), smem, st,
                          jobs, twy, twz, sign);
    }
}

template <int W>
cudaError_t planes_split_w(const float2 *twy, const float2 *twz, const PlaneJobs &jobs, int sign, cudaStream_t st)
{
    static_assert(W % kSplitLines == 0, "split plane passes take whole line groups");
    const size_t sy = (size_t)(W + PadMat<W>::size(kSplitLines)) * sizeof(float2);
    const size_t sz = (size_t)(W + PadMat<kSplitLines>::size(W)) * sizeof(float2);
    cudaError_t e = smem_attr((const void *)k_plane_lines_y_s<W>, sy);
    if (e == cudaSuccess) e = smem_attr((const void *)k_plane_lines_z_s<W>, sz);
    if (e != cudaSuccess) return e;
    const dim3 grid(W / 2 + 1, W / kSplitLines, jobs.njobs);
    e = launch_pdl(k_plane_lines_y_s<W>, grid, dim3(kSplitThreads), sy, st, jobs, twy, sign);
    if (e != cudaSuccess) return e;
    return launch_pdl(k_plane_lines_z_s<W>, grid, dim3(kSplitThreads), sz, st, jobs, twz, sign);
}

template <int W>
cudaError_t growth_rows_w(const float2 *tw, const GrowthJobs &jobs, const float *lut, const float *A, float *H,
                          float *U, float *BACK, float *Udbg, int *err, cudaStream_t st)
{
    // The block-level pass measured faster than the warp-level one at 128^3
    // (200 vs 211 us for 4 channels x 16 kernels); LENIA_GROWTH_WARP selects
    // the warp-level pass.
#ifdef LENIA_GROWTH_WARP
    if constexpr (W % kGwRowsBlock == 0 && (kGwRows * W) % 32 == 0) {
#else
    if constexpr (false) {
#endif
        using G = GrowthWarpShape<W>;
        const size_t smem = G::smem(jobs.K, jobs.C);
        cudaError_t e = smem_attr((const void *)k_growth_warp<W>, smem);
        if (e != cudaSuccess) return e;
        k_growth_warp<W><<<W * (W / kGwRowsBlock), kGwWarps * 32, smem, st>>>(jobs, tw, lut, A, H, U, BACK, Udbg,
                                                                              err);
        return cudaGetLastError();
    } else {
        using S = RowShape<W, true>;
        const size_t smem = (size_t)(W + S::PM::size(S::TY)) * sizeof(float2) + (size_t)256 * jobs.K * sizeof(float) +
                            (size_t)jobs.C * S::T * sizeof(float);
        auto kern = jobs.exact_bell ? k_growth_rows_s<W, true> : k_growth_rows_s<W, false>;
        cudaError_t e = smem_attr((const void *)kern, smem);
        if (e != cudaSuccess) return e;
        return launch_pdl(kern, dim3(W * (W / S::TY)), dim3(kGrowthThreads), smem, st, jobs, tw, lut, A, H, U, BACK,
                          Udbg, err);
    }
}

template <int W>
cudaError_t blur_rows_w(const float2 *tw, const BlurJobs &jobs, cudaStream_t st)
{
    using S = RowShape<W>;
    const size_t smem = (size_t)(W + S::PM::size(S::TY)) * sizeof(float2);
    cudaError_t e = smem_attr((const void *)k_blur_rows_s<W, BlurJobs>, smem);
    if (e != cudaSuccess) return e;
    return launch_pdl(k_blur_rows_s<W, BlurJobs>, dim3(W * (W / S::TY), (jobs.nfields + 1) / 2),
                      dim3(kFastRowThreads), smem, st, jobs, tw);
}

// Batched forms: the same kernels over device job lists (grid y = entries).
template <int W>
cudaError_t fwd_rows_list_w(const float2 *tw, RowPairList jobs, cudaStream_t st)
{
    using S = RowShape<W>;
    const size_t smem = (size_t)(W + S::PM::size(S::TY)) * sizeof(float2);
    cudaError_t e = smem_attr((const void *)k_fwd_rows_s<W, RowPairList>, smem);
    if (e != cudaSuccess || jobs.n == 0) return e;
    // the jobs run as grid.y, at most kMaxGridY per launch
    for (int j0 = 0; j0 < jobs.n && e == cudaSuccess; j0 += kMaxGridY) {
        const RowPairList part{jobs.j + j0, std::min(jobs.n - j0, kMaxGridY)};
        k_fwd_rows_s<W, RowPairList><<<dim3(W * (W / S::TY), part.n), kFastRowThreads, smem, st>>>(part, tw);
        e = cudaGetLastError();
    }
    return e;
}

template <int W>
cudaError_t planes_list_w(const float2 *twy, const float2 *twz, PlaneJobList jobs, int sign, cudaStream_t st)
{
    static_assert(!planes_persistent<W>(), "batched plane passes take one plane per block");
    const size_t smem = (size_t)(2 * W + PadMat<W>::size(W)) * sizeof(float2);
    cudaError_t e = smem_attr((const void *)k_planes_s<W, PlaneJobList>, smem);
    if (e != cudaSuccess || jobs.n == 0) return e;
    for (int j0 = 0; j0 < jobs.n && e == cudaSuccess; j0 += kMaxGridY) {
        const PlaneJobList part{jobs.j + j0, std::min(jobs.n - j0, kMaxGridY)};
        k_planes_s<W, PlaneJobList><<<dim3(W / 2 + 1, part.n), kFastPlaneThreads, smem, st>>>(part, twy, twz, sign);
        e = cudaGetLastError();
    }
    return e;
}

template <int W>
cudaError_t inv_rows_list_w(const float2 *tw, InvPairList jobs, cudaStream_t st)
{
    using S = RowShape<W>;
    const size_t smem = (size_t)(W + S::PM::size(S::TY)) * sizeof(float2);
    cudaError_t e = smem_attr((const void *)k_blur_rows_s<W, InvPairList>, smem);
    if (e != cudaSuccess || jobs.n == 0) return e;
    for (int j0 = 0; j0 < jobs.n && e == cudaSuccess; j0 += kMaxGridY) {
        const InvPairList part{jobs.j + j0, std::min(jobs.n - j0, kMaxGridY)};
        k_blur_rows_s<W, InvPairList><<<dim3(W * (W / S::TY), part.n), kFastRowThreads, smem, st>>>(part, tw);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace

#define LENIA_FAST_SIZES(X) X(24) X(32) X(36) X(44) X(48) X(64) X(96) X(128)
// Row transforms also for 256: a 256 x 256 plane does not fit shared memory,
// so the plane transforms of that size run as the runtime-sized split passes.
#define LENIA_FAST_ROW_SIZES(X) LENIA_FAST_SIZES(X) X(256)

bool fast_supported(const Dims &d)
{
    if (d.W != d.H) return false;
    switch (d.W) {
#define CASE(n) case n:
        LENIA_FAST_SIZES(CASE)
#undef CASE
        return true;
    default: return false;
    }
}

bool fast_rows_supported(const Dims &d)
{
    if (d.W != d.H) return false;
    switch (d.W) {
#define CASE(n) case n:
        LENIA_FAST_ROW_SIZES(CASE)
#undef CASE
        return true;
    default: return false;
    }
}

cudaError_t launch_fwd_rows_fast(const Dims &d, const float2 *tw_x, const FwdRowJobs &jobs, cudaStream_t st)
{
    switch (d.W) {
#define CASE(n) case n: return fwd_rows_w<n>(d, tw_x, jobs, st);
        LENIA_FAST_ROW_SIZES(CASE)
#undef CASE
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_planes_fast(const Dims &d, const float2 *tw_y, const float2 *tw_z, const PlaneJobs &jobs, int sign,
                               cudaStream_t st)
{
    switch (d.W) {
#define CASE(n) case n: return planes_w<n>(d, tw_y, tw_z, jobs, sign, st);
        LENIA_FAST_SIZES(CASE)
#undef CASE
    default: return cudaErrorInvalidValue;
    }
}

bool fast_split_planes_supported(const Dims &d) { return d.W == d.H && d.W == 256; }

// Grid sizes of the batched launches: the size-specialised kernels with one
// plane per block.
#define LENIA_LIST_SIZES(X) X(24) X(32) X(36) X(44) X(48) X(64) X(96)

bool list_size_supported(int W)
{
    switch (W) {
#define CASE(n) case n:
        LENIA_LIST_SIZES(CASE)
#undef CASE
        return true;
    default: return false;
    }
}

cudaError_t launch_fwd_rows_list(int W, const float2 *tw_x, RowPairList jobs, cudaStream_t st)
{
    switch (W) {
#define CASE(n) case n: return fwd_rows_list_w<n>(tw_x, jobs, st);
        LENIA_LIST_SIZES(CASE)
#undef CASE
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_planes_list(int W, const float2 *tw_y, const float2 *tw_z, PlaneJobList jobs, int sign,
                               cudaStream_t st)
{
    switch (W) {
#define CASE(n) case n: return planes_list_w<n>(tw_y, tw_z, jobs, sign, st);
        LENIA_LIST_SIZES(CASE)
#undef CASE
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_inv_rows_list(int W, const float2 *tw_x_inv, InvPairList jobs, cudaStream_t st)
{
    switch (W) {
#define CASE(n) case n: return inv_rows_list_w<n>(tw_x_inv, jobs, st);
        LENIA_LIST_SIZES(CASE)
#undef CASE
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_planes_split_fast(const Dims &d, const float2 *tw_y, const float2 *tw_z, const PlaneJobs &jobs,
                                     int sign, cudaStream_t st)
{
    if (d.W == 256 && d.H == 256) return planes_split_w<256>(tw_y, tw_z, jobs, sign, st);
    return cudaErrorInvalidValue;
}

cudaError_t launch_growth_rows_fast(const Dims &d, const float2 *tw_x_inv, const GrowthJobs &jobs,
                                    const float *lut_rows, const float *A, float *H, float *U_SUM, float *BACK,
                                    float *U_dbg, int *err_flag, cudaStream_t st)
{
    switch (d.W) {
#define CASE(n) \
    case n: return growth_rows_w<n>(tw_x_inv, jobs, lut_rows, A, H, U_SUM, BACK, U_dbg, err_flag, st);
        LENIA_FAST_ROW_SIZES(CASE)
#undef CASE
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_blur_rows_fast(const Dims &d, const float2 *tw_x_inv, const BlurJobs &jobs, cudaStream_t st)
{
    switch (d.W) {
#define CASE(n) case n: return blur_rows_w<n>(tw_x_inv, jobs, st);
        LENIA_FAST_ROW_SIZES(CASE)
#undef CASE
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace lenia
