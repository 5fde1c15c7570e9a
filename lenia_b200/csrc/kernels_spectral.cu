// Spectral convolution of the 3D Flow Lenia step (lenia.cpp:435-594,
// reintegration.cpp:13-188) on sm_100a.
//
// The reference runs a full complex 3D FFTW transform per channel (forward)
// and per kernel (inverse).  Here every transform is the project's LFFT
// (lfft_device.cuh) arranged as a half-spectrum convolution:
//   fwd_rows   two real fields packed as a + i b, x-transform per row, split
//              into the two half spectra kx in [0, W/2], stored [kx][z][y];
//   planes     per kx plane (D x H complex in shared memory) the y- then
//              z-transform, optionally multiplied first by the real kernel
//              spectrum (octant-compressed, read through |k| symmetry);
//   growth     per row tile two kernels packed as S0 + i S1, extended over
//              kx by Hermitian symmetry, inverse x-transform, u = re/N,
//              im/N, then the growth-table accumulation of mt_fft_step
//              (lenia.cpp:501-538) in kernel order and the early growth into
//              BACK (lenia.cpp:542-592), all in one kernel.
// The same arrangement is written out on the CPU (oracle/restate) so results
// can be compared bit for bit.
#include "lenia_internal.h"
#include "growth_common.cuh"

namespace lenia {

// ------------------------------------------------------------ forward rows

template <int CAP>
__global__ void __launch_bounds__(kRowThreads) k_fwd_rows(Dims d, FftPlan px, const float2 *__restrict__ tw_x,
                                                          FwdRowJobs jobs, int TY)
{
    extern __shared__ float2 smem[];
    float2 *tw = smem;
    float2 *buf = smem + d.W;
    const int W = d.W, H = d.H, D = d.D;
    const int tiles_y = H / TY;
    const int z = blockIdx.x / tiles_y;
    const int y0 = (blockIdx.x % tiles_y) * TY;
    const int pair = blockIdx.y;
    const float *fa = jobs.in[2 * pair];
    const float *fb = jobs.in[2 * pair + 1];
    float2 *oa = jobs.out[2 * pair];
    float2 *ob = jobs.out[2 * pair + 1];

    for (int i = threadIdx.x; i < W; i += blockDim.x) tw[i] = tw_x[i];
    const long long base = ((long long)z * H + y0) * W;
    for (int e = threadIdx.x; e < TY * W; e += blockDim.x) {
        float a = fa[base + e];
        float b = fb ? fb[base + e] : 0.0f;
        buf[e] = make_float2(a, b);
    }
    __syncthreads();
    fft_lines<CAP>(buf, px, TY, 1, W, tw, -1, false);
    const int KX = d.KX;
    for (int e = threadIdx.x; e < TY * KX; e += blockDim.x) {
        const int ty = e % TY, kx = e / TY;
        const float2 p = buf[ty * W + kx];
        const float2 q = buf[ty * W + (W - kx) % W];
        const long long o = ((long long)kx * D + z) * H + y0 + ty;
        oa[o] = make_float2((p.x + q.x) * 0.5f, (p.y - q.y) * 0.5f);
        if (ob) ob[o] = make_float2((p.y + q.y) * 0.5f, (q.x - p.x) * 0.5f);
    }
}

// ------------------------------------------------------------------ planes

__global__ void __launch_bounds__(kPlaneThreads) k_planes(Dims d, FftPlan py, FftPlan pz,
                                                          const float2 *__restrict__ tw_y,
                                                          const float2 *__restrict__ tw_z, PlaneJobs jobs,
                                                          int sign)
{
    extern __shared__ float2 smem[];
    const int H = d.H, D = d.D;
    float2 *twy = smem;
    float2 *twz = smem + H;
    float2 *buf = smem + H + D;
    const int kx = blockIdx.x;
    const int job = blockIdx.y;
    const float2 *src = jobs.src[job] + (long long)kx * D * H;
    float2 *dst = jobs.dst[job] + (long long)kx * D * H;
    const float *kc = jobs.kc[job];
    for (int i = threadIdx.x; i < H; i += blockDim.x) twy[i] = tw_y[i];
    for (int i = threadIdx.x; i < D; i += blockDim.x) twz[i] = tw_z[i];
    const int KZ = D / 2 + 1, KY = H / 2 + 1;
    if (kc) {
        const float *kp = kc + (long long)kx * KZ * KY;
        for (int e = threadIdx.x; e < D * H; e += blockDim.x) {
            const int z = e / H, y = e % H;
            const int oz = z <= D - z ? z : D - z;
            const int oy = y <= H - y ? y : H - y;
            const float k = kp[oz * KY + oy];
            const float2 t = src[e];
            buf[e] = make_float2(t.x * k, t.y * k);
        }
    } else {
        for (int e = threadIdx.x; e < D * H; e += blockDim.x) buf[e] = src[e];
    }
    __syncthreads();
    fft_lines<kPlaneCap>(buf, py, D, 1, H, twy, sign, false);
    fft_lines<kPlaneCap>(buf, pz, H, H, 1, twz, sign, true);
    for (int e = threadIdx.x; e < D * H; e += blockDim.x) dst[e] = buf[e];
}

// Planes larger than shared memory: the same two line transforms as
// k_planes, each as its own pass through global memory.  Pass y transforms
// TZ consecutive z-lines of one kx plane (after the optional kernel product);
// pass z transforms TY consecutive y-columns.  Every line goes through the
// same 1-D transform as in k_planes, so results are identical.
__global__ void __launch_bounds__(kPlaneThreads) k_plane_lines_y(Dims d, FftPlan py, const float2 *__restrict__ tw_y,
                                                                 PlaneJobs jobs, int sign, int TZ)
{
    extern __shared__ float2 smem[];
    const int H = d.H, D = d.D;
    float2 *twy = smem;
    float2 *buf = smem + H;
    const int kx = blockIdx.x;
    const int z0 = blockIdx.y * TZ;
    const int job = blockIdx.z;
    const long long base = ((long long)kx * D + z0) * H;
    const float2 *src = jobs.src[job] + base;
    float2 *dst = jobs.dst[job] + base;
    const float *kc = jobs.kc[job];
    for (int i = threadIdx.x; i < H; i += blockDim.x) twy[i] = tw_y[i];
    const int KZ = D / 2 + 1, KY = H / 2 + 1;
    if (kc) {
        const float *kp = kc + (long long)kx * KZ * KY;
        for (int e = threadIdx.x; e < TZ * H; e += blockDim.x) {
            const int z = z0 + e / H, y = e % H;
            const int oz = z <= D - z ? z : D - z;
            const int oy = y <= H - y ? y : H - y;
            const float k = kp[oz * KY + oy];
            const float2 t = src[e];
            buf[e] = make_float2(t.x * k, t.y * k);
        }
    } else {
        for (int e = threadIdx.x; e < TZ * H; e += blockDim.x) buf[e] = src[e];
    }
    __syncthreads();
    fft_lines<kPlaneCap>(buf, py, TZ, 1, H, twy, sign, false);
    for (int e = threadIdx.x; e < TZ * H; e += blockDim.x) dst[e] = buf[e];
}

__global__ void __launch_bounds__(kPlaneThreads) k_plane_lines_z(Dims d, FftPlan pz, const float2 *__restrict__ tw_z,
                                                                 PlaneJobs jobs, int sign, int TY)
{
    extern __shared__ float2 smem[];
    const int H = d.H, D = d.D;
    float2 *twz = smem;
    float2 *buf = smem + D;
    const int kx = blockIdx.x;
    const int y0 = blockIdx.y * TY;
    const int job = blockIdx.z;
    float2 *dst = jobs.dst[job] + (long long)kx * D * H + y0;
    for (int i = threadIdx.x; i < D; i += blockDim.x) twz[i] = tw_z[i];
    for (int e = threadIdx.x; e < D * TY; e += blockDim.x) {
        const int z = e / TY, t = e % TY;
        buf[e] = dst[(long long)z * H + t];
    }
    __syncthreads();
    fft_lines<kPlaneCap>(buf, pz, TY, TY, 1, twz, sign, true);
    for (int e = threadIdx.x; e < D * TY; e += blockDim.x) {
        const int z = e / TY, t = e % TY;
        dst[(long long)z * H + t] = buf[e];
    }
}

// ------------------------------------------------- inverse rows: growth

// Builds the packed row spectrum of kernels (s0, s1) for one row tile.
__device__ __forceinline__ void load_packed_rows(float2 *buf, const Dims &d, const float2 *s0, const float2 *s1,
                                                 int z, int y0, int TY)
{
    const int W = d.W, H = d.H, D = d.D, KX = d.KX;
    for (int e = threadIdx.x; e < TY * W; e += blockDim.x) {
        const int ty = e % TY, kx = e / TY;
        const int m = kx < KX ? kx : W - kx;
        const long long o = ((long long)m * D + z) * H + y0 + ty;
        const float2 a = s0[o];
        const float2 b = s1 ? s1[o] : make_float2(0.0f, 0.0f);
        float2 r;
        if (kx < KX) r = make_float2(a.x - b.y, a.y + b.x);
        else r = make_float2(a.x + b.y, b.x - a.y);
        buf[ty * W + kx] = r;
    }
}

template <int CAP>
__global__ void __launch_bounds__(kRowThreads) k_growth_rows(Dims d, FftPlan px, const float2 *__restrict__ tw_x,
                                                             GrowthJobs jobs, const float *__restrict__ lut_rows,
                                                             const float *__restrict__ A, float *__restrict__ Hout,
                                                             float *__restrict__ Uout, float *__restrict__ BACK,
                                                             float *__restrict__ Udbg, int *err_flag, int TY)
{
    extern __shared__ float2 smem[];
    const int W = d.W, H = d.H;
    const int C = jobs.C, K = jobs.K;
    const int T = TY * W;
    float2 *tw = smem;
    float2 *buf = tw + W;
    float *lut = (float *)(buf + T);
    float *hacc = lut + 256 * K;
    float *uacc = hacc + C * T;
    const int tiles_y = H / TY;
    const int z = blockIdx.x / tiles_y;
    const int y0 = (blockIdx.x % tiles_y) * TY;
    const long long base = ((long long)z * H + y0) * W;
    const float nf = (float)d.N;

    for (int i = threadIdx.x; i < W; i += blockDim.x) tw[i] = tw_x[i];
    for (int i = threadIdx.x; i < 256 * K; i += blockDim.x) lut[i] = lut_rows[i];
    for (int i = threadIdx.x; i < C * T; i += blockDim.x) {
        hacc[i] = 0.0f;
        uacc[i] = 0.0f;
    }
    int bad = 0;
    for (int k0 = 0; k0 < K; k0 += 2) {
        const int k1 = k0 + 1 < K ? k0 + 1 : -1;
        load_packed_rows(buf, d, jobs.spec[k0], k1 >= 0 ? jobs.spec[k1] : nullptr, z, y0, TY);
        __syncthreads();
        fft_lines<CAP>(buf, px, TY, 1, W, tw, +1, false);
        for (int e = threadIdx.x; e < T; e += blockDim.x) {
            const float2 zz = buf[e];
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const int k = q == 0 ? k0 : k1;
                if (k < 0) continue;
                const float u = (q == 0 ? zz.x : zz.y) / nf;
                const int c = jobs.c1[k];
                const float h = jobs.h[k];
                uacc[c * T + e] = uacc[c * T + e] + u;
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
                float g;
                if (jobs.asymptotic[c]) g = (l - A[(long long)c * d.N + base + e]) * h;
                else g = l * h;
                hacc[c * T + e] = hacc[c * T + e] + g;
                if (Udbg) Udbg[(long long)k * d.N + base + e] = u;
            }
        }
        __syncthreads();
    }
    for (int c = 0; c < C; c++) {
        for (int e = threadIdx.x; e < T; e += blockDim.x) {
            const long long o = (long long)c * d.N + base + e;
            const float hv = hacc[c * T + e];
            Hout[o] = hv;
            const float us = uacc[c * T + e];
            Uout[o] = us;
            if (!isfinite(us)) bad = 1;  // a NaN u indexes the table at 0: test the sum
            if (jobs.growth_rt) BACK[o] = early_growth(A[o], hv, jobs.timestep, jobs.soft_clip[c]);
        }
    }
    if (bad && err_flag) atomicOr(err_flag, 1);
}

// --------------------------------------------------- inverse rows: blur

template <int CAP>
__global__ void __launch_bounds__(kRowThreads) k_blur_rows(Dims d, FftPlan px, const float2 *__restrict__ tw_x,
                                                           BlurJobs jobs, int TY)
{
    extern __shared__ float2 smem[];
    const int W = d.W, H = d.H;
    const int T = TY * W;
    float2 *tw = smem;
    float2 *buf = tw + W;
    const int tiles_y = H / TY;
    const int z = blockIdx.x / tiles_y;
    const int y0 = (blockIdx.x % tiles_y) * TY;
    const int pair = blockIdx.y;
    const long long base = ((long long)z * H + y0) * W;
    const float nf = (float)d.N;
    for (int i = threadIdx.x; i < W; i += blockDim.x) tw[i] = tw_x[i];
    const int f0 = 2 * pair, f1 = 2 * pair + 1 < jobs.nfields ? 2 * pair + 1 : -1;
    load_packed_rows(buf, d, jobs.spec[f0], f1 >= 0 ? jobs.spec[f1] : nullptr, z, y0, TY);
    __syncthreads();
    fft_lines<CAP>(buf, px, TY, 1, W, tw, +1, false);
    for (int e = threadIdx.x; e < T; e += blockDim.x) {
        const float2 zz = buf[e];
        jobs.out[f0][base + e] = zz.x / nf;
        if (f1 >= 0) jobs.out[f1][base + e] = zz.y / nf;
    }
}

// ------------------------------------------------------ kernel building

// Value of kernel cell (gx, gy, gz) as init_kernel places it
// (lenia.cpp:215-245): r = the offset in [-W/2, W/2) whose emod is g.
__device__ __forceinline__ float kernel_value(const LeniaKernelParams &kp, int rx, int ry, int rz)
{
    const float x = fabsf((float)rx), y = fabsf((float)ry), z = fabsf((float)rz);
    float dist = sqrtf(x * x + y * y + z * z);
    dist = dist / (float)kp.radius * (float)kp.beta_size / kp.r_a;
    if (!(dist < (float)kp.beta_size)) return 0.0f;
    const int fi = (int)floorf(dist);
    const int index = fi < kp.beta_size - 1 ? fi : kp.beta_size - 1;
    return kp.b[index] * bell_dev(fmodf(dist, 1.0f), 0.5f, 0.15f);
}

__global__ void k_kernel_values(Dims d, const LeniaKernelParams *__restrict__ kps, float *grids)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.N) return;
    const int k = blockIdx.y;
    const int gx = (int)(i % d.W), gy = (int)((i / d.W) % d.H), gz = (int)(i / ((long long)d.W * d.H));
    const int rx = gx < d.W / 2 ? gx : gx - d.W;
    const int ry = gy < d.H / 2 ? gy : gy - d.H;
    const int rz = gz < d.D / 2 ? gz : gz - d.D;
    grids[(long long)k * d.N + i] = kernel_value(kps[k], rx, ry, rz);
}

// Sum of the cell values in the reference's (r_x, r_y, r_z) loop order, in
// float (lenia.cpp:215-243); the normalisation (lenia.cpp:250-257) follows.
// Cells outside the box |r| <= bound hold +0 and leave the sum unchanged.
// The block stages the box's values 256 at a time into one of two shared
// buffers while thread 0 adds up the other one in order (one barrier per
// chunk; four values per shared-memory load); k_kernel_scale then divides.
__global__ void k_kernel_normalise(Dims d, const LeniaKernelParams *__restrict__ kps, float *grids,
                                   float *ksum, int blur)
{
    __shared__ __align__(16) float chunk[2][256];
    const int k = blockIdx.x;
    float *g = grids + (long long)k * d.N;
    int bx, by;
    if (blur) {
        bx = by = 2;
    } else {
        const LeniaKernelParams &kp = kps[k];
        const float ext = (float)kp.radius * kp.r_a;
        bx = by = (int)ceilf(ext) + 2;
    }
    const int ow = d.W / 2, oh = d.H / 2;
    const int x0 = bx < ow ? -bx : -ow, x1 = bx < ow ? bx : ow - 1;
    const int yl = by < oh ? -by : -oh, yh = by < oh ? by : oh - 1;
    const int nx = x1 - x0 + 1, ny = yh - yl + 1;
    const long long cnt = (long long)nx * ny * nx;
    // value c of the box in the reference's (r_x, r_y, r_z) loop order
    auto stage = [&](long long c0, float *dst) {
        const long long c = c0 + threadIdx.x;
        float v = 0.0f;
        if (c < cnt) {
            const int rz = (int)(c % nx) + x0;
            const int ry = (int)((c / nx) % ny) + yl;
            const int rx = (int)(c / ((long long)nx * ny)) + x0;
            const int gx = rx < 0 ? rx + d.W : rx, gy = ry < 0 ? ry + d.H : ry, gz = rz < 0 ? rz + d.D : rz;
            v = g[gx + (long long)gy * d.W + (long long)gz * d.W * d.H];
        }
        dst[threadIdx.x] = v;
    };
    float s = 0.0f;
    if (cnt > 0) stage(0, chunk[0]);
    __syncthreads();
    int it = 0;
    for (long long c0 = 0; c0 < cnt; c0 += 256, it++) {
        if (c0 + 256 < cnt) stage(c0 + 256, chunk[(it + 1) & 1]);
        if (threadIdx.x == 0) {
            const float4 *q = reinterpret_cast<const float4 *>(chunk[it & 1]);
            const int lim = cnt - c0 < 256 ? (int)(cnt - c0) : 256;
            int j = 0;
            for (; j + 4 <= lim; j += 4) {
                const float4 v = q[j / 4];
                s = s + v.x;
                s = s + v.y;
                s = s + v.z;
                s = s + v.w;
            }
            for (; j < lim; j++) s = s + chunk[it & 1][j];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) ksum[k] = s;
}

// The normalisation itself (lenia.cpp:250-257): every cell of kernel grid
// blockIdx.y divided by its sum, over a grid of blocks.
__global__ void k_kernel_scale(Dims d, float *grids, const float *__restrict__ ksum)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.N) return;
    float *g = grids + (long long)blockIdx.y * d.N;
    g[i] = g[i] / ksum[blockIdx.y];
}

// precompute_blur_kernel (reintegration.cpp:37-73): 5^3 exp(-d^2/s^3), s = 1.5.
__global__ void k_blur_values(Dims d, float *grid)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.N) return;
    const int gx = (int)(i % d.W), gy = (int)((i / d.W) % d.H), gz = (int)(i / ((long long)d.W * d.H));
    const int rx = gx < d.W / 2 ? gx : gx - d.W;
    const int ry = gy < d.H / 2 ? gy : gy - d.H;
    const int rz = gz < d.D / 2 ? gz : gz - d.D;
    float v = 0.0f;
    if (rx >= -2 && rx <= 2 && ry >= -2 && ry <= 2 && rz >= -2 && rz <= 2) {
        const float x = fabsf((float)rx), y = fabsf((float)ry), z = fabsf((float)rz);
        const float s = 1.5f;
        const float dist = x * x + y * y + z * z;
        // expf of the reference, evaluated as the correctly rounded float of
        // the double exponential (equal to the host libm on these arguments)
        v = (float)exp((double)(-dist / (s * s * s)));
    }
    grid[i] = v;
}

__global__ void k_compress(Dims d, const float2 *__restrict__ spec, float *kc)
{
    const int KZ = d.D / 2 + 1, KY = d.H / 2 + 1;
    const long long total = (long long)d.KX * KZ * KY;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int ky = (int)(i % KY), kz = (int)((i / KY) % KZ), kx = (int)(i / ((long long)KY * KZ));
    kc[i] = spec[((long long)kx * d.D + kz) * d.H + ky].x;
}

// Rows of the growth table for each kernel: LUT[m][s][u] for the kernel's
// truncated m and s indices (lenia.h:79-84).
__global__ void k_lut_rows(const LeniaKernelParams *__restrict__ kps, float *rows, int *bases)
{
    const int k = blockIdx.x, u = threadIdx.x;
    const int mi = (int)(kps[k].m * 255);
    const int si = (int)(kps[k].s * 255);
    const long long base = (long long)mi * 65536 + (long long)si * 256;
    rows[k * 256 + u] = lut_flat_dev(base + u);
    if (u == 0) bases[k] = (int)base;
}

// ------------------------------------------------------------- launches

static bool fits(const FftPlan &p, int nlines, int threads, int cap)
{
    for (int s = 0; s < p.nstages; s++) {
        const int r = p.radix[s];
        const long long total = (long long)nlines * (p.n / r);
        if (total > (long long)(cap / r) * threads) return false;
    }
    return true;
}

int row_tile(const Dims &d, const FftPlan &px)
{
    if (d.ty > 0 && d.H % d.ty == 0 && fits(px, d.ty, kRowThreads, kRowCap)) return d.ty;
    for (int ty = 32; ty >= 1; ty /= 2)
        if (d.H % ty == 0 && fits(px, ty, kRowThreads, kRowCap)) return ty;
    return 0;
}

constexpr long long kPlaneSmem = 200 * 1024;

// Lines per block of the split plane passes (0: none fits).
static int split_tile(int n_lines, int n, const FftPlan &p, int other)
{
    for (int t = 64; t >= 1; t /= 2)
        if (n_lines % t == 0 && fits(p, t, kPlaneThreads, kPlaneCap) &&
            (long long)t * n * 8 + (long long)other * 8 <= kPlaneSmem)
            return t;
    return 0;
}

bool plane_fits(const Dims &d, const FftPlan &py, const FftPlan &pz);

// Whether the plane transforms run, in one pass or in two.
bool planes_supported(const Dims &d, const FftPlan &py, const FftPlan &pz)
{
    return plane_fits(d, py, pz) || (split_tile(d.D, d.H, py, d.H) > 0 && split_tile(d.H, d.D, pz, d.D) > 0);
}

bool plane_fits(const Dims &d, const FftPlan &py, const FftPlan &pz)
{
    return (long long)d.D * d.H * 8 + (d.H + d.D) * 8 <= 200 * 1024 && fits(py, d.D, kPlaneThreads, kPlaneCap) &&
           fits(pz, d.H, kPlaneThreads, kPlaneCap);
}

static cudaError_t set_smem(const void *fn, size_t bytes)
{
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t launch_fwd_rows(const Dims &d, const FftPlan &px, const float2 *tw_x, const FwdRowJobs &jobs,
                            cudaStream_t st)
{
    if (fast_rows_supported(d)) return launch_fwd_rows_fast(d, tw_x, jobs, st);
    const int TY = row_tile(d, px);
    if (TY == 0) return cudaErrorInvalidValue;
    const size_t smem = (size_t)(d.W + TY * d.W) * sizeof(float2);
    cudaError_t e = set_smem((const void *)k_fwd_rows<kRowCap>, smem);
    if (e != cudaSuccess) return e;
    dim3 grid(d.D * (d.H / TY), jobs.npairs);
    k_fwd_rows<kRowCap><<<grid, kRowThreads, smem, st>>>(d, px, tw_x, jobs, TY);
    return cudaGetLastError();
}

cudaError_t launch_planes(const Dims &d, const FftPlan &py, const FftPlan &pz, const float2 *tw_y,
                          const float2 *tw_z, const PlaneJobs &jobs, int sign, cudaStream_t st)
{
    if (fast_supported(d)) return launch_planes_fast(d, tw_y, tw_z, jobs, sign, st);
    if (fast_split_planes_supported(d)) return launch_planes_split_fast(d, tw_y, tw_z, jobs, sign, st);
    if (!plane_fits(d, py, pz)) {
        const int TZ = split_tile(d.D, d.H, py, d.H), TY = split_tile(d.H, d.D, pz, d.D);
        if (TZ == 0 || TY == 0) return cudaErrorInvalidValue;
        const size_t sy = ((size_t)TZ * d.H + d.H) * sizeof(float2), sz = ((size_t)d.D * TY + d.D) * sizeof(float2);
        cudaError_t e = set_smem((const void *)k_plane_lines_y, sy);
        if (e == cudaSuccess) e = set_smem((const void *)k_plane_lines_z, sz);
        if (e != cudaSuccess) return e;
        k_plane_lines_y<<<dim3(d.KX, d.D / TZ, jobs.njobs), kPlaneThreads, sy, st>>>(d, py, tw_y, jobs, sign, TZ);
        k_plane_lines_z<<<dim3(d.KX, d.H / TY, jobs.njobs), kPlaneThreads, sz, st>>>(d, pz, tw_z, jobs, sign, TY);
        return cudaGetLastError();
    }
    const size_t smem = (size_t)(d.H + d.D + (long long)d.D * d.H) * sizeof(float2);
    cudaError_t e = set_smem((const void *)k_planes, smem);
    if (e != cudaSuccess) return e;
    dim3 grid(d.KX, jobs.njobs);
    k_planes<<<grid, kPlaneThreads, smem, st>>>(d, py, pz, tw_y, tw_z, jobs, sign);
    return cudaGetLastError();
}

cudaError_t launch_growth_rows(const Dims &d, const FftPlan &px, const float2 *tw_x_inv, const GrowthJobs &jobs,
                               const float *lut_rows, const float *A, float *H, float *U_SUM, float *BACK,
                               float *U_dbg, int *err_flag, cudaStream_t st)
{
    if (fast_rows_supported(d))
        return launch_growth_rows_fast(d, tw_x_inv, jobs, lut_rows, A, H, U_SUM, BACK, U_dbg, err_flag, st);
    int TY = row_tile(d, px);
    if (TY == 0) return cudaErrorInvalidValue;
    auto smem_for = [&](int ty) {
        return (size_t)(d.W + ty * d.W) * sizeof(float2) + (size_t)256 * jobs.K * sizeof(float) +
               (size_t)2 * jobs.C * ty * d.W * sizeof(float);
    };
    while (TY > 1 && smem_for(TY) > 200 * 1024) TY /= 2;
    const size_t smem = smem_for(TY);
    cudaError_t e = set_smem((const void *)k_growth_rows<kRowCap>, smem);
    if (e != cudaSuccess) return e;
    dim3 grid(d.D * (d.H / TY));
    k_growth_rows<kRowCap><<<grid, kRowThreads, smem, st>>>(d, px, tw_x_inv, jobs, lut_rows, A, H, U_SUM, BACK,
                                                            U_dbg, err_flag, TY);
    return cudaGetLastError();
}

cudaError_t launch_blur_rows(const Dims &d, const FftPlan &px, const float2 *tw_x_inv, const BlurJobs &jobs,
                             cudaStream_t st)
{
    if (fast_rows_supported(d)) return launch_blur_rows_fast(d, tw_x_inv, jobs, st);
    const int TY = row_tile(d, px);
    if (TY == 0) return cudaErrorInvalidValue;
    const size_t smem = (size_t)(d.W + TY * d.W) * sizeof(float2);
    cudaError_t e = set_smem((const void *)k_blur_rows<kRowCap>, smem);
    if (e != cudaSuccess) return e;
    dim3 grid(d.D * (d.H / TY), (jobs.nfields + 1) / 2);
    k_blur_rows<kRowCap><<<grid, kRowThreads, smem, st>>>(d, px, tw_x_inv, jobs, TY);
    return cudaGetLastError();
}

cudaError_t launch_kernel_grids(const Dims &d, const LeniaKernelParams *kp_dev, int K, float *grids, float *ksum,
                                cudaStream_t st)
{
    if (K == 0) return cudaSuccess;
    dim3 grid((unsigned)((d.N + 255) / 256), K);
    k_kernel_values<<<grid, 256, 0, st>>>(d, kp_dev, grids);
    k_kernel_normalise<<<K, 256, 0, st>>>(d, kp_dev, grids, ksum, 0);
    k_kernel_scale<<<dim3((unsigned)((d.N + 255) / 256), K), 256, 0, st>>>(d, grids, ksum);
    return cudaGetLastError();
}

cudaError_t launch_blur_grid(const Dims &d, float *grid, float *ksum, cudaStream_t st)
{
    k_blur_values<<<(unsigned)((d.N + 255) / 256), 256, 0, st>>>(d, grid);
    k_kernel_normalise<<<1, 256, 0, st>>>(d, nullptr, grid, ksum, 1);
    k_kernel_scale<<<dim3((unsigned)((d.N + 255) / 256), 1), 256, 0, st>>>(d, grid, ksum);
    return cudaGetLastError();
}

cudaError_t launch_compress(const Dims &d, const float2 *spec, float *kc, cudaStream_t st)
{
    const long long total = (long long)d.KX * (d.D / 2 + 1) * (d.H / 2 + 1);
    k_compress<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(d, spec, kc);
    return cudaGetLastError();
}

cudaError_t launch_lut_rows(const LeniaKernelParams *kp_dev, int K, float *lut_rows, int *lut_base, cudaStream_t st)
{
    if (K == 0) return cudaSuccess;
    k_lut_rows<<<K, 256, 0, st>>>(kp_dev, lut_rows, lut_base);
    return cudaGetLastError();
}

}  // namespace lenia
