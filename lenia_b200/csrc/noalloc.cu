// lenia_convolve_noalloc: the growth stage's convolution of one field with one
// kernel, for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: an application that embeds this library
// inside its own memory manager and has already reserved the device memory it
// is allowed to use, or a host loop that must not take the implicit
// device-wide synchronisation an allocation can cause.  For them this entry
// point keeps every intermediate buffer in one file-scope __device__ array of
// fixed size (kNoAllocBytes below: 4,439,040 bytes, about 4.4 MB), which each
// GPU that loads the library holds until the process exits.  The caller passes the input
// field and the output buffer, both in device memory.
//
// The array is shared by every call and keeps the last call's contents; every
// element a call reads is written earlier in the same call, so nothing needs
// clearing.  Calls that overlap on the GPU (different streams or threads
// without ordering) race on the array and give wrong results.
//
// The first call on a device looks up the array's device address with
// cudaGetSymbolAddress while that device is current (the host-side name of a
// __device__ array is not a device address) and keeps it for later calls on
// that device.  cudaDeviceReset unloads the library's device code, so the
// kept address is stale afterwards: do not call this entry point on a device
// after resetting it in the same process.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <atomic>

#include "lenia_internal.h"

using namespace lenia;

namespace {

constexpr int kNoAllocMaxCells = 64 * 64 * 64;        // largest grid accepted
constexpr int kNoAllocMaxDim = 64;
constexpr long long kNoAllocMaxHS = 33LL * 64 * 64;   // half-spectrum entries at 64^3
constexpr long long kNoAllocMaxKH = 33LL * 33 * 33;   // octant kernel entries at 64^3

// Layout of the scratch array (offsets in bytes, each 256-byte aligned).
constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kOffGrid = 0;                                                   // kernel grid, N floats
constexpr size_t kOffSpecField = kOffGrid + align256(kNoAllocMaxCells * 4);        // field half spectrum
constexpr size_t kOffSpecKern = kOffSpecField + align256(kNoAllocMaxHS * 8);      // kernel half spectrum
constexpr size_t kOffSpecOut = kOffSpecKern + align256(kNoAllocMaxHS * 8);        // product after planes
constexpr size_t kOffKc = kOffSpecOut + align256(kNoAllocMaxHS * 8);              // octant kernel spectrum
constexpr size_t kOffTw = kOffKc + align256(kNoAllocMaxKH * 4);                   // 4 twiddle tables
constexpr size_t kOffParams = kOffTw + align256(4 * kNoAllocMaxDim * 8);          // kernel parameters
constexpr size_t kOffSum = kOffParams + align256(sizeof(LeniaKernelParams));     // normalisation sum
constexpr size_t kNoAllocBytes = kOffSum + 256;
static_assert(kNoAllocBytes == 4439040, "the documented size of the scratch array (about 4.4 MB)");

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch per device, filled on first use.
// Atomic: host threads may make their first calls on a device at the same
// time (each stores the same address).
constexpr int kMaxDevices = 64;
std::atomic<unsigned char *> g_scratch_ptr[kMaxDevices] = {};

struct TwiddleArgs {
    float2 xf[kNoAllocMaxDim], xi[kNoAllocMaxDim], yf[kNoAllocMaxDim], yi[kNoAllocMaxDim];
};

// Writes the twiddle tables and the kernel parameters into the scratch array
// (both come by value, so no host-to-device copy is needed).
__global__ void k_noalloc_setup(TwiddleArgs tw, LeniaKernelParams kp, float2 *tw_dst, LeniaKernelParams *kp_dst,
                                int W, int H)
{
    for (int i = threadIdx.x; i < W; i += blockDim.x) {
        tw_dst[i] = tw.xf[i];
        tw_dst[kNoAllocMaxDim + i] = tw.xi[i];
    }
    for (int i = threadIdx.x; i < H; i += blockDim.x) {
        tw_dst[2 * kNoAllocMaxDim + i] = tw.yf[i];
        tw_dst[3 * kNoAllocMaxDim + i] = tw.yi[i];
    }
    if (threadIdx.x == 0) *kp_dst = kp;
}

void host_twiddles(int n, int sign, float2 *out)
{
    const double pi = 3.14159265358979323846;
    for (int i = 0; i < n; i++) {
        const double ang = (2.0 * pi * (double)i) / (double)n;
        const double c = cos(ang), s = sin(ang);
        out[i].x = (float)c;
        out[i].y = (float)(sign < 0 ? -s : s);
    }
}

bool dim_ok(int n)
{
    int r[kMaxStages];
    return n >= 8 && n <= kNoAllocMaxDim && n % 4 == 0 && fft_factor(n, r) > 0;
}

}  // namespace

namespace lenia {
bool plane_fits(const Dims &d, const FftPlan &py, const FftPlan &pz);
int row_tile(const Dims &d, const FftPlan &px);
}  // namespace lenia

extern "C" lenia_status lenia_convolve_noalloc(int width, int height, const float *field, const LeniaKernelParams *kernel,
                                               float *u_out, void *stream)
{
    if (!field || !kernel || !u_out) return LENIA_ERR_INVALID_ARG;
    if (!dim_ok(width) || !dim_ok(height)) {
        fprintf(stderr,
                "lenia_convolve_noalloc: grid %d x %d x %d is outside the fixed scratch space: width and height must "
                "be multiples of 4 in [8, %d] with prime factors in {2,3,5,7,11}\n",
                width, height, width, kNoAllocMaxDim);
        return LENIA_ERR_INVALID_ARG;
    }
    if (kernel->radius < 1 || kernel->beta_size < 1 || kernel->beta_size > LENIA_MAX_BETA || !(kernel->r_a > 0.0f))
        return LENIA_ERR_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return LENIA_ERR_NO_DEVICE;
    unsigned char *scratch = g_scratch_ptr[dev].load(std::memory_order_acquire);
    if (!scratch) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            fprintf(stderr, "lenia_convolve_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return LENIA_ERR_CUDA;
        }
        scratch = (unsigned char *)p;
        g_scratch_ptr[dev].store(scratch, std::memory_order_release);
    }
    cudaStream_t st = (cudaStream_t)stream;

    Dims d;
    d.W = width;
    d.H = height;
    d.D = width;
    d.N = (long long)width * height * width;
    d.KX = width / 2 + 1;
    d.HS = (long long)d.KX * d.D * d.H;
    d.P = (long long)(width + 8) * (height + 8) * (width + 8);
    FftPlan px, py;
    px.n = width;
    px.nstages = fft_factor(width, px.radix);
    py.n = height;
    py.nstages = fft_factor(height, py.radix);
    if (row_tile(d, px) == 0 || !plane_fits(d, py, px)) return LENIA_ERR_UNSUPPORTED;

    float *grid = (float *)(scratch + kOffGrid);
    float2 *spec_field = (float2 *)(scratch + kOffSpecField);
    float2 *spec_kern = (float2 *)(scratch + kOffSpecKern);
    float2 *spec_out = (float2 *)(scratch + kOffSpecOut);
    float *kc = (float *)(scratch + kOffKc);
    float2 *tw = (float2 *)(scratch + kOffTw);
    LeniaKernelParams *kp_dev = (LeniaKernelParams *)(scratch + kOffParams);
    float *ksum = (float *)(scratch + kOffSum);
    float2 *tw_xf = tw, *tw_xi = tw + kNoAllocMaxDim, *tw_yf = tw + 2 * kNoAllocMaxDim, *tw_yi = tw + 3 * kNoAllocMaxDim;

    TwiddleArgs ta;
    memset(&ta, 0, sizeof(ta));
    host_twiddles(width, -1, ta.xf);
    host_twiddles(width, +1, ta.xi);
    host_twiddles(height, -1, ta.yf);
    host_twiddles(height, +1, ta.yi);
    k_noalloc_setup<<<1, 128, 0, st>>>(ta, *kernel, tw, kp_dev, width, height);
    cudaError_t e = cudaGetLastError();

    // the kernel's grid and octant spectrum, as lenia_create builds them
    if (e == cudaSuccess) e = launch_kernel_grids(d, kp_dev, 1, grid, ksum, st);
    FwdRowJobs fj;
    memset(&fj, 0, sizeof(fj));
    fj.npairs = 1;
    fj.in[0] = grid;
    fj.out[0] = spec_kern;
    if (e == cudaSuccess) e = launch_fwd_rows(d, px, tw_xf, fj, st);
    // the field's half spectrum, as the growth stage builds it for a lone channel
    fj.in[0] = field;
    fj.out[0] = spec_field;
    if (e == cudaSuccess) e = launch_fwd_rows(d, px, tw_xf, fj, st);
    PlaneJobs pj;
    memset(&pj, 0, sizeof(pj));
    pj.njobs = 2;
    pj.src[0] = pj.dst[0] = spec_kern;
    pj.src[1] = pj.dst[1] = spec_field;
    if (e == cudaSuccess) e = launch_planes(d, py, px, tw_yf, tw_xf, pj, -1, st);
    if (e == cudaSuccess) e = launch_compress(d, spec_kern, kc, st);
    memset(&pj, 0, sizeof(pj));
    pj.njobs = 1;
    pj.src[0] = spec_field;
    pj.dst[0] = spec_out;
    pj.kc[0] = kc;
    if (e == cudaSuccess) e = launch_planes(d, py, px, tw_yi, tw_xi, pj, +1, st);
    BlurJobs bj;
    memset(&bj, 0, sizeof(bj));
    bj.nfields = 1;
    bj.spec[0] = spec_out;
    bj.out[0] = u_out;
    if (e == cudaSuccess) e = launch_blur_rows(d, px, tw_xi, bj, st);
    if (e != cudaSuccess) {
        fprintf(stderr, "lenia_convolve_noalloc: %s\n", cudaGetErrorString(e));
        return LENIA_ERR_CUDA;
    }
    return LENIA_OK;
}
