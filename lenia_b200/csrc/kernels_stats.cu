// Statistics of a grid for labelling runs (no counterpart in the reference):
// per channel, in double precision,
//   0 mass           sum a
//   1-6 moments      sum a cos(2 pi x / W), sum a sin(2 pi x / W), the same
//                    for y (H) and z (W): the torus-aware centroid and spread
//   7 max            max a
//   8 fill           number of cells with a > threshold
// Two passes with a fixed summation order (each thread walks its cells in a
// fixed order, blocks reduce in a fixed tree, the second pass adds the block
// partials in order), so the result is the same on every run.
#include "lenia_internal.h"

namespace lenia {

namespace {

constexpr int kStatThreads = 256;

// Block reduction of the nine statistics (slot 7, the max, by maximum).
__device__ __forceinline__ void stat_reduce(double *s, double (&v)[kStats])
{
    const int t = threadIdx.x;
#pragma unroll
    for (int j = 0; j < kStats; j++) s[j * kStatThreads + t] = v[j];
    __syncthreads();
    for (int o = kStatThreads / 2; o > 0; o >>= 1) {
        if (t < o) {
#pragma unroll
            for (int j = 0; j < kStats; j++) {
                const double a = s[j * kStatThreads + t], b = s[j * kStatThreads + t + o];
                s[j * kStatThreads + t] = j == 7 ? (b > a ? b : a) : a + b;
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kStatThreads) k_stats_partial(const float *__restrict__ A, int W, int H, long long N,
                                                                const double *__restrict__ trig, float fill,
                                                                double *__restrict__ partial, int nblk)
{
    __shared__ double s[kStats * kStatThreads];
    const int c = blockIdx.y;
    const long long per = (N + nblk - 1) / nblk;
    const long long beg = blockIdx.x * per, end = beg + per < N ? beg + per : N;
    const float *a = A + (long long)c * N;
    const double *cx = trig, *sx = trig + W, *cy = trig + 2 * W, *sy = trig + 2 * W + H;
    double v[kStats] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (long long i = beg + threadIdx.x; i < end; i += kStatThreads) {
        const int x = (int)(i % W), y = (int)((i / W) % H), z = (int)(i / ((long long)W * H));
        const double m = (double)__ldg(a + i);
        v[0] += m;
        v[1] += m * cx[x];
        v[2] += m * sx[x];
        v[3] += m * cy[y];
        v[4] += m * sy[y];
        v[5] += m * cx[z];
        v[6] += m * sx[z];
        v[7] = m > v[7] ? m : v[7];
        v[8] += (float)m > fill ? 1.0 : 0.0;
    }
    stat_reduce(s, v);
    if (threadIdx.x < kStats) partial[((long long)c * nblk + blockIdx.x) * kStats + threadIdx.x] = s[threadIdx.x * kStatThreads];
}

// One block per channel; thread j adds statistic j of the block partials in order.
__global__ void k_stats_final(const double *__restrict__ partial, int nblk, double *__restrict__ out)
{
    const int c = blockIdx.x, j = threadIdx.x;
    if (j >= kStats) return;
    double r = 0.0;
    for (int b = 0; b < nblk; b++) {
        const double v = partial[((long long)c * nblk + b) * kStats + j];
        r = j == 7 ? (v > r ? v : r) : r + v;
    }
    out[c * kStats + j] = r;
}

// Channel totals for mass conservation: the same fixed-order two-pass sum.
__global__ void __launch_bounds__(kStatThreads) k_mass_partial(const float *__restrict__ A, long long N,
                                                               double *__restrict__ partial, int nblk)
{
    __shared__ double s[kStatThreads];
    const int c = blockIdx.y, t = threadIdx.x;
    const long long per = (N + nblk - 1) / nblk;
    const long long beg = blockIdx.x * per, end = beg + per < N ? beg + per : N;
    const float *a = A + (long long)c * N;
    double v = 0.0;
    for (long long i = beg + t; i < end; i += kStatThreads) v += (double)__ldg(a + i);
    s[t] = v;
    __syncthreads();
    for (int o = kStatThreads / 2; o > 0; o >>= 1) {
        if (t < o) s[t] = s[t] + s[t + o];
        __syncthreads();
    }
    if (t == 0) partial[(long long)c * nblk + blockIdx.x] = s[0];
}

__global__ void k_mass_final(const double *__restrict__ partial, int nblk, int C, double *__restrict__ out)
{
    const int c = threadIdx.x;
    if (c >= C) return;
    double r = 0.0;
    for (int b = 0; b < nblk; b++) r = r + partial[(long long)c * nblk + b];
    out[c] = r;
}

// A_c *= float(target_c / total_c) (no change for an empty channel).
__global__ void k_mass_scale(float *__restrict__ A, long long N, int C, const double *__restrict__ target,
                             const double *__restrict__ total)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)C * N) return;
    const int c = (int)(i / N);
    const double m = total[c];
    if (!(m > 0.0)) return;
    A[i] = A[i] * (float)(target[c] / m);
}

}  // namespace

cudaError_t launch_mass_totals(const float *A, const Dims &d, int C, double *partial, int nblk, double *out,
                               cudaStream_t st)
{
    k_mass_partial<<<dim3(nblk, C), kStatThreads, 0, st>>>(A, d.N, partial, nblk);
    k_mass_final<<<1, 32, 0, st>>>(partial, nblk, C, out);
    return cudaGetLastError();
}

cudaError_t launch_mass_scale(float *A, const Dims &d, int C, const double *target, const double *total,
                              cudaStream_t st)
{
    const long long n = (long long)C * d.N;
    k_mass_scale<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(A, d.N, C, target, total);
    return cudaGetLastError();
}

cudaError_t launch_stats(const float *A, const Dims &d, int C, const double *trig, float fill, double *partial,
                         int nblk, double *out, cudaStream_t st)
{
    k_stats_partial<<<dim3(nblk, C), kStatThreads, 0, st>>>(A, d.W, d.H, d.N, trig, fill, partial, nblk);
    k_stats_final<<<C, 32, 0, st>>>(partial, nblk, out);
    return cudaGetLastError();
}

}  // namespace lenia
