// Compile-time-sized LFFT (the contract is in lfft_device.cuh): the same
// butterflies, twiddles and stage order, with the transform length, radix
// plan and batch shape known to the compiler, so every index is constant
// arithmetic.  Data live in a padded shared-memory matrix so that the
// Stockham reads and writes are free of bank conflicts.
#pragma once

#include "lfft_device.cuh"

namespace lenia {

// Radix plan of lfft_device.cuh, as constant expressions.
constexpr int plan_count(int n)
{
    int k = 0;
    while (n % 8 == 0) { k++; n /= 8; }
    if (n % 4 == 0) { k++; n /= 4; }
    if (n % 2 == 0) { k++; n /= 2; }
    const int odd[4] = {3, 5, 7, 11};
    for (int i = 0; i < 4; i++)
        while (n % odd[i] == 0) { k++; n /= odd[i]; }
    return n == 1 ? k : -1;
}

constexpr int plan_radix(int n, int s)
{
    int k = 0;
    while (n % 8 == 0) { if (k++ == s) return 8; n /= 8; }
    if (n % 4 == 0) { if (k++ == s) return 4; n /= 4; }
    if (n % 2 == 0) { if (k++ == s) return 2; n /= 2; }
    const int odd[4] = {3, 5, 7, 11};
    for (int i = 0; i < 4; i++)
        while (n % odd[i] == 0) { if (k++ == s) return odd[i]; n /= odd[i]; }
    return 0;
}

// Product of the radices before stage s (Ns of the Stockham stage).
constexpr int plan_ns(int n, int s)
{
    int p = 1;
    for (int i = 0; i < s; i++) p *= plan_radix(n, i);
    return p;
}

// A padded row-major matrix of float2: one spare slot every 16 columns and an
// odd row pitch, so rows and columns are both conflict-free to walk.
template <int NC>
struct PadMat {
    static constexpr int RP0 = NC + NC / 16;
    static constexpr int RP = (RP0 % 2 == 0) ? RP0 + 1 : RP0;
    static __device__ __forceinline__ int at(int r, int c) { return r * RP + c + (c >> 4); }
    static constexpr int size(int nrows) { return nrows * RP; }
};

// One Stockham stage.  COLS = false: NLINES rows of length N along the
// matrix columns (contiguous); COLS = true: NLINES matrix columns of length N
// along the rows.  THREADS threads with indices `tid` take part; WARP selects
// a warp-scope barrier (the lines belong to one warp) instead of the block's;
// P selects the paired butterflies of lfft_device.cuh (same bits).
template <int N, int S, int NLINES, bool COLS, int NC, int THREADS, bool WARP, bool P = false>
__device__ __forceinline__ void static_stage(float2 *buf, const float2 *tw, int sign, int tid)
{
    constexpr int R = plan_radix(N, S);
    constexpr int NS = plan_ns(N, S);
    constexpr int M = N / R;
    constexpr int TOTAL = NLINES * M;
    constexpr int NB = (TOTAL + THREADS - 1) / THREADS;
    constexpr int TSTEP = N / (NS * R);
    using PM = PadMat<NC>;
    float2 v[NB][R];
#pragma unroll
    for (int i = 0; i < NB; i++) {
        const int b = tid + i * THREADS;
        if (TOTAL % THREADS == 0 || b < TOTAL) {
            int l, j;
            if (COLS) { l = b % NLINES; j = b / NLINES; }
            else { j = b % M; l = b / M; }
#pragma unroll
            for (int r = 0; r < R; r++) v[i][r] = COLS ? buf[PM::at(j + r * M, l)] : buf[PM::at(l, j + r * M)];
        }
    }
    if (WARP) __syncwarp();
    else __syncthreads();
#pragma unroll
    for (int i = 0; i < NB; i++) {
        const int b = tid + i * THREADS;
        if (TOTAL % THREADS == 0 || b < TOTAL) {
            int l, j;
            if (COLS) { l = b % NLINES; j = b / NLINES; }
            else { j = b % M; l = b / M; }
            const int jm = j % NS;
            if (NS > 1 && jm != 0) {
#pragma unroll
                for (int r = 1; r < R; r++) v[i][r] = cmul(v[i][r], tw[r * jm * TSTEP]);
            }
            dft_small<R, P>(v[i], sign, tw, N);
            const int base = (j / NS) * NS * R + jm;
#pragma unroll
            for (int r = 0; r < R; r++) {
                if (COLS) buf[PM::at(base + r * NS, l)] = v[i][r];
                else buf[PM::at(l, base + r * NS)] = v[i][r];
            }
        }
    }
    if (WARP) __syncwarp();
    else __syncthreads();
}

// Stages S .. END-1 of the plan (END defaults to the whole plan).
template <int N, int S, int NLINES, bool COLS, int NC, int THREADS, bool WARP, int END = plan_count(N),
          bool P = false>
__device__ __forceinline__ void static_stages(float2 *buf, const float2 *tw, int sign, int tid)
{
    if constexpr (S < END) {
        static_stage<N, S, NLINES, COLS, NC, THREADS, WARP, P>(buf, tw, sign, tid);
        static_stages<N, S + 1, NLINES, COLS, NC, THREADS, WARP, END, P>(buf, tw, sign, tid);
    }
}

// Whole transform of NLINES lines held in a PadMat<NC>, by the whole block.
template <int N, int NLINES, bool COLS, int NC, int THREADS, bool P = false>
__device__ __forceinline__ void static_fft(float2 *buf, const float2 *tw, int sign)
{
    static_assert(plan_count(N) > 0, "unsupported transform length");
    static_stages<N, 0, NLINES, COLS, NC, THREADS, false, plan_count(N), P>(buf, tw, sign, threadIdx.x);
}

// Whole transform of NLINES rows owned by one warp (lane = threadIdx.x & 31).
template <int N, int NLINES, int NC>
__device__ __forceinline__ void warp_fft_rows(float2 *buf, const float2 *tw, int sign)
{
    static_assert(plan_count(N) > 0, "unsupported transform length");
    static_stages<N, 0, NLINES, false, NC, 32, true>(buf, tw, sign, threadIdx.x & 31);
}

// Largest divisor of n not above 16: rows per tile of the row kernels.
constexpr int row_tile_for(int n)
{
    for (int t = 16; t > 1; t--)
        if (n % t == 0) return t;
    return 1;
}

}  // namespace lenia
