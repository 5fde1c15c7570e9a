// Device side of LFFT, the project's mixed-radix Stockham FFT.
//
// Contract (shared with the CPU restatement used by the tests):
//   radix plan      greedy 8s, then one 4, then one 2, then 3s, 5s, 7s, 11s;
//   stage (Ns, R)   for j in [0, n/R): v[r] = x[j + r*n/R]; if (j % Ns) v[r] *=
//                   tw[r*(j%Ns)*(n/(Ns*R))] for r >= 1; v = DFT_R(v);
//                   y[(j/Ns)*Ns*R + j%Ns + r*Ns] = v[r];
//   twiddles        tw[t] = (cos 2 pi t/n, sign * sin 2 pi t/n) in double,
//                   stored as float (computed on the host at plan time);
//   arithmetic      complex product (a*c - b*d, a*d + b*c) with no fused
//                   multiply-add (this file is compiled with -fmad=false);
//   butterflies     as below: radix 8 = two radix-4 halves joined with
//                   sqrt(1/2) = 0x1.6a09e6p-1f, radix 3 with sqrt(3)/2 =
//                   0x1.bb67aep-1f, radices 5/7/11 as direct sums whose roots
//                   are tw[t*n/R].
// A transform of the same data therefore gives the same bits on the CPU and
// on the GPU, whichever kernel runs it.
#pragma once

#include <cuda_runtime.h>

namespace lenia {

constexpr int kMaxStages = 12;

struct FftPlan {
    int n;
    int nstages;
    int radix[kMaxStages];
};

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 w)
{
    return make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}

// Paired forms (P = true): the same per-lane operations issued as paired FP32
// instructions (two lanes per issue on sm_100), so the bits are those of the
// scalar forms.  The difference is a + (-1) * b with one rounding, which is
// a - b exactly (signed zeros included).  The product by a constant w takes
// the four products as two paired multiplies, (a.x w.x, a.y w.x) and
// (a.x w.y, a.y w.y), then (a.x w.x - a.y w.y, a.y w.x + a.x w.y): the
// roundings of cmul.  They hold more registers, so only kernels bound by
// instruction issue use them.
// A paired product that feeds a paired sum directly is contracted into one
// paired fma even under -fmad=false and the _rn forms (measured on sm_100a:
// __fadd2_rn(c, __fmul2_rn(a, b)) gave the fused result wherever one and two
// roundings differ).  So no paired sum here takes a paired product: the
// products of cmul_const meet scalar sums, and csub_t's fma multiplies by -1
// exactly.
template <bool P>
__device__ __forceinline__ float2 cadd_t(float2 a, float2 b)
{
    if constexpr (P) return __fadd2_rn(a, b);
    else return cadd(a, b);
}
template <bool P>
__device__ __forceinline__ float2 csub_t(float2 a, float2 b)
{
    if constexpr (P) return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
    else return csub(a, b);
}
template <bool P>
__device__ __forceinline__ float2 cmul_const(float2 a, float wx, float wy)
{
    if constexpr (P) {
        const float2 p = __fmul2_rn(a, make_float2(wx, wx));
        const float2 q = __fmul2_rn(a, make_float2(wy, wy));
        return make_float2(p.x - q.y, p.y + q.x);
    } else {
        return cmul(a, make_float2(wx, wy));
    }
}
// sign * i * a (exact)
__device__ __forceinline__ float2 cmul_si(float2 a, int sign)
{
    return sign > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <bool P = false>
__device__ __forceinline__ void dft2(float2 *v)
{
    float2 a = v[0], b = v[1];
    v[0] = cadd_t<P>(a, b);
    v[1] = csub_t<P>(a, b);
}

template <bool P = false>
__device__ __forceinline__ void dft4(float2 *v, int sign)
{
    float2 t0 = cadd_t<P>(v[0], v[2]);
    float2 t1 = csub_t<P>(v[0], v[2]);
    float2 t2 = cadd_t<P>(v[1], v[3]);
    float2 t3 = csub_t<P>(v[1], v[3]);
    float2 u = cmul_si(t3, sign);
    v[0] = cadd_t<P>(t0, t2);
    v[1] = cadd(t1, u);  // lanes cross: scalar
    v[2] = csub_t<P>(t0, t2);
    v[3] = csub(t1, u);
}

template <bool P = false>
__device__ __forceinline__ void dft8(float2 *v, int sign)
{
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    dft4<P>(e, sign);
    dft4<P>(o, sign);
    const float h = 0x1.6a09e6p-1f;
    const float sh = (float)sign * h;
    float2 o1 = cmul_const<P>(o[1], h, sh);
    float2 o2 = cmul_si(o[2], sign);
    float2 o3 = cmul_const<P>(o[3], -h, sh);
    v[0] = cadd_t<P>(e[0], o[0]);
    v[4] = csub_t<P>(e[0], o[0]);
    v[1] = cadd_t<P>(e[1], o1);
    v[5] = csub_t<P>(e[1], o1);
    v[2] = cadd(e[2], o2);  // lanes cross: scalar
    v[6] = csub(e[2], o2);
    v[3] = cadd_t<P>(e[3], o3);
    v[7] = csub_t<P>(e[3], o3);
}

__device__ __forceinline__ void dft3(float2 *v, int sign)
{
    const float s3 = 0x1.bb67aep-1f;
    float2 d = csub(v[1], v[2]);
    float2 t1 = cadd(v[1], v[2]);
    float2 y0 = cadd(v[0], t1);
    float2 m = make_float2(v[0].x - t1.x * 0.5f, v[0].y - t1.y * 0.5f);
    float2 q = cmul_si(d, sign);
    float2 e = make_float2(q.x * s3, q.y * s3);
    v[0] = y0;
    v[1] = cadd(m, e);
    v[2] = csub(m, e);
}

template <int R>
__device__ __forceinline__ void dft_generic(float2 *v, const float2 *tw, int n)
{
    float2 w[R];
    float2 y[R];
#pragma unroll
    for (int t = 0; t < R; t++) w[t] = tw[t * (n / R)];
#pragma unroll
    for (int k = 0; k < R; k++) {
        float2 acc = v[0];
#pragma unroll
        for (int j = 1; j < R; j++) acc = cadd(acc, cmul(v[j], w[(j * k) % R]));
        y[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < R; k++) v[k] = y[k];
}

template <int R, bool P = false>
__device__ __forceinline__ void dft_small(float2 *v, int sign, const float2 *tw, int n)
{
    if constexpr (R == 2) dft2<P>(v);
    else if constexpr (R == 3) dft3(v, sign);
    else if constexpr (R == 4) dft4<P>(v, sign);
    else if constexpr (R == 8) dft8<P>(v, sign);
    else dft_generic<R>(v, tw, n);
}

// One Stockham stage of radix R over `nlines` lines of length n held in shared
// memory, in place.  Element j of line l lives at buf[l*ls + j*es].  Every
// thread of the block loads its butterflies' inputs into registers, the block
// synchronises, then every thread computes and stores; CAP bounds the values
// a thread holds (nlines*n/blockDim <= CAP - R + 1 is required).
// `line_fast` maps consecutive threads to consecutive lines (use it when the
// lines, not the elements, are contiguous in shared memory).
template <int R, int CAP>
__device__ __forceinline__ void stage_inplace(float2 *buf, int n, int nlines, int es, int ls,
                                              int ns, const float2 *tw, int sign, bool line_fast)
{
    constexpr int NB = CAP / R;
    const int m = n / R;
    const int total = nlines * m;
    const int T = blockDim.x;
    float2 v[NB][R];
    int jj[NB], ll[NB];
#pragma unroll
    for (int i = 0; i < NB; i++) {
        const int b = threadIdx.x + i * T;
        jj[i] = -1;
        if (b < total) {
            int l, j;
            if (line_fast) { l = b % nlines; j = b / nlines; }
            else { j = b % m; l = b / m; }
            jj[i] = j;
            ll[i] = l;
#pragma unroll
            for (int r = 0; r < R; r++) v[i][r] = buf[l * ls + (j + r * m) * es];
        }
    }
    __syncthreads();
    const int tstep = n / (ns * R);
#pragma unroll
    for (int i = 0; i < NB; i++) {
        const int j = jj[i];
        if (j >= 0) {
            const int jm = j % ns;
            if (jm != 0) {
#pragma unroll
                for (int r = 1; r < R; r++) v[i][r] = cmul(v[i][r], tw[r * jm * tstep]);
            }
            dft_small<R>(v[i], sign, tw, n);
            const int base = (j / ns) * ns * R + jm;
            const int l = ll[i];
#pragma unroll
            for (int r = 0; r < R; r++) buf[l * ls + (base + r * ns) * es] = v[i][r];
        }
    }
    __syncthreads();
}

// Full in-place transform of `nlines` lines (all threads of the block).
template <int CAP>
__device__ void fft_lines(float2 *buf, const FftPlan &p, int nlines, int es, int ls,
                          const float2 *tw, int sign, bool line_fast)
{
    int ns = 1;
    for (int s = 0; s < p.nstages; s++) {
        const int r = p.radix[s];
        switch (r) {
        case 2: stage_inplace<2, CAP>(buf, p.n, nlines, es, ls, ns, tw, sign, line_fast); break;
        case 3: stage_inplace<3, CAP>(buf, p.n, nlines, es, ls, ns, tw, sign, line_fast); break;
        case 4: stage_inplace<4, CAP>(buf, p.n, nlines, es, ls, ns, tw, sign, line_fast); break;
        case 5: stage_inplace<5, CAP>(buf, p.n, nlines, es, ls, ns, tw, sign, line_fast); break;
        case 7: stage_inplace<7, CAP>(buf, p.n, nlines, es, ls, ns, tw, sign, line_fast); break;
        case 8: stage_inplace<8, CAP>(buf, p.n, nlines, es, ls, ns, tw, sign, line_fast); break;
        default: stage_inplace<11, CAP>(buf, p.n, nlines, es, ls, ns, tw, sign, line_fast); break;
        }
        ns *= r;
    }
}

}  // namespace lenia
