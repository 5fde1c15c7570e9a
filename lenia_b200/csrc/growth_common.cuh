// Device helpers of the growth and early-growth arithmetic, shared by the
// spectral kernels (each translation unit gets its own inline copy).
#pragma once

#include <cuda_runtime.h>

namespace lenia {

// bell() of render.h:674-677: float argument arithmetic, double exponential.
__device__ __forceinline__ float bell_dev(float x, float m, float s)
{
    const float qf = (x - m) / s;
    const double q = (double)qf;
    return (float)exp(-(q * q) / 2.0);
}

// Entry f of the reference's 256^3 growth table (lenia.cpp:93-101).
__device__ __forceinline__ float lut_flat_dev(long long f)
{
    if (f < 0 || f >= 256LL * 256 * 256) return 0.0f;
    const int m = (int)(f >> 16), s = (int)((f >> 8) & 255), u = (int)(f & 255);
    return bell_dev((float)u / 255, (float)m / 255, (float)s / 255);
}

// fastexp of reintegration.h:149-170: degree-7 Taylor polynomial, Horner.
__device__ __forceinline__ float fastexp_dev(float x)
{
    const float a0 = 1.0f, a1 = 1.0f, a2 = 1.0f / 2, a3 = 1.0f / 2 / 3, a4 = 1.0f / 2 / 3 / 4,
                a5 = 1.0f / 2 / 3 / 4 / 5, a6 = 1.0f / 2 / 3 / 4 / 5 / 6, a7 = 1.0f / 2 / 3 / 4 / 5 / 6 / 7;
    float r = a7 * x + a6;
    r = r * x + a5;
    r = r * x + a4;
    r = r * x + a3;
    r = r * x + a2;
    r = r * x + a1;
    r = r * x + a0;
    return r;
}

// Early growth into BACK (lenia.cpp:542-592): clamp(g + h dt, 0, 1), or the
// soft clip 1 / (1 + fastexp(-4 (g + h dt - 0.5))) clamped.
__device__ __forceinline__ float early_growth(float g, float h, float dt, int soft)
{
    float v = g + h * dt;
    if (soft) {
        v = -4.0f * (v - 0.5f);
        v = fastexp_dev(v);
        v = 1.0f + v;
        v = 1.0f / v;
    }
    v = v > 0.0f ? v : 0.0f;
    v = v < 1.0f ? v : 1.0f;
    return v;
}

}  // namespace lenia
