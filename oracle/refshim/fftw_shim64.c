/*
 * Oracle test infrastructure: a second FFTW stand-in, used only to measure how
 * sensitive the reference's step is to the rounding of its FFT.
 *
 * It computes the same unnormalised DFT that FFTW documents
 *   X[k] = sum_j x[j] exp(sign * 2 pi i j k / n)
 * but in double precision throughout (input widened to double, the three
 * axis passes in double, one rounding to float at the end), so its result is
 * the correctly rounded transform up to double-precision error, where the
 * float stand-in (fftw_shim.c) rounds after every butterfly.  Linked with the
 * unmodified reference sources it gives a second, equally valid build of the
 * reference; the two builds' trajectories show how far two correct FFTs let
 * the reference's own step drift apart.
 *
 * Power-of-two lengths use an iterative radix-2 transform; other lengths a
 * direct O(n^2) sum (both in double).
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct lenia_fftwf_plan_s {
    int n0, n1, n2, sign;
};

typedef struct { double re, im; } zc;

fftwf_plan fftwf_plan_dft_3d(int n0, int n1, int n2, fftwf_complex *in, fftwf_complex *out,
                             int sign, unsigned flags)
{
    (void)in; (void)out; (void)flags;
    fftwf_plan p = (fftwf_plan)malloc(sizeof(*p));
    p->n0 = n0; p->n1 = n1; p->n2 = n2; p->sign = sign;
    return p;
}

static void dft_line(zc *x, int n, int sign, zc *tmp)
{
    const double pi = 3.14159265358979323846;
    if ((n & (n - 1)) == 0) {
        /* bit-reversal permutation, then log2(n) butterfly passes */
        for (int i = 1, j = 0; i < n; i++) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) { zc t = x[i]; x[i] = x[j]; x[j] = t; }
        }
        for (int len = 2; len <= n; len <<= 1) {
            for (int k = 0; k < len / 2; k++) {
                const double a = sign * 2.0 * pi * (double)k / (double)len;
                const double wr = cos(a), wi = sin(a);
                for (int s = 0; s < n; s += len) {
                    zc u = x[s + k], v = x[s + k + len / 2];
                    const double vr = v.re * wr - v.im * wi, vi = v.re * wi + v.im * wr;
                    x[s + k].re = u.re + vr; x[s + k].im = u.im + vi;
                    x[s + k + len / 2].re = u.re - vr; x[s + k + len / 2].im = u.im - vi;
                }
            }
        }
        return;
    }
    for (int k = 0; k < n; k++) {
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < n; j++) {
            const double a = sign * 2.0 * pi * (double)(((long)j * k) % n) / (double)n;
            const double c = cos(a), s = sin(a);
            sr += x[j].re * c - x[j].im * s;
            si += x[j].re * s + x[j].im * c;
        }
        tmp[k].re = sr; tmp[k].im = si;
    }
    memcpy(x, tmp, sizeof(zc) * (size_t)n);
}

void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out)
{
    const int d = p->n0, h = p->n1, w = p->n2;
    const size_t n = (size_t)d * h * w;
    int mx = w > h ? w : h;
    if (d > mx) mx = d;
    zc *z = (zc *)malloc(sizeof(zc) * n);
    zc *line = (zc *)malloc(sizeof(zc) * (size_t)mx);
    zc *tmp = (zc *)malloc(sizeof(zc) * (size_t)mx);
    for (size_t i = 0; i < n; i++) { z[i].re = in[i][0]; z[i].im = in[i][1]; }
    /* along w, h, then d (fastest to slowest) */
    for (long r = 0; r < (long)d * h; r++) dft_line(z + r * w, w, p->sign, tmp);
    for (int zz = 0; zz < d; zz++)
        for (int x = 0; x < w; x++) {
            zc *b = z + (size_t)zz * h * w + x;
            for (int y = 0; y < h; y++) line[y] = b[(size_t)y * w];
            dft_line(line, h, p->sign, tmp);
            for (int y = 0; y < h; y++) b[(size_t)y * w] = line[y];
        }
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            zc *b = z + (size_t)y * w + x;
            for (int zz = 0; zz < d; zz++) line[zz] = b[(size_t)zz * h * w];
            dft_line(line, d, p->sign, tmp);
            for (int zz = 0; zz < d; zz++) b[(size_t)zz * h * w] = line[zz];
        }
    for (size_t i = 0; i < n; i++) { out[i][0] = (float)z[i].re; out[i][1] = (float)z[i].im; }
    free(tmp);
    free(line);
    free(z);
}

void fftwf_destroy_plan(fftwf_plan p) { free(p); }
