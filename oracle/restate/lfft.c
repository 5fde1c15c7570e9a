/*
 * Oracle test infrastructure: LFFT, the project's mixed-radix Stockham FFT,
 * written out on the CPU.  The file header of lfft.h states the contract.
 * Build with -ffp-contract=off so that no multiply-add is fused.
 */
#include "lfft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define LFFT_PI 3.14159265358979323846

static inline lcf c_add(lcf a, lcf b) { lcf r = {a.re + b.re, a.im + b.im}; return r; }
static inline lcf c_sub(lcf a, lcf b) { lcf r = {a.re - b.re, a.im - b.im}; return r; }
static inline lcf c_mul(lcf a, lcf w)
{
    lcf r = {a.re * w.re - a.im * w.im, a.re * w.im + a.im * w.re};
    return r;
}
/* sign * i * a, exact */
static inline lcf c_mul_si(lcf a, int sign)
{
    lcf r;
    if (sign > 0) { r.re = -a.im; r.im = a.re; }
    else          { r.re = a.im;  r.im = -a.re; }
    return r;
}

int lfft_factor(int n, int *radix)
{
    int k = 0;
    if (n < 1) return -1;
    while (n % 8 == 0 && k < LFFT_MAX_STAGES) { radix[k++] = 8; n /= 8; }
    if (n % 4 == 0) { radix[k++] = 4; n /= 4; }
    if (n % 2 == 0) { radix[k++] = 2; n /= 2; }
    static const int odd[4] = {3, 5, 7, 11};
    for (int i = 0; i < 4; i++)
        while (n % odd[i] == 0 && k < LFFT_MAX_STAGES) { radix[k++] = odd[i]; n /= odd[i]; }
    if (n != 1) return -1;
    return k;
}

int lfft_plan_init(lfft_plan *p, int n)
{
    memset(p, 0, sizeof(*p));
    p->n = n;
    p->nstages = lfft_factor(n, p->radix);
    if (p->nstages < 0) return -1;
    p->tw_fwd = (lcf *)malloc(sizeof(lcf) * (size_t)n);
    p->tw_inv = (lcf *)malloc(sizeof(lcf) * (size_t)n);
    for (int t = 0; t < n; t++) {
        double ang = (2.0 * LFFT_PI * (double)t) / (double)n;
        double c = cos(ang), s = sin(ang);
        p->tw_fwd[t].re = (float)c;
        p->tw_fwd[t].im = (float)(-s);
        p->tw_inv[t].re = (float)c;
        p->tw_inv[t].im = (float)s;
    }
    return 0;
}

void lfft_plan_free(lfft_plan *p)
{
    free(p->tw_fwd);
    free(p->tw_inv);
    p->tw_fwd = p->tw_inv = NULL;
}

static void dft2(lcf *v)
{
    lcf a = v[0], b = v[1];
    v[0] = c_add(a, b);
    v[1] = c_sub(a, b);
}

static void dft4(lcf *v, int sign)
{
    lcf t0 = c_add(v[0], v[2]);
    lcf t1 = c_sub(v[0], v[2]);
    lcf t2 = c_add(v[1], v[3]);
    lcf t3 = c_sub(v[1], v[3]);
    lcf u = c_mul_si(t3, sign);
    v[0] = c_add(t0, t2);
    v[1] = c_add(t1, u);
    v[2] = c_sub(t0, t2);
    v[3] = c_sub(t1, u);
}

static void dft8(lcf *v, int sign)
{
    lcf e[4] = {v[0], v[2], v[4], v[6]};
    lcf o[4] = {v[1], v[3], v[5], v[7]};
    dft4(e, sign);
    dft4(o, sign);
    const float h = 0x1.6a09e6p-1f; /* sqrt(1/2) rounded to float */
    lcf w1 = {h, sign * h};
    lcf w3 = {-h, sign * h};
    lcf o1 = c_mul(o[1], w1);
    lcf o2 = c_mul_si(o[2], sign);
    lcf o3 = c_mul(o[3], w3);
    v[0] = c_add(e[0], o[0]);
    v[4] = c_sub(e[0], o[0]);
    v[1] = c_add(e[1], o1);
    v[5] = c_sub(e[1], o1);
    v[2] = c_add(e[2], o2);
    v[6] = c_sub(e[2], o2);
    v[3] = c_add(e[3], o3);
    v[7] = c_sub(e[3], o3);
}

static void dft3(lcf *v, int sign)
{
    const float s3 = 0x1.bb67aep-1f; /* sqrt(3)/2 rounded to float */
    lcf d = c_sub(v[1], v[2]);
    lcf t1 = c_add(v[1], v[2]);
    lcf y0 = c_add(v[0], t1);
    lcf m = {v[0].re - t1.re * 0.5f, v[0].im - t1.im * 0.5f};
    lcf q = c_mul_si(d, sign);
    lcf e = {q.re * s3, q.im * s3};
    v[0] = y0;
    v[1] = c_add(m, e);
    v[2] = c_sub(m, e);
}

/* Direct DFT for the odd radices 5, 7, 11: y_k = v_0 + sum_j v_j W[(j k) % R],
 * the roots W[t] read from the length-n twiddle table at t * n / R. */
static void dft_generic(lcf *v, int r, const lcf *tw, int n)
{
    lcf w[11];
    lcf y[11];
    for (int t = 0; t < r; t++) w[t] = tw[t * (n / r)];
    for (int k = 0; k < r; k++) {
        lcf acc = v[0];
        for (int j = 1; j < r; j++) acc = c_add(acc, c_mul(v[j], w[(j * k) % r]));
        y[k] = acc;
    }
    for (int k = 0; k < r; k++) v[k] = y[k];
}

static void dft_small(lcf *v, int r, int sign, const lcf *tw, int n)
{
    switch (r) {
    case 2: dft2(v); break;
    case 3: dft3(v, sign); break;
    case 4: dft4(v, sign); break;
    case 8: dft8(v, sign); break;
    default: dft_generic(v, r, tw, n); break;
    }
}

void lfft_1d(const lfft_plan *p, lcf *x, long stride, int sign, lcf *work)
{
    const int n = p->n;
    const lcf *tw = sign < 0 ? p->tw_fwd : p->tw_inv;
    lcf *a = work, *b = work + n;
    for (int i = 0; i < n; i++) a[i] = x[(long)i * stride];
    int ns = 1;
    for (int s = 0; s < p->nstages; s++) {
        const int r = p->radix[s];
        const int m = n / r;
        const int tstep = n / (ns * r);
        for (int j = 0; j < m; j++) {
            lcf v[11];
            const int jm = j % ns;
            for (int q = 0; q < r; q++) v[q] = a[j + q * m];
            if (jm != 0)
                for (int q = 1; q < r; q++) v[q] = c_mul(v[q], tw[q * jm * tstep]);
            dft_small(v, r, sign, tw, n);
            const int base = (j / ns) * ns * r + jm;
            for (int q = 0; q < r; q++) b[base + q * ns] = v[q];
        }
        lcf *t = a; a = b; b = t;
        ns *= r;
    }
    for (int i = 0; i < n; i++) x[(long)i * stride] = a[i];
}

void lfft_3d_c2c(lcf *x, int w, int h, int d, int sign)
{
    lfft_plan pw, ph, pd;
    lfft_plan_init(&pw, w);
    lfft_plan_init(&ph, h);
    lfft_plan_init(&pd, d);
    int mx = w > h ? w : h;
    if (d > mx) mx = d;
    const long plane = (long)w * h;
    /* lines are independent: any thread order gives the same bits */
#pragma omp parallel
    {
        lcf *work = (lcf *)malloc(sizeof(lcf) * 2 * (size_t)mx);
#pragma omp for schedule(static)
        for (long zy = 0; zy < (long)d * h; zy++)
            lfft_1d(&pw, x + (zy / h) * plane + (zy % h) * w, 1, sign, work);
#pragma omp for schedule(static)
        for (long zx = 0; zx < (long)d * w; zx++)
            lfft_1d(&ph, x + (zx / w) * plane + (zx % w), w, sign, work);
#pragma omp for schedule(static)
        for (long yx = 0; yx < (long)h * w; yx++)
            lfft_1d(&pd, x + (yx / w) * w + (yx % w), plane, sign, work);
        free(work);
    }
    lfft_plan_free(&pw);
    lfft_plan_free(&ph);
    lfft_plan_free(&pd);
}
