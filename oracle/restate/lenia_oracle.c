/*
 * ORACLE — test infrastructure only.  A CPU restatement of the 3D Flow Lenia
 * step of lostnthought/Lenia, written from the reference's semantics with the
 * grid size, channel count and kernel count as runtime values.  Each function
 * cites the reference file:line it follows.  Tests (and bench.py's CPU
 * baseline) load it through ctypes; the product library never does.
 *
 * Parity pin: with fft_mode ORA_FFT_C2C this restatement reproduces, bit for
 * bit, the reference's own sources compiled here (oracle/_ref/libleniaref.so,
 * 32x32x32) on every stage and mode (tests/test_oracle_pin.py), the two builds
 * sharing the LFFT engine in place of FFTW.  With ORA_FFT_HALF it follows the
 * CUDA library's half-spectrum convolution (described below) so that
 * GPU and CPU trajectories can be compared bit for bit; every other stage is
 * the same code in both modes.
 *
 * Layout: unpadded, channel-major, x fastest (IDX of render.h:334).  The
 * reference's 4-cell padding is replaced by read rules that reproduce what its
 * halo cells hold (transposition.cpp): a face cell (one coordinate outside the
 * grid) holds the copy its border routine writes; an edge or corner cell (two
 * or more coordinates outside) is never written and reads 0.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "lfft.h"
#include "oracle_api.h"

#define ORA_FFT_C2C 0
#define ORA_FFT_HALF 1

enum { B_TORUS = 0, B_WALL = 1, B_NONE = 2 };
enum { G_NOGROWTH = 0, G_RT = 1, G_TRANSPOSITION = 2 };
enum { M_SRT = 0, M_RT = 1, M_ADV = 2 };
enum { GR_CENTRAL_DIFF = 0, GR_SOBEL = 1 };

typedef struct {
    ora_params p;
    int W, H, D; /* x, y, z extents; D == W as in the reference */
    long N;      /* cells */
    int C, K;
    int fft_mode;
    ora_kernel *kern;
    float *kgrid;       /* K*N spatial kernels (lenia.cpp:199-257) */
    float *lut;         /* K*256 growth table rows (lenia.cpp:93-101) */
    int *lut_base;      /* K flat offsets m*65536 + s*256 into the 256^3 table */
    float *blur_grid;   /* N (reintegration.cpp:13-73) */
    /* C2C spectra (reference structure) */
    lcf *T;             /* C*N */
    lcf *kg;            /* K*N */
    lcf *blur_kg;       /* N */
    /* half spectra (library structure) */
    long HS;            /* (W/2+1)*D*H */
    float *khat;        /* K * (W/2+1)*(D/2+1)*(H/2+1) */
    float *blur_hat;
    /* fields */
    float *A, *V, *GA, *SUM, *H_, *U_SUM, *BACK, *NA, *NU, *PREALPHA, *ALPHA, *F, *MU, *TT,
        *U_S, *SUM_S, *U, *H_RB, *U_SUM_RB, *RBB;
    /* PREALPHA is MAX_CHANNELS*N floats as in the reference (lenia.cpp:41),
     * because sobel_convolve_h writes it at c*P + i (Q20). */
    long P; /* padded cells (W+8)(H+8)(W+8), render.h:293 */
} ora_world;

static inline long IDXW(const ora_world *w, int x, int y, int z)
{
    return (long)x + (long)y * w->W + (long)z * w->W * w->H;
}

/* ---------------------------------------------------------------- helpers */

/* _mm_min_ps / _mm_max_ps semantics: second operand unless the comparison holds. */
static inline float smin(float a, float b) { return a < b ? a : b; }
static inline float smax(float a, float b) { return a > b ? a : b; }
static inline float clampf(float a, float lo, float hi) { return smin(smax(a, lo), hi); }

static inline int emod(int a, int b)
{
    int r = a % b;
    return r < 0 ? r + b : r;
}

/* bell() of render.h:674-677: float argument arithmetic, double exp. */
static inline float bell(float x, float m, float s)
{
    double q = (double)((x - m) / s);
    return (float)exp(-(q * q) / 2.0);
}

/* fastexp of reintegration.h:149-170: degree-7 Taylor polynomial, Horner. */
static inline float fastexp(float x)
{
    const float a0 = 1.0f, a1 = 1.0f, a2 = 1.0f / 2, a3 = 1.0f / 2 / 3, a4 = 1.0f / 2 / 3 / 4,
                a5 = 1.0f / 2 / 3 / 4 / 5, a6 = 1.0f / 2 / 3 / 4 / 5 / 6,
                a7 = 1.0f / 2 / 3 / 4 / 5 / 6 / 7;
    float r = a7 * x + a6;
    r = r * x + a5;
    r = r * x + a4;
    r = r * x + a3;
    r = r * x + a2;
    r = r * x + a1;
    r = r * x + a0;
    return r;
}

/* Growth-table entry at flat index f of BELL_LUT (lenia.cpp:93-101). */
static float lut_flat(long f)
{
    if (f < 0 || f >= 256L * 256 * 256) return 0.0f;
    int m = (int)(f >> 16), s = (int)((f >> 8) & 255), u = (int)(f & 255);
    return bell((float)u / 255, (float)m / 255, (float)s / 255);
}

float ora_bell_lut(int m, int s, int u) { return lut_flat((long)m * 65536 + s * 256 + u); }

/* bell_lookup (lenia.h:79-84): truncating index into the 256^3 table; with
 * exact_bell (no counterpart in the reference) the bell itself. */
static inline float growth_lookup(const ora_world *w, int k, float u)
{
    /* exact_bell: the function the table samples, at u itself */
    if (w->p.exact_bell) return bell(u, w->kern[k].m, w->kern[k].s);
    int ui = (int)(u * 255);
    if (ui >= 0 && ui < 256) return w->lut[k * 256 + ui];
    return lut_flat((long)w->lut_base[k] + ui);
}

/* ------------------------------------------------------------ halo reads */

/* Fields whose halo faces transpose_borders fills (MU, ALPHA, V, F, GRID,
 * BACK: transposition.cpp:671-876): (int)dd periodic layers on faces only. */
static inline float tb_read(const ora_world *w, const float *f, int x, int y, int z)
{
    int dd = (int)w->p.dd;
    int ox = (x < 0 || x >= w->W), oy = (y < 0 || y >= w->H), oz = (z < 0 || z >= w->D);
    int no = ox + oy + oz;
    if (no == 0) return f[IDXW(w, x, y, z)];
    if (no > 1) return 0.0f;
    if (x < -dd || x >= w->W + dd || y < -dd || y >= w->H + dd || z < -dd || z >= w->D + dd)
        return 0.0f;
    if (x < 0) x += w->W; else if (x >= w->W) x -= w->W;
    if (y < 0) y += w->H; else if (y >= w->H) y -= w->H;
    if (z < 0) z += w->D; else if (z >= w->D) z -= w->D;
    return f[IDXW(w, x, y, z)];
}

/* Fields whose one-cell halo faces the gradient border routines fill
 * (transposition.cpp:6-665): torus copies the opposite face, wall replicates
 * the nearest interior cell, none writes zero. */
static inline float gb_read(const ora_world *w, const float *f, int x, int y, int z, int border)
{
    int ox = (x < 0 || x >= w->W), oy = (y < 0 || y >= w->H), oz = (z < 0 || z >= w->D);
    int no = ox + oy + oz;
    if (no == 0) return f[IDXW(w, x, y, z)];
    if (no > 1 || border == B_NONE) return 0.0f;
    if (x < -1 || x > w->W || y < -1 || y > w->H || z < -1 || z > w->D) return 0.0f;
    if (border == B_TORUS) {
        if (x < 0) x += w->W; else if (x >= w->W) x -= w->W;
        if (y < 0) y += w->H; else if (y >= w->H) y -= w->H;
        if (z < 0) z += w->D; else if (z >= w->D) z -= w->D;
    } else {
        if (x < 0) x = 0; else if (x >= w->W) x = w->W - 1;
        if (y < 0) y = 0; else if (y >= w->H) y = w->H - 1;
        if (z < 0) z = 0; else if (z >= w->D) z = w->D - 1;
    }
    return f[IDXW(w, x, y, z)];
}

/* ------------------------------------------------------ kernel building */

/* init_kernel (lenia.cpp:199-257): ring shells, normalised by the sum of the
 * cell values accumulated in float in (r_x, r_y, r_z) loop order. */
static void build_kernel_grid(const ora_world *w, const ora_kernel *kp, float *grid)
{
    const int W = w->W, H = w->H;
    const int ow = W / 2, oh = H / 2;
    const int bs = kp->beta_size;
    const int r = kp->radius;
    float k_cells = 0.0f;
    memset(grid, 0, sizeof(float) * w->N);
    for (int rx = -ow; rx < ow; rx++)
        for (int ry = -oh; ry < oh; ry++)
            for (int rz = -ow; rz < ow; rz++) {
                float x = fabsf((float)rx), y = fabsf((float)ry), z = fabsf((float)rz);
                float dist = sqrtf(x * x + y * y + z * z);
                dist = dist / (float)r * (float)bs / kp->r_a;
                if (dist < (float)bs) {
                    int fi = (int)floorf(dist);
                    int index = fi < bs - 1 ? fi : bs - 1;
                    float fin = kp->b[index] * bell(fmodf(dist, 1.0f), 0.5f, 0.15f);
                    grid[emod(rx, W) + (long)emod(ry, H) * W + (long)emod(rz, W) * W * H] = fin;
                    k_cells += fin;
                }
            }
    for (long i = 0; i < w->N; i++) grid[i] /= k_cells;
}

/* precompute_blur_kernel (reintegration.cpp:13-73): 5^3 exp(-d^2/s^3), s=1.5. */
static void build_blur_grid(const ora_world *w, float *grid)
{
    const int W = w->W, H = w->H;
    const float s = 1.5f;
    float k_cells = 0.0f;
    memset(grid, 0, sizeof(float) * w->N);
    for (int rx = -2; rx <= 2; rx++)
        for (int ry = -2; ry <= 2; ry++)
            for (int rz = -2; rz <= 2; rz++) {
                float x = fabsf((float)rx), y = fabsf((float)ry), z = fabsf((float)rz);
                float dist = x * x + y * y + z * z;
                float g = expf(-dist / (s * s * s));
                grid[emod(rx, W) + (long)emod(ry, H) * W + (long)emod(rz, W) * W * H] = g;
                k_cells += g;
            }
    for (long i = 0; i < w->N; i++) grid[i] /= k_cells;
}

/* --------------------------------------------------- half-spectrum path */
/*
 * The CUDA library's convolution:
 *   forward  two real fields a, b packed as a + i b; x-FFT per row; split into
 *            the two half spectra kx in [0, W/2]; then per kx plane the
 *            y-FFT and z-FFT.  Layout [kx][z][y], y fastest.
 *   kernels  real part of the forward transform of the kernel grid, kept on
 *            the octant kx<=W/2, kz<=D/2, ky<=H/2 and read back through
 *            |k| symmetry.
 *   inverse  per kx plane: multiply by the real kernel value, inverse y-FFT,
 *            inverse z-FFT; then per (z, y) row two kernels packed as
 *            S0 + i S1 extended to the full x range by Hermitian symmetry,
 *            inverse x-FFT, u0 = re / N, u1 = im / N.
 */

typedef struct {
    lfft_plan px, py, pz;
    lcf *work;
} hs_plans;

static void hs_plans_init(const ora_world *w, hs_plans *pl)
{
    lfft_plan_init(&pl->px, w->W);
    lfft_plan_init(&pl->py, w->H);
    lfft_plan_init(&pl->pz, w->D);
}

static void hs_plans_free(hs_plans *pl)
{
    lfft_plan_free(&pl->px);
    lfft_plan_free(&pl->py);
    lfft_plan_free(&pl->pz);
}

static inline long hs_idx(const ora_world *w, int kx, int z, int y)
{
    return ((long)kx * w->D + z) * w->H + y;
}

/* Forward transform of real fields fa (and fb, or zero) into half spectra. */
static void hs_forward_pair(const ora_world *w, hs_plans *pl, const float *fa, const float *fb,
                            lcf *oa, lcf *ob)
{
    const int W = w->W, H = w->H, D = w->D, KX = W / 2 + 1;
#pragma omp parallel
    {
        lcf *row = (lcf *)malloc(sizeof(lcf) * W);
        lcf *work = (lcf *)malloc(sizeof(lcf) * 2 * (W > H ? (W > D ? W : D) : (H > D ? H : D)));
#pragma omp for schedule(static)
        for (long zy = 0; zy < (long)D * H; zy++) {
            int z = (int)(zy / H), y = (int)(zy % H);
            const long base = IDXW(w, 0, y, z);
            for (int x = 0; x < W; x++) {
                row[x].re = fa[base + x];
                row[x].im = fb ? fb[base + x] : 0.0f;
            }
            lfft_1d(&pl->px, row, 1, -1, work);
            for (int kx = 0; kx < KX; kx++) {
                lcf p = row[kx], q = row[(W - kx) % W];
                lcf xa = {(p.re + q.re) * 0.5f, (p.im - q.im) * 0.5f};
                oa[hs_idx(w, kx, z, y)] = xa;
                if (ob) {
                    lcf xb = {(p.im + q.im) * 0.5f, (q.re - p.re) * 0.5f};
                    ob[hs_idx(w, kx, z, y)] = xb;
                }
            }
        }
#pragma omp for schedule(static)
        for (long kz = 0; kz < (long)KX * D; kz++) {
            int kx = (int)(kz / D), z = (int)(kz % D);
            lfft_1d(&pl->py, oa + hs_idx(w, kx, z, 0), 1, -1, work);
            if (ob) lfft_1d(&pl->py, ob + hs_idx(w, kx, z, 0), 1, -1, work);
        }
#pragma omp for schedule(static)
        for (long ky = 0; ky < (long)KX * H; ky++) {
            int kx = (int)(ky / H), y = (int)(ky % H);
            lfft_1d(&pl->pz, oa + hs_idx(w, kx, 0, y), H, -1, work);
            if (ob) lfft_1d(&pl->pz, ob + hs_idx(w, kx, 0, y), H, -1, work);
        }
        free(row);
        free(work);
    }
}

static inline float khat_at(const ora_world *w, const float *kh, int kx, int z, int y)
{
    int kz = z <= w->D - z ? z : w->D - z;
    int ky = y <= w->H - y ? y : w->H - y;
    return kh[((long)kx * (w->D / 2 + 1) + kz) * (w->H / 2 + 1) + ky];
}

/* Real, octant-compressed kernel spectrum from a full half spectrum. */
static void hs_compress_kernel(const ora_world *w, const lcf *spec, float *kh)
{
    const int KX = w->W / 2 + 1, KZ = w->D / 2 + 1, KY = w->H / 2 + 1;
    for (int kx = 0; kx < KX; kx++)
        for (int kz = 0; kz < KZ; kz++)
            for (int ky = 0; ky < KY; ky++)
                kh[((long)kx * KZ + kz) * KY + ky] = spec[hs_idx(w, kx, kz, ky)].re;
}

/* Multiply a half spectrum by a real kernel and run the inverse plane passes. */
static void hs_inverse_planes(const ora_world *w, hs_plans *pl, const lcf *src, const float *kh,
                              lcf *dst)
{
    const int W = w->W, H = w->H, D = w->D, KX = W / 2 + 1;
#pragma omp parallel
    {
        lcf *work = (lcf *)malloc(sizeof(lcf) * 2 * (H > D ? H : D));
#pragma omp for schedule(static)
        for (long kz = 0; kz < (long)KX * D; kz++) {
            int kx = (int)(kz / D), z = (int)(kz % D);
            for (int y = 0; y < H; y++) {
                lcf t = src[hs_idx(w, kx, z, y)];
                float k = khat_at(w, kh, kx, z, y);
                lcf r = {t.re * k, t.im * k};
                dst[hs_idx(w, kx, z, y)] = r;
            }
            lfft_1d(&pl->py, dst + hs_idx(w, kx, z, 0), 1, +1, work);
        }
#pragma omp for schedule(static)
        for (long ky = 0; ky < (long)KX * H; ky++) {
            int kx = (int)(ky / H), y = (int)(ky % H);
            lfft_1d(&pl->pz, dst + hs_idx(w, kx, 0, y), H, +1, work);
        }
        free(work);
    }
}

/* Final inverse x pass for two planes-transformed spectra packed together. */
static void hs_inverse_rows_pair(const ora_world *w, hs_plans *pl, const lcf *s0, const lcf *s1,
                                 float *u0, float *u1)
{
    const int W = w->W, H = w->H, D = w->D, KX = W / 2 + 1;
    const float nf = (float)w->N;
#pragma omp parallel
    {
        lcf *row = (lcf *)malloc(sizeof(lcf) * W);
        lcf *work = (lcf *)malloc(sizeof(lcf) * 2 * W);
#pragma omp for schedule(static)
        for (long zy = 0; zy < (long)D * H; zy++) {
            int z = (int)(zy / H), y = (int)(zy % H);
            for (int kx = 0; kx < W; kx++) {
                lcf a, b, zz;
                if (kx < KX) {
                    a = s0[hs_idx(w, kx, z, y)];
                    if (s1) b = s1[hs_idx(w, kx, z, y)]; else { b.re = 0.0f; b.im = 0.0f; }
                    zz.re = a.re - b.im;
                    zz.im = a.im + b.re;
                } else {
                    int m = W - kx;
                    a = s0[hs_idx(w, m, z, y)];
                    if (s1) b = s1[hs_idx(w, m, z, y)]; else { b.re = 0.0f; b.im = 0.0f; }
                    zz.re = a.re + b.im;
                    zz.im = b.re - a.im;
                }
                row[kx] = zz;
            }
            lfft_1d(&pl->px, row, 1, +1, work);
            const long base = IDXW(w, 0, y, z);
            for (int x = 0; x < W; x++) {
                u0[base + x] = row[x].re / nf;
                if (u1) u1[base + x] = row[x].im / nf;
            }
        }
        free(row);
        free(work);
    }
}

/* ------------------------------------------------------------- world */

static float *zalloc(long n) { return (float *)calloc((size_t)n, sizeof(float)); }

static void compute_lut_rows(ora_world *w)
{
    for (int k = 0; k < w->K; k++) {
        int mi = (int)(w->kern[k].m * 255);
        int si = (int)(w->kern[k].s * 255);
        w->lut_base[k] = mi * 65536 + si * 256;
        for (int u = 0; u < 256; u++) w->lut[k * 256 + u] = lut_flat((long)w->lut_base[k] + u);
    }
}

static void compute_kernel_spectra(ora_world *w)
{
    for (int k = 0; k < w->K; k++) build_kernel_grid(w, &w->kern[k], w->kgrid + (long)k * w->N);
    build_blur_grid(w, w->blur_grid);
    if (w->fft_mode == ORA_FFT_C2C) {
        for (int k = 0; k < w->K; k++) {
            lcf *dst = w->kg + (long)k * w->N;
            for (long i = 0; i < w->N; i++) { dst[i].re = w->kgrid[(long)k * w->N + i]; dst[i].im = 0.0f; }
            lfft_3d_c2c(dst, w->W, w->H, w->D, -1);
        }
        for (long i = 0; i < w->N; i++) { w->blur_kg[i].re = w->blur_grid[i]; w->blur_kg[i].im = 0.0f; }
        lfft_3d_c2c(w->blur_kg, w->W, w->H, w->D, -1);
    } else {
        hs_plans pl;
        hs_plans_init(w, &pl);
        lcf *sa = (lcf *)malloc(sizeof(lcf) * w->HS), *sb = (lcf *)malloc(sizeof(lcf) * w->HS);
        const long KH = (long)(w->W / 2 + 1) * (w->D / 2 + 1) * (w->H / 2 + 1);
        for (int k = 0; k < w->K; k += 2) {
            const float *gb = k + 1 < w->K ? w->kgrid + (long)(k + 1) * w->N : NULL;
            hs_forward_pair(w, &pl, w->kgrid + (long)k * w->N, gb, sa, gb ? sb : NULL);
            hs_compress_kernel(w, sa, w->khat + (long)k * KH);
            if (gb) hs_compress_kernel(w, sb, w->khat + (long)(k + 1) * KH);
        }
        hs_forward_pair(w, &pl, w->blur_grid, NULL, sa, NULL);
        hs_compress_kernel(w, sa, w->blur_hat);
        free(sa);
        free(sb);
        hs_plans_free(&pl);
    }
}

static void compute_spectra_c2c(ora_world *w)
{
    if (w->fft_mode != ORA_FFT_C2C) return;
    for (int c = 0; c < w->C; c++) {
        lcf *t = w->T + (long)c * w->N;
        for (long i = 0; i < w->N; i++) { t[i].re = w->A[(long)c * w->N + i]; t[i].im = 0.0f; }
        lfft_3d_c2c(t, w->W, w->H, w->D, -1);
    }
}

void *ora_create(const ora_params *p, const ora_kernel *k, int nk, int fft_mode)
{
    ora_world *w = (ora_world *)calloc(1, sizeof(ora_world));
    w->p = *p;
    w->W = p->width;
    w->H = p->height;
    w->D = p->width;
    w->N = (long)w->W * w->H * w->D;
    w->C = p->channels;
    w->K = nk;
    w->fft_mode = fft_mode;
    w->kern = (ora_kernel *)malloc(sizeof(ora_kernel) * (nk > 0 ? nk : 1));
    memcpy(w->kern, k, sizeof(ora_kernel) * nk);
    const long N = w->N, C = w->C;
    w->kgrid = zalloc((long)nk * N + 1);
    w->lut = zalloc((long)nk * 256 + 1);
    w->lut_base = (int *)calloc((size_t)nk + 1, sizeof(int));
    w->blur_grid = zalloc(N);
    w->HS = (long)(w->W / 2 + 1) * w->D * w->H;
    if (fft_mode == ORA_FFT_C2C) {
        w->T = (lcf *)calloc((size_t)(C * N), sizeof(lcf));
        w->kg = (lcf *)calloc((size_t)((long)nk * N + 1), sizeof(lcf));
        w->blur_kg = (lcf *)calloc((size_t)N, sizeof(lcf));
    } else {
        const long KH = (long)(w->W / 2 + 1) * (w->D / 2 + 1) * (w->H / 2 + 1);
        w->khat = zalloc((long)nk * KH + 1);
        w->blur_hat = zalloc(KH);
    }
    w->A = zalloc(C * N);
    w->V = zalloc(3 * C * N);
    w->GA = zalloc(C * N);
    w->SUM = zalloc(N);
    w->H_ = zalloc(C * N);
    w->U_SUM = zalloc(C * N);
    w->BACK = zalloc(C * N);
    w->NA = zalloc(3 * N);
    w->NU = zalloc(3 * C * N);
    w->PREALPHA = zalloc(ORA_MAX_CHANNELS * N);
    w->P = (long)(w->W + 8) * (w->H + 8) * (w->W + 8);
    w->ALPHA = zalloc(C * N);
    w->F = zalloc(3 * C * N);
    w->MU = zalloc(3 * C * N);
    w->TT = zalloc(C * N);
    w->U_S = zalloc(C * N);
    w->SUM_S = zalloc(N);
    w->U = zalloc((long)nk * N + 1);
    w->H_RB = zalloc(C * N);
    w->U_SUM_RB = zalloc(C * N);
    w->RBB = zalloc(C * N);
    compute_lut_rows(w);
    compute_kernel_spectra(w);
    return w;
}

void ora_destroy(void *h)
{
    ora_world *w = (ora_world *)h;
    if (!w) return;
    float *fs[] = {w->kgrid, w->lut, w->blur_grid, w->khat, w->blur_hat, w->A, w->V, w->GA,
                   w->SUM, w->H_, w->U_SUM, w->BACK, w->NA, w->NU, w->PREALPHA, w->ALPHA, w->F,
                   w->MU, w->TT, w->U_S, w->SUM_S, w->U, w->H_RB, w->U_SUM_RB, w->RBB};
    for (size_t i = 0; i < sizeof(fs) / sizeof(fs[0]); i++) free(fs[i]);
    free(w->lut_base);
    free(w->T);
    free(w->kg);
    free(w->blur_kg);
    free(w->kern);
    free(w);
}

/* Parameters other than the grid shape, channel count and kernels. */
void ora_set_params(void *h, const ora_params *p)
{
    ora_world *w = (ora_world *)h;
    ora_params q = *p;
    q.width = w->p.width;
    q.height = w->p.height;
    q.channels = w->p.channels;
    w->p = q;
}

/* New world state (reference: every array zero, then the seeded fields). */
void ora_set_state(void *h, const float *A, const float *V, const float *GA, const float *SUM)
{
    ora_world *w = (ora_world *)h;
    const long N = w->N, C = w->C;
    float *fs[] = {w->A, w->GA, w->H_, w->U_SUM, w->BACK, w->ALPHA, w->TT, w->U_S,
                   w->H_RB, w->U_SUM_RB, w->RBB};
    for (size_t i = 0; i < sizeof(fs) / sizeof(fs[0]); i++) memset(fs[i], 0, sizeof(float) * C * N);
    memset(w->PREALPHA, 0, sizeof(float) * ORA_MAX_CHANNELS * N);
    memset(w->V, 0, sizeof(float) * 3 * C * N);
    memset(w->NU, 0, sizeof(float) * 3 * C * N);
    memset(w->F, 0, sizeof(float) * 3 * C * N);
    memset(w->MU, 0, sizeof(float) * 3 * C * N);
    memset(w->NA, 0, sizeof(float) * 3 * N);
    memset(w->SUM, 0, sizeof(float) * N);
    memset(w->SUM_S, 0, sizeof(float) * N);
    memset(w->U, 0, sizeof(float) * w->K * N);
    if (A) memcpy(w->A, A, sizeof(float) * C * N);
    if (V) memcpy(w->V, V, sizeof(float) * 3 * C * N);
    if (GA) memcpy(w->GA, GA, sizeof(float) * C * N);
    if (SUM) memcpy(w->SUM, SUM, sizeof(float) * N);
    compute_spectra_c2c(w);
}

/* -------------------------------------------------------------- stages */

/* SIM_EVENT_FFT: fft_step (lenia.cpp:435-491).  Saves H and U_SUM into the
 * mesh snapshots, zeroes the accumulators, and computes u_k for every kernel
 * (Re of the inverse transform / N, the value mt_fft_step indexes with). */
static void ev_fft(ora_world *w)
{
    const long N = w->N, C = w->C;
    memcpy(w->U_SUM_RB, w->U_SUM, sizeof(float) * C * N);
    memcpy(w->H_RB, w->H_, sizeof(float) * C * N);
    memset(w->U_SUM, 0, sizeof(float) * C * N);
    memset(w->H_, 0, sizeof(float) * C * N);
    memset(w->NA, 0, sizeof(float) * 3 * N);
    memset(w->NU, 0, sizeof(float) * 3 * C * N);
    const float nf = (float)N;
    if (w->fft_mode == ORA_FFT_C2C) {
        lcf *tmp = (lcf *)malloc(sizeof(lcf) * N);
        for (int k = 0; k < w->K; k++) {
            const lcf *t = w->T + (long)w->kern[k].c0 * N;
            const lcf *g = w->kg + (long)k * N;
            for (long i = 0; i < N; i++) {
                tmp[i].re = t[i].re * g[i].re - t[i].im * g[i].im;
                tmp[i].im = t[i].re * g[i].im + t[i].im * g[i].re;
            }
            lfft_3d_c2c(tmp, w->W, w->H, w->D, +1);
            for (long i = 0; i < N; i++) w->U[(long)k * N + i] = tmp[i].re / nf;
        }
        free(tmp);
    } else {
        hs_plans pl;
        hs_plans_init(w, &pl);
        const long HS = w->HS;
        const long KH = (long)(w->W / 2 + 1) * (w->D / 2 + 1) * (w->H / 2 + 1);
        lcf *spec = (lcf *)malloc(sizeof(lcf) * HS * (C > 0 ? C : 1));
        for (int c = 0; c < C; c += 2) {
            const float *fb = c + 1 < C ? w->A + (c + 1) * N : NULL;
            hs_forward_pair(w, &pl, w->A + c * N, fb, spec + c * HS, fb ? spec + (c + 1) * HS : NULL);
        }
        lcf *s0 = (lcf *)malloc(sizeof(lcf) * HS), *s1 = (lcf *)malloc(sizeof(lcf) * HS);
        for (int k = 0; k < w->K; k += 2) {
            hs_inverse_planes(w, &pl, spec + (long)w->kern[k].c0 * HS, w->khat + (long)k * KH, s0);
            int two = k + 1 < w->K;
            if (two)
                hs_inverse_planes(w, &pl, spec + (long)w->kern[k + 1].c0 * HS,
                                  w->khat + (long)(k + 1) * KH, s1);
            hs_inverse_rows_pair(w, &pl, s0, two ? s1 : NULL, w->U + (long)k * N,
                                 two ? w->U + (long)(k + 1) * N : NULL);
        }
        free(s0);
        free(s1);
        free(spec);
        hs_plans_free(&pl);
    }
}

/* SIM_EVENT_FFT_MT: mt_fft_step (lenia.cpp:496-594), the growth accumulation
 * in kernel order and the early growth into BACK. */
static void ev_fft_mt(ora_world *w)
{
    const long N = w->N;
    /* render.cpp:399-403 (with the intended sizes) */
    if (w->p.gradient_mode == GR_CENTRAL_DIFF && w->p.sobel_border == B_NONE) {
        memset(w->U_S, 0, sizeof(float) * w->C * N);
        memset(w->SUM_S, 0, sizeof(float) * N);
    }
    for (int k = 0; k < w->K; k++) {
        const int c = w->kern[k].c1;
        const float h = w->kern[k].h;
        const float *u = w->U + (long)k * N;
        float *Hc = w->H_ + (long)c * N, *Us = w->U_SUM + (long)c * N;
        const float *g = w->A + (long)c * N;
        const int asym = w->p.asymptotic[c];
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; i++) {
            Us[i] = Us[i] + u[i];
            float l = growth_lookup(w, k, u[i]);
            if (asym) Hc[i] = Hc[i] + (l - g[i]) * h;
            else Hc[i] = Hc[i] + l * h;
        }
    }
    if (w->p.growth_type != G_NOGROWTH && w->p.growth_type != G_TRANSPOSITION) {
        const float t = w->p.timestep;
        for (int c = 0; c < w->C; c++) {
            const float *g = w->A + (long)c * N, *hh = w->H_ + (long)c * N;
            float *b = w->BACK + (long)c * N;
            const int sc = w->p.soft_clip[c];
#pragma omp parallel for schedule(static)
            for (long i = 0; i < N; i++) {
                float v = g[i] + hh[i] * t;
                if (sc) {
                    v = -4.0f * (v - 0.5f);
                    v = fastexp(v);
                    v = 1.0f + v;
                    v = 1.0f / v;
                }
                b[i] = clampf(v, 0.0f, 1.0f);
            }
        }
    }
}

/* SIM_EVENT_BLUR: h_sum_blur (reintegration.cpp:89-178) when
 * BLUR_CENTRAL_DIFF is set, else the intended copy H -> U_S, SUM -> SUM_S.
 * Only central-difference mode reads U_S / SUM_S (render.cpp:411). */
static void ev_blur(ora_world *w)
{
    const long N = w->N, C = w->C;
    if (w->p.gradient_mode != GR_CENTRAL_DIFF) return;
    if (!w->p.blur_central_diff) {
        memcpy(w->U_S, w->H_, sizeof(float) * C * N);
        memcpy(w->SUM_S, w->SUM, sizeof(float) * N);
        return;
    }
    const float nf = (float)N;
    if (w->fft_mode == ORA_FFT_C2C) {
        lcf *a = (lcf *)malloc(sizeof(lcf) * N), *t = (lcf *)malloc(sizeof(lcf) * N);
        for (int f = 0; f <= C; f++) {
            const float *src = f < C ? w->H_ + f * N : w->SUM;
            float *dst = f < C ? w->U_S + f * N : w->SUM_S;
            for (long i = 0; i < N; i++) { a[i].re = src[i]; a[i].im = 0.0f; }
            lfft_3d_c2c(a, w->W, w->H, w->D, -1);
            for (long i = 0; i < N; i++) {
                t[i].re = a[i].re * w->blur_kg[i].re - a[i].im * w->blur_kg[i].im;
                t[i].im = a[i].re * w->blur_kg[i].im + a[i].im * w->blur_kg[i].re;
            }
            lfft_3d_c2c(t, w->W, w->H, w->D, +1);
            for (long i = 0; i < N; i++) dst[i] = t[i].re / nf;
        }
        free(a);
        free(t);
    } else {
        hs_plans pl;
        hs_plans_init(w, &pl);
        const long HS = w->HS;
        lcf *sa = (lcf *)malloc(sizeof(lcf) * HS), *sb = (lcf *)malloc(sizeof(lcf) * HS);
        lcf *pa = (lcf *)malloc(sizeof(lcf) * HS), *pb = (lcf *)malloc(sizeof(lcf) * HS);
        for (int f = 0; f <= C; f += 2) {
            const float *fa = f < C ? w->H_ + f * N : w->SUM;
            float *da = f < C ? w->U_S + f * N : w->SUM_S;
            const float *fb = NULL;
            float *db = NULL;
            if (f + 1 <= C) {
                fb = f + 1 < C ? w->H_ + (f + 1) * N : w->SUM;
                db = f + 1 < C ? w->U_S + (f + 1) * N : w->SUM_S;
            }
            hs_forward_pair(w, &pl, fa, fb, sa, fb ? sb : NULL);
            hs_inverse_planes(w, &pl, sa, w->blur_hat, pa);
            if (fb) hs_inverse_planes(w, &pl, sb, w->blur_hat, pb);
            hs_inverse_rows_pair(w, &pl, pa, fb ? pb : NULL, da, db);
        }
        free(sa); free(sb); free(pa); free(pb);
        hs_plans_free(&pl);
    }
}

/* Sobel coefficient tables of lenia.h:30-71 as products: smoothing weight
 * 1-2-1 on two axes times the difference -1/0/+1 on the third.  Indexed
 * [dx+1][dy+1][dz+1] the reference's tables differentiate along dz (sx),
 * dx (sy) and dy (sz). */
static inline float sob_w(int d) { return d == 0 ? 2.0f : 1.0f; }
static inline float sob_sx(int dx, int dy, int dz) { return sob_w(dx) * sob_w(dy) * (float)dz; }
static inline float sob_sy(int dx, int dy, int dz) { return (float)dx * sob_w(dy) * sob_w(dz); }
static inline float sob_sz(int dx, int dy, int dz) { return sob_w(dx) * (float)dy * sob_w(dz); }

/* Gradient of one field into out (3 blocks of N): sum_sobel / h_sobel
 * (reintegration.cpp:191-259) or sum_central_diff / h_central_diff
 * (reintegration.cpp:260-315). */
static void gradient_field(const ora_world *w, const float *f, float *ox, float *oy, float *oz)
{
    const int W = w->W, H = w->H, D = w->D;
    const int border = w->p.sobel_border;
    if (w->p.gradient_mode == GR_SOBEL) {
#pragma omp parallel for schedule(static)
        for (int z = 0; z < D; z++)
            for (int y = 0; y < H; y++)
                for (int x = 0; x < W; x++) {
                    float ax = 0.0f, ay = 0.0f, az = 0.0f;
                    for (int dz = -1; dz <= 1; dz++)
                        for (int dy = -1; dy <= 1; dy++)
                            for (int dx = -1; dx <= 1; dx++) {
                                float v = gb_read(w, f, x + dx, y + dy, z + dz, border);
                                ax = ax + v * sob_sx(dx, dy, dz);
                                ay = ay + v * sob_sy(dx, dy, dz);
                                az = az + v * sob_sz(dx, dy, dz);
                            }
                    long i = IDXW(w, x, y, z);
                    ox[i] = ax;
                    oy[i] = ay;
                    oz[i] = az;
                }
    } else {
#pragma omp parallel for schedule(static)
        for (int z = 0; z < D; z++)
            for (int y = 0; y < H; y++)
                for (int x = 0; x < W; x++) {
                    long i = IDXW(w, x, y, z);
                    ox[i] = (gb_read(w, f, x + 1, y, z, border) - gb_read(w, f, x - 1, y, z, border)) * 0.5f;
                    oy[i] = (gb_read(w, f, x, y + 1, z, border) - gb_read(w, f, x, y - 1, z, border)) * 0.5f;
                    oz[i] = (gb_read(w, f, x, y, z + 1, border) - gb_read(w, f, x, y, z - 1, border)) * 0.5f;
                }
    }
}

/* SIM_EVENT_SOBEL_ONE: sobel_convolve (lenia.cpp:597-612), NA = grad SUM. */
static void ev_sobel_one(ora_world *w)
{
    const long N = w->N;
    const float *src = w->p.gradient_mode == GR_SOBEL ? w->SUM : w->SUM_S;
    gradient_field(w, src, w->NA, w->NA + N, w->NA + 2 * N);
}

/* SIM_EVENT_SOBEL_TWO: sobel_convolve_h (lenia.cpp:616-676), NU = grad H,
 * ALPHA = |GRID - GA|, PREALPHA = clamp((GRID/theta_A)^2, 0, 1) (Q3: the
 * ALPHA_MODE switch and N have no effect).
 * Q20: lenia.cpp:652-670 offsets the unpadded GA and PREALPHA arrays by the
 * padded channel stride CPOFFSET(c) = c*P while compute_f reads PREALPHA at
 * c*N + i.  The in-bounds effect is reproduced: PREALPHA is written at
 * c*P + i (writes past MAX_CHANNELS*N are dropped; in the reference's
 * declaration-order layout they land in SUM, which is cleared before its next
 * read) and ALPHA reads GA at c*P + i (reads past MAX_CHANNELS*N read 0). */
static void ev_sobel_two(ora_world *w)
{
    const long N = w->N, C = w->C, P = w->P, LIM = (long)ORA_MAX_CHANNELS * N;
    for (int c = 0; c < C; c++) {
        const float *src = (w->p.gradient_mode == GR_SOBEL ? w->H_ : w->U_S) + c * N;
        gradient_field(w, src, w->NU + c * N, w->NU + (C + c) * N, w->NU + (2 * C + c) * N);
    }
    const float ta = w->p.theta_a;
    const int fix = w->p.alpha_index_fix;
    for (int c = 0; c < C; c++) {
        const long off = fix ? c * N : c * P;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < N; i++) {
            float g = w->A[c * N + i];
            const long f = off + i;
            float ga = f < C * N ? w->GA[f] : 0.0f;
            w->ALPHA[c * N + i] = fabsf(g - ga);
            float pg = g / ta;
            pg = pg * pg;
            if (f < LIM) w->PREALPHA[f] = clampf(pg, 0.0f, 1.0f);
        }
    }
}

/* SIM_EVENT_F: compute_f (lenia.cpp:679-719). */
static void ev_f(ora_world *w)
{
    const long N = w->N, C = w->C;
#pragma omp parallel for schedule(static)
    for (long ci = 0; ci < C * N; ci++) {
        long i = ci % N;
        float a = w->PREALPHA[ci];
        float a1 = 1.0f - a;
        for (int d = 0; d < 3; d++)
            w->F[d * C * N + ci] = w->NU[d * C * N + ci] * a1 - w->NA[d * N + i] * a;
    }
}

/* SIM_EVENT_MU: compute_{f,velocity}_mu[_wall] (reintegration.cpp:321-602)
 * with compute_vel (reintegration.h:173-205). */
static void ev_mu(ora_world *w)
{
    const long N = w->N, C = w->C;
    const float dt = w->p.timestep, damp = w->p.v_damp, sigma = w->p.sigma;
    const float ma = w->p.dd - w->p.sigma;
    const float gws = (float)w->W - sigma, ghs = (float)w->H - sigma;
    const int wall = w->p.border == B_WALL;
    const int muvel = w->p.mu_vel;
#pragma omp parallel for schedule(static)
    for (long ci = 0; ci < C * N; ci++) {
        long i = ci % N;
        int x = (int)(i % w->W), y = (int)((i / w->W) % w->H), z = (int)(i / ((long)w->W * w->H));
        float pos[3] = {(float)x + 0.5f, (float)y + 0.5f, (float)z + 0.5f};
        float f[3], v[3];
        for (int d = 0; d < 3; d++) {
            f[d] = w->F[d * C * N + ci];
            v[d] = w->V[d * C * N + ci];
        }
        if (muvel)
            for (int d = 0; d < 3; d++) v[d] = (v[d] + f[d]) * damp;
        for (int d = 0; d < 3; d++) {
            float m = (muvel ? v[d] : f[d]) * dt;
            m = smax(m, -ma);
            m = smin(m, ma);
            m = pos[d] + m;
            if (wall) {
                m = smax(m, sigma);
                m = smin(m, d == 1 ? ghs : gws);
            }
            w->MU[d * C * N + ci] = m;
        }
        if (!muvel)
            for (int d = 0; d < 3; d++) v[d] = (v[d] + f[d]) * damp;
        for (int d = 0; d < 3; d++) w->V[d * C * N + ci] = v[d];
    }
}

static inline float torus_wrap(float m, int ext)
{
    const float half = (float)(ext / 2);
    if (m > half) m = m - (float)ext;
    if (m < -half) m = m + (float)ext;
    return m;
}

/* SIM_EVENT_REINTEGRATION: reintegration_step (lenia.cpp:727-918) with
 * srt, rt_border_torus, rt_border_other, adv_vel, adv_f
 * (reintegration.cpp:607-1410) and the oscillators. */
static void ev_reintegration(ora_world *w)
{
    const long N = w->N, C = w->C;
    const int W = w->W, H = w->H, D = w->D;
    const float sigma = w->p.sigma;
    const float s2 = 1 / (4 * sigma * sigma);
    const float s23 = 1 / (2 * sigma * sigma * sigma);
    const float sn = s2 * (1 - w->p.s_norm) + (w->p.s_norm * s23);
    const float clip = smin(2.0f * sigma, 1.0f);
    const float si = 0.5f + sigma;
    const int use_grid = w->p.growth_type == G_NOGROWTH || w->p.growth_type == G_TRANSPOSITION;
    const float *ARR = use_grid ? w->A : w->BACK;
    const int mode = w->p.mode_type;
    const int torus = w->p.border == B_TORUS;
    const int dd = (int)w->p.dd;
    const int crt = w->p.rt_all_channels ? (int)C : (C < 3 ? (int)C : 3);

    if (mode == M_SRT || mode == M_RT) {
#pragma omp parallel for schedule(static)
        for (int z = 0; z < D; z++)
            for (int y = 0; y < H; y++)
                for (int x = 0; x < W; x++) {
                    const long di = IDXW(w, x, y, z);
                    const float px = (float)x + 0.5f, py = (float)y + 0.5f, pz = (float)z + 0.5f;
                    for (int c = 0; c < crt; c++) {
                        const float *mux = w->MU + c * N, *muy = w->MU + (C + c) * N,
                                    *muz = w->MU + (2 * C + c) * N, *arr = ARR + c * N;
                        float tt = w->TT[c * N + di];
                        if (mode == M_SRT) {
                            float mx = fabsf(px - mux[di]), my = fabsf(py - muy[di]), mz = fabsf(pz - muz[di]);
                            mx = clampf(si - mx, 0.0f, clip);
                            my = clampf(si - my, 0.0f, clip);
                            mz = clampf(si - mz, 0.0f, clip);
                            float wgt = arr[di] * mx;
                            wgt = wgt * my;
                            wgt = wgt * mz;
                            wgt = wgt * sn;
                            tt = tt + wgt;
                        } else {
                            for (int dz = -dd; dz <= dd; dz++)
                                for (int dy = -dd; dy <= dd; dy++)
                                    for (int dx = -dd; dx <= dd; dx++) {
                                        int sx = x + dx, sy = y + dy, sz = z + dz;
                                        float mx = px - tb_read(w, mux, sx, sy, sz);
                                        float my = py - tb_read(w, muy, sx, sy, sz);
                                        float mz = pz - tb_read(w, muz, sx, sy, sz);
                                        if (torus) {
                                            mx = torus_wrap(mx, W);
                                            my = torus_wrap(my, H);
                                            mz = torus_wrap(mz, D);
                                        }
                                        mx = fabsf(mx); my = fabsf(my); mz = fabsf(mz);
                                        mx = si - mx; my = si - my; mz = si - mz;
                                        mx = smax(mx, 0.0f); my = smax(my, 0.0f); mz = smax(mz, 0.0f);
                                        mx = smin(mx, clip); my = smin(my, clip); mz = smin(mz, clip);
                                        float wgt = tb_read(w, arr, sx, sy, sz) * mx;
                                        wgt = wgt * my;
                                        wgt = wgt * mz;
                                        wgt = wgt * sn;
                                        tt = tt + wgt;
                                    }
                        }
                        w->TT[c * N + di] = tt;
                    }
                }
    } else if (mode == M_ADV) {
        const float dt = w->p.timestep, ma = w->p.dd - w->p.sigma;
        const float *vel = w->p.adv_vel ? w->V : w->F;
#pragma omp parallel for schedule(static)
        for (int z = 0; z < D; z++)
            for (int y = 0; y < H; y++)
                for (int x = 0; x < W; x++) {
                    const long di = IDXW(w, x, y, z);
                    const float pos[3] = {(float)x + 0.5f, (float)y + 0.5f, (float)z + 0.5f};
                    const float ext[3] = {(float)W, (float)H, (float)W};
                    for (int c = 0; c < C; c++) {
                        float X[3], Fr[3];
                        int I0[3];
                        for (int d = 0; d < 3; d++) {
                            float v = vel[(d * C + c) * N + di] * dt;
                            v = smin(smax(v, -ma), ma);
                            float q = (pos[d] - 0.5f) - v;
                            q = q + ext[d];
                            q = q - floorf(q / ext[d]) * ext[d];
                            float q0 = floorf(q);
                            X[d] = q;
                            I0[d] = (int)q0;
                            Fr[d] = q - q0;
                        }
                        const float *arr = ARR + c * N;
                        const float fx = Fr[0], fy = Fr[1], fz = Fr[2];
                        const float nfx = 1.0f - fx, nfy = 1.0f - fy, nfz = 1.0f - fz;
                        const int x0 = I0[0], y0 = I0[1], z0 = I0[2];
                        float s = tb_read(w, arr, x0, y0, z0) * nfx * nfy * nfz;
                        s = s + tb_read(w, arr, x0 + 1, y0, z0) * fx * nfy * nfz;
                        s = s + tb_read(w, arr, x0, y0 + 1, z0) * nfx * fy * nfz;
                        s = s + tb_read(w, arr, x0 + 1, y0 + 1, z0) * fx * fy * nfz;
                        s = s + tb_read(w, arr, x0, y0, z0 + 1) * nfx * nfy * fz;
                        s = s + tb_read(w, arr, x0 + 1, y0, z0 + 1) * fx * nfy * fz;
                        s = s + tb_read(w, arr, x0, y0 + 1, z0 + 1) * nfx * fy * fz;
                        s = s + tb_read(w, arr, x0 + 1, y0 + 1, z0 + 1) * fx * fy * fz;
                        w->TT[c * N + di] = s;
                        (void)X;
                    }
                }
    }

    if (w->p.osc_la || w->p.osc_flow || w->p.osc_div_flow) {
        const float *fl = w->p.osc_vel ? w->V : w->F;
#pragma omp parallel for schedule(static)
        for (int z = 0; z < D; z++)
            for (int y = 0; y < H; y++)
                for (int x = 0; x < W; x++) {
                    const long di = IDXW(w, x, y, z);
                    for (int c = 0; c < C; c++) {
                        const float *g = w->A + c * N;
                        float fx1 = tb_read(w, g, x + 1, y, z), fx0 = tb_read(w, g, x - 1, y, z);
                        float fy1 = tb_read(w, g, x, y + 1, z), fy0 = tb_read(w, g, x, y - 1, z);
                        float fz1 = tb_read(w, g, x, y, z + 1), fz0 = tb_read(w, g, x, y, z - 1);
                        float dxv = fx1 - fx0, dyv = fy1 - fy0, dzv = fz1 - fz0;
                        float tt = w->TT[c * N + di];
                        if (w->p.osc_la) {
                            float la = fx1 + fx0 + fy1 + fy0 + fz1 + fz0 - 6 * g[di];
                            tt = tt + la * w->p.osc_la_amt;
                        }
                        if (w->p.osc_flow) {
                            float flow = fl[c * N + di] * dxv + fl[(C + c) * N + di] * dyv +
                                         fl[(2 * C + c) * N + di] * dzv;
                            tt = tt + flow * w->p.osc_flow_amt;
                        }
                        if (w->p.osc_div_flow) {
                            const float *fxs = fl + c * N, *fys = fl + (C + c) * N, *fzs = fl + (2 * C + c) * N;
                            const float *al = w->ALPHA + c * N;
                            float jx = tb_read(w, fxs, x + 1, y, z) * tb_read(w, al, x + 1, y, z) -
                                       tb_read(w, fxs, x - 1, y, z) * tb_read(w, al, x - 1, y, z);
                            float jy = tb_read(w, fys, x, y + 1, z) * tb_read(w, al, x, y + 1, z) -
                                       tb_read(w, fys, x, y - 1, z) * tb_read(w, al, x, y - 1, z);
                            float jz = tb_read(w, fzs, x, y, z + 1) * tb_read(w, al, x, y, z + 1) -
                                       tb_read(w, fzs, x, y, z - 1) * tb_read(w, al, x, y, z - 1);
                            float divj = jx + jy + jz;
                            tt = tt + divj * w->p.osc_div_flow_amt;
                        }
                        w->TT[c * N + di] = tt;
                    }
                }
    }
    memset(w->SUM, 0, sizeof(float) * N);
}

/* SIM_EVENT_TRM: transpose_to_row_major (lenia.cpp:924-1044): growth or
 * clamp, moving averages, new GRID, SUM = STA * sum_c TT (Q2), TT cleared,
 * spectra recomputed from the complete new grid (Q10 fixed). */
static void ev_trm(ora_world *w)
{
    const long N = w->N, C = w->C;
    const float t = w->p.timestep;
    if (w->p.growth_type == G_TRANSPOSITION) {
        for (int c = 0; c < C; c++) {
            float *tt = w->TT + c * N;
            const float *g = w->A + c * N, *hh = w->H_ + c * N;
            float *b = w->BACK + c * N;
            if (w->p.soft_clip[c]) {
                for (long i = 0; i < N; i++) {
                    float v = g[i] + hh[i] * t;
                    v = -4.0f * (v - 0.5f);
                    v = fastexp(v);
                    v = 1.0f + v;
                    v = 1.0f / v;
                    b[i] = clampf(v, 0.0f, 1.0f);
                }
            } else {
                for (long i = 0; i < N; i++) tt[i] = clampf(tt[i] + hh[i] * t, 0.0f, 1.0f);
            }
        }
    } else {
        for (long i = 0; i < C * N; i++) w->TT[i] = clampf(w->TT[i], 0.0f, 1.0f);
    }
    const float stam = 1.0f - w->p.sta, stas = w->p.sta;
    const float gtas = w->p.gta, gtam = 1.0f - w->p.gta;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < N; i++) {
        float ttsum = 0.0f;
        for (int c = 0; c < C; c++) {
            float tt = w->TT[c * N + i];
            ttsum = ttsum + tt;
            w->TT[c * N + i] = 0.0f;
            w->GA[c * N + i] = gtam * w->GA[c * N + i] + tt * gtas;
            w->A[c * N + i] = tt;
        }
        w->SUM[i] = stam * w->SUM[i] + ttsum * stas;
    }
    compute_spectra_c2c(w);
}

/* SIM_EVENT_TMB: transpose_mesh_borders (transposition.cpp:881-995) only
 * fills halo faces of the mesh snapshots; with the snapshot taken in the same
 * step (Q12) the interior RBB is the current grid (main.cpp:226-236). */
static void ev_tmb(ora_world *w)
{
    memcpy(w->RBB, w->A, sizeof(float) * w->C * w->N);
}

void ora_run_event(void *h, int ev)
{
    ora_world *w = (ora_world *)h;
    switch (ev) {
    case ORA_EV_FFT: ev_fft(w); break;
    case ORA_EV_FFT_MT: ev_fft_mt(w); break;
    case ORA_EV_BLUR: ev_blur(w); break;
    case ORA_EV_TSB: break; /* halo faces are read rules, see gb_read */
    case ORA_EV_SOBEL_ONE: ev_sobel_one(w); break;
    case ORA_EV_SOBEL_TWO: ev_sobel_two(w); break;
    case ORA_EV_F: ev_f(w); break;
    case ORA_EV_MU: ev_mu(w); break;
    case ORA_EV_TB: break; /* halo faces are read rules, see tb_read */
    case ORA_EV_REINTEGRATION: ev_reintegration(w); break;
    case ORA_EV_TRM: ev_trm(w); break;
    case ORA_EV_TMB: ev_tmb(w); break;
    default: break;
    }
}

void ora_step(void *h, int nsteps)
{
    for (int s = 0; s < nsteps; s++)
        for (int ev = 0; ev < ORA_EV_MAX; ev++) ora_run_event(h, ev);
}

static float *field_ptr(ora_world *w, int field, long *count)
{
    const long N = w->N, C = w->C;
    switch (field) {
    case ORA_A: *count = C * N; return w->A;
    case ORA_V: *count = 3 * C * N; return w->V;
    case ORA_GA: *count = C * N; return w->GA;
    case ORA_SUM: *count = N; return w->SUM;
    case ORA_H: *count = C * N; return w->H_;
    case ORA_U_SUM: *count = C * N; return w->U_SUM;
    case ORA_BACK: *count = C * N; return w->BACK;
    case ORA_NA: *count = 3 * N; return w->NA;
    case ORA_NU: *count = 3 * C * N; return w->NU;
    case ORA_PREALPHA: *count = C * N; return w->PREALPHA;
    case ORA_ALPHA: *count = C * N; return w->ALPHA;
    case ORA_F: *count = 3 * C * N; return w->F;
    case ORA_MU: *count = 3 * C * N; return w->MU;
    case ORA_TT: *count = C * N; return w->TT;
    case ORA_U_S: *count = C * N; return w->U_S;
    case ORA_SUM_S: *count = N; return w->SUM_S;
    case ORA_U: *count = (long)w->K * N; return w->U;
    case ORA_H_RB: *count = C * N; return w->H_RB;
    case ORA_U_SUM_RB: *count = C * N; return w->U_SUM_RB;
    case ORA_RBB: *count = C * N; return w->RBB;
    default: *count = 0; return NULL;
    }
}

long ora_get_field(void *h, int field, float *out)
{
    long n;
    float *p = field_ptr((ora_world *)h, field, &n);
    if (!p) return -1;
    memcpy(out, p, sizeof(float) * n);
    return n;
}

/* Overwrites a field (stage-injection tests).  Setting A recomputes the C2C
 * spectra as TRM would. */
long ora_set_field(void *h, int field, const float *in)
{
    ora_world *w = (ora_world *)h;
    long n;
    float *p = field_ptr(w, field, &n);
    if (!p) return -1;
    memcpy(p, in, sizeof(float) * n);
    if (field == ORA_A) compute_spectra_c2c(w);
    return n;
}

void ora_get_kernel_grid(void *h, int k, float *out)
{
    ora_world *w = (ora_world *)h;
    memcpy(out, w->kgrid + (long)k * w->N, sizeof(float) * w->N);
}

void ora_get_blur_grid(void *h, float *out)
{
    ora_world *w = (ora_world *)h;
    memcpy(out, w->blur_grid, sizeof(float) * w->N);
}

/* Octant-compressed real kernel spectrum (half-spectrum mode only). */
long ora_get_kernel_hat(void *h, int k, float *out)
{
    ora_world *w = (ora_world *)h;
    if (!w->khat) return -1;
    const long KH = (long)(w->W / 2 + 1) * (w->D / 2 + 1) * (w->H / 2 + 1);
    memcpy(out, k < 0 ? w->blur_hat : w->khat + (long)k * KH, sizeof(float) * KH);
    return KH;
}

/* Full C2C kernel spectrum (C2C mode only), complex interleaved. */
long ora_get_kernel_spectrum(void *h, int k, float *out)
{
    ora_world *w = (ora_world *)h;
    if (!w->kg) return -1;
    memcpy(out, k < 0 ? w->blur_kg : w->kg + (long)k * w->N, sizeof(lcf) * w->N);
    return w->N;
}

void ora_get_lut_row(void *h, int k, float *out256)
{
    ora_world *w = (ora_world *)h;
    memcpy(out256, w->lut + k * 256, sizeof(float) * 256);
}

/* Half-spectrum forward transform of one or two real fields (unit tests of
 * the CUDA FFT).  Outputs are [kx][z][y] complex. */
void ora_hs_forward(void *h, const float *fa, const float *fb, float *oa, float *ob)
{
    ora_world *w = (ora_world *)h;
    hs_plans pl;
    hs_plans_init(w, &pl);
    hs_forward_pair(w, &pl, fa, fb, (lcf *)oa, (lcf *)ob);
    hs_plans_free(&pl);
}

/* One 1D LFFT of n complex values in place. */
void ora_lfft_1d(float *x, int n, int sign)
{
    lfft_plan p;
    if (lfft_plan_init(&p, n) != 0) return;
    lcf *work = (lcf *)malloc(sizeof(lcf) * 2 * n);
    lfft_1d(&p, (lcf *)x, 1, sign, work);
    free(work);
    lfft_plan_free(&p);
}

int ora_lfft_factor(int n, int *radix) { return lfft_factor(n, radix); }
