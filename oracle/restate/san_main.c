/*
 * Oracle test infrastructure: a host harness for the address and
 * undefined-behaviour sanitizer build of the C restatement
 * (`make -C oracle sanitize` -> _build/san/oracle_san).
 *
 * It drives the restatement through every path the parity tests use, on
 * small grids: each border rule, both gradients, the blur pass, SRT, RT
 * (dd 1 and 2) and advection, both FFT structures, the oscillators, the
 * non-default channel options, several steps each, every field read back,
 * and marching cubes of the result with one and two slabs.  The sanitizers
 * report any out-of-bounds access, use after free, leak or undefined
 * operation; the process exits non-zero on the first report or when a
 * result is not finite where the step keeps it finite.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mc_tables.h"
#include "oracle_api.h"

void *ora_create(const ora_params *p, const ora_kernel *k, int nk, int fft_mode);
void ora_destroy(void *h);
void ora_set_state(void *h, const float *A, const float *V, const float *GA, const float *SUM);
void ora_step(void *h, int nsteps);
long ora_get_field(void *h, int field, float *out);

static uint32_t rng_state = 12345u;

static float urand(void)
{
    rng_state = rng_state * 1664525u + 1013904223u;
    return (float)(rng_state >> 8) / 16777216.0f;
}

static ora_params base_params(int w, int c)
{
    ora_params p;
    memset(&p, 0, sizeof(p));
    p.width = w;
    p.height = w;
    p.channels = c;
    p.timestep = 0.2f;
    p.theta_a = 2.0f;
    p.n_alpha = 2.0f;
    p.s_norm = 1.0f;
    p.gta = 0.5f;
    p.sta = 0.5f;
    p.v_damp = 0.9f;
    p.iso_value = 0.5f;
    p.sigma = 0.65f;
    p.dd = 1.0f;
    p.growth_type = 1;
    p.mode_type = 1;
    p.sobel_border = 0;
    p.border = 0;
    p.gradient_mode = 0;
    p.adv_vel = 1;
    return p;
}

static int run_case(const char *name, const ora_params *p, int fft_mode, int steps)
{
    const int C = p->channels, W = p->width, H = p->height;
    const long N = (long)W * H * W;
    ora_kernel ks[6];
    const int nk = C * 2 < 6 ? C * 2 : 6;
    for (int k = 0; k < nk; k++) {
        memset(&ks[k], 0, sizeof(ks[k]));
        ks[k].radius = W / 4;
        ks[k].beta_size = 1 + k % 3;
        for (int b = 0; b < ks[k].beta_size; b++) ks[k].b[b] = urand();
        ks[k].r_a = 1.0f;
        ks[k].m = 0.1f + 0.4f * urand();
        ks[k].s = 0.01f + 0.17f * urand();
        ks[k].h = 0.01f + 0.99f * urand();
        ks[k].c0 = k % C;
        ks[k].c1 = (k + 1) % C;
    }
    void *h = ora_create(p, ks, nk, fft_mode);
    if (!h) {
        fprintf(stderr, "%s: ora_create failed\n", name);
        return 1;
    }
    float *A = calloc((size_t)C * N, sizeof(float));
    for (int c = 0; c < C; c++)
        for (int z = W / 4; z < 3 * W / 4; z++)
            for (int y = H / 4; y < 3 * H / 4; y++)
                for (int x = W / 4; x < 3 * W / 4; x++) A[c * N + x + (long)y * W + (long)z * W * H] = urand();
    ora_set_state(h, A, NULL, NULL, NULL);
    ora_step(h, steps);
    int bad = 0;
    float *buf = malloc(sizeof(float) * 16 * (size_t)C * N);
    for (int f = 0; f < ORA_NFIELDS; f++) {
        const long n = ora_get_field(h, f, buf);
        if (f == ORA_A) {
            for (long i = 0; i < n; i++)
                if (!isfinite(buf[i])) bad = 1;
            memcpy(A, buf, sizeof(float) * (size_t)C * N);
        }
    }
    if (bad) fprintf(stderr, "%s: non-finite grid after %d steps\n", name, steps);
    for (int slabs = 1; slabs <= 2 && !bad; slabs++) {
        const long cap = 1L << 20;
        unsigned char *cases = calloc((size_t)C * N, 1), *unsure = calloc(cap, 1);
        float *pos = calloc(3 * cap, sizeof(float)), *nrm = calloc(3 * cap, sizeof(float));
        float *fnrm = calloc(cap, sizeof(float));
        int *vch = calloc(cap, sizeof(int));
        unsigned *idx = calloc(cap, sizeof(unsigned));
        const float *fields[1] = {A};
        long nv = 0, ni = 0;
        const int rc = ora_mesh_fields(fields, NULL, 1, NULL, W, H, C, p->iso_value, 3.5f, NULL, slabs, 1, 0, cases,
                                       pos, nrm, vch, unsure, cap, idx, fnrm, cap, &nv, &ni);
        if (rc != 0) {
            fprintf(stderr, "%s: mesh returned %d\n", name, rc);
            bad = 1;
        }
        free(cases);
        free(unsure);
        free(pos);
        free(nrm);
        free(fnrm);
        free(vch);
        free(idx);
    }
    free(buf);
    free(A);
    ora_destroy(h);
    printf("%-28s %s\n", name, bad ? "FAILED" : "ok");
    return bad;
}

int main(void)
{
    int fails = 0;
    for (int fft = 0; fft <= 1; fft++) {
        ora_params p = base_params(16, 2);
        char name[64];
        snprintf(name, sizeof(name), "rt torus cd fft%d", fft);
        fails += run_case(name, &p, fft, 3);
        p.gradient_mode = 1;
        p.sobel_border = 1;
        p.border = 1;
        snprintf(name, sizeof(name), "rt wall sobel fft%d", fft);
        fails += run_case(name, &p, fft, 3);
    }
    {
        ora_params p = base_params(16, 3);
        p.sobel_border = 2;
        p.border = 2;
        p.blur_central_diff = 1;
        fails += run_case("rt none cd blur", &p, 1, 3);
        p.blur_central_diff = 0;
        p.mode_type = 0;
        fails += run_case("srt none", &p, 1, 3);
        p.mode_type = 2;
        fails += run_case("adv vel", &p, 1, 3);
        p.adv_vel = 0;
        fails += run_case("adv f", &p, 1, 3);
        p.mode_type = 1;
        p.dd = 2.0f;
        p.sigma = 0.9f;
        fails += run_case("rt dd2", &p, 1, 2);
    }
    {
        ora_params p = base_params(16, 4);
        p.gradient_mode = 1;
        p.mu_vel = 1;
        p.osc_la = 1;
        p.osc_flow = 1;
        p.osc_div_flow = 1;
        p.osc_la_amt = 0.01f;
        p.osc_flow_amt = 0.01f;
        p.osc_div_flow_amt = 0.01f;
        p.growth_type = 2;
        p.soft_clip[1] = 1;
        p.asymptotic[2] = 1;
        fails += run_case("osc transposition 4ch", &p, 1, 2);
        p.rt_all_channels = 1;
        p.alpha_index_fix = 1;
        p.exact_bell = 1;
        fails += run_case("options on", &p, 1, 2);
    }
    {
        ora_params p = base_params(20, 2);
        p.height = 12;
        fails += run_case("20 x 12 x 20", &p, 0, 2);
    }
    printf("%d case(s) failed\n", fails);
    return fails != 0;
}
