/*
 * Oracle test infrastructure: serial step driver for the reference build.
 *
 * The reference's lenia.cpp, reintegration.cpp, transposition.cpp and mesh.cpp
 * are compiled unmodified (oracle/Makefile) and linked with this file, which
 *   - defines the globals that main.cpp / render.cpp normally define
 *     (main.cpp:9-98, render.cpp:85), with the same defaults;
 *   - replays the 12-event step of render.cpp:357-604 serially, thread slab 0
 *     then slab 1 for every event, with these fix-ups:
 *       * the step always starts at SIM_EVENT_FFT with T = FFT(GRID)
 *         (main.cpp:198/321 would start the first step at FFT_MT);
 *       * with BLUR_CENTRAL_DIFF off, the H -> U_S and SUM -> SUM_S copy is
 *         the intended full copy (reintegration.cpp:179-186 copies
 *         MAX_CHANNELS times too many bytes) and the FFT_MT memsets clear
 *         exactly U_S and SUM_S (render.cpp:399-403 overruns SUM_S);
 *       * after SIM_EVENT_TRM the spectra T[c] are recomputed from the
 *         complete `val` (lenia.cpp:1039-1044 races the two slabs);
 *   - optionally runs each event's two slabs on two threads at once
 *     (ref_step_slabs), as the reference's SIM_THREADS = 2 sim threads do
 *     between the barriers of render.cpp:357-604;
 *   - exposes a C API for ctypes (ref_*).
 * It copies no reference code; it calls the reference's functions.
 */
#include "render.h"
#include "lenia.h"
#include "reintegration.h"
#include "transposition.h"
#include "mesh.h"
#include "marching_cubes.h"

#include <stdint.h>

#include <thread>
#include <vector>

#include "../restate/oracle_api.h"

/* ---- globals normally defined by main.cpp / render.cpp ---------------- */
bool redraw_config = true;
HINSTANCE hinst;
IDirect3DDevice9 *Device = 0;
IDirect3DVertexBuffer9 *cell_verts[2];
IDirect3DVertexBuffer9 *kernel_verts;
IDirect3DIndexBuffer9 *cvi[2];
int kernel_vcnt = 0;
volatile bool halted = false;
int voffset[2];
int ioffset[2];
volatile int running = 0;
int Width = 1280;
int Height = 768;
float move_speed = 1.0f;
float dt = 0.0f;
ViewType VIEWS = VIEW_U;
bool BLUR_CENTRAL_DIFF = false;
float GTA = 0.1f;
float STA = 0.1f;
float V_BETA = 0.9f;
float V_DAMP = 0.9f;
float neighborhood = 50.0f;
float ISO_VALUE = 0.5f;
float N = 2;
float THETA_A = 1;
float timestep = 0.1f;
int channels = 3;
bool ADV_VEL = true;
bool OSC_LA = false;
float OSC_LA_AMT = -0.001f;
bool OSC_FLOW = false;
float OSC_FLOW_AMT = -0.001f;
bool OSC_DIV_FLOW = false;
float OSC_DIV_FLOW_AMT = -0.001f;
bool OSC_VEL = false;
float S_NORM = 0.0f;
bool MU_VEL = false;
Border SOBEL_BORDER = BORDER_NONE;
Border BORDER = BORDER_NONE;
AlphaMode ALPHA_MODE = ALPHA_GRID;
GrowthType GROWTH_TYPE = GROWTH_RT;
ModeType MODE_TYPE = MODE_SRT;
GradientType GRADIENT_MODE = GRADIENT_SOBEL;
Kernel blur_kernel;
Kernel kernels[MAX_KERNELS];
int kernel_count = 0;
OffsetTable off_table;
ChannelData ch[MAX_CHANNELS];
fftwf_plan reverse_fft;
fftwf_plan forward_fft;
volatile LONG sim_threads_running;
volatile LONG sim_thread_gen;
volatile LONG sim_worker_gen[SIM_THREADS];
volatile LONG mesh_threads_running;
volatile LONG mesh_thread_gen;
volatile LONG mesh_worker_gen[MESH_THREADS];
volatile LONG render_gen;
volatile LONG mesh_render_gen;
SIM_EVENTS current_sim_event;
MESH_EVENTS current_mesh_event;
TD sim_td[8];
TD mesh_td[8];
int cur_buf = 0;
EdgeInfo EI[12];

/* Arrays defined in lenia.cpp / reintegration.cpp that the driver reads. */
extern fftwf_complex val[MAX_CHANNELS][GRID_SIZE];
extern fftwf_complex T[MAX_CHANNELS][GRID_SIZE];
extern fftwf_complex TEMP[MAX_KERNELS][GRID_SIZE];
extern fftwf_complex U[MAX_KERNELS][GRID_SIZE];
extern float PREALPHA[GRID_SIZE * MAX_CHANNELS];
extern float BELL_LUT[BELL_LUT_SIZE];

/* The kernel-preview mesh is rendering only (render.cpp:216-352). */
void rebuild_kernel_mesh(Vertex *v) { (void)v; }

/* rand()/srand() of the reference's platform (the MSVC C runtime): the linear
 * congruential generator x = 214013 x + 2531011 (mod 2^32), returning bits
 * 16..30.  Defined here with protected visibility so that the reference's
 * calls in this library bind to it instead of the C library's generator. */
static unsigned g_rand_state = 1;
extern "C" __attribute__((visibility("protected"))) void srand(unsigned seed) noexcept { g_rand_state = seed; }
extern "C" __attribute__((visibility("protected"))) int rand(void) noexcept
{
    g_rand_state = g_rand_state * 214013u + 2531011u;
    return (int)((g_rand_state >> 16) & 0x7fff);
}

/* Corner positions of a cube in the order mesh.cpp:19-32 samples them. */
static const int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1},
                                  {0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {0, 1, 1}};

/* EI (render.cpp:87-150) derived from geometry: the edge joining corners a and
 * b starts at their component-wise minimum and runs along the axis where they
 * differ. */
static void derive_edge_info(void)
{
    for (int e = 0; e < 12; e++) {
        int a = EDGE_TO_VERTICES[e][0], b = EDGE_TO_VERTICES[e][1];
        int o[3], axis = 0;
        for (int d = 0; d < 3; d++) {
            o[d] = kCorner[a][d] < kCorner[b][d] ? kCorner[a][d] : kCorner[b][d];
            if (kCorner[a][d] != kCorner[b][d]) axis = d;
        }
        EI[e].offset = ivec3(o[0], o[1], o[2]);
        EI[e].corner_a = a;
        EI[e].corner_b = b;
        EI[e].axis = (AXIS)axis;
    }
}

static bool g_initialised = false;

static void zero_all_state(void)
{
    memset(val, 0, sizeof(val));
    memset(GRID, 0, sizeof(GRID));
    memset(BACK, 0, sizeof(BACK));
    memset(T, 0, sizeof(T));
    memset(TEMP, 0, sizeof(TEMP));
    memset(U, 0, sizeof(U));
    memset(GA, 0, sizeof(GA));
    memset(ALPHA, 0, sizeof(ALPHA));
    memset(PREALPHA, 0, sizeof(PREALPHA));
    memset(SUM, 0, sizeof(SUM));
    memset(SUM_S, 0, sizeof(SUM_S));
    memset(U_S, 0, sizeof(U_S));
    memset(U_SUM_RB, 0, sizeof(U_SUM_RB));
    memset(U_SUM, 0, sizeof(U_SUM));
    memset(RBB, 0, sizeof(RBB));
    memset(H_RB, 0, sizeof(H_RB));
    memset(H, 0, sizeof(H));
    memset(NA_x, 0, sizeof(NA_x));
    memset(NA_y, 0, sizeof(NA_y));
    memset(NA_z, 0, sizeof(NA_z));
    memset(NU_x, 0, sizeof(NU_x));
    memset(NU_y, 0, sizeof(NU_y));
    memset(NU_z, 0, sizeof(NU_z));
    memset(F_x, 0, sizeof(F_x));
    memset(F_y, 0, sizeof(F_y));
    memset(F_z, 0, sizeof(F_z));
    memset(V_x, 0, sizeof(V_x));
    memset(V_y, 0, sizeof(V_y));
    memset(V_z, 0, sizeof(V_z));
    memset(MU_x, 0, sizeof(MU_x));
    memset(MU_y, 0, sizeof(MU_y));
    memset(MU_z, 0, sizeof(MU_z));
    memset(TT, 0, sizeof(TT));
}

extern "C" {

int ref_grid_width(void) { return GRID_WIDTH; }
int ref_grid_height(void) { return GRID_HEIGHT; }
int ref_max_kernels(void) { return MAX_KERNELS; }
int ref_max_channels(void) { return MAX_CHANNELS; }
int ref_padding(void) { return PADDING; }

/* One-time set-up in the order d3d::EnterMsgLoop / Setup use
 * (main.cpp:302-310, render.cpp:813, 903). */
void ref_init(void)
{
    if (g_initialised) return;
    init_pos_array();
    off_table.dd = 1.0f;
    off_table.sigma = 0.5f;
    off_table.X = off_table.Y = off_table.Z = NULL;
    init_gaussian_kernel();
    init_offset_table(NULL);
    init_bell_lut();
    derive_edge_info();
    init_fftw_plans();
    blur_kernel.radius = 2;
    blur_kernel.beta_size = 1;
    precompute_blur_kernel(&blur_kernel);
    for (int i = 0; i < 8; i++) sim_td[i].id = i;
    g_initialised = true;
}

void ref_set_params(const ora_params *p)
{
    channels = p->channels;
    timestep = p->timestep;
    THETA_A = p->theta_a;
    N = p->n_alpha;
    S_NORM = p->s_norm;
    GTA = p->gta;
    STA = p->sta;
    V_DAMP = p->v_damp;
    V_BETA = p->v_beta;
    ISO_VALUE = p->iso_value;
    off_table.sigma = p->sigma;
    off_table.dd = p->dd;
    init_offset_table(NULL);
    ALPHA_MODE = (AlphaMode)p->alpha_mode;
    GROWTH_TYPE = (GrowthType)p->growth_type;
    MODE_TYPE = (ModeType)p->mode_type;
    SOBEL_BORDER = (Border)p->sobel_border;
    BORDER = (Border)p->border;
    GRADIENT_MODE = (GradientType)p->gradient_mode;
    ADV_VEL = p->adv_vel != 0;
    MU_VEL = p->mu_vel != 0;
    BLUR_CENTRAL_DIFF = p->blur_central_diff != 0;
    OSC_LA = p->osc_la != 0;
    OSC_FLOW = p->osc_flow != 0;
    OSC_DIV_FLOW = p->osc_div_flow != 0;
    OSC_VEL = p->osc_vel != 0;
    OSC_LA_AMT = p->osc_la_amt;
    OSC_FLOW_AMT = p->osc_flow_amt;
    OSC_DIV_FLOW_AMT = p->osc_div_flow_amt;
    for (int c = 0; c < MAX_CHANNELS; c++) {
        ch[c].asymptotic = p->asymptotic[c] != 0;
        ch[c].soft_clip = p->soft_clip[c] != 0;
    }
}

/* Fills kernels[] and runs init_kernel (lenia.cpp:199-261) on each. */
int ref_set_kernels(const ora_kernel *k, int n)
{
    if (n < 0 || n > MAX_KERNELS) return -1;
    kernel_count = n;
    for (int i = 0; i < n; i++) {
        Kernel *d = &kernels[i];
        d->radius = k[i].radius;
        d->beta_size = k[i].beta_size;
        for (int b = 0; b < MAX_BETA; b++) d->b[b] = k[i].b[b];
        d->r_a = k[i].r_a;
        d->m = k[i].m;
        d->s = k[i].s;
        d->h = k[i].h;
        d->c0 = k[i].c0;
        d->c1 = k[i].c1;
        init_kernel(d);
    }
    return 0;
}

/* Kernel k's spatial grid (real part of Kernel::grid) and spectrum kg. */
void ref_get_kernel_grid(int k, float *out)
{
    for (int i = 0; i < GRID_SIZE; i++) out[i] = kernels[k].grid[i][0];
}
void ref_get_kernel_spectrum(int k, float *out_complex)
{
    memcpy(out_complex, kernels[k].kg, sizeof(fftwf_complex) * GRID_SIZE);
}
void ref_get_blur_spectrum(float *out_complex)
{
    memcpy(out_complex, blur_kernel.kg, sizeof(fftwf_complex) * GRID_SIZE);
}
void ref_get_blur_grid(float *out)
{
    for (int i = 0; i < GRID_SIZE; i++) out[i] = blur_kernel.grid[i][0];
}
float ref_bell_lut(int m, int s, int u) { return BELL_LUT[m * 65536 + s * 256 + u]; }

static void recompute_spectra(void)
{
    for (int c = 0; c < channels; c++) fftwf_execute_dft(forward_fft, val[c], T[c]);
}

/* New world: every array zero, then A, V (3 blocks), GA and SUM (interior)
 * from the caller, val = A and T = FFT(val).  Any pointer may be NULL. */
void ref_set_state(const float *A, const float *V, const float *GAin, const float *SUMin)
{
    zero_all_state();
    const int n = GRID_SIZE;
    for (int c = 0; c < channels; c++)
        for (int z = 0; z < GRID_WIDTH; z++)
            for (int y = 0; y < GRID_HEIGHT; y++)
                for (int x = 0; x < GRID_WIDTH; x++) {
                    int i = IDX(x, y, z);
                    int p = CPIDX(PIDX(x, y, z), c);
                    float a = A ? A[c * n + i] : 0.0f;
                    GRID[p] = a;
                    val[c][i][0] = a;
                    val[c][i][1] = 0.0f;
                    if (V) {
                        V_x[p] = V[(0 * channels + c) * n + i];
                        V_y[p] = V[(1 * channels + c) * n + i];
                        V_z[p] = V[(2 * channels + c) * n + i];
                    }
                    if (GAin) GA[c * n + i] = GAin[c * n + i];
                }
    if (SUMin)
        for (int z = 0; z < GRID_WIDTH; z++)
            for (int y = 0; y < GRID_HEIGHT; y++)
                for (int x = 0; x < GRID_WIDTH; x++) SUM[PIDX(x, y, z)] = SUMin[IDX(x, y, z)];
    recompute_spectra();
}

/* Slab threads: 0 runs the slabs one after the other on the calling thread;
 * 1 runs slab 1 on a second thread while the caller runs slab 0 and joins it
 * before the next event (the reference's barrier per event). */
static int g_slab_threads = 0;

static void run_both(void (*fn)(TD *))
{
    if (g_slab_threads) {
        std::thread other(fn, &sim_td[1]);
        fn(&sim_td[0]);
        other.join();
        for (int t = 2; t < SIM_THREADS; t++) fn(&sim_td[t]);
        return;
    }
    for (int t = 0; t < SIM_THREADS; t++) fn(&sim_td[t]);
}

/* One event for both slabs, mirroring the switch of render.cpp:376-592. */
void ref_run_event(int ev)
{
    switch (ev) {
    case ORA_EV_FFT:
        run_both(fft_step);
        break;
    case ORA_EV_FFT_MT:
        run_both(mt_fft_step);
        if (GRADIENT_MODE == GRADIENT_CENTRAL_DIFF && SOBEL_BORDER == BORDER_NONE) {
            memset(U_S, 0, sizeof(U_S));
            memset(SUM_S, 0, sizeof(SUM_S));
        }
        break;
    case ORA_EV_BLUR:
        if (GRADIENT_MODE == GRADIENT_CENTRAL_DIFF) {
            if (BLUR_CENTRAL_DIFF) {
                run_both(h_sum_blur);
            } else {
                memcpy(U_S, H, sizeof(U_S));
                memcpy(SUM_S, SUM, sizeof(SUM_S));
            }
        }
        break;
    case ORA_EV_TSB:
        if (GRADIENT_MODE == GRADIENT_SOBEL) {
            if (SOBEL_BORDER == BORDER_TORUS) run_both(transpose_sobel_borders);
            else if (SOBEL_BORDER == BORDER_WALL) run_both(wall_sobel_borders);
            else if (SOBEL_BORDER == BORDER_NONE) run_both(zero_sobel_borders);
        } else {
            if (SOBEL_BORDER == BORDER_TORUS) run_both(transpose_central_diff_borders);
            else if (SOBEL_BORDER == BORDER_WALL) run_both(wall_central_diff_borders);
        }
        break;
    case ORA_EV_SOBEL_ONE:
        run_both(sobel_convolve);
        break;
    case ORA_EV_SOBEL_TWO:
        run_both(sobel_convolve_h);
        break;
    case ORA_EV_F:
        run_both(compute_f);
        break;
    case ORA_EV_MU:
        if (MU_VEL) {
            if (BORDER == BORDER_WALL) run_both(compute_velocity_mu_wall);
            else run_both(compute_velocity_mu);
        } else {
            if (BORDER == BORDER_WALL) run_both(compute_f_mu_wall);
            else run_both(compute_f_mu);
        }
        break;
    case ORA_EV_TB:
        run_both(transpose_borders);
        break;
    case ORA_EV_REINTEGRATION:
        run_both(reintegration_step);
        break;
    case ORA_EV_TRM:
        run_both(transpose_to_row_major);
        recompute_spectra();
        break;
    case ORA_EV_TMB:
        run_both(transpose_mesh_borders);
        /* mesh snapshot of the grid interior (main.cpp:226-236), taken in the
         * same step as its halo faces */
        for (int c = 0; c < MAX_CHANNELS; c++)
            for (int z = 0; z < GRID_WIDTH; z++)
                for (int y = 0; y < GRID_HEIGHT; y++)
                    for (int x = 0; x < GRID_WIDTH; x++)
                        RBB[CPIDX(PIDX(x, y, z), c)] = GRID[CPIDX(PIDX(x, y, z), c)];
        break;
    default:
        break;
    }
}

void ref_step(int nsteps)
{
    for (int s = 0; s < nsteps; s++)
        for (int ev = 0; ev < ORA_EV_MAX; ev++) ref_run_event(ev);
}

/* ref_step with the two slabs of every event on two threads at once. */
void ref_step_slabs(int nsteps)
{
    g_slab_threads = 1;
    ref_step(nsteps);
    g_slab_threads = 0;
}

static void get_padded(const float *src, int nch, float *out)
{
    const int n = GRID_SIZE;
    for (int c = 0; c < nch; c++)
        for (int z = 0; z < GRID_WIDTH; z++)
            for (int y = 0; y < GRID_HEIGHT; y++)
                for (int x = 0; x < GRID_WIDTH; x++)
                    out[c * n + IDX(x, y, z)] = src[CPIDX(PIDX(x, y, z), c)];
}

/* Copies a field, unpadded and channel-major, into `out`; returns the
 * number of floats written or -1. */
int ref_get_field(int field, float *out)
{
    const int n = GRID_SIZE, C = channels;
    switch (field) {
    case ORA_A: get_padded(GRID, C, out); return C * n;
    case ORA_V:
        get_padded(V_x, C, out); get_padded(V_y, C, out + C * n); get_padded(V_z, C, out + 2 * C * n);
        return 3 * C * n;
    case ORA_GA: memcpy(out, GA, sizeof(float) * C * n); return C * n;
    case ORA_SUM: get_padded(SUM, 1, out); return n;
    case ORA_H: get_padded(H, C, out); return C * n;
    case ORA_U_SUM: get_padded(U_SUM, C, out); return C * n;
    case ORA_BACK: get_padded(BACK, C, out); return C * n;
    case ORA_NA:
        memcpy(out, NA_x, sizeof(float) * n); memcpy(out + n, NA_y, sizeof(float) * n);
        memcpy(out + 2 * n, NA_z, sizeof(float) * n);
        return 3 * n;
    case ORA_NU:
        memcpy(out, NU_x, sizeof(float) * C * n); memcpy(out + C * n, NU_y, sizeof(float) * C * n);
        memcpy(out + 2 * C * n, NU_z, sizeof(float) * C * n);
        return 3 * C * n;
    case ORA_PREALPHA: memcpy(out, PREALPHA, sizeof(float) * C * n); return C * n;
    case ORA_ALPHA: get_padded(ALPHA, C, out); return C * n;
    case ORA_F:
        get_padded(F_x, C, out); get_padded(F_y, C, out + C * n); get_padded(F_z, C, out + 2 * C * n);
        return 3 * C * n;
    case ORA_MU:
        get_padded(MU_x, C, out); get_padded(MU_y, C, out + C * n); get_padded(MU_z, C, out + 2 * C * n);
        return 3 * C * n;
    case ORA_TT: get_padded(TT, C, out); return C * n;
    case ORA_U_S: get_padded(U_S, C, out); return C * n;
    case ORA_SUM_S: get_padded(SUM_S, 1, out); return n;
    case ORA_U:
        for (int k = 0; k < kernel_count; k++)
            for (int i = 0; i < n; i++) out[k * n + i] = U[k][i][0] / GRID_SIZE;
        return kernel_count * n;
    case ORA_H_RB: get_padded(H_RB, C, out); return C * n;
    case ORA_U_SUM_RB: get_padded(U_SUM_RB, C, out); return C * n;
    case ORA_RBB: get_padded(RBB, C, out); return C * n;
    default: return -1;
    }
}

/* A padded field as the reference stores it: MAX_CHANNELS blocks of
 * GRID_PADDED floats (SUM, SUM_S: one block).  Returns floats written. */
int ref_get_padded(int field, float *out)
{
    const float *src = NULL;
    int blocks = MAX_CHANNELS;
    switch (field) {
    case ORA_A: src = GRID; break;
    case ORA_H: src = H; break;
    case ORA_U_S: src = U_S; break;
    case ORA_BACK: src = BACK; break;
    case ORA_ALPHA: src = ALPHA; break;
    case ORA_TT: src = TT; break;
    case ORA_SUM: src = SUM; blocks = 1; break;
    case ORA_SUM_S: src = SUM_S; blocks = 1; break;
    default: return -1;
    }
    memcpy(out, src, sizeof(float) * GRID_PADDED * blocks);
    return GRID_PADDED * blocks;
}

/* generate_random (lenia.cpp:370-429) after srand(seed), with the channel
 * count set by ref_set_params: writes the kernels it draws (up to max_k) and
 * the neighbourhood; the seeded grid (seed_grid_gaussian) is then in GRID
 * (ref_get_field A).  Returns kernel_count. */
int ref_generate_random(unsigned seed, ora_kernel *out, int max_k, float *neighborhood_out)
{
    static std::vector<char> kverts;
    static IDirect3DVertexBuffer9 kvb;
    kverts.resize((size_t)GRID_SIZE * 6 * MAX_KERNELS * sizeof(Vertex));
    kvb.mem = kverts.data();
    kvb.bytes = kverts.size();
    kernel_verts = &kvb;
    srand(seed);
    generate_random();
    for (int i = 0; i < kernel_count && i < max_k; i++) {
        const Kernel &k = kernels[i];
        out[i].radius = k.radius;
        out[i].beta_size = k.beta_size;
        for (int e = 0; e < 12; e++) out[i].b[e] = e < k.beta_size ? k.b[e] : 0.0f;
        out[i].r_a = k.r_a;
        out[i].m = k.m;
        out[i].s = k.s;
        out[i].h = k.h;
        out[i].c0 = k.c0;
        out[i].c1 = k.c1;
    }
    *neighborhood_out = neighborhood;
    return kernel_count;
}

/* Spectrum T[c] (complex, N entries). */
void ref_get_spectrum(int c, float *out_complex)
{
    memcpy(out_complex, T[c], sizeof(fftwf_complex) * GRID_SIZE);
}

/* One mesh of view 0 (NORMAL), 1 (U) or 2 (H), as mesh_thread_loop picks
 * them (render.cpp:625-636): the buffer reset of reset_mesh_generation
 * (render.cpp:182-200), generate_mesh_v1/v2/v3 (mesh.cpp) for every mesh
 * thread on RBB, U_SUM_RB, H_RB (filled by the step and ORA_EV_TMB), and the
 * concatenation of render.cpp:161-179 (thread order; indices offset by the
 * vertices before them).  stitch_borders (main.cpp:101-163) is not run.
 * Writes positions and normals (3 floats per vertex) and indices; returns 0,
 * or -1 when the output capacity is too small. */
int ref_mesh(int view, float *pos, float *nrm, long max_v, unsigned *idx, long max_i, long *n_v, long *n_i)
{
    static Vertex *vbuf[MESH_THREADS];
    static DWORD *ibuf[MESH_THREADS];
    const long cap = 3 * 15L * GRID_WIDTH * GRID_HEIGHT * GRID_WIDTH * MAX_CHANNELS;
    cur_buf = 0;
    memset(V1_EDGES, -1, sizeof(V1_EDGES));
    memset(V2_EDGES, -1, sizeof(V2_EDGES));
    memset(V3_EDGES, -1, sizeof(V3_EDGES));
    for (int t = 0; t < MESH_THREADS; t++) {
        if (!vbuf[t]) {
            vbuf[t] = (Vertex *)malloc(sizeof(Vertex) * cap);
            ibuf[t] = (DWORD *)malloc(sizeof(DWORD) * cap);
            if (!vbuf[t] || !ibuf[t]) return -1;
        }
        TD *td = &mesh_td[t];
        td->id = t;
        td->v = vbuf[t];
        td->ib = ibuf[t];
        td->vidx[cur_buf] = 0;
        td->iidx[cur_buf] = 0;
        td->lower_stitches = 0;
        td->upper_stitches = 0;
        memset(td->lower_border, -1, sizeof(td->lower_border));
        memset(td->upper_border, -1, sizeof(td->upper_border));
        memset(td->lower_indices, 0, sizeof(td->lower_indices));
        memset(td->upper_indices, 0, sizeof(td->upper_indices));
        if (view == 1) generate_mesh_v2(td);
        else if (view == 2) generate_mesh_v3(td);
        else generate_mesh_v1(td);
    }
    long nv = 0, ni = 0;
    for (int t = 0; t < MESH_THREADS; t++) {
        const TD *td = &mesh_td[t];
        for (int i = 0; i < td->iidx[cur_buf]; i++) {
            if (ni < max_i) idx[ni] = (unsigned)(td->ib[i] + nv);
            ni++;
        }
        for (int i = 0; i < td->vidx[cur_buf]; i++) {
            if (nv < max_v) {
                const Vertex &v = td->v[i];
                pos[3 * nv] = v._x;
                pos[3 * nv + 1] = v._y;
                pos[3 * nv + 2] = v._z;
                nrm[3 * nv] = v._nx;
                nrm[3 * nv + 1] = v._ny;
                nrm[3 * nv + 2] = v._nz;
            }
            nv++;
        }
    }
    *n_v = nv;
    *n_i = ni;
    return (nv > max_v || ni > max_i) ? -1 : 0;
}

}  /* extern "C" */
