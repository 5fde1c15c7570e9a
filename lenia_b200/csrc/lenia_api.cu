// C ABI of the B200 3D Flow Lenia step (include/lenia_b200.h): world
// lifetime, validation, FFT plans, field I/O and the stream-ordered step.
//
// One step issues, in the reference's event order (render.cpp:376-583):
//   GROWTH     fwd_rows + planes (forward) + planes (inverse, x kernel) +
//              growth_rows                                   FFT, FFT_MT
//   BLUR       (central difference with blur) the same chain with the blur
//              kernel, storing U_S and SUM_S                  BLUR
//   FLOW       one fused stencil kernel                       TSB .. TB
//   TRANSPORT  one fused gather kernel                        REINTEGRATION, TRM
//   SNAPSHOT   (when enabled) grid copy for meshing           TMB
#include <math.h>
#include <stdio.h>
#include <stdarg.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <utility>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "direct_conv.h"
#include "lenia_internal.h"

using namespace lenia;

namespace lenia {
int row_tile(const Dims &d, const FftPlan &px);
bool plane_fits(const Dims &d, const FftPlan &py, const FftPlan &pz);
bool planes_supported(const Dims &d, const FftPlan &py, const FftPlan &pz);

int fft_factor(int n, int *radix)
{
    int k = 0;
    if (n < 1) return -1;
    while (n % 8 == 0 && k < kMaxStages) { radix[k++] = 8; n /= 8; }
    if (n % 4 == 0) { radix[k++] = 4; n /= 4; }
    if (n % 2 == 0) { radix[k++] = 2; n /= 2; }
    const int odd[4] = {3, 5, 7, 11};
    for (int i = 0; i < 4; i++)
        while (n % odd[i] == 0 && k < kMaxStages) { radix[k++] = odd[i]; n /= odd[i]; }
    return n == 1 ? k : -1;
}
}  // namespace lenia

namespace {

constexpr double kPi = 3.14159265358979323846;

// Twiddles tw[t] = (cos 2 pi t/n, sign sin 2 pi t/n): double, stored as float.
std::vector<float2> twiddles(int n, int sign)
{
    std::vector<float2> t(n);
    for (int i = 0; i < n; i++) {
        const double ang = (2.0 * kPi * (double)i) / (double)n;
        const double c = cos(ang), s = sin(ang);
        t[i].x = (float)c;
        t[i].y = (float)(sign < 0 ? -s : s);
    }
    return t;
}

template <typename T>
T *dalloc(size_t count, cudaError_t &err)
{
    T *p = nullptr;
    if (err != cudaSuccess || count == 0) return nullptr;
    err = cudaMalloc((void **)&p, count * sizeof(T));
    if (err == cudaSuccess) err = cudaMemset(p, 0, count * sizeof(T));
    return err == cudaSuccess ? p : nullptr;
}

}  // namespace

enum KernelId {
    KID_FWD_ROWS = 0,
    KID_PLANES_FWD,
    KID_PLANES_INV,
    KID_GROWTH_ROWS,
    KID_BLUR_FWD_ROWS,
    KID_BLUR_PLANES_FWD,
    KID_BLUR_PLANES_INV,
    KID_BLUR_ROWS,
    KID_FLOW,
    KID_TRANSPORT,
    KID_DIRECT_PAD,
    KID_DIRECT_CONV,
    KID_GROWTH_U,
    KID_MASS,
    KID_INV_ROWS,
    KID_MAX
};
const char *const kKernelNames[KID_MAX] = {"fwd_rows",          "planes_fwd",          "planes_inv",
                                           "growth_rows",       "blur_fwd_rows",       "blur_planes_fwd",
                                           "blur_planes_inv",   "blur_rows",           "flow",
                                           "transport",         "direct_pad",          "direct_conv",
                                           "growth_u",          "mass",                "inverse_rows"};

struct ProfRec {
    int kid;
    cudaEvent_t a, b;
};

struct lenia_world {
    LeniaWorldDesc desc;
    std::vector<LeniaKernelParams> kernels;
    Dims d;
    int C = 0, K = 0;
    FftPlan px, py;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;  // created by lenia_create
    int device = 0;
    bool debug = false, snapshots = false;
    bool shared_scratch = false;  // the per-step buffers belong to a batch lane (see lenia_batch)
    int launches = 0;
    std::string err;
    // device state
    float *A = nullptr, *A_next = nullptr, *V = nullptr, *GA = nullptr, *SUM = nullptr;
    float *H = nullptr, *H_RB = nullptr, *U_SUM = nullptr, *U_SUM_RB = nullptr, *BACK = nullptr;
    float *MU = nullptr, *F = nullptr, *ALPHA = nullptr, *U_S = nullptr, *SUM_S = nullptr, *RBB = nullptr;
    // The grid buffer (A or A_next) whose contents RBB stands for while the
    // snapshot copy is deferred (null: RBB holds the snapshot itself).  The
    // copy is made only when RBB is read out, or before that buffer is
    // written (the transport two steps later, lenia_set_field of A).
    const float *rbb_src = nullptr;
    float *NA = nullptr, *NU = nullptr, *PREALPHA = nullptr, *TT = nullptr, *U = nullptr;
    float2 *XS = nullptr;   // (C+1) half spectra
    float2 *S = nullptr;    // max(K, C+1) half spectra
    float *Kc = nullptr;    // K octant kernel spectra
    float *blur_hat = nullptr;
    float *lut_rows = nullptr;
    int *lut_base = nullptr;
    float *ksum = nullptr;  // K + 1 normalisation sums
    LeniaKernelParams *kp_dev = nullptr;
    float2 *tw_x_fwd = nullptr, *tw_x_inv = nullptr, *tw_y_fwd = nullptr, *tw_y_inv = nullptr;
    int *err_flag = nullptr;
    unsigned wait_polls = kDefaultTileWaitPolls;  // first wait for a tile copy (lenia_set_wait_limit)
    double *stats_trig = nullptr, *stats_partial = nullptr;  // lenia_world_stats buffers (allocated on first use)
    int lut_base_host[kMaxKernels];
    bool blur_valid = false;  // U_S / SUM_S hold a blur result
    int conv_mode = LENIA_CONV_FFT;
    int growth_split = 0;         // FFT growth as inverse rows storing u_k, then the growth from u_k
    DirectConv *dconv = nullptr;  // plan of the direct convolution modes
    // conserve_mass: the channel totals to restore, this step's totals, partials
    double *mass_target = nullptr, *mass_total = nullptr, *mass_partial = nullptr;
    // profiling
    bool profile = false;
    std::vector<ProfRec> prof_pending;
    std::vector<cudaEvent_t> prof_free;
    double prof_ms[KID_MAX] = {};
    long long prof_n[KID_MAX] = {};
};

namespace {

cudaEvent_t prof_event(lenia_world *w)
{
    if (!w->prof_free.empty()) {
        cudaEvent_t e = w->prof_free.back();
        w->prof_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Brackets the launches issued between prof_begin and prof_end.
// An NVTX range on the host timeline (header-only NVTX 3: a no-op unless a
// profiler such as Nsight Systems injects itself).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// One kernel launch of a step: an NVTX range named after the kernel and,
// with profiling on, CUDA events around it on the world's stream.
struct ProfScope {
    lenia_world *w;
    int kid;
    cudaEvent_t a = nullptr;
    NvtxRange range;
    ProfScope(lenia_world *w_, int kid_) : w(w_), kid(kid_), range(kKernelNames[kid_])
    {
        if (w->profile) {
            a = prof_event(w);
            cudaEventRecord(a, w->stream);
        }
    }
    ~ProfScope()
    {
        if (a) {
            cudaEvent_t b = prof_event(w);
            cudaEventRecord(b, w->stream);
            w->prof_pending.push_back({kid, a, b});
        }
    }
};

lenia_status fail(lenia_world *w, lenia_status s, const char *fmt, ...)
{
    if (w) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        w->err = buf;
    }
    return s;
}

lenia_status cuda_fail(lenia_world *w, cudaError_t e, const char *what)
{
    if (e == cudaErrorMemoryAllocation) return fail(w, LENIA_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
    return fail(w, LENIA_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

bool dim_ok(int n)
{
    int r[kMaxStages];
    return n >= 8 && n <= 256 && n % 4 == 0 && fft_factor(n, r) > 0;
}

lenia_status validate_desc(lenia_world *w, const LeniaWorldDesc *d)
{
    if (!d) return fail(w, LENIA_ERR_INVALID_ARG, "desc is NULL");
    if (!dim_ok(d->width) || !dim_ok(d->height))
        return fail(w, LENIA_ERR_INVALID_ARG,
                    "width/height must be in [8,256], multiples of 4, with prime factors in {2,3,5,7,11} "
                    "(got %d x %d)", d->width, d->height);
    if (d->channels < 1 || d->channels > LENIA_MAX_CHANNELS)
        return fail(w, LENIA_ERR_INVALID_ARG, "channels must be 1..%d", LENIA_MAX_CHANNELS);
    if (!(d->sigma > 0.0f) || !(d->dd >= 1.0f) || d->dd >= 5.0f)
        return fail(w, LENIA_ERR_INVALID_ARG, "need sigma > 0 and 1 <= dd < 5 (the reference pads 4 cells)");
    if (d->growth_type < 0 || d->growth_type > 2 || d->mode_type < 0 || d->mode_type > 2 || d->border < 0 ||
        d->border > 2 || d->sobel_border < 0 || d->sobel_border > 2 || d->gradient_mode < 0 || d->gradient_mode > 1)
        return fail(w, LENIA_ERR_INVALID_ARG, "mode enum out of range");
    return LENIA_OK;
}

lenia_status validate_kernels(lenia_world *w, const LeniaKernelParams *k, int n, int channels)
{
    if (n < 0 || n > LENIA_MAX_KERNELS) return fail(w, LENIA_ERR_INVALID_ARG, "n_kernels must be 0..%d", LENIA_MAX_KERNELS);
    if (n > 0 && !k) return fail(w, LENIA_ERR_INVALID_ARG, "kernels is NULL");
    for (int i = 0; i < n; i++) {
        if (k[i].radius < 1 || k[i].beta_size < 1 || k[i].beta_size > LENIA_MAX_BETA || !(k[i].r_a > 0.0f))
            return fail(w, LENIA_ERR_INVALID_ARG, "kernel %d: need radius >= 1, 1 <= beta_size <= %d, r_a > 0", i,
                        LENIA_MAX_BETA);
        if (k[i].c0 < 0 || k[i].c0 >= channels || k[i].c1 < 0 || k[i].c1 >= channels)
            return fail(w, LENIA_ERR_INVALID_ARG, "kernel %d: channel out of range", i);
    }
    return LENIA_OK;
}

StepParams step_params(const lenia_world *w)
{
    const LeniaWorldDesc &s = w->desc;
    StepParams p;
    memset(&p, 0, sizeof(p));
    p.d = w->d;
    p.C = w->C;
    p.timestep = s.timestep;
    p.theta_a = s.theta_a;
    {
        int ex = 0;
        const float m = frexpf(s.theta_a, &ex);  // theta_a = m * 2^ex, m in [0.5, 1)
        p.inv_theta_a = (m == 0.5f && ex - 1 >= -126 && ex - 1 <= 126) ? ldexpf(1.0f, 1 - ex) : 0.0f;
    }
    p.s_norm = s.s_norm;
    p.gta = s.gta;
    p.sta = s.sta;
    p.v_damp = s.v_damp;
    p.sigma = s.sigma;
    p.dd_f = s.dd;
    p.dd = (int)s.dd;
    p.growth_type = s.growth_type;
    p.mode_type = s.mode_type;
    p.sobel_border = s.sobel_border;
    p.border = s.border;
    p.gradient_mode = s.gradient_mode;
    p.adv_vel = s.adv_vel;
    p.mu_vel = s.mu_vel;
    p.blur = s.blur_central_diff;
    p.osc_la = s.osc_la;
    p.osc_flow = s.osc_flow;
    p.osc_div_flow = s.osc_div_flow;
    p.osc_vel = s.osc_vel;
    p.osc_la_amt = s.osc_la_amt;
    p.osc_flow_amt = s.osc_flow_amt;
    p.osc_div_flow_amt = s.osc_div_flow_amt;
    for (int c = 0; c < kMaxChannels; c++) {
        p.asymptotic[c] = s.asymptotic[c];
        p.soft_clip[c] = s.soft_clip[c];
    }
    p.rt_all_channels = s.rt_all_channels;
    p.alpha_index_fix = s.alpha_index_fix;
    // off_table.ma (lenia.cpp:143) and the reintegration constants
    // (lenia.cpp:730-736, reintegration.cpp:610, 328-329), in float.
    const float sigma = s.sigma;
    p.ma = s.dd - s.sigma;
    const float s2 = 1 / (4 * sigma * sigma);
    const float s23 = 1 / (2 * sigma * sigma * sigma);
    p.sn = s2 * (1 - s.s_norm) + (s.s_norm * s23);
    p.clip = 2.0f * sigma < 1.0f ? 2.0f * sigma : 1.0f;
    p.si = 0.5f + sigma;
    p.gws = (float)w->d.W - sigma;
    p.ghs = (float)w->d.H - sigma;
    p.wait_polls = w->wait_polls;
    return p;
}

bool needs_F(const LeniaWorldDesc &s)
{
    return (s.mode_type == LENIA_MODE_ADV && !s.adv_vel) || ((s.osc_flow || s.osc_div_flow) && !s.osc_vel);
}

lenia_status ensure_optional(lenia_world *w)
{
    cudaError_t e = cudaSuccess;
    const size_t CN = (size_t)w->C * w->d.N;
    if ((w->debug || needs_F(w->desc)) && !w->F) w->F = dalloc<float>(3 * CN, e);
    if ((w->debug || w->desc.osc_div_flow) && !w->ALPHA) w->ALPHA = dalloc<float>(CN, e);
    if (w->debug) {
        if (!w->NA) w->NA = dalloc<float>(3 * (size_t)w->d.N, e);
        if (!w->NU) w->NU = dalloc<float>(3 * CN, e);
        if (!w->PREALPHA) w->PREALPHA = dalloc<float>(CN, e);
        if (!w->TT) w->TT = dalloc<float>(CN, e);
        if (!w->U && w->K > 0) w->U = dalloc<float>((size_t)w->K * w->d.N, e);
    }
    if (w->snapshots && !w->RBB) w->RBB = dalloc<float>(CN, e);
    if (e != cudaSuccess) return cuda_fail(w, e, "allocating optional fields");
    return LENIA_OK;
}

// Kernel spectra, growth-table rows and the blur spectrum.
lenia_status build_kernels(lenia_world *w)
{
    cudaError_t e = cudaSuccess;
    const Dims &d = w->d;
    const int K = w->K;
    cudaStream_t st = w->stream;
    if (K > 0) {
        e = cudaMemcpyAsync(w->kp_dev, w->kernels.data(), sizeof(LeniaKernelParams) * K, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_fail(w, e, "copying kernels");
    }
    float *grids = nullptr;
    size_t ng = (size_t)std::max(K, 1) * d.N;
    e = cudaMallocAsync((void **)&grids, ng * sizeof(float), st);
    if (e != cudaSuccess) return cuda_fail(w, e, "kernel grid scratch");
    if ((e = launch_kernel_grids(d, w->kp_dev, K, grids, w->ksum, st)) != cudaSuccess) goto out;
    if (w->dconv) {
        direct_destroy(w->dconv);
        w->dconv = nullptr;
    }
    if (w->conv_mode != LENIA_CONV_FFT) {
        if (!w->U && K > 0) w->U = dalloc<float>((size_t)K * d.N, e);
        if (e != cudaSuccess) goto out;
        if ((e = direct_create(d, w->C, w->kernels.data(), K, w->conv_mode, &w->dconv)) != cudaSuccess) goto out;
        if ((e = direct_build(w->dconv, grids, st)) != cudaSuccess) goto out;
    }
    for (int k0 = 0; k0 < K; k0 += 2 * kMaxPairs) {
        FwdRowJobs fj;
        memset(&fj, 0, sizeof(fj));
        PlaneJobs pj;
        memset(&pj, 0, sizeof(pj));
        for (int k = k0; k < K && k < k0 + 2 * kMaxPairs; k += 2) {
            const int p = fj.npairs++;
            fj.in[2 * p] = grids + (size_t)k * d.N;
            fj.out[2 * p] = w->S + (size_t)k * d.HS;
            fj.in[2 * p + 1] = k + 1 < K ? grids + (size_t)(k + 1) * d.N : nullptr;
            fj.out[2 * p + 1] = k + 1 < K ? w->S + (size_t)(k + 1) * d.HS : nullptr;
        }
        if ((e = launch_fwd_rows(d, w->px, w->tw_x_fwd, fj, st)) != cudaSuccess) goto out;
        for (int k = k0; k < K && k < k0 + 2 * kMaxPairs; k++) {
            if (pj.njobs == kMaxKernels + 8) {
                if ((e = launch_planes(d, w->py, w->px, w->tw_y_fwd, w->tw_x_fwd, pj, -1, st)) != cudaSuccess) goto out;
                pj.njobs = 0;
            }
            pj.src[pj.njobs] = w->S + (size_t)k * d.HS;
            pj.dst[pj.njobs] = w->S + (size_t)k * d.HS;
            pj.kc[pj.njobs] = nullptr;
            pj.njobs++;
        }
        if (pj.njobs && (e = launch_planes(d, w->py, w->px, w->tw_y_fwd, w->tw_x_fwd, pj, -1, st)) != cudaSuccess)
            goto out;
    }
    for (int k = 0; k < K; k++) {
        const size_t kh = (size_t)d.KX * (d.D / 2 + 1) * (d.H / 2 + 1);
        if ((e = launch_compress(d, w->S + (size_t)k * d.HS, w->Kc + k * kh, st)) != cudaSuccess) goto out;
    }
    // blur kernel (precompute_blur_kernel, reintegration.cpp:13-78)
    if ((e = launch_blur_grid(d, grids, w->ksum + K, st)) != cudaSuccess) goto out;
    {
        FwdRowJobs fj;
        memset(&fj, 0, sizeof(fj));
        fj.npairs = 1;
        fj.in[0] = grids;
        fj.out[0] = w->S;
        if ((e = launch_fwd_rows(d, w->px, w->tw_x_fwd, fj, st)) != cudaSuccess) goto out;
        PlaneJobs pj;
        memset(&pj, 0, sizeof(pj));
        pj.njobs = 1;
        pj.src[0] = w->S;
        pj.dst[0] = w->S;
        if ((e = launch_planes(d, w->py, w->px, w->tw_y_fwd, w->tw_x_fwd, pj, -1, st)) != cudaSuccess) goto out;
        if ((e = launch_compress(d, w->S, w->blur_hat, st)) != cudaSuccess) goto out;
    }
    if ((e = launch_lut_rows(w->kp_dev, K, w->lut_rows, w->lut_base, st)) != cudaSuccess) goto out;
    if (K > 0) {
        e = cudaMemcpyAsync(w->lut_base_host, w->lut_base, sizeof(int) * K, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) goto out;
    }
out:
    cudaFreeAsync(grids, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(w, e, "building kernels");
    return LENIA_OK;
}

void free_world(lenia_world *w)
{
    float *fs[] = {w->A, w->A_next, w->V, w->GA, w->SUM, w->H_RB, w->U_SUM_RB, w->RBB, w->NA, w->NU, w->PREALPHA,
                   w->TT, w->U, w->Kc, w->blur_hat, w->lut_rows, w->ksum};
    for (float *p : fs)
        if (p) cudaFree(p);
    void *vs[] = {w->lut_base, w->kp_dev, w->tw_x_fwd, w->tw_x_inv, w->tw_y_fwd, w->tw_y_inv, w->err_flag,
                  w->stats_trig, w->stats_partial, w->mass_target, w->mass_total, w->mass_partial};
    for (void *p : vs)
        if (p) cudaFree(p);
    direct_destroy(w->dconv);
    w->dconv = nullptr;
    if (!w->shared_scratch) {
        void *sc[] = {w->H, w->U_SUM, w->BACK, w->MU, w->F, w->ALPHA, w->U_S, w->SUM_S, w->XS, w->S};
        for (void *p : sc)
            if (p) cudaFree(p);
    }
}

// Grid statistics of the world's current A into dst (device, C x kStats
// doubles), on the world's stream.
lenia_status world_stats_async(lenia_world *w, float fill, double *dst)
{
    cudaError_t e = cudaSuccess;
    if (!w->stats_trig) {
        const int W = w->d.W, H = w->d.H;
        std::vector<double> t(2 * (size_t)W + 2 * (size_t)H);
        const double pi = 3.14159265358979323846;
        for (int x = 0; x < W; x++) {
            t[x] = cos(2.0 * pi * x / W);
            t[W + x] = sin(2.0 * pi * x / W);
        }
        for (int y = 0; y < H; y++) {
            t[2 * W + y] = cos(2.0 * pi * y / H);
            t[2 * W + H + y] = sin(2.0 * pi * y / H);
        }
        w->stats_trig = dalloc<double>(t.size(), e);
        w->stats_partial = dalloc<double>((size_t)w->C * kStatBlocks * kStats, e);
        if (e == cudaSuccess)
            e = cudaMemcpy(w->stats_trig, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(w, e, "statistics buffers");
    }
    e = launch_stats(w->A, w->d, w->C, w->stats_trig, fill, w->stats_partial, kStatBlocks, dst, w->stream);
    if (e != cudaSuccess) return cuda_fail(w, e, "statistics");
    return LENIA_OK;
}

constexpr int kMassBlocks = 64;

// conserve_mass: records the current channel totals of A as the totals every
// later step restores (allocates its buffers on first use; stream-ordered).
lenia_status mass_record_target(lenia_world *w)
{
    cudaError_t e = cudaSuccess;
    if (!w->mass_target) {
        w->mass_target = dalloc<double>(kMaxChannels, e);
        w->mass_total = dalloc<double>(kMaxChannels, e);
        w->mass_partial = dalloc<double>((size_t)kMaxChannels * kMassBlocks, e);
        if (e != cudaSuccess) return cuda_fail(w, e, "mass conservation buffers");
    }
    e = launch_mass_totals(w->A, w->d, w->C, w->mass_partial, kMassBlocks, w->mass_target, w->stream);
    if (e != cudaSuccess) return cuda_fail(w, e, "mass totals");
    return LENIA_OK;
}

}  // namespace

// The conserve_mass target totals (one double per channel) of a world that
// has recorded them: copied out (synchronises the world's stream; returns the
// channel count, 0 when none are recorded) or replaced (stream-ordered).
int lenia::mass_target_get(lenia_world *w, double *host, int n)
{
    if (!w || !w->mass_target || n < w->C) return 0;
    if (cudaStreamSynchronize(w->stream) != cudaSuccess) return 0;
    if (cudaMemcpy(host, w->mass_target, sizeof(double) * w->C, cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
    return w->C;
}

lenia_status lenia::mass_target_set(lenia_world *w, const double *host, int n)
{
    if (!w || n != w->C) return LENIA_ERR_INVALID_ARG;
    if (!w->mass_target) {
        const lenia_status s = mass_record_target(w);
        if (s != LENIA_OK) return s;
    }
    const cudaError_t e =
        cudaMemcpyAsync(w->mass_target, host, sizeof(double) * n, cudaMemcpyHostToDevice, w->stream);
    if (e == cudaSuccess) return cudaStreamSynchronize(w->stream) == cudaSuccess ? LENIA_OK : LENIA_ERR_CUDA;
    return cuda_fail(w, e, "mass target");
}

namespace {

// Per-step buffers a batch lane lends to its worlds (they run one after
// another on the lane's stream).
struct WorldScratch {
    float *H, *U_SUM, *BACK, *MU, *F, *ALPHA, *U_S, *SUM_S;
    float2 *XS, *S;
};

// ---------------------------------------------------------------- stages

// The growth stage's jobs of a world (kernel spectra, targets, weights,
// growth-table rows, channel flags).
GrowthJobs growth_jobs(const lenia_world *w)
{
    const Dims &d = w->d;
    GrowthJobs gj;
    memset(&gj, 0, sizeof(gj));
    gj.K = w->K;
    gj.C = w->C;
    for (int k = 0; k < w->K; k++) {
        gj.spec[k] = w->S + (size_t)k * d.HS;
        gj.c1[k] = w->kernels[k].c1;
        gj.h[k] = w->kernels[k].h;
        gj.lut_base[k] = w->lut_base_host[k];
    }
    for (int c = 0; c < kMaxChannels; c++) {
        gj.asymptotic[c] = w->desc.asymptotic[c];
        gj.soft_clip[c] = w->desc.soft_clip[c];
    }
    gj.growth_rt = w->desc.growth_type == LENIA_GROWTH_RT;
    gj.timestep = w->desc.timestep;
    gj.exact_bell = w->desc.exact_bell;
    for (int k = 0; k < w->K; k++) {
        gj.m[k] = w->kernels[k].m;
        gj.s[k] = w->kernels[k].s;
    }
    return gj;
}

// The flow stage's buffers of a world (its current grid).
FlowBuffers flow_buffers(const lenia_world *w)
{
    FlowBuffers b;
    memset(&b, 0, sizeof(b));
    const bool cd = w->desc.gradient_mode == LENIA_GRADIENT_CENTRAL_DIFF;
    // Without the blur, U_S and SUM_S are plain copies of H and SUM
    // (the intended h_sum_blur copy): read H and SUM directly.
    b.H = (cd && w->blur_valid) ? w->U_S : w->H;
    b.SUM = (cd && w->blur_valid) ? w->SUM_S : w->SUM;
    b.A = w->A;
    b.GA = w->GA;
    b.V = w->V;
    b.MU = w->MU;
    b.F = (w->debug || needs_F(w->desc)) ? w->F : nullptr;
    b.ALPHA = (w->debug || w->desc.osc_div_flow) ? w->ALPHA : nullptr;
    b.err = w->err_flag;
    if (w->debug) {
        b.NA = w->NA;
        b.NU = w->NU;
        b.PREALPHA = w->PREALPHA;
    }
    return b;
}

// The transport stage's buffers of a world (current grid A, new grid A_next).
TransportBuffers transport_buffers(const lenia_world *w)
{
    TransportBuffers b;
    memset(&b, 0, sizeof(b));
    const bool use_grid =
        w->desc.growth_type == LENIA_GROWTH_NOGROWTH || w->desc.growth_type == LENIA_GROWTH_TRANSPOSITION;
    b.A = w->A;
    b.A_out = w->A_next;
    b.ARR = use_grid ? w->A : w->BACK;
    b.MU = w->MU;
    b.H = w->H;
    b.V = w->V;
    b.F = w->F;
    b.ALPHA = w->ALPHA;
    b.GA = w->GA;
    b.SUM = w->SUM;
    b.BACK = w->BACK;
    b.TT = w->debug ? w->TT : nullptr;
    b.err = w->err_flag;
    return b;
}

lenia_status stage_growth(lenia_world *w)
{
    const Dims &d = w->d;
    cudaStream_t st = w->stream;
    cudaError_t e;
    if (w->snapshots) {
        std::swap(w->H, w->H_RB);
        std::swap(w->U_SUM, w->U_SUM_RB);
    }
    const GrowthJobs gj = growth_jobs(w);
    if (w->conv_mode != LENIA_CONV_FFT) {
        // direct convolution on the tensor cores, then the growth from u_k
        if (!w->dconv && w->K > 0) return fail(w, LENIA_ERR_INVALID_ARG, "direct convolution has no plan");
        if (w->dconv) {
            {
                ProfScope ps(w, KID_DIRECT_PAD);
                if ((e = direct_pad(w->dconv, w->A, st)) != cudaSuccess) return cuda_fail(w, e, "direct_pad");
            }
            {
                ProfScope ps(w, KID_DIRECT_CONV);
                if ((e = direct_convolve(w->dconv, w->U, w->err_flag, st)) != cudaSuccess)
                    return cuda_fail(w, e, "direct_conv");
            }
            w->launches += 2;
        }
        {
            ProfScope ps(w, KID_GROWTH_U);
            if ((e = launch_growth_from_u(d, gj, w->lut_rows, w->U, w->A, w->H, w->U_SUM, w->BACK, w->err_flag, st)) !=
                cudaSuccess)
                return cuda_fail(w, e, "growth_u");
        }
        w->launches++;
        return LENIA_OK;
    }
    // forward transforms of the grid channels, packed in pairs
    FwdRowJobs fj;
    memset(&fj, 0, sizeof(fj));
    for (int c = 0; c < w->C; c += 2) {
        const int p = fj.npairs++;
        fj.in[2 * p] = w->A + (size_t)c * d.N;
        fj.out[2 * p] = w->XS + (size_t)c * d.HS;
        fj.in[2 * p + 1] = c + 1 < w->C ? w->A + (size_t)(c + 1) * d.N : nullptr;
        fj.out[2 * p + 1] = c + 1 < w->C ? w->XS + (size_t)(c + 1) * d.HS : nullptr;
    }
    {
        ProfScope ps(w, KID_FWD_ROWS);
        if ((e = launch_fwd_rows(d, w->px, w->tw_x_fwd, fj, st)) != cudaSuccess) return cuda_fail(w, e, "fwd_rows");
    }
    PlaneJobs pj;
    memset(&pj, 0, sizeof(pj));
    pj.njobs = w->C;
    for (int c = 0; c < w->C; c++) {
        pj.src[c] = w->XS + (size_t)c * d.HS;
        pj.dst[c] = w->XS + (size_t)c * d.HS;
        pj.kc[c] = nullptr;
    }
    {
        ProfScope ps(w, KID_PLANES_FWD);
        if ((e = launch_planes(d, w->py, w->px, w->tw_y_fwd, w->tw_x_fwd, pj, -1, st)) != cudaSuccess)
            return cuda_fail(w, e, "planes (forward)");
    }
    w->launches += 2;
    if (w->K > 0) {
        const size_t kh = (size_t)d.KX * (d.D / 2 + 1) * (d.H / 2 + 1);
        memset(&pj, 0, sizeof(pj));
        pj.njobs = w->K;
        for (int k = 0; k < w->K; k++) {
            pj.src[k] = w->XS + (size_t)w->kernels[k].c0 * d.HS;
            pj.dst[k] = w->S + (size_t)k * d.HS;
            pj.kc[k] = w->Kc + k * kh;
        }
        ProfScope ps(w, KID_PLANES_INV);
        if ((e = launch_planes(d, w->py, w->px, w->tw_y_inv, w->tw_x_inv, pj, +1, st)) != cudaSuccess)
            return cuda_fail(w, e, "planes (inverse)");
        w->launches++;
    }
    if (w->growth_split && w->K > 0) {
        // two passes: the inverse row transforms store u_k of every kernel
        // (kernel pairs as in the fused pass, sixteen fields per launch),
        // then the growth from u_k
        if (!w->U) return fail(w, LENIA_ERR_INVALID_ARG, "the split growth has no u_k buffer");
        for (int k0 = 0; k0 < w->K; k0 += kBlurFields) {
            BlurJobs bj;
            memset(&bj, 0, sizeof(bj));
            bj.nfields = std::min(w->K - k0, kBlurFields);
            for (int i = 0; i < bj.nfields; i++) {
                bj.spec[i] = w->S + (size_t)(k0 + i) * d.HS;
                bj.out[i] = w->U + (size_t)(k0 + i) * d.N;
            }
            ProfScope ps(w, KID_INV_ROWS);
            if ((e = launch_blur_rows(d, w->px, w->tw_x_inv, bj, st)) != cudaSuccess)
                return cuda_fail(w, e, "inverse rows");
            w->launches++;
        }
        ProfScope ps(w, KID_GROWTH_U);
        if ((e = launch_growth_from_u(d, gj, w->lut_rows, w->U, w->A, w->H, w->U_SUM, w->BACK, w->err_flag, st)) !=
            cudaSuccess)
            return cuda_fail(w, e, "growth_u");
        w->launches++;
        return LENIA_OK;
    }
    {
        ProfScope ps(w, KID_GROWTH_ROWS);
        if ((e = launch_growth_rows(d, w->px, w->tw_x_inv, gj, w->lut_rows, w->A, w->H, w->U_SUM, w->BACK,
                                    w->debug ? w->U : nullptr, w->err_flag, st)) != cudaSuccess)
            return cuda_fail(w, e, "growth_rows");
    }
    w->launches++;
    return LENIA_OK;
}

lenia_status stage_blur(lenia_world *w)
{
    const LeniaWorldDesc &s = w->desc;
    if (s.gradient_mode != LENIA_GRADIENT_CENTRAL_DIFF || !s.blur_central_diff) {
        w->blur_valid = false;
        return LENIA_OK;
    }
    const Dims &d = w->d;
    cudaStream_t st = w->stream;
    cudaError_t e;
    const int nf = w->C + 1;  // H_0..H_{C-1}, SUM
    FwdRowJobs fj;
    memset(&fj, 0, sizeof(fj));
    auto field_in = [&](int f) -> const float * { return f < w->C ? w->H + (size_t)f * d.N : w->SUM; };
    auto field_out = [&](int f) -> float * { return f < w->C ? w->U_S + (size_t)f * d.N : w->SUM_S; };
    for (int f = 0; f < nf; f += 2) {
        const int p = fj.npairs++;
        fj.in[2 * p] = field_in(f);
        fj.out[2 * p] = w->XS + (size_t)f * d.HS;
        fj.in[2 * p + 1] = f + 1 < nf ? field_in(f + 1) : nullptr;
        fj.out[2 * p + 1] = f + 1 < nf ? w->XS + (size_t)(f + 1) * d.HS : nullptr;
    }
    {
        ProfScope ps(w, KID_BLUR_FWD_ROWS);
        if ((e = launch_fwd_rows(d, w->px, w->tw_x_fwd, fj, st)) != cudaSuccess)
            return cuda_fail(w, e, "blur fwd_rows");
    }
    PlaneJobs pj;
    memset(&pj, 0, sizeof(pj));
    pj.njobs = nf;
    for (int f = 0; f < nf; f++) {
        pj.src[f] = w->XS + (size_t)f * d.HS;
        pj.dst[f] = w->XS + (size_t)f * d.HS;
    }
    {
        ProfScope ps(w, KID_BLUR_PLANES_FWD);
        if ((e = launch_planes(d, w->py, w->px, w->tw_y_fwd, w->tw_x_fwd, pj, -1, st)) != cudaSuccess)
            return cuda_fail(w, e, "blur planes (forward)");
    }
    for (int f = 0; f < nf; f++) {
        pj.src[f] = w->XS + (size_t)f * d.HS;
        pj.dst[f] = w->S + (size_t)f * d.HS;
        pj.kc[f] = w->blur_hat;
    }
    {
        ProfScope ps(w, KID_BLUR_PLANES_INV);
        if ((e = launch_planes(d, w->py, w->px, w->tw_y_inv, w->tw_x_inv, pj, +1, st)) != cudaSuccess)
            return cuda_fail(w, e, "blur planes (inverse)");
    }
    BlurJobs bj;
    memset(&bj, 0, sizeof(bj));
    bj.nfields = nf;
    for (int f = 0; f < nf; f++) {
        bj.spec[f] = w->S + (size_t)f * d.HS;
        bj.out[f] = field_out(f);
    }
    {
        ProfScope ps(w, KID_BLUR_ROWS);
        if ((e = launch_blur_rows(d, w->px, w->tw_x_inv, bj, st)) != cudaSuccess) return cuda_fail(w, e, "blur rows");
    }
    w->launches += 4;
    w->blur_valid = true;
    return LENIA_OK;
}

lenia_status stage_flow(lenia_world *w)
{
    lenia_status s = ensure_optional(w);
    if (s != LENIA_OK) return s;
    const StepParams p = step_params(w);
    const FlowBuffers b = flow_buffers(w);
    cudaError_t e;
    {
        ProfScope ps(w, KID_FLOW);
        e = launch_flow(p, b, w->stream);
    }
    if (e != cudaSuccess) return cuda_fail(w, e, "flow");
    w->launches++;
    return LENIA_OK;
}

cudaError_t rbb_materialize(lenia_world *w);

lenia_status stage_transport(lenia_world *w)
{
    const StepParams p = step_params(w);
    const TransportBuffers b = transport_buffers(w);
    cudaError_t e;
    // the new grid overwrites A_next: a deferred snapshot of it is copied first
    if (w->rbb_src == w->A_next && (e = rbb_materialize(w)) != cudaSuccess) return cuda_fail(w, e, "snapshot");
    {
        ProfScope ps(w, KID_TRANSPORT);
        e = launch_transport(p, b, w->stream);
    }
    if (e != cudaSuccess) return cuda_fail(w, e, "transport");
    std::swap(w->A, w->A_next);
    w->launches++;
    if (w->desc.conserve_mass) {
        // the new grid's channel totals (double, fixed order), then the
        // rescaling that restores the recorded totals
        if (!w->mass_target) return fail(w, LENIA_ERR_INVALID_ARG, "conserve_mass has no recorded totals");
        ProfScope ps(w, KID_MASS);
        if ((e = launch_mass_totals(w->A, w->d, w->C, w->mass_partial, kMassBlocks, w->mass_total, w->stream)) !=
                cudaSuccess ||
            (e = launch_mass_scale(w->A, w->d, w->C, w->mass_target, w->mass_total, w->stream)) != cudaSuccess)
            return cuda_fail(w, e, "mass conservation");
        w->launches += 3;
    }
    return LENIA_OK;
}

// RBB := the grid buffer it stands for, if the copy was deferred.
cudaError_t rbb_materialize(lenia_world *w)
{
    if (!w->rbb_src || !w->RBB) return cudaSuccess;
    const float *src = w->rbb_src;
    w->rbb_src = nullptr;
    return cudaMemcpyAsync(w->RBB, src, sizeof(float) * w->C * w->d.N, cudaMemcpyDeviceToDevice, w->stream);
}

// The snapshot of the grid the step produced (render.cpp's copy to RBB).
// The copy itself is deferred: until RBB is read or the grid buffer is
// written again, RBB's contents are that buffer's, which meshing reads in
// place.
lenia_status stage_snapshot(lenia_world *w)
{
    lenia_status s = ensure_optional(w);
    if (s != LENIA_OK) return s;
    if (!w->RBB) return LENIA_OK;
    w->rbb_src = w->A;
    return LENIA_OK;
}

float *field_ptr(lenia_world *w, int field, size_t *count)
{
    const size_t N = w->d.N, CN = (size_t)w->C * N;
    const bool cd_plain = !w->blur_valid;
    switch (field) {
    case LENIA_FIELD_A: *count = CN; return w->A;
    case LENIA_FIELD_V: *count = 3 * CN; return w->V;
    case LENIA_FIELD_GA: *count = CN; return w->GA;
    case LENIA_FIELD_SUM: *count = N; return w->SUM;
    case LENIA_FIELD_H: *count = CN; return w->H;
    case LENIA_FIELD_U_SUM: *count = CN; return w->U_SUM;
    case LENIA_FIELD_BACK: *count = CN; return w->BACK;
    case LENIA_FIELD_NA: *count = 3 * N; return w->NA;
    case LENIA_FIELD_NU: *count = 3 * CN; return w->NU;
    case LENIA_FIELD_PREALPHA: *count = CN; return w->PREALPHA;
    case LENIA_FIELD_ALPHA: *count = CN; return w->ALPHA;
    case LENIA_FIELD_F: *count = 3 * CN; return w->F;
    case LENIA_FIELD_MU: *count = 3 * CN; return w->MU;
    case LENIA_FIELD_TT: *count = CN; return w->TT;
    case LENIA_FIELD_U_S: *count = CN; return cd_plain ? w->H : w->U_S;
    case LENIA_FIELD_SUM_S: *count = N; return cd_plain ? w->SUM : w->SUM_S;
    case LENIA_FIELD_U: *count = (size_t)w->K * N; return w->U;
    case LENIA_FIELD_H_RB: *count = CN; return w->snapshots ? w->H_RB : nullptr;
    case LENIA_FIELD_U_SUM_RB: *count = CN; return w->snapshots ? w->U_SUM_RB : nullptr;
    case LENIA_FIELD_RBB: *count = CN; return w->RBB;
    default: *count = 0; return nullptr;
    }
}

// The stream a world created for itself.
void destroy_streams(lenia_world *w)
{
    if (w->own_stream) cudaStreamDestroy(w->own_stream);
    w->own_stream = nullptr;
}

// A world; with `shared`, the per-step buffers are the lane's and the
// kernels are built on `stream` (which the world then uses).
lenia_status create_world(const LeniaWorldDesc *desc, const LeniaKernelParams *kernels, int n_kernels,
                          const WorldScratch *shared, cudaStream_t stream, lenia_world **out)
{
    if (!out) return LENIA_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return LENIA_ERR_NO_DEVICE;
    }
    lenia_world *w = new lenia_world();
    lenia_status s = validate_desc(w, desc);
    if (s == LENIA_OK) s = validate_kernels(w, kernels, n_kernels, desc->channels);
    if (s != LENIA_OK) {
        fprintf(stderr, "lenia_create: %s\n", w->err.c_str());
        delete w;
        return s;
    }
    w->desc = *desc;
    w->kernels.assign(kernels, kernels + n_kernels);
    w->C = desc->channels;
    w->K = n_kernels;
    Dims &d = w->d;
    d.W = desc->width;
    d.H = desc->height;
    d.D = desc->width;
    d.N = (long long)d.W * d.H * d.D;
    d.KX = d.W / 2 + 1;
    d.HS = (long long)d.KX * d.D * d.H;
    d.P = (long long)(d.W + 8) * (d.H + 8) * (d.W + 8);
    w->px.n = d.W;
    w->px.nstages = fft_factor(d.W, w->px.radix);
    w->py.n = d.H;
    w->py.nstages = fft_factor(d.H, w->py.radix);
    if (row_tile(d, w->px) == 0 || !planes_supported(d, w->py, w->px)) {
        delete w;
        return LENIA_ERR_UNSUPPORTED;
    }
    cudaGetDevice(&w->device);
    cudaError_t e = cudaSuccess;
    const size_t N = d.N, CN = (size_t)w->C * N;
    w->A = dalloc<float>(CN, e);
    w->A_next = dalloc<float>(CN, e);
    w->V = dalloc<float>(3 * CN, e);
    w->GA = dalloc<float>(CN, e);
    w->SUM = dalloc<float>(N, e);
    if (shared) {
        w->shared_scratch = true;
        w->H = shared->H;
        w->U_SUM = shared->U_SUM;
        w->BACK = shared->BACK;
        w->MU = shared->MU;
        w->F = shared->F;
        w->ALPHA = shared->ALPHA;
        w->U_S = shared->U_S;
        w->SUM_S = shared->SUM_S;
        w->XS = shared->XS;
        w->S = shared->S;
    } else {
        w->H = dalloc<float>(CN, e);
        w->H_RB = dalloc<float>(CN, e);
        w->U_SUM = dalloc<float>(CN, e);
        w->U_SUM_RB = dalloc<float>(CN, e);
        w->BACK = dalloc<float>(CN, e);
        w->MU = dalloc<float>(3 * CN, e);
        w->U_S = dalloc<float>(CN, e);
        w->SUM_S = dalloc<float>(N, e);
        w->XS = dalloc<float2>((size_t)(w->C + 1) * d.HS, e);
        w->S = dalloc<float2>((size_t)std::max(w->K, w->C + 1) * d.HS, e);
    }
    const size_t kh = (size_t)d.KX * (d.D / 2 + 1) * (d.H / 2 + 1);
    w->Kc = dalloc<float>(std::max(w->K, 1) * kh, e);
    w->blur_hat = dalloc<float>(kh, e);
    w->lut_rows = dalloc<float>(256 * (size_t)std::max(w->K, 1), e);
    w->lut_base = dalloc<int>(std::max(w->K, 1), e);
    w->ksum = dalloc<float>(w->K + 1, e);
    w->kp_dev = dalloc<LeniaKernelParams>(kMaxKernels, e);
    w->tw_x_fwd = dalloc<float2>(d.W, e);
    w->tw_x_inv = dalloc<float2>(d.W, e);
    w->tw_y_fwd = dalloc<float2>(d.H, e);
    w->tw_y_inv = dalloc<float2>(d.H, e);
    w->err_flag = dalloc<int>(1, e);
    if (e == cudaSuccess) {
        auto a = twiddles(d.W, -1), b = twiddles(d.W, +1), c = twiddles(d.H, -1), dd = twiddles(d.H, +1);
        e = cudaMemcpy(w->tw_x_fwd, a.data(), sizeof(float2) * d.W, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(w->tw_x_inv, b.data(), sizeof(float2) * d.W, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(w->tw_y_fwd, c.data(), sizeof(float2) * d.H, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(w->tw_y_inv, dd.data(), sizeof(float2) * d.H, cudaMemcpyHostToDevice);
    }
    if (shared) {
        w->stream = stream;
    } else {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&w->own_stream, cudaStreamNonBlocking);
        w->stream = w->own_stream;
    }
    if (e != cudaSuccess) {
        s = e == cudaErrorMemoryAllocation ? LENIA_ERR_OOM : LENIA_ERR_CUDA;
        fprintf(stderr, "lenia_create: %s\n", cudaGetErrorString(e));
        free_world(w);
        destroy_streams(w);
        delete w;
        return s;
    }
    s = build_kernels(w);
    if (s == LENIA_OK && w->desc.conserve_mass) s = mass_record_target(w);
    if (s != LENIA_OK) {
        fprintf(stderr, "lenia_create: %s\n", w->err.c_str());
        free_world(w);
        destroy_streams(w);
        delete w;
        return s;
    }
    *out = w;
    return LENIA_OK;
}

}  // namespace

extern "C" {

const char *lenia_version(void) { return "lenia_b200 0.1 (sm_100a)"; }

lenia_status lenia_create(const LeniaWorldDesc *desc, const LeniaKernelParams *kernels, int n_kernels,
                          lenia_world **out)
{
    return create_world(desc, kernels, n_kernels, nullptr, nullptr, out);
}

lenia_status lenia_destroy(lenia_world *w)
{
    if (!w) return LENIA_ERR_INVALID_ARG;
    cudaStreamSynchronize(w->stream);
    for (const ProfRec &r : w->prof_pending) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (cudaEvent_t e : w->prof_free) cudaEventDestroy(e);
    free_world(w);
    destroy_streams(w);
    delete w;
    return LENIA_OK;
}

lenia_status lenia_set_params(lenia_world *w, const LeniaWorldDesc *desc)
{
    if (!w) return LENIA_ERR_INVALID_ARG;
    lenia_status s = validate_desc(w, desc);
    if (s != LENIA_OK) return s;
    if (desc->width != w->desc.width || desc->height != w->desc.height || desc->channels != w->desc.channels)
        return fail(w, LENIA_ERR_INVALID_ARG, "set_params cannot change the grid shape or channel count");
    w->desc = *desc;
    if (desc->conserve_mass) return mass_record_target(w);
    return LENIA_OK;
}

lenia_status lenia_set_kernels(lenia_world *w, const LeniaKernelParams *kernels, int n_kernels)
{
    if (!w) return LENIA_ERR_INVALID_ARG;
    lenia_status s = validate_kernels(w, kernels, n_kernels, w->C);
    if (s != LENIA_OK) return s;
    const Dims &d = w->d;
    cudaError_t e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) return cuda_fail(w, e, "set_kernels");
    if (n_kernels > w->K) {
        // grow the per-kernel buffers
        const size_t kh = (size_t)d.KX * (d.D / 2 + 1) * (d.H / 2 + 1);
        cudaFree(w->S);
        cudaFree(w->Kc);
        cudaFree(w->lut_rows);
        cudaFree(w->lut_base);
        cudaFree(w->ksum);
        if (w->U) { cudaFree(w->U); w->U = nullptr; }
        e = cudaSuccess;
        w->S = dalloc<float2>((size_t)std::max(n_kernels, w->C + 1) * d.HS, e);
        w->Kc = dalloc<float>(n_kernels * kh, e);
        w->lut_rows = dalloc<float>(256 * (size_t)n_kernels, e);
        w->lut_base = dalloc<int>(n_kernels, e);
        w->ksum = dalloc<float>(n_kernels + 1, e);
        if (e != cudaSuccess) return cuda_fail(w, e, "set_kernels");
    }
    w->kernels.assign(kernels, kernels + n_kernels);
    w->K = n_kernels;
    return build_kernels(w);
}

size_t lenia_field_size(const lenia_world *w, int field)
{
    if (!w) return 0;
    size_t n = 0;
    field_ptr(const_cast<lenia_world *>(w), field, &n);
    return n;
}

lenia_status lenia_set_field(lenia_world *w, int field, const float *src, size_t count, int on_device)
{
    if (!w || !src) return LENIA_ERR_INVALID_ARG;
    if (field == LENIA_FIELD_U_S || field == LENIA_FIELD_SUM_S) {
        // the blur stage owns these; writing them selects them as flow inputs
        w->blur_valid = true;
    }
    if (field == LENIA_FIELD_H_RB || field == LENIA_FIELD_U_SUM_RB || field == LENIA_FIELD_RBB) {
        w->snapshots = true;
    }
    lenia_status s = ensure_optional(w);
    if (s != LENIA_OK) return s;
    size_t n = 0;
    float *p = field_ptr(w, field, &n);
    if (!p) return fail(w, LENIA_ERR_INVALID_ARG, "field %d is not available (enable debug?)", field);
    if (count != n) return fail(w, LENIA_ERR_INVALID_ARG, "field %d holds %zu floats, got %zu", field, n, count);
    cudaError_t e = cudaSuccess;
    if (field == LENIA_FIELD_RBB) w->rbb_src = nullptr;  // replaced whole
    else if (field == LENIA_FIELD_A && w->rbb_src == w->A) e = rbb_materialize(w);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p, src, count * sizeof(float),
                                    on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, w->stream);
    if (e == cudaSuccess && !on_device) e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) return cuda_fail(w, e, "set_field");
    if (field == LENIA_FIELD_A && w->desc.conserve_mass) return mass_record_target(w);
    return LENIA_OK;
}

lenia_status lenia_get_field(lenia_world *w, int field, float *dst, size_t count, int on_device)
{
    if (!w || !dst) return LENIA_ERR_INVALID_ARG;
    size_t n = 0;
    float *p = field_ptr(w, field, &n);
    if (!p) return fail(w, LENIA_ERR_INVALID_ARG, "field %d is not available (enable debug?)", field);
    if (count != n) return fail(w, LENIA_ERR_INVALID_ARG, "field %d holds %zu floats, got %zu", field, n, count);
    cudaError_t e = field == LENIA_FIELD_RBB ? rbb_materialize(w) : cudaSuccess;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dst, p, count * sizeof(float), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                            w->stream);
    if (e == cudaSuccess && !on_device) e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) return cuda_fail(w, e, "get_field");
    return LENIA_OK;
}

lenia_status lenia_step_stage(lenia_world *w, int stage)
{
    if (!w) return LENIA_ERR_INVALID_ARG;
    switch (stage) {
    case LENIA_STAGE_GROWTH: return stage_growth(w);
    case LENIA_STAGE_BLUR: return stage_blur(w);
    case LENIA_STAGE_FLOW: return stage_flow(w);
    case LENIA_STAGE_TRANSPORT: return stage_transport(w);
    case LENIA_STAGE_SNAPSHOT: return stage_snapshot(w);
    default: return fail(w, LENIA_ERR_INVALID_ARG, "unknown stage %d", stage);
    }
}

lenia_status lenia_step(lenia_world *w, int n_steps)
{
    if (!w || n_steps < 0) return LENIA_ERR_INVALID_ARG;
    NvtxRange range("lenia_step");
    lenia_status s = ensure_optional(w);
    if (s != LENIA_OK) return s;
    for (int i = 0; i < n_steps; i++) {
        w->launches = 0;
        if ((s = stage_growth(w)) != LENIA_OK) return s;
        if ((s = stage_blur(w)) != LENIA_OK) return s;
        if ((s = stage_flow(w)) != LENIA_OK) return s;
        if ((s = stage_transport(w)) != LENIA_OK) return s;
        if (w->snapshots && (s = stage_snapshot(w)) != LENIA_OK) return s;
    }
    return LENIA_OK;
}

lenia_status lenia_set_stream(lenia_world *w, void *stream)
{
    if (!w) return LENIA_ERR_INVALID_ARG;
    cudaError_t e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) return cuda_fail(w, e, "set_stream");
    w->stream = (cudaStream_t)stream;
    return LENIA_OK;
}

lenia_status lenia_sync(lenia_world *w)
{
    if (!w) return LENIA_ERR_INVALID_ARG;
    cudaError_t e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) return cuda_fail(w, e, "sync");
    int flag = 0;
    e = cudaMemcpy(&flag, w->err_flag, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(w, e, "sync");
    if (flag) {
        cudaMemset(w->err_flag, 0, sizeof(int));
        if (flag & 2)
            return fail(w, LENIA_ERR_TIMEOUT,
                        "a bounded wait ran out (a tile copy of the flow or transport stage, or the direct "
                        "convolution's copy/MMA/drain pipeline)");
        return fail(w, LENIA_ERR_NONFINITE, "non-finite u (NaN or infinite) met in the growth stage");
    }
    return LENIA_OK;
}

lenia_status lenia_set_wait_limit(lenia_world *w, long long polls)
{
    if (!w) return LENIA_ERR_INVALID_ARG;
    if (polls > 0xffffffffLL) return fail(w, LENIA_ERR_INVALID_ARG, "wait limit %lld above 2^32 - 1", polls);
    w->wait_polls = polls < 0 ? kDefaultTileWaitPolls : (unsigned)polls;
    return LENIA_OK;
}

lenia_status lenia_set_debug(lenia_world *w, int on)
{
    if (!w) return LENIA_ERR_INVALID_ARG;
    w->debug = on != 0;
    return ensure_optional(w);
}

lenia_status lenia_set_conv_mode(lenia_world *w, int mode)
{
    if (!w) return LENIA_ERR_INVALID_ARG;
    if (mode < LENIA_CONV_FFT || mode > LENIA_CONV_DIRECT_BF16X3)
        return fail(w, LENIA_ERR_INVALID_ARG, "unknown convolution mode %d", mode);
    if (mode != LENIA_CONV_FFT)
        for (const LeniaKernelParams &k : w->kernels)
            if ((float)k.radius * k.r_a > 64.0f)
                return fail(w, LENIA_ERR_UNSUPPORTED, "direct convolution needs radius * r_a <= 64");
    cudaError_t e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) return cuda_fail(w, e, "set_conv_mode");
    const int old = w->conv_mode;
    w->conv_mode = mode;
    lenia_status s = build_kernels(w);
    if (s != LENIA_OK && old != mode) {
        const std::string why = w->err;
        w->conv_mode = old;
        build_kernels(w);
        w->err = why;
    }
    return s;
}

int lenia_get_conv_mode(lenia_world *w) { return w ? w->conv_mode : -1; }

lenia_status lenia_set_tuning(lenia_world *w, int row_tile, int growth_split)
{
    if (!w) return LENIA_ERR_INVALID_ARG;
    if (row_tile < 0 || row_tile > 32 || (row_tile & (row_tile - 1)))
        return fail(w, LENIA_ERR_INVALID_ARG, "row tile %d is not 0 or a power of two up to 32", row_tile);
    cudaError_t e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) return cuda_fail(w, e, "set_tuning");
    if (growth_split && !w->U && w->K > 0) {
        w->U = dalloc<float>((size_t)w->K * w->d.N, e);
        if (e != cudaSuccess) return cuda_fail(w, e, "u_k buffer");
    }
    w->d.ty = row_tile;
    w->growth_split = growth_split != 0;
    return LENIA_OK;
}

// Times the growth stage (the convolution and the growth table) for every
// allowed convolution mode and, on the FFT path's runtime-sized kernels, every
// row tile that fits; keeps the fastest.  The grid state is untouched: the
// growth stage only writes H, U_SUM and BACK, which the next step recomputes
// (the mesh snapshot pair is not rotated while timing).
lenia_status lenia_autotune(lenia_world *w, int modes, LeniaTuneResult *out)
{
    if (!w || !out) return LENIA_ERR_INVALID_ARG;
    if ((modes & ~7) || !(modes & 7)) return fail(w, LENIA_ERR_INVALID_ARG, "autotune: mode mask %d", modes);
    cudaError_t e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) return cuda_fail(w, e, "autotune");
    memset(out, 0, sizeof(*out));
    for (int i = 0; i < 3; i++) out->ms[i] = -1.0f;
    const bool snaps = w->snapshots;
    const int launches = w->launches;
    const int mode0 = w->conv_mode, ty0 = w->d.ty, split0 = w->growth_split;
    w->snapshots = false;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    std::vector<int> tiles = {0};
    if (!fast_rows_supported(w->d)) {
        tiles.clear();
        for (int ty = 32; ty >= 1; ty /= 2) {
            Dims t = w->d;
            t.ty = ty;
            if (row_tile(t, w->px) == ty) tiles.push_back(ty);
        }
    }
    int best_mode = -1, best_ty = 0, best_split = 0;
    float best = 1e30f;
    lenia_status s = LENIA_OK;
    for (int mode = 0; mode < 3 && s == LENIA_OK; mode++) {
        if (!((modes >> mode) & 1)) continue;
        if (w->conv_mode != mode) {
            w->conv_mode = mode;
            if (build_kernels(w) != LENIA_OK) continue;  // e.g. a radius the direct modes do not take
        }
        // FFT: every row tile, with the fused growth and with the split one
        std::vector<std::pair<int, int>> cand;
        if (mode == LENIA_CONV_FFT) {
            for (int ty : tiles)
                for (int split = 0; split < 2; split++) cand.push_back({ty, split});
        } else {
            cand.push_back({ty0, 0});
        }
        for (const auto &c : cand) {
            const int ty = c.first;
            if (c.second && !w->U && w->K > 0) {
                w->U = dalloc<float>((size_t)w->K * w->d.N, e);
                if (e != cudaSuccess) {
                    s = cuda_fail(w, e, "u_k buffer");
                    break;
                }
            }
            w->d.ty = ty;
            w->growth_split = c.second;
            if ((s = stage_growth(w)) != LENIA_OK) break;  // warm-up
            cudaEventRecord(a, w->stream);
            for (int r = 0; r < 3 && s == LENIA_OK; r++) s = stage_growth(w);
            cudaEventRecord(b, w->stream);
            if (s != LENIA_OK) break;
            if ((e = cudaEventSynchronize(b)) != cudaSuccess) {
                s = cuda_fail(w, e, "autotune timing");
                break;
            }
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, a, b);
            ms /= 3.0f;
            if (out->ms[mode] < 0.0f || ms < out->ms[mode]) out->ms[mode] = ms;
            if (ms < best) {
                best = ms;
                best_mode = mode;
                best_ty = ty;
                best_split = c.second;
            }
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    w->snapshots = snaps;
    w->launches = launches;
    if (s == LENIA_OK && best_mode < 0) s = fail(w, LENIA_ERR_UNSUPPORTED, "autotune: no allowed mode runs");
    const int keep_mode = s == LENIA_OK ? best_mode : mode0;
    w->d.ty = s == LENIA_OK ? best_ty : ty0;
    w->growth_split = s == LENIA_OK ? best_split : split0;
    if (w->conv_mode != keep_mode) {
        w->conv_mode = keep_mode;
        const lenia_status s2 = build_kernels(w);
        if (s == LENIA_OK) s = s2;
    }
    out->conv_mode = w->conv_mode;
    out->row_tile = w->d.ty;
    out->growth_split = w->growth_split;
    return s;
}

lenia_status lenia_conv_macs(lenia_world *w, double *issued, double *useful)
{
    if (!w) return LENIA_ERR_INVALID_ARG;
    double a = 0.0, b = 0.0;
    if (w->dconv) direct_counts(w->dconv, &a, &b);
    if (issued) *issued = a;
    if (useful) *useful = b;
    return LENIA_OK;
}

lenia_status lenia_set_snapshots(lenia_world *w, int on)
{
    if (!w) return LENIA_ERR_INVALID_ARG;
    w->snapshots = on != 0;
    return ensure_optional(w);
}

lenia_status lenia_set_profiling(lenia_world *w, int on)
{
    if (!w) return LENIA_ERR_INVALID_ARG;
    w->profile = on != 0;
    return LENIA_OK;
}

int lenia_profile_read(lenia_world *w, double *ms, long long *launches, int n)
{
    if (!w) return -1;
    cudaStreamSynchronize(w->stream);
    for (const ProfRec &r : w->prof_pending) {
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess) {
            w->prof_ms[r.kid] += t;
            w->prof_n[r.kid] += 1;
        }
        w->prof_free.push_back(r.a);
        w->prof_free.push_back(r.b);
    }
    w->prof_pending.clear();
    for (int k = 0; k < KID_MAX && k < n; k++) {
        if (ms) ms[k] = w->prof_ms[k];
        if (launches) launches[k] = w->prof_n[k];
        w->prof_ms[k] = 0.0;
        w->prof_n[k] = 0;
    }
    return KID_MAX;
}

lenia_status lenia_mesh_world(lenia_world *w, int view, lenia_mesher *m, long long *n_vertices,
                              long long *n_triangles)
{
    if (!w || !m) return LENIA_ERR_INVALID_ARG;
    if (view < LENIA_VIEW_NORMAL || view > LENIA_VIEW_H)
        return fail(w, LENIA_ERR_INVALID_ARG, "unknown view %d", view);
    if (!w->snapshots || !w->RBB) return fail(w, LENIA_ERR_INVALID_ARG, "meshing reads the snapshots: enable them");
    if (mesher_fields(m) != view + 1)
        return fail(w, LENIA_ERR_INVALID_ARG, "view %d meshes %d fields, the mesher %d", view, view + 1,
                    mesher_fields(m));
    if (mesher_field_floats(m) != (long long)w->C * w->d.N)
        return fail(w, LENIA_ERR_INVALID_ARG, "mesher shape does not match the world");
    // the snapshots, and the arrays their +1 faces copy (transposition.cpp:881-995);
    // a deferred grid snapshot is read where it lies
    const float *rbb = w->rbb_src ? w->rbb_src : w->RBB;
    const float *fields[3] = {rbb, w->U_SUM_RB, w->H_RB};
    const float *halos[3] = {rbb, w->U_SUM, w->H};
    const lenia_status s = lenia_mesher_run(m, fields, halos, w->stream, n_vertices, n_triangles);
    if (s != LENIA_OK) return fail(w, s, "mesh: %s", lenia_mesher_last_error(m));
    return LENIA_OK;
}

lenia_status lenia_world_stats(lenia_world *w, float fill_threshold, double *out)
{
    if (!w || !out) return LENIA_ERR_INVALID_ARG;
    double *dev = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&dev, sizeof(double) * w->C * kStats, w->stream);
    if (e != cudaSuccess) return cuda_fail(w, e, "statistics");
    lenia_status s = world_stats_async(w, fill_threshold, dev);
    if (s == LENIA_OK) {
        e = cudaMemcpyAsync(out, dev, sizeof(double) * w->C * kStats, cudaMemcpyDeviceToHost, w->stream);
        if (e == cudaSuccess) e = cudaFreeAsync(dev, w->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
        if (e != cudaSuccess) s = cuda_fail(w, e, "statistics");
    } else {
        cudaFreeAsync(dev, w->stream);
    }
    return s;
}

const char *lenia_kernel_name(int kid) { return kid >= 0 && kid < KID_MAX ? kKernelNames[kid] : nullptr; }

int lenia_launches_per_step(const lenia_world *w) { return w ? w->launches : 0; }

const char *lenia_last_error(const lenia_world *w) { return w ? w->err.c_str() : "null world"; }

}  // extern "C"

// ---------------------------------------------------------------- batches
//
// Many independent worlds stepped together.  Each world keeps only what
// lives from step to step (A, V, GA, SUM, its kernel spectra and growth-table
// rows); the buffers a step produces and consumes (H, U_SUM, BACK, MU, U_S,
// SUM_S, F, ALPHA and the half spectra) belong to a lane, a stream whose
// worlds run one after another.  Lanes run concurrently.  One step of every
// world is captured into a CUDA graph once and replayed: two graphs, since a
// step swaps each world's A and A_next.  Every world runs the single-world
// code above, so its fields are bit-identical to a world stepped alone.

struct BatchLane {
    cudaStream_t stream = nullptr;
    cudaEvent_t join = nullptr;
    WorldScratch sc = {};
    std::vector<int> worlds;
};

// Worlds stepped by the batched launches (one launch per stage and grid size
// over all worlds of a wave, see capture_grouped): a wave is a set of worlds
// whose per-step buffers fit the shared scratch pool at once; waves run one
// after another and reuse the pool.
struct GroupSize {                 // the jobs of one grid size in a wave
    int W = 0;
    const float2 *tw_x_fwd = nullptr, *tw_x_inv = nullptr, *tw_y_fwd = nullptr, *tw_y_inv = nullptr;
    RowPairJob *fwd = nullptr;     // forward rows of the current grid (per parity)
    int n_fwd = 0;
    PlaneJob *planes_fwd = nullptr, *planes_inv = nullptr;
    int n_planes_fwd = 0, n_planes_inv = 0;
    InvPairJob *inv = nullptr;
    int n_inv = 0;
};
struct GroupWave {
    std::vector<int> worlds;
    std::vector<GroupSize> sizes;
    BatchWorldDev *ws = nullptr;   // world table
    WorkItem *growth = nullptr, *flow = nullptr, *rt[4] = {}, *adv = nullptr;  // rt: [torus * 2 + clip1]
    int n_growth = 0, n_flow = 0, n_rt[4] = {}, n_adv = 0;
};
struct GroupPlan {                 // per step parity (the grid and its double buffer swap)
    std::vector<GroupWave> waves;
    std::vector<void *> allocs;    // device tables of this plan
    int launches = 0;
};

struct lenia_batch {
    std::vector<lenia_world *> worlds;
    std::vector<BatchLane> lanes;
    cudaStream_t stream = nullptr;  // graph launches, field copies
    cudaStream_t own_stream = nullptr;
    cudaEvent_t fork = nullptr;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    int parity = 0;
    std::string err;
    // batched launches
    std::vector<char> grouped;      // per world: stepped by the batched launches
    GroupPlan plan[2];
    unsigned char *pool = nullptr;  // shared per-step scratch of a wave
    size_t pool_bytes = 0;
    cudaStream_t group_stream = nullptr;
    cudaEvent_t group_join = nullptr;
    int lane_launches[2] = {0, 0};
    bool group_on = true;           // lenia_batch_set_batched_launches
};

namespace {

lenia_status bfail(lenia_batch *b, lenia_status s, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (b) b->err = buf;
    return s;
}

void free_plan(GroupPlan &p)
{
    for (void *q : p.allocs)
        if (q) cudaFree(q);
    p = GroupPlan();
}

void free_batch(lenia_batch *b)
{
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (cudaGraphExec_t &g : b->exec)
        if (g) cudaGraphExecDestroy(g);
    if (b->group_stream) cudaStreamSynchronize(b->group_stream);
    for (GroupPlan &p : b->plan) free_plan(p);
    if (b->pool) cudaFree(b->pool);
    if (b->group_join) cudaEventDestroy(b->group_join);
    if (b->group_stream) cudaStreamDestroy(b->group_stream);
    for (lenia_world *w : b->worlds) {
        free_world(w);
        delete w;
    }
    for (BatchLane &l : b->lanes) {
        if (l.stream) cudaStreamSynchronize(l.stream);
        void *sc[] = {l.sc.H, l.sc.U_SUM, l.sc.BACK, l.sc.MU, l.sc.F, l.sc.ALPHA, l.sc.U_S, l.sc.SUM_S, l.sc.XS, l.sc.S};
        for (void *p : sc)
            if (p) cudaFree(p);
        if (l.join) cudaEventDestroy(l.join);
        if (l.stream) cudaStreamDestroy(l.stream);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
}

// One step of a world on its current stream (lenia_step without snapshots).
lenia_status step_once(lenia_world *w)
{
    lenia_status s;
    w->launches = 0;
    if ((s = stage_growth(w)) != LENIA_OK) return s;
    if ((s = stage_blur(w)) != LENIA_OK) return s;
    if ((s = stage_flow(w)) != LENIA_OK) return s;
    return stage_transport(w);
}

// ---- batched launches ---------------------------------------------------
//
// Worlds that take the batched launches: cubic grids of a size with
// one-block-per-plane transforms (24 .. 96), the FFT convolution (stepped in
// its split form, inverse rows storing u_k then the growth from u_k: the
// same bits as the fused form), no debug outputs, snapshots, mass
// conservation, blur, F or ALPHA, and a transport that is the tiled gather
// with dd = 1 or the per-cell kernel.  Per wave and stage one launch per
// grid size (transforms) or one launch over all the wave's worlds (growth
// from u_k, flow, transport), each block working on one block of one world
// through a device work list.

// Per-step buffers of one wave: at most 48 GB, and at most a third of the
// device memory that is free or already held by the batch's pool when the
// plan is built (the pool is allocated once and reused by every wave).
constexpr size_t kWaveScratchMax = 48ull << 30;

size_t wave_scratch_budget(size_t held)
{
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return held > (4ull << 30) ? held : (4ull << 30);
    }
    const size_t third = (free_b + held) / 3;
    const size_t budget = third < kWaveScratchMax ? third : kWaveScratchMax;
    return budget > held ? budget : held;
}

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

bool group_eligible(const lenia_world *w)
{
    const LeniaWorldDesc &s = w->desc;
    if (w->d.W != w->d.H || !list_size_supported(w->d.W)) return false;
    if (w->conv_mode != LENIA_CONV_FFT || w->K < 1 || w->C < 1) return false;
    if (w->debug || w->snapshots || s.conserve_mass) return false;
    if (s.gradient_mode == LENIA_GRADIENT_CENTRAL_DIFF && s.blur_central_diff) return false;
    if (needs_F(s) || s.osc_div_flow) return false;
    return transport_form(step_params(w)) != 2;
}

// The per-step buffers of a world in a wave: H, U_SUM, BACK, MU, u_k, the
// channels' half spectra and the kernels' inverse half spectra.
size_t group_scratch_bytes(const lenia_world *w)
{
    const size_t N = (size_t)w->d.N, CN = (size_t)w->C * N, HS = (size_t)w->d.HS;
    return 3 * align256(CN * 4) + align256(3 * CN * 4) + align256((size_t)w->K * N * 4) +
           align256((size_t)w->C * HS * 8) + align256((size_t)w->K * HS * 8);
}

template <typename T>
T *plan_copy(GroupPlan &plan, const std::vector<T> &v, cudaError_t &e)
{
    if (e != cudaSuccess || v.empty()) return nullptr;
    T *p = nullptr;
    e = cudaMalloc((void **)&p, sizeof(T) * v.size());
    if (e != cudaSuccess) return nullptr;
    plan.allocs.push_back(p);
    e = cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
    return p;
}

// Builds the batched launches' tables for the worlds' current grids (the
// step of graph `which`): waves, the scratch pool, world tables, job lists
// and work items.
lenia_status build_plan(lenia_batch *b, int which)
{
    GroupPlan &plan = b->plan[which];
    free_plan(plan);
    const int n = (int)b->worlds.size();
    b->grouped.assign(n, 0);
    std::vector<int> ids;
    for (int i = 0; i < n && b->group_on; i++)
        if (group_eligible(b->worlds[i])) ids.push_back(i);
    std::stable_sort(ids.begin(), ids.end(), [&](int a, int c) { return b->worlds[a]->d.N > b->worlds[c]->d.N; });
    size_t used = 0, need = 0;
    const size_t budget = wave_scratch_budget(b->pool_bytes);
    for (int i : ids) {
        const size_t sb = group_scratch_bytes(b->worlds[i]);
        if (plan.waves.empty() || (used + sb > budget && !plan.waves.back().worlds.empty())) {
            plan.waves.emplace_back();
            used = 0;
        }
        plan.waves.back().worlds.push_back(i);
        used += sb;
        need = std::max(need, used);
    }
    cudaError_t e = cudaSuccess;
    if (need > b->pool_bytes) {
        if (b->pool) cudaFree(b->pool);
        b->pool = nullptr;
        b->pool_bytes = 0;
        e = cudaMalloc((void **)&b->pool, need);
        if (e != cudaSuccess) return bfail(b, LENIA_ERR_OOM, "batched launches: scratch pool of %zu bytes", need);
        b->pool_bytes = need;
    }
    for (GroupWave &wv : plan.waves) {
        std::vector<BatchWorldDev> table(wv.worlds.size());
        std::vector<WorkItem> growth, flow, rt[4], adv;
        struct SizeJobs {
            std::vector<RowPairJob> fwd;
            std::vector<PlaneJob> pf, pi;
            std::vector<InvPairJob> inv;
        };
        std::vector<int> sizes;
        std::vector<SizeJobs> jobs;
        unsigned char *base = b->pool;
        for (size_t j = 0; j < wv.worlds.size() && e == cudaSuccess; j++) {
            lenia_world *w = b->worlds[wv.worlds[j]];
            const Dims &d = w->d;
            const size_t N = (size_t)d.N, CN = (size_t)w->C * N, HS = (size_t)d.HS;
            auto take = [&](size_t bytes) {
                unsigned char *q = base;
                base += align256(bytes);
                return q;
            };
            float *H = (float *)take(CN * 4), *U_SUM = (float *)take(CN * 4), *BACK = (float *)take(CN * 4);
            float *MU = (float *)take(3 * CN * 4), *U = (float *)take((size_t)w->K * N * 4);
            float2 *XS = (float2 *)take((size_t)w->C * HS * 8), *S = (float2 *)take((size_t)w->K * HS * 8);
            BatchWorldDev &t = table[j];
            memset((void *)&t, 0, sizeof(t));
            t.p = step_params(w);
            t.fb = flow_buffers(w);
            t.fb.H = H;
            t.fb.MU = MU;
            t.tb = transport_buffers(w);
            if (t.tb.ARR == w->BACK) t.tb.ARR = BACK;
            t.tb.MU = MU;
            t.tb.H = H;
            t.tb.BACK = BACK;
            t.gj = growth_jobs(w);
            for (int k = 0; k < w->K; k++) t.gj.spec[k] = S + (size_t)k * HS;
            t.ord = channel_order(t.gj);
            t.lut_rows = w->lut_rows;
            t.U = U;
            t.A = w->A;
            t.H = H;
            t.U_SUM = U_SUM;
            t.BACK = BACK;
            t.err = w->err_flag;
            const int wj = (int)j;
            e = flow_tensor_maps(t.p, t.fb, &t.tm_sum, &t.tm_h);
            const int nf = flow_blocks(d, &t.flow_gx);
            for (int blk = 0; blk < nf; blk++) flow.push_back({wj, blk});
            for (int blk = 0, ng = growth_from_u_blocks(d); blk < ng; blk++) growth.push_back({wj, blk});
            if (transport_form(t.p) == 1) {
                if (e == cudaSuccess) e = transport_tensor_maps(t.p, t.tb, 1, &t.tm_mu, &t.tm_arr);
                const int nt = transport_rt_blocks(d, &t.transport_gx);
                const int v = (t.p.border == kBorderTorus ? 2 : 0) + (t.p.clip == 1.0f ? 1 : 0);
                for (int blk = 0; blk < nt; blk++) rt[v].push_back({wj, blk});
            } else {
                for (int blk = 0, nt = transport_adv_blocks(d); blk < nt; blk++) adv.push_back({wj, blk});
            }
            // the transforms, paired as a single world's launches pair them
            const size_t si = std::find(sizes.begin(), sizes.end(), d.W) - sizes.begin();
            if (si == sizes.size()) {
                sizes.push_back(d.W);
                jobs.emplace_back();
                GroupSize g;
                g.W = d.W;
                g.tw_x_fwd = w->tw_x_fwd;
                g.tw_x_inv = w->tw_x_inv;
                g.tw_y_fwd = w->tw_y_fwd;
                g.tw_y_inv = w->tw_y_inv;
                wv.sizes.push_back(g);
            }
            SizeJobs &sj = jobs[si];
            for (int c = 0; c < w->C; c += 2) {
                RowPairJob r;
                r.in[0] = w->A + (size_t)c * N;
                r.out[0] = XS + (size_t)c * HS;
                r.in[1] = c + 1 < w->C ? w->A + (size_t)(c + 1) * N : nullptr;
                r.out[1] = c + 1 < w->C ? XS + (size_t)(c + 1) * HS : nullptr;
                sj.fwd.push_back(r);
            }
            for (int c = 0; c < w->C; c++) sj.pf.push_back({XS + (size_t)c * HS, XS + (size_t)c * HS, nullptr});
            const size_t kh = (size_t)d.KX * (d.D / 2 + 1) * (d.H / 2 + 1);
            for (int k = 0; k < w->K; k++)
                sj.pi.push_back({XS + (size_t)w->kernels[k].c0 * HS, S + (size_t)k * HS, w->Kc + k * kh});
            for (int k = 0; k < w->K; k += 2) {
                InvPairJob q;
                q.spec[0] = S + (size_t)k * HS;
                q.out[0] = U + (size_t)k * N;
                q.spec[1] = k + 1 < w->K ? S + (size_t)(k + 1) * HS : nullptr;
                q.out[1] = k + 1 < w->K ? U + (size_t)(k + 1) * N : nullptr;
                sj.inv.push_back(q);
            }
        }
        wv.ws = plan_copy(plan, table, e);
        wv.growth = plan_copy(plan, growth, e);
        wv.n_growth = (int)growth.size();
        wv.flow = plan_copy(plan, flow, e);
        wv.n_flow = (int)flow.size();
        for (int v = 0; v < 4; v++) {
            wv.rt[v] = plan_copy(plan, rt[v], e);
            wv.n_rt[v] = (int)rt[v].size();
            plan.launches += wv.n_rt[v] > 0;
        }
        wv.adv = plan_copy(plan, adv, e);
        wv.n_adv = (int)adv.size();
        plan.launches += 2 + (wv.n_adv > 0);
        for (size_t si = 0; si < sizes.size(); si++) {
            GroupSize &g = wv.sizes[si];
            g.fwd = plan_copy(plan, jobs[si].fwd, e);
            g.n_fwd = (int)jobs[si].fwd.size();
            g.planes_fwd = plan_copy(plan, jobs[si].pf, e);
            g.n_planes_fwd = (int)jobs[si].pf.size();
            g.planes_inv = plan_copy(plan, jobs[si].pi, e);
            g.n_planes_inv = (int)jobs[si].pi.size();
            g.inv = plan_copy(plan, jobs[si].inv, e);
            g.n_inv = (int)jobs[si].inv.size();
            // each job list runs in launches of at most 65535 jobs (grid.y)
            for (const int n : {g.n_fwd, g.n_planes_fwd, g.n_planes_inv, g.n_inv}) plan.launches += (n + 65534) / 65535;
        }
        if (e != cudaSuccess) break;
    }
    if (e != cudaSuccess) {
        free_plan(plan);
        b->grouped.assign(n, 0);
        return bfail(b, e == cudaErrorMemoryAllocation ? LENIA_ERR_OOM : LENIA_ERR_CUDA, "batched launches: %s",
                     cudaGetErrorString(e));
    }
    for (int i : ids) b->grouped[i] = 1;
    return LENIA_OK;
}

// The batched launches of one step on stream st.
cudaError_t launch_plan(const GroupPlan &plan, cudaStream_t st)
{
    cudaError_t e = cudaSuccess;
    for (const GroupWave &wv : plan.waves) {
        for (const GroupSize &g : wv.sizes)
            if (e == cudaSuccess) e = launch_fwd_rows_list(g.W, g.tw_x_fwd, RowPairList{g.fwd, g.n_fwd}, st);
        for (const GroupSize &g : wv.sizes)
            if (e == cudaSuccess)
                e = launch_planes_list(g.W, g.tw_y_fwd, g.tw_x_fwd, PlaneJobList{g.planes_fwd, g.n_planes_fwd}, -1, st);
        for (const GroupSize &g : wv.sizes)
            if (e == cudaSuccess)
                e = launch_planes_list(g.W, g.tw_y_inv, g.tw_x_inv, PlaneJobList{g.planes_inv, g.n_planes_inv}, +1, st);
        for (const GroupSize &g : wv.sizes)
            if (e == cudaSuccess) e = launch_inv_rows_list(g.W, g.tw_x_inv, InvPairList{g.inv, g.n_inv}, st);
        if (e == cudaSuccess) e = launch_growth_from_u_multi(wv.ws, wv.growth, wv.n_growth, st);
        if (e == cudaSuccess) e = launch_flow_multi(wv.ws, wv.flow, wv.n_flow, st);
        for (int v = 0; v < 4; v++)
            if (e == cudaSuccess) e = launch_transport_rt_multi(wv.ws, wv.rt[v], wv.n_rt[v], v >= 2, v & 1, st);
        if (e == cudaSuccess) e = launch_transport_adv_multi(wv.ws, wv.adv, wv.n_adv, st);
    }
    return e;
}

// Captures one step of every world, lanes forked from and joined to the
// batch stream, into exec[which]; worlds that take the batched launches run
// on the group stream beside the lanes.
lenia_status capture_step(lenia_batch *b, int which)
{
    lenia_status s = build_plan(b, which);
    if (s != LENIA_OK) return s;
    // captured on the batch's own stream (the caller's stream, which the
    // graph is launched on, may be one that cannot be captured)
    cudaStream_t cs = b->own_stream;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return bfail(b, LENIA_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e));
    e = cudaEventRecord(b->fork, cs);
    int lane_launches = 0;
    if (e == cudaSuccess && !b->plan[which].waves.empty()) {
        e = cudaStreamWaitEvent(b->group_stream, b->fork, 0);
        if (e == cudaSuccess) e = launch_plan(b->plan[which], b->group_stream);
        if (e == cudaSuccess) e = cudaEventRecord(b->group_join, b->group_stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, b->group_join, 0);
    }
    for (size_t l = 0; l < b->lanes.size() && e == cudaSuccess && s == LENIA_OK; l++) {
        BatchLane &lane = b->lanes[l];
        e = cudaStreamWaitEvent(lane.stream, b->fork, 0);
        for (int i : lane.worlds) {
            if (e != cudaSuccess || s != LENIA_OK) break;
            if (b->grouped[i]) continue;
            lenia_world *w = b->worlds[i];
            w->stream = lane.stream;
            s = step_once(w);
            lane_launches += w->launches;
            if (s != LENIA_OK) b->err = "world " + std::to_string(i) + ": " + w->err;
        }
        if (e == cudaSuccess) e = cudaEventRecord(lane.join, lane.stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, lane.join, 0);
    }
    b->lane_launches[which] = lane_launches;
    // the batched launches wrote the worlds' next grids
    for (size_t i = 0; i < b->worlds.size(); i++)
        if (b->grouped[i]) std::swap(b->worlds[i]->A, b->worlds[i]->A_next);

    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
    for (lenia_world *w : b->worlds) w->stream = b->stream;
    if (s != LENIA_OK) {
        if (graph) cudaGraphDestroy(graph);
        return s;
    }
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec[which], graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) return bfail(b, LENIA_ERR_CUDA, "capturing the batch step: %s", cudaGetErrorString(e));
    return LENIA_OK;
}

bool batch_field_ok(int field)
{
    return field == LENIA_FIELD_A || field == LENIA_FIELD_V || field == LENIA_FIELD_GA || field == LENIA_FIELD_SUM;
}

}  // namespace

extern "C" {

lenia_status lenia_batch_create(const LeniaWorldDesc *descs, const LeniaKernelParams *kernels,
                                const int *kernel_counts, int n_worlds, int lanes, lenia_batch **out)
{
    if (!descs || !kernel_counts || !out || n_worlds < 1 || lanes < 0) return LENIA_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return LENIA_ERR_NO_DEVICE;
    }
    for (int i = 0; i < n_worlds; i++) {
        const LeniaWorldDesc &d = descs[i];
        if (d.width < 8 || d.width > 256 || d.height < 8 || d.height > 256 || d.channels < 1 ||
            d.channels > LENIA_MAX_CHANNELS || kernel_counts[i] < 0 || kernel_counts[i] > LENIA_MAX_KERNELS)
            return LENIA_ERR_INVALID_ARG;
    }
    lenia_batch *b = new lenia_batch();
    const int L = std::max(1, std::min(lanes == 0 ? 64 : lanes, n_worlds));
    b->lanes.resize(L);
    // longest processing time first: the largest world to the lightest lane
    std::vector<int> order(n_worlds);
    for (int i = 0; i < n_worlds; i++) order[i] = i;
    auto cells = [&](int i) {
        return (long long)descs[i].width * descs[i].height * descs[i].width * descs[i].channels *
               (1 + kernel_counts[i]);
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return cells(a) > cells(c); });
    std::vector<long long> load(L, 0);
    for (int i : order) {
        const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        b->lanes[l].worlds.push_back(i);
        load[l] += cells(i);
    }
    std::vector<size_t> koff(n_worlds + 1, 0);
    for (int i = 0; i < n_worlds; i++) koff[i + 1] = koff[i] + kernel_counts[i];
    b->worlds.assign(n_worlds, nullptr);
    cudaError_t e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking);
    b->stream = b->own_stream;
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->group_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->group_join, cudaEventDisableTiming);
    lenia_status s = LENIA_OK;
    for (BatchLane &lane : b->lanes) {
        if (e != cudaSuccess || s != LENIA_OK) break;
        std::sort(lane.worlds.begin(), lane.worlds.end());
        e = cudaStreamCreateWithFlags(&lane.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&lane.join, cudaEventDisableTiming);
        // scratch sized for the lane's largest needs
        size_t cn = 0, n = 0, xs = 0, sk = 0;
        bool need_f = false, need_alpha = false;
        for (int i : lane.worlds) {
            const LeniaWorldDesc &d = descs[i];
            const size_t N = (size_t)d.width * d.height * d.width;
            const size_t hs = (size_t)(d.width / 2 + 1) * d.width * d.height;
            cn = std::max(cn, (size_t)d.channels * N);
            n = std::max(n, N);
            xs = std::max(xs, (size_t)(d.channels + 1) * hs);
            sk = std::max(sk, (size_t)std::max(kernel_counts[i], d.channels + 1) * hs);
            need_f = need_f || needs_F(d);
            need_alpha = need_alpha || d.osc_div_flow;
        }
        WorldScratch &sc = lane.sc;
        sc.H = dalloc<float>(cn, e);
        sc.U_SUM = dalloc<float>(cn, e);
        sc.BACK = dalloc<float>(cn, e);
        sc.MU = dalloc<float>(3 * cn, e);
        sc.U_S = dalloc<float>(cn, e);
        sc.SUM_S = dalloc<float>(n, e);
        sc.F = need_f ? dalloc<float>(3 * cn, e) : nullptr;
        sc.ALPHA = need_alpha ? dalloc<float>(cn, e) : nullptr;
        sc.XS = dalloc<float2>(xs, e);
        sc.S = dalloc<float2>(sk, e);
        for (int i : lane.worlds) {
            if (e != cudaSuccess || s != LENIA_OK) break;
            s = create_world(&descs[i], kernels ? kernels + koff[i] : nullptr, kernel_counts[i], &sc, lane.stream,
                             &b->worlds[i]);
            if (s != LENIA_OK) bfail(b, s, "world %d could not be created", i);
        }
    }
    if (e == cudaSuccess && s == LENIA_OK) {
        for (BatchLane &lane : b->lanes)
            if (e == cudaSuccess) e = cudaStreamSynchronize(lane.stream);
        for (lenia_world *w : b->worlds) w->stream = b->stream;
    }
    if (e != cudaSuccess && s == LENIA_OK) s = e == cudaErrorMemoryAllocation ? LENIA_ERR_OOM : LENIA_ERR_CUDA;
    if (s == LENIA_OK) s = capture_step(b, 0);
    if (s == LENIA_OK) s = capture_step(b, 1);
    if (s != LENIA_OK) {
        fprintf(stderr, "lenia_batch_create: %s\n", b->err.empty() ? cudaGetErrorString(e) : b->err.c_str());
        b->worlds.erase(std::remove(b->worlds.begin(), b->worlds.end(), nullptr), b->worlds.end());
        free_batch(b);
        delete b;
        return s;
    }
    *out = b;
    return LENIA_OK;
}

lenia_status lenia_batch_destroy(lenia_batch *b)
{
    if (!b) return LENIA_ERR_INVALID_ARG;
    free_batch(b);
    delete b;
    return LENIA_OK;
}

int lenia_batch_size(const lenia_batch *b) { return b ? (int)b->worlds.size() : 0; }

lenia_status lenia_batch_set_stream(lenia_batch *b, void *stream)
{
    if (!b) return LENIA_ERR_INVALID_ARG;
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return bfail(b, LENIA_ERR_CUDA, "set_stream: %s", cudaGetErrorString(e));
    b->stream = (cudaStream_t)stream;
    for (lenia_world *w : b->worlds) w->stream = b->stream;
    return LENIA_OK;
}

lenia_status lenia_batch_set_field(lenia_batch *b, int world, int field, const float *src, size_t count, int on_device)
{
    if (!b || world < 0 || world >= (int)b->worlds.size()) return LENIA_ERR_INVALID_ARG;
    if (!batch_field_ok(field)) return bfail(b, LENIA_ERR_INVALID_ARG, "a batch world keeps only A, V, GA and SUM");
    const lenia_status s = lenia_set_field(b->worlds[world], field, src, count, on_device);
    if (s != LENIA_OK) b->err = b->worlds[world]->err;
    return s;
}

lenia_status lenia_batch_get_field(lenia_batch *b, int world, int field, float *dst, size_t count, int on_device)
{
    if (!b || world < 0 || world >= (int)b->worlds.size()) return LENIA_ERR_INVALID_ARG;
    if (!batch_field_ok(field)) return bfail(b, LENIA_ERR_INVALID_ARG, "a batch world keeps only A, V, GA and SUM");
    const lenia_status s = lenia_get_field(b->worlds[world], field, dst, count, on_device);
    if (s != LENIA_OK) b->err = b->worlds[world]->err;
    return s;
}

lenia_status lenia_batch_step(lenia_batch *b, int n_steps)
{
    if (!b || n_steps < 0) return LENIA_ERR_INVALID_ARG;
    NvtxRange range("lenia_batch_step");
    for (int i = 0; i < n_steps; i++) {
        const cudaError_t e = cudaGraphLaunch(b->exec[b->parity], b->stream);
        if (e != cudaSuccess) return bfail(b, LENIA_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e));
        for (lenia_world *w : b->worlds) std::swap(w->A, w->A_next);
        b->parity ^= 1;
    }
    return LENIA_OK;
}

lenia_status lenia_batch_sync(lenia_batch *b)
{
    if (!b) return LENIA_ERR_INVALID_ARG;
    for (size_t i = 0; i < b->worlds.size(); i++) {
        const lenia_status s = lenia_sync(b->worlds[i]);
        if (s != LENIA_OK) return bfail(b, s, "world %zu: %s", i, b->worlds[i]->err.c_str());
    }
    return LENIA_OK;
}

// Per grid shape (width, height): lenia_autotune on the first world of that
// shape, its choice applied to every world of the shape; then both step
// graphs are captured again.
lenia_status lenia_batch_autotune(lenia_batch *b, int modes, LeniaTuneResult *per_world)
{
    if (!b) return LENIA_ERR_INVALID_ARG;
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return bfail(b, LENIA_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
    std::vector<int> done(b->worlds.size(), 0);
    for (size_t i = 0; i < b->worlds.size(); i++) {
        if (done[i]) continue;
        lenia_world *rep = b->worlds[i];
        LeniaTuneResult r;
        lenia_status s = lenia_autotune(rep, modes, &r);
        if (s != LENIA_OK) return bfail(b, s, "world %zu: %s", i, rep->err.c_str());
        for (size_t j = i; j < b->worlds.size(); j++) {
            lenia_world *w = b->worlds[j];
            if (done[j] || w->d.W != rep->d.W || w->d.H != rep->d.H) continue;
            done[j] = 1;
            w->d.ty = r.row_tile;
            if (r.growth_split && !w->U && w->K > 0) {
                cudaError_t ea = cudaSuccess;
                w->U = dalloc<float>((size_t)w->K * w->d.N, ea);
                if (ea != cudaSuccess) return bfail(b, LENIA_ERR_OOM, "world %zu: u_k buffer", j);
            }
            w->growth_split = r.growth_split;
            if (w->conv_mode != r.conv_mode) {
                w->conv_mode = r.conv_mode;
                if ((s = build_kernels(w)) != LENIA_OK) return bfail(b, s, "world %zu: %s", j, w->err.c_str());
            }
            w->stream = b->stream;
            if (per_world) per_world[j] = r;
        }
    }
    for (cudaGraphExec_t &g : b->exec)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    // the worlds' host pointers hold the current grid: the graph of the
    // current parity is captured first (each capture swaps A and A_next)
    lenia_status s = capture_step(b, b->parity);
    if (s == LENIA_OK) s = capture_step(b, b->parity ^ 1);
    return s;
}

lenia_status lenia_batch_stats(lenia_batch *b, float fill_threshold, double *out)
{
    if (!b || !out) return LENIA_ERR_INVALID_ARG;
    size_t total = 0;
    for (const lenia_world *w : b->worlds) total += (size_t)w->C * kStats;
    double *dev = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&dev, sizeof(double) * total, b->stream);
    if (e != cudaSuccess) return bfail(b, LENIA_ERR_CUDA, "statistics: %s", cudaGetErrorString(e));
    size_t off = 0;
    for (size_t i = 0; i < b->worlds.size(); i++) {
        lenia_world *w = b->worlds[i];
        const lenia_status s = world_stats_async(w, fill_threshold, dev + off);
        if (s != LENIA_OK) {
            cudaFreeAsync(dev, b->stream);
            return bfail(b, s, "world %zu: %s", i, w->err.c_str());
        }
        off += (size_t)w->C * kStats;
    }
    e = cudaMemcpyAsync(out, dev, sizeof(double) * total, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaFreeAsync(dev, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return bfail(b, LENIA_ERR_CUDA, "statistics: %s", cudaGetErrorString(e));
    return LENIA_OK;
}

lenia_status lenia_batch_set_batched_launches(lenia_batch *b, int on)
{
    if (!b) return LENIA_ERR_INVALID_ARG;
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return bfail(b, LENIA_ERR_CUDA, "set_batched_launches: %s", cudaGetErrorString(e));
    b->group_on = on != 0;
    for (cudaGraphExec_t &g : b->exec)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    lenia_status s = capture_step(b, b->parity);
    if (s == LENIA_OK) s = capture_step(b, b->parity ^ 1);
    return s;
}

int lenia_batch_grouped_worlds(const lenia_batch *b)
{
    if (!b) return 0;
    int n = 0;
    for (char g : b->grouped) n += g != 0;
    return n;
}

int lenia_batch_launches_per_step(const lenia_batch *b)
{
    if (!b) return 0;
    return b->lane_launches[b->parity] + b->plan[b->parity].launches;
}

const char *lenia_batch_last_error(const lenia_batch *b) { return b ? b->err.c_str() : "null batch"; }

}  // extern "C"
