// Internal declarations shared by the host code (lenia_api.cu) and the CUDA
// kernels of the 3D Flow Lenia step.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/lenia_b200.h"
#include "lfft_device.cuh"

namespace lenia {

constexpr int kMaxKernels = 64;
constexpr int kMaxChannels = 4;
constexpr int kMaxPairs = 40;       // packed real-field pairs in one forward launch
constexpr int kPlaneThreads = 512;  // block size of the plane transform
constexpr int kPlaneCap = 32;       // values per thread in the plane transform
constexpr int kRowThreads = 256;    // block size of the row transforms
constexpr int kRowCap = 32;
// default poll limit of the first wait for a tile copy (StepParams::wait_polls)
constexpr unsigned kDefaultTileWaitPolls = 1u << 24;

enum { kBorderTorus = 0, kBorderWall = 1, kBorderNone = 2 };
enum { kGrowthNone = 0, kGrowthRT = 1, kGrowthTransposition = 2 };
enum { kModeSRT = 0, kModeRT = 1, kModeADV = 2 };
enum { kGradCentralDiff = 0, kGradSobel = 1 };

struct Dims {
    int W, H, D;  // x, y, z extents (D == W)
    long long N;  // cells
    int KX;       // W/2 + 1
    long long HS; // KX * D * H complex entries of a half spectrum
    long long P;  // (W+8)(H+8)(W+8): the reference's padded block (Q20)
    int ty = 0;   // row tile of the runtime-sized row transforms (0: the largest that fits)
};

// Forward row pass: up to kMaxPairs pairs of real fields -> half spectra.
struct FwdRowJobs {
    const float *in[2 * kMaxPairs];
    float2 *out[2 * kMaxPairs];
    int npairs;
};

// Plane pass: one job per (array); a job transforms every kx plane of it.
struct PlaneJobs {
    const float2 *src[kMaxKernels + 8];
    float2 *dst[kMaxKernels + 8];
    const float *kc[kMaxKernels + 8];  // octant kernel spectrum, or null
    int njobs;
};

// Inverse row pass with the growth epilogue.
struct GrowthJobs {
    const float2 *spec[kMaxKernels];
    int c1[kMaxKernels];
    float h[kMaxKernels];
    int lut_base[kMaxKernels];
    int K;
    int C;
    int asymptotic[kMaxChannels];
    int soft_clip[kMaxChannels];
    int growth_rt;  // write BACK
    float timestep;
    int exact_bell;            // growth = bell(u, m, s) instead of the table entry
    float m[kMaxKernels];      // growth centre and width per kernel (exact_bell)
    float s[kMaxKernels];
};

// Inverse row pass storing field/N (the blur, and u_k of the split growth).
constexpr int kBlurFields = 16;  // >= 2 * kMaxChannels + 2, the blur's fields
struct BlurJobs {
    const float2 *spec[kBlurFields];
    float *out[kBlurFields];
    int nfields;
};

// Everything the flow and transport kernels read, by value.
struct StepParams {
    Dims d;
    int C;
    float timestep, theta_a, s_norm, gta, sta, v_damp, sigma, dd_f;
    int dd;
    int growth_type, mode_type, sobel_border, border, gradient_mode;
    int adv_vel, mu_vel, blur;
    int osc_la, osc_flow, osc_div_flow, osc_vel;
    float osc_la_amt, osc_flow_amt, osc_div_flow_amt;
    int asymptotic[kMaxChannels], soft_clip[kMaxChannels];
    int rt_all_channels, alpha_index_fix;
    // derived (computed on the host in the reference's float expressions)
    float ma, sn, clip, si, gws, ghs;
    // 1 / theta_a when theta_a is a power of two whose reciprocal is a
    // normal float (then a / theta_a == a * inv_theta_a for every a: both are
    // the correctly rounded value of the same real number), else 0
    float inv_theta_a;
    // poll limit of the first wait for each tile copy in the flow and
    // transport kernels (lenia_set_wait_limit); a block whose wait runs out
    // records the timeout, drains its copies in flight and returns
    unsigned wait_polls;
};

struct FlowBuffers {
    const float *H;      // H (Sobel) or U_S (central difference), C*N
    const float *SUM;    // SUM (Sobel) or SUM_S, N
    const float *A;      // C*N
    const float *GA;     // C*N (ALPHA only)
    float *V;            // 3*C*N, updated in place
    float *MU;           // 3*C*N
    float *F;            // 3*C*N or null
    float *ALPHA;        // C*N or null
    float *NA, *NU, *PREALPHA;  // debug outputs or null (PREALPHA: 4*N flat)
    int *err;            // bit 2 set when a tile copy did not complete in time
};

struct TransportBuffers {
    const float *A;      // current grid, C*N
    float *A_out;        // new grid, C*N
    const float *ARR;    // GRID or BACK, C*N
    const float *MU;     // 3*C*N
    const float *H;      // C*N (growth by transposition)
    const float *V;      // 3*C*N (advection, oscillators)
    const float *F;      // 3*C*N or null
    const float *ALPHA;  // C*N or null
    float *GA;           // C*N, updated in place
    float *SUM;          // N
    float *BACK;         // C*N (transposition soft clip)
    float *TT;           // debug: pre-clamp TT, or null
    int *err;            // bit 2 set when a tile copy did not complete in time
};

// ---- batches of worlds as one launch per stage -------------------------
// Job lists in device memory: one launch transforms the fields of many
// worlds of one grid size (each entry is what a single world's launch would
// take; entries of different worlds never share a transform).
struct RowPairJob {       // forward rows: two real fields -> half spectra
    const float *in[2];   // in[1] may be null
    float2 *out[2];
};
struct PlaneJob {         // plane pass of one half spectrum
    const float2 *src;
    float2 *dst;
    const float *kc;      // octant kernel spectrum, or null
};
struct InvPairJob {       // inverse rows: two half spectra -> fields / N
    const float2 *spec[2];  // spec[1] may be null
    float *out[2];
};
struct RowPairList { const RowPairJob *j; int n; };
struct PlaneJobList { const PlaneJob *j; int n; };
struct InvPairList { const InvPairJob *j; int n; };

// The kernels grouped by target channel c1, in kernel order within a group
// (the order of the growth from u_k).
struct ChannelOrder {
    int k[kMaxKernels];
};

// Everything a world's growth-from-u, flow and transport launches take, in
// device memory for the batched launches (tensor maps first: 64-byte aligned).
struct alignas(64) BatchWorldDev {
    CUtensorMap tm_sum, tm_h;    // flow: SUM and H tiles
    CUtensorMap tm_mu, tm_arr;   // transport: MU and ARR tiles
    StepParams p;
    FlowBuffers fb;
    TransportBuffers tb;
    GrowthJobs gj;
    ChannelOrder ord;
    const float *lut_rows, *U, *A;
    float *H, *U_SUM, *BACK;
    int *err;
    int flow_gx;                 // flow blocks along x*y (the launch's x extent for this world)
    int transport_gx;            // transport (tiled) blocks along x*y
};

// One block of a batched launch: world index and the block's index within
// that world's own launch (flattened x fastest).
struct WorkItem {
    int world;
    int block;
};

// Batched launches (kernels_*.cu): grid sizes W < 128 (the one-block-per-plane
// transforms); the job lists, world table and work items live in device memory.
bool list_size_supported(int W);
cudaError_t launch_fwd_rows_list(int W, const float2 *tw_x, RowPairList jobs, cudaStream_t st);
cudaError_t launch_planes_list(int W, const float2 *tw_y, const float2 *tw_z, PlaneJobList jobs, int sign,
                               cudaStream_t st);
cudaError_t launch_inv_rows_list(int W, const float2 *tw_x_inv, InvPairList jobs, cudaStream_t st);
cudaError_t launch_growth_from_u_multi(const BatchWorldDev *ws, const WorkItem *items, int n_items, cudaStream_t st);
cudaError_t launch_flow_multi(const BatchWorldDev *ws, const WorkItem *items, int n_items, cudaStream_t st);
// RT with dd = 1 (the tiled gather) for worlds sharing torus/clip-1 flags; ADV per cell
cudaError_t launch_transport_rt_multi(const BatchWorldDev *ws, const WorkItem *items, int n_items, bool torus,
                                      bool clip1, cudaStream_t st);
cudaError_t launch_transport_adv_multi(const BatchWorldDev *ws, const WorkItem *items, int n_items, cudaStream_t st);
// Tensor maps of a world's flow and tiled-transport launches (for the world
// table of the batched launches); the transport kernel form of a world
// (1: tiled, dd = 1; 2: tiled, dd = 2; 0: per cell).
cudaError_t flow_tensor_maps(const StepParams &p, const FlowBuffers &b, CUtensorMap *tm_sum, CUtensorMap *tm_h);
cudaError_t transport_tensor_maps(const StepParams &p, const TransportBuffers &b, int dd, CUtensorMap *tm_mu,
                                  CUtensorMap *tm_arr);
int transport_form(const StepParams &p);
// Blocks of a world's own launches (the work-item counts of the batched ones).
int flow_blocks(const Dims &d, int *gx);
int transport_rt_blocks(const Dims &d, int *gx);
int transport_adv_blocks(const Dims &d);
int growth_from_u_blocks(const Dims &d);
ChannelOrder channel_order(const GrowthJobs &jobs);

// Programmatic dependent launch between the kernels of a step (forward rows,
// planes, growth, flow, transport): a kernel lets the next one launch once
// all its blocks run (pdl_trigger), and waits for the previous kernel's
// completion and memory (pdl_wait) after its constant set-up and before it
// reads or writes any field.  Without the launch attribute both are no-ops.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Launch wrappers (kernels_*.cu); all are asynchronous on `st`.
cudaError_t launch_fwd_rows(const Dims &d, const FftPlan &px, const float2 *tw_x, const FwdRowJobs &jobs,
                            cudaStream_t st);
cudaError_t launch_planes(const Dims &d, const FftPlan &py, const FftPlan &pz, const float2 *tw_y,
                          const float2 *tw_z, const PlaneJobs &jobs, int sign, cudaStream_t st);
cudaError_t launch_growth_rows(const Dims &d, const FftPlan &px, const float2 *tw_x_inv, const GrowthJobs &jobs,
                               const float *lut_rows, const float *A, float *H, float *U_SUM, float *BACK,
                               float *U_dbg, int *err_flag, cudaStream_t st);
cudaError_t launch_blur_rows(const Dims &d, const FftPlan &px, const float2 *tw_x_inv, const BlurJobs &jobs,
                             cudaStream_t st);
cudaError_t launch_kernel_grids(const Dims &d, const LeniaKernelParams *kp_dev, int K, float *grids,
                                float *ksum, cudaStream_t st);
cudaError_t launch_blur_grid(const Dims &d, float *grid, float *ksum, cudaStream_t st);
cudaError_t launch_compress(const Dims &d, const float2 *spec, float *kc, cudaStream_t st);
cudaError_t launch_lut_rows(const LeniaKernelParams *kp_dev, int K, float *lut_rows, int *lut_base,
                            cudaStream_t st);
cudaError_t launch_flow(const StepParams &p, const FlowBuffers &b, cudaStream_t st);
cudaError_t launch_transport(const StepParams &p, const TransportBuffers &b, cudaStream_t st);

// Size-specialised spectral kernels (kernels_spectral_fast.cu) for cubic
// grids of the sizes they are instantiated for.
bool fast_supported(const Dims &d);
// The size-specialised row transforms (forward rows, growth, blur) also
// serve cubic grids whose planes use the runtime-sized plane passes.
bool fast_rows_supported(const Dims &d);
// Plane transforms of such grids as two line passes with compile-time plans.
bool fast_split_planes_supported(const Dims &d);
cudaError_t launch_planes_split_fast(const Dims &d, const float2 *tw_y, const float2 *tw_z, const PlaneJobs &jobs,
                                     int sign, cudaStream_t st);
cudaError_t launch_fwd_rows_fast(const Dims &d, const float2 *tw_x, const FwdRowJobs &jobs, cudaStream_t st);
cudaError_t launch_planes_fast(const Dims &d, const float2 *tw_y, const float2 *tw_z, const PlaneJobs &jobs, int sign,
                               cudaStream_t st);
cudaError_t launch_growth_rows_fast(const Dims &d, const float2 *tw_x_inv, const GrowthJobs &jobs,
                                    const float *lut_rows, const float *A, float *H, float *U_SUM, float *BACK,
                                    float *U_dbg, int *err_flag, cudaStream_t st);
cudaError_t launch_blur_rows_fast(const Dims &d, const float2 *tw_x_inv, const BlurJobs &jobs, cudaStream_t st);

// Grid statistics for labelling (kernels_stats.cu): per channel kStats
// doubles; trig holds cos, sin of 2 pi x / W (W each) then of 2 pi y / H.
constexpr int kStats = 9;
constexpr int kStatBlocks = 64;
cudaError_t launch_stats(const float *A, const Dims &d, int C, const double *trig, float fill, double *partial,
                         int nblk, double *out, cudaStream_t st);
// Per-channel totals of A in double (fixed summation order) into out[C], and
// the rescaling A_c *= float(target_c / total_c) that restores them.
cudaError_t launch_mass_totals(const float *A, const Dims &d, int C, double *partial, int nblk, double *out,
                               cudaStream_t st);
cudaError_t launch_mass_scale(float *A, const Dims &d, int C, const double *target, const double *total,
                              cudaStream_t st);

// The conserve_mass target totals of a world (lenia_api.cu): copied out to
// `host` (n >= channels; returns the channel count, 0 when none are
// recorded) or replaced from it (n == channels).
int mass_target_get(lenia_world *w, double *host, int n);
lenia_status mass_target_set(lenia_world *w, const double *host, int n);

// Host FFT plans and twiddle tables (lenia_api.cu).
int fft_factor(int n, int *radix);

// Marching-cubes mesher (kernels_mesh.cu): floats of each field it meshes,
// and the number of fields.
long long mesher_field_floats(const lenia_mesher *m);
int mesher_fields(const lenia_mesher *m);

}  // namespace lenia
