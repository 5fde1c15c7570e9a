/*
 * lenia_b200 — C ABI of the B200-native 3D Flow Lenia step.
 *
 * The reference (lostnthought/Lenia) has no library boundary: its step API is
 * a set of `void stage(TD *t)` functions over process-global arrays
 * (lenia.h:5-28, reintegration.h:207-240, transposition.h:4-11, mesh.h:7-9),
 * configured by writing globals (main.cpp:27-66) and driven by a 12-event
 * state machine (render.cpp:357-604).  This header replaces that surface with
 * an opaque world handle: the globals become LeniaWorldDesc, the Kernel struct
 * becomes LeniaKernelParams, the arrays become fields read and written through
 * lenia_get_field / lenia_set_field, and the event sequence becomes
 * lenia_step (whole steps) or lenia_step_stage (one stage group).
 *
 * Plain C types only; all device work runs on one CUDA stream per world.
 * Every entry point returns a lenia_status; lenia_last_error() describes the
 * last failure on a world.  There is no CPU fallback: without a CUDA device
 * lenia_create fails with LENIA_ERR_NO_DEVICE.
 */
#ifndef LENIA_B200_H
#define LENIA_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LENIA_MAX_CHANNELS 4 /* MAX_CHANNELS, render.h:34 */
#define LENIA_MAX_BETA 12    /* MAX_BETA, render.h:35 */
#define LENIA_MAX_KERNELS 64 /* render.h:33 fixes 12; runtime here */

typedef enum lenia_status {
    LENIA_OK = 0,
    LENIA_ERR_INVALID_ARG = 1,
    LENIA_ERR_OOM = 2,
    LENIA_ERR_CUDA = 3,
    LENIA_ERR_TIMEOUT = 4,
    LENIA_ERR_NONFINITE = 5,
    LENIA_ERR_NO_DEVICE = 6,
    LENIA_ERR_UNSUPPORTED = 7
} lenia_status;

/* Enumerations, in the reference's order (render.h:128-223). */
enum { LENIA_GROWTH_NOGROWTH = 0, LENIA_GROWTH_RT = 1, LENIA_GROWTH_TRANSPOSITION = 2 };
enum { LENIA_MODE_SRT = 0, LENIA_MODE_RT = 1, LENIA_MODE_ADV = 2 };
enum { LENIA_BORDER_TORUS = 0, LENIA_BORDER_WALL = 1, LENIA_BORDER_NONE = 2 };
enum { LENIA_GRADIENT_CENTRAL_DIFF = 0, LENIA_GRADIENT_SOBEL = 1 };

/* The reference's scalar and mode globals (main.cpp:27-56, main.cpp:304,
 * render.h:125-233) plus the per-channel flags (ChannelData, render.h:486-492).
 * The grid is width x height x width (x, y, z), GRID_WIDTH/GRID_HEIGHT of
 * render.h:27-29, here chosen at run time. */
typedef struct LeniaWorldDesc {
    int width;
    int height;
    int channels;
    float timestep;
    float theta_a;
    float n_alpha;   /* N: accepted, unused (as in the reference) */
    float s_norm;
    float gta;
    float sta;
    float v_damp;
    float v_beta;    /* accepted, unused (as in the reference) */
    float iso_value;
    float sigma;     /* off_table.sigma */
    float dd;        /* off_table.dd, truncated to int */
    int alpha_mode;  /* accepted, no effect (as in the reference) */
    int growth_type;
    int mode_type;
    int sobel_border;
    int border;
    int gradient_mode;
    int adv_vel;
    int mu_vel;
    int blur_central_diff;
    int osc_la;
    int osc_flow;
    int osc_div_flow;
    int osc_vel;
    float osc_la_amt;
    float osc_flow_amt;
    float osc_div_flow_amt;
    int asymptotic[LENIA_MAX_CHANNELS];
    int soft_clip[LENIA_MAX_CHANNELS];
    int rt_all_channels; /* 0 = reference: SRT/RT transport channels 0-2 only */
    int alpha_index_fix; /* 0 = reference: PREALPHA/GA read at the padded offset */
    int exact_bell;      /* 0 = reference: growth from the 256^3 table at the truncated
                          * indices of u, m and s (Q1, lenia.h:79-84); 1 = bell(u, m, s)
                          * evaluated for each cell (no quantisation of u) */
    int conserve_mass;   /* 0 = reference; 1 = after every step each channel is rescaled
                          * so that its total (summed in double on the GPU, fixed order)
                          * equals the total it had when the grid was last written
                          * (lenia_set_field of A, lenia_create, lenia_set_params) */
} LeniaWorldDesc;

/* One kernel: the parameter part of `Kernel` (render.h:347-361). */
typedef struct LeniaKernelParams {
    int radius;
    int beta_size;
    float b[LENIA_MAX_BETA];
    float r_a;
    float m;
    float s;
    float h;
    int c0; /* source channel */
    int c1; /* destination channel */
} LeniaKernelParams;

/* Fields (the reference's arrays, render.h:277-328, lenia.cpp:9-89), each
 * unpadded, channel-major, x fastest (IDX, render.h:334).  Vector fields are
 * three blocks x, y, z.  Fields marked (debug) exist only after
 * lenia_set_debug(w, 1). */
typedef enum LeniaField {
    LENIA_FIELD_A = 0,         /* GRID, C*N */
    LENIA_FIELD_V = 1,         /* V_x,V_y,V_z, 3*C*N */
    LENIA_FIELD_GA = 2,        /* C*N */
    LENIA_FIELD_SUM = 3,       /* N */
    LENIA_FIELD_H = 4,         /* C*N */
    LENIA_FIELD_U_SUM = 5,     /* C*N */
    LENIA_FIELD_BACK = 6,      /* C*N */
    LENIA_FIELD_NA = 7,        /* 3*N (debug) */
    LENIA_FIELD_NU = 8,        /* 3*C*N (debug) */
    LENIA_FIELD_PREALPHA = 9,  /* C*N (debug) */
    LENIA_FIELD_ALPHA = 10,    /* C*N (debug, or with OSC_DIV_FLOW) */
    LENIA_FIELD_F = 11,        /* 3*C*N (debug, or when advection/oscillators read it) */
    LENIA_FIELD_MU = 12,       /* 3*C*N */
    LENIA_FIELD_TT = 13,       /* C*N (debug: TT before the transposition epilogue) */
    LENIA_FIELD_U_S = 14,      /* C*N (central difference) */
    LENIA_FIELD_SUM_S = 15,    /* N (central difference) */
    LENIA_FIELD_U = 16,        /* K*N: u_k per kernel (debug, or a direct convolution mode) */
    LENIA_FIELD_H_RB = 17,     /* C*N: H of the previous step */
    LENIA_FIELD_U_SUM_RB = 18, /* C*N: U_SUM of the previous step */
    LENIA_FIELD_RBB = 19       /* C*N: grid snapshot for meshing */
} LeniaField;

/* Stage groups of one step, each a run of the reference's events
 * (render.h:181-197). */
typedef enum LeniaStage {
    LENIA_STAGE_GROWTH = 0,    /* SIM_EVENT_FFT + FFT_MT: u_k, H, U_SUM, BACK */
    LENIA_STAGE_BLUR = 1,      /* SIM_EVENT_BLUR: U_S, SUM_S */
    LENIA_STAGE_FLOW = 2,      /* TSB, SOBEL_ONE, SOBEL_TWO, F, MU, TB: V, MU */
    LENIA_STAGE_TRANSPORT = 3, /* REINTEGRATION + TRM: A, GA, SUM */
    LENIA_STAGE_SNAPSHOT = 4   /* TMB: RBB */
} LeniaStage;

typedef struct lenia_world lenia_world;

/* Creates a world on the current CUDA device: validates the description
 * (width/height in [8,256], multiples of 4, prime factors in {2,3,5,7,11};
 * channels 1..4; kernels 0..64 with channels in range), allocates device
 * state, builds the kernels (init_kernel, lenia.cpp:199-261), the growth
 * table rows (init_bell_lut, lenia.cpp:93-101) and the blur kernel
 * (precompute_blur_kernel, reintegration.cpp:13-78).  All fields start at 0. */
lenia_status lenia_create(const LeniaWorldDesc *desc, const LeniaKernelParams *kernels,
                          int n_kernels, lenia_world **out);
lenia_status lenia_destroy(lenia_world *w);

/* Replaces scalars and modes (same grid shape and channel count): the
 * reference's UI edits of the globals (config.cpp:406-520). */
lenia_status lenia_set_params(lenia_world *w, const LeniaWorldDesc *desc);
/* Replaces the kernel set (init_kernel per kernel, lenia.cpp:199-261). */
lenia_status lenia_set_kernels(lenia_world *w, const LeniaKernelParams *kernels, int n_kernels);

/* Copies `count` floats into / out of a field.  `on_device` = 1 means the
 * pointer is device memory; 0 means host memory (pageable or pinned).
 * Field sizes are listed at LeniaField; count must match.  Device copies are
 * queued on the world's stream and return at once: order other streams'
 * use of the pointer after them (lenia_sync, or events).  Host copies
 * return when done. */
lenia_status lenia_set_field(lenia_world *w, int field, const float *src, size_t count, int on_device);
lenia_status lenia_get_field(lenia_world *w, int field, float *dst, size_t count, int on_device);
/* Number of floats of a field (0 if the field does not exist). */
size_t lenia_field_size(const lenia_world *w, int field);

/* Advances n_steps full steps (the 12 events FFT..TMB of render.cpp:376-583,
 * TMB only when snapshots are on).  Stream-ordered; returns when queued. */
lenia_status lenia_step(lenia_world *w, int n_steps);
/* Runs one stage group of the current step (per-stage parity hooks). */
lenia_status lenia_step_stage(lenia_world *w, int stage);

/* Uses `stream` (a cudaStream_t) for all later work of this world. */
lenia_status lenia_set_stream(lenia_world *w, void *stream);
/* Waits for the world's stream and reports device-side errors. */
lenia_status lenia_sync(lenia_world *w);
/* 1: keep the intermediate fields marked (debug) in LeniaField. */
lenia_status lenia_set_debug(lenia_world *w, int on);
/* No counterpart in the reference (it has no error handling, lenia.h:73).
 * Poll limit of the first wait of each block of the flow and transport
 * kernels for a tile copy into shared memory.  When a block's wait runs out,
 * the block records LENIA_ERR_TIMEOUT (reported by the next lenia_sync),
 * waits with the library's fixed long limit for the copies it still has in
 * flight, and returns without writing its tile's outputs; the world stays
 * usable.  polls < 0 restores the default (2^24 polls); 0 makes every such
 * wait give up at once (for tests of the timeout path). */
lenia_status lenia_set_wait_limit(lenia_world *w, long long polls);
/* 1: keep the mesh snapshots H_RB / U_SUM_RB / RBB every step.  RBB (the
 * grid after the step) is copied only when it is read out or before the
 * grid buffer it equals is overwritten; meshing reads that buffer in place. */
lenia_status lenia_set_snapshots(lenia_world *w, int on);

/* 1: bracket every kernel launch with CUDA events on the world's stream and
 * accumulate per-kernel device time (read with lenia_profile_read). */
lenia_status lenia_set_profiling(lenia_world *w, int on);
/* Synchronises, then writes per-kernel totals (milliseconds, launches) for
 * up to `n` kernel ids and clears them; returns the number of kernel ids. */
int lenia_profile_read(lenia_world *w, double *ms, long long *launches, int n);
/* Name of kernel id `kid` of lenia_profile_read (NULL past the last). */
const char *lenia_kernel_name(int kid);

/* ------------------------------------------------------- convolution modes
 * How the growth stage computes u_k = K_k (*) A_c0 (the reference: FFTW,
 * lenia.cpp:435-491).  LENIA_CONV_FFT is the half-spectrum FP32 FFT path.
 * The direct modes run the same periodic convolution in the spatial domain on
 * the tcgen05 tensor cores with FP32 accumulation: DIRECT_BF16 rounds grid
 * and kernel taps to BF16; DIRECT_BF16X3 splits each into hi + lo BF16 parts
 * and sums hi*hi + hi*lo + lo*hi.  Direct modes need every kernel's
 * radius * r_a <= 64 and keep u_k of every kernel in HBM (K x N floats). */
enum { LENIA_CONV_FFT = 0, LENIA_CONV_DIRECT_BF16 = 1, LENIA_CONV_DIRECT_BF16X3 = 2 };
/* Selects the convolution mode (rebuilds the kernel tables; synchronous). */
lenia_status lenia_set_conv_mode(lenia_world *w, int mode);
int lenia_get_conv_mode(lenia_world *w);
/* Tensor multiply-adds one direct convolution issues and the useful ones
 * (nonzero taps x cells x products per tap); both 0 in FFT mode. */
lenia_status lenia_conv_macs(lenia_world *w, double *issued, double *useful);

/* No counterpart in the reference.  Measures the growth stage on this world's
 * stream for every convolution mode whose bit is set in `modes` (bit i = mode
 * i; LENIA_CONV_FFT and LENIA_CONV_DIRECT_BF16X3 give FP32-level results,
 * DIRECT_BF16 does not), and for the FFT path every row tile its
 * runtime-sized kernels take (grids without size-specialised kernels), each
 * with the fused and the split growth (lenia_set_tuning), then keeps the
 * fastest.  The grid state is left as it was.  Synchronous. */
typedef struct LeniaTuneResult {
    int conv_mode;    /* the mode kept */
    int row_tile;     /* rows per block of the FFT row transforms (0: built-in choice) */
    float ms[3];      /* growth-stage milliseconds per mode, best variant; -1: not measured */
    int growth_split; /* FFT growth as two passes (see lenia_set_tuning) */
} LeniaTuneResult;
lenia_status lenia_autotune(lenia_world *w, int modes, LeniaTuneResult *out);
/* No counterpart in the reference.  The FFT path's tuning, as lenia_autotune
 * sets it: row_tile = rows per block of the runtime-sized row transforms (0:
 * the largest that fits; size-specialised grids ignore it); growth_split = 1
 * runs the growth stage as two passes, the inverse row transforms storing u_k
 * of every kernel (K x N floats, allocated here) and then the growth from
 * u_k, instead of one fused pass.  Results are identical either way. */
lenia_status lenia_set_tuning(lenia_world *w, int row_tile, int growth_split);

/* No counterpart in the reference.  u_out = Re(IFFT(FFT(field) * K^))/N for
 * one field and one kernel, computed exactly as a world's growth stage computes
 * u for that kernel, for callers that cannot allocate device memory: every
 * intermediate buffer lives in one fixed __device__ array (4,439,040 bytes,
 * about 4.4 MB per GPU, held until exit), so this call allocates nothing.  field and u_out are
 * device pointers of width*height*width floats; grids up to 64^3 are accepted
 * (larger ones return LENIA_ERR_INVALID_ARG).  Calls share that array, so
 * calls that overlap on the GPU race; the first call on a device looks up the
 * array's address (cudaGetSymbolAddress) with that device current and keeps
 * it, so after a cudaDeviceReset of that device the kept address is stale and
 * this call must not be used on it again in the same process. */
lenia_status lenia_convolve_noalloc(int width, int height, const float *field, const LeniaKernelParams *kernel,
                                    float *u_out, void *stream);

/* ---- Checkpoints --------------------------------------------------------
 *
 * The save/load that config.cpp:75-262 sketches (commented out in the
 * reference): the parameters, the kernels and every field that carries over
 * between steps (A, V, GA, SUM), as a versioned little-endian binary with a
 * CRC-32 trailer.  desc and kernels are the world's (the caller's copies);
 * step is a counter stored alongside. */
lenia_status lenia_save(lenia_world *w, const LeniaWorldDesc *desc, const LeniaKernelParams *kernels, int n_kernels,
                        unsigned long long step, const char *path);
/* Creates a world on the current device from a checkpoint; a wrong magic,
 * checksum or field size gives LENIA_ERR_INVALID_ARG, another version
 * LENIA_ERR_UNSUPPORTED.  step (optional) receives the stored counter. */
lenia_status lenia_load(const char *path, lenia_world **out, unsigned long long *step);

/* ---- Batches of worlds -------------------------------------------------
 *
 * Many independent worlds (any mix of sizes, channels, kernel sets and
 * modes) stepped together: the reference has no counterpart beyond calling
 * its step once per world.  Each world keeps only the fields that live from
 * step to step (A, V, GA, SUM); the buffers of one step belong to a lane, a
 * stream whose worlds run one after another, and lanes run concurrently.
 * Worlds that qualify (cubic grids of 24 .. 96 cells per side, FFT
 * convolution, no debug outputs, snapshots, mass conservation, blur, F or
 * ALPHA, transport by the dd = 1 gather or per cell) are instead stepped by
 * batched launches: per stage one launch per grid size (the transforms) or
 * one launch for all of them (growth from u_k, flow, transport), whose
 * blocks each take one block of one world from a device work list, in waves
 * whose per-step buffers share one scratch pool (at most 48 GB and a third of
 * the device memory free when the step is captured).  One step
 * of every world is captured once into a CUDA graph and replayed, so a batch
 * step is one graph launch.  Every world computes exactly what a world of
 * lenia_create computes (bit-identical fields). */
typedef struct lenia_batch lenia_batch;

/* descs[n_worlds]; kernels: every world's kernels one after another,
 * kernel_counts[i] of them for world i; lanes: concurrent streams (0 = up to
 * 64).  Worlds start at 0, like lenia_create's. */
lenia_status lenia_batch_create(const LeniaWorldDesc *descs, const LeniaKernelParams *kernels,
                                const int *kernel_counts, int n_worlds, int lanes, lenia_batch **out);
lenia_status lenia_batch_destroy(lenia_batch *b);
int lenia_batch_size(const lenia_batch *b);
/* Field copies of world `world` (A, V, GA or SUM; as lenia_set_field /
 * lenia_get_field), ordered with the steps on the batch's stream. */
lenia_status lenia_batch_set_field(lenia_batch *b, int world, int field, const float *src, size_t count,
                                   int on_device);
lenia_status lenia_batch_get_field(lenia_batch *b, int world, int field, float *dst, size_t count, int on_device);
/* n_steps graph launches on the batch's stream; returns when queued. */
lenia_status lenia_batch_step(lenia_batch *b, int n_steps);
/* Uses `stream` (a cudaStream_t) for later steps and copies. */
lenia_status lenia_batch_set_stream(lenia_batch *b, void *stream);
/* Waits for the batch and reports the first world's device-side error. */
lenia_status lenia_batch_sync(lenia_batch *b);
/* No counterpart in the reference.  lenia_autotune (above) on the
 * first world of every grid shape in the batch, its choice (convolution mode,
 * row tile) applied to every world of that shape, then the batch's step graphs
 * captured again.  per_world: n_worlds results, or NULL.  Synchronous. */
lenia_status lenia_batch_autotune(lenia_batch *b, int modes, LeniaTuneResult *per_world);
/* Kernel launches one batch step contains (all worlds). */
int lenia_batch_launches_per_step(const lenia_batch *b);
/* No counterpart in the reference.  on = 0 steps every world through its own
 * launches on the lanes, on = 1 (the default) lets the worlds that qualify
 * take the batched launches; the step graphs are captured again.  The fields
 * are the same either way.  Synchronous. */
lenia_status lenia_batch_set_batched_launches(lenia_batch *b, int on);
/* Worlds the batched launches step (the rest run on the lanes). */
int lenia_batch_grouped_worlds(const lenia_batch *b);
const char *lenia_batch_last_error(const lenia_batch *b);

/* ---- Statistics for labelling runs --------------------------------------
 *
 * No counterpart in the reference.  Per channel of the grid A, in double
 * precision with a fixed summation order (identical on every run):
 *   0 mass sum a;  1-6 sum a cos(2 pi x / W), sum a sin(2 pi x / W), the same
 *   for y (H) and z (W) - the torus-aware centroid and spread;  7 max a;
 *   8 number of cells with a > fill_threshold. */
#define LENIA_STATS 9
/* out: channels x LENIA_STATS doubles (host memory).  Synchronises. */
lenia_status lenia_world_stats(lenia_world *w, float fill_threshold, double *out);
/* out: every world's channels x LENIA_STATS doubles, in world order (host). */
lenia_status lenia_batch_stats(lenia_batch *b, float fill_threshold, double *out);

/* ---- Proposal network ----------------------------------------------------
 *
 * No counterpart in the reference.  A multilayer perceptron n_in -> hidden ->
 * hidden -> hidden -> 1 with GELU, trained and evaluated by this library's
 * own kernels: every matrix product (forward, weight gradient, activation
 * gradient) runs on the tcgen05 tensor cores with bfloat16 operands (weights,
 * activations, and dz in the backward products, rounded to nearest even) and
 * float32 accumulation in tensor memory; the loss is binary cross-entropy on
 * the logit, and Adam updates float32 master weights.  Parameters are laid
 * out layer by layer, W (out x in, row-major) then b. */
typedef struct lenia_mlp lenia_mlp;
lenia_status lenia_mlp_create(int n_in, int hidden, unsigned long long seed, lenia_mlp **out);
lenia_status lenia_mlp_destroy(lenia_mlp *m);
long long lenia_mlp_param_count(const lenia_mlp *m);
lenia_status lenia_mlp_get_params(lenia_mlp *m, float *out, size_t n);
lenia_status lenia_mlp_set_params(lenia_mlp *m, const float *src, size_t n);
/* Gradients of the last lenia_mlp_gradients / lenia_mlp_train_step. */
lenia_status lenia_mlp_get_grads(lenia_mlp *m, float *out, size_t n);
/* x: B x n_in (device, row-major); logits: B floats (device); on `stream`. */
lenia_status lenia_mlp_forward(lenia_mlp *m, const float *x, int B, float *logits, void *stream);
/* Loss (mean binary cross-entropy, host) and gradients of a batch; y: B
 * targets in {0, 1} (device).  Synchronises the stream. */
lenia_status lenia_mlp_gradients(lenia_mlp *m, const float *x, const float *y, int B, float *loss_out, void *stream);
/* lenia_mlp_gradients, then one Adam step (0.9, 0.999, 1e-8) with learning
 * rate lr and decoupled weight decay wd. */
lenia_status lenia_mlp_train_step(lenia_mlp *m, const float *x, const float *y, int B, float lr, float wd,
                                  float *loss_out, void *stream);
const char *lenia_mlp_last_error(const lenia_mlp *m);

/* ---- Marching cubes --------------------------------------------------
 *
 * Replaces generate_mesh_v1/v2/v3 (mesh.cpp:34-431, 434-1109, 1115-2037)
 * with the buffer reset and concatenation around them (render.cpp:153-212):
 * an iso-surface of every channel of one to three fields meshed together, one
 * vertex per intersected grid edge and field, face normals summed into the
 * vertices, and a triangle index buffer.  The reference's D3D vertex buffers
 * (position, normal, colour) become flat arrays; the colour becomes the
 * vertex's channel.  Cube (gx, gy, gz), gx, gy, gz in [0, width), reads its
 * corners at +1 from the periodic copy of the field's halo source on the
 * +x/+y/+z faces and 0 on the halo edges (transpose_mesh_borders,
 * transposition.cpp:881-995).
 *
 * The triangle table is this library's own (the reference's is third-party
 * data): built from geometry, it has the same triangle count as the
 * reference's for every one of the 256 cases (lenia_mc_triangle_table). */

/* The reference's views (render.cpp:625-636): NORMAL meshes RBB (v1); U adds
 * U_SUM_RB shifted along x (v2); H adds U_SUM_RB along x and H_RB along z (v3). */
enum { LENIA_VIEW_NORMAL = 0, LENIA_VIEW_U = 1, LENIA_VIEW_H = 2 };

typedef struct LeniaMeshDesc {
    int width;            /* grid width (= depth) */
    int height;
    int channels;         /* meshed channels 0 .. channels-1 of every field */
    int fields;           /* 1..3 fields meshed together; per cube their triangles follow in field order */
    float iso_value;      /* ISO_VALUE (render.h:61): a corner is inside when value > iso_value */
    float cell_size;      /* CELL_SIZE (render.h:26), 3.5 */
    float offset[3][3];   /* per field, added to x, y, z after interpolation where nonzero */
    int slabs;            /* z ranges meshed with separate vertex maps, as the MESH_THREADS (render.h:15)
                             mesh threads split z (mesh.cpp:42-43): 2 reproduces the reference, 1 gives one
                             mesh without seam duplicates */
    int share_channels;   /* 1: one vertex map per field for all channels, as V1_EDGES is cleared only per
                             mesh (render.cpp:182), so a channel reuses the vertex an earlier channel put on
                             the same edge; 0: a vertex map per field and channel */
} LeniaMeshDesc;

/* Arrays of the last mesh (lenia_mesher_get).  Vertices are numbered in the
 * order the reference creates them: by slab, then channel, then cube
 * (x fastest), then field, then triangle slot. */
typedef enum LeniaMeshArray {
    LENIA_MESH_POSITIONS = 0,      /* float, 3 per vertex */
    LENIA_MESH_NORMALS = 1,        /* float, 3 per vertex: unnormalised sums of face normals (B-A)x(C-A) */
    LENIA_MESH_VERTEX_CHANNEL = 2, /* int32, 1 per vertex: channel + channels * field of the creating triangle */
    LENIA_MESH_INDICES = 3,        /* uint32, 3 per triangle */
    LENIA_MESH_FACE_NORMALS = 4,   /* float, 3 per triangle */
    LENIA_MESH_CASES = 5           /* uint8, fields * channels * width * height * width: case index per cube */
} LeniaMeshArray;

typedef struct lenia_mesher lenia_mesher;

/* Fills a description for one of the reference's views (two slabs, channels
 * sharing vertex maps, CELL_SIZE 3.5, offsets width * 3.5). */
lenia_status lenia_mesh_desc_for_view(int view, int width, int height, int channels, float iso_value,
                                      LeniaMeshDesc *out);
/* Creates a mesher on the current CUDA device for fields of desc's shape
 * (width/height in [2, 512], channels 1..4, fields 1..3, slabs 1..width). */
lenia_status lenia_mesher_create(const LeniaMeshDesc *desc, lenia_mesher **out);
lenia_status lenia_mesher_destroy(lenia_mesher *m);
/* Meshes desc.fields fields (device pointers, each channels * width * height *
 * width floats, channel-major, x fastest) on `stream` (a cudaStream_t; NULL =
 * default).  halos: per field the array whose periodic copy the +1 faces
 * hold (NULL, or a NULL entry: the field itself).  Synchronises once, to size
 * the output, and returns the counts; the arrays are then ready on `stream`.
 * Output buffers grow as needed. */
lenia_status lenia_mesher_run(lenia_mesher *m, const float *const *fields, const float *const *halos, void *stream,
                              long long *n_vertices, long long *n_triangles);
/* Copies one LeniaMeshArray of the last mesh, on the stream of the last run
 * (which must still exist); `count` is in elements and must equal the array's
 * size.  on_device: dst is device memory. */
lenia_status lenia_mesher_get(lenia_mesher *m, int which, void *dst, size_t count, int on_device);
/* lenia_mesher_run on a world's snapshots for a view (snapshots on; a mesher
 * of view + 1 fields): RBB, U_SUM_RB, H_RB, whose +1 faces copy RBB, U_SUM
 * and H, on the world's stream. */
lenia_status lenia_mesh_world(lenia_world *w, int view, lenia_mesher *m, long long *n_vertices,
                              long long *n_triangles);
/* Writes the triangle table (256 cases x 16 edge indices, -1 after the last
 * triangle; edges numbered as EDGE_TO_VERTICES, marching_cubes.h:17-22) and
 * returns 0.  Host-only: needs no device. */
int lenia_mc_triangle_table(int *table);
/* Description of the last failure on m (never NULL). */
const char *lenia_mesher_last_error(const lenia_mesher *m);

/* Number of kernel launches the last lenia_step issued per step. */
int lenia_launches_per_step(const lenia_world *w);
/* Human-readable description of the last failure on w (never NULL). */
const char *lenia_last_error(const lenia_world *w);
/* Library version string. */
const char *lenia_version(void);

#ifdef __cplusplus
}
#endif
#endif
