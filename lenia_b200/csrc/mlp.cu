// A small multilayer perceptron trained on the GPU by this file's own
// kernels: the proposal network of the persistent-pattern search (no
// counterpart in the reference).
//
//   n_in -> hidden -> hidden -> hidden -> 1, GELU (0.5 x (1 + erf(x / sqrt 2)))
//   after every hidden layer, a logit out; binary cross-entropy on the logit.
//
// Precision: every matrix product takes bfloat16 operands (round to nearest
// even) and accumulates in float32 in tensor memory: the forward products
// (activations x weights), and both backward products (the weight gradient
// dz^T x activations and the activation gradient dz x W, with dz rounded to
// bfloat16 as it enters them).  Biases, pre-activations, dz, gradients and
// the Adam state are float32, and the Adam update runs on float32 master
// weights, whose bfloat16 copies (W and W^T) are refreshed after each update.
//
// Kernels: one tcgen05 matrix product C = A B^T (both operands K-major
// bfloat16 in global memory, staged by TMA, FP32 accumulators in tensor
// memory) with per-use epilogues (bias + GELU writing the next layer's
// operands, the logit, the weight gradient, the activation gradient through
// GELU'), the loss with its gradient, column sums for the bias gradients,
// Adam, and the bfloat16 packing of weights and inputs.
#include <cuda.h>
#include <cuda_bf16.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <random>
#include <string>
#include <vector>

#include "lenia_internal.h"
#include "tma.cuh"

using namespace lenia;

namespace {

constexpr int kMlpLayers = 4;

// ---- tcgen05 matrix product ------------------------------------------------
// C[M x N] = sum_k A[m, k] B[n, k]: A (M x K) and B (N x K) bfloat16, each row
// K-contiguous with a row stride that is a multiple of 8 elements; reads past
// a matrix's true extent (rows, or k >= K) return zero (TMA fill), so the
// operands need no padding in memory.  One CTA owns 128 rows of C and all of
// its N <= 256 columns (the MMA is 128 x Np x 16, Np = N rounded up to 16).
// K streams through shared memory in chunks of 64 in a three-stage pipeline:
// per chunk, per 8-element k slice, one TMA box of 128 A rows and one of Np B
// rows, each landing as a column of 8 x 16-byte core matrices (the canonical
// K-major layout without swizzle: core matrices adjacent in M/N 128 bytes
// apart, adjacent in K `rows` x 16 bytes apart).  Thread 0 issues the copies,
// thread 32 the MMAs; after the last MMA sixteen warps read the accumulator
// (warp w: lanes 32(w % 4)..+31 = rows, every fourth 32-column group from
// 32(w / 4)) and run the epilogue (its GELU evaluations are the long part).
constexpr int kGemmM = 128;
constexpr int kGemmKC = 64;      // K per stage
constexpr int kGemmStages = 3;
constexpr int kGemmThreads = 512;  // 16 warps: 4 per tensor-memory lane quadrant in the epilogue
constexpr int kGemmHeader = 1024;
constexpr unsigned long long kGemmWaitNs = 2000000000ull;  // 2 s per wait
constexpr unsigned kGemmWaitPolls = 1u << 30;

enum GemmMode { kEpiHidden = 0, kEpiLogit = 1, kEpiWeightGrad = 2, kEpiActGrad = 3 };

struct TcGemm {
    int M, N, K;       // rows and columns of C, reduction length
    int Np;            // MMA N (N rounded up to 16)
    int mode;
    int kper;                    // K per CTA row (blockIdx.y): a multiple of 64
    float *ws;                   // split K (gridDim.y > 1): partial sums [y][M][N]
    const float *bias;           // kEpiHidden, kEpiLogit
    float *c32;                  // float32 result (z, logit, dW or dz)
    long long ldc;
    const float *zin;            // kEpiActGrad: pre-activation of the layer below
    long long ldz;
    __nv_bfloat16 *ob;           // kEpiHidden / kEpiActGrad: bfloat16 copy, row-major
    long long ldo;
    __nv_bfloat16 *obt;          // ... and transposed ([n][m])
    long long ldot;
    int *err;                    // bit 2 set when a wait ran out
};

__device__ __forceinline__ unsigned long long gemm_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for phase `parity`; false after kGemmWaitNs (or kGemmWaitPolls polls).
__device__ bool gemm_wait(uint64_t *bar, unsigned parity)
{
    const uint32_t a = smem_addr(bar);
    unsigned long long t0 = 0;
    for (unsigned i = 0; i < kGemmWaitPolls; i++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 255u) == 0) {
            const unsigned long long t = gemm_ns();
            if (i == 0) t0 = t;
            else if (t - t0 > kGemmWaitNs) return false;
        }
    }
    return false;
}

// Shared-memory matrix descriptor without swizzle (start, leading byte offset
// = between core matrices along K, stride byte offset = along M/N, all in
// 16-byte units; bit 46: descriptor version of sm_100).
__device__ __forceinline__ uint64_t gemm_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];\n" ::"r"(smem_addr(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float z)
{
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

__global__ void __launch_bounds__(kGemmThreads, 1) k_tc_gemm(TcGemm g, const __grid_constant__ CUtensorMap tma,
                                                            const __grid_constant__ CUtensorMap tmb)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t *full = (uint64_t *)smem;            // [kGemmStages]
    uint64_t *empty = full + kGemmStages;         // [kGemmStages]
    uint64_t *done = empty + kGemmStages;         // accumulator complete
    uint32_t *tmem_slot = (uint32_t *)(smem + 256);
    int *s_bad = (int *)(smem + 260);
    int *s_issued = (int *)(smem + 264);
    int *s_consumed = (int *)(smem + 268);
    unsigned char *stages = smem + kGemmHeader;
    const uint32_t a_bytes = 8u * kGemmM * 16u, b_bytes = 8u * (uint32_t)g.Np * 16u;
    const uint32_t stage_bytes = a_bytes + b_bytes;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kGemmM;
    // this CTA's share of K: [kbeg, kend), whole 64-element chunks except at K
    const int Kp = (g.K + 15) / 16 * 16;
    const int kbeg = blockIdx.y * g.kper;
    const int kend = min(Kp, kbeg + g.kper);
    const int nchunks = (kend - kbeg + kGemmKC - 1) / kGemmKC;
    const uint32_t ncols = g.Np <= 32 ? 32u : g.Np <= 64 ? 64u : g.Np <= 128 ? 128u : 256u;
    // kind::f16, D float32, A and B bfloat16, both K-major, N >> 3, M >> 4
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(g.Np >> 3) << 17) |
                           ((uint32_t)(kGemmM >> 4) << 24);

    if (threadIdx.x == 0) {
        for (int i = 0; i < kGemmStages; i++) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        mbar_init(done, 1);
        *s_bad = 0;
        *s_issued = 0;
        *s_consumed = 0;
        mbar_init_fence();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(tmem_slot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (threadIdx.x == 0) {
        // copies: chunk i into stage i % kGemmStages once its previous MMAs are done
        int i = 0;
        for (; i < nchunks; i++) {
            const int s = i % kGemmStages;
            if (i >= kGemmStages && !gemm_wait(&empty[s], (unsigned)(i / kGemmStages - 1) & 1u)) {
                atomicOr(s_bad, 1);
                break;
            }
            if (*(volatile int *)s_bad) break;
            const int k0 = kbeg + i * kGemmKC;
            const int nk = min(8, (kend - k0) / 8);  // 8-element k slices in this chunk
            unsigned char *sa = stages + (size_t)s * stage_bytes, *sb = sa + a_bytes;
            mbar_arrive_expect_tx(&full[s], (unsigned)nk * (kGemmM * 16u + (unsigned)g.Np * 16u));
            for (int c = 0; c < nk; c++) {
                tma_load_2d(sa + (size_t)c * kGemmM * 16, &tma, k0 + 8 * c, m0, &full[s]);
                tma_load_2d(sb + (size_t)c * g.Np * 16, &tmb, k0 + 8 * c, 0, &full[s]);
            }
        }
        *(volatile int *)s_issued = i;
    } else if (threadIdx.x == 32) {
        int i = 0;
        for (; i < nchunks; i++) {
            const int s = i % kGemmStages;
            if (!gemm_wait(&full[s], (unsigned)(i / kGemmStages) & 1u)) {
                atomicOr(s_bad, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const int k0 = kbeg + i * kGemmKC;
            const int nm = min(4, (kend - k0) / 16);
            const uint32_t sa = smem_addr(stages + (size_t)s * stage_bytes), sb = sa + a_bytes;
            for (int j = 0; j < nm; j++) {
                const uint64_t da = gemm_desc(sa + (uint32_t)j * 2u * kGemmM * 16u, kGemmM * 16u, 128u);
                const uint64_t db = gemm_desc(sb + (uint32_t)j * 2u * (uint32_t)g.Np * 16u, (uint32_t)g.Np * 16u, 128u);
                const uint32_t acc = (i > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_addr(&empty[s]))
                         : "memory");
        }
        *(volatile int *)s_consumed = i;
        // completes once every MMA issued above has finished
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         smem_addr(done))
                     : "memory");
    }
    if (!gemm_wait(done, 0u)) atomicOr(s_bad, 1);
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    __syncthreads();
    const bool bad = *(volatile int *)s_bad != 0;

    if (!bad) {
        const int quad = warp & 3, part = warp >> 2;
        const int m = m0 + quad * 32 + lane;
        const bool row_ok = m < g.M;
        for (int c0 = 32 * part; c0 < g.Np; c0 += 128) {
            uint32_t v[32];
            tmem_ld32(tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)c0, v);
            if (!row_ok) continue;
#pragma unroll
            for (int j = 0; j < 32; j++) {
                const int n = c0 + j;
                if (n >= g.N) break;
                const float acc = __uint_as_float(v[j]);
                if (g.ws) {
                    g.ws[((long long)blockIdx.y * g.M + m) * g.N + n] = acc;
                } else if (g.mode == kEpiHidden) {
                    const float z = acc + g.bias[n];
                    g.c32[(long long)m * g.ldc + n] = z;
                    const __nv_bfloat16 a = __float2bfloat16_rn(gelu(z));
                    g.ob[(long long)m * g.ldo + n] = a;
                    g.obt[(long long)n * g.ldot + m] = a;
                } else if (g.mode == kEpiLogit) {
                    g.c32[(long long)m * g.ldc + n] = acc + g.bias[n];
                } else if (g.mode == kEpiWeightGrad) {
                    g.c32[(long long)m * g.ldc + n] = acc;
                } else {
                    const float dz = acc * gelu_grad(g.zin[(long long)m * g.ldz + n]);
                    g.c32[(long long)m * g.ldc + n] = dz;
                    const __nv_bfloat16 b = __float2bfloat16_rn(dz);
                    g.ob[(long long)m * g.ldo + n] = b;
                    g.obt[(long long)n * g.ldot + m] = b;
                }
            }
        }
    } else if (threadIdx.x == 0) {
        // a wait ran out: record it, and let the copies still in flight land
        // (bounded) before the block's shared memory is released
        if (g.err) atomicOr(g.err, 2);
        const int issued = *(volatile int *)s_issued, consumed = *(volatile int *)s_consumed;
        for (int i = consumed; i < issued; i++) gemm_wait(&full[i % kGemmStages], (unsigned)(i / kGemmStages) & 1u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(ncols) : "memory");
}

// c[m][n] = sum over s = 0, 1, ... of ws[s][m][n] (fixed order).
__global__ void k_split_sum(const float *__restrict__ ws, int ns, int M, int N, float *__restrict__ c, long long ldc)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long mn = (long long)M * N;
    if (i >= mn) return;
    float s = ws[i];
    for (int k = 1; k < ns; k++) s += ws[(long long)k * mn + i];
    const int m = (int)(i / N), n = (int)(i - (long long)m * N);
    c[(long long)m * ldc + n] = s;
}

size_t gemm_smem(int Np) { return kGemmHeader + (size_t)kGemmStages * (8u * kGemmM * 16u + 8u * (unsigned)Np * 16u); }

// A bfloat16 matrix in global memory: rows x cols, row stride ld (a multiple of 8).
struct Bf16Mat {
    __nv_bfloat16 *p = nullptr;
    int rows = 0, cols = 0;
    long long ld = 0;
};

int round_up(int x, int m) { return (x + m - 1) / m * m; }

// Tensor map of the first `rows` rows and `cols` columns of m (reads past
// either extent return zero) with a box of 8 columns x box_rows rows: one k
// slice of an operand tile.
cudaError_t gemm_map(CUtensorMap *map, const Bf16Mat &m, int rows, int cols, int box_rows)
{
    const unsigned long long dims[2] = {(unsigned long long)cols, (unsigned long long)rows};
    const unsigned long long strides[1] = {(unsigned long long)m.ld * 2ull};
    const unsigned box[2] = {8u, (unsigned)box_rows};
    return encode_tensor_map_strided(map, m.p, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, dims, strides, box);
}

// C = A B^T for the first M rows of A and N rows of B (each K columns wide).
// ksplit > 1 (weight gradients only) splits K over that many CTA rows, each
// writing its partial product to ws (ksplit x M x N floats); k_split_sum
// then adds the partials in split order into g.c32.
cudaError_t tc_gemm(const Bf16Mat &A, int M, const Bf16Mat &B, int N, int K, TcGemm g, cudaStream_t st,
                    int ksplit = 1, float *ws = nullptr)
{
    if (M < 1 || N < 1 || N > 256 || K < 1 || A.cols < K || B.cols < K || A.rows < M || B.rows < N)
        return cudaErrorInvalidValue;
    g.M = M;
    g.N = N;
    g.K = K;
    g.Np = round_up(N, 16);
    const int Kp = round_up(K, 16);
    if (ksplit < 1 || (ksplit > 1 && (!ws || g.mode != kEpiWeightGrad))) return cudaErrorInvalidValue;
    g.kper = round_up((Kp + ksplit - 1) / ksplit, kGemmKC);
    ksplit = (Kp + g.kper - 1) / g.kper;
    g.ws = ksplit > 1 ? ws : nullptr;
    CUtensorMap ta, tb;
    cudaError_t e = gemm_map(&ta, A, M, K, kGemmM);
    if (e == cudaSuccess) e = gemm_map(&tb, B, N, K, g.Np);
    if (e != cudaSuccess) return e;
    const size_t smem = gemm_smem(g.Np);
    e = cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((M + kGemmM - 1) / kGemmM, ksplit);
    k_tc_gemm<<<grid, kGemmThreads, smem, st>>>(g, ta, tb);
    e = cudaGetLastError();
    if (e == cudaSuccess && ksplit > 1) {
        const long long n = (long long)M * N;
        k_split_sum<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(ws, ksplit, M, N, g.c32, g.ldc);
        e = cudaGetLastError();
    }
    return e;
}

// dst[r][c] = bf16(src[r][c]) (or of src[c][r] with transpose) for r < rows,
// c < cols of dst.
__global__ void k_pack_bf16(const float *__restrict__ src, long long lds, int transpose, __nv_bfloat16 *dst,
                            long long ldd, int rows, int cols)
{
    const long long n = (long long)rows * cols;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / cols), c = (int)(i - (long long)r * cols);
        const float v = transpose ? src[(long long)c * lds + r] : src[(long long)r * lds + c];
        dst[(long long)r * ldd + c] = __float2bfloat16_rn(v);
    }
}

// Binary cross-entropy on logits, mean over the batch: per-row loss into
// rowloss, gradient (sigmoid(z) - y) / B into dz (float32) and its bfloat16
// copies dzb (row b, column 0) and dzbt (row 0, column b).
__global__ void k_bce(const float *__restrict__ z, const float *__restrict__ y, float *__restrict__ dz,
                      __nv_bfloat16 *__restrict__ dzb, long long lddzb, __nv_bfloat16 *__restrict__ dzbt,
                      float *__restrict__ rowloss, int B)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B) return;
    const float zi = z[i], yi = y[i];
    const float s = 1.0f / (1.0f + expf(-zi));
    // log(1 + e^-|z|) + max(z, 0) - z y
    rowloss[i] = log1pf(expf(-fabsf(zi))) + fmaxf(zi, 0.0f) - zi * yi;
    const float g = (s - yi) / (float)B;
    dz[i] = g;
    const __nv_bfloat16 gb = __float2bfloat16_rn(g);
    dzb[(long long)i * lddzb] = gb;
    dzbt[i] = gb;
}

// db[n] = sum over rows of dz[m, n] (rows summed in order; one thread per column)
__global__ void k_colsum(const float *__restrict__ dz, int M, int N, float *__restrict__ db)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.0f;
    for (int m = 0; m < M; m++) s += dz[(long long)m * N + n];
    db[n] = s;
}

// Sum of the first n values (one block, fixed order).
__global__ void k_sum(const float *__restrict__ v, int n, float *__restrict__ out)
{
    __shared__ float s[256];
    float a = 0.0f;
    for (int i = threadIdx.x; i < n; i += 256) a += v[i];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m1,
                       float *__restrict__ m2, long long n, float lr, float b1, float b2, float eps, float c1,
                       float c2, float wd)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i] + wd * w[i];
        m1[i] = b1 * m1[i] + (1.0f - b1) * gi;
        m2[i] = b2 * m2[i] + (1.0f - b2) * gi * gi;
        const float mh = m1[i] / c1, vh = m2[i] / c2;
        w[i] -= lr * mh / (sqrtf(vh) + eps);
    }
}

unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096); }

}  // namespace

struct lenia_mlp {
    int dims[kMlpLayers + 1];            // n_in, h, h, h, 1
    long long woff[kMlpLayers], boff[kMlpLayers], nparams;
    float *params = nullptr, *grads = nullptr, *m1 = nullptr, *m2 = nullptr;
    // bfloat16 copies of the weights: W (out x in) for the forward products,
    // W^T (in x out) for the activation gradients
    Bf16Mat wb[kMlpLayers], wtb[kMlpLayers];
    // per batch (capacity cap rows): the input and every hidden activation in
    // bfloat16, row-major and transposed; pre-activations z (float32)
    Bf16Mat xb, xbt, ab[kMlpLayers - 1], abt[kMlpLayers - 1];
    float *z[kMlpLayers] = {};
    // dz of the layer being differentiated, ping-pong by layer parity:
    // float32 (bias gradients), bfloat16 row-major and transposed
    float *dz[2] = {};
    Bf16Mat dzb[2], dzbt[2];
    Bf16Mat dzb_out, dzbt_out;           // dz of the logit layer (one column)
    float *dz_out = nullptr, *rowloss = nullptr, *loss = nullptr;
    float *ws = nullptr;                 // split-K partial weight gradients
    int ksplit = 1;                      // K (batch) splits of the weight gradients
    int *err = nullptr;
    int cap = 0;
    long long step = 0;
    std::string err_msg;
};

namespace {

lenia_status mlp_fail(lenia_mlp *m, cudaError_t e, const char *where)
{
    if (m) m->err_msg = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? LENIA_ERR_OOM : LENIA_ERR_CUDA;
}

void free_mat(Bf16Mat &b)
{
    if (b.p) cudaFree(b.p);
    b = Bf16Mat();
}

cudaError_t alloc_mat(Bf16Mat &b, int rows, int cols)
{
    free_mat(b);
    b.rows = rows;
    b.cols = cols;
    b.ld = round_up(cols, 8);
    cudaError_t e = cudaMalloc((void **)&b.p, sizeof(__nv_bfloat16) * (size_t)rows * b.ld);
    if (e == cudaSuccess) e = cudaMemset(b.p, 0, sizeof(__nv_bfloat16) * (size_t)rows * b.ld);
    return e;
}

void free_acts(lenia_mlp *m)
{
    free_mat(m->xb);
    free_mat(m->xbt);
    for (int l = 0; l < kMlpLayers - 1; l++) {
        free_mat(m->ab[l]);
        free_mat(m->abt[l]);
    }
    for (int l = 0; l < kMlpLayers; l++) {
        if (m->z[l]) cudaFree(m->z[l]);
        m->z[l] = nullptr;
    }
    for (int i = 0; i < 2; i++) {
        if (m->dz[i]) cudaFree(m->dz[i]);
        m->dz[i] = nullptr;
        free_mat(m->dzb[i]);
        free_mat(m->dzbt[i]);
    }
    free_mat(m->dzb_out);
    free_mat(m->dzbt_out);
    float **bufs[] = {&m->dz_out, &m->rowloss, &m->ws};
    for (float **p : bufs) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    m->cap = 0;
}

cudaError_t ensure_batch(lenia_mlp *m, int B)
{
    if (B <= m->cap) return cudaSuccess;
    free_acts(m);
    const int cap = round_up(B, 128);
    const int n_in = m->dims[0], h = m->dims[1];
    cudaError_t e = alloc_mat(m->xb, cap, n_in);
    if (e == cudaSuccess) e = alloc_mat(m->xbt, n_in, cap);
    for (int l = 0; l < kMlpLayers - 1 && e == cudaSuccess; l++) {
        e = alloc_mat(m->ab[l], cap, h);
        if (e == cudaSuccess) e = alloc_mat(m->abt[l], h, cap);
    }
    for (int l = 0; l < kMlpLayers && e == cudaSuccess; l++)
        e = cudaMalloc((void **)&m->z[l], sizeof(float) * (size_t)cap * m->dims[l + 1]);
    for (int i = 0; i < 2 && e == cudaSuccess; i++) {
        e = cudaMalloc((void **)&m->dz[i], sizeof(float) * (size_t)cap * h);
        if (e == cudaSuccess) e = alloc_mat(m->dzb[i], cap, h);
        if (e == cudaSuccess) e = alloc_mat(m->dzbt[i], h, cap);
    }
    if (e == cudaSuccess) e = alloc_mat(m->dzb_out, cap, 1);
    if (e == cudaSuccess) e = alloc_mat(m->dzbt_out, 1, cap);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->dz_out, sizeof(float) * (size_t)cap);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->rowloss, sizeof(float) * (size_t)cap);
    // the weight gradients reduce over the batch: about 256 batch rows per CTA
    // row, at most 64 CTA rows
    m->ksplit = std::max(1, std::min(64, cap / 256));
    int widest = 0;
    for (int l = 0; l < kMlpLayers; l++) widest = std::max(widest, m->dims[l] * m->dims[l + 1]);
    if (e == cudaSuccess && m->ksplit > 1)
        e = cudaMalloc((void **)&m->ws, sizeof(float) * (size_t)m->ksplit * widest);
    if (e == cudaSuccess) m->cap = cap;
    return e;
}

cudaError_t pack(const float *src, long long lds, bool transpose, Bf16Mat &dst, int rows, int cols, cudaStream_t st)
{
    k_pack_bf16<<<blocks_for((long long)rows * cols), 256, 0, st>>>(src, lds, transpose ? 1 : 0, dst.p, dst.ld, rows,
                                                                    cols);
    return cudaGetLastError();
}

// Refreshes the bfloat16 weight copies from the float32 master weights.
cudaError_t refresh_weights(lenia_mlp *m, cudaStream_t st)
{
    cudaError_t e = cudaSuccess;
    for (int l = 0; l < kMlpLayers && e == cudaSuccess; l++) {
        const int K = m->dims[l], N = m->dims[l + 1];
        const float *W = m->params + m->woff[l];
        e = pack(W, K, false, m->wb[l], N, K, st);
        if (e == cudaSuccess) e = pack(W, K, true, m->wtb[l], K, N, st);
    }
    return e;
}

TcGemm epi(int mode)
{
    TcGemm g;
    memset(&g, 0, sizeof(g));
    g.mode = mode;
    return g;
}

// Forward pass of B rows: z of every layer; the hidden activations in
// bfloat16 (row-major for the next product, transposed for the weight
// gradients).
cudaError_t forward(lenia_mlp *m, const float *x, int B, cudaStream_t st)
{
    const int n_in = m->dims[0];
    cudaError_t e = pack(x, n_in, false, m->xb, B, n_in, st);
    if (e == cudaSuccess) e = pack(x, n_in, true, m->xbt, n_in, B, st);
    for (int l = 0; l < kMlpLayers && e == cudaSuccess; l++) {
        const int K = m->dims[l], N = m->dims[l + 1];
        const Bf16Mat &in = l == 0 ? m->xb : m->ab[l - 1];
        TcGemm g = epi(l + 1 < kMlpLayers ? kEpiHidden : kEpiLogit);
        g.bias = m->params + m->boff[l];
        g.c32 = m->z[l];
        g.ldc = N;
        if (l + 1 < kMlpLayers) {
            g.ob = m->ab[l].p;
            g.ldo = m->ab[l].ld;
            g.obt = m->abt[l].p;
            g.ldot = m->abt[l].ld;
        }
        g.err = m->err;
        e = tc_gemm(in, B, m->wb[l], N, K, g, st);
    }
    return e;
}

}  // namespace

extern "C" {

lenia_status lenia_mlp_create(int n_in, int hidden, unsigned long long seed, lenia_mlp **out)
{
    if (!out || n_in < 1 || hidden < 1 || hidden > 256 || n_in > 256) return LENIA_ERR_INVALID_ARG;
    *out = nullptr;
    lenia_mlp *m = new lenia_mlp();
    m->dims[0] = n_in;
    m->dims[1] = m->dims[2] = m->dims[3] = hidden;
    m->dims[4] = 1;
    long long off = 0;
    for (int l = 0; l < kMlpLayers; l++) {
        m->woff[l] = off;
        off += (long long)m->dims[l] * m->dims[l + 1];
        m->boff[l] = off;
        off += m->dims[l + 1];
    }
    m->nparams = off;
    // He-style initialisation, uniform in +-sqrt(6 / fan_in); biases 0
    std::vector<float> init(off, 0.0f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < kMlpLayers; l++) {
        const float lim = sqrtf(6.0f / (float)m->dims[l]);
        std::uniform_real_distribution<float> u(-lim, lim);
        for (long long i = 0; i < (long long)m->dims[l] * m->dims[l + 1]; i++) init[m->woff[l] + i] = u(rng);
    }
    cudaError_t e = cudaMalloc((void **)&m->params, sizeof(float) * off);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->grads, sizeof(float) * off);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->m1, sizeof(float) * off);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->m2, sizeof(float) * off);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(m->err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(m->params, init.data(), sizeof(float) * off, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m->grads, 0, sizeof(float) * off);
    if (e == cudaSuccess) e = cudaMemset(m->m1, 0, sizeof(float) * off);
    if (e == cudaSuccess) e = cudaMemset(m->m2, 0, sizeof(float) * off);
    for (int l = 0; l < kMlpLayers && e == cudaSuccess; l++) {
        e = alloc_mat(m->wb[l], m->dims[l + 1], m->dims[l]);
        if (e == cudaSuccess) e = alloc_mat(m->wtb[l], m->dims[l], m->dims[l + 1]);
    }
    if (e == cudaSuccess) e = refresh_weights(m, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        lenia_mlp_destroy(m);
        return e == cudaErrorMemoryAllocation ? LENIA_ERR_OOM : LENIA_ERR_CUDA;
    }
    *out = m;
    return LENIA_OK;
}

lenia_status lenia_mlp_destroy(lenia_mlp *m)
{
    if (!m) return LENIA_ERR_INVALID_ARG;
    free_acts(m);
    for (int l = 0; l < kMlpLayers; l++) {
        free_mat(m->wb[l]);
        free_mat(m->wtb[l]);
    }
    float *bufs[] = {m->params, m->grads, m->m1, m->m2, m->loss};
    for (float *p : bufs)
        if (p) cudaFree(p);
    if (m->err) cudaFree(m->err);
    delete m;
    return LENIA_OK;
}

long long lenia_mlp_param_count(const lenia_mlp *m) { return m ? m->nparams : 0; }

// Parameters as float32, layer by layer: W (out x in, row-major) then b.
lenia_status lenia_mlp_get_params(lenia_mlp *m, float *out, size_t n)
{
    if (!m || !out || (long long)n != m->nparams) return LENIA_ERR_INVALID_ARG;
    const cudaError_t e = cudaMemcpy(out, m->params, sizeof(float) * n, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? LENIA_OK : mlp_fail(m, e, "get_params");
}

lenia_status lenia_mlp_set_params(lenia_mlp *m, const float *src, size_t n)
{
    if (!m || !src || (long long)n != m->nparams) return LENIA_ERR_INVALID_ARG;
    cudaError_t e = cudaMemcpy(m->params, src, sizeof(float) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = refresh_weights(m, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return e == cudaSuccess ? LENIA_OK : mlp_fail(m, e, "set_params");
}

// Gradients of the last lenia_mlp_train_step (or lenia_mlp_gradients), same layout.
lenia_status lenia_mlp_get_grads(lenia_mlp *m, float *out, size_t n)
{
    if (!m || !out || (long long)n != m->nparams) return LENIA_ERR_INVALID_ARG;
    const cudaError_t e = cudaMemcpy(out, m->grads, sizeof(float) * n, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? LENIA_OK : mlp_fail(m, e, "get_grads");
}

// Logits of B rows of x (device, B x n_in row-major) into logits (device, B).
lenia_status lenia_mlp_forward(lenia_mlp *m, const float *x, int B, float *logits, void *stream)
{
    if (!m || !x || !logits || B < 1) return LENIA_ERR_INVALID_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = ensure_batch(m, B);
    if (e == cudaSuccess) e = forward(m, x, B, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(logits, m->z[kMlpLayers - 1], sizeof(float) * B, cudaMemcpyDeviceToDevice, st);
    return e == cudaSuccess ? LENIA_OK : mlp_fail(m, e, "forward");
}

// Loss and gradients of a batch (x: B x n_in, y: B targets in {0, 1}, both
// device) without updating the parameters; *loss_out (host) = mean BCE.
lenia_status lenia_mlp_gradients(lenia_mlp *m, const float *x, const float *y, int B, float *loss_out, void *stream)
{
    if (!m || !x || !y || B < 1) return LENIA_ERR_INVALID_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = ensure_batch(m, B);
    if (e == cudaSuccess) e = forward(m, x, B, st);
    if (e != cudaSuccess) return mlp_fail(m, e, "forward");
    k_bce<<<(B + 255) / 256, 256, 0, st>>>(m->z[kMlpLayers - 1], y, m->dz_out, m->dzb_out.p, m->dzb_out.ld,
                                           m->dzbt_out.p, m->rowloss, B);
    e = cudaGetLastError();
    for (int l = kMlpLayers - 1; l >= 0 && e == cudaSuccess; l--) {
        const int K = m->dims[l], N = m->dims[l + 1];
        const bool top = l == kMlpLayers - 1;
        const float *dz = top ? m->dz_out : m->dz[l & 1];
        const Bf16Mat &dzb = top ? m->dzb_out : m->dzb[l & 1];
        const Bf16Mat &dzbt = top ? m->dzbt_out : m->dzbt[l & 1];
        const Bf16Mat &inT = l == 0 ? m->xbt : m->abt[l - 1];
        // dW[n, k] = sum_b dz[b, n] in[b, k]: A = dz^T (N x B), B = in^T (K x B)
        TcGemm gw = epi(kEpiWeightGrad);
        gw.c32 = m->grads + m->woff[l];
        gw.ldc = K;
        gw.err = m->err;
        e = tc_gemm(dzbt, N, inT, K, B, gw, st, std::min(m->ksplit, std::max(1, B / 256)), m->ws);
        if (e == cudaSuccess) {
            k_colsum<<<(N + 255) / 256, 256, 0, st>>>(dz, B, N, m->grads + m->boff[l]);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && l > 0) {
            // dz_{l-1}[b, k] = (sum_n dz[b, n] W[n, k]) gelu'(z_{l-1}[b, k]):
            // A = dz (B x N), B = W^T (K x N)
            const int o = (l - 1) & 1;
            TcGemm ga = epi(kEpiActGrad);
            ga.c32 = m->dz[o];
            ga.ldc = K;
            ga.zin = m->z[l - 1];
            ga.ldz = K;
            ga.ob = m->dzb[o].p;
            ga.ldo = m->dzb[o].ld;
            ga.obt = m->dzbt[o].p;
            ga.ldot = m->dzbt[o].ld;
            ga.err = m->err;
            e = tc_gemm(dzb, B, m->wtb[l], K, N, ga, st);
        }
    }
    int err = 0;
    if (e == cudaSuccess) {
        k_sum<<<1, 256, 0, st>>>(m->rowloss, B, m->loss);
        float l = 0.0f;
        e = cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&err, m->err, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (loss_out) *loss_out = l / (float)B;
    }
    if (e == cudaSuccess && err) {
        m->err_msg = "a tensor-core product timed out waiting for its operands";
        cudaMemsetAsync(m->err, 0, sizeof(int), st);
        return LENIA_ERR_TIMEOUT;
    }
    return e == cudaSuccess ? LENIA_OK : mlp_fail(m, e, "backward");
}

// One Adam step (beta1 0.9, beta2 0.999, eps 1e-8, decoupled weight decay wd)
// on a batch; *loss_out (host, optional) = the batch's mean BCE before the step.
lenia_status lenia_mlp_train_step(lenia_mlp *m, const float *x, const float *y, int B, float lr, float wd,
                                  float *loss_out, void *stream)
{
    lenia_status s = lenia_mlp_gradients(m, x, y, B, loss_out, stream);
    if (s != LENIA_OK) return s;
    m->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)m->step), c2 = 1.0f - powf(b2, (float)m->step);
    cudaStream_t st = (cudaStream_t)stream;
    k_adam<<<blocks_for(m->nparams), 256, 0, st>>>(m->params, m->grads, m->m1, m->m2, m->nparams, lr, b1, b2, 1e-8f,
                                                   c1, c2, wd);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = refresh_weights(m, st);
    return e == cudaSuccess ? LENIA_OK : mlp_fail(m, e, "adam");
}

const char *lenia_mlp_last_error(const lenia_mlp *m) { return m ? m->err_msg.c_str() : "null mlp"; }

}  // extern "C"
