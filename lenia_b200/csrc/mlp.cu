// A small multilayer perceptron trained on the GPU by this file's own
// kernels: the proposal network of the persistent-pattern search (no
// counterpart in the reference).
//
//   n_in -> hidden -> hidden -> hidden -> 1, GELU (0.5 x (1 + erf(x / sqrt 2)))
//   after every hidden layer, a logit out; binary cross-entropy on the logit.
//
// Precision: weights and activations enter every matrix product rounded to
// bfloat16 (round to nearest even); products accumulate in float32; biases,
// pre-activations, gradients and the Adam state are float32, and the Adam
// update runs on float32 master weights.
//
// Kernels: one tiled matrix product with strides (so that the forward
// product, both backward products and their transposes share it), a fused
// bias + GELU epilogue, the loss with its gradient, the GELU derivative,
// column sums for the bias gradients, and Adam.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <random>
#include <string>
#include <vector>

#include "lenia_internal.h"

namespace {

constexpr int kTile = 64;    // output tile of the product (64 x 64)
constexpr int kTileK = 16;   // reduction step staged in shared memory
constexpr int kMlpLayers = 4;

__device__ __forceinline__ float to_bf16(float x)
{
    // round to nearest even at bit 16; NaN stays NaN
    unsigned u = __float_as_uint(x);
    if ((u & 0x7f800000u) == 0x7f800000u) return x;
    u += 0x7fffu + ((u >> 16) & 1u);
    return __uint_as_float(u & 0xffff0000u);
}

// C[m, n] (+)= sum_k A(m, k) B(n, k) (+ bias[n]), with A(m, k) = A[m sam + k sak]
// and B(n, k) = B[n sbn + k sbk]; operands optionally rounded to bfloat16 as
// they are staged.  256 threads, each computing 4 x 4 outputs of a 64 x 64
// tile; the sum over k runs in increasing k.
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, const float *__restrict__ A, long long sam,
                                              long long sak, const float *__restrict__ B, long long sbn,
                                              long long sbk, float *__restrict__ C, long long scm, long long scn,
                                              const float *__restrict__ bias, int round_a, int round_b, int accumulate)
{
    __shared__ float sa[kTileK][kTile + 1];
    __shared__ float sb[kTileK][kTile + 1];
    const int m0 = blockIdx.y * kTile, n0 = blockIdx.x * kTile;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += kTileK) {
        for (int e = threadIdx.x; e < kTileK * kTile; e += 256) {
            const int kk = e / kTile, r = e % kTile;
            const int k = k0 + kk;
            float a = 0.0f, b = 0.0f;
            if (m0 + r < M && k < K) {
                a = A[(long long)(m0 + r) * sam + (long long)k * sak];
                if (round_a) a = to_bf16(a);
            }
            if (n0 + r < N && k < K) {
                b = B[(long long)(n0 + r) * sbn + (long long)k * sbk];
                if (round_b) b = to_bf16(b);
            }
            sa[kk][r] = a;
            sb[kk][r] = b;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kTileK; kk++) {
            float av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; i++) av[i] = sa[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; j++) bv[j] = sb[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int m = m0 + ty * 4 + i, n = n0 + tx * 4 + j;
            if (m >= M || n >= N) continue;
            float v = acc[i][j];
            if (bias) v += bias[n];
            float *c = C + (long long)m * scm + (long long)n * scn;
            *c = accumulate ? *c + v : v;
        }
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float z)
{
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

__global__ void k_gelu(const float *__restrict__ z, float *__restrict__ a, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[i] = gelu(z[i]);
}

// dz = da * gelu'(z)
__global__ void k_gelu_back(const float *__restrict__ z, const float *__restrict__ da, float *__restrict__ dz,
                            long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dz[i] = da[i] * gelu_grad(z[i]);
}

// Binary cross-entropy on logits, mean over the batch: per-row loss into
// rowloss, gradient (sigmoid(z) - y) / B into dz.
__global__ void k_bce(const float *__restrict__ z, const float *__restrict__ y, float *__restrict__ dz,
                      float *__restrict__ rowloss, int B)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B) return;
    const float zi = z[i], yi = y[i];
    const float s = 1.0f / (1.0f + expf(-zi));
    // log(1 + e^-|z|) + max(z, 0) - z y
    rowloss[i] = log1pf(expf(-fabsf(zi))) + fmaxf(zi, 0.0f) - zi * yi;
    dz[i] = (s - yi) / (float)B;
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
    float *z[kMlpLayers] = {}, *a[kMlpLayers] = {};  // pre-activations, activations per layer
    float *dz = nullptr, *da = nullptr, *rowloss = nullptr, *loss = nullptr;
    int cap = 0;                         // batch capacity of the activation buffers
    long long step = 0;
    std::string err;
};

namespace {

lenia_status mlp_fail(lenia_mlp *m, cudaError_t e, const char *where)
{
    if (m) m->err = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? LENIA_ERR_OOM : LENIA_ERR_CUDA;
}

void free_acts(lenia_mlp *m)
{
    for (int l = 0; l < kMlpLayers; l++) {
        if (m->z[l]) cudaFree(m->z[l]);
        if (m->a[l]) cudaFree(m->a[l]);
        m->z[l] = m->a[l] = nullptr;
    }
    float **bufs[] = {&m->dz, &m->da, &m->rowloss};
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
    cudaError_t e = cudaSuccess;
    int widest = 0;
    for (int l = 0; l <= kMlpLayers; l++) widest = m->dims[l] > widest ? m->dims[l] : widest;
    for (int l = 0; l < kMlpLayers && e == cudaSuccess; l++) {
        e = cudaMalloc((void **)&m->z[l], sizeof(float) * (size_t)B * m->dims[l + 1]);
        if (e == cudaSuccess) e = cudaMalloc((void **)&m->a[l], sizeof(float) * (size_t)B * m->dims[l + 1]);
    }
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->dz, sizeof(float) * (size_t)B * widest);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->da, sizeof(float) * (size_t)B * widest);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->rowloss, sizeof(float) * (size_t)B);
    if (e == cudaSuccess) m->cap = B;
    return e;
}

// C[M x N] = X[M x K] W^T + b (row-major X, W[N x K]), operands rounded to bf16.
cudaError_t gemm_forward(const float *X, const float *Wt, const float *b, float *C, int M, int N, int K,
                         cudaStream_t st)
{
    dim3 grid((N + kTile - 1) / kTile, (M + kTile - 1) / kTile);
    k_gemm<<<grid, 256, 0, st>>>(M, N, K, X, K, 1, Wt, K, 1, C, N, 1, b, 1, 1, 0);
    return cudaGetLastError();
}

cudaError_t forward(lenia_mlp *m, const float *x, int B, cudaStream_t st)
{
    cudaError_t e = cudaSuccess;
    const float *in = x;
    for (int l = 0; l < kMlpLayers && e == cudaSuccess; l++) {
        const int K = m->dims[l], N = m->dims[l + 1];
        e = gemm_forward(in, m->params + m->woff[l], m->params + m->boff[l], m->z[l], B, N, K, st);
        if (e != cudaSuccess) break;
        if (l + 1 < kMlpLayers) {
            const long long n = (long long)B * N;
            k_gelu<<<blocks_for(n), 256, 0, st>>>(m->z[l], m->a[l], n);
            e = cudaGetLastError();
            in = m->a[l];
        }
    }
    return e;
}

}  // namespace

extern "C" {

lenia_status lenia_mlp_create(int n_in, int hidden, unsigned long long seed, lenia_mlp **out)
{
    if (!out || n_in < 1 || hidden < 1) return LENIA_ERR_INVALID_ARG;
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
    if (e == cudaSuccess) e = cudaMemcpy(m->params, init.data(), sizeof(float) * off, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m->grads, 0, sizeof(float) * off);
    if (e == cudaSuccess) e = cudaMemset(m->m1, 0, sizeof(float) * off);
    if (e == cudaSuccess) e = cudaMemset(m->m2, 0, sizeof(float) * off);
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
    float *bufs[] = {m->params, m->grads, m->m1, m->m2, m->loss};
    for (float *p : bufs)
        if (p) cudaFree(p);
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
    const cudaError_t e = cudaMemcpy(m->params, src, sizeof(float) * n, cudaMemcpyHostToDevice);
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
    k_bce<<<(B + 255) / 256, 256, 0, st>>>(m->z[kMlpLayers - 1], y, m->dz, m->rowloss, B);
    for (int l = kMlpLayers - 1; l >= 0 && e == cudaSuccess; l--) {
        const int K = m->dims[l], N = m->dims[l + 1];
        const float *in = l > 0 ? m->a[l - 1] : x;
        // dW[n, k] = sum_b dz[b, n] in[b, k]  (dz float, in rounded to bf16)
        dim3 gw((K + kTile - 1) / kTile, (N + kTile - 1) / kTile);
        k_gemm<<<gw, 256, 0, st>>>(N, K, B, m->dz, 1, N, in, 1, K, m->grads + m->woff[l], K, 1, nullptr, 0, 1, 0);
        k_colsum<<<(N + 255) / 256, 256, 0, st>>>(m->dz, B, N, m->grads + m->boff[l]);
        if (l > 0) {
            // da[b, k] = sum_n dz[b, n] W[n, k]  (W rounded to bf16), then through GELU
            dim3 gd((K + kTile - 1) / kTile, (B + kTile - 1) / kTile);
            k_gemm<<<gd, 256, 0, st>>>(B, K, N, m->dz, N, 1, m->params + m->woff[l], 1, K, m->da, K, 1, nullptr, 0, 1,
                                       0);
            const long long n = (long long)B * K;
            k_gelu_back<<<blocks_for(n), 256, 0, st>>>(m->z[l - 1], m->da, m->dz, n);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        k_sum<<<1, 256, 0, st>>>(m->rowloss, B, m->loss);
        float l = 0.0f;
        e = cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (loss_out) *loss_out = l / (float)B;
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
    k_adam<<<blocks_for(m->nparams), 256, 0, (cudaStream_t)stream>>>(m->params, m->grads, m->m1, m->m2, m->nparams, lr,
                                                                    b1, b2, 1e-8f, c1, c2, wd);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LENIA_OK : mlp_fail(m, e, "adam");
}

const char *lenia_mlp_last_error(const lenia_mlp *m) { return m ? m->err.c_str() : "null mlp"; }

}  // extern "C"
