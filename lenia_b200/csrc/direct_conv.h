// Direct convolution of the growth stage on the tcgen05 tensor cores
// (kernels_direct.cu): the plan of one world and its launches.
#pragma once

#include <cuda_runtime.h>

#include "lenia_internal.h"

namespace lenia {

struct DirectConv;

// Plan for a world's grid and kernels in mode LENIA_CONV_DIRECT_BF16 or
// LENIA_CONV_DIRECT_BF16X3 (allocates its buffers; synchronous).
cudaError_t direct_create(const Dims &d, int C, const LeniaKernelParams *kernels, int K, int mode, DirectConv **out);
void direct_destroy(DirectConv *dc);
// Kernel strips from the normalised kernel grids (K x N floats); synchronous.
cudaError_t direct_build(DirectConv *dc, const float *grids, cudaStream_t st);
// Padded BF16 (hi, lo) copy of the grid A (C x N floats).
cudaError_t direct_pad(DirectConv *dc, const float *A, cudaStream_t st);
// u_k of every kernel into U (K x N floats) from the padded copy.
cudaError_t direct_convolve(DirectConv *dc, float *U, int *err, cudaStream_t st);
// Tensor multiply-adds issued per convolution, and the useful ones (nonzero
// taps x cells x products per tap).
void direct_counts(const DirectConv *dc, double *issued_macs, double *useful_macs);
size_t direct_smem(const DirectConv *dc);
int direct_stages(const DirectConv *dc);
int direct_radius(const DirectConv *dc);

// Growth accumulation from stored u_k (H, U_SUM, BACK), per cell.
cudaError_t launch_growth_from_u(const Dims &d, const GrowthJobs &jobs, const float *lut_rows, const float *U,
                                 const float *A, float *H, float *U_SUM, float *BACK, int *err_flag, cudaStream_t st);

}  // namespace lenia
