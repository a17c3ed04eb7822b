/*
 * Host shim used only to compile the reference's kernel headers
 * (gpuFunctions_undir.cuh) as plain C++ for the oracle/_ref harness.
 * Kernel qualifiers vanish and the launch geometry is one thread, so every
 * grid-stride loop in the reference runs serially in index order.
 */
#ifndef DYNCOLOR_REF_SHIM_CUDA_RUNTIME_H
#define DYNCOLOR_REF_SHIM_CUDA_RUNTIME_H
#define __global__
#define __device__
#define __host__
struct dc_shim_dim3 {
  unsigned x, y, z;
};
static dc_shim_dim3 threadIdx = {0, 0, 0};
static dc_shim_dim3 blockIdx = {0, 0, 0};
static dc_shim_dim3 blockDim = {1, 1, 1};
static dc_shim_dim3 gridDim = {1, 1, 1};
#endif
