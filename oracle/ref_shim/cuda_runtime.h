/*
 * Host shim used only to compile the reference's kernel headers
 * (gpuFunctions_undir.cuh) as plain C++ for the oracle/_ref harness.
 * Kernel qualifiers vanish.  By default the launch geometry is one thread, so
 * every grid-stride loop in the reference runs serially in index order.  The
 * harness's timing mode "launches" a kernel on T host threads by calling it
 * from every thread of an OpenMP team with blockDim.x = T and threadIdx.x
 * the thread's number: the grid-stride loops then split their items over
 * the threads, which race on the shared arrays as the reference's GPU
 * threads do.
 */
#ifndef DYNCOLOR_REF_SHIM_CUDA_RUNTIME_H
#define DYNCOLOR_REF_SHIM_CUDA_RUNTIME_H
#define __global__
#define __device__
#define __host__
struct dc_shim_dim3 {
  unsigned x, y, z;
};
static thread_local dc_shim_dim3 threadIdx = {0, 0, 0};
static dc_shim_dim3 blockIdx = {0, 0, 0};
static dc_shim_dim3 blockDim = {1, 1, 1};
static dc_shim_dim3 gridDim = {1, 1, 1};
#endif
