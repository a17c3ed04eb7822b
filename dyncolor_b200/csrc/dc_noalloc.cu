// dc_noalloc.cu -- colouring validation that allocates no memory.
//
// Some callers cannot let a library call cudaMalloc: a serving process whose
// device memory is fully budgeted to resident graphs, an application whose
// own allocator (for example PyTorch's caching allocator) owns every device
// byte, or code that must not introduce the implicit device synchronisation
// cudaMalloc/cudaFree can cause.  dc_validate_csr_noalloc serves them: it
// checks a colouring of a CSR the caller already holds in device memory and
// keeps its scratch (result counters and a bitmap of conflicted vertices) in
// the file-scope device array below, which every GPU that loads the library
// holds until the process exits.
#include <algorithm>

#include "../../include/dyncolor.h"
#include "dc_device.cuh"

namespace dc {

namespace {

// Scratch layout (32-bit words):
//   [0..1]  monochromatic edges (u64)
//   [2..3]  conflicted vertices (u64)
//   [4]     max colour
//   [5]     error flags (1: negative colour, 2: neighbour id outside [0,n))
//   [16..)  one bit per vertex: "has a monochromatic edge"
constexpr int kHeaderWords = 16;
constexpr long long kNoAllocMaxVertices = 1ll << 24;  // 16,777,216 vertices: a 2 MiB bitmap
constexpr long long kScratchWords = kHeaderWords + kNoAllocMaxVertices / 32;

static __device__ __align__(256) unsigned int g_noalloc_scratch[kScratchWords];

constexpr int kNoAllocThreads = 256;

__global__ void noalloc_clear_kernel(unsigned int* scratch, long long words) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < words;
       i += (long long)gridDim.x * blockDim.x)
    scratch[i] = 0u;
}

// validate (HI/gpuFunctions_undir.cuh:289-305) over a caller-owned CSR: one
// warp per row, counting each monochromatic edge once (u > v).
__global__ void noalloc_validate_kernel(int n, const long long* off, const int* len, const int* adj,
                                        const int* color, unsigned int* scratch) {
  unsigned long long* edges = reinterpret_cast<unsigned long long*>(scratch);
  unsigned long long* verts = reinterpret_cast<unsigned long long*>(scratch + 2);
  unsigned int* bits = scratch + kHeaderWords;
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  long long bad = 0, newly = 0;
  int cmax = 0;
  unsigned err = 0;
  for (long long v = gw; v < n; v += nw) {
    const int cv = color[v];
    if (cv < 0) err |= 1u;
    cmax = max(cmax, cv);
    const long long o = off[v];
    const int L = len[v];
    for (int s = lane_id(); s < L; s += 32) {
      const int u = adj[o + s];
      if (u < 0) continue;  // tombstone
      if (u >= n) {
        err |= 2u;
        continue;
      }
      if (u > v && color[u] == cv) {
        ++bad;
        const unsigned bu = 1u << (u & 31), bv = 1u << (v & 31);
        if (!(atomicOr(&bits[u >> 5], bu) & bu)) ++newly;
        if (!(atomicOr(&bits[v >> 5], bv) & bv)) ++newly;
      }
    }
  }
  bad = warp_sum_ll(bad);
  newly = warp_sum_ll(newly);
  cmax = __reduce_max_sync(0xffffffffu, cmax);
  err = __reduce_or_sync(0xffffffffu, err);
  if (lane_id() == 0) {
    if (bad) atomicAdd(edges, (unsigned long long)bad);
    if (newly) atomicAdd(verts, (unsigned long long)newly);
    atomicMax(reinterpret_cast<int*>(scratch + 4), cmax);
    if (err) atomicOr(scratch + 5, err);
  }
}

}  // namespace

}  // namespace dc

extern "C" dc_status dc_validate_csr_noalloc(int32_t n, const int64_t* d_row_off, const int32_t* d_row_len,
                                             const int32_t* d_adj, const int32_t* d_colors, void* stream,
                                             int64_t* conflicts, int64_t* conflicted_vertices,
                                             int32_t* max_color) {
  using namespace dc;
  if (n < 0 || n > kNoAllocMaxVertices) return DC_E_INVAL;  // bitmap holds 2^24 vertices
  if (!conflicts || (n > 0 && (!d_row_off || !d_row_len || !d_adj || !d_colors))) return DC_E_INVAL;
  cudaGetLastError();  // an error left by the caller's own earlier work is not this call's
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The call waits for its stream at the end, which a capturing stream does
  // not allow.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
    cudaGetLastError();
    return DC_E_CUDA;
  }
  if (cap != cudaStreamCaptureStatusNone) return DC_E_STATE;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                 cudaSuccess) {
    cudaGetLastError();
    return DC_E_CUDA;
  }
  // The device address of the scratch array, looked up on every call with
  // the caller's device current.  In host code the array's name is only a
  // host-side stand-in and must never be handed to a kernel; and an address
  // kept from an earlier call could belong to a module that a device reset
  // has since unloaded, so none is kept.  The lookup allocates nothing.
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
    cudaGetLastError();
    return DC_E_CUDA;
  }
  unsigned int* scratch = static_cast<unsigned int*>(p);
  // The array keeps the previous call's contents: clear the header and the
  // bitmap words this call uses.
  const long long words = kHeaderWords + ((long long)n + 31) / 32;
  const int cgrid = (int)std::min<long long>((words + kNoAllocThreads - 1) / kNoAllocThreads, 1024);
  noalloc_clear_kernel<<<cgrid, kNoAllocThreads, 0, s>>>(scratch, words);
  if (n > 0) {
    const long long per_sm = 2048 / kNoAllocThreads;  // resident blocks of 256 threads per SM
    const int vgrid = (int)std::min<long long>(((long long)n * 32 + kNoAllocThreads - 1) / kNoAllocThreads,
                                               (long long)std::max(sms, 1) * per_sm);
    noalloc_validate_kernel<<<vgrid, kNoAllocThreads, 0, s>>>(
        n, reinterpret_cast<const long long*>(d_row_off), d_row_len, d_adj, d_colors, scratch);
  }
  if (cudaGetLastError() != cudaSuccess) return DC_E_CUDA;
  unsigned int head[6];
  if (cudaMemcpyAsync(head, scratch, sizeof(head), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return DC_E_CUDA;
  }
  if (head[5] != 0u) return DC_E_INVAL;  // negative colour or neighbour id outside [0, n)
  *conflicts = (int64_t)(((unsigned long long)head[1] << 32) | head[0]);
  if (conflicted_vertices) *conflicted_vertices = (int64_t)(((unsigned long long)head[3] << 32) | head[2]);
  if (max_color) *max_color = (int32_t)head[4];
  return DC_OK;
}
