// dc_device.cuh -- device helpers shared by the persistent kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "dc_internal.h"

namespace dc {

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ int warp_id() { return threadIdx.x >> 5; }

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned ld_volatile_u32(const unsigned* p) {
  return *reinterpret_cast<const volatile unsigned*>(p);
}

template <class T>
__device__ __forceinline__ T ld_cg(const T* p) {
  return __ldcg(p);
}

// Software grid barrier for a cooperative (all-CTAs-resident) launch.
// `target` is per-CTA state starting at 0.  Every wait is bounded by
// `timeout_ns` of globaltimer; on expiry the CTA raises ST_TIMEOUT and the
// abort flag, and every CTA then returns false from its next wait so the
// kernel exits instead of hanging.
__device__ __forceinline__ bool grid_sync(DevState* st, unsigned& target, unsigned long long timeout_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    target += gridDim.x;
    __threadfence();
    atomicAdd(&st->bar_arrived, 1u);
    int ok = 1;
    const unsigned long long t0 = globaltimer_ns();
    unsigned spins = 0;
    while (true) {
      const unsigned a = ld_acquire_u32(&st->bar_arrived);
      if ((int)(a - target) >= 0) break;
      if (ld_volatile_u32(&st->bar_abort)) {
        ok = 0;
        break;
      }
      if ((++spins & 255u) == 0 && globaltimer_ns() - t0 > timeout_ns) {
        atomicOr(&st->status, ST_TIMEOUT);
        atomicExch(&st->bar_abort, 1u);
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ int warp_incl_scan(int x) {
  const int lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

__device__ __forceinline__ long long warp_sum_ll(long long x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// Block-wide exclusive scan of one int per thread (blockDim.x == kThreads).
// `sw` is shared scratch of kWarps+1 ints.  Returns the exclusive prefix and
// the block total in *total.
__device__ __forceinline__ int block_excl_scan(int v, int* sw, int* total) {
  const int lane = lane_id(), w = warp_id();
  const int incl = warp_incl_scan(v);
  if (lane == 31) sw[w] = incl;
  __syncthreads();
  if (w == 0) {
    int s = lane < kWarps ? sw[lane] : 0;
    s = warp_incl_scan(s);
    if (lane < kWarps) sw[lane] = s;
  }
  __syncthreads();
  const int base = w > 0 ? sw[w - 1] : 0;
  *total = sw[kWarps - 1];
  __syncthreads();
  return base + incl - v;
}

__device__ __forceinline__ long long block_sum_ll(long long v, long long* sw) {
  v = warp_sum_ll(v);
  if (lane_id() == 0) sw[warp_id()] = v;
  __syncthreads();
  long long t = 0;
  for (int i = 0; i < kWarps; ++i) t += sw[i];
  __syncthreads();
  return t;
}

// Warp-aggregated atomicAdd of `val` (per lane, may be 0) on a 64-bit
// counter.  All 32 lanes must call.  Returns this lane's exclusive base.
__device__ __forceinline__ unsigned long long warp_atomic_add(unsigned long long* ctr, int val) {
  const int incl = warp_incl_scan(val);
  const int tot = __shfl_sync(0xffffffffu, incl, 31);
  unsigned long long base = 0;
  if (tot > 0 && lane_id() == 31) base = atomicAdd(ctr, (unsigned long long)tot);
  base = __shfl_sync(0xffffffffu, base, 31);
  return base + (unsigned long long)(incl - val);
}

// Marks bit v in a bitmap; returns true for the call that set it.
__device__ __forceinline__ bool mark_bit(unsigned* bm, int v) {
  const unsigned bit = 1u << (v & 31);
  unsigned* w = bm + (v >> 5);
  if (ld_cg(w) & bit) return false;
  const unsigned old = atomicOr(w, bit);
  return (old & bit) == 0;
}

// LDF priority, HB/gpuFunctions_undir.cuh:104-113: a is prior to b when its
// degree property is larger, ties broken by the lower vertex id.
__device__ __forceinline__ bool is_prior(int pa, int a, int pb, int b) {
  return pa > pb || (pa == pb && a < b);
}

// Key of one directed change entry: row, neighbour, op (0 delete, 1 insert).
__device__ __forceinline__ unsigned long long make_key(int row, int nbr, int op, int B) {
  return ((unsigned long long)row << (B + 1)) | ((unsigned long long)nbr << 1) |
         (unsigned long long)op;
}
__device__ __forceinline__ int key_row(unsigned long long k, int B) { return (int)(k >> (B + 1)); }
__device__ __forceinline__ int key_nbr(unsigned long long k, int B) {
  return (int)((k >> 1) & ((1ull << B) - 1));
}
__device__ __forceinline__ int key_op(unsigned long long k) { return (int)(k & 1ull); }

}  // namespace dc
