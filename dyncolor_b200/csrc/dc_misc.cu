// dc_misc.cu -- validation, colour bound and adjacency repacking kernels.
#include "dc_device.cuh"

namespace dc {

namespace {

constexpr int kMiscThreads = 256;

// validate (HI/gpuFunctions_undir.cuh:289-305): live edges {u,v}, u<v, with
// equal colours; one warp per row instead of one thread for the graph.
__global__ void validate_kernel(GraphDev g, unsigned long long* out) {
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  long long bad = 0;
  for (long long v = gw; v < g.n; v += nw) {
    const long long o = g.off[v];
    const int L = g.len[v];
    const int cv = g.color[v];
    for (int s = lane_id(); s < L; s += 32) {
      const int u = g.adj[o + s];
      if (u > v && g.color[u] == cv) ++bad;
    }
  }
  bad = warp_sum_ll(bad);
  if (lane_id() == 0 && bad) atomicAdd(out, (unsigned long long)bad);
}

__global__ void color_max_kernel(GraphDev g, DevState* st) {
  int m = 0;
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < g.n;
       v += (long long)gridDim.x * blockDim.x)
    m = max(m, g.color[v]);
  m = __reduce_max_sync(0xffffffffu, m);
  if (lane_id() == 0) atomicMax(&st->cmax, m);
}

__global__ void count_live_kernel(GraphDev g, unsigned long long* out) {
  long long s = 0;
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < g.n;
       v += (long long)gridDim.x * blockDim.x)
    s += g.live[v];
  s = warp_sum_ll(s);
  if (lane_id() == 0 && s) atomicAdd(out, (unsigned long long)s);
}

__global__ void color_unmark_kernel(GraphDev g) {
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < g.n;
       v += (long long)gridDim.x * blockDim.x)
    g.color[v] &= kColorMask;
}

// gid[v] = graph of v (first[] ascending, first[0] = 0, first[ngraphs] = n),
// then the number of live adjacency entries joining two graphs.
__global__ void partition_gid_kernel(GraphDev g, const int* first, int ngraphs, int* gid) {
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < g.n;
       v += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = ngraphs;  // largest j with first[j] <= v
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (first[mid] <= v) lo = mid; else hi = mid;
    }
    gid[v] = lo;
  }
}

__global__ void partition_cross_kernel(GraphDev g, const int* gid, unsigned long long* cross) {
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  long long bad = 0;
  for (long long v = gw; v < g.n; v += nw) {
    const long long o = g.off[v];
    const int L = g.len[v];
    const int gv = gid[v];
    for (int s = lane_id(); s < L; s += 32) {
      const int u = g.adj[o + s];
      if (u >= 0 && gid[u] != gv) ++bad;
    }
  }
  bad = warp_sum_ll(bad);
  if (lane_id() == 0 && bad) atomicAdd(cross, (unsigned long long)bad);
}

__device__ __forceinline__ long long packed_cap(int live, float slack) {
  if (live <= 0) return 0;
  long long want = (long long)ceilf((float)live * slack);
  if (want < (long long)live + 4) want = (long long)live + 4;
  return (want + 3) & ~3ll;
}

// repack step 1: per-block sums of the new capacities
__global__ void repack_caps_kernel(GraphDev g, float slack, long long* bsum) {
  __shared__ long long sw[kMiscThreads / 32];
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long c = v < g.n ? packed_cap(g.live[v], slack) : 0;
  c = warp_sum_ll(c);
  if (lane_id() == 0) sw[warp_id()] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int i = 0; i < kMiscThreads / 32; ++i) t += sw[i];
    bsum[blockIdx.x] = t;
  }
}

// repack step 2: exclusive scan of the block sums (one CTA, sequential chunks)
__global__ void repack_scan_kernel(long long* bsum, long long nb, unsigned long long* used) {
  __shared__ long long sw[kMiscThreads / 32 + 1];
  long long run = 0;
  for (long long c0 = 0; c0 < nb; c0 += kMiscThreads) {
    const long long i = c0 + threadIdx.x;
    const long long x = i < nb ? bsum[i] : 0;
    long long incl = x;
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane_id() >= o) incl += y;
    }
    if (lane_id() == 31) sw[warp_id()] = incl;
    __syncthreads();
    long long wbase = 0, tot = 0;
    for (int w = 0; w < kMiscThreads / 32; ++w) {
      if (w < warp_id()) wbase += sw[w];
      tot += sw[w];
    }
    if (i < nb) bsum[i] = run + wbase + incl - x;
    __syncthreads();
    run += tot;
  }
  if (threadIdx.x == 0) *used = (unsigned long long)run;
}

// repack step 3: per-vertex offsets
__global__ void repack_offsets_kernel(GraphDev g, float slack, const long long* bsum, long long* off2,
                                      int* cap2) {
  __shared__ long long sw[kMiscThreads / 32];
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long c = v < g.n ? packed_cap(g.live[v], slack) : 0;
  long long incl = c;
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane_id() >= o) incl += y;
  }
  if (lane_id() == 31) sw[warp_id()] = incl;
  __syncthreads();
  long long wbase = 0;
  for (int w = 0; w < warp_id(); ++w) wbase += sw[w];
  if (v < g.n) {
    off2[v] = bsum[blockIdx.x] + wbase + incl - c;
    cap2[v] = (int)c;
  }
}

// repack step 4: order-preserving copy of the live slots, one warp per row;
// the new row lengths go to len2 so the old layout stays whole until the swap
__global__ void repack_copy_kernel(GraphDev g, const long long* off2, int* len2, int* adj2, long long cap_slots,
                                   unsigned* status) {
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long v = gw; v < g.n; v += nw) {
    const long long o = g.off[v];
    const int L = g.len[v];
    const long long no = off2[v];
    int cur = 0;
    for (int s0 = 0; s0 < L; s0 += 32) {
      const int s = s0 + lane_id();
      const int x = s < L ? g.adj[o + s] : kTomb;
      const unsigned bal = __ballot_sync(0xffffffffu, x >= 0);
      if (x >= 0) {
        const long long pos = no + cur + __popc(bal & lanemask_lt());
        if (pos < cap_slots)
          adj2[pos] = x;
        else
          atomicOr(status, ST_OVERFLOW);
      }
      cur += __popc(bal);
    }
    __syncwarp();
    if (lane_id() == 0) len2[v] = cur;
  }
}

// Resident pool: rows of vertices [v0, v0 + nv) copied out in row order
// (tombstones dropped, ids made local by subtracting `base`); row i's live
// entries land at out[pre[i] ..).  One warp per row.
__global__ void range_gather_kernel(GraphDev g, int base, int v0, int nv, const long long* pre, int* out) {
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long i = gw; i < nv; i += nw) {
    const long long v = v0 + i;
    const long long o = g.off[v];
    const int L = g.len[v];
    int* dst = out + pre[i];
    const long long room = pre[i + 1] - pre[i];  // live[v] as the host read it
    int cur = 0;
    for (int s0 = 0; s0 < L; s0 += 32) {
      const int s = s0 + lane_id();
      const int x = s < L ? g.adj[o + s] : kTomb;
      const unsigned bal = __ballot_sync(0xffffffffu, x >= 0);
      const int at = cur + __popc(bal & lanemask_lt());
      if (x >= 0 && at < room) dst[at] = x - base;
      cur += __popc(bal);
    }
  }
}

// The inverse: row i (vertex v0 + i, whose off/len were already written)
// takes in[pre[i] .. pre[i] + len) with `base` added to every id.
__global__ void range_scatter_kernel(GraphDev g, int base, int v0, int nv, const long long* pre, const int* in) {
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long i = gw; i < nv; i += nw) {
    const long long v = v0 + i;
    const long long o = g.off[v];
    const int L = g.len[v];
    const int* src = in + pre[i];
    for (int s = lane_id(); s < L; s += 32) g.adj[o + s] = src[s] + base;
  }
}

__global__ void fill_kernel(int* p, long long count, int value) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x)
    p[i] = value;
}

}  // namespace

static int misc_grid(long long work, int per_block) {
  long long b = (work + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return (int)b;
}

cudaError_t launch_validate(const GraphDev& g, unsigned long long* out, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  validate_kernel<<<misc_grid((long long)g.n * 32, kMiscThreads), kMiscThreads, 0, s>>>(g, out);
  return cudaGetLastError();
}

cudaError_t launch_color_max(const GraphDev& g, DevState* st, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(&st->cmax, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  color_max_kernel<<<misc_grid(g.n, kMiscThreads), kMiscThreads, 0, s>>>(g, st);
  return cudaGetLastError();
}

cudaError_t launch_count_live(const GraphDev& g, unsigned long long* out, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  count_live_kernel<<<misc_grid(g.n, kMiscThreads), kMiscThreads, 0, s>>>(g, out);
  return cudaGetLastError();
}

cudaError_t launch_color_unmark(const GraphDev& g, cudaStream_t s) {
  color_unmark_kernel<<<misc_grid(g.n, kMiscThreads), kMiscThreads, 0, s>>>(g);
  return cudaGetLastError();
}

cudaError_t launch_partition(const GraphDev& g, const int* first, int ngraphs, int* gid,
                             unsigned long long* cross, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(cross, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  partition_gid_kernel<<<misc_grid(g.n, kMiscThreads), kMiscThreads, 0, s>>>(g, first, ngraphs, gid);
  partition_cross_kernel<<<misc_grid((long long)g.n * 32, kMiscThreads), kMiscThreads, 0, s>>>(g, gid, cross);
  return cudaGetLastError();
}

// scratch must hold ceil(n / 256) + 1 long longs.  Steps 1-2: per-block
// offsets in scratch and the packed total in *total.
cudaError_t launch_packed_total(const GraphDev& g, float slack, long long* scratch, unsigned long long* total,
                                cudaStream_t s) {
  const long long nb = ((long long)g.n + kMiscThreads - 1) / kMiscThreads;
  if (nb == 0) return cudaMemsetAsync(total, 0, sizeof(unsigned long long), s);
  repack_caps_kernel<<<(unsigned)nb, kMiscThreads, 0, s>>>(g, slack, scratch);
  repack_scan_kernel<<<1, kMiscThreads, 0, s>>>(scratch, nb, total);
  return cudaGetLastError();
}

// Steps 3-4 with the scratch of launch_packed_total.
cudaError_t launch_repack_copy(const GraphDev& g, float slack, const long long* scratch, long long* off2, int* cap2,
                               int* len2, int* adj2, long long cap_slots, unsigned* status, cudaStream_t s) {
  const long long nb = ((long long)g.n + kMiscThreads - 1) / kMiscThreads;
  if (nb == 0) return cudaSuccess;
  repack_offsets_kernel<<<(unsigned)nb, kMiscThreads, 0, s>>>(g, slack, scratch, off2, cap2);
  repack_copy_kernel<<<misc_grid((long long)g.n * 32, kMiscThreads), kMiscThreads, 0, s>>>(
      g, off2, len2, adj2, cap_slots, status);
  return cudaGetLastError();
}

cudaError_t launch_range_gather(const GraphDev& g, int base, int v0, int nv, const long long* pre, int* out,
                                cudaStream_t s) {
  if (nv <= 0) return cudaSuccess;
  range_gather_kernel<<<misc_grid((long long)nv * 32, kMiscThreads), kMiscThreads, 0, s>>>(g, base, v0, nv, pre, out);
  return cudaGetLastError();
}

cudaError_t launch_range_scatter(const GraphDev& g, int base, int v0, int nv, const long long* pre, const int* in,
                                 cudaStream_t s) {
  if (nv <= 0) return cudaSuccess;
  range_scatter_kernel<<<misc_grid((long long)nv * 32, kMiscThreads), kMiscThreads, 0, s>>>(g, base, v0, nv, pre, in);
  return cudaGetLastError();
}

cudaError_t launch_fill(int* p, long long count, int value, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  fill_kernel<<<misc_grid(count, kMiscThreads), kMiscThreads, 0, s>>>(p, count, value);
  return cudaGetLastError();
}

}  // namespace dc
