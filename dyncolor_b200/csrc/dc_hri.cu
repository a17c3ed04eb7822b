// dc_hri.cu -- heavy-row index of the recolouring loop, rebuilt before
// every recolour launch (after the structural update of the batch).
//
//   count     rows with at least min_live live slots, per length class
//             floor(log2(live))
//   classify  those rows get an index i, longest class first (arrival
//             order within a class; the order never affects results), and
//             the changed-colour bitmap is cleared
//   offsets   one CTA: exclusive scans of the rows' live counts (ordered
//             copies) and of their change-list capacities; rows past the
//             buffers' capacity (the shortest) lose their index and are
//             scanned in full
//   fill (HI) one CTA per row: counting sort of the row's live neighbours
//             by colour, descending (colours >= kHriBins - 1 share the first
//             bin), written as (colour << 32) | neighbour; the first
//             cap_hist rows also keep their per-colour counts
//   split (HB) one CTA per row: the neighbours prior to the row's vertex in
//             LDF order first, then the rest, as 4-byte ids
#include "dc_device.cuh"

namespace dc {

namespace {

constexpr int kHriThreads = 512;

__device__ __forceinline__ int hri_bin(int c) { return c < kHriBins - 1 ? c : kHriBins - 1; }

// Change-list capacity of a row with `live` slots: a neighbour joins the
// list once per launch (at its first colour change), so it never overflows.
__device__ __forceinline__ long long xcap(int live) { return live; }

// Length class of a row with live >= 1 slots: floor(log2(live)).
__device__ __forceinline__ int len_class(int live) { return 31 - __clz(live); }

// Calls f(v) for every vertex the index covers: all of them, or those of
// h.ranges (one index space over the ranges, binary search for the range).
template <typename F>
__device__ __forceinline__ void for_each_vertex(const GraphDev& g, const HriBufs& h, F f) {
  const long long nt = (long long)gridDim.x * blockDim.x;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (!h.ranges) {
    for (long long v = t; v < g.n; v += nt) f((int)v);
    return;
  }
  const int cnt = h.ranges[0];
  const long long total = h.ranges[1];
  const int* r = h.ranges + 2;  // (first vertex, vertices before) per range
  for (long long x = t; x < total; x += nt) {
    int lo = 0, hi = cnt - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if ((long long)r[2 * mid + 1] <= x) lo = mid; else hi = mid - 1;
    }
    f(r[2 * lo] + (int)(x - r[2 * lo + 1]));
  }
}

// Rows with at least min_live live slots, counted per length class.
__global__ void hri_count_kernel(GraphDev g, HriBufs h) {
  __shared__ unsigned s_cnt[32];
  if (threadIdx.x < 32) s_cnt[threadIdx.x] = 0u;
  __syncthreads();
  for_each_vertex(g, h, [&](int v) {
    const int L = g.live[v];
    if (L >= h.min_live) atomicAdd(&s_cnt[len_class(L)], 1u);
  });
  __syncthreads();
  if (threadIdx.x < 32 && s_cnt[threadIdx.x] != 0u)
    atomicAdd(&h.bcnt[threadIdx.x], (unsigned long long)s_cnt[threadIdx.x]);
}

// Index i of every such row, class by class from the longest (so when the
// copies outgrow their buffer, the rows that lose their index are the
// shortest), in arrival order within a class; clears the changed-colour
// bitmap of the covered vertices.
__global__ void hri_classify_kernel(GraphDev g, HriBufs h, DevState* st) {
  __shared__ unsigned long long s_base[32];
  if (threadIdx.x < 32) {
    unsigned long long b = 0;
    for (int c = 31; c > (int)threadIdx.x; --c) b += h.bcnt[c];
    s_base[threadIdx.x] = b;
    if (blockIdx.x == 0 && threadIdx.x == 0) st->hcount = b + h.bcnt[0];
  }
  __syncthreads();
  for_each_vertex(g, h, [&](int v) {
    int id = -1;
    const int L = g.live[v];
    if (L >= h.min_live) {
      const int c = len_class(L);
      const unsigned long long i = s_base[c] + atomicAdd(&h.bcnt[32 + c], 1ull);
      if ((long long)i < h.cap_rows) {
        id = (int)i;
        h.hrow[i] = v;
      }
    }
    h.hid[v] = id;
    if (h.bmF && h.ranges) atomicAnd(&h.bmF[v >> 5], ~(1u << (v & 31)));
  });
  if (h.bmF && !h.ranges) {
    const long long nt = (long long)gridDim.x * blockDim.x;
    const long long words = ((long long)g.n + 31) / 32 + 1;
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += nt) h.bmF[w] = 0u;
  }
}

// Single CTA.  hoff / xoff get exclusive prefixes; rows whose copy or list
// would pass the buffers lose their index.
__global__ void hri_offsets_kernel(GraphDev g, HriBufs h, DevState* st) {
  __shared__ long long sw[kHriThreads / 32];
  __shared__ long long s_tot[2];
  const long long R = min((long long)ld_cg(&st->hcount), h.cap_rows);
  long long run_p = 0, run_x = 0;
  for (long long c0 = 0; c0 < R; c0 += kHriThreads) {
    const long long i = c0 + threadIdx.x;
    const int L = i < R ? g.live[h.hrow[i]] : 0;
    const long long xp = (i < R && h.xv) ? xcap(L) : 0;  // HB keeps no change lists
    // two block scans (pairs, list capacity)
    long long vals[2] = {(long long)L, xp};
    long long excl[2];
    for (int k = 0; k < 2; ++k) {
      long long incl = vals[k];
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane_id() >= o) incl += y;
      }
      if (lane_id() == 31) sw[warp_id()] = incl;
      __syncthreads();
      long long wbase = 0, tot = 0;
      for (int w = 0; w < kHriThreads / 32; ++w) {
        if (w < warp_id()) wbase += sw[w];
        tot += sw[w];
      }
      excl[k] = wbase + incl - vals[k];
      if (threadIdx.x == 0) s_tot[k] = tot;
      __syncthreads();
    }
    if (i < R) {
      const long long po = run_p + excl[0], xo = run_x + excl[1];
      h.hoff[i] = po;
      h.xoff[i] = xo;
      h.xcnt[i] = 0;
      if (po + L > h.cap_pairs || xo + xp > h.cap_exc) h.hid[h.hrow[i]] = -1;  // no room: full scans
    }
    run_p += s_tot[0];
    run_x += s_tot[1];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    h.hoff[R] = min(run_p, h.cap_pairs);
    h.xoff[R] = min(run_x, h.cap_exc);
  }
}

__global__ void __launch_bounds__(kHriThreads) hri_fill_kernel(GraphDev g, HriBufs h, DevState* st) {
  __shared__ int hist[kHriBins];
  __shared__ int sw[kHriThreads / 32 + 1];
  const long long R = min((long long)ld_cg(&st->hcount), h.cap_rows);
  for (long long i = blockIdx.x; i < R; i += gridDim.x) {
    const int v = h.hrow[i];
    if (h.hid[v] != (int)i) continue;  // lost its index in the offsets pass (uniform per CTA)
    const long long o = g.off[v];
    const int L = g.len[v];
    const long long base = h.hoff[i];
    const long long room = h.hoff[i + 1] - base;  // == live[v]
    for (int b = threadIdx.x; b < kHriBins; b += kHriThreads) hist[b] = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < L; s += kHriThreads) {
      const int u = g.adj[o + s];
      if (u >= 0) atomicAdd(&hist[hri_bin(g.color[u] & kColorMask)], 1);
    }
    __syncthreads();
    // the mex of the loop reads the per-colour counts of the first cap_hist rows
    if (i < h.cap_hist)
      for (int b = threadIdx.x; b < kHriBins; b += kHriThreads) h.hist[i * kHriBins + b] = hist[b];
    // descending bins: start of bin b = sum of the counts of bins above b.
    // Thread t owns bins [2t, 2t + 1] counted from the top.
    {
      const int b0 = kHriBins - 1 - 2 * threadIdx.x, b1 = b0 - 1;
      const int c0 = hist[b0], c1 = hist[b1];
      int incl = c0 + c1;
      for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane_id() >= off) incl += y;
      }
      if (lane_id() == 31) sw[warp_id()] = incl;
      __syncthreads();
      int wbase = 0;
      for (int w = 0; w < warp_id(); ++w) wbase += sw[w];
      const int start = wbase + incl - (c0 + c1);
      __syncthreads();
      hist[b0] = start;  // becomes the bin's write cursor
      hist[b1] = start + c0;
    }
    __syncthreads();
    for (int s = threadIdx.x; s < L; s += kHriThreads) {
      const int u = g.adj[o + s];
      if (u < 0) continue;
      const int c = g.color[u] & kColorMask;
      const int pos = atomicAdd(&hist[hri_bin(c)], 1);
      if (pos < room)
        h.pairs[base + pos] = ((unsigned long long)(unsigned)c << 32) | (unsigned)u;
      else
        atomicOr(&st->status, ST_OVERFLOW);
    }
    __syncthreads();
  }
}

static_assert(kHriBins == 2 * kHriThreads, "fill scan: two bins per thread");

// HB: one CTA per row: the row's live neighbours prior to v in LDF order
// (HB/gpuFunctions_undir.cuh:104-113) first, then the others.  The
// prior-filtered mex of v only needs the first part.
__global__ void __launch_bounds__(kHriThreads) hri_split_kernel(GraphDev g, HriBufs h, DevState* st) {
  __shared__ int s_cur[2];
  __shared__ int sw[kHriThreads / 32];
  const long long R = min((long long)ld_cg(&st->hcount), h.cap_rows);
  for (long long i = blockIdx.x; i < R; i += gridDim.x) {
    const int v = h.hrow[i];
    if (h.hid[v] != (int)i) continue;  // uniform per CTA
    const long long o = g.off[v];
    const int L = g.len[v];
    const int pv = g.prop[v];
    const long long base = h.hoff[i];
    const long long room = h.hoff[i + 1] - base;
    int nh = 0;
    for (int s = threadIdx.x; s < L; s += kHriThreads) {
      const int u = g.adj[o + s];
      if (u >= 0 && is_prior(g.prop[u], u, pv, v)) ++nh;
    }
    nh = (int)warp_sum_ll(nh);
    if (lane_id() == 0) sw[warp_id()] = nh;
    __syncthreads();
    if (threadIdx.x == 0) {
      int t = 0;
      for (int w = 0; w < kHriThreads / 32; ++w) t += sw[w];
      s_cur[0] = 0;
      s_cur[1] = t;
      h.hsplit[i] = t;
    }
    __syncthreads();
    for (int s = threadIdx.x; s < L; s += kHriThreads) {
      const int u = g.adj[o + s];
      if (u < 0) continue;
      const int pos = atomicAdd(&s_cur[is_prior(g.prop[u], u, pv, v) ? 0 : 1], 1);
      if (pos < room)
        h.ids[base + pos] = u;
      else
        atomicOr(&st->status, ST_OVERFLOW);
    }
    __syncthreads();
  }
}

}  // namespace

cudaError_t launch_hri_build(const GraphDev& g, const HriBufs& h, DevState* st, int variant, cudaStream_t s) {
  if (h.min_live <= 0 || g.n <= 0) return cudaSuccess;
  long long b = ((long long)g.n + kHriThreads - 1) / kHriThreads;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  cudaError_t e = cudaMemsetAsync(h.bcnt, 0, 64 * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  hri_count_kernel<<<(unsigned)b, kHriThreads, 0, s>>>(g, h);
  hri_classify_kernel<<<(unsigned)b, kHriThreads, 0, s>>>(g, h, st);
  hri_offsets_kernel<<<1, kHriThreads, 0, s>>>(g, h, st);
  if (variant == DC_HB)
    hri_split_kernel<<<148 * 4, kHriThreads, 0, s>>>(g, h, st);
  else
    hri_fill_kernel<<<148 * 4, kHriThreads, 0, s>>>(g, h, st);
  return cudaGetLastError();
}

}  // namespace dc
