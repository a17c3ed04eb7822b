// dc_recolor.cu -- seeding + recolouring loop of one update batch, as one
// cooperative persistent launch with software grid barriers.
//
// Snapshot schedule: every reference kernel launch is one step whose reads
// see the state at the start of the step.  A step that computes colours
// (REDUCE) writes them to ncolor[]; the following COMMIT step publishes them.
//
//   HI  (HI/gpuFunctions_undir.cuh:147-284, HI/Color_main.cu:146-202)
//     D1  deletions: target = endpoint with the larger colour (tie: node2)
//     D2  mex of every target                           -> ncolor
//     D3  commit where the colour changed; frontier F0 += target
//     I1  insertions whose colours were equal before the batch and still are
//     I2  saturation size (distinct neighbour colours) of both endpoints
//     I3  target = endpoint with the smaller saturation (tie: node2)
//     I4  mex of every target                           -> ncolor
//     I5  commit unconditionally; F0 += target
//   HB  (HB/gpuFunctions_undir.cuh:104-314, HB/Color_main.cu:160-224)
//     H1  every endpoint of (equal-colour insertions + deletions)
//     H2  mex over neighbours prior in LDF order        -> ncolor
//     H3  commit where the colour changed; F0 += vertex
//   loop (both), until the frontier is empty (HI) or nothing changed (HB):
//     E   findEligibleNeighbors over F  -> next frontier Q (deduped by a
//         mark bit in the colour word)
//     R   recolorNeighbor's mex over Q  -> ncolor
//     C   commit Q (HI also saves the previous colour), Q becomes F
//     A   (HI with the heavy-row index) vertices whose colour changed for
//         the first time join the change lists of their indexed neighbours
//
// Heavy-row index (built by dc_hri.cu before the launch, for batches large
// enough to use it): HI's E and R read an indexed row through its
// colour-ordered copy and change list instead of gathering every
// neighbour's colour; HB's prior-filtered mex reads only the prior part of
// an indexed row.  Results are the same as the full scans.
//
// Work is split by row length: rows of <= kSmall slots ("class A") are
// processed 32 at a time by one warp with a warp-level load-balanced search
// over their slots; longer rows become units of up to unit_slots slots, one
// warp per unit.  A row of several units combines its partial colour masks
// in a global mask slot; the unit that finishes last computes the result.
#include "dc_device.cuh"

namespace dc {

namespace {

enum Mode { M_MEX_ALL = 0, M_MEX_PRIOR = 1, M_DISTINCT = 2 };

constexpr int kCtaBuf = 4096;  // vertices a CTA stages for the next queue during a find-eligible phase

struct Shared {
  unsigned mask[kWarps][kMaskWords];  // per-warp colour window
  int pbuf[kWarps][64];               // per-warp buffer of newly marked vertices
  long long swll[kWarps];
  int cbuf[kCtaBuf];                  // the CTA's newly marked vertices, pushed at the end of the phase
  int ccnt;                           // entries claimed in cbuf (may pass kCtaBuf)
  int sw[kWarps + 1];                 // block-scan scratch
  unsigned long long qbase[2];        // queue positions the CTA's bulk push got (items, units)
};

__device__ __forceinline__ long long grab(unsigned long long* ctr) {
  unsigned long long x = 0;
  if (lane_id() == 0) x = atomicAdd(ctr, 1ull);
  return (long long)__shfl_sync(0xffffffffu, x, 0);
}

// Hands out the work items [0, total) of a phase to warps, `per` items per
// atomic on the phase's counter: a counter takes one atomic at a time, so a
// phase of hundreds of thousands of items would otherwise be bound by the
// counter alone.  `per` grows with the items per warp (at most 32), keeping
// the tail imbalance small.
struct Grabber {
  unsigned long long* ctr;
  long long total, per, cur, end;
  __device__ Grabber(unsigned long long* c, long long t, long long nwarps) : ctr(c), total(t), cur(0), end(0) {
    per = t / (8 * nwarps);
    per = per < 1 ? 1 : (per > 32 ? 32 : per);
  }
  // Warp-uniform.
  __device__ __forceinline__ bool next(long long& i) {
    if (cur >= end) {
      cur = grab(ctr) * per;
      if (cur >= total) return false;
      end = min(total, cur + per);
    }
    i = cur++;
    return true;
  }
};

// Mask words a row of L slots needs in a colour window: the mex of at most
// L colours is at most L, so colours >= min(L, kMaskBits) never matter;
// saturation sizes need the whole window.  At least 2 words (colours < 64
// are folded in from per-lane registers).
__device__ __forceinline__ int mask_words(int L, int mode) {
  if (mode == M_DISTINCT) return kMaskWords;
  const int limit = min(L, kMaskBits);
  return min(kMaskWords, max(2, (limit + 31) / 32 + 1));
}

// Work units of a row: a row of L slots pushed with unit size CH is cut
// into row_units(L, CH) units.  Consumers recover the span of every unit
// from L and the unit count alone (the queue need not record CH): the units
// split the row evenly, in multiples of 128 slots.  (Cutting hub rows into
// quarter units as well was measured 21 % slower on the headline: the extra
// units' mask combining costs more than the shorter units save.)
__device__ __forceinline__ int row_units(int L, int CH) { return L > CH ? (L + CH - 1) / CH : 1; }
__device__ __forceinline__ int unit_span(int L, int nch) {
  const int s = (L + nch - 1) / nch;
  return (s + 127) & ~127;
}

// Pushes u (or nothing when u < 0) into a queue.  Rows of more than one
// unit get a global mask region [done counter, mask words...].  All 32 lanes
// must call.
__device__ __forceinline__ void warp_push(const QueueBufs& qb, QCount* qc, const int* len, int u,
                                          bool allowA, int mode, int CH, unsigned* status) {
  const int L = u >= 0 ? len[u] : 0;
  const bool isA = u >= 0 && allowA && L <= kSmall;
  const bool isU = u >= 0 && !isA;
  const unsigned long long pa = warp_atomic_add(&qc->countA, isA ? 1 : 0);
  if (isA) {
    if ((long long)pa < qb.capA)
      qb.itemsA[pa] = u;
    else
      atomicOr(status, ST_OVERFLOW);
  }
  int c = 0;
  if (isU) c = row_units(L, CH);
  const unsigned long long pu = warp_atomic_add(&qc->countU, c);
  if (isU) {
    int ms = -1;
    if (c > 1) {
      const int words = (mask_words(L, mode) + 1 + 3) & ~3;
      const unsigned long long mo = atomicAdd(&qc->masks, (unsigned long long)words);
      if ((long long)(mo + words) > qb.capM) {
        atomicOr(status, ST_OVERFLOW);
        return;
      }
      uint4* m = reinterpret_cast<uint4*>(qb.gmask + mo);
      for (int i = 0; i < words / 4; ++i) m[i] = make_uint4(0, 0, 0, 0);
      ms = (int)mo;
    }
    for (int q = 0; q < c; ++q) {
      if ((long long)(pu + q) < qb.capU)
        qb.units[pu + q] = make_int4(u, q, ms, c);
      else
        atomicOr(status, ST_OVERFLOW);
    }
  }
}

// Slots per work unit for a queue pushed while processing a phase of
// `items` work items with `nwarps` warps: the configured size while the
// phase keeps every warp busy, a half or a quarter of it (at least 128, a
// multiple of 128) when it does not.
__device__ __forceinline__ int unit_slots_for(long long items, long long nwarps, int ch) {
  int d = 1;
  if (items < nwarps / 2)
    d = 4;
  else if (items < 2 * nwarps)
    d = 2;
  const int c = (ch / d) & ~127;
  return c < 128 ? 128 : c;
}

// Largest j (0..31) with excl_j <= s, excl held one value per lane and
// non-decreasing across lanes.  All lanes must call.
__device__ __forceinline__ int find_owner(int excl, int s) {
  int j = 0;
#pragma unroll
  for (int step = 16; step >= 1; step >>= 1) {
    const int e = __shfl_sync(0xffffffffu, excl, j + step);
    if (e <= s) j += step;
  }
  return j;
}

// First zero bit of the window sm[0..nw) (words >= nw count as zero);
// -1 when all kMaskBits bits are set.  All lanes must call.
__device__ __forceinline__ int first_zero(const unsigned* sm, int nw) {
  for (int k0 = 0; k0 < nw; k0 += 32) {
    const int k = k0 + lane_id();
    const unsigned word = k < nw ? sm[k] : 0u;
    const unsigned bal = __ballot_sync(0xffffffffu, word != 0xffffffffu);
    if (bal) {
      const int l = __ffs(bal) - 1;
      const unsigned wd = __shfl_sync(0xffffffffu, word, l);
      return (k0 + l) * 32 + __ffs(~wd) - 1;
    }
  }
  return nw < kMaskWords ? nw * 32 : -1;
}

struct Env {
  struct {
    unsigned* bmA;
    unsigned* bmB;
    unsigned* bmC;
    int* ncolor;
  } p;
  GraphDev g;
  DevState* st;
  int variant;
  int CH;   // unit size of the seeding phases' pushes
  int CHp;  // unit size of the units this phase pushes (row_units)
  long long nwarps;  // warps of the grid
  long long my_scanned;
  // HB: (degree property << 32) | colour word per vertex, so one 8-byte
  // gather gives both; the next-frontier mark lives in its colour half
  unsigned long long* cp;
  // HI: heavy-row index (hri_on false: every row is scanned in full)
  HriBufs hri;
  bool hri_on;
  bool hri_mex;          // the loop's mex may use the index (its change lists are complete)
  bool hri_split;        // HB: indexed rows list their prior neighbours first
  Shared* sh;            // the CTA's shared memory
  bool cta_stage;        // flush() stages vertices in the CTA buffer (the phase ends with cta_push)
  long long read_delta;  // entries read minus entries the rules cover
  // batched mode (all nullptr for one graph)
  const int* gid;
  int* gpush;        // HI: pushes into the next frontier per graph, this iteration
  int* gchg;         // HB: colour changes per graph, this iteration
  const int* gskip;  // HB: graphs whose last recolour step changed nothing are not expanded
  int* gf0;          // frontier F0 vertices per graph
};

// ---------------------------------------------------------------------
// slow paths (single warp, whole row): colour windows beyond the first
// ---------------------------------------------------------------------
__device__ int slow_mex(Env& E, unsigned* sm, int v, int mode, int w_first = kMaskBits) {
  const GraphDev& g = E.g;
  const long long o = g.off[v];
  const int L = g.len[v];
  const int pv = mode == M_MEX_PRIOR ? g.prop[v] : 0;
  for (int w0 = w_first;; w0 += kMaskBits) {
    for (int k = lane_id(); k < kMaskWords; k += 32) sm[k] = 0;
    __syncwarp();
    for (int s0 = 0; s0 < L; s0 += 32) {
      const int s = s0 + lane_id();
      if (s < L) {
        const int u = g.adj[o + s];
        if (u >= 0 && (mode != M_MEX_PRIOR || is_prior(g.prop[u], u, pv, v))) {
          const int c = (g.color[u] & kColorMask) - w0;
          if (c >= 0 && c < kMaskBits) atomicOr(&sm[c >> 5], 1u << (c & 31));
        }
      }
    }
    __syncwarp();
    const int r = first_zero(sm, kMaskWords);
    __syncwarp();
    if (r >= 0) return w0 + r;
    if (w0 > L) return w0;  // unreachable: the mex never exceeds the row length
  }
}

__device__ int slow_distinct(Env& E, unsigned* sm, int v, int cmax) {
  const GraphDev& g = E.g;
  const long long o = g.off[v];
  const int L = g.len[v];
  int total = 0;
  for (int w0 = kMaskBits; w0 <= cmax; w0 += kMaskBits) {
    for (int k = lane_id(); k < kMaskWords; k += 32) sm[k] = 0;
    __syncwarp();
    for (int s0 = 0; s0 < L; s0 += 32) {
      const int s = s0 + lane_id();
      if (s < L) {
        const int u = g.adj[o + s];
        if (u >= 0) {
          const int c = (g.color[u] & kColorMask) - w0;
          if (c >= 0 && c < kMaskBits) atomicOr(&sm[c >> 5], 1u << (c & 31));
        }
      }
    }
    __syncwarp();
    int cnt = 0;
    for (int k = lane_id(); k < kMaskWords; k += 32) cnt += __popc(sm[k]);
    total += (int)warp_sum_ll(cnt);
    __syncwarp();
  }
  return total;
}

// ---------------------------------------------------------------------
// REDUCE: colour results of a queue into out[]
// ---------------------------------------------------------------------
// Folds per-lane masks of colours < 64 into words 0 and 1 of the window.
__device__ __forceinline__ void fold_low(unsigned* sm, unsigned long long lm) {
  const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)lm);
  const unsigned hi = __reduce_or_sync(0xffffffffu, (unsigned)(lm >> 32));
  __syncwarp();
  if (lane_id() == 0) {
    sm[0] |= lo;
    sm[1] |= hi;
  }
  __syncwarp();
}

// HI mex of an indexed row v inside the loop, from the index instead of a
// gather per neighbour: colour c is present iff some neighbour that kept
// its launch-start colour has colour c (the row's count of unchanged
// neighbours of launch-start colour c is above 0: the build counted every
// colour and the append phase takes one off for each neighbour's first
// change), or some changed neighbour has colour c now (its change list).
// Every unit of the row gathers the current colours of its slice of the
// change list into the row's mask; the unit that finishes last reads the
// counts 32 colours at a time from 0.  Returns false when the row has no
// usable index (the caller scans it).
__device__ bool reduce_heavy(Env& E, Shared& sh, const QueueBufs& qb, int4 un, int* out) {
  const HriBufs& H = E.hri;
  const int v = un.x;
  const int hi = H.hid[v];
  if (hi < 0 || hi >= H.cap_hist || ld_cg(&E.st->hri_off) != 0u) return false;
  const long long xb = H.xoff[hi];
  const int xc = ld_cg(&H.xcnt[hi]);
  if ((long long)xc > H.xoff[hi + 1] - xb) return false;  // change list overflowed
  const int nch = un.w;
  const int nw = mask_words(E.g.len[v], M_MEX_ALL);  // as the queue push sized the row's mask
  unsigned* sm = sh.mask[warp_id()];
  for (int k = lane_id(); k < nw; k += 32) sm[k] = 0;
  __syncwarp();
  const int us = unit_span(E.g.len[v], nch);
  const long long e0 = (long long)un.y * us;
  const long long e1 = min((long long)xc, e0 + us);
  for (long long r0 = e0; r0 < e1; r0 += 128) {
    int cc[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const long long idx = r0 + j * 32 + lane_id();
      cc[j] = idx < e1 ? (E.g.color[H.xv[xb + idx]] & kColorMask) : -1;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (cc[j] >= 0 && cc[j] < nw * 32) atomicOr(&sm[cc[j] >> 5], 1u << (cc[j] & 31));
  }
  __syncwarp();
  if (lane_id() == 0 && e1 > e0) E.read_delta += e1 - e0;
  if (nch > 1) {
    unsigned* gm = qb.gmask + un.z;  // [0]: finished units, [1..nw]: mask
    for (int k = lane_id(); k < nw; k += 32) {
      const unsigned x = sm[k];
      if (x) atomicOr(&gm[1 + k], x);
    }
    __threadfence();
    __syncwarp();
    int last = 0;
    if (lane_id() == 0) last = atomicAdd(&gm[0], 1u) == (unsigned)(nch - 1);
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return true;
    __threadfence();
    for (int k = lane_id(); k < nw; k += 32) sm[k] = ld_cg(&gm[1 + k]);
    __syncwarp();
  }
  const long long live = H.hoff[hi + 1] - H.hoff[hi];
  const int* cnt = H.hist + (long long)hi * kHriBins;
  int r = -1;
  for (int c0 = 0; c0 < kHriBins - 1; c0 += 32) {
    const int c = c0 + lane_id();
    bool pres = true;
    if (c < kHriBins - 1) pres = ld_cg(&cnt[c]) > 0 || (c < nw * 32 && ((sm[c >> 5] >> (c & 31)) & 1u));
    const unsigned bal = __ballot_sync(0xffffffffu, pres);
    if (bal != 0xffffffffu) {
      r = c0 + __ffs(~bal) - 1;
      break;
    }
  }
  long long extra = 0;
  if (r < 0) {
    // every colour below the shared top bin is present: scan the row
    extra = E.g.len[v];
    r = slow_mex(E, sm, v, M_MEX_ALL, 0);
  }
  if (lane_id() == 0) {
    out[v] = r;
    E.my_scanned += live;  // the rule covers every live entry
    E.read_delta += extra - live;
  }
  __syncwarp();
  return true;
}

// HB mex over the prior neighbours of an indexed row v (seeding and loop):
// only the first hsplit entries of its copy are prior to v, so only their
// colours are gathered.  The whole row is handled by its first unit.
__device__ bool reduce_split(Env& E, Shared& sh, int4 un, int* out) {
  const HriBufs& H = E.hri;
  const int v = un.x;
  const int hi = H.hid[v];
  if (hi < 0) return false;
  if (un.y != 0) return true;
  const long long pb = H.hoff[hi];
  const long long live = H.hoff[hi + 1] - pb;
  const int nh = H.hsplit[hi];
  if (lane_id() == 0) E.my_scanned += live;  // the rule covers every live entry
  unsigned* sm = sh.mask[warp_id()];
  const int nw = mask_words(nh + 1, M_MEX_ALL);  // the mex of nh colours is at most nh
  for (int k = lane_id(); k < nw; k += 32) sm[k] = 0;
  __syncwarp();
  unsigned long long lm = 0;
  for (int r0 = 0; r0 < nh; r0 += 128) {
    int cc[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int idx = r0 + j * 32 + lane_id();
      cc[j] = idx < nh ? (E.g.color[H.ids[pb + idx]] & kColorMask) : -1;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = cc[j];
      if (c < 0) continue;
      if (c < 64)
        lm |= 1ull << c;
      else if (c < nw * 32)
        atomicOr(&sm[c >> 5], 1u << (c & 31));
    }
  }
  fold_low(sm, lm);
  int r = first_zero(sm, nw);
  __syncwarp();
  if (r < 0) r = slow_mex(E, sm, v, M_MEX_PRIOR);  // every colour of the window present
  if (lane_id() == 0) {
    out[v] = r;
    E.read_delta += nh - live;
  }
  __syncwarp();
  return true;
}

__device__ void reduce_unit(Env& E, Shared& sh, const QueueBufs& qb, int4 un, int mode, int* out) {
  if (E.hri_mex && mode == M_MEX_ALL && reduce_heavy(E, sh, qb, un, out)) return;
  if (E.hri_split && mode == M_MEX_PRIOR && reduce_split(E, sh, un, out)) return;
  const GraphDev& g = E.g;
  const int v = un.x, chunk = un.y, ms = un.z, nch = un.w;
  const int L = g.len[v];
  const long long o = g.off[v];
  const int us = unit_span(L, nch);
  const int s_lo = chunk * us;
  const int s_hi = min(L, s_lo + us);
  const int limit = mode == M_DISTINCT ? kMaskBits : min(L, kMaskBits);
  const int nw = mask_words(L, mode);
  unsigned* sm = sh.mask[warp_id()];
  for (int k = lane_id(); k < nw; k += 32) sm[k] = 0;
  __syncwarp();
  const int pv = mode == M_MEX_PRIOR ? g.prop[v] : 0;
  unsigned long long lm = 0;  // colours < 64 seen by this lane
  // Four slots per lane per round, lane l taking slots r0 + l + 32 j: every
  // load is coalesced across the warp, and because rows are kept sorted by
  // neighbour id, the colour gathers of one instruction fall on nearby
  // addresses in dense rows.  Four independent gathers are in flight.
  // The ids of round r + 1 are loaded before the colour gathers of round r
  // are consumed, so each round waits on one dependent load, not two.
  int nx[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int sidx = s_lo + j * 32 + lane_id();
    nx[j] = sidx < s_hi ? __ldg(g.adj + o + sidx) : -1;
  }
  for (int r0 = s_lo; r0 < s_hi; r0 += 128) {
    int uu[4];
    bool ok[4];
    int cc[4], pp[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      uu[j] = nx[j];
      const int sidx = r0 + 128 + j * 32 + lane_id();
      nx[j] = sidx < s_hi ? __ldg(g.adj + o + sidx) : -1;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) ok[j] = uu[j] >= 0;
    if (mode == M_MEX_PRIOR) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const unsigned long long x = ok[j] ? E.cp[uu[j]] : 0ull;
        cc[j] = (int)((unsigned)x & (unsigned)kColorMask);
        pp[j] = (int)(x >> 32);
      }
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) cc[j] = ok[j] ? (g.color[uu[j]] & kColorMask) : 0;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (!ok[j]) continue;
      ++E.my_scanned;
      if (mode == M_MEX_PRIOR && !is_prior(pp[j], uu[j], pv, v)) continue;
      const int c = cc[j];
      if (c < 64)
        lm |= 1ull << c;
      else if (c < limit)
        atomicOr(&sm[c >> 5], 1u << (c & 31));
    }
  }
  fold_low(sm, lm);
  if (nch > 1) {
    unsigned* gm = qb.gmask + ms;  // [0]: finished units, [1..nw]: mask
    for (int k = lane_id(); k < nw; k += 32) {
      const unsigned x = sm[k];
      if (x) atomicOr(&gm[1 + k], x);
    }
    __threadfence();
    __syncwarp();
    int last = 0;
    if (lane_id() == 0) last = atomicAdd(&gm[0], 1u) == (unsigned)(nch - 1);
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return;
    __threadfence();
    for (int k = lane_id(); k < nw; k += 32) sm[k] = ld_cg(&gm[1 + k]);
    __syncwarp();
  }
  int r;
  if (mode == M_DISTINCT) {
    int cnt = 0;
    for (int k = lane_id(); k < nw; k += 32) cnt += __popc(sm[k]);
    r = (int)warp_sum_ll(cnt);
    __syncwarp();
    const int cmax = ld_cg(&E.st->cmax);
    if (cmax >= kMaskBits) r += slow_distinct(E, sm, v, cmax);
  } else {
    r = first_zero(sm, nw);
    __syncwarp();
    if (r < 0) r = slow_mex(E, sm, v, mode);
  }
  if (lane_id() == 0) out[v] = r;
  __syncwarp();
}

// Class A batch: 32 rows of <= kSmall slots.  MEX modes only.  Each lane
// handles four slots per round (a warp-level load-balanced search finds the
// row of every slot) so four gathers are in flight.
__device__ void reduce_batchA(Env& E, Shared& sh, const QueueBufs& qb, long long cA, long long b,
                              int mode, int* out) {
  const GraphDev& g = E.g;
  const long long idx = b * 32 + lane_id();
  const bool valid = idx < cA;
  const int v = valid ? qb.itemsA[idx] : 0;
  const int L = valid ? g.len[v] : 0;
  const long long o = valid ? g.off[v] : 0;
  const int pv = (valid && mode == M_MEX_PRIOR) ? g.prop[v] : 0;
  unsigned long long* m64 = reinterpret_cast<unsigned long long*>(sh.mask[warp_id()]);
  m64[lane_id()] = 0ull;
  __syncwarp();
  const int incl = warp_incl_scan(L);
  const int T = __shfl_sync(0xffffffffu, incl, 31);
  const int excl = incl - L;
  for (int s0 = 0; s0 < T; s0 += 128) {
    int jj[4], vj[4], pj[4], uu[4], cc[4], pp[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int s = s0 + r * 32 + lane_id();
      jj[r] = find_owner(excl, s);
      vj[r] = __shfl_sync(0xffffffffu, v, jj[r]);
      const long long oj = __shfl_sync(0xffffffffu, o, jj[r]);
      const int ej = __shfl_sync(0xffffffffu, excl, jj[r]);
      pj[r] = __shfl_sync(0xffffffffu, pv, jj[r]);
      uu[r] = s < T ? g.adj[oj + (s - ej)] : -1;
    }
    if (mode == M_MEX_PRIOR) {
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const unsigned long long x = uu[r] >= 0 ? E.cp[uu[r]] : 0ull;
        cc[r] = (int)((unsigned)x & (unsigned)kColorMask);
        pp[r] = (int)(x >> 32);
      }
    } else {
#pragma unroll
      for (int r = 0; r < 4; ++r) cc[r] = uu[r] >= 0 ? (g.color[uu[r]] & kColorMask) : 0;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      if (uu[r] < 0) continue;
      ++E.my_scanned;
      if (mode == M_MEX_PRIOR && !is_prior(pp[r], uu[r], pj[r], vj[r])) continue;
      if (cc[r] < 64) atomicOr(&m64[jj[r]], 1ull << cc[r]);
    }
  }
  __syncwarp();
  if (valid) out[v] = __ffsll((long long)~m64[lane_id()]) - 1;
  __syncwarp();
}

__device__ void phase_reduce(Env& E, Shared& sh, const QueueBufs& qb, const QCount* qc,
                             unsigned long long* ctr, int mode, int* out) {
  const long long cA = min((long long)ld_cg(&qc->countA), qb.capA);
  const long long cU = min((long long)ld_cg(&qc->countU), qb.capU);
  const long long nAb = (cA + 31) / 32;
  const long long total = cU + nAb;
  Grabber gb(ctr, total, E.nwarps);
  long long i;
  while (gb.next(i)) {
    if (i < cU)
      reduce_unit(E, sh, qb, qb.units[i], mode, out);
    else
      reduce_batchA(E, sh, qb, cA, i - cU, mode, out);
  }
}

// ---------------------------------------------------------------------
// EXPAND: findEligibleNeighbors of frontier F into queue N (bitmap bmB)
//   HI: HI/gpuFunctions_undir.cuh:229-260
//   HB: HB/gpuFunctions_undir.cuh:259-291
// ---------------------------------------------------------------------
struct Rule {
  int v, cv, pv;  // frontier vertex, its colour, prev colour (HI) / prop (HB)
};

// Decides for one live slot (v -> u) which vertex to mark, given u's colour
// cu and (HB) degree property pu.
__device__ __forceinline__ void eligible(const Env& E, const Rule& R, int u, int cu, int pu, bool* mu,
                                         bool* mv) {
  if (E.variant == DC_HI) {
    *mu = (R.cv == cu && R.v < u) || (R.pv < cu);
    *mv = false;
  } else {
    const bool pr = is_prior(R.pv, R.v, pu, u);
    *mu = pr;
    *mv = (R.cv == cu) && !pr;
  }
}

// Newly marked vertices collect in a per-warp shared buffer and are pushed
// into the next queue 32 at a time, so every push round (row length gather,
// class split, queue counters) runs with a full warp.
struct PushBuf {
  int* buf;  // sh.pbuf[warp]
  int cnt;   // warp-uniform
};

__device__ __forceinline__ void flush(Env& E, PushBuf& pb, const QueueBufs& nq, QCount* nc, int k) {
  int u = lane_id() < k ? pb.buf[lane_id()] : -1;
  __syncwarp();
  if (E.cta_stage) {
    // stage in the CTA buffer (one shared atomic); what does not fit goes
    // to the queue directly
    int base = 0;
    if (lane_id() == 0) base = atomicAdd(&E.sh->ccnt, k);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (u >= 0 && base + lane_id() < kCtaBuf) {
      E.sh->cbuf[base + lane_id()] = u;
      u = -1;
    }
    if (__any_sync(0xffffffffu, u >= 0)) {
      if (E.gpush && u >= 0) atomicAdd(&E.gpush[E.gid[u]], 1);
      warp_push(nq, nc, E.g.len, u, true, M_MEX_ALL, E.CHp, &E.st->status);
    }
  } else {
    if (E.gpush && u >= 0) atomicAdd(&E.gpush[E.gid[u]], 1);
    warp_push(nq, nc, E.g.len, u, true, M_MEX_ALL, E.CHp, &E.st->status);
  }
  // keep the remainder at the front
  const int rest = pb.cnt - k;
  if (lane_id() < rest) pb.buf[lane_id()] = pb.buf[k + lane_id()];  // rest <= 31 < k
  __syncwarp();
  pb.cnt = rest;
}

// Pushes the CTA buffer into the queue after every warp of the CTA has
// finished the phase: one pair of queue atomics for the whole CTA (block
// scans of the class-A items and of the work units), then every thread
// writes its entries.  All threads of the CTA call it.
__device__ void cta_push(Env& E, const QueueBufs& qb, QCount* qc) {
  Shared& sh = *E.sh;
  __syncthreads();
  const int cnt = min(sh.ccnt, kCtaBuf);
  const int CH = E.CHp;
  for (int b0 = 0; b0 < cnt; b0 += kThreads) {
    const int i = b0 + (int)threadIdx.x;
    const int u = i < cnt ? sh.cbuf[i] : -1;
    const int L = u >= 0 ? E.g.len[u] : 0;
    const bool isA = u >= 0 && L <= kSmall;
    const int c = (u >= 0 && !isA) ? row_units(L, CH) : 0;
    if (E.gpush && u >= 0) atomicAdd(&E.gpush[E.gid[u]], 1);
    int totA = 0, totU = 0;
    const int ea = block_excl_scan(isA ? 1 : 0, sh.sw, &totA);
    const int eu = block_excl_scan(c, sh.sw, &totU);
    if (threadIdx.x == 0 && totA) sh.qbase[0] = atomicAdd(&qc->countA, (unsigned long long)totA);
    if (threadIdx.x == 32 && totU) sh.qbase[1] = atomicAdd(&qc->countU, (unsigned long long)totU);
    __syncthreads();
    if (isA) {
      const unsigned long long pa = sh.qbase[0] + ea;
      if ((long long)pa < qb.capA)
        qb.itemsA[pa] = u;
      else
        atomicOr(&E.st->status, ST_OVERFLOW);
    }
    if (c > 0) {
      int ms = -1;
      bool ok = true;
      if (c > 1) {
        const int words = (mask_words(L, M_MEX_ALL) + 1 + 3) & ~3;
        const unsigned long long mo = atomicAdd(&qc->masks, (unsigned long long)words);
        if ((long long)(mo + words) > qb.capM) {
          atomicOr(&E.st->status, ST_OVERFLOW);
          ok = false;
        } else {
          uint4* m = reinterpret_cast<uint4*>(qb.gmask + mo);
          for (int w = 0; w < words / 4; ++w) m[w] = make_uint4(0, 0, 0, 0);
          ms = (int)mo;
        }
      }
      const unsigned long long pu = sh.qbase[1] + eu;
      for (int q = 0; ok && q < c; ++q) {
        if ((long long)(pu + q) < qb.capU)
          qb.units[pu + q] = make_int4(u, q, ms, c);
        else
          atomicOr(&E.st->status, ST_OVERFLOW);
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) sh.ccnt = 0;
}

// The word that holds u's next-frontier mark: its colour word (HI) or the
// colour half of its packed word (HB).
__device__ __forceinline__ unsigned* mark_word(const Env& E, int u) {
  return E.cp ? reinterpret_cast<unsigned*>(E.cp + u) : reinterpret_cast<unsigned*>(E.g.color + u);
}

// Claims u for the next frontier: sets the mark bit of its colour word
// unless the preloaded word already has it (the atomic decides races), and
// appends the vertices this warp marked first to the warp buffer.  All
// lanes must call.
__device__ __forceinline__ void claim(Env& E, PushBuf& pb, const QueueBufs& nq, QCount* nc, int u,
                                      bool want, unsigned word) {
  bool got = false;
  if (want && !(word & kMarkBit))
    got = !(atomicOr(mark_word(E, u), kMarkBit) & kMarkBit);
  const unsigned bal = __ballot_sync(0xffffffffu, got);
  if (!bal) return;
  if (got) pb.buf[pb.cnt + __popc(bal & lanemask_lt())] = u;
  __syncwarp();
  pb.cnt += __popc(bal);
  if (pb.cnt >= 32) flush(E, pb, nq, nc, 32);
}

// claim() for four candidates per lane at once: their mark atomics are all
// in flight before any result is used.  All lanes must call.
__device__ __forceinline__ void claim4(Env& E, PushBuf& pb, const QueueBufs& nq, QCount* nc, const int* uu,
                                       const bool* want, const unsigned* ww) {
  unsigned old[4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
    old[j] = (want[j] && !(ww[j] & kMarkBit)) ? atomicOr(mark_word(E, uu[j]), kMarkBit) : kMarkBit;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const bool got = !(old[j] & kMarkBit);
    const unsigned bal = __ballot_sync(0xffffffffu, got);
    if (!bal) continue;
    if (got) pb.buf[pb.cnt + __popc(bal & lanemask_lt())] = uu[j];
    __syncwarp();
    pb.cnt += __popc(bal);
    if (pb.cnt >= 32) flush(E, pb, nq, nc, 32);
  }
}

// HI findEligibleNeighbors over one unit of an indexed row v: the unit's
// slice of the colour-ordered copy (candidates are the neighbours whose
// colour at index time is above prev[v], equal to color[v], or in the shared
// top bin; a slice that starts below both is skipped after one load), then
// the same slice of v's change list.  Every candidate's current colour is
// gathered and the reference's rule applied to it.
__device__ void expand_heavy(Env& E, PushBuf& pb, int4 un, const Rule& R, int hi, long long xb, int xc,
                             const QueueBufs& nq, QCount* nc) {
  const HriBufs& H = E.hri;
  const int us = unit_span(E.g.len[un.x], un.w);
  const long long p0 = H.hoff[hi] + (long long)un.y * us;
  const long long p1 = min(H.hoff[hi + 1], p0 + us);
  long long reads = 0;
  if (p0 < p1) {
    const int sf = (int)(H.pairs[p0] >> 32);
    const bool skip = sf < kHriBins - 1 && sf <= R.pv && sf < R.cv;
    reads = 1;
    if (lane_id() == 0) E.my_scanned += p1 - p0;  // the rule covers every live entry
    if (!skip) {
      for (long long r0 = p0; r0 < p1; r0 += 128) {
        reads = min(p1, r0 + 128) - p0;
        int uu[4];
        unsigned ww[4];
        bool mu[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const long long idx = r0 + j * 32 + lane_id();
          uu[j] = -1;
          if (idx < p1) {
            const unsigned long long x = H.pairs[idx];
            const int c0 = (int)(x >> 32);
            if (c0 >= kHriBins - 1 || c0 > R.pv || c0 == R.cv) uu[j] = (int)(unsigned)x;
          }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) ww[j] = uu[j] >= 0 ? (unsigned)E.g.color[uu[j]] : kMarkBit;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int cu = (int)(ww[j] & (unsigned)kColorMask);
          mu[j] = uu[j] >= 0 && ((R.cv == cu && R.v < uu[j]) || (R.pv < cu));
        }
        claim4(E, pb, nq, nc, uu, mu, ww);
        // the copy is in descending colour order: once a round ends below
        // both thresholds, so does the rest of the slice
        const int sl = (int)(H.pairs[min(r0 + 127, p1 - 1)] >> 32);
        if (sl < kHriBins - 1 && sl <= R.pv && sl < R.cv) break;
      }
    }
  }
  const long long e0 = (long long)un.y * us;
  const long long e1 = min((long long)xc, e0 + us);
  if (e0 < e1) {
    reads += e1 - e0;
    for (long long r0 = e0; r0 < e1; r0 += 128) {
      int uu[4];
      unsigned ww[4];
      bool mu[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const long long idx = r0 + j * 32 + lane_id();
        uu[j] = idx < e1 ? H.xv[xb + idx] : -1;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) ww[j] = uu[j] >= 0 ? (unsigned)E.g.color[uu[j]] : kMarkBit;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int cu = (int)(ww[j] & (unsigned)kColorMask);
        mu[j] = uu[j] >= 0 && ((R.cv == cu && R.v < uu[j]) || (R.pv < cu));
      }
      claim4(E, pb, nq, nc, uu, mu, ww);
    }
  }
  if (lane_id() == 0) E.read_delta += reads - (p1 > p0 ? p1 - p0 : 0);
}

// First colour change of v since the index was built (c0: its colour
// until then): queue v's row, in chunks, for the append phase.  An item is
// (v, chunk | bin << 21), bin = c0's count bin.  An overflowing queue turns
// the index off for the rest of the batch.
constexpr int kAppendChunk = 512;  // slots per append-phase item: 4 rounds of 4 loads per lane
constexpr int kChunkBits = 21;     // rows of up to 2^21 append chunks (2^30 slots)

__device__ __forceinline__ void push_first(Env& E, int v, int c0) {
  const int L = E.g.len[v];
  const int c = L > 0 ? (L + kAppendChunk - 1) / kAppendChunk : 0;
  if (c == 0) return;
  const unsigned long long b = atomicAdd(&E.st->a_count, (unsigned long long)c);
  if ((long long)(b + c) > E.hri.cap_a) {
    atomicExch(&E.st->hri_off, 1u);
    return;
  }
  const int bin = c0 < kHriBins - 1 ? c0 : kHriBins - 1;
  for (int q = 0; q < c; ++q) E.hri.alist[b + q] = make_int2(v, q | (bin << kChunkBits));
}

// Append phase: every vertex whose colour changed for the first time since
// the index was built joins the change list of each indexed neighbour, and
// leaves that neighbour's count of unchanged neighbours of its launch-start
// colour.
__device__ void phase_append(Env& E, unsigned long long* ctr) {
  const HriBufs& H = E.hri;
  // an overflowed queue has unwritten items, and the index is off anyway
  if (ld_cg(&E.st->hri_off) != 0u) return;
  const long long cnt = min((long long)ld_cg(&E.st->a_count), H.cap_a);
  Grabber gb(ctr, cnt, E.nwarps);
  long long i;
  while (gb.next(i)) {
    const int2 it = H.alist[i];
    const int v = it.x;
    const int chunk = it.y & ((1 << kChunkBits) - 1);
    const int bin = it.y >> kChunkBits;
    const int L = E.g.len[v];
    const long long o = E.g.off[v];
    const int s_lo = chunk * kAppendChunk, s_hi = min(L, s_lo + kAppendChunk);
    for (int r0 = s_lo; r0 < s_hi; r0 += 128) {
      int uu[4], hh[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int sidx = r0 + j * 32 + lane_id();
        uu[j] = sidx < s_hi ? E.g.adj[o + sidx] : -1;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) hh[j] = uu[j] >= 0 ? H.hid[uu[j]] : -1;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (hh[j] < 0) continue;
        const int h = hh[j];
        const int slot = atomicAdd(&H.xcnt[h], 1);
        if ((long long)slot < H.xoff[h + 1] - H.xoff[h]) H.xv[H.xoff[h] + slot] = v;
        if (h < H.cap_hist && bin < kHriBins - 1) atomicSub(&H.hist[(long long)h * kHriBins + bin], 1);
      }
    }
  }
}

__device__ void expand_unit(Env& E, PushBuf& pb, int4 un, const QueueBufs& nq, QCount* nc) {
  const GraphDev& g = E.g;
  const int v = un.x;
  if (E.gskip && ld_cg(&E.gskip[E.gid[v]]) == 0) return;  // its graph has stopped
  const int L = g.len[v];
  const long long o = g.off[v];
  const int us = unit_span(L, un.w);
  const int s_lo = un.y * us;
  const int s_hi = min(L, s_lo + us);
  Rule R;
  R.v = v;
  R.cv = g.color[v] & kColorMask;
  R.pv = E.variant == DC_HI ? g.prev[v] : g.prop[v];
  if (E.hri_on) {
    const int hi = E.hri.hid[v];
    if (hi >= 0 && ld_cg(&E.st->hri_off) == 0u) {
      const long long xb = E.hri.xoff[hi];
      const int xc = ld_cg(&E.hri.xcnt[hi]);
      if ((long long)xc <= E.hri.xoff[hi + 1] - xb) {  // its change list is complete
        expand_heavy(E, pb, un, R, hi, xb, xc, nq, nc);
        return;
      }
    }
  }
  bool markv = false;
  int nx[4];  // ids of the next round, loaded one round ahead
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int sidx = s_lo + j * 32 + lane_id();
    nx[j] = sidx < s_hi ? __ldg(g.adj + o + sidx) : -1;
  }
  for (int r0 = s_lo; r0 < s_hi; r0 += 128) {
    int uu[4], cc[4], pp[4];
    unsigned ww[4];
    bool mu[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      uu[j] = nx[j];
      const int sidx = r0 + 128 + j * 32 + lane_id();
      nx[j] = sidx < s_hi ? __ldg(g.adj + o + sidx) : -1;
    }
    // one gather gives u's colour and its next-frontier mark (HB: and its
    // degree property)
    if (E.cp) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const unsigned long long x = uu[j] >= 0 ? E.cp[uu[j]] : (unsigned long long)kMarkBit;
        ww[j] = (unsigned)x;
        pp[j] = (int)(x >> 32);
      }
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) ww[j] = uu[j] >= 0 ? (unsigned)g.color[uu[j]] : kMarkBit;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) cc[j] = (int)(ww[j] & (unsigned)kColorMask);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      mu[j] = false;
      if (uu[j] < 0) continue;
      ++E.my_scanned;
      bool mv;
      eligible(E, R, uu[j], cc[j], pp[j], &mu[j], &mv);
      markv |= mv;
    }
    claim4(E, pb, nq, nc, uu, mu, ww);
  }
  const bool mv = __any_sync(0xffffffffu, markv);
  claim(E, pb, nq, nc, v, mv && lane_id() == 0, mv ? ld_cg(mark_word(E, v)) : kMarkBit);
}

__device__ void expand_batchA(Env& E, PushBuf& pb, const QueueBufs& fq, long long cA, long long b,
                              const QueueBufs& nq, QCount* nc) {
  const GraphDev& g = E.g;
  const long long idx = b * 32 + lane_id();
  bool valid = idx < cA;
  const int v = valid ? fq.itemsA[idx] : 0;
  if (valid && E.gskip && ld_cg(&E.gskip[E.gid[v]]) == 0) valid = false;  // its graph has stopped
  const int L = valid ? g.len[v] : 0;
  const long long o = valid ? g.off[v] : 0;
  const int cv = valid ? (g.color[v] & kColorMask) : 0;
  const int pv = valid ? (E.variant == DC_HI ? g.prev[v] : g.prop[v]) : 0;
  const int incl = warp_incl_scan(L);
  const int T = __shfl_sync(0xffffffffu, incl, 31);
  const int excl = incl - L;
  for (int s0 = 0; s0 < T; s0 += 128) {
    Rule R[4];
    int uu[4], cc[4], pp[4];
    unsigned ww[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int s = s0 + r * 32 + lane_id();
      const int j = find_owner(excl, s);
      R[r].v = __shfl_sync(0xffffffffu, v, j);
      R[r].cv = __shfl_sync(0xffffffffu, cv, j);
      R[r].pv = __shfl_sync(0xffffffffu, pv, j);
      const long long oj = __shfl_sync(0xffffffffu, o, j);
      const int ej = __shfl_sync(0xffffffffu, excl, j);
      uu[r] = s < T ? g.adj[oj + (s - ej)] : -1;
    }
    if (E.cp) {
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const unsigned long long x = uu[r] >= 0 ? E.cp[uu[r]] : (unsigned long long)kMarkBit;
        ww[r] = (unsigned)x;
        pp[r] = (int)(x >> 32);
      }
    } else {
#pragma unroll
      for (int r = 0; r < 4; ++r) ww[r] = uu[r] >= 0 ? (unsigned)g.color[uu[r]] : kMarkBit;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) cc[r] = (int)(ww[r] & (unsigned)kColorMask);
    bool mu[4], mv[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      mu[r] = false;
      mv[r] = false;
      if (uu[r] >= 0) {
        ++E.my_scanned;
        eligible(E, R[r], uu[r], cc[r], pp[r], &mu[r], &mv[r]);
      }
    }
    claim4(E, pb, nq, nc, uu, mu, ww);
    if (E.variant == DC_HB) {
#pragma unroll
      for (int r = 0; r < 4; ++r)
        claim(E, pb, nq, nc, R[r].v, mv[r], mv[r] ? ld_cg(mark_word(E, R[r].v)) : kMarkBit);
    }
  }
}

__device__ void phase_expand(Env& E, Shared& sh, const QueueBufs& fq, const QCount* fc,
                             const QueueBufs& nq, QCount* nc, unsigned long long* ctr) {
  const long long cA = min((long long)ld_cg(&fc->countA), fq.capA);
  const long long cU = min((long long)ld_cg(&fc->countU), fq.capU);
  const long long nAb = (cA + 31) / 32;
  const long long total = cU + nAb;
  PushBuf pb;
  pb.buf = sh.pbuf[warp_id()];
  pb.cnt = 0;
  Grabber gb(ctr, total, E.nwarps);
  long long i;
  while (gb.next(i)) {
    if (i < cU)
      expand_unit(E, pb, fq.units[i], nq, nc);
    else
      expand_batchA(E, pb, fq, cA, i - cU, nq, nc);
  }
  if (pb.cnt > 0) flush(E, pb, nq, nc, pb.cnt);
  if (E.cta_stage) cta_push(E, nq, nc);
}

// ---------------------------------------------------------------------
// COMMIT and line phases
// ---------------------------------------------------------------------
enum Commit {
  C_LOOP = 0,     // prev (HI) and colour from ncolor (clears the frontier mark)
  C_SEED_DEL = 1, // HI deleteEdge: commit if changed, F0 += v, clear bmA
  C_SEED_INS = 2, // HI insEdge: commit always, F0 += v, clear bmC
  C_SEED_HB = 3,  // HB processChangeEdge: commit if changed, F0 += v, clear bmA
  C_CLEAR_A = 4,  // clear bmA only
  C_CLEAR_B = 5   // clear bmB only
};

// Item i of a queue: class A items first, then units with chunk 0.
__device__ __forceinline__ int queue_item(const QueueBufs& qb, long long cA, long long total, long long i) {
  if (i < cA) return qb.itemsA[i];
  if (i < total) {
    const int4 un = qb.units[i - cA];
    if (un.y == 0) return un.x;
  }
  return -1;
}

// Pushes u into the next frontier through the warp buffer (all lanes call).
__device__ __forceinline__ void push_ready(Env& E, PushBuf& pb, const QueueBufs& nq, QCount* nc, int u, bool want) {
  const unsigned bal = __ballot_sync(0xffffffffu, want);
  if (!bal) return;
  if (want) pb.buf[pb.cnt + __popc(bal & lanemask_lt())] = u;
  __syncwarp();
  pb.cnt += __popc(bal);
  if (pb.cnt >= 32) flush(E, pb, nq, nc, 32);
}

// HB findEligibleNeighbors for a dense frontier, by pulling: rather than
// every frontier vertex walking its whole row (every entry covered by the
// rule), every vertex u asks whether it is marked, and stops at the first
// reason.  u is marked iff a neighbour prior to u is in the frontier, or u
// is in the frontier and a neighbour prior to u has u's colour -- the same
// set the rule marks from the frontier side (HB/gpuFunctions_undir.cuh:
// 259-291).  Frontier membership is a bitmap built from the queue first.
constexpr int kPullLane = 256;  // rows up to this length are walked by one lane

// Sets the membership bit of every frontier vertex and counts the entries
// the rule covers (the frontier rows' live entries).
__device__ void phase_mark_frontier(Env& E, const QueueBufs& fq, const QCount* fc, unsigned* inF,
                                    long long gwarp, long long nwarps) {
  const long long cA = min((long long)ld_cg(&fc->countA), fq.capA);
  const long long cU = min((long long)ld_cg(&fc->countU), fq.capU);
  const long long total = cA + cU;
  long long cov = 0;
  for (long long i0 = gwarp * 32; i0 < total; i0 += nwarps * 32) {
    const int v = queue_item(fq, cA, total, i0 + lane_id());
    if (v < 0) continue;
    if (E.gskip && ld_cg(&E.gskip[E.gid[v]]) == 0) continue;  // its graph has stopped
    atomicOr(&inF[v >> 5], 1u << (v & 31));
    cov += E.g.live[v];
  }
  cov = warp_sum_ll(cov);
  if (lane_id() == 0) {
    E.my_scanned += cov;
    E.read_delta -= cov;
  }
}

__device__ __forceinline__ bool in_bits(const unsigned* bm, int v) { return (ld_cg(&bm[v >> 5]) >> (v & 31)) & 1u; }

// Index of u's heavy row, or -1.  Checked against the row list, because a
// pool launch indexes its own graphs' rows only and the entries of other
// vertices are left from earlier launches.
__device__ __forceinline__ int heavy_row(const Env& E, int u) {
  const int hi = E.hri.hid[u];
  if (hi < 0 || hi >= E.hri.cap_rows || (unsigned long long)hi >= ld_cg(&E.st->hcount)) return -1;
  return E.hri.hrow[hi] == u ? hi : -1;
}

// Walks u's neighbours until one prior to u is in the frontier, or -- when
// u is in the frontier -- has u's colour.  One lane, four neighbours per
// step (their ids, then their packed words, then their membership bits, each
// four loads in flight).
__device__ __forceinline__ bool pull_lane(const Env& E, const unsigned* inF, int u, long long& reads) {
  const GraphDev& g = E.g;
  const int L = g.len[u];
  const long long o = g.off[u];
  const int pu = g.prop[u];
  const bool fu = in_bits(inF, u);
  const int cu = (int)((unsigned)E.cp[u] & (unsigned)kColorMask);
  const int hi = (E.hri_split && L >= E.hri.min_live) ? heavy_row(E, u) : -1;
  if (hi >= 0) {
    // an indexed row lists its prior neighbours first: only they can mark u
    const long long pb = E.hri.hoff[hi];
    const int nh = E.hri.hsplit[hi];
    for (int s0 = 0; s0 < nh; s0 += 4) {
      int w[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) w[j] = s0 + j < nh ? E.hri.ids[pb + s0 + j] : -1;
#pragma unroll
      for (int j = 0; j < 4; ++j) reads += w[j] >= 0;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (w[j] >= 0 && (in_bits(inF, w[j]) || (fu && (g.color[w[j]] & kColorMask) == cu)))
          return true;
    }
    return false;
  }
  for (int s0 = 0; s0 < L; s0 += 4) {
    int w[4];
    unsigned long long x[4];
    bool pr[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) w[j] = s0 + j < L ? g.adj[o + s0 + j] : -1;
#pragma unroll
    for (int j = 0; j < 4; ++j) x[j] = w[j] >= 0 ? E.cp[w[j]] : 0ull;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      pr[j] = w[j] >= 0 && is_prior((int)(x[j] >> 32), w[j], pu, u);
      reads += w[j] >= 0;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (pr[j] && (in_bits(inF, w[j]) || (fu && (int)((unsigned)x[j] & (unsigned)kColorMask) == cu))) return true;
  }
  return false;
}

// Long rows four at a time: lane group g (8 lanes) walks row rows[g], 8
// entries per step, until a hit or the row's end; the warp loops while any
// group is still walking.  All lanes call; returns this group's verdict.
__device__ bool pull_group(const Env& E, const unsigned* inF, int x, long long& reads) {
  const GraphDev& g = E.g;
  const int grp = lane_id() >> 3, sub = lane_id() & 7;
  const unsigned gmask = 0xffu << (grp * 8);
  int lim = 0, pu = 0, cu = 0;
  long long base = 0;
  bool fu = false, idx = false;
  if (x >= 0) {
    pu = g.prop[x];
    fu = in_bits(inF, x);
    cu = (int)((unsigned)E.cp[x] & (unsigned)kColorMask);
    const int hi = E.hri_split ? heavy_row(E, x) : -1;
    if (hi >= 0) {
      idx = true;
      base = E.hri.hoff[hi];
      lim = E.hri.hsplit[hi];
    } else {
      base = g.off[x];
      lim = g.len[x];
    }
  }
  bool done = x < 0, m = false;
  for (int s0 = 0;; s0 += 8) {
    const bool act = !done && s0 < lim;
    if (!__any_sync(0xffffffffu, act)) break;
    bool hit = false;
    if (act) {
      const int s = s0 + sub;
      if (s < lim) {
        ++reads;
        if (idx) {
          const int w = E.hri.ids[base + s];
          hit = in_bits(inF, w) || (fu && (g.color[w] & kColorMask) == cu);
        } else {
          const int w = g.adj[base + s];
          if (w >= 0) {
            const unsigned long long xx = E.cp[w];
            hit = is_prior((int)(xx >> 32), w, pu, x) &&
                  (in_bits(inF, w) || (fu && (int)((unsigned)xx & (unsigned)kColorMask) == cu));
          }
        }
      }
    }
    const unsigned bal = __ballot_sync(0xffffffffu, hit) & gmask;
    if (act) {
      if (bal) {
        m = true;
        done = true;
      } else if (s0 + 8 >= lim) {
        done = true;
      }
    }
  }
  return m;
}

// Every vertex of the launch's graphs (all vertices, or the vertex ranges
// of a pool launch) decides whether it joins the next frontier; lanes take
// rows of up to kPullLane slots, the warp then takes the longer rows of its
// 32 vertices four at a time (8 lanes each).
__device__ void phase_pull_hb(Env& E, Shared& sh, const unsigned* inF, const int* ranges, const QueueBufs& nq,
                              QCount* nc, long long gwarp, long long nwarps) {
  const GraphDev& g = E.g;
  PushBuf pb;
  pb.buf = sh.pbuf[warp_id()];
  pb.cnt = 0;
  long long reads = 0;
  const long long total = ranges ? (long long)ranges[1] : (long long)g.n;
  for (long long b0 = gwarp * 32; b0 < total; b0 += nwarps * 32) {
    const long long x = b0 + lane_id();
    int u = -1;
    if (x < total) {
      if (ranges) {
        const int* r = ranges + 2;
        int lo = 0, hi = ranges[0] - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) / 2;
          if ((long long)r[2 * mid + 1] <= x) lo = mid; else hi = mid - 1;
        }
        u = r[2 * lo] + (int)(x - r[2 * lo + 1]);
      } else {
        u = (int)x;
      }
    }
    if (u >= 0 && E.gskip && ld_cg(&E.gskip[E.gid[u]]) == 0) u = -1;  // its graph has stopped
    const bool lng = u >= 0 && g.len[u] > kPullLane;
    bool want = false;
    if (u >= 0 && !lng) want = pull_lane(E, inF, u, reads);
    push_ready(E, pb, nq, nc, u, want);
    unsigned todo = __ballot_sync(0xffffffffu, lng);
    while (todo) {
      int rows[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        rows[k] = -1;
        if (todo) {
          const int l = __ffs(todo) - 1;
          todo &= todo - 1;
          rows[k] = __shfl_sync(0xffffffffu, u, l);
        }
      }
      const int grp = lane_id() >> 3;
      const int x = grp == 0 ? rows[0] : grp == 1 ? rows[1] : grp == 2 ? rows[2] : rows[3];
      const bool m = pull_group(E, inF, x, reads);
      push_ready(E, pb, nq, nc, x, m && (lane_id() & 7) == 0);
    }
  }
  if (pb.cnt > 0) flush(E, pb, nq, nc, pb.cnt);
  reads = warp_sum_ll(reads);
  if (lane_id() == 0) E.read_delta += reads;
  if (E.cta_stage) cta_push(E, nq, nc);
}

__device__ void phase_commit(Env& E, const QueueBufs& qb, const QCount* qc, int kind,
                             const QueueBufs* f0, QCount* f0c, long long gwarp, long long nwarps,
                             unsigned long long* items_stat, int* chg_flag) {
  const GraphDev& g = E.g;
  const long long cA = min((long long)ld_cg(&qc->countA), qb.capA);
  const long long cU = min((long long)ld_cg(&qc->countU), qb.capU);
  const long long total = cA + cU;
  long long items = 0;
  int cmax_local = -1;
  bool changed = false;
  for (long long i0 = gwarp * 32; i0 < total; i0 += nwarps * 32) {
    const int v = queue_item(qb, cA, total, i0 + lane_id());
    int push = -1;
    int first = -1;  // first colour change since the heavy-row index was built
    int first_c0 = 0;  // its colour until then
    if (v >= 0) {
      ++items;
      switch (kind) {
        case C_LOOP: {
          const int nc = ld_cg(&E.p.ncolor[v]);
          const int oc = ld_cg(g.color + v) & kColorMask;
          if (E.variant == DC_HI) g.prev[v] = oc;
          if (nc != oc) {
            changed = true;
            if (E.gchg) atomicAdd(&E.gchg[E.gid[v]], 1);
            if (E.hri_on && mark_bit(E.hri.bmF, v)) {
              first = v;
              first_c0 = oc;
            }
          }
          g.color[v] = nc;  // also clears the frontier mark
          if (E.cp) reinterpret_cast<unsigned*>(E.cp + v)[0] = (unsigned)nc;
          cmax_local = max(cmax_local, nc);
          break;
        }
        case C_SEED_DEL:
        case C_SEED_HB: {
          const int nc = ld_cg(&E.p.ncolor[v]);
          const int oc = g.color[v];
          if (nc != oc) {
            if (E.hri_on && mark_bit(E.hri.bmF, v)) {
              first = v;
              first_c0 = oc;
            }
            if (kind == C_SEED_DEL) g.prev[v] = oc;
            g.color[v] = nc;
            if (E.cp) reinterpret_cast<unsigned*>(E.cp + v)[0] = (unsigned)nc;
            cmax_local = max(cmax_local, nc);
            push = v;
          }
          E.p.bmA[v >> 5] = 0u;
          break;
        }
        case C_SEED_INS: {
          const int nc = ld_cg(&E.p.ncolor[v]);
          if (E.hri_on && nc != g.color[v] && mark_bit(E.hri.bmF, v)) {
            first = v;
            first_c0 = g.color[v];
          }
          g.prev[v] = g.color[v];
          g.color[v] = nc;
          cmax_local = max(cmax_local, nc);
          push = v;
          E.p.bmC[v >> 5] = 0u;
          break;
        }
        case C_CLEAR_A:
          E.p.bmA[v >> 5] = 0u;
          break;
        default:
          E.p.bmB[v >> 5] = 0u;
          break;
      }
    }
    if (first >= 0) push_first(E, first, first_c0);
    if (f0) {
      const bool claim = push >= 0 && mark_bit(E.p.bmB, push);
      if (claim && E.gf0) atomicAdd(&E.gf0[E.gid[push]], 1);
      warp_push(*f0, f0c, g.len, claim ? push : -1, true, M_MEX_ALL, E.CHp, &E.st->status);
    }
  }
  const int m = __reduce_max_sync(0xffffffffu, cmax_local);
  if (lane_id() == 0 && m >= 0) atomicMax(&E.st->cmax, m);
  const long long it = warp_sum_ll(items);
  if (lane_id() == 0 && it && items_stat) atomicAdd(items_stat, (unsigned long long)it);
  if (chg_flag && __any_sync(0xffffffffu, changed) && lane_id() == 0) atomicExch(chg_flag, 1);
}

}  // namespace

// One instantiation per variant, so each gets its own register allocation
// and no per-entry variant branches.
template <int V>
__global__ void __launch_bounds__(kThreads, 2) recolor_kernel(RecolorParams p) {
  __shared__ Shared sh;
  Env E;
  E.p.bmA = p.bmA;
  E.p.bmB = p.bmB;
  E.p.bmC = p.bmC;
  E.p.ncolor = p.ncolor;
  E.g = p.g;
  E.st = p.st;
  E.variant = V;
  E.CH = p.unit_slots;
  E.CHp = p.unit_slots;
  E.my_scanned = 0;
  E.gid = p.gid;
  E.gpush = nullptr;
  E.gchg = nullptr;
  E.gskip = nullptr;
  E.gf0 = p.gid ? p.gf0 : nullptr;
  E.cp = V == DC_HB ? p.cp : nullptr;
  E.hri = p.hri;
  E.hri_on = V == DC_HI && p.hri.min_live > 0;
  E.hri_mex = false;  // set once the seeding's changes are in the change lists
  E.hri_split = V == DC_HB && p.hri.min_live > 0;
  E.read_delta = 0;
  E.sh = &sh;
  E.cta_stage = false;
  E.nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  if (threadIdx.x == 0) sh.ccnt = 0;
  DevState* st = p.st;
  const GraphDev& g = E.g;
  unsigned bar = 0;
  int ps = 0;  // phase sequence for the work-grab ring
  const long long gthreads = (long long)gridDim.x * blockDim.x;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long gwarp = gtid >> 5, nwarps = gthreads >> 5;
  const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
  auto ctr = [&]() -> unsigned long long* {
    if (leader) st->wctr[(ps + 1) % 3] = 0ull;  // next phase's counter (last used 2 phases ago)
    return &st->wctr[ps % 3];
  };
  // Phase timer: CTA 0 thread 0 reads %globaltimer after each barrier and
  // charges the elapsed time to the phase kind that just ended.
  unsigned long long t_last = leader ? globaltimer_ns() : 0ull;
  if (leader) st->t_recolor[0] = t_last;
  unsigned long long acc[6] = {0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
  auto lap = [&](int kind) {
    if (leader) {
      const unsigned long long t = globaltimer_ns();
      acc[kind] += t - t_last;
      t_last = t;
    }
  };
  const QueueBufs& B0 = p.qb[0];  // F0 and even loop queues
  const QueueBufs& B1 = p.qb[1];  // odd loop queues, HI insertion targets
  const QueueBufs& B2 = p.qb[2];  // seeding sets
  const dc_change* ch = p.ch;
  const long long K = p.k_dev ? *p.k_dev : p.k;
  // The structural launch failed (invalid line, pool exhausted, ...): the
  // batch is not applied.  Uniform: nothing writes pre_status here.
  if (ld_cg(&st->pre_status) != 0u) return;

  // ======================= seeding =======================
  if (V == DC_HI) {
    // D1: deletion targets (and remember which insertions had equal colours)
    for (long long i0 = gwarp * 32; i0 < K; i0 += nwarps * 32) {
      const long long i = i0 + lane_id();
      int t = -1;
      if (i < K) {
        const dc_change c = ch[i];
        if (c.inst == 0) {
          t = g.color[c.node1] > g.color[c.node2] ? c.node1 : c.node2;
        }
        p.lflag[i] = (c.inst == 1 && g.color[c.node1] == g.color[c.node2]) ? 1 : 0;
      }
      const bool claim = t >= 0 && mark_bit(p.bmA, t);
      warp_push(B2, &st->q[Q_S1], g.len, claim ? t : -1, true, M_MEX_ALL, E.CH, &st->status);
    }
    if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
    // D2
    phase_reduce(E, sh, B2, &st->q[Q_S1], ctr(), M_MEX_ALL, p.ncolor);
    ++ps;
    if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
    // D3
    phase_commit(E, B2, &st->q[Q_S1], C_SEED_DEL, &B0, &st->q[Q_LOOP0], gwarp, nwarps,
                 &st->seed_targets, nullptr);
    if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
    // I1: insertions still monochromatic -> both endpoints
    for (long long i0 = gwarp * 32; i0 < K; i0 += nwarps * 32) {
      const long long i = i0 + lane_id();
      int a = -1, b = -1;
      if (i < K && p.lflag[i]) {
        const dc_change c = ch[i];
        if (g.color[c.node1] == g.color[c.node2]) {
          a = c.node1;
          b = c.node2;
          p.lflag[i] = 2;
        }
      }
      const bool ca = a >= 0 && mark_bit(p.bmA, a);
      warp_push(B2, &st->q[Q_S2E], g.len, ca ? a : -1, false, M_DISTINCT, E.CH, &st->status);
      const bool cb = b >= 0 && mark_bit(p.bmA, b);
      warp_push(B2, &st->q[Q_S2E], g.len, cb ? b : -1, false, M_DISTINCT, E.CH, &st->status);
    }
    if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
    // I2: saturation sizes
    phase_reduce(E, sh, B2, &st->q[Q_S2E], ctr(), M_DISTINCT, p.sat);
    ++ps;
    if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
    // I3: targets; release the endpoint set
    for (long long i0 = gwarp * 32; i0 < K; i0 += nwarps * 32) {
      const long long i = i0 + lane_id();
      int t = -1;
      if (i < K && p.lflag[i] == 2) {
        const dc_change c = ch[i];
        t = ld_cg(&p.sat[c.node1]) < ld_cg(&p.sat[c.node2]) ? c.node1 : c.node2;
      }
      const bool claim = t >= 0 && mark_bit(p.bmC, t);
      warp_push(B1, &st->q[Q_S2T], g.len, claim ? t : -1, true, M_MEX_ALL, E.CH, &st->status);
    }
    phase_commit(E, B2, &st->q[Q_S2E], C_CLEAR_A, nullptr, nullptr, gwarp, nwarps, nullptr,
                 nullptr);
    if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
    // I4
    phase_reduce(E, sh, B1, &st->q[Q_S2T], ctr(), M_MEX_ALL, p.ncolor);
    ++ps;
    if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
    // I5
    phase_commit(E, B1, &st->q[Q_S2T], C_SEED_INS, &B0, &st->q[Q_LOOP0], gwarp, nwarps,
                 &st->seed_targets, nullptr);
    if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
  } else {
    // packed (degree property, colour) words for this launch's gathers;
    // the barrier after H1 publishes them before H2 reads any
    for (long long v = gtid; v < g.n; v += gthreads)
      E.cp[v] = ((unsigned long long)(unsigned)g.prop[v] << 32) | (unsigned)(g.color[v] & kColorMask);
    // H1: endpoints of equal-colour insertions and of all deletions
    for (long long i0 = gwarp * 32; i0 < K; i0 += nwarps * 32) {
      const long long i = i0 + lane_id();
      int a = -1, b = -1;
      if (i < K) {
        const dc_change c = ch[i];
        if (c.inst == 0 || (c.inst == 1 && g.color[c.node1] == g.color[c.node2])) {
          a = c.node1;
          b = c.node2;
        }
      }
      const bool ca = a >= 0 && mark_bit(p.bmA, a);
      warp_push(B2, &st->q[Q_S1], g.len, ca ? a : -1, true, M_MEX_ALL, E.CH, &st->status);
      const bool cb = b >= 0 && mark_bit(p.bmA, b);
      warp_push(B2, &st->q[Q_S1], g.len, cb ? b : -1, true, M_MEX_ALL, E.CH, &st->status);
    }
    if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
    // H2
    phase_reduce(E, sh, B2, &st->q[Q_S1], ctr(), M_MEX_PRIOR, p.ncolor);
    ++ps;
    if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
    // H3
    phase_commit(E, B2, &st->q[Q_S1], C_SEED_HB, &B0, &st->q[Q_LOOP0], gwarp, nwarps,
                 &st->seed_targets, nullptr);
    if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
  }
  // F0 is complete: release its marks so the loop can mark into bmB.
  phase_commit(E, B0, &st->q[Q_LOOP0], C_CLEAR_B, nullptr, nullptr, gwarp, nwarps, nullptr,
               nullptr);
  if (p.gid) {
    // a graph whose seeding recoloured nothing never enters the loop
    for (long long gg = gtid; gg < p.ngraphs; gg += gthreads) p.gstate[gg] = ld_cg(&p.gf0[gg]) > 0 ? 1 : 2;
  }
  if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
  // rows of vertices the seeding recoloured join their indexed neighbours'
  // change lists before the loop reads them
  if (E.hri_on && ld_cg(&st->a_count) > 0) {
    phase_append(E, ctr());
    ++ps;
    if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
  }
  E.hri_mex = E.hri_on;
  lap(0);

  // ======================= loop =======================
  {
    int fs = Q_LOOP0;  // counter slot of the frontier
    int fb = 0;        // buffer of the frontier
    const QCount* f0c = &st->q[Q_LOOP0];
    long long it = 0;
    const int rmode = V == DC_HI ? M_MEX_ALL : M_MEX_PRIOR;
    bool go = (ld_cg(&f0c->countA) + ld_cg(&f0c->countU)) > 0;
    while (go) {
      if (it >= p.iter_cap) {
        if (leader) atomicOr(&st->status, ST_ITER);
        break;
      }
      ++it;
      const int ns = (fs + 1) % 3;
      const int nb = fb ^ 1;
      // E
      if (leader) {
        QCount* z = &st->q[(fs + 2) % 3];
        z->countA = 0;
        z->countU = 0;
        z->masks = 0;
        st->a_count = 0;  // every warp read it before the append phase's barrier
      }
      const int ring = (int)(it & 1);
      if (p.gid) {
        int* cur = p.gcnt + (long long)ring * p.ngraphs;
        int* prv = p.gcnt + (long long)(ring ^ 1) * p.ngraphs;
        if (V == DC_HB) {
          // graphs with no colour change in the previous iteration are done
          // (the reference's loop would have ended for them)
          if (it > 1) {
            for (long long gg = gtid; gg < p.ngraphs; gg += gthreads)
              if (p.gstate[gg] == 1 && ld_cg(&prv[gg]) == 0) {
                p.gstate[gg] = 2;
                p.giters[gg] = (int)(it - 1);
              }
          }
          E.gskip = it > 1 ? prv : nullptr;
          E.gpush = nullptr;
        } else {
          E.gpush = cur;
          E.gskip = nullptr;
        }
      }
      // Work units of the next frontier are cut smaller when this one is
      // small, so a small phase is not set by a few long units.
      {
        const long long items = (long long)ld_cg(&st->q[fs].countU) + ((long long)ld_cg(&st->q[fs].countA) + 31) / 32;
        E.CHp = unit_slots_for(items, nwarps, p.unit_slots);
      }
      // HB with a frontier of more than a sixteenth of the launch's vertices pulls
      const bool pull = V == DC_HB && (long long)(ld_cg(&st->q[fs].countA) + ld_cg(&st->q[fs].countU)) * 16 >
                                          (p.ranges ? (long long)p.ranges[1] : (long long)g.n);
      E.cta_stage = true;
      if (pull) {
        phase_mark_frontier(E, p.qb[fb], &st->q[fs], p.bmC, gwarp, nwarps);
        if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
        phase_pull_hb(E, sh, p.bmC, p.ranges, p.qb[nb], &st->q[ns], gwarp, nwarps);
      } else {
        phase_expand(E, sh, p.qb[fb], &st->q[fs], p.qb[nb], &st->q[ns], ctr());
        ++ps;
      }
      E.cta_stage = false;
      if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
      lap(1);
      const QCount* nc = &st->q[ns];
      const long long nq = (long long)(ld_cg(&nc->countA) + ld_cg(&nc->countU));
      if (V == DC_HI && nq == 0) break;
      // R
      if (leader) st->chg[(it + 1) & 1] = 0;
      if (p.gid) {
        int* cur = p.gcnt + (long long)ring * p.ngraphs;
        int* nxt = p.gcnt + (long long)(ring ^ 1) * p.ngraphs;
        for (long long gg = gtid; gg < p.ngraphs; gg += gthreads) {
          // HI: a running graph whose next frontier is empty is done
          if (V == DC_HI && p.gstate[gg] == 1 && ld_cg(&cur[gg]) == 0) {
            p.gstate[gg] = 2;
            p.giters[gg] = (int)it;
          }
          nxt[gg] = 0;  // next iteration's counters (last read before this phase)
        }
        E.gchg = V == DC_HB ? cur : nullptr;
      }
      phase_reduce(E, sh, p.qb[nb], nc, ctr(), rmode, p.ncolor);
      ++ps;
      if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
      lap(2);
      // C
      phase_commit(E, p.qb[nb], nc, C_LOOP, nullptr, nullptr, gwarp, nwarps, &st->frontier_total,
                   &st->chg[it & 1]);
      if (pull) {
        // clear the frontier membership bits for the next pulling iteration
        const long long words = ((long long)g.n + 31) / 32 + 1;
        for (long long w = gtid; w < words; w += gthreads) p.bmC[w] = 0u;
      }
      if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
      if (E.hri_on && ld_cg(&st->a_count) > 0) {
        phase_append(E, ctr());
        ++ps;
        if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
      }
      lap(3);
      if (V == DC_HB && ld_cg(&st->chg[it & 1]) == 0) break;
      fs = ns;
      fb = nb;
    }
    if (p.gid) {
      // graphs still running stop with the union's last iteration
      for (long long gg = gtid; gg < p.ngraphs; gg += gthreads)
        if (p.gstate[gg] == 1) p.giters[gg] = (int)it;
    }
    if (leader) {
      st->iterations = (unsigned long long)it;
      for (int i = 0; i < 6; ++i) st->phase_ns[i] = acc[i];
      st->t_recolor[1] = globaltimer_ns();
    }
  }
  const long long sc = warp_sum_ll(E.my_scanned);
  const long long rd = warp_sum_ll(E.read_delta);
  if (lane_id() == 0 && sc) {
    atomicAdd(&st->slots_scanned, (unsigned long long)sc);
    atomicAdd(&st->slots_read, (unsigned long long)(sc + rd));  // entries actually read
  }
}

// ---------------------------------------------------------------------
// Initial colouring: greedy lowest free colour in a priority order, as a
// Jones-Plassmann schedule (no reference counterpart: the reference takes
// its initial colours from an external tool, MG/README.txt:19-22).
//
// A vertex is coloured once every neighbour before it in the order is
// coloured, with the smallest colour none of those neighbours has.  Its
// neighbours after it are then exactly the uncoloured ones, so every vertex
// gets the colour the sequential greedy pass in that order gives it; the
// rounds only run the independent vertices of the order side by side.
// Order: larger g.prop first, ties by lower id (isPrior_RelativeOrdering's
// comparison); with g.prop all zero it is the vertex-id order.
//   P   pred[v] = neighbours before v         (all vertices, in units)
//   F   frontier F0 = vertices with pred 0
//   round (until the frontier is empty):
//     R  mex over the neighbours before v      -> ncolor
//     D  commit the colour; every neighbour after v loses one pred, and the
//        ones that reach 0 form the next frontier
// ---------------------------------------------------------------------
namespace {

// P over one unit (or a class-A batch of 32 rows): counts the neighbours of
// each row that come before it.
__device__ void pred_unit(Env& E, int4 un, int* pred) {
  const GraphDev& g = E.g;
  const int v = un.x;
  const int L = g.len[v];
  const long long o = g.off[v];
  const int us = unit_span(L, un.w);
  const int s_lo = un.y * us, s_hi = min(L, s_lo + us);
  const int pv = g.prop[v];
  int cnt = 0;
  for (int s0 = s_lo; s0 < s_hi; s0 += 32) {
    const int sidx = s0 + lane_id();
    const int u = sidx < s_hi ? g.adj[o + sidx] : -1;
    if (u >= 0 && is_prior(g.prop[u], u, pv, v)) ++cnt;
  }
  cnt = (int)warp_sum_ll(cnt);
  if (lane_id() == 0 && cnt) atomicAdd(&pred[v], cnt);
}

__device__ void pred_batchA(Env& E, const QueueBufs& qb, long long cA, long long b, int* pred) {
  const GraphDev& g = E.g;
  const long long idx = b * 32 + lane_id();
  if (idx >= cA) return;
  const int v = qb.itemsA[idx];
  const int L = g.len[v];
  const long long o = g.off[v];
  const int pv = g.prop[v];
  int cnt = 0;
  for (int s = 0; s < L; ++s) {
    const int u = g.adj[o + s];
    if (u >= 0 && is_prior(g.prop[u], u, pv, v)) ++cnt;
  }
  if (cnt) atomicAdd(&pred[v], cnt);
}

// Commits v's colour (its first unit) into the colour word and the packed
// word.
__device__ __forceinline__ int commit_init(Env& E, int v) {
  const int c = ld_cg(&E.p.ncolor[v]);
  E.g.color[v] = c;
  reinterpret_cast<unsigned*>(E.cp + v)[0] = (unsigned)c;
  return c;
}

// D over one unit: every neighbour after v loses one pred; those reaching 0
// are ready.
__device__ void release_unit(Env& E, PushBuf& pb, int4 un, int* pred, const QueueBufs& nq, QCount* nc,
                             int& cmax) {
  const GraphDev& g = E.g;
  const int v = un.x;
  if (un.y == 0 && lane_id() == 0) cmax = max(cmax, commit_init(E, v));
  const int L = g.len[v];
  const long long o = g.off[v];
  const int us = unit_span(L, un.w);
  const int s_lo = un.y * us, s_hi = min(L, s_lo + us);
  const int pv = g.prop[v];
  for (int s0 = s_lo; s0 < s_hi; s0 += 32) {
    const int sidx = s0 + lane_id();
    const int u = sidx < s_hi ? g.adj[o + sidx] : -1;
    bool ready = false;
    if (u >= 0 && is_prior(pv, v, g.prop[u], u)) ready = atomicSub(&pred[u], 1) == 1;
    push_ready(E, pb, nq, nc, u, ready);
  }
}

__device__ void release_batchA(Env& E, PushBuf& pb, const QueueBufs& qb, long long cA, long long b, int* pred,
                               const QueueBufs& nq, QCount* nc, int& cmax) {
  const GraphDev& g = E.g;
  const long long idx = b * 32 + lane_id();
  const bool valid = idx < cA;
  const int v = valid ? qb.itemsA[idx] : 0;
  if (valid) cmax = max(cmax, commit_init(E, v));
  const int L = valid ? g.len[v] : 0;
  const long long o = valid ? g.off[v] : 0;
  const int pv = valid ? g.prop[v] : 0;
  const int Lmax = __reduce_max_sync(0xffffffffu, L);
  for (int s = 0; s < Lmax; ++s) {
    const int u = s < L ? g.adj[o + s] : -1;
    bool ready = false;
    if (u >= 0 && is_prior(pv, v, g.prop[u], u)) ready = atomicSub(&pred[u], 1) == 1;
    push_ready(E, pb, nq, nc, u, ready);
  }
}

}  // namespace

__global__ void __launch_bounds__(kThreads, 2) init_color_kernel(RecolorParams p) {
  __shared__ Shared sh;
  Env E;
  E.p.bmA = p.bmA;
  E.p.bmB = p.bmB;
  E.p.bmC = p.bmC;
  E.p.ncolor = p.ncolor;
  E.g = p.g;
  E.st = p.st;
  E.variant = DC_HB;  // the prior-filtered mex of HB
  E.CH = p.unit_slots;
  E.CHp = p.unit_slots;
  E.my_scanned = 0;
  E.gid = nullptr;
  E.gpush = nullptr;
  E.gchg = nullptr;
  E.gskip = nullptr;
  E.gf0 = nullptr;
  E.cp = p.cp;
  E.hri = p.hri;
  E.hri_on = false;
  E.hri_mex = false;
  E.hri_split = false;
  E.read_delta = 0;
  E.sh = &sh;
  E.cta_stage = false;
  E.nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  DevState* st = p.st;
  const GraphDev& g = E.g;
  int* pred = p.pred;
  unsigned bar = 0;
  int ps = 0;
  const long long gthreads = (long long)gridDim.x * blockDim.x;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long gwarp = gtid >> 5, nwarps = gthreads >> 5;
  const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
  auto ctr = [&]() -> unsigned long long* {
    if (leader) st->wctr[(ps + 1) % 3] = 0ull;
    return &st->wctr[ps % 3];
  };
  if (leader) st->t_recolor[0] = globaltimer_ns();
  // every vertex into the all-rows queue; packed (priority, colour) words
  for (long long i0 = gwarp * 32; i0 < g.n; i0 += nwarps * 32) {
    const long long v = i0 + lane_id();
    if (v < g.n) {
      pred[v] = 0;
      E.cp[v] = ((unsigned long long)(unsigned)g.prop[v] << 32);
    }
    warp_push(p.qb[2], &st->q[Q_S1], g.len, v < g.n ? (int)v : -1, true, M_MEX_ALL, E.CH, &st->status);
  }
  if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
  // P
  {
    const QueueBufs& qb = p.qb[2];
    const QCount* qc = &st->q[Q_S1];
    const long long cA = min((long long)ld_cg(&qc->countA), qb.capA);
    const long long cU = min((long long)ld_cg(&qc->countU), qb.capU);
    const long long total = cU + (cA + 31) / 32;
    Grabber gb(ctr(), total, E.nwarps);
    long long i;
    while (gb.next(i)) {
      if (i < cU)
        pred_unit(E, qb.units[i], pred);
      else
        pred_batchA(E, qb, cA, i - cU, pred);
    }
    ++ps;
  }
  if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
  // F0
  for (long long i0 = gwarp * 32; i0 < g.n; i0 += nwarps * 32) {
    const long long v = i0 + lane_id();
    const bool r = v < g.n && ld_cg(&pred[v]) == 0;
    warp_push(p.qb[0], &st->q[Q_LOOP0], g.len, r ? (int)v : -1, true, M_MEX_ALL, E.CH, &st->status);
  }
  if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
  int fs = Q_LOOP0, fb = 0;
  long long it = 0;
  int cmax = -1;
  while (ld_cg(&st->q[fs].countA) + ld_cg(&st->q[fs].countU) > 0) {
    if (it >= p.iter_cap) {
      if (leader) atomicOr(&st->status, ST_ITER);
      break;
    }
    ++it;
    const int ns = (fs + 1) % 3;
    const int nb = fb ^ 1;
    if (leader) {
      QCount* z = &st->q[(fs + 2) % 3];
      z->countA = 0;
      z->countU = 0;
      z->masks = 0;
    }
    // R: the mex over the neighbours before each frontier vertex
    phase_reduce(E, sh, p.qb[fb], &st->q[fs], ctr(), M_MEX_PRIOR, p.ncolor);
    ++ps;
    if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
    // D
    {
      const QueueBufs& fq = p.qb[fb];
      const QCount* fc = &st->q[fs];
      const long long cA = min((long long)ld_cg(&fc->countA), fq.capA);
      const long long cU = min((long long)ld_cg(&fc->countU), fq.capU);
      const long long total = cU + (cA + 31) / 32;
      PushBuf pb;
      pb.buf = sh.pbuf[warp_id()];
      pb.cnt = 0;
      Grabber gb(ctr(), total, E.nwarps);
      long long i;
      while (gb.next(i)) {
        if (i < cU)
          release_unit(E, pb, fq.units[i], pred, p.qb[nb], &st->q[ns], cmax);
        else
          release_batchA(E, pb, fq, cA, i - cU, pred, p.qb[nb], &st->q[ns], cmax);
      }
      if (pb.cnt > 0) flush(E, pb, p.qb[nb], &st->q[ns], pb.cnt);
      ++ps;
    }
    if (!grid_sync(st, bar, p.bar_timeout_ns)) return;
    fs = ns;
    fb = nb;
  }
  const int m = __reduce_max_sync(0xffffffffu, cmax);
  if (lane_id() == 0 && m >= 0) atomicMax(&st->cmax, m);
  if (leader) {
    st->iterations = (unsigned long long)it;
    st->t_recolor[1] = globaltimer_ns();
  }
}

cudaError_t launch_init_color(const RecolorParams& p, int grid, cudaStream_t s) {
  RecolorParams q = p;
  void* args[] = {&q};
  return cudaLaunchCooperativeKernel((const void*)init_color_kernel, dim3(grid), dim3(kThreads), args, 0, s);
}

cudaError_t launch_recolor(const RecolorParams& p, int grid, cudaStream_t s) {
  RecolorParams q = p;
  void* args[] = {&q};
  const void* fn = p.variant == DC_HB ? (const void*)recolor_kernel<DC_HB> : (const void*)recolor_kernel<DC_HI>;
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), args, 0, s);
}

int recolor_kernel_occupancy() {
  int a = 0, b = 0, c = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, recolor_kernel<DC_HI>, kThreads, 0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, recolor_kernel<DC_HB>, kThreads, 0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, init_color_kernel, kThreads, 0) != cudaSuccess)
    return 0;
  const int ab = a < b ? a : b;
  return ab < c ? ab : c;
}

}  // namespace dc
