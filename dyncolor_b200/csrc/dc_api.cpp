// dc_api.cpp -- C ABI of libdyncolor (include/dyncolor.h).
//
// Host orchestration only: argument checks, device allocations, the two
// cooperative launches of a batch (structural update, then seeding +
// recolouring loop), pool growth and retry, statistics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/dyncolor.h"
#include "dc_ctx.h"

using namespace dc;


namespace dc {
namespace host {

int key_bits_for(int n) {
  int B = 1;
  while (B < 31 && (1ll << B) < (long long)n) ++B;
  return B;
}

GraphDev graph_dev(const dc_ctx* c) {
  GraphDev g;
  g.n = c->n;
  g.key_bits = c->key_bits;
  g.off = c->off;
  g.len = c->len;
  g.cap = c->cap;
  g.live = c->live;
  g.adj = c->adj;
  g.pool_cap = c->pool_cap;
  g.color = c->color;
  g.prev = c->prev;
  g.prop = c->prop;
  return g;
}

int unit_slots(const dc_ctx* c) { return c->opt.unit_slots; }

// Recolour scratch depends on n and on the pool capacity (work units).
dc_status ensure_recolor_scratch(dc_ctx* ctx) {
  if (ctx->rc_pool_cap == ctx->pool_cap) return DC_OK;
  const long long n = std::max(ctx->n, 1);
  // the loop cuts units down to an eighth of unit_slots (at least 128) when
  // a frontier is small
  const long long CH = std::max<long long>(128, (unit_slots(ctx) / 8) & ~127ll);
  const long long capU = n + ctx->pool_cap / CH + 64;
  // mask words: a multi-unit row (length L > its unit size) takes at most
  // L/32 + 7 words in the mex modes and 132 words for saturation sizes
  // (buffer 2, cut at unit_slots)
  const long long capM_mex = ctx->pool_cap / 32 + 8 * (ctx->pool_cap / CH) + 1024;
  const long long capM_dist = std::max(capM_mex, 132 * (ctx->pool_cap / unit_slots(ctx)) + 1024);
  const long long words = (n + 31) / 32 + 1;
  dc_status s;
  for (int b = 0; b < 3; ++b) {
    QueueBufs& q = ctx->qb[b];
    if ((s = dalloc(ctx, &q.itemsA, n, "queue items")) != DC_OK) return s;
    if ((s = dalloc(ctx, &q.units, capU, "queue units")) != DC_OK) return s;
    const long long capM = b == 2 ? capM_dist : capM_mex;
    if ((s = dalloc(ctx, &q.gmask, capM, "queue masks")) != DC_OK) return s;
    q.capA = n;
    q.capU = capU;
    q.capM = capM;
  }
  if (ctx->opt.heavy_min_live > 0) {
    // heavy-row index: rows that do not fit lose their index (and are scanned in full)
    const bool hi = ctx->opt.variant == DC_HI;
    HriBufs& h = ctx->hri;
    h.min_live = ctx->opt.heavy_min_live;
    h.cap_rows = std::min<long long>(n + 1, ctx->pool_cap / h.min_live + 1);
    // R-MAT scale 24 (1.57 G pool slots): rows >= 2048 hold 236 M slots, rows
    // >= 256 339 M, rows >= 128 414 M.  HB's 4-byte ids get twice the entries
    // in the same bytes.
    h.cap_pairs = hi ? ctx->pool_cap / 4 + 4096 : ctx->pool_cap / 2 + 8192;
    h.cap_exc = hi ? h.cap_pairs : 1;       // a row's change list holds at most its live neighbours
    h.cap_a = hi ? n / 8 + ctx->pool_cap / 512 + 1024 : 1;  // items of 512 slots
    h.cap_hist = hi ? std::min<long long>(h.cap_rows, 1ll << 16) : 0;
    if ((s = dalloc(ctx, &h.hrow, h.cap_rows, "heavy rows")) != DC_OK) return s;
    if ((s = dalloc(ctx, &h.hoff, h.cap_rows + 1, "heavy-row offsets")) != DC_OK) return s;
    if ((s = dalloc(ctx, &h.xoff, h.cap_rows + 1, "change-list offsets")) != DC_OK) return s;
    if ((s = dalloc(ctx, &h.xcnt, h.cap_rows, "change-list counts")) != DC_OK) return s;
    if ((s = dalloc(ctx, &h.hsplit, h.cap_rows, "priority splits")) != DC_OK) return s;
    if ((s = dalloc(ctx, &h.bcnt, 64, "row length classes")) != DC_OK) return s;
    if (hi) {
      if ((s = dalloc(ctx, &h.pairs, h.cap_pairs, "ordered neighbours")) != DC_OK) return s;
      if ((s = dalloc(ctx, &h.xv, h.cap_exc, "change lists")) != DC_OK) return s;
      if ((s = dalloc(ctx, &h.alist, h.cap_a, "append queue")) != DC_OK) return s;
      if ((s = dalloc(ctx, &h.hist, h.cap_hist * kHriBins, "heavy-row colour counts")) != DC_OK) return s;
    } else {
      if ((s = dalloc(ctx, &h.ids, h.cap_pairs, "split neighbours")) != DC_OK) return s;
    }
  }
  if (!ctx->bmA) {
    if ((s = dalloc(ctx, &ctx->bmA, words, "bitmap")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->bmB, words, "bitmap")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->bmC, words, "bitmap")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->ncolor, n, "ncolor")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->sat, n, "sat")) != DC_OK) return s;
    if (ctx->opt.variant == DC_HB && (s = dalloc(ctx, &ctx->cp, n, "packed words")) != DC_OK) return s;
    if (ctx->opt.heavy_min_live > 0) {
      HriBufs& h = ctx->hri;
      if ((s = dalloc(ctx, &h.hid, n, "heavy-row ids")) != DC_OK) return s;
      if (ctx->opt.variant == DC_HI && (s = dalloc(ctx, &h.bmF, words, "changed-colour bitmap")) != DC_OK)
        return s;
    }
    DC_CK(cudaMemsetAsync(ctx->bmA, 0, words * 4, ctx->stream));
    DC_CK(cudaMemsetAsync(ctx->bmB, 0, words * 4, ctx->stream));
    DC_CK(cudaMemsetAsync(ctx->bmC, 0, words * 4, ctx->stream));
  }
  ctx->rc_pool_cap = ctx->pool_cap;
  return DC_OK;
}

dc_status reset_bitmaps(dc_ctx* ctx) {
  const long long words = ((long long)std::max(ctx->n, 1) + 31) / 32 + 1;
  DC_CK(cudaMemsetAsync(ctx->bmA, 0, words * 4, ctx->stream));
  DC_CK(cudaMemsetAsync(ctx->bmB, 0, words * 4, ctx->stream));
  DC_CK(cudaMemsetAsync(ctx->bmC, 0, words * 4, ctx->stream));
  return DC_OK;
}

// Batch scratch depends on k (lines) and on the pool capacity (row units).
dc_status ensure_batch_scratch(dc_ctx* ctx, long long k) {
  const bool grow_k = k > ctx->kcap;
  const bool grow_pool = ctx->k_pool_cap != ctx->pool_cap;
  if (!grow_k && !grow_pool) return DC_OK;
  dc_status s;
  const long long G = std::max(ctx->grid_struct, 1);
  if (grow_k) {
    const long long kk = std::max<long long>(k, 1024);
    const long long k2 = 2 * kk;
    if ((s = dalloc(ctx, &ctx->d_ch, kk, "changes")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->lflag, kk, "line flags")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->keysA, k2, "keys")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->keysB, k2, "keys")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->net, k2, "net")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->tof, k2, "tof")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->present, k2, "present")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->rank, k2, "rank")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->tbeg, k2 + 1, "tbeg")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->trow, k2, "trow")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->rowdel, k2, "rowdel")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->tins, k2, "tins")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->tnoff, k2, "tnoff")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->tncap, k2, "tncap")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->tnlive, k2, "tnlive")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->trel, k2, "trel")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->cursor, k2, "cursor")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->delpos, k2, "delpos")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->hist, G * 256, "hist")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->dscan, G * 256 + 256, "dscan")) != DC_OK) return s;
    if ((s = dalloc(ctx, &ctx->cta_cnt, G, "cta counts")) != DC_OK) return s;
    ctx->kcap = kk;
  }
  const long long cu = 2 * ctx->kcap + ctx->pool_cap / kStructChunk + 64;
  if ((s = dalloc(ctx, &ctx->units, cu, "row units")) != DC_OK) return s;
  if ((s = dalloc(ctx, &ctx->relunits, cu, "relocation units")) != DC_OK) return s;
  ctx->cap_units = cu;
  ctx->cap_rel = cu;
  ctx->k_pool_cap = ctx->pool_cap;
  return DC_OK;
}

void free_batch_scratch(dc_ctx* ctx) {
  dfree(ctx, &ctx->d_ch);
  dfree(ctx, &ctx->lflag);
  dfree(ctx, &ctx->keysA);
  dfree(ctx, &ctx->keysB);
  dfree(ctx, &ctx->net);
  dfree(ctx, &ctx->tof);
  dfree(ctx, &ctx->present);
  dfree(ctx, &ctx->rank);
  dfree(ctx, &ctx->tbeg);
  dfree(ctx, &ctx->trow);
  dfree(ctx, &ctx->rowdel);
  dfree(ctx, &ctx->tins);
  dfree(ctx, &ctx->tnoff);
  dfree(ctx, &ctx->tncap);
  dfree(ctx, &ctx->tnlive);
  dfree(ctx, &ctx->trel);
  dfree(ctx, &ctx->cursor);
  dfree(ctx, &ctx->delpos);
  dfree(ctx, &ctx->units);
  dfree(ctx, &ctx->relunits);
  dfree(ctx, &ctx->hist);
  dfree(ctx, &ctx->dscan);
  dfree(ctx, &ctx->cta_cnt);
  ctx->kcap = 0;
  ctx->k_pool_cap = -1;
}

StructParams struct_params(dc_ctx* ctx, const dc_change* ch, const int* la, const int* lb, long long k) {
  StructParams p{};
  p.g = graph_dev(ctx);
  p.ch = ch;
  p.la = la;
  p.lb = lb;
  p.k = k;
  p.slack = ctx->opt.slack;
  p.keysA = ctx->keysA;
  p.keysB = ctx->keysB;
  p.hist = ctx->hist;
  p.dscan = ctx->dscan;
  p.cta_cnt = ctx->cta_cnt;
  p.net = ctx->net;
  p.tof = ctx->tof;
  p.present = ctx->present;
  p.rank = ctx->rank;
  p.tbeg = ctx->tbeg;
  p.trow = ctx->trow;
  p.rowdel = ctx->rowdel;
  p.tins = ctx->tins;
  p.tnoff = ctx->tnoff;
  p.tncap = ctx->tncap;
  p.tnlive = ctx->tnlive;
  p.trel = ctx->trel;
  p.cursor = ctx->cursor;
  p.delpos = ctx->delpos;
  p.units = ctx->units;
  p.relunits = ctx->relunits;
  p.cap_units = ctx->cap_units;
  p.cap_rel = ctx->cap_rel;
  p.gid = ctx->ngraphs > 0 ? ctx->gid : nullptr;
  p.bar_timeout_ns = (unsigned long long)ctx->opt.barrier_timeout_ms * 1000000ull;
  p.st = ctx->st;
  return p;
}

RecolorParams recolor_params(dc_ctx* ctx, const dc_change* ch, long long k) {
  RecolorParams p{};
  p.g = graph_dev(ctx);
  p.ch = ch;
  p.k = k;
  p.variant = ctx->opt.variant;
  p.unit_slots = unit_slots(ctx);
  p.iter_cap = ctx->opt.iter_cap;
  for (int b = 0; b < 3; ++b) p.qb[b] = ctx->qb[b];
  p.bmA = ctx->bmA;
  p.bmB = ctx->bmB;
  p.bmC = ctx->bmC;
  p.ncolor = ctx->ncolor;
  p.sat = ctx->sat;
  p.cp = ctx->cp;
  p.hri = ctx->hri;
  p.lflag = ctx->lflag;
  if (ctx->ngraphs > 0) {
    p.gid = ctx->gid;
    p.ngraphs = ctx->ngraphs;
    p.gcnt = ctx->gcnt;
    p.gf0 = ctx->gf0;
    p.giters = ctx->giters;
    p.gstate = ctx->gstate;
  }
  p.bar_timeout_ns = (unsigned long long)ctx->opt.barrier_timeout_ms * 1000000ull;
  p.st = ctx->st;
  return p;
}

// Clears the per-launch part of DevState and snapshots the pool counter.
dc_status reset_state(dc_ctx* ctx) {
  const size_t off = offsetof(DevState, bar_arrived);
  DC_CK(cudaMemsetAsync(reinterpret_cast<char*>(ctx->st) + off, 0, sizeof(DevState) - off, ctx->stream));
  DC_CK(cudaMemcpyAsync(&ctx->st->pool_used_start, &ctx->st->pool_used, sizeof(unsigned long long),
                        cudaMemcpyDeviceToDevice, ctx->stream));
  return DC_OK;
}

dc_status read_state(dc_ctx* ctx) {
  DC_CK(cudaMemcpyAsync(ctx->h_st, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
  DC_CK(cudaStreamSynchronize(ctx->stream));
  return DC_OK;
}

void drop_graph(dc_ctx* ctx);

// Moves the adjacency into a fresh pool of new_cap slots (tombstones dropped).
// Packed size of every row (tombstones dropped, rows at the repack slack).
dc_status packed_total(dc_ctx* ctx, long long* total, long long** scratch_out) {
  const long long n = std::max(ctx->n, 1);
  long long* scratch = nullptr;
  dc_status s;
  if ((s = dalloc(ctx, &scratch, n / 256 + 2, "repack scratch")) != DC_OK) return s;
  cudaError_t e = launch_packed_total(graph_dev(ctx), ctx->opt.slack, scratch, ctx->d_scalar, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ctx->h_scalar, ctx->d_scalar, 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    dfree(ctx, &scratch);
    return cuda_fail(ctx, "packed total", e);
  }
  *total = (long long)ctx->h_scalar[0];
  if (scratch_out)
    *scratch_out = scratch;
  else
    dfree(ctx, &scratch);
  return DC_OK;
}

// Moves the adjacency into a fresh pool of new_cap slots (tombstones
// dropped).  Nothing changes when the packed rows need more than new_cap.
dc_status repack(dc_ctx* ctx, long long new_cap) {
  long long total = 0;
  long long* scratch = nullptr;
  dc_status s;
  if ((s = packed_total(ctx, &total, &scratch)) != DC_OK) return s;
  if (total > new_cap) {
    dfree(ctx, &scratch);
    return fail(ctx, DC_E_NOMEM, "compaction needs " + std::to_string(total) + " adjacency slots, the pool has " +
                                     std::to_string(new_cap));
  }
  long long* off2 = nullptr;
  int* cap2 = nullptr;
  int* len2 = nullptr;
  int* adj2 = nullptr;
  const long long n = std::max(ctx->n, 1);
  auto drop = [&]() {
    dfree(ctx, &scratch);
    dfree(ctx, &off2);
    dfree(ctx, &cap2);
    dfree(ctx, &len2);
    dfree(ctx, &adj2);
  };
  // a context that compacts often keeps the previous arrays as the next
  // compaction's target instead of freeing and reallocating gigabytes
  if (ctx->keep_spare && ctx->spare.adj && ctx->spare.adj_cap >= new_cap) {
    off2 = ctx->spare.off;
    cap2 = ctx->spare.cap;
    len2 = ctx->spare.len;
    adj2 = ctx->spare.adj;
    ctx->spare = dc_ctx::Spare{};
  } else if ((s = dalloc(ctx, &off2, n, "repack offsets")) != DC_OK ||
             (s = dalloc(ctx, &cap2, n, "repack caps")) != DC_OK ||
             (s = dalloc(ctx, &len2, n, "repack lengths")) != DC_OK ||
             (s = dalloc(ctx, &adj2, new_cap, "repack pool")) != DC_OK) {
    drop();
    return s;
  }
  DC_CK(cudaMemsetAsync(&ctx->st->status, 0, sizeof(unsigned), ctx->stream));
  DC_CK(launch_repack_copy(graph_dev(ctx), ctx->opt.slack, scratch, off2, cap2, len2, adj2, new_cap,
                           &ctx->st->status, ctx->stream));
  if ((s = read_state(ctx)) != DC_OK) return s;
  if (ctx->h_st->status & ST_OVERFLOW) {
    drop();
    return fail(ctx, DC_E_INTERNAL, "repack: a row outgrew its packed size");
  }
  ctx->h_scalar[1] = (unsigned long long)total;
  DC_CK(cudaMemcpyAsync(&ctx->st->pool_used, ctx->h_scalar + 1, 8, cudaMemcpyHostToDevice, ctx->stream));
  DC_CK(cudaStreamSynchronize(ctx->stream));
  dfree(ctx, &scratch);
  if (ctx->keep_spare) {
    dfree(ctx, &ctx->spare.off);  // a spare too small for this compaction
    dfree(ctx, &ctx->spare.cap);
    dfree(ctx, &ctx->spare.len);
    dfree(ctx, &ctx->spare.adj);
    ctx->spare.off = ctx->off;
    ctx->spare.cap = ctx->cap;
    ctx->spare.len = ctx->len;
    ctx->spare.adj = ctx->adj;
    ctx->spare.adj_cap = ctx->pool_cap;
  } else {
    dfree(ctx, &ctx->off);
    dfree(ctx, &ctx->cap);
    dfree(ctx, &ctx->len);
    dfree(ctx, &ctx->adj);
  }
  ctx->off = off2;
  ctx->cap = cap2;
  ctx->len = len2;
  ctx->adj = adj2;
  ctx->pool_cap = new_cap;
  drop_graph(ctx);  // a captured batch graph names the old arrays
  return DC_OK;
}

// Runs one batch (or a load) already resident on the device.
// Enqueues one attempt of a batch (or load) on the context's stream, ending
// with the copy of the device state into pinned host memory.  k_dev, when
// set, makes the kernels read the line count from device memory, so a
// captured graph of this sequence serves every batch.
dc_status enqueue_batch(dc_ctx* ctx, const dc_change* d_ch, const int* la, const int* lb, long long k,
                        bool recolor, const long long* k_dev) {
  dc_status s;
  const bool events = k_dev == nullptr;  // events recorded inside a captured graph cannot be timed
  if (events) DC_CK(cudaEventRecord(ctx->ev0, ctx->stream));
  if ((s = reset_state(ctx)) != DC_OK) return s;
  StructParams sp = struct_params(ctx, d_ch, la, lb, k);
  sp.k_dev = k_dev;
  DC_CK(launch_struct(sp, ctx->grid_struct, ctx->stream));
  if (events) DC_CK(cudaEventRecord(ctx->evm, ctx->stream));
  if (recolor) {
    if (ctx->ngraphs > 0) {
      const size_t G = (size_t)ctx->ngraphs;
      DC_CK(cudaMemsetAsync(ctx->gcnt, 0, 2 * G * sizeof(int), ctx->stream));
      DC_CK(cudaMemsetAsync(ctx->gf0, 0, G * sizeof(int), ctx->stream));
      DC_CK(cudaMemsetAsync(ctx->giters, 0, G * sizeof(int), ctx->stream));
      DC_CK(cudaMemsetAsync(ctx->gstate, 0, G * sizeof(int), ctx->stream));
    }
    DC_CK(cudaMemcpyAsync(&ctx->st->pre_status, &ctx->st->status, sizeof(unsigned),
                          cudaMemcpyDeviceToDevice, ctx->stream));
    // fresh grid barrier and work counters for the second cooperative launch
    const size_t b0 = offsetof(DevState, bar_arrived);
    const size_t b1 = offsetof(DevState, wctr) + sizeof(((DevState*)nullptr)->wctr);
    DC_CK(cudaMemsetAsync(reinterpret_cast<char*>(ctx->st) + b0, 0, b1 - b0, ctx->stream));
    RecolorParams rp = recolor_params(ctx, d_ch, k);
    rp.k_dev = k_dev;
    rp.ranges = ctx->index_n > 0 ? ctx->d_ranges : nullptr;
    if (ctx->use_index) {
      HriBufs hb = ctx->hri;
      hb.ranges = ctx->index_n > 0 ? ctx->d_ranges : nullptr;
      rp.hri.ranges = hb.ranges;
      DC_CK(launch_hri_build(graph_dev(ctx), hb, ctx->st, ctx->opt.variant, ctx->stream));
    }
    else
      rp.hri.min_live = 0;  // this batch scans every row
    DC_CK(launch_recolor(rp, ctx->grid_recolor, ctx->stream));
  }
  if (events) DC_CK(cudaEventRecord(ctx->ev1, ctx->stream));
  DC_CK(cudaMemcpyAsync(ctx->h_st, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
  return DC_OK;
}

void drop_graph(dc_ctx* ctx) {
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  if (ctx->cgraph) cudaGraphDestroy(ctx->cgraph);
  ctx->gexec = nullptr;
  ctx->cgraph = nullptr;
}

// Captures the batch sequence (lines in ctx->d_ch, count in st->batch_k)
// into a CUDA graph; recaptured whenever a buffer it names was reallocated.
dc_status ensure_graph(dc_ctx* ctx) {
  const long long key[6] = {ctx->kcap, ctx->k_pool_cap, ctx->rc_pool_cap, ctx->ngraphs,
                            (long long)(uintptr_t)ctx->d_ch,
                            (ctx->use_index ? 1 : 0) + (ctx->index_n > 0 ? 2 : 0)};
  if (ctx->gexec && std::memcmp(key, ctx->graph_key, sizeof(key)) == 0) return DC_OK;
  drop_graph(ctx);
  DC_CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  dc_status s = enqueue_batch(ctx, ctx->d_ch, nullptr, nullptr, 0, true, &ctx->st->batch_k);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  if (s != DC_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  if (e != cudaSuccess) return cuda_fail(ctx, "cudaStreamEndCapture", e);
  ctx->cgraph = g;
  e = cudaGraphInstantiate(&ctx->gexec, g, 0);
  if (e != cudaSuccess) {
    drop_graph(ctx);
    return cuda_fail(ctx, "cudaGraphInstantiate", e);
  }
  std::memcpy(ctx->graph_key, key, sizeof(key));
  return DC_OK;
}

// Runs one batch (or a load) already resident on the device.
dc_status run_batch(dc_ctx* ctx, const dc_change* d_ch, const int* la, const int* lb, long long k,
                    bool recolor, dc_stats* out) {
  dc_status s;
  if ((s = ensure_batch_scratch(ctx, k)) != DC_OK) return s;
  if ((s = ensure_recolor_scratch(ctx)) != DC_OK) return s;
  // The heavy-row index is rebuilt for every row of the graph at each
  // launch; it pays off when the batch is large enough to start long
  // cascades through those rows, and a small batch on a big graph (or one
  // graph's batch in a pool of many) would mostly pay for the build.
  ctx->use_index = recolor && ctx->hri.min_live > 0 &&
                   k * kIndexBatchRatio >= (ctx->index_n > 0 ? ctx->index_n : (long long)ctx->n);
  bool compacted = false;
  for (int attempt = 0;; ++attempt) {
    const bool graph = ctx->opt.cuda_graph && recolor && attempt == 0;
    ctx->last_graph = graph;
    if (graph) {
      if (d_ch != ctx->d_ch)
        DC_CK(cudaMemcpyAsync(ctx->d_ch, d_ch, (size_t)k * sizeof(dc_change), cudaMemcpyDeviceToDevice,
                              ctx->stream));
      if ((s = ensure_graph(ctx)) != DC_OK) return s;
      *ctx->h_k = k;
      DC_CK(cudaEventRecord(ctx->ev0, ctx->stream));
      DC_CK(cudaMemcpyAsync(&ctx->st->batch_k, ctx->h_k, sizeof(long long), cudaMemcpyHostToDevice,
                            ctx->stream));
      DC_CK(cudaGraphLaunch(ctx->gexec, ctx->stream));
      DC_CK(cudaEventRecord(ctx->ev1, ctx->stream));
    } else {
      if ((s = enqueue_batch(ctx, d_ch, la, lb, k, recolor, nullptr)) != DC_OK) return s;
    }
    DC_CK(cudaStreamSynchronize(ctx->stream));
    const unsigned stt = ctx->h_st->status;
    if ((stt & ST_POOL) && !(stt & (ST_OVERFLOW | ST_TIMEOUT | ST_INVAL)) && attempt < 4) {
      long long grow = std::max<long long>(ctx->pool_cap, 4ll * k + 4096);
      if (ctx->max_pool_cap > 0) {
        // a budgeted pool: grow up to the cap, else compact once in place
        grow = std::max<long long>(0, std::min(grow, ctx->max_pool_cap - ctx->pool_cap));
        if (grow == 0 && compacted) break;
        compacted = compacted || grow == 0;
      }
      if ((s = repack(ctx, ctx->pool_cap + grow)) != DC_OK) return s;
      if ((s = ensure_batch_scratch(ctx, k)) != DC_OK) return s;
      if ((s = ensure_recolor_scratch(ctx)) != DC_OK) return s;
      continue;
    }
    break;
  }
  const DevState& h = *ctx->h_st;
  float ms = 0.f, ms_s = 0.f, ms_r = 0.f;
  // (a failure here only loses the timing; clear it so no later call sees it)
  if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) != cudaSuccess) ms = -1.f;
  if (ctx->last_graph) {
    // launch split from the kernels' own %globaltimer stamps
    ms_s = h.t_struct[1] > h.t_struct[0] ? (float)((h.t_struct[1] - h.t_struct[0]) * 1e-6) : -1.f;
    ms_r = h.t_recolor[1] > h.t_recolor[0] ? (float)((h.t_recolor[1] - h.t_recolor[0]) * 1e-6) : -1.f;
  } else {
    if (cudaEventElapsedTime(&ms_s, ctx->ev0, ctx->evm) != cudaSuccess) ms_s = -1.f;
    if (cudaEventElapsedTime(&ms_r, ctx->evm, ctx->ev1) != cudaSuccess) ms_r = -1.f;
  }
  cudaGetLastError();
  dc_status rc = DC_OK;
  if (h.status & ST_INVAL)
    rc = fail(ctx, DC_E_INVAL, "change line with a vertex id outside [0,n) or a self-loop");
  else if (h.status & ST_TIMEOUT) {
    // the launch stopped between steps: the graph and colours are partial
    ctx->broken = true;
    return fail(ctx, DC_E_TIMEOUT, "a device-side grid barrier timed out");
  }
  else if (h.status & ST_OVERFLOW)
    rc = fail(ctx, DC_E_INTERNAL, "device-side capacity guard fired");
  else if (h.status & ST_POOL)
    rc = fail(ctx, DC_E_NOMEM, "adjacency pool exhausted");
  else if (h.status & ST_ITER)
    rc = fail(ctx, DC_E_ITER_LIMIT, "recolour loop reached the iteration cap");
  if (rc != DC_OK && recolor) {
    dc_status s2 = reset_bitmaps(ctx);
    if (s2 != DC_OK) return s2;
    DC_CK(launch_color_unmark(graph_dev(ctx), ctx->stream));
  }
  if (out) {
    std::memset(out, 0, sizeof(*out));
    out->iterations = (int64_t)h.iterations;
    out->seed_targets = (int64_t)h.seed_targets;
    out->frontier_total = (int64_t)h.frontier_total;
    out->slots_scanned = (int64_t)h.slots_scanned;
    out->edges_inserted = (int64_t)(h.edges_inserted / 2);
    out->edges_deleted = (int64_t)(h.edges_deleted / 2);
    out->rows_relocated = (int64_t)h.rows_relocated;
    out->status = rc;
    out->max_color = h.cmax;
    out->device_ms = ms;
    out->struct_ms = ms_s;
    out->recolor_ms = ms_r;
    for (int i = 0; i < 6; ++i) out->phase_ms[i] = (double)h.phase_ns[i] * 1e-6;
    out->slots_read = (int64_t)h.slots_read;
    out->pairs = 0;
  }
  return rc;
}

bool ready(dc_ctx* ctx) { return ctx && ctx->n >= 0; }

dc_status gate(dc_ctx* ctx) {
  if (!ctx) return DC_E_INVAL;
  if (ctx->broken) return fail(ctx, DC_E_STATE, "context unusable after a device-side wait timed out; destroy it");
  if (ctx->n < 0) return fail(ctx, DC_E_STATE, "no graph loaded");
  return DC_OK;
}

}  // namespace host
}  // namespace dc

using namespace dc::host;

extern "C" {

const char* dc_status_str(dc_status s) {
  switch (s) {
    case DC_OK: return "ok";
    case DC_E_INVAL: return "invalid argument";
    case DC_E_NOMEM: return "out of memory";
    case DC_E_CUDA: return "CUDA error";
    case DC_E_ITER_LIMIT: return "iteration cap reached";
    case DC_E_STATE: return "call out of order";
    case DC_E_TIMEOUT: return "device wait timed out";
    case DC_E_INTERNAL: return "internal capacity guard";
  }
  return "unknown";
}

dc_status dc_options_default(dc_options* opt) {
  if (!opt) return DC_E_INVAL;
  std::memset(opt, 0, sizeof(*opt));
  opt->variant = DC_HI;
  opt->device = 0;
  opt->stream = nullptr;
  opt->iter_cap = 1 << 20;
  opt->slack = 1.25f;
  opt->blocks_per_sm = 0;
  opt->reserve_slots = 0;
  opt->unit_slots = kUnitSlotsDefault;
  opt->heavy_min_live = 0;  // per variant: dc_create picks it
  opt->barrier_timeout_ms = kBarrierTimeoutMsDefault;
  return DC_OK;
}

dc_status dc_create(dc_ctx** out, const dc_options* opt) {
  if (!out) return DC_E_INVAL;
  *out = nullptr;
  dc_options o;
  if (opt)
    o = *opt;
  else
    dc_options_default(&o);
  if (o.variant != DC_HI && o.variant != DC_HB) return DC_E_INVAL;
  if (o.iter_cap <= 0) o.iter_cap = 1 << 20;
  if (!(o.slack > 1.0f)) o.slack = 1.25f;
  if (o.unit_slots <= 0) o.unit_slots = kUnitSlotsDefault;
  if (o.unit_slots % 128 != 0 || o.unit_slots < 128) return DC_E_INVAL;
  if (o.heavy_min_live == 0) o.heavy_min_live = o.variant == DC_HB ? kHeavyMinLiveHB : kHeavyMinLive;
  if (o.heavy_min_live < 0) o.heavy_min_live = 0;  // off
  if (o.heavy_min_live > 0 && o.heavy_min_live < 64) o.heavy_min_live = 64;
  if (o.barrier_timeout_ms <= 0) o.barrier_timeout_ms = kBarrierTimeoutMsDefault;
  dc_ctx* ctx = new (std::nothrow) dc_ctx();
  if (!ctx) return DC_E_NOMEM;
  ctx->opt = o;
  ctx->device = o.device;
  auto bail = [&](dc_status s) {
    dc_destroy(ctx);
    return s;
  };
  if (cudaSetDevice(o.device) != cudaSuccess) {
    cudaGetLastError();
    return bail(DC_E_CUDA);
  }
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, o.device);
  cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, o.device);
  if (!coop || ctx->sms <= 0) return bail(DC_E_CUDA);
  int occ_s = struct_kernel_occupancy();
  int occ_r = recolor_kernel_occupancy();
  if (occ_s <= 0 || occ_r <= 0) return bail(DC_E_CUDA);
  if (o.blocks_per_sm > 0) {
    occ_s = std::min(occ_s, o.blocks_per_sm);
    occ_r = std::min(occ_r, o.blocks_per_sm);
  }
  ctx->grid_struct = ctx->sms * occ_s;
  ctx->grid_recolor = ctx->sms * occ_r;
  if (o.grid_ctas > 0) {
    ctx->grid_struct = std::min(ctx->grid_struct, (int)o.grid_ctas);
    ctx->grid_recolor = std::min(ctx->grid_recolor, (int)o.grid_ctas);
  }
  if (o.stream) {
    ctx->stream = (cudaStream_t)o.stream;
  } else {
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(DC_E_CUDA);
    ctx->own_stream = true;
  }
  if (cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
      cudaEventCreate(&ctx->evm) != cudaSuccess)
    return bail(DC_E_CUDA);
  if (cudaMalloc((void**)&ctx->st, sizeof(DevState)) != cudaSuccess) return bail(DC_E_NOMEM);
  if (cudaMemset(ctx->st, 0, sizeof(DevState)) != cudaSuccess) return bail(DC_E_CUDA);
  if (cudaMallocHost((void**)&ctx->h_st, sizeof(DevState)) != cudaSuccess) return bail(DC_E_NOMEM);
  if (cudaMalloc((void**)&ctx->d_scalar, 16) != cudaSuccess) return bail(DC_E_NOMEM);
  if (cudaMallocHost((void**)&ctx->h_scalar, 16) != cudaSuccess) return bail(DC_E_NOMEM);
  if (cudaMallocHost((void**)&ctx->h_k, sizeof(long long)) != cudaSuccess) return bail(DC_E_NOMEM);
  *out = ctx;
  return DC_OK;
}

void dc_destroy(dc_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // start from a clean error state
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_batch_scratch(ctx);
  for (int b = 0; b < 3; ++b) {
    dfree(ctx, &ctx->qb[b].itemsA);
    dfree(ctx, &ctx->qb[b].units);
    dfree(ctx, &ctx->qb[b].gmask);
  }
  dfree(ctx, &ctx->bmA);
  dfree(ctx, &ctx->bmB);
  dfree(ctx, &ctx->bmC);
  dfree(ctx, &ctx->ncolor);
  dfree(ctx, &ctx->sat);
  dfree(ctx, &ctx->cp);
  dfree(ctx, &ctx->hri.hid);
  dfree(ctx, &ctx->hri.bmF);
  dfree(ctx, &ctx->hri.hrow);
  dfree(ctx, &ctx->hri.hoff);
  dfree(ctx, &ctx->hri.xoff);
  dfree(ctx, &ctx->hri.xcnt);
  dfree(ctx, &ctx->hri.pairs);
  dfree(ctx, &ctx->hri.ids);
  dfree(ctx, &ctx->hri.xv);
  dfree(ctx, &ctx->hri.alist);
  dfree(ctx, &ctx->hri.hist);
  dfree(ctx, &ctx->hri.hsplit);
  dfree(ctx, &ctx->hri.bcnt);
  dfree(ctx, &ctx->d_ranges);
  dfree(ctx, &ctx->off);
  dfree(ctx, &ctx->len);
  dfree(ctx, &ctx->cap);
  dfree(ctx, &ctx->live);
  dfree(ctx, &ctx->adj);
  dfree(ctx, &ctx->spare.off);
  dfree(ctx, &ctx->spare.cap);
  dfree(ctx, &ctx->spare.len);
  dfree(ctx, &ctx->spare.adj);
  dfree(ctx, &ctx->color);
  dfree(ctx, &ctx->prev);
  dfree(ctx, &ctx->prop);
  dfree(ctx, &ctx->first);
  dfree(ctx, &ctx->gid);
  dfree(ctx, &ctx->gcnt);
  dfree(ctx, &ctx->gf0);
  dfree(ctx, &ctx->giters);
  dfree(ctx, &ctx->gstate);
  dfree(ctx, &ctx->st);
  dfree(ctx, &ctx->d_scalar);
  if (ctx->h_st) cudaFreeHost(ctx->h_st);
  if (ctx->h_scalar) cudaFreeHost(ctx->h_scalar);
  if (ctx->h_k) cudaFreeHost(ctx->h_k);
  drop_graph(ctx);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->evm) cudaEventDestroy(ctx->evm);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

dc_status dc_graph_load_edges(dc_ctx* ctx, int32_t n, const int32_t* a, const int32_t* b, int64_t m) {
  if (!ctx) return DC_E_INVAL;
  if (ctx->broken) return gate(ctx);
  if (ctx->n >= 0) return fail(ctx, DC_E_STATE, "graph already loaded");
  if (n < 0 || m < 0 || (m > 0 && (!a || !b))) return fail(ctx, DC_E_INVAL, "bad graph arguments");
  // pieces of kLoadPiece lines keep the sort keys and scratch in range; the
  // pool of 2 * m * slack slots is the only size limit past this one
  if (m > (1ll << 36)) return fail(ctx, DC_E_INVAL, "more than 2^36 edge lines");
  for (int64_t i = 0; i < m; ++i)
    if (a[i] < 0 || a[i] >= n || b[i] < 0 || b[i] >= n || a[i] == b[i])
      return fail(ctx, DC_E_INVAL, "edge " + std::to_string(i) + " has an id outside [0,n) or is a self-loop");
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // start from a clean error state
  ctx->n = n;
  ctx->key_bits = key_bits_for(n);
  const long long nn = std::max(n, 1);
  dc_status s;
  if ((s = dalloc(ctx, &ctx->off, nn, "row offsets")) != DC_OK) return s;
  if ((s = dalloc(ctx, &ctx->len, nn, "row lengths")) != DC_OK) return s;
  if ((s = dalloc(ctx, &ctx->cap, nn, "row capacities")) != DC_OK) return s;
  if ((s = dalloc(ctx, &ctx->live, nn, "row live counts")) != DC_OK) return s;
  if ((s = dalloc(ctx, &ctx->color, nn, "colours")) != DC_OK) return s;
  if ((s = dalloc(ctx, &ctx->prev, nn, "previous colours")) != DC_OK) return s;
  if ((s = dalloc(ctx, &ctx->prop, nn, "degree property")) != DC_OK) return s;
  DC_CK(cudaMemsetAsync(ctx->off, 0, nn * sizeof(long long), ctx->stream));
  DC_CK(cudaMemsetAsync(ctx->len, 0, nn * sizeof(int), ctx->stream));
  DC_CK(cudaMemsetAsync(ctx->cap, 0, nn * sizeof(int), ctx->stream));
  DC_CK(cudaMemsetAsync(ctx->live, 0, nn * sizeof(int), ctx->stream));
  DC_CK(cudaMemsetAsync(ctx->color, 0, nn * sizeof(int), ctx->stream));
  DC_CK(cudaMemsetAsync(ctx->prev, 0xff, nn * sizeof(int), ctx->stream));  // -1
  DC_CK(cudaMemsetAsync(ctx->prop, 0, nn * sizeof(int), ctx->stream));
  const double slack = ctx->opt.slack;
  long long pool = (long long)std::ceil(2.0 * (double)m * slack) + 8ll * nn + 4096;
  pool = std::max<long long>(pool, ctx->opt.reserve_slots);
  if (ctx->max_pool_cap > 0) pool = ctx->max_pool_cap;  // a budgeted pool takes its whole budget at once
  ctx->pool_cap = pool;
  if ((s = dalloc(ctx, &ctx->adj, pool, "adjacency pool")) != DC_OK) return s;
  DC_CK(cudaMemsetAsync(ctx->st, 0, sizeof(DevState), ctx->stream));
  if (m > 0) {
    // Large edge lists go in pieces so the sort scratch stays bounded; every
    // piece is an insertion batch into the rows built so far.
    const long long piece = std::min<long long>(m, kLoadPiece);
    int* da = nullptr;
    int* db = nullptr;
    if ((s = dalloc(ctx, &da, piece, "load pairs")) != DC_OK) return s;
    if ((s = dalloc(ctx, &db, piece, "load pairs")) != DC_OK) {
      dfree(ctx, &da);
      return s;
    }
    for (long long at = 0; at < m && s == DC_OK; at += piece) {
      const long long len = std::min<long long>(piece, m - at);
      cudaMemcpyAsync(da, a + at, (size_t)len * 4, cudaMemcpyHostToDevice, ctx->stream);
      cudaMemcpyAsync(db, b + at, (size_t)len * 4, cudaMemcpyHostToDevice, ctx->stream);
      s = run_batch(ctx, nullptr, da, db, len, false, nullptr);
    }
    dfree(ctx, &da);
    dfree(ctx, &db);
    // load-sized scratch is not needed by typical batches
    free_batch_scratch(ctx);
    if (s != DC_OK) return s;
  } else {
    if ((s = ensure_recolor_scratch(ctx)) != DC_OK) return s;
  }
  DC_CK(cudaStreamSynchronize(ctx->stream));
  return DC_OK;
}

dc_status dc_colors_set(dc_ctx* ctx, const int32_t* colors, int32_t n) {
  if (dc_status g_ = gate(ctx)) return g_;
  if (n != ctx->n || (n > 0 && !colors)) return fail(ctx, DC_E_INVAL, "colour array size differs from n");
  for (int32_t v = 0; v < n; ++v)
    if (colors[v] < 0 || colors[v] > kColorMask)
      return fail(ctx, DC_E_INVAL, "colour outside [0, 2^30) at vertex " + std::to_string(v));
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // start from a clean error state
  if (n > 0) DC_CK(cudaMemcpyAsync(ctx->color, colors, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
  DC_CK(launch_color_max(graph_dev(ctx), ctx->st, ctx->stream));
  DC_CK(cudaStreamSynchronize(ctx->stream));
  return DC_OK;
}

dc_status dc_colors_init(dc_ctx* ctx, int32_t order) {
  if (dc_status g_ = gate(ctx)) return g_;
  if (order != DC_ORDER_ID && order != DC_ORDER_LDF) return fail(ctx, DC_E_INVAL, "unknown colouring order");
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // start from a clean error state
  dc_status s;
  if ((s = ensure_recolor_scratch(ctx)) != DC_OK) return s;
  const long long n = std::max(ctx->n, 1);
  int* prio = nullptr;
  int* pred = nullptr;
  unsigned long long* cp = nullptr;
  auto drop = [&]() {
    dfree(ctx, &prio);
    dfree(ctx, &pred);
    dfree(ctx, &cp);
  };
  if ((s = dalloc(ctx, &prio, n, "colouring priorities")) != DC_OK ||
      (s = dalloc(ctx, &pred, n, "colouring predecessor counts")) != DC_OK ||
      (s = dalloc(ctx, &cp, n, "colouring packed words")) != DC_OK) {
    drop();
    return s;
  }
  cudaError_t e;
  if (order == DC_ORDER_LDF)
    e = cudaMemcpyAsync(prio, ctx->live, (size_t)n * 4, cudaMemcpyDeviceToDevice, ctx->stream);
  else
    e = cudaMemsetAsync(prio, 0, (size_t)n * 4, ctx->stream);
  if (e == cudaSuccess) {
    // fresh counters, queues and grid barrier for the launch
    const size_t off = offsetof(DevState, bar_arrived);
    e = cudaMemsetAsync(reinterpret_cast<char*>(ctx->st) + off, 0, sizeof(DevState) - off, ctx->stream);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(&ctx->st->cmax, 0, sizeof(int), ctx->stream);
  if (e == cudaSuccess) {
    RecolorParams rp = recolor_params(ctx, nullptr, 0);
    rp.g.prop = prio;
    rp.cp = cp;
    rp.pred = pred;
    rp.hri.min_live = 0;
    rp.iter_cap = n + 1;  // every round colours at least one vertex
    e = launch_init_color(rp, ctx->grid_recolor, ctx->stream);
  }
  if (e != cudaSuccess) {
    drop();
    return cuda_fail(ctx, "initial colouring launch", e);
  }
  s = read_state(ctx);
  drop();
  if (s != DC_OK) return s;
  const unsigned st = ctx->h_st->status;
  if (st & ST_TIMEOUT) {
    ctx->broken = true;
    return fail(ctx, DC_E_TIMEOUT, "a device-side grid barrier timed out");
  }
  if (st & (ST_OVERFLOW | ST_ITER)) return fail(ctx, DC_E_INTERNAL, "initial colouring: a capacity guard fired");
  return DC_OK;
}

dc_status dc_colors_init_greedy(dc_ctx* ctx) { return dc_colors_init(ctx, DC_ORDER_ID); }

dc_status dc_apply_batch(dc_ctx* ctx, const dc_change* changes, int64_t k, dc_stats* out) {
  if (dc_status g_ = gate(ctx)) return g_;
  if (k < 0 || (k > 0 && !changes)) return fail(ctx, DC_E_INVAL, "bad batch arguments");
  if (k > (1ll << 30)) return fail(ctx, DC_E_INVAL, "more than 2^30 change lines");
  if (out) std::memset(out, 0, sizeof(*out));
  if (k == 0) return DC_OK;
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // start from a clean error state
  dc_status s;
  if ((s = ensure_batch_scratch(ctx, k)) != DC_OK) return s;
  DC_CK(cudaMemcpyAsync(ctx->d_ch, changes, (size_t)k * sizeof(dc_change), cudaMemcpyHostToDevice,
                        ctx->stream));
  return run_batch(ctx, ctx->d_ch, nullptr, nullptr, k, true, out);
}

dc_status dc_apply_batch_device(dc_ctx* ctx, const dc_change* d_changes, int64_t k, dc_stats* out) {
  if (dc_status g_ = gate(ctx)) return g_;
  if (k < 0 || (k > 0 && !d_changes)) return fail(ctx, DC_E_INVAL, "bad batch arguments");
  if (k > (1ll << 30)) return fail(ctx, DC_E_INVAL, "more than 2^30 change lines");
  if (out) std::memset(out, 0, sizeof(*out));
  if (k == 0) return DC_OK;
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // start from a clean error state
  return run_batch(ctx, d_changes, nullptr, nullptr, k, true, out);
}

dc_status dc_colors_read(dc_ctx* ctx, int32_t* out, int32_t n) {
  if (dc_status g_ = gate(ctx)) return g_;
  if (n != ctx->n || (n > 0 && !out)) return fail(ctx, DC_E_INVAL, "output size differs from n");
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // start from a clean error state
  if (n > 0) DC_CK(cudaMemcpyAsync(out, ctx->color, (size_t)n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  DC_CK(cudaStreamSynchronize(ctx->stream));
  return DC_OK;
}

dc_status dc_colors_device(dc_ctx* ctx, int32_t** d_colors) {
  if (dc_status g_ = gate(ctx)) return g_;
  if (!d_colors) return DC_E_INVAL;
  *d_colors = ctx->color;
  return DC_OK;
}

dc_status dc_prop_read(dc_ctx* ctx, int32_t* out, int32_t n) {
  if (dc_status g_ = gate(ctx)) return g_;
  if (n != ctx->n || (n > 0 && !out)) return fail(ctx, DC_E_INVAL, "output size differs from n");
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // start from a clean error state
  if (n > 0) DC_CK(cudaMemcpyAsync(out, ctx->prop, (size_t)n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  DC_CK(cudaStreamSynchronize(ctx->stream));
  return DC_OK;
}

dc_status dc_validate(dc_ctx* ctx, int64_t* conflicts) {
  if (dc_status g_ = gate(ctx)) return g_;
  if (!conflicts) return DC_E_INVAL;
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // start from a clean error state
  DC_CK(launch_validate(graph_dev(ctx), ctx->d_scalar, ctx->stream));
  DC_CK(cudaMemcpyAsync(ctx->h_scalar, ctx->d_scalar, 8, cudaMemcpyDeviceToHost, ctx->stream));
  DC_CK(cudaStreamSynchronize(ctx->stream));
  *conflicts = (int64_t)ctx->h_scalar[0];
  return DC_OK;
}

dc_status dc_neighbors(dc_ctx* ctx, int32_t v, int32_t* out, int32_t cap, int32_t* deg) {
  if (dc_status g_ = gate(ctx)) return g_;
  if (v < 0 || v >= ctx->n || !deg || (cap > 0 && !out)) return fail(ctx, DC_E_INVAL, "bad vertex");
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // start from a clean error state
  long long o = 0;
  int L = 0;
  DC_CK(cudaMemcpyAsync(&o, ctx->off + v, 8, cudaMemcpyDeviceToHost, ctx->stream));
  DC_CK(cudaMemcpyAsync(&L, ctx->len + v, 4, cudaMemcpyDeviceToHost, ctx->stream));
  DC_CK(cudaStreamSynchronize(ctx->stream));
  std::vector<int> row((size_t)std::max(L, 1));
  if (L > 0) {
    DC_CK(cudaMemcpyAsync(row.data(), ctx->adj + o, (size_t)L * 4, cudaMemcpyDeviceToHost, ctx->stream));
    DC_CK(cudaStreamSynchronize(ctx->stream));
  }
  int d = 0;
  for (int i = 0; i < L; ++i) {
    if (row[i] < 0) continue;
    if (d < cap) out[d] = row[i];
    ++d;
  }
  *deg = d;
  return DC_OK;
}

dc_status dc_graph_info_get(dc_ctx* ctx, dc_graph_info* info) {
  if (dc_status g_ = gate(ctx)) return g_;
  if (!info) return DC_E_INVAL;
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // start from a clean error state
  DC_CK(launch_count_live(graph_dev(ctx), ctx->d_scalar, ctx->stream));
  DC_CK(cudaMemcpyAsync(ctx->h_scalar, ctx->d_scalar, 8, cudaMemcpyDeviceToHost, ctx->stream));
  DC_CK(cudaMemcpyAsync(ctx->h_scalar + 1, &ctx->st->pool_used, 8, cudaMemcpyDeviceToHost, ctx->stream));
  DC_CK(cudaStreamSynchronize(ctx->stream));
  info->n = ctx->n;
  info->edges = (int64_t)(ctx->h_scalar[0] / 2);
  info->slots_used = (int64_t)ctx->h_scalar[1];
  info->slots_capacity = ctx->pool_cap;
  info->device_bytes = ctx->bytes;
  return DC_OK;
}

dc_status dc_compact(dc_ctx* ctx) {
  if (dc_status g_ = gate(ctx)) return g_;
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // start from a clean error state
  dc_status s = repack(ctx, ctx->pool_cap);
  if (s != DC_OK) return s;
  if ((s = ensure_recolor_scratch(ctx)) != DC_OK) return s;
  DC_CK(cudaStreamSynchronize(ctx->stream));
  return DC_OK;
}

dc_status dc_partition_set(dc_ctx* ctx, int32_t ngraphs, const int32_t* first) {
  if (dc_status g_ = gate(ctx)) return g_;
  if (ngraphs <= 0 || !first) return fail(ctx, DC_E_INVAL, "bad partition arguments");
  if (first[0] != 0 || first[ngraphs] != ctx->n)
    return fail(ctx, DC_E_INVAL, "partition must start at 0 and end at n");
  for (int32_t g = 0; g < ngraphs; ++g)
    if (first[g + 1] < first[g]) return fail(ctx, DC_E_INVAL, "partition offsets must not decrease");
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // start from a clean error state
  const long long G = ngraphs;
  dc_status s;
  if ((s = dalloc(ctx, &ctx->first, G + 1, "partition offsets")) != DC_OK) return s;
  if ((s = dalloc(ctx, &ctx->gid, std::max(ctx->n, 1), "graph ids")) != DC_OK) return s;
  if ((s = dalloc(ctx, &ctx->gcnt, 2 * G, "graph counters")) != DC_OK) return s;
  if ((s = dalloc(ctx, &ctx->gf0, G, "graph counters")) != DC_OK) return s;
  if ((s = dalloc(ctx, &ctx->giters, G, "graph iterations")) != DC_OK) return s;
  if ((s = dalloc(ctx, &ctx->gstate, G, "graph states")) != DC_OK) return s;
  DC_CK(cudaMemcpyAsync(ctx->first, first, (size_t)(G + 1) * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  DC_CK(cudaMemsetAsync(ctx->giters, 0, (size_t)G * sizeof(int), ctx->stream));
  DC_CK(launch_partition(graph_dev(ctx), ctx->first, ngraphs, ctx->gid, ctx->d_scalar, ctx->stream));
  DC_CK(cudaMemcpyAsync(ctx->h_scalar, ctx->d_scalar, 8, cudaMemcpyDeviceToHost, ctx->stream));
  DC_CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->h_scalar[0] != 0) {
    ctx->ngraphs = 0;
    return fail(ctx, DC_E_INVAL, std::to_string(ctx->h_scalar[0]) + " adjacency entries join two graphs");
  }
  ctx->ngraphs = ngraphs;
  return DC_OK;
}

dc_status dc_graph_iterations(dc_ctx* ctx, int64_t* out, int32_t ngraphs) {
  if (dc_status g_ = gate(ctx)) return g_;
  if (ctx->ngraphs == 0) return fail(ctx, DC_E_STATE, "no partition set");
  if (ngraphs != ctx->ngraphs || !out) return fail(ctx, DC_E_INVAL, "output size differs from the partition");
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // start from a clean error state
  std::vector<int> tmp((size_t)ngraphs);
  DC_CK(cudaMemcpyAsync(tmp.data(), ctx->giters, (size_t)ngraphs * sizeof(int), cudaMemcpyDeviceToHost,
                        ctx->stream));
  DC_CK(cudaStreamSynchronize(ctx->stream));
  for (int32_t g = 0; g < ngraphs; ++g) out[g] = tmp[(size_t)g];
  return DC_OK;
}

const char* dc_last_error(const dc_ctx* ctx) {
  if (!ctx) return "null context";
  return ctx->err.c_str();
}

}  // extern "C"
