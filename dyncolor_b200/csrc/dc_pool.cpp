// dc_pool.cpp -- resident multi-graph pool (include/dyncolor_pool.h).
//
// One union context holds every resident graph: graph g owns the vertex ids
// [first, first + n) while resident, gid[v] = g there and gid[v] = G (free)
// elsewhere, so the batched-mode kernels keep the graphs apart and count
// each graph's iterations.  The adjacency pool of the union is the row
// budget: rows of a reloaded graph are appended packed at the pool's tail,
// and a full pool is compacted (tombstones and spilled graphs' rows
// dropped) before graphs are evicted.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/dyncolor_pool.h"
#include "dc_ctx.h"

using namespace dc;
using namespace dc::host;

namespace {

constexpr long long kChunkVertices = 1ll << 20;  // rows per gather / scatter launch
constexpr long long kStageDefault = 1ll << 25;   // staging slots (128 MiB)
constexpr long long kPoolLoadPiece = 1ll << 24;  // edge pairs per structural launch of a graph load

struct PGraph {
  int n = 0;
  bool resident = false;
  int first = -1;
  unsigned long long last_use = 0;
  long long packed = 0;  // adjacency slots the graph takes when reloaded packed
  int max_color = 0;
  bool host_valid = false;  // the pinned copy below is the graph's state
  int* h_color = nullptr;   // n each, pinned
  int* h_prev = nullptr;
  int* h_prop = nullptr;
  int* h_live = nullptr;
  long long* h_pre = nullptr;  // n + 1: row starts in h_rows
  int* h_rows = nullptr;       // live neighbours, local ids, row after row
  long long rows_cap = 0;
};

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Row capacity of a packed row: the rule of the device repack (dc_misc.cu).
long long packed_cap_host(int live, float slack) {
  if (live <= 0) return 0;
  long long want = (long long)std::ceil((float)live * slack);
  if (want < (long long)live + 4) want = (long long)live + 4;
  return (want + 3) & ~3ll;
}

}  // namespace

struct dc_pool {
  dc_pool_options opt{};
  dc_ctx* u = nullptr;
  int G = 0;  // graph capacity; gid G marks free vertex ids
  std::vector<PGraph> graphs;
  std::map<int, int> freemap;  // free vertex-id ranges: start -> length
  unsigned long long clock = 0;
  int* stage = nullptr;
  long long stage_cap = 0;
  long long* d_pre = nullptr;     // kChunkVertices + 1
  long long* h_prerel = nullptr;  // pinned, kChunkVertices + 1
  long long* h_off = nullptr;     // pinned, hv_cap
  int* h_cap = nullptr;           // pinned, hv_cap
  long long hv_cap = 0;
  dc_change* h_lines = nullptr;   // pinned union batch
  long long lines_cap = 0;
  int* h_giters = nullptr;        // pinned, G + 1
  int* h_ranges = nullptr;        // pinned: the index ranges of a launch (HriBufs::ranges)
  std::unordered_map<void*, long long> hsizes;
  long long host_bytes = 0;
  long long budget = 0;  // adjacency slots for the packed rows of resident graphs
  long long hard = 0;    // the pool never grows past this
  dc_pool_info info{};
};

namespace {

dc_status pfail(dc_pool* P, dc_status s, const std::string& what) { return fail(P->u, s, what); }

template <class T>
dc_status halloc(dc_pool* P, T** p, long long count) {
  if (*p) {
    auto it = P->hsizes.find((void*)*p);
    if (it != P->hsizes.end()) {
      P->host_bytes -= it->second;
      P->hsizes.erase(it);
    }
    cudaFreeHost(*p);
    *p = nullptr;
  }
  if (count <= 0) count = 1;
  const size_t bytes = (size_t)count * sizeof(T);
  if (cudaMallocHost((void**)p, bytes) != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return pfail(P, DC_E_NOMEM, "cudaMallocHost (" + std::to_string(bytes) + " bytes)");
  }
  P->hsizes[(void*)*p] = (long long)bytes;
  P->host_bytes += (long long)bytes;
  return DC_OK;
}

template <class T>
void hfree(dc_pool* P, T** p) {
  if (!*p) return;
  auto it = P->hsizes.find((void*)*p);
  if (it != P->hsizes.end()) {
    P->host_bytes -= it->second;
    P->hsizes.erase(it);
  }
  cudaFreeHost(*p);
  *p = nullptr;
}

// ---- vertex-id ranges ------------------------------------------------------

bool find_range(const dc_pool* P, int n, int* start) {
  if (n == 0) {
    *start = 0;
    return true;
  }
  int best = -1, best_len = 0;
  for (const auto& r : P->freemap)
    if (r.second >= n && (best < 0 || r.second < best_len)) {
      best = r.first;
      best_len = r.second;
    }
  if (best < 0) return false;
  *start = best;
  return true;
}

// [start, start + n) lies inside one free range (which may have merged with
// its neighbours since find_range).
void take_range(dc_pool* P, int start, int n) {
  if (n == 0) return;
  auto it = P->freemap.upper_bound(start);
  --it;
  const int s = it->first, l = it->second;
  P->freemap.erase(it);
  if (start > s) P->freemap[s] = start - s;
  if (s + l > start + n) P->freemap[start + n] = s + l - (start + n);
}

void give_range(dc_pool* P, int start, int n) {
  if (n == 0) return;
  int s = start, l = n;
  auto next = P->freemap.lower_bound(start);
  if (next != P->freemap.end() && next->first == s + l) {
    l += next->second;
    next = P->freemap.erase(next);
  }
  if (next != P->freemap.begin()) {
    auto prev = std::prev(next);
    if (prev->first + prev->second == s) {
      s = prev->first;
      l += prev->second;
      P->freemap.erase(prev);
    }
  }
  P->freemap[s] = l;
}

int lru_victim(const dc_pool* P, const std::vector<char>& locked) {
  int best = -1;
  for (int i = 0; i < (int)P->graphs.size(); ++i) {
    const PGraph& g = P->graphs[(size_t)i];
    if (!g.resident || (i < (int)locked.size() && locked[(size_t)i])) continue;
    if (best < 0 || g.last_use < P->graphs[(size_t)best].last_use) best = i;
  }
  return best;
}

dc_status read_used(dc_pool* P, long long* used) {
  dc_ctx* ctx = P->u;
  DC_CK(cudaMemcpyAsync(ctx->h_scalar, &ctx->st->pool_used, 8, cudaMemcpyDeviceToHost, ctx->stream));
  DC_CK(cudaStreamSynchronize(ctx->stream));
  *used = (long long)ctx->h_scalar[0];
  return DC_OK;
}

// Compacts the pool to max(budget, packed rows + extra) slots: back to the
// budget when the resident rows allow it, past it (up to the hard limit)
// when the graphs that must stay resident need more.
dc_status compact(dc_pool* P, long long extra) {
  dc_ctx* ctx = P->u;
  const double t0 = now_ms();
  long long T = 0;
  dc_status s = packed_total(ctx, &T, nullptr);
  if (s != DC_OK) return s;
  const long long target = (std::max(P->budget, T + extra) + 3) & ~3ll;
  if (target > P->hard)
    return pfail(P, DC_E_NOMEM, "resident rows need " + std::to_string(T + extra) +
                                    " adjacency slots, past the pool's hard limit of " + std::to_string(P->hard));
  if ((s = repack(ctx, target)) != DC_OK) return s;
  ctx->max_pool_cap = target;  // growth inside a launch stops here
  if (target > P->budget) ++P->info.overbudget;
  ++P->info.compactions;
  DC_CK(cudaStreamSynchronize(ctx->stream));
  P->info.compact_ms += now_ms() - t0;
  return DC_OK;
}

// Splits rows [0, n) into chunks of at most kChunkVertices rows and
// stage_cap slots; a row longer than the stage grows the stage.
dc_status next_chunk(dc_pool* P, const long long* pre, int n, int v0, int* v1) {
  const long long lim = std::min<long long>(n, (long long)v0 + kChunkVertices);
  if (pre[v0 + 1] - pre[v0] > P->stage_cap) {
    dc_status s = dalloc(P->u, &P->stage, pre[v0 + 1] - pre[v0], "pool staging");
    if (s != DC_OK) return s;
    P->stage_cap = pre[v0 + 1] - pre[v0];
  }
  // largest v with pre[v] - pre[v0] <= stage_cap, v <= lim
  long long lo = v0 + 1, hi = lim;
  while (lo < hi) {
    const long long mid = (lo + hi + 1) / 2;
    if (pre[mid] - pre[v0] <= P->stage_cap) lo = mid; else hi = mid - 1;
  }
  *v1 = (int)lo;
  return DC_OK;
}

dc_status upload_prerel(dc_pool* P, const long long* pre, int v0, int v1) {
  dc_ctx* ctx = P->u;
  for (int i = 0; i <= v1 - v0; ++i) P->h_prerel[i] = pre[v0 + i] - pre[v0];
  DC_CK(cudaMemcpyAsync(P->d_pre, P->h_prerel, (size_t)(v1 - v0 + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
  return DC_OK;
}

// The graph's pinned host slot: per-vertex arrays, and rows for at least
// `rows` ids.  Rows grow by half again when they outgrow the slot, so a
// graph that keeps growing is not re-pinned at every spill (pinning costs
// far more per byte than copying).
dc_status host_slot(dc_pool* P, PGraph& g, long long rows) {
  dc_status s;
  const int n = g.n;
  if (!g.h_color) {
    if ((s = halloc(P, &g.h_color, n)) != DC_OK) return s;
    if ((s = halloc(P, &g.h_prev, n)) != DC_OK) return s;
    if ((s = halloc(P, &g.h_prop, n)) != DC_OK) return s;
    if ((s = halloc(P, &g.h_live, n)) != DC_OK) return s;
    if ((s = halloc(P, &g.h_pre, (long long)n + 1)) != DC_OK) return s;
  }
  if (rows > g.rows_cap) {
    const long long cap = std::max(rows, g.rows_cap + g.rows_cap / 2);
    if ((s = halloc(P, &g.h_rows, cap)) != DC_OK) return s;
    g.rows_cap = cap;
  }
  return DC_OK;
}

// Moves a resident graph to pinned host memory and frees its vertex ids.
dc_status spill(dc_pool* P, int gi) {
  dc_ctx* ctx = P->u;
  PGraph& g = P->graphs[(size_t)gi];
  if (!g.resident) return DC_OK;
  const double t0 = now_ms();
  const int f = g.first, n = g.n;
  dc_status s;
  if ((s = host_slot(P, g, 0)) != DC_OK) return s;
  const size_t nb = (size_t)n * 4;
  if (n > 0) {
    DC_CK(cudaMemcpyAsync(g.h_live, ctx->live + f, nb, cudaMemcpyDeviceToHost, ctx->stream));
    DC_CK(cudaMemcpyAsync(g.h_color, ctx->color + f, nb, cudaMemcpyDeviceToHost, ctx->stream));
    DC_CK(cudaMemcpyAsync(g.h_prev, ctx->prev + f, nb, cudaMemcpyDeviceToHost, ctx->stream));
    DC_CK(cudaMemcpyAsync(g.h_prop, ctx->prop + f, nb, cudaMemcpyDeviceToHost, ctx->stream));
    DC_CK(cudaStreamSynchronize(ctx->stream));
  }
  long long packed = 0;
  int maxc = 0;
  g.h_pre[0] = 0;
  for (int v = 0; v < n; ++v) {
    g.h_pre[v + 1] = g.h_pre[v] + g.h_live[v];
    packed += packed_cap_host(g.h_live[v], ctx->opt.slack);
    maxc = std::max(maxc, g.h_color[v]);
  }
  const long long S = g.h_pre[n];
  if ((s = host_slot(P, g, S)) != DC_OK) return s;
  const GraphDev gd = graph_dev(ctx);
  for (int v0 = 0; v0 < n;) {
    int v1 = v0;
    if ((s = next_chunk(P, g.h_pre, n, v0, &v1)) != DC_OK) return s;
    if ((s = upload_prerel(P, g.h_pre, v0, v1)) != DC_OK) return s;
    DC_CK(launch_range_gather(gd, f, f + v0, v1 - v0, P->d_pre, P->stage, ctx->stream));
    const long long cnt = g.h_pre[v1] - g.h_pre[v0];
    if (cnt > 0)
      DC_CK(cudaMemcpyAsync(g.h_rows + g.h_pre[v0], P->stage, (size_t)cnt * 4, cudaMemcpyDeviceToHost,
                            ctx->stream));
    DC_CK(cudaStreamSynchronize(ctx->stream));  // stage and h_prerel are reused
    v0 = v1;
  }
  if (n > 0) {
    // the ids become free: isolated, uncoloured, outside every graph
    DC_CK(cudaMemsetAsync(ctx->len + f, 0, nb, ctx->stream));
    DC_CK(cudaMemsetAsync(ctx->cap + f, 0, nb, ctx->stream));
    DC_CK(cudaMemsetAsync(ctx->live + f, 0, nb, ctx->stream));
    DC_CK(cudaMemsetAsync(ctx->color + f, 0, nb, ctx->stream));
    DC_CK(cudaMemsetAsync(ctx->prev + f, 0xff, nb, ctx->stream));
    DC_CK(cudaMemsetAsync(ctx->prop + f, 0, nb, ctx->stream));
    DC_CK(launch_fill(ctx->gid + f, n, P->G, ctx->stream));
    DC_CK(cudaStreamSynchronize(ctx->stream));
  }
  give_range(P, f, n);
  g.resident = false;
  g.first = -1;
  g.host_valid = true;
  g.packed = packed;
  g.max_color = maxc;
  ++P->info.spills;
  P->info.spill_bytes += (long long)nb * 4 + S * 4;
  P->info.spill_ms += now_ms() - t0;
  return DC_OK;
}

// Finds vertex ids [start, start + n) and `need` free slots at the pool's
// tail: evicts least recently used unlocked graphs until the packed rows of
// the resident graphs plus `need` fit the budget (or nothing is left to
// evict), then compacts when the tail is short.  *base = the tail's start.
dc_status make_room(dc_pool* P, int n, long long need, const std::vector<char>& locked, int* start,
                    long long* base) {
  dc_ctx* ctx = P->u;
  dc_status s;
  if (need > P->hard)
    return pfail(P, DC_E_NOMEM, "a graph needs " + std::to_string(need) + " adjacency slots; the pool's hard limit is " +
                                    std::to_string(P->hard));
  while (!find_range(P, n, start)) {
    const int v = lru_victim(P, locked);
    if (v < 0) return pfail(P, DC_E_NOMEM, "vertex capacity exhausted by graphs this launch needs");
    if ((s = spill(P, v)) != DC_OK) return s;
  }
  long long T = 0;
  if ((s = packed_total(ctx, &T, nullptr)) != DC_OK) return s;
  while (T + need > P->budget) {
    const int v = lru_victim(P, locked);
    if (v < 0) break;  // the locked graphs alone exceed the budget
    if ((s = spill(P, v)) != DC_OK) return s;
    T -= P->graphs[(size_t)v].packed;
  }
  long long used = 0;
  if ((s = read_used(P, &used)) != DC_OK) return s;
  if (used + need > ctx->pool_cap || (ctx->pool_cap > P->budget && T + need <= P->budget)) {
    if ((s = compact(P, need)) != DC_OK) return s;
    if ((s = read_used(P, &used)) != DC_OK) return s;
  }
  if (used + need > ctx->pool_cap) return pfail(P, DC_E_NOMEM, "adjacency pool short after compaction");
  *base = used;
  return DC_OK;
}

// After a launch found the pool short (an exhausted launch changes
// nothing): evicts the least recently used unlocked graph, or, with none
// left, grows the pool past the budget toward the hard limit.
dc_status relieve(dc_pool* P, const std::vector<char>& locked, long long lines) {
  dc_ctx* ctx = P->u;
  const int v = lru_victim(P, locked);
  dc_status s;
  if (v >= 0) {
    if ((s = spill(P, v)) != DC_OK) return s;
    return compact(P, 0);
  }
  if (ctx->pool_cap >= P->hard)
    return pfail(P, DC_E_NOMEM, "the graphs of this launch outgrew the pool's hard limit");
  const long long target =
      std::min(P->hard, ctx->pool_cap + std::max(ctx->pool_cap / 2, 4 * lines + 4096)) & ~3ll;
  if ((s = repack(ctx, target)) != DC_OK) return s;
  ctx->max_pool_cap = target;
  ++P->info.overbudget;
  ++P->info.compactions;
  return DC_OK;
}

// Brings a spilled graph back: packed rows appended at the pool's tail.
dc_status restore(dc_pool* P, int gi, const std::vector<char>& locked) {
  dc_ctx* ctx = P->u;
  PGraph& g = P->graphs[(size_t)gi];
  if (g.resident) return DC_OK;
  const double t0 = now_ms();
  const int n = g.n;
  int f = 0;
  long long base = 0;
  dc_status s;
  if ((s = make_room(P, n, g.packed, locked, &f, &base)) != DC_OK) return s;
  if (n > P->hv_cap) {
    if ((s = halloc(P, &P->h_off, n)) != DC_OK) return s;
    if ((s = halloc(P, &P->h_cap, n)) != DC_OK) return s;
    P->hv_cap = n;
  }
  long long at = base;
  for (int v = 0; v < n; ++v) {
    const long long c = packed_cap_host(g.h_live[v], ctx->opt.slack);
    P->h_off[v] = at;
    P->h_cap[v] = (int)c;
    at += c;
  }
  const size_t nb = (size_t)n * 4;
  if (n > 0) {
    DC_CK(cudaMemcpyAsync(ctx->off + f, P->h_off, (size_t)n * 8, cudaMemcpyHostToDevice, ctx->stream));
    DC_CK(cudaMemcpyAsync(ctx->cap + f, P->h_cap, nb, cudaMemcpyHostToDevice, ctx->stream));
    DC_CK(cudaMemcpyAsync(ctx->len + f, g.h_live, nb, cudaMemcpyHostToDevice, ctx->stream));
    DC_CK(cudaMemcpyAsync(ctx->live + f, g.h_live, nb, cudaMemcpyHostToDevice, ctx->stream));
    DC_CK(cudaMemcpyAsync(ctx->color + f, g.h_color, nb, cudaMemcpyHostToDevice, ctx->stream));
    DC_CK(cudaMemcpyAsync(ctx->prev + f, g.h_prev, nb, cudaMemcpyHostToDevice, ctx->stream));
    DC_CK(cudaMemcpyAsync(ctx->prop + f, g.h_prop, nb, cudaMemcpyHostToDevice, ctx->stream));
    DC_CK(launch_fill(ctx->gid + f, n, gi, ctx->stream));
  }
  const GraphDev gd = graph_dev(ctx);
  for (int v0 = 0; v0 < n;) {
    int v1 = v0;
    if ((s = next_chunk(P, g.h_pre, n, v0, &v1)) != DC_OK) return s;
    if ((s = upload_prerel(P, g.h_pre, v0, v1)) != DC_OK) return s;
    const long long cnt = g.h_pre[v1] - g.h_pre[v0];
    if (cnt > 0)
      DC_CK(cudaMemcpyAsync(P->stage, g.h_rows + g.h_pre[v0], (size_t)cnt * 4, cudaMemcpyHostToDevice,
                            ctx->stream));
    DC_CK(launch_range_scatter(gd, f, f + v0, v1 - v0, P->d_pre, P->stage, ctx->stream));
    DC_CK(cudaStreamSynchronize(ctx->stream));  // stage and h_prerel are reused
    v0 = v1;
  }
  ctx->h_scalar[1] = (unsigned long long)at;
  DC_CK(cudaMemcpyAsync(&ctx->st->pool_used, ctx->h_scalar + 1, 8, cudaMemcpyHostToDevice, ctx->stream));
  DC_CK(cudaMemcpyAsync(ctx->h_scalar, &ctx->st->cmax, 4, cudaMemcpyDeviceToHost, ctx->stream));
  DC_CK(cudaStreamSynchronize(ctx->stream));
  int cmax = 0;
  std::memcpy(&cmax, ctx->h_scalar, 4);
  if (g.max_color > cmax) {
    std::memcpy(ctx->h_scalar, &g.max_color, 4);
    DC_CK(cudaMemcpyAsync(&ctx->st->cmax, ctx->h_scalar, 4, cudaMemcpyHostToDevice, ctx->stream));
    DC_CK(cudaStreamSynchronize(ctx->stream));
  }
  take_range(P, f, n);
  g.resident = true;
  g.first = f;
  g.host_valid = false;
  ++P->info.restores;
  P->info.restore_bytes += (long long)nb * 4 + (long long)n * 8 + g.h_pre[n] * 4;
  P->info.restore_ms += now_ms() - t0;
  return DC_OK;
}

bool pool_ready(const dc_pool* P) { return P && P->u && !P->u->broken; }
// Status for a pool that is not ready: DC_E_STATE after a device-side wait
// timed out in its union context, else DC_E_INVAL.
dc_status pool_gate(const dc_pool* P) { return (P && P->u && P->u->broken) ? DC_E_STATE : DC_E_INVAL; }

}  // namespace

extern "C" {

dc_status dc_pool_options_default(dc_pool_options* opt) {
  if (!opt) return DC_E_INVAL;
  std::memset(opt, 0, sizeof(*opt));
  opt->variant = DC_HI;
  opt->max_graphs = 1024;
  opt->vertex_capacity = 1 << 22;
  opt->pool_slots = 1ll << 28;
  opt->iter_cap = 1 << 20;
  opt->slack = 1.25f;
  opt->unit_slots = kUnitSlotsDefault;
  opt->stage_slots = kStageDefault;
  return DC_OK;
}

dc_status dc_pool_create(dc_pool** out, const dc_pool_options* opt) {
  if (!out) return DC_E_INVAL;
  *out = nullptr;
  dc_pool_options o;
  if (opt)
    o = *opt;
  else
    dc_pool_options_default(&o);
  if (o.max_graphs <= 0) o.max_graphs = 1024;
  if (o.stage_slots <= 0) o.stage_slots = kStageDefault;
  if (o.vertex_capacity <= 0 || o.pool_slots <= 0 || o.max_graphs >= (1 << 30)) return DC_E_INVAL;
  dc_options co;
  dc_options_default(&co);
  co.variant = o.variant;
  co.device = o.device;
  co.stream = o.stream;
  co.iter_cap = o.iter_cap;
  co.slack = o.slack;
  co.blocks_per_sm = o.blocks_per_sm;
  co.grid_ctas = o.grid_ctas;
  co.unit_slots = o.unit_slots;
  co.cuda_graph = o.cuda_graph;
  dc_pool* P = new (std::nothrow) dc_pool();
  if (!P) return DC_E_NOMEM;
  P->opt = o;
  // Off unless asked for: a launch then builds the heavy-row index over its
  // own graphs' rows only, but on the served benchmark (graphs of 2^14 to
  // 2^20 vertices, batches up to 1M lines) launches ran 1.75x slower with
  // it than with plain scans.
  co.heavy_min_live = o.heavy_min_live > 0 ? o.heavy_min_live : -1;
  dc_status s = dc_create(&P->u, &co);
  if (s != DC_OK) {
    delete P;
    return s;
  }
  dc_ctx* ctx = P->u;
  auto bail = [&](dc_status st) {
    dc_pool_destroy(P);
    return st;
  };
  P->budget = (o.pool_slots + 3) & ~3ll;
  P->hard = std::max(P->budget, (o.pool_slots_max > 0 ? o.pool_slots_max : 2 * o.pool_slots) & ~3ll);
  ctx->max_pool_cap = P->budget;
  ctx->keep_spare = true;  // a pool compacts often
  if ((s = dc_graph_load_edges(ctx, o.vertex_capacity, nullptr, nullptr, 0)) != DC_OK) return bail(s);
  P->G = o.max_graphs;
  const long long G1 = (long long)P->G + 1;
  if ((s = dalloc(ctx, &ctx->gid, o.vertex_capacity, "graph ids")) != DC_OK) return bail(s);
  if ((s = dalloc(ctx, &ctx->gcnt, 2 * G1, "graph counters")) != DC_OK) return bail(s);
  if ((s = dalloc(ctx, &ctx->gf0, G1, "graph counters")) != DC_OK) return bail(s);
  if ((s = dalloc(ctx, &ctx->giters, G1, "graph iterations")) != DC_OK) return bail(s);
  if ((s = dalloc(ctx, &ctx->gstate, G1, "graph states")) != DC_OK) return bail(s);
  if (launch_fill(ctx->gid, o.vertex_capacity, P->G, ctx->stream) != cudaSuccess ||
      cudaMemsetAsync(ctx->giters, 0, (size_t)G1 * 4, ctx->stream) != cudaSuccess)
    return bail(DC_E_CUDA);
  ctx->ngraphs = (int)G1;
  if ((s = dalloc(ctx, &P->stage, o.stage_slots, "pool staging")) != DC_OK) return bail(s);
  P->stage_cap = o.stage_slots;
  if ((s = dalloc(ctx, &P->d_pre, kChunkVertices + 1, "pool chunk offsets")) != DC_OK) return bail(s);
  if ((s = halloc(P, &P->h_prerel, kChunkVertices + 1)) != DC_OK) return bail(s);
  if ((s = halloc(P, &P->h_giters, G1)) != DC_OK) return bail(s);
  if ((s = halloc(P, &P->h_ranges, 2 * G1 + 2)) != DC_OK) return bail(s);
  if ((s = dalloc(P->u, &P->u->d_ranges, 2 * G1 + 2, "index ranges")) != DC_OK) return bail(s);
  P->u->ranges_cap = 2 * G1 + 2;
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return bail(DC_E_CUDA);
  P->freemap[0] = o.vertex_capacity;
  *out = P;
  return DC_OK;
}

void dc_pool_destroy(dc_pool* P) {
  if (!P) return;
  if (P->u) {
    cudaSetDevice(P->u->device);
    cudaGetLastError();
    if (P->u->stream) cudaStreamSynchronize(P->u->stream);
    dfree(P->u, &P->stage);
    dfree(P->u, &P->d_pre);
  }
  for (PGraph& g : P->graphs) {
    hfree(P, &g.h_color);
    hfree(P, &g.h_prev);
    hfree(P, &g.h_prop);
    hfree(P, &g.h_live);
    hfree(P, &g.h_pre);
    hfree(P, &g.h_rows);
  }
  hfree(P, &P->h_prerel);
  hfree(P, &P->h_off);
  hfree(P, &P->h_cap);
  hfree(P, &P->h_lines);
  hfree(P, &P->h_giters);
  hfree(P, &P->h_ranges);
  if (P->u) dc_destroy(P->u);
  delete P;
}

dc_status dc_pool_add_graph(dc_pool* P, int32_t n, const int32_t* a, const int32_t* b, int64_t m,
                            const int32_t* colors, int32_t* graph) {
  if (!pool_ready(P)) return pool_gate(P);
  if (!graph) return DC_E_INVAL;
  dc_ctx* ctx = P->u;
  if (n < 0 || m < 0 || (m > 0 && (!a || !b)) || (n > 0 && !colors))
    return pfail(P, DC_E_INVAL, "bad graph arguments");
  if ((int)P->graphs.size() >= P->G) return pfail(P, DC_E_INVAL, "the pool holds max_graphs graphs already");
  if (n > P->opt.vertex_capacity) return pfail(P, DC_E_NOMEM, "graph larger than the pool's vertex capacity");
  for (int64_t i = 0; i < m; ++i)
    if (a[i] < 0 || a[i] >= n || b[i] < 0 || b[i] >= n || a[i] == b[i])
      return pfail(P, DC_E_INVAL, "edge " + std::to_string(i) + " has an id outside [0,n) or is a self-loop");
  int maxc = 0;
  for (int32_t v = 0; v < n; ++v) {
    if (colors[v] < 0 || colors[v] > kColorMask)
      return pfail(P, DC_E_INVAL, "colour outside [0, 2^30) at vertex " + std::to_string(v));
    maxc = std::max(maxc, colors[v]);
  }
  cudaSetDevice(ctx->device);
  cudaGetLastError();
  const int gi = (int)P->graphs.size();
  P->graphs.emplace_back();
  P->graphs.back().n = n;
  std::vector<char> locked(P->graphs.size(), 0);
  locked[(size_t)gi] = 1;
  auto undo = [&](dc_status st) {
    P->graphs.pop_back();
    return st;
  };
  // the structural kernel gives every new row packed_cap(degree) slots
  const long long need = (long long)std::ceil(2.0 * (double)m * ctx->opt.slack) + 8ll * n;
  int f = 0;
  long long base = 0;
  dc_status s;
  if ((s = make_room(P, n, std::min(need, P->budget), locked, &f, &base)) != DC_OK) return undo(s);
  take_range(P, f, n);
  PGraph& g = P->graphs[(size_t)gi];
  g.resident = true;
  g.first = f;
  g.max_color = maxc;
  g.last_use = ++P->clock;
  if (n > 0) {
    DC_CK(launch_fill(ctx->gid + f, n, gi, ctx->stream));
    DC_CK(cudaMemcpyAsync(ctx->color + f, colors, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
  }
  if (m > 0) {
    const long long piece = std::min<long long>(m, kPoolLoadPiece);
    std::vector<int> sa((size_t)piece), sb((size_t)piece);
    int* da = nullptr;
    int* db = nullptr;
    if ((s = dalloc(ctx, &da, piece, "load pairs")) != DC_OK) return s;
    if ((s = dalloc(ctx, &db, piece, "load pairs")) != DC_OK) {
      dfree(ctx, &da);
      return s;
    }
    for (long long at = 0; at < m && s == DC_OK; at += piece) {
      const long long len = std::min<long long>(piece, m - at);
      for (long long i = 0; i < len; ++i) {
        sa[(size_t)i] = a[at + i] + f;
        sb[(size_t)i] = b[at + i] + f;
      }
      cudaMemcpyAsync(da, sa.data(), (size_t)len * 4, cudaMemcpyHostToDevice, ctx->stream);
      cudaMemcpyAsync(db, sb.data(), (size_t)len * 4, cudaMemcpyHostToDevice, ctx->stream);
      for (;;) {
        s = run_batch(ctx, nullptr, da, db, len, false, nullptr);
        if (s != DC_E_NOMEM) break;
        // the rows outgrew the estimate: make room and retry
        if ((s = relieve(P, locked, len)) != DC_OK) break;
      }
    }
    dfree(ctx, &da);
    dfree(ctx, &db);
    if (s != DC_OK) return s;  // the graph stays registered and resident, partly loaded
  }
  // cmax bound and the exact packed size
  std::vector<int> live((size_t)std::max(n, 1));
  if (n > 0) DC_CK(cudaMemcpyAsync(live.data(), ctx->live + f, (size_t)n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  DC_CK(cudaMemcpyAsync(ctx->h_scalar, &ctx->st->cmax, 4, cudaMemcpyDeviceToHost, ctx->stream));
  DC_CK(cudaStreamSynchronize(ctx->stream));
  long long packed = 0;
  for (int v = 0; v < n; ++v) packed += packed_cap_host(live[(size_t)v], ctx->opt.slack);
  g.packed = packed;
  // the host slot is pinned now, while the graph is registered, not at its
  // first spill in the middle of serving
  long long live_total = 0;
  for (int v = 0; v < n; ++v) live_total += live[(size_t)v];
  if ((s = host_slot(P, g, live_total + live_total / 4)) != DC_OK) return s;
  int cmax = 0;
  std::memcpy(&cmax, ctx->h_scalar, 4);
  if (maxc > cmax) {
    std::memcpy(ctx->h_scalar, &maxc, 4);
    DC_CK(cudaMemcpyAsync(&ctx->st->cmax, ctx->h_scalar, 4, cudaMemcpyHostToDevice, ctx->stream));
    DC_CK(cudaStreamSynchronize(ctx->stream));
  }
  *graph = gi;
  return DC_OK;
}

dc_status dc_pool_apply(dc_pool* P, const dc_pool_request* reqs, int32_t count, dc_pool_result* results,
                        dc_stats* stats) {
  if (!pool_ready(P)) return pool_gate(P);
  dc_ctx* ctx = P->u;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (count < 0 || (count > 0 && !reqs)) return pfail(P, DC_E_INVAL, "bad request arguments");
  std::vector<char> locked(P->graphs.size(), 0);
  long long K = 0, nsum = 0, slots = 0;
  for (int32_t i = 0; i < count; ++i) {
    const dc_pool_request& r = reqs[i];
    if (r.graph < 0 || r.graph >= (int)P->graphs.size())
      return pfail(P, DC_E_INVAL, "request " + std::to_string(i) + ": unknown graph");
    if (locked[(size_t)r.graph])
      return pfail(P, DC_E_INVAL, "request " + std::to_string(i) + ": a second batch for one graph in a launch");
    if (r.k < 0 || (r.k > 0 && !r.lines)) return pfail(P, DC_E_INVAL, "request " + std::to_string(i) + ": bad lines");
    const int n = P->graphs[(size_t)r.graph].n;
    for (int64_t j = 0; j < r.k; ++j) {
      const dc_change& c = r.lines[j];
      if (c.inst != 0 && c.inst != 1) continue;  // ignored line
      if (c.node1 < 0 || c.node1 >= n || c.node2 < 0 || c.node2 >= n || c.node1 == c.node2)
        return pfail(P, DC_E_INVAL, "request " + std::to_string(i) + " line " + std::to_string(j) +
                                        ": vertex id outside [0,n) or a self-loop");
    }
    locked[(size_t)r.graph] = 1;
    K += r.k;
    nsum += n;
    slots += P->graphs[(size_t)r.graph].packed;
  }
  if (nsum > P->opt.vertex_capacity || slots > P->hard)
    return pfail(P, DC_E_NOMEM, "the graphs of this launch do not fit the pool together");
  if (K > (1ll << 30)) return pfail(P, DC_E_INVAL, "more than 2^30 change lines in one launch");
  cudaSetDevice(ctx->device);
  cudaGetLastError();
  dc_status s;
  for (int32_t i = 0; i < count; ++i) {
    PGraph& g = P->graphs[(size_t)reqs[i].graph];
    const bool was = g.resident;
    if ((s = restore(P, reqs[i].graph, locked)) != DC_OK) return s;
    if (results) {
      results[i].restored = was ? 0 : 1;
      results[i].iterations = 0;
    }
  }
  if (K > P->lines_cap) {
    if ((s = halloc(P, &P->h_lines, K)) != DC_OK) return s;
    P->lines_cap = K;
  }
  long long w = 0;
  for (int32_t i = 0; i < count; ++i) {
    const dc_pool_request& r = reqs[i];
    const int f = P->graphs[(size_t)r.graph].first;
    dc_change* dst = P->h_lines + w;
#pragma omp parallel for schedule(static) if (r.k > (1 << 16))
    for (int64_t j = 0; j < r.k; ++j) {
      dst[j].node1 = r.lines[j].node1 + f;
      dst[j].node2 = r.lines[j].node2 + f;
      dst[j].inst = r.lines[j].inst;
    }
    w += r.k;
  }
  if (K > 0) {
    // the launch's graphs: the only rows its heavy-row index needs
    {
      int* r = P->h_ranges;
      long long tot = 0;
      r[0] = count;
      for (int32_t i = 0; i < count; ++i) {
        const PGraph& g = P->graphs[(size_t)reqs[i].graph];
        r[2 + 2 * i] = g.first;
        r[3 + 2 * i] = (int)tot;
        tot += g.n;
      }
      r[1] = (int)tot;
      DC_CK(cudaMemcpyAsync(ctx->d_ranges, r, (size_t)(2 + 2 * count) * sizeof(int), cudaMemcpyHostToDevice,
                            ctx->stream));
      ctx->index_n = std::max<long long>(tot, 1);
    }
    for (;;) {
      s = dc_apply_batch(ctx, P->h_lines, K, stats);
      if (s != DC_E_NOMEM) break;
      // rows grew past the pool: make room and retry
      dc_status s2 = relieve(P, locked, K);
      if (s2 != DC_OK) return s2;
    }
    if (s != DC_OK && s != DC_E_ITER_LIMIT) return s;
    DC_CK(cudaMemcpyAsync(P->h_giters, ctx->giters, (size_t)(P->G + 1) * 4, cudaMemcpyDeviceToHost, ctx->stream));
    DC_CK(cudaStreamSynchronize(ctx->stream));
    if (results)
      for (int32_t i = 0; i < count; ++i) results[i].iterations = P->h_giters[reqs[i].graph];
  } else {
    s = DC_OK;
  }
  for (int32_t i = 0; i < count; ++i) P->graphs[(size_t)reqs[i].graph].last_use = ++P->clock;
  ++P->info.launches;
  return s;
}

dc_status dc_pool_colors_read(dc_pool* P, int32_t graph, int32_t* out, int32_t n) {
  if (!pool_ready(P)) return pool_gate(P);
  dc_ctx* ctx = P->u;
  if (graph < 0 || graph >= (int)P->graphs.size()) return pfail(P, DC_E_INVAL, "unknown graph");
  const PGraph& g = P->graphs[(size_t)graph];
  if (n != g.n || (n > 0 && !out)) return pfail(P, DC_E_INVAL, "output size differs from the graph's n");
  if (n == 0) return DC_OK;
  if (g.resident) {
    cudaSetDevice(ctx->device);
    cudaGetLastError();
    DC_CK(cudaMemcpyAsync(out, ctx->color + g.first, (size_t)n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    DC_CK(cudaStreamSynchronize(ctx->stream));
  } else {
    std::memcpy(out, g.h_color, (size_t)n * 4);
  }
  return DC_OK;
}

dc_status dc_pool_spill(dc_pool* P, int32_t graph) {
  if (!pool_ready(P)) return pool_gate(P);
  if (graph < 0 || graph >= (int)P->graphs.size()) return pfail(P, DC_E_INVAL, "unknown graph");
  cudaSetDevice(P->u->device);
  cudaGetLastError();
  return spill(P, graph);
}

dc_status dc_pool_graph_size(dc_pool* P, int32_t graph, int32_t* n, int64_t* slots, int32_t* resident) {
  if (!pool_ready(P)) return pool_gate(P);
  if (graph < 0 || graph >= (int)P->graphs.size()) return pfail(P, DC_E_INVAL, "unknown graph");
  const PGraph& g = P->graphs[(size_t)graph];
  if (n) *n = g.n;
  if (slots) *slots = g.packed;
  if (resident) *resident = g.resident ? 1 : 0;
  return DC_OK;
}

dc_status dc_pool_info_get(dc_pool* P, dc_pool_info* info) {
  if (!pool_ready(P)) return pool_gate(P);
  if (!info) return DC_E_INVAL;
  cudaSetDevice(P->u->device);
  cudaGetLastError();
  long long used = 0;
  dc_status s = read_used(P, &used);
  if (s != DC_OK) return s;
  *info = P->info;
  info->graphs = (int32_t)P->graphs.size();
  info->resident = 0;
  info->resident_vertices = 0;
  for (const PGraph& g : P->graphs)
    if (g.resident) {
      ++info->resident;
      info->resident_vertices += g.n;
    }
  info->vertex_capacity = P->opt.vertex_capacity;
  info->pool_slots_used = used;
  info->pool_slots = P->u->pool_cap;
  info->pool_slots_budget = P->budget;
  info->pool_slots_max = P->hard;
  info->device_bytes = P->u->bytes;
  info->host_bytes = P->host_bytes;
  return DC_OK;
}

const char* dc_pool_last_error(const dc_pool* P) {
  if (!P || !P->u) return "null pool";
  return dc_last_error(P->u);
}

}  // extern "C"
