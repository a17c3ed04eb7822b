// dc_ctx.h -- the context object behind the C ABI and the host helpers the
// single-graph API (dc_api.cpp) and the resident pool (dc_pool.cpp) share.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <unordered_map>

#include "../../include/dyncolor.h"
#include "dc_internal.h"

using dc::DevState;
using dc::QueueBufs;
using dc::HriBufs;

struct dc_ctx {
  dc_options opt{};
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sms = 0;
  int grid_struct = 0;
  int grid_recolor = 0;
  std::string err;
  bool broken = false;  // a device-side wait timed out: every later call is refused
  long long bytes = 0;  // device bytes held (dalloc / dfree)
  std::unordered_map<void*, long long> sizes;

  // graph
  int n = -1;
  int key_bits = 1;
  long long pool_cap = 0;
  long long max_pool_cap = 0;  // > 0: pool growth stops here (a resident pool's budget)
  bool keep_spare = false;      // compactions reuse the previous arrays (resident pools)
  struct Spare {
    long long* off = nullptr;
    int* cap = nullptr;
    int* len = nullptr;
    int* adj = nullptr;
    long long adj_cap = 0;
  } spare;
  long long* off = nullptr;
  int* len = nullptr;
  int* cap = nullptr;
  int* live = nullptr;
  int* adj = nullptr;
  int* color = nullptr;
  int* prev = nullptr;
  int* prop = nullptr;
  DevState* st = nullptr;
  DevState* h_st = nullptr;  // pinned
  unsigned long long* d_scalar = nullptr;
  unsigned long long* h_scalar = nullptr;  // pinned

  // recolour scratch (sized by n and pool_cap)
  long long rc_pool_cap = -1;
  QueueBufs qb[3]{};
  unsigned* bmA = nullptr;
  unsigned* bmB = nullptr;
  unsigned* bmC = nullptr;
  int* ncolor = nullptr;
  int* sat = nullptr;
  unsigned long long* cp = nullptr;  // HB: packed (degree property, colour) per vertex
  HriBufs hri{};                     // HI: heavy-row index (min_live 0: off)

  // batch scratch (sized by k and pool_cap)
  long long kcap = 0;
  long long k_pool_cap = -1;
  dc_change* d_ch = nullptr;
  unsigned char* lflag = nullptr;
  unsigned long long* keysA = nullptr;
  unsigned long long* keysB = nullptr;
  unsigned long long* net = nullptr;
  int* tof = nullptr;
  unsigned char* present = nullptr;
  int* rank = nullptr;
  int* tbeg = nullptr;
  int* trow = nullptr;
  int* rowdel = nullptr;
  int* tins = nullptr;
  long long* tnoff = nullptr;
  int* tncap = nullptr;
  int* tnlive = nullptr;
  int* trel = nullptr;
  int* cursor = nullptr;
  long long* delpos = nullptr;
  int2* units = nullptr;
  int2* relunits = nullptr;
  long long cap_units = 0;
  long long cap_rel = 0;
  unsigned* hist = nullptr;
  unsigned* dscan = nullptr;
  unsigned* cta_cnt = nullptr;

  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evm = nullptr;

  // captured batch graph
  cudaGraph_t cgraph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  long long graph_key[6] = {0, 0, 0, 0, 0, 0};
  bool use_index = false;  // this batch builds and uses the heavy-row index
  int* d_ranges = nullptr;  // vertex ranges of the next batch's index (HriBufs::ranges), or unused
  long long ranges_cap = 0; // ints
  long long index_n = 0;    // > 0: the next batch's index covers d_ranges' vertices, this many
  long long* h_k = nullptr;  // pinned line count for the captured graph
  bool last_graph = false;   // the last batch ran from the captured graph

  // batched mode: disjoint union of ngraphs graphs
  int ngraphs = 0;
  int* first = nullptr;   // ngraphs + 1
  int* gid = nullptr;     // n
  int* gcnt = nullptr;    // 2 * ngraphs
  int* gf0 = nullptr;     // ngraphs
  int* giters = nullptr;  // ngraphs
  int* gstate = nullptr;  // ngraphs
};

namespace dc {
namespace host {

inline dc_status fail(dc_ctx* c, dc_status s, const std::string& what) {
  if (c) c->err = what;
  return s;
}

inline dc_status cuda_fail(dc_ctx* c, const char* what, cudaError_t e) {
  return fail(c, e == cudaErrorMemoryAllocation ? DC_E_NOMEM : DC_E_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

#define DC_CK(call)                                      \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(ctx, #call, e_); \
  } while (0)

template <class T>
inline dc_status dalloc(dc_ctx* ctx, T** p, long long count, const char* what) {
  if (*p) {
    auto it = ctx->sizes.find((void*)*p);
    if (it != ctx->sizes.end()) {
      ctx->bytes -= it->second;
      ctx->sizes.erase(it);
    }
    cudaFree(*p);
    *p = nullptr;
  }
  if (count <= 0) count = 1;
  const size_t bytes = (size_t)count * sizeof(T);
  cudaError_t e = cudaMalloc((void**)p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return fail(ctx, DC_E_NOMEM, std::string("cudaMalloc ") + what + " (" + std::to_string(bytes) + " bytes)");
  }
  ctx->bytes += (long long)bytes;
  ctx->sizes[(void*)*p] = (long long)bytes;
  return DC_OK;
}

template <class T>
inline void dfree(dc_ctx* ctx, T** p) {
  if (*p) {
    auto it = ctx->sizes.find((void*)*p);
    if (it != ctx->sizes.end()) {
      ctx->bytes -= it->second;
      ctx->sizes.erase(it);
    }
    cudaFree(*p);
    *p = nullptr;
  }
}

int key_bits_for(int n);
GraphDev graph_dev(const dc_ctx* c);
dc_status ensure_recolor_scratch(dc_ctx* ctx);
dc_status reset_bitmaps(dc_ctx* ctx);
dc_status read_state(dc_ctx* ctx);
dc_status repack(dc_ctx* ctx, long long new_cap);
dc_status packed_total(dc_ctx* ctx, long long* total, long long** scratch_out);
dc_status run_batch(dc_ctx* ctx, const dc_change* d_ch, const int* la, const int* lb, long long k, bool recolor,
                    dc_stats* out);
bool ready(dc_ctx* ctx);
// DC_OK when the context holds a graph and is usable, else the status to return.
dc_status gate(dc_ctx* ctx);

}  // namespace host
}  // namespace dc
