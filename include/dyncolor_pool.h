/*
 * dyncolor_pool.h -- resident multi-graph pool of libdyncolor (served mode).
 *
 * The reference recolours one graph per process run (HI/Color_main.cu:21-216):
 * every update batch pays a process start, a graph load and a launch
 * sequence.  A pool keeps many graphs resident in one device context under
 * a fixed budget of adjacency slots, and recolours the update batches of
 * several graphs in the same launches.
 *
 *  - Every graph occupies a contiguous range of the pool's vertex ids while
 *    it is resident, and is independent of the others: each ends a launch
 *    with the colours and loop-iteration count a separate run of its batch
 *    would give (the snapshot schedule of dyncolor.h, applied per graph).
 *  - Admission is by budget.  A graph that is not resident is held in pinned
 *    host memory (its rows, colours, previous colours and degree property);
 *    bringing it back evicts the least recently used graphs that the current
 *    launch does not touch until the packed rows of the resident graphs fit
 *    pool_slots, and compacts the adjacency pool when its free tail is too
 *    short.  Spill and reload are exact copies.  Only when the graphs of one
 *    launch alone need more than pool_slots does the pool grow past it, up
 *    to pool_slots_max; otherwise the call fails with DC_E_NOMEM.
 *  - Lines use each graph's own vertex ids [0, n).  Lines with an inst other
 *    than 0 or 1 are ignored, as readin_changes ignores them.
 *
 * A pool is used by one host thread at a time.
 */
#ifndef DYNCOLOR_POOL_H
#define DYNCOLOR_POOL_H
#include "dyncolor.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dc_pool dc_pool;

typedef struct {
  int32_t variant;         /* DC_HI or DC_HB, for every graph of the pool */
  int32_t device;          /* CUDA device ordinal */
  void* stream;            /* cudaStream_t to run on; NULL: the library creates one */
  int32_t max_graphs;      /* graphs that can be registered; <= 0: 1024 */
  int32_t vertex_capacity; /* vertex ids for resident graphs (sum of their n at most) */
  int64_t pool_slots;      /* adjacency slots (4 bytes each) for resident rows: the row budget */
  int64_t iter_cap;        /* recolour-loop iteration cap; <= 0: 1<<20 */
  float slack;             /* row capacity = live * slack when a row is (re)allocated; <= 1: 1.25 */
  int32_t blocks_per_sm;   /* persistent-kernel CTAs per SM; 0: from occupancy */
  int32_t unit_slots;      /* adjacency slots per warp work unit; 0: 4096 */
  int32_t cuda_graph;      /* 1: replay each launch from a captured CUDA graph */
  int64_t stage_slots;     /* device staging for spill and reload (4-byte slots); <= 0: 2^25 */
  int64_t pool_slots_max;  /* hard limit: when the graphs of one launch alone outgrow pool_slots, the
                              pool grows up to this many slots (and shrinks back at the next
                              compaction that allows it); <= 0: 2 * pool_slots */
  int32_t grid_ctas;       /* CTAs of the persistent launches (dc_options.grid_ctas); 0: all */
  int32_t heavy_min_live;  /* > 0: dc_options.heavy_min_live (a launch indexes only the rows of its
                              own graphs, when its lines are at least 1/256 of their vertices);
                              <= 0: off, every row is scanned */
  int32_t reserved[6];
} dc_pool_options;

/* One update batch for one graph. */
typedef struct {
  int32_t graph;           /* id returned by dc_pool_add_graph */
  int32_t pad;
  const dc_change* lines;  /* host array of k lines in the graph's own vertex ids */
  int64_t k;
} dc_pool_request;

typedef struct {
  int64_t iterations;      /* recolour-loop iterations this graph took in the launch */
  int32_t restored;        /* 1: the graph was reloaded from host memory for this launch */
  int32_t pad;
} dc_pool_result;

typedef struct {
  int32_t graphs;          /* registered */
  int32_t resident;
  int64_t resident_vertices;
  int64_t vertex_capacity;
  int64_t pool_slots_used; /* adjacency pool slots handed out (live rows and garbage) */
  int64_t pool_slots;      /* current adjacency pool size */
  int64_t pool_slots_budget;
  int64_t pool_slots_max;
  int64_t overbudget;      /* compactions or launches that took the pool past its budget */
  int64_t spills;
  int64_t restores;
  int64_t spill_bytes;     /* device -> host bytes moved by spills */
  int64_t restore_bytes;   /* host -> device bytes moved by reloads */
  double spill_ms;         /* host wall time inside spills */
  double restore_ms;       /* host wall time inside reloads (compaction included) */
  int64_t launches;
  int64_t compactions;
  int64_t device_bytes;    /* device memory held by the pool */
  int64_t host_bytes;      /* pinned host memory held by the pool */
  double compact_ms;       /* host wall time inside compactions */
} dc_pool_info;

dc_status dc_pool_options_default(dc_pool_options* opt);
dc_status dc_pool_create(dc_pool** out, const dc_pool_options* opt);
void dc_pool_destroy(dc_pool* pool);

/* Registers a graph with the semantics of dc_graph_load_edges + dc_colors_set
 * and makes it resident (evicting others if needed).  *graph gets its id. */
dc_status dc_pool_add_graph(dc_pool* pool, int32_t n, const int32_t* a, const int32_t* b, int64_t m,
                            const int32_t* colors, int32_t* graph);

/* Applies `count` update batches, each to a different graph, in one launch
 * sequence; results[i] (optional) belongs to reqs[i].  stats (optional)
 * describes the whole launch.  On an error no graph has changed, except
 * DC_E_ITER_LIMIT (partial colourings, as dc_apply_batch). */
dc_status dc_pool_apply(dc_pool* pool, const dc_pool_request* reqs, int32_t count, dc_pool_result* results,
                        dc_stats* stats);

dc_status dc_pool_colors_read(dc_pool* pool, int32_t graph, int32_t* out, int32_t n);
/* Moves a graph to pinned host memory now (it is reloaded on its next use). */
dc_status dc_pool_spill(dc_pool* pool, int32_t graph);
/* n, adjacency slots the graph takes when reloaded (as of its last load or
 * spill), and whether it is resident. */
dc_status dc_pool_graph_size(dc_pool* pool, int32_t graph, int32_t* n, int64_t* slots, int32_t* resident);
dc_status dc_pool_info_get(dc_pool* pool, dc_pool_info* info);
const char* dc_pool_last_error(const dc_pool* pool);

#ifdef __cplusplus
}
#endif
#endif /* DYNCOLOR_POOL_H */
