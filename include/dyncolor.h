/*
 * dyncolor.h -- C ABI of the B200 incremental graph-recoloring library
 * (libdyncolor.so).
 *
 * It replaces the host phases of the reference's single-GPU drivers
 * (DynColorHeuristicIndependent "HI" and DynColorHeuristicBased "HB"):
 *
 *   graph-load          read_graphEdges + transfer_data_to_GPU
 *                       HI/all_structure_undir.cuh:156-183,
 *                       HB/all_structure_undir.cuh:158-186,
 *                       HI/supportingFunctions.cu:19-101
 *   initial-color       read_Input_Color   HI/all_structure_undir.cuh:130-150
 *   apply-update-batch  readin_changes + deleteEdgeFromAdj + deleteEdge /
 *                       insEdge (HI) or processChangeEdge (HB) + the
 *                       findEligibleNeighbors / compact / recolorNeighbor loop
 *                       HI/all_structure_undir.cuh:78-128,
 *                       HI/gpuFunctions_undir.cuh:118-284,
 *                       HB/gpuFunctions_undir.cuh:104-314,
 *                       HI/Color_main.cu:146-202, HB/Color_main.cu:160-224
 *   read-colors         the managed vertexcolor array, HI/Color_main.cu:211-216
 *   validate            validate kernel, HI/gpuFunctions_undir.cuh:289-305
 *
 * Semantics.  Every reference kernel launch is one step; all reads of a step
 * see the state at the start of the step and its writes land at the end
 * (the reference's kernels race; this library fixes that schedule).  Tie
 * breaks and rules are the reference's; saturation masks are exact over the
 * whole colour range.  The adjacency is a set: inserting an existing edge
 * is a no-op, a deletion removes the edge, and inside one batch every
 * insertion is applied before every deletion (a delete of the same edge
 * wins), as in the reference.
 *
 * Ownership: host arrays passed in are caller-owned and copied; device state
 * is library-owned.  A context is used by one host thread at a time.
 * Every call returns a dc_status; none exits the process.
 */
#ifndef DYNCOLOR_H
#define DYNCOLOR_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  DC_OK = 0,
  DC_E_INVAL = 1,      /* bad argument: id out of range, self-loop, negative colour, ... */
  DC_E_NOMEM = 2,      /* device or host allocation failed */
  DC_E_CUDA = 3,       /* a CUDA runtime call failed (see dc_last_error) */
  DC_E_ITER_LIMIT = 4, /* the recolour loop hit options.iter_cap; colours are partial */
  DC_E_STATE = 5,      /* call out of order (e.g. apply before load) */
  DC_E_TIMEOUT = 6,    /* a device-side wait gave up (grid barrier); the context refuses every
                          later call but dc_destroy/dc_last_error with DC_E_STATE */
  DC_E_INTERNAL = 7    /* a device-side capacity guard fired */
} dc_status;

typedef enum {
  DC_HI = 0, /* heuristic-independent: order by colour value */
  DC_HB = 1  /* heuristic-based: largest-degree-first priority */
} dc_variant;

/* One change line "node1 node2 weight inst" of the reference's change file
 * (changeEdge, HI/all_structure_undir.cuh:41-45): inst 1 inserts, inst 0
 * deletes, any other value is ignored like readin_changes ignores it. */
typedef struct {
  int32_t node1;
  int32_t node2;
  int32_t inst;
} dc_change;

typedef struct {
  int32_t variant;       /* dc_variant */
  int32_t device;        /* CUDA device ordinal */
  void* stream;          /* cudaStream_t to run on; NULL: the library creates one */
  int64_t iter_cap;      /* recolour-loop iteration cap; <= 0: 1<<20 */
  float slack;           /* row capacity = live * slack when a row is (re)allocated; <= 1: 1.25 */
  int32_t blocks_per_sm; /* persistent-kernel CTAs per SM; 0: from occupancy */
  int64_t reserve_slots; /* initial adjacency pool size hint in slots; 0: automatic */
  int32_t unit_slots;    /* adjacency slots per warp work unit (multiple of 128); 0: 4096 */
  int32_t cuda_graph;    /* 1: replay each batch's launches from a captured CUDA graph */
  int32_t heavy_min_live; /* rows with at least this many live slots get a per-batch index (HI: by
                             colour, HB: by priority) used by batches of at least n/256 lines;
                             0: 2048 for HI, 256 for HB; < 0: off.  Results are the same either
                             way. */
  int32_t barrier_timeout_ms; /* limit of every device-side grid-barrier wait; 0: 20,000 ms.  A wait
                                 that runs out ends the launch with DC_E_TIMEOUT instead of hanging,
                                 and the context then refuses further work (DC_E_STATE). */
  int32_t grid_ctas;      /* CTAs of the persistent launches; 0: SMs x blocks_per_sm (or the
                             occupancy).  Fewer CTAs leave SMs to launches on other streams. */
  int32_t reserved[3];
} dc_options;

typedef struct {
  int64_t iterations;     /* executions of the recolour loop body */
  int64_t seed_targets;   /* distinct vertices recomputed by the seeding steps */
  int64_t frontier_total; /* sum over iterations of the recolour frontier size */
  int64_t slots_scanned;  /* live adjacency entries read by seeding + loop */
  int64_t edges_inserted; /* net structural insertions (new edges) */
  int64_t edges_deleted;  /* net structural deletions (edges removed) */
  int64_t rows_relocated; /* adjacency rows moved to new capacity */
  int32_t status;         /* dc_status of the batch */
  int32_t max_color;      /* an upper bound of every colour after the batch */
  double device_ms;       /* device time of the batch (CUDA events) */
  double struct_ms;       /* of which the structural-update launch */
  double recolor_ms;      /* of which the seeding + recolour launch */
  double phase_ms[6];     /* recolour launch split: seeding, find-eligible, mex, commit,
                             2 reserved */
  int64_t slots_read;     /* adjacency entries the kernels actually read (the loop
                             reads each frontier row once per iteration) */
  int64_t pairs;          /* frontier-internal edges the fused loop deferred */
} dc_stats;

typedef struct {
  int32_t n;              /* vertices */
  int64_t edges;          /* live undirected edges */
  int64_t slots_used;     /* adjacency pool slots handed out */
  int64_t slots_capacity; /* adjacency pool capacity in slots */
  int64_t device_bytes;   /* device memory held by the context */
} dc_graph_info;

typedef struct dc_ctx dc_ctx;

/* Fills *opt with defaults (variant HI, device 0, library stream). */
dc_status dc_options_default(dc_options* opt);

/* Creates a context on opt->device. */
dc_status dc_create(dc_ctx** out, const dc_options* opt);
void dc_destroy(dc_ctx* ctx);

/* graph-load (read_graphEdges + transfer_data_to_GPU).  Pair i adds the
 * undirected edge (a[i], b[i]); duplicate pairs collapse; self-loops and ids
 * outside [0, n) are rejected with DC_E_INVAL before anything changes.  The
 * HB degree property counts every pair (duplicates too), like
 * HB/all_structure_undir.cuh:176-178.  Resets colours to 0.  May be called
 * once per context. */
dc_status dc_graph_load_edges(dc_ctx* ctx, int32_t n, const int32_t* a, const int32_t* b,
                              int64_t m);

/* initial-color (read_Input_Color): colours must lie in [0, 2^30). */
dc_status dc_colors_set(dc_ctx* ctx, const int32_t* colors, int32_t n);

/* Orders of the initial colouring. */
typedef enum {
  DC_ORDER_ID = 0, /* vertex-id order */
  DC_ORDER_LDF = 1 /* largest live degree first, ties by lower id */
} dc_order;

/* Initial colouring of the resident graph, not in the reference (whose
 * initial colours come from an external tool, MG/README.txt:19-22): the
 * greedy lowest-free colouring in the given order over the current edge set,
 * computed on the device as a Jones-Plassmann schedule (a vertex is coloured
 * as soon as every neighbour before it in the order is).  The colours equal
 * the sequential greedy pass in that order: with DC_ORDER_ID they are
 * dcg_greedy_color's on the same edges.  DC_ORDER_LDF re-seeds a colouring
 * with the largest-degree-first order, which usually needs fewer colours. */
dc_status dc_colors_init(dc_ctx* ctx, int32_t order);

/* dc_colors_init(ctx, DC_ORDER_ID). */
dc_status dc_colors_init_greedy(dc_ctx* ctx);

/* apply-update-batch from host memory (any host pointer; pinned is fastest).
 * Validates every line first (DC_E_INVAL leaves the state untouched).  Runs
 * the structural update and the recolouring on the context's stream and
 * waits for it.  *out (optional) receives the statistics. */
dc_status dc_apply_batch(dc_ctx* ctx, const dc_change* changes, int64_t k, dc_stats* out);

/* apply-update-batch with the change lines already in device memory. */
dc_status dc_apply_batch_device(dc_ctx* ctx, const dc_change* d_changes, int64_t k,
                                dc_stats* out);

/* read-colors into host memory (n = number of vertices). */
dc_status dc_colors_read(dc_ctx* ctx, int32_t* out, int32_t n);
/* Device pointer of the colour array (valid until the next load/destroy). */
dc_status dc_colors_device(dc_ctx* ctx, int32_t** d_colors);
/* HB degree property, host copy. */
dc_status dc_prop_read(dc_ctx* ctx, int32_t* out, int32_t n);

/* validate: number of live edges {u,v} with equal colours (0 = proper). */
dc_status dc_validate(dc_ctx* ctx, int64_t* conflicts);

/* Adjacency of v (live neighbours, any order) into out[cap]; *deg gets the
 * live degree (may exceed cap). */
dc_status dc_neighbors(dc_ctx* ctx, int32_t v, int32_t* out, int32_t cap, int32_t* deg);

dc_status dc_graph_info_get(dc_ctx* ctx, dc_graph_info* info);

/* Batched mode (no counterpart in the reference, which runs one graph per
 * process): declares the loaded graph to be the disjoint union of ngraphs
 * independent graphs, graph g owning vertices [first[g], first[g+1])
 * (first[0] = 0, first[ngraphs] = n).  DC_E_INVAL if an edge joins two
 * graphs.  Afterwards every batch is applied to all graphs in the same
 * launches, each graph exactly as if it were recoloured alone: HB stops
 * expanding a graph as soon as one of its recolour steps changes nothing,
 * and change lines that join two graphs are rejected. */
dc_status dc_partition_set(dc_ctx* ctx, int32_t ngraphs, const int32_t* first);

/* Batched mode: loop iterations each graph ran in the last batch (what a
 * separate run of that graph would report). */
dc_status dc_graph_iterations(dc_ctx* ctx, int64_t* out, int32_t ngraphs);

/* Re-packs the adjacency (drops tombstones, re-applies slack). */
dc_status dc_compact(dc_ctx* ctx);

/* Colouring check that allocates no device or host memory (no counterpart
 * in the reference).  For callers that cannot let a library call
 * cudaMalloc: a serving process whose device memory is fully budgeted, an
 * application whose own allocator owns every device byte, or code that must
 * avoid the device synchronisation cudaMalloc/cudaFree can cause.  Checks
 * the colouring of a CSR the caller holds in device memory (row r has
 * d_row_len[r] entries from d_adj[d_row_off[r]]; negative entries are
 * skipped as deleted) on the current device and `stream`, and returns the
 * number of monochromatic edges {u,v}, of vertices on such an edge, and the
 * largest colour.  A row that lists the same neighbour twice counts a
 * monochromatic edge once per copy (the library's own rows never do).
 * n must not exceed 16,777,216 (2^24): the scratch bitmap is a fixed 2 MiB
 * device array inside the library, held by every GPU that loads it until
 * the process exits.  Every call looks up that array's device address with
 * the caller's device current (no allocation).  All calls share the array:
 * calls that overlap on the GPU (other streams, other host threads) race.
 * The call waits for `stream` before returning, so it must not be made on a
 * stream that is being captured (DC_E_STATE).  conflicted_vertices and
 * max_color may be NULL.  DC_E_INVAL: n out of range, a negative colour or a
 * neighbour id outside [0, n). */
dc_status dc_validate_csr_noalloc(int32_t n, const int64_t* d_row_off, const int32_t* d_row_len,
                                  const int32_t* d_adj, const int32_t* d_colors, void* stream,
                                  int64_t* conflicts, int64_t* conflicted_vertices,
                                  int32_t* max_color);

/* Last error text of the context (never NULL). */
const char* dc_last_error(const dc_ctx* ctx);
const char* dc_status_str(dc_status s);

#ifdef __cplusplus
}
#endif
#endif
