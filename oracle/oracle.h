/*
 * oracle.h -- CPU restatement of DynColor's single-GPU recoloring path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the parity tests,
 * `__graft_entry__.smoke()` and the CPU-baseline leg of `bench.py` compare
 * the CUDA path against.  Nothing in the product (the dyncolor_b200 package,
 * libdyncolor.so) links, loads or calls it.
 *
 * It restates, in plain C, the reference's host and kernel logic:
 *   - text/host side: read_graphEdges, readin_changes
 *       HI/all_structure_undir.cuh:78-128, 156-183
 *       HB/all_structure_undir.cuh:78-129, 158-186 (LDF degree property)
 *   - structural delete: deleteEdgeFromAdj   HI/gpuFunctions_undir.cuh:118-142
 *   - HI seeding:  deleteEdge, insEdge       HI/gpuFunctions_undir.cuh:147-223
 *   - HB seeding:  processChangeEdge          HB/gpuFunctions_undir.cuh:222-249
 *   - loop: findEligibleNeighbors, compact, recolorNeighbor
 *       HI/gpuFunctions_undir.cuh:229-284, HB/gpuFunctions_undir.cuh:259-314,
 *       HI/compactor.cuh:79-173, HI/Color_main.cu:176-202,
 *       HB/Color_main.cu:198-224
 *   - validate                               HI/gpuFunctions_undir.cuh:289-305
 *
 * with exact multi-word saturation masks (the reference's 32-bit arithmetic
 * is only exact while every color is <= 30).
 *
 * Two schedules:
 *   ORC_SERIAL   -- every kernel's grid-stride loop run by one thread in
 *                   index order with writes visible immediately; this is
 *                   what the reference's own code does with one thread, and
 *                   is pinned bit-exactly against it (oracle/_ref).
 *   ORC_SNAPSHOT -- every kernel launch is one step: all reads in a step see
 *                   the state at the start of the step, writes land at the
 *                   end.  Targets of a step are de-duplicated; HB's
 *                   processChangeEdge treats node1 and node2 of every change
 *                   as independent targets of one step.  This is the
 *                   deterministic schedule the CUDA path implements.
 */
#ifndef DYNCOLOR_ORACLE_H
#define DYNCOLOR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_HI = 0, ORC_HB = 1 };
enum { ORC_SNAPSHOT = 0, ORC_SERIAL = 1 };
enum {
  ORC_OK = 0,
  ORC_E_INVAL = 1,
  ORC_E_NOMEM = 2,
  ORC_E_ITER_LIMIT = 4
};

/* One change line: node1 node2 inst (inst 1 = insert, 0 = delete, other
 * values are ignored like readin_changes does). HI/all_structure_undir.cuh:41-45 */
typedef struct {
  int32_t node1;
  int32_t node2;
  int32_t inst;
} orc_change;

typedef struct {
  int64_t iterations;      /* executions of the while(change) body */
  int64_t seed_targets;    /* distinct vertices recomputed by the seeding steps */
  int64_t frontier_total;  /* sum over iterations of |recolor frontier| */
  int64_t slots_scanned;   /* live adjacency entries read by all steps */
  int64_t changed_vertices;/* vertices whose final color differs from the start */
  int32_t status;          /* ORC_OK or ORC_E_ITER_LIMIT */
  int32_t max_color;       /* max color after the batch */
  int64_t internal_pairs;  /* instrumentation: sum over iterations of live
                              directed edges with both ends in the recolor
                              frontier (only with orc_set_instrument(1)) */
} orc_stats;

typedef struct orc_graph orc_graph;

orc_graph* orc_create(int32_t n);
void orc_destroy(orc_graph* g);
/* read_graphEdges: every pair adds a->b and b->a (no de-duplication) and
 * bumps the LDF degree property of both ends. */
int orc_load_edges(orc_graph* g, const int32_t* a, const int32_t* b, int64_t m);
/* read_Input_Color */
int orc_set_colors(orc_graph* g, const int32_t* colors);
int orc_get_colors(const orc_graph* g, int32_t* out);
int orc_get_prop(const orc_graph* g, int32_t* out);
/* readin_changes + deleteEdgeFromAdj + seeding + loop */
int orc_apply_batch(orc_graph* g, int variant, int schedule,
                    const orc_change* ch, int64_t k, int64_t iter_cap,
                    orc_stats* st);
/* validate: number of live adjacency entries (u,v), u<v, with equal colors */
int64_t orc_conflicts(const orc_graph* g);
/* number of live distinct neighbours of v (set semantics) */
int32_t orc_live_degree(const orc_graph* g, int32_t v);
/* distinct live neighbours of v, ascending, into out[cap]; returns their count */
int32_t orc_neighbors(const orc_graph* g, int32_t v, int32_t* out, int32_t cap);
/* 1 if colors[v] == mex{colors[u] : u neighbour of v, u < v} for every v */
int orc_is_greedy_id_order(const orc_graph* g);
/* Greedy lowest-free colour in vertex-id order (same rule as above). */
int orc_greedy_id_order(orc_graph* g);
/* Greedy lowest-free colour with vertices taken in order[0..n). */
int orc_greedy_in_order(orc_graph* g, const int32_t* order);
int32_t orc_num_vertices(const orc_graph* g);
void orc_set_threads(int nthreads);
void orc_set_instrument(int on);

#ifdef __cplusplus
}
#endif
#endif
