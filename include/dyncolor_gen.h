/*
 * dyncolor_gen.h -- seeded workload generators of libdyncolor (host C++,
 * OpenMP).  They produce the synthetic inputs the benchmarks and tests run
 * on; the reference itself ships no generator (it reads text files, see
 * HI/all_structure_undir.cuh:78-183), so these have no reference
 * counterpart.  Every generator is deterministic for a given seed,
 * independent of the thread count.
 */
#ifndef DYNCOLOR_GEN_H
#define DYNCOLOR_GEN_H
#include <stdint.h>

#include "dyncolor.h"

#ifdef __cplusplus
extern "C" {
#endif

/* m R-MAT samples over 2^scale vertices with quadrant probabilities a, b, c
 * (d = 1-a-b-c), no noise and no vertex permutation.  Raw pairs: may hold
 * self-loops and duplicates.  Vertex ids >= n (when n < 2^scale) are folded
 * by modulo n. */
int dcg_rmat(int32_t scale, int32_t n, int64_t m, double a, double b, double c, uint64_t seed,
             int32_t* out_a, int32_t* out_b);

/* m uniform pairs over [0, n). */
int dcg_uniform_pairs(int32_t n, int64_t m, uint64_t seed, int32_t* out_a, int32_t* out_b);

/* Chung-Lu sampling: expected degree of vertex i is
 *   w_i = max_deg * (1 + i/i0)^(-1/(gamma-1)),
 * i0 chosen so that the mean of w is avg_deg; m = n*avg_deg/2 pairs with
 * both endpoints drawn proportionally to w.  Writes at most m_cap pairs and
 * returns the number written (negative on error). */
int64_t dcg_chung_lu(int32_t n, double gamma, double avg_deg, double max_deg, uint64_t seed,
                     int32_t* out_a, int32_t* out_b, int64_t m_cap);

/* Drops self-loops, orders every pair (min, max), sorts and removes
 * duplicates in place.  Returns the new number of pairs. */
int64_t dcg_dedup(int32_t n, int32_t* a, int32_t* b, int64_t m);

/* Greedy lowest-free colour in vertex-id order over the undirected edge
 * list: colors[v] = mex{colors[u] : u < v, u ~ v}. */
int dcg_greedy_color(int32_t n, const int32_t* a, const int32_t* b, int64_t m, int32_t* colors);

/* Edge set used to draw update batches against the current graph. */
typedef struct dcg_edgeset dcg_edgeset;

/* Takes a deduplicated edge list (as from dcg_dedup). */
dcg_edgeset* dcg_edgeset_create(int32_t n, const int32_t* a, const int32_t* b, int64_t m);
void dcg_edgeset_destroy(dcg_edgeset* s);
int64_t dcg_edgeset_size(const dcg_edgeset* s);

enum {
  DCG_INS_UNIFORM = 0, /* both endpoints uniform over [0, n) */
  DCG_INS_RMAT = 1,    /* endpoints from R-MAT(scale, a, b, c) */
  DCG_INS_DEGREE = 2   /* one endpoint proportional to degree, the other uniform */
};

/* Draws one batch: k_del deletions of distinct edges present in the
 * original edge list and not deleted yet (uniform), and k_ins insertions of
 * distinct pairs absent from the current graph and not deleted by this batch
 * (self-loops excluded), then applies it to the set.  Lines are shuffled.  out holds k_del + k_ins
 * lines.  Returns the number of lines written. */
int64_t dcg_edgeset_sample_batch(dcg_edgeset* s, int64_t k_del, int64_t k_ins, int32_t ins_mode,
                                 int32_t scale, double a, double b, double c, uint64_t seed,
                                 dc_change* out);

#ifdef __cplusplus
}
#endif
#endif
