/*
 * oracle.c -- CPU restatement of DynColor's recoloring path (test
 * infrastructure only; see oracle.h for what it restates and why).
 *
 * The adjacency is kept the way the reference keeps it: every row is a list
 * of slots, insertions append (duplicates allowed), deletions tombstone every
 * matching slot (HI/all_structure_undir.cuh:26-29 ColWt{col,flag},
 * HI/gpuFunctions_undir.cuh:118-142).  A tombstoned slot is stored as a
 * negative number.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

struct orc_graph {
  int32_t n;
  int32_t** row;  /* row[v][i] >= 0: live neighbour; < 0: tombstone */
  int32_t* len;
  int32_t* cap;
  int32_t* color;
  int32_t* prev; /* previosVertexcolor, HI only; starts at -1 */
  int32_t* prop; /* vertex_prop (LDF degree), HB only */
};

/* ------------------------------------------------------------------ */
/* small helpers                                                       */
/* ------------------------------------------------------------------ */

static int row_reserve(orc_graph* g, int32_t v, int64_t need) {
  if (need <= g->cap[v]) return 0;
  int64_t nc = g->cap[v] ? (int64_t)g->cap[v] * 2 : 4;
  if (nc < need) nc = need;
  if (nc > 0x7fffffff) return -1;
  int32_t* p = (int32_t*)realloc(g->row[v], (size_t)nc * sizeof(int32_t));
  if (!p) return -1;
  g->row[v] = p;
  g->cap[v] = (int32_t)nc;
  return 0;
}

static int row_push(orc_graph* g, int32_t v, int32_t x) {
  if (row_reserve(g, v, (int64_t)g->len[v] + 1)) return -1;
  g->row[v][g->len[v]++] = x;
  return 0;
}

/* isPrior_RelativeOrdering, HB/gpuFunctions_undir.cuh:104-113:
 * a is prior to b when it has the larger degree property, ties -> lower id. */
static inline int is_prior(const int32_t* prop, int32_t a, int32_t b) {
  if (prop[a] != prop[b]) return prop[a] > prop[b];
  return a < b;
}

/* Per-thread stamp table used to build exact colour sets without clearing. */
typedef struct {
  uint32_t* stamp;
  int64_t size;
  uint32_t gen;
} scratch_t;

static int scratch_fit(scratch_t* s, int64_t size) {
  if (size <= s->size) return 0;
  uint32_t* p = (uint32_t*)calloc((size_t)size, sizeof(uint32_t));
  if (!p) return -1;
  free(s->stamp);
  s->stamp = p;
  s->size = size;
  s->gen = 0;
  return 0;
}

static inline uint32_t scratch_next(scratch_t* s) {
  if (++s->gen == 0) {
    memset(s->stamp, 0, (size_t)s->size * sizeof(uint32_t));
    s->gen = 1;
  }
  return s->gen;
}

/* Smallest colour not used by a live neighbour of v (HI computeSC +
 * FirstZeroBit, HI/gpuFunctions_undir.cuh:36-69, with exact masks).  When
 * prop != NULL only neighbours prior to v count (HB findMinAvailableColor,
 * HB/gpuFunctions_undir.cuh:118-129).  The mex of a set of at most L values
 * is at most L, so only colours <= len(v) need recording. */
static int32_t mex_of(const orc_graph* g, int32_t v, const int32_t* color,
                      const int32_t* prop, scratch_t* s, int64_t* scanned) {
  const int32_t* r = g->row[v];
  int32_t L = g->len[v];
  uint32_t gen = scratch_next(s);
  int64_t live = 0;
  for (int32_t i = 0; i < L; ++i) {
    int32_t u = r[i];
    if (u < 0) continue;
    ++live;
    if (prop && !is_prior(prop, u, v)) continue;
    int32_t c = color[u];
    if (c >= 0 && c <= L) s->stamp[c] = gen;
  }
  if (scanned) *scanned += live;
  int32_t c = 0;
  while (c <= L && s->stamp[c] == gen) ++c;
  return c;
}

/* Number of distinct colours among live neighbours of v: the saturation
 * size HI insEdge compares (BitCount over the full mask,
 * HI/gpuFunctions_undir.cuh:203-209). */
static int32_t distinct_of(const orc_graph* g, int32_t v, const int32_t* color,
                           scratch_t* s, int64_t* scanned) {
  const int32_t* r = g->row[v];
  int32_t L = g->len[v];
  uint32_t gen = scratch_next(s);
  int32_t cnt = 0;
  int64_t live = 0;
  for (int32_t i = 0; i < L; ++i) {
    int32_t u = r[i];
    if (u < 0) continue;
    ++live;
    int32_t c = color[u];
    if (s->stamp[c] != gen) {
      s->stamp[c] = gen;
      ++cnt;
    }
  }
  if (scanned) *scanned += live;
  return cnt;
}

static int32_t max_color(const orc_graph* g) {
  int32_t m = -1;
  for (int32_t v = 0; v < g->n; ++v)
    if (g->color[v] > m) m = g->color[v];
  return m;
}

static int32_t max_len(const orc_graph* g) {
  int32_t m = 0;
  for (int32_t v = 0; v < g->n; ++v)
    if (g->len[v] > m) m = g->len[v];
  return m;
}

static int g_threads = 0;
void orc_set_threads(int nthreads) { g_threads = nthreads; }
static int g_instrument = 0;
void orc_set_instrument(int on) { g_instrument = on; }

static int nthreads_now(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* graph / colour I/O                                                  */
/* ------------------------------------------------------------------ */

orc_graph* orc_create(int32_t n) {
  if (n < 0) return NULL;
  orc_graph* g = (orc_graph*)calloc(1, sizeof(orc_graph));
  if (!g) return NULL;
  g->n = n;
  size_t nn = n > 0 ? (size_t)n : 1;
  g->row = (int32_t**)calloc(nn, sizeof(int32_t*));
  g->len = (int32_t*)calloc(nn, sizeof(int32_t));
  g->cap = (int32_t*)calloc(nn, sizeof(int32_t));
  g->color = (int32_t*)calloc(nn, sizeof(int32_t));
  g->prev = (int32_t*)malloc(nn * sizeof(int32_t));
  g->prop = (int32_t*)calloc(nn, sizeof(int32_t));
  if (!g->row || !g->len || !g->cap || !g->color || !g->prev || !g->prop) {
    orc_destroy(g);
    return NULL;
  }
  /* cudaMemset(previosVertexcolor, -1, ...) HI/supportingFunctions.cu:89 */
  for (int32_t v = 0; v < n; ++v) g->prev[v] = -1;
  return g;
}

void orc_destroy(orc_graph* g) {
  if (!g) return;
  if (g->row)
    for (int32_t v = 0; v < g->n; ++v) free(g->row[v]);
  free(g->row);
  free(g->len);
  free(g->cap);
  free(g->color);
  free(g->prev);
  free(g->prop);
  free(g);
}

int32_t orc_num_vertices(const orc_graph* g) { return g->n; }

/* read_graphEdges, HI/all_structure_undir.cuh:156-183 and
 * HB/all_structure_undir.cuh:158-186: "a b w" adds a to row b and b to row
 * a, and (HB) bumps vertex_prop of both ends.  Self-loops and ids outside
 * [0,n) are rejected before anything is modified. */
int orc_load_edges(orc_graph* g, const int32_t* a, const int32_t* b, int64_t m) {
  if (m < 0) return ORC_E_INVAL;
  for (int64_t i = 0; i < m; ++i) {
    if (a[i] < 0 || a[i] >= g->n || b[i] < 0 || b[i] >= g->n || a[i] == b[i])
      return ORC_E_INVAL;
  }
  /* reserve exact room first so large loads do not realloc repeatedly */
  int64_t* add = (int64_t*)calloc(g->n > 0 ? (size_t)g->n : 1, sizeof(int64_t));
  if (!add) return ORC_E_NOMEM;
  for (int64_t i = 0; i < m; ++i) {
    add[a[i]]++;
    add[b[i]]++;
  }
  for (int32_t v = 0; v < g->n; ++v) {
    if (add[v] && row_reserve(g, v, g->len[v] + add[v])) {
      free(add);
      return ORC_E_NOMEM;
    }
  }
  free(add);
  for (int64_t i = 0; i < m; ++i) {
    row_push(g, b[i], a[i]);
    row_push(g, a[i], b[i]);
    g->prop[a[i]] += 1;
    g->prop[b[i]] += 1;
  }
  return ORC_OK;
}

/* read_Input_Color, HI/all_structure_undir.cuh:130-150 */
int orc_set_colors(orc_graph* g, const int32_t* colors) {
  for (int32_t v = 0; v < g->n; ++v)
    if (colors[v] < 0) return ORC_E_INVAL;
  memcpy(g->color, colors, (size_t)g->n * sizeof(int32_t));
  return ORC_OK;
}

int orc_get_colors(const orc_graph* g, int32_t* out) {
  memcpy(out, g->color, (size_t)g->n * sizeof(int32_t));
  return ORC_OK;
}

int orc_get_prop(const orc_graph* g, int32_t* out) {
  memcpy(out, g->prop, (size_t)g->n * sizeof(int32_t));
  return ORC_OK;
}

int32_t orc_live_degree(const orc_graph* g, int32_t v) {
  /* distinct live neighbours */
  int32_t L = g->len[v];
  int32_t cnt = 0;
  for (int32_t i = 0; i < L; ++i) {
    int32_t u = g->row[v][i];
    if (u < 0) continue;
    int dup = 0;
    for (int32_t j = 0; j < i; ++j)
      if (g->row[v][j] == u) {
        dup = 1;
        break;
      }
    cnt += !dup;
  }
  return cnt;
}

static int cmp_i32(const void* x, const void* y) {
  int32_t a = *(const int32_t*)x, b = *(const int32_t*)y;
  return (a > b) - (a < b);
}

int32_t orc_neighbors(const orc_graph* g, int32_t v, int32_t* out, int32_t cap) {
  int32_t L = g->len[v];
  int32_t* tmp = (int32_t*)malloc((size_t)(L > 0 ? L : 1) * sizeof(int32_t));
  int32_t c = 0;
  for (int32_t i = 0; i < L; ++i)
    if (g->row[v][i] >= 0) tmp[c++] = g->row[v][i];
  qsort(tmp, (size_t)c, sizeof(int32_t), cmp_i32);
  int32_t u = 0;
  for (int32_t i = 0; i < c; ++i)
    if (i == 0 || tmp[i] != tmp[i - 1]) {
      if (u < cap) out[u] = tmp[i];
      ++u;
    }
  free(tmp);
  return u;
}

/* validate, HI/gpuFunctions_undir.cuh:289-305 (counted once per u<v slot) */
int64_t orc_conflicts(const orc_graph* g) {
  int64_t bad = 0;
  for (int32_t v = 0; v < g->n; ++v)
    for (int32_t i = 0; i < g->len[v]; ++i) {
      int32_t u = g->row[v][i];
      if (u > v && g->color[u] == g->color[v]) ++bad;
    }
  return bad;
}

int orc_is_greedy_id_order(const orc_graph* g) {
  scratch_t s = {0};
  if (scratch_fit(&s, (int64_t)max_len(g) + 2)) return -1;
  int ok = 1;
  for (int32_t v = 0; v < g->n && ok; ++v) {
    uint32_t gen = scratch_next(&s);
    int32_t L = g->len[v];
    for (int32_t i = 0; i < L; ++i) {
      int32_t u = g->row[v][i];
      if (u >= 0 && u < v && g->color[u] <= L) s.stamp[g->color[u]] = gen;
    }
    int32_t c = 0;
    while (c <= L && s.stamp[c] == gen) ++c;
    ok = (c == g->color[v]);
  }
  free(s.stamp);
  return ok;
}

int orc_greedy_id_order(orc_graph* g) {
  scratch_t s = {0};
  if (scratch_fit(&s, (int64_t)max_len(g) + 2)) return ORC_E_NOMEM;
  for (int32_t v = 0; v < g->n; ++v) {
    uint32_t gen = scratch_next(&s);
    int32_t L = g->len[v];
    for (int32_t i = 0; i < L; ++i) {
      int32_t u = g->row[v][i];
      if (u >= 0 && u < v && g->color[u] <= L) s.stamp[g->color[u]] = gen;
    }
    int32_t c = 0;
    while (c <= L && s.stamp[c] == gen) ++c;
    g->color[v] = c;
  }
  free(s.stamp);
  return ORC_OK;
}

/* Greedy lowest-free colour with the vertices taken in the given order
 * (order[i] = the i-th vertex coloured); the colour of a vertex is the mex
 * over its neighbours coloured before it.  Checker for the device's
 * initial colouring in any order. */
int orc_greedy_in_order(orc_graph* g, const int32_t* order) {
  scratch_t s = {0};
  if (scratch_fit(&s, (int64_t)max_len(g) + 2)) return ORC_E_NOMEM;
  uint8_t* done = (uint8_t*)calloc(g->n > 0 ? (size_t)g->n : 1, 1);
  if (!done) {
    free(s.stamp);
    return ORC_E_NOMEM;
  }
  for (int32_t i = 0; i < g->n; ++i) {
    int32_t v = order[i];
    if (v < 0 || v >= g->n || done[v]) {
      free(done);
      free(s.stamp);
      return ORC_E_INVAL;
    }
    uint32_t gen = scratch_next(&s);
    int32_t L = g->len[v];
    for (int32_t j = 0; j < L; ++j) {
      int32_t u = g->row[v][j];
      if (u >= 0 && done[u] && g->color[u] <= L) s.stamp[g->color[u]] = gen;
    }
    int32_t c = 0;
    while (c <= L && s.stamp[c] == gen) ++c;
    g->color[v] = c;
    done[v] = 1;
  }
  free(done);
  free(s.stamp);
  return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* batch application                                                   */
/* ------------------------------------------------------------------ */

typedef struct {
  orc_graph* g;
  int variant;
  int nt;
  scratch_t* sc; /* one per thread */
  uint8_t* mark; /* affected_marked */
  int32_t* list; /* affectedNodeList */
  int64_t count; /* *counter */
  int32_t* tmp;  /* snapshot results, aligned with a target list */
  int64_t scanned;
} run_t;

/* compactor: flags -> ascending vertex ids (HI/compactor.cuh:79-173) */
static void compact(run_t* R) {
  int64_t c = 0;
  for (int32_t v = 0; v < R->g->n; ++v)
    if (R->mark[v]) R->list[c++] = v;
  R->count = c;
}

static inline int tid(void) {
#ifdef _OPENMP
  return omp_get_thread_num();
#else
  return 0;
#endif
}

/* findEligibleNeighbors.  It writes only flags, so its result does not
 * depend on the schedule.
 *   HI: HI/gpuFunctions_undir.cuh:229-260
 *   HB: HB/gpuFunctions_undir.cuh:259-291 */
static void find_eligible(run_t* R) {
  orc_graph* g = R->g;
  const int32_t* color = g->color;
  const int32_t* prev = g->prev;
  const int32_t* prop = g->prop;
  int64_t scanned = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : scanned) num_threads(R->nt)
  for (int64_t i = 0; i < R->count; ++i) {
    int32_t node = R->list[i];
    const int32_t* r = g->row[node];
    int32_t L = g->len[node];
    for (int32_t j = 0; j < L; ++j) {
      int32_t u = r[j];
      if (u < 0) continue;
      ++scanned;
      if (R->variant == ORC_HI) {
        if (color[node] == color[u] && node < u) __atomic_store_n(&R->mark[u], 1, __ATOMIC_RELAXED);
        if (prev[node] < color[u]) __atomic_store_n(&R->mark[u], 1, __ATOMIC_RELAXED);
      } else {
        if (color[node] == color[u]) {
          int32_t cand = is_prior(prop, node, u) ? u : node;
          __atomic_store_n(&R->mark[cand], 1, __ATOMIC_RELAXED);
        }
        if (is_prior(prop, node, u)) __atomic_store_n(&R->mark[u], 1, __ATOMIC_RELAXED);
      }
    }
  }
  R->scanned += scanned;
}

/* Computes, from the current state, the new colour of every target in
 * list[0..cnt) into R->tmp (snapshot step).  HB uses the prior-filtered
 * mex, HI the plain one. */
static void snapshot_mex(run_t* R, const int32_t* list, int64_t cnt) {
  orc_graph* g = R->g;
  const int32_t* prop = R->variant == ORC_HB ? g->prop : NULL;
  int64_t scanned = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : scanned) num_threads(R->nt)
  for (int64_t i = 0; i < cnt; ++i)
    R->tmp[i] = mex_of(g, list[i], g->color, prop, &R->sc[tid()], &scanned);
  R->scanned += scanned;
}

/* Adds v to a de-duplicated target list. */
static inline void add_target(int32_t v, uint8_t* seen, int32_t* out, int64_t* cnt) {
  if (!seen[v]) {
    seen[v] = 1;
    out[(*cnt)++] = v;
  }
}

static int64_t seed_hi_snapshot(run_t* R, const orc_change* ch, const int64_t* del,
                                int64_t ndel, const int64_t* ins, int64_t nins,
                                uint8_t* seen, int32_t* tgt, int* change) {
  orc_graph* g = R->g;
  int32_t* color = g->color;
  int64_t seeds = 0;
  /* deleteEdge (HI/gpuFunctions_undir.cuh:147-177): target = endpoint with
   * the larger colour, tie -> node2; recolour to the mex if it differs. */
  int64_t nt = 0;
  for (int64_t i = 0; i < ndel; ++i) {
    const orc_change* c = &ch[del[i]];
    int32_t t = color[c->node1] > color[c->node2] ? c->node1 : c->node2;
    add_target(t, seen, tgt, &nt);
  }
  snapshot_mex(R, tgt, nt);
  for (int64_t i = 0; i < nt; ++i) {
    int32_t t = tgt[i];
    seen[t] = 0;
    if (R->tmp[i] != color[t]) {
      g->prev[t] = color[t];
      color[t] = R->tmp[i];
      R->mark[t] = 1;
      *change = 1;
    }
  }
  seeds += nt;
  /* insEdge (HI/gpuFunctions_undir.cuh:182-223): if the colours are still
   * equal, the endpoint with the smaller saturation size (tie -> node2) is
   * recoloured unconditionally. */
  int64_t ne = 0;
  int32_t* ends = (int32_t*)malloc((size_t)(2 * nins + 1) * sizeof(int32_t));
  int32_t* sat = (int32_t*)malloc((size_t)(2 * nins + 1) * sizeof(int32_t));
  int32_t* where = (int32_t*)malloc((size_t)(g->n > 0 ? g->n : 1) * sizeof(int32_t));
  for (int64_t i = 0; i < nins; ++i) {
    const orc_change* c = &ch[ins[i]];
    if (color[c->node1] != color[c->node2]) continue;
    add_target(c->node1, seen, ends, &ne);
    add_target(c->node2, seen, ends, &ne);
  }
  int64_t scanned = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : scanned) num_threads(R->nt)
  for (int64_t i = 0; i < ne; ++i) sat[i] = distinct_of(g, ends[i], color, &R->sc[tid()], &scanned);
  R->scanned += scanned;
  for (int64_t i = 0; i < ne; ++i) {
    where[ends[i]] = (int32_t)i;
    seen[ends[i]] = 0;
  }
  nt = 0;
  for (int64_t i = 0; i < nins; ++i) {
    const orc_change* c = &ch[ins[i]];
    if (color[c->node1] != color[c->node2]) continue;
    int32_t s1 = sat[where[c->node1]], s2 = sat[where[c->node2]];
    int32_t t = s1 < s2 ? c->node1 : c->node2;
    add_target(t, seen, tgt, &nt);
  }
  snapshot_mex(R, tgt, nt);
  for (int64_t i = 0; i < nt; ++i) {
    int32_t t = tgt[i];
    seen[t] = 0;
    g->prev[t] = color[t];
    color[t] = R->tmp[i];
    R->mark[t] = 1;
    *change = 1;
  }
  seeds += nt;
  free(ends);
  free(sat);
  free(where);
  return seeds;
}

static int64_t seed_hi_serial(run_t* R, const orc_change* ch, const int64_t* del,
                              int64_t ndel, const int64_t* ins, int64_t nins, int* change) {
  orc_graph* g = R->g;
  int32_t* color = g->color;
  scratch_t* s = &R->sc[0];
  for (int64_t i = 0; i < ndel; ++i) {
    const orc_change* c = &ch[del[i]];
    int32_t t = color[c->node1] > color[c->node2] ? c->node1 : c->node2;
    int32_t m = mex_of(g, t, color, NULL, s, &R->scanned);
    if (m != color[t]) {
      g->prev[t] = color[t];
      color[t] = m;
      R->mark[t] = 1;
      *change = 1;
    }
  }
  for (int64_t i = 0; i < nins; ++i) {
    const orc_change* c = &ch[ins[i]];
    if (color[c->node1] != color[c->node2]) continue;
    int32_t s1 = distinct_of(g, c->node1, color, s, &R->scanned);
    int32_t s2 = distinct_of(g, c->node2, color, s, &R->scanned);
    int32_t t = s1 < s2 ? c->node1 : c->node2;
    int32_t m = mex_of(g, t, color, NULL, s, &R->scanned);
    g->prev[t] = color[t];
    color[t] = m;
    R->mark[t] = 1;
    *change = 1;
  }
  return ndel + nins;
}

/* processChangeEdge, HB/gpuFunctions_undir.cuh:222-249.  Snapshot form:
 * every endpoint of every listed change is one de-duplicated target of a
 * single step. */
static int64_t seed_hb_snapshot(run_t* R, const orc_change* ch, const int64_t* lst,
                                int64_t nl, uint8_t* seen, int32_t* tgt, int* change) {
  orc_graph* g = R->g;
  int64_t nt = 0;
  for (int64_t i = 0; i < nl; ++i) {
    add_target(ch[lst[i]].node1, seen, tgt, &nt);
    add_target(ch[lst[i]].node2, seen, tgt, &nt);
  }
  snapshot_mex(R, tgt, nt);
  for (int64_t i = 0; i < nt; ++i) {
    int32_t t = tgt[i];
    seen[t] = 0;
    if (R->tmp[i] != g->color[t]) {
      g->color[t] = R->tmp[i];
      R->mark[t] = 1;
      *change = 1;
    }
  }
  return nt;
}

static int64_t seed_hb_serial(run_t* R, const orc_change* ch, const int64_t* lst,
                              int64_t nl, int* change) {
  orc_graph* g = R->g;
  scratch_t* s = &R->sc[0];
  for (int64_t i = 0; i < nl; ++i) {
    int32_t ends[2] = {ch[lst[i]].node1, ch[lst[i]].node2};
    for (int e = 0; e < 2; ++e) {
      int32_t node = ends[e];
      int32_t m = mex_of(g, node, g->color, g->prop, s, &R->scanned);
      if (m != g->color[node]) {
        g->color[node] = m;
        R->mark[node] = 1;
        *change = 1;
      }
    }
  }
  return 2 * nl;
}

int orc_apply_batch(orc_graph* g, int variant, int schedule, const orc_change* ch,
                    int64_t k, int64_t iter_cap, orc_stats* st) {
  if (variant != ORC_HI && variant != ORC_HB) return ORC_E_INVAL;
  if (schedule != ORC_SNAPSHOT && schedule != ORC_SERIAL) return ORC_E_INVAL;
  if (k < 0) return ORC_E_INVAL;
  for (int64_t i = 0; i < k; ++i) {
    if (ch[i].inst != 0 && ch[i].inst != 1) continue;
    if (ch[i].node1 < 0 || ch[i].node1 >= g->n || ch[i].node2 < 0 ||
        ch[i].node2 >= g->n || ch[i].node1 == ch[i].node2)
      return ORC_E_INVAL;
  }
  orc_stats S;
  memset(&S, 0, sizeof(S));
  int32_t n = g->n;
  size_t nn = n > 0 ? (size_t)n : 1;
  int32_t* start = (int32_t*)malloc(nn * sizeof(int32_t));
  int64_t* del = (int64_t*)malloc((size_t)(k + 1) * sizeof(int64_t));
  int64_t* ins = (int64_t*)malloc((size_t)(k + 1) * sizeof(int64_t));
  int64_t* lst = (int64_t*)malloc((size_t)(k + 1) * sizeof(int64_t));
  if (!start || !del || !ins || !lst) {
    free(start);
    free(del);
    free(ins);
    free(lst);
    return ORC_E_NOMEM;
  }
  memcpy(start, g->color, nn * sizeof(int32_t) * (n > 0));
  int64_t ndel = 0, nins = 0, nl = 0;

  /* readin_changes: HI/all_structure_undir.cuh:78-128,
   * HB/all_structure_undir.cuh:78-129.  Insertions go into the adjacency
   * straight away (so a delete of the same edge in the batch wins), and are
   * kept as seeds only when their colours are equal at read time.  HB keeps
   * every deletion as a seed too and moves the degree property by one per
   * line. */
  for (int64_t i = 0; i < k; ++i) {
    int32_t a = ch[i].node1, b = ch[i].node2;
    if (ch[i].inst == 1) {
      if (row_push(g, b, a) || row_push(g, a, b)) {
        free(start); free(del); free(ins); free(lst);
        return ORC_E_NOMEM;
      }
      if (g->color[a] == g->color[b]) {
        ins[nins++] = i;
        lst[nl++] = i;
      }
      g->prop[a] += 1;
      g->prop[b] += 1;
    } else if (ch[i].inst == 0) {
      del[ndel++] = i;
      lst[nl++] = i;
      g->prop[a] -= 1;
      g->prop[b] -= 1;
    }
  }
  /* deleteEdgeFromAdj: tombstone every copy in both rows. */
  for (int64_t i = 0; i < ndel; ++i) {
    int32_t a = ch[del[i]].node1, b = ch[del[i]].node2;
    for (int32_t j = 0; j < g->len[b]; ++j)
      if (g->row[b][j] == a) g->row[b][j] = -1 - a;
    for (int32_t j = 0; j < g->len[a]; ++j)
      if (g->row[a][j] == b) g->row[a][j] = -1 - b;
  }

  run_t R;
  memset(&R, 0, sizeof(R));
  R.g = g;
  R.variant = variant;
  R.nt = schedule == ORC_SERIAL ? 1 : nthreads_now();
  R.sc = (scratch_t*)calloc((size_t)R.nt, sizeof(scratch_t));
  R.mark = (uint8_t*)calloc(nn, 1);
  R.list = (int32_t*)malloc(nn * sizeof(int32_t));
  R.tmp = (int32_t*)malloc(nn * sizeof(int32_t));
  uint8_t* seen = (uint8_t*)calloc(nn, 1);
  int32_t* tgt = (int32_t*)malloc(nn * sizeof(int32_t));
  int rc = ORC_OK;
  int64_t need = (int64_t)max_len(g) + 2;
  int32_t mc = max_color(g);
  if (mc + 2 > need) need = (int64_t)mc + 2;
  if (!R.sc || !R.mark || !R.list || !R.tmp || !seen || !tgt) rc = ORC_E_NOMEM;
  for (int t = 0; t < R.nt && rc == ORC_OK; ++t)
    if (scratch_fit(&R.sc[t], need)) rc = ORC_E_NOMEM;

  if (rc == ORC_OK) {
    int change = 0;
    if (variant == ORC_HI) {
      S.seed_targets = schedule == ORC_SNAPSHOT
                           ? seed_hi_snapshot(&R, ch, del, ndel, ins, nins, seen, tgt, &change)
                           : seed_hi_serial(&R, ch, del, ndel, ins, nins, &change);
    } else {
      S.seed_targets = schedule == ORC_SNAPSHOT
                           ? seed_hb_snapshot(&R, ch, lst, nl, seen, tgt, &change)
                           : seed_hb_serial(&R, ch, lst, nl, &change);
    }
    /* The colour bound may have grown during seeding. */
    compact(&R);
    /* HI/Color_main.cu:176-202, HB/Color_main.cu:198-224 */
    while (change > 0) {
      if (S.iterations >= iter_cap) {
        S.status = ORC_E_ITER_LIMIT;
        break;
      }
      S.iterations++;
      change = 0;
      memset(R.mark, 0, nn);
      find_eligible(&R);
      compact(&R);
      memset(R.mark, 0, nn);
      S.frontier_total += R.count;
      if (g_instrument) {
        /* edges with both ends in this frontier (R.list), via a membership array */
        uint8_t* inq = (uint8_t*)calloc(nn, 1);
        for (int64_t i = 0; i < R.count; ++i) inq[R.list[i]] = 1;
        for (int64_t i = 0; i < R.count; ++i) {
          int32_t t = R.list[i];
          for (int32_t j = 0; j < g->len[t]; ++j) {
            int32_t u = g->row[t][j];
            if (u >= 0 && inq[u]) S.internal_pairs++;
          }
        }
        free(inq);
      }
      /* recolorNeighbor: HI/gpuFunctions_undir.cuh:264-284 (always sets
       * change), HB/gpuFunctions_undir.cuh:295-314 (only on a change). */
      if (schedule == ORC_SNAPSHOT) {
        snapshot_mex(&R, R.list, R.count);
        for (int64_t i = 0; i < R.count; ++i) {
          int32_t t = R.list[i];
          if (variant == ORC_HI) {
            g->prev[t] = g->color[t];
            g->color[t] = R.tmp[i];
            change = 1;
          } else if (R.tmp[i] != g->color[t]) {
            g->color[t] = R.tmp[i];
            change = 1;
          }
        }
      } else {
        const int32_t* prop = variant == ORC_HB ? g->prop : NULL;
        for (int64_t i = 0; i < R.count; ++i) {
          int32_t t = R.list[i];
          int32_t m = mex_of(g, t, g->color, prop, &R.sc[0], &R.scanned);
          if (variant == ORC_HI) {
            g->prev[t] = g->color[t];
            g->color[t] = m;
            change = 1;
          } else if (m != g->color[t]) {
            g->color[t] = m;
            change = 1;
          }
        }
      }
    }
    S.slots_scanned = R.scanned;
    int64_t changed = 0;
    for (int32_t v = 0; v < n; ++v) changed += (g->color[v] != start[v]);
    S.changed_vertices = changed;
    S.max_color = max_color(g);
  }
  for (int t = 0; R.sc && t < R.nt; ++t) free(R.sc[t].stamp);
  free(R.sc);
  free(R.mark);
  free(R.list);
  free(R.tmp);
  free(seen);
  free(tgt);
  free(start);
  free(del);
  free(ins);
  free(lst);
  if (st) *st = S;
  if (rc != ORC_OK) return rc;
  return S.status;
}
