// dc_internal.h -- host/device shared layouts of libdyncolor (not part of the
// public C ABI).  Plain structs of pointers and sizes; no torch types.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/dyncolor.h"

namespace dc {

// Device status bits (DevState::status).
enum : unsigned {
  ST_INVAL = 1u << 0,     // a change line is invalid (id out of range / self-loop)
  ST_POOL = 1u << 1,      // adjacency pool exhausted: host grows it and retries
  ST_ITER = 1u << 2,      // iteration cap reached
  ST_TIMEOUT = 1u << 3,   // a grid barrier gave up waiting
  ST_OVERFLOW = 1u << 4,  // an internal capacity guard fired
};

constexpr int kThreads = 512;       // threads per CTA of the persistent kernels
constexpr int kWarps = kThreads / 32;
constexpr int kSmall = 32;          // rows up to this many slots are "class A" (warp-batched)
constexpr int kMaskWords = 128;     // colour window per warp: 4096 colours
constexpr int kMaskBits = kMaskWords * 32;
constexpr int kStructChunk = 1024;  // slots per unit in the structural row scans
constexpr int kTomb = -1;           // tombstoned adjacency slot
// During the recolour loop, bit 30 of color[v] marks v for the next
// frontier; colours are below 2^30.  The commit's store clears it.
constexpr unsigned kMarkBit = 1u << 30;
constexpr int kColorMask = (1 << 30) - 1;
constexpr int kNumQueues = 6;       // logical queue counter slots
constexpr int kUnitSlotsDefault = 4096;  // adjacency slots per warp work unit
constexpr long long kLoadPiece = 1ll << 27;  // edge pairs per structural launch of a graph load
constexpr int kBarrierTimeoutMsDefault = 20000;  // grid-barrier wait limit unless the options set one

// Logical queue counter slots.
enum { Q_LOOP0 = 0, Q_LOOP1 = 1, Q_LOOP2 = 2, Q_S1 = 3, Q_S2E = 4, Q_S2T = 5 };

struct QCount {
  unsigned long long countA;  // class A items
  unsigned long long countU;  // work units (class B/C)
  unsigned long long masks;   // multi-unit mask words handed out
  unsigned long long pad;
};

// Lives in device memory.  Fields up to `pool_used_start` persist across
// batches; everything from `bar_arrived` on is cleared before every batch,
// and bar_arrived .. wctr again before every launch.
struct DevState {
  int cmax;                        // upper bound of every colour value
  int pad0;
  unsigned long long pool_used;    // adjacency pool slots handed out
  long long batch_k;               // line count, read by kernels of a captured batch graph
  unsigned long long pool_used_start;
  // ---- cleared before every kernel launch (bar_arrived .. wctr) ----
  unsigned bar_arrived;
  unsigned bar_abort;
  int chg[2];                      // HB loop: "a colour changed" flags, ring by iteration
  unsigned long long wctr[3];      // work-grab counters (ring by phase)
  // ---- cleared before every batch (bar_arrived .. end) ----
  unsigned status;
  unsigned pre_status;             // status of the structural launch, copied before the recolour launch
  // structural kernel
  unsigned long long nvalid;       // valid change lines
  unsigned long long nnet;         // netted (row, nbr) entries
  unsigned long long ntouched;     // touched rows
  unsigned long long ndel;         // slots to tombstone
  unsigned long long nunits;       // row-scan units
  unsigned long long nrel;         // relocation copy units
  // recolour kernel
  QCount q[kNumQueues];
  // statistics
  unsigned long long iterations;
  unsigned long long seed_targets;
  unsigned long long frontier_total;
  unsigned long long slots_scanned;
  unsigned long long edges_inserted;  // directed entries (2 per undirected edge)
  unsigned long long edges_deleted;
  unsigned long long rows_relocated;
  unsigned long long slots_read;      // adjacency entries the kernels actually read
  unsigned long long t_struct[2];     // %globaltimer at the start and end of the structural launch
  unsigned long long t_recolor[2];    // same for the recolour launch
  unsigned long long phase_ns[6];     // recolour launch: seeding, find-eligible, mex, commit, 2 spare
  // heavy-row index
  unsigned long long hcount;          // rows found with at least min_live live slots
  unsigned long long a_count;         // (vertex, chunk) items waiting for the append phase
  unsigned hri_off;                   // 1: the index is incomplete for this batch; full scans only
  unsigned pad1;
  long long read_delta;               // adjacency/index entries read minus entries scanned
};

struct GraphDev {
  int n;
  int key_bits;          // B with n-1 < 2^B
  long long* off;        // row start in adj, multiple of 4
  int* len;              // slots in use (live + tombstones)
  int* cap;              // slots reserved, multiple of 4
  int* live;             // live slots
  int* adj;              // adjacency pool
  long long pool_cap;
  int* color;
  int* prev;             // HI previosVertexcolor
  int* prop;             // HB vertex_prop
};

struct QueueBufs {
  int* itemsA;           // class A items
  int4* units;           // {vertex, chunk, mask word offset, chunks}
  unsigned* gmask;       // per multi-unit row: [done counter, mask words...], 4-word aligned
  long long capA, capU, capM;  // capM in 32-bit words
};

struct StructParams {
  GraphDev g;
  const dc_change* ch;   // change lines (update batch) or NULL
  const int* la;         // graph-load pairs when ch == NULL
  const int* lb;
  long long k;           // number of lines
  const long long* k_dev;  // when set, the line count is read from here (captured graphs)
  float slack;
  unsigned long long* keysA;  // 2k
  unsigned long long* keysB;  // 2k
  unsigned* hist;        // grid * 256
  unsigned* dscan;       // grid * 256 (digit prefix over CTAs) + 256 totals
  unsigned* cta_cnt;     // grid
  unsigned long long* net;    // 2k netted keys
  int* tof;              // 2k: touched-row index of each net entry
  unsigned char* present;// 2k
  int* rank;             // 2k
  int* tbeg;             // touched rows + 1: first net entry
  int* trow;             // touched row id
  int* rowdel;           // per touched row: slots deleted
  int* tins;             // per touched row: new neighbours
  long long* tnoff;      // per touched row: new offset
  int* tncap;
  int* tnlive;
  int* trel;
  int* cursor;
  long long* delpos;     // absolute slot positions to tombstone
  int2* units;           // row-scan units {touched row, chunk}
  int2* relunits;        // relocation copy units
  long long cap_units;
  long long cap_rel;
  const int* gid;        // batched mode: vertex -> graph; lines must stay inside a graph
  unsigned long long bar_timeout_ns;  // limit of every grid-barrier wait
  DevState* st;
};

// Heavy-row index.  Per batch, every row with at least `min_live` live
// slots gets a copy of its neighbours.  HI: ordered by their colour at the
// start of the recolour launch (descending), and a list of its neighbours
// whose colour has changed since.  HB: its neighbours prior to it first.
// HI's findEligibleNeighbors marks a neighbour u of v only if
// color[u] > prev[v] or color[u] == color[v], so for such a row it reads
// the head of the ordered copy, the segment of colour color[v], and the
// list, instead of gathering every neighbour's colour.
constexpr int kHeavyMinLive = 2048;   // HI
constexpr int kHeavyMinLiveHB = 256;  // HB: its index only splits rows by priority, cheap to build
// A batch uses the index when lines * kIndexBatchRatio >= n.
constexpr long long kIndexBatchRatio = 256;
constexpr int kHriBins = 1024;  // exact colour order below 1023; colours >= 1023 share the first bin
struct HriBufs {
  int* hid;                   // n: index of v's ordered copy, or -1
  int* hrow;                  // cap_rows: vertex of index i
  long long* hoff;            // cap_rows + 1: start of row i in pairs
  unsigned long long* pairs;  // HI, cap_pairs: (colour << 32) | neighbour
  int* ids;                   // HB, cap_pairs: neighbour ids (see hsplit)
  long long* xoff;           // cap_rows + 1: start of row i's change list
  int* xcnt;                  // cap_rows: entries appended to row i's change list (> capacity: overflow)
  int* xv;                    // cap_exc: changed neighbours
  unsigned* bmF;              // n/32 + 1: colour changed since the index was built
  int2* alist;                // cap_a: (vertex, chunk) of first changes, for the append phase
  int* hist;                  // cap_hist * kHriBins: row i's count of neighbours per launch-start colour
                              // that have not changed colour since (the append phase takes them off)
  int* hsplit;                // HB, cap_rows: row i's copy (in ids) holds its prior neighbours first,
                              // hsplit[i] of them, then the rest
  unsigned long long* bcnt;   // 64: rows per length class, then the classes' cursors (build scratch)
  long long cap_rows, cap_pairs, cap_exc, cap_a, cap_hist;
  int min_live;               // 0: no index
  // Vertex ranges the index covers (nullptr: every vertex): [count, total,
  // then per range its first vertex and the vertices before it in the
  // ranges' concatenation].  A resident pool's launch touches only its own
  // graphs, so their rows alone are indexed; hid of other vertices is never
  // read during that launch.
  const int* ranges;
};

struct RecolorParams {
  GraphDev g;
  const dc_change* ch;
  long long k;
  const long long* k_dev;  // when set, the line count is read from here (captured graphs)
  int variant;
  int unit_slots;        // slots per work unit (multiple of 128)
  long long iter_cap;
  QueueBufs qb[3];
  unsigned* bmA;
  unsigned* bmB;
  unsigned* bmC;
  int* ncolor;           // n
  int* sat;              // n
  unsigned long long* cp;  // HB: n packed (degree property, colour) words
  HriBufs hri;             // HI: heavy-row index (hri.min_live == 0: off)
  unsigned char* lflag;  // k
  int* pred;             // initial colouring: neighbours still to be coloured before each vertex
  const int* ranges;     // vertex ranges of the launch's graphs (HriBufs::ranges layout), nullptr: all
  // Batched mode: the graph is a disjoint union of independent graphs.
  const int* gid;        // vertex -> graph (nullptr: one graph)
  int ngraphs;
  int* gcnt;             // 2 * ngraphs: per-iteration activity of each graph (ring by parity)
  int* gf0;              // ngraphs: vertices each graph put in frontier F0
  int* giters;           // ngraphs: loop iterations of each graph
  int* gstate;           // ngraphs: 0 not started, 1 running, 2 done
  unsigned long long bar_timeout_ns;  // limit of every grid-barrier wait
  DevState* st;
};

// Launchers (dc_struct.cu / dc_recolor.cu / dc_misc.cu).  They return the
// CUDA error of the launch.
cudaError_t launch_struct(const StructParams& p, int grid, cudaStream_t s);
cudaError_t launch_recolor(const RecolorParams& p, int grid, cudaStream_t s);
// Initial colouring (greedy lowest free colour in a priority order) as a
// Jones-Plassmann launch: p.g.prop holds each vertex's priority value (ties
// and the id order: lower id first), p.cp and p.pred are n-sized scratch, the
// colours land in p.g.color.
cudaError_t launch_init_color(const RecolorParams& p, int grid, cudaStream_t s);
int struct_kernel_occupancy();
int recolor_kernel_occupancy();
cudaError_t launch_validate(const GraphDev& g, unsigned long long* out, cudaStream_t s);
cudaError_t launch_color_max(const GraphDev& g, DevState* st, cudaStream_t s);
cudaError_t launch_count_live(const GraphDev& g, unsigned long long* out, cudaStream_t s);
// Clears loop marks left in the colour array by an aborted launch.
cudaError_t launch_color_unmark(const GraphDev& g, cudaStream_t s);
// Batched mode: gid[v] from graph start offsets; counts edges crossing graphs.
cudaError_t launch_partition(const GraphDev& g, const int* first, int ngraphs, int* gid,
                             unsigned long long* cross, cudaStream_t s);
// Repacking rows of g into new arrays with the given slack, in two parts:
// the packed total (scratch: ceil(n / 256) + 1 long longs), then the copy
// into off2/cap2/len2/adj2 (g itself is only read).
cudaError_t launch_packed_total(const GraphDev& g, float slack, long long* scratch, unsigned long long* total,
                                cudaStream_t s);
cudaError_t launch_repack_copy(const GraphDev& g, float slack, const long long* scratch, long long* off2, int* cap2,
                               int* len2, int* adj2, long long cap_slots, unsigned* status, cudaStream_t s);
// Resident pool: copy the rows of vertices [v0, v0 + nv) out to / in from a
// packed buffer (row i at pre[i]), with vertex ids shifted by -base / +base.
cudaError_t launch_range_gather(const GraphDev& g, int base, int v0, int nv, const long long* pre, int* out,
                                cudaStream_t s);
cudaError_t launch_range_scatter(const GraphDev& g, int base, int v0, int nv, const long long* pre, const int* in,
                                 cudaStream_t s);
cudaError_t launch_fill(int* p, long long count, int value, cudaStream_t s);
// Builds the heavy-row index of the current graph and colours (dc_hri.cu):
// HI orders rows by colour, HB splits them by LDF priority.
cudaError_t launch_hri_build(const GraphDev& g, const HriBufs& h, DevState* st, int variant, cudaStream_t s);

}  // namespace dc
