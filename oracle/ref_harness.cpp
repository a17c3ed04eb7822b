/*
 * ref_harness.cpp -- runs the reference's OWN kernel bodies and text readers
 * on the CPU (test infrastructure only; built into oracle/_ref/, never part
 * of the product).
 *
 * Compiled once per variant with -DREF_HI or -DREF_HB and -I pointing at the
 * reference's source directory, so that
 *   all_structure_undir.cuh   (read_graphEdges / read_Input_Color / readin_changes)
 *   gpuFunctions_undir.cuh    (deleteEdgeFromAdj, deleteEdge, insEdge,
 *                              processChangeEdge, findEligibleNeighbors,
 *                              recolorNeighbor)
 * are used unmodified.  The shim in ref_shim/ makes the launch geometry one
 * thread.  This file re-states only the driver (HI/Color_main.cu:31-247,
 * HB/Color_main.cu:32-256, HI/supportingFunctions.cu:19-101) with a host
 * compaction in place of cuCompactor (ascending ids, HI/compactor.cuh:79-173),
 * and always allocates the frontier buffers (the reference allocates them
 * only when the batch has deletions, HI/supportingFunctions.cu:69-95).
 *
 * Two schedules:
 *   serial   -- each kernel called once over all its items (index order).
 *   snapshot -- each kernel item is run alone against a copy of the state at
 *               the start of the step; the writes of all items are merged
 *               afterwards (a write conflict aborts).  HB's
 *               processChangeEdge becomes HB's recolorNeighbor body applied
 *               to the de-duplicated endpoints of the change list.
 *
 * usage: ref_{hi,hb} serial|snapshot graph nodes edges prevColor changes out [iter_cap]
 * out: "iterations <n> status <0|4>\n" then one colour per line.
 *
 * Timing mode (for the reference arm of the benchmark):
 *   ref_{hi,hb} bench graph.bin nodes edges colors.bin ch1[,ch2,...] out
 *               [iter_cap [budget_ms [max_fail [threads]]]]
 *   Every kernel is launched on `threads` host threads (default: all of
 *   OpenMP's): each thread runs the kernel's grid-stride loop over its share
 *   of the items, racing on the shared arrays as the reference's GPU threads
 *   do.  A step stops at iter_cap loop iterations or once its timed work
 *   passes budget_ms, with status 4, so a timing run ends in bounded time;
 *   after max_fail such steps in a row (default: never) the rest are skipped.
 * graph.bin holds int32 pairs (a0 b0 a1 b1 ...) turned into the adjacency the
 * way read_graphEdges does; colors.bin holds one int32 per vertex.  Every
 * change file is one step applied to the initial graph and colouring (the
 * state is restored between steps, untimed).  The timed region of a step is
 * readin_changes + deleteEdgeFromAdj + seeding + loop (the CSR flatten
 * between them is not timed); out gets one line per step:
 * "iterations <n> status <s> time_ms <t>".
 */
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "gpuFunctions_undir.cuh"

namespace {

struct State {
  int n = 0;
  std::vector<int> color, prev, affected;
  int change = 0;
};

// Runs one snapshot step: run_item(j) is called for every item against the
// state as it was when the step began; all writes are merged at the end.
template <class F>
bool snapshot_step(State& S, int nitems, F run_item) {
  const std::vector<int> c0 = S.color, p0 = S.prev, a0 = S.affected;
  const int ch0 = S.change;
  std::vector<int> nc = c0, np = p0, na = a0;
  std::vector<char> wc(S.n, 0), wp(S.n, 0), wa(S.n, 0);
  int nch = ch0;
  for (int j = 0; j < nitems; ++j) {
    S.color = c0;
    S.prev = p0;
    S.affected = a0;
    S.change = ch0;
    run_item(j);
    for (int v = 0; v < S.n; ++v) {
      if (S.color[v] != c0[v]) {
        if (wc[v] && nc[v] != S.color[v]) return false;
        wc[v] = 1;
        nc[v] = S.color[v];
      }
      if (S.prev[v] != p0[v]) {
        if (wp[v] && np[v] != S.prev[v]) return false;
        wp[v] = 1;
        np[v] = S.prev[v];
      }
      if (S.affected[v] != a0[v]) {
        if (wa[v] && na[v] != S.affected[v]) return false;
        wa[v] = 1;
        na[v] = S.affected[v];
      }
    }
    if (S.change != ch0) nch = S.change;
  }
  S.color = nc;
  S.prev = np;
  S.affected = na;
  S.change = nch;
  return true;
}

// Runs kernel body f as a launch of `threads` host threads (see the shim).
template <class F>
void launch(int threads, F f) {
  if (threads <= 1) {
    f();
    return;
  }
  blockDim.x = (unsigned)threads;
#pragma omp parallel num_threads(threads)
  {
    threadIdx.x = (unsigned)omp_get_thread_num();
    f();
    threadIdx.x = 0;
  }
  blockDim.x = 1;
}

int compact(const State& S, std::vector<int>& list) {
  int c = 0;
  for (int v = 0; v < S.n; ++v)
    if (S.affected[v] == 1) list[c++] = v;
  return c;
}

}  // namespace

namespace {

struct Graph {
  int nodes = 0;
  std::vector<ColList> adj;
#ifndef REF_HI
  std::vector<int> prop;
#endif
};

struct StepResult {
  long iterations = 0;
  int status = 0;
  double ms = 0;
  bool ok = true;
};

// One update batch as the reference driver applies it
// (HI/Color_main.cu:62-202, HB/Color_main.cu:71-224).
StepResult run_step(Graph& G, State& S, const char* changes, bool snapshot, long iter_cap,
                    double budget_ms = 0.0, int threads = 1) {
  using clk = std::chrono::steady_clock;
  StepResult R;
  const int nodes = G.nodes;
  int totalInsertion = 0;
#ifdef REF_HI
  int maxColor = -1;
  for (int v = 0; v < nodes; ++v) maxColor = std::max(maxColor, S.color[v]);
  const int W = maxColor / 32 + 2;  // HI/Color_main.cu:69
  std::vector<changeEdge> allChange_Ins, allChange_Del;
  clk::time_point t0 = clk::now();
  readin_changes(const_cast<char*>(changes), allChange_Ins, allChange_Del, G.adj, totalInsertion,
                 S.color.data());
#else
  std::vector<changeEdge> allChange, allChange_Del;
  clk::time_point t0 = clk::now();
  readin_changes(const_cast<char*>(changes), allChange, allChange_Del, G.adj, totalInsertion,
                 S.color.data(), G.prop.data());
#endif
  R.ms += std::chrono::duration<double, std::milli>(clk::now() - t0).count();
  // CSR flatten, HI/supportingFunctions.cu:27-33 (not timed)
  std::vector<int> tracker(nodes + 1, 0);
  std::vector<ColWt> full;
  size_t total = 0;
  for (int i = 0; i < nodes; ++i) total += G.adj[i].size();
  full.reserve(total + 1);
  for (int i = 0; i < nodes; ++i) {
    tracker[i + 1] = tracker[i] + (int)G.adj[i].size();
    full.insert(full.end(), G.adj[i].begin(), G.adj[i].end());
  }
  full.push_back(ColWt{0, -1});  // keeps data() valid for an empty graph
  t0 = clk::now();
  ColWt* adj = full.data();
  int* trk = tracker.data();
  std::vector<int> list(nodes > 0 ? nodes : 1, 0);
  int counter = 0;
  int one = 1;
  bool ok = true;

  if (!allChange_Del.empty())
    launch(threads, [&] { deleteEdgeFromAdj(allChange_Del.data(), (int)allChange_Del.size(), adj, trk); });

#ifdef REF_HI
  if (!allChange_Del.empty()) {
    if (snapshot) {
      ok = ok && snapshot_step(S, (int)allChange_Del.size(), [&](int j) {
        deleteEdge(&allChange_Del[j], S.color.data(), S.prev.data(), 1, adj, trk,
                   S.affected.data(), &S.change, W);
      });
    } else {
      launch(threads, [&] {
        deleteEdge(allChange_Del.data(), S.color.data(), S.prev.data(), (int)allChange_Del.size(), adj, trk,
                   S.affected.data(), &S.change, W);
      });
    }
  }
  if (!allChange_Ins.empty()) {
    if (snapshot) {
      ok = ok && snapshot_step(S, (int)allChange_Ins.size(), [&](int j) {
        insEdge(&allChange_Ins[j], S.color.data(), S.prev.data(), 1, adj, trk,
                S.affected.data(), &S.change, W);
      });
    } else {
      launch(threads, [&] {
        insEdge(allChange_Ins.data(), S.color.data(), S.prev.data(), (int)allChange_Ins.size(), adj, trk,
                S.affected.data(), &S.change, W);
      });
    }
  }
#else
  int* prop = G.prop.data();
  if (snapshot) {
    std::vector<int> ends;
    std::vector<char> seen(nodes, 0);
    for (const changeEdge& c : allChange) {
      int e[2] = {c.node1, c.node2};
      for (int x : e)
        if (!seen[x]) {
          seen[x] = 1;
          ends.push_back(x);
        }
    }
    ok = ok && snapshot_step(S, (int)ends.size(), [&](int j) {
      recolorNeighbor(&ends[j], S.color.data(), adj, trk, S.affected.data(), &one, &S.change,
                      prop);
    });
  } else if (!allChange.empty()) {
    launch(threads, [&] {
      processChangeEdge(allChange.data(), S.color.data(), (int)allChange.size(), adj, trk, S.affected.data(),
                        &S.change, prop);
    });
  }
#endif

  long it = 0;
  counter = compact(S, list);
  while (ok && S.change > 0) {
    // the iteration cap, or (timing mode) the time budget of the step
    if (it >= iter_cap ||
        (budget_ms > 0 && std::chrono::duration<double, std::milli>(clk::now() - t0).count() + R.ms > budget_ms)) {
      R.status = 4;
      break;
    }
    ++it;
    S.change = 0;
    std::fill(S.affected.begin(), S.affected.end(), 0);
    launch(threads, [&] {
#ifdef REF_HI
      findEligibleNeighbors(list.data(), adj, trk, S.affected.data(), S.prev.data(), S.color.data(), &counter);
#else
      findEligibleNeighbors(list.data(), adj, trk, S.affected.data(), S.color.data(), &counter, prop);
#endif
    });
    counter = compact(S, list);
    std::fill(S.affected.begin(), S.affected.end(), 0);
    if (snapshot) {
      ok = snapshot_step(S, counter, [&](int j) {
#ifdef REF_HI
        recolorNeighbor(&list[j], S.color.data(), S.prev.data(), adj, trk, S.affected.data(), &one,
                        &S.change, W);
#else
        recolorNeighbor(&list[j], S.color.data(), adj, trk, S.affected.data(), &one, &S.change,
                        prop);
#endif
      });
    } else {
      launch(threads, [&] {
#ifdef REF_HI
        recolorNeighbor(list.data(), S.color.data(), S.prev.data(), adj, trk, S.affected.data(), &counter,
                        &S.change, W);
#else
        recolorNeighbor(list.data(), S.color.data(), adj, trk, S.affected.data(), &counter, &S.change, prop);
#endif
      });
    }
  }
  R.ms += std::chrono::duration<double, std::milli>(clk::now() - t0).count();
  R.iterations = it;
  R.ok = ok;
  return R;
}

}  // namespace

int main(int argc, char* argv[]) {
  if (argc < 8) {
    std::fprintf(stderr,
                 "usage: %s serial|snapshot|bench graph nodes edges prevColor changes out [iter_cap]\n",
                 argv[0]);
    return 2;
  }
  const bool bench = std::strcmp(argv[1], "bench") == 0;
  const bool snapshot = std::strcmp(argv[1], "snapshot") == 0;
  const int nodes = std::atoi(argv[3]);
  const long iter_cap = argc > 8 ? std::atol(argv[8]) : 100000;
  const double budget_ms = argc > 9 ? std::atof(argv[9]) : 0.0;  // bench mode: per-step time budget
  const int max_fail = argc > 10 ? std::atoi(argv[10]) : 0;       // bench mode: stop after this many
  const int threads = argc > 11 ? std::atoi(argv[11]) : omp_get_max_threads();
  Graph G;
  G.nodes = nodes;
  G.adj.resize(nodes);
  State S;
  S.n = nodes;
  S.color.assign(nodes, 0);
  S.prev.assign(nodes, -1);  // cudaMemset(previosVertexcolor, -1)
  S.affected.assign(nodes, 0);
#ifndef REF_HI
  G.prop.assign(nodes, 0);
#endif
  if (bench) {
    // binary inputs, same adjacency as read_graphEdges builds
    FILE* fg = std::fopen(argv[2], "rb");
    FILE* fc = std::fopen(argv[5], "rb");
    if (!fg || !fc) return 2;
    std::vector<int> pair(2 * 65536);
    size_t got;
    while ((got = std::fread(pair.data(), sizeof(int), pair.size(), fg)) >= 2) {
      for (size_t i = 0; i + 1 < got; i += 2) {
        const int n1 = pair[i], n2 = pair[i + 1];
        G.adj[n2].push_back(ColWt{n1, 0});
        G.adj[n1].push_back(ColWt{n2, 0});
#ifndef REF_HI
        G.prop[n1] += 1;
        G.prop[n2] += 1;
#endif
      }
    }
    std::fclose(fg);
    if (std::fread(S.color.data(), sizeof(int), nodes, fc) != (size_t)nodes) return 2;
    std::fclose(fc);
  } else {
#ifdef REF_HI
    int maxColor = -1;
    read_Input_Color(S.color.data(), argv[5], &maxColor);
    read_graphEdges(G.adj, argv[2]);
#else
    read_Input_Color(S.color.data(), argv[5]);
    read_graphEdges(G.adj, argv[2], G.prop.data());
#endif
  }
  FILE* f = std::fopen(argv[7], "w");
  if (!f) return 2;
  if (!bench) {
    const StepResult R = run_step(G, S, argv[6], snapshot, iter_cap);
    if (!R.ok) {
      std::fprintf(stderr, "snapshot write conflict\n");
      std::fclose(f);
      return 3;
    }
    std::fprintf(f, "iterations %ld status %d\n", R.iterations, R.status);
    for (int v = 0; v < nodes; ++v) std::fprintf(f, "%d\n", S.color[v]);
    std::fclose(f);
    return 0;
  }
  // bench: every comma-separated change file is one step on the initial state
  const State S0 = S;
#ifndef REF_HI
  const std::vector<int> prop0 = G.prop;
#endif
  std::string list = argv[6];
  size_t pos = 0;
  int fails = 0;
  while (pos <= list.size()) {
    size_t comma = list.find(',', pos);
    if (comma == std::string::npos) comma = list.size();
    const std::string file = list.substr(pos, comma - pos);
    pos = comma + 1;
    if (file.empty()) continue;
    // rows an insertion may grow: every vertex named by the file
    std::vector<std::pair<int, size_t>> sizes;
    if (FILE* cf = std::fopen(file.c_str(), "r")) {
      int x, y, w, t;
      while (std::fscanf(cf, "%d %d %d %d", &x, &y, &w, &t) == 4) {
        if (x >= 0 && x < nodes) sizes.emplace_back(x, G.adj[x].size());
        if (y >= 0 && y < nodes) sizes.emplace_back(y, G.adj[y].size());
      }
      std::fclose(cf);
    }
    const StepResult R = run_step(G, S, file.c_str(), false, iter_cap, budget_ms, threads);
    std::fprintf(f, "iterations %ld status %d time_ms %.3f threads %d\n", R.iterations, R.status, R.ms, threads);
    std::fflush(f);
    fails = R.status != 0 ? fails + 1 : 0;
    for (auto it = sizes.rbegin(); it != sizes.rend(); ++it) G.adj[it->first].resize(it->second);
    S = S0;
#ifndef REF_HI
    G.prop = prop0;
#endif
    if (max_fail > 0 && fails >= max_fail) break;
  }
  std::fclose(f);
  return 0;
}
