// dc_cli.cpp -- the `dyncolor` command: the reference drivers' argv and text
// files on top of the C ABI (include/dyncolor.h).
//
//   dyncolor <graph> <nodes> <edges> <prevColor> <changes>
//            [--variant hi|hb] [--out colors.txt] [--device N] [--iter-cap N]
//
// argv as in HI/Color_main.cu:21-37 and HB/Color_main.cu:22-38 (graph file,
// vertex count, edge count, input colour file, change file); `edges` is
// advisory, as in the reference, which only sized an allocation with it.
// Text formats as read by the reference (HI/all_structure_undir.cuh:78-183,
// HB/all_structure_undir.cuh:78-186):
//   graph      "a b w" per line: the undirected edge {a, b}; w is ignored
//   prevColor  "node color" per line
//   changes    "a b w inst" per line: inst 1 inserts, 0 deletes, other
//              values are ignored
// Lines are read 127 characters at a time (a longer line continues as the
// next one) and parsed with sscanf, like the reference's fgets/sscanf loop;
// the last line needs no newline.  Where the reference's behaviour is
// undefined the command refuses instead: a line that does not parse is
// skipped (the reference would reuse the previous line's numbers), and a
// vertex id outside [0, nodes) is an error (the reference throws or writes
// out of bounds).
//
// Output: the reference's timing lines, the highest colour id used, one
// "##Error found: u v" line per monochromatic edge (validate,
// HI/gpuFunctions_undir.cuh:289-305, at most 100 lines, then a count), and
// with --out the colours as "node color" lines in the colour file's format.
// Exit status 0 when the colouring is proper, 1 when it is not, 2 on a usage,
// input or device error.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dyncolor.h"

namespace {

using Clock = std::chrono::steady_clock;

double us_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::micro>(Clock::now() - t0).count();
}

// Calls f(line) for every line of path read the reference's way (fgets into
// a 128-byte buffer).  Returns false when the file cannot be opened.
template <class F>
bool for_each_line(const char* path, F f) {
  FILE* fp = std::fopen(path, "r");
  if (!fp) return false;
  char line[128];
  while (std::fgets(line, sizeof(line), fp) != nullptr) f(line);
  std::fclose(fp);
  return true;
}

int usage() {
  std::fprintf(stderr,
               "usage: dyncolor <graph> <nodes> <edges> <prevColor> <changes> [--variant hi|hb] "
               "[--out colors.txt] [--device N] [--iter-cap N]\n");
  return 2;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 6) return usage();
  const char* graph_path = argv[1];
  const long long nodes_ll = std::atoll(argv[2]);
  const char* color_path = argv[4];
  const char* change_path = argv[5];
  int variant = DC_HI;
  const char* out_path = nullptr;
  int device = 0;
  long long iter_cap = 0;
  for (int i = 6; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--variant" && i + 1 < argc) {
      const std::string v = argv[++i];
      if (v == "hi")
        variant = DC_HI;
      else if (v == "hb")
        variant = DC_HB;
      else
        return usage();
    } else if (a == "--out" && i + 1 < argc) {
      out_path = argv[++i];
    } else if (a == "--device" && i + 1 < argc) {
      device = std::atoi(argv[++i]);
    } else if (a == "--iter-cap" && i + 1 < argc) {
      iter_cap = std::atoll(argv[++i]);
    } else {
      return usage();
    }
  }
  if (nodes_ll < 0 || nodes_ll > 0x7fffffffll) {
    std::fprintf(stderr, "nodes must lie in [0, 2^31)\n");
    return 2;
  }
  const int nodes = (int)nodes_ll;

  // read_Input_Color (HI/all_structure_undir.cuh:130-150)
  std::vector<int32_t> colors((size_t)nodes, 0);
  int max_color = -1;
  bool bad_input = false;
  if (!for_each_line(color_path, [&](const char* line) {
        int v, c;
        if (std::sscanf(line, "%d %d", &v, &c) != 2) return;
        if (v < 0 || v >= nodes || c < 0) {
          bad_input = true;
          return;
        }
        colors[(size_t)v] = c;
        if (c > max_color) max_color = c;
      })) {
    std::fprintf(stderr, "cannot open %s\n", color_path);
    return 2;
  }
  if (bad_input) {
    std::fprintf(stderr, "%s: a vertex id outside [0, %d) or a negative colour\n", color_path, nodes);
    return 2;
  }
  std::printf("Max color id in input graph: %d\n", max_color);

  // read_graphEdges (HI/all_structure_undir.cuh:156-183)
  std::printf("Reading input graph...\n");
  Clock::time_point t0 = Clock::now();
  std::vector<int32_t> ea, eb;
  if (!for_each_line(graph_path, [&](const char* line) {
        int a, b, w;
        if (std::sscanf(line, "%d %d %d", &a, &b, &w) < 2) return;
        ea.push_back(a);
        eb.push_back(b);
      })) {
    std::fprintf(stderr, "cannot open %s\n", graph_path);
    return 2;
  }
  std::printf("Reading input graph completed\n");
  std::printf("Time taken to read input graph: %lld microseconds\n", (long long)us_since(t0));

  // readin_changes (HI/all_structure_undir.cuh:78-128)
  std::printf("Reading input changed edges data...\n");
  t0 = Clock::now();
  std::vector<dc_change> changes;
  long long total_insertion = 0;
  if (!for_each_line(change_path, [&](const char* line) {
        int a, b, w, inst;
        if (std::sscanf(line, "%d %d %d %d", &a, &b, &w, &inst) != 4) return;
        changes.push_back(dc_change{a, b, inst});
        if (inst == 1) ++total_insertion;
      })) {
    std::fprintf(stderr, "cannot open %s\n", change_path);
    return 2;
  }
  std::printf("Reading input changed edges data completed. totalInsertion:%lld\n", total_insertion);
  std::printf("Time taken to read input changed edges: %lld microseconds\n", (long long)us_since(t0));

  dc_options opt;
  dc_options_default(&opt);
  opt.variant = variant;
  opt.device = device;
  if (iter_cap > 0) opt.iter_cap = iter_cap;
  dc_ctx* ctx = nullptr;
  dc_status s = dc_create(&ctx, &opt);
  if (s != DC_OK) {
    std::fprintf(stderr, "dc_create: %s\n", dc_status_str(s));
    return 2;
  }
  auto fail = [&](const char* what, dc_status st) {
    std::fprintf(stderr, "%s: %s: %s\n", what, dc_status_str(st), dc_last_error(ctx));
    dc_destroy(ctx);
    return 2;
  };
  std::printf("Transferring graph data from CPU to GPU\n");
  t0 = Clock::now();
  s = dc_graph_load_edges(ctx, nodes, ea.data(), eb.data(), (int64_t)ea.size());
  if (s != DC_OK) return fail("graph", s);
  s = dc_colors_set(ctx, colors.data(), nodes);
  if (s != DC_OK) return fail("colours", s);
  std::printf("**Time taken to transfer graph data from CPU to GPU: %.3f milliseconds**\n", us_since(t0) / 1e3);

  dc_stats st;
  std::memset(&st, 0, sizeof(st));
  s = dc_apply_batch(ctx, changes.data(), (int64_t)changes.size(), &st);
  if (s != DC_OK && s != DC_E_ITER_LIMIT) return fail("apply batch", s);
  std::printf("**Time taken for the structural update of the batch: %.3f milliseconds**\n", st.struct_ms);
  std::printf("**Time taken for processing affected neighbors: %.3f milliseconds** (%lld iterations)\n",
              st.recolor_ms, (long long)st.iterations);
  std::printf("****Total Time for Vertex Color Update: %.3f milliseconds****\n", st.device_ms);
  if (s == DC_E_ITER_LIMIT) std::printf("iteration cap reached: the colouring is partial\n");

  s = dc_colors_read(ctx, colors.data(), nodes);
  if (s != DC_OK) return fail("read colours", s);
  int hi_color = -1;
  for (int v = 0; v < nodes; ++v)
    if (colors[(size_t)v] > hi_color) hi_color = colors[(size_t)v];
  std::printf("highest color id used: %d\n", hi_color);

  // validate (HI/gpuFunctions_undir.cuh:289-305): the count on the device,
  // and the edges themselves when there are any
  int64_t conflicts = 0;
  s = dc_validate(ctx, &conflicts);
  if (s != DC_OK) return fail("validate", s);
  if (conflicts > 0) {
    int printed = 0;
    std::vector<int32_t> row;
    for (int v = 0; v < nodes && printed < 100; ++v) {
      int32_t deg = 0;
      if (dc_neighbors(ctx, v, nullptr, 0, &deg) != DC_OK) break;
      row.resize((size_t)deg > 0 ? (size_t)deg : 1);
      if (dc_neighbors(ctx, v, row.data(), deg, &deg) != DC_OK) break;
      for (int32_t i = 0; i < deg && printed < 100; ++i)
        if (row[(size_t)i] > v && colors[(size_t)row[(size_t)i]] == colors[(size_t)v]) {
          std::printf("##Error found: %d %d\n", v, row[(size_t)i]);
          ++printed;
        }
    }
    std::printf("##%lld monochromatic edges\n", (long long)conflicts);
  }
  dc_destroy(ctx);

  if (out_path) {
    FILE* fo = std::fopen(out_path, "w");
    if (!fo) {
      std::fprintf(stderr, "cannot write %s\n", out_path);
      return 2;
    }
    for (int v = 0; v < nodes; ++v) std::fprintf(fo, "%d %d\n", v, colors[(size_t)v]);
    std::fclose(fo);
  }
  return conflicts == 0 ? 0 : 1;
}
