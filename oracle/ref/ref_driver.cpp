// Oracle driver around the reference's UNMODIFIED hot path (core/graph.hpp),
// compiled from the reference's own headers with the OpenMP stand-in under
// oracle/ref/shim.  Test infrastructure only: it produces golden values and the
// timed CPU baseline; nothing in the product links it.
//
// It differs from the reference's src/{bfs,sssp,sswp,wcc}{,_inc,_inc_batch}.cpp
// drivers in four ways: |V| is passed explicitly (the reference infers
// max id + 1, src/sssp.cpp:40-46); weights are splitmix64(src<<32|dst)%255+1
// (the reference uses (src+dst)%128, src/sssp.cpp:59); per-vertex values,
// parents and a per-step value checksum are written out (the reference prints
// histograms, src/sssp_inc.cpp:354-416); the number of updates is capped (the
// reference runs to the end of the file).  The per-algorithm hooks are the
// reference drivers' a8 hooks restated: BFS src/bfs.cpp:76-91, SSSP
// src/sssp.cpp:67-91, SSWP src/sswp.cpp:76-91, WCC src/wcc.cpp:62-86.
//
// Usage:
//   ref_driver build <algo> <graph.bin> <V> <root> <out|-> [repeats warmup]
//   ref_driver inc   <algo> <graph.bin> <V> <root> <rate> <steps> <out|->
//   ref_driver batch <algo> <graph.bin> <V> <root> <rate> <batch> <nbatches> <out|->
// algo: bfs | sssp | sswp | wcc.  Output files: <out>.val <out>.par <out>.pw
// (uint64 per vertex; par == V means no parent) and <out>.sums (uint64 per step).
// One JSON line with timings goes to stdout.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "core/graph.hpp"
#include "core/io.hpp"
#include "core/type.hpp"

extern "C" {
#include "rg_gen.h"
}

namespace {

using clk = std::chrono::steady_clock;
double secs(clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); }

enum Algo { BFS, SSSP, SSWP, WCC };

Algo parse_algo(const char *s) {
  if (!strcmp(s, "bfs")) return BFS;
  if (!strcmp(s, "sssp")) return SSSP;
  if (!strcmp(s, "sswp")) return SSWP;
  if (!strcmp(s, "wcc")) return WCC;
  fprintf(stderr, "unknown algo %s\n", s);
  exit(2);
}

// Edge construction: weighted graphs carry the splitmix weight.
template <typename G>
typename G::edge_type make_edge(uint64_t s, uint64_t d);
template <>
Graph<void>::edge_type make_edge<Graph<void>>(uint64_t s, uint64_t d) { return {s, d}; }
template <>
Graph<uint64_t>::edge_type make_edge<Graph<uint64_t>>(uint64_t s, uint64_t d) {
  return {s, d, rg_gen_weight(s, d)};
}

template <typename E>
uint64_t edge_w(const E &e) { return (uint64_t)e.data; }

template <typename G>
struct Hooks;

// a8 hooks as lambdas-in-structs.  R = uint64_t counters, DataType = uint64_t.
template <typename G>
struct Hooks {
  Algo algo;
  uint64_t root;
  static constexpr uint64_t BFS_MAXL = 65536;        // src/bfs.cpp:66
  static constexpr uint64_t SSSP_MAXL = 134217728;   // src/sssp.cpp:66, src/sswp.cpp:66

  auto continue_reduce() const {
    return [](uint64_t, uint64_t total, uint64_t local) -> std::pair<bool, uint64_t> {
      return std::make_pair(local > 0, total + local);
    };
  }
  auto active_result() const {
    return [](uint64_t old_result, uint64_t, uint64_t, uint64_t, uint64_t, uint64_t) -> uint64_t {
      return old_result + 1;
    };
  }
  auto update() const {
    Algo a = algo;
    return [a](uint64_t, uint64_t, uint64_t s, uint64_t d, typename G::adjedge_type e) -> std::pair<bool, uint64_t> {
      uint64_t w = (uint64_t)e.data;
      switch (a) {
        case BFS: return std::make_pair(s + 1 < d, s + 1);
        case SSSP: return std::make_pair(s + w < d, s + w);
        case SSWP: { uint64_t m = std::min(s, w); return std::make_pair(m > d, m); }
        default: return std::make_pair(s < d, s);
      }
    };
  }
  auto equal() const {
    Algo a = algo;
    return [a](uint64_t, uint64_t, uint64_t s, uint64_t d, typename G::adjedge_type e) -> bool {
      uint64_t w = (uint64_t)e.data;
      switch (a) {
        case BFS: return s + 1 == d;
        case SSSP: return s + w == d;
        case SSWP: return std::min(s, w) == d;
        default: return s == d;
      }
    };
  }
  auto init() const {
    Algo a = algo;
    uint64_t r = root;
    return [a, r](uint64_t vid) -> std::pair<uint64_t, bool> {
      switch (a) {
        case BFS: return {vid == r ? 0 : BFS_MAXL, vid == r};
        case SSSP: return {vid == r ? 0 : SSSP_MAXL, vid == r};
        case SSWP: return {vid == r ? SSSP_MAXL : 0, vid == r};
        default: return {vid, true};
      }
    };
  }
};

struct Out {
  std::string prefix;
  void write(const char *ext, const std::vector<uint64_t> &v) const {
    if (prefix == "-") return;
    std::string p = prefix + ext;
    FILE *f = fopen(p.c_str(), "wb");
    if (!f) { perror(p.c_str()); exit(3); }
    fwrite(v.data(), 8, v.size(), f);
    fclose(f);
  }
};

template <typename G, typename L>
void dump_labels(const Out &out, const L &labels, uint64_t V) {
  std::vector<uint64_t> val(V), par(V), pw(V);
  for (uint64_t v = 0; v < V; v++) {
    val[v] = labels[v].data;
    par[v] = labels[v].parent.nbr;
    pw[v] = (uint64_t)labels[v].parent.data;
  }
  out.write(".val", val);
  out.write(".par", par);
  out.write(".pw", pw);
}

template <typename L>
uint64_t checksum(const L &labels, uint64_t V, std::vector<uint64_t> &tmp) {
  for (uint64_t v = 0; v < V; v++) tmp[v] = labels[v].data;
  return rg_gen_value_checksum(tmp.data(), V);
}

template <typename G>
int run(int argc, char **argv) {
  const char *mode = argv[1];
  Algo algo = parse_algo(argv[2]);
  auto raw = mmap_binary(argv[3]);
  std::pair<uint64_t, uint64_t> *edges = raw.first;
  uint64_t E = raw.second;
  uint64_t V = std::stoull(argv[4]);
  uint64_t root = std::stoull(argv[5]);
  bool symmetric = (algo == WCC), directed = (algo != WCC);
  bool inc_mode = strcmp(mode, "build") != 0;
  // WCC incremental drivers construct (symmetric, !dual) (src/wcc_inc.cpp:56);
  // every other driver uses dual = true.
  bool dual = !(algo == WCC && inc_mode);

  double rate = 1.0;
  uint64_t steps = 0, batch = 1;
  std::string prefix;
  uint64_t repeats = 1, warmup = 0;
  if (!strcmp(mode, "build")) {
    prefix = argv[6];
    if (argc > 8) { repeats = std::stoull(argv[7]); warmup = std::stoull(argv[8]); }
  } else if (!strcmp(mode, "inc")) {
    rate = std::stod(argv[6]); steps = std::stoull(argv[7]); prefix = argv[8];
  } else if (!strcmp(mode, "batch")) {
    rate = std::stod(argv[6]); batch = std::stoull(argv[7]); steps = std::stoull(argv[8]); prefix = argv[9];
  } else {
    fprintf(stderr, "unknown mode %s\n", mode);
    return 2;
  }
  for (uint64_t i = 0; i < E; i++)
    if (edges[i].first >= V || edges[i].second >= V) { fprintf(stderr, "edge %lu out of range\n", i); return 4; }
  uint64_t imported = inc_mode ? (uint64_t)(E * rate) : E;   // src/sssp_inc.cpp:190-191

  G graph(V, E, symmetric, dual);
  Hooks<G> h{algo, root};
  auto t0 = clk::now();
#pragma omp parallel for
  for (uint64_t i = 0; i < imported; i++)
    graph.add_edge(make_edge<G>(edges[i].first, edges[i].second), directed);
  auto t1 = clk::now();

  auto labels = graph.template alloc_vertex_tree_array<uint64_t>();
  std::vector<double> build_times;
  for (uint64_t r = 0; r < warmup + repeats; r++) {
    auto b0 = clk::now();
    graph.template build_tree<uint64_t, uint64_t>(h.init(), h.continue_reduce(), h.update(), h.active_result(), labels);
    auto b1 = clk::now();
    if (r >= warmup) build_times.push_back(secs(b0, b1));
  }
  Out out{prefix};
  std::vector<uint64_t> tmp(V), sums;
  uint64_t n_tree_add = 0, n_tree_del = 0;
  double upd = 0.0;

  if (!strcmp(mode, "inc")) {
    uint64_t end = std::min(E, imported + steps);
    for (uint64_t i = imported; i < end; i++) {
      auto u0 = clk::now();
      {
        auto e = make_edge<G>(edges[i].first, edges[i].second);
        if (graph.add_edge(e, directed) == 0) {
          n_tree_add++;
          graph.template update_tree_add<uint64_t, uint64_t>(h.continue_reduce(), h.update(), h.active_result(), labels, e, directed);
        }
      }
      {
        auto e = make_edge<G>(edges[i - imported].first, edges[i - imported].second);
        if (graph.del_edge(e, directed) == 1) {
          n_tree_del++;
          graph.template update_tree_del<uint64_t, uint64_t>(h.init(), h.continue_reduce(), h.update(), h.active_result(), h.equal(), labels, e, directed);
        }
      }
      upd += secs(u0, clk::now());
      sums.push_back(checksum(labels, V, tmp));
    }
  } else if (!strcmp(mode, "batch")) {
    std::vector<typename G::edge_type> added(batch), deled(batch);
    uint64_t nb = 0;
    for (uint64_t b0 = imported; b0 < E && nb < steps; b0 += batch, nb++) {
      uint64_t b1 = std::min(b0 + batch, E);
      auto u0 = clk::now();
      {
        std::atomic_uint64_t len(0);
#pragma omp parallel for if (b1 - b0 > 1024)
        for (uint64_t i = b0; i < b1; i++) {
          auto e = make_edge<G>(edges[i].first, edges[i].second);
          if (graph.add_edge(e, directed) == 0) added[len.fetch_add(1)] = e;
        }
        n_tree_add += len.load();
        graph.template update_tree_add<uint64_t, uint64_t>(h.continue_reduce(), h.update(), h.active_result(), labels, added, len.load(), directed);
      }
      {
        std::atomic_uint64_t len(0);
#pragma omp parallel for if (b1 - b0 > 1024)
        for (uint64_t i = b0; i < b1; i++) {
          auto e = make_edge<G>(edges[i - imported].first, edges[i - imported].second);
          if (graph.del_edge(e, directed) == 1) deled[len.fetch_add(1)] = e;
        }
        n_tree_del += len.load();
        graph.template update_tree_del<uint64_t, uint64_t>(h.init(), h.continue_reduce(), h.update(), h.active_result(), h.equal(), labels, deled, len.load(), directed);
      }
      upd += secs(u0, clk::now());
      sums.push_back(checksum(labels, V, tmp));
    }
  }

  dump_labels<G>(out, labels, V);
  if (inc_mode) out.write(".sums", sums);
  double bsum = 0;
  for (double t : build_times) bsum += t;
  printf("{\"mode\": \"%s\", \"algo\": \"%s\", \"V\": %lu, \"E\": %lu, \"imported\": %lu, \"threads\": %d, "
         "\"load_s\": %.6f, \"build_s\": %.6f, \"build_times\": [",
         mode, argv[2], V, E, imported, omp_get_max_threads(), secs(t0, t1), build_times.empty() ? 0.0 : bsum / build_times.size());
  for (size_t i = 0; i < build_times.size(); i++) printf("%s%.6f", i ? ", " : "", build_times[i]);
  printf("], \"update_s\": %.6f, \"steps\": %lu, \"tree_add\": %lu, \"tree_del\": %lu, \"checksum\": %lu}\n",
         upd, (uint64_t)sums.size(), n_tree_add, n_tree_del, checksum(labels, V, tmp));
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 7) {
    fprintf(stderr, "usage: ref_driver build|inc|batch algo graph.bin V root ...\n");
    return 2;
  }
  Algo a = parse_algo(argv[2]);
  if (a == BFS || a == WCC) return run<Graph<void>>(argc, argv);
  return run<Graph<uint64_t>>(argc, argv);
}
