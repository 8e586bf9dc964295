// Command-line drivers with the reference's names and arguments, on the GPU:
//
//   bfs  | sssp | sswp  graph root                                  (src/sssp.cpp)
//   wcc                 graph                                       (src/wcc.cpp)
//   *_inc               graph [root] imported_rate                  (src/sssp_inc.cpp)
//   *_inc_batch         graph [root] imported_rate batch_size       (src/sssp_inc_batch.cpp)
//   *_inc_rt            graph [root] imported_rate timeout_ms percent clients
//                                                                   (src/sssp_inc_rt.cpp)
//
// One binary; the name it is called by (argv[0], via the links the build
// makes) picks the algorithm and the mode.  The graph file is the reference's
// binary edge list (core/io.hpp:26-36): (u64 src, u64 dst) pairs, host order,
// no header; |V| = max id + 1 (src/sssp.cpp:40-46).  Weights are
// (src + dst) % 128 as in the reference drivers (src/sssp.cpp:59), or
// splitmix64(src<<32|dst) % 255 + 1 with RG_WEIGHTS=splitmix.  Timings go to
// stderr with the reference's labels, value histograms to stdout.
// RG_DUMP_VALUES=<path> writes the final value of every vertex (u64 each).
#include <fcntl.h>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "rg_gen.h"
#include "risgraph_b200.h"

namespace {

using clk = std::chrono::high_resolution_clock;

double secs(clk::time_point a, clk::time_point b) {
  return 1e-6 * (double)std::chrono::duration_cast<std::chrono::microseconds>(b - a).count();
}

// mmap_binary (core/io.hpp:26-36)
std::pair<const uint64_t *, uint64_t> mmap_binary(const char *path) {
  int fd = open(path, O_RDONLY);
  if (fd < 0) {
    std::perror("open");
    std::exit(1);
  }
  struct stat st;
  fstat(fd, &st);
  uint64_t n = (uint64_t)st.st_size / 16;
  void *p = n ? mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0) : nullptr;
  if (n && p == MAP_FAILED) {
    std::perror("mmap");
    std::exit(1);
  }
  close(fd);
  return {reinterpret_cast<const uint64_t *>(p), n};
}

struct Cfg {
  std::string algo, mode;
  int A = 0;
  bool weighted = false, symmetric = false, splitmix = false;
  uint64_t maxl = 0;
};

uint64_t weight_of(const Cfg &c, uint64_t s, uint64_t d) {
  if (!c.weighted) return 0;
  return c.splitmix ? rg_gen_weight(s, d) : (s + d) % 128;
}

rg_edge edge_of(const Cfg &c, const uint64_t *raw, uint64_t i) {
  return rg_edge{raw[2 * i], raw[2 * i + 1], weight_of(c, raw[2 * i], raw[2 * i + 1])};
}

void check(int rc, const char *what) {
  if (rc != RG_OK) {
    std::fprintf(stderr, "%s: %s\n", what, rg_last_error());
    std::exit(1);
  }
}

std::vector<uint64_t> values_of(rg_graph *g, uint64_t V) {
  std::vector<uint64_t> v(V);
  check(rg_get_labels(g, v.data(), nullptr, nullptr), "rg_get_labels");
  return v;
}

// The drivers' closing output: value histogram (stdout) or, for WCC, the
// number of components (stderr, src/wcc.cpp:100-110).
void report(const Cfg &c, rg_graph *g, uint64_t V, uint64_t root) {
  std::vector<uint64_t> v = values_of(g, V);
  if (c.algo == "wcc") {
    uint64_t k = 0;
    for (uint64_t i = 0; i < V; i++) k += v[i] == i;
    std::fprintf(stderr, "number of communities: %lu\n", (unsigned long)k);
    return;
  }
  std::map<uint64_t, uint64_t> h;
  uint64_t visited = 0;
  for (uint64_t i = 0; i < V; i++)
    if (v[i] != c.maxl) {
      h[v[i]]++;
      visited++;
    }
  if (c.algo == "bfs") {
    std::fprintf(stderr, "%lu visited vertices: %lu\n", (unsigned long)root, (unsigned long)visited);
    uint64_t want = 0;
    for (const auto &kv : h) {  // layer sizes up to the first empty layer (src/bfs_inc_batch.cpp:204-215)
      if (kv.first != want) break;
      std::printf("%lu ", (unsigned long)kv.second);
      want++;
    }
    std::printf("\n");
  } else {
    for (const auto &kv : h) std::printf("%lu: %lu, ", (unsigned long)kv.first, (unsigned long)kv.second);
    std::printf("\n");
  }
  std::fflush(stdout);
}

void dump(rg_graph *g, uint64_t V) {
  const char *path = std::getenv("RG_DUMP_VALUES");
  if (!path || !*path) return;
  std::vector<uint64_t> v = values_of(g, V);
  FILE *f = std::fopen(path, "wb");
  if (!f || std::fwrite(v.data(), 8, V, f) != V) {
    std::fprintf(stderr, "cannot write %s\n", path);
    std::exit(1);
  }
  std::fclose(f);
}

void build(const Cfg &c, rg_graph *g, uint64_t root) {
  auto t0 = clk::now();
  check(rg_build_tree(g, c.A, root, nullptr), "rg_build_tree");
  std::fprintf(stderr, "exec: %.6lfs\n", secs(t0, clk::now()));
}

// sliding window of src/sssp_inc.cpp:251-326: step i inserts raw[i] and deletes
// raw[i - imported]; each update is applied alone (add_edge + update_tree_* on
// the multiplicity transition, fused on the device).
void run_inc(const Cfg &c, rg_graph *g, const uint64_t *raw, uint64_t E, uint64_t imported, bool directed) {
  const uint64_t print_int = c.algo == "bfs" || c.algo == "wcc" ? 1000000 : 10000000;
  auto t0 = clk::now(), pre = t0;
  for (uint64_t i = imported; i < E; i++) {
    if ((i - imported) % print_int == 0 && i != imported) {
      auto now = clk::now();
      std::fprintf(stderr, "%lu, time: %.6lfs, edges/sec: %.6lf\n", (unsigned long)(i - imported), secs(pre, now),
                   print_int / secs(pre, now));
      pre = now;
    }
    rg_edge a = edge_of(c, raw, i), d = edge_of(c, raw, i - imported);
    check(rg_apply_add(g, c.A, &a, 1, directed, nullptr), "add");
    check(rg_apply_del(g, c.A, &d, 1, directed, nullptr), "del");
  }
  std::fprintf(stderr, "exec: %.6lfs\n", secs(t0, clk::now()));
}

// batches of src/sssp_inc_batch.cpp:136-181: all inserts of the batch, then all
// deletes.
void run_batch(const Cfg &c, rg_graph *g, const uint64_t *raw, uint64_t E, uint64_t imported, uint64_t batch,
               bool directed) {
  std::vector<rg_edge> add(batch), del(batch);
  uint64_t num_batches = 0;
  auto t0 = clk::now();
  for (uint64_t lo = imported; lo < E; lo += batch) {
    uint64_t hi = std::min(lo + batch, E), n = hi - lo;
    for (uint64_t i = lo; i < hi; i++) {
      add[i - lo] = edge_of(c, raw, i);
      del[i - lo] = edge_of(c, raw, i - imported);
    }
    check(rg_apply_add(g, c.A, add.data(), n, directed, nullptr), "add batch");
    check(rg_apply_del(g, c.A, del.data(), n, directed, nullptr), "del batch");
    num_batches++;
  }
  const double ns = 1e9 * secs(t0, clk::now());
  std::fprintf(stderr, "wall_times = %lf us\n", 1e-3 * ns);
  std::fprintf(stderr, "wall_mean = %lf us\n", num_batches ? 1e-3 * ns / num_batches : 0.0);
}

// src/sssp_inc_rt.cpp:119-441: `clients` closed-loop clients send the sliding
// window's updates to the served path until the window reaches the end of the
// file; per-update latency percentiles and the fraction within timeout_ms.
void run_rt(const Cfg &c, rg_graph *g, const uint64_t *raw, uint64_t E, uint64_t imported, uint32_t timeout_ms,
            double percent, uint64_t clients, bool directed) {
  rg_server *srv = nullptr;
  // an epoch aims at a fifth of the timeout (the reference breaks at 0.8 of it)
  check(rg_server_create(0, std::max(0.05, timeout_ms * 0.2), 1 << 16, 0, &srv), "rg_server_create");
  uint32_t inst = 0;
  check(rg_server_attach(srv, g, c.A, directed, &inst), "rg_server_attach");
  const uint64_t total = 2 * (E - imported);
  const uint64_t C = std::max<uint64_t>(1, clients);
  std::vector<uint64_t> lat;
  lat.reserve(total);
  auto t0 = clk::now();
  if (!c.weighted || c.splitmix) {
    // the built-in closed-loop load (its weights are rg_gen_weight's)
    rg_load_config lc{};
    lc.instance = inst;
    lc.clients = (uint32_t)C;
    lc.duration_s = 1e9;
    lc.max_updates = total;
    lc.pairs = raw;
    lc.n_pairs = E;
    lc.imported = imported;
    lc.weighted = c.weighted ? 1 : 0;
    lc.seed = 1;
    lat.resize(total);
    lc.latencies_ns = lat.data();
    lc.latencies_cap = total;
    rg_load_result r{};
    check(rg_server_run_load(srv, &lc, 1, &r), "rg_server_run_load");
    lat.resize(std::min<uint64_t>(r.completed, total));
  } else {
    // the reference's (s+d)%128 weights: explicit requests, one in flight per client
    std::vector<rg_completion> comp(4096);
    uint64_t issued = 0, outstanding = 0;
    auto issue = [&](uint64_t tag) {
      const uint64_t s = issued++;
      const bool add = (s & 1) == 0;
      const uint64_t idx = add ? imported + s / 2 : s / 2;
      rg_request q{inst, add ? 0u : 1u, raw[2 * idx], raw[2 * idx + 1], weight_of(c, raw[2 * idx], raw[2 * idx + 1]),
                   tag};
      check(rg_server_submit(srv, &q, 1), "rg_server_submit");
      outstanding++;
    };
    for (uint64_t k = 0; k < C && issued < total; k++) issue(k);
    while (outstanding) {
      uint64_t n = 0;
      check(rg_server_poll(srv, comp.data(), comp.size(), &n), "rg_server_poll");
      if (!n) {
        std::this_thread::yield();
        continue;
      }
      for (uint64_t i = 0; i < n; i++) {
        lat.push_back(comp[i].done_ns - comp[i].submit_ns);
        outstanding--;
        if (issued < total) issue(comp[i].tag);
      }
    }
  }
  const double wall = secs(t0, clk::now());
  check(rg_server_detach(srv, inst), "rg_server_detach");
  rg_server_destroy(srv);
  const uint64_t done = lat.size();
  std::sort(lat.begin(), lat.end());
  uint64_t timeouts = 0;
  double sum = 0;
  for (uint64_t x : lat) {
    sum += (double)x;
    timeouts += x > (uint64_t)timeout_ms * 1000000ull;
  }
  auto P = [&](double q) {
    return lat.empty() ? 0.0 : 1e-3 * (double)lat[std::min(lat.size() - 1, (size_t)(lat.size() * q))];
  };
  std::fprintf(stderr, "target success rate: %lf\n", percent);
  std::fprintf(stderr, "exec:       %.6lfs\n", wall);
  std::fprintf(stderr, "Throughput: %lf\n", done / wall);
  std::fprintf(stderr, "Success:    %lf\n", done ? 1.0 - (double)timeouts / done : 0.0);
  std::fprintf(stderr, "Mean:       %lf us\n", done ? 1e-3 * sum / done : 0.0);
  const double qs[] = {0.25, 0.5, 0.75, 0.9, 0.99, 0.999, 0.9999, 0.99999, 0.999999, 0.9999999, 0.99999999};
  const char *names[] = {"P25:", "P50:", "P75:", "P90:", "P99:", "P999:", "P9999:", "P99999:", "P999999:",
                         "P9999999:", "P99999999:"};
  for (int i = 0; i < 11; i++) std::fprintf(stderr, "%-11s %lfus\n", names[i], P(qs[i]));
  std::fprintf(stderr, "Max:        %lfus\n", lat.empty() ? 0.0 : 1e-3 * (double)lat.back());
}

int usage(const char *name, const Cfg &c) {
  const char *root = c.algo == "wcc" ? "" : " root";
  if (c.mode.empty()) std::fprintf(stderr, "usage: %s graph%s\n", name, root);
  else if (c.mode == "_inc") std::fprintf(stderr, "usage: %s graph%s imported_rate\n", name, root);
  else if (c.mode == "_inc_batch") std::fprintf(stderr, "usage: %s graph%s imported_rate batch_size\n", name, root);
  else std::fprintf(stderr, "usage: %s graph%s imported_rate timeout_ms percent clients\n", name, root);
  return 1;
}

}  // namespace

int main(int argc, char **argv) {
  std::string name = argv[0];
  name = name.substr(name.find_last_of('/') + 1);
  Cfg c;
  for (const char *a : {"bfs", "sssp", "sswp", "wcc"})
    if (name.rfind(a, 0) == 0 && (name.size() == std::strlen(a) || name[std::strlen(a)] == '_')) c.algo = a;
  if (c.algo.empty()) {
    std::fprintf(stderr, "%s: call as bfs|sssp|sswp|wcc[_inc|_inc_batch|_inc_rt]\n", name.c_str());
    return 1;
  }
  c.mode = name.substr(c.algo.size());
  if (!c.mode.empty() && c.mode != "_inc" && c.mode != "_inc_batch" && c.mode != "_inc_rt") return usage(argv[0], c);
  c.A = c.algo == "bfs" ? RG_BFS : c.algo == "sssp" ? RG_SSSP : c.algo == "sswp" ? RG_SSWP : RG_WCC;
  c.weighted = c.algo == "sssp" || c.algo == "sswp";
  c.symmetric = c.algo == "wcc";
  c.maxl = c.algo == "bfs" ? 65536 : 134217728;
  const char *wenv = std::getenv("RG_WEIGHTS");
  c.splitmix = wenv && std::string(wenv) == "splitmix";
  const int has_root = c.algo == "wcc" ? 0 : 1;
  const int need = 2 + has_root + (c.mode.empty() ? 0 : 1) + (c.mode == "_inc_batch" ? 1 : 0) +
                   (c.mode == "_inc_rt" ? 3 : 0);
  if (argc < need) return usage(argv[0], c);
  const uint64_t root = has_root ? std::stoull(argv[2]) : 0;
  const double rate = c.mode.empty() ? 1.0 : std::stod(argv[2 + has_root]);

  auto t0 = clk::now();
  auto [raw, E] = mmap_binary(argv[1]);
  uint64_t V = 0;
#pragma omp parallel for reduction(max : V)
  for (uint64_t i = 0; i < 2 * E; i++) V = std::max(V, raw[i] + 1);
  std::fprintf(stderr, "read: %.6lfs\n", secs(t0, clk::now()));
  std::fprintf(stderr, "|E|=%lu\n", (unsigned long)E);
  if (has_root && root >= V) {
    std::fprintf(stderr, "VertexId error.\n");
    return 1;
  }
  const bool directed = !c.symmetric;
  // WCC keeps in-edges only for plain runs (Graph(..., true, false) in src/wcc_inc.cpp:56)
  const bool dual = !(c.algo == "wcc" && !c.mode.empty());
  rg_graph *g = nullptr;
  check(rg_create(V, E, c.symmetric, dual, 0, c.weighted, &g), "rg_create");
  const uint64_t imported = c.mode.empty() ? E : (uint64_t)(E * rate);
  {
    auto t = clk::now();
    const uint64_t chunk = 1ull << 24;
    std::vector<rg_edge> buf;
    for (uint64_t lo = 0; lo < imported; lo += chunk) {
      const uint64_t hi = std::min(imported, lo + chunk);
      if (c.weighted && !c.splitmix) {
        buf.resize(hi - lo);
#pragma omp parallel for
        for (uint64_t i = lo; i < hi; i++) buf[i - lo] = edge_of(c, raw, i);
        check(rg_add_edges(g, buf.data(), hi - lo, directed, nullptr), "rg_add_edges");
      } else {
        check(rg_add_pairs(g, raw + 2 * lo, hi - lo, directed, nullptr), "rg_add_pairs");
      }
    }
    std::fprintf(stderr, "add: %.6lfs\n", secs(t, clk::now()));
  }
  build(c, g, root);
  if (c.mode.empty()) {
    report(c, g, V, root);
  } else {
    if (c.mode == "_inc") {
      run_inc(c, g, raw, E, imported, directed);
    } else if (c.mode == "_inc_batch") {
      const uint64_t batch = std::max<uint64_t>(1, std::stoull(argv[3 + has_root]));
      run_batch(c, g, raw, E, imported, batch, directed);
    } else {
      run_rt(c, g, raw, E, imported, (uint32_t)std::stoul(argv[3 + has_root]), std::stod(argv[4 + has_root]),
             std::stoull(argv[5 + has_root]), directed);
    }
    report(c, g, V, root);
    dump(g, V);
    // self-check of the drivers: a rebuild from scratch gives the same tree
    std::vector<uint64_t> inc = values_of(g, V);
    build(c, g, root);
    report(c, g, V, root);
    if (values_of(g, V) != inc) {
      std::fprintf(stderr, "incremental values differ from a rebuild\n");
      return 2;
    }
    rg_destroy(g);
    return 0;
  }
  dump(g, V);
  rg_destroy(g);
  return 0;
}
