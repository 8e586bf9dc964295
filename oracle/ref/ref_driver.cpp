// Oracle driver around the reference's UNMODIFIED hot path (core/graph.hpp),
// compiled from the reference's own headers with the OpenMP stand-in under
// oracle/ref/shim.  Test infrastructure only: it produces golden values and the
// timed CPU baselines; nothing in the product links it.
//
// It differs from the reference's src/{bfs,sssp,sswp,wcc}{,_inc,_inc_batch,_inc_rt}.cpp
// drivers in four ways: |V| is passed explicitly (the reference infers
// max id + 1, src/sssp.cpp:40-46); weights are splitmix64(src<<32|dst)%255+1
// (the reference uses (src+dst)%128, src/sssp.cpp:59); per-vertex values,
// parents and a per-step value checksum are written out (the reference prints
// histograms, src/sssp_inc.cpp:354-416); the number of updates is capped (the
// reference runs to the end of the file, and its _inc_rt loop reads one past
// the end, src/sssp_inc_rt.cpp:235,273).  The per-algorithm hooks are the
// reference drivers' a8 hooks restated: BFS src/bfs.cpp:76-91, SSSP
// src/sssp.cpp:67-91, SSWP src/sswp.cpp:76-91, WCC src/wcc.cpp:62-86.
//
// Usage:
//   ref_driver build  <algo> <graph> <V> <root> <out|-> [repeats warmup]
//   ref_driver inc    <algo> <graph> <V> <root> <rate> <steps> <out|->
//   ref_driver batch  <algo> <graph> <V> <root> <rate> <batch> <nbatches> <out|->
//   ref_driver sweep  <algo> <graph> <V> <root> <rate> <spec> <out|->
//   ref_driver replay <algo> <graph> <V> <root> <loaded> <batchfile> <out|->
//   ref_driver rt     <algo> <graph> <V> <root> <rate> <clients,...> <timeout_ms> <max_updates> <out|->
// algo: bfs | sssp | sswp | wcc.
// graph: a file in the reference's binary format (core/io.hpp:26-36), or
//   rmat:<scale>:<seed>            the 16*2^scale-edge RMAT stream of rg_gen_rmat (longer
//                                  when a window below reaches past its end)
//   mix:<scale>:<edges>:<seed>     the ER+RMAT mix of rg_gen_er_rmat_mix
// generated in memory (a/b/c = .57/.19/.19), so no other library is needed;
// a suffix @<lo>:<hi> keeps edges [lo, hi) of the list only (the window a
// sliding-window run has reached).
// V: vertex count (0 = 2^scale for a generated graph).  root: a vertex id or
// "maxdeg" (highest out-degree, lowest id on ties).
// sweep spec: comma-separated <batch>x<count> items, run as consecutive
//   sliding-window batches (each inserts the next `batch` edges and deletes the
//   `batch` oldest loaded ones, src/sssp_inc_batch.cpp:136-181).
// replay batchfile: records of uint64 n_add, n_del, then n_add (src,dst) pairs
//   and n_del (src,dst) pairs; each record is one batch (all inserts, then all
//   deletes) after the first `loaded` edges of the graph were added.
// rt: the reference's latency-aware epoch loop (src/sssp_inc_rt.cpp:119-441)
//   with closed-loop clients and its adaptive unsafe-update threshold, one run
//   of max_updates updates per listed client count, each run continuing the
//   sliding window where the previous one stopped.
// Output files: <out>.val <out>.par <out>.pw (uint64 per vertex; par == V means
// no parent) and <out>.sums (uint64 per step or batch).  One JSON line with
// timings goes to stdout.
#include <parallel/algorithm>

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "core/graph.hpp"
#include "core/io.hpp"
#include "core/mvvec.hpp"
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

// The input edge list: mapped from a file or generated into memory.
struct Input {
  std::pair<uint64_t, uint64_t> *edges = nullptr;
  uint64_t n = 0;
  uint64_t scale = 0;
  std::vector<uint64_t> owned;
};

Input load_input(const char *spec_arg) {
  Input in;
  unsigned sc = 0;
  unsigned long long seed = 0, ne = 0, lo = 0, hi = 0;
  std::string spec(spec_arg);
  bool window = false;
  size_t at = spec.find('@');
  if (at != std::string::npos) {
    if (sscanf(spec.c_str() + at + 1, "%llu:%llu", &lo, &hi) != 2 || lo > hi) {
      fprintf(stderr, "bad window in %s\n", spec_arg);
      exit(2);
    }
    window = true;
    spec.resize(at);
  }
  if (sscanf(spec.c_str(), "rmat:%u:%llu", &sc, &seed) == 2) {
    in.scale = sc;
    // the stream continues past 16 * 2^scale edges when a window reaches beyond
    // (the generator is counter-based: a longer stream keeps the same prefix)
    in.n = std::max<unsigned long long>(16ull << sc, window ? hi : 0);
    in.owned.resize(2 * in.n);
    rg_gen_rmat(sc, 0, in.n, 0.57, 0.19, 0.19, seed, in.owned.data());
  } else if (sscanf(spec.c_str(), "mix:%u:%llu:%llu", &sc, &ne, &seed) == 3) {
    in.scale = sc;
    in.n = ne;
    in.owned.resize(2 * in.n);
    rg_gen_er_rmat_mix(sc, 0, in.n, 0.57, 0.19, 0.19, seed, in.owned.data());
  } else {
    auto raw = mmap_binary(spec.c_str());
    in.edges = raw.first;
    in.n = raw.second;
  }
  if (!in.owned.empty()) in.edges = reinterpret_cast<std::pair<uint64_t, uint64_t> *>(in.owned.data());
  if (window) {   // edges [lo, hi) of the list only
    hi = std::min<unsigned long long>(hi, in.n);
    lo = std::min(lo, hi);
    in.edges += lo;
    in.n = hi - lo;
  }
  return in;
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
uint64_t adj_w(const E &e) { return (uint64_t)e.data; }
template <>
uint64_t adj_w<AdjEdge<void>>(const AdjEdge<void> &) { return 0; }

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
      uint64_t w = adj_w(e);
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
      uint64_t w = adj_w(e);
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
  uint64_t unreached() const { return algo == BFS ? BFS_MAXL : algo == SSSP ? SSSP_MAXL : 0; }
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
    pw[v] = adj_w(labels[v].parent);
  }
  out.write(".val", val);
  out.write(".par", par);
  out.write(".pw", pw);
}

template <typename L>
uint64_t checksum(const L &labels, uint64_t V, std::vector<uint64_t> &tmp) {
#pragma omp parallel for schedule(static)
  for (uint64_t v = 0; v < V; v++) tmp[v] = labels[v].data;
  return rg_gen_value_checksum(tmp.data(), V);
}

// Reached vertices (value differs from the unreached sentinel; every vertex for
// WCC) and the stored edges out of them: adjacency entries with multiplicity > 0
// (core/storage.hpp:345-398 keeps one entry per distinct (nbr, data)).
template <typename G, typename L>
std::pair<uint64_t, uint64_t> reached(G &graph, const L &labels, uint64_t V, const Hooks<G> &h) {
  uint64_t vr = 0, er = 0;
#pragma omp parallel for reduction(+ : vr, er) schedule(dynamic, 4096)
  for (uint64_t v = 0; v < V; v++) {
    if (h.algo != WCC && labels[v].data == h.unreached()) continue;
    vr++;
    auto range = graph.get_outgoing_adjlist_range(v);
    for (auto it = range.first; it != range.second; ++it)
      if (it->num) er++;
  }
  return {vr, er};
}

void json_times(const char *key, const std::vector<double> &t) {
  printf(", \"%s\": [", key);
  for (size_t i = 0; i < t.size(); i++) printf("%s%.9f", i ? ", " : "", t[i]);
  printf("]");
}

// One sliding-window batch of src/sssp_inc_batch.cpp:141-175: add the edges of
// `adds` and repair for those whose multiplicity went 0 -> 1, then delete the
// edges of `dels` and repair for those that went 1 -> 0.
template <typename G, typename L>
void apply_batch(G &graph, const Hooks<G> &h, L &labels, const std::pair<uint64_t, uint64_t> *adds, uint64_t na,
                 const std::pair<uint64_t, uint64_t> *dels, uint64_t nd, bool directed,
                 std::vector<typename G::edge_type> &buf, uint64_t &n_tree_add, uint64_t &n_tree_del) {
  if (buf.size() < std::max(na, nd)) buf.resize(std::max(na, nd));
  {
    std::atomic_uint64_t len(0);
#pragma omp parallel for if (na > 1024)
    for (uint64_t i = 0; i < na; i++) {
      auto e = make_edge<G>(adds[i].first, adds[i].second);
      if (graph.add_edge(e, directed) == 0) buf[len.fetch_add(1)] = e;
    }
    n_tree_add += len.load();
    graph.template update_tree_add<uint64_t, uint64_t>(h.continue_reduce(), h.update(), h.active_result(), labels, buf,
                                                       len.load(), directed);
  }
  {
    std::atomic_uint64_t len(0);
#pragma omp parallel for if (nd > 1024)
    for (uint64_t i = 0; i < nd; i++) {
      auto e = make_edge<G>(dels[i].first, dels[i].second);
      if (graph.del_edge(e, directed) == 1) buf[len.fetch_add(1)] = e;
    }
    n_tree_del += len.load();
    graph.template update_tree_del<uint64_t, uint64_t>(h.init(), h.continue_reduce(), h.update(), h.active_result(),
                                                       h.equal(), labels, buf, len.load(), directed);
  }
}

// The epoch loop of src/sssp_inc_rt.cpp:119-441, restated over this driver's
// hooks: in each epoch every thread serves its share of closed-loop clients,
// applying safe updates at once (need_update_tree_* false) and queueing unsafe
// ones, blocking their clients, until the oldest queued update has waited 80 %
// of the timeout or the queue passes the adaptive threshold; then the unsafe
// updates are applied one by one in arrival order, each with its tree repair
// and its history record (MVVec::set of every modified vertex).  Latency of an
// update = time from its client's previous completion to its own.  Inserts come
// from the edges after `imported`, deletes from the oldest loaded edges.
template <typename G, typename L>
void run_rt(G &graph, const Hooks<G> &h, L &labels, const std::pair<uint64_t, uint64_t> *edges, uint64_t E,
            uint64_t imported, uint64_t &add_base, uint64_t &del_base, uint64_t clients, uint32_t timeout_ms,
            uint64_t max_updates, bool directed,
            double target_timeout_rate, std::vector<uint64_t> &latency, double &seconds, uint64_t &n_updates,
            uint64_t &n_timeouts, uint64_t &epochs) {
  using hclk = std::chrono::steady_clock;
  using edge_t = typename G::edge_type;
  struct Pending {
    edge_t edge;
    hclk::time_point when;
    hclk::time_point *client_time;
  };
  const uint64_t T = (uint64_t)omp_get_max_threads();
  const uint64_t per_thread = (clients + T - 1) / T;
  std::vector<std::vector<hclk::time_point>> last_time(T);
  std::vector<std::vector<uint64_t>> blocked(T);
  std::vector<uint64_t> next_client(T, 0), n_clients(T, 0), add_next(T), del_next(T);
  std::vector<std::vector<uint64_t>> lat(T);
  auto t_begin = hclk::now();
  for (uint64_t t = 0; t < T; t++) {
    uint64_t lo = per_thread * t;
    n_clients[t] = lo < clients ? std::min(per_thread * (t + 1), clients) - lo : 0;
    last_time[t].assign(std::max<uint64_t>(n_clients[t], 1), t_begin);
    blocked[t].assign(std::max<uint64_t>(n_clients[t], 1), 0);
    add_next[t] = add_base + t;
    del_next[t] = del_base + t;
  }
  const uint64_t add_end = std::min(E, add_base + (max_updates + 1) / 2);
  const uint64_t del_end = std::min(imported, del_base + max_updates / 2);
  std::vector<Pending> adds, dels;
  std::mutex add_mu, del_mu;
  std::atomic<uint64_t> done(0), timeouts(0);
  uint64_t threshold = T, last_to = 0, last_up = 0;
  auto history = graph.template alloc_history_array<uint64_t>();
  uint64_t version = 0;
  const auto timeout = std::chrono::milliseconds(timeout_ms);
  epochs = 0;
  auto start = hclk::now();
  while (done.load() < max_updates) {
    epochs++;
    adds.clear();
    dels.clear();
    std::atomic<uint64_t> n_unsafe(0);
    std::atomic<int64_t> first_ns(INT64_MAX);
    std::atomic<uint64_t> progress(0);
#pragma omp parallel
    {
      const uint64_t t = (uint64_t)omp_get_thread_num();
      const uint64_t nc = n_clients[t];
      uint64_t left = nc, nc_i = next_client[t], local = 0;
      bool is_add = epochs & 1, add_out = false, del_out = false;
      while (nc && left && (!add_out || !del_out)) {
        is_add = !is_add;
        auto now = hclk::now();
        int64_t f = first_ns.load(std::memory_order_relaxed);
        if (n_unsafe.load(std::memory_order_relaxed) > threshold ||
            (f != INT64_MAX && now.time_since_epoch().count() - f > (int64_t)(0.8 * timeout_ms * 1e6)))
          break;
        do { nc_i = (nc_i + 1) % nc; } while (blocked[t][nc_i] == epochs);
        uint64_t i;
        if (is_add) {
          i = add_next[t];
          if (i >= add_end) { add_out = true; continue; }
          add_next[t] += T;
        } else {
          i = del_next[t];
          if (i >= del_end) { del_out = true; continue; }
          del_next[t] += T;
        }
        local++;
        auto e = make_edge<G>(edges[i].first, edges[i].second);
        bool unsafe = is_add ? graph.need_update_tree_add(h.update(), labels, e, directed)
                             : graph.need_update_tree_del(labels, e, directed);
        if (unsafe) {
          {
            std::lock_guard<std::mutex> lk(is_add ? add_mu : del_mu);
            (is_add ? adds : dels).push_back(Pending{e, now, &last_time[t][nc_i]});
          }
          int64_t expect = INT64_MAX;
          first_ns.compare_exchange_strong(expect, now.time_since_epoch().count());
          n_unsafe.fetch_add(1, std::memory_order_relaxed);
          blocked[t][nc_i] = epochs;
          left--;
        } else {
          if (is_add) graph.add_edge(e, directed);
          else graph.del_edge(e, directed);
          auto end = hclk::now();
          auto d = end - last_time[t][nc_i];
          lat[t].push_back((uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(d).count());
          if (d > timeout) timeouts.fetch_add(1, std::memory_order_relaxed);
          last_time[t][nc_i] = end;
        }
      }
      next_client[t] = nc_i;
      progress.fetch_add(local, std::memory_order_relaxed);
    }
    // unsafe updates one by one, in arrival order
    std::sort(adds.begin(), adds.end(), [](const Pending &a, const Pending &b) { return a.when < b.when; });
    std::sort(dels.begin(), dels.end(), [](const Pending &a, const Pending &b) { return a.when < b.when; });
    size_t ia = 0, id = 0;
    while (ia < adds.size() || id < dels.size()) {
      bool take_add = id >= dels.size() || (ia < adds.size() && adds[ia].when < dels[id].when);
      Pending &p = take_add ? adds[ia++] : dels[id++];
      version++;
      graph.clear_modified();
      if (take_add) {
        if (graph.add_edge(p.edge, directed) == 0)
          graph.template update_tree_add<uint64_t, uint64_t>(h.continue_reduce(), h.update(), h.active_result(),
                                                             labels, p.edge, directed);
      } else {
        if (graph.del_edge(p.edge, directed) == 1)
          graph.template update_tree_del<uint64_t, uint64_t>(h.init(), h.continue_reduce(), h.update(),
                                                             h.active_result(), h.equal(), labels, p.edge, directed);
      }
      graph.template stream_vertices_hybrid<uint64_t>(
          [&](uint64_t vid) {
            history.set(vid, version, labels[vid].data);
            return 0;
          },
          graph.get_modified());
      auto end = hclk::now();
      auto d = end - *p.client_time;
      lat[0].push_back((uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(d).count());
      if (d > timeout) timeouts.fetch_add(1, std::memory_order_relaxed);
      *p.client_time = end;
    }
    uint64_t got = progress.load();
    done.fetch_add(got);
    if (got == 0) break;   // every client's stream is exhausted
    // the adaptive threshold of src/sssp_inc_rt.cpp:394-412
    if (epochs % 3 == 0) {
      uint64_t gto = timeouts.load(), gup = done.load();
      uint64_t lto = gto - last_to, lup = gup - last_up;
      if (lup && (double)lto / lup > 0.8 * target_timeout_rate) threshold = std::max<uint64_t>(threshold * 9 / 10, T);
      if (lup && (double)lto / lup < 0.8 * target_timeout_rate && gup && (double)gto / gup < target_timeout_rate)
        threshold = std::min<uint64_t>(threshold < 1000 ? threshold + 10 : threshold * 101 / 100, 1000000);
      last_to = gto;
      last_up = gup;
    }
  }
  seconds = secs(start, hclk::now());
  for (uint64_t t = 0; t < T; t++) {   // the next run starts past every index taken
    add_base = std::max(add_base, std::min(add_next[t], add_end));
    del_base = std::max(del_base, std::min(del_next[t], del_end));
  }
  n_updates = done.load();
  n_timeouts = timeouts.load();
  for (auto &v : lat) latency.insert(latency.end(), v.begin(), v.end());
  __gnu_parallel::sort(latency.begin(), latency.end());
}

template <typename G>
int run(int argc, char **argv) {
  const char *mode = argv[1];
  Algo algo = parse_algo(argv[2]);
  Input in = load_input(argv[3]);
  std::pair<uint64_t, uint64_t> *edges = in.edges;
  uint64_t E = in.n;
  uint64_t V = std::stoull(argv[4]);
  if (V == 0) V = 1ull << in.scale;
  uint64_t root = 0;
  if (!strcmp(argv[5], "maxdeg")) root = rg_gen_max_out_degree_vertex(&edges[0].first, E, V);
  else root = std::stoull(argv[5]);
  bool symmetric = (algo == WCC), directed = (algo != WCC);
  bool inc_mode = strcmp(mode, "build") != 0;
  bool rt_mode = !strcmp(mode, "rt");
  // WCC incremental drivers construct (symmetric, !dual) (src/wcc_inc.cpp:56);
  // every other driver uses dual = true.  The _inc_rt drivers trace modified
  // vertices for the history (src/sssp_inc_rt.cpp:58).
  bool dual = !(algo == WCC && inc_mode);

  double rate = 1.0;
  uint64_t steps = 0, batch = 1, loaded = 0, max_updates = 0;
  uint32_t timeout_ms = 1;
  std::string prefix, spec, batchfile;
  uint64_t repeats = 1, warmup = 0;
  auto need = [&](int n) {
    if (argc < n) { fprintf(stderr, "%s: missing arguments\n", mode); exit(2); }
  };
  if (!strcmp(mode, "build")) {
    need(7);
    prefix = argv[6];
    if (argc > 8) { repeats = std::stoull(argv[7]); warmup = std::stoull(argv[8]); }
  } else if (!strcmp(mode, "inc")) {
    need(9);
    rate = std::stod(argv[6]); steps = std::stoull(argv[7]); prefix = argv[8];
  } else if (!strcmp(mode, "batch")) {
    need(10);
    rate = std::stod(argv[6]); batch = std::stoull(argv[7]); steps = std::stoull(argv[8]); prefix = argv[9];
  } else if (!strcmp(mode, "sweep")) {
    need(9);
    rate = std::stod(argv[6]); spec = argv[7]; prefix = argv[8];
  } else if (!strcmp(mode, "replay")) {
    need(9);
    loaded = std::stoull(argv[6]); batchfile = argv[7]; prefix = argv[8];
  } else if (rt_mode) {
    need(11);
    rate = std::stod(argv[6]); spec = argv[7]; timeout_ms = (uint32_t)std::stoul(argv[8]);
    max_updates = std::stoull(argv[9]); prefix = argv[10];
  } else {
    fprintf(stderr, "unknown mode %s\n", mode);
    return 2;
  }
  for (uint64_t i = 0; i < E; i++)
    if (edges[i].first >= V || edges[i].second >= V) { fprintf(stderr, "edge %lu out of range\n", i); return 4; }
  uint64_t imported = inc_mode ? (uint64_t)(E * rate) : E;   // src/sssp_inc.cpp:190-191
  if (!strcmp(mode, "replay")) imported = std::min(loaded, E);

  G graph(V, E, symmetric, dual, rt_mode);
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
  std::vector<double> times;
  uint64_t n_tree_add = 0, n_tree_del = 0;
  double upd = 0.0;
  std::vector<typename G::edge_type> buf;
  std::string extra;

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
      double dt = secs(u0, clk::now());
      upd += dt;
      times.push_back(dt);
      sums.push_back(checksum(labels, V, tmp));
    }
  } else if (!strcmp(mode, "batch") || !strcmp(mode, "sweep")) {
    std::vector<std::pair<uint64_t, uint64_t>> plan;   // (batch size, count)
    if (!strcmp(mode, "batch")) {
      plan.push_back({batch, steps});
    } else {
      const char *p = spec.c_str();
      while (*p) {
        unsigned long long b = 0, c = 0;
        int used = 0;
        if (sscanf(p, "%llux%llu%n", &b, &c, &used) != 2 || b == 0) { fprintf(stderr, "bad sweep spec\n"); return 2; }
        plan.push_back({b, c});
        p += used;
        if (*p == ',') p++;
      }
    }
    uint64_t b0 = imported;
    for (auto &pc : plan) {
      for (uint64_t k = 0; k < pc.second && b0 < E; k++) {
        uint64_t b1 = std::min(b0 + pc.first, E);
        auto u0 = clk::now();
        apply_batch(graph, h, labels, &edges[b0], b1 - b0, &edges[b0 - imported], b1 - b0, directed, buf, n_tree_add,
                    n_tree_del);
        double dt = secs(u0, clk::now());
        upd += dt;
        times.push_back(dt);
        sums.push_back(checksum(labels, V, tmp));
        b0 = b1;
      }
    }
  } else if (!strcmp(mode, "replay")) {
    FILE *f = fopen(batchfile.c_str(), "rb");
    if (!f) { perror(batchfile.c_str()); return 3; }
    std::vector<std::pair<uint64_t, uint64_t>> a, d;
    uint64_t hdr[2];
    while (fread(hdr, 8, 2, f) == 2) {
      a.resize(hdr[0]);
      d.resize(hdr[1]);
      if (fread(a.data(), 16, hdr[0], f) != hdr[0] || fread(d.data(), 16, hdr[1], f) != hdr[1]) {
        fprintf(stderr, "truncated batch file\n");
        return 3;
      }
      for (auto &e : a) if (e.first >= V || e.second >= V) { fprintf(stderr, "replay edge out of range\n"); return 4; }
      for (auto &e : d) if (e.first >= V || e.second >= V) { fprintf(stderr, "replay edge out of range\n"); return 4; }
      auto u0 = clk::now();
      apply_batch(graph, h, labels, a.data(), a.size(), d.data(), d.size(), directed, buf, n_tree_add, n_tree_del);
      double dt = secs(u0, clk::now());
      upd += dt;
      times.push_back(dt);
      sums.push_back(checksum(labels, V, tmp));
    }
    fclose(f);
  } else if (rt_mode) {
    // one run per client count, back to back; each continues the window where
    // the previous one stopped
    extra = ", \"runs\": [";
    uint64_t add_base = imported, del_base = 0;
    const char *p = spec.c_str();
    for (int k = 0; *p; k++) {
      unsigned long long c = 0;
      int used = 0;
      if (sscanf(p, "%llu%n", &c, &used) != 1 || c == 0) { fprintf(stderr, "bad client list\n"); return 2; }
      p += used;
      if (*p == ',') p++;
      std::vector<uint64_t> lat;
      double s = 0;
      uint64_t nu = 0, nto = 0, ep = 0;
      run_rt(graph, h, labels, edges, E, imported, add_base, del_base, c, timeout_ms, max_updates, directed, 0.001,
             lat, s, nu, nto, ep);
      upd += s;
      auto pct = [&](double q) {
        return lat.empty() ? 0.0 : 1e-3 * lat[std::min(lat.size() - 1, (size_t)(lat.size() * q))];
      };
      char b[512];
      snprintf(b, sizeof(b),
               "%s{\"clients\": %llu, \"updates\": %lu, \"timeouts\": %lu, \"epochs\": %lu, "
               "\"updates_per_s\": %.3f, \"p50_us\": %.3f, \"p99_us\": %.3f, \"p999_us\": %.3f, \"max_us\": %.3f}",
               k ? ", " : "", c, nu, nto, ep, s > 0 ? nu / s : 0.0, pct(0.5), pct(0.99), pct(0.999),
               lat.empty() ? 0.0 : 1e-3 * lat.back());
      extra += b;
    }
    extra += "]";
  }

  dump_labels<G>(out, labels, V);
  if (inc_mode) out.write(".sums", sums);
  double bsum = 0;
  for (double t : build_times) bsum += t;
  printf("{\"mode\": \"%s\", \"algo\": \"%s\", \"V\": %lu, \"E\": %lu, \"imported\": %lu, \"root\": %lu, "
         "\"threads\": %d, \"load_s\": %.6f, \"build_s\": %.6f, \"build_times\": [",
         mode, argv[2], V, E, imported, root, omp_get_max_threads(), secs(t0, t1),
         build_times.empty() ? 0.0 : bsum / build_times.size());
  for (size_t i = 0; i < build_times.size(); i++) printf("%s%.6f", i ? ", " : "", build_times[i]);
  printf("]");
  if (!inc_mode) {
    auto r = reached(graph, labels, V, h);
    printf(", \"V_r\": %lu, \"E_r\": %lu", r.first, r.second);
  } else if (!rt_mode) {
    json_times("times", times);
  }
  printf("%s, \"update_s\": %.6f, \"steps\": %lu, \"tree_add\": %lu, \"tree_del\": %lu, \"checksum\": %lu}\n",
         extra.c_str(), upd, (uint64_t)sums.size(), n_tree_add, n_tree_del, checksum(labels, V, tmp));
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 7) {
    fprintf(stderr, "usage: ref_driver build|inc|batch|sweep|replay|rt algo graph V root ...\n");
    return 2;
  }
  Algo a = parse_algo(argv[2]);
  if (a == BFS || a == WCC) return run<Graph<void>>(argc, argv);
  return run<Graph<uint64_t>>(argc, argv);
}
