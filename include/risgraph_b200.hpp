// risgraph_b200.hpp: C++ facade over the C ABI of risgraph_b200.h with the
// method names and argument meaning of the reference's
// template<EdgeData> class Graph (core/graph.hpp:41-1908), so that a driver
// written against the reference reads the same:
//
//   rg::Graph<uint64_t> graph(num_vertices, raw_edges_len, false, true);
//   graph.add_edge({src, dst, w}, true);
//   auto labels = graph.alloc_vertex_tree_array<uint64_t>();
//   graph.build_tree(rg::SSSP{root}, labels);
//   if (!graph.add_edge(e, true)) graph.update_tree_add(rg::SSSP{root}, labels, e, true);
//
// The reference takes the per-algorithm semantics as lambdas (update_func,
// init_label_func, ...); a C ABI cannot, so the four hook sets of its drivers
// (src/bfs.cpp:76-91, src/sssp.cpp:67-91, src/sswp.cpp:76-91, src/wcc.cpp:62-86)
// are the tag types BFS, SSSP, SSWP and WCC below.  Labels live on the GPU;
// VertexTreeArray is the host view, read back lazily the first time an entry
// is read after a tree call.  Errors throw std::runtime_error with the
// reference's messages ("VertexId error.", core/graph.hpp:205,231).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "risgraph_b200.h"

namespace rg {

inline void check(int status) {
  if (status != RG_OK) {
    const char *msg = rg_last_error();
    throw std::runtime_error(msg && *msg ? msg : rg_status_string(status));
  }
}

// Hook sets (init_label_func / update_func / equal_func of the drivers).
struct BFS {
  uint64_t root;
  static constexpr int algo = RG_BFS;
  static constexpr uint64_t MAXL = 65536;  // src/bfs.cpp:66
};
struct SSSP {
  uint64_t root;
  static constexpr int algo = RG_SSSP;
  static constexpr uint64_t MAXL = 134217728;  // src/sssp.cpp:66
};
struct SSWP {
  uint64_t root;
  static constexpr int algo = RG_SSWP;
  static constexpr uint64_t MAXL = 134217728;  // root value; others start at 0 (src/sswp.cpp)
};
struct WCC {
  uint64_t root = 0;  // unused: every vertex starts with its own id
  static constexpr int algo = RG_WCC;
  static constexpr uint64_t MAXL = ~0ull;
};

// Edge<EdgeData> / AdjEdge<EdgeData> (core/type.hpp:21-81).  EdgeData = void
// is the unweighted graph.
template <typename D>
struct Edge {
  uint64_t src, dst;
  D data;
};
template <>
struct Edge<void> {
  uint64_t src, dst;
};
template <typename D>
struct AdjEdge {
  uint64_t nbr;
  D data;
};
template <>
struct AdjEdge<void> {
  uint64_t nbr;
};

// VertexTree<EdgeData, DataType> (core/graph.hpp:54-59).
template <typename D, typename T>
struct VertexTree {
  AdjEdge<D> parent;
  T data;
};

template <typename D>
class Graph;

// Host view of the device label array.
template <typename D, typename T>
class VertexTreeArray {
 public:
  const VertexTree<D, T> &operator[](uint64_t v) const {
    sync();
    return host_[v];
  }
  uint64_t size() const { return host_.size(); }
  void invalidate() { stale_ = true; }
  // force the read-back now (e.g. before timing stops)
  void sync() const {
    if (!stale_) return;
    std::vector<uint64_t> val(host_.size()), par(host_.size()), pw(host_.size());
    check(rg_get_labels(g_, val.data(), par.data(), pw.data()));
    for (uint64_t v = 0; v < host_.size(); v++) {
      host_[v].data = (T)val[v];
      host_[v].parent.nbr = par[v];
      set_w(host_[v].parent, pw[v]);
    }
    stale_ = false;
  }

 private:
  friend class Graph<D>;
  template <typename E>
  static void set_w(AdjEdge<E> &a, uint64_t w) { a.data = (E)w; }
  static void set_w(AdjEdge<void> &, uint64_t) {}
  VertexTreeArray(rg_graph *g, uint64_t n) : g_(g), host_(n) {}
  rg_graph *g_;
  mutable std::vector<VertexTree<D, T>> host_;
  mutable bool stale_ = true;
};

template <typename D>
class Graph {
 public:
  using edge_type = Edge<D>;
  using adjedge_type = AdjEdge<D>;
  static constexpr bool weighted = !std::is_void<D>::value;

  // Graph(vertices, hint_edges, symmetric, dual, trace_modified) (core/graph.hpp:61-100)
  Graph(uint64_t vertices, uint64_t hint_edges = 0, bool symmetric = false, bool dual = true,
        bool trace_modified = false)
      : V_(vertices) {
    check(rg_create(vertices, hint_edges, symmetric, dual, trace_modified, weighted ? 1 : 0, &g_));
  }
  ~Graph() {
    if (g_) rg_destroy(g_);
  }
  Graph(const Graph &) = delete;
  Graph &operator=(const Graph &) = delete;

  uint64_t get_num_vertices() const { return V_; }
  rg_graph *handle() const { return g_; }

  // add_edge / del_edge (core/graph.hpp:203-253): returns the old multiplicity.
  uint64_t add_edge(const edge_type &e, bool directed) { return edge_op(&e, 1, directed, true); }
  uint64_t del_edge(const edge_type &e, bool directed) { return edge_op(&e, 1, directed, false); }
  // batched forms: old[i] for edge i
  void add_edges(const edge_type *e, uint64_t n, bool directed, uint64_t *old = nullptr) {
    edge_ops(e, n, directed, true, old);
  }
  void del_edges(const edge_type *e, uint64_t n, bool directed, uint64_t *old = nullptr) {
    edge_ops(e, n, directed, false, old);
  }
  // reference binary-format pairs (core/io.hpp:26-36), weights by rg_gen_weight
  void add_pairs(const uint64_t *pairs, uint64_t n, bool directed) { check(rg_add_pairs(g_, pairs, n, directed, nullptr)); }

  uint64_t get_edge_num(const edge_type &e) {
    rg_edge x = to_c(e);
    uint64_t num = 0;
    check(rg_get_edge_num(g_, &x, 1, &num));
    return num;
  }

  template <typename T>
  VertexTreeArray<D, T> alloc_vertex_tree_array() {
    return VertexTreeArray<D, T>(g_, V_);
  }

  // build_tree (core/graph.hpp:873-985); returns the number of label updates.
  template <typename H, typename T>
  uint64_t build_tree(const H &hooks, VertexTreeArray<D, T> &labels) {
    uint64_t total = 0;
    check(rg_build_tree(g_, H::algo, hooks.root, &total));
    labels.invalidate();
    return total;
  }

  // update_tree_add single (:1124-1160) and batch (:1162-1218)
  template <typename H, typename T>
  uint64_t update_tree_add(const H &hooks, VertexTreeArray<D, T> &labels, const edge_type &e, bool directed) {
    return update_tree_add(hooks, labels, &e, 1, directed);
  }
  template <typename H, typename T>
  uint64_t update_tree_add(const H &, VertexTreeArray<D, T> &labels, const edge_type *e, uint64_t n, bool directed) {
    std::vector<rg_edge> x = to_c(e, n);
    uint64_t total = 0;
    check(rg_update_tree_add(g_, H::algo, x.data(), n, directed, &total));
    labels.invalidate();
    return total;
  }
  // update_tree_del single (:1622-1656) and batch (:1658-1718)
  template <typename H, typename T>
  uint64_t update_tree_del(const H &hooks, VertexTreeArray<D, T> &labels, const edge_type &e, bool directed) {
    return update_tree_del(hooks, labels, &e, 1, directed);
  }
  template <typename H, typename T>
  uint64_t update_tree_del(const H &, VertexTreeArray<D, T> &labels, const edge_type *e, uint64_t n, bool directed) {
    std::vector<rg_edge> x = to_c(e, n);
    uint64_t total = 0;
    check(rg_update_tree_del(g_, H::algo, x.data(), n, directed, &total));
    labels.invalidate();
    return total;
  }

  // need_update_tree_add (:987-1000) / need_update_tree_del (:1220-1233)
  template <typename H, typename T>
  bool need_update_tree_add(const H &, const VertexTreeArray<D, T> &, const edge_type &e, bool directed) {
    return classify(H::algo, e, false, directed);
  }
  template <typename H, typename T>
  bool need_update_tree_del(const H &, const VertexTreeArray<D, T> &, const edge_type &e, bool directed) {
    return classify(H::algo, e, true, directed);
  }

  // add_edge + update_tree_add of the 0->1 transitions, fused on the device
  // (the step of src/sssp_inc_batch.cpp:141-157); likewise for deletes.
  template <typename H, typename T>
  void apply_add(const H &, VertexTreeArray<D, T> &labels, const edge_type *e, uint64_t n, bool directed) {
    std::vector<rg_edge> x = to_c(e, n);
    check(rg_apply_add(g_, H::algo, x.data(), n, directed, nullptr));
    labels.invalidate();
  }
  template <typename H, typename T>
  void apply_del(const H &, VertexTreeArray<D, T> &labels, const edge_type *e, uint64_t n, bool directed) {
    std::vector<rg_edge> x = to_c(e, n);
    check(rg_apply_del(g_, H::algo, x.data(), n, directed, nullptr));
    labels.invalidate();
  }

  // get_modified / clear_modified (core/graph.hpp:117-130)
  std::vector<uint64_t> get_modified() {
    std::vector<uint64_t> out(V_);
    uint64_t n = 0;
    check(rg_get_modified(g_, out.data(), V_, &n));
    out.resize(n);
    return out;
  }
  void clear_modified() { check(rg_clear_modified(g_)); }

  // get_outgoing_degree / get_incoming_degree for all vertices at once
  void get_degrees(std::vector<uint64_t> &out, std::vector<uint64_t> &in) {
    out.resize(V_);
    in.resize(V_);
    check(rg_get_degrees(g_, out.data(), in.data()));
  }

 private:
  static rg_edge to_c(const edge_type &e) {
    rg_edge x{e.src, e.dst, 0};
    if constexpr (weighted) x.data = (uint64_t)e.data;
    return x;
  }
  static std::vector<rg_edge> to_c(const edge_type *e, uint64_t n) {
    std::vector<rg_edge> x(n);
    for (uint64_t i = 0; i < n; i++) x[i] = to_c(e[i]);
    return x;
  }
  uint64_t edge_op(const edge_type *e, uint64_t n, bool directed, bool add) {
    uint64_t old = 0;
    edge_ops(e, n, directed, add, &old);
    return old;
  }
  void edge_ops(const edge_type *e, uint64_t n, bool directed, bool add, uint64_t *old) {
    std::vector<rg_edge> x = to_c(e, n);
    check(add ? rg_add_edges(g_, x.data(), n, directed, old) : rg_del_edges(g_, x.data(), n, directed, old));
  }
  bool classify(int algo, const edge_type &e, bool del, bool directed) {
    rg_edge x = to_c(e);
    uint8_t is_del = del ? 1 : 0, unsafe = 0;
    check(rg_classify(g_, algo, &x, &is_del, 1, directed, &unsafe));
    return unsafe != 0;
  }
  rg_graph *g_ = nullptr;
  uint64_t V_;
};

}  // namespace rg
