// C-ABI entry points of librisgraph_b200 (declared in include/risgraph_b200.h).
// Argument checking happens here, on the host, before any device work, so
// malformed input returns a status and never reaches a kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>

#include "rg_internal.cuh"

namespace rg {

static thread_local std::string tl_err;

void set_error(const std::string &msg) { tl_err = msg; }

int cuda_fail(cudaError_t e, const char *what) {
  tl_err = std::string(what) + ": " + cudaGetErrorString(e);
  return RG_ECUDA;
}

}  // namespace rg

namespace {

using rg::Graph;

constexpr uint64_t CHUNK_EDGES = 1ull << 24;

int check_graph(rg_graph *g) {
  if (!g) {
    rg::set_error("null graph");
    return RG_EINVAL;
  }
  cudaError_t e = cudaSetDevice(g->g.device);
  if (e != cudaSuccess) return rg::cuda_fail(e, "cudaSetDevice");
  return RG_OK;
}

int check_edges(const Graph &g, const rg_edge *edges, const uint64_t *pairs, uint64_t n) {
  if (n && !edges && !pairs) {
    rg::set_error("null edge array");
    return RG_EINVAL;
  }
  for (uint64_t i = 0; i < n; i++) {
    uint64_t s = pairs ? pairs[2 * i] : edges[i].src, d = pairs ? pairs[2 * i + 1] : edges[i].dst;
    if (s >= g.V || d >= g.V) {
      rg::set_error("VertexId error.");  // core/graph.hpp:205,231
      return RG_EINVAL_VID;
    }
    if (!pairs && g.weighted && edges[i].data >= rg::W_LIMIT) {
      rg::set_error("edge weight >= 2^64 - 2^27 (the reference's u64 sums would wrap)");
      return RG_EINVAL_WEIGHT;
    }
  }
  return RG_OK;
}

// The edges as the device takes them: weights above W_RAW_MAX replaced by
// their codes (assigned on first sight), in `buf`; the input itself when no
// weight needs a code (the common case costs one scan).
int device_edges(Graph &g, const rg_edge *edges, uint64_t n, std::vector<rg_edge> &buf, const rg_edge **out) {
  *out = edges;
  if (!g.weighted || !edges) return RG_OK;
  uint64_t i = 0;
  while (i < n && edges[i].data <= rg::W_RAW_MAX) i++;
  if (i == n) return RG_OK;
  buf.assign(edges, edges + n);
  std::lock_guard<std::mutex> lk(g.wmu);
  for (; i < n; i++) {
    uint64_t w = buf[i].data;
    if (w <= rg::W_RAW_MAX) continue;
    auto it = g.wcode.find(w);
    if (it == g.wcode.end()) {
      if (rg::W_CODE_BASE + g.wfull.size() >= rg::W_CODE_END) {
        rg::set_error("more than 2^31 - 2^27 distinct edge weights above 2^27");
        return RG_ENOSPACE;
      }
      it = g.wcode.emplace(w, (uint32_t)(rg::W_CODE_BASE + g.wfull.size())).first;
      g.wfull.push_back(w);
    }
    buf[i].data = it->second;
  }
  *out = buf.data();
  return RG_OK;
}

// Parent weights read back: codes to full weights.
void host_weights(Graph &g, uint64_t *w, uint64_t n) {
  std::lock_guard<std::mutex> lk(g.wmu);
  if (g.wfull.empty()) return;
  for (uint64_t i = 0; i < n; i++)
    if (w[i] >= rg::W_CODE_BASE && w[i] - rg::W_CODE_BASE < g.wfull.size()) w[i] = g.wfull[w[i] - rg::W_CODE_BASE];
}

int check_algo(const Graph &g, int algo) {
  if (algo < RG_BFS || algo > RG_WCC) {
    rg::set_error("unknown algorithm");
    return RG_EINVAL;
  }
  if (g.algo != algo) {
    rg::set_error("labels were not built for this algorithm (call rg_build_tree first)");
    return RG_ESTATE;
  }
  return RG_OK;
}

// add/del over edges or pairs, chunked; tree repair of each chunk's candidates
// when `apply` (the final values are the unique fixpoint either way).
int edge_updates(rg_graph *gh, const rg_edge *edges, const uint64_t *pairs, uint64_t n, int directed,
                 uint64_t *old_num, bool add, bool apply) {
  Graph &g = gh->g;
  int rc = check_edges(g, edges, pairs, n);
  if (rc) return rc;
  std::vector<rg_edge> wbuf;
  if ((rc = device_edges(g, edges, n, wbuf, &edges))) return rc;
  // small batches (single updates, served epochs): one fused graph launch
  if (apply && n && n <= g.fused_max && !g.profiling) return rg::apply_small(g, edges, pairs, n, directed, add, old_num);
  const int what = add ? 1 : 2;
  for (uint64_t b = 0; b < n; b += CHUNK_EDGES) {
    uint64_t m = std::min(CHUNK_EDGES, n - b), nops = 0;
    rc = rg::stage_edges(g, edges ? edges + b : nullptr, pairs ? pairs + 2 * b : nullptr, m, directed, &nops);
    if (rc) return rc;
    // storage update, candidate list and tree repair in one submission
    rc = rg::storage_enqueue(g, add, m, nops, directed, apply);
    if (!rc && apply) rc = rg::tree_enqueue(g, what, m, directed, true);
    if (!rc && old_num) rc = rg::storage_copy_old(g, m);
    if (!rc) rc = rg::sync_ctl(g);
    if (rc) return rc;
    if (add && g.h_ctl[rg::C_ERR] == RG_ENOSPACE && g.h_ctl[rg::C_AUX] == 1) {
      // growth ran out of pool: compact, then replay from the growth step
      rc = rg::storage_recover(g);
      if (!rc) rc = rg::storage_replay(g, m, nops, directed, apply);
      if (!rc && apply) rc = rg::tree_enqueue(g, what, m, directed, true);
      if (!rc && old_num) rc = rg::storage_copy_old(g, m);
      if (!rc) rc = rg::sync_ctl(g);
      if (rc) return rc;
    }
    if ((rc = rg::storage_error(g))) return rc;
    if (apply && (rc = rg::tree_after_sync(g, what, nullptr))) return rc;
    if (old_num) std::memcpy(old_num + b, rg::storage_old_host(g), m * 8);
  }
  return RG_OK;
}

int tree_updates(rg_graph *gh, int algo, const rg_edge *edges, uint64_t n, int directed, uint64_t *total, bool add) {
  Graph &g = gh->g;
  int rc = check_algo(g, algo);
  if (rc) return rc;
  if ((rc = check_edges(g, edges, nullptr, n))) return rc;
  std::vector<rg_edge> wbuf;
  if ((rc = device_edges(g, edges, n, wbuf, &edges))) return rc;
  uint64_t sum = 0;
  for (uint64_t b = 0; b < n; b += CHUNK_EDGES) {
    uint64_t m = std::min(CHUNK_EDGES, n - b), nops = 0, t = 0;
    if ((rc = rg::stage_edges(g, edges + b, nullptr, m, directed, &nops))) return rc;
    rc = add ? rg::tree_add(g, m, directed, false, &t) : rg::tree_del(g, m, directed, false, &t);
    if (rc) return rc;
    sum += t;
  }
  if (total) *total = sum;
  return RG_OK;
}

}  // namespace

extern "C" {

const char *rg_status_string(int s) {
  switch (s) {
    case RG_OK: return "ok";
    case RG_EINVAL: return "invalid argument";
    case RG_EINVAL_VID: return "VertexId error.";
    case RG_EINVAL_WEIGHT: return "edge weight out of range";
    case RG_ENOMEM_HBM: return "device memory exhausted";
    case RG_ENOSPACE: return "edge pool or index full";
    case RG_ETIMEOUT: return "bounded device wait timed out";
    case RG_ECUDA: return "CUDA error";
    case RG_ESTATE: return "invalid state";
  }
  return "unknown status";
}

const char *rg_last_error(void) { return rg::tl_err.c_str(); }

int rg_create(uint64_t vertices, uint64_t hint_edges, int symmetric, int dual, int trace_modified, int weighted,
              rg_graph **out) {
  if (!out) {
    rg::set_error("null output pointer");
    return RG_EINVAL;
  }
  *out = nullptr;
  if (vertices == 0 || vertices >= (1ull << 31)) {
    rg::set_error("vertices must be in [1, 2^31)");
    return RG_EINVAL;
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    rg::set_error(std::string("no CUDA device: ") + cudaGetErrorString(e));
    return RG_ECUDA;
  }
  rg_graph *gh = new (std::nothrow) rg_graph();
  if (!gh) return RG_ENOMEM_HBM;
  Graph &g = gh->g;
  g.V = vertices;
  g.hint = hint_edges ? hint_edges : vertices * 16;  // core/graph.hpp:64
  g.symmetric = symmetric ? 1 : 0;
  g.dual = dual ? 1 : 0;
  g.trace = trace_modified ? 1 : 0;
  g.weighted = weighted ? 1 : 0;
  cudaGetDevice(&g.device);
  cudaDeviceGetAttribute(&g.num_sms, cudaDevAttrMultiProcessorCount, g.device);
  int rc = RG_OK;
  if ((e = cudaStreamCreateWithFlags(&g.own_stream, cudaStreamNonBlocking)) != cudaSuccess) rc = rg::cuda_fail(e, "stream");
  g.stream = g.own_stream;
  if (!rc && (e = cudaEventCreate(&g.pev[0])) != cudaSuccess) rc = rg::cuda_fail(e, "event");
  if (!rc && (e = cudaEventCreate(&g.pev[1])) != cudaSuccess) rc = rg::cuda_fail(e, "event");
  if (!rc && (e = cudaHostAlloc(&g.h_ctl, sizeof(unsigned long long) * rg::C_COUNT, cudaHostAllocMapped)) != cudaSuccess)
    rc = rg::cuda_fail(e, "cudaHostAlloc(ctl)");
  if (!rc && (e = cudaHostGetDevicePointer(&g.h_ctl_dev, g.h_ctl, 0)) != cudaSuccess)
    rc = rg::cuda_fail(e, "cudaHostGetDevicePointer(ctl)");
  if (!rc) rc = rg::storage_alloc(g);
  if (!rc) rc = rg::tree_alloc(g);
  if (rc) {
    rg_destroy(gh);
    return rc;
  }
  *out = gh;
  return RG_OK;
}

int rg_destroy(rg_graph *gh) {
  if (!gh) return RG_EINVAL;
  Graph &g = gh->g;
  cudaSetDevice(g.device);
  if (g.stream) cudaStreamSynchronize(g.stream);
  rg::storage_free(g);
  rg::history_free(g);
  cudaFree(g.d.lab); cudaFree(g.d.val32); cudaFree(g.d.stamp); cudaFree(g.d.inv); cudaFree(g.d.chk); cudaFree(g.d.heavy); cudaFree(g.d.modstamp); cudaFree(g.d.modq);
  cudaFree(g.q[0]); cudaFree(g.q[1]); cudaFree(g.tree); cudaFree(g.scratch64); cudaFree(g.hubq); cudaFree(g.d.ctl);
  cudaFree(g.lb_P); cudaFree(g.lb_tile); cudaFree(g.cub_tmp); cudaFree(g.act);
  cudaFree(g.sell_ent); cudaFree(g.sell_off); cudaFree(g.sell_row); cudaFree(g.sell_hub); cudaFree(g.sell_piece);
  cudaFree(g.sell_cnt); cudaFree(g.sell_hub_off); cudaFree(g.sell_piece_best); cudaFree(g.lb_sums);
  if (g.h_ctl) cudaFreeHost(g.h_ctl);
  if (g.pev[0]) cudaEventDestroy(g.pev[0]);
  if (g.pev[1]) cudaEventDestroy(g.pev[1]);
  for (auto &l : g.loops)
    if (l.exec) cudaGraphExecDestroy(l.exec);
  for (auto &l : g.dels)
    if (l.exec) cudaGraphExecDestroy(l.exec);
  for (auto &l : g.applies)
    if (l.exec) cudaGraphExecDestroy(l.exec);
  for (auto &l : g.mixes)
    if (l.exec) cudaGraphExecDestroy(l.exec);
  for (auto &l : g.rests)
    if (l.exec) cudaGraphExecDestroy(l.exec);
  if (g.cap_stream) cudaStreamDestroy(g.cap_stream);
  cudaFree(g.d.trace);
  cudaFree(g.ptrace_buf);
  if (g.own_stream) cudaStreamDestroy(g.own_stream);
  delete gh;
  return RG_OK;
}

int rg_add_edges(rg_graph *g, const rg_edge *edges, uint64_t n, int directed, uint64_t *old_num) {
  int rc = check_graph(g);
  return rc ? rc : edge_updates(g, edges, nullptr, n, directed, old_num, true, false);
}

int rg_del_edges(rg_graph *g, const rg_edge *edges, uint64_t n, int directed, uint64_t *old_num) {
  int rc = check_graph(g);
  return rc ? rc : edge_updates(g, edges, nullptr, n, directed, old_num, false, false);
}

int rg_add_pairs(rg_graph *g, const uint64_t *pairs, uint64_t n, int directed, uint64_t *old_num) {
  int rc = check_graph(g);
  return rc ? rc : edge_updates(g, nullptr, pairs, n, directed, old_num, true, false);
}

int rg_del_pairs(rg_graph *g, const uint64_t *pairs, uint64_t n, int directed, uint64_t *old_num) {
  int rc = check_graph(g);
  return rc ? rc : edge_updates(g, nullptr, pairs, n, directed, old_num, false, false);
}

int rg_apply_add(rg_graph *g, int algo, const rg_edge *edges, uint64_t n, int directed, uint64_t *old_num) {
  int rc = check_graph(g);
  if (!rc) rc = check_algo(g->g, algo);
  return rc ? rc : edge_updates(g, edges, nullptr, n, directed, old_num, true, true);
}

int rg_apply_del(rg_graph *g, int algo, const rg_edge *edges, uint64_t n, int directed, uint64_t *old_num) {
  int rc = check_graph(g);
  if (!rc) rc = check_algo(g->g, algo);
  return rc ? rc : edge_updates(g, edges, nullptr, n, directed, old_num, false, true);
}

int rg_apply_add_del(rg_graph *g, int algo, const rg_edge *adds, uint64_t n_add, const rg_edge *dels, uint64_t n_del,
                     int directed) {
  int rc = check_graph(g);
  if (!rc) rc = check_algo(g->g, algo);
  if (!rc) rc = check_edges(g->g, adds, nullptr, n_add);
  if (!rc) rc = check_edges(g->g, dels, nullptr, n_del);
  if (rc) return rc;
  if (n_add && n_del && n_add <= g->g.fused_max && n_del <= g->g.fused_max && !g->g.profiling) {
    std::vector<rg_edge> abuf, dbuf;
    const rg_edge *a = adds, *d = dels;
    if (!rc) rc = device_edges(g->g, adds, n_add, abuf, &a);
    if (!rc) rc = device_edges(g->g, dels, n_del, dbuf, &d);
    return rc ? rc : rg::apply_add_del_small(g->g, a, n_add, d, n_del, directed);
  }
  // (edge_updates codes the weights itself)
  rc = edge_updates(g, adds, nullptr, n_add, directed, nullptr, true, true);
  return rc ? rc : edge_updates(g, dels, nullptr, n_del, directed, nullptr, false, true);
}

int rg_apply_add_pairs(rg_graph *g, int algo, const uint64_t *pairs, uint64_t n, int directed, uint64_t *old_num) {
  int rc = check_graph(g);
  if (!rc) rc = check_algo(g->g, algo);
  return rc ? rc : edge_updates(g, nullptr, pairs, n, directed, old_num, true, true);
}

int rg_apply_del_pairs(rg_graph *g, int algo, const uint64_t *pairs, uint64_t n, int directed, uint64_t *old_num) {
  int rc = check_graph(g);
  if (!rc) rc = check_algo(g->g, algo);
  return rc ? rc : edge_updates(g, nullptr, pairs, n, directed, old_num, false, true);
}

int rg_get_edge_num(rg_graph *gh, const rg_edge *edges, uint64_t n, uint64_t *num) {
  int rc = check_graph(gh);
  if (rc) return rc;
  Graph &g = gh->g;
  if ((rc = check_edges(g, edges, nullptr, n))) return rc;
  if (!num) { rg::set_error("null output"); return RG_EINVAL; }
  std::vector<rg_edge> wbuf;
  if ((rc = device_edges(g, edges, n, wbuf, &edges))) return rc;
  for (uint64_t b = 0; b < n; b += CHUNK_EDGES) {
    uint64_t m = std::min(CHUNK_EDGES, n - b), nops = 0;
    if ((rc = rg::stage_edges(g, edges + b, nullptr, m, 1, &nops))) return rc;
    if ((rc = rg::storage_num(g, nops, num + b))) return rc;
  }
  return RG_OK;
}

int rg_get_degrees(rg_graph *gh, uint64_t *out_degree, uint64_t *in_degree) {
  int rc = check_graph(gh);
  if (rc) return rc;
  Graph &g = gh->g;
  if (out_degree) RG_CUDA(cudaMemcpyAsync(out_degree, g.d.out.deg, g.V * 8, cudaMemcpyDeviceToHost, g.stream));
  if (in_degree) RG_CUDA(cudaMemcpyAsync(in_degree, g.d.in.deg, g.V * 8, cudaMemcpyDeviceToHost, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  return RG_OK;
}

int rg_build_tree(rg_graph *gh, int algo, uint64_t root, uint64_t *total) {
  int rc = check_graph(gh);
  if (rc) return rc;
  Graph &g = gh->g;
  if (algo < RG_BFS || algo > RG_WCC) { rg::set_error("unknown algorithm"); return RG_EINVAL; }
  if (algo != RG_WCC && root >= g.V) { rg::set_error("VertexId error."); return RG_EINVAL_VID; }
  return rg::tree_build(g, algo, algo == RG_WCC ? 0 : root, total);
}

int rg_update_tree_add(rg_graph *g, int algo, const rg_edge *edges, uint64_t n, int directed, uint64_t *total) {
  int rc = check_graph(g);
  return rc ? rc : tree_updates(g, algo, edges, n, directed, total, true);
}

int rg_update_tree_del(rg_graph *g, int algo, const rg_edge *edges, uint64_t n, int directed, uint64_t *total) {
  int rc = check_graph(g);
  return rc ? rc : tree_updates(g, algo, edges, n, directed, total, false);
}

int rg_classify(rg_graph *gh, int algo, const rg_edge *edges, const uint8_t *is_del, uint64_t n, int directed,
                uint8_t *unsafe) {
  int rc = check_graph(gh);
  if (rc) return rc;
  Graph &g = gh->g;
  if ((rc = check_algo(g, algo))) return rc;
  if ((rc = check_edges(g, edges, nullptr, n))) return rc;
  if (!unsafe) { rg::set_error("null output"); return RG_EINVAL; }
  std::vector<rg_edge> wbuf;
  if ((rc = device_edges(g, edges, n, wbuf, &edges))) return rc;
  for (uint64_t b = 0; b < n; b += CHUNK_EDGES) {
    uint64_t m = std::min(CHUNK_EDGES, n - b), nops = 0;
    if ((rc = rg::stage_edges(g, edges + b, nullptr, m, directed, &nops))) return rc;
    // flags ride in the scratch area after the 16-byte-aligned label unpack space
    uint8_t *d_flags = reinterpret_cast<uint8_t *>(rg::op_cand(g));  // >= m bytes
    uint8_t *d_is_del = nullptr;
    if (is_del) {
      d_is_del = reinterpret_cast<uint8_t *>(g.scratch64);
      if (m > g.V * 8) { rg::set_error("classify batch larger than scratch"); return RG_EINVAL; }
      RG_CUDA(cudaMemcpyAsync(d_is_del, is_del + b, m, cudaMemcpyHostToDevice, g.stream));
    }
    if ((rc = rg::tree_classify(g, m, directed, d_is_del, d_flags))) return rc;
    RG_CUDA(cudaMemcpyAsync(unsafe + b, d_flags, m, cudaMemcpyDeviceToHost, g.stream));
    RG_CUDA(cudaStreamSynchronize(g.stream));
  }
  return RG_OK;
}

int rg_get_labels(rg_graph *gh, uint64_t *value, uint64_t *parent, uint64_t *parent_w) {
  int rc = check_graph(gh);
  if (!rc) rc = rg::tree_labels(gh->g, value, parent, parent_w);
  if (!rc && parent_w && gh->g.weighted) host_weights(gh->g, parent_w, gh->g.V);
  return rc;
}

int rg_get_modified(rg_graph *gh, uint64_t *vids, uint64_t cap, uint64_t *n) {
  int rc = check_graph(gh);
  if (rc) return rc;
  Graph &g = gh->g;
  if (!g.trace) { rg::set_error("graph was created without trace_modified"); return RG_ESTATE; }
  RG_CUDA(cudaMemcpyAsync(g.h_ctl, g.d.ctl, sizeof(unsigned long long) * rg::C_COUNT, cudaMemcpyDeviceToHost, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  uint64_t m = g.h_ctl[rg::C_MODN];
  if (n) *n = m;
  uint64_t k = std::min(m, cap);
  if (vids && k) {
    uint32_t *tmp = new (std::nothrow) uint32_t[k];
    if (!tmp) return RG_EINVAL;
    cudaError_t e = cudaMemcpy(tmp, g.d.modq, k * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { delete[] tmp; return rg::cuda_fail(e, "copy modified"); }
    for (uint64_t i = 0; i < k; i++) vids[i] = tmp[i];
    delete[] tmp;
  }
  return RG_OK;
}

int rg_clear_modified(rg_graph *gh) {
  int rc = check_graph(gh);
  if (rc) return rc;
  Graph &g = gh->g;
  if (++g.mod_epoch == 0xFFFFFFFFu) {
    RG_CUDA(cudaMemsetAsync(g.d.modstamp, 0, g.V * 4, g.stream));
    g.mod_epoch = 1;
  }
  RG_CUDA(cudaMemsetAsync(&g.d.ctl[rg::C_MODN], 0, 8, g.stream));
  unsigned long long ep = g.mod_epoch;
  RG_CUDA(cudaMemcpyAsync(&g.d.ctl[rg::C_MODEPOCH], &ep, 8, cudaMemcpyHostToDevice, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  return RG_OK;
}

int rg_history_enable(rg_graph *gh, uint64_t capacity_nodes) {
  int rc = check_graph(gh);
  return rc ? rc : rg::history_enable(gh->g, capacity_nodes);
}

int rg_history_record(rg_graph *gh, uint64_t version, int all_vertices) {
  int rc = check_graph(gh);
  if (!rc) rc = rg::history_record(gh->g, version, all_vertices);
  if (!rc) rc = rg_clear_modified(gh);
  return rc;
}

int rg_history_get(rg_graph *gh, const uint64_t *vids, uint64_t n, uint64_t version, uint64_t *values,
                   uint8_t *found) {
  int rc = check_graph(gh);
  if (rc) return rc;
  if (n && (!vids || !values)) {
    rg::set_error("null array");
    return RG_EINVAL;
  }
  return rg::history_get(gh->g, vids, n, version, values, found);
}

int rg_history_gc(rg_graph *gh, uint64_t version) {
  int rc = check_graph(gh);
  return rc ? rc : rg::history_gc(gh->g, version);
}

int rg_history_nodes(rg_graph *gh, uint64_t *used, uint64_t *capacity) {
  if (!gh) return RG_EINVAL;
  if (used) *used = gh->g.hist_used;
  if (capacity) *capacity = gh->g.hist_cap;
  return RG_OK;
}

int rg_value_checksum(rg_graph *gh, uint64_t *checksum) {
  int rc = check_graph(gh);
  if (rc) return rc;
  if (!checksum) { rg::set_error("null output"); return RG_EINVAL; }
  return rg::tree_checksum(gh->g, checksum);
}

int rg_last_stats(rg_graph *gh, uint64_t *levels, uint64_t *invalidated, uint64_t *recomputes) {
  if (!gh) return RG_EINVAL;
  if (levels) *levels = gh->g.st_levels;
  if (invalidated) *invalidated = gh->g.st_invalidated;
  if (recomputes) *recomputes = gh->g.st_recomputes;
  return RG_OK;
}

int rg_set_stream(rg_graph *gh, void *cuda_stream) {
  int rc = check_graph(gh);
  if (rc) return rc;
  Graph &g = gh->g;
  RG_CUDA(cudaStreamSynchronize(g.stream));
  g.stream = cuda_stream ? (cudaStream_t)cuda_stream : g.own_stream;
  return RG_OK;
}

int rg_get_stream(rg_graph *gh, void **cuda_stream) {
  if (!gh || !cuda_stream) return RG_EINVAL;
  *cuda_stream = (void *)gh->g.stream;
  return RG_OK;
}

int rg_launch_count(rg_graph *gh, uint64_t *launches) {
  if (!gh || !launches) return RG_EINVAL;
  *launches = gh->g.launches;
  return RG_OK;
}

int rg_profile(rg_graph *gh, int enable) {
  if (!gh) return RG_EINVAL;
  gh->g.profiling = enable ? 1 : 0;
  return RG_OK;
}

int rg_profile_read(rg_graph *gh, uint64_t *launches, double *ms) {
  if (!gh) return RG_EINVAL;
  if (launches) *launches = gh->g.prof_launches;
  if (ms) *ms = gh->g.prof_ms;
  gh->g.prof_launches = 0;
  gh->g.prof_ms = 0.0;
  return RG_OK;
}

int rg_level_trace(rg_graph *gh, uint64_t *sizes, uint64_t cap, uint64_t *levels, uint64_t *edges_scanned) {
  int rc = check_graph(gh);
  if (rc) return rc;
  Graph &g = gh->g;
  RG_CUDA(cudaMemcpyAsync(g.h_ctl, g.d.ctl, sizeof(unsigned long long) * rg::C_COUNT, cudaMemcpyDeviceToHost, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  uint64_t n = std::min<uint64_t>(g.h_ctl[rg::C_LEVEL], rg::TRACE_CAP);
  if (levels) *levels = n;
  if (edges_scanned) *edges_scanned = g.h_ctl[rg::C_EDGES];
  if (sizes && cap && n) {
    uint64_t k = std::min(cap, n);
    RG_CUDA(cudaMemcpy(sizes, g.d.trace, k * 8, cudaMemcpyDeviceToHost));
  }
  return RG_OK;
}

int rg_level_stamps(rg_graph *gh, uint64_t *ns, uint64_t cap, uint64_t *levels) {
  int rc = check_graph(gh);
  if (rc) return rc;
  Graph &g = gh->g;
  RG_CUDA(cudaMemcpyAsync(g.h_ctl, g.d.ctl, sizeof(unsigned long long) * rg::C_COUNT, cudaMemcpyDeviceToHost, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  uint64_t n = std::min<uint64_t>(g.h_ctl[rg::C_LEVEL], rg::TRACE_CAP);
  if (levels) *levels = n;
  if (ns && cap) {
    uint64_t k = std::min(cap, n + 1);
    RG_CUDA(cudaMemcpy(ns, g.d.trace + rg::TRACE_CAP, k * 8, cudaMemcpyDeviceToHost));
  }
  return RG_OK;
}

int rg_phase_trace(rg_graph *gh, uint64_t *ns) {
  if (!gh || !ns) return RG_EINVAL;
  Graph &g = gh->g;
  if (!g.ptrace_buf) {
    std::memset(ns, 0, RG_PHASE_SLOTS * 8);
    return RG_OK;
  }
  RG_CUDA(cudaMemcpy(ns, g.ptrace_buf, RG_PHASE_SLOTS * 8, cudaMemcpyDeviceToHost));
  return RG_OK;
}

int rg_level_times(rg_graph *gh, double *ms, uint64_t cap, uint64_t *levels) {
  if (!gh) return RG_EINVAL;
  Graph &g = gh->g;
  if (levels) *levels = g.st_level_ms.size();
  for (uint64_t i = 0; ms && i < cap && i < g.st_level_ms.size(); i++) ms[i] = g.st_level_ms[i];
  return RG_OK;
}

int rg_set_option(rg_graph *gh, int option, uint64_t value) {
  if (!gh) return RG_EINVAL;
  Graph &g = gh->g;
  switch (option) {
    case RG_OPT_DENSE_PULL:
      if (value > 2) return RG_EINVAL;
      g.dense_pull = (int)value;
      return RG_OK;
    case RG_OPT_DENSE_DIV: g.dense_div = value ? value : 1; return RG_OK;
    case RG_OPT_LBS_MIN: g.lbs_min = value; return RG_OK;
    case RG_OPT_BFS_BOTTOM_UP: g.bfs_bottom_up = value ? 1 : 0; return RG_OK;
    case RG_OPT_RECOMPUTE_MIN: g.recompute_min = value; return RG_OK;
    case RG_OPT_BFS_BU_DIV: g.bu_div = value ? value : 1; return RG_OK;
    case RG_OPT_PULL_DIV: g.pull_div = value ? value : 1; return RG_OK;
    case RG_OPT_TINY_EDGES: g.tiny_edges = value; return RG_OK;
    case RG_OPT_PULL_SPLIT:
      if (value > 2) break;
      g.pull_split = (int)value;
      return RG_OK;
    case RG_OPT_MAX_LEVELS: g.max_levels = value; return RG_OK;
    case RG_OPT_PULL_GROUPS:
      if (value < 2 || value > 16) break;
      g.pull_groups = value;
      return RG_OK;
    case RG_OPT_FUSED_MAX:
      if (value > rg::SMALL_EDGES) break;
      g.fused_max = value;
      return RG_OK;
    case RG_OPT_PHASE_TRACE:
      if (value > 1) break;
      g.phase_trace = (int)value;
      g.d.ptrace = value ? g.ptrace_buf : nullptr;
      return RG_OK;
    case RG_OPT_INLINE_MAX:
      if (value > rg::INLINE_MAX_EDGES) break;
      g.inline_max = value;
      return RG_OK;
    case RG_OPT_CLUSTER_EDGES:
      if (value > (1ull << 20)) break;
      g.cluster_edges = value;
      return RG_OK;
  }
  rg::set_error("unknown option");
  return RG_EINVAL;
}

int rg_get_option(rg_graph *gh, int option, uint64_t *value) {
  if (!gh || !value) return RG_EINVAL;
  Graph &g = gh->g;
  switch (option) {
    case RG_OPT_DENSE_PULL: *value = (uint64_t)g.dense_pull; return RG_OK;
    case RG_OPT_DENSE_DIV: *value = g.dense_div; return RG_OK;
    case RG_OPT_LBS_MIN: *value = g.lbs_min; return RG_OK;
    case RG_OPT_BFS_BOTTOM_UP: *value = (uint64_t)g.bfs_bottom_up; return RG_OK;
    case RG_OPT_RECOMPUTE_MIN: *value = g.recompute_min; return RG_OK;
    case RG_OPT_BFS_BU_DIV: *value = g.bu_div; return RG_OK;
    case RG_OPT_PULL_DIV: *value = g.pull_div; return RG_OK;
    case RG_OPT_TINY_EDGES: *value = g.tiny_edges; return RG_OK;
    case RG_OPT_PULL_SPLIT: *value = (uint64_t)g.pull_split; return RG_OK;
    case RG_OPT_MAX_LEVELS: *value = g.max_levels; return RG_OK;
    case RG_OPT_PULL_GROUPS: *value = g.pull_groups; return RG_OK;
    case RG_OPT_FUSED_MAX: *value = g.fused_max; return RG_OK;
    case RG_OPT_PHASE_TRACE: *value = (uint64_t)g.phase_trace; return RG_OK;
    case RG_OPT_INLINE_MAX: *value = g.inline_max; return RG_OK;
    case RG_OPT_CLUSTER_EDGES: *value = g.cluster_edges; return RG_OK;
  }
  rg::set_error("unknown option");
  return RG_EINVAL;
}

int rg_device_bytes(rg_graph *gh, uint64_t *bytes) {
  if (!gh || !bytes) return RG_EINVAL;
  *bytes = gh->g.bytes;
  return RG_OK;
}

}  // extern "C"
