// Versioned label history (rg_history_* in include/risgraph_b200.h): the
// device form of the reference's MVVec (core/mvvec.hpp:23-162), which the
// _inc_rt drivers fill with the value of every vertex an update modified,
// tagged with the update's version (src/sssp_inc_rt.cpp:338-343), so that a
// reader can ask for a vertex's value as of an earlier version.
//
// Layout: per vertex the index of its newest node (head[v], NIL if none);
// nodes {begin version, previous node, value} in a bump-allocated pool, so a
// vertex's history is a chain from newest to oldest.  set() follows MVVec::set:
// a new node only when the value changed at a newer version, an overwrite when
// the version is the same.  gc(t) keeps, per vertex, the nodes newer than t and
// the newest node at or before t (MVVec::gc), then packs the pool.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include "rg_internal.cuh"

namespace rg {
namespace {

constexpr unsigned long long NIL = ~0ull;
constexpr int HT_TPB = 256;

__global__ void k_hist_fill(unsigned long long *head, uint64_t V) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += stride) head[v] = NIL;
}

// One vertex's set (single writer per vertex in one call: the modified list
// holds each vertex once).
__device__ __forceinline__ void hist_set(const DevGraph &g, HistNode *nodes, unsigned long long *head,
                                         unsigned long long *top, uint64_t cap, unsigned long long *err, uint32_t v,
                                         uint64_t version) {
  const uint64_t value = ld_val(&g.lab[v]);
  const unsigned long long cur = head[v];
  if (cur != NIL && nodes[cur].begin == version) {
    nodes[cur].value = value;  // overwrite the same version
    return;
  }
  if (cur != NIL && (nodes[cur].begin > version || nodes[cur].value == value)) return;
  const unsigned long long idx = atomicAdd(top, 1ull);
  if (idx >= cap) {
    atomicCAS(err, 0ull, (unsigned long long)RG_ENOSPACE);
    return;
  }
  nodes[idx] = HistNode{version, cur, value};
  head[v] = idx;
}

__global__ void k_hist_record_modified(DevGraph g, HistNode *nodes, unsigned long long *head,
                                       unsigned long long *top, uint64_t cap, unsigned long long *err,
                                       uint64_t version) {
  const uint64_t n = g.ctl[C_MODN];
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride)
    hist_set(g, nodes, head, top, cap, err, g.modq[i], version);
}

__global__ void k_hist_record_all(DevGraph g, HistNode *nodes, unsigned long long *head, unsigned long long *top,
                                  uint64_t cap, unsigned long long *err, uint64_t version) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < g.V; v += stride)
    hist_set(g, nodes, head, top, cap, err, (uint32_t)v, version);
}

// MVVec::get: the newest node at or before `version`.
__global__ void k_hist_get(const HistNode *nodes, const unsigned long long *head, const uint32_t *vids, uint64_t n,
                           uint64_t version, uint64_t *out, uint8_t *found) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    unsigned long long c = head[vids[i]];
    while (c != NIL && nodes[c].begin > version) c = nodes[c].pre;
    out[i] = c == NIL ? 0 : nodes[c].value;
    found[i] = c != NIL;
  }
}

// gc: the number of nodes each vertex keeps (newer than t, plus the newest at
// or before t).
__global__ void k_hist_keep(const HistNode *nodes, const unsigned long long *head, uint64_t V, uint64_t t,
                            uint64_t *keep) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v <= V; v += stride) {
    uint64_t k = 0;
    if (v < V)
      for (unsigned long long c = head[v]; c != NIL; c = nodes[c].pre) {
        k++;
        if (nodes[c].begin <= t) break;
      }
    keep[v] = k;
  }
}

// Copy the kept chain of every vertex to [off[v], off[v] + keep) of the new
// pool, newest first, relinking the previous pointers.
__global__ void k_hist_pack(const HistNode *nodes, unsigned long long *head, uint64_t V, const uint64_t *off,
                            const uint64_t *keep, HistNode *out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += stride) {
    const uint64_t k = keep[v], o = off[v];
    unsigned long long c = head[v];
    for (uint64_t j = 0; j < k; j++) {
      HistNode x = nodes[c];
      c = x.pre;
      x.pre = j + 1 < k ? o + j + 1 : NIL;
      out[o + j] = x;
    }
    head[v] = k ? o : NIL;
  }
}

int grid(const Graph &g, uint64_t n) {
  uint64_t b = (n + HT_TPB - 1) / HT_TPB;
  b = b < (uint64_t)g.num_sms * 8 ? b : (uint64_t)g.num_sms * 8;
  return (int)(b ? b : 1);
}

}  // namespace

int history_enable(Graph &g, uint64_t capacity) {
  if (g.hist_nodes) {
    set_error("history already enabled");
    return RG_ESTATE;
  }
  if (!g.trace) {
    set_error("history needs a graph created with trace_modified");
    return RG_ESTATE;
  }
  if (capacity == 0) {
    set_error("history capacity must be positive");
    return RG_EINVAL;
  }
  cudaError_t e = cudaMalloc(&g.hist_nodes, capacity * sizeof(HistNode));
  if (e == cudaSuccess) e = cudaMalloc(&g.hist_head, g.V * 8);
  if (e == cudaSuccess) e = cudaMalloc(&g.hist_ctl, 16);
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaFree(g.hist_nodes);
    cudaFree(g.hist_head);
    g.hist_nodes = nullptr;
    g.hist_head = nullptr;
    set_error("device allocation failed: history");
    return RG_ENOMEM_HBM;
  }
  g.hist_cap = capacity;
  g.bytes += capacity * sizeof(HistNode) + g.V * 8 + 16;
  count_launch(g);
  k_hist_fill<<<grid(g, g.V), HT_TPB, 0, g.stream>>>(g.hist_head, g.V);
  RG_CUDA(cudaMemsetAsync(g.hist_ctl, 0, 16, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  return RG_OK;
}

int history_record(Graph &g, uint64_t version, int all) {
  if (!g.hist_nodes) {
    set_error("history not enabled");
    return RG_ESTATE;
  }
  unsigned long long *top = g.hist_ctl, *err = g.hist_ctl + 1;
  count_launch(g);
  if (all)
    k_hist_record_all<<<grid(g, g.V), HT_TPB, 0, g.stream>>>(g.d, g.hist_nodes, g.hist_head, top, g.hist_cap, err,
                                                               version);
  else
    k_hist_record_modified<<<g.num_sms * 4, HT_TPB, 0, g.stream>>>(g.d, g.hist_nodes, g.hist_head, top, g.hist_cap,
                                                                   err, version);
  RG_CUDA(cudaGetLastError());
  unsigned long long h[2];
  RG_CUDA(cudaMemcpyAsync(h, g.hist_ctl, 16, cudaMemcpyDeviceToHost, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  g.hist_used = h[0] < g.hist_cap ? h[0] : g.hist_cap;
  if (h[1]) {
    // keep the pool consistent: the nodes that did not fit were not linked
    RG_CUDA(cudaMemsetAsync(err, 0, 8, g.stream));
    unsigned long long used = g.hist_used;
    RG_CUDA(cudaMemcpyAsync(top, &used, 8, cudaMemcpyHostToDevice, g.stream));
    RG_CUDA(cudaStreamSynchronize(g.stream));
    set_error("history pool is full (call rg_history_gc or enable a larger pool)");
    return RG_ENOSPACE;
  }
  return RG_OK;
}

int history_get(Graph &g, const uint64_t *vids, uint64_t n, uint64_t version, uint64_t *values, uint8_t *found) {
  if (!g.hist_nodes) {
    set_error("history not enabled");
    return RG_ESTATE;
  }
  if (!n) return RG_OK;
  for (uint64_t i = 0; i < n; i++)
    if (vids[i] >= g.V) {
      set_error("VertexId error.");
      return RG_EINVAL_VID;
    }
  uint32_t *dv = nullptr;
  uint64_t *dout = nullptr;
  uint8_t *dfound = nullptr;
  std::vector<uint32_t> v32(vids, vids + n);
  cudaError_t e = cudaMalloc(&dv, n * 4);
  if (e == cudaSuccess) e = cudaMalloc(&dout, n * 8);
  if (e == cudaSuccess) e = cudaMalloc(&dfound, n);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dv, v32.data(), n * 4, cudaMemcpyHostToDevice, g.stream);
  if (e == cudaSuccess) {
    count_launch(g);
    k_hist_get<<<grid(g, n), HT_TPB, 0, g.stream>>>(g.hist_nodes, g.hist_head, dv, n, version, dout, dfound);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(values, dout, n * 8, cudaMemcpyDeviceToHost, g.stream);
  if (e == cudaSuccess && found) e = cudaMemcpyAsync(found, dfound, n, cudaMemcpyDeviceToHost, g.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g.stream);
  cudaFree(dv);
  cudaFree(dout);
  cudaFree(dfound);
  if (e != cudaSuccess) return cuda_fail(e, "history read");
  return RG_OK;
}

int history_gc(Graph &g, uint64_t version) {
  if (!g.hist_nodes) {
    set_error("history not enabled");
    return RG_ESTATE;
  }
  const uint64_t V = g.V;
  uint64_t *keep = g.scratch64;  // V + 1 entries
  uint64_t *off = nullptr;
  HistNode *fresh = nullptr;
  cudaError_t e = cudaMalloc(&off, (V + 1) * 8);
  if (e == cudaSuccess) e = cudaMalloc(&fresh, g.hist_cap * sizeof(HistNode));
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaFree(off);
    set_error("device allocation failed: history gc");
    return RG_ENOMEM_HBM;
  }
  count_launch(g, 2);
  k_hist_keep<<<grid(g, V + 1), HT_TPB, 0, g.stream>>>(g.hist_nodes, g.hist_head, V, version, keep);
  size_t tb = g.cub_tmp_bytes;
  e = cub::DeviceScan::ExclusiveSum(g.cub_tmp, tb, keep, off, V + 1, g.stream);
  if (e == cudaSuccess) {
    k_hist_pack<<<grid(g, V), HT_TPB, 0, g.stream>>>(g.hist_nodes, g.hist_head, V, off, keep, fresh);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(g.hist_ctl, off + V, 8, cudaMemcpyDeviceToDevice, g.stream);
  unsigned long long used = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&used, off + V, 8, cudaMemcpyDeviceToHost, g.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g.stream);
  cudaFree(off);
  if (e != cudaSuccess) {
    cudaFree(fresh);
    return cuda_fail(e, "history gc");
  }
  cudaFree(g.hist_nodes);
  g.hist_nodes = fresh;
  g.hist_used = used;
  return RG_OK;
}

void history_free(Graph &g) {
  cudaFree(g.hist_nodes);
  cudaFree(g.hist_head);
  cudaFree(g.hist_ctl);
  g.hist_nodes = nullptr;
  g.hist_head = nullptr;
  g.hist_ctl = nullptr;
}

}  // namespace rg
