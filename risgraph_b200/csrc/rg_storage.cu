// Device-resident dynamic adjacency with multiplicity counts: the B200 form of
// the reference's IndexedEdgeStorage (core/storage.hpp:282-430) and of
// Graph::add_edge / del_edge (core/graph.hpp:203-253).
//
// A batch of edge updates runs as a short fixed sequence of kernels with no host
// decision in between:
//   unpack   -> directed ops (two per undirected edge, as add_edge(e,false) does)
//   lookup   -> find (src,dst,w) in the edge index, creating the record and
//               reserving a slot at the end of the src (and dst) segment if new
//   grow     -> move segments that ran out of capacity to a larger pool region
//   write    -> store the new entries, still DEAD (multiplicity 0)
//   count    -> atomic multiplicity update returning the old count; the 0->1
//               and 1->0 transitions flip the DEAD bit
//   edge_old -> per-edge old count with the reference's undirected conventions,
//               plus the candidate list for tree repair (0->1 adds, 1->0 dels)
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include <cub/device/device_scan.cuh>

#include "rg_internal.cuh"
#include "rg_storage_dev.cuh"

namespace rg {

namespace {

constexpr int TPB = 256;

using namespace sdev;

#define GRID_STRIDE(j, n) \
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x, _st = (uint64_t)gridDim.x * blockDim.x; j < (n); j += _st)

__global__ void k_unpack_edges(const rg_edge *e, uint64_t n, int directed, int weighted, OpView ops) {
  GRID_STRIDE(i, n) unpack_edge(e, i, directed, weighted, ops);
}

__global__ void k_unpack_pairs(const uint64_t *p, uint64_t n, int directed, int weighted, OpView ops) {
  GRID_STRIDE(i, n) unpack_pair(p, i, directed, weighted, ops);
}

__global__ void k_lookup(DevGraph g, OpView ops, uint64_t nops, int create) {
  GRID_STRIDE(j, nops) lookup_op(g, ops, j, create);
}

// One CTA per growing vertex.
template <bool W>
__global__ void k_grow(DevDir dir, unsigned long long *ctl, int which) {
  __shared__ GrowShared sh;
  const unsigned long long n = ctl[which];
  for (unsigned long long k = blockIdx.x; k < n; k += gridDim.x) grow_vertex<W>(dir, ctl, dir.grow[k], sh);
}

// Pool compaction: segments keep their capacity and slot order, but are
// packed back to back into a fresh pool (regions abandoned by growth are
// reclaimed).  Slot positions inside a segment do not change, so edge records
// stay valid.
__global__ void k_caps_u64(const uint32_t *cap, uint64_t V, uint64_t *out) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += stride) out[v] = cap[v];
}

template <bool W>
__global__ void k_compact(DevDir dir, const void *old_pool, void *new_pool, uint32_t *new_owner,
                          const uint64_t *new_off, uint64_t V) {
  using E = typename std::conditional<W, uint2, uint32_t>::type;
  const E *src = reinterpret_cast<const E *>(old_pool);
  E *dst = reinterpret_cast<E *>(new_pool);
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t v = warp; v < V; v += nwarps) {
    uint32_t len = dir.len[v], cap = dir.cap[v];
    uint32_t n = len < cap ? len : cap;
    uint64_t from = dir.off[v], to = new_off[v];
    for (uint32_t i = lane; i < n; i += 32) {
      dst[to + i] = src[from + i];
      new_owner[to + i] = (uint32_t)v;
    }
    __syncwarp();
    if (lane == 0) dir.off[v] = to;
  }
}

template <bool W>
__global__ void k_write_new(DevGraph g, OpView ops, uint64_t nops) {
  if (g.ctl[C_ERR]) return;  // a failed growth is compacted and replayed by the host
  GRID_STRIDE(j, nops) write_new_op<W>(g, ops, j);
}

template <bool W>
__global__ void k_count(DevGraph g, OpView ops, uint64_t nops, int add) {
  if (g.ctl[C_ERR]) return;
  GRID_STRIDE(j, nops) count_op<W>(g, ops, j, add);
}

__global__ void k_edge_old(OpView ops, uint64_t n, int directed, int add, int collect, uint64_t *old_out,
                           uint32_t *cand, unsigned long long *ctl) {
  if (ctl[C_ERR]) return;
  GRID_STRIDE(i, n) edge_old(ops, i, directed, add, collect, old_out, cand, ctl);
}

__global__ void k_get_num(DevGraph g, OpView ops, uint64_t nops, uint64_t *out) {
  GRID_STRIDE(j, nops) {
    uint32_t rid = ops.rid[j];
    out[j] = rid == UNSET ? 0 : g.rec_num[rid];
  }
}

int grid_for(const Graph &g, uint64_t n) {
  uint64_t b = (n + TPB - 1) / TPB;
  uint64_t cap = (uint64_t)g.num_sms * 16;
  if (b > cap) b = cap;
  if (b == 0) b = 1;
  return (int)b;
}

int ensure_ops(Graph &g, uint64_t nops, uint64_t n_edges) {
  if (nops <= g.ops_cap && g.ops) return RG_OK;
  uint64_t cap = std::max<uint64_t>(nops, 1024);
  cap = std::max<uint64_t>(cap, g.ops_cap * 2);
  cap = (cap + 63) & ~63ull;  // keeps the u64 old-count array 8-byte aligned
  if (g.ops) cudaFree(g.ops);
  g.ops = nullptr;
  // O_NARR u32 arrays + candidate list (n_edges u32) + u64 old per edge
  size_t bytes = (size_t)cap * (O_NARR + 1) * 4 + (size_t)cap * 8;
  cudaError_t e = cudaMalloc(&g.ops, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(ops)");
  g.ops_cap = cap;
  (void)n_edges;
  return RG_OK;
}

int ensure_stage(Graph &g, size_t bytes) {
  if (bytes > g.stage_dev_bytes) {
    if (g.stage_dev) cudaFree(g.stage_dev);
    g.stage_dev = nullptr;
    size_t b = std::max(bytes, g.stage_dev_bytes * 2);
    cudaError_t e = cudaMalloc(&g.stage_dev, b);
    if (e != cudaSuccess) { g.stage_dev_bytes = 0; return cuda_fail(e, "cudaMalloc(stage)"); }
    g.stage_dev_bytes = b;
  }
  if (bytes > g.stage_host_bytes) {
    if (g.stage_host) cudaFreeHost(g.stage_host);
    g.stage_host = nullptr;
    size_t b = std::max(bytes, g.stage_host_bytes * 2);
    cudaError_t e = cudaHostAlloc(&g.stage_host, b, cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(&g.stage_host_dev, g.stage_host, 0);
    if (e != cudaSuccess) { g.stage_host_bytes = 0; return cuda_fail(e, "cudaHostAlloc(stage)"); }
    g.stage_host_bytes = b;
  }
  return RG_OK;
}

uint64_t *old_dev(Graph &g) {
  return reinterpret_cast<uint64_t *>(g.ops + (uint64_t)(O_NARR + 1) * g.ops_cap);
}

// Read the device error word; also syncs the stream.
int finish(Graph &g, bool need_old, uint64_t *old_num, uint64_t n) {
  RG_CUDA(cudaMemcpyAsync(g.h_ctl, g.d.ctl, sizeof(unsigned long long) * C_COUNT, cudaMemcpyDeviceToHost, g.stream));
  if (need_old && old_num)
    RG_CUDA(cudaMemcpyAsync(old_num, old_dev(g), n * 8, cudaMemcpyDeviceToHost, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  if (g.h_ctl[C_ERR]) {
    int code = (int)g.h_ctl[C_ERR];
    set_error(code == RG_ENOSPACE ? (g.h_ctl[C_AUX] == 1 ? "device edge pool is full" : "device edge index is full")
                                  : "device error");
    cudaMemsetAsync(&g.d.ctl[C_ERR], 0, 8, g.stream);
    return code;
  }
  return RG_OK;
}

}  // namespace

int storage_reserve(Graph &g, uint64_t n_edges) {
  int rc = ensure_ops(g, 2 * n_edges, n_edges);
  if (!rc) rc = ensure_stage(g, n_edges * sizeof(rg_edge));
  return rc;
}

uint32_t *op_src(Graph &g) { return g.ops + (uint64_t)O_SRC * g.ops_cap; }
uint32_t *op_dst(Graph &g) { return g.ops + (uint64_t)O_DST * g.ops_cap; }
uint32_t *op_w(Graph &g) { return g.ops + (uint64_t)O_W * g.ops_cap; }
uint32_t *op_cand(Graph &g) { return g.ops + (uint64_t)O_NARR * g.ops_cap; }

static uint64_t next_pow2(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

int storage_alloc(Graph &g) {
  uint64_t V = g.V;
  uint64_t keys = g.hint * (g.symmetric ? 2 : 1);
  if (keys < 1024) keys = 1024;
  uint64_t ht_cap = next_pow2(keys + keys / 2);  // load <= 2/3 at the hint
  uint64_t rec_cap = ht_cap - ht_cap / 8;
  uint64_t pool_cap = 2 * keys + 8 * V + 1024;  // slack for growth; compaction reclaims the rest
  size_t esz = g.weighted ? 8 : 4;
  auto alloc = [&](void **p, size_t bytes, const char *what) -> int {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error(std::string("device allocation failed: ") + what);
      return RG_ENOMEM_HBM;
    }
    g.bytes += bytes;
    return RG_OK;
  };
  int rc;
  DevGraph &d = g.d;
  d.V = (uint32_t)V;
  d.weighted = g.weighted;
  d.symmetric = g.symmetric;
  for (int dir = 0; dir < (g.symmetric ? 1 : 2); dir++) {
    DevDir &D = dir == 0 ? d.out : d.in;
    if ((rc = alloc((void **)&D.off, V * 8 + 8, "segment offsets"))) return rc;
    if ((rc = alloc((void **)&D.len, V * 4 + 4, "segment lengths"))) return rc;
    if ((rc = alloc((void **)&D.cap, V * 4 + 4, "segment capacities"))) return rc;
    if ((rc = alloc((void **)&D.deg, V * 8 + 8, "degrees"))) return rc;
    if ((rc = alloc((void **)&D.grow, V * 4 + 4, "grow list"))) return rc;
    if ((rc = alloc(&D.pool, pool_cap * esz, "edge pool"))) return rc;
    if ((rc = alloc((void **)&D.pool_top, 8, "pool top"))) return rc;
    if ((rc = alloc((void **)&D.owner, pool_cap * 4, "slot owners"))) return rc;
    RG_CUDA(cudaMemset(D.owner, 0xff, pool_cap * 4));
    D.pool_cap = pool_cap;
    RG_CUDA(cudaMemset(D.off, 0, V * 8 + 8));
    RG_CUDA(cudaMemset(D.len, 0, V * 4 + 4));
    RG_CUDA(cudaMemset(D.cap, 0, V * 4 + 4));
    RG_CUDA(cudaMemset(D.deg, 0, V * 8 + 8));
    RG_CUDA(cudaMemset(D.pool_top, 0, 8));
  }
  if (g.symmetric) d.in = d.out;  // incoming == outgoing (core/graph.hpp:167,183,194)
  if ((rc = alloc((void **)&d.ht, ht_cap * 16, "edge index"))) return rc;
  RG_CUDA(cudaMemset(d.ht, 0xff, ht_cap * 16));
  d.ht_mask = ht_cap - 1;
  if ((rc = alloc((void **)&d.rec_num, rec_cap * 4, "edge records"))) return rc;
  if ((rc = alloc((void **)&d.rec_out, rec_cap * 4, "edge records"))) return rc;
  if ((rc = alloc((void **)&d.rec_in, rec_cap * 4, "edge records"))) return rc;
  if ((rc = alloc((void **)&d.rec_top, 8, "record top"))) return rc;
  RG_CUDA(cudaMemset(d.rec_top, 0, 8));
  d.rec_cap = rec_cap;
  return RG_OK;
}

void storage_free(Graph &g) {
  DevGraph &d = g.d;
  for (int dir = 0; dir < (g.symmetric ? 1 : 2); dir++) {
    DevDir &D = dir == 0 ? d.out : d.in;
    cudaFree(D.off); cudaFree(D.len); cudaFree(D.cap); cudaFree(D.deg); cudaFree(D.grow);
    cudaFree(D.pool); cudaFree(D.pool_top); cudaFree(D.owner);
  }
  cudaFree(d.ht); cudaFree(d.rec_num); cudaFree(d.rec_out); cudaFree(d.rec_in); cudaFree(d.rec_top);
  if (g.ops) cudaFree(g.ops);
  if (g.stage_dev) cudaFree(g.stage_dev);
  if (g.stage_host) cudaFreeHost(g.stage_host);
  g.ops = nullptr; g.stage_dev = nullptr; g.stage_host = nullptr;
}

int stage_edges(Graph &g, const rg_edge *edges, const uint64_t *pairs, uint64_t n, int directed, uint64_t *nops) {
  uint64_t k = directed ? n : 2 * n;
  *nops = k;
  int rc = ensure_ops(g, k, n);
  if (rc) return rc;
  size_t bytes = pairs ? n * 16 : n * sizeof(rg_edge);
  if ((rc = ensure_stage(g, bytes))) return rc;
  if (n == 0) return RG_OK;
  std::memcpy(g.stage_host, pairs ? (const void *)pairs : (const void *)edges, bytes);
  RG_CUDA(cudaMemcpyAsync(g.stage_dev, g.stage_host, bytes, cudaMemcpyHostToDevice, g.stream));
  OpView ops = op_view(g);
  count_launch(g);
  if (pairs)
    k_unpack_pairs<<<grid_for(g, n), TPB, 0, g.stream>>>((const uint64_t *)g.stage_dev, n, directed, g.weighted, ops);
  else
    k_unpack_edges<<<grid_for(g, n), TPB, 0, g.stream>>>((const rg_edge *)g.stage_dev, n, directed, g.weighted, ops);
  RG_CUDA(cudaGetLastError());
  return RG_OK;
}

static int grow_dir(Graph &g, DevDir &dir, int which) {
  int grid = g.num_sms * 8;
  count_launch(g);
  if (g.weighted) k_grow<true><<<grid, TPB, 0, g.stream>>>(dir, g.d.ctl, which);
  else k_grow<false><<<grid, TPB, 0, g.stream>>>(dir, g.d.ctl, which);
  RG_CUDA(cudaGetLastError());
  return RG_OK;
}

// Pack one direction's segments into a fresh pool (see k_compact).
static int compact_dir(Graph &g, DevDir &dir) {
  const uint64_t V = g.V;
  uint64_t *offs = nullptr;
  void *tmp = nullptr, *fresh = nullptr;
  uint32_t *fresh_owner = nullptr;
  size_t tmp_bytes = 0;
  const size_t esz = g.weighted ? 8 : 4;
  int rc = RG_OK;
  count_launch(g);
  k_caps_u64<<<g.num_sms * 8, TPB, 0, g.stream>>>(dir.cap, V, g.scratch64);
  RG_CUDA(cudaMemsetAsync(g.scratch64 + V, 0, 8, g.stream));
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, g.scratch64, g.scratch64, V + 1, g.stream);
  cudaError_t e = cudaMalloc(&tmp, tmp_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&offs, (V + 1) * 8);
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaFree(tmp);
    set_error("device allocation failed: pool compaction");
    return RG_ENOMEM_HBM;
  }
  cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, g.scratch64, offs, V + 1, g.stream);
  uint64_t total = 0;
  RG_CUDA(cudaMemcpyAsync(&total, offs + V, 8, cudaMemcpyDeviceToHost, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  if (total > dir.pool_cap) {
    set_error("device edge pool is full even after compaction");
    rc = RG_ENOSPACE;
  } else if ((e = cudaMalloc(&fresh, dir.pool_cap * esz)) != cudaSuccess ||
             (e = cudaMalloc(&fresh_owner, dir.pool_cap * 4)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(fresh);
    set_error("device allocation failed: pool compaction");
    rc = RG_ENOMEM_HBM;
  } else {
    count_launch(g);
    cudaMemsetAsync(fresh_owner, 0xff, dir.pool_cap * 4, g.stream);
    if (g.weighted)
      k_compact<true><<<g.num_sms * 16, TPB, 0, g.stream>>>(dir, dir.pool, fresh, fresh_owner, offs, V);
    else
      k_compact<false><<<g.num_sms * 16, TPB, 0, g.stream>>>(dir, dir.pool, fresh, fresh_owner, offs, V);
    unsigned long long top = total;
    cudaMemcpyAsync(dir.pool_top, &top, 8, cudaMemcpyHostToDevice, g.stream);
    e = cudaStreamSynchronize(g.stream);
    if (e != cudaSuccess) rc = cuda_fail(e, "pool compaction");
    cudaFree(dir.pool);
    cudaFree(dir.owner);
    dir.pool = fresh;
    dir.owner = fresh_owner;
    g.layout_version++;  // cached level-loop graphs hold the old pool pointers
  }
  cudaFree(tmp);
  cudaFree(offs);
  if (g.symmetric) g.d.in = g.d.out;
  return rc;
}

// Pool exhaustion during growth: compact both directions; the caller then
// replays the batch from the growth step (storage_replay).
int storage_recover(Graph &g) {
  RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_ERR], 0, 8, g.stream));
  RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_AUX], 0, 8, g.stream));
  int rc = compact_dir(g, g.d.out);
  if (!rc && !g.symmetric) rc = compact_dir(g, g.d.in);
  return rc;
}

static int enqueue_after_lookup(Graph &g, uint64_t n, uint64_t nops, int directed, bool collect) {
  OpView ops = op_view(g);
  int rc = grow_dir(g, g.d.out, C_GROWN_OUT);
  if (!rc && !g.symmetric) rc = grow_dir(g, g.d.in, C_GROWN_IN);
  if (rc) return rc;
  count_launch(g, 3);
  if (collect) RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_CANDN], 0, 8, g.stream));
  if (g.weighted) {
    k_write_new<true><<<grid_for(g, nops), TPB, 0, g.stream>>>(g.d, ops, nops);
    k_count<true><<<grid_for(g, nops), TPB, 0, g.stream>>>(g.d, ops, nops, 1);
  } else {
    k_write_new<false><<<grid_for(g, nops), TPB, 0, g.stream>>>(g.d, ops, nops);
    k_count<false><<<grid_for(g, nops), TPB, 0, g.stream>>>(g.d, ops, nops, 1);
  }
  k_edge_old<<<grid_for(g, n), TPB, 0, g.stream>>>(ops, n, directed, 1, collect, old_dev(g), op_cand(g), g.d.ctl);
  RG_CUDA(cudaGetLastError());
  return RG_OK;
}

// Storage kernels of one staged batch, enqueued without waiting.  Each kernel
// after the growth step skips its work once the device error word is set.
int storage_enqueue(Graph &g, bool add, uint64_t n, uint64_t nops, int directed, bool collect) {
  OpView ops = op_view(g);
  g.adj_version++;
  if (collect) RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_CANDN], 0, 8, g.stream));
  if (!nops) return RG_OK;
  if (add) {
    RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_GROWN_OUT], 0, 16, g.stream));
    count_launch(g);
    k_lookup<<<grid_for(g, nops), TPB, 0, g.stream>>>(g.d, ops, nops, 1);
    RG_CUDA(cudaGetLastError());
    return enqueue_after_lookup(g, n, nops, directed, collect);
  }
  count_launch(g, 3);
  k_lookup<<<grid_for(g, nops), TPB, 0, g.stream>>>(g.d, ops, nops, 0);
  if (g.weighted) k_count<true><<<grid_for(g, nops), TPB, 0, g.stream>>>(g.d, ops, nops, 0);
  else k_count<false><<<grid_for(g, nops), TPB, 0, g.stream>>>(g.d, ops, nops, 0);
  k_edge_old<<<grid_for(g, n), TPB, 0, g.stream>>>(ops, n, directed, 0, collect, old_dev(g), op_cand(g), g.d.ctl);
  RG_CUDA(cudaGetLastError());
  return RG_OK;
}

int storage_replay(Graph &g, uint64_t n, uint64_t nops, int directed, bool collect) {
  if (!nops) return RG_OK;
  return enqueue_after_lookup(g, n, nops, directed, collect);
}

// Per-edge old counts into the pinned staging buffer (read after the sync).
int storage_copy_old(Graph &g, uint64_t n) {
  if (n) RG_CUDA(cudaMemcpyAsync(g.stage_host, old_dev(g), n * 8, cudaMemcpyDeviceToHost, g.stream));
  return RG_OK;
}

const uint64_t *storage_old_host(Graph &g) { return reinterpret_cast<const uint64_t *>(g.stage_host); }

int sync_ctl(Graph &g) {
  RG_CUDA(cudaMemcpyAsync(g.h_ctl, g.d.ctl, sizeof(unsigned long long) * C_COUNT, cudaMemcpyDeviceToHost, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  return RG_OK;
}

// Device error left by the storage kernels, as a status (clears it).
int storage_error(Graph &g) {
  if (!g.h_ctl[C_ERR]) return RG_OK;
  int code = (int)g.h_ctl[C_ERR];
  set_error(code == RG_ENOSPACE ? (g.h_ctl[C_AUX] == 1 ? "device edge pool is full" : "device edge index is full")
                                : "device error");
  cudaMemsetAsync(&g.d.ctl[C_ERR], 0, 8, g.stream);
  cudaMemsetAsync(&g.d.ctl[C_AUX], 0, 8, g.stream);
  return code;
}

int storage_num(Graph &g, uint64_t nops, uint64_t *num) {
  OpView ops = op_view(g);
  if (nops) {
    count_launch(g, 2);
    k_lookup<<<grid_for(g, nops), TPB, 0, g.stream>>>(g.d, ops, nops, 0);
    k_get_num<<<grid_for(g, nops), TPB, 0, g.stream>>>(g.d, ops, nops, old_dev(g));
    RG_CUDA(cudaGetLastError());
  }
  return finish(g, true, num, nops);
}

}  // namespace rg
