// rg_build_tree_csr_static: a full build_tree that allocates nothing.
//
// Some callers cannot allocate device memory at the point where they need a
// dependency tree: a serving process whose memory is owned by another
// framework's pool and carved up at start-up (any cudaMalloc later would break
// the budget or fail), or a latency-critical path where cudaMalloc / cudaFree
// would synchronise the device and stall unrelated work.  For them this entry
// point runs the same level-synchronous push relaxation as rg_build_tree on a
// caller-owned CSR graph, writing into caller-owned output arrays, and keeps
// all of its working memory (labels, two frontier queues, dedup stamps and a
// few counters) in one file-scope static __device__ array of fixed size.
//
// Limits and sharing rules:
//  * at most RG_STATIC_MAX_VERTICES vertices (larger graphs are rejected with
//    RG_EINVAL before anything runs);
//  * the scratch array (about 28 MB) is held on every GPU where this library's
//    device code has been loaded, for the life of the process;
//  * every call shares that one array, and it keeps the previous call's
//    contents: each call clears the parts that must start at zero itself, but
//    two calls whose work overlaps on the GPU (different streams, or different
//    host threads) race on it and both results are undefined;
//  * the device address of the array is looked up once per device, on the
//    first call made with that device current (cudaGetSymbolAddress).  With
//    lazy module loading (the CUDA default) that lookup is also what loads this
//    library's device code, and with it the array, onto the device; a call
//    with vertices == 0 and all pointers NULL does only this set-up, so that a
//    caller can take the array at start-up, before another pool claims the
//    device's memory;
//  * each call is synchronous (a counter read-back per level) and must not be
//    made on a stream under capture.
#include <cuda_runtime.h>

#include <mutex>

#include "rg_internal.cuh"

namespace rg {
namespace {

constexpr uint64_t SMAX = RG_STATIC_MAX_VERTICES;
// layout in 8-byte words: labels (2 words/vertex), queue 0, queue 1, stamps
// (u32 each, packed two per word), then the counters
constexpr uint64_t W_LAB = 0;
constexpr uint64_t W_Q0 = W_LAB + 2 * SMAX;
constexpr uint64_t W_Q1 = W_Q0 + SMAX / 2;
constexpr uint64_t W_STAMP = W_Q1 + SMAX / 2;
constexpr uint64_t W_CTL = W_STAMP + SMAX / 2;
constexpr uint64_t W_TOTAL = W_CTL + 32;

// The scratch: labels, frontier queues, stamps, counters.  Host code must use
// the address from cudaGetSymbolAddress, never the symbol itself.
static __device__ __align__(256) unsigned long long rg_static_scratch[W_TOTAL];

struct View {
  ulonglong2 *lab;
  uint32_t *q[2];
  uint32_t *stamp;
  unsigned long long *ctl;  // [0],[1] queue lengths, [2] error
};

View view_of(unsigned long long *base) {
  View v;
  v.lab = reinterpret_cast<ulonglong2 *>(base + W_LAB);
  v.q[0] = reinterpret_cast<uint32_t *>(base + W_Q0);
  v.q[1] = reinterpret_cast<uint32_t *>(base + W_Q1);
  v.stamp = reinterpret_cast<uint32_t *>(base + W_STAMP);
  v.ctl = base + W_CTL;
  return v;
}

template <int A>
__global__ void k_static_init(View s, uint64_t V, uint64_t root) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += stride) {
    s.lab[v] = make_ulonglong2(Hook<A>::init(v, root), pack_parent(NONE, 0));
    if (Hook<A>::all_active) s.q[0][v] = (uint32_t)v;
    else if (v == root) s.q[0][0] = (uint32_t)v;
  }
}

// Variant of the push level of rg_tree.cu for a plain CSR: one warp per
// frontier vertex, lanes striding over its edges.
// Malformed CSR input (offsets decreasing or past `edges`, a column >= V) is
// skipped and reported through ctl[2]; nothing is read or written out of range.
template <int A, bool W>
__global__ void k_static_push(View s, uint64_t V, uint64_t E, const uint64_t *row, const uint32_t *col,
                              const uint32_t *wgt, int in_q, uint32_t st) {
  const uint32_t *fin = s.q[in_q];
  uint32_t *fout = s.q[in_q ^ 1];
  unsigned long long *fout_n = &s.ctl[in_q ^ 1];
  const uint64_t n = s.ctl[in_q];
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = lane_id();
  for (uint64_t i = warp; i < n; i += nwarps) {
    const uint32_t u = fin[i];
    const uint64_t su = ld_val(&s.lab[u]);
    const uint64_t b = row[u], e = row[u + 1];
    if (b > e || e > E) {
      if (lane == 0) s.ctl[2] = RG_EINVAL;
      continue;
    }
    for (uint64_t kb = b; kb < e; kb += 32) {
      const uint64_t k = kb + lane;
      bool upd = false;
      uint32_t v = 0;
      if (k < e && col[k] >= V) {
        s.ctl[2] = RG_EINVAL_VID;
      } else if (k < e) {
        v = col[k];
        const uint32_t w = W ? wgt[k] : 0u;
        const uint64_t nv = Hook<A>::combine(su, w);
        ulonglong2 c = ld_lab(&s.lab[v]);
        while (Hook<A>::better(nv, c.x)) {
          ulonglong2 want = make_ulonglong2(nv, pack_parent(u, w));
          ulonglong2 old = cas128(&s.lab[v], c, want);
          if (old.x == c.x && old.y == c.y) { upd = true; break; }
          c = old;
        }
      }
      bool app = upd && atomicExch(&s.stamp[v], st) != st;
      warp_append(app, v, fout, fout_n, FULL);
    }
  }
}

__global__ void k_static_out(View s, uint64_t V, uint64_t *values, uint64_t *parents) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += stride) {
    ulonglong2 l = s.lab[v];
    if (values) values[v] = l.x;
    uint32_t p = (uint32_t)l.y;
    if (parents) parents[v] = p == NONE ? V : (uint64_t)p;
  }
}

std::mutex g_addr_mu;
unsigned long long *g_addr[64] = {nullptr};

// Per-device address of rg_static_scratch, looked up with that device current.
int scratch_address(unsigned long long **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) {
    set_error("device ordinal out of range");
    return RG_EINVAL;
  }
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, rg_static_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(rg_static_scratch)");
    g_addr[dev] = reinterpret_cast<unsigned long long *>(p);
  }
  *out = g_addr[dev];
  return RG_OK;
}

template <int A, bool W>
int run(uint64_t V, uint64_t E, uint64_t root, const uint64_t *row, const uint32_t *col, const uint32_t *wgt,
        uint64_t *values, uint64_t *parents, cudaStream_t stream) {
  unsigned long long *base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  View s = view_of(base);
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // stamps and counters must start at zero; the rest is overwritten
  RG_CUDA(cudaMemsetAsync(s.stamp, 0, V * 4, stream));
  RG_CUDA(cudaMemsetAsync(s.ctl, 0, 32 * 8, stream));
  unsigned long long n = Hook<A>::all_active ? V : 1;
  RG_CUDA(cudaMemcpyAsync(&s.ctl[0], &n, 8, cudaMemcpyHostToDevice, stream));
  k_static_init<A><<<sms * 8, 256, 0, stream>>>(s, V, root);
  RG_CUDA(cudaGetLastError());
  int q = 0;
  for (uint32_t st = 1; n; st++) {
    if (st > 4 * V + 1024) {
      set_error("push levels did not converge");
      return RG_ETIMEOUT;
    }
    RG_CUDA(cudaMemsetAsync(&s.ctl[q ^ 1], 0, 8, stream));
    uint64_t blocks = (n * 32 + 255) / 256;
    if (blocks > (uint64_t)sms * 16) blocks = (uint64_t)sms * 16;
    k_static_push<A, W><<<(unsigned)blocks, 256, 0, stream>>>(s, V, E, row, col, wgt, q, st);
    RG_CUDA(cudaGetLastError());
    unsigned long long c[3] = {0, 0, 0};
    RG_CUDA(cudaMemcpyAsync(c, s.ctl, sizeof(c), cudaMemcpyDeviceToHost, stream));
    RG_CUDA(cudaStreamSynchronize(stream));
    if (c[2]) {
      set_error(c[2] == RG_EINVAL_VID ? "rg_build_tree_csr_static: column index >= vertices"
                                      : "rg_build_tree_csr_static: row offsets decrease or exceed edges");
      return (int)c[2];
    }
    n = c[q ^ 1];
    q ^= 1;
  }
  k_static_out<<<sms * 8, 256, 0, stream>>>(s, V, values, parents);
  RG_CUDA(cudaGetLastError());
  RG_CUDA(cudaStreamSynchronize(stream));
  return RG_OK;
}

}  // namespace
}  // namespace rg

extern "C" int rg_build_tree_csr_static(int algo, uint64_t root, uint64_t vertices, uint64_t edges,
                                        const uint64_t *row_offsets, const uint32_t *columns,
                                        const uint32_t *weights, uint64_t *values, uint64_t *parents,
                                        void *cuda_stream) {
  using namespace rg;
  if (vertices == 0 && !row_offsets && !columns && !weights && !values && !parents) {
    // set-up only: load the module and look the array's address up on this device
    unsigned long long *base = nullptr;
    return scratch_address(&base);
  }
  if (vertices == 0 || vertices > RG_STATIC_MAX_VERTICES) {
    set_error("rg_build_tree_csr_static: vertices must be in [1, RG_STATIC_MAX_VERTICES]");
    return RG_EINVAL;
  }
  if (!row_offsets || (!columns && vertices) || (!values && !parents)) {
    set_error("rg_build_tree_csr_static: null CSR or output pointer");
    return RG_EINVAL;
  }
  if ((algo == RG_SSSP || algo == RG_SSWP) && !weights) {
    set_error("rg_build_tree_csr_static: SSSP and SSWP need edge weights");
    return RG_EINVAL;
  }
  if (algo != RG_WCC && root >= vertices) {
    set_error("VertexId error.");
    return RG_EINVAL_VID;
  }
  cudaStream_t st = (cudaStream_t)cuda_stream;
  const uint64_t V = vertices, E = edges;
  switch (algo) {
    case RG_BFS: return run<RG_BFS, false>(V, E, root, row_offsets, columns, nullptr, values, parents, st);
    case RG_SSSP: return run<RG_SSSP, true>(V, E, root, row_offsets, columns, weights, values, parents, st);
    case RG_SSWP: return run<RG_SSWP, true>(V, E, root, row_offsets, columns, weights, values, parents, st);
    case RG_WCC: return run<RG_WCC, false>(V, E, 0, row_offsets, columns, nullptr, values, parents, st);
  }
  set_error("unknown algorithm");
  return RG_EINVAL;
}
