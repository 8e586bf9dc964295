// Dependency-tree kernels: the B200 form of Graph::build_tree,
// update_tree_add / do_update_tree_add, update_tree_del / do_update_tree_del,
// need_update_tree_* and update_label (core/graph.hpp:873-1887).
//
// Frontiers are device queues of u32 vertex ids deduplicated per level by a
// stamp word per vertex (the reference's ActiveSet keeps duplicates,
// core/actset.hpp:114-147; duplicates only repeat work).  One level of push
// relaxation is one launch of k_push (+ k_push_hub for split hub lists):
//   * each warp takes 32 frontier vertices, scans their degrees with shuffles
//     and walks the concatenated edge slots 32 at a time, so consecutive lanes
//     read consecutive slots (coalesced 8-byte {nbr,w} loads) whatever the
//     degree mix;
//   * lists longer than HUB slots are cut into CHUNK-slot tasks that any warp
//     of the hub kernel picks up (CTA-per-hub balance without a scan);
//   * a relaxation reads the 16-byte label of the target from L2, and only when
//     update_func improves it does a 128-bit CAS of {value, parent|weight}
//     (update_label, core/graph.hpp:1799-1826); successes are appended to the
//     next frontier with one warp-aggregated atomic.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include <cub/device/device_scan.cuh>

#include "rg_internal.cuh"

namespace rg {

namespace {

constexpr int TPB = 256;
constexpr uint32_t HUB = 64;     // longer lists of a small frontier are split into
constexpr uint32_t CHUNK = 64;   // CHUNK-slot tasks so no warp walks a long list alone
constexpr uint64_t LBS_MIN_FRONTIER = 2048;  // smaller frontiers use k_push

template <bool W>
struct PoolT;
template <>
struct PoolT<true> {
  using E = uint2;
  static __device__ __forceinline__ uint32_t nbr(E e) { return e.x; }
  static __device__ __forceinline__ uint32_t wt(E e) { return e.y; }
};
template <>
struct PoolT<false> {
  using E = uint32_t;
  static __device__ __forceinline__ uint32_t nbr(E e) { return e; }
  static __device__ __forceinline__ uint32_t wt(E) { return 0u; }
};

__device__ __forceinline__ uint32_t seg_len(const DevDir &d, uint32_t v) {
  uint32_t l = d.len[v], c = d.cap[v];
  return l < c ? l : c;
}

// update_label (core/graph.hpp:1799-1826): CAS {value, parent} while the new
// value still improves the current one.
template <int A>
__device__ __forceinline__ bool relax(ulonglong2 *lab, uint32_t u, uint64_t su, uint32_t v, uint32_t w) {
  uint64_t nv = Hook<A>::combine(su, w);
  ulonglong2 cur = ld_lab(&lab[v]);
  while (Hook<A>::better(nv, cur.x)) {
    ulonglong2 want = make_ulonglong2(nv, pack_parent(u, w));
    ulonglong2 old = cas128(&lab[v], cur, want);
    if (old.x == cur.x && old.y == cur.y) return true;
    cur = old;
  }
  return false;
}

__device__ __forceinline__ void warp_add_result(unsigned long long local, unsigned long long *dst) {
  for (int o = 16; o; o >>= 1) local += __shfl_down_sync(FULL, local, o);
  if (lane_id() == 0 && local) atomicAdd(dst, local);
}

__device__ __forceinline__ void mark_modified(const DevGraph &g, bool pred, uint32_t v, uint32_t mst) {
  bool app = pred && atomicExch(&g.modstamp[v], mst) != mst;
  warp_append(app, v, g.modq, &g.ctl[C_MODN], FULL);
}

// One push level over a frontier list (stream_edges / stream_edges_sparse
// push lambdas, core/graph.hpp:910-935, :1017-1042, :1083-1104).
template <int A, bool W>
__global__ void __launch_bounds__(TPB) k_push(DevGraph g, const uint32_t *fin, const unsigned long long *fin_n,
                                              uint32_t *fout, unsigned long long *fout_n, uint32_t st,
                                              uint64_t *hubq, unsigned long long *hub_n, uint32_t mst) {
  using P = PoolT<W>;
  const typename P::E *pool = reinterpret_cast<const typename P::E *>(g.out.pool);
  const uint64_t n = *fin_n;
  const int lane = lane_id();
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long local = 0, scanned = 0;
  for (uint64_t base = warp * 32; base < n; base += nwarps * 32) {
    uint64_t i = base + lane;
    uint32_t u = 0, len = 0;
    uint64_t off = 0, su = 0;
    if (i < n) {
      u = fin[i];
      len = seg_len(g.out, u);
      off = g.out.off[u];
      su = ld_val(&g.lab[u]);
      if (len > HUB) {
        uint32_t nch = (len + CHUNK - 1) / CHUNK;
        unsigned long long k = atomicAdd(hub_n, (unsigned long long)nch);
        for (uint32_t c = 0; c < nch; c++) hubq[k + c] = (uint64_t)u | ((uint64_t)c << 32);
        len = 0;
      }
    }
    uint32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += t;
    }
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    if (lane == 0) scanned += total;
    for (uint32_t kb = 0; kb < total; kb += 32) {
      const uint32_t k = kb + lane;
      const bool valid = k < total;
      int owner = 0;
#pragma unroll
      for (int step = 16; step; step >>= 1) {
        uint32_t t = __shfl_sync(FULL, incl, owner + step - 1);
        if (t <= k) owner += step;
      }
      const uint32_t ou = __shfl_sync(FULL, u, owner);
      const uint64_t ooff = __shfl_sync(FULL, off, owner);
      const uint64_t osu = __shfl_sync(FULL, su, owner);
      const uint32_t ostart = __shfl_sync(FULL, incl - len, owner);
      bool upd = false;
      uint32_t v = 0;
      if (valid) {
        typename P::E e = pool[ooff + (k - ostart)];
        uint32_t nb = P::nbr(e);
        if (!(nb & DEAD)) {
          v = nb;
          upd = relax<A>(g.lab, ou, osu, v, P::wt(e));
        }
      }
      local += upd;
      bool app = upd && atomicExch(&g.stamp[v], st) != st;
      warp_append(app, v, fout, fout_n, FULL);
      if (mst) mark_modified(g, upd, v, mst);
    }
  }
  if (lane == 0 && scanned) atomicAdd(&g.ctl[C_EDGES], scanned);
  warp_add_result(local, &g.ctl[C_RESULT]);
}

// Hub chunks: CHUNK consecutive slots of one long list per warp iteration.
template <int A, bool W>
__global__ void __launch_bounds__(TPB) k_push_hub(DevGraph g, const uint64_t *hubq, const unsigned long long *hub_n,
                                                  uint32_t *fout, unsigned long long *fout_n, uint32_t st,
                                                  uint32_t mst) {
  using P = PoolT<W>;
  const typename P::E *pool = reinterpret_cast<const typename P::E *>(g.out.pool);
  const uint64_t n = *hub_n;
  const int lane = lane_id();
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long local = 0, scanned = 0;
  for (uint64_t t = warp; t < n; t += nwarps) {
    const uint64_t task = hubq[t];
    const uint32_t u = (uint32_t)task, c = (uint32_t)(task >> 32);
    const uint32_t len = seg_len(g.out, u);
    const uint64_t off = g.out.off[u];
    const uint64_t su = ld_val(&g.lab[u]);
    const uint32_t start = c * CHUNK, end = min(len, start + CHUNK);
    if (lane == 0 && end > start) scanned += end - start;
    for (uint32_t kb = start; kb < end; kb += 32) {
      const uint32_t k = kb + lane;
      bool upd = false;
      uint32_t v = 0;
      if (k < end) {
        typename P::E e = pool[off + k];
        uint32_t nb = P::nbr(e);
        if (!(nb & DEAD)) {
          v = nb;
          upd = relax<A>(g.lab, u, su, v, P::wt(e));
        }
      }
      local += upd;
      bool app = upd && atomicExch(&g.stamp[v], st) != st;
      warp_append(app, v, fout, fout_n, FULL);
      if (mst) mark_modified(g, upd, v, mst);
    }
  }
  if (lane == 0 && scanned) atomicAdd(&g.ctl[C_EDGES], scanned);
  warp_add_result(local, &g.ctl[C_RESULT]);
}

// Relaxation of N independent candidate edges held by one thread (u[k] -> v[k]
// with weight w[k], source value su[k], target record cur[k] already loaded).
// All CASes are issued before any result is used, then all stamp exchanges,
// then one warp-wide append for every new frontier entry of the warp: the
// success path costs three round trips per N edges instead of three per edge.
template <int A, int N>
__device__ __forceinline__ void relax_batch(const DevGraph &g, const bool (&on)[N], const uint32_t (&u)[N],
                                            const uint32_t (&v)[N], const uint32_t (&w)[N],
                                            const uint64_t (&su)[N], ulonglong2 (&cur)[N], uint32_t st,
                                            uint32_t *fout, unsigned long long *fout_n, unsigned long long &local,
                                            uint32_t mst) {
  bool pend[N], upd[N];
  ulonglong2 want[N], old[N];
#pragma unroll
  for (int k = 0; k < N; k++) {
    const uint64_t nv = Hook<A>::combine(su[k], w[k]);
    pend[k] = on[k] && Hook<A>::better(nv, cur[k].x);
    want[k] = make_ulonglong2(nv, pack_parent(u[k], w[k]));
    upd[k] = false;
  }
#pragma unroll
  for (int k = 0; k < N; k++)
    if (pend[k]) old[k] = cas128(&g.lab[v[k]], cur[k], want[k]);
#pragma unroll
  for (int k = 0; k < N; k++) {
    if (!pend[k]) continue;
    if (old[k].x == cur[k].x && old[k].y == cur[k].y) {
      upd[k] = true;
      continue;
    }
    cur[k] = old[k];
    while (Hook<A>::better(want[k].x, cur[k].x)) {  // lost a race: retry while still better
      ulonglong2 o = cas128(&g.lab[v[k]], cur[k], want[k]);
      if (o.x == cur[k].x && o.y == cur[k].y) {
        upd[k] = true;
        break;
      }
      cur[k] = o;
    }
  }
  uint32_t ex[N];
#pragma unroll
  for (int k = 0; k < N; k++)
    if (upd[k]) ex[k] = atomicExch(&g.stamp[v[k]], st);
  uint32_t cnt = 0;
#pragma unroll
  for (int k = 0; k < N; k++) {
    local += upd[k];
    cnt += (upd[k] && ex[k] != st);
  }
  // one atomic per warp for all new entries
  uint32_t incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(FULL, incl, o);
    if (lane_id() >= o) incl += t;
  }
  const uint32_t total = __shfl_sync(FULL, incl, 31);
  if (total) {
    unsigned long long base = 0;
    if (lane_id() == 31) base = atomicAdd(fout_n, (unsigned long long)total);
    base = __shfl_sync(FULL, base, 31) + (incl - cnt);
#pragma unroll
    for (int k = 0; k < N; k++)
      if (upd[k] && ex[k] != st) fout[base++] = v[k];
  }
  if (mst) {
#pragma unroll
    for (int k = 0; k < N; k++) mark_modified(g, upd[k], v[k], mst);
  }
}

// ---- edge-balanced push for large frontiers -------------------------------
// The frontier's degrees are prefix-summed (P), the concatenated edge range
// [0, P[n]) is cut into LB_TILE-edge tiles, and each CTA takes whole tiles:
// the frontier entries a tile touches are staged in shared memory, and each
// thread relaxes LB_ITEMS edges strided by the block size (coalesced pool
// reads).  The edge loads of a thread are all issued before the label loads,
// and those before any CAS, so each thread keeps LB_ITEMS independent memory
// round trips in flight instead of one.
constexpr int LB_TPB = 256;
constexpr int LB_ITEMS = 4;
constexpr uint32_t LB_TILE = LB_TPB * LB_ITEMS;
constexpr uint32_t LB_CAP = 1025;  // staged entries per tile (sparser tiles search P in global memory)

__global__ void k_gather_deg(DevGraph g, const uint32_t *fin, uint64_t n, uint64_t *deg) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= n; i += stride)
    deg[i] = i < n ? seg_len(g.out, fin[i]) : 0;
}

// tile_lo[t] = last frontier index whose edge range starts at or before t*LB_TILE.
__global__ void k_partition(const uint64_t *P, uint64_t n, uint32_t *tile_lo) {
  const uint64_t T = P[n];
  const uint64_t ntiles = (T + LB_TILE - 1) / LB_TILE;
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t <= ntiles; t += stride) {
    uint64_t x = t < ntiles ? t * LB_TILE : T;
    uint64_t lo = 0, hi = n;  // largest i in [0, n] with P[i] <= x
    while (lo < hi) {
      uint64_t mid = (lo + hi + 1) >> 1;
      if (__ldg(&P[mid]) <= x) lo = mid;
      else hi = mid - 1;
    }
    tile_lo[t] = (uint32_t)(lo < n ? lo : (n ? n - 1 : 0));
  }
}

template <int A, bool W>
__global__ void __launch_bounds__(LB_TPB, 3) k_push_lbs(DevGraph g, const uint32_t *fin, uint64_t n, const uint64_t *P,
                                                     const uint32_t *tile_lo, uint32_t *fout,
                                                     unsigned long long *fout_n, uint32_t st, uint32_t mst) {
  using P_ = PoolT<W>;
  const typename P_::E *pool = reinterpret_cast<const typename P_::E *>(g.out.pool);
  __shared__ uint32_t s_rel[LB_CAP];
  __shared__ uint32_t s_u[LB_CAP];
  __shared__ uint64_t s_base[LB_CAP];
  __shared__ uint64_t s_su[LB_CAP];
  const uint64_t T = P[n];
  const uint64_t ntiles = (T + LB_TILE - 1) / LB_TILE;
  unsigned long long local = 0;
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint64_t t0 = t * LB_TILE;
    const uint64_t t1 = min(t0 + LB_TILE, T);
    const uint32_t lo = tile_lo[t];
    const uint32_t hi = tile_lo[t + 1];
    const uint32_t m = hi - lo + 1;
    const bool staged = m <= LB_CAP;
    if (staged) {
      for (uint32_t j = threadIdx.x; j < m; j += LB_TPB) {
        uint64_t pj = P[lo + j];
        uint32_t u = fin[lo + j];
        s_rel[j] = pj <= t0 ? 0u : (uint32_t)(pj - t0);
        s_u[j] = u;
        s_base[j] = g.out.off[u] - pj;
        s_su[j] = ld_val(&g.lab[u]);
      }
    }
    __syncthreads();
    uint64_t slot[LB_ITEMS], su[LB_ITEMS];
    uint32_t uu[LB_ITEMS];
#pragma unroll
    for (int k = 0; k < LB_ITEMS; k++) {
      const uint64_t e = t0 + (uint64_t)k * LB_TPB + threadIdx.x;
      slot[k] = ~0ull;
      if (e < t1) {
        uint32_t j;
        if (staged) {
          const uint32_t er = (uint32_t)(e - t0);
          uint32_t a = 0, b = m - 1;  // largest j with s_rel[j] <= er
          while (a < b) {
            uint32_t mid = (a + b + 1) >> 1;
            if (s_rel[mid] <= er) a = mid;
            else b = mid - 1;
          }
          j = a;
          slot[k] = s_base[j] + e;
          uu[k] = s_u[j];
          su[k] = s_su[j];
        } else {
          uint64_t a = lo, b = hi;  // many empty entries: search P directly
          while (a < b) {
            uint64_t mid = (a + b + 1) >> 1;
            if (P[mid] <= e) a = mid;
            else b = mid - 1;
          }
          uint32_t u = fin[a];
          slot[k] = g.out.off[u] + (e - P[a]);
          uu[k] = u;
          su[k] = ld_val(&g.lab[u]);
        }
      }
    }
    bool on[LB_ITEMS];
    uint32_t vv[LB_ITEMS], ww[LB_ITEMS];
#pragma unroll
    for (int k = 0; k < LB_ITEMS; k++) {
      on[k] = false;
      vv[k] = 0;
      ww[k] = 0;
      if (slot[k] != ~0ull) {
        typename P_::E ent = __ldg(&pool[slot[k]]);
        vv[k] = P_::nbr(ent);
        ww[k] = P_::wt(ent);
        on[k] = !(vv[k] & DEAD);
      } else {
        uu[k] = 0;
        su[k] = 0;
      }
    }
    ulonglong2 cur[LB_ITEMS];
#pragma unroll
    for (int k = 0; k < LB_ITEMS; k++) cur[k] = on[k] ? ld_lab(&g.lab[vv[k]]) : make_ulonglong2(0, 0);
    relax_batch<A, LB_ITEMS>(g, on, uu, vv, ww, su, cur, st, fout, fout_n, local, mst);
    __syncthreads();
  }
  warp_add_result(local, &g.ctl[C_RESULT]);
  if (threadIdx.x == 0 && blockIdx.x == 0) atomicAdd(&g.ctl[C_EDGES], T);
}

// ---- edge-centric push for dense levels -----------------------------------
// When the frontier holds a large share of the vertices (the reference switches
// to its dense mode at the same point, core/graph.hpp:334), streaming the whole
// out-pool beats locating every frontier segment: slot i belongs to owner[i]
// and is relaxed when its owner is active in this level (act[owner] == id).
// Reads of owner[] and of the pool are fully coalesced; there is no staging,
// search or barrier, and each thread keeps DN_ITEMS slots in flight.
constexpr int DN_TPB = 256;
constexpr int DN_ITEMS = 4;
constexpr uint64_t DENSE_DIV = 20;  // dense when frontier >= V / DENSE_DIV

__global__ void k_mark_active(const uint32_t *fin, uint64_t n, uint32_t *act, uint32_t id) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) act[fin[i]] = id;
}

template <int A, bool W>
__global__ void __launch_bounds__(DN_TPB, 3) k_push_dense(DevGraph g, const uint32_t *act, uint32_t act_id,
                                                       uint32_t *fout, unsigned long long *fout_n, uint32_t st,
                                                       uint32_t mst) {
  using P_ = PoolT<W>;
  const typename P_::E *pool = reinterpret_cast<const typename P_::E *>(g.out.pool);
  const uint64_t top = *g.out.pool_top;
  const uint64_t slots = top < g.out.pool_cap ? top : g.out.pool_cap;
  const uint64_t tile = (uint64_t)DN_TPB * DN_ITEMS;
  unsigned long long local = 0, scanned = 0;
  for (uint64_t base = blockIdx.x * tile; base < slots; base += (uint64_t)gridDim.x * tile) {
    uint32_t o[DN_ITEMS];
#pragma unroll
    for (int k = 0; k < DN_ITEMS; k++) {
      const uint64_t i = base + (uint64_t)k * DN_TPB + threadIdx.x;
      o[k] = i < slots ? __ldg(&g.out.owner[i]) : NONE;
    }
    bool a[DN_ITEMS];
#pragma unroll
    for (int k = 0; k < DN_ITEMS; k++) a[k] = o[k] != NONE && __ldg(&act[o[k]]) == act_id;
    uint32_t vv[DN_ITEMS], ww[DN_ITEMS];
    uint64_t su[DN_ITEMS];
#pragma unroll
    for (int k = 0; k < DN_ITEMS; k++) {
      vv[k] = 0;
      ww[k] = 0;
      su[k] = 0;
      if (a[k]) {
        typename P_::E ent = __ldg(&pool[base + (uint64_t)k * DN_TPB + threadIdx.x]);
        su[k] = ld_val(&g.lab[o[k]]);
        vv[k] = P_::nbr(ent);
        ww[k] = P_::wt(ent);
        a[k] = !(vv[k] & DEAD);
        scanned++;
      }
    }
    ulonglong2 cur[DN_ITEMS];
#pragma unroll
    for (int k = 0; k < DN_ITEMS; k++) cur[k] = a[k] ? ld_lab(&g.lab[vv[k]]) : make_ulonglong2(0, 0);
    relax_batch<A, DN_ITEMS>(g, a, o, vv, ww, su, cur, st, fout, fout_n, local, mst);
  }
  warp_add_result(local, &g.ctl[C_RESULT]);
  warp_add_result(scanned, &g.ctl[C_EDGES]);
}

// Bottom-up BFS level for full builds (the reference's dense pull,
// core/graph.hpp:936-976, specialised to BFS): every unreached vertex scans
// its in-edges and takes the first in-neighbour at depth d as its parent,
// stopping there.  Used when the frontier is large; each vertex is written
// only by its own thread, so no atomics on labels.
template <bool W>
__global__ void k_bfs_bottom_up(DevGraph g, uint64_t d, uint32_t *fout, unsigned long long *fout_n) {
  using P_ = PoolT<W>;
  const typename P_::E *pool = reinterpret_cast<const typename P_::E *>(g.in.pool);
  const uint64_t V = g.V;
  unsigned long long local = 0, scanned = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x; base < V; base += stride) {
    const uint64_t v = base + threadIdx.x;
    bool found = false;
    if (v < V && ld_val(&g.lab[v]) == BFS_MAXL) {
      const uint32_t len = seg_len(g.in, (uint32_t)v);
      const uint64_t off = g.in.off[v];
      for (uint32_t k = 0; k < len; k++) {
        const typename P_::E e = __ldg(&pool[off + k]);
        const uint32_t u = P_::nbr(e);
        scanned++;
        if (u & DEAD) continue;
        if (ld_val(&g.lab[u]) == d) {
          g.lab[v] = make_ulonglong2(d + 1, pack_parent(u, P_::wt(e)));
          found = true;
          break;
        }
      }
    }
    local += found;
    warp_append(found, (uint32_t)v, fout, fout_n, FULL);
  }
  warp_add_result(local, &g.ctl[C_RESULT]);
  warp_add_result(scanned, &g.ctl[C_EDGES]);
}

// build_tree init (core/graph.hpp:886-896): every label to init_label_func,
// parent to empty; the active set is the root, or every vertex (WCC).
template <int A>
__global__ void k_init(DevGraph g, uint64_t root, uint32_t *fout) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < g.V; v += stride) {
    g.lab[v] = make_ulonglong2(Hook<A>::init(v, root), pack_parent(NONE, 0));
    if (Hook<A>::all_active) fout[v] = (uint32_t)v;
    else if (v == root) fout[0] = (uint32_t)v;
  }
}

// Seed relaxations of update_tree_add (single :1140-1153, batch :1180-1214):
// relax each inserted edge, both orientations when undirected.
template <int A>
__global__ void k_seed_add(DevGraph g, const uint32_t *os, const uint32_t *od, const uint32_t *ow, const uint32_t *cand,
                           const unsigned long long *cand_n, uint64_t n_all, int directed, uint32_t *fout,
                           unsigned long long *fout_n, uint32_t st, uint32_t mst) {
  const uint64_t n = cand ? *cand_n : n_all;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long local = 0;
  for (uint64_t base = warp * 32; base < n; base += nwarps * 32) {
    uint64_t i = base + lane_id();
    for (int dir = 0; dir < (directed ? 1 : 2); dir++) {
      bool upd = false;
      uint32_t v = 0;
      if (i < n) {
        uint64_t e = cand ? cand[i] : i;
        uint64_t op = directed ? e : 2 * e + dir;
        uint32_t u = os[op];
        v = od[op];
        upd = relax<A>(g.lab, u, ld_val(&g.lab[u]), v, ow[op]);
      }
      local += upd;
      bool app = upd && atomicExch(&g.stamp[v], st) != st;
      warp_append(app, v, fout, fout_n, FULL);
      if (mst) mark_modified(g, upd, v, mst);
    }
  }
  warp_add_result(local, &g.ctl[C_RESULT]);
}

// Seeds of update_tree_del (single :1640-1649, batch :1680-1714): a deleted
// edge that is dst's parent edge invalidates dst.
__global__ void k_seed_del(DevGraph g, const uint32_t *os, const uint32_t *od, const uint32_t *ow, const uint32_t *cand,
                           const unsigned long long *cand_n, uint64_t n_all, int directed, uint32_t tag_inv,
                           uint32_t *fout, unsigned long long *fout_n) {
  const uint64_t n = cand ? *cand_n : n_all;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t base = warp * 32; base < n; base += nwarps * 32) {
    uint64_t i = base + lane_id();
    for (int dir = 0; dir < (directed ? 1 : 2); dir++) {
      bool app = false;
      uint32_t v = 0;
      if (i < n) {
        uint64_t e = cand ? cand[i] : i;
        uint64_t op = directed ? e : 2 * e + dir;
        uint32_t u = os[op];
        v = od[op];
        if (ld_meta(&g.lab[v]) == pack_parent(u, ow[op])) app = atomicExch(&g.inv[v], tag_inv) != tag_inv;
      }
      warp_append(app, v, fout, fout_n, FULL);
    }
  }
}

// has_parents (core/graph.hpp:1889-1907): does x's parent chain reach a root
// without meeting a vertex invalidated (or rescued) by this repair?  The chain
// guard (0.1 |V| steps) requests a full recompute, as the reference does.
__device__ __forceinline__ bool has_parents(const DevGraph &g, uint32_t x, uint32_t tag_inv, uint64_t limit) {
  uint64_t num = 0;
  for (;;) {
    uint32_t t = ld_u32(&g.inv[x]);
    if (t == tag_inv || t == tag_inv + 1) return true;
    uint32_t p = (uint32_t)ld_meta(&g.lab[x]);
    if (p == NONE) return false;
    x = p;
    if (++num > limit) {
      atomicExch(&g.ctl[C_RECOMPUTE], 1ull);
      return true;
    }
  }
}

// Rescue (core/graph.hpp:1323-1361): an invalidated dst keeps its value when an
// in-neighbour satisfies equal_func and has a clean parent chain; the parent
// moves to that in-edge.  One warp per frontier vertex.
template <int A, bool W>
__global__ void __launch_bounds__(TPB) k_rescue(DevGraph g, const uint32_t *fin, const unsigned long long *fin_n,
                                                uint32_t tag_inv, uint64_t limit) {
  using P = PoolT<W>;
  const typename P::E *pool = reinterpret_cast<const typename P::E *>(g.in.pool);
  const uint64_t n = *fin_n;
  const int lane = lane_id();
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t idx = warp; idx < n; idx += nwarps) {
    const uint32_t d = fin[idx];
    if (ld_u32(&g.inv[d]) != tag_inv) continue;
    const uint64_t sd = ld_val(&g.lab[d]);
    const uint32_t len = seg_len(g.in, d);
    const uint64_t off = g.in.off[d];
    for (uint32_t kb = 0; kb < len; kb += 32) {
      const uint32_t k = kb + lane;
      bool ok = false;
      uint32_t src = 0, w = 0;
      if (k < len) {
        typename P::E e = pool[off + k];
        src = P::nbr(e);
        w = P::wt(e);
        if (!(src & DEAD) && Hook<A>::combine(ld_val(&g.lab[src]), w) == sd) ok = !has_parents(g, src, tag_inv, limit);
      }
      unsigned b = __ballot_sync(FULL, ok);
      bool done = false;
      while (b) {
        int l = __ffs(b) - 1;
        b &= b - 1;
        bool won = false;
        if (lane == l) {
          won = atomicCAS(&g.inv[d], tag_inv, tag_inv + 1) == tag_inv;
          if (won) reinterpret_cast<unsigned long long *>(&g.lab[d])[1] = pack_parent(src, w);
        }
        won = __shfl_sync(FULL, won, l);
        if (won) { done = true; break; }
      }
      if (done || __shfl_sync(FULL, ld_u32(&g.inv[d]), 0) != tag_inv) break;
    }
  }
}

// Collect and expand (core/graph.hpp:1363-1417): a still-invalid vertex joins
// the reset set; its tree children (parent == (u,w)) are invalidated next.
template <int A, bool W>
__global__ void __launch_bounds__(TPB) k_expand(DevGraph g, const uint32_t *fin, const unsigned long long *fin_n,
                                                uint32_t *tree, uint32_t *fout, unsigned long long *fout_n,
                                                uint32_t tag_inv) {
  using P = PoolT<W>;
  const typename P::E *pool = reinterpret_cast<const typename P::E *>(g.out.pool);
  const uint64_t n = *fin_n;
  const int lane = lane_id();
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t idx = warp; idx < n; idx += nwarps) {
    const uint32_t u = fin[idx];
    if (ld_u32(&g.inv[u]) != tag_inv) continue;
    if (lane == 0) {
      unsigned long long k = atomicAdd(&g.ctl[C_TREEN], 1ull);
      tree[k] = u;
    }
    const uint32_t len = seg_len(g.out, u);
    const uint64_t off = g.out.off[u];
    for (uint32_t kb = 0; kb < len; kb += 32) {
      const uint32_t k = kb + lane;
      bool app = false;
      uint32_t v = 0;
      if (k < len) {
        typename P::E e = pool[off + k];
        v = P::nbr(e);
        if (!(v & DEAD) && ld_meta(&g.lab[v]) == pack_parent(u, P::wt(e))) {
          uint32_t t = ld_u32(&g.inv[v]);
          if (t != tag_inv && t != tag_inv + 1) app = atomicCAS(&g.inv[v], t, tag_inv) == t;
        }
      }
      warp_append(app, v, fout, fout_n, FULL);
    }
  }
}

// Reset the invalid set to init (core/graph.hpp:1420-1430).
template <int A>
__global__ void k_reset(DevGraph g, const uint32_t *tree, const unsigned long long *tree_n, uint64_t root,
                        uint32_t mst) {
  const uint64_t n = *tree_n;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t base = warp * 32; base < n; base += nwarps * 32) {
    uint64_t i = base + lane_id();
    uint32_t u = 0;
    if (i < n) {
      u = tree[i];
      g.lab[u] = make_ulonglong2(Hook<A>::init(u, root), pack_parent(NONE, 0));
    }
    if (mst) mark_modified(g, i < n, u, mst);
  }
}

// One transposed pull over the reset set (core/graph.hpp:1433-1511): each
// vertex takes its best in-neighbour by update_func.  One warp per vertex.
template <int A, bool W>
__global__ void __launch_bounds__(TPB) k_pull(DevGraph g, const uint32_t *fin, const unsigned long long *fin_n,
                                              uint32_t mst) {
  using P = PoolT<W>;
  const typename P::E *pool = reinterpret_cast<const typename P::E *>(g.in.pool);
  const uint64_t n = *fin_n;
  const int lane = lane_id();
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long local = 0;
  for (uint64_t idx = warp; idx < n; idx += nwarps) {
    const uint32_t d = fin[idx];
    const uint32_t len = seg_len(g.in, d);
    const uint64_t off = g.in.off[d];
    uint64_t best = ld_val(&g.lab[d]), bsu = 0;
    uint32_t bsrc = NONE, bw = 0;
    for (uint32_t k = lane; k < len; k += 32) {
      typename P::E e = pool[off + k];
      uint32_t s = P::nbr(e);
      if (s & DEAD) continue;
      uint64_t su = ld_val(&g.lab[s]);
      uint64_t nv = Hook<A>::combine(su, P::wt(e));
      if (Hook<A>::better(nv, best)) { best = nv; bsrc = s; bw = P::wt(e); bsu = su; }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      uint64_t ob = __shfl_down_sync(FULL, best, o);
      uint64_t osu = __shfl_down_sync(FULL, bsu, o);
      uint32_t os = __shfl_down_sync(FULL, bsrc, o);
      uint32_t ow = __shfl_down_sync(FULL, bw, o);
      if (os != NONE && (bsrc == NONE || Hook<A>::better(ob, best))) { best = ob; bsu = osu; bsrc = os; bw = ow; }
    }
    bool upd = false;
    if (lane == 0 && bsrc != NONE) upd = relax<A>(g.lab, bsrc, bsu, d, bw);
    local += upd;
    if (mst) mark_modified(g, __shfl_sync(FULL, upd, 0) && lane == 0, d, mst);
  }
  warp_add_result(local, &g.ctl[C_RESULT]);
}

// need_update_tree_add (core/graph.hpp:987-1000) / need_update_tree_del
// (:1220-1233) per edge.
template <int A>
__global__ void k_classify(DevGraph g, const uint32_t *os, const uint32_t *od, const uint32_t *ow, uint64_t n,
                           int directed, const uint8_t *is_del, uint8_t *unsafe) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    bool del = is_del && is_del[i];
    bool r = false;
    for (int dir = 0; dir < (directed ? 1 : 2); dir++) {
      uint64_t op = directed ? i : 2 * i + dir;
      uint32_t u = os[op], v = od[op], w = ow[op];
      if (del) r = r || ld_meta(&g.lab[v]) == pack_parent(u, w);
      else r = r || Hook<A>::better(Hook<A>::combine(ld_val(&g.lab[u]), w), ld_val(&g.lab[v]));
    }
    unsafe[i] = r;
  }
}

__global__ void k_unpack_labels(DevGraph g, uint64_t *val, uint64_t *par, uint64_t *pw) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < g.V; v += stride) {
    ulonglong2 l = g.lab[v];
    if (val) val[v] = l.x;
    uint32_t p = (uint32_t)l.y;
    if (par) par[v] = p == NONE ? (uint64_t)g.V : (uint64_t)p;
    if (pw) pw[v] = p == NONE ? 0 : (l.y >> 32);
  }
}

__global__ void k_checksum(DevGraph g) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long h = 0;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < g.V; v += stride)
    h += splitmix64(g.lab[v].x ^ (v * 0x9E3779B97F4A7C15ull));
  for (int o = 16; o; o >>= 1) h += __shfl_down_sync(FULL, h, o);
  if (lane_id() == 0) atomicAdd(&g.ctl[C_CHECKSUM], h);
}

// ---------------------------------------------------------------- host side

int grid_warps(const Graph &g, uint64_t warps) {
  uint64_t b = (warps * 32 + TPB - 1) / TPB;
  uint64_t cap = (uint64_t)g.num_sms * 16;
  if (b > cap) b = cap;
  return (int)(b ? b : 1);
}

uint32_t next_stamp(Graph &g) {
  if (++g.stamp_epoch == 0xFFFFFFFFu) {
    cudaMemsetAsync(g.d.stamp, 0, (size_t)g.V * 4, g.stream);
    g.stamp_epoch = 1;
  }
  return g.stamp_epoch;
}

uint32_t mod_stamp(Graph &g) { return g.trace ? g.mod_epoch : 0u; }

int read_ctl(Graph &g) {
  RG_CUDA(cudaMemcpyAsync(g.h_ctl, g.d.ctl, sizeof(unsigned long long) * C_COUNT, cudaMemcpyDeviceToHost, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  return RG_OK;
}

// Push levels to a fixpoint from the frontier (fin, *fin_n) with n0 entries
// (do_update_tree_add, core/graph.hpp:1013-1111; build_tree :898-983).
template <int A, bool W>
int push_levels(Graph &g, const uint32_t *fin, unsigned long long *fin_n, uint64_t n0, bool bfs_levels = false) {
  const uint32_t *cur = fin;
  unsigned long long *cur_n = fin_n;
  uint64_t n = n0;
  unsigned long long *hub_n = &g.d.ctl[C_HUBN];
  // Values move monotonically, so levels are bounded; the cap only turns a
  // logic error into a status instead of an endless loop.
  const uint64_t max_levels = 4 * (uint64_t)g.V + 1024;
  for (uint64_t lvl = 0; n; lvl++) {
    if (lvl > max_levels) {
      set_error("push levels did not converge");
      return RG_ETIMEOUT;
    }
    g.st_frontier.push_back(n);
    int nb = (cur == g.q[0]) ? 1 : 0;
    uint32_t *next = g.q[nb];
    unsigned long long *next_n = &g.d.ctl[C_QN0 + nb];
    RG_CUDA(cudaMemsetAsync(next_n, 0, 8, g.stream));
    RG_CUDA(cudaMemsetAsync(hub_n, 0, 8, g.stream));
    uint32_t st = next_stamp(g);
    if (g.profiling) RG_CUDA(cudaEventRecord(g.pev[0], g.stream));
    if (A == RG_BFS && bfs_levels && n * DENSE_DIV >= g.V) {
      // full BFS build: the frontier is exactly depth lvl; pull bottom-up
      count_launch(g);
      k_bfs_bottom_up<W><<<g.num_sms * 8, TPB, 0, g.stream>>>(g.d, lvl, next, next_n);
    } else if (n * DENSE_DIV >= g.V) {
      if (++g.act_epoch == 0xFFFFFFFFu) {
        RG_CUDA(cudaMemsetAsync(g.act, 0, (size_t)g.V * 4, g.stream));
        g.act_epoch = 1;
      }
      count_launch(g, 2);
      k_mark_active<<<grid_warps(g, (n + 31) / 32), TPB, 0, g.stream>>>(cur, n, g.act, g.act_epoch);
      k_push_dense<A, W><<<g.num_sms * 3, DN_TPB, 0, g.stream>>>(g.d, g.act, g.act_epoch, next, next_n, st,
                                                                 mod_stamp(g));
    } else if (n >= LBS_MIN_FRONTIER) {
      count_launch(g, 4);
      k_gather_deg<<<grid_warps(g, (n + 32) / 32), TPB, 0, g.stream>>>(g.d, cur, n, g.scratch64);
      size_t tb = g.cub_tmp_bytes;
      RG_CUDA(cub::DeviceScan::ExclusiveSum(g.cub_tmp, tb, g.scratch64, g.lb_P, n + 1, g.stream));
      k_partition<<<g.num_sms * 4, TPB, 0, g.stream>>>(g.lb_P, n, g.lb_tile);
      k_push_lbs<A, W><<<g.num_sms * 3, LB_TPB, 0, g.stream>>>(g.d, cur, n, g.lb_P, g.lb_tile, next, next_n, st,
                                                               mod_stamp(g));
    } else {
      count_launch(g, 2);
      k_push<A, W><<<grid_warps(g, (n + 31) / 32), TPB, 0, g.stream>>>(g.d, cur, cur_n, next, next_n, st, g.hubq,
                                                                        hub_n, mod_stamp(g));
      k_push_hub<A, W><<<g.num_sms * 8, TPB, 0, g.stream>>>(g.d, g.hubq, hub_n, next, next_n, st, mod_stamp(g));
    }
    RG_CUDA(cudaGetLastError());
    if (g.profiling) RG_CUDA(cudaEventRecord(g.pev[1], g.stream));
    int rc = read_ctl(g);
    if (rc) return rc;
    if (g.profiling) {
      float ms = 0.f;
      RG_CUDA(cudaEventElapsedTime(&ms, g.pev[0], g.pev[1]));
      g.prof_ms += ms;
      g.prof_launches += 1;
      g.st_level_ms.push_back(ms);
    }
    n = g.h_ctl[C_QN0 + nb];
    cur = next;
    cur_n = next_n;
    g.st_levels++;
  }
  return RG_OK;
}

template <int A, bool W>
int build_impl(Graph &g, uint64_t root) {
  RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_RESULT], 0, 8, g.stream));
  RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_QN0], 0, 8, g.stream));
  count_launch(g);
  k_init<A><<<g.num_sms * 16, TPB, 0, g.stream>>>(g.d, root, g.q[0]);
  RG_CUDA(cudaGetLastError());
  uint64_t n0 = Hook<A>::all_active ? g.V : 1;
  unsigned long long hn = n0;
  RG_CUDA(cudaMemcpyAsync(&g.d.ctl[C_QN0], &hn, 8, cudaMemcpyHostToDevice, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  if (g.trace) {
    // every label is rewritten; the modified list becomes "all vertices" lazily
    // through the same dedup stamps.
  }
  return push_levels<A, W>(g, g.q[0], &g.d.ctl[C_QN0], n0, /*bfs_levels=*/true);
}

template <int A, bool W>
int add_impl(Graph &g, uint64_t n_edges, int directed, bool from_cands) {
  RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_RESULT], 0, 8, g.stream));
  RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_QN0], 0, 8, g.stream));
  uint32_t st = next_stamp(g);
  count_launch(g);
  k_seed_add<A><<<grid_warps(g, (n_edges + 31) / 32), TPB, 0, g.stream>>>(
      g.d, op_src(g), op_dst(g), op_w(g), from_cands ? op_cand(g) : nullptr, &g.d.ctl[C_CANDN], n_edges, directed,
      g.q[0], &g.d.ctl[C_QN0], st, mod_stamp(g));
  RG_CUDA(cudaGetLastError());
  int rc = read_ctl(g);
  if (rc) return rc;
  return push_levels<A, W>(g, g.q[0], &g.d.ctl[C_QN0], g.h_ctl[C_QN0]);
}

template <int A, bool W>
int del_impl(Graph &g, uint64_t n_edges, int directed, bool from_cands) {
  RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_RESULT], 0, 8, g.stream));
  RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_QN0], 0, 8, g.stream));
  RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_TREEN], 0, 8, g.stream));
  RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_RECOMPUTE], 0, 8, g.stream));
  if (++g.inv_epoch >= 0x7FFFFFFFu) {
    RG_CUDA(cudaMemsetAsync(g.d.inv, 0, (size_t)g.V * 4, g.stream));
    g.inv_epoch = 1;
  }
  const uint32_t tag = 2 * g.inv_epoch;   // tag: invalidated; tag+1: rescued
  count_launch(g);
  k_seed_del<<<grid_warps(g, (n_edges + 31) / 32), TPB, 0, g.stream>>>(
      g.d, op_src(g), op_dst(g), op_w(g), from_cands ? op_cand(g) : nullptr, &g.d.ctl[C_CANDN], n_edges, directed, tag,
      g.q[0], &g.d.ctl[C_QN0]);
  RG_CUDA(cudaGetLastError());
  int rc = read_ctl(g);
  if (rc) return rc;
  uint64_t n = g.h_ctl[C_QN0];
  if (n == 0) return RG_OK;
  const uint64_t limit = (uint64_t)((double)g.V * 0.1);
  const uint64_t big = std::max<uint64_t>((uint64_t)(0.05 * (double)g.V), 2000000);
  const uint32_t *cur = g.q[0];
  unsigned long long *cur_n = &g.d.ctl[C_QN0];
  bool recompute = false;
  for (uint64_t i = 0; n; i++) {
    // full recompute fallback (core/graph.hpp:1252)
    if (i <= 10 && g.h_ctl[C_TREEN] + n > big) { recompute = true; break; }
    int nb = (cur == g.q[0]) ? 1 : 0;
    uint32_t *next = g.q[nb];
    unsigned long long *next_n = &g.d.ctl[C_QN0 + nb];
    RG_CUDA(cudaMemsetAsync(next_n, 0, 8, g.stream));
    count_launch(g, 2);
    k_rescue<A, W><<<grid_warps(g, n), TPB, 0, g.stream>>>(g.d, cur, cur_n, tag, limit);
    k_expand<A, W><<<grid_warps(g, n), TPB, 0, g.stream>>>(g.d, cur, cur_n, g.tree, next, next_n, tag);
    RG_CUDA(cudaGetLastError());
    if ((rc = read_ctl(g))) return rc;
    if (g.h_ctl[C_RECOMPUTE]) { recompute = true; break; }
    n = g.h_ctl[C_QN0 + nb];
    cur = next;
    cur_n = next_n;
    g.st_levels++;
  }
  if (recompute) {
    g.st_recomputes++;
    uint64_t keep = 0;
    RG_CUDA(cudaMemsetAsync(g.d.inv, 0, (size_t)g.V * 4, g.stream));
    g.inv_epoch = 0;
    (void)keep;
    return build_impl<A, W>(g, g.root);
  }
  uint64_t nt = g.h_ctl[C_TREEN];
  g.st_invalidated += nt;
  if (nt == 0) return RG_OK;
  count_launch(g, 2);
  k_reset<A><<<grid_warps(g, (nt + 31) / 32), TPB, 0, g.stream>>>(g.d, g.tree, &g.d.ctl[C_TREEN], g.root,
                                                                   mod_stamp(g));
  k_pull<A, W><<<grid_warps(g, nt), TPB, 0, g.stream>>>(g.d, g.tree, &g.d.ctl[C_TREEN], mod_stamp(g));
  RG_CUDA(cudaGetLastError());
  return push_levels<A, W>(g, g.tree, &g.d.ctl[C_TREEN], nt);
}

template <int A>
int dispatch_w(Graph &g, int what, uint64_t a, int directed, bool from_cands) {
  if (g.weighted) {
    if (what == 0) return build_impl<A, true>(g, a);
    if (what == 1) return add_impl<A, true>(g, a, directed, from_cands);
    return del_impl<A, true>(g, a, directed, from_cands);
  }
  if (what == 0) return build_impl<A, false>(g, a);
  if (what == 1) return add_impl<A, false>(g, a, directed, from_cands);
  return del_impl<A, false>(g, a, directed, from_cands);
}

int dispatch(Graph &g, int algo, int what, uint64_t a, int directed, bool from_cands) {
  switch (algo) {
    case RG_BFS: return dispatch_w<RG_BFS>(g, what, a, directed, from_cands);
    case RG_SSSP: return dispatch_w<RG_SSSP>(g, what, a, directed, from_cands);
    case RG_SSWP: return dispatch_w<RG_SSWP>(g, what, a, directed, from_cands);
    case RG_WCC: return dispatch_w<RG_WCC>(g, what, a, directed, from_cands);
  }
  set_error("unknown algorithm");
  return RG_EINVAL;
}

}  // namespace

int tree_alloc(Graph &g) {
  uint64_t V = g.V;
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
  if ((rc = alloc((void **)&g.d.lab, V * 16 + 16, "labels"))) return rc;
  if ((rc = alloc((void **)&g.d.stamp, V * 4 + 4, "frontier stamps"))) return rc;
  if ((rc = alloc((void **)&g.d.inv, V * 4 + 4, "invalidation tags"))) return rc;
  if ((rc = alloc((void **)&g.d.modstamp, V * 4 + 4, "modified stamps"))) return rc;
  if ((rc = alloc((void **)&g.d.modq, V * 4 + 4, "modified list"))) return rc;
  if ((rc = alloc((void **)&g.q[0], V * 4 + 4, "frontier"))) return rc;
  if ((rc = alloc((void **)&g.q[1], V * 4 + 4, "frontier"))) return rc;
  if ((rc = alloc((void **)&g.tree, V * 4 + 4, "reset set"))) return rc;
  if ((rc = alloc((void **)&g.scratch64, V * 8 + 8, "scratch"))) return rc;
  g.hubq_cap = g.d.out.pool_cap / CHUNK + V / HUB + 1024;
  if ((rc = alloc((void **)&g.hubq, g.hubq_cap * 8, "hub tasks"))) return rc;
  if ((rc = alloc((void **)&g.lb_P, V * 8 + 16, "frontier degree prefix"))) return rc;
  if ((rc = alloc((void **)&g.act, V * 4 + 4, "dense-level activity"))) return rc;
  RG_CUDA(cudaMemset(g.act, 0, V * 4 + 4));
  if ((rc = alloc((void **)&g.lb_tile, (g.d.out.pool_cap / LB_TILE + 4) * 4, "tile partition"))) return rc;
  g.cub_tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, g.cub_tmp_bytes, g.scratch64, g.lb_P, V + 1);
  if ((rc = alloc(&g.cub_tmp, g.cub_tmp_bytes + 256, "scan scratch"))) return rc;
  if ((rc = alloc((void **)&g.d.ctl, sizeof(unsigned long long) * C_COUNT, "control block"))) return rc;
  RG_CUDA(cudaMemset(g.d.ctl, 0, sizeof(unsigned long long) * C_COUNT));
  RG_CUDA(cudaMemset(g.d.stamp, 0, V * 4 + 4));
  RG_CUDA(cudaMemset(g.d.inv, 0, V * 4 + 4));
  RG_CUDA(cudaMemset(g.d.modstamp, 0, V * 4 + 4));
  // labels start as "no parent", value 0 until build_tree (alloc_vertex_tree_array, :255-262)
  RG_CUDA(cudaMemset(g.d.lab, 0, V * 16 + 16));
  for (uint64_t v = 0; v < 1; v++) {}
  return RG_OK;
}

int tree_build(Graph &g, int algo, uint64_t root, uint64_t *total) {
  g.st_levels = g.st_invalidated = g.st_recomputes = 0;
  g.st_frontier.clear();
  g.st_level_ms.clear();
  cudaMemsetAsync(&g.d.ctl[C_EDGES], 0, 8, g.stream);
  g.algo = algo;
  g.root = root;
  int rc = dispatch(g, algo, 0, root, 1, false);
  if (rc) return rc;
  if (total) *total = g.h_ctl[C_RESULT];
  return RG_OK;
}

int tree_add(Graph &g, uint64_t n_edges, int directed, bool from_cands, uint64_t *total) {
  g.st_levels = g.st_invalidated = g.st_recomputes = 0;
  g.st_frontier.clear();
  g.st_level_ms.clear();
  cudaMemsetAsync(&g.d.ctl[C_EDGES], 0, 8, g.stream);
  int rc = dispatch(g, g.algo, 1, n_edges, directed, from_cands);
  if (rc) return rc;
  if (total) *total = g.h_ctl[C_RESULT];
  return RG_OK;
}

int tree_del(Graph &g, uint64_t n_edges, int directed, bool from_cands, uint64_t *total) {
  g.st_levels = g.st_invalidated = g.st_recomputes = 0;
  g.st_frontier.clear();
  g.st_level_ms.clear();
  cudaMemsetAsync(&g.d.ctl[C_EDGES], 0, 8, g.stream);
  int rc = dispatch(g, g.algo, 2, n_edges, directed, from_cands);
  if (rc) return rc;
  if (total) *total = g.h_ctl[C_RESULT];
  return RG_OK;
}

int tree_classify(Graph &g, uint64_t n, int directed, const uint8_t *is_del_dev, uint8_t *unsafe_dev) {
  int grid = grid_warps(g, (n + 31) / 32);
  count_launch(g);
  switch (g.algo) {
    case RG_BFS: k_classify<RG_BFS><<<grid, TPB, 0, g.stream>>>(g.d, op_src(g), op_dst(g), op_w(g), n, directed, is_del_dev, unsafe_dev); break;
    case RG_SSSP: k_classify<RG_SSSP><<<grid, TPB, 0, g.stream>>>(g.d, op_src(g), op_dst(g), op_w(g), n, directed, is_del_dev, unsafe_dev); break;
    case RG_SSWP: k_classify<RG_SSWP><<<grid, TPB, 0, g.stream>>>(g.d, op_src(g), op_dst(g), op_w(g), n, directed, is_del_dev, unsafe_dev); break;
    default: k_classify<RG_WCC><<<grid, TPB, 0, g.stream>>>(g.d, op_src(g), op_dst(g), op_w(g), n, directed, is_del_dev, unsafe_dev); break;
  }
  RG_CUDA(cudaGetLastError());
  return RG_OK;
}

int tree_labels(Graph &g, uint64_t *val, uint64_t *par, uint64_t *pw) {
  uint64_t *outs[3] = {val, par, pw};
  for (int k = 0; k < 3; k++) {
    if (!outs[k]) continue;
    count_launch(g);
    k_unpack_labels<<<g.num_sms * 8, TPB, 0, g.stream>>>(g.d, k == 0 ? g.scratch64 : nullptr,
                                                          k == 1 ? g.scratch64 : nullptr, k == 2 ? g.scratch64 : nullptr);
    RG_CUDA(cudaGetLastError());
    RG_CUDA(cudaMemcpyAsync(outs[k], g.scratch64, g.V * 8, cudaMemcpyDeviceToHost, g.stream));
  }
  RG_CUDA(cudaStreamSynchronize(g.stream));
  return RG_OK;
}

int tree_checksum(Graph &g, uint64_t *sum) {
  RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_CHECKSUM], 0, 8, g.stream));
  count_launch(g);
  k_checksum<<<g.num_sms * 8, TPB, 0, g.stream>>>(g.d);
  RG_CUDA(cudaGetLastError());
  int rc = read_ctl(g);
  if (rc) return rc;
  *sum = g.h_ctl[C_CHECKSUM];
  return RG_OK;
}

}  // namespace rg
