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
#include <cstring>
#include <type_traits>

#include <cooperative_groups.h>
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "rg_internal.cuh"
#include "rg_storage_dev.cuh"

namespace rg {

namespace {

constexpr int TPB = 256;
constexpr uint32_t HUB = 64;     // longer lists of a small frontier are split into
constexpr uint32_t CHUNK = 64;   // CHUNK-slot tasks so no warp walks a long list alone

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
__device__ __forceinline__ bool relax(const DevGraph &g, uint32_t u, uint64_t su, uint32_t v, uint32_t w) {
  const uint64_t nv = Hook<A>::combine(su, w);
  if (!Hook<A>::better(nv, ld_v32(g.val32, v))) return false;
  ulonglong2 cur = ld_lab(&g.lab[v]);
  while (Hook<A>::better(nv, cur.x)) {
    ulonglong2 want = make_ulonglong2(nv, pack_parent(u, w));
    ulonglong2 old = cas128(&g.lab[v], cur, want);
    if (old.x == cur.x && old.y == cur.y) {
      mirror_improve<A>(g.val32, v, nv);
      return true;
    }
    cur = old;
  }
  return false;
}

// relax without the 4-byte value filter: the label itself is the first load,
// so that an improving edge costs two round trips (load, CAS) instead of
// three.  For latency-bound single-CTA levels, where the filter saves no
// bandwidth worth having.
template <int A>
__device__ __forceinline__ bool relax_lab(const DevGraph &g, uint32_t u, uint64_t su, uint32_t v, uint32_t w) {
  const uint64_t nv = Hook<A>::combine(su, w);
  ulonglong2 cur = ld_lab(&g.lab[v]);
  while (Hook<A>::better(nv, cur.x)) {
    ulonglong2 want = make_ulonglong2(nv, pack_parent(u, w));
    ulonglong2 old = cas128(&g.lab[v], cur, want);
    if (old.x == cur.x && old.y == cur.y) {
      mirror_improve<A>(g.val32, v, nv);
      return true;
    }
    cur = old;
  }
  return false;
}

__device__ __forceinline__ void warp_add_result(unsigned long long local, unsigned long long *dst) {
  for (int o = 16; o; o >>= 1) local += __shfl_down_sync(FULL, local, o);
  if (lane_id() == 0 && local) atomicAdd(dst, local);
}

// Record v in the modified list (trace_modified graphs); the epoch is read
// from the control block so cached graphs follow rg_clear_modified.
__device__ __forceinline__ void mark_modified(const DevGraph &g, bool pred, uint32_t v, uint32_t /*on*/) {
  const uint32_t mst = (uint32_t)g.ctl[C_MODEPOCH];
  bool app = pred && atomicExch(&g.modstamp[v], mst) != mst;
  warp_append(app, v, g.modq, &g.ctl[C_MODN], FULL);
}

// One push level over a frontier list (stream_edges / stream_edges_sparse
// push lambdas, core/graph.hpp:910-935, :1017-1042, :1083-1104).
template <int A, bool W>
__global__ void __launch_bounds__(TPB) k_push(DevGraph g, const uint32_t *fin, const unsigned long long *fin_n,
                                              uint32_t *fout, unsigned long long *fout_n, uint64_t *hubq,
                                              unsigned long long *hub_n, uint32_t mst) {
  if (g.ctl[C_MODE] != M_SPARSE) return;
  const uint32_t st = (uint32_t)g.ctl[C_STAMP];
  using P = PoolT<W>;
  const typename P::E *pool = reinterpret_cast<const typename P::E *>(g.out.pool);
  const uint64_t n = *fin_n;
  const int lane = lane_id();
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long local = 0, scanned = 0;
  // vertices per warp: as few as the frontier allows (at most 32), so that a
  // frontier smaller than 32 x the grid's warps still spreads over every warp
  // instead of leaving a few warps to walk 32 lists each
  const uint64_t per = (n + nwarps - 1) / nwarps;
  const uint32_t vpw = per >= 32 ? 32u : (per ? (uint32_t)per : 1u);
  for (uint64_t base = warp * vpw; base < n; base += nwarps * vpw) {
    uint64_t i = base + lane;
    uint32_t u = 0, len = 0;
    uint64_t off = 0, su = 0;
    uint32_t hub_c = 0;            // tasks of this lane's hub list
    unsigned long long hub_k = 0;  // where they go in the task queue
    if (lane < vpw && i < n) {
      u = fin[i];
      len = seg_len(g.out, u);
      off = g.out.off[u];
      su = ld_v32(g.val32, u);
      if (len > HUB) {
        hub_c = (len + CHUNK - 1) / CHUNK;
        hub_k = atomicAdd(hub_n, (unsigned long long)hub_c);
        len = 0;
      }
    }
    // the whole warp writes each hub's task list (a hub of 100K slots has 1,563
    // tasks: one lane writing them alone took longer than the rest of the level)
    for (unsigned hm = __ballot_sync(FULL, hub_c != 0); hm; hm &= hm - 1) {
      const int src = __ffs(hm) - 1;
      const uint32_t hu = __shfl_sync(FULL, u, src), hc = __shfl_sync(FULL, hub_c, src);
      const unsigned long long hk = __shfl_sync(FULL, hub_k, src);
      for (uint32_t c = lane; c < hc; c += 32) hubq[hk + c] = (uint64_t)hu | ((uint64_t)c << 32);
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
          upd = relax<A>(g,ou, osu, v, P::wt(e));
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
                                                  uint32_t *fout, unsigned long long *fout_n, uint32_t mst) {
  if (g.ctl[C_MODE] != M_SPARSE) return;
  const uint32_t st = (uint32_t)g.ctl[C_STAMP];
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
    const uint64_t su = ld_v32(g.val32, u);
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
          upd = relax<A>(g,u, su, v, P::wt(e));
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
// with weight w[k], source value su[k]), in two steps.
// relax_filter reads the 32-bit value mirror of every target and keeps the
// candidates whose update_func value improves it; it returns whether any lane
// of the warp kept one, so a warp whose candidates all fail (the common case
// in late levels) skips the commit entirely.
template <int A, int N>
__device__ __forceinline__ bool relax_filter(const DevGraph &g, bool (&on)[N], const uint32_t (&v)[N],
                                             const uint32_t (&w)[N], const uint64_t (&su)[N]) {
  uint64_t dv[N];
#pragma unroll
  for (int k = 0; k < N; k++) dv[k] = on[k] ? ld_v32(g.val32, v[k]) : 0;
  bool any = false;
#pragma unroll
  for (int k = 0; k < N; k++) {
    on[k] = on[k] && Hook<A>::better(Hook<A>::combine(su[k], w[k]), dv[k]);
    any |= on[k];
  }
  return __any_sync(FULL, any);
}

// relax_commit (all lanes of the warp): issues every CAS of the kept
// candidates before any result is used, then the stamp exchanges, then one
// warp-wide append for every new frontier entry of the warp, so the success
// path costs three round trips per N edges instead of three per edge.
template <int A, int N>
__device__ __forceinline__ void relax_commit(const DevGraph &g, const bool (&on)[N], const uint32_t (&u)[N],
                                             const uint32_t (&v)[N], const uint32_t (&w)[N],
                                             const uint64_t (&su)[N], uint32_t st, uint32_t *fout,
                                             unsigned long long *fout_n, unsigned long long &local, uint32_t mst) {
  bool pend[N], upd[N];
  ulonglong2 want[N], old[N], cur[N];
#pragma unroll
  for (int k = 0; k < N; k++) {
    pend[k] = on[k];
    want[k] = make_ulonglong2(Hook<A>::combine(su[k], w[k]), pack_parent(u[k], w[k]));
    upd[k] = false;
  }
#pragma unroll
  for (int k = 0; k < N; k++) cur[k] = pend[k] ? ld_lab(&g.lab[v[k]]) : make_ulonglong2(0, 0);
#pragma unroll
  for (int k = 0; k < N; k++) pend[k] = pend[k] && Hook<A>::better(want[k].x, cur[k].x);
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
    if (upd[k]) {
      mirror_improve<A>(g.val32, v[k], want[k].x);
      ex[k] = atomicExch(&g.stamp[v[k]], st);
    }
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

template <int A, int N>
__device__ __forceinline__ void relax_batch(const DevGraph &g, const bool (&on)[N], const uint32_t (&u)[N],
                                            const uint32_t (&v)[N], const uint32_t (&w)[N],
                                            const uint64_t (&su)[N], uint32_t st, uint32_t *fout,
                                            unsigned long long *fout_n, unsigned long long &local, uint32_t mst) {
  bool keep[N];
#pragma unroll
  for (int k = 0; k < N; k++) keep[k] = on[k];
  if (relax_filter<A, N>(g, keep, v, w, su)) relax_commit<A, N>(g, keep, u, v, w, su, st, fout, fout_n, local, mst);
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

// Exclusive prefix of the frontier's degrees into P[0..n] (P[n] = total),
// with n read on the device: every block owns one contiguous range; pass 1
// sums the ranges, pass 2 scans the range sums in one block, pass 3 scans
// each range with its offset.
constexpr int SC_BLOCKS = 512;
constexpr int SC_TPB = 256;

__device__ __forceinline__ void scan_range(uint64_t n1, int b, uint64_t &lo, uint64_t &hi) {
  const uint64_t per = (n1 + SC_BLOCKS - 1) / SC_BLOCKS;
  lo = min(n1, (uint64_t)b * per);
  hi = min(n1, lo + per);
}

__global__ void __launch_bounds__(SC_TPB) k_scan_sums(DevGraph g, const uint32_t *fin,
                                                      const unsigned long long *fin_n, uint64_t *deg,
                                                      uint64_t *sums) {
  using BR = cub::BlockReduce<uint64_t, SC_TPB>;
  __shared__ typename BR::TempStorage tmp;
  const uint64_t n = *fin_n;
  uint64_t lo, hi;
  scan_range(n + 1, blockIdx.x, lo, hi);
  uint64_t s = 0;
  for (uint64_t i = lo + threadIdx.x; i < hi; i += SC_TPB) {
    const uint64_t d = i < n ? seg_len(g.out, fin[i]) : 0;
    deg[i] = d;
    s += d;
  }
  s = BR(tmp).Sum(s);
  if (threadIdx.x == 0) sums[blockIdx.x] = s;
}

__global__ void __launch_bounds__(SC_BLOCKS) k_scan_top(uint64_t *sums) {
  using BS = cub::BlockScan<uint64_t, SC_BLOCKS>;
  __shared__ typename BS::TempStorage tmp;
  uint64_t v = sums[threadIdx.x];
  BS(tmp).ExclusiveSum(v, v);
  sums[threadIdx.x] = v;
}

__global__ void __launch_bounds__(SC_TPB) k_scan_final(const unsigned long long *fin_n, const uint64_t *deg,
                                                       const uint64_t *sums, uint64_t *P) {
  using BS = cub::BlockScan<uint64_t, SC_TPB>;
  __shared__ typename BS::TempStorage tmp;
  __shared__ uint64_t carry;
  const uint64_t n = *fin_n;
  uint64_t lo, hi;
  scan_range(n + 1, blockIdx.x, lo, hi);
  if (threadIdx.x == 0) carry = sums[blockIdx.x];
  __syncthreads();
  for (uint64_t base = lo; base < hi; base += SC_TPB) {
    const uint64_t i = base + threadIdx.x;
    uint64_t d = i < hi ? deg[i] : 0, x, total;
    BS(tmp).ExclusiveSum(d, x, total);
    if (i < hi) P[i] = carry + x;
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
}

// tile_lo[t] = last frontier index whose edge range starts at or before t*LB_TILE.
__global__ void k_partition(const uint64_t *P, const unsigned long long *fin_n, uint32_t *tile_lo) {
  const uint64_t n = *fin_n;
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
__global__ void __launch_bounds__(LB_TPB, 3) k_push_lbs(DevGraph g, const uint32_t *fin,
                                                     const unsigned long long *fin_n, const uint64_t *P,
                                                     const uint32_t *tile_lo, uint32_t *fout,
                                                     unsigned long long *fout_n, uint32_t mst) {
  const uint64_t n = *fin_n;
  const uint32_t st = (uint32_t)g.ctl[C_STAMP];
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
        s_su[j] = ld_v32(g.val32, u);
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
          su[k] = ld_v32(g.val32, u);
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
    relax_batch<A, LB_ITEMS>(g, on, uu, vv, ww, su, st, fout, fout_n, local, mst);
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

__global__ void k_mark_active(DevGraph g, const uint32_t *fin, const unsigned long long *fin_n, uint32_t *act) {
  if (g.ctl[C_MODE] != M_DENSE_PUSH) return;
  const uint32_t id = (uint32_t)g.ctl[C_ACT];
  const uint64_t n = *fin_n;
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) act[fin[i]] = id;
}

template <int A, bool W>
__global__ void __launch_bounds__(DN_TPB, 3) k_push_dense(DevGraph g, const uint32_t *act, uint32_t *fout,
                                                       unsigned long long *fout_n, uint32_t mst) {
  if (g.ctl[C_MODE] != M_DENSE_PUSH) return;
  const uint32_t act_id = (uint32_t)g.ctl[C_ACT];
  const uint32_t st = (uint32_t)g.ctl[C_STAMP];
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
    bool a[DN_ITEMS], any = false;
#pragma unroll
    for (int k = 0; k < DN_ITEMS; k++) {
      a[k] = o[k] != NONE && __ldg(&act[o[k]]) == act_id;
      any |= a[k];
    }
    if (!__any_sync(FULL, any)) continue;  // no active owner in the warp's slots
    uint32_t vv[DN_ITEMS], ww[DN_ITEMS];
    uint64_t su[DN_ITEMS];
#pragma unroll
    for (int k = 0; k < DN_ITEMS; k++) {
      vv[k] = 0;
      ww[k] = 0;
      su[k] = 0;
      if (a[k]) {
        typename P_::E ent = __ldg(&pool[base + (uint64_t)k * DN_TPB + threadIdx.x]);
        su[k] = ld_v32(g.val32, o[k]);
        vv[k] = P_::nbr(ent);
        ww[k] = P_::wt(ent);
        a[k] = !(vv[k] & DEAD);
        scanned++;
      }
    }
    relax_batch<A, DN_ITEMS>(g, a, o, vv, ww, su, st, fout, fout_n, local, mst);
  }
  warp_add_result(local, &g.ctl[C_RESULT]);
  warp_add_result(scanned, &g.ctl[C_EDGES]);
}

// ---- dense pull over in-edges ----------------------------------------------
// The reference's dense mode (stream_edges dense lambda, core/graph.hpp:936-976):
// every vertex takes the best update_func value over its in-edges.  For full
// builds the live in-edges are copied once per adjacency version into a sliced
// ELLPACK layout (SELL-32): rows sorted by length, 32 consecutive rows per
// slice, a slice stored column-major so that lane l of a warp reads row l and
// the 32 lanes of a warp read 32 consecutive entries.  A row is a vertex's
// in-list, or for a hub (in-list longer than PULL_HUB) one of the equal pieces
// its list is cut into, so every row holds at most PULL_HUB entries and the
// warps stay balanced.  A pull level is one warp per slice with no search and
// no atomics on labels: a vertex row is written only by its own lane; a piece
// leaves its best in a side array and k_pull_hub_fix combines the pieces of
// each hub.
constexpr uint32_t PULL_HUB = 576;
constexpr int PS_TPB = 256;
// Split pull levels (RG_OPT_PULL_SPLIT): a level runs in two launches, first
// the slices of the longest in-lists (width >= PULL_SPLIT: the hubs and their
// pieces), then k_pull_hub_fix, then every other slice.  The second launch
// reads the hubs' values of this level (a value cached in L1 by the first
// launch is not carried into the second), where one launch reads them stale
// from L1 for most of the level, so values move along hub paths faster and
// fewer levels pull.  On RMAT-22 the WCC build pulls 2 levels instead of 3
// (1.15 ms against 1.47 unsplit), SSSP 4 instead of 5 (3.96 x E entries read
// against 4.88; 1.70 ms against 1.73).  The first launch has few, long slices
// and leaves part of the GPU idle at its end; SSWP, whose values settle in
// fewer levels anyway, loses more there than it saves (2.05 ms against 1.89),
// so by default SSSP and WCC split and SSWP does not.  Pieces of at most 576
// entries and a split at width 288 keep the first launch within one wave of
// resident warps (2,168 slices for 2,368 warps on RMAT-22; with 512 / 256 it
// was 2,590 slices, and its last warp ran 42 iterations instead of 36).
// Without the split the level is one launch over every slice, k_pull_hub_fix,
// and an empty launch (every level runs the same three kernels).
constexpr uint32_t PULL_SPLIT = 288;
// every hub piece (at least PULL_HUB / 2 entries) must fall in the first launch
static_assert(PULL_SPLIT <= PULL_HUB / 2, "hub pieces must be pulled before k_pull_hub_fix");
// In-list entries a lane keeps in flight: 16 for 8-byte weighted entries; 8 for
// 4-byte ones, plus the next 8 prefetched (measured best on RMAT-22).
template <bool W>
struct PullDepth {
  static constexpr int N = W ? 16 : 8;
  static constexpr bool prefetch = !W;
};

template <bool W>
struct SellE;
template <>
struct SellE<true> {
  using E = uint2;
  static __device__ __forceinline__ E none() { return make_uint2(NONE, 0u); }
  static __device__ __forceinline__ E make(uint32_t u, uint32_t w) { return make_uint2(u, w); }
  static __device__ __forceinline__ uint32_t nbr(E e) { return e.x; }
  static __device__ __forceinline__ uint32_t wt(E e) { return e.y; }
};
template <>
struct SellE<false> {
  using E = uint32_t;
  static __device__ __forceinline__ E none() { return NONE; }
  static __device__ __forceinline__ E make(uint32_t u, uint32_t) { return u; }
  static __device__ __forceinline__ uint32_t nbr(E e) { return e; }
  static __device__ __forceinline__ uint32_t wt(E) { return 0u; }
};

// Pieces of a hub of in-list length len: equal lengths of at most PULL_HUB.
__device__ __forceinline__ uint32_t hub_pieces(uint32_t len) { return (len + PULL_HUB - 1) / PULL_HUB; }

// Hubs (in-list longer than PULL_HUB) with their piece counts.
__global__ void k_sell_hubs(DevGraph g, uint32_t *hub_v, uint64_t *hub_np, unsigned long long *cnt) {
  const uint64_t V = g.V;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += stride) {
    const uint32_t d = seg_len(g.in, (uint32_t)v);
    if (d > PULL_HUB) {
      const unsigned long long h = atomicAdd(cnt, 1ull);
      hub_v[h] = (uint32_t)v;
      hub_np[h] = hub_pieces(d);
    }
  }
}

// Row keys of the vertices: in-list length, 0 for hubs (their rows are pieces).
__global__ void k_sell_keys(DevGraph g, uint32_t *key, uint32_t *id) {
  const uint64_t V = g.V;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += stride) {
    const uint32_t d = seg_len(g.in, (uint32_t)v);
    key[v] = d > PULL_HUB ? 0u : d;
    id[v] = (uint32_t)v;
  }
}

// Piece rows of every hub (id V + piece index), their keys and the piece table.
__global__ void k_sell_pieces(DevGraph g, const uint32_t *hub_v, const uint64_t *piece_off, uint64_t nh, uint32_t *key,
                              uint32_t *id, uint32_t *piece_v, uint32_t *piece_start, uint32_t *piece_len) {
  const uint64_t V = g.V;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t h = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; h < nh; h += stride) {
    const uint32_t v = hub_v[h];
    const uint32_t d = seg_len(g.in, v);
    const uint64_t p0 = piece_off[h];
    const uint32_t np = hub_pieces(d), base = d / np, extra = d % np;
    uint32_t start = 0;
    for (uint32_t k = 0; k < np; k++) {
      const uint32_t n = base + (k < extra ? 1u : 0u);
      key[V + p0 + k] = n;
      id[V + p0 + k] = (uint32_t)(V + p0 + k);
      piece_v[p0 + k] = v;
      piece_start[p0 + k] = start;
      piece_len[p0 + k] = n;
      start += n;
    }
  }
}

__global__ void k_sell_count(const uint32_t *key, uint64_t n, unsigned long long *rows) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x; base < n; base += stride) {
    const uint64_t i = base + threadIdx.x;
    const unsigned b = __ballot_sync(FULL, i < n && key[i] > 0);
    if (lane_id() == 0 && b) atomicAdd(rows, (unsigned long long)__popc(b));
  }
}

// Slice sizes (entries): 32 x the length of the slice's first (longest) row.
__global__ void k_sell_sizes(const uint32_t *sorted_key, uint64_t slices, uint64_t *size) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s <= slices; s += stride)
    size[s] = s < slices ? 32ull * sorted_key[s * 32] : 0;
}

// Copy the live in-entries of each row into its column; pad with NONE.
template <bool W>
__global__ void k_sell_fill(DevGraph g, const uint32_t *row_id, uint64_t rows, uint64_t slices, const uint64_t *off,
                            const uint32_t *piece_v, const uint32_t *piece_start, const uint32_t *piece_len,
                            typename SellE<W>::E *ent) {
  using P_ = PoolT<W>;
  using S_ = SellE<W>;
  const typename P_::E *pool = reinterpret_cast<const typename P_::E *>(g.in.pool);
  const uint64_t V = g.V;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < slices * 32; r += stride) {
    const uint64_t s = r >> 5, lane = r & 31;
    const uint64_t o0 = off[s], width = (off[s + 1] - o0) >> 5;
    uint64_t j = 0;
    if (r < rows) {
      const uint32_t id = row_id[r];
      uint32_t v, k0, n;
      if (id < V) {
        v = id;
        k0 = 0;
        n = seg_len(g.in, v);
      } else {
        v = piece_v[id - V];
        k0 = piece_start[id - V];
        n = piece_len[id - V];
      }
      const uint64_t so = g.in.off[v] + k0;
      for (uint32_t k = 0; k < n && j < width; k++) {
        const typename P_::E e = pool[so + k];
        const uint32_t u = P_::nbr(e);
        if (u & DEAD) continue;
        ent[o0 + j * 32 + lane] = S_::make(u, P_::wt(e));
        j++;
      }
    }
    for (; j < width; j++) ent[o0 + j * 32 + lane] = S_::none();
  }
}

// Writes v's pulled best when it improves v's value (single writer per vertex).
template <int A>
__device__ __forceinline__ bool pull_commit(const DevGraph &g, bool has, uint32_t v, uint64_t best, uint32_t bsrc,
                                            uint32_t bw) {
  if (!has || !Hook<A>::better(best, ld_v32(g.val32, v))) return false;
  g.lab[v] = make_ulonglong2(best, pack_parent(bsrc, bw));
  g.val32[v] = (uint32_t)best;
  return true;
}

// Commit of one pulled row (all lanes of the warp call it).
template <int A>
__device__ __forceinline__ void pull_row_done(const DevGraph &g, bool active, uint32_t id, bool has, uint64_t best,
                                              uint32_t bsrc, uint32_t bw, ulonglong2 *piece_best, uint32_t *fout,
                                              unsigned long long *fout_n, uint32_t mst, unsigned long long &local) {
  bool upd = false;
  if (active && id < g.V) {
    upd = pull_commit<A>(g, has, id, best, bsrc, bw);
  } else if (active) {
    // a hub piece: its best waits for k_pull_hub_fix
    piece_best[id - g.V] = make_ulonglong2(best, has ? pack_parent(bsrc, bw) : ~0ull);
  }
  local += upd;
  warp_append(upd, id, fout, fout_n, FULL);
  if (mst) mark_modified(g, upd, id, mst);
}

template <int A, bool W>
__device__ __forceinline__ void pull_take(const typename SellE<W>::E &e, uint32_t sv, bool &has, uint64_t &best,
                                          uint32_t &bsrc, uint32_t &bw) {
  using S_ = SellE<W>;
  if (S_::nbr(e) == NONE) return;
  const uint64_t c = Hook<A>::combine(sv, S_::wt(e));
  if (!has || Hook<A>::better(c, best)) {
    has = true;
    best = c;
    bsrc = S_::nbr(e);
    bw = S_::wt(e);
  }
}

// Source values through L1: the values of popular sources stay there.  A value
// cached before its owner improved in this level is only older, and that owner
// is in the next frontier anyway.
__device__ __forceinline__ uint32_t pull_src_val(const DevGraph &g, uint32_t u) {
  return u != NONE ? __ldca(&g.val32[u]) : 0u;
}

// Slices are sorted by width (the length of their longest row).  Wide slices
// (more than 8 entries per row) take a warp each and stream their rows 16 (or
// 8 + 8 prefetched) entries at a time; narrower slices are taken G at a time
// (G = 2, 4, 8 for widths up to 8, 4, 2) so that every lane still keeps 16
// entries in flight per round trip.  cls[0..2]: first slice of width <= 8, 4, 2.
struct PullClasses {
  uint64_t c8, c4, c2;
};

template <int A, bool W, int G>
__device__ __forceinline__ void pull_narrow(const DevGraph &g, const typename SellE<W>::E *ent, const uint64_t *off,
                                            const uint32_t *row_id, uint64_t rows, uint64_t lo, uint64_t hi,
                                            ulonglong2 *piece_best, uint32_t *fout, unsigned long long *fout_n,
                                            uint32_t mst, unsigned long long &local, uint64_t warp, uint64_t nwarps) {
  using S_ = SellE<W>;
  constexpr int NP = 16 / G;
  const int lane = lane_id();
  for (uint64_t s0 = lo + warp * G; s0 < hi; s0 += nwarps * G) {
    typename S_::E e[16];
#pragma unroll
    for (int gi = 0; gi < G; gi++) {
      const uint64_t s = s0 + gi;
      const uint64_t o = s < hi ? off[s] : 0, w = s < hi ? (off[s + 1] - o) >> 5 : 0;
#pragma unroll
      for (int k = 0; k < NP; k++) e[gi * NP + k] = k < w ? __ldcs(&ent[o + (uint64_t)k * 32 + lane]) : S_::none();
    }
    uint32_t sv[16];
#pragma unroll
    for (int k = 0; k < 16; k++) sv[k] = pull_src_val(g, S_::nbr(e[k]));
#pragma unroll
    for (int gi = 0; gi < G; gi++) {
      const uint64_t s = s0 + gi;
      const uint64_t r = s * 32 + lane;
      const bool active = s < hi && r < rows;
      bool has = false;
      uint64_t best = 0;
      uint32_t bsrc = 0, bw = 0;
#pragma unroll
      for (int k = 0; k < NP; k++) pull_take<A, W>(e[gi * NP + k], sv[gi * NP + k], has, best, bsrc, bw);
      pull_row_done<A>(g, active, active ? row_id[r] : 0u, has, best, bsrc, bw, piece_best, fout, fout_n, mst, local);
    }
  }
}

// One launch covers the wide slices [s_lo, s_hi), and the narrow classes
// when `rest` is set.
template <int A, bool W>
__global__ void __launch_bounds__(PS_TPB) k_pull_sell(DevGraph g, const typename SellE<W>::E *ent, const uint64_t *off,
                                                      const uint32_t *row_id, uint64_t rows, uint64_t slices,
                                                      PullClasses cls, uint64_t s_lo, uint64_t s_hi, int rest,
                                                      ulonglong2 *piece_best, uint32_t *fout,
                                                      unsigned long long *fout_n, uint32_t mst) {
  if (g.ctl[C_MODE] != M_PULL) return;
  using S_ = SellE<W>;
  const int lane = lane_id();
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long local = 0;
  for (uint64_t s = s_lo + warp; s < s_hi; s += nwarps) {
    const uint64_t r = s * 32 + lane;
    const bool active = r < rows;
    const uint32_t id = active ? row_id[r] : 0u;
    const uint64_t o0 = off[s], width = (off[s + 1] - o0) >> 5;
    const typename S_::E *col = ent + o0 + lane;
    bool has = false;
    uint64_t best = 0;
    uint32_t bsrc = 0, bw = 0;
    constexpr int N = PullDepth<W>::N;
    typename S_::E ne[N];
    if constexpr (PullDepth<W>::prefetch) {
#pragma unroll
      for (int k = 0; k < N; k++) ne[k] = k < width ? __ldcs(&col[(uint64_t)k * 32]) : S_::none();
    }
    for (uint64_t j = 0; j < width; j += N) {
      typename S_::E e[N];
#pragma unroll
      for (int k = 0; k < N; k++) {
        if constexpr (PullDepth<W>::prefetch) {
          e[k] = ne[k];
          ne[k] = j + N + k < width ? __ldcs(&col[(j + N + k) * 32]) : S_::none();
        } else {
          e[k] = j + k < width ? __ldcs(&col[(j + k) * 32]) : S_::none();
        }
      }
      uint32_t sv[N];  // every hook's values fit 32 bits
#pragma unroll
      for (int k = 0; k < N; k++) sv[k] = pull_src_val(g, S_::nbr(e[k]));
#pragma unroll
      for (int k = 0; k < N; k++) pull_take<A, W>(e[k], sv[k], has, best, bsrc, bw);
    }
    pull_row_done<A>(g, active, id, has, best, bsrc, bw, piece_best, fout, fout_n, mst, local);
  }
  if (!rest) {
    warp_add_result(local, &g.ctl[C_RESULT]);
    return;
  }
  pull_narrow<A, W, 2>(g, ent, off, row_id, rows, cls.c8, cls.c4, piece_best, fout, fout_n, mst, local, warp, nwarps);
  pull_narrow<A, W, 4>(g, ent, off, row_id, rows, cls.c4, cls.c2, piece_best, fout, fout_n, mst, local, warp, nwarps);
  pull_narrow<A, W, 8>(g, ent, off, row_id, rows, cls.c2, slices, piece_best, fout, fout_n, mst, local, warp, nwarps);
  warp_add_result(local, &g.ctl[C_RESULT]);
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&g.ctl[C_EDGES], off[slices]);
}

// First slice whose width is at most 8, 4, 2 (slice widths never increase).
__global__ void k_sell_classes(const uint32_t *sorted_key, uint64_t slices, unsigned long long *cls) {
  // cls[3]: first slice narrower than PULL_SPLIT
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < slices; s += stride) {
    const uint32_t w = sorted_key[s * 32], wp = s ? sorted_key[(s - 1) * 32] : 0xFFFFFFFFu;
    if (w <= 8 && wp > 8) cls[0] = s;
    if (w <= 4 && wp > 4) cls[1] = s;
    if (w <= 2 && wp > 2) cls[2] = s;
    if (w < PULL_SPLIT && wp >= PULL_SPLIT) cls[3] = s;
  }
}

// One warp per hub: best of its pieces, one write.
template <int A>
__global__ void k_pull_hub_fix(DevGraph g, const uint32_t *hub_v, const uint64_t *piece_off, uint64_t nh,
                               const ulonglong2 *piece_best, uint32_t *fout, unsigned long long *fout_n, uint32_t mst) {
  if (g.ctl[C_MODE] != M_PULL) return;
  const int lane = lane_id();
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long local = 0;
  for (uint64_t h0 = warp * 32; h0 < nh; h0 += nwarps * 32) {
    // lane l owns hub h0 + l; the warp scans the pieces of its 32 hubs
    const uint64_t h = h0 + lane;
    bool has = false;
    uint64_t best = 0, meta = 0;
    uint32_t v = 0;
    if (h < nh) {
      v = hub_v[h];
      for (uint64_t p = piece_off[h]; p < piece_off[h + 1]; p++) {
        const ulonglong2 b = piece_best[p];
        if (b.y == ~0ull) continue;
        if (!has || Hook<A>::better(b.x, best)) {
          has = true;
          best = b.x;
          meta = b.y;
        }
      }
    }
    const bool upd = h < nh && pull_commit<A>(g, has, v, best, (uint32_t)meta, (uint32_t)(meta >> 32));
    local += upd;
    warp_append(upd, v, fout, fout_n, FULL);
    if (mst) mark_modified(g, upd, v, mst);
  }
  warp_add_result(local, &g.ctl[C_RESULT]);
}

// Bottom-up BFS level for full builds (the reference's dense pull,
// core/graph.hpp:936-976, specialised to BFS): every unreached vertex scans
// its in-edges and takes the first in-neighbour at depth d as its parent,
// stopping there.  Used when the frontier is large; each vertex is written
// only by its own thread, so no atomics on labels.
template <bool W>
__global__ void k_bfs_bottom_up(DevGraph g, uint32_t *fout, unsigned long long *fout_n) {
  if (g.ctl[C_MODE] != M_BOTTOM_UP) return;
  const uint64_t d = g.ctl[C_DEPTH];
  using P_ = PoolT<W>;
  const typename P_::E *pool = reinterpret_cast<const typename P_::E *>(g.in.pool);
  const uint64_t V = g.V;
  unsigned long long local = 0, scanned = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x; base < V; base += stride) {
    const uint64_t v = base + threadIdx.x;
    bool found = false;
    if (v < V && ld_v32(g.val32, (uint32_t)v) == BFS_MAXL) {
      const uint32_t len = seg_len(g.in, (uint32_t)v);
      const uint64_t off = g.in.off[v];
      for (uint32_t k = 0; k < len; k++) {
        const typename P_::E e = __ldg(&pool[off + k]);
        const uint32_t u = P_::nbr(e);
        scanned++;
        if (u & DEAD) continue;
        if (__ldca(&g.val32[u]) == d) {  // a stale value only hides a parent found this level
          g.lab[v] = make_ulonglong2(d + 1, pack_parent(u, P_::wt(e)));
          g.val32[v] = (uint32_t)(d + 1);
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

// ---- small frontiers: several levels in one CTA -----------------------------
// Incremental repairs and the tail of a build run many levels whose frontier
// is a handful of vertices; one launch per level would cost more than the
// work.  k_push_tiny takes a frontier of at most TINY_N vertices and
// TINY_EDGES out-slots and keeps relaxing level after level inside one CTA
// (CTA barriers between levels), until the frontier empties or outgrows those
// limits; the frontier it leaves is in the level's output queue, as after any
// other level kernel.  Each slot is found by a binary search of the frontier's
// degree prefix in shared memory.
constexpr uint32_t TINY_N = 1024;
constexpr uint64_t TINY_EDGES = 1ull << 20;
constexpr int TINY_TPB = 1024;

//
// tiny_levels is that loop as a device function for a CTA of TINY_TPB threads:
// it leaves the frontier in q_final (one of q_in, q_out) with its count in
// *n_final.  first_begun: k_level_begin did the first level's bookkeeping (the
// level counter, stamp, depth and trace); otherwise the loop does it for every
// level, the first included.
template <int A, bool W>
__device__ __forceinline__ void tiny_levels(const DevGraph &g, uint32_t *q_in, unsigned long long *n_in,
                                            uint32_t *q_out, unsigned long long *n_out, uint32_t *q_final,
                                            unsigned long long *n_final, uint64_t max_levels, uint64_t max_edges,
                                            uint32_t mst, bool first_begun) {
  using P_ = PoolT<W>;
  using Scan = cub::BlockScan<uint32_t, TINY_TPB>;
  __shared__ typename Scan::TempStorage scan_tmp;
  __shared__ uint32_t s_pref[TINY_N + 1];
  __shared__ uint32_t s_v[TINY_N];
  __shared__ uint64_t s_off[TINY_N];
  __shared__ uint32_t s_su[TINY_N];
  __shared__ int s_go;
  const typename P_::E *pool = reinterpret_cast<const typename P_::E *>(g.out.pool);
  unsigned long long *c = g.ctl;
  const unsigned tid = threadIdx.x;
  uint32_t *cur = q_in, *nxt = q_out;
  unsigned long long *cur_n = n_in, *nxt_n = n_out;
  unsigned long long local = 0, scanned = 0;
  for (bool first = true;; first = false) {
    const uint64_t n = *cur_n;
    // stage the frontier and its degree prefix
    uint32_t d = 0;
    if (n <= TINY_N && tid < n) {
      const uint32_t u = cur[tid];
      s_v[tid] = u;
      s_off[tid] = g.out.off[u];
      s_su[tid] = (uint32_t)ld_v32(g.val32, u);
      d = seg_len(g.out, u);
    }
    uint32_t excl, total;
    Scan(scan_tmp).ExclusiveSum(d, excl, total);
    if (tid < TINY_N) s_pref[tid] = excl;
    if (tid == 0) {
      s_pref[TINY_N] = total;
      bool go = n > 0 && n <= TINY_N && total <= max_edges;
      if ((!first || !first_begun) && go) {
        // a new level: the bookkeeping k_level_begin does for the first one
        const uint64_t lvl = c[C_LEVEL];
        go = lvl < max_levels;
        if (go) {
          c[C_STAMP] += 1;
          c[C_DEPTH] = lvl;
          if (lvl < TRACE_CAP) {
            g.trace[lvl] = n;
            g.trace[TRACE_CAP + lvl] = global_ns();
          }
          c[C_LEVEL] = lvl + 1;
          *nxt_n = 0;
        }
      }
      s_go = go;
    }
    __syncthreads();
    if (!s_go) break;
    const uint32_t st = (uint32_t)c[C_STAMP];
    for (uint32_t base = 0; base < total; base += TINY_TPB) {
      const uint32_t e = base + tid;
      bool upd = false;
      uint32_t v = 0;
      if (e < total) {
        uint32_t lo = 0, hi = (uint32_t)n - 1;
        while (lo < hi) {
          const uint32_t mid = (lo + hi + 1) >> 1;
          if (s_pref[mid] <= e) lo = mid;
          else hi = mid - 1;
        }
        const typename P_::E ent = __ldg(&pool[s_off[lo] + (e - s_pref[lo])]);
        v = P_::nbr(ent);
        scanned++;
        if (!(v & DEAD)) upd = relax_lab<A>(g, s_v[lo], s_su[lo], v, P_::wt(ent));
      }
      local += upd;
      const bool app = upd && atomicExch(&g.stamp[v], st) != st;
      warp_append(app, v, nxt, nxt_n, FULL);
      if (mst) mark_modified(g, upd, v, mst);
    }
    __syncthreads();  // the next level reads the queue this one wrote
    uint32_t *t = cur;
    cur = nxt;
    nxt = t;
    unsigned long long *tn = cur_n;
    cur_n = nxt_n;
    nxt_n = tn;
  }
  if (cur != q_final) {
    const uint64_t n = *cur_n;
    for (uint64_t i = tid; i < n; i += TINY_TPB) q_final[i] = cur[i];
    __syncthreads();
    if (tid == 0) *n_final = n;
  }
  __syncthreads();
  warp_add_result(local, &c[C_RESULT]);
  warp_add_result(scanned, &c[C_EDGES]);
}

// The frontier is left in the output queue of the level the launch stands for.
template <int A, bool W>
__global__ void __launch_bounds__(TINY_TPB) k_push_tiny(DevGraph g, uint32_t *q_in, unsigned long long *n_in,
                                                        uint32_t *q_out, unsigned long long *n_out,
                                                        uint64_t max_levels, uint64_t max_edges, uint32_t mst) {
  if (g.ctl[C_MODE] != M_TINY) return;
  tiny_levels<A, W>(g, q_in, n_in, q_out, n_out, q_out, n_out, max_levels, max_edges, mst, true);
}

// ---- cluster levels ------------------------------------------------------------
// A frontier too large for one CTA but at most CL_TPB vertices per CTA of a
// thread-block cluster (16 CTAs where the GPU schedules a cluster that size,
// else 8; one per SM) runs in k_push_cluster: successive levels inside one
// launch, separated by the hardware cluster barrier (barrier.cluster, with
// release/acquire ordering of the global queue and labels) instead of kernel
// boundaries and a conditional node per level, which cost 25-40 us per
// mid-size level in the graph-driven loop.  Each CTA stages CL_TPB frontier
// vertices (offset, value, degree prefix) in its shared memory; the level's
// out-slots are spread evenly over every thread of the cluster, and a thread
// finds the vertex of its slot in the owning CTA's shared memory through
// distributed shared memory.  Every decision that ends the loop is made from
// values that all CTAs read alike (the frontier size after a barrier, the
// CTAs' slot totals in global memory), so that every CTA passes the same
// barriers.  The loop ends when the frontier empties or outgrows the cluster
// (more than CL_TPB vertices per CTA or max_edges slots), leaving the frontier
// in the level's output queue like tiny_levels.
constexpr int CL_TPB = 1024;
constexpr int CL_MAX_CTAS = 16;
constexpr uint64_t CL_EDGES = 1ull << 20;  // largest slot limit of a cluster level

template <int A, bool W>
__global__ void __launch_bounds__(CL_TPB, 1)
    k_push_cluster(DevGraph g, uint32_t *q_in, unsigned long long *n_in, uint32_t *q_out, unsigned long long *n_out,
                   unsigned long long *tot, uint64_t max_levels, uint64_t max_edges, uint32_t mst) {
  namespace cgr = cooperative_groups;
  if (g.ctl[C_MODE] != M_CLUSTER) return;  // the same in every CTA
  cgr::cluster_group cluster = cgr::this_cluster();
  using P_ = PoolT<W>;
  using Scan = cub::BlockScan<uint32_t, CL_TPB>;
  __shared__ typename Scan::TempStorage scan_tmp;
  __shared__ uint32_t s_pref[CL_TPB + 1];
  __shared__ uint32_t s_v[CL_TPB];
  __shared__ uint64_t s_off[CL_TPB];
  __shared__ uint32_t s_su[CL_TPB];
  __shared__ uint64_t s_base[CL_MAX_CTAS + 1];
  const typename P_::E *pool = reinterpret_cast<const typename P_::E *>(g.out.pool);
  unsigned long long *c = g.ctl;
  const unsigned tid = threadIdx.x;
  const unsigned nc = cluster.num_blocks(), r = cluster.block_rank();
  const uint64_t cap = (uint64_t)nc * CL_TPB;  // frontier vertices the cluster stages
  uint32_t *cur = q_in, *nxt = q_out;
  unsigned long long *cur_n = n_in, *nxt_n = n_out;
  unsigned long long local = 0, scanned = 0;
  uint64_t n = 0;
  for (bool first = true;; first = false) {
    // values every CTA reads alike: written before the last barrier (or the launch)
    n = __ldcg(cur_n);
    const unsigned long long st0 = __ldcg(&c[C_STAMP]), lvl = __ldcg(&c[C_LEVEL]);
    const bool book = !first;  // k_level_begin did the first level's bookkeeping
    const uint64_t i = (uint64_t)r * CL_TPB + tid;
    uint32_t d = 0;
    if (n <= cap && i < n) {
      const uint32_t u = __ldcg(&cur[i]);
      s_v[tid] = u;
      s_off[tid] = g.out.off[u];
      s_su[tid] = (uint32_t)ld_v32(g.val32, u);
      d = seg_len(g.out, u);
    }
    uint32_t excl, total;
    Scan(scan_tmp).ExclusiveSum(d, excl, total);
    s_pref[tid] = excl;
    if (tid == 0) {
      s_pref[CL_TPB] = total;
      tot[r] = total;
      // the output count: the input of the level before this one, read by every CTA
      // before the last barrier
      if (r == 0 && book) *nxt_n = 0;
    }
    cluster.sync();  // A: totals and stage visible, output count cleared
    if (tid < 32) {
      // the CTAs' slot totals, loaded together and scanned in one warp
      const uint64_t t = tid < nc ? __ldcg(&tot[tid]) : 0;
      uint64_t incl = t;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(FULL, incl, o);
        if (tid >= (unsigned)o) incl += y;
      }
      if (tid <= nc) s_base[tid] = incl - t;  // entry nc: the level's slots
    }
    __syncthreads();
    const uint64_t S = s_base[nc];
    const bool go = n > 0 && n <= cap && (first || (S <= max_edges && lvl < max_levels));
    if (!go) break;  // the same in every CTA
    if (book && r == 0 && tid == 0) {
      c[C_STAMP] = st0 + 1;
      c[C_DEPTH] = lvl;
      if (lvl < TRACE_CAP) {
        g.trace[lvl] = n;
        g.trace[TRACE_CAP + lvl] = global_ns();
      }
      c[C_LEVEL] = lvl + 1;
    }
    const uint32_t st = (uint32_t)(book ? st0 + 1 : st0);
    for (uint64_t base = 0; base < S; base += cap) {
      const uint64_t e = base + i;
      bool upd = false;
      uint32_t v = 0;
      if (e < S) {
        unsigned k = 0;  // the CTA that staged slot e: largest k with s_base[k] <= e
        while (k + 1 < nc && s_base[k + 1] <= e) k++;
        const uint32_t el = (uint32_t)(e - s_base[k]);
        const uint32_t *rp = cluster.map_shared_rank(s_pref, k);
        const uint64_t left = n - (uint64_t)k * CL_TPB;
        const uint64_t nk = left < CL_TPB ? left : CL_TPB;
        uint32_t lo = 0, hi = (uint32_t)nk - 1;  // largest j with rp[j] <= el
        while (lo < hi) {
          const uint32_t mid = (lo + hi + 1) >> 1;
          if (rp[mid] <= el) lo = mid;
          else hi = mid - 1;
        }
        const uint64_t off = *cluster.map_shared_rank(&s_off[lo], k);
        const uint32_t u = *cluster.map_shared_rank(&s_v[lo], k);
        const uint32_t su = *cluster.map_shared_rank(&s_su[lo], k);
        const typename P_::E ent = __ldg(&pool[off + (el - rp[lo])]);
        v = P_::nbr(ent);
        scanned++;
        if (!(v & DEAD)) upd = relax_lab<A>(g, u, su, v, P_::wt(ent));
      }
      local += upd;
      const bool app = upd && atomicExch(&g.stamp[v], st) != st;
      warp_append(app, v, nxt, nxt_n, FULL);
      if (mst) mark_modified(g, upd, v, mst);
    }
    cluster.sync();  // B: this level's queue and labels visible; nobody reads a peer's stage any more
    uint32_t *t = cur;
    cur = nxt;
    nxt = t;
    unsigned long long *tn = cur_n;
    cur_n = nxt_n;
    nxt_n = tn;
  }
  // the frontier that ended the loop goes to the launch's output queue
  if (cur != q_out) {
    for (uint64_t k = (uint64_t)r * CL_TPB + tid; k < n; k += cap) q_out[k] = __ldcg(&cur[k]);
    if (r == 0 && tid == 0) *n_out = n;
  }
  warp_add_result(local, &c[C_RESULT]);
  warp_add_result(scanned, &c[C_EDGES]);
}

// ---- device-driven level loop ------------------------------------------------
// A tree call runs k_prologue, its seed kernel, then a CUDA graph whose WHILE
// node repeats a pair of levels (queue 0 -> 1, then 1 -> 0).  Each level
// starts with k_level_begin, which reads the frontier size and picks the level
// mode and stamp on the device; every level kernel returns at once unless the
// mode is its own; k_loop_cond stops the loop when the frontier is empty.  No
// host round trip happens between levels (the reference's driver decides
// between levels on the host, core/graph.hpp:898-983, :1013-1111).

// stamp: the control block's C_STAMP when the caller read it already.
__device__ __forceinline__ void prologue_ctl(unsigned long long *c, unsigned long long inv_tag,
                                             const unsigned long long *stamp = nullptr) {
  c[C_INVTAG] = inv_tag;
  c[C_INVITER] = 0;
  c[C_OVER] = 0;
  c[C_QN0] = 0;
  c[C_QN1] = 0;
  c[C_HUBN] = 0;
  c[C_RESULT] = 0;
  c[C_TREEN] = 0;
  c[C_RECOMPUTE] = 0;
  c[C_LEVEL] = 0;
  c[C_EDGES] = 0;
  c[C_MODE] = M_EMPTY;
  c[C_KLAUNCH] = 0;
  c[C_HVR] = 0;
  c[C_HVE] = 0;
  c[C_HVP] = 0;
  c[C_STAMP] = (stamp ? *stamp : c[C_STAMP]) + 1;
}

__global__ void k_prologue(DevGraph g, unsigned long long inv_tag) { prologue_ctl(g.ctl, inv_tag); }

// Kernels a level of each mode launches (k_level_begin not included).
__host__ __device__ __forceinline__ int mode_launches(unsigned long long mode) {
  switch (mode) {
    case M_SPARSE: return 2;
    case M_PULL: return 3;
    case M_DENSE_PUSH: return 2;
    case M_BOTTOM_UP: return 1;
    case M_LBS: return 5;
    case M_TINY: return 1;
    case M_CLUSTER: return 1;
  }
  return 0;
}

struct LevelCfg {
  uint64_t dense_div;
  uint64_t lbs_min;
  uint64_t bu_div;    // BFS builds go bottom-up once frontier * bu_div >= |V|
  uint64_t pull_div;  // builds pull once frontier * pull_div >= |V|
  uint64_t pull_split;  // pull levels run in two launches
  uint64_t tiny_edges;
  uint64_t max_levels;  // level bound baked into the loop graphs
  uint64_t pull_groups;  // launches of a split pull level
  uint64_t cl_edges;     // out-slot limit of a cluster level (0: no cluster levels)
  uint64_t cl_v;         // frontier vertices a cluster stages (its CTAs x CL_TPB)
  int allow_pull;
  int bottom_up;
};

// Picks the level mode from the frontier size (the reference's push/pull rule
// at core/graph.hpp:334 and its vertex/edge-centric rule at :595-612 play the
// same role); inside a graph it also selects the SWITCH case to run.
// Threads of k_level_begin (they sum small frontiers' degrees).  256, not
// 1024: the kernel starts every level, and in served mode the epochs of other
// instances occupy the SMs, where a 1024-thread CTA waits longer for room.
constexpr int LVB_TPB = 256;
// A frontier that both a tiny level and a cluster level could take goes to the
// cluster when it has more out-slots than this: one CTA walks them
// 1024 at a time, the cluster 16,384 at a time.
constexpr uint64_t CL_TINY_PREF = 4096;

__global__ void __launch_bounds__(LVB_TPB) k_level_begin(DevGraph g, const uint32_t *fin,
                                                         const unsigned long long *fin_n, unsigned long long *fout_n,
                                                         LevelCfg cfg, int use_switch, cudaGraphConditionalHandle sw) {
  using BR = cub::BlockReduce<unsigned long long, LVB_TPB>;
  __shared__ typename BR::TempStorage br_tmp;
  const uint64_t n0 = *fin_n;
  unsigned long long d = 0;
  if ((cfg.tiny_edges && n0 && n0 <= TINY_N) || (cfg.cl_edges && n0 && n0 <= cfg.cl_v)) {
    // eight frontier entries per thread in flight (a frontier of up to 16K vertices)
    for (uint64_t i0 = threadIdx.x; i0 < n0; i0 += 8 * LVB_TPB) {
      uint32_t u[8];
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const uint64_t i = i0 + (uint64_t)k * LVB_TPB;
        u[k] = i < n0 ? fin[i] : NONE;
      }
#pragma unroll
      for (int k = 0; k < 8; k++) d += u[k] != NONE ? seg_len(g.out, u[k]) : 0u;
    }
  }
  // a tree reduction: 1024 threads adding into one shared word contend for it
  const unsigned long long s_edges = BR(br_tmp).Sum(d);  // valid in thread 0
  if (threadIdx.x != 0) return;
  const bool tiny = cfg.tiny_edges && n0 && n0 <= TINY_N && s_edges <= cfg.tiny_edges;
  const bool clus = cfg.cl_edges && n0 && n0 <= cfg.cl_v && s_edges <= cfg.cl_edges;
  unsigned long long *c = g.ctl;
  const uint64_t n = n0;
  const uint64_t lvl = c[C_LEVEL];
  *fout_n = 0;
  c[C_HUBN] = 0;
  c[C_STAMP] += 1;
  c[C_DEPTH] = lvl;
  const bool dense = n * cfg.dense_div >= g.V;
  unsigned long long mode = M_SPARSE;
  if (n == 0) mode = M_EMPTY;
  else if (cfg.bottom_up && n * cfg.bu_div >= g.V) mode = M_BOTTOM_UP;
  // pull once the frontier passes |V| / pull_div, and keep pulling until it
  // falls below 4x that (the frontier's first large levels are hub-heavy, its
  // last ones are not: the direction switch of Beamer et al., by vertex count)
  else if (cfg.allow_pull && n * (c[C_MODE] == M_PULL ? (cfg.pull_div + 3) / 4 : cfg.pull_div) >= g.V) mode = M_PULL;
  else if (tiny && !(clus && s_edges > CL_TINY_PREF)) mode = M_TINY;
  else if (clus) mode = M_CLUSTER;
  else if (dense) mode = M_DENSE_PUSH;
  else if (n >= cfg.lbs_min) mode = M_LBS;
  if (mode == M_DENSE_PUSH) c[C_ACT] += 1;
  c[C_MODE] = mode;
  if (use_switch) c[C_KLAUNCH] += 1 + mode_launches(mode) + (mode == M_PULL ? cfg.pull_groups - 2 : 0);
  if (n) {
    if (lvl < TRACE_CAP) {
      g.trace[lvl] = n;
      g.trace[TRACE_CAP + lvl] = global_ns();  // the level's start on the device clock
    }
    c[C_LEVEL] = lvl + 1;
  }
  if (use_switch) cudaGraphSetConditional(sw, (unsigned)mode);
}

__global__ void k_loop_cond(DevGraph g, const unsigned long long *n_after, uint64_t max_levels,
                            cudaGraphConditionalHandle handle) {
  const uint64_t n = *n_after;
  const uint64_t lvl = g.ctl[C_LEVEL];
  g.ctl[C_KLAUNCH] += 1;
  // the end of the levels so far (the next level's start overwrites it)
  if (lvl < TRACE_CAP) g.trace[TRACE_CAP + lvl] = global_ns();
  if (n && lvl >= max_levels) atomicCAS(&g.ctl[C_ERR], 0ull, (unsigned long long)RG_ETIMEOUT);
  cudaGraphSetConditional(handle, (n && lvl < max_levels) ? 1u : 0u);
}

// Deletion repair loop control (do_update_tree_del, core/graph.hpp:1250-1418):
// one invalidation level per k_inv_begin; the full-recompute fallback
// (:1252) stops the loop and turns the rest of the repair into no-ops.
__global__ void k_inv_begin(DevGraph g, const unsigned long long *fin_n, unsigned long long *fout_n, uint64_t big) {
  unsigned long long *c = g.ctl;
  const uint64_t n = *fin_n;
  *fout_n = 0;
  c[C_HVR] = 0;
  c[C_HVE] = 0;
  c[C_KLAUNCH] += 5;  // this kernel, k_rescue, k_rescue_heavy, k_expand, k_expand_heavy
  if (n == 0 || c[C_RECOMPUTE]) return;
  const uint64_t it = c[C_INVITER];
  if (it <= 10 && c[C_TREEN] + n > big) c[C_RECOMPUTE] = 1;
  c[C_INVITER] = it + 1;
}

// in_graph = 0: launched by the host (profile mode); the condition goes to
// C_HOSTCOND instead of the WHILE node's handle.
__global__ void k_inv_cond(DevGraph g, const unsigned long long *n_after, uint64_t max_iter,
                           cudaGraphConditionalHandle handle, int in_graph) {
  unsigned long long *c = g.ctl;
  const uint64_t n = *n_after;
  c[C_KLAUNCH] += 1;
  const unsigned go = (n && !c[C_RECOMPUTE] && c[C_INVITER] < max_iter) ? 1u : 0u;
  if (in_graph) cudaGraphSetConditional(handle, go);
  else c[C_HOSTCOND] = go;
}

__global__ void k_copy_frontier(DevGraph g, const uint32_t *src, const unsigned long long *src_n, uint32_t *dst,
                                unsigned long long *dst_n) {
  if (blockIdx.x == 0 && threadIdx.x == 0) g.ctl[C_KLAUNCH] += 4;  // k_reset, k_pull, k_pull_heavy, this kernel
  if (g.ctl[C_RECOMPUTE]) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *dst_n = 0;
    return;
  }
  const uint64_t n = *src_n;
  if (blockIdx.x == 0 && threadIdx.x == 0) *dst_n = n;
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = src[i];
}

// build_tree init (core/graph.hpp:886-896): every label to init_label_func,
// parent to empty; the active set is the root, or every vertex (WCC).
template <int A>
__global__ void k_init(DevGraph g, uint64_t root, uint32_t *fout) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < g.V; v += stride) {
    g.lab[v] = make_ulonglong2(Hook<A>::init(v, root), pack_parent(NONE, 0));
    g.val32[v] = (uint32_t)Hook<A>::init(v, root);
    if (Hook<A>::all_active) fout[v] = (uint32_t)v;
    else if (v == root) fout[0] = (uint32_t)v;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    g.ctl[C_QN0] = Hook<A>::all_active ? g.V : 1;
    g.ctl[C_ROOT] = root;
  }
}

// Seed relaxations of update_tree_add (single :1140-1153, batch :1180-1214):
// relax each inserted edge, both orientations when undirected.
template <int A>
__device__ __forceinline__ unsigned long long seed_add(const DevGraph &g, const uint32_t *os, const uint32_t *od,
                                                       const uint32_t *ow, const uint32_t *cand, uint64_t n,
                                                       int directed, uint32_t *fout, unsigned long long *fout_n,
                                                       uint32_t mst, uint64_t warp, uint64_t nwarps) {
  const uint32_t st = (uint32_t)g.ctl[C_STAMP];
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
        upd = relax<A>(g, u, ld_v32(g.val32, u), v, ow[op]);
      }
      local += upd;
      bool app = upd && atomicExch(&g.stamp[v], st) != st;
      warp_append(app, v, fout, fout_n, FULL);
      if (mst) mark_modified(g, upd, v, mst);
    }
  }
  return local;
}

template <int A>
__global__ void k_seed_add(DevGraph g, const uint32_t *os, const uint32_t *od, const uint32_t *ow, const uint32_t *cand,
                           const unsigned long long *cand_n, uint64_t n_all, int directed, uint32_t *fout,
                           unsigned long long *fout_n, uint32_t mst) {
  const uint64_t n = cand ? *cand_n : n_all;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long local = seed_add<A>(g, os, od, ow, cand, n, directed, fout, fout_n, mst, warp, nwarps);
  warp_add_result(local, &g.ctl[C_RESULT]);
}

// Seeds of update_tree_del (single :1640-1649, batch :1680-1714): a deleted
// edge that is dst's parent edge invalidates dst.
__device__ __forceinline__ void seed_del(const DevGraph &g, const uint32_t *os, const uint32_t *od, const uint32_t *ow,
                                         const uint32_t *cand, uint64_t n, int directed, uint32_t *fout,
                                         unsigned long long *fout_n, uint64_t warp, uint64_t nwarps) {
  const uint32_t tag_inv = (uint32_t)g.ctl[C_INVTAG];
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

__global__ void k_seed_del(DevGraph g, const uint32_t *os, const uint32_t *od, const uint32_t *ow, const uint32_t *cand,
                           const unsigned long long *cand_n, uint64_t n_all, int directed, uint32_t *fout,
                           unsigned long long *fout_n) {
  const uint64_t n = cand ? *cand_n : n_all;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  seed_del(g, os, od, ow, cand, n, directed, fout, fout_n, warp, nwarps);
}

// has_parents (core/graph.hpp:1889-1907): does x's parent chain reach a root
// without meeting a vertex invalidated (or rescued) by this repair?  The chain
// guard (0.1 |V| steps) requests a full recompute, as the reference does.
//
// A chain found clear stays clear for the rest of the repair: tags only go to
// the tree descendants of vertices tagged before (the seeds are tagged first),
// and only tagged vertices change parent, so an untagged chain never gains a
// tag.  The walk therefore stops at a vertex marked clear earlier in this
// repair (chk == the repair's tag), and a clear walk marks the first vertices
// of its chain, so that walks from their descendants end there.
//
// The three words of a step are loaded together, so that a step costs one
// round trip to memory rather than three.
__device__ __forceinline__ bool has_parents(const DevGraph &g, uint32_t x0, uint32_t tag_inv, uint64_t limit) {
  uint64_t num = 0;
  uint32_t x = x0;
  for (;;) {
    const uint32_t ck = ld_u32(&g.chk[x]);
    const uint32_t t = ld_u32(&g.inv[x]);
    const uint32_t p = (uint32_t)ld_meta(&g.lab[x]);
    if (ck == tag_inv) break;
    if (t == tag_inv || t == tag_inv + 1) return true;
    if (p == NONE) break;
    x = p;
    if (++num > limit) {
      atomicExch(&g.ctl[C_RECOMPUTE], 1ull);
      return true;
    }
  }
  x = x0;
  for (int k = 0; k < 16 && x != NONE && ld_u32(&g.chk[x]) != tag_inv; k++) {
    g.chk[x] = tag_inv;
    x = (uint32_t)ld_meta(&g.lab[x]);
  }
  return false;
}

// Rescue (core/graph.hpp:1323-1361): an invalidated dst keeps its value when an
// in-neighbour satisfies equal_func and has a clean parent chain; the parent
// moves to that in-edge.  One warp per frontier vertex.
// Heavy vertices: a warp per vertex would scan an RMAT hub's 10^5 edges 32 at
// a time.  The warp-per-vertex passes of the deletion repair (rescue, expand,
// the pull over the reset set) queue the vertices whose list is longer than
// HEAVY_DEG instead, and a second kernel spreads each queued vertex's list over
// every warp of the grid.  Without a queue (the one-CTA repair, which hands
// heavy vertices over to the grid-wide one) or when it is full, the warp scans
// the whole list itself.
constexpr uint32_t HEAVY_DEG = 2048;

__device__ __forceinline__ bool queue_heavy(uint32_t *hv, unsigned long long *hv_n, uint64_t hv_cap, uint32_t v,
                                            int lane) {
  unsigned long long k = 0;
  if (lane == 0) k = atomicAdd(hv_n, 1ull);
  k = __shfl_sync(FULL, k, 0);
  if (k < hv_cap) {
    if (lane == 0) hv[k] = v;
    return true;
  }
  return false;
}

template <int A, bool W>
__device__ __forceinline__ void rescue_warps(const DevGraph &g, const uint32_t *fin, uint64_t n, uint64_t limit,
                                             uint64_t warp, uint64_t nwarps, uint32_t *hv = nullptr,
                                             unsigned long long *hv_n = nullptr, uint64_t hv_cap = 0) {
  const uint32_t tag_inv = (uint32_t)g.ctl[C_INVTAG];
  using P = PoolT<W>;
  const typename P::E *pool = reinterpret_cast<const typename P::E *>(g.in.pool);
  const int lane = lane_id();
  for (uint64_t idx = warp; idx < n; idx += nwarps) {
    const uint32_t d = fin[idx];
    // (the vertex's words in one round trip)
    const uint32_t td = ld_u32(&g.inv[d]);
    const uint64_t sd = ld_v32(g.val32, d);
    const uint32_t len = seg_len(g.in, d);
    const uint64_t off = g.in.off[d];
    if (td != tag_inv) continue;
    if (hv && len > HEAVY_DEG && queue_heavy(hv, hv_n, hv_cap, d, lane)) continue;
    for (uint32_t kb = 0; kb < len; kb += 32) {
      const uint32_t k = kb + lane;
      bool ok = false;
      uint32_t src = 0, w = 0;
      if (k < len) {
        typename P::E e = pool[off + k];
        src = P::nbr(e);
        w = P::wt(e);
        if (!(src & DEAD) && Hook<A>::combine(ld_v32(g.val32, src), w) == sd) ok = !has_parents(g, src, tag_inv, limit);
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

template <int A, bool W>
__global__ void __launch_bounds__(TPB) k_rescue(DevGraph g, const uint32_t *fin, const unsigned long long *fin_n,
                                                uint64_t limit) {
  if (g.ctl[C_RECOMPUTE]) return;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  rescue_warps<A, W>(g, fin, *fin_n, limit, warp, nwarps, g.heavy, &g.ctl[C_HVR], g.heavy_cap);
}

// Rescue of the queued heavy vertices: for each in turn, every warp scans a
// 32-entry stride of its in-list; the first valid candidate wins the CAS.
template <int A, bool W>
__global__ void __launch_bounds__(TPB) k_rescue_heavy(DevGraph g, uint64_t limit) {
  if (g.ctl[C_RECOMPUTE]) return;
  const uint32_t tag_inv = (uint32_t)g.ctl[C_INVTAG];
  using P = PoolT<W>;
  const typename P::E *pool = reinterpret_cast<const typename P::E *>(g.in.pool);
  const int lane = lane_id();
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t nh = min(g.ctl[C_HVR], (unsigned long long)g.heavy_cap);
  for (uint64_t h = 0; h < nh; h++) {
    const uint32_t d = g.heavy[h];
    const uint64_t sd = ld_v32(g.val32, d);
    const uint32_t len = seg_len(g.in, d);
    const uint64_t off = g.in.off[d];
    for (uint64_t kb = warp * 32; kb < len; kb += nwarps * 32) {
      if (__shfl_sync(FULL, ld_u32(&g.inv[d]), 0) != tag_inv) break;  // rescued by another warp
      const uint64_t k = kb + lane;
      bool ok = false;
      uint32_t src = 0, w = 0;
      if (k < len) {
        typename P::E e = pool[off + k];
        src = P::nbr(e);
        w = P::wt(e);
        if (!(src & DEAD) && Hook<A>::combine(ld_v32(g.val32, src), w) == sd) ok = !has_parents(g, src, tag_inv, limit);
      }
      unsigned b = __ballot_sync(FULL, ok);
      if (b) {
        const int l = __ffs(b) - 1;
        if (lane == l && atomicCAS(&g.inv[d], tag_inv, tag_inv + 1) == tag_inv)
          reinterpret_cast<unsigned long long *>(&g.lab[d])[1] = pack_parent(src, w);
        break;
      }
    }
  }
}

// Collect and expand (core/graph.hpp:1363-1417): a still-invalid vertex joins
// the reset set; its tree children (parent == (u,w)) are invalidated next.
template <int A, bool W>
__device__ __forceinline__ void expand_warps(const DevGraph &g, const uint32_t *fin, uint64_t n, uint32_t *tree,
                                             uint32_t *fout, unsigned long long *fout_n, uint64_t warp,
                                             uint64_t nwarps, uint32_t *hv = nullptr,
                                             unsigned long long *hv_n = nullptr, uint64_t hv_cap = 0) {
  const uint32_t tag_inv = (uint32_t)g.ctl[C_INVTAG];
  using P = PoolT<W>;
  const typename P::E *pool = reinterpret_cast<const typename P::E *>(g.out.pool);
  const int lane = lane_id();
  for (uint64_t idx = warp; idx < n; idx += nwarps) {
    const uint32_t u = fin[idx];
    // (the vertex's words in one round trip; its slot in the reset set is
    // taken here and written after the scan, off the critical path)
    const uint32_t tu = ld_u32(&g.inv[u]);
    const uint32_t len = seg_len(g.out, u);
    const uint64_t off = g.out.off[u];
    if (tu != tag_inv) continue;
    unsigned long long slot = 0;
    if (lane == 0) slot = atomicAdd(&g.ctl[C_TREEN], 1ull);
    if (!(hv && len > HEAVY_DEG && queue_heavy(hv, hv_n, hv_cap, u, lane))) {
      for (uint32_t kb = 0; kb < len; kb += 32) {
        const uint32_t k = kb + lane;
        bool app = false;
        uint32_t v = 0;
        if (k < len) {
          typename P::E e = pool[off + k];
          v = P::nbr(e);
          if (!(v & DEAD)) {
            const uint64_t meta = ld_meta(&g.lab[v]);
            const uint32_t t = ld_u32(&g.inv[v]);
            if (meta == pack_parent(u, P::wt(e)) && t != tag_inv && t != tag_inv + 1)
              app = atomicCAS(&g.inv[v], t, tag_inv) == t;
          }
        }
        warp_append(app, v, fout, fout_n, FULL);
      }
    }
    if (lane == 0) tree[slot] = u;
  }
}

// Expansion of the queued heavy vertices: their tree children, found by every
// warp over a stride of the out-list.
template <int A, bool W>
__global__ void __launch_bounds__(TPB) k_expand_heavy(DevGraph g, uint32_t *fout, unsigned long long *fout_n) {
  if (g.ctl[C_RECOMPUTE]) return;
  const uint32_t tag_inv = (uint32_t)g.ctl[C_INVTAG];
  using P = PoolT<W>;
  const typename P::E *pool = reinterpret_cast<const typename P::E *>(g.out.pool);
  const int lane = lane_id();
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t *hv = g.heavy + g.heavy_cap;
  const uint64_t nh = min(g.ctl[C_HVE], (unsigned long long)g.heavy_cap);
  for (uint64_t h = 0; h < nh; h++) {
    const uint32_t u = hv[h];
    const uint32_t len = seg_len(g.out, u);
    const uint64_t off = g.out.off[u];
    for (uint64_t kb = warp * 32; kb < len; kb += nwarps * 32) {
      const uint64_t k = kb + lane;
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

template <int A, bool W>
__global__ void __launch_bounds__(TPB) k_expand(DevGraph g, const uint32_t *fin, const unsigned long long *fin_n,
                                                uint32_t *tree, uint32_t *fout, unsigned long long *fout_n) {
  if (g.ctl[C_RECOMPUTE]) return;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  expand_warps<A, W>(g, fin, *fin_n, tree, fout, fout_n, warp, nwarps, g.heavy + g.heavy_cap, &g.ctl[C_HVE],
                     g.heavy_cap);
}

// Reset the invalid set to init (core/graph.hpp:1420-1430).
template <int A>
__device__ __forceinline__ void reset_warps(const DevGraph &g, const uint32_t *tree, uint64_t n, uint32_t mst,
                                            uint64_t warp, uint64_t nwarps) {
  const uint64_t root = g.ctl[C_ROOT];
  for (uint64_t base = warp * 32; base < n; base += nwarps * 32) {
    uint64_t i = base + lane_id();
    uint32_t u = 0;
    if (i < n) {
      u = tree[i];
      g.lab[u] = make_ulonglong2(Hook<A>::init(u, root), pack_parent(NONE, 0));
      g.val32[u] = (uint32_t)Hook<A>::init(u, root);
    }
    if (mst) mark_modified(g, i < n, u, mst);
  }
}

template <int A>
__global__ void k_reset(DevGraph g, const uint32_t *tree, const unsigned long long *tree_n, uint32_t mst) {
  if (g.ctl[C_RECOMPUTE]) return;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  reset_warps<A>(g, tree, *tree_n, mst, warp, nwarps);
}

// One transposed pull over the reset set (core/graph.hpp:1433-1511): each
// vertex takes its best in-neighbour by update_func.  One warp per vertex.
template <int A, bool W>
__device__ __forceinline__ unsigned long long pull_warps(const DevGraph &g, const uint32_t *fin, uint64_t n,
                                                         uint32_t mst, uint64_t warp, uint64_t nwarps,
                                                         uint32_t *hv = nullptr, unsigned long long *hv_n = nullptr,
                                                         uint64_t hv_cap = 0) {
  using P = PoolT<W>;
  const typename P::E *pool = reinterpret_cast<const typename P::E *>(g.in.pool);
  const int lane = lane_id();
  unsigned long long local = 0;
  for (uint64_t idx = warp; idx < n; idx += nwarps) {
    const uint32_t d = fin[idx];
    const uint32_t len = seg_len(g.in, d);
    const uint64_t off = g.in.off[d];
    if (hv && len > HEAVY_DEG && queue_heavy(hv, hv_n, hv_cap, d, lane)) continue;
    uint64_t best = ld_v32(g.val32, d), bsu = 0;
    uint32_t bsrc = NONE, bw = 0;
    for (uint32_t k = lane; k < len; k += 32) {
      typename P::E e = pool[off + k];
      uint32_t s = P::nbr(e);
      if (s & DEAD) continue;
      uint64_t su = ld_v32(g.val32, s);
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
    if (lane == 0 && bsrc != NONE) upd = relax<A>(g,bsrc, bsu, d, bw);
    local += upd;
    if (mst) mark_modified(g, __shfl_sync(FULL, upd, 0) && lane == 0, d, mst);
  }
  return local;
}

template <int A, bool W>
__global__ void __launch_bounds__(TPB) k_pull(DevGraph g, const uint32_t *fin, const unsigned long long *fin_n,
                                              uint32_t mst) {
  if (g.ctl[C_RECOMPUTE]) return;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long local =
      pull_warps<A, W>(g, fin, *fin_n, mst, warp, nwarps, g.heavy + 2 * g.heavy_cap, &g.ctl[C_HVP], g.heavy_cap);
  warp_add_result(local, &g.ctl[C_RESULT]);
}

// The pull of the queued heavy reset vertices: every warp takes the best of a
// stride of the in-list and relaxes the vertex with it (the CAS keeps the best).
template <int A, bool W>
__global__ void __launch_bounds__(TPB) k_pull_heavy(DevGraph g, uint32_t mst) {
  if (g.ctl[C_RECOMPUTE]) return;
  using P = PoolT<W>;
  const typename P::E *pool = reinterpret_cast<const typename P::E *>(g.in.pool);
  const int lane = lane_id();
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t *hv = g.heavy + 2 * g.heavy_cap;
  const uint64_t nh = min(g.ctl[C_HVP], (unsigned long long)g.heavy_cap);
  unsigned long long local = 0;
  for (uint64_t h = 0; h < nh; h++) {
    const uint32_t d = hv[h];
    const uint32_t len = seg_len(g.in, d);
    const uint64_t off = g.in.off[d];
    if (warp * 32 >= len) continue;
    uint64_t best = ld_v32(g.val32, d), bsu = 0;
    uint32_t bsrc = NONE, bw = 0;
    for (uint64_t k = warp * 32 + lane; k < len; k += nwarps * 32) {
      typename P::E e = pool[off + k];
      uint32_t s = P::nbr(e);
      if (s & DEAD) continue;
      uint64_t su = ld_v32(g.val32, s);
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
    if (lane == 0 && bsrc != NONE) upd = relax<A>(g, bsrc, bsu, d, bw);
    local += upd;
    if (mst) mark_modified(g, __shfl_sync(FULL, upd, 0) && lane == 0, d, mst);
  }
  warp_add_result(local, &g.ctl[C_RESULT]);
}

// Small deletion repairs in one CTA: the invalidation levels (rescue, expand),
// the reset and the pull with CTA barriers in place of launches, then the
// reset set copied to queue 0 for the push loop.  When a level's frontier or
// the reset set outgrows one CTA it hands over to the multi-CTA repair (the
// IF node it opens), with the frontier left in queue 0 where that repair
// starts.
constexpr int DT_TPB = 1024;
constexpr uint64_t DEL_TINY_N = 1024, DEL_TINY_TREE = 8192;

// del_tiny_levels is that repair as a device function for a CTA of DT_TPB
// threads; it returns true when it hands over.
template <int A, bool W>
__device__ __forceinline__ bool del_tiny_levels(const DevGraph &g, uint32_t *q0, uint32_t *q1, uint32_t *tree,
                                                uint64_t limit, uint64_t big, uint64_t max_iter, uint32_t mst) {
  __shared__ int s_go;
  unsigned long long *c = g.ctl;
  const unsigned tid = threadIdx.x;
  const uint64_t warp = tid >> 5, nwarps = DT_TPB / 32;
  uint32_t *cur = q0, *nxt = q1;
  unsigned long long *cur_n = &c[C_QN0], *nxt_n = &c[C_QN1];
  for (;;) {
    // a heavy vertex (a list longer than HEAVY_DEG) in this level's frontier,
    // or in the reset set once the levels are done, goes to the grid-wide repair
    int heavy = 0;
    {
      const uint64_t n0 = *cur_n;
      if (n0 && n0 <= DEL_TINY_N) {
        for (uint64_t i = tid; i < n0; i += DT_TPB)
          heavy |= seg_len(g.in, cur[i]) > HEAVY_DEG || seg_len(g.out, cur[i]) > HEAVY_DEG;
      } else if (n0 == 0) {
        const uint64_t tn = c[C_TREEN];
        if (tn <= DEL_TINY_TREE)
          for (uint64_t i = tid; i < tn; i += DT_TPB) heavy |= seg_len(g.in, tree[i]) > HEAVY_DEG;
      }
    }
    heavy = __syncthreads_or(heavy);
    if (tid == 0) {
      const uint64_t n = *cur_n;
      int go = 1;  // 1: run this level; 0: invalidation done; 2: hand over
      if (n == 0 || c[C_RECOMPUTE]) {
        go = 0;
      } else if (n > DEL_TINY_N || heavy) {
        go = 2;
      } else {
        const uint64_t it = c[C_INVITER];
        if (it >= max_iter) {
          go = 0;
        } else if (it <= 10 && c[C_TREEN] + n > big) {  // core/graph.hpp:1252
          c[C_RECOMPUTE] = 1;
          go = 0;
        } else {
          c[C_INVITER] = it + 1;
          *nxt_n = 0;
        }
      }
      if (go == 0 && (c[C_TREEN] > DEL_TINY_TREE || heavy) && !c[C_RECOMPUTE]) go = 2;
      s_go = go;
    }
    __syncthreads();
    if (s_go != 1) break;
    const uint64_t n = *cur_n;
    rescue_warps<A, W>(g, cur, n, limit, warp, nwarps);
    __syncthreads();
    expand_warps<A, W>(g, cur, n, tree, nxt, nxt_n, warp, nwarps);
    __syncthreads();
    uint32_t *t = cur;
    cur = nxt;
    nxt = t;
    unsigned long long *tn = cur_n;
    cur_n = nxt_n;
    nxt_n = tn;
  }
  if (s_go == 2) {
    // the multi-CTA repair continues from queue 0
    if (cur != q0) {
      const uint64_t n = *cur_n;
      for (uint64_t i = tid; i < n; i += DT_TPB) q0[i] = cur[i];
      __syncthreads();
      if (tid == 0) c[C_QN0] = n;
    }
    __syncthreads();
    return true;
  }
  unsigned long long local = 0;
  const bool recompute = c[C_RECOMPUTE] != 0;
  if (!recompute) {
    const uint64_t tn = c[C_TREEN];
    reset_warps<A>(g, tree, tn, mst, warp, nwarps);
    __syncthreads();
    local = pull_warps<A, W>(g, tree, tn, mst, warp, nwarps);
    __syncthreads();
    for (uint64_t i = tid; i < tn; i += DT_TPB) q0[i] = tree[i];
    __syncthreads();
    if (tid == 0) c[C_QN0] = tn;
  } else if (tid == 0) {
    c[C_QN0] = 0;
  }
  warp_add_result(local, &c[C_RESULT]);
  __syncthreads();
  return false;
}

// in_graph = 0: launched by the host (profile mode); the hand-over decision
// goes to C_HOSTCOND instead of the IF node's handle.
template <int A, bool W>
__global__ void __launch_bounds__(DT_TPB) k_del_tiny(DevGraph g, uint32_t *q0, uint32_t *q1, uint32_t *tree,
                                                     uint64_t limit, uint64_t big, uint64_t max_iter, uint32_t mst,
                                                     cudaGraphConditionalHandle standard, int in_graph) {
  const bool over = del_tiny_levels<A, W>(g, q0, q1, tree, limit, big, max_iter, mst);
  if (threadIdx.x == 0) {
    g.ctl[C_KLAUNCH] += 1;
    if (in_graph) cudaGraphSetConditional(standard, over ? 1u : 0u);
    else g.ctl[C_HOSTCOND] = over ? 1 : 0;
  }
}

// The hand-over decision of the fused apply kernel's deletion repair, for the
// IF node of the grid-wide repair (a kernel sets the handle of a conditional
// node in its own graph).
__global__ void k_handover(DevGraph g, cudaGraphConditionalHandle standard) {
  g.ctl[C_KLAUNCH] += 1;
  cudaGraphSetConditional(standard, g.ctl[C_OVER] ? 1u : 0u);
}

// Fused small-batch apply: one CTA runs the storage steps of a batch of at
// most SMALL_EDGES edges (unpack from the mapped staging buffer, lookup/create,
// growth, new-slot write, multiplicity count, candidates) and the seeding of
// the tree repair, with CTA barriers where the multi-kernel path has kernel
// boundaries.  A small repair then runs in the same CTA: the one-CTA deletion
// repair (del_tiny_levels) for a delete batch, and push levels while the
// frontier stays small (tiny_levels).  The kernel ends by writing the control
// block to the host's mapped copy; C_LEFT there tells the host what is left
// for the graphs it launches next (the level loop; the grid-wide deletion
// repair when the one-CTA repair handed over, C_OVER).  A safe update (the
// common case, need_update_tree_* false) and most unsafe single updates cost
// this one kernel and no conditional node: a conditional node costs about
// 10 us even when its condition is false.  A storage error (edge
// index or pool full) stops before the count step, leaving the op arrays for
// the host's compaction and replay, exactly like the multi-kernel path.
constexpr int FS_TPB = 1024;
static_assert(FS_TPB == TINY_TPB && FS_TPB == DT_TPB, "the fused kernel runs the one-CTA repairs");

// What the fused kernel's in-place repair needs besides queue 0.
struct FusedRepair {
  uint32_t *q1, *tree;
  uint64_t limit;       // has_parents chain guard
  uint64_t big;         // invalidated-set size that asks for a full recompute
  uint64_t max_iter;    // invalidation levels
  uint64_t max_levels;  // level bound of the push loop
  uint64_t tiny_edges;  // out-slot limit of an in-place push level (0: none in place)
};

// The control block to the host's mapped copy, by the whole CTA after its
// last update (the host reads it once the stream has synchronised).
__device__ __forceinline__ void ctl_to_host(const DevGraph &g, unsigned long long *ctl_host) {
  __syncthreads();
  if (threadIdx.x < C_COUNT) ctl_host[threadIdx.x] = g.ctl[threadIdx.x];
  __threadfence_system();
}

// A batch's header as the fused kernels read it.
struct StagedBatch {
  uint64_t n, pairs, want, inv_tag;
  unsigned long long stamp;  // C_STAMP at the kernel's start (used by its first batch)
};

// A batch of at most INLINE_EDGES edges travels inside the kernel's parameters
// (the launch carries it to the SM), so the kernel reads no staging buffer
// across the bus: single updates and the served path's small epochs skip the
// one PCIe round trip (about 6 us) that staging from mapped memory costs.
// words[] holds the batch as the caller gave it: rg_edge records (3 words per
// edge) or (src, dst) pairs (2 words).
constexpr unsigned INLINE_EDGES = INLINE_MAX_EDGES;
struct InlineBatch {
  uint64_t n, pairs, want, inv_tag;
  uint64_t words[3 * INLINE_EDGES];
};

// The batch crosses the bus in 16-byte loads into device scratch: the first
// APPLY_SPEC chunks in the same round trip as the header (thread hdr_t reads
// the header, threads chunk_t .. chunk_t + APPLY_SPEC - 1 the chunks), the
// rest in apply_batch once the header gives the size.  The host wrote both
// before the launch; they are read past any cache.
constexpr unsigned APPLY_SPEC = 256;

__device__ __forceinline__ void stage_batch(const DevGraph &g, const ApplyHdr *hdr, const char *data, uint4 *scratch,
                                            StagedBatch &sb, unsigned hdr_t, unsigned chunk_t) {
  const unsigned tid = threadIdx.x;
  const uint4 *raw = reinterpret_cast<const uint4 *>(data);
  if (tid >= chunk_t && tid < chunk_t + APPLY_SPEC) scratch[tid - chunk_t] = __ldcv(&raw[tid - chunk_t]);
  if (tid == hdr_t) {
    sb.stamp = g.ctl[C_STAMP];
    sb.n = __ldcv(&hdr->n);
    sb.pairs = __ldcv(&hdr->pairs);
    sb.want = __ldcv(&hdr->want_old);
    sb.inv_tag = __ldcv(&hdr->inv_tag);
  }
}

// One staged batch through the storage steps, the seeding and the in-place
// repair, by all threads of the CTA after a barrier.  Returns 0 when nothing
// is left, 1 when the repair left work for the graph nodes after the kernel
// (C_OVER set when the deletion repair handed over), 2 after a storage error
// or when it skipped the batch.  inl: the batch's words in the kernel's
// parameters (an inline batch), or null when they were staged into scratch.
template <int A, bool W>
__device__ __forceinline__ int apply_batch(const DevGraph &g, sdev::OpView ops, const StagedBatch &sb,
                                           const char *data, uint64_t *old_host, uint32_t *cand, int add, int directed,
                                           uint32_t *q0, uint32_t mst, int second, const FusedRepair &fr,
                                           uint4 *scratch, const uint64_t *inl = nullptr) {
  __shared__ int s_skip;
  unsigned long long *c = g.ctl;
  const unsigned tid = threadIdx.x;
  // phase trace (RG_OPT_PHASE_TRACE): thread 0 stamps the device clock
  unsigned long long *tr = g.ptrace ? g.ptrace + 16 * second : nullptr;
  auto stamp = [&](int k) {
    if (tr && tid == 0) tr[k] = global_ns();
  };
  if (tid == 0) {
    // the second batch of a submission does nothing after an error in the first
    s_skip = second && c[C_ERR] != 0;
    if (!s_skip) {
      const unsigned long long kl = c[C_KLAUNCH];
      prologue_ctl(c, sb.inv_tag, second ? nullptr : &sb.stamp);
      if (second) c[C_KLAUNCH] = kl;  // the count covers the whole submission
      c[C_CANDN] = 0;
      c[C_GROWN_OUT] = 0;
      c[C_GROWN_IN] = 0;
    }
  }
  __syncthreads();
  if (s_skip) return 2;
  if (tr && tid == 0) tr[15] = 1;
  stamp(RG_PH_BEGIN);
  const uint64_t n = sb.n < SMALL_EDGES ? sb.n : SMALL_EDGES;
  const uint64_t nops = directed ? n : 2 * n;
  const int weighted = W ? 1 : 0;
  const uint64_t chunks = (n * (sb.pairs ? 16 : sizeof(rg_edge)) + 15) / 16;
  if (!inl && chunks > APPLY_SPEC) {
    const uint4 *raw = reinterpret_cast<const uint4 *>(data);
    for (uint64_t k = APPLY_SPEC + tid; k < chunks; k += FS_TPB) scratch[k] = __ldcv(&raw[k]);
    __syncthreads();
  }
  // staged words are read past L1 (this CTA wrote them); inline ones are parameters
  const uint64_t *words = inl ? inl : reinterpret_cast<const uint64_t *>(scratch);
  auto word = [&](uint64_t k) -> uint64_t { return inl ? inl[k] : __ldcg(&words[k]); };
  if (sb.pairs) {
    for (uint64_t i = tid; i < n; i += FS_TPB) {
      uint64_t s64 = word(2 * i), d64 = word(2 * i + 1);
      uint32_t w = weighted ? (uint32_t)(splitmix64((s64 << 32) | d64) % 255 + 1) : 0u;
      sdev::put_ops(ops, i, (uint32_t)s64, (uint32_t)d64, w, directed);
    }
  } else {
    for (uint64_t i = tid; i < n; i += FS_TPB) {
      uint64_t s64 = word(3 * i), d64 = word(3 * i + 1), w64 = word(3 * i + 2);
      sdev::put_ops(ops, i, (uint32_t)s64, (uint32_t)d64, weighted ? (uint32_t)w64 : 0u, directed);
    }
  }
  __syncthreads();
  stamp(RG_PH_UNPACK);
  for (uint64_t j = tid; j < nops; j += FS_TPB) sdev::lookup_op(g, ops, j, add);
  __syncthreads();
  stamp(RG_PH_LOOKUP);
  if (add) {
    // each warp grows its own vertices (a vertex is in a grow list once); the
    // copies of long lists (a hub's) are left to the whole CTA below
    constexpr unsigned BIG = 16;
    __shared__ sdev::GrowClaim s_big[BIG];
    __shared__ int s_big_in[BIG];
    __shared__ unsigned s_nbig;
    if (tid == 0) s_nbig = 0;
    __syncthreads();
    const unsigned gw = tid >> 5, gl = tid & 31;
    for (int in = 0; in < (g.symmetric ? 1 : 2); in++) {
      const DevDir &dir = in ? g.in : g.out;
      const unsigned long long nv = c[in ? C_GROWN_IN : C_GROWN_OUT];
      for (unsigned long long k = gw; k < nv; k += FS_TPB / 32) {
        const uint32_t v = dir.grow[k];
        // a slot may be free (taken below, or the warp copies after all);
        // lane 0's view keeps the choice uniform across the warp
        const bool more = __shfl_sync(FULL, s_nbig < BIG ? 1 : 0, 0) != 0;
        sdev::GrowClaim cl;
        if (sdev::grow_vertex_warp<W>(dir, c, v, gl, more, &cl)) {
          unsigned slot = 0;
          if (gl == 0) slot = atomicAdd(&s_nbig, 1u);
          slot = __shfl_sync(FULL, slot, 0);
          if (slot < BIG) {
            if (gl == 0) {
              s_big[slot] = cl;
              s_big_in[slot] = in;
            }
          } else {
            sdev::grow_copy<W>(dir, cl, gl, 32);
            __syncwarp();
            if (gl == 0) sdev::grow_publish(dir, cl);
          }
        }
      }
    }
    __syncthreads();
    const unsigned nbig = s_nbig < BIG ? s_nbig : BIG;
    for (unsigned b = 0; b < nbig; b++) sdev::grow_copy<W>(s_big_in[b] ? g.in : g.out, s_big[b], tid, FS_TPB);
    __syncthreads();
    if (tid < nbig) sdev::grow_publish(s_big_in[tid] ? g.in : g.out, s_big[tid]);
  }
  __syncthreads();
  stamp(RG_PH_GROW);
  if (c[C_ERR]) return 2;
  if (add) {
    for (uint64_t j = tid; j < nops; j += FS_TPB) sdev::write_new_op<W>(g, ops, j);
    __syncthreads();
    stamp(RG_PH_WRITE);
  }
  for (uint64_t j = tid; j < nops; j += FS_TPB) sdev::count_op<W>(g, ops, j, add);
  __syncthreads();
  stamp(RG_PH_COUNT);
  for (uint64_t i = tid; i < n; i += FS_TPB) sdev::edge_old(ops, i, directed, add, 1, sb.want ? old_host : nullptr, cand, c);
  __syncthreads();
  stamp(RG_PH_OLD);
  const uint64_t ncand = c[C_CANDN];
  const uint64_t warp = tid >> 5, nwarps = FS_TPB / 32;
  if (add) {
    unsigned long long local = seed_add<A>(g, ops.src, ops.dst, ops.w, cand, ncand, directed, q0, &c[C_QN0], mst, warp, nwarps);
    warp_add_result(local, &c[C_RESULT]);
  } else {
    seed_del(g, ops.src, ops.dst, ops.w, cand, ncand, directed, q0, &c[C_QN0], warp, nwarps);
  }
  __syncthreads();
  stamp(RG_PH_SEED);
  bool over = false;
  if (c[C_QN0] && !c[C_ERR]) {
    if (!add) over = del_tiny_levels<A, W>(g, q0, fr.q1, fr.tree, fr.limit, fr.big, fr.max_iter, mst);
    stamp(RG_PH_DELREPAIR);
    if (!over && fr.tiny_edges && c[C_QN0])
      tiny_levels<A, W>(g, q0, &c[C_QN0], fr.q1, &c[C_QN1], q0, &c[C_QN0], fr.max_levels, fr.tiny_edges, mst, false);
  }
  const bool left = over || (c[C_QN0] && !c[C_ERR]);
  __syncthreads();  // every thread has read the counts before the next batch resets them
  stamp(RG_PH_END);
  if (tid == 0) c[C_OVER] = over ? 1 : 0;
  return left ? 1 : 0;
}

template <int A, bool W>
__global__ void __launch_bounds__(FS_TPB)
    k_apply_small(DevGraph g, sdev::OpView ops, const ApplyHdr *hdr, const char *data, uint64_t *old_host,
                  uint32_t *cand, int add, int directed, uint32_t *q0, uint32_t mst, int second, FusedRepair fr,
                  uint4 *scratch, unsigned long long *ctl_host) {
  __shared__ StagedBatch sb;
  if (g.ptrace && threadIdx.x == 0) {
    g.ptrace[32 + 2 * second] = global_ns();
    g.ptrace[16 * second + 15] = 0;
    if (!second) g.ptrace[31] = 0;  // a single batch: no delete batch ran
  }
  stage_batch(g, hdr, data, scratch, sb, 0, 32);
  __syncthreads();
  if (g.ptrace && threadIdx.x == 0) g.ptrace[33 + 2 * second] = global_ns();
  const int r = apply_batch<A, W>(g, ops, sb, data, old_host, cand, add, directed, q0, mst, second, fr, scratch);
  if (threadIdx.x == 0) g.ctl[C_LEFT] = r == 1 ? (add ? 1 : 2) : 0;
  ctl_to_host(g, ctl_host);
}

// An insert batch and then a delete batch in one kernel (both staged in one
// round trip): the delete batch runs here too when the insert batch's repair
// finished in place.  C_LEFT tells the host what is left: 1 the insert
// batch's level loop and then the whole delete batch, 2 the delete batch's
// repair.
template <int A, bool W>
__global__ void __launch_bounds__(FS_TPB)
    k_apply_mixed(DevGraph g, sdev::OpView ops, const ApplyHdr *hdr1, const char *data1, const ApplyHdr *hdr2,
                  const char *data2, uint32_t *cand, int directed, uint32_t *q0, uint32_t mst, FusedRepair fr,
                  uint4 *scratch1, uint4 *scratch2, unsigned long long *ctl_host) {
  __shared__ StagedBatch sb1, sb2;
  if (g.ptrace && threadIdx.x == 0) {
    g.ptrace[32] = g.ptrace[34] = global_ns();
    g.ptrace[15] = g.ptrace[31] = 0;
  }
  stage_batch(g, hdr1, data1, scratch1, sb1, 0, 32);
  stage_batch(g, hdr2, data2, scratch2, sb2, 32 + APPLY_SPEC, 64 + APPLY_SPEC);
  __syncthreads();
  if (g.ptrace && threadIdx.x == 0) g.ptrace[33] = g.ptrace[35] = global_ns();
  int r = apply_batch<A, W>(g, ops, sb1, data1, nullptr, cand, 1, directed, q0, mst, 0, fr, scratch1);
  unsigned long long lf = r == 1 ? 1 : 0;
  if (r == 0) {
    r = apply_batch<A, W>(g, ops, sb2, data2, nullptr, cand, 0, directed, q0, mst, 1, fr, scratch2);
    lf = r == 1 ? 2 : 0;
  }
  if (threadIdx.x == 0) g.ctl[C_LEFT] = lf;
  ctl_to_host(g, ctl_host);
}

// The header of an inline batch (its size clamped to what the parameters hold).
__device__ __forceinline__ void inline_header(const DevGraph &g, const InlineBatch &ib, StagedBatch &sb) {
  if (threadIdx.x == 0) {
    sb.stamp = g.ctl[C_STAMP];
    sb.n = ib.n < INLINE_EDGES ? ib.n : INLINE_EDGES;
    sb.pairs = ib.pairs;
    sb.want = ib.want;
    sb.inv_tag = ib.inv_tag;
  }
}

// k_apply_small for an inline batch (launched directly, not from a graph).
template <int A, bool W>
__global__ void __launch_bounds__(FS_TPB)
    k_apply_small_inl(DevGraph g, sdev::OpView ops, const __grid_constant__ InlineBatch ib, uint64_t *old_host,
                      uint32_t *cand, int add, int directed, uint32_t *q0, uint32_t mst, FusedRepair fr,
                      unsigned long long *ctl_host) {
  __shared__ StagedBatch sb;
  if (g.ptrace && threadIdx.x == 0) {
    g.ptrace[32] = g.ptrace[33] = global_ns();
    g.ptrace[15] = 0;
    g.ptrace[31] = 0;
  }
  inline_header(g, ib, sb);
  __syncthreads();
  const int r = apply_batch<A, W>(g, ops, sb, nullptr, old_host, cand, add, directed, q0, mst, 0, fr, nullptr, ib.words);
  if (threadIdx.x == 0) g.ctl[C_LEFT] = r == 1 ? (add ? 1 : 2) : 0;
  ctl_to_host(g, ctl_host);
}

// k_apply_mixed for two inline batches.  When the insert batch leaves work,
// the host continues exactly as after k_apply_mixed: the delete batch is in
// the staging buffer too (the host wrote it there before the launch).
template <int A, bool W>
__global__ void __launch_bounds__(FS_TPB)
    k_apply_mixed_inl(DevGraph g, sdev::OpView ops, const __grid_constant__ InlineBatch ib1,
                      const __grid_constant__ InlineBatch ib2, uint32_t *cand, int directed, uint32_t *q0,
                      uint32_t mst, FusedRepair fr, unsigned long long *ctl_host) {
  __shared__ StagedBatch sb1, sb2;
  if (g.ptrace && threadIdx.x == 0) {
    g.ptrace[32] = g.ptrace[33] = g.ptrace[34] = g.ptrace[35] = global_ns();
    g.ptrace[15] = g.ptrace[31] = 0;
  }
  inline_header(g, ib1, sb1);
  inline_header(g, ib2, sb2);
  __syncthreads();
  int r = apply_batch<A, W>(g, ops, sb1, nullptr, nullptr, cand, 1, directed, q0, mst, 0, fr, nullptr, ib1.words);
  unsigned long long lf = r == 1 ? 1 : 0;
  if (r == 0) {
    r = apply_batch<A, W>(g, ops, sb2, nullptr, nullptr, cand, 0, directed, q0, mst, 1, fr, nullptr, ib2.words);
    lf = r == 1 ? 2 : 0;
  }
  if (threadIdx.x == 0) g.ctl[C_LEFT] = lf;
  ctl_to_host(g, ctl_host);
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
      else r = r || Hook<A>::better(Hook<A>::combine(ld_v32(g.val32, u), w), ld_val(&g.lab[v]));
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

uint32_t mod_stamp(Graph &g) { return g.trace ? 1u : 0u; }

int read_ctl(Graph &g) {
  RG_CUDA(cudaMemcpyAsync(g.h_ctl, g.d.ctl, sizeof(unsigned long long) * C_COUNT, cudaMemcpyDeviceToHost, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  return RG_OK;
}

// Stamps and dense-level activity ids count up on the device, one per level.
// A call runs at most max_levels levels, so clearing the arrays whenever the
// last observed counter is within that margin of 2^32 keeps them unique.
int guard_counters(Graph &g) {
  const uint64_t margin = 8 * (uint64_t)g.V + (1ull << 16);
  if (g.h_ctl[C_STAMP] + margin >= 0xFFFFFFFFull) {
    RG_CUDA(cudaMemsetAsync(g.d.stamp, 0, (size_t)g.V * 4 + 4, g.stream));
    RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_STAMP], 0, 8, g.stream));
    g.h_ctl[C_STAMP] = 0;
  }
  if (g.h_ctl[C_ACT] + margin >= 0xFFFFFFFFull) {
    RG_CUDA(cudaMemsetAsync(g.act, 0, (size_t)g.V * 4 + 4, g.stream));
    RG_CUDA(cudaMemsetAsync(&g.d.ctl[C_ACT], 0, 8, g.stream));
    g.h_ctl[C_ACT] = 0;
  }
  return RG_OK;
}

// Sliced-ELL copy of the in-edges for dense pull levels, rebuilt only after
// the adjacency changed (one degree sort and one copy per version).
template <bool W>
int prepare_pull_w(Graph &g) {
  const uint64_t V = g.V;
  unsigned long long *cnt = g.sell_cnt;
  unsigned long long h[2] = {0, 0};
  auto grow = [&](void **p, uint64_t &cap, uint64_t want, size_t esz) -> int {
    if (want <= cap && *p) return RG_OK;
    if (*p) {
      cudaFree(*p);
      g.bytes -= cap * esz;
    }
    *p = nullptr;
    cap = 0;
    const uint64_t c = want + want / 8 + 64;
    if (cudaMalloc(p, c * esz) != cudaSuccess) {
      cudaGetLastError();
      set_error("device allocation failed: pull preparation");
      return RG_ENOMEM_HBM;
    }
    cap = c;
    g.bytes += c * esz;
    return RG_OK;
  };
  int rc = RG_OK;
  // 1. hubs and their piece offsets (the hub arrays are sized for every vertex
  //    once, so their addresses stay fixed for the cached level-loop graph)
  if ((rc = grow((void **)&g.sell_hub, g.sell_hub_cap, V + 1, 4))) return rc;
  uint64_t off_cap = g.sell_hub_cap;
  if (!g.sell_hub_off) {
    if (cudaMalloc(&g.sell_hub_off, off_cap * 8) != cudaSuccess) {
      cudaGetLastError();
      set_error("device allocation failed: pull preparation");
      return RG_ENOMEM_HBM;
    }
    g.bytes += off_cap * 8;
  }
  RG_CUDA(cudaMemsetAsync(cnt, 0, 16, g.stream));
  count_launch(g);
  k_sell_hubs<<<g.num_sms * 8, TPB, 0, g.stream>>>(g.d, g.sell_hub, g.sell_hub_off, cnt);
  RG_CUDA(cudaMemcpyAsync(h, cnt, 8, cudaMemcpyDeviceToHost, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  const uint64_t nh = h[0];
  RG_CUDA(cudaMemsetAsync(g.sell_hub_off + nh, 0, 8, g.stream));
  size_t tb = g.cub_tmp_bytes;
  RG_CUDA(cub::DeviceScan::ExclusiveSum(g.cub_tmp, tb, g.sell_hub_off, g.sell_hub_off, nh + 1, g.stream));
  uint64_t P = 0;
  RG_CUDA(cudaMemcpyAsync(&P, g.sell_hub_off + nh, 8, cudaMemcpyDeviceToHost, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  const uint64_t n = V + P;
  // 2. piece table, piece results and row ids
  if ((rc = grow((void **)&g.sell_piece, g.sell_piece_cap, 3 * (P + 1), 4))) return rc;
  if ((rc = grow((void **)&g.sell_piece_best, g.sell_best_cap, P + 1, 16))) return rc;
  if ((rc = grow((void **)&g.sell_row, g.sell_row_cap, n, 4))) return rc;
  uint32_t *pv = g.sell_piece, *pst = pv + (P + 1), *pln = pst + (P + 1);
  // 3. keys and ids of all rows (vertices, then pieces), sorted by length
  uint32_t *key0 = nullptr;
  void *tmp = nullptr;
  if (cudaMalloc(&key0, n * 4 * 3 + 64) != cudaSuccess) {
    cudaGetLastError();
    set_error("device allocation failed: pull preparation");
    return RG_ENOMEM_HBM;
  }
  uint32_t *id0 = key0 + n, *key1 = id0 + n;
  count_launch(g, nh ? 2 : 1);
  k_sell_keys<<<g.num_sms * 8, TPB, 0, g.stream>>>(g.d, key0, id0);
  if (nh) k_sell_pieces<<<g.num_sms * 2, TPB, 0, g.stream>>>(g.d, g.sell_hub, g.sell_hub_off, nh, key0, id0, pv, pst, pln);
  cudaError_t e = cudaGetLastError();
  tb = 0;
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, key0, key1, id0, g.sell_row, (int)n, 0, 32, g.stream);
  if (e == cudaSuccess) e = cudaMalloc(&tmp, tb + 256);
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairsDescending(tmp, tb, key0, key1, id0, g.sell_row, (int)n, 0, 32, g.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(cnt + 1, 0, 8, g.stream);
  if (e == cudaSuccess) {
    count_launch(g);
    k_sell_count<<<g.num_sms * 4, TPB, 0, g.stream>>>(key1, n, cnt + 1);
    e = cudaMemcpyAsync(h, cnt, 16, cudaMemcpyDeviceToHost, g.stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(g.stream);
  cudaFree(tmp);
  const uint64_t rows = h[1], slices = (rows + 31) / 32;
  // 4. slice offsets (rows count hub pieces too, so there can be more than |V|)
  uint64_t total = 0;
  if (e == cudaSuccess && (rc = grow((void **)&g.sell_off, g.sell_off_cap, slices + 1, 8))) {
    cudaFree(key0);
    return rc;
  }
  if (e == cudaSuccess) {
    count_launch(g);
    k_sell_sizes<<<g.num_sms * 4, TPB, 0, g.stream>>>(key1, slices, g.scratch64);
    tb = g.cub_tmp_bytes;
    e = cub::DeviceScan::ExclusiveSum(g.cub_tmp, tb, g.scratch64, g.sell_off, slices + 1, g.stream);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&total, g.sell_off + slices, 8, cudaMemcpyDeviceToHost, g.stream);
  unsigned long long cls[4] = {slices, slices, slices, slices};
  if (e == cudaSuccess) e = cudaMemcpyAsync(g.sell_cnt + 2, cls, 32, cudaMemcpyHostToDevice, g.stream);
  if (e == cudaSuccess) {
    count_launch(g);
    k_sell_classes<<<g.num_sms * 4, TPB, 0, g.stream>>>(key1, slices, g.sell_cnt + 2);
    e = cudaMemcpyAsync(cls, g.sell_cnt + 2, 32, cudaMemcpyDeviceToHost, g.stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(g.stream);
  cudaFree(key0);
  if (e != cudaSuccess) return cuda_fail(e, "pull preparation");
  // 5. the entries
  if ((rc = grow(&g.sell_ent, g.sell_cap, total, W ? 8 : 4))) return rc;
  count_launch(g);
  k_sell_fill<W><<<g.num_sms * 8, TPB, 0, g.stream>>>(g.d, g.sell_row, rows, slices, g.sell_off, pv, pst, pln,
                                                      reinterpret_cast<typename SellE<W>::E *>(g.sell_ent));
  RG_CUDA(cudaGetLastError());
  g.sell_hubs = nh;
  g.sell_rows = rows;
  g.sell_slices = slices;
  // classes are nested: a slice of width <= 2 is also <= 4 and <= 8
  g.sell_cls[2] = cls[2];
  g.sell_cls[1] = std::min<uint64_t>(cls[1], g.sell_cls[2]);
  g.sell_cls[0] = std::min<uint64_t>(cls[0], g.sell_cls[1]);
  g.sell_split = std::min<uint64_t>(cls[3], g.sell_cls[0]);
  g.sell_off_host.resize(slices + 1);
  RG_CUDA(cudaMemcpyAsync(g.sell_off_host.data(), g.sell_off, (slices + 1) * 8, cudaMemcpyDeviceToHost, g.stream));
  RG_CUDA(cudaStreamSynchronize(g.stream));
  g.sell_epoch++;
  g.pull_version = g.adj_version;
  return RG_OK;
}

// Dense build levels pull (sliced ELL) for SSSP / SSWP / WCC by default; BFS
// builds use their bottom-up levels.  RG_OPT_DENSE_PULL 0 / 1 force push / pull.
bool pull_on(const Graph &g, int A) { return g.dense_pull == 1 || (g.dense_pull == 2 && A != RG_BFS); }

// Two-launch pull levels: RG_OPT_PULL_SPLIT 1 always, 0 never, 2 (default) for SSSP and WCC.
bool pull_split_on(const Graph &g, int A) {
  return g.pull_split == 1 || (g.pull_split == 2 && (A == RG_SSSP || A == RG_WCC));
}

int prepare_pull(Graph &g) {
  if (g.pull_version == g.adj_version) return RG_OK;
  return g.weighted ? prepare_pull_w<true>(g) : prepare_pull_w<false>(g);
}

// Slice bounds of the launches that follow the hub launch of a split pull
// level: [mid, b1), [b1, b2), ..., [b_k, c8), the narrow classes with the last
// launch; groups - 1 launches holding about equal shares of the entries of
// slices [mid, end).
std::vector<uint64_t> pull_group_bounds(const Graph &g, uint64_t mid, uint64_t c8, uint64_t groups) {
  std::vector<uint64_t> b{mid};
  const uint64_t k = groups > 2 ? groups - 1 : 1;
  const std::vector<uint64_t> &off = g.sell_off_host;
  if (k > 1 && off.size() == g.sell_slices + 1 && mid <= c8 && c8 <= g.sell_slices) {
    const uint64_t e0 = off[mid], e1 = off[g.sell_slices];
    for (uint64_t i = 1; i < k; i++) {
      const uint64_t target = e0 + (e1 - e0) * i / k;
      uint64_t s = (uint64_t)(std::lower_bound(off.begin() + mid, off.begin() + c8, target) - off.begin());
      s = std::min(std::max(s, b.back()), c8);
      if (s > b.back() && s < c8) b.push_back(s);
    }
  }
  b.push_back(c8);
  return b;
}

uint64_t max_levels_of(const Graph &g) { return g.max_levels ? g.max_levels : 4 * (uint64_t)g.V + 1024; }

// Kernels of one level mode for one half-level (queue half -> queue half^1).
template <int A, bool W>
int enqueue_mode(Graph &g, cudaStream_t s, int half, unsigned long long mode) {
  const uint32_t *fin = g.q[half];
  unsigned long long *fin_n = &g.d.ctl[C_QN0 + half];
  uint32_t *fout = g.q[half ^ 1];
  unsigned long long *fout_n = &g.d.ctl[C_QN0 + (half ^ 1)];
  unsigned long long *hub_n = &g.d.ctl[C_HUBN];
  const uint32_t mst = mod_stamp(g);
  switch (mode) {
    case M_SPARSE:
      k_push<A, W><<<g.num_sms * 16, TPB, 0, s>>>(g.d, fin, fin_n, fout, fout_n, g.hubq, hub_n, mst);
      k_push_hub<A, W><<<g.num_sms * 8, TPB, 0, s>>>(g.d, g.hubq, hub_n, fout, fout_n, mst);
      break;
    case M_PULL: {
      const auto *ent = reinterpret_cast<const typename SellE<W>::E *>(g.sell_ent);
      const PullClasses cls{g.sell_cls[0], g.sell_cls[1], g.sell_cls[2]};
      const bool split = pull_split_on(g, A);
      const uint64_t mid = split ? g.sell_split : cls.c8;  // end of the first launch's wide slices
      k_pull_sell<A, W><<<g.num_sms * 8, PS_TPB, 0, s>>>(g.d, ent, g.sell_off, g.sell_row, g.sell_rows, g.sell_slices,
                                                         cls, 0, mid, split ? 0 : 1, g.sell_piece_best, fout, fout_n,
                                                         mst);
      k_pull_hub_fix<A><<<(unsigned)std::max<uint64_t>(1, (g.sell_hubs + 255) / 256), 256, 0, s>>>(
          g.d, g.sell_hub, g.sell_hub_off, g.sell_hubs, g.sell_piece_best, fout, fout_n, mst);
      // the other rows, in widest-first groups of equal entries: each group
      // reads the values the groups before it set in this level
      const std::vector<uint64_t> b = pull_group_bounds(g, mid, cls.c8, split ? g.pull_groups : 2);
      for (size_t i = 0; i + 1 < b.size(); i++)
        k_pull_sell<A, W><<<g.num_sms * 8, PS_TPB, 0, s>>>(g.d, ent, g.sell_off, g.sell_row, g.sell_rows,
                                                           g.sell_slices, cls, b[i], b[i + 1],
                                                           (split && i + 2 == b.size()) ? 1 : 0, g.sell_piece_best,
                                                           fout, fout_n, mst);
      break;
    }
    case M_DENSE_PUSH:
      k_mark_active<<<g.num_sms * 8, TPB, 0, s>>>(g.d, fin, fin_n, g.act);
      k_push_dense<A, W><<<g.num_sms * 3, DN_TPB, 0, s>>>(g.d, g.act, fout, fout_n, mst);
      break;
    case M_TINY:
      k_push_tiny<A, W><<<1, TINY_TPB, 0, s>>>(g.d, g.q[half], fin_n, g.q[half ^ 1], fout_n, max_levels_of(g),
                                               std::min<uint64_t>(g.tiny_edges, TINY_EDGES), mst);
      break;
    case M_BOTTOM_UP:
      k_bfs_bottom_up<W><<<g.num_sms * 8, TPB, 0, s>>>(g.d, fout, fout_n);
      break;
    case M_CLUSTER: {
      if (!g.cl_ctas) break;  // never selected then
      cudaLaunchConfig_t lc = {};
      lc.gridDim = dim3((unsigned)g.cl_ctas);
      lc.blockDim = dim3(CL_TPB);
      lc.stream = s;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = (unsigned)g.cl_ctas;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      lc.attrs = at;
      lc.numAttrs = 1;
      uint32_t *qi = g.q[half], *qo = g.q[half ^ 1];
      if (cudaLaunchKernelEx(&lc, k_push_cluster<A, W>, g.d, qi, fin_n, qo, fout_n,
                             reinterpret_cast<unsigned long long *>(g.lb_sums), max_levels_of(g),
                             std::min<uint64_t>(g.cluster_edges, CL_EDGES), mst) != cudaSuccess)
        return RG_ECUDA;
      break;
    }
    case M_LBS:
      k_scan_sums<<<SC_BLOCKS, SC_TPB, 0, s>>>(g.d, fin, fin_n, g.scratch64, g.lb_sums);
      k_scan_top<<<1, SC_BLOCKS, 0, s>>>(g.lb_sums);
      k_scan_final<<<SC_BLOCKS, SC_TPB, 0, s>>>(fin_n, g.scratch64, g.lb_sums, g.lb_P);
      k_partition<<<g.num_sms * 4, TPB, 0, s>>>(g.lb_P, fin_n, g.lb_tile);
      k_push_lbs<A, W><<<g.num_sms * 3, LB_TPB, 0, s>>>(g.d, fin, fin_n, g.lb_P, g.lb_tile, fout, fout_n, mst);
      break;
    default:
      break;
  }
  return cudaGetLastError() == cudaSuccess ? RG_OK : RG_ECUDA;
}

// Hash of every level-mode knob: cached graphs bake them into kernel arguments.
uint64_t cfg_key(const LevelCfg &c) {
  uint64_t h = splitmix64(c.dense_div);
  h = splitmix64(h ^ c.lbs_min);
  h = splitmix64(h ^ c.bu_div);
  h = splitmix64(h ^ c.pull_div);
  h = splitmix64(h ^ c.pull_split);
  h = splitmix64(h ^ c.tiny_edges);
  h = splitmix64(h ^ c.max_levels);
  h = splitmix64(h ^ c.pull_groups);
  h = splitmix64(h ^ c.cl_edges);
  h = splitmix64(h ^ c.cl_v);
  return splitmix64(h ^ ((uint64_t)c.allow_pull << 1) ^ (uint64_t)c.bottom_up);
}

LevelCfg level_cfg(const Graph &g, int A, bool build_variant) {
  LevelCfg cfg;
  cfg.dense_div = g.dense_div;
  cfg.lbs_min = g.lbs_min;
  cfg.allow_pull = (build_variant && pull_on(g, A)) ? 1 : 0;
  cfg.bottom_up = (A == RG_BFS && build_variant && g.bfs_bottom_up) ? 1 : 0;
  cfg.bu_div = g.bu_div;
  cfg.pull_div = g.pull_div;
  cfg.pull_split = pull_split_on(g, A) ? 1 : 0;
  cfg.tiny_edges = g.tiny_edges < TINY_EDGES ? g.tiny_edges : TINY_EDGES;
  cfg.max_levels = max_levels_of(g);
  cfg.pull_groups = cfg.pull_split ? std::max<uint64_t>(2, g.pull_groups) : 2;
  cfg.cl_edges = g.cl_ctas ? std::min<uint64_t>(g.cluster_edges, CL_EDGES) : 0;
  cfg.cl_v = (uint64_t)g.cl_ctas * CL_TPB;
  return cfg;
}

uint64_t recompute_threshold(const Graph &g) {
  return std::max<uint64_t>((uint64_t)(0.05 * (double)g.V), g.recompute_min);
}

// The level loop as a node of a CUDA graph:
//   WHILE (frontier non-empty) {
//     k_level_begin(q0 -> q1) ; SWITCH(mode) { sparse | pull | dense push | bottom-up | edge-balanced }
//     k_level_begin(q1 -> q0) ; SWITCH(mode) { ... }
//     k_loop_cond
//   }
// added to `graph` after `deps`.
template <int A, bool W>
int add_level_loop(Graph &g, cudaGraph_t graph, const cudaGraphNode_t *deps, size_t ndeps, const LevelCfg &cfg,
                   cudaGraphNode_t *out) {
  if (!g.cap_stream) RG_CUDA(cudaStreamCreateWithFlags(&g.cap_stream, cudaStreamNonBlocking));
  int rc = RG_OK;
  cudaError_t e = cudaSuccess;
  do {
    cudaGraphConditionalHandle wh;
    if ((e = cudaGraphConditionalHandleCreate(&wh, graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess) break;
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = wh;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    if ((e = cudaGraphAddNode(out, graph, deps, ndeps, &wp)) != cudaSuccess) break;
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    cudaGraphNode_t prev = nullptr;
    for (int half = 0; half < 2 && e == cudaSuccess && !rc; half++) {
      cudaGraphConditionalHandle sw;
      if ((e = cudaGraphConditionalHandleCreate(&sw, body, 0, 0)) != cudaSuccess) break;
      const uint32_t *fin = g.q[half];
      const unsigned long long *fin_n = &g.d.ctl[C_QN0 + half];
      unsigned long long *fout_n = &g.d.ctl[C_QN0 + (half ^ 1)];
      int use_switch = 1;
      LevelCfg c = cfg;
      void *args[] = {(void *)&g.d, (void *)&fin, (void *)&fin_n, (void *)&fout_n, (void *)&c, (void *)&use_switch,
                      (void *)&sw};
      cudaKernelNodeParams kp = {};
      kp.func = (void *)k_level_begin;
      kp.gridDim = dim3(1);
      kp.blockDim = dim3(LVB_TPB);
      kp.kernelParams = args;
      cudaGraphNode_t kn;
      if ((e = cudaGraphAddKernelNode(&kn, body, prev ? &prev : nullptr, prev ? 1 : 0, &kp)) != cudaSuccess) break;
      cudaGraphNodeParams sp = {};
      sp.type = cudaGraphNodeTypeConditional;
      sp.conditional.handle = sw;
      sp.conditional.type = cudaGraphCondTypeSwitch;
      sp.conditional.size = M_COUNT;
      cudaGraphNode_t sn;
      if ((e = cudaGraphAddNode(&sn, body, &kn, 1, &sp)) != cudaSuccess) break;
      for (unsigned long long m = 1; m < M_COUNT && e == cudaSuccess && !rc; m++) {
        if (m == M_PULL && !cfg.allow_pull) continue;
        if (m == M_BOTTOM_UP && !cfg.bottom_up) continue;
        if (m == M_CLUSTER && !cfg.cl_edges) continue;
        cudaGraph_t cg = sp.conditional.phGraph_out[m];
        if ((e = cudaStreamBeginCaptureToGraph(g.cap_stream, cg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed)) !=
            cudaSuccess)
          break;
        rc = enqueue_mode<A, W>(g, g.cap_stream, half, m);
        e = cudaStreamEndCapture(g.cap_stream, &cg);
      }
      prev = sn;
    }
    if (e != cudaSuccess || rc) break;
    const unsigned long long *n_after = &g.d.ctl[C_QN0];
    uint64_t maxl = max_levels_of(g);
    void *cargs[] = {(void *)&g.d, (void *)&n_after, (void *)&maxl, (void *)&wh};
    cudaKernelNodeParams cp = {};
    cp.func = (void *)k_loop_cond;
    cp.gridDim = dim3(1);
    cp.blockDim = dim3(1);
    cp.kernelParams = cargs;
    cudaGraphNode_t cn;
    e = cudaGraphAddKernelNode(&cn, body, &prev, 1, &cp);
  } while (0);
  if (e != cudaSuccess) return cuda_fail(e, "building the level-loop graph");
  return rc;
}

// Deletion repair as nodes of a CUDA graph (do_update_tree_del,
// core/graph.hpp:1235-1612):
//   k_del_tiny (small repairs in one CTA) -> IF (it handed over) {
//     WHILE (invalidated frontier non-empty and no recompute) {
//       k_inv_begin ; k_rescue ; k_expand     (queue 0 -> 1)
//       k_inv_begin ; k_rescue ; k_expand     (queue 1 -> 0)
//       k_inv_cond }
//     k_reset ; k_pull ; k_copy_frontier (reset set -> queue 0 for the push loop) }
// *out is the IF node.  With `fused` (the fused apply kernel ran the one-CTA
// repair and left its hand-over decision in C_OVER) the first node is
// k_handover instead of k_del_tiny.
template <int A, bool W>
int add_del_repair(Graph &g, cudaGraph_t graph, const cudaGraphNode_t *deps, size_t ndeps, cudaGraphNode_t *out,
                   bool fused = false) {
  if (!g.cap_stream) RG_CUDA(cudaStreamCreateWithFlags(&g.cap_stream, cudaStreamNonBlocking));
  const uint64_t big = recompute_threshold(g);
  const uint64_t limit = (uint64_t)((double)g.V * 0.1);  // has_parents guard, core/graph.hpp:1900
  uint32_t mst = mod_stamp(g);
  const int gridw = g.num_sms * 16;
  cudaError_t e = cudaSuccess;
  do {
    cudaGraphConditionalHandle th;
    if ((e = cudaGraphConditionalHandleCreate(&th, graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess) break;
    uint32_t *q0 = g.q[0], *q1 = g.q[1], *tr = g.tree;
    uint64_t max_iter = (uint64_t)g.V + 2;
    int in_graph = 1;
    void *ta[] = {(void *)&g.d, (void *)&q0, (void *)&q1, (void *)&tr, (void *)&limit, (void *)&big,
                  (void *)&max_iter, (void *)&mst, (void *)&th, (void *)&in_graph};
    void *hoa[] = {(void *)&g.d, (void *)&th};
    cudaKernelNodeParams tp = {};
    tp.func = fused ? (void *)k_handover : (void *)k_del_tiny<A, W>;
    tp.gridDim = dim3(1);
    tp.blockDim = dim3(fused ? 1 : DT_TPB);
    tp.kernelParams = fused ? hoa : ta;
    cudaGraphNode_t tn;
    if ((e = cudaGraphAddKernelNode(&tn, graph, deps, ndeps, &tp)) != cudaSuccess) break;
    cudaGraphNodeParams ip = {};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = th;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    if ((e = cudaGraphAddNode(out, graph, &tn, 1, &ip)) != cudaSuccess) break;
    graph = ip.conditional.phGraph_out[0];  // the multi-CTA repair below goes into the IF body
    deps = nullptr;
    ndeps = 0;
    cudaGraphConditionalHandle wh;
    if ((e = cudaGraphConditionalHandleCreate(&wh, graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess) break;
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = wh;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wnode;
    if ((e = cudaGraphAddNode(&wnode, graph, deps, ndeps, &wp)) != cudaSuccess) break;
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    if ((e = cudaStreamBeginCaptureToGraph(g.cap_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed)) !=
        cudaSuccess)
      break;
    for (int half = 0; half < 2; half++) {
      unsigned long long *fin_n = &g.d.ctl[C_QN0 + half], *fout_n = &g.d.ctl[C_QN0 + (half ^ 1)];
      k_inv_begin<<<1, 1, 0, g.cap_stream>>>(g.d, fin_n, fout_n, big);
      k_rescue<A, W><<<gridw, TPB, 0, g.cap_stream>>>(g.d, g.q[half], fin_n, limit);
      k_rescue_heavy<A, W><<<gridw, TPB, 0, g.cap_stream>>>(g.d, limit);
      k_expand<A, W><<<gridw, TPB, 0, g.cap_stream>>>(g.d, g.q[half], fin_n, g.tree, g.q[half ^ 1], fout_n);
      k_expand_heavy<A, W><<<gridw, TPB, 0, g.cap_stream>>>(g.d, g.q[half ^ 1], fout_n);
    }
    k_inv_cond<<<1, 1, 0, g.cap_stream>>>(g.d, &g.d.ctl[C_QN0], (uint64_t)g.V + 2, wh, 1);
    if ((e = cudaStreamEndCapture(g.cap_stream, &body)) != cudaSuccess) break;
    // k_reset -> k_pull -> k_copy_frontier after the loop
    unsigned long long *tree_n = &g.d.ctl[C_TREEN], *q0_n = &g.d.ctl[C_QN0];
    const uint32_t *tree = g.tree;
    void *ra[] = {(void *)&g.d, (void *)&tree, (void *)&tree_n, (void *)&mst};
    void *ca[] = {(void *)&g.d, (void *)&tree, (void *)&tree_n, (void *)&q0, (void *)&q0_n};
    cudaKernelNodeParams kp = {};
    kp.gridDim = dim3(gridw);
    kp.blockDim = dim3(TPB);
    kp.func = (void *)k_reset<A>;
    kp.kernelParams = ra;
    cudaGraphNode_t n1, n2;
    if ((e = cudaGraphAddKernelNode(&n1, graph, &wnode, 1, &kp)) != cudaSuccess) break;
    kp.func = (void *)k_pull<A, W>;
    if ((e = cudaGraphAddKernelNode(&n2, graph, &n1, 1, &kp)) != cudaSuccess) break;
    void *ha[] = {(void *)&g.d, (void *)&mst};
    kp.func = (void *)k_pull_heavy<A, W>;
    kp.kernelParams = ha;
    cudaGraphNode_t n2h;
    if ((e = cudaGraphAddKernelNode(&n2h, graph, &n2, 1, &kp)) != cudaSuccess) break;
    kp.func = (void *)k_copy_frontier;
    kp.gridDim = dim3(g.num_sms * 4);
    kp.kernelParams = ca;
    cudaGraphNode_t n3;
    e = cudaGraphAddKernelNode(&n3, graph, &n2h, 1, &kp);
  } while (0);
  if (e != cudaSuccess) return cuda_fail(e, "building the deletion-repair graph");
  return RG_OK;
}

// Cached standalone level loop per (algorithm, weighting, variant), rebuilt
// when the pool is relocated by a compaction or an option changes.
template <int A, bool W>
int loop_exec(Graph &g, bool build_variant, cudaGraphExec_t *out) {
  const LevelCfg cfg = level_cfg(g, A, build_variant);
  LoopGraph &slot = g.loops[(A * 2 + (W ? 1 : 0)) * 2 + (build_variant ? 1 : 0)];
  const uint64_t key = cfg_key(cfg) ^ splitmix64(g.layout_version) ^ splitmix64(build_variant ? g.sell_epoch + 5 : 0);
  if (slot.exec && slot.key == key) {
    *out = slot.exec;
    return RG_OK;
  }
  if (slot.exec) {
    cudaGraphExecDestroy(slot.exec);
    slot.exec = nullptr;
  }
  cudaGraph_t graph;
  RG_CUDA(cudaGraphCreate(&graph, 0));
  cudaGraphNode_t node;
  int rc = add_level_loop<A, W>(g, graph, nullptr, 0, cfg, &node);
  if (!rc) {
    cudaError_t e = cudaGraphInstantiate(&slot.exec, graph, 0);
    if (e != cudaSuccess) {
      slot.exec = nullptr;
      rc = cuda_fail(e, "instantiating the level-loop graph");
    }
  }
  cudaGraphDestroy(graph);
  if (rc) return rc;
  slot.key = key;
  *out = slot.exec;
  return RG_OK;
}

// Push levels to a fixpoint from the frontier in queue 0 (do_update_tree_add,
// core/graph.hpp:1013-1111; build_tree :898-983).  Enqueues one graph launch;
// with profiling on, the host runs the same kernels level by level (syncing)
// so each level can be timed.
template <int A, bool W>
int push_levels(Graph &g, bool build_variant) {
  if (build_variant && pull_on(g, A)) {
    int rc = prepare_pull(g);
    if (rc) return rc;
  }
  if (!g.profiling) {
    cudaGraphExec_t exec;
    int rc = loop_exec<A, W>(g, build_variant, &exec);
    if (rc) return rc;
    RG_CUDA(cudaGraphLaunch(exec, g.stream));
    return RG_OK;
  }
  const LevelCfg cfg = level_cfg(g, A, build_variant);
  int rc = read_ctl(g);
  if (rc) return rc;
  for (int half = 0; g.h_ctl[C_QN0 + half]; half ^= 1) {
    if (g.h_ctl[C_LEVEL] >= max_levels_of(g)) {
      set_error("push levels did not converge");
      return RG_ETIMEOUT;
    }
    RG_CUDA(cudaEventRecord(g.pev[0], g.stream));
    count_launch(g);
    k_level_begin<<<1, LVB_TPB, 0, g.stream>>>(g.d, g.q[half], &g.d.ctl[C_QN0 + half], &g.d.ctl[C_QN0 + (half ^ 1)],
                                                cfg, 0, cudaGraphConditionalHandle{});
    if ((rc = read_ctl(g))) return rc;
    const unsigned long long mode = g.h_ctl[C_MODE];
    count_launch(g, mode_launches(mode));
    if ((rc = enqueue_mode<A, W>(g, g.stream, half, mode))) return rc;
    RG_CUDA(cudaEventRecord(g.pev[1], g.stream));
    if ((rc = read_ctl(g))) return rc;
    float ms = 0.f;
    RG_CUDA(cudaEventElapsedTime(&ms, g.pev[0], g.pev[1]));
    g.prof_ms += ms;
    g.prof_launches += 1;
    g.st_level_ms.push_back(ms);
  }
  return RG_OK;
}


// Cached standalone deletion repair (the push loop follows as its own graph).
template <int A, bool W>
int del_exec(Graph &g, bool fused, cudaGraphExec_t *out) {
  LoopGraph &slot = g.dels[(A * 2 + (W ? 1 : 0)) * 2 + (fused ? 1 : 0)];
  const uint64_t key = (g.layout_version << 40) ^ recompute_threshold(g);
  if (slot.exec && slot.key == key) {
    *out = slot.exec;
    return RG_OK;
  }
  if (slot.exec) {
    cudaGraphExecDestroy(slot.exec);
    slot.exec = nullptr;
  }
  cudaGraph_t graph;
  RG_CUDA(cudaGraphCreate(&graph, 0));
  cudaGraphNode_t last;
  int rc = add_del_repair<A, W>(g, graph, nullptr, 0, &last, fused);
  if (!rc) {
    cudaError_t e = cudaGraphInstantiate(&slot.exec, graph, 0);
    if (e != cudaSuccess) {
      slot.exec = nullptr;
      rc = cuda_fail(e, "instantiating the deletion-repair graph");
    }
  }
  cudaGraphDestroy(graph);
  if (rc) return rc;
  slot.key = key;
  *out = slot.exec;
  return RG_OK;
}

// The deletion repair of add_del_repair launched kernel by kernel from the
// host (profile mode): the same kernels in the same order, with the IF and
// WHILE decisions read back through C_HOSTCOND, so that every kernel is a
// plain launch a profiler lists.
template <int A, bool W>
int del_repair_stepped(Graph &g) {
  const uint64_t big = recompute_threshold(g);
  const uint64_t limit = (uint64_t)((double)g.V * 0.1);  // has_parents guard, core/graph.hpp:1900
  const uint32_t mst = mod_stamp(g);
  const int gridw = g.num_sms * 16;
  const uint64_t max_iter = (uint64_t)g.V + 2;
  count_launch(g);
  k_del_tiny<A, W><<<1, DT_TPB, 0, g.stream>>>(g.d, g.q[0], g.q[1], g.tree, limit, big, max_iter, mst,
                                               cudaGraphConditionalHandle{}, 0);
  RG_CUDA(cudaGetLastError());
  int rc = read_ctl(g);
  if (rc) return rc;
  if (!g.h_ctl[C_HOSTCOND]) return RG_OK;
  for (uint64_t it = 0;; it++) {
    if (it > max_iter) {
      set_error("deletion repair did not converge");
      return RG_ETIMEOUT;
    }
    for (int half = 0; half < 2; half++) {
      unsigned long long *fin_n = &g.d.ctl[C_QN0 + half], *fout_n = &g.d.ctl[C_QN0 + (half ^ 1)];
      count_launch(g, 5);
      k_inv_begin<<<1, 1, 0, g.stream>>>(g.d, fin_n, fout_n, big);
      k_rescue<A, W><<<gridw, TPB, 0, g.stream>>>(g.d, g.q[half], fin_n, limit);
      k_rescue_heavy<A, W><<<gridw, TPB, 0, g.stream>>>(g.d, limit);
      k_expand<A, W><<<gridw, TPB, 0, g.stream>>>(g.d, g.q[half], fin_n, g.tree, g.q[half ^ 1], fout_n);
      k_expand_heavy<A, W><<<gridw, TPB, 0, g.stream>>>(g.d, g.q[half ^ 1], fout_n);
    }
    count_launch(g);
    k_inv_cond<<<1, 1, 0, g.stream>>>(g.d, &g.d.ctl[C_QN0], max_iter, cudaGraphConditionalHandle{}, 0);
    RG_CUDA(cudaGetLastError());
    if ((rc = read_ctl(g))) return rc;
    if (!g.h_ctl[C_HOSTCOND]) break;
  }
  count_launch(g, 4);
  k_reset<A><<<gridw, TPB, 0, g.stream>>>(g.d, g.tree, &g.d.ctl[C_TREEN], mst);
  k_pull<A, W><<<gridw, TPB, 0, g.stream>>>(g.d, g.tree, &g.d.ctl[C_TREEN], mst);
  k_pull_heavy<A, W><<<gridw, TPB, 0, g.stream>>>(g.d, mst);
  k_copy_frontier<<<g.num_sms * 4, TPB, 0, g.stream>>>(g.d, g.tree, &g.d.ctl[C_TREEN], g.q[0], &g.d.ctl[C_QN0]);
  RG_CUDA(cudaGetLastError());
  return RG_OK;
}

template <int A, bool W>
int build_enqueue(Graph &g, uint64_t root) {
  int rc = guard_counters(g);
  if (rc) return rc;
  count_launch(g, 2);
  k_prologue<<<1, 1, 0, g.stream>>>(g.d, 0ull);
  k_init<A><<<g.num_sms * 16, TPB, 0, g.stream>>>(g.d, root, g.q[0]);
  RG_CUDA(cudaGetLastError());
  return push_levels<A, W>(g, true);
}

template <int A, bool W>
int add_enqueue(Graph &g, uint64_t n_edges, int directed, bool from_cands) {
  int rc = guard_counters(g);
  if (rc) return rc;
  count_launch(g, 2);
  k_prologue<<<1, 1, 0, g.stream>>>(g.d, 0ull);
  k_seed_add<A><<<grid_warps(g, (n_edges + 31) / 32), TPB, 0, g.stream>>>(
      g.d, op_src(g), op_dst(g), op_w(g), from_cands ? op_cand(g) : nullptr, &g.d.ctl[C_CANDN], n_edges, directed,
      g.q[0], &g.d.ctl[C_QN0], mod_stamp(g));
  RG_CUDA(cudaGetLastError());
  return push_levels<A, W>(g, false);
}

template <int A, bool W>
int del_enqueue(Graph &g, uint64_t n_edges, int directed, bool from_cands) {
  int rc = guard_counters(g);
  if (rc) return rc;
  if (++g.inv_epoch >= 0x7FFFFFFFu) {
    RG_CUDA(cudaMemsetAsync(g.d.inv, 0, (size_t)g.V * 4, g.stream));
    RG_CUDA(cudaMemsetAsync(g.d.chk, 0, (size_t)g.V * 4, g.stream));
    g.inv_epoch = 1;
  }
  const unsigned long long tag = 2ull * g.inv_epoch;  // tag: invalidated; tag+1: rescued
  count_launch(g, 2);
  k_prologue<<<1, 1, 0, g.stream>>>(g.d, tag);
  k_seed_del<<<grid_warps(g, (n_edges + 31) / 32), TPB, 0, g.stream>>>(
      g.d, op_src(g), op_dst(g), op_w(g), from_cands ? op_cand(g) : nullptr, &g.d.ctl[C_CANDN], n_edges, directed,
      g.q[0], &g.d.ctl[C_QN0]);
  RG_CUDA(cudaGetLastError());
  if (g.profiling) {
    rc = del_repair_stepped<A, W>(g);
  } else {
    cudaGraphExec_t exec;
    if ((rc = del_exec<A, W>(g, false, &exec))) return rc;
    RG_CUDA(cudaGraphLaunch(exec, g.stream));
  }
  if (rc) return rc;
  return push_levels<A, W>(g, false);
}

// After the stream has been synchronised and h_ctl read: errors, statistics
// and the full-recompute fallback of a deletion repair.
template <int A, bool W>
int after_sync(Graph &g, int what) {
  if (g.h_ctl[C_ERR]) {
    int code = (int)g.h_ctl[C_ERR];
    set_error(code == RG_ETIMEOUT ? "push levels did not converge" : "device error in tree update");
    cudaMemsetAsync(&g.d.ctl[C_ERR], 0, 8, g.stream);
    return code;
  }
  g.launches += g.h_ctl[C_KLAUNCH];  // kernels run inside graphs, counted on the device
  g.st_levels = g.h_ctl[C_LEVEL];
  if (what == 2) {
    g.st_invalidated = g.h_ctl[C_TREEN];
    if (g.h_ctl[C_RECOMPUTE]) {
      g.st_recomputes++;
      RG_CUDA(cudaMemsetAsync(g.d.inv, 0, (size_t)g.V * 4, g.stream));
      RG_CUDA(cudaMemsetAsync(g.d.chk, 0, (size_t)g.V * 4, g.stream));
      g.inv_epoch = 0;
      int rc = build_enqueue<A, W>(g, g.root);
      if (!rc) rc = read_ctl(g);
      if (!rc) rc = after_sync<A, W>(g, 0);
      return rc;
    }
  }
  return RG_OK;
}

template <int A, bool W>
int run_what(Graph &g, int what, uint64_t a, int directed, bool from_cands, int phase) {
  if (phase == 1) return after_sync<A, W>(g, what);
  if (what == 0) return build_enqueue<A, W>(g, a);
  if (what == 1) return add_enqueue<A, W>(g, a, directed, from_cands);
  return del_enqueue<A, W>(g, a, directed, from_cands);
}

template <int A>
int dispatch_w(Graph &g, int what, uint64_t a, int directed, bool from_cands, int phase) {
  if (g.weighted) return run_what<A, true>(g, what, a, directed, from_cands, phase);
  return run_what<A, false>(g, what, a, directed, from_cands, phase);
}

// phase 0: enqueue the call's device work; phase 1: finish it after a sync.
int dispatch(Graph &g, int algo, int what, uint64_t a, int directed, bool from_cands, int phase) {
  switch (algo) {
    case RG_BFS: return dispatch_w<RG_BFS>(g, what, a, directed, from_cands, phase);
    case RG_SSSP: return dispatch_w<RG_SSSP>(g, what, a, directed, from_cands, phase);
    case RG_SSWP: return dispatch_w<RG_SSWP>(g, what, a, directed, from_cands, phase);
    case RG_WCC: return dispatch_w<RG_WCC>(g, what, a, directed, from_cands, phase);
  }
  set_error("unknown algorithm");
  return RG_EINVAL;
}

}  // namespace

// CTAs of the cluster-level kernel: 16 where this GPU schedules a cluster of
// sixteen 1024-thread CTAs, else the portable 8; 0 (cluster levels off) when
// neither can run.
template <int A, bool W>
void cluster_allow(cudaError_t &e) {
  cudaError_t x = cudaFuncSetAttribute(k_push_cluster<A, W>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (x != cudaSuccess) e = x;
}

static void cluster_setup(Graph &g) {
  cudaError_t e = cudaSuccess;
  cluster_allow<RG_BFS, false>(e);
  cluster_allow<RG_BFS, true>(e);
  cluster_allow<RG_SSSP, false>(e);
  cluster_allow<RG_SSSP, true>(e);
  cluster_allow<RG_SSWP, false>(e);
  cluster_allow<RG_SSWP, true>(e);
  cluster_allow<RG_WCC, false>(e);
  cluster_allow<RG_WCC, true>(e);
  g.cl_ctas = 0;
  for (int n : {CL_MAX_CTAS, 8}) {
    if (e != cudaSuccess && n > 8) continue;  // without the attribute only the portable size
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)n);
    lc.blockDim = dim3(CL_TPB);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)n;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k_push_cluster<RG_SSSP, true>, &lc) == cudaSuccess && clusters > 0) {
      g.cl_ctas = n;
      break;
    }
  }
  cudaGetLastError();
}

int tree_alloc(Graph &g) {
  uint64_t V = g.V;
  cluster_setup(g);
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
  if ((rc = alloc((void **)&g.d.val32, V * 4 + 4, "label value mirror"))) return rc;
  RG_CUDA(cudaMemset(g.d.val32, 0, V * 4 + 4));
  if ((rc = alloc((void **)&g.d.stamp, V * 4 + 4, "frontier stamps"))) return rc;
  if ((rc = alloc((void **)&g.d.inv, V * 4 + 4, "invalidation tags"))) return rc;
  if ((rc = alloc((void **)&g.d.chk, V * 4 + 4, "clear-chain marks"))) return rc;
  // at most (edge slots / HEAVY_DEG) vertices have a longer list
  g.d.heavy_cap = std::max(g.d.out.pool_cap, g.d.in.pool_cap) / HEAVY_DEG + 1024;
  if ((rc = alloc((void **)&g.d.heavy, 3 * g.d.heavy_cap * 4, "heavy-vertex lists"))) return rc;
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
  if ((rc = alloc((void **)&g.lb_sums, SC_BLOCKS * 8, "scan block sums"))) return rc;
  if ((rc = alloc((void **)&g.sell_cnt, 64, "pull counters"))) return rc;
  RG_CUDA(cudaMemset(g.act, 0, V * 4 + 4));
  if ((rc = alloc((void **)&g.lb_tile, (g.d.out.pool_cap / LB_TILE + 4) * 4, "tile partition"))) return rc;
  g.cub_tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, g.cub_tmp_bytes, g.scratch64, g.lb_P, V + 1);
  if ((rc = alloc(&g.cub_tmp, g.cub_tmp_bytes + 256, "scan scratch"))) return rc;
  if ((rc = alloc((void **)&g.d.ctl, sizeof(unsigned long long) * C_COUNT, "control block"))) return rc;
  RG_CUDA(cudaMemset(g.d.ctl, 0, sizeof(unsigned long long) * C_COUNT));
  {
    unsigned long long one = 1;
    RG_CUDA(cudaMemcpy(&g.d.ctl[C_MODEPOCH], &one, 8, cudaMemcpyHostToDevice));
  }
  // frontier sizes, then the levels' start stamps (one more: the end of the last)
  if ((rc = alloc((void **)&g.d.trace, (2 * TRACE_CAP + 1) * 8, "level trace"))) return rc;
  if ((rc = alloc((void **)&g.ptrace_buf, RG_PHASE_SLOTS * 8, "phase trace"))) return rc;
  RG_CUDA(cudaMemset(g.ptrace_buf, 0, RG_PHASE_SLOTS * 8));
  g.d.ptrace = g.phase_trace ? g.ptrace_buf : nullptr;
  RG_CUDA(cudaMemset(g.d.stamp, 0, V * 4 + 4));
  RG_CUDA(cudaMemset(g.d.inv, 0, V * 4 + 4));
  RG_CUDA(cudaMemset(g.d.chk, 0, V * 4 + 4));
  RG_CUDA(cudaMemset(g.d.modstamp, 0, V * 4 + 4));
  // labels start as "no parent", value 0 until build_tree (alloc_vertex_tree_array, :255-262)
  RG_CUDA(cudaMemset(g.d.lab, 0, V * 16 + 16));
  return RG_OK;
}

static void reset_stats(Graph &g) {
  g.st_levels = g.st_invalidated = g.st_recomputes = 0;
  g.st_level_ms.clear();
}

int tree_enqueue(Graph &g, int what, uint64_t n_edges, int directed, bool from_cands) {
  reset_stats(g);
  return dispatch(g, g.algo, what, n_edges, directed, from_cands, 0);
}

int tree_after_sync(Graph &g, int what, uint64_t *total) {
  int rc = dispatch(g, g.algo, what, 0, 1, false, 1);
  if (rc) return rc;
  if (total) *total = g.h_ctl[C_RESULT];
  return RG_OK;
}

int tree_build(Graph &g, int algo, uint64_t root, uint64_t *total) {
  reset_stats(g);
  g.algo = algo;
  g.root = root;
  int rc = dispatch(g, algo, 0, root, 1, false, 0);
  if (!rc) rc = read_ctl(g);
  if (!rc) rc = tree_after_sync(g, 0, total);
  return rc;
}

int tree_add(Graph &g, uint64_t n_edges, int directed, bool from_cands, uint64_t *total) {
  int rc = tree_enqueue(g, 1, n_edges, directed, from_cands);
  if (!rc) rc = read_ctl(g);
  if (!rc) rc = tree_after_sync(g, 1, total);
  return rc;
}

int tree_del(Graph &g, uint64_t n_edges, int directed, bool from_cands, uint64_t *total) {
  int rc = tree_enqueue(g, 2, n_edges, directed, from_cands);
  if (!rc) rc = read_ctl(g);
  if (!rc) rc = tree_after_sync(g, 2, total);
  return rc;
}

FusedRepair fused_repair(const Graph &g, const LevelCfg &cfg) {
  FusedRepair fr = {};
  fr.q1 = g.q[1];
  fr.tree = g.tree;
  fr.limit = (uint64_t)((double)g.V * 0.1);  // has_parents guard, core/graph.hpp:1900
  fr.big = recompute_threshold(g);
  fr.max_iter = (uint64_t)g.V + 2;
  fr.max_levels = cfg.max_levels;
  fr.tiny_edges = cfg.tiny_edges;
  return fr;
}

// The fused kernel for one batch as a graph node after `deps`: k_apply_small
// with the header at hdr_off of the staging buffer (second: the delete batch
// of an insert+delete submission, whose edges start at apply_data2_off()).
template <int A, bool W>
int add_apply_kernel(Graph &g, cudaGraph_t graph, const cudaGraphNode_t *deps, size_t ndeps, bool add, int directed,
                     uint64_t hdr_off, int second, const LevelCfg &cfg, cudaGraphNode_t *out) {
  sdev::OpView ops = sdev::op_view(g);
  char *base = reinterpret_cast<char *>(g.stage_host_dev);
  const ApplyHdr *hdr = reinterpret_cast<const ApplyHdr *>(base + hdr_off);
  const char *data = base + APPLY_DATA_OFF + (second ? apply_data2_off() : 0);
  uint64_t *old_host = reinterpret_cast<uint64_t *>(base + apply_old_off());
  uint4 *scratch = reinterpret_cast<uint4 *>(g.stage_dev);
  uint32_t *cand = op_cand(g);
  int a_add = add ? 1 : 0, a_dir = directed ? 1 : 0, a_second = second;
  uint32_t *q0 = g.q[0];
  uint32_t mst = mod_stamp(g);
  FusedRepair fr = fused_repair(g, cfg);
  unsigned long long *ctl_host = g.h_ctl_dev;
  void *args[] = {(void *)&g.d,    (void *)&ops, (void *)&hdr, (void *)&data,   (void *)&old_host,
                  (void *)&cand,   (void *)&a_add, (void *)&a_dir, (void *)&q0, (void *)&mst,
                  (void *)&a_second, (void *)&fr, (void *)&scratch, (void *)&ctl_host};
  cudaKernelNodeParams kp = {};
  kp.func = (void *)k_apply_small<A, W>;
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(FS_TPB);
  kp.kernelParams = args;
  cudaError_t e = cudaGraphAddKernelNode(out, graph, deps, ndeps, &kp);
  return e == cudaSuccess ? RG_OK : cuda_fail(e, "building the fused apply graph");
}

uint64_t apply_key(const Graph &g, const LevelCfg &cfg) {
  return splitmix64(g.layout_version) ^ splitmix64((uint64_t)(uintptr_t)g.ops ^ (g.ops_cap << 1)) ^
         splitmix64((uint64_t)(uintptr_t)g.d.ptrace + 17) ^ splitmix64((uint64_t)(uintptr_t)g.h_ctl_dev + 19) ^
         splitmix64((uint64_t)(uintptr_t)g.stage_host_dev + 7) ^ splitmix64((uint64_t)(uintptr_t)g.stage_dev + 13) ^
         cfg_key(cfg) ^ splitmix64(recompute_threshold(g) + 11);
}

// A cached graph: `build` adds its nodes; rebuilt when `key` changes.
template <typename F>
int cached_graph(LoopGraph &slot, uint64_t key, F build, const char *what, cudaGraphExec_t *out) {
  if (slot.exec && slot.key == key) {
    *out = slot.exec;
    return RG_OK;
  }
  if (slot.exec) {
    cudaGraphExecDestroy(slot.exec);
    slot.exec = nullptr;
  }
  cudaGraph_t graph;
  RG_CUDA(cudaGraphCreate(&graph, 0));
  int rc = build(graph);
  if (!rc) {
    cudaError_t e = cudaGraphInstantiate(&slot.exec, graph, 0);
    if (e != cudaSuccess) {
      slot.exec = nullptr;
      rc = cuda_fail(e, what);
    }
  }
  cudaGraphDestroy(graph);
  if (rc) return rc;
  slot.key = key;
  *out = slot.exec;
  return RG_OK;
}

// Insert batch then delete batch: one node, k_apply_mixed (both batches, and
// their repairs while they stay small).
template <int A, bool W>
int mixed_exec(Graph &g, int directed, cudaGraphExec_t *out) {
  const LevelCfg cfg = level_cfg(g, A, false);
  auto build = [&](cudaGraph_t graph) -> int {
    sdev::OpView ops = sdev::op_view(g);
    char *base = reinterpret_cast<char *>(g.stage_host_dev);
    const ApplyHdr *hdr1 = reinterpret_cast<const ApplyHdr *>(base);
    const ApplyHdr *hdr2 = reinterpret_cast<const ApplyHdr *>(base + APPLY_HDR2);
    const char *data1 = base + APPLY_DATA_OFF, *data2 = base + APPLY_DATA_OFF + apply_data2_off();
    uint4 *scr1 = reinterpret_cast<uint4 *>(g.stage_dev);
    uint4 *scr2 = reinterpret_cast<uint4 *>(reinterpret_cast<char *>(g.stage_dev) + apply_data2_off());
    uint32_t *cand = op_cand(g), *q0 = g.q[0];
    int a_dir = directed ? 1 : 0;
    uint32_t mst = mod_stamp(g);
    FusedRepair fr = fused_repair(g, cfg);
    unsigned long long *ctl_host = g.h_ctl_dev;
    void *args[] = {(void *)&g.d,  (void *)&ops,   (void *)&hdr1, (void *)&data1, (void *)&hdr2,
                    (void *)&data2, (void *)&cand, (void *)&a_dir, (void *)&q0,   (void *)&mst,
                    (void *)&fr,   (void *)&scr1,  (void *)&scr2, (void *)&ctl_host};
    cudaKernelNodeParams kp = {};
    kp.func = (void *)k_apply_mixed<A, W>;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(FS_TPB);
    kp.kernelParams = args;
    cudaGraphNode_t kn;
    cudaError_t e = cudaGraphAddKernelNode(&kn, graph, nullptr, 0, &kp);
    return e == cudaSuccess ? RG_OK : cuda_fail(e, "building the fused insert+delete graph");
  };
  return cached_graph(g.mixes[(A * 2 + (W ? 1 : 0)) * 2 + (directed ? 1 : 0)], apply_key(g, cfg), build,
                      "instantiating the fused insert+delete graph", out);
}

// After k_apply_mixed left the insert batch's level loop: that loop, then the
// delete batch in its own fused kernel (k_apply_small, second batch).
template <int A, bool W>
int rest_exec(Graph &g, int directed, cudaGraphExec_t *out) {
  const LevelCfg cfg = level_cfg(g, A, false);
  auto build = [&](cudaGraph_t graph) -> int {
    cudaGraphNode_t loop, kn;
    int rc = add_level_loop<A, W>(g, graph, nullptr, 0, cfg, &loop);
    if (!rc) rc = add_apply_kernel<A, W>(g, graph, &loop, 1, false, directed, APPLY_HDR2, 1, cfg, &kn);
    return rc;
  };
  return cached_graph(g.rests[(A * 2 + (W ? 1 : 0)) * 2 + (directed ? 1 : 0)], apply_key(g, cfg), build,
                      "instantiating the insert loop + delete batch graph", out);
}

// One batch: one node, k_apply_small.  Its parameters hold the op, staging and
// pool addresses, so it is rebuilt when any of them moves.
template <int A, bool W>
int apply_exec(Graph &g, bool add, int directed, cudaGraphExec_t *out) {
  const LevelCfg cfg = level_cfg(g, A, false);
  auto build = [&](cudaGraph_t graph) -> int {
    cudaGraphNode_t kn;
    return add_apply_kernel<A, W>(g, graph, nullptr, 0, add, directed, 0, 0, cfg, &kn);
  };
  return cached_graph(g.applies[((A * 2 + (W ? 1 : 0)) * 2 + (add ? 1 : 0)) * 2 + (directed ? 1 : 0)],
                      apply_key(g, cfg), build, "instantiating the fused apply graph", out);
}

// What a fused kernel left (C_LEFT in the host's copy of the control block):
// 1 the insert batch's level loop; 2 the delete batch's repair, that is the
// grid-wide deletion repair when the one-CTA repair handed over (k_handover
// reads C_OVER) and then the level loop.  Ends with the control block read
// back.
template <int A, bool W>
int finish_left(Graph &g, unsigned long long left) {
  int rc = RG_OK;
  if (left == 2) {
    cudaGraphExec_t de;
    if ((rc = del_exec<A, W>(g, true, &de))) return rc;
    RG_CUDA(cudaGraphLaunch(de, g.stream));
  }
  cudaGraphExec_t le;
  if ((rc = loop_exec<A, W>(g, false, &le))) return rc;
  RG_CUDA(cudaGraphLaunch(le, g.stream));
  return read_ctl(g);
}

// An inline batch from the caller's edges (n <= INLINE_EDGES).
InlineBatch inline_batch(const void *src, uint64_t n, bool pairs, bool want, uint64_t inv_tag) {
  InlineBatch ib;
  ib.n = n;
  ib.pairs = pairs ? 1 : 0;
  ib.want = want ? 1 : 0;
  ib.inv_tag = inv_tag;
  std::memset(ib.words, 0, sizeof(ib.words));
  std::memcpy(ib.words, src, n * (pairs ? 16 : sizeof(rg_edge)));
  return ib;
}

// One batch of at most INLINE_EDGES edges: k_apply_small_inl, launched
// directly with the batch in its parameters.
template <int A, bool W>
int launch_apply_inline(Graph &g, const InlineBatch &ib, bool add, int directed) {
  const LevelCfg cfg = level_cfg(g, A, false);
  uint64_t *old_host = reinterpret_cast<uint64_t *>(reinterpret_cast<char *>(g.stage_host_dev) + apply_old_off());
  k_apply_small_inl<A, W><<<1, FS_TPB, 0, g.stream>>>(g.d, sdev::op_view(g), ib, old_host, op_cand(g), add ? 1 : 0,
                                                      directed ? 1 : 0, g.q[0], mod_stamp(g), fused_repair(g, cfg),
                                                      g.h_ctl_dev);
  RG_CUDA(cudaGetLastError());
  return RG_OK;
}

// An insert batch and a delete batch of at most INLINE_EDGES edges each:
// k_apply_mixed_inl.
template <int A, bool W>
int launch_mixed_inline(Graph &g, const InlineBatch &ib1, const InlineBatch &ib2, int directed) {
  const LevelCfg cfg = level_cfg(g, A, false);
  k_apply_mixed_inl<A, W><<<1, FS_TPB, 0, g.stream>>>(g.d, sdev::op_view(g), ib1, ib2, op_cand(g), directed ? 1 : 0,
                                                      g.q[0], mod_stamp(g), fused_repair(g, cfg), g.h_ctl_dev);
  RG_CUDA(cudaGetLastError());
  return RG_OK;
}

template <int A, bool W>
int apply_small_t(Graph &g, const rg_edge *edges, const uint64_t *pairs, uint64_t n, int directed, bool add,
                  uint64_t *old_num) {
  int rc = storage_reserve(g, 3 * SMALL_EDGES);  // op arrays and staging sized once for the small path
  if (rc) return rc;
  char *st = reinterpret_cast<char *>(g.stage_host);
  ApplyHdr *h = reinterpret_cast<ApplyHdr *>(st);
  std::memcpy(st + APPLY_DATA_OFF, pairs ? (const void *)pairs : (const void *)edges,
              n * (pairs ? 16 : sizeof(rg_edge)));
  h->n = n;
  h->pairs = pairs ? 1 : 0;
  h->want_old = old_num ? 1 : 0;
  h->inv_tag = 0;
  h->data_off = 0;
  g.adj_version++;
  if ((rc = guard_counters(g))) return rc;
  if (!add) {
    if (++g.inv_epoch >= 0x7FFFFFFFu) {
      RG_CUDA(cudaMemsetAsync(g.d.inv, 0, (size_t)g.V * 4, g.stream));
      RG_CUDA(cudaMemsetAsync(g.d.chk, 0, (size_t)g.V * 4, g.stream));
      g.inv_epoch = 1;
    }
    h->inv_tag = 2ull * g.inv_epoch;  // tag: invalidated; tag+1: rescued
  }
  reset_stats(g);
  count_launch(g);
  if (n <= g.inline_max) {
    const InlineBatch ib = inline_batch(pairs ? (const void *)pairs : (const void *)edges, n, pairs != nullptr,
                                        old_num != nullptr, h->inv_tag);
    if ((rc = launch_apply_inline<A, W>(g, ib, add, directed))) return rc;
  } else {
    cudaGraphExec_t exec;
    if ((rc = apply_exec<A, W>(g, add, directed, &exec))) return rc;
    RG_CUDA(cudaGraphLaunch(exec, g.stream));
  }
  RG_CUDA(cudaStreamSynchronize(g.stream));
  const int what = add ? 1 : 2;
  bool replayed = false;
  if (add && g.h_ctl[C_ERR] == RG_ENOSPACE && g.h_ctl[C_AUX] == 1) {
    // growth ran out of pool: compact, then replay from the growth step
    const uint64_t nops = directed ? n : 2 * n;
    rc = storage_recover(g);
    if (!rc) rc = storage_replay(g, n, nops, directed, true);
    if (!rc) rc = dispatch(g, A, what, n, directed, true, 0);
    if (!rc && old_num) rc = storage_copy_old(g, n);
    if (!rc) rc = sync_ctl(g);
    if (rc) return rc;
    replayed = true;
  }
  if ((rc = storage_error(g))) return rc;
  if (!replayed && g.h_ctl[C_LEFT] && (rc = finish_left<A, W>(g, g.h_ctl[C_LEFT]))) return rc;
  if ((rc = after_sync<A, W>(g, what))) return rc;
  if (old_num) std::memcpy(old_num, replayed ? (const void *)storage_old_host(g) : (const void *)(st + apply_old_off()),
                           n * 8);
  return RG_OK;
}

template <int A, bool W>
int apply_add_del_t(Graph &g, const rg_edge *adds, uint64_t n_add, const rg_edge *dels, uint64_t n_del,
                    int directed) {
  int rc = storage_reserve(g, 3 * SMALL_EDGES);
  if (rc) return rc;
  char *st = reinterpret_cast<char *>(g.stage_host);
  ApplyHdr *h1 = reinterpret_cast<ApplyHdr *>(st), *h2 = reinterpret_cast<ApplyHdr *>(st + APPLY_HDR2);
  std::memcpy(st + APPLY_DATA_OFF, adds, n_add * sizeof(rg_edge));
  std::memcpy(st + APPLY_DATA_OFF + apply_data2_off(), dels, n_del * sizeof(rg_edge));
  *h1 = ApplyHdr{n_add, 0, 0, 0, 0};
  *h2 = ApplyHdr{n_del, 0, 0, 0, apply_data2_off()};
  g.adj_version++;
  if ((rc = guard_counters(g))) return rc;
  if (++g.inv_epoch >= 0x7FFFFFFFu) {
    RG_CUDA(cudaMemsetAsync(g.d.inv, 0, (size_t)g.V * 4, g.stream));
    RG_CUDA(cudaMemsetAsync(g.d.chk, 0, (size_t)g.V * 4, g.stream));
    g.inv_epoch = 1;
  }
  h2->inv_tag = 2ull * g.inv_epoch;
  reset_stats(g);
  count_launch(g);
  if (n_add <= g.inline_max && n_del <= g.inline_max) {
    // both batches in the parameters; the staging buffer keeps them too for
    // the graphs that run when the insert batch leaves work
    const InlineBatch ib1 = inline_batch(adds, n_add, false, false, 0);
    const InlineBatch ib2 = inline_batch(dels, n_del, false, false, h2->inv_tag);
    if ((rc = launch_mixed_inline<A, W>(g, ib1, ib2, directed))) return rc;
  } else {
    cudaGraphExec_t exec;
    if ((rc = mixed_exec<A, W>(g, directed, &exec))) return rc;
    RG_CUDA(cudaGraphLaunch(exec, g.stream));
  }
  RG_CUDA(cudaStreamSynchronize(g.stream));
  if (g.h_ctl[C_ERR] == RG_ENOSPACE && g.h_ctl[C_AUX] == 1) {
    // the insert phase ran out of pool during growth (the delete phase did not
    // run): compact, replay the inserts, then apply the deletes on their own
    const uint64_t nops = directed ? n_add : 2 * n_add;
    rc = storage_recover(g);
    if (!rc) rc = storage_replay(g, n_add, nops, directed, true);
    if (!rc) rc = dispatch(g, A, 1, n_add, directed, true, 0);
    if (!rc) rc = sync_ctl(g);
    if (!rc) rc = storage_error(g);
    if (!rc) rc = after_sync<A, W>(g, 1);
    if (rc) return rc;
    return n_del ? apply_small_t<A, W>(g, dels, nullptr, n_del, directed, false, nullptr) : RG_OK;
  }
  if ((rc = storage_error(g))) return rc;
  unsigned long long left = g.h_ctl[C_LEFT];
  if (left == 1) {
    // the insert batch's level loop, then the delete batch in its own kernel
    cudaGraphExec_t re;
    if ((rc = rest_exec<A, W>(g, directed, &re))) return rc;
    count_launch(g);
    RG_CUDA(cudaGraphLaunch(re, g.stream));
    RG_CUDA(cudaStreamSynchronize(g.stream));
    if ((rc = storage_error(g))) return rc;
    left = g.h_ctl[C_LEFT];
  }
  if (left == 2 && (rc = finish_left<A, W>(g, 2))) return rc;
  return after_sync<A, W>(g, 2);
}

int apply_add_del_small(Graph &g, const rg_edge *adds, uint64_t n_add, const rg_edge *dels, uint64_t n_del,
                        int directed) {
  const bool W = g.weighted != 0;
  switch (g.algo) {
    case RG_BFS: return W ? apply_add_del_t<RG_BFS, true>(g, adds, n_add, dels, n_del, directed)
                          : apply_add_del_t<RG_BFS, false>(g, adds, n_add, dels, n_del, directed);
    case RG_SSSP: return W ? apply_add_del_t<RG_SSSP, true>(g, adds, n_add, dels, n_del, directed)
                           : apply_add_del_t<RG_SSSP, false>(g, adds, n_add, dels, n_del, directed);
    case RG_SSWP: return W ? apply_add_del_t<RG_SSWP, true>(g, adds, n_add, dels, n_del, directed)
                           : apply_add_del_t<RG_SSWP, false>(g, adds, n_add, dels, n_del, directed);
    case RG_WCC: return W ? apply_add_del_t<RG_WCC, true>(g, adds, n_add, dels, n_del, directed)
                          : apply_add_del_t<RG_WCC, false>(g, adds, n_add, dels, n_del, directed);
  }
  set_error("labels were not built (call rg_build_tree first)");
  return RG_ESTATE;
}

int apply_small(Graph &g, const rg_edge *edges, const uint64_t *pairs, uint64_t n, int directed, bool add,
                uint64_t *old_num) {
  const bool W = g.weighted != 0;
  switch (g.algo) {
    case RG_BFS: return W ? apply_small_t<RG_BFS, true>(g, edges, pairs, n, directed, add, old_num)
                          : apply_small_t<RG_BFS, false>(g, edges, pairs, n, directed, add, old_num);
    case RG_SSSP: return W ? apply_small_t<RG_SSSP, true>(g, edges, pairs, n, directed, add, old_num)
                           : apply_small_t<RG_SSSP, false>(g, edges, pairs, n, directed, add, old_num);
    case RG_SSWP: return W ? apply_small_t<RG_SSWP, true>(g, edges, pairs, n, directed, add, old_num)
                           : apply_small_t<RG_SSWP, false>(g, edges, pairs, n, directed, add, old_num);
    case RG_WCC: return W ? apply_small_t<RG_WCC, true>(g, edges, pairs, n, directed, add, old_num)
                          : apply_small_t<RG_WCC, false>(g, edges, pairs, n, directed, add, old_num);
  }
  set_error("labels were not built (call rg_build_tree first)");
  return RG_ESTATE;
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
