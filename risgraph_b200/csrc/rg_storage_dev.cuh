// Device side of the edge storage (the B200 form of IndexedEdgeStorage,
// core/storage.hpp:282-430, and Graph::add_edge / del_edge,
// core/graph.hpp:203-253), as per-item functions.  rg_storage.cu wraps each
// step in a grid-stride kernel for large batches; the fused small-batch apply
// kernel of rg_tree.cu runs the same steps inside one CTA.
#pragma once
#include <type_traits>

#include "rg_internal.cuh"

namespace rg {
namespace sdev {

// Op arrays (u32 each, ops_cap entries) of a staged batch.  O_MUL: multiplicity
// delta of the op (1; 2 for an undirected self-loop, whose two add_edge calls
// hit the same key; 0 = no-op).
enum OpArr { O_SRC = 0, O_DST, O_W, O_RID, O_OLD, O_MUL, O_SPARE, O_FLAG, O_NARR };

struct OpView {
  uint32_t *src, *dst, *w, *rid, *old, *mul, *spare, *flag;
};

inline OpView op_view(Graph &g) {
  OpView v;
  uint32_t **f = reinterpret_cast<uint32_t **>(&v);
  for (int i = 0; i < O_NARR; i++) f[i] = g.ops + (uint64_t)i * g.ops_cap;
  return v;
}

__device__ __forceinline__ uint64_t ht_hash(uint32_t s, uint32_t d, uint32_t w) {
  return splitmix64(((uint64_t)s << 32 | d) ^ splitmix64((uint64_t)w + 0x5851F42D4C957F2Dull));
}

__device__ __forceinline__ void set_err(unsigned long long *ctl, int code) {
  atomicCAS(&ctl[C_ERR], 0ull, (unsigned long long)code);
}

// Directed ops of edge i: one when directed; (s,d) and (d,s) when undirected
// (add_edge(e,false), core/graph.hpp:206-211).  An undirected self-loop is a
// single op of delta 2 on its one key, so concurrent duplicates still see a
// serial sequence of counts.
__device__ __forceinline__ void put_ops(OpView ops, uint64_t i, uint32_t s, uint32_t d, uint32_t w, int directed) {
  if (directed) {
    ops.src[i] = s; ops.dst[i] = d; ops.w[i] = w; ops.mul[i] = 1;
  } else {
    ops.src[2 * i] = s; ops.dst[2 * i] = d; ops.w[2 * i] = w; ops.mul[2 * i] = s == d ? 2 : 1;
    ops.src[2 * i + 1] = d; ops.dst[2 * i + 1] = s; ops.w[2 * i + 1] = w; ops.mul[2 * i + 1] = s == d ? 0 : 1;
  }
}

__device__ __forceinline__ void unpack_edge(const rg_edge *e, uint64_t i, int directed, int weighted, OpView ops) {
  uint32_t s = (uint32_t)e[i].src, d = (uint32_t)e[i].dst, w = weighted ? (uint32_t)e[i].data : 0u;
  put_ops(ops, i, s, d, w, directed);
}

// Reference file format pairs; weights are the pure function of the endpoints
// used by every implementation here (splitmix64(src<<32|dst) % 255 + 1).
__device__ __forceinline__ void unpack_pair(const uint64_t *p, uint64_t i, int directed, int weighted, OpView ops) {
  uint64_t s64 = p[2 * i], d64 = p[2 * i + 1];
  uint32_t s = (uint32_t)s64, d = (uint32_t)d64;
  uint32_t w = weighted ? (uint32_t)(splitmix64((s64 << 32) | d64) % 255 + 1) : 0u;
  put_ops(ops, i, s, d, w, directed);
}

// Find the record of op j's (s,d,w); create it (and reserve its slots at the
// end of the src / dst segments) when `create`.  Vertices whose segment just
// ran out of capacity go to the direction's grow list.  Lanes of a warp that
// reserve slots of the same vertex together take consecutive slots with one
// atomic (a hub is the source of many edges of one batch).
__device__ __forceinline__ void lookup_op(const DevGraph &g, OpView ops, uint64_t j, int create) {
  uint32_t s = ops.src[j], d = ops.dst[j], w = ops.w[j];
  if (ops.mul[j] == 0) { ops.rid[j] = UNSET; ops.flag[j] = 0; return; }
  ulonglong2 key = make_ulonglong2((uint64_t)s | ((uint64_t)d << 32), (uint64_t)w);
  uint64_t h = ht_hash(s, d, w) & g.ht_mask;
  uint32_t rid = UNSET, mine = UNSET;
  int created = 0;
  for (uint64_t probe = 0; probe <= g.ht_mask; probe++) {
    ulonglong2 e = __ldcg(&g.ht[h]);
    if ((uint32_t)e.x == NONE) {
      if (!create) break;
      if (mine == UNSET) {
        // (no fence before the claim below: a thread that finds this record
        // in the index only takes its id; the record's fields are read after
        // the kernel or CTA barrier that ends the lookup step).  The lanes
        // that claim together take their ids with one atomic.
        const unsigned m = __activemask();
        const int leader = __ffs(m) - 1, lane = threadIdx.x & 31;
        unsigned long long r = 0;
        if (lane == leader) r = atomicAdd(g.rec_top, (unsigned long long)__popc(m));
        r = __shfl_sync(m, r, leader) + __popc(m & ((1u << lane) - 1));
        if (r >= g.rec_cap) { set_err(g.ctl, RG_ENOSPACE); break; }
        mine = (uint32_t)r;
        g.rec_num[mine] = 0;
        g.rec_out[mine] = UNSET;
        g.rec_in[mine] = UNSET;
      }
      ulonglong2 want = make_ulonglong2(key.x, key.y | ((uint64_t)mine << 32));
      ulonglong2 old = cas128(&g.ht[h], make_ulonglong2(~0ull, ~0ull), want);
      if (old.x == ~0ull && old.y == ~0ull) { rid = mine; created = 1; break; }
      e = old;
    }
    // A 16-byte load racing with the claiming CAS may see the new (src,dst)
    // half with the old (all-ones) half; re-read atomically before deciding.
    if (e.x == key.x && (uint32_t)e.y != w) e = cas128(&g.ht[h], make_ulonglong2(~0ull, ~0ull), make_ulonglong2(~0ull, ~0ull));
    if (e.x == key.x && (uint32_t)e.y == w) { rid = (uint32_t)(e.y >> 32); break; }
    h = (h + 1) & g.ht_mask;
  }
  if (create && rid == UNSET && mine == UNSET) set_err(g.ctl, RG_ENOSPACE);
  ops.rid[j] = rid;
  ops.flag[j] = created;
  if (created) {
    // both directions' slots are reserved before either result is used, so
    // that the two atomics are in flight together
    const unsigned am = __activemask();
    const int lane = threadIdx.x & 31;
    const unsigned mo = __match_any_sync(am, s), mi = g.symmetric ? 0u : __match_any_sync(am, d);
    const int lo = __ffs(mo) - 1, li = __ffs(mi) - 1;
    uint32_t bo = 0, bi = 0;
    if (lane == lo) bo = atomicAdd(&g.out.len[s], (uint32_t)__popc(mo));
    if (!g.symmetric && lane == li) bi = atomicAdd(&g.in.len[d], (uint32_t)__popc(mi));
    const uint32_t co = g.out.cap[s], ci = g.symmetric ? 0u : g.in.cap[d];
    const unsigned lt = (1u << lane) - 1;
    const uint32_t po = __shfl_sync(mo, bo, lo) + __popc(mo & lt);
    g.rec_out[rid] = po;
    if (po == co) {
      unsigned long long k = atomicAdd(&g.ctl[C_GROWN_OUT], 1ull);
      g.out.grow[k] = s;
    }
    if (!g.symmetric) {
      const uint32_t pi = __shfl_sync(mi, bi, li) + __popc(mi & lt);
      g.rec_in[rid] = pi;
      if (pi == ci) {
        unsigned long long k = atomicAdd(&g.ctl[C_GROWN_IN], 1ull);
        g.in.grow[k] = d;
      }
    }
  }
}

// Grow vertex v of a direction, cooperatively by the calling CTA: a new region
// from the pool bump pointer, then a copy of the existing slots.  Initial loads
// (cap 0) get exactly len + len/8 + 2; a full pool sets RG_ENOSPACE with
// C_AUX = 1 (the host compacts and replays).  All threads of the CTA call it.
struct GrowShared {
  uint64_t new_off;
  uint32_t copy, new_cap;
};

template <bool W>
__device__ __forceinline__ void grow_vertex(DevDir dir, unsigned long long *ctl, uint32_t v, GrowShared &sh) {
  using E = typename std::conditional<W, uint2, uint32_t>::type;
  E *pool = reinterpret_cast<E *>(dir.pool);
  if (threadIdx.x == 0) {
    uint32_t len = dir.len[v], cap = dir.cap[v];
    sh.new_cap = 0;
    if (len > cap) {  // (a retry after compaction skips vertices already grown)
      uint64_t want = cap ? (uint64_t)cap * 2 : (uint64_t)len + len / 8 + 2;
      while (want < len) want *= 2;
      if (want > 0xFFFFFFF0ull) want = 0xFFFFFFF0ull;
      unsigned long long off = atomicAdd(dir.pool_top, (unsigned long long)want);
      if (off + want > dir.pool_cap) {
        atomicCAS(&ctl[C_ERR], 0ull, (unsigned long long)RG_ENOSPACE);
        ctl[C_AUX] = 1;
      } else {
        sh.new_cap = (uint32_t)want;
        sh.new_off = off;
      }
    }
    sh.copy = len < cap ? len : cap;
  }
  __syncthreads();
  if (sh.new_cap) {
    uint64_t from = dir.off[v];
    uint32_t old_cap = dir.cap[v];
    for (uint32_t i = threadIdx.x; i < sh.copy; i += blockDim.x) {
      pool[sh.new_off + i] = pool[from + i];
      dir.owner[sh.new_off + i] = v;
    }
    for (uint32_t i = threadIdx.x; i < old_cap; i += blockDim.x) dir.owner[from + i] = NONE;
    __syncthreads();
    if (threadIdx.x == 0) {
      dir.off[v] = sh.new_off;
      dir.cap[v] = sh.new_cap;
    }
  }
  __syncthreads();
}

// The same growth done by one warp, so that the warps of one CTA grow
// different vertices at once (the grow list names each vertex once).  The
// claim (new region from the bump pointer), the copy and the publication of
// the new offset and capacity are separate steps, so that a long list can be
// copied by the whole CTA instead (grow_vertex_warp returns such a claim
// uncopied when `defer` is set).
struct GrowClaim {
  unsigned long long new_off, from;
  uint32_t new_cap, copy, old_cap, v;
};

// What vertex v's growth needs: *want slots (0 when v has room; a retry
// after compaction skips vertices already grown), and the claim without its
// new region.
__device__ __forceinline__ GrowClaim grow_want(DevDir dir, uint32_t v, unsigned long long *want) {
  GrowClaim cl = {0, 0, 0, 0, 0, v};
  const uint32_t len = dir.len[v], cap = dir.cap[v];
  *want = 0;
  if (len > cap) {
    uint64_t w = cap ? (uint64_t)cap * 2 : (uint64_t)len + len / 8 + 2;
    while (w < len) w *= 2;
    if (w > 0xFFFFFFF0ull) w = 0xFFFFFFF0ull;
    *want = w;
    cl.from = dir.off[v];
    cl.old_cap = cap;
  }
  cl.copy = len < cap ? len : cap;
  return cl;
}

__device__ __forceinline__ GrowClaim grow_claim_warp(DevDir dir, unsigned long long *ctl, uint32_t v, int lane) {
  GrowClaim cl = {0, 0, 0, 0, 0, v};
  if (lane == 0) {
    unsigned long long want;
    cl = grow_want(dir, v, &want);
    if (want) {
      unsigned long long off = atomicAdd(dir.pool_top, want);
      if (off + want > dir.pool_cap) {
        atomicCAS(&ctl[C_ERR], 0ull, (unsigned long long)RG_ENOSPACE);
        ctl[C_AUX] = 1;
      } else {
        cl.new_cap = (uint32_t)want;
        cl.new_off = off;
      }
    }
  }
  cl.new_cap = __shfl_sync(0xFFFFFFFFu, cl.new_cap, 0);
  cl.new_off = __shfl_sync(0xFFFFFFFFu, cl.new_off, 0);
  cl.from = __shfl_sync(0xFFFFFFFFu, cl.from, 0);
  cl.copy = __shfl_sync(0xFFFFFFFFu, cl.copy, 0);
  cl.old_cap = __shfl_sync(0xFFFFFFFFu, cl.old_cap, 0);
  return cl;
}

// Copies a claimed vertex's slots (thread t of n threads), four loads in
// flight per thread before their stores.
template <bool W>
__device__ __forceinline__ void grow_copy(DevDir dir, const GrowClaim &cl, uint32_t t, uint32_t n) {
  using E = typename std::conditional<W, uint2, uint32_t>::type;
  E *pool = reinterpret_cast<E *>(dir.pool);
  for (uint32_t b = 0; b < cl.copy; b += 4 * n) {
    E x[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint32_t i = b + k * n + t;
      if (i < cl.copy) x[k] = pool[cl.from + i];
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint32_t i = b + k * n + t;
      if (i < cl.copy) {
        pool[cl.new_off + i] = x[k];
        dir.owner[cl.new_off + i] = cl.v;
      }
    }
  }
  for (uint32_t i = t; i < cl.old_cap; i += n) dir.owner[cl.from + i] = NONE;
}

__device__ __forceinline__ void grow_publish(DevDir dir, const GrowClaim &cl) {
  dir.off[cl.v] = cl.new_off;
  dir.cap[cl.v] = cl.new_cap;
}

// Returns true when the claim was left uncopied for the caller (`defer` and a
// copy of more than GROW_WARP_MAX slots).
constexpr uint32_t GROW_WARP_MAX = 2048;

template <bool W>
__device__ __forceinline__ bool grow_vertex_warp(DevDir dir, unsigned long long *ctl, uint32_t v, int lane,
                                                 bool defer = false, GrowClaim *out = nullptr) {
  const GrowClaim cl = grow_claim_warp(dir, ctl, v, lane);
  if (!cl.new_cap) return false;
  if (defer && cl.copy > GROW_WARP_MAX) {
    *out = cl;
    return true;
  }
  grow_copy<W>(dir, cl, (uint32_t)lane, 32);
  __syncwarp();
  if (lane == 0) grow_publish(dir, cl);
  __syncwarp();
  return false;
}

// Store op j's new entries (created by lookup), still DEAD (multiplicity 0).
template <bool W>
__device__ __forceinline__ void write_new_op(const DevGraph &g, OpView ops, uint64_t j) {
  using E = typename std::conditional<W, uint2, uint32_t>::type;
  E *po = reinterpret_cast<E *>(g.out.pool);
  E *pi = reinterpret_cast<E *>(g.in.pool);
  if (!ops.flag[j]) return;
  uint32_t s = ops.src[j], d = ops.dst[j], w = ops.w[j], rid = ops.rid[j];
  uint32_t ps = g.rec_out[rid];
  if (ps < g.out.cap[s]) {
    if constexpr (W) po[g.out.off[s] + ps] = make_uint2(d | DEAD, w);
    else po[g.out.off[s] + ps] = d | DEAD;
    g.out.owner[g.out.off[s] + ps] = s;
  }
  if (!g.symmetric) {
    uint32_t pd = g.rec_in[rid];
    if (pd < g.in.cap[d]) {
      if constexpr (W) pi[g.in.off[d] + pd] = make_uint2(s | DEAD, w);
      else pi[g.in.off[d] + pd] = s | DEAD;
      g.in.owner[g.in.off[d] + pd] = d;
    }
  }
}

template <bool W>
__device__ __forceinline__ void set_alive(const DevDir &dir, uint32_t v, uint32_t pos, uint32_t nbr, bool alive) {
  using E = typename std::conditional<W, uint2, uint32_t>::type;
  E *pool = reinterpret_cast<E *>(dir.pool);
  if (pos >= dir.cap[v]) return;
  uint32_t x = alive ? nbr : (nbr | DEAD);
  if constexpr (W) reinterpret_cast<uint32_t *>(&pool[dir.off[v] + pos])[0] = x;
  else pool[dir.off[v] + pos] = x;
}

// Multiplicity update of op j (update_edge, core/storage.hpp:390-396); the
// 0->1 and 1->0 transitions flip the DEAD bit.  ops.old = count before.
template <bool W>
__device__ __forceinline__ void count_op(const DevGraph &g, OpView ops, uint64_t j, int add) {
  uint32_t rid = ops.rid[j];
  uint32_t s = ops.src[j], d = ops.dst[j];
  if (rid == UNSET) { ops.old[j] = 0; return; }
  const uint32_t mul = ops.mul[j];
  uint32_t old;
  if (add) {
    old = atomicAdd(&g.rec_num[rid], mul);
    atomicAdd(&g.out.deg[s], (unsigned long long)mul);
    if (!g.symmetric) atomicAdd(&g.in.deg[d], (unsigned long long)mul);
    if (old == 0) {
      set_alive<W>(g.out, s, g.rec_out[rid], d, true);
      if (!g.symmetric) set_alive<W>(g.in, d, g.rec_in[rid], s, true);
    }
  } else {
    // update_edge(-1): the count never goes below zero
    old = g.rec_num[rid];
    while (old > 0) {
      uint32_t nv = old >= mul ? old - mul : 0u;
      uint32_t seen = atomicCAS(&g.rec_num[rid], old, nv);
      if (seen == old) break;
      old = seen;
    }
    uint32_t dropped = old < mul ? old : mul;
    if (dropped) {
      atomicAdd(&g.out.deg[s], 0ull - dropped);
      if (!g.symmetric) atomicAdd(&g.in.deg[d], 0ull - dropped);
    }
    if (old != 0 && old <= mul) {
      set_alive<W>(g.out, s, g.rec_out[rid], d, false);
      if (!g.symmetric) set_alive<W>(g.in, d, g.rec_in[rid], s, false);
    }
  }
  ops.old[j] = old;
}

// Per-edge old multiplicity with add_edge/del_edge's undirected conventions
// (core/graph.hpp:206-211: second orientation's count, minus one for a
// self-loop on add; :232-237 for delete) and the tree-repair candidates:
// 0->1 adds (src/sssp_inc_batch.cpp:148) and 1->0 deletes (:166).
__device__ __forceinline__ void edge_old(OpView ops, uint64_t i, int directed, int add, int collect,
                                         uint64_t *old_out, uint32_t *cand, unsigned long long *ctl) {
  uint32_t o;
  if (directed) {
    o = ops.old[i];
  } else {
    const uint32_t s = ops.src[2 * i], d = ops.dst[2 * i];
    if (s == d) {
      // add returns old+1-1, delete the second call's old (max(old-1,0))
      uint32_t a = ops.old[2 * i];
      o = add ? a : (a ? a - 1 : 0);
    } else {
      // both orientations move together; the canonical (lower src) key gives a
      // serial count sequence even when (s,d) and (d,s) share a batch
      o = ops.old[2 * i + (s < d ? 0 : 1)];
    }
  }
  if (old_out) old_out[i] = o;
  if (collect && (add ? o == 0 : o == 1)) {
    unsigned long long k = atomicAdd(&ctl[C_CANDN], 1ull);
    cand[k] = (uint32_t)i;
  }
}

}  // namespace sdev
}  // namespace rg
