// Internal device layout and helpers of librisgraph_b200.
//
// HBM layout (per graph):
//   labels   ulonglong2 lab[V]        {value u64, parent u32 | parent_w u32 << 32}
//                                      parent == NONE (0xFFFFFFFF) means no parent.
//                                      Updated as one 16-byte record with a 128-bit CAS,
//                                      the role of the reference's 16-byte CAS / vertex lock
//                                      in update_label (core/graph.hpp:1765-1887).
//   adjacency, per direction (out; in unless symmetric):
//            u64 off[V], u32 len[V], u32 cap[V], u64 deg[V]
//            pool: weighted   uint2  {nbr | DEAD, w}
//                  unweighted uint32  nbr | DEAD
//            A vertex's edges are the contiguous slots [off, off+len) of the pool.
//            DEAD marks a multiplicity-0 entry, the reference's never-compacted num==0
//            tombstone (core/storage.hpp:391-396, skipped at core/graph.hpp:916).
//   edge index: open-addressing table of uint4 {src, dst, w, rec} keyed by (src,dst,w)
//            -> record rec: num (multiplicity), out slot, in slot.  One probe sequence
//            finds an edge whatever its vertex's degree (the reference scans lists below
//            512 entries and hashes above, core/storage.hpp:358-386).
//   frontier queues, dedup stamps, invalidation tags, small control block.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "risgraph_b200.h"

namespace rg {

constexpr uint32_t NONE = 0xFFFFFFFFu;
constexpr uint32_t DEAD = 0x80000000u;
constexpr uint32_t VID_MASK = 0x7FFFFFFFu;
constexpr uint32_t UNSET = 0xFFFFFFFFu;
constexpr uint64_t BFS_MAXL = 65536ull;        // src/bfs.cpp:66
constexpr uint64_t SSSP_MAXL = 134217728ull;   // src/sssp.cpp:66, src/sswp.cpp:66
constexpr unsigned FULL = 0xFFFFFFFFu;

// Control block counters (device, u64 each).
enum Ctl : int {
  C_QN0 = 0,       // frontier length, queue 0
  C_QN1 = 1,       // frontier length, queue 1
  C_HUBN = 2,      // hub chunk tasks this level
  C_RESULT = 3,    // successful label updates (active_result_func sum)
  C_CANDN = 4,     // candidate edges for tree repair
  C_TREEN = 5,     // invalidated (reset) vertices
  C_GROWN_OUT = 6, // vertices whose out segment must grow
  C_GROWN_IN = 7,
  C_ERR = 8,       // first error code raised on the device
  C_RECOMPUTE = 9, // parent-chain guard tripped (has_parents, core/graph.hpp:1900-1903)
  C_MODN = 10,     // modified list length
  C_CHECKSUM = 11,
  C_AUX = 12,
  C_EDGES = 13,    // edge slots scanned by push levels (work counter)
  // device-driven level loop (written by k_level_begin, read by level kernels)
  C_LEVEL = 16,    // levels run in the current loop
  C_STAMP = 17,    // frontier dedup stamp of the current level
  C_ACT = 18,      // activity id of the current dense push level
  C_MODE = 19,     // mode of the current level (LevelMode)
  C_DEPTH = 20,    // BFS depth of the current frontier (full builds)
  C_MODEPOCH = 21, // modified-list epoch (trace_modified graphs)
  C_KLAUNCH = 22,  // kernels run by the level-loop graph of the current call
  C_INVTAG = 23,   // invalidation tag of the current deletion repair (tag+1 = rescued)
  C_INVITER = 24,  // invalidation levels run by the current deletion repair
  C_ROOT = 25,     // root of the label set (init_label_func argument)
  C_HOSTCOND = 26, // a loop condition for the host, when profile mode steps a loop from the host
  C_HVR = 27,      // heavy vertices queued by the rescue pass of this invalidation level
  C_HVE = 28,      // ... by the expand pass
  C_HVP = 29,      // ... by the pull over the reset set
  C_OVER = 30,     // the fused apply's one-CTA deletion repair handed over to the grid-wide one
  C_LEFT = 31,     // what a fused kernel left to the host (1: insert batch's level loop [and the delete batch], 2: delete batch's repair)
  C_COUNT = 32
};

enum LevelMode : unsigned long long {
  M_EMPTY = 0,      // frontier empty: every level kernel returns at once
  M_SPARSE = 1,     // k_push + k_push_hub over the frontier list
  M_PULL = 2,       // k_pull_hubs + k_pull_sell over all in-edges
  M_DENSE_PUSH = 3, // k_push_dense over all out-slots of active vertices
  M_BOTTOM_UP = 4,  // k_bfs_bottom_up (full BFS builds)
  M_LBS = 5,        // edge-balanced push (degree scan + tile partition + k_push_lbs)
  M_TINY = 6,       // k_push_tiny: one CTA runs successive small levels
  M_CLUSTER = 7,    // k_push_cluster: one thread-block cluster runs successive mid-size levels
  M_COUNT = 8
};
constexpr int TRACE_CAP = 4096;

struct DevDir {
  uint64_t *off;
  uint32_t *len;
  uint32_t *cap;
  unsigned long long *deg;
  void *pool;
  uint64_t pool_cap;
  unsigned long long *pool_top;
  uint32_t *grow;   // vertices to grow
  uint32_t *owner;  // per pool slot: the vertex whose segment holds it (NONE if unused)
};

struct DevGraph {
  uint32_t V;
  int weighted, symmetric;
  DevDir out, in;
  ulonglong2 *ht;
  uint64_t ht_mask;
  uint32_t *rec_num, *rec_out, *rec_in;
  unsigned long long *rec_top;
  uint64_t rec_cap;
  ulonglong2 *lab;
  uint32_t *val32;   // 32-bit mirror of lab[].x for reads (equal at kernel boundaries)
  uint32_t *stamp;
  uint32_t *inv;
  uint32_t *chk;     // repair tag of the vertices whose parent chain was found clear in that repair
  uint32_t *heavy;   // 3 lists of heavy_cap vertices: rescue, expand, pull (deletion repair)
  uint64_t heavy_cap;
  uint32_t *modstamp;
  uint32_t *modq;
  unsigned long long *ctl;
  unsigned long long *trace;  // frontier size per level (TRACE_CAP entries)
  unsigned long long *ptrace; // fused-path phase stamps (RG_PHASE_SLOTS), or null when not traced
};

// ---- per-algorithm hooks (a8): update_func = better(combine(s,w), d);
//      equal_func = combine(s,w) == d; init_label_func = init/active. ----
template <int A>
struct Hook;
template <>
struct Hook<RG_BFS> {  // src/bfs.cpp:76-91
  static __host__ __device__ __forceinline__ uint64_t combine(uint64_t s, uint64_t) { return s + 1; }
  static __host__ __device__ __forceinline__ bool better(uint64_t a, uint64_t b) { return a < b; }
  static __host__ __device__ __forceinline__ uint64_t init(uint64_t v, uint64_t r) { return v == r ? 0 : BFS_MAXL; }
  static constexpr bool all_active = false;
};
template <>
struct Hook<RG_SSSP> {  // src/sssp.cpp:67-91
  static __host__ __device__ __forceinline__ uint64_t combine(uint64_t s, uint64_t w) { return s + w; }
  static __host__ __device__ __forceinline__ bool better(uint64_t a, uint64_t b) { return a < b; }
  static __host__ __device__ __forceinline__ uint64_t init(uint64_t v, uint64_t r) { return v == r ? 0 : SSSP_MAXL; }
  static constexpr bool all_active = false;
};
template <>
struct Hook<RG_SSWP> {  // src/sswp.cpp:76-91
  static __host__ __device__ __forceinline__ uint64_t combine(uint64_t s, uint64_t w) { return s < w ? s : w; }
  static __host__ __device__ __forceinline__ bool better(uint64_t a, uint64_t b) { return a > b; }
  static __host__ __device__ __forceinline__ uint64_t init(uint64_t v, uint64_t r) { return v == r ? SSSP_MAXL : 0; }
  static constexpr bool all_active = false;
};
template <>
struct Hook<RG_WCC> {  // src/wcc.cpp:62-86
  static __host__ __device__ __forceinline__ uint64_t combine(uint64_t s, uint64_t) { return s; }
  static __host__ __device__ __forceinline__ bool better(uint64_t a, uint64_t b) { return a < b; }
  static __host__ __device__ __forceinline__ uint64_t init(uint64_t v, uint64_t) { return v; }
  static constexpr bool all_active = true;
};

// Values of all four hook sets stay below 2^31 (BFS <= 65536, SSSP/SSWP <=
// 2^27, WCC < |V| < 2^31), so a 32-bit mirror holds them exactly.  After a
// successful CAS of the 16-byte record the mirror moves the same way with a
// fire-and-forget atomic; readers may see it lag within a kernel (a weaker
// value only costs a wasted CAS or a later relaxation), never run ahead.
template <int A>
__device__ __forceinline__ void mirror_improve(uint32_t *m, uint32_t v, uint64_t nv) {
  if constexpr (A == RG_SSWP) atomicMax(&m[v], (uint32_t)nv);
  else atomicMin(&m[v], (uint32_t)nv);
}
__device__ __forceinline__ uint64_t ld_v32(const uint32_t *m, uint32_t v) { return __ldcg(&m[v]); }

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t pack_parent(uint32_t p, uint32_t w) {
  return (uint64_t)p | ((uint64_t)w << 32);
}

// ---- memory access helpers ----
__device__ __forceinline__ ulonglong2 cas128(ulonglong2 *addr, ulonglong2 cmp, ulonglong2 val) {
  ulonglong2 old;
  asm volatile(
      "{\n\t.reg .b128 d, b, c;\n\t"
      "mov.b128 b, {%2, %3};\n\t"
      "mov.b128 c, {%4, %5};\n\t"
      "atom.relaxed.gpu.global.cas.b128 d, [%6], b, c;\n\t"
      "mov.b128 {%0, %1}, d;\n\t}"
      : "=l"(old.x), "=l"(old.y)
      : "l"(cmp.x), "l"(cmp.y), "l"(val.x), "l"(val.y), "l"(addr)
      : "memory");
  return old;
}

// Coherent (L2) 16-byte load: labels are written by other SMs inside a launch.
__device__ __forceinline__ ulonglong2 ld_lab(const ulonglong2 *p) { return __ldcg(p); }
__device__ __forceinline__ uint64_t ld_val(const ulonglong2 *p) {
  return __ldcg(reinterpret_cast<const unsigned long long *>(p));
}
__device__ __forceinline__ uint64_t ld_meta(const ulonglong2 *p) {
  return __ldcg(reinterpret_cast<const unsigned long long *>(p) + 1);
}
__device__ __forceinline__ uint32_t ld_u32(const uint32_t *p) { return __ldcg(p); }

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// The device clock in ns (%globaltimer), for the phase trace.
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Warp-aggregated append of `v` by every lane with pred set (all lanes of mask
// must call).  Returns nothing; writes q[base + rank].
__device__ __forceinline__ void warp_append(bool pred, uint32_t v, uint32_t *q, unsigned long long *cnt,
                                            unsigned mask) {
  unsigned b = __ballot_sync(mask, pred);
  if (!b) return;
  int leader = __ffs(b) - 1;
  unsigned long long base = 0;
  if (lane_id() == leader) base = atomicAdd(cnt, (unsigned long long)__popc(b));
  base = __shfl_sync(mask, base, leader);
  if (pred) q[base + __popc(b & ((1u << lane_id()) - 1))] = v;
}

// Header of a small update batch in the graph's mapped pinned staging buffer,
// read by the fused apply kernel.  A submission holds up to two headers (an
// insert batch at offset 0, a delete batch at APPLY_HDR2); the edges follow at
// APPLY_DATA_OFF + data_off (0, or apply_data2_off() for the delete batch of
// an insert+delete submission: fixed, so that the kernel reads the edges
// without waiting for the header), and the per-edge old counts of a single
// batch are written back at apply_old_off().
struct ApplyHdr {
  uint64_t n;         // edges in the batch
  uint64_t pairs;     // 1: reference-format (src,dst) pairs, 0: rg_edge records
  uint64_t inv_tag;   // invalidation tag of a deletion repair
  uint64_t want_old;  // 1: write the old counts back
  uint64_t data_off;  // offset of the batch's edges from APPLY_DATA_OFF
};
constexpr uint64_t APPLY_HDR2 = 64;
constexpr uint64_t APPLY_DATA_OFF = 128;
constexpr uint64_t SMALL_EDGES = 2048;  // largest batch of the fused single-CTA apply path
constexpr uint64_t INLINE_MAX_EDGES = 16;  // largest batch carried in the fused kernel's parameters
inline uint64_t apply_old_off() { return APPLY_DATA_OFF + 2 * SMALL_EDGES * sizeof(rg_edge); }
// the delete batch of an insert+delete submission starts here, from APPLY_DATA_OFF
inline uint64_t apply_data2_off() { return SMALL_EDGES * sizeof(rg_edge); }

// A node of the versioned label history (rg_history.cu).
struct HistNode {
  uint64_t begin;           // version the value holds from
  unsigned long long pre;   // older node of the same vertex, ~0 if none
  uint64_t value;
};

// A cached, instantiated level-loop graph.
struct LoopGraph {
  cudaGraphExec_t exec = nullptr;
  uint64_t key = 0;
  int launches = 0;
};

// ---- host-side graph object ----
struct Graph {
  DevGraph d{};
  uint64_t V = 0, hint = 0;
  int symmetric = 0, dual = 1, trace = 0, weighted = 0;
  int algo = -1;
  uint64_t root = 0;
  cudaStream_t stream = nullptr;
  int device = 0;
  int num_sms = 148;
  // frontier queues (V entries each)
  uint32_t *q[2] = {nullptr, nullptr};
  uint32_t *tree = nullptr;   // invalidated set
  uint64_t *hubq = nullptr;   // hub chunk tasks (vertex | chunk << 32)
  uint64_t hubq_cap = 0;
  // staging for update batches
  void *stage_dev = nullptr;
  size_t stage_dev_bytes = 0;
  void *stage_host = nullptr;  // pinned, mapped
  void *stage_host_dev = nullptr;  // device view of stage_host
  size_t stage_host_bytes = 0;
  uint32_t *ops = nullptr;     // s,d,w,rid,old... per directed op (SoA inside)
  uint64_t ops_cap = 0;
  unsigned long long *h_ctl = nullptr;      // pinned, mapped mirror of ctl
  unsigned long long *h_ctl_dev = nullptr;  // its device view (the fused kernels write it)
  uint32_t stamp_epoch = 0;
  uint32_t inv_epoch = 0;
  uint32_t mod_epoch = 1;
  uint64_t *scratch64 = nullptr;  // V+1 u64 (unpack labels, frontier degrees, compaction)
  uint64_t *lb_P = nullptr;       // V+1 u64 frontier degree prefix
  uint32_t *lb_tile = nullptr;    // tile partition of the edge range
  uint64_t *lb_sums = nullptr;    // per-block sums of the device-side frontier scan
  uint32_t *act = nullptr;        // V: level id of the dense level a vertex is active in
  uint32_t act_epoch = 0;
  // sliced-ELL copy of the in-edges for dense pull levels, valid while adj_version == pull_version
  void *sell_ent = nullptr;       // entries, slice-major, column-major inside a slice
  uint64_t sell_cap = 0;          // entries allocated
  uint64_t *sell_off = nullptr;   // slice offsets (entries), slices + 1
  uint64_t sell_off_cap = 0;
  uint32_t *sell_row = nullptr;   // row ids by length, descending: vertex id, or |V| + hub piece index
  uint64_t sell_row_cap = 0;
  uint32_t *sell_hub = nullptr;   // hub vertices (in-list longer than a row)
  uint64_t sell_hub_cap = 0;
  uint64_t *sell_hub_off = nullptr;  // first piece of each hub (prefix of piece counts)
  uint32_t *sell_piece = nullptr;  // pieces: vertex[P+1], start[P+1], length[P+1]
  uint64_t sell_piece_cap = 0;
  ulonglong2 *sell_piece_best = nullptr;  // best {value, parent | w << 32} of each piece in a pull level
  uint64_t sell_best_cap = 0;
  unsigned long long *sell_cnt = nullptr;
  uint64_t sell_hubs = 0, sell_rows = 0, sell_slices = 0, sell_epoch = 0;
  uint64_t sell_cls[3] = {0, 0, 0};  // first slice of width <= 8, 4, 2
  uint64_t sell_split = 0;           // first slice of the second launch of a pull level
  std::vector<uint64_t> sell_off_host;  // host copy of sell_off (launch bounds of grouped pull levels)
  uint64_t pull_groups = 2;          // launches of a split pull level (RG_OPT_PULL_GROUPS)
  uint64_t pull_div = 64;
  int pull_split = 2;  // two-launch pull levels: 1 always, 0 never, 2 SSSP and WCC
  // versioned label history (off until rg_history_enable)
  HistNode *hist_nodes = nullptr;
  unsigned long long *hist_head = nullptr, *hist_ctl = nullptr;  // ctl: pool top, error
  uint64_t hist_cap = 0, hist_used = 0;
  uint64_t tiny_edges = 32768;  // frontiers with at most this many out-slots run in k_push_tiny (0: off)
  uint64_t adj_version = 1, pull_version = 0;
  int dense_pull = 2;  // dense build levels: 1 = pull over in-edges, 0 = edge-centric push, 2 = pull for WCC only
  uint64_t dense_div = 20, lbs_min = 2048, recompute_min = 2000000;
  uint64_t max_levels = 0;  // bound on the levels of one tree call (0: 4 |V| + 1024)
  // largest batch of the fused single-CTA apply path (<= SMALL_EDGES); measured on RMAT-24
  // SSSP, larger batches run faster on the grid-wide kernels
  uint64_t fused_max = 2048;
  int phase_trace = 0;            // RG_OPT_PHASE_TRACE
  uint64_t inline_max = 16;       // RG_OPT_INLINE_MAX: largest fused batch passed in the launch parameters
  uint64_t cluster_edges = 65536;  // RG_OPT_CLUSTER_EDGES: out-slot limit of a cluster level (0: off)
  int cl_ctas = 0;                  // CTAs of the cluster kernel (16 where the GPU schedules it, else 8)
  unsigned long long *ptrace_buf = nullptr;  // its device buffer (allocated with the labels)
  int bfs_bottom_up = 1;
  uint64_t bu_div = 64;  // measured on RMAT-22: the second BFS level (2% of |V|, most edges) already pays
  // device-driven level loops: [algo][weighted][build variant]; deletion repair: [algo][weighted]
  LoopGraph loops[16];
  LoopGraph dels[16];
  LoopGraph rests[16];  // after an insert+delete kernel left the insert batch's loop: loop -> delete batch
  // fused small-batch apply graphs: [algo][weighted][add][directed]; insert+delete pairs: [algo][weighted][directed]
  LoopGraph applies[32];
  LoopGraph mixes[16];
  cudaStream_t cap_stream = nullptr;
  uint64_t layout_version = 1;  // bumped when pool buffers move (compaction)
  void *cub_tmp = nullptr;
  size_t cub_tmp_bytes = 0;
  // stats of the last tree call
  uint64_t st_levels = 0, st_invalidated = 0, st_recomputes = 0;
  std::vector<uint64_t> st_frontier;  // frontier size entering each push level
  std::vector<double> st_level_ms;    // device time of each push level (profiling on)
  uint64_t bytes = 0;
  std::string err;
  cudaStream_t own_stream = nullptr;
  // kernel accounting
  uint64_t launches = 0;
  int profiling = 0;
  cudaEvent_t pev[2] = {nullptr, nullptr};
  uint64_t prof_launches = 0;
  double prof_ms = 0.0;
  // weights above W_RAW_MAX travel as 32-bit codes (see weight_code): code -> weight
  std::mutex wmu;
  std::unordered_map<uint64_t, uint32_t> wcode;
  std::vector<uint64_t> wfull;
};

// Edge weights on the device are 32-bit.  A weight above W_RAW_MAX = 2^27 (the
// SSSP/SSWP sentinel MAXL, src/sssp.cpp:66) can never lower an SSSP value
// (s + w >= 2^27 >= d for every label d) and never limits an SSWP value
// (min(s, w) = s, since s <= 2^27), so its exact size only matters to read it
// back: such weights are exchanged on the host for distinct codes in
// (2^27, 2^31), every comparison the hooks make gives the same answer, equal
// weights stay one edge and different ones stay different edges, and
// rg_get_labels turns a parent's code back into its full weight.  Weights at or
// above W_LIMIT = 2^64 - 2^27 are refused: there the reference's u64 sum s + w
// wraps around (a negative weight).
constexpr uint64_t W_RAW_MAX = 1ull << 27;
constexpr uint64_t W_CODE_BASE = W_RAW_MAX + 1, W_CODE_END = 1ull << 31;
constexpr uint64_t W_LIMIT = 0ull - (1ull << 27);

// Kernel launch bookkeeping (every launch site calls count_launch).
inline void count_launch(Graph &g, int n = 1) { g.launches += (uint64_t)n; }

// Error plumbing (thread-local last error message).
void set_error(const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
#define RG_CUDA(call)                                  \
  do {                                                 \
    cudaError_t _e = (call);                           \
    if (_e != cudaSuccess) return rg::cuda_fail(_e, #call); \
  } while (0)

// ---- storage (rg_storage.cu) ----
int storage_alloc(Graph &g);
void storage_free(Graph &g);
// Stage n edges (rg_edge or reference pairs) into the device op arrays as
// directed ops (2 per edge when undirected).  Returns number of ops.
int stage_edges(Graph &g, const rg_edge *edges, const uint64_t *pairs, uint64_t n, int directed, uint64_t *nops);
// One staged batch: storage_enqueue launches the multiplicity update (and, when
// collect, the tree-repair candidate list) without waiting; after sync_ctl,
// storage_error reports a device error.  A pool exhausted by growth is
// recovered by storage_recover + storage_replay.  storage_copy_old enqueues
// the per-edge old counts into pinned memory, read with storage_old_host
// after the sync.
int storage_enqueue(Graph &g, bool add, uint64_t n_edges, uint64_t nops, int directed, bool collect);
int storage_replay(Graph &g, uint64_t n_edges, uint64_t nops, int directed, bool collect);
int storage_recover(Graph &g);
int storage_copy_old(Graph &g, uint64_t n_edges);
const uint64_t *storage_old_host(Graph &g);
int storage_error(Graph &g);
int sync_ctl(Graph &g);
// Size the staging and op buffers for batches of up to n_edges edges now, so
// that later batches of that size allocate nothing.
int storage_reserve(Graph &g, uint64_t n_edges);
int storage_num(Graph &g, uint64_t nops, uint64_t *num);
// op array accessors (device pointers)
uint32_t *op_src(Graph &g);
uint32_t *op_dst(Graph &g);
uint32_t *op_w(Graph &g);
uint32_t *op_cand(Graph &g);   // candidate edge indices after storage_add/del(collect)

// ---- trees (rg_tree.cu) ----
int tree_build(Graph &g, int algo, uint64_t root, uint64_t *total);
// Repair for candidate edges: edges [0,n) given as staged ops (cands == nullptr:
// all staged edges are candidates; else indices in op_cand with count in ctl).
int tree_add(Graph &g, uint64_t n_edges, int directed, bool from_cands, uint64_t *total);
int tree_del(Graph &g, uint64_t n_edges, int directed, bool from_cands, uint64_t *total);
// Split form used to fuse storage and repair into one submission:
// tree_enqueue (what: 1 add, 2 del) launches without waiting; after the caller
// has synchronised and read the control block, tree_after_sync finishes it.
int tree_enqueue(Graph &g, int what, uint64_t n_edges, int directed, bool from_cands);
int tree_after_sync(Graph &g, int what, uint64_t *total);
int tree_classify(Graph &g, uint64_t n_edges, int directed, const uint8_t *is_del_dev, uint8_t *unsafe_dev);
int tree_labels(Graph &g, uint64_t *val, uint64_t *par, uint64_t *pw);
int tree_checksum(Graph &g, uint64_t *sum);
int tree_alloc(Graph &g);
// Fused small-batch apply (n <= SMALL_EDGES): storage update, candidate
// selection and seeding in one single-CTA kernel, the repair loops behind a
// conditional node, one graph launch and one synchronisation in all.
int apply_small(Graph &g, const rg_edge *edges, const uint64_t *pairs, uint64_t n, int directed, bool add,
                uint64_t *old_num);
// Versioned label history (rg_history.cu).
int history_enable(Graph &g, uint64_t capacity);
int history_record(Graph &g, uint64_t version, int all);
int history_get(Graph &g, const uint64_t *vids, uint64_t n, uint64_t version, uint64_t *values, uint8_t *found);
int history_gc(Graph &g, uint64_t version);
void history_free(Graph &g);
// An insert batch and a delete batch (each <= SMALL_EDGES) in one graph launch:
// the two fused applies back to back, the delete one skipped if the insert
// one stopped on a storage error.
int apply_add_del_small(Graph &g, const rg_edge *adds, uint64_t n_add, const rg_edge *dels, uint64_t n_del,
                        int directed);

}  // namespace rg

// The opaque handle of the C ABI.
struct rg_graph {
  rg::Graph g;
};
