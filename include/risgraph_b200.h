/* risgraph_b200: B200-native (sm_100a) incremental dependency-tree maintenance
 * for BFS / SSSP / SSWP / WCC under edge insertions and deletions.
 *
 * Drop-in C ABI for the hot path of the reference's header-only
 * template<EdgeData> class Graph (core/graph.hpp:41-1908).  The reference takes
 * its per-algorithm semantics as lambda template parameters; a C ABI cannot, so
 * an algorithm enum selects the four hook sets the reference's drivers define
 * (src/bfs.cpp:76-91, src/sssp.cpp:67-91, src/sswp.cpp:76-91, src/wcc.cpp:62-86).
 * The adjacency and the label array live in device memory (HBM); the host
 * mirror is filled on rg_get_labels.  Plain pointers and sizes only; no
 * exceptions cross the ABI: every call returns an rg_status.
 *
 * Threading: one CUDA stream per graph; calls on one graph are serialised by
 * the caller (the reference's build_tree / update_tree_* are single-caller,
 * core/graph.hpp:1728).  Distinct graphs may be used from distinct threads.
 * Every call returns after its device work has completed.
 *
 * Limits of the device layout: vertices < 2^31 (the reference stores 48-bit
 * ids, core/type.hpp:23); edge weights are uint64 as in the reference
 * (core/type.hpp:25) below 2^64 - 2^27, where the reference's u64 sum
 * value + weight would wrap around; edge multiplicities are 32-bit (the
 * reference's are 16-bit, core/type.hpp:24).  Weights above 2^27 (the
 * SSSP/SSWP sentinel) are kept on the device as 32-bit codes, which every
 * hook compares exactly as the full weight, and read back in full.
 * Out-of-range input returns an error, never a fault. */
#ifndef RISGRAPH_B200_H
#define RISGRAPH_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference throws std::runtime_error("VertexId error.")
 * for ids >= |V| (core/graph.hpp:205,231); here that is RG_EINVAL_VID. */
typedef enum {
  RG_OK = 0,
  RG_EINVAL = 1,        /* bad argument (null graph, bad algorithm, size) */
  RG_EINVAL_VID = 2,    /* vertex id >= |V| */
  RG_EINVAL_WEIGHT = 3, /* weight >= 2^64 - 2^27 on a weighted graph */
  RG_ENOMEM_HBM = 4,    /* device allocation failed / HBM budget exceeded */
  RG_ENOSPACE = 5,      /* edge pool or edge index full */
  RG_ETIMEOUT = 6,      /* a bounded device wait gave up */
  RG_ECUDA = 7,         /* CUDA runtime error (message in rg_last_error) */
  RG_ESTATE = 8         /* call not valid in the graph's current state */
} rg_status;

/* Algorithms: the a8 hook sets of the reference drivers. */
typedef enum { RG_BFS = 0, RG_SSSP = 1, RG_SSWP = 2, RG_WCC = 3 } rg_algo;

/* Edge<EdgeData> (core/type.hpp:57-81): src, dst, data (weight; ignored on
 * unweighted graphs). 24 bytes, host byte order. */
typedef struct {
  uint64_t src, dst, data;
} rg_edge;

typedef struct rg_graph rg_graph;

/* Graph(vertices, hint_edges, symmetric, dual, trace_modified)
 * (core/graph.hpp:61-100), plus `weighted` (Graph<uint64_t> vs Graph<void>).
 * hint_edges sizes the device edge pool and index (0 = 16 * vertices, the
 * reference's default at :64). */
int rg_create(uint64_t vertices, uint64_t hint_edges, int symmetric, int dual, int trace_modified,
              int weighted, rg_graph **out);
int rg_destroy(rg_graph *g);

/* Graph::add_edge / del_edge for n edges (core/graph.hpp:203-253), applied as
 * one batch.  old_num[i] (nullable) receives the multiplicity before edge i,
 * with the reference's undirected conventions (:206-211, :232-237). */
int rg_add_edges(rg_graph *g, const rg_edge *edges, uint64_t n, int directed, uint64_t *old_num);
int rg_del_edges(rg_graph *g, const rg_edge *edges, uint64_t n, int directed, uint64_t *old_num);

/* The same for edges given in the reference's binary file format
 * (mmap_binary, core/io.hpp:26-36): n (src,dst) uint64 pairs.  Weights are
 * splitmix64(src<<32|dst) % 255 + 1 on weighted graphs (rg_gen_weight). */
int rg_add_pairs(rg_graph *g, const uint64_t *pairs, uint64_t n, int directed, uint64_t *old_num);
int rg_del_pairs(rg_graph *g, const uint64_t *pairs, uint64_t n, int directed, uint64_t *old_num);

/* Graph::get_edge_num (core/graph.hpp:198-201) for n edges. */
int rg_get_edge_num(rg_graph *g, const rg_edge *edges, uint64_t n, uint64_t *num);

/* get_outgoing_degree / get_incoming_degree (core/graph.hpp:165-174) for all
 * vertices: sum of multiplicities (IndexedEdgeStorage::get_degree,
 * core/storage.hpp:329).  Either pointer may be NULL. */
int rg_get_degrees(rg_graph *g, uint64_t *out_degree, uint64_t *in_degree);

/* Graph::build_tree (core/graph.hpp:873-985) with the hooks of `algo` rooted
 * at `root` (ignored for WCC).  Sets the graph's label algorithm and root for
 * the update calls below.  total (nullable) = number of label updates. */
int rg_build_tree(rg_graph *g, int algo, uint64_t root, uint64_t *total);

/* Graph::update_tree_add for one edge (n == 1, core/graph.hpp:1124-1160) or a
 * batch (core/graph.hpp:1162-1218).  The edges are already in the adjacency. */
int rg_update_tree_add(rg_graph *g, int algo, const rg_edge *edges, uint64_t n, int directed, uint64_t *total);

/* Graph::update_tree_del for one edge (core/graph.hpp:1622-1656) or a batch
 * (core/graph.hpp:1658-1718).  The edges are already removed. */
int rg_update_tree_del(rg_graph *g, int algo, const rg_edge *edges, uint64_t n, int directed, uint64_t *total);

/* need_update_tree_add (core/graph.hpp:987-1000) and need_update_tree_del
 * (core/graph.hpp:1220-1233) for n edges: unsafe[i] = 1 when edge i needs a
 * tree repair.  is_del (nullable = all adds) selects the hook per edge. */
int rg_classify(rg_graph *g, int algo, const rg_edge *edges, const uint8_t *is_del, uint64_t n, int directed,
                uint8_t *unsafe);

/* The batch driver step of src/sssp_inc_batch.cpp:141-157 (resp. :159-175)
 * fused on the device: add (resp. delete) the n edges, then repair the tree for
 * exactly those whose multiplicity went 0->1 (resp. 1->0).  No host decision
 * in between.  old_num as for rg_add_edges. */
int rg_apply_add(rg_graph *g, int algo, const rg_edge *edges, uint64_t n, int directed, uint64_t *old_num);
int rg_apply_del(rg_graph *g, int algo, const rg_edge *edges, uint64_t n, int directed, uint64_t *old_num);

/* One step of src/sssp_inc_batch.cpp:141-175: rg_apply_add of `adds`, then
 * rg_apply_del of `dels`, as one device submission with one synchronisation
 * when both batches hold at most RG_OPT_FUSED_MAX edges (default 2048; two
 * submissions otherwise). */
int rg_apply_add_del(rg_graph *g, int algo, const rg_edge *adds, uint64_t n_add, const rg_edge *dels, uint64_t n_del,
                     int directed);

/* rg_apply_add / rg_apply_del over reference-format pairs (see rg_add_pairs). */
int rg_apply_add_pairs(rg_graph *g, int algo, const uint64_t *pairs, uint64_t n, int directed, uint64_t *old_num);
int rg_apply_del_pairs(rg_graph *g, int algo, const uint64_t *pairs, uint64_t n, int directed, uint64_t *old_num);

/* Labels (VertexTree, core/graph.hpp:54-59): value, parent vertex (== |V| for
 * none, as empty_parent at :90) and parent edge weight.  Any pointer may be NULL. */
int rg_get_labels(rg_graph *g, uint64_t *value, uint64_t *parent, uint64_t *parent_w);

/* Vertices whose label changed since rg_clear_modified (trace_modified graphs;
 * get_modified / clear_modified, core/graph.hpp:117-130).  Writes up to cap ids. */
int rg_get_modified(rg_graph *g, uint64_t *vids, uint64_t cap, uint64_t *n);
int rg_clear_modified(rg_graph *g);

/* Versioned label history: the device form of MVVec (core/mvvec.hpp:23-162),
 * which the _inc_rt drivers fill after every update with the value of each
 * modified vertex at the update's version (src/sssp_inc_rt.cpp:338-343).
 * Needs a trace_modified graph.  rg_history_enable reserves capacity_nodes
 * history nodes (24 bytes each).  rg_history_record stores, at `version`, the
 * current value of every vertex modified since the last rg_clear_modified (all
 * vertices when all_vertices, e.g. version 0 right after rg_build_tree), then
 * clears the modified list; as MVVec::set, a vertex gets a new node only when
 * its value changed, and a repeated version overwrites.  RG_ENOSPACE when the
 * pool is full (nodes that fit are kept).  rg_history_get returns each vertex's
 * value as of `version` (MVVec::get: the newest node at or before it); found[i]
 * = 0 when the vertex has no node that old.  rg_history_gc(version) drops the
 * nodes no reader at or after `version` can see (MVVec::gc) and packs the pool. */
int rg_history_enable(rg_graph *g, uint64_t capacity_nodes);
int rg_history_record(rg_graph *g, uint64_t version, int all_vertices);
int rg_history_get(rg_graph *g, const uint64_t *vids, uint64_t n, uint64_t version, uint64_t *values,
                   uint8_t *found);
int rg_history_gc(rg_graph *g, uint64_t version);
int rg_history_nodes(rg_graph *g, uint64_t *used, uint64_t *capacity);

/* Checksum of the value array on the device (same definition as
 * rg_gen_value_checksum), so per-step checks need no label copy. */
int rg_value_checksum(rg_graph *g, uint64_t *checksum);

/* Counters of the last tree call: levels run, vertices invalidated by deletion
 * repair, full recomputes.  Any pointer may be NULL. */
int rg_last_stats(rg_graph *g, uint64_t *levels, uint64_t *invalidated, uint64_t *recomputes);

/* Run this graph's device work on a caller-provided cudaStream_t (NULL:
 * back to the graph's own stream), e.g. to time it with events on that stream
 * or to order it after the caller's copies.  rg_get_stream returns the stream
 * in use.  No reference counterpart: the reference runs on host threads. */
int rg_set_stream(rg_graph *g, void *cuda_stream);
int rg_get_stream(rg_graph *g, void **cuda_stream);

/* Kernel accounting.  rg_launch_count: kernels this graph has launched since
 * creation.  rg_profile(g, 1) brackets every level-relaxation launch (the
 * push kernels) with CUDA events on the launching stream; rg_profile_read
 * returns their number and summed device time in milliseconds since the last
 * read.  No reference counterpart (the reference prints phase wall times). */
int rg_launch_count(rg_graph *g, uint64_t *launches);
int rg_profile(rg_graph *g, int enable);
int rg_profile_read(rg_graph *g, uint64_t *launches, double *ms);

/* Frontier size entering each push level of the last tree call (up to cap
 * entries), the number of levels, and the edge slots those levels scanned.
 * The reference prints the same per-level counts through
 * continue_reduce_print_func (src/sssp.cpp:71-75). */
int rg_level_trace(rg_graph *g, uint64_t *sizes, uint64_t cap, uint64_t *levels, uint64_t *edges_scanned);
/* Device time (ms, CUDA events) of each push level of the last tree call,
 * recorded only while rg_profile is on. */
int rg_level_times(rg_graph *g, double *ms, uint64_t cap, uint64_t *levels);
/* Device-clock start (ns, %globaltimer) of each level of the last tree call,
 * stamped on the device by the level loop itself, so it covers graph-launched
 * calls too; entry `levels` is the end of the last level.  Writes
 * min(cap, levels + 1) entries.  No counterpart in the reference (it times
 * whole calls with wall clocks, src/sssp.cpp:96-99). */
int rg_level_stamps(rg_graph *g, uint64_t *ns, uint64_t cap, uint64_t *levels);

/* Device-clock stamps (ns, %globaltimer) of the last fused submission while
 * RG_OPT_PHASE_TRACE is on: RG_PHASE_SLOTS words.  Batch b (0: the insert
 * batch or a single batch, 1: the delete batch of rg_apply_add_del) owns
 * words 16*b + RG_PH_*; word 16*b + 15 is 1 when that batch ran in the fused
 * kernel.  Words 32 + 2*b and 33 + 2*b: start of the kernel that ran batch b
 * and the end of its staging (header and edges across the bus).  The
 * reference has no counterpart (it times phases with wall clocks). */
#define RG_PHASE_SLOTS 64
enum {
  RG_PH_BEGIN = 0,      /* control block reset */
  RG_PH_UNPACK = 1,     /* edges unpacked into the op arrays */
  RG_PH_LOOKUP = 2,     /* edge index lookups / inserts */
  RG_PH_GROW = 3,       /* segment growth */
  RG_PH_WRITE = 4,      /* new slots written (insert batches) */
  RG_PH_COUNT = 5,      /* multiplicities updated */
  RG_PH_OLD = 6,        /* per-edge old counts and repair candidates */
  RG_PH_SEED = 7,       /* repair seeds */
  RG_PH_DELREPAIR = 8,  /* one-CTA deletion repair (delete batches) */
  RG_PH_END = 9         /* in-place push levels, end of the batch */
};
int rg_phase_trace(rg_graph *g, uint64_t *ns);

/* Strategy knobs of the level engine (the reference hard-codes its own:
 * push/pull switch at core/graph.hpp:334, vertex- vs edge-centric cost model
 * at :595-612, recompute threshold at :1252).  Values are per graph.
 *   RG_OPT_DENSE_PULL     build levels may pull over in-edges: 1 always, 0 never,
 *                         2 (default) for SSSP / SSWP / WCC (BFS goes bottom-up)
 *   RG_OPT_PULL_DIV       a build level pulls when frontier * div >= |V| (default 64)
 *   RG_OPT_TINY_EDGES     frontiers of at most 1024 vertices and this many out-slots
 *                         run level after level in one CTA (default 32768, max 2^20,
 *                         0 = off)
 *   RG_OPT_DENSE_DIV      a level is dense when frontier * div >= |V|
 *   RG_OPT_LBS_MIN        frontiers at least this large use the edge-balanced push
 *   RG_OPT_BFS_BOTTOM_UP  1: full BFS builds pull bottom-up on large levels
 *   RG_OPT_BFS_BU_DIV     a BFS build level goes bottom-up when frontier * div >= |V|
 *                         (default 64; Beamer's direction switch by frontier size)
 *   RG_OPT_RECOMPUTE_MIN  deletion repair falls back to a full build when the
 *                         invalidated set exceeds max(this, |V|/20)
 *   RG_OPT_PULL_SPLIT     pull levels run the longest in-lists in a first launch
 *                         so the rest read this level's hub values: 1 always,
 *                         0 never, 2 (default) for SSSP and WCC
 *   RG_OPT_MAX_LEVELS     bound on the relaxation levels of one tree call
 *                         (0, the default: 4 |V| + 1024).  A call that reaches
 *                         it stops with RG_ETIMEOUT and leaves the labels
 *                         partly updated; the graph stays usable and the next
 *                         rg_build_tree restores them.
 *   RG_OPT_PULL_GROUPS    launches of a split pull level (2..16, default 2): the
 *                         hub slices first, then the other rows, widest first, in
 *                         groups - 1 launches of about equal entries; each launch
 *                         reads the values the earlier ones set in this level.
 *   RG_OPT_FUSED_MAX      update batches of at most this many edges (0..2048,
 *                         default 2048) take the fused single-CTA path of
 *                         rg_apply_*: storage and small repairs in one
 *                         submission; larger batches run grid-wide kernels.
 *   RG_OPT_PHASE_TRACE    1: the fused path stamps the device clock at its
 *                         phase boundaries (rg_phase_trace); default 0.
 *   RG_OPT_INLINE_MAX     fused batches of at most this many edges (0..16,
 *                         default 16; 0: never) travel inside the kernel's
 *                         launch parameters instead of a staging buffer that
 *                         the kernel reads across the bus.
 *   RG_OPT_CLUSTER_EDGES  frontiers too large for one CTA but of at most 16 x
 *                         1024 vertices (8 x 1024 where the GPU schedules no
 *                         16-CTA cluster) and this many out-slots (default
 *                         65536, at most 2^20; 0: never) run their levels in
 *                         one thread-block cluster, one launch for successive
 *                         levels; a frontier that a tiny level could take goes
 *                         to the cluster when it has more than 4096 slots. */
typedef enum {
  RG_OPT_DENSE_PULL = 0,
  RG_OPT_DENSE_DIV = 1,
  RG_OPT_LBS_MIN = 2,
  RG_OPT_BFS_BOTTOM_UP = 3,
  RG_OPT_RECOMPUTE_MIN = 4,
  RG_OPT_BFS_BU_DIV = 5,
  RG_OPT_PULL_DIV = 6,
  RG_OPT_TINY_EDGES = 7,
  RG_OPT_PULL_SPLIT = 8,
  RG_OPT_MAX_LEVELS = 9,
  RG_OPT_PULL_GROUPS = 10,
  RG_OPT_FUSED_MAX = 11,
  RG_OPT_PHASE_TRACE = 12,
  RG_OPT_INLINE_MAX = 13,
  RG_OPT_CLUSTER_EDGES = 14
} rg_option;
int rg_set_option(rg_graph *g, int option, uint64_t value);
int rg_get_option(rg_graph *g, int option, uint64_t *value);

/* Autotuner of the options above for this graph and algorithm: coordinate
 * descent over candidate values of the pull / bottom-up divisor, the dense
 * divisor, the edge-balanced minimum and the small-frontier size, timing `reps`
 * full builds per trial (and, when n_sample > 0, insert + delete round trips
 * of the sample batch, which leave the graph unchanged, for the small-frontier
 * size).  The chosen values stay set on the graph.  Every trial must give the
 * same values (checked by checksum); the labels end as after rg_build_tree.
 * No reference counterpart: the reference's thresholds are constants. */
typedef struct {
  double build_ms_before, build_ms_after;  /* median build time */
  double apply_ms_before, apply_ms_after;  /* median sample round trip (0 without a sample) */
  uint64_t options[16];                    /* chosen values, indexed by rg_option */
  uint64_t trials;
} rg_tune_report;
int rg_autotune(rg_graph *g, int algo, uint64_t root, const rg_edge *sample, uint64_t n_sample, int directed,
                int reps, rg_tune_report *out);

/* Device bytes held by the graph. */
int rg_device_bytes(rg_graph *g, uint64_t *bytes);

/* Allocation-free build_tree for callers that may not allocate device memory
 * when they need a tree: a process whose device memory belongs to another
 * framework's pool and is fixed at start-up, or a latency-critical path where
 * cudaMalloc/cudaFree would synchronise the device.  No counterpart in the
 * reference (its build_tree, core/graph.hpp:873-985, works on the Graph's own
 * storage); this computes the same values with the same hooks.
 *
 * Input: a CSR graph in caller-owned DEVICE memory: row_offsets[vertices+1]
 * (uint64, non-decreasing, last <= edges), columns[edges] (uint32 < vertices),
 * weights[edges] (uint32; required for RG_SSSP and RG_SSWP, ignored for RG_BFS
 * and RG_WCC; NULL with SSSP/SSWP is RG_EINVAL).  Output: values[vertices]
 * and parents[vertices] (parent == vertices for none) in caller-owned device
 * memory; either may be NULL, not both.  Runs on cuda_stream (NULL = default)
 * and is synchronous: it reads a frontier count back to the host after every
 * level and returns when the tree is written, so it must not be called on a
 * stream that is being captured.  No cudaMalloc/cudaFree or allocating library
 * call: the working memory is one static device array of about 28 MB, held by
 * every GPU that loads the library's device code until exit, which bounds the
 * graph to RG_STATIC_MAX_VERTICES vertices (larger graphs: RG_EINVAL).  All
 * calls share that array: calls that overlap on the GPU race and give
 * undefined results.
 *
 * Set-up: CUDA loads a library's device code lazily by default
 * (CUDA_MODULE_LOADING=LAZY), so the 28 MB are only taken on a device when
 * this library's device code is first used there.  The first call on each
 * device (with that device current) looks the array's address up, which
 * loads the module.  A caller whose memory is later claimed by a pool fixed at
 * start-up should therefore make a set-up call at start-up, before the pool
 * reserves its memory: vertices == 0 with every pointer NULL only does this
 * per-device set-up and returns RG_OK (or run with CUDA_MODULE_LOADING=EAGER).
 * Malformed CSR input returns RG_EINVAL / RG_EINVAL_VID without touching
 * memory out of range. */
#define RG_STATIC_MAX_VERTICES (1u << 20)
int rg_build_tree_csr_static(int algo, uint64_t root, uint64_t vertices, uint64_t edges,
                             const uint64_t *row_offsets, const uint32_t *columns, const uint32_t *weights,
                             uint64_t *values, uint64_t *parents, void *cuda_stream);

/* ---- Served mode ----------------------------------------------------------
 * Stands in for the reference's latency-aware epoch loop of the _inc_rt
 * drivers (src/sssp_inc_rt.cpp:119-441): clients submit single edge updates;
 * the server batches, per graph instance, every update that arrived while the
 * previous batch was on the GPU (continuous batching), applies it as one
 * fused add batch + delete batch (safe updates cost only the multiplicity
 * update; unsafe ones share one repair), and completes all of them together.
 * Each instance has its own worker thread and CUDA stream, so instances of
 * different sizes overlap on the device.  Instances are admitted against an
 * HBM budget.  The epoch cap adapts so that one epoch stays within the target
 * latency (the reference adapts its unsafe-update threshold at :394-412).
 * With per_update = 1 every update is applied alone (one update per launch
 * sequence): the baseline the batched server is measured against. */
typedef struct rg_server rg_server;

typedef struct {
  uint32_t instance;  /* from rg_server_attach */
  uint32_t type;      /* 0 = add edge, 1 = delete edge */
  uint64_t src, dst, data;
  uint64_t tag;       /* caller's id, returned in the completion */
} rg_request;

typedef struct {
  uint64_t tag;
  uint64_t submit_ns, done_ns;  /* CLOCK_MONOTONIC */
  uint32_t instance, type;
  int32_t status;               /* rg_status of the batch that applied it */
  uint32_t epoch_size;
  uint64_t version;             /* the instance's epochs so far, this one included */
} rg_completion;

typedef struct {
  uint64_t completed, epochs, largest_epoch;
  double p50_us, p99_us, p999_us, max_us, mean_us;
} rg_server_stats;

int rg_server_create(uint64_t hbm_budget_bytes, double target_epoch_ms, uint64_t max_epoch, int per_update,
                     rg_server **out);
/* Admit a graph (labels already built with rg_build_tree for `algo`).
 * RG_ENOMEM_HBM when its device bytes would exceed the budget.  While
 * attached the graph runs no cluster levels (RG_OPT_CLUSTER_EDGES reads 0;
 * detach gives the value back): with other instances' epochs on the GPU a
 * level that needs a GPC of free SMs at once would wait for them. */
int rg_server_attach(rg_server *s, rg_graph *g, int algo, int directed, uint32_t *instance);
int rg_server_detach(rg_server *s, uint32_t instance);
/* Record the label history (rg_history_record of the modified vertices) after
 * every epoch of the instance, at versions 1, 2, ...; the graph needs
 * trace_modified and rg_history_enable.  version (nullable) receives the last
 * version recorded so far. */
int rg_server_history(rg_server *s, uint32_t instance, int enable, uint64_t *version);
/* Thread-safe; timestamps the requests. */
int rg_server_submit(rg_server *s, const rg_request *reqs, uint64_t n);
/* Drain up to cap completions (n = number written). */
int rg_server_poll(rg_server *s, rg_completion *out, uint64_t cap, uint64_t *n);
/* Wait until every submitted request has completed (timeout_ms; RG_ETIMEOUT). */
int rg_server_drain(rg_server *s, uint64_t timeout_ms);
int rg_server_stats_get(rg_server *s, rg_server_stats *st, int reset);
int rg_server_destroy(rg_server *s);

/* Closed-loop client load (the reference's simulated clients, one outstanding
 * update each, src/sssp_inc_rt.cpp:196-311), with exponential think time of
 * mean think_us between a completion and the client's next update (Poisson
 * arrivals per client).  Update number s (counted from `offset`, so that a
 * load can continue the window of an earlier one) inserts pairs[imported + s/2]
 * when s is even and deletes pairs[s/2] (the oldest loaded edge) when s is
 * odd: the sliding window of src/sssp_inc.cpp:251-326.
 * Weights as in rg_add_pairs when `weighted`.  The load stops issuing after
 * duration_s seconds or max_updates updates (0 = no cap), or when the window
 * reaches the end of `pairs`, and returns once all issued updates completed.
 * Every delete removes a loaded copy, so the final graph, and hence the final
 * values, depend only on the number of updates issued, not on their order.
 * open_loop = 1 makes each client an open Poisson source instead: it issues at
 * exponential intervals of mean think_us whether or not its earlier updates
 * have completed (the offered load no longer adapts to the server). */
typedef struct {
  uint32_t instance;
  uint32_t clients;
  double think_us;
  double duration_s;
  uint64_t max_updates;
  uint64_t offset;
  const uint64_t *pairs;
  uint64_t n_pairs, imported;
  int weighted;
  int open_loop;
  uint64_t seed;
  uint64_t *latencies_ns;  /* optional: every completed update's latency, in completion order */
  uint64_t latencies_cap;
} rg_load_config;

typedef struct {
  uint64_t completed, adds, dels, failed;
  double seconds, updates_per_s;
  double p50_us, p99_us, p999_us, max_us, mean_us;
  uint64_t epochs;        /* epochs of this instance during the load */
  double mean_epoch;      /* updates per epoch */
} rg_load_result;

/* Runs the loads of n configs concurrently (one generator thread each). */
int rg_server_run_load(rg_server *s, const rg_load_config *cfgs, uint64_t n, rg_load_result *results);

/* rg_server_poll that waits up to timeout_us microseconds for a first
 * completion when none is queued (the network front end's completion thread
 * uses it instead of polling in a loop). */
int rg_server_poll_wait(rg_server *s, rg_completion *out, uint64_t cap, uint64_t *n, uint64_t timeout_us);

/* ---- Network front end and write-ahead log --------------------------------
 * The reference's served driver (src/all_inc_rpc.cpp) takes updates from
 * remote clients as ClientUpdateRequest structs (core/rpc.hpp:19-32) and
 * answers each with a ClientUpdateResponse (:34-38); before serving, the first
 * connection's first requests are clock-synchronisation requests answered with
 * {0, 0} (src/all_inc_rpc.cpp:277-290, src/rpc_client.cpp:83-90).  With a WAL,
 * every update is appended to a 4 KB log block and applied only once its block
 * is durable; the blocks are written one after another (group commit,
 * src/all_inc_rpc.cpp:306-335,572-589).  The reference moves the structs over
 * UCX; here they move over TCP, byte for byte in the reference's x86-64
 * layout below. */
typedef struct {
  uint32_t client_id;
  uint32_t type;              /* 0 add, 1 delete, 2 end (ClientUpdateRequest::Type) */
  uint64_t src, dst, data;
  int64_t request_time_ns;    /* the client's std::chrono::high_resolution_clock */
} rg_client_update_request;   /* 40 bytes (core/rpc.hpp:19-32) */

typedef struct {
  uint32_t client_id;
  uint32_t pad;
  uint64_t version_id;        /* label version after the update (the instance's epoch count) */
} rg_client_update_response;  /* 16 bytes (core/rpc.hpp:34-38) */

/* One WAL record (the WAL struct of src/all_inc_rpc.cpp:306-316): 32 bytes.
 * A block is 4096 bytes: uint64 version (1, 2, ...; block k sits at byte
 * (k - 1) * 4096), uint64 record count, then up to 127 records. */
typedef struct {
  uint32_t type;       /* 0 add, 1 delete */
  uint32_t client_id;
  uint64_t src, dst, data;
} rg_wal_record;

typedef struct rg_frontend rg_frontend;

typedef struct {
  uint64_t connections, requests, updates, sync_requests, wal_blocks, failed;
  int64_t time_offset_ns;     /* mean (server clock - request_time) of the sync requests */
  double p50_us, p99_us, p999_us, max_us, mean_us;  /* request_time + offset -> response sent */
} rg_frontend_stats;

/* Serve `instance` of server s on a TCP listener at host:port (port 0 picks a
 * free port; rg_frontend_port reports it).  wal_path (nullable) enables the
 * write-ahead log, truncated at start.  sync_requests: how many clock-sync
 * requests open the first connection (the reference's clients send 1024;
 * 0 = none).  The front end drains the server's completion queue, so s should
 * be a server nothing else polls.  Each connection may carry many clients;
 * responses on a connection leave in request order.  A request the server
 * would refuse (vertex id or weight out of range) is answered at once with
 * version_id ~0 and is neither logged nor applied. */
int rg_frontend_start(rg_server *s, uint32_t instance, const char *host, uint16_t port, const char *wal_path,
                      uint32_t sync_requests, rg_frontend **out);
int rg_frontend_port(rg_frontend *f, uint16_t *port);
int rg_frontend_stats_get(rg_frontend *f, rg_frontend_stats *st);
/* Stops accepting, stops reading the connections, waits (up to timeout_ms:
 * RG_ETIMEOUT) for the updates already taken to complete and be answered,
 * flushes the WAL and frees the front end. */
int rg_frontend_stop(rg_frontend *f, uint64_t timeout_ms);

/* Read the records of a WAL file in order (blocks 1, 2, ... until a block is
 * missing, empty or out of sequence); n = records found (all of them, even
 * beyond cap).  No GPU needed. */
int rg_wal_read(const char *path, rg_wal_record *out, uint64_t cap, uint64_t *n);
/* Re-apply a WAL to a graph whose labels are built for `algo`: the records
 * in order, runs of adds and runs of deletes as batches (rg_apply_add /
 * rg_apply_del), which gives the graph and values of the logged run. */
int rg_wal_replay(rg_graph *g, int algo, const char *path, int directed, uint64_t *applied);

const char *rg_status_string(int status);
/* Last error message of the calling thread ("" if none). */
const char *rg_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
