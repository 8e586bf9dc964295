/* CPU restatement of RisGraph's incremental dependency-tree hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity checker: only tests/, the
 * package's smoke check and bench.py's CPU-baseline leg may load it.  The
 * product path (librisgraph_b200.so) never calls it.
 *
 * Sequential, deterministic C that follows the reference function by function
 * (citations are to the reference's core/graph.hpp, core/storage.hpp and the
 * src/ drivers).  Values are the reference's exactly; parents are the ones a
 * sequential run of the reference's algorithm picks (the reference's own
 * parents depend on thread races, so parents are checked structurally).
 * Pinned against the reference itself, compiled from its own sources by
 * oracle/ref/Makefile, through the fixtures in tests/golden/. */
#ifndef RG_ORACLE_H
#define RG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { RGO_BFS = 0, RGO_SSSP = 1, RGO_SSWP = 2, RGO_WCC = 3 };

typedef struct rgo_graph rgo_graph;

rgo_graph *rgo_create(uint64_t vertices, uint64_t hint_edges, int symmetric, int dual, int weighted);
void rgo_destroy(rgo_graph *g);

uint64_t rgo_add_edge(rgo_graph *g, uint64_t src, uint64_t dst, uint64_t w, int directed);
uint64_t rgo_del_edge(rgo_graph *g, uint64_t src, uint64_t dst, uint64_t w, int directed);
uint64_t rgo_get_edge_num(rgo_graph *g, uint64_t src, uint64_t dst, uint64_t w);
uint64_t rgo_get_outgoing_degree(rgo_graph *g, uint64_t v);
uint64_t rgo_get_incoming_degree(rgo_graph *g, uint64_t v);

uint64_t rgo_build_tree(rgo_graph *g, int algo, uint64_t root);
uint64_t rgo_update_tree_add(rgo_graph *g, int algo, uint64_t root, uint64_t src, uint64_t dst, uint64_t w, int directed);
uint64_t rgo_update_tree_add_batch(rgo_graph *g, int algo, uint64_t root, const uint64_t *src, const uint64_t *dst,
                                   const uint64_t *w, uint64_t n, int directed);
uint64_t rgo_update_tree_del(rgo_graph *g, int algo, uint64_t root, uint64_t src, uint64_t dst, uint64_t w, int directed);
uint64_t rgo_update_tree_del_batch(rgo_graph *g, int algo, uint64_t root, const uint64_t *src, const uint64_t *dst,
                                   const uint64_t *w, uint64_t n, int directed);
int rgo_need_update_tree_add(rgo_graph *g, int algo, uint64_t src, uint64_t dst, uint64_t w, int directed);
int rgo_need_update_tree_del(rgo_graph *g, uint64_t src, uint64_t dst, uint64_t w, int directed);

/* val/par/pw may be NULL.  par == vertices means "no parent". */
void rgo_get_labels(rgo_graph *g, uint64_t *val, uint64_t *par, uint64_t *pw);
uint64_t rgo_recomputes(rgo_graph *g);

/* Whole driver loops of the reference drivers src/sssp_inc.cpp (:251-326) and
 * src/sssp_inc_batch.cpp (:136-181) over an edge list in the reference format.
 * Weighted graphs use rg_gen_weight.  sums[k] = value checksum after step k. */
uint64_t rgo_run_inc(rgo_graph *g, int algo, uint64_t root, const uint64_t *pairs, uint64_t n_edges,
                     uint64_t imported, uint64_t steps, uint64_t *sums);
uint64_t rgo_run_batch(rgo_graph *g, int algo, uint64_t root, const uint64_t *pairs, uint64_t n_edges,
                       uint64_t imported, uint64_t batch, uint64_t n_batches, uint64_t *sums);
/* Bulk add of pairs[0..n) (weights from rg_gen_weight when weighted). */
void rgo_load(rgo_graph *g, const uint64_t *pairs, uint64_t n, int directed);

/* Structural check of a dependency tree (any implementation's):
 * returns 0 if every vertex with a parent p has a live edge (p->v, pw) and
 * equal_func(val[p], pw, val[v]) holds, every vertex without a parent holds its
 * init value, and the parent graph is acyclic; otherwise 1 + the first bad vertex
 * (in *bad_kind: 1 missing edge, 2 not tight, 3 init mismatch, 4 cycle). */
uint64_t rgo_validate_tree(rgo_graph *g, int algo, uint64_t root, const uint64_t *val, const uint64_t *par,
                           const uint64_t *pw, int *bad_kind);

#ifdef __cplusplus
}
#endif
#endif
