/* CPU restatement of RisGraph's incremental dependency-tree hot path.
 * TEST INFRASTRUCTURE ONLY (the parity checker); see rg_oracle.h.
 * Every function names the reference code it follows. */
#include "rg_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "rg_gen.h"

/* ---- per-algorithm hooks: src/bfs.cpp:76-91, src/sssp.cpp:67-91,
 *      src/sswp.cpp:76-91, src/wcc.cpp:62-86 ---- */
#define BFS_MAXL 65536ull      /* src/bfs.cpp:66 */
#define SSSP_MAXL 134217728ull /* src/sssp.cpp:66, src/sswp.cpp:66 */

static inline int hk_update(int algo, uint64_t s, uint64_t d, uint64_t w, uint64_t *nv) {
  switch (algo) {
    case RGO_BFS: *nv = s + 1; return s + 1 < d;
    case RGO_SSSP: *nv = s + w; return s + w < d;
    case RGO_SSWP: { uint64_t m = s < w ? s : w; *nv = m; return m > d; }
    default: *nv = s; return s < d;
  }
}
static inline int hk_equal(int algo, uint64_t s, uint64_t d, uint64_t w) {
  switch (algo) {
    case RGO_BFS: return s + 1 == d;
    case RGO_SSSP: return s + w == d;
    case RGO_SSWP: return (s < w ? s : w) == d;
    default: return s == d;
  }
}
static inline uint64_t hk_init(int algo, uint64_t v, uint64_t root, int *active) {
  switch (algo) {
    case RGO_BFS: *active = (v == root); return v == root ? 0 : BFS_MAXL;
    case RGO_SSSP: *active = (v == root); return v == root ? 0 : SSSP_MAXL;
    case RGO_SSWP: *active = (v == root); return v == root ? SSSP_MAXL : 0;
    default: *active = 1; return v;
  }
}

/* ---- dynamic adjacency: core/storage.hpp:282-430 (IndexedEdgeStorage) ---- */
typedef struct { uint64_t nbr, w; uint16_t num; } adj_t;   /* AdjEdge, core/type.hpp:21-54 */
typedef struct { adj_t *e; uint64_t len, cap, degree; } list_t;

/* key (vid, nbr, w) -> position in list; stands in for the per-list
 * dense_hash_map of core/storage.hpp:358-386 (lookup result is identical). */
typedef struct { uint64_t *k0, *k1, *k2; uint64_t *pos; uint64_t cap, cnt; } index_t;

typedef struct {
  list_t *lists;
  index_t idx;
} storage_t;

typedef struct { uint64_t *v; uint64_t len, cap; } vlist_t;

struct rgo_graph {
  uint64_t V, hint_edges;
  int symmetric, dual, weighted;
  storage_t out, in;
  uint64_t *val, *par, *pw;
  int64_t *inv;
  int64_t inv_idx;
  vlist_t a_in, a_out, a_tree;
  uint8_t *bm_in, *bm_out;
  uint64_t recomputes;
};

static inline uint64_t mix3(uint64_t a, uint64_t b, uint64_t c) {
  return rg_gen_splitmix64(a * 0x9E3779B97F4A7C15ull ^ rg_gen_splitmix64(b ^ rg_gen_splitmix64(c)));
}

static void index_grow(index_t *ix);
static uint64_t index_find(index_t *ix, uint64_t a, uint64_t b, uint64_t c, int *found) {
  uint64_t m = ix->cap - 1, h = mix3(a, b, c) & m;
  for (;;) {
    if (ix->pos[h] == UINT64_MAX) { *found = 0; return h; }
    if (ix->k0[h] == a && ix->k1[h] == b && ix->k2[h] == c) { *found = 1; return h; }
    h = (h + 1) & m;
  }
}
static void index_alloc(index_t *ix, uint64_t cap) {
  ix->cap = cap;
  ix->cnt = 0;
  ix->k0 = malloc(cap * 8); ix->k1 = malloc(cap * 8); ix->k2 = malloc(cap * 8);
  ix->pos = malloc(cap * 8);
  memset(ix->pos, 0xff, cap * 8);
}
static void index_grow(index_t *ix) {
  index_t old = *ix;
  index_alloc(ix, old.cap * 2);
  for (uint64_t i = 0; i < old.cap; i++) {
    if (old.pos[i] == UINT64_MAX) continue;
    int f;
    uint64_t h = index_find(ix, old.k0[i], old.k1[i], old.k2[i], &f);
    ix->k0[h] = old.k0[i]; ix->k1[h] = old.k1[i]; ix->k2[h] = old.k2[i]; ix->pos[h] = old.pos[i];
    ix->cnt++;
  }
  free(old.k0); free(old.k1); free(old.k2); free(old.pos);
}

/* IndexedEdgeStorage::update_edge, core/storage.hpp:345-398: find (nbr,w) or
 * append it with num 0; num += update only if the result stays >= 0 (16-bit);
 * degree += update unless a delete found num == 0; return the old num. */
static uint64_t storage_update(storage_t *st, uint64_t vid, uint64_t nbr, uint64_t w, int update) {
  index_t *ix = &st->idx;
  if (2 * (ix->cnt + 1) > ix->cap) index_grow(ix);
  int found;
  uint64_t h = index_find(ix, vid, nbr, w, &found);
  list_t *l = &st->lists[vid];
  uint64_t p;
  if (!found) {
    if (l->len == l->cap) {
      l->cap = l->cap ? 2 * l->cap : 4;
      l->e = realloc(l->e, l->cap * sizeof(adj_t));
    }
    p = l->len++;
    l->e[p].nbr = nbr; l->e[p].w = w; l->e[p].num = 0;
    ix->k0[h] = vid; ix->k1[h] = nbr; ix->k2[h] = w; ix->pos[h] = p;
    ix->cnt++;
  } else {
    p = ix->pos[h];
  }
  uint64_t cur = l->e[p].num;
  if ((int)l->e[p].num + update >= 0) l->e[p].num = (uint16_t)(l->e[p].num + update);
  l->degree += (uint64_t)((update > 0 || cur >= (uint64_t)(-(int64_t)update)) * (int64_t)update);
  return cur;
}

static uint64_t storage_num(storage_t *st, uint64_t vid, uint64_t nbr, uint64_t w) {
  int found;
  uint64_t h = index_find(&st->idx, vid, nbr, w, &found);
  if (!found) return 0;
  return st->lists[vid].e[st->idx.pos[h]].num;
}

static void vl_push(vlist_t *l, uint64_t v) {
  if (l->len == l->cap) {
    l->cap = l->cap ? 2 * l->cap : 1024;
    l->v = realloc(l->v, l->cap * 8);
  }
  l->v[l->len++] = v;
}
static void vl_swap(vlist_t *a, vlist_t *b) { vlist_t t = *a; *a = *b; *b = t; }

/* Graph ctor, core/graph.hpp:61-100 (empty parent = nbr V, :90). */
rgo_graph *rgo_create(uint64_t V, uint64_t hint_edges, int symmetric, int dual, int weighted) {
  rgo_graph *g = calloc(1, sizeof(rgo_graph));
  g->V = V;
  g->hint_edges = hint_edges ? hint_edges : V * 16;
  g->symmetric = symmetric; g->dual = dual; g->weighted = weighted;
  g->out.lists = calloc(V ? V : 1, sizeof(list_t));
  index_alloc(&g->out.idx, 1024);
  if (!symmetric) {
    g->in.lists = calloc(V ? V : 1, sizeof(list_t));
    index_alloc(&g->in.idx, 1024);
  }
  g->val = calloc(V ? V : 1, 8);
  g->par = malloc((V ? V : 1) * 8);
  g->pw = calloc(V ? V : 1, 8);
  for (uint64_t v = 0; v < V; v++) g->par[v] = V;
  g->inv = calloc(V ? V : 1, 8);
  g->bm_in = calloc(V ? V : 1, 1);
  g->bm_out = calloc(V ? V : 1, 1);
  return g;
}

static void storage_free(storage_t *st, uint64_t V) {
  if (!st->lists) return;
  for (uint64_t v = 0; v < V; v++) free(st->lists[v].e);
  free(st->lists);
  free(st->idx.k0); free(st->idx.k1); free(st->idx.k2); free(st->idx.pos);
}

void rgo_destroy(rgo_graph *g) {
  if (!g) return;
  storage_free(&g->out, g->V);
  storage_free(&g->in, g->V);
  free(g->val); free(g->par); free(g->pw); free(g->inv);
  free(g->a_in.v); free(g->a_out.v); free(g->a_tree.v);
  free(g->bm_in); free(g->bm_out);
  free(g);
}

static inline uint64_t key_w(rgo_graph *g, uint64_t w) { return g->weighted ? w : 0; }

/* Graph::add_edge, core/graph.hpp:203-227 (undirected form :206-211). */
uint64_t rgo_add_edge(rgo_graph *g, uint64_t s, uint64_t d, uint64_t w, int directed) {
  w = key_w(g, w);
  if (!directed) {
    rgo_add_edge(g, s, d, w, 1);
    return rgo_add_edge(g, d, s, w, 1) - (s == d);
  }
  uint64_t cur = storage_update(&g->out, s, d, w, 1);
  if (!g->symmetric) storage_update(&g->in, d, s, w, 1);
  return cur;
}

/* Graph::del_edge, core/graph.hpp:229-253. */
uint64_t rgo_del_edge(rgo_graph *g, uint64_t s, uint64_t d, uint64_t w, int directed) {
  w = key_w(g, w);
  if (!directed) {
    rgo_del_edge(g, s, d, w, 1);
    return rgo_del_edge(g, d, s, w, 1);
  }
  uint64_t cur = storage_update(&g->out, s, d, w, -1);
  if (!g->symmetric) storage_update(&g->in, d, s, w, -1);
  return cur;
}

uint64_t rgo_get_edge_num(rgo_graph *g, uint64_t s, uint64_t d, uint64_t w) {
  return storage_num(&g->out, s, d, key_w(g, w));
}
uint64_t rgo_get_outgoing_degree(rgo_graph *g, uint64_t v) { return g->out.lists[v].degree; }
uint64_t rgo_get_incoming_degree(rgo_graph *g, uint64_t v) {
  return g->symmetric ? g->out.lists[v].degree : g->in.lists[v].degree;
}

static inline list_t *out_list(rgo_graph *g, uint64_t v) { return &g->out.lists[v]; }
static inline list_t *in_list(rgo_graph *g, uint64_t v) {
  return g->symmetric ? &g->out.lists[v] : &g->in.lists[v];
}

/* update_label, core/graph.hpp:1765-1887: under the vertex lock (or 16-byte CAS),
 * if update_func still improves dst, write value and parent (src, w). */
static inline int update_label(rgo_graph *g, int algo, uint64_t src, uint64_t dst, uint64_t w) {
  uint64_t nv;
  if (!hk_update(algo, g->val[src], g->val[dst], w, &nv)) return 0;
  g->val[dst] = nv;
  g->par[dst] = src;
  g->pw[dst] = w;
  return 1;
}

/* Push lambda shared by build_tree (:910-935), do_update_tree_add (:1017-1042)
 * and the final push of do_update_tree_del (:1517-1541). */
static uint64_t push_vertex(rgo_graph *g, int algo, uint64_t src, vlist_t *next, uint8_t *next_bm) {
  uint64_t res = 0;
  list_t *l = out_list(g, src);
  for (uint64_t i = 0; i < l->len; i++) {
    adj_t e = l->e[i];
    if (e.num == 0) continue;
    uint64_t nv;
    if (hk_update(algo, g->val[src], g->val[e.nbr], e.w, &nv) && update_label(g, algo, src, e.nbr, e.w)) {
      if (next) vl_push(next, e.nbr);
      if (next_bm) next_bm[e.nbr] = 1;
      res++;
    }
  }
  return res;
}

/* Pull lambda (:936-976): best in-neighbour by update_func, then update_label. */
static uint64_t pull_vertex(rgo_graph *g, int algo, uint64_t dst, vlist_t *next, uint8_t *next_bm) {
  list_t *l = in_list(g, dst);
  uint64_t new_label = g->val[dst], new_src = UINT64_MAX, new_w = 0;
  for (uint64_t i = 0; i < l->len; i++) {
    adj_t e = l->e[i];
    if (e.num == 0) continue;
    uint64_t nv;
    if (hk_update(algo, g->val[e.nbr], new_label, e.w, &nv)) {
      new_label = nv; new_src = e.nbr; new_w = e.w;
    }
  }
  if (new_src == UINT64_MAX) return 0;
  if (update_label(g, algo, new_src, dst, new_w)) {
    if (next) vl_push(next, dst);
    if (next_bm) next_bm[dst] = 1;
    return 1;
  }
  return 0;
}

/* Graph::build_tree, core/graph.hpp:873-985, with stream_edges(Bitmap)
 * (:323-396): push over active out-edges, or pull over all in-edges when
 * active_edges >= V and >= hint/20 and the graph is dual (:334). */
uint64_t rgo_build_tree(rgo_graph *g, int algo, uint64_t root) {
  uint64_t V = g->V;
  memset(g->bm_in, 0, V);
  for (uint64_t v = 0; v < V; v++) {
    int act;
    g->val[v] = hk_init(algo, v, root, &act);
    g->par[v] = V;
    g->pw[v] = 0;
    if (act) g->bm_in[v] = 1;
  }
  uint64_t total = 0;
  for (;;) {
    memset(g->bm_out, 0, V);
    uint64_t active_edges = 0;
    for (uint64_t v = 0; v < V; v++)
      if (g->bm_in[v]) active_edges += out_list(g, v)->degree;
    int sparse = (active_edges < V || active_edges < g->hint_edges / 20 || !g->dual);
    uint64_t local = 0;
    if (sparse) {
      for (uint64_t v = 0; v < V; v++)
        if (g->bm_in[v] && out_list(g, v)->degree) local += push_vertex(g, algo, v, NULL, g->bm_out);
    } else {
      for (uint64_t v = 0; v < V; v++)
        if (in_list(g, v)->degree) local += pull_vertex(g, algo, v, NULL, g->bm_out);
    }
    uint8_t *t = g->bm_in; g->bm_in = g->bm_out; g->bm_out = t;
    total += local;
    if (!local) break;
  }
  return total;
}

/* do_update_tree_add, core/graph.hpp:1002-1116: push levels from active_in
 * (stream_edges_hybrid on a sparse set is always push, :577-614). */
static uint64_t do_update_tree_add(rgo_graph *g, int algo) {
  uint64_t total = 0;
  for (;;) {
    g->a_out.len = 0;
    uint64_t local = 0;
    for (uint64_t i = 0; i < g->a_in.len; i++) {
      uint64_t v = g->a_in.v[i];
      if (out_list(g, v)->degree) local += push_vertex(g, algo, v, &g->a_out, NULL);
    }
    vl_swap(&g->a_in, &g->a_out);
    total += local;
    if (!local) break;
  }
  return total;
}

/* Seed relax of one directed edge, core/graph.hpp:1140-1153 / :1185-1197. */
static uint64_t seed_add(rgo_graph *g, int algo, uint64_t s, uint64_t d, uint64_t w) {
  uint64_t nv;
  if (!hk_update(algo, g->val[s], g->val[d], w, &nv)) return 0;
  if (update_label(g, algo, s, d, w)) {
    vl_push(&g->a_in, d);
    return 1;
  }
  return 0;
}

/* update_tree_add (single edge), core/graph.hpp:1124-1160. */
uint64_t rgo_update_tree_add(rgo_graph *g, int algo, uint64_t root, uint64_t s, uint64_t d, uint64_t w, int directed) {
  (void)root;
  w = key_w(g, w);
  if (!directed) {
    uint64_t l = rgo_update_tree_add(g, algo, root, s, d, w, 1);
    uint64_t r = rgo_update_tree_add(g, algo, root, d, s, w, 1);
    return l + r;
  }
  uint64_t nv;
  if (!hk_update(algo, g->val[s], g->val[d], w, &nv)) return 0;
  g->a_in.len = 0;
  uint64_t total = seed_add(g, algo, s, d, w);
  return total + do_update_tree_add(g, algo);
}

/* update_tree_add (batch), core/graph.hpp:1162-1218. */
uint64_t rgo_update_tree_add_batch(rgo_graph *g, int algo, uint64_t root, const uint64_t *src, const uint64_t *dst,
                                   const uint64_t *w, uint64_t n, int directed) {
  if (n == 1) return rgo_update_tree_add(g, algo, root, src[0], dst[0], w ? w[0] : 0, directed);
  g->a_in.len = 0;
  uint64_t total = 0;
  for (uint64_t i = 0; i < n; i++) {
    uint64_t ww = key_w(g, w ? w[i] : 0);
    total += seed_add(g, algo, src[i], dst[i], ww);
    if (directed) continue;
    total += seed_add(g, algo, dst[i], src[i], ww);
  }
  if (g->a_in.len == 0) return total;
  return total + do_update_tree_add(g, algo);
}

/* need_update_tree_add, core/graph.hpp:987-1000. */
int rgo_need_update_tree_add(rgo_graph *g, int algo, uint64_t s, uint64_t d, uint64_t w, int directed) {
  w = key_w(g, w);
  uint64_t nv;
  int r = hk_update(algo, g->val[s], g->val[d], w, &nv);
  if (!directed) r = r || hk_update(algo, g->val[d], g->val[s], w, &nv);
  return r;
}

static inline int parent_is(rgo_graph *g, uint64_t d, uint64_t s, uint64_t w) {
  return g->par[d] == s && g->pw[d] == w;
}

/* need_update_tree_del, core/graph.hpp:1220-1233. */
int rgo_need_update_tree_del(rgo_graph *g, uint64_t s, uint64_t d, uint64_t w, int directed) {
  w = key_w(g, w);
  int r = parent_is(g, d, s, w);
  if (!directed) r = r || parent_is(g, s, d, w);
  return r;
}

/* has_parents, core/graph.hpp:1889-1907. */
static int has_parents(rgo_graph *g, uint64_t x, int *need_recompute) {
  uint64_t num = 0;
  for (;;) {
    if (g->inv[x] == g->inv_idx || g->inv[x] == -g->inv_idx) return 1;
    if (g->par[x] != g->V) x = g->par[x];
    else break;
    if ((double)(++num) > (double)g->V * 0.1) {
      *need_recompute = 1;
      return 1;
    }
  }
  return 0;
}

/* do_update_tree_del, core/graph.hpp:1235-1612. */
static uint64_t do_update_tree_del(rgo_graph *g, int algo, uint64_t root) {
  uint64_t V = g->V, size_tree = 0;
  int need_recompute = 0;
  for (uint64_t i = 0, active_vertices = g->a_in.len; i < V && active_vertices; i++) {
    /* full recompute fallback, :1252-1322 */
    if (need_recompute || (i <= 10 && (double)(size_tree + active_vertices) > 0.05 * (double)V &&
                           size_tree + active_vertices > 2000000)) {
      memset(g->inv, 0, V * 8);
      g->recomputes++;
      return rgo_build_tree(g, algo, root);
    }
    /* rescue over in-edges (transposed push), :1323-1361 */
    if (i <= 5 || active_vertices < 8192 * 2) {
      for (uint64_t k = 0; k < g->a_in.len; k++) {
        uint64_t dst = g->a_in.v[k];
        list_t *l = in_list(g, dst);
        for (uint64_t j = 0; j < l->len; j++) {
          adj_t e = l->e[j];
          if (e.num == 0) continue;
          if (hk_equal(algo, g->val[e.nbr], g->val[dst], e.w) && g->inv[dst] == g->inv_idx &&
              !has_parents(g, e.nbr, &need_recompute)) {
            g->inv[dst] = -g->inv_idx;
            g->par[dst] = e.nbr;
            g->pw[dst] = e.w;
          }
        }
      }
    }
    if (need_recompute) continue;
    /* collect the still-invalid set, :1363-1380 */
    g->a_out.len = 0;
    for (uint64_t k = 0; k < g->a_in.len; k++) {
      uint64_t vid = g->a_in.v[k];
      if (g->inv[vid] == g->inv_idx) {
        vl_push(&g->a_out, vid);
        vl_push(&g->a_tree, vid);
        size_tree++;
      } else if (g->inv[vid] == -g->inv_idx) {
        g->inv[vid] = 0;
      }
    }
    /* invalidate tree children through out-edges, :1381-1417 */
    g->a_in.len = 0;
    active_vertices = 0;
    for (uint64_t k = 0; k < g->a_out.len; k++) {
      uint64_t src = g->a_out.v[k];
      list_t *l = out_list(g, src);
      if (!l->degree) continue;
      for (uint64_t j = 0; j < l->len; j++) {
        adj_t e = l->e[j];
        if (e.num == 0) continue;
        if (parent_is(g, e.nbr, src, e.w) && g->inv[e.nbr] == 0) {
          g->inv[e.nbr] = g->inv_idx;
          vl_push(&g->a_in, e.nbr);
          active_vertices++;
        }
      }
    }
  }
  /* reset the invalid set, :1420-1430 */
  for (uint64_t k = 0; k < g->a_tree.len; k++) {
    uint64_t vid = g->a_tree.v[k];
    int act;
    g->val[vid] = hk_init(algo, vid, root, &act);
    g->par[vid] = V;
    g->pw[vid] = 0;
    g->inv[vid] = 0;
  }
  vl_swap(&g->a_in, &g->a_tree);
  /* one transposed pull over the reset set, :1433-1511 */
  uint64_t total = 0;
  for (uint64_t k = 0; k < g->a_in.len; k++) {
    uint64_t dst = g->a_in.v[k];
    if (in_list(g, dst)->degree) total += pull_vertex(g, algo, dst, NULL, NULL);
  }
  /* push to a fixpoint, :1513-1608 */
  return total + do_update_tree_add(g, algo);
}

/* update_tree_del (single edge), core/graph.hpp:1622-1656. */
uint64_t rgo_update_tree_del(rgo_graph *g, int algo, uint64_t root, uint64_t s, uint64_t d, uint64_t w, int directed) {
  w = key_w(g, w);
  if (!directed) {
    uint64_t l = rgo_update_tree_del(g, algo, root, s, d, w, 1);
    uint64_t r = rgo_update_tree_del(g, algo, root, d, s, w, 1);
    return l + r;
  }
  if (!parent_is(g, d, s, w)) return 0;
  g->a_in.len = 0;
  g->a_tree.len = 0;
  vl_push(&g->a_in, d);
  g->inv_idx++;
  g->inv[d] = g->inv_idx;
  return do_update_tree_del(g, algo, root);
}

/* update_tree_del (batch), core/graph.hpp:1658-1718. */
uint64_t rgo_update_tree_del_batch(rgo_graph *g, int algo, uint64_t root, const uint64_t *src, const uint64_t *dst,
                                   const uint64_t *w, uint64_t n, int directed) {
  if (n == 1) return rgo_update_tree_del(g, algo, root, src[0], dst[0], w ? w[0] : 0, directed);
  g->a_in.len = 0;
  g->a_tree.len = 0;
  g->inv_idx++;
  for (uint64_t i = 0; i < n; i++) {
    uint64_t ww = key_w(g, w ? w[i] : 0);
    for (int dir = 0; dir < (directed ? 1 : 2); dir++) {
      uint64_t s = dir ? dst[i] : src[i], d = dir ? src[i] : dst[i];
      if (parent_is(g, d, s, ww) && g->inv[d] != g->inv_idx) {
        g->inv[d] = g->inv_idx;
        vl_push(&g->a_in, d);
      }
    }
  }
  if (g->a_in.len == 0) return 0;
  return do_update_tree_del(g, algo, root);
}

void rgo_get_labels(rgo_graph *g, uint64_t *val, uint64_t *par, uint64_t *pw) {
  if (val) memcpy(val, g->val, g->V * 8);
  if (par) memcpy(par, g->par, g->V * 8);
  if (pw) memcpy(pw, g->pw, g->V * 8);
}

uint64_t rgo_recomputes(rgo_graph *g) { return g->recomputes; }

static inline uint64_t edge_weight(rgo_graph *g, uint64_t s, uint64_t d) {
  return g->weighted ? rg_gen_weight(s, d) : 0;
}

void rgo_load(rgo_graph *g, const uint64_t *pairs, uint64_t n, int directed) {
  for (uint64_t i = 0; i < n; i++) {
    uint64_t s = pairs[2 * i], d = pairs[2 * i + 1];
    rgo_add_edge(g, s, d, edge_weight(g, s, d), directed);
  }
}

/* Sliding window of src/sssp_inc.cpp:251-326: insert raw[i], repair on 0->1;
 * delete raw[i-imported], repair on 1->0. */
uint64_t rgo_run_inc(rgo_graph *g, int algo, uint64_t root, const uint64_t *pairs, uint64_t n_edges,
                     uint64_t imported, uint64_t steps, uint64_t *sums) {
  int directed = algo != RGO_WCC;
  uint64_t end = imported + steps < n_edges ? imported + steps : n_edges, k = 0;
  for (uint64_t i = imported; i < end; i++, k++) {
    uint64_t s = pairs[2 * i], d = pairs[2 * i + 1], w = edge_weight(g, s, d);
    if (rgo_add_edge(g, s, d, w, directed) == 0) rgo_update_tree_add(g, algo, root, s, d, w, directed);
    s = pairs[2 * (i - imported)]; d = pairs[2 * (i - imported) + 1]; w = edge_weight(g, s, d);
    if (rgo_del_edge(g, s, d, w, directed) == 1) rgo_update_tree_del(g, algo, root, s, d, w, directed);
    if (sums) sums[k] = rg_gen_value_checksum(g->val, g->V);
  }
  return k;
}

/* Batches of src/sssp_inc_batch.cpp:136-181: all inserts of the batch (repair
 * the 0->1 ones together), then all deletes (repair the 1->0 ones together). */
uint64_t rgo_run_batch(rgo_graph *g, int algo, uint64_t root, const uint64_t *pairs, uint64_t n_edges,
                       uint64_t imported, uint64_t batch, uint64_t n_batches, uint64_t *sums) {
  int directed = algo != RGO_WCC;
  uint64_t *bs = malloc(batch * 8), *bd = malloc(batch * 8), *bw = malloc(batch * 8);
  uint64_t nb = 0;
  for (uint64_t b0 = imported; b0 < n_edges && nb < n_batches; b0 += batch, nb++) {
    uint64_t b1 = b0 + batch < n_edges ? b0 + batch : n_edges, len = 0;
    for (uint64_t i = b0; i < b1; i++) {
      uint64_t s = pairs[2 * i], d = pairs[2 * i + 1], w = edge_weight(g, s, d);
      if (rgo_add_edge(g, s, d, w, directed) == 0) { bs[len] = s; bd[len] = d; bw[len] = w; len++; }
    }
    rgo_update_tree_add_batch(g, algo, root, bs, bd, bw, len, directed);
    len = 0;
    for (uint64_t i = b0; i < b1; i++) {
      uint64_t j = i - imported;
      uint64_t s = pairs[2 * j], d = pairs[2 * j + 1], w = edge_weight(g, s, d);
      if (rgo_del_edge(g, s, d, w, directed) == 1) { bs[len] = s; bd[len] = d; bw[len] = w; len++; }
    }
    rgo_update_tree_del_batch(g, algo, root, bs, bd, bw, len, directed);
    if (sums) sums[nb] = rg_gen_value_checksum(g->val, g->V);
  }
  free(bs); free(bd); free(bw);
  return nb;
}

uint64_t rgo_validate_tree(rgo_graph *g, int algo, uint64_t root, const uint64_t *val, const uint64_t *par,
                           const uint64_t *pw, int *bad_kind) {
  uint64_t V = g->V;
  *bad_kind = 0;
  for (uint64_t v = 0; v < V; v++) {
    int act;
    if (par[v] >= V) {
      if (val[v] != hk_init(algo, v, root, &act)) { *bad_kind = 3; return v + 1; }
      continue;
    }
    uint64_t p = par[v], w = key_w(g, pw[v]);
    if (storage_num(&g->out, p, v, w) == 0) { *bad_kind = 1; return v + 1; }
    if (!hk_equal(algo, val[p], val[v], w)) { *bad_kind = 2; return v + 1; }
  }
  /* acyclicity: colour walk with path marks */
  uint8_t *state = calloc(V ? V : 1, 1);
  for (uint64_t v = 0; v < V; v++) {
    if (state[v]) continue;
    uint64_t x = v;
    while (x < V && state[x] == 0) { state[x] = 1; x = par[x]; }
    if (x < V && state[x] == 1) { free(state); *bad_kind = 4; return x + 1; }
    x = v;
    while (x < V && state[x] == 1) { state[x] = 2; x = par[x]; }
  }
  free(state);
  return 0;
}
