// Autotuner of the level-mode knobs (rg_autotune in include/risgraph_b200.h).
//
// The level engine picks each level's kernel from the frontier size with a few
// thresholds (rg_option): when a build level pulls, when BFS goes bottom-up,
// when a push level is dense or edge-balanced, and up to which size a frontier
// stays in one CTA.  The best values depend on the graph's degree distribution
// and on the algorithm, so this tuner measures them on the graph itself:
// coordinate descent over each knob's candidate values, timing full builds
// (and, when the caller passes a sample batch, insert+delete round trips of
// that batch, which leave the graph as it was), keeping the fastest value of
// each knob in turn.  Every trial's values are checked against the first
// build's checksum: the knobs only choose kernels, so a different checksum is
// an error, never a trade-off.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <vector>

#include "rg_internal.cuh"

namespace {

double median(std::vector<double> v) {
  std::sort(v.begin(), v.end());
  return v.empty() ? 0.0 : v[v.size() / 2];
}

struct Tuner {
  rg_graph *g;
  int algo;
  uint64_t root;
  const rg_edge *sample;
  uint64_t n_sample;
  int directed;
  int reps;
  uint64_t want_sum = 0;
  uint64_t trials = 0;

  int build_ms(double *ms) {
    std::vector<double> t;
    int rc = rg_build_tree(g, algo, root, nullptr);  // warm-up: rebuilds cached graphs after a knob change
    for (int r = 0; !rc && r < reps; r++) {
      auto a = std::chrono::steady_clock::now();
      rc = rg_build_tree(g, algo, root, nullptr);
      t.push_back(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count());
    }
    uint64_t sum = 0;
    if (!rc) rc = rg_value_checksum(g, &sum);
    if (!rc && sum != want_sum) {
      rg::set_error("autotune: a level-mode setting changed the values");
      rc = RG_ESTATE;
    }
    trials++;
    *ms = median(t);
    return rc;
  }

  // builds plus sample round trips, for the knob that both use
  int both_ms(double *ms) {
    double a = 0, b = 0;
    int rc = build_ms(&a);
    if (!rc) rc = apply_ms(&b);
    *ms = a + b;
    return rc;
  }

  // insert + delete of the sample (the graph returns to its state)
  int apply_ms(double *ms) {
    if (!n_sample) {
      *ms = 0;
      return RG_OK;
    }
    std::vector<double> t;
    int rc = RG_OK;
    for (int r = 0; !rc && r <= reps; r++) {
      auto a = std::chrono::steady_clock::now();
      rc = rg_apply_add(g, algo, sample, n_sample, directed, nullptr);
      if (!rc) rc = rg_apply_del(g, algo, sample, n_sample, directed, nullptr);
      if (r) t.push_back(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count());
    }
    uint64_t sum = 0;
    if (!rc) rc = rg_value_checksum(g, &sum);
    if (!rc && sum != want_sum) {
      rg::set_error("autotune: the sample round trip changed the values");
      rc = RG_ESTATE;
    }
    trials++;
    *ms = median(t);
    return rc;
  }

  // best value of one knob by `measure` (build_ms or apply_ms)
  template <typename M>
  int tune(int option, const std::vector<uint64_t> &cands, M measure, double *best_ms) {
    uint64_t best = 0;
    int rc = rg_get_option(g, option, &best);
    if (rc) return rc;
    double cur = 0;
    if ((rc = (this->*measure)(&cur))) return rc;
    for (uint64_t c : cands) {
      if (c == best) continue;
      if ((rc = rg_set_option(g, option, c))) return rc;
      double ms = 0;
      if ((rc = (this->*measure)(&ms))) return rc;
      if (ms < cur * 0.95) {  // a clear win only (timings move by a few percent)
        cur = ms;
        best = c;
      }
    }
    if ((rc = rg_set_option(g, option, best))) return rc;
    *best_ms = cur;
    return RG_OK;
  }
};

}  // namespace

extern "C" int rg_autotune(rg_graph *g, int algo, uint64_t root, const rg_edge *sample, uint64_t n_sample,
                           int directed, int reps, rg_tune_report *out) {
  if (!g || !out || (n_sample && !sample)) return RG_EINVAL;
  Tuner t{g, algo, root, sample, n_sample, directed, reps > 0 ? reps : 5};
  int rc = rg_build_tree(g, algo, root, nullptr);
  if (!rc) rc = rg_value_checksum(g, &t.want_sum);
  if (rc) return rc;
  *out = rg_tune_report{};
  if ((rc = t.build_ms(&out->build_ms_before))) return rc;
  if ((rc = t.apply_ms(&out->apply_ms_before))) return rc;
  constexpr int NOPT = RG_OPT_CLUSTER_EDGES + 1;
  uint64_t orig[NOPT];
  for (int o = 0; o < NOPT; o++) rg_get_option(g, o, &orig[o]);
  double ms = 0;
  // build knobs
  if (algo == RG_BFS) {
    if ((rc = t.tune(RG_OPT_BFS_BU_DIV, {16, 32, 64, 128, 256}, &Tuner::build_ms, &ms))) return rc;
  } else {
    if ((rc = t.tune(RG_OPT_PULL_DIV, {16, 32, 64, 128, 256}, &Tuner::build_ms, &ms))) return rc;
  }
  if (algo != RG_BFS && (rc = t.tune(RG_OPT_PULL_SPLIT, {0, 1}, &Tuner::build_ms, &ms))) return rc;
  if ((rc = t.tune(RG_OPT_DENSE_DIV, {10, 20, 40, 80}, &Tuner::build_ms, &ms))) return rc;
  if ((rc = t.tune(RG_OPT_LBS_MIN, {512, 2048, 8192, 32768, 131072}, &Tuner::build_ms, &ms))) return rc;
  // small-frontier knob: builds and the sample's round trips together
  if ((rc = t.tune(RG_OPT_TINY_EDGES, {0, 8192, 32768, 131072}, &Tuner::both_ms, &ms))) return rc;
  // mid-size frontiers in one thread-block cluster: builds and round trips together
  if ((rc = t.tune(RG_OPT_CLUSTER_EDGES, {0, 16384, 65536, 262144}, &Tuner::both_ms, &ms))) return rc;
  if ((rc = t.build_ms(&out->build_ms_after))) return rc;
  if ((rc = t.apply_ms(&out->apply_ms_after))) return rc;
  if (out->build_ms_after + out->apply_ms_after > 1.05 * (out->build_ms_before + out->apply_ms_before)) {
    // the knobs interact; when their combination lost, keep the settings the graph had
    for (int o = 0; o < NOPT; o++) rg_set_option(g, o, orig[o]);
    if ((rc = t.build_ms(&out->build_ms_after))) return rc;
    if ((rc = t.apply_ms(&out->apply_ms_after))) return rc;
  }
  for (int o = 0; o <= RG_OPT_CLUSTER_EDGES; o++) rg_get_option(g, o, &out->options[o]);
  out->trials = t.trials;
  // leave the labels of a fresh build, as rg_build_tree would
  return rg_build_tree(g, algo, root, nullptr);
}
