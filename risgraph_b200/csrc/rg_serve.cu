// Served mode (rg_server_* in include/risgraph_b200.h): continuous batching of
// single-edge updates over several resident graph instances.
//
// The reference serves updates from simulated clients in epochs
// (src/sssp_inc_rt.cpp:119-441): inside an epoch, safe updates are applied at
// once and unsafe ones are queued, then the unsafe queue is applied one update
// at a time; the epoch ends when the oldest queued update has waited 0.8 of the
// timeout or the queue passed an adaptive threshold (:139-148, :394-412).
//
// Here every instance owns a worker thread and the graph's own CUDA stream.
// The worker takes everything that queued while its previous epoch was on the
// GPU (up to an adaptive cap) and applies it as one add batch and one delete
// batch through the fused storage + repair submission (rg_apply_add_del, one
// launch for both when they are small): safe updates cost only their
// multiplicity change, unsafe ones share one repair.  Batching changes no result: the values after an epoch are
// the unique fixpoint of the graph after the epoch's updates.  The one order
// that batching could change, a delete of an edge followed by an insert of the
// same edge (adds run before deletes), ends the epoch before the insert.
// Instances never share a stream or a lock on the apply path, so epochs of
// different instances overlap on the device.
#include <cuda_runtime.h>
#include <sys/prctl.h>
#include <time.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <queue>
#include <random>
#include <thread>
#include <unordered_set>
#include <vector>

#include "rg_gen.h"
#include "rg_internal.cuh"

namespace {

// How long an idle instance worker spins for the next request before it
// sleeps on its condition variable.
constexpr uint64_t SPIN_NS = 200000;

uint64_t now_ns() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (uint64_t)ts.tv_sec * 1000000000ull + (uint64_t)ts.tv_nsec;
}

struct Item {
  rg_request r;
  uint64_t submit_ns;
};

// Completions of one instance while a load runs on it.
struct Sink {
  std::mutex mu;
  std::condition_variable cv;
  std::vector<rg_completion> items;
};

struct Instance {
  uint32_t id = 0;
  rg_graph *g = nullptr;
  int algo = 0, directed = 1;
  uint64_t bytes = 0;
  std::mutex mu;  // q, stop, sink
  std::condition_variable cv;
  std::deque<Item> q;
  std::atomic<uint64_t> qn{0};  // q.size(), readable without the lock
  bool stop = false;
  Sink *sink = nullptr;
  std::thread worker;
  uint64_t cap = 1;  // epoch cap, worker-owned
  std::atomic<int> history{0};  // record the label history after every epoch
  uint64_t version = 0;         // history version, worker-owned
  std::atomic<uint64_t> epochs{0}, applied{0};
  uint64_t cluster_edges = 0;  // the graph's RG_OPT_CLUSTER_EDGES, given back at detach
};

// Key of an edge for the delete-then-insert check: canonical orientation on
// undirected graphs, where (u,v) and (v,u) name one edge.
uint64_t edge_key(const rg_request &r, int directed) {
  uint64_t a = r.src, b = r.dst;
  if (!directed && a > b) std::swap(a, b);
  uint64_t h = rg_gen_splitmix64(a * 0x9E3779B97F4A7C15ull ^ rg_gen_splitmix64(b));
  return rg_gen_splitmix64(h ^ r.data);
}

double pct(const std::vector<uint64_t> &sorted, double q) {
  if (sorted.empty()) return 0.0;
  size_t i = std::min(sorted.size() - 1, (size_t)(q * (double)sorted.size()));
  return sorted[i] * 1e-3;
}

}  // namespace

struct rg_server {
  uint64_t budget = 0, used = 0;
  double target_ms = 0.5;
  uint64_t max_epoch = 1;
  int per_update = 0;
  std::mutex mu;  // inst, used
  std::vector<std::shared_ptr<Instance>> inst;
  std::mutex cmu;  // everything below
  std::condition_variable ccv;
  std::vector<rg_completion> done;
  uint64_t submitted = 0, completed = 0, epochs = 0, largest = 0;
  std::vector<uint64_t> lat;
};

namespace {

std::shared_ptr<Instance> find(rg_server *s, uint32_t id) {
  std::lock_guard<std::mutex> lk(s->mu);
  if (id >= s->inst.size()) return nullptr;
  return s->inst[id];
}

void worker_main(rg_server *s, Instance *in) {
  std::vector<Item> batch;
  std::vector<rg_edge> adds, dels;
  std::vector<rg_completion> out;
  std::unordered_set<uint64_t> deleted;
  for (;;) {
    Sink *sink = nullptr;
    {
      std::unique_lock<std::mutex> lk(in->mu);
      if (in->q.empty() && !in->stop) {
        // Wait for the next request spinning first: waking a sleeping thread
        // through the condition variable costs tens of microseconds on a
        // virtualised host, as much as applying a single update.
        lk.unlock();
        const uint64_t until = now_ns() + SPIN_NS;
        while (in->qn.load(std::memory_order_acquire) == 0 && now_ns() < until) {
#if defined(__x86_64__)
          __builtin_ia32_pause();
#endif
        }
        lk.lock();
      }
      in->cv.wait(lk, [&] { return in->stop || !in->q.empty(); });
      if (in->q.empty()) break;  // stopped and drained
      const uint64_t lim = s->per_update ? 1 : in->cap;
      batch.clear();
      deleted.clear();
      while (!in->q.empty() && batch.size() < lim) {
        const Item &it = in->q.front();
        const uint64_t k = edge_key(it.r, in->directed);
        if (it.r.type == 0 && deleted.count(k)) break;  // delete-then-insert: next epoch
        if (it.r.type == 1) deleted.insert(k);
        batch.push_back(it);
        in->q.pop_front();
        in->qn.fetch_sub(1, std::memory_order_relaxed);
      }
      sink = in->sink;
    }
    adds.clear();
    dels.clear();
    for (const Item &it : batch) (it.r.type ? dels : adds).push_back(rg_edge{it.r.src, it.r.dst, it.r.data});
    const uint64_t t0 = now_ns();
    int rc = RG_OK;
    if (!adds.empty() && !dels.empty())
      rc = rg_apply_add_del(in->g, in->algo, adds.data(), adds.size(), dels.data(), dels.size(), in->directed);
    else if (!adds.empty())
      rc = rg_apply_add(in->g, in->algo, adds.data(), adds.size(), in->directed, nullptr);
    else if (!dels.empty())
      rc = rg_apply_del(in->g, in->algo, dels.data(), dels.size(), in->directed, nullptr);
    // the modified vertices of the epoch go to the label history at the next
    // version (src/sssp_inc_rt.cpp:338-343 records after every update)
    if (!rc && in->history.load(std::memory_order_relaxed)) rc = rg_history_record(in->g, ++in->version, 0);
    const uint64_t t1 = now_ns();
    // Adapt the cap to keep one epoch within the target (cf. the threshold
    // update of src/sssp_inc_rt.cpp:394-412, driven by time instead of timeouts).
    const double ms = (t1 - t0) * 1e-6;
    // (epochs cost a fixed ~50 us plus a small share per update, so the cap
    // grows while an epoch stays under 3/4 of the target)
    if (ms > s->target_ms && in->cap > 1) {
      in->cap = std::max<uint64_t>(1, in->cap * 3 / 4);
    } else if (batch.size() >= in->cap && ms < 0.75 * s->target_ms) {
      in->cap = std::min<uint64_t>(s->max_epoch, in->cap + in->cap / 4 + 1);
    }
    const uint64_t version = in->epochs.fetch_add(1, std::memory_order_relaxed) + 1;
    in->applied.fetch_add(batch.size(), std::memory_order_relaxed);
    out.clear();
    for (const Item &it : batch)
      out.push_back(rg_completion{it.r.tag, it.submit_ns, t1, in->id, it.r.type, rc, (uint32_t)batch.size(), version});
    {
      std::lock_guard<std::mutex> lk(s->cmu);
      for (const rg_completion &c : out) s->lat.push_back(c.done_ns - c.submit_ns);
      if (!sink) s->done.insert(s->done.end(), out.begin(), out.end());
      s->completed += out.size();
      s->epochs++;
      s->largest = std::max<uint64_t>(s->largest, out.size());
    }
    s->ccv.notify_all();
    if (sink) {
      {
        std::lock_guard<std::mutex> lk(sink->mu);
        sink->items.insert(sink->items.end(), out.begin(), out.end());
      }
      sink->cv.notify_one();
    }
  }
}

int check_request(const Instance &in, const rg_request &r) {
  const rg::Graph &g = in.g->g;
  if (r.type > 1) {
    rg::set_error("request type must be 0 (add) or 1 (delete)");
    return RG_EINVAL;
  }
  if (r.src >= g.V || r.dst >= g.V) {
    rg::set_error("VertexId error.");
    return RG_EINVAL_VID;
  }
  if (g.weighted && r.data >= rg::W_LIMIT) {
    rg::set_error("edge weight >= 2^64 - 2^27 (the reference's u64 sums would wrap)");
    return RG_EINVAL_WEIGHT;
  }
  return RG_OK;
}

// One client load (see rg_load_config).  The clients that may issue are kept
// in a min-heap by the time they issue next, so one generator thread serves
// thousands of clients without scanning them all on every wake-up; its timed
// waits run with a 1 us timer slack (the default 50 us would add to the think
// times).
void run_load(rg_server *s, Instance *in, const rg_load_config &c, Sink &sink, rg_load_result &r) {
  prctl(PR_SET_TIMERSLACK, 1000UL, 0, 0, 0);
  const uint32_t C = std::max<uint32_t>(1, c.clients);
  std::mt19937_64 rng(c.seed);
  std::exponential_distribution<double> think(1.0);
  const bool open = c.open_loop != 0;
  // an open source needs a finite rate
  const double think_ns = c.think_us > 0 ? c.think_us * 1e3 : (open ? 1e3 : 0.0);
  const uint64_t limit = c.max_updates ? c.max_updates : ~0ull;
  const uint64_t t_start = now_ns();
  const uint64_t t_stop = t_start + (uint64_t)(std::max(0.0, c.duration_s) * 1e9);
  using Ev = std::pair<uint64_t, uint32_t>;  // (issue time, client)
  std::priority_queue<Ev, std::vector<Ev>, std::greater<Ev>> due;
  for (uint32_t k = 0; k < C; k++) due.push({open ? t_start + (uint64_t)(think(rng) * think_ns) : t_start, k});
  std::vector<rg_request> reqs;
  std::vector<rg_completion> got;
  std::vector<uint64_t> lat;
  uint64_t issued = 0, outstanding = 0, last_done = t_start, e0 = in->epochs.load(), a0 = in->applied.load();
  bool issuing = true;
  double sum_us = 0;
  for (;;) {
    uint64_t now = now_ns();
    if (now >= t_stop) issuing = false;
    if (issuing) {
      reqs.clear();
      while (issuing && !due.empty() && due.top().first <= now) {
        const Ev ev = due.top();
        const uint64_t sn = c.offset + issued;
        const bool is_add = (sn & 1) == 0;
        const uint64_t idx = is_add ? c.imported + sn / 2 : sn / 2;
        // (a delete's index is below the insert's before it: the window end bounds both)
        if (issued >= limit || idx >= c.n_pairs) {
          issuing = false;
          break;
        }
        due.pop();
        const uint64_t u = c.pairs[2 * idx], v = c.pairs[2 * idx + 1];
        reqs.push_back(rg_request{in->id, is_add ? 0u : 1u, u, v, c.weighted ? rg_gen_weight(u, v) : 0, ev.second});
        // open: Poisson arrivals, independent of completions; closed: next issue after the completion
        if (open) due.push({ev.first + (uint64_t)(think(rng) * think_ns), ev.second});
        issued++;
      }
      if (!reqs.empty()) {
        int rc = rg_server_submit(s, reqs.data(), reqs.size());
        if (rc) {
          // nothing of this call was queued
          r.failed += reqs.size();
          issuing = false;
        } else {
          outstanding += reqs.size();
          for (const rg_request &q : reqs) (q.type ? r.dels : r.adds)++;
        }
      }
    }
    if (!issuing && outstanding == 0) break;
    const uint64_t wake = (issuing && !due.empty()) ? due.top().first : ~0ull;
    {
      std::unique_lock<std::mutex> lk(sink.mu);
      if (sink.items.empty()) {
        now = now_ns();
        if (wake == ~0ull) {
          // a completion is due; bound the wait so a stuck worker cannot hang the load
          if (!sink.cv.wait_for(lk, std::chrono::seconds(60), [&] { return !sink.items.empty(); })) {
            r.failed += outstanding;
            break;
          }
        } else if (wake > now) {
          sink.cv.wait_for(lk, std::chrono::nanoseconds(wake - now), [&] { return !sink.items.empty(); });
        }
      }
      got.clear();
      got.swap(sink.items);
    }
    for (const rg_completion &d : got) {
      outstanding--;
      r.completed++;
      if (d.status) r.failed++;
      if (c.latencies_ns && lat.size() < c.latencies_cap) c.latencies_ns[lat.size()] = d.done_ns - d.submit_ns;
      lat.push_back(d.done_ns - d.submit_ns);
      sum_us += (d.done_ns - d.submit_ns) * 1e-3;
      last_done = std::max(last_done, d.done_ns);
      if (!open) due.push({d.done_ns + (uint64_t)(think_ns > 0 ? think(rng) * think_ns : 0.0), (uint32_t)d.tag});
    }
  }
  std::sort(lat.begin(), lat.end());
  r.seconds = (last_done - t_start) * 1e-9;
  r.updates_per_s = r.seconds > 0 ? r.completed / r.seconds : 0.0;
  r.p50_us = pct(lat, 0.50);
  r.p99_us = pct(lat, 0.99);
  r.p999_us = pct(lat, 0.999);
  r.max_us = lat.empty() ? 0.0 : lat.back() * 1e-3;
  r.mean_us = lat.empty() ? 0.0 : sum_us / lat.size();
  r.epochs = in->epochs.load() - e0;
  r.mean_epoch = r.epochs ? (double)(in->applied.load() - a0) / r.epochs : 0.0;
}

}  // namespace

namespace rg {
// The checks rg_server_submit makes, for one request (the network front end
// refuses a bad update before it reaches the log).
int server_check(rg_server *s, const rg_request &r) {
  std::shared_ptr<Instance> in = find(s, r.instance);
  if (!in) {
    set_error("unknown instance");
    return RG_EINVAL;
  }
  return check_request(*in, r);
}
}  // namespace rg

extern "C" {

int rg_server_create(uint64_t hbm_budget_bytes, double target_epoch_ms, uint64_t max_epoch, int per_update,
                     rg_server **out) {
  if (!out || !(target_epoch_ms > 0)) return RG_EINVAL;
  rg_server *s = new (std::nothrow) rg_server();
  if (!s) return RG_ENOMEM_HBM;
  s->budget = hbm_budget_bytes;
  s->target_ms = target_epoch_ms;
  s->max_epoch = std::max<uint64_t>(1, max_epoch);
  s->per_update = per_update ? 1 : 0;
  *out = s;
  return RG_OK;
}

int rg_server_attach(rg_server *s, rg_graph *g, int algo, int directed, uint32_t *instance) {
  if (!s || !g || !instance) return RG_EINVAL;
  if (algo < RG_BFS || algo > RG_WCC) return RG_EINVAL;
  if (g->g.algo != algo) {
    rg::set_error("labels were not built for this algorithm (call rg_build_tree first)");
    return RG_ESTATE;
  }
  auto in = std::make_shared<Instance>();
  in->g = g;
  in->algo = algo;
  in->directed = directed ? 1 : 0;
  in->cap = std::min<uint64_t>(s->max_epoch, 64);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (const auto &p : s->inst)
      if (p && p->g == g) {
        rg::set_error("graph is already attached");
        return RG_ESTATE;
      }
    // size the staging buffers for the largest epoch before admission, so the
    // apply path allocates nothing while instances run
    cudaSetDevice(g->g.device);
    int rc = rg::storage_reserve(g->g, s->per_update ? 1 : s->max_epoch);
    if (rc) return rc;
    in->bytes = g->g.bytes;
    if (s->budget && s->used + in->bytes > s->budget) {
      rg::set_error("HBM budget exceeded");
      return RG_ENOMEM_HBM;
    }
    s->used += in->bytes;
    in->id = (uint32_t)s->inst.size();
    s->inst.push_back(in);
  }
  // No cluster levels while served: the epochs of other instances keep SMs
  // busy, and a level that needs a whole GPC's worth of free SMs at once then
  // waits for them (p99 went from 0.4 to 4 ms in the six-instance mix).
  in->cluster_edges = g->g.cluster_edges;
  g->g.cluster_edges = 0;
  Instance *raw = in.get();
  in->worker = std::thread([s, raw] { worker_main(s, raw); });
  *instance = in->id;
  return RG_OK;
}

int rg_server_history(rg_server *s, uint32_t instance, int enable, uint64_t *version) {
  if (!s) return RG_EINVAL;
  std::shared_ptr<Instance> in = find(s, instance);
  if (!in) {
    rg::set_error("unknown instance");
    return RG_EINVAL;
  }
  if (enable && !in->g->g.hist_nodes) {
    rg::set_error("enable the graph's history (rg_history_enable) first");
    return RG_ESTATE;
  }
  in->history.store(enable ? 1 : 0);
  if (version) *version = in->version;  // the worker's latest recorded version
  return RG_OK;
}

int rg_server_detach(rg_server *s, uint32_t instance) {
  if (!s) return RG_EINVAL;
  std::shared_ptr<Instance> in;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (instance >= s->inst.size() || !s->inst[instance]) return RG_EINVAL;
    in = s->inst[instance];
    s->inst[instance].reset();
  }
  {
    std::lock_guard<std::mutex> lk(in->mu);
    in->stop = true;  // the worker finishes what is queued, then exits
  }
  in->cv.notify_all();
  in->worker.join();
  in->g->g.cluster_edges = in->cluster_edges;
  std::lock_guard<std::mutex> lk(s->mu);
  s->used -= in->bytes;
  return RG_OK;
}

int rg_server_submit(rg_server *s, const rg_request *reqs, uint64_t n) {
  if (!s || (n && !reqs)) return RG_EINVAL;
  std::vector<std::shared_ptr<Instance>> ins(n);
  for (uint64_t i = 0; i < n; i++) {
    if (!(ins[i] = find(s, reqs[i].instance))) {
      rg::set_error("unknown instance");
      return RG_EINVAL;
    }
    int rc = check_request(*ins[i], reqs[i]);
    if (rc) return rc;
  }
  for (uint64_t i = 0; i < n; i++) {
    std::lock_guard<std::mutex> lk(ins[i]->mu);
    if (ins[i]->stop) {
      rg::set_error("instance is being detached");
      return RG_ESTATE;
    }
  }
  {
    std::lock_guard<std::mutex> lk(s->cmu);
    s->submitted += n;
  }
  const uint64_t t = now_ns();
  for (uint64_t i = 0; i < n;) {
    Instance *in = ins[i].get();
    uint64_t j = i;
    {
      std::lock_guard<std::mutex> lk(in->mu);
      for (; j < n && ins[j].get() == in; j++) in->q.push_back(Item{reqs[j], t});
      in->qn.fetch_add(j - i, std::memory_order_release);
    }
    in->cv.notify_one();
    i = j;
  }
  return RG_OK;
}

int rg_server_poll(rg_server *s, rg_completion *out, uint64_t cap, uint64_t *n) {
  if (!s || !n || (cap && !out)) return RG_EINVAL;
  std::lock_guard<std::mutex> lk(s->cmu);
  const uint64_t k = std::min<uint64_t>(cap, s->done.size());
  std::copy(s->done.begin(), s->done.begin() + k, out);
  s->done.erase(s->done.begin(), s->done.begin() + k);
  *n = k;
  return RG_OK;
}

int rg_server_poll_wait(rg_server *s, rg_completion *out, uint64_t cap, uint64_t *n, uint64_t timeout_us) {
  if (!s || !n || (cap && !out)) return RG_EINVAL;
  std::unique_lock<std::mutex> lk(s->cmu);
  s->ccv.wait_for(lk, std::chrono::microseconds(timeout_us), [&] { return !s->done.empty(); });
  const uint64_t k = std::min<uint64_t>(cap, s->done.size());
  std::copy(s->done.begin(), s->done.begin() + k, out);
  s->done.erase(s->done.begin(), s->done.begin() + k);
  *n = k;
  return RG_OK;
}

int rg_server_drain(rg_server *s, uint64_t timeout_ms) {
  if (!s) return RG_EINVAL;
  std::unique_lock<std::mutex> lk(s->cmu);
  bool ok = s->ccv.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return s->completed >= s->submitted; });
  return ok ? RG_OK : RG_ETIMEOUT;
}

int rg_server_stats_get(rg_server *s, rg_server_stats *st, int reset) {
  if (!s || !st) return RG_EINVAL;
  std::lock_guard<std::mutex> lk(s->cmu);
  std::vector<uint64_t> v(s->lat);
  std::sort(v.begin(), v.end());
  double sum = 0;
  for (uint64_t x : v) sum += x * 1e-3;
  st->completed = v.size();
  st->epochs = s->epochs;
  st->largest_epoch = s->largest;
  st->p50_us = pct(v, 0.50);
  st->p99_us = pct(v, 0.99);
  st->p999_us = pct(v, 0.999);
  st->max_us = v.empty() ? 0.0 : v.back() * 1e-3;
  st->mean_us = v.empty() ? 0.0 : sum / v.size();
  if (reset) {
    s->lat.clear();
    s->epochs = 0;
    s->largest = 0;
  }
  return RG_OK;
}

int rg_server_run_load(rg_server *s, const rg_load_config *cfgs, uint64_t n, rg_load_result *results) {
  if (!s || (n && (!cfgs || !results))) return RG_EINVAL;
  std::vector<std::shared_ptr<Instance>> ins(n);
  std::vector<std::unique_ptr<Sink>> sinks(n);
  for (uint64_t i = 0; i < n; i++) {
    if (!(ins[i] = find(s, cfgs[i].instance)) || !cfgs[i].pairs || cfgs[i].imported > cfgs[i].n_pairs) {
      rg::set_error("bad load config");
      return RG_EINVAL;
    }
    const rg::Graph &g = ins[i]->g->g;
    for (uint64_t k = 0; k < 2 * cfgs[i].n_pairs; k++)
      if (cfgs[i].pairs[k] >= g.V) {
        rg::set_error("VertexId error.");
        return RG_EINVAL_VID;
      }
    sinks[i].reset(new Sink());
  }
  int rc = RG_OK;
  uint64_t set = 0;
  for (; set < n; set++) {
    std::lock_guard<std::mutex> lk(ins[set]->mu);
    if (ins[set]->sink) {
      rg::set_error("a load already runs on this instance");
      rc = RG_ESTATE;
      break;
    }
    ins[set]->sink = sinks[set].get();
  }
  if (!rc) {
    std::vector<std::thread> th;
    for (uint64_t i = 0; i < n; i++) {
      results[i] = rg_load_result{};
      th.emplace_back([&, i] { run_load(s, ins[i].get(), cfgs[i], *sinks[i], results[i]); });
    }
    for (auto &t : th) t.join();
  }
  for (uint64_t i = 0; i < set; i++) {
    std::lock_guard<std::mutex> lk(ins[i]->mu);
    ins[i]->sink = nullptr;
  }
  return rc;
}

int rg_server_destroy(rg_server *s) {
  if (!s) return RG_EINVAL;
  std::vector<uint32_t> ids;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (const auto &p : s->inst)
      if (p) ids.push_back(p->id);
  }
  for (uint32_t id : ids) rg_server_detach(s, id);
  delete s;
  return RG_OK;
}

}  // extern "C"
