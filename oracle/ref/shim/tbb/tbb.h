// OpenMP-backed stand-in for the handful of TBB names that the reference's
// core/graph.hpp, core/actset.hpp, core/mmapalloc.hpp and src/*_inc_rt.cpp use.
// Test infrastructure only: it lets the reference's own hot path compile here so
// that it can serve as the parity oracle and the CPU baseline.  Written from the
// published TBB interface (names and call shapes), not from TBB sources.
//
// Names provided (uses in the reference):
//   task_scheduler_init            core/graph.hpp:85
//   blocked_range<T>               core/graph.hpp:414,468,528; core/actset.hpp:168
//   affinity_partitioner           core/graph.hpp:1736
//   parallel_reduce(range, identity, body, join[, partitioner])  core/graph.hpp:414,468,528
//   parallel_for(range, body)      core/actset.hpp:168
//   enumerable_thread_specific<T>  core/graph.hpp:526,1737; core/actset.hpp:166;
//                                  core/mmapalloc.hpp:160; src/*_inc_rt.cpp:152-156
//   parallel_sort(begin, end[, cmp])  src/*_inc_rt.cpp:424; src/*_inc_clf.cpp:158
#pragma once
#include <omp.h>
#include <algorithm>
#include <cstdint>
#include <functional>
#include <list>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>

namespace tbb {

class task_scheduler_init {
 public:
  explicit task_scheduler_init(int = -1) {}
};

class affinity_partitioner {};
class auto_partitioner {};
class simple_partitioner {};

template <typename T>
class blocked_range {
 public:
  using const_iterator = T;
  blocked_range() : b_(), e_(), g_(1) {}
  blocked_range(T b, T e, size_t grain = 1) : b_(b), e_(e), g_(grain ? grain : 1) {}
  T begin() const { return b_; }
  T end() const { return e_; }
  size_t grainsize() const { return g_; }
  size_t size() const { return (size_t)(e_ - b_); }
  bool empty() const { return !(b_ < e_); }

 private:
  T b_, e_;
  size_t g_;
};

namespace shim_detail {
// Number of grain-sized chunks of a range.
template <typename T>
inline uint64_t chunks(const blocked_range<T> &r) {
  uint64_t n = (uint64_t)(r.end() - r.begin());
  return (n + r.grainsize() - 1) / r.grainsize();
}
template <typename T>
inline blocked_range<T> chunk(const blocked_range<T> &r, uint64_t c) {
  T b = r.begin() + (T)(c * r.grainsize());
  T e = b + (T)r.grainsize();
  if (e > r.end() || e < b) e = r.end();
  return blocked_range<T>(b, e, r.grainsize());
}
}  // namespace shim_detail

// Functional parallel_reduce: body(subrange, acc) returns acc folded over the
// subrange; join combines per-thread partials.
template <typename Range, typename Value, typename Body, typename Join>
Value parallel_reduce(const Range &range, const Value &identity, const Body &body, const Join &join) {
  uint64_t n = shim_detail::chunks(range);
  if (n == 0) return identity;
  int nt = omp_in_parallel() ? 1 : omp_get_max_threads();
  std::vector<Value> part(nt, identity);
  std::vector<char> used(nt, 0);
#pragma omp parallel num_threads(nt)
  {
    int t = omp_get_thread_num();
    Value acc = identity;
    bool any = false;
#pragma omp for schedule(dynamic, 1)
    for (uint64_t c = 0; c < n; c++) {
      acc = body(shim_detail::chunk(range, c), acc);
      any = true;
    }
    part[t] = acc;
    used[t] = any;
  }
  Value res = identity;
  bool first = true;
  for (int t = 0; t < nt; t++) {
    if (!used[t]) continue;
    res = first ? part[t] : join(res, part[t]);
    first = false;
  }
  return res;
}

template <typename Range, typename Value, typename Body, typename Join, typename Part>
Value parallel_reduce(const Range &range, const Value &identity, const Body &body, const Join &join, Part &) {
  return parallel_reduce(range, identity, body, join);
}

template <typename Range, typename Body>
void parallel_for(const Range &range, const Body &body) {
  uint64_t n = shim_detail::chunks(range);
  if (n == 0) return;
  int nt = omp_in_parallel() ? 1 : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (uint64_t c = 0; c < n; c++) body(shim_detail::chunk(range, c));
}

template <typename Range, typename Body, typename Part>
void parallel_for(const Range &range, const Body &body, Part &) {
  parallel_for(range, body);
}

// One T per calling OS thread, created on first local() from a factory.
template <typename T>
class enumerable_thread_specific {
 public:
  enumerable_thread_specific() : make_([] { return std::make_unique<T>(); }) {}
  template <typename A0, typename... An>
  explicit enumerable_thread_specific(A0 &&a0, An &&...an) {
    auto args = std::make_shared<std::tuple<std::decay_t<A0>, std::decay_t<An>...>>(
        std::forward<A0>(a0), std::forward<An>(an)...);
    make_ = [args] {
      return std::apply([](auto &...xs) { return std::make_unique<T>(xs...); }, *args);
    };
  }
  enumerable_thread_specific(const enumerable_thread_specific &) = delete;
  enumerable_thread_specific &operator=(const enumerable_thread_specific &) = delete;

  T &local() {
    std::lock_guard<std::mutex> g(mu_);
    auto id = std::this_thread::get_id();
    auto it = idx_.find(id);
    if (it != idx_.end()) return *it->second;
    items_.push_back(make_());
    T *p = items_.back().get();
    idx_.emplace(id, p);
    return *p;
  }

  struct iterator {
    typename std::list<std::unique_ptr<T>>::iterator it;
    T &operator*() const { return **it; }
    T *operator->() const { return it->get(); }
    iterator &operator++() { ++it; return *this; }
    bool operator!=(const iterator &o) const { return it != o.it; }
    bool operator==(const iterator &o) const { return it == o.it; }
  };
  iterator begin() { return iterator{items_.begin()}; }
  iterator end() { return iterator{items_.end()}; }
  size_t size() const { return items_.size(); }
  void clear() { std::lock_guard<std::mutex> g(mu_); items_.clear(); idx_.clear(); }

 private:
  std::function<std::unique_ptr<T>()> make_;
  std::mutex mu_;
  std::list<std::unique_ptr<T>> items_;
  std::unordered_map<std::thread::id, T *> idx_;
};

template <typename It>
void parallel_sort(It b, It e) { std::sort(b, e); }
template <typename It, typename Cmp>
void parallel_sort(It b, It e, const Cmp &cmp) { std::sort(b, e, cmp); }

}  // namespace tbb
