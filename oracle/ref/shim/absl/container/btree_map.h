// Declarations only: the reference's core/storage.hpp:28-81,216-277 names these
// abseil templates in alternative edge indexes that Graph never instantiates
// (Graph uses storage::index::DenseHashMap, core/graph.hpp:47).  Test
// infrastructure only; ordered std containers stand in where a type is needed.
#pragma once
#include <functional>
#include <map>
#include <memory>
#include <utility>

namespace absl {
namespace container_internal {
template <typename Key, typename Value, typename Compare, typename Alloc, int TargetNodeSize, bool Multi>
struct map_params {};
template <typename Params>
class btree {};
template <typename Tree>
class btree_map_container {};
}  // namespace container_internal

template <typename Key, typename Value, typename Compare = std::less<Key>,
          typename Alloc = std::allocator<std::pair<const Key, Value>>>
using btree_map = std::map<Key, Value, Compare, Alloc>;
}  // namespace absl
