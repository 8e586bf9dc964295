// Declaration stand-in for an abseil name used only by an unused index
// adaptor of the reference (core/storage.hpp:265-278).  Test infrastructure only.
#pragma once
#include <functional>
#include <memory>
#include <unordered_map>
#include <utility>

namespace absl {
template <typename Key, typename Value, typename Hash = std::hash<Key>, typename Eq = std::equal_to<Key>,
          typename Alloc = std::allocator<std::pair<const Key, Value>>>
using node_hash_map = std::unordered_map<Key, Value, Hash, Eq, Alloc>;
}  // namespace absl
