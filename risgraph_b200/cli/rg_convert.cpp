// Text edge list -> the binary edge-list format the drivers read
// ((u64 src, u64 dst) pairs, host order, no header; core/io.hpp:26-36), with
// the names of the reference's converters (utils/convert_to_binary*.cpp):
//
//   convert_to_binary            < "src dst" lines  > graph.bin   (input order)
//   convert_to_binary_random     < "src dst" lines  > graph.bin   (shuffled)
//   convert_to_binary_timestamp  < "src dst t" lines > graph.bin  (sorted by t, then src, dst)
//
// Without RG_SHUFFLE_SEED the shuffle is std::random_shuffle over the
// (src, dst) pairs with the C library's default rand() state, as
// utils/convert_to_binary_random.cpp:28 does, so on the same C++ library the
// output is byte-identical to the reference's.  With RG_SHUFFLE_SEED set it is
// a Fisher-Yates shuffle driven by splitmix64 from that seed, which gives the
// same file on every platform.  Input is read in large blocks; any run of
// characters other than digits separates numbers (scanf("%lu") would also
// take a sign).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "rg_gen.h"

namespace {

// Streams unsigned decimal numbers from stdin.
struct Reader {
  std::vector<char> buf = std::vector<char>(1 << 22);
  size_t pos = 0, len = 0;
  bool eof = false;
  int next_char() {
    if (pos == len) {
      if (eof) return -1;
      len = std::fread(buf.data(), 1, buf.size(), stdin);
      pos = 0;
      if (len == 0) {
        eof = true;
        return -1;
      }
    }
    return (unsigned char)buf[pos++];
  }
  bool next(uint64_t &x) {
    int c = next_char();
    while (c != -1 && (c < '0' || c > '9')) c = next_char();
    if (c == -1) return false;
    x = 0;
    while (c >= '0' && c <= '9') {
      x = x * 10 + (uint64_t)(c - '0');
      c = next_char();
    }
    return true;
  }
};

void write_pairs(const std::vector<uint64_t> &p) {
  if (!p.empty() && std::fwrite(p.data(), 8, p.size(), stdout) != p.size()) {
    std::perror("write");
    std::exit(1);
  }
}

}  // namespace

int main(int argc, char **argv) {
  (void)argc;
  std::string name = argv[0];
  name = name.substr(name.find_last_of('/') + 1);
  const bool random = name == "convert_to_binary_random";
  const bool timestamp = name == "convert_to_binary_timestamp";
  if (!random && !timestamp && name != "convert_to_binary") {
    std::fprintf(stderr, "%s: call as convert_to_binary[_random|_timestamp]\n", name.c_str());
    return 1;
  }
  Reader in;
  if (timestamp) {
    struct E {
      uint64_t t, s, d;
    };
    std::vector<E> e;
    uint64_t s, d, t;
    while (in.next(s) && in.next(d) && in.next(t)) e.push_back({t, s, d});
    std::sort(e.begin(), e.end(), [](const E &a, const E &b) {
      return a.t != b.t ? a.t < b.t : (a.s != b.s ? a.s < b.s : a.d < b.d);
    });
    std::vector<uint64_t> p(2 * e.size());
    for (size_t i = 0; i < e.size(); i++) {
      p[2 * i] = e[i].s;
      p[2 * i + 1] = e[i].d;
    }
    write_pairs(p);
    return 0;
  }
  std::vector<uint64_t> p;
  uint64_t s, d;
  while (in.next(s) && in.next(d)) {
    p.push_back(s);
    p.push_back(d);
  }
  if (random && !std::getenv("RG_SHUFFLE_SEED")) {
    std::vector<std::pair<uint64_t, uint64_t>> e(p.size() / 2);
    for (size_t i = 0; i < e.size(); i++) e[i] = {p[2 * i], p[2 * i + 1]};
    std::random_shuffle(e.begin(), e.end());
    for (size_t i = 0; i < e.size(); i++) {
      p[2 * i] = e[i].first;
      p[2 * i + 1] = e[i].second;
    }
  } else if (random) {
    uint64_t state = std::strtoull(std::getenv("RG_SHUFFLE_SEED"), nullptr, 10);
    const size_t n = p.size() / 2;
    for (size_t i = n; i > 1; i--) {
      state = rg_gen_splitmix64(state);
      const size_t j = (size_t)(state % i);
      std::swap(p[2 * (i - 1)], p[2 * j]);
      std::swap(p[2 * (i - 1) + 1], p[2 * j + 1]);
    }
  }
  write_pairs(p);
  return 0;
}
