// Replays a sequence of operations through the reference's UNMODIFIED MVVec
// (core/mvvec.hpp:23-162), the versioned label history of the _inc_rt drivers
// (src/sssp_inc_rt.cpp:338-343).  Test infrastructure only.
//
// Usage: mvvec_driver <length> <ops.bin> <out.bin>
// ops.bin holds uint64 records of four words (op, a, b, c):
//   op 0: set(id = a, timestamp = b, data = c)
//   op 1: get(id = a, timestamp = b); the result is appended to out.bin
//   op 2: gc(timestamp = a) over every id
// A get must name a timestamp at or after the id's first set (MVVec::get
// asserts otherwise, core/mvvec.hpp:81-82).
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "core/mvvec.hpp"

int main(int argc, char **argv) {
  if (argc != 4) {
    fprintf(stderr, "usage: mvvec_driver <length> <ops.bin> <out.bin>\n");
    return 2;
  }
  const uint64_t length = std::stoull(argv[1]);
  FILE *f = fopen(argv[2], "rb");
  if (!f) { perror(argv[2]); return 3; }
  std::vector<uint64_t> ops;
  uint64_t rec[4];
  while (fread(rec, 8, 4, f) == 4) ops.insert(ops.end(), rec, rec + 4);
  fclose(f);
  MVVec<uint64_t> mv(length);
  std::vector<uint64_t> out;
  for (size_t i = 0; i < ops.size(); i += 4) {
    const uint64_t op = ops[i], a = ops[i + 1], b = ops[i + 2], c = ops[i + 3];
    if ((op == 0 || op == 1) && a >= length) { fprintf(stderr, "id %lu out of range\n", a); return 4; }
    if (op == 0) mv.set(a, b, c);
    else if (op == 1) out.push_back(mv.get(a, b));
    else if (op == 2) mv.gc(a);
    else { fprintf(stderr, "bad op %lu\n", op); return 4; }
  }
  FILE *o = fopen(argv[3], "wb");
  if (!o) { perror(argv[3]); return 3; }
  fwrite(out.data(), 8, out.size(), o);
  fclose(o);
  printf("{\"ops\": %zu, \"gets\": %zu}\n", ops.size() / 4, out.size());
  return 0;
}
