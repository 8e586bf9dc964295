/* Synthetic graph generation in the reference's 16-byte binary edge format
 * (core/io.hpp:26-36).  See include/rg_gen.h for the contract. */
#include "rg_gen.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

uint64_t rg_gen_splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

uint64_t rg_gen_weight(uint64_t src, uint64_t dst) {
  return rg_gen_splitmix64((src << 32) | dst) % 255 + 1;
}

/* Threshold for probability p on the full 64-bit range. */
static uint64_t prob_to_u64(double p) {
  if (p <= 0.0) return 0;
  if (p >= 1.0) return UINT64_MAX;
  return (uint64_t)(p * 18446744073709551616.0);
}

static inline void rmat_edge(uint32_t scale, uint64_t idx, uint64_t ta, uint64_t tab, uint64_t tabc,
                             uint64_t seed, uint64_t *s, uint64_t *d) {
  uint64_t state = rg_gen_splitmix64(seed ^ rg_gen_splitmix64(idx + 0x632BE59BD9B4E019ull));
  uint64_t src = 0, dst = 0;
  for (uint32_t l = 0; l < scale; l++) {
    state += 0x9E3779B97F4A7C15ull;
    uint64_t r = rg_gen_splitmix64(state);
    uint64_t sb, db;
    if (r < ta) { sb = 0; db = 0; }
    else if (r < tab) { sb = 0; db = 1; }
    else if (r < tabc) { sb = 1; db = 0; }
    else { sb = 1; db = 1; }
    src = (src << 1) | sb;
    dst = (dst << 1) | db;
  }
  *s = src;
  *d = dst;
}

void rg_gen_rmat(uint32_t scale, uint64_t first, uint64_t n, double a, double b, double c,
                 uint64_t seed, uint64_t *pairs) {
  uint64_t ta = prob_to_u64(a), tab = prob_to_u64(a + b), tabc = prob_to_u64(a + b + c);
#pragma omp parallel for schedule(static)
  for (uint64_t i = 0; i < n; i++) {
    rmat_edge(scale, first + i, ta, tab, tabc, seed, &pairs[2 * i], &pairs[2 * i + 1]);
  }
}

void rg_gen_er_rmat_mix(uint32_t scale, uint64_t first, uint64_t n, double a, double b, double c,
                        uint64_t seed, uint64_t *pairs) {
  uint64_t ta = prob_to_u64(a), tab = prob_to_u64(a + b), tabc = prob_to_u64(a + b + c);
  uint64_t mask = (scale >= 64) ? UINT64_MAX : ((1ull << scale) - 1);
#pragma omp parallel for schedule(static)
  for (uint64_t i = 0; i < n; i++) {
    uint64_t idx = first + i;
    if ((idx & 1) == 0) {
      uint64_t h = rg_gen_splitmix64(seed ^ rg_gen_splitmix64(idx ^ 0xD1B54A32D192ED03ull));
      pairs[2 * i] = h & mask;
      pairs[2 * i + 1] = rg_gen_splitmix64(h) & mask;
    } else {
      rmat_edge(scale, idx, ta, tab, tabc, seed, &pairs[2 * i], &pairs[2 * i + 1]);
    }
  }
}

void rg_gen_weights(const uint64_t *pairs, uint64_t n, uint64_t *weights) {
#pragma omp parallel for schedule(static)
  for (uint64_t i = 0; i < n; i++) weights[i] = rg_gen_weight(pairs[2 * i], pairs[2 * i + 1]);
}

uint64_t rg_gen_max_out_degree_vertex(const uint64_t *pairs, uint64_t n, uint64_t nv) {
  uint64_t *deg = (uint64_t *)calloc(nv ? nv : 1, sizeof(uint64_t));
  if (!deg) return 0;
  for (uint64_t i = 0; i < n; i++) {
    uint64_t s = pairs[2 * i];
    if (s < nv) deg[s]++;
  }
  uint64_t best = 0;
  for (uint64_t v = 1; v < nv; v++)
    if (deg[v] > deg[best]) best = v;
  free(deg);
  return best;
}

int rg_gen_write_binary(const char *path, const uint64_t *pairs, uint64_t n) {
  FILE *f = fopen(path, "wb");
  if (!f) return -1;
  uint64_t done = 0;
  while (done < n) {
    uint64_t chunk = n - done > (1ull << 24) ? (1ull << 24) : n - done;
    if (fwrite(pairs + 2 * done, 16, chunk, f) != chunk) { fclose(f); return -2; }
    done += chunk;
  }
  return fclose(f) == 0 ? 0 : -3;
}

uint64_t rg_gen_value_checksum(const uint64_t *val, uint64_t nv) {
  uint64_t h = 0;
#pragma omp parallel for reduction(+ : h) schedule(static)
  for (uint64_t v = 0; v < nv; v++) h += rg_gen_splitmix64(val[v] ^ (v * 0x9E3779B97F4A7C15ull));
  return h;
}
