/* Synthetic evolving-graph inputs in the reference's binary edge-list format.
 *
 * The reference reads its input with mmap_binary (core/io.hpp:26-36): a file of
 * (uint64 src, uint64 dst) pairs in host byte order with no header, and infers
 * |V| = max id + 1 (src/sssp.cpp:40-46).  Its converters (utils/convert_to_binary*.cpp)
 * turn text edge lists into that format.  These entry points generate the
 * benchmark graphs directly in that format:
 *   - RMAT (a,b,c,d probabilities, duplicates and self-loops kept), each edge
 *     drawn from a counter-based stream keyed by (seed, edge index), so the
 *     order of the list is already a seeded random order and the output does
 *     not depend on the thread count;
 *   - an Erdos-Renyi + RMAT mix (even indices uniform endpoints, odd indices RMAT);
 *   - edge weights splitmix64(src<<32|dst) % 255 + 1, a pure function of the
 *     endpoints, so every implementation derives identical weights.
 * Plain C ABI, no device code. */
#ifndef RG_GEN_H
#define RG_GEN_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* splitmix64 finaliser applied to x + 0x9E3779B97F4A7C15 (Steele, Lea, Flood 2014). */
uint64_t rg_gen_splitmix64(uint64_t x);

/* Edge weight in [1,255]: splitmix64(src<<32 | dst) % 255 + 1. */
uint64_t rg_gen_weight(uint64_t src, uint64_t dst);

/* Fill pairs[2*i], pairs[2*i+1] with (src,dst) of RMAT edges first..first+n-1 of
 * the stream (scale bits per endpoint). */
void rg_gen_rmat(uint32_t scale, uint64_t first, uint64_t n, double a, double b, double c,
                 uint64_t seed, uint64_t *pairs);

/* Erdos-Renyi + RMAT mix over 2^scale vertices: edge i is uniform when i is even,
 * RMAT when i is odd. */
void rg_gen_er_rmat_mix(uint32_t scale, uint64_t first, uint64_t n, double a, double b, double c,
                        uint64_t seed, uint64_t *pairs);

/* Weights for n pairs. */
void rg_gen_weights(const uint64_t *pairs, uint64_t n, uint64_t *weights);

/* Vertex with the highest out-degree among the n pairs (duplicates counted),
 * lowest id on ties; vertices must be < nv. */
uint64_t rg_gen_max_out_degree_vertex(const uint64_t *pairs, uint64_t n, uint64_t nv);

/* Write n pairs to path in the reference format. Returns 0 on success. */
int rg_gen_write_binary(const char *path, const uint64_t *pairs, uint64_t n);

/* Checksum of a per-vertex value array: sum over v of splitmix64(val[v] ^ (v * 0x9E3779B97F4A7C15)),
 * wrapping.  Position-dependent and order-independent, so it can be computed in parallel. */
uint64_t rg_gen_value_checksum(const uint64_t *val, uint64_t nv);

#ifdef __cplusplus
}
#endif
#endif
