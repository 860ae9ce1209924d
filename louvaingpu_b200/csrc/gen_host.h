/*
 * Seeded synthetic graph generators (host, C ABI).  Every generator returns a
 * symmetric edge list (both directions of each undirected edge), without self
 * loops, with duplicate edges merged, sorted by (src, dst).
 */
#ifndef LVG_GEN_HOST_H
#define LVG_GEN_HOST_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct lvggen_graph lvggen_graph;

/* Stochastic block model: n vertices in `blocks` near-equal blocks; each
 * unordered pair is an edge with probability p_in (same block) or p_out;
 * integer weights uniform in [w_lo, w_hi]. */
lvggen_graph* lvggen_sbm(int32_t n, int32_t blocks, double p_in, double p_out, int32_t w_lo, int32_t w_hi,
                         uint64_t seed);

/* LFR-style benchmark: power-law degrees (exponent deg_exp on [d_min, d_max]),
 * power-law community sizes (exponent com_exp on [c_min, c_max]), a fraction
 * mu of each vertex's edges leaving its community; configuration-model wiring
 * inside communities and across them; unit weights. */
lvggen_graph* lvggen_lfr(int32_t n, double deg_exp, int32_t d_min, int32_t d_max, double com_exp, int32_t c_min,
                         int32_t c_max, double mu, uint64_t seed);

/* R-MAT: edge_factor * 2^scale generated edges with quadrant probabilities
 * (a, b, c, 1-a-b-c), vertex labels not permuted; self loops dropped,
 * duplicates merged by summing weights; integer weights uniform in [w_lo, w_hi]. */
lvggen_graph* lvggen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, int32_t w_lo,
                          int32_t w_hi, uint64_t seed);

int32_t lvggen_n_vertices(const lvggen_graph* g);
int64_t lvggen_n_entries(const lvggen_graph* g);
void lvggen_copy(const lvggen_graph* g, int32_t* src, int32_t* dst, float* w);
/* Planted community of every vertex (SBM blocks, LFR communities); -1 for R-MAT. */
void lvggen_truth(const lvggen_graph* g, int32_t* membership);
void lvggen_free(lvggen_graph* g);

#ifdef __cplusplus
}
#endif
#endif
