/*
 * Seeded synthetic graphs generated on the device, for the benchmark shapes
 * that are too large to build on the host (R-MAT scale 25, thousands of
 * batched SBMs).  The reference ships no generator; these exist so that its
 * workloads can be produced straight into HBM.  The generated lists are in
 * the form lvg_load_edges_device and lvg_batch_run_device take.
 */
#ifndef LVG_GEN_H
#define LVG_GEN_H
#include <stdint.h>

#include "lvg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lvg_dgraph lvg_dgraph;   /* generated graph(s), device memory */

/* R-MAT: edge_factor * 2^scale edges with quadrant probabilities
 * (a, b, c, 1-a-b-c), labels not permuted; self loops dropped, duplicate
 * edges merged by summing their weights; integer weights uniform in
 * [w_lo, w_hi]; symmetric list sorted by (src, dst).  The result equals the
 * host generator's (lvggen_rmat) entry for entry.  stream may be NULL. */
lvg_status lvg_gen_rmat(int32_t device, void* stream, int32_t scale, int32_t edge_factor, double a, double b,
                        double c, int32_t w_lo, int32_t w_hi, uint64_t seed, lvg_dgraph** out);

/* n_graphs independent stochastic block models packed into one list: graph g
 * has n[g] vertices in blocks[g] near-equal blocks (block k = vertices
 * floor(n*k/blocks) .. floor(n*(k+1)/blocks)-1); every unordered pair is an
 * edge with probability p_in[g] (same block) or p_out[g]; integer weights
 * uniform in [w_lo, w_hi]; seeds[g] seeds graph g alone, so a graph does not
 * depend on its batch.  Vertex ids are local to each graph; graph g owns
 * entries entry_off[g] .. entry_off[g+1] (lvg_dgraph_offsets), sorted by
 * (src, dst), both directions listed.  The packed list holds at most
 * 2^31 - 1 entries. */
lvg_status lvg_gen_sbm_batch(int32_t device, void* stream, int32_t n_graphs, const int32_t* n,
                             const int32_t* blocks, const double* p_in, const double* p_out, int32_t w_lo,
                             int32_t w_hi, const uint64_t* seeds, lvg_dgraph** out);

/* Sizes: number of graphs, entries, vertices (sum over graphs). */
lvg_status lvg_dgraph_info(const lvg_dgraph* g, int32_t* n_graphs, int64_t* n_entries, int64_t* n_vertices);
/* Device pointers of the packed list (valid until lvg_dgraph_free). */
lvg_status lvg_dgraph_arrays(const lvg_dgraph* g, const int32_t** src, const int32_t** dst, const float** w);
/* Host copies of the offsets: entry_off[n_graphs+1], vertex_off[n_graphs+1]. */
lvg_status lvg_dgraph_offsets(const lvg_dgraph* g, int64_t* entry_off, int32_t* vertex_off);
/* Copy the packed list into host arrays of n_entries elements (each nullable). */
lvg_status lvg_dgraph_copy_to_host(const lvg_dgraph* g, int32_t* src, int32_t* dst, float* w);
void lvg_dgraph_free(lvg_dgraph* g);
/* Message of the last failed generator call on this thread. */
const char* lvg_gen_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
