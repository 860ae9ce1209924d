/*
 * CPU oracle for the Louvain hot path of LouvainGPU -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain C++ restatement of the reference's method, used as the
 * checker by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline
 * leg.  Nothing in the product (louvaingpu_b200/) links, loads or calls it.
 *
 * PARITY UNPINNED: the reference cannot be compiled or run here (CUDPP 2.3 and
 * Boost.Python are absent, its Thrust calls do not compile against CUDA 12.9,
 * and it uses the pre-Volta __shfl_down that sm_100a lacks), and it ships no
 * test, golden vector or fixture.  The oracle is pinned instead by
 * hand-derived known answers (tests/golden/) and by networkx modularity.
 *
 * Two arithmetic modes:
 *   ORC_FP64  -- community totals, degrees, gains and Q in FP64 (the method the
 *                GPU path implements, bit-exact for integer-valued weights);
 *   ORC_REF32 -- the reference's own types: int community totals with
 *                float->int truncation, float degrees, gains and Q
 *                (StatusCUDA.h:27-41, OneLevelKernel.cu:52-78,307-315,427-451).
 */
#ifndef LVG_ORACLE_H
#define LVG_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_FP64 = 0, ORC_REF32 = 1 };

typedef struct orc_csr orc_csr;   /* opaque: CSR of one level */
typedef struct orc_run orc_run;   /* opaque: a full dendrogram run */

/* Build the level CSR from a level input list (NeighbourCompute.cu:42-117,
 * InitKernel.cu:154-243).  Returns NULL on bad input. */
orc_csr* orc_csr_build(int32_t n_vertices, int64_t n_entries, const int32_t* src,
                       const int32_t* dst, const float* w);
void     orc_csr_free(orc_csr*);
int64_t  orc_csr_nnz(const orc_csr*);
double   orc_csr_m(const orc_csr*);
/* Copy out: off[V+1], col[nnz], w[nnz], k[V], loopw[V], has_loop[V]. Any may be NULL. */
void     orc_csr_get(const orc_csr*, int64_t* off, int32_t* col, float* w, double* k,
                     float* loopw, uint8_t* has_loop);

/* One synchronous decision pass of the move phase (OneLevelKernel.cu:248-422)
 * from the committed state (comm, tot, size).  Outputs per vertex: the chosen
 * community after the singleton-pair rule, the isolated-merge candidate (-1 if
 * none), and the number of distinct neighbour communities. */
void orc_move_decide(const orc_csr*, const int32_t* comm, const double* tot,
                     const int32_t* size, int32_t* next, int32_t* cand, int32_t* nseg,
                     int n_threads);

/* orc_move_decide restricted to the n_verts vertices listed in verts (a
 * bounded sample of one pass); outputs are written at those positions.
 * Returns the seconds the decisions took (scratch set-up excluded). */
double orc_move_decide_subset(const orc_csr*, const int32_t* comm, const double* tot,
                            const int32_t* size, const int32_t* verts, int64_t n_verts,
                            int32_t* next, int32_t* cand, int32_t* nseg, int n_threads);

/* Deterministic fixed-tree FP64 sum used for Q on both sides. */
double orc_tree_sum(const double* x, int64_t n);

/* Q of the committed totals: sum_c in_c/m - (tot_c/2m)^2 (OneLevelKernel.cu:427-451). */
double orc_q_totals(const double* tot, const double* in, int32_t n, double m);

/* Renumber by smallest member index (RenumberKernel.cu:63-221).
 * newid[i] = new community of vertex i; returns the community count. */
int32_t orc_renumber(int32_t n_vertices, const int32_t* comm, int32_t* newid);

/* Coarsen a level input list under part[] (InducedGraphKernel.cu:28-113).
 * Two calls: with out_* NULL returns the output count; then fills the outputs. */
int64_t orc_induce(int32_t n_vertices, int64_t n_entries, const int32_t* src,
                   const int32_t* dst, const float* w, const int32_t* part,
                   int32_t* out_src, int32_t* out_dst, float* out_w);

/* Full run (LouvainCPP.cpp:209-553).  max_passes/max_levels < 0: unbounded. */
typedef struct {
  int32_t mode;            /* ORC_FP64 or ORC_REF32 */
  int32_t n_threads;       /* OpenMP threads, <= 0 for all */
  double pass_min_gain;    /* __MIN = 1e-7 (OneLevelKernel.cu:425) */
  double level_min_gain;   /* 1e-7 (LouvainCPP.cpp:55,466) */
  int32_t max_passes;
  int32_t max_levels;
} orc_config;

orc_run* orc_run_louvain(int32_t n_vertices, int64_t n_entries, const int32_t* src,
                         const int32_t* dst, const float* w, const orc_config* cfg);
void     orc_run_free(orc_run*);
int32_t  orc_run_status(const orc_run*);      /* 0 ok, 4 not converged */
int32_t  orc_run_levels(const orc_run*);
/* Per-level facts: vertices, input entries, CSR entries, communities, passes,
 * Q at level start, returned Q of the one-level phase. */
void     orc_run_level_info(const orc_run*, int32_t level, int32_t* n_vertices,
                            int64_t* n_entries, int64_t* nnz, int32_t* n_comms,
                            int32_t* passes, double* q_start, double* q_level);
/* part[n_vertices of that level] = renumbered community of each level vertex. */
void     orc_run_level_partition(const orc_run*, int32_t level, int32_t* part);
/* labels before renumbering (community ids as vertex indices of that level). */
void     orc_run_level_labels(const orc_run*, int32_t level, int32_t* labels);
/* per-pass Q trace of a level (the value tested against pass_min_gain). */
int32_t  orc_run_level_qtrace(const orc_run*, int32_t level, double* q, int32_t cap);
/* Composed partition of the level-0 vertices after levels 0..level. */
void     orc_run_partition(const orc_run*, int32_t level, int32_t* part);
double   orc_run_seconds(const orc_run*);
int64_t  orc_run_pass_entries(const orc_run*);  /* sum over levels of nnz * passes */

/* Newman modularity in FP64 of a partition over the doubled input list. */
double orc_modularity_fp64(int32_t n_vertices, int64_t n_entries, const int32_t* src,
                           const int32_t* dst, const float* w, const int32_t* part);

#ifdef __cplusplus
}
#endif
#endif
