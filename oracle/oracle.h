/*
 * oracle.h -- CPU restatement of graph-gpu's serial BFS / PageRank algorithms
 * and of the graph builders they run on.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links or calls
 * this code; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it, and only as the checker.  Parity is pinned: tests compare every
 * function here with the reference's own CPU code compiled from its sources
 * (oracle/_ref, built by oracle/Makefile) and with the committed golden
 * fixtures under tests/golden/ that were produced from that build.
 *
 * Conventions follow the reference: vertex ids and CSR offsets are uint32,
 * an unreached vertex has distance 0xFFFFFFFF (src/cpu/bfs_cpu.hpp:14), and
 * PageRank is double precision with d = 0.85 (src/cpu/pagerank_cpu.hpp:4-8).
 */
#ifndef GRAPH_ORACLE_H
#define GRAPH_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_UNREACHED 0xFFFFFFFFu
#define ORC_FLAG_DIRECTED 1u
#define ORC_FLAG_SORTED 2u
#define ORC_FLAG_DEDUP 4u

/* A CSR owned by the oracle (malloc'd arrays) or a borrowed view. */
typedef struct {
    uint64_t n, m;
    uint32_t flags;
    uint32_t* row_ptr; /* n + 1 */
    uint32_t* col_idx; /* m */
} orc_csr;

/* One BFS level record (src/util/trace.hpp:7-14). */
typedef struct {
    uint32_t level;
    uint32_t direction; /* 'T' or 'B' */
    uint64_t frontier;
    uint64_t edges;
} orc_level;

void orc_csr_free(orc_csr* g);

/* SplitMix64 stream (src/util/rng.hpp:8-26). */
uint64_t orc_rng_next(uint64_t* state);
uint64_t orc_rng_below(uint64_t* state, uint64_t bound);
double orc_rng_uniform(uint64_t* state);

/* Graph builders (src/graph/csr.cpp:112-163, src/graph/generators.cpp). */
orc_csr* orc_from_edge_list(uint64_t n, const uint32_t* eu, const uint32_t* ev, uint64_t ne,
                            int directed);
orc_csr* orc_gen_path(uint32_t n);
orc_csr* orc_gen_star(uint32_t leaves);
orc_csr* orc_gen_complete(uint32_t n);
orc_csr* orc_gen_two_components(void);
orc_csr* orc_gen_empty(uint32_t n);
orc_csr* orc_gen_grid2d(uint32_t rows, uint32_t cols);
orc_csr* orc_gen_rmat(uint32_t scale, uint32_t edgefactor, int directed, uint64_t seed);
/* R-MAT with an explicit generated-edge count (same quadrant draw). */
orc_csr* orc_gen_rmat_edges(uint32_t scale, uint64_t edges, int directed, uint64_t seed);
/* The raw R-MAT endpoint pairs of orc_gen_rmat_edges, before fromEdgeList. */
void orc_rmat_draw(uint32_t scale, uint64_t edges, uint64_t seed, uint32_t* eu, uint32_t* ev);

/* Transforms (src/graph/transform.cpp:9-76) and the random ordering
 * (src/graph/reorder.cpp:20-25). */
orc_csr* orc_transpose(const orc_csr* g);
orc_csr* orc_symmetrize(const orc_csr* g);
orc_csr* orc_permute(const orc_csr* g, const uint32_t* perm);
void orc_random_perm(uint64_t n, uint64_t seed, uint32_t* perm);
/* Orderings on a symmetric graph (src/graph/reorder.cpp:27-99): perm[old] =
 * new; "degree" = descending degree (ties by id), "rcm" = reverse
 * Cuthill-McKee per component.  locality (:111-125). */
void orc_reorder_degree(const orc_csr* g, uint32_t* perm);
void orc_reorder_rcm(const orc_csr* g, uint32_t* perm);
void orc_locality(const orc_csr* g, double* mean_gap, double* same_block64);
/* Structural check (src/graph/csr.cpp:86-104): 0 if valid. */
int orc_validate(const orc_csr* g);

/* BFS (src/cpu/bfs_cpu.cpp:27-45 and :227-283). */
void orc_bfs_serial(const orc_csr* g, uint32_t source, uint32_t* dist);
/* Returns the number of levels (also written to trace when cap allows). */
int orc_bfs_do(const orc_csr* g, uint32_t source, uint32_t* dist, double alpha, double beta,
               orc_level* trace, int cap);

/* Sources like gbench (src/bench/main.cpp:130-169); returns the count. */
int orc_pick_sources(const orc_csr* g, int count, uint64_t seed, int any_component,
                     uint32_t* out);
/* Undirected edges of the component reached in dist (src/bench/main.cpp:329-332). */
uint64_t orc_component_edges(const orc_csr* g, const uint32_t* dist);

/* PageRank (src/cpu/pagerank_cpu.cpp:20-53). in = transpose of the graph. */
void orc_out_degrees(const orc_csr* g, uint32_t* outdeg);
int orc_pagerank_serial(const orc_csr* in, const uint32_t* outdeg, double* r, double damping,
                        int iters, double tol, double* last_delta);
/* checkRanks (src/cpu/pagerank_cpu.hpp:42-60), on float or double results. */
void orc_check_ranks_f32(const double* ref, const float* got, uint64_t n, double* l1,
                         double* max_rel_top, double* sum);
void orc_check_ranks_f64(const double* ref, const double* got, uint64_t n, double* l1,
                         double* max_rel_top, double* sum);
/* gsNoWorseThanJacobi (src/cpu/pagerank_cpu.hpp:80-84). */
int orc_gs_no_worse(double gs_l1, double gs_rel, double gs_sum, double j_l1, double j_rel);

/* SNAP edge list (plain or gzip text) -> CSR (src/graph/snap.cpp:17-149).
 * Lines: blank or whitespace-only lines and lines whose first non-blank byte
 * is '#' or '%' are skipped; otherwise two decimal ids separated by spaces or
 * tabs, anything after the second id ignored.  Ids are relabelled densely in
 * increasing raw-id order; directed = 0 adds both directions; lists sorted,
 * duplicates and self-loops dropped.  Returns 0, or 1 with the reference's
 * error message in msg (the first failing line in file order wins). */
typedef struct {
    uint64_t lines, raw_max_id, n, m_before, m;
} orc_convert_stats;
int orc_convert_snap(const char* path, int directed, orc_csr** out, orc_convert_stats* st,
                     char* msg, size_t cap);

/* Reference two-layer-ReLU MLP (forward, backward of the mean squared error)
 * used to check the GPU selector-training kernels.  Layout: w1[h][f], b1[h],
 * w2[h][h], b2[h], w3[o][h], b3[o]; x[b][f], y[b][o] (targets), mask[b][o]
 * (1 where a target exists).  Returns the loss; grads has the same layout as
 * params. */
double orc_mlp_loss_grad(int nf, int nh, int no, const float* params, int batch, const float* x,
                         const float* y, const float* mask, float* grads);
void orc_mlp_forward(int nf, int nh, int no, const float* params, int batch, const float* x,
                     float* out);

#ifdef __cplusplus
}
#endif
#endif
