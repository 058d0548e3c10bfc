/*
 * graph_b200.h -- C ABI of the B200 (sm_100a) BFS / PageRank library.
 *
 * This is the drop-in boundary for graph-gpu's GPU hot paths.  Each entry point
 * names the reference interface it replaces (paths inside the reference
 * project).  Plain pointers and sizes only; no exceptions cross the ABI:
 * every function returns a gb_status and gb_last_error() holds the message of
 * the calling thread's last failure.
 *
 * Threading: a handle owns one CUDA stream and its device buffers; it is not
 * thread-safe (as the reference's single encoder, src/metal/primitives.hpp:1-12).
 * All work is asynchronous on that stream and synchronised before return.
 * Graphs: CSR with uint32 offsets/ids (src/graph/csr.hpp:29-45), m < 2^32.
 */
#ifndef GRAPH_B200_H
#define GRAPH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GB_UNREACHED 0xFFFFFFFFu /* cpu::kUnreached, src/cpu/bfs_cpu.hpp:14 */

typedef enum {
    GB_OK = 0,
    GB_ERR_ARG = 1,         /* invalid argument: std::runtime_error in the reference */
    GB_ERR_CUDA = 2,        /* CUDA runtime / kernel failure (reference: exit(1)) */
    GB_ERR_OOM = 3,         /* device allocation failed */
    GB_ERR_TIMEOUT = 4,     /* a bounded device wait (grid barrier) gave up */
    GB_ERR_STATE = 5,       /* call out of order (e.g. ranks before run) */
    GB_ERR_IO = 6,          /* .bin read/write failure */
    GB_ERR_CAPACITY = 7     /* output buffer too small */
} gb_status;

const char* gb_last_error(void);
/* The device the library will use (name, SM count, compute capability);
 * also creates its CUDA context, so that later calls do not pay for it. */
int gb_device_info(char* name, size_t cap, int* sm_count, int* cc_major, int* cc_minor);

/* ------------------------------------------------------------ host graphs */

#define GB_FLAG_DIRECTED 1u /* graph::kFlagDirected, src/graph/csr.hpp:14-18 */
#define GB_FLAG_SORTED 2u
#define GB_FLAG_DEDUP 4u

/* A host CSR whose arrays the library allocated; release with gb_csr_free. */
typedef struct {
    uint64_t n, m;
    uint32_t flags;
    uint32_t* row_ptr; /* n + 1 */
    uint32_t* col_idx; /* m */
} gb_csr;

void gb_csr_free(gb_csr* g);
/* graph::load / graph::save, "GGPUCSR1" format (src/graph/csr.cpp:30-84). */
int gb_csr_load(const char* path, gb_csr* out);
int gb_csr_save(const gb_csr* g, const char* path);
/* graph::load for a discrete GPU (src/graph/csr.cpp:54-84 maps the file and
 * lets the GPU read it in place; here it has to cross PCIe): the same checks
 * and result as gb_csr_load, with both arrays in page-locked host memory read
 * by several threads, so every later upload runs at full PCIe speed.
 * gb_csr_free releases them. */
int gb_csr_load_pinned(const char* path, gb_csr* out);
/* graph::validate (src/graph/csr.cpp:86-104); msg gets "" when valid. */
int gb_csr_validate(const gb_csr* g, char* msg, size_t cap);
/* graph::fromEdgeList (src/graph/csr.cpp:146-163). */
int gb_csr_from_edges(uint64_t n, const uint32_t* eu, const uint32_t* ev, uint64_t ne, int directed,
                      gb_csr* out);
/* graph::transpose / symmetrize / permute (src/graph/transform.cpp:9-76). */
int gb_csr_transpose(const gb_csr* g, gb_csr* out);
int gb_csr_symmetrize(const gb_csr* g, gb_csr* out);
int gb_csr_permute(const gb_csr* g, const uint32_t* perm, gb_csr* out);
/* The same four operations on the GPU (host arrays in and out, results
 * identical to the functions above): one 64-bit (row, column) key per output
 * entry, a radix sort, then the duplicate / self-loop rule of each operation.
 * fromEdgeList (src/graph/csr.cpp:146-163), transpose, symmetrize and permute
 * (src/graph/transform.cpp:9-76).  gb_csr_symmetrize_gpu needs a
 * duplicate-free directed input (flag bit 2), as every generator and
 * fromEdgeList produce; undirected inputs come back unchanged.  Inputs are
 * checked on the device before use (ids below n, row_ptr from 0 to m, perm a
 * permutation). */
int gb_csr_from_edges_gpu(uint64_t n, const uint32_t* eu, const uint32_t* ev, uint64_t ne, int directed,
                          gb_csr* out);
int gb_csr_transpose_gpu(const gb_csr* g, gb_csr* out);
int gb_csr_symmetrize_gpu(const gb_csr* g, gb_csr* out);
int gb_csr_permute_gpu(const gb_csr* g, const uint32_t* perm, gb_csr* out);
/* gb_pick_sources with the largest connected component found on the GPU
 * (largestComponent, src/bench/main.cpp:130-149: hooking + pointer jumping,
 * components rooted at their smallest vertex, the first of the largest kept);
 * same sources as gb_pick_sources.  Symmetric graphs only. */
int gb_pick_sources_gpu(const gb_csr* g, int count, uint64_t seed, int any_component, uint32_t* out,
                        int* k);
/* SNAP edge list (plain text or gzip) -> CSR, parsed and compacted on the
 * GPU: graph::convertSnap (src/graph/snap.cpp:85-149, ConvertStats in
 * src/graph/snap.hpp:9-16) with the line rules of forEachEdge (:17-81):
 * '#' / '%' comment lines, blank lines, ' ' / '\t' separators, '\r' before a
 * line's text, extra columns ignored; ids relabelled densely in increasing
 * raw-id order; undirected (directed = 0) adds both directions; lists sorted,
 * duplicates and self-loops dropped; flags Sorted | Dedup (| Directed).
 * Errors (GB_ERR_ARG, the reference's messages): "<path>: malformed line N",
 * "<path>: vertex ID too large on line N", "line longer than 4 MB in <path>"
 * (first failing line in file order), "too many edges for uint32 offsets";
 * GB_ERR_IO: "cannot open <path>", "gzread failed on <path>".
 * chunk_bytes: text bytes per device chunk (0 = 64 MiB; at least 4 MiB + 1). */
typedef struct {
    uint64_t lines;      /* edge lines parsed */
    uint64_t raw_max_id; /* largest raw id (0 when there are no edges) */
    uint64_t n;          /* vertices after relabelling */
    uint64_t m_before;   /* entries before duplicate / self-loop removal */
    uint64_t m;          /* entries of the result */
    double seconds;
} gb_convert_stats;
int gb_csr_from_snap_gpu(const char* path, int directed, uint64_t chunk_bytes, gb_csr* out,
                         gb_convert_stats* stats);
/* The converter of gconvert (src/graph/convert.cpp:11-45): text -> .bin. */
int gb_convert_snap_gpu(const char* in_path, const char* out_path, int directed,
                        gb_convert_stats* stats);
/* reorder::compute(..., "random", seed) (src/graph/reorder.cpp:20-25). */
int gb_random_perm(uint64_t n, uint64_t seed, uint32_t* perm);
/* reorder::compute(sym, ordering, seed) (src/graph/reorder.cpp:94-100) on a
 * symmetric graph: perm[old] = new for "original", "random" (seed),
 * "degree" (descending degree, ties by id, :27-38) or "rcm" (reverse
 * Cuthill-McKee per component, :40-92).  gb_reorder runs on the host,
 * gb_reorder_gpu computes "degree" and "rcm" on the GPU (same permutation;
 * "original" and "random" stay on the host).  Unknown names: GB_ERR_ARG. */
int gb_reorder(const gb_csr* sym, const char* ordering, uint64_t seed, uint32_t* perm);
int gb_reorder_gpu(const gb_csr* sym, const char* ordering, uint64_t seed, uint32_t* perm);
/* reorder::locality (src/graph/reorder.cpp:111-125): mean |u - v| over the
 * stored entries and the fraction with u / 64 == v / 64. */
int gb_locality(const gb_csr* g, double* mean_gap, double* same_block64);
/* The hub-first adjacency layout of gb_bfs_hub_first applied to a host CSR on
 * the GPU: every list sorted by descending neighbour degree, ties by id
 * (docs/REPORT.md:743-744).  out->flags drops GB_FLAG_SORTED. */
int gb_csr_hub_first_gpu(const gb_csr* g, gb_csr* out);

/* Generators: src/graph/generators.cpp:8-75 (same graphs, byte for byte). */
int gb_gen_path(uint32_t n, gb_csr* out);
int gb_gen_star(uint32_t leaves, gb_csr* out);
int gb_gen_complete(uint32_t n, gb_csr* out);
int gb_gen_two_components(gb_csr* out);
int gb_gen_empty(uint32_t n, gb_csr* out);
int gb_gen_grid2d(uint32_t rows, uint32_t cols, gb_csr* out);
int gb_gen_rmat(uint32_t scale, uint64_t edges, int directed, uint64_t seed, gb_csr* out);
/* Benchmark-shaped graphs without a reference counterpart (new generators):
 * road: rows x cols grid, drop_frac of edges removed, diag_frac * n random
 *       (+-1, +-1) links, max degree <= 8;
 * web:  directed, geometric out-degree (mean out_mean), targets by Zipf rank
 *       popularity (in-degree exponent s), ids permuted;
 * chung_lu: undirected, weights ~ (i + i0)^(-1/(gamma-1)), mean degree mean_deg,
 *       w_max capped at sqrt(sum w), ids permuted. */
int gb_gen_road(uint32_t rows, uint32_t cols, double drop_frac, double diag_frac, uint64_t seed,
                gb_csr* out);
int gb_gen_web(uint32_t n, double out_mean, double zipf_s, uint64_t seed, gb_csr* out);
int gb_gen_chung_lu(uint32_t n, double gamma, double mean_deg, uint64_t seed, gb_csr* out);
/* gbench's pickSources (src/bench/main.cpp:130-169); returns count via *k. */
int gb_pick_sources(const gb_csr* g, int count, uint64_t seed, int any_component, uint32_t* out,
                    int* k);

/* -------------------------------------------------------------------- BFS */

/* Variants: the gbench names of src/bench/main.cpp:79-81 plus new ones. */
typedef enum {
    GB_BFS_VERTEX = 0,     /* gpu_vertex: GpuBfs::runVertex, src/metal/bfs_gpu.mm:115 */
    GB_BFS_NAIVE = 1,      /* gpu_naive:  runNaive,  bfs_gpu.mm:141 */
    GB_BFS_BINNED = 2,     /* gpu_binned: runBinned, bfs_gpu.mm:177-236 */
    GB_BFS_EDGE = 3,       /* gpu_edge:   runEdge,   bfs_gpu.mm:277-305 */
    GB_BFS_DO = 4,         /* gpu_do:     runDO (host loop, one sync per level), bfs_gpu.mm:326-429 */
    GB_BFS_PERSISTENT = 5, /* gpu_do_persistent: every level in one cooperative launch;
                              also what `hybrid` (bfs_gpu.mm:307-325) maps to */
    GB_BFS_BATCH = 6       /* the 64-source batched kernel (gb_bfs_run_batch; gb_bfs_run_many;
                              autotune) */
} gb_bfs_variant;

typedef enum { GB_SELECT_RULE = 0, GB_SELECT_LEARNED = 1 } gb_selector;

/* Strategies a persistent-kernel level can run (the learned selector's classes). */
typedef enum {
    GB_STRAT_TD_EPT1 = 0, /* top-down, CTA-tiled edge-balanced expansion, 1 edge/thread/round */
    GB_STRAT_TD_EPT2 = 1,
    GB_STRAT_TD_EPT4 = 2,
    GB_STRAT_TD_WARP = 3, /* top-down, warp per frontier vertex (degree-binned form) */
    GB_STRAT_BU = 4,      /* bottom-up over the frontier bitmap */
    GB_NUM_STRATS = 5
} gb_strategy;

/* GpuBfsOptions (src/metal/bfs_gpu.hpp:23-33) plus the new fields. */
typedef struct {
    uint32_t tg;         /* threads per block of the level kernels (multiple of 32, 32..1024) */
    uint32_t small_max;  /* gpu_binned: degree <  small_max -> thread-cooperative */
    uint32_t large_min;  /* gpu_binned: degree >= large_min -> block per vertex */
    uint32_t ept;        /* gpu_edge / gpu_do top-down: edges per thread */
    double alpha, beta;  /* direction rule (cpu::bfsDO, src/cpu/bfs_cpu.cpp:227-283) */
    uint32_t selector;   /* gb_selector, persistent variant only */
    int32_t force_strategy; /* >= 0: persistent kernel runs every level with it (profiling) */
    uint32_t hub_min;    /* persistent: degree at which a vertex is split across blocks */
    uint32_t block;      /* persistent / batched: threads per block (256 or 512) */
    uint64_t spin_limit; /* grid-barrier wait bound in polls (0 = default, ~ seconds) */
    uint32_t grid_blocks; /* persistent / batched: blocks in the grid (0 = every resident block) */
    float sel_margin;    /* learned selector: it departs from the alpha/beta rule's direction only
                            when it predicts the other direction faster by this much (log2 of
                            the time ratio); its top-down strategy choice is free.  0 = pure
                            argmin.  A direction change costs work the per-level predictions do
                            not see (a bottom-up to top-down switch rebuilds the queue). */
    uint32_t in_flight;  /* gb_bfs_run_many, persistent variant: traversals run at once (1..16; 0 = 1),
                            each a cooperative grid of grid_blocks (0 = every resident block /
                            in_flight) with its own state and stream.  A traversal's levels are
                            bound by dependent loads and the grid barrier, so two or more of
                            them on a share of the SMs each overlap those waits. */
} gb_bfs_options;

void gb_bfs_default_options(gb_bfs_options* o);

/* util::BfsLevel (src/util/trace.hpp:7-14) plus the strategy that ran. */
typedef struct {
    uint32_t level;
    char direction; /* 'T' or 'B' */
    char device;    /* always 'G' */
    uint8_t strategy;
    uint8_t pad;
    uint64_t frontier;
    uint64_t edges;
    double time_ms;
} gb_level;

typedef struct gb_bfs gb_bfs;

/* GpuBfs(ctx, g) (src/metal/bfs_gpu.hpp:37): one upload of a symmetric CSR. */
int gb_bfs_create(const uint32_t* row_ptr, const uint32_t* col_idx, uint64_t n, uint64_t m,
                  gb_bfs** out);
int gb_bfs_destroy(gb_bfs* h);
/* GpuBfs from a symmetric .bin file (graph::load + GpuBfs(ctx, g),
 * src/graph/csr.cpp:54-84, src/metal/bfs_gpu.hpp:37): the adjacency streams
 * from the file into the handle's device memory through two pinned staging
 * buffers, read and copy overlapped, with no host copy of the whole graph.
 * A directed file is rejected (GB_ERR_ARG): BFS runs on the symmetric graph.
 * n_out / m_out (may be null) receive the graph's sizes. */
int gb_bfs_create_from_file(const char* path, gb_bfs** out, uint64_t* n_out, uint64_t* m_out);
/* GpuBfs::run* (src/metal/bfs_gpu.hpp:43-66).  out_host: n entries written on
 * return, or NULL to leave the result in device memory (gb_bfs_device_dist).
 * trace: optional per-level records (cap entries, *nlev = levels run). */
int gb_bfs_run(gb_bfs* h, int variant, uint32_t source, uint32_t* out_host,
               const gb_bfs_options* opt, gb_level* trace, size_t cap, size_t* nlev);
/* The per-source loop of gbench (src/bench/main.cpp:324-364: one run per
 * source, each timed) as one call.  For GB_BFS_PERSISTENT the traversals
 * follow one another on the handle's stream with no host round trip between
 * them; with out_host, the depths of traversal i are packed on the device,
 * copied to the host on a second stream and widened there while the next
 * traversals run.  Other variants run the sources one by one as gb_bfs_run.
 * out_host: source i writes n entries at out_host + i * stride (stride 0:
 * every source writes the same n entries, which end with the last source's
 * depths; else stride >= n), or NULL (the last source's depths stay on the
 * device, gb_bfs_device_dist, whose pointer may change with this call).
 * gpu_ms, levels (each may be NULL): count entries, device time and level
 * count of each traversal.  Every source is checked before any runs.
 * For GB_BFS_BATCH the sources run 64 to a launch of the batched kernel and
 * each row is then packed, copied and widened as above; gpu_ms[i] is the
 * launch's device time shared evenly over its sources and levels[i] the
 * launch's level count. */
int gb_bfs_run_many(gb_bfs* h, int variant, const uint32_t* sources, uint32_t count, uint32_t* out_host,
                    uint64_t stride, const gb_bfs_options* opt, float* gpu_ms, uint32_t* levels);
/* 64-source batched BFS in one persistent launch (replaces the per-source loop
 * of src/bench/main.cpp:324-364).  k <= 64 sources; out_host: k * n entries,
 * source-major (out_host[i * n + v] = depth of v from sources[i]), or NULL. */
int gb_bfs_run_batch(gb_bfs* h, const uint32_t* sources, int k, uint32_t* out_host,
                     const gb_bfs_options* opt, gb_level* trace, size_t cap, size_t* nlev);
/* lastGpuMs / lastLevels (src/metal/bfs_gpu.hpp:70-72): device time of the
 * last run (CUDA events on the handle's stream) and its level count. */
double gb_bfs_last_gpu_ms(const gb_bfs* h);
uint32_t gb_bfs_last_levels(const gb_bfs* h);
/* Device pointer of the last single-source result (n uint32), for callers that
 * keep results on the GPU (GpuBfs::dist(), src/metal/bfs_gpu.hpp:40); read it
 * again after gb_bfs_run_many, which may move the result to another buffer. */
const uint32_t* gb_bfs_device_dist(const gb_bfs* h);
/* The CUDA stream the handle launches on (cudaStream_t as void*). */
void* gb_bfs_stream(const gb_bfs* h);
/* GpuBfs::graph() (src/metal/bfs_gpu.hpp:39): the graph the handle traverses,
 * as a host CSR (the reference returns a view of its unified-memory buffers;
 * a discrete GPU copies the device arrays back).  Adjacency in the handle's
 * order (hub-first after gb_bfs_hub_first, which drops GB_FLAG_SORTED); flags
 * are the file's for gb_bfs_create_from_file handles, else 0.  Release with
 * gb_csr_free. */
int gb_bfs_graph(const gb_bfs* h, gb_csr* out);
/* Hub-first adjacency (the reference's proposed "hub-first neighbor order
 * inside adjacency lists", docs/REPORT.md:386-398 and 743-744): re-sorts the
 * handle's device copy of every adjacency list by descending neighbour degree,
 * ties by id.  Depths are unchanged; bottom-up levels find a frontier parent
 * sooner, so the "edges" of bottom-up trace records count fewer entries than
 * in the caller's order.  Stays in effect for the handle's lifetime. */
int gb_bfs_hub_first(gb_bfs* h);

/* Learned selector: load MLP parameters (layout of gb_selector_param_count) for
 * single-source (which = 0) or batched (which = 1) persistent runs. */
int gb_selector_shape(int* n_features, int* n_hidden, int* n_outputs);
size_t gb_selector_param_count(void);
int gb_bfs_set_selector(gb_bfs* h, int which, const float* params, size_t count);
/* Selector training kernels (GPU): loss + gradient of the masked MSE over a
 * batch (checked against the CPU oracle), and a full Adam training loop. */
int gb_mlp_loss_grad(const float* params, int batch, const float* x, const float* y,
                     const float* mask, float* grads_out, double* loss_out);
int gb_mlp_forward(const float* params, int batch, const float* x, float* out);
int gb_mlp_train(float* params_inout, int rows, const float* x, const float* y, const float* mask,
                 int epochs, int batch, float lr, uint64_t seed, float* final_loss);
/* Training data: run the single-source persistent BFS once per strategy, the
 * strategy forced at every level (a level's vertex set does not depend on it),
 * and record each level's features (gb_selector_shape) and its device time
 * under every strategy (us, min over `repeats` runs after a warm-up run).
 * rows_out: [cap][n_features] features, times_out: [cap][GB_NUM_STRATS].
 * Returns the number of rows via *rows. */
int gb_bfs_profile_levels(gb_bfs* h, uint32_t source, const gb_bfs_options* opt, int repeats,
                          float* feats_out, float* times_out, size_t cap, size_t* rows);
int gb_bfs_profile_batch_levels(gb_bfs* h, const uint32_t* sources, int k, const gb_bfs_options* opt,
                                int repeats, float* feats_out, float* times_out, size_t cap,
                                size_t* rows);

/* Autotuner (replaces scripts/sweep_balanced.sh, sweep_tg.sh, sweep_do.sh):
 * times candidate small_max/large_min and tg (gpu_binned), ept and tg
 * (gpu_edge, gpu_do), block size, grid size and hub_min cut (persistent, GB_BFS_BATCH)
 * on the given sources and writes the fastest into *o. */
int gb_bfs_autotune(gb_bfs* h, int variant, const uint32_t* sources, int k, gb_bfs_options* o);

/* --------------------------------------------------------------- PageRank */

typedef enum {
    GB_PR_PUSH = 0,          /* gpu_push          (src/shaders/pagerank.metal:228-267) */
    GB_PR_PULL_SCALAR = 1,   /* gpu_pull_scalar   (:306-312) */
    GB_PR_PULL_VECTOR = 2,   /* gpu_pull_vector   (:317-327) */
    GB_PR_PULL_ADAPTIVE = 3, /* gpu_pull_adaptive (:338-381) */
    GB_PR_PULL_GS = 4,       /* gpu_pull_gs       (src/metal/pagerank_gpu.mm:88-192) */
    GB_PR_PULL_F64 = 5,      /* double-precision Jacobi pull: the GPU oracle for FP32 runs */
    GB_PR_PULL_BLOCKED = 6   /* gpu_pull_blocked: Jacobi pull with the contributions staged in
                                shared memory, one 16K-vertex part at a time (TMA bulk copies),
                                over a per-row-block, per-part edge list; no reference counterpart
                                (a B200 layout of gpu_pull_*, src/metal/pagerank_gpu.mm:276-297) */
} gb_pr_variant;

/* GpuPrOptions (src/metal/pagerank_gpu.hpp:27-36). */
typedef struct {
    float damping;
    int32_t iters;     /* fixed mode: iterations; tol mode: cap */
    double tol;        /* > 0: stop when the L1 change < tol */
    double tol_rel;    /* > 0 (tol mode): also require max relative change < tol_rel */
    uint32_t tg;       /* threads per block of the main kernels */
    uint32_t small_max, large_min; /* adaptive bins (in-degree) */
    uint32_t inplace;  /* any pull variant: update contrib in place (GS-style) */
} gb_pr_options;

void gb_pr_default_options(gb_pr_options* o);

/* GpuPrResult (src/metal/pagerank_gpu.hpp:38-44). */
typedef struct {
    int32_t iters;
    int32_t floor_stop; /* tol mode: stopped because the L1 change stagnated */
    double last_delta;  /* tol mode: L1 change of the last iteration (FP64 on the GPU) */
    double last_max_rel;
    double gpu_ms;
} gb_pr_result;

typedef struct gb_pr gb_pr;

/* GpuPageRank(ctx, out, in, outdeg, needOut, needIn) (src/metal/pagerank_gpu.hpp:49-50).
 * out_* may be NULL when the push variant is not needed, in_* when no pull is. */
int gb_pr_create(uint64_t n, const uint32_t* out_row_ptr, const uint32_t* out_col_idx,
                 uint64_t out_m, const uint32_t* in_row_ptr, const uint32_t* in_col_idx,
                 uint64_t in_m, const uint32_t* outdeg, gb_pr** out);
int gb_pr_destroy(gb_pr* h);
/* prepareAdaptive / prepareGS (src/metal/pagerank_gpu.mm:70-192). */
int gb_pr_prepare_adaptive(gb_pr* h, uint32_t small_max, uint32_t large_min);
int gb_pr_prepare_gs(gb_pr* h, uint32_t pair_max_outdeg);
/* gsColored / gsSets / gsDeferred (src/metal/pagerank_gpu.hpp:82-84). */
int gb_pr_gs_info(const gb_pr* h, int* colored, uint64_t* sets, uint64_t* deferred);
/* GpuPageRank::run (src/metal/pagerank_gpu.mm:336-407). */
int gb_pr_run(gb_pr* h, int variant, const gb_pr_options* opt, gb_pr_result* res);
/* ranks() in the caller's ids (src/metal/pagerank_gpu.mm:194-203). */
int gb_pr_ranks(gb_pr* h, float* out_host);
/* FP64 ranks of the last GB_PR_PULL_F64 run. */
int gb_pr_ranks_f64(gb_pr* h, double* out_host);
int gb_pr_autotune(gb_pr* h, gb_pr_options* o);
void* gb_pr_stream(const gb_pr* h);

/* --------------------------------------------------- primitives (tests) */

/* Exclusive scan / sum / max of uint32 (src/metal/primitives.hpp:18-65),
 * host arrays in and out; total may be NULL. */
int gb_prim_scan(const uint32_t* in, uint64_t n, uint32_t* out, uint32_t* total);
/* Exclusive scan of device memory that allocates no device memory.  It has no
 * counterpart in the reference (src/metal/primitives.mm:69-101 allocates its
 * block-sum buffers per call); it exists for callers that cannot allocate at
 * the point of the scan, such as a program whose device memory is all held by
 * its own pool, or a stream pipeline that must avoid cudaMalloc / cudaFree
 * because they can wait for the whole device.
 *   in, out (in == out allowed), total, timeout_flag: device pointers on the
 *   current device; total and timeout_flag may be NULL.  out[i] = in[0] + ...
 *   + in[i-1] (mod 2^32), *total = sum of all n; *timeout_flag = 1 if a
 *   look-back wait ran out (the result is then invalid), else 0.
 *   stream: a cudaStream_t (NULL = the default stream).  The call only
 *   enqueues work: results are ready when the stream reaches them.
 * Limit: n <= 8,388,608 (4096 tiles of 2048); larger n returns
 * GB_ERR_CAPACITY and enqueues nothing.  The look-back scratch is one fixed
 * 32 KiB array per device inside the library, cleared on the stream by each
 * call before its kernel; calls whose kernels overlap on the same GPU (other
 * streams, other host threads) race on it and give undefined results, so
 * order them.  The first call on each device looks up that array's address
 * with the device current; make it before any stream capture begins.  A call
 * under a different context of that device (after cudaDeviceReset, or under a
 * context the caller created) looks the address up again. */
int gb_prim_scan_device_noalloc(const uint32_t* in, uint64_t n, uint32_t* out, uint32_t* total,
                                uint32_t* timeout_flag, void* stream);
int gb_prim_reduce(const uint32_t* in, uint64_t n, uint32_t* sum, uint32_t* max);
/* queueToBitmap then bitmapToQueue (src/metal/primitives.mm:103-123). */
int gb_prim_queue_bitmap(const uint32_t* queue, uint64_t size, uint64_t n, uint32_t* bitmap_out,
                         uint32_t* queue_out, uint64_t* count_out);
/* Grid barrier with a wait that cannot complete (expects one more block than
 * runs); must return GB_ERR_TIMEOUT after spin_limit polls, context intact. */
int gb_debug_barrier_timeout(uint64_t spin_limit);

#ifdef __cplusplus
}
#endif
#endif
