/*
 * cuts_b200.h -- C ABI of the B200 subgraph-isomorphism counting engine.
 *
 * Plain C types only (no C++ or torch types).  Every function returns an
 * int status (CUTS_OK == 0); on failure cuts_last_error() returns a
 * thread-local message.  Handles own their device memory; the caller frees
 * them.  A handle is not thread-safe; use one per host thread.
 *
 * Each entry point names the reference (cuTS) interface it replaces.
 */
#ifndef CUTS_B200_H
#define CUTS_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CUTS_OK 0
#define CUTS_ERR_ARG 1        /* invalid argument */
#define CUTS_ERR_IO 2         /* file cannot be opened / read */
#define CUTS_ERR_PARSE 3      /* malformed graph text */
#define CUTS_ERR_CUDA 4       /* CUDA runtime error */
#define CUTS_ERR_NOMEM 5      /* host or device allocation failed */
#define CUTS_ERR_QUERY 6      /* query unsupported (disconnected, too large) */
#define CUTS_ERR_CAPACITY 7   /* a level exceeds its capacity */
#define CUTS_ERR_LIMIT 8      /* graph exceeds a size limit of the layout */
#define CUTS_ERR_BUDGET 9     /* stopped by the caller's time budget */

#define CUTS_MAX_QUERY 16     /* query vertices (reference: QUERY_NODES 12) */

/* cuts_count flags */
#define CUTS_FLAG_SYMMETRY_BREAK 1u  /* count one embedding per automorphism
                                        orbit and scale by |Aut(Q)| (exact;
                                        query must be loop-free) */
#define CUTS_FLAG_NO_CLOSED_FORM 2u  /* enumerate the last level even when a
                                        closed form exists */
#define CUTS_FLAG_NO_FUSE 4u         /* materialise the level before the counted
                                        one even when it could be fused */
#define CUTS_FLAG_NO_ORBIT_FOLD 8u   /* with CUTS_FLAG_SYMMETRY_BREAK: break the
                                        whole query's symmetry even when the last
                                        vertex is a pendant whose removal leaves
                                        a more symmetric core */
#define CUTS_FLAG_NO_PAIR_FOLD 16u   /* enumerate the second-to-last level even
                                        when the last two vertices are pendants
                                        on the same earlier vertex, whose pairs
                                        have a closed form */

/* order modes for cuts_plan */
#define CUTS_ORDER_SCORE 0    /* greedy score order (score.cpp) */
#define CUTS_ORDER_LEARNED 1  /* learned cost model, score order fallback */

typedef struct cuts_graph_s *cuts_graph;   /* data graph resident on one GPU */
typedef struct cuts_query_s *cuts_query;   /* query graph + matching order */
typedef struct cuts_hgraph_s *cuts_hgraph; /* data graph in host memory (CSR) */

const char *cuts_last_error(void);
const char *cuts_version(void);

/* ---- host graph: loader, generators, writer ------------------------ */

/* Parse a graph file into a host CSR.  Replaces file_reader (util.cpp:
 * 19-52) and the CSR build of Graph::Graph (graph.cpp:18-61). */
int cuts_hgraph_load(const char *path, cuts_hgraph *out);
/* Seeded undirected Erdos-Renyi G(n, p), both arcs per edge.  No reference
 * counterpart (the reference reads SNAP files only). */
int cuts_hgraph_gen_er(uint32_t n, double p, uint64_t seed, cuts_hgraph *out);
/* Seeded undirected Chung-Lu graph with exactly m distinct edges, weights
 * min(cap, wmin * U^(-1/(gamma-1))).  No reference counterpart. */
int cuts_hgraph_gen_chung_lu(uint32_t n, uint64_t m, double gamma, double wmin, double cap,
                             uint64_t seed, cuts_hgraph *out);
int cuts_hgraph_info(cuts_hgraph h, uint32_t *n, uint64_t *arcs, int *symmetric,
                     uint32_t *max_degree);
/* Copy the CSR out (arrays sized n+1 / arcs; in_* ignored when symmetric). */
int cuts_hgraph_csr(cuts_hgraph h, uint64_t *out_off, uint32_t *out_adj, uint64_t *in_off,
                    uint32_t *in_adj);
/* Write the reference text format (line 1 = V, then "s<TAB>t"). */
int cuts_hgraph_write(cuts_hgraph h, const char *path);
/* Binary CSR cache of a host graph: saving once makes later loads skip text
 * parsing and sorting (the reference re-parses the text on every run,
 * util.cpp:19-52). */
int cuts_hgraph_save_binary(cuts_hgraph h, const char *path);
int cuts_hgraph_load_binary(const char *path, cuts_hgraph *out);
/* Make a host graph resident on `device` (the host graph stays valid).
 * Replaces malloc_graph_gpu_memory (gpu_memory_allocation.cu:26-37). */
int cuts_graph_upload(cuts_hgraph h, int device, cuts_graph *out);
void cuts_hgraph_free(cuts_hgraph h);

/* Seeded random connected undirected query: a random spanning tree plus each
 * other pair with probability p.  Writes both arcs of each edge into
 * src/dst (capacity k*k each) and their number into *narcs.  No reference
 * counterpart. */
int cuts_gen_random_query(uint32_t k, double p, uint64_t seed, uint32_t *narcs, uint32_t *src,
                          uint32_t *dst);

/* ---- data graph --------------------------------------------------- */

/* Load a graph file (line 1 = V, then "s<TAB>t" arcs) and make it resident
 * on `device`.  Replaces Graph::Graph(1, file) (graph.cpp:18-61, util.cpp:
 * 19-52) followed by malloc_graph_gpu_memory (gpu_memory_allocation.cu:
 * 26-37). */
int cuts_graph_load(const char *path, int device, cuts_graph *out);

/* The same from host CSR arrays (offsets n+1, sorted duplicate-free lists).
 * in_off/in_adj NULL means the graph is symmetric (in-lists == out-lists).
 * Replaces malloc_graph_gpu_memory (gpu_memory_allocation.cu:26-37). */
int cuts_graph_from_csr(uint32_t n, const uint64_t *out_off, const uint32_t *out_adj,
                        const uint64_t *in_off, const uint32_t *in_adj, int device,
                        cuts_graph *out);

/* n, distinct arcs, 1 if symmetric, maximum list length. */
int cuts_graph_info(cuts_graph g, uint32_t *n, uint64_t *arcs, int *symmetric,
                    uint32_t *max_degree);

/* Cap (in entries) of each intermediate trie level; 0 = automatic (sized
 * from free device memory).  Smaller caps force more chunks.  Replaces the
 * fixed GPU_TABLE_LIMIT (common.h:25, gpu_memory_allocation.cu:56-59). */
int cuts_graph_set_level_cap(cuts_graph g, uint64_t entries);

/* Size in bytes of the trie-level arena (allocated at the first count; 0 =
 * automatic: 384 B per arc within [256 MB, 64 GB] and 60% of free memory).
 * Frees the current arena; the next count allocates the new size. */
int cuts_graph_set_arena_bytes(cuts_graph g, uint64_t bytes);

/* Tile of the fused count of the last two levels: a parent whose candidate
 * set S holds more than `split` vertices is split into groups of 32 handed
 * to all warps (the hub split); 0 = the default (256, the size that fits
 * one warp's shared-memory tile).  Replaces nothing in the reference, whose
 * per-warp candidate tile is the fixed MAX_NE = 112 (common.h:31). */
int cuts_graph_set_fuse_split(cuts_graph g, uint32_t split);

void cuts_graph_free(cuts_graph g);

/* ---- query graph -------------------------------------------------- */

/* Load a query file and compute the score order.  Replaces
 * Graph::Graph(0, file) (graph.cpp:18-61) + sort_search_order
 * (graph.cpp:62-134). */
int cuts_query_load(const char *path, cuts_query *out);

/* Query from an arc list (k vertices, arcs as given; add both arcs for an
 * undirected edge).  Duplicates collapse, as in util.cpp:46-47. */
int cuts_query_from_arcs(uint32_t k, uint32_t narcs, const uint32_t *src,
                         const uint32_t *dst, cuts_query *out);

/* Number of query vertices and the current order (k entries). */
int cuts_query_info(cuts_query q, uint32_t *k, uint32_t *order);

/* P/C join lists of the current order over level positions (graph.cpp:
 * 94-133): p_off/c_off have k+1 entries, p/c at most k*k. */
int cuts_query_joins(cuts_query q, uint32_t *p_off, uint32_t *p, uint32_t *c_off,
                     uint32_t *c);

/* Replace the order (a permutation whose every prefix is connected). */
int cuts_query_set_order(cuts_query q, const uint32_t *order);

/* The first j positions of q's matching order as a query of its own (a
 * new handle, freed with cuts_query_free): it keeps q's degree signatures,
 * tests them at every level and counts plainly (no symmetry breaking), so its
 * per-level sizes are exactly the sizes of q's first j trie levels -- the
 * cheap way to log them when q's full count is out of reach.  No reference
 * counterpart. */
int cuts_query_prefix(cuts_query q, uint32_t j, cuts_query *out);

/* The per-level plan the kernels run for the current order, for a data
 * graph that is symmetric or not and the given flags: 12 words per level,
 * {joined lists, signature test, closed form, folded into the level before,
 * guaranteed-member mask, greater-than mask, less-than mask, fused with the
 * level before, orbit-fold positions, signature in-degree, signature
 * out-degree, pendant-pair fold (1 independent pendants, 2 ordered pendants,
 * both on one list: the level counts the last two levels' pairs)}.  Host only;
 * no reference counterpart (the reference derives joins per launch,
 * device_funcs.cu:103-127). */
int cuts_query_plan_levels(cuts_query q, int data_symmetric, uint32_t flags, uint32_t *out,
                           uint64_t *aut);

/* |Aut(Q)| (arc-preserving permutations). */
int cuts_query_automorphisms(cuts_query q, uint64_t *count);

void cuts_query_free(cuts_query q);

/* ---- counting ----------------------------------------------------- */

/* Count embeddings of q in g (reference semantics: injective, arc
 * preserving, degree signature filter).  chunks >= 1 splits the root level
 * into that many slices, as the reference's trunks argument does; memory
 * driven chunking is automatic on top of it.  *ms = device time from the
 * first kernel to the last, as the reference times it.  Replaces search()
 * (host_funcs.cu:115-171) and search_dfs_bfs_strategy() (host_funcs.cu:
 * 39-114) after the graphs are resident. */
int cuts_count(cuts_graph g, cuts_query q, uint32_t chunks, uint32_t flags,
               uint64_t *count, float *ms);

/* As cuts_count, and also reports per-level sizes |L_0|..|L_{k-1}|
 * (level_sizes has k entries; with CUTS_FLAG_SYMMETRY_BREAK they are the
 * constrained sizes) and statistics in stats[8]:
 *   [0] kernels launched, [1] chunks expanded,
 *   [2] algorithmic bytes of the last-level kernel (computed by an extra
 *       untimed pass, only when stats[2] is nonzero on entry),
 *   [3] last-level kernel device time in ns, [4] expansion kernel time in
 *       ns, [5] last-level launches, [6] expansion launches (event pairs
 *       around every launch, only when stats[3] is nonzero on entry),
 *   [7] reserved. */
int cuts_count_ex(cuts_graph g, cuts_query q, uint32_t chunks, uint32_t flags,
                  uint64_t *count, float *ms, uint64_t *level_sizes, uint64_t *stats);

/* Count only the roots u with u % nshards == shard, the rank striding of
 * the reference's multi-node level 0 (device_funcs.cu:267-279,
 * main_mpi.cu:257-376); the shard counts of 0..nshards-1 sum to the count,
 * and so do the per-level sizes (level_sizes: k entries, may be NULL). */
int cuts_count_sharded(cuts_graph g, cuts_query q, uint32_t chunks, uint32_t flags,
                       uint32_t shard, uint32_t nshards, uint64_t *count, float *ms,
                       uint64_t *level_sizes);

/* cuts_count_sharded with the statistics of cuts_count_ex (stats[8], same
 * layout and the same opt-in entries). */
int cuts_count_sharded_ex(cuts_graph g, cuts_query q, uint32_t chunks, uint32_t flags,
                          uint32_t shard, uint32_t nshards, uint64_t *count, float *ms,
                          uint64_t *level_sizes, uint64_t *stats);

/* As cuts_count, but stops with CUTS_ERR_BUDGET once budget_ms has passed:
 * the host checks between chunks, and every kernel of the run stops taking
 * work once budget_ms of device time has passed since the run's first
 * kernel, so one oversized chunk cannot overrun the budget by more than the
 * work items already in flight. */
int cuts_count_budget(cuts_graph g, cuts_query q, uint32_t chunks, uint32_t flags,
                      double budget_ms, uint64_t *count, float *ms, uint64_t *level_sizes);

/* The root stripe u % nshards == shard of cuts_count, under a time budget
 * (0 = none): the per-level sizes of a stripe, scaled by nshards, estimate the
 * full run's.  Used to log training data for the learned order cheaply. */
int cuts_count_sample(cuts_graph g, cuts_query q, uint32_t shard, uint32_t nshards,
                      uint32_t flags, double budget_ms, uint64_t *count, float *ms,
                      uint64_t *level_sizes);

/* Write every embedding to `path` in the reference's ans.txt line format
 * "(q,d)(q,d)..." in matching order (util.cpp:53-74).  Returns the number
 * of lines in *count.  Line order is unspecified, as in the reference. */
int cuts_dump(cuts_graph g, cuts_query q, const char *path, uint64_t *count);

/* The matches of cuts_dump whose root (the data vertex matched at the first
 * position of the order) is among the roots u with u % nshards == shard, in
 * the engine's vertex numbering; the shards 0..nshards-1 together write every
 * line of cuts_dump once.  Bounds one call's output on large graphs, where
 * the reference holds every match in a 200 GB managed table
 * (gpu_memory_allocation.cu:60-68) before writing ans.txt (util.cpp:53-74). */
int cuts_dump_sharded(cuts_graph g, cuts_query q, uint32_t shard, uint32_t nshards, const char *path,
                      uint64_t *count);

/* Reference in-process API (host_funcs.h:21-25): load both files, make the
 * data graph resident, count, print "<data>,<query>,<ms>ms,<count>" and,
 * when write_to_disk != 0, write ans.txt in the working directory.
 * trunks == 0 runs search(); trunks >= 1 runs search_dfs_bfs_strategy().
 * The count (every embedding, as the reference's) is found with exact
 * symmetry breaking unless the environment sets CUTS_PLAIN=1. */
int cuts_search(const char *query_file, const char *data_file, int write_to_disk,
                uint32_t trunks, uint64_t *count, float *ms);

/* ---- learned matching order ---------------------------------------- */

/* The cost model of the learned order: an FP32 MLP in -> 64 -> 64 -> 1
 * (ReLU) predicting log(1 + |L_i|) from per-step order features, trained and
 * evaluated by this library's own kernels.  No reference counterpart: the
 * reference has only the greedy score order (graph.cpp:62-93). */
#define CUTS_FEATURES 16
typedef struct cuts_mlp_s *cuts_mlp;
int cuts_mlp_create(uint32_t in_dim, uint64_t seed, int device, cuts_mlp *out);
int cuts_mlp_param_count(cuts_mlp m, uint32_t *n);
int cuts_mlp_get_params(cuts_mlp m, float *params);
int cuts_mlp_set_params(cuts_mlp m, const float *params);
/* Mean squared error over n rows and its gradient (n_params floats). */
int cuts_mlp_loss_grad(cuts_mlp m, const float *X, const float *y, uint32_t n, float *loss,
                       float *grad);
/* Adam, `epochs` passes over mini-batches of `batch` rows (0 = full batch). */
int cuts_mlp_train(cuts_mlp m, const float *X, const float *y, uint32_t n, uint32_t epochs,
                   uint32_t batch, float lr, float *final_loss);
int cuts_mlp_predict(cuts_mlp m, const float *X, uint32_t n, float *y);
void cuts_mlp_free(cuts_mlp m);

/* Feature rows (k x CUTS_FEATURES) of the given order on graph g, with the
 * parent-level feature taken from level_sizes (teacher forcing). */
int cuts_query_features(cuts_query q, cuts_graph g, const uint32_t *order,
                        const uint64_t *level_sizes, float *features);

/* Choose and set the query's order.  CUTS_ORDER_SCORE: the score order
 * (graph.cpp:62-93).  CUTS_ORDER_LEARNED: search connected-prefix orders
 * (exhaustive, or a beam of `beam` prefixes when beam > 0) with the model m
 * and keep the best unless its predicted work is not `margin` times below
 * the score order's, in which case the score order stays.  order_out (k),
 * pred_work and score_work (predicted work of the chosen and of the score
 * order) may be NULL. */
int cuts_plan(cuts_query q, cuts_graph g, int mode, cuts_mlp m, uint32_t beam, double margin,
              uint32_t *order_out, double *pred_work, double *score_work);

/* The max_orders complete orders with the least predicted work under the
 * model m (same search as cuts_plan), least first, without changing the
 * query's order: orders_out holds max_orders x k entries, work_out (may be
 * NULL) max_orders values; *n_out receives how many were found.  Lets a
 * caller measure a few proposals on a root stripe and keep the fastest. */
int cuts_plan_candidates(cuts_query q, cuts_graph g, cuts_mlp m, uint32_t beam, uint32_t max_orders,
                         uint32_t *orders_out, double *work_out, uint32_t *n_out);

/* ---- batched counting -------------------------------------------- */

/* Count nq queries against one resident graph in one persistent launch.
 * counts[nq] receives exact per-query counts; status[nq] (may be NULL)
 * receives 0 or a CUTS_ERR_* code per query.  No reference counterpart
 * (the reference runs one query per process). */
int cuts_count_batch(cuts_graph g, const cuts_query *qs, uint32_t nq, uint32_t flags,
                     uint64_t *counts, int *status, float *ms);

/* A reusable batch: the launch is captured once in a CUDA graph and replayed
 * by every cuts_batch_run.  tune[3] = {grain (level-1 candidates per task),
 * tasks per work-counter grab, max blocks per SM}; NULL or 0 entries take
 * the defaults.  The query handles must outlive the batch. */
typedef struct cuts_batch_s *cuts_batch;
int cuts_batch_create(cuts_graph g, const cuts_query *qs, uint32_t nq, uint32_t flags,
                      const uint32_t *tune, cuts_batch *out);
/* budget_ms > 0 stops the launch after that much device time; unfinished
 * queries get status CUTS_ERR_BUDGET and a partial count.  *ms is the
 * device time of the launch. */
int cuts_batch_run(cuts_batch b, double budget_ms, uint64_t *counts, int *status, float *ms);
/* tasks in the launch, launch blocks */
/* Per-query limit for later cuts_batch_run calls: each query may use ms of
 * the whole GPU (its warp time summed over the launch's warps, up to ms x the
 * launch's warps); a query past it reports CUTS_ERR_BUDGET while the others
 * carry on.  0 = no limit (the default).  No reference counterpart: the
 * reference runs one query per process. */
int cuts_batch_set_query_budget(cuts_batch b, double ms);
/* Later cuts_batch_run calls take only the tasks t with t % nshards == shard
 * (tasks are (query, root, level-1 range)), so one launch per GPU with
 * shard = rank partitions every query's count; sum the per-query counts over
 * ranks.  Plays the part of the reference's rank striping of roots
 * (device_funcs.cu:273, main_mpi.cu) for a batch. */
int cuts_batch_set_shard(cuts_batch b, uint32_t shard, uint32_t nshards);
int cuts_batch_info(cuts_batch b, uint64_t *tasks, uint32_t *blocks);
void cuts_batch_free(cuts_batch b);

/* ---- allocation-free counting ------------------------------------- */

/* For callers that cannot allocate GPU memory themselves -- code inside a
 * host framework that owns every device allocation (a pool that must
 * account for all bytes, a sandboxed plugin): count up to 64 queries in one
 * launch using only buffers the caller passes in.  No reference counterpart.
 *
 * Inputs, in the caller's device memory: info_out[2v] = offset of v's
 * out-list in adj, info_out[2v+1] = its length (u32 pairs, 8-byte aligned);
 * info_in likewise for in-lists, or NULL for a symmetric graph; adj (u32).
 * The caller guarantees what the resident-graph path validates on upload:
 * every list strictly increasing (sorted, no duplicates), every id below n,
 * every (offset, length) inside adj, and for info_in == NULL every arc's
 * reverse present.  These are not checked here: duplicates give wrong
 * counts and out-of-range ids read out of bounds.
 * Output: counts[nq] (u64, device memory), overwritten with the exact count
 * of each query (not touched when nq == 0; zeros when n == 0).  Work is
 * queued on `stream` (a cudaStream_t, NULL = the default stream) and the
 * call returns without waiting: the query plans travel as kernel
 * parameters, so no host buffer has to outlive the call.  Synchronise the
 * stream before reading counts.
 *
 * Calls no cudaMalloc, cudaFree or other allocating routine.  The engine's
 * own scratch for this path (query plans, work counter) is a fixed array of
 * about 42 KB in device memory that every GPU loading this library holds
 * until the process exits.  The first call on a device looks up that
 * array's device address and the launch shape, with the device current;
 * make that first call before any stream capture.  Every call shares the
 * array and clears what must start at zero, so calls that overlap on the
 * GPU (other streams, other threads) race: serialise them.
 *
 * Limits, rejected with CUTS_ERR_LIMIT: more than 64 queries, a query of
 * more than 10 vertices, a level joining more than 8 lists.
 * CUTS_FLAG_SYMMETRY_BREAK is rejected (CUTS_ERR_ARG). */
int cuts_count_noalloc(const uint32_t *info_out, const uint32_t *info_in, const uint32_t *adj,
                       uint32_t n, const cuts_query *qs, uint32_t nq, uint32_t flags,
                       uint64_t *counts, void *stream);

#ifdef __cplusplus
}
#endif
#endif
