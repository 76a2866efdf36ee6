/*
 * dyngb200.h -- the C ABI of dyng_b200: dynG's batch-dynamic single-source shortest-path update
 * (dyng::sssp::compute / dyng::sssp::update on resources::cuda()) rebuilt for NVIDIA B200
 * (sm_100a).  Plain pointers and sizes, no C++ or torch types.
 *
 * Every entry point returns a dyngb200_status; on failure dyngb200_last_error_message() holds a
 * message for the calling thread.  The statuses mirror the reference's exception classes
 * (cpp/include/dyng/core/error.hpp): invalid_argument_error, not_supported_error,
 * stale_result_error, out_of_memory_error, cuda_error, capacity_error, internal_error.
 *
 * Memory: graphs and trees live in device memory.  Batch and array arguments name their memory
 * space (DYNGB200_HOST or DYNGB200_DEVICE).  A call is complete on the host when it returns: the
 * context's stream is synchronized once at the end of compute/update (the control block is
 * read), as the reference's fused engine does (cpp/src/algorithms/sssp/cuda.cu:183-195).
 *
 * Threading: a context, graph or tree is not thread-safe; distinct graphs and trees may be used
 * concurrently from different contexts (cpp/include/dyng/graph/graph.hpp:63-70).
 */
#ifndef DYNGB200_H
#define DYNGB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DYNGB200_ABI_VERSION 1

typedef enum dyngb200_status {
  DYNGB200_OK = 0,
  DYNGB200_INVALID_ARGUMENT = 1, /* invalid_argument_error */
  DYNGB200_NOT_SUPPORTED = 2,    /* not_supported_error */
  DYNGB200_STALE_RESULT = 3,     /* stale_result_error */
  DYNGB200_OUT_OF_MEMORY = 4,    /* out_of_memory_error */
  DYNGB200_CUDA_ERROR = 5,       /* cuda_error */
  DYNGB200_CAPACITY = 6,         /* capacity_error */
  DYNGB200_INTERNAL = 7          /* internal_error */
} dyngb200_status;

typedef enum dyngb200_memory { DYNGB200_HOST = 0, DYNGB200_DEVICE = 1 } dyngb200_memory;

/* dyng::engine (cpp/include/dyng/core/types.hpp): a tunable that never changes the result
 * (sssp.cpp:195-226).  FUSED: one cooperative persistent kernel for the applier and one for the
 * sssp step, every loop decision on the device, one host synchronization per call; refused with
 * NOT_SUPPORTED, before anything changes, on a device without cooperative launch.  OPERATORS:
 * ordinary launches (one per applier step, one per sssp phase and per near-far step) with the
 * loop on the host, which reads a few counters after each step; runs on any device.  AUTOMATIC:
 * FUSED where the device offers cooperative launch, OPERATORS otherwise.  The stats report the
 * engine that ran (engine_used). */
typedef enum dyngb200_engine {
  DYNGB200_ENGINE_AUTOMATIC = 0,
  DYNGB200_ENGINE_FUSED = 1,
  DYNGB200_ENGINE_OPERATORS = 2
} dyngb200_engine;

typedef struct dyngb200_context_s* dyngb200_context; /* resources::cuda() */
typedef struct dyngb200_scheduler_s* dyngb200_scheduler; /* the learned scheduler (bf16 MLP) */
typedef struct dyngb200_graph_s* dyngb200_graph;     /* graph<int32,int64,int32> on the device */
typedef struct dyngb200_tree_s* dyngb200_tree;       /* sssp::result<int32> */

/* graph_properties + batch_semantics (cpp/include/dyng/graph/graph_properties.hpp:67-241).
 * dyngb200_props_default() gives the reference's defaults; mosp_compatible() is sorted = 0,
 * allow_multi = 1. */
typedef struct dyngb200_props {
  int32_t directed;            /* 1: directed; 0: every batch edge (u,v) changes both directions */
  int32_t sorted;              /* row_order::sorted (1) or append (0) */
  int32_t allow_multi;         /* multi_edges::allow (1) or forbid (0) */
  int32_t on_existing_insert;  /* 0 upsert, 1 error, 2 ignore */
  int32_t on_missing_delete;   /* 0 ignore, 1 error */
  int32_t on_self_loop;        /* 0 keep, 1 drop, 2 error */
  int32_t deletions_first;     /* 1: deletions, then insertions */
  int32_t allow_vertex_growth; /* 1: insertions may name new vertices */
  double headroom;             /* spare slots per slack row, as a fraction of its degree */
} dyngb200_props;

/* edge_batch_view<int32, int32> (cpp/include/dyng/graph/edge_batch.hpp:38-76). Insertion weights
 * are insertion-major: num_weights per insertion. */
typedef struct dyngb200_batch {
  const int32_t* insert_src;
  const int32_t* insert_dst;
  const int32_t* insert_weights;
  int64_t num_insertions;
  const int32_t* delete_src;
  const int32_t* delete_dst;
  int64_t num_deletions;
  int32_t num_weights;
  int32_t memory; /* dyngb200_memory of all five arrays */
} dyngb200_batch;

/* apply_summary (cpp/include/dyng/graph/apply_summary.hpp). */
typedef struct dyngb200_apply_summary {
  int64_t inserted_edges;
  int64_t deleted_edges;
  int64_t updated_edges;
  int64_t ignored_insertions;
  int64_t ignored_deletions;
  int64_t dropped_self_loops;
  int64_t inserted_vertices;
  int64_t num_vertices_after;
} dyngb200_apply_summary;

/* sssp::stats (cpp/include/dyng/sssp.hpp:100-117) plus the schedule that ran and device times. */
typedef struct dyngb200_stats {
  dyngb200_apply_summary batch;
  int64_t invalidated; /* deterministic */
  int64_t affected;    /* deterministic: vertices whose distance or parent changed */
  int64_t iterations;  /* schedule-dependent */
  int64_t epochs;      /* schedule-dependent */
  int64_t pushes;      /* schedule-dependent */
  int32_t packed_parents;
  int32_t engine_used; /* dyngb200_engine that ran: FUSED or OPERATORS */
  int64_t delta;       /* near-far width that ran */
  int64_t max_weight;  /* bound weight of the packing */
  int32_t grid_blocks; /* persistent grid that ran (operators engine: its launches' grid) */
  int32_t invalidation; /* 0 pointer jumping, 1 subtree walk */
  float apply_ms;      /* device time of the batch applier */
  float sssp_ms;       /* device time of the sssp kernel */
  int64_t rounds;      /* pointer-jumping rounds */
  int64_t touched;     /* vertices the commit rewrote (their distance or parent changed) */
  /* Work of the sssp kernel, for its algorithmic traffic: [0] vertex visits of the pointer-jumping
   * rounds, [1] jumps, [2] invalidated, [3] pull candidates, [4] pulled in-slots, [5] word reads of
   * the pull, [6] pushed vertices, [7] scanned out-slots, [8] target word reads, [9] successful
   * atomicMin, [10] frontier appends, [11] vertices the commit compared, [12] atomicMin attempts (successful
   * or not); the first near-far step's balance: [13] the slowest warp's busy ns, [14] the warps'
   * summed busy ns, [15] warps, [16..18] the warps' summed ns in light / medium / heavy rows,
   * [19..21] the slowest warp's ns in each; [22] vertices seeded for pointer jumping; [23]
   * successful atomicMin of the pull, [24] frontier appends of the pull, [25] change pairs
   * visited by the roots and insertion-head passes; [26] rows and [27] slots of the subtree
   * walk (the walk invalidation); [28] change stamps the commit scanned ([11] then counts the
   * stamped vertices it compared); [29..31] zero.  [9] and [10] count the near-far loop only. */
  int64_t work[32];
  /* Device time of the kernel's phases (ms): setup+roots, pointer jumping, invalidation, pull,
   * first split, near-far loop, unpack. */
  float phase_ms[7];
  /* Trace of the first 64 steps of the near-far loop: light frontier size (negative: an epoch
   * with that many far vertices), heavy chunks, and the step's start in microseconds since the
   * kernel began. */
  /* The first 64 near-far steps: light frontier entries, heavy-row chunks (bit 30 set: the step
   * ran block-local, in the small-frontier mode), and the time since the kernel began. */
  int32_t trace_len;
  int32_t trace_light[64];
  int32_t trace_heavy[64];
  float trace_us[64];
  /* The learned scheduler's view of the update (filled when a scheduler ran or the schedule asked
   * for record_features): the 12 batch features and the class each head chose (-1: none; -2:
   * the features were outside the scheduler's trained range, the plain schedule ran). */
  float features[12];
  int32_t schedule_classes[3];
  int64_t kernel_launches; /* kernels of this library the call launched */
  float pj_round_us[24];    /* start of each pointer-jumping round, us since the kernel began */
  float pj_done_us[24];     /* the last block's arrival at the barrier ending each round */
  /* The batch applier kernel: the end of each of its steps (us since it began; 0: not reached):
   * [1] checks, [2] pairs, [3] matching, [4] resolution, then (append-order rows) three ordering
   * steps, then allocation, mutation, moves and appends, row descriptors; [11] the finalize. */
  float apply_step_us[12];
  /* Host time of the call (us): [0] checks, index room and batch staging, [1] queuing the batch
   * applier, [2] queuing the sssp kernel and the read-back, [3] waiting for the device. */
  float host_us[4];
} dyngb200_stats;

/* sssp::options (cpp/include/dyng/sssp.hpp:78-94). */
typedef struct dyngb200_options {
  int64_t delta;           /* near-far width; 0 = automatic (the reference's defaultDelta) */
  int32_t objective;       /* weight column, fixed at compute() */
  int32_t cuda_engine;     /* dyngb200_engine */
  int32_t validate_inputs; /* O(n) checks of imported trees */
} dyngb200_options;

/* The schedule of one update: what the learned scheduler chooses.  A tunable only: every field
 * changes the order of work, never the distances or parents.  Zero fields mean "the fixed
 * heuristic": delta from the options, the occupancy grid, pointer-jumping invalidation. */
typedef struct dyngb200_schedule {
  int64_t delta;          /* near-far bucket width (0: heuristic) */
  int32_t grid_blocks;    /* persistent grid size (0: occupancy x SMs) */
  int32_t invalidation;   /* 0 heuristic/pointer jumping, 1 subtree walk */
  int32_t small_frontier; /* frontiers up to this many vertices run on one block (0: 256, < 0: off) */
  int32_t heavy_degree;   /* rows longer than this are split across warps (0: default) */
  int32_t record_features; /* nonzero: compute the scheduler's features into the stats */
} dyngb200_schedule;

/* ---- errors ------------------------------------------------------------------------------ */
const char* dyngb200_last_error_message(void);
const char* dyngb200_status_name(dyngb200_status s);
int dyngb200_abi_version(void);

/* ---- context: resources::cuda(device) (cpp/include/dyng/core/resources.hpp) --------------- */
/* stream: a cudaStream_t, or NULL for a stream owned by the context. */
dyngb200_status dyngb200_context_create(int device, void* stream, dyngb200_context* out);
dyngb200_status dyngb200_context_destroy(dyngb200_context ctx);
dyngb200_status dyngb200_context_synchronize(dyngb200_context ctx);
void dyngb200_props_default(dyngb200_props* props);
void dyngb200_props_mosp_compatible(dyngb200_props* props);

/* ---- test support (the reference's tests/support: failing_allocator.hpp:18-143, the counting
 * resource of sssp_cuda_test.cpp:622-655, resources_access::force_cooperative_launch used at
 * sssp_cuda_test.cpp:106-150).  Failures made on the host: nothing here faults a GPU. ------- */
typedef struct dyngb200_test_hooks {
  /* A grid barrier of the persistent kernel gives up after this long without progress (0: the
   * library's 5 s); it then records a timeout, every block leaves the kernel and the call
   * reports INTERNAL with the tree poisoned. */
  int64_t barrier_timeout_ns;
  /* Blocks every grid barrier waits for beyond the launched ones (0: none).  Nothing ever
   * arrives for them, so every barrier's wait runs out after barrier_timeout_ns. */
  int32_t barrier_extra_arrivals;
  /* Nonzero: the context behaves as on a device without cooperative launch: calls asking for
   * the fused engine are refused with NOT_SUPPORTED before anything changes, automatic ones run
   * the operators engine (graph_apply its applier as one launch per step). */
  int32_t no_cooperative_launch;
  /* Which persistent kernel the phantom arrivals hold up: 0 both, 1 the batch applier (its first
   * barrier comes before any change: the call fails with the graph and the tree unchanged), 2 the
   * sssp kernel (after the batch is applied: the tree is poisoned). */
  int32_t barrier_kernel;
} dyngb200_test_hooks;
/* Set (hooks) or clear (NULL) the test hooks of a context. */
dyngb200_status dyngb200_context_set_test_hooks(dyngb200_context ctx,
                                                const dyngb200_test_hooks* hooks);
/* Device allocations the library has made in this process (every DevBuf growth; frees are not
 * counted): after warm-up, a steady stream of same-size updates adds none. */
dyngb200_status dyngb200_debug_device_allocations(int64_t* count);
/* The nth device allocation from now fails as cudaMalloc would (OUT_OF_MEMORY); 0 disarms. */
dyngb200_status dyngb200_debug_fail_device_allocation(int64_t nth);

/* ---- graph (cpp/include/dyng/graph/graph.hpp:143-195, 332-487) ----------------------------- */
/* graph<int32,int64,int32>::from_edges: weights insertion-major (num_weights per edge). */
dyngb200_status dyngb200_graph_from_edges(dyngb200_context ctx, int64_t num_vertices,
                                          const int32_t* src, const int32_t* dst,
                                          const int32_t* weights, int64_t num_edges,
                                          int32_t num_weights, int32_t memory,
                                          const dyngb200_props* props, dyngb200_graph* out);
/* graph::from_csr: row_ptr has num_vertices + 1 entries, weights objective-major. */
dyngb200_status dyngb200_graph_from_csr(dyngb200_context ctx, int64_t num_vertices,
                                        const int64_t* row_ptr, const int32_t* col,
                                        const int32_t* weights, int32_t num_weights,
                                        int32_t memory, const dyngb200_props* props,
                                        dyngb200_graph* out);
dyngb200_status dyngb200_graph_destroy(dyngb200_graph g);
/* num_vertices / num_edges / num_weights / version (graph.hpp:332-354). */
dyngb200_status dyngb200_graph_info(dyngb200_graph g, int64_t* num_vertices, int64_t* num_edges,
                                    int32_t* num_weights, uint64_t* version);
/* graph::apply (graph.hpp:474): the batch alone, on the device.  weight_increased (optional,
 * host, num_effective_insertions x num_weights bytes) receives the classification. */
dyngb200_status dyngb200_graph_apply(dyngb200_context ctx, dyngb200_graph g,
                                     const dyngb200_batch* batch,
                                     dyngb200_apply_summary* summary);
/* graph::apply plus the weight-increase classification of apply_host.cpp:348-393: host buffer
 * weight_increased receives num_insertions x num_weights bytes (1: the insertion raised that
 * objective's weight of the first (u,v) of row u). */
dyngb200_status dyngb200_graph_apply_classified(dyngb200_context ctx, dyngb200_graph g,
                                                const dyngb200_batch* batch,
                                                dyngb200_apply_summary* summary,
                                                uint8_t* weight_increased);
/* graph::to_csr (graph.hpp:487) plus the in-edge mirror; host buffers sized from
 * dyngb200_graph_info (row_ptr n+1, col m, weights k*m objective-major); any pointer may be NULL. */
dyngb200_status dyngb200_graph_to_csr(dyngb200_context ctx, dyngb200_graph g, int64_t* row_ptr,
                                      int32_t* col, int32_t* weights, int64_t* in_row_ptr,
                                      int32_t* in_col, int32_t* in_weights);
/* Device memory held by the graph, in bytes. */
dyngb200_status dyngb200_graph_device_bytes(dyngb200_graph g, int64_t* bytes);
/* The slack-row storage behind a graph (no reference counterpart: the reference's CSR has no
 * slack).  Figures as of the last completed call on the graph. */
typedef struct dyngb200_graph_storage {
  int64_t vertex_capacity;         /* rows allocated per side */
  int64_t arena_slots;             /* slots of each side's arena */
  int64_t out_top, in_top;         /* slots handed out (rows, their slack, abandoned space) */
  int64_t out_garbage, in_garbage; /* slots abandoned by rows that moved */
  int64_t index_slots;             /* edge index capacity (0 for multigraphs) */
  int64_t arena_growths;           /* arena enlargements, done on the device */
  int64_t compactions;             /* compactions, done on the device */
  int64_t index_builds;            /* edge index (re)builds */
  double grow_ms, compact_ms, index_ms; /* host time of the above, summed (includes the wait) */
  double maintenance_ms_max;       /* the longest single growth, compaction or index build */
} dyngb200_graph_storage;
dyngb200_status dyngb200_graph_storage_get(dyngb200_graph g, dyngb200_graph_storage* out);

/* ---- sssp (cpp/include/dyng/sssp.hpp:415-489) -------------------------------------------- */
/* sssp::compute(resources::cuda(), g, source, opt) (sssp.hpp:415-421). opt may be NULL. */
dyngb200_status dyngb200_sssp_compute(dyngb200_context ctx, dyngb200_graph g, int32_t source,
                                      const dyngb200_options* opt, dyngb200_tree* out,
                                      dyngb200_stats* stats);
/* sssp::update(resources::cuda(), g, batch, tree) (sssp.hpp:484-489). */
dyngb200_status dyngb200_sssp_update(dyngb200_context ctx, dyngb200_graph g,
                                     const dyngb200_batch* batch, dyngb200_tree tree,
                                     dyngb200_stats* stats);
/* dyng::update_each(resources::cuda(), g, batch, results) (update.hpp:331) for sssp results,
 * e.g. the K objectives of a multi-weight graph: the batch is applied once and every tree is
 * updated (one stats per tree, in order).  Errors found before the batch is applied, for any
 * tree, leave the graph and all trees unchanged; an error after it poisons that tree only, the
 * others are still updated, and the first error is returned. */
dyngb200_status dyngb200_sssp_update_each(dyngb200_context ctx, dyngb200_graph g,
                                          const dyngb200_batch* batch, dyngb200_tree* trees,
                                          int32_t count, dyngb200_stats* stats);
/* ---- mosp (cpp/include/dyng/mosp.hpp): K objectives, the combined graph, the MOSP tree ------ */
/* mosp::options (mosp.hpp:79-101).  preferences: NULL / num_preferences 0 for all ones, else one
 * per objective, each >= 1 (a lower value is a higher priority), lcm <= 2^20. */
typedef struct dyngb200_mosp_options {
  int32_t num_objectives;       /* the first K weight columns; 0 = every column (K <= 64) */
  int32_t num_preferences;
  const int32_t* preferences;
  int64_t delta;                /* near-far width of the K sssp updates; 0 = automatic */
  int32_t compute_path_costs;   /* path costs at compute() / update() (1 by default) */
  int32_t validate_inputs;      /* from_arrays: sssp's checks of every imported tree */
} dyngb200_mosp_options;
/* mosp::stats (mosp.hpp:115-125). */
typedef struct dyngb200_mosp_stats {
  dyngb200_apply_summary batch;
  int64_t affected;          /* vertices whose combined distance or MOSP parent changed */
  int64_t combined_edges;
  int64_t preference_scale;  /* L = lcm(preferences): combined distances are in units of 1/L */
  int64_t iterations;        /* summed over the K sssp updates and the combined solve */
  int32_t converged;
  float combine_ms, solve_ms, costs_ms; /* host time of the finalize stages (with their waits) */
} dyngb200_mosp_stats;
typedef struct dyngb200_mosp_s* dyngb200_mosp;
/* mosp::compute(resources::cuda(), g, source, opt) (mosp.hpp:444-449); opt may be NULL. */
dyngb200_status dyngb200_mosp_compute(dyngb200_context ctx, dyngb200_graph g, int32_t source,
                                      const dyngb200_mosp_options* opt, dyngb200_mosp* out);
/* mosp::result::from_arrays (mosp.hpp:300-347): K trees of g (distances[k], parents[k]: n
 * values each, in `memory`), imported as sssp::result::from_arrays imports one tree, then the
 * combined graph, the MOSP tree and the path costs.  K must equal the objectives opt selects. */
dyngb200_status dyngb200_mosp_from_arrays(dyngb200_context ctx, dyngb200_graph g, int32_t source,
                                          int32_t num_trees, const int64_t* const* distances,
                                          const int32_t* const* parents, int64_t n,
                                          int32_t memory, int32_t canonicalize,
                                          const dyngb200_mosp_options* opt, dyngb200_mosp* out);
/* mosp::update(resources::cuda(), g, batch, r) (mosp.hpp:502-506): the batch applied once, the
 * K trees updated (dyng::update_each), then the combined graph solved again.  objective_stats:
 * NULL or K entries.  An error before the batch is applied changes nothing; an error after it
 * leaves the result unusable (stale_result_error on every access). */
dyngb200_status dyngb200_mosp_update(dyngb200_context ctx, dyngb200_graph g,
                                     const dyngb200_batch* batch, dyngb200_mosp r,
                                     dyngb200_mosp_stats* stats, dyngb200_stats* objective_stats);
dyngb200_status dyngb200_mosp_destroy(dyngb200_mosp r);
/* K, n, L, the source and the graph version the result matches. */
dyngb200_status dyngb200_mosp_info(dyngb200_mosp r, int32_t* num_objectives, int64_t* num_vertices,
                                   int64_t* preference_scale, int32_t* source,
                                   uint64_t* graph_version);
/* The sssp tree of one objective (mosp::result::distances(k) / parents(k)): a borrowed handle,
 * owned by r and valid until r is destroyed; do not destroy it. */
dyngb200_status dyngb200_mosp_tree(dyngb200_mosp r, int32_t objective, dyngb200_tree* out);
/* combined_distances() / combined_parents(): n values each into buffers in `memory` (either may
 * be NULL). */
dyngb200_status dyngb200_mosp_combined(dyngb200_mosp r, int64_t* distances, int32_t* parents,
                                       int32_t memory);
/* path_costs(): n x K values, vertex-major, into a host buffer; INVALID_ARGUMENT if they were
 * not computed at the last compute() / update(). */
dyngb200_status dyngb200_mosp_path_costs(dyngb200_mosp r, int64_t* costs);
/* The path costs along the current MOSP tree over the first `columns` weight columns of g
 * (MOSP's mospCosts.txt covers every column of the graph), n x columns into a host buffer. */
dyngb200_status dyngb200_mosp_path_costs_columns(dyngb200_context ctx, dyngb200_graph g,
                                                 dyngb200_mosp r, int32_t columns, int64_t* costs);
/* result::set_options: delta, compute_path_costs and validate_inputs change (from the next
 * update); num_objectives and preferences must stay the same. */
dyngb200_status dyngb200_mosp_set_options(dyngb200_mosp r, const dyngb200_mosp_options* opt);

/* sssp::update with an explicit schedule (the learned scheduler's entry point; no reference
 * counterpart beyond options::delta / options::cuda_engine, which are tunables the same way). */
dyngb200_status dyngb200_sssp_update_scheduled(dyngb200_context ctx, dyngb200_graph g,
                                               const dyngb200_batch* batch, dyngb200_tree tree,
                                               const dyngb200_schedule* schedule,
                                               dyngb200_stats* stats);

/* sssp::compute into caller-owned device arrays, allocating nothing.  No counterpart in the
 * reference.  For callers that cannot allocate device memory while they run: serving processes
 * that reserve their whole memory budget at start-up and treat any later allocation as a fault,
 * and host frameworks that own the device allocator.  The graph
 * (on the current device) and the outputs -- distances: int64 x num_vertices, parents: int32 x
 * num_vertices, both device memory -- come from the caller; the kernel's scratch is a fixed
 * device array of about 6 MB inside this library that every GPU which loads it holds until exit, so
 * graphs are limited to 65,536 vertices (larger ones are rejected with INVALID_ARGUMENT).  The
 * first call on a device looks up that array's device address; make it before any stream
 * capture.  All calls share the array: calls that overlap on the GPU (other streams, other host
 * threads) race, so serialize them.  objective / delta as in dyngb200_options; stream: a
 * cudaStream_t or NULL.  The results equal dyngb200_sssp_compute's. */
dyngb200_status dyngb200_sssp_compute_static_scratch(dyngb200_graph g, int32_t source,
                                                     int32_t objective, int64_t delta,
                                                     int64_t* distances, int32_t* parents,
                                                     void* stream);

/* ---- the learned scheduler (no reference counterpart) --------------------------------------
 * A 12 -> 64 -> 64 -> 15 MLP with bf16 weights and activations and fp32 accumulation.  Its three
 * softmax heads pick the schedule of one update: the near-far width class (8 classes: the
 * automatic width times 4^(c - 2)), the invalidation / small-frontier class (4: pointer jumping
 * with the small-frontier switch at 256, pointer jumping without it, subtree walk at 256, subtree
 * walk without it) and the persistent-grid class (3: 1/4, 1/2, all of the occupancy grid).  The
 * features are computed on the device from the batch, the graph and the tree's record of its
 * previous update; the schedule never changes distances or parents.
 * Features (12, float): log2(1 + batch operations), insertion fraction, fraction of deletions
 * that remove a tree edge, log2(1 + mean / max out-degree of the batch's sources), log2(1 + n),
 * log2(1 + m / n), log2(1 + automatic width), and of the tree's previous update log2(1 + x) of:
 * invalidated vertices, first near-far frontier, largest of the next three, steps.
 * Labels: 3 int32 per sample (width, switch, grid class).  Parameters: dyngb200_scheduler_num_params
 * floats, W1[64x12] b1[64] W2[64x64] b2[64] W3[15x64] b3[15] (row-major, out x in); the feature
 * standardization (f - mean) * scale is applied on the device. */
#define DYNGB200_SCHED_FEATURES 12
#define DYNGB200_SCHED_OUTPUTS 15
int64_t dyngb200_scheduler_num_params(void);
dyngb200_status dyngb200_scheduler_create(dyngb200_context ctx, uint64_t seed,
                                          dyngb200_scheduler* out);
dyngb200_status dyngb200_scheduler_destroy(dyngb200_scheduler s);
/* NULL pointers leave that part unchanged; new parameters reset the optimizer state. */
dyngb200_status dyngb200_scheduler_set_params(dyngb200_context ctx, dyngb200_scheduler s,
                                              const float* params, const float* feature_mean,
                                              const float* feature_scale);
dyngb200_status dyngb200_scheduler_get_params(dyngb200_context ctx, dyngb200_scheduler s,
                                              float* params, float* feature_mean,
                                              float* feature_scale);
/* The raw feature range the scheduler was trained on (12 floats each; NULL, NULL: no range).
 * An update whose features fall outside it keeps the plain schedule (its stats report schedule
 * classes -2): the network never extrapolates. */
dyngb200_status dyngb200_scheduler_set_feature_range(dyngb200_scheduler s, const float* lo,
                                                     const float* hi);
dyngb200_status dyngb200_scheduler_get_feature_range(dyngb200_scheduler s, float* lo, float* hi,
                                                     int32_t* has_range);
/* Logits (n x 15, host) of raw feature rows (n x 12, host), by the device kernels. */
dyngb200_status dyngb200_scheduler_forward(dyngb200_context ctx, dyngb200_scheduler s,
                                           const float* features, int64_t n, float* logits);
/* Mean loss (cross-entropy summed over the heads) and its gradient over all n samples, without
 * a step; grads: num_params floats (host) or NULL. */
dyngb200_status dyngb200_scheduler_gradients(dyngb200_context ctx, dyngb200_scheduler s,
                                             const float* features, const int32_t* labels,
                                             int64_t n, float* grads, double* loss);
/* Minibatch Adam on the device over `epochs` seeded shuffles; final_loss: the mean loss of the
 * last pass. */
dyngb200_status dyngb200_scheduler_train(dyngb200_context ctx, dyngb200_scheduler s,
                                         const float* features, const int32_t* labels, int64_t n,
                                         int32_t epochs, int32_t batch_size, float learning_rate,
                                         uint64_t seed, double* final_loss);
/* sssp::update with the schedule the scheduler picks on the device for this batch (stats carry
 * the features and the chosen classes).  Results equal dyngb200_sssp_update's. */
dyngb200_status dyngb200_sssp_update_learned(dyngb200_context ctx, dyngb200_graph g,
                                             const dyngb200_batch* batch, dyngb200_tree tree,
                                             dyngb200_scheduler scheduler, dyngb200_stats* stats);

/* ---- the serving loop (no reference counterpart) ----------------------------------------------
 * Several graphs resident on one GPU, each with its shortest-path tree, updated by batches that
 * arrive at any time from any host thread.  One dispatcher thread runs the updates: the batches
 * of one graph apply in arrival order (each result equals running the same batches alone, in
 * order); each round queues the oldest small batch of every waiting graph on one stream and waits
 * once (continuous batching); a batch larger than small_changes runs in a round of its own.
 * Admission: a graph is registered only if its workspace fits beside hbm_reserve_bytes of free
 * device memory, a batch is dispatched only if its scratch estimate fits beyond that reserve
 * (else its wait returns OUT_OF_MEMORY).  Registered graphs and trees belong to the server until
 * it is destroyed: do not use them elsewhere meanwhile. */
typedef struct dyngb200_server_s* dyngb200_server;
typedef struct dyngb200_server_config {
  int32_t device;
  int32_t max_group;         /* updates queued before one wait (0: 8) */
  int64_t small_changes;     /* batches up to this many changes share a round (0: 65536) */
  int64_t hbm_reserve_bytes; /* device memory admission keeps free (0: 1 GiB) */
  int32_t lanes;             /* 0 or 2: large batches run on their own lane, on two thirds of the
                                SMs' block slots, beside rounds of small ones on the rest;
                                1: one lane (a large batch holds every SM while it runs);
                                3..8: lanes - 1 small lanes share the rest in fixed parts, so
                                small batches of different graphs run side by side (the large
                                lane is lane lanes - 1) */
} dyngb200_server_config;
typedef struct dyngb200_request_times {
  double queued_ms;   /* submit -> dispatch */
  double service_ms;  /* dispatch -> result */
  double total_ms;    /* submit -> result */
  int32_t group_size; /* updates in the request's round */
  double begin_ms;    /* host time queuing this update's work (staging, launches) */
  double round_ms;    /* dispatch -> the round's work complete on the GPU */
  double copy_ms;     /* inside submit: the batch copied into the server's pinned buffer */
  int32_t lane;       /* 0: a round of small batches (or every round with one lane); 1: large */
} dyngb200_request_times;
typedef struct dyngb200_server_info {
  int64_t submitted;
  int64_t completed;
  int64_t failed;
  int64_t rounds;
  int64_t max_group;
  int64_t waiting;
  int64_t admission_us_max; /* longest free-memory query (a helper thread's), microseconds */
  int64_t lanes;            /* lanes in use (2 once a graph shows the GPU holds the split) */
  int64_t large_rounds;     /* rounds of the large lane */
} dyngb200_server_info;
/* learned: a scheduler used for every update (NULL: the fixed heuristic). */
dyngb200_status dyngb200_server_create(const dyngb200_server_config* config,
                                       dyngb200_scheduler learned, dyngb200_server* out);
dyngb200_status dyngb200_server_add_graph(dyngb200_server s, dyngb200_graph g, dyngb200_tree t,
                                          int32_t* slot);
/* The batch is copied (its arrays may be reused when the call returns); memory: any space. */
dyngb200_status dyngb200_server_submit(dyngb200_server s, int32_t slot,
                                       const dyngb200_batch* batch, uint64_t* ticket);
/* Blocks until the request is done; returns the update's own status (its message in
 * dyngb200_last_error_message).  Each ticket is waited for once; stats / times may be NULL. */
dyngb200_status dyngb200_server_wait(dyngb200_server s, uint64_t ticket, dyngb200_stats* stats,
                                     dyngb200_request_times* times);
dyngb200_status dyngb200_server_drain(dyngb200_server s);
dyngb200_status dyngb200_server_info_get(dyngb200_server s, dyngb200_server_info* info);
/* Finishes every submitted request, then stops the dispatcher. */
dyngb200_status dyngb200_server_destroy(dyngb200_server s);

/* ---- snapshots (recording scheduler traces: one batch under many schedules) ---------------- */
/* A new graph with g's contents (its own identity: trees of g are not bound to it). */
dyngb200_status dyngb200_graph_clone(dyngb200_context ctx, dyngb200_graph g, dyngb200_graph* out);
/* src's contents into dst, which keeps its identity (trees bound to dst stay bound). */
dyngb200_status dyngb200_graph_copy_from(dyngb200_context ctx, dyngb200_graph dst,
                                         dyngb200_graph src);
dyngb200_status dyngb200_tree_copy_from(dyngb200_context ctx, dyngb200_tree dst, dyngb200_tree src);

/* ---- tree: sssp::result (sssp.hpp:153-310) ------------------------------------------------ */
/* result::from_arrays (sssp.hpp:253-302): arrays in `memory`, n entries each. */
dyngb200_status dyngb200_tree_from_arrays(dyngb200_context ctx, dyngb200_graph g, int32_t source,
                                          const int64_t* distances, const int32_t* parents,
                                          int64_t n, int32_t memory, int32_t canonicalize,
                                          const dyngb200_options* opt, dyngb200_tree* out);
/* result::clone (sssp.hpp:245). */
dyngb200_status dyngb200_tree_clone(dyngb200_context ctx, dyngb200_tree t, dyngb200_tree* out);
dyngb200_status dyngb200_tree_destroy(dyngb200_tree t);
/* result::distances() / parents() copied into `dst` (n entries, in `memory`). */
dyngb200_status dyngb200_tree_distances(dyngb200_context ctx, dyngb200_tree t, int64_t* dst,
                                        int32_t memory);
dyngb200_status dyngb200_tree_parents(dyngb200_context ctx, dyngb200_tree t, int32_t* dst,
                                      int32_t memory);
/* The device arrays themselves (valid until the next update of t). */
dyngb200_status dyngb200_tree_device_arrays(dyngb200_tree t, const int64_t** distances,
                                            const int32_t** parents);
/* source(), num vertices, graph_version(), poisoned, get_options(). */
dyngb200_status dyngb200_tree_info(dyngb200_tree t, int32_t* source, int64_t* num_vertices,
                                   uint64_t* graph_version, int32_t* poisoned,
                                   dyngb200_options* opt);
/* result::set_options (sssp.hpp:214-222): objective must stay. */
dyngb200_status dyngb200_tree_set_options(dyngb200_tree t, const dyngb200_options* opt);

#ifdef __cplusplus
}
#endif

#endif /* DYNGB200_H */
