// Host-side objects of the dyng_b200 library: the execution context (resources::cuda()), the
// device-resident slack-row graph and the shortest-path tree.  Not part of the public ABI.
#pragma once

#include "common.cuh"

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/dyngb200.h"

namespace dyngb200 {

// A library error carrying the C-ABI status it maps to.
struct Error : std::runtime_error {
  dyngb200_status status;
  Error(dyngb200_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

#define DYNGB200_CUDA(call)                                                                     \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) {                                                                    \
      if (e_ == cudaErrorMemoryAllocation) {                                                    \
        cudaGetLastError();                                                                     \
        throw ::dyngb200::Error(DYNGB200_OUT_OF_MEMORY,                                         \
                                std::string("CUDA out of memory at ") + #call);                 \
      }                                                                                         \
      throw ::dyngb200::Error(DYNGB200_CUDA_ERROR, std::string(cudaGetErrorString(e_)) + " at " \
                                                       + #call);                               \
    }                                                                                           \
  } while (0)

inline void expects(bool ok, const std::string& msg,
                    dyngb200_status s = DYNGB200_INVALID_ARGUMENT) {
  if (!ok) throw Error(s, msg);
}

// memory.cu: device memory from a per-device pool that keeps freed memory (cudaMalloc /
// cudaFree semantics otherwise: a free waits for the device first).
void* device_alloc(size_t bytes, int* device);
void device_free(void* p, int device) noexcept;
void device_pool_reserve(size_t bytes);        // pre-fill the current device's pool
long long device_pool_idle_bytes(int device);  // pooled bytes not in use
long long device_alloc_count();                // device_alloc calls of this process so far
void device_alloc_fail_at(long long nth);      // the nth device_alloc from now fails (0: none)

// A device buffer that grows on demand (contents are not preserved unless asked).
template <typename T>
struct DevBuf {
  T* ptr = nullptr;
  size_t count = 0;
  int dev = 0;  // the device of ptr
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void swap(DevBuf& o) noexcept {
    std::swap(ptr, o.ptr);
    std::swap(count, o.count);
    std::swap(dev, o.dev);
  }
  void release() {
    if (ptr) device_free(ptr, dev);
    ptr = nullptr;
    count = 0;
  }
  // Ensure room for n elements; keeps the first `keep` elements when it reallocates.
  void reserve(size_t n, cudaStream_t stream = 0, size_t keep = 0) {
    if (n <= count) return;
    int d = 0;
    T* fresh = static_cast<T*>(device_alloc((n ? n : 1) * sizeof(T), &d));
    if (ptr && keep) {
      const cudaError_t e = cudaMemcpyAsync(fresh, ptr, keep * sizeof(T), cudaMemcpyDeviceToDevice,
                                            stream);
      const cudaError_t e2 = e == cudaSuccess ? cudaStreamSynchronize(stream) : e;
      if (e2 != cudaSuccess) {
        device_free(fresh, d);
        DYNGB200_CUDA(e2);
      }
    }
    if (ptr) device_free(ptr, dev);
    ptr = fresh;
    count = n;
    dev = d;
  }
};

// Pinned host buffer.
template <typename T>
struct HostBuf {
  T* ptr = nullptr;
  size_t count = 0;
  HostBuf() = default;
  HostBuf(const HostBuf&) = delete;
  HostBuf& operator=(const HostBuf&) = delete;
  ~HostBuf() {
    if (ptr) cudaFreeHost(ptr);
  }
  void reserve(size_t n) {
    if (n <= count) return;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    DYNGB200_CUDA(cudaMallocHost(&ptr, (n ? n : 1) * sizeof(T)));
    count = n;
  }
};

// The control block of one update, written by the kernels and read back once at the end.
struct UpdateCtl {
  unsigned error;
  int pad0;
  long long err_index;
  // Step 0 / applier
  long long n_old, n_after;
  long long batch_ins_max;  // largest insertion weight of the objective (at least 1)
  long long max_w;          // max(column max before the batch, batch_ins_max)
  long long delta;
  int pairs;
  int rows_out, rows_in;
  int chunks_out, chunks_in;
  int relocated_out, relocated_in;
  int pad1;
  u64 top_out, top_in;  // tentative arena tops
  u64 seg_top;          // append-order rows: segments reserved so far
  int committing;       // the applier passed its allocation step: the graph is being changed
  int applied;          // the applier finished: the graph holds the batch
  long long summary[8];  // apply_summary fields in dyngb200_apply_summary order
  // sssp
  int packing_bits;
  int repacked;
  u64 max_distance;
  int cand_count;       // light pull candidates
  int frontier_count;   // vertices the pull (or the head offers) improved
  int near_cnt[3];      // light near-frontier lists, triple-buffered counters
  int near_med_cnt[3];  // medium rows of the near frontier
  int walk_cnt[3];      // subtree-walk levels
  int walk_med_cnt[3];
  int cand_med_count;   // medium pull candidates
  int far_count, far2_count;
  u64 heavy_cnt[3];     // (slots << 40 | chunks) of the heavy near-frontier lists
  u64 walk_heavy[3];
  u64 pull_heavy;       // heavy pull candidates
  // push steps hand out medium rows and heavy chunks to warps through these cursors (per step,
  // triple-buffered like the list counters)
  int med_cursor[3];
  int pad_cursor;
  unsigned long long heavy_cursor[3];
  int touched_count;
  int active[3];
  int rounds;
  int iterations, epochs;
  int levels;
  long long pushes;
  long long invalidated;
  long long affected;
  u64 minimum;
  int changed;         // the batch holds a deleted or weight-increased edge
  int last_generation; // last stamp generation the kernel used
  // the schedule of this launch (0 fields: the heuristic); see dyngb200_schedule
  long long sched_delta;
  int sched_small;     // small-frontier size (0: off)
  int sched_walk;      // subtree-walk invalidation
  int sched_heavy;     // heavy-row threshold (0: 256)
  int active_blocks;   // persistent grid size (0: all launched blocks)
  // learned scheduler: feature accumulators (tree-edge deletions, degree sum, max degree,
  // touched sources) and the feature vector of this update
  long long feat_acc[4];
  float features[12];
  int sched_classes[3];  // the chosen class of each head (-1: no scheduler)
  int loop_state[6];   // near-far state handed from block 0 back to the grid
  long long loop_pushes;
  u64 loop_threshold;
  // work counters (algorithmic traffic) and phase timestamps of the sssp kernel
  long long work[32];
  unsigned long long phase_ns[8];
  // trace of the first 64 push iterations / epochs: (light count, heavy chunks, ns since start)
  int trace_n[64];
  int trace_h[64];
  unsigned trace_t[64];
  int trace_len;
  unsigned long long apply_ns[12];  // the applier kernel: start, then the end of each step
  unsigned pj_t[24];  // start of each pointer-jumping round (ns since the kernel began)
  unsigned pj_done[24];  // the last block's arrival at the barrier ending each round
  // grid barrier: one arrival counter and the generation word the blocks wait on, each on its own
  // 128-byte line (the polling of the generation does not slow the arrivals)
  alignas(128) unsigned bar_count;
  alignas(128) unsigned bar_gen;
  unsigned bar_err;  // the error word as the last arrival saw it (read after bar_gen moves)
  // progress of a block that works alone (the small-frontier loop of block 0): the blocks waiting
  // at a grid barrier meanwhile restart their time limit whenever it moves
  alignas(128) unsigned heartbeat;
};

// Persistent blocks the pointer-jumping survivor lists of the sssp kernel support.
constexpr int kPjMaxBlocks = 1024;

// Scratch memory of a context, sized on demand and reused (the reference's workspace pool).
struct Workspace {
  // applier
  DevBuf<u64> pair_key;
  DevBuf<int> pair_d, pair_t, pair_first, pair_last, pair_out_pos, pair_in_pos, pair_out_pos2,
      pair_in_pos2, pair_flags, pair_out_row, pair_in_row, pair_out_rank, pair_in_rank, pair_list;
  DevBuf<unsigned char> pair_inc;  // pairs x k weight-increase flags
  DevBuf<int> touch_out_stamp, touch_in_stamp, row_slot_out, row_slot_in;
  DevBuf<int> rows_out, rows_in;  // touched row ids
  DevBuf<int> row_dels_out, row_dels_in, row_apps_out, row_apps_in, row_reloc_out, row_reloc_in;
  DevBuf<unsigned> row_new_start_out, row_new_start_in;
  DevBuf<unsigned> row_append_at_out, row_append_at_in;  // first append slot of each touched row
  DevBuf<int> row_new_cap_out, row_new_cap_in, row_live_out, row_live_in;
  DevBuf<int> row_seg_offsets, row_seg;  // append order: appended pairs per row
  DevBuf<long long> col_ins_max, col_sum_delta, col_removed_at_max, col_written_max,
      col_written_at_max;
  // batch staging
  DevBuf<int32_t> b_ins_src, b_ins_dst, b_ins_w, b_del_src, b_del_dst;
  // sssp
  DevBuf<int> stamp, touch_stamp, flag, in_far, ancestor;
  DevBuf<int> pj_blk;  // per-block survivor counts of pointer jumping
  DevBuf<long long> batch_extrema;  // update_each: per-objective insertion weight range, max id
  DevBuf<int> candidates, frontier, near_a, near_b, far_a, far_b, heavy_a, heavy_b, pull_heavy,
      touched, cand_med, near_med_a, near_med_b;
  DevBuf<UpdateCtl> ctl;
  HostBuf<UpdateCtl> host_ctl;
  DevBuf<unsigned long long> op_counts;  // the operators engine's step counters
  HostBuf<unsigned long long> op_host;
  int generation = 0;     // stamp generations (sssp)
  int touch_generation = 0;  // row-touch generations (applier)
  long long n_sized = 0;
  long long pairs_sized = 0;
  long long pairs_active = 0;  // pair-table size of the current batch (<= pairs_sized)

  void reserve_vertices(long long n_cap, cudaStream_t s);
  void reserve_batch(long long ops, int k, cudaStream_t s);
  int next_generation(int count, cudaStream_t s);  // reserves `count` sssp generations
  int next_touch_generation(cudaStream_t s);
};

struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sm_count = 0;
  int coop_supported = 0;
  long long launches = 0;  // kernels this context has launched (reported per call in the stats)
  int update_blocks_per_sm = 0;
  int apply_blocks_per_sm = 0;
  int compute_blocks_per_sm = 0;
  // cap on the update's persistent grid (0: occupancy x SMs); the serving loop's lanes split the
  // SMs' block slots between two concurrent persistent kernels with it
  int max_update_blocks = 0;
  Workspace ws;
  // the learned scheduler's hook: when set, the next update runs with this schedule
  dyngb200_schedule schedule{};
  int schedule_set = 0;
  // test hooks (dyngb200_context_set_test_hooks): the grid barrier's time limit without progress
  // (0: kBarrierTimeoutNs), blocks every grid barrier waits for beyond the launched ones (they
  // never arrive: the barrier's wait runs out), and a device taken as one without cooperative launch
  long long test_barrier_timeout_ns = 0;
  int test_barrier_extra = 0;
  int test_barrier_kernel = 0;  // the phantom arrivals: 0 every kernel, 1 the applier, 2 sssp
  int test_no_cooperative = 0;
  // the timing events of an update (before the applier, between the kernels, after the sssp
  // kernel): created at the first update and reused (a context has one update in flight at a
  // time), destroyed with the context
  cudaEvent_t update_events[3] = {nullptr, nullptr, nullptr};
};

// The persistent kernels need cooperative launch; checked before anything of a call changes.
void require_cooperative(const Context& ctx);
// The engines (sssp.cpp:195-226 of the reference): the fused persistent kernels need cooperative
// launch; the operators engine (ordinary launches, the loop on the host) runs anywhere;
// `automatic` takes the fused engine where the device offers cooperative launch.
bool cooperative_available(const Context& ctx);
// Throws NOT_SUPPORTED for the fused engine on a device without cooperative launch (before
// anything changes); returns whether the call runs the operators engine.
bool select_engine(const Context& ctx, int requested);
// A graph an update left incomplete refuses further use.
struct Graph;
void require_intact(const Graph& g);

struct Graph {
  uint64_t id = 0;
  uint64_t version = 0;
  // an update stopped part-way through changing the graph (a grid barrier of the applier timed
  // out after its first change): the graph refuses further use
  bool broken = false;
  dyngb200_props props{};
  int k = 1;
  long long n = 0, m = 0;  // host mirrors after the last completed call
  long long n_cap = 0, arena_cap = 0;
  long long arena_growths = 0, compactions = 0, index_builds = 0;
  double grow_ms = 0, compact_ms = 0, index_ms = 0, maintenance_ms_max = 0;
  DevBuf<RowDesc> out_desc, in_desc;
  DevBuf<int32_t> out_cap, in_cap, out_dead, in_dead;
  DevBuf<int32_t> out_col, in_col;
  DevBuf<int32_t> out_w, in_w;
  DevBuf<GraphCounters> counters;
  DevBuf<ColumnStats> columns;
  DevBuf<u64> ekey;  // edge index (simple graphs)
  DevBuf<unsigned> eout, ein;
  long long ecap = 0;
  GraphCounters host_counters{};
  std::vector<ColumnStats> host_columns;
  // pinned landing area of the per-update read-back: the counters, then the column statistics
  // (both 8-byte aligned PODs; sized in ColumnStats units)
  HostBuf<ColumnStats> pinned;
  int device = 0;

  GraphView view() {
    // the kernels read rows with 16-byte loads: every weight column must start aligned
    expects(arena_cap % 4 == 0, "graph: the arena size is not a multiple of 4 slots",
            DYNGB200_INTERNAL);
    GraphView v{};
    v.out_desc = out_desc.ptr;
    v.out_cap = out_cap.ptr;
    v.out_dead = out_dead.ptr;
    v.out_col = out_col.ptr;
    v.out_w = out_w.ptr;
    v.in_desc = in_desc.ptr;
    v.in_cap = in_cap.ptr;
    v.in_dead = in_dead.ptr;
    v.in_col = in_col.ptr;
    v.in_w = in_w.ptr;
    v.arena_cap = arena_cap;
    v.n_cap = n_cap;
    v.k = k;
    v.sorted = props.sorted;
    v.allow_multi = props.allow_multi;
    v.counters = counters.ptr;
    v.columns = columns.ptr;
    v.ekey = ekey.ptr;
    v.eout = eout.ptr;
    v.ein = ein.ptr;
    v.emask = ecap - 1;
    return v;
  }
};

// What the last update of a tree looked like (the learned scheduler's history features),
// written by the sssp kernel on the device.
struct TreeHistory {
  long long invalidated;
  int frontier[4];  // sizes of the first four near-far steps
  int iterations;   // near-far iterations + epochs
  int rounds;       // pointer-jumping rounds
};

struct Tree {
  DevBuf<TreeHistory> hist;
  bool canonical = true;  // every parent is the lowest-id tight in-neighbour (compute, canonicalize)
  uint64_t graph_id = 0;
  uint64_t version = 0;
  int32_t source = 0;
  dyngb200_options opt{};
  long long n = 0, cap = 0;
  DevBuf<int64_t> dist;
  DevBuf<int32_t> parent;
  DevBuf<u64> packed;
  int packed_bits = -1;  // format of `packed` (-1: not valid, repack before use)
  bool trusted = true;   // built by compute() or validated: no parent cycle possible
  bool poisoned = false;
  int device = 0;
};

// The learned scheduler: a 12 -> 64 -> 64 -> 15 MLP (bf16 weights and activations, fp32
// accumulation), three softmax heads: near-far width class (8), invalidation / small-frontier
// switch class (4), persistent-grid class (3).
constexpr int kMlpIn = 12, kMlpHidden = 64, kMlpOut = 15;
constexpr int kMlpParams = kMlpHidden * kMlpIn + kMlpHidden + kMlpHidden * kMlpHidden + kMlpHidden +
                           kMlpOut * kMlpHidden + kMlpOut;
struct Scheduler {
  int device = 0;
  DevBuf<float> params;       // fp32 master weights
  DevBuf<uint16_t> wbf16;     // bf16 copies of W1, W2, W3 (biases stay fp32)
  DevBuf<float> grads, m, v;  // gradient and Adam moments
  DevBuf<float> x;            // training features
  DevBuf<int> y;              // training labels (3 per sample)
  DevBuf<int> idx;            // the shuffle of one training pass
  DevBuf<float> out;          // logits / losses
  DevBuf<double> loss;
  long long step = 0;
  float feat_mean[kMlpIn] = {};
  float feat_scale[kMlpIn] = {};  // features are standardized: (f - mean) * scale
  // the raw feature range it was trained on: an update whose features leave it keeps the plain
  // schedule (no extrapolation)
  float feat_lo[kMlpIn] = {};
  float feat_hi[kMlpIn] = {};
  bool has_range = false;
};

// mlp.cu
struct StagedBatch;
void scheduler_refresh(Scheduler& s, cudaStream_t st);  // bf16 copies from the master weights
void scheduler_init(Context& ctx, Scheduler& s, uint64_t seed);
void scheduler_set(Context& ctx, Scheduler& s, const float* params, const float* mean,
                   const float* scale);
void scheduler_get(Context& ctx, const Scheduler& s, float* params, float* mean, float* scale);
void scheduler_forward(Context& ctx, Scheduler& s, const float* x, long long n, float* logits);
void scheduler_gradients(Context& ctx, Scheduler& s, const float* x, const int32_t* y, long long n,
                         float* grads, double* loss);
void scheduler_train(Context& ctx, Scheduler& s, const float* x, const int32_t* y, long long n,
                     int epochs, int batch, float lr, uint64_t seed, double* final_loss);
// What the batch applier's first block needs to compute the batch features (and, with a
// scheduler, its schedule) into the control block (mlp_common.cuh)
struct InferArgs;
void learned_infer_args(Context& ctx, Tree& t, const Scheduler* sch, InferArgs* out);

// graph.cu
void graph_build(Context& ctx, Graph& g, long long n, const int64_t* row_ptr, const int32_t* col,
                 const int32_t* w_objective_major, long long m);
void graph_export(Context& ctx, Graph& g, int64_t* row_ptr, int32_t* col, int32_t* w,
                  int64_t* in_row_ptr, int32_t* in_col, int32_t* in_w);
void graph_grow(Context& ctx, Graph& g, long long need_n, long long need_arena_out,
                long long need_arena_in);
void graph_rescan_columns(Context& ctx, Graph& g);
void graph_index_build(Context& ctx, Graph& g, long long extra, long long min_cap = 0);
void graph_index_reserve(Context& ctx, Graph& g, long long inserts);
void graph_refresh_host(Context& ctx, Graph& g);
void graph_copy(Context& ctx, Graph& dst, const Graph& src);

// Launches the batch applier (Step 0 checks, grouping, matching, resolution, allocation and the
// mutation of the slack rows).  `objective` >= 0 also records the sssp change classification for
// that weight column; tree arrays are not touched.  Work is queued on ctx.stream.
struct StagedBatch {
  const int32_t* ins_src;
  const int32_t* ins_dst;
  const int32_t* ins_w;
  long long ni;
  const int32_t* del_src;
  const int32_t* del_dst;
  long long nd;
};
void apply_launch(Context& ctx, Graph& g, const StagedBatch& b, int objective,
                  long long delta_opt, const dyngb200_schedule* sched, Tree* tree = nullptr,
                  const Scheduler* learned = nullptr, bool stepped = false);
void schedule_into(const dyngb200_schedule& sched, UpdateCtl& init);
StagedBatch stage_batch(Context& ctx, const dyngb200_batch& batch, int k);

// sssp.cu
void sssp_compute(Context& ctx, Graph& g, Tree& t, dyngb200_stats* st);
void sssp_update(Context& ctx, Graph& g, Tree& t, const dyngb200_batch& batch,
                 const dyngb200_schedule& sched, dyngb200_stats* st,
                 const Scheduler* learned = nullptr);
// An update split in two for callers that queue several updates (of different graphs, each with
// its own context) on one stream before waiting: begin() stages the batch and queues the work,
// end() waits, retries on capacity and fills the stats.
struct PendingUpdate {
  Context* ctx = nullptr;
  Graph* g = nullptr;
  Tree* t = nullptr;
  dyngb200_schedule sched{};
  const Scheduler* learned = nullptr;
  StagedBatch b{};
  int blocks = 0;
  bool operators = false;  // the operators engine (ordinary launches, the loop on the host)
  long long launches0 = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;  // the context's update events
  double host_us[4] = {};  // see dyngb200_stats::host_us
  PendingUpdate() = default;
  PendingUpdate(const PendingUpdate&) = delete;
  PendingUpdate& operator=(const PendingUpdate&) = delete;
  ~PendingUpdate();
};
void sssp_update_begin(Context& ctx, Graph& g, Tree& t, const dyngb200_batch& batch,
                       const dyngb200_schedule& sched, const Scheduler* learned,
                       PendingUpdate& u);
void sssp_update_end(PendingUpdate& u, dyngb200_stats* st);
// The update's persistent kernel: blocks an SM holds at once, and the grid an update launches
// (occupancy x SMs, or Context::max_update_blocks when smaller).
int update_blocks_per_sm(Context& ctx);
int update_grid_blocks(Context& ctx);
void sssp_update_each(Context& ctx, Graph& g, const dyngb200_batch& batch, Tree* const* trees,
                      int count, dyngb200_stats* stats);
void graph_apply(Context& ctx, Graph& g, const dyngb200_batch& batch,
                 dyngb200_apply_summary* summary, unsigned char* weight_increased);
void tree_reserve(Context& ctx, Tree& t, long long n_cap);
void tree_repack(Context& ctx, Tree& t, int bits);
void tree_canonicalize(Context& ctx, Graph& g, Tree& t);
void tree_copy(Context& ctx, Tree& dst, const Tree& src);
void sssp_compute_static(Graph& g, int32_t source, int objective, long long delta,
                         int64_t* distances, int32_t* parents, cudaStream_t s);

}  // namespace dyngb200
