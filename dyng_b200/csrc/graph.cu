// The device-resident slack-row graph and the batch applier.
//
// Layout in HBM (one graph):
//   out_desc[v] = {start, len}   slack row of v in the out arena (len counts tombstones)
//   out_cap[v], out_dead[v]      slots owned by the row, tombstones inside it
//   out_col[arena], out_w[k][arena]   neighbour ids and k weight columns (objective-major);
//                                      rows start on 16-byte boundaries (multiples of 4 slots)
//   in_*                          the same for the in-edge mirror (source ids)
// A deleted edge becomes a tombstone (column -1) in both rows; insertions append after the last
// slot.  A row that runs out of slots moves to the top of its arena, compacted, with new slack.
// Row order is the order of the reference's compact rows under row_order::append; under
// row_order::sorted the export sorts (the sssp kernels do not depend on the order).
//
// The applier reproduces apply_batch_host (reference cpp/src/graph/apply_host.cpp:57-395):
// Step 0 (self-loops, vertex growth, undirected expansion), deletions of the first alive match,
// upserts of the first alive match or appends, and the weight-increase classification
// (apply_host.cpp:348-393) -- restated per (u, v) pair: every outcome of a pair depends only on
// its number of existing matches c, its deletions d and insertions t and the first / last
// insertion, so the pairs are grouped by a hash table instead of rebuilding rows in batch order.
#include "internal.hpp"
#include "grid_sync.cuh"
#include "mlp_common.cuh"
#include "scan.cuh"


#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>

namespace dyngb200 {

namespace {

constexpr u64 kEmptyKey = ~0ULL;
constexpr int kBlock = 256;

__device__ __forceinline__ u64 pair_key(int32_t u, int32_t v) {
  return (static_cast<u64>(static_cast<uint32_t>(u)) << 32) | static_cast<uint32_t>(v);
}

// Per-thread column statistics deltas of weight column 0, in registers (the other columns go to
// the global counters directly); flushed once per warp at the end of a step.  Scalars, not
// arrays indexed by the column: every thread of the persistent grid carries them, and an array
// indexed at run time would live in local memory.
struct ColumnAcc {
  long long sum;
  long long removed_at_max;
  long long written_max;
  long long written_at_max;
  int bad;
};

struct ApplyParams {
  GraphView g;
  const int32_t* ins_src;
  const int32_t* ins_dst;
  const int32_t* ins_w;
  long long ni;
  const int32_t* del_src;
  const int32_t* del_dst;
  long long nd;
  int k;
  int objective;
  dyngb200_props props;
  long long delta_opt;
  // pair table
  u64* key;
  int mask;
  int* d;
  int* t;
  int* first;
  int* last;
  int* out_pos;
  int* in_pos;
  int* out_pos2;
  int* in_pos2;
  int* flags;
  int* out_rank;
  int* in_rank;
  int* out_count;  // matches in the out row (multi-edge graphs)
  int* in_count;
  int* list;
  unsigned char* inc;
  // touched rows
  int* touch_out_stamp;
  int* touch_in_stamp;
  int* row_slot_out;
  int* row_slot_in;
  int touch_gen;
  int* rows_out;
  int* rows_in;
  int* dels_out;
  int* dels_in;
  int* apps_out;
  int* apps_in;
  int* reloc_out;
  int* reloc_in;
  unsigned* new_start_out;
  unsigned* new_start_in;
  unsigned* append_at_out;  // the arena slot of the row's first appended edge
  unsigned* append_at_in;
  int* new_cap_out;
  int* new_cap_in;
  int* live_out;
  int* live_in;
  // column statistics deltas (k entries each)
  long long* col_sum_delta;
  long long* col_removed_at_max;
  long long* col_written_max;
  long long* col_written_at_max;
  UpdateCtl* ctl;
  // append-order rows: each touched out row's segment and the pairs appended to it, in order
  int* seg_offsets;
  int* seg;
  // the learned scheduler's batch features, accumulated by k_validate when `feat` is set: the
  // tree the update repairs (parent array, its vertex count)
  const int32_t* feat_parent;
  long long feat_tree_n;
  int feat;
};

// Pair flags.
enum : int {
  kPairDelete = 1,       // the batch deletes (u,v) at least once: a changed edge
  kPairIncreased = 2,    // the objective's weight of (u,v) increased: a changed edge
  kPairHead = 4,         // the batch inserts (u,v): v is an insertion head
  kPairAppend = 8,       // a new slot is appended to both rows
  kPairUpsert = 16,      // an existing slot receives the insertion's weights
  kPairUseFirst = 32,    // the first insertion's weights (ignore semantics), else the last's
};

__device__ __forceinline__ int find_pair(const ApplyParams& p, u64 k) {
  unsigned h = static_cast<unsigned>(mix64(k)) & static_cast<unsigned>(p.mask);
  for (int probe = 0; probe <= p.mask; ++probe) {
    const u64 cur = p.key[h];
    if (cur == k) return static_cast<int>(h);
    if (cur == kEmptyKey) return -1;
    h = (h + 1) & static_cast<unsigned>(p.mask);
  }
  return -1;
}

// ---- A: Step 0 checks, vertex growth, largest insertion weight --------------------------------
__device__ void ph_validate(const ApplyParams& p, BlockRed& R, long long tid, long long threads) {
  UpdateCtl* c = p.ctl;
  const long long total = p.ni + p.nd;
  const long long n = c->n_old;
  long long top = 0;
  long long wmax = 1;
  int dropped = 0;
  // scheduler features: tree-edge deletions, source out-degree sum / max / count
  long long f_tree = 0, f_deg = 0, f_max = 0, f_srcs = 0;
  for (long long i = tid; i < total; i += threads) {
    if (p.feat) {
      const bool del = i >= p.ni;
      const long long j = del ? i - p.ni : i;
      const int32_t u = del ? p.del_src[j] : p.ins_src[j];
      if (u >= 0 && u < n) {
        const long long deg = p.g.out_desc[u].len;
        f_deg += deg;
        f_max = deg > f_max ? deg : f_max;
        ++f_srcs;
      }
      if (del && p.feat_parent) {
        const int32_t v = p.del_dst[j];
        if (u >= 0 && v >= 0 && u < p.feat_tree_n && v < p.feat_tree_n &&
            (p.feat_parent[v] == u || (!p.props.directed && p.feat_parent[u] == v)))
          ++f_tree;
      }
    }
    if (i < p.ni) {
      const int32_t u = p.ins_src[i], v = p.ins_dst[i];
      if (p.objective >= 0) {
        const long long w = p.ins_w[i * p.k + p.objective];
        if (w < 1) {
          set_error(&c->error, kErrInvalidBatch);
          atomicMin(&c->err_index, i);
        }
        wmax = max(wmax, w);
      }
      if (u < 0 || v < 0 || (!p.props.allow_vertex_growth && (u >= n || v >= n)) ||
          u == INT32_MAX || v == INT32_MAX) {
        set_error(&c->error, kErrInvalidBatch);
        atomicMin(&c->err_index, i);
        continue;
      }
      if (u == v && p.props.on_self_loop != 0) {
        if (p.props.on_self_loop == 2) {
          set_error(&c->error, kErrInvalidBatch);
          atomicMin(&c->err_index, i);
        }
        ++dropped;
        continue;
      }
      top = max(top, static_cast<long long>(max(u, v)) + 1);
    } else {
      const long long j = i - p.ni;
      const int32_t u = p.del_src[j], v = p.del_dst[j];
      if (u < 0 || v < 0) {
        set_error(&c->error, kErrInvalidBatch);
        atomicMin(&c->err_index, p.ni + j);
        continue;
      }
      if (u == v && p.props.on_self_loop != 0) {
        if (p.props.on_self_loop == 2) {
          set_error(&c->error, kErrInvalidBatch);
          atomicMin(&c->err_index, p.ni + j);
        }
        ++dropped;
      }
    }
  }
  red_max(R, 0, top);
  red_max(R, 1, wmax);
  red_sum(R, 2, dropped);
  red_sum(R, 3, f_tree);
  red_sum(R, 4, f_deg);
  red_max(R, 5, f_max);
  red_sum(R, 6, f_srcs);
  __syncthreads();
  long long t;
  switch (threadIdx.x) {
    case 0: if ((t = red_maximum(R, 0, 0)) > 0) atomicMax(&c->n_after, t); break;
    case 1: if (p.objective >= 0 && (t = red_maximum(R, 1, 1)) > 1) atomicMax(&c->batch_ins_max, t); break;
    case 2: if ((t = red_total(R, 2)) != 0) atomicAdd(reinterpret_cast<unsigned long long*>(&c->summary[5]), static_cast<unsigned long long>(t)); break;
    case 3: if (p.feat && (t = red_total(R, 3)) != 0) atomicAdd(reinterpret_cast<unsigned long long*>(&c->feat_acc[0]), static_cast<unsigned long long>(t)); break;
    case 4: if (p.feat && (t = red_total(R, 4)) != 0) atomicAdd(reinterpret_cast<unsigned long long*>(&c->feat_acc[1]), static_cast<unsigned long long>(t)); break;
    case 5: if (p.feat && (t = red_maximum(R, 5, 0)) > 0) atomicMax(&c->feat_acc[2], t); break;
    case 6: if (p.feat && (t = red_total(R, 6)) != 0) atomicAdd(reinterpret_cast<unsigned long long*>(&c->feat_acc[3]), static_cast<unsigned long long>(t)); break;
    default: break;
  }
}

// ---- the per-batch reset: an empty pair table and zero column deltas ---------------------------
__device__ void ph_clear(const ApplyParams& p, long long tid, long long threads) {
  const long long cap = static_cast<long long>(p.mask) + 1;
  const int k = p.k > 0 ? p.k : 1;
  // every field a new pair starts from, written here by coalesced passes over the table rather
  // than by the thread that inserts the pair (one scattered 32-byte sector per field and pair)
  for (long long i = tid; i < cap; i += threads) {
    p.key[i] = ~0ULL;
    p.d[i] = 0;
    p.t[i] = 0;
    p.first[i] = 0x7f7f7f7f;
    p.last[i] = -1;
    p.out_pos[i] = -1;
    p.in_pos[i] = -1;
    p.out_pos2[i] = -1;
    p.in_pos2[i] = -1;
    p.out_count[i] = 0;
    p.in_count[i] = 0;
    if (i < k) {
      p.col_sum_delta[i] = 0;
      p.col_removed_at_max[i] = 0;
      p.col_written_max[i] = 0;
      p.col_written_at_max[i] = 0;
    }
  }
}

// ---- B: the plan (one thread): capacity, packing bound, near-far width ------------------------
__device__ void ph_plan(const ApplyParams& p) {
  UpdateCtl* c = p.ctl;
  const GraphCounters* gc = p.g.counters;
  c->n_after = max(c->n_after, c->n_old);
  if (c->n_after > p.g.n_cap) {
    set_error(&c->error, kErrCapacity);
  }
  c->top_out = gc->out_top;
  c->top_in = gc->in_top;
  if (p.objective >= 0) {
    const ColumnStats cs = p.g.columns[p.objective];
    c->max_w = max(cs.max_w, c->batch_ins_max);
    if (!distances_fit(c->n_after, c->max_w)) {
      set_error(&c->error, kErrInvalidBatch);
      c->err_index = -2;  // distances do not fit in 62 bits
    }
    const long long m = gc->m;
    c->delta = p.delta_opt > 0 ? p.delta_opt : default_delta(m > 1 ? m : 1, gc->n, cs.sum_w);
    u64 bound = 0;
    const Packing pk = choose_packing(c->n_after, c->max_w, &bound);
    c->packing_bits = pk.bits;
    c->max_distance = bound;
  }
}

// Block-staged list appends of k_pairs: new pairs and newly touched rows are collected in shared
// memory and copied to the global lists with one atomicAdd per block and list at the end of the
// kernel (a full stage falls back to direct global appends, warp-aggregated atomics on one
// counter per list).  3,072 entries per list (36 KB, 38 KB of shared memory per block with the
// reductions, three blocks per SM still resident) hold a 1M-change batch's new pairs and touched
// rows over 444 blocks; with 1,024 the overflow appends had made the pair step 2.6x slower there.
constexpr int kPairStageCap = 3072;
struct PairStage {
  int cnt[3];
  int base[3];
  int data[3][kPairStageCap];  // 0: pair slots, 1: out rows, 2: in rows
};

__device__ __forceinline__ void place_row(const ApplyParams& p, int side, int32_t r, int slot) {
  (side == 0 ? p.rows_out : p.rows_in)[slot] = r;
  (side == 0 ? p.row_slot_out : p.row_slot_in)[r] = slot;
  (side == 0 ? p.dels_out : p.dels_in)[slot] = 0;
  (side == 0 ? p.apps_out : p.apps_in)[slot] = 0;
}

__device__ __forceinline__ void stage_put(PairStage& st, const ApplyParams& p, int list, int v) {
  const int pos = atomicAdd(&st.cnt[list], 1);
  if (pos < kPairStageCap) {
    st.data[list][pos] = v;
    return;
  }
  UpdateCtl* c = p.ctl;
  if (list == 0) {
    p.list[append_slot(&c->pairs)] = v;
  } else {
    const int side = list - 1;
    place_row(p, side, v, append_slot(side == 0 ? &c->rows_out : &c->rows_in));
  }
}

__device__ void touch_row(PairStage& st, const ApplyParams& p, int side, int32_t r) {
  int* stamp = side == 0 ? p.touch_out_stamp : p.touch_in_stamp;
  if (atomicExch(&stamp[r], p.touch_gen) == p.touch_gen) return;
  stage_put(st, p, 1 + side, r);
}

__device__ void add_op(PairStage& st, const ApplyParams& p, int32_t u, int32_t v, int kind,
                       int index) {
  const u64 k = pair_key(u, v);
  unsigned h = static_cast<unsigned>(mix64(k)) & static_cast<unsigned>(p.mask);
  int slot = -1;
  for (int probe = 0; probe <= p.mask; ++probe) {
    const u64 prev = atomicCAS(&p.key[h], kEmptyKey, k);
    if (prev == kEmptyKey) {
      slot = static_cast<int>(h);  // its fields were set by the clear step
      stage_put(st, p, 0, slot);
      touch_row(st, p, 0, u);
      touch_row(st, p, 1, v);
      break;
    }
    if (prev == k) {
      slot = static_cast<int>(h);
      break;
    }
    h = (h + 1) & static_cast<unsigned>(p.mask);
  }
  if (slot < 0) {
    set_error(&p.ctl->error, kErrInternal);
    return;
  }
  if (kind == 0) {
    atomicAdd(&p.d[slot], 1);
  } else {
    atomicAdd(&p.t[slot], 1);
    atomicMin(&p.first[slot], index);
    atomicMax(&p.last[slot], index);
  }
}

// ---- C: group the effective operations by (u, v) pair ------------------------------------------
__device__ void ph_pairs(const ApplyParams& p, PairStage& st, BlockRed& R, long long tid, long long threads) {
  UpdateCtl* c = p.ctl;
  if (threadIdx.x < 3) st.cnt[threadIdx.x] = 0;
  __syncthreads();
  const long long total = p.ni + p.nd;
  const long long n_after = c->n_after;
  long long missing = 0;
  for (long long i = tid; i < total; i += threads) {
    if (i < p.ni) {
      const int32_t u = p.ins_src[i], v = p.ins_dst[i];
      if (u == v && p.props.on_self_loop != 0) continue;
      add_op(st, p, u, v, 1, static_cast<int>(i));
      if (!p.props.directed && u != v) add_op(st, p, v, u, 1, static_cast<int>(i));
    } else {
      const long long j = i - p.ni;
      const int32_t u = p.del_src[j], v = p.del_dst[j];
      if (u == v && p.props.on_self_loop != 0) continue;
      if (u >= n_after || v >= n_after) {
        missing += (!p.props.directed && u != v) ? 2 : 1;
        if (p.props.on_missing_delete == 1) {
          set_error(&c->error, kErrInvalidBatch);
          atomicMin(&c->err_index, p.ni + j);
        }
        continue;
      }
      add_op(st, p, u, v, 0, static_cast<int>(j));
      if (!p.props.directed && u != v) add_op(st, p, v, u, 0, static_cast<int>(j));
    }
  }
  red_sum(R, 0, missing);
  // flush the stages: one global atomic per list and block
  __syncthreads();
  if (threadIdx.x < 3) {
    const int n = min(st.cnt[threadIdx.x], kPairStageCap);
    int* counter = threadIdx.x == 0 ? &c->pairs : (threadIdx.x == 1 ? &c->rows_out : &c->rows_in);
    st.base[threadIdx.x] = n > 0 ? atomicAdd(counter, n) : 0;
  } else if (threadIdx.x == 3) {
    const long long t = red_total(R, 0);
    if (t != 0)
      atomicAdd(reinterpret_cast<unsigned long long*>(&c->summary[4]), static_cast<unsigned long long>(t));
  }
  __syncthreads();
  for (int list = 0; list < 3; ++list) {
    const int n = min(st.cnt[list], kPairStageCap);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int pos = st.base[list] + i;
      if (list == 0) p.list[pos] = st.data[0][i];
      else place_row(p, list - 1, st.data[list][i], pos);
    }
  }
}

// ---- D: match existing slots (simple graphs: at most one slot per pair, found in the edge
// index; positions are absolute arena slots) ------------------------------------------------------
__device__ void ph_match(const ApplyParams& p, long long tid, long long threads) {
  UpdateCtl* c = p.ctl;
  const int pairs = c->pairs;
  for (long long i = tid; i < pairs; i += threads) {
    const int slot = p.list[i];
    const long long e = index_find(p.g, p.key[slot]);
    if (e >= 0) {
      p.out_pos[slot] = static_cast<int>(p.g.eout[e]);
      p.in_pos[slot] = static_cast<int>(p.g.ein[e]);
      p.out_count[slot] = 1;
      p.in_count[slot] = 1;
    }
    p.in_pos2[slot] = static_cast<int>(e);  // index slot of the pair (or -1)
  }
}

// Multi-edge graphs: one thread per pair walks its rows in order (the first alive matches).
// Records c, the first match and the match the insertions address (see resolve).
__device__ void ph_scan_multi(const ApplyParams& p, long long tid, long long threads) {
  // one warp per pair: the lanes read a row 32 slots at a time, the matches ranked by a ballot
  UpdateCtl* c = p.ctl;
  const int pairs = c->pairs;
  const int lane = threadIdx.x & 31;
  for (long long i = tid >> 5; i < pairs; i += threads >> 5) {
    const int slot = p.list[i];
    const u64 key = p.key[slot];
    const int32_t u = static_cast<int32_t>(key >> 32), v = static_cast<int32_t>(key & 0xffffffffu);
    const int d = p.d[slot];
    for (int side = 0; side < 2; ++side) {
      const int32_t r = side == 0 ? u : v;
      const int32_t want = side == 0 ? v : u;
      if (r >= c->n_old) continue;
      const RowDesc desc = (side == 0 ? p.g.out_desc : p.g.in_desc)[r];
      const int32_t* col = (side == 0 ? p.g.out_col : p.g.in_col) + desc.start;
      // first match, and match number d (the first survivor of the deletions); absolute slots
      int count = 0, first = -1, target = -1;
      for (int base = 0; base < desc.len; base += 32) {
        const int e = base + lane;
        const unsigned ballot = __ballot_sync(0xffffffffu, e < desc.len && col[e] == want);
        if (ballot == 0) continue;
        if (first < 0) first = static_cast<int>(desc.start) + base + __ffs(ballot) - 1;
        const int found = __popc(ballot);
        if (target < 0 && d >= count && d < count + found) {
          unsigned rest = ballot;
          for (int k = d - count; k > 0; --k) rest &= rest - 1;  // drop the lower matches
          target = static_cast<int>(desc.start) + base + __ffs(rest) - 1;
        }
        count += found;
      }
      if (lane == 0) {
        if (side == 0) {
          p.out_count[slot] = count;
          p.out_pos[slot] = first;
          p.out_pos2[slot] = target;
        } else {
          p.in_count[slot] = count;
          p.in_pos[slot] = first;
          p.in_pos2[slot] = target;
        }
      }
    }
  }
}


// ---- E: resolve every pair (counts, policies, classification, per-row slot demand) -------------
__device__ void ph_resolve(const ApplyParams& p, BlockRed& R, long long tid, long long threads) {
  UpdateCtl* c = p.ctl;
  const int pairs = c->pairs;
  const bool del_first = p.props.deletions_first != 0;
  const int policy = p.props.on_existing_insert;
  long long acc[5] = {0, 0, 0, 0, 0};
  for (long long i = tid; i < pairs; i += threads) {
    const int slot = p.list[i];
    const u64 key = p.key[slot];
    const int32_t u = static_cast<int32_t>(key >> 32), v = static_cast<int32_t>(key & 0xffffffffu);
    const int d = p.d[slot];
    const int t = p.t[slot];
    const int cnt = p.out_count[slot];
    if (cnt != p.in_count[slot]) {
      set_error(&c->error, kErrInternal);  // the in-edge mirror disagrees with the out rows
      continue;
    }
    // Positions in storage: orig[0] is out_pos / in_pos; the addressed match (multi-edge graphs)
    // is out_pos2 / in_pos2 (simple graphs: cnt <= 1, so match 0 is the only one).
    const bool appended = t >= 1 && (del_first ? cnt <= d : cnt == 0);
    const int seq = cnt + (appended ? 1 : 0);  // S = original matches, then the appended slot
    const int removed = del_first ? min(cnt, d) : min(seq, d);
    // Which element of S receives the insertion's weights (-1 none).
    int target = -1;
    if (t >= 1) target = appended ? cnt : (del_first ? d : 0);
    const bool target_survives = target >= removed;
    int flags = 0;
    if (d > 0) flags |= kPairDelete;
    if (t > 0) flags |= kPairHead;
    long long inserted = 0, updated = 0, ignored_ins = 0;
    if (t >= 1) {
      if (appended) {
        inserted = 1;
        if (policy == 0) updated = t - 1;
        else if (policy == 2) ignored_ins = t - 1;
        else if (t > 1) set_error(&c->error, kErrInvalidBatch);
      } else {
        if (policy == 0) updated = t;
        else if (policy == 2) ignored_ins = t;
        else set_error(&c->error, kErrInvalidBatch);
      }
    }
    const long long deleted = removed;
    const long long ignored_del = d - removed;
    if (ignored_del > 0 && p.props.on_missing_delete == 1) set_error(&c->error, kErrInvalidBatch);
    const bool writes_weights = t >= 1 && (appended || policy == 0);
    const bool use_first = appended && policy == 2;
    if (appended && target_survives) flags |= kPairAppend;
    if (!appended && t >= 1 && policy == 0 && target_survives) flags |= kPairUpsert;
    if (use_first) flags |= kPairUseFirst;
    acc[0] += inserted;
    acc[1] += deleted;
    acc[2] += updated;
    acc[3] += ignored_ins;
    acc[4] += ignored_del;
    // Weight-increase classification (apply_host.cpp:348-393): first (u,v) before vs after.
    const int ins_index = use_first ? p.first[slot] : p.last[slot];
    const int final_idx = removed;  // S[removed] is the first (u,v) after the batch
    const bool final_exists = final_idx < seq;
    const bool orig_exists = cnt >= 1 && u < c->n_old;
    // storage position of S[final_idx] when it is an original slot (final_idx is 0 or d)
    int final_pos = -1;
    if (final_exists && final_idx < cnt) {
      final_pos = final_idx == 0 ? p.out_pos[slot] : p.out_pos2[slot];
    }
    for (int j = 0; j < p.k; ++j) {
      unsigned char inc = 0;
      if (orig_exists && final_exists) {
        const long long w0 = p.g.out_w[j * p.g.arena_cap + p.out_pos[slot]];
        long long wf;
        if (final_idx == target && writes_weights) {
          wf = p.ins_w[static_cast<long long>(ins_index) * p.k + j];
        } else {
          wf = p.g.out_w[j * p.g.arena_cap + final_pos];
        }
        inc = wf > w0 ? 1 : 0;
      }
      p.inc[static_cast<long long>(slot) * p.k + j] = inc;
      if (j == p.objective && inc) flags |= kPairIncreased;
    }
    p.flags[slot] = flags;
    // per-row demand: tombstones for removed originals, one slot per surviving append
    const int tomb = min(removed, cnt);
    const int app = (flags & kPairAppend) ? 1 : 0;
    if (tomb || app) {
      const int so = p.row_slot_out[u];
      const int si = p.row_slot_in[v];
      if (tomb) {
        atomicAdd(&p.dels_out[so], tomb);
        atomicAdd(&p.dels_in[si], tomb);
      }
      if (app) {
        p.out_rank[slot] = atomicAdd(&p.apps_out[so], 1);
        p.in_rank[slot] = atomicAdd(&p.apps_in[si], 1);
      }
    }
  }
  for (int f = 0; f < 5; ++f) red_sum(R, f, acc[f]);
  __syncthreads();
  if (threadIdx.x < 5) {
    const long long t = red_total(R, threadIdx.x);
    if (t != 0)
      atomicAdd(reinterpret_cast<unsigned long long*>(&c->summary[threadIdx.x]), static_cast<unsigned long long>(t));
  }
}

// Warp-wide reservation on a shared counter: every lane asks for `amount` (0: none), one atomic
// for the warp, each lane gets the start of its own range.  All 32 lanes must call.
__device__ __forceinline__ u64 warp_reserve(u64 amount, u64* counter) {
  const int lane = threadIdx.x & 31;
  u64 incl = amount;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u64 t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  const u64 total = __shfl_sync(0xffffffffu, incl, 31);
  u64 base = 0;
  if (lane == 31 && total > 0) base = atomicAdd(counter, total);
  base = __shfl_sync(0xffffffffu, base, 31);
  return base + incl - amount;
}

// ---- F: per touched row: stay in place or move to the top of the arena -------------------------
// A row that overflows its slack (or is mostly tombstones) gets a new place at the arena top.  The warps iterate together so that the arena
// space of a warp's relocated rows is reserved with one atomic per side.
__device__ void ph_alloc(const ApplyParams& p, BlockRed& R, long long tid, long long threads) {
  UpdateCtl* c = p.ctl;
  const int rows_out = c->rows_out, rows_in = c->rows_in;
  const int total = rows_out + rows_in;
  const double headroom = p.props.headroom;
  const int lane = threadIdx.x & 31;
  long long moved_out = 0, moved_in = 0;  // relocated rows (lane 0 of each warp counts)
  for (long long i0 = tid & ~31LL; i0 < total; i0 += threads) {
    const int i = i0 + lane;
    const bool active = i < total;
    const int side = i < rows_out ? 0 : 1;
    const int s = side == 0 ? i : i - rows_out;
    int reloc = 0, new_cap = 0, live = 0;
    unsigned start = 0, tail = 0;
    if (active) {
      const int32_t r = (side == 0 ? p.rows_out : p.rows_in)[s];
      const bool existing = r < c->n_old;
      const RowDesc desc = existing ? (side == 0 ? p.g.out_desc : p.g.in_desc)[r] : RowDesc{0, 0};
      const int cap = existing ? (side == 0 ? p.g.out_cap : p.g.in_cap)[r] : 0;
      const int dead = existing ? (side == 0 ? p.g.out_dead : p.g.in_dead)[r] : 0;
      const int dels = (side == 0 ? p.dels_out : p.dels_in)[s];
      const int apps = (side == 0 ? p.apps_out : p.apps_in)[s];
      live = desc.len - dead - dels;
      const int tomb = dead + dels;
      const bool compact = tomb > 8 && tomb * 4 > desc.len;
      start = desc.start;
      tail = desc.start + desc.len;
      new_cap = cap;
      if (desc.len + apps > cap || compact) {
        reloc = 1;
        const long long want = static_cast<long long>(live) + apps;
        long long extra = static_cast<long long>(ceil(static_cast<double>(want) * headroom));
        if (extra < 4) extra = 4;
        new_cap = static_cast<int>((want + extra + 3) & ~3LL);
      }
    }
    const u64 at_out = warp_reserve(reloc && side == 0 ? static_cast<u64>(new_cap) : 0, &c->top_out);
    const u64 at_in = warp_reserve(reloc && side == 1 ? static_cast<u64>(new_cap) : 0, &c->top_in);
    const unsigned n_out = __popc(__ballot_sync(0xffffffffu, reloc && side == 0));
    const unsigned n_in = __popc(__ballot_sync(0xffffffffu, reloc && side == 1));
    if (lane == 0) {
      moved_out += n_out;
      moved_in += n_in;
    }
    if (!active) continue;
    if (reloc) {
      const u64 at = side == 0 ? at_out : at_in;
      if (at + new_cap > static_cast<u64>(p.g.arena_cap) || at + new_cap > 0xffffffffULL) {
        set_error(&c->error, kErrCapacity);
      }
      start = static_cast<unsigned>(at);
      tail = start + live;
    }
    (side == 0 ? p.reloc_out : p.reloc_in)[s] = reloc;
    (side == 0 ? p.new_start_out : p.new_start_in)[s] = start;
    (side == 0 ? p.append_at_out : p.append_at_in)[s] = tail;
    (side == 0 ? p.new_cap_out : p.new_cap_in)[s] = new_cap;
    (side == 0 ? p.live_out : p.live_in)[s] = live;
  }
  red_sum(R, 0, moved_out);
  red_sum(R, 1, moved_in);
  __syncthreads();
  if (threadIdx.x < 2) {
    const long long t = red_total(R, threadIdx.x);
    if (t != 0) atomicAdd(threadIdx.x == 0 ? &c->relocated_out : &c->relocated_in, static_cast<int>(t));
  }
}

__device__ __forceinline__ void acc_init(ColumnAcc& a) {
  a.sum = a.removed_at_max = a.written_max = a.written_at_max = 0;
  a.bad = 0;
}
__device__ __forceinline__ void column_out(const ApplyParams& p, ColumnAcc& a, int j, long long w,
                                           long long old_max) {
  if (j == 0) {
    a.sum -= w;
    a.removed_at_max += w == old_max;
    a.bad -= w < 1;
    return;
  }
  atomicAdd(reinterpret_cast<unsigned long long*>(&p.col_sum_delta[j]),
            static_cast<unsigned long long>(-w));
  if (w == old_max) atomicAdd(reinterpret_cast<unsigned long long*>(&p.col_removed_at_max[j]), 1ULL);
  if (w < 1) atomicSub(&p.g.columns[j].bad, 1);
}
__device__ __forceinline__ void column_in(const ApplyParams& p, ColumnAcc& a, int j, long long w) {
  if (j == 0) {
    a.sum += w;
    a.written_max = max(a.written_max, w);
    a.bad += w < 1;
    return;
  }
  atomicAdd(reinterpret_cast<unsigned long long*>(&p.col_sum_delta[j]),
            static_cast<unsigned long long>(w));
  atomicMax(&p.col_written_max[j], w);
  if (w < 1) atomicAdd(&p.g.columns[j].bad, 1);
}
// The block's column-0 accumulators into reduction slots base .. base + 4 (all threads call).
__device__ __forceinline__ void acc_stage(BlockRed& R, const ColumnAcc& a, int base) {
  red_sum(R, base, a.sum);
  red_sum(R, base + 1, a.removed_at_max);
  red_max(R, base + 2, a.written_max);
  red_sum(R, base + 3, a.written_at_max);
  red_sum(R, base + 4, a.bad);
}
// After the barrier that follows acc_stage: thread `base + i` commits value i (one atomic per
// block and value).
__device__ __forceinline__ void acc_commit(const ApplyParams& p, const BlockRed& R, int base) {
  const int i = static_cast<int>(threadIdx.x) - base;
  if (i < 0 || i > 4) return;
  if (i == 2) {
    const long long t = red_maximum(R, base + 2, 0);
    if (t > 0) atomicMax(&p.col_written_max[0], t);
    return;
  }
  const long long t = red_total(R, base + i);
  if (t == 0) return;
  if (i == 4) {
    atomicAdd(&p.g.columns[0].bad, static_cast<int>(t));
    return;
  }
  long long* target = i == 0 ? &p.col_sum_delta[0]
                             : (i == 1 ? &p.col_removed_at_max[0] : &p.col_written_at_max[0]);
  atomicAdd(reinterpret_cast<unsigned long long*>(target), static_cast<unsigned long long>(t));
}
// A block's signed counter into one global atomic (called by the committing thread).
__device__ __forceinline__ void commit_add(long long t, long long* target) {
  if (t != 0) atomicAdd(reinterpret_cast<unsigned long long*>(target), static_cast<unsigned long long>(t));
}

// ---- G: tombstones and upserts in place -------------------------------------------------------
// Simple graphs: one thread per pair, the matching slots from the edge index.  Multigraphs: one
// warp per pair walking both rows in order (lanes over 32 slots at a time, the matches ranked by
// a ballot), so a hub row is read once, coalesced, instead of slot by slot by one thread.
__device__ void ph_mutate(const ApplyParams& p, BlockRed& R, long long tid, long long threads) {
  UpdateCtl* c = p.ctl;
  const int pairs = c->pairs;
  const bool del_first = p.props.deletions_first != 0;
  const bool multi = p.g.allow_multi != 0;
  const int lane = threadIdx.x & 31;
  ColumnAcc acc;
  acc_init(acc);
  long long idx_deleted = 0;
  const long long first_i = multi ? tid >> 5 : tid;
  const long long step = multi ? threads >> 5 : threads;
  for (long long i = first_i; i < pairs; i += step) {
    const int slot = p.list[i];
    const u64 key = p.key[slot];
    const int32_t u = static_cast<int32_t>(key >> 32), v = static_cast<int32_t>(key & 0xffffffffu);
    const int d = p.d[slot];
    const int t = p.t[slot];
    const int cnt = p.out_count[slot];
    const int flags = p.flags[slot];
    const bool appended = (flags & kPairAppend) || (t >= 1 && (del_first ? cnt <= d : cnt == 0));
    const int seq = cnt + (appended ? 1 : 0);
    const int removed = del_first ? min(cnt, d) : min(seq, d);
    const int tomb = min(removed, cnt);
    const int ins_index = (flags & kPairUseFirst) ? p.first[slot] : p.last[slot];
    if (!tomb && !(flags & kPairUpsert)) continue;
    const int target = del_first ? d : 0;  // the original match an upsert addresses
    if (!multi) {
      // simple graphs: the single matching slot, absolute positions from the edge index
      for (int side = 0; side < 2; ++side) {
        int32_t* col = side == 0 ? p.g.out_col : p.g.in_col;
        int32_t* w = side == 0 ? p.g.out_w : p.g.in_w;
        const int pos = side == 0 ? p.out_pos[slot] : p.in_pos[slot];
        if (tomb) {
          col[pos] = kDead;
          if (side == 0)
            for (int j = 0; j < p.k; ++j)
              column_out(p, acc, j, w[j * p.g.arena_cap + pos], p.g.columns[j].max_w);
        } else {
          for (int j = 0; j < p.k; ++j) {
            const long long nw = p.ins_w[static_cast<long long>(ins_index) * p.k + j];
            if (side == 0) {
              column_out(p, acc, j, w[j * p.g.arena_cap + pos], p.g.columns[j].max_w);
              column_in(p, acc, j, nw);
            }
            w[j * p.g.arena_cap + pos] = static_cast<int32_t>(nw);
          }
        }
      }
      if (tomb && !(flags & kPairAppend)) {
        // the edge is gone: its index key becomes a deleted marker
        p.g.ekey[p.in_pos2[slot]] = kKeyDeleted;
        ++idx_deleted;
      }
      continue;
    }
    for (int side = 0; side < 2; ++side) {
      const int32_t r = side == 0 ? u : v;
      const int32_t want = side == 0 ? v : u;
      const RowDesc desc = (side == 0 ? p.g.out_desc : p.g.in_desc)[r];
      int32_t* col = (side == 0 ? p.g.out_col : p.g.in_col) + desc.start;
      int32_t* w = (side == 0 ? p.g.out_w : p.g.in_w) + desc.start;
      // multi-edge graphs: the row in order, 32 slots per step; a match's rank is the number of
      // matches before it (the first `tomb` become tombstones, rank `target` takes the upsert)
      int seen = 0;
      for (int base = 0; base < desc.len && seen < cnt; base += 32) {
        const int e = base + lane;
        const bool match = e < desc.len && col[e] == want;
        const unsigned ballot = __ballot_sync(0xffffffffu, match);
        if (match) {
          const int rank = seen + __popc(ballot & ((1u << lane) - 1));
          if (rank < tomb) {
            col[e] = kDead;
            if (side == 0)
              for (int j = 0; j < p.k; ++j)
                column_out(p, acc, j, w[j * p.g.arena_cap + e], p.g.columns[j].max_w);
          } else if (rank < cnt && (flags & kPairUpsert) && rank == target) {
            for (int j = 0; j < p.k; ++j) {
              const long long nw = p.ins_w[static_cast<long long>(ins_index) * p.k + j];
              if (side == 0) {
                column_out(p, acc, j, w[j * p.g.arena_cap + e], p.g.columns[j].max_w);
                column_in(p, acc, j, nw);
              }
              w[j * p.g.arena_cap + e] = static_cast<int32_t>(nw);
            }
          }
        }
        seen += __popc(ballot);
      }
    }
  }
  acc_stage(R, acc, 0);
  red_sum(R, 5, idx_deleted);
  __syncthreads();
  acc_commit(p, R, 0);
  if (threadIdx.x == 5) {
    const long long t = red_total(R, 5);
    commit_add(-t, &p.g.counters->idx_live);
    commit_add(t, &p.g.counters->idx_dead);
  }
}

// ---- H: move relocated rows (live slots, in order) ---------------------------------------------
// A warp takes the touched rows 32 at a time, each lane reading one row's relocation flag and
// length; the warp then moves the flagged rows that hold slots one after another (lanes over the
// row's slots).  Most relocated rows are empty (a vertex without edges has no slack: its first
// edge relocates it, at R-MAT scale 22 about 70k rows per 100k-change batch), and they have
// nothing to move, so they take no warp step.
__device__ void ph_move(const ApplyParams& p, long long tid, long long threads) {
  UpdateCtl* c = p.ctl;
  const int lane = threadIdx.x & 31;
  const long long warp = tid >> 5;
  const long long warps = threads >> 5;
  const int rows_out = c->rows_out, rows_in = c->rows_in;
  const long long total = static_cast<long long>(rows_out) + rows_in;
  for (long long g0 = warp * 32; g0 < total; g0 += warps * 32) {
    const long long mine = g0 + lane;
    bool flagged = false;
    if (mine < total) {
      const int side = mine < rows_out ? 0 : 1;
      const int s = side == 0 ? static_cast<int>(mine) : static_cast<int>(mine - rows_out);
      const int32_t r = (side == 0 ? p.rows_out : p.rows_in)[s];
      if ((side == 0 ? p.reloc_out : p.reloc_in)[s] != 0 && r < c->n_old)
        flagged = (side == 0 ? p.g.out_desc : p.g.in_desc)[r].len > 0;
    }
    unsigned todo = __ballot_sync(0xffffffffu, flagged);
    while (todo) {
      const long long i = g0 + __ffs(todo) - 1;
      todo &= todo - 1;
      const int side = i < rows_out ? 0 : 1;
      const int s = side == 0 ? static_cast<int>(i) : static_cast<int>(i - rows_out);
      const int32_t r = (side == 0 ? p.rows_out : p.rows_in)[s];
      const RowDesc desc = (side == 0 ? p.g.out_desc : p.g.in_desc)[r];
      const unsigned dst = (side == 0 ? p.new_start_out : p.new_start_in)[s];
      int32_t* col = side == 0 ? p.g.out_col : p.g.in_col;
      int32_t* w = side == 0 ? p.g.out_w : p.g.in_w;
      int written = 0;
      for (int base = 0; base < desc.len; base += 32) {
        const int e = base + lane;
        const int32_t x = e < desc.len ? col[desc.start + e] : kDead;
        const bool live = x >= 0;
        const unsigned ballot = __ballot_sync(0xffffffffu, live);
        const int pos = written + __popc(ballot & ((1u << lane) - 1));
        if (live) {
          col[dst + pos] = x;
          for (int j = 0; j < p.k; ++j)
            w[j * p.g.arena_cap + dst + pos] = w[j * p.g.arena_cap + desc.start + e];
          if (!p.g.allow_multi) {
            const long long ie = index_find(p.g, side == 0 ? edge_key(r, x) : edge_key(x, r));
            if (ie >= 0) (side == 0 ? p.g.eout : p.g.ein)[ie] = dst + pos;
            else set_error(&c->error, kErrInternal);
          }
        }
        written += __popc(ballot);
      }
    }
  }
}

// ---- I: append the new slots ---------------------------------------------------------------------
__device__ void ph_append(const ApplyParams& p, BlockRed& R, long long tid, long long threads) {
  UpdateCtl* c = p.ctl;
  const int pairs = c->pairs;
  ColumnAcc acc;
  acc_init(acc);
  long long idx_new = 0, idx_reused = 0;
  for (long long i = tid; i < pairs; i += threads) {
    const int slot = p.list[i];
    const int flags = p.flags[slot];
    if (!(flags & kPairAppend)) continue;
    const u64 key = p.key[slot];
    const int32_t u = static_cast<int32_t>(key >> 32), v = static_cast<int32_t>(key & 0xffffffffu);
    const int ins_index = (flags & kPairUseFirst) ? p.first[slot] : p.last[slot];
    // both sides' loads first (they are independent), then the stores; the row's first append
    // slot (after its live slots if it moved, after its old length if not) was set by the alloc
    // step, so one scattered row field is read per side
    const int s0 = p.row_slot_out[u], s1 = p.row_slot_in[v];
    const int rk0 = p.out_rank[slot], rk1 = p.in_rank[slot];
    const unsigned placed[2] = {p.append_at_out[s0] + rk0, p.append_at_in[s1] + rk1};
    p.g.out_col[placed[0]] = v;
    p.g.in_col[placed[1]] = u;
    for (int j = 0; j < p.k; ++j) {
      const long long nw = p.ins_w[static_cast<long long>(ins_index) * p.k + j];
      p.g.out_w[j * p.g.arena_cap + placed[0]] = static_cast<int32_t>(nw);
      p.g.in_w[j * p.g.arena_cap + placed[1]] = static_cast<int32_t>(nw);
      column_in(p, acc, j, nw);
    }
    if (!p.g.allow_multi) {
      // the edge index follows the new slots (an edge deleted and re-inserted keeps its key)
      bool inserted = false, reused = false;
      const long long ie = index_find_or_insert(p.g, key, &inserted, &reused);
      if (ie < 0) {
        set_error(&c->error, kErrInternal);
        continue;
      }
      if (inserted) {
        ++idx_new;
        idx_reused += reused ? 1 : 0;
      }
      p.g.eout[ie] = placed[0];
      p.g.ein[ie] = placed[1];
    }
  }
  acc_stage(R, acc, 0);
  red_sum(R, 5, idx_new);
  red_sum(R, 6, idx_reused);
  __syncthreads();
  acc_commit(p, R, 0);
  if (threadIdx.x == 5) commit_add(red_total(R, 5), &p.g.counters->idx_live);
  if (threadIdx.x == 6) commit_add(-red_total(R, 6), &p.g.counters->idx_dead);
}

// ---- J: new row descriptors ----------------------------------------------------------------------
__device__ void ph_rows_final(const ApplyParams& p, BlockRed& R, long long tid, long long threads) {
  UpdateCtl* c = p.ctl;
  const int rows_out = c->rows_out, rows_in = c->rows_in;
  long long garbage_out = 0, garbage_in = 0, dead_delta_out = 0, dead_delta_in = 0;
  for (long long i = tid; i < rows_out + rows_in; i += threads) {
    const int side = i < rows_out ? 0 : 1;
    const int s = side == 0 ? i : i - rows_out;
    const int32_t r = (side == 0 ? p.rows_out : p.rows_in)[s];
    const bool existing = r < c->n_old;
    RowDesc* descs = side == 0 ? p.g.out_desc : p.g.in_desc;
    const RowDesc desc = existing ? descs[r] : RowDesc{0, 0};
    int* caps = side == 0 ? p.g.out_cap : p.g.in_cap;
    int* deads = side == 0 ? p.g.out_dead : p.g.in_dead;
    const int old_cap = existing ? caps[r] : 0;
    const int old_dead = existing ? deads[r] : 0;
    const int dels = (side == 0 ? p.dels_out : p.dels_in)[s];
    const int apps = (side == 0 ? p.apps_out : p.apps_in)[s];
    RowDesc nd;
    if ((side == 0 ? p.reloc_out : p.reloc_in)[s]) {
      nd.start = (side == 0 ? p.new_start_out : p.new_start_in)[s];
      nd.len = (side == 0 ? p.live_out : p.live_in)[s] + apps;
      caps[r] = (side == 0 ? p.new_cap_out : p.new_cap_in)[s];
      deads[r] = 0;
      (side == 0 ? garbage_out : garbage_in) += old_cap;
      (side == 0 ? dead_delta_out : dead_delta_in) -= old_dead;
    } else {
      nd.start = desc.start;
      nd.len = desc.len + apps;
      deads[r] = old_dead + dels;
      (side == 0 ? dead_delta_out : dead_delta_in) += dels;
    }
    descs[r] = nd;
  }
  GraphCounters* gc = p.g.counters;
  red_sum(R, 8, garbage_out);
  red_sum(R, 9, garbage_in);
  red_sum(R, 10, dead_delta_out);
  red_sum(R, 11, dead_delta_in);
  __syncthreads();
  if (threadIdx.x == 8 || threadIdx.x == 9) {
    const long long t = red_total(R, threadIdx.x);
    if (t != 0) atomicAdd(threadIdx.x == 8 ? &gc->out_garbage : &gc->in_garbage, static_cast<u64>(t));
  }
  if (threadIdx.x == 10) commit_add(red_total(R, 10), &gc->dead_out);
  if (threadIdx.x == 11) commit_add(red_total(R, 11), &gc->dead_in);
}

// Count the weights written by the batch that equal the new maximum (for count_at_max).
__device__ void ph_count_written_max(const ApplyParams& p, BlockRed& R, long long tid, long long threads) {
  UpdateCtl* c = p.ctl;
  const int pairs = c->pairs;
  ColumnAcc acc;
  acc_init(acc);
  for (long long i = tid; i < pairs; i += threads) {
    const int slot = p.list[i];
    const int flags = p.flags[slot];
    if (!(flags & (kPairAppend | kPairUpsert))) continue;
    const int ins_index = (flags & kPairUseFirst) ? p.first[slot] : p.last[slot];
    for (int j = 0; j < p.k; ++j) {
      const long long nw = p.ins_w[static_cast<long long>(ins_index) * p.k + j];
      const long long target = max(p.col_written_max[j], p.g.columns[j].max_w);
      if (nw == target) {
        if (j == 0) ++acc.written_at_max;
        else atomicAdd(reinterpret_cast<unsigned long long*>(&p.col_written_at_max[j]), 1ULL);
      }
    }
  }
  red_sum(R, 12, acc.written_at_max);
  __syncthreads();
  if (threadIdx.x == 12) commit_add(red_total(R, 12), &p.col_written_at_max[0]);
}

// One thread: graph counters and column statistics after the batch.
__device__ void ph_finalize(const ApplyParams& p) {
  UpdateCtl* c = p.ctl;
  GraphCounters* gc = p.g.counters;
  gc->n = c->n_after;
  gc->m += c->summary[0] - c->summary[1];
  gc->out_top = c->top_out;
  gc->in_top = c->top_in;
  c->summary[6] = c->n_after - c->n_old;
  c->summary[7] = c->n_after;
  c->applied = 1;
  for (int j = 0; j < p.k; ++j) {
    ColumnStats cs = p.g.columns[j];
    cs.sum_w += p.col_sum_delta[j];
    const long long wmax = p.col_written_max[j];
    if (wmax > cs.max_w) {
      cs.max_w = wmax;
      cs.count_at_max = p.col_written_at_max[j];
    } else {
      cs.count_at_max += p.col_written_at_max[j] - p.col_removed_at_max[j];
      if (cs.count_at_max <= 0) cs.dirty = 1;
    }
    if (gc->m == 0) {
      cs.max_w = 1;
      cs.count_at_max = 0;
      cs.sum_w = 0;
      cs.dirty = 0;
    }
    cs.bad = p.g.columns[j].bad;  // maintained by atomics during the mutation
    p.g.columns[j] = cs;
  }
}

// Column statistics by a full pass over the live slots (after a maximum edge was deleted): one
// warp per row, its lanes over the row's slots (coalesced; a hub row does not hold up a thread).
__global__ void k_rescan_columns(GraphView g, long long n, long long* out) {
  // out: per objective [max, count, sum]
  const int lane = threadIdx.x & 31;
  const long long warps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
  for (int j = 0; j < g.k; ++j) {
    long long mx = 0, sum = 0;
    for (long long v = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5; v < n;
         v += warps) {
      const RowDesc desc = g.out_desc[v];
      for (int e = lane; e < desc.len; e += 32) {
        if (g.out_col[desc.start + e] < 0) continue;
        const long long w = g.out_w[j * g.arena_cap + desc.start + e];
        mx = max(mx, w);
        sum += w;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    if (lane == 0) {
      if (mx > 0) atomicMax(&out[3 * j], mx);
      if (sum != 0)
        atomicAdd(reinterpret_cast<unsigned long long*>(&out[3 * j + 2]),
                  static_cast<unsigned long long>(sum));
    }
  }
}

__global__ void k_rescan_count(GraphView g, long long n, long long* out) {
  const int lane = threadIdx.x & 31;
  const long long warps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
  for (int j = 0; j < g.k; ++j) {
    const long long mx = out[3 * j];
    long long cnt = 0;
    for (long long v = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5; v < n;
         v += warps) {
      const RowDesc desc = g.out_desc[v];
      for (int e = lane; e < desc.len; e += 32) {
        if (g.out_col[desc.start + e] < 0) continue;
        cnt += g.out_w[j * g.arena_cap + desc.start + e] == mx;
      }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0 && cnt != 0)
      atomicAdd(reinterpret_cast<unsigned long long*>(&out[3 * j + 1]),
                static_cast<unsigned long long>(cnt));
  }
}

// Append order (row_order::append): the new slots of a row follow the batch order of their first
// insertion, as the reference appends them (apply_host.cpp:214-246).  The atomic ranks of
// k_resolve are replaced by the rank among the row's appended pairs ordered by first insertion.
// Append-order rows: a segment of the segment array per touched out row, sized by its appended
// pairs.  The segments only have to be disjoint (each row sorts its own), so a warp reserves its
// rows' segments with one atomic instead of a scan in row order.
__device__ void ph_row_offsets(const ApplyParams& p, int* offsets, long long tid, long long threads) {
  UpdateCtl* c = p.ctl;
  const int rows = c->rows_out;
  const int lane = threadIdx.x & 31;
  for (long long i0 = tid & ~31LL; i0 < rows; i0 += threads) {
    const long long i = i0 + lane;
    const u64 a = i < rows ? static_cast<u64>(p.apps_out[i]) : 0;
    const u64 at = warp_reserve(a, &c->seg_top);
    if (i < rows) offsets[i] = static_cast<int>(at);
  }
}

__device__ void ph_fill_segments(const ApplyParams& p, const int* offsets, int* seg, long long tid, long long threads) {
  UpdateCtl* c = p.ctl;
  const int pairs = c->pairs;
  for (long long i = tid; i < pairs; i += threads) {
    const int slot = p.list[i];
    if (!(p.flags[slot] & kPairAppend)) continue;
    const int32_t u = static_cast<int32_t>(p.key[slot] >> 32);
    seg[offsets[p.row_slot_out[u]] + p.out_rank[slot]] = slot;
  }
}

__device__ void ph_sort_segments(const ApplyParams& p, const int* offsets, int* seg, long long tid, long long threads) {
  UpdateCtl* c = p.ctl;
  const int rows = c->rows_out;
  for (long long s = tid; s < rows; s += threads) {
    const int a = p.apps_out[s];
    if (a <= 0) continue;
    int* base = seg + offsets[s];
    for (int i = 1; i < a; ++i) {
      const int x = base[i];
      const int key = p.first[x];
      int j = i - 1;
      while (j >= 0 && p.first[base[j]] > key) {
        base[j + 1] = base[j];
        --j;
      }
      base[j + 1] = x;
    }
    for (int i = 0; i < a; ++i) p.out_rank[base[i]] = i;
  }
}

// The classification per batch insertion (the weight-increase mask of apply_host.cpp:348-393):
// insertion i reads the flags of its pair (u, v).
__global__ void k_insert_flags(ApplyParams p, unsigned char* out) {
  UpdateCtl* c = p.ctl;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < p.ni;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int32_t u = p.ins_src[i], v = p.ins_dst[i];
    int slot = -1;
    if (!c->error && u >= 0 && v >= 0) slot = find_pair(p, pair_key(u, v));
    for (int j = 0; j < p.k; ++j)
      out[i * p.k + j] = slot >= 0 ? p.inc[static_cast<long long>(slot) * p.k + j] : 0;
  }
}

// Edge index construction: every live out-slot (u, x) inserts its key with the out position,
// then every live in-slot (v, y) records the in position of key (y, v).
__global__ void k_index_clear(GraphView g) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i <= g.emask;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    g.ekey[i] = kKeyEmpty;
}

// One warp per row, the lanes over its slots: hub rows (tens of thousands of slots in R-MAT
// graphs) do not serialise one thread.
__global__ void k_index_out(GraphView g, long long n, unsigned* error) {
  const int lane = threadIdx.x & 31;
  const long long warps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
  long long live = 0;
  for (long long u = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; u < n;
       u += warps) {
    const RowDesc d = g.out_desc[u];
    for (int e = lane; e < d.len; e += 32) {
      const int32_t x = g.out_col[d.start + e];
      if (x < 0) continue;
      bool reused = false;
      const long long ie = index_insert(g, edge_key(static_cast<int32_t>(u), x), &reused);
      if (ie < 0) {
        atomicOr(error, kErrCapacity);  // a full table: the build fails, no other walk needed
        return;
      }
      g.eout[ie] = d.start + e;
      ++live;
    }
  }
  if (live) atomicAdd(reinterpret_cast<unsigned long long*>(&g.counters->idx_live),
                      static_cast<unsigned long long>(live));
}

__global__ void k_index_in(GraphView g, long long n, unsigned* error) {
  const int lane = threadIdx.x & 31;
  const long long warps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
  for (long long v = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; v < n;
       v += warps) {
    const RowDesc d = g.in_desc[v];
    for (int e = lane; e < d.len; e += 32) {
      const int32_t y = g.in_col[d.start + e];
      if (y < 0) continue;
      const long long ie = index_find(g, edge_key(y, static_cast<int32_t>(v)));
      if (ie < 0) {
        atomicOr(error, kErrInternal);
        return;
      }
      g.ein[ie] = d.start + e;
    }
  }
}

// Compaction of one side, on the device: the live slots of every row (col >= 0), in storage
// order, packed into a fresh arena with new slack (slack_cap of the live length).  One warp per
// row; the row descriptors are rewritten in place by the warp that read them.
__device__ __forceinline__ long long row_slack(long long len, double headroom) {
  if (len <= 0) return 0;
  long long extra = static_cast<long long>(ceil(static_cast<double>(len) * headroom));
  if (extra < 4) extra = 4;
  return (len + extra + 3) & ~3LL;
}

__global__ void k_compact_count(const RowDesc* desc, const int32_t* col, long long n,
                                double headroom, long long* cap) {
  const int lane = threadIdx.x & 31;
  const long long warps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
  for (long long v = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; v < n;
       v += warps) {
    const RowDesc d = desc[v];
    int live = 0;
    for (int e = lane; e < d.len; e += 32) live += col[d.start + e] >= 0;
    for (int o = 16; o > 0; o >>= 1) live += __shfl_down_sync(0xffffffffu, live, o);
    if (lane == 0) cap[v] = row_slack(live, headroom);
  }
}

__global__ void k_compact_copy(RowDesc* desc, int32_t* cap_out, int32_t* dead,
                               const int32_t* col, const int32_t* w, long long old_arena,
                               const long long* start, int32_t* ncol, int32_t* nw,
                               long long new_arena, int k, long long n) {
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const long long warps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
  for (long long v = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; v < n;
       v += warps) {
    const RowDesc d = desc[v];
    const long long to = start[v];
    int at = 0;
    for (int e0 = 0; e0 < d.len; e0 += 32) {
      const int e = e0 + lane;
      const int32_t x = e < d.len ? col[d.start + e] : kDead;
      const unsigned live = __ballot_sync(0xffffffffu, x >= 0);
      if (x >= 0) {
        const long long dst = to + at + __popc(live & below);
        ncol[dst] = x;
        for (int j = 0; j < k; ++j)
          nw[j * new_arena + dst] = w[j * old_arena + d.start + e];
      }
      at += __popc(live);
    }
    __syncwarp();
    if (lane == 0) {
      desc[v] = RowDesc{static_cast<uint32_t>(to), at};
      cap_out[v] = static_cast<int32_t>(start[v + 1] - to);
      dead[v] = 0;
    }
  }
}

// ---- the applier as one cooperative persistent kernel -------------------------------------------
// Steps A-J of the batch applier (apply_host.cpp:57-395 restated per pair, above) in one launch:
// each step is a grid-stride pass of every block, and a grid barrier separates the steps that
// depend on one another (grid_sync.cuh).  Every block leaves a barrier with the same snapshot of
// the error word, so an error (an invalid batch, a capacity shortfall) stops all blocks at the same
// point, before anything of the graph changes: the steps that mutate the graph (G-J) run only after
// the allocation step found room for the whole batch.  Block 0 computes the plan and, for the
// learned scheduler, the batch features and the schedule while the other blocks group the pairs.
//
// The block footprint (256 threads, at most 80 registers by the launch bounds, the shared memory
// below) stays within the sssp kernel's, so the grids the serving loop's lanes size for the sssp
// kernel's block slots are co-resident for this kernel too.
struct ApplyLaunch {
  InferArgs infer;
  int infer_on;   // block 0 computes the batch features (and, with weights, the schedule)
  unsigned long long barrier_limit_ns;  // 0: kBarrierTimeoutNs
  int barrier_extra;                    // test hook: arrivals that never come (0 outside tests)
};

union ApplySmem {
  PairStage pairs;
  InferShared infer;
};

__global__ void __launch_bounds__(kBlock, 3) k_apply(ApplyParams p, ApplyLaunch L) {
  __shared__ ApplySmem sm;
  __shared__ BlockRed red;
  UpdateCtl* c = p.ctl;
  const long long tid = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  const long long threads = static_cast<long long>(gridDim.x) * blockDim.x;
  const unsigned arrivals = gridDim.x + static_cast<unsigned>(L.barrier_extra > 0 ? L.barrier_extra : 0);
  const unsigned long long limit = L.barrier_limit_ns > 0 ? L.barrier_limit_ns : kBarrierTimeoutNs;
  unsigned gen = gs_ld_volatile(&c->bar_gen);
  unsigned err = 0;
  // step timestamps (block 0's view): apply_ns[0] the start, then the end of each step
  int stamp = 0;
  auto mark = [&]() {
    ++stamp;
    if (tid == 0 && stamp < 12) c->apply_ns[stamp] = global_ns();
  };
  if (tid == 0) c->apply_ns[0] = global_ns();
  // A: Step 0 checks (and the scheduler's feature sums); this batch's pair table cleared
  ph_clear(p, tid, threads);
  ph_validate(p, red, tid, threads);
  if (!grid_sync(c, gen, arrivals, limit, &err)) return;
  mark();
  // B: the plan, then the features and schedule, by block 0
  if (blockIdx.x == 0) {
    if (threadIdx.x == 0) ph_plan(p);
    if (L.infer_on) {
      __syncthreads();
      infer_schedule_block(L.infer, c, p.g.counters, p.ni, p.nd, sm.infer);
    }
    __syncthreads();  // the pair stage below reuses the inference's shared memory
  }
  // an invalid batch or a vertex capacity shortfall ends the call here (nothing has changed; the
  // host reads the plan for the retry): every block decides on the same values
  if (err != 0 || max(c->n_after, c->n_old) > p.g.n_cap) return;
  // C: the operations grouped by (u, v) pair; while block 0 runs the inference the other blocks
  // share the pairs among themselves (the inference is then off the critical path)
  const long long skip = L.infer_on ? blockDim.x : 0;
  const long long ptid = (L.infer_on && blockIdx.x == 0) ? (1LL << 62) : tid - skip;
  ph_pairs(p, sm.pairs, red, ptid, threads - skip);
  if (!grid_sync(c, gen, arrivals, limit, &err) || err != 0) return;
  mark();
  // D: the live slot of each pair
  if (p.g.allow_multi) ph_scan_multi(p, tid, threads);
  else ph_match(p, tid, threads);
  if (!grid_sync(c, gen, arrivals, limit, &err) || err != 0) return;
  mark();
  // E: the outcome of each pair, its weight-increase class, the rows' demand
  ph_resolve(p, red, tid, threads);
  if (!grid_sync(c, gen, arrivals, limit, &err) || err != 0) return;
  mark();
  if (!p.props.sorted) {
    // append order: the order of the pairs appended to each row
    ph_row_offsets(p, p.seg_offsets, tid, threads);
    if (!grid_sync(c, gen, arrivals, limit, &err) || err != 0) return;
  mark();
    ph_fill_segments(p, p.seg_offsets, p.seg, tid, threads);
    if (!grid_sync(c, gen, arrivals, limit, &err) || err != 0) return;
  mark();
    ph_sort_segments(p, p.seg_offsets, p.seg, tid, threads);
    if (!grid_sync(c, gen, arrivals, limit, &err) || err != 0) return;
  mark();
  }
  // F: room for every touched row (the last point where an error leaves the graph untouched);
  // the barrier's last arrival records that the graph is about to change (any block past it
  // sees `committing` set, so a stop from here on is reported as leaving the graph incomplete)
  ph_alloc(p, red, tid, threads);
  if (!grid_sync(c, gen, arrivals, limit, &err, &c->committing) || err != 0) return;
  mark();
  // G: tombstones and upserts in place
  ph_mutate(p, red, tid, threads);
  if (!grid_sync(c, gen, arrivals, limit, &err) || err != 0) return;
  mark();
  // H, I: relocated rows moved and new slots appended (disjoint slots)
  ph_move(p, tid, threads);
  ph_append(p, red, tid, threads);
  if (!grid_sync(c, gen, arrivals, limit, &err) || err != 0) return;
  mark();
  // J: row descriptors, the written maxima, then counters and column statistics
  ph_rows_final(p, red, tid, threads);
  ph_count_written_max(p, red, tid, threads);
  if (!grid_sync(c, gen, arrivals, limit, &err) || err != 0) return;
  mark();
  if (tid == 0) {
    ph_finalize(p);
    c->apply_ns[11] = global_ns();
  }
}

// ---- the applier as ordinary launches, one per step ----------------------------------------------
// The same steps A-J for a device without cooperative launch and for the operators engine: the
// end of a launch stands in for each grid barrier.  Every launch but the first two starts by
// reading the error word and the capacity check of the plan, which all its blocks see alike (the
// previous launch has finished), so an error stops the sequence at the same step as the fused
// kernel's barrier snapshot does.  The plan (and the scheduler's inference) runs as a launch of
// one block; `mark` >= 0 records the end of the previous step in apply_ns[mark].
enum ApplyStep {
  kStepValidate, kStepPlan, kStepPairs, kStepMatch, kStepResolve, kStepRowOffsets,
  kStepFillSegments, kStepSortSegments, kStepAlloc, kStepMutate, kStepMove, kStepAppend,
  kStepRows, kStepFinalize
};

__global__ void __launch_bounds__(kBlock, 3) k_apply_step(ApplyParams p, ApplyLaunch L, int step,
                                                          int mark) {
  __shared__ ApplySmem sm;
  __shared__ BlockRed red;
  UpdateCtl* c = p.ctl;
  const long long tid = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  const long long threads = static_cast<long long>(gridDim.x) * blockDim.x;
  if (tid == 0 && mark >= 0 && mark < 12) c->apply_ns[mark] = global_ns();
  if (step == kStepValidate) {
    ph_clear(p, tid, threads);
    ph_validate(p, red, tid, threads);
    return;
  }
  if (step == kStepPlan) {
    if (threadIdx.x == 0) ph_plan(p);
    if (L.infer_on) {
      __syncthreads();
      infer_schedule_block(L.infer, c, p.g.counters, p.ni, p.nd, sm.infer);
    }
    return;
  }
  if (gs_ld_volatile(&c->error) != 0 || max(c->n_after, c->n_old) > p.g.n_cap) return;
  switch (step) {
    case kStepPairs: ph_pairs(p, sm.pairs, red, tid, threads); break;
    case kStepMatch:
      if (p.g.allow_multi) ph_scan_multi(p, tid, threads);
      else ph_match(p, tid, threads);
      break;
    case kStepResolve: ph_resolve(p, red, tid, threads); break;
    case kStepRowOffsets: ph_row_offsets(p, p.seg_offsets, tid, threads); break;
    case kStepFillSegments: ph_fill_segments(p, p.seg_offsets, p.seg, tid, threads); break;
    case kStepSortSegments: ph_sort_segments(p, p.seg_offsets, p.seg, tid, threads); break;
    case kStepAlloc: ph_alloc(p, red, tid, threads); break;
    case kStepMutate:
      // past the allocation step with no error: the graph is about to change
      if (tid == 0) c->committing = 1;
      ph_mutate(p, red, tid, threads);
      break;
    case kStepMove: ph_move(p, tid, threads); break;  // H and I touch disjoint slots
    case kStepAppend: ph_append(p, red, tid, threads); break;
    case kStepRows:
      ph_rows_final(p, red, tid, threads);
      ph_count_written_max(p, red, tid, threads);
      break;
    case kStepFinalize:
      if (tid == 0) {
        ph_finalize(p);
        c->apply_ns[11] = global_ns();
      }
      break;
    default: break;
  }
}

int grid_for(long long work, int block, int sm_count) {
  long long g = (work + block - 1) / block;
  const long long cap = static_cast<long long>(sm_count) * 8;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return static_cast<int>(g);
}

long long round4(long long x) { return (x + 3) & ~3LL; }

long long slack_cap(long long len, double headroom) {
  if (len <= 0) return 0;
  long long extra = static_cast<long long>(std::ceil(static_cast<double>(len) * headroom));
  if (extra < 4) extra = 4;
  return round4(len + extra);
}

ApplyParams make_params(Context& ctx, Graph& g, const StagedBatch& b, int objective,
                        long long delta_opt) {
  Workspace& ws = ctx.ws;
  ApplyParams p{};
  p.g = g.view();
  p.ins_src = b.ins_src;
  p.ins_dst = b.ins_dst;
  p.ins_w = b.ins_w;
  p.ni = b.ni;
  p.del_src = b.del_src;
  p.del_dst = b.del_dst;
  p.nd = b.nd;
  p.k = g.k;
  p.objective = objective;
  p.props = g.props;
  p.delta_opt = delta_opt;
  p.key = ws.pair_key.ptr;
  p.mask = static_cast<int>(ws.pairs_active - 1);
  p.d = ws.pair_d.ptr;
  p.t = ws.pair_t.ptr;
  p.first = ws.pair_first.ptr;
  p.last = ws.pair_last.ptr;
  p.out_pos = ws.pair_out_pos.ptr;
  p.in_pos = ws.pair_in_pos.ptr;
  p.out_pos2 = ws.pair_out_pos2.ptr;
  p.in_pos2 = ws.pair_in_pos2.ptr;
  p.flags = ws.pair_flags.ptr;
  p.out_rank = ws.pair_out_rank.ptr;
  p.in_rank = ws.pair_in_rank.ptr;
  p.out_count = ws.pair_out_row.ptr;
  p.in_count = ws.pair_in_row.ptr;
  p.list = ws.pair_list.ptr;
  p.inc = ws.pair_inc.ptr;
  p.touch_out_stamp = ws.touch_out_stamp.ptr;
  p.touch_in_stamp = ws.touch_in_stamp.ptr;
  p.row_slot_out = ws.row_slot_out.ptr;
  p.row_slot_in = ws.row_slot_in.ptr;
  p.rows_out = ws.rows_out.ptr;
  p.rows_in = ws.rows_in.ptr;
  p.dels_out = ws.row_dels_out.ptr;
  p.dels_in = ws.row_dels_in.ptr;
  p.apps_out = ws.row_apps_out.ptr;
  p.apps_in = ws.row_apps_in.ptr;
  p.reloc_out = ws.row_reloc_out.ptr;
  p.reloc_in = ws.row_reloc_in.ptr;
  p.new_start_out = ws.row_new_start_out.ptr;
  p.new_start_in = ws.row_new_start_in.ptr;
  p.append_at_out = ws.row_append_at_out.ptr;
  p.append_at_in = ws.row_append_at_in.ptr;
  p.new_cap_out = ws.row_new_cap_out.ptr;
  p.new_cap_in = ws.row_new_cap_in.ptr;
  p.live_out = ws.row_live_out.ptr;
  p.live_in = ws.row_live_in.ptr;
  p.col_sum_delta = ws.col_sum_delta.ptr;
  p.col_removed_at_max = ws.col_removed_at_max.ptr;
  p.col_written_max = ws.col_written_max.ptr;
  p.col_written_at_max = ws.col_written_at_max.ptr;
  p.ctl = ws.ctl.ptr;
  return p;
}

}  // namespace

// ------------------------------------------------------------------------------------------------
// Workspace
// ------------------------------------------------------------------------------------------------
void Workspace::reserve_vertices(long long n_cap, cudaStream_t s) {
  pj_blk.reserve(2 * kPjMaxBlocks, s);
  op_counts.reserve(8, s);
  op_host.reserve(8);
  if (n_cap <= n_sized) return;
  // buffers are released before they are reallocated: until every one is back, the workspace
  // counts as unsized (a failed allocation makes the next call start over, never skip)
  n_sized = 0;
  const size_t n = static_cast<size_t>(n_cap);
  for (DevBuf<int>* b : {&touch_out_stamp, &touch_in_stamp, &stamp, &touch_stamp}) {
    b->release();
    b->reserve(n, s);
    DYNGB200_CUDA(cudaMemsetAsync(b->ptr, 0, n * sizeof(int), s));
  }
  for (DevBuf<int>* b : {&flag, &in_far}) {
    b->release();
    b->reserve(n, s);
    DYNGB200_CUDA(cudaMemsetAsync(b->ptr, 0, n * sizeof(int), s));
  }
  for (DevBuf<int>* b : {&row_slot_out, &row_slot_in, &ancestor, &candidates, &frontier, &near_a,
                         &near_b, &far_a, &far_b, &touched, &cand_med, &near_med_a, &near_med_b}) {
    b->release();
    b->reserve(n, s);
  }
  for (DevBuf<int>* b : {&heavy_a, &heavy_b, &pull_heavy}) {  // int2 entries
    b->release();
    b->reserve(2 * n, s);
  }
  generation = 0;
  touch_generation = 0;
  n_sized = n_cap;
}

void Workspace::reserve_batch(long long ops, int k, cudaStream_t s) {
  // pair table: a power of two, at least twice the number of directed operations
  long long cap = 1024;
  while (cap < 2 * ops) cap <<= 1;
  if (cap > pairs_sized) {
    const size_t c = static_cast<size_t>(cap);
    pairs_sized = 0;  // unsized until every table is back (see reserve_vertices)
    pair_key.release();
    pair_key.reserve(c, s);
    for (DevBuf<int>* b : {&pair_d, &pair_t, &pair_first, &pair_last, &pair_out_pos, &pair_in_pos,
                           &pair_out_pos2, &pair_in_pos2, &pair_flags, &pair_out_row,
                           &pair_in_row, &pair_out_rank, &pair_in_rank, &pair_list}) {
      b->release();
      b->reserve(c, s);
    }
    for (DevBuf<int>* b : {&rows_out, &rows_in, &row_dels_out, &row_dels_in, &row_apps_out,
                           &row_apps_in, &row_reloc_out, &row_reloc_in, &row_new_cap_out,
                           &row_new_cap_in, &row_live_out, &row_live_in}) {
      b->release();
      b->reserve(c, s);
    }
    row_new_start_out.release();
    row_new_start_out.reserve(c, s);
    row_new_start_in.release();
    row_new_start_in.reserve(c, s);
    row_append_at_out.release();
    row_append_at_out.reserve(c, s);
    row_append_at_in.release();
    row_append_at_in.reserve(c, s);
    pairs_sized = cap;
  }
  pairs_active = cap;
  const size_t inc = static_cast<size_t>(pairs_sized) * static_cast<size_t>(k > 0 ? k : 1);
  pair_inc.reserve(inc, s);
  for (DevBuf<long long>* b : {&col_ins_max, &col_sum_delta, &col_removed_at_max,
                               &col_written_max, &col_written_at_max}) {
    b->reserve(static_cast<size_t>(k > 0 ? k : 1), s);
  }
  ctl.reserve(1, s);
  host_ctl.reserve(1);
}

int Workspace::next_generation(int count, cudaStream_t s) {
  if (generation > INT32_MAX / 2) {
    DYNGB200_CUDA(cudaMemsetAsync(stamp.ptr, 0, stamp.count * sizeof(int), s));
    DYNGB200_CUDA(cudaMemsetAsync(touch_stamp.ptr, 0, touch_stamp.count * sizeof(int), s));
    generation = 0;
  }
  const int g = generation + 1;
  generation += count;
  return g;
}

int Workspace::next_touch_generation(cudaStream_t s) {
  if (touch_generation > INT32_MAX / 2) {
    DYNGB200_CUDA(cudaMemsetAsync(touch_out_stamp.ptr, 0, touch_out_stamp.count * sizeof(int), s));
    DYNGB200_CUDA(cudaMemsetAsync(touch_in_stamp.ptr, 0, touch_in_stamp.count * sizeof(int), s));
    touch_generation = 0;
  }
  return ++touch_generation;
}

// ------------------------------------------------------------------------------------------------
// Build, export, growth
// ------------------------------------------------------------------------------------------------
namespace {

// Host layout of one side: row descriptors, caps, the arena (col + k weight columns).
struct HostSide {
  std::vector<RowDesc> desc;
  std::vector<int32_t> cap, dead;
  std::vector<int32_t> col;
  std::vector<int32_t> w;  // k x arena
  long long top = 0;
};

void layout_side(long long n, long long n_cap, int k, const int64_t* row_ptr, const int32_t* col,
                 const int32_t* w, long long m, double headroom, long long arena_cap,
                 HostSide& out) {
  out.desc.assign(static_cast<size_t>(n_cap), RowDesc{0, 0});
  out.cap.assign(static_cast<size_t>(n_cap), 0);
  out.dead.assign(static_cast<size_t>(n_cap), 0);
  long long top = 0;
  for (long long v = 0; v < n; ++v) {
    const long long len = row_ptr[v + 1] - row_ptr[v];
    const long long cap = slack_cap(len, headroom);
    out.desc[v] = RowDesc{static_cast<uint32_t>(top), static_cast<int32_t>(len)};
    out.cap[v] = static_cast<int32_t>(cap);
    top += cap;
  }
  out.top = top;
  out.col.assign(static_cast<size_t>(top), kDead);
  out.w.assign(static_cast<size_t>(top) * static_cast<size_t>(k), 0);
  for (long long v = 0; v < n; ++v) {
    const long long len = row_ptr[v + 1] - row_ptr[v];
    const long long s = out.desc[v].start;
    std::memcpy(&out.col[s], col + row_ptr[v], static_cast<size_t>(len) * sizeof(int32_t));
    for (int j = 0; j < k; ++j)
      std::memcpy(&out.w[static_cast<size_t>(j) * top + s], w + static_cast<size_t>(j) * m + row_ptr[v],
                  static_cast<size_t>(len) * sizeof(int32_t));
  }
  (void)arena_cap;
}

long long needed_top(long long n, const int64_t* row_ptr, double headroom) {
  long long top = 0;
  for (long long v = 0; v < n; ++v) top += slack_cap(row_ptr[v + 1] - row_ptr[v], headroom);
  return top;
}

void upload_side(Context& ctx, const HostSide& h, long long n_cap, long long arena_cap, int k,
                 DevBuf<RowDesc>& desc, DevBuf<int32_t>& cap, DevBuf<int32_t>& dead,
                 DevBuf<int32_t>& col, DevBuf<int32_t>& w) {
  cudaStream_t s = ctx.stream;
  desc.release();
  cap.release();
  dead.release();
  col.release();
  w.release();
  desc.reserve(static_cast<size_t>(n_cap));
  cap.reserve(static_cast<size_t>(n_cap));
  dead.reserve(static_cast<size_t>(n_cap));
  col.reserve(static_cast<size_t>(arena_cap));
  w.reserve(static_cast<size_t>(arena_cap) * static_cast<size_t>(k > 0 ? k : 1));
  DYNGB200_CUDA(cudaMemcpyAsync(desc.ptr, h.desc.data(), n_cap * sizeof(RowDesc),
                                cudaMemcpyHostToDevice, s));
  DYNGB200_CUDA(cudaMemcpyAsync(cap.ptr, h.cap.data(), n_cap * sizeof(int32_t),
                                cudaMemcpyHostToDevice, s));
  DYNGB200_CUDA(cudaMemcpyAsync(dead.ptr, h.dead.data(), n_cap * sizeof(int32_t),
                                cudaMemcpyHostToDevice, s));
  if (h.top > 0) {
    DYNGB200_CUDA(cudaMemcpyAsync(col.ptr, h.col.data(), h.top * sizeof(int32_t),
                                  cudaMemcpyHostToDevice, s));
    for (int j = 0; j < k; ++j)
      DYNGB200_CUDA(cudaMemcpyAsync(w.ptr + static_cast<size_t>(j) * arena_cap,
                                    h.w.data() + static_cast<size_t>(j) * h.top,
                                    h.top * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  }
  DYNGB200_CUDA(cudaStreamSynchronize(s));
}

// Transposition with the reference's order: inside an in-row the sources appear in out-edge
// order (apply_host.cpp:470-518).
void transpose_host(long long n, long long m, int k, const int64_t* row_ptr, const int32_t* col,
                    const int32_t* w, std::vector<int64_t>& irp, std::vector<int32_t>& icol,
                    std::vector<int32_t>& iw) {
  irp.assign(static_cast<size_t>(n) + 1, 0);
  for (long long e = 0; e < m; ++e) irp[static_cast<size_t>(col[e]) + 1]++;
  for (long long v = 0; v < n; ++v) irp[v + 1] += irp[v];
  icol.resize(static_cast<size_t>(m));
  iw.resize(static_cast<size_t>(m) * static_cast<size_t>(k));
  std::vector<int64_t> cursor(irp.begin(), irp.end() - 1);
  for (long long u = 0; u < n; ++u) {
    for (int64_t e = row_ptr[u]; e < row_ptr[u + 1]; ++e) {
      const int64_t pos = cursor[col[e]]++;
      icol[pos] = static_cast<int32_t>(u);
      for (int j = 0; j < k; ++j)
        iw[static_cast<size_t>(j) * m + pos] = w[static_cast<size_t>(j) * m + e];
    }
  }
}

}  // namespace

void graph_build(Context& ctx, Graph& g, long long n, const int64_t* row_ptr, const int32_t* col,
                 const int32_t* w, long long m) {
  const int k = g.k;
  const double headroom = g.props.headroom;
  std::vector<int64_t> irp;
  std::vector<int32_t> icol, iw;
  transpose_host(n, m, k, row_ptr, col, w, irp, icol, iw);
  const long long n_cap = n + 1024 + n / 16;
  const long long top_out = needed_top(n, row_ptr, headroom);
  const long long top_in = needed_top(n, irp.data(), headroom);
  long long arena = std::max(top_out, top_in);
  arena = round4(arena + std::max(arena / 2, 1LL << 16));
  expects(arena < 0xffffffffLL, "graph: the slack arena exceeds 2^32 slots", DYNGB200_CAPACITY);
  HostSide out, in;
  layout_side(n, n_cap, k, row_ptr, col, w, m, headroom, arena, out);
  layout_side(n, n_cap, k, irp.data(), icol.data(), iw.data(), m, headroom, arena, in);
  g.n = n;
  g.m = m;
  g.n_cap = n_cap;
  g.arena_cap = arena;
  upload_side(ctx, out, n_cap, arena, k, g.out_desc, g.out_cap, g.out_dead, g.out_col, g.out_w);
  upload_side(ctx, in, n_cap, arena, k, g.in_desc, g.in_cap, g.in_dead, g.in_col, g.in_w);
  GraphCounters gc{};
  gc.n = n;
  gc.m = m;
  gc.out_top = static_cast<u64>(out.top);
  gc.in_top = static_cast<u64>(in.top);
  g.counters.reserve(1);
  g.host_columns.assign(static_cast<size_t>(k > 0 ? k : 1), ColumnStats{1, 0, 0, 0, 0});
  for (int j = 0; j < k; ++j) {
    ColumnStats cs{1, 0, 0, 0, 0};
    long long mx = 0;
    for (long long e = 0; e < m; ++e) mx = std::max<long long>(mx, w[static_cast<size_t>(j) * m + e]);
    long long cnt = 0, sum = 0;
    for (long long e = 0; e < m; ++e) {
      const long long x = w[static_cast<size_t>(j) * m + e];
      sum += x;
      cnt += x == mx;
    }
    int bad = 0;
    for (long long e = 0; e < m; ++e) bad += w[static_cast<size_t>(j) * m + e] < 1;
    cs.max_w = m > 0 ? std::max<long long>(mx, 1) : 1;
    cs.count_at_max = m > 0 ? cnt : 0;
    cs.sum_w = sum;
    cs.bad = bad;
    g.host_columns[j] = cs;
  }
  g.columns.reserve(g.host_columns.size());
  DYNGB200_CUDA(cudaMemcpyAsync(g.counters.ptr, &gc, sizeof(gc), cudaMemcpyHostToDevice, ctx.stream));
  DYNGB200_CUDA(cudaMemcpyAsync(g.columns.ptr, g.host_columns.data(),
                                g.host_columns.size() * sizeof(ColumnStats),
                                cudaMemcpyHostToDevice, ctx.stream));
  DYNGB200_CUDA(cudaStreamSynchronize(ctx.stream));
  g.host_counters = gc;
  if (!g.props.allow_multi) graph_index_build(ctx, g, 0);
}

namespace {
// Host time of one storage maintenance step (growth, compaction, index build), added to the
// graph's totals when it ends.
struct MaintenanceTimer {
  Graph& g;
  double& total;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  MaintenanceTimer(Graph& graph, double& sum) : g(graph), total(sum) {}
  ~MaintenanceTimer() {
    const double ms = std::chrono::duration<double, std::milli>(
                          std::chrono::steady_clock::now() - t0).count();
    total += ms;
    g.maintenance_ms_max = std::max(g.maintenance_ms_max, ms);
  }
};
}  // namespace

// (Re)build the edge index with room for `extra` more edges and at least `min_cap` slots.
// Slots of an edge index for the graph's edges plus `extra` insertions (load <= 1/3 after the
// build), at least min_cap.  A rebuild comes when live plus deleted keys pass 60 %: with a third
// the graph can grow by 80 % of its edges before the next one (at R-MAT scale 22 a rebuild takes
// 60-85 ms; at a half, 1M-change batches met one every 15 batches).
static long long index_want(const Graph& g, long long extra, long long min_cap) {
  long long want = 1024;
  while (want < 3 * (g.host_counters.m + extra) + 65536 || want < min_cap) want <<= 1;
  return want;
}

void graph_index_build(Context& ctx, Graph& g, long long extra, long long min_cap) {
  MaintenanceTimer timer(g, g.index_ms);
  ++g.index_builds;
  cudaStream_t s = ctx.stream;
  Workspace& ws = ctx.ws;
  ws.ctl.reserve(1, s);  // before the index changes: every allocation comes first
  const long long want = index_want(g, extra, min_cap);
  if (want != g.ecap) {
    // the new arrays first: a failed allocation leaves the old index, whole, in place
    DevBuf<u64> key;
    DevBuf<unsigned> out, in;
    key.reserve(static_cast<size_t>(want));
    out.reserve(static_cast<size_t>(want));
    in.reserve(static_cast<size_t>(want));
    g.ekey.swap(key);
    g.eout.swap(out);
    g.ein.swap(in);
    g.ecap = want;
  }
  GraphCounters gc = g.host_counters;
  gc.idx_live = 0;
  gc.idx_dead = 0;
  DYNGB200_CUDA(cudaMemcpyAsync(g.counters.ptr, &gc, sizeof(gc), cudaMemcpyHostToDevice, s));
  DYNGB200_CUDA(cudaMemsetAsync(&ws.ctl.ptr->error, 0, sizeof(unsigned), s));
  GraphView v = g.view();
  const int grid = ctx.sm_count * 8;
  ctx.launches += 3;
  k_index_clear<<<grid, kBlock, 0, s>>>(v);
  k_index_out<<<grid, kBlock, 0, s>>>(v, gc.n, &ws.ctl.ptr->error);
  k_index_in<<<grid, kBlock, 0, s>>>(v, gc.n, &ws.ctl.ptr->error);
  DYNGB200_CUDA(cudaGetLastError());
  unsigned err = 0;
  DYNGB200_CUDA(cudaMemcpyAsync(&err, &ws.ctl.ptr->error, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  DYNGB200_CUDA(cudaMemcpyAsync(&g.host_counters, g.counters.ptr, sizeof(GraphCounters),
                                cudaMemcpyDeviceToHost, s));
  DYNGB200_CUDA(cudaStreamSynchronize(s));
  expects(err == 0, "graph: the edge index could not be built (duplicate edges?)", DYNGB200_INTERNAL);
}

// Before a batch of `inserts` insertions: rebuild the index when deleted markers or the batch
// would push it past 60% load.
void graph_index_reserve(Context& ctx, Graph& g, long long inserts) {
  if (g.props.allow_multi) return;
  const GraphCounters& gc = g.host_counters;
  if (static_cast<double>(gc.idx_live + gc.idx_dead + inserts) > 0.6 * static_cast<double>(g.ecap))
    graph_index_build(ctx, g, inserts);
}

void graph_refresh_host(Context& ctx, Graph& g) {
  DYNGB200_CUDA(cudaMemcpyAsync(&g.host_counters, g.counters.ptr, sizeof(GraphCounters),
                                cudaMemcpyDeviceToHost, ctx.stream));
  DYNGB200_CUDA(cudaMemcpyAsync(g.host_columns.data(), g.columns.ptr,
                                g.host_columns.size() * sizeof(ColumnStats),
                                cudaMemcpyDeviceToHost, ctx.stream));
  DYNGB200_CUDA(cudaStreamSynchronize(ctx.stream));
  g.n = g.host_counters.n;
  g.m = g.host_counters.m;
}

namespace {

// Download one side as raw slack rows.
void download_side(Context& ctx, Graph& g, int side, long long n, std::vector<RowDesc>& desc,
                   std::vector<int32_t>& col, std::vector<int32_t>& w, long long& top) {
  cudaStream_t s = ctx.stream;
  top = static_cast<long long>(side == 0 ? g.host_counters.out_top : g.host_counters.in_top);
  desc.resize(static_cast<size_t>(n));
  col.resize(static_cast<size_t>(top));
  w.resize(static_cast<size_t>(top) * static_cast<size_t>(g.k));
  DYNGB200_CUDA(cudaMemcpyAsync(desc.data(), (side == 0 ? g.out_desc : g.in_desc).ptr,
                                n * sizeof(RowDesc), cudaMemcpyDeviceToHost, s));
  if (top > 0) {
    DYNGB200_CUDA(cudaMemcpyAsync(col.data(), (side == 0 ? g.out_col : g.in_col).ptr,
                                  top * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    for (int j = 0; j < g.k; ++j)
      DYNGB200_CUDA(cudaMemcpyAsync(w.data() + static_cast<size_t>(j) * top,
                                    (side == 0 ? g.out_w : g.in_w).ptr +
                                        static_cast<size_t>(j) * g.arena_cap,
                                    top * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  }
  DYNGB200_CUDA(cudaStreamSynchronize(s));
}

// Compact CSR of one side: live slots per row, stably sorted by neighbour when `sort`.
void side_to_csr(long long n, int k, const std::vector<RowDesc>& desc,
                 const std::vector<int32_t>& col, const std::vector<int32_t>& w, long long top,
                 bool sort, std::vector<int64_t>& rp, std::vector<int32_t>& ocol,
                 std::vector<int32_t>& ow) {
  rp.assign(static_cast<size_t>(n) + 1, 0);
  for (long long v = 0; v < n; ++v) {
    long long live = 0;
    for (int e = 0; e < desc[v].len; ++e) live += col[desc[v].start + e] >= 0;
    rp[v + 1] = rp[v] + live;
  }
  const long long m = rp[n];
  ocol.resize(static_cast<size_t>(m));
  ow.resize(static_cast<size_t>(m) * static_cast<size_t>(k));
  std::vector<long long> idx;
  for (long long v = 0; v < n; ++v) {
    idx.clear();
    for (int e = 0; e < desc[v].len; ++e)
      if (col[desc[v].start + e] >= 0) idx.push_back(desc[v].start + e);
    if (sort)
      std::stable_sort(idx.begin(), idx.end(),
                       [&](long long a, long long b) { return col[a] < col[b]; });
    long long out = rp[v];
    for (long long e : idx) {
      ocol[out] = col[e];
      for (int j = 0; j < k; ++j)
        ow[static_cast<size_t>(j) * m + out] = w[static_cast<size_t>(j) * top + e];
      ++out;
    }
  }
}

}  // namespace

void graph_export(Context& ctx, Graph& g, int64_t* row_ptr, int32_t* col, int32_t* w,
                  int64_t* in_row_ptr, int32_t* in_col, int32_t* in_w) {
  require_intact(g);
  graph_refresh_host(ctx, g);
  const long long n = g.n;
  for (int side = 0; side < 2; ++side) {
    int64_t* rp_dst = side == 0 ? row_ptr : in_row_ptr;
    int32_t* col_dst = side == 0 ? col : in_col;
    int32_t* w_dst = side == 0 ? w : in_w;
    if (!rp_dst && !col_dst && !w_dst) continue;
    std::vector<RowDesc> desc;
    std::vector<int32_t> c, ww;
    long long top = 0;
    download_side(ctx, g, side, n, desc, c, ww, top);
    std::vector<int64_t> rp;
    std::vector<int32_t> oc, ow;
    // out rows: sorted by neighbour under row_order::sorted; in rows: always by source
    side_to_csr(n, g.k, desc, c, ww, top, side == 1 || g.props.sorted, rp, oc, ow);
    if (rp_dst) std::memcpy(rp_dst, rp.data(), rp.size() * sizeof(int64_t));
    if (col_dst) std::memcpy(col_dst, oc.data(), oc.size() * sizeof(int32_t));
    if (w_dst) std::memcpy(w_dst, ow.data(), ow.size() * sizeof(int32_t));
  }
}

// Compaction on the device: both sides packed into fresh arenas sized for the live slots plus
// the demand of the batch that ran out of room (need_* = the tops that batch reached), then the
// edge index rebuilt over the new slot positions.  Storage order inside every row is kept.
void graph_compact(Context& ctx, Graph& g, long long need_out, long long need_in) {
  MaintenanceTimer timer(g, g.compact_ms);
  cudaStream_t s = ctx.stream;
  const long long n = g.n;
  const int k = g.k > 0 ? g.k : 1;
  const int grid = ctx.sm_count * 8;
  DevBuf<long long> cap, start;
  cap.reserve(static_cast<size_t>(n) + 1);
  start.reserve(static_cast<size_t>(n) + 1);
  long long top[2] = {0, 0};
  DevBuf<long long> temp;
  temp.reserve(static_cast<size_t>(scan_scratch(n + 1)));
  const long long demand[2] = {
      std::max(0LL, need_out - static_cast<long long>(g.host_counters.out_top)),
      std::max(0LL, need_in - static_cast<long long>(g.host_counters.in_top))};
  // pass 1: the new tops of both sides decide the one arena size the sides share
  for (int side = 0; side < 2; ++side) {
    DYNGB200_CUDA(cudaMemsetAsync(cap.ptr + n, 0, sizeof(long long), s));
    ctx.launches += 1;
    k_compact_count<<<grid, kBlock, 0, s>>>((side == 0 ? g.out_desc : g.in_desc).ptr,
                                            (side == 0 ? g.out_col : g.in_col).ptr, n,
                                            g.props.headroom, cap.ptr);
    DYNGB200_CUDA(cudaGetLastError());
    ctx.launches += exclusive_scan(cap.ptr, start.ptr, n + 1, temp.ptr, s);
    DYNGB200_CUDA(cudaMemcpyAsync(&top[side], start.ptr + n, sizeof(long long),
                                  cudaMemcpyDeviceToHost, s));
    DYNGB200_CUDA(cudaStreamSynchronize(s));
  }
  long long base = std::max(top[0] + demand[0], top[1] + demand[1]);
  const long long arena = round4(base + std::max(base / 2, 1LL << 16));
  expects(arena < 0xffffffffLL, "graph: the slack arena exceeds 2^32 slots", DYNGB200_CAPACITY);
  // pass 2: the new arenas of both sides are allocated before either side's rows move (the row
  // descriptors are rewritten in place, and both sides share arena_cap): a failed allocation
  // leaves the graph as it was
  DevBuf<int32_t> ncol[2], nw[2];
  for (int side = 0; side < 2; ++side) {
    ncol[side].reserve(static_cast<size_t>(arena));
    nw[side].reserve(static_cast<size_t>(arena) * static_cast<size_t>(k));
  }
  // the edge index is rebuilt over the moved slots below: its arrays (when it grows) and the
  // control block are allocated now, so the rebuild cannot fail on an allocation after the
  // slots moved (the old index would point at other edges' slots)
  const long long index_cap = g.props.allow_multi ? g.ecap : index_want(g, 0, g.ecap);
  DevBuf<u64> ikey;
  DevBuf<unsigned> iout, iin;
  if (index_cap != g.ecap) {
    ikey.reserve(static_cast<size_t>(index_cap));
    iout.reserve(static_cast<size_t>(index_cap));
    iin.reserve(static_cast<size_t>(index_cap));
  }
  ctx.ws.ctl.reserve(1, s);
  for (int side = 0; side < 2; ++side) {
    DevBuf<int32_t>& col = side == 0 ? g.out_col : g.in_col;
    DevBuf<int32_t>& w = side == 0 ? g.out_w : g.in_w;
    RowDesc* desc = (side == 0 ? g.out_desc : g.in_desc).ptr;
    DYNGB200_CUDA(cudaMemsetAsync(cap.ptr + n, 0, sizeof(long long), s));
    ctx.launches += 2;
    k_compact_count<<<grid, kBlock, 0, s>>>(desc, col.ptr, n, g.props.headroom, cap.ptr);
    ctx.launches += exclusive_scan(cap.ptr, start.ptr, n + 1, temp.ptr, s);
    DYNGB200_CUDA(cudaMemsetAsync(ncol[side].ptr, 0xff,
                                  static_cast<size_t>(arena) * sizeof(int32_t), s));
    k_compact_copy<<<grid, kBlock, 0, s>>>(desc, (side == 0 ? g.out_cap : g.in_cap).ptr,
                                           (side == 0 ? g.out_dead : g.in_dead).ptr, col.ptr,
                                           w.ptr, g.arena_cap, start.ptr, ncol[side].ptr,
                                           nw[side].ptr, arena, g.k, n);
    DYNGB200_CUDA(cudaGetLastError());
  }
  DYNGB200_CUDA(cudaStreamSynchronize(s));
  g.out_col.swap(ncol[0]);
  g.out_w.swap(nw[0]);
  g.in_col.swap(ncol[1]);
  g.in_w.swap(nw[1]);
  g.arena_cap = arena;
  if (index_cap != g.ecap) {
    g.ekey.swap(ikey);
    g.eout.swap(iout);
    g.ein.swap(iin);
    g.ecap = index_cap;
  }
  ++g.compactions;
  GraphCounters& gc = g.host_counters;
  gc.out_top = static_cast<u64>(top[0]);
  gc.in_top = static_cast<u64>(top[1]);
  gc.out_garbage = gc.in_garbage = 0;
  gc.dead_out = gc.dead_in = 0;
  if (!g.props.allow_multi) {
    graph_index_build(ctx, g, 0, g.ecap);  // same room as before; uploads the counters too
  } else {
    DYNGB200_CUDA(cudaMemcpyAsync(g.counters.ptr, &gc, sizeof(gc), cudaMemcpyHostToDevice, s));
    DYNGB200_CUDA(cudaStreamSynchronize(s));
  }
}

// Grow the vertex capacity and/or the arenas.  Heavily fragmented arenas are compacted instead.
void graph_grow(Context& ctx, Graph& g, long long need_n, long long need_out, long long need_in) {
  graph_refresh_host(ctx, g);
  const long long m = g.m;
  const long long garbage = static_cast<long long>(
      std::max(g.host_counters.out_garbage, g.host_counters.in_garbage));
  const bool compact = garbage > m / 2 + 1024;
  if (!compact && (need_out > g.arena_cap || need_in > g.arena_cap)) {
    MaintenanceTimer timer(g, g.grow_ms);
    // more arena on the device: the used part of each column copied to a 1.5x larger arena at
    // the same slot offsets (row descriptors and the edge index stay valid)
    const long long top = static_cast<long long>(std::max(g.host_counters.out_top,
                                                          g.host_counters.in_top));
    // a multiple of 4 slots: weight column j starts at j * arena_cap, and rows are read with
    // 16-byte loads
    const long long new_cap = round4(std::max(
        std::max(need_out, need_in) + (need_out + need_in) / 4, g.arena_cap + g.arena_cap / 2));
    expects(new_cap < (1LL << 32), "graph: the slack arena would pass 2^32 slots",
            DYNGB200_CAPACITY);
    const size_t k = static_cast<size_t>(g.k > 0 ? g.k : 1);
    // all four new arrays before anything is swapped: the weight columns' stride is arena_cap,
    // so the arrays and arena_cap change together or not at all
    DevBuf<int32_t> fresh[4];
    DevBuf<int32_t>* cur[4] = {&g.out_col, &g.in_col, &g.out_w, &g.in_w};
    for (int a = 0; a < 4; ++a)
      fresh[a].reserve(static_cast<size_t>(new_cap) * (a < 2 ? 1 : k));
    for (int a = 0; a < 4; ++a) {
      const size_t cols = a < 2 ? 1 : k;
      for (size_t j = 0; j < cols; ++j)
        DYNGB200_CUDA(cudaMemcpyAsync(fresh[a].ptr + j * new_cap, cur[a]->ptr + j * g.arena_cap,
                                      static_cast<size_t>(top) * sizeof(int32_t),
                                      cudaMemcpyDeviceToDevice, ctx.stream));
    }
    DYNGB200_CUDA(cudaStreamSynchronize(ctx.stream));
    for (int a = 0; a < 4; ++a) cur[a]->swap(fresh[a]);
    g.arena_cap = new_cap;
    ++g.arena_growths;
  }
  if (compact) graph_compact(ctx, g, need_out, need_in);
  if (need_n > g.n_cap) {
    const long long new_cap = std::max(need_n + 1024, g.n_cap * 2);
    // every new array before anything is swapped (a failed allocation changes nothing)
    DevBuf<RowDesc> fdesc[2];
    DevBuf<int32_t> fint[4];
    DevBuf<RowDesc>* cdesc[2] = {&g.out_desc, &g.in_desc};
    DevBuf<int32_t>* cint[4] = {&g.out_cap, &g.in_cap, &g.out_dead, &g.in_dead};
    for (auto& f : fdesc) f.reserve(static_cast<size_t>(new_cap));
    for (auto& f : fint) f.reserve(static_cast<size_t>(new_cap));
    for (int a = 0; a < 2; ++a) {
      DYNGB200_CUDA(cudaMemsetAsync(fdesc[a].ptr, 0, new_cap * sizeof(RowDesc), ctx.stream));
      DYNGB200_CUDA(cudaMemcpyAsync(fdesc[a].ptr, cdesc[a]->ptr, g.n_cap * sizeof(RowDesc),
                                    cudaMemcpyDeviceToDevice, ctx.stream));
    }
    for (int a = 0; a < 4; ++a) {
      DYNGB200_CUDA(cudaMemsetAsync(fint[a].ptr, 0, new_cap * sizeof(int32_t), ctx.stream));
      DYNGB200_CUDA(cudaMemcpyAsync(fint[a].ptr, cint[a]->ptr, g.n_cap * sizeof(int32_t),
                                    cudaMemcpyDeviceToDevice, ctx.stream));
    }
    DYNGB200_CUDA(cudaStreamSynchronize(ctx.stream));
    for (int a = 0; a < 2; ++a) cdesc[a]->swap(fdesc[a]);
    for (int a = 0; a < 4; ++a) cint[a]->swap(fint[a]);
    g.n_cap = new_cap;
  }
}

void graph_rescan_columns(Context& ctx, Graph& g) {
  DevBuf<long long> out;
  const size_t k = static_cast<size_t>(g.k > 0 ? g.k : 1);
  out.reserve(3 * k);
  DYNGB200_CUDA(cudaMemsetAsync(out.ptr, 0, 3 * k * sizeof(long long), ctx.stream));
  const int grid = grid_for(32 * g.n, kBlock, ctx.sm_count);  // a warp per row
  ctx.launches += 2;
  k_rescan_columns<<<grid, kBlock, 0, ctx.stream>>>(g.view(), g.n, out.ptr);
  k_rescan_count<<<grid, kBlock, 0, ctx.stream>>>(g.view(), g.n, out.ptr);
  std::vector<long long> h(3 * k);
  DYNGB200_CUDA(cudaMemcpyAsync(h.data(), out.ptr, 3 * k * sizeof(long long),
                                cudaMemcpyDeviceToHost, ctx.stream));
  DYNGB200_CUDA(cudaStreamSynchronize(ctx.stream));
  for (int j = 0; j < g.k; ++j) {
    ColumnStats cs{std::max<long long>(h[3 * j], 1), h[3 * j + 1], h[3 * j + 2], 0,
                   g.host_columns[j].bad};
    if (h[3 * j] == 0) cs.count_at_max = 0;
    g.host_columns[j] = cs;
  }
  DYNGB200_CUDA(cudaMemcpyAsync(g.columns.ptr, g.host_columns.data(),
                                g.host_columns.size() * sizeof(ColumnStats),
                                cudaMemcpyHostToDevice, ctx.stream));
  DYNGB200_CUDA(cudaStreamSynchronize(ctx.stream));
}

// ------------------------------------------------------------------------------------------------
// The applier (queued on ctx.stream; the caller reads the control block once at the end)
// ------------------------------------------------------------------------------------------------
StagedBatch stage_batch(Context& ctx, const dyngb200_batch& batch, int k) {
  StagedBatch b{};
  b.ni = batch.num_insertions;
  b.nd = batch.num_deletions;
  if (batch.memory == DYNGB200_DEVICE) {
    b.ins_src = batch.insert_src;
    b.ins_dst = batch.insert_dst;
    b.ins_w = batch.insert_weights;
    b.del_src = batch.delete_src;
    b.del_dst = batch.delete_dst;
    return b;
  }
  Workspace& ws = ctx.ws;
  cudaStream_t s = ctx.stream;
  const size_t ni = static_cast<size_t>(b.ni), nd = static_cast<size_t>(b.nd);
  ws.b_ins_src.reserve(ni + 1);
  ws.b_ins_dst.reserve(ni + 1);
  ws.b_ins_w.reserve(ni * static_cast<size_t>(k > 0 ? k : 1) + 1);
  ws.b_del_src.reserve(nd + 1);
  ws.b_del_dst.reserve(nd + 1);
  if (ni) {
    DYNGB200_CUDA(cudaMemcpyAsync(ws.b_ins_src.ptr, batch.insert_src, ni * 4, cudaMemcpyHostToDevice, s));
    DYNGB200_CUDA(cudaMemcpyAsync(ws.b_ins_dst.ptr, batch.insert_dst, ni * 4, cudaMemcpyHostToDevice, s));
    if (k > 0)
      DYNGB200_CUDA(cudaMemcpyAsync(ws.b_ins_w.ptr, batch.insert_weights, ni * k * 4,
                                    cudaMemcpyHostToDevice, s));
  }
  if (nd) {
    DYNGB200_CUDA(cudaMemcpyAsync(ws.b_del_src.ptr, batch.delete_src, nd * 4, cudaMemcpyHostToDevice, s));
    DYNGB200_CUDA(cudaMemcpyAsync(ws.b_del_dst.ptr, batch.delete_dst, nd * 4, cudaMemcpyHostToDevice, s));
  }
  b.ins_src = ws.b_ins_src.ptr;
  b.ins_dst = ws.b_ins_dst.ptr;
  b.ins_w = ws.b_ins_w.ptr;
  b.del_src = ws.b_del_src.ptr;
  b.del_dst = ws.b_del_dst.ptr;
  return b;
}

// Blocks of the applier kernel per SM (asked once per context).
static int apply_blocks_per_sm(Context& ctx) {
  if (ctx.apply_blocks_per_sm == 0) {
    int per_sm = 0;
    DYNGB200_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_apply, kBlock, 0));
    expects(per_sm >= 1, "graph::apply: the applier kernel does not fit on an SM",
            DYNGB200_NOT_SUPPORTED);
    ctx.apply_blocks_per_sm = per_sm;
  }
  return ctx.apply_blocks_per_sm;
}

// The batch applier (Steps A-J), queued on ctx.stream as one cooperative launch (or, `stepped`,
// as one ordinary launch per step); the caller reads the control block once at the end.
// `objective` >= 0 also records the sssp change classification for that weight column and the
// plan (packing, default width); tree arrays are not touched.  With `tree` and a scheduler (or a
// schedule asking for features), block 0 of the launch computes the batch features and the
// schedule into the control block.
void apply_launch(Context& ctx, Graph& g, const StagedBatch& b, int objective, long long delta_opt,
                  const dyngb200_schedule* sched, Tree* tree, const Scheduler* learned,
                  bool stepped) {
  if (!stepped) require_cooperative(ctx);
  Workspace& ws = ctx.ws;
  cudaStream_t s = ctx.stream;
  const long long dir = g.props.directed ? 1 : 2;
  const long long ops = (b.ni + b.nd) * dir;
  // every allocation first: a failed one leaves the graph as it was
  ws.reserve_vertices(g.n_cap, s);
  ws.reserve_batch(ops, g.k, s);
  if (!g.props.sorted) {
    const size_t cap = static_cast<size_t>(ws.pairs_sized);
    ws.row_seg_offsets.reserve(cap);
    ws.row_seg.reserve(cap);
  }
  const int blocks = std::min(apply_blocks_per_sm(ctx) * ctx.sm_count, update_grid_blocks(ctx));
  const int touch_gen = ws.next_touch_generation(s);
  UpdateCtl init{};
  init.err_index = INT64_MAX;
  init.n_old = g.n;
  init.n_after = g.n;
  init.batch_ins_max = 1;
  init.minimum = kPackedInf;
  if (sched) schedule_into(*sched, init);
  *ws.host_ctl.ptr = init;
  DYNGB200_CUDA(cudaMemcpyAsync(ws.ctl.ptr, ws.host_ctl.ptr, sizeof(UpdateCtl),
                                cudaMemcpyHostToDevice, s));
  ApplyParams p = make_params(ctx, g, b, objective, delta_opt);
  p.touch_gen = touch_gen;
  p.seg_offsets = ws.row_seg_offsets.ptr;
  p.seg = ws.row_seg.ptr;
  ApplyLaunch L{};
  // the learned scheduler's batch features come from the validation pass (the batch, the old
  // rows and the tree before anything changes); its inference follows the plan's default width
  const bool features = tree && (learned || (sched && sched->record_features));
  if (features) {
    p.feat = 1;
    p.feat_parent = tree->parent.ptr;
    p.feat_tree_n = tree->n;
    L.infer_on = 1;
    learned_infer_args(ctx, *tree, learned, &L.infer);
  }
  L.barrier_limit_ns = ctx.test_barrier_timeout_ns > 0
                           ? static_cast<unsigned long long>(ctx.test_barrier_timeout_ns)
                           : 0;
  L.barrier_extra = ctx.test_barrier_kernel == 2 ? 0 : ctx.test_barrier_extra;
  if (stepped) {
    // the steps in the fused kernel's order; apply_ns gets the same marks (the start of the
    // applier, then the end of each step of the fused kernel)
    int mark = 0;
    auto step = [&](int which, int grid) {
      // the plan and the pairs, and the moves and the appends, are one step each in the fused
      // kernel: the second of each pair records no mark
      const bool second = which == kStepPairs || which == kStepAppend;
      k_apply_step<<<grid, kBlock, 0, s>>>(p, L, which, second ? -1 : mark);
      if (!second) ++mark;
      ++ctx.launches;
      DYNGB200_CUDA(cudaGetLastError());
    };
    step(kStepValidate, blocks);
    step(kStepPlan, 1);
    step(kStepPairs, blocks);
    step(kStepMatch, blocks);
    step(kStepResolve, blocks);
    if (!g.props.sorted) {
      step(kStepRowOffsets, blocks);
      step(kStepFillSegments, blocks);
      step(kStepSortSegments, blocks);
    }
    step(kStepAlloc, blocks);
    step(kStepMutate, blocks);
    step(kStepMove, blocks);
    step(kStepAppend, blocks);
    step(kStepRows, blocks);
    step(kStepFinalize, 1);
    return;
  }
  void* args[] = {&p, &L};
  ++ctx.launches;
  DYNGB200_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&k_apply), dim3(blocks),
                                            dim3(kBlock), args, 0, s));
}

// graph::apply on its own (no tree): the applier, one read-back, growth and retry on capacity.
void graph_apply(Context& ctx, Graph& g, const dyngb200_batch& batch,
                 dyngb200_apply_summary* summary, unsigned char* weight_increased) {
  Workspace& ws = ctx.ws;
  cudaStream_t s = ctx.stream;
  require_intact(g);
  graph_index_reserve(ctx, g, batch.num_insertions * (g.props.directed ? 1 : 2));
  const StagedBatch b = stage_batch(ctx, batch, g.k);
  UpdateCtl r{};
  DevBuf<unsigned char> flags;
  // allocated before the applier is queued: a failed allocation leaves the graph as it was
  if (weight_increased && b.ni > 0) flags.reserve(static_cast<size_t>(b.ni) * g.k);
  for (int attempt = 0;; ++attempt) {
    apply_launch(ctx, g, b, -1, 0, nullptr, nullptr, nullptr, !cooperative_available(ctx));
    if (weight_increased && b.ni > 0) {
      ApplyParams p = make_params(ctx, g, b, -1, 0);
      k_insert_flags<<<grid_for(b.ni, kBlock, ctx.sm_count), kBlock, 0, s>>>(p, flags.ptr);
      ++ctx.launches;
      DYNGB200_CUDA(cudaGetLastError());
      DYNGB200_CUDA(cudaMemcpyAsync(weight_increased, flags.ptr, static_cast<size_t>(b.ni) * g.k,
                                    cudaMemcpyDeviceToHost, s));
    }
    DYNGB200_CUDA(cudaMemcpyAsync(ws.host_ctl.ptr, ws.ctl.ptr, sizeof(UpdateCtl),
                                  cudaMemcpyDeviceToHost, s));
    DYNGB200_CUDA(cudaMemcpyAsync(&g.host_counters, g.counters.ptr, sizeof(GraphCounters),
                                  cudaMemcpyDeviceToHost, s));
    DYNGB200_CUDA(cudaMemcpyAsync(g.host_columns.data(), g.columns.ptr,
                                  g.host_columns.size() * sizeof(ColumnStats),
                                  cudaMemcpyDeviceToHost, s));
    DYNGB200_CUDA(cudaStreamSynchronize(s));
    r = *ws.host_ctl.ptr;
    if ((r.error & kErrCapacity) && attempt < 4) {
      graph_grow(ctx, g, r.n_after > g.n_cap ? r.n_after : 0, static_cast<long long>(r.top_out),
                 static_cast<long long>(r.top_in));
      continue;
    }
    break;
  }
  if (r.committing && !r.applied) {
    g.broken = true;
    throw Error(DYNGB200_INTERNAL,
                "graph::apply: the batch applier stopped part-way through applying the batch; "
                "the graph is incomplete");
  }
  if (r.error & kErrCapacity) throw Error(DYNGB200_CAPACITY, "graph::apply: capacity exceeded");
  if (r.error & kErrInvalidBatch) {
    std::string msg = "graph::apply: invalid batch";
    if (r.err_index != INT64_MAX) msg += " (operation " + std::to_string(r.err_index) + ")";
    throw Error(DYNGB200_INVALID_ARGUMENT, msg);
  }
  if (r.error) throw Error(DYNGB200_INTERNAL, "graph::apply: internal error");
  g.version += 1;
  g.n = g.host_counters.n;
  g.m = g.host_counters.m;
  if (summary) std::memcpy(summary, r.summary, sizeof(*summary));
}

}  // namespace dyngb200

namespace dyngb200 {

template <typename T>
static void copy_buf(DevBuf<T>& dst, const DevBuf<T>& src, cudaStream_t s) {
  if (!src.ptr) return;
  dst.reserve(src.count);
  DYNGB200_CUDA(cudaMemcpyAsync(dst.ptr, src.ptr, src.count * sizeof(T), cudaMemcpyDeviceToDevice, s));
}

// Device contents and host mirrors of `src` into `dst` (same device); dst keeps its identity, so
// trees bound to dst stay bound to it.
void graph_copy(Context& ctx, Graph& dst, const Graph& src) {
  cudaStream_t s = ctx.stream;
  copy_buf(dst.out_desc, src.out_desc, s);
  copy_buf(dst.in_desc, src.in_desc, s);
  copy_buf(dst.out_cap, src.out_cap, s);
  copy_buf(dst.in_cap, src.in_cap, s);
  copy_buf(dst.out_dead, src.out_dead, s);
  copy_buf(dst.in_dead, src.in_dead, s);
  copy_buf(dst.out_col, src.out_col, s);
  copy_buf(dst.in_col, src.in_col, s);
  copy_buf(dst.out_w, src.out_w, s);
  copy_buf(dst.in_w, src.in_w, s);
  copy_buf(dst.counters, src.counters, s);
  copy_buf(dst.columns, src.columns, s);
  copy_buf(dst.ekey, src.ekey, s);
  copy_buf(dst.eout, src.eout, s);
  copy_buf(dst.ein, src.ein, s);
  dst.version = src.version;
  dst.props = src.props;
  dst.k = src.k;
  dst.n = src.n;
  dst.m = src.m;
  dst.n_cap = src.n_cap;
  dst.arena_cap = src.arena_cap;
  dst.ecap = src.ecap;
  dst.host_counters = src.host_counters;
  dst.host_columns = src.host_columns;
  dst.device = src.device;
  DYNGB200_CUDA(cudaStreamSynchronize(s));
}

}  // namespace dyngb200
