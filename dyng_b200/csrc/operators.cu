// The operators engine of sssp::update and sssp::compute: the same algorithm as the fused
// persistent kernel (sssp.cu), as a sequence of ordinary kernel launches whose loop is driven
// from the host, which reads a few counters after each step (the reference's engine::operators,
// cpp/src/algorithms/sssp/operators.cuh and its host loop in operators.cu: one synchronisation
// per push iteration and per threshold raise).  Between the roots and the first push the counts
// stay on the device (the heads, the pull, the first threshold and split read them there), so an
// update synchronises once for the roots, once per four pointer-jumping rounds or per walk level,
// once for the first split, and once per push step or threshold raise.
//
// It needs no cooperative launch, so it is what engine::automatic runs on a device without one
// (as the reference does, sssp.cpp:195-226), and what options::cuda_engine = operators asks for.
// Every kernel is a grid-stride pass over its list or over the vertices (any grid size); rows are
// read by one warp each (the lanes over the row's slots, their minimum or their offers combined
// in the warp).  The fixed point is the fused kernel's: one 64-bit atomicMin per offer on the
// packed (distance << b | parent) word, so the distances, parents, `invalidated` and `affected`
// equal the fused engine's (and the oracle's) bit for bit.  Invalidation runs pointer jumping
// over every vertex (full passes, at most ceil(log2 n) + 1, a parent cycle reported past that),
// or, when the schedule asks for it on a tree that cannot hold a cycle, walks the invalidated
// subtrees level by level over the out-rows.
#include "internal.hpp"
#include "sssp_params.cuh"

#include <algorithm>
#include <cstddef>
#include <string>

namespace dyngb200 {

namespace {

constexpr int kOpBlock = 256;
constexpr int kMarked = -2;  // pointer jumping: an invalidated ancestor was reached
// Rows longer than kOpHeavy slots are not read by one warp: the warp that meets one lists its
// kOpChunk-slot chunks, and a second launch reads every chunk with its own warp.
constexpr int kOpHeavy = 2048;
constexpr int kOpChunk = 1024;
// Pointer-jumping rounds launched between two host synchronisations.
constexpr int kOpRoundsPerSync = 4;

// The counters one step leaves for the host.
struct OpCounts {
  int next;        // entries appended to the next list (near frontier, walk level, pull frontier)
  int far;         // entries on the far pile being appended to
  int candidates;  // vertices the pull re-evaluates
  unsigned moved;  // pointer jumping: bit r set when a chain moved on in round r and goes on
  int heavy;       // chunks listed for the heavy-row launch
  int in_count;    // length of the list a split reads (set by k_op_threshold)
  int source;      // compute: the source, staged for its copy into the frontier
  unsigned long long minimum;    // smallest distance of a list (kPackedInf: none)
  unsigned long long threshold;  // the near-far threshold of the current split and pushes
};

// Lists the chunks of a heavy row as (vertex, first slot) entries and returns how many it listed:
// all of them, or those that fit below `cap` (the caller reads the rest of the row itself).  Every
// entry below min(oc->heavy, cap) is written by the warp that reserved it.  Called by a whole warp.
__device__ __forceinline__ int op_list_chunks(int v, int len, int2* heavy, long long cap,
                                              OpCounts* oc) {
  const int chunks = (len + kOpChunk - 1) / kOpChunk;
  int base = 0;
  if ((threadIdx.x & 31) == 0) base = atomicAdd(&oc->heavy, chunks);
  base = __shfl_sync(0xffffffffu, base, 0);
  const long long room = cap - base;
  const int listed = room <= 0 ? 0 : static_cast<int>(min(static_cast<long long>(chunks), room));
  for (int q = threadIdx.x & 31; q < listed; q += 32) heavy[base + q] = make_int2(v, q * kOpChunk);
  return listed;
}

__device__ __forceinline__ Packing packing_of(int bits) {
  Packing pk;
  pk.bits = bits;
  pk.no_parent = bits ? (1ULL << bits) - 1 : 0;
  return pk;
}

__device__ __forceinline__ bool op_claim(int* stamp, int v, int generation) {
  return atomicExch(&stamp[v], generation) != generation;
}

__device__ __forceinline__ void op_invalidate(const SsspParams& p, int v, OpCounts* oc) {
  p.packed[v] = kPackedInf;
  p.touch_stamp[v] = p.touch_gen;
  p.candidates[append_slot(&oc->candidates)] = v;
}

__device__ __forceinline__ long long op_tid() {
  return blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
}
__device__ __forceinline__ long long op_threads() {
  return static_cast<long long>(gridDim.x) * blockDim.x;
}

// Sum of a per-thread count over the block, added to a global counter by one atomic.
__device__ __forceinline__ void op_block_add(long long v, long long* target) {
  __shared__ unsigned long long s_sum;
  if (threadIdx.x == 0) s_sum = 0;
  __syncthreads();
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0) atomicAdd(&s_sum, static_cast<unsigned long long>(v));
  __syncthreads();
  if (threadIdx.x == 0 && s_sum != 0)
    atomicAdd(reinterpret_cast<unsigned long long*>(target), s_sum);
}

// The persistent words in this call's format and the vertices the batch added (update); every
// word INF but the source's (compute).
__global__ void k_op_setup(SsspParams p, int bits, u64 maxd, long long n) {
  const Packing pk = packing_of(bits);
  UpdateCtl* c = p.ctl;
  for (long long v = op_tid(); v < n; v += op_threads()) {
    if (p.from_scratch) {
      p.packed[v] = v == p.source ? pk.pack(0, -1) : kPackedInf;
      continue;
    }
    if (v >= p.tree_n) {
      p.dist[v] = kInfinity;
      p.parent[v] = -1;
      p.packed[v] = kPackedInf;
      continue;
    }
    if (p.tree_bits != bits) {
      const long long d = p.dist[v];
      u64 word = kPackedInf;
      if (d < kInfinity / 2) {
        if (d < 0 || static_cast<u64>(d) > maxd) atomicOr(&c->error, kErrOverflow);
        else word = pk.pack(static_cast<u64>(d), p.parent[v]);
      }
      p.packed[v] = word;
    }
  }
}

// Roots (fused.cuh:178-197): the heads v of deleted or weight-increased tree edges (u, v) are
// invalidated; for the walk they are also its first level.  `changed` records whether the batch
// holds a changed edge (1) and a root (2).
__global__ void k_op_roots(SsspParams p, int gen_inv, int* level, int walk, OpCounts* oc) {
  UpdateCtl* c = p.ctl;
  const int pairs = c->pairs;
  long long inval = 0;
  int changed = 0;
  for (long long i = op_tid(); i < pairs; i += op_threads()) {
    const int slot = p.pair_list[i];
    const int f = p.pair_flags[slot];
    const bool increased = p.use_inc ? p.inc[static_cast<long long>(slot) * p.k + p.objective] != 0
                                     : (f & kPairIncreased) != 0;
    if (!(f & kPairDelete) && !increased) continue;
    changed |= 1;
    const u64 key = p.pair_key[slot];
    const int32_t u = static_cast<int32_t>(key >> 32);
    const int32_t v = static_cast<int32_t>(key & 0xffffffffu);
    if (v < p.tree_n && p.parent[v] == u && op_claim(p.stamp, v, gen_inv)) {
      changed |= 2;
      op_invalidate(p, v, oc);
      ++inval;
      if (walk) level[append_slot(&oc->next)] = v;
    }
  }
  const int any = __syncthreads_or(changed & 1);
  const int roots = __syncthreads_or(changed & 2);
  if (threadIdx.x == 0 && any) atomicOr(&c->changed, roots ? 3 : 1);
  op_block_add(inval, &c->invalidated);
}

// One level of the subtree walk: every child y of a level vertex u (parent[y] == u) is
// invalidated and joins the next level.  One warp per level vertex, its lanes over the out-row.
__global__ void k_op_walk(SsspParams p, int gen_inv, const int* level, int count, int* next,
                          OpCounts* oc) {
  const int lane = threadIdx.x & 31;
  long long inval = 0;
  for (long long i = op_tid() >> 5; i < count; i += op_threads() >> 5) {
    const int u = level[i];
    const RowDesc d = p.g.out_desc[u];
    for (int e = lane; e < d.len; e += 32) {
      const int y = p.g.out_col[d.start + e];
      if (y < 0 || y >= p.tree_n || p.parent[y] != u) continue;
      if (!op_claim(p.stamp, y, gen_inv)) continue;
      op_invalidate(p, y, oc);
      ++inval;
      next[append_slot(&oc->next)] = y;
    }
  }
  op_block_add(inval, &p.ctl->invalidated);
}

// Pointer jumping (fused.cuh:199-234): the first ancestors (kMarked for a root, -1 for a child of
// the source, whose chain ends at once), then rounds over every vertex until no chain moves.
// Invariant: ancestor[x] >= 0 implies no root on the tree path from x up to ancestor[x]; a
// vertex whose ancestor is invalidated is invalidated on the spot.  A round may read an ancestor
// word another thread of the same round writes: either value keeps the invariant.
__global__ void k_op_pj_start(SsspParams p, int gen_inv, long long n) {
  for (long long v = op_tid(); v < n; v += op_threads()) {
    const int pa = v < p.tree_n ? p.parent[v] : -1;
    p.ancestor[v] = p.stamp[v] == gen_inv ? kMarked : (pa == p.source ? -1 : pa);
  }
}

// Round `round` returns at once when no chain moved on in the round before it (the rounds are
// launched a few at a time between host synchronisations; a round after the last one that moved
// would change nothing anyway, every ancestor being negative by then).
__global__ void k_op_pj_round(SsspParams p, int gen_inv, long long n, OpCounts* oc, int round) {
  if (round > 0 && !((oc->moved >> (round - 1)) & 1u)) return;
  long long inval = 0;
  int jumped = 0;
  for (long long v = op_tid(); v < n; v += op_threads()) {
    const int a = ld_cg(&p.ancestor[v]);
    if (a < 0) continue;
    int na = ld_cg(&p.ancestor[a]);
    if (na == p.source) na = -1;  // reaching the source ends a chain
    if (na == kMarked) {
      p.ancestor[v] = kMarked;
      p.stamp[v] = gen_inv;
      op_invalidate(p, static_cast<int>(v), oc);
      ++inval;
    } else {
      p.ancestor[v] = na;
      jumped |= na >= 0;
    }
  }
  if (__syncthreads_or(jumped) && threadIdx.x == 0) atomicOr(&oc->moved, 1u << round);
  op_block_add(inval, &p.ctl->invalidated);
}

// Insertion heads (fused.cuh:236-256): pulled, or (canonical trees) offered the inserted edge.
__global__ void k_op_heads(SsspParams p, int bits, u64 maxd, int gen_inv, int gen_pull,
                           OpCounts* oc) {
  const Packing pk = packing_of(bits);
  const int pairs = p.ctl->pairs;
  for (long long i = op_tid(); i < pairs; i += op_threads()) {
    const int slot = p.pair_list[i];
    const int f = p.pair_flags[slot];
    if (!(f & kPairHead)) continue;
    const u64 key = p.pair_key[slot];
    const int32_t v = static_cast<int32_t>(key & 0xffffffffu);
    if (v == p.source) continue;
    if (!p.offer_heads) {
      if (op_claim(p.stamp, v, gen_inv)) p.candidates[append_slot(&oc->candidates)] = v;
      continue;
    }
    if (!(f & (kPairAppend | kPairUpsert))) continue;  // no new weight on (u,v)
    if (ld_cg(&p.stamp[v]) == gen_inv) continue;       // invalidated: pulled anyway
    const int32_t u = static_cast<int32_t>(key >> 32);
    const u64 word = ld_cg(&p.packed[u]);
    if (word == kPackedInf) continue;
    const int ins = (f & kPairUseFirst) ? p.pair_first[slot] : p.pair_last[slot];
    const u64 nd = pk.dist(word) +
                   static_cast<u64>(p.ins_w[static_cast<long long>(ins) * p.k + p.objective]);
    if (nd > maxd) continue;
    const u64 cand = pk.pack(nd, u);
    if (cand >= ld_cg(&p.packed[v])) continue;
    const u64 old = atomicMin(&p.packed[v], cand);
    if (cand < old) p.touch_stamp[v] = p.touch_gen;
    if (nd < pk.dist(old) && op_claim(p.stamp, v, gen_pull))
      p.frontier[append_slot(&oc->next)] = v;
  }
}

// The pull (fused.cuh:258-285): every candidate takes the minimum over its in-row of
// pack(d(y) + w, y); with an offer it joins the frontier.  One warp per candidate; heavy rows
// are listed by chunks for k_op_pull_heavy.
__device__ __forceinline__ void op_pull_range(const SsspParams& p, const Packing& pk, u64 maxd,
                                              int gen_pull, int v, const RowDesc& d, int e0,
                                              int e1, OpCounts* oc) {
  const int lane = threadIdx.x & 31;
  const int32_t* wcol = p.g.in_w + static_cast<long long>(p.objective) * p.g.arena_cap;
  u64 best = kPackedInf;
  for (int e = e0 + lane; e < e1; e += 32) {
    const int y = p.g.in_col[d.start + e];
    if (y < 0) continue;
    // the source's word is distance 0 for good
    const u64 word = y == p.source ? 0 : ld_cg(&p.packed[y]);
    if (word == kPackedInf) continue;
    const u64 nd = (y == p.source ? 0 : pk.dist(word)) + static_cast<u64>(wcol[d.start + e]);
    if (nd > maxd) continue;
    best = min(best, pk.pack(nd, y));
  }
  for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
  if (lane == 0 && best != kPackedInf) {
    const u64 old = atomicMin(&p.packed[v], best);
    if (best < old) p.touch_stamp[v] = p.touch_gen;
    if (op_claim(p.stamp, v, gen_pull)) p.frontier[append_slot(&oc->next)] = v;
  }
}

__global__ void k_op_pull(SsspParams p, int bits, u64 maxd, int gen_pull, int2* heavy,
                          long long heavy_cap, OpCounts* oc) {
  const Packing pk = packing_of(bits);
  const int count = ld_cg(&oc->candidates);  // left by the roots, the invalidation and the heads
  for (long long i = op_tid() >> 5; i < count; i += op_threads() >> 5) {
    const int v = p.candidates[i];
    const RowDesc d = p.g.in_desc[v];
    const int listed = d.len > kOpHeavy ? op_list_chunks(v, d.len, heavy, heavy_cap, oc) : 0;
    if (listed * kOpChunk < d.len)
      op_pull_range(p, pk, maxd, gen_pull, v, d, listed * kOpChunk, d.len, oc);
  }
}

__global__ void k_op_pull_heavy(SsspParams p, int bits, u64 maxd, int gen_pull, const int2* heavy,
                                long long heavy_cap, OpCounts* oc) {
  const Packing pk = packing_of(bits);
  const long long count = min(static_cast<long long>(ld_cg(&oc->heavy)), heavy_cap);
  for (long long i = op_tid() >> 5; i < count; i += op_threads() >> 5) {
    const int2 h = heavy[i];
    const RowDesc d = p.g.in_desc[h.x];
    op_pull_range(p, pk, maxd, gen_pull, h.x, d, h.y, min(d.len, h.y + kOpChunk), oc);
  }
}

// The smallest distance of a list's vertices (none: kPackedInf).
__global__ void k_op_min(SsspParams p, int bits, const int* list, const int* count_at,
                         OpCounts* oc) {
  const Packing pk = packing_of(bits);
  const int count = ld_cg(count_at);
  u64 local = kPackedInf;
  for (long long i = op_tid(); i < count; i += op_threads()) {
    const u64 word = ld_cg(&p.packed[list[i]]);
    if (word != kPackedInf) local = min(local, pk.dist(word));
  }
  for (int o = 16; o > 0; o >>= 1) local = min(local, __shfl_down_sync(0xffffffffu, local, o));
  if ((threadIdx.x & 31) == 0 && local != kPackedInf) atomicMin(&oc->minimum, local);
}

// A list split at the threshold: below it into the near frontier (claimed once per step), the
// rest onto the far pile (the first split: once, by the vertex's flag; a split of the far pile:
// the entries that stay).  Entries taken off the far pile lose the flag.
// The threshold of a split, on the device: the first one min + delta, each later one
// max(threshold, min) + delta (fused.cuh:288-417); the list to split moves to `in_count`, and the
// near frontier and the far pile it fills start empty.  One thread.
__global__ void k_op_threshold(OpCounts* oc, u64 delta, int first, int from_far) {
  const u64 m = oc->minimum;
  if (first) {
    oc->threshold = (m == kPackedInf ? 0 : m) + delta;
  } else {
    const u64 t = oc->threshold;
    oc->threshold = (m == kPackedInf ? t : max(t, m)) + delta;
  }
  oc->minimum = kPackedInf;
  oc->in_count = from_far ? oc->far : oc->next;
  oc->next = 0;
  oc->far = 0;
}

__global__ void k_op_split(SsspParams p, int bits, int gen, const int* list, int from_far,
                           int* near, int* far, OpCounts* oc) {
  const Packing pk = packing_of(bits);
  const u64 threshold = ld_cg(&oc->threshold);
  const int count = ld_cg(&oc->in_count);
  for (long long i = op_tid(); i < count; i += op_threads()) {
    const int v = list[i];
    const u64 word = ld_cg(&p.packed[v]);
    const u64 d = word == kPackedInf ? kPackedInf : pk.dist(word);
    if (d < threshold) {
      if (from_far) p.in_far[v] = 0;
      if (op_claim(p.stamp, v, gen)) near[append_slot(&oc->next)] = v;
    } else if (from_far || atomicExch(&p.in_far[v], 1) == 0) {
      far[append_slot(&oc->far)] = v;
    }
  }
}

// One push step of the near-far loop (fused.cuh:288-417): every near vertex u offers
// pack(d(u) + w, u) to its out-neighbours; an improved neighbour joins the next near frontier
// (below the threshold) or the far pile.  One warp per near vertex; heavy rows are listed by
// chunks for k_op_push_heavy.
__device__ __forceinline__ void op_push_range(const SsspParams& p, const Packing& pk, u64 maxd,
                                              u64 threshold, int gen, int u, u64 du,
                                              const RowDesc& d, int e0, int e1, int* next,
                                              int* far, OpCounts* oc) {
  const int32_t* wcol = p.g.out_w + static_cast<long long>(p.objective) * p.g.arena_cap;
  for (int e = e0 + (threadIdx.x & 31); e < e1; e += 32) {
    const int y = p.g.out_col[d.start + e];
    if (y < 0 || y == p.source) continue;
    const u64 nd = du + static_cast<u64>(wcol[d.start + e]);
    if (nd > maxd) continue;
    const u64 cand = pk.pack(nd, u);
    if (cand >= ld_cg(&p.packed[y])) continue;
    const u64 old = atomicMin(&p.packed[y], cand);
    if (cand < old) p.touch_stamp[y] = p.touch_gen;
    if (nd >= pk.dist(old)) continue;
    if (nd < threshold) {
      if (op_claim(p.stamp, y, gen)) next[append_slot(&oc->next)] = y;
    } else if (atomicExch(&p.in_far[y], 1) == 0) {
      far[append_slot(&oc->far)] = y;
    }
  }
}

__global__ void k_op_push(SsspParams p, int bits, u64 maxd, u64 threshold, int gen,
                          const int* near, int count, int* next, int* far, int2* heavy,
                          long long heavy_cap, OpCounts* oc) {
  const Packing pk = packing_of(bits);
  for (long long i = op_tid() >> 5; i < count; i += op_threads() >> 5) {
    const int u = near[i];
    const u64 wu = ld_cg(&p.packed[u]);
    if (wu == kPackedInf) continue;
    const RowDesc d = p.g.out_desc[u];
    const int listed = d.len > kOpHeavy ? op_list_chunks(u, d.len, heavy, heavy_cap, oc) : 0;
    if (listed * kOpChunk < d.len)
      op_push_range(p, pk, maxd, threshold, gen, u, pk.dist(wu), d, listed * kOpChunk, d.len,
                    next, far, oc);
  }
}

__global__ void k_op_push_heavy(SsspParams p, int bits, u64 maxd, u64 threshold, int gen,
                                int* next, int* far, const int2* heavy, long long heavy_cap,
                                OpCounts* oc) {
  const Packing pk = packing_of(bits);
  const long long count = min(static_cast<long long>(ld_cg(&oc->heavy)), heavy_cap);
  for (long long i = op_tid() >> 5; i < count; i += op_threads() >> 5) {
    const int2 h = heavy[i];
    const u64 wu = ld_cg(&p.packed[h.x]);  // the word the listing warp read, or a smaller one
    const RowDesc d = p.g.out_desc[h.x];
    op_push_range(p, pk, maxd, threshold, gen, h.x, pk.dist(wu), d, h.y,
                  min(d.len, h.y + kOpChunk), next, far, oc);
  }
}

// The commit (fused.cuh:419-494), packed words: every vertex (compute) or every vertex whose word
// this call changed (update) gets its (distance, parent); the changed ones are counted.
__global__ void k_op_unpack(SsspParams p, int bits, long long n) {
  const Packing pk = packing_of(bits);
  long long affected = 0;
  for (long long v = op_tid(); v < n; v += op_threads()) {
    if (!p.from_scratch && ld_cg(&p.touch_stamp[v]) != p.touch_gen) continue;
    const u64 word = ld_cg(&p.packed[v]);
    const long long d = word == kPackedInf ? kInfinity : static_cast<long long>(pk.dist(word));
    const int32_t par = word == kPackedInf ? -1 : pk.parent(word);
    if (p.dist[v] != d || p.parent[v] != par) {
      p.dist[v] = d;
      p.parent[v] = par;
      ++affected;
    }
  }
  if (!p.from_scratch) op_block_add(affected, &p.ctl->affected);
}

// The commit, distance-only words: the distances written, the parents recovered as the lowest-id
// tight in-neighbour (three passes, as in the fused kernel).
__global__ void k_op_dist_prepare(SsspParams p, long long n) {
  for (long long v = op_tid(); v < n; v += op_threads()) {
    const u64 word = ld_cg(&p.packed[v]);
    const long long d = word == kPackedInf ? kInfinity : static_cast<long long>(word);
    if (!p.from_scratch) {
      p.ancestor[v] = p.parent[v];
      p.candidates[v] = d != p.dist[v] ? 1 : 0;
    }
    p.dist[v] = d;
    p.parent[v] = (word == kPackedInf || v == p.source) ? -1 : INT32_MAX;
  }
}

__global__ void k_op_dist_parents(SsspParams p, long long n) {
  const int32_t* wcol = p.g.out_w + static_cast<long long>(p.objective) * p.g.arena_cap;
  const int lane = threadIdx.x & 31;
  for (long long u = op_tid() >> 5; u < n; u += op_threads() >> 5) {
    const u64 du = ld_cg(&p.packed[u]);
    if (du == kPackedInf) continue;
    const RowDesc d = p.g.out_desc[u];
    for (int e = lane; e < d.len; e += 32) {
      const int x = p.g.out_col[d.start + e];
      if (x < 0 || x == p.source) continue;
      if (du + static_cast<u64>(wcol[d.start + e]) == ld_cg(&p.packed[x]))
        atomicMin(&p.parent[x], static_cast<int32_t>(u));
    }
  }
}

__global__ void k_op_dist_count(SsspParams p, long long n) {
  long long affected = 0;
  for (long long v = op_tid(); v < n; v += op_threads())
    affected += (ld_cg(&p.candidates[v]) != 0 || ld_cg(&p.ancestor[v]) != ld_cg(&p.parent[v]));
  op_block_add(affected, &p.ctl->affected);
}

// The run's counters and the tree's history into the control block (what the fused kernel
// writes at its end).
struct OpSummary {
  int iterations, epochs, rounds, active, levels, last_generation, error;
  long long pushes;
  int frontier[4];
};

__global__ void k_op_finish(SsspParams p, OpSummary s) {
  UpdateCtl* c = p.ctl;
  c->iterations = s.iterations;
  c->epochs = s.epochs;
  c->pushes = s.pushes;
  c->rounds = s.rounds;
  c->levels = s.levels;
  if (s.rounds > 0) c->active[(s.rounds - 1) % 3] = s.active;
  c->last_generation = s.last_generation;
  if (s.error) atomicOr(&c->error, static_cast<unsigned>(s.error));
  c->work[2] = c->invalidated;
  if (p.hist) {
    TreeHistory h{};
    h.invalidated = c->invalidated;
    for (int i = 0; i < 4; ++i) h.frontier[i] = s.frontier[i];
    h.iterations = s.iterations + s.epochs;
    h.rounds = s.rounds;
    *p.hist = h;
  }
}

}  // namespace

int operators_grid(const Context& ctx) { return std::max(1, ctx.sm_count * 8); }

void run_operators(Context& ctx, const SsspParams& p) {
  cudaStream_t s = ctx.stream;
  Workspace& ws = ctx.ws;
  UpdateCtl* c = p.ctl;
  expects(ws.op_counts.ptr != nullptr && ws.op_host.ptr != nullptr,
          "sssp: the workspace was not reserved", DYNGB200_INTERNAL);
  static_assert(sizeof(OpCounts) <= 8 * sizeof(unsigned long long), "the step counters fit");
  OpCounts* oc = reinterpret_cast<OpCounts*>(ws.op_counts.ptr);
  OpCounts* hc = reinterpret_cast<OpCounts*>(ws.op_host.ptr);
  const int grid = operators_grid(ctx);
  int2* heavy = p.heavy_a;  // (vertex, first slot) chunks of the heavy rows of one launch
  const long long heavy_cap = static_cast<long long>(ws.heavy_a.count / 2);
  auto read_ctl = [&]() {
    DYNGB200_CUDA(cudaMemcpyAsync(ws.host_ctl.ptr, c, sizeof(UpdateCtl), cudaMemcpyDeviceToHost, s));
    DYNGB200_CUDA(cudaStreamSynchronize(s));
    return *ws.host_ctl.ptr;
  };
  // the plan (the applier's, or compute's upload) and any error found before the engine: an
  // error leaves the control block to the caller as it is
  const UpdateCtl plan = read_ctl();
  if (plan.error != 0) return;
  const long long n = plan.n_after;
  const int bits = plan.packing_bits;
  const u64 maxd = plan.max_distance;
  const long long delta_sel = plan.sched_delta > 0
                                  ? plan.sched_delta
                                  : (p.delta_override > 0 ? p.delta_override : plan.delta);
  const u64 delta = static_cast<u64>(delta_sel > 0 ? delta_sel : 1);
  // the step counters live in pinned memory (hc) and on the device (oc); the host changes hc
  // and copies it over oc before a step, and copies oc back into hc after the steps it reads
  auto put = [&]() {
    DYNGB200_CUDA(cudaMemcpyAsync(oc, hc, sizeof(OpCounts), cudaMemcpyHostToDevice, s));
  };
  auto get = [&]() {
    DYNGB200_CUDA(cudaMemcpyAsync(hc, oc, sizeof(OpCounts), cudaMemcpyDeviceToHost, s));
  };
  auto wait = [&]() { DYNGB200_CUDA(cudaStreamSynchronize(s)); };
  auto launched = [&](int k) {
    ctx.launches += k;
    DYNGB200_CUDA(cudaGetLastError());
  };
  OpSummary sum{};
  int gen = p.generation;
  int* lists[2] = {p.near_a, p.near_b};
  int* fars[2] = {p.far_a, p.far_b};
  *hc = OpCounts{};
  hc->minimum = kPackedInf;
  if (n > 0) {
    k_op_setup<<<grid, kOpBlock, 0, s>>>(p, bits, maxd, n);
    launched(1);
  }
  bool frontier = false;  // the pull's frontier (p.frontier, oc->next entries) is ready
  if (p.from_scratch) {
    if (n > 0) {
      hc->source = p.source;  // staged in pinned memory: copied in stream order
      DYNGB200_CUDA(cudaMemcpyAsync(p.frontier, &hc->source, sizeof(int), cudaMemcpyHostToDevice,
                                    s));
      hc->next = 1;
      put();
      frontier = true;
    }
  } else {
    const int gen_inv = ++gen;
    const int gen_pull = ++gen;
    const bool walk = plan.sched_walk != 0 && p.tree_trusted != 0;
    // ---- roots, and the repack's overflow check: one synchronisation for both ----------------
    put();
    k_op_roots<<<grid, kOpBlock, 0, s>>>(p, gen_inv, lists[0], walk ? 1 : 0, oc);
    launched(1);
    get();
    DYNGB200_CUDA(cudaMemcpyAsync(ws.host_ctl.ptr, c, sizeof(UpdateCtl), cudaMemcpyDeviceToHost, s));
    wait();
    const UpdateCtl after_roots = *ws.host_ctl.ptr;
    if (after_roots.error != 0) return;  // an input distance that does not fit: nothing written
    if (walk) {
      // ---- invalidation by a walk down the old tree, level by level --------------------------
      int level = hc->next, cur = 0;
      while (level > 0) {
        if (sum.levels > n + 1) {
          sum.error |= kErrNotConverged;
          break;
        }
        hc->next = 0;
        put();
        k_op_walk<<<grid, kOpBlock, 0, s>>>(p, gen_inv, lists[cur], level, lists[cur ^ 1], oc);
        launched(1);
        get();
        wait();
        level = hc->next;
        cur ^= 1;
        ++sum.levels;
      }
    } else {
      // ---- invalidation by pointer jumping: when roots exist, or (a tree imported without
      // validation) when any edge changed, so that a parent cycle is still reported -------------
      const int changed = after_roots.changed;
      if ((changed & 2) || (!p.tree_trusted && (changed & 1))) {
        int max_rounds = 0;
        while ((1LL << max_rounds) < n) ++max_rounds;
        ++max_rounds;
        k_op_pj_start<<<grid, kOpBlock, 0, s>>>(p, gen_inv, n);
        launched(1);
        hc->moved = 0;
        put();
        // kOpRoundsPerSync rounds per host synchronisation; sum.rounds counts the rounds up to
        // and including the first in which no chain moved on (all of them if every one moved)
        for (int first = 0; first < max_rounds; first += kOpRoundsPerSync) {
          const int last = std::min(max_rounds, first + kOpRoundsPerSync);
          for (int round = first; round < last; ++round)
            k_op_pj_round<<<grid, kOpBlock, 0, s>>>(p, gen_inv, n, oc, round);
          launched(last - first);
          get();
          wait();
          int round = first;
          while (round < last && ((hc->moved >> round) & 1u)) ++round;
          sum.rounds = std::min(round + 1, last);
          sum.active = (hc->moved >> (sum.rounds - 1)) & 1u;
          if (round < last) break;
        }
      }
    }
    // ---- insertion heads, then the pull over every candidate (its count read on the device) --
    if (sum.error == 0) {
      hc->next = 0;
      hc->heavy = 0;
      put();
      k_op_heads<<<grid, kOpBlock, 0, s>>>(p, bits, maxd, gen_inv, gen_pull, oc);
      k_op_pull<<<grid, kOpBlock, 0, s>>>(p, bits, maxd, gen_pull, heavy, heavy_cap, oc);
      k_op_pull_heavy<<<grid, kOpBlock, 0, s>>>(p, bits, maxd, gen_pull, heavy, heavy_cap, oc);
      launched(3);
      frontier = true;
    }
  }
  // ---- the near-far loop: one host synchronisation per push step or threshold raise -----------
  const long long iteration_cap = 4 * n + 64;
  if (frontier && sum.error == 0) {
    int cur = 0, far_cur = 0;
    // the first threshold and split, with the frontier's length and minimum on the device
    k_op_min<<<grid, kOpBlock, 0, s>>>(p, bits, p.frontier, &oc->next, oc);
    k_op_threshold<<<1, 1, 0, s>>>(oc, delta, 1, 0);
    ++gen;
    k_op_split<<<grid, kOpBlock, 0, s>>>(p, bits, gen, p.frontier, 0, lists[cur], fars[far_cur],
                                         oc);
    launched(3);
    get();
    wait();
    int near_count = hc->next, far_count = hc->far;
    while (near_count > 0 || far_count > 0) {
      const int step = sum.iterations + sum.epochs;
      if (step < 4) sum.frontier[step] = near_count > 0 ? near_count : -far_count;
      if (near_count > 0) {
        if (++sum.iterations > iteration_cap) {
          sum.error |= kErrNotConverged;
          break;
        }
        sum.pushes += near_count;
        ++gen;
        hc->next = 0;
        hc->heavy = 0;
        put();
        const u64 threshold = hc->threshold;
        k_op_push<<<grid, kOpBlock, 0, s>>>(p, bits, maxd, threshold, gen, lists[cur], near_count,
                                            lists[cur ^ 1], fars[far_cur], heavy, heavy_cap, oc);
        k_op_push_heavy<<<grid, kOpBlock, 0, s>>>(p, bits, maxd, threshold, gen, lists[cur ^ 1],
                                                  fars[far_cur], heavy, heavy_cap, oc);
        launched(2);
        get();
        wait();
        cur ^= 1;
        near_count = hc->next;
        far_count = hc->far;
        continue;
      }
      // the near frontier is empty: raise the threshold past the far pile and split the pile
      ++sum.epochs;
      k_op_min<<<grid, kOpBlock, 0, s>>>(p, bits, fars[far_cur], &oc->far, oc);
      k_op_threshold<<<1, 1, 0, s>>>(oc, delta, 0, 1);
      ++gen;
      k_op_split<<<grid, kOpBlock, 0, s>>>(p, bits, gen, fars[far_cur], 1, lists[cur],
                                           fars[far_cur ^ 1], oc);
      launched(3);
      get();
      wait();
      far_cur ^= 1;
      near_count = hc->next;
      far_count = hc->far;
    }
  }
  // ---- commit ---------------------------------------------------------------------------------
  if (n > 0 && sum.error == 0) {
    if (bits > 0) {
      k_op_unpack<<<grid, kOpBlock, 0, s>>>(p, bits, n);
      launched(1);
    } else {
      k_op_dist_prepare<<<grid, kOpBlock, 0, s>>>(p, n);
      k_op_dist_parents<<<grid, kOpBlock, 0, s>>>(p, n);
      launched(2);
      if (!p.from_scratch) {
        k_op_dist_count<<<grid, kOpBlock, 0, s>>>(p, n);
        launched(1);
      }
    }
  }
  sum.last_generation = gen;
  k_op_finish<<<1, 1, 0, s>>>(p, sum);
  launched(1);
}

}  // namespace dyngb200
