// The sssp kernels: one persistent cooperative kernel per compute() / update() that runs subtree
// invalidation, the pull pass, the near-far push loop and the commit, with every loop decision
// taken on the device (the schedule of the reference's fused engine,
// cpp/src/algorithms/sssp/fused.cuh:155-495), on the slack rows of the device graph.
//
// What differs from the reference's kernel (the results do not):
//   - the packed (distance << b | parent) words persist between updates in the tree, so an update
//     does not pack all n vertices; the unpack compares every word with its (distance, parent)
//     and writes the changed ones (`affected`), so the relaxations keep no list of written words;
//   - frontier rows longer than `heavy_degree` are split into 1024-slot chunks spread over all
//     warps (one 64-bit atomic reserves a list slot and its chunk range together), shorter rows
//     of 32+ slots are scanned by a whole warp, the rest by one lane each;
//   - the grid barrier is this file's own, with a time limit after which it records kErrTimeout
//     and every block leaves the kernel (no unbounded spin).
#include "internal.hpp"
#include "grid_sync.cuh"
#include "sssp_params.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>

namespace dyngb200 {

namespace {

constexpr int kThreads = 256;
constexpr int kHeavyChunk = 256;

enum Mode { kPush = 0, kPull = 1, kWalk = 2 };

__device__ __forceinline__ unsigned ld_volatile(const unsigned* p) { return gs_ld_volatile(p); }

// Shared-memory staging of list appends.  A lane appends into its block's stage with a
// warp-aggregated shared-memory atomic (ballot + popc); at the end of the phase the block copies
// the stage to the global list with ONE global atomicAdd for its slot range, so the global list
// counters see one atomic per block and phase instead of one per warp group.  A full stage falls
// back to the global list directly.  Stages: the next frontier (near list, pull frontier or walk
// level), the far pile, the touched list and the pull candidates.
constexpr int kStages = 6;
constexpr int kStageCap = 768;
enum StageId { kStNext = 0, kStFar = 1, kStTouched = 2, kStCand = 3, kStNextMed = 4, kStCandMed = 5 };

struct StageSet {
  int cnt[kStages];
  int base[kStages];
  int* list[kStages];
  int* count[kStages];
  int data[kStages][kStageCap];
};

__shared__ StageSet g_stage;
__shared__ int g_nblk;  // blocks taking part in this launch (the schedule's grid size)
__shared__ int g_bar_arrivals;  // arrivals a grid barrier waits for (g_nblk, plus test phantoms)
__shared__ unsigned long long g_bar_limit;  // the barrier's time limit without progress (ns)

__device__ __forceinline__ void staged_append(int id, int* list, int* count, int v) {
  const unsigned mask = __activemask();
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  const int rank = __popc(mask & ((1u << lane) - 1));
  int base = 0;
  if (lane == leader) {
    base = atomicAdd(&g_stage.cnt[id], __popc(mask));
    g_stage.list[id] = list;
    g_stage.count[id] = count;
  }
  base = __shfl_sync(mask, base, leader);
  const int pos = base + rank;
  if (pos < kStageCap) g_stage.data[id][pos] = v;
  else list[append_slot(count)] = v;
}

__device__ __forceinline__ void stage_init() {
  if (threadIdx.x < kStages) g_stage.cnt[threadIdx.x] = 0;
  __syncthreads();
}

// Copy every non-empty stage to its global list (all threads of the block).
__device__ __forceinline__ void stage_flush() {
  __syncthreads();
  if (threadIdx.x < kStages) {
    const int id = threadIdx.x;
    const int n = min(g_stage.cnt[id], kStageCap);
    g_stage.base[id] = n > 0 ? atomicAdd(g_stage.count[id], n) : 0;
  }
  __syncthreads();
#pragma unroll
  for (int id = 0; id < kStages; ++id) {
    const int n = min(g_stage.cnt[id], kStageCap);
    int* list = g_stage.list[id];
    const int b = g_stage.base[id];
    for (int i = threadIdx.x; i < n; i += blockDim.x) list[b + i] = g_stage.data[id][i];
  }
  __syncthreads();
  if (threadIdx.x < kStages) g_stage.cnt[threadIdx.x] = 0;
}

// Grid-wide barrier over co-resident blocks (cooperative launch, grid_sync.cuh).  Flushes the
// block's stages first.  Returns false once any block has recorded a timeout; the caller then
// leaves the kernel.  *err (optional) receives the error word as every block sees it.
__device__ __forceinline__ bool grid_barrier(UpdateCtl* c, unsigned& gen, unsigned* err = nullptr) {
  stage_flush();
  unsigned e = 0;
  const bool ok = grid_sync(c, gen, static_cast<unsigned>(g_bar_arrivals), g_bar_limit, &e);
  if (err) *err = e;
  return ok;
}

// A vertex whose packed word this update changed: the commit compares only these with the stored
// (distance, parent) (a plain store: every writer stores the same value).
__device__ __forceinline__ void touch(const SsspParams& p, int v) { p.touch_stamp[v] = p.touch_gen; }

__device__ __forceinline__ bool claim(int* stamp, int v, int generation) {
  return atomicExch(&stamp[v], generation) != generation;
}

// The block's minimum into *target with one atomic per block (every thread of the block calls).
__device__ __forceinline__ void block_min_into(u64 v, u64* target) {
  __shared__ u64 s_min[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_down_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) s_min[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    u64 m = kPackedInf;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) m = min(m, s_min[w]);
    if (m != kPackedInf) atomicMin(target, m);
  }
  __syncthreads();
}

// The block's sum into *target with one atomic per block (every thread of the block calls).
__device__ __forceinline__ void block_sum_into(long long v, long long* target) {
  __shared__ long long s_sum[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s_sum[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += s_sum[w];
    if (t != 0)
      atomicAdd(reinterpret_cast<unsigned long long*>(target), static_cast<unsigned long long>(t));
  }
  __syncthreads();
}

// Rows are sorted into three classes when they join a frontier: light (up to 32 slots: their
// slots are dealt over the lanes of one warp), medium (up to `heavy_degree` slots: one row per
// warp) and heavy (split into kHeavyChunk-slot chunks spread over all warps; one 64-bit atomic
// reserves the list slot and the chunk range together, so chunk bases grow with the slot index).
constexpr int kLightMax = 32;

struct ListSet {
  int* light;
  int* light_cnt;
  int* med;
  int* med_cnt;
  int2* heavy;
  u64* heavy_cnt;
  int stage_light;
  int stage_med;
};

__device__ __forceinline__ void list_append(const ListSet& L, int v, int len, int heavy_degree) {
  if (len > heavy_degree) {
    const u64 chunks = static_cast<u64>((len + kHeavyChunk - 1) / kHeavyChunk);
    const u64 prev = atomicAdd(L.heavy_cnt, (1ULL << 40) | chunks);
    L.heavy[static_cast<int>(prev >> 40)] =
        make_int2(v, static_cast<int>(prev & ((1ULL << 40) - 1)));
  } else if (len > kLightMax) {
    staged_append(L.stage_med, L.med, L.med_cnt, v);
  } else {
    staged_append(L.stage_light, L.light, L.light_cnt, v);
  }
}

// A vertex to re-evaluate by the pull pass (classified by in-degree).
__device__ __forceinline__ void add_candidate(const SsspParams& p, int v) {
  const ListSet L{p.candidates, &p.ctl->cand_count, p.cand_med, &p.ctl->cand_med_count,
                  p.pull_heavy, &p.ctl->pull_heavy, kStCand, kStCandMed};
  list_append(L, v, p.g.in_desc[v].len, p.heavy_degree);
}

// Per-thread state of one expansion: where improved vertices go, and work counters.
struct Ctx {
  Packing pk;
  u64 maxd;
  u64 threshold;
  int gen;       // claim generation of the appends
  ListSet next;  // push: next near frontier; walk: next level; pull: the frontier (light only)
  int* far;
  int* far_cnt;
  unsigned slots, words, atomics, appends, rows;
  unsigned tries;  // atomicMin attempts on packed words (successful or not)
};

// One slot of a row.  push: owner u relaxes (u -> y); pull: in-neighbour y offers to the owner;
// walk: y is invalidated if its old parent is the owner.
template <int MODE>
__device__ __forceinline__ void visit(const SsspParams& p, Ctx& X, int owner, u64 odu, int y,
                                      int w) {
  ++X.slots;
  if (y < 0) return;  // tombstone
  if (MODE == kWalk) {
    if (y < p.tree_n && p.parent[y] == owner && claim(p.stamp, y, X.gen)) {
      p.packed[y] = kPackedInf;
      touch(p, y);
      add_candidate(p, y);
      ++X.appends;
      list_append(X.next, y, p.g.out_desc[y].len, p.heavy_degree);
    }
    return;
  }
  int src, dst;
  u64 du;
  if (MODE == kPush) {
    if (y == p.source) return;
    src = owner;
    dst = y;
    du = odu;
  } else {
    // the source's word is distance 0 for good: no load (it is the hottest address of a pull)
    const u64 word = y == p.source ? 0 : ld_cg(&p.packed[y]);
    ++X.words;
    if (word == kPackedInf) return;
    src = y;
    dst = owner;
    du = y == p.source ? 0 : X.pk.dist(word);
  }
  const u64 nd = du + static_cast<u64>(w);
  if (nd > X.maxd) return;
  const u64 cand = X.pk.pack(nd, src);
  if (MODE == kPush) ++X.words;
  if (cand >= ld_cg(&p.packed[dst])) return;
  ++X.tries;
  const u64 old = atomicMin(&p.packed[dst], cand);
  if (cand < old) {
    ++X.atomics;
    touch(p, dst);
  }
  if (nd < X.pk.dist(old)) {
    if (MODE == kPull) {
      if (claim(p.stamp, dst, X.gen)) {
        ++X.appends;
        staged_append(kStNext, X.next.light, X.next.light_cnt, dst);
      }
    } else if (nd < X.threshold) {
      if (claim(p.stamp, dst, X.gen)) {
        ++X.appends;
        list_append(X.next, dst, p.g.out_desc[dst].len, p.heavy_degree);
      }
    } else if (atomicExch(&p.in_far[dst], 1) == 0) {
      ++X.appends;
      staged_append(kStFar, X.far, X.far_cnt, dst);
    }
  }
}

// The pull's offer of in-neighbour y over an in-slot of weight w: packed (d(y) + w, y), or INF.
__device__ __forceinline__ u64 pull_candidate(const SsspParams& p, Ctx& X, int y, int w) {
  ++X.slots;
  if (y < 0) return kPackedInf;
  // the source's word is distance 0 for good: no load (it is the hottest address of a pull)
  const u64 word = y == p.source ? 0 : ld_cg(&p.packed[y]);
  ++X.words;
  if (word == kPackedInf) return kPackedInf;
  const u64 nd = (y == p.source ? 0 : X.pk.dist(word)) + static_cast<u64>(w);
  if (nd > X.maxd) return kPackedInf;
  return X.pk.pack(nd, y);
}

// The best offer of a pull for `owner`: keep it if smaller; on a distance decrease the owner
// joins the frontier of the near-far loop.
__device__ __forceinline__ void offer_owner(const SsspParams& p, Ctx& X, int owner, u64 cand) {
  // no read of the owner's word first: pull owners are mostly invalidated (their word is INF),
  // so the atomicMin nearly always wins and the read would only add a round trip
  ++X.tries;
  // atomicMin and claim together (see push_commit): a lost race appends the owner anyway
  const u64 old = atomicMin(&p.packed[owner], cand);
  const bool claimed = claim(p.stamp, owner, X.gen);
  if (cand < old) {
    ++X.atomics;
    touch(p, owner);
  }
  if (claimed) {
    ++X.appends;
    staged_append(kStNext, X.next.light, X.next.light_cnt, owner);
  }
}

// The push split in two stages, so that a lane issues the loads of several slots before it
// commits any of them: prepare computes the offer and loads the target's current word; commit
// does the atomicMin and the frontier bookkeeping (the same steps as visit<kPush>).
struct Offer {
  int dst;
  u64 cand;
  u64 cur;
};

__device__ __forceinline__ void push_prepare(const SsspParams& p, Ctx& X, int u, u64 du, int y,
                                             int w, Offer& r) {
  ++X.slots;
  r.dst = y;
  r.cand = kPackedInf;
  r.cur = 0;
  if (y < 0 || y == p.source) return;
  const u64 nd = du + static_cast<u64>(w);
  if (nd > X.maxd) return;
  r.cand = X.pk.pack(nd, u);
  ++X.words;
  r.cur = ld_cg(&p.packed[y]);
}

__device__ __forceinline__ void push_commit(const SsspParams& p, Ctx& X, const Offer& r) {
  if (r.cand >= r.cur) return;  // also skips "no offer" (cand == INF)
  const int dst = r.dst;
  const u64 nd = X.pk.dist(r.cand);
  const bool near = nd < X.threshold;
  ++X.tries;
  // The atomicMin, the claim (of the next near frontier, or of the far pile) and the row length
  // are independent: issued together, they cost one round trip instead of three.  The claim is
  // taken on the offer alone (the target's word read before was larger): when another lane's
  // smaller word wins the atomicMin meanwhile, the vertex is still appended and is pushed once
  // more with its current word -- redundant, never wrong.
  const int len = near ? p.g.out_desc[dst].len : 0;
  const u64 old = atomicMin(&p.packed[dst], r.cand);
  const bool claimed = near ? claim(p.stamp, dst, X.gen) : atomicExch(&p.in_far[dst], 1) == 0;
  if (r.cand < old) {
    ++X.atomics;
    touch(p, dst);
  }
  if (!claimed) return;
  ++X.appends;
  if (near) list_append(X.next, dst, len, p.heavy_degree);
  else staged_append(kStFar, X.far, X.far_cnt, dst);
}

template <int MODE>
__device__ __forceinline__ const int32_t* row_col(const SsspParams& p) {
  return MODE == kPull ? p.g.in_col : p.g.out_col;
}
template <int MODE>
__device__ __forceinline__ const int32_t* row_w(const SsspParams& p) {
  return (MODE == kPull ? p.g.in_w : p.g.out_w) + static_cast<long long>(p.objective) * p.g.arena_cap;
}

// Slots [e0, e1) of one row by the 32 lanes of a warp: lane l takes the 4-slot groups l, l+32, ...
// with one 16-byte load of columns and one of weights (rows start on 4-slot boundaries and own at
// least round_up(len, 4) slots, so a group never leaves its row).
template <int MODE>
__device__ __forceinline__ void warp_slots(const SsspParams& p, Ctx& X, int owner, u64 odu,
                                           unsigned start, int e0, int e1) {
  const int lane = threadIdx.x & 31;
  const int32_t* col = row_col<MODE>(p) + start;
  const int32_t* wt = row_w<MODE>(p) + start;
  const int g1 = (e1 + 3) >> 2;
  if (MODE == kPull) {
    // one owner: the warp's minimum over the slots, one offer
    u64 best = kPackedInf;
    for (int grp = (e0 >> 2) + lane; grp < g1; grp += 32) {
      const int e = grp << 2;
      const int4 c4 = __ldg(reinterpret_cast<const int4*>(col + e));
      const int4 w4 = __ldg(reinterpret_cast<const int4*>(wt + e));
      if (e + 0 < e1) best = min(best, pull_candidate(p, X, c4.x, w4.x));
      if (e + 1 < e1) best = min(best, pull_candidate(p, X, c4.y, w4.y));
      if (e + 2 < e1) best = min(best, pull_candidate(p, X, c4.z, w4.z));
      if (e + 3 < e1) best = min(best, pull_candidate(p, X, c4.w, w4.w));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, off));
    if (lane == 0 && best != kPackedInf) offer_owner(p, X, owner, best);
    return;
  }
  if (MODE == kPush) {
    for (int grp = (e0 >> 2) + lane; grp < g1; grp += 32) {
      const int e = grp << 2;
      const int4 c4 = __ldg(reinterpret_cast<const int4*>(col + e));
      const int4 w4 = __ldg(reinterpret_cast<const int4*>(wt + e));
      Offer r0, r1, r2, r3;
      push_prepare(p, X, owner, odu, e + 0 < e1 ? c4.x : -1, w4.x, r0);
      push_prepare(p, X, owner, odu, e + 1 < e1 ? c4.y : -1, w4.y, r1);
      push_prepare(p, X, owner, odu, e + 2 < e1 ? c4.z : -1, w4.z, r2);
      push_prepare(p, X, owner, odu, e + 3 < e1 ? c4.w : -1, w4.w, r3);
      push_commit(p, X, r0);
      push_commit(p, X, r1);
      push_commit(p, X, r2);
      push_commit(p, X, r3);
    }
    return;
  }
  for (int grp = (e0 >> 2) + lane; grp < g1; grp += 32) {
    const int e = grp << 2;
    const int4 c4 = __ldg(reinterpret_cast<const int4*>(col + e));
    const int4 w4 = MODE == kWalk ? make_int4(0, 0, 0, 0) : __ldg(reinterpret_cast<const int4*>(wt + e));
    if (e + 0 < e1) visit<MODE>(p, X, owner, odu, c4.x, w4.x);
    if (e + 1 < e1) visit<MODE>(p, X, owner, odu, c4.y, w4.y);
    if (e + 2 < e1) visit<MODE>(p, X, owner, odu, c4.z, w4.z);
    if (e + 3 < e1) visit<MODE>(p, X, owner, odu, c4.w, w4.w);
  }
}

// Up to 32 rows, one per lane (len 0: none).  Rows of 32+ slots are scanned by the whole warp in
// turn; the shorter rows are concatenated and their slots dealt round-robin to the lanes (the
// owner of slot e is found by a binary search over the lanes' exclusive prefix sums).
template <int MODE>
__device__ __forceinline__ void warp_rows(const SsspParams& p, Ctx& X, int owner, u64 odu,
                                          unsigned start, int len) {
  const int lane = threadIdx.x & 31;
  unsigned big = __ballot_sync(0xffffffffu, len > kLightMax);
  while (big) {
    const int leader = __ffs(big) - 1;
    big &= big - 1;
    warp_slots<MODE>(p, X, __shfl_sync(0xffffffffu, owner, leader),
                     __shfl_sync(0xffffffffu, odu, leader), __shfl_sync(0xffffffffu, start, leader),
                     0, __shfl_sync(0xffffffffu, len, leader));
  }
  const int mine = len <= kLightMax ? len : 0;
  int incl = mine;
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  const int excl = incl - mine;
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  const int32_t* col = row_col<MODE>(p);
  const int32_t* wt = row_w<MODE>(p);
  if (MODE == kPush) {
    // two slots per lane and step: both offers prepared before either commits
    for (int base = 0; base < total; base += 64) {
      Offer r[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int e = base + 32 * q + lane;
        int j = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const int cand = j + step;
          if (__shfl_sync(0xffffffffu, excl, cand) <= e) j = cand;
        }
        const int o = __shfl_sync(0xffffffffu, owner, j);
        const u64 d = __shfl_sync(0xffffffffu, odu, j);
        const unsigned s = __shfl_sync(0xffffffffu, start, j);
        const int ex = __shfl_sync(0xffffffffu, excl, j);
        if (e < total) {
          const unsigned slot = s + static_cast<unsigned>(e - ex);
          push_prepare(p, X, o, d, col[slot], wt[slot], r[q]);
        } else {
          r[q].cand = kPackedInf;
          r[q].cur = 0;
          r[q].dst = -1;
        }
      }
      push_commit(p, X, r[0]);
      push_commit(p, X, r[1]);
    }
    return;
  }
  for (int base = 0; base < total; base += 32) {
    const int e = base + lane;
    int j = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const int cand = j + step;
      if (__shfl_sync(0xffffffffu, excl, cand) <= e) j = cand;
    }
    const int o = __shfl_sync(0xffffffffu, owner, j);
    const u64 d = __shfl_sync(0xffffffffu, odu, j);
    const unsigned s = __shfl_sync(0xffffffffu, start, j);
    const int ex = __shfl_sync(0xffffffffu, excl, j);
    if (MODE == kPull) {
      // the lanes of one owner are contiguous: a segmented minimum, then one offer per owner
      u64 best = kPackedInf;
      if (e < total) {
        const unsigned slot = s + static_cast<unsigned>(e - ex);
        best = pull_candidate(p, X, col[slot], wt[slot]);
      }
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const u64 other = __shfl_down_sync(0xffffffffu, best, off);
        const int oj = __shfl_down_sync(0xffffffffu, j, off);
        if (lane + off < 32 && oj == j) best = min(best, other);
      }
      const int pj = __shfl_up_sync(0xffffffffu, j, 1);
      if (e < total && (lane == 0 || pj != j) && best != kPackedInf) offer_owner(p, X, o, best);
    } else if (e < total) {
      const unsigned slot = s + static_cast<unsigned>(e - ex);
      visit<MODE>(p, X, o, d, col[slot], MODE == kWalk ? 0 : wt[slot]);
    }
  }
}

// The heavy entry whose chunk range holds chunk `ch`: a 32-ary search by the whole warp (each
// lane probes one pivot per step), so a lookup costs about log32(count) dependent loads.
__device__ __forceinline__ int find_heavy(const int2* list, int count, long long ch) {
  const int lane = threadIdx.x & 31;
  int lo = 0, hi = count;  // answer in [lo, hi)
  while (hi - lo > 1) {
    const int stride = (hi - lo + 31) >> 5;
    const int probe = lo + lane * stride;
    const bool ok = probe < hi && static_cast<long long>(__ldcg(&list[probe].y)) <= ch;
    const unsigned bal = __ballot_sync(0xffffffffu, ok);
    const int last = 31 - __clz(bal);  // lane 0 always holds (list[lo].y <= ch)
    lo = lo + last * stride;
    hi = min(hi, lo + stride);
  }
  return lo;
}

// Expand a frontier: light rows in balanced groups of up to 32 per warp, medium rows one per warp,
// heavy rows in kHeavyChunk-slot chunks over all warps.  push / walk expand out-rows, pull
// expands in-rows.  With cursors (zero at the start of the step), medium rows and heavy chunks go
// to whichever warp asks next, so a warp that finished its light rows early takes more of them;
// without, warp w takes rows w, w + nwarps, ...
template <int MODE>
__device__ void expand(const SsspParams& p, Ctx& X, const int* light, int light_count,
                       const int* med, int med_count, const int2* heavy, u64 heavy_cnt,
                       long long gwarp, long long nwarps, long long* probe = nullptr,
                       int* med_cursor = nullptr, unsigned long long* heavy_cursor = nullptr) {
  const int lane = threadIdx.x & 31;
  unsigned long long t_part = probe ? global_ns() : 0;
  // probe: the warp's time in each part, summed into probe[0..2], maxed into probe[3..5]; the
  // block's warps meet in shared memory first (one global atomic per block and value)
  __shared__ long long s_part[6];
  if (probe && threadIdx.x < 6) s_part[threadIdx.x] = 0;
  if (probe) __syncthreads();
  auto part_done = [&](int part) {
    if (!probe) return;
    const unsigned long long now = global_ns();
    if (lane == 0) {
      const long long d = static_cast<long long>(now - t_part);
      atomicAdd(reinterpret_cast<unsigned long long*>(&s_part[part]), static_cast<unsigned long long>(d));
      atomicMax(&s_part[3 + part], d);
    }
    t_part = now;
  };
  const RowDesc* descs = MODE == kPull ? p.g.in_desc : p.g.out_desc;
  // light: `per` consecutive vertices per warp, balanced so that every warp runs the same
  // number of rounds
  if (light_count > 0) {
    const long long rounds = (light_count + nwarps * 32 - 1) / (nwarps * 32);
    long long per = (light_count + rounds * nwarps - 1) / (rounds * nwarps);
    per = per < 1 ? 1 : (per > 32 ? 32 : per);
    for (long long base = gwarp * per; base < light_count; base += nwarps * per) {
      const long long i = base + lane;
      int owner = -1;
      u64 du = 0;
      RowDesc desc{0, 0};
      if (lane < per && i < light_count) {
        owner = ld_cg(&light[i]);
        ++X.rows;
        // the descriptor is loaded beside the owner's word, not after it (one round trip)
        desc = descs[owner];
        if (MODE == kPush) {
          const u64 word = ld_cg(&p.packed[owner]);
          if (word != kPackedInf) du = X.pk.dist(word);
          else desc.len = 0;
        }
      }
      warp_rows<MODE>(p, X, owner, du, desc.start, desc.len);
    }
  }
  part_done(0);
  // medium: one row per warp
  auto medium_row = [&](long long i) {
    const int owner = ld_cg(&med[i]);
    const RowDesc desc = descs[owner];  // beside the owner's word
    u64 du = 0;
    if (MODE == kPush) {
      const u64 word = ld_cg(&p.packed[owner]);
      if (word == kPackedInf) return;
      du = X.pk.dist(word);
    }
    if (lane == 0) ++X.rows;
    warp_slots<MODE>(p, X, owner, du, desc.start, 0, desc.len);
  };
  // the cursors balance many rows or chunks over the warps; with at most one per warp the fixed
  // split is as balanced and spares every warp an atomic on one shared address
  if (med_cursor && med_count > nwarps) {
    // runs of rows per grab, so that a step makes at most about 4 grabs per warp (one cursor
    // address takes every grab of the step)
    const int run = 1 + static_cast<int>(med_count / (4 * nwarps));
    for (;;) {
      int i = 0;
      if (lane == 0) i = atomicAdd(med_cursor, run);
      i = __shfl_sync(0xffffffffu, i, 0);
      if (i >= med_count) break;
      const int end = min(med_count, i + run);
      for (; i < end; ++i) medium_row(i);
    }
  } else {
    for (long long i = gwarp; i < med_count; i += nwarps) medium_row(i);
  }
  part_done(1);
  // heavy: chunks
  const int hcount = static_cast<int>(heavy_cnt >> 40);
  const long long chunks = static_cast<long long>(heavy_cnt & ((1ULL << 40) - 1));
  auto heavy_chunk = [&](long long ch) {
    const int h = find_heavy(heavy, hcount, ch);
    const int owner = __ldcg(&heavy[h].x);
    const int base = __ldcg(&heavy[h].y);
    const RowDesc desc = descs[owner];  // beside the owner's word
    u64 du = 0;
    if (MODE == kPush) {
      const u64 word = ld_cg(&p.packed[owner]);
      if (word == kPackedInf) return;
      du = X.pk.dist(word);
    }
    if (ch == base && lane == 0) ++X.rows;
    const int e0 = static_cast<int>(ch - base) * kHeavyChunk;
    const int e1 = min(desc.len, e0 + kHeavyChunk);
    warp_slots<MODE>(p, X, owner, du, desc.start, e0, e1);
  };
  if (heavy_cursor && chunks > nwarps) {
    const long long run = 1 + chunks / (4 * nwarps);
    for (;;) {
      unsigned long long ch = 0;
      if (lane == 0) ch = atomicAdd(heavy_cursor, static_cast<unsigned long long>(run));
      ch = __shfl_sync(0xffffffffu, ch, 0);
      if (static_cast<long long>(ch) >= chunks) break;
      const long long end = min(chunks, static_cast<long long>(ch) + run);
      for (long long c = static_cast<long long>(ch); c < end; ++c) heavy_chunk(c);
    }
  } else {
    for (long long ch = gwarp; ch < chunks; ch += nwarps) heavy_chunk(ch);
  }
  part_done(2);
  if (probe) {
    __syncthreads();
    if (threadIdx.x < 3)
      atomicAdd(reinterpret_cast<unsigned long long*>(&probe[threadIdx.x]),
                static_cast<unsigned long long>(s_part[threadIdx.x]));
    else if (threadIdx.x < 6)
      atomicMax(&probe[threadIdx.x], s_part[threadIdx.x]);
  }
}


__device__ __forceinline__ void invalidate(const SsspParams& p, int v) {
  p.packed[v] = kPackedInf;
  touch(p, v);
  add_candidate(p, v);
}

// State of the near-far loop carried across a switch between the whole grid and one block.
struct LoopState {
  int gen;
  int it;           // push iterations so far (selects the list buffers and counter slots)
  int iterations;
  int epochs;
  int far_parity;   // which of far_a / far_b is the current far pile
  int done;
  long long pushes;
  u64 threshold;
};

constexpr int kSmallFarMax = 4096;

__device__ __forceinline__ void block_barrier() {
  stage_flush();
  __threadfence();
  __syncthreads();
}

// The near-far loop (fused.cuh:288-417) run by the whole grid (BLOCK = false) or by block 0 alone
// (BLOCK = true, between block barriers: frontiers of up to `small` vertices do not pay for a grid
// barrier per step).  Returns 0 when the loop is finished, 1 when the grid should hand over to
// block 0 (small frontier) or block 0 back to the grid, -1 on a timeout.
template <bool BLOCK>
__device__ int near_far(const SsspParams& p, Ctx& X, LoopState& S, unsigned& bar, u64 delta,
                        long long iteration_cap, int small) {
  UpdateCtl* c = p.ctl;
  const long long tid = BLOCK ? threadIdx.x : blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  const long long threads = BLOCK ? blockDim.x : static_cast<long long>(g_nblk) * blockDim.x;
  const long long gwarp = tid >> 5;
  const long long nwarps = threads >> 5;
  const bool leader = BLOCK ? threadIdx.x == 0 : tid == 0;
  int* lists[2] = {p.near_a, p.near_b};
  int* mlists[2] = {p.near_med_a, p.near_med_b};
  int2* hlists[2] = {p.heavy_a, p.heavy_b};
  const Packing pk = X.pk;
  while (true) {
    // alone, block 0 shows the waiting blocks that it makes progress (no result is read back)
    if (BLOCK && threadIdx.x == 0) atomicAdd(&c->heartbeat, 1u);
    const int cs = S.it % 3;
    const int nc = ld_cg(&c->near_cnt[cs]);
    const int mc = ld_cg(&c->near_med_cnt[cs]);
    const u64 hc = ld_cg(&c->heavy_cnt[cs]);
    const int far_count = ld_cg(&c->far_count);
    const bool near_work = nc > 0 || mc > 0 || (hc >> 40) > 0;
    const bool fits_block =
        (hc >> 40) == 0 && nc + mc <= small && (near_work || far_count <= kSmallFarMax);
    if (!near_work && far_count == 0) return 0;
    if (small > 0 && (BLOCK ? !fits_block : fits_block)) return 1;
    int* far = S.far_parity ? p.far_b : p.far_a;
    int* far2 = S.far_parity ? p.far_a : p.far_b;
    const int step = S.iterations + S.epochs;
    if (leader && blockIdx.x == 0 && step < 64) {
      c->trace_n[step] = near_work ? nc + mc : -far_count;
      c->trace_h[step] = static_cast<int>(hc & 0xffffffffu) | (BLOCK ? 0x40000000 : 0);
      c->trace_t[step] = static_cast<unsigned>(global_ns() - c->phase_ns[0]);
      c->trace_len = step + 1;
    }
    if (near_work) {
      ++S.iterations;
      if (S.iterations > iteration_cap) {
        if (leader) atomicOr(&c->error, kErrNotConverged);
        return 0;
      }
      S.pushes += nc + mc + static_cast<long long>(hc >> 40);
      X.gen = ++S.gen;
      const int nb = (S.it + 1) & 1;
      X.next = ListSet{lists[nb], &c->near_cnt[(S.it + 1) % 3], mlists[nb],
                       &c->near_med_cnt[(S.it + 1) % 3], hlists[nb],
                       &c->heavy_cnt[(S.it + 1) % 3], kStNext, kStNextMed};
      X.far = far;
      X.far_cnt = &c->far_count;
      X.threshold = S.threshold;
      if (leader) {
        c->near_cnt[(S.it + 2) % 3] = 0;
        c->near_med_cnt[(S.it + 2) % 3] = 0;
        c->heavy_cnt[(S.it + 2) % 3] = 0;
        c->med_cursor[(S.it + 2) % 3] = 0;
        c->heavy_cursor[(S.it + 2) % 3] = 0;
      }
      const unsigned long long t_busy = (!BLOCK && step == 0) ? global_ns() : 0;
      expand<kPush>(p, X, lists[S.it & 1], nc, mlists[S.it & 1], mc, hlists[S.it & 1], hc, gwarp,
                    nwarps, (!BLOCK && step == 0) ? &c->work[16] : nullptr, &c->med_cursor[cs],
                    &c->heavy_cursor[cs]);
      if (!BLOCK && step == 0) {
        // balance of the first step: the slowest warp's and the summed busy time, and warps
        // (met per block in shared memory: one global atomic per block and value)
        __shared__ long long s_busy[2];
        if (threadIdx.x == 0) s_busy[0] = s_busy[1] = 0;
        __syncthreads();
        const long long busy = static_cast<long long>(global_ns() - t_busy);
        if ((threadIdx.x & 31) == 0) {
          atomicMax(&s_busy[0], busy);
          atomicAdd(reinterpret_cast<unsigned long long*>(&s_busy[1]),
                    static_cast<unsigned long long>(busy));
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          atomicMax(&c->work[13], s_busy[0]);
          atomicAdd(reinterpret_cast<unsigned long long*>(&c->work[14]),
                    static_cast<unsigned long long>(s_busy[1]));
          atomicAdd(reinterpret_cast<unsigned long long*>(&c->work[15]),
                    static_cast<unsigned long long>(blockDim.x >> 5));
        }
      }
      if (BLOCK) block_barrier();
      else if (!grid_barrier(c, bar)) return -1;
      ++S.it;
      continue;
    }
    // near frontier empty: raise the threshold past the far pile
    ++S.epochs;
    u64 local = kPackedInf;
    for (long long i = tid; i < far_count; i += threads) {
      const u64 word = ld_cg(&p.packed[ld_cg(&far[i])]);
      if (word != kPackedInf) local = min(local, pk.dist(word));
    }
    block_min_into(local, &c->minimum);
    if (BLOCK) block_barrier();
    else if (!grid_barrier(c, bar)) return -1;
    S.threshold = max(S.threshold, ld_cg(reinterpret_cast<const u64*>(&c->minimum))) + delta;
    ++S.gen;
    const ListSet now{lists[S.it & 1], &c->near_cnt[cs], mlists[S.it & 1], &c->near_med_cnt[cs],
                      hlists[S.it & 1], &c->heavy_cnt[cs], kStNext, kStNextMed};
    for (long long i = tid; i < far_count; i += threads) {
      const int v = ld_cg(&far[i]);
      const u64 word = ld_cg(&p.packed[v]);
      const u64 d = word == kPackedInf ? kPackedInf : pk.dist(word);
      if (d < S.threshold) {
        p.in_far[v] = 0;
        if (claim(p.stamp, v, S.gen)) list_append(now, v, p.g.out_desc[v].len, p.heavy_degree);
      } else {
        staged_append(kStFar, far2, &c->far2_count, v);
      }
    }
    if (BLOCK) block_barrier();
    else if (!grid_barrier(c, bar)) return -1;
    if (leader) {
      c->far_count = ld_cg(&c->far2_count);
      c->far2_count = 0;
      c->minimum = kPackedInf;
    }
    if (BLOCK) block_barrier();
    else if (!grid_barrier(c, bar)) return -1;
    S.far_parity ^= 1;
  }
}

__global__ void __launch_bounds__(kThreads, 3) k_sssp(SsspParams p) {
  UpdateCtl* c = p.ctl;
  if (ld_volatile(&c->error) != 0) return;
  // The schedule lives in the control block (written by the host, or by the scheduler's
  // inference kernel on the device): blocks beyond its grid size leave at once.
  const int nblk = c->active_blocks > 0 && c->active_blocks < static_cast<int>(gridDim.x)
                       ? c->active_blocks
                       : static_cast<int>(gridDim.x);
  if (static_cast<int>(blockIdx.x) >= nblk) return;
  if (threadIdx.x == 0) {
    g_nblk = nblk;
    g_bar_arrivals = nblk + (p.barrier_extra > 0 ? p.barrier_extra : 0);
    g_bar_limit = p.barrier_limit_ns > 0 ? p.barrier_limit_ns : kBarrierTimeoutNs;
  }
  if (c->sched_heavy > 0) p.heavy_degree = c->sched_heavy;
  p.small_frontier = c->sched_small;
  p.walk = c->sched_walk && p.tree_trusted ? 1 : 0;
  if (c->sched_delta > 0) p.delta_override = c->sched_delta;
  stage_init();
  // the barrier generation continues from the previous kernel on this control block (the applier)
  unsigned bar = ld_volatile(&c->bar_gen);
  const long long tid = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  const long long threads = static_cast<long long>(nblk) * blockDim.x;
  const int lane = threadIdx.x & 31;
  const long long gwarp = tid >> 5;
  const long long nwarps = threads >> 5;
  const long long n = c->n_after;
  Ctx X;
  X.pk.bits = c->packing_bits;
  X.pk.no_parent = X.pk.bits ? (1ULL << X.pk.bits) - 1 : 0;
  X.maxd = c->max_distance;
  X.threshold = 0;
  X.slots = X.words = X.atomics = X.appends = X.rows = X.tries = 0;
  const Packing pk = X.pk;
  const u64 delta = static_cast<u64>(p.delta_override > 0 ? p.delta_override : c->delta);
  int gen = p.generation;
  int frontier_count = 0;
  // work counters (see dyngb200_stats::work)
  long long w_visits = 0, w_jumps = 0, w_inval = 0;
  unsigned pull_slots = 0, pull_words = 0, pull_rows = 0, unpacked = 0;
  unsigned pull_atomics = 0, pull_appends = 0, pair_visits = 0, walk_rows = 0, walk_slots = 0;
  if (tid == 0) c->phase_ns[0] = global_ns();

  if (p.from_scratch) {
    for (long long v = tid; v < n; v += threads)
      p.packed[v] = v == p.source ? pk.pack(0, -1) : kPackedInf;
    if (tid == 0) p.frontier[0] = p.source;
    frontier_count = 1;
    if (!grid_barrier(c, bar)) return;
  } else {
    const int gen_inv = ++gen;
    const int gen_pull = ++gen;
    // ---- the persistent words in this update's format; growth -------------------------------
    if (p.tree_bits != pk.bits) {
      for (long long v = tid; v < n; v += threads) {
        if (v >= p.tree_n) {
          p.dist[v] = kInfinity;
          p.parent[v] = -1;
        }
        const long long d = p.dist[v];
        u64 word = kPackedInf;
        if (d < kInfinity / 2) {
          if (d < 0 || static_cast<u64>(d) > X.maxd) atomicOr(&c->error, kErrOverflow);
          else word = pk.pack(static_cast<u64>(d), p.parent[v]);
        }
        p.packed[v] = word;
      }
    } else {
      for (long long v = p.tree_n + tid; v < n; v += threads) {
        p.dist[v] = kInfinity;
        p.parent[v] = -1;
        p.packed[v] = kPackedInf;
      }
    }
    // ---- roots: heads v of changed edges (u,v) with parent[v] == u ---------------------------
    const int pairs = c->pairs;
    int changed = 0;
    for (long long i = tid; i < pairs; i += threads) {
      ++pair_visits;
      const int slot = p.pair_list[i];
      const int f = p.pair_flags[slot];
      const bool increased = p.use_inc ? p.inc[static_cast<long long>(slot) * p.k + p.objective] != 0
                                       : (f & kPairIncreased) != 0;
      if ((f & kPairDelete) || increased) {
        changed = 1;
        const u64 key = p.pair_key[slot];
        const int32_t u = static_cast<int32_t>(key >> 32);
        const int32_t v = static_cast<int32_t>(key & 0xffffffffu);
        if (v < p.tree_n && p.parent[v] == u && claim(p.stamp, v, gen_inv)) {
          // roots are invalidated here (stamp = gen_inv marks the invalidated vertices)
          invalidate(p, static_cast<int>(v));
          ++w_inval;
          changed = 2;
          if (p.walk) {
            const ListSet W0{p.near_a, &c->walk_cnt[0], p.near_med_a, &c->walk_med_cnt[0],
                             p.heavy_a, &c->walk_heavy[0], kStNext, kStNextMed};
            list_append(W0, v, p.g.out_desc[v].len, p.heavy_degree);
          }
        }
      }
    }
    {
      // one atomic per block (not per warp) into the shared flag word
      const int any1 = __syncthreads_or(changed != 0);
      const int any2 = __syncthreads_or(changed == 2);
      if (threadIdx.x == 0 && any1) atomicOr(&c->changed, any2 ? 3 : 1);
    }
    unsigned roots_err = 0;
    if (!grid_barrier(c, bar, &roots_err)) return;
    if (roots_err) return;  // every block sees the same snapshot: all leave together
    if (tid == 0) c->phase_ns[1] = global_ns();
    // pointer jumping runs when roots exist, or (a tree imported without validation) when any
    // edge changed, so that a parent cycle is still reported as the reference reports it
    const int changed_bits = ld_cg(&c->changed);
    const bool any_changed = (changed_bits & 2) || (!p.tree_trusted && (changed_bits & 1));
    if (!p.walk) {
      // ---- subtree invalidation by pointer jumping (fused.cuh:199-234) ------------------------
      // ancestor[v]: >= 0 the current ancestor, -1 the chain ended without a root, kMarked:
      // invalidated.  Invariant: ancestor[x] >= 0 implies no root on the tree path from x up to
      // (excluding) ancestor[x].  A vertex whose ancestor is invalidated is invalidated on the
      // spot, so no scan follows the rounds.
      constexpr int kMarked = -2;
      int max_rounds = 0;
      while ((1LL << max_rounds) < n) ++max_rounds;
      ++max_rounds;
      if (any_changed) {
        // Round 0 visits every vertex; a vertex whose new ancestor is still a vertex (it jumps
        // again) is written to its block's survivor region (heavy_a / heavy_b, `span` (vertex,
        // ancestor) entries per block) with no global atomic.  Later rounds see the regions, concatenated in block
        // order, as one list (each block scans the per-block counts) and split it evenly over
        // the blocks: a block visits at most `span` entries, so its survivors fit its region.
        __shared__ int s_pj_cnt;
        __shared__ int s_prefix[kPjMaxBlocks + 1];
        const long long span = (n + nblk - 1) / nblk;
        const long long lo = static_cast<long long>(blockIdx.x) * span;
        // ancestor[] starts as the parents with the roots marked, written by a sequential pass
        // over all vertices, so that every round gathers one random word per vertex
        // (ancestor[a]) instead of two (parent[a] and stamp[a]; a round 0 that gathered both
        // instead of this pass measured 18 % slower at R-MAT scale 22)
        // a child of the source has no ancestor that can be a root: its chain ends at once
        // (and nothing ever gathers ancestor[source], which every chain would reach)
        auto first_ancestor = [&](int st, int pa) {
          return st == gen_inv ? kMarked : (pa == p.source ? -1 : pa);
        };
        // 16-byte loads, two quads per thread in flight (a one-word loop was latency-bound at
        // about a quarter of the bandwidth); the tail, and unaligned arrays, word by word
        const bool vec = ((reinterpret_cast<uintptr_t>(p.stamp) | reinterpret_cast<uintptr_t>(p.parent) |
                           reinterpret_cast<uintptr_t>(p.ancestor)) & 15) == 0;
        const long long quads = vec ? min(n, p.tree_n) >> 2 : 0;
        for (long long q0 = tid; q0 < quads; q0 += 2 * threads) {
          int4 st[2], pa[2];
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const long long q = q0 + j * threads;
            if (q < quads) {
              st[j] = __ldcg(reinterpret_cast<const int4*>(p.stamp) + q);
              pa[j] = __ldcg(reinterpret_cast<const int4*>(p.parent) + q);
            }
          }
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const long long q = q0 + j * threads;
            if (q < quads)
              reinterpret_cast<int4*>(p.ancestor)[q] =
                  make_int4(first_ancestor(st[j].x, pa[j].x), first_ancestor(st[j].y, pa[j].y),
                            first_ancestor(st[j].z, pa[j].z), first_ancestor(st[j].w, pa[j].w));
          }
        }
        for (long long v = 4 * quads + tid; v < n; v += threads)
          p.ancestor[v] = first_ancestor(ld_cg(&p.stamp[v]), v < p.tree_n ? p.parent[v] : -1);
        if (tid == 0) c->work[22] = n;
        if (!grid_barrier(c, bar)) return;
        for (int round = 0; round < max_rounds; ++round) {
          if (tid == 0) {
            c->rounds = round + 1;
            if (round < 24) c->pj_t[round] = static_cast<unsigned>(global_ns() - c->phase_ns[0]);
          }
          if (threadIdx.x == 0) s_pj_cnt = 0;
          long long total = n;
          if (round > 0) {
            const int* cnt = p.pj_blk + ((round - 1) & 1) * kPjMaxBlocks;
            for (int q = threadIdx.x; q < nblk; q += blockDim.x) s_prefix[q + 1] = ld_cg(&cnt[q]);
            if (threadIdx.x == 0) s_prefix[0] = 0;
            __syncthreads();
            if (threadIdx.x < 32) {
              // inclusive scan of s_prefix[1..nblk] by warp 0: chunks of `per`, then the chunk sums
              const int per = (nblk + 31) / 32;
              const int b0 = 1 + lane * per, b1 = min(nblk + 1, b0 + per);
              int run = 0;
              for (int q = b0; q < b1; ++q) {
                run += s_prefix[q];
                s_prefix[q] = run;
              }
              int incl = run;
              for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
              }
              const int before = incl - run;
              for (int q = b0; q < b1; ++q) s_prefix[q] += before;
            }
            __syncthreads();
            total = s_prefix[nblk];
          } else {
            __syncthreads();
          }
          const long long vspan = (total + nblk - 1) / nblk;
          const long long vlo = static_cast<long long>(blockIdx.x) * vspan;
          const long long vhi = min(total, vlo + vspan);
          // survivor entries are (vertex, its ancestor): a round gathers only ancestor[a]
          const int2* cur = (round & 1) ? p.heavy_a : p.heavy_b;  // the previous round's regions
          int2* next = ((round & 1) ? p.heavy_b : p.heavy_a) + lo;  // this block's region
          int jumping = 0;
          // four entries per thread and step, their loads issued together; the warps iterate
          // together (the bound is tested on the warp's first entry) for the ballots below
          for (long long i0 = vlo + (threadIdx.x & ~31); i0 < vhi; i0 += 4LL * blockDim.x) {
            int vv[4], a[4], na[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const long long i = i0 + lane + q * blockDim.x;
              a[q] = -1;
              if (i >= vhi) {
                vv[q] = -1;
              } else if (round == 0) {
                vv[q] = static_cast<int>(i);
              } else {
                // the region holding entry i: the last block whose prefix is <= i
                int lo_b = 0, hi_b = nblk;
                while (hi_b - lo_b > 1) {
                  const int mid = (lo_b + hi_b) >> 1;
                  if (s_prefix[mid] <= i) lo_b = mid;
                  else hi_b = mid;
                }
                const int2 e = __ldcg(&cur[static_cast<long long>(lo_b) * span + (i - s_prefix[lo_b])]);
                vv[q] = e.x;
                a[q] = e.y;
              }
            }
            if (round == 0) {
#pragma unroll
              for (int q = 0; q < 4; ++q) a[q] = vv[q] < 0 ? -1 : ld_cg(&p.ancestor[vv[q]]);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              na[q] = a[q] < 0 ? a[q] : ld_cg(&p.ancestor[a[q]]);
              if (na[q] == p.source) na[q] = -1;  // reaching the source ends a chain
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int v = vv[q];
              bool survives = false;
              if (v >= 0) {
                ++w_visits;
                if (a[q] >= 0) {
                  ++w_jumps;
                  if (na[q] == kMarked) {
                    p.ancestor[v] = kMarked;
                    p.stamp[v] = gen_inv;
                    invalidate(p, v);
                    ++w_inval;
                  } else {
                    p.ancestor[v] = na[q];
                    survives = na[q] >= 0;
                  }
                }
              }
              // warp-aggregated append to the block's survivor region
              const unsigned m = __ballot_sync(0xffffffffu, survives);
              if (m) {
                int base = 0;
                if (lane == 0) base = atomicAdd(&s_pj_cnt, __popc(m));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (survives) next[base + __popc(m & ((1u << lane) - 1))] = make_int2(v, na[q]);
                jumping = 1;
              }
            }
          }
          __syncthreads();
          if (threadIdx.x == 0) p.pj_blk[(round & 1) * kPjMaxBlocks + blockIdx.x] = s_pj_cnt;
          (void)jumping;
          if (!grid_barrier(c, bar)) return;
          if (tid == 0 && round < 24)
            c->pj_done[round] = static_cast<unsigned>(global_ns() - c->phase_ns[0]);
          // every block reads the survivor counts itself: none left, the rounds are done (no
          // flag that every warp with a survivor would store)
          {
            const int* cnt = p.pj_blk + (round & 1) * kPjMaxBlocks;
            int mine = 0;
            for (int q = threadIdx.x; q < nblk; q += blockDim.x) mine |= ld_cg(&cnt[q]);
            const int any = __syncthreads_or(mine != 0);
            if (tid == 0) c->active[round % 3] = any;  // the host's parent-cycle check
            if (!any) break;
          }
        }
      }
      if (tid == 0) c->phase_ns[2] = global_ns();
    } else {
      // ---- subtree invalidation by a walk down the old tree's edges, level by level ---------
      X.gen = gen_inv;
      int level = 0;
      while (true) {
        const int cs = level % 3;
        const int nc = ld_cg(&c->walk_cnt[cs]);
        const int mc = ld_cg(&c->walk_med_cnt[cs]);
        const u64 hc = ld_cg(&c->walk_heavy[cs]);
        if (nc == 0 && mc == 0 && (hc >> 40) == 0) break;
        if (level > n + 1) {
          if (tid == 0) atomicOr(&c->error, kErrNotConverged);
          break;
        }
        const int nb = (level + 1) & 1;
        X.next = ListSet{nb ? p.near_b : p.near_a, &c->walk_cnt[(level + 1) % 3],
                         nb ? p.near_med_b : p.near_med_a, &c->walk_med_cnt[(level + 1) % 3],
                         nb ? p.heavy_b : p.heavy_a, &c->walk_heavy[(level + 1) % 3], kStNext,
                         kStNextMed};
        if (tid == 0) {
          c->walk_cnt[(level + 2) % 3] = 0;
          c->walk_med_cnt[(level + 2) % 3] = 0;
          c->walk_heavy[(level + 2) % 3] = 0;
        }
        const int cb = level & 1;
        expand<kWalk>(p, X, cb ? p.near_b : p.near_a, nc, cb ? p.near_med_b : p.near_med_a, mc,
                      cb ? p.heavy_b : p.heavy_a, hc, gwarp, nwarps);
        if (!grid_barrier(c, bar)) return;
        ++level;
      }
      w_inval += X.appends;
      walk_rows = X.rows;
      walk_slots = X.slots;
      X.appends = X.rows = X.slots = 0;
      if (tid == 0) {
        c->levels = level;
        c->phase_ns[2] = global_ns();
      }
    }
    if (!grid_barrier(c, bar)) return;
    if (tid == 0) c->phase_ns[3] = global_ns();
    // ---- insertion heads: pulled, or (canonical trees) offered the inserted edge ----------------
    for (long long i = tid; i < pairs; i += threads) {
      ++pair_visits;
      const int slot = p.pair_list[i];
      const int f = p.pair_flags[slot];
      if (!(f & kPairHead)) continue;
      const u64 key = p.pair_key[slot];
      const int32_t v = static_cast<int32_t>(key & 0xffffffffu);
      if (v == p.source) continue;
      if (!p.offer_heads) {
        if (claim(p.stamp, v, gen_inv)) add_candidate(p, v);
        continue;
      }
      if (!(f & (kPairAppend | kPairUpsert))) continue;       // no new weight on (u,v)
      if (ld_cg(&p.stamp[v]) == gen_inv) continue;              // invalidated: pulled anyway
      const int32_t u = static_cast<int32_t>(key >> 32);
      const u64 word = ld_cg(&p.packed[u]);
      if (word == kPackedInf) continue;
      const int ins = (f & kPairUseFirst) ? p.pair_first[slot] : p.pair_last[slot];
      const u64 nd = pk.dist(word) + static_cast<u64>(p.ins_w[static_cast<long long>(ins) * p.k +
                                                              p.objective]);
      if (nd > X.maxd) continue;
      const u64 cand = pk.pack(nd, u);
      if (cand >= ld_cg(&p.packed[v])) continue;
      const u64 old = atomicMin(&p.packed[v], cand);
      if (cand < old) touch(p, v);
      if (nd < pk.dist(old) && claim(p.stamp, v, gen_pull))
        staged_append(kStNext, p.frontier, &c->frontier_count, v);
    }
    block_sum_into(w_inval, &c->invalidated);
    if (!grid_barrier(c, bar)) return;
    if (tid == 0) c->phase_ns[4] = global_ns();
    // ---- pull pass (fused.cuh:258-285): every candidate takes its best in-neighbour ----------
    {
      Ctx Y = X;
      Y.gen = gen_pull;
      Y.next = ListSet{p.frontier, &c->frontier_count, nullptr, nullptr, nullptr, nullptr, kStNext,
                       kStNextMed};
      Y.slots = Y.words = Y.atomics = Y.appends = Y.rows = Y.tries = 0;
      expand<kPull>(p, Y, p.candidates, ld_cg(&c->cand_count), p.cand_med,
                    ld_cg(&c->cand_med_count), p.pull_heavy, ld_cg(&c->pull_heavy), gwarp, nwarps);
      pull_slots = Y.slots;
      pull_words = Y.words;
      pull_rows = Y.rows;
      pull_atomics = Y.atomics;
      pull_appends = Y.appends;
      X.tries += Y.tries;
    }
    if (!grid_barrier(c, bar)) return;
    frontier_count = ld_cg(&c->frontier_count);
  }
  if (tid == 0) c->phase_ns[5] = global_ns();

  // ---- near-far propagation (fused.cuh:288-417) ------------------------------------------------
  u64 local = kPackedInf;
  for (long long i = tid; i < frontier_count; i += threads) {
    const u64 word = ld_cg(&p.packed[ld_cg(&p.frontier[i])]);
    if (word != kPackedInf) local = min(local, pk.dist(word));
  }
  block_min_into(local, &c->minimum);
  if (!grid_barrier(c, bar)) return;
  const u64 smallest = ld_cg(reinterpret_cast<const u64*>(&c->minimum));
  X.threshold = (smallest == kPackedInf ? 0 : smallest) + delta;
  int* lists[2] = {p.near_a, p.near_b};
  int* mlists[2] = {p.near_med_a, p.near_med_b};
  int2* hlists[2] = {p.heavy_a, p.heavy_b};
  int* far = p.far_a;
  X.far_cnt = &c->far_count;
  ++gen;
  for (long long i = tid; i < frontier_count; i += threads) {
    const int v = ld_cg(&p.frontier[i]);
    const u64 word = ld_cg(&p.packed[v]);
    const u64 d = word == kPackedInf ? kPackedInf : pk.dist(word);
    if (d < X.threshold) {
      if (claim(p.stamp, v, gen))
        list_append(ListSet{lists[0], &c->near_cnt[0], mlists[0], &c->near_med_cnt[0], hlists[0],
                            &c->heavy_cnt[0], kStNext, kStNextMed},
                    v, p.g.out_desc[v].len, p.heavy_degree);
    } else if (atomicExch(&p.in_far[v], 1) == 0) {
      staged_append(kStFar, far, &c->far_count, v);
    }
  }
  if (!grid_barrier(c, bar)) return;
  if (tid == 0) c->minimum = kPackedInf;
  if (!grid_barrier(c, bar)) return;
  LoopState S{gen, 0, 0, 0, 0, 0, 0, X.threshold};
  const long long iteration_cap = 4 * n + 64;
  const int small = p.small_frontier;
  while (true) {
    const int r = near_far<false>(p, X, S, bar, delta, iteration_cap, small);
    if (r < 0) return;
    if (r == 0) break;
    // a small frontier: block 0 runs the loop alone while the other blocks wait at one barrier
    if (blockIdx.x == 0) {
      const int rb = near_far<true>(p, X, S, bar, delta, iteration_cap, small);
      if (threadIdx.x == 0) {
        S.done = rb == 0 ? 1 : 0;
        c->loop_state[0] = S.gen;
        c->loop_state[1] = S.it;
        c->loop_state[2] = S.iterations;
        c->loop_state[3] = S.epochs;
        c->loop_state[4] = S.far_parity;
        c->loop_state[5] = S.done;
        c->loop_pushes = S.pushes;
        c->loop_threshold = S.threshold;
      }
    }
    if (!grid_barrier(c, bar)) return;
    S.gen = ld_cg(&c->loop_state[0]);
    S.it = ld_cg(&c->loop_state[1]);
    S.iterations = ld_cg(&c->loop_state[2]);
    S.epochs = ld_cg(&c->loop_state[3]);
    S.far_parity = ld_cg(&c->loop_state[4]);
    S.done = ld_cg(&c->loop_state[5]);
    S.pushes = ld_cg(&c->loop_pushes);
    S.threshold = ld_cg(&c->loop_threshold);
    if (S.done) break;
  }
  gen = S.gen;
  const int iterations = S.iterations, epochs = S.epochs;
  const long long pushes = S.pushes;
  if (tid == 0) c->phase_ns[6] = global_ns();

  // ---- commit: unpack (fused.cuh:419-494) ------------------------------------------------------
  long long affected = 0;
  if (pk.bits > 0) {
    if (p.from_scratch) {
      for (long long v = tid; v < n; v += threads) {
        const u64 word = ld_cg(&p.packed[v]);
        p.dist[v] = word == kPackedInf ? kInfinity : static_cast<long long>(pk.dist(word));
        p.parent[v] = word == kPackedInf ? -1 : pk.parent(word);
      }
    } else {
      // only a vertex whose packed word this update changed can change its (distance, parent):
      // the stamps of every vertex are scanned (4 bytes each, 16-byte loads) and the stamped
      // ones compared with the stored pair; the changed ones are written and counted
      const bool vec = (reinterpret_cast<uintptr_t>(p.touch_stamp) & 15) == 0;
      const long long quads = vec ? n >> 2 : 0;
      auto commit = [&](long long v) {
        ++unpacked;
        const u64 word = ld_cg(&p.packed[v]);
        const long long d = word == kPackedInf ? kInfinity : static_cast<long long>(pk.dist(word));
        const int32_t par = word == kPackedInf ? -1 : pk.parent(word);
        if (p.dist[v] != d || p.parent[v] != par) {
          p.dist[v] = d;
          p.parent[v] = par;
          ++affected;
        }
      };
      for (long long q0 = tid; q0 < quads; q0 += 2 * threads) {
        int4 ts[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const long long q = q0 + j * threads;
          ts[j] = q < quads ? __ldcg(reinterpret_cast<const int4*>(p.touch_stamp) + q)
                            : make_int4(0, 0, 0, 0);
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const long long v = 4 * (q0 + j * threads);
          if (ts[j].x == p.touch_gen) commit(v);
          if (ts[j].y == p.touch_gen) commit(v + 1);
          if (ts[j].z == p.touch_gen) commit(v + 2);
          if (ts[j].w == p.touch_gen) commit(v + 3);
        }
      }
      for (long long v = 4 * quads + tid; v < n; v += threads)
        if (ld_cg(&p.touch_stamp[v]) == p.touch_gen) commit(v);
      if (tid == 0) c->work[28] = n;  // stamps scanned
    }
  } else {
    // distance-only words: recover the lowest-id tight parent of every vertex
    for (long long v = tid; v < n; v += threads) {
      const u64 word = ld_cg(&p.packed[v]);
      const long long d = word == kPackedInf ? kInfinity : static_cast<long long>(word);
      if (!p.from_scratch) {
        p.ancestor[v] = p.parent[v];
        p.candidates[v] = d != p.dist[v] ? 1 : 0;
      }
      p.dist[v] = d;
      p.parent[v] = (word == kPackedInf || v == p.source) ? -1 : INT32_MAX;
    }
    if (!grid_barrier(c, bar)) return;
    const int32_t* wcol = p.g.out_w + static_cast<long long>(p.objective) * p.g.arena_cap;
    for (long long u = tid; u < n; u += threads) {
      const u64 du = ld_cg(&p.packed[u]);
      if (du == kPackedInf) continue;
      const RowDesc desc = p.g.out_desc[u];
      for (int e = 0; e < desc.len; ++e) {
        const int x = p.g.out_col[desc.start + e];
        if (x < 0 || x == p.source) continue;
        if (du + static_cast<u64>(wcol[desc.start + e]) == ld_cg(&p.packed[x]))
          atomicMin(&p.parent[x], static_cast<int32_t>(u));
      }
    }
    if (!grid_barrier(c, bar)) return;
    if (!p.from_scratch) {
      for (long long v = tid; v < n; v += threads)
        affected += (ld_cg(&p.candidates[v]) != 0 || ld_cg(&p.ancestor[v]) != ld_cg(&p.parent[v]));
    }
  }
  // the work counters, one atomic per block and counter
  {
    __shared__ BlockRed red;
    red_sum(red, 0, affected);
    red_sum(red, 1, w_visits);
    red_sum(red, 2, w_jumps);
    red_sum(red, 3, pull_rows);
    red_sum(red, 4, pull_slots);
    red_sum(red, 5, pull_words);
    red_sum(red, 6, X.rows);
    red_sum(red, 7, X.slots);
    red_sum(red, 8, X.words);
    red_sum(red, 9, X.atomics);
    red_sum(red, 10, X.tries);
    red_sum(red, 11, X.appends);
    red_sum(red, 12, unpacked);
    red_sum(red, 13, pull_atomics);
    red_sum(red, 14, pull_appends);
    red_sum(red, 15, pair_visits);
    red_sum(red, 16, walk_rows);
    red_sum(red, 17, walk_slots);
    __syncthreads();
    if (threadIdx.x < 18) {
      // reduction slot -> work counter (slot 0: affected)
      const int w = threadIdx.x < 10 ? static_cast<int>(threadIdx.x) - 1 + (threadIdx.x >= 3 ? 1 : 0)
                                     : (threadIdx.x == 10 ? 12 : (threadIdx.x == 11 ? 10 : (threadIdx.x == 12 ? 11 : static_cast<int>(threadIdx.x) + 10)));
      const long long t = red_total(red, threadIdx.x);
      long long* target = threadIdx.x == 0 ? &c->affected : &c->work[w];
      if (t != 0)
        atomicAdd(reinterpret_cast<unsigned long long*>(target), static_cast<unsigned long long>(t));
    }
  }
  if (tid == 0) {
    c->work[2] = ld_cg(&c->invalidated);  // complete: summed before the heads' barrier
    c->phase_ns[7] = global_ns();
    c->iterations = iterations;
    c->epochs = epochs;
    c->pushes = pushes;
    c->last_generation = gen;
    if (p.hist) {
      TreeHistory h{};
      h.invalidated = ld_cg(&c->invalidated);
      const int len = ld_cg(&c->trace_len);
      for (int i = 0; i < 4; ++i) h.frontier[i] = i < len ? ld_cg(&c->trace_n[i]) : 0;
      h.iterations = iterations + epochs;
      h.rounds = ld_cg(&c->rounds);
      *p.hist = h;
    }
  }
}

// Canonicalise an imported tree (sssp.cpp:377-396): for every edge (u,v) with
// dist[u] + w == dist[v] and u < parent[v], parent[v] becomes u.  Lowest id wins via atomicMin.
// One warp per row, its lanes over the row's slots.
__global__ void k_canonicalize(GraphView g, int objective, int32_t source, long long n,
                               const long long* dist, int32_t* parent) {
  const int32_t* wcol = g.out_w + static_cast<long long>(objective) * g.arena_cap;
  const int lane = threadIdx.x & 31;
  const long long warps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
  for (long long u = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5; u < n;
       u += warps) {
    const long long du = dist[u];
    if (du >= kInfinity / 2) continue;
    const RowDesc desc = g.out_desc[u];
    for (int e = lane; e < desc.len; e += 32) {
      const int v = g.out_col[desc.start + e];
      if (v < 0 || v == source) continue;
      if (du + wcol[desc.start + e] == dist[v]) atomicMin(&parent[v], static_cast<int32_t>(u));
    }
  }
}

__global__ void k_pack(long long n, int bits, const long long* dist, const int32_t* parent,
                       u64* packed) {
  Packing pk;
  pk.bits = bits;
  pk.no_parent = bits ? (1ULL << bits) - 1 : 0;
  for (long long v = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; v < n;
       v += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long d = dist[v];
    packed[v] = d >= kInfinity / 2 ? kPackedInf : pk.pack(static_cast<u64>(d), parent[v]);
  }
}

}  // namespace

// Blocks of the persistent kernel an SM holds at once (its occupancy, asked once per context).
int update_blocks_per_sm(Context& ctx) {
  if (ctx.update_blocks_per_sm == 0) {
    int per_sm = 0;
    DYNGB200_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sssp, kThreads, 0));
    expects(per_sm >= 1, "sssp: the persistent kernel does not fit on an SM", DYNGB200_NOT_SUPPORTED);
    ctx.update_blocks_per_sm = per_sm;
  }
  expects(ctx.update_blocks_per_sm * ctx.sm_count <= kPjMaxBlocks,
          "sssp: more persistent blocks than the pointer-jumping lists support", DYNGB200_NOT_SUPPORTED);
  return ctx.update_blocks_per_sm;
}

// The update's persistent grid: occupancy x SMs, or the context's cap when it is smaller.
int update_grid_blocks(Context& ctx) {
  const int full = update_blocks_per_sm(ctx) * ctx.sm_count;
  return ctx.max_update_blocks > 0 && ctx.max_update_blocks < full ? ctx.max_update_blocks : full;
}

// Blocks of the persistent kernel (co-resident: cooperative launch).
// The schedule's fields in the control block (0 / unset: the heuristic).
void schedule_into(const dyngb200_schedule& sched, UpdateCtl& init) {
  init.sched_delta = sched.delta > 0 ? sched.delta : 0;
  init.sched_small = sched.small_frontier > 0 ? sched.small_frontier
                                              : (sched.small_frontier < 0 ? 0 : kDefaultSmall);
  init.sched_walk = sched.invalidation == 1 ? 1 : 0;
  init.sched_heavy = sched.heavy_degree > 0 ? sched.heavy_degree : 0;
  init.active_blocks = sched.grid_blocks > 0 ? sched.grid_blocks : 0;
}

static int persistent_blocks(Context& ctx, const dyngb200_schedule& sched) {
  (void)sched;  // the schedule's grid size is applied on the device (active_blocks)
  return update_grid_blocks(ctx);
}

void require_intact(const Graph& g) {
  expects(!g.broken,
          "graph: an earlier update stopped part-way through applying its batch (a grid barrier "
          "of the batch applier timed out), so the graph is incomplete; build it again",
          DYNGB200_INTERNAL);
}

bool cooperative_available(const Context& ctx) {
  return ctx.coop_supported != 0 && ctx.test_no_cooperative == 0;
}

void require_cooperative(const Context& ctx) {
  expects(cooperative_available(ctx),
          "sssp: the fused engine needs cooperative launch, which this device does not offer; "
          "use cuda_engine automatic or operators (the multi-kernel engine runs without it)",
          DYNGB200_NOT_SUPPORTED);
}

bool select_engine(const Context& ctx, int requested) {
  expects(requested >= DYNGB200_ENGINE_AUTOMATIC && requested <= DYNGB200_ENGINE_OPERATORS,
          "sssp: unknown cuda_engine " + std::to_string(requested));
  if (requested == DYNGB200_ENGINE_FUSED) require_cooperative(ctx);
  return requested == DYNGB200_ENGINE_OPERATORS ||
         (requested == DYNGB200_ENGINE_AUTOMATIC && !cooperative_available(ctx));
}

static void launch(Context& ctx, SsspParams& p, int blocks) {
  require_cooperative(ctx);
  void* args[] = {&p};
  ++ctx.launches;
  DYNGB200_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&k_sssp), dim3(blocks),
                                            dim3(kThreads), args, 0, ctx.stream));
}

static SsspParams base_params(Context& ctx, Graph& g, Tree& t) {
  Workspace& ws = ctx.ws;
  SsspParams p{};
  p.g = g.view();
  p.objective = t.opt.objective;
  p.source = t.source;
  p.dist = reinterpret_cast<long long*>(t.dist.ptr);
  p.parent = t.parent.ptr;
  p.packed = t.packed.ptr;
  p.stamp = ws.stamp.ptr;
  p.touch_stamp = ws.touch_stamp.ptr;
  p.flag = ws.flag.ptr;
  p.in_far = ws.in_far.ptr;
  p.ancestor = ws.ancestor.ptr;
  p.candidates = ws.candidates.ptr;
  p.frontier = ws.frontier.ptr;
  p.near_a = ws.near_a.ptr;
  p.near_b = ws.near_b.ptr;
  p.far_a = ws.far_a.ptr;
  p.far_b = ws.far_b.ptr;
  p.heavy_a = reinterpret_cast<int2*>(ws.heavy_a.ptr);
  p.heavy_b = reinterpret_cast<int2*>(ws.heavy_b.ptr);
  p.pull_heavy = reinterpret_cast<int2*>(ws.pull_heavy.ptr);
  p.cand_med = ws.cand_med.ptr;
  p.near_med_a = ws.near_med_a.ptr;
  p.near_med_b = ws.near_med_b.ptr;
  p.touched = ws.touched.ptr;
  p.ctl = ws.ctl.ptr;
  p.hist = t.hist.ptr;
  expects(ws.pj_blk.ptr != nullptr, "sssp: the workspace was not reserved", DYNGB200_INTERNAL);
  p.pj_blk = ws.pj_blk.ptr;  // reserved by Workspace::reserve_vertices
  p.barrier_limit_ns = ctx.test_barrier_timeout_ns > 0
                           ? static_cast<unsigned long long>(ctx.test_barrier_timeout_ns)
                           : 0;
  p.barrier_extra = ctx.test_barrier_kernel == 1 ? 0 : ctx.test_barrier_extra;
  return p;
}

// compute(): the persistent kernel from the source (fused.cuh:167-176).
void sssp_compute(Context& ctx, Graph& g, Tree& t, dyngb200_stats* st) {
  require_intact(g);
  const bool operators = select_engine(ctx, t.opt.cuda_engine);
  const long long launches0 = ctx.launches;
  Workspace& ws = ctx.ws;
  cudaStream_t s = ctx.stream;
  ws.reserve_vertices(g.n_cap, s);
  ws.reserve_batch(0, g.k, s);
  // heavy lists hold int2 entries: sized 2 x n_cap ints each by reserve_vertices
  const long long n = g.n;
  if (g.host_columns[t.opt.objective].dirty) graph_rescan_columns(ctx, g);
  const ColumnStats cs = g.host_columns[t.opt.objective];
  expects(cs.bad == 0, "sssp::compute: an edge has a weight below 1 in objective " +
                           std::to_string(t.opt.objective) + "; sssp needs weights in [1, 2^31 - 1]");
  expects(distances_fit(n, cs.max_w), "sssp::compute: distances do not fit in 62 bits");
  UpdateCtl init{};
  init.err_index = INT64_MAX;
  init.n_old = n;
  init.n_after = n;
  init.max_w = cs.max_w;
  init.delta = t.opt.delta > 0 ? t.opt.delta
                               : default_delta(g.m > 1 ? g.m : 1, n, cs.sum_w);
  u64 bound = 0;
  const Packing pk = choose_packing(n, cs.max_w, &bound);
  init.packing_bits = pk.bits;
  init.max_distance = bound;
  init.minimum = kPackedInf;
  const dyngb200_schedule sched = ctx.schedule_set ? ctx.schedule : dyngb200_schedule{};
  schedule_into(sched, init);
  *ws.host_ctl.ptr = init;
  DYNGB200_CUDA(cudaMemcpyAsync(ws.ctl.ptr, ws.host_ctl.ptr, sizeof(UpdateCtl),
                                cudaMemcpyHostToDevice, s));
  tree_reserve(ctx, t, g.n_cap);
  SsspParams p = base_params(ctx, g, t);
  p.from_scratch = 1;
  p.tree_bits = pk.bits;
  p.tree_n = n;
  p.generation = ws.next_generation(1, s);
  p.touch_gen = 1;
  p.heavy_degree = 256;
  const int blocks = persistent_blocks(ctx, sched);
  cudaEvent_t e0, e1;
  DYNGB200_CUDA(cudaEventCreate(&e0));
  DYNGB200_CUDA(cudaEventCreate(&e1));
  DYNGB200_CUDA(cudaEventRecord(e0, s));
  if (n > 0) {
    if (operators) run_operators(ctx, p);
    else launch(ctx, p, blocks);
  }
  DYNGB200_CUDA(cudaEventRecord(e1, s));
  DYNGB200_CUDA(cudaMemcpyAsync(ws.host_ctl.ptr, ws.ctl.ptr, sizeof(UpdateCtl),
                                cudaMemcpyDeviceToHost, s));
  DYNGB200_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const UpdateCtl& r = *ws.host_ctl.ptr;
  if (r.error & kErrTimeout) throw Error(DYNGB200_INTERNAL, "sssp: a grid barrier timed out");
  if (r.error & kErrNotConverged)
    throw Error(DYNGB200_INTERNAL, "sssp: the near-far loop did not converge");
  ws.generation = std::max(ws.generation, r.last_generation);
  t.packed_bits = pk.bits;
  t.n = n;
  if (st) {
    std::memset(st, 0, sizeof(*st));
    st->iterations = r.iterations;
    st->epochs = r.epochs;
    st->pushes = r.pushes;
    st->packed_parents = pk.bits > 0;
    st->engine_used = operators ? DYNGB200_ENGINE_OPERATORS : DYNGB200_ENGINE_FUSED;
    st->delta = init.delta;
    st->max_weight = cs.max_w;
    st->grid_blocks = operators ? operators_grid(ctx)
                                : (init.active_blocks > 0 && init.active_blocks < blocks
                                       ? init.active_blocks
                                       : blocks);
    st->sssp_ms = ms;
    st->kernel_launches = ctx.launches - launches0;
    st->affected = r.affected;
    for (int i = 0; i < 32; ++i) st->work[i] = r.work[i];
    st->trace_len = r.trace_len;
    for (int i = 0; i < r.trace_len && i < 64; ++i) {
      st->trace_light[i] = r.trace_n[i];
      st->trace_heavy[i] = r.trace_h[i];
      st->trace_us[i] = r.trace_t[i] * 1e-3f;
    }
  }
}

// update(): the applier, then the persistent kernel, then one read-back of the control block.
// The pinned read-back area of a graph: the counters first, then the column statistics.
constexpr size_t kCounterSlots = (sizeof(GraphCounters) + sizeof(ColumnStats) - 1) / sizeof(ColumnStats);

// One attempt of an update, queued on the context's stream: the applier, the persistent kernel,
// and the read-back of the control block, counters and column statistics into pinned memory.
static double us_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
}

static void enqueue_attempt(PendingUpdate& u) {
  const auto h0 = std::chrono::steady_clock::now();
  Context& ctx = *u.ctx;
  Graph& g = *u.g;
  Tree& t = *u.t;
  Workspace& ws = ctx.ws;
  cudaStream_t s = ctx.stream;
  tree_reserve(ctx, t, g.n_cap);
  // every allocation of the attempt comes before the applier is queued: a failed one leaves the
  // graph as it was
  g.pinned.reserve(kCounterSlots + g.host_columns.size());
  DYNGB200_CUDA(cudaEventRecord(u.e0, s));
  apply_launch(ctx, g, u.b, t.opt.objective, t.opt.delta, &u.sched, &t, u.learned, u.operators);
  DYNGB200_CUDA(cudaEventRecord(u.e1, s));
  u.host_us[1] += us_since(h0);
  const auto h1 = std::chrono::steady_clock::now();
  SsspParams p = base_params(ctx, g, t);
  p.from_scratch = 0;
  p.tree_n = t.n;
  p.tree_bits = t.packed_bits;
  p.pair_key = ws.pair_key.ptr;
  p.pair_list = ws.pair_list.ptr;
  p.pair_flags = ws.pair_flags.ptr;
  p.pair_first = ws.pair_first.ptr;
  p.pair_last = ws.pair_last.ptr;
  p.ins_w = u.b.ins_w;
  p.k = g.k;
  p.offer_heads = t.canonical ? 1 : 0;
  p.tree_trusted = t.trusted ? 1 : 0;
  p.generation = ws.next_generation(1, s);
  p.touch_gen = p.generation;
  p.heavy_degree = 256;
  if (u.operators) run_operators(ctx, p);
  else launch(ctx, p, u.blocks);
  DYNGB200_CUDA(cudaEventRecord(u.e2, s));
  DYNGB200_CUDA(cudaMemcpyAsync(ws.host_ctl.ptr, ws.ctl.ptr, sizeof(UpdateCtl),
                                cudaMemcpyDeviceToHost, s));
  DYNGB200_CUDA(cudaMemcpyAsync(g.pinned.ptr, g.counters.ptr, sizeof(GraphCounters),
                                cudaMemcpyDeviceToHost, s));
  DYNGB200_CUDA(cudaMemcpyAsync(g.pinned.ptr + kCounterSlots, g.columns.ptr,
                                g.host_columns.size() * sizeof(ColumnStats),
                                cudaMemcpyDeviceToHost, s));
  u.host_us[2] += us_since(h1);
}

PendingUpdate::~PendingUpdate() = default;  // the events belong to the context

// update(), first half: host checks that need no device result, the batch staged on the device
// and the first attempt queued.  Nothing waits for the GPU here (batches in pinned host memory
// or device memory), so several updates of different graphs on one stream queue back to back.
void sssp_update_begin(Context& ctx, Graph& g, Tree& t, const dyngb200_batch& batch,
                       const dyngb200_schedule& sched, const Scheduler* learned,
                       PendingUpdate& u) {
  const auto h0 = std::chrono::steady_clock::now();
  u.ctx = &ctx;
  u.g = &g;
  u.t = &t;
  u.sched = sched;
  u.learned = learned;
  u.launches0 = ctx.launches;
  require_intact(g);
  // before the batch is staged or applied: nothing changes
  u.operators = select_engine(ctx, t.opt.cuda_engine);
  if (g.host_columns[t.opt.objective].dirty) graph_rescan_columns(ctx, g);
  graph_index_reserve(ctx, g, batch.num_insertions * (g.props.directed ? 1 : 2));
  u.b = stage_batch(ctx, batch, g.k);
  u.blocks = persistent_blocks(ctx, sched);
  for (cudaEvent_t& e : ctx.update_events)
    if (!e) DYNGB200_CUDA(cudaEventCreate(&e));
  u.e0 = ctx.update_events[0];
  u.e1 = ctx.update_events[1];
  u.e2 = ctx.update_events[2];
  u.host_us[0] = us_since(h0);
  enqueue_attempt(u);
}

// update(), second half: waits for the queued attempt, grows and retries on a capacity error
// (nothing was changed), then the error translation, the commit bookkeeping and the stats.
// After the commit: the tree's errors (poisoning it), its new state and the stats.
static void finish_tree(Context& ctx, Graph& g, Tree& t, const UpdateCtl& r, int blocks,
                        bool operators, float apply_ms, float sssp_ms, const Scheduler* learned,
                        const dyngb200_schedule& sched, long long launches0,
                        dyngb200_stats* st) {
  if (r.error & kErrInternal) {
    t.poisoned = true;
    throw Error(DYNGB200_INTERNAL, "sssp::update: the in-edge mirror disagrees with the rows");
  }
  if (r.error & kErrOverflow) {
    t.poisoned = true;
    throw Error(DYNGB200_INVALID_ARGUMENT,
                "sssp::update: an input distance is negative or larger than (n - 1) * max "
                "weight; the initial tree does not belong to this graph");
  }
  int max_rounds = 0;
  while ((1LL << max_rounds) < r.n_after) ++max_rounds;
  ++max_rounds;
  if (r.rounds == max_rounds && r.rounds > 0 && r.active[(r.rounds - 1) % 3] != 0) {
    t.poisoned = true;
    throw Error(DYNGB200_INVALID_ARGUMENT,
                "sssp: the input shortest-path tree has a parent cycle (pointer jumping did not "
                "reach a root in ceil(log2 n) + 1 rounds)");
  }
  if (r.error & (kErrTimeout | kErrNotConverged)) {
    t.poisoned = true;
    throw Error(DYNGB200_INTERNAL, (r.error & kErrTimeout)
                                       ? "sssp::update: a grid barrier timed out"
                                       : "sssp::update: the near-far loop did not converge");
  }
  t.n = r.n_after;
  t.packed_bits = r.packing_bits;
  if (st) {
    std::memset(st, 0, sizeof(*st));
    std::memcpy(&st->batch, r.summary, sizeof(st->batch));
    st->invalidated = r.invalidated;
    st->affected = r.affected;
    st->iterations = r.iterations;
    st->epochs = r.epochs;
    st->pushes = r.pushes;
    st->packed_parents = r.packing_bits > 0;
    st->engine_used = operators ? DYNGB200_ENGINE_OPERATORS : DYNGB200_ENGINE_FUSED;
    st->delta = r.sched_delta > 0 ? r.sched_delta : r.delta;
    st->max_weight = r.max_w;
    st->grid_blocks = operators ? operators_grid(ctx)
                                : (r.active_blocks > 0 && r.active_blocks < blocks ? r.active_blocks
                                                                                   : blocks);
    st->invalidation = (r.sched_walk && t.trusted) ? 1 : 0;
    st->apply_ms = apply_ms;
    st->sssp_ms = sssp_ms;
    st->rounds = r.rounds;
    st->touched = r.affected;
    for (int i = 0; i < 32; ++i) st->work[i] = r.work[i];
    st->trace_len = r.trace_len;
    for (int i = 0; i < r.trace_len && i < 64; ++i) {
      st->trace_light[i] = r.trace_n[i];
      st->trace_heavy[i] = r.trace_h[i];
      st->trace_us[i] = r.trace_t[i] * 1e-3f;
    }
    const bool scheduled = learned || sched.record_features;
    for (int i = 0; i < 12; ++i) st->features[i] = scheduled ? r.features[i] : 0.0f;
    for (int i = 0; i < 3; ++i) st->schedule_classes[i] = learned ? r.sched_classes[i] : -1;
    st->kernel_launches = ctx.launches - launches0;
    for (int i = 0; i < 24 && i < r.rounds; ++i) st->pj_round_us[i] = r.pj_t[i] * 1e-3f;
    for (int i = 0; i < 24 && i < r.rounds; ++i) st->pj_done_us[i] = r.pj_done[i] * 1e-3f;
    for (int i = 1; i < 12; ++i)
      st->apply_step_us[i] = r.apply_ns[i] > r.apply_ns[0]
                                 ? static_cast<float>((r.apply_ns[i] - r.apply_ns[0]) * 1e-3)
                                 : 0.0f;
    for (int i = 0; i < 7; ++i)
      st->phase_ms[i] = r.phase_ns[i + 1] > r.phase_ns[i]
                            ? static_cast<float>((r.phase_ns[i + 1] - r.phase_ns[i]) * 1e-6)
                            : 0.0f;
  }
}

void sssp_update_end(PendingUpdate& u, dyngb200_stats* st) {
  Context& ctx = *u.ctx;
  Graph& g = *u.g;
  Tree& t = *u.t;
  Workspace& ws = ctx.ws;
  const Scheduler* learned = u.learned;
  const dyngb200_schedule& sched = u.sched;
  const int blocks = u.blocks;
  const long long launches0 = u.launches0;
  UpdateCtl r{};
  for (int attempt = 0;; ++attempt) {
    const auto w0 = std::chrono::steady_clock::now();
    DYNGB200_CUDA(cudaStreamSynchronize(ctx.stream));
    u.host_us[3] += us_since(w0);
    r = *ws.host_ctl.ptr;
    g.host_counters = *reinterpret_cast<const GraphCounters*>(g.pinned.ptr);
    std::memcpy(g.host_columns.data(), g.pinned.ptr + kCounterSlots,
                g.host_columns.size() * sizeof(ColumnStats));
    ws.generation = std::max(ws.generation, r.last_generation);
    if ((r.error & kErrCapacity) && attempt < 4) {
      // nothing was changed: grow the vertex capacity or the arenas and run again
      graph_grow(ctx, g, r.n_after > g.n_cap ? r.n_after : 0,
                 static_cast<long long>(r.top_out), static_cast<long long>(r.top_in));
      enqueue_attempt(u);
      continue;
    }
    break;
  }
  float apply_ms = 0, sssp_ms = 0;
  cudaEventElapsedTime(&apply_ms, u.e0, u.e1);
  cudaEventElapsedTime(&sssp_ms, u.e1, u.e2);
  if (!r.applied) {
    if (r.committing) {
      // the applier stopped between its first change and its last: the graph is incomplete
      g.broken = true;
      t.poisoned = true;
      throw Error(DYNGB200_INTERNAL,
                  (r.error & kErrTimeout)
                      ? "sssp::update: a grid barrier of the batch applier timed out part-way "
                        "through applying the batch; the graph is incomplete"
                      : "sssp::update: the batch applier found the in-edge mirror inconsistent "
                        "part-way through applying the batch; the graph is incomplete");
    }
    // found before the commit: the graph and the tree are unchanged
    std::string msg = "sssp::update: invalid batch";
    if (r.err_index == -2) msg = "sssp::update: distances do not fit in 62 bits";
    else if (r.err_index != INT64_MAX) msg += " (operation " + std::to_string(r.err_index) + ")";
    if (r.error & kErrCapacity) throw Error(DYNGB200_CAPACITY, "sssp::update: capacity exceeded");
    if (r.error & kErrInvalidBatch) throw Error(DYNGB200_INVALID_ARGUMENT, msg);
    if (r.error & kErrTimeout)
      throw Error(DYNGB200_INTERNAL,
                  "sssp::update: a grid barrier of the batch applier timed out before the batch "
                  "was applied; the graph and the tree are unchanged");
    throw Error(DYNGB200_INTERNAL,
                "sssp::update: the batch applier found the in-edge mirror inconsistent with the "
                "rows; the graph and the tree are unchanged");
  }
  // the batch is committed from here on
  g.version += 1;
  g.n = g.host_counters.n;
  g.m = g.host_counters.m;
  t.version = g.version;
  finish_tree(ctx, g, t, r, blocks, u.operators, apply_ms, sssp_ms, learned, sched, launches0,
              st);
  if (st)
    for (int i = 0; i < 4; ++i) st->host_us[i] = static_cast<float>(u.host_us[i]);
}

// update(): sssp::update(resources::cuda(), g, batch, tree) (sssp.hpp:484-489).
void sssp_update(Context& ctx, Graph& g, Tree& t, const dyngb200_batch& batch,
                 const dyngb200_schedule& sched, dyngb200_stats* st, const Scheduler* learned) {
  PendingUpdate u;
  sssp_update_begin(ctx, g, t, batch, sched, learned, u);
  sssp_update_end(u, st);
}

// ---- update_each: one batch, the trees of several objectives -------------------------------

namespace {
// Per objective j of a batch: out[2j] = the largest insertion weight, out[2j + 1] = the smallest;
// out[2k] = the largest vertex id + 1 the batch names.
__global__ void k_batch_extrema(const int32_t* ins_src, const int32_t* ins_dst,
                                const int32_t* ins_w, long long ni, const int32_t* del_src,
                                const int32_t* del_dst, long long nd, int k, long long* out) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < ni + nd;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const bool ins = i < ni;
    const long long j = ins ? i : i - ni;
    const long long u = ins ? ins_src[j] : del_src[j];
    const long long v = ins ? ins_dst[j] : del_dst[j];
    atomicMax(&out[2 * k], max(u, v) + 1);
    if (ins) {
      for (int c = 0; c < k; ++c) {
        const long long w = ins_w[j * k + c];
        atomicMax(&out[2 * c], w);
        atomicMin(&out[2 * c + 1], w);
      }
    }
  }
}
}  // namespace

// The sssp part of an update for a tree of another objective than the one the batch was applied
// with: the applier's state (pairs, flags, summary) is still in the workspace; the plan of this
// objective comes from the graph as it was before the batch (`pre_*`).
static void sssp_rerun(Context& ctx, Graph& g, Tree& t, const UpdateCtl& applied,
                       const std::vector<ColumnStats>& pre_cols, const GraphCounters& pre_counters,
                       long long batch_max_w, const int32_t* ins_w, dyngb200_stats* st) {
  const long long launches0 = ctx.launches;
  Workspace& ws = ctx.ws;
  cudaStream_t s = ctx.stream;
  const int obj = t.opt.objective;
  const bool operators = select_engine(ctx, t.opt.cuda_engine);
  UpdateCtl init{};
  init.err_index = INT64_MAX;
  init.n_old = applied.n_old;
  init.n_after = applied.n_after;
  init.pairs = applied.pairs;
  std::memcpy(init.summary, applied.summary, sizeof(init.summary));
  init.batch_ins_max = std::max<long long>(1, batch_max_w);
  init.max_w = std::max<long long>(pre_cols[obj].max_w, init.batch_ins_max);
  init.delta = t.opt.delta > 0 ? t.opt.delta
                               : default_delta(std::max<long long>(pre_counters.m, 1),
                                               pre_counters.n, pre_cols[obj].sum_w);
  u64 bound = 0;
  const Packing pk = choose_packing(init.n_after, init.max_w, &bound);
  init.packing_bits = pk.bits;
  init.max_distance = bound;
  init.minimum = kPackedInf;
  const dyngb200_schedule sched{};
  schedule_into(sched, init);
  *ws.host_ctl.ptr = init;
  tree_reserve(ctx, t, g.n_cap);
  cudaEvent_t e1, e2;
  DYNGB200_CUDA(cudaEventCreate(&e1));
  DYNGB200_CUDA(cudaEventCreate(&e2));
  DYNGB200_CUDA(cudaMemcpyAsync(ws.ctl.ptr, ws.host_ctl.ptr, sizeof(UpdateCtl),
                                cudaMemcpyHostToDevice, s));
  const int blocks = persistent_blocks(ctx, sched);
  SsspParams p = base_params(ctx, g, t);
  p.from_scratch = 0;
  p.tree_n = t.n;
  p.tree_bits = t.packed_bits;
  p.pair_key = ws.pair_key.ptr;
  p.pair_list = ws.pair_list.ptr;
  p.pair_flags = ws.pair_flags.ptr;
  p.pair_first = ws.pair_first.ptr;
  p.pair_last = ws.pair_last.ptr;
  p.ins_w = ins_w;
  p.k = g.k;
  p.inc = ws.pair_inc.ptr;
  p.use_inc = 1;
  p.offer_heads = t.canonical ? 1 : 0;
  p.tree_trusted = t.trusted ? 1 : 0;
  p.generation = ws.next_generation(1, s);
  p.touch_gen = p.generation;
  p.heavy_degree = 256;
  DYNGB200_CUDA(cudaEventRecord(e1, s));
  if (operators) run_operators(ctx, p);
  else launch(ctx, p, blocks);
  DYNGB200_CUDA(cudaEventRecord(e2, s));
  DYNGB200_CUDA(cudaMemcpyAsync(ws.host_ctl.ptr, ws.ctl.ptr, sizeof(UpdateCtl),
                                cudaMemcpyDeviceToHost, s));
  DYNGB200_CUDA(cudaStreamSynchronize(s));
  const UpdateCtl r = *ws.host_ctl.ptr;
  ws.generation = std::max(ws.generation, r.last_generation);
  float sssp_ms = 0;
  cudaEventElapsedTime(&sssp_ms, e1, e2);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  t.version = g.version;
  finish_tree(ctx, g, t, r, blocks, operators, 0.0f, sssp_ms, nullptr, sched, launches0, st);
}

// update_each (update.hpp:331): the batch is applied once; every tree is brought up to date.
// Errors found before the batch is applied (for any of the objectives) leave the graph and every
// tree unchanged; an error after it poisons that tree only, the others are still updated, and the
// first error is rethrown.
void sssp_update_each(Context& ctx, Graph& g, const dyngb200_batch& batch, Tree* const* trees,
                      int count, dyngb200_stats* stats) {
  require_intact(g);
  for (int i = 0; i < count; ++i) select_engine(ctx, trees[i]->opt.cuda_engine);
  cudaStream_t s = ctx.stream;
  for (int i = 0; i < count; ++i)
    if (g.host_columns[trees[i]->opt.objective].dirty) graph_rescan_columns(ctx, g);
  const StagedBatch b = stage_batch(ctx, batch, g.k);
  // before the batch is applied: every objective's weights and 62-bit bound
  const int k = g.k;
  std::vector<long long> ext(2 * k + 1, 0);
  for (int c = 0; c < k; ++c) ext[2 * c + 1] = INT64_MAX;
  DevBuf<long long>& d_ext = ctx.ws.batch_extrema;  // kept: steady-state calls allocate nothing
  d_ext.reserve(ext.size());
  DYNGB200_CUDA(cudaMemcpyAsync(d_ext.ptr, ext.data(), ext.size() * sizeof(long long),
                                cudaMemcpyHostToDevice, s));
  if (b.ni + b.nd > 0) {
    k_batch_extrema<<<std::max(1, ctx.sm_count * 4), kThreads, 0, s>>>(
        b.ins_src, b.ins_dst, b.ins_w, b.ni, b.del_src, b.del_dst, b.nd, k, d_ext.ptr);
    ++ctx.launches;
    DYNGB200_CUDA(cudaGetLastError());
  }
  DYNGB200_CUDA(cudaMemcpyAsync(ext.data(), d_ext.ptr, ext.size() * sizeof(long long),
                                cudaMemcpyDeviceToHost, s));
  DYNGB200_CUDA(cudaStreamSynchronize(s));
  const long long n_bound = std::max<long long>(g.n, ext[2 * k]);
  for (int i = 0; i < count; ++i) {
    const int obj = trees[i]->opt.objective;
    if (b.ni > 0)
      expects(ext[2 * obj + 1] >= 1, "dyng::update_each: an insertion weight of objective " +
                                         std::to_string(obj) + " is below 1");
    const long long mw = std::max<long long>(g.host_columns[obj].max_w, b.ni > 0 ? ext[2 * obj] : 1);
    expects(distances_fit(n_bound, mw),
            "dyng::update_each: distances of objective " + std::to_string(obj) +
                " do not fit in 62 bits");
  }
  const std::vector<ColumnStats> pre_cols = g.host_columns;
  const GraphCounters pre_counters = g.host_counters;
  const uint64_t version0 = g.version;
  // the first tree applies the batch (an error before the commit leaves everything unchanged)
  std::string first_msg;
  dyngb200_status first_status = DYNGB200_OK;
  try {
    sssp_update(ctx, g, *trees[0], batch, dyngb200_schedule{}, stats ? &stats[0] : nullptr);
  } catch (const Error& e) {
    if (g.version == version0) throw;  // nothing was applied
    first_status = e.status;
    first_msg = e.what();
  }
  const UpdateCtl applied = *ctx.ws.host_ctl.ptr;
  for (int i = 1; i < count; ++i) {
    try {
      const int obj = trees[i]->opt.objective;
      sssp_rerun(ctx, g, *trees[i], applied, pre_cols, pre_counters,
                 b.ni > 0 ? ext[2 * obj] : 1, b.ins_w, stats ? &stats[i] : nullptr);
    } catch (const Error& e) {
      trees[i]->poisoned = true;
      if (first_status == DYNGB200_OK) {
        first_status = e.status;
        first_msg = e.what();
      }
    }
  }
  if (first_status != DYNGB200_OK) throw Error(first_status, first_msg);
}

// Tree arrays sized for the graph's vertex capacity (contents kept).
void tree_reserve(Context& ctx, Tree& t, long long n_cap) {
  if (!t.hist.ptr) {
    t.hist.reserve(1);
    DYNGB200_CUDA(cudaMemsetAsync(t.hist.ptr, 0, sizeof(TreeHistory), ctx.stream));
  }
  if (t.cap >= n_cap) return;
  const size_t keep = static_cast<size_t>(t.n);
  t.dist.reserve(static_cast<size_t>(n_cap), ctx.stream, keep);
  t.parent.reserve(static_cast<size_t>(n_cap), ctx.stream, keep);
  t.packed.reserve(static_cast<size_t>(n_cap), ctx.stream, keep);
  t.cap = n_cap;
}
// Contents of `src` into `dst` (same device); dst stays bound to its own graph handle.
void tree_copy(Context& ctx, Tree& dst, const Tree& src) {
  cudaStream_t s = ctx.stream;
  dst.version = src.version;
  dst.source = src.source;
  dst.opt = src.opt;
  dst.packed_bits = src.packed_bits;
  dst.trusted = src.trusted;
  dst.canonical = src.canonical;
  dst.poisoned = src.poisoned;
  dst.device = src.device;
  dst.n = src.n;
  tree_reserve(ctx, dst, std::max(src.cap, src.n));
  if (src.n > 0) {
    const size_t n = static_cast<size_t>(src.n);
    DYNGB200_CUDA(cudaMemcpyAsync(dst.dist.ptr, src.dist.ptr, n * sizeof(int64_t),
                                  cudaMemcpyDeviceToDevice, s));
    DYNGB200_CUDA(cudaMemcpyAsync(dst.parent.ptr, src.parent.ptr, n * sizeof(int32_t),
                                  cudaMemcpyDeviceToDevice, s));
    DYNGB200_CUDA(cudaMemcpyAsync(dst.packed.ptr, src.packed.ptr, n * sizeof(u64),
                                  cudaMemcpyDeviceToDevice, s));
  }
  if (src.hist.ptr)
    DYNGB200_CUDA(cudaMemcpyAsync(dst.hist.ptr, src.hist.ptr, sizeof(TreeHistory),
                                  cudaMemcpyDeviceToDevice, s));
  DYNGB200_CUDA(cudaStreamSynchronize(s));
}

void tree_canonicalize(Context& ctx, Graph& g, Tree& t) {
  const int grid = ctx.sm_count * 8;
  ++ctx.launches;
  k_canonicalize<<<grid, kThreads, 0, ctx.stream>>>(g.view(), t.opt.objective, t.source, t.n,
                                                    reinterpret_cast<const long long*>(t.dist.ptr),
                                                    t.parent.ptr);
  DYNGB200_CUDA(cudaGetLastError());
}

void tree_repack(Context& ctx, Tree& t, int bits) {
  const int grid = ctx.sm_count * 8;
  ++ctx.launches;
  k_pack<<<grid, kThreads, 0, ctx.stream>>>(t.n, bits, reinterpret_cast<const long long*>(t.dist.ptr),
                                            t.parent.ptr, t.packed.ptr);
  DYNGB200_CUDA(cudaGetLastError());
  t.packed_bits = bits;
}

// ------------------------------------------------------------------------------------------------
// compute() without allocation: the scratch of the persistent kernel in a fixed device array.
//
// For callers that must not allocate device memory once they are running: serving processes that
// reserve their whole device-memory budget at start-up and treat any later allocation as a fault,
// and host frameworks that own the device allocator and hand this library only the buffers it
// reads and writes.  The caller passes the graph (already built) and the two output arrays; every
// other byte the kernel needs lives in `g_static_scratch` below, a file-scope device array of
// kStaticScratchBytes that every GPU which loads this library holds until the process exits.
// ------------------------------------------------------------------------------------------------
constexpr long long kStaticMaxVertices = 1LL << 16;
// control block + packed words (8 B) + 15 int lists / stamp arrays + 3 int2 lists, per vertex
constexpr long long kStaticScratchBytes =
    4096 + kStaticMaxVertices * (8 + 15 * 4 + 3 * 8);

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

namespace {

constexpr int kMaxStaticDevices = 64;
unsigned char* g_static_ptr[kMaxStaticDevices] = {};
std::mutex g_static_mutex;

// The device address of g_static_scratch on the current device: looked up once per device (the
// array's host-side name is only a stand-in, never a device address).
unsigned char* static_scratch_for(int device) {
  expects(device >= 0 && device < kMaxStaticDevices, "static scratch: device out of range");
  std::lock_guard<std::mutex> lock(g_static_mutex);
  if (!g_static_ptr[device]) {
    void* ptr = nullptr;
    DYNGB200_CUDA(cudaGetSymbolAddress(&ptr, g_static_scratch));
    g_static_ptr[device] = static_cast<unsigned char*>(ptr);
  }
  return g_static_ptr[device];
}

}  // namespace

void sssp_compute_static(Graph& g, int32_t source, int objective, long long delta,
                         int64_t* distances, int32_t* parents, cudaStream_t s) {
  require_intact(g);
  const long long n = g.n;
  expects(n <= kStaticMaxVertices,
          "sssp::compute (static scratch): the graph has " + std::to_string(n) +
              " vertices; this entry point serves graphs of at most " +
              std::to_string(kStaticMaxVertices));
  expects(objective >= 0 && objective < g.k, "sssp::compute (static scratch): objective out of range");
  expects(source >= 0 && source < n, "sssp::compute (static scratch): source out of range");
  expects(delta >= 0, "sssp::compute (static scratch): delta must be >= 0");
  expects(distances && parents, "sssp::compute (static scratch): null output array");
  const ColumnStats cs = g.host_columns[objective];
  expects(!cs.dirty, "sssp::compute (static scratch): the graph's weight statistics need a rescan; "
                     "run sssp::compute or sssp::update on it once first");
  expects(cs.bad == 0, "sssp::compute (static scratch): an edge has a weight below 1");
  expects(distances_fit(n, cs.max_w), "sssp::compute (static scratch): distances do not fit in 62 bits");
  int device = 0;
  DYNGB200_CUDA(cudaGetDevice(&device));
  expects(device == g.device, "sssp::compute (static scratch): the graph belongs to another device");
  unsigned char* base = static_scratch_for(device);
  // carve the array: control block, packed words, int arrays, int2 lists
  static_assert(sizeof(UpdateCtl) <= 4096, "the control block fills the array's first 4 KB");
  const long long N = kStaticMaxVertices;
  auto* ctl = reinterpret_cast<UpdateCtl*>(base);
  auto* packed = reinterpret_cast<u64*>(base + 4096);
  int* ints = reinterpret_cast<int*>(base + 4096 + 8 * N);
  int2* pairs = reinterpret_cast<int2*>(base + 4096 + 8 * N + 15 * 4 * N);
  SsspParams p{};
  p.g = g.view();
  p.objective = objective;
  p.source = source;
  p.from_scratch = 1;
  p.dist = reinterpret_cast<long long*>(distances);
  p.parent = parents;
  p.packed = packed;
  p.stamp = ints + 0 * N;
  p.touch_stamp = ints + 1 * N;
  p.in_far = ints + 2 * N;
  p.flag = ints + 3 * N;
  p.ancestor = ints + 4 * N;
  p.candidates = ints + 5 * N;
  p.frontier = ints + 6 * N;
  p.near_a = ints + 7 * N;
  p.near_b = ints + 8 * N;
  p.far_a = ints + 9 * N;
  p.far_b = ints + 10 * N;
  p.touched = ints + 11 * N;
  p.cand_med = ints + 12 * N;
  p.near_med_a = ints + 13 * N;
  p.near_med_b = ints + 14 * N;
  p.heavy_a = pairs;
  p.heavy_b = pairs + N;
  p.pull_heavy = pairs + 2 * N;
  p.ctl = ctl;
  p.generation = 1;
  p.touch_gen = 1;
  p.heavy_degree = 256;
  p.small_frontier = kDefaultSmall;
  u64 bound = 0;
  const Packing pk = choose_packing(n, cs.max_w, &bound);
  p.tree_bits = pk.bits;
  p.tree_n = n;
  // the array keeps the previous call's contents: stamps and far marks must start at zero
  DYNGB200_CUDA(cudaMemsetAsync(ints, 0, 3 * N * sizeof(int), s));
  UpdateCtl init{};
  init.err_index = INT64_MAX;
  init.n_old = n;
  init.n_after = n;
  init.max_w = cs.max_w;
  init.delta = delta > 0 ? delta : default_delta(g.m > 1 ? g.m : 1, n, cs.sum_w);
  init.packing_bits = pk.bits;
  init.max_distance = bound;
  init.minimum = kPackedInf;
  init.sched_small = kDefaultSmall;
  DYNGB200_CUDA(cudaMemcpyAsync(ctl, &init, sizeof(UpdateCtl), cudaMemcpyHostToDevice, s));
  int sm = 0, coop = 0, per_sm = 0;
  DYNGB200_CUDA(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, device));
  DYNGB200_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
  expects(coop != 0, "sssp: the fused engine needs cooperative launch", DYNGB200_NOT_SUPPORTED);
  DYNGB200_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sssp, kThreads, 0));
  expects(per_sm >= 1, "sssp: the persistent kernel does not fit on an SM", DYNGB200_NOT_SUPPORTED);
  if (n > 0) {
    void* args[] = {&p};
    DYNGB200_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&k_sssp),
                                              dim3(per_sm * sm), dim3(kThreads), args, 0, s));
  }
  UpdateCtl r{};
  DYNGB200_CUDA(cudaMemcpyAsync(&r, ctl, sizeof(UpdateCtl), cudaMemcpyDeviceToHost, s));
  DYNGB200_CUDA(cudaStreamSynchronize(s));
  if (r.error & kErrTimeout) throw Error(DYNGB200_INTERNAL, "sssp: a grid barrier timed out");
  if (r.error & kErrNotConverged)
    throw Error(DYNGB200_INTERNAL, "sssp: the near-far loop did not converge");
}

}  // namespace dyngb200
