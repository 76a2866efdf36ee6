// Shared device/host definitions of the dyng_b200 library (CUDA 12.9, sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace dyngb200 {

using u64 = unsigned long long;

constexpr int64_t kInfinity = INT64_MAX / 4;  // sssp_infinity of the reference (problem.hpp:340)
constexpr u64 kPackedInf = ~0ULL;
constexpr int32_t kDead = -1;  // tombstone in a slack row's column slot
constexpr int kDefaultSmall = 256;  // the heuristic: frontiers up to 256 vertices run on one block

// Device error bits (the sticky error word; the reference's util/device_error_flags.hpp:9-43
// has capacity / invalid_input / parent_cycle / internal).
enum : unsigned {
  kErrCapacity = 1u << 0,       // vertex or arena capacity exceeded: the host grows and retries
  kErrInvalidBatch = 1u << 1,   // negative id, weight < 1, growth not allowed, policy error
  kErrParentCycle = 1u << 2,    // pointer jumping still active in its last round
  kErrOverflow = 1u << 3,       // an input distance does not fit the packing bound
  kErrInternal = 1u << 4,       // mirror mismatch or another broken invariant
  kErrTimeout = 1u << 5,        // a bounded wait ran out (grid barrier, loop cap)
  kErrNotConverged = 1u << 6,   // the near-far loop exceeded its iteration cap
};

// One slack row: entries [start, start + len) of the arena, `len` counting tombstones.
struct RowDesc {
  uint32_t start;
  int32_t len;
};

// Per-objective column statistics kept on the device (max weight, how many edges carry it, sum).
struct ColumnStats {
  long long max_w;
  long long count_at_max;
  long long sum_w;
  int dirty;  // count_at_max reached 0: max_w is only an upper bound until rescanned
  int bad;    // weights below 1 (sssp refuses the column while any is left)
};

// Device-resident graph counters.
struct GraphCounters {
  long long n;          // vertices
  long long m;          // live edges
  u64 out_top, in_top;  // arena allocation tops (entries)
  u64 out_garbage, in_garbage;  // entries abandoned by relocated rows
  long long dead_out, dead_in;  // tombstones still stored
  long long idx_live, idx_dead; // edge index: live keys and deleted markers
};

// The device view of one slack-row graph (out-rows plus the in-edge mirror).
struct GraphView {
  RowDesc* out_desc;
  int32_t* out_cap;
  int32_t* out_dead;
  int32_t* out_col;
  int32_t* out_w;  // k columns of arena_cap entries each (objective-major)
  RowDesc* in_desc;
  int32_t* in_cap;
  int32_t* in_dead;
  int32_t* in_col;
  int32_t* in_w;
  long long arena_cap;
  long long n_cap;
  int k;
  int sorted;       // row_order::sorted (export order only)
  int allow_multi;  // multi_edges::allow
  GraphCounters* counters;
  ColumnStats* columns;  // k entries
  // Edge index (simple graphs): open addressing on (u << 32 | v) -> absolute slot of the edge in
  // the out arena and in the in arena.  emask + 1 entries; empty keys ~0, deleted ~0 - 1.
  unsigned long long* ekey;
  unsigned* eout;
  unsigned* ein;
  long long emask;
};

constexpr unsigned long long kKeyEmpty = ~0ULL;
constexpr unsigned long long kKeyDeleted = ~0ULL - 1;

__host__ __device__ inline int parent_bits_for(long long n) {
  int bits = 1;
  while (((1ULL << bits) - 1) < static_cast<u64>(n)) ++bits;
  return bits;
}

// Packed (distance << bits | parent) words; bits == 0 holds the distance alone (the format of the
// reference's kernels.cuh:51-92).
struct Packing {
  int bits;
  u64 no_parent;
  __host__ __device__ u64 pack(u64 d, int32_t p) const {
    if (bits == 0) return d;
    return (d << bits) | (p < 0 ? no_parent : static_cast<u64>(p));
  }
  __host__ __device__ u64 dist(u64 w) const { return w >> bits; }
  __host__ __device__ int32_t parent(u64 w) const {
    const u64 p = w & no_parent;
    return p == no_parent ? -1 : static_cast<int32_t>(p);
  }
  __host__ __device__ u64 max_distance() const { return (kPackedInf >> bits) - 1; }
};

// The CUDA engines' packing rule (cuda.cu:225-234): packed if (n-1)*max_w fits next to the parent
// bits, distance-only otherwise.
__host__ __device__ inline Packing choose_packing(long long n, long long max_w, u64* bound) {
  const u64 w = static_cast<u64>(max_w > 1 ? max_w : 1);
  const u64 hops = static_cast<u64>(n - 1 > 1 ? n - 1 : 1);
  *bound = w * hops;
  Packing p;
  p.bits = parent_bits_for(n);
  p.no_parent = (1ULL << p.bits) - 1;
  if (*bound <= p.max_distance()) return p;
  p.bits = 0;
  p.no_parent = 0;
  return p;
}

// The reference's default near-far width (sssp.cpp:136-145): max(1, 32 * avg weight / avg degree).
__host__ __device__ inline long long default_delta(long long m, long long n, long long wsum) {
  if (m <= 0 || n <= 0) return 1;
  const double avg_w = static_cast<double>(wsum) / static_cast<double>(m);
  const double avg_deg = static_cast<double>(m) / static_cast<double>(n);
  const long long d = static_cast<long long>(32.0 * avg_w / avg_deg);
  return d > 1 ? d : 1;
}

// The 62-bit check (sssp.cpp:147-152).
__host__ __device__ inline bool distances_fit(long long n, long long max_w) {
  const u64 w = static_cast<u64>(max_w > 1 ? max_w : 1);
  const u64 hops = static_cast<u64>(n - 1 > 1 ? n - 1 : 1);
  const u64 output_max = static_cast<u64>(kInfinity / 2 - 1);
  return w <= output_max / hops;
}

#ifdef __CUDACC__
__device__ __forceinline__ u64 mix64(u64 x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  return x;
}

__device__ __forceinline__ u64 edge_key(int32_t u, int32_t v) {
  return (static_cast<u64>(static_cast<uint32_t>(u)) << 32) | static_cast<uint32_t>(v);
}

// Slot of a live key in the edge index, or -1.
__device__ __forceinline__ long long index_find(const GraphView& g, u64 key) {
  long long h = static_cast<long long>(mix64(key) & static_cast<u64>(g.emask));
  for (long long probe = 0; probe <= g.emask; ++probe) {
    const u64 cur = g.ekey[h];
    if (cur == key) return h;
    if (cur == kKeyEmpty) return -1;
    h = (h + 1) & g.emask;
  }
  return -1;
}

// Claim a slot for a key that is not in the index (an empty or deleted slot); -1 if full.
// *reused tells whether a deleted marker was replaced.
__device__ __forceinline__ long long index_insert(const GraphView& g, u64 key, bool* reused) {
  long long h = static_cast<long long>(mix64(key) & static_cast<u64>(g.emask));
  for (long long probe = 0; probe <= g.emask; ++probe) {
    u64 cur = g.ekey[h];
    while (cur == kKeyEmpty || cur == kKeyDeleted) {
      const u64 prev = atomicCAS(&g.ekey[h], cur, key);
      if (prev == cur) {
        *reused = cur == kKeyDeleted;
        return h;
      }
      cur = prev;
    }
    h = (h + 1) & g.emask;
  }
  return -1;
}

// The slot of `key`: found along its probe chain, or else claimed (the first deleted slot of the
// chain, else the empty slot that ends it).  One walk of the chain instead of a find and an
// insert.  Concurrent calls must not insert the same key (the applier inserts each pair once).
__device__ __forceinline__ long long index_find_or_insert(const GraphView& g, u64 key,
                                                          bool* inserted, bool* reused) {
  long long h = static_cast<long long>(mix64(key) & static_cast<u64>(g.emask));
  long long first_deleted = -1;
  for (long long probe = 0; probe <= g.emask; ++probe) {
    const u64 cur = g.ekey[h];
    if (cur == key) {
      *inserted = false;
      return h;
    }
    if (cur == kKeyDeleted && first_deleted < 0) first_deleted = h;
    if (cur == kKeyEmpty) break;
    h = (h + 1) & g.emask;
  }
  // not in the index: claim the first deleted slot seen, else insert from scratch
  if (first_deleted >= 0 && atomicCAS(&g.ekey[first_deleted], kKeyDeleted, key) == kKeyDeleted) {
    *inserted = true;
    *reused = true;
    return first_deleted;
  }
  *inserted = true;
  return index_insert(g, key, reused);
}

__device__ __forceinline__ int ld_cg(const int* p) { return __ldcg(p); }
__device__ __forceinline__ u64 ld_cg(const u64* p) { return __ldcg(p); }
__device__ __forceinline__ long long ld_cg(const long long* p) { return __ldcg(p); }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Warp-aggregated reservation of one slot of a shared list (one atomicAdd per converged group).
__device__ __forceinline__ int append_slot(int* counter) {
  const unsigned mask = __activemask();
  const int leader = __ffs(mask) - 1;
  const int lane = threadIdx.x & 31;
  const int rank = __popc(mask & ((1u << lane) - 1));
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(mask));
  base = __shfl_sync(mask, base, leader);
  return base + rank;
}

__device__ __forceinline__ void set_error(unsigned* word, unsigned bits) { atomicOr(word, bits); }
#endif

}  // namespace dyngb200
