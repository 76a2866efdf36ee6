// dyng::mosp on the device: K shortest-path trees of one graph (the sssp trees of its first K
// weight columns), the combined graph they span, its shortest-path tree (the MOSP tree) and the
// K objective values of every MOSP path.  The reference's cpp/include/dyng/mosp.hpp and
// cpp/src/algorithms/mosp/mosp.cpp (compute / update / from_arrays, the finalize step at
// mosp.cpp:259-350); the combined graph of mosp/cuda.cu and mosp/sequential.cpp:33-170; the path
// costs of mosp/sequential.cpp:172-232.
//
// The finalize step, all on the device after the K trees are current:
//   1. the combined graph: vertex v's in-row lists its distinct parents among the K trees, edge
//      (p, v) weighted base - sum of the preference terms of the trees that hold it
//      (base = L (K + 1), term_i = L / Pref_i, L = lcm(Pref)); in-rows have a fixed stride
//      round4(K), out-rows are counted, scanned and filled.  The combined graph is a graph of
//      this library (slack rows, no edge index), so
//   2. the MOSP tree is sssp::compute on it: the same persistent kernel, lowest-id ties, default
//      width from the combined graph's edges and weight sum (as the reference), packing bound
//      `base`;
//   3. `affected` compares the new MOSP tree with the previous one (two trees, swapped);
//   4. path costs: the first edge p -> v of each tree edge in the graph's row order (the edge
//      index of a simple graph, else a warp-per-row scan keeping the lowest slot), then pointer
//      jumping that sums the weights along the tree in log(depth) rounds; copied to the host
//      (the reference keeps path costs in host memory on every backend).
#include "handles.hpp"

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

namespace dyngb200 {

constexpr int kMospMaxObjectives = 64;             // mosp::max_objectives (mosp.hpp:68)
constexpr long long kMospMaxScale = 1LL << 20;     // mosp::max_preference_scale (mosp.hpp:76)
constexpr unsigned kNoSlot = 0xffffffffu;

namespace {

constexpr int kMospBlock = 256;

struct CombineInput {
  const int32_t* parents[kMospMaxObjectives];  // the K trees' parent arrays
  int32_t terms[kMospMaxObjectives];           // L / Pref_i
  int32_t base;                                // L (K + 1)
  int num_k;
  int32_t source;
  long long n;
};

// Parent k of v carries a combined edge if it is the first occurrence of its value among the K
// parents; its weight is base minus the terms of every tree that holds the same parent
// (mosp/sequential.cpp:33-55).
__device__ __forceinline__ bool combined_edge(const CombineInput& in, long long v, int k,
                                              int32_t& p, int32_t& w) {
  p = in.parents[k][v];
  if (p < 0) return false;
  for (int j = 0; j < k; ++j)
    if (in.parents[j][v] == p) return false;
  int32_t wt = in.base - in.terms[k];
  for (int j = k + 1; j < in.num_k; ++j)
    if (in.parents[j][v] == p) wt -= in.terms[j];
  w = wt;
  return true;
}

// In-rows of the combined graph (stride slots per vertex), the out-degree of every parent, and
// the edge count and weight sum (one atomic pair per warp).
__global__ void k_mosp_in_rows(CombineInput in, GraphView cg, int stride, long long n_cap,
                               int* out_count, unsigned long long* totals) {
  const int lane = threadIdx.x & 31;
  const long long step = static_cast<long long>(gridDim.x) * blockDim.x;
  const long long first = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  // every lane runs the same number of iterations (the warp reduction below)
  for (long long v0 = first - lane; v0 < n_cap; v0 += step) {
    const long long v = v0 + lane;
    long long edges = 0, wsum = 0;
    if (v < n_cap) {
      const long long at = v * stride;
      int cnt = 0;
      if (v < in.n && v != in.source) {
        for (int k = 0; k < in.num_k; ++k) {
          int32_t p, w;
          if (!combined_edge(in, v, k, p, w)) continue;
          cg.in_col[at + cnt] = p;
          cg.in_w[at + cnt] = w;
          atomicAdd(&out_count[p], 1);
          ++cnt;
          wsum += w;
        }
      }
      for (int c = cnt; c < stride; ++c) cg.in_col[at + c] = kDead;
      cg.in_desc[v] = RowDesc{static_cast<uint32_t>(at), cnt};
      cg.in_cap[v] = stride;
      cg.in_dead[v] = 0;
      edges = cnt;
    }
    for (int o = 16; o > 0; o >>= 1) {
      edges += __shfl_down_sync(0xffffffffu, edges, o);
      wsum += __shfl_down_sync(0xffffffffu, wsum, o);
    }
    if (lane == 0 && edges) {
      atomicAdd(&totals[0], static_cast<unsigned long long>(edges));
      atomicAdd(&totals[1], static_cast<unsigned long long>(wsum));
    }
  }
}

// Out-row capacities: round4(out-degree) slots, so rows start on 16-byte boundaries.
__global__ void k_mosp_out_caps(const int* out_count, long long n_cap, long long* cap) {
  for (long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; p < n_cap;
       p += static_cast<long long>(gridDim.x) * blockDim.x)
    cap[p] = (static_cast<long long>(out_count[p]) + 3) & ~3LL;
}

__global__ void k_mosp_out_desc(GraphView cg, const int* out_count, const long long* start,
                                long long n_cap, int* fill) {
  for (long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; p < n_cap;
       p += static_cast<long long>(gridDim.x) * blockDim.x) {
    cg.out_desc[p] = RowDesc{static_cast<uint32_t>(start[p]), out_count[p]};
    cg.out_cap[p] = static_cast<int32_t>(start[p + 1] - start[p]);
    cg.out_dead[p] = 0;
    fill[p] = 0;
  }
}

// Out-rows from the in-rows (the order inside a row does not matter: the solve breaks ties by
// the lowest parent id, whatever the order of its pushes).
__global__ void k_mosp_out_fill(GraphView cg, long long n, int* fill) {
  for (long long v = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; v < n;
       v += static_cast<long long>(gridDim.x) * blockDim.x) {
    const RowDesc d = cg.in_desc[v];
    for (int c = 0; c < d.len; ++c) {
      const int32_t p = cg.in_col[d.start + c];
      const RowDesc o = cg.out_desc[p];
      const int pos = atomicAdd(&fill[p], 1);
      cg.out_col[o.start + pos] = static_cast<int32_t>(v);
      cg.out_w[o.start + pos] = cg.in_w[d.start + c];
    }
  }
}

// Vertices whose (distance, parent) differ between the previous MOSP tree (n_old vertices; the
// rest count as unreachable) and the new one.
__global__ void k_mosp_changed(const int64_t* od, const int32_t* op, long long n_old,
                               const int64_t* nd, const int32_t* np, long long n,
                               unsigned long long* count) {
  long long c = 0;
  for (long long v = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; v < n;
       v += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int64_t d0 = v < n_old ? od[v] : kInfinity;
    const int32_t p0 = v < n_old ? op[v] : -1;
    c += (d0 != nd[v] || p0 != np[v]) ? 1 : 0;
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, static_cast<unsigned long long>(c));
}

// The first slot of every MOSP tree edge (p, v) in row p, by a scan of the out-rows (one warp
// per row; slots are in row order, so the lowest slot is the first edge).
__global__ void k_mosp_first_scan(GraphView g, long long n, const int32_t* cpar, int32_t source,
                                  unsigned* first) {
  const int lane = threadIdx.x & 31;
  const long long warps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
  for (long long p = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; p < n;
       p += warps) {
    const RowDesc d = g.out_desc[p];
    for (int e = lane; e < d.len; e += 32) {
      const int32_t x = g.out_col[d.start + e];
      if (x >= 0 && x != source && cpar[x] == p) atomicMin(&first[x], d.start + e);
    }
  }
}

// The same through the edge index of a simple graph (one edge per pair).
__global__ void k_mosp_first_index(GraphView g, long long n, const int32_t* cpar, int32_t source,
                                   unsigned* first) {
  for (long long v = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; v < n;
       v += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int32_t p = cpar[v];
    if (p < 0 || v == source) continue;
    const long long ie = index_find(g, edge_key(p, static_cast<int32_t>(v)));
    if (ie >= 0) first[v] = g.eout[ie];
  }
}

// Pointer-jumping state: acc[v] = the weights from anc[v] down to v (C columns), anc[v] = the
// tree ancestor the sum starts at (-1 once the sum reaches the source).  A tree edge that is not
// an edge of the graph records its head in *missing (the lowest such vertex).
__global__ void k_mosp_costs_init(GraphView g, long long n, const int32_t* cpar, int32_t source,
                                  const unsigned* first, int columns, int64_t* acc, int32_t* anc,
                                  int* missing) {
  for (long long v = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; v < n;
       v += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int32_t p = v == source ? -1 : cpar[v];
    int64_t* a = acc + v * columns;
    if (v == source) {
      for (int j = 0; j < columns; ++j) a[j] = 0;
      anc[v] = -1;
      continue;
    }
    if (p < 0) {
      for (int j = 0; j < columns; ++j) a[j] = kInfinity;
      anc[v] = -1;
      continue;
    }
    const unsigned slot = first[v];
    if (slot == kNoSlot) {
      atomicMin(missing, static_cast<int>(v));
      for (int j = 0; j < columns; ++j) a[j] = kInfinity;
      anc[v] = -1;
      continue;
    }
    for (int j = 0; j < columns; ++j)
      a[j] = g.out_w[static_cast<long long>(j) * g.arena_cap + slot];
    anc[v] = p;
  }
}

__global__ void k_mosp_costs_jump(long long n, int columns, const int64_t* acc_in,
                                  const int32_t* anc_in, int64_t* acc_out, int32_t* anc_out,
                                  int* more) {
  int again = 0;
  for (long long v = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; v < n;
       v += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int32_t a = anc_in[v];
    const int64_t* src = acc_in + v * columns;
    int64_t* dst = acc_out + v * columns;
    if (a < 0) {
      for (int j = 0; j < columns; ++j) dst[j] = src[j];
      anc_out[v] = -1;
      continue;
    }
    const int64_t* up = acc_in + static_cast<long long>(a) * columns;
    for (int j = 0; j < columns; ++j) dst[j] = src[j] + up[j];
    const int32_t next = anc_in[a];
    anc_out[v] = next;
    again |= next >= 0;
  }
  if (__any_sync(0xffffffffu, again) && (threadIdx.x & 31) == 0) *more = 1;
}

}  // namespace
