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
//      jumping that sums the weights along the tree in log(depth) rounds; kept on the device and
//      copied into the caller's host buffer when read (path_costs() is host memory, as in the
//      reference).
#include "handles.hpp"
#include "scan.cuh"


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

// ---- the result object ---------------------------------------------------------------------------

struct Mosp {
  int device = 0;
  int32_t source = 0;
  int num_k = 0;
  long long scale = 1;  // L = lcm(preferences)
  std::vector<int32_t> preferences;
  dyngb200_mosp_options opt{};
  std::vector<std::unique_ptr<dyngb200_tree_s>> trees;  // the K sssp trees
  Graph combined;      // the combined graph of the last finalize step
  Tree mosp[2];        // the MOSP tree: current and spare
  int cur = 0;
  DevBuf<int64_t> costs;  // n x K of the last compute() / update(), copied out when read
  bool has_costs = false;
  bool poisoned = false;
  uint64_t graph_id = 0, version = 0;
  // scratch of the finalize step
  DevBuf<int> out_count, fill, anc[2], missing;
  DevBuf<long long> cap, start;
  DevBuf<long long> scan_temp;  // tile totals of the out-row scan
  DevBuf<unsigned long long> totals;
  DevBuf<unsigned> first;
  DevBuf<int64_t> acc[2];

  Tree& tree() { return mosp[cur]; }
};

namespace {

long long preference_scale(const std::vector<int32_t>& prefs, int num_k, const char* what) {
  if (prefs.empty()) return 1;
  expects(static_cast<int>(prefs.size()) == num_k,
          std::string(what) + ": options.preferences has " + std::to_string(prefs.size()) +
              " values for " + std::to_string(num_k) +
              " objective(s) (one per objective, or none)");
  long long scale = 1;
  for (size_t i = 0; i < prefs.size(); ++i) {
    const long long p = prefs[i];
    expects(p >= 1, std::string(what) + ": options.preferences[" + std::to_string(i) + "] is " +
                        std::to_string(p) + "; a preference must be >= 1 (a lower value is a "
                        "higher priority)");
    scale = scale / std::gcd(scale, p) * p;
    expects(scale <= kMospMaxScale, std::string(what) + ": lcm(options.preferences) exceeds 2^20 "
                                                        "(the combined weights are scaled by it)");
  }
  return scale;
}

// The objectives and the scale the options select (mosp.cpp:134-153).
void resolve(Mosp& m, const Graph& g, const dyngb200_mosp_options& o, const char* what) {
  expects(o.delta >= 0, std::string(what) + ": options.delta must be >= 0 (0 = automatic), got " +
                            std::to_string(o.delta));
  expects(o.num_objectives >= 0 && o.num_objectives <= g.k,
          std::string(what) + ": options.num_objectives " + std::to_string(o.num_objectives) +
              " is out of range [0, " + std::to_string(g.k) + "] (the graph has " +
              std::to_string(g.k) + " weight column(s); 0 = all)");
  const int k = o.num_objectives > 0 ? o.num_objectives : g.k;
  expects(k >= 1, std::string(what) + ": mosp needs at least one weight column");
  expects(k <= kMospMaxObjectives, std::string(what) + ": " + std::to_string(k) +
                                       " objectives; mosp supports at most 64 (set "
                                       "options.num_objectives)");
  expects(o.num_preferences >= 0 && (o.num_preferences == 0 || o.preferences != nullptr),
          std::string(what) + ": options.preferences is null");
  std::vector<int32_t> prefs(o.preferences, o.preferences + o.num_preferences);
  m.scale = preference_scale(prefs, k, what);
  m.preferences = prefs;
  m.num_k = k;
  m.opt = o;
  m.opt.preferences = nullptr;  // kept in m.preferences
  m.opt.num_objectives = k;
}

void throw_status(dyngb200_status st) {
  if (st != DYNGB200_OK) throw Error(st, last_error());
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct FinalizeCounts {
  long long affected = 0;
  long long combined_edges = 0;
  long long iterations = 0;
  double combine_ms = 0, solve_ms = 0, costs_ms = 0;
};

// Path costs over the first `columns` weight columns of g along the current MOSP tree (n x
// columns, vertex-major): returns the scratch buffer that holds them (m.acc[0] or m.acc[1]).
int mosp_path_costs(Context& ctx, Graph& g, Mosp& m, int columns) {
  cudaStream_t s = ctx.stream;
  const long long n = g.n;
  const Tree& t = m.tree();
  const int grid = ctx.sm_count * 8;
  m.first.reserve(static_cast<size_t>(std::max(n, 1LL)));
  m.missing.reserve(2);  // [0] the lowest vertex without its tree edge, [1] "jump again"
  int* more_flag = m.missing.ptr + 1;
  for (int b = 0; b < 2; ++b) {
    m.anc[b].reserve(static_cast<size_t>(std::max(n, 1LL)));
    m.acc[b].reserve(static_cast<size_t>(std::max(n, 1LL)) * columns);
  }
  DYNGB200_CUDA(cudaMemsetAsync(m.first.ptr, 0xff, n * sizeof(unsigned), s));
  const int big = 0x7fffffff;
  DYNGB200_CUDA(cudaMemcpyAsync(m.missing.ptr, &big, sizeof(int), cudaMemcpyHostToDevice, s));
  const GraphView gv = g.view();
  if (g.props.allow_multi)
    k_mosp_first_scan<<<grid, kMospBlock, 0, s>>>(gv, n, t.parent.ptr, m.source, m.first.ptr);
  else
    k_mosp_first_index<<<grid, kMospBlock, 0, s>>>(gv, n, t.parent.ptr, m.source, m.first.ptr);
  k_mosp_costs_init<<<grid, kMospBlock, 0, s>>>(gv, n, t.parent.ptr, m.source, m.first.ptr,
                                                columns, m.acc[0].ptr, m.anc[0].ptr,
                                                m.missing.ptr);
  ctx.launches += 2;
  DYNGB200_CUDA(cudaGetLastError());
  int b = 0;
  for (int round = 0; round < 64; ++round) {
    DYNGB200_CUDA(cudaMemsetAsync(more_flag, 0, sizeof(int), s));
    k_mosp_costs_jump<<<grid, kMospBlock, 0, s>>>(n, columns, m.acc[b].ptr, m.anc[b].ptr,
                                                  m.acc[1 - b].ptr, m.anc[1 - b].ptr, more_flag);
    ++ctx.launches;
    DYNGB200_CUDA(cudaGetLastError());
    b = 1 - b;
    int more = 0;
    DYNGB200_CUDA(cudaMemcpyAsync(&more, more_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    DYNGB200_CUDA(cudaStreamSynchronize(s));
    if (!more) break;
  }
  int missing = big;
  DYNGB200_CUDA(cudaMemcpyAsync(&missing, m.missing.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
  DYNGB200_CUDA(cudaStreamSynchronize(s));
  if (missing != big) {
    int32_t p = -1;
    DYNGB200_CUDA(cudaMemcpy(&p, t.parent.ptr + missing, sizeof(int32_t), cudaMemcpyDeviceToHost));
    throw Error(DYNGB200_INVALID_ARGUMENT,
                "mosp: the MOSP tree edge (" + std::to_string(p) + ", " + std::to_string(missing) +
                    ") is not an edge of the graph (do the trees belong to this graph?)");
  }
  return b;
}

// Steps 2-3 of MOSP_Update on the current K trees (mosp.cpp:259-301): the combined graph, its
// tree, `affected` (count_affected) and the path costs.
FinalizeCounts mosp_finalize(Context& ctx, Graph& g, Mosp& m, bool count_affected) {
  FinalizeCounts out;
  cudaStream_t s = ctx.stream;
  const long long n = g.n;
  const long long n_cap = std::max(g.n_cap, n);
  const int K = m.num_k;
  const int stride = (K + 3) & ~3;
  auto t0 = std::chrono::steady_clock::now();
  // --- 1. the combined graph --------------------------------------------------------------------
  Graph& cg = m.combined;
  cg.device = g.device;
  cg.k = 1;
  cg.props = g.props;
  cg.props.directed = 1;
  cg.props.allow_multi = 1;  // no edge index: the solve reads rows only
  if (cg.n_cap < n_cap) {
    for (DevBuf<RowDesc>* d : {&cg.out_desc, &cg.in_desc}) d->reserve(static_cast<size_t>(n_cap));
    for (DevBuf<int32_t>* d : {&cg.out_cap, &cg.in_cap, &cg.out_dead, &cg.in_dead})
      d->reserve(static_cast<size_t>(n_cap));
    cg.n_cap = n_cap;
  }
  // in-rows: stride slots per vertex; out-rows: round4(degree) each, at most K n + 3 n_cap
  const long long arena = std::max(n_cap * stride, K * n + 3 * n_cap + 4);
  expects(arena < 0xffffffffLL, "mosp: the combined graph needs more than 2^32 row slots");
  for (DevBuf<int32_t>* d : {&cg.in_col, &cg.in_w, &cg.out_col, &cg.out_w})
    d->reserve(static_cast<size_t>(arena));
  cg.arena_cap = (arena + 3) & ~3LL;
  if (cg.arena_cap > static_cast<long long>(cg.out_col.count)) {
    for (DevBuf<int32_t>* d : {&cg.in_col, &cg.in_w, &cg.out_col, &cg.out_w})
      d->reserve(static_cast<size_t>(cg.arena_cap));
  }
  cg.counters.reserve(1);
  cg.columns.reserve(1);
  m.out_count.reserve(static_cast<size_t>(n_cap));
  m.fill.reserve(static_cast<size_t>(n_cap));
  m.cap.reserve(static_cast<size_t>(n_cap) + 1);
  m.start.reserve(static_cast<size_t>(n_cap) + 1);
  m.totals.reserve(2);
  m.scan_temp.reserve(static_cast<size_t>(scan_scratch(n_cap + 1)));
  DYNGB200_CUDA(cudaMemsetAsync(m.out_count.ptr, 0, n_cap * sizeof(int), s));
  DYNGB200_CUDA(cudaMemsetAsync(m.totals.ptr, 0, 2 * sizeof(unsigned long long), s));
  DYNGB200_CUDA(cudaMemsetAsync(m.cap.ptr + n_cap, 0, sizeof(long long), s));
  DYNGB200_CUDA(cudaMemsetAsync(cg.out_col.ptr, 0xff, cg.arena_cap * sizeof(int32_t), s));
  CombineInput in{};
  for (int k = 0; k < K; ++k) {
    in.parents[k] = m.trees[k]->t.parent.ptr;
    in.terms[k] = static_cast<int32_t>(m.preferences.empty() ? m.scale : m.scale / m.preferences[k]);
  }
  in.base = static_cast<int32_t>(m.scale * (K + 1));
  in.num_k = K;
  in.source = m.source;
  in.n = n;
  const int grid = ctx.sm_count * 8;
  const GraphView cv = cg.view();
  k_mosp_in_rows<<<grid, kMospBlock, 0, s>>>(in, cv, stride, n_cap, m.out_count.ptr, m.totals.ptr);
  k_mosp_out_caps<<<grid, kMospBlock, 0, s>>>(m.out_count.ptr, n_cap, m.cap.ptr);
  ctx.launches += exclusive_scan(m.cap.ptr, m.start.ptr, n_cap + 1, m.scan_temp.ptr, s);
  k_mosp_out_desc<<<grid, kMospBlock, 0, s>>>(cv, m.out_count.ptr, m.start.ptr, n_cap, m.fill.ptr);
  k_mosp_out_fill<<<grid, kMospBlock, 0, s>>>(cv, n, m.fill.ptr);
  ctx.launches += 5;
  DYNGB200_CUDA(cudaGetLastError());
  unsigned long long totals[2] = {0, 0};
  DYNGB200_CUDA(cudaMemcpyAsync(totals, m.totals.ptr, sizeof(totals), cudaMemcpyDeviceToHost, s));
  DYNGB200_CUDA(cudaStreamSynchronize(s));
  out.combined_edges = static_cast<long long>(totals[0]);
  GraphCounters gc{};
  gc.n = n;
  gc.m = out.combined_edges;
  gc.out_top = static_cast<u64>(cg.arena_cap);
  gc.in_top = static_cast<u64>(n_cap * stride);
  cg.host_counters = gc;
  cg.n = n;
  cg.m = gc.m;
  // the packing bound of the solve is `base` (mosp.cpp:319: max_weight = base)
  const ColumnStats cs{in.base, 0, static_cast<long long>(totals[1]), 0, 0};
  cg.host_columns.assign(1, cs);
  DYNGB200_CUDA(cudaMemcpyAsync(cg.counters.ptr, &cg.host_counters, sizeof(GraphCounters),
                                cudaMemcpyHostToDevice, s));
  DYNGB200_CUDA(cudaMemcpyAsync(cg.columns.ptr, cg.host_columns.data(), sizeof(ColumnStats),
                                cudaMemcpyHostToDevice, s));
  out.combine_ms = ms_since(t0);
  // --- 2. the MOSP tree: sssp::compute on the combined graph ----------------------------------
  t0 = std::chrono::steady_clock::now();
  Tree& prev = m.mosp[m.cur];
  Tree& next = m.mosp[1 - m.cur];
  next.source = m.source;
  next.opt = dyngb200_options{0, 0, DYNGB200_ENGINE_AUTOMATIC, 1};
  next.device = g.device;
  next.n = n;
  dyngb200_stats st{};
  sssp_compute(ctx, cg, next, &st);
  out.iterations = st.iterations;
  // --- 3. affected ------------------------------------------------------------------------------
  if (count_affected) {
    DYNGB200_CUDA(cudaMemsetAsync(m.totals.ptr, 0, sizeof(unsigned long long), s));
    const long long n_old = prev.dist.ptr ? std::min(prev.n, n) : 0;
    k_mosp_changed<<<grid, kMospBlock, 0, s>>>(prev.dist.ptr, prev.parent.ptr, n_old,
                                               next.dist.ptr, next.parent.ptr, n, m.totals.ptr);
    ++ctx.launches;
    DYNGB200_CUDA(cudaGetLastError());
    DYNGB200_CUDA(cudaMemcpyAsync(totals, m.totals.ptr, sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, s));
    DYNGB200_CUDA(cudaStreamSynchronize(s));
    out.affected = static_cast<long long>(totals[0]);
  }
  m.cur = 1 - m.cur;
  out.solve_ms = ms_since(t0);
  // --- 4. path costs ----------------------------------------------------------------------------
  t0 = std::chrono::steady_clock::now();
  m.has_costs = false;
  if (m.opt.compute_path_costs) {
    const int b = mosp_path_costs(ctx, g, m, K);
    m.costs.swap(m.acc[b]);  // kept on the device; dyngb200_mosp_path_costs copies them out
    m.has_costs = true;
  }
  out.costs_ms = ms_since(t0);
  return out;
}

}  // namespace dyngb200

struct dyngb200_mosp_s {
  dyngb200::Mosp m;
};

using dyngb200::guarded;

namespace {

using namespace dyngb200;

dyngb200_mosp_options default_mosp_options() {
  dyngb200_mosp_options o{};
  o.compute_path_costs = 1;
  o.validate_inputs = 1;
  return o;
}

Mosp& usable(dyngb200_mosp r, const char* what) {
  expects(r != nullptr, std::string(what) + ": null result");
  expects(!r->m.poisoned,
          std::string(what) + ": the result was left unusable by a failed update; recompute it "
                              "with mosp::compute() (or import valid trees with from_arrays())",
          DYNGB200_STALE_RESULT);
  return r->m;
}

dyngb200_options objective_options(const Mosp& m, int k) {
  return dyngb200_options{m.opt.delta, k, DYNGB200_ENGINE_AUTOMATIC, m.opt.validate_inputs};
}

}  // namespace

extern "C" {

dyngb200_status dyngb200_mosp_compute(dyngb200_context ctx, dyngb200_graph g, int32_t source,
                                      const dyngb200_mosp_options* opt, dyngb200_mosp* out) {
  return guarded([&] {
    expects(ctx && g && out, "mosp::compute: null argument");
    Context& c = ctx->ctx;
    Graph& gr = g->g;
    DeviceGuard guard(c.device);
    expects(gr.device == c.device, "mosp::compute: the graph belongs to another device");
    auto h = std::make_unique<dyngb200_mosp_s>();
    Mosp& m = h->m;
    resolve(m, gr, opt ? *opt : default_mosp_options(), "mosp::compute");
    expects(source >= 0 && source < gr.n, "mosp::compute: source " + std::to_string(source) +
                                              " is out of range [0, " + std::to_string(gr.n) + ")");
    m.source = source;
    m.device = c.device;
    for (int k = 0; k < m.num_k; ++k) {
      const dyngb200_options o = objective_options(m, k);
      dyngb200_tree t = nullptr;
      throw_status(dyngb200_sssp_compute(ctx, g, source, &o, &t, nullptr));
      m.trees.emplace_back(t);
    }
    mosp_finalize(c, gr, m, false);
    m.graph_id = gr.id;
    m.version = gr.version;
    *out = h.release();
  });
}

dyngb200_status dyngb200_mosp_from_arrays(dyngb200_context ctx, dyngb200_graph g, int32_t source,
                                          int32_t num_trees, const int64_t* const* distances,
                                          const int32_t* const* parents, int64_t n,
                                          int32_t memory, int32_t canonicalize,
                                          const dyngb200_mosp_options* opt, dyngb200_mosp* out) {
  return guarded([&] {
    expects(ctx && g && out, "mosp::result::from_arrays: null argument");
    Context& c = ctx->ctx;
    Graph& gr = g->g;
    DeviceGuard guard(c.device);
    auto h = std::make_unique<dyngb200_mosp_s>();
    Mosp& m = h->m;
    resolve(m, gr, opt ? *opt : default_mosp_options(), "mosp::result::from_arrays");
    expects(num_trees == m.num_k, "mosp::result::from_arrays: " + std::to_string(num_trees) +
                                      " trees for " + std::to_string(m.num_k) + " objective(s)");
    expects(distances && parents, "mosp::result::from_arrays: null array list");
    m.source = source;
    m.device = c.device;
    for (int k = 0; k < m.num_k; ++k) {
      const dyngb200_options o = objective_options(m, k);
      dyngb200_tree t = nullptr;
      throw_status(dyngb200_tree_from_arrays(ctx, g, source, distances[k], parents[k], n, memory,
                                             canonicalize, &o, &t));
      m.trees.emplace_back(t);
    }
    mosp_finalize(c, gr, m, false);
    m.graph_id = gr.id;
    m.version = gr.version;
    *out = h.release();
  });
}

dyngb200_status dyngb200_mosp_update(dyngb200_context ctx, dyngb200_graph g,
                                     const dyngb200_batch* batch, dyngb200_mosp r,
                                     dyngb200_mosp_stats* stats, dyngb200_stats* objective_stats) {
  return guarded([&] {
    expects(ctx && g && batch, "mosp::update: null argument");
    Mosp& m = usable(r, "mosp::update");
    Context& c = ctx->ctx;
    Graph& gr = g->g;
    DeviceGuard guard(c.device);
    std::vector<Tree*> ts;
    for (auto& t : m.trees) {
      expect_tree_current(gr, t->t, "mosp::update");
      ts.push_back(&t->t);
    }
    expect_batch(gr, *batch, "mosp::update");
    std::vector<dyngb200_stats> st(static_cast<size_t>(m.num_k));
    const uint64_t version0 = gr.version;
    FinalizeCounts f;
    try {
      sssp_update_each(c, gr, *batch, ts.data(), m.num_k, st.data());
      f = mosp_finalize(c, gr, m, true);
    } catch (...) {
      if (gr.version != version0) m.poisoned = true;  // the batch was applied: K trees stale
      throw;
    }
    m.version = gr.version;
    if (objective_stats)
      std::memcpy(objective_stats, st.data(), st.size() * sizeof(dyngb200_stats));
    if (stats) {
      dyngb200_mosp_stats o{};
      o.batch = st[0].batch;
      o.affected = f.affected;
      o.combined_edges = f.combined_edges;
      o.preference_scale = m.scale;
      o.iterations = f.iterations;
      for (const auto& x : st) o.iterations += x.iterations;
      o.converged = 1;
      o.combine_ms = static_cast<float>(f.combine_ms);
      o.solve_ms = static_cast<float>(f.solve_ms);
      o.costs_ms = static_cast<float>(f.costs_ms);
      *stats = o;
    }
  });
}

dyngb200_status dyngb200_mosp_destroy(dyngb200_mosp r) {
  return guarded([&] { delete r; });
}

dyngb200_status dyngb200_mosp_info(dyngb200_mosp r, int32_t* num_objectives, int64_t* num_vertices,
                                   int64_t* preference_scale, int32_t* source,
                                   uint64_t* graph_version) {
  return guarded([&] {
    expects(r != nullptr, "mosp::result: null result");
    const Mosp& m = r->m;
    if (num_objectives) *num_objectives = m.num_k;
    if (num_vertices) *num_vertices = m.mosp[m.cur].n;
    if (preference_scale) *preference_scale = m.scale;
    if (source) *source = m.source;
    if (graph_version) *graph_version = m.version;
  });
}

dyngb200_status dyngb200_mosp_tree(dyngb200_mosp r, int32_t objective, dyngb200_tree* out) {
  return guarded([&] {
    Mosp& m = usable(r, "mosp::result::parents");
    expects(out != nullptr, "mosp::result: null output");
    expects(objective >= 0 && objective < m.num_k,
            "mosp::result: objective " + std::to_string(objective) + " is out of range [0, " +
                std::to_string(m.num_k) + ")");
    *out = m.trees[static_cast<size_t>(objective)].get();
  });
}

dyngb200_status dyngb200_mosp_combined(dyngb200_mosp r, int64_t* distances, int32_t* parents,
                                       int32_t memory) {
  return guarded([&] {
    Mosp& m = usable(r, "mosp::result::combined_distances");
    DeviceGuard guard(m.device);
    const Tree& t = m.tree();
    const cudaMemcpyKind kind =
        memory == DYNGB200_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (distances && t.n > 0)
      DYNGB200_CUDA(cudaMemcpy(distances, t.dist.ptr, t.n * sizeof(int64_t), kind));
    if (parents && t.n > 0)
      DYNGB200_CUDA(cudaMemcpy(parents, t.parent.ptr, t.n * sizeof(int32_t), kind));
  });
}

dyngb200_status dyngb200_mosp_path_costs(dyngb200_mosp r, int64_t* costs) {
  return guarded([&] {
    Mosp& m = usable(r, "mosp::result::path_costs");
    expects(m.has_costs, "mosp::result::path_costs: the path costs were not computed "
                         "(options.compute_path_costs was false at the last compute() or update())");
    const size_t count = static_cast<size_t>(m.mosp[m.cur].n) * static_cast<size_t>(m.num_k);
    expects(costs != nullptr || count == 0, "mosp::result::path_costs: null output");
    DeviceGuard guard(m.device);
    if (count) DYNGB200_CUDA(cudaMemcpy(costs, m.costs.ptr, count * sizeof(int64_t),
                                        cudaMemcpyDeviceToHost));
  });
}

dyngb200_status dyngb200_mosp_path_costs_columns(dyngb200_context ctx, dyngb200_graph g,
                                                 dyngb200_mosp r, int32_t columns, int64_t* costs) {
  return guarded([&] {
    expects(ctx && g, "mosp path costs: null argument");
    Mosp& m = usable(r, "mosp path costs");
    Graph& gr = g->g;
    DeviceGuard guard(ctx->ctx.device);
    expects(gr.id == m.graph_id && gr.version == m.version,
            "mosp path costs: the result does not match the graph's current version",
            DYNGB200_STALE_RESULT);
    expects(columns >= 1 && columns <= gr.k, "mosp path costs: columns " +
                                                 std::to_string(columns) + " is out of range [1, " +
                                                 std::to_string(gr.k) + "]");
    const int b = mosp_path_costs(ctx->ctx, gr, m, columns);
    const size_t count = static_cast<size_t>(gr.n) * static_cast<size_t>(columns);
    expects(costs != nullptr || count == 0, "mosp path costs: null output");
    if (count) DYNGB200_CUDA(cudaMemcpy(costs, m.acc[b].ptr, count * sizeof(int64_t),
                                        cudaMemcpyDeviceToHost));
  });
}

dyngb200_status dyngb200_mosp_set_options(dyngb200_mosp r, const dyngb200_mosp_options* opt) {
  return guarded([&] {
    Mosp& m = usable(r, "mosp::result::set_options");
    expects(opt != nullptr, "mosp::result::set_options: null options");
    expects(opt->delta >= 0, "mosp::result::set_options: options.delta must be >= 0");
    const int k = opt->num_objectives;
    expects(k == 0 || k == m.num_k, "mosp::result::set_options: num_objectives is fixed at compute()");
    std::vector<int32_t> prefs(opt->preferences, opt->preferences + opt->num_preferences);
    const bool same = prefs == m.preferences ||
                      (prefs.empty() && std::all_of(m.preferences.begin(), m.preferences.end(),
                                                    [](int32_t p) { return p == 1; })) ||
                      (m.preferences.empty() && std::all_of(prefs.begin(), prefs.end(),
                                                            [](int32_t p) { return p == 1; }) &&
                       static_cast<int>(prefs.size()) == m.num_k);
    expects(same, "mosp::result::set_options: preferences are fixed at compute()");
    m.opt.delta = opt->delta;
    m.opt.compute_path_costs = opt->compute_path_costs;
    m.opt.validate_inputs = opt->validate_inputs;
    for (auto& t : m.trees) t->t.opt.delta = opt->delta;
  });
}

}  // extern "C"
