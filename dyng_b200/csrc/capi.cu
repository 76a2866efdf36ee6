// The C ABI (include/dyngb200.h): handles, argument checks on the host, error translation, and
// the host-side parts of the reference's API that are not on the device path (graph
// construction with the reference's normalisation, tree import and validation).
#include "internal.hpp"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "handles.hpp"

namespace dyngb200 {

void expect_tree_current(const Graph& g, const Tree& t, const char* what) {
  if (t.poisoned)
    throw Error(DYNGB200_STALE_RESULT,
                std::string(what) + ": the result was left unusable by a failed update; recompute "
                                    "it with sssp::compute() (or import a valid tree)");
  if (t.graph_id != g.id || t.version != g.version)
    throw Error(DYNGB200_STALE_RESULT,
                std::string(what) + ": the result does not match the graph's current version");
  if (t.device != g.device)
    throw Error(DYNGB200_INVALID_ARGUMENT, std::string(what) + ": result on another device");
}

void expect_batch(const Graph& g, const dyngb200_batch& b, const char* what) {
  expects(b.num_insertions >= 0 && b.num_deletions >= 0, std::string(what) + ": negative sizes");
  expects(b.num_insertions == 0 || b.num_weights == g.k,
          std::string(what) + ": the batch has " + std::to_string(b.num_weights) +
              " weight(s) per insertion but the graph has " + std::to_string(g.k));
  expects(b.num_insertions == 0 || (b.insert_src && b.insert_dst && (g.k == 0 || b.insert_weights)),
          std::string(what) + ": null insertion arrays");
  expects(b.num_deletions == 0 || (b.delete_src && b.delete_dst),
          std::string(what) + ": null deletion arrays");
  expects(b.num_insertions + b.num_deletions < (1LL << 30),
          std::string(what) + ": a batch holds at most 2^30 operations");
}

std::string& last_error() {
  thread_local std::string message;
  return message;
}

void context_init(Context& c, int device, void* stream) {
  c.device = device;
  DYNGB200_CUDA(cudaDeviceGetAttribute(&c.sm_count, cudaDevAttrMultiProcessorCount, device));
  DYNGB200_CUDA(cudaDeviceGetAttribute(&c.coop_supported, cudaDevAttrCooperativeLaunch, device));
  if (stream) {
    c.stream = static_cast<cudaStream_t>(stream);
  } else {
    DYNGB200_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    c.own_stream = true;
  }
}

}  // namespace dyngb200

namespace {

using namespace dyngb200;

std::atomic<uint64_t> g_next_graph_id{1};

// Copy n elements of an array in `memory` to a host vector.
template <typename T>
std::vector<T> to_host(Context& ctx, const T* p, size_t n, int memory) {
  std::vector<T> out(n);
  if (n == 0) return out;
  expects(p != nullptr, "null array");
  if (memory == DYNGB200_DEVICE) {
    DYNGB200_CUDA(cudaMemcpyAsync(out.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost, ctx.stream));
    DYNGB200_CUDA(cudaStreamSynchronize(ctx.stream));
  } else {
    std::memcpy(out.data(), p, n * sizeof(T));
  }
  return out;
}

// The reference's construction (apply_host.cpp:527-660): counting sort by source keeping input
// order; under multi_edges::forbid a stable sort by destination merges repeats (first position,
// last weights), then append order restores first positions; under allow + sorted a stable sort.
// Weights come as item-major (num_weights per item).
void build_rows(long long n, int k, const std::vector<int32_t>& src, const std::vector<int32_t>& dst,
                const std::vector<long long>& item, const int32_t* weights_item_major,
                const dyngb200_props& props, std::vector<int64_t>& row_ptr,
                std::vector<int32_t>& col, std::vector<int32_t>& w) {
  const size_t count = src.size();
  std::vector<int64_t> start(static_cast<size_t>(n) + 1, 0);
  for (int32_t u : src) start[static_cast<size_t>(u) + 1]++;
  for (long long u = 0; u < n; ++u) start[u + 1] += start[u];
  std::vector<int64_t> order(count);
  {
    std::vector<int64_t> cursor(start.begin(), start.end() - 1);
    for (size_t i = 0; i < count; ++i) order[cursor[src[i]]++] = static_cast<int64_t>(i);
  }
  struct Item {
    int32_t v;
    int64_t first, last;
  };
  std::vector<Item> kept;
  kept.reserve(count);
  row_ptr.assign(static_cast<size_t>(n) + 1, 0);
  std::vector<Item> row;
  for (long long u = 0; u < n; ++u) {
    row.clear();
    for (int64_t j = start[u]; j < start[u + 1]; ++j) row.push_back({dst[order[j]], j, order[j]});
    if (!props.allow_multi) {
      bool sorted_unique = true;
      for (size_t r = 1; r < row.size() && sorted_unique; ++r)
        sorted_unique = row[r - 1].v < row[r].v;
      if (!sorted_unique) {
        std::stable_sort(row.begin(), row.end(),
                         [](const Item& a, const Item& b) { return a.v < b.v; });
        size_t wpos = 0;
        for (size_t r = 0; r < row.size(); ++r) {
          if (wpos > 0 && row[wpos - 1].v == row[r].v) {
            row[wpos - 1].last = row[r].last;
          } else {
            row[wpos++] = row[r];
          }
        }
        row.resize(wpos);
        if (!props.sorted)
          std::sort(row.begin(), row.end(),
                    [](const Item& a, const Item& b) { return a.first < b.first; });
      }
    } else if (props.sorted) {
      std::stable_sort(row.begin(), row.end(), [](const Item& a, const Item& b) { return a.v < b.v; });
    }
    row_ptr[u + 1] = row_ptr[u] + static_cast<int64_t>(row.size());
    kept.insert(kept.end(), row.begin(), row.end());
  }
  const size_t m = kept.size();
  col.resize(m);
  w.resize(m * static_cast<size_t>(k));
  for (size_t e = 0; e < m; ++e) {
    col[e] = kept[e].v;
    const long long it = item[static_cast<size_t>(kept[e].last)];
    for (int j = 0; j < k; ++j)
      w[static_cast<size_t>(j) * m + e] = weights_item_major[it * k + j];
  }
}

void expect_props(const dyngb200_props& p) {
  expects(p.on_existing_insert >= 0 && p.on_existing_insert <= 2, "props.on_existing_insert");
  expects(p.on_missing_delete >= 0 && p.on_missing_delete <= 1, "props.on_missing_delete");
  expects(p.on_self_loop >= 0 && p.on_self_loop <= 2, "props.on_self_loop");
  expects(p.headroom >= 0 && p.headroom <= 16, "props.headroom must lie in [0, 16]");
}

dyngb200_graph_s* new_graph(Context& ctx, long long n, std::vector<int32_t>& src, std::vector<int32_t>& dst,
                 std::vector<long long>& item, const int32_t* weights_item_major, int k,
                 const dyngb200_props& props) {
  std::vector<int64_t> rp;
  std::vector<int32_t> col, w;
  build_rows(n, k, src, dst, item, weights_item_major, props, rp, col, w);
  auto* h = new dyngb200_graph_s();
  Graph& g = h->g;
  g.id = g_next_graph_id.fetch_add(1);
  g.props = props;
  g.k = k;
  g.device = ctx.device;
  try {
    graph_build(ctx, g, n, rp.data(), col.data(), w.data(), static_cast<long long>(col.size()));
  } catch (...) {
    delete h;
    throw;
  }
  return h;
}

// The O(n) checks of validate_inputs (sssp.cpp:398-460), in vertex order.
void validate_tree(int32_t source, const std::vector<int64_t>& d, const std::vector<int32_t>& p,
                   long long bound) {
  const long long n = static_cast<long long>(d.size());
  expects(d[source] == 0, "sssp: the source " + std::to_string(source) + " must have distance 0");
  expects(p[source] == -1, "sssp: the source " + std::to_string(source) + " must have parent -1");
  for (long long v = 0; v < n; ++v) {
    const int64_t dv = d[v];
    const int32_t pv = p[v];
    if (dv >= kInfinity / 2) {
      expects(pv == -1, "sssp: unreachable vertex " + std::to_string(v) + " has a parent");
      continue;
    }
    expects(dv >= 0 && dv <= bound, "sssp: the distance of vertex " + std::to_string(v) +
                                        " is outside [0, (n - 1) * max weight]");
    if (v == source) continue;
    expects(pv >= 0, "sssp: reachable vertex " + std::to_string(v) + " has no parent");
    expects(d[pv] < kInfinity / 2,
            "sssp: vertex " + std::to_string(v) + " has an unreachable parent");
  }
  std::vector<char> state(static_cast<size_t>(n), 0);
  state[source] = 2;
  std::vector<int32_t> path;
  for (long long v = 0; v < n; ++v) {
    if (state[v] != 0 || d[v] >= kInfinity / 2) continue;
    path.clear();
    int32_t u = static_cast<int32_t>(v);
    while (state[u] == 0) {
      state[u] = 1;
      path.push_back(u);
      u = p[u];
    }
    expects(state[u] == 2, "sssp: the input shortest-path tree has a parent cycle through vertex " +
                               std::to_string(u));
    for (int32_t x : path) state[x] = 2;
  }
}

}  // namespace

extern "C" {

const char* dyngb200_last_error_message(void) { return last_error().c_str(); }

const char* dyngb200_status_name(dyngb200_status s) {
  switch (s) {
    case DYNGB200_OK: return "ok";
    case DYNGB200_INVALID_ARGUMENT: return "invalid_argument";
    case DYNGB200_NOT_SUPPORTED: return "not_supported";
    case DYNGB200_STALE_RESULT: return "stale_result";
    case DYNGB200_OUT_OF_MEMORY: return "out_of_memory";
    case DYNGB200_CUDA_ERROR: return "cuda_error";
    case DYNGB200_CAPACITY: return "capacity";
    case DYNGB200_INTERNAL: return "internal";
  }
  return "unknown";
}

int dyngb200_abi_version(void) { return DYNGB200_ABI_VERSION; }

void dyngb200_props_default(dyngb200_props* p) {
  if (!p) return;
  *p = dyngb200_props{1, 1, 0, 0, 0, 0, 1, 1, 0.125};
}

void dyngb200_props_mosp_compatible(dyngb200_props* p) {
  if (!p) return;
  *p = dyngb200_props{1, 0, 1, 0, 0, 0, 1, 1, 0.125};
}

dyngb200_status dyngb200_context_create(int device, void* stream, dyngb200_context* out) {
  return guarded([&] {
    expects(out != nullptr, "context_create: null output");
    int count = 0;
    DYNGB200_CUDA(cudaGetDeviceCount(&count));
    expects(device >= 0 && device < count, "context_create: no CUDA device " + std::to_string(device),
            DYNGB200_NOT_SUPPORTED);
    DeviceGuard guard(device);
    auto h = std::make_unique<dyngb200_context_s>();
    context_init(h->ctx, device, stream);
    *out = h.release();
  });
}

dyngb200_status dyngb200_context_destroy(dyngb200_context ctx) {
  return guarded([&] {
    if (!ctx) return;
    DeviceGuard guard(ctx->ctx.device);
    cudaStreamSynchronize(ctx->ctx.stream);
    for (cudaEvent_t e : ctx->ctx.update_events)
      if (e) cudaEventDestroy(e);
    if (ctx->ctx.own_stream) cudaStreamDestroy(ctx->ctx.stream);
    delete ctx;
  });
}

dyngb200_status dyngb200_context_synchronize(dyngb200_context ctx) {
  return guarded([&] {
    expects(ctx != nullptr, "null context");
    DYNGB200_CUDA(cudaStreamSynchronize(ctx->ctx.stream));
  });
}

dyngb200_status dyngb200_context_set_test_hooks(dyngb200_context ctx,
                                                const dyngb200_test_hooks* hooks) {
  return guarded([&] {
    expects(ctx != nullptr, "context_set_test_hooks: null context");
    const dyngb200_test_hooks h = hooks ? *hooks : dyngb200_test_hooks{0, 0, 0, 0};
    expects(h.barrier_timeout_ns >= 0 && h.barrier_extra_arrivals >= 0,
            "context_set_test_hooks: negative limit or arrivals");
    expects(h.barrier_kernel >= 0 && h.barrier_kernel <= 2,
            "context_set_test_hooks: barrier_kernel is 0, 1 or 2");
    ctx->ctx.test_barrier_kernel = h.barrier_kernel;
    ctx->ctx.test_barrier_timeout_ns = h.barrier_timeout_ns;
    ctx->ctx.test_barrier_extra = h.barrier_extra_arrivals;
    ctx->ctx.test_no_cooperative = h.no_cooperative_launch != 0 ? 1 : 0;
  });
}

dyngb200_status dyngb200_debug_device_allocations(int64_t* count) {
  return guarded([&] {
    expects(count != nullptr, "debug_device_allocations: null argument");
    *count = device_alloc_count();
  });
}

dyngb200_status dyngb200_debug_fail_device_allocation(int64_t nth) {
  return guarded([&] {
    expects(nth >= 0, "debug_fail_device_allocation: negative count");
    device_alloc_fail_at(nth);
  });
}

dyngb200_status dyngb200_graph_from_edges(dyngb200_context ctx, int64_t n, const int32_t* src,
                                          const int32_t* dst, const int32_t* weights,
                                          int64_t num_edges, int32_t num_weights, int32_t memory,
                                          const dyngb200_props* props, dyngb200_graph* out) {
  return guarded([&] {
    expects(ctx && out, "graph_from_edges: null argument");
    expects(n >= 0 && n < INT32_MAX, "graph_from_edges: num_vertices out of range");
    expects(num_edges >= 0 && num_weights >= 1, "graph_from_edges: sizes");
    dyngb200_props pr;
    dyngb200_props_default(&pr);
    if (props) pr = *props;
    expect_props(pr);
    Context& c = ctx->ctx;
    DeviceGuard guard(c.device);
    auto s = to_host(c, src, static_cast<size_t>(num_edges), memory);
    auto d = to_host(c, dst, static_cast<size_t>(num_edges), memory);
    auto w = to_host(c, weights, static_cast<size_t>(num_edges) * num_weights, memory);
    std::vector<int32_t> fs, fd;
    std::vector<long long> item;
    fs.reserve(s.size());
    fd.reserve(s.size());
    item.reserve(s.size());
    for (int64_t i = 0; i < num_edges; ++i) {
      const int32_t u = s[i], v = d[i];
      expects(u >= 0 && u < n && v >= 0 && v < n,
              "graph_from_edges: edge " + std::to_string(i) + " is out of range");
      if (u == v && pr.on_self_loop != 0) {
        expects(pr.on_self_loop != 2, "graph_from_edges: self-loop under self_loop::error");
        continue;
      }
      fs.push_back(u);
      fd.push_back(v);
      item.push_back(i);
      if (!pr.directed && u != v) {
        fs.push_back(v);
        fd.push_back(u);
        item.push_back(i);
      }
    }
    *out = new_graph(c, n, fs, fd, item, w.data(), num_weights, pr);
  });
}

dyngb200_status dyngb200_graph_from_csr(dyngb200_context ctx, int64_t n, const int64_t* row_ptr,
                                        const int32_t* col, const int32_t* weights,
                                        int32_t num_weights, int32_t memory,
                                        const dyngb200_props* props, dyngb200_graph* out) {
  return guarded([&] {
    expects(ctx && out && row_ptr, "graph_from_csr: null argument");
    expects(n >= 0 && n < INT32_MAX && num_weights >= 1, "graph_from_csr: sizes");
    dyngb200_props pr;
    dyngb200_props_default(&pr);
    if (props) pr = *props;
    expect_props(pr);
    Context& c = ctx->ctx;
    DeviceGuard guard(c.device);
    auto rp = to_host(c, row_ptr, static_cast<size_t>(n) + 1, memory);
    expects(rp[0] == 0, "graph_from_csr: row_ptr[0] must be 0");
    for (int64_t u = 0; u < n; ++u) expects(rp[u + 1] >= rp[u], "graph_from_csr: row_ptr not monotone");
    const int64_t m = rp[n];
    auto cl = to_host(c, col, static_cast<size_t>(m), memory);
    auto w = to_host(c, weights, static_cast<size_t>(m) * num_weights, memory);
    std::vector<int32_t> fs, fd;
    std::vector<long long> item;
    std::vector<int32_t> witems(static_cast<size_t>(m) * num_weights);
    for (int64_t e = 0; e < m; ++e)
      for (int j = 0; j < num_weights; ++j)
        witems[static_cast<size_t>(e) * num_weights + j] = w[static_cast<size_t>(j) * m + e];
    fs.reserve(static_cast<size_t>(m));
    fd.reserve(static_cast<size_t>(m));
    item.reserve(static_cast<size_t>(m));
    for (int64_t u = 0; u < n; ++u) {
      for (int64_t e = rp[u]; e < rp[u + 1]; ++e) {
        const int32_t v = cl[e];
        expects(v >= 0 && v < n, "graph_from_csr: neighbour out of range");
        if (static_cast<int32_t>(u) == v && pr.on_self_loop != 0) {
          expects(pr.on_self_loop != 2, "graph_from_csr: self-loop under self_loop::error");
          continue;
        }
        fs.push_back(static_cast<int32_t>(u));
        fd.push_back(v);
        item.push_back(e);
      }
    }
    *out = new_graph(c, n, fs, fd, item, witems.data(), num_weights, pr);
  });
}

dyngb200_status dyngb200_graph_destroy(dyngb200_graph g) {
  return guarded([&] {
    if (!g) return;
    DeviceGuard guard(g->g.device);
    delete g;
  });
}

dyngb200_status dyngb200_graph_info(dyngb200_graph g, int64_t* n, int64_t* m, int32_t* k,
                                    uint64_t* version) {
  return guarded([&] {
    expects(g != nullptr, "graph_info: null graph");
    if (n) *n = g->g.n;
    if (m) *m = g->g.m;
    if (k) *k = g->g.k;
    if (version) *version = g->g.version;
  });
}

dyngb200_status dyngb200_graph_device_bytes(dyngb200_graph g, int64_t* bytes) {
  return guarded([&] {
    expects(g && bytes, "graph_device_bytes: null argument");
    const Graph& x = g->g;
    const long long k = x.k;
    *bytes = 2 * (x.n_cap * (8 + 4 + 4) + x.arena_cap * (4 + 4 * k)) + 16 * x.ecap;
  });
}

dyngb200_status dyngb200_graph_storage_get(dyngb200_graph g, dyngb200_graph_storage* out) {
  return guarded([&] {
    expects(g && out, "graph_storage_get: null argument");
    const Graph& x = g->g;
    out->vertex_capacity = x.n_cap;
    out->arena_slots = x.arena_cap;
    out->out_top = static_cast<int64_t>(x.host_counters.out_top);
    out->in_top = static_cast<int64_t>(x.host_counters.in_top);
    out->out_garbage = static_cast<int64_t>(x.host_counters.out_garbage);
    out->in_garbage = static_cast<int64_t>(x.host_counters.in_garbage);
    out->index_slots = x.props.allow_multi ? 0 : x.ecap;
    out->arena_growths = x.arena_growths;
    out->compactions = x.compactions;
    out->index_builds = x.index_builds;
    out->grow_ms = x.grow_ms;
    out->compact_ms = x.compact_ms;
    out->index_ms = x.index_ms;
    out->maintenance_ms_max = x.maintenance_ms_max;
  });
}

dyngb200_status dyngb200_graph_apply(dyngb200_context ctx, dyngb200_graph g,
                                     const dyngb200_batch* batch, dyngb200_apply_summary* summary) {
  return guarded([&] {
    expects(ctx && g && batch, "graph_apply: null argument");
    DeviceGuard guard(ctx->ctx.device);
    expect_batch(g->g, *batch, "graph::apply");
    graph_apply(ctx->ctx, g->g, *batch, summary, nullptr);
  });
}

dyngb200_status dyngb200_graph_apply_classified(dyngb200_context ctx, dyngb200_graph g,
                                                const dyngb200_batch* batch,
                                                dyngb200_apply_summary* summary,
                                                uint8_t* weight_increased) {
  return guarded([&] {
    expects(ctx && g && batch, "graph_apply: null argument");
    DeviceGuard guard(ctx->ctx.device);
    expect_batch(g->g, *batch, "graph::apply");
    graph_apply(ctx->ctx, g->g, *batch, summary, weight_increased);
  });
}

dyngb200_status dyngb200_graph_to_csr(dyngb200_context ctx, dyngb200_graph g, int64_t* row_ptr,
                                      int32_t* col, int32_t* weights, int64_t* in_row_ptr,
                                      int32_t* in_col, int32_t* in_weights) {
  return guarded([&] {
    expects(ctx && g, "graph_to_csr: null argument");
    DeviceGuard guard(ctx->ctx.device);
    graph_export(ctx->ctx, g->g, row_ptr, col, weights, in_row_ptr, in_col, in_weights);
  });
}

dyngb200_status dyngb200_sssp_compute(dyngb200_context ctx, dyngb200_graph g, int32_t source,
                                      const dyngb200_options* opt, dyngb200_tree* out,
                                      dyngb200_stats* stats) {
  return guarded([&] {
    expects(ctx && g && out, "sssp::compute: null argument");
    Context& c = ctx->ctx;
    Graph& gr = g->g;
    DeviceGuard guard(c.device);
    dyngb200_options o{0, 0, DYNGB200_ENGINE_AUTOMATIC, 1};
    if (opt) o = *opt;
    expects(o.delta >= 0, "sssp: options.delta must be >= 0 (0 = automatic)");
    expects(o.objective >= 0 && o.objective < gr.k, "sssp::compute: options.objective " +
                                                        std::to_string(o.objective) +
                                                        " is out of range");
    expects(gr.device == c.device, "sssp::compute: the graph belongs to another device");
    expects(source >= 0 && source < gr.n, "sssp::compute: source " + std::to_string(source) +
                                              " is out of range [0, " + std::to_string(gr.n) + ")");
    auto h = std::make_unique<dyngb200_tree_s>();
    Tree& t = h->t;
    t.graph_id = gr.id;
    t.version = gr.version;
    t.source = source;
    t.opt = o;
    t.device = c.device;
    t.n = gr.n;
    sssp_compute(c, gr, t, stats);
    *out = h.release();
  });
}

dyngb200_status dyngb200_sssp_compute_static_scratch(dyngb200_graph g, int32_t source,
                                                     int32_t objective, int64_t delta,
                                                     int64_t* distances, int32_t* parents,
                                                     void* stream) {
  return guarded([&] {
    expects(g != nullptr, "sssp::compute (static scratch): null graph");
    sssp_compute_static(g->g, source, objective, delta, distances, parents,
                        static_cast<cudaStream_t>(stream));
  });
}

dyngb200_status dyngb200_sssp_update(dyngb200_context ctx, dyngb200_graph g,
                                     const dyngb200_batch* batch, dyngb200_tree tree,
                                     dyngb200_stats* stats) {
  return guarded([&] {
    expects(ctx && g && batch && tree, "sssp::update: null argument");
    Context& c = ctx->ctx;
    DeviceGuard guard(c.device);
    expect_tree_current(g->g, tree->t, "sssp::update");
    expect_batch(g->g, *batch, "sssp::update");
    const dyngb200_schedule sched = c.schedule_set ? c.schedule : dyngb200_schedule{};
    sssp_update(c, g->g, tree->t, *batch, sched, stats);
  });
}

dyngb200_status dyngb200_sssp_update_scheduled(dyngb200_context ctx, dyngb200_graph g,
                                               const dyngb200_batch* batch, dyngb200_tree tree,
                                               const dyngb200_schedule* schedule,
                                               dyngb200_stats* stats) {
  return guarded([&] {
    expects(ctx && g && batch && tree, "sssp::update: null argument");
    Context& c = ctx->ctx;
    DeviceGuard guard(c.device);
    expect_tree_current(g->g, tree->t, "sssp::update");
    expect_batch(g->g, *batch, "sssp::update");
    dyngb200_schedule sched{};
    if (schedule) sched = *schedule;
    expects(sched.delta >= 0 && sched.grid_blocks >= 0 && sched.heavy_degree >= 0,
            "sssp::update: negative schedule field");
    sssp_update(c, g->g, tree->t, *batch, sched, stats);
  });
}

dyngb200_status dyngb200_sssp_update_each(dyngb200_context ctx, dyngb200_graph g,
                                          const dyngb200_batch* batch, dyngb200_tree* trees,
                                          int32_t count, dyngb200_stats* stats) {
  return guarded([&] {
    expects(ctx && g && batch && trees, "dyng::update_each: null argument");
    expects(count >= 1, "dyng::update_each: the list of results is empty (applying a batch "
                        "without updating any result would leave every result stale; use "
                        "graph_apply)");
    Context& c = ctx->ctx;
    DeviceGuard guard(c.device);
    std::vector<Tree*> ts(static_cast<size_t>(count));
    for (int i = 0; i < count; ++i) {
      expects(trees[i] != nullptr, "dyng::update_each: result " + std::to_string(i) + " is null");
      for (int j = 0; j < i; ++j)
        expects(trees[j] != trees[i], "dyng::update_each: result " + std::to_string(i) +
                                          " is listed twice");
      expect_tree_current(g->g, trees[i]->t, "dyng::update_each");
      ts[i] = &trees[i]->t;
    }
    expect_batch(g->g, *batch, "dyng::update_each");
    sssp_update_each(c, g->g, *batch, ts.data(), count, stats);
  });
}

dyngb200_status dyngb200_sssp_update_learned(dyngb200_context ctx, dyngb200_graph g,
                                             const dyngb200_batch* batch, dyngb200_tree tree,
                                             dyngb200_scheduler scheduler, dyngb200_stats* stats) {
  return guarded([&] {
    expects(ctx && g && batch && tree && scheduler, "sssp::update: null argument");
    Context& c = ctx->ctx;
    DeviceGuard guard(c.device);
    expects(scheduler->s.device == c.device, "sssp::update: the scheduler belongs to another device");
    expect_tree_current(g->g, tree->t, "sssp::update");
    expect_batch(g->g, *batch, "sssp::update");
    sssp_update(c, g->g, tree->t, *batch, dyngb200_schedule{}, stats, &scheduler->s);
  });
}

int64_t dyngb200_scheduler_num_params(void) { return kMlpParams; }

dyngb200_status dyngb200_scheduler_create(dyngb200_context ctx, uint64_t seed,
                                          dyngb200_scheduler* out) {
  return guarded([&] {
    expects(ctx && out, "scheduler_create: null argument");
    DeviceGuard guard(ctx->ctx.device);
    auto h = std::make_unique<dyngb200_scheduler_s>();
    scheduler_init(ctx->ctx, h->s, seed);
    *out = h.release();
  });
}

dyngb200_status dyngb200_scheduler_destroy(dyngb200_scheduler s) {
  return guarded([&] {
    if (!s) return;
    DeviceGuard guard(s->s.device);
    delete s;
  });
}

dyngb200_status dyngb200_scheduler_set_params(dyngb200_context ctx, dyngb200_scheduler s,
                                              const float* params, const float* feature_mean,
                                              const float* feature_scale) {
  return guarded([&] {
    expects(ctx && s, "scheduler_set_params: null argument");
    DeviceGuard guard(ctx->ctx.device);
    expects(s->s.device == ctx->ctx.device, "scheduler: the scheduler belongs to another device");
    scheduler_set(ctx->ctx, s->s, params, feature_mean, feature_scale);
  });
}

dyngb200_status dyngb200_scheduler_get_params(dyngb200_context ctx, dyngb200_scheduler s,
                                              float* params, float* feature_mean,
                                              float* feature_scale) {
  return guarded([&] {
    expects(ctx && s, "scheduler_get_params: null argument");
    DeviceGuard guard(ctx->ctx.device);
    scheduler_get(ctx->ctx, s->s, params, feature_mean, feature_scale);
  });
}

dyngb200_status dyngb200_scheduler_set_feature_range(dyngb200_scheduler s, const float* lo,
                                                     const float* hi) {
  return guarded([&] {
    expects(s != nullptr, "scheduler_set_feature_range: null scheduler");
    expects((lo == nullptr) == (hi == nullptr),
            "scheduler_set_feature_range: give both bounds or neither");
    Scheduler& x = s->s;
    x.has_range = lo != nullptr;
    for (int i = 0; i < kMlpIn; ++i) {
      if (lo) expects(lo[i] <= hi[i], "scheduler_set_feature_range: lower bound above upper");
      x.feat_lo[i] = lo ? lo[i] : 0.0f;
      x.feat_hi[i] = hi ? hi[i] : 0.0f;
    }
  });
}

dyngb200_status dyngb200_scheduler_get_feature_range(dyngb200_scheduler s, float* lo, float* hi,
                                                     int32_t* has_range) {
  return guarded([&] {
    expects(s != nullptr, "scheduler_get_feature_range: null scheduler");
    const Scheduler& x = s->s;
    if (has_range) *has_range = x.has_range ? 1 : 0;
    for (int i = 0; i < kMlpIn; ++i) {
      if (lo) lo[i] = x.feat_lo[i];
      if (hi) hi[i] = x.feat_hi[i];
    }
  });
}

dyngb200_status dyngb200_scheduler_forward(dyngb200_context ctx, dyngb200_scheduler s,
                                           const float* features, int64_t n, float* logits) {
  return guarded([&] {
    expects(ctx && s && (n == 0 || (features && logits)), "scheduler_forward: null argument");
    DeviceGuard guard(ctx->ctx.device);
    scheduler_forward(ctx->ctx, s->s, features, n, logits);
  });
}

dyngb200_status dyngb200_scheduler_gradients(dyngb200_context ctx, dyngb200_scheduler s,
                                             const float* features, const int32_t* labels,
                                             int64_t n, float* grads, double* loss) {
  return guarded([&] {
    expects(ctx && s && features && labels, "scheduler_gradients: null argument");
    DeviceGuard guard(ctx->ctx.device);
    scheduler_gradients(ctx->ctx, s->s, features, labels, n, grads, loss);
  });
}

dyngb200_status dyngb200_scheduler_train(dyngb200_context ctx, dyngb200_scheduler s,
                                         const float* features, const int32_t* labels, int64_t n,
                                         int32_t epochs, int32_t batch_size, float learning_rate,
                                         uint64_t seed, double* final_loss) {
  return guarded([&] {
    expects(ctx && s && features && labels, "scheduler_train: null argument");
    DeviceGuard guard(ctx->ctx.device);
    scheduler_train(ctx->ctx, s->s, features, labels, n, epochs, batch_size, learning_rate, seed,
                    final_loss);
  });
}

dyngb200_status dyngb200_graph_clone(dyngb200_context ctx, dyngb200_graph g, dyngb200_graph* out) {
  return guarded([&] {
    expects(ctx && g && out, "graph_clone: null argument");
    DeviceGuard guard(ctx->ctx.device);
    expects(g->g.device == ctx->ctx.device, "graph_clone: the graph belongs to another device");
    auto h = std::make_unique<dyngb200_graph_s>();
    h->g.id = g_next_graph_id.fetch_add(1);
    graph_copy(ctx->ctx, h->g, g->g);
    *out = h.release();
  });
}

dyngb200_status dyngb200_graph_copy_from(dyngb200_context ctx, dyngb200_graph dst,
                                         dyngb200_graph src) {
  return guarded([&] {
    expects(ctx && dst && src, "graph_copy_from: null argument");
    DeviceGuard guard(ctx->ctx.device);
    expects(dst->g.device == ctx->ctx.device && src->g.device == ctx->ctx.device,
            "graph_copy_from: both graphs must live on the context's device");
    if (dst != src) graph_copy(ctx->ctx, dst->g, src->g);
  });
}

dyngb200_status dyngb200_tree_copy_from(dyngb200_context ctx, dyngb200_tree dst,
                                        dyngb200_tree src) {
  return guarded([&] {
    expects(ctx && dst && src, "tree_copy_from: null argument");
    DeviceGuard guard(ctx->ctx.device);
    expects(dst->t.device == ctx->ctx.device && src->t.device == ctx->ctx.device,
            "tree_copy_from: both trees must live on the context's device");
    expects(!src->t.poisoned, "tree_copy_from: the source was left unusable by a failed update",
            DYNGB200_STALE_RESULT);
    if (dst != src) tree_copy(ctx->ctx, dst->t, src->t);
  });
}

dyngb200_status dyngb200_tree_from_arrays(dyngb200_context ctx, dyngb200_graph g, int32_t source,
                                          const int64_t* distances, const int32_t* parents,
                                          int64_t n, int32_t memory, int32_t canonicalize,
                                          const dyngb200_options* opt, dyngb200_tree* out) {
  return guarded([&] {
    expects(ctx && g && out, "from_arrays: null argument");
    Context& c = ctx->ctx;
    Graph& gr = g->g;
    DeviceGuard guard(c.device);
    dyngb200_options o{0, 0, DYNGB200_ENGINE_AUTOMATIC, 1};
    if (opt) o = *opt;
    expects(o.delta >= 0, "sssp: options.delta must be >= 0");
    expects(o.objective >= 0 && o.objective < gr.k, "from_arrays: objective out of range");
    expects(source >= 0 && source < gr.n, "sssp::result::from_arrays: source out of range");
    expects(n == gr.n, "sssp::result::from_arrays: " + std::to_string(n) + " entries for " +
                           std::to_string(gr.n) + " vertices");
    if (gr.host_columns[o.objective].dirty) graph_rescan_columns(c, gr);
    const ColumnStats cs = gr.host_columns[o.objective];
    expects(cs.bad == 0, "sssp::result::from_arrays: an edge has a weight below 1");
    auto d = to_host(c, distances, static_cast<size_t>(n), memory);
    auto p = to_host(c, parents, static_cast<size_t>(n), memory);
    for (int64_t v = 0; v < n; ++v) {
      if (d[v] >= kInfinity / 2) d[v] = kInfinity;
      expects(p[v] >= -1 && p[v] < n, "sssp::result::from_arrays: vertex " + std::to_string(v) +
                                          " has parent " + std::to_string(p[v]) +
                                          ", outside [-1, " + std::to_string(n) + ")");
    }
    auto h = std::make_unique<dyngb200_tree_s>();
    Tree& t = h->t;
    t.graph_id = gr.id;
    t.version = gr.version;
    t.source = source;
    t.opt = o;
    t.device = c.device;
    t.n = n;
    tree_reserve(c, t, gr.n_cap);
    DYNGB200_CUDA(cudaMemcpyAsync(t.dist.ptr, d.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice,
                                  c.stream));
    DYNGB200_CUDA(cudaMemcpyAsync(t.parent.ptr, p.data(), n * sizeof(int32_t),
                                  cudaMemcpyHostToDevice, c.stream));
    if (canonicalize) {
      tree_canonicalize(c, gr, t);
      DYNGB200_CUDA(cudaMemcpyAsync(p.data(), t.parent.ptr, n * sizeof(int32_t),
                                    cudaMemcpyDeviceToHost, c.stream));
      DYNGB200_CUDA(cudaStreamSynchronize(c.stream));
    }
    if (o.validate_inputs) {
      expects(distances_fit(n, cs.max_w), "sssp::result::from_arrays: distances do not fit in 62 bits");
      validate_tree(source, d, p, cs.max_w * std::max<long long>(n - 1, 1));
    }
    t.trusted = o.validate_inputs != 0;
    t.canonical = canonicalize != 0;
    // the persistent packed words in the format of the graph's current bound
    u64 bound = 0;
    const Packing pk = choose_packing(n, cs.max_w, &bound);
    tree_repack(c, t, pk.bits);
    DYNGB200_CUDA(cudaStreamSynchronize(c.stream));
    *out = h.release();
  });
}

dyngb200_status dyngb200_tree_clone(dyngb200_context ctx, dyngb200_tree tree, dyngb200_tree* out) {
  return guarded([&] {
    expects(ctx && tree && out, "clone: null argument");
    Context& c = ctx->ctx;
    DeviceGuard guard(c.device);
    const Tree& s = tree->t;
    expects(!s.poisoned, "sssp::result::clone: the result was left unusable by a failed update",
            DYNGB200_STALE_RESULT);
    auto h = std::make_unique<dyngb200_tree_s>();
    Tree& t = h->t;
    t.graph_id = s.graph_id;
    t.version = s.version;
    t.source = s.source;
    t.opt = s.opt;
    t.n = s.n;
    t.device = c.device;
    t.packed_bits = s.packed_bits;
    t.trusted = s.trusted;
    t.canonical = s.canonical;
    tree_reserve(c, t, std::max(s.cap, s.n));
    if (s.n > 0) {
      DYNGB200_CUDA(cudaMemcpyPeerAsync(t.dist.ptr, c.device, s.dist.ptr, s.device,
                                        s.n * sizeof(int64_t), c.stream));
      DYNGB200_CUDA(cudaMemcpyPeerAsync(t.parent.ptr, c.device, s.parent.ptr, s.device,
                                        s.n * sizeof(int32_t), c.stream));
      DYNGB200_CUDA(cudaMemcpyPeerAsync(t.packed.ptr, c.device, s.packed.ptr, s.device,
                                        s.n * sizeof(u64), c.stream));
    }
    if (s.hist.ptr)
      DYNGB200_CUDA(cudaMemcpyPeerAsync(t.hist.ptr, c.device, s.hist.ptr, s.device,
                                        sizeof(TreeHistory), c.stream));
    DYNGB200_CUDA(cudaStreamSynchronize(c.stream));
    *out = h.release();
  });
}

dyngb200_status dyngb200_tree_destroy(dyngb200_tree t) {
  return guarded([&] {
    if (!t) return;
    DeviceGuard guard(t->t.device);
    delete t;
  });
}

dyngb200_status dyngb200_tree_distances(dyngb200_context ctx, dyngb200_tree t, int64_t* dst,
                                        int32_t memory) {
  return guarded([&] {
    expects(ctx && t && dst, "distances: null argument");
    expects(!t->t.poisoned, "sssp::result: the result was left unusable by a failed update",
            DYNGB200_STALE_RESULT);
    DeviceGuard guard(ctx->ctx.device);
    DYNGB200_CUDA(cudaMemcpyAsync(dst, t->t.dist.ptr, t->t.n * sizeof(int64_t),
                                  memory == DYNGB200_DEVICE ? cudaMemcpyDeviceToDevice
                                                            : cudaMemcpyDeviceToHost,
                                  ctx->ctx.stream));
    DYNGB200_CUDA(cudaStreamSynchronize(ctx->ctx.stream));
  });
}

dyngb200_status dyngb200_tree_parents(dyngb200_context ctx, dyngb200_tree t, int32_t* dst,
                                      int32_t memory) {
  return guarded([&] {
    expects(ctx && t && dst, "parents: null argument");
    expects(!t->t.poisoned, "sssp::result: the result was left unusable by a failed update",
            DYNGB200_STALE_RESULT);
    DeviceGuard guard(ctx->ctx.device);
    DYNGB200_CUDA(cudaMemcpyAsync(dst, t->t.parent.ptr, t->t.n * sizeof(int32_t),
                                  memory == DYNGB200_DEVICE ? cudaMemcpyDeviceToDevice
                                                            : cudaMemcpyDeviceToHost,
                                  ctx->ctx.stream));
    DYNGB200_CUDA(cudaStreamSynchronize(ctx->ctx.stream));
  });
}

dyngb200_status dyngb200_tree_device_arrays(dyngb200_tree t, const int64_t** d,
                                            const int32_t** p) {
  return guarded([&] {
    expects(t != nullptr, "device_arrays: null tree");
    expects(!t->t.poisoned, "sssp::result: the result was left unusable by a failed update",
            DYNGB200_STALE_RESULT);
    if (d) *d = t->t.dist.ptr;
    if (p) *p = t->t.parent.ptr;
  });
}

dyngb200_status dyngb200_tree_info(dyngb200_tree t, int32_t* source, int64_t* n,
                                   uint64_t* version, int32_t* poisoned, dyngb200_options* opt) {
  return guarded([&] {
    expects(t != nullptr, "tree_info: null tree");
    if (source) *source = t->t.source;
    if (n) *n = t->t.n;
    if (version) *version = t->t.version;
    if (poisoned) *poisoned = t->t.poisoned ? 1 : 0;
    if (opt) *opt = t->t.opt;
  });
}

dyngb200_status dyngb200_tree_set_options(dyngb200_tree t, const dyngb200_options* opt) {
  return guarded([&] {
    expects(t && opt, "set_options: null argument");
    expects(!t->t.poisoned, "set_options: poisoned result", DYNGB200_STALE_RESULT);
    expects(opt->objective == t->t.opt.objective, "set_options: the objective must stay the same");
    expects(opt->delta >= 0, "set_options: options.delta must be >= 0");
    t->t.opt = *opt;
  });
}

}  // extern "C"
