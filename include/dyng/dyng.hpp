// dyng/dyng.hpp -- a C++17 face over include/dyngb200.h for callers written against dynG's C++
// API (cpp/include/dyng/dyng.hpp and the headers it gathers).  Header-only; link with
// dyng_b200/libdyngb200.so.  It covers the batch-dynamic SSSP path on resources::cuda():
//
//   auto res = dyng::resources::cuda();
//   dyng::edge_list<std::int32_t, std::int32_t> edges{4, {0, 0, 2, 1}, {1, 2, 1, 3}, {4, 1, 2, 1}, 1};
//   auto g = dyng::graph<>::from_edges(res, edges.view());
//   auto tree = dyng::sssp::compute(res, g, 0);
//   dyng::edge_batch<std::int32_t, std::int32_t> batch;
//   batch.delete_edge(2, 1);
//   batch.insert_edge(2, 3, {1});
//   auto st = dyng::sssp::update(res, g, batch.view(), tree);
//   for (auto d : dyng::to_vector(res, tree.distances())) std::cout << d << ' ';
//
// Statuses become the reference's exception classes (cpp/include/dyng/core/error.hpp).  Only
// the CUDA backend exists here: resources::sequential() and resources::openmp() throw
// not_supported_error.  Ids and weights are int32, edge offsets int64, distances int64 (the
// graph<int32, int64, int32> and result<int32> instantiations of sssp.hpp:323-371).
#ifndef DYNG_B200_DYNG_HPP
#define DYNG_B200_DYNG_HPP

#include <cstdint>
#include <functional>
#include <initializer_list>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../dyngb200.h"

namespace dyng {

// ---- errors (core/error.hpp) ------------------------------------------------------------------
struct error : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct invalid_argument_error : error {
  using error::error;
};
struct not_supported_error : error {
  using error::error;
};
struct stale_result_error : error {
  using error::error;
};
struct out_of_memory_error : error {
  using error::error;
};
struct cuda_error : error {
  using error::error;
};
struct capacity_error : error {
  using error::error;
};
struct internal_error : error {
  using error::error;
};

namespace detail {
inline void check(dyngb200_status s) {
  if (s == DYNGB200_OK) return;
  const std::string msg = dyngb200_last_error_message();
  switch (s) {
    case DYNGB200_INVALID_ARGUMENT: throw invalid_argument_error(msg);
    case DYNGB200_NOT_SUPPORTED: throw not_supported_error(msg);
    case DYNGB200_STALE_RESULT: throw stale_result_error(msg);
    case DYNGB200_OUT_OF_MEMORY: throw out_of_memory_error(msg);
    case DYNGB200_CUDA_ERROR: throw cuda_error(msg);
    case DYNGB200_CAPACITY: throw capacity_error(msg);
    default: throw internal_error(msg);
  }
}
template <typename T>
constexpr bool is_i32 = std::is_same_v<T, std::int32_t>;
}  // namespace detail

enum class memory_space { host = DYNGB200_HOST, device = DYNGB200_DEVICE };
enum class engine { automatic = DYNGB200_ENGINE_AUTOMATIC, fused = DYNGB200_ENGINE_FUSED,
                    operators = DYNGB200_ENGINE_OPERATORS };

// ---- resources (core/resources.hpp) ------------------------------------------------------------
class resources {
 public:
  static resources cuda(int device = 0, void* stream = nullptr) {
    dyngb200_context c = nullptr;
    detail::check(dyngb200_context_create(device, stream, &c));
    return resources(std::shared_ptr<dyngb200_context_s>(c, [](dyngb200_context p) {
      dyngb200_context_destroy(p);
    }));
  }
  static resources sequential() {
    throw not_supported_error("dyng_b200: only the cuda backend is built (resources::cuda())");
  }
  static resources openmp(int = 0) {
    throw not_supported_error("dyng_b200: only the cuda backend is built (resources::cuda())");
  }
  void synchronize() const { detail::check(dyngb200_context_synchronize(ctx_.get())); }
  dyngb200_context handle() const { return ctx_.get(); }

 private:
  explicit resources(std::shared_ptr<dyngb200_context_s> c) : ctx_(std::move(c)) {}
  std::shared_ptr<dyngb200_context_s> ctx_;
};

// A view of a typed array in host or device memory (array_view of core/array.hpp).  A device
// view of this library carries the copy that reads it (the owner's accessor).
template <typename T>
struct array_view {
  const T* data = nullptr;
  std::int64_t size = 0;
  memory_space space = memory_space::host;
  std::function<void(const resources&, T*)> read_to_host;
};

// Copy of a view into a host vector (dyng::to_vector).
template <typename T>
std::vector<T> to_vector(const resources& res, const array_view<T>& v) {
  std::vector<T> out(static_cast<size_t>(v.size));
  if (v.size == 0) return out;
  if (v.space == memory_space::host) {
    out.assign(v.data, v.data + v.size);
  } else {
    if (!v.read_to_host) throw invalid_argument_error("to_vector: a device view without owner");
    v.read_to_host(res, out.data());
  }
  return out;
}

// ---- graph properties and edge lists (graph/graph_properties.hpp, io/edge_list) ----------------
struct graph_properties {
  dyngb200_props p{};
  graph_properties() { dyngb200_props_default(&p); }
  static graph_properties mosp_compatible() {
    graph_properties g;
    dyngb200_props_mosp_compatible(&g.p);
    return g;
  }
};

template <typename V, typename W>
struct edge_list_view {
  std::int64_t num_vertices = 0;
  array_view<V> src, dst;
  array_view<W> weights;  // num_weights per edge, edge-major
  int num_weights = 1;
};

template <typename V = std::int32_t, typename W = std::int32_t>
struct edge_list {
  static_assert(detail::is_i32<V> && detail::is_i32<W>, "dyng_b200: int32 ids and weights");
  std::int64_t num_vertices = 0;
  std::vector<V> src, dst;
  std::vector<W> weights;
  int num_weights = 1;
  edge_list_view<V, W> view() const {
    edge_list_view<V, W> v;
    v.num_vertices = num_vertices;
    v.src = {src.data(), static_cast<std::int64_t>(src.size()), memory_space::host, {}};
    v.dst = {dst.data(), static_cast<std::int64_t>(dst.size()), memory_space::host, {}};
    v.weights = {weights.data(), static_cast<std::int64_t>(weights.size()), memory_space::host, {}};
    v.num_weights = num_weights;
    return v;
  }
};

// ---- edge batches (graph/edge_batch.hpp:38-404) ------------------------------------------------
template <typename V = std::int32_t, typename W = std::int32_t>
struct edge_batch_view {
  array_view<V> insert_src, insert_dst;
  array_view<W> insert_weights;  // num_weights per insertion
  array_view<V> delete_src, delete_dst;
  int num_weights = 1;
  std::int64_t num_insertions() const { return insert_src.size; }
  std::int64_t num_deletions() const { return delete_src.size; }
  dyngb200_batch native() const {
    dyngb200_batch b{};
    b.insert_src = insert_src.data;
    b.insert_dst = insert_dst.data;
    b.insert_weights = insert_weights.data;
    b.num_insertions = insert_src.size;
    b.delete_src = delete_src.data;
    b.delete_dst = delete_dst.data;
    b.num_deletions = delete_src.size;
    b.num_weights = num_weights;
    b.memory = static_cast<std::int32_t>(insert_src.size ? insert_src.space : delete_src.space);
    return b;
  }
};

template <typename V = std::int32_t, typename W = std::int32_t>
class edge_batch {
  static_assert(detail::is_i32<V> && detail::is_i32<W>, "dyng_b200: int32 ids and weights");

 public:
  explicit edge_batch(int num_weights = 1) : k_(num_weights) {}
  void insert_edge(V u, V v, std::initializer_list<W> w) {
    if (static_cast<int>(w.size()) != k_)
      throw invalid_argument_error("edge_batch::insert_edge: wrong number of weights");
    is_.push_back(u);
    id_.push_back(v);
    iw_.insert(iw_.end(), w.begin(), w.end());
  }
  void delete_edge(V u, V v) {
    ds_.push_back(u);
    dd_.push_back(v);
  }
  void clear() {
    is_.clear();
    id_.clear();
    iw_.clear();
    ds_.clear();
    dd_.clear();
  }
  edge_batch_view<V, W> view() const {
    edge_batch_view<V, W> b;
    b.insert_src = {is_.data(), static_cast<std::int64_t>(is_.size()), memory_space::host, {}};
    b.insert_dst = {id_.data(), static_cast<std::int64_t>(id_.size()), memory_space::host, {}};
    b.insert_weights = {iw_.data(), static_cast<std::int64_t>(iw_.size()), memory_space::host, {}};
    b.delete_src = {ds_.data(), static_cast<std::int64_t>(ds_.size()), memory_space::host, {}};
    b.delete_dst = {dd_.data(), static_cast<std::int64_t>(dd_.size()), memory_space::host, {}};
    b.num_weights = k_;
    return b;
  }

 private:
  int k_;
  std::vector<V> is_, id_, ds_, dd_;
  std::vector<W> iw_;
};

struct apply_summary : dyngb200_apply_summary {};

// ---- graph (graph/graph.hpp:96-508) ------------------------------------------------------------
template <typename V = std::int32_t, typename E = std::int64_t, typename W = std::int32_t>
class graph {
  static_assert(detail::is_i32<V> && std::is_same_v<E, std::int64_t> && detail::is_i32<W>,
                "dyng_b200 builds graph<int32, int64, int32>");

 public:
  static graph from_edges(const resources& res, const edge_list_view<V, W>& e,
                          const graph_properties& props = {}) {
    dyngb200_graph h = nullptr;
    detail::check(dyngb200_graph_from_edges(res.handle(), e.num_vertices, e.src.data, e.dst.data,
                                            e.weights.data, e.src.size, e.num_weights,
                                            static_cast<std::int32_t>(e.src.space), &props.p, &h));
    return graph(h);
  }
  static graph from_csr(const resources& res, std::int64_t num_vertices, const E* row_ptr,
                        const V* col_ind, const W* weights, int num_weights = 1,
                        const graph_properties& props = {},
                        memory_space space = memory_space::host) {
    dyngb200_graph h = nullptr;
    detail::check(dyngb200_graph_from_csr(res.handle(), num_vertices, row_ptr, col_ind, weights,
                                          num_weights, static_cast<std::int32_t>(space), &props.p,
                                          &h));
    return graph(h);
  }
  apply_summary apply(const resources& res, const edge_batch_view<V, W>& b) {
    apply_summary s{};
    const dyngb200_batch nb = b.native();
    detail::check(dyngb200_graph_apply(res.handle(), h_.get(), &nb, &s));
    return s;
  }
  std::int64_t num_vertices() const { return info().n; }
  std::int64_t num_edges() const { return info().m; }
  int num_weights() const { return info().k; }
  std::uint64_t version() const { return info().version; }
  dyngb200_graph handle() const { return h_.get(); }

 private:
  struct info_t {
    std::int64_t n, m;
    std::int32_t k;
    std::uint64_t version;
  };
  info_t info() const {
    info_t i{};
    detail::check(dyngb200_graph_info(h_.get(), &i.n, &i.m, &i.k, &i.version));
    return i;
  }
  explicit graph(dyngb200_graph h)
      : h_(h, [](dyngb200_graph p) { dyngb200_graph_destroy(p); }) {}
  std::shared_ptr<dyngb200_graph_s> h_;
};

// ---- sssp (sssp.hpp:78-489) --------------------------------------------------------------------
namespace sssp {

struct options {
  std::int64_t delta = 0;
  int objective = 0;
  engine cuda_engine = engine::automatic;
  bool validate_inputs = true;
  dyngb200_options native() const {
    return dyngb200_options{delta, objective, static_cast<std::int32_t>(cuda_engine),
                            validate_inputs ? 1 : 0};
  }
};

// sssp::stats (sssp.hpp:100-117), plus the schedule that ran and the device times.
struct stats : dyngb200_stats {};

constexpr std::int64_t infinite_distance = INT64_MAX / 4;

template <typename V = std::int32_t, typename D = std::int64_t>
class result {
  static_assert(detail::is_i32<V> && std::is_same_v<D, std::int64_t>,
                "dyng_b200 builds result<int32, int64>");

 public:
  // result::from_arrays (sssp.hpp:253-302): host arrays of n entries each.
  template <typename E, typename W>
  static result from_arrays(const resources& res, const graph<V, E, W>& g, V source,
                            const std::vector<D>& distances, const std::vector<V>& parents,
                            bool canonicalize = true, const options& opt = {}) {
    if (distances.size() != parents.size())
      throw invalid_argument_error("from_arrays: distances and parents differ in length");
    const dyngb200_options o = opt.native();
    dyngb200_tree t = nullptr;
    detail::check(dyngb200_tree_from_arrays(res.handle(), g.handle(), source, distances.data(),
                                            parents.data(),
                                            static_cast<std::int64_t>(distances.size()),
                                            DYNGB200_HOST, canonicalize ? 1 : 0, &o, &t));
    return result(t);
  }
  result clone(const resources& res) const {
    dyngb200_tree t = nullptr;
    detail::check(dyngb200_tree_clone(res.handle(), h_.get(), &t));
    return result(t);
  }
  V source() const { return info().source; }
  std::uint64_t graph_version() const { return info().version; }
  bool poisoned() const { return info().poisoned != 0; }
  options get_options() const {
    const dyngb200_options o = info().opt;
    return options{o.delta, o.objective, static_cast<engine>(o.cuda_engine), o.validate_inputs != 0};
  }
  void set_options(const options& opt) {
    const dyngb200_options o = opt.native();
    detail::check(dyngb200_tree_set_options(h_.get(), &o));
  }
  // Device views of the distances and parents (valid until the next update of this result).
  array_view<D> distances() const {
    const std::int64_t* d = nullptr;
    detail::check(dyngb200_tree_device_arrays(h_.get(), &d, nullptr));
    auto h = h_;
    return {d, info().n, memory_space::device, [h](const resources& r, D* out) {
              detail::check(dyngb200_tree_distances(r.handle(), h.get(), out, DYNGB200_HOST));
            }};
  }
  array_view<V> parents() const {
    const std::int32_t* p = nullptr;
    detail::check(dyngb200_tree_device_arrays(h_.get(), nullptr, &p));
    auto h = h_;
    return {p, info().n, memory_space::device, [h](const resources& r, V* out) {
              detail::check(dyngb200_tree_parents(r.handle(), h.get(), out, DYNGB200_HOST));
            }};
  }
  dyngb200_tree handle() const { return h_.get(); }
  explicit result(dyngb200_tree t) : h_(t, [](dyngb200_tree p) { dyngb200_tree_destroy(p); }) {}

 private:
  struct info_t {
    std::int32_t source;
    std::int64_t n;
    std::uint64_t version;
    std::int32_t poisoned;
    dyngb200_options opt;
  };
  info_t info() const {
    info_t i{};
    detail::check(dyngb200_tree_info(h_.get(), &i.source, &i.n, &i.version, &i.poisoned, &i.opt));
    return i;
  }
  std::shared_ptr<dyngb200_tree_s> h_;
};

// sssp::compute(resources::cuda(), g, source, opt) (sssp.hpp:415-421).
template <typename V, typename E, typename W>
result<V> compute(const resources& res, const graph<V, E, W>& g, V source,
                  const options& opt = {}) {
  const dyngb200_options o = opt.native();
  dyngb200_tree t = nullptr;
  detail::check(dyngb200_sssp_compute(res.handle(), g.handle(), source, &o, &t, nullptr));
  return result<V>(t);
}

// sssp::update(resources::cuda(), g, batch, tree) (sssp.hpp:484-489).
template <typename V, typename E, typename W>
stats update(const resources& res, graph<V, E, W>& g, const edge_batch_view<V, W>& batch,
             result<V>& tree) {
  stats st{};
  const dyngb200_batch b = batch.native();
  detail::check(dyngb200_sssp_update(res.handle(), g.handle(), &b, tree.handle(), &st));
  return st;
}

}  // namespace sssp

// ---- mosp (mosp.hpp:79-506) ----------------------------------------------------------------------
namespace mosp {

inline constexpr int max_objectives = 64;
inline constexpr std::int64_t max_preference_scale = std::int64_t{1} << 20;

// mosp::options (mosp.hpp:79-101).
struct options {
  std::vector<std::int32_t> preferences;
  std::int64_t delta = 0;
  engine cuda_engine = engine::automatic;
  bool compute_path_costs = true;
  bool validate_inputs = true;
  int num_objectives = 0;
  dyngb200_mosp_options native() const {
    dyngb200_mosp_options o{};
    o.num_objectives = num_objectives;
    o.num_preferences = static_cast<std::int32_t>(preferences.size());
    o.preferences = preferences.empty() ? nullptr : preferences.data();
    o.delta = delta;
    o.compute_path_costs = compute_path_costs ? 1 : 0;
    o.validate_inputs = validate_inputs ? 1 : 0;
    return o;
  }
};

// mosp::stats (mosp.hpp:115-125): the batch, `affected`, the combined graph's edges, L and the
// K sssp updates in objective order.
struct stats : dyngb200_mosp_stats {
  std::vector<sssp::stats> objectives;
};

// mosp::result (mosp.hpp:138-348): the K trees, the MOSP tree and the path costs.
template <typename V = std::int32_t, typename D = std::int64_t>
class result {
  static_assert(detail::is_i32<V> && std::is_same_v<D, std::int64_t>,
                "dyng_b200 builds mosp::result<int32, int64>");

 public:
  // result::from_arrays (mosp.hpp:300-347): K host trees of n entries each.
  template <typename E, typename W>
  static result from_arrays(const resources& res, const graph<V, E, W>& g, V source,
                            const std::vector<std::vector<D>>& distances,
                            const std::vector<std::vector<V>>& parents,
                            bool canonicalize = true, const options& opt = {}) {
    if (distances.size() != parents.size())
      throw invalid_argument_error("mosp::result::from_arrays: as many distance as parent arrays");
    std::vector<const std::int64_t*> dp;
    std::vector<const std::int32_t*> pp;
    std::int64_t n = distances.empty() ? 0 : static_cast<std::int64_t>(distances[0].size());
    for (std::size_t k = 0; k < distances.size(); ++k) {
      if (static_cast<std::int64_t>(distances[k].size()) != n ||
          static_cast<std::int64_t>(parents[k].size()) != n)
        throw invalid_argument_error("mosp::result::from_arrays: arrays of different lengths");
      dp.push_back(distances[k].data());
      pp.push_back(parents[k].data());
    }
    const dyngb200_mosp_options o = opt.native();
    dyngb200_mosp m = nullptr;
    detail::check(dyngb200_mosp_from_arrays(res.handle(), g.handle(), source,
                                            static_cast<std::int32_t>(dp.size()), dp.data(),
                                            pp.data(), n, DYNGB200_HOST, canonicalize ? 1 : 0, &o,
                                            &m));
    return result(m, opt);
  }
  int num_objectives() const { return info().k; }
  V source() const { return info().source; }
  std::int64_t preference_scale() const { return info().scale; }
  std::uint64_t graph_version() const { return info().version; }
  const options& get_options() const { return opt_; }
  void set_options(const options& opt) {
    const dyngb200_mosp_options o = opt.native();
    detail::check(dyngb200_mosp_set_options(h_.get(), &o));
    opt_ = opt;
  }
  // The trees of the objectives and the MOSP tree: device views (read with dyng::to_vector),
  // valid until the next update of this result.
  array_view<D> distances(int objective) const {
    const dyngb200_tree t = tree(objective);
    const std::int64_t* d = nullptr;
    detail::check(dyngb200_tree_device_arrays(t, &d, nullptr));
    auto h = h_;
    return {d, info().n, memory_space::device, [h, t](const resources& r, D* out) {
              detail::check(dyngb200_tree_distances(r.handle(), t, out, DYNGB200_HOST));
            }};
  }
  array_view<V> parents(int objective) const {
    const dyngb200_tree t = tree(objective);
    const std::int32_t* p = nullptr;
    detail::check(dyngb200_tree_device_arrays(t, nullptr, &p));
    auto h = h_;
    return {p, info().n, memory_space::device, [h, t](const resources& r, V* out) {
              detail::check(dyngb200_tree_parents(r.handle(), t, out, DYNGB200_HOST));
            }};
  }
  array_view<D> combined_distances() const {
    auto h = h_;
    return {nullptr, info().n, memory_space::device, [h](const resources&, D* out) {
              detail::check(dyngb200_mosp_combined(h.get(), out, nullptr, DYNGB200_HOST));
            }};
  }
  array_view<V> combined_parents() const {
    auto h = h_;
    return {nullptr, info().n, memory_space::device, [h](const resources&, V* out) {
              detail::check(dyngb200_mosp_combined(h.get(), nullptr, out, DYNGB200_HOST));
            }};
  }
  // n x K, vertex-major (costs[v * K + k]); host memory, as the reference's path_costs().
  std::vector<D> path_costs() const {
    const info_t i = info();
    std::vector<D> out(static_cast<std::size_t>(i.n) * static_cast<std::size_t>(i.k));
    detail::check(dyngb200_mosp_path_costs(h_.get(), out.data()));
    return out;
  }
  dyngb200_mosp handle() const { return h_.get(); }
  result(dyngb200_mosp m, const options& opt)
      : h_(m, [](dyngb200_mosp p) { dyngb200_mosp_destroy(p); }), opt_(opt) {}

 private:
  struct info_t {
    std::int32_t k;
    std::int64_t n;
    std::int64_t scale;
    std::int32_t source;
    std::uint64_t version;
  };
  info_t info() const {
    info_t i{};
    detail::check(dyngb200_mosp_info(h_.get(), &i.k, &i.n, &i.scale, &i.source, &i.version));
    return i;
  }
  dyngb200_tree tree(int objective) const {
    dyngb200_tree t = nullptr;
    detail::check(dyngb200_mosp_tree(h_.get(), objective, &t));
    return t;
  }
  std::shared_ptr<dyngb200_mosp_s> h_;
  options opt_;
};

// mosp::compute(resources::cuda(), g, source, opt) (mosp.hpp:444-449).
template <typename V, typename E, typename W>
result<V> compute(const resources& res, const graph<V, E, W>& g, V source,
                  const options& opt = {}) {
  const dyngb200_mosp_options o = opt.native();
  dyngb200_mosp m = nullptr;
  detail::check(dyngb200_mosp_compute(res.handle(), g.handle(), source, &o, &m));
  return result<V>(m, opt);
}

// mosp::update(resources::cuda(), g, batch, r) (mosp.hpp:502-506).
template <typename V, typename E, typename W>
stats update(const resources& res, graph<V, E, W>& g, const edge_batch_view<V, W>& batch,
             result<V>& r) {
  stats st{};
  st.objectives.resize(static_cast<std::size_t>(r.num_objectives()));
  const dyngb200_batch b = batch.native();
  detail::check(dyngb200_mosp_update(res.handle(), g.handle(), &b, r.handle(), &st,
                                     st.objectives.data()));
  return st;
}

}  // namespace mosp
}  // namespace dyng

#endif  // DYNG_B200_DYNG_HPP
