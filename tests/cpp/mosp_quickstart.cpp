// dyng::mosp through include/dyng/dyng.hpp: the two-objective graph of the reference's
// mosp_test.cpp:249-269 (0->1->3 best for objective 0, 0->2->3 for objective 1), compute with
// the default preferences and with Pref = {2, 1}, then one update.  Prints the combined
// distances, the MOSP tree and the costs of vertex 3 per case.
#include <dyng/dyng.hpp>

#include <iostream>

static void show(const dyng::resources& res, const dyng::mosp::result<>& r) {
  for (auto d : dyng::to_vector(res, r.combined_distances())) std::cout << d << ' ';
  std::cout << '|';
  for (auto p : dyng::to_vector(res, r.combined_parents())) std::cout << ' ' << p;
  const auto c = r.path_costs();
  const int k = r.num_objectives();
  std::cout << " | " << c[3 * k] << ' ' << c[3 * k + 1] << " | L " << r.preference_scale() << '\n';
}

int main() {
  auto res = dyng::resources::cuda();
  // two weights per edge, edge-major: (1, 5), (5, 1), (1, 5), (5, 1)
  dyng::edge_list<std::int32_t, std::int32_t> edges{4, {0, 0, 1, 2}, {1, 2, 3, 3},
                                                    {1, 5, 5, 1, 1, 5, 5, 1}, 2};
  auto g = dyng::graph<>::from_edges(res, edges.view());
  auto r = dyng::mosp::compute(res, g, /*source=*/0);
  show(res, r);
  dyng::mosp::options opt;
  opt.preferences = {2, 1};
  auto q = dyng::mosp::compute(res, g, 0, opt);
  show(res, q);
  dyng::edge_batch<std::int32_t, std::int32_t> batch(2);
  batch.delete_edge(1, 3);
  const auto st = dyng::mosp::update(res, g, batch.view(), r);
  show(res, r);
  std::cout << "affected " << st.affected << " objectives " << st.objectives.size() << '\n';
  return 0;
}
