// The reference's C++ quickstart (README.md:67-83) against include/dyng/dyng.hpp, on the CUDA
// backend; prints "0 4 1 2 | invalidated 2".  Then an error path: a stale result is rejected
// with dyng::stale_result_error.
#include <dyng/dyng.hpp>

#include <iostream>

int main() {
  auto res = dyng::resources::cuda();
  dyng::edge_list<std::int32_t, std::int32_t> edges{4, {0, 0, 2, 1}, {1, 2, 1, 3}, {4, 1, 2, 1}, 1};
  auto g = dyng::graph<>::from_edges(res, edges.view());
  auto tree = dyng::sssp::compute(res, g, /*source=*/0);
  dyng::edge_batch<std::int32_t, std::int32_t> batch;
  batch.delete_edge(2, 1);
  batch.insert_edge(2, 3, {1});
  auto old = tree.clone(res);
  auto st = dyng::sssp::update(res, g, batch.view(), tree);
  for (auto d : dyng::to_vector(res, tree.distances())) std::cout << d << ' ';
  std::cout << "| invalidated " << st.invalidated << '\n';
  try {
    dyng::sssp::update(res, g, batch.view(), old);
    std::cout << "stale result accepted\n";
    return 1;
  } catch (const dyng::stale_result_error&) {
    std::cout << "stale_result_error\n";
  }
  try {
    (void)dyng::resources::sequential();
    return 1;
  } catch (const dyng::not_supported_error&) {
    std::cout << "not_supported_error\n";
  }
  return 0;
}
