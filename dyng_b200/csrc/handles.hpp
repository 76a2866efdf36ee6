// The opaque handle types of the C ABI and the host-side argument checks shared by the C-ABI
// translation units.  Not part of the public ABI.
#pragma once

#include "internal.hpp"

#include <new>
#include <string>

struct dyngb200_context_s {
  dyngb200::Context ctx;
};
struct dyngb200_graph_s {
  dyngb200::Graph g;
};
struct dyngb200_tree_s {
  dyngb200::Tree t;
};
struct dyngb200_scheduler_s {
  dyngb200::Scheduler s;
};

namespace dyngb200 {

// The tree must belong to the graph's current version and be usable (stale_result_error).
void expect_tree_current(const Graph& g, const Tree& t, const char* what);
// Sizes, weight count and array pointers of a batch.
void expect_batch(const Graph& g, const dyngb200_batch& b, const char* what);
// Makes `dev` the calling thread's current device for a scope.
struct DeviceGuard {
  int prev = 0;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != prev) cudaSetDevice(prev);
  }
};

// Context set-up: device attributes and the stream (a caller's stream, or one of its own).
void context_init(Context& c, int device, void* stream);

// The calling thread's last error message (dyngb200_last_error_message).
std::string& last_error();

// Runs a C-ABI body: exceptions become statuses, their messages the thread's last error.
template <typename F>
dyngb200_status guarded(F&& f) {
  try {
    f();
    last_error().clear();
    return DYNGB200_OK;
  } catch (const Error& e) {
    last_error() = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    last_error() = "out of host memory";
    return DYNGB200_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    last_error() = e.what();
    return DYNGB200_INTERNAL;
  }
}

}  // namespace dyngb200
