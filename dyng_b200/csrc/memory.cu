// Device memory of the library: one stream-ordered pool per device that keeps what is freed.
//
// Graphs, trees and workspaces grow while they are in use (slack arenas, the edge index, batch
// scratch).  With plain cudaMalloc / cudaFree every growth asks the driver for memory, and on a
// busy machine a driver allocation or free has been seen to take half a second, stalling every
// update queued behind it.  Here the memory freed by a buffer stays in the pool (release
// threshold: never) and the next buffer that grows is carved from it without the driver.
//
// Allocation and free keep the semantics of cudaMalloc / cudaFree: both run on the pool's own
// stream and wait for it, and a free first waits for the device (as cudaFree does), so a buffer
// is never reused while a kernel on any stream may still touch it.
#include "internal.hpp"

#include <atomic>
#include <cstdint>
#include <mutex>
#include <unordered_map>

namespace dyngb200 {

namespace {

struct DevicePool {
  cudaMemPool_t pool = nullptr;
  cudaStream_t stream = nullptr;
};

std::mutex& pools_mutex() {
  static std::mutex m;
  return m;
}

// Pools live to the end of the process (buffers may be released from static destructors).
std::unordered_map<int, DevicePool>& pools() {
  static auto* p = new std::unordered_map<int, DevicePool>();
  return *p;
}

DevicePool& pool_of(int device) {
  std::lock_guard<std::mutex> lk(pools_mutex());
  auto it = pools().find(device);
  if (it != pools().end()) return it->second;
  DevicePool dp;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  DYNGB200_CUDA(cudaMemPoolCreate(&dp.pool, &props));
  uint64_t keep_all = UINT64_MAX;
  DYNGB200_CUDA(cudaMemPoolSetAttribute(dp.pool, cudaMemPoolAttrReleaseThreshold, &keep_all));
  DYNGB200_CUDA(cudaStreamCreateWithFlags(&dp.stream, cudaStreamNonBlocking));
  return pools().emplace(device, dp).first->second;
}

int current_device() {
  int d = 0;
  DYNGB200_CUDA(cudaGetDevice(&d));
  return d;
}

std::atomic<long long> g_alloc_count{0};
std::atomic<long long> g_fail_countdown{0};

}  // namespace

long long device_alloc_count() { return g_alloc_count.load(); }

void device_alloc_fail_at(long long nth) { g_fail_countdown.store(nth > 0 ? nth : 0); }

void* device_alloc(size_t bytes, int* device) {
  g_alloc_count.fetch_add(1);
  // the test hook of the allocation-failure sweeps: one allocation fails as cudaMalloc would
  // (nothing is allocated, the call reports out-of-memory)
  long long left = g_fail_countdown.load();
  while (left > 0 && !g_fail_countdown.compare_exchange_weak(left, left - 1)) {
  }
  if (left == 1)
    throw Error(DYNGB200_OUT_OF_MEMORY, "CUDA out of memory (an injected allocation failure)");
  const int d = current_device();
  DevicePool& dp = pool_of(d);
  void* p = nullptr;
  DYNGB200_CUDA(cudaMallocFromPoolAsync(&p, bytes ? bytes : 1, dp.pool, dp.stream));
  DYNGB200_CUDA(cudaStreamSynchronize(dp.stream));
  *device = d;
  return p;
}

void device_free(void* p, int device) noexcept {
  if (!p) return;
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return;
  if (prev != device) cudaSetDevice(device);
  DevicePool* dp = nullptr;
  {
    std::lock_guard<std::mutex> lk(pools_mutex());
    auto it = pools().find(device);
    if (it != pools().end()) dp = &it->second;
  }
  if (dp) {
    cudaDeviceSynchronize();  // as cudaFree: nothing in flight may still use the memory
    cudaFreeAsync(p, dp->stream);
    cudaStreamSynchronize(dp->stream);
  }
  if (prev != device) cudaSetDevice(prev);
}

void device_pool_reserve(size_t bytes) {
  if (bytes == 0) return;
  int d = 0;
  void* p = device_alloc(bytes, &d);
  device_free(p, d);
}

long long device_pool_idle_bytes(int device) {
  DevicePool* dp = nullptr;
  {
    std::lock_guard<std::mutex> lk(pools_mutex());
    auto it = pools().find(device);
    if (it != pools().end()) dp = &it->second;
  }
  if (!dp) return 0;
  uint64_t reserved = 0, used = 0;
  if (cudaMemPoolGetAttribute(dp->pool, cudaMemPoolAttrReservedMemCurrent, &reserved) !=
          cudaSuccess ||
      cudaMemPoolGetAttribute(dp->pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess)
    return 0;
  return reserved > used ? static_cast<long long>(reserved - used) : 0;
}

}  // namespace dyngb200
