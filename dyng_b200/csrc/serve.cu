// The serving loop: several graphs resident on one GPU, each with its own shortest-path tree,
// fed by batches that arrive at any time from any host thread.
//
// - Requests wait in per-graph FIFO queues, so the batches of one graph apply in arrival order
//   and every result is the one the same batches would give alone, one after the other.  A graph
//   is in at most one round at a time.
// - Lanes, each a dispatcher thread with its own stream: one large lane and one or more small
//   lanes.  A small lane runs rounds of small batches: the oldest waiting request of every free
//   graph (round-robin), all of their updates queued on the lane's stream before one wait
//   (sssp_update_begin / sssp_update_end), so the host work of one update overlaps the GPU work of
//   the previous ones and a round needs one host-device synchronisation.  The large lane runs one
//   large batch at a time.
// - The persistent kernel holds every SM it is given, so a small batch behind a large one would
//   wait for all of it.  While the large lane runs, its persistent grid is capped at (occupancy -
//   1) blocks per SM and the small lane's at one block per SM: the two grids together fill the
//   SMs' block slots exactly, so both are co-resident whatever the order of their blocks (no grid
//   barrier can wait on a block that has no slot).  With one small lane, a small round that
//   starts while the large lane is idle takes the whole grid, and a large batch waits for such a
//   round to end first.  With several small lanes the one-block-per-SM layer is split between
//   them in fixed shares: small batches of different graphs run side by side, each on the same
//   grid whatever else runs (a steady service time), and the grids of all lanes still sum to the
//   block slots.
// - Admission by free HBM: a graph is registered only if its workspace fits beside the reserve,
//   and a batch is dispatched only if its estimated scratch fits in the free device memory beyond
//   the reserve; otherwise it fails with OUT_OF_MEMORY instead of taking the device down.
// - Every graph has its own context (workspace, control block), pointed at the stream of the
//   lane that runs it.
#include "handles.hpp"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

struct dyngb200_server_s;

namespace dyngb200 {

using Clock = std::chrono::steady_clock;

struct ServerGraph;

// Page-locked host memory for the copies of queued batches: one slab of the back-pressure cap,
// allocated when the server starts and carved first-fit (free extents kept sorted and merged), so
// serving never asks the driver for host memory: a cudaMallocHost under load took milliseconds
// and held up the other lanes' CUDA calls meanwhile.
class PinnedSlab {
 public:
  void init(size_t ints) {
    mem_.reserve(ints);
    free_.clear();
    free_[0] = mem_.count;
  }
  // Room for n int32 values (nullptr: no free extent is large enough).
  int32_t* take(size_t n) {
    n = round(n);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      const size_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > n) free_[off + n] = len - n;
      return mem_.ptr + off;
    }
    return nullptr;
  }
  void give(int32_t* p, size_t n) {
    n = round(n);
    size_t off = static_cast<size_t>(p - mem_.ptr);
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + n == next->first) {  // merge with the extent after
      n += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {  // merge with the extent before
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += n;
        return;
      }
    }
    free_[off] = n;
  }
  bool owns(const int32_t* p) const { return p >= mem_.ptr && p < mem_.ptr + mem_.count; }

 private:
  static size_t round(size_t n) { return (std::max<size_t>(n, 1) + 63) & ~static_cast<size_t>(63); }
  HostBuf<int32_t> mem_;
  std::map<size_t, size_t> free_;  // offset -> length, in int32 values
};

struct ServerRequest {
  uint64_t ticket = 0;
  int slot = 0;
  int32_t* data = nullptr;   // pinned copy of the batch's five arrays (in the slab, or in `own`)
  size_t data_n = 0;
  std::unique_ptr<HostBuf<int32_t>> own;  // a batch larger than the slab: its own pinned copy
  dyngb200_batch batch{};
  long long ops = 0;
  Clock::time_point arrival, ready, start, begun, synced, finish;
  int group_size = 0;
  int lane = 0;
  ServerGraph* graph = nullptr;  // set when a lane takes the request
  bool done = false;
  dyngb200_status status = DYNGB200_OK;
  std::string message;
  dyngb200_stats stats{};
};

struct ServerGraph {
  std::unique_ptr<Context> ctx;
  Graph* g = nullptr;
  Tree* t = nullptr;
  std::deque<ServerRequest*> queue;
  bool busy = false;  // in a lane's round
};

class Server {
 public:
  Server(const dyngb200_server_config& cfg, const Scheduler* learned);
  ~Server();
  int add_graph(Graph& g, Tree& t);
  uint64_t submit(int slot, const dyngb200_batch& b);
  ServerRequest wait(uint64_t ticket);
  void drain();
  dyngb200_server_info info();

 private:
  void run(int lane);
  bool take_round(int lane, std::vector<ServerRequest*>& group, int& cap);
  void monitor();
  void dispatch(int lane, std::vector<ServerRequest*>& group, int cap);
  long long estimate_bytes(const ServerGraph& sg, const ServerRequest& r) const;
  void release_copy(ServerRequest& r);  // the caller holds mu_

  dyngb200_server_config cfg_{};
  const Scheduler* learned_ = nullptr;
  std::vector<cudaStream_t> streams_;  // one per lane: the small lanes', then the large lane's
  std::vector<std::unique_ptr<ServerGraph>> graphs_;
  std::unordered_map<uint64_t, std::unique_ptr<ServerRequest>> requests_;
  PinnedSlab slab_;
  std::mutex mu_;
  std::condition_variable work_cv_, done_cv_;
  std::vector<std::thread> workers_;
  std::thread monitor_;  // samples the free device memory for admission (off the dispatcher)
  std::condition_variable monitor_cv_;
  long long free_sample_ = -1;   // bytes free at the last sample (-1: none)
  long long admitted_since_ = 0; // scratch estimates admitted after that sample
  bool stop_ = false;
  uint64_t next_ticket_ = 1;
  size_t next_graph_ = 0;  // round-robin start
  // lanes: 1 until the first graph shows the GPU holds two persistent grids side by side
  int lanes_ = 1;
  int want_lanes_ = 2;  // the configured lanes (small ones plus the large one)
  int full_blocks_ = 0, small_blocks_ = 0;  // persistent grid: whole, the small lanes' layer
  std::vector<int> small_cap_;  // with several small lanes: each one's share of the layer
  bool large_running_ = false;  // the large lane's round is in flight
  bool large_wants_ = false;    // a large batch waits for a whole-grid small round to end
  bool small_full_ = false;     // a small round runs on the whole grid
  long long waiting_ = 0, running_ = 0;
  long long held_bytes_ = 0;  // pinned copies of queued batches (submit waits above the cap)
  static constexpr long long kHeldCap = 1LL << 30;
  static constexpr double kLargeMaxWaitMs = 5.0;  // a large batch waits at most this long
  static constexpr int kMaxLanes = 8;
  dyngb200_server_info info_{};
};

}  // namespace dyngb200

namespace dyngb200 {

// Bytes of the pinned copy a queued request holds.
long long held_of(const ServerRequest& r) {
  const long long ni = r.batch.num_insertions, nd = r.batch.num_deletions;
  const long long k = r.batch.num_weights > 0 ? r.batch.num_weights : 0;
  return (2 * ni + ni * k + 2 * nd) * static_cast<long long>(sizeof(int32_t));
}

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

Server::Server(const dyngb200_server_config& cfg, const Scheduler* learned)
    : cfg_(cfg), learned_(learned) {
  if (cfg_.max_group <= 0) cfg_.max_group = 8;
  if (cfg_.small_changes <= 0) cfg_.small_changes = 65536;
  if (cfg_.hbm_reserve_bytes <= 0) cfg_.hbm_reserve_bytes = 1LL << 30;
  expects(!learned_ || learned_->device == cfg_.device,
          "server: the scheduler belongs to another device");
  expects(cfg_.lanes >= 0 && cfg_.lanes <= kMaxLanes,
          "server: lanes is 0 (two), 1 or up to " + std::to_string(kMaxLanes));
  want_lanes_ = cfg_.lanes == 0 ? 2 : cfg_.lanes;
  DYNGB200_CUDA(cudaSetDevice(cfg_.device));
  streams_.assign(static_cast<size_t>(want_lanes_), nullptr);
  slab_.init(static_cast<size_t>(kHeldCap / sizeof(int32_t)));
  for (auto& st : streams_) DYNGB200_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  size_t free_b = 0, total_b = 0;
  DYNGB200_CUDA(cudaMemGetInfo(&free_b, &total_b));
  free_sample_ = static_cast<long long>(free_b);
  for (int lane = 0; lane < want_lanes_; ++lane)
    workers_.emplace_back([this, lane] { run(lane); });
  monitor_ = std::thread([this] { monitor(); });
}

// The free-memory query can take tens to hundreds of milliseconds on a busy machine, and while
// it runs the driver delays device allocations (an arena growth waited 0.3 s behind it): it runs
// here, every kMonitorMs, and the dispatcher reads the last sample minus what it admitted since.
void Server::monitor() {
  cudaSetDevice(cfg_.device);
  constexpr int kMonitorMs = 250;
  std::unique_lock<std::mutex> lk(mu_);
  while (!stop_) {
    monitor_cv_.wait_for(lk, std::chrono::milliseconds(kMonitorMs), [&] { return stop_; });
    if (stop_) break;
    lk.unlock();
    size_t free_b = 0, total_b = 0;
    const Clock::time_point q0 = Clock::now();
    const bool ok = cudaMemGetInfo(&free_b, &total_b) == cudaSuccess;
    const long long pooled = device_pool_idle_bytes(cfg_.device);  // free to the library too
    const long long us =
        std::chrono::duration_cast<std::chrono::microseconds>(Clock::now() - q0).count();
    lk.lock();
    info_.admission_us_max = std::max<long long>(info_.admission_us_max, us);
    if (ok) {
      free_sample_ = static_cast<long long>(free_b) + pooled;
      admitted_since_ = 0;
    }
  }
}

Server::~Server() {
  {
    std::unique_lock<std::mutex> lk(mu_);
    stop_ = true;
  }
  work_cv_.notify_all();
  monitor_cv_.notify_all();
  for (auto& w : workers_)
    if (w.joinable()) w.join();
  if (monitor_.joinable()) monitor_.join();
  graphs_.clear();
  for (auto& st : streams_)
    if (st) cudaStreamDestroy(st);
}

int Server::add_graph(Graph& g, Tree& t) {
  expects(g.device == cfg_.device, "server::add_graph: the graph belongs to another device");
  DeviceGuard guard(cfg_.device);
  expect_tree_current(g, t, "server::add_graph");
  auto sg = std::make_unique<ServerGraph>();
  sg->ctx = std::make_unique<Context>();
  context_init(*sg->ctx, cfg_.device, streams_[0]);
  // admission: the context's per-vertex workspace (~100 B per vertex of capacity) must fit
  size_t free_b = 0, total_b = 0;
  DYNGB200_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const long long need = 100LL * g.n_cap + (16LL << 20);
  if (static_cast<long long>(free_b) - need < cfg_.hbm_reserve_bytes)
    throw Error(DYNGB200_OUT_OF_MEMORY,
                "server::add_graph: the graph's workspace (" + std::to_string(need) +
                    " bytes) does not fit beside the reserve of " +
                    std::to_string(cfg_.hbm_reserve_bytes) + " bytes (" +
                    std::to_string(free_b) + " free)");
  sg->ctx->ws.reserve_vertices(g.n_cap, streams_[0]);
  DYNGB200_CUDA(cudaStreamSynchronize(streams_[0]));
  // the split: the large lane's grid takes all but one block slot per SM, the small lane's one
  const int per_sm = update_blocks_per_sm(*sg->ctx);
  // room for the graph to grow (index doublings, arena growths) kept in the device pool, so that
  // growth while serving does not wait for the driver
  const long long graph_bytes =
      2 * (g.n_cap * 16 + g.arena_cap * (4 + 4LL * g.k)) + 16 * g.ecap;
  if (static_cast<long long>(free_b) - need - graph_bytes > 2 * cfg_.hbm_reserve_bytes)
    device_pool_reserve(static_cast<size_t>(graph_bytes));
  sg->g = &g;
  sg->t = &t;
  std::unique_lock<std::mutex> lk(mu_);
  if (graphs_.empty()) {
    full_blocks_ = per_sm * sg->ctx->sm_count;
    small_blocks_ = sg->ctx->sm_count;
    lanes_ = want_lanes_ >= 2 && per_sm >= 2 ? want_lanes_ : 1;
    // several small lanes share the one-block-per-SM layer in equal parts
    const int small_lanes = lanes_ - 1;
    small_cap_.assign(static_cast<size_t>(std::max(small_lanes, 1)), small_blocks_);
    if (small_lanes > 1)
      for (int l = 0; l < small_lanes; ++l)
        small_cap_[l] = small_blocks_ / small_lanes + (l < small_blocks_ % small_lanes ? 1 : 0);
  }
  graphs_.push_back(std::move(sg));
  return static_cast<int>(graphs_.size()) - 1;
}

void Server::release_copy(ServerRequest& r) {
  if (r.data && slab_.owns(r.data)) slab_.give(r.data, r.data_n);
  r.data = nullptr;
  r.own.reset();
}

uint64_t Server::submit(int slot, const dyngb200_batch& b) {
  {
    std::unique_lock<std::mutex> lk(mu_);
    expects(slot >= 0 && slot < static_cast<int>(graphs_.size()),
            "server::submit: no graph in slot " + std::to_string(slot));
    expect_batch(*graphs_[slot]->g, b, "server::submit");
  }
  auto r = std::make_unique<ServerRequest>();
  r->slot = slot;
  r->arrival = Clock::now();
  const long long ni = b.num_insertions, nd = b.num_deletions;
  const int k = b.num_weights > 0 ? b.num_weights : 0;
  const size_t total = static_cast<size_t>(2 * ni + ni * k + 2 * nd);
  const long long bytes = static_cast<long long>(total * sizeof(int32_t));
  {
    // backpressure: queued batches hold at most kHeldCap bytes of pinned copies, all in the
    // slab (waiting for room when the free extents are too small); a batch larger than the slab
    // gets a copy of its own once nothing else is held
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] {
      if (held_bytes_ > 0 && held_bytes_ + bytes > kHeldCap) return false;
      r->data = slab_.take(total);
      return r->data != nullptr || held_bytes_ == 0;
    });
    held_bytes_ += bytes;
  }
  uint64_t ticket = 0;
  try {
    if (!r->data) {
      r->own = std::make_unique<HostBuf<int32_t>>();
      r->own->reserve(total);
      r->data = r->own->ptr;
    }
    r->data_n = total;
    int32_t* p = r->data;
    auto put = [&](const int32_t* src, long long count) {
      if (count > 0) {
        if (b.memory == DYNGB200_DEVICE)
          DYNGB200_CUDA(cudaMemcpy(p, src, count * sizeof(int32_t), cudaMemcpyDeviceToHost));
        else
          std::memcpy(p, src, count * sizeof(int32_t));
      }
      int32_t* at = p;
      p += count;
      return at;
    };
    r->batch = b;
    r->batch.insert_src = put(b.insert_src, ni);
    r->batch.insert_dst = put(b.insert_dst, ni);
    r->batch.insert_weights = put(b.insert_weights, ni * k);
    r->batch.delete_src = put(b.delete_src, nd);
    r->batch.delete_dst = put(b.delete_dst, nd);
    r->batch.memory = DYNGB200_HOST;
    r->ops = ni + nd;
    r->ready = Clock::now();
    std::unique_lock<std::mutex> lk(mu_);
    expects(!stop_, "server::submit: the server is shutting down");
    r->ticket = next_ticket_++;
    ticket = r->ticket;
    graphs_[slot]->queue.push_back(r.get());
    requests_.emplace(ticket, std::move(r));
    ++waiting_;
    ++info_.submitted;
  } catch (...) {
    std::unique_lock<std::mutex> lk(mu_);
    held_bytes_ -= bytes;
    if (r) release_copy(*r);
    done_cv_.notify_all();
    throw;
  }
  work_cv_.notify_all();  // either lane may be the one that takes it
  return ticket;
}

ServerRequest Server::wait(uint64_t ticket) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = requests_.find(ticket);
  expects(it != requests_.end(), "server::wait: unknown ticket " + std::to_string(ticket));
  ServerRequest* r = it->second.get();
  done_cv_.wait(lk, [&] { return r->done; });
  ServerRequest out;
  out.ticket = r->ticket;
  out.slot = r->slot;
  out.ops = r->ops;
  out.arrival = r->arrival;
  out.ready = r->ready;
  out.start = r->start;
  out.begun = r->begun;
  out.synced = r->synced;
  out.finish = r->finish;
  out.group_size = r->group_size;
  out.lane = r->lane;
  out.done = true;
  out.status = r->status;
  out.message = r->message;
  out.stats = r->stats;
  requests_.erase(it);
  return out;
}

void Server::drain() {
  std::unique_lock<std::mutex> lk(mu_);
  done_cv_.wait(lk, [&] { return waiting_ == 0 && running_ == 0; });
}

dyngb200_server_info Server::info() {
  std::unique_lock<std::mutex> lk(mu_);
  dyngb200_server_info i = info_;
  i.waiting = waiting_;
  i.lanes = lanes_;
  return i;
}

// Scratch a batch may need beyond what its graph holds: staging, the applier's pair tables and
// row lists, and the slack arenas growing by a batch's worth of appends in both directions.
long long Server::estimate_bytes(const ServerGraph& sg, const ServerRequest& r) const {
  const long long dir = sg.g->props.directed ? 1 : 2;
  const long long k = sg.g->k;
  return r.ops * (20 + dir * (96 + 2 * (4 + 4 * k) * 3 / 2)) + (1LL << 20);
}

// Picks the next round of `lane` (the caller holds mu_): true when it took requests, or failed
// some by admission (they are done); `cap` is the persistent grid of the round (0: whole).
bool Server::take_round(int lane, std::vector<ServerRequest*>& group, int& cap) {
  cap = 0;
  const size_t ng = graphs_.size();
  if (waiting_ == 0 || ng == 0 || lane >= lanes_) return false;
  const bool known = free_sample_ >= 0;
  long long free_left = known ? free_sample_ - admitted_since_ - cfg_.hbm_reserve_bytes : 0;
  bool failed = false;
  // take the head of graph gi into this round: admitted, or failed by admission (then done)
  auto take = [&](size_t gi) {
    ServerGraph& sg = *graphs_[gi];
    ServerRequest* r = sg.queue.front();
    sg.queue.pop_front();
    --waiting_;
    r->start = Clock::now();
    r->lane = lane;
    r->graph = &sg;
    const long long need = estimate_bytes(sg, *r);
    if (known && need > free_left) {
      // admission: the batch's scratch does not fit beside the reserve; fail it, keep the rest
      r->status = DYNGB200_OUT_OF_MEMORY;
      r->message = "server: admission refused: the batch needs about " + std::to_string(need) +
                   " bytes of device memory beyond the reserve, " +
                   std::to_string(std::max(free_left, 0LL)) + " are free";
      r->finish = Clock::now();
      r->done = true;
      ++info_.failed;
      held_bytes_ -= held_of(*r);
      release_copy(*r);
      failed = true;
      return;
    }
    free_left -= need;
    admitted_since_ += need;
    sg.busy = true;
    group.push_back(r);
  };
  auto head = [&](size_t gi, bool large) {
    const ServerGraph& sg = *graphs_[gi];
    return !sg.busy && !sg.queue.empty() && (sg.queue.front()->ops > cfg_.small_changes) == large;
  };
  auto small_heads = [&] {
    for (size_t step = 0; step < ng && static_cast<int>(group.size()) < cfg_.max_group; ++step) {
      const size_t gi = (next_graph_ + step) % ng;
      if (head(gi, false)) take(gi);
    }
    next_graph_ = (next_graph_ + 1) % ng;
  };
  size_t oldest_large = ng;
  for (size_t gi = 0; gi < ng; ++gi)
    if (head(gi, true) && (oldest_large == ng || graphs_[gi]->queue.front()->arrival <
                                                     graphs_[oldest_large]->queue.front()->arrival))
      oldest_large = gi;
  if (lanes_ == 1) {
    // One lane: small batches first; a large batch runs in a round of its own when no small head
    // waits, or once it has waited kLargeMaxWaitMs (no starvation).
    const bool overdue =
        oldest_large < ng &&
        ms_between(graphs_[oldest_large]->queue.front()->arrival, Clock::now()) > kLargeMaxWaitMs;
    if (!overdue) small_heads();
    if (group.empty() && !failed && oldest_large < ng) take(oldest_large);
  } else if (lane < lanes_ - 1) {
    small_heads();
    if (!group.empty()) {
      if (lanes_ == 2) {
        cap = large_running_ || large_wants_ ? small_blocks_ : 0;
        small_full_ = cap == 0;
      } else {
        cap = small_cap_[lane];
      }
    }
  } else {
    if (oldest_large == ng) {
      large_wants_ = false;
      return false;
    }
    if (small_full_) {  // a whole-grid small round is in flight: wait for it
      large_wants_ = true;
      return false;
    }
    large_wants_ = false;
    take(oldest_large);
    if (!group.empty()) {
      cap = full_blocks_ - small_blocks_;
      large_running_ = true;
      ++info_.large_rounds;
    }
  }
  return !group.empty() || failed;
}

void Server::run(int lane) {
  cudaSetDevice(cfg_.device);
  std::vector<ServerRequest*> group;
  for (;;) {
    group.clear();
    int cap = 0;
    {
      std::unique_lock<std::mutex> lk(mu_);
      for (;;) {
        if (stop_ && waiting_ == 0) return;
        if (take_round(lane, group, cap)) break;
        work_cv_.wait(lk);
      }
      running_ += static_cast<long long>(group.size());
    }
    done_cv_.notify_all();  // admission failures are done
    if (!group.empty()) dispatch(lane, group, cap);
    {
      std::unique_lock<std::mutex> lk(mu_);
      running_ -= static_cast<long long>(group.size());
      if (!group.empty()) {
        ++info_.rounds;
        info_.max_group =
            std::max<long long>(info_.max_group, static_cast<long long>(group.size()));
        if (lanes_ >= 2 && lane == lanes_ - 1) large_running_ = false;
        if (lanes_ == 2 && lane == 0) small_full_ = false;
      }
    }
    work_cv_.notify_all();  // graphs freed, a lane's grid released: the other lane may go on
    done_cv_.notify_all();
  }
}

// One round: every update of the group queued on the lane's stream, then one wait, then each
// update's results.  Distinct graphs, distinct contexts: no scratch is shared inside a round.
void Server::dispatch(int lane, std::vector<ServerRequest*>& group, int cap) {
  const size_t n = group.size();
  cudaStream_t stream = streams_[lane];
  std::vector<std::unique_ptr<PendingUpdate>> pending(n);
  std::vector<char> begun(n, 0);
  for (size_t i = 0; i < n; ++i) {
    ServerRequest* r = group[i];
    ServerGraph& sg = *r->graph;
    r->group_size = static_cast<int>(n);
    sg.ctx->stream = stream;  // the graph's previous round, on either lane, has completed
    sg.ctx->max_update_blocks = cap;
    try {
      expect_tree_current(*sg.g, *sg.t, "sssp::update");
      pending[i] = std::make_unique<PendingUpdate>();
      sssp_update_begin(*sg.ctx, *sg.g, *sg.t, r->batch, dyngb200_schedule{}, learned_,
                        *pending[i]);
      begun[i] = 1;
      r->begun = Clock::now();
    } catch (const Error& e) {
      r->status = e.status;
      r->message = e.what();
    } catch (const std::exception& e) {
      r->status = DYNGB200_INTERNAL;
      r->message = e.what();
    }
  }
  cudaStreamSynchronize(stream);  // errors surface in sssp_update_end
  const Clock::time_point synced = Clock::now();
  for (size_t i = 0; i < n; ++i) {
    ServerRequest* r = group[i];
    ServerGraph& sg = *r->graph;
    r->synced = synced;
    if (!begun[i]) r->begun = r->start;
    if (begun[i]) {
      try {
        sssp_update_end(*pending[i], &r->stats);
      } catch (const Error& e) {
        r->status = e.status;
        r->message = e.what();
      } catch (const std::exception& e) {
        r->status = DYNGB200_INTERNAL;
        r->message = e.what();
      }
    }
    pending[i].reset();
    sg.ctx->max_update_blocks = 0;
    const long long bytes = held_of(*r);
    r->finish = Clock::now();
    std::unique_lock<std::mutex> lk(mu_);
    release_copy(*r);
    held_bytes_ -= bytes;
    sg.busy = false;
    r->done = true;  // a waiter may take (and free) the request from here on
    if (r->status == DYNGB200_OK) ++info_.completed;
    else ++info_.failed;
  }
}

}  // namespace dyngb200

struct dyngb200_server_s {
  std::unique_ptr<dyngb200::Server> s;
};

using dyngb200::guarded;

extern "C" {

dyngb200_status dyngb200_server_create(const dyngb200_server_config* config,
                                       dyngb200_scheduler learned, dyngb200_server* out) {
  return guarded([&] {
    dyngb200::expects(config && out, "server_create: null argument");
    int count = 0;
    DYNGB200_CUDA(cudaGetDeviceCount(&count));
    dyngb200::expects(config->device >= 0 && config->device < count,
                      "server_create: no CUDA device " + std::to_string(config->device),
                      DYNGB200_NOT_SUPPORTED);
    auto h = std::make_unique<dyngb200_server_s>();
    h->s = std::make_unique<dyngb200::Server>(*config, learned ? &learned->s : nullptr);
    *out = h.release();
  });
}

dyngb200_status dyngb200_server_add_graph(dyngb200_server s, dyngb200_graph g, dyngb200_tree t,
                                          int32_t* slot) {
  return guarded([&] {
    dyngb200::expects(s && g && t && slot, "server_add_graph: null argument");
    *slot = s->s->add_graph(g->g, t->t);
  });
}

dyngb200_status dyngb200_server_submit(dyngb200_server s, int32_t slot,
                                       const dyngb200_batch* batch, uint64_t* ticket) {
  return guarded([&] {
    dyngb200::expects(s && batch && ticket, "server_submit: null argument");
    *ticket = s->s->submit(slot, *batch);
  });
}

dyngb200_status dyngb200_server_wait(dyngb200_server s, uint64_t ticket, dyngb200_stats* stats,
                                     dyngb200_request_times* times) {
  dyngb200::ServerRequest r;
  const dyngb200_status st = guarded([&] {
    dyngb200::expects(s != nullptr, "server_wait: null server");
    r = s->s->wait(ticket);
  });
  if (st != DYNGB200_OK) return st;
  if (stats) *stats = r.stats;
  if (times) {
    times->queued_ms = dyngb200::ms_between(r.arrival, r.start);
    times->service_ms = dyngb200::ms_between(r.start, r.finish);
    times->total_ms = dyngb200::ms_between(r.arrival, r.finish);
    times->group_size = r.group_size;
    const bool ran = r.synced.time_since_epoch().count() != 0;
    times->begin_ms = ran ? dyngb200::ms_between(r.start, r.begun) : 0.0;
    times->round_ms = ran ? dyngb200::ms_between(r.start, r.synced) : 0.0;
    times->copy_ms = dyngb200::ms_between(r.arrival, r.ready);
    times->lane = r.lane;
  }
  dyngb200::last_error() = r.message;
  return r.status;
}

dyngb200_status dyngb200_server_drain(dyngb200_server s) {
  return guarded([&] {
    dyngb200::expects(s != nullptr, "server_drain: null server");
    s->s->drain();
  });
}

dyngb200_status dyngb200_server_info_get(dyngb200_server s, dyngb200_server_info* info) {
  return guarded([&] {
    dyngb200::expects(s && info, "server_info: null argument");
    *info = s->s->info();
  });
}

dyngb200_status dyngb200_server_destroy(dyngb200_server s) {
  return guarded([&] { delete s; });
}

}  // extern "C"
