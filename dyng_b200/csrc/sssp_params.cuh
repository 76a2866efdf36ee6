// The launch parameters of the sssp engines (the fused persistent kernel in sssp.cu and the
// operators engine in operators.cu): the graph, the tree arrays, the applier's pair table and
// the workspace lists, as one struct passed by value.
#pragma once

#include "internal.hpp"

namespace dyngb200 {

struct SsspParams {
  GraphView g;
  int objective;
  int32_t source;
  int from_scratch;
  long long* dist;
  int32_t* parent;
  u64* packed;
  int tree_bits;         // format of the persistent words (-1: none); another format is rebuilt
  long long tree_n;      // vertices the tree held before this call (growth fills the rest)
  int walk;              // invalidation by a subtree walk instead of pointer jumping
  int tree_trusted;      // computed or validated: no parent cycle possible
  int offer_heads;       // canonical tree: insertion heads take the inserted edge's offer
  // pairs of the applier (update only) and the batch weights
  const u64* pair_key;
  const int* pair_list;
  const int* pair_flags;
  const int* pair_first;
  const int* pair_last;
  const int32_t* ins_w;
  int k;
  // scratch
  int* stamp;
  int* touch_stamp;
  int* flag;
  int* in_far;
  int* ancestor;
  int* candidates;
  int* frontier;
  int* near_a;
  int* near_b;
  int* far_a;
  int* far_b;
  int2* heavy_a;
  int2* heavy_b;
  int2* pull_heavy;
  int* cand_med;
  int* near_med_a;
  int* near_med_b;
  int* touched;
  int generation;
  int touch_gen;
  int heavy_degree;
  long long delta_override;
  int small_frontier;    // frontiers up to this size run on block 0 alone (0: never)
  UpdateCtl* ctl;
  TreeHistory* hist;
  int* pj_blk;           // survivor counts of the pointer-jumping rounds: 2 x kPjMaxBlocks
  const unsigned char* inc;  // the applier's weight-increase flags (pairs x k)
  int use_inc;           // 1: changed edges of `objective` from inc[] (a batch applied for another
                         // objective), 0: from the pair flags
  // the grid barrier: its time limit without progress (0: kBarrierTimeoutNs) and blocks it waits
  // for beyond the launched ones (0 outside tests; a phantom block makes every wait run out)
  unsigned long long barrier_limit_ns;
  int barrier_extra;
};

// Pair flags of the applier (graph.cu).
constexpr int kPairDelete = 1, kPairIncreased = 2, kPairHead = 4, kPairAppend = 8,
              kPairUpsert = 16, kPairUseFirst = 32;

// The operators engine: the update (or a from-scratch compute) as a sequence of ordinary kernel
// launches on ctx.stream with the loop driven from the host (operators.cu).  `p` is what the fused
// kernel would be launched with; the control block already holds the plan (the applier's, or
// compute's upload).  The final counters are left in the control block as the fused kernel leaves
// them.
void run_operators(Context& ctx, const SsspParams& p);
// The operators engine's grid (blocks of every launch but the one-block ones).
int operators_grid(const Context& ctx);

}  // namespace dyngb200
