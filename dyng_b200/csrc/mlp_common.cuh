// The learned scheduler's shared definitions: the parameter layout of the 12 -> 64 -> 64 -> 15
// MLP, the bf16 helpers, the feature standardization and the per-update inference, which the
// batch applier's first block runs on the device (mlp.cu holds training and batch inference).
#pragma once

#include "internal.hpp"

#include <cuda_bf16.h>

namespace dyngb200 {

constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpHidden * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kMlpOut * kMlpHidden;
static_assert(kOffB3 + kMlpOut == kMlpParams, "parameter layout");
// bf16 weight copies: W1, W2, W3 back to back
constexpr int kBfW1 = 0;
constexpr int kBfW2 = kBfW1 + kMlpHidden * kMlpIn;
constexpr int kBfW3 = kBfW2 + kMlpHidden * kMlpHidden;
constexpr int kBfCount = kBfW3 + kMlpOut * kMlpHidden;

// heads: width class (8 logits), switch class (4), grid class (3)
__host__ __device__ constexpr int head_begin(int h) { return h == 0 ? 0 : (h == 1 ? 8 : 12); }
__host__ __device__ constexpr int head_size(int h) { return h == 0 ? 8 : (h == 1 ? 4 : 3); }

__device__ __forceinline__ float bf(uint16_t h) {
  return __uint_as_float(static_cast<unsigned>(h) << 16);
}
// round-to-nearest-even fp32 -> bf16 (the rounding of __float2bfloat16)
__device__ __forceinline__ uint16_t to_bf(float f) {
  return __bfloat16_as_ushort(__float2bfloat16(f));
}
__device__ __forceinline__ float round_bf(float f) { return bf(to_bf(f)); }

// Feature standardization, passed by value: x' = (x - mean) * scale.
struct FeatNorm {
  float mean[kMlpIn];
  float scale[kMlpIn];
  float lo[kMlpIn], hi[kMlpIn];  // the trained range (used by inference when `ranged`)
  int ranged;
};

__device__ __forceinline__ float lg(double v) { return static_cast<float>(log2(1.0 + (v > 0 ? v : 0))); }

// Shared memory of the inference (one block).
struct InferShared {
  float f[kMlpIn];
  float xs[kMlpIn];
  float h1[kMlpHidden], h2[kMlpHidden], lo[kMlpOut];
  __align__(16) uint16_t sw[kBfCount];  // the bf16 weights
};

// What the inference of one update reads besides the control block.
struct InferArgs {
  const float* params;       // fp32 master weights (biases); nullptr: the features only
  const uint16_t* w;         // bf16 copies of W1, W2, W3
  FeatNorm nrm;
  const TreeHistory* hist;   // the tree's record of its previous update
  int blocks;                // the full persistent grid (the grid classes scale it)
};

// The 12 features of one update, the MLP on them and the schedule it picks, by one block of at
// least 64 threads (every thread calls it).  Runs after the plan (the default width is in
// c->delta) and before the sssp kernel reads the schedule fields.  a.params == nullptr: the
// features only (recording traces).
static __device__ __forceinline__ void infer_schedule_block(const InferArgs& a, UpdateCtl* c,
                                                  const GraphCounters* gc, long long ni,
                                                  long long nd, InferShared& sh) {
  static_assert(kBfCount % 8 == 0, "bf16 weights are staged 8 at a time");
  const float* params = a.params;
  const uint16_t* w = a.w;
  const FeatNorm& nrm = a.nrm;
  const TreeHistory* hist = a.hist;
  const int blocks = a.blocks;
  float* f = sh.f;
  float* xs = sh.xs;
  float* h1 = sh.h1;
  float* h2 = sh.h2;
  float* lo = sh.lo;
  uint16_t* sw = sh.sw;
  const int lane = threadIdx.x;
  if (params && threadIdx.x >= 32) {
    const uint4* src = reinterpret_cast<const uint4*>(w);
    uint4* dst = reinterpret_cast<uint4*>(sw);
    for (int i = threadIdx.x - 32; i < kBfCount / 8; i += blockDim.x - 32) dst[i] = src[i];
  }
  if (lane == 0) {
    const long long ops = ni + nd;
    const long long n = gc->n, m = gc->m;
    const long long srcs = c->feat_acc[3];
    TreeHistory h{};
    if (hist) h = *hist;
    int fmax = 0;
    for (int i = 1; i < 4; ++i) fmax = max(fmax, h.frontier[i]);
    f[0] = lg(static_cast<double>(ops));
    f[1] = ops > 0 ? static_cast<float>(ni) / static_cast<float>(ops) : 0.0f;
    f[2] = nd > 0 ? static_cast<float>(c->feat_acc[0]) / static_cast<float>(nd) : 0.0f;
    f[3] = lg(srcs > 0 ? static_cast<double>(c->feat_acc[1]) / srcs : 0.0);
    f[4] = lg(static_cast<double>(c->feat_acc[2]));
    f[5] = lg(static_cast<double>(n));
    f[6] = lg(n > 0 ? static_cast<double>(m) / n : 0.0);
    f[7] = lg(static_cast<double>(c->delta));
    f[8] = lg(static_cast<double>(h.invalidated));
    f[9] = lg(static_cast<double>(abs(h.frontier[0])));
    f[10] = lg(static_cast<double>(abs(fmax)));
    f[11] = lg(static_cast<double>(h.iterations));
  }
  __syncthreads();
  if (lane < kMlpIn) c->features[lane] = f[lane];
  if (!params) {
    if (lane < 3) c->sched_classes[lane] = -1;
    return;
  }
  // outside the trained range the network would extrapolate: keep the plain schedule
  bool outside = false;
  if (nrm.ranged)
    for (int i = 0; i < kMlpIn; ++i) outside |= f[i] < nrm.lo[i] || f[i] > nrm.hi[i];
  if (outside) {
    if (lane < 3) c->sched_classes[lane] = -2;
    return;
  }
  // the MLP with one thread per output, in the arithmetic (and order) of warp_forward
  if (lane < kMlpIn) xs[lane] = round_bf((f[lane] - nrm.mean[lane]) * nrm.scale[lane]);
  __syncthreads();
  if (lane < kMlpHidden) {
    float acc = params[kOffB1 + lane];
    for (int i = 0; i < kMlpIn; ++i) acc = fmaf(bf(sw[kBfW1 + lane * kMlpIn + i]), xs[i], acc);
    h1[lane] = round_bf(fmaxf(acc, 0.0f));
  }
  __syncthreads();
  if (lane < kMlpHidden) {
    float acc = params[kOffB2 + lane];
    for (int i = 0; i < kMlpHidden; ++i) acc = fmaf(bf(sw[kBfW2 + lane * kMlpHidden + i]), h1[i], acc);
    h2[lane] = round_bf(fmaxf(acc, 0.0f));
  }
  __syncthreads();
  if (lane < kMlpOut) {
    float acc = params[kOffB3 + lane];
    for (int i = 0; i < kMlpHidden; ++i) acc = fmaf(bf(sw[kBfW3 + lane * kMlpHidden + i]), h2[i], acc);
    lo[lane] = acc;
  }
  __syncthreads();
  if (lane == 0) {
    int cls[3];
    for (int head = 0; head < 3; ++head) {
      const int b = head_begin(head);
      int best = 0;
      for (int j = 1; j < head_size(head); ++j)
        if (lo[b + j] > lo[b + best]) best = j;
      cls[head] = best;
      c->sched_classes[head] = best;
    }
    // width: the plan's default times 4^(class - 2)
    const long long base = c->delta > 0 ? c->delta : 1;
    long long d = base;
    if (cls[0] >= 2) {
      const int sh = 2 * (cls[0] - 2);
      d = base > (1LL << 40) >> sh ? (1LL << 40) : base << sh;
    } else {
      d = base >> (2 * (2 - cls[0]));
    }
    c->sched_delta = d > 0 ? d : 1;
    c->sched_walk = cls[1] >= 2 ? 1 : 0;
    c->sched_small = (cls[1] & 1) ? 0 : kDefaultSmall;
    c->active_blocks = cls[2] == 2 ? 0 : max(1, blocks >> (2 - cls[2]));
  }
}

}  // namespace dyngb200
