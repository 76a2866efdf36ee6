// The learned scheduler: a small bf16 MLP with hand-written training and inference kernels.
//
// Input: 12 batch features (standardized on the device); layers 12 -> 64 -> 64 -> 15 with ReLU;
// weights and activations in bf16, every dot product accumulated in fp32; three softmax heads:
//   - near-far width class (8): the plan's default width times 4^(c - 2), c = 0..7;
//   - switch class (4): invalidation by pointer jumping (pull-style, bottom-up) or by a subtree
//     walk (push-style, top-down) x small-frontier switch off / at 256 vertices;
//   - persistent-grid class (3): 1/2, 1 or 2 blocks of 256 threads per SM.
// A schedule never changes the distances or parents (the kernels reach the same fixed point);
// the fixed heuristic -- the default width, pointer jumping, the full occupancy grid -- is the
// fallback when no scheduler is given.
//
// Training: cross-entropy summed over the heads, mean over the batch, Adam on fp32 master weights
// whose bf16 copies the forward pass reads.  The gradients are accumulated per block in shared
// memory and folded into global memory with one atomicAdd per parameter and block.
#include "internal.hpp"
#include "mlp_common.cuh"

#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <vector>

namespace dyngb200 {

namespace {

// One sample's forward pass by one warp.  x: 12 standardized features; on return h1 / h2 hold
// the bf16-rounded ReLU activations (shared memory of this warp) and logits the 15 outputs.
__device__ __forceinline__ void warp_forward(const float* params, const uint16_t* w, const float* x,
                                             float* h1, float* h2, float* logits) {
  const int lane = threadIdx.x & 31;
  float xb[kMlpIn];
#pragma unroll
  for (int i = 0; i < kMlpIn; ++i) xb[i] = round_bf(x[i]);
  for (int o = lane; o < kMlpHidden; o += 32) {
    float acc = params[kOffB1 + o];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) acc = fmaf(bf(w[kBfW1 + o * kMlpIn + i]), xb[i], acc);
    h1[o] = round_bf(fmaxf(acc, 0.0f));
  }
  __syncwarp();
  for (int o = lane; o < kMlpHidden; o += 32) {
    float acc = params[kOffB2 + o];
    for (int i = 0; i < kMlpHidden; ++i) acc = fmaf(bf(w[kBfW2 + o * kMlpHidden + i]), h1[i], acc);
    h2[o] = round_bf(fmaxf(acc, 0.0f));
  }
  __syncwarp();
  if (lane < kMlpOut) {
    float acc = params[kOffB3 + lane];
    for (int i = 0; i < kMlpHidden; ++i) acc = fmaf(bf(w[kBfW3 + lane * kMlpHidden + i]), h2[i], acc);
    logits[lane] = acc;
  }
  __syncwarp();
}

__device__ __forceinline__ void load_features(const float* x, const FeatNorm& nrm, float* xs) {
  const int lane = threadIdx.x & 31;
  if (lane < kMlpIn) xs[lane] = (x[lane] - nrm.mean[lane]) * nrm.scale[lane];
  __syncwarp();
}

// Forward pass of a batch of raw feature rows: one warp per sample, logits [n x 15].
__global__ void k_mlp_forward(const float* params, const uint16_t* w, FeatNorm nrm, const float* x,
                              int n, float* logits) {
  __shared__ float sh[8][2 * kMlpHidden + kMlpOut + kMlpIn];
  const int wid = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  float* h1 = sh[wid];
  float* h2 = h1 + kMlpHidden;
  float* lo = h2 + kMlpHidden;
  float* xs = lo + kMlpOut;
  for (long long s = blockIdx.x * 8LL + wid; s < n; s += gridDim.x * 8LL) {
    load_features(x + s * kMlpIn, nrm, xs);
    warp_forward(params, w, xs, h1, h2, lo);
    if (lane < kMlpOut) logits[s * kMlpOut + lane] = lo[lane];
    __syncwarp();
  }
}

// Softmax of one head over lanes [begin, begin + size) of `lo`; returns the lane's probability
// (0 outside the head).
__device__ __forceinline__ float head_softmax(const float* lo, int head, int lane, float* loss,
                                              int label) {
  const int b = head_begin(head), sz = head_size(head);
  float mx = -INFINITY;
  for (int j = 0; j < sz; ++j) mx = fmaxf(mx, lo[b + j]);
  float sum = 0.0f;
  for (int j = 0; j < sz; ++j) sum += expf(lo[b + j] - mx);
  if (loss) *loss = logf(sum) + mx - lo[b + label];
  const int j = lane - b;
  return (j >= 0 && j < sz) ? expf(lo[b + j] - mx) / sum : 0.0f;
}

// Loss and gradients of samples idx[begin .. begin + count) (idx == nullptr: the identity),
// scaled by 1/count: cross-entropy summed over the three heads.  loss_out accumulates the summed
// loss times loss_scale.  The rounding of weights and
// activations to bf16 passes the gradient straight through.  One warp per sample; each block
// accumulates the gradient in shared memory, then adds it to `grads` once.
__global__ void __launch_bounds__(256) k_mlp_grad(const float* params, const uint16_t* w,
                                                  FeatNorm nrm, const float* x, const int* y,
                                                  const int* idx, long long begin, int count,
                                                  float* grads, double* loss_out,
                                                  double loss_scale) {
  __shared__ float acc[kMlpParams];
  __shared__ float sh[8][3 * kMlpHidden + 2 * kMlpOut + kMlpIn];
  __shared__ double block_loss;
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) acc[i] = 0.0f;
  if (threadIdx.x == 0) block_loss = 0.0;
  __syncthreads();
  const int wid = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  float* h1 = sh[wid];
  float* h2 = h1 + kMlpHidden;
  float* dh = h2 + kMlpHidden;
  float* lo = dh + kMlpHidden;
  float* dlo = lo + kMlpOut;
  float* xs = dlo + kMlpOut;
  const float inv = 1.0f / static_cast<float>(count > 0 ? count : 1);
  double warp_loss = 0.0;
  for (long long r = blockIdx.x * 8LL + wid; r < count; r += gridDim.x * 8LL) {
    const long long s = idx ? idx[begin + r] : begin + r;
    load_features(x + s * kMlpIn, nrm, xs);
    warp_forward(params, w, xs, h1, h2, lo);
    // dlogits = softmax - onehot, per head
    float g = 0.0f;
    for (int head = 0; head < 3; ++head) {
      const int label = y[s * 3 + head];
      float l = 0.0f;
      const float pr = head_softmax(lo, head, lane, &l, label);
      if (lane == 0) warp_loss += l;
      const int j = lane - head_begin(head);
      if (j >= 0 && j < head_size(head)) g = pr - (j == label ? 1.0f : 0.0f);
    }
    if (lane < kMlpOut) dlo[lane] = g * inv;
    __syncwarp();
    // layer 3: dW3[o][i] = dlo[o] h2[i]; dh2[i] = sum_o dlo[o] W3[o][i] (h2 > 0)
    if (lane < kMlpOut) atomicAdd(&acc[kOffB3 + lane], dlo[lane]);
    for (int i = lane; i < kMlpHidden; i += 32) {
      float d = 0.0f;
      for (int o = 0; o < kMlpOut; ++o) {
        atomicAdd(&acc[kOffW3 + o * kMlpHidden + i], dlo[o] * h2[i]);
        d = fmaf(dlo[o], bf(w[kBfW3 + o * kMlpHidden + i]), d);
      }
      dh[i] = h2[i] > 0.0f ? d : 0.0f;
    }
    __syncwarp();
    // layer 2: dW2[o][i] = dh2[o] h1[i]; dh1[i] = sum_o dh2[o] W2[o][i] (h1 > 0)
    for (int o = lane; o < kMlpHidden; o += 32) atomicAdd(&acc[kOffB2 + o], dh[o]);
    float dh1[2];
    for (int t = 0; t < 2; ++t) {
      const int i = lane + 32 * t;
      float d = 0.0f;
      for (int o = 0; o < kMlpHidden; ++o) {
        const float go = dh[o];
        if (go != 0.0f) {
          atomicAdd(&acc[kOffW2 + o * kMlpHidden + i], go * h1[i]);
          d = fmaf(go, bf(w[kBfW2 + o * kMlpHidden + i]), d);
        }
      }
      dh1[t] = h1[i] > 0.0f ? d : 0.0f;
    }
    __syncwarp();
    for (int t = 0; t < 2; ++t) dh[lane + 32 * t] = dh1[t];
    __syncwarp();
    // layer 1: dW1[o][i] = dh1[o] x[i]
    for (int o = lane; o < kMlpHidden; o += 32) {
      const float go = dh[o];
      atomicAdd(&acc[kOffB1 + o], go);
      if (go != 0.0f)
        for (int i = 0; i < kMlpIn; ++i) atomicAdd(&acc[kOffW1 + o * kMlpIn + i], go * round_bf(xs[i]));
    }
    __syncwarp();
  }
  if (lane == 0 && warp_loss != 0.0) atomicAdd(&block_loss, warp_loss);
  __syncthreads();
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x)
    if (acc[i] != 0.0f) atomicAdd(&grads[i], acc[i]);
  if (threadIdx.x == 0 && loss_out) atomicAdd(loss_out, block_loss * loss_scale);
}

// Index of a parameter's bf16 copy (-1: a bias, which stays fp32).
__device__ __forceinline__ int bf_index(int i) {
  if (i < kOffB1) return kBfW1 + (i - kOffW1);
  if (i >= kOffW2 && i < kOffB2) return kBfW2 + (i - kOffW2);
  if (i >= kOffW3 && i < kOffB3) return kBfW3 + (i - kOffW3);
  return -1;
}

// Adam step (bias-corrected) on the fp32 master weights, then their bf16 copies.
__global__ void k_adam(float* params, const float* grads, float* m, float* v, uint16_t* w, float lr,
                       float beta1, float beta2, float eps, float corr1, float corr2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpParams; i += gridDim.x * blockDim.x) {
    const float g = grads[i];
    const float mi = beta1 * m[i] + (1.0f - beta1) * g;
    const float vi = beta2 * v[i] + (1.0f - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float p = params[i] - lr * (mi / corr1) / (sqrtf(vi / corr2) + eps);
    params[i] = p;
    const int b = bf_index(i);
    if (b >= 0) w[b] = to_bf(p);
  }
}

__global__ void k_refresh_bf16(const float* params, uint16_t* w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpParams; i += gridDim.x * blockDim.x) {
    const int b = bf_index(i);
    if (b >= 0) w[b] = to_bf(params[i]);
  }
}

FeatNorm norm_of(const Scheduler& s) {
  FeatNorm nrm;
  for (int i = 0; i < kMlpIn; ++i) {
    nrm.mean[i] = s.feat_mean[i];
    nrm.scale[i] = s.feat_scale[i];
    nrm.lo[i] = s.feat_lo[i];
    nrm.hi[i] = s.feat_hi[i];
  }
  nrm.ranged = s.has_range ? 1 : 0;
  return nrm;
}

}  // namespace

void scheduler_refresh(Scheduler& s, cudaStream_t st) {
  k_refresh_bf16<<<8, 256, 0, st>>>(s.params.ptr, s.wbf16.ptr);
  DYNGB200_CUDA(cudaGetLastError());
}

// He-uniform weights from a seeded splitmix sequence, zero biases, identity standardization.
void scheduler_init(Context& ctx, Scheduler& s, uint64_t seed) {
  s.device = ctx.device;
  s.params.reserve(kMlpParams);
  s.wbf16.reserve(kBfCount);
  s.grads.reserve(kMlpParams);
  s.m.reserve(kMlpParams);
  s.v.reserve(kMlpParams);
  s.loss.reserve(1);
  std::vector<float> h(kMlpParams, 0.0f);
  uint64_t state = seed;
  auto uniform = [&]() {
    state += 0x9e3779b97f4a7c15ULL;
    uint64_t z = state;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    z ^= z >> 31;
    return static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
  };
  auto fill = [&](int off, int rows, int cols) {
    const double bound = std::sqrt(6.0 / cols);
    for (int i = 0; i < rows * cols; ++i) h[off + i] = static_cast<float>(uniform() * bound);
  };
  fill(kOffW1, kMlpHidden, kMlpIn);
  fill(kOffW2, kMlpHidden, kMlpHidden);
  fill(kOffW3, kMlpOut, kMlpHidden);
  for (int i = 0; i < kMlpIn; ++i) {
    s.feat_mean[i] = 0.0f;
    s.feat_scale[i] = 1.0f;
  }
  scheduler_set(ctx, s, h.data(), nullptr, nullptr);
}

void scheduler_set(Context& ctx, Scheduler& s, const float* params, const float* mean,
                   const float* scale) {
  cudaStream_t st = ctx.stream;
  if (params) {
    DYNGB200_CUDA(cudaMemcpyAsync(s.params.ptr, params, kMlpParams * sizeof(float),
                                  cudaMemcpyHostToDevice, st));
    DYNGB200_CUDA(cudaMemsetAsync(s.m.ptr, 0, kMlpParams * sizeof(float), st));
    DYNGB200_CUDA(cudaMemsetAsync(s.v.ptr, 0, kMlpParams * sizeof(float), st));
    s.step = 0;
    scheduler_refresh(s, st);
  }
  for (int i = 0; i < kMlpIn; ++i) {
    if (mean) s.feat_mean[i] = mean[i];
    if (scale) s.feat_scale[i] = scale[i];
  }
  DYNGB200_CUDA(cudaStreamSynchronize(st));
}

void scheduler_get(Context& ctx, const Scheduler& s, float* params, float* mean, float* scale) {
  if (params) {
    DYNGB200_CUDA(cudaMemcpyAsync(params, s.params.ptr, kMlpParams * sizeof(float),
                                  cudaMemcpyDeviceToHost, ctx.stream));
    DYNGB200_CUDA(cudaStreamSynchronize(ctx.stream));
  }
  for (int i = 0; i < kMlpIn; ++i) {
    if (mean) mean[i] = s.feat_mean[i];
    if (scale) scale[i] = s.feat_scale[i];
  }
}

static void upload_samples(Context& ctx, Scheduler& s, const float* x, const int32_t* y,
                           long long n) {
  const size_t nn = static_cast<size_t>(n > 0 ? n : 1);
  s.x.reserve(nn * kMlpIn);
  if (n > 0)
    DYNGB200_CUDA(cudaMemcpyAsync(s.x.ptr, x, n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice,
                                  ctx.stream));
  if (y) {
    s.y.reserve(nn * 3);
    if (n > 0)
      DYNGB200_CUDA(cudaMemcpyAsync(s.y.ptr, y, n * 3 * sizeof(int32_t), cudaMemcpyHostToDevice,
                                    ctx.stream));
  }
}

static void check_labels(const int32_t* y, long long n) {
  for (long long i = 0; i < n; ++i)
    for (int h = 0; h < 3; ++h)
      expects(y[i * 3 + h] >= 0 && y[i * 3 + h] < head_size(h),
              "scheduler: label " + std::to_string(y[i * 3 + h]) + " of sample " +
                  std::to_string(i) + " is outside head " + std::to_string(h));
}

void scheduler_forward(Context& ctx, Scheduler& s, const float* x, long long n, float* logits) {
  expects(n >= 0, "scheduler_forward: n must be >= 0");
  if (n == 0) return;
  expects(n <= INT32_MAX, "scheduler_forward: too many samples");
  upload_samples(ctx, s, x, nullptr, n);
  s.out.reserve(static_cast<size_t>(n) * kMlpOut);
  const int grid = static_cast<int>(std::min<long long>((n + 7) / 8, 1024));
  k_mlp_forward<<<grid, 256, 0, ctx.stream>>>(s.params.ptr, s.wbf16.ptr, norm_of(s), s.x.ptr,
                                              static_cast<int>(n), s.out.ptr);
  DYNGB200_CUDA(cudaGetLastError());
  DYNGB200_CUDA(cudaMemcpyAsync(logits, s.out.ptr, n * kMlpOut * sizeof(float),
                                cudaMemcpyDeviceToHost, ctx.stream));
  DYNGB200_CUDA(cudaStreamSynchronize(ctx.stream));
}

static int grad_grid(long long count) {
  return static_cast<int>(std::max<long long>(1, std::min<long long>((count + 7) / 8, 148)));
}

void scheduler_gradients(Context& ctx, Scheduler& s, const float* x, const int32_t* y, long long n,
                         float* grads, double* loss) {
  expects(n > 0, "scheduler_gradients: needs at least one sample");
  expects(n <= INT32_MAX, "scheduler_gradients: too many samples");
  check_labels(y, n);
  upload_samples(ctx, s, x, y, n);
  cudaStream_t st = ctx.stream;
  DYNGB200_CUDA(cudaMemsetAsync(s.grads.ptr, 0, kMlpParams * sizeof(float), st));
  DYNGB200_CUDA(cudaMemsetAsync(s.loss.ptr, 0, sizeof(double), st));
  k_mlp_grad<<<grad_grid(n), 256, 0, st>>>(s.params.ptr, s.wbf16.ptr, norm_of(s), s.x.ptr, s.y.ptr,
                                           nullptr, 0, static_cast<int>(n), s.grads.ptr,
                                           s.loss.ptr, 1.0 / static_cast<double>(n));
  DYNGB200_CUDA(cudaGetLastError());
  if (grads)
    DYNGB200_CUDA(cudaMemcpyAsync(grads, s.grads.ptr, kMlpParams * sizeof(float),
                                  cudaMemcpyDeviceToHost, st));
  double l = 0;
  DYNGB200_CUDA(cudaMemcpyAsync(&l, s.loss.ptr, sizeof(double), cudaMemcpyDeviceToHost, st));
  DYNGB200_CUDA(cudaStreamSynchronize(st));
  if (loss) *loss = l;
}

// Minibatch Adam over `epochs` passes of a seeded shuffle; returns the mean loss of the last pass
// (measured on the minibatches as they were trained).
void scheduler_train(Context& ctx, Scheduler& s, const float* x, const int32_t* y, long long n,
                     int epochs, int batch, float lr, uint64_t seed, double* final_loss) {
  expects(n > 0 && n <= INT32_MAX, "scheduler_train: needs 1 .. 2^31 - 1 samples");
  expects(epochs >= 1 && batch >= 1 && lr > 0.0f, "scheduler_train: bad epochs, batch or lr");
  check_labels(y, n);
  upload_samples(ctx, s, x, y, n);
  cudaStream_t st = ctx.stream;
  s.idx.reserve(static_cast<size_t>(n));
  std::vector<int32_t> perm(static_cast<size_t>(n));
  uint64_t state = seed;
  auto next = [&]() {
    state += 0x9e3779b97f4a7c15ULL;
    uint64_t z = state;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
  };
  const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  double l = 0;
  for (int e = 0; e < epochs; ++e) {
    for (long long i = 0; i < n; ++i) perm[i] = static_cast<int32_t>(i);
    for (long long i = n - 1; i > 0; --i) std::swap(perm[i], perm[next() % (i + 1)]);
    DYNGB200_CUDA(cudaMemcpyAsync(s.idx.ptr, perm.data(), n * sizeof(int32_t),
                                  cudaMemcpyHostToDevice, st));
    DYNGB200_CUDA(cudaMemsetAsync(s.loss.ptr, 0, sizeof(double), st));
    for (long long b0 = 0; b0 < n; b0 += batch) {
      const int count = static_cast<int>(std::min<long long>(batch, n - b0));
      DYNGB200_CUDA(cudaMemsetAsync(s.grads.ptr, 0, kMlpParams * sizeof(float), st));
      k_mlp_grad<<<grad_grid(count), 256, 0, st>>>(
          s.params.ptr, s.wbf16.ptr, norm_of(s), s.x.ptr, s.y.ptr, s.idx.ptr, b0, count,
          s.grads.ptr, s.loss.ptr, 1.0 / static_cast<double>(n));
      ++s.step;
      const float corr1 = 1.0f - std::pow(beta1, static_cast<float>(s.step));
      const float corr2 = 1.0f - std::pow(beta2, static_cast<float>(s.step));
      k_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(s.params.ptr, s.grads.ptr, s.m.ptr, s.v.ptr,
                                                       s.wbf16.ptr, lr, beta1, beta2, eps, corr1,
                                                       corr2);
    }
    DYNGB200_CUDA(cudaGetLastError());
  }
  DYNGB200_CUDA(cudaMemcpyAsync(&l, s.loss.ptr, sizeof(double), cudaMemcpyDeviceToHost, st));
  DYNGB200_CUDA(cudaStreamSynchronize(st));
  if (final_loss) *final_loss = l;
}

// Queued by the applier after its plan (its validation pass accumulated the batch features in
// the control block): the features and, with a scheduler, the schedule the MLP picks, written
// into the control block that the persistent kernel reads.
void learned_infer_args(Context& ctx, Tree& t, const Scheduler* sch, InferArgs* out) {
  InferArgs a{};
  a.params = sch ? sch->params.ptr : nullptr;
  a.w = sch ? sch->wbf16.ptr : nullptr;
  if (sch) a.nrm = norm_of(*sch);
  a.hist = t.hist.ptr;
  a.blocks = update_grid_blocks(ctx);
  *out = a;
}

}  // namespace dyngb200
