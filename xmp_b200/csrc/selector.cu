// Learned kernel-configuration selector: an MLP that maps a problem shape to
// a predicted log2(time) for every candidate slot, trained on the exhaustive
// tuner's measurements.  Its forward pass, backward pass, Adam update and
// grid inference are the CUDA kernels below (no framework): the selector
// only chooses a schedule, so every result it leads to stays bit-exact.
//
// Network: x[4] -> relu(W1 x + b1)[64] -> relu(W2 h1 + b2)[64] -> W3 h2 + b3 [48].
// Inputs (scaled logs): op - 1, (log2 bits - 10)/4, (log2 count - 13)/7,
// (log2(exp_bits + 1) - 7)/7.  Loss: mean squared error of log2(ms) over the
// valid (shape, slot) pairs.
#include "tune.h"
#include <math.h>
#include <string.h>
#include <vector>

using namespace xmpb;

namespace xmpb {

constexpr int kIn = 4, kH = XMP_SELECTOR_HIDDEN, kOut = XMP_TUNE_CANDIDATES;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kIn * kH, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH,
              kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH * kOut, kParams = kOffB3 + kOut;
static_assert(kParams == XMP_SELECTOR_PARAMS, "parameter layout");

static void features(const xmpTuneShape_t &s, float *x) {
  x[0] = (float)s.op - 1.0f;
  x[1] = (log2f((float)std::max(s.bits, 1u)) - 10.0f) / 4.0f;
  x[2] = (log2f((float)std::max(s.count, 1u)) - 13.0f) / 7.0f;
  x[3] = (log2f((float)s.exp_bits + 1.0f) - 7.0f) / 7.0f;
}

// out[b][j] = act(sum_i in[b][i] W[i][j] + bias[j])
__global__ void dense_fwd(const float *in, int in_dim, const float *W, const float *bias, float *out, int out_dim,
                          int n, int relu) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * out_dim) return;
  int b = t / out_dim, j = t % out_dim;
  float acc = bias[j];
  for (int i = 0; i < in_dim; i++) acc = fmaf(in[b * in_dim + i], W[i * out_dim + j], acc);
  out[t] = relu ? fmaxf(acc, 0.0f) : acc;
}

// dpred = d(mean sq err)/dpred on valid entries; loss accumulated (sum of squares)
__global__ void mse_grad(const float *pred, const float *target, const float *mask, float inv_count, int total,
                         float *dpred, float *loss_sum) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  float d = (pred[t] - target[t]) * mask[t];
  dpred[t] = 2.0f * d * inv_count;
  atomicAdd(loss_sum, d * d * inv_count);
}

// dW[i][j] = sum_b in[b][i] dout[b][j];  db[j] = sum_b dout[b][j]
__global__ void dense_bwd_w(const float *in, int in_dim, const float *dout, int out_dim, int n, float *dW,
                            float *db) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < in_dim * out_dim) {
    int i = t / out_dim, j = t % out_dim;
    float acc = 0.0f;
    for (int b = 0; b < n; b++) acc = fmaf(in[b * in_dim + i], dout[b * out_dim + j], acc);
    dW[t] = acc;
  } else if (t < in_dim * out_dim + out_dim) {
    int j = t - in_dim * out_dim;
    float acc = 0.0f;
    for (int b = 0; b < n; b++) acc += dout[b * out_dim + j];
    db[j] = acc;
  }
}

// din[b][i] = (sum_j dout[b][j] W[i][j]) * [act[b][i] > 0]
__global__ void dense_bwd_in(const float *dout, int out_dim, const float *W, const float *act, int in_dim, int n,
                             float *din) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * in_dim) return;
  int b = t / in_dim, i = t % in_dim;
  float acc = 0.0f;
  for (int j = 0; j < out_dim; j++) acc = fmaf(dout[b * out_dim + j], W[i * out_dim + j], acc);
  din[t] = act[t] > 0.0f ? acc : 0.0f;
}

__global__ void adam_step(float *p, const float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                          float c1, float c2) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  float gi = g[t];
  float mi = b1 * m[t] + (1.0f - b1) * gi, vi = b2 * v[t] + (1.0f - b2) * gi * gi;
  m[t] = mi;
  v[t] = vi;
  p[t] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// One grid cell per thread: forward pass with the weights in shared memory,
// argmin over the cell's valid slots (valid: bit mask per (op, limbs)).
// The table is filled from an ensemble of `members` networks (parameters
// back to back): a cell's predicted log2(time) per slot is the members'
// mean, and the cell takes the valid slot with the smallest.  Averaging
// independently seeded networks generalises to untimed precisions better
// than any one of them.
__global__ void grid_infer(const float *params, int members, const uint64_t *valid, uint8_t *table) {
  __shared__ float w[kParams];
  const int cells = 3 * kGridMaxLimbs * kGridCountBuckets * kGridExpBuckets;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  int eb = 0, cb = 0, nl = 1, op = 0;
  uint64_t vmask = 0;
  if (c < cells) {
    eb = c % kGridExpBuckets;
    cb = (c / kGridExpBuckets) % kGridCountBuckets;
    nl = (c / (kGridExpBuckets * kGridCountBuckets)) % kGridMaxLimbs + 1;
    op = c / (kGridExpBuckets * kGridCountBuckets * kGridMaxLimbs);
    vmask = valid[op * kGridMaxLimbs + nl - 1];
    if (op != xmpTunePowm && eb != 0) vmask = 0;
  }
  // the cell stands for counts in [2^cb, 2^(cb+1)) and exponents in [2^eb, 2^(eb+1)): use the geometric
  // middle.  Batches smaller than the smallest one the tuner times (2^6) leave the GPU just as idle as
  // that one, so they take its choice instead of an extrapolation below the data.
  float x[kIn];
  x[0] = (float)op - 1.0f;
  x[1] = (log2f(32.0f * nl) - 10.0f) / 4.0f;
  x[2] = (fmaxf((float)cb, (float)kSelectorMinCountLog2) + 0.5f - 13.0f) / 7.0f;
  x[3] = op == xmpTunePowm ? ((float)eb + 0.5f - 7.0f) / 7.0f : (0.0f - 7.0f) / 7.0f;
  float acc[kOut];
  for (int j = 0; j < kOut; j++) acc[j] = 0.0f;
  // every thread of the block takes part in the loads of every member, cell or not
  for (int m = 0; m < members; m++) {
    __syncthreads();
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) w[i] = params[(size_t)m * kParams + i];
    __syncthreads();
    if (vmask == 0) continue;
    float h1[kH], h2[kH];
    for (int j = 0; j < kH; j++) {
      float a = w[kOffB1 + j];
      for (int i = 0; i < kIn; i++) a = fmaf(x[i], w[kOffW1 + i * kH + j], a);
      h1[j] = fmaxf(a, 0.0f);
    }
    for (int j = 0; j < kH; j++) {
      float a = w[kOffB2 + j];
      for (int i = 0; i < kH; i++) a = fmaf(h1[i], w[kOffW2 + i * kH + j], a);
      h2[j] = fmaxf(a, 0.0f);
    }
    for (int j = 0; j < kOut; j++) {
      if (!((vmask >> j) & 1ull)) continue;
      float a = w[kOffB3 + j];
      for (int i = 0; i < kH; i++) a = fmaf(h2[i], w[kOffW3 + i * kOut + j], a);
      acc[j] += a;
    }
  }
  if (c >= cells) return;
  int best = 0xff;
  float best_v = 1e30f;
  for (int j = 0; j < kOut; j++) {
    if (!((vmask >> j) & 1ull)) continue;
    if (acc[j] < best_v) {
      best_v = acc[j];
      best = j;
    }
  }
  table[c] = (uint8_t)best;
}

// Device buffers for one forward/backward pass over n samples.
struct Net {
  xmpHandle_t h;
  int n = 0;
  float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;
  float *x = nullptr, *h1 = nullptr, *h2 = nullptr, *y = nullptr, *t = nullptr, *mask = nullptr;
  float *dy = nullptr, *dh2 = nullptr, *dh1 = nullptr, *loss = nullptr;
  std::vector<void *> owned;
  float inv_count = 0.0f;

  explicit Net(xmpHandle_t hh) : h(hh) {}
  ~Net() {
    cudaStreamSynchronize(h->stream);
    for (void *p : owned) h->df(p);
  }
  float *alloc(size_t count) {
    void *p = h->da(count * sizeof(float));
    if (p) owned.push_back(p);
    return (float *)p;
  }
  xmpError_t setup(const xmpTuneShape_t *shapes, const float *ms, int nn) {
    n = nn;
    params = alloc(kParams);
    grads = alloc(kParams);
    m = alloc(kParams);
    v = alloc(kParams);
    x = alloc((size_t)n * kIn);
    h1 = alloc((size_t)n * kH);
    h2 = alloc((size_t)n * kH);
    y = alloc((size_t)n * kOut);
    t = alloc((size_t)n * kOut);
    mask = alloc((size_t)n * kOut);
    dy = alloc((size_t)n * kOut);
    dh2 = alloc((size_t)n * kH);
    dh1 = alloc((size_t)n * kH);
    loss = alloc(1);
    if (owned.size() != 14) return xmpErrorInvalidCudaMalloc;
    std::vector<float> hx((size_t)n * kIn), ht((size_t)n * kOut, 0.0f), hm((size_t)n * kOut, 0.0f);
    size_t valid = 0;
    for (int b = 0; b < n; b++) {
      features(shapes[b], &hx[(size_t)b * kIn]);
      if (ms)
        for (int j = 0; j < kOut; j++) {
          float v = ms[(size_t)b * kOut + j];
          if (v > 0.0f && isfinite(v)) {
            ht[(size_t)b * kOut + j] = log2f(v);
            hm[(size_t)b * kOut + j] = 1.0f;
            valid++;
          }
        }
    }
    inv_count = valid ? 1.0f / (float)valid : 0.0f;
    cudaMemcpyAsync(x, hx.data(), hx.size() * 4, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(t, ht.data(), ht.size() * 4, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(mask, hm.data(), hm.size() * 4, cudaMemcpyHostToDevice, h->stream);
    cudaMemsetAsync(m, 0, kParams * 4, h->stream);
    cudaMemsetAsync(v, 0, kParams * 4, h->stream);
    return check_cuda();
  }
  void forward() {
    cudaStream_t s = h->stream;
    dense_fwd<<<grid_for((uint64_t)n * kH, 128), 128, 0, s>>>(x, kIn, params + kOffW1, params + kOffB1, h1, kH, n, 1);
    dense_fwd<<<grid_for((uint64_t)n * kH, 128), 128, 0, s>>>(h1, kH, params + kOffW2, params + kOffB2, h2, kH, n, 1);
    dense_fwd<<<grid_for((uint64_t)n * kOut, 128), 128, 0, s>>>(h2, kH, params + kOffW3, params + kOffB3, y, kOut, n,
                                                                 0);
  }
  void backward() {
    cudaStream_t s = h->stream;
    cudaMemsetAsync(loss, 0, 4, s);
    mse_grad<<<grid_for((uint64_t)n * kOut, 128), 128, 0, s>>>(y, t, mask, inv_count, n * kOut, dy, loss);
    dense_bwd_w<<<grid_for(kH * kOut + kOut, 128), 128, 0, s>>>(h2, kH, dy, kOut, n, grads + kOffW3, grads + kOffB3);
    dense_bwd_in<<<grid_for((uint64_t)n * kH, 128), 128, 0, s>>>(dy, kOut, params + kOffW3, h2, kH, n, dh2);
    dense_bwd_w<<<grid_for(kH * kH + kH, 128), 128, 0, s>>>(h1, kH, dh2, kH, n, grads + kOffW2, grads + kOffB2);
    dense_bwd_in<<<grid_for((uint64_t)n * kH, 128), 128, 0, s>>>(dh2, kH, params + kOffW2, h1, kH, n, dh1);
    dense_bwd_w<<<grid_for(kIn * kH + kH, 128), 128, 0, s>>>(x, kIn, dh1, kH, n, grads + kOffW1, grads + kOffB1);
  }
};

// He-uniform initial weights, zero biases, from a splitmix64 stream.
static void init_params(float *p, uint64_t seed) {
  uint64_t s = seed;
  auto uni = [&]() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (float)((z >> 11) * (1.0 / 9007199254740992.0)) * 2.0f - 1.0f;
  };
  memset(p, 0, sizeof(float) * kParams);
  for (int i = 0; i < kIn * kH; i++) p[kOffW1 + i] = uni() * sqrtf(6.0f / kIn);
  for (int i = 0; i < kH * kH; i++) p[kOffW2 + i] = uni() * sqrtf(6.0f / kH);
  for (int i = 0; i < kH * kOut; i++) p[kOffW3 + i] = uni() * sqrtf(6.0f / kH);
  for (int j = 0; j < kOut; j++) p[kOffB3 + j] = 0.0f;
}

// The selector trained on this library's own B200 timings, compiled in by
// the build (xmp_b200/tuning/b200_selector.f32 as exact hex-float literals):
// every new handle loads it, the way the reference's kernels read their
// compiled-in tune tables.
#if __has_include("default_selector.inc")
#include "default_selector.inc"
#endif

const float *default_selector_params(int *members) {
#ifdef XMPB_DEFAULT_SELECTOR_COUNT
  static_assert(XMPB_DEFAULT_SELECTOR_COUNT % kParams == 0, "embedded selector has the wrong shape");
  *members = XMPB_DEFAULT_SELECTOR_COUNT / kParams;
  return kDefaultSelector;
#else
  *members = 0;
  return nullptr;
#endif
}

xmpError_t selector_fill_table(xmpHandle_t h, const float *params, int members, std::vector<uint8_t> *table) {
  const size_t cells = (size_t)3 * kGridMaxLimbs * kGridCountBuckets * kGridExpBuckets;
  std::vector<uint64_t> valid((size_t)3 * kGridMaxLimbs, 0);
  for (int op = 0; op < 3; op++)
    for (int nl = 1; nl <= kGridMaxLimbs; nl++) {
      uint64_t mk = 0;
      for (int s = 0; s < kCand; s++) {
        bool ok;
        if (op == xmpTunePowm) {
          PowmConfig c;
          ok = powm_candidate(nl, s, &c);
        } else {
          ElemConfig c;
          ok = elem_candidate(op, nl, s, &c);
        }
        if (ok) mk |= 1ull << s;
      }
      valid[(size_t)op * kGridMaxLimbs + nl - 1] = mk;
    }
  float *dp = (float *)h->da((size_t)members * kParams * 4);
  uint64_t *dv = (uint64_t *)h->da(valid.size() * 8);
  uint8_t *dt = (uint8_t *)h->da(cells);
  xmpError_t e = xmpErrorSuccess;
  if (!dp || !dv || !dt) {
    e = xmpErrorInvalidCudaMalloc;
  } else {
    cudaMemcpyAsync(dp, params, (size_t)members * kParams * 4, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(dv, valid.data(), valid.size() * 8, cudaMemcpyHostToDevice, h->stream);
    grid_infer<<<grid_for(cells, 128), 128, 0, h->stream>>>(dp, members, dv, dt);
    table->resize(cells);
    cudaMemcpyAsync(table->data(), dt, cells, cudaMemcpyDeviceToHost, h->stream);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) e = xmpErrorCuda;
  }
  if (dp) h->df(dp);
  if (dv) h->df(dv);
  if (dt) h->df(dt);
  if (e != xmpErrorSuccess) return e;
  return check_cuda();
}

}  // namespace xmpb

extern "C" {

xmpError_t XMPAPI xmpSelectorTrain(xmpHandle_t h, const xmpTuneShape_t *shapes, const float *ms, int32_t n,
                                   int32_t epochs, float lr, uint64_t seed, int32_t init_from_params, float *params,
                                   float *final_loss) {
  if (!h || !shapes || !ms || n <= 0 || epochs < 0 || !params) return xmpErrorInvalidParameter;
  DeviceGuard guard(h->device);
  Net net(h);
  xmpError_t e = net.setup(shapes, ms, n);
  if (e != xmpErrorSuccess) return e;
  std::vector<float> p0(kParams);
  if (init_from_params)
    memcpy(p0.data(), params, kParams * 4);
  else
    init_params(p0.data(), seed);
  cudaMemcpyAsync(net.params, p0.data(), kParams * 4, cudaMemcpyHostToDevice, h->stream);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float c1 = 1.0f, c2 = 1.0f;
  for (int ep = 0; ep < epochs; ep++) {
    net.forward();
    net.backward();
    c1 *= b1;
    c2 *= b2;
    adam_step<<<grid_for(kParams, 128), 128, 0, h->stream>>>(net.params, net.grads, net.m, net.v, kParams, lr, b1, b2,
                                                             eps, 1.0f - c1, 1.0f - c2);
  }
  net.forward();
  net.backward();
  float loss = 0.0f;
  cudaMemcpyAsync(params, net.params, kParams * 4, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(&loss, net.loss, 4, cudaMemcpyDeviceToHost, h->stream);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return xmpErrorCuda;
  if (final_loss) *final_loss = loss;
  return check_cuda();
}

xmpError_t XMPAPI xmpSelectorGradients(xmpHandle_t h, const float *params, const xmpTuneShape_t *shapes,
                                       const float *ms, int32_t n, float *loss, float *grads) {
  if (!h || !params || !shapes || !ms || n <= 0 || !grads) return xmpErrorInvalidParameter;
  DeviceGuard guard(h->device);
  Net net(h);
  xmpError_t e = net.setup(shapes, ms, n);
  if (e != xmpErrorSuccess) return e;
  cudaMemcpyAsync(net.params, params, kParams * 4, cudaMemcpyHostToDevice, h->stream);
  net.forward();
  net.backward();
  float l = 0.0f;
  cudaMemcpyAsync(grads, net.grads, kParams * 4, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(&l, net.loss, 4, cudaMemcpyDeviceToHost, h->stream);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return xmpErrorCuda;
  if (loss) *loss = l;
  return check_cuda();
}

xmpError_t XMPAPI xmpSelectorPredict(xmpHandle_t h, const float *params, const xmpTuneShape_t *shapes, int32_t n,
                                     float *pred) {
  if (!h || !params || !shapes || n <= 0 || !pred) return xmpErrorInvalidParameter;
  DeviceGuard guard(h->device);
  Net net(h);
  xmpError_t e = net.setup(shapes, nullptr, n);
  if (e != xmpErrorSuccess) return e;
  cudaMemcpyAsync(net.params, params, kParams * 4, cudaMemcpyHostToDevice, h->stream);
  net.forward();
  cudaMemcpyAsync(pred, net.y, (size_t)n * kOut * 4, cudaMemcpyDeviceToHost, h->stream);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return xmpErrorCuda;
  return check_cuda();
}

}  // extern "C"
