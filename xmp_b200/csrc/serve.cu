// Continuous-batching modular-exponentiation server (no counterpart in the
// reference, whose xmpIntegersPowm is one synchronous batch per call,
// src/powm.cu:250-307).
//
// Keys (odd moduli) are registered per precision class and kept on the device
// with their Montgomery constant R^2 mod m (computed once by r2_kernel; the
// per-key n' = -m^-1 mod 2^32 is two Newton steps inside the kernel).
// Requests carry 1..max_wave_ops exponentiations under one key.  A scheduler
// thread turns pending requests into launch waves: the ops are copied into
// pinned staging, one copy moves them to the device, a staging kernel
// interleaves them into a contiguous range of op slots, the powm kernel runs
// on those slots with the key's constants gathered through a per-slot key
// index, and the results come back with one copy.  Request exponents are
// treated as secret: the kernel is the constant-schedule form (a fixed window
// over the exponent's whole precision, the same multiplications for every
// exponent value).  While the GPU is nearly idle, small waves of up to 2048
// bits run one op per CTA (cta.cuh); everything else runs on the lane
// kernels.  Waves go out on a pool of
// streams, so requests that arrive while others are on the GPU start as soon
// as slots are free and run alongside them.  The slot rings (one per class,
// sized from the HBM budget) are the admission control: a request waits on
// the host while its class has no room.  Every wait is on the host (event
// polls, condition variables with timeouts); no kernel waits on anything.
#include "powm.h"
#include "serve_sched.h"
#include "tune.h"
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

using namespace xmpb;

namespace xmpb {
namespace serve {

static int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// rows (count x nlimbs words, compact) -> interleaved elements dst_first.. of
// an array with `stride` elements per limb group; z selects one of two pairs.
__global__ void rows_to_slots(const uint32_t *__restrict__ rows0, uint32_t *__restrict__ dst0,
                              const uint32_t *__restrict__ rows1, uint32_t *__restrict__ dst1, uint32_t nlimbs,
                              uint32_t stride, uint32_t dst_first, uint32_t count) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const uint32_t g = blockIdx.y;
  const uint32_t *row = (blockIdx.z ? rows1 : rows0) + (size_t)k * nlimbs;
  uint32_t *dst = blockIdx.z ? dst1 : dst0;
  const uint32_t j = g * 4;
  uint4 v;
  if ((nlimbs & 3) == 0) {
    v = __ldg(reinterpret_cast<const uint4 *>(row) + g);
  } else {
    v.x = j < nlimbs ? row[j] : 0;
    v.y = j + 1 < nlimbs ? row[j + 1] : 0;
    v.z = j + 2 < nlimbs ? row[j + 2] : 0;
    v.w = j + 3 < nlimbs ? row[j + 3] : 0;
  }
  reinterpret_cast<uint4 *>(dst)[(size_t)g * stride + dst_first + k] = v;
}

// interleaved elements src_first.. -> compact rows
__global__ void slots_to_rows(const uint32_t *__restrict__ src, uint32_t nlimbs, uint32_t stride, uint32_t src_first,
                              uint32_t *__restrict__ rows, uint32_t count) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const uint32_t g = blockIdx.y;
  const uint4 v = __ldg(reinterpret_cast<const uint4 *>(src) + (size_t)g * stride + src_first + k);
  uint32_t *row = rows + (size_t)k * nlimbs;
  const uint32_t j = g * 4;
  if ((nlimbs & 3) == 0) {
    reinterpret_cast<uint4 *>(row)[g] = v;
  } else {
    if (j < nlimbs) row[j] = v.x;
    if (j + 1 < nlimbs) row[j + 1] = v.y;
    if (j + 2 < nlimbs) row[j + 2] = v.z;
    if (j + 3 < nlimbs) row[j + 3] = v.w;
  }
}

enum ReqState : int { kPending = 0, kRunning = 1, kDone = 2, kFailed = 3 };

struct Req {
  uint64_t id = 0;
  uint32_t cls = 0, key = 0, nops = 0;
  const uint32_t *base = nullptr, *exp = nullptr;
  uint32_t *out = nullptr;
  int64_t t_arrival = 0, t_enqueue = 0, t_done = 0;
  int state = kPending;
};

struct Wave {
  uint32_t first = 0, taken = 0, ops = 0;
  int stream = 0;
  cudaEvent_t ev = nullptr;
  std::vector<Req *> reqs;
  std::vector<uint32_t> offs;
  bool finished = false;
};

constexpr int kBuckets = 20;  // waves of 2^b .. 2^(b+1)-1 ops

struct Class {
  uint32_t precision = 0, n = 0, ngroups = 0, cap = 0;
  // keys
  uint32_t kcap = 0, nkeys = 0;
  uint32_t *key_mod = nullptr, *key_r2 = nullptr;
  std::vector<uint32_t> host_mod;  // compact rows, for the synchronous baseline
  // op slots
  uint32_t slots = 0;
  SlotRing ring;
  uint32_t *slot_base = nullptr, *slot_exp = nullptr, *slot_out = nullptr, *slot_key = nullptr;
  uint32_t *rows_base = nullptr, *rows_exp = nullptr, *rows_out = nullptr;  // device compact staging
  uint32_t *pin_base = nullptr, *pin_exp = nullptr, *pin_out = nullptr, *pin_key = nullptr;
  uint32_t *table = nullptr;
  size_t table_words = 0;  // per slot
  PowmConfig cfg[kBuckets];
  const PowmKernelEntry *entry[kBuckets] = {};
  bool cta[kBuckets] = {};  // waves of this size run one op per CTA (cta_limbs-limb operands)
  uint32_t cta_limbs = 0;
  bool urgent = false;  // the largest precision: its waves bound the latency tail, so they get priority streams
  // scheduler-owned queues
  std::deque<Req *> pending;
  uint32_t pending_ops = 0;
  std::deque<Wave *> inflight;
  uint32_t inflight_ops = 0;
  bool stalled = false;
};

}  // namespace serve
}  // namespace xmpb

using namespace xmpb::serve;

struct _xmpServer_t {
  xmpHandle_t h = nullptr;
  int device = 0;
  xmpServerConfig_t cfg{};
  WavePolicy policy;
  std::vector<Class> classes;
  std::vector<std::pair<uint32_t, uint32_t>> keys;  // global key -> (class, key within class)
  std::vector<cudaStream_t> streams;
  std::vector<int> stream_waves;
  std::vector<bool> stream_high;  // created at the device's greatest stream priority
  int next_stream = 0;
  std::vector<cudaEvent_t> event_pool;
  cudaStream_t setup = nullptr;
  std::vector<void *> device_allocs;
  std::vector<void *> host_allocs;
  size_t device_bytes = 0;

  std::thread thread;
  std::mutex mu;                     // incoming, requests, states, error, stats
  std::mutex setup_mu;               // AddKeys
  std::condition_variable cv_work;   // scheduler wake-up
  std::condition_variable cv_done;   // request completion
  std::deque<Req *> incoming;
  std::unordered_map<uint64_t, Req *> requests;
  uint64_t next_id = 1;
  bool stop = false;
  xmpError_t error = xmpErrorSuccess;
  uint64_t outstanding = 0;  // submitted, not yet done
  xmpServerStats_t stats{};
};

namespace xmpb {
namespace serve {

static int bucket_of(uint32_t ops) {
  int b = 0;
  while (b + 1 < kBuckets && (1u << (b + 1)) <= ops) b++;
  return b;
}

static void *dev_alloc(xmpServer_t s, size_t bytes) {
  void *p = s->h->da(bytes);
  if (p) {
    s->device_allocs.push_back(p);
    s->device_bytes += bytes;
  }
  return p;
}

static void *host_alloc(xmpServer_t s, size_t bytes) {
  void *p = nullptr;
  if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) != cudaSuccess) return nullptr;
  s->host_allocs.push_back(p);
  return p;
}

static void free_all(xmpServer_t s) {
  for (void *p : s->device_allocs) s->h->df(p);
  for (void *p : s->host_allocs) cudaFreeHost(p);
  for (auto st : s->streams) cudaStreamDestroy(st);
  for (auto ev : s->event_pool) cudaEventDestroy(ev);
  if (s->setup) cudaStreamDestroy(s->setup);
  for (auto &c : s->classes)
    for (Wave *w : c.inflight) {
      if (w->ev) cudaEventDestroy(w->ev);
      delete w;
    }
  for (auto &kv : s->requests) delete kv.second;
}

// Configuration per wave-size bucket: the tuner's choice (an exact tuned entry
// or the learned selector) when it runs at the class's Montgomery radix, else
// the built-in heuristic restricted to that radix.
static void choose_configs(xmpServer_t s, Class &c) {
  for (int b = 0; b < kBuckets; b++) {
    const uint32_t ops = 1u << b;
    PowmConfig cfg;
    bool ok = tuner_lookup_powm(s->h, c.n, c.precision, ops, &cfg) && cfg.dist == kDistLanes &&
              (uint32_t)(cfg.tpi * cfg.limbs) == c.cap && powm_find(cfg.tpi, cfg.limbs);
    if (!ok) cfg = powm_default_config(c.n, c.precision, ops, xmpAlgorithmDefault, s->h->sm_count, c.cap);
    // requests carry private exponents: the constant-schedule kernel, fixed window over the full precision
    cfg.window = window_for_bits(c.precision, false);
    c.cfg[b] = cfg;
    c.entry[b] = powm_find(cfg.tpi, cfg.limbs);
    // small waves on a quiet GPU: one op per CTA (its constant-schedule form), at a lone op's lowest
    // latency (one op: 3.6 vs 8.4 ms at 2048 bits, 9.2 vs 15.7 ms at 3072, 20.4 vs 30.0 ms at 4096)
    c.cta_limbs = powm_cta_limbs(c.n);
    c.cta[b] = c.cta_limbs != 0 && ops <= s->h->sm_count && powm_cta_preferred(c.n, ops, s->h->sm_count);
  }
}

static void fail_all(xmpServer_t s, xmpError_t e) {
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->error == xmpErrorSuccess) s->error = e;
  s->cv_done.notify_all();
}

static cudaEvent_t take_event(xmpServer_t s) {
  if (!s->event_pool.empty()) {
    cudaEvent_t e = s->event_pool.back();
    s->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  return e;
}

// `load`: the class's ops in flight with this wave (picks the lane kernel's bucket); `gpu_load`: all
// classes' ops in flight with this wave.  A wave runs one op per CTA only while the GPU is otherwise
// nearly idle: CTAs of a lone op are fast but share SMs poorly (measured: with one op per CTA for
// every wave of up to two ops per SM, a 70%-load mix of 2048-4096-bit requests had a 166 ms p99
// against 58 ms on the lane kernels alone).
static bool launch_wave(xmpServer_t s, Class &c, Wave *w, uint32_t load, uint32_t gpu_load) {
  const uint32_t n = c.n;
  const size_t row_bytes = (size_t)n * 4;
  for (size_t r = 0; r < w->reqs.size(); r++) {
    Req *q = w->reqs[r];
    const uint32_t at = w->first + w->offs[r];
    memcpy(c.pin_base + (size_t)at * n, q->base, q->nops * row_bytes);
    memcpy(c.pin_exp + (size_t)at * n, q->exp, q->nops * row_bytes);
    for (uint32_t j = 0; j < q->nops; j++) c.pin_key[at + j] = q->key;
  }
  // the stream with the fewest waves in flight (an idle one when there is one),
  // of the class's priority when one of those is as free, rotating among
  // equals so consecutive waves land on different streams
  const int ns = (int)s->streams.size();
  int si = -1;
  for (int j = 0; j < ns; j++) {
    const int k = (s->next_stream + j) % ns;
    if (si < 0 || s->stream_waves[k] < s->stream_waves[si] ||
        (s->stream_waves[k] == s->stream_waves[si] && s->stream_high[k] == c.urgent &&
         s->stream_high[si] != c.urgent))
      si = k;
  }
  s->next_stream = si + 1;
  cudaStream_t st = s->streams[si];
  w->stream = si;
  s->stream_waves[si]++;
  const size_t off = (size_t)w->first * n;
  const size_t bytes = (size_t)w->ops * row_bytes;
  if (cudaMemcpyAsync(c.rows_base + off, c.pin_base + off, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(c.rows_exp + off, c.pin_exp + off, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(c.slot_key + w->first, c.pin_key + w->first, (size_t)w->ops * 4, cudaMemcpyHostToDevice,
                      st) != cudaSuccess)
    return false;
  rows_to_slots<<<dim3(div_up(w->ops, 128), c.ngroups, 2), 128, 0, st>>>(
      c.rows_base + off, c.slot_base, c.rows_exp + off, c.slot_exp, n, c.slots, w->first, w->ops);
  const int b = bucket_of(load);
  const PowmConfig &cfg = c.cfg[b];
  PowmArgs a;
  a.base = ArrayView{c.slot_base, n, c.slots, c.slots, nullptr, 0};
  a.exp = ArrayView{c.slot_exp, n, c.slots, c.slots, nullptr, 0};
  a.mod = ArrayView{c.key_mod, n, c.kcap, c.kcap, c.slot_key, c.slots};
  a.r2 = ArrayView{c.key_r2, n, c.kcap, c.kcap, c.slot_key, c.slots};
  a.out = OutView{c.slot_out, n, c.slots, c.slots, nullptr};
  a.start = w->first;
  a.count = w->ops;
  a.window = cfg.window;
  a.table = c.table + (size_t)w->first * c.table_words;
  if (c.cta[b] && gpu_load <= s->h->sm_count) {
    if (!powm_cta_launch(c.cta_limbs, true, a, w->ops, st)) return false;
  } else {
    c.entry[b]->launch_ct(a, grid_for((uint64_t)w->ops * cfg.tpi, 128), st);
  }
  slots_to_rows<<<dim3(div_up(w->ops, 128), c.ngroups), 128, 0, st>>>(c.slot_out, n, c.slots, w->first,
                                                                         c.rows_out + off, w->ops);
  if (cudaMemcpyAsync(c.pin_out + off, c.rows_out + off, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return false;
  w->ev = take_event(s);
  if (!w->ev || cudaEventRecord(w->ev, st) != cudaSuccess) return false;
  return cudaGetLastError() == cudaSuccess;
}

// Completed waves: results to the callers' buffers, slots back to the ring.
static bool poll_completions(xmpServer_t s, bool *progress) {
  for (auto &c : s->classes) {
    for (Wave *w : c.inflight) {
      if (w->finished) continue;
      cudaError_t q = cudaEventQuery(w->ev);
      if (q == cudaErrorNotReady) continue;
      if (q != cudaSuccess) return false;
      const int64_t t = now_ns();
      for (size_t r = 0; r < w->reqs.size(); r++) {
        Req *rq = w->reqs[r];
        memcpy(rq->out, c.pin_out + (size_t)(w->first + w->offs[r]) * c.n, (size_t)rq->nops * c.n * 4);
      }
      {
        std::lock_guard<std::mutex> lk(s->mu);
        for (Req *rq : w->reqs) {
          rq->t_done = t;
          rq->state = kDone;
          s->stats.requests_completed++;
          s->stats.ops_completed += rq->nops;
          s->outstanding--;
        }
      }
      s->cv_done.notify_all();
      w->finished = true;
      s->stream_waves[w->stream]--;
      *progress = true;
    }
    while (!c.inflight.empty() && c.inflight.front()->finished) {
      Wave *w = c.inflight.front();
      c.inflight.pop_front();
      c.ring.release(w->taken);
      c.inflight_ops -= w->ops;
      s->event_pool.push_back(w->ev);
      delete w;
    }
  }
  return true;
}

// Forms and launches waves while a stream is idle, oldest pending request
// first across classes.  A wave's configuration follows the class's load (its
// ops plus those already in flight): lone requests get the lowest-latency
// kernel, and as the GPU fills the choice moves to the highest-throughput one.
static bool launch_ready(xmpServer_t s, bool *progress) {
  int idle = 0;
  for (int w : s->stream_waves) idle += w == 0;
  std::vector<bool> blocked(s->classes.size(), false);
  while (true) {
    int best = -1;
    for (size_t i = 0; i < s->classes.size(); i++) {
      const Class &c = s->classes[i];
      if (blocked[i] || !s->policy.should_launch(c.pending_ops, (uint32_t)idle)) continue;
      if (best < 0 || c.pending.front()->t_enqueue < s->classes[best].pending.front()->t_enqueue) best = (int)i;
    }
    if (best < 0) break;
    Class &c = s->classes[best];
    const uint32_t limit = std::min(s->policy.max_wave_ops, c.ring.largest_free());
    uint32_t take = 0;
    size_t k = 0;
    while (k < c.pending.size() && take + c.pending[k]->nops <= limit) take += c.pending[k++]->nops;
    if (k == 0) {
      // no op slots for the oldest request of this class: it waits for completions
      if (!c.stalled) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stats.admission_stalls++;
      }
      c.stalled = true;
      blocked[best] = true;
      continue;
    }
    c.stalled = false;
    Wave *w = new Wave();
    if (!c.ring.alloc(take, &w->first, &w->taken)) {
      delete w;
      return false;  // cannot happen: take <= largest_free
    }
    w->ops = take;
    uint32_t off = 0;
    for (size_t j = 0; j < k; j++) {
      Req *r = c.pending.front();
      c.pending.pop_front();
      c.pending_ops -= r->nops;
      r->state = kRunning;
      w->reqs.push_back(r);
      w->offs.push_back(off);
      off += r->nops;
    }
    const uint32_t load = c.inflight_ops + take;
    uint32_t gpu_load = take;
    for (const auto &cc : s->classes) gpu_load += cc.inflight_ops;
    c.inflight.push_back(w);
    c.inflight_ops += take;
    if (!launch_wave(s, c, w, load, gpu_load)) return false;
    idle--;
    *progress = true;
    std::lock_guard<std::mutex> lk(s->mu);
    s->stats.waves++;
  }
  uint32_t total_inflight = 0;
  for (auto &c : s->classes) total_inflight += c.inflight_ops;
  std::lock_guard<std::mutex> lk(s->mu);
  s->stats.max_inflight_ops = std::max(s->stats.max_inflight_ops, total_inflight);
  return true;
}

static void scheduler(xmpServer_t s) {
  cudaSetDevice(s->device);
  std::vector<Req *> moved;
  bool failed = false;
  while (true) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      moved.assign(s->incoming.begin(), s->incoming.end());
      s->incoming.clear();
      if (s->stop) break;
    }
    for (Req *r : moved) {
      Class &c = s->classes[r->cls];
      c.pending.push_back(r);
      c.pending_ops += r->nops;
    }
    if (failed) {
      // after a CUDA failure nothing more is launched; pending requests fail
      std::lock_guard<std::mutex> lk(s->mu);
      for (auto &c : s->classes) {
        for (Req *r : c.pending) {
          r->state = kFailed;
          s->outstanding--;
        }
        c.pending.clear();
        c.pending_ops = 0;
      }
      s->cv_done.notify_all();
    }
    bool progress = false;
    if (!failed && !(poll_completions(s, &progress) && launch_ready(s, &progress))) {
      failed = true;
      fail_all(s, xmpErrorCuda);
      continue;
    }
    if (!progress) {
      bool busy = false;
      for (auto &c : s->classes) busy |= !c.inflight.empty() || !c.pending.empty();
      std::unique_lock<std::mutex> lk(s->mu);
      if (s->incoming.empty() && !s->stop) {
        // short sleeps while work is on the device (event polling), longer when idle
        s->cv_work.wait_for(lk, std::chrono::microseconds(busy ? 20 : 2000));
      }
    }
  }
  // shutdown: let the device finish what was launched
  for (auto &c : s->classes)
    for (Wave *w : c.inflight)
      if (!w->finished && w->ev) cudaEventSynchronize(w->ev);
  std::lock_guard<std::mutex> lk(s->mu);
  for (auto &c : s->classes) {
    for (Req *r : c.pending) r->state = kFailed;
    for (Wave *w : c.inflight)
      for (Req *r : w->reqs)
        if (r->state != kDone) r->state = kFailed;
  }
  s->cv_done.notify_all();
}

static int find_class(xmpServer_t s, uint32_t precision) {
  for (size_t i = 0; i < s->classes.size(); i++)
    if (s->classes[i].precision == precision) return (int)i;
  return -1;
}

}  // namespace serve
}  // namespace xmpb

extern "C" {

xmpError_t XMPAPI xmpServerCreate(xmpHandle_t h, const uint32_t *precisions, uint32_t n_classes,
                                  const xmpServerConfig_t *config, xmpServer_t *out) {
  if (!h || !out || !precisions || n_classes == 0 || n_classes > 16) return xmpErrorInvalidParameter;
  *out = nullptr;
  DeviceGuard guard(h->device);
  xmpServer_t s = new _xmpServer_t();
  s->h = h;
  s->device = h->device;
  if (config) s->cfg = *config;
  xmpServerConfig_t &cf = s->cfg;
  if (cf.hbm_budget == 0) cf.hbm_budget = (size_t)8 << 30;
  if (cf.max_wave_ops == 0) cf.max_wave_ops = 4096;
  if (cf.streams == 0) cf.streams = 32;
  if (cf.max_keys == 0) cf.max_keys = 4096;
  if (cf.max_slots == 0) cf.max_slots = 1u << 18;
  cf.max_wave_ops = std::min(cf.max_wave_ops, 1u << 19);
  s->policy.max_wave_ops = cf.max_wave_ops;
  auto fail = [&](xmpError_t e) {
    free_all(s);
    delete s;
    return e;
  };
  const uint32_t granule = 128;
  // ---- classes: radix, configurations, per-slot footprint ----
  s->classes.resize(n_classes);
  size_t key_bytes = 0, per_slot_total = 0;
  std::vector<size_t> per_slot(n_classes);
  for (uint32_t i = 0; i < n_classes; i++) {
    Class &c = s->classes[i];
    if (precisions[i] == 0 || precisions[i] % 32 != 0) return fail(xmpErrorInvalidPrecision);
    for (uint32_t j = 0; j < i; j++)
      if (precisions[j] == precisions[i]) return fail(xmpErrorInvalidParameter);
    c.precision = precisions[i];
    c.n = precisions[i] / 32;
    c.ngroups = div_up(c.n, 4);
    // Montgomery radix: the smallest register-kernel capacity that holds n limbs
    uint32_t cap = 0;
    for (const auto &e : powm_registry()) {
      uint32_t k = (uint32_t)e.tpi * e.limbs;
      if (k >= c.n && (cap == 0 || k < cap)) cap = k;
    }
    if (cap == 0) return fail(xmpErrorUnsupported);
    c.cap = cap;
    choose_configs(s, c);
    size_t tw = 0;
    for (int b = 0; b < kBuckets; b++) {
      if (!c.entry[b]) return fail(xmpErrorUnsupported);
      tw = std::max(tw, (size_t)cap * powm_table_entries(c.cfg[b].window, false));
    }
    c.table_words = tw;
    c.kcap = round_up(cf.max_keys, 32);
    key_bytes += 2 * (size_t)c.ngroups * 16 * c.kcap;
    // interleaved base/exp/out + key index + compact base/exp/out + window table
    per_slot[i] = 3 * (size_t)c.ngroups * 16 + 4 + 3 * (size_t)c.n * 4 + tw * 4;
    per_slot_total += per_slot[i];
  }
  if (cf.hbm_budget <= key_bytes) return fail(xmpErrorIncreaseScratchLimit);
  // equal slot counts per class, within the budget
  uint64_t slots = (cf.hbm_budget - key_bytes) / per_slot_total;
  slots = std::min<uint64_t>(slots, cf.max_slots) / granule * granule;
  if (slots < granule) return fail(xmpErrorIncreaseScratchLimit);
  for (uint32_t i = 0; i < n_classes; i++) {
    Class &c = s->classes[i];
    c.slots = (uint32_t)slots;
    c.ring = SlotRing(c.slots, granule);
    const size_t gbytes = (size_t)c.ngroups * 16;
    c.key_mod = (uint32_t *)dev_alloc(s, gbytes * c.kcap);
    c.key_r2 = (uint32_t *)dev_alloc(s, gbytes * c.kcap);
    c.slot_base = (uint32_t *)dev_alloc(s, gbytes * c.slots);
    c.slot_exp = (uint32_t *)dev_alloc(s, gbytes * c.slots);
    c.slot_out = (uint32_t *)dev_alloc(s, gbytes * c.slots);
    c.slot_key = (uint32_t *)dev_alloc(s, (size_t)4 * c.slots);
    c.rows_base = (uint32_t *)dev_alloc(s, (size_t)c.n * 4 * c.slots);
    c.rows_exp = (uint32_t *)dev_alloc(s, (size_t)c.n * 4 * c.slots);
    c.rows_out = (uint32_t *)dev_alloc(s, (size_t)c.n * 4 * c.slots);
    c.table = (uint32_t *)dev_alloc(s, c.table_words * 4 * c.slots);
    if (!c.key_mod || !c.key_r2 || !c.slot_base || !c.slot_exp || !c.slot_out || !c.slot_key || !c.rows_base ||
        !c.rows_exp || !c.rows_out || !c.table)
      return fail(xmpErrorInvalidCudaMalloc);
    if (cudaMemset(c.key_mod, 0, gbytes * c.kcap) != cudaSuccess ||
        cudaMemset(c.key_r2, 0, gbytes * c.kcap) != cudaSuccess)
      return fail(xmpErrorCuda);
    c.pin_base = (uint32_t *)host_alloc(s, (size_t)c.n * 4 * c.slots);
    c.pin_exp = (uint32_t *)host_alloc(s, (size_t)c.n * 4 * c.slots);
    c.pin_out = (uint32_t *)host_alloc(s, (size_t)c.n * 4 * c.slots);
    c.pin_key = (uint32_t *)host_alloc(s, (size_t)4 * c.slots);
    if (!c.pin_base || !c.pin_exp || !c.pin_out || !c.pin_key) return fail(xmpErrorInvalidCudaMalloc);
  }
  // ---- streams and the scheduler ----
  if (cudaStreamCreateWithFlags(&s->setup, cudaStreamNonBlocking) != cudaSuccess) return fail(xmpErrorCuda);
  // Half of the streams at the device's greatest priority: the block scheduler
  // gives their CTAs the SMs first, and the largest class (whose operations
  // take longest and so set the latency tail) launches there by preference.
  int prio_low = 0, prio_high = 0;
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  uint32_t biggest = 0;
  for (uint32_t i = 1; i < n_classes; i++)
    if (s->classes[i].precision > s->classes[biggest].precision) biggest = i;
  if (n_classes > 1) s->classes[biggest].urgent = true;
  for (uint32_t i = 0; i < cf.streams; i++) {
    cudaStream_t st;
    const bool high = n_classes > 1 && i % 2 == 0;
    if (cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, high ? prio_high : prio_low) != cudaSuccess)
      return fail(xmpErrorCuda);
    s->streams.push_back(st);
    s->stream_waves.push_back(0);
    s->stream_high.push_back(high);
  }
  s->stats.classes = n_classes;
  s->stats.device_bytes = s->device_bytes;
  s->thread = std::thread(scheduler, s);
  *out = s;
  return xmpErrorSuccess;
}

xmpError_t XMPAPI xmpServerDestroy(xmpServer_t s) {
  if (!s) return xmpErrorInvalidParameter;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->thread.joinable()) s->thread.join();
  DeviceGuard guard(s->device);
  free_all(s);
  delete s;
  return xmpErrorSuccess;
}

xmpError_t XMPAPI xmpServerAddKeys(xmpServer_t s, uint32_t precision, const uint32_t *moduli, uint32_t count,
                                   uint32_t *first_key) {
  if (!s || !moduli || !first_key) return xmpErrorInvalidParameter;
  const int ci = find_class(s, precision);
  if (ci < 0) return xmpErrorInvalidPrecision;
  if (count == 0) return xmpErrorInvalidCount;
  Class &c = s->classes[ci];
  for (uint32_t k = 0; k < count; k++)
    if ((moduli[(size_t)k * c.n] & 1u) == 0) return xmpErrorInvalidParameter;  // Montgomery needs odd moduli
  std::lock_guard<std::mutex> setup(s->setup_mu);
  if (c.nkeys + (uint64_t)count > c.kcap) return xmpErrorInvalidCount;
  DeviceGuard guard(s->device);
  const size_t bytes = (size_t)count * c.n * 4;
  uint32_t *rows = (uint32_t *)s->h->da(bytes);
  if (!rows) return xmpErrorInvalidCudaMalloc;
  xmpError_t e = xmpErrorSuccess;
  if (cudaMemcpyAsync(rows, moduli, bytes, cudaMemcpyHostToDevice, s->setup) != cudaSuccess) e = xmpErrorCuda;
  if (!e) {
    // one pair (grid.z = 1): the second pair is never read
    rows_to_slots<<<dim3(div_up(count, 128), c.ngroups, 1), 128, 0, s->setup>>>(rows, c.key_mod, nullptr, nullptr,
                                                                                 c.n, c.kcap, c.nkeys, count);
    PowmArgs a;
    a.mod = ArrayView{c.key_mod, c.n, c.kcap, c.kcap, nullptr, 0};
    a.out = OutView{c.key_r2, c.n, c.kcap, c.kcap, nullptr};
    a.start = c.nkeys;
    a.count = count;
    c.entry[0]->launch_r2(a, grid_for((uint64_t)count * c.cfg[0].tpi, 128), s->setup);
    if (cudaStreamSynchronize(s->setup) != cudaSuccess) e = xmpErrorCuda;
  }
  s->h->df(rows);
  if (e) return e;
  c.host_mod.insert(c.host_mod.end(), moduli, moduli + (size_t)count * c.n);
  std::lock_guard<std::mutex> lk(s->mu);
  *first_key = (uint32_t)s->keys.size();
  for (uint32_t k = 0; k < count; k++) s->keys.emplace_back((uint32_t)ci, c.nkeys + k);
  c.nkeys += count;
  return xmpErrorSuccess;
}

static xmpError_t make_request(xmpServer_t s, uint32_t key, uint32_t nops, const uint32_t *bases,
                               const uint32_t *exps, uint32_t *out, Req **rq) {
  if (!bases || !exps || !out) return xmpErrorInvalidParameter;
  if (key >= s->keys.size()) return xmpErrorInvalidParameter;
  const auto kc = s->keys[key];
  const Class &c = s->classes[kc.first];
  if (nops == 0 || nops > s->cfg.max_wave_ops || nops > c.slots) return xmpErrorInvalidCount;
  Req *r = new Req();
  r->cls = kc.first;
  r->key = kc.second;
  r->nops = nops;
  r->base = bases;
  r->exp = exps;
  r->out = out;
  *rq = r;
  return xmpErrorSuccess;
}

xmpError_t XMPAPI xmpServerSubmit(xmpServer_t s, uint32_t key, uint32_t nops, const uint32_t *bases,
                                  const uint32_t *exps, uint32_t *out, uint64_t *request) {
  if (!s || !request) return xmpErrorInvalidParameter;
  Req *r = nullptr;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->error) return s->error;
    xmpError_t e = make_request(s, key, nops, bases, exps, out, &r);
    if (e) return e;
    r->id = s->next_id++;
    r->t_arrival = r->t_enqueue = now_ns();
    s->requests[r->id] = r;
    s->incoming.push_back(r);
    s->outstanding++;
    s->stats.requests_submitted++;
    *request = r->id;
  }
  s->cv_work.notify_one();
  return xmpErrorSuccess;
}

xmpError_t XMPAPI xmpServerWait(xmpServer_t s, uint64_t request, uint32_t timeout_us, int32_t *done) {
  if (!s || !done) return xmpErrorInvalidParameter;
  *done = 0;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->requests.find(request);
  if (it == s->requests.end()) return xmpErrorInvalidParameter;
  Req *r = it->second;
  auto ready = [&] { return r->state == kDone || r->state == kFailed || s->error != xmpErrorSuccess; };
  if (timeout_us) s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), ready);
  if (r->state == kDone) {
    *done = 1;
    s->requests.erase(it);
    delete r;
    return xmpErrorSuccess;
  }
  if (r->state == kFailed || s->error) return s->error ? s->error : xmpErrorCuda;
  return xmpErrorSuccess;
}

xmpError_t XMPAPI xmpServerStats(xmpServer_t s, xmpServerStats_t *stats) {
  if (!s || !stats) return xmpErrorInvalidParameter;
  std::lock_guard<std::mutex> lk(s->mu);
  *stats = s->stats;
  return s->error;
}

xmpError_t XMPAPI xmpServerReplay(xmpServer_t s, uint32_t n, const uint32_t *keys, const uint32_t *nops,
                                  const uint64_t *arrival_ns, const uint32_t *const *bases,
                                  const uint32_t *const *exps, uint32_t *const *outs, int32_t mode,
                                  uint64_t *latency_ns, double *seconds) {
  if (!s || !keys || !nops || !arrival_ns || !bases || !exps || !outs || !latency_ns || !seconds ||
      (mode != 0 && mode != 1))
    return xmpErrorInvalidParameter;
  for (uint32_t i = 1; i < n; i++)
    if (arrival_ns[i] < arrival_ns[i - 1]) return xmpErrorInvalidParameter;
  std::vector<Req *> rs(n, nullptr);
  auto cleanup = [&]() {
    for (Req *r : rs) delete r;
  };
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->error) return s->error;
    if (s->outstanding) return xmpErrorInvalidParameter;  // replay needs an idle server
    for (uint32_t i = 0; i < n; i++) {
      xmpError_t e = make_request(s, keys[i], nops[i], bases[i], exps[i], outs[i], &rs[i]);
      if (e) {
        cleanup();
        return e;
      }
    }
  }
  auto wait_until = [](int64_t t) {
    while (true) {
      int64_t d = t - now_ns();
      if (d <= 0) return;
      if (d > 300000) std::this_thread::sleep_for(std::chrono::nanoseconds(d - 200000));
    }
  };
  xmpError_t err = xmpErrorSuccess;
  const int64_t t0 = now_ns() + 1000000;
  if (mode == 0) {
    for (uint32_t i = 0; i < n; i++) {
      Req *r = rs[i];
      r->t_arrival = t0 + (int64_t)arrival_ns[i];
      wait_until(r->t_arrival);
      {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = 0;
        r->t_enqueue = now_ns();
        s->incoming.push_back(r);
        s->outstanding++;
        s->stats.requests_submitted++;
      }
      s->cv_work.notify_one();
    }
    std::unique_lock<std::mutex> lk(s->mu);
    for (uint32_t i = 0; i < n; i++) {
      Req *r = rs[i];
      s->cv_done.wait(lk, [&] { return r->state == kDone || r->state == kFailed || s->error != xmpErrorSuccess; });
      if (r->state != kDone) {
        err = s->error ? s->error : xmpErrorCuda;
        break;
      }
    }
    if (err) {
      // requests still known to the scheduler must outlive it: keep them (leak) rather than free under it
      rs.clear();
      return err;
    }
  } else {
    // plain synchronous per-request launches through the public API
    xmpHandle_t h = s->h;
    std::vector<uint32_t> maxops(s->classes.size(), 0);
    for (Req *r : rs) maxops[r->cls] = std::max(maxops[r->cls], r->nops);
    std::vector<xmpIntegers_t> B(s->classes.size()), E(s->classes.size()), M(s->classes.size()),
        O(s->classes.size());
    for (size_t c = 0; c < s->classes.size() && !err; c++) {
      if (!maxops[c]) continue;
      const uint32_t p = s->classes[c].precision;
      if ((err = xmpIntegersCreate(h, &B[c], p, maxops[c])) || (err = xmpIntegersCreate(h, &E[c], p, maxops[c])) ||
          (err = xmpIntegersCreate(h, &M[c], p, 1)) || (err = xmpIntegersCreate(h, &O[c], p, maxops[c])))
        break;
    }
    for (uint32_t i = 0; i < n && !err; i++) {
      Req *r = rs[i];
      const Class &c = s->classes[r->cls];
      r->t_arrival = t0 + (int64_t)arrival_ns[i];
      wait_until(r->t_arrival);
      uint32_t words = 0;
      void *mrow = (void *)(c.host_mod.data() + (size_t)r->key * c.n);
      if ((err = xmpIntegersImport(h, B[r->cls], c.n, -1, 4, 0, 0, (void *)r->base, r->nops)) ||
          (err = xmpIntegersImport(h, E[r->cls], c.n, -1, 4, 0, 0, (void *)r->exp, r->nops)) ||
          (err = xmpIntegersImport(h, M[r->cls], c.n, -1, 4, 0, 0, mrow, 1)) ||
          (err = xmpIntegersPowm(h, O[r->cls], B[r->cls], E[r->cls], M[r->cls], r->nops)) ||
          (err = xmpIntegersExport(h, r->out, &words, -1, 4, 0, 0, O[r->cls], r->nops)))
        break;
      r->t_done = now_ns();
      r->state = kDone;
    }
    for (size_t c = 0; c < s->classes.size(); c++)
      for (xmpIntegers_t x : {B[c], E[c], M[c], O[c]})
        if (x) xmpIntegersDestroy(h, x);
    if (err) {
      cleanup();
      return err;
    }
  }
  int64_t last = t0;
  for (uint32_t i = 0; i < n; i++) {
    latency_ns[i] = (uint64_t)std::max<int64_t>(0, rs[i]->t_done - rs[i]->t_arrival);
    last = std::max(last, rs[i]->t_done);
  }
  *seconds = (double)(last - t0) * 1e-9;
  cleanup();
  return xmpErrorSuccess;
}

}  // extern "C"
