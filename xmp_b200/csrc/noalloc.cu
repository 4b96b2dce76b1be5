// xmpIntegersPowmNoAlloc: modular exponentiation for callers that must not
// allocate device memory.
//
// Who needs it: code where cudaMalloc/cudaFree are not affordable or not
// available -- a latency-critical serving path (cudaMalloc and cudaFree
// synchronise the device and stall every other stream), or a process whose
// device memory is owned by another allocator (a framework's caching pool or
// a fixed arena) that hands out only the operand buffers.  The regular
// xmpIntegersPowm grows the handle's scratch arena with the handle's
// allocator; this entry point instead keeps the exponentiation window tables
// in a fixed, file-scope device array, so the call itself allocates nothing.
//
// Scratch: kNoAllocScratchBytes (16 MiB) of `__device__` memory.  Every GPU
// that loads this library holds it until the process exits.  The array is
// shared by all calls on a device and keeps the last call's contents; the
// kernel writes every table slot before reading it, so nothing needs
// clearing.  Calls whose kernels overlap on the GPU (different streams, or
// several host threads) race on this array: serialise them.
//
// Device address: host code cannot pass the array's name to a kernel (on the
// host it is a stand-in, not a device address).  The address is looked up with
// cudaGetSymbolAddress while the device is current, on the first call in each
// CUDA context, and cached under that context's unique id (cuCtxGetId), so a
// context created after cudaDeviceReset, or another context a driver-API
// caller makes current, gets its own lookup rather than a stale address.
// Make the first call in a context before any stream capture.
#include "powm.h"
#include <cuda.h>
#include <mutex>

namespace xmpb {

constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocScratchBytes / 4];

// Driver entry points for the current context's id, fetched through the
// runtime (the library does not link libcuda).  Without them every call looks
// the address up again.
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

static bool current_context_id(unsigned long long *id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (CtxGetCurrentFn)f;
    f = nullptr;
    q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (CtxGetIdFn)f;
    cudaGetLastError();
  });
  if (!get_current || !get_id) return false;
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return false;
  return get_id(ctx, id) == CUDA_SUCCESS;
}

// Small cache: context id -> device address of g_noalloc_scratch in it.
constexpr int kNoAllocCacheEntries = 64;
struct NoAllocCacheEntry {
  unsigned long long ctx_id;
  void *addr;
};
static NoAllocCacheEntry g_noalloc_cache[kNoAllocCacheEntries];
static int g_noalloc_cache_next;
static std::mutex g_noalloc_mu;

static xmpError_t noalloc_scratch(void **addr) {
  unsigned long long id = 0;
  const bool have_id = current_context_id(&id);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (have_id) {
    for (const auto &e : g_noalloc_cache)
      if (e.addr && e.ctx_id == id) {
        *addr = e.addr;
        return xmpErrorSuccess;
      }
  }
  void *p = nullptr;
  cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (err != cudaSuccess || p == nullptr) {
    cudaGetLastError();
    return xmpErrorCuda;
  }
  // a context that did not exist before the lookup (the runtime made the primary one current) has an id now
  if (have_id || current_context_id(&id)) {
    g_noalloc_cache[g_noalloc_cache_next] = NoAllocCacheEntry{id, p};
    g_noalloc_cache_next = (g_noalloc_cache_next + 1) % kNoAllocCacheEntries;
  }
  *addr = p;
  return xmpErrorSuccess;
}

}  // namespace xmpb

using namespace xmpb;

extern "C" xmpError_t XMPAPI xmpIntegersPowmNoAlloc(cudaStream_t stream, uint32_t *out, const uint32_t *base,
                                                     const uint32_t *exp, const uint32_t *mod, uint32_t precision,
                                                     uint32_t exp_precision, uint32_t stride, uint32_t count) {
  if (count == 0) return xmpErrorSuccess;
  if (!out || !base || !exp || !mod) return xmpErrorInvalidParameter;
  if (stride < count) return xmpErrorInvalidCount;
  if (precision == 0 || precision % 32 != 0 || exp_precision == 0 || exp_precision % 32 != 0)
    return xmpErrorInvalidPrecision;
  const uintptr_t align = (uintptr_t)out | (uintptr_t)base | (uintptr_t)exp | (uintptr_t)mod;
  if (align % 16 != 0) return xmpErrorInvalidParameter;

  int device = 0, sms = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return xmpErrorInvalidDevice;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return xmpErrorCuda;

  const uint32_t nlimbs = precision / 32;
  // Register distributions only (up to 16,384 bits): the digit-serial kernel needs per-instance arrays
  // far larger than the fixed scratch.
  PowmConfig cfg = powm_default_config(nlimbs, exp_precision, count, xmpAlgorithmDefault, (uint32_t)sms);
  if (cfg.dist != kDistLanes || !powm_config_valid(cfg, nlimbs)) return xmpErrorUnsupported;
  // Shrink the window until the tables fit the fixed array; beyond that the batch is too large.
  while (powm_table_bytes(cfg, nlimbs, count) > kNoAllocScratchBytes && cfg.window > 1) cfg.window--;
  if (powm_table_bytes(cfg, nlimbs, count) > kNoAllocScratchBytes) return xmpErrorIncreaseScratchLimit;
  const PowmKernelEntry *k = powm_find(cfg.tpi, cfg.limbs);
  if (!k) return xmpErrorUnsupported;

  void *scratch = nullptr;
  xmpError_t e = noalloc_scratch(&scratch);
  if (e != xmpErrorSuccess) return e;

  PowmArgs a;
  a.base = ArrayView{const_cast<uint32_t *>(base), nlimbs, stride, count, nullptr, 0};
  a.exp = ArrayView{const_cast<uint32_t *>(exp), exp_precision / 32, stride, count, nullptr, 0};
  a.mod = ArrayView{const_cast<uint32_t *>(mod), nlimbs, stride, count, nullptr, 0};
  a.out = OutView{out, nlimbs, stride, count, nullptr};
  a.start = 0;
  a.count = count;
  a.window = (uint32_t)cfg.window;
  a.table = (uint32_t *)scratch;
  k->launch(a, grid_for((uint64_t)count * cfg.tpi, 128), stream);
  return cudaPeekAtLastError() == cudaSuccess ? xmpErrorSuccess : xmpErrorCuda;
}
