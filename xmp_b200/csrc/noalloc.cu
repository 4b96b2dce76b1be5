// xmpIntegersPowmNoAlloc: modular exponentiation for callers that must not
// allocate device memory.
//
// Who needs it: code that runs where cudaMalloc/cudaFree are not allowed or
// not affordable -- inside a CUDA stream capture (allocation is illegal
// while capturing), on a latency-critical serving path (cudaMalloc and
// cudaFree synchronise the device and stall every other stream), or in a
// process whose device memory is owned by another allocator (a framework's
// caching pool or a fixed arena) that hands out only the operand buffers.
// The regular xmpIntegersPowm grows the handle's scratch arena with the
// handle's allocator; this entry point instead keeps the exponentiation
// window tables in a fixed, file-scope device array, so the call itself
// allocates nothing.
//
// Scratch: kNoAllocScratchBytes (16 MiB) of `__device__` memory.  Every GPU
// that loads this library holds it until the process exits.  The array is
// shared by all calls on a device and keeps the last call's contents; the
// kernel writes every table slot before reading it, so nothing needs
// clearing.  Calls whose kernels overlap on the GPU (different streams, or
// several host threads) race on this array: serialise them.
//
// Device address: host code cannot pass the array's name to a kernel (on the
// host it is a stand-in, not a device address).  The first call on each
// device looks the address up with cudaGetSymbolAddress while that device is
// current and caches it; make that first call before any stream capture.
#include "powm.h"
#include <mutex>

namespace xmpb {

constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocScratchBytes / 4];

constexpr int kNoAllocMaxDevices = 256;
static void *g_noalloc_addr[kNoAllocMaxDevices];
static std::mutex g_noalloc_mu;

static xmpError_t noalloc_scratch(int device, void **addr) {
  if (device < 0 || device >= kNoAllocMaxDevices) return xmpErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return xmpErrorCuda;
    }
    g_noalloc_addr[device] = p;
  }
  *addr = g_noalloc_addr[device];
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
  xmpError_t e = noalloc_scratch(device, &scratch);
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
