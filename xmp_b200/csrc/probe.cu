// INT32 multiply-add throughput microbenchmark (libxmpprobe.so): measures the
// roofline denominator for the integer kernels on the device it runs on.
//   mode 0: independent mad.lo.u32 chains (plain IMAD issue rate)
//   mode 1: mad.lo.cc / madc.hi.cc carry-chain rows shaped like the Montgomery
//           inner loop (2L multiply-adds + 2 carry adds per row, L = 8)
// Every instruction is inline PTX so the count per thread is exact; the
// result is written out so nothing is dead.
#include <cuda_runtime.h>
#include <stdint.h>
#include "carry.cuh"

using namespace xmpb;

#define PROBE_API extern "C" __attribute__((visibility("default")))

__global__ void __launch_bounds__(256) imad_plain(uint32_t *out, int iters, uint32_t seed) {
  uint32_t a[8], c[8];
  const uint32_t b = seed | 1u;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    a[k] = seed ^ (threadIdx.x * 2654435761u + k);
    c[k] = k * 7919u;
  }
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 8; u++) {
#pragma unroll
      for (int k = 0; k < 8; k++) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(b), "r"(c[k]));
    }
  }
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s ^= a[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) imad_rows(uint32_t *out, int iters, uint32_t seed) {
  uint32_t a[8], r[8], c0 = 0, c1 = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    a[k] = seed ^ (threadIdx.x * 2654435761u + k);
    r[k] = k;
  }
  uint32_t w = seed | 1u;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 4; u++) {
      r[0] = mad_lo_cc(a[0], w, r[0]);
#pragma unroll
      for (int k = 1; k < 8; k++) r[k] = madc_lo_cc(a[k], w, r[k]);
      c0 = addc_cc(c0, 0u);
      c1 = addc(c1, 0u);
      r[1] = mad_hi_cc(a[0], w, r[1]);
#pragma unroll
      for (int k = 2; k < 8; k++) r[k] = madc_hi_cc(a[k - 1], w, r[k]);
      c0 = madc_hi_cc(a[7], w, c0);
      c1 = addc(c1, 0u);
      w += r[0];
    }
  }
  uint32_t s = c0 ^ c1;
#pragma unroll
  for (int k = 0; k < 8; k++) s ^= r[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

PROBE_API int xmpb_probe_imad(int mode, int blocks_per_sm, int iters, double *imads, double *ms) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int threads = 256, blocks = sms * blocks_per_sm;
  uint32_t *out = nullptr;
  cudaError_t e = cudaMalloc(&out, (size_t)blocks * threads * 4);
  if (e != cudaSuccess) return (int)e;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  auto launch = [&](int it) {
    switch (mode) {
      case 0: imad_plain<<<blocks, threads>>>(out, it, 12345u); break;
      default: imad_rows<<<blocks, threads>>>(out, it, 12345u); break;
    }
  };
  launch(iters / 8 + 1);  // warm-up
  cudaEventRecord(t0);
  launch(iters);
  cudaEventRecord(t1);
  e = cudaEventSynchronize(t1);
  float f = 0;
  cudaEventElapsedTime(&f, t0, t1);
  *ms = f;
  // multiply-adds per thread per iteration (both modes: 64)
  *imads = (double)blocks * threads * iters * 64.0;
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(out);
  return e == cudaSuccess ? (int)cudaGetLastError() : (int)e;
}
