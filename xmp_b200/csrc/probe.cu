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

// mode 2: independent mad.wide.u32 (64-bit product + 64-bit addend), 2 multiply-adds each
// mode 3: independent mad.hi.u32
// mode 4: rows written with 64-bit C arithmetic, t = a*w + r + c (compiler-chosen instructions)
// mode 5: low-half chains only (mad.lo.cc / madc.lo.cc), 8 per row
// mode 6: add.cc / addc.cc chains (no multiplies), counted as adds
__global__ void __launch_bounds__(256) imad_wide(uint32_t *out, int iters, uint32_t seed) {
  uint64_t acc[8];
  uint32_t a[8];
  const uint32_t b = seed | 1u;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    a[k] = seed ^ (threadIdx.x * 2654435761u + k);
    acc[k] = k;
  }
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 8; u++) {
#pragma unroll
      for (int k = 0; k < 8; k++) asm volatile("mad.wide.u32 %0, %1, %2, %0;" : "+l"(acc[k]) : "r"(a[k]), "r"(b));
    }
  }
  uint64_t s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s ^= acc[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = (uint32_t)s ^ (uint32_t)(s >> 32);
}

__global__ void __launch_bounds__(256) imad_hi(uint32_t *out, int iters, uint32_t seed) {
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
      for (int k = 0; k < 8; k++) asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(b), "r"(c[k]));
    }
  }
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s ^= a[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) imad_rows64(uint32_t *out, int iters, uint32_t seed) {
  uint32_t a[8], r[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    a[k] = seed ^ (threadIdx.x * 2654435761u + k);
    r[k] = k;
  }
  uint32_t w = seed | 1u, top = 0;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 4; u++) {
      uint64_t c = 0;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        uint64_t t = (uint64_t)a[k] * w + r[k] + c;
        r[k] = (uint32_t)t;
        c = t >> 32;
      }
      top += (uint32_t)c;
      w += r[0];
    }
  }
  uint32_t s = top;
#pragma unroll
  for (int k = 0; k < 8; k++) s ^= r[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) imad_lochain(uint32_t *out, int iters, uint32_t seed) {
  uint32_t a[8], r[8], c0 = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    a[k] = seed ^ (threadIdx.x * 2654435761u + k);
    r[k] = k;
  }
  uint32_t w = seed | 1u;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 8; u++) {
      r[0] = mad_lo_cc(a[0], w, r[0]);
#pragma unroll
      for (int k = 1; k < 8; k++) r[k] = madc_lo_cc(a[k], w, r[k]);
      c0 = addc(c0, 0u);
      w += r[1];
    }
  }
  uint32_t s = c0;
#pragma unroll
  for (int k = 0; k < 8; k++) s ^= r[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) iadd_chain(uint32_t *out, int iters, uint32_t seed) {
  uint32_t a[8], r[8], c0 = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    a[k] = seed ^ (threadIdx.x * 2654435761u + k);
    r[k] = k;
  }
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 8; u++) {
      r[0] = add_cc(r[0], a[0]);
#pragma unroll
      for (int k = 1; k < 8; k++) r[k] = addc_cc(r[k], a[k]);
      c0 = addc(c0, 0u);
      a[u & 7] ^= r[7];
    }
  }
  uint32_t s = c0;
#pragma unroll
  for (int k = 0; k < 8; k++) s ^= r[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// mode 7: Montgomery-shaped rows on wide products: p_k = a_k*w + r_k (mad.wide, addend zero-extended),
//         then one add chain r_k = lo(p_k) + hi(p_{k-1}); two dependent rows per step, 8 limbs
// mode 8: same rows with p_k = a_k*w (mul.wide) and two add chains (r_k += lo(p_k), += hi(p_{k-1}))
__device__ __forceinline__ uint64_t madw(uint32_t a, uint32_t b, uint64_t c) {
  uint64_t r;
  asm volatile("mad.wide.u32 %0, %1, %2, %3;" : "=l"(r) : "r"(a), "r"(b), "l"(c));
  return r;
}
__device__ __forceinline__ uint64_t mulw(uint32_t a, uint32_t b) {
  uint64_t r;
  asm volatile("mul.wide.u32 %0, %1, %2;" : "=l"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t lo32(uint64_t v) { return (uint32_t)v; }
__device__ __forceinline__ uint32_t hi32(uint64_t v) { return (uint32_t)(v >> 32); }

template <int MODE>
__global__ void __launch_bounds__(256) wide_rows(uint32_t *out, int iters, uint32_t seed) {
  uint32_t a[8], n[8], r[8], c0 = 0, c1 = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    a[k] = seed ^ (threadIdx.x * 2654435761u + k);
    n[k] = a[k] * 7u + 1u;
    r[k] = k;
  }
  uint32_t w = seed | 1u;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const uint32_t *src = (u & 1) ? n : a;
      uint64_t p[8];
      if (MODE == 7) {
#pragma unroll
        for (int k = 0; k < 8; k++) p[k] = madw(src[k], w, (uint64_t)r[k]);
        r[0] = lo32(p[0]);
        r[1] = add_cc(lo32(p[1]), hi32(p[0]));
#pragma unroll
        for (int k = 2; k < 8; k++) r[k] = addc_cc(lo32(p[k]), hi32(p[k - 1]));
        c0 = addc_cc(c0, hi32(p[7]));
        c1 = addc(c1, 0u);
      } else {
#pragma unroll
        for (int k = 0; k < 8; k++) p[k] = mulw(src[k], w);
        r[0] = add_cc(r[0], lo32(p[0]));
#pragma unroll
        for (int k = 1; k < 8; k++) r[k] = addc_cc(r[k], lo32(p[k]));
        c0 = addc_cc(c0, 0u);
        c1 = addc(c1, 0u);
        r[1] = add_cc(r[1], hi32(p[0]));
#pragma unroll
        for (int k = 2; k < 8; k++) r[k] = addc_cc(r[k], hi32(p[k - 1]));
        c0 = addc_cc(c0, hi32(p[7]));
        c1 = addc(c1, 0u);
      }
      w = r[0] * 0x9e3779b9u;
    }
  }
  uint32_t s = c0 ^ c1;
#pragma unroll
  for (int k = 0; k < 8; k++) s ^= r[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// mode 9: independent mad.wide.u32 with a 32-bit addend (zero-extended), both halves consumed
__global__ void __launch_bounds__(256) wide_addend32(uint32_t *out, int iters, uint32_t seed) {
  uint32_t a[8], r[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    a[k] = seed ^ (threadIdx.x * 2654435761u + k);
    r[k] = k;
  }
  const uint32_t w = seed | 1u;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 8; u++) {
#pragma unroll
      for (int k = 0; k < 8; k++) {
        uint64_t p = madw(a[k], w, (uint64_t)r[k]);
        r[k] = lo32(p) ^ hi32(p);
      }
    }
  }
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s ^= r[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Runs the probe on the current device; *imads = multiply-adds executed,
// *ms = kernel time from CUDA events.  Returns a cudaError_t value.
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
      case 1: imad_rows<<<blocks, threads>>>(out, it, 12345u); break;
      case 2: imad_wide<<<blocks, threads>>>(out, it, 12345u); break;
      case 3: imad_hi<<<blocks, threads>>>(out, it, 12345u); break;
      case 4: imad_rows64<<<blocks, threads>>>(out, it, 12345u); break;
      case 5: imad_lochain<<<blocks, threads>>>(out, it, 12345u); break;
      case 7: wide_rows<7><<<blocks, threads>>>(out, it, 12345u); break;
      case 8: wide_rows<8><<<blocks, threads>>>(out, it, 12345u); break;
      case 9: wide_addend32<<<blocks, threads>>>(out, it, 12345u); break;
      default: iadd_chain<<<blocks, threads>>>(out, it, 12345u); break;
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
  // multiply-adds per thread per iteration (a mad.wide counts as two: low and high halves)
  const double per_iter_by_mode[10] = {64.0, 64.0, 128.0, 64.0, 64.0, 64.0, 64.0, 64.0, 64.0, 128.0};
  double per_iter = per_iter_by_mode[mode < 0 || mode > 9 ? 6 : mode];
  *imads = (double)blocks * threads * iters * per_iter;
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(out);
  return e == cudaSuccess ? (int)cudaGetLastError() : (int)e;
}
