// PTX carry-chain primitives (replaces the PTXInliner/PTXChain layer,
// src/include/ptx/ptx.h:31-168).  Each wrapper is one PTX integer instruction;
// `asm volatile` keeps the statements of a chain in program order so the
// carry flag written by one `.cc` instruction is the one read by the next.
// Only the 32-bit IMAD formulation is provided: sm_100 has full-rate 32-bit
// multiply-add, so the reference's 16-bit XMAD emulation has no counterpart.
#pragma once
#include <stdint.h>

namespace xmpb {

__device__ __forceinline__ uint32_t add_cc(uint32_t a, uint32_t b) {
  uint32_t r;
  asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t addc_cc(uint32_t a, uint32_t b) {
  uint32_t r;
  asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t addc(uint32_t a, uint32_t b) {
  uint32_t r;
  asm volatile("addc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t sub_cc(uint32_t a, uint32_t b) {
  uint32_t r;
  asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t subc_cc(uint32_t a, uint32_t b) {
  uint32_t r;
  asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t subc(uint32_t a, uint32_t b) {
  uint32_t r;
  asm volatile("subc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
// r = lo(a*b) + c, carry out
__device__ __forceinline__ uint32_t mad_lo_cc(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r;
  asm volatile("mad.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
}
__device__ __forceinline__ uint32_t madc_lo_cc(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r;
  asm volatile("madc.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
}
__device__ __forceinline__ uint32_t mad_hi_cc(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r;
  asm volatile("mad.hi.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
}
__device__ __forceinline__ uint32_t madc_hi_cc(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r;
  asm volatile("madc.hi.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
}
__device__ __forceinline__ uint32_t madc_hi(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r;
  asm volatile("madc.hi.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
}
__device__ __forceinline__ uint32_t madc_lo(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r;
  asm volatile("madc.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
}

// a + carry-in (no carry-out) issued as a multiply-add (a*1 + 0 + CC), so the
// chain's last step can go to the FMA pipe instead of the integer ALU, which
// the carry-producing adds keep busy.
__device__ __forceinline__ uint32_t addc_fma(uint32_t a) {
  uint32_t r;
  asm volatile("madc.lo.u32 %0, %1, 1, 0;" : "=r"(r) : "r"(a));
  return r;
}

// Full 64-bit product a*b (one wide multiply); no carry flag involved, so the
// compiler may schedule it freely between carry chains.
__device__ __forceinline__ uint64_t mul_wide(uint32_t a, uint32_t b) {
  uint64_t r;
  asm("mul.wide.u32 %0, %1, %2;" : "=l"(r) : "r"(a), "r"(b));
  return r;
}

// -n^{-1} mod 2^32 for odd n by Newton-Hensel lifting: x <- x(2 - n x) doubles
// the number of correct low bits; n*n == 1 mod 8 gives 3 bits to start.
__host__ __device__ __forceinline__ uint32_t neg_inv32(uint32_t n) {
  uint32_t x = n;
  x = x * (2u - n * x);
  x = x * (2u - n * x);
  x = x * (2u - n * x);
  x = x * (2u - n * x);
  return 0u - x;
}

}  // namespace xmpb
