// Bit-sliced byte classification: the character classes the structural
// index needs, for 32 bytes at a time, as 32-bit masks (bit j = byte j).
//
// The 32 bytes (eight little-endian 32-bit registers) are transposed into
// eight bit planes -- plane k holds bit k of every byte -- and each class is
// then a product of plane literals, a handful of three-input logic ops for
// all 32 bytes.  The transpose is a byte permutation (register i gathers
// bytes i, 8+i, 16+i, 24+i) followed by three exchange stages, each of which
// swaps one bit of the register index with one bit of the bit-in-byte index.
//
// Host and device: the same code runs in the CPU unit test.
#pragma once

#include <cstdint>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace gpjb {

// byte permute: bytes 0-3 of x then 0-3 of y, selected by the nibbles of s
__host__ __device__ __forceinline__ uint32_t perm_bytes(uint32_t x, uint32_t y, uint32_t s) {
#if defined(__CUDA_ARCH__)
  return __byte_perm(x, y, s);
#else
  const uint64_t v = (uint64_t(y) << 32) | x;
  uint32_t r = 0;
  for (int n = 0; n < 4; ++n) r |= uint32_t((v >> (8 * ((s >> (4 * n)) & 7u))) & 0xFFu) << (8 * n);
  return r;
#endif
}

// 4x4 byte transpose: out[i] = byte i of a, b, c, d
__host__ __device__ __forceinline__ void byte_transpose4(uint32_t a, uint32_t b, uint32_t c,
                                                         uint32_t d, uint32_t &o0, uint32_t &o1,
                                                         uint32_t &o2, uint32_t &o3) {
  const uint32_t t0 = perm_bytes(a, b, 0x5140u);  // a0 b0 a1 b1
  const uint32_t t1 = perm_bytes(a, b, 0x7362u);  // a2 b2 a3 b3
  const uint32_t t2 = perm_bytes(c, d, 0x5140u);  // c0 d0 c1 d1
  const uint32_t t3 = perm_bytes(c, d, 0x7362u);  // c2 d2 c3 d3
  o0 = perm_bytes(t0, t2, 0x5410u);               // a0 b0 c0 d0
  o1 = perm_bytes(t0, t2, 0x7632u);               // a1 b1 c1 d1
  o2 = perm_bytes(t1, t3, 0x5410u);
  o3 = perm_bytes(t1, t3, 0x7632u);
}

// Swaps bit j of the register index (a: 0, b: 1) with bit j of the
// bit-in-byte index; S = 2^j, M = positions whose bit-in-byte index has bit
// j set.
template <int S, uint32_t M>
__host__ __device__ __forceinline__ void exchange(uint32_t &a, uint32_t &b) {
  const uint32_t na = (a & ~M) | ((b << S) & M);
  const uint32_t nb = (b & M) | ((a >> S) & ~M);
  a = na;
  b = nb;
}

struct GroupClasses {
  uint32_t bs, qt, nl, op, cl, sp;
};

// r[m] holds bytes 4m .. 4m+3 (little-endian).
__host__ __device__ __forceinline__ GroupClasses classify32(const uint32_t *r) {
  uint32_t p[8];
  byte_transpose4(r[0], r[2], r[4], r[6], p[0], p[1], p[2], p[3]);
  byte_transpose4(r[1], r[3], r[5], r[7], p[4], p[5], p[6], p[7]);
  // p[i] now holds byte 8c+i at bits 8c..8c+7
  exchange<1, 0xAAAAAAAAu>(p[0], p[1]);
  exchange<1, 0xAAAAAAAAu>(p[2], p[3]);
  exchange<1, 0xAAAAAAAAu>(p[4], p[5]);
  exchange<1, 0xAAAAAAAAu>(p[6], p[7]);
  exchange<2, 0xCCCCCCCCu>(p[0], p[2]);
  exchange<2, 0xCCCCCCCCu>(p[1], p[3]);
  exchange<2, 0xCCCCCCCCu>(p[4], p[6]);
  exchange<2, 0xCCCCCCCCu>(p[5], p[7]);
  exchange<4, 0xF0F0F0F0u>(p[0], p[4]);
  exchange<4, 0xF0F0F0F0u>(p[1], p[5]);
  exchange<4, 0xF0F0F0F0u>(p[2], p[6]);
  exchange<4, 0xF0F0F0F0u>(p[3], p[7]);
  // p[k] = plane k: bit j = bit k of byte j
  const uint32_t a = ~p[7] & p[6] & p[4];    // 01x1xxxx
  const uint32_t x = a & p[3] & p[0];        // 01x11xx1
  const uint32_t b = ~p[7] & ~p[6] & ~p[0];  // 00xxxxx0
  const uint32_t c = b & p[1] & ~p[2];       // 00xxx010
  GroupClasses g;
  g.op = x & ~p[2] & p[1];                          // '{' 0x7B, '[' 0x5B
  g.cl = x & p[2] & ~p[1];                          // '}' 0x7D, ']' 0x5D
  g.bs = a & ~p[5] & p[3] & p[2] & ~p[1] & ~p[0];   // '\\' 0x5C
  g.qt = c & p[5] & ~p[4] & ~p[3];                  // '"' 0x22
  g.nl = c & ~p[5] & ~p[4] & p[3];                  // '\n' 0x0A
  g.sp = (c & p[5] & p[4] & p[3]) |                 // ':' 0x3A
         (b & ~p[1] & p[2] & p[5] & ~p[4] & p[3]);  // ',' 0x2C
  return g;
}

}  // namespace gpjb
