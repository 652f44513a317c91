// Look-back descriptors of the structural indexer: one 64-bit word per tile.
//   bits 0-1   status (0 = not ready, 1 = aggregate, 2 = inclusive prefix)
//   bit  2     string parity: string state after the span if it starts
//              outside a string (for a constant span: the state after it)
//   bits 3-10  depth change if the span starts outside a string (mod 256)
//   bits 11-18 depth change if it starts inside a string (mod 256)
//   bit  19    constant: the span starts at a file start (state and depth
//              restart there), so its result does not depend on what came
//              before; inclusive prefixes are constant too
//   bits 20-63 newline count (runs on across files)
// A span is a function from the (string state, depth) entering it to the
// pair leaving it; composition of such functions is associative, which is
// what lets one warp fold 128 predecessors per step.
//
// Host and device: the CPU unit test checks the packed composition against
// the field-wise one and for associativity.
#pragma once

#include <cstdint>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace gpjb {

constexpr uint64_t kStatusAgg = 1, kStatusIncl = 2;

struct Agg {
  uint32_t p;   // string parity (or final state for a constant span)
  uint32_t d0;  // depth change starting outside a string (mod 256)
  uint32_t d1;  // depth change starting inside a string (mod 256)
  uint32_t c;   // 1 = constant span
  uint64_t n;   // newlines
};

__host__ __device__ __forceinline__ Agg agg_identity() { return Agg{0u, 0u, 0u, 0u, 0ull}; }

// `a` covers the bytes before `b`.
__host__ __device__ __forceinline__ Agg agg_combine(const Agg &a, const Agg &b) {
  Agg r;
  r.n = a.n + b.n;
  if (b.c) {  // b restarts: what came before only adds newlines
    r.p = b.p;
    r.d0 = b.d0;
    r.d1 = b.d1;
    r.c = 1u;
  } else if (a.c) {  // constant a: b sees a's final state
    r.p = a.p ^ b.p;
    r.d0 = r.d1 = (a.d0 + (a.p ? b.d1 : b.d0)) & 0xFFu;
    r.c = 1u;
  } else {
    r.p = a.p ^ b.p;
    r.d0 = (a.d0 + (a.p ? b.d1 : b.d0)) & 0xFFu;
    r.d1 = (a.d1 + (a.p ? b.d0 : b.d1)) & 0xFFu;
    r.c = 0u;
  }
  return r;
}

__host__ __device__ __forceinline__ uint64_t agg_pack(uint64_t status, const Agg &a) {
  return status | (uint64_t(a.p & 1u) << 2) | (uint64_t(a.d0 & 0xFFu) << 3) |
         (uint64_t(a.d1 & 0xFFu) << 11) | (uint64_t(a.c & 1u) << 19) | (a.n << 20);
}

__host__ __device__ __forceinline__ Agg agg_unpack(uint64_t v) {
  Agg a;
  a.p = uint32_t(v >> 2) & 1u;
  a.d0 = uint32_t(v >> 3) & 0xFFu;
  a.d1 = uint32_t(v >> 11) & 0xFFu;
  a.c = uint32_t(v >> 19) & 1u;
  a.n = v >> 20;
  return a;
}

// agg_combine on packed descriptors, branch-free; the status bits of the
// result are 0 (the identity is the word 0).
__host__ __device__ __forceinline__ uint64_t desc_combine(uint64_t a, uint64_t b) {
  const uint32_t al = uint32_t(a), bl = uint32_t(b);
  const uint32_t ap = (al >> 2) & 1u, ac = (al >> 19) & 1u, bc = (bl >> 19) & 1u;
  const uint32_t ad0 = (al >> 3) & 0xFFu, ad1 = (al >> 11) & 0xFFu;
  const uint32_t bd0 = (bl >> 3) & 0xFFu, bd1 = (bl >> 11) & 0xFFu;
  const uint32_t d0 = (ad0 + (ap ? bd1 : bd0)) & 0xFFu;
  const uint32_t d1 = ac ? d0 : ((ad1 + (ap ? bd0 : bd1)) & 0xFFu);
  const uint32_t mixed = (((al ^ bl) >> 2) & 1u) << 2 | (d0 << 3) | (d1 << 11) | (ac << 19);
  const uint32_t lo = bc ? (bl & 0xFFFFCu) : mixed;
  return (((a >> 20) + (b >> 20)) << 20) | lo;
}

}  // namespace gpjb
