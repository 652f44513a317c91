// Bit-level building blocks of the structural indexer (sm_100a).
//
// Every helper works on 64-bit words where bit b of word w stands for byte
// 64*w + b of the partition, LSB first -- the layout of the reference's
// escape/quote/string/leveled bitmaps (Xinyu-Li-123/15418-project,
// src/gpjson/index/kernels/sharemem/*.cu).
#pragma once

#include <cstdint>

#include "classify.cuh"

namespace gpjb {

// Classes of one 64-byte word.  Only the characters the index needs:
//   bs  '\\'        qt '"'        nl '\n'
//   op  '{' '['     cl '}' ']'    sp ':' ','
struct WordClasses {
  uint64_t bs, qt, nl, op, cl, sp;
};

// Classifies 64 bytes held as 16 registers (r[0] = bytes 0..3), two
// bit-sliced groups of 32 bytes (classify.cuh).
__device__ __forceinline__ WordClasses classify64(const uint32_t (&r)[16]) {
  const GroupClasses lo = classify32(r);
  const GroupClasses hi = classify32(r + 8);
  auto join = [](uint32_t a, uint32_t b) -> uint64_t {
    return (static_cast<uint64_t>(b) << 32) | a;
  };
  WordClasses w;
  w.bs = join(lo.bs, hi.bs);
  w.qt = join(lo.qt, hi.qt);
  w.nl = join(lo.nl, hi.nl);
  w.op = join(lo.op, hi.op);
  w.cl = join(lo.cl, hi.cl);
  w.sp = join(lo.sp, hi.sp);
  return w;
}

// ---------------------------------------------------------------------------
// Escape bitmap of one word.
//
// Bit i is set iff the byte-serial machine "bit i = carry; carry = (byte is
// '\\') ? !carry : 0" (sharemem/uncombined/escape-index.cu:29-96) would set
// it, given the carry entering the word.  Bit-parallel form: inside a run of
// backslashes that starts at s, the positions s+1 .. end that sit an odd
// distance from s are escaped.  Runs starting on even bits escape odd
// positions, runs starting on odd bits escape even positions.  An escaped
// backslash at bit 0 (carry_in = 1) does not start a run.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t escaped_bits(uint64_t bs, uint32_t carry_in) {
  constexpr uint64_t kEven = 0x5555555555555555ull;
  const uint64_t cin = static_cast<uint64_t>(carry_in & 1u);
  const uint64_t b = bs & ~cin;
  const uint64_t starts = b & ~(b << 1);
  // Adding 1 at every odd start ripples through that run and clears it, so
  // what stays set under b are the runs that start on even bits.
  const uint64_t even_runs = (b + (starts & ~kEven)) & b;
  // escaped: the odd positions after an even-started run, the even positions
  // after an odd-started one -- the run bits on the other parity, shifted up
  // once (one three-input mask per half instead of two shifts and masks)
  const uint64_t pre = (even_runs & kEven) | (b & ~even_runs & ~kEven);
  return (pre << 1) | cin;
}

// Carry the reference passes from a word to the next: parity of the run of
// backslashes that ends the word, counted inside the word only
// (sharemem/uncombined/escape-carry-index.cu:95-164).  An all-backslash word
// gives __clzll(0) = 64 -> parity 0.
__device__ __forceinline__ uint32_t trailing_escape_parity(uint64_t bs) {
  return static_cast<uint32_t>(__clzll(static_cast<long long>(~bs))) & 1u;
}

// Inclusive prefix-XOR inside one word (sharemem/string-index.cu:16-21).
__device__ __forceinline__ uint64_t prefix_xor(uint64_t x) {
  x ^= x << 1;
  x ^= x << 2;
  x ^= x << 4;
  x ^= x << 8;
  x ^= x << 16;
  x ^= x << 32;
  return x;
}

__device__ __forceinline__ int popc64(uint64_t x) { return __popcll(x); }

}  // namespace gpjb
