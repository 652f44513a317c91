// Bit-level building blocks of the structural indexer (sm_100a).
//
// Every helper works on 64-bit words where bit b of word w stands for byte
// 64*w + b of the partition, LSB first -- the layout of the reference's
// escape/quote/string/leveled bitmaps (Xinyu-Li-123/15418-project,
// src/gpjson/index/kernels/sharemem/*.cu).
#pragma once

#include <cstdint>

namespace gpjb {

// ---------------------------------------------------------------------------
// Byte classification (SWAR on 4 bytes per 32-bit register).
//
// eq_flags(x, pat, mask) sets bit 7 of every byte of x whose value equals the
// pattern byte under `mask` and whose own bit 7 is clear; every other bit of
// the result is 0.  With mask = 0x7F the test is plain equality; with
// mask = 0x5F bit 5 is ignored, which folds '{'/'[' (0x7B/0x5B) and '}'/']'
// (0x7D/0x5D) into one test each.  All pattern bytes are ASCII (< 0x80).
//   t = (x ^ pat) & mask          -> 0 in a byte iff the byte matches
//   y = t + 0x7F                  -> bit 7 of a byte set iff t != 0 (no carry
//                                    leaves the byte since t <= 0x7F)
//   ~(y | x) & 0x80               -> match and ASCII
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t eq_partial(uint32_t x, uint32_t pat,
                                               uint32_t mask) {
  return ((x ^ pat) & mask) + 0x7F7F7F7Fu;
}
__device__ __forceinline__ uint32_t eq_flags(uint32_t x, uint32_t pat,
                                             uint32_t mask) {
  return ~(eq_partial(x, pat, mask) | x) & 0x80808080u;
}

// Gathers the bit-7 flags of 16 consecutive bytes (4 registers, byte 0 of f0
// first) into a 16-bit mask.  __dp4a multiplies each flag byte (0x80 or 0)
// by a power-of-two weight and sums, i.e. it is a "movemask" of four bytes:
// f0 lands on bits 7..10, f1 on bits 11..14.
__device__ __forceinline__ uint32_t gather16(uint32_t f0, uint32_t f1,
                                             uint32_t f2, uint32_t f3) {
  const uint32_t lo = __dp4a(f1, 0x80402010u, __dp4a(f0, 0x08040201u, 0u));
  const uint32_t hi = __dp4a(f3, 0x80402010u, __dp4a(f2, 0x08040201u, 0u));
  return (lo >> 7) | (hi << 1);
}

// Classes of one 64-byte word.  Only the characters the index needs:
//   bs  '\\'        qt '"'        nl '\n'
//   op  '{' '['     cl '}' ']'    sp ':' ','
struct WordClasses {
  uint64_t bs, qt, nl, op, cl, sp;
};

// Classifies 64 bytes held as 16 registers (r[0] = bytes 0..3).
__device__ __forceinline__ WordClasses classify64(const uint32_t (&r)[16]) {
  constexpr uint32_t kM7 = 0x7F7F7F7Fu, kM5 = 0x5F5F5F5Fu;
  uint32_t g_bs[4], g_qt[4], g_nl[4], g_op[4], g_cl[4], g_sp[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    uint32_t f_bs[4], f_qt[4], f_nl[4], f_op[4], f_cl[4], f_sp[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t x = r[4 * c + k];
      f_bs[k] = eq_flags(x, 0x5C5C5C5Cu, kM7);
      f_qt[k] = eq_flags(x, 0x22222222u, kM7);
      f_nl[k] = eq_flags(x, 0x0A0A0A0Au, kM7);
      f_op[k] = eq_flags(x, 0x5B5B5B5Bu, kM5);
      f_cl[k] = eq_flags(x, 0x5D5D5D5Du, kM5);
      // ':' or ',': ~((y_colon & y_comma) | x) & 0x80
      f_sp[k] = ~((eq_partial(x, 0x3A3A3A3Au, kM7) &
                   eq_partial(x, 0x2C2C2C2Cu, kM7)) | x) & 0x80808080u;
    }
    g_bs[c] = gather16(f_bs[0], f_bs[1], f_bs[2], f_bs[3]);
    g_qt[c] = gather16(f_qt[0], f_qt[1], f_qt[2], f_qt[3]);
    g_nl[c] = gather16(f_nl[0], f_nl[1], f_nl[2], f_nl[3]);
    g_op[c] = gather16(f_op[0], f_op[1], f_op[2], f_op[3]);
    g_cl[c] = gather16(f_cl[0], f_cl[1], f_cl[2], f_cl[3]);
    g_sp[c] = gather16(f_sp[0], f_sp[1], f_sp[2], f_sp[3]);
  }
  auto join = [](const uint32_t (&g)[4]) -> uint64_t {
    const uint32_t lo = __byte_perm(g[0], g[1], 0x5410);
    const uint32_t hi = __byte_perm(g[2], g[3], 0x5410);
    return (static_cast<uint64_t>(hi) << 32) | lo;
  };
  WordClasses w;
  w.bs = join(g_bs);
  w.qt = join(g_qt);
  w.nl = join(g_nl);
  w.op = join(g_op);
  w.cl = join(g_cl);
  w.sp = join(g_sp);
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
  const uint64_t odd_runs = b & ~even_runs;
  return ((even_runs << 1) & ~kEven) | ((odd_runs << 1) & kEven) | cin;
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
