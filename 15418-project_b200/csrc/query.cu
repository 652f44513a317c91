// JSONPath query kernel: one thread per record interprets the byte IR over
// the leveled bitmaps and the string mask and writes (start, end) byte
// offsets per result slot.  Semantics follow
// src/gpjson/query/kernels/orig/query.cu:144-454 of the reference; the IR is
// passed in the kernel parameters and staged in shared memory instead of a
// process-global __constant__ array (query.cu:11), so launches on different
// streams do not race.  Positions are 64-bit internally; with partitions
// below 2 GiB every value equals the reference's int arithmetic.
#include "query.cuh"

namespace gpjb {
namespace {

enum : uint8_t {
  OP_END = 0x00,
  OP_STORE_RESULT = 0x01,
  OP_MOVE_UP = 0x02,
  OP_MOVE_DOWN = 0x03,
  OP_MOVE_TO_KEY = 0x04,
  OP_MOVE_TO_INDEX = 0x05,
  OP_MOVE_TO_INDEX_REVERSE = 0x06,
  OP_MARK_POSITION = 0x07,
  OP_RESET_POSITION = 0x08,
  OP_EXPRESSION_STRING_EQUALS = 0x09,
  // Extensions of this build (never emitted for the reference's syntax):
  OP_NUMBER_COMPARE = 0x0A,  // numeric filter: cmp byte, varint length, number text
  OP_DESCEND_KEY = 0x0B,     // "..name" as the last step: varint length, key bytes
  OP_EXPECT_AT_MOST = 0x0C,  // "[*]" element-count check: varint limit
  OP_EXPECT_FOLLOWING = 0x0D,  // "[a:-b]": varint count of elements that must follow
};

// Last bitmap word read, per thread: consecutive searches of a record mostly
// start in the word the previous search ended in.
template <typename Pos>
struct WordCache {
  const uint64_t *bm = nullptr;
  Pos idx = -1;
  uint64_t val = 0;
};

template <typename Pos>
struct Rec {
  const uint8_t *in;
  Pos n;
  const uint64_t *S;
  const uint64_t *LB;
  Pos W;
  const uint8_t *ir;  // shared memory
  int ir_len;
  int base;    // bitmap level of query level 0
  int levels;  // levels present in LB
  unsigned int *status;  // kQueryStatusOverflow is OR-ed here (may be null)
};

// Per-thread interpreter state indexed by query level, in shared memory
// (slot [level * stride + thread]): the end of each open level and the
// current array index at it.  `nlev` levels are held: the deepest level the
// IR can reach (query_ir_levels), at most kMaxQueryLevels.
template <typename Pos>
struct LevelState {
  Pos *end;
  int32_t *index;
  int stride, nlev;
  __device__ __forceinline__ Pos &level_end(int l) const { return end[l * stride]; }
  __device__ __forceinline__ int32_t &curr_index(int l) const { return index[l * stride]; }
};

// The reference reads file[] unguarded; well-formed JSON never leaves the
// partition.  Out-of-range reads return 0 here.
template <typename Pos>
__device__ __forceinline__ uint8_t at(const Rec<Pos> &c, Pos i) {
  return (i >= 0 && i < c.n) ? c.in[i] : uint8_t(0);
}
template <typename Pos>
__device__ __forceinline__ uint8_t ir_at(const Rec<Pos> &c, int i) {
  return (i >= 0 && i < c.ir_len) ? c.ir[i] : uint8_t(0);
}

template <typename Pos>
__device__ __forceinline__ uint64_t cached_word(WordCache<Pos> &wc, const uint64_t *bm, Pos W,
                                                Pos i) {
  if (wc.bm == bm && wc.idx == i) return wc.val;
  const uint64_t v = (i >= 0 && i < W) ? bm[i] : 0ull;
  wc.bm = bm;
  wc.idx = i;
  wc.val = v;
  return v;
}

__device__ __forceinline__ uint64_t mask_through_bit(int b) {
  return b == 63 ? ~0ull : ((1ull << (b + 1)) - 1ull);
}

// query.cu:39-77
template <typename Pos>
__device__ Pos prev_bit(WordCache<Pos> &wc, const uint64_t *bm, Pos W, Pos min_index,
                        Pos line_index) {
  if (line_index < min_index) return -1;
  Pos wi = line_index >> 6;
  Pos base = wi * 64;
  uint64_t word = cached_word(wc, bm, W, wi) & mask_through_bit(int(line_index - base));
  while (base + 63 >= min_index) {
    uint64_t cand = word;
    const Pos first = min_index - base;
    if (first > 0) cand &= ~mask_through_bit(int(first - 1));
    if (cand != 0) return base + 63 - __clzll(static_cast<long long>(cand));
    if (wi == 0) break;
    --wi;
    base -= 64;
    if (base + 63 < min_index) break;
    word = cached_word(wc, bm, W, wi);
  }
  return -1;
}

// Leveled-bitmap words of a query level, or null for a level the index does
// not hold (it has no structural characters).
template <typename Pos>
__device__ __forceinline__ const uint64_t *level_words(const Rec<Pos> &c, int level) {
  const int l = level + c.base;
  return (l < 0 || l >= c.levels) ? nullptr : c.LB + uint64_t(c.W) * uint64_t(l);
}

// query.cu:79-115
template <typename Pos>
__device__ Pos next_struct(const Rec<Pos> &c, WordCache<Pos> &wc, Pos level_end, Pos line_index,
                           const uint64_t *lvl) {
  if (line_index >= level_end || lvl == nullptr) return level_end;
  Pos wi = line_index >> 6;
  Pos base = wi * 64;
  {
    uint64_t cand = cached_word(wc, lvl, c.W, wi) & (~0ull << (line_index - base));
    const Pos last = level_end - base;
    if (last < 63) cand &= mask_through_bit(int(last));
    if (cand != 0) return base + __ffsll(static_cast<long long>(cand)) - 1;
  }
  // A long gap (a string value, a skipped member) spans several words: scan
  // them two at a time with one 16-byte load per aligned pair.  Words past W
  // are zero, so the scan may stop there.
  ++wi;
  base += 64;
  while (base <= level_end && wi < c.W) {
    const bool pair = ((reinterpret_cast<uintptr_t>(lvl + wi) & 15u) == 0) && wi + 1 < c.W;
    uint64_t w0, w1 = 0ull;
    if (pair) {
      const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(lvl + wi);
      w0 = v.x;
      w1 = v.y;
    } else {
      w0 = lvl[wi];
    }
    uint64_t cand = w0;
    Pos last = level_end - base;
    if (last < 63) cand &= mask_through_bit(int(last));
    if (cand != 0) {
      wc.bm = lvl;
      wc.idx = wi;
      wc.val = w0;
      return base + __ffsll(static_cast<long long>(cand)) - 1;
    }
    ++wi;
    base += 64;
    if (!pair) continue;
    if (base > level_end) break;
    cand = w1;
    last = level_end - base;
    if (last < 63) cand &= mask_through_bit(int(last));
    if (cand != 0) {
      wc.bm = lvl;
      wc.idx = wi;
      wc.val = w1;
      return base + __ffsll(static_cast<long long>(cand)) - 1;
    }
    ++wi;
    base += 64;
  }
  return level_end;
}

// query.cu:117-128
template <typename Pos>
__device__ Pos prev_struct(const Rec<Pos> &c, WordCache<Pos> &wc, Pos level_start, Pos line_index,
                           const uint64_t *lvl) {
  if (line_index <= level_start || lvl == nullptr) return level_start;
  const Pos s = prev_bit(wc, lvl, c.W, level_start, line_index);
  return s == -1 ? level_start : s;
}

// query.cu:130-140 (LEB128).  Unsigned arithmetic reinterpreted as int, as
// the reference's int result wraps; an operand longer than five bytes (never
// produced by the compiler) reads as -1.
template <typename Pos>
__device__ int read_varint(const Rec<Pos> &c, int &pos) {
  uint32_t value = 0, byte = 0;
  int shift = 0;
  while (((byte = ir_at(c, pos++)) & 0x80u) != 0) {
    value |= (byte & 0x7Fu) << shift;
    shift += 7;
    if (shift > 28) return -1;
  }
  return int(value | (byte << shift));
}


// ---- Extensions of this build (the reference's compiler rejects them) ----
//
// Exact decimal comparison of two JSON numbers (no floating point): a number
// is 0.d1d2d3... x 10^E with d1 != 0, or zero; exponents saturate at
// +-10^15.  Bytes come from a getter so the same code reads the partition
// (bounds-checked) and the IR.
struct DecNum {
  bool neg, zero;
  int64_t E, nd, first, int_len, int_pos, frac_pos;
};

constexpr int64_t kExpLimit = 1000000000000000ll;

__device__ __forceinline__ bool is_digit(uint8_t c) { return c >= '0' && c <= '9'; }

template <class Get>
__device__ __forceinline__ uint8_t dec_digit(const Get &get, const DecNum &x, int64_t k) {
  return get(k < x.int_len ? x.int_pos + k : x.frac_pos + (k - x.int_len));
}

// Parses bytes [0, len) of the getter as one JSON number (RFC 8259).
template <class Get>
__device__ bool dec_parse(const Get &get, int64_t len, DecNum &o) {
  int64_t i = 0;
  o.neg = false;
  if (i < len && get(i) == '-') {
    o.neg = true;
    ++i;
  }
  if (i >= len) return false;
  o.int_pos = i;
  const uint8_t c0 = get(i);
  if (c0 == '0') {
    ++i;
  } else if (c0 >= '1' && c0 <= '9') {
    while (i < len && is_digit(get(i))) ++i;
  } else {
    return false;
  }
  o.int_len = i - o.int_pos;
  int64_t frac_len = 0;
  o.frac_pos = i;
  if (i < len && get(i) == '.') {
    ++i;
    o.frac_pos = i;
    while (i < len && is_digit(get(i))) ++i;
    frac_len = i - o.frac_pos;
    if (frac_len == 0) return false;
  }
  int64_t ex = 0;
  if (i < len && (get(i) == 'e' || get(i) == 'E')) {
    ++i;
    bool eneg = false;
    if (i < len && (get(i) == '+' || get(i) == '-')) {
      eneg = get(i) == '-';
      ++i;
    }
    const int64_t es = i;
    while (i < len && is_digit(get(i))) {
      if (ex < kExpLimit) ex = ex * 10 + (get(i) - '0');
      ++i;
    }
    if (i == es) return false;
    if (ex > kExpLimit) ex = kExpLimit;
    if (eneg) ex = -ex;
  }
  if (i != len) return false;
  const int64_t total = o.int_len + frac_len;
  int64_t z = 0;
  while (z < total && dec_digit(get, o, z) == '0') ++z;
  o.zero = z == total;
  o.first = z;
  o.nd = total - z;
  o.E = o.int_len - z + ex;
  return true;
}

template <class GetA, class GetB>
__device__ int dec_cmp(const GetA &ga, const DecNum &a, const GetB &gb, const DecNum &b) {
  const int sa = a.zero ? 0 : (a.neg ? -1 : 1);
  const int sb = b.zero ? 0 : (b.neg ? -1 : 1);
  if (sa != sb) return sa < sb ? -1 : 1;
  if (sa == 0) return 0;
  int mag = 0;
  if (a.E != b.E) {
    mag = a.E > b.E ? 1 : -1;
  } else {
    const int64_t n = a.nd > b.nd ? a.nd : b.nd;
    for (int64_t k = 0; k < n && mag == 0; ++k) {
      const uint8_t da = k < a.nd ? dec_digit(ga, a, a.first + k) : uint8_t('0');
      const uint8_t db = k < b.nd ? dec_digit(gb, b, b.first + k) : uint8_t('0');
      if (da != db) mag = da > db ? 1 : -1;
    }
  }
  return sa > 0 ? mag : -mag;
}

__device__ __forceinline__ bool cmp_holds(int op, int r) {
  switch (op) {
  case 0: return r == 0;
  case 1: return r != 0;
  case 2: return r < 0;
  case 3: return r <= 0;
  case 4: return r > 0;
  case 5: return r >= 0;
  default: return false;
  }
}

template <typename Pos>
__device__ __forceinline__ void raise_status(const Rec<Pos> &c, unsigned int bits) {
  if (c.status != nullptr) atomicOr(c.status, bits);
}

// Does the string before the ':' at `colon` equal the key (the test of
// MOVE_TO_KEY, query.cu:254-302)?
template <typename Pos>
__device__ bool key_at_colon(const Rec<Pos> &c, WordCache<Pos> &sc, Pos line_start, Pos colon,
                             int key_pos, int key_len) {
  const Pos string_end = prev_bit(sc, c.S, c.W, Pos(line_start + 1), Pos(colon - 1));
  const Pos string_start = string_end - key_len;
  if (string_start < line_start || at(c, string_start) != '"') return false;
  for (int i = 0; i < key_len; ++i)
    if (ir_at(c, key_pos + i) != at(c, Pos(string_start + i + 1))) return false;
  return true;
}

template <typename Pos, typename OutT, bool kExt>
__device__ void run_record(const Rec<Pos> &c, const LevelState<Pos> &L, Pos line_start,
                           Pos line_end, int num_results, OutT *out) {
  if (line_start < 0 || line_start >= c.n || line_end < 0) return;
  if (line_end >= c.n) line_end = c.n - 1;
  while (line_end > line_start && at(c, line_end) != '}') --line_end;
  while (line_start < line_end && at(c, line_start) != '{') ++line_start;
  if (line_start == line_end) return;

  Pos line_index = line_start;
  int level = 0;
  int qp = 0;
  // Step bound of one search loop.  On well-formed JSON every step lands on a
  // new structural character of the record, so the bound is never reached;
  // on malformed input the reference's loops can revisit the same character
  // forever, and the record is abandoned instead.
  const Pos max_steps = (line_end - line_start) + 2;
  Pos steps = 0;
  WordCache<Pos> lbc, sc;  // leveled-bitmap and string-mask words
  L.level_end(0) = line_end;
  L.curr_index(0) = -1;
  for (int i = 1; i < L.nlev; ++i) {
    L.level_end(i) = -1;
    L.curr_index(i) = -1;
  }
  // marks belong to filter expressions only: rare, kept in local memory
  Pos marked_pos[kMaxQueryLevels];
  int marked_level[kMaxQueryLevels];
  int marked = -1;
  int stored = 0;
  int key_pos = 0;
  int key_len = 0;
  int target = 0;

#define LEVEL_OK(l) ((l) >= 0 && (l) < L.nlev)
  for (;;) {
    const uint8_t op = ir_at(c, qp++);
    switch (op) {
    case OP_END:
      return;
    case OP_STORE_RESULT: {
      if (!LEVEL_OK(level)) return;
      const Pos lend = L.level_end(level);
      Pos end_str = lend;
      while (at(c, line_index) == ' ' && line_index < lend) ++line_index;
      while (end_str > line_index && at(c, end_str - 1) == ' ') --end_str;
      if (stored < num_results) {
        out[2 * stored] = OutT(line_index);
        out[2 * stored + 1] = OutT(end_str);
      } else if constexpr (kExt) {
        raise_status(c, kQueryStatusOverflow);  // only extension IR gets here
      }
      ++stored;
      break;
    }
    case OP_MOVE_UP:
      if (!LEVEL_OK(level)) return;
      line_index = L.level_end(level);
      L.level_end(level) = -1;
      --level;
      break;
    case OP_MOVE_DOWN:
      ++level;
      if (!LEVEL_OK(level) || level < 1) return;
      if (L.level_end(level) == -1) {
        L.level_end(level) =
            next_struct(c, lbc, L.level_end(level - 1), Pos(line_index + 1),
                        level_words(c, level - 1));
        while (at(c, line_index) == ' ') ++line_index;
      }
      break;
    case OP_MOVE_TO_KEY: {
      key_len = read_varint(c, qp);
      key_pos = qp;
      qp += key_len;
      if (key_len < 0 || !LEVEL_OK(level)) return;
      if (at(c, line_index) != '{') return;
      const Pos lend = L.level_end(level);
      const uint64_t *lvl = level_words(c, level);
      steps = 0;
      for (;;) {
        if (++steps > max_steps) return;
        // Every position this step may inspect follows from the bitmaps
        // alone: the next structural character, the key string that would
        // end before it, and the structural character after it.  Their
        // bytes are then loaded together rather than one after another.
        const Pos p1 = next_struct(c, lbc, lend, Pos(line_index + 1), lvl);
        const Pos p2 = next_struct(c, lbc, lend, Pos(p1 + 1), lvl);
        const Pos string_end = prev_bit(sc, c.S, c.W, Pos(line_start + 1), Pos(p1 - 1));
        const Pos string_start = string_end - key_len;
        const uint8_t b1 = at(c, p1), b2 = at(c, p2), bq = at(c, string_start);
        line_index = p1;
        if (b1 == ':') {
          bool mismatch = string_start < line_start || bq != '"';
          for (int i = 0; !mismatch && i < key_len; ++i) {
            if (ir_at(c, key_pos + i) != at(c, Pos(string_start + i + 1))) mismatch = true;
          }
          if (mismatch) {
            line_index = p2;
            if (b2 == '}') return;
            continue;
          }
        }
        break;
      }
      ++line_index;
      break;
    }
    case OP_MOVE_TO_INDEX: {
      target = read_varint(c, qp);
      if (!LEVEL_OK(level)) return;
      const uint8_t ch = at(c, line_index);
      if (ch != '[' && ch != ',' && ch != ']') return;
      int32_t ci = ch == '[' ? 0 : L.curr_index(level) + 1;
      const Pos lend = L.level_end(level);
      const uint64_t *lvl = level_words(c, level);
      steps = 0;
      bool fail = false;
      for (;;) {
        if (++steps > max_steps) {
          fail = true;
          break;
        }
        if (ci < target) {
          ++line_index;
          line_index = next_struct(c, lbc, lend, line_index, lvl);
          if (at(c, line_index) == ',') {
            ++ci;
            continue;
          }
          fail = true;
          break;
        }
        if (ci > target) {
          --line_index;
          line_index = prev_struct(c, lbc, Pos(0), line_index, lvl);
          --ci;
          continue;
        }
        break;
      }
      L.curr_index(level) = ci;
      if (fail) return;
      if (at(c, line_index) == ']') return;
      ++line_index;
      break;
    }
    case OP_MOVE_TO_INDEX_REVERSE: {
      target = read_varint(c, qp);
      if (!LEVEL_OK(level)) return;
      line_index = L.level_end(level) - 1;
      while (at(c, line_index) == ' ') --line_index;
      const uint8_t ch = at(c, line_index);
      if (ch != ']' && ch != ',' && ch != '[') return;
      int32_t ci = ch == ']' ? 0 : L.curr_index(level) + 1;
      const Pos lend = L.level_end(level);
      const uint64_t *lvl = level_words(c, level);
      steps = 0;
      bool fail = false;
      for (;;) {
        if (++steps > max_steps) {
          fail = true;
          break;
        }
        if (ci < target) {
          --line_index;
          line_index = prev_struct(c, lbc, Pos(0), line_index, lvl);
          if (at(c, line_index) == ',' || ci + 1 == target) {
            ++ci;
            continue;
          }
          fail = true;
          break;
        }
        if (ci > target) {
          ++line_index;
          line_index = next_struct(c, lbc, lend, line_index, lvl);
          --ci;
          continue;
        }
        break;
      }
      L.curr_index(level) = ci;
      if (fail) return;
      ++line_index;
      break;
    }
    case OP_MARK_POSITION:
      if (marked + 1 >= kMaxQueryLevels) return;
      ++marked;
      marked_pos[marked] = line_index;
      marked_level[marked] = level;
      break;
    case OP_RESET_POSITION:
      if (marked < 0) return;
      line_index = marked_pos[marked];
      level = marked_level[marked];
      --marked;
      for (int i = level + 1; i < L.nlev; ++i) {
        if (i < 0) continue;
        if (L.level_end(i) == -1) break;
        L.level_end(i) = -1;
      }
      break;
    case OP_EXPRESSION_STRING_EQUALS: {
      key_len = read_varint(c, qp);
      key_pos = qp;
      qp += key_len;
      if (key_len < 0 || !LEVEL_OK(level)) return;
      const Pos lend = L.level_end(level);
      while (at(c, line_index) == ' ' && line_index < lend) ++line_index;
      Pos string_end = lend - 1;
      while (line_index < string_end && at(c, string_end) == ' ') --string_end;
      if (string_end - line_index + 1 != key_len) return;
      for (int i = 0; i < key_len; ++i) {
        if (ir_at(c, key_pos + i) != at(c, Pos(line_index + i))) return;
      }
      break;
    }
    case OP_NUMBER_COMPARE: {
      if constexpr (!kExt) return;
      const int cmp = ir_at(c, qp++);
      const int lit_len = read_varint(c, qp);
      const int lit_pos = qp;
      qp += lit_len;
      if (lit_len < 0 || lit_pos + lit_len > c.ir_len || !LEVEL_OK(level)) return;
      const Pos lend = L.level_end(level);
      while (at(c, line_index) == ' ' && line_index < lend) ++line_index;
      Pos value_end = lend - 1;
      while (line_index < value_end && at(c, value_end) == ' ') --value_end;
      if (line_index < 0 || value_end >= c.n || value_end < line_index) return;
      const Pos v0 = line_index;
      auto gv = [&](int64_t i) { return at(c, Pos(v0 + i)); };
      auto gl = [&](int64_t i) { return ir_at(c, int(lit_pos + i)); };
      DecNum v, lit;
      if (!dec_parse(gv, int64_t(value_end - line_index) + 1, v)) return;
      if (!dec_parse(gl, int64_t(lit_len), lit)) return;
      if (!cmp_holds(cmp, dec_cmp(gv, v, gl, lit))) return;
      break;
    }
    case OP_DESCEND_KEY: {
      if constexpr (!kExt) return;
      key_len = read_varint(c, qp);
      key_pos = qp;
      qp += key_len;
      if (key_len < 0 || !LEVEL_OK(level)) return;
      // every member named key inside the current value, at any level the
      // index holds, in document order (by the position of its ':')
      const Pos hi = L.level_end(level);
      for (Pos w = line_index >> 6; w * 64 < hi && w < c.W; ++w) {
        uint64_t cand = 0;
        for (int l = level; l + c.base < c.levels; ++l) {
          const uint64_t *lw = level_words(c, l);
          if (lw != nullptr) cand |= lw[w];
        }
        const Pos base = w * 64;
        if (line_index > base) cand &= ~0ull << (line_index - base);
        if (hi - base < 64) cand &= (1ull << (hi - base)) - 1ull;
        while (cand != 0) {
          const Pos p = base + Pos(__ffsll(static_cast<long long>(cand)) - 1);
          cand &= cand - 1;
          if (at(c, p) != ':') continue;
          int lv = level;
          while (lv + c.base < c.levels &&
                 ((level_words(c, lv)[w] >> (p - base)) & 1ull) == 0ull)
            ++lv;
          if (!key_at_colon(c, sc, line_start, p, key_pos, key_len)) continue;
          const Pos vend = next_struct(c, lbc, hi, Pos(p + 1), level_words(c, lv));
          Pos vs = p + 1;
          while (at(c, vs) == ' ' && vs < vend) ++vs;
          Pos ve = vend;
          while (ve > vs && at(c, ve - 1) == ' ') --ve;
          if (stored < num_results) {
            out[2 * stored] = OutT(vs);
            out[2 * stored + 1] = OutT(ve);
          } else {
            raise_status(c, kQueryStatusOverflow);
          }
          ++stored;
        }
      }
      break;
    }
    case OP_EXPECT_AT_MOST: {
      if constexpr (!kExt) return;
      const int limit = read_varint(c, qp);
      if (limit < 0 || !LEVEL_OK(level)) return;
      if (limit == 0 || at(c, line_index) != '[') break;
      // K commas at this level before the closing bracket: K+1 elements
      const Pos lend = L.level_end(level);
      const uint64_t *lvl = level_words(c, level);
      Pos p = line_index;
      int commas = 0;
      steps = 0;
      while (commas < limit) {
        if (++steps > max_steps) break;
        p = next_struct(c, lbc, lend, Pos(p + 1), lvl);
        if (at(c, p) != ',') break;
        ++commas;
      }
      if (commas >= limit) raise_status(c, kQueryStatusOverflow);
      break;
    }
    case OP_EXPECT_FOLLOWING: {
      if constexpr (!kExt) return;
      const int need = read_varint(c, qp);
      if (need < 0 || !LEVEL_OK(level)) return;
      // The element must exist (an empty array has no element 0) and be
      // followed by `need` commas at this level before the closing bracket;
      // otherwise it is among the last `need` (and so is every later one):
      // the record is done.
      const Pos lend = L.level_end(level);
      const uint64_t *lvl = level_words(c, level);
      Pos p = line_index;
      while (p < lend && at(c, p) == ' ') ++p;
      if (at(c, p) == ']') return;
      p = line_index - 1;
      int commas = 0;
      steps = 0;
      while (commas < need) {
        if (++steps > max_steps) return;
        p = next_struct(c, lbc, lend, Pos(p + 1), lvl);
        if (at(c, p) != ',') return;
        ++commas;
      }
      break;
    }
    default:
      break;
    }
    if (qp > c.ir_len + 1) return;
  }
#undef LEVEL_OK
}

// kExt: the IR holds extension opcodes (numeric filters, "..name", the
// element checks of "[*]" and the open slices); reference-syntax IR runs the
// variant without them.
template <typename Pos, typename OutT, bool kExt>
__global__ void __launch_bounds__(256)
    query_kernel(const QueryLaunch q, const __grid_constant__ IrBlob ir, OutT *out, int nlev) {
  __shared__ uint8_t s_ir[kMaxQueryIrBytes];
  extern __shared__ __align__(8) uint8_t s_levels[];  // Pos[nlev][bdim], int32[nlev][bdim]
  for (int i = threadIdx.x; i < q.ir_len; i += blockDim.x) s_ir[i] = ir.bytes[i];
  __syncthreads();
  const Rec<Pos> c{q.in, Pos(q.n), q.S, q.LB, Pos(q.W), s_ir, q.ir_len, q.base_level,
                   q.num_levels, q.status};
  Pos *ends = reinterpret_cast<Pos *>(s_levels);
  int32_t *idx = reinterpret_cast<int32_t *>(ends + nlev * blockDim.x);
  const LevelState<Pos> L{ends + threadIdx.x, idx + threadIdx.x, int(blockDim.x), nlev};
  const int64_t stride = int64_t(blockDim.x) * gridDim.x;
  for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < q.num_lines;
       r += stride) {
    OutT *o = out + r * int64_t(q.num_results) * 2;
    for (int i = 0; i < 2 * q.num_results; ++i) o[i] = OutT(-1);
    const int64_t start = q.NL[r];
    const int64_t end = (r + 1 < q.num_lines) ? q.NL[r + 1] : q.n - 1;
    run_record<Pos, OutT, kExt>(c, L, Pos(start), Pos(end), q.num_results, o);
  }
}

// At most 48 registers (five 256-thread blocks per SM): the kernel waits on
// memory, and more resident warps hide more of it (measured 6 % faster on the
// c3 file table than at 64 registers; 40 registers was slower again).
template <bool kExt>
__global__ void __launch_bounds__(256, 5)
    batch_query_kernel(const BatchQueryLaunch q, const __grid_constant__ IrBlob ir, int nlev) {
  __shared__ uint8_t s_ir[kMaxQueryIrBytes];
  extern __shared__ __align__(8) uint8_t s_levels[];  // int32[nlev][bdim] x 2
  for (int i = threadIdx.x; i < kMaxQueryIrBytes; i += blockDim.x) s_ir[i] = ir.bytes[i];
  __syncthreads();
  int32_t *ends = reinterpret_cast<int32_t *>(s_levels);
  const LevelState<int32_t> L{ends + threadIdx.x, ends + nlev * blockDim.x + threadIdx.x,
                              int(blockDim.x), nlev};
  const uint64_t records = q.totals[kTotRecords];
  // Records go to warps 32 at a time from a counter, so a warp whose records
  // were quick takes more instead of every warp doing the same number of
  // rounds (the launch ends with its slowest warp); without a counter each
  // thread strides over the records.
  const bool fed = q.record_counter != nullptr;
  const uint64_t stride = uint64_t(blockDim.x) * gridDim.x;
  uint64_t r = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  for (;; r += stride) {
    if (fed) {
      unsigned long long base = 0;
      if ((threadIdx.x & 31u) == 0) base = atomicAdd(q.record_counter, 32ull);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (base >= records) break;
      r = base + (threadIdx.x & 31u);
      if (r >= records) continue;
    } else if (r >= records) {
      break;
    }
    uint32_t lo = 0, hi = q.num_files;  // file_info[lo].rec_off <= r
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (q.file_info[uint64_t(mid) * kFileInfoWords + kFiRecOff] <= r) lo = mid;
      else hi = mid;
    }
    const uint64_t *row = q.file_info + uint64_t(lo) * kFileInfoWords;
    const IndexFile F = q.files[lo];
    const BatchQueryGroup g = q.groups[row[kFiQuery] < uint64_t(q.num_groups) ? row[kFiQuery] : 0];
    const uint64_t i = r - row[kFiRecOff];
    const uint64_t lines = row[kFiLines];
    int32_t *o = q.out + row[kFiOutOff] + i * uint64_t(g.num_results) * 2u;
    for (int k = 0; k < 2 * g.num_results; ++k) o[k] = -1;
    if (F.n == 0) continue;
    const int64_t *nl = q.NL + row[kFiNlOff];
    const int64_t start = nl[i];
    const int64_t end = (i + 1 < lines) ? nl[i + 1] : int64_t(F.n) - 1;
    // batch files are below 2 GiB (int32 results): 32-bit positions
    const Rec<int32_t> c{q.in + F.in_off, int32_t(F.n), q.S + F.s_off, q.LB + F.lb_off,
                         int32_t((F.n + 63u) / 64u), s_ir + g.ir_off, g.ir_len, g.base_level,
                         F.levels, q.file_status ? q.file_status + lo : q.status};
    run_record<int32_t, int32_t, kExt>(c, L, int32_t(start), int32_t(end), g.num_results, o);
  }
}

}  // namespace

int query_ir_levels(const uint8_t *ir, int len) {
  // Follows the interpreter's level changes along the IR (it has no jumps;
  // reset returns to a marked level) to find the deepest level it can reach.
  int level = 0, deepest = 0, marked = 0;
  int marks[kMaxQueryLevels] = {};
  auto skip_varint = [&](int &p, int *value) {
    uint32_t v = 0, b = 0;
    int shift = 0;
    while (p < len && ((b = ir[p++]) & 0x80u) != 0 && shift <= 28) {
      v |= (b & 0x7Fu) << shift;
      shift += 7;
    }
    if (value != nullptr) *value = int(v | (shift <= 28 ? (b << shift) : 0u));
  };
  for (int p = 0; p < len;) {
    const uint8_t op = ir[p++];
    if (op == OP_END) break;
    int n = 0;
    switch (op) {
    case OP_MOVE_UP: --level; break;
    case OP_MOVE_DOWN: ++level; break;
    case OP_MOVE_TO_KEY:
    case OP_EXPRESSION_STRING_EQUALS:
      skip_varint(p, &n);
      if (n > 0) p += n;
      break;
    case OP_MOVE_TO_INDEX:
    case OP_MOVE_TO_INDEX_REVERSE:
    case OP_EXPECT_AT_MOST:
    case OP_EXPECT_FOLLOWING: skip_varint(p, nullptr); break;
    case OP_NUMBER_COMPARE:
      ++p;  // comparator
      skip_varint(p, &n);
      if (n > 0) p += n;
      break;
    case OP_DESCEND_KEY:
      skip_varint(p, &n);
      if (n > 0) p += n;
      break;
    case OP_MARK_POSITION:
      if (marked < kMaxQueryLevels) marks[marked++] = level;
      break;
    case OP_RESET_POSITION:
      if (marked > 0) level = marks[--marked];
      break;
    default: break;
    }
    if (level > deepest) deepest = level;
  }
  return deepest + 1 < kMaxQueryLevels ? deepest + 1 : kMaxQueryLevels;
}

bool query_ir_uses_extensions(const uint8_t *ir, int len) {
  auto skip_varint = [&](int &p) -> int {
    uint32_t v = 0, b = 0;
    int shift = 0;
    while (p < len && ((b = ir[p++]) & 0x80u) != 0 && shift <= 28) {
      v |= (b & 0x7Fu) << shift;
      shift += 7;
    }
    return int(v | (shift <= 28 ? (b << shift) : 0u));
  };
  for (int p = 0; p < len;) {
    const uint8_t op = ir[p++];
    switch (op) {
    case OP_END: return false;
    case OP_NUMBER_COMPARE:
    case OP_DESCEND_KEY:
    case OP_EXPECT_AT_MOST:
    case OP_EXPECT_FOLLOWING: return true;
    case OP_MOVE_TO_KEY:
    case OP_EXPRESSION_STRING_EQUALS: {
      const int n = skip_varint(p);
      if (n > 0) p += n;
      break;
    }
    case OP_MOVE_TO_INDEX:
    case OP_MOVE_TO_INDEX_REVERSE: skip_varint(p); break;
    default: break;
    }
  }
  return false;
}

cudaError_t batch_query_launch(const BatchQueryLaunch &q, const IrBlob &ir, int grid,
                               int block, cudaStream_t stream) {
  int nlev = 1;
  bool ext = false;
  for (int g = 0; g < q.num_groups; ++g) {
    const int l = query_ir_levels(ir.bytes + q.groups[g].ir_off, q.groups[g].ir_len);
    if (l > nlev) nlev = l;
    ext = ext || query_ir_uses_extensions(ir.bytes + q.groups[g].ir_off, q.groups[g].ir_len);
  }
  const size_t smem = size_t(nlev) * size_t(block) * 8u;
  if (q.record_counter != nullptr) {
    const cudaError_t e = cudaMemsetAsync(q.record_counter, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
  }
  if (ext) batch_query_kernel<true><<<grid, block, smem, stream>>>(q, ir, nlev);
  else batch_query_kernel<false><<<grid, block, smem, stream>>>(q, ir, nlev);
  return cudaGetLastError();
}

cudaError_t query_launch(const QueryLaunch &q, const IrBlob &ir, int grid,
                         int block, cudaStream_t stream) {
  if (q.num_lines <= 0 || q.n <= 0) return cudaSuccess;
  if (block <= 0) block = 256;
  if (block > 256) block = 256;
  if (grid <= 0) grid = int((q.num_lines + block - 1) / block);
  const int nlev = query_ir_levels(ir.bytes, q.ir_len);
  const bool ext = query_ir_uses_extensions(ir.bytes, q.ir_len);
  if (q.out64 != nullptr) {
    const size_t smem = size_t(nlev) * size_t(block) * 12u;
    if (ext) query_kernel<int64_t, int64_t, true><<<grid, block, smem, stream>>>(q, ir, q.out64, nlev);
    else query_kernel<int64_t, int64_t, false><<<grid, block, smem, stream>>>(q, ir, q.out64, nlev);
  } else {
    // int32 results imply a partition below 2 GiB: 32-bit positions
    const size_t smem = size_t(nlev) * size_t(block) * 8u;
    if (ext) query_kernel<int32_t, int32_t, true><<<grid, block, smem, stream>>>(q, ir, q.out32, nlev);
    else query_kernel<int32_t, int32_t, false><<<grid, block, smem, stream>>>(q, ir, q.out32, nlev);
  }
  return cudaGetLastError();
}

}  // namespace gpjb
