/*
 * CPU oracle for the GpJSON structural index and JSONPath query path.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arm of bench.py as the checker and the CPU
 * baseline.  The product library never links or calls it.
 *
 * The code below is a plain, byte-serial restatement of the reference
 * (Xinyu-Li-123/15418-project).  Each function names the reference lines it
 * follows; where the reference reads out of bounds on malformed input (its
 * release build compiles the asserts out), this restatement reads a 0 byte
 * instead, and says so at that spot.
 */
#include "gpjson_oracle.h"

#include <stdlib.h>
#include <string.h>

uint64_t orc_num_words(uint64_t n) { return (n + 63u) / 64u; }

/* tests/index/newline_index_test.cpp:27-35 (expected_newline_index) and
 * src/gpjson/index/sharemem_index_builder.cu:343-349 (num_lines = count + 1,
 * slot 0 = 0). */
uint64_t orc_newline_index(const uint8_t *in, uint64_t n, int64_t *out,
                           uint64_t cap) {
  uint64_t lines = 1;
  if (cap > 0) out[0] = 0;
  for (uint64_t i = 0; i < n; ++i) {
    if (in[i] == '\n') {
      if (lines < cap) out[lines] = (int64_t)i;
      ++lines;
    }
  }
  return lines;
}

/* Escape bitmap with the SHAREMEM word-local carry:
 *  - carry into word w is the parity of the trailing '\\' run inside word w-1
 *    only, read backward from its last in-file byte
 *    (src/gpjson/index/kernels/sharemem/uncombined/escape-carry-index.cu:95-164);
 *  - inside a word the state machine is "bit i = carry; carry = (byte=='\\')
 *    ? !carry : 0" (sharemem/uncombined/escape-index.cu:29-96).
 * An all-backslash word therefore passes carry 0 on, whatever came before. */
void orc_escape_index(const uint8_t *in, uint64_t n, uint64_t *E) {
  const uint64_t W = orc_num_words(n);
  for (uint64_t w = 0; w < W; ++w) {
    int carry = 0;
    if (w > 0) {
      /* backward read of word w-1 (always a full word) */
      const uint64_t base = (w - 1) * 64u;
      for (int b = 63; b >= 0; --b) {
        if (in[base + (uint64_t)b] == '\\') carry ^= 1;
        else break;
      }
    }
    uint64_t word = 0;
    const uint64_t base = w * 64u;
    for (int b = 0; b < 64 && base + (uint64_t)b < n; ++b) {
      if (carry) word |= (uint64_t)1 << b;
      carry = (in[base + (uint64_t)b] == '\\') ? !carry : 0;
    }
    E[w] = word;
  }
}

/* tests/index/string_index_test.cpp:28-34 counts the whole preceding run. */
void orc_escape_index_unbounded(const uint8_t *in, uint64_t n, uint64_t *E) {
  const uint64_t W = orc_num_words(n);
  memset(E, 0, W * sizeof(uint64_t));
  int carry = 0;
  for (uint64_t i = 0; i < n; ++i) {
    if (carry) E[i / 64u] |= (uint64_t)1 << (i % 64u);
    carry = (in[i] == '\\') ? !carry : 0;
  }
}

/* sharemem/quote-index.cu:29-95: Q bit = '"' and not escaped. */
void orc_quote_index(const uint8_t *in, uint64_t n, const uint64_t *E,
                     uint64_t *Q) {
  const uint64_t W = orc_num_words(n);
  for (uint64_t w = 0; w < W; ++w) {
    uint64_t word = 0;
    for (int b = 0; b < 64 && w * 64u + (uint64_t)b < n; ++b) {
      const uint64_t bit = (uint64_t)1 << b;
      if (in[w * 64u + (uint64_t)b] == '"' && (E[w] & bit) == 0) word |= bit;
    }
    Q[w] = word;
  }
}

/* sharemem_index_builder.cu:206-217 (inclusive XOR scan of per-word quote
 * parity) + sharemem/string-index.cu:3-31 (shift-xor cascade, then xor with
 * all ones when the carried parity is 1).  Bits past the end of the data keep
 * the in-string state at the end, exactly like the cascade does. */
void orc_string_index(const uint64_t *Q, uint64_t W, uint64_t *S) {
  uint64_t state = 0; /* 0 or all ones */
  for (uint64_t w = 0; w < W; ++w) {
    uint64_t x = Q[w];
    uint64_t out = 0;
    for (int b = 0; b < 64; ++b) {
      if ((x >> b) & 1u) state = ~state;
      out |= (state & 1u) << b;
    }
    S[w] = out;
  }
}

/* sharemem/leveled-bitmaps-carry-index.cu:202-277 + the char scan of
 * sharemem_index_builder.cu:281-301 + sharemem/leveled-bitmaps-index.cu:210-316
 * collapse into one running signed-char depth that starts at -1 and wraps
 * modulo 256.  Per byte outside strings:
 *   '{' '['  -> depth++, then set bit at level depth
 *   '}' ']'  -> set bit at level depth, then depth--
 *   ':' ','  -> set bit at level depth
 * and a bit is stored only when 0 <= depth < num_levels
 * (also tests/index/leveled_bitmap_index_test.cpp:57-92). */
void orc_leveled_bitmap_index(const uint8_t *in, uint64_t n, const uint64_t *S,
                              int num_levels, uint64_t *LB) {
  const uint64_t W = orc_num_words(n);
  memset(LB, 0, W * (uint64_t)num_levels * sizeof(uint64_t));
  int8_t level = -1;
  for (uint64_t i = 0; i < n; ++i) {
    const uint64_t w = i / 64u;
    const uint64_t bit = (uint64_t)1 << (i % 64u);
    if (S[w] & bit) continue;
    const uint8_t c = in[i];
    if (c == '{' || c == '[') {
      level = (int8_t)(level + 1);
      if (level >= 0 && level < num_levels) LB[(uint64_t)level * W + w] |= bit;
    } else if (c == '}' || c == ']') {
      if (level >= 0 && level < num_levels) LB[(uint64_t)level * W + w] |= bit;
      level = (int8_t)(level - 1);
    } else if (c == ':' || c == ',') {
      if (level >= 0 && level < num_levels) LB[(uint64_t)level * W + w] |= bit;
    }
  }
}

uint64_t orc_build_index(const uint8_t *in, uint64_t n, int num_levels,
                         uint64_t *E, uint64_t *Q, uint64_t *S, uint64_t *LB,
                         int64_t *NL, uint64_t nl_cap) {
  const uint64_t W = orc_num_words(n);
  uint64_t *e = E;
  uint64_t *tmp = 0;
  if (e == 0) {
    tmp = (uint64_t *)malloc((W ? W : 1) * sizeof(uint64_t));
    e = tmp;
  }
  /* Q goes into the S buffer when not requested, as the reference does
   * (sharemem_index_builder.cu:194-197); the scan below reads word w before
   * writing it, so it runs in place. */
  uint64_t *q = Q ? Q : S;
  orc_escape_index(in, n, e);
  orc_quote_index(in, n, e, q);
  orc_string_index(q, W, S);
  orc_leveled_bitmap_index(in, n, S, num_levels, LB);
  free(tmp);
  return orc_newline_index(in, n, NL, nl_cap);
}

/* ------------------------------------------------------------------------ */
/* Query interpreter: src/gpjson/query/kernels/orig/query.cu:144-454         */
/* ------------------------------------------------------------------------ */

enum {
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
  /* Extensions of this build (never emitted for the reference's syntax):
   * numeric filters, recursive descent to a member name, the element count
   * check of a bounded "[*]" or open slice, and the check that an element is
   * not among the last b of its array ("[a:-b]"). */
  OP_NUMBER_COMPARE = 0x0A,
  OP_DESCEND_KEY = 0x0B,
  OP_EXPECT_AT_MOST = 0x0C,
  OP_EXPECT_FOLLOWING = 0x0D
};
#define ORC_MAX_LEVELS 16 /* query.cu:20 MAX_NUM_LEVELS */

typedef struct {
  const uint8_t *in;
  int64_t n;
  const uint64_t *S;
  const uint64_t *LB;
  int64_t W;
  const uint8_t *ir;
  int64_t ir_len;
  int levels; /* levels held by LB */
  int base;   /* bitmap level of query level 0 */
  uint32_t status; /* ORC_STATUS_* bits raised by the records */
} qctx;

/* The reference indexes file[] without bounds checks; on well-formed JSON it
 * never leaves the partition.  Here a read outside [0, n) yields 0. */
static inline uint8_t at(const qctx *c, int64_t i) {
  return (i >= 0 && i < c->n) ? c->in[i] : 0;
}
static inline uint64_t word_at(const uint64_t *bm, int64_t W, int64_t i) {
  return (i >= 0 && i < W) ? bm[i] : 0;
}
static inline uint8_t ir_at(const qctx *c, int64_t i) {
  return (i >= 0 && i < c->ir_len) ? c->ir[i] : 0;
}

/* query.cu:34-37 */
static inline uint64_t mask_through_bit(int bit_offset) {
  return bit_offset == 63 ? ~(uint64_t)0 : (((uint64_t)1 << (bit_offset + 1)) - 1);
}

static inline int clz64(uint64_t x) { return __builtin_clzll(x); }
static inline int ffs64(uint64_t x) { return __builtin_ffsll((long long)x); }

/* query.cu:39-77 find_previous_bitmap_bit */
static int64_t find_previous_bitmap_bit(const uint64_t *bitmap, int64_t W,
                                        int64_t min_index, int64_t line_index) {
  if (line_index < min_index) return -1;
  int64_t word_index = line_index / 64;
  int64_t word_base = word_index * 64;
  uint64_t word = word_at(bitmap, W, word_index);
  word &= mask_through_bit((int)(line_index - word_base));
  while (word_base + 63 >= min_index) {
    uint64_t candidate = word;
    const int64_t first_bit = min_index - word_base;
    if (first_bit > 0) candidate &= ~mask_through_bit((int)(first_bit - 1));
    if (candidate != 0) return word_base + 63 - clz64(candidate);
    if (word_index == 0) break;
    --word_index;
    word_base -= 64;
    if (word_base + 63 < min_index) break;
    word = word_at(bitmap, W, word_index);
  }
  return -1;
}

/* query.cu:79-115 find_next_structural_char */
static int64_t find_next_structural_char(const qctx *c, int64_t level_end,
                                         int64_t line_index, int level) {
  if (line_index >= level_end) return level_end;
  if (level + c->base < 0 || level + c->base >= c->levels) return level_end;
  const uint64_t *lvl = c->LB + (uint64_t)c->W * (uint64_t)(level + c->base);
  int64_t word_index = line_index / 64;
  int64_t word_base = word_index * 64;
  uint64_t word = word_at(lvl, c->W, word_index);
  word &= ~(uint64_t)0 << (line_index - word_base);
  while (word_base <= level_end) {
    uint64_t candidate = word;
    const int64_t last_bit = level_end - word_base;
    if (last_bit < 63) candidate &= mask_through_bit((int)last_bit);
    if (candidate != 0) return word_base + ffs64(candidate) - 1;
    ++word_index;
    word_base += 64;
    if (word_base > level_end) break;
    word = word_at(lvl, c->W, word_index);
  }
  return level_end;
}

/* query.cu:117-128 find_previous_structural_char */
static int64_t find_previous_structural_char(const qctx *c, int64_t level_start,
                                             int64_t line_index, int level) {
  if (line_index <= level_start) return level_start;
  if (level + c->base < 0 || level + c->base >= c->levels) return level_start;
  const uint64_t *lvl = c->LB + (uint64_t)c->W * (uint64_t)(level + c->base);
  const int64_t s = find_previous_bitmap_bit(lvl, c->W, level_start, line_index);
  return s == -1 ? level_start : s;
}

/* query.cu:130-140 read_varint (LEB128).  Unsigned arithmetic reinterpreted
 * as int, as the reference's int result wraps; an operand longer than five
 * bytes (never produced by the compiler) reads as -1. */
static int read_varint(const qctx *c, int64_t *pos) {
  uint32_t value = 0, byte = 0;
  int shift = 0;
  while (((byte = ir_at(c, (*pos)++)) & 0x80u) != 0) {
    value |= (byte & 0x7Fu) << shift;
    shift += 7;
    if (shift > 28) return -1;
  }
  return (int)(value | (byte << shift));
}


/* ---- Extensions of this build (the reference rejects these queries) ----
 *
 * Numeric filter [?(@ <op> <number>)]: the value at the current position,
 * trimmed of ' ' like EXPRESSION_STRING_EQUALS trims it (query.cu:414-441),
 * must be a JSON number (RFC 8259 grammar) and compare as <op> against the
 * literal; otherwise the record is abandoned.  The comparison is exact
 * decimal arithmetic on the digit strings (no floating point): a number is
 * 0.d1d2d3... x 10^E with d1 != 0, or zero; exponents saturate at +-10^15. */
typedef struct {
  int neg, zero;
  int64_t E;       /* decimal exponent of 0.d1d2... */
  int64_t nd;      /* significant digits (from the first nonzero digit) */
  int64_t first;   /* index of the first significant digit in int+frac digits */
  int64_t int_len; /* digits before the point */
  const uint8_t *ip, *fp; /* integer and fraction digits */
} orc_num;

#define ORC_EXP_LIMIT 1000000000000000LL

static int is_digit(uint8_t c) { return c >= '0' && c <= '9'; }

static uint8_t num_digit(const orc_num *x, int64_t k) { /* k-th of int+frac digits */
  return k < x->int_len ? x->ip[k] : x->fp[k - x->int_len];
}

/* Parses p[0..len) as one JSON number; 0 if it is not one. */
static int num_parse(const uint8_t *p, int64_t len, orc_num *o) {
  int64_t i = 0;
  o->neg = 0;
  if (i < len && p[i] == '-') {
    o->neg = 1;
    ++i;
  }
  if (i >= len) return 0;
  const int64_t int_start = i;
  if (p[i] == '0') {
    ++i;
  } else if (p[i] >= '1' && p[i] <= '9') {
    while (i < len && is_digit(p[i])) ++i;
  } else {
    return 0;
  }
  o->ip = p + int_start;
  o->int_len = i - int_start;
  int64_t frac_len = 0;
  o->fp = p + i;
  if (i < len && p[i] == '.') {
    ++i;
    o->fp = p + i;
    while (i < len && is_digit(p[i])) ++i;
    frac_len = (p + i) - o->fp;
    if (frac_len == 0) return 0;
  }
  int64_t ex = 0;
  if (i < len && (p[i] == 'e' || p[i] == 'E')) {
    ++i;
    int eneg = 0;
    if (i < len && (p[i] == '+' || p[i] == '-')) {
      eneg = p[i] == '-';
      ++i;
    }
    const int64_t es = i;
    while (i < len && is_digit(p[i])) {
      if (ex < ORC_EXP_LIMIT) ex = ex * 10 + (p[i] - '0');
      ++i;
    }
    if (i == es) return 0;
    if (ex > ORC_EXP_LIMIT) ex = ORC_EXP_LIMIT;
    if (eneg) ex = -ex;
  }
  if (i != len) return 0;
  const int64_t total = o->int_len + frac_len;
  int64_t z = 0;
  while (z < total && num_digit(o, z) == '0') ++z;
  o->zero = z == total;
  o->first = z;
  o->nd = total - z;
  o->E = o->int_len - z + ex;
  return 1;
}

/* -1, 0, 1 as a <, ==, > b. */
static int num_cmp(const orc_num *a, const orc_num *b) {
  const int sa = a->zero ? 0 : (a->neg ? -1 : 1);
  const int sb = b->zero ? 0 : (b->neg ? -1 : 1);
  if (sa != sb) return sa < sb ? -1 : 1;
  if (sa == 0) return 0;
  int mag = 0;
  if (a->E != b->E) {
    mag = a->E > b->E ? 1 : -1;
  } else {
    const int64_t n = a->nd > b->nd ? a->nd : b->nd;
    for (int64_t k = 0; k < n && mag == 0; ++k) {
      const uint8_t da = k < a->nd ? num_digit(a, a->first + k) : '0';
      const uint8_t db = k < b->nd ? num_digit(b, b->first + k) : '0';
      if (da != db) mag = da > db ? 1 : -1;
    }
  }
  return sa > 0 ? mag : -mag;
}

/* Comparators of OP_NUMBER_COMPARE. */
enum { CMP_EQ = 0, CMP_NE = 1, CMP_LT = 2, CMP_LE = 3, CMP_GT = 4, CMP_GE = 5 };

static int cmp_holds(int op, int r) {
  switch (op) {
  case CMP_EQ: return r == 0;
  case CMP_NE: return r != 0;
  case CMP_LT: return r < 0;
  case CMP_LE: return r <= 0;
  case CMP_GT: return r > 0;
  case CMP_GE: return r >= 0;
  default: return 0;
  }
}

static int level_bit(const qctx *c, int level, int64_t pos) {
  const int l = level + c->base;
  if (l < 0 || l >= c->levels || pos < 0 || pos / 64 >= c->W) return 0;
  return (int)((c->LB[(uint64_t)c->W * (uint64_t)l + (uint64_t)(pos / 64)] >> (pos % 64)) & 1u);
}

/* Does the string before the ':' at `colon` equal the key (the test of
 * MOVE_TO_KEY, query.cu:254-302)? */
static int key_matches(const qctx *c, int64_t line_start, int64_t colon, int64_t key_pos,
                       int key_len) {
  const int64_t string_end = find_previous_bitmap_bit(c->S, c->W, line_start + 1, colon - 1);
  const int64_t string_start = string_end - key_len;
  if (string_start < line_start || at(c, string_start) != '"') return 0;
  for (int i = 0; i < key_len; ++i)
    if (ir_at(c, key_pos + i) != at(c, string_start + i + 1)) return 0;
  return 1;
}

/* One record: query.cu:150-451.  out points at this record's 2*num_results
 * slots, already filled with -1. */
static void query_record(qctx *c, int64_t line_start, int64_t line_end,
                         int num_results, int64_t *out) {
  if (line_start < 0 || line_start >= c->n || line_end < 0) return;
  if (line_end >= c->n) line_end = c->n - 1;
  while (line_end > line_start && at(c, line_end) != '}') --line_end;
  while (line_start < line_end && at(c, line_start) != '{') ++line_start;
  if (line_start == line_end) return;

  int64_t line_index = line_start;
  int current_level = 0;
  int64_t query_pos = 0;
  /* Step bound of one search loop (not in the reference): on well-formed JSON
   * each step lands on a new structural character of the record, so it is
   * never reached; on malformed input the reference's loops can revisit one
   * character forever, and the record is abandoned instead. */
  const int64_t max_steps = (line_end - line_start) + 2;
  int64_t steps = 0;
  int64_t level_end[ORC_MAX_LEVELS];
  level_end[0] = line_end;
  for (int i = 1; i < ORC_MAX_LEVELS; ++i) level_end[i] = -1;
  int64_t marked_pos[ORC_MAX_LEVELS];
  int marked_pos_level[ORC_MAX_LEVELS];
  int marked_pos_index = -1;
  int num_results_index = 0;
  int64_t key_pos = 0;
  int key_len = 0;
  int target_index = 0;
  int64_t curr_index[ORC_MAX_LEVELS];
  for (int i = 0; i < ORC_MAX_LEVELS; ++i) curr_index[i] = -1;

/* The reference has no guard for these; the compiler never emits IR that
 * reaches them.  Leaving the record keeps the restatement memory safe. */
#define LEVEL_OK(l) ((l) >= 0 && (l) < ORC_MAX_LEVELS)
/* Where the reference's kernel has a device assert, the oracle records in
 * the status that the condition failed (ORC_STATUS_REF_ASSERT) and carries
 * on: test harnesses check it before handing an input to the reference. */
#define REF_ASSERT(cond)                                                     \
  do {                                                                       \
    if (!(cond)) c->status |= ORC_STATUS_REF_ASSERT;                         \
  } while (0)

  for (;;) {
    const uint8_t op = ir_at(c, query_pos++);
    switch (op) {
    case OP_END:
      return;

    case OP_STORE_RESULT: { /* query.cu:213-231 */
      if (!LEVEL_OK(current_level)) return;
      int64_t end_str = level_end[current_level];
      while (at(c, line_index) == ' ' && line_index < level_end[current_level])
        ++line_index;
      while (end_str > line_index && at(c, end_str - 1) == ' ') --end_str;
      REF_ASSERT(line_index <= end_str); /* query.cu:230 */
      if (num_results_index < num_results) {
        out[num_results_index * 2] = line_index;
        out[num_results_index * 2 + 1] = end_str;
      } else {
        c->status |= ORC_STATUS_OVERFLOW; /* only extension queries get here */
      }
      ++num_results_index;
      break;
    }

    case OP_MOVE_UP: /* query.cu:233-237 */
      if (!LEVEL_OK(current_level)) return;
      line_index = level_end[current_level];
      level_end[current_level] = -1;
      --current_level;
      break;

    case OP_MOVE_DOWN: /* query.cu:239-252 */
      ++current_level;
      if (!LEVEL_OK(current_level) || current_level < 1) return;
      if (level_end[current_level] == -1) {
        level_end[current_level] = find_next_structural_char(
            c, level_end[current_level - 1], line_index + 1, current_level - 1);
        while (at(c, line_index) == ' ') ++line_index;
      }
      break;

    case OP_MOVE_TO_KEY: /* query.cu:254-302 */
      key_len = read_varint(c, &query_pos);
      key_pos = query_pos;
      query_pos += key_len;
      if (key_len < 0 || !LEVEL_OK(current_level)) return;
      if (at(c, line_index) == '{') {
        steps = 0;
        for (;;) { /* search_key */
          if (++steps > max_steps) return;
          ++line_index;
          line_index = find_next_structural_char(c, level_end[current_level],
                                                 line_index, current_level);
          REF_ASSERT(at(c, line_index) == ':' || at(c, line_index) == '}'); /* query.cu:265 */
          if (at(c, line_index) == ':') {
            const int64_t string_end = find_previous_bitmap_bit(
                c->S, c->W, line_start + 1, line_index - 1);
            const int64_t string_start = string_end - key_len;
            int mismatch = 0;
            if (string_start < line_start || at(c, string_start) != '"') {
              mismatch = 1;
            } else {
              for (int i = 0; i < key_len; ++i) {
                if (ir_at(c, key_pos + i) != at(c, string_start + i + 1)) {
                  mismatch = 1;
                  break;
                }
              }
            }
            if (mismatch) {
              ++line_index;
              line_index = find_next_structural_char(
                  c, level_end[current_level], line_index, current_level);
              /* query.cu:276, 290 */
              REF_ASSERT(at(c, line_index) == ',' || at(c, line_index) == '}');
              if (at(c, line_index) == '}') return;
              continue; /* goto search_key */
            }
          }
          break;
        }
        ++line_index;
      } else {
        return;
      }
      break;

    case OP_MOVE_TO_INDEX: /* query.cu:304-346 */
      target_index = read_varint(c, &query_pos);
      if (!LEVEL_OK(current_level)) return;
      {
        const uint8_t ch = at(c, line_index);
        if (ch == '[' || ch == ',' || ch == ']') {
          if (ch == '[') curr_index[current_level] = 0;
          else ++curr_index[current_level];
          steps = 0;
          for (;;) { /* search_index */
            if (++steps > max_steps) return;
            if (curr_index[current_level] < target_index) {
              ++line_index;
              line_index = find_next_structural_char(
                  c, level_end[current_level], line_index, current_level);
              /* query.cu:321 */
              REF_ASSERT(at(c, line_index) == ',' || at(c, line_index) == ']');
              if (at(c, line_index) == ',') {
                ++curr_index[current_level];
                continue;
              }
              return;
            }
            if (curr_index[current_level] > target_index) {
              --line_index;
              line_index =
                  find_previous_structural_char(c, 0, line_index, current_level);
              /* query.cu:334 */
              REF_ASSERT(at(c, line_index) == ',' || at(c, line_index) == '[');
              --curr_index[current_level];
              continue;
            }
            break;
          }
          if (at(c, line_index) == ']') return;
          ++line_index;
        } else {
          return;
        }
      }
      break;

    case OP_MOVE_TO_INDEX_REVERSE: /* query.cu:348-392 */
      target_index = read_varint(c, &query_pos);
      if (!LEVEL_OK(current_level)) return;
      line_index = level_end[current_level] - 1;
      while (at(c, line_index) == ' ') --line_index;
      {
        const uint8_t ch = at(c, line_index);
        if (ch == ']' || ch == ',' || ch == '[') {
          if (ch == ']') curr_index[current_level] = 0;
          else ++curr_index[current_level];
          steps = 0;
          for (;;) { /* search_index_reverse */
            if (++steps > max_steps) return;
            if (curr_index[current_level] < target_index) {
              --line_index;
              line_index =
                  find_previous_structural_char(c, 0, line_index, current_level);
              /* query.cu:370 */
              REF_ASSERT(at(c, line_index) == ',' || at(c, line_index) == '[');
              if (at(c, line_index) == ',' ||
                  curr_index[current_level] + 1 == target_index) {
                ++curr_index[current_level];
                continue;
              }
              return;
            }
            if (curr_index[current_level] > target_index) {
              ++line_index;
              line_index = find_next_structural_char(
                  c, level_end[current_level], line_index, current_level);
              /* query.cu:384 */
              REF_ASSERT(at(c, line_index) == ',' || at(c, line_index) == ']');
              --curr_index[current_level];
              continue;
            }
            break;
          }
          ++line_index;
        } else {
          return;
        }
      }
      break;

    case OP_MARK_POSITION: /* query.cu:394-399 */
      if (marked_pos_index + 1 >= ORC_MAX_LEVELS) return;
      ++marked_pos_index;
      marked_pos[marked_pos_index] = line_index;
      marked_pos_level[marked_pos_index] = current_level;
      break;

    case OP_RESET_POSITION: /* query.cu:401-412 */
      if (marked_pos_index < 0) return;
      line_index = marked_pos[marked_pos_index];
      current_level = marked_pos_level[marked_pos_index];
      --marked_pos_index;
      for (int i = current_level + 1; i < ORC_MAX_LEVELS; ++i) {
        if (i < 0) continue;
        if (level_end[i] == -1) break;
        level_end[i] = -1;
      }
      break;

    case OP_EXPRESSION_STRING_EQUALS: /* query.cu:414-441 */
      key_len = read_varint(c, &query_pos);
      key_pos = query_pos;
      query_pos += key_len;
      if (key_len < 0 || !LEVEL_OK(current_level)) return;
      while (at(c, line_index) == ' ' && line_index < level_end[current_level])
        ++line_index;
      {
        int64_t string_end = level_end[current_level] - 1;
        while (line_index < string_end && at(c, string_end) == ' ') --string_end;
        /* query.cu:430: a string filter on a value that is not a string */
        REF_ASSERT(at(c, line_index) == '"' && at(c, string_end) == '"');
        const int64_t string_length = string_end - line_index + 1;
        if (string_length != key_len) return;
        for (int i = 0; i < key_len; ++i) {
          if (ir_at(c, key_pos + i) != at(c, line_index + i)) return;
        }
      }
      break;

    case OP_NUMBER_COMPARE: { /* extension: numeric filter */
      const int cmp = ir_at(c, query_pos++);
      const int lit_len = read_varint(c, &query_pos);
      const int64_t lit_pos = query_pos;
      query_pos += lit_len;
      if (lit_len < 0 || lit_pos + lit_len > c->ir_len || !LEVEL_OK(current_level)) return;
      while (at(c, line_index) == ' ' && line_index < level_end[current_level]) ++line_index;
      int64_t value_end = level_end[current_level] - 1;
      while (line_index < value_end && at(c, value_end) == ' ') --value_end;
      if (line_index < 0 || value_end >= c->n || value_end < line_index) return;
      orc_num v, lit;
      if (!num_parse(c->in + line_index, value_end - line_index + 1, &v)) return;
      if (!num_parse(c->ir + lit_pos, lit_len, &lit)) return;
      if (!cmp_holds(cmp, num_cmp(&v, &lit))) return;
      break;
    }

    case OP_DESCEND_KEY: { /* extension: "..name" as the last step */
      key_len = read_varint(c, &query_pos);
      key_pos = query_pos;
      query_pos += key_len;
      if (key_len < 0 || !LEVEL_OK(current_level)) return;
      const int64_t hi = level_end[current_level];
      /* every member named key inside the current value, at any level the
       * index holds, in document order (by the position of its ':') */
      for (int64_t p = line_index; p < hi; ++p) {
        if (at(c, p) != ':') continue;
        int lv = -1;
        for (int l = current_level; l + c->base < c->levels; ++l) {
          if (level_bit(c, l, p)) {
            lv = l;
            break;
          }
        }
        if (lv < 0 || !key_matches(c, line_start, p, key_pos, key_len)) continue;
        const int64_t vend = find_next_structural_char(c, hi, p + 1, lv);
        int64_t vs = p + 1;
        while (at(c, vs) == ' ' && vs < vend) ++vs;
        int64_t ve = vend;
        while (ve > vs && at(c, ve - 1) == ' ') --ve;
        if (num_results_index < num_results) {
          out[num_results_index * 2] = vs;
          out[num_results_index * 2 + 1] = ve;
        } else {
          c->status |= ORC_STATUS_OVERFLOW;
        }
        ++num_results_index;
      }
      break;
    }

    case OP_EXPECT_AT_MOST: { /* extension: "[*]" bounded to K elements */
      const int limit = read_varint(c, &query_pos);
      if (limit < 0 || !LEVEL_OK(current_level)) return;
      if (limit == 0 || at(c, line_index) != '[') break;
      /* K commas at this level before the closing bracket: K+1 elements */
      int64_t p = line_index;
      int commas = 0;
      steps = 0;
      while (commas < limit) {
        if (++steps > max_steps) break;
        p = find_next_structural_char(c, level_end[current_level], p + 1, current_level);
        if (at(c, p) != ',') break;
        ++commas;
      }
      if (limit > 0 && commas >= limit) c->status |= ORC_STATUS_OVERFLOW;
      break;
    }

    case OP_EXPECT_FOLLOWING: { /* extension: "[a:-b]", after MOVE_TO_INDEX */
      const int need = read_varint(c, &query_pos);
      if (need < 0 || !LEVEL_OK(current_level)) return;
      /* The element must exist (an empty array has no element 0) and be
       * followed by `need` commas at this level before the closing bracket;
       * otherwise it is among the last `need` (and so is every later one):
       * the record is done. */
      int64_t p = line_index;
      while (p < level_end[current_level] && at(c, p) == ' ') ++p;
      if (at(c, p) == ']') return;
      p = line_index - 1;
      int commas = 0;
      steps = 0;
      while (commas < need) {
        if (++steps > max_steps) return;
        p = find_next_structural_char(c, level_end[current_level], p + 1, current_level);
        if (at(c, p) != ',') return;
        ++commas;
      }
      break;
    }

    default: /* the reference asserts; release builds fall through */
      break;
    }
    if (query_pos > c->ir_len + 1) return; /* ran off the IR */
  }
#undef LEVEL_OK
}

int orc_query(const uint8_t *in, uint64_t n, const int64_t *NL,
              uint64_t num_lines, const uint64_t *S, const uint64_t *LB,
              uint64_t W, int num_levels, int base_level, const uint8_t *ir,
              uint64_t ir_len, int num_results, int64_t *out) {
  return orc_query_status(in, n, NL, num_lines, S, LB, W, num_levels, base_level, ir, ir_len,
                          num_results, out, NULL);
}

int orc_query_status(const uint8_t *in, uint64_t n, const int64_t *NL,
                     uint64_t num_lines, const uint64_t *S, const uint64_t *LB,
                     uint64_t W, int num_levels, int base_level, const uint8_t *ir,
                     uint64_t ir_len, int num_results, int64_t *out, uint32_t *status) {
  qctx c = {in, (int64_t)n, S, LB, (int64_t)W, ir, (int64_t)ir_len, num_levels, base_level, 0u};
  for (uint64_t r = 0; r < num_lines; ++r) {
    int64_t *o = out + r * (uint64_t)num_results * 2u;
    for (int i = 0; i < 2 * num_results; ++i) o[i] = -1;
    if (n == 0) continue;
    const int64_t line_start = NL[r];
    const int64_t line_end = (r + 1 < num_lines) ? NL[r + 1] : (int64_t)n - 1;
    query_record(&c, line_start, line_end, num_results, o);
  }
  if (status != NULL) *status = c.status;
  return 0;
}
