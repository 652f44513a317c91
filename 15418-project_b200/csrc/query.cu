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
};

// Last bitmap word read, per thread: consecutive searches of a record mostly
// start in the word the previous search ended in.
struct WordCache {
  const uint64_t *bm = nullptr;
  int64_t idx = -1;
  uint64_t val = 0;
};

struct Rec {
  const uint8_t *in;
  int64_t n;
  const uint64_t *S;
  const uint64_t *LB;
  int64_t W;
  const uint8_t *ir;  // shared memory
  int ir_len;
  int base;    // bitmap level of query level 0
  int levels;  // levels present in LB
};

// The reference reads file[] unguarded; well-formed JSON never leaves the
// partition.  Out-of-range reads return 0 here.
__device__ __forceinline__ uint8_t at(const Rec &c, int64_t i) {
  return (i >= 0 && i < c.n) ? c.in[i] : uint8_t(0);
}
__device__ __forceinline__ uint64_t word_at(const uint64_t *bm, int64_t W,
                                            int64_t i) {
  return (i >= 0 && i < W) ? bm[i] : 0ull;
}
__device__ __forceinline__ uint8_t ir_at(const Rec &c, int64_t i) {
  return (i >= 0 && i < c.ir_len) ? c.ir[i] : uint8_t(0);
}

__device__ __forceinline__ uint64_t cached_word(WordCache &wc, const uint64_t *bm, int64_t W,
                                                int64_t i) {
  if (wc.bm == bm && wc.idx == i) return wc.val;
  const uint64_t v = word_at(bm, W, i);
  wc.bm = bm;
  wc.idx = i;
  wc.val = v;
  return v;
}

__device__ __forceinline__ uint64_t mask_through_bit(int b) {
  return b == 63 ? ~0ull : ((1ull << (b + 1)) - 1ull);
}

// query.cu:39-77
__device__ int64_t prev_bit(WordCache &wc, const uint64_t *bm, int64_t W, int64_t min_index,
                            int64_t line_index) {
  if (line_index < min_index) return -1;
  int64_t wi = line_index >> 6;
  int64_t base = wi * 64;
  uint64_t word = cached_word(wc, bm, W, wi) & mask_through_bit(int(line_index - base));
  while (base + 63 >= min_index) {
    uint64_t cand = word;
    const int64_t first = min_index - base;
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

// query.cu:79-115
__device__ int64_t next_struct(const Rec &c, WordCache &wc, int64_t level_end,
                               int64_t line_index, int level) {
  if (line_index >= level_end) return level_end;
  // a level the index does not hold has no structural characters
  if (level + c.base < 0 || level + c.base >= c.levels) return level_end;
  const uint64_t *lvl = c.LB + uint64_t(c.W) * uint64_t(level + c.base);
  int64_t wi = line_index >> 6;
  int64_t base = wi * 64;
  uint64_t word = cached_word(wc, lvl, c.W, wi) & (~0ull << (line_index - base));
  while (base <= level_end) {
    uint64_t cand = word;
    const int64_t last = level_end - base;
    if (last < 63) cand &= mask_through_bit(int(last));
    if (cand != 0) return base + __ffsll(static_cast<long long>(cand)) - 1;
    ++wi;
    base += 64;
    if (base > level_end) break;
    word = cached_word(wc, lvl, c.W, wi);
  }
  return level_end;
}

// query.cu:117-128
__device__ int64_t prev_struct(const Rec &c, WordCache &wc, int64_t level_start,
                               int64_t line_index, int level) {
  if (line_index <= level_start) return level_start;
  if (level + c.base < 0 || level + c.base >= c.levels) return level_start;
  const uint64_t *lvl = c.LB + uint64_t(c.W) * uint64_t(level + c.base);
  const int64_t s = prev_bit(wc, lvl, c.W, level_start, line_index);
  return s == -1 ? level_start : s;
}

// query.cu:130-140 (LEB128).  Unsigned arithmetic reinterpreted as int, as
// the reference's int result wraps; an operand longer than five bytes (never
// produced by the compiler) reads as -1.
__device__ int read_varint(const Rec &c, int64_t &pos) {
  uint32_t value = 0, byte = 0;
  int shift = 0;
  while (((byte = ir_at(c, pos++)) & 0x80u) != 0) {
    value |= (byte & 0x7Fu) << shift;
    shift += 7;
    if (shift > 28) return -1;
  }
  return int(value | (byte << shift));
}

template <typename OutT>
__device__ void run_record(const Rec &c, int64_t line_start, int64_t line_end,
                           int num_results, OutT *out) {
  if (line_start < 0 || line_start >= c.n || line_end < 0) return;
  if (line_end >= c.n) line_end = c.n - 1;
  while (line_end > line_start && at(c, line_end) != '}') --line_end;
  while (line_start < line_end && at(c, line_start) != '{') ++line_start;
  if (line_start == line_end) return;

  int64_t line_index = line_start;
  int level = 0;
  int64_t qp = 0;
  // Step bound of one search loop.  On well-formed JSON every step lands on a
  // new structural character of the record, so the bound is never reached;
  // on malformed input the reference's loops can revisit the same character
  // forever, and the record is abandoned instead.
  const int64_t max_steps = (line_end - line_start) + 2;
  int64_t steps = 0;
  WordCache lbc, sc;  // leveled-bitmap and string-mask words
  int64_t level_end[kMaxQueryLevels];
  level_end[0] = line_end;
#pragma unroll
  for (int i = 1; i < kMaxQueryLevels; ++i) level_end[i] = -1;
  int64_t marked_pos[kMaxQueryLevels];
  int marked_level[kMaxQueryLevels];
  int marked = -1;
  int stored = 0;
  int64_t key_pos = 0;
  int key_len = 0;
  int target = 0;
  int64_t curr_index[kMaxQueryLevels];
#pragma unroll
  for (int i = 0; i < kMaxQueryLevels; ++i) curr_index[i] = -1;

#define LEVEL_OK(l) ((l) >= 0 && (l) < kMaxQueryLevels)
  for (;;) {
    const uint8_t op = ir_at(c, qp++);
    switch (op) {
    case OP_END:
      return;
    case OP_STORE_RESULT: {
      if (!LEVEL_OK(level)) return;
      int64_t end_str = level_end[level];
      while (at(c, line_index) == ' ' && line_index < level_end[level]) ++line_index;
      while (end_str > line_index && at(c, end_str - 1) == ' ') --end_str;
      if (stored < num_results) {
        out[2 * stored] = OutT(line_index);
        out[2 * stored + 1] = OutT(end_str);
      }
      ++stored;
      break;
    }
    case OP_MOVE_UP:
      if (!LEVEL_OK(level)) return;
      line_index = level_end[level];
      level_end[level] = -1;
      --level;
      break;
    case OP_MOVE_DOWN:
      ++level;
      if (!LEVEL_OK(level) || level < 1) return;
      if (level_end[level] == -1) {
        level_end[level] = next_struct(c, lbc, level_end[level - 1], line_index + 1, level - 1);
        while (at(c, line_index) == ' ') ++line_index;
      }
      break;
    case OP_MOVE_TO_KEY:
      key_len = read_varint(c, qp);
      key_pos = qp;
      qp += key_len;
      if (key_len < 0 || !LEVEL_OK(level)) return;
      if (at(c, line_index) != '{') return;
      steps = 0;
      for (;;) {
        if (++steps > max_steps) return;
        ++line_index;
        line_index = next_struct(c, lbc, level_end[level], line_index, level);
        if (at(c, line_index) == ':') {
          const int64_t string_end = prev_bit(sc, c.S, c.W, line_start + 1, line_index - 1);
          const int64_t string_start = string_end - key_len;
          bool mismatch = string_start < line_start || at(c, string_start) != '"';
          for (int i = 0; !mismatch && i < key_len; ++i) {
            if (ir_at(c, key_pos + i) != at(c, string_start + i + 1)) mismatch = true;
          }
          if (mismatch) {
            ++line_index;
            line_index = next_struct(c, lbc, level_end[level], line_index, level);
            if (at(c, line_index) == '}') return;
            continue;
          }
        }
        break;
      }
      ++line_index;
      break;
    case OP_MOVE_TO_INDEX: {
      target = read_varint(c, qp);
      if (!LEVEL_OK(level)) return;
      const uint8_t ch = at(c, line_index);
      if (ch != '[' && ch != ',' && ch != ']') return;
      if (ch == '[') curr_index[level] = 0;
      else ++curr_index[level];
      steps = 0;
      for (;;) {
        if (++steps > max_steps) return;
        if (curr_index[level] < target) {
          ++line_index;
          line_index = next_struct(c, lbc, level_end[level], line_index, level);
          if (at(c, line_index) == ',') {
            ++curr_index[level];
            continue;
          }
          return;
        }
        if (curr_index[level] > target) {
          --line_index;
          line_index = prev_struct(c, lbc, 0, line_index, level);
          --curr_index[level];
          continue;
        }
        break;
      }
      if (at(c, line_index) == ']') return;
      ++line_index;
      break;
    }
    case OP_MOVE_TO_INDEX_REVERSE: {
      target = read_varint(c, qp);
      if (!LEVEL_OK(level)) return;
      line_index = level_end[level] - 1;
      while (at(c, line_index) == ' ') --line_index;
      const uint8_t ch = at(c, line_index);
      if (ch != ']' && ch != ',' && ch != '[') return;
      if (ch == ']') curr_index[level] = 0;
      else ++curr_index[level];
      steps = 0;
      for (;;) {
        if (++steps > max_steps) return;
        if (curr_index[level] < target) {
          --line_index;
          line_index = prev_struct(c, lbc, 0, line_index, level);
          if (at(c, line_index) == ',' || curr_index[level] + 1 == target) {
            ++curr_index[level];
            continue;
          }
          return;
        }
        if (curr_index[level] > target) {
          ++line_index;
          line_index = next_struct(c, lbc, level_end[level], line_index, level);
          --curr_index[level];
          continue;
        }
        break;
      }
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
      for (int i = level + 1; i < kMaxQueryLevels; ++i) {
        if (i < 0) continue;
        if (level_end[i] == -1) break;
        level_end[i] = -1;
      }
      break;
    case OP_EXPRESSION_STRING_EQUALS: {
      key_len = read_varint(c, qp);
      key_pos = qp;
      qp += key_len;
      if (key_len < 0 || !LEVEL_OK(level)) return;
      while (at(c, line_index) == ' ' && line_index < level_end[level]) ++line_index;
      int64_t string_end = level_end[level] - 1;
      while (line_index < string_end && at(c, string_end) == ' ') --string_end;
      if (string_end - line_index + 1 != key_len) return;
      for (int i = 0; i < key_len; ++i) {
        if (ir_at(c, key_pos + i) != at(c, line_index + i)) return;
      }
      break;
    }
    default:
      break;
    }
    if (qp > int64_t(c.ir_len) + 1) return;
  }
#undef LEVEL_OK
}

template <typename OutT>
__global__ void __launch_bounds__(256)
    query_kernel(const QueryLaunch q, const __grid_constant__ IrBlob ir, OutT *out) {
  __shared__ uint8_t s_ir[kMaxQueryIrBytes];
  for (int i = threadIdx.x; i < q.ir_len; i += blockDim.x) s_ir[i] = ir.bytes[i];
  __syncthreads();
  const Rec c{q.in, q.n, q.S, q.LB, q.W, s_ir, q.ir_len, q.base_level, q.num_levels};
  const int64_t stride = int64_t(blockDim.x) * gridDim.x;
  for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < q.num_lines;
       r += stride) {
    OutT *o = out + r * int64_t(q.num_results) * 2;
    for (int i = 0; i < 2 * q.num_results; ++i) o[i] = OutT(-1);
    const int64_t start = q.NL[r];
    const int64_t end = (r + 1 < q.num_lines) ? q.NL[r + 1] : q.n - 1;
    run_record<OutT>(c, start, end, q.num_results, o);
  }
}

__global__ void __launch_bounds__(256)
    batch_query_kernel(const BatchQueryLaunch q, const __grid_constant__ IrBlob ir) {
  __shared__ uint8_t s_ir[kMaxQueryIrBytes];
  for (int i = threadIdx.x; i < kMaxQueryIrBytes; i += blockDim.x) s_ir[i] = ir.bytes[i];
  __syncthreads();
  const uint64_t records = q.totals[kTotRecords];
  const uint64_t stride = uint64_t(blockDim.x) * gridDim.x;
  for (uint64_t r = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < records; r += stride) {
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
    const Rec c{q.in + F.in_off, int64_t(F.n), q.S + F.s_off, q.LB + F.lb_off,
                int64_t((F.n + 63u) / 64u), s_ir + g.ir_off, g.ir_len, g.base_level, F.levels};
    run_record<int32_t>(c, start, end, g.num_results, o);
  }
}

}  // namespace

cudaError_t batch_query_launch(const BatchQueryLaunch &q, const IrBlob &ir, int grid,
                               int block, cudaStream_t stream) {
  batch_query_kernel<<<grid, block, 0, stream>>>(q, ir);
  return cudaGetLastError();
}

cudaError_t query_launch(const QueryLaunch &q, const IrBlob &ir, int grid,
                         int block, cudaStream_t stream) {
  if (q.num_lines <= 0 || q.n <= 0) return cudaSuccess;
  if (block <= 0) block = 256;
  if (block > 256) block = 256;
  if (grid <= 0) grid = int((q.num_lines + block - 1) / block);
  if (q.out64 != nullptr) {
    query_kernel<int64_t><<<grid, block, 0, stream>>>(q, ir, q.out64);
  } else {
    query_kernel<int32_t><<<grid, block, 0, stream>>>(q, ir, q.out32);
  }
  return cudaGetLastError();
}

}  // namespace gpjb
