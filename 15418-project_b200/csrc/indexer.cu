// Fused single-pass structural indexer for sm_100a.
//
// One launch replaces the reference's whole SharememIndexBuilder chain
// (src/gpjson/index/sharemem_index_builder.cu:443-458: nine kernels, three
// thrust scans, four scalar copies, seven passes over the input).  Persistent
// CTAs take 32 KiB tiles in ticket order, stage each in shared memory with
// one TMA tensor load (128-byte swizzle so that every thread reads its own
// 128-byte row with conflict-free 16-byte loads), and compute per 64-byte
// word:
//   escape bitmap E   (word-local carry rule, escape-index.cu:29-96)
//   quote bitmap  Q   = '"' & ~E                     (quote-index.cu:29-95)
//   string mask   S   = prefix-XOR of Q over the file (string-index.cu:3-31)
//   depth             = -1 + running sum of '{[' minus '}]' outside strings,
//                       signed char                  (leveled-bitmaps-*.cu)
//   leveled bitmaps   LB[level*W + w]
//   newline index     NL = [0, offsets of every '\n'] (newline-*.cu)
// The three file-wide carries (string parity, depth, newline count) cross
// tiles through a decoupled look-back.  A tile's depth change depends on the
// string state it starts in, so its look-back descriptor holds the change for
// both start states; descriptors compose associatively.
#include "bits.cuh"
#include "descriptor.cuh"
#include "indexer.cuh"

#include <cudaTypedefs.h>

namespace gpjb {
namespace {

__device__ __forceinline__ uint64_t ld_relaxed(const unsigned long long *p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(unsigned long long *p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Every wait is bounded: after this many polls (with back-off) the kernel
// records an error bit and carries on with neutral values, so a broken
// invariant surfaces as an error status on the host instead of a hang.
constexpr uint32_t kSpinLimit = 1u << 22;

// One warp.  Walks back over the predecessors of `tile` (whose own aggregate
// is already published), 32 * K per round (K descriptors per lane, loaded
// together so one round costs one memory round trip), and returns the tile's
// exclusive prefix.  The fold works on packed descriptors: two shuffles and
// one branch-free composition per step.  Rounds of 32 (K = 1) were measured
// faster than rounds of 64 or 128 on the configured workloads: a nearby
// inclusive descriptor is the usual case, and fewer polled lines wait on
// fewer unpublished tiles; the batch autotuner also tries K = 2.

__device__ __forceinline__ uint64_t shfl_down_u64(uint64_t v, int off) {
  const uint32_t lo = __shfl_down_sync(0xFFFFFFFFu, uint32_t(v), off);
  const uint32_t hi = __shfl_down_sync(0xFFFFFFFFu, uint32_t(v >> 32), off);
  return (uint64_t(hi) << 32) | lo;
}
__device__ __forceinline__ uint64_t shfl_u64(uint64_t v, int src) {
  const uint32_t lo = __shfl_sync(0xFFFFFFFFu, uint32_t(v), src);
  const uint32_t hi = __shfl_sync(0xFFFFFFFFu, uint32_t(v >> 32), src);
  return (uint64_t(hi) << 32) | lo;
}

template <int kLookbackPerLane>
__device__ Agg lookback(const IndexLaunch &P, uint32_t tile) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) return agg_identity();

  uint64_t later = 0;  // packed identity
  int64_t base = int64_t(tile) - 1;  // newest tile of the window
  for (;;) {
    // lane l covers tiles base - l*K - j, j = 0 (newest) .. K-1 (oldest),
    // K = kLookbackPerLane
    uint64_t s[kLookbackPerLane];
#pragma unroll
    for (int j = 0; j < kLookbackPerLane; ++j) s[j] = 0;  // not yet published
    uint32_t polls = 0;
    for (;;) {
      // only descriptors not yet published are (re)read: the lines of the
      // newest tiles are the ones every look-back polls
      bool ready = true;
#pragma unroll
      for (int j = 0; j < kLookbackPerLane; ++j) {
        const int64_t idx = base - int64_t(kLookbackPerLane) * lane - j;
        if ((s[j] & 3u) == 0) s[j] = (idx >= 0) ? ld_relaxed(&P.tile_state[idx]) : kStatusIncl;
        ready = ready && ((s[j] & 3u) != 0);
      }
      if (__all_sync(0xFFFFFFFFu, ready)) break;
      if (++polls > P.lookback_spin_limit) {
        if (lane == 0) atomicOr(P.error, kErrLookbackTimeout);
#pragma unroll
        for (int j = 0; j < kLookbackPerLane; ++j)
          if ((s[j] & 3u) == 0) s[j] = kStatusIncl;
        break;
      }
      __nanosleep(polls < 4096 ? 32 : 500);
    }
    // fold the lane's descriptors newest-first, stopping at an inclusive one
    uint64_t v = 0;
    bool has_incl = false;
#pragma unroll
    for (int j = 0; j < kLookbackPerLane; ++j) {
      if (!has_incl) {
        v = desc_combine(s[j], v);
        has_incl = (s[j] & 3u) == kStatusIncl;
      }
    }
    const uint32_t incl = __ballot_sync(0xFFFFFFFFu, has_incl);
    const int limit = incl ? (__ffs(incl) - 1) : 31;
    if (lane > limit) v = 0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint64_t o = shfl_down_u64(v, off);  // tiles further back
      if (lane + off < 32) v = desc_combine(o, v);
    }
    later = desc_combine(shfl_u64(v, 0), later);
    if (incl) break;
    base -= 32 * kLookbackPerLane;
  }
  return agg_unpack(later);
}

// ----------------------------------------------------------------------------
// Leveled bitmaps of one word.  Walks the open/close events of the word in
// order; separators between two events share one depth.  Depth arithmetic is
// signed char, as in sharemem/leveled-bitmaps-index.cu:270-300.
// ----------------------------------------------------------------------------
template <int LMAX>
__device__ __forceinline__ void add_level(uint64_t (&lb)[LMAX], int d, uint64_t m) {
  // levels >= L are computed but never stored; d outside [0, LMAX) matches none
#pragma unroll
  for (int l = 0; l < LMAX; ++l) lb[l] |= (d == l) ? m : 0ull;
}

template <int LMAX>
__device__ __forceinline__ int leveled_word(uint64_t op, uint64_t cl,
                                            uint64_t sp, int depth,
                                            uint64_t (&lb)[LMAX]) {
#pragma unroll
  for (int l = 0; l < LMAX; ++l) lb[l] = 0;
  uint64_t ev = op | cl;
  int d = depth;
  uint64_t acc = 0, done = 0;
  while (ev) {  // branch-free body: lanes only differ in the trip count
    const uint64_t bit = ev & (0 - ev);
    const uint64_t below = bit - 1;
    acc |= sp & below & ~done;
    const bool open = (op & bit) != 0;
    add_level<LMAX>(lb, d, open ? acc : (acc | bit));
    d = int(int8_t(open ? d + 1 : d - 1));
    acc = open ? bit : 0ull;
    done = below | bit;
    ev &= ev - 1;
  }
  add_level<LMAX>(lb, d, acc | (sp & ~done));
  return d;
}

__device__ __forceinline__ uint64_t valid_mask(uint64_t w, uint64_t n) {
  const uint64_t base = w * 64u;
  if (base + 64u <= n) return ~0ull;
  if (base >= n) return 0ull;
  return (1ull << (n - base)) - 1ull;
}

__device__ __forceinline__ void store2(uint64_t *dst, uint64_t w, uint64_t W,
                                       uint64_t a, uint64_t b) {
  // dst + w is 16-byte aligned whenever the element offset is even
  if (w + 1 < W) {
    if (((reinterpret_cast<uintptr_t>(dst + w)) & 15u) == 0) {
      *reinterpret_cast<ulonglong2 *>(dst + w) = make_ulonglong2(a, b);
    } else {
      dst[w] = a;
      dst[w + 1] = b;
    }
  } else if (w < W) {
    dst[w] = a;
  }
}

// Loads 64 bytes [base, base+64) of `in` as 16 registers, zero at and past n.
__device__ __forceinline__ void load_word_global(const uint8_t *in, uint64_t n,
                                                 uint64_t base, uint32_t (&r)[16]) {
  if (base + 64u <= n && (reinterpret_cast<uintptr_t>(in + base) & 15u) == 0) {
    const uint4 *p = reinterpret_cast<const uint4 *>(in + base);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const uint4 v = __ldg(p + c);
      r[4 * c + 0] = v.x;
      r[4 * c + 1] = v.y;
      r[4 * c + 2] = v.z;
      r[4 * c + 3] = v.w;
    }
    return;
  }
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    uint32_t v = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const uint64_t i = base + uint64_t(4 * k + b);
      if (i < n) v |= uint32_t(in[i]) << (8 * b);
    }
    r[k] = v;
  }
}

// Reads word `half` (0 or 1) of row `row` from the swizzled tile: chunk j of
// a row sits at chunk position j ^ (row & 7) (TMA 128-byte swizzle).
__device__ __forceinline__ void load_word_smem(const uint8_t *tile, int row,
                                               int half, uint32_t (&r)[16]) {
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int j = 4 * half + c;
    const uint4 v = *reinterpret_cast<const uint4 *>(
        tile + row * 128 + ((j ^ (row & 7)) << 4));
    r[4 * c + 0] = v.x;
    r[4 * c + 1] = v.y;
    r[4 * c + 2] = v.z;
    r[4 * c + 3] = v.w;
  }
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Locates the file of `tile`: binary search over the files' first tiles.
__device__ __forceinline__ uint32_t file_of_tile(const IndexLaunch &P, uint32_t tile) {
  uint32_t lo = 0, hi = P.num_files;  // invariant: files[lo].first_tile <= tile
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (P.files[mid].first_tile <= tile) lo = mid;
    else hi = mid;
  }
  return lo;
}

// ----------------------------------------------------------------------------
// mbarrier and named-barrier helpers.  Every wait is bounded.
// ----------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;"
      " selp.u32 %0, 1, 0, p; }"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}
// false: gave up after kSpinLimit polls, or the CTA is aborting
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity,
                                          const volatile uint32_t *abort) {
  for (uint32_t polls = 0; !mbar_try(bar, parity);) {
    if (++polls > kSpinLimit || *abort) return false;
  }
  return true;
}

// Named barrier of the compute warps (the control warp never joins it).
template <int NT>
__device__ __forceinline__ void compute_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
}
// The same barrier, returning the OR of `pred` over the compute threads: a
// decision every compute thread takes identically.
template <int NT>
__device__ __forceinline__ bool compute_sync_or(bool pred) {
  uint32_t r;
  asm volatile(
      "{ .reg .pred p, q; setp.ne.u32 p, %1, 0; barrier.red.or.pred q, 1, %2, p;"
      " selp.u32 %0, 1, 0, q; }"
      : "=r"(r)
      : "r"(uint32_t(pred)), "n"(NT)
      : "memory");
  return r != 0;
}

// A tile's look-back aggregate from its local scans: string parity, depth
// sums packed as (change if the tile starts outside a string) | (total << 16),
// newline count.
__device__ __forceinline__ Agg tile_aggregate(uint32_t par, uint32_t dd, uint32_t nl,
                                              bool file_start) {
  Agg a;
  a.p = par;
  a.d0 = dd & 0xFFu;
  a.d1 = ((dd >> 16) - dd) & 0xFFu;  // total - d0
  a.c = file_start ? 1u : 0u;
  if (file_start) a.d1 = a.d0;  // a file starts outside any string
  a.n = nl;
  return a;
}

// ----------------------------------------------------------------------------
// Persistent pipelined indexer.
//
// A CTA is NT compute threads (one 128-byte row of a tile each) plus one
// control warp.  The compute warps run, for their k-th tile, phase A
// (classification, escapes, local scans: everything that does not need the
// file-wide prefix; it ends by publishing the tile's look-back aggregate) and
// then phase B of tile k-1 (string mask, leveled bitmaps, newline index:
// everything that does).  The control warp claims the CTA's next tile the
// moment phase A of the current one ends, stages it into the free one of two
// shared-memory buffers with a TMA tensor load, and resolves the prefix of
// the current tile by decoupled look-back while the compute warps run phase
// B of the previous tile and phase A of the next.
//
// Claiming just in time keeps the time from a tile's claim to its aggregate
// the same for every CTA (phase B of one tile plus phase A of the next), so
// a tile's predecessors, claimed earlier, have mostly published theirs by
// the time it looks back.  Tiles are claimed only by running CTAs, in
// increasing order per CTA, and a CTA's compute warps always work on its
// smallest unfinished tile, so every wait ends.
// ----------------------------------------------------------------------------
constexpr int kStages = 2;
constexpr uint32_t kEndTile = 0xFFFFFFFFu;

struct StageMeta {  // written by the control warp with each fill
  uint32_t tile;    // kEndTile: no more tiles for this CTA
  uint32_t file_idx;
  uint32_t halo;    // escape carry into the tile
  uint32_t valid;   // bytes of the file in the tile
  uint32_t smem_rows;  // rows 0 .. smem_rows-1 are read from the staged copy
  uint32_t pad;
  IndexFile F;
};

struct TileMeta {  // a tile between its phase A and its phase B
  uint32_t tile, file_idx;
  IndexFile F;
  uint32_t par, dd, nl;  // tile aggregate: string parity, packed depth sums, newlines
  uint32_t c_in, d_in;   // prefix from the look-back
  unsigned long long n_in;
  // Where phase B writes, computed once per tile: the file's S and level-0
  // words from the tile's first word on, the file's word count and the
  // tile's first word.  store_flags: kTileInside when every word of the
  // tile lies inside the file (the stores need no bounds check), kTileSAligned
  // when the S row of every thread starts on 16 bytes, bit kTileLevelAligned
  // + l when level l's rows do, and kTileAllAligned when all of them do.
  uint64_t *S_tile, *LB_tile;
  uint64_t W, lw_tile;
  uint32_t store_flags;
};
constexpr uint32_t kTileInside = 1u, kTileSAligned = 2u, kTileAllAligned = 4u,
                   kTileLevelAligned = 8u;

template <int NT>
struct PipeSmem {
  static constexpr int NW = NT / 32;
  uint8_t tiles[kStages][NT * 128];
  unsigned long long full[kStages];
  unsigned long long agg[2];
  unsigned long long pref[2];
  StageMeta stage[kStages];
  TileMeta tm[2];
  uint32_t last_tp[NW], warp_par[NW], warp_dd[NW], warp_nl[NW];
  uint32_t abort;
};

// Shared-memory staging of the leveled bitmaps (phase B): per warp and
// level, one 64-bit slot for each of the warp's 64 words; a lane only ever
// touches the slots of its own two words.  Level LMAX is a sink for the
// masks of depths that are not stored, so the walk writes without a branch.
constexpr int kSharedLevels = 8;  // LMAX up to this stages in shared memory
// Indexes of up to four levels can walk quarters with two or more bracket
// events from a per-warp list (every lane takes one), the rest in the lane
// that owns them (kList); otherwise every lane walks its own four quarters.
template <int LMAX>
__host__ __device__ constexpr bool walk_list_allowed() {
  return LMAX <= 4;
}
template <int NT, int LMAX, bool kList>
struct LevelScratch {
  static constexpr int NW = NT / 32;
  uint64_t lb[NW][LMAX + 1][64];
  uint4 items[kList ? NW : 1][128];  // O, C, P, start depth | quarter << 8
};

// One thread's row between phase A and phase B.
struct RowState {
  uint64_t op0, cl0, sp0, nl0, op1, cl1, sp1, nl1;
  uint64_t Sl0, Sl1;
  uint32_t pex, par0, dd_ex, nl_ex;
};

// The leveled-bitmap scratch follows the pipeline state (8-byte aligned);
// kernels for more than kSharedLevels levels do not allocate it.
template <int NT>
__host__ __device__ constexpr size_t level_scratch_offset() {
  return (sizeof(PipeSmem<NT>) + 15u) & ~size_t(15);
}

// Claims the next tile and stages it into buffer s (warp-collective).
template <int NT, bool kTma>
__device__ __forceinline__ void control_fill(const IndexLaunch &P, PipeSmem<NT> &sm,
                                             const CUtensorMap *tmap, int s, bool &ended,
                                             uint32_t &tile_out) {
  constexpr uint64_t TILE_BYTES = uint64_t(NT) * 128u;
  const int lane = threadIdx.x & 31;
  uint32_t t = 0;
  if (lane == 0) t = P.tile_begin + atomicAdd(P.tile_counter, 1u);
  t = __shfl_sync(0xFFFFFFFFu, t, 0);
  const uint32_t full = smem_u32(&sm.full[s]);
  if (t >= P.tile_end) {
    ended = true;
    tile_out = kEndTile;
    if (lane == 0) {
      sm.stage[s].tile = kEndTile;
      mbar_arrive(full);
      mbar_arrive(full);
    }
    return;
  }
  // Every CTA claims about one tile per iteration, so the tiles claimed one
  // iteration from now are about gridDim.x tiles ahead: that tile's bytes are
  // prefetched into L2.  The copy needs only the tile's first input row: one
  // load from the row table of a file table, none for a single file.
  const uint32_t ahead = t + gridDim.x;
  const bool has_ahead = ahead < P.tile_end;
  uint32_t f = 0;
  IndexFile F;
  uint64_t row0 = 0, pf_row = ~0ull;
  bool first = false, have_F = true;
  if (P.files == nullptr) {
    F = P.single;
    row0 = uint64_t(t) * NT;
    first = t == 0;
    if (has_ahead) pf_row = uint64_t(ahead) * NT;
  } else if (P.tile_row != nullptr && P.tile_file != nullptr) {
    const uint32_t tr = P.tile_row[t];
    f = P.tile_file[t];
    const uint32_t ta = has_ahead ? P.tile_row[ahead] : 0u;
    row0 = tr & 0x7FFFFFFFu;
    first = (tr >> 31) != 0;
    if (has_ahead) pf_row = ta & 0x7FFFFFFFu;
    have_F = false;  // loaded after the copy is issued
  } else {
    uint32_t fa = 0;
    if (P.tile_file) {
      f = P.tile_file[t];
      if (has_ahead) fa = P.tile_file[ahead];
    } else {
      f = file_of_tile(P, t);
      if (has_ahead) fa = file_of_tile(P, ahead);
    }
    F = P.files[f];
    const uint32_t ktile = t - F.first_tile;
    row0 = (F.in_off + uint64_t(ktile) * TILE_BYTES) / 128u;
    first = ktile == 0;
    if (has_ahead) {
      const IndexFile A = P.files[fa];
      pf_row = (A.in_off + uint64_t(ahead - A.first_tile) * TILE_BYTES) / 128u;
    }
  }
  // The stage's barrier takes two arrivals: one with the copy's byte count
  // as soon as the copy is issued, one once the escape carry (a dependent
  // global load) and the tile's file are written, so the copy waits for
  // neither.
  if (lane == 0) {
    if constexpr (kTma) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive_tx(full, uint32_t(TILE_BYTES));
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(sm.tiles[s])),
          "l"(tmap), "r"(0), "r"(int32_t(row0)), "r"(full)
          : "memory");
      if (pf_row != ~0ull && (pf_row + NT) * 128u <= P.full_rows * 128u)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(P.in + pf_row * 128u),
                     "r"(uint32_t(TILE_BYTES))
                     : "memory");
    } else {
      mbar_arrive(full);
    }
  }
  if (!have_F) F = P.files[f];
  // escape carry: parity of the backslash run ending the word before the
  // tile, counted inside that word (all 64 bytes read at once)
  uint32_t halo = 0;
  if (!first) {
    const uint8_t *w = P.in + row0 * 128u - 64u;
    const uint32_t lo = __ballot_sync(0xFFFFFFFFu, w[lane] != '\\');
    const uint32_t hi = __ballot_sync(0xFFFFFFFFu, w[32 + lane] != '\\');
    const uint64_t not_bs = (uint64_t(hi) << 32) | lo;
    halo = uint32_t(__clzll(static_cast<long long>(not_bs))) & 1u;
  }
  if (lane == 0) {
    // the tile's bytes of the file, and the rows the compute threads read
    // from the staged copy (whole rows inside the file and the tensor map)
    const uint64_t byte0 = uint64_t(t - F.first_tile) * TILE_BYTES;
    const uint32_t valid = uint32_t(min(TILE_BYTES, F.n - byte0));
    uint32_t smem_rows = 0;
    if (kTma && row0 < P.full_rows)
      smem_rows = uint32_t(min(uint64_t(valid / 128u), P.full_rows - row0));
    sm.stage[s].tile = t;
    sm.stage[s].file_idx = f;
    sm.stage[s].F = F;
    sm.stage[s].halo = halo;
    sm.stage[s].valid = valid;
    sm.stage[s].smem_rows = smem_rows;
    mbar_arrive(full);
  }
  tile_out = t;
}

template <int NT, bool kTma, int kLB>
__device__ void control_warp(const IndexLaunch &P, PipeSmem<NT> &sm, const CUtensorMap *tmap) {
  static_assert(kLB == 1 || kLB == 2, "look-back descriptors per lane");
  const int lane = threadIdx.x & 31;
  const volatile uint32_t *abort = &sm.abort;
  uint32_t stage_tile[kStages] = {kEndTile, kEndTile};
  bool ended = false;
  control_fill<NT, kTma>(P, sm, tmap, 0, ended, stage_tile[0]);
  uint32_t k = 0;
  for (;; ++k) {
    const int s = int(k & 1u);
    const uint32_t tile = stage_tile[s];
    if (tile == kEndTile) break;
    const int j = int(k & 1u);
    if (!mbar_wait(smem_u32(&sm.agg[j]), (k >> 1) & 1u, abort)) {
      if (lane == 0) {
        atomicOr(P.error, kErrPipelineTimeout);
        sm.abort = 1;
      }
      break;
    }
    // phase A of tile k is done: claim and stage tile k+1 at once (the
    // other buffer was read by phase A of tile k-1), then resolve k's prefix
    if (!ended) control_fill<NT, kTma>(P, sm, tmap, s ^ 1, ended, stage_tile[s ^ 1]);
    stage_tile[s] = kEndTile;

    TileMeta &tm = sm.tm[j];
    const IndexFile F = tm.F;
    const bool file_start = tile == F.first_tile;
    const Agg local = tile_aggregate(tm.par, tm.dd, tm.nl, file_start);
    const Agg prefix = lookback<kLB>(P, tile);
    if (lane == 0) {
      const Agg incl = agg_combine(prefix, local);
      st_relaxed(&P.tile_state[tile], agg_pack(kStatusIncl, incl));
      tm.c_in = file_start ? 0u : prefix.p;
      tm.d_in = file_start ? 0u : prefix.d0;
      tm.n_in = prefix.n;
      if (P.files == nullptr && tile + 1 == P.num_tiles) {
        P.summary[0] = incl.n + 1u;  // lines = newlines + 1
        P.summary[1] = incl.p;
        P.summary[2] = uint64_t(int64_t(int8_t(uint8_t(incl.d0 - 1u))));
      }
      if (file_start && prefix.n + tm.file_idx < P.nl_cap) P.NL[prefix.n + tm.file_idx] = 0;
      mbar_arrive(smem_u32(&sm.pref[j]));
    }
    __syncwarp();
  }
  // no TMA may still be writing this CTA's shared memory when it exits: a
  // staged tile not yet consumed is the one of iteration k (buffer k & 1) or
  // k + 1 (the other buffer)
  if constexpr (kTma) {
#pragma unroll
    for (int s = 0; s < kStages; ++s) {
      if (stage_tile[s] == kEndTile) continue;
      const uint32_t kk = (uint32_t(s) == (k & 1u)) ? k : k + 1u;
      for (uint32_t polls = 0; !mbar_try(smem_u32(&sm.full[s]), (kk >> 1) & 1u) &&
                               polls < kSpinLimit;
           ++polls) {
      }
    }
  }
}

template <int LMAX, bool kTma, int NT>
__device__ __forceinline__ void phase_a(const IndexLaunch &P, PipeSmem<NT> &sm, int s, uint32_t k,
                                        RowState &st) {
  constexpr int NWARPS = NT / 32;
  constexpr uint64_t TILE_BYTES = uint64_t(NT) * 128u;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const StageMeta &m = sm.stage[s];
  const uint32_t tile = m.tile;
  const IndexFile F = m.F;
  const uint32_t ktile = tile - F.first_tile;
  const uint64_t byte0 = uint64_t(ktile) * TILE_BYTES;
  const uint32_t valid = m.valid;
  const uint32_t row_byte = uint32_t(tid) * 128u;
  const uint64_t lw0 = byte0 / 64u + 2u * uint64_t(tid);
  const bool row_in_smem = kTma && uint32_t(tid) < m.smem_rows;
  // rows past the end of the file read as zero bytes (no class)
  const uint32_t lim = valid > row_byte ? valid - row_byte : 0u;
  const uint8_t *rp = P.in + F.in_off + byte0 + row_byte;
  uint32_t r[16];
  if (row_in_smem) load_word_smem(sm.tiles[s], tid, 0, r);
  else load_word_global(rp, lim, 0, r);
  const WordClasses c0 = classify64(r);
  if (row_in_smem) load_word_smem(sm.tiles[s], tid, 1, r);
  else load_word_global(rp, lim, 64, r);
  const WordClasses c1 = classify64(r);
  const uint32_t tp0 = trailing_escape_parity(c0.bs);
  const uint32_t tp1 = trailing_escape_parity(c1.bs);
  if (lane == 31) sm.last_tp[warp] = tp1;
  compute_sync<NT>();  // (1) last_tp; every row of buffer s has been read
  uint32_t cin0 = __shfl_up_sync(0xFFFFFFFFu, tp1, 1);
  if (lane == 0) cin0 = (warp == 0) ? m.halo : sm.last_tp[warp - 1];

  const uint64_t E0 = escaped_bits(c0.bs, cin0);
  const uint64_t E1 = escaped_bits(c1.bs, tp0);
  const uint64_t Q0 = c0.qt & ~E0;
  const uint64_t Q1 = c1.qt & ~E1;
  const uint64_t Sl0 = prefix_xor(Q0);
  const uint64_t Sl1 = prefix_xor(Q1);
  // a word's quote parity is the top bit of its in-word prefix-XOR
  const uint32_t par0 = uint32_t(Sl0 >> 63);
  const uint32_t par1 = uint32_t(Sl1 >> 63);
  if (P.E != nullptr) {
    const uint64_t W = (F.n + 63u) / 64u;
    store2(P.E + F.s_off, lw0, W, E0 & valid_mask(lw0, F.n), E1 & valid_mask(lw0 + 1, F.n));
    store2(P.Q + F.s_off, lw0, W, Q0, Q1);
  }

  // depth change of each word if it starts outside a string, and in total
  const int d00 = popc64(c0.op & ~Sl0) - popc64(c0.cl & ~Sl0);
  const int t0 = popc64(c0.op) - popc64(c0.cl);
  const int d10 = popc64(c1.op & ~Sl1) - popc64(c1.cl & ~Sl1);
  const int t1 = popc64(c1.op) - popc64(c1.cl);
  const int thr_d0 = d00 + (par0 ? (t1 - d10) : d10);
  const int thr_t = t0 + t1;
  const uint32_t thr_par = par0 ^ par1;
  const uint32_t thr_nl = uint32_t(popc64(c0.nl) + popc64(c1.nl));

  const uint32_t lt_mask = (1u << lane) - 1u;
  const uint32_t par_ballot = __ballot_sync(0xFFFFFFFFu, thr_par);
  uint32_t pex = uint32_t(__popc(par_ballot & lt_mask)) & 1u;
  if (lane == 0) sm.warp_par[warp] = uint32_t(__popc(par_ballot)) & 1u;
  compute_sync<NT>();  // (2)
  // the warps' parities as one bit mask (lane w reads warp w's)
  const uint32_t wpar =
      __ballot_sync(0xFFFFFFFFu, lane < NWARPS && sm.warp_par[lane < NWARPS ? lane : 0] != 0u);
  pex ^= uint32_t(__popc(wpar & ((1u << warp) - 1u))) & 1u;
  const uint32_t tile_par = uint32_t(__popc(wpar)) & 1u;
  // depth changes are only needed mod 256: two 16-bit lanes cannot overflow
  // over at most 256 threads (256 * 255 < 65536)
  const int dt0 = pex ? (thr_t - thr_d0) : thr_d0;
  const uint32_t dd = (uint32_t(dt0) & 0xFFu) | ((uint32_t(thr_t) & 0xFFu) << 16);
  uint32_t dd_inc = dd, nl_inc = thr_nl;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t a = __shfl_up_sync(0xFFFFFFFFu, dd_inc, off);
    const uint32_t b = __shfl_up_sync(0xFFFFFFFFu, nl_inc, off);
    if (lane >= off) {
      dd_inc += a;
      nl_inc += b;
    }
  }
  if (lane == 31) {
    sm.warp_dd[warp] = dd_inc;
    sm.warp_nl[warp] = nl_inc;
  }
  compute_sync<NT>();  // (3)
  // inclusive scan of the warps' sums over lanes 0 .. NWARPS-1
  uint32_t wdd = lane < NWARPS ? sm.warp_dd[lane < NWARPS ? lane : 0] : 0u;
  uint32_t wnl = lane < NWARPS ? sm.warp_nl[lane < NWARPS ? lane : 0] : 0u;
#pragma unroll
  for (int off = 1; off < NWARPS; off <<= 1) {
    const uint32_t a = __shfl_up_sync(0xFFFFFFFFu, wdd, off);
    const uint32_t b = __shfl_up_sync(0xFFFFFFFFu, wnl, off);
    if (lane >= off) {
      wdd += a;
      wnl += b;
    }
  }
  const int prev_warp = warp > 0 ? warp - 1 : 0;
  const uint32_t before_dd = __shfl_sync(0xFFFFFFFFu, wdd, prev_warp);
  const uint32_t before_nl = __shfl_sync(0xFFFFFFFFu, wnl, prev_warp);
  const uint32_t tile_dd = __shfl_sync(0xFFFFFFFFu, wdd, NWARPS - 1);
  const uint32_t tile_nl = __shfl_sync(0xFFFFFFFFu, wnl, NWARPS - 1);
  const uint32_t dd_ex = dd_inc - dd + (warp > 0 ? before_dd : 0u);
  const uint32_t nl_ex = nl_inc - thr_nl + (warp > 0 ? before_nl : 0u);
  if (tid == 0) {
    // publish the aggregate at once: look-backs of later tiles wait for it
    if (tile != 0)
      st_relaxed(&P.tile_state[tile],
                 agg_pack(kStatusAgg, tile_aggregate(tile_par, tile_dd, tile_nl, ktile == 0)));
    TileMeta &tm = sm.tm[k & 1u];
    tm.tile = tile;
    tm.file_idx = m.file_idx;
    tm.F = F;
    tm.par = tile_par;
    tm.dd = tile_dd;
    tm.nl = tile_nl;
    const uint64_t W = (F.n + 63u) / 64u;
    const uint64_t lw_tile = byte0 / 64u;
    tm.W = W;
    tm.lw_tile = lw_tile;
    tm.S_tile = P.S + F.s_off + lw_tile;
    tm.LB_tile = P.LB + F.lb_off + lw_tile;
    uint32_t flags = lw_tile + 2u * NT <= W ? kTileInside : 0u;
    if ((reinterpret_cast<uintptr_t>(tm.S_tile) & 15u) == 0) flags |= kTileSAligned;
    bool all = (flags & kTileSAligned) != 0;
    for (int l = 0; l < F.levels && l < 24; ++l) {
      if ((reinterpret_cast<uintptr_t>(tm.LB_tile + uint64_t(l) * W) & 15u) == 0)
        flags |= 1u << (kTileLevelAligned + l);
      else
        all = false;
    }
    tm.store_flags = flags | (all ? kTileAllAligned : 0u);
    mbar_arrive(smem_u32(&sm.agg[k & 1u]));
  }
  st.op0 = c0.op;
  st.cl0 = c0.cl;
  st.sp0 = c0.sp;
  st.nl0 = c0.nl;
  st.op1 = c1.op;
  st.cl1 = c1.cl;
  st.sp1 = c1.sp;
  st.nl1 = c1.nl;
  st.Sl0 = Sl0;
  st.Sl1 = Sl1;
  st.pex = pex;
  st.par0 = par0;
  st.dd_ex = dd_ex;
  st.nl_ex = nl_ex;
}

// Leveled bitmaps of one lane's two words, walked as event sequences in
// 32-bit quarters (word 0 low, word 0 high, word 1 low, word 1 high; each
// quarter starts at the depth the quarters before it leave), so every step
// is 32-bit integer work.  Separators between two events share one depth;
// an opening bracket belongs to the level it opens, a closing one to the
// level it closes (signed-char depth, sharemem/leveled-bitmaps-index.cu:
// 270-300).  Each mask is OR-ed into the shared-memory slot of its level and
// quarter; the lane reads its two words' slots back once all are written.
template <int LMAX, int NT, bool kList>
__device__ __forceinline__ void leveled_lane(LevelScratch<NT, LMAX, kList> &ls, uint64_t O0,
                                             uint64_t C0, uint64_t P0, uint64_t O1, uint64_t C1,
                                             uint64_t P1, int depth0, uint64_t (&lb0)[LMAX],
                                             uint64_t (&lb1)[LMAX]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t *slot64 = &ls.lb[warp][0][2 * lane];  // [level * 64 + word]
#pragma unroll
  for (int l = 0; l < LMAX; ++l) {
    slot64[l * 64] = 0ull;
    slot64[l * 64 + 1] = 0ull;
  }
  uint32_t *slot = reinterpret_cast<uint32_t *>(slot64);  // [level * 128 + quarter]
  // The signed-char depth is kept modulo 256 in the low byte of d: depths 0
  // .. LMAX-1 are the bytes 0 .. LMAX-1, negative depths the bytes 128 ..
  // 255, and every byte from LMAX up selects the sink level.
  uint32_t d = uint32_t(depth0);
  if constexpr (kList) {
    // A quarter with at most one event takes two masks, written here; a
    // quarter with more goes to the warp's list, ordered by quarter then
    // lane, and each lane walks one listed quarter per pass.  A warp then
    // iterates about as often as its busiest listed quarter needs, not as
    // often as its busiest lane needs in each of the four quarters.  Every
    // (level, quarter) slot has one writer: the owner or the lane walking it.
    uint32_t *wslot = reinterpret_cast<uint32_t *>(&ls.lb[warp][0][0]);  // [level * 128 + q]
    uint4 *items = ls.items[warp];
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t listed = 0;
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const uint64_t Ow = h < 2 ? O0 : O1, Cw = h < 2 ? C0 : C1, Pw = h < 2 ? P0 : P1;
      const uint32_t O = uint32_t((h & 1) ? (Ow >> 32) : Ow);
      const uint32_t C = uint32_t((h & 1) ? (Cw >> 32) : Cw);
      const uint32_t Pm = uint32_t((h & 1) ? (Pw >> 32) : Pw);
      const uint32_t PO = Pm | O, ev = O | C;
      const uint32_t q = uint32_t(lane) * 4u + uint32_t(h);
      const bool heavy = (ev & (ev - 1u)) != 0u;
      const uint32_t hb = __ballot_sync(0xFFFFFFFFu, heavy);
      if (heavy) {
        items[listed + __popc(hb & lt)] = make_uint4(O, C, Pm, (d & 0xFFu) | (q << 8));
      } else {
        // bit: the event, or 0 (below then covers the whole quarter)
        const uint32_t bit = ev & (0u - ev);
        const uint32_t below = bit - 1u;
        wslot[min(d & 0xFFu, uint32_t(LMAX)) * 128 + q] |= (below & PO) | (bit & ~O);
        const uint32_t d1 = d + ((O & bit) ? 1u : (bit ? 0xFFFFFFFFu : 0u));
        wslot[min(d1 & 0xFFu, uint32_t(LMAX)) * 128 + q] |= PO & ~below;
      }
      listed += __popc(hb);
      d += uint32_t(__popc(O)) - uint32_t(__popc(C));
    }
    __syncwarp();
    for (uint32_t i = uint32_t(lane); i < listed; i += 32u) {
      const uint4 it = items[i];
      const uint32_t O = it.x, C = it.y, PO = it.z | it.x, q = it.w >> 8;
      uint32_t dq = it.w, ev = O | C, below_prev = 0u;
      while (ev) {  // the walk of the per-lane loop below
        const uint32_t bit = ev & (0u - ev);
        const uint32_t below = bit - 1u;
        wslot[min(dq & 0xFFu, uint32_t(LMAX)) * 128 + q] |= ((below ^ below_prev) & PO) | (bit & ~O);
        dq += (O & bit) ? 1u : 0xFFFFFFFFu;
        below_prev = below;
        ev ^= bit;
      }
      wslot[min(dq & 0xFFu, uint32_t(LMAX)) * 128 + q] |= PO & ~below_prev;
    }
    __syncwarp();
  } else {
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const uint64_t Ow = h < 2 ? O0 : O1, Cw = h < 2 ? C0 : C1, Pw = h < 2 ? P0 : P1;
      const uint32_t O = uint32_t((h & 1) ? (Ow >> 32) : Ow);
      const uint32_t C = uint32_t((h & 1) ? (Cw >> 32) : Cw);
      const uint32_t Pm = uint32_t((h & 1) ? (Pw >> 32) : Pw);
      // Between two consecutive events the only bits of P | O are the
      // separators and, when the earlier event opens a level, its own bit:
      // exactly the bits of that run's level.
      const uint32_t PO = Pm | O;
      uint32_t ev = O | C, below_prev = 0u;
      while (ev) {  // branch-free body: lanes only differ in the trip count
        const uint32_t bit = ev & (0u - ev);
        const uint32_t below = bit - 1u;
        // the run since the last event, and a closing bracket, which joins
        // the level it closes
        const uint32_t m = ((below ^ below_prev) & PO) | (bit & ~O);
        slot[min(d & 0xFFu, uint32_t(LMAX)) * 128 + h] |= m;
        d += (O & bit) ? 1u : 0xFFFFFFFFu;
        below_prev = below;
        ev ^= bit;
      }
      // the run after the quarter's last event
      slot[min(d & 0xFFu, uint32_t(LMAX)) * 128 + h] |= PO & ~below_prev;
    }
  }
#pragma unroll
  for (int l = 0; l < LMAX; ++l) {
    lb0[l] = slot64[l * 64];
    lb1[l] = slot64[l * 64 + 1];
  }
}

template <int LMAX, int NT, bool kList>
__device__ __forceinline__ void phase_b(const IndexLaunch &P, PipeSmem<NT> &sm,
                                        LevelScratch<NT, LMAX, kList> &ls, uint32_t k,
                                        const RowState &st) {
  const int tid = threadIdx.x;
  const int j = int(k & 1u);
  if (!mbar_wait(smem_u32(&sm.pref[j]), (k >> 1) & 1u, &sm.abort)) {
    atomicOr(P.error, kErrPipelineTimeout);
    sm.abort = 1;
    return;
  }
  const TileMeta &tm = sm.tm[j];
  const uint64_t W = tm.W;
  const uint64_t lw0 = tm.lw_tile + 2u * uint64_t(tid);
  const int levels = tm.F.levels;
  const uint32_t flags = tm.store_flags;
  const uint32_t c_in = tm.c_in, d_in = tm.d_in;
  const uint64_t nl_base = tm.n_in + st.nl_ex + tm.file_idx;  // slot of my first newline - 1

  const uint32_t car0 = c_in ^ st.pex;
  const uint32_t car1 = car0 ^ st.par0;
  const uint64_t S0 = st.Sl0 ^ (car0 ? ~0ull : 0ull);
  const uint64_t S1 = st.Sl1 ^ (car1 ? ~0ull : 0ull);
  const uint32_t a_ex = st.dd_ex & 0xFFu, t_ex = (st.dd_ex >> 16) & 0xFFu;
  const int depth0 = int(int8_t(uint8_t(d_in - 1u + (c_in ? (t_ex - a_ex) : a_ex))));

  uint64_t *const S_tile = tm.S_tile, *const LB_tile = tm.LB_tile;
  // A row of two words, inside the file: one 16-byte store where aligned.
  auto put2 = [tid](uint64_t *row, bool aligned, uint64_t a, uint64_t b) {
    if (aligned) {
      *reinterpret_cast<ulonglong2 *>(row + 2 * tid) = make_ulonglong2(a, b);
    } else {
      row[2 * tid] = a;
      row[2 * tid + 1] = b;
    }
  };
  const bool inside = (flags & kTileInside) != 0;
  if (inside) {
    put2(S_tile, (flags & kTileSAligned) != 0, S0, S1);
  } else {
    store2(S_tile - tm.lw_tile, lw0, W, S0, S1);
  }
  if (levels > 0) {
    uint64_t lb0[LMAX], lb1[LMAX];
    const uint64_t O0 = st.op0 & ~S0, C0 = st.cl0 & ~S0, P0 = st.sp0 & ~S0;
    const uint64_t O1 = st.op1 & ~S1, C1 = st.cl1 & ~S1, P1 = st.sp1 & ~S1;
    if constexpr (LMAX <= kSharedLevels) {
      leveled_lane<LMAX, NT, kList>(ls, O0, C0, P0, O1, C1, P1, depth0, lb0, lb1);
    } else {
      const int depth1 = leveled_word<LMAX>(O0, C0, P0, depth0, lb0);
      leveled_word<LMAX>(O1, C1, P1, depth1, lb1);
    }
    if (inside && (flags & kTileAllAligned) != 0) {
#pragma unroll
      for (int l = 0; l < LMAX; ++l) {
        if (l < levels)
          *reinterpret_cast<ulonglong2 *>(LB_tile + uint64_t(l) * W + 2 * tid) =
              make_ulonglong2(lb0[l], lb1[l]);
      }
    } else if (inside) {
#pragma unroll
      for (int l = 0; l < LMAX; ++l) {
        if (l < levels)
          put2(LB_tile + uint64_t(l) * W, ((flags >> (kTileLevelAligned + l)) & 1u) != 0, lb0[l],
               lb1[l]);
      }
    } else {
#pragma unroll
      for (int l = 0; l < LMAX; ++l) {
        if (l < levels) store2(LB_tile - tm.lw_tile + uint64_t(l) * W, lw0, W, lb0[l], lb1[l]);
      }
    }
  }
  // newline offsets (every '\n' counts, strings or not), file-local
  uint64_t kk = nl_base;
  uint64_t m = st.nl0;
  while (m) {
    const int b = __ffsll(static_cast<long long>(m)) - 1;
    if (kk + 1 < P.nl_cap) P.NL[kk + 1] = int64_t(lw0 * 64u + uint64_t(b));
    ++kk;
    m &= m - 1;
  }
  m = st.nl1;
  while (m) {
    const int b = __ffsll(static_cast<long long>(m)) - 1;
    if (kk + 1 < P.nl_cap) P.NL[kk + 1] = int64_t((lw0 + 1) * 64u + uint64_t(b));
    ++kk;
    m &= m - 1;
  }
}

// LMAX: levels the kernel can store; kTma: tiles staged by TMA; NT: compute
// threads; kList: the listed leveled walk; kLB: look-back descriptors per
// lane.
template <int LMAX, bool kTma, int NT, bool kList, int kLB>
__global__ void __launch_bounds__(NT + 32, LMAX > 8 ? 1 : (NT <= 128 ? 4 : 2))
    index_kernel(const __grid_constant__ CUtensorMap tmap, const IndexLaunch P) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // the 128-byte-swizzled TMA destinations need 1024-byte alignment
  uint8_t *smem_base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  PipeSmem<NT> &sm = *reinterpret_cast<PipeSmem<NT> *>(smem_base);
  LevelScratch<NT, LMAX, kList> &ls = *reinterpret_cast<LevelScratch<NT, LMAX, kList> *>(
      smem_base + level_scratch_offset<NT>());
  const int tid = threadIdx.x;
  if (tid == NT) {
    // barriers must be initialised before anyone polls them: shared memory
    // may still hold barriers of an earlier CTA on this SM
#pragma unroll
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_u32(&sm.full[s]), 2);  // copy issued + escape carry written
      sm.stage[s].tile = kEndTile;
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      mbar_init(smem_u32(&sm.agg[j]), 1);
      mbar_init(smem_u32(&sm.pref[j]), 1);
    }
    sm.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid >= NT) {
    control_warp<NT, kTma, kLB>(P, sm, &tmap);
    return;
  }
  RowState prev{};
  uint32_t k = 0;
  for (;; ++k) {
    const int s = int(k & 1u);
    bool stop = !mbar_wait(smem_u32(&sm.full[s]), (k >> 1) & 1u, &sm.abort);
    if (stop) {
      atomicOr(P.error, kErrTmaTimeout);
      sm.abort = 1;
    }
    // one decision for all compute threads: buffer s is read only when every
    // one of them saw it filled
    stop = compute_sync_or<NT>(stop || *static_cast<volatile uint32_t *>(&sm.abort) != 0 ||
                               sm.stage[s].tile == kEndTile);
    if (stop) break;
    RowState cur;
    phase_a<LMAX, kTma, NT>(P, sm, s, k, cur);
    if (k > 0) phase_b<LMAX, NT, kList>(P, sm, ls, k - 1, prev);
    prev = cur;
  }
  if (k > 0 && !*static_cast<volatile uint32_t *>(&sm.abort))
    phase_b<LMAX, NT, kList>(P, sm, ls, k - 1, prev);
}

template <int LMAX, bool kTma, int NT, bool kList, int kLB>
cudaError_t launch_kernel(const IndexLaunch &L, const CUtensorMap &map, cudaStream_t stream) {
  auto kernel = index_kernel<LMAX, kTma, NT, kList, kLB>;
  constexpr size_t smem = level_scratch_offset<NT>() +
                          (LMAX <= kSharedLevels ? sizeof(LevelScratch<NT, LMAX, kList>) : 0) +
                          1024;  // + alignment slack
  static int grid_per_device[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (grid_per_device[dev] == 0) {
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, NT + 32, smem);
    if (e != cudaSuccess) return e;
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    grid_per_device[dev] = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  }
  const uint32_t grid = min(L.tile_end - L.tile_begin, uint32_t(grid_per_device[dev]));
  kernel<<<grid, NT + 32, smem, stream>>>(map, L);
  return cudaGetLastError();
}

template <int LMAX, int NT, bool kList, int kLB>
cudaError_t launch_tma(const IndexLaunch &L, const CUtensorMap *map, bool use_tma,
                       cudaStream_t stream) {
  if (use_tma) return launch_kernel<LMAX, true, NT, kList, kLB>(L, *map, stream);
  CUtensorMap dummy{};
  return launch_kernel<LMAX, false, NT, kList, kLB>(L, dummy, stream);
}

// The launch variant (IndexLaunch::variant) picks the walk and the look-back
// granularity where both forms exist (up to four levels); deeper indexes
// always walk per lane with rounds of 32 descriptors.
template <int LMAX, int NT>
cudaError_t launch_levels(const IndexLaunch &L, const CUtensorMap *map, bool use_tma,
                          cudaStream_t stream) {
  if constexpr (walk_list_allowed<LMAX>()) {
    const bool lanes = (L.variant & kIndexVariantLaneWalk) != 0;
    const bool wide = (L.variant & kIndexVariantWideLookback) != 0;
    if (lanes && wide) return launch_tma<LMAX, NT, false, 2>(L, map, use_tma, stream);
    if (lanes) return launch_tma<LMAX, NT, false, 1>(L, map, use_tma, stream);
    if (wide) return launch_tma<LMAX, NT, true, 2>(L, map, use_tma, stream);
    return launch_tma<LMAX, NT, true, 1>(L, map, use_tma, stream);
  } else {
    return launch_tma<LMAX, NT, false, 1>(L, map, use_tma, stream);
  }
}

template <int NT>
cudaError_t launch_threads(const IndexLaunch &L, const CUtensorMap *map, bool use_tma,
                           cudaStream_t stream) {
  const int lv = L.num_levels;
  if (lv <= 2) return launch_levels<2, NT>(L, map, use_tma, stream);
  if (lv <= 4) return launch_levels<4, NT>(L, map, use_tma, stream);
  if (lv <= 8) return launch_levels<8, NT>(L, map, use_tma, stream);
  return launch_levels<kMaxLevels, NT>(L, map, use_tma, stream);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault,
                                &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      p = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

}  // namespace

void index_bind_scratch(IndexLaunch &L, void *scratch) {
  auto *base = static_cast<unsigned char *>(scratch);
  L.tile_state = reinterpret_cast<unsigned long long *>(base);
  unsigned char *tail = base + uint64_t(L.num_tiles) * 8u;
  L.summary = reinterpret_cast<unsigned long long *>(tail);        // 4 x u64
  L.tile_counter = reinterpret_cast<unsigned int *>(tail + 32);
  L.error = reinterpret_cast<unsigned int *>(tail + 36);
}

bool index_make_tensor_map(CUtensorMap *map, const uint8_t *in, uint64_t n, int threads) {
  const uint64_t rows = n / 128u;
  if (rows == 0 || (reinterpret_cast<uintptr_t>(in) & 15u) != 0) return false;
  auto fn = encode_fn();
  if (fn == nullptr) return false;
  const cuuint64_t dims[2] = {128u, rows};
  const cuuint64_t strides[1] = {128u};
  const cuuint32_t box[2] = {128u, uint32_t(threads)};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2,
                        const_cast<uint8_t *>(in), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

cudaError_t index_clear_scratch(const IndexLaunch &L, cudaStream_t stream) {
  return cudaMemsetAsync(L.tile_state, 0, uint64_t(L.num_tiles) * 8u + 64u, stream);
}

cudaError_t index_clear_counter(const IndexLaunch &L, cudaStream_t stream) {
  return cudaMemsetAsync(L.tile_counter, 0, sizeof(unsigned int), stream);
}

cudaError_t index_launch_range(const IndexLaunch &L, const CUtensorMap *map, bool use_tma,
                               cudaStream_t stream, uint32_t t0, uint32_t t1, int threads) {
  if (t1 > L.num_tiles) t1 = L.num_tiles;
  if (t0 >= t1) return cudaSuccess;
  IndexLaunch R = L;
  R.tile_begin = t0;
  R.tile_end = t1;
  if (threads == 128) return launch_threads<128>(R, map, use_tma, stream);
  return launch_threads<256>(R, map, use_tma, stream);
}

cudaError_t index_launch(const IndexLaunch &L, const CUtensorMap *map, bool use_tma,
                         cudaStream_t stream, int threads) {
  if (L.num_tiles == 0) return cudaSuccess;
  cudaError_t e = index_clear_scratch(L, stream);
  if (e != cudaSuccess) return e;
  return index_launch_range(L, map, use_tma, stream, 0u, L.num_tiles, threads);
}
}  // namespace gpjb

namespace gpjb {
namespace {

constexpr int kFinalizeThreads = 1024;

__global__ void __launch_bounds__(kFinalizeThreads)
    finalize_files_kernel(const IndexLaunch P, const uint32_t *query_of_file,
                          const uint32_t *slots_of_query, uint64_t *info, uint64_t *totals) {
  __shared__ unsigned long long s_warp_rec[32], s_warp_out[32];
  __shared__ unsigned long long s_carry_rec, s_carry_out;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    s_carry_rec = 0;
    s_carry_out = 0;
  }
  __syncthreads();
  for (uint32_t base = 0; base < P.num_files; base += kFinalizeThreads) {
    const uint32_t f = base + uint32_t(tid);
    uint64_t lines = 0, nl_off = 0, out_ints = 0, in_string = 0, bytes = 0;
    int64_t depth = -1;
    uint32_t q = 0;
    if (f < P.num_files) {
      const IndexFile F = P.files[f];
      const uint32_t next_first = (f + 1 < P.num_files) ? P.files[f + 1].first_tile : P.num_tiles;
      // newlines before the file = inclusive count of the tile before it
      const uint64_t n_start = F.first_tile > 0 ? agg_unpack(P.tile_state[F.first_tile - 1]).n : 0;
      const uint64_t n_end = next_first > 0 ? agg_unpack(P.tile_state[next_first - 1]).n : 0;
      lines = n_end - n_start + 1u;
      nl_off = n_start + f;
      bytes = F.n;
      if (next_first > F.first_tile) {
        const Agg last = agg_unpack(P.tile_state[next_first - 1]);
        in_string = last.p;
        depth = int64_t(int8_t(uint8_t(last.d0 - 1u)));
      } else if (nl_off < P.nl_cap) {
        P.NL[nl_off] = 0;  // an empty file has no tile to write it
      }
      q = query_of_file ? query_of_file[f] : 0u;
      out_ints = lines * uint64_t(slots_of_query ? slots_of_query[q] : 0u) * 2u;
    }
    // block-wide exclusive scans of lines and result ints
    unsigned long long rec_inc = lines, out_inc = out_ints;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const unsigned long long a = __shfl_up_sync(0xFFFFFFFFu, rec_inc, off);
      const unsigned long long b = __shfl_up_sync(0xFFFFFFFFu, out_inc, off);
      if (lane >= off) {
        rec_inc += a;
        out_inc += b;
      }
    }
    if (lane == 31) {
      s_warp_rec[warp] = rec_inc;
      s_warp_out[warp] = out_inc;
    }
    __syncthreads();
    unsigned long long rec_ex = rec_inc - lines + s_carry_rec;
    unsigned long long out_ex = out_inc - out_ints + s_carry_out;
    for (int w = 0; w < warp; ++w) {
      rec_ex += s_warp_rec[w];
      out_ex += s_warp_out[w];
    }
    if (f < P.num_files) {
      uint64_t *row = info + uint64_t(f) * kFileInfoWords;
      row[kFiLines] = lines;
      row[kFiNlOff] = nl_off;
      row[kFiRecOff] = rec_ex;
      row[kFiOutOff] = out_ex;
      row[kFiInString] = in_string;
      row[kFiDepth] = uint64_t(depth);
      row[kFiBytes] = bytes;
      row[kFiQuery] = q;
    }
    __syncthreads();
    if (tid == kFinalizeThreads - 1) {
      s_carry_rec = rec_ex + lines;
      s_carry_out = out_ex + out_ints;
    }
    __syncthreads();
  }
  if (tid == 0) {
    const uint64_t n_total = P.num_tiles > 0 ? agg_unpack(P.tile_state[P.num_tiles - 1]).n : 0;
    totals[kTotRecords] = s_carry_rec;
    totals[kTotResultInts] = s_carry_out;
    totals[kTotNlSlots] = n_total + P.num_files;
    totals[kTotError] = *P.error;
  }
}

}  // namespace

cudaError_t index_finalize_files(const IndexLaunch &L, const uint32_t *query_of_file,
                                 const uint32_t *slots_of_query, uint64_t *file_info,
                                 uint64_t *totals, cudaStream_t stream) {
  finalize_files_kernel<<<1, kFinalizeThreads, 0, stream>>>(L, query_of_file, slots_of_query,
                                                             file_info, totals);
  return cudaGetLastError();
}

}  // namespace gpjb
