// Fused single-pass structural indexer for sm_100a.
//
// One launch replaces the reference's whole SharememIndexBuilder chain
// (src/gpjson/index/sharemem_index_builder.cu:443-458: nine kernels, three
// thrust scans, four scalar copies, seven passes over the input).  Each CTA
// takes one 32 KiB tile in ticket order, stages it in shared memory with one
// TMA tensor load (128-byte swizzle so that every thread reads its own
// 128-byte row with conflict-free 16-byte loads), and computes per 64-byte
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

// Warp 0 only.  Publishes the tile's aggregate, then walks back over its
// predecessors, 128 per round (4 consecutive descriptors per lane, loaded
// together so one round costs one memory round trip), and returns the tile's
// exclusive prefix.  The fold works on packed descriptors: two shuffles and
// one branch-free composition per step.
constexpr int kLookbackPerLane = 4;

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

__device__ Agg lookback(const IndexLaunch &P, uint32_t tile, const Agg &local) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) return agg_identity();
  if (lane == 0) st_relaxed(&P.tile_state[tile], agg_pack(kStatusAgg, local));

  uint64_t later = 0;  // packed identity
  int64_t base = int64_t(tile) - 1;  // newest tile of the window
  for (;;) {
    // lane l covers tiles base - 4l - j, j = 0 (newest) .. 3 (oldest)
    uint64_t s[kLookbackPerLane];
    uint32_t polls = 0;
    for (;;) {
      bool ready = true;
#pragma unroll
      for (int j = 0; j < kLookbackPerLane; ++j) {
        const int64_t idx = base - int64_t(kLookbackPerLane) * lane - j;
        s[j] = (idx >= 0) ? ld_relaxed(&P.tile_state[idx]) : kStatusIncl;
        ready = ready && ((s[j] & 3u) != 0);
      }
      if (__all_sync(0xFFFFFFFFu, ready)) break;
      if (++polls > kSpinLimit) {
        if (lane == 0) atomicOr(P.error, kErrLookbackTimeout);
#pragma unroll
        for (int j = 0; j < kLookbackPerLane; ++j)
          if ((s[j] & 3u) == 0) s[j] = kStatusIncl;
        break;
      }
      __nanosleep(polls < 64 ? 20 : 500);
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

// NT threads per CTA, two 64-byte words per thread: a tile is NT * 128 bytes
// (NT rows of 128 B, one TMA box).
template <int LMAX, bool kTma, int NT>
__global__ void __launch_bounds__(NT)
    index_kernel(const __grid_constant__ CUtensorMap tmap, const IndexLaunch P) {
  constexpr int NWARPS = NT / 32;
  constexpr uint64_t TILE_BYTES = uint64_t(NT) * 128u;
  static_assert(NT % 32 == 0 && NT <= 256, "one TMA box of at most 256 rows per tile");
  __shared__ __align__(1024) uint8_t s_tile[kTma ? TILE_BYTES : 16];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ uint32_t s_tile_id, s_file_idx;
  __shared__ IndexFile s_file;
  __shared__ uint32_t s_halo;
  __shared__ uint32_t s_last_tp[NWARPS];
  __shared__ uint32_t s_warp_par[NWARPS];
  __shared__ uint32_t s_warp_dd[NWARPS];
  __shared__ uint32_t s_warp_nl[NWARPS];
  __shared__ uint32_t s_prefix_p, s_prefix_d;
  __shared__ unsigned long long s_prefix_n;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;

  if (tid == 0) {
    const uint32_t t = atomicAdd(P.tile_counter, 1u);
    s_tile_id = t;
    if (P.files == nullptr) {
      s_file_idx = 0;
      s_file = P.single;
    } else if (t < P.num_tiles) {
      const uint32_t f = P.tile_file ? P.tile_file[t] : file_of_tile(P, t);
      s_file_idx = f;
      s_file = P.files[f];
    }
    if constexpr (kTma) {
      // the barrier must be initialised before any thread polls it: shared
      // memory may still hold a barrier of an earlier CTA on this SM
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_bar)));
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
  }
  __syncthreads();
  const uint32_t tile = s_tile_id;
  if (tile >= P.num_tiles) return;  // cannot happen with grid == num_tiles
  const IndexFile F = s_file;
  const uint32_t file_idx = s_file_idx;
  const uint32_t ktile = tile - F.first_tile;             // tile within the file
  const bool file_start = ktile == 0;
  const uint64_t byte0 = uint64_t(ktile) * TILE_BYTES;    // tile start within the file
  const uint64_t valid = min(TILE_BYTES, F.n - byte0);    // bytes of the file in the tile
  const uint64_t W = (F.n + 63u) / 64u;                   // words of the file
  const uint8_t *fin = P.in + F.in_off;                   // file bytes
  const int64_t row0 = int64_t((F.in_off + byte0) / 128u);

  if constexpr (kTma) {
    if (tid == 0) {
      const uint32_t bar = smem_u32(&s_bar);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile(
          "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
          "r"(uint32_t(TILE_BYTES))
          : "memory");
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(s_tile)),
          "l"(&tmap), "r"(0), "r"(int32_t(row0)), "r"(bar)
          : "memory");
    }
  }
  // Escape carry into the tile: parity of the backslash run that ends the
  // previous word of the same file (read backward, at most 64 bytes).
  if (tid == 0) {
    uint32_t p = 0;
    if (!file_start) {
      for (int k = 1; k <= 64; ++k) {
        if (fin[byte0 - uint64_t(k)] == '\\') p ^= 1u;
        else break;
      }
    }
    s_halo = p;
  }

  // Thread `tid` owns tile row `tid`: bytes [128 tid, 128 tid + 128) of the
  // tile, i.e. words lw0 and lw0 + 1 of the file.
  const uint64_t row_byte = uint64_t(tid) * 128u;
  const uint64_t lw0 = byte0 / 64u + 2u * uint64_t(tid);
  const bool row_in_smem = kTma && row_byte + 128u <= valid &&
                           row0 + tid < int64_t(P.full_rows);
  if constexpr (kTma) {
    const uint32_t bar = smem_u32(&s_bar);
    uint32_t done = 0, polls = 0;
    while (!done) {
      asm volatile(
          "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;"
          " selp.u32 %0, 1, 0, p; }"
          : "=r"(done)
          : "r"(bar)
          : "memory");
      if (!done && ++polls > kSpinLimit) {
        atomicOr(P.error, kErrTmaTimeout);
        break;
      }
    }
  }
  uint32_t r[16];
  WordClasses c0, c1;
  if (row_in_smem) {
    load_word_smem(s_tile, tid, 0, r);
    c0 = classify64(r);
    load_word_smem(s_tile, tid, 1, r);
    c1 = classify64(r);
  } else {
    // rows past the end of the file read as zero bytes (no class)
    const uint64_t lim = valid > row_byte ? valid - row_byte : 0u;
    const uint8_t *rp = fin + byte0 + row_byte;
    load_word_global(rp, lim, 0, r);
    c0 = classify64(r);
    load_word_global(rp, lim, 64, r);
    c1 = classify64(r);
  }

  // --- escape carries between words --------------------------------------
  const uint32_t tp0 = trailing_escape_parity(c0.bs);
  const uint32_t tp1 = trailing_escape_parity(c1.bs);
  if (lane == 31) s_last_tp[warp] = tp1;
  __syncthreads();  // (1) s_last_tp, s_halo; every thread is past the barrier wait
  if constexpr (kTma) {
    if (tid == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(&s_bar)));
  }
  uint32_t cin0 = __shfl_up_sync(0xFFFFFFFFu, tp1, 1);
  if (lane == 0) cin0 = (warp == 0) ? s_halo : s_last_tp[warp - 1];

  const uint64_t E0 = escaped_bits(c0.bs, cin0);
  const uint64_t E1 = escaped_bits(c1.bs, tp0);
  const uint64_t Q0 = c0.qt & ~E0;
  const uint64_t Q1 = c1.qt & ~E1;
  const uint64_t Sl0 = prefix_xor(Q0);
  const uint64_t Sl1 = prefix_xor(Q1);
  const uint32_t par0 = uint32_t(popc64(Q0)) & 1u;
  const uint32_t par1 = uint32_t(popc64(Q1)) & 1u;

  // depth change of each word if it starts outside a string, and in total
  const int d00 = popc64(c0.op & ~Sl0) - popc64(c0.cl & ~Sl0);
  const int t0 = popc64(c0.op) - popc64(c0.cl);
  const int d10 = popc64(c1.op & ~Sl1) - popc64(c1.cl & ~Sl1);
  const int t1 = popc64(c1.op) - popc64(c1.cl);
  const int thr_d0 = d00 + (par0 ? (t1 - d10) : d10);
  const int thr_t = t0 + t1;
  const uint32_t thr_par = par0 ^ par1;
  const uint32_t thr_nl = uint32_t(popc64(c0.nl) + popc64(c1.nl));

  // --- tile-local exclusive scans ------------------------------------------
  const uint32_t lt_mask = (1u << lane) - 1u;
  const uint32_t par_ballot = __ballot_sync(0xFFFFFFFFu, thr_par);
  uint32_t pex = uint32_t(__popc(par_ballot & lt_mask)) & 1u;
  if (lane == 0) s_warp_par[warp] = uint32_t(__popc(par_ballot)) & 1u;
  __syncthreads();  // (2)
  for (int w = 0; w < warp; ++w) pex ^= s_warp_par[w];
  uint32_t tile_par = 0;
#pragma unroll
  for (int w = 0; w < NWARPS; ++w) tile_par ^= s_warp_par[w];

  // depth changes are only needed mod 256: two 16-bit lanes cannot overflow
  // over at most 256 threads (256 * 255 < 65536)
  const int dt0 = pex ? (thr_t - thr_d0) : thr_d0;
  uint32_t dd = (uint32_t(dt0) & 0xFFu) | ((uint32_t(thr_t) & 0xFFu) << 16);
  uint32_t nl = thr_nl;
  uint32_t dd_inc = dd, nl_inc = nl;
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
    s_warp_dd[warp] = dd_inc;
    s_warp_nl[warp] = nl_inc;
  }
  __syncthreads();  // (3)
  uint32_t dd_ex = dd_inc - dd, nl_ex = nl_inc - nl;
  uint32_t tile_dd = 0, tile_nl = 0;
#pragma unroll
  for (int w = 0; w < NWARPS; ++w) {
    if (w < warp) {
      dd_ex += s_warp_dd[w];
      nl_ex += s_warp_nl[w];
    }
    tile_dd += s_warp_dd[w];
    tile_nl += s_warp_nl[w];
  }

  // --- decoupled look-back --------------------------------------------------
  if (warp == 0) {
    Agg local;
    local.p = tile_par;
    local.d0 = tile_dd & 0xFFu;
    local.d1 = ((tile_dd >> 16) - tile_dd) & 0xFFu;  // total - d0
    local.c = file_start ? 1u : 0u;
    if (file_start) local.d1 = local.d0;  // a file starts outside any string
    local.n = tile_nl;
    const Agg prefix = lookback(P, tile, local);
    if (lane == 0) {
      const Agg incl = agg_combine(prefix, local);
      st_relaxed(&P.tile_state[tile], agg_pack(kStatusIncl, incl));
      // a file start ignores the string state and depth of what precedes it
      s_prefix_p = file_start ? 0u : prefix.p;
      s_prefix_d = file_start ? 0u : prefix.d0;
      s_prefix_n = prefix.n;
      if (P.files == nullptr && tile + 1 == P.num_tiles) {
        P.summary[0] = incl.n + 1u;  // lines = newlines + 1
        P.summary[1] = incl.p;
        P.summary[2] = uint64_t(int64_t(int8_t(uint8_t(incl.d0 - 1u))));
      }
      // newline index of the file starts with 0, at (newlines before it) + f
      if (file_start && prefix.n + file_idx < P.nl_cap) P.NL[prefix.n + file_idx] = 0;
    }
  }
  __syncthreads();  // (4)
  const uint32_t c_in = s_prefix_p;
  const uint32_t d_in = s_prefix_d;
  const uint64_t nl_base = s_prefix_n + nl_ex + file_idx;  // slot of my first newline - 1

  // --- outputs ----------------------------------------------------------------
  const uint32_t car0 = c_in ^ pex;
  const uint32_t car1 = car0 ^ par0;
  const uint64_t S0 = Sl0 ^ (car0 ? ~0ull : 0ull);
  const uint64_t S1 = Sl1 ^ (car1 ? ~0ull : 0ull);
  const uint32_t a_ex = dd_ex & 0xFFu, t_ex = (dd_ex >> 16) & 0xFFu;
  const int depth0 = int(int8_t(uint8_t(d_in - 1u + (c_in ? (t_ex - a_ex) : a_ex))));

  store2(P.S + F.s_off, lw0, W, S0, S1);
  if (P.E != nullptr) {
    store2(P.E + F.s_off, lw0, W, E0 & valid_mask(lw0, F.n), E1 & valid_mask(lw0 + 1, F.n));
    store2(P.Q + F.s_off, lw0, W, Q0, Q1);
  }

  if (F.levels > 0) {
    uint64_t lb0[LMAX], lb1[LMAX];
    const int depth1 =
        leveled_word<LMAX>(c0.op & ~S0, c0.cl & ~S0, c0.sp & ~S0, depth0, lb0);
    leveled_word<LMAX>(c1.op & ~S1, c1.cl & ~S1, c1.sp & ~S1, depth1, lb1);
#pragma unroll
    for (int l = 0; l < LMAX; ++l) {
      if (l < F.levels) store2(P.LB + F.lb_off + uint64_t(l) * W, lw0, W, lb0[l], lb1[l]);
    }
  }

  // newline offsets (every '\n' counts, strings or not), file-local
  uint64_t k = nl_base;
  uint64_t m = c0.nl;
  while (m) {
    const int b = __ffsll(static_cast<long long>(m)) - 1;
    if (k + 1 < P.nl_cap) P.NL[k + 1] = int64_t(lw0 * 64u + uint64_t(b));
    ++k;
    m &= m - 1;
  }
  m = c1.nl;
  while (m) {
    const int b = __ffsll(static_cast<long long>(m)) - 1;
    if (k + 1 < P.nl_cap) P.NL[k + 1] = int64_t((lw0 + 1) * 64u + uint64_t(b));
    ++k;
    m &= m - 1;
  }
}

template <int LMAX, int NT>
cudaError_t launch_levels(const IndexLaunch &L, const CUtensorMap *map, bool use_tma,
                          cudaStream_t stream) {
  const dim3 grid(L.num_tiles), block(NT);
  if (use_tma) {
    index_kernel<LMAX, true, NT><<<grid, block, 0, stream>>>(*map, L);
  } else {
    CUtensorMap dummy{};
    index_kernel<LMAX, false, NT><<<grid, block, 0, stream>>>(dummy, L);
  }
  return cudaGetLastError();
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

cudaError_t index_launch(const IndexLaunch &L, const CUtensorMap *map, bool use_tma,
                         cudaStream_t stream, int threads) {
  if (L.num_tiles == 0) return cudaSuccess;
  const uint64_t scratch = uint64_t(L.num_tiles) * 8u + 64u;
  cudaError_t e = cudaMemsetAsync(L.tile_state, 0, scratch, stream);
  if (e != cudaSuccess) return e;
  if (threads == 128) return launch_threads<128>(L, map, use_tma, stream);
  return launch_threads<256>(L, map, use_tma, stream);
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
