// Serving loop over the index and query kernels (gpj_server_* in
// include/gpjson_b200.h).
//
// Requests are admitted in arrival order whenever one of num_slots streams is
// free and the request's device footprint fits the arena; idle resident
// indexes are evicted least-recently-used first to make room.  Each admitted
// request runs on its own stream, so copies, index builds and queries of
// different requests overlap on the GPU:
//
//   builder:  H2D input -> index kernel -> D2H summary  [event]
//             -> queries -> D2H results                 [event] -> done
//
// Builds are batched: the cache-miss requests admitted in one scheduler pass
// are indexed together by ONE file-table launch of the indexer (the batch
// path's multi-file mode, with every file addressed inside the device
// arena), followed by the per-file finalize kernel and one D2H of the file
// rows; each request's resident index keeps its own input, string-mask and
// leveled-bitmap block, and its newline index is a slice of the pass's
// shared newline block, freed when the last of its residents goes.
//   hit:      queries -> D2H results                    [event] -> done
//   waiter:   (another request is building the same key) waits for that
//             build, then runs its queries like a hit
//
// The scheduler thread owns every CUDA call and the device arena; API calls
// from other threads only touch the queues, the pinned result arena and the
// statistics, all under `mu`.  The device arena is one cudaMalloc made at
// creation, carved by a host-side best-fit allocator, so the loop itself
// never calls cudaMalloc or cudaFree.  A block returns to the arena only
// after the event that follows its last use has completed.
#include "indexer.cuh"
#include "query.cuh"

#include "gpjson_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <iterator>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace gpjb {
int report_error(int code, const char *message);  // capi.cu
}

namespace {

constexpr uint64_t kAlign = 256;
inline uint64_t align_up(uint64_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }
inline uint64_t block_size(uint64_t x) { return align_up(std::max<uint64_t>(x, 1)); }

uint64_t now_ns() {
  return uint64_t(std::chrono::duration_cast<std::chrono::nanoseconds>(
                      std::chrono::steady_clock::now().time_since_epoch())
                      .count());
}

// Best-fit offset allocator over [0, size): free ranges indexed by offset
// (to coalesce neighbours) and by size (to find the smallest fit).  Every
// block is a multiple of 256 bytes and starts on a 256-byte boundary.
class OffsetArena {
 public:
  void reset(uint64_t size) {
    free_.clear();
    by_size_.clear();
    size_ = size & ~(kAlign - 1);
    used_ = peak_ = 0;
    if (size_ > 0) insert(0, size_);
  }
  bool alloc(uint64_t bytes, uint64_t *off) {
    bytes = block_size(bytes);
    auto it = by_size_.lower_bound(bytes);
    if (it == by_size_.end()) return false;
    const uint64_t s = it->first, o = it->second;
    erase(o, s);
    if (s > bytes) insert(o + bytes, s - bytes);
    used_ += bytes;
    peak_ = std::max(peak_, used_);
    *off = o;
    return true;
  }
  void release(uint64_t off, uint64_t bytes) {
    bytes = block_size(bytes);
    used_ -= bytes;
    uint64_t o = off, s = bytes;
    auto next = free_.lower_bound(o);
    if (next != free_.end() && next->first == o + s) {
      s += next->second;
      erase(next->first, next->second);
    }
    auto it = free_.lower_bound(o);
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == o) {
        o = prev->first;
        s += prev->second;
        erase(prev->first, prev->second);
      }
    }
    insert(o, s);
  }
  // Keeps the first `keep` bytes of a block of `bytes` and frees the rest.
  void shrink(uint64_t off, uint64_t bytes, uint64_t keep) {
    bytes = block_size(bytes);
    keep = block_size(keep);
    if (keep < bytes) release(off + keep, bytes - keep);
  }
  uint64_t size() const { return size_; }
  uint64_t used() const { return used_; }
  uint64_t peak() const { return peak_; }

 private:
  void insert(uint64_t o, uint64_t s) {
    free_[o] = s;
    by_size_.emplace(s, o);
  }
  void erase(uint64_t o, uint64_t s) {
    free_.erase(o);
    auto r = by_size_.equal_range(s);
    for (auto i = r.first; i != r.second; ++i)
      if (i->second == o) {
        by_size_.erase(i);
        break;
      }
  }
  std::map<uint64_t, uint64_t> free_;
  std::multimap<uint64_t, uint64_t> by_size_;
  uint64_t size_ = 0, used_ = 0, peak_ = 0;
};

struct Request;

// One grouped build: the newline index of all its files (packed: file f at
// its finalize row's slot), and a metadata block (file table, look-back
// scratch, file rows, totals) with its pinned host mirror, freed once every
// member has read its row.
struct Group {
  uint64_t nl_off = 0, nl_bytes = 0, nl_cap = 0;
  int64_t *NL = nullptr;
  uint64_t meta_off = 0, meta_bytes = 0;
  uint64_t host_off = 0, host_bytes = 0;
  const uint64_t *h_rows = nullptr;  // 8 words per file, then the 4 totals
  uint32_t files = 0;
  int pending = 0;  // members that have not read their row yet
  int refs = 0;     // pending members + residents whose newline index lives here
};

// An index in the device arena: the input copy, string mask and leveled
// bitmaps in one block, the newline index in another (shrunk to its exact
// size once the line count is known).
struct Resident {
  uint64_t key = 0;  // 0: private to one request, freed with it
  uint64_t size = 0;
  int levels = 0;
  uint64_t main_off = 0, main_bytes = 0;
  uint64_t nl_off = 0, nl_bytes = 0, nl_cap = 0;
  Group *nl_group = nullptr;  // newline index inside a grouped build's block
  uint8_t *d_input = nullptr;
  uint64_t *S = nullptr;
  uint64_t *LB = nullptr;
  int64_t *NL = nullptr;
  uint64_t W = 0;
  uint64_t lines = 0;
  bool ready = false;
  int refs = 0;
  bool in_lru = false;
  std::list<Resident *>::iterator lru_it;
  std::vector<Request *> waiters;
};

enum class St { Pending, WaitGroup, Indexing, WaitIndex, WaitMemory, QueryReady, Querying, Done };

// One batched query launch: every query of every request whose index became
// ready in the same scheduler pass runs in ONE launch of the multi-file query
// kernel; each (request, query) pair is one "file" of its table.  Its device
// metadata (file table, file rows, totals, one status word per pair) and the
// pinned host mirror are freed when the last of its requests finishes.
struct QBatch {
  uint64_t meta_off = 0, meta_bytes = 0;
  uint64_t host_off = 0, host_bytes = 0;
  int refs = 0;
};

struct Request {
  uint64_t id = 0;
  uint64_t key = 0;
  const uint8_t *h_input = nullptr;
  uint64_t n = 0;
  std::vector<gpj_batch_query> queries;
  std::vector<std::vector<uint8_t>> irs;
  int levels_needed = 1;
  uint64_t slots_total = 0;
  St state = St::Pending;
  int slot = -1;
  Resident *res = nullptr;
  bool builder = false;
  bool rebuild_pending = false;  // waiting for memory to rebuild a truncated NL
  bool rebuild_copy = false;     // that rebuild must copy the input first
  Group *group = nullptr;        // the grouped build indexing this request
  uint32_t group_file = 0;       // its file (row) in that build
  QBatch *qbatch = nullptr;      // the batched query launch running its queries
  uint32_t status_words = 0;     // its per-query status words in the slot's pinned words
  bool wait_host = false;        // waiting for pinned result memory
  uint64_t work_off = 0, work_bytes = 0, scratch_bytes = 0, result_cap_ints = 0;
  bool has_work = false;
  uint64_t host_off = 0, host_bytes = 0;
  bool has_host = false;
  bool done = false;  // under the server mutex: visible to API callers
  gpj_response resp{};
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t event = nullptr;
  unsigned long long *pinned = nullptr;  // index summary (4 words), counter, error
};

}  // namespace

struct gpj_server {
  gpj_server_config cfg{};
  bool cache_on = true;
  bool sleep_poll = false;
  bool group_builds = true;
  // TMA view of the whole device arena (rows of 128 bytes) for grouped builds
  CUtensorMap arena_map{};
  bool arena_tma = false;
  std::vector<Request *> tick;  // cache misses admitted in this pass, not built yet
  std::unordered_map<Group *, std::unique_ptr<Group>> groups;
  std::vector<Request *> qready;  // requests whose queries run in this pass's batch
  std::unordered_map<QBatch *, std::unique_ptr<QBatch>> qbatches;

  uint8_t *d_arena = nullptr;
  OffsetArena dev;  // scheduler thread only
  int32_t *h_arena = nullptr;
  OffsetArena host;  // under mu
  unsigned long long *h_pinned = nullptr;
  unsigned int *d_status = nullptr;  // one query-status word per slot

  std::vector<Slot> slots;
  std::vector<int> free_slots;  // scheduler thread only

  std::mutex mu;
  std::condition_variable cv_sched, cv_done;
  std::deque<Request *> pending;                                  // under mu
  std::unordered_map<uint64_t, std::unique_ptr<Request>> requests;  // under mu
  std::deque<uint64_t> done_unreported;                           // under mu
  gpj_server_stats stats{};                                       // under mu
  bool stop = false;                                              // under mu
  bool clear_requested = false;                                   // under mu
  uint64_t next_id = 1;                                           // under mu
  // released requests, deleted by the scheduler between its passes (a pass
  // may still hold their pointers)
  std::vector<std::unique_ptr<Request>> graveyard;                // under mu

  // scheduler thread only
  std::unordered_map<uint64_t, Resident *> cache;
  std::list<Resident *> lru;  // idle resident indexes, most recent first
  std::vector<Request *> active;
  std::unordered_map<Resident *, std::unique_ptr<Resident>> residents;
  std::thread thread;

  // ---- device arena -------------------------------------------------------
  void unlink_lru(Resident *r) {
    if (r->in_lru) {
      lru.erase(r->lru_it);
      r->in_lru = false;
    }
  }
  void unref_group(Group *g) {
    if (--g->refs > 0) return;
    if (g->nl_bytes) dev.release(g->nl_off, g->nl_bytes);
    if (g->meta_bytes) dev.release(g->meta_off, g->meta_bytes);
    if (g->host_bytes) host_free(g->host_off, g->host_bytes);
    groups.erase(g);
  }
  // A member has read its row: the metadata block is done with once all have.
  void group_row_read(Group *g) {
    if (--g->pending == 0) {
      if (g->meta_bytes) dev.release(g->meta_off, g->meta_bytes);
      if (g->host_bytes) host_free(g->host_off, g->host_bytes);
      g->meta_bytes = g->host_bytes = 0;
    }
    unref_group(g);
  }
  void free_resident(Resident *r) {
    unlink_lru(r);
    if (r->key != 0) {
      auto it = cache.find(r->key);
      if (it != cache.end() && it->second == r) cache.erase(it);
    }
    if (r->main_bytes) dev.release(r->main_off, r->main_bytes);
    if (r->nl_bytes) dev.release(r->nl_off, r->nl_bytes);
    r->main_bytes = r->nl_bytes = 0;
    if (r->nl_group != nullptr) {
      unref_group(r->nl_group);
      r->nl_group = nullptr;
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      if (r->key != 0 && r->ready) {
        stats.resident_indexes--;
        stats.resident_bytes -= r->size;
      }
      stats.arena_used = dev.used();
    }
    residents.erase(r);
  }
  bool evict_one() {
    if (lru.empty()) return false;
    Resident *victim = lru.back();
    free_resident(victim);
    std::lock_guard<std::mutex> lk(mu);
    stats.evictions++;
    return true;
  }
  // Allocates from the device arena, evicting idle indexes while it does not fit.
  bool dev_alloc(uint64_t bytes, uint64_t *off) {
    for (;;) {
      if (dev.alloc(bytes, off)) {
        std::lock_guard<std::mutex> lk(mu);
        stats.arena_used = dev.used();
        stats.arena_peak = dev.peak();
        return true;
      }
      if (!evict_one()) return false;
    }
  }
  void dev_free(uint64_t off, uint64_t bytes) {
    dev.release(off, bytes);
    std::lock_guard<std::mutex> lk(mu);
    stats.arena_used = dev.used();
  }
  bool host_alloc(uint64_t bytes, uint64_t *off) {
    std::lock_guard<std::mutex> lk(mu);
    return host.alloc(bytes, off);
  }
  void host_free(uint64_t off, uint64_t bytes) {
    std::lock_guard<std::mutex> lk(mu);
    host.release(off, bytes);
  }
  uint8_t *dptr(uint64_t off) const { return d_arena + off; }

  // ---- request lifecycle ----------------------------------------------------
  void release_work(Request *r) {
    if (r->has_work) dev_free(r->work_off, r->work_bytes);
    r->has_work = false;
  }
  void unref(Request *r) {
    Resident *res = r->res;
    r->res = nullptr;
    if (res == nullptr) return;
    res->refs--;
    if (res->refs > 0) return;
    if (res->key == 0 || !res->ready) {
      free_resident(res);
    } else {
      lru.push_front(res);
      res->lru_it = lru.begin();
      res->in_lru = true;
    }
  }
  void unref_qbatch(QBatch *b) {
    if (--b->refs > 0) return;
    if (b->meta_bytes) dev_free(b->meta_off, b->meta_bytes);
    if (b->host_bytes) host_free(b->host_off, b->host_bytes);
    qbatches.erase(b);
  }
  void finish(Request *r, int status, const std::string &msg) {
    if (r->qbatch != nullptr) {
      unref_qbatch(r->qbatch);
      r->qbatch = nullptr;
    }
    {
      auto it = std::find(qready.begin(), qready.end(), r);
      if (it != qready.end()) qready.erase(it);
    }
    release_work(r);
    if (status != GPJ_OK && r->has_host) {
      host_free(r->host_off, r->host_bytes);
      r->has_host = false;
    }
    unref(r);
    if (r->slot >= 0) {
      free_slots.push_back(r->slot);
      r->slot = -1;
    }
    auto it = std::find(active.begin(), active.end(), r);
    if (it != active.end()) active.erase(it);
    r->state = St::Done;
    std::lock_guard<std::mutex> lk(mu);
    r->resp.status = status;
    std::snprintf(r->resp.message, sizeof(r->resp.message), "%s", msg.c_str());
    r->resp.done_ns = now_ns();
    if (status == GPJ_OK) {
      const uint64_t exact = r->resp.result_ints * 4u;
      host.shrink(r->host_off, r->host_bytes, exact);
      r->host_bytes = block_size(exact);
      r->resp.h_results = h_arena + r->host_off / 4u;
      stats.completed++;
      stats.bytes_served += r->n;
    } else {
      r->resp.h_results = nullptr;
      r->resp.result_ints = 0;
      stats.failed++;
    }
    r->done = true;
    done_unreported.push_back(r->id);
    cv_done.notify_all();
  }
  // A failed build fails the requests waiting for it too.
  void fail_build(Request *r, int status, const std::string &msg) {
    Resident *res = r->res;
    if (res != nullptr) {
      std::vector<Request *> waiters;
      waiters.swap(res->waiters);
      if (res->key != 0) {
        auto it = cache.find(res->key);
        if (it != cache.end() && it->second == res) cache.erase(it);
        res->key = 0;  // freed with its last user
      }
      for (Request *w : waiters) finish(w, status, msg);
    }
    finish(r, status, msg);
  }

  int cuda_status(cudaError_t e) {
    (void)cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? GPJ_ERR_OOM : GPJ_ERR_CUDA;
  }

  // Enqueues (copy and) index build of the request's resident index.
  bool enqueue_build(Request *r, bool copy) {
    Resident *res = r->res;
    Slot &s = slots[r->slot];
    cudaError_t e = cudaSuccess;
    if (copy && res->size > 0)
      e = cudaMemcpyAsync(res->d_input, r->h_input, res->size, cudaMemcpyHostToDevice, s.stream);
    if (e == cudaSuccess && res->size == 0) {
      // no tiles: NL = [0], one line; the summary is set here (no kernel)
      e = cudaMemsetAsync(res->NL, 0, 8, s.stream);
      std::memset(s.pinned, 0, 64);
      s.pinned[0] = 1ull;
    } else if (e == cudaSuccess) {
      gpjb::IndexLaunch L;
      L.single.n = res->size;
      L.single.levels = res->levels;
      L.num_levels = res->levels;
      L.full_rows = res->size / 128u;
      L.S = res->S;
      L.LB = res->LB;
      L.NL = res->NL;
      L.nl_cap = res->nl_cap;
      L.num_tiles = uint32_t(gpjb::index_num_tiles(res->size));
      L.in = res->d_input;
      gpjb::index_bind_scratch(L, dptr(r->work_off));
      CUtensorMap map;
      const bool tma = gpjb::index_make_tensor_map(&map, res->d_input, res->size);
      e = gpjb::index_launch(L, tma ? &map : nullptr, tma, s.stream);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(s.pinned, L.summary, 40, cudaMemcpyDeviceToHost, s.stream);
    }
    if (e == cudaSuccess) e = cudaEventRecord(s.event, s.stream);
    if (e != cudaSuccess) {
      fail_build(r, cuda_status(e), std::string("index build: ") + cudaGetErrorString(e));
      return false;
    }
    if (res->size > 0) {
      std::lock_guard<std::mutex> lk(mu);
      stats.index_launches++;
    }
    r->state = St::Indexing;
    return true;
  }

  // Makes sure the request's device and host result blocks hold its exact
  // result ints; false: no memory now (the request waits).
  bool ensure_results(Request *r, uint64_t ints) {
    r->wait_host = false;
    if (!r->has_work || r->result_cap_ints < ints) {
      release_work(r);
      uint64_t off = 0;
      if (!dev_alloc(ints * 4u, &off)) return false;
      r->work_off = off;
      r->work_bytes = block_size(ints * 4u);
      r->scratch_bytes = 0;
      r->result_cap_ints = ints;
      r->has_work = true;
    }
    if (!r->has_host || r->host_bytes < ints * 4u) {
      if (r->has_host) host_free(r->host_off, r->host_bytes);
      r->has_host = false;
      uint64_t off = 0;
      if (!host_alloc(ints * 4u, &off)) {
        r->wait_host = true;  // freed by gpj_server_release, not by eviction
        return false;
      }
      r->host_off = off;
      r->host_bytes = block_size(ints * 4u);
      r->has_host = true;
    }
    return true;
  }

  // Launches the queries of a request whose index is ready, then the copy of
  // its results to the pinned arena.
  // The queries of a request whose index is ready join this pass's batched
  // launch (flush_queries); an empty file runs alone (no kernel).
  void launch_queries(Request *r) {
    Resident *res = r->res;
    const uint64_t ints = res->lines * r->slots_total * 2u;
    if (!ensure_results(r, ints)) {
      r->state = St::WaitMemory;
      return;
    }
    if (res->size == 0 || !group_builds) {
      launch_queries_alone(r);
      return;
    }
    r->state = St::QueryReady;
    qready.push_back(r);
  }

  void launch_queries_alone(Request *r) {
    Resident *res = r->res;
    const uint64_t lines = res->lines;
    const uint64_t ints = lines * r->slots_total * 2u;
    if (!ensure_results(r, ints)) {
      r->state = St::WaitMemory;
      return;
    }
    r->status_words = 0;
    Slot &s = slots[r->slot];
    int32_t *d_out = reinterpret_cast<int32_t *>(dptr(r->work_off + r->scratch_bytes));
    cudaError_t e = cudaSuccess;
    uint64_t off = 0;
    for (size_t q = 0; q < r->queries.size(); ++q) {
      r->resp.result_offset[q] = off;
      off += lines * r->queries[q].num_result_slots * 2u;
    }
    unsigned int *d_status = this->d_status + r->slot;
    auto *h_status = reinterpret_cast<unsigned int *>(s.pinned + 7);
    *h_status = 0;
    if (res->size == 0) {
      if (ints > 0) e = cudaMemsetAsync(d_out, 0xFF, ints * 4u, s.stream);
    } else {
      e = cudaMemsetAsync(d_status, 0, 4, s.stream);
      for (size_t q = 0; q < r->queries.size() && e == cudaSuccess; ++q) {
        const gpj_batch_query &bq = r->queries[q];
        gpjb::QueryLaunch ql;
        ql.in = res->d_input;
        ql.n = int64_t(res->size);
        ql.NL = res->NL;
        ql.num_lines = int64_t(lines);
        ql.S = res->S;
        ql.LB = res->LB;
        ql.W = int64_t(res->W);
        ql.ir_len = int(bq.ir_len);
        ql.num_results = int(bq.num_result_slots);
        ql.num_levels = res->levels;
        ql.base_level = int(bq.base_level);
        ql.out32 = d_out + r->resp.result_offset[q];
        ql.status = d_status;
        if (bq.num_result_slots == 0) continue;
        gpjb::IrBlob blob;
        std::memset(blob.bytes, 0, sizeof(blob.bytes));
        std::memcpy(blob.bytes, r->irs[q].data(), r->irs[q].size());
        e = gpjb::query_launch(ql, blob, 0, 256, s.stream);
      }
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_status, d_status, 4, cudaMemcpyDeviceToHost, s.stream);
    }
    if (e == cudaSuccess && ints > 0)
      e = cudaMemcpyAsync(h_arena + r->host_off / 4u, d_out, ints * 4u, cudaMemcpyDeviceToHost,
                          s.stream);
    if (e == cudaSuccess) e = cudaEventRecord(s.event, s.stream);
    if (e != cudaSuccess) {
      finish(r, cuda_status(e), std::string("query: ") + cudaGetErrorString(e));
      return;
    }
    r->resp.num_lines = lines;
    r->resp.result_ints = ints;
    r->state = St::Querying;
  }

  // The builder's index kernel finished: check it, publish the index, start
  // the queries of the builder and of every request waiting for it.
  void on_index_done(Request *r) {
    Resident *res = r->res;
    if (r->group != nullptr) {
      on_group_member_done(r);
      return;
    }
    const unsigned long long *p = slots[r->slot].pinned;
    const uint64_t lines = p[0];
    const uint32_t err = reinterpret_cast<const uint32_t *>(p)[9];
    if (res->size > 0 && err != 0) {
      fail_build(r, GPJ_ERR_TIMEOUT,
                 "index kernel: a bounded wait gave up (error bits " + std::to_string(err) + ")");
      return;
    }
    if (lines > res->nl_cap) {
      // the newline index was truncated: rebuild with the exact capacity
      {
        std::lock_guard<std::mutex> lk(mu);
        stats.rebuilds++;
      }
      dev_free(res->nl_off, res->nl_bytes);
      res->nl_bytes = 0;
      res->nl_cap = lines;
      r->rebuild_pending = true;
      retry_rebuild(r);
      return;
    }
    if (res->nl_bytes > block_size(lines * 8u)) {
      dev.shrink(res->nl_off, res->nl_bytes, lines * 8u);
      res->nl_bytes = block_size(lines * 8u);
    }
    publish_index(r, lines);
  }

  // A member of a grouped build: its row of the finalize output gives its
  // line count and newline slot; the totals give the launch's error bits and
  // the newline slots the group needed.
  void on_group_member_done(Request *r) {
    Resident *res = r->res;
    Group *g = r->group;
    r->group = nullptr;
    const uint64_t *row = g->h_rows + uint64_t(r->group_file) * 8u;
    const uint64_t *tot = g->h_rows + uint64_t(g->files) * 8u;
    const uint64_t lines = row[gpjb::kFiLines];
    const uint64_t err = tot[gpjb::kTotError];
    if (err != 0) {
      group_row_read(g);
      fail_build(r, GPJ_ERR_TIMEOUT,
                 "grouped index build: a bounded wait gave up (error bits " + std::to_string(err) +
                     ")");
      return;
    }
    if (tot[gpjb::kTotNlSlots] > g->nl_cap) {
      // the group's newline block was too small: this member's index is
      // built again on its own with its exact line count
      group_row_read(g);
      {
        std::lock_guard<std::mutex> lk(mu);
        stats.rebuilds++;
      }
      res->nl_cap = lines;
      r->rebuild_pending = true;
      retry_rebuild(r);
      return;
    }
    res->NL = g->NL + row[gpjb::kFiNlOff];
    res->nl_group = g;
    g->refs++;  // held by the resident until it is freed
    group_row_read(g);
    publish_index(r, lines);
  }

  // The index of a builder is complete: publish it and start the queries of
  // the builder and of every request waiting for it.
  void publish_index(Request *r, uint64_t lines) {
    Resident *res = r->res;
    res->lines = lines;
    res->ready = true;
    if (res->key != 0) {
      std::lock_guard<std::mutex> lk(mu);
      stats.resident_indexes++;
      stats.resident_bytes += res->size;
      stats.arena_used = dev.used();
    }
    const uint64_t t = now_ns();
    std::vector<Request *> waiters;
    waiters.swap(res->waiters);
    r->resp.index_ready_ns = t;
    launch_queries(r);
    for (Request *w : waiters) {
      w->resp.index_ready_ns = t;
      launch_queries(w);
    }
  }
  void retry_rebuild(Request *r) {
    Resident *res = r->res;
    uint64_t off = 0;
    if (!dev_alloc(res->nl_cap * 8u, &off)) {
      r->state = St::WaitMemory;
      return;
    }
    res->nl_off = off;
    res->nl_bytes = block_size(res->nl_cap * 8u);
    res->NL = reinterpret_cast<int64_t *>(dptr(off));
    r->rebuild_pending = false;
    const bool copy = r->rebuild_copy;
    r->rebuild_copy = false;
    enqueue_build(r, copy);
  }

  // 1: admitted (or finished with an error), 0: does not fit yet.
  int try_admit(Request *r) {
    Resident *res = nullptr;
    if (cache_on && r->key != 0) {
      auto it = cache.find(r->key);
      if (it != cache.end()) {
        Resident *e = it->second;
        if (e->size == r->n && e->levels >= r->levels_needed) {
          res = e;
        } else if (e->refs == 0 && e->ready) {
          free_resident(e);  // stale shape: replaced below
          std::lock_guard<std::mutex> lk(mu);
          stats.evictions++;
        }
      }
    }
    const bool build = (res == nullptr);
    const bool cacheable = build && cache_on && r->key != 0 && cache.find(r->key) == cache.end();
    const int levels =
        build ? std::min(GPJ_MAX_LEVELS, cacheable ? std::max(r->levels_needed, cfg.cache_levels)
                                                   : r->levels_needed)
              : res->levels;
    const uint64_t n = r->n;
    const uint64_t W = (n + 63u) / 64u;
    const uint64_t in_bytes = align_up(n), s_bytes = align_up(W * 8u),
                   lb_bytes = align_up(W * 8u * uint64_t(levels));
    const uint64_t main_bytes = block_size(in_bytes + s_bytes + lb_bytes);
    const uint64_t nl_cap = n / 32u + 1024u;
    const uint64_t scratch = build ? align_up(gpjb::index_scratch_bytes(n)) : 0u;
    const uint64_t lines_guess = build ? nl_cap : (res->ready ? res->lines : res->nl_cap);
    const uint64_t ints = lines_guess * r->slots_total * 2u;
    const uint64_t work_bytes = block_size(scratch + ints * 4u);
    // a build of this pass is grouped with the others: its newline index goes
    // to the group's shared block, allocated when the pass ends
    const bool grouped = build && group_builds;
    const uint64_t need = work_bytes + (build ? main_bytes + block_size(nl_cap * 8u) : 0u);
    if (need > dev.size()) {
      finish(r, GPJ_ERR_OOM,
             "request needs " + std::to_string(need) + " bytes of device memory; the budget is " +
                 std::to_string(dev.size()));
      return 1;
    }
    if (block_size(ints * 4u) > host.size()) {
      finish(r, GPJ_ERR_OOM, "request results exceed the pinned result arena");
      return 1;
    }
    // pin a resident hit before allocating (allocation may evict idle indexes)
    if (!build) {
      res->refs++;
      unlink_lru(res);
    }
    uint64_t main_off = 0, nl_off = 0, work_off = 0, host_off = 0;
    bool ok_main = !build, ok_nl = !build, ok_work = false, ok_host = false;
    if (build) ok_main = dev_alloc(main_bytes, &main_off);
    if (build && ok_main) ok_nl = grouped || dev_alloc(nl_cap * 8u, &nl_off);
    if (ok_main && ok_nl) ok_work = dev_alloc(work_bytes, &work_off);
    if (ok_work) ok_host = host_alloc(ints * 4u, &host_off);
    if (!ok_host) {
      if (ok_work) dev_free(work_off, work_bytes);
      if (build && ok_nl && !grouped) dev_free(nl_off, nl_cap * 8u);
      if (build && ok_main) dev_free(main_off, main_bytes);
      if (!build) {
        res->refs--;
        if (res->refs == 0 && res->ready) {
          lru.push_front(res);
          res->lru_it = lru.begin();
          res->in_lru = true;
        }
      }
      if (active.empty() && lru.empty()) {
        finish(r, GPJ_ERR_OOM,
               ok_work ? "pinned result arena full: release finished responses"
                       : "request does not fit the device arena");
        return 1;
      }
      return 0;
    }
    r->work_off = work_off;
    r->work_bytes = work_bytes;
    r->scratch_bytes = scratch;
    r->result_cap_ints = ints;
    r->has_work = true;
    r->host_off = host_off;
    r->host_bytes = block_size(ints * 4u);
    r->has_host = true;
    r->slot = free_slots.back();
    free_slots.pop_back();
    r->resp.admit_ns = now_ns();
    active.push_back(r);
    if (build) {
      auto owned = std::make_unique<Resident>();
      res = owned.get();
      residents.emplace(res, std::move(owned));
      res->key = cacheable ? r->key : 0u;
      res->size = n;
      res->levels = levels;
      res->main_off = main_off;
      res->main_bytes = main_bytes;
      res->nl_off = nl_off;
      res->nl_bytes = grouped ? 0u : block_size(nl_cap * 8u);
      res->nl_cap = nl_cap;
      res->W = W;
      res->d_input = dptr(main_off);
      res->S = reinterpret_cast<uint64_t *>(dptr(main_off + in_bytes));
      res->LB = reinterpret_cast<uint64_t *>(dptr(main_off + in_bytes + s_bytes));
      res->NL = grouped ? nullptr : reinterpret_cast<int64_t *>(dptr(nl_off));
      res->refs = 1;
      if (cacheable) cache[r->key] = res;
      r->res = res;
      r->builder = true;
      {
        std::lock_guard<std::mutex> lk(mu);
        stats.cache_misses++;
        stats.bytes_indexed += n;
      }
      if (grouped) {
        r->state = St::WaitGroup;
        tick.push_back(r);
      } else {
        enqueue_build(r, true);
      }
    } else {
      r->res = res;
      r->resp.cache_hit = 1;
      {
        std::lock_guard<std::mutex> lk(mu);
        stats.cache_hits++;
      }
      if (res->ready) {
        r->resp.index_ready_ns = r->resp.admit_ns;
        launch_queries(r);
      } else {
        r->state = St::WaitIndex;
        res->waiters.push_back(r);
      }
    }
    return 1;
  }

  bool query_overflow(const Request *r) const {
    const unsigned long long *p = slots[r->slot].pinned;
    unsigned int bits = 0;
    if (r->status_words == 0) {
      bits = *reinterpret_cast<const unsigned int *>(p + 7);
    } else {
      const auto *w = reinterpret_cast<const unsigned int *>(p + 4);
      for (uint32_t k = 0; k < r->status_words; ++k) bits |= w[k];
    }
    return (bits & gpjb::kQueryStatusOverflow) != 0;
  }

  // One launch of the multi-file query kernel for every request in qready:
  // a "file" per (request, query) pair, addressed inside the device arena
  // (input, bitmaps, newline index, results), with its own status word; then
  // per request a D2H of its results and status words and its event.
  void flush_queries() {
    if (qready.empty()) return;
    std::vector<Request *> reqs;
    reqs.swap(qready);
    // pairs and distinct query IRs (the kernel takes up to kMaxBatchGroups)
    struct Pair { Request *r; uint32_t q; uint32_t group; };
    std::vector<Pair> pairs;
    std::vector<const Request *> group_req;
    std::vector<uint32_t> group_q;
    std::vector<Request *> in_batch, alone;
    uint64_t ir_bytes = 0;
    for (Request *r : reqs) {
      std::vector<Pair> mine;
      bool fits = true;
      uint64_t added_ir = 0;
      std::vector<std::pair<const Request *, uint32_t>> new_groups;
      for (uint32_t q = 0; q < r->queries.size(); ++q) {
        const gpj_batch_query &bq = r->queries[q];
        uint32_t g = 0;
        bool found = false;
        for (; g < group_req.size(); ++g) {
          const gpj_batch_query &o = group_req[g]->queries[group_q[g]];
          if (o.num_result_slots == bq.num_result_slots && o.base_level == bq.base_level &&
              group_req[g]->irs[group_q[g]] == r->irs[q]) {
            found = true;
            break;
          }
        }
        if (!found) {
          for (size_t k = 0; k < new_groups.size(); ++k) {
            const Request *nr = new_groups[k].first;
            const uint32_t nq = new_groups[k].second;
            if (nr->queries[nq].num_result_slots == bq.num_result_slots &&
                nr->queries[nq].base_level == bq.base_level && nr->irs[nq] == r->irs[q]) {
              g = uint32_t(group_req.size() + k);
              found = true;
              break;
            }
          }
        }
        if (!found) {
          g = uint32_t(group_req.size() + new_groups.size());
          new_groups.emplace_back(r, q);
          added_ir += r->irs[q].size();
        }
        mine.push_back(Pair{r, q, g});
      }
      if (group_req.size() + new_groups.size() > size_t(gpjb::kMaxBatchGroups) ||
          ir_bytes + added_ir > uint64_t(gpjb::kMaxQueryIrBytes))
        fits = false;
      if (!fits) {
        alone.push_back(r);
        continue;
      }
      for (auto &ng : new_groups) {
        group_req.push_back(ng.first);
        group_q.push_back(ng.second);
      }
      ir_bytes += added_ir;
      pairs.insert(pairs.end(), mine.begin(), mine.end());
      in_batch.push_back(r);
    }
    for (Request *r : alone) launch_queries_alone(r);
    if (in_batch.empty()) return;
    const uint64_t V = pairs.size();
    const uint64_t files_bytes = align_up(V * sizeof(gpjb::IndexFile));
    const uint64_t rows_bytes = align_up(V * 64u + 32u);
    const uint64_t meta_bytes = files_bytes + rows_bytes + align_up(V * 4u);
    const uint64_t host_bytes = files_bytes + rows_bytes;
    auto owned = std::make_unique<QBatch>();
    QBatch *b = owned.get();
    bool ok = dev_alloc(meta_bytes, &b->meta_off);
    if (ok) b->meta_bytes = block_size(meta_bytes);
    ok = ok && host_alloc(host_bytes, &b->host_off);
    if (ok) b->host_bytes = block_size(host_bytes);
    if (!ok) {
      if (b->meta_bytes) dev_free(b->meta_off, b->meta_bytes);
      for (Request *r : in_batch) launch_queries_alone(r);
      return;
    }
    auto *h_files = reinterpret_cast<gpjb::IndexFile *>(
        reinterpret_cast<uint8_t *>(h_arena) + b->host_off);
    auto *h_rows = reinterpret_cast<uint64_t *>(
        reinterpret_cast<uint8_t *>(h_arena) + b->host_off + files_bytes);
    auto *d_files = reinterpret_cast<gpjb::IndexFile *>(dptr(b->meta_off));
    auto *d_rows = reinterpret_cast<uint64_t *>(dptr(b->meta_off + files_bytes));
    auto *d_stat = reinterpret_cast<unsigned int *>(dptr(b->meta_off + files_bytes + rows_bytes));
    uint64_t records = 0;
    for (uint64_t v = 0; v < V; ++v) {
      const Pair &pr = pairs[v];
      Request *r = pr.r;
      const Resident *res = r->res;
      const gpj_batch_query &bq = r->queries[pr.q];
      uint64_t off = 0;
      for (uint32_t q = 0; q < pr.q; ++q) off += res->lines * r->queries[q].num_result_slots * 2u;
      r->resp.result_offset[pr.q] = off;
      gpjb::IndexFile F;
      F.in_off = uint64_t(res->d_input - d_arena);
      F.n = res->size;
      F.s_off = uint64_t(reinterpret_cast<uint8_t *>(res->S) - d_arena) / 8u;
      F.lb_off = uint64_t(reinterpret_cast<uint8_t *>(res->LB) - d_arena) / 8u;
      F.first_tile = 0;
      F.levels = res->levels;
      h_files[v] = F;
      uint64_t *row = h_rows + v * 8u;
      const uint64_t out_int = (r->work_off + r->scratch_bytes) / 4u + off;
      row[gpjb::kFiLines] = res->lines;
      row[gpjb::kFiNlOff] = uint64_t(reinterpret_cast<uint8_t *>(res->NL) - d_arena) / 8u;
      row[gpjb::kFiRecOff] = records;
      row[gpjb::kFiOutOff] = out_int;
      row[gpjb::kFiInString] = 0;
      row[gpjb::kFiDepth] = 0;
      row[gpjb::kFiBytes] = res->size;
      row[gpjb::kFiQuery] = pr.group;
      records += bq.num_result_slots > 0 ? res->lines : 0u;
      if (bq.num_result_slots == 0) row[gpjb::kFiLines] = 0;
    }
    uint64_t *h_tot = h_rows + V * 8u;
    h_tot[gpjb::kTotRecords] = records;
    h_tot[gpjb::kTotResultInts] = 0;
    h_tot[gpjb::kTotNlSlots] = 0;
    h_tot[gpjb::kTotError] = 0;
    gpjb::BatchQueryLaunch ql;
    ql.in = d_arena;
    ql.S = reinterpret_cast<const uint64_t *>(d_arena);
    ql.LB = reinterpret_cast<const uint64_t *>(d_arena);
    ql.NL = reinterpret_cast<const int64_t *>(d_arena);
    ql.files = d_files;
    ql.num_files = uint32_t(V);
    ql.file_info = d_rows;
    ql.totals = d_rows + V * 8u;
    ql.out = reinterpret_cast<int32_t *>(d_arena);
    ql.file_status = d_stat;
    ql.num_groups = int(group_req.size());
    gpjb::IrBlob blob;
    std::memset(blob.bytes, 0, sizeof(blob.bytes));
    int ir_off = 0;
    for (size_t g = 0; g < group_req.size(); ++g) {
      const Request *gr = group_req[g];
      const uint32_t gq = group_q[g];
      std::memcpy(blob.bytes + ir_off, gr->irs[gq].data(), gr->irs[gq].size());
      ql.groups[g].ir_off = ir_off;
      ql.groups[g].ir_len = int(gr->irs[gq].size());
      ql.groups[g].num_results = int(gr->queries[gq].num_result_slots);
      ql.groups[g].base_level = int(gr->queries[gq].base_level);
      ir_off += int(gr->irs[gq].size());
    }
    Slot &s0 = slots[in_batch[0]->slot];
    cudaError_t e = cudaMemcpyAsync(d_files, h_files, files_bytes + V * 64u + 32u,
                                    cudaMemcpyHostToDevice, s0.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_stat, 0, V * 4u, s0.stream);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cfg.device);
    const uint64_t blocks = (records + 127u) / 128u;
    const int grid = int(std::max<uint64_t>(1, std::min<uint64_t>(blocks, uint64_t(sms) * 8u)));
    if (e == cudaSuccess && records > 0) e = gpjb::batch_query_launch(ql, blob, grid, 128, s0.stream);
    b->refs = int(in_batch.size());
    qbatches.emplace(b, std::move(owned));
    uint64_t v = 0;
    for (Request *r : in_batch) {
      Slot &s = slots[r->slot];
      const uint64_t ints = r->res->lines * r->slots_total * 2u;
      const uint32_t nq = uint32_t(r->queries.size());
      r->qbatch = b;
      r->status_words = nq;
      if (e == cudaSuccess && ints > 0)
        e = cudaMemcpyAsync(h_arena + r->host_off / 4u, dptr(r->work_off + r->scratch_bytes),
                            ints * 4u, cudaMemcpyDeviceToHost, s0.stream);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(reinterpret_cast<unsigned int *>(s.pinned + 4), d_stat + v, nq * 4u,
                            cudaMemcpyDeviceToHost, s0.stream);
      if (e == cudaSuccess) e = cudaEventRecord(s.event, s0.stream);
      v += nq;
      r->resp.num_lines = r->res->lines;
      r->resp.result_ints = ints;
      r->state = St::Querying;
    }
    if (e != cudaSuccess) {
      const std::string msg = std::string("batched query: ") + cudaGetErrorString(e);
      const int code = cuda_status(e);
      for (Request *r : in_batch) finish(r, code, msg);
    }
  }

  bool advance() {
    bool any = false;
    const std::vector<Request *> snap(active);
    for (Request *r : snap) {
      if (r->state == St::Indexing || r->state == St::Querying) {
        const cudaError_t e = cudaEventQuery(slots[r->slot].event);
        if (e == cudaErrorNotReady) continue;
        any = true;
        if (e != cudaSuccess) {
          const std::string msg = std::string("device work failed: ") + cudaGetErrorString(e);
          if (r->state == St::Indexing) fail_build(r, cuda_status(e), msg);
          else finish(r, cuda_status(e), msg);
        } else if (r->state == St::Indexing) {
          on_index_done(r);
        } else if (query_overflow(r)) {
          finish(r, GPJ_ERR_CAPACITY,
                 "a record has more results than result slots; the results are truncated");
        } else {
          finish(r, GPJ_OK, "");
        }
      } else if (r->state == St::WaitMemory) {
        if (r->rebuild_pending) retry_rebuild(r);
        else launch_queries(r);
        if (r->state != St::WaitMemory) any = true;
      }
      // St::WaitIndex progresses with its builder
    }
    if (any || active.empty()) return any;
    // Every admitted request waits for device memory, nothing runs that
    // could free some and nothing is left to evict: fail the oldest waiter.
    for (Request *r : active)
      if (r->state == St::Indexing || r->state == St::Querying || r->wait_host) return false;
    if (!lru.empty()) return false;
    for (Request *r : active)
      if (r->state == St::WaitMemory) {
        if (r->rebuild_pending)
          fail_build(r, GPJ_ERR_OOM, "no device memory to rebuild the newline index");
        else
          finish(r, GPJ_ERR_OOM, "no device memory for the results");
        return true;
      }
    return false;
  }

  bool admit() {
    bool any = false;
    for (;;) {
      Request *r = nullptr;
      {
        std::lock_guard<std::mutex> lk(mu);
        if (pending.empty() || free_slots.empty()) break;
        r = pending.front();
      }
      if (try_admit(r) == 0) break;
      {
        std::lock_guard<std::mutex> lk(mu);
        pending.pop_front();
      }
      any = true;
    }
    flush_tick();
    return any;
  }

  // ---- grouped builds --------------------------------------------------------
  // A build that leaves the group path: its own newline block, then the
  // single-file launch (or a wait for memory, retried by advance()).
  void build_alone(Request *r) {
    Resident *res = r->res;
    uint64_t off = 0;
    if (!dev_alloc(res->nl_cap * 8u, &off)) {
      r->rebuild_pending = true;
      r->rebuild_copy = true;
      r->state = St::WaitMemory;
      return;
    }
    res->nl_off = off;
    res->nl_bytes = block_size(res->nl_cap * 8u);
    res->NL = reinterpret_cast<int64_t *>(dptr(off));
    enqueue_build(r, true);
  }

  void flush_tick() {
    if (tick.empty()) return;
    std::vector<Request *> members;
    members.swap(tick);
    if (members.size() == 1 || !enqueue_group(members))
      for (Request *r : members) build_alone(r);
  }

  // Indexes every member with one file-table launch on the first member's
  // stream: H2D of the inputs and the file table, indexer, finalize, one D2H
  // of the file rows and totals; every member's event is recorded after it.
  // false: no memory for the group's blocks (nothing was enqueued).
  bool enqueue_group(const std::vector<Request *> &members) {
    const uint32_t G = uint32_t(members.size());
    uint64_t tiles = 0, nl_cap = 0;
    int levels = 0;
    for (Request *r : members) {
      tiles += gpjb::tiles_for(r->res->size, gpjb::kIndexThreads);
      nl_cap += r->res->nl_cap;
      levels = std::max(levels, r->res->levels);
    }
    const uint64_t files_bytes = align_up(uint64_t(G) * sizeof(gpjb::IndexFile));
    const uint64_t scratch_bytes = align_up(tiles * 8u + 64u);
    const uint64_t rows_bytes = uint64_t(G) * 64u + 32u;
    const uint64_t meta_bytes = files_bytes + scratch_bytes + align_up(rows_bytes);
    const uint64_t host_bytes = files_bytes + align_up(rows_bytes);
    auto owned = std::make_unique<Group>();
    Group *g = owned.get();
    bool ok = dev_alloc(nl_cap * 8u, &g->nl_off);
    if (ok) g->nl_bytes = block_size(nl_cap * 8u);
    ok = ok && dev_alloc(meta_bytes, &g->meta_off);
    if (ok) g->meta_bytes = block_size(meta_bytes);
    ok = ok && host_alloc(host_bytes, &g->host_off);
    if (ok) g->host_bytes = block_size(host_bytes);
    if (!ok) {
      if (g->nl_bytes) dev_free(g->nl_off, g->nl_bytes);
      if (g->meta_bytes) dev_free(g->meta_off, g->meta_bytes);
      return false;
    }
    g->nl_cap = nl_cap;
    g->NL = reinterpret_cast<int64_t *>(dptr(g->nl_off));
    g->files = G;
    auto *h_files = reinterpret_cast<gpjb::IndexFile *>(
        reinterpret_cast<uint8_t *>(h_arena) + g->host_off);
    g->h_rows = reinterpret_cast<const uint64_t *>(
        reinterpret_cast<uint8_t *>(h_arena) + g->host_off + files_bytes);
    uint64_t first = 0;
    for (uint32_t f = 0; f < G; ++f) {
      const Resident *res = members[f]->res;
      gpjb::IndexFile F;
      F.in_off = res->main_off;
      F.n = res->size;
      F.s_off = uint64_t(reinterpret_cast<uint8_t *>(res->S) - d_arena) / 8u;
      F.lb_off = uint64_t(reinterpret_cast<uint8_t *>(res->LB) - d_arena) / 8u;
      F.first_tile = uint32_t(first);
      F.levels = res->levels;
      h_files[f] = F;
      first += gpjb::tiles_for(res->size, gpjb::kIndexThreads);
    }
    auto *d_files = reinterpret_cast<gpjb::IndexFile *>(dptr(g->meta_off));
    auto *d_rows = reinterpret_cast<uint64_t *>(dptr(g->meta_off + files_bytes + scratch_bytes));
    gpjb::IndexLaunch L;
    L.in = d_arena;
    L.full_rows = dev.size() / 128u;
    L.files = d_files;
    L.num_files = G;
    L.num_levels = levels;
    L.S = reinterpret_cast<uint64_t *>(d_arena);
    L.LB = reinterpret_cast<uint64_t *>(d_arena);
    L.NL = g->NL;
    L.nl_cap = nl_cap;
    L.num_tiles = uint32_t(tiles);
    gpjb::index_bind_scratch(L, dptr(g->meta_off + files_bytes));
    Slot &s = slots[members[0]->slot];
    cudaError_t e = cudaSuccess;
    for (Request *r : members)
      if (e == cudaSuccess && r->res->size > 0)
        e = cudaMemcpyAsync(r->res->d_input, r->h_input, r->res->size, cudaMemcpyHostToDevice,
                            s.stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_files, h_files, uint64_t(G) * sizeof(gpjb::IndexFile),
                          cudaMemcpyHostToDevice, s.stream);
    if (e == cudaSuccess && tiles > 0)
      e = gpjb::index_launch(L, arena_tma ? &arena_map : nullptr, arena_tma, s.stream);
    if (e == cudaSuccess && tiles == 0)
      e = gpjb::index_clear_scratch(L, s.stream);
    if (e == cudaSuccess)
      e = gpjb::index_finalize_files(L, nullptr, nullptr, d_rows, d_rows + uint64_t(G) * 8u,
                                     s.stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(const_cast<uint64_t *>(g->h_rows), d_rows, rows_bytes,
                          cudaMemcpyDeviceToHost, s.stream);
    for (Request *r : members) {
      if (e == cudaSuccess) e = cudaEventRecord(slots[r->slot].event, s.stream);
    }
    groups.emplace(g, std::move(owned));
    g->pending = int(G);
    g->refs = int(G);
    {
      std::lock_guard<std::mutex> lk(mu);
      stats.index_launches++;
    }
    for (uint32_t f = 0; f < G; ++f) {
      Request *r = members[f];
      r->group = g;
      r->group_file = f;
      r->state = St::Indexing;
    }
    if (e != cudaSuccess) {
      const std::string msg = std::string("grouped index build: ") + cudaGetErrorString(e);
      const int code = cuda_status(e);
      for (Request *r : members) {
        r->group = nullptr;
        group_row_read(g);
        fail_build(r, code, msg);
      }
    }
    return true;
  }

  void clear_idle() {
    while (evict_one()) {
    }
  }

  void loop() {
    cudaSetDevice(cfg.device);
    for (;;) {
      bool clear = false;
      {
        std::lock_guard<std::mutex> lk(mu);
        graveyard.clear();
        clear = clear_requested;
      }
      if (clear) {
        clear_idle();
        std::lock_guard<std::mutex> lk(mu);
        clear_requested = false;
        cv_done.notify_all();
      }
      bool progressed = advance();
      progressed = admit() || progressed;
      flush_queries();
      std::unique_lock<std::mutex> lk(mu);
      stats.in_flight = active.size();
      stats.pending = pending.size();
      if (stop && pending.empty() && active.empty()) break;
      if (progressed || clear_requested) continue;
      if (!active.empty()) {
        lk.unlock();
        if (sleep_poll) std::this_thread::sleep_for(std::chrono::microseconds(20));
        else std::this_thread::yield();
      } else if (pending.empty()) {
        cv_sched.wait(lk, [&] { return stop || clear_requested || !pending.empty(); });
      } else {
        // the head request waits for pinned result memory: woken by a release
        cv_sched.wait_for(lk, std::chrono::microseconds(200));
      }
    }
  }
};

namespace {

int fail(int code, const std::string &msg) { return gpjb::report_error(code, msg.c_str()); }

void free_server(gpj_server *s) {
  for (auto &sl : s->slots) {
    if (sl.event) cudaEventDestroy(sl.event);
    if (sl.stream) cudaStreamDestroy(sl.stream);
  }
  if (s->d_arena) cudaFree(s->d_arena);
  if (s->h_arena) cudaFreeHost(s->h_arena);
  if (s->h_pinned) cudaFreeHost(s->h_pinned);
  if (s->d_status) cudaFree(s->d_status);
  delete s;
}

}  // namespace

extern "C" {

int gpj_server_create(const gpj_server_config *config, gpj_server **out) {
  if (out == nullptr) return fail(GPJ_ERR_INVALID_ARGUMENT, "gpj_server_create: null out");
  *out = nullptr;
  gpj_server_config cfg{};
  if (config != nullptr) cfg = *config;
  if (cfg.num_slots <= 0) cfg.num_slots = 32;
  if (cfg.num_slots > 1024) return fail(GPJ_ERR_INVALID_ARGUMENT, "num_slots must be <= 1024");
  if (cfg.hbm_budget_bytes == 0) cfg.hbm_budget_bytes = 1ull << 30;
  if (cfg.host_result_bytes == 0) cfg.host_result_bytes = 256ull << 20;
  if (cfg.cache_levels <= 0) cfg.cache_levels = 4;
  if (cfg.cache_levels > GPJ_MAX_LEVELS)
    return fail(GPJ_ERR_INVALID_ARGUMENT, "cache_levels must be <= 22");
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) {
    (void)cudaGetLastError();
    return fail(GPJ_ERR_CUDA, "gpj_server_create: no CUDA device");
  }
  if (cudaSetDevice(cfg.device) != cudaSuccess) {
    (void)cudaGetLastError();
    return fail(GPJ_ERR_CUDA, "gpj_server_create: cudaSetDevice failed");
  }
  auto *s = new (std::nothrow) gpj_server;
  if (s == nullptr) return fail(GPJ_ERR_OOM, "gpj_server_create: out of host memory");
  s->cfg = cfg;
  s->cache_on = (cfg.flags & GPJ_SERVER_NO_CACHE) == 0;
  s->sleep_poll = (cfg.flags & GPJ_SERVER_SLEEP_POLL) != 0;
  s->group_builds = (cfg.flags & GPJ_SERVER_NO_GROUPS) == 0;
  std::string err;
  int code = GPJ_OK;
  cudaError_t e = cudaMalloc(&s->d_arena, cfg.hbm_budget_bytes);
  if (e != cudaSuccess) {
    code = e == cudaErrorMemoryAllocation ? GPJ_ERR_OOM : GPJ_ERR_CUDA;
    err = std::string("device arena: ") + cudaGetErrorString(e);
  }
  if (code == GPJ_OK) {
    e = cudaHostAlloc(reinterpret_cast<void **>(&s->h_arena), cfg.host_result_bytes,
                      cudaHostAllocDefault);
    if (e != cudaSuccess) {
      code = GPJ_ERR_OOM;
      err = std::string("pinned result arena: ") + cudaGetErrorString(e);
    }
  }
  if (code == GPJ_OK) {
    e = cudaHostAlloc(reinterpret_cast<void **>(&s->h_pinned), uint64_t(cfg.num_slots) * 64u,
                      cudaHostAllocDefault);
    if (e != cudaSuccess) {
      code = GPJ_ERR_OOM;
      err = std::string("pinned slot words: ") + cudaGetErrorString(e);
    }
  }
  if (code == GPJ_OK) {
    e = cudaMalloc(reinterpret_cast<void **>(&s->d_status), uint64_t(cfg.num_slots) * 4u);
    if (e == cudaSuccess) e = cudaMemset(s->d_status, 0, uint64_t(cfg.num_slots) * 4u);
    if (e != cudaSuccess) {
      code = GPJ_ERR_CUDA;
      err = std::string("query status words: ") + cudaGetErrorString(e);
    }
  }
  if (code == GPJ_OK) {
    s->slots.resize(size_t(cfg.num_slots));
    for (int i = 0; i < cfg.num_slots && code == GPJ_OK; ++i) {
      Slot &sl = s->slots[size_t(i)];
      sl.pinned = s->h_pinned + size_t(i) * 8u;
      if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&sl.event, cudaEventDisableTiming) != cudaSuccess) {
        code = GPJ_ERR_CUDA;
        err = "stream/event creation failed";
      }
      s->free_slots.push_back(cfg.num_slots - 1 - i);
    }
  }
  if (code != GPJ_OK) {
    (void)cudaGetLastError();
    free_server(s);
    cudaSetDevice(prev);
    return fail(code, "gpj_server_create: " + err);
  }
  s->dev.reset(cfg.hbm_budget_bytes);
  s->host.reset(cfg.host_result_bytes);
  // grouped builds read every file inside the arena through one TMA view
  s->arena_tma = gpjb::index_make_tensor_map(&s->arena_map, s->d_arena, s->dev.size(),
                                             gpjb::kIndexThreads);
  s->stats.arena_bytes = s->dev.size();
  s->thread = std::thread([s] { s->loop(); });
  cudaSetDevice(prev);
  *out = s;
  return GPJ_OK;
}

namespace {
// Checks one request and copies it (and its IRs) into a new Request.
int make_request(const gpj_request *req, std::unique_ptr<Request> *out) {
  if (req->num_queries == 0 || req->num_queries > GPJ_SERVER_MAX_QUERIES || req->queries == nullptr)
    return fail(GPJ_ERR_INVALID_ARGUMENT, "gpj_server_submit: 1 to 8 queries per request");
  if (req->size_bytes > 0x7FFFFFFFull)
    return fail(GPJ_ERR_EXECUTION, "partition size exceeds CUDA int range");
  if (req->size_bytes > 0 && req->h_input == nullptr)
    return fail(GPJ_ERR_INVALID_ARGUMENT, "gpj_server_submit: null input");
  auto r = std::make_unique<Request>();
  r->key = req->file_key;
  r->h_input = req->h_input;
  r->n = req->size_bytes;
  r->levels_needed = 1;
  for (uint32_t q = 0; q < req->num_queries; ++q) {
    const gpj_batch_query &bq = req->queries[q];
    if (bq.h_ir == nullptr || bq.ir_len == 0)
      return fail(GPJ_ERR_INVALID_ARGUMENT, "gpj_server_submit: empty query IR");
    if (bq.ir_len > uint64_t(GPJ_MAX_QUERY_IR))
      return fail(GPJ_ERR_EXECUTION, "Compiled query IR exceeds constant memory buffer");
    if (bq.num_levels > uint32_t(GPJ_MAX_LEVELS))
      return fail(GPJ_ERR_INVALID_ARGUMENT, "num_levels must be in [0, 22]");
    if (bq.base_level > 0 && bq.base_level >= bq.num_levels)
      return fail(GPJ_ERR_EXECUTION, "Query requires more bitmap levels than the index provides");
    r->queries.push_back(bq);
    r->irs.emplace_back(bq.h_ir, bq.h_ir + bq.ir_len);
    r->queries.back().h_ir = nullptr;
    r->levels_needed = std::max(r->levels_needed, int(bq.num_levels));
    r->slots_total += bq.num_result_slots;
  }
  r->resp.arrival_ns = req->arrival_ns ? req->arrival_ns : now_ns();
  *out = std::move(r);
  return GPJ_OK;
}
}  // namespace

int gpj_server_submit_many(gpj_server *s, const gpj_request *reqs, uint32_t count,
                           uint64_t *request_ids) {
  if (s == nullptr || (count > 0 && (reqs == nullptr || request_ids == nullptr)))
    return fail(GPJ_ERR_INVALID_ARGUMENT, "gpj_server_submit_many: null argument");
  std::vector<std::unique_ptr<Request>> made(count);
  for (uint32_t i = 0; i < count; ++i) {
    const int rc = make_request(&reqs[i], &made[i]);
    if (rc != GPJ_OK) return rc;  // nothing was queued
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return fail(GPJ_ERR_EXECUTION, "gpj_server_submit: server is shutting down");
  for (uint32_t i = 0; i < count; ++i) {
    Request *r = made[i].get();
    r->id = s->next_id++;
    request_ids[i] = r->id;
    s->pending.push_back(r);
    s->requests.emplace(r->id, std::move(made[i]));
  }
  s->stats.submitted += count;
  s->cv_sched.notify_one();
  return GPJ_OK;
}

int gpj_server_submit(gpj_server *s, const gpj_request *req, uint64_t *request_id) {
  if (s == nullptr || req == nullptr || request_id == nullptr)
    return fail(GPJ_ERR_INVALID_ARGUMENT, "gpj_server_submit: null argument");
  return gpj_server_submit_many(s, req, 1, request_id);
}

int gpj_server_poll(gpj_server *s, uint64_t *ids, uint32_t capacity, uint32_t *count,
                    int64_t timeout_us) {
  if (s == nullptr || count == nullptr || (capacity > 0 && ids == nullptr))
    return fail(GPJ_ERR_INVALID_ARGUMENT, "gpj_server_poll: null argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto ready = [&] { return !s->done_unreported.empty(); };
  if (timeout_us < 0) s->cv_done.wait(lk, ready);
  else if (timeout_us > 0) s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), ready);
  uint32_t k = 0;
  while (k < capacity && !s->done_unreported.empty()) {
    ids[k++] = s->done_unreported.front();
    s->done_unreported.pop_front();
  }
  *count = k;
  return GPJ_OK;
}

int gpj_server_wait(gpj_server *s, uint64_t id, int64_t timeout_us) {
  if (s == nullptr) return fail(GPJ_ERR_INVALID_ARGUMENT, "gpj_server_wait: null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->requests.find(id);
  if (it == s->requests.end()) return fail(GPJ_ERR_OUT_OF_RANGE, "unknown request id");
  Request *r = it->second.get();
  auto done = [&] { return r->done; };
  if (timeout_us < 0) s->cv_done.wait(lk, done);
  else s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), done);
  if (!done()) return fail(GPJ_ERR_TIMEOUT, "request still running");
  return GPJ_OK;
}

int gpj_server_response(gpj_server *s, uint64_t id, gpj_response *out) {
  if (s == nullptr || out == nullptr)
    return fail(GPJ_ERR_INVALID_ARGUMENT, "gpj_server_response: null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->requests.find(id);
  if (it == s->requests.end()) return fail(GPJ_ERR_OUT_OF_RANGE, "unknown request id");
  if (!it->second->done) return fail(GPJ_ERR_TIMEOUT, "request still running");
  *out = it->second->resp;
  return GPJ_OK;
}

int gpj_server_release(gpj_server *s, uint64_t id) {
  if (s == nullptr) return fail(GPJ_ERR_INVALID_ARGUMENT, "gpj_server_release: null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->requests.find(id);
  if (it == s->requests.end()) return fail(GPJ_ERR_OUT_OF_RANGE, "unknown request id");
  Request *r = it->second.get();
  if (!r->done) return fail(GPJ_ERR_TIMEOUT, "request still running");
  if (r->has_host) s->host.release(r->host_off, r->host_bytes);
  r->has_host = false;
  s->graveyard.push_back(std::move(it->second));
  s->requests.erase(it);
  s->cv_sched.notify_one();
  return GPJ_OK;
}

int gpj_server_stats_get(gpj_server *s, gpj_server_stats *out) {
  if (s == nullptr || out == nullptr)
    return fail(GPJ_ERR_INVALID_ARGUMENT, "gpj_server_stats_get: null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  out->arena_bytes = s->dev.size();
  return GPJ_OK;
}

int gpj_server_clear_cache(gpj_server *s) {
  if (s == nullptr) return fail(GPJ_ERR_INVALID_ARGUMENT, "gpj_server_clear_cache: null server");
  // the scheduler owns the device arena: ask it and wait
  std::unique_lock<std::mutex> lk(s->mu);
  s->clear_requested = true;
  s->cv_sched.notify_one();
  s->cv_done.wait(lk, [&] { return !s->clear_requested; });
  return GPJ_OK;
}

int gpj_server_destroy(gpj_server *s) {
  if (s == nullptr) return GPJ_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (Request *r : s->pending) {
      r->resp.status = GPJ_ERR_EXECUTION;
      std::snprintf(r->resp.message, sizeof(r->resp.message), "server destroyed");
      r->state = St::Done;
      r->done = true;
    }
    s->pending.clear();
    s->stop = true;
    s->cv_sched.notify_one();
  }
  if (s->thread.joinable()) s->thread.join();
  cudaSetDevice(s->cfg.device);
  free_server(s);
  return GPJ_OK;
}

}  // extern "C"
