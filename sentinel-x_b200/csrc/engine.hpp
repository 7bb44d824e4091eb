// Internal declarations shared by the engine's host translation units:
// device buffers, streams and slots, the engine / profile-set / target-set
// objects behind the C ABI handles, and the functions one file defines for
// another (packing: pack.cu; the search scheduler: scheduler.cu; device
// domain-definition passes: domain_passes.cu; C ABI: engine.cu, score.cu,
// static_entry.cu).
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/sxhmm.h"
#include "internal.hpp"
#include "shapes.hpp"

using namespace sx;
using sxk::BinRegion;
using sxk::DevProfile;
using sxk::MsvTile;
using sxk::PairRec;
using sxk::Thresholds;

// defined with their kernels in long.cuh / plain.cuh
namespace sxk {
struct LongPair;
struct PlainProfile;
}  // namespace sxk

namespace sxe {

// last error message of the calling thread (sx_last_error)
extern thread_local std::string g_err;

// Names the kernels of one entry-point call for profilers (a no-op unless a
// tool is attached), e.g. ncu --nvtx --nvtx-include "sx_search/".
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

// Wall-clock phases of one sx_search, printed to stderr when the environment
// variable SXHMM_PROFILE is set (a diagnostic for tuning placements; it adds
// clock reads only).
struct PhaseLog {
  bool on = std::getenv("SXHMM_PROFILE") != nullptr;
  std::mutex mu;  // entries may come from the host pool's thread
  std::vector<std::pair<std::string, double>> v;
  void add(const std::string& name, std::chrono::steady_clock::time_point t0) {
    if (!on) return;
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::lock_guard<std::mutex> g(mu);
    v.emplace_back(name, ms);
  }
  void print() {
    if (!on) return;
    std::lock_guard<std::mutex> g(mu);
    std::string o = "[sxhmm profile]";
    char buf[96];
    for (const auto& p : v) {
      snprintf(buf, sizeof buf, " %s=%.1fms", p.first.c_str(), p.second);
      o += buf;
    }
    fprintf(stderr, "%s\n", o.c_str());
  }
};
// Records msg as the calling thread's last error and returns code.
int fail(int code, const std::string& msg);


struct CudaError {
  int code;
  std::string msg;
};

#define CK(call)                                                                                      \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess)                                                                            \
      throw CudaError{e_ == cudaErrorMemoryAllocation ? SX_ENOMEM : SX_ECUDA,                         \
                      std::string(#call) + ": " + cudaGetErrorString(e_)};                            \
  } while (0)

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  bool owned = true;  // false: a view into memory someone else frees
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p && owned) cudaFree(p);
    p = nullptr;
    n = 0;
    owned = true;
  }
  void view(void* at, size_t count) {
    release();
    p = static_cast<T*>(at);
    n = count;
    owned = false;
  }
  // Grow-only, contents undefined.  A buffer that must grow takes a quarter
  // more than asked: the scratch of a stream of searches (survivor lists,
  // envelope planes) varies from call to call, and each regrowth is a
  // cudaFree -- which waits for the whole device -- and a fresh cudaMalloc.
  void alloc(size_t count) {
    if (count <= n && p) return;
    release();
    const size_t want = std::max<size_t>(count, 1);
    const size_t ask = want + want / 4;
    if (cudaMalloc(&p, ask * sizeof(T)) == cudaSuccess) {
      n = ask;
      return;
    }
    cudaGetLastError();
    p = nullptr;
    CK(cudaMalloc(&p, want * sizeof(T)));
    n = want;
  }
  void upload(const T* src, size_t count, cudaStream_t s) {
    alloc(count);
    if (count) CK(cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
};

// Page-locked host buffer (grow-only): device-to-host copies into it run at
// full link speed and never fault in fresh pages.
template <typename T>
struct PinnedBuf {
  T* p = nullptr;
  size_t n = 0;
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
  ~PinnedBuf() { release(); }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count <= n && p) return;
    release();
    CK(cudaHostAlloc((void**)&p, std::max<size_t>(count, 1) * sizeof(T), cudaHostAllocDefault));
    n = std::max<size_t>(count, 1);
  }
};

// Launch tables of every kernel instantiation (filled once).
const KernelTables& kernels();

// ---- thread pool helper ----------------------------------------------------
template <typename F>
void parallel_for(size_t n, int nthreads, F&& f) {
  if (n == 0) return;
  const int nt = std::max(1, std::min<int>(nthreads, (int)n));
  std::atomic<size_t> next{0};
  auto work = [&]() {
    for (;;) {
      const size_t i = next.fetch_add(1);
      if (i >= n) break;
      f(i);
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nt; t++) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
}

// Smallest f32 statistic s with pass(s) true, assuming pass is monotone
// (false below the boundary, true above); +inf if it never passes, -inf if it
// always passes on the finite range.
template <typename Pred>
float f32_boundary(Pred pass) {
  auto key = [](float f) {
    int32_t i;
    memcpy(&i, &f, 4);
    return i >= 0 ? i : (int32_t)(0x80000000u - (uint32_t)i) * -1;  // monotone int order
  };
  (void)key;
  // order-preserving map float <-> int64 over finite floats
  auto to_ord = [](float f) -> int64_t {
    uint32_t u;
    memcpy(&u, &f, 4);
    return (u & 0x80000000u) ? -(int64_t)(u & 0x7fffffffu) : (int64_t)u;
  };
  auto from_ord = [](int64_t o) -> float {
    uint32_t u = o < 0 ? (0x80000000u | (uint32_t)(-o)) : (uint32_t)o;
    float f;
    memcpy(&f, &u, 4);
    return f;
  };
  int64_t lo = to_ord(-3.0e38f), hi = to_ord(3.0e38f);
  if (pass(from_ord(lo))) return -INFINITY;
  if (!pass(from_ord(hi))) return INFINITY;
  while (hi - lo > 1) {  // invariant: !pass(lo), pass(hi)
    const int64_t mid = lo + (hi - lo) / 2;
    if (pass(from_ord(mid))) hi = mid;
    else lo = mid;
  }
  return from_ord(hi);
}

// Device blocks recycled between target sets, so that a caller streaming
// batches of targets through one engine does not pay a cudaMalloc/cudaFree
// pair (and the device-wide synchronisation of cudaFree) per batch.
// Host buffers of packed residues, recycled across target sets so that a
// caller streaming batches of targets writes into pages already touched.
// Page-locked host memory for the packed residues of target sets, so their
// copy to the device runs at the bus's rate rather than through the driver's
// pageable staging; plain heap memory when the pinned allocation fails.
// Growing a vector leaves the new elements uninitialised (the packers write
// every byte).
template <typename T>
struct PinnedAlloc {
  using value_type = T;
  PinnedAlloc() = default;
  template <typename U>
  PinnedAlloc(const PinnedAlloc<U>&) {}
  // Each block starts with a 64-byte header recording how it was obtained,
  // so it is freed the same way even after the CUDA context is gone.
  static constexpr size_t kHead = 64;
  T* allocate(size_t n) {
    const size_t bytes = std::max<size_t>(n, 1) * sizeof(T) + kHead;
    void* p = nullptr;
    uint32_t pinned = 1;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      pinned = 0;
      p = std::malloc(bytes);
      if (!p) throw std::bad_alloc();
    }
    std::memcpy(p, &pinned, sizeof pinned);
    return reinterpret_cast<T*>(static_cast<char*>(p) + kHead);
  }
  void deallocate(T* q, size_t) {
    void* p = reinterpret_cast<char*>(q) - kHead;
    uint32_t pinned = 0;
    std::memcpy(&pinned, p, sizeof pinned);
    if (pinned) {
      if (cudaFreeHost(p) != cudaSuccess) cudaGetLastError();
    } else {
      std::free(p);
    }
  }
  template <typename U>
  void construct(U* p) noexcept {}  // default-initialise: no fill
  template <typename U, typename... A>
  void construct(U* p, A&&... a) {
    ::new ((void*)p) U(std::forward<A>(a)...);
  }
  template <typename U>
  bool operator==(const PinnedAlloc<U>&) const { return true; }
  template <typename U>
  bool operator!=(const PinnedAlloc<U>&) const { return false; }
};
using HostBytes = std::vector<uint8_t, PinnedAlloc<uint8_t>>;

class HostBytePool {
 public:
  HostBytes take(size_t bytes) {
    std::lock_guard<std::mutex> g(mu_);
    for (size_t i = 0; i < free_.size(); i++)
      if (free_[i].capacity() >= bytes) {
        HostBytes v = std::move(free_[i]);
        free_.erase(free_.begin() + (std::ptrdiff_t)i);
        v.clear();
        return v;
      }
    HostBytes v;
    v.reserve(bytes);
    return v;
  }
  void give(HostBytes&& v) {
    if (!v.capacity()) return;
    std::lock_guard<std::mutex> g(mu_);
    free_.push_back(std::move(v));
    if (free_.size() > 2)  // keep the two largest
      free_.erase(std::min_element(free_.begin(), free_.end(),
                                   [](const auto& x, const auto& y) { return x.capacity() < y.capacity(); }));
  }

 private:
  std::mutex mu_;
  std::vector<HostBytes> free_;
};

class BlockPool {
 public:
  ~BlockPool() {
    for (auto& b : free_) cudaFree(b.first);
  }
  // A block of at least `bytes`; its size is returned in `got`.
  void* take(size_t bytes, size_t& got) {
    {
      std::lock_guard<std::mutex> g(mu_);
      size_t best = free_.size();
      for (size_t i = 0; i < free_.size(); i++)
        if (free_[i].second >= bytes && (best == free_.size() || free_[i].second < free_[best].second)) best = i;
      if (best < free_.size()) {
        auto b = free_[best];
        free_.erase(free_.begin() + (std::ptrdiff_t)best);
        got = b.second;
        return b.first;
      }
    }
    void* p = nullptr;
    CK(cudaMalloc(&p, std::max<size_t>(bytes, 256)));
    got = std::max<size_t>(bytes, 256);
    return p;
  }
  void give(void* p, size_t bytes) {
    std::lock_guard<std::mutex> g(mu_);
    free_.emplace_back(p, bytes);
    if (free_.size() > kKeep) {  // drop the smallest
      auto it = std::min_element(free_.begin(), free_.end(),
                                 [](const auto& a, const auto& b) { return a.second < b.second; });
      cudaFree(it->first);
      free_.erase(it);
    }
  }

 private:
  static constexpr size_t kKeep = 2;
  std::mutex mu_;
  std::vector<std::pair<void*, size_t>> free_;
};

// A main stream with auxiliary streams that fan out from it and join back
// into it, all of one scheduling priority.
struct Streams {
  static constexpr int kAux = 8;
  int naux = kAux;  // auxiliary streams in use
  cudaStream_t main = nullptr;
  cudaStream_t aux[kAux] = {};  // independent launches (shapes, bins) run side by side
  cudaEvent_t fork_ev = nullptr, join_ev[kAux] = {};
  void create(int priority, int n_aux) {
    naux = std::max(1, std::min(n_aux, kAux));
    CK(cudaStreamCreateWithPriority(&main, cudaStreamNonBlocking, priority));
    for (int a = 0; a < naux; a++) {
      CK(cudaStreamCreateWithPriority(&aux[a], cudaStreamNonBlocking, priority));
      CK(cudaEventCreateWithFlags(&join_ev[a], cudaEventDisableTiming));
    }
    CK(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
  }
  void destroy() {
    if (main) cudaStreamSynchronize(main);
    for (int a = 0; a < naux; a++)
      if (aux[a]) cudaStreamSynchronize(aux[a]);
    for (int a = 0; a < naux; a++) {
      if (aux[a]) cudaStreamDestroy(aux[a]);
      if (join_ev[a]) cudaEventDestroy(join_ev[a]);
    }
    if (fork_ev) cudaEventDestroy(fork_ev);
    if (main) cudaStreamDestroy(main);
  }
};

// Set once a host job has copied a slot's row buffers out; the engine thread
// waits for it before it reuses those buffers for a later block.
struct RowsTicket {
  std::mutex mu;
  std::condition_variable cv;
  bool done = false;
  void set() {
    {
      std::lock_guard<std::mutex> g(mu);
      done = true;
    }
    cv.notify_all();
  }
  void wait() {
    std::unique_lock<std::mutex> g(mu);
    cv.wait(g, [&] { return done; });
  }
};

// Streams, events and survivor lists of one block of a search.  A search
// keeps two blocks in flight: block b+1's MSV runs on one slot while block
// b's later stages, row passes and host re-check use the other.  MSV goes to
// the low-priority streams, everything after it to the high-priority ones,
// so the short, latency-bound later stages of block b get SMs as soon as
// block b+1's MSV CTAs retire and MSV fills the rest of the GPU.
struct Slot {
  Streams hi, lo;
  cudaEvent_t ev[8] = {};
  cudaEvent_t msv_done = nullptr;
  // grow-only device scratch
  DevBuf<PairRec> lists[4];
  DevBuf<BinRegion> bins[4];
  DevBuf<unsigned> counts;  // 4 stages x kMaxBins
  DevBuf<unsigned> overflow;
  DevBuf<unsigned> cursor;  // kMaxBins pair cursors of the Viterbi launches
  DevBuf<double> cells;     // DP cells entering each stage (stats)
  DevBuf<MsvTile> tiles;
  DevBuf<sxk::PackedTile> ptiles;  // packed pre-screen tiles
  DevBuf<int32_t> rlist;           // pre-screen survivors: target indices, rcap per profile of the block
  DevBuf<unsigned> rcount;         // survivors per profile of the block
  cudaEvent_t pre_done = nullptr;  // pre-screen finished (its time, for the stats)
  // packed Viterbi pre-screen: the bias filter's survivors of pre-screened
  // profiles, vcap per profile of the block, and the pre-screen's tiles
  DevBuf<PairRec> vlist;
  DevBuf<unsigned> vcount;
  DevBuf<sxk::VitTile> vtiles;
  DevBuf<double> vstats;           // cells bounded, cells passed, pairs passed
  cudaEvent_t bias_done = nullptr, vpre_done = nullptr;
  // Forward/Backward row passes of the block's final pairs, in buffers of
  // their own: the engine thread queues them and moves on to the next block;
  // a host job waits for them, copies the rows out and releases the buffers.
  DevBuf<PairRec> rrecs;
  DevBuf<BinRegion> rbins;
  DevBuf<unsigned> rcnt;
  DevBuf<int64_t> roff;
  DevBuf<float> rows_f, rows_b;
  cudaEvent_t rows_t0 = nullptr, rows_t1 = nullptr;
  cudaStream_t rows_copy = nullptr;  // device-to-host copies of the rows (host job)
  std::shared_ptr<RowsTicket> rows_busy;
  void create() {
    int least = 0, greatest = 0;
    CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    // 2 slots x (9 + 6) streams + 1 envelope stream = 31, within the 32
    // hardware work queues a process can have (CUDA_DEVICE_MAX_CONNECTIONS=32):
    // with fewer queues, streams share them and a high-priority launch can
    // wait behind queued MSV work
    hi.create(greatest, 8);
    lo.create(least, 5);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    CK(cudaEventCreate(&pre_done));
    CK(cudaEventCreate(&bias_done));
    CK(cudaEventCreate(&vpre_done));
    CK(cudaEventCreate(&rows_t0));
    CK(cudaEventCreate(&rows_t1));
    CK(cudaStreamCreateWithFlags(&rows_copy, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&msv_done, cudaEventDisableTiming));
  }
  void destroy() {
    hi.destroy();
    lo.destroy();
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (msv_done) cudaEventDestroy(msv_done);
    if (pre_done) cudaEventDestroy(pre_done);
    if (bias_done) cudaEventDestroy(bias_done);
    if (vpre_done) cudaEventDestroy(vpre_done);
    if (rows_busy) rows_busy->wait();
    if (rows_t0) cudaEventDestroy(rows_t0);
    if (rows_t1) cudaEventDestroy(rows_t1);
    if (rows_copy) {
      cudaStreamSynchronize(rows_copy);
      cudaStreamDestroy(rows_copy);
    }
  }
};

}  // namespace sxe

using namespace sxe;

// ---- engine objects ----------------------------------------------------------
struct sx_engine {
  int device = 0;
  int host_threads = 1;
  uint32_t flags = 0;
  int64_t batch_bytes = 0;
  int num_sms = 148;
  static constexpr int kAux = Streams::kAux;
  Slot sl[2];
  // slot 0 under the names the single-batch entry points use
  cudaStream_t& stream = sl[0].hi.main;
  cudaStream_t (&aux)[kAux] = sl[0].hi.aux;
  cudaEvent_t& fork_ev = sl[0].hi.fork_ev;
  cudaEvent_t (&join_ev)[kAux] = sl[0].hi.join_ev;
  cudaEvent_t (&ev)[8] = sl[0].ev;
  DevBuf<PairRec> (&lists)[4] = sl[0].lists;
  DevBuf<BinRegion> (&bins)[4] = sl[0].bins;
  DevBuf<unsigned>& counts = sl[0].counts;
  DevBuf<unsigned>& overflow = sl[0].overflow;
  DevBuf<MsvTile>& tiles = sl[0].tiles;
  std::mutex mu;
  sx_search_stats stats{};
  int pipeline_blocks = 0;  // profile blocks per search; 0 = by workload size
  // kernel shape per profile length, set by a tuner (sx_set_shape_table):
  // [0] MSV, [1] Viterbi; empty or -1 = the built-in choice
  std::vector<int16_t> shape_table[2];
  int64_t mem_free = 0;     // device memory free when the engine was created
  // Lifetime: profile and target sets point at their engine.  sx_destroy
  // releases the engine's streams at once, but the engine object itself lives
  // until the last of its sets is freed, so a set freed after its engine (a
  // garbage-collected binding, say) never touches freed memory.
  std::mutex life_mu;
  int64_t live_sets = 0;
  bool destroyed = false;
  BlockPool target_blocks;  // device memory of freed target sets
  HostBytePool target_bytes;  // host residue buffers of freed target sets
  // envelope passes of the host domain definition (used by the host pool's
  // driver thread, one batch at a time)
  cudaStream_t env_stream = nullptr;  // the passes' copies; their launches fan out over the slots' streams
  cudaEvent_t env_ev = nullptr;
  DevBuf<sxk::EnvRec> env_recs;
  DevBuf<float> env_planes, env_rows, env_aux, env_out;
  DevBuf<double> env_fac;
  DevBuf<sxk::TraceRec> trc_recs;  // stochastic-trace passes of multi-domain regions
  DevBuf<int32_t> trc_pool, trc_count, trc_status;
  DevBuf<float> trc_cols;
  DevBuf<sxk::LongPair> long_pairs;  // pairs of profiles longer than kMaxM
  DevBuf<float> long_scratch, long_out, long_rows_f, long_rows_b;
  DevBuf<int64_t> long_row_off;
  DevBuf<Thresholds> thr;
  DevBuf<float> rows_f, rows_b;
  DevBuf<int64_t> row_off;
  DevBuf<float> scores;
  DevBuf<int32_t> slots, plist;
  DevBuf<sxk::AdjPair> adj_pairs;
  DevBuf<float> adj_f, adj_out;
  PinnedBuf<float> adj_host;  // staging of the adjoint's counts on their way to the caller
  DevBuf<double> adj_d, adj_lnz;
};

struct sx_profiles {
  sx_engine* eng = nullptr;
  std::vector<ProfileHost> h;
  std::vector<DevProfile> dp;
  std::vector<int> msv_shape;
  DevBuf<DevProfile> d_prof;
  DevBuf<sxk::PlainProfile> d_pprof;  // plain one-pair-per-block layout
  DevBuf<float> d_plain;
  DevBuf<float4> d_msv;
  DevBuf<uint2> d_qimg;  // quantized MSV images of the pre-screen (int16, 4 columns per uint2)
  DevBuf<float4> d_vit;  // Viterbi lane-group images
  DevBuf<uint4> d_qvimg;  // quantized Viterbi images of the packed pre-screen
  DevBuf<float> d_vfb;
  DevBuf<double> d_bias;
  // the filter thresholds of the last search options seen (they depend on the
  // profiles' statistics and F1/F2/F3 alone): a stream of searches with one
  // configuration computes them once
  mutable std::mutex th_mu;
  mutable std::vector<Thresholds> th_cache;
  mutable double th_key[4] = {-1, -1, -1, -1};
};

struct sx_targets {
  sx_engine* eng = nullptr;
  std::vector<std::string> ids;  // caller's names (sx_targets_create); empty for digital sets
  HostBytes dsq;  // packed digital residues, each target 16-byte aligned (page-locked)
  std::vector<int64_t> off;
  std::vector<int32_t> len;
  std::vector<int32_t> order;  // indices sorted by length, longest first
  double residues = 0;
  DevBuf<uint8_t> d_res;
  DevBuf<int64_t> d_off;
  DevBuf<int32_t> d_len;
  DevBuf<float4> d_tpar;  // MSV tloop, tmove, null score
  DevBuf<float4> d_xsc;   // multihit loop, move (log), loop, move (prob)
  DevBuf<int32_t> d_order;
  void* block = nullptr;  // one device block holding all d_* arrays (engine pool)
  size_t block_bytes = 0;
  ~sx_targets() {
    if (block) eng->target_blocks.give(block, block_bytes);
    eng->target_bytes.give(std::move(dsq));
  }
};

struct sx_hits {
  std::vector<sx_hit> hits;
  std::vector<sx_domain> doms;
};

namespace sxe {

constexpr float kSlackBits = 1.0e-3f;  // device-log decisions: never reject what the reference keeps

struct FinalPair {
  int32_t p, t;
  float usc, filtersc, vsc;
  int32_t slot;
};

// Host copies of one chunk of raw Forward/Backward special rows.
struct RowsChunk {
  std::vector<float> f, b;    // rows of every pair of the chunk, back to back
  std::vector<int64_t> off;   // offset of pair q's rows in f and b
  std::vector<size_t> which;  // pair q's index in the caller's list
};

// One batch's requests and the places for their results.
struct EnvSource {
  const DomainBatch* db;
  const std::vector<EnvRequest>* reqs;
  std::vector<EnvFactors>* F;
  std::vector<EnvDeviceOut>* D;
};

struct RegionSource {
  DomainBatch* db;
  const std::vector<RegionRequest>* regs;
};
struct RegionPassStats {
  int64_t launches = 0, device = 0, redone = 0;
  double cells = 0;
};

int vit_blocks(int num_sms, int shape, unsigned n);
int warp_ctas(int num_sms, unsigned n);
std::vector<int16_t> default_shape_table(int kind);
int shape_for(const sx_engine* E, int kind, int m);
void pack_profiles(sx_profiles* P);
void pack_targets(sx_targets* T);
void append_target(sx_targets* T, const uint8_t* dig, size_t l);
std::vector<Thresholds> make_thresholds(const std::vector<ProfileHost>& H, const SearchOpts& o);
void fork_aux(Streams& X);
void join_aux(Streams& X);
void note_free_memory(sx_engine* E);
int64_t scratch_budget(const sx_engine* E, int64_t want);
int report(const sx_profiles* P, const sx_targets* T, const sx_search_cfg* cfg,
           std::vector<std::vector<std::pair<int32_t, HitOut>>>& per_profile, sx_hits* out);
int check_cutoffs(const sx_profiles* P, int kind);
size_t msv_smem(int s);
void launch_msv(sx_engine* E, Slot& S, Streams& X, const sx_profiles* P, const sx_targets* T, const std::vector<std::vector<MsvTile>>& tiles,
                const int32_t* d_list, float* d_scores, const int32_t* d_slot, PairRec* surv, const BinRegion* bins,
                unsigned* counts, const unsigned* rcount = nullptr, unsigned rcap = 0, int p0 = 0);
double elapsed_ms(cudaEvent_t a, cudaEvent_t b);
int long_grid(const sx_engine* E, size_t n);
int64_t long_stride(const sx_profiles* P, const std::vector<sxk::LongPair>& v, size_t a, size_t b);
void long_scores(sx_engine* E, const sx_profiles* P, const sx_targets* T, const std::vector<sxk::LongPair>& v,
                 bool viterbi, std::vector<float>& out);
int run_search(sx_engine* E, const sx_profiles* P, const sx_targets* T, const sx_search_cfg* cfg, sx_hits* out);
int64_t envelope_passes(sx_engine* E, const sx_profiles* P, const sx_targets* T, std::vector<EnvSource>& srcs,
                        int nthr, PhaseLog* plog = nullptr);
RegionPassStats region_passes(sx_engine* E, const sx_profiles* P, const sx_targets* T,
                              std::vector<RegionSource>& srcs, int nthr);

// Device Forward and Backward with row output for `pairs`, in chunks bounded
// by `row_budget` floats per direction; hands each chunk's host copy to
// consume(RowsChunk&&) as soon as it has arrived.
template <typename Consume>
void rows_pass(sx_engine* E, Slot& S, const sx_profiles* P, const sx_targets* T, const std::vector<FinalPair>& pairs,
               Consume&& consume) {
  if (pairs.empty()) return;
  const auto& K = kernels();
  const int64_t row_budget = std::max<int64_t>(scratch_budget(E, E->batch_bytes / 2) / (int64_t)sizeof(float), 1 << 20);
  size_t i0 = 0;
  while (i0 < pairs.size()) {
    // chunk [i0, i1)
    size_t i1 = i0;
    int64_t used = 0;
    while (i1 < pairs.size()) {
      const int64_t need = 6 * ((int64_t)T->len[pairs[i1].t] + 1);
      if (i1 > i0 && used + need > row_budget) break;
      used += need;
      i1++;
    }
    // group by vbin, assign row offsets
    std::vector<std::vector<size_t>> byb(kNumVbins);
    for (size_t i = i0; i < i1; i++) byb[P->dp[pairs[i].p].vbin].push_back(i);
    std::vector<PairRec> recs;
    RowsChunk c;
    std::vector<BinRegion> reg(kNumVbins);
    std::vector<unsigned> cnt(kNumVbins, 0);
    int64_t ro = 0;
    for (int b = 0; b < kNumVbins; b++) {
      reg[b].off = (int64_t)recs.size();
      reg[b].cap = (uint32_t)byb[b].size();
      reg[b].pad = 0;
      cnt[b] = (unsigned)byb[b].size();
      for (size_t i : byb[b]) {
        const FinalPair& f = pairs[i];
        PairRec r{f.p, f.t, f.usc, f.filtersc, f.vsc, 0.f, f.slot, 0};
        recs.push_back(r);
        c.off.push_back(ro);
        c.which.push_back(i);
        ro += 6 * ((int64_t)T->len[f.t] + 1);
      }
    }
    cudaStream_t s = S.hi.main;
    S.lists[3].upload(recs.data(), recs.size(), s);
    E->row_off.upload(c.off.data(), c.off.size(), s);
    S.bins[3].upload(reg.data(), reg.size(), s);
    S.counts.alloc(4 * kMaxBins);
    CK(cudaMemcpyAsync(S.counts.p + 3 * kMaxBins, cnt.data(), sizeof(unsigned) * kNumVbins, cudaMemcpyHostToDevice, s));
    E->rows_f.alloc((size_t)ro);
    E->rows_b.alloc((size_t)ro);
    // rows the kernels never touch are zero
    CK(cudaMemsetAsync(E->rows_f.p, 0, sizeof(float) * (size_t)ro, s));
    CK(cudaMemsetAsync(E->rows_b.p, 0, sizeof(float) * (size_t)ro, s));
    fork_aux(S.hi);
    for (int b = 0; b < kNumVbins; b++) {
      if (!cnt[b]) continue;
      const int blocks = warp_ctas(E->num_sms, cnt[b]);
      cudaStream_t sa = S.hi.aux[(2 * b) % S.hi.naux], sb = S.hi.aux[(2 * b + 1) % S.hi.naux];
      K.fwd[b]<<<blocks, 32, 0, sa>>>(S.lists[3].p, S.counts.p + 3 * kMaxBins, S.bins[3].p, b, nullptr, nullptr,
                                       nullptr, S.overflow.p, P->d_prof.p, E->thr.p, P->d_vfb.p, T->d_res.p,
                                       T->d_off.p, T->d_len.p, T->d_xsc.p, 0.f, E->rows_f.p, E->row_off.p);
      K.bwd[b]<<<blocks, 32, 0, sb>>>(S.lists[3].p, S.counts.p + 3 * kMaxBins, S.bins[3].p, b, P->d_prof.p,
                                       P->d_vfb.p, T->d_res.p, T->d_off.p, T->d_len.p, T->d_xsc.p, E->rows_b.p,
                                       E->row_off.p);
      E->stats.kernel_launches += 2;
    }
    CK(cudaGetLastError());
    join_aux(S.hi);
    c.f.resize((size_t)ro);
    c.b.resize((size_t)ro);
    CK(cudaMemcpyAsync(c.f.data(), E->rows_f.p, sizeof(float) * (size_t)ro, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(c.b.data(), E->rows_b.p, sizeof(float) * (size_t)ro, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    consume(std::move(c));
    i0 = i1;
  }
}

// rows_pass with each chunk consumed on the calling thread: sink(i, fwd_rows,
// bwd_rows) for every pair, spread over the engine's host threads.
template <typename Sink>
void rows_pass_sync(sx_engine* E, const sx_profiles* P, const sx_targets* T, const std::vector<FinalPair>& pairs,
                    Sink&& sink) {
  rows_pass(E, E->sl[0], P, T, pairs, [&](RowsChunk&& c) {
    parallel_for(c.which.size(), E->host_threads,
                 [&](size_t q) { sink(c.which[q], c.f.data() + c.off[q], c.b.data() + c.off[q]); });
  });
}

// Raw Forward/Backward special rows of long-profile pairs, in chunks bounded
// by the scratch budget; consume(first, n, fwd, bwd, off) per chunk, pair
// first + q having its rows at fwd + off[q] and bwd + off[q].
using LongRowsSink = std::function<void(size_t, size_t, const float*, const float*, const std::vector<int64_t>&)>;
void long_rows(sx_engine* E, const sx_profiles* P, const sx_targets* T, const std::vector<sxk::LongPair>& v,
               const LongRowsSink& consume);

}  // namespace sxe
