// sxhmm engine: device data layout, the batched hmmsearch cascade on one
// B200, and the C ABI declared in include/sxhmm.h.
//
// Flow of sx_search (replaces the rayon pair loop of search_profiles,
// src/hmmer/search.rs:213-234, and score_target, src/hmmer/pipeline.rs:154):
//   1. MSV over every (profile, target) pair: CTA tiles of (profile, slice of
//      the length-sorted targets); exact F1 decision; survivors appended to
//      per-shape lists.
//   2. composition-bias filter, 3. Viterbi, 4. Forward score: each a
//      pair-list kernel over the previous stage's survivors; decisions that
//      involve a device logarithm are taken with a small slack so the device
//      never rejects a pair the reference keeps.
//   5. host: exact re-check of every decision with the reference's libm;
//      device Forward/Backward passes that emit the raw special rows of the
//      final pairs (chunked); host posterior domain definition, envelope
//      rescoring and reporting on a thread pool.
// Steps 1-5 run per block of profiles; a block's host domain definition is
// queued to a background pool and overlaps the device work of later blocks.
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
#include "long.cuh"
#include "tuned_shapes.inc"

using namespace sx;
using sxk::BinRegion;
using sxk::DevProfile;
using sxk::MsvTile;
using sxk::PairRec;
using sxk::Thresholds;

namespace {

thread_local std::string g_err;

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
  std::vector<std::pair<std::string, double>> v;
  void add(const char* name, std::chrono::steady_clock::time_point t0) {
    if (on) v.emplace_back(name, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
  }
  void print() const {
    if (!on) return;
    std::string o = "[sxhmm profile]";
    char buf[96];
    for (const auto& p : v) {
      snprintf(buf, sizeof buf, " %s=%.1fms", p.first.c_str(), p.second);
      o += buf;
    }
    fprintf(stderr, "%s\n", o.c_str());
  }
};

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

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
  void alloc(size_t count) {  // grow-only, contents undefined
    if (count <= n && p) return;
    release();
    CK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    n = std::max<size_t>(count, 1);
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

const KernelTables& kernels() {
  static const KernelTables t = [] {
    KernelTables k;
    fill_msv_tables(k);
    fill_msv16_tables(k);
    fill_vit_tables(k);
    fill_vit16_tables(k);
    fill_vbin_tables(k);
    fill_env_tables(k);
    return k;
  }();
  return t;
}

// Pick the MSV shape with the fewest issued instructions per useful DP cell.
// Per row a warp issues about 2.75*C instructions of cell work (FADD, FMNMX,
// a share of FMNMX3 and LDS.128) plus ~44 of per-row overhead (residue
// extraction, shuffles, specials) and 2 per butterfly step; it advances 32/G
// targets by M cells each (fitted to ncu instruction counts on B200).
int choose_msv_shape(int m) {
  int best = -1;
  double best_cost = 1e30;
  for (int s = 0; s < kNumMsvShapes; s++) {
    const int g = kMsvShapes[s].g, c = kMsvShapes[s].c;
    if (g * c < m) continue;
    const double instr = 2.75 * c + 44.0 + 2.0 * std::log2((double)g);
    const double cost = instr / ((32.0 / g) * m);
    if (cost < best_cost * 0.999) {
      best_cost = cost;
      best = s;
    }
  }
  return best;
}
// Viterbi shape: per row a lane does ~19 instructions per column (16 lane-ops
// plus 9 loads per 4 columns) and ~50 of overhead; lanes per pair cost
// lazy-F carry rounds and butterfly steps; C >= 24 halves occupancy.
int choose_vit_shape(int m) {
  int best = -1;
  double best_cost = 1e30;
  for (int s = 0; s < kNumVitShapes; s++) {
    const int g = kVitShapes[s].g, c = kVitShapes[s].c;
    if (g * c < m) continue;
    // per-row lane instructions; register-held transitions save the 8 loads per 4 columns
    const double per_row = (kVitShapes[s].rt ? 9.0 : 19.0) * c + 50.0 + 12.0 * std::log2((double)g);
    const double occ = vit_ctas_per_sm(kVitShapes[s]) == 2 ? 1.0 : 0.5;
    const double cost = per_row * g / (32.0 * m) / occ;
    if (cost < best_cost * 0.999) {
      best_cost = cost;
      best = s;
    }
  }
  return best;
}
// Persistent grid for a lane-group Viterbi launch of `n` pairs: the CTAs that
// fit on the GPU at once (two per SM for C <= 16, whose registers are capped
// at 128, one otherwise), fewer if the pairs need fewer groups.
int vit_blocks(int num_sms, int shape, unsigned n) {
  const int g = kVitShapes[shape].g, per_sm = vit_ctas_per_sm(kVitShapes[shape]);
  return (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)n * g + 255) / 256, (int64_t)num_sms * per_sm));
}

// Packed Viterbi pre-screen shape of a profile: the narrowest that covers M;
// -1 when none does.
int choose_vit16_shape(int m) {
  for (int s = 0; s < kNumVit16Shapes; s++)
    if (kVit16Shapes[s].g * kVit16Shapes[s].c >= m) return s;
  return -1;
}

// Forward/Backward pass kernels run one warp per pair in one-warp CTAs, so a
// warp that finishes frees its SM slot at once instead of holding it until
// the longest pair of a larger CTA is done.
int warp_ctas(int num_sms, unsigned n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)n, (int64_t)num_sms * 32));
}

int choose_vbin(int m) {
  const int need = (m + 31) / 32;
  for (int b = 0; b < kNumVbins; b++)
    if (kVcBins[b] >= need) return b;
  return -1;
}

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
class HostBytePool {
 public:
  std::vector<uint8_t> take(size_t bytes) {
    std::lock_guard<std::mutex> g(mu_);
    for (size_t i = 0; i < free_.size(); i++)
      if (free_[i].capacity() >= bytes) {
        std::vector<uint8_t> v = std::move(free_[i]);
        free_.erase(free_.begin() + (std::ptrdiff_t)i);
        v.clear();
        return v;
      }
    std::vector<uint8_t> v;
    v.reserve(bytes);
    return v;
  }
  void give(std::vector<uint8_t>&& v) {
    if (!v.capacity()) return;
    std::lock_guard<std::mutex> g(mu_);
    free_.push_back(std::move(v));
    if (free_.size() > 2)  // keep the two largest
      free_.erase(std::min_element(free_.begin(), free_.end(),
                                   [](const auto& x, const auto& y) { return x.capacity() < y.capacity(); }));
  }

 private:
  std::mutex mu_;
  std::vector<std::vector<uint8_t>> free_;
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
    // 2 slots x (9 + 6) streams + 2 envelope streams = 32, the
    // most hardware work queues a process can have (CUDA_DEVICE_MAX_CONNECTIONS=32):
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

}  // namespace

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
  cudaStream_t env_stream = nullptr, env_stream2 = nullptr;  // Backward runs beside Forward
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
};

struct sx_targets {
  sx_engine* eng = nullptr;
  std::vector<std::string> ids;  // caller's names (sx_targets_create); empty for digital sets
  std::vector<uint8_t> dsq;  // packed digital residues, each target 16-byte aligned
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

namespace {

// Fan independent launches out over the auxiliary streams and join them back
// into the engine stream.
void fork_aux(Streams& X) {
  CK(cudaEventRecord(X.fork_ev, X.main));
  for (int a = 0; a < X.naux; a++) CK(cudaStreamWaitEvent(X.aux[a], X.fork_ev, 0));
}
void join_aux(Streams& X) {
  for (int a = 0; a < X.naux; a++) {
    CK(cudaEventRecord(X.join_ev[a], X.aux[a]));
    CK(cudaStreamWaitEvent(X.main, X.join_ev[a], 0));
  }
}

// The built-in shape table of a kind: for Viterbi the shapes measured fastest
// per range of M on B200 (tuned_shapes.inc, written by sxhmm/tune.py); none for
// MSV, whose cost model was fitted to ncu instruction counts.
std::vector<int16_t> default_shape_table(int kind) {
  std::vector<int16_t> t;
  if (kind != 1) return t;
  t.assign(kMaxM + 1, -1);
  for (const auto& r : kTunedVit) {
    int idx = -1;
    for (int s = 0; s < kNumVitShapes; s++)
      if (kVitShapes[s].g == r[2] && kVitShapes[s].c == r[3] && kVitShapes[s].rt == r[4]) idx = s;
    if (idx < 0 || kVitShapes[idx].g * kVitShapes[idx].c < r[1]) continue;
    for (int m = std::max(r[0], 0); m <= r[1] && m <= kMaxM; m++) t[(size_t)m] = (int16_t)idx;
  }
  return t;
}

// Kernel shape for a profile of length m: the engine's table where it has an
// entry, else the cost model (kind 0 MSV, 1 Viterbi).
int shape_for(const sx_engine* E, int kind, int m) {
  const auto& t = E->shape_table[kind];
  if (m >= 0 && (size_t)m < t.size() && t[(size_t)m] >= 0) return t[(size_t)m];
  return kind == 0 ? choose_msv_shape(m) : choose_vit_shape(m);
}

// ---- profile packing --------------------------------------------------------
// The images of a profile the warp-chunked and lane-group kernels read.
void pack_images(const ProfileHost& h, const DevProfile& d, float4* msv, float4* vit, float* vfb) {
  const int m = h.m;
  // MSV image: residue row x, float4 chunk c4 of lane j at (x*NC4 + c4)*G + j;
  // lane j's column c is k = j*C + c + 1.
  {
    const int G = d.msv_g, C = d.msv_c, NC4 = C / 4;
    float4* base = msv + d.msv_off;
    for (int x = 0; x < 25; x++)
      for (int j = 0; j < G; j++)
        for (int c4 = 0; c4 < NC4; c4++) {
          float v[4];
          for (int e = 0; e < 4; e++) {
            const int k = j * C + c4 * 4 + e + 1;
            v[e] = k <= m ? h.msc_row(x)[k] : kNegInf;
          }
          base[((size_t)x * NC4 + c4) * G + j] = make_float4(v[0], v[1], v[2], v[3]);
        }
  }
  // Viterbi image: rows 0..24 log-odds, 25..32 transitions (mm im dm at k-1, bm mi ii at k,
  // md dd at k-1), lane-major float4 chunks as for MSV
  {
    const int G = kVitShapes[d.vshape].g, C = kVitShapes[d.vshape].c, NC4 = C / 4;
    float4* base = vit + d.vit_off;
    auto row = [&](int r, const std::function<float(int)>& f, float pad) {
      for (int j = 0; j < G; j++)
        for (int c4 = 0; c4 < NC4; c4++) {
          float v[4];
          for (int e = 0; e < 4; e++) {
            const int k = j * C + c4 * 4 + e + 1;
            v[e] = k <= m ? f(k) : pad;
          }
          base[((size_t)r * NC4 + c4) * G + j] = make_float4(v[0], v[1], v[2], v[3]);
        }
    };
    for (int x = 0; x < 25; x++) row(x, [&](int k) { return h.msc_row(x)[k]; }, kNegInf);
    const auto& t = h.t;
    row(25, [&](int k) { return t[TMM][k - 1]; }, kNegInf);
    row(26, [&](int k) { return t[TIM][k - 1]; }, kNegInf);
    row(27, [&](int k) { return t[TDM][k - 1]; }, kNegInf);
    row(28, [&](int k) { return t[TBM][k]; }, kNegInf);
    // no insert state at node M: -inf from k = M on keeps I_M.. at -inf
    row(29, [&](int k) { return k < m ? t[TMI][k] : kNegInf; }, kNegInf);
    row(30, [&](int k) { return k < m ? t[TII][k] : kNegInf; }, kNegInf);
    row(31, [&](int k) { return t[TMD][k - 1]; }, kNegInf);
    row(32, [&](int k) { return t[TDD][k - 1]; }, kNegInf);
  }
  // warp-chunked image: row r, lane l, column c (k = l*vc + c + 1) at (r*vc + c)*32 + l
  {
    const int vc = d.vc;
    float* base = vfb + d.vfb_off;
    auto put = [&](int r, const std::function<float(int)>& f, float pad) {
      for (int l = 0; l < 32; l++)
        for (int c = 0; c < vc; c++) {
          const int k = l * vc + c + 1;
          base[((size_t)r * vc + c) * 32 + l] = k <= m ? f(k) : pad;
        }
    };
    for (int x = 0; x < 25; x++) {
      put(sxk::kRowMsc + x, [&](int k) { return h.msc_row(x)[k]; }, kNegInf);
      put(sxk::kRowMo + x, [&](int k) { return h.mo_row(x)[k]; }, 0.0f);
    }
    const auto& t = h.t;
    const auto& p = h.p;
    auto shl = [&](const std::vector<float>& v) { return [&v](int k) { return v[k - 1]; }; };
    auto at = [&](const std::vector<float>& v) { return [&v](int k) { return v[k]; }; };
    put(sxk::kRowVit + 0, shl(t[TMM]), kNegInf);
    put(sxk::kRowVit + 1, shl(t[TIM]), kNegInf);
    put(sxk::kRowVit + 2, shl(t[TDM]), kNegInf);
    put(sxk::kRowVit + 3, at(t[TBM]), kNegInf);
    put(sxk::kRowVit + 4, at(t[TMI]), kNegInf);
    put(sxk::kRowVit + 5, at(t[TII]), kNegInf);
    put(sxk::kRowVit + 6, shl(t[TMD]), kNegInf);
    put(sxk::kRowVit + 7, shl(t[TDD]), kNegInf);
    put(sxk::kRowFwd + 0, at(p[TBM]), 0.0f);
    put(sxk::kRowFwd + 1, shl(p[TMM]), 0.0f);
    put(sxk::kRowFwd + 2, shl(p[TIM]), 0.0f);
    put(sxk::kRowFwd + 3, shl(p[TDM]), 0.0f);
    put(sxk::kRowFwd + 4, at(p[TMI]), 0.0f);
    put(sxk::kRowFwd + 5, at(p[TII]), 0.0f);
    put(sxk::kRowFwd + 6, shl(p[TMD]), 0.0f);
    put(sxk::kRowFwd + 7, shl(p[TDD]), 0.0f);
    put(sxk::kRowBwd + 0, at(p[TMM]), 0.0f);
    put(sxk::kRowBwd + 1, at(p[TMI]), 0.0f);
    put(sxk::kRowBwd + 2, at(p[TMD]), 0.0f);
    put(sxk::kRowBwd + 3, at(p[TIM]), 0.0f);
    put(sxk::kRowBwd + 4, at(p[TII]), 0.0f);
    put(sxk::kRowBwd + 5, at(p[TDM]), 0.0f);
    put(sxk::kRowBwd + 6, at(p[TDD]), 0.0f);
    put(sxk::kRowBwd + 7, at(p[TBM]), 0.0f);
  }
}

// Quantized MSV image of the packed pre-screen (prescreen.cuh): the match
// scores in units of 2^-9 nat rounded up after adding 2^-12 nat, clamped up to
// -16 nats (-inf included), -32 nats past column M, in the lane-major chunk
// layout of the profile's f32 MSV image (4 columns per uint2).  Returns the
// largest rounded score of a real column; the profile's cap is 32767 minus it.
int pack_qimage(const ProfileHost& h, const DevProfile& d, uint2* out) {
  const int m = h.m, G = d.msv_g, C = d.msv_c, NC4 = C / 4;
  int emax = sxk::kQ16EFloor;
  auto q = [&](int x, int k) -> int {
    if (k > m) return sxk::kQ16EPad;
    const float e = h.msc_row(x)[k];
    if (!(e > -1e30f)) return sxk::kQ16EFloor;  // -inf (and NaN, which no configured profile has)
    const double u = std::ceil(((double)e + std::ldexp(1.0, -12)) * 512.0);
    const int v = (int)std::max<double>(u, (double)sxk::kQ16EFloor);
    emax = std::max(emax, v);
    return v;
  };
  uint2* base = out + d.q_off;
  for (int x = 0; x < 25; x++)
    for (int j = 0; j < G; j++)
      for (int c4 = 0; c4 < NC4; c4++) {
        int v[4];
        for (int e = 0; e < 4; e++) v[e] = q(x, j * C + c4 * 4 + e + 1);
        uint2 w;
        w.x = (uint32_t)(v[0] & 0xffff) | ((uint32_t)(v[1] & 0xffff) << 16);
        w.y = (uint32_t)(v[2] & 0xffff) | ((uint32_t)(v[3] & 0xffff) << 16);
        base[((size_t)x * NC4 + c4) * G + j] = w;
      }
  return emax;
}

// Quantized Viterbi image of the packed pre-screen (prescreen.cuh
// vit16_kernel), in units of 2^-9 nat: every score rounded up after adding
// 2^-12 nat; match scores clamped up to -8 nats, transitions clamped to
// [-8 nats, 0] (t_bm to [-16 nats, 0]); -inf scores and columns past M take
// the floor.  8 transition rows (each column's score in both int16 halves of
// a word, 4 columns per uint4), then 25 match-score rows (4 columns per
// uint2), lane-major like the f32 Viterbi image, at width G*C of the
// profile's pre-screen shape.  Returns the largest rounded match score.
int pack_qvimage(const ProfileHost& h, const DevProfile& d, uint4* out) {
  const int m = h.m, G = kVit16Shapes[d.qv_shape].g, C = kVit16Shapes[d.qv_shape].c, NC4 = C / 4;
  auto up = [](float v) { return std::ceil(((double)v + std::ldexp(1.0, -12)) * 512.0); };
  int emax = sxk::kV16EFloor;
  auto em = [&](int x, int k) -> int {
    if (k > m) return sxk::kV16EFloor;
    const float e = h.msc_row(x)[k];
    if (!(e > -1e30f)) return sxk::kV16EFloor;
    const int v = (int)std::max<double>(up(e), (double)sxk::kV16EFloor);
    emax = std::max(emax, v);
    return v;
  };
  auto tq = [&](float t, int floor) -> int {
    if (!(t > -1e30f)) return floor;
    return (int)std::max<double>(std::min<double>(up(t), 0.0), (double)floor);
  };
  const auto& t = h.t;
  // transition row q of column k (the f32 Viterbi image's rows 25..32)
  auto tr = [&](int q, int k) -> int {
    if (k > m) return q == 3 ? sxk::kV16BmFloor : sxk::kV16TFloor;
    switch (q) {
      case 0: return tq(t[TMM][k - 1], sxk::kV16TFloor);
      case 1: return tq(t[TIM][k - 1], sxk::kV16TFloor);
      case 2: return tq(t[TDM][k - 1], sxk::kV16TFloor);
      case 3: return tq(t[TBM][k], sxk::kV16BmFloor);
      case 4: return k < m ? tq(t[TMI][k], sxk::kV16TFloor) : sxk::kV16TFloor;
      case 5: return k < m ? tq(t[TII][k], sxk::kV16TFloor) : sxk::kV16TFloor;
      case 6: return tq(t[TMD][k - 1], sxk::kV16TFloor);
      default: return tq(t[TDD][k - 1], sxk::kV16TFloor);
    }
  };
  auto dup = [](int v) { return ((uint32_t)v & 0xffffu) * 0x10001u; };
  uint4* base = out + d.qv_off;
  const size_t row4 = (size_t)NC4 * G;
  for (int q = 0; q < 8; q++)
    for (int j = 0; j < G; j++)
      for (int c4 = 0; c4 < NC4; c4++) {
        const int k = j * C + c4 * 4 + 1;
        base[(q * NC4 + c4) * G + j] = make_uint4(dup(tr(q, k)), dup(tr(q, k + 1)), dup(tr(q, k + 2)), dup(tr(q, k + 3)));
      }
  uint2* es = reinterpret_cast<uint2*>(base + 8 * row4);
  for (int x = 0; x < 25; x++)
    for (int j = 0; j < G; j++)
      for (int c4 = 0; c4 < NC4; c4++) {
        int v[4];
        for (int e = 0; e < 4; e++) v[e] = em(x, j * C + c4 * 4 + e + 1);
        uint2 w;
        w.x = (uint32_t)(v[0] & 0xffff) | ((uint32_t)(v[1] & 0xffff) << 16);
        w.y = (uint32_t)(v[2] & 0xffff) | ((uint32_t)(v[3] & 0xffff) << 16);
        es[((size_t)x * NC4 + c4) * G + j] = w;
      }
  return emax;
}
// uint4 entries of a quantized Viterbi image of shape s
int64_t qvimage_size(int s) {
  const int64_t row4 = (int64_t)(kVit16Shapes[s].c / 4) * kVit16Shapes[s].g;
  return 8 * row4 + 25 * row4 / 2;
}

// Composition-bias filter table (src/hmmer/pipeline.rs:110-131): 54 doubles.
void pack_bias(const ProfileHost& h, double* b) {
  const int m = h.m;
  for (int x = 0; x < 25; x++) b[x] = b[25 + x] = 1.0;
  for (int x = 0; x < NRES; x++) b[25 + x] = (double)h.compo[x] / (double)kBackground[x];
  for (int code = 20; code <= 23; code++) {
    const Degenerate& dg = degenerate(code);
    double e0 = 0, e1 = 0, z = 0;
    for (int q = 0; q < dg.n; q++) {
      e0 += (double)kBackground[dg.members[q]];
      e1 += (double)h.compo[dg.members[q]];
      z += (double)kBackground[dg.members[q]];
    }
    b[code] = e0 / z;
    b[25 + code] = e1 / z;
  }
  const double l0 = 400.0, l1 = (double)m / 8.0;
  b[50] = l0 / (l0 + 1.0);
  b[51] = 1.0 / (l0 + 1.0);
  b[52] = 1.0 / (l1 + 1.0);
  b[53] = l1 / (l1 + 1.0);
}

void pack_profiles(sx_profiles* P) {
  const size_t np = P->h.size();
  P->dp.resize(np);
  P->msv_shape.resize(np);
  int64_t msv_total = 0, vfb_total = 0, vit_total = 0, q_total = 0, qv_total = 0;
  for (size_t i = 0; i < np; i++) {
    const ProfileHost& h = P->h[i];
    DevProfile& d = P->dp[i];
    memset(&d, 0, sizeof d);
    d.m = h.m;
    d.msv_tbm = h.msv_tbm;
    if (is_long(h.m)) {  // no warp-chunked, MSV or Viterbi images: the long kernels read the plain image
      P->msv_shape[i] = -1;
      d.vbin = d.vshape = -1;
      d.msv_off = msv_total;
      d.vfb_off = vfb_total;
      d.vit_off = vit_total;
      d.q_off = -1;
      d.qv_shape = -1;
      d.qv_off = -1;
      continue;
    }
    const int s = shape_for(P->eng, 0, h.m);
    const int vb = choose_vbin(h.m);
    if (s < 0 || vb < 0) throw CudaError{SX_EINVAL, "profile '" + h.name + "': no kernel shape for M=" + std::to_string(h.m)};
    P->msv_shape[i] = s;
    d.msv_g = kMsvShapes[s].g;
    d.msv_c = kMsvShapes[s].c;
    d.vbin = vb;
    d.vc = kVcBins[vb];
    d.msv_off = msv_total;
    msv_total += 25LL * (d.msv_c / 4) * d.msv_g;
    d.q_off = q_total;
    q_total += 25LL * (d.msv_c / 4) * d.msv_g;
    d.q_tbm = (int32_t)std::ceil(((double)h.msv_tbm + std::ldexp(1.0, -17)) * 1048576.0);
    d.vfb_off = vfb_total;
    vfb_total += (int64_t)sxk::kImgRows * 32 * d.vc;
    d.vshape = shape_for(P->eng, 1, h.m);
    if (d.vshape < 0) throw CudaError{SX_EINVAL, "profile '" + h.name + "' too long for the Viterbi shapes"};
    d.vit_off = vit_total;
    vit_total += 33LL * (kVitShapes[d.vshape].c / 4) * kVitShapes[d.vshape].g;
    d.qv_shape = choose_vit16_shape(h.m);
    d.qv_off = -1;
    if (d.qv_shape >= 0) {
      d.qv_off = qv_total;
      qv_total += qvimage_size(d.qv_shape);
    }
  }
  std::vector<float4> msv((size_t)msv_total);
  std::vector<float4> vit((size_t)std::max<int64_t>(vit_total, 1));
  std::vector<float> vfb((size_t)vfb_total);
  std::vector<double> bias(np * 54);
  std::vector<uint2> qimg((size_t)std::max<int64_t>(q_total, 1));
  std::vector<uint4> qvimg((size_t)std::max<int64_t>(qv_total, 1));
  for (size_t i = 0; i < np; i++) {
    if (P->dp[i].vbin >= 0) {
      pack_images(P->h[i], P->dp[i], msv.data(), vit.data(), vfb.data());
      // a profile whose rounded scores leave less than half of the int16
      // range as headroom (scores above +16 nats) stays on the exact kernel
      const int emax = pack_qimage(P->h[i], P->dp[i], qimg.data());
      if (emax < 8192) P->dp[i].q_cap = 32767 - emax;
      else P->dp[i].q_off = -1;
      // the Viterbi pre-screen takes the MSV pre-screen's profiles (whose
      // bias-filter survivors fit the per-profile lists of the MSV rescoring)
      // whose rounded match scores leave at least half of the int16 range
      DevProfile& d = P->dp[i];
      if (d.qv_shape >= 0 && d.q_off >= 0) {
        const int vmax = pack_qvimage(P->h[i], d, qvimg.data());
        if (vmax < 8192) d.qv_cap = 32767 - vmax;
        else d.qv_shape = -1;
      } else {
        d.qv_shape = -1;
      }
    }
    pack_bias(P->h[i], bias.data() + i * 54);
  }
  // plain layout: 25 msc rows then mm mi md im ii dm dd bm, each M+1 long;
  // long profiles add the 25 odds rows and the 8 probability rows (same order),
  // the image of the long kernels
  std::vector<sxk::PlainProfile> pprof(np);
  int64_t plain_total = 0;
  for (size_t i = 0; i < np; i++) {
    pprof[i].off = plain_total;
    pprof[i].m = P->h[i].m;
    pprof[i].pad = 0;
    plain_total += (is_long(P->h[i].m) ? (int64_t)sxk::kLongRows : 33LL) * (P->h[i].m + 1);
  }
  std::vector<float> plain((size_t)std::max<int64_t>(plain_total, 1));
  for (size_t i = 0; i < np; i++) {
    const ProfileHost& h = P->h[i];
    const size_t w = (size_t)h.m + 1;
    float* b = plain.data() + pprof[i].off;
    memcpy(b, h.msc.data(), sizeof(float) * 25 * w);
    const int order[8] = {TMM, TMI, TMD, TIM, TII, TDM, TDD, TBM};
    for (int q = 0; q < 8; q++) memcpy(b + (25 + q) * w, h.t[order[q]].data(), sizeof(float) * w);
    if (is_long(h.m)) {
      memcpy(b + sxk::kLMo * w, h.mo.data(), sizeof(float) * 25 * w);
      for (int q = 0; q < 8; q++) memcpy(b + (sxk::kLP + q) * w, h.p[order[q]].data(), sizeof(float) * w);
    }
  }
  cudaStream_t s = P->eng->stream;
  P->d_pprof.upload(pprof.data(), np, s);
  P->d_plain.upload(plain.data(), plain.size(), s);
  P->d_prof.upload(P->dp.data(), np, s);
  P->d_msv.upload(msv.data(), msv.size(), s);
  P->d_qimg.upload(qimg.data(), qimg.size(), s);
  P->d_qvimg.upload(qvimg.data(), qvimg.size(), s);
  P->d_vit.upload(vit.data(), vit.size(), s);
  P->d_vfb.upload(vfb.data(), vfb.size(), s);
  P->d_bias.upload(bias.data(), bias.size(), s);
  CK(cudaStreamSynchronize(s));
}

// ---- target packing ---------------------------------------------------------
void pack_targets(sx_targets* T) {
  const size_t n = T->len.size();
  std::vector<float4> tpar(n), xsc(n);
  T->residues = 0;
  // the length constants depend on L alone: computed once per distinct length
  std::unordered_map<int64_t, std::pair<float4, float4>> by_len;
  for (size_t i = 0; i < n; i++) {
    const int64_t l = T->len[i];
    auto it = by_len.find(l);
    if (it == by_len.end()) {
      const float lf = (float)l;
      // MSV length model (src/hmmer/dp.rs:98-100) and the multihit Xsc (model.rs:284-312)
      const float tloop = std::log(lf / (lf + 3.0f));
      const float tmove = std::log(3.0f / (lf + 3.0f));
      const SpecialTr st = special_transitions(l, true);
      it = by_len.emplace(l, std::make_pair(make_float4(tloop, tmove, null1_score(l), 0.0f),
                                            make_float4(st.loop, st.move, st.ploop, st.pmove))).first;
    }
    tpar[i] = it->second.first;
    xsc[i] = it->second.second;
    T->residues += (double)l;
  }
  // indices by length, longest first, ties in input order (a counting sort
  // when the lengths allow one)
  T->order.resize(n);
  int32_t mx = 0;
  for (size_t i = 0; i < n; i++) mx = std::max(mx, T->len[i]);
  if (mx <= (1 << 22)) {
    std::vector<int32_t> start((size_t)mx + 2, 0);
    for (size_t i = 0; i < n; i++) start[(size_t)(mx - T->len[i]) + 1]++;
    for (size_t k = 1; k < start.size(); k++) start[k] += start[k - 1];
    for (size_t i = 0; i < n; i++) T->order[(size_t)start[(size_t)(mx - T->len[i])]++] = (int32_t)i;
  } else {
    std::iota(T->order.begin(), T->order.end(), 0);
    std::stable_sort(T->order.begin(), T->order.end(), [&](int a, int b) { return T->len[a] > T->len[b]; });
  }
  cudaStream_t s = T->eng->stream;
  // all arrays in one pooled block, each 256-byte aligned
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t o_res = 0, o_off = o_res + up(T->dsq.size()), o_len = o_off + up(8 * n), o_tpar = o_len + up(4 * n);
  const size_t o_xsc = o_tpar + up(16 * n), o_order = o_xsc + up(16 * n), total = o_order + up(4 * n);
  if (T->block) T->eng->target_blocks.give(T->block, T->block_bytes);
  T->block = T->eng->target_blocks.take(total, T->block_bytes);
  char* b = static_cast<char*>(T->block);
  T->d_res.view(b + o_res, T->dsq.size());
  T->d_off.view(b + o_off, n);
  T->d_len.view(b + o_len, n);
  T->d_tpar.view(b + o_tpar, n);
  T->d_xsc.view(b + o_xsc, n);
  T->d_order.view(b + o_order, n);
  auto put = [&](void* dst, const void* src, size_t bytes) {
    if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
  };
  put(T->d_res.p, T->dsq.data(), T->dsq.size());
  put(T->d_off.p, T->off.data(), 8 * n);
  put(T->d_len.p, T->len.data(), 4 * n);
  put(T->d_tpar.p, tpar.data(), 16 * n);
  put(T->d_xsc.p, xsc.data(), 16 * n);
  put(T->d_order.p, T->order.data(), 4 * n);
  CK(cudaStreamSynchronize(s));
}

void append_target(sx_targets* T, const uint8_t* dig, size_t l) {
  const int64_t o = (int64_t)T->dsq.size();
  T->off.push_back(o);
  T->len.push_back((int32_t)l);
  T->dsq.insert(T->dsq.end(), dig, dig + l);
  // pad to a 16-byte boundary; kernels read up to 48 bytes past a target
  size_t padded = (T->dsq.size() + 15) & ~(size_t)15;
  T->dsq.resize(padded, SYM_STAR);
}

// ---- thresholds ---------------------------------------------------------------
// Per profile, the smallest f32 bit statistic that passes each filter
// (pipeline.rs:164-183).  The tails are monotone in the statistic, except the
// Gumbel survival around its branch at 1e-5; a threshold within 2% of that
// point disables device filtering for the stage (the host still decides).
std::vector<Thresholds> make_thresholds(const std::vector<ProfileHost>& H, const SearchOpts& o) {
  std::vector<Thresholds> th(H.size());
  auto near_branch = [](double f) { return f > 0.98e-5 && f < 1.02e-5; };
  for (size_t i = 0; i < H.size(); i++) {
    const ProfileHost& h = H[i];
    Thresholds& t = th[i];
    if (!o.filters || !h.calibrated()) {
      t.s1 = t.s2 = t.s3 = -INFINITY;
      t.exact = 0;
      continue;
    }
    t.exact = 1;
    const double mmu = h.msv[0], mlam = h.msv[1], vmu = h.vit[0], vlam = h.vit[1], ftau = h.fwd[0], flam = h.fwd[1];
    t.s1 = near_branch(o.f1) ? -INFINITY : f32_boundary([&](float s) { return !(gumbel_survival((double)s, mmu, mlam) > o.f1); });
    t.s2 = near_branch(o.f2) ? -INFINITY : f32_boundary([&](float s) { return !(gumbel_survival((double)s, vmu, vlam) > o.f2); });
    t.s3 = f32_boundary([&](float s) { return !(std::exp(exp_tail_logsurv((double)s, ftau, flam)) > o.f3); });
    if (std::isnan(t.s1)) t.s1 = -INFINITY;
    if (std::isnan(t.s2)) t.s2 = -INFINITY;
    if (std::isnan(t.s3)) t.s3 = -INFINITY;
  }
  return th;
}

constexpr float kSlackBits = 1.0e-3f;  // device-log decisions: never reject what the reference keeps

struct StageLists {
  std::vector<BinRegion> reg;
  int64_t total = 0;
};

StageLists make_regions(const std::vector<double>& want) {
  StageLists s;
  s.reg.resize(kMaxBins);
  int64_t off = 0;
  for (int b = 0; b < kMaxBins; b++) {
    const uint32_t cap = b < (int)want.size() ? (uint32_t)std::min<double>(std::max(want[b], 0.0), 4.0e9) : 0u;
    s.reg[b].off = off;
    s.reg[b].cap = cap;
    s.reg[b].pad = 0;
    off += cap;
  }
  s.total = off;
  return s;
}

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

// Device memory free when the engine was created (0 = unknown).  Queried once:
// with the query at the start of every search, a stream of end-to-end
// searches ran tens of milliseconds slower per call.
void note_free_memory(sx_engine* E) {
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    cudaGetLastError();
    fr = 0;
  }
  E->mem_free = (int64_t)fr;
}
// Bytes a pass may take for its scratch: the configured budget, capped by half
// of the device memory that was free when the engine was created (other
// processes on the GPU, other engines), and never below 64 MB.
int64_t scratch_budget(const sx_engine* E, int64_t want) {
  if (E->mem_free <= 0) return want;
  return std::max<int64_t>(std::min<int64_t>(want, E->mem_free / 2), 64LL << 20);
}

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

// Row passes of a block's final pairs queued without waiting: when all of
// their rows fit one chunk, the kernels go to slot S's high-priority streams
// with the slot's own row buffers and the call returns a fetch function; a
// host job calls it, which waits for the kernels, copies the rows out on the
// slot's copy stream, adds the passes' device time to *dev_ms and releases
// the buffers.  Returns an empty function when the rows need more than one
// chunk (the caller then takes the synchronous rows_pass).
constexpr int kRowsWarps = 8;  // warps (pairs) per CTA of the asynchronous row passes
std::function<RowsChunk()> rows_pass_async(sx_engine* E, Slot& S, const sx_profiles* P, const sx_targets* T,
                                           const std::vector<FinalPair>& pairs, std::mutex* ms_mu, double* dev_ms) {
  const auto& K = kernels();
  const int64_t row_budget = std::max<int64_t>(scratch_budget(E, E->batch_bytes / 2) / (int64_t)sizeof(float), 1 << 20);
  int64_t ro = 0;
  for (const FinalPair& f : pairs) ro += 6 * ((int64_t)T->len[f.t] + 1);
  if (pairs.empty() || ro > row_budget) return {};
  if (S.rows_busy) S.rows_busy->wait();  // an earlier block's rows are still being read
  std::vector<std::vector<size_t>> byb(kNumVbins);
  for (size_t i = 0; i < pairs.size(); i++) byb[P->dp[pairs[i].p].vbin].push_back(i);
  // longest first: the warps of a CTA then carry similar lengths, and the
  // longest chains start first
  for (auto& v : byb)
    std::stable_sort(v.begin(), v.end(), [&](size_t a, size_t b) { return T->len[pairs[a].t] > T->len[pairs[b].t]; });
  std::vector<PairRec> recs;
  auto c = std::make_shared<RowsChunk>();
  std::vector<BinRegion> reg(kNumVbins);
  std::vector<unsigned> cnt(kNumVbins, 0);
  ro = 0;
  for (int b = 0; b < kNumVbins; b++) {
    reg[b].off = (int64_t)recs.size();
    reg[b].cap = (uint32_t)byb[b].size();
    reg[b].pad = 0;
    cnt[b] = (unsigned)byb[b].size();
    for (size_t i : byb[b]) {
      const FinalPair& f = pairs[i];
      recs.push_back({f.p, f.t, f.usc, f.filtersc, f.vsc, 0.f, f.slot, 0});
      c->off.push_back(ro);
      c->which.push_back(i);
      ro += 6 * ((int64_t)T->len[f.t] + 1);
    }
  }
  cudaStream_t s = S.hi.main;
  S.rrecs.upload(recs.data(), recs.size(), s);
  S.roff.upload(c->off.data(), c->off.size(), s);
  S.rbins.upload(reg.data(), reg.size(), s);
  S.rcnt.upload(cnt.data(), cnt.size(), s);
  S.rows_f.alloc((size_t)ro);
  S.rows_b.alloc((size_t)ro);
  CK(cudaEventRecord(S.rows_t0, s));
  // rows the kernels never touch are zero
  CK(cudaMemsetAsync(S.rows_f.p, 0, sizeof(float) * (size_t)ro, s));
  CK(cudaMemsetAsync(S.rows_b.p, 0, sizeof(float) * (size_t)ro, s));
  fork_aux(S.hi);
  for (int b = 0; b < kNumVbins; b++) {
    if (!cnt[b]) continue;
    // The row passes are latency-bound chains that run for milliseconds
    // beside the next block's MSV: packed kRowsWarps to a CTA they hold the
    // registers of a few SMs instead of one MSV CTA slot on nearly every SM.
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)cnt[b] + kRowsWarps - 1) / kRowsWarps,
                                                                   (int64_t)E->num_sms * 32 / kRowsWarps));
    cudaStream_t sa = S.hi.aux[(2 * b) % S.hi.naux], sb = S.hi.aux[(2 * b + 1) % S.hi.naux];
    K.fwd[b]<<<blocks, 32 * kRowsWarps, 0, sa>>>(S.rrecs.p, S.rcnt.p, S.rbins.p, b, nullptr, nullptr, nullptr, S.overflow.p,
                                     P->d_prof.p, E->thr.p, P->d_vfb.p, T->d_res.p, T->d_off.p, T->d_len.p,
                                     T->d_xsc.p, 0.f, S.rows_f.p, S.roff.p);
    K.bwd[b]<<<blocks, 32 * kRowsWarps, 0, sb>>>(S.rrecs.p, S.rcnt.p, S.rbins.p, b, P->d_prof.p, P->d_vfb.p, T->d_res.p,
                                     T->d_off.p, T->d_len.p, T->d_xsc.p, S.rows_b.p, S.roff.p);
    E->stats.kernel_launches += 2;
  }
  CK(cudaGetLastError());
  join_aux(S.hi);
  CK(cudaEventRecord(S.rows_t1, s));
  auto ticket = std::make_shared<RowsTicket>();
  S.rows_busy = ticket;
  Slot* SP = &S;
  const int device = E->device;
  return [SP, c, ro, ticket, ms_mu, dev_ms, device]() -> RowsChunk {
    struct Release {  // the buffers are free again, even if a copy failed
      RowsTicket& t;
      ~Release() { t.set(); }
    } rel{*ticket};
    Slot& S = *SP;
    CK(cudaSetDevice(device));
    CK(cudaStreamWaitEvent(S.rows_copy, S.rows_t1, 0));
    c->f.resize((size_t)ro);
    c->b.resize((size_t)ro);
    CK(cudaMemcpyAsync(c->f.data(), S.rows_f.p, sizeof(float) * (size_t)ro, cudaMemcpyDeviceToHost, S.rows_copy));
    CK(cudaMemcpyAsync(c->b.data(), S.rows_b.p, sizeof(float) * (size_t)ro, cudaMemcpyDeviceToHost, S.rows_copy));
    CK(cudaStreamSynchronize(S.rows_copy));
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, S.rows_t0, S.rows_t1) != cudaSuccess) cudaGetLastError();
    {
      std::lock_guard<std::mutex> g(*ms_mu);
      *dev_ms += ms;
    }
    return std::move(*c);
  };
}

// Background host work: one driver thread runs the queued jobs in order, each
// over `threads` workers, while the engine thread keeps the device busy with
// later profile blocks.
class HostQueue {
 public:
  explicit HostQueue(int threads) : threads_(std::max(1, threads)), th_([this] { loop(); }) {}
  ~HostQueue() { finish(); }
  void push(std::function<void(int)> job) {
    {
      std::lock_guard<std::mutex> g(mu_);
      q_.push_back(std::move(job));
    }
    cv_.notify_one();
  }
  // Runs what is queued to completion and stops the driver; returns its busy
  // milliseconds.
  double finish() {
    {
      std::lock_guard<std::mutex> g(mu_);
      done_ = true;
    }
    cv_.notify_one();
    if (th_.joinable()) th_.join();
    return busy_ms_;
  }

 private:
  void loop() {
    for (;;) {
      std::function<void(int)> job;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return done_ || !q_.empty(); });
        if (q_.empty()) return;
        job = std::move(q_.front());
        q_.pop_front();
      }
      const auto t0 = std::chrono::steady_clock::now();
      job(threads_);
      busy_ms_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
  }
  const int threads_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<std::function<void(int)>> q_;
  bool done_ = false;
  double busy_ms_ = 0;
  std::thread th_;  // last member: starts once the others exist
};

struct PairResult {
  bool hit = false;
  HitOut h;
};

// search.rs:131-210: thresholds, E-values, domain c-/i-E-values, reported flags.
int report(const sx_profiles* P, const sx_targets* T, const sx_search_cfg* cfg,
           std::vector<std::vector<std::pair<int32_t, HitOut>>>& per_profile, sx_hits* out) {
  const double z = std::max(std::isnan(cfg->z) ? (double)T->len.size() : cfg->z, 1.0);
  for (size_t pi = 0; pi < P->h.size(); pi++) {
    const ProfileHost& h = P->h[pi];
    bool is_e = false;
    double e_seq = 0, e_dom = 0;
    float t_seq = 0, t_dom = 0;
    switch (cfg->cutoff_kind) {
      case SX_CUT_EVALUE: is_e = true; e_seq = cfg->seq_threshold; e_dom = cfg->dom_threshold; break;
      case SX_CUT_BITS: t_seq = (float)cfg->seq_threshold; t_dom = (float)cfg->dom_threshold; break;
      case SX_CUT_GA: t_seq = h.ga[0]; t_dom = h.ga[1]; break;
      case SX_CUT_NC: t_seq = h.nc[0]; t_dom = h.nc[1]; break;
      case SX_CUT_TC: t_seq = h.tc[0]; t_dom = h.tc[1]; break;
    }
    auto& raws = per_profile[pi];
    std::sort(raws.begin(), raws.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    const size_t first_hit = out->hits.size();
    for (auto& [ti, r] : raws) {
      const double evalue = std::exp(r.lnp) * z;
      const bool keep = is_e ? (evalue <= e_seq) : (r.bits >= t_seq);
      if (!keep) continue;
      sx_hit hh{};
      hh.profile_index = (int32_t)pi;
      hh.target_index = ti;
      hh.qlen = h.m;
      hh.tlen = T->len[ti];
      hh.score = r.bits;
      hh.bias = r.bias;
      hh.evalue = evalue;
      hh.nexpected = r.nexpected;
      hh.ndomains = (int32_t)r.domains.size();
      hh.domain_offset = (int32_t)out->doms.size();
      for (const DomainOut& d : r.domains) {
        sx_domain dd{};
        dd.score = d.bits;
        dd.bias = d.bias;
        dd.c_evalue = NAN;
        dd.i_evalue = std::exp(d.lnp) * z;
        dd.hmm_from = (int32_t)d.kali; dd.hmm_to = (int32_t)d.mali;
        dd.ali_from = (int32_t)d.iali; dd.ali_to = (int32_t)d.jali;
        dd.env_from = (int32_t)d.ienv; dd.env_to = (int32_t)d.jenv;
        dd.reported = 0;
        out->doms.push_back(dd);
      }
      out->hits.push_back(hh);
    }
    const double dom_z = (double)std::max<size_t>(out->hits.size() - first_hit, 1);
    for (size_t q = first_hit; q < out->hits.size(); q++) {
      const sx_hit& hh = out->hits[q];
      for (int d = 0; d < hh.ndomains; d++) {
        sx_domain& dd = out->doms[hh.domain_offset + d];
        const double p_dom = dd.i_evalue / z;
        dd.c_evalue = p_dom * dom_z;
        dd.reported = is_e ? (dd.c_evalue <= e_dom) : (dd.score >= t_dom);
      }
    }
  }
  return SX_OK;
}

int check_cutoffs(const sx_profiles* P, int kind) {
  for (const ProfileHost& h : P->h) {
    if (kind == SX_CUT_GA && !h.has_ga) return fail(SX_ECUTOFF, "GA bit thresholds unavailable on model " + h.name);
    if (kind == SX_CUT_NC && !h.has_nc) return fail(SX_ECUTOFF, "NC bit thresholds unavailable on model " + h.name);
    if (kind == SX_CUT_TC && !h.has_tc) return fail(SX_ECUTOFF, "TC bit thresholds unavailable on model " + h.name);
  }
  if (kind < SX_CUT_EVALUE || kind > SX_CUT_TC) return fail(SX_EINVAL, "unknown cutoff kind " + std::to_string(kind));
  return SX_OK;
}

// MSV tiles: for every profile, slices of the length-sorted target order with
// roughly equal residue counts.
// MSV tiles of every (profile in [p0, p1), target) pair, grouped by kernel shape.
std::vector<std::vector<MsvTile>> make_all_pairs_tiles(const sx_engine* E, const sx_profiles* P, const sx_targets* T,
                                                       int p0, int p1) {
  std::vector<std::vector<MsvTile>> by_shape(kNumMsvShapes);
  const int nt = (int)T->len.size();
  if (nt == 0 || p1 <= p0) return by_shape;
  const int np = p1 - p0;
  const int waves = 16;
  int nslices = (int)std::ceil((double)waves * E->num_sms * 2 / std::max(1, np));
  nslices = std::max(1, std::min(nslices, std::max(1, nt / 32)));
  // slice boundaries with ~equal residues
  std::vector<int> cut(nslices + 1, nt);
  cut[0] = 0;
  {
    double acc = 0, per = T->residues / nslices;
    int s = 1;
    for (int q = 0; q < nt && s < nslices; q++) {
      acc += T->len[T->order[q]];
      if (acc >= per * s) cut[s++] = q + 1;
    }
  }
  std::vector<int> pord(np);
  std::iota(pord.begin(), pord.end(), p0);
  std::stable_sort(pord.begin(), pord.end(), [&](int a, int b) { return P->h[a].m > P->h[b].m; });
  for (int pi : pord)
    if (P->msv_shape[pi] >= 0)
      for (int s = 0; s < nslices; s++)
        if (cut[s + 1] > cut[s]) by_shape[P->msv_shape[pi]].push_back({pi, cut[s], cut[s + 1], 0});
  return by_shape;
}

// Shared memory of an MSV-shaped CTA (f32 image or interleaved packed image:
// both 16 bytes per chunk of 4 columns), one shifted copy per quarter-warp group.
size_t msv_smem(int s) {
  const int g = kMsvShapes[s].g, c = kMsvShapes[s].c;
  const int ncopy = g < 8 ? 8 / g : 1;
  const size_t rowp = ((size_t)(c / 4) * g + 7) & ~(size_t)7;
  return (size_t)ncopy * (25 * rowp + 8 + g) * sizeof(float4);
}

void launch_msv(sx_engine* E, Slot& S, Streams& X, const sx_profiles* P, const sx_targets* T, const std::vector<std::vector<MsvTile>>& tiles,
                const int32_t* d_list, float* d_scores, const int32_t* d_slot, PairRec* surv, const BinRegion* bins,
                unsigned* counts, const unsigned* rcount = nullptr, unsigned rcap = 0, int p0 = 0) {
  const auto& K = kernels();
  std::vector<MsvTile> all;
  std::vector<size_t> start(kNumMsvShapes + 1, 0);
  for (int s = 0; s < kNumMsvShapes; s++) {
    start[s] = all.size();
    all.insert(all.end(), tiles[s].begin(), tiles[s].end());
  }
  start[kNumMsvShapes] = all.size();
  if (all.empty()) return;
  S.tiles.upload(all.data(), all.size(), X.main);
  // biggest launches first, each on its own auxiliary stream
  std::vector<int> order;
  for (int s = 0; s < kNumMsvShapes; s++)
    if (start[s + 1] > start[s]) order.push_back(s);
  std::vector<double> work(kNumMsvShapes, 0.0);
  for (int s : order)
    for (size_t q = start[s]; q < start[s + 1]; q++) work[s] += (double)all[q].end - all[q].begin;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
  fork_aux(X);
  int lane = 0;
  for (int s : order) {
    const size_t nt = start[s + 1] - start[s];
    const size_t smem = msv_smem(s);
    CK(cudaFuncSetAttribute((const void*)K.msv[s], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    K.msv[s]<<<(unsigned)nt, 256, smem, X.aux[lane++ % X.naux]>>>(
        S.tiles.p + start[s], P->d_prof.p, E->thr.p, P->d_msv.p, T->d_res.p, T->d_off.p, T->d_len.p, T->d_tpar.p,
        d_list, d_scores, d_slot, surv, bins, counts, S.overflow.p, rcount, rcap, p0);
    E->stats.kernel_launches++;
  }
  CK(cudaGetLastError());
  join_aux(X);
}

// The block's pre-screened profiles: pairs of one MSV shape (similar M
// adjacent) as tiles over slices of the length-sorted targets, grouped by shape.
std::vector<std::vector<sxk::PackedTile>> make_packed_tiles(const sx_engine* E, const sx_profiles* P,
                                                            const sx_targets* T, const std::vector<int>& prof) {
  std::vector<std::vector<sxk::PackedTile>> by_shape(kNumMsvShapes);
  const int nt = (int)T->len.size();
  if (nt == 0 || prof.empty()) return by_shape;
  std::vector<std::vector<int>> group(kNumMsvShapes);
  for (int pi : prof) group[P->msv_shape[pi]].push_back(pi);
  std::vector<std::pair<int, int>> pairs;  // (pa, pb), pb = -1 for the odd one
  for (auto& g : group) {
    std::stable_sort(g.begin(), g.end(), [&](int a, int b) { return P->h[a].m > P->h[b].m; });
    for (size_t q = 0; q < g.size(); q += 2) pairs.emplace_back(g[q], q + 1 < g.size() ? g[q + 1] : -1);
  }
  const int np = (int)pairs.size();
  int nslices = (int)std::ceil(16.0 * E->num_sms * 2 / std::max(1, np));
  nslices = std::max(1, std::min(nslices, std::max(1, nt / 32)));
  std::vector<int> cut(nslices + 1, nt);
  cut[0] = 0;
  {
    double acc = 0, per = T->residues / nslices;
    int s = 1;
    for (int q = 0; q < nt && s < nslices; q++) {
      acc += T->len[T->order[q]];
      if (acc >= per * s) cut[s++] = q + 1;
    }
  }
  for (const auto& pr : pairs)
    for (int s = 0; s < nslices; s++)
      if (cut[s + 1] > cut[s]) by_shape[P->msv_shape[pr.first]].push_back({pr.first, pr.second, cut[s], cut[s + 1]});
  return by_shape;
}

// Packed pre-screen of a block (profiles `prof`, all with a quantized image):
// the pairs whose bound passes F1 land in the per-profile rescoring lists of
// slot S (region (p - p0) * rcap of S.rlist, counts in S.rcount).
void launch_prescreen(sx_engine* E, Slot& S, Streams& X, const sx_profiles* P, const sx_targets* T,
                      const std::vector<int>& prof, unsigned rcap, int p0) {
  const auto& K = kernels();
  auto tiles = make_packed_tiles(E, P, T, prof);
  std::vector<sxk::PackedTile> all;
  std::vector<size_t> start(kNumMsvShapes + 1, 0);
  for (int s = 0; s < kNumMsvShapes; s++) {
    start[s] = all.size();
    all.insert(all.end(), tiles[s].begin(), tiles[s].end());
  }
  start[kNumMsvShapes] = all.size();
  if (all.empty()) return;
  S.ptiles.upload(all.data(), all.size(), X.main);
  std::vector<int> order;
  std::vector<double> work(kNumMsvShapes, 0.0);
  for (int s = 0; s < kNumMsvShapes; s++)
    if (start[s + 1] > start[s]) {
      order.push_back(s);
      for (size_t q = start[s]; q < start[s + 1]; q++) work[s] += (double)all[q].end - all[q].begin;
    }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
  fork_aux(X);
  int lane = 0;
  for (int s : order) {
    const size_t smem = msv_smem(s);
    CK(cudaFuncSetAttribute((const void*)K.msv16[s], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    K.msv16[s]<<<(unsigned)(start[s + 1] - start[s]), 256, smem, X.aux[lane++ % X.naux]>>>(
        S.ptiles.p + start[s], P->d_prof.p, E->thr.p, P->d_qimg.p, T->d_res.p, T->d_off.p, T->d_len.p, T->d_tpar.p,
        T->d_order.p, S.rlist.p, rcap, S.rcount.p, p0, S.overflow.p, nullptr, nullptr, 0);
    E->stats.kernel_launches++;
  }
  CK(cudaGetLastError());
  join_aux(X);
}

// Exact MSV of the pre-screen's survivors: per profile `nsub` strided
// sub-tiles over its rescoring list; scores and F1 decisions as in a full
// MSV pass (survivors appended to the stage-0 lists).
void launch_rescore(sx_engine* E, Slot& S, Streams& X, const sx_profiles* P, const sx_targets* T,
                    const std::vector<int>& prof, unsigned rcap, int p0) {
  std::vector<std::vector<MsvTile>> tiles(kNumMsvShapes);
  const int nsub = std::max(2, std::min(32, (int)std::ceil(4.0 * E->num_sms / std::max<size_t>(1, prof.size()))));
  for (int pi : prof)
    for (int q = 0; q < nsub; q++) tiles[P->msv_shape[pi]].push_back({pi, q, nsub, 0});
  launch_msv(E, S, X, P, T, tiles, S.rlist.p, nullptr, nullptr, S.lists[0].p, S.bins[0].p, S.counts.p, S.rcount.p,
             rcap, p0);
}

// Per-profile lists of the packed Viterbi pre-screen: with `list` set, the
// bias filter hands the survivors of pre-screened profiles over in them.
struct VitScreen {
  PairRec* list = nullptr;
  unsigned cap = 0;
  unsigned* count = nullptr;
  int p0 = 0;
};

// One filter stage over per-vbin lists: stage `si` reads lists[si] and writes lists[si+1].
void launch_stage(sx_engine* E, Slot& S, const sx_profiles* P, const sx_targets* T, int si, const std::vector<unsigned>& nin,
                  const VitScreen& vs = VitScreen{}) {
  const auto& K = kernels();
  cudaStream_t s = S.hi.main;
  unsigned* cin = S.counts.p + si * kMaxBins;
  unsigned* cout = S.counts.p + (si + 1) * kMaxBins;
  if (si == 0) {
    unsigned mx = 0;
    for (int b = 0; b < kNumVbins; b++) mx = std::max(mx, nin[b]);
    if (!mx) return;
    dim3 grid((unsigned)std::min<int64_t>((mx + 255) / 256, (int64_t)E->num_sms * 8), kNumVbins);
    sxk::bias_kernel<<<grid, 256, 0, s>>>(S.lists[0].p, cin, S.bins[0].p, S.lists[1].p, S.bins[1].p, cout,
                                          S.overflow.p, P->d_bias.p, E->thr.p, T->d_res.p, T->d_off.p, T->d_len.p,
                                          kSlackBits, nullptr, P->d_prof.p, vs.list, vs.cap, vs.count, vs.p0);
    E->stats.kernel_launches++;
  } else {
    if (si == 1) {
      S.cursor.alloc(kMaxBins);
      CK(cudaMemsetAsync(S.cursor.p, 0, sizeof(unsigned) * kMaxBins, S.hi.main));
    }
    fork_aux(S.hi);
    int lane = 0;
    const int nb = si == 1 ? kNumVitShapes : kNumVbins;
    for (int b = 0; b < nb; b++) {
      if (!nin[b]) continue;
      cudaStream_t s = S.hi.aux[lane++ % S.hi.naux];
      if (si == 1 && (E->flags & SX_FLAG_PLAIN)) {
        sxk::plain_viterbi_kernel<<<(unsigned)std::min<int64_t>(nin[b], (int64_t)E->num_sms * 64), sxk::kPlainThreads,
                                    0, S.hi.main>>>(S.lists[1].p, cin, S.bins[1].p, b, S.lists[2].p, S.bins[2].p,
                                                    cout, S.overflow.p, P->d_pprof.p, P->d_plain.p, E->thr.p,
                                                    T->d_res.p, T->d_off.p, T->d_len.p, T->d_xsc.p, kSlackBits,
                                                    P->d_prof.p);
        E->stats.kernel_launches++;
        continue;
      }
      if (si == 1) {
        const int vblocks = vit_blocks(E->num_sms, b, nin[b]);
        K.vitg[b]<<<vblocks, 256, 0, s>>>(S.lists[1].p, cin, S.bins[1].p, b, S.lists[2].p, S.bins[2].p, cout,
                                          S.overflow.p, P->d_prof.p, E->thr.p, P->d_vit.p, T->d_res.p, T->d_off.p,
                                          T->d_len.p, T->d_xsc.p, kSlackBits, nullptr, S.cursor.p);
      } else
        K.fwd_scan[b]<<<warp_ctas(E->num_sms, nin[b]), 32, 0, s>>>(S.lists[2].p, cin, S.bins[2].p, b, S.lists[3].p,
                                                               S.bins[3].p, cout,
                                        S.overflow.p, P->d_prof.p, E->thr.p, P->d_vfb.p, T->d_res.p, T->d_off.p,
                                        T->d_len.p, T->d_xsc.p, kSlackBits, nullptr, nullptr);
      E->stats.kernel_launches++;
    }
    join_aux(S.hi);
  }
  CK(cudaGetLastError());
}

// Packed Viterbi pre-screen of a block's bias-filter survivors (profiles
// `prof`, per-profile lists in `vs`, `count[p - p0]` pairs in each): a
// profile's list is cut into strided sub-tiles of about twelve rounds of the
// pairs a CTA holds at once (fewer leave a CTA's slot idle behind its longest
// target too often), larger M first, one launch per shape on the
// slot's high-priority auxiliary streams; pairs whose bound passes F2 go to
// the Viterbi lists (lists[1]), S.vstats collects cells and passes.
void launch_vprescreen(sx_engine* E, Slot& S, const sx_profiles* P, const sx_targets* T, const std::vector<int>& prof,
                       const VitScreen& vs, const std::vector<unsigned>& count) {
  const auto& K = kernels();
  std::vector<std::vector<sxk::VitTile>> by_shape(kNumVit16Shapes);
  std::vector<int> order(prof);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return P->h[a].m > P->h[b].m; });
  for (int pi : order) {
    const unsigned n = std::min(count[pi - vs.p0], vs.cap);
    if (!n) continue;
    const Vit16Shape& v = kVit16Shapes[P->dp[pi].qv_shape];
    const unsigned per = 12u * (unsigned)(vit16_threads(v) / 32) * (unsigned)(32 / v.g) * 2u;  // pairs per sub-tile
    const int nsub = (int)std::min<unsigned>(256u, (n + per - 1) / per);
    for (int q = 0; q < nsub; q++) by_shape[P->dp[pi].qv_shape].push_back({pi, q, nsub, 0});
  }
  std::vector<sxk::VitTile> all;
  std::vector<size_t> start(kNumVit16Shapes + 1, 0);
  for (int s = 0; s < kNumVit16Shapes; s++) {
    start[s] = all.size();
    all.insert(all.end(), by_shape[s].begin(), by_shape[s].end());
  }
  start[kNumVit16Shapes] = all.size();
  if (all.empty()) return;
  S.vtiles.upload(all.data(), all.size(), S.hi.main);
  fork_aux(S.hi);
  int lane = 0;
  for (int s = kNumVit16Shapes - 1; s >= 0; s--) {  // widest first
    if (start[s + 1] == start[s]) continue;
    const int smem = vit16_smem(kVit16Shapes[s]);
    CK(cudaFuncSetAttribute((const void*)K.vit16[s], cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    K.vit16[s]<<<(unsigned)(start[s + 1] - start[s]), vit16_threads(kVit16Shapes[s]), smem,
                 S.hi.aux[lane++ % S.hi.naux]>>>(
        S.vtiles.p + start[s], P->d_prof.p, E->thr.p, P->d_qvimg.p, T->d_res.p, T->d_off.p, T->d_len.p, T->d_xsc.p,
        vs.list, vs.cap, vs.count, vs.p0, S.lists[1].p, S.bins[1].p, S.counts.p + kMaxBins, S.overflow.p, kSlackBits,
        nullptr, S.vstats.p);
    E->stats.kernel_launches++;
  }
  CK(cudaGetLastError());
  join_aux(S.hi);
}

double elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

// The device passes of a DomainBatch: for every envelope request the
// full-matrix Forward and Backward (their raw special rows come back to the
// host), the host's posterior factors, then the posterior / null2 /
// optimal-accuracy pass.  One warp per envelope; batches bounded by the
// memory of their matrix planes.  Runs on the host pool's driver thread.
// One batch's requests and the places for their results.
struct EnvSource {
  const DomainBatch* db;
  const std::vector<EnvRequest>* reqs;
  std::vector<EnvFactors>* F;
  std::vector<EnvDeviceOut>* D;
};

int64_t envelope_passes(sx_engine* E, const sx_profiles* P, const sx_targets* T, std::vector<EnvSource>& srcs,
                        int nthr, PhaseLog* plog = nullptr) {
  // every request of every batch, as (batch, request)
  std::vector<std::pair<uint32_t, uint32_t>> items;
  for (size_t b = 0; b < srcs.size(); b++) {
    const size_t nr = srcs[b].reqs->size();
    srcs[b].F->assign(nr, EnvFactors{});
    srcs[b].D->assign(nr, EnvDeviceOut{});
    for (size_t r = 0; r < nr; r++) items.emplace_back((uint32_t)b, (uint32_t)r);
  }
  const size_t nr = items.size();
  int64_t launches = 0;
  if (!nr) return 0;
  auto req = [&](size_t x) -> const EnvRequest& { return (*srcs[items[x].first].reqs)[items[x].second]; };
  auto fac_of = [&](size_t x) -> EnvFactors& { return (*srcs[items[x].first].F)[items[x].second]; };
  auto out_of = [&](size_t x) -> EnvDeviceOut& { return (*srcs[items[x].first].D)[items[x].second]; };
  const auto& K = kernels();
  cudaStream_t s = E->env_stream;
  // Planes of every envelope of a search at once when they fit: each batch
  // is one round of latency-bound passes (the longest envelope sets its
  // time) plus a host round trip, so fewer, larger batches finish sooner.
  const int64_t budget = scratch_budget(E, std::max<int64_t>(4 * E->batch_bytes, 256LL << 20));
  std::vector<size_t> order(nr);
  std::iota(order.begin(), order.end(), (size_t)0);
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t x, size_t y) { return P->dp[req(x).p].vbin < P->dp[req(y).p].vbin; });
  size_t a = 0;
  while (a < nr) {
    size_t b = a;
    int64_t planes = 0, rowsz = 0, aux = 0, fac = 0;
    std::vector<sxk::EnvRec> recs;
    while (b < nr) {
      const EnvRequest& q = req(order[b]);
      const int vc = kVcBins[P->dp[q.p].vbin];
      const int64_t lr = q.j - q.i + 1;
      const int64_t need = 5 * (lr + 1) * 32 * vc;
      if (b > a && (planes + need) * (int64_t)sizeof(float) > budget) break;
      sxk::EnvRec r{};
      r.p = q.p;
      r.t = q.t;
      r.i0 = (int32_t)(q.i - 1);
      r.lr = (int32_t)lr;
      r.ploop = q.st.ploop;
      r.pmove = q.st.pmove;
      r.pe_loop = q.st.pe_loop;
      r.pe_move = q.st.pe_move;
      r.plane_off = planes;
      r.row_off = rowsz;
      r.aux_off = aux;
      r.fac_off = fac;
      r.out_off = (int64_t)(b - a) * sxk::kEnvOut;
      planes += need;
      rowsz += 12 * (lr + 1);
      aux += 8 * (lr + 1);
      fac += lr + 1;
      recs.push_back(r);
      b++;
    }
    const size_t n = b - a;
    const auto tb0 = std::chrono::steady_clock::now();
    E->env_recs.upload(recs.data(), n, s);
    E->env_planes.alloc((size_t)planes);
    E->env_rows.alloc((size_t)rowsz);
    E->env_aux.alloc((size_t)aux);
    E->env_fac.alloc((size_t)fac);
    E->env_out.alloc(n * sxk::kEnvOut);
    // one launch per vbin: requests are sorted by vbin
    auto each_bin = [&](auto&& launch) {
      size_t x = 0;
      while (x < n) {
        const int vb = P->dp[req(order[a + x]).p].vbin;
        size_t y = x;
        while (y < n && P->dp[req(order[a + y]).p].vbin == vb) y++;
        const int cnt = (int)(y - x);
        launch(vb, (int)x, cnt, (int)std::min<int64_t>(cnt, (int64_t)E->num_sms * 32));
        x = y;
      }
    };
    // Forward on the envelope stream, Backward beside it on the second one
    CK(cudaEventRecord(E->env_ev, s));
    CK(cudaStreamWaitEvent(E->env_stream2, E->env_ev, 0));
    each_bin([&](int vb, int x0, int cnt, int blocks) {
      K.envf[vb]<<<blocks, 32, 0, s>>>(E->env_recs.p + x0, cnt, P->d_prof.p, P->d_vfb.p, T->d_res.p, T->d_off.p,
                                       E->env_planes.p, E->env_rows.p);
      K.envb[vb]<<<blocks, 32, 0, E->env_stream2>>>(E->env_recs.p + x0, cnt, P->d_prof.p, P->d_vfb.p, T->d_res.p,
                                                    T->d_off.p, E->env_planes.p, E->env_rows.p);
      launches += 2;
    });
    CK(cudaGetLastError());
    CK(cudaEventRecord(E->env_ev, E->env_stream2));
    CK(cudaStreamWaitEvent(s, E->env_ev, 0));
    std::vector<float> hrows((size_t)rowsz);
    CK(cudaMemcpyAsync(hrows.data(), E->env_rows.p, sizeof(float) * (size_t)rowsz, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (plog) plog->add("env_fb_pass", tb0);
    const auto tb1 = std::chrono::steady_clock::now();
    parallel_for(n, nthr, [&](size_t x) {
      const sxk::EnvRec& r = recs[x];
      const auto& it = items[order[a + x]];
      srcs[it.first].db->factors(it.second, hrows.data() + r.row_off,
                                 hrows.data() + r.row_off + 6 * ((int64_t)r.lr + 1), fac_of(order[a + x]));
    });
    std::vector<float> haux((size_t)aux, 0.0f);
    std::vector<double> hfac((size_t)fac, 0.0);
    for (size_t x = 0; x < n; x++) {
      const EnvFactors& f = fac_of(order[a + x]);
      if (!f.ok) continue;
      const sxk::EnvRec& r = recs[x];
      const size_t w = (size_t)r.lr + 1;
      std::copy(f.pn.begin(), f.pn.end(), haux.begin() + r.aux_off);
      std::copy(f.pj.begin(), f.pj.end(), haux.begin() + r.aux_off + w);
      std::copy(f.pc.begin(), f.pc.end(), haux.begin() + r.aux_off + 2 * w);
      std::copy(f.fac.begin(), f.fac.end(), hfac.begin() + r.fac_off);
    }
    if (plog) plog->add("env_factors_host", tb1);
    const auto tb2 = std::chrono::steady_clock::now();
    CK(cudaMemcpyAsync(E->env_aux.p, haux.data(), sizeof(float) * (size_t)aux, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(E->env_fac.p, hfac.data(), sizeof(double) * (size_t)fac, cudaMemcpyHostToDevice, s));
    each_bin([&](int vb, int x0, int cnt, int blocks) {
      const size_t psm = sxk::env_post_smem(kVcBins[vb]);
      CK(cudaFuncSetAttribute((const void*)K.envp[vb], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm));
      K.envp[vb]<<<blocks, 32, psm, s>>>(E->env_recs.p + x0, cnt, P->d_prof.p, P->d_vfb.p, E->env_planes.p,
                                       E->env_aux.p, E->env_fac.p, E->env_out.p);
      launches += 1;
    });
    CK(cudaGetLastError());
    std::vector<float> hout(n * sxk::kEnvOut);
    CK(cudaMemcpyAsync(hout.data(), E->env_out.p, sizeof(float) * hout.size(), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (plog) plog->add("env_post_pass", tb2);
    for (size_t x = 0; x < n; x++) {
      const float* o = hout.data() + x * sxk::kEnvOut;
      EnvDeviceOut& d = out_of(order[a + x]);
      for (int k = 0; k < NRES; k++) d.v[k] = o[k];
      d.si = o[20];
      d.found = o[21] != 0.0f;
      d.i0 = (int32_t)o[22];
      d.i1 = (int32_t)o[23];
      d.k0 = (int32_t)o[24];
      d.k1 = (int32_t)o[25];
    }
    a = b;
  }
  return launches;
}

// The device passes of the stochastic traces of multi-domain regions: the
// region's multihit Forward matrix (M, I and D planes in the diagonal
// layout), then one warp per region samples the trace ensemble and sums the
// per-position null2; the samples come back compacted into one pool.  The host finishes each region
// (logs, clustering) with DomainBatch::expand, and redoes on its own any
// region the device flagged.  Runs after the cascade, like envelope_passes.
struct RegionSource {
  DomainBatch* db;
  const std::vector<RegionRequest>* regs;
};
struct RegionPassStats {
  int64_t launches = 0, device = 0, redone = 0;
  double cells = 0;
};

RegionPassStats region_passes(sx_engine* E, const sx_profiles* P, const sx_targets* T,
                              std::vector<RegionSource>& srcs, int nthr) {
  RegionPassStats st;
  std::vector<std::pair<uint32_t, uint32_t>> items;
  for (size_t b = 0; b < srcs.size(); b++)
    for (size_t r = 0; r < srcs[b].regs->size(); r++) items.emplace_back((uint32_t)b, (uint32_t)r);
  const size_t nr = items.size();
  if (!nr) return st;
  auto reg = [&](size_t x) -> const RegionRequest& { return (*srcs[items[x].first].regs)[items[x].second]; };
  sxk::TraceConsts tc{};
  tc.lcg0 = DomainBatch::trace_lcg_start();
  for (int d = 0; d < 4; d++) {
    const Degenerate& g = degenerate(20 + d);
    tc.deg_n[d] = g.n;
    for (int q = 0; q < g.n; q++) tc.deg_m[d][q] = (int8_t)g.members[q];
  }
  const auto& K = kernels();
  cudaStream_t s = E->env_stream;
  // a batch is one latency-bound wave of 200-trace chains: keep the batches few
  const int64_t budget = scratch_budget(E, std::max<int64_t>(E->batch_bytes * 2, 1LL << 30));
  constexpr int64_t kPoolPerRegion = 1024;
  // column tables of the profiles that have regions (exact copies of the host's
  // probabilities and match odds), uploaded once
  std::unordered_map<int32_t, int64_t> col_of;
  std::vector<float> hcols;
  for (size_t x = 0; x < nr; x++) {
    const int32_t p = reg(x).p;
    if (col_of.count(p)) continue;
    const ProfileHost& h = P->h[p];
    col_of[p] = (int64_t)hcols.size();
    for (int k = 1; k <= h.m; k++) {
      const float c[8] = {h.p[TBM][k], h.p[TMM][k - 1], h.p[TIM][k - 1], h.p[TDM][k - 1],
                          h.p[TMI][k],  h.p[TII][k],     h.p[TMD][k - 1], h.p[TDD][k - 1]};
      hcols.insert(hcols.end(), c, c + 8);
      for (int x2 = 0; x2 < sxk::kTraceRes; x2++) hcols.push_back(h.mo_row(x2)[k]);
    }
  }
  E->trc_cols.upload(hcols.data(), hcols.size(), s);  // sampled domains per region, on average, before regions are redone
  std::vector<size_t> order(nr);
  std::iota(order.begin(), order.end(), (size_t)0);
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t x, size_t y) { return P->dp[reg(x).p].vbin < P->dp[reg(y).p].vbin; });
  size_t a = 0;
  while (a < nr) {
    size_t b = a;
    int64_t planes = 0, rowsz = 0, n2 = 0;
    std::vector<sxk::EnvRec> frecs;
    std::vector<sxk::TraceRec> trecs;
    while (b < nr) {
      const RegionRequest& g = reg(order[b]);
      const int64_t lr = g.j - g.i + 1;
      const int64_t need = 3 * sxk::diag_plane(lr, P->h[g.p].m);
      if (b > a && (planes + need) * (int64_t)sizeof(float) > budget) break;
      sxk::EnvRec f{};
      f.p = g.p;
      f.t = g.t;
      f.i0 = (int32_t)(g.i - 1);
      f.lr = (int32_t)lr;
      f.ploop = g.st.ploop;
      f.pmove = g.st.pmove;
      f.pe_loop = g.st.pe_loop;
      f.pe_move = g.st.pe_move;
      f.plane_off = planes;
      f.row_off = rowsz;
      sxk::TraceRec t{};
      t.m = P->h[g.p].m;
      t.t = f.t;
      t.i0 = f.i0;
      t.lr = f.lr;
      t.ploop = f.ploop;
      t.pmove = f.pmove;
      t.pe_loop = f.pe_loop;
      t.pe_move = f.pe_move;
      t.plane_off = planes;
      t.row_off = rowsz;
      t.n2_off = n2;
      t.col_off = col_of[g.p];
      planes += need;
      rowsz += 6 * (lr + 1);
      n2 += lr + 1;
      st.cells += (double)P->h[g.p].m * (double)lr;
      frecs.push_back(f);
      trecs.push_back(t);
      b++;
    }
    const size_t n = b - a;
    const int64_t pool_cap = std::min<int64_t>((int64_t)n * kPoolPerRegion, INT32_MAX / sxk::kTraceRecord);
    E->env_recs.upload(frecs.data(), n, s);
    E->trc_recs.upload(trecs.data(), n, s);
    E->env_planes.alloc((size_t)planes);
    E->env_rows.alloc((size_t)rowsz);
    E->env_aux.alloc((size_t)n2);
    E->trc_pool.alloc((size_t)pool_cap * sxk::kTraceRecord);
    E->trc_count.alloc(1);
    E->trc_status.alloc(n);
    CK(cudaMemsetAsync(E->trc_count.p, 0, sizeof(int32_t), s));
    // the region Forward passes, one launch per vbin (regions are sorted by
    // vbin), then one trace launch over the batch
    for (size_t x = 0; x < n;) {
      const int vb = P->dp[reg(order[a + x]).p].vbin;
      size_t y = x;
      while (y < n && P->dp[reg(order[a + y]).p].vbin == vb) y++;
      const int cnt = (int)(y - x);
      K.regf[vb]<<<(int)std::min<int64_t>(cnt, (int64_t)E->num_sms * 32), 32, 0, s>>>(
          E->env_recs.p + x, cnt, P->d_prof.p, P->d_vfb.p, T->d_res.p, T->d_off.p, E->env_planes.p, E->env_rows.p);
      st.launches += 1;
      x = y;
    }
    sxk::env_trace_kernel<<<(int)std::min<int64_t>(((int64_t)n + 3) / 4, (int64_t)E->num_sms * 16), 128, 0, s>>>(
        E->trc_recs.p, (int)n, E->trc_cols.p, T->d_res.p, T->d_off.p, E->env_planes.p, E->env_rows.p, E->env_aux.p,
        E->trc_pool.p, E->trc_count.p, (int32_t)pool_cap, 0, E->trc_status.p, tc);
    st.launches += 1;
    CK(cudaGetLastError());
    std::vector<float> hn2((size_t)n2);
    std::vector<int32_t> hstatus(n);
    int32_t count = 0;
    CK(cudaMemcpyAsync(hn2.data(), E->env_aux.p, sizeof(float) * (size_t)n2, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hstatus.data(), E->trc_status.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&count, E->trc_count.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const int64_t used = std::min<int64_t>(count, pool_cap);
    std::vector<int32_t> hpool((size_t)used * sxk::kTraceRecord);
    if (used > 0) {
      CK(cudaMemcpyAsync(hpool.data(), E->trc_pool.p, sizeof(int32_t) * hpool.size(), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
    }
    // samples per region, in pool order (a warp reserves each trace's block in
    // trace order, so pool order within a region is trace order)
    std::vector<std::vector<TraceSample>> per(n);
    for (int64_t q = 0; q < used; q++) {
      const int32_t* o = hpool.data() + q * sxk::kTraceRecord;
      if (o[0] < 0 || (size_t)o[0] >= n) continue;
      per[(size_t)o[0]].push_back({o[1], (int64_t)o[2], (int64_t)o[3], o[4], o[5]});
    }
    std::atomic<int64_t> redone{0};
    parallel_for(n, nthr, [&](size_t x) {
      const auto& it = items[order[a + x]];
      const bool ok = hstatus[x] == 0;
      if (!ok) redone++;
      srcs[it.first].db->expand(it.second, per[x], hn2.data() + trecs[x].n2_off, ok);
    });
    st.redone += redone.load();
    st.device += (int64_t)n - redone.load();
    a = b;
  }
  return st;
}

// ---- profiles longer than kMaxM ----------------------------------------------
// One CTA per pair; each CTA keeps kLongArrays rows of M+1 floats in scratch.
constexpr int kLongCtasPerSm = 8;

int long_grid(const sx_engine* E, size_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)n, (int64_t)E->num_sms * kLongCtasPerSm));
}
int64_t long_stride(const sx_profiles* P, const std::vector<sxk::LongPair>& v, size_t a, size_t b) {
  int m = 0;
  for (size_t i = a; i < b; i++) m = std::max(m, P->h[v[i].p].m);
  return (int64_t)sxk::kLongArrays * (m + 1);
}

// MSV (viterbi = false) or Viterbi scores of long-profile pairs.
void long_scores(sx_engine* E, const sx_profiles* P, const sx_targets* T, const std::vector<sxk::LongPair>& v,
                 bool viterbi, std::vector<float>& out) {
  out.assign(v.size(), kNegInf);
  if (v.empty()) return;
  cudaStream_t s = E->stream;
  const int grid = long_grid(E, v.size());
  const int64_t stride = long_stride(P, v, 0, v.size());
  E->long_pairs.upload(v.data(), v.size(), s);
  E->long_scratch.alloc((size_t)grid * (size_t)stride);
  E->long_out.alloc(v.size());
  if (viterbi)
    sxk::long_viterbi_kernel<<<grid, sxk::kPlainThreads, 0, s>>>(E->long_pairs.p, (int)v.size(), P->d_pprof.p,
                                                                P->d_plain.p, T->d_res.p, T->d_off.p, T->d_len.p,
                                                                T->d_xsc.p, E->long_scratch.p, stride, E->long_out.p);
  else
    sxk::long_msv_kernel<<<grid, sxk::kPlainThreads, 0, s>>>(E->long_pairs.p, (int)v.size(), P->d_pprof.p,
                                                            P->d_plain.p, P->d_prof.p, T->d_res.p, T->d_off.p,
                                                            T->d_len.p, T->d_tpar.p, E->long_scratch.p, stride,
                                                            E->long_out.p);
  CK(cudaGetLastError());
  E->stats.kernel_launches++;
  CK(cudaMemcpyAsync(out.data(), E->long_out.p, sizeof(float) * v.size(), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
}

// Raw Forward/Backward special rows of long-profile pairs, in chunks bounded
// by the scratch budget; consume(first, n, fwd, bwd, off) per chunk, pair
// first + q having its rows at fwd + off[q] and bwd + off[q].
template <typename F>
void long_rows(sx_engine* E, const sx_profiles* P, const sx_targets* T, const std::vector<sxk::LongPair>& v,
               F&& consume) {
  cudaStream_t s = E->stream;
  const int64_t budget = std::max<int64_t>(scratch_budget(E, E->batch_bytes / 2) / (int64_t)sizeof(float), 1 << 20);
  size_t i0 = 0;
  while (i0 < v.size()) {
    size_t i1 = i0;
    int64_t used = 0;
    std::vector<int64_t> off;
    while (i1 < v.size()) {
      const int64_t need = 6 * ((int64_t)T->len[v[i1].t] + 1);
      if (i1 > i0 && used + need > budget) break;
      off.push_back(used);
      used += need;
      i1++;
    }
    const size_t n = i1 - i0;
    const int grid = long_grid(E, n);
    const int64_t stride = long_stride(P, v, i0, i1);
    E->long_pairs.upload(v.data() + i0, n, s);
    E->long_row_off.upload(off.data(), n, s);
    E->long_scratch.alloc((size_t)grid * (size_t)stride);
    E->long_rows_f.alloc((size_t)used);
    E->long_rows_b.alloc((size_t)used);
    sxk::long_rows_kernel<<<grid, sxk::kPlainThreads, 0, s>>>(E->long_pairs.p, (int)n, P->d_pprof.p, P->d_plain.p,
                                                             T->d_res.p, T->d_off.p, T->d_len.p, T->d_xsc.p,
                                                             E->long_scratch.p, stride, E->long_rows_f.p,
                                                             E->long_rows_b.p, E->long_row_off.p);
    CK(cudaGetLastError());
    E->stats.kernel_launches++;
    std::vector<float> f((size_t)used), b((size_t)used);
    CK(cudaMemcpyAsync(f.data(), E->long_rows_f.p, sizeof(float) * (size_t)used, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(b.data(), E->long_rows_b.p, sizeof(float) * (size_t)used, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    consume(i0, n, f.data(), b.data(), off);
    i0 = i1;
  }
}

// Contiguous ranges of profile indices with about equal filtered DP cells.
// Each range runs through the device cascade as one block; the host domain
// definition of a block overlaps the device work of the blocks after it.
std::vector<std::pair<int, int>> profile_blocks(const sx_engine* E, const sx_profiles* P, const sx_targets* T,
                                                const std::vector<Thresholds>& th) {
  constexpr double kCellsPerBlock = 2.5e11;  // ~80 ms of B200 cascade
  constexpr int kMaxBlocks = 5;  // more blocks cost more than their shorter tail saves
  const int np = (int)P->h.size();
  std::vector<double> w(np, 0.0);
  double total = 0;
  int nfilt = 0;
  for (int pi = 0; pi < np; pi++)
    if (th[pi].exact) {
      w[pi] = (double)std::max(P->h[pi].m, 1) * std::max(T->residues, 1.0);
      total += w[pi];
      nfilt++;
    }
  std::vector<std::pair<int, int>> out;
  if (nfilt == 0 || T->len.empty()) return out;
  int nb = E->pipeline_blocks > 0 ? E->pipeline_blocks
                                  : (int)std::min<double>(kMaxBlocks, std::max(1.0, std::floor(total / kCellsPerBlock)));
  nb = std::max(1, std::min(nb, nfilt));
  // relative block sizes: the last two blocks of an automatic partition of
  // four or more are smaller (0.6 and 0.3 of the others), so the work left
  // after the last MSV stage -- that block's later device stages and its
  // domain definition on the host -- is short
  std::vector<double> rel(nb, 1.0);
  if (E->pipeline_blocks <= 0 && nb >= 4) {
    rel[nb - 2] = 0.6;
    rel[nb - 1] = 0.3;
  }
  std::vector<double> cum(nb + 1, 0.0);
  for (int b = 0; b < nb; b++) cum[b + 1] = cum[b] + rel[b];
  int p0 = 0;
  double acc = 0;
  for (int pi = 0; pi < np; pi++) {
    acc += w[pi];
    if ((int)out.size() < nb - 1 && acc >= total * cum[out.size() + 1] / cum[nb]) {
      out.emplace_back(p0, pi + 1);
      p0 = pi + 1;
    }
  }
  if (p0 < np) out.emplace_back(p0, np);
  return out;
}

// One block of filtered profiles [p0, p1) going through the device cascade.
struct BlockRun {
  int p0 = 0, p1 = 0;
  int attempt = 0;  // survivor-list sizing attempt; lists grow 4x per overflow
  std::vector<int> screened;  // profiles that go through the packed pre-screen
  unsigned rcap = 0;          // rescoring-list capacity per profile
  std::vector<int> vscreened;  // profiles whose bias survivors go through the packed Viterbi pre-screen
  StageLists L[4];
  std::vector<double> pairs_in_bin, pairs_in_vs;
  double cells_total = 0;
};
constexpr int kListAttempts = 4;

// Sizes the block's survivor lists, clears its counters and queues its MSV on
// slot S; returns without waiting for the device.
void cascade_launch(sx_engine* E, Slot& S, const sx_profiles* P, const sx_targets* T,
                    const std::vector<Thresholds>& th, BlockRun& R) {
  const size_t nt = T->len.size();
  cudaStream_t s = S.lo.main;
  if (R.attempt == 0) {  // capacity per bin from the number of pairs it holds
    R.pairs_in_bin.assign(kMaxBins, 0.0);
    R.pairs_in_vs.assign(kMaxBins, 0.0);
    R.cells_total = 0;
    for (int pi = R.p0; pi < R.p1; pi++)
      if (th[pi].exact && P->dp[pi].vbin >= 0) {
        R.pairs_in_bin[P->dp[pi].vbin] += (double)nt;
        R.pairs_in_vs[P->dp[pi].vshape] += (double)nt;
        R.cells_total += (double)P->h[pi].m * T->residues;
      }
  }
  // the last attempt sizes every list for all of its pairs and cannot overflow
  const bool full = R.attempt >= kListAttempts - 1;
  const double scale = std::pow(4.0, (double)R.attempt);
  std::vector<double> w1(kMaxBins), w1v(kMaxBins), w3(kMaxBins);
  for (int b = 0; b < kMaxBins; b++) {
    const double pb = R.pairs_in_bin[b], pv = R.pairs_in_vs[b];
    w1[b] = full ? pb : std::min(pb, scale * (0.06 * pb + 8192));
    w1v[b] = full ? pv : std::min(pv, scale * (0.06 * pv + 8192));
    w3[b] = full ? pb : std::min(pb, scale * (0.01 * pb + 4096));
  }
  R.L[0] = make_regions(w1);
  R.L[1] = make_regions(w1v);
  R.L[2] = make_regions(w3);
  R.L[3] = make_regions(w3);
  for (int q = 0; q < 4; q++) {
    S.lists[q].alloc((size_t)R.L[q].total);
    S.bins[q].upload(R.L[q].reg.data(), kMaxBins, s);
  }
  CK(cudaMemsetAsync(S.counts.p, 0, sizeof(unsigned) * 4 * kMaxBins, s));
  CK(cudaMemsetAsync(S.overflow.p, 0, sizeof(unsigned), s));
  S.cells.alloc(4);
  CK(cudaMemsetAsync(S.cells.p, 0, sizeof(double) * 4, s));
  // stage 0: MSV over all pairs of the block's filtered profiles
  CK(cudaEventRecord(S.ev[0], s));
  if (E->flags & SX_FLAG_PLAIN) {
    const int64_t last = (int64_t)R.p1 * (int64_t)nt;
    for (int64_t first = (int64_t)R.p0 * (int64_t)nt; first < last; first += (1LL << 30)) {
      const int64_t n = std::min<int64_t>(last - first, 1LL << 30);
      sxk::plain_msv_kernel<<<(unsigned)n, sxk::kPlainThreads, 0, s>>>(
          first, (int)nt, P->d_pprof.p, P->d_plain.p, P->d_prof.p, E->thr.p, T->d_res.p, T->d_off.p, T->d_len.p,
          T->d_tpar.p, S.lists[0].p, S.bins[0].p, S.counts.p, S.overflow.p);
      E->stats.kernel_launches++;
    }
    CK(cudaGetLastError());
  } else {
    // Profiles with a quantized image go through the packed pre-screen, then
    // the exact MSV of its survivors; the others straight through the exact
    // kernel.  Either way the stage-0 lists receive exactly the pairs whose
    // f32 MSV score passes F1.
    R.screened.clear();
    if (!(E->flags & SX_FLAG_NO_PRESCREEN) && nt > 0)
      for (int pi = R.p0; pi < R.p1; pi++)
        if (th[pi].exact && P->dp[pi].q_off >= 0) R.screened.push_back(pi);
    R.rcap = (unsigned)(full ? nt : std::min<double>((double)nt, scale * (0.05 * (double)nt + 1024)));
    if ((int64_t)(R.p1 - R.p0) * (int64_t)R.rcap >= (int64_t)INT32_MAX) R.screened.clear();
    std::vector<char> scr(R.p1 - R.p0, 0);
    for (int pi : R.screened) scr[pi - R.p0] = 1;
    auto tiles = make_all_pairs_tiles(E, P, T, R.p0, R.p1);
    for (auto& v : tiles)
      v.erase(std::remove_if(v.begin(), v.end(),
                             [&](const MsvTile& t) { return !th[t.p].exact || scr[t.p - R.p0]; }),
              v.end());
    launch_msv(E, S, S.lo, P, T, tiles, T->d_order.p, nullptr, nullptr, S.lists[0].p, S.bins[0].p, S.counts.p);
    if (!R.screened.empty()) {
      S.rlist.alloc((size_t)(R.p1 - R.p0) * R.rcap);
      S.rcount.alloc((size_t)(R.p1 - R.p0));
      CK(cudaMemsetAsync(S.rcount.p, 0, sizeof(unsigned) * (R.p1 - R.p0), s));
      launch_prescreen(E, S, S.lo, P, T, R.screened, R.rcap, R.p0);
      CK(cudaEventRecord(S.pre_done, s));
      launch_rescore(E, S, S.lo, P, T, R.screened, R.rcap, R.p0);
    }
    // Viterbi pre-screen: every MSV-pre-screened profile with a quantized
    // Viterbi image; its bias survivors (at most its rescoring list) go to
    // per-profile lists of the same capacity
    R.vscreened.clear();
    for (int pi : R.screened)
      if (P->dp[pi].qv_shape >= 0) R.vscreened.push_back(pi);
    if (!R.vscreened.empty()) {
      S.vlist.alloc((size_t)(R.p1 - R.p0) * R.rcap);
      S.vcount.alloc((size_t)(R.p1 - R.p0));
      S.vstats.alloc(3);
      CK(cudaMemsetAsync(S.vcount.p, 0, sizeof(unsigned) * (R.p1 - R.p0), s));
      CK(cudaMemsetAsync(S.vstats.p, 0, sizeof(double) * 3, s));
    }
  }
  CK(cudaEventRecord(S.ev[1], s));
  CK(cudaEventRecord(S.msv_done, s));
}

// Drives the block's bias, Viterbi and Forward pre-screen stages on slot S,
// then gathers the survivors and re-checks them exactly on the host, appending
// the pairs that pass to `finals`.  Returns false if a survivor list
// overflowed; the caller then relaunches the block (with larger lists).
bool cascade_finish(sx_engine* E, Slot& S, const sx_profiles* P, const sx_targets* T,
                    const std::vector<Thresholds>& th, const SearchOpts& o, BlockRun& R,
                    std::vector<FinalPair>& finals) {
  cudaStream_t s = S.hi.main;
  CK(cudaStreamWaitEvent(s, S.msv_done, 0));
  std::vector<unsigned> cnt(4 * kMaxBins);
  for (int si = 0; si < 3; si++) {
    CK(cudaMemcpyAsync(cnt.data(), S.counts.p, sizeof(unsigned) * 4 * kMaxBins, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    std::vector<unsigned> nin(kMaxBins);
    for (int b = 0; b < kMaxBins; b++) nin[b] = std::min(cnt[si * kMaxBins + b], R.L[si].reg[b].cap);
    CK(cudaEventRecord(S.ev[2 + si], s));
    if (si == 0 && !R.vscreened.empty()) {
      const VitScreen vs{S.vlist.p, R.rcap, S.vcount.p, R.p0};
      launch_stage(E, S, P, T, si, nin, vs);
      CK(cudaEventRecord(S.bias_done, s));
      std::vector<unsigned> vc((size_t)(R.p1 - R.p0));
      CK(cudaMemcpyAsync(vc.data(), S.vcount.p, sizeof(unsigned) * vc.size(), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      launch_vprescreen(E, S, P, T, R.vscreened, vs, vc);
      CK(cudaEventRecord(S.vpre_done, s));
      continue;
    }
    launch_stage(E, S, P, T, si, nin);
    if (si >= 1) {  // cells entering Viterbi (si = 1) and the Forward pre-screen (si = 2), for the stats
      unsigned mx = 0;
      for (int b = 0; b < kMaxBins; b++) mx = std::max(mx, nin[b]);
      if (mx) {
        dim3 grid((unsigned)std::min<int64_t>((mx + 255) / 256, (int64_t)E->num_sms * 4), kMaxBins);
        sxk::stage_cells_kernel<<<grid, 256, 0, S.hi.aux[0]>>>(S.lists[si].p, S.counts.p + si * kMaxBins,
                                                                S.bins[si].p, P->d_prof.p, T->d_len.p,
                                                                S.cells.p + si);
        E->stats.kernel_launches++;
      }
    }
  }
  CK(cudaEventRecord(S.ev[5], s));
  unsigned ovf = 0;
  double scells[4] = {0, 0, 0, 0};
  join_aux(S.hi);  // the cell counts run on an auxiliary stream
  CK(cudaMemcpyAsync(cnt.data(), S.counts.p, sizeof(unsigned) * 4 * kMaxBins, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&ovf, S.overflow.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(scells, S.cells.p, sizeof(double) * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (ovf && R.attempt < kListAttempts - 1) {  // a survivor list was too small
    R.attempt++;
    return false;
  }
  // stats
  double pairs_all = 0;
  for (int b = 0; b < kMaxBins; b++) pairs_all += R.pairs_in_bin[b];
  E->stats.pairs_in[0] += (int64_t)pairs_all;
  E->stats.cells[0] += R.cells_total;
  // Viterbi pre-screen: its input are bias survivors, its passes part of
  // the exact Viterbi's input
  int64_t v_in = 0, v_pass = 0;
  double v_stats[3] = {0, 0, 0};
  if (!R.vscreened.empty()) {
    std::vector<unsigned> vc((size_t)(R.p1 - R.p0));
    CK(cudaMemcpyAsync(vc.data(), S.vcount.p, sizeof(unsigned) * vc.size(), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(v_stats, S.vstats.p, sizeof(double) * 3, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int pi : R.vscreened) v_in += std::min(vc[pi - R.p0], R.rcap);
    v_pass = (int64_t)v_stats[2];
    E->stats.vprescreen_pairs_in += v_in;
    E->stats.vprescreen_pairs_out += v_pass;
    E->stats.vprescreen_cells += v_stats[0];
    E->stats.vprescreen_ms += elapsed_ms(S.bias_done, S.vpre_done);
  }
  for (int si = 0; si < 4; si++) {
    int64_t c = 0;
    for (int b = 0; b < kMaxBins; b++) c += cnt[si * kMaxBins + b];
    if (si == 1) c += v_in - v_pass;  // bias survivors: the pre-screen's input in place of its passes
    E->stats.pairs_out[si] += c;
    if (si < 3) E->stats.pairs_in[si + 1] += c;
  }
  // cells entering Viterbi: the exact kernel's input, with the pre-screen's
  // passes replaced by all the pairs it bounded
  E->stats.cells[2] += scells[1] - v_stats[1] + v_stats[0];
  E->stats.cells[3] += scells[2];
  E->stats.ms[0] += elapsed_ms(S.ev[0], S.ev[1]);
  if (!R.screened.empty()) {
    std::vector<unsigned> rc((size_t)(R.p1 - R.p0));
    CK(cudaMemcpyAsync(rc.data(), S.rcount.p, sizeof(unsigned) * rc.size(), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    double cells = 0;
    for (int pi : R.screened) {
      E->stats.prescreen_pairs_out += std::min(rc[pi - R.p0], R.rcap);
      cells += (double)P->h[pi].m;
    }
    E->stats.prescreen_pairs_in += (int64_t)R.screened.size() * (int64_t)T->len.size();
    E->stats.prescreen_cells += cells * T->residues;
    E->stats.prescreen_ms += elapsed_ms(S.ev[0], S.pre_done);
    E->stats.rescore_ms += elapsed_ms(S.pre_done, S.ev[1]);
  }
  E->stats.ms[1] += elapsed_ms(S.ev[2], R.vscreened.empty() ? S.ev[3] : S.bias_done);
  E->stats.ms[2] += elapsed_ms(S.ev[3], S.ev[4]);
  if (!R.vscreened.empty()) E->stats.ms[2] += elapsed_ms(S.bias_done, S.vpre_done);
  E->stats.ms[3] += elapsed_ms(S.ev[4], S.ev[5]);
  // gather stage-3 survivors
  std::vector<PairRec> surv;
  for (int b = 0; b < kNumVbins; b++) {
    const unsigned n = std::min(cnt[3 * kMaxBins + b], R.L[3].reg[b].cap);
    if (!n) continue;
    const size_t o0 = surv.size();
    surv.resize(o0 + n);
    CK(cudaMemcpyAsync(surv.data() + o0, S.lists[3].p + R.L[3].reg[b].off, sizeof(PairRec) * n,
                       cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  // exact host re-check of F1 / bias / F2 with the reference's libm
  std::vector<char> keep(surv.size(), 0);
  parallel_for(surv.size(), E->host_threads, [&](size_t i) {
    PairRec& r = surv[i];
    const ProfileHost& h = P->h[r.p];
    const uint8_t* d = T->dsq.data() + T->off[r.t];
    const int64_t l = T->len[r.t];
    const float nullsc = null1_score(l);
    if (gumbel_survival((double)((r.usc - nullsc) / kLn2f), h.msv[0], h.msv[1]) > o.f1) return;
    const float fsc = composition_bias_score(h, d, l);
    r.filtersc = fsc;
    if (gumbel_survival((double)((r.usc - fsc) / kLn2f), h.msv[0], h.msv[1]) > o.f1) return;
    if (gumbel_survival((double)((r.vsc - fsc) / kLn2f), h.vit[0], h.vit[1]) > o.f2) return;
    keep[i] = 1;
  });
  for (size_t i = 0; i < surv.size(); i++)
    if (keep[i]) finals.push_back({surv[i].p, surv[i].t, surv[i].usc, surv[i].filtersc, surv[i].vsc, -1});
  return true;
}

int run_search(sx_engine* E, const sx_profiles* P, const sx_targets* T, const sx_search_cfg* cfg, sx_hits* out) {
  int rc = check_cutoffs(P, cfg->cutoff_kind);
  if (rc) return rc;
  E->stats = sx_search_stats{};
  SearchOpts o;
  o.filters = cfg->filters != 0;
  o.null2 = cfg->null2 != 0;
  o.f1 = cfg->f1;
  o.f2 = cfg->f2;
  o.f3 = cfg->f3;
  const size_t np = P->h.size(), nt = T->len.size();
  cudaStream_t s = E->stream;
  std::vector<Thresholds> th = make_thresholds(P->h, o);
  // profiles longer than kMaxM take the long pass instead of the cascade
  std::vector<int> longs;
  std::vector<char> long_exact(np, 0);
  for (size_t pi = 0; pi < np; pi++)
    if (is_long(P->h[pi].m)) {
      longs.push_back((int)pi);
      long_exact[pi] = (char)th[pi].exact;
      th[pi].exact = 0;
    }
  E->thr.upload(th.data(), th.size(), s);
  for (Slot& S : E->sl) {
    S.overflow.alloc(1);
    S.counts.alloc(4 * kMaxBins);
  }
  const auto t_start = std::chrono::steady_clock::now();

  // Profiles searched with filters go through the cascade in blocks; those
  // without (uncalibrated, or --max) send every target straight to
  // Forward/Backward as a last block.
  struct BlockOut {
    std::vector<FinalPair> finals;
    std::vector<PairResult> res;
  };
  std::vector<std::unique_ptr<BlockOut>> outs;
  std::atomic<int64_t> n_domain{0};
  double rows_ms = 0;
  // errors raised on the host pool's thread, reported after it is joined
  std::mutex host_err_mu;
  int host_err_code = 0;
  std::string host_err_msg;
  std::atomic<int64_t> n_env{0}, env_launches{0};
  // batches whose host phase is done; their envelope passes run after the cascade
  struct PendingBatch {
    BlockOut* B;
    std::vector<size_t> which;
    std::vector<char> begun;
    std::unique_ptr<DomainBatch> db;
    std::vector<EnvRequest> reqs;
    std::vector<EnvFactors> F;
    std::vector<EnvDeviceOut> D;
    bool dev_regions = false;  // its multi-domain regions wait for the device trace passes
  };
  std::vector<std::unique_ptr<PendingBatch>> pending;  // appended by the pool's driver thread only
  HostQueue hq(E->host_threads);  // declared after what its jobs use, so it is joined first
  // device rows of a block's final pairs; their domain definition is queued
  // and runs while the engine thread moves on to the next block
  // Domain definition of a block runs on the host pool, hidden behind the
  // device work of later blocks, while that host work stays well below the
  // block's device time; past that (hit-heavy blocks) the envelopes' full-
  // matrix passes go to the device.  Host: ~44 ns per DP cell of the final
  // pairs per thread; device cascade ~4.4e12 cells/s (B200, Pfam-scale).
  auto device_envelopes = [&](const BlockOut* B, double block_cells) {
    if (E->flags & SX_FLAG_ENV_DEVICE) return true;
    if (E->flags & SX_FLAG_ENV_HOST) return false;
    double fin = 0;
    for (const auto& f : B->finals) fin += (double)P->h[f.p].m * (double)T->len[f.t];
    const double host_ms = fin * 44e-9 * 1e3 / std::max(1, E->host_threads);
    const double dev_ms = block_cells / 4.4e12 * 1e3;
    return host_ms > 0.5 * dev_ms + 5.0;
  };
  // Stochastic traces of a block's multi-domain regions: on the host pool at
  // once (hidden behind later device work) unless their estimated host time
  // exceeds the device trace pass.  Host: ~19 ns per DP cell of a region's
  // Forward matrix, traces included, per thread.  Device: one warp per region
  // runs its 200 traces as one dependent chain of ~200 (L + M) steps at
  // ~0.75 us each (B200), so a pass lasts about one chain per wave of
  // concurrent regions (20 per SM), plus ~30 ms of copies and host clustering.
  auto device_traces = [&](const std::vector<RegionRequest>& regs, int nthr) {
    if (E->flags & SX_FLAG_TRACE_DEVICE) return true;
    if (E->flags & SX_FLAG_TRACE_HOST) return false;
    double cells = 0, chain = 0;
    for (const RegionRequest& g : regs) {
      const double lr = (double)(g.j - g.i + 1), m = (double)P->h[g.p].m;
      cells += m * lr;
      chain = std::max(chain, 200.0 * (lr + m) * 0.75e-3);
    }
    const double waves = std::ceil((double)regs.size() / (20.0 * E->num_sms));
    return cells * 19e-6 / std::max(1, nthr) > 30.0 + waves * chain;
  };
  std::mutex rows_ms_mu;
  auto rows_and_queue = [&](Slot& S, BlockOut* B, bool dev_env) {
    B->res.resize(B->finals.size());
    // the host job of one chunk of rows: `get` hands it the rows (at once, or
    // after waiting for the asynchronous row passes)
    auto queue_chunk = [&, B, dev_env](std::function<RowsChunk()> get) {
      hq.push([&, B, dev_env, get](int nthr) {
        try {
          auto ch = std::make_shared<RowsChunk>(get());
          const size_t nq = ch->which.size();
          // largest pairs first, for an even finish across the workers
          std::vector<size_t> ord(nq);
          std::iota(ord.begin(), ord.end(), (size_t)0);
          auto cost = [&](size_t q) {
            const FinalPair& f = B->finals[ch->which[q]];
            return (double)P->h[f.p].m * (double)T->len[f.t];
          };
          std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return cost(a) > cost(b); });
          if (!dev_env) {  // F3 and the whole domain definition on the host (pipeline.rs:179-293)
            parallel_for(ord.size(), nthr, [&](size_t rr) {
              const size_t q = ord[rr];
              const size_t i = ch->which[q];
              const FinalPair& f = B->finals[i];
              const ProfileHost& h = P->h[f.p];
              const int64_t l = T->len[f.t];
              const float* fr = ch->f.data() + ch->off[q];
              const float* br = ch->b.data() + ch->off[q];
              const float fwdsc = forward_score_from_rows(h, l, fr);
              if (th[f.p].exact &&
                  std::exp(exp_tail_logsurv((double)((fwdsc - f.filtersc) / kLn2f), h.fwd[0], h.fwd[1])) > o.f3)
                return;
              n_domain++;
              B->res[i].hit = define_domains(h, T->dsq.data() + T->off[f.t], l, RawRows{fr, br}, fwdsc, o, B->res[i].h);
            });
            return;
          }
          // F3 (pipeline.rs:179-183), posterior decoding and regions on the
          // host; the stochastic traces of multi-domain regions and the
          // envelopes' full-matrix passes wait until the cascade is done
          auto pb = std::make_unique<PendingBatch>();
          pb->B = B;
          pb->which = ch->which;
          pb->begun.assign(nq, 0);
          pb->db = std::make_unique<DomainBatch>(o, nq);
          DomainBatch& db = *pb->db;
          std::vector<char>& begun = pb->begun;
          parallel_for(ord.size(), nthr, [&](size_t rr) {
            const size_t q = ord[rr];
            const FinalPair& f = B->finals[ch->which[q]];
            const ProfileHost& h = P->h[f.p];
            const int64_t l = T->len[f.t];
            const float* fr = ch->f.data() + ch->off[q];
            const float* br = ch->b.data() + ch->off[q];
            const float fwdsc = forward_score_from_rows(h, l, fr);
            if (th[f.p].exact &&
                std::exp(exp_tail_logsurv((double)((fwdsc - f.filtersc) / kLn2f), h.fwd[0], h.fwd[1])) > o.f3)
              return;
            n_domain++;
            db.begin(q, h, f.p, T->dsq.data() + T->off[f.t], l, f.t, RawRows{fr, br}, fwdsc, true);
            begun[q] = 1;
          });
          const std::vector<RegionRequest>& regs = db.regions();
          pb->dev_regions = !regs.empty() && device_traces(regs, nthr);
          if (!regs.empty() && !pb->dev_regions)
            parallel_for(regs.size(), nthr, [&](size_t r) { db.expand(r, {}, nullptr, false); });
          pending.push_back(std::move(pb));
        } catch (const CudaError& ce) {
          std::lock_guard<std::mutex> g(host_err_mu);
          if (!host_err_code) {
            host_err_code = ce.code;
            host_err_msg = ce.msg;
          }
        } catch (const std::bad_alloc&) {
          std::lock_guard<std::mutex> g(host_err_mu);
          if (!host_err_code) {
            host_err_code = SX_ENOMEM;
            host_err_msg = "sx_search: host allocation failed during domain definition";
          }
        }
      });
    };
    auto fetch = rows_pass_async(E, S, P, T, B->finals, &rows_ms_mu, &rows_ms);
    if (fetch) {
      queue_chunk(std::move(fetch));
      return;
    }
    // rows larger than one chunk: passes in turn, each chunk queued as it arrives
    const auto t0 = std::chrono::steady_clock::now();
    rows_pass(E, S, P, T, B->finals, [&](RowsChunk&& c) {
      auto ch = std::make_shared<RowsChunk>(std::move(c));
      queue_chunk([ch]() { return std::move(*ch); });
    });
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::lock_guard<std::mutex> g(rows_ms_mu);
    rows_ms += ms;
  };

  std::vector<int> unfiltered;
  for (size_t pi = 0; pi < np; pi++)
    if (!th[pi].exact && !is_long(P->h[pi].m)) unfiltered.push_back((int)pi);
  int64_t nfinal = 0;
  // software pipeline over two slots: block b+1's MSV is queued on the device
  // before block b's later stages are driven, so it fills the GPU around
  // their latency-bound tails and around block b's row passes
  const auto pb = profile_blocks(E, P, T, th);
  std::vector<BlockRun> runs(pb.size());
  for (size_t b = 0; b < pb.size(); b++) {
    runs[b].p0 = pb[b].first;
    runs[b].p1 = pb[b].second;
  }
  if (!runs.empty()) {
    // other slots' kernels read the thresholds uploaded on slot 0's stream
    CK(cudaStreamSynchronize(s));
    cascade_launch(E, E->sl[0], P, T, th, runs[0]);
  }
  for (size_t b = 0; b < runs.size(); b++) {
    Slot& S = E->sl[b % 2];
    if (b + 1 < runs.size()) cascade_launch(E, E->sl[(b + 1) % 2], P, T, th, runs[b + 1]);
    outs.push_back(std::make_unique<BlockOut>());
    BlockOut* B = outs.back().get();
    while (!cascade_finish(E, S, P, T, th, o, runs[b], B->finals)) cascade_launch(E, S, P, T, th, runs[b]);
    nfinal += (int64_t)B->finals.size();
    rows_and_queue(S, B, device_envelopes(B, runs[b].cells_total));
  }
  if (!unfiltered.empty() && nt > 0) {
    outs.push_back(std::make_unique<BlockOut>());
    BlockOut* B = outs.back().get();
    for (int pi : unfiltered)
      for (size_t t = 0; t < nt; t++) B->finals.push_back({pi, (int32_t)t, 0.f, 0.f, 0.f, -1});
    nfinal += (int64_t)B->finals.size();
    rows_and_queue(E->sl[0], B, !(E->flags & SX_FLAG_ENV_HOST));  // every pair reaches domain definition
  }
  const auto t_dev = std::chrono::steady_clock::now();
  PhaseLog plog;
  plog.add("cascade_and_rows", t_start);
  E->stats.ms[5] = hq.finish();
  plog.add("host_pool_drain", t_dev);
  if (host_err_code) return fail(host_err_code, host_err_msg);
  // every multi-domain region's trace ensemble, then every envelope of the
  // search through the device passes at once, on an idle GPU, then each
  // pair's scores
  RegionPassStats rstats;
  {
    const auto t_env = std::chrono::steady_clock::now();
    std::vector<RegionSource> rsrc;
    for (auto& pb : pending)
      if (pb->dev_regions) rsrc.push_back({pb->db.get(), &pb->db->regions()});
    rstats = region_passes(E, P, T, rsrc, E->host_threads);
    plog.add("region_passes", t_env);
    env_launches += rstats.launches;
    for (auto& pb : pending) {
      pb->reqs = pb->db->requests();
      n_env += (int64_t)pb->reqs.size();
    }
    std::vector<EnvSource> srcs;
    for (auto& pb : pending) srcs.push_back({pb->db.get(), &pb->reqs, &pb->F, &pb->D});
    const auto t_ep = std::chrono::steady_clock::now();
    env_launches += envelope_passes(E, P, T, srcs, E->host_threads, &plog);
    plog.add("envelope_passes", t_ep);
    const auto t_fin = std::chrono::steady_clock::now();
    std::vector<std::pair<PendingBatch*, size_t>> todo;
    for (auto& pb : pending)
      for (size_t q = 0; q < pb->which.size(); q++)
        if (pb->begun[q]) todo.emplace_back(pb.get(), q);
    parallel_for(todo.size(), E->host_threads, [&](size_t x) {
      PendingBatch& pb = *todo[x].first;
      const size_t q = todo[x].second;
      const size_t i = pb.which[q];
      pb.B->res[i].hit = pb.db->finish(q, pb.F, pb.D, pb.B->res[i].h);
    });
    plog.add("finish", t_fin);
    E->stats.ms[5] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_env).count();
  }
  // profiles longer than kMaxM: MSV on the device, the exact host checks of the
  // F1 / bias / F2 filters on its scores (those cascade_finish re-runs), the
  // Viterbi scores of the survivors, then the rows of the final pairs, F3 and
  // domain definition on the host pool
  if (!longs.empty() && nt > 0) {
    outs.push_back(std::make_unique<BlockOut>());
    BlockOut* B = outs.back().get();
    std::vector<sxk::LongPair> filt;
    for (int pi : longs)
      for (size_t t = 0; t < nt; t++) {
        if (long_exact[pi]) filt.push_back({pi, (int32_t)t});
        else B->finals.push_back({pi, (int32_t)t, 0.f, 0.f, 0.f, -1});
      }
    std::vector<float> usc, vsc, fsc(filt.size(), 0.f);
    long_scores(E, P, T, filt, false, usc);
    std::vector<char> pass1(filt.size(), 0);
    parallel_for(filt.size(), E->host_threads, [&](size_t i) {
      const ProfileHost& h = P->h[filt[i].p];
      const int64_t l = T->len[filt[i].t];
      const float nullsc = null1_score(l);
      if (gumbel_survival((double)((usc[i] - nullsc) / kLn2f), h.msv[0], h.msv[1]) > o.f1) return;
      fsc[i] = composition_bias_score(h, T->dsq.data() + T->off[filt[i].t], l);
      if (gumbel_survival((double)((usc[i] - fsc[i]) / kLn2f), h.msv[0], h.msv[1]) > o.f1) return;
      pass1[i] = 1;
    });
    std::vector<sxk::LongPair> surv;
    std::vector<size_t> from;
    for (size_t i = 0; i < filt.size(); i++)
      if (pass1[i]) {
        surv.push_back(filt[i]);
        from.push_back(i);
      }
    long_scores(E, P, T, surv, true, vsc);
    for (size_t q = 0; q < surv.size(); q++) {
      const size_t i = from[q];
      const ProfileHost& h = P->h[surv[q].p];
      if (gumbel_survival((double)((vsc[q] - fsc[i]) / kLn2f), h.vit[0], h.vit[1]) > o.f2) continue;
      B->finals.push_back({surv[q].p, surv[q].t, usc[i], fsc[i], vsc[q], -1});
    }
    for (const sxk::LongPair& q : filt) {
      E->stats.pairs_in[0]++;
      E->stats.cells[0] += (double)P->h[q.p].m * (double)T->len[q.t];
    }
    B->res.resize(B->finals.size());
    std::vector<sxk::LongPair> fin(B->finals.size());
    for (size_t i = 0; i < fin.size(); i++) fin[i] = {B->finals[i].p, B->finals[i].t};
    nfinal += (int64_t)fin.size();
    long_rows(E, P, T, fin, [&](size_t first, size_t n, const float* f, const float* b, const std::vector<int64_t>& off) {
      parallel_for(n, E->host_threads, [&](size_t q) {
        const size_t i = first + q;
        const FinalPair& fp = B->finals[i];
        const ProfileHost& h = P->h[fp.p];
        const int64_t l = T->len[fp.t];
        const float* fr = f + off[q];
        const float* br = b + off[q];
        const float fwdsc = forward_score_from_rows(h, l, fr);
        if (long_exact[fp.p] &&
            std::exp(exp_tail_logsurv((double)((fwdsc - fp.filtersc) / kLn2f), h.fwd[0], h.fwd[1])) > o.f3)
          return;
        n_domain++;
        B->res[i].hit = define_domains(h, T->dsq.data() + T->off[fp.t], l, RawRows{fr, br}, fwdsc, o, B->res[i].h);
      });
    });
  }
  E->stats.kernel_launches += env_launches.load();
  E->stats.pairs_out[5] = n_env.load();
  E->stats.pairs_in[6] = rstats.device + rstats.redone;
  E->stats.pairs_out[6] = rstats.device;
  E->stats.cells[6] = rstats.cells;
  const auto t_end = std::chrono::steady_clock::now();
  E->stats.pairs_in[4] = nfinal;
  E->stats.pairs_out[4] = n_domain.load();
  E->stats.pairs_in[5] = n_domain.load();
  E->stats.ms[4] = rows_ms;
  E->stats.ms[6] = std::chrono::duration<double, std::milli>(t_end - t_start).count();
  E->stats.ms[7] = std::chrono::duration<double, std::milli>(t_end - t_dev).count();
  plog.add("total", t_start);
  plog.print();
  std::vector<std::vector<std::pair<int32_t, HitOut>>> per(np);
  for (auto& B : outs) {
    for (const auto& f : B->finals) E->stats.cells[4] += (double)P->h[f.p].m * T->len[f.t];
    for (size_t i = 0; i < B->finals.size(); i++)
      if (B->res[i].hit) per[B->finals[i].p].emplace_back(B->finals[i].t, std::move(B->res[i].h));
  }
  return report(P, T, cfg, per, out);
}

}  // namespace

// ================================================================ C ABI
extern "C" {

const char* sx_last_error(void) { return g_err.c_str(); }

int sx_create(const sx_opts* opts, sx_engine** out) {
  if (!out) return fail(SX_EINVAL, "sx_create: out is NULL");
  *out = nullptr;
  auto e = std::make_unique<sx_engine>();
  e->device = opts ? opts->device : 0;
  e->flags = opts ? opts->flags : 0;
  e->host_threads = (opts && opts->host_threads > 0) ? opts->host_threads : (int)std::thread::hardware_concurrency();
  e->host_threads = std::max(1, e->host_threads);
  e->batch_bytes = (opts && opts->batch_bytes > 0) ? opts->batch_bytes : (2LL << 30);
  e->pipeline_blocks = (opts && opts->pipeline_blocks > 0) ? opts->pipeline_blocks : 0;
  try {
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (e->device < 0 || e->device >= ndev)
      return fail(SX_EINVAL, "sx_create: device " + std::to_string(e->device) + " not present (" +
                                 std::to_string(ndev) + " devices)");
    CK(cudaSetDevice(e->device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, e->device));
    if (prop.major < 10)
      return fail(SX_EINVAL, std::string("sx_create: device is ") + prop.name + " (sm_" + std::to_string(prop.major) +
                                 std::to_string(prop.minor) + "); this library is built for sm_100a");
    e->num_sms = prop.multiProcessorCount;
    for (Slot& S : e->sl) S.create();
    {
      int least = 0, greatest = 0;
      CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
      CK(cudaStreamCreateWithPriority(&e->env_stream, cudaStreamNonBlocking, greatest));
      CK(cudaStreamCreateWithPriority(&e->env_stream2, cudaStreamNonBlocking, greatest));
      CK(cudaEventCreateWithFlags(&e->env_ev, cudaEventDisableTiming));
    }
    note_free_memory(e.get());
    for (int kind = 0; kind < 2; kind++) e->shape_table[kind] = default_shape_table(kind);
    (void)kernels();
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  }
  *out = e.release();
  return SX_OK;
}

void sx_destroy(sx_engine* e) {
  if (!e) return;
  cudaSetDevice(e->device);
  for (Slot& S : e->sl) S.destroy();
  for (cudaStream_t st : {e->env_stream, e->env_stream2})
    if (st) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
  if (e->env_ev) cudaEventDestroy(e->env_ev);
  e->env_stream = e->env_stream2 = nullptr;
  e->env_ev = nullptr;
  bool last;
  {
    std::lock_guard<std::mutex> g(e->life_mu);
    e->destroyed = true;
    last = e->live_sets == 0;
  }
  if (last) delete e;
}

// A set handed to the caller keeps its engine object alive (see sx_engine).
static void engine_ref(sx_engine* e) {
  std::lock_guard<std::mutex> g(e->life_mu);
  e->live_sets++;
}
static void engine_unref(sx_engine* e) {
  bool last;
  {
    std::lock_guard<std::mutex> g(e->life_mu);
    last = --e->live_sets == 0 && e->destroyed;
  }
  if (last) delete e;
}

static int finish_profiles(sx_engine* e, std::unique_ptr<sx_profiles> p, sx_profiles** out) {
  try {
    CK(cudaSetDevice(e->device));
    pack_profiles(p.get());
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  }
  engine_ref(e);
  *out = p.release();
  return SX_OK;
}

int sx_profiles_load_text(sx_engine* e, const char* text, size_t len, const char* source, sx_profiles** out) {
  if (!e || !out || (!text && len)) return fail(SX_EINVAL, "sx_profiles_load_text: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(e->mu);
  auto p = std::make_unique<sx_profiles>();
  p->eng = e;
  std::string err;
  if (!load_profiles_text(text ? text : "", len, source ? source : "<stream>", p->h, err)) return fail(SX_EINVAL, err);
  return finish_profiles(e, std::move(p), out);
}

int sx_profiles_from_arrays(sx_engine* e, const sx_profile_arrays* a, size_t n, sx_profiles** out) {
  if (!e || !out || (n && !a)) return fail(SX_EINVAL, "sx_profiles_from_arrays: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(e->mu);
  auto p = std::make_unique<sx_profiles>();
  p->eng = e;
  p->h.resize(n);
  for (size_t i = 0; i < n; i++) {
    const sx_profile_arrays& s = a[i];
    const std::string at = "sx_profiles_from_arrays: profile " + std::to_string(i);
    if (!s.name || !s.msc || !s.mo || !s.t || !s.p || !s.compo) return fail(SX_EINVAL, at + ": NULL field");
    if (s.m < 1) return fail(SX_EINVAL, at + ": M must be at least 1");
    ProfileHost& h = p->h[i];
    const size_t w = (size_t)s.m + 1;
    h.name = s.name;
    h.has_acc = s.acc != nullptr;
    h.has_desc = s.desc != nullptr;
    if (s.acc) h.acc = s.acc;
    if (s.desc) h.desc = s.desc;
    h.m = s.m;
    h.msc.assign(s.msc, s.msc + NSYM * w);
    h.mo.assign(s.mo, s.mo + NSYM * w);
    for (int q = 0; q < NTR; q++) {
      h.t[q].assign(s.t + q * w, s.t + (q + 1) * w);
      h.p[q].assign(s.p + q * w, s.p + (q + 1) * w);
    }
    h.msv_tbm = s.msv_tbm;
    std::copy(s.compo, s.compo + NRES, h.compo);
    h.has_ga = s.has_cutoffs & 1;
    h.has_tc = (s.has_cutoffs >> 1) & 1;
    h.has_nc = (s.has_cutoffs >> 2) & 1;
    for (int q = 0; q < 2; q++) {
      h.ga[q] = h.has_ga ? s.ga[q] : NAN;
      h.tc[q] = h.has_tc ? s.tc[q] : NAN;
      h.nc[q] = h.has_nc ? s.nc[q] : NAN;
    }
    h.has_msv = s.has_stats & 1;
    h.has_vit = (s.has_stats >> 1) & 1;
    h.has_fwd = (s.has_stats >> 2) & 1;
    for (int q = 0; q < 2; q++) {
      h.msv[q] = h.has_msv ? s.msv[q] : NAN;
      h.vit[q] = h.has_vit ? s.viterbi[q] : NAN;
      h.fwd[q] = h.has_fwd ? s.forward[q] : NAN;
    }
  }
  return finish_profiles(e, std::move(p), out);
}

int sx_profiles_load_file(sx_engine* e, const char* path, sx_profiles** out) {
  if (!e || !out || !path) return fail(SX_EINVAL, "sx_profiles_load_file: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(e->mu);
  auto p = std::make_unique<sx_profiles>();
  p->eng = e;
  std::string err;
  bool io = false;
  if (!load_profiles_file(path, p->h, err, io)) return fail(io ? SX_EIO : SX_EINVAL, err);
  return finish_profiles(e, std::move(p), out);
}

int sx_profiles_save(const sx_profiles* p, const char* path) {
  if (!p || !path) return fail(SX_EINVAL, "sx_profiles_save: NULL argument");
  std::string err;
  if (!save_profiles_binary(p->h, path, err)) return fail(SX_EIO, "sx_profiles_save: " + err);
  return SX_OK;
}

int sx_profiles_load_binary(sx_engine* e, const char* path, sx_profiles** out) {
  if (!e || !out || !path) return fail(SX_EINVAL, "sx_profiles_load_binary: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(e->mu);
  auto p = std::make_unique<sx_profiles>();
  p->eng = e;
  std::string err;
  bool io = false;
  if (!load_profiles_binary(path, p->h, err, io)) return fail(io ? SX_EIO : SX_EINVAL, "sx_profiles_load_binary: " + err);
  return finish_profiles(e, std::move(p), out);
}

int32_t sx_profiles_count(const sx_profiles* p) { return p ? (int32_t)p->h.size() : 0; }

int sx_profiles_info(const sx_profiles* p, int32_t i, sx_profile_info* out) {
  if (!p || !out || i < 0 || i >= (int32_t)p->h.size()) return fail(SX_EINVAL, "sx_profiles_info: bad index");
  const ProfileHost& h = p->h[i];
  out->name = h.name.c_str();
  out->acc = h.has_acc ? h.acc.c_str() : nullptr;
  out->desc = h.has_desc ? h.desc.c_str() : nullptr;
  out->m = h.m;
  out->calibrated = h.calibrated();
  for (int q = 0; q < 2; q++) {
    out->ga[q] = h.has_ga ? h.ga[q] : NAN;
    out->tc[q] = h.has_tc ? h.tc[q] : NAN;
    out->nc[q] = h.has_nc ? h.nc[q] : NAN;
    out->msv[q] = h.has_msv ? h.msv[q] : NAN;
    out->viterbi[q] = h.has_vit ? h.vit[q] : NAN;
    out->forward[q] = h.has_fwd ? h.fwd[q] : NAN;
  }
  return SX_OK;
}

void sx_profiles_free(sx_profiles* p) {
  if (!p) return;
  sx_engine* e = p->eng;
  cudaSetDevice(e->device);
  delete p;
  engine_unref(e);
}

static int finish_targets(sx_engine* e, std::unique_ptr<sx_targets> t, sx_targets** out) {
  t->dsq.resize(t->dsq.size() + 64, SYM_STAR);  // read slack past the last target
  try {
    CK(cudaSetDevice(e->device));
    pack_targets(t.get());
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  }
  engine_ref(e);
  *out = t.release();
  return SX_OK;
}

int sx_targets_create(sx_engine* e, const char* const* ids, const uint8_t* const* seqs, const size_t* lens, size_t n,
                      sx_targets** out) {
  if (!e || !out || (n && (!seqs || !lens))) return fail(SX_EINVAL, "sx_targets_create: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(e->mu);
  auto t = std::make_unique<sx_targets>();
  t->eng = e;
  size_t total = 64;  // an upper bound of the packed size
  for (size_t i = 0; i < n; i++) total += (lens[i] + 15) & ~(size_t)15;
  t->dsq = e->target_bytes.take(total);
  std::vector<uint8_t> dig;
  for (size_t i = 0; i < n; i++) {
    dig.clear();
    for (size_t q = 0; q < lens[i]; q++) {
      const uint8_t b = seqs[i][q];
      if (b == ' ' || b == '\t' || b == '\n' || b == '\r' || b == '\f' || b == '\v') continue;
      dig.push_back(kDigitize[b]);
    }
    if (dig.size() > (size_t)INT32_MAX) return fail(SX_EINVAL, "sx_targets_create: sequence too long");
    append_target(t.get(), dig.data(), dig.size());
    t->ids.push_back(ids && ids[i] ? ids[i] : std::to_string(i));
  }
  return finish_targets(e, std::move(t), out);
}

int sx_targets_create_digital(sx_engine* e, const uint8_t* dsq, const int64_t* offsets, const int64_t* lens, size_t n,
                              sx_targets** out) {
  if (!e || !out || (n && (!dsq || !offsets || !lens))) return fail(SX_EINVAL, "sx_targets_create_digital: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(e->mu);
  auto t = std::make_unique<sx_targets>();
  t->eng = e;
  size_t total = 64;
  for (size_t i = 0; i < n; i++) {
    if (lens[i] < 0 || offsets[i] < 0 || lens[i] > INT32_MAX) return fail(SX_EINVAL, "sx_targets_create_digital: bad length");
    total += ((size_t)lens[i] + 15) & ~(size_t)15;
  }
  t->dsq = e->target_bytes.take(total);
  t->off.reserve(n);
  t->len.reserve(n);
  for (size_t i = 0; i < n; i++) {
    const uint8_t* d = dsq + offsets[i];
    uint8_t hi = 0;  // max code, a loop the compiler vectorises; positions only on failure
    for (int64_t q = 0; q < lens[i]; q++) hi = std::max(hi, d[q]);
    if (hi > SYM_STAR)
      for (int64_t q = 0; q < lens[i]; q++)
        if (d[q] > SYM_STAR)
          return fail(SX_EINVAL, "sx_targets_create_digital: residue code " + std::to_string(d[q]) +
                                     " out of range in target " + std::to_string(i));
    append_target(t.get(), d, (size_t)lens[i]);
  }
  return finish_targets(e, std::move(t), out);
}

int64_t sx_targets_count(const sx_targets* t) { return t ? (int64_t)t->len.size() : 0; }

void sx_targets_free(sx_targets* t) {
  if (!t) return;
  sx_engine* e = t->eng;
  cudaSetDevice(e->device);
  delete t;
  engine_unref(e);
}

int sx_search(sx_engine* e, const sx_profiles* p, const sx_targets* t, const sx_search_cfg* cfg, sx_hits** out) {
  if (!e || !p || !t || !cfg || !out) return fail(SX_EINVAL, "sx_search: NULL argument");
  if (p->eng != e || t->eng != e) return fail(SX_EINVAL, "sx_search: profiles/targets belong to another engine");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(e->mu);
  NvtxRange nv("sx_search");
  auto h = std::make_unique<sx_hits>();
  try {
    CK(cudaSetDevice(e->device));
    const int rc = run_search(e, p, t, cfg, h.get());
    if (rc) return rc;
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  } catch (const std::bad_alloc&) {
    return fail(SX_ENOMEM, "sx_search: host allocation failed");
  }
  *out = h.release();
  return SX_OK;
}

int sx_search_many(sx_engine* e, const sx_profiles* const* sets, size_t n, const sx_targets* t,
                   const sx_search_cfg* cfg, sx_hits** out) {
  if (!e || !t || !cfg || !out || (n && !sets)) return fail(SX_EINVAL, "sx_search_many: NULL argument");
  for (size_t i = 0; i < n; i++) out[i] = nullptr;
  if (t->eng != e) return fail(SX_EINVAL, "sx_search_many: targets belong to another engine");
  for (size_t i = 0; i < n; i++)
    if (!sets[i] || sets[i]->eng != e)
      return fail(SX_EINVAL, "sx_search_many: profile set " + std::to_string(i) + " is NULL or of another engine");
  std::lock_guard<std::mutex> lk(e->mu);
  // the first set sx_search would reject decides the error
  for (size_t i = 0; i < n; i++) {
    const int rc = check_cutoffs(sets[i], cfg->cutoff_kind);
    if (rc) return rc;
  }
  // One combined set.  Search and report treat every profile on its own
  // (per-profile thresholds, E-values over the same targets, per-profile
  // domain Z), so slicing the combined hits by profile range is exact.
  std::vector<size_t> first(n + 1, 0);
  auto all = std::make_unique<sx_profiles>();
  all->eng = e;
  for (size_t i = 0; i < n; i++) {
    first[i] = all->h.size();
    all->h.insert(all->h.end(), sets[i]->h.begin(), sets[i]->h.end());
  }
  first[n] = all->h.size();
  std::vector<std::unique_ptr<sx_hits>> parts(n);
  try {
    CK(cudaSetDevice(e->device));
    sx_hits hits;
    if (!all->h.empty()) {
      pack_profiles(all.get());
      const int rc = run_search(e, all.get(), t, cfg, &hits);
      if (rc) return rc;
    }
    size_t q = 0;
    for (size_t i = 0; i < n; i++) {
      parts[i] = std::make_unique<sx_hits>();
      sx_hits& part = *parts[i];
      while (q < hits.hits.size() && (size_t)hits.hits[q].profile_index < first[i + 1]) {
        sx_hit hh = hits.hits[q++];
        const sx_domain* d = hits.doms.data() + hh.domain_offset;
        hh.profile_index -= (int32_t)first[i];
        hh.domain_offset = (int32_t)part.doms.size();
        part.doms.insert(part.doms.end(), d, d + hh.ndomains);
        part.hits.push_back(hh);
      }
    }
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  } catch (const std::bad_alloc&) {
    return fail(SX_ENOMEM, "sx_search_many: host allocation failed");
  }
  for (size_t i = 0; i < n; i++) out[i] = parts[i].release();
  return SX_OK;
}

size_t sx_hits_count(const sx_hits* h) { return h ? h->hits.size() : 0; }
const sx_hit* sx_hits_array(const sx_hits* h) { return h && !h->hits.empty() ? h->hits.data() : nullptr; }
size_t sx_hits_domain_count(const sx_hits* h) { return h ? h->doms.size() : 0; }
const sx_domain* sx_hits_domains(const sx_hits* h) { return h && !h->doms.empty() ? h->doms.data() : nullptr; }
void sx_hits_free(sx_hits* h) { delete h; }

int sx_shape_count(int kind) { return kind == 0 ? kNumMsvShapes : kind == 1 ? kNumVitShapes : -1; }

int sx_shape_info(int kind, int index, int32_t* g, int32_t* c, int32_t* rt) {
  if (kind < 0 || kind > 1 || index < 0 || index >= sx_shape_count(kind) || !g || !c || !rt)
    return fail(SX_EINVAL, "sx_shape_info: bad kind or index");
  if (kind == 0) {
    *g = kMsvShapes[index].g;
    *c = kMsvShapes[index].c;
    *rt = 0;
  } else {
    *g = kVitShapes[index].g;
    *c = kVitShapes[index].c;
    *rt = kVitShapes[index].rt;
  }
  return SX_OK;
}

int sx_shape_for(const sx_engine* e, int kind, int32_t m) {
  if (!e || kind < 0 || kind > 1 || m < 0) return -1;
  return is_long(m) ? -1 : shape_for(e, kind, m);
}

int sx_set_shape_table(sx_engine* e, int kind, const int32_t* shape_by_m, size_t len) {
  if (!e || kind < 0 || kind > 1 || (len && !shape_by_m)) return fail(SX_EINVAL, "sx_set_shape_table: bad argument");
  if (len != 0 && len != (size_t)kMaxM + 1)
    return fail(SX_EINVAL, "sx_set_shape_table: the table has one entry per M = 0.." + std::to_string(kMaxM));
  std::vector<int16_t> t = len ? std::vector<int16_t>(len, -1) : default_shape_table(kind);
  for (size_t m = 0; m < len; m++) {
    const int s = shape_by_m[m];
    if (s < 0) continue;
    if (s >= sx_shape_count(kind)) return fail(SX_EINVAL, "sx_set_shape_table: shape " + std::to_string(s) + " unknown");
    const int cols = kind == 0 ? kMsvShapes[s].g * kMsvShapes[s].c : kVitShapes[s].g * kVitShapes[s].c;
    if (cols < (int)m)
      return fail(SX_EINVAL, "sx_set_shape_table: shape " + std::to_string(s) + " holds " + std::to_string(cols) +
                                 " columns, fewer than M=" + std::to_string(m));
    t[m] = (int16_t)s;
  }
  std::lock_guard<std::mutex> lk(e->mu);
  e->shape_table[kind] = std::move(t);
  return SX_OK;
}

int sx_last_search_stats(const sx_engine* e, sx_search_stats* out) {
  if (!e || !out) return fail(SX_EINVAL, "sx_last_search_stats: NULL argument");
  *out = e->stats;
  return SX_OK;
}

int sx_score_pairs(sx_engine* e, const sx_profiles* p, const sx_targets* t, const int32_t* pair_profile,
                   const int32_t* pair_target, size_t npairs, float* msv, float* viterbi, float* forward,
                   float* backward, float* bias) {
  if (!e || !p || !t || (npairs && (!pair_profile || !pair_target))) return fail(SX_EINVAL, "sx_score_pairs: NULL argument");
  if (p->eng != e || t->eng != e) return fail(SX_EINVAL, "sx_score_pairs: profiles/targets belong to another engine");
  std::lock_guard<std::mutex> lk(e->mu);
  NvtxRange nv("sx_score_pairs");
  const size_t np = p->h.size(), nt = t->len.size();
  for (size_t i = 0; i < npairs; i++)
    if (pair_profile[i] < 0 || (size_t)pair_profile[i] >= np || pair_target[i] < 0 || (size_t)pair_target[i] >= nt)
      return fail(SX_EINVAL, "sx_score_pairs: pair " + std::to_string(i) + " out of range");
  if (!npairs) return SX_OK;
  try {
    CK(cudaSetDevice(e->device));
    cudaStream_t s = e->stream;
    e->stats = sx_search_stats{};
    std::vector<Thresholds> th(np, Thresholds{-INFINITY, -INFINITY, -INFINITY, 0});
    e->thr.upload(th.data(), th.size(), s);
    e->overflow.alloc(1);
    CK(cudaMemsetAsync(e->overflow.p, 0, sizeof(unsigned), s));
    e->scores.alloc(npairs);
    // pairs of profiles longer than kMaxM go through the long kernels
    std::vector<size_t> lng;
    std::vector<sxk::LongPair> lpairs;
    for (size_t i = 0; i < npairs; i++)
      if (is_long(p->h[pair_profile[i]].m)) {
        lng.push_back(i);
        lpairs.push_back({pair_profile[i], pair_target[i]});
      }
    if (msv) {
      // list sorted by (profile, length desc); tiles per profile over that list
      std::vector<int32_t> idx(npairs);
      std::iota(idx.begin(), idx.end(), 0);
      std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
        if (pair_profile[a] != pair_profile[b]) return pair_profile[a] < pair_profile[b];
        return t->len[pair_target[a]] > t->len[pair_target[b]];
      });
      std::vector<int32_t> lst(npairs), slot(npairs);
      for (size_t q = 0; q < npairs; q++) {
        lst[q] = pair_target[idx[q]];
        slot[q] = idx[q];
      }
      std::vector<std::vector<MsvTile>> tiles(kNumMsvShapes);
      size_t q = 0;
      while (q < npairs) {
        size_t r = q;
        const int pp = pair_profile[idx[q]];
        while (r < npairs && pair_profile[idx[r]] == pp) r++;
        if (p->msv_shape[pp] >= 0)
          for (size_t a = q; a < r; a += 4096)
            tiles[p->msv_shape[pp]].push_back({pp, (int32_t)a, (int32_t)std::min(r, a + 4096), 0});
        q = r;
      }
      e->plist.upload(lst.data(), npairs, s);
      e->slots.upload(slot.data(), npairs, s);
      launch_msv(e, e->sl[0], e->sl[0].hi, p, t, tiles, e->plist.p, e->scores.p, e->slots.p, nullptr, nullptr, nullptr);
      CK(cudaMemcpyAsync(msv, e->scores.p, sizeof(float) * npairs, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      if (!lng.empty()) {
        std::vector<float> v;
        long_scores(e, p, t, lpairs, false, v);
        for (size_t q = 0; q < lng.size(); q++) msv[lng[q]] = v[q];
      }
    }
    if (bias || viterbi) {
      // pair lists per vbin, every pair carries its slot
      std::vector<PairRec> recs;
      std::vector<BinRegion> reg(kMaxBins);
      std::vector<unsigned> cnt(kMaxBins, 0);
      std::vector<std::vector<int32_t>> byb(kMaxBins);
      // long-profile pairs sit in an extra bin that only the bias pass reads
      for (size_t i = 0; i < npairs; i++) {
        const int vs = p->dp[pair_profile[i]].vshape;
        byb[vs >= 0 ? vs : kNumVitShapes].push_back((int32_t)i);
      }
      for (int b = 0; b < kMaxBins; b++) {
        reg[b].off = (int64_t)recs.size();
        reg[b].cap = (uint32_t)byb[b].size();
        reg[b].pad = 0;
        cnt[b] = (unsigned)byb[b].size();
        for (int32_t i : byb[b]) recs.push_back({pair_profile[i], pair_target[i], 0.f, 0.f, 0.f, 0.f, i, 0});
      }
      e->lists[0].upload(recs.data(), recs.size(), s);
      e->bins[0].upload(reg.data(), reg.size(), s);
      e->counts.alloc(4 * kMaxBins);
      CK(cudaMemcpyAsync(e->counts.p, cnt.data(), sizeof(unsigned) * kMaxBins, cudaMemcpyHostToDevice, s));
      const auto& K = kernels();
      if (bias) {
        unsigned mx = *std::max_element(cnt.begin(), cnt.end());
        dim3 grid((unsigned)std::max<int64_t>(1, std::min<int64_t>((mx + 255) / 256, (int64_t)e->num_sms * 8)),
                  kNumVitShapes + 1);
        sxk::bias_kernel<<<grid, 256, 0, s>>>(e->lists[0].p, e->counts.p, e->bins[0].p, nullptr, nullptr, nullptr,
                                              e->overflow.p, p->d_bias.p, e->thr.p, t->d_res.p, t->d_off.p, t->d_len.p,
                                              0.f, e->scores.p, p->d_prof.p);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(bias, e->scores.p, sizeof(float) * npairs, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
      }
      if (viterbi) {
        e->sl[0].cursor.alloc(kMaxBins);
        CK(cudaMemsetAsync(e->sl[0].cursor.p, 0, sizeof(unsigned) * kMaxBins, s));
        CK(cudaEventRecord(e->ev[0], s));
        for (int b = 0; b < kNumVitShapes; b++) {
          if (!cnt[b]) continue;
          const int blocks = vit_blocks(e->num_sms, b, cnt[b]);
          K.vitg[b]<<<blocks, 256, 0, s>>>(e->lists[0].p, e->counts.p, e->bins[0].p, b, nullptr, nullptr, nullptr,
                                           e->overflow.p, p->d_prof.p, e->thr.p, p->d_vit.p, t->d_res.p, t->d_off.p,
                                           t->d_len.p, t->d_xsc.p, 0.f, e->scores.p, e->sl[0].cursor.p);
        }
        CK(cudaGetLastError());
        CK(cudaEventRecord(e->ev[1], s));
        CK(cudaMemcpyAsync(viterbi, e->scores.p, sizeof(float) * npairs, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        e->stats.ms[2] = elapsed_ms(e->ev[0], e->ev[1]);  // the Viterbi launches, for tuners
        for (size_t i = 0; i < npairs; i++)
          if (!is_long(p->h[pair_profile[i]].m)) e->stats.cells[2] += (double)p->h[pair_profile[i]].m * t->len[pair_target[i]];
        if (!lng.empty()) {
          std::vector<float> v;
          long_scores(e, p, t, lpairs, true, v);
          for (size_t q = 0; q < lng.size(); q++) viterbi[lng[q]] = v[q];
        }
      }
    }
    if (forward || backward) {
      auto put = [&](size_t i, const float* fr, const float* br) {
        const ProfileHost& h = p->h[pair_profile[i]];
        const int64_t l = t->len[pair_target[i]];
        if (l == 0 || h.m == 0) {
          if (forward) forward[i] = kNegInf;
          if (backward) backward[i] = kNegInf;
          return;
        }
        if (forward) forward[i] = forward_score_from_rows(h, l, fr);
        if (backward) backward[i] = backward_score_from_rows(l, br);
      };
      std::vector<FinalPair> fp;
      for (size_t i = 0; i < npairs; i++)
        if (!is_long(p->h[pair_profile[i]].m)) fp.push_back({pair_profile[i], pair_target[i], 0.f, 0.f, 0.f, (int32_t)i});
      rows_pass_sync(e, p, t, fp, [&](size_t q, const float* fr, const float* br) { put((size_t)fp[q].slot, fr, br); });
      long_rows(e, p, t, lpairs, [&](size_t first, size_t n, const float* f, const float* b, const std::vector<int64_t>& off) {
        for (size_t q = 0; q < n; q++) put(lng[first + q], f + off[q], b + off[q]);
      });
    }
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  }
  return SX_OK;
}

int sx_score_prescreens(sx_engine* e, const sx_profiles* p, const sx_targets* t, const int32_t* pair_profile,
                        const int32_t* pair_target, size_t npairs, float* msv_bound, float* fwd_scan,
                        float* vit_bound) {
  if (!e || !p || !t || (npairs && (!pair_profile || !pair_target)))
    return fail(SX_EINVAL, "sx_score_prescreens: NULL argument");
  if (p->eng != e || t->eng != e) return fail(SX_EINVAL, "sx_score_prescreens: profiles/targets belong to another engine");
  std::lock_guard<std::mutex> lk(e->mu);
  const size_t np = p->h.size(), nt = t->len.size();
  for (size_t i = 0; i < npairs; i++)
    if (pair_profile[i] < 0 || (size_t)pair_profile[i] >= np || pair_target[i] < 0 || (size_t)pair_target[i] >= nt)
      return fail(SX_EINVAL, "sx_score_prescreens: pair " + std::to_string(i) + " out of range");
  if (npairs > (size_t)INT32_MAX) return fail(SX_EINVAL, "sx_score_prescreens: too many pairs");
  for (size_t i = 0; i < npairs; i++) {
    if (msv_bound) msv_bound[i] = NAN;
    if (fwd_scan) fwd_scan[i] = NAN;
    if (vit_bound) vit_bound[i] = NAN;
  }
  if (!npairs) return SX_OK;
  try {
    CK(cudaSetDevice(e->device));
    cudaStream_t s = e->stream;
    const auto& K = kernels();
    std::vector<Thresholds> th(np, Thresholds{-INFINITY, -INFINITY, -INFINITY, 0});
    e->thr.upload(th.data(), th.size(), s);
    e->overflow.alloc(1);
    CK(cudaMemsetAsync(e->overflow.p, 0, sizeof(unsigned), s));
    if (msv_bound) {
      // pairs of pre-screened profiles, sorted by (profile, length desc); one
      // profile per tile (the high half is padding)
      std::vector<int32_t> idx;
      for (size_t i = 0; i < npairs; i++)
        if (p->dp[pair_profile[i]].vbin >= 0 && p->dp[pair_profile[i]].q_off >= 0) idx.push_back((int32_t)i);
      std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
        if (pair_profile[a] != pair_profile[b]) return pair_profile[a] < pair_profile[b];
        return t->len[pair_target[a]] > t->len[pair_target[b]];
      });
      const size_t n = idx.size();
      if (n) {
        std::vector<int32_t> lst(n), slot(n);
        for (size_t q = 0; q < n; q++) {
          lst[q] = pair_target[idx[q]];
          slot[q] = idx[q];
        }
        std::vector<std::vector<sxk::PackedTile>> tiles(kNumMsvShapes);
        size_t q = 0;
        while (q < n) {
          size_t r = q;
          const int pp = pair_profile[idx[q]];
          while (r < n && pair_profile[idx[r]] == pp) r++;
          for (size_t a = q; a < r; a += 4096)
            tiles[p->msv_shape[pp]].push_back({pp, -1, (int32_t)a, (int32_t)std::min(r, a + 4096)});
          q = r;
        }
        e->plist.upload(lst.data(), n, s);
        e->slots.upload(slot.data(), n, s);
        e->scores.alloc(npairs);
        std::vector<float> nanv(npairs, NAN);
        CK(cudaMemcpyAsync(e->scores.p, nanv.data(), sizeof(float) * npairs, cudaMemcpyHostToDevice, s));
        Slot& S = e->sl[0];
        for (int sh = 0; sh < kNumMsvShapes; sh++) {
          if (tiles[sh].empty()) continue;
          S.ptiles.upload(tiles[sh].data(), tiles[sh].size(), s);
          const size_t smem = msv_smem(sh);
          CK(cudaFuncSetAttribute((const void*)K.msv16[sh], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
          K.msv16[sh]<<<(unsigned)tiles[sh].size(), 256, smem, s>>>(
              S.ptiles.p, p->d_prof.p, e->thr.p, p->d_qimg.p, t->d_res.p, t->d_off.p, t->d_len.p, t->d_tpar.p,
              e->plist.p, nullptr, 0, nullptr, 0, e->overflow.p, e->scores.p, e->slots.p, 0);
          CK(cudaGetLastError());
          CK(cudaStreamSynchronize(s));  // the tile buffer is reused by the next shape
        }
        CK(cudaMemcpyAsync(msv_bound, e->scores.p, sizeof(float) * npairs, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
      }
    }
    if (vit_bound) {
      // pairs of Viterbi-pre-screened profiles, one list per profile; one
      // launch per profile (its list at p0 = the profile, count at index 0)
      std::vector<std::vector<int32_t>> byp(np);
      for (size_t i = 0; i < npairs; i++)
        if (p->dp[pair_profile[i]].qv_shape >= 0) byp[pair_profile[i]].push_back((int32_t)i);
      std::vector<PairRec> recs;
      std::vector<int64_t> seg;
      std::vector<int> profs;
      std::vector<unsigned> cnt;
      for (size_t pi = 0; pi < np; pi++) {
        if (byp[pi].empty()) continue;
        profs.push_back((int)pi);
        seg.push_back((int64_t)recs.size());
        cnt.push_back((unsigned)byp[pi].size());
        for (int32_t i : byp[pi]) recs.push_back({(int32_t)pi, pair_target[i], 0.f, 0.f, 0.f, 0.f, i, 0});
      }
      if (!recs.empty()) {
        Slot& S = e->sl[0];
        S.vlist.upload(recs.data(), recs.size(), s);
        S.vcount.upload(cnt.data(), cnt.size(), s);
        constexpr int kSub = 8;
        std::vector<sxk::VitTile> tiles;
        for (int pi : profs)
          for (int q = 0; q < kSub; q++) tiles.push_back({pi, q, kSub, 0});
        S.vtiles.upload(tiles.data(), tiles.size(), s);
        e->scores.alloc(npairs);
        std::vector<float> nanv(npairs, NAN);
        CK(cudaMemcpyAsync(e->scores.p, nanv.data(), sizeof(float) * npairs, cudaMemcpyHostToDevice, s));
        for (size_t q = 0; q < profs.size(); q++) {
          const int sh = p->dp[profs[q]].qv_shape;
          const int smem = vit16_smem(kVit16Shapes[sh]);
          CK(cudaFuncSetAttribute((const void*)K.vit16[sh], cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
          K.vit16[sh]<<<kSub, vit16_threads(kVit16Shapes[sh]), smem, s>>>(S.vtiles.p + q * kSub, p->d_prof.p, e->thr.p, p->d_qvimg.p, t->d_res.p,
                                             t->d_off.p, t->d_len.p, t->d_xsc.p, S.vlist.p + seg[q], cnt[q],
                                             S.vcount.p + q, profs[q], nullptr, nullptr, nullptr, e->overflow.p,
                                             kSlackBits, e->scores.p, nullptr);
        }
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(vit_bound, e->scores.p, sizeof(float) * npairs, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
      }
    }
    if (fwd_scan) {
      // every pair through the F3 pre-screen with a threshold of -inf: all of
      // them come out of the kernel carrying its Forward estimate
      std::vector<PairRec> recs;
      std::vector<BinRegion> reg(kMaxBins);
      std::vector<unsigned> cnt(kMaxBins, 0);
      std::vector<std::vector<int32_t>> byb(kMaxBins);
      for (size_t i = 0; i < npairs; i++)
        if (p->dp[pair_profile[i]].vbin >= 0) byb[p->dp[pair_profile[i]].vbin].push_back((int32_t)i);
      for (int b = 0; b < kMaxBins; b++) {
        reg[b].off = (int64_t)recs.size();
        reg[b].cap = (uint32_t)byb[b].size();
        reg[b].pad = 0;
        cnt[b] = (unsigned)byb[b].size();
        for (int32_t i : byb[b]) recs.push_back({pair_profile[i], pair_target[i], 0.f, 0.f, 0.f, 0.f, i, 0});
      }
      if (!recs.empty()) {
        Slot& S = e->sl[0];
        S.lists[2].upload(recs.data(), recs.size(), s);
        S.lists[3].alloc(recs.size());
        S.bins[2].upload(reg.data(), reg.size(), s);
        S.bins[3].upload(reg.data(), reg.size(), s);
        e->counts.alloc(4 * kMaxBins);
        CK(cudaMemcpyAsync(e->counts.p + 2 * kMaxBins, cnt.data(), sizeof(unsigned) * kMaxBins, cudaMemcpyHostToDevice, s));
        CK(cudaMemsetAsync(e->counts.p + 3 * kMaxBins, 0, sizeof(unsigned) * kMaxBins, s));
        for (int b = 0; b < kNumVbins; b++) {
          if (!cnt[b]) continue;
          K.fwd_scan[b]<<<warp_ctas(e->num_sms, cnt[b]), 32, 0, s>>>(
              S.lists[2].p, e->counts.p + 2 * kMaxBins, S.bins[2].p, b, S.lists[3].p, S.bins[3].p,
              e->counts.p + 3 * kMaxBins, e->overflow.p, p->d_prof.p, e->thr.p, p->d_vfb.p, t->d_res.p, t->d_off.p,
              t->d_len.p, t->d_xsc.p, kSlackBits, nullptr, nullptr);
        }
        CK(cudaGetLastError());
        std::vector<PairRec> out(recs.size());
        CK(cudaMemcpyAsync(out.data(), S.lists[3].p, sizeof(PairRec) * out.size(), cudaMemcpyDeviceToHost, s));
        std::vector<unsigned> oc(kMaxBins);
        CK(cudaMemcpyAsync(oc.data(), e->counts.p + 3 * kMaxBins, sizeof(unsigned) * kMaxBins, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (int b = 0; b < kNumVbins; b++)
          for (unsigned q = 0; q < std::min(oc[b], cnt[b]); q++) {
            const PairRec& r = out[reg[b].off + q];
            fwd_scan[r.slot] = r.fwd;
          }
      }
    }
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  }
  return SX_OK;
}

int sx_posterior_grad(sx_engine* e, const sx_profiles* p, const sx_targets* t, const int32_t* pair_profile,
                      const int32_t* pair_target, size_t npairs, int32_t m, float* d_msc, float* d_isc,
                      float* d_trans, double* lnz) {
  if (!e || !p || !t || (npairs && (!pair_profile || !pair_target || !d_msc || !d_isc || !d_trans || !lnz)))
    return fail(SX_EINVAL, "sx_posterior_grad: NULL argument");
  if (p->eng != e || t->eng != e) return fail(SX_EINVAL, "sx_posterior_grad: profiles/targets belong to another engine");
  std::lock_guard<std::mutex> lk(e->mu);
  const size_t np = p->h.size(), nt = t->len.size();
  for (size_t i = 0; i < npairs; i++) {
    if (pair_profile[i] < 0 || (size_t)pair_profile[i] >= np || pair_target[i] < 0 || (size_t)pair_target[i] >= nt)
      return fail(SX_EINVAL, "sx_posterior_grad: pair " + std::to_string(i) + " out of range");
    if (p->h[pair_profile[i]].m != m)
      return fail(SX_EINVAL, "sx_posterior_grad: pair " + std::to_string(i) + " uses a profile of M=" +
                                 std::to_string(p->h[pair_profile[i]].m) + ", expected " + std::to_string(m));
    if (is_long(m))
      return fail(SX_EINVAL, "sx_posterior_grad: profiles of M > " + std::to_string(kMaxM) + " are not supported");
  }
  if (!npairs) return SX_OK;
  const int W = m + 1;
  const size_t out_per = (size_t)(25 + 25 + 8) * W;
  try {
    CK(cudaSetDevice(e->device));
    cudaStream_t s = e->stream;
    const int vb = p->dp[pair_profile[0]].vbin, VC = kVcBins[vb];
    const auto& K = kernels();
    const int64_t budget = scratch_budget(e, std::max<int64_t>(e->batch_bytes, 64LL << 20));
    size_t i0 = 0;
    while (i0 < npairs) {
      // chunk: scratch floats per pair ~ (L/S + S + 2) * 3 * 32 * VC + 6 (L+1) + out, doubles (L+1)
      std::vector<sxk::AdjPair> ap;
      int64_t fo = 0, dd = 0;
      size_t i1 = i0;
      while (i1 < npairs) {
        const int64_t L = t->len[pair_target[i1]];
        const int S = std::max<int>(1, (int)std::ceil(std::sqrt((double)std::max<int64_t>(L, 1))));
        const int64_t rowf = 3LL * 32 * VC;
        const int64_t need_f = (L / S + 1) * rowf + (S + 1) * rowf + 6 * (L + 1);
        if (i1 > i0 && (fo + need_f + (int64_t)(i1 - i0 + 1) * (int64_t)out_per) * 4 + (dd + L + 1) * 8 > budget)
          break;
        sxk::AdjPair a{};
        a.p = pair_profile[i1];
        a.t = pair_target[i1];
        a.S = S;
        a.ck_off = fo;
        a.seg_off = a.ck_off + (L / S + 1) * rowf;
        a.sp_off = a.seg_off + (S + 1) * rowf;
        a.out_off = (int64_t)(i1 - i0) * (int64_t)out_per;  // outputs packed per pair in their own buffer
        a.ls_off = dd;
        fo = a.sp_off + 6 * (L + 1);
        dd += L + 1;
        ap.push_back(a);
        i1++;
      }
      const int n = (int)ap.size();
      e->adj_pairs.upload(ap.data(), ap.size(), s);
      e->adj_f.alloc((size_t)fo);
      e->adj_out.alloc((size_t)n * out_per);
      e->adj_d.alloc((size_t)std::max<int64_t>(dd, 1));
      e->adj_lnz.alloc((size_t)n);
      CK(cudaMemsetAsync(e->adj_out.p, 0, sizeof(float) * out_per * (size_t)n, s));
      const int blocks = std::max(1, std::min((n + 3) / 4, e->num_sms * 32));
      K.adjf[vb]<<<blocks, 128, 0, s>>>(e->adj_pairs.p, n, p->d_prof.p, p->d_vfb.p, t->d_res.p, t->d_off.p,
                                        t->d_len.p, t->d_xsc.p, e->adj_f.p, e->adj_d.p, e->adj_lnz.p);
      K.adjb[vb]<<<blocks, 128, 0, s>>>(e->adj_pairs.p, n, p->d_prof.p, p->d_vfb.p, t->d_res.p, t->d_off.p,
                                        t->d_len.p, t->d_xsc.p, e->adj_f.p, e->adj_d.p, e->adj_lnz.p, e->adj_out.p);
      CK(cudaGetLastError());
      // scatter the packed [25W | 25W | 8W] outputs straight into the caller's three arrays
      // one copy into page-locked staging, then the host threads split the
      // counts into the caller's three arrays (and fault in their pages)
      e->adj_host.alloc(out_per * (size_t)n);
      CK(cudaMemcpyAsync(e->adj_host.p, e->adj_out.p, sizeof(float) * out_per * (size_t)n, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(lnz + i0, e->adj_lnz.p, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      const float* hs = e->adj_host.p;
      parallel_for((size_t)n, e->host_threads, [&](size_t q) {
        const float* src = hs + q * out_per;
        memcpy(d_msc + (i0 + q) * 25 * W, src, sizeof(float) * 25 * W);
        memcpy(d_isc + (i0 + q) * 25 * W, src + 25 * W, sizeof(float) * 25 * W);
        memcpy(d_trans + (i0 + q) * 8 * W, src + 50 * W, sizeof(float) * 8 * W);
      });
      i0 = i1;
    }
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  }
  return SX_OK;
}

}  // extern "C"

// ================================================================ no-allocation entry point
//
// sx_score_viterbi_static: Viterbi scores for explicit pairs without any
// allocation.  Its working memory -- the caller's pair indices, the pair
// records grouped by kernel shape, the per-shape list descriptors and the
// output staging -- lives in one file-scope device array of fixed size,
// reserved on every GPU that loads this library for as long as the process
// runs.  The host side uses only stack storage.
namespace {

constexpr size_t kStaticMaxPairs = 8192;
constexpr size_t kStaticPairIdxOff = 0;                                                    // int32 pp[], pt[]
constexpr size_t kStaticRecOff = kStaticPairIdxOff + 2 * kStaticMaxPairs * sizeof(int32_t);  // PairRec[]
constexpr size_t kStaticBinOff = kStaticRecOff + kStaticMaxPairs * sizeof(PairRec);         // BinRegion[]
constexpr size_t kStaticCountOff = kStaticBinOff + 16 * sizeof(BinRegion);                  // unsigned[16]
constexpr size_t kStaticFlagOff = kStaticCountOff + 16 * sizeof(unsigned);                  // unsigned
constexpr size_t kStaticScoreOff = (kStaticFlagOff + 4 + 255) & ~(size_t)255;               // float[]
constexpr size_t kStaticScratchBytes = kStaticScoreOff + kStaticMaxPairs * sizeof(float);
static_assert(kNumVbins <= 16, "static scratch holds at most 16 pair lists");

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

struct StaticLayout {
  int32_t off[16], n[16];
};

// Scatter the caller's pairs into per-shape lists at host-computed offsets
// and publish the list descriptors the Viterbi kernels read.
__global__ void static_bucket_kernel(unsigned char* scratch, int npairs, const DevProfile* __restrict__ profs,
                                     StaticLayout lay) {
  const int32_t* pp = reinterpret_cast<const int32_t*>(scratch + kStaticPairIdxOff);
  const int32_t* pt = pp + kStaticMaxPairs;
  PairRec* recs = reinterpret_cast<PairRec*>(scratch + kStaticRecOff);
  BinRegion* bins = reinterpret_cast<BinRegion*>(scratch + kStaticBinOff);
  unsigned* counts = reinterpret_cast<unsigned*>(scratch + kStaticCountOff);
  __shared__ unsigned cursor[16];
  if (threadIdx.x < 16) {
    cursor[threadIdx.x] = 0;
    if (threadIdx.x < kNumVbins) {
      bins[threadIdx.x].off = lay.off[threadIdx.x];
      bins[threadIdx.x].cap = (uint32_t)lay.n[threadIdx.x];
      bins[threadIdx.x].pad = 0;
      counts[threadIdx.x] = (unsigned)lay.n[threadIdx.x];
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < npairs; i += blockDim.x) {
    const int b = profs[pp[i]].vbin;
    const unsigned pos = (unsigned)lay.off[b] + atomicAdd(&cursor[b], 1u);
    PairRec r;
    r.p = pp[i]; r.t = pt[i]; r.usc = r.filtersc = r.vsc = r.fwd = 0.f; r.slot = i; r.pad = 0;
    recs[pos] = r;
  }
}

// Device address of g_static_scratch for each device, looked up once per
// device context (with that device current): on the first call on the device,
// and again after the device's context has been replaced (cudaDeviceReset
// destroys the primary context and the module that holds the array, so an
// address cached before it would dangle).  The context is told apart by the
// driver's context id, reached through the runtime's driver entry points so
// the library needs no link to libcuda.
std::mutex g_static_mu;
struct StaticAddr {
  void* ptr = nullptr;
  unsigned long long ctx_id = 0;
};
StaticAddr g_static_addr[128];

typedef int (*CtxGetCurrentFn)(void** ctx);
typedef int (*CtxGetIdFn)(void* ctx, unsigned long long* id);

// Id of the calling thread's current context, or 0 when the driver cannot
// report one (the cached address is then kept for the process lifetime).
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
  });
  if (!get_current || !get_id) return 0;
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

int static_scratch_ptr(int device, unsigned char** out) {
  if (device < 0 || device >= 128) return fail(SX_EINVAL, "sx_score_viterbi_static: device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_static_mu);
  StaticAddr& a = g_static_addr[device];
  const unsigned long long ctx = current_context_id();
  if (!a.ptr || ctx != a.ctx_id) {
    void* ptr = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&ptr, g_static_scratch);
    if (rc != cudaSuccess || !ptr)
      return fail(SX_ECUDA, std::string("sx_score_viterbi_static: cudaGetSymbolAddress: ") + cudaGetErrorString(rc));
    a.ptr = ptr;
    a.ctx_id = ctx;
  }
  *out = static_cast<unsigned char*>(a.ptr);
  return SX_OK;
}

}  // namespace

extern "C" int sx_score_viterbi_static(sx_engine* e, const sx_profiles* p, const sx_targets* t,
                                       const int32_t* pair_profile, const int32_t* pair_target, size_t npairs,
                                       float* viterbi) {
  if (!e || !p || !t || (npairs && (!pair_profile || !pair_target || !viterbi)))
    return fail(SX_EINVAL, "sx_score_viterbi_static: NULL argument");
  if (p->eng != e || t->eng != e)
    return fail(SX_EINVAL, "sx_score_viterbi_static: profiles/targets belong to another engine");
  if (npairs > kStaticMaxPairs)
    return fail(SX_EINVAL, "sx_score_viterbi_static: " + std::to_string(npairs) + " pairs exceed the fixed limit of " +
                               std::to_string(kStaticMaxPairs) + " per call");
  std::lock_guard<std::mutex> lk(e->mu);
  const size_t np = p->h.size(), nt = t->len.size();
  StaticLayout lay{};
  for (size_t i = 0; i < npairs; i++) {
    if (pair_profile[i] < 0 || (size_t)pair_profile[i] >= np || pair_target[i] < 0 || (size_t)pair_target[i] >= nt)
      return fail(SX_EINVAL, "sx_score_viterbi_static: pair " + std::to_string(i) + " out of range");
    if (p->dp[pair_profile[i]].vbin < 0)
      return fail(SX_EINVAL, "sx_score_viterbi_static: profiles of M > " + std::to_string(kMaxM) + " are not supported");
    lay.n[p->dp[pair_profile[i]].vbin]++;
  }
  if (!npairs) return SX_OK;
  for (int b = 1; b < kNumVbins; b++) lay.off[b] = lay.off[b - 1] + lay.n[b - 1];
  try {
    CK(cudaSetDevice(e->device));
    unsigned char* scratch = nullptr;
    const int rc = static_scratch_ptr(e->device, &scratch);
    if (rc) return rc;
    cudaStream_t s = e->stream;
    CK(cudaMemcpyAsync(scratch + kStaticPairIdxOff, pair_profile, npairs * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(scratch + kStaticPairIdxOff + kStaticMaxPairs * sizeof(int32_t), pair_target,
                       npairs * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(scratch + kStaticFlagOff, 0, sizeof(unsigned), s));
    static_bucket_kernel<<<1, 1024, 0, s>>>(scratch, (int)npairs, p->d_prof.p, lay);
    const auto& K = kernels();
    const PairRec* recs = reinterpret_cast<const PairRec*>(scratch + kStaticRecOff);
    const BinRegion* bins = reinterpret_cast<const BinRegion*>(scratch + kStaticBinOff);
    const unsigned* counts = reinterpret_cast<const unsigned*>(scratch + kStaticCountOff);
    unsigned* flag = reinterpret_cast<unsigned*>(scratch + kStaticFlagOff);
    float* scores = reinterpret_cast<float*>(scratch + kStaticScoreOff);
    for (int b = 0; b < kNumVbins; b++) {
      if (!lay.n[b]) continue;
      const int blocks = (int)std::min<int64_t>((lay.n[b] + 7) / 8, (int64_t)e->num_sms * 16);
      K.vit[b]<<<blocks, 256, 0, s>>>(recs, counts, bins, b, nullptr, nullptr, nullptr, flag, p->d_prof.p, nullptr,
                                      p->d_vfb.p, t->d_res.p, t->d_off.p, t->d_len.p, t->d_xsc.p, 0.f, scores);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(viterbi, scores, npairs * sizeof(float), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  }
  return SX_OK;
}
