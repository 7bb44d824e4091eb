// The search scheduler: profile blocks through the device filter cascade on a
// two-slot pipeline of prioritised streams, the exact host re-checks between
// stages, the Forward/Backward row passes of the final pairs, domain
// definition on the host pool, profiles longer than the lane-group kernels
// take, and the report.
#include "engine.hpp"
#include "long.cuh"

namespace sxe {


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
  // Each launch lasts about its longest chain (rows x columns of its
  // longest pair); the launches go longest first to the least-loaded
  // auxiliary stream, so the long bins start at once and the short ones
  // queue behind other short ones
  std::vector<double> load(S.hi.naux, 0.0);
  auto pick_stream = [&](double est) {
    const int a = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    load[a] += est;
    return S.hi.aux[a];
  };
  std::vector<std::pair<double, int>> order;
  for (int b = 0; b < kNumVbins; b++) {
    if (!cnt[b]) continue;
    int64_t longest = 0;
    for (size_t i : byb[b]) longest = std::max<int64_t>(longest, T->len[pairs[i].t]);
    order.emplace_back((double)longest * kVcBins[b], b);
  }
  std::stable_sort(order.begin(), order.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
  fork_aux(S.hi);
  for (const auto& ob : order) {
    const int b = ob.second;
    // The row passes are latency-bound chains that run for milliseconds
    // beside the next block's MSV: packed kRowsWarps to a CTA they hold the
    // registers of a few SMs instead of one MSV CTA slot on nearly every SM.
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)cnt[b] + kRowsWarps - 1) / kRowsWarps,
                                                                   (int64_t)E->num_sms * 32 / kRowsWarps));
    cudaStream_t sa = pick_stream(ob.first), sb = pick_stream(ob.first);
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
                unsigned* counts, const unsigned* rcount, unsigned rcap, int p0) {
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
    // widest bins first, each to the least-loaded auxiliary stream: a bin's
    // launch lasts about its longest row chain, which grows with the width
    const int nb = si == 1 ? kNumVitShapes : kNumVbins;
    std::vector<std::pair<int, int>> order;  // (columns, bin)
    for (int b = 0; b < nb; b++)
      if (nin[b]) order.emplace_back(si == 1 ? kVitShapes[b].g * kVitShapes[b].c : 32 * kVcBins[b], b);
    std::stable_sort(order.begin(), order.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    std::vector<double> load(S.hi.naux, 0.0);
    for (const auto& ob : order) {
      const int b = ob.second;
      const int a = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      load[a] += (double)ob.first;
      cudaStream_t s = S.hi.aux[a];
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
// profile's list is cut into strided sub-tiles of about 24 rounds of the
// pairs a CTA holds at once (with 6 a CTA's slot idles behind its longest
// target too often: 69 ms against 59), larger M first, one launch per shape on the
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
    const unsigned per = 24u * (unsigned)(vit16_threads(v) / 32) * (unsigned)(32 / v.g) * 2u;  // pairs per sub-tile
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
void long_rows(sx_engine* E, const sx_profiles* P, const sx_targets* T, const std::vector<sxk::LongPair>& v,
               const LongRowsSink& consume) {
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
  // four or more are smaller (0.7 and 0.4 of the others), so the work left
  // after the last MSV stage -- that block's later device stages and its
  // domain definition -- is short (Pfam-scale: 1,1,1,0.7,0.4 449 ms per
  // search; 0.6,0.3 454; 1,0.5 461; five equal blocks 487)
  std::vector<double> rel(nb, 1.0);
  if (E->pipeline_blocks <= 0 && nb >= 4) {
    rel[nb - 2] = 0.7;
    rel[nb - 1] = 0.4;
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
  std::vector<Thresholds> th;
  {
    const double key[4] = {o.filters ? 1.0 : 0.0, o.f1, o.f2, o.f3};
    std::lock_guard<std::mutex> g(P->th_mu);
    if (P->th_cache.size() != np || std::memcmp(key, P->th_key, sizeof key) != 0) {
      P->th_cache = make_thresholds(P->h, o);
      std::memcpy(P->th_key, key, sizeof key);
    }
    th = P->th_cache;
  }
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
  // with SXHMM_PROFILE: each block's milestones, milliseconds since the call began
  PhaseLog timeline;
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
  auto device_envelopes = [&](const BlockOut* B, double block_cells, bool last_of_several) {
    if (E->flags & SX_FLAG_ENV_DEVICE) return true;
    if (E->flags & SX_FLAG_ENV_HOST) return false;
    // the last block's host work is hidden behind nothing: its envelopes go
    // to the device passes, which run them all at once (Pfam-scale search
    // 461 -> 452 ms, the tail after the last device stage 49 -> 33 ms)
    if (last_of_several) return true;
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
    const size_t bi = outs.size() - 1;
    auto queue_chunk = [&, B, dev_env, bi](std::function<RowsChunk()> get) {
      hq.push([&, B, dev_env, get, bi](int nthr) {
        try {
          auto ch = std::make_shared<RowsChunk>(get());
          timeline.add("b" + std::to_string(bi) + "_rows", t_start);
          struct Done {
            PhaseLog& tl;
            size_t bi;
            std::chrono::steady_clock::time_point t0;
            ~Done() { tl.add("b" + std::to_string(bi) + "_host", t0); }
          } done{timeline, bi, t_start};
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
    timeline.add("b" + std::to_string(b) + "_cascade", t_start);
    nfinal += (int64_t)B->finals.size();
    rows_and_queue(S, B, device_envelopes(B, runs[b].cells_total, b + 1 == runs.size() && runs.size() > 1));
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
  timeline.print();
  std::vector<std::vector<std::pair<int32_t, HitOut>>> per(np);
  for (auto& B : outs) {
    for (const auto& f : B->finals) E->stats.cells[4] += (double)P->h[f.p].m * T->len[f.t];
    for (size_t i = 0; i < B->finals.size(); i++)
      if (B->res[i].hit) per[B->finals[i].p].emplace_back(B->finals[i].t, std::move(B->res[i].h));
  }
  return report(P, T, cfg, per, out);
}

}  // namespace sxe
