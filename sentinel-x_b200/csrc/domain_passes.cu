// The device passes of host domain definition, run after a search's cascade:
// envelope rescoring (full-matrix Forward/Backward, then posterior, null2 and
// optimal accuracy) and the stochastic-trace ensembles of multi-domain regions.
#include "engine.hpp"

namespace sxe {

// The per-bin launches of a pass fan out over the two slots' high-priority
// auxiliary streams, idle once the cascade is done: a launch holds only as
// many warps as its bin has envelopes (tens), and on one stream the bins of a
// pass would run one after another -- the pass taking the sum of its bins'
// longest chains instead of the largest one.
struct FanOut {
  sx_engine* E;
  cudaStream_t origin;
  std::vector<cudaStream_t> lanes;
  size_t next = 0;
  FanOut(sx_engine* e, cudaStream_t s) : E(e), origin(s) {
    CK(cudaEventRecord(E->env_ev, s));
    for (Slot& S : E->sl) {
      CK(cudaStreamWaitEvent(S.hi.main, E->env_ev, 0));
      fork_aux(S.hi);
      for (int a = 0; a < S.hi.naux; a++) lanes.push_back(S.hi.aux[a]);
    }
  }
  cudaStream_t take() { return lanes[next++ % lanes.size()]; }
  // the origin stream waits for every launch made
  void join() {
    for (Slot& S : E->sl) {
      join_aux(S.hi);
      CK(cudaEventRecord(E->env_ev, S.hi.main));
      CK(cudaStreamWaitEvent(origin, E->env_ev, 0));
    }
  }
};

// The device passes of a DomainBatch: for every envelope request the
// full-matrix Forward and Backward (their raw special rows come back to the
// host), the host's posterior factors, then the posterior / null2 /
// optimal-accuracy pass.  One warp per envelope; batches bounded by the
// memory of their matrix planes.  Runs on the host pool's driver thread.
int64_t envelope_passes(sx_engine* E, const sx_profiles* P, const sx_targets* T, std::vector<EnvSource>& srcs,
                        int nthr, PhaseLog* plog) {
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
    // Forward and Backward of every bin at once, each launch on a stream of its own
    {
      FanOut fan(E, s);
      each_bin([&](int vb, int x0, int cnt, int blocks) {
        K.envf[vb]<<<blocks, 32, 0, fan.take()>>>(E->env_recs.p + x0, cnt, P->d_prof.p, P->d_vfb.p, T->d_res.p,
                                                  T->d_off.p, E->env_planes.p, E->env_rows.p);
        K.envb[vb]<<<blocks, 32, 0, fan.take()>>>(E->env_recs.p + x0, cnt, P->d_prof.p, P->d_vfb.p, T->d_res.p,
                                                  T->d_off.p, E->env_planes.p, E->env_rows.p);
        launches += 2;
      });
      CK(cudaGetLastError());
      fan.join();
    }
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
    FanOut fan(E, s);
    each_bin([&](int vb, int x0, int cnt, int blocks) {
      const size_t psm = sxk::env_post_smem(kVcBins[vb]);
      CK(cudaFuncSetAttribute((const void*)K.envp[vb], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm));
      K.envp[vb]<<<blocks, 32, psm, fan.take()>>>(E->env_recs.p + x0, cnt, P->d_prof.p, P->d_vfb.p, E->env_planes.p,
                                       E->env_aux.p, E->env_fac.p, E->env_out.p);
      launches += 1;
    });
    CK(cudaGetLastError());
    fan.join();
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
    // vbin) on streams of their own, then one trace launch over the batch
    FanOut fan(E, s);
    for (size_t x = 0; x < n;) {
      const int vb = P->dp[reg(order[a + x]).p].vbin;
      size_t y = x;
      while (y < n && P->dp[reg(order[a + y]).p].vbin == vb) y++;
      const int cnt = (int)(y - x);
      K.regf[vb]<<<(int)std::min<int64_t>(cnt, (int64_t)E->num_sms * 32), 32, 0, fan.take()>>>(
          E->env_recs.p + x, cnt, P->d_prof.p, P->d_vfb.p, T->d_res.p, T->d_off.p, E->env_planes.p, E->env_rows.p);
      st.launches += 1;
      x = y;
    }
    CK(cudaGetLastError());
    fan.join();
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

}  // namespace sxe
