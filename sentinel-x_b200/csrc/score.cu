// C ABI: stage scores, pre-screen bounds and the adjoint for explicit pairs.
#include "engine.hpp"
#include "long.cuh"

extern "C" {

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
