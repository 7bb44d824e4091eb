// TEST INFRASTRUCTURE ONLY — flat C interface to the CPU oracle so the
// Python tests and bench.py's CPU-baseline leg can drive it through ctypes.
#include <atomic>
#include <chrono>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "sx_oracle.hpp"

namespace sxo {
double forward_logspace_f64(const Profile& p, const uint8_t* dsq, size_t l, bool multihit, int kind, size_t idx,
                            double delta);
double expected_counts_f64(const Profile& p, const uint8_t* dsq, size_t l, bool multihit, double* d_msc,
                           double* d_isc, double* d_t, double* d_tbm, double* bsc);
double posterior_f64(const Profile& p, const uint8_t* dsq, size_t l, bool multihit, double* pm, double* pi);
}  // namespace sxo

using namespace sxo;

struct OrSet {
  std::vector<Hmm> hmms;
  std::vector<Profile> profiles;
};

struct OrHit {
  int32_t profile_index, target_index;
  float score, bias;
  double evalue;
  float nexpected;
  int32_t ndom, dom_offset;
};
struct OrDom {
  float score, bias;
  double c_evalue, i_evalue;
  int32_t hmm_from, hmm_to, ali_from, ali_to, env_from, env_to, reported, pad;
};
struct OrResults {
  std::vector<OrHit> hits;
  std::vector<OrDom> doms;
};
struct OrStage {  // StageTrace, flat
  float usc, filtersc, vsc, fwdsc, bcksc, nullsc;
  int32_t stage_reached, pass_f1, pass_bias, pass_f2, pass_f3, is_hit;
  float bits, bias;
  int32_t ndom, nregions;
};
struct OrCfg {
  int32_t cutoff_kind;  // 0 E, 1 bits, 2 GA, 3 NC, 4 TC
  int32_t filters, null2, has_z;
  double seq, dom, f1, f2, f3, z;
};

static thread_local std::string g_err;

static void make_targets(int64_t nt, const uint8_t* seq, const int64_t* off, const int64_t* len, Targets& t) {
  t.ids.resize((size_t)nt);
  t.dsq.resize((size_t)nt);
  for (int64_t i = 0; i < nt; i++) {
    t.ids[i] = std::to_string(i);
    t.dsq[i].assign(seq + off[i], seq + off[i] + len[i]);
  }
}
static SearchConfig make_cfg(const OrCfg* c) {
  SearchConfig s;
  s.cutoff.kind = (CutoffKind)c->cutoff_kind;
  s.cutoff.seq = c->seq;
  s.cutoff.dom = c->dom;
  s.pipeline.filters = c->filters != 0;
  s.pipeline.null2 = c->null2 != 0;
  s.pipeline.f1 = c->f1;
  s.pipeline.f2 = c->f2;
  s.pipeline.f3 = c->f3;
  if (c->has_z) s.z = c->z;
  return s;
}

extern "C" {

const char* or_last_error() { return g_err.c_str(); }

OrSet* or_load_text(const char* text, int64_t n, const char* source) {
  auto* s = new OrSet;
  if (!parse_hmm_text(std::string(text, (size_t)n), source ? source : "<stream>", s->hmms, g_err)) {
    delete s;
    return nullptr;
  }
  for (auto& h : s->hmms) s->profiles.push_back(configure(h));
  return s;
}
OrSet* or_load_file(const char* path) {
  auto* s = new OrSet;
  if (!parse_hmm_path(path, s->hmms, g_err)) {
    delete s;
    return nullptr;
  }
  for (auto& h : s->hmms) s->profiles.push_back(configure(h));
  return s;
}
void or_free(OrSet* s) { delete s; }
int32_t or_count(const OrSet* s) { return (int32_t)s->profiles.size(); }
int32_t or_m(const OrSet* s, int32_t i) { return (int32_t)s->profiles[i].m; }
const char* or_name(const OrSet* s, int32_t i) { return s->profiles[i].name.c_str(); }
// Header fields: ga/tc/nc (seq,dom; NaN if absent) and stats (mu/tau, lambda; NaN if absent)
void or_header(const OrSet* s, int32_t i, float* cut6, double* stats6) {
  const Profile& p = s->profiles[i];
  const std::optional<std::pair<float, float>>* c[3] = {&p.ga, &p.tc, &p.nc};
  for (int q = 0; q < 3; q++) {
    cut6[2 * q] = *c[q] ? (*c[q])->first : NAN;
    cut6[2 * q + 1] = *c[q] ? (*c[q])->second : NAN;
  }
  const std::optional<std::pair<double, double>>* st[3] = {&p.stats.msv, &p.stats.viterbi, &p.stats.forward};
  for (int q = 0; q < 3; q++) {
    stats6[2 * q] = *st[q] ? (*st[q])->first : NAN;
    stats6[2 * q + 1] = *st[q] ? (*st[q])->second : NAN;
  }
}
// Configured profile arrays: msc/mo (25*(M+1)), t (8*(M+1): mm mi md im ii dm dd bm), p (8*(M+1)), msv_tbm
void or_profile_arrays(const OrSet* s, int32_t i, float* msc, float* mo, float* t8, float* p8, float* msv_tbm,
                       float* compo) {
  const Profile& p = s->profiles[i];
  const size_t w = p.m + 1;
  std::memcpy(msc, p.msc.data(), sizeof(float) * NCODE * w);
  std::memcpy(mo, p.mo.data(), sizeof(float) * NCODE * w);
  const std::vector<float>* tv[8] = {&p.t_mm, &p.t_mi, &p.t_md, &p.t_im, &p.t_ii, &p.t_dm, &p.t_dd, &p.t_bm};
  const std::vector<float>* pv[8] = {&p.p_mm, &p.p_mi, &p.p_md, &p.p_im, &p.p_ii, &p.p_dm, &p.p_dd, &p.p_bm};
  for (int q = 0; q < 8; q++) {
    std::memcpy(t8 + q * w, tv[q]->data(), sizeof(float) * w);
    std::memcpy(p8 + q * w, pv[q]->data(), sizeof(float) * w);
  }
  *msv_tbm = p.msv_tbm;
  std::memcpy(compo, p.compo.data(), sizeof(float) * K);
}

int64_t or_encode(const char* s, int64_t n, uint8_t* out) {
  auto v = encode(std::string(s, (size_t)n));
  std::memcpy(out, v.data(), v.size());
  return (int64_t)v.size();
}

float or_msv(const OrSet* s, int32_t pi, const uint8_t* dsq, int64_t l) {
  DpBuf b;
  return msv(s->profiles[pi], dsq, (size_t)l, b);
}
float or_viterbi(const OrSet* s, int32_t pi, const uint8_t* dsq, int64_t l) {
  DpBuf b;
  return viterbi_score(s->profiles[pi], dsq, (size_t)l, Xsc::make((size_t)l, true), b);
}
// Forward (multihit, target-length config). If sp5 != null it receives the
// specials N,B,E,J,C rows (5*(L+1)).
float or_forward(const OrSet* s, int32_t pi, const uint8_t* dsq, int64_t l, float* sp5) {
  DpBuf b;
  Specials sp;
  float r = forward(s->profiles[pi], dsq, (size_t)l, Xsc::make((size_t)l, true), b, sp5 ? &sp : nullptr);
  if (sp5) {
    const std::vector<float>* v[5] = {&sp.n, &sp.b, &sp.e, &sp.j, &sp.c};
    for (int q = 0; q < 5; q++) std::memcpy(sp5 + q * (l + 1), v[q]->data(), sizeof(float) * (l + 1));
  }
  return r;
}
float or_backward(const OrSet* s, int32_t pi, const uint8_t* dsq, int64_t l, float* sp5) {
  DpBuf b;
  Specials sp;
  float r = backward(s->profiles[pi], dsq, (size_t)l, Xsc::make((size_t)l, true), b, sp);
  if (sp5) {
    const std::vector<float>* v[5] = {&sp.n, &sp.b, &sp.e, &sp.j, &sp.c};
    for (int q = 0; q < 5; q++) std::memcpy(sp5 + q * (l + 1), v[q]->data(), sizeof(float) * (l + 1));
  }
  return r;
}
float or_bias(const OrSet* s, int32_t pi, const uint8_t* dsq, int64_t l) {
  return bias_filter_score(s->profiles[pi], dsq, (size_t)l);
}
float or_null(int64_t l) { return null_score((size_t)l); }
void or_xsc(int64_t l, int32_t multihit, float* out16) {
  Xsc x = Xsc::make((size_t)l, multihit != 0);
  float v[16] = {x.n_loop, x.n_move, x.j_loop, x.j_move, x.c_loop, x.c_move, x.e_move, x.e_loop,
                 x.p.n_loop, x.p.n_move, x.p.j_loop, x.p.j_move, x.p.c_loop, x.p.c_move, x.p.e_move, x.p.e_loop};
  std::memcpy(out16, v, sizeof v);
}
double or_gumbel_surv(double x, double mu, double lam) { return gumbel_surv(x, mu, lam); }
double or_exp_logsurv(double x, double tau, double lam) { return exp_logsurv(x, tau, lam); }
float or_logsum(float a, float b) { return logsum(a, b); }

// Full pipeline for one pair, with the stage record.
void or_score_pair(const OrSet* s, int32_t pi, const uint8_t* dsq, int64_t l, const OrCfg* c, OrStage* out) {
  Workspace ws;
  StageTrace tr;
  SearchConfig sc = make_cfg(c);
  auto h = score_target(s->profiles[pi], dsq, (size_t)l, sc.pipeline, ws, &tr);
  out->usc = tr.usc; out->filtersc = tr.filtersc; out->vsc = tr.vsc; out->fwdsc = tr.fwdsc;
  out->bcksc = tr.bcksc; out->nullsc = tr.nullsc; out->stage_reached = tr.stage_reached;
  out->pass_f1 = tr.pass_f1; out->pass_bias = tr.pass_bias; out->pass_f2 = tr.pass_f2; out->pass_f3 = tr.pass_f3;
  out->is_hit = h.has_value();
  out->bits = h ? h->bits : NAN;
  out->bias = h ? h->bias : NAN;
  out->ndom = h ? (int32_t)h->domains.size() : 0;
  out->nregions = h ? (int32_t)h->nregions : 0;
}

OrResults* or_search(const OrSet* s, int64_t nt, const uint8_t* seq, const int64_t* off, const int64_t* len,
                     const OrCfg* c, int32_t nthreads) {
  Targets t;
  make_targets(nt, seq, off, len, t);
  std::vector<Hit> hits;
  if (!search_profiles(s->profiles, t, make_cfg(c), nthreads, hits, g_err)) return nullptr;
  auto* r = new OrResults;
  std::vector<int32_t> pidx;
  for (auto& h : hits) {
    int32_t p = 0;
    for (size_t q = 0; q < s->profiles.size(); q++)
      if (s->profiles[q].name == h.profile) { p = (int32_t)q; break; }
    OrHit oh{p, (int32_t)h.target_index, h.score, h.bias, h.evalue, h.nexpected, (int32_t)h.domains.size(),
             (int32_t)r->doms.size()};
    r->hits.push_back(oh);
    for (auto& d : h.domains)
      r->doms.push_back({d.score, d.bias, d.c_evalue, d.i_evalue, (int32_t)d.hmm_from, (int32_t)d.hmm_to,
                         (int32_t)d.ali_from, (int32_t)d.ali_to, (int32_t)d.env_from, (int32_t)d.env_to,
                         (int32_t)d.reported, 0});
  }
  return r;
}
int64_t or_results_nhits(const OrResults* r) { return (int64_t)r->hits.size(); }
int64_t or_results_ndoms(const OrResults* r) { return (int64_t)r->doms.size(); }
void or_results_copy(const OrResults* r, OrHit* hits, OrDom* doms) {
  std::memcpy(hits, r->hits.data(), sizeof(OrHit) * r->hits.size());
  std::memcpy(doms, r->doms.data(), sizeof(OrDom) * r->doms.size());
}
void or_results_free(OrResults* r) { delete r; }

// Timed CPU baseline: score_target over pairs (p, t) in profile-major order
// starting at pair index `start`, on `nthreads` threads with a dynamic pair
// index, stopping once `time_limit_s` has elapsed (or all pairs are done).
// Writes pairs done, cells (sum M*L) and wall seconds.
void or_time_pairs(const OrSet* s, int64_t nt, const uint8_t* seq, const int64_t* off, const int64_t* len,
                   const OrCfg* c, int32_t nthreads, int64_t start, int64_t max_pairs, double time_limit_s,
                   int64_t* pairs_done, double* cells, double* seconds, int64_t* nhits) {
  SearchConfig sc = make_cfg(c);
  const int64_t np = (int64_t)s->profiles.size() * nt;
  const int64_t end = std::min<int64_t>(np, start + max_pairs);
  std::atomic<int64_t> next{start}, done{0}, hitc{0};
  std::atomic<double> cellsum{0.0};
  std::atomic<bool> stop{false};
  auto t0 = std::chrono::steady_clock::now();
  auto worker = [&]() {
    Workspace ws;
    double mycells = 0;
    int64_t mydone = 0, myhits = 0;
    for (;;) {
      if (stop.load(std::memory_order_relaxed)) break;
      int64_t idx = next.fetch_add(1);
      if (idx >= end) break;
      int64_t pi = idx / nt, ti = idx % nt;
      auto h = score_target(s->profiles[pi], seq + off[ti], (size_t)len[ti], sc.pipeline, ws);
      if (h) myhits++;
      mycells += (double)s->profiles[pi].m * (double)len[ti];
      mydone++;
      if ((mydone & 63) == 0) {
        double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > time_limit_s) stop = true;
      }
    }
    done += mydone;
    hitc += myhits;
    double cur = cellsum.load();
    while (!cellsum.compare_exchange_weak(cur, cur + mycells)) {}
  };
  std::vector<std::thread> th;
  for (int t = 1; t < std::max(1, nthreads); t++) th.emplace_back(worker);
  worker();
  for (auto& t : th) t.join();
  *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  *pairs_done = done.load();
  *cells = cellsum.load();
  *nhits = hitc.load();
}

// Scores of every profile x every target (profile-major) for calibration:
// msv, viterbi_score and forward, on `nthreads` threads.
void or_score_all(const OrSet* s, int64_t nt, const uint8_t* seq, const int64_t* off, const int64_t* len,
                  int32_t nthreads, float* msv_out, float* vit_out, float* fwd_out) {
  const int64_t np = (int64_t)s->profiles.size();
  std::atomic<int64_t> next{0};
  auto worker = [&]() {
    DpBuf b;
    for (;;) {
      const int64_t idx = next.fetch_add(1);
      if (idx >= np * nt) break;
      const int64_t pi = idx / nt, ti = idx % nt;
      const Profile& p = s->profiles[pi];
      const uint8_t* d = seq + off[ti];
      const size_t l = (size_t)len[ti];
      Xsc xs = Xsc::make(l, true);
      if (msv_out) msv_out[idx] = msv(p, d, l, b);
      if (vit_out) vit_out[idx] = viterbi_score(p, d, l, xs, b);
      if (fwd_out) fwd_out[idx] = forward(p, d, l, xs, b, nullptr);
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < std::max(1, nthreads); t++) th.emplace_back(worker);
  worker();
  for (auto& t : th) t.join();
}

// ---- matrices for envelope / posterior checks ----
// Full-matrix forward+backward+decode of dsq with Xsc(L_cfg, multihit): writes
// pm, pi ((L+1)*(M+1)) and pn,pj,pc (L+1) and returns the forward score.
float or_decode(const OrSet* s, int32_t pi, const uint8_t* dsq, int64_t l, int64_t l_cfg, int32_t multihit, float* pm,
                float* pii, float* pn, float* pj, float* pc, float* bsc) {
  Matrix fx, bx;
  Posterior pp;
  const Profile& p = s->profiles[pi];
  Xsc xs = Xsc::make((size_t)l_cfg, multihit != 0);
  float f = forward_matrix(p, dsq, (size_t)l, xs, fx);
  float b = backward_matrix(p, dsq, (size_t)l, xs, bx);
  if (bsc) *bsc = b;
  decode(p, xs, fx, bx, pp);
  const size_t n = ((size_t)l + 1) * (p.m + 1);
  std::memcpy(pm, pp.pm.data(), sizeof(float) * n);
  std::memcpy(pii, pp.pi.data(), sizeof(float) * n);
  std::memcpy(pn, pp.pn.data(), sizeof(float) * (l + 1));
  std::memcpy(pj, pp.pj.data(), sizeof(float) * (l + 1));
  std::memcpy(pc, pp.pc.data(), sizeof(float) * (l + 1));
  return f;
}
// viterbi_trace coordinates (max 64 domains): writes 4 ints per domain.
int32_t or_viterbi_trace(const OrSet* s, int32_t pi, const uint8_t* dsq, int64_t l, int32_t* out4, int32_t cap) {
  auto tr = viterbi_trace(s->profiles[pi], dsq, (size_t)l, Xsc::make((size_t)l, true));
  int32_t n = 0;
  for (auto& a : tr) {
    if (n >= cap) break;
    out4[4 * n] = (int32_t)a.iali; out4[4 * n + 1] = (int32_t)a.jali;
    out4[4 * n + 2] = (int32_t)a.kali; out4[4 * n + 3] = (int32_t)a.mali;
    n++;
  }
  return (int32_t)tr.size();
}

// ---- FP64 log-space yardstick ----
double or_forward_f64(const OrSet* s, int32_t pi, const uint8_t* dsq, int64_t l, int32_t multihit, int32_t kind,
                      int64_t idx, double delta) {
  return forward_logspace_f64(s->profiles[pi], dsq, (size_t)l, multihit != 0, kind, (size_t)idx, delta);
}
double or_expected_counts_f64(const OrSet* s, int32_t pi, const uint8_t* dsq, int64_t l, int32_t multihit,
                              double* d_msc, double* d_isc, double* d_t, double* d_tbm, double* bsc) {
  return expected_counts_f64(s->profiles[pi], dsq, (size_t)l, multihit != 0, d_msc, d_isc, d_t, d_tbm, bsc);
}
double or_posterior_f64(const OrSet* s, int32_t pi, const uint8_t* dsq, int64_t l, int32_t multihit, double* pm,
                        double* pii) {
  return posterior_f64(s->profiles[pi], dsq, (size_t)l, multihit != 0, pm, pii);
}

}  // extern "C"
