// Host-side domain definition for the sxhmm engine: everything in
// score_target after the Backward pass (src/hmmer/pipeline.rs:187-293), for the
// few pairs that survive the device cascade.
//
// Inputs are the device's raw Forward/Backward special rows (scaled values and
// per-row rescale factors); this file turns them into log-space rows with the
// same libm calls the reference makes, then runs posterior decoding, the
// rt1/rt2/rt3 region heuristics, envelope rescoring (full-matrix Forward,
// Backward, posterior decoding, null2 by expectation, optimal-accuracy
// coordinates with a Viterbi-trace fallback), the 200-sample stochastic-trace
// clustering of multi-domain regions and the final bit scores.  Every f32/f64
// operation is in the reference's order, so results are bit-identical to it.
#include <algorithm>
#include <cassert>
#include <cstring>
#include <optional>

#include "internal.hpp"

namespace sx {
namespace {

constexpr float kRescale = 1.0e4f;

inline float lnpos(float x) { return x > 0.0f ? std::log(x) : kNegInf; }
inline float fmax_gt(float a, float b) { return a > b ? a : b; }

float logsum2(float a, float b) {  // ln(e^a + e^b), src/hmmer/dp.rs:32-40
  float hi = a > b ? a : b, lo = a > b ? b : a;
  float d = hi - lo;
  if (!(d < 30.0f)) return hi;
  return hi + std::log1p(std::exp(-d));
}

// Log-space special rows N B E J C, rows 0..L.
struct LogRows {
  std::vector<float> n, b, e, j, c;
  void reset(int64_t l) {
    for (auto* v : {&n, &b, &e, &j, &c}) v->assign((size_t)l + 1, kNegInf);
  }
};

// Full probability-space DP matrix of one envelope (rows 0..Lr, cols 0..M).
struct Mat {
  int m = 0;
  int64_t l = 0;
  std::vector<float> mm, im, dm;
  std::vector<double> lnscale;
  LogRows sp;
  std::vector<float> xn, xb, xe, xj, xc, scale;
  void reset(int m_, int64_t l_) {
    m = m_;
    l = l_;
    const size_t n = (size_t)(l + 1) * (size_t)(m + 1);
    for (auto* v : {&mm, &im, &dm}) v->assign(n, 0.0f);
    lnscale.assign((size_t)l + 2, 0.0);
    sp.reset(l);
    for (auto* v : {&xn, &xb, &xe, &xj, &xc}) v->assign((size_t)l + 1, 0.0f);
    scale.assign((size_t)l + 1, 1.0f);
  }
};

struct Post {
  int m = 0;
  int64_t l = 0;
  std::vector<float> pm, pi, pn, pj, pc;
};

struct Coords {
  int64_t i0, i1;
  int k0, k1;
};

// Easel's fast LCG seeded through esl_mix3 (src/hmmer/dp.rs:965-1023).
class Lcg {
 public:
  explicit Lcg(uint32_t seed) : seed_(seed) { reset(); }
  void reset() {
    uint32_t a = seed_, b = 87654321u, c = 12345678u;
    a -= b; a -= c; a ^= c >> 13;
    b -= c; b -= a; b ^= a << 8;
    c -= a; c -= b; c ^= b >> 13;
    a -= b; a -= c; a ^= c >> 12;
    b -= c; b -= a; b ^= a << 16;
    c -= a; c -= b; c ^= b >> 5;
    a -= b; a -= c; a ^= c >> 3;
    b -= c; b -= a; b ^= a << 10;
    c -= a; c -= b; c ^= b >> 15;
    x_ = c ? c : 42u;
  }
  double uniform() {
    x_ = x_ * 69069u + 1u;
    return (double)x_ / 4294967296.0;
  }
  uint32_t state() const { return x_; }

 private:
  uint32_t seed_, x_ = 0;
};

// esl_vec_FNorm (Kahan sum) then esl_rnd_FChoose (src/hmmer/dp.rs:1026-1059).
template <int N>
int choose(Lcg& rng, float (&v)[N]) {
  float s = 0.0f, comp = 0.0f;
  for (int i = 0; i < N; i++) {
    float y = v[i] - comp;
    float t = s + y;
    comp = (t - s) - y;
    s = t;
  }
  if (s != 0.0f)
    for (int i = 0; i < N; i++) v[i] /= s;
  else
    for (int i = 0; i < N; i++) v[i] = 1.0f / (float)N;
  double norm = 0.0;
  for (int i = 0; i < N; i++) norm += (double)v[i];
  const double roll = rng.uniform();
  double acc = 0.0;
  for (int i = 0; i < N; i++) {
    acc += (double)v[i];
    if (roll < acc / norm) return i;
  }
  return N - 1;
}

struct Sampled {
  int64_t sqfrom = 0, sqto = 0;
  int hmmfrom = 0, hmmto = 0;
  std::vector<int> nodes;
};

struct Sample {  // p7_spcoord_s
  size_t trace;
  int64_t i, j;
  int k, m;
};

// Full-matrix workspaces of envelope rescoring: one set per thread, reused by
// every EnvelopeScorer the thread creates (a fresh set per pair faulted in
// megabytes of new pages every time).  Each use re-initialises what it reads,
// and a thread runs one scorer at a time; `in_use` checks that last point
// (a scorer constructed while another one of the same thread is alive would
// share, and overwrite, its matrices).
struct ScorerWork {
  Mat fx, bx;
  Post pp;
  std::vector<float> om, oi, od;
  bool in_use = false;
};
// Claims the thread's workspace for the lifetime of one EnvelopeScorer.
struct WorkClaim {
  ScorerWork& w;
  explicit WorkClaim(ScorerWork& ws) : w(ws) {
    assert(!w.in_use && "two EnvelopeScorer objects alive on one thread");
    w.in_use = true;
  }
  ~WorkClaim() { w.in_use = false; }
  WorkClaim(const WorkClaim&) = delete;
  WorkClaim& operator=(const WorkClaim&) = delete;
};
ScorerWork& scorer_work() {
  thread_local ScorerWork w;
  return w;
}

class EnvelopeScorer {
 public:
  EnvelopeScorer(const ProfileHost& p, const uint8_t* dsq, int64_t l, const SearchOpts& o)
      : p_(p), dsq_(dsq), l_(l), o_(o), w_((size_t)p.m + 1) {}

  // Full-matrix Forward of sub[0..lr) with special transitions `st`
  // (src/hmmer/dp.rs:442-513).
  float forward_full(const uint8_t* sub, int64_t lr, const SpecialTr& st, Mat& fx) {
    const int m = p_.m;
    fx.reset(m, lr);
    if (lr == 0 || m == 0) return kNegInf;
    float xn = 1.0f, xb = st.pmove, xj = 0.0f, xc = 0.0f;
    double lnscale = 0.0;
    fx.sp.n[0] = 0.0f;
    fx.sp.b[0] = lnpos(xb);
    fx.xn[0] = xn;
    fx.xb[0] = xb;
    const float *pbm = p_.p[TBM].data(), *pmm = p_.p[TMM].data(), *pim = p_.p[TIM].data(), *pdm = p_.p[TDM].data();
    const float *pmi = p_.p[TMI].data(), *pii = p_.p[TII].data(), *pmd = p_.p[TMD].data(), *pdd = p_.p[TDD].data();
    for (int64_t i = 1; i <= lr; i++) {
      const uint8_t x = sub[i - 1];
      const float* eo = p_.mo_row(x);
      const float ins = x != SYM_STAR ? 1.0f : 0.0f;
      float* mc = &fx.mm[(size_t)i * w_];
      float* ic = &fx.im[(size_t)i * w_];
      float* dc = &fx.dm[(size_t)i * w_];
      const float* mp = mc - w_;
      const float* ip = ic - w_;
      const float* dp = dc - w_;
      float xe = 0.0f;
      for (int k = 1; k <= m; k++) {
        float mv = (xb * pbm[k] + mp[k - 1] * pmm[k - 1] + ip[k - 1] * pim[k - 1] + dp[k - 1] * pdm[k - 1]) * eo[k];
        mc[k] = mv;
        ic[k] = k < m ? (mp[k] * pmi[k] + ip[k] * pii[k]) * ins : 0.0f;
        float dv = mc[k - 1] * pmd[k - 1] + dc[k - 1] * pdd[k - 1];
        dc[k] = dv;
        xe += mv + dv;
      }
      xj = xj * st.ploop + xe * st.pe_loop;
      xc = xc * st.ploop + xe * st.pe_move;
      xn *= st.ploop;
      xb = xn * st.pmove + xj * st.pmove;
      if (xe > kRescale) {
        const float inv = 1.0f / xe;
        for (int k = 1; k <= m; k++) {
          mc[k] *= inv;
          ic[k] *= inv;
          dc[k] *= inv;
        }
        xn *= inv;
        xb *= inv;
        xj *= inv;
        xc *= inv;
        lnscale += std::log((double)xe);
        fx.scale[i] = xe;
        xe = 1.0f;
      }
      fx.xn[i] = xn; fx.xb[i] = xb; fx.xe[i] = xe; fx.xj[i] = xj; fx.xc[i] = xc;
      fx.lnscale[i] = lnscale;
      const float ls = (float)lnscale;
      fx.sp.n[i] = lnpos(xn) + ls; fx.sp.b[i] = lnpos(xb) + ls; fx.sp.e[i] = lnpos(xe) + ls;
      fx.sp.j[i] = lnpos(xj) + ls; fx.sp.c[i] = lnpos(xc) + ls;
    }
    return (float)((double)lnpos(xc * st.pmove) + lnscale);
  }

  // Full-matrix Backward (src/hmmer/dp.rs:516-601).
  float backward_full(const uint8_t* sub, int64_t lr, const SpecialTr& st, Mat& bx) {
    const int m = p_.m;
    bx.reset(m, lr);
    if (lr == 0 || m == 0) return kNegInf;
    const float *pbm = p_.p[TBM].data(), *pmm = p_.p[TMM].data(), *pim = p_.p[TIM].data(), *pdm = p_.p[TDM].data();
    const float *pmi = p_.p[TMI].data(), *pii = p_.p[TII].data(), *pmd = p_.p[TMD].data(), *pdd = p_.p[TDD].data();
    float xc = st.pmove;
    float xe = xc * st.pe_move;
    float xj = 0.0f, xn = 0.0f;
    {
      float* mL = &bx.mm[(size_t)lr * w_];
      float* dL = &bx.dm[(size_t)lr * w_];
      mL[m] = xe;
      dL[m] = xe;
      for (int k = m - 1; k >= 1; k--) {
        mL[k] = xe + dL[k + 1] * pmd[k];
        dL[k] = xe + dL[k + 1] * pdd[k];
      }
    }
    double lnscale = 0.0;
    bx.lnscale[lr] = 0.0;
    bx.sp.c[lr] = lnpos(xc);
    bx.sp.e[lr] = lnpos(xe);
    for (int64_t i = lr - 1; i >= 1; i--) {
      const uint8_t xnext = sub[i];
      const float* eo = p_.mo_row(xnext);
      const float ins = xnext != SYM_STAR ? 1.0f : 0.0f;
      const float* mn = &bx.mm[(size_t)(i + 1) * w_];
      const float* in = &bx.im[(size_t)(i + 1) * w_];
      float* mc = &bx.mm[(size_t)i * w_];
      float* ic = &bx.im[(size_t)i * w_];
      float* dc = &bx.dm[(size_t)i * w_];
      float xb = 0.0f;
      for (int k = 1; k <= m; k++) xb += mn[k] * pbm[k] * eo[k];
      xj = xj * st.ploop + xb * st.pmove;
      xc *= st.ploop;
      xe = xj * st.pe_loop + xc * st.pe_move;
      xn = xn * st.ploop + xb * st.pmove;
      mc[m] = xe;
      dc[m] = xe;
      ic[m] = 0.0f;
      float rowmax = std::fmax(std::fmax(std::fmax(std::fmax(xb, xe), xn), xj), xc);
      for (int k = m - 1; k >= 1; k--) {
        const float mnext = mn[k + 1] * eo[k + 1];
        const float iv = in[k] * ins;
        const float mv = mnext * pmm[k] + iv * pmi[k] + xe + dc[k + 1] * pmd[k];
        mc[k] = mv;
        ic[k] = mnext * pim[k] + iv * pii[k];
        dc[k] = mnext * pdm[k] + dc[k + 1] * pdd[k] + xe;
        if (mv > rowmax) rowmax = mv;
      }
      if (rowmax > kRescale) {
        const float inv = 1.0f / rowmax;
        for (int k = 1; k <= m; k++) {
          mc[k] *= inv;
          ic[k] *= inv;
          dc[k] *= inv;
        }
        xb *= inv;
        xe *= inv;
        xn *= inv;
        xj *= inv;
        xc *= inv;
        lnscale += std::log((double)rowmax);
      }
      bx.lnscale[i] = lnscale;
      const float ls = (float)lnscale;
      bx.sp.n[i] = lnpos(xn) + ls; bx.sp.b[i] = lnpos(xb) + ls; bx.sp.e[i] = lnpos(xe) + ls;
      bx.sp.j[i] = lnpos(xj) + ls; bx.sp.c[i] = lnpos(xc) + ls;
    }
    const float* eo = p_.mo_row(sub[0]);
    const float* m1 = &bx.mm[w_];
    float b = 0.0f;
    for (int k = 1; k <= m; k++) b += m1[k] * pbm[k] * eo[k];
    bx.lnscale[0] = lnscale;
    bx.sp.b[0] = lnpos(b) + (float)lnscale;
    bx.sp.n[0] = logsum2(bx.sp.n[1] + st.loop, bx.sp.b[0] + st.move);
    return bx.sp.n[0];
  }

  // Posterior decoding (src/hmmer/dp.rs:1278-1306).
  void posterior(const SpecialTr& st, const Mat& fx, const Mat& bx, Post& pp) {
    const int m = p_.m;
    const int64_t l = fx.l;
    pp.m = m;
    pp.l = l;
    pp.pm.assign((size_t)(l + 1) * w_, 0.0f);
    pp.pi.assign((size_t)(l + 1) * w_, 0.0f);
    for (auto* v : {&pp.pn, &pp.pj, &pp.pc}) v->assign((size_t)l + 1, 0.0f);
    const double overall = (double)bx.sp.n[0];
    for (int64_t i = 1; i <= l; i++) {
      const size_t row = (size_t)i * w_;
      const double fac = std::exp(fx.lnscale[i] + bx.lnscale[i] - overall);
      for (int k = 1; k <= m; k++) {
        pp.pm[row + k] = (float)((double)fx.mm[row + k] * (double)bx.mm[row + k] * fac);
        if (k < m) pp.pi[row + k] = (float)((double)fx.im[row + k] * (double)bx.im[row + k] * fac);
      }
      pp.pn[i] = (float)std::exp((double)(fx.sp.n[i - 1] + bx.sp.n[i] + st.loop) - overall);
      pp.pj[i] = (float)std::exp((double)(fx.sp.j[i - 1] + bx.sp.j[i] + st.loop) - overall);
      pp.pc[i] = (float)std::exp((double)(fx.sp.c[i - 1] + bx.sp.c[i] + st.loop) - overall);
    }
  }

  // ln null2 odds by posterior expectation (src/hmmer/dp.rs:1310-1350).
  void null2_posterior(const Post& pp, float out[NSYM]) {
    const int m = p_.m;
    const int64_t l = pp.l;
    std::vector<float> sm(w_, 0.0f);
    float si = 0.0f, sn = 0.0f, sj = 0.0f, sc = 0.0f;
    for (int64_t i = 1; i <= l; i++) {
      const size_t row = (size_t)i * w_;
      for (int k = 1; k <= m; k++) {
        sm[k] += pp.pm[row + k];
        si += pp.pi[row + k];
      }
      sn += pp.pn[i];
      sj += pp.pj[i];
      sc += pp.pc[i];
    }
    const float norm = 1.0f / (float)std::max<int64_t>(l, 1);
    const float xfactor = sn * norm + sc * norm + sj * norm;
    const float isum = si * norm;
    float n2[NSYM];
    for (int x = 0; x < NRES; x++) {
      const float* row = p_.mo_row(x);
      float v = 0.0f;
      for (int k = 1; k <= m; k++) v += sm[k] * norm * row[k];
      n2[x] = v + isum + xfactor;
    }
    average_degenerate(n2);
    for (int x = 0; x < NSYM; x++) out[x] = n2[x] > 0.0f ? std::log(n2[x]) : kNegInf;
  }

  static void average_degenerate(float* n2) {  // esl_abc_FAvgScVec
    for (int code = 20; code <= 23; code++) {
      const Degenerate& d = degenerate(code);
      float s = 0.0f;
      for (int q = 0; q < d.n; q++) s += n2[d.members[q]];
      n2[code] = s / (float)d.n;
    }
    n2[SYM_STAR] = 1.0f;
  }

  // Optimal-accuracy alignment coordinates (src/hmmer/dp.rs:1355-1564).
  std::optional<Coords> oa_coords(const SpecialTr& st, const Post& pp) {
    const int m = p_.m;
    const int64_t l = pp.l;
    if (l == 0 || m == 0) return std::nullopt;
    const size_t n = (size_t)(l + 1) * w_;
    om_.assign(n, kNegInf);
    oi_.assign(n, kNegInf);
    od_.assign(n, kNegInf);
    std::vector<float> xe(l + 1, kNegInf), xn(l + 1, kNegInf), xj(l + 1, kNegInf), xb(l + 1, kNegInf),
        xc(l + 1, kNegInf);
    xn[0] = 0.0f;
    xb[0] = 0.0f;
    const float *pbm = p_.p[TBM].data(), *pmm = p_.p[TMM].data(), *pim = p_.p[TIM].data(), *pdm = p_.p[TDM].data();
    const float *pmi = p_.p[TMI].data(), *pii = p_.p[TII].data(), *pmd = p_.p[TMD].data(), *pdd = p_.p[TDD].data();
    auto gate = [](float t, float v) { return t > 0.0f ? v : 0.0f; };
    for (int64_t i = 1; i <= l; i++) {
      const size_t pr = (size_t)(i - 1) * w_, cr = (size_t)i * w_;
      float emax = kNegInf;
      for (int k = 1; k <= m; k++) {
        float sv = gate(pbm[k], xb[i - 1]);
        if (k >= 2) {
          sv = std::fmax(sv, gate(pmm[k - 1], om_[pr + k - 1]));
          sv = std::fmax(sv, gate(pim[k - 1], oi_[pr + k - 1]));
          sv = std::fmax(sv, gate(pdm[k - 1], od_[pr + k - 1]));
        } else {
          sv = std::fmax(sv, 0.0f);
        }
        const float mv = sv + pp.pm[cr + k];
        om_[cr + k] = mv;
        emax = std::fmax(emax, mv);
        oi_[cr + k] = std::fmax(gate(pmi[k], om_[pr + k]), gate(pii[k], oi_[pr + k])) + pp.pi[cr + k];
      }
      od_[cr + 1] = kNegInf;
      for (int k = 2; k <= m; k++) {
        od_[cr + k] = std::fmax(gate(pmd[k - 1], om_[cr + k - 1]), gate(pdd[k - 1], od_[cr + k - 1]));
        emax = std::fmax(emax, od_[cr + k]);
      }
      xe[i] = emax;
      float t1 = st.ploop == 0.0f ? 0.0f : xj[i - 1] + pp.pj[i];
      float t2 = st.pe_loop == 0.0f ? 0.0f : xe[i];
      xj[i] = std::fmax(t1, t2);
      t1 = st.ploop == 0.0f ? 0.0f : xc[i - 1] + pp.pc[i];
      t2 = st.pe_move == 0.0f ? 0.0f : xe[i];
      xc[i] = std::fmax(t1, t2);
      xn[i] = st.ploop == 0.0f ? 0.0f : xn[i - 1] + pp.pn[i];
      t1 = st.pmove == 0.0f ? 0.0f : xn[i];
      t2 = st.pmove == 0.0f ? 0.0f : xj[i];
      xb[i] = std::fmax(t1, t2);
    }
    // traceback
    enum S { SC, SE, SM, SI, SD, SB, SJ, SN } s0 = SC;
    const int q_stripes = std::max(2, (m - 1) / 4 + 1);
    int64_t i = l;
    int k = 0;
    bool got_first = false, got_last = false;
    Coords cd{0, 0, 0, 0};
    const size_t limit = 8 * (size_t)(l + 2) * (size_t)(m + 2) + 64;
    auto dis = [](float t, float v) { return t == 0.0f ? kNegInf : v; };
    for (size_t guard = 1; guard <= limit; guard++) {
      S s1;
      if (s0 == SC) {
        if (i == 0) break;
        const float a = st.ploop == 0.0f ? kNegInf : xc[i - 1] + pp.pc[i];
        const float b = st.pe_move == 0.0f ? kNegInf : xe[i];
        s1 = a > b ? SC : SE;
      } else if (s0 == SE) {
        const size_t row = (size_t)i * w_;
        float mx = kNegInf;
        int pick = 0;
        S pst = SM;
        for (int q = 0; q < q_stripes; q++) {
          for (int r = 0; r < 4; r++) {
            const int kk = r * q_stripes + q + 1;
            if (kk <= m && om_[row + kk] >= mx) { mx = om_[row + kk]; pick = kk; pst = SM; }
          }
          for (int r = 0; r < 4; r++) {
            const int kk = r * q_stripes + q + 1;
            if (kk <= m && od_[row + kk] > mx) { mx = od_[row + kk]; pick = kk; pst = SD; }
          }
        }
        if (pick == 0) break;
        k = pick;
        s1 = pst;
      } else if (s0 == SM) {
        if (i < 1 || k < 1) break;  // no predecessor left (reachable only when every path is -inf)
        if (!got_last) { got_last = true; cd.i1 = i; cd.k1 = k; }
        got_first = true;
        cd.i0 = i;
        cd.k0 = k;
        const size_t prow = (size_t)(i - 1) * w_;
        float path[4] = {kNegInf, kNegInf, kNegInf, dis(pbm[k], xb[i - 1])};
        if (k >= 2) {
          path[0] = dis(pmm[k - 1], om_[prow + k - 1]);
          path[1] = dis(pim[k - 1], oi_[prow + k - 1]);
          path[2] = dis(pdm[k - 1], od_[prow + k - 1]);
        }
        int best = 0;
        for (int t = 1; t < 4; t++)
          if (path[t] > path[best]) best = t;
        k -= 1;
        i -= 1;
        s1 = best == 0 ? SM : best == 1 ? SI : best == 2 ? SD : SB;
      } else if (s0 == SD) {
        if (k < 1) break;
        const size_t row = (size_t)i * w_;
        float a = kNegInf, b = kNegInf;
        if (k >= 2) {
          a = dis(pmd[k - 1], om_[row + k - 1]);
          b = dis(pdd[k - 1], od_[row + k - 1]);
        }
        k -= 1;
        s1 = a >= b ? SM : SD;
      } else if (s0 == SI) {
        if (i < 1 || k < 1) break;
        const size_t prow = (size_t)(i - 1) * w_;
        const float a = dis(pmi[k], om_[prow + k]);
        const float b = dis(pii[k], oi_[prow + k]);
        i -= 1;
        s1 = a >= b ? SM : SI;
      } else if (s0 == SB) {
        const float a = st.pmove == 0.0f ? kNegInf : xn[i];
        const float b = st.pmove == 0.0f ? kNegInf : xj[i];
        if (a > b) s1 = SN;
        else break;
      } else {
        break;
      }
      if ((s1 == SN || s1 == SJ || s1 == SC) && s1 == s0) i -= 1;
      if (s1 == SN) break;
      s0 = s1;
    }
    if (got_first && got_last) return cd;
    return std::nullopt;
  }

  // First B..E segment of the Viterbi path (src/hmmer/dp.rs:691-904).
  std::optional<Coords> viterbi_first(const uint8_t* sub, int64_t lr, const SpecialTr& st) {
    const int m = p_.m;
    if (lr == 0 || m == 0) return std::nullopt;
    const size_t n = (size_t)(lr + 1) * w_;
    std::vector<float> vm(n, kNegInf), vi(n, kNegInf), vd(n, kNegInf);
    std::vector<uint8_t> bm(n, 0), bi(n, 0), bd(n, 0);
    std::vector<float> xn(lr + 1, kNegInf), xb(lr + 1, kNegInf), xj(lr + 1, kNegInf), xc(lr + 1, kNegInf);
    std::vector<int> esrc(lr + 1, 0);
    std::vector<char> edel(lr + 1, 0), bj(lr + 1, 0), je(lr + 1, 0), ce(lr + 1, 0);
    const float *tbm = p_.t[TBM].data(), *tmm = p_.t[TMM].data(), *tim = p_.t[TIM].data(), *tdm = p_.t[TDM].data();
    const float *tmi = p_.t[TMI].data(), *tii = p_.t[TII].data(), *tmd = p_.t[TMD].data(), *tdd = p_.t[TDD].data();
    xn[0] = 0.0f;
    xb[0] = st.move;
    for (int64_t i = 1; i <= lr; i++) {
      const uint8_t x = sub[i - 1];
      const float* rs = p_.msc_row(x);
      const bool ins_ok = x != SYM_STAR;
      float best = kNegInf;
      int bk = 0;
      bool bdel = false;
      for (int k = 1; k <= m; k++) {
        const size_t pc = (size_t)(i - 1) * w_ + k, cc = (size_t)i * w_ + k;
        const float c0 = vm[pc - 1] + tmm[k - 1], c1 = vi[pc - 1] + tim[k - 1], c2 = vd[pc - 1] + tdm[k - 1];
        const float c3 = xb[i - 1] + tbm[k];
        float sc = c0;
        uint8_t ptr = 0;
        if (c1 > sc) { sc = c1; ptr = 1; }
        if (c2 > sc) { sc = c2; ptr = 2; }
        if (c3 > sc) { sc = c3; ptr = 3; }
        vm[cc] = sc + rs[k];
        bm[cc] = ptr;
        if (k < m && ins_ok) {
          const float a = vm[pc] + tmi[k], b = vi[pc] + tii[k];
          if (a >= b) { vi[cc] = a; bi[cc] = 0; } else { vi[cc] = b; bi[cc] = 1; }
        }
        const float a = vm[cc - 1] + tmd[k - 1], b = vd[cc - 1] + tdd[k - 1];
        if (a >= b) { vd[cc] = a; bd[cc] = 0; } else { vd[cc] = b; bd[cc] = 1; }
        if (vm[cc] > best) { best = vm[cc]; bk = k; bdel = false; }
        if (vd[cc] > best) { best = vd[cc]; bk = k; bdel = true; }
      }
      esrc[i] = bk;
      edel[i] = bdel;
      const float jl = xj[i - 1] + st.loop, jv = best + st.e_loop;
      if (jv > jl) { xj[i] = jv; je[i] = 1; } else xj[i] = jl;
      const float cl = xc[i - 1] + st.loop, cv = best + st.e_move;
      if (cv > cl) { xc[i] = cv; ce[i] = 1; } else xc[i] = cl;
      xn[i] = xn[i - 1] + st.loop;
      const float bn = xn[i] + st.move, bjv = xj[i] + st.move;
      if (bjv > bn) { xb[i] = bjv; bj[i] = 1; } else xb[i] = bn;
    }
    if (!(xc[lr] > kNegInf)) return std::nullopt;
    enum S { SC, SE, SM, SI, SD, SB, SJ, SN } s = SC;
    int64_t i = lr;
    int k = 0;
    bool open = false;
    int64_t end_i = 0;
    int end_k = 0;
    std::optional<Coords> first;
    const size_t limit = 4 * (size_t)(lr + 2) * (size_t)(m + 2);
    for (size_t guard = 1; guard <= limit; guard++) {
      if (s == SC) {
        if (i == 0) break;
        if (ce[i]) s = SE; else i -= 1;
      } else if (s == SE) {
        if (esrc[i] == 0) break;
        k = esrc[i];
        s = edel[i] ? SD : SM;
        open = true;
        end_i = i;
        end_k = k;
      } else if (s == SM) {
        const uint8_t ptr = bm[(size_t)i * w_ + k];
        if (ptr == 0) { s = SM; k--; i--; }
        else if (ptr == 1) { s = SI; k--; i--; }
        else if (ptr == 2) { s = SD; k--; i--; }
        else {
          if (open) {  // segments come out last-to-first; keep the earliest
            first = Coords{i, end_i, k, end_k};
            open = false;
          }
          s = SB;
          i--;
        }
      } else if (s == SI) {
        s = bi[(size_t)i * w_ + k] == 0 ? SM : SI;
        i--;
      } else if (s == SD) {
        s = bd[(size_t)i * w_ + k] == 0 ? SM : SD;
        k--;
      } else if (s == SB) {
        s = bj[i] ? SJ : SN;
      } else if (s == SJ) {
        if (je[i]) s = SE; else i--;
      } else {
        break;
      }
    }
    return first;
  }

  // One stochastic traceback (src/hmmer/dp.rs:1075-1258).
  void sample_trace(const Mat& fx, const SpecialTr& st, Lcg& rng, std::vector<Sampled>& out) {
    out.clear();
    const int m = p_.m;
    const int q_stripes = std::max(2, (m > 0 ? m - 1 : 0) / 4 + 1);
    const float *pbm = p_.p[TBM].data(), *pmm = p_.p[TMM].data(), *pim = p_.p[TIM].data(), *pdm = p_.p[TDM].data();
    const float *pmi = p_.p[TMI].data(), *pii = p_.p[TII].data(), *pmd = p_.p[TMD].data(), *pdd = p_.p[TDD].data();
    enum S { SC, SE, SM, SI, SD, SB, SJ, SN } s0 = SC;
    int64_t i = fx.l;
    int k = 0;
    bool have = false;
    Sampled cur;
    const size_t limit = 8 * (size_t)(fx.l + 2) * (size_t)(m + 2) + 64;
    for (size_t guard = 1; guard <= limit; guard++) {
      S s1;
      if (s0 == SC) {
        if (i == 0) break;
        float path[2] = {fx.xc[i - 1] * st.ploop, fx.xe[i] * st.pe_move * fx.scale[i]};
        s1 = choose(rng, path) == 0 ? SC : SE;
      } else if (s0 == SE) {
        const double roll = rng.uniform();
        const float norm = (float)(1.0 / (double)fx.xe[i]);
        const size_t row = (size_t)i * w_;
        double acc = 0.0;
        int pick = 0;
        S pst = SM;
        for (int pass = 0; pick == 0 && pass < 1000; pass++) {
          for (int q = 0; q < q_stripes && pick == 0; q++) {
            for (int r = 0; r < 4 && pick == 0; r++) {
              const int kk = r * q_stripes + q + 1;
              if (kk <= m) {
                acc += (double)(fx.mm[row + kk] * norm);
                if (roll < acc) { pick = kk; pst = SM; }
              }
            }
            for (int r = 0; r < 4 && pick == 0; r++) {
              const int kk = r * q_stripes + q + 1;
              if (kk <= m) {
                acc += (double)(fx.dm[row + kk] * norm);
                if (roll < acc) { pick = kk; pst = SD; }
              }
            }
          }
          if (pick == 0 && acc <= 0.0) break;
        }
        if (pick == 0) break;
        k = pick;
        cur = Sampled();
        have = true;
        s1 = pst;
      } else if (s0 == SM) {
        if (have) {
          if (cur.sqto == 0) { cur.sqto = i; cur.hmmto = k; }
          cur.sqfrom = i;
          cur.hmmfrom = k;
          cur.nodes.push_back(k);
        }
        const size_t prow = (size_t)(i - 1) * w_;
        float path[4] = {fx.xb[i - 1] * pbm[k], 0.0f, 0.0f, 0.0f};
        if (k >= 2) {
          path[1] = fx.mm[prow + k - 1] * pmm[k - 1];
          path[2] = fx.im[prow + k - 1] * pim[k - 1];
          path[3] = fx.dm[prow + k - 1] * pdm[k - 1];
        }
        const int c = choose(rng, path);
        k -= 1;
        i -= 1;
        s1 = c == 0 ? SB : c == 1 ? SM : c == 2 ? SI : SD;
      } else if (s0 == SD) {
        const size_t row = (size_t)i * w_;
        float path[2] = {0.0f, 0.0f};
        if (k >= 2) {
          path[0] = fx.mm[row + k - 1] * pmd[k - 1];
          path[1] = fx.dm[row + k - 1] * pdd[k - 1];
        }
        const int c = choose(rng, path);
        k -= 1;
        s1 = c == 0 ? SM : SD;
      } else if (s0 == SI) {
        if (have) cur.nodes.push_back(k);
        const size_t prow = (size_t)(i - 1) * w_;
        float path[2] = {fx.mm[prow + k] * pmi[k], fx.im[prow + k] * pii[k]};
        const int c = choose(rng, path);
        i -= 1;
        s1 = c == 0 ? SM : SI;
      } else if (s0 == SB) {
        if (have) {
          out.push_back(std::move(cur));
          cur = Sampled();
          have = false;
        }
        float path[2] = {fx.xn[i] * st.pmove, fx.xj[i] * st.pmove};
        s1 = choose(rng, path) == 0 ? SN : SJ;
      } else if (s0 == SJ) {
        if (i == 0) break;
        float path[2] = {fx.xj[i - 1] * st.ploop, fx.xe[i] * st.pe_loop * fx.scale[i]};
        s1 = choose(rng, path) == 0 ? SJ : SE;
      } else {
        if (i == 0) break;
        s1 = SN;
      }
      if ((s1 == SN || s1 == SJ || s1 == SC) && s1 == s0) i -= 1;
      s0 = s1;
    }
    std::reverse(out.begin(), out.end());
  }

  // Envelope rescoring (rescore_isolated_domain; src/hmmer/pipeline.rs:545-591).
  bool rescore(int64_t i, int64_t j, std::vector<float>& n2sc, bool null2_done, DomainOut& d, float& envsc,
               float& domcorr) {
    if (i == 0 || j < i || j > l_) return false;
    const uint8_t* sub = dsq_ + (i - 1);
    const int64_t lr = j - i + 1;
    const SpecialTr st = special_transitions(l_, false);
    envsc = forward_full(sub, lr, st, fx_);
    if (!std::isfinite(envsc)) return false;
    const float bsc = backward_full(sub, lr, st, bx_);
    if (!std::isfinite(bsc)) return false;
    posterior(st, fx_, bx_, pp_);
    domcorr = 0.0f;
    if (o_.null2) {
      if (!null2_done) {
        float n2[NSYM];
        null2_posterior(pp_, n2);
        for (int64_t pos = i; pos <= j; pos++) {
          const float v = n2[dsq_[pos - 1]];
          n2sc[pos] = std::isfinite(v) ? v : 0.0f;
        }
      }
      for (int64_t pos = i; pos <= j; pos++) domcorr += n2sc[pos];
    }
    d.ienv = i;
    d.jenv = j;
    if (auto oa = oa_coords(st, pp_)) {
      d.iali = i - 1 + oa->i0; d.jali = i - 1 + oa->i1; d.kali = oa->k0; d.mali = oa->k1;
    } else if (auto vt = viterbi_first(sub, lr, st)) {
      d.iali = i - 1 + vt->i0; d.jali = i - 1 + vt->i1; d.kali = vt->k0; d.mali = vt->k1;
    } else {
      d.iali = i; d.jali = j; d.kali = 1; d.mali = p_.m;
    }
    return true;
  }

  // Multi-domain region: 200 sampled traces, position-specific null2 and
  // single-linkage clusters (src/hmmer/pipeline.rs:360-477).
  std::vector<std::pair<int64_t, int64_t>> trace_ensemble(int64_t ireg, int64_t jreg, std::vector<float>& n2sc) {
    constexpr int kSamples = 200;
    const uint8_t* sub = dsq_ + (ireg - 1);
    const int64_t lr = jreg - ireg + 1;
    const SpecialTr st = special_transitions(l_, true);
    forward_full(sub, lr, st, fx_);
    Lcg rng(42);
    for (int64_t v = ireg; v <= jreg; v++) n2sc[v] = 0.0f;
    std::vector<Sample> sp;
    std::vector<Sampled> doms;
    float n2[NSYM] = {0};
    for (int t = 0; t < kSamples; t++) {
      sample_trace(fx_, st, rng, doms);
      int64_t pos = 1;
      for (const Sampled& d : doms) {
        sp.push_back({(size_t)t, d.sqfrom + ireg - 1, d.sqto + ireg - 1, d.hmmfrom, d.hmmto});
        const float ld = (float)std::max<size_t>(d.nodes.size(), 1);
        for (int x = 0; x < NRES; x++) {
          const float* row = p_.mo_row(x);
          float v = 0.0f;
          for (int kk : d.nodes) v += row[kk];
          n2[x] = v / ld;
        }
        average_degenerate(n2);
        for (; pos <= d.sqfrom; pos++) n2sc[ireg + pos - 1] += 1.0f;
        for (; pos <= d.sqto; pos++) n2sc[ireg + pos - 1] += n2[dsq_[ireg + pos - 2]];
      }
      for (; pos <= lr; pos++) n2sc[ireg + pos - 1] += 1.0f;
    }
    for (int64_t v = ireg; v <= jreg; v++) n2sc[v] = std::log(n2sc[v] / (float)kSamples);
    return cluster(sp, kSamples);
  }

 private:
  static bool linked(const Sample& a, const Sample& b) {  // link_spsamples, pipeline.rs:308-327
    int64_t nov = std::min(a.j, b.j) - std::max(a.i, b.i) + 1;
    float n = (float)std::min(a.j - a.i + 1, b.j - b.i + 1);
    if ((float)nov / n < 0.8f) return false;
    nov = (int64_t)std::min(a.m, b.m) - (int64_t)std::max(a.k, b.k);
    n = (float)std::min(a.m - a.k + 1, b.m - b.k + 1);
    if ((float)nov / n < 0.8f) return false;
    if (std::llabs((a.i - a.k) - (b.i - b.k)) <= 4) return true;
    return std::llabs((a.j - a.m) - (b.j - b.m)) <= 4;
  }

 public:
  static std::vector<std::pair<int64_t, int64_t>> cluster(const std::vector<Sample>& sp, int nsamples) {
    const size_t n = sp.size();
    // esl_cluster_SingleLinkage traversal (pipeline.rs:330-355)
    std::vector<size_t> pool(n), stack;
    for (size_t x = 0; x < n; x++) pool[x] = n - x - 1;
    std::vector<size_t> cid(n, 0);
    size_t nc = 0;
    while (!pool.empty()) {
      stack.push_back(pool.back());
      pool.pop_back();
      while (!stack.empty()) {
        const size_t x = stack.back();
        stack.pop_back();
        cid[x] = nc;
        for (size_t ii = pool.size(); ii-- > 0;) {
          if (linked(sp[x], sp[pool[ii]])) {
            stack.push_back(pool[ii]);
            pool[ii] = pool.back();
            pool.pop_back();
          }
        }
      }
      nc++;
    }
    struct Sig { int64_t i, j; float prob; };
    std::vector<Sig> sig;
    std::vector<int64_t> vi, vj, vk, vm;
    for (size_t c = 0; c < nc; c++) {
      size_t ninc = 0;
      bool any = false;
      size_t last = 0;
      vi.clear(); vj.clear(); vk.clear(); vm.clear();
      for (size_t h = 0; h < n; h++) {
        if (cid[h] != c) continue;
        if (!any || last != sp[h].trace) ninc++;
        any = true;
        last = sp[h].trace;
        vi.push_back(sp[h].i); vj.push_back(sp[h].j); vk.push_back(sp[h].k); vm.push_back(sp[h].m);
      }
      if ((float)ninc / (float)nsamples < 0.25f) continue;
      const size_t thr = (size_t)std::ceil((float)ninc * 0.02f);
      const int64_t bi = endpoint(vi, thr, true), bk = endpoint(vk, thr, true);
      const int64_t bj = endpoint(vj, thr, false), bm = endpoint(vm, thr, false);
      if (bi > bj || bk > bm) continue;
      sig.push_back({bi, bj, (float)ninc / (float)nsamples});
    }
    std::stable_sort(sig.begin(), sig.end(), [](const Sig& a, const Sig& b) { return a.i < b.i; });
    std::vector<char> dom(sig.size(), 0);
    for (size_t d = 0; d < sig.size(); d++) {
      for (size_t d2 = d + 1; d2 < sig.size(); d2++) {
        const int64_t nov = std::min(sig[d].j, sig[d2].j) - std::max(sig[d].i, sig[d2].i) + 1;
        if (nov == 0) break;
        const float nn = (float)std::min(sig[d].j - sig[d].i + 1, sig[d2].j - sig[d2].i + 1);
        if ((float)nov / nn >= 0.8f) {
          if (sig[d].prob > sig[d2].prob) dom[d2] = 1;
          else dom[d] = 1;
        }
      }
    }
    std::vector<std::pair<int64_t, int64_t>> out;
    for (size_t d = 0; d < sig.size(); d++)
      if (!dom[d]) out.emplace_back(sig[d].i, sig[d].j);
    return out;
  }

 private:
  // Leftmost (left=true) or rightmost endpoint whose count reaches thr, else
  // the most frequent one (pipeline.rs:489-525).
  static int64_t endpoint(const std::vector<int64_t>& v, size_t thr, bool left) {
    int64_t lo = INT64_MAX, hi = 0;
    for (int64_t x : v) { lo = std::min(lo, x); hi = std::max(hi, x); }
    std::vector<size_t> cnt((size_t)(hi - lo + 1), 0);
    for (int64_t x : v) cnt[(size_t)(x - lo)]++;
    if (left) {
      for (size_t o = 0; o < cnt.size(); o++)
        if (cnt[o] >= thr) return lo + (int64_t)o;
    } else {
      for (size_t o = cnt.size(); o-- > 0;)
        if (cnt[o] >= thr) return lo + (int64_t)o;
    }
    size_t best = 0;
    for (size_t o = 0; o < cnt.size(); o++)
      if (cnt[o] > cnt[best]) best = o;
    return lo + (int64_t)best;
  }

  const ProfileHost& p_;
  const uint8_t* dsq_;
  const int64_t l_;
  const SearchOpts& o_;
  const size_t w_;
  ScorerWork& ws_ = scorer_work();
  WorkClaim claim_{ws_};
  Mat& fx_ = ws_.fx;
  Mat& bx_ = ws_.bx;
  Post& pp_ = ws_.pp;
  std::vector<float>& om_ = ws_.om;
  std::vector<float>& oi_ = ws_.oi;
  std::vector<float>& od_ = ws_.od;
};

// Log-space rows from the device's raw scaled rows.  Forward rows: slots
// N B E J C scale per row i = 1..L (src/hmmer/dp.rs:270-292).
void forward_log_rows(const ProfileHost& p, int64_t l, const float* raw, LogRows& sp, double& lnscale_out) {
  (void)p;
  const SpecialTr st = special_transitions(l, true);
  sp.reset(l);
  sp.n[0] = 0.0f;
  sp.b[0] = lnpos(st.pmove);
  double lnscale = 0.0;
  for (int64_t i = 1; i <= l; i++) {
    const float* r = raw + 6 * i;
    if (r[5] > 0.0f) lnscale += std::log((double)r[5]);
    const float ls = (float)lnscale;
    sp.n[i] = lnpos(r[0]) + ls;
    sp.b[i] = lnpos(r[1]) + ls;
    sp.e[i] = lnpos(r[2]) + ls;
    sp.j[i] = lnpos(r[3]) + ls;
    sp.c[i] = lnpos(r[4]) + ls;
  }
  lnscale_out = lnscale;
}

// Backward rows: row L holds C and E; rows L-1..1 the five specials and the
// row's rescale factor; row 0 the raw B sum in slot 1 (src/hmmer/dp.rs:314-391).
float backward_log_rows(int64_t l, const float* raw, LogRows& sp) {
  const SpecialTr st = special_transitions(l, true);
  sp.reset(l);
  sp.c[l] = lnpos(raw[6 * l + 4]);
  sp.e[l] = lnpos(raw[6 * l + 2]);
  double lnscale = 0.0;
  for (int64_t i = l - 1; i >= 1; i--) {
    const float* r = raw + 6 * i;
    if (r[5] > 0.0f) lnscale += std::log((double)r[5]);
    const float ls = (float)lnscale;
    sp.n[i] = lnpos(r[0]) + ls;
    sp.b[i] = lnpos(r[1]) + ls;
    sp.e[i] = lnpos(r[2]) + ls;
    sp.j[i] = lnpos(r[3]) + ls;
    sp.c[i] = lnpos(r[4]) + ls;
  }
  sp.b[0] = lnpos(raw[1]) + (float)lnscale;
  sp.n[0] = logsum2(sp.n[1] + st.loop, sp.b[0] + st.move);
  return sp.n[0];
}

bool is_multidomain(const std::vector<float>& btot, const std::vector<float>& etot, int64_t i, int64_t j) {
  float mx = -1.0f;
  for (int64_t jj = i; jj <= j; jj++) {
    const float v = std::fmin(etot[jj] - etot[i - 1], btot[j] - btot[jj - 1]);
    if (v > mx) mx = v;
  }
  return mx >= 0.20f;
}

}  // namespace

float forward_score_from_rows(const ProfileHost& p, int64_t l, const float* fwd_rows) {
  if (l <= 0) return kNegInf;  // no row was computed; the reference's xc stays 0
  LogRows sp;
  double lnscale;
  forward_log_rows(p, l, fwd_rows, sp, lnscale);
  const SpecialTr st = special_transitions(l, true);
  const float xc = fwd_rows[6 * l + 4];
  return (float)((double)lnpos(xc * st.pmove) + lnscale);
}

float backward_score_from_rows(int64_t l, const float* bwd_rows) {
  if (l <= 0) return kNegInf;
  LogRows sp;
  return backward_log_rows(l, bwd_rows, sp);
}

namespace {

struct Env {
  DomainOut d;
  float envsc, domcorr;
};

// Sequence and domain scores of a pair from its rescored envelopes
// (src/hmmer/pipeline.rs:247-293).
void assemble_hit(const ProfileHost& p, int64_t l, float fwdsc, float nullsc, int64_t nregions,
                  const std::vector<float>& n2sc, const std::vector<Env>& envs, const SearchOpts& o, HitOut& out) {
  const float omega = std::log(1.0f / 256.0f);
  float seqbias = 0.0f;
  if (o.null2) {
    float s = 0.0f;
    for (int64_t q = 1; q <= l; q++) s += n2sc[q];
    seqbias = logsum2(0.0f, omega + s);
  }
  float pre_score = (fwdsc - nullsc) / kLn2f;
  float seq_score = (fwdsc - (nullsc + seqbias)) / kLn2f;
  const float lml = std::log((float)l / ((float)l + 3.0f));
  float sum = 0.0f, sum_bias = 0.0f;
  int64_t ld_tot = 0;
  for (const Env& e : envs) {
    const bool keep = o.null2 ? (e.envsc - e.domcorr > 0.0f) : (e.envsc > 0.0f);
    if (keep) {
      sum += e.envsc;
      ld_tot += e.d.jenv - e.d.ienv + 1;
      sum_bias += e.domcorr;
    }
  }
  const float sum_seqbias = o.null2 ? logsum2(0.0f, omega + sum_bias) : 0.0f;
  sum += (float)(l - std::min(ld_tot, l)) * lml;
  const float pre2 = (sum - nullsc) / kLn2f;
  const float sum_score = (sum - (nullsc + sum_seqbias)) / kLn2f;
  if (ld_tot > 0 && sum_score > seq_score) {
    seq_score = sum_score;
    pre_score = pre2;
  }
  const double ftau = p.has_fwd ? p.fwd[0] : NAN, flam = p.has_fwd ? p.fwd[1] : NAN;
  out.bits = seq_score;
  out.bias = pre_score - seq_score;
  out.lnp = p.has_fwd ? exp_tail_logsurv((double)seq_score, ftau, flam) : NAN;
  out.nregions = nregions;
  out.domains.clear();
  for (const Env& e : envs) {
    const int64_t ld = e.d.jenv - e.d.ienv + 1;
    const float dombias = o.null2 ? logsum2(0.0f, omega + e.domcorr) : 0.0f;
    DomainOut d = e.d;
    d.bits = (e.envsc + (float)(l - ld) * lml - (nullsc + dombias)) / kLn2f;
    d.bias = dombias / kLn2f;
    d.lnp = p.has_fwd ? exp_tail_logsurv((double)d.bits, ftau, flam) : NAN;
    out.domains.push_back(d);
  }
}

}  // namespace

namespace {

// Posterior decoding of the special states and region identification
// (p7_GDomainDecoding + p7_domaindef_ByPosteriorHeuristics,
// src/hmmer/pipeline.rs:187-245): calls on_region(i, j, multidomain) for each
// region in order.  Returns false when fwdsc is not finite.
template <typename F>
bool decode_regions(const ProfileHost& p, int64_t l, const RawRows& rows, float fwdsc, float& nexpected,
                    F&& on_region) {
  if (!std::isfinite(fwdsc)) return false;
  const SpecialTr xs = special_transitions(l, true);
  LogRows f, b;
  double lnscale_f;
  forward_log_rows(p, l, rows.fwd, f, lnscale_f);
  const float bcksc = backward_log_rows(l, rows.bwd, b);
  const float overall = std::isfinite(bcksc) ? bcksc : fwdsc;
  std::vector<float> btot((size_t)l + 1, 0.0f), etot((size_t)l + 1, 0.0f), mocc((size_t)l + 1, 0.0f);
  for (int64_t i = 1; i <= l; i++) {
    btot[i] = btot[i - 1] + std::exp(f.b[i - 1] + b.b[i - 1] - overall);
    etot[i] = etot[i - 1] + std::exp(f.e[i] + b.e[i] - overall);
    const float njc = std::exp(f.n[i - 1] + b.n[i] + xs.loop - overall) +
                      std::exp(f.j[i - 1] + b.j[i] + xs.loop - overall) +
                      std::exp(f.c[i - 1] + b.c[i] + xs.loop - overall);
    mocc[i] = 1.0f - njc;
  }
  nexpected = btot[l];
  int64_t start = -1;
  bool triggered = false;
  for (int64_t j = 1; j <= l; j++) {
    if (!triggered) {
      if (mocc[j] - (btot[j] - btot[j - 1]) < 0.10f || start == -1) start = j;
      if (mocc[j] >= 0.25f) triggered = true;
    } else if (mocc[j] - (etot[j] - etot[j - 1]) < 0.10f) {
      const int64_t ri = std::max<int64_t>(start, 1);
      on_region(ri, j, is_multidomain(btot, etot, ri, j));
      start = -1;
      triggered = false;
    }
  }
  return true;
}

}  // namespace

bool define_domains(const ProfileHost& p, const uint8_t* dsq, int64_t l, const RawRows& rows, float fwdsc,
                    const SearchOpts& o, HitOut& out) {
  EnvelopeScorer es(p, dsq, l, o);
  std::vector<float> n2sc((size_t)l + 1, 0.0f);
  std::vector<Env> envs;
  int64_t nregions = 0;
  const bool ok = decode_regions(p, l, rows, fwdsc, out.nexpected, [&](int64_t ri, int64_t j, bool multi) {
    nregions++;
    Env e;
    if (multi) {
      for (auto [ei, ej] : es.trace_ensemble(ri, j, n2sc))
        if (es.rescore(ei, ej, n2sc, true, e.d, e.envsc, e.domcorr)) envs.push_back(e);
    } else if (es.rescore(ri, j, n2sc, false, e.d, e.envsc, e.domcorr)) {
      envs.push_back(e);
    }
  });
  if (!ok || nregions == 0 || envs.empty()) return false;
  assemble_hit(p, l, fwdsc, null1_score(l), nregions, n2sc, envs, o, out);
  return true;
}

// ---- batched domain definition (device envelope passes) ----------------------
struct DomainBatch::Impl {
  struct Pending {
    int64_t i, j;
    bool null2_done;
    bool pass;         // false: rescore rejects the envelope before any pass
    int64_t req = -1;  // index into reqs
    int32_t region = -1;  // >= 0: placeholder for the envelopes of this region's trace ensemble
  };
  struct PairState {
    bool begun = false;
    const ProfileHost* p = nullptr;
    const uint8_t* dsq = nullptr;
    int64_t l = 0;
    int32_t pi = 0, ti = 0;
    float fwdsc = 0, nexpected = 0;
    int64_t nregions = 0;
    std::vector<float> n2sc;
    std::vector<Pending> pend;
    std::vector<std::pair<int64_t, int64_t>> regions;                   // multi-domain regions left to the device
    std::vector<std::vector<std::pair<int64_t, int64_t>>> region_envs;  // their clustered envelopes
  };
  SearchOpts o;
  std::vector<PairState> pairs;
  std::vector<RegionRequest> regs;
  bool regs_built = false;
  std::vector<EnvRequest> reqs;
};

DomainBatch::DomainBatch(const SearchOpts& o, size_t npairs) : impl_(new Impl) {
  impl_->o = o;
  impl_->pairs.resize(npairs);
}
DomainBatch::~DomainBatch() = default;

void DomainBatch::begin(size_t q, const ProfileHost& p, int32_t pi, const uint8_t* dsq, int64_t l, int32_t ti,
                        const RawRows& rows, float fwdsc, bool device_regions) {
  Impl::PairState& st = impl_->pairs[q];
  st.p = &p;
  st.dsq = dsq;
  st.l = l;
  st.pi = pi;
  st.ti = ti;
  st.fwdsc = fwdsc;
  st.n2sc.assign((size_t)l + 1, 0.0f);
  EnvelopeScorer es(p, dsq, l, impl_->o);
  auto add = [&](int64_t i, int64_t j, bool null2_done) {
    st.pend.push_back({i, j, null2_done, !(i == 0 || j < i || j > l), -1});
  };
  st.begun = decode_regions(p, l, rows, fwdsc, st.nexpected, [&](int64_t ri, int64_t j, bool multi) {
    st.nregions++;
    if (multi && device_regions) {  // traced on the device; expand() fills in the envelopes
      st.pend.push_back({ri, j, true, true, -1, (int32_t)st.regions.size()});
      st.regions.emplace_back(ri, j);
    } else if (multi) {  // stochastic traces and clustering here; their envelopes are batched
      for (auto [ei, ej] : es.trace_ensemble(ri, j, st.n2sc)) add(ei, ej, true);
    } else {
      add(ri, j, false);
    }
  });
}

const std::vector<RegionRequest>& DomainBatch::regions() {
  Impl& I = *impl_;
  if (I.regs_built) return I.regs;
  I.regs_built = true;
  for (size_t q = 0; q < I.pairs.size(); q++) {
    Impl::PairState& st = I.pairs[q];
    if (!st.begun || st.regions.empty()) continue;
    st.region_envs.assign(st.regions.size(), {});
    const SpecialTr multi = special_transitions(st.l, true);
    for (size_t r = 0; r < st.regions.size(); r++)
      I.regs.push_back({(int32_t)q, st.pi, st.ti, st.regions[r].first, st.regions[r].second, multi, (int32_t)r});
  }
  return I.regs;
}

// The rest of region_trace_ensemble (src/hmmer/pipeline.rs:360-477) after the
// device's traces: the position-specific null2 from the per-position sums,
// then single-linkage clustering of the sampled domains.
void DomainBatch::expand(size_t r, const std::vector<TraceSample>& samples, const float* n2sum, bool ok) {
  Impl& I = *impl_;
  const RegionRequest& g = I.regs[r];
  Impl::PairState& st = I.pairs[(size_t)g.pair];
  auto& envs = st.region_envs[(size_t)g.local];
  if (!ok) {
    EnvelopeScorer es(*st.p, st.dsq, st.l, I.o);
    envs = es.trace_ensemble(g.i, g.j, st.n2sc);
    return;
  }
  constexpr int kSamples = 200;
  for (int64_t v = g.i; v <= g.j; v++) st.n2sc[(size_t)v] = std::log(n2sum[v - g.i + 1] / (float)kSamples);
  std::vector<Sample> sp(samples.size());
  for (size_t x = 0; x < samples.size(); x++)
    sp[x] = {(size_t)samples[x].trace, samples[x].i, samples[x].j, samples[x].k, samples[x].m};
  envs = EnvelopeScorer::cluster(sp, kSamples);
}

uint32_t DomainBatch::trace_lcg_start() { return Lcg(42).state(); }

const std::vector<EnvRequest>& DomainBatch::requests() {
  Impl& I = *impl_;
  I.reqs.clear();
  for (size_t q = 0; q < I.pairs.size(); q++) {
    Impl::PairState& st = I.pairs[q];
    if (!st.begun) continue;
    if (!st.regions.empty()) {  // each region placeholder becomes its envelopes, in order
      std::vector<Impl::Pending> flat;
      for (const Impl::Pending& e : st.pend) {
        if (e.region < 0) {
          flat.push_back(e);
          continue;
        }
        for (auto [ei, ej] : st.region_envs[(size_t)e.region])
          flat.push_back({ei, ej, true, !(ei == 0 || ej < ei || ej > st.l), -1, -1});
      }
      st.pend.swap(flat);
      st.regions.clear();
    }
    const SpecialTr uni = special_transitions(st.l, false);
    for (Impl::Pending& e : st.pend) {
      if (!e.pass) continue;
      e.req = (int64_t)I.reqs.size();
      I.reqs.push_back({(int32_t)q, st.pi, st.ti, e.i, e.j, e.null2_done, uni});
    }
  }
  return I.reqs;
}

// forward_matrix's score and backward_matrix's row 0 from the raw rows, then
// decode's per-row factor and N/J/C posteriors (src/hmmer/dp.rs:442-601,
// 1278-1306), with the libm the reference uses.
void DomainBatch::factors(size_t r, const float* fr, const float* br, EnvFactors& f) const {
  const EnvRequest& q = impl_->reqs[r];
  const SpecialTr& st = q.st;
  const int64_t lr = q.j - q.i + 1;
  const size_t n = (size_t)lr + 1;
  f.ok = false;
  std::vector<double> lnf(n, 0.0), lnb(n, 0.0);
  std::vector<float> fn(n, kNegInf), fj(n, kNegInf), fc(n, kNegInf), bn(n, kNegInf), bj(n, kNegInf),
      bc(n, kNegInf);
  fn[0] = 0.0f;
  double lnscale = 0.0;
  for (int64_t i = 1; i <= lr; i++) {
    const float* x = fr + 6 * i;
    if (x[5] > 0.0f) lnscale += std::log((double)x[5]);
    lnf[i] = lnscale;
    const float ls = (float)lnscale;
    fn[i] = lnpos(x[0]) + ls;
    fj[i] = lnpos(x[3]) + ls;
    fc[i] = lnpos(x[4]) + ls;
  }
  f.envsc = (float)((double)lnpos(fr[6 * lr + 4] * st.pmove) + lnscale);
  if (!std::isfinite(f.envsc)) return;
  bc[lr] = lnpos(br[6 * lr + 4]);
  lnscale = 0.0;
  for (int64_t i = lr - 1; i >= 1; i--) {
    const float* x = br + 6 * i;
    if (x[5] > 0.0f) lnscale += std::log((double)x[5]);
    lnb[i] = lnscale;
    const float ls = (float)lnscale;
    bn[i] = lnpos(x[0]) + ls;
    bj[i] = lnpos(x[3]) + ls;
    bc[i] = lnpos(x[4]) + ls;
  }
  const float b0 = lnpos(br[1]) + (float)lnscale;
  const float bsc = logsum2(bn[1] + st.loop, b0 + st.move);
  if (!std::isfinite(bsc)) return;
  const double overall = (double)bsc;
  f.fac.assign(n, 0.0);
  f.pn.assign(n, 0.0f);
  f.pj.assign(n, 0.0f);
  f.pc.assign(n, 0.0f);
  f.sn = f.sj = f.sc = 0.0f;
  for (int64_t i = 1; i <= lr; i++) {
    f.fac[i] = std::exp(lnf[i] + lnb[i] - overall);
    f.pn[i] = (float)std::exp((double)(fn[i - 1] + bn[i] + st.loop) - overall);
    f.pj[i] = (float)std::exp((double)(fj[i - 1] + bj[i] + st.loop) - overall);
    f.pc[i] = (float)std::exp((double)(fc[i - 1] + bc[i] + st.loop) - overall);
    f.sn += f.pn[i];
    f.sj += f.pj[i];
    f.sc += f.pc[i];
  }
  f.ok = true;
}

// The rest of rescore_isolated_domain (src/hmmer/pipeline.rs:545-591) for every
// envelope of pair q, then the pair's scores.
bool DomainBatch::finish(size_t q, const std::vector<EnvFactors>& F, const std::vector<EnvDeviceOut>& D,
                         HitOut& out) {
  Impl::PairState& st = impl_->pairs[q];
  const SearchOpts& o = impl_->o;
  if (!st.begun) return false;
  out.nexpected = st.nexpected;
  EnvelopeScorer es(*st.p, st.dsq, st.l, o);
  const SpecialTr uni = special_transitions(st.l, false);
  std::vector<Env> envs;
  for (const Impl::Pending& e : st.pend) {
    if (e.req < 0) continue;
    const EnvFactors& f = F[(size_t)e.req];
    if (!f.ok) continue;
    const EnvDeviceOut& d = D[(size_t)e.req];
    const int64_t lr = e.j - e.i + 1;
    Env v;
    v.envsc = f.envsc;
    v.domcorr = 0.0f;
    if (o.null2) {
      if (!e.null2_done) {  // null2 by posterior expectation (dp.rs:1310-1350)
        const float norm = 1.0f / (float)std::max<int64_t>(lr, 1);
        const float xfactor = f.sn * norm + f.sc * norm + f.sj * norm;
        const float isum = d.si * norm;
        float n2[NSYM];
        for (int x = 0; x < NRES; x++) n2[x] = d.v[x] + isum + xfactor;
        EnvelopeScorer::average_degenerate(n2);
        float lg[NSYM];
        for (int x = 0; x < NSYM; x++) lg[x] = n2[x] > 0.0f ? std::log(n2[x]) : kNegInf;
        for (int64_t pos = e.i; pos <= e.j; pos++) {
          const float w = lg[st.dsq[pos - 1]];
          st.n2sc[pos] = std::isfinite(w) ? w : 0.0f;
        }
      }
      for (int64_t pos = e.i; pos <= e.j; pos++) v.domcorr += st.n2sc[pos];
    }
    v.d.ienv = e.i;
    v.d.jenv = e.j;
    if (d.found) {
      v.d.iali = e.i - 1 + d.i0; v.d.jali = e.i - 1 + d.i1; v.d.kali = d.k0; v.d.mali = d.k1;
    } else if (auto vt = es.viterbi_first(st.dsq + (e.i - 1), lr, uni)) {
      v.d.iali = e.i - 1 + vt->i0; v.d.jali = e.i - 1 + vt->i1; v.d.kali = vt->k0; v.d.mali = vt->k1;
    } else {
      v.d.iali = e.i; v.d.jali = e.j; v.d.kali = 1; v.d.mali = st.p->m;
    }
    envs.push_back(v);
  }
  if (st.nregions == 0 || envs.empty()) return false;
  assemble_hit(*st.p, st.l, st.fwdsc, null1_score(st.l), st.nregions, st.n2sc, envs, o, out);
  return true;
}


float composition_bias_score(const ProfileHost& p, const uint8_t* dsq, int64_t l) {
  const double l0 = 400.0, l1 = (double)p.m / 8.0;
  const double t00 = l0 / (l0 + 1.0), t01 = 1.0 / (l0 + 1.0), t10 = 1.0 / (l1 + 1.0), t11 = l1 / (l1 + 1.0);
  double eo0[NSYM], eo1[NSYM];
  for (int x = 0; x < NSYM; x++) eo0[x] = eo1[x] = 1.0;
  for (int x = 0; x < NRES; x++) eo1[x] = (double)p.compo[x] / (double)kBackground[x];
  for (int code = 20; code <= 23; code++) {
    const Degenerate& d = degenerate(code);
    double e0 = 0, e1 = 0, z = 0;
    for (int q = 0; q < d.n; q++) {
      e0 += (double)kBackground[d.members[q]];
      e1 += (double)p.compo[d.members[q]];
      z += (double)kBackground[d.members[q]];
    }
    eo0[code] = e0 / z;
    eo1[code] = e1 / z;
  }
  eo0[SYM_STAR] = eo1[SYM_STAR] = 1.0;
  const double tiny = std::numeric_limits<double>::min();
  double logsc = 0.0;
  double d0 = eo0[dsq[0]] * 0.999, d1 = eo1[dsq[0]] * 0.001;
  double mx = std::fmax(std::fmax(d0, d1), tiny);
  d0 /= mx;
  d1 /= mx;
  logsc += std::log(mx);
  for (int64_t i = 1; i < l; i++) {
    const int x = dsq[i];
    const double n0 = (d0 * t00 + d1 * t10) * eo0[x];
    const double n1 = (d0 * t01 + d1 * t11) * eo1[x];
    mx = std::fmax(std::fmax(n0, n1), tiny);
    d0 = n0 / mx;
    d1 = n1 / mx;
    logsc += std::log(mx);
  }
  logsc += std::log(d0 + d1);
  const double p1 = (double)l / ((double)l + 1.0);
  return (float)(logsc + (double)l * std::log(p1) + std::log(1.0 - p1));
}

}  // namespace sx
