// TEST INFRASTRUCTURE ONLY — FP64 log-space Plan7 Forward/Backward.
//
// Not a restatement of a reference function: it is the independent
// high-precision yardstick the FP32 odds-space Forward (src/hmmer/dp.rs:229-298)
// and the device kernels are measured against, and the source of the expected
// state/transition counts (= gradients of the Forward log score with respect
// to the log-space emission and transition scores) that the adjoint kernel is
// checked with.  Same state graph as dp.rs: local multihit entry B->M_k with
// t_bm, free exits M_k->E and D_k->E, insert emissions scored 0 except at node
// M and on '*', N/J/C loops from Xsc.
#include <cmath>
#include <vector>

#include "sx_oracle.hpp"

namespace sxo {

static inline double lse(double a, double b) {
  if (a == -INFINITY) return b;
  if (b == -INFINITY) return a;
  double hi = a > b ? a : b, lo = a > b ? b : a;
  return hi + std::log1p(std::exp(lo - hi));
}

struct Lsp {  // per-profile scores promoted to f64, with an optional perturbation
  size_t m;
  std::vector<double> msc, t[7], tbm, isc;  // isc[x*(M+1)+k]: insert emission score (0 / -inf)
};

// kind: 0 none, 1 msc[x][k] (idx = x*(M+1)+k), 2 isc[x][k], 3+q transition q at node k (idx = k), 10 t_bm[k]
static Lsp promote(const Profile& p, int kind, size_t idx, double delta) {
  Lsp s;
  s.m = p.m;
  const size_t w = p.m + 1;
  s.msc.assign(p.msc.begin(), p.msc.end());
  const std::vector<float>* tv[7] = {&p.t_mm, &p.t_mi, &p.t_md, &p.t_im, &p.t_ii, &p.t_dm, &p.t_dd};
  for (int q = 0; q < 7; q++) s.t[q].assign(tv[q]->begin(), tv[q]->end());
  s.tbm.assign(p.t_bm.begin(), p.t_bm.end());
  s.isc.assign((size_t)NCODE * w, -INFINITY);
  for (int x = 0; x < NCODE; x++)
    for (size_t k = 1; k < p.m; k++) s.isc[(size_t)x * w + k] = (x == CODE_STAR) ? -INFINITY : 0.0;
  if (kind == 1) s.msc[idx] += delta;
  else if (kind == 2) s.isc[idx] += delta;
  else if (kind >= 3 && kind < 10) s.t[kind - 3][idx] += delta;
  else if (kind == 10) s.tbm[idx] += delta;
  return s;
}

struct LogMats {
  size_t m, l;
  std::vector<double> M, I, D;        // (L+1)*(M+2)
  std::vector<double> N, B, E, J, C;  // L+1
};

static double fwd64(const Lsp& s, const uint8_t* dsq, size_t l, const Xsc& xs, LogMats& f) {
  const size_t m = s.m, w = m + 2;
  f.m = m; f.l = l;
  f.M.assign((l + 1) * w, -INFINITY); f.I.assign((l + 1) * w, -INFINITY); f.D.assign((l + 1) * w, -INFINITY);
  for (auto* v : {&f.N, &f.B, &f.E, &f.J, &f.C}) v->assign(l + 1, -INFINITY);
  const double nl = xs.n_loop, nm = xs.n_move, jl = xs.j_loop, jm = xs.j_move, cl = xs.c_loop, em = xs.e_move,
               el = xs.e_loop;
  f.N[0] = 0.0;
  f.B[0] = nm;
  for (size_t i = 1; i <= l; i++) {
    uint8_t x = dsq[i - 1];
    const size_t pr = (i - 1) * w, cr = i * w;
    double e = -INFINITY;
    for (size_t k = 1; k <= m; k++) {
      double v = f.B[i - 1] + s.tbm[k];
      if (k >= 2) {
        v = lse(v, f.M[pr + k - 1] + s.t[T_MM][k - 1]);
        v = lse(v, f.I[pr + k - 1] + s.t[T_IM][k - 1]);
        v = lse(v, f.D[pr + k - 1] + s.t[T_DM][k - 1]);
      }
      f.M[cr + k] = v + s.msc[(size_t)x * (m + 1) + k];
      if (k < m) f.I[cr + k] = lse(f.M[pr + k] + s.t[T_MI][k], f.I[pr + k] + s.t[T_II][k]) + s.isc[(size_t)x * (m + 1) + k];
      if (k >= 2) f.D[cr + k] = lse(f.M[cr + k - 1] + s.t[T_MD][k - 1], f.D[cr + k - 1] + s.t[T_DD][k - 1]);
      e = lse(e, lse(f.M[cr + k], f.D[cr + k]));
    }
    f.E[i] = e;
    f.J[i] = lse(f.J[i - 1] + jl, e + el);
    f.C[i] = lse(f.C[i - 1] + cl, e + em);
    f.N[i] = f.N[i - 1] + nl;
    f.B[i] = lse(f.N[i] + nm, f.J[i] + jm);
  }
  return f.C[l] + xs.c_move;
}

static double bwd64(const Lsp& s, const uint8_t* dsq, size_t l, const Xsc& xs, LogMats& b) {
  const size_t m = s.m, w = m + 2;
  b.m = m; b.l = l;
  b.M.assign((l + 1) * w, -INFINITY); b.I.assign((l + 1) * w, -INFINITY); b.D.assign((l + 1) * w, -INFINITY);
  for (auto* v : {&b.N, &b.B, &b.E, &b.J, &b.C}) v->assign(l + 1, -INFINITY);
  const double nl = xs.n_loop, nm = xs.n_move, jl = xs.j_loop, jm = xs.j_move, cl = xs.c_loop, em = xs.e_move,
               el = xs.e_loop;
  for (size_t i = l + 1; i-- > 0;) {
    const size_t cr = i * w, nr = (i + 1) * w;
    // specials at row i (state occupied after emitting residue i)
    if (i == l) {
      b.C[i] = xs.c_move;
      b.J[i] = -INFINITY;
      b.N[i] = -INFINITY;
      b.B[i] = -INFINITY;
    } else {
      uint8_t xn = dsq[i];
      double bb = -INFINITY;
      for (size_t k = 1; k <= m; k++) bb = lse(bb, s.tbm[k] + s.msc[(size_t)xn * (m + 1) + k] + b.M[nr + k]);
      b.B[i] = bb;
      b.C[i] = b.C[i + 1] + cl;
      b.J[i] = lse(b.J[i + 1] + jl, bb + jm);
      b.N[i] = lse(b.N[i + 1] + nl, bb + nm);
    }
    b.E[i] = lse(b.J[i] + el, b.C[i] + em);
    if (i == 0) break;
    for (size_t k = m; k >= 1; k--) {
      double mv = b.E[i], iv = -INFINITY, dv = b.E[i];
      if (k < m) {
        dv = lse(dv, s.t[T_DD][k] + b.D[cr + k + 1]);
        mv = lse(mv, s.t[T_MD][k] + b.D[cr + k + 1]);
        if (i < l) {
          uint8_t xn = dsq[i];
          double nextm = s.msc[(size_t)xn * (m + 1) + k + 1] + b.M[nr + k + 1];
          double nexti = s.isc[(size_t)xn * (m + 1) + k] + b.I[nr + k];
          mv = lse(mv, lse(s.t[T_MM][k] + nextm, s.t[T_MI][k] + nexti));
          iv = lse(s.t[T_IM][k] + nextm, s.t[T_II][k] + nexti);
          dv = lse(dv, s.t[T_DM][k] + nextm);
        }
      }
      b.M[cr + k] = mv;
      b.I[cr + k] = iv;
      b.D[cr + k] = dv;
    }
  }
  return b.N[0];
}

double forward_logspace_f64(const Profile& p, const uint8_t* dsq, size_t l, bool multihit, int kind, size_t idx,
                            double delta) {
  if (l == 0 || p.m == 0) return -INFINITY;
  Lsp s = promote(p, kind, idx, delta);
  LogMats f;
  return fwd64(s, dsq, l, Xsc::make(l, multihit), f);
}

// Expected counts (all natural-log-score gradients of the Forward score):
//   d_msc[x*(M+1)+k], d_isc[x*(M+1)+k]  (25 x (M+1) each)
//   d_t[q*(M+1)+k] for q in MM MI MD IM II DM DD (source node k)
//   d_tbm[k]
// Returns lnZ from the forward pass and writes the backward score to *bsc.
double expected_counts_f64(const Profile& p, const uint8_t* dsq, size_t l, bool multihit, double* d_msc,
                           double* d_isc, double* d_t, double* d_tbm, double* bsc) {
  const size_t m = p.m, w1 = m + 1, w = m + 2;
  for (size_t q = 0; q < (size_t)NCODE * w1; q++) { d_msc[q] = 0; d_isc[q] = 0; }
  for (size_t q = 0; q < 7 * w1; q++) d_t[q] = 0;
  for (size_t q = 0; q < w1; q++) d_tbm[q] = 0;
  if (l == 0 || m == 0) return -INFINITY;
  Lsp s = promote(p, 0, 0, 0);
  Xsc xs = Xsc::make(l, multihit);
  LogMats f, b;
  double z = fwd64(s, dsq, l, xs, f);
  double zb = bwd64(s, dsq, l, xs, b);
  if (bsc) *bsc = zb;
  for (size_t i = 1; i <= l; i++) {
    uint8_t x = dsq[i - 1];
    const size_t cr = i * w, nr = (i + 1) * w, pr = (i - 1) * w;
    for (size_t k = 1; k <= m; k++) {
      d_msc[(size_t)x * w1 + k] += std::exp(f.M[cr + k] + b.M[cr + k] - z);
      if (k < m) d_isc[(size_t)x * w1 + k] += std::exp(f.I[cr + k] + b.I[cr + k] - z);
      // entry B(i-1) -> M_k at row i
      d_tbm[k] += std::exp(f.B[i - 1] + s.tbm[k] + s.msc[(size_t)x * w1 + k] + b.M[cr + k] - z);
      if (k >= 2) {
        double em = s.msc[(size_t)x * w1 + k] + b.M[cr + k];
        d_t[T_MM * w1 + k - 1] += std::exp(f.M[pr + k - 1] + s.t[T_MM][k - 1] + em - z);
        d_t[T_IM * w1 + k - 1] += std::exp(f.I[pr + k - 1] + s.t[T_IM][k - 1] + em - z);
        d_t[T_DM * w1 + k - 1] += std::exp(f.D[pr + k - 1] + s.t[T_DM][k - 1] + em - z);
        d_t[T_MD * w1 + k - 1] += std::exp(f.M[cr + k - 1] + s.t[T_MD][k - 1] + b.D[cr + k] - z);
        d_t[T_DD * w1 + k - 1] += std::exp(f.D[cr + k - 1] + s.t[T_DD][k - 1] + b.D[cr + k] - z);
      }
      if (k < m && i < l) {
        uint8_t xn = dsq[i];
        double ei = s.isc[(size_t)xn * w1 + k] + b.I[nr + k];
        d_t[T_MI * w1 + k] += std::exp(f.M[cr + k] + s.t[T_MI][k] + ei - z);
        d_t[T_II * w1 + k] += std::exp(f.I[cr + k] + s.t[T_II][k] + ei - z);
      }
    }
  }
  return z;
}

// FP64 log-space posterior of M_k / I_k at residue i, (L+1)*(M+1) each.
double posterior_f64(const Profile& p, const uint8_t* dsq, size_t l, bool multihit, double* pm, double* pi) {
  const size_t m = p.m, w1 = m + 1, w = m + 2;
  for (size_t q = 0; q < (l + 1) * w1; q++) { pm[q] = 0; pi[q] = 0; }
  if (l == 0 || m == 0) return -INFINITY;
  Lsp s = promote(p, 0, 0, 0);
  Xsc xs = Xsc::make(l, multihit);
  LogMats f, b;
  double z = fwd64(s, dsq, l, xs, f);
  bwd64(s, dsq, l, xs, b);
  for (size_t i = 1; i <= l; i++)
    for (size_t k = 1; k <= m; k++) {
      pm[i * w1 + k] = std::exp(f.M[i * w + k] + b.M[i * w + k] - z);
      if (k < m) pi[i * w1 + k] = std::exp(f.I[i * w + k] + b.I[i * w + k] - z);
    }
  return z;
}

}  // namespace sxo
