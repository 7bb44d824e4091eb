// TEST INFRASTRUCTURE ONLY — CPU oracle (see sx_oracle.hpp).  Each function
// cites the reference file:line it restates.  Build: oracle/Makefile.
#include "sx_oracle.hpp"

#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <thread>

namespace sxo {

// ---------------------------------------------------------------- alphabet
// src/hmmer/alphabet.rs:36-39
const float BG[K] = {0.0787945f, 0.0151600f, 0.0535222f, 0.0668298f, 0.0397062f, 0.0695071f, 0.0229198f,
                     0.0590092f, 0.0594422f, 0.0963728f, 0.0237718f, 0.0414386f, 0.0482904f, 0.0395639f,
                     0.0540978f, 0.0683364f, 0.0540687f, 0.0673417f, 0.0114135f, 0.0304133f};

// src/hmmer/alphabet.rs:42-54
std::vector<int> degenerate_members(uint8_t code) {
  switch (code) {
    case CODE_B: return {2, 11};
    case CODE_J: return {7, 9};
    case CODE_Z: return {3, 13};
    case CODE_X: {
      std::vector<int> v(20);
      for (int i = 0; i < 20; i++) v[i] = i;
      return v;
    }
    default: return {};
  }
}

// src/hmmer/alphabet.rs:58-88
uint8_t encode_residue(uint8_t b) {
  uint8_t c = (b >= 'a' && b <= 'z') ? (uint8_t)(b - 32) : b;
  switch (c) {
    case 'A': return 0;
    case 'C': case 'U': return 1;
    case 'D': return 2;
    case 'E': return 3;
    case 'F': return 4;
    case 'G': return 5;
    case 'H': return 6;
    case 'I': return 7;
    case 'K': case 'O': return 8;
    case 'L': return 9;
    case 'M': return 10;
    case 'N': return 11;
    case 'P': return 12;
    case 'Q': return 13;
    case 'R': return 14;
    case 'S': return 15;
    case 'T': return 16;
    case 'V': return 17;
    case 'W': return 18;
    case 'Y': return 19;
    case 'B': return CODE_B;
    case 'J': return CODE_J;
    case 'Z': return CODE_Z;
    case 'X': return CODE_X;
    case '*': case '-': case '.': case '_': case '~': return CODE_STAR;
    default: return (c >= 'A' && c <= 'Z') ? CODE_X : CODE_STAR;
  }
}

// src/hmmer/alphabet.rs:91-93 (ASCII whitespace dropped)
std::vector<uint8_t> encode(const std::string& seq) {
  std::vector<uint8_t> out;
  out.reserve(seq.size());
  for (unsigned char b : seq) {
    if (b == ' ' || b == '\t' || b == '\n' || b == '\r' || b == '\f') continue;
    out.push_back(encode_residue(b));
  }
  return out;
}

// ---------------------------------------------------------------- model
// src/hmmer/model.rs:248-260
std::vector<float> Hmm::occupancy() const {
  std::vector<float> occ(m + 1, 0.0f);
  if (m == 0) return occ;
  occ[1] = t[0][T_MI] + t[0][T_MM];
  for (size_t k = 2; k <= m; k++) {
    const auto& tk = t[k - 1];
    occ[k] = occ[k - 1] * (tk[T_MM] + tk[T_MI]) + (1.0f - occ[k - 1]) * tk[T_DM];
  }
  return occ;
}

static inline float lnp_f(float p) { return p > 0.0f ? (float)std::log((double)p) : NEG_INF; }

// src/hmmer/model.rs:146-245
Profile configure(const Hmm& h) {
  Profile p;
  const size_t m = h.m, w = m + 1;
  p.msc.assign((size_t)NCODE * w, NEG_INF);
  for (size_t k = 1; k <= m; k++) {
    float sc[NCODE];
    for (int x = 0; x < NCODE; x++) sc[x] = NEG_INF;
    for (int x = 0; x < K; x++) {
      double pr = (double)h.mat[k][x];
      sc[x] = pr > 0.0 ? (float)std::log(pr / (double)BG[x]) : NEG_INF;
    }
    for (uint8_t code = 20; code <= 23; code++) {
      float num = 0.0f, den = 0.0f;
      for (int y : degenerate_members(code)) {
        num += sc[y] * BG[y];
        den += BG[y];
      }
      sc[code] = den > 0.0f ? num / den : 0.0f;
    }
    sc[CODE_STAR] = NEG_INF;
    for (int x = 0; x < NCODE; x++) p.msc[(size_t)x * w + k] = sc[x];
  }
  auto vec = [&]() { return std::vector<float>(w, NEG_INF); };
  p.t_mm = vec(); p.t_mi = vec(); p.t_md = vec(); p.t_im = vec(); p.t_ii = vec(); p.t_dm = vec(); p.t_dd = vec();
  for (size_t k = 1; k < m; k++) {
    const auto& t = h.t[k];
    p.t_mm[k] = lnp_f(t[T_MM]);
    p.t_mi[k] = lnp_f(t[T_MI]);
    p.t_md[k] = lnp_f(t[T_MD]);
    p.t_im[k] = lnp_f(t[T_IM]);
    p.t_ii[k] = lnp_f(t[T_II]);
    p.t_dm[k] = lnp_f(t[T_DM]);
    p.t_dd[k] = lnp_f(t[T_DD]);
  }
  if (m >= 1) {
    p.t_dm[1] = NEG_INF;
    p.t_dd[1] = NEG_INF;
  }
  std::vector<float> occ = h.occupancy();
  float z = 0.0f;
  for (size_t k = 1; k < occ.size(); k++) z += occ[k] * (float)(m - k + 1);
  p.t_bm = vec();
  for (size_t k = 1; k <= m; k++)
    p.t_bm[k] = (z > 0.0f && occ[k] > 0.0f) ? (float)std::log((double)(occ[k] / z)) : NEG_INF;
  float mf = (float)m;
  p.msv_tbm = std::log(2.0f / (mf * (mf + 1.0f)));
  auto ex = [](const std::vector<float>& v) {
    std::vector<float> o(v.size());
    for (size_t i = 0; i < v.size(); i++) o[i] = std::exp(v[i]);
    return o;
  };
  p.mo = ex(p.msc);
  p.p_mm = ex(p.t_mm); p.p_mi = ex(p.t_mi); p.p_md = ex(p.t_md); p.p_im = ex(p.t_im);
  p.p_ii = ex(p.t_ii); p.p_dm = ex(p.t_dm); p.p_dd = ex(p.t_dd); p.p_bm = ex(p.t_bm);
  p.name = h.name; p.acc = h.acc; p.desc = h.desc; p.m = m;
  if (h.compo) p.compo = *h.compo;
  else for (int x = 0; x < K; x++) p.compo[x] = BG[x];
  p.ga = h.ga; p.tc = h.tc; p.nc = h.nc; p.stats = h.stats;
  return p;
}

// src/hmmer/model.rs:284-312
Xsc Xsc::make(size_t l, bool multihit) {
  float nj = multihit ? 1.0f : 0.0f;
  float pmove = (2.0f + nj) / ((float)l + 2.0f + nj);
  float ploop = 1.0f - pmove;
  float lloop = (float)std::log((double)ploop);
  float lmove = (float)std::log((double)pmove);
  Xsc x;
  x.n_loop = x.j_loop = x.c_loop = lloop;
  x.n_move = x.j_move = x.c_move = lmove;
  if (multihit) { x.e_move = -LN2F; x.e_loop = -LN2F; x.p.e_move = 0.5f; x.p.e_loop = 0.5f; }
  else { x.e_move = 0.0f; x.e_loop = NEG_INF; x.p.e_move = 1.0f; x.p.e_loop = 0.0f; }
  x.p.n_loop = x.p.j_loop = x.p.c_loop = ploop;
  x.p.n_move = x.p.j_move = x.p.c_move = pmove;
  return x;
}

// src/hmmer/model.rs:334-337
float null_score(size_t l) {
  float p1 = (float)l / ((float)l + 1.0f);
  return (float)((double)l * std::log((double)p1) + std::log(1.0 - (double)p1));
}

// ---------------------------------------------------------------- parser
// src/hmmer/parse.rs:66-236 (record parser), 259-298 (token helpers)
namespace {
std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) a++;
  while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}
std::string trim_start(const std::string& s) {
  size_t a = 0;
  while (a < s.size() && std::isspace((unsigned char)s[a])) a++;
  return s.substr(a);
}
std::vector<std::string> split_ws(const std::string& s) {
  std::vector<std::string> out;
  size_t i = 0, n = s.size();
  while (i < n) {
    while (i < n && std::isspace((unsigned char)s[i])) i++;
    size_t j = i;
    while (j < n && !std::isspace((unsigned char)s[j])) j++;
    if (j > i) out.push_back(s.substr(i, j - i));
    i = j;
  }
  return out;
}
bool parse_f64(const std::string& t, double& v) {
  if (t.empty()) return false;
  char* end = nullptr;
  v = std::strtod(t.c_str(), &end);
  return end == t.c_str() + t.size();
}
bool parse_f32(const std::string& t, float& v) {
  if (t.empty()) return false;
  char* end = nullptr;
  v = std::strtof(t.c_str(), &end);
  return end == t.c_str() + t.size();
}
bool parse_usize(const std::string& t, size_t& v) {
  if (t.empty()) return false;
  size_t i = (t[0] == '+') ? 1 : 0;
  if (i == t.size()) return false;
  size_t acc = 0;
  for (; i < t.size(); i++) {
    if (t[i] < '0' || t[i] > '9') return false;
    acc = acc * 10 + (size_t)(t[i] - '0');
  }
  v = acc;
  return true;
}
// parse.rs:268-277
bool tok_prob(const std::string& tok, float& out, std::string& err) {
  if (tok == "*") { out = 0.0f; return true; }
  double v;
  if (!parse_f64(tok, v)) { err = "non-numeric probability token \"" + tok + "\""; return false; }
  if (!std::isfinite(v) || v < 0.0) { err = "invalid -ln(p) value \"" + tok + "\""; return false; }
  out = (float)std::exp(-v);
  return true;
}
// parse.rs:279-287
bool fill_probs(const std::vector<std::string>& toks, size_t off, float* out, std::string& err) {
  if (toks.size() < off + K) {
    err = "expected 20 values, found " + std::to_string(toks.size() - std::min(off, toks.size()));
    return false;
  }
  for (int i = 0; i < K; i++) if (!tok_prob(toks[off + i], out[i], err)) return false;
  return true;
}
// parse.rs:289-298
bool fill_trans(const std::string& line, float* out, std::string& err) {
  auto toks = split_ws(line);
  if (toks.size() < 7) { err = "expected 7 transition values, found " + std::to_string(toks.size()); return false; }
  for (int i = 0; i < 7; i++) if (!tok_prob(toks[i], out[i], err)) return false;
  return true;
}

struct Reader {
  std::vector<std::string> lines;
  size_t pos = 0;
  size_t lineno = 0;
  std::string source;
  bool next(std::string& l) {
    if (pos >= lines.size()) return false;
    l = lines[pos++];
    lineno++;
    return true;
  }
  std::string errmsg(const std::string& m) const { return source + " line " + std::to_string(lineno) + ": " + m; }
};

// returns 1 = record, 0 = EOF, -1 = error
int parse_record(Reader& r, Hmm& h, std::string& err) {
  std::string first, line;
  for (;;) {
    if (!r.next(first)) return 0;
    if (trim(first).empty()) continue;
    break;
  }
  if (first.rfind("HMMER3", 0) != 0) {
    if (first.rfind("HMMER2", 0) == 0) { err = r.errmsg("HMMER2 format is not supported; convert with `hmmconvert`"); return -1; }
    err = r.errmsg("expected 'HMMER3/x' header, found \"" + first + "\"");
    return -1;
  }
  h = Hmm();
  bool alph_ok = false;
  auto need = [&](const char* what, std::string& out) -> bool {
    if (!r.next(out)) { err = r.source + ": unexpected end of file (" + what + ")"; return false; }
    return true;
  };
  for (;;) {
    if (!need("header", line)) return -1;
    std::string tr = trim_start(line);
    if (tr.rfind("HMM ", 0) == 0 || tr == "HMM" || tr.rfind("HMM\t", 0) == 0) break;
    size_t sp = 0;
    while (sp < tr.size() && !std::isspace((unsigned char)tr[sp])) sp++;
    std::string tag = tr.substr(0, sp);
    std::string rest = sp < tr.size() ? trim(tr.substr(sp + 1)) : std::string();
    if (tag == "NAME") h.name = rest;
    else if (tag == "ACC") h.acc = rest;
    else if (tag == "DESC") h.desc = rest;
    else if (tag == "LENG") {
      if (!parse_usize(rest, h.m)) { err = r.errmsg("bad LENG value \"" + rest + "\""); return -1; }
    } else if (tag == "ALPH") {
      std::string lo = rest;
      for (auto& c : lo) c = (char)std::tolower((unsigned char)c);
      if (lo != "amino") {
        err = r.errmsg("profile '" + h.name + "' has alphabet '" + rest + "'; only protein (amino) profiles are supported");
        return -1;
      }
      alph_ok = true;
    } else if (tag == "GA" || tag == "TC" || tag == "NC") {
      auto c = cutoff_pair(rest);
      if (!c) { err = r.errmsg("bad " + tag + " line"); return -1; }
      if (tag == "GA") h.ga = c; else if (tag == "TC") h.tc = c; else h.nc = c;
    } else if (tag == "STATS") {
      auto f = split_ws(rest);
      if (f.size() >= 4) {
        double a, b;
        if (!parse_f64(f[2], a) || !parse_f64(f[3], b)) { err = r.errmsg("bad STATS value"); return -1; }
        if (f[1] == "MSV") h.stats.msv = std::make_pair(a, b);
        else if (f[1] == "VITERBI") h.stats.viterbi = std::make_pair(a, b);
        else if (f[1] == "FORWARD") h.stats.forward = std::make_pair(a, b);
      }
    }
  }
  if (h.m == 0) { err = r.errmsg("profile '" + h.name + "' has no LENG"); return -1; }
  if (!alph_ok) { err = r.errmsg("profile '" + h.name + "' has no ALPH line"); return -1; }
  if (!need("transition header", line)) return -1;
  h.mat.assign(h.m + 1, std::array<float, K>{});
  h.t.assign(h.m + 1, std::array<float, 7>{});
  std::string l1, body_first;
  if (!need("model body", l1)) return -1;
  if (trim_start(l1).rfind("COMPO", 0) == 0) {
    auto toks = split_ws(l1);
    std::array<float, K> c{};
    std::string e;
    if (!fill_probs(toks, 1, c.data(), e)) { err = r.errmsg("COMPO: " + e); return -1; }
    h.compo = c;
    if (!need("node-0 insert line", body_first)) return -1;
  } else {
    body_first = l1;
  }
  if (split_ws(body_first).size() < (size_t)K) { err = r.errmsg("truncated node-0 insert line"); return -1; }
  std::string tr0;
  if (!need("node-0 transitions", tr0)) return -1;
  {
    std::string e;
    if (!fill_trans(tr0, h.t[0].data(), e)) { err = r.errmsg("node 0 transitions: " + e); return -1; }
  }
  for (size_t k = 1; k <= h.m; k++) {
    std::string ml, il, tl, e;
    if (!need("match line", ml)) return -1;
    auto toks = split_ws(ml);
    size_t idx;
    if (toks.empty() || !parse_usize(toks[0], idx)) { err = r.errmsg("bad match-line node index"); return -1; }
    if (idx != k) { err = r.errmsg("node index " + std::to_string(idx) + ", expected " + std::to_string(k)); return -1; }
    if (toks.size() < 1 + (size_t)K) { err = r.errmsg("truncated match emissions at node " + std::to_string(k)); return -1; }
    if (!fill_probs(toks, 1, h.mat[k].data(), e)) { err = r.errmsg("node " + std::to_string(k) + ": " + e); return -1; }
    if (!need("insert line", il)) return -1;
    if (split_ws(il).size() < (size_t)K) { err = r.errmsg("truncated insert emissions at node " + std::to_string(k)); return -1; }
    if (!need("transition line", tl)) return -1;
    if (!fill_trans(tl, h.t[k].data(), e)) { err = r.errmsg("node " + std::to_string(k) + " transitions: " + e); return -1; }
  }
  for (;;) {
    std::string l;
    if (!r.next(l)) break;
    std::string t = trim(l);
    if (t.empty()) continue;
    if (t == "//") break;
    err = r.errmsg("expected '//', found \"" + l + "\"");
    return -1;
  }
  return 1;
}
}  // namespace

std::optional<std::pair<float, float>> cutoff_pair(const std::string& rest) {
  std::string cleaned = rest;
  for (auto& c : cleaned) if (c == ';') c = ' ';
  auto toks = split_ws(cleaned);
  if (toks.empty()) return std::nullopt;
  float a;
  if (!parse_f32(toks[0], a)) return std::nullopt;
  float b = a;
  if (toks.size() > 1) {
    float bb;
    if (parse_f32(toks[1], bb)) b = bb;
  }
  return std::make_pair(a, b);
}

bool parse_hmm_text(const std::string& text, const std::string& source, std::vector<Hmm>& out, std::string& err) {
  Reader r;
  r.source = source;
  size_t i = 0;
  while (i < text.size()) {
    size_t j = text.find('\n', i);
    if (j == std::string::npos) j = text.size();
    std::string l = text.substr(i, j - i);
    while (!l.empty() && (l.back() == '\r' || l.back() == '\n')) l.pop_back();
    r.lines.push_back(l);
    i = j + 1;
  }
  out.clear();
  for (;;) {
    Hmm h;
    int rc = parse_record(r, h, err);
    if (rc == 0) return true;
    if (rc < 0) return false;
    out.push_back(std::move(h));
  }
}

bool parse_hmm_path(const std::string& path, std::vector<Hmm>& out, std::string& err) {
  gzFile f = gzopen(path.c_str(), "rb");  // transparently reads plain or gzip
  if (!f) { err = "opening HMM file " + path; return false; }
  std::string text;
  char buf[1 << 16];
  int n;
  while ((n = gzread(f, buf, sizeof buf)) > 0) text.append(buf, (size_t)n);
  gzclose(f);
  return parse_hmm_text(text, path, out, err);
}

// ---------------------------------------------------------------- dp
static inline float fmax_r(float a, float b) { return a > b ? a : b; }  // dp.rs:21-27

// dp.rs:32-40
float logsum(float a, float b) {
  float hi, lo;
  if (a > b) { hi = a; lo = b; } else { hi = b; lo = a; }
  float d = hi - lo;
  if (!(d < 30.0f)) return hi;
  return hi + std::log1p(std::exp(-d));
}

static inline float lnf(float x) { return x > 0.0f ? std::log(x) : NEG_INF; }  // dp.rs:200-206

void Specials::reset(size_t l) {
  for (auto* v : {&n, &b, &e, &j, &c}) v->assign(l + 1, NEG_INF);
}

static void rows6(DpBuf& buf, size_t w, float fill) {
  for (auto* v : {&buf.a, &buf.b, &buf.c, &buf.d, &buf.e, &buf.f}) v->assign(w, fill);
}

// dp.rs:92-145 (msv_kernel; the 8-wide e8 grouping only reorders exact maxes)
float msv(const Profile& p, const uint8_t* dsq, size_t l, DpBuf& buf) {
  const size_t m = p.m;
  if (l == 0 || m == 0) return NEG_INF;
  float lf = (float)l;
  float tloop = std::log(lf / (lf + 3.0f));
  float tmove = std::log(3.0f / (lf + 3.0f));
  float tbmk = p.msv_tbm;
  float tec = -LN2F, tej = -LN2F;
  rows6(buf, m + 1, NEG_INF);
  float* prev = buf.a.data();
  float* cur = buf.b.data();
  float xn = 0.0f, xb = tmove, xj = NEG_INF, xc = NEG_INF;
  for (size_t i = 0; i < l; i++) {
    const float* rs = p.msc_row(dsq[i]);
    float be = xb + tbmk;
    float xe = NEG_INF;
    for (size_t k = 1; k <= m; k++) {
      float v = rs[k] + fmax_r(prev[k - 1], be);
      cur[k] = v;
      xe = fmax_r(xe, v);
    }
    cur[0] = NEG_INF;
    xj = fmax_r(xj + tloop, xe + tej);
    xc = fmax_r(xc + tloop, xe + tec);
    xn += tloop;
    xb = fmax_r(xn + tmove, xj + tmove);
    std::swap(prev, cur);
  }
  return xc + tmove;
}

// dp.rs:152-189
float viterbi_score(const Profile& p, const uint8_t* dsq, size_t l, const Xsc& xs, DpBuf& buf) {
  const size_t m = p.m;
  if (l == 0 || m == 0) return NEG_INF;
  const size_t w = m + 1;
  rows6(buf, w, NEG_INF);
  float *mp = buf.a.data(), *ip = buf.b.data(), *dp = buf.c.data();
  float *mc = buf.d.data(), *ic = buf.e.data(), *dc = buf.f.data();
  float xn = 0.0f, xb = xs.n_move, xj = NEG_INF, xc = NEG_INF;
  for (size_t i = 0; i < l; i++) {
    uint8_t x = dsq[i];
    const float* rs = p.msc_row(x);
    bool ins_ok = x != CODE_STAR;
    mc[0] = NEG_INF; ic[0] = NEG_INF; dc[0] = NEG_INF;
    float xe = NEG_INF;
    for (size_t k = 1; k <= m; k++) {
      float sc = fmax_r(fmax_r(mp[k - 1] + p.t_mm[k - 1], ip[k - 1] + p.t_im[k - 1]),
                        fmax_r(xb + p.t_bm[k], dp[k - 1] + p.t_dm[k - 1]));
      float mv = sc + rs[k];
      mc[k] = mv;
      ic[k] = (k < m && ins_ok) ? fmax_r(mp[k] + p.t_mi[k], ip[k] + p.t_ii[k]) : NEG_INF;
      float dv = fmax_r(mc[k - 1] + p.t_md[k - 1], dc[k - 1] + p.t_dd[k - 1]);
      dc[k] = dv;
      xe = fmax_r(xe, fmax_r(mv, dv));
    }
    xj = fmax_r(xj + xs.j_loop, xe + xs.e_loop);
    xc = fmax_r(xc + xs.c_loop, xe + xs.e_move);
    xn += xs.n_loop;
    xb = fmax_r(xn + xs.n_move, xj + xs.j_move);
    std::swap(mp, mc); std::swap(ip, ic); std::swap(dp, dc);
  }
  return xc + xs.c_move;
}

static constexpr float RESCALE = 1.0e4f;  // dp.rs:197

// dp.rs:229-298
float forward(const Profile& p, const uint8_t* dsq, size_t l, const Xsc& xs, DpBuf& buf, Specials* sp) {
  const size_t m = p.m;
  if (l == 0 || m == 0) return NEG_INF;
  if (sp) sp->reset(l);
  const XscP xp = xs.p;
  const size_t w = m + 1;
  rows6(buf, w, 0.0f);
  float *mp = buf.a.data(), *ip = buf.b.data(), *dp = buf.c.data();
  float *mc = buf.d.data(), *ic = buf.e.data(), *dc = buf.f.data();
  float xn = 1.0f, xb = xp.n_move, xj = 0.0f, xc = 0.0f;
  double lnscale = 0.0;
  if (sp) { sp->n[0] = 0.0f; sp->b[0] = lnf(xb); }
  for (size_t i0 = 0; i0 < l; i0++) {
    uint8_t x = dsq[i0];
    const float* eo = p.mo_row(x);
    float ins = x != CODE_STAR ? 1.0f : 0.0f;
    float xe = 0.0f;
    for (size_t k = 1; k <= m; k++) {
      float mv = (xb * p.p_bm[k] + mp[k - 1] * p.p_mm[k - 1] + ip[k - 1] * p.p_im[k - 1] + dp[k - 1] * p.p_dm[k - 1]) * eo[k];
      mc[k] = mv;
      ic[k] = k < m ? (mp[k] * p.p_mi[k] + ip[k] * p.p_ii[k]) * ins : 0.0f;
      float dv = mc[k - 1] * p.p_md[k - 1] + dc[k - 1] * p.p_dd[k - 1];
      dc[k] = dv;
      xe += mv + dv;
    }
    xj = xj * xp.j_loop + xe * xp.e_loop;
    xc = xc * xp.c_loop + xe * xp.e_move;
    xn *= xp.n_loop;
    xb = xn * xp.n_move + xj * xp.j_move;
    if (xe > RESCALE) {
      float inv = 1.0f / xe;
      for (size_t k = 1; k <= m; k++) { mc[k] *= inv; ic[k] *= inv; dc[k] *= inv; }
      xn *= inv; xb *= inv; xj *= inv; xc *= inv;
      lnscale += std::log((double)xe);
      xe = 1.0f;
    }
    if (sp) {
      size_t i = i0 + 1;
      float ls = (float)lnscale;
      sp->n[i] = lnf(xn) + ls; sp->b[i] = lnf(xb) + ls; sp->e[i] = lnf(xe) + ls;
      sp->j[i] = lnf(xj) + ls; sp->c[i] = lnf(xc) + ls;
    }
    std::swap(mp, mc); std::swap(ip, ic); std::swap(dp, dc);
  }
  return (float)((double)lnf(xc * xp.c_move) + lnscale);
}

// dp.rs:301-392
float backward(const Profile& p, const uint8_t* dsq, size_t l, const Xsc& xs, DpBuf& buf, Specials& sp) {
  const size_t m = p.m;
  sp.reset(l);
  if (l == 0 || m == 0) return NEG_INF;
  const XscP xp = xs.p;
  const size_t w = m + 1;
  rows6(buf, w, 0.0f);
  float *mn = buf.a.data(), *inx = buf.b.data(), *dn = buf.c.data();
  float *mc = buf.d.data(), *ic = buf.e.data(), *dc = buf.f.data();
  float xc = xp.c_move;
  float xe = xc * xp.e_move;
  float xj = 0.0f, xn = 0.0f, xb;
  mn[m] = xe;
  dn[m] = xe;
  for (size_t k = m - 1; k >= 1; k--) {
    mn[k] = xe + dn[k + 1] * p.p_md[k];
    dn[k] = xe + dn[k + 1] * p.p_dd[k];
  }
  double lnscale = 0.0;
  sp.c[l] = lnf(xc);
  sp.e[l] = lnf(xe);
  for (size_t i = l - 1; i >= 1; i--) {
    uint8_t xnext = dsq[i];
    const float* eo = p.mo_row(xnext);
    float ins = xnext != CODE_STAR ? 1.0f : 0.0f;
    float b = 0.0f;
    for (size_t k = 1; k <= m; k++) b += mn[k] * p.p_bm[k] * eo[k];
    xb = b;
    xj = xj * xp.j_loop + xb * xp.j_move;
    xc *= xp.c_loop;
    xe = xj * xp.e_loop + xc * xp.e_move;
    xn = xn * xp.n_loop + xb * xp.n_move;
    mc[m] = xe; dc[m] = xe; ic[m] = 0.0f;
    float rowmax = std::fmax(std::fmax(std::fmax(std::fmax(xb, xe), xn), xj), xc);
    for (size_t k = m - 1; k >= 1; k--) {
      float mnext = mn[k + 1] * eo[k + 1];
      float iv = inx[k] * ins;
      float mv = mnext * p.p_mm[k] + iv * p.p_mi[k] + xe + dc[k + 1] * p.p_md[k];
      mc[k] = mv;
      ic[k] = mnext * p.p_im[k] + iv * p.p_ii[k];
      dc[k] = mnext * p.p_dm[k] + dc[k + 1] * p.p_dd[k] + xe;
      if (mv > rowmax) rowmax = mv;
    }
    if (rowmax > RESCALE) {
      float inv = 1.0f / rowmax;
      for (size_t k = 1; k <= m; k++) { mc[k] *= inv; ic[k] *= inv; dc[k] *= inv; }
      xb *= inv; xe *= inv; xn *= inv; xj *= inv; xc *= inv;
      lnscale += std::log((double)rowmax);
    }
    float ls = (float)lnscale;
    sp.n[i] = lnf(xn) + ls; sp.b[i] = lnf(xb) + ls; sp.e[i] = lnf(xe) + ls;
    sp.j[i] = lnf(xj) + ls; sp.c[i] = lnf(xc) + ls;
    std::swap(mn, mc); std::swap(inx, ic); std::swap(dn, dc);
  }
  const float* eo = p.mo_row(dsq[0]);
  float b = 0.0f;
  for (size_t k = 1; k <= m; k++) b += mn[k] * p.p_bm[k] * eo[k];
  float ls = (float)lnscale;
  sp.b[0] = lnf(b) + ls;
  sp.n[0] = logsum(sp.n[1] + xs.n_loop, sp.b[0] + xs.n_move);
  return sp.n[0];
}

// dp.rs:420-439
void Matrix::reset(size_t m_, size_t l_) {
  m = m_; l = l_;
  size_t n = (l + 1) * (m + 1);
  for (auto* v : {&mm, &im, &dm}) v->assign(n, 0.0f);
  lnscale.assign(l + 2, 0.0);
  sp.reset(l);
  for (auto* v : {&xn, &xb, &xe, &xj, &xc}) v->assign(l + 1, 0.0f);
  scale.assign(l + 1, 1.0f);
}

// dp.rs:442-513
float forward_matrix(const Profile& p, const uint8_t* dsq, size_t l, const Xsc& xs, Matrix& fx) {
  const size_t m = p.m;
  fx.reset(m, l);
  if (l == 0 || m == 0) return NEG_INF;
  const XscP xp = xs.p;
  const size_t w = m + 1;
  float xn = 1.0f, xb = xp.n_move, xj = 0.0f, xc = 0.0f;
  double lnscale = 0.0;
  fx.sp.n[0] = 0.0f;
  fx.sp.b[0] = lnf(xb);
  fx.xn[0] = xn;
  fx.xb[0] = xb;
  for (size_t i = 1; i <= l; i++) {
    uint8_t x = dsq[i - 1];
    const float* eo = p.mo_row(x);
    float ins = x != CODE_STAR ? 1.0f : 0.0f;
    size_t pb = (i - 1) * w, cb = i * w;
    float xe = 0.0f;
    for (size_t k = 1; k <= m; k++) {
      float mv = (xb * p.p_bm[k] + fx.mm[pb + k - 1] * p.p_mm[k - 1] + fx.im[pb + k - 1] * p.p_im[k - 1] +
                  fx.dm[pb + k - 1] * p.p_dm[k - 1]) * eo[k];
      fx.mm[cb + k] = mv;
      fx.im[cb + k] = k < m ? (fx.mm[pb + k] * p.p_mi[k] + fx.im[pb + k] * p.p_ii[k]) * ins : 0.0f;
      float dv = fx.mm[cb + k - 1] * p.p_md[k - 1] + fx.dm[cb + k - 1] * p.p_dd[k - 1];
      fx.dm[cb + k] = dv;
      xe += mv + dv;
    }
    xj = xj * xp.j_loop + xe * xp.e_loop;
    xc = xc * xp.c_loop + xe * xp.e_move;
    xn *= xp.n_loop;
    xb = xn * xp.n_move + xj * xp.j_move;
    if (xe > RESCALE) {
      float inv = 1.0f / xe;
      for (size_t k = 1; k <= m; k++) { fx.mm[cb + k] *= inv; fx.im[cb + k] *= inv; fx.dm[cb + k] *= inv; }
      xn *= inv; xb *= inv; xj *= inv; xc *= inv;
      lnscale += std::log((double)xe);
      fx.scale[i] = xe;
      xe = 1.0f;
    }
    fx.xn[i] = xn; fx.xb[i] = xb; fx.xe[i] = xe; fx.xj[i] = xj; fx.xc[i] = xc;
    fx.lnscale[i] = lnscale;
    float ls = (float)lnscale;
    fx.sp.n[i] = lnf(xn) + ls; fx.sp.b[i] = lnf(xb) + ls; fx.sp.e[i] = lnf(xe) + ls;
    fx.sp.j[i] = lnf(xj) + ls; fx.sp.c[i] = lnf(xc) + ls;
  }
  return (float)((double)lnf(xc * xp.c_move) + lnscale);
}

// dp.rs:516-601
float backward_matrix(const Profile& p, const uint8_t* dsq, size_t l, const Xsc& xs, Matrix& bx) {
  const size_t m = p.m;
  bx.reset(m, l);
  if (l == 0 || m == 0) return NEG_INF;
  const XscP xp = xs.p;
  const size_t w = m + 1;
  float xc = xp.c_move;
  float xe = xc * xp.e_move;
  float xj = 0.0f, xn = 0.0f;
  size_t base = l * w;
  bx.mm[base + m] = xe;
  bx.dm[base + m] = xe;
  for (size_t k = m - 1; k >= 1; k--) {
    bx.mm[base + k] = xe + bx.dm[base + k + 1] * p.p_md[k];
    bx.dm[base + k] = xe + bx.dm[base + k + 1] * p.p_dd[k];
  }
  double lnscale = 0.0;
  bx.lnscale[l] = 0.0;
  bx.sp.c[l] = lnf(xc);
  bx.sp.e[l] = lnf(xe);
  for (size_t i = l - 1; i >= 1; i--) {
    uint8_t xnext = dsq[i];
    const float* eo = p.mo_row(xnext);
    float ins = xnext != CODE_STAR ? 1.0f : 0.0f;
    size_t nb = (i + 1) * w, cb = i * w;
    float xb = 0.0f;
    for (size_t k = 1; k <= m; k++) xb += bx.mm[nb + k] * p.p_bm[k] * eo[k];
    xj = xj * xp.j_loop + xb * xp.j_move;
    xc *= xp.c_loop;
    xe = xj * xp.e_loop + xc * xp.e_move;
    xn = xn * xp.n_loop + xb * xp.n_move;
    bx.mm[cb + m] = xe; bx.dm[cb + m] = xe; bx.im[cb + m] = 0.0f;
    float rowmax = std::fmax(std::fmax(std::fmax(std::fmax(xb, xe), xn), xj), xc);
    for (size_t k = m - 1; k >= 1; k--) {
      float mnext = bx.mm[nb + k + 1] * eo[k + 1];
      float iv = bx.im[nb + k] * ins;
      float mv = mnext * p.p_mm[k] + iv * p.p_mi[k] + xe + bx.dm[cb + k + 1] * p.p_md[k];
      bx.mm[cb + k] = mv;
      bx.im[cb + k] = mnext * p.p_im[k] + iv * p.p_ii[k];
      bx.dm[cb + k] = mnext * p.p_dm[k] + bx.dm[cb + k + 1] * p.p_dd[k] + xe;
      if (mv > rowmax) rowmax = mv;
    }
    if (rowmax > RESCALE) {
      float inv = 1.0f / rowmax;
      for (size_t k = 1; k <= m; k++) { bx.mm[cb + k] *= inv; bx.im[cb + k] *= inv; bx.dm[cb + k] *= inv; }
      xb *= inv; xe *= inv; xn *= inv; xj *= inv; xc *= inv;
      lnscale += std::log((double)rowmax);
    }
    bx.lnscale[i] = lnscale;
    float ls = (float)lnscale;
    bx.sp.n[i] = lnf(xn) + ls; bx.sp.b[i] = lnf(xb) + ls; bx.sp.e[i] = lnf(xe) + ls;
    bx.sp.j[i] = lnf(xj) + ls; bx.sp.c[i] = lnf(xc) + ls;
  }
  const float* eo = p.mo_row(dsq[0]);
  float b = 0.0f;
  for (size_t k = 1; k <= m; k++) b += bx.mm[w + k] * p.p_bm[k] * eo[k];
  bx.lnscale[0] = lnscale;
  bx.sp.b[0] = lnf(b) + (float)lnscale;
  bx.sp.n[0] = logsum(bx.sp.n[1] + xs.n_loop, bx.sp.b[0] + xs.n_move);
  return bx.sp.n[0];
}

// dp.rs:605-664
std::array<float, NCODE> null2_by_expectation(const Profile& p, const uint8_t* dsq, size_t l, const Xsc& xs,
                                              const Matrix& fx, const Matrix& bx) {
  (void)dsq;
  const size_t m = p.m, w = m + 1;
  double overall = (double)bx.sp.n[0];
  std::vector<double> pm(w, 0.0), pi(w, 0.0), rm(w, 0.0), ri(w, 0.0);
  double pncj = 0.0;
  for (size_t i = 1; i <= l; i++) {
    size_t row = i * w;
    double fac = std::exp(fx.lnscale[i] + bx.lnscale[i] - overall);
    double denom = 0.0;
    for (size_t k = 1; k <= m; k++) {
      double vm = (double)fx.mm[row + k] * (double)bx.mm[row + k] * fac;
      rm[k] = vm;
      denom += vm;
      double vi = k < m ? (double)fx.im[row + k] * (double)bx.im[row + k] * fac : 0.0;
      ri[k] = vi;
      denom += vi;
    }
    double n = std::exp((double)(fx.sp.n[i - 1] + bx.sp.n[i] + xs.n_loop) - overall);
    double j = std::exp((double)(fx.sp.j[i - 1] + bx.sp.j[i] + xs.j_loop) - overall);
    double c = std::exp((double)(fx.sp.c[i - 1] + bx.sp.c[i] + xs.c_loop) - overall);
    denom += n + j + c;
    if (denom > 0.0 && std::isfinite(denom)) {
      double inv = 1.0 / denom;
      for (size_t k = 1; k <= m; k++) { pm[k] += rm[k] * inv; pi[k] += ri[k] * inv; }
      pncj += (n + j + c) * inv;
    }
  }
  double ld = (double)std::max<size_t>(l, 1);
  double null2[NCODE] = {0};
  double isum = 0.0;
  for (double v : pi) isum += v;
  isum /= ld;
  double xfactor = pncj / ld;
  for (int x = 0; x < K; x++) {
    const float* row = p.mo_row((uint8_t)x);
    double v = 0.0;
    for (size_t k = 1; k <= m; k++) v += (pm[k] / ld) * (double)row[k];
    null2[x] = v + isum + xfactor;
  }
  for (uint8_t code = 20; code <= 23; code++) {
    auto mem = degenerate_members(code);
    double s = 0.0;
    for (int y : mem) s += null2[y];
    null2[code] = s / (double)mem.size();
  }
  null2[CODE_STAR] = 1.0;
  std::array<float, NCODE> out;
  for (int x = 0; x < NCODE; x++) out[x] = null2[x] > 0.0 ? (float)std::log(null2[x]) : NEG_INF;
  return out;
}

// dp.rs:691-904
std::vector<AliCoords> viterbi_trace(const Profile& p, const uint8_t* dsq, size_t l, const Xsc& xs) {
  const size_t m = p.m;
  if (l == 0 || m == 0) return {};
  const size_t w = m + 1, n = (l + 1) * w;
  enum : uint8_t { PMM = 0, PIM = 1, PDM = 2, PBM = 3, PMI = 0, PII = 1, PMD = 0, PDD = 1 };
  std::vector<float> vm(n, NEG_INF), vi(n, NEG_INF), vd(n, NEG_INF);
  std::vector<uint8_t> pm(n, 0), pi(n, 0), pd(n, 0);
  std::vector<float> xn(l + 1, NEG_INF), xb(l + 1, NEG_INF), xe(l + 1, NEG_INF), xj(l + 1, NEG_INF), xc(l + 1, NEG_INF);
  std::vector<std::pair<size_t, bool>> e_src(l + 1, {0, false});
  std::vector<char> b_from_j(l + 1, 0), j_from_e(l + 1, 0), c_from_e(l + 1, 0);
  xn[0] = 0.0f;
  xb[0] = xs.n_move;
  for (size_t i = 1; i <= l; i++) {
    uint8_t x = dsq[i - 1];
    const float* rs = p.msc_row(x);
    bool ins_ok = x != CODE_STAR;
    float best_e = NEG_INF;
    std::pair<size_t, bool> best_src{0, false};
    for (size_t k = 1; k <= m; k++) {
      size_t pc = (i - 1) * w + k, cc = i * w + k;
      float c0 = vm[pc - 1] + p.t_mm[k - 1];
      float c1 = vi[pc - 1] + p.t_im[k - 1];
      float c2 = vd[pc - 1] + p.t_dm[k - 1];
      float c3 = xb[i - 1] + p.t_bm[k];
      float sc = c0;
      uint8_t ptr = PMM;
      if (c1 > sc) { sc = c1; ptr = PIM; }
      if (c2 > sc) { sc = c2; ptr = PDM; }
      if (c3 > sc) { sc = c3; ptr = PBM; }
      vm[cc] = sc + rs[k];
      pm[cc] = ptr;
      if (k < m && ins_ok) {
        float a = vm[pc] + p.t_mi[k], b = vi[pc] + p.t_ii[k];
        if (a >= b) { vi[cc] = a; pi[cc] = PMI; } else { vi[cc] = b; pi[cc] = PII; }
      }
      float a = vm[cc - 1] + p.t_md[k - 1], b = vd[cc - 1] + p.t_dd[k - 1];
      if (a >= b) { vd[cc] = a; pd[cc] = PMD; } else { vd[cc] = b; pd[cc] = PDD; }
      if (vm[cc] > best_e) { best_e = vm[cc]; best_src = {k, false}; }
      if (vd[cc] > best_e) { best_e = vd[cc]; best_src = {k, true}; }
    }
    xe[i] = best_e;
    e_src[i] = best_src;
    float jl = xj[i - 1] + xs.j_loop, je = best_e + xs.e_loop;
    if (je > jl) { xj[i] = je; j_from_e[i] = 1; } else xj[i] = jl;
    float cl = xc[i - 1] + xs.c_loop, ce = best_e + xs.e_move;
    if (ce > cl) { xc[i] = ce; c_from_e[i] = 1; } else xc[i] = cl;
    xn[i] = xn[i - 1] + xs.n_loop;
    float bn = xn[i] + xs.n_move, bj = xj[i] + xs.j_move;
    if (bj > bn) { xb[i] = bj; b_from_j[i] = 1; } else xb[i] = bn;
  }
  if (!(xc[l] > NEG_INF)) return {};
  enum St { C, E, M, I, D, B, J, N };
  std::vector<AliCoords> out;
  St st = C;
  size_t k = 0, i = l;
  bool have_end = false;
  size_t end_j = 0, end_m = 0;
  size_t guard = 0;
  for (;;) {
    guard++;
    if (guard > 4 * (l + 2) * (m + 2)) break;
    switch (st) {
      case C:
        if (i == 0) goto done;
        if (c_from_e[i]) st = E; else i -= 1;
        break;
      case E: {
        auto [kk, del] = e_src[i];
        if (kk == 0) goto done;
        k = kk;
        st = del ? D : M;
        have_end = true; end_j = i; end_m = kk;
        break;
      }
      case M: {
        uint8_t ptr = pm[i * w + k];
        if (ptr == PMM) { st = M; k -= 1; i -= 1; }
        else if (ptr == PIM) { st = I; k -= 1; i -= 1; }
        else if (ptr == PDM) { st = D; k -= 1; i -= 1; }
        else {
          if (have_end) { out.push_back({i, end_j, k, end_m}); have_end = false; }
          st = B;
          i -= 1;
        }
        break;
      }
      case I:
        st = (pi[i * w + k] == PMI) ? M : I;
        i -= 1;
        break;
      case D:
        if (pd[i * w + k] == PMD) st = M; else st = D;
        k -= 1;
        break;
      case B: st = b_from_j[i] ? J : N; break;
      case J:
        if (j_from_e[i]) st = E; else i -= 1;
        break;
      case N: goto done;
    }
  }
done:
  std::reverse(out.begin(), out.end());
  return out;
}

// dp.rs:965-1023
static uint32_t esl_mix3(uint32_t a, uint32_t b, uint32_t c) {
  a -= b; a -= c; a ^= c >> 13;
  b -= c; b -= a; b ^= a << 8;
  c -= a; c -= b; c ^= b >> 13;
  a -= b; a -= c; a ^= c >> 12;
  b -= c; b -= a; b ^= a << 16;
  c -= a; c -= b; c ^= b >> 5;
  a -= b; a -= c; a ^= c >> 3;
  b -= c; b -= a; b ^= a << 10;
  c -= a; c -= b; c ^= b >> 15;
  return c;
}
EslRng::EslRng(uint32_t s) : seed(s), x(0) { reseed(); }
void EslRng::reseed() {
  x = esl_mix3(seed, 87654321u, 12345678u);
  if (x == 0) x = 42;
}
double EslRng::next() {
  x = x * 69069u + 1u;
  return (double)x / 4294967296.0;
}

// dp.rs:1026-1045
template <size_t N>
static void esl_fnorm(std::array<float, N>& v) {
  float sum = 0.0f, c = 0.0f;
  for (float xx : v) {
    float y = xx - c;
    float t = sum + y;
    c = (t - sum) - y;
    sum = t;
  }
  if (sum != 0.0f) for (auto& xx : v) xx /= sum;
  else for (auto& xx : v) xx = 1.0f / (float)N;
}
// dp.rs:1048-1059
template <size_t N>
static size_t esl_fchoose(EslRng& rng, const std::array<float, N>& p) {
  double norm = 0.0;
  for (float xx : p) norm += (double)xx;
  double roll = rng.next();
  double sum = 0.0;
  for (size_t i = 0; i < N; i++) {
    sum += (double)p[i];
    if (roll < sum / norm) return i;
  }
  return N - 1;
}

// dp.rs:1075-1258
std::vector<SampledDomain> stochastic_trace(const Profile& p, const Matrix& fx, const Xsc& xs, EslRng& rng) {
  enum St { C, E, M, I, D, B, J, N };
  const XscP xp = xs.p;
  const size_t m = p.m, w = m + 1;
  const size_t q_stripes = std::max<size_t>(2, (m > 0 ? m - 1 : 0) / 4 + 1);
  std::vector<SampledDomain> doms;
  std::optional<SampledDomain> cur;
  St s0 = C;
  size_t i = fx.l, k = 0, guard = 0;
  const size_t limit = 8 * (fx.l + 2) * (m + 2) + 64;
  for (;;) {
    guard++;
    if (guard > limit) break;
    St s1;
    switch (s0) {
      case C: {
        if (i == 0) goto done;
        std::array<float, 2> path = {fx.xc[i - 1] * xp.c_loop, fx.xe[i] * xp.e_move * fx.scale[i]};
        esl_fnorm(path);
        s1 = esl_fchoose(rng, path) == 0 ? C : E;
        break;
      }
      case E: {
        double roll = rng.next();
        float norm = (float)(1.0 / (double)fx.xe[i]);
        size_t row = i * w;
        double sum = 0.0;
        bool picked = false;
        size_t pk = 0;
        St pst = M;
        int passes = 0;
        while (!picked && passes < 1000) {
          passes++;
          for (size_t q = 0; q < q_stripes && !picked; q++) {
            for (size_t r = 0; r < 4; r++) {
              size_t kk = r * q_stripes + q + 1;
              if (kk <= m) {
                sum += (double)(fx.mm[row + kk] * norm);
                if (roll < sum) { picked = true; pk = kk; pst = M; break; }
              }
            }
            if (picked) break;
            for (size_t r = 0; r < 4; r++) {
              size_t kk = r * q_stripes + q + 1;
              if (kk <= m) {
                sum += (double)(fx.dm[row + kk] * norm);
                if (roll < sum) { picked = true; pk = kk; pst = D; break; }
              }
            }
          }
          if (picked) break;
          if (sum <= 0.0) break;
        }
        if (!picked) goto done;
        k = pk;
        cur = SampledDomain();
        s1 = pst;
        break;
      }
      case M: {
        if (cur) {
          if (cur->sqto == 0) { cur->sqto = i; cur->hmmto = k; }
          cur->sqfrom = i;
          cur->hmmfrom = k;
          cur->nodes.push_back(k);
        }
        size_t prow = (i - 1) * w;
        float mpv = 0, ipv = 0, dpv = 0, tmm = 0, tim = 0, tdm = 0;
        if (k >= 2) {
          mpv = fx.mm[prow + k - 1]; ipv = fx.im[prow + k - 1]; dpv = fx.dm[prow + k - 1];
          tmm = p.p_mm[k - 1]; tim = p.p_im[k - 1]; tdm = p.p_dm[k - 1];
        }
        std::array<float, 4> path = {fx.xb[i - 1] * p.p_bm[k], mpv * tmm, ipv * tim, dpv * tdm};
        esl_fnorm(path);
        size_t c = esl_fchoose(rng, path);
        k -= 1;
        i -= 1;
        s1 = c == 0 ? B : c == 1 ? M : c == 2 ? I : D;
        break;
      }
      case D: {
        size_t row = i * w;
        float mpv = 0, dpv = 0, tmd = 0, tdd = 0;
        if (k >= 2) { mpv = fx.mm[row + k - 1]; dpv = fx.dm[row + k - 1]; tmd = p.p_md[k - 1]; tdd = p.p_dd[k - 1]; }
        std::array<float, 2> path = {mpv * tmd, dpv * tdd};
        esl_fnorm(path);
        size_t c = esl_fchoose(rng, path);
        k -= 1;
        s1 = c == 0 ? M : D;
        break;
      }
      case I: {
        if (cur) cur->nodes.push_back(k);
        size_t prow = (i - 1) * w;
        std::array<float, 2> path = {fx.mm[prow + k] * p.p_mi[k], fx.im[prow + k] * p.p_ii[k]};
        esl_fnorm(path);
        size_t c = esl_fchoose(rng, path);
        i -= 1;
        s1 = c == 0 ? M : I;
        break;
      }
      case B: {
        if (cur) { doms.push_back(std::move(*cur)); cur.reset(); }
        std::array<float, 2> path = {fx.xn[i] * xp.n_move, fx.xj[i] * xp.j_move};
        esl_fnorm(path);
        s1 = esl_fchoose(rng, path) == 0 ? N : J;
        break;
      }
      case J: {
        if (i == 0) goto done;
        std::array<float, 2> path = {fx.xj[i - 1] * xp.j_loop, fx.xe[i] * xp.e_loop * fx.scale[i]};
        esl_fnorm(path);
        s1 = esl_fchoose(rng, path) == 0 ? J : E;
        break;
      }
      case N:
      default:
        if (i == 0) goto done;
        s1 = N;
        break;
    }
    if ((s1 == N || s1 == J || s1 == C) && s1 == s0) i -= 1;
    s0 = s1;
  }
done:
  std::reverse(doms.begin(), doms.end());
  return doms;
}

// dp.rs:1278-1306
void decode(const Profile& p, const Xsc& xs, const Matrix& fx, const Matrix& bx, Posterior& pp) {
  const size_t m = p.m, l = fx.l, w = m + 1;
  pp.m = m; pp.l = l;
  pp.pm.assign((l + 1) * w, 0.0f);
  pp.pi.assign((l + 1) * w, 0.0f);
  for (auto* v : {&pp.pn, &pp.pj, &pp.pc}) v->assign(l + 1, 0.0f);
  double overall = (double)bx.sp.n[0];
  for (size_t i = 1; i <= l; i++) {
    size_t row = i * w;
    double fac = std::exp(fx.lnscale[i] + bx.lnscale[i] - overall);
    for (size_t k = 1; k <= m; k++) {
      pp.pm[row + k] = (float)((double)fx.mm[row + k] * (double)bx.mm[row + k] * fac);
      if (k < m) pp.pi[row + k] = (float)((double)fx.im[row + k] * (double)bx.im[row + k] * fac);
    }
    pp.pn[i] = (float)std::exp((double)(fx.sp.n[i - 1] + bx.sp.n[i] + xs.n_loop) - overall);
    pp.pj[i] = (float)std::exp((double)(fx.sp.j[i - 1] + bx.sp.j[i] + xs.j_loop) - overall);
    pp.pc[i] = (float)std::exp((double)(fx.sp.c[i - 1] + bx.sp.c[i] + xs.c_loop) - overall);
  }
}

// dp.rs:1310-1350
std::array<float, NCODE> null2_from_posterior(const Profile& p, const Posterior& pp) {
  const size_t m = p.m, l = pp.l, w = m + 1;
  std::vector<float> sm(w, 0.0f);
  float si = 0.0f, sn = 0.0f, sj = 0.0f, sc = 0.0f;
  for (size_t i = 1; i <= l; i++) {
    size_t row = i * w;
    for (size_t k = 1; k <= m; k++) { sm[k] += pp.pm[row + k]; si += pp.pi[row + k]; }
    sn += pp.pn[i]; sj += pp.pj[i]; sc += pp.pc[i];
  }
  float norm = 1.0f / (float)std::max<size_t>(l, 1);
  float xfactor = sn * norm + sc * norm + sj * norm;
  float isum = si * norm;
  float null2[NCODE] = {0};
  for (int x = 0; x < K; x++) {
    const float* row = p.mo_row((uint8_t)x);
    float v = 0.0f;
    for (size_t k = 1; k <= m; k++) v += sm[k] * norm * row[k];
    null2[x] = v + isum + xfactor;
  }
  for (uint8_t code = 20; code <= 23; code++) {
    auto mem = degenerate_members(code);
    float s = 0.0f;
    for (int y : mem) s += null2[y];
    null2[code] = s / (float)mem.size();
  }
  null2[CODE_STAR] = 1.0f;
  std::array<float, NCODE> out;
  for (int x = 0; x < NCODE; x++) out[x] = null2[x] > 0.0f ? std::log(null2[x]) : NEG_INF;
  return out;
}

// dp.rs:1355-1564
std::optional<AliCoords> optimal_accuracy_coords(const Profile& p, const Xsc& xs, const Posterior& pp) {
  const size_t m = p.m, l = pp.l;
  if (l == 0 || m == 0) return std::nullopt;
  const size_t w = m + 1, n = (l + 1) * w;
  const XscP xp = xs.p;
  std::vector<float> om(n, NEG_INF), oi(n, NEG_INF), od(n, NEG_INF);
  std::vector<float> xe(l + 1, NEG_INF), xn(l + 1, NEG_INF), xj(l + 1, NEG_INF), xb(l + 1, NEG_INF), xc(l + 1, NEG_INF);
  xn[0] = 0.0f;
  xb[0] = 0.0f;
  auto gate = [](float t, float v) { return t > 0.0f ? v : 0.0f; };
  for (size_t i = 1; i <= l; i++) {
    size_t pr = (i - 1) * w, cr = i * w;
    float emax = NEG_INF;
    for (size_t k = 1; k <= m; k++) {
      float sv = gate(p.p_bm[k], xb[i - 1]);
      if (k >= 2) {
        sv = std::fmax(sv, gate(p.p_mm[k - 1], om[pr + k - 1]));
        sv = std::fmax(sv, gate(p.p_im[k - 1], oi[pr + k - 1]));
        sv = std::fmax(sv, gate(p.p_dm[k - 1], od[pr + k - 1]));
      } else {
        sv = std::fmax(sv, 0.0f);
      }
      float mv = sv + pp.pm[cr + k];
      om[cr + k] = mv;
      emax = std::fmax(emax, mv);
      float iv = std::fmax(gate(p.p_mi[k], om[pr + k]), gate(p.p_ii[k], oi[pr + k])) + pp.pi[cr + k];
      oi[cr + k] = iv;
    }
    od[cr + 1] = NEG_INF;
    for (size_t k = 2; k <= m; k++) {
      float a = gate(p.p_md[k - 1], om[cr + k - 1]);
      float b = gate(p.p_dd[k - 1], od[cr + k - 1]);
      od[cr + k] = std::fmax(a, b);
      emax = std::fmax(emax, od[cr + k]);
    }
    xe[i] = emax;
    float t1 = xp.j_loop == 0.0f ? 0.0f : xj[i - 1] + pp.pj[i];
    float t2 = xp.e_loop == 0.0f ? 0.0f : xe[i];
    xj[i] = std::fmax(t1, t2);
    t1 = xp.c_loop == 0.0f ? 0.0f : xc[i - 1] + pp.pc[i];
    t2 = xp.e_move == 0.0f ? 0.0f : xe[i];
    xc[i] = std::fmax(t1, t2);
    xn[i] = xp.n_loop == 0.0f ? 0.0f : xn[i - 1] + pp.pn[i];
    t1 = xp.n_move == 0.0f ? 0.0f : xn[i];
    t2 = xp.j_move == 0.0f ? 0.0f : xj[i];
    xb[i] = std::fmax(t1, t2);
  }
  enum St { C, E, M, I, D, B, J, N };
  const size_t q_stripes = std::max<size_t>(2, (m - 1) / 4 + 1);
  St s0 = C;
  size_t i = l, k = 0, guard = 0;
  const size_t limit = 8 * (l + 2) * (m + 2) + 64;
  bool have_first = false, have_last = false;
  size_t fi = 0, fk = 0, li = 0, lk = 0;
  auto dis = [](float t, float v) { return t == 0.0f ? NEG_INF : v; };
  for (;;) {
    guard++;
    if (guard > limit) break;
    St s1;
    switch (s0) {
      case C: {
        if (i == 0) goto done;
        float a = xp.c_loop == 0.0f ? NEG_INF : xc[i - 1] + pp.pc[i];
        float b = xp.e_move == 0.0f ? NEG_INF : xe[i];
        s1 = a > b ? C : E;
        break;
      }
      case E: {
        size_t row = i * w;
        float mx = NEG_INF;
        bool picked = false;
        size_t pk = 0;
        St pst = M;
        for (size_t q = 0; q < q_stripes; q++) {
          for (size_t r = 0; r < 4; r++) {
            size_t kk = r * q_stripes + q + 1;
            if (kk <= m && om[row + kk] >= mx) { mx = om[row + kk]; picked = true; pk = kk; pst = M; }
          }
          for (size_t r = 0; r < 4; r++) {
            size_t kk = r * q_stripes + q + 1;
            if (kk <= m && od[row + kk] > mx) { mx = od[row + kk]; picked = true; pk = kk; pst = D; }
          }
        }
        if (!picked) goto done;
        k = pk;
        s1 = pst;
        break;
      }
      case M: {
        if (!have_last) { have_last = true; li = i; lk = k; }
        have_first = true; fi = i; fk = k;
        size_t prow = (i - 1) * w;
        float mv = NEG_INF, iv = NEG_INF, dv = NEG_INF;
        if (k >= 2) {
          mv = dis(p.p_mm[k - 1], om[prow + k - 1]);
          iv = dis(p.p_im[k - 1], oi[prow + k - 1]);
          dv = dis(p.p_dm[k - 1], od[prow + k - 1]);
        }
        float bv = dis(p.p_bm[k], xb[i - 1]);
        float path[4] = {mv, iv, dv, bv};
        int best = 0;
        for (int t = 1; t < 4; t++) if (path[t] > path[best]) best = t;
        k -= 1;
        i -= 1;
        s1 = best == 0 ? M : best == 1 ? I : best == 2 ? D : B;
        break;
      }
      case D: {
        size_t row = i * w;
        float a = NEG_INF, b = NEG_INF;
        if (k >= 2) { a = dis(p.p_md[k - 1], om[row + k - 1]); b = dis(p.p_dd[k - 1], od[row + k - 1]); }
        k -= 1;
        s1 = a >= b ? M : D;
        break;
      }
      case I: {
        size_t prow = (i - 1) * w;
        float a = dis(p.p_mi[k], om[prow + k]);
        float b = dis(p.p_ii[k], oi[prow + k]);
        i -= 1;
        s1 = a >= b ? M : I;
        break;
      }
      case B: {
        float a = xp.n_move == 0.0f ? NEG_INF : xn[i];
        float b = xp.j_move == 0.0f ? NEG_INF : xj[i];
        if (a > b) s1 = N;
        else goto done;
        break;
      }
      case J:
      case N:
      default:
        goto done;
    }
    if ((s1 == N || s1 == J || s1 == C) && s1 == s0) i -= 1;
    if (s1 == N) break;
    s0 = s1;
  }
done:
  if (have_first && have_last) return AliCoords{fi, li, fk, lk};
  return std::nullopt;
}

// ---------------------------------------------------------------- pipeline
// pipeline.rs:87-95
double gumbel_surv(double x, double mu, double lambda) {
  double y = lambda * (x - mu);
  double ey = -std::exp(-y);
  if (std::fabs(ey) < 1e-5) return -ey;
  return 1.0 - std::exp(ey);
}
// pipeline.rs:98-104
double exp_logsurv(double x, double tau, double lambda) {
  if (x < tau) return 0.0;
  return -lambda * (x - tau);
}

// pipeline.rs:107-150
float bias_filter_score(const Profile& p, const uint8_t* dsq, size_t l) {
  const double l0 = 400.0, l1 = (double)p.m / 8.0;
  const double t[2][2] = {{l0 / (l0 + 1.0), 1.0 / (l0 + 1.0)}, {1.0 / (l1 + 1.0), l1 / (l1 + 1.0)}};
  const double pi[2] = {0.999, 0.001};
  double eo[NCODE][2];
  for (int x = 0; x < NCODE; x++) { eo[x][0] = 1.0; eo[x][1] = 1.0; }
  for (int x = 0; x < K; x++) { eo[x][0] = 1.0; eo[x][1] = (double)p.compo[x] / (double)BG[x]; }
  for (uint8_t code = 20; code <= 23; code++) {
    double e0 = 0, e1 = 0, z = 0;
    for (int y : degenerate_members(code)) { e0 += (double)BG[y]; e1 += (double)p.compo[y]; z += (double)BG[y]; }
    eo[code][0] = e0 / z;
    eo[code][1] = e1 / z;
  }
  eo[CODE_STAR][0] = 1.0;
  eo[CODE_STAR][1] = 1.0;
  double logsc = 0.0;
  size_t x1 = dsq[0];
  double d0 = eo[x1][0] * pi[0], d1 = eo[x1][1] * pi[1];
  double mx = std::fmax(std::fmax(d0, d1), std::numeric_limits<double>::min());
  d0 /= mx; d1 /= mx;
  logsc += std::log(mx);
  for (size_t i = 1; i < l; i++) {
    size_t x = dsq[i];
    double n0 = (d0 * t[0][0] + d1 * t[1][0]) * eo[x][0];
    double n1 = (d0 * t[0][1] + d1 * t[1][1]) * eo[x][1];
    mx = std::fmax(std::fmax(n0, n1), std::numeric_limits<double>::min());
    d0 = n0 / mx; d1 = n1 / mx;
    logsc += std::log(mx);
  }
  logsc += std::log(d0 + d1);
  double p1 = (double)l / ((double)l + 1.0);
  return (float)(logsc + (double)l * std::log(p1) + std::log(1.0 - p1));
}

namespace {
struct SpCoord { size_t idx, i, j, k, m; };

// pipeline.rs:308-327
bool sp_link(const SpCoord& h1, const SpCoord& h2) {
  int64_t nov = (int64_t)std::min(h1.j, h2.j) - (int64_t)std::max(h1.i, h2.i) + 1;
  float n = (float)std::min(h1.j - h1.i + 1, h2.j - h2.i + 1);
  if ((float)nov / n < 0.8f) return false;
  nov = (int64_t)std::min(h1.m, h2.m) - (int64_t)std::max(h1.k, h2.k);
  n = (float)std::min(h1.m - h1.k + 1, h2.m - h2.k + 1);
  if ((float)nov / n < 0.8f) return false;
  int64_t d1 = (int64_t)h1.i - (int64_t)h1.k, d2 = (int64_t)h2.i - (int64_t)h2.k;
  if (std::llabs(d1 - d2) <= 4) return true;
  d1 = (int64_t)h1.j - (int64_t)h1.m;
  d2 = (int64_t)h2.j - (int64_t)h2.m;
  return std::llabs(d1 - d2) <= 4;
}

// pipeline.rs:330-355
size_t single_linkage(const std::vector<SpCoord>& v, std::vector<size_t>& c) {
  size_t n = v.size();
  std::vector<size_t> a(n), b;
  for (size_t x = 0; x < n; x++) a[x] = n - x - 1;
  c.assign(n, 0);
  size_t nc = 0;
  while (!a.empty()) {
    size_t v0 = a.back();
    a.pop_back();
    b.push_back(v0);
    while (!b.empty()) {
      size_t x = b.back();
      b.pop_back();
      c[x] = nc;
      size_t ii = a.size();
      while (ii > 0) {
        ii--;
        if (sp_link(v[x], v[a[ii]])) {
          size_t wv = a[ii];
          a[ii] = a.back();
          a.pop_back();
          b.push_back(wv);
        }
      }
    }
    nc++;
  }
  return nc;
}

// pipeline.rs:489-525
std::vector<size_t> endpoint_counts(const std::vector<size_t>& vals, size_t lo, size_t hi) {
  std::vector<size_t> epc(hi - lo + 1, 0);
  for (size_t v : vals) epc[v - lo]++;
  return epc;
}
size_t argmax_u(const std::vector<size_t>& v) {
  size_t best = 0;
  for (size_t i = 0; i < v.size(); i++) if (v[i] > v[best]) best = i;
  return best;
}
size_t leftmost(const std::vector<size_t>& vals, size_t lo, size_t hi, size_t thr) {
  auto epc = endpoint_counts(vals, lo, hi);
  for (size_t o = 0; o < epc.size(); o++) if (epc[o] >= thr) return lo + o;
  return lo + argmax_u(epc);
}
size_t rightmost(const std::vector<size_t>& vals, size_t lo, size_t hi, size_t thr) {
  auto epc = endpoint_counts(vals, lo, hi);
  for (size_t o = epc.size(); o-- > 0;) if (epc[o] >= thr) return lo + o;
  return lo + argmax_u(epc);
}

// pipeline.rs:527-536
bool is_multidomain(const std::vector<float>& btot, const std::vector<float>& etot, size_t i, size_t j, float rt3) {
  float mx = -1.0f;
  for (size_t jj = i; jj <= j; jj++) {
    float v = std::fmin(etot[jj] - etot[i - 1], btot[j] - btot[jj - 1]);
    if (v > mx) mx = v;
  }
  return mx >= rt3;
}

// pipeline.rs:360-477
std::vector<std::pair<size_t, size_t>> region_trace_ensemble(const Profile& p, const uint8_t* dsq, size_t ireg,
                                                              size_t jreg, size_t l, Workspace& ws,
                                                              std::vector<float>& n2sc) {
  const size_t NSAMPLES = 200;
  const uint8_t* sub = dsq + (ireg - 1);
  size_t lr = jreg - ireg + 1;
  Xsc xs = Xsc::make(l, true);
  forward_matrix(p, sub, lr, xs, ws.fx);
  EslRng rng(42);
  for (size_t v = ireg; v <= jreg; v++) n2sc[v] = 0.0f;
  std::vector<SpCoord> sp;
  const size_t w = p.m + 1;
  float null2[NCODE] = {0};
  for (size_t t = 0; t < NSAMPLES; t++) {
    auto doms = stochastic_trace(p, ws.fx, xs, rng);
    size_t pos = 1;
    for (const auto& d : doms) {
      sp.push_back({t, d.sqfrom + ireg - 1, d.sqto + ireg - 1, d.hmmfrom, d.hmmto});
      float ld = (float)std::max<size_t>(d.nodes.size(), 1);
      for (int x = 0; x < K; x++) {
        const float* row = p.mo.data() + (size_t)x * w;
        float v = 0.0f;
        for (size_t kk : d.nodes) v += row[kk];
        null2[x] = v / ld;
      }
      for (uint8_t code = 20; code <= 23; code++) {
        auto mem = degenerate_members(code);
        float s = 0.0f;
        for (int y : mem) s += null2[y];
        null2[code] = s / (float)mem.size();
      }
      null2[CODE_STAR] = 1.0f;
      while (pos <= d.sqfrom) { n2sc[ireg + pos - 1] += 1.0f; pos++; }
      while (pos <= d.sqto) { n2sc[ireg + pos - 1] += null2[dsq[ireg + pos - 2]]; pos++; }
    }
    while (pos <= lr) { n2sc[ireg + pos - 1] += 1.0f; pos++; }
  }
  for (size_t v = ireg; v <= jreg; v++) n2sc[v] = std::log(n2sc[v] / (float)NSAMPLES);

  std::vector<size_t> assign;
  size_t nc = single_linkage(sp, assign);
  struct Sig { size_t i, j; float prob; };
  std::vector<Sig> sigc;
  for (size_t c = 0; c < nc; c++) {
    size_t ninc = 0;
    bool have_last = false;
    size_t last = 0;
    for (size_t h = 0; h < sp.size(); h++) {
      if (assign[h] == c) {
        if (!have_last || last != sp[h].idx) ninc++;
        have_last = true;
        last = sp[h].idx;
      }
    }
    if ((float)ninc / (float)NSAMPLES < 0.25f) continue;
    std::vector<size_t> vi, vj, vk, vm;
    for (size_t h = 0; h < sp.size(); h++)
      if (assign[h] == c) { vi.push_back(sp[h].i); vj.push_back(sp[h].j); vk.push_back(sp[h].k); vm.push_back(sp[h].m); }
    auto mm = [](const std::vector<size_t>& v) {
      size_t lo = SIZE_MAX, hi = 0;
      for (size_t x : v) { lo = std::min(lo, x); hi = std::max(hi, x); }
      return std::make_pair(lo, hi);
    };
    auto [imin, imax] = mm(vi);
    auto [jmin, jmax] = mm(vj);
    auto [kmin, kmax] = mm(vk);
    auto [mmin, mmax] = mm(vm);
    size_t thr = (size_t)std::ceil((float)ninc * 0.02f);
    size_t best_i = leftmost(vi, imin, imax, thr);
    size_t best_k = leftmost(vk, kmin, kmax, thr);
    size_t best_j = rightmost(vj, jmin, jmax, thr);
    size_t best_m = rightmost(vm, mmin, mmax, thr);
    if (best_i > best_j || best_k > best_m) continue;
    sigc.push_back({best_i, best_j, (float)ninc / (float)NSAMPLES});
  }
  std::stable_sort(sigc.begin(), sigc.end(), [](const Sig& a, const Sig& b) { return a.i < b.i; });
  std::vector<char> dominated(sigc.size(), 0);
  for (size_t d = 0; d < sigc.size(); d++) {
    for (size_t d2 = d + 1; d2 < sigc.size(); d2++) {
      int64_t nov = (int64_t)std::min(sigc[d].j, sigc[d2].j) - (int64_t)std::max(sigc[d].i, sigc[d2].i) + 1;
      if (nov == 0) break;
      float n = (float)std::min(sigc[d].j - sigc[d].i + 1, sigc[d2].j - sigc[d2].i + 1);
      if ((float)nov / n >= 0.8f) {
        if (sigc[d].prob > sigc[d2].prob) dominated[d2] = 1;
        else dominated[d] = 1;
      }
    }
  }
  std::vector<std::pair<size_t, size_t>> out;
  for (size_t d = 0; d < sigc.size(); d++) if (!dominated[d]) out.push_back({sigc[d].i, sigc[d].j});
  return out;
}

struct Envelope { size_t ie, je; float envsc, domcorr; size_t ia, ja, ka, ma; };

// pipeline.rs:545-591
std::optional<Envelope> rescore(const Profile& p, const uint8_t* dsq, size_t i, size_t j, size_t l,
                                const PipelineConfig& cfg, Workspace& ws, std::vector<float>& n2sc, bool null2_done) {
  if (i == 0 || j < i || j > l) return std::nullopt;
  const uint8_t* sub = dsq + (i - 1);
  size_t lsub = j - i + 1;
  Xsc xs = Xsc::make(l, false);
  float envsc = forward_matrix(p, sub, lsub, xs, ws.fx);
  if (!std::isfinite(envsc)) return std::nullopt;
  float bsc = backward_matrix(p, sub, lsub, xs, ws.bx);
  if (!std::isfinite(bsc)) return std::nullopt;
  decode(p, xs, ws.fx, ws.bx, ws.pp);
  float domcorr = 0.0f;
  if (cfg.null2) {
    if (!null2_done) {
      auto n2 = null2_from_posterior(p, ws.pp);
      for (size_t pos = i; pos <= j; pos++) {
        float v = n2[dsq[pos - 1]];
        n2sc[pos] = std::isfinite(v) ? v : 0.0f;
      }
    }
    for (size_t pos = i; pos <= j; pos++) domcorr += n2sc[pos];
  }
  Envelope e{i, j, envsc, domcorr, 0, 0, 0, 0};
  auto oa = optimal_accuracy_coords(p, xs, ws.pp);
  if (oa) {
    e.ia = i - 1 + oa->iali; e.ja = i - 1 + oa->jali; e.ka = oa->kali; e.ma = oa->mali;
  } else {
    auto tr = viterbi_trace(p, sub, lsub, xs);
    if (!tr.empty()) { e.ia = i - 1 + tr[0].iali; e.ja = i - 1 + tr[0].jali; e.ka = tr[0].kali; e.ma = tr[0].mali; }
    else { e.ia = i; e.ja = j; e.ka = 1; e.ma = p.m; }
  }
  return e;
}
}  // namespace

// pipeline.rs:154-294
std::optional<RawHit> score_target(const Profile& p, const uint8_t* dsq, size_t l, const PipelineConfig& cfg,
                                   Workspace& ws, StageTrace* tr) {
  if (l == 0 || p.m == 0) return std::nullopt;
  float nullsc = null_score(l);
  Xsc xs = Xsc::make(l, true);
  bool calibrated = p.stats.is_calibrated();
  if (tr) tr->nullsc = nullsc;
  float fwdsc;
  if (cfg.filters && calibrated) {
    auto [mmu, mlam] = *p.stats.msv;
    float usc = msv(p, dsq, l, ws.buf);
    if (tr) { tr->usc = usc; tr->stage_reached = 1; }
    if (gumbel_surv((double)((usc - nullsc) / LN2F), mmu, mlam) > cfg.f1) return std::nullopt;
    if (tr) tr->pass_f1 = true;
    float filtersc = bias_filter_score(p, dsq, l);
    if (tr) { tr->filtersc = filtersc; tr->stage_reached = 2; }
    if (gumbel_surv((double)((usc - filtersc) / LN2F), mmu, mlam) > cfg.f1) return std::nullopt;
    if (tr) tr->pass_bias = true;
    auto [vmu, vlam] = *p.stats.viterbi;
    float vsc = viterbi_score(p, dsq, l, xs, ws.buf);
    if (tr) { tr->vsc = vsc; tr->stage_reached = 3; }
    if (gumbel_surv((double)((vsc - filtersc) / LN2F), vmu, vlam) > cfg.f2) return std::nullopt;
    if (tr) tr->pass_f2 = true;
    auto [ftau, flam] = *p.stats.forward;
    fwdsc = forward(p, dsq, l, xs, ws.buf, &ws.fsp);
    if (tr) { tr->fwdsc = fwdsc; tr->stage_reached = 4; }
    if (std::exp(exp_logsurv((double)((fwdsc - filtersc) / LN2F), ftau, flam)) > cfg.f3) return std::nullopt;
    if (tr) tr->pass_f3 = true;
  } else {
    fwdsc = forward(p, dsq, l, xs, ws.buf, &ws.fsp);
    if (tr) { tr->fwdsc = fwdsc; tr->stage_reached = 4; }
  }
  if (!std::isfinite(fwdsc)) return std::nullopt;
  float bcksc = backward(p, dsq, l, xs, ws.buf, ws.bsp);
  if (tr) { tr->bcksc = bcksc; tr->stage_reached = 5; }
  float overall = std::isfinite(bcksc) ? bcksc : fwdsc;

  const Specials& f = ws.fsp;
  const Specials& b = ws.bsp;
  std::vector<float> btot(l + 1, 0.0f), etot(l + 1, 0.0f), mocc(l + 1, 0.0f);
  for (size_t i = 1; i <= l; i++) {
    btot[i] = btot[i - 1] + std::exp(f.b[i - 1] + b.b[i - 1] - overall);
    etot[i] = etot[i - 1] + std::exp(f.e[i] + b.e[i] - overall);
    float njc = std::exp(f.n[i - 1] + b.n[i] + xs.n_loop - overall) + std::exp(f.j[i - 1] + b.j[i] + xs.j_loop - overall) +
                std::exp(f.c[i - 1] + b.c[i] + xs.c_loop - overall);
    mocc[i] = 1.0f - njc;
  }
  float nexpected = btot[l];

  const float rt1 = 0.25f, rt2 = 0.10f, rt3 = 0.20f;
  std::vector<float> n2sc(l + 1, 0.0f);
  std::vector<Envelope> envs;
  size_t nregions = 0;
  int64_t i = -1;
  bool triggered = false;
  for (size_t j = 1; j <= l; j++) {
    if (!triggered) {
      if (mocc[j] - (btot[j] - btot[j - 1]) < rt2 || i == -1) i = (int64_t)j;
      if (mocc[j] >= rt1) triggered = true;
    } else if (mocc[j] - (etot[j] - etot[j - 1]) < rt2) {
      size_t ri = (size_t)std::max<int64_t>(i, 1);
      nregions++;
      if (is_multidomain(btot, etot, ri, j, rt3)) {
        auto envs_r = region_trace_ensemble(p, dsq, ri, j, l, ws, n2sc);
        for (auto [ei, ej] : envs_r) {
          auto d = rescore(p, dsq, ei, ej, l, cfg, ws, n2sc, true);
          if (d) envs.push_back(*d);
        }
      } else {
        auto d = rescore(p, dsq, ri, j, l, cfg, ws, n2sc, false);
        if (d) envs.push_back(*d);
      }
      i = -1;
      triggered = false;
    }
  }
  if (nregions == 0 || envs.empty()) return std::nullopt;

  const float omega_ln = std::log(1.0f / 256.0f);
  float seqbias = 0.0f;
  if (cfg.null2) {
    float s = 0.0f;
    for (size_t q = 1; q <= l; q++) s += n2sc[q];
    seqbias = logsum(0.0f, omega_ln + s);
  }
  float pre_score = (fwdsc - nullsc) / LN2F;
  float seq_score = (fwdsc - (nullsc + seqbias)) / LN2F;
  const float ln_multi_loop = std::log((float)l / ((float)l + 3.0f));
  float sum = 0.0f, sum_bias = 0.0f;
  size_t ld_tot = 0;
  for (const auto& e : envs) {
    bool keep = cfg.null2 ? (e.envsc - e.domcorr > 0.0f) : (e.envsc > 0.0f);
    if (keep) { sum += e.envsc; ld_tot += e.je - e.ie + 1; sum_bias += e.domcorr; }
  }
  float sum_seqbias = cfg.null2 ? logsum(0.0f, omega_ln + sum_bias) : 0.0f;
  sum += (float)(l - std::min(ld_tot, l)) * ln_multi_loop;
  float pre2 = (sum - nullsc) / LN2F;
  float sum_score = (sum - (nullsc + sum_seqbias)) / LN2F;
  if (ld_tot > 0 && sum_score > seq_score) { seq_score = sum_score; pre_score = pre2; }

  double ftau = NAN, flam = NAN;
  if (p.stats.forward) { ftau = p.stats.forward->first; flam = p.stats.forward->second; }
  double lnp = (calibrated || p.stats.forward) ? exp_logsurv((double)seq_score, ftau, flam) : NAN;

  RawHit h;
  h.bits = seq_score;
  h.bias = pre_score - seq_score;
  h.lnp = lnp;
  h.nexpected = nexpected;
  h.nregions = nregions;
  for (const auto& e : envs) {
    size_t ld = e.je - e.ie + 1;
    float dombias = cfg.null2 ? logsum(0.0f, omega_ln + e.domcorr) : 0.0f;
    float bits = (e.envsc + (float)(l - ld) * ln_multi_loop - (nullsc + dombias)) / LN2F;
    double dlnp = p.stats.forward ? exp_logsurv((double)bits, ftau, flam) : NAN;
    h.domains.push_back({e.ie, e.je, e.ia, e.ja, e.ka, e.ma, bits, dombias / LN2F, dlnp});
  }
  return h;
}

// ---------------------------------------------------------------- search
namespace {
struct Threshold { bool is_e; double e_seq, e_dom; float t_seq, t_dom; };

// search.rs:131-148
bool thresholds(const Profile& p, const Cutoff& c, Threshold& th, std::string& err) {
  th = Threshold{false, 0, 0, 0, 0};
  auto use = [&](const std::optional<std::pair<float, float>>& v, const char* nm) {
    if (!v) { err = std::string(nm) + " bit thresholds unavailable on model " + p.name; return false; }
    th.t_seq = v->first; th.t_dom = v->second;
    return true;
  };
  switch (c.kind) {
    case CutoffKind::Evalue: th.is_e = true; th.e_seq = c.seq; th.e_dom = c.dom; return true;
    case CutoffKind::Bits: th.t_seq = (float)c.seq; th.t_dom = (float)c.dom; return true;
    case CutoffKind::Gathering: return use(p.ga, "GA");
    case CutoffKind::Noise: return use(p.nc, "NC");
    case CutoffKind::Trusted: return use(p.tc, "TC");
  }
  return true;
}

// search.rs:157-210
void report(const Profile& p, std::vector<std::pair<size_t, RawHit>>& raws, const Targets& targets, const Threshold& th,
            double z, std::vector<Hit>& out) {
  std::vector<Hit> hits;
  for (auto& [ti, r] : raws) {
    double evalue = std::exp(r.lnp) * z;
    bool keep = th.is_e ? (evalue <= th.e_seq) : (r.bits >= th.t_seq);
    if (!keep) continue;
    Hit h;
    h.profile = p.name; h.acc = p.acc; h.qlen = p.m;
    h.target = targets.ids[ti]; h.target_index = ti; h.tlen = targets.dsq[ti].size();
    h.score = r.bits; h.bias = r.bias; h.evalue = evalue; h.nexpected = r.nexpected;
    for (const auto& d : r.domains) {
      h.domains.push_back({d.bits, d.bias, NAN, std::exp(d.lnp) * z, d.kali, d.mali, d.iali, d.jali, d.ienv, d.jenv, false});
    }
    hits.push_back(std::move(h));
  }
  double dom_z = (double)std::max<size_t>(hits.size(), 1);
  for (auto& h : hits) {
    for (auto& d : h.domains) {
      double p_dom = d.i_evalue / z;
      d.c_evalue = p_dom * dom_z;
      d.reported = th.is_e ? (d.c_evalue <= th.e_dom) : (d.score >= th.t_dom);
    }
  }
  for (auto& h : hits) out.push_back(std::move(h));
}
}  // namespace

// search.rs:213-234
bool search_profiles(const std::vector<Profile>& profiles, const Targets& targets, const SearchConfig& cfg,
                     int nthreads, std::vector<Hit>& out, std::string& err) {
  double z = std::max(cfg.z ? *cfg.z : (double)targets.ids.size(), 1.0);
  std::vector<Threshold> ths(profiles.size());
  for (size_t i = 0; i < profiles.size(); i++)
    if (!thresholds(profiles[i], cfg.cutoff, ths[i], err)) return false;
  const size_t nt = targets.ids.size();
  const size_t npairs = profiles.size() * nt;
  std::vector<std::optional<RawHit>> res(npairs);
  std::atomic<size_t> next{0};
  auto worker = [&]() {
    Workspace ws;
    for (;;) {
      size_t idx = next.fetch_add(1);
      if (idx >= npairs) break;
      size_t pi = idx / nt, ti = idx % nt;
      const auto& d = targets.dsq[ti];
      res[idx] = score_target(profiles[pi], d.data(), d.size(), cfg.pipeline, ws);
    }
  };
  int nth = std::max(1, nthreads);
  std::vector<std::thread> th;
  for (int t = 1; t < nth; t++) th.emplace_back(worker);
  worker();
  for (auto& t : th) t.join();
  out.clear();
  for (size_t pi = 0; pi < profiles.size(); pi++) {
    std::vector<std::pair<size_t, RawHit>> raws;
    for (size_t ti = 0; ti < nt; ti++)
      if (res[pi * nt + ti]) raws.push_back({ti, std::move(*res[pi * nt + ti])});
    report(profiles[pi], raws, targets, ths[pi], z, out);
  }
  return true;
}

}  // namespace sxo
