// HMMER3 profile ingest for the sxhmm engine: text (or gzip) -> configured
// ProfileHost records.
//
// Semantics follow the reference parser and profile configuration
// (src/hmmer/parse.rs:107-298, src/hmmer/model.rs:146-260): the same accepted
// header tags, the same -ln(p) decoding (f64 exp, then f32), the same
// f64-vs-f32 logarithms in the configured scores, and error texts of the same
// shape ("<source> line N: ...").  The implementation is a single pass over a
// memory buffer with a line cursor.
#include <zlib.h>

#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "internal.hpp"

namespace sx {

const float kBackground[NRES] = {0.0787945f, 0.0151600f, 0.0535222f, 0.0668298f, 0.0397062f, 0.0695071f,
                                 0.0229198f, 0.0590092f, 0.0594422f, 0.0963728f, 0.0237718f, 0.0414386f,
                                 0.0482904f, 0.0395639f, 0.0540978f, 0.0683364f, 0.0540687f, 0.0673417f,
                                 0.0114135f, 0.0304133f};

const Degenerate& degenerate(int code) {
  static const Degenerate tab[4] = {
      {2, {2, 11}},                                                                     // B: D N
      {2, {7, 9}},                                                                      // J: I L
      {2, {3, 13}},                                                                     // Z: E Q
      {20, {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19}},  // X: all
  };
  return tab[code - 20];
}

static std::array<uint8_t, 256> make_digitize() {
  std::array<uint8_t, 256> t{};
  for (int c = 0; c < 256; c++) t[c] = SYM_STAR;
  const char* aa = "ACDEFGHIKLMNPQRSTVWY";
  for (int c = 'A'; c <= 'Z'; c++) t[c] = 23;  // unknown letters score as X
  for (int i = 0; i < 20; i++) t[(uint8_t)aa[i]] = (uint8_t)i;
  t['U'] = 1;   // selenocysteine scores as C
  t['O'] = 8;   // pyrrolysine scores as K
  t['B'] = 20; t['J'] = 21; t['Z'] = 22; t['X'] = 23;
  for (int c = 'a'; c <= 'z'; c++) t[c] = t[c - 32];
  return t;
}
static const std::array<uint8_t, 256> kDig = make_digitize();
const uint8_t kDigitize[256] = {
#define R(i) kDig[i]
#define R8(i) R(i), R(i + 1), R(i + 2), R(i + 3), R(i + 4), R(i + 5), R(i + 6), R(i + 7)
#define R64(i) R8(i), R8(i + 8), R8(i + 16), R8(i + 24), R8(i + 32), R8(i + 40), R8(i + 48), R8(i + 56)
    R64(0), R64(64), R64(128), R64(192)
#undef R64
#undef R8
#undef R
};

namespace {

inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f' || c == '\v'; }

// A view of one line split into whitespace-separated tokens.
struct Tokens {
  std::vector<std::pair<const char*, size_t>> v;
  void split(const char* b, const char* e) {
    v.clear();
    while (b < e) {
      while (b < e && is_ws(*b)) b++;
      const char* s = b;
      while (b < e && !is_ws(*b)) b++;
      if (b > s) v.emplace_back(s, (size_t)(b - s));
    }
  }
  std::string str(size_t i) const { return std::string(v[i].first, v[i].second); }
  size_t size() const { return v.size(); }
};

class Cursor {
 public:
  Cursor(const char* text, size_t len, std::string source) : p_(text), end_(text + len), src_(std::move(source)) {}
  // Next line without its trailing "\n"/"\r" characters; false at end of input.
  bool next(const char** b, const char** e) {
    if (p_ >= end_) return false;
    const char* nl = static_cast<const char*>(memchr(p_, '\n', (size_t)(end_ - p_)));
    const char* le = nl ? nl : end_;
    *b = p_;
    *e = le;
    while (*e > *b && ((*e)[-1] == '\r' || (*e)[-1] == '\n')) (*e)--;
    p_ = nl ? nl + 1 : end_;
    line_++;
    return true;
  }
  std::string at(const std::string& msg) const { return src_ + " line " + std::to_string(line_) + ": " + msg; }
  std::string eof(const char* what) const { return src_ + ": unexpected end of file (" + what + ")"; }

 private:
  const char* p_;
  const char* end_;
  std::string src_;
  size_t line_ = 0;
};

bool blank(const char* b, const char* e) {
  for (; b < e; b++)
    if (!is_ws(*b)) return false;
  return true;
}
bool starts(const char* b, const char* e, const char* pre) {
  size_t n = strlen(pre);
  return (size_t)(e - b) >= n && memcmp(b, pre, n) == 0;
}

bool to_double(const std::pair<const char*, size_t>& t, double& v) {
  char buf[64];
  if (t.second == 0 || t.second >= sizeof buf) return false;
  memcpy(buf, t.first, t.second);
  buf[t.second] = 0;
  char* endp;
  v = strtod(buf, &endp);
  return endp == buf + t.second;
}
bool to_float(const std::string& s, float& v) {
  if (s.empty()) return false;
  char* endp;
  v = strtof(s.c_str(), &endp);
  return endp == s.c_str() + s.size();
}
bool to_size(const std::string& s, size_t& v) {
  size_t i = (!s.empty() && s[0] == '+') ? 1 : 0;
  if (i >= s.size()) return false;
  size_t acc = 0;
  for (; i < s.size(); i++) {
    if (s[i] < '0' || s[i] > '9') return false;
    acc = acc * 10 + (size_t)(s[i] - '0');
  }
  v = acc;
  return true;
}

// "-ln p" token -> p as f32 via f64 exp; "*" is p = 0 (parse.rs:268-277).
bool neglog_prob(const std::pair<const char*, size_t>& t, float& out, std::string& why) {
  if (t.second == 1 && t.first[0] == '*') {
    out = 0.0f;
    return true;
  }
  double v;
  std::string tok(t.first, t.second);
  if (!to_double(t, v)) {
    why = "non-numeric probability token \"" + tok + "\"";
    return false;
  }
  if (!std::isfinite(v) || v < 0.0) {
    why = "invalid -ln(p) value \"" + tok + "\"";
    return false;
  }
  out = (float)std::exp(-v);
  return true;
}

bool probs(const Tokens& tk, size_t first, size_t n, float* out, std::string& why) {
  if (tk.size() < first + n) {
    why = "expected " + std::to_string(n) + (n == 7 ? " transition values" : " values") + ", found " +
          std::to_string(tk.size() > first ? tk.size() - first : 0);
    return false;
  }
  for (size_t i = 0; i < n; i++)
    if (!neglog_prob(tk.v[first + i], out[i], why)) return false;
  return true;
}

// GA/TC/NC value pair; Pfam appends ';' (parse.rs:260-266).
bool cutoff_values(const std::string& rest, float out[2]) {
  std::string s = rest;
  for (char& c : s)
    if (c == ';') c = ' ';
  Tokens tk;
  tk.split(s.data(), s.data() + s.size());
  if (tk.size() == 0 || !to_float(tk.str(0), out[0])) return false;
  out[1] = out[0];
  float b;
  if (tk.size() > 1 && to_float(tk.str(1), b)) out[1] = b;
  return true;
}

struct RawModel {
  size_t m = 0;
  std::vector<std::array<float, NRES>> mat;
  std::vector<std::array<float, 7>> tr;
  bool has_compo = false;
  std::array<float, NRES> compo{};
};

// One record; returns 1 ok, 0 end of input, -1 error.
int read_record(Cursor& cur, ProfileHost& ph, RawModel& rm, std::string& err) {
  const char *b, *e;
  for (;;) {
    if (!cur.next(&b, &e)) return 0;
    if (!blank(b, e)) break;
  }
  if (!starts(b, e, "HMMER3")) {
    if (starts(b, e, "HMMER2")) {
      err = cur.at("HMMER2 format is not supported; convert with `hmmconvert`");
      return -1;
    }
    err = cur.at("expected 'HMMER3/x' header, found \"" + std::string(b, e) + "\"");
    return -1;
  }
  ph = ProfileHost();
  rm = RawModel();
  bool alph = false;
  Tokens tk;
  for (;;) {
    if (!cur.next(&b, &e)) {
      err = cur.eof("header");
      return -1;
    }
    const char* s = b;
    while (s < e && is_ws(*s)) s++;
    if ((e - s == 3 && memcmp(s, "HMM", 3) == 0) || starts(s, e, "HMM ") || starts(s, e, "HMM\t")) break;
    const char* te = s;
    while (te < e && !is_ws(*te)) te++;
    std::string tag(s, te);
    const char* rb = te < e ? te + 1 : te;
    while (rb < e && is_ws(*rb)) rb++;
    const char* re = e;
    while (re > rb && is_ws(re[-1])) re--;
    std::string rest(rb, re);
    if (tag == "NAME") {
      ph.name = rest;
    } else if (tag == "ACC") {
      ph.acc = rest;
      ph.has_acc = true;
    } else if (tag == "DESC") {
      ph.desc = rest;
      ph.has_desc = true;
    } else if (tag == "LENG") {
      size_t m;
      if (!to_size(rest, m)) {
        err = cur.at("bad LENG value \"" + rest + "\"");
        return -1;
      }
      rm.m = m;
    } else if (tag == "ALPH") {
      std::string lo = rest;
      for (char& c : lo) c = (char)tolower((unsigned char)c);
      if (lo != "amino") {
        err = cur.at("profile '" + ph.name + "' has alphabet '" + rest +
                     "'; only protein (amino) profiles are supported");
        return -1;
      }
      alph = true;
    } else if (tag == "GA" || tag == "TC" || tag == "NC") {
      float v[2];
      if (!cutoff_values(rest, v)) {
        err = cur.at("bad " + tag + " line");
        return -1;
      }
      float* dst = tag == "GA" ? ph.ga : tag == "TC" ? ph.tc : ph.nc;
      (tag == "GA" ? ph.has_ga : tag == "TC" ? ph.has_tc : ph.has_nc) = true;
      dst[0] = v[0];
      dst[1] = v[1];
    } else if (tag == "STATS") {
      tk.split(rest.data(), rest.data() + rest.size());
      if (tk.size() >= 4) {
        double a, c;
        if (!to_double(tk.v[2], a) || !to_double(tk.v[3], c)) {
          err = cur.at("bad STATS value");
          return -1;
        }
        std::string which = tk.str(1);
        if (which == "MSV") { ph.msv[0] = a; ph.msv[1] = c; ph.has_msv = true; }
        else if (which == "VITERBI") { ph.vit[0] = a; ph.vit[1] = c; ph.has_vit = true; }
        else if (which == "FORWARD") { ph.fwd[0] = a; ph.fwd[1] = c; ph.has_fwd = true; }
      }
    }
  }
  if (rm.m == 0) {
    err = cur.at("profile '" + ph.name + "' has no LENG");
    return -1;
  }
  if (!alph) {
    err = cur.at("profile '" + ph.name + "' has no ALPH line");
    return -1;
  }
  if (!cur.next(&b, &e)) {  // transition-order line
    err = cur.eof("transition header");
    return -1;
  }
  const size_t m = rm.m;
  rm.mat.assign(m + 1, std::array<float, NRES>{});
  rm.tr.assign(m + 1, std::array<float, 7>{});
  std::string why;
  if (!cur.next(&b, &e)) {
    err = cur.eof("model body");
    return -1;
  }
  {
    const char* s = b;
    while (s < e && is_ws(*s)) s++;
    if (starts(s, e, "COMPO")) {
      tk.split(b, e);
      if (!probs(tk, 1, NRES, rm.compo.data(), why)) {
        err = cur.at("COMPO: " + why);
        return -1;
      }
      rm.has_compo = true;
      if (!cur.next(&b, &e)) {
        err = cur.eof("node-0 insert line");
        return -1;
      }
    }
  }
  tk.split(b, e);
  if (tk.size() < (size_t)NRES) {
    err = cur.at("truncated node-0 insert line");
    return -1;
  }
  if (!cur.next(&b, &e)) {
    err = cur.eof("node-0 transitions");
    return -1;
  }
  tk.split(b, e);
  if (!probs(tk, 0, 7, rm.tr[0].data(), why)) {
    err = cur.at("node 0 transitions: " + why);
    return -1;
  }
  for (size_t k = 1; k <= m; k++) {
    if (!cur.next(&b, &e)) {
      err = cur.eof("match line");
      return -1;
    }
    tk.split(b, e);
    size_t idx;
    if (tk.size() == 0 || !to_size(tk.str(0), idx)) {
      err = cur.at("bad match-line node index");
      return -1;
    }
    if (idx != k) {
      err = cur.at("node index " + std::to_string(idx) + ", expected " + std::to_string(k));
      return -1;
    }
    if (tk.size() < 1 + (size_t)NRES) {
      err = cur.at("truncated match emissions at node " + std::to_string(k));
      return -1;
    }
    if (!probs(tk, 1, NRES, rm.mat[k].data(), why)) {
      err = cur.at("node " + std::to_string(k) + ": " + why);
      return -1;
    }
    if (!cur.next(&b, &e)) {
      err = cur.eof("insert line");
      return -1;
    }
    tk.split(b, e);
    if (tk.size() < (size_t)NRES) {
      err = cur.at("truncated insert emissions at node " + std::to_string(k));
      return -1;
    }
    if (!cur.next(&b, &e)) {
      err = cur.eof("transition line");
      return -1;
    }
    tk.split(b, e);
    if (!probs(tk, 0, 7, rm.tr[k].data(), why)) {
      err = cur.at("node " + std::to_string(k) + " transitions: " + why);
      return -1;
    }
  }
  while (cur.next(&b, &e)) {
    if (blank(b, e)) continue;
    const char* s = b;
    while (s < e && is_ws(*s)) s++;
    const char* t = e;
    while (t > s && is_ws(t[-1])) t--;
    if (t - s == 2 && s[0] == '/' && s[1] == '/') break;
    err = cur.at("expected '//', found \"" + std::string(b, e) + "\"");
    return -1;
  }
  return 1;
}

inline float ln_or_neginf(float p) { return p > 0.0f ? (float)std::log((double)p) : kNegInf; }

// p7_ProfileConfig in local multihit mode (src/hmmer/model.rs:146-245).
void configure_profile(const RawModel& rm, ProfileHost& ph) {
  const int m = (int)rm.m;
  const size_t w = (size_t)m + 1;
  ph.m = m;
  ph.msc.assign((size_t)NSYM * w, kNegInf);
  for (int k = 1; k <= m; k++) {
    float sc[NSYM];
    for (int x = 0; x < NRES; x++) {
      double pr = (double)rm.mat[k][x];
      sc[x] = pr > 0.0 ? (float)std::log(pr / (double)kBackground[x]) : kNegInf;
    }
    for (int code = 20; code <= 23; code++) {  // background-weighted expected score
      const Degenerate& d = degenerate(code);
      float num = 0.0f, den = 0.0f;
      for (int q = 0; q < d.n; q++) {
        num += sc[d.members[q]] * kBackground[d.members[q]];
        den += kBackground[d.members[q]];
      }
      sc[code] = den > 0.0f ? num / den : 0.0f;
    }
    sc[SYM_STAR] = kNegInf;
    for (int x = 0; x < NSYM; x++) ph.msc[(size_t)x * w + k] = sc[x];
  }
  for (int q = 0; q < NTR; q++) ph.t[q].assign(w, kNegInf);
  for (int k = 1; k < m; k++)
    for (int q = 0; q < 7; q++) ph.t[q][k] = ln_or_neginf(rm.tr[k][q]);
  if (m >= 1) ph.t[TDM][1] = ph.t[TDD][1] = kNegInf;  // no D_1 in local mode
  // match occupancy (p7_hmm_CalculateOccupancy) and occupancy-weighted entry
  std::vector<float> occ(w, 0.0f);
  if (m >= 1) {
    occ[1] = rm.tr[0][1] + rm.tr[0][0];
    for (int k = 2; k <= m; k++) {
      const auto& t = rm.tr[k - 1];
      occ[k] = occ[k - 1] * (t[0] + t[1]) + (1.0f - occ[k - 1]) * t[5];
    }
  }
  float z = 0.0f;
  for (int k = 1; k <= m; k++) z += occ[k] * (float)(m - k + 1);
  for (int k = 1; k <= m; k++)
    ph.t[TBM][k] = (z > 0.0f && occ[k] > 0.0f) ? (float)std::log((double)(occ[k] / z)) : kNegInf;
  const float mf = (float)m;
  ph.msv_tbm = std::log(2.0f / (mf * (mf + 1.0f)));
  ph.mo.resize(ph.msc.size());
  for (size_t i = 0; i < ph.msc.size(); i++) ph.mo[i] = std::exp(ph.msc[i]);
  for (int q = 0; q < NTR; q++) {
    ph.p[q].resize(w);
    for (size_t k = 0; k < w; k++) ph.p[q][k] = std::exp(ph.t[q][k]);
  }
  for (int x = 0; x < NRES; x++) ph.compo[x] = rm.has_compo ? rm.compo[x] : kBackground[x];
}

}  // namespace

bool load_profiles_text(const char* text, size_t len, const std::string& source, std::vector<ProfileHost>& out,
                        std::string& err) {
  Cursor cur(text, len, source);
  out.clear();
  RawModel rm;
  for (;;) {
    ProfileHost ph;
    int rc = read_record(cur, ph, rm, err);
    if (rc == 0) return true;
    if (rc < 0) return false;
    configure_profile(rm, ph);
    out.push_back(std::move(ph));
  }
}

bool load_profiles_file(const std::string& path, std::vector<ProfileHost>& out, std::string& err, bool& io_error) {
  io_error = false;
  gzFile f = gzopen(path.c_str(), "rb");  // reads gzip (by magic) or plain text
  if (!f) {
    io_error = true;
    err = "opening HMM file " + path + ": " + strerror(errno);
    return false;
  }
  gzbuffer(f, 1 << 20);
  std::string text;
  std::vector<char> buf(1 << 20);
  int n;
  while ((n = gzread(f, buf.data(), (unsigned)buf.size())) > 0) text.append(buf.data(), (size_t)n);
  int zerr = 0;
  const char* zmsg = gzerror(f, &zerr);
  gzclose(f);
  if (n < 0 || (zerr != Z_OK && zerr != Z_BUF_ERROR)) {
    io_error = true;
    err = "reading " + path + ": " + (zmsg ? zmsg : "read error");
    return false;
  }
  return load_profiles_text(text.data(), text.size(), path, out, err);
}

SpecialTr special_transitions(int64_t l, bool multihit) {
  SpecialTr s;
  const float nj = multihit ? 1.0f : 0.0f;
  s.pmove = (2.0f + nj) / ((float)l + 2.0f + nj);
  s.ploop = 1.0f - s.pmove;
  s.loop = (float)std::log((double)s.ploop);
  s.move = (float)std::log((double)s.pmove);
  if (multihit) {
    s.e_move = s.e_loop = -kLn2f;
    s.pe_move = s.pe_loop = 0.5f;
  } else {
    s.e_move = 0.0f;
    s.e_loop = kNegInf;
    s.pe_move = 1.0f;
    s.pe_loop = 0.0f;
  }
  return s;
}

float null1_score(int64_t l) {
  const float p1 = (float)l / ((float)l + 1.0f);
  return (float)((double)l * std::log((double)p1) + std::log(1.0 - (double)p1));
}

double gumbel_survival(double x, double mu, double lambda) {
  const double y = lambda * (x - mu);
  const double ey = -std::exp(-y);
  return std::fabs(ey) < 1e-5 ? -ey : 1.0 - std::exp(ey);
}

double exp_tail_logsurv(double x, double tau, double lambda) { return x < tau ? 0.0 : -lambda * (x - tau); }

// ---- binary cache of configured profiles ---------------------------------------
// Layout (little-endian): "SXPROF01", u32 version = 1, u32 count, then per
// profile: string name, u8 has_acc, string acc, u8 has_desc, string desc,
// i32 M, u8 flags (GA TC NC MSV VIT FWD), f32 ga[2] tc[2] nc[2],
// f64 msv[2] vit[2] fwd[2], f32 msv_tbm, f32 compo[20], f32 msc[25(M+1)],
// mo[25(M+1)], t[8(M+1)], p[8(M+1)]; finally u64 FNV-1a of everything after
// the magic.  Strings are u32 length + bytes.
namespace {

constexpr char kBinMagic[8] = {'S', 'X', 'P', 'R', 'O', 'F', '0', '1'};
constexpr uint32_t kBinVersion = 1;

uint64_t fnv1a(const uint8_t* p, size_t n) {
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < n; i++) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

class ByteWriter {
 public:
  template <typename T>
  void put(const T& v) { raw(&v, sizeof v); }
  void raw(const void* p, size_t n) {
    const uint8_t* b = static_cast<const uint8_t*>(p);
    buf.insert(buf.end(), b, b + n);
  }
  void str(const std::string& s) {
    put<uint32_t>((uint32_t)s.size());
    raw(s.data(), s.size());
  }
  void floats(const std::vector<float>& v) { raw(v.data(), sizeof(float) * v.size()); }
  std::vector<uint8_t> buf;
};

class ByteReader {
 public:
  ByteReader(const uint8_t* p, size_t n) : p_(p), n_(n) {}
  template <typename T>
  bool get(T& v) { return raw(&v, sizeof v); }
  bool raw(void* out, size_t n) {
    if (n > n_ - o_) return false;
    std::memcpy(out, p_ + o_, n);
    o_ += n;
    return true;
  }
  bool str(std::string& s) {
    uint32_t n = 0;
    if (!get(n) || n > n_ - o_) return false;
    s.assign(reinterpret_cast<const char*>(p_ + o_), n);
    o_ += n;
    return true;
  }
  bool floats(std::vector<float>& v, size_t n) {
    if (n > (n_ - o_) / sizeof(float)) return false;
    v.resize(n);
    return raw(v.data(), sizeof(float) * n);
  }
  size_t left() const { return n_ - o_; }

 private:
  const uint8_t* p_;
  size_t n_, o_ = 0;
};

}  // namespace

bool save_profiles_binary(const std::vector<ProfileHost>& in, const std::string& path, std::string& err) {
  ByteWriter w;
  w.put<uint32_t>(kBinVersion);
  w.put<uint32_t>((uint32_t)in.size());
  for (const ProfileHost& h : in) {
    w.str(h.name);
    w.put<uint8_t>(h.has_acc);
    w.str(h.acc);
    w.put<uint8_t>(h.has_desc);
    w.str(h.desc);
    w.put<int32_t>(h.m);
    const uint8_t flags = (uint8_t)(h.has_ga | h.has_tc << 1 | h.has_nc << 2 | h.has_msv << 3 | h.has_vit << 4 |
                                    h.has_fwd << 5);
    w.put(flags);
    w.raw(h.ga, sizeof h.ga);
    w.raw(h.tc, sizeof h.tc);
    w.raw(h.nc, sizeof h.nc);
    w.raw(h.msv, sizeof h.msv);
    w.raw(h.vit, sizeof h.vit);
    w.raw(h.fwd, sizeof h.fwd);
    w.put(h.msv_tbm);
    w.raw(h.compo, sizeof h.compo);
    w.floats(h.msc);
    w.floats(h.mo);
    for (int q = 0; q < NTR; q++) w.floats(h.t[q]);
    for (int q = 0; q < NTR; q++) w.floats(h.p[q]);
  }
  const uint64_t sum = fnv1a(w.buf.data(), w.buf.size());
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = path + ": " + std::strerror(errno);
    return false;
  }
  bool ok = std::fwrite(kBinMagic, 1, sizeof kBinMagic, f) == sizeof kBinMagic;
  ok = ok && std::fwrite(w.buf.data(), 1, w.buf.size(), f) == w.buf.size();
  ok = ok && std::fwrite(&sum, 1, sizeof sum, f) == sizeof sum;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) err = path + ": write failed";
  return ok;
}

bool load_profiles_binary(const std::string& path, std::vector<ProfileHost>& out, std::string& err, bool& io_error) {
  io_error = false;
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) {
    io_error = true;
    err = path + ": " + std::strerror(errno);
    return false;
  }
  std::vector<uint8_t> all;
  std::vector<uint8_t> chunk(1 << 16);
  size_t got;
  while ((got = std::fread(chunk.data(), 1, chunk.size(), f)) > 0) all.insert(all.end(), chunk.data(), chunk.data() + got);
  const bool rerr = std::ferror(f) != 0;
  std::fclose(f);
  if (rerr) {
    io_error = true;
    err = path + ": read failed";
    return false;
  }
  if (all.size() < sizeof kBinMagic + 8 + 8 || std::memcmp(all.data(), kBinMagic, sizeof kBinMagic) != 0) {
    err = path + ": not a profile cache (bad magic)";
    return false;
  }
  const uint8_t* body = all.data() + sizeof kBinMagic;
  const size_t nbody = all.size() - sizeof kBinMagic - 8;
  uint64_t sum = 0;
  std::memcpy(&sum, body + nbody, 8);
  if (fnv1a(body, nbody) != sum) {
    err = path + ": checksum mismatch (truncated or corrupt)";
    return false;
  }
  ByteReader r(body, nbody);
  uint32_t version = 0, count = 0;
  if (!r.get(version) || version != kBinVersion) {
    err = path + ": unsupported cache version " + std::to_string(version);
    return false;
  }
  if (!r.get(count)) {
    err = path + ": truncated header";
    return false;
  }
  out.clear();
  out.resize(count);
  for (uint32_t i = 0; i < count; i++) {
    ProfileHost& h = out[i];
    uint8_t has_acc = 0, has_desc = 0, flags = 0;
    bool ok = r.str(h.name) && r.get(has_acc) && r.str(h.acc) && r.get(has_desc) && r.str(h.desc) && r.get(h.m) &&
              r.get(flags) && r.raw(h.ga, sizeof h.ga) && r.raw(h.tc, sizeof h.tc) && r.raw(h.nc, sizeof h.nc) &&
              r.raw(h.msv, sizeof h.msv) && r.raw(h.vit, sizeof h.vit) && r.raw(h.fwd, sizeof h.fwd) &&
              r.get(h.msv_tbm) && r.raw(h.compo, sizeof h.compo);
    if (ok && (h.m < 1 || h.m > (1 << 20))) ok = false;
    const size_t w = ok ? (size_t)h.m + 1 : 0;
    ok = ok && r.floats(h.msc, NSYM * w) && r.floats(h.mo, NSYM * w);
    for (int q = 0; q < NTR && ok; q++) ok = r.floats(h.t[q], w);
    for (int q = 0; q < NTR && ok; q++) ok = r.floats(h.p[q], w);
    if (!ok) {
      err = path + ": malformed record for profile " + std::to_string(i);
      out.clear();
      return false;
    }
    h.has_acc = has_acc != 0;
    h.has_desc = has_desc != 0;
    h.has_ga = flags & 1;
    h.has_tc = (flags >> 1) & 1;
    h.has_nc = (flags >> 2) & 1;
    h.has_msv = (flags >> 3) & 1;
    h.has_vit = (flags >> 4) & 1;
    h.has_fwd = (flags >> 5) & 1;
  }
  if (r.left() != 0) {
    err = path + ": trailing bytes after the last profile";
    out.clear();
    return false;
  }
  return true;
}

}  // namespace sx
