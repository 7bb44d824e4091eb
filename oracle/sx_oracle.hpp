// TEST INFRASTRUCTURE ONLY — the CPU oracle for the hmmsearch path.
//
// A line-by-line C++17 restatement of the reference Rust engine
// (src/hmmer/{alphabet,parse,model,dp,pipeline,search}.rs of raw-lab/sentinel-x),
// used only by tests/, the smoke check and bench.py's CPU-baseline leg as the
// checker.  The product library never links, imports or calls anything here.
//
// Numerics: compiled with -ffp-contract=off and without -ffast-math so every
// f32/f64 operation rounds exactly as the Rust code does (Rust never fuses
// a*b+c).  Transcendentals come from glibc (logf/expf/log1pf/log/exp), which is
// what Rust's std uses on x86_64-unknown-linux-gnu.
//
// Parity pin: tests/test_oracle_golden.py checks this oracle against the
// reference's own HMMER 3.4 fixture (src/hmmer/testdata/hmmer34_*; tolerance
// 0.1 bits and exact coordinates, src/hmmer/search.rs:316-355) and against the
// known answers of the reference's unit tests.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <limits>
#include <optional>
#include <string>
#include <utility>
#include <vector>

namespace sxo {

constexpr int K = 20;       // canonical residues (src/hmmer/alphabet.rs:20)
constexpr int NCODE = 25;   // + B J Z X * (src/hmmer/alphabet.rs:23)
constexpr uint8_t CODE_B = 20, CODE_J = 21, CODE_Z = 22, CODE_X = 23, CODE_STAR = 24;
constexpr float NEG_INF = -std::numeric_limits<float>::infinity();
constexpr float LN2F = 0.693147182464599609375f;  // std::f32::consts::LN_2

extern const float BG[K];  // src/hmmer/alphabet.rs:36-39

uint8_t encode_residue(uint8_t b);                    // alphabet.rs:58-88
std::vector<uint8_t> encode(const std::string& seq);  // alphabet.rs:91-93
std::vector<int> degenerate_members(uint8_t code);    // alphabet.rs:42-54

enum { T_MM = 0, T_MI, T_MD, T_IM, T_II, T_DM, T_DD };

struct Stats {  // src/hmmer/model.rs:26-40
  std::optional<std::pair<double, double>> msv, viterbi, forward;
  bool is_calibrated() const { return msv && viterbi && forward; }
};

struct Hmm {  // src/hmmer/model.rs:53-71
  std::string name;
  std::optional<std::string> acc, desc;
  size_t m = 0;
  std::vector<std::array<float, K>> mat;
  std::vector<std::array<float, 7>> t;
  std::optional<std::array<float, K>> compo;
  std::optional<std::pair<float, float>> ga, tc, nc;
  Stats stats;
  std::vector<float> occupancy() const;
};

struct Profile {  // src/hmmer/model.rs:74-113
  std::string name;
  std::optional<std::string> acc, desc;
  size_t m = 0;
  std::vector<float> msc;  // msc[x*(M+1)+k]
  std::vector<float> t_mm, t_mi, t_md, t_im, t_ii, t_dm, t_dd, t_bm;
  float msv_tbm = 0;
  std::vector<float> mo;
  std::vector<float> p_mm, p_mi, p_md, p_im, p_ii, p_dm, p_dd, p_bm;
  std::array<float, K> compo{};
  std::optional<std::pair<float, float>> ga, tc, nc;
  Stats stats;
  const float* msc_row(uint8_t x) const { return msc.data() + (size_t)x * (m + 1); }
  const float* mo_row(uint8_t x) const { return mo.data() + (size_t)x * (m + 1); }
};

Profile configure(const Hmm& h);  // model.rs:146-245

struct XscP { float n_loop, n_move, j_loop, j_move, c_loop, c_move, e_move, e_loop; };
struct Xsc {  // model.rs:265-312
  float n_loop, n_move, j_loop, j_move, c_loop, c_move, e_move, e_loop;
  XscP p;
  static Xsc make(size_t l, bool multihit);
};
float null_score(size_t l);  // model.rs:334-337

// ---- parser (src/hmmer/parse.rs) ----
struct ParseError { std::string msg; };
// Parses every record of an in-memory HMMER3 text.  On error returns false and
// fills err (message text mirrors parse.rs: "<source> line N: ...").
bool parse_hmm_text(const std::string& text, const std::string& source, std::vector<Hmm>& out, std::string& err);
bool parse_hmm_path(const std::string& path, std::vector<Hmm>& out, std::string& err);  // gzip-aware
std::optional<std::pair<float, float>> cutoff_pair(const std::string& rest);           // parse.rs:260-266

// ---- dp (src/hmmer/dp.rs) ----
float logsum(float a, float b);
struct DpBuf { std::vector<float> a, b, c, d, e, f; };
struct Specials {
  std::vector<float> n, b, e, j, c;
  void reset(size_t l);
};
float msv(const Profile& p, const uint8_t* dsq, size_t l, DpBuf& buf);
float viterbi_score(const Profile& p, const uint8_t* dsq, size_t l, const Xsc& xs, DpBuf& buf);
float forward(const Profile& p, const uint8_t* dsq, size_t l, const Xsc& xs, DpBuf& buf, Specials* sp);
float backward(const Profile& p, const uint8_t* dsq, size_t l, const Xsc& xs, DpBuf& buf, Specials& sp);

struct Matrix {
  size_t m = 0, l = 0;
  std::vector<float> mm, im, dm;
  std::vector<double> lnscale;
  Specials sp;
  std::vector<float> xn, xb, xe, xj, xc, scale;
  void reset(size_t m, size_t l);
};
float forward_matrix(const Profile& p, const uint8_t* dsq, size_t l, const Xsc& xs, Matrix& fx);
float backward_matrix(const Profile& p, const uint8_t* dsq, size_t l, const Xsc& xs, Matrix& bx);
std::array<float, NCODE> null2_by_expectation(const Profile& p, const uint8_t* dsq, size_t l, const Xsc& xs,
                                              const Matrix& fx, const Matrix& bx);

struct AliCoords { size_t iali, jali, kali, mali; };
std::vector<AliCoords> viterbi_trace(const Profile& p, const uint8_t* dsq, size_t l, const Xsc& xs);

struct EslRng {
  uint32_t seed, x;
  explicit EslRng(uint32_t s);
  void reseed();
  double next();
};
struct SampledDomain { size_t sqfrom = 0, sqto = 0, hmmfrom = 0, hmmto = 0; std::vector<size_t> nodes; };
std::vector<SampledDomain> stochastic_trace(const Profile& p, const Matrix& fx, const Xsc& xs, EslRng& rng);

struct Posterior {
  size_t m = 0, l = 0;
  std::vector<float> pm, pi, pn, pj, pc;
};
void decode(const Profile& p, const Xsc& xs, const Matrix& fx, const Matrix& bx, Posterior& pp);
std::array<float, NCODE> null2_from_posterior(const Profile& p, const Posterior& pp);
std::optional<AliCoords> optimal_accuracy_coords(const Profile& p, const Xsc& xs, const Posterior& pp);

// ---- pipeline (src/hmmer/pipeline.rs) ----
struct PipelineConfig { bool filters = true, null2 = true; double f1 = 0.02, f2 = 1e-3, f3 = 1e-5; };
struct RawDomain { size_t ienv, jenv, iali, jali, kali, mali; float bits, bias; double lnp; };
struct RawHit {
  float bits, bias;
  double lnp;
  std::vector<RawDomain> domains;
  float nexpected;
  size_t nregions;
};
struct Workspace { DpBuf buf; Specials fsp, bsp; Matrix fx, bx; Posterior pp; };
double gumbel_surv(double x, double mu, double lambda);
double exp_logsurv(double x, double tau, double lambda);
float bias_filter_score(const Profile& p, const uint8_t* dsq, size_t l);

// Per-stage record of one pair (filled by score_target when non-null): the
// stage scores and the decisions, so tests can compare the GPU cascade
// stage by stage.
struct StageTrace {
  float usc = NAN, filtersc = NAN, vsc = NAN, fwdsc = NAN, bcksc = NAN, nullsc = NAN;
  int stage_reached = 0;  // 1 msv, 2 bias, 3 viterbi, 4 forward, 5 domains
  bool pass_f1 = false, pass_bias = false, pass_f2 = false, pass_f3 = false;
};
std::optional<RawHit> score_target(const Profile& p, const uint8_t* dsq, size_t l, const PipelineConfig& cfg,
                                   Workspace& ws, StageTrace* tr = nullptr);

// ---- search (src/hmmer/search.rs) ----
enum class CutoffKind { Evalue = 0, Bits = 1, Gathering = 2, Noise = 3, Trusted = 4 };
struct Cutoff { CutoffKind kind = CutoffKind::Evalue; double seq = 10.0, dom = 10.0; };
struct SearchConfig { Cutoff cutoff; PipelineConfig pipeline; std::optional<double> z; };
struct Targets { std::vector<std::string> ids; std::vector<std::vector<uint8_t>> dsq; };
struct DomainHit {
  float score, bias;
  double c_evalue, i_evalue;
  size_t hmm_from, hmm_to, ali_from, ali_to, env_from, env_to;
  bool reported;
};
struct Hit {
  std::string profile;
  std::optional<std::string> acc;
  size_t qlen;
  std::string target;
  size_t target_index, tlen;
  float score, bias;
  double evalue;
  float nexpected;
  std::vector<DomainHit> domains;
};
// search_profiles (search.rs:213-234), pair loop on `nthreads` std::threads
// with one Workspace per thread and a dynamic pair index (the rayon map_init
// loop).  Returns false with err on a missing cutoff.
bool search_profiles(const std::vector<Profile>& profiles, const Targets& targets, const SearchConfig& cfg,
                     int nthreads, std::vector<Hit>& out, std::string& err);

}  // namespace sxo
