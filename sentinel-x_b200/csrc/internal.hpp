// Internal host-side types of the sxhmm engine.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <limits>
#include <memory>
#include <string>
#include <vector>

namespace sx {

constexpr int NRES = 20;   // canonical residues, HMMER order ACDEFGHIKLMNPQRSTVWY
constexpr int NSYM = 25;   // + B J Z X and the nonresidue '*'
constexpr uint8_t SYM_STAR = 24;
constexpr float kNegInf = -std::numeric_limits<float>::infinity();
constexpr float kLn2f = 0.693147182464599609375f;  // f32 rounding of ln 2

// HMMER3's amino-acid background (p7_AminoFrequencies), src/hmmer/alphabet.rs:36-39.
extern const float kBackground[NRES];
// Members of the degenerate codes B, J, Z, X (src/hmmer/alphabet.rs:42-54).
struct Degenerate {
  int n;
  int members[20];
};
const Degenerate& degenerate(int code);  // code in 20..23
// ASCII -> digital code (src/hmmer/alphabet.rs:58-88): case-insensitive, U->C,
// O->K, gap/stop characters -> '*', other letters -> X, everything else -> '*'.
extern const uint8_t kDigitize[256];

// Transition slots of a node, in HMMER file order.
enum Tr { TMM = 0, TMI, TMD, TIM, TII, TDM, TDD, TBM, NTR };

// One configured profile (HMMER p7_ProfileConfig, local multihit;
// src/hmmer/model.rs:146-245).  Vectors have M+1 entries indexed by node k.
struct ProfileHost {
  std::string name, acc, desc;
  bool has_acc = false, has_desc = false;
  int m = 0;
  bool has_ga = false, has_tc = false, has_nc = false;
  float ga[2] = {NAN, NAN}, tc[2] = {NAN, NAN}, nc[2] = {NAN, NAN};
  bool has_msv = false, has_vit = false, has_fwd = false;
  double msv[2] = {NAN, NAN}, vit[2] = {NAN, NAN}, fwd[2] = {NAN, NAN};
  bool calibrated() const { return has_msv && has_vit && has_fwd; }
  std::vector<float> msc;  // [NSYM][M+1] log-odds match scores (nats)
  std::vector<float> mo;   // [NSYM][M+1] match odds exp(msc)
  std::vector<float> t[NTR];  // log-space transitions, node k (t[TBM] = local entry B->M_k)
  std::vector<float> p[NTR];  // probability-space copies
  float msv_tbm = 0;
  float compo[NRES];
  const float* msc_row(int x) const { return msc.data() + (size_t)x * (m + 1); }
  const float* mo_row(int x) const { return mo.data() + (size_t)x * (m + 1); }
};

// Parse (plain or gzip) HMMER3 text and configure every profile.  Returns
// false with `err` set (messages follow src/hmmer/parse.rs: "<source> line N: ...").
bool load_profiles_text(const char* text, size_t len, const std::string& source, std::vector<ProfileHost>& out,
                        std::string& err);
bool load_profiles_file(const std::string& path, std::vector<ProfileHost>& out, std::string& err, bool& io_error);

// Binary cache of configured profiles (hmmfile.cpp): magic, version, count,
// the ProfileHost fields of every profile, FNV-1a checksum of the payload.
bool save_profiles_binary(const std::vector<ProfileHost>& in, const std::string& path, std::string& err);
bool load_profiles_binary(const std::string& path, std::vector<ProfileHost>& out, std::string& err, bool& io_error);

// Length-dependent special transitions (p7_ReconfigLength; src/hmmer/model.rs:284-312).
struct SpecialTr {
  float loop, move;    // N/J/C loop and move, log space
  float e_move, e_loop;
  float ploop, pmove;  // probability space
  float pe_move, pe_loop;
};
SpecialTr special_transitions(int64_t l, bool multihit);
float null1_score(int64_t l);  // src/hmmer/model.rs:334-337

// ---- host-side domain definition (the per-hit tail of score_target) ----
struct SearchOpts {
  bool filters = true, null2 = true;
  double f1 = 0.02, f2 = 1e-3, f3 = 1e-5;
};

struct DomainOut {
  int64_t ienv, jenv, iali, jali, kali, mali;
  float bits, bias;
  double lnp;
};
struct HitOut {
  float bits, bias;
  double lnp;
  float nexpected;
  int64_t nregions;
  std::vector<DomainOut> domains;
};

// Raw, still-scaled Forward / Backward special-state rows produced on the
// device: per row i the five values N B E J C and the row's rescale factor
// (0 when the row was not rescaled).
struct RawRows {
  const float* fwd;  // (L+1) x 6, row 0 unused
  const float* bwd;  // (L+1) x 6; row 0 holds the B sum in slot 1
};

// From the raw rows: exact Forward/Backward scores and special rows (using
// the same libm as the reference), then posterior decoding, region
// identification, envelope rescoring, null2 and final scores
// (src/hmmer/pipeline.rs:187-293).  Returns false when the pair yields no hit.
// `fwdsc_out` receives the Forward score (for the F3 decision by the caller).
float forward_score_from_rows(const ProfileHost& p, int64_t l, const float* fwd_rows);
float backward_score_from_rows(int64_t l, const float* bwd_rows);
// Batched domain definition: the same results as define_domains, with the
// full-matrix envelope passes of every pair of a batch done elsewhere (on
// the device).  Phases: begin() per pair (decoding, regions; the stochastic
// traces of multi-domain regions either here or, with device_regions, by the
// caller: regions() -> device trace passes -> expand() per region, which
// clusters the samples on the host) -> requests() -> the caller runs the
// Forward and Backward envelope passes -> factors() per request -> the caller
// runs the posterior / null2 / optimal-accuracy pass -> finish() per pair.
struct EnvRequest {
  int32_t pair;     // index of the pair in the batch
  int32_t p, t;     // profile and target indices
  int64_t i, j;     // envelope, 1-based residues of the target
  bool null2_done;  // null2 already set by the region's stochastic traces
  SpecialTr st;     // unihit special transitions of the target's length
};
struct EnvFactors {
  bool ok = false;  // Forward and Backward envelope scores finite
  float envsc = 0;
  std::vector<double> fac;        // exp(lnF[i] + lnB[i] - lnZ), rows 0..lr
  std::vector<float> pn, pj, pc;  // N/J/C posteriors, rows 0..lr
  float sn = 0, sj = 0, sc = 0;   // their sums over rows 1..lr, in order
};
struct EnvDeviceOut {
  float v[NRES];  // sum_k (sm[k] * norm) * mo[x][k]
  float si;       // sum of insert posteriors, row-major
  bool found;     // optimal-accuracy traceback found a domain
  int32_t i0, i1, k0, k1;
};
// A multi-domain region whose stochastic traces run on the device.
struct RegionRequest {
  int32_t pair;   // index of the pair in the batch
  int32_t p, t;   // profile and target indices
  int64_t i, j;   // region, 1-based residues of the target
  SpecialTr st;   // multihit special transitions of the target's length
  int32_t local;  // the region's number within its pair
};
// One sampled domain of a region's trace ensemble (p7_spcoord_s), target coordinates.
struct TraceSample {
  int32_t trace;
  int64_t i, j;
  int32_t k, m;
};
class DomainBatch {
 public:
  DomainBatch(const SearchOpts& o, size_t npairs);
  ~DomainBatch();
  // device_regions: the stochastic traces of multi-domain regions are left to
  // the caller (regions() -> device passes -> expand()); otherwise they run here.
  void begin(size_t q, const ProfileHost& p, int32_t pi, const uint8_t* dsq, int64_t l, int32_t ti,
             const RawRows& rows, float fwdsc, bool device_regions = false);
  const std::vector<RegionRequest>& regions();  // built on the first call, after every begin()
  // Region r's trace ensemble: its samples in trace order and the per-position
  // null2 sums (positions 1..lr); ok = false redoes the ensemble on the host.
  void expand(size_t r, const std::vector<TraceSample>& samples, const float* n2sum, bool ok);
  // LCG state the device trace streams start from (seed 42 through esl_mix3).
  static uint32_t trace_lcg_start();
  const std::vector<EnvRequest>& requests();
  void factors(size_t r, const float* fwd_rows, const float* bwd_rows, EnvFactors& f) const;
  bool finish(size_t q, const std::vector<EnvFactors>& f, const std::vector<EnvDeviceOut>& d, HitOut& out);

 private:
  struct Impl;
  std::unique_ptr<Impl> impl_;
};

bool define_domains(const ProfileHost& p, const uint8_t* dsq, int64_t l, const RawRows& rows, float fwdsc,
                    const SearchOpts& o, HitOut& out);

// bias_filter_score (src/hmmer/pipeline.rs:107-150), exact host version.
float composition_bias_score(const ProfileHost& p, const uint8_t* dsq, int64_t l);

// P-values (src/hmmer/pipeline.rs:87-104).
double gumbel_survival(double x, double mu, double lambda);
double exp_tail_logsurv(double x, double tau, double lambda);

}  // namespace sx
