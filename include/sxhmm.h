/*
 * sxhmm — B200 hmmsearch engine, C ABI.
 *
 * Drop-in for the hmmsearch engine of raw-lab/sentinel-x (src/hmmer).  The
 * boundary sits below `search_profiles` (src/hmmer/search.rs:213): parsing,
 * profile configuration and reporting keep the reference's semantics on the
 * host; the (profile x target) pair loop and the per-pair pipeline
 * (`score_target`, src/hmmer/pipeline.rs:154) run on one NVIDIA B200.
 *
 * Conventions: every call returns SX_OK (0) or an SX_E* error class; the
 * message of the last error on the calling thread is sx_last_error().  Inputs
 * are borrowed for the duration of a call.  Objects returned through `out`
 * pointers belong to the library until the matching *_free.  No call aborts or
 * exits the process.  Calls on one engine are serialised by the engine.
 */
#ifndef SXHMM_H
#define SXHMM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error classes ---------------------------------------------------- */
#define SX_OK 0
#define SX_EINVAL 1    /* bad argument / malformed input (e.g. a .hmm parse error)  */
#define SX_ECUTOFF 2   /* GA/NC/TC cutoff requested but absent (search.rs:135-146)  */
#define SX_ENOMEM 3    /* host or device allocation failed / admission refused     */
#define SX_ECUDA 4     /* CUDA runtime error                                        */
#define SX_ETIMEOUT 5  /* a bounded device wait gave up                             */
#define SX_EIO 6       /* file could not be opened or read                          */

/* Cutoff kinds (hmmsearch -E/--domE, -T/--domT, --cut_ga/nc/tc;
 * src/hmmer/search.rs:26-38). */
#define SX_CUT_EVALUE 0
#define SX_CUT_BITS 1
#define SX_CUT_GA 2
#define SX_CUT_NC 3
#define SX_CUT_TC 4

/* Engine options. */
#define SX_FLAG_PLAIN 1u /* run the plain one-pair-per-block kernels instead of the batched cascade */
/* Where the envelope rescoring of domain definition runs (default: chosen per
 * profile block; the device when the host's share would not hide behind the
 * device cascade).  Results are identical either way. */
#define SX_FLAG_ENV_DEVICE 2u /* always on the device */
#define SX_FLAG_ENV_HOST 4u   /* always on the host */
/* Where the stochastic-trace ensembles of multi-domain regions (200 sampled
 * traces each, region_trace_ensemble) run when a block's envelopes go to the
 * device (default: chosen per profile block; the device when the block's
 * regions would cost the host pool more than one device trace pass takes).
 * Results are identical either way. */
#define SX_FLAG_TRACE_HOST 8u    /* always on the host */
#define SX_FLAG_TRACE_DEVICE 16u /* always on the device (with the envelopes) */
/* MSV runs as a packed int16x2 pre-screen (an upper bound of the f32 score for
 * two profiles per 32-bit lane) followed by the exact f32 MSV of the pairs whose
 * bound passes F1; this flag runs the exact kernel on every pair instead.
 * Results are identical either way. */
#define SX_FLAG_NO_PRESCREEN 32u

typedef struct sx_engine sx_engine;
typedef struct sx_profiles sx_profiles;
typedef struct sx_targets sx_targets;
typedef struct sx_hits sx_hits;

typedef struct {
  int32_t device;       /* CUDA device ordinal                                       */
  int32_t host_threads; /* host threads for domain definition; 0 = all cores         */
  uint32_t flags;       /* SX_FLAG_*                                                 */
  int32_t pipeline_blocks; /* profile blocks per search whose host domain definition
                              overlaps the next block's device cascade; 0 = automatic */
  int64_t batch_bytes;  /* device bytes per streamed batch; 0 = 2 GiB                */
} sx_opts;

/* PipelineConfig + SearchConfig (src/hmmer/pipeline.rs:27-42,
 * src/hmmer/search.rs:42-47).  z = NaN means "number of targets". */
typedef struct {
  int32_t cutoff_kind;  /* SX_CUT_* */
  int32_t filters;      /* 0 = hmmsearch --max */
  int32_t null2;        /* 0 = --nonull2 */
  int32_t reserved;
  double seq_threshold; /* E-value or bits, per cutoff_kind (ignored for GA/NC/TC) */
  double dom_threshold;
  double f1, f2, f3;
  double z;
} sx_search_cfg;

/* One reported target: `Hit` (src/hmmer/search.rs:101-116). */
typedef struct {
  int32_t profile_index; /* index in the sx_profiles set */
  int32_t target_index;  /* index in the sx_targets set  */
  int32_t qlen, tlen;
  float score, bias;
  double evalue;
  float nexpected;
  int32_t ndomains;
  int32_t domain_offset; /* first domain in sx_hits_domains() */
  int32_t reserved;
} sx_hit;

/* One domain: `DomainHit` (src/hmmer/search.rs:84-97). */
typedef struct {
  float score, bias;
  double c_evalue, i_evalue;
  int32_t hmm_from, hmm_to, ali_from, ali_to, env_from, env_to;
  int32_t reported;
  int32_t reserved;
} sx_domain;

/* Header of one profile: name, accession, M, cutoffs and STATS
 * (src/hmmer/model.rs:53-71). Missing values are NaN; strings live as long
 * as the sx_profiles set. */
typedef struct {
  const char* name;
  const char* acc;  /* NULL if absent */
  const char* desc; /* NULL if absent */
  int32_t m;
  int32_t calibrated;
  float ga[2], tc[2], nc[2];
  double msv[2], viterbi[2], forward[2]; /* (mu|tau, lambda) */
} sx_profile_info;

/* ---- engine ------------------------------------------------------------ */
/* New: one engine per device.  sx_destroy releases the engine's streams at
 * once; profile and target sets of the engine may still be freed afterwards
 * (the engine's memory goes when its last set does), but no other call may
 * name the engine or its sets after sx_destroy. */
int sx_create(const sx_opts* opts, sx_engine** out);
void sx_destroy(sx_engine* e);
/* Message of the last error on this thread ("" if none). */
const char* sx_last_error(void);

/* ---- profiles ---------------------------------------------------------- */
/* Replaces open_hmm + HmmReader + Hmm::configure (src/hmmer/parse.rs:42-236,
 * src/hmmer/model.rs:146-245): parses a HMMER3/b..f file (gzip detected by
 * magic bytes), configures every profile and uploads it to the device. */
int sx_profiles_load_file(sx_engine* e, const char* path, sx_profiles** out);
/* Same from an in-memory HMMER3 text; `source` names it in error messages. */
int sx_profiles_load_text(sx_engine* e, const char* text, size_t len, const char* source, sx_profiles** out);
/* One profile already configured by the caller, as the plain arrays of
 * `Profile` (src/hmmer/model.rs:75-113): the input of search_profiles(&[Profile],
 * ...) (src/hmmer/search.rs:213).  w = m + 1; every array is read during the
 * call only. */
typedef struct {
  const char* name;     /* required */
  const char* acc;      /* NULL if absent */
  const char* desc;     /* NULL if absent */
  int32_t m;            /* model length M, 1..2048 */
  int32_t has_cutoffs;  /* bit 0 GA, bit 1 TC, bit 2 NC */
  const float* msc;     /* [25][w] match log-odds msc[x*w+k] (column 0 -inf) */
  const float* mo;      /* [25][w] match odds */
  const float* t;       /* [8][w] log transitions of node k: mm mi md im ii dm dd, then bm (B->M_k) */
  const float* p;       /* [8][w] probability-space copies, same order */
  const float* compo;   /* [20] composition used by the bias filter */
  float msv_tbm;        /* ln(2/(M(M+1))) */
  float ga[2], tc[2], nc[2];
  int32_t has_stats;    /* bit 0 MSV, bit 1 Viterbi, bit 2 Forward */
  double msv[2], viterbi[2], forward[2]; /* (mu|tau, lambda) */
} sx_profile_arrays;
/* Uploads n configured profiles (replaces nothing on the reference side: its
 * callers hand `&[Profile]` to search_profiles directly). */
int sx_profiles_from_arrays(sx_engine* e, const sx_profile_arrays* profiles, size_t n, sx_profiles** out);
/* A binary cache of configured profiles: sx_profiles_save writes the set in
 * the library's own format (little-endian, versioned, checksummed) and
 * sx_profiles_load_binary reads it back without parsing or configuring, for
 * large libraries such as Pfam-A.  No counterpart in the reference. */
int sx_profiles_save(const sx_profiles* p, const char* path);
int sx_profiles_load_binary(sx_engine* e, const char* path, sx_profiles** out);
int32_t sx_profiles_count(const sx_profiles* p);
int sx_profiles_info(const sx_profiles* p, int32_t i, sx_profile_info* out);
void sx_profiles_free(sx_profiles* p);

/* ---- targets ----------------------------------------------------------- */
/* Replaces Targets::new (src/hmmer/search.rs:56-67): digitises ASCII protein
 * sequences (src/hmmer/alphabet.rs:58-93) and uploads them.  ids may be NULL. */
int sx_targets_create(sx_engine* e, const char* const* ids, const uint8_t* const* seqs, const size_t* lens, size_t n,
                      sx_targets** out);
/* Already-digitised residues (codes 0..24) packed back to back: target i is
 * dsq[offsets[i] .. offsets[i]+lens[i]). */
int sx_targets_create_digital(sx_engine* e, const uint8_t* dsq, const int64_t* offsets, const int64_t* lens, size_t n,
                              sx_targets** out);
int64_t sx_targets_count(const sx_targets* t);
void sx_targets_free(sx_targets* t);

/* ---- search ------------------------------------------------------------ */
/* Replaces search_profiles (src/hmmer/search.rs:213-234): every profile x
 * every target through MSV -> bias -> Viterbi -> Forward filters, Backward,
 * posterior domain definition, envelope rescoring, null2 and reporting.  Hits
 * come out in profile order, then target order, like the reference. */
int sx_search(sx_engine* e, const sx_profiles* p, const sx_targets* t, const sx_search_cfg* cfg, sx_hits** out);
/* Batched sx_search for callers that issue many small searches over the same
 * targets (BUSCO: one single-profile search per file, src/busco/mod.rs:297-304;
 * CheckV: one search per HMM file, src/checkv/mod.rs:370-371).  The n profile
 * sets run as one device search; out[i] receives exactly the hits
 * sx_search(e, sets[i], t, cfg, ...) returns (profile_index relative to set i).
 * Fails, with out[] all NULL, if sx_search would fail for any set. */
int sx_search_many(sx_engine* e, const sx_profiles* const* sets, size_t n, const sx_targets* t,
                   const sx_search_cfg* cfg, sx_hits** out);
size_t sx_hits_count(const sx_hits* h);
const sx_hit* sx_hits_array(const sx_hits* h);
size_t sx_hits_domain_count(const sx_hits* h);
const sx_domain* sx_hits_domains(const sx_hits* h);
void sx_hits_free(sx_hits* h);

/* Per-stage counters of the last sx_search on this engine: pairs entering and
 * leaving each stage, DP cells per stage and milliseconds per stage.
 * stage: 0 MSV, 1 bias, 2 Viterbi, 3 Forward pre-screen (device, CUDA
 * events), 4 Forward/Backward row passes of the final pairs (device + copies),
 * 5 domain definition (busy time of the host pool, which overlaps the
 * device stages of later profile blocks), 6 whole call (host clock), 7 host
 * time after the last device work (the part of stage 5 not hidden).
 * pairs_out[5] counts the envelopes rescored by the device passes.
 * Slot 6: stochastic-trace ensembles of multi-domain regions on the device:
 * pairs_in[6] regions sent, pairs_out[6] regions the device completed (the
 * rest are redone on the host), cells[6] DP cells of their Forward matrices. */
typedef struct {
  int64_t pairs_in[8], pairs_out[8];
  double cells[8];
  double ms[8];
  int64_t kernel_launches;
  /* the packed MSV pre-screen (part of stage 0): pairs it bounded, pairs
   * whose bound passed F1 (rescored exactly), its DP cells, the device time
   * of the pre-screen and of the exact rescoring */
  int64_t prescreen_pairs_in, prescreen_pairs_out;
  double prescreen_cells, prescreen_ms, rescore_ms;
  /* the packed Viterbi pre-screen (part of stage 2): bias-filter survivors
   * it bounded, those whose bound passed F2 (scored exactly; the exact
   * Viterbi also takes the pairs of profiles it does not handle), its DP
   * cells and device time */
  int64_t vprescreen_pairs_in, vprescreen_pairs_out;
  double vprescreen_cells, vprescreen_ms;
} sx_search_stats;
int sx_last_search_stats(const sx_engine* e, sx_search_stats* out);

/* ---- kernel shapes (for tuners) ------------------------------------------ */
/* kind 0: MSV lane-group shapes (G lanes x C columns per lane); kind 1:
 * Viterbi lane-group shapes (G, C, transitions held in registers).  A profile
 * of M <= 2048 nodes runs with the shape the engine's table gives for M, else
 * with the built-in choice.  sx_set_shape_table takes one entry per M =
 * 0..2048 (-1 = the cost model; a shape must hold G*C >= M columns), or len
 * = 0 to restore the built-in table (for Viterbi the shapes measured fastest
 * per range of M on B200); it applies to profile sets loaded afterwards. */
int sx_shape_count(int kind);
int sx_shape_info(int kind, int index, int32_t* g, int32_t* c, int32_t* rt);
int sx_shape_for(const sx_engine* e, int kind, int32_t m);
int sx_set_shape_table(sx_engine* e, int kind, const int32_t* shape_by_m, size_t len);

/* ---- stage scores for explicit pairs ----------------------------------- */
/* Scores of msv (dp.rs:69), viterbi_score (dp.rs:152), forward (dp.rs:229),
 * backward (dp.rs:301) and bias_filter_score (pipeline.rs:107) for each pair
 * (pair_profile[i], pair_target[i]), target-length configured and multihit
 * as in score_target.  Any output pointer may be NULL to skip that stage. */
int sx_score_pairs(sx_engine* e, const sx_profiles* p, const sx_targets* t, const int32_t* pair_profile,
                   const int32_t* pair_target, size_t npairs, float* msv, float* viterbi, float* forward,
                   float* backward, float* bias);

/* ---- pre-screen bounds for explicit pairs (diagnostics) ------------------ */
/* No counterpart in the reference: the two conservative screens the device
 * cascade runs in front of exact stages, for tests and tuning.
 *   msv_bound: the packed int16x2 MSV pre-screen's upper bound of the f32 MSV
 *     score (nats; +inf when the pair hit the int16 headroom cap and passes
 *     unconditionally).  It is >= the msv score of sx_score_pairs for every
 *     pair; NaN for profiles the pre-screen does not handle (M > 2048, or
 *     match scores above +16 nats).
 *   fwd_scan: the F3 pre-screen's Forward score (nats), evaluated in a
 *     parallel order that differs from the reference's; its difference from
 *     the exact Forward score is bounded by (L+1)(2M + 6 VC + 64) 2^-24 nats,
 *     taken twice (VC = columns per lane of the profile's warp-chunked image);
 *     NaN for M > 2048.
 *   vit_bound: the packed int16x2 Viterbi pre-screen's upper bound of the
 *     f32 Viterbi score (nats; +inf when capped).  It is >= the viterbi score
 *     of sx_score_pairs for every pair; NaN for empty targets and for
 *     profiles the pre-screen does not handle (M > 512, profiles outside the
 *     MSV pre-screen, match scores above +16 nats).
 * Any output pointer may be NULL to skip that screen. */
int sx_score_prescreens(sx_engine* e, const sx_profiles* p, const sx_targets* t, const int32_t* pair_profile,
                        const int32_t* pair_target, size_t npairs, float* msv_bound, float* fwd_scan,
                        float* vit_bound);

/* ---- adjoint ----------------------------------------------------------- */
/* Gradient of each pair's Forward log score lnZ (multihit, target-length
 * config; dp.rs:229-298) with respect to the profile's log-space scores:
 *   d_msc [npairs][25][M+1]  match emission scores msc[x][k]
 *   d_isc [npairs][25][M+1]  insert emission scores (0 in the model)
 *   d_trans[npairs][8][M+1]  transitions MM MI MD IM II DM DD of source node k,
 *                            then the local entry B->M_k
 * i.e. the posterior expected counts of each emission and transition (the
 * quantities decode(), dp.rs:1278-1306, sums for domain definition).  All
 * pairs must use profiles of one length M (= m).  lnz[npairs] receives lnZ.
 * The Forward pass keeps sqrt(L) checkpoint rows and Backward recomputes the
 * rows between checkpoints, so device scratch is O(M sqrt(L)) per pair. */
int sx_posterior_grad(sx_engine* e, const sx_profiles* p, const sx_targets* t, const int32_t* pair_profile,
                      const int32_t* pair_target, size_t npairs, int32_t m, float* d_msc, float* d_isc,
                      float* d_trans, double* lnz);

/* ---- scoring without allocation ----------------------------------------- */
/* No counterpart in the reference.  Viterbi scores (as sx_score_pairs computes
 * them) for up to 8192 pairs per call, for callers that must not allocate GPU
 * memory during the call: for example a host program that shares the GPU with
 * another runtime whose caching allocator already holds nearly all device
 * memory, or a latency-bound caller that cannot absorb the device-wide
 * synchronisation a cudaMalloc/cudaFree can imply.  Instead of engine scratch
 * it uses one fixed device array of about 360 KB that every GPU holding this
 * library keeps reserved until the process exits.  The first call on a device
 * looks up that array's device address (and the first call after the device's
 * context was replaced, e.g. by cudaDeviceReset, looks it up again); make that
 * first call before any stream capture begins on the device.  Profiles and
 * targets must belong to the engine passed (SX_EINVAL otherwise).  More than 8192 pairs is an SX_EINVAL
 * error.  All calls on a device share the array: calls that overlap on the
 * GPU (for example from two engines on one device) race; calls on one engine
 * are serialised.  Inputs and outputs are host arrays, as for sx_score_pairs. */
int sx_score_viterbi_static(sx_engine* e, const sx_profiles* p, const sx_targets* t, const int32_t* pair_profile,
                            const int32_t* pair_target, size_t npairs, float* viterbi);

#ifdef __cplusplus
}
#endif
#endif /* SXHMM_H */
