// sxhmm engine: the C ABI of include/sxhmm.h -- engine lifecycle, profile
// and target sets, the search entry points, hits, shape tables and stats.
// The rest of the engine: shared objects and declarations in engine.hpp,
// shape choice and device images in pack.cu, the search scheduler in
// scheduler.cu, the device domain-definition passes in domain_passes.cu,
// explicit-pair scoring in score.cu, the allocation-free entry point in
// static_entry.cu.
//
// Flow of sx_search (replaces the rayon pair loop of search_profiles,
// src/hmmer/search.rs:213-234, and score_target, src/hmmer/pipeline.rs:154):
//   1. MSV over every (profile, target) pair: CTA tiles of (profile, slice of
//      the length-sorted targets); exact F1 decision; survivors appended to
//      per-shape lists.
//   2. composition-bias filter, 3. Viterbi, 4. Forward score: each a
//      pair-list kernel over the previous stage's survivors; decisions that
//      involve a device logarithm are taken with a small slack so the device
//      never rejects a pair the reference keeps.
//   5. host: exact re-check of every decision with the reference's libm;
//      device Forward/Backward passes that emit the raw special rows of the
//      final pairs (chunked); host posterior domain definition, envelope
//      rescoring and reporting on a thread pool.
// Steps 1-5 run per block of profiles; a block's host domain definition is
// queued to a background pool and overlaps the device work of later blocks.
#include "engine.hpp"

namespace sxe {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

const KernelTables& kernels() {
  static const KernelTables t = [] {
    KernelTables k;
    fill_msv_tables(k);
    fill_msv16_tables(k);
    fill_vit_tables(k);
    fill_vit16_tables(k);
    fill_vbin_tables(k);
    fill_env_tables(k);
    return k;
  }();
  return t;
}

}  // namespace sxe

// ================================================================ C ABI
extern "C" {

const char* sx_last_error(void) { return g_err.c_str(); }

int sx_create(const sx_opts* opts, sx_engine** out) {
  if (!out) return fail(SX_EINVAL, "sx_create: out is NULL");
  *out = nullptr;
  auto e = std::make_unique<sx_engine>();
  e->device = opts ? opts->device : 0;
  e->flags = opts ? opts->flags : 0;
  e->host_threads = (opts && opts->host_threads > 0) ? opts->host_threads : (int)std::thread::hardware_concurrency();
  e->host_threads = std::max(1, e->host_threads);
  e->batch_bytes = (opts && opts->batch_bytes > 0) ? opts->batch_bytes : (2LL << 30);
  e->pipeline_blocks = (opts && opts->pipeline_blocks > 0) ? opts->pipeline_blocks : 0;
  try {
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (e->device < 0 || e->device >= ndev)
      return fail(SX_EINVAL, "sx_create: device " + std::to_string(e->device) + " not present (" +
                                 std::to_string(ndev) + " devices)");
    CK(cudaSetDevice(e->device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, e->device));
    if (prop.major < 10)
      return fail(SX_EINVAL, std::string("sx_create: device is ") + prop.name + " (sm_" + std::to_string(prop.major) +
                                 std::to_string(prop.minor) + "); this library is built for sm_100a");
    e->num_sms = prop.multiProcessorCount;
    for (Slot& S : e->sl) S.create();
    {
      int least = 0, greatest = 0;
      CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
      CK(cudaStreamCreateWithPriority(&e->env_stream, cudaStreamNonBlocking, greatest));
      CK(cudaEventCreateWithFlags(&e->env_ev, cudaEventDisableTiming));
    }
    note_free_memory(e.get());
    for (int kind = 0; kind < 2; kind++) e->shape_table[kind] = default_shape_table(kind);
    (void)kernels();
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  }
  *out = e.release();
  return SX_OK;
}

void sx_destroy(sx_engine* e) {
  if (!e) return;
  cudaSetDevice(e->device);
  for (Slot& S : e->sl) S.destroy();
  if (e->env_stream) {
    cudaStreamSynchronize(e->env_stream);
    cudaStreamDestroy(e->env_stream);
  }
  if (e->env_ev) cudaEventDestroy(e->env_ev);
  e->env_stream = nullptr;
  e->env_ev = nullptr;
  bool last;
  {
    std::lock_guard<std::mutex> g(e->life_mu);
    e->destroyed = true;
    last = e->live_sets == 0;
  }
  if (last) delete e;
}

// A set handed to the caller keeps its engine object alive (see sx_engine).
static void engine_ref(sx_engine* e) {
  std::lock_guard<std::mutex> g(e->life_mu);
  e->live_sets++;
}
static void engine_unref(sx_engine* e) {
  bool last;
  {
    std::lock_guard<std::mutex> g(e->life_mu);
    last = --e->live_sets == 0 && e->destroyed;
  }
  if (last) delete e;
}

static int finish_profiles(sx_engine* e, std::unique_ptr<sx_profiles> p, sx_profiles** out) {
  try {
    CK(cudaSetDevice(e->device));
    pack_profiles(p.get());
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  }
  engine_ref(e);
  *out = p.release();
  return SX_OK;
}

int sx_profiles_load_text(sx_engine* e, const char* text, size_t len, const char* source, sx_profiles** out) {
  if (!e || !out || (!text && len)) return fail(SX_EINVAL, "sx_profiles_load_text: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(e->mu);
  auto p = std::make_unique<sx_profiles>();
  p->eng = e;
  std::string err;
  if (!load_profiles_text(text ? text : "", len, source ? source : "<stream>", p->h, err)) return fail(SX_EINVAL, err);
  return finish_profiles(e, std::move(p), out);
}

int sx_profiles_from_arrays(sx_engine* e, const sx_profile_arrays* a, size_t n, sx_profiles** out) {
  if (!e || !out || (n && !a)) return fail(SX_EINVAL, "sx_profiles_from_arrays: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(e->mu);
  auto p = std::make_unique<sx_profiles>();
  p->eng = e;
  p->h.resize(n);
  for (size_t i = 0; i < n; i++) {
    const sx_profile_arrays& s = a[i];
    const std::string at = "sx_profiles_from_arrays: profile " + std::to_string(i);
    if (!s.name || !s.msc || !s.mo || !s.t || !s.p || !s.compo) return fail(SX_EINVAL, at + ": NULL field");
    if (s.m < 1) return fail(SX_EINVAL, at + ": M must be at least 1");
    ProfileHost& h = p->h[i];
    const size_t w = (size_t)s.m + 1;
    h.name = s.name;
    h.has_acc = s.acc != nullptr;
    h.has_desc = s.desc != nullptr;
    if (s.acc) h.acc = s.acc;
    if (s.desc) h.desc = s.desc;
    h.m = s.m;
    h.msc.assign(s.msc, s.msc + NSYM * w);
    h.mo.assign(s.mo, s.mo + NSYM * w);
    for (int q = 0; q < NTR; q++) {
      h.t[q].assign(s.t + q * w, s.t + (q + 1) * w);
      h.p[q].assign(s.p + q * w, s.p + (q + 1) * w);
    }
    h.msv_tbm = s.msv_tbm;
    std::copy(s.compo, s.compo + NRES, h.compo);
    h.has_ga = s.has_cutoffs & 1;
    h.has_tc = (s.has_cutoffs >> 1) & 1;
    h.has_nc = (s.has_cutoffs >> 2) & 1;
    for (int q = 0; q < 2; q++) {
      h.ga[q] = h.has_ga ? s.ga[q] : NAN;
      h.tc[q] = h.has_tc ? s.tc[q] : NAN;
      h.nc[q] = h.has_nc ? s.nc[q] : NAN;
    }
    h.has_msv = s.has_stats & 1;
    h.has_vit = (s.has_stats >> 1) & 1;
    h.has_fwd = (s.has_stats >> 2) & 1;
    for (int q = 0; q < 2; q++) {
      h.msv[q] = h.has_msv ? s.msv[q] : NAN;
      h.vit[q] = h.has_vit ? s.viterbi[q] : NAN;
      h.fwd[q] = h.has_fwd ? s.forward[q] : NAN;
    }
  }
  return finish_profiles(e, std::move(p), out);
}

int sx_profiles_load_file(sx_engine* e, const char* path, sx_profiles** out) {
  if (!e || !out || !path) return fail(SX_EINVAL, "sx_profiles_load_file: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(e->mu);
  auto p = std::make_unique<sx_profiles>();
  p->eng = e;
  std::string err;
  bool io = false;
  if (!load_profiles_file(path, p->h, err, io)) return fail(io ? SX_EIO : SX_EINVAL, err);
  return finish_profiles(e, std::move(p), out);
}

int sx_profiles_save(const sx_profiles* p, const char* path) {
  if (!p || !path) return fail(SX_EINVAL, "sx_profiles_save: NULL argument");
  std::string err;
  if (!save_profiles_binary(p->h, path, err)) return fail(SX_EIO, "sx_profiles_save: " + err);
  return SX_OK;
}

int sx_profiles_load_binary(sx_engine* e, const char* path, sx_profiles** out) {
  if (!e || !out || !path) return fail(SX_EINVAL, "sx_profiles_load_binary: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(e->mu);
  auto p = std::make_unique<sx_profiles>();
  p->eng = e;
  std::string err;
  bool io = false;
  if (!load_profiles_binary(path, p->h, err, io)) return fail(io ? SX_EIO : SX_EINVAL, "sx_profiles_load_binary: " + err);
  return finish_profiles(e, std::move(p), out);
}

int32_t sx_profiles_count(const sx_profiles* p) { return p ? (int32_t)p->h.size() : 0; }

int sx_profiles_info(const sx_profiles* p, int32_t i, sx_profile_info* out) {
  if (!p || !out || i < 0 || i >= (int32_t)p->h.size()) return fail(SX_EINVAL, "sx_profiles_info: bad index");
  const ProfileHost& h = p->h[i];
  out->name = h.name.c_str();
  out->acc = h.has_acc ? h.acc.c_str() : nullptr;
  out->desc = h.has_desc ? h.desc.c_str() : nullptr;
  out->m = h.m;
  out->calibrated = h.calibrated();
  for (int q = 0; q < 2; q++) {
    out->ga[q] = h.has_ga ? h.ga[q] : NAN;
    out->tc[q] = h.has_tc ? h.tc[q] : NAN;
    out->nc[q] = h.has_nc ? h.nc[q] : NAN;
    out->msv[q] = h.has_msv ? h.msv[q] : NAN;
    out->viterbi[q] = h.has_vit ? h.vit[q] : NAN;
    out->forward[q] = h.has_fwd ? h.fwd[q] : NAN;
  }
  return SX_OK;
}

void sx_profiles_free(sx_profiles* p) {
  if (!p) return;
  sx_engine* e = p->eng;
  cudaSetDevice(e->device);
  delete p;
  engine_unref(e);
}

static int finish_targets(sx_engine* e, std::unique_ptr<sx_targets> t, sx_targets** out) {
  t->dsq.resize(t->dsq.size() + 64, SYM_STAR);  // read slack past the last target
  try {
    CK(cudaSetDevice(e->device));
    pack_targets(t.get());
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  }
  engine_ref(e);
  *out = t.release();
  return SX_OK;
}

int sx_targets_create(sx_engine* e, const char* const* ids, const uint8_t* const* seqs, const size_t* lens, size_t n,
                      sx_targets** out) {
  if (!e || !out || (n && (!seqs || !lens))) return fail(SX_EINVAL, "sx_targets_create: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(e->mu);
  auto t = std::make_unique<sx_targets>();
  t->eng = e;
  size_t total = 64;  // an upper bound of the packed size
  for (size_t i = 0; i < n; i++) total += (lens[i] + 15) & ~(size_t)15;
  t->dsq = e->target_bytes.take(total);
  std::vector<uint8_t> dig;
  for (size_t i = 0; i < n; i++) {
    dig.clear();
    for (size_t q = 0; q < lens[i]; q++) {
      const uint8_t b = seqs[i][q];
      if (b == ' ' || b == '\t' || b == '\n' || b == '\r' || b == '\f' || b == '\v') continue;
      dig.push_back(kDigitize[b]);
    }
    if (dig.size() > (size_t)INT32_MAX) return fail(SX_EINVAL, "sx_targets_create: sequence too long");
    append_target(t.get(), dig.data(), dig.size());
    t->ids.push_back(ids && ids[i] ? ids[i] : std::to_string(i));
  }
  return finish_targets(e, std::move(t), out);
}

int sx_targets_create_digital(sx_engine* e, const uint8_t* dsq, const int64_t* offsets, const int64_t* lens, size_t n,
                              sx_targets** out) {
  if (!e || !out || (n && (!dsq || !offsets || !lens))) return fail(SX_EINVAL, "sx_targets_create_digital: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(e->mu);
  auto t = std::make_unique<sx_targets>();
  t->eng = e;
  size_t total = 64;
  for (size_t i = 0; i < n; i++) {
    if (lens[i] < 0 || offsets[i] < 0 || lens[i] > INT32_MAX) return fail(SX_EINVAL, "sx_targets_create_digital: bad length");
    total += ((size_t)lens[i] + 15) & ~(size_t)15;
  }
  t->dsq = e->target_bytes.take(total);
  // packed offsets first; then each target is checked, copied and padded
  // with '*' to its 16-byte boundary, targets spread over the host threads
  // (sets of a few MB and more: a Pfam-scale set of 50,000 targets is
  // repacked for every search of a streaming caller)
  t->off.resize(n);
  t->len.resize(n);
  int64_t o = 0;
  for (size_t i = 0; i < n; i++) {
    t->off[i] = o;
    t->len[i] = (int32_t)lens[i];
    o += (lens[i] + 15) & ~(int64_t)15;
  }
  t->dsq.resize((size_t)o);
  uint8_t* out8 = t->dsq.data();
  std::atomic<size_t> bad{SIZE_MAX};
  const size_t nchunk = o >= (1 << 22) ? std::min<size_t>(n, 8 * (size_t)e->host_threads) : 1;
  parallel_for(nchunk, e->host_threads, [&](size_t c) {
    for (size_t i = n * c / nchunk; i < n * (c + 1) / nchunk; i++) {
      const uint8_t* d = dsq + offsets[i];
      uint8_t hi = 0;  // max code, a loop the compiler vectorises; positions only on failure
      for (int64_t q = 0; q < lens[i]; q++) hi = std::max(hi, d[q]);
      if (hi > SYM_STAR) {
        size_t cur = bad.load();
        while (i < cur && !bad.compare_exchange_weak(cur, i)) {
        }
        return;
      }
      uint8_t* w = out8 + t->off[i];
      if (lens[i]) std::memcpy(w, d, (size_t)lens[i]);
      const int64_t pad = ((lens[i] + 15) & ~(int64_t)15) - lens[i];
      if (pad) std::memset(w + lens[i], SYM_STAR, (size_t)pad);
    }
  });
  if (bad.load() != SIZE_MAX) {
    const size_t i = bad.load();
    const uint8_t* d = dsq + offsets[i];
    for (int64_t q = 0; q < lens[i]; q++)
      if (d[q] > SYM_STAR)
        return fail(SX_EINVAL, "sx_targets_create_digital: residue code " + std::to_string(d[q]) +
                                   " out of range in target " + std::to_string(i));
  }
  return finish_targets(e, std::move(t), out);
}

int64_t sx_targets_count(const sx_targets* t) { return t ? (int64_t)t->len.size() : 0; }

void sx_targets_free(sx_targets* t) {
  if (!t) return;
  sx_engine* e = t->eng;
  cudaSetDevice(e->device);
  delete t;
  engine_unref(e);
}

int sx_search(sx_engine* e, const sx_profiles* p, const sx_targets* t, const sx_search_cfg* cfg, sx_hits** out) {
  if (!e || !p || !t || !cfg || !out) return fail(SX_EINVAL, "sx_search: NULL argument");
  if (p->eng != e || t->eng != e) return fail(SX_EINVAL, "sx_search: profiles/targets belong to another engine");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(e->mu);
  NvtxRange nv("sx_search");
  auto h = std::make_unique<sx_hits>();
  try {
    CK(cudaSetDevice(e->device));
    const int rc = run_search(e, p, t, cfg, h.get());
    if (rc) return rc;
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  } catch (const std::bad_alloc&) {
    return fail(SX_ENOMEM, "sx_search: host allocation failed");
  }
  *out = h.release();
  return SX_OK;
}

int sx_search_many(sx_engine* e, const sx_profiles* const* sets, size_t n, const sx_targets* t,
                   const sx_search_cfg* cfg, sx_hits** out) {
  if (!e || !t || !cfg || !out || (n && !sets)) return fail(SX_EINVAL, "sx_search_many: NULL argument");
  for (size_t i = 0; i < n; i++) out[i] = nullptr;
  if (t->eng != e) return fail(SX_EINVAL, "sx_search_many: targets belong to another engine");
  for (size_t i = 0; i < n; i++)
    if (!sets[i] || sets[i]->eng != e)
      return fail(SX_EINVAL, "sx_search_many: profile set " + std::to_string(i) + " is NULL or of another engine");
  std::lock_guard<std::mutex> lk(e->mu);
  // the first set sx_search would reject decides the error
  for (size_t i = 0; i < n; i++) {
    const int rc = check_cutoffs(sets[i], cfg->cutoff_kind);
    if (rc) return rc;
  }
  // One combined set.  Search and report treat every profile on its own
  // (per-profile thresholds, E-values over the same targets, per-profile
  // domain Z), so slicing the combined hits by profile range is exact.
  std::vector<size_t> first(n + 1, 0);
  auto all = std::make_unique<sx_profiles>();
  all->eng = e;
  for (size_t i = 0; i < n; i++) {
    first[i] = all->h.size();
    all->h.insert(all->h.end(), sets[i]->h.begin(), sets[i]->h.end());
  }
  first[n] = all->h.size();
  std::vector<std::unique_ptr<sx_hits>> parts(n);
  try {
    CK(cudaSetDevice(e->device));
    sx_hits hits;
    if (!all->h.empty()) {
      pack_profiles(all.get());
      const int rc = run_search(e, all.get(), t, cfg, &hits);
      if (rc) return rc;
    }
    size_t q = 0;
    for (size_t i = 0; i < n; i++) {
      parts[i] = std::make_unique<sx_hits>();
      sx_hits& part = *parts[i];
      while (q < hits.hits.size() && (size_t)hits.hits[q].profile_index < first[i + 1]) {
        sx_hit hh = hits.hits[q++];
        const sx_domain* d = hits.doms.data() + hh.domain_offset;
        hh.profile_index -= (int32_t)first[i];
        hh.domain_offset = (int32_t)part.doms.size();
        part.doms.insert(part.doms.end(), d, d + hh.ndomains);
        part.hits.push_back(hh);
      }
    }
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  } catch (const std::bad_alloc&) {
    return fail(SX_ENOMEM, "sx_search_many: host allocation failed");
  }
  for (size_t i = 0; i < n; i++) out[i] = parts[i].release();
  return SX_OK;
}

size_t sx_hits_count(const sx_hits* h) { return h ? h->hits.size() : 0; }
const sx_hit* sx_hits_array(const sx_hits* h) { return h && !h->hits.empty() ? h->hits.data() : nullptr; }
size_t sx_hits_domain_count(const sx_hits* h) { return h ? h->doms.size() : 0; }
const sx_domain* sx_hits_domains(const sx_hits* h) { return h && !h->doms.empty() ? h->doms.data() : nullptr; }
void sx_hits_free(sx_hits* h) { delete h; }

int sx_shape_count(int kind) { return kind == 0 ? kNumMsvShapes : kind == 1 ? kNumVitShapes : -1; }

int sx_shape_info(int kind, int index, int32_t* g, int32_t* c, int32_t* rt) {
  if (kind < 0 || kind > 1 || index < 0 || index >= sx_shape_count(kind) || !g || !c || !rt)
    return fail(SX_EINVAL, "sx_shape_info: bad kind or index");
  if (kind == 0) {
    *g = kMsvShapes[index].g;
    *c = kMsvShapes[index].c;
    *rt = 0;
  } else {
    *g = kVitShapes[index].g;
    *c = kVitShapes[index].c;
    *rt = kVitShapes[index].rt;
  }
  return SX_OK;
}

int sx_shape_for(const sx_engine* e, int kind, int32_t m) {
  if (!e || kind < 0 || kind > 1 || m < 0) return -1;
  return is_long(m) ? -1 : shape_for(e, kind, m);
}

int sx_set_shape_table(sx_engine* e, int kind, const int32_t* shape_by_m, size_t len) {
  if (!e || kind < 0 || kind > 1 || (len && !shape_by_m)) return fail(SX_EINVAL, "sx_set_shape_table: bad argument");
  if (len != 0 && len != (size_t)kMaxM + 1)
    return fail(SX_EINVAL, "sx_set_shape_table: the table has one entry per M = 0.." + std::to_string(kMaxM));
  std::vector<int16_t> t = len ? std::vector<int16_t>(len, -1) : default_shape_table(kind);
  for (size_t m = 0; m < len; m++) {
    const int s = shape_by_m[m];
    if (s < 0) continue;
    if (s >= sx_shape_count(kind)) return fail(SX_EINVAL, "sx_set_shape_table: shape " + std::to_string(s) + " unknown");
    const int cols = kind == 0 ? kMsvShapes[s].g * kMsvShapes[s].c : kVitShapes[s].g * kVitShapes[s].c;
    if (cols < (int)m)
      return fail(SX_EINVAL, "sx_set_shape_table: shape " + std::to_string(s) + " holds " + std::to_string(cols) +
                                 " columns, fewer than M=" + std::to_string(m));
    t[m] = (int16_t)s;
  }
  std::lock_guard<std::mutex> lk(e->mu);
  e->shape_table[kind] = std::move(t);
  return SX_OK;
}

int sx_last_search_stats(const sx_engine* e, sx_search_stats* out) {
  if (!e || !out) return fail(SX_EINVAL, "sx_last_search_stats: NULL argument");
  *out = e->stats;
  return SX_OK;
}

}  // extern "C"
