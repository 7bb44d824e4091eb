#include "engine.hpp"

// ================================================================ no-allocation entry point
//
// sx_score_viterbi_static: Viterbi scores for explicit pairs without any
// allocation.  Its working memory -- the caller's pair indices, the pair
// records grouped by kernel shape, the per-shape list descriptors and the
// output staging -- lives in one file-scope device array of fixed size,
// reserved on every GPU that loads this library for as long as the process
// runs.  The host side uses only stack storage.
namespace {

constexpr size_t kStaticMaxPairs = 8192;
constexpr size_t kStaticPairIdxOff = 0;                                                    // int32 pp[], pt[]
constexpr size_t kStaticRecOff = kStaticPairIdxOff + 2 * kStaticMaxPairs * sizeof(int32_t);  // PairRec[]
constexpr size_t kStaticBinOff = kStaticRecOff + kStaticMaxPairs * sizeof(PairRec);         // BinRegion[]
constexpr size_t kStaticCountOff = kStaticBinOff + 16 * sizeof(BinRegion);                  // unsigned[16]
constexpr size_t kStaticFlagOff = kStaticCountOff + 16 * sizeof(unsigned);                  // unsigned
constexpr size_t kStaticScoreOff = (kStaticFlagOff + 4 + 255) & ~(size_t)255;               // float[]
constexpr size_t kStaticScratchBytes = kStaticScoreOff + kStaticMaxPairs * sizeof(float);
static_assert(kNumVbins <= 16, "static scratch holds at most 16 pair lists");

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

struct StaticLayout {
  int32_t off[16], n[16];
};

// Scatter the caller's pairs into per-shape lists at host-computed offsets
// and publish the list descriptors the Viterbi kernels read.
__global__ void static_bucket_kernel(unsigned char* scratch, int npairs, const DevProfile* __restrict__ profs,
                                     StaticLayout lay) {
  const int32_t* pp = reinterpret_cast<const int32_t*>(scratch + kStaticPairIdxOff);
  const int32_t* pt = pp + kStaticMaxPairs;
  PairRec* recs = reinterpret_cast<PairRec*>(scratch + kStaticRecOff);
  BinRegion* bins = reinterpret_cast<BinRegion*>(scratch + kStaticBinOff);
  unsigned* counts = reinterpret_cast<unsigned*>(scratch + kStaticCountOff);
  __shared__ unsigned cursor[16];
  if (threadIdx.x < 16) {
    cursor[threadIdx.x] = 0;
    if (threadIdx.x < kNumVbins) {
      bins[threadIdx.x].off = lay.off[threadIdx.x];
      bins[threadIdx.x].cap = (uint32_t)lay.n[threadIdx.x];
      bins[threadIdx.x].pad = 0;
      counts[threadIdx.x] = (unsigned)lay.n[threadIdx.x];
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < npairs; i += blockDim.x) {
    const int b = profs[pp[i]].vbin;
    const unsigned pos = (unsigned)lay.off[b] + atomicAdd(&cursor[b], 1u);
    PairRec r;
    r.p = pp[i]; r.t = pt[i]; r.usc = r.filtersc = r.vsc = r.fwd = 0.f; r.slot = i; r.pad = 0;
    recs[pos] = r;
  }
}

// Device address of g_static_scratch for each device, looked up once per
// device context (with that device current): on the first call on the device,
// and again after the device's context has been replaced (cudaDeviceReset
// destroys the primary context and the module that holds the array, so an
// address cached before it would dangle).  The context is told apart by the
// driver's context id, reached through the runtime's driver entry points so
// the library needs no link to libcuda.
std::mutex g_static_mu;
struct StaticAddr {
  void* ptr = nullptr;
  unsigned long long ctx_id = 0;
};
StaticAddr g_static_addr[128];

typedef int (*CtxGetCurrentFn)(void** ctx);
typedef int (*CtxGetIdFn)(void* ctx, unsigned long long* id);

// Id of the calling thread's current context, or 0 when the driver cannot
// report one (the cached address is then kept for the process lifetime).
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
  });
  if (!get_current || !get_id) return 0;
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

int static_scratch_ptr(int device, unsigned char** out) {
  if (device < 0 || device >= 128) return fail(SX_EINVAL, "sx_score_viterbi_static: device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_static_mu);
  StaticAddr& a = g_static_addr[device];
  const unsigned long long ctx = current_context_id();
  if (!a.ptr || ctx != a.ctx_id) {
    void* ptr = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&ptr, g_static_scratch);
    if (rc != cudaSuccess || !ptr)
      return fail(SX_ECUDA, std::string("sx_score_viterbi_static: cudaGetSymbolAddress: ") + cudaGetErrorString(rc));
    a.ptr = ptr;
    a.ctx_id = ctx;
  }
  *out = static_cast<unsigned char*>(a.ptr);
  return SX_OK;
}

}  // namespace

extern "C" int sx_score_viterbi_static(sx_engine* e, const sx_profiles* p, const sx_targets* t,
                                       const int32_t* pair_profile, const int32_t* pair_target, size_t npairs,
                                       float* viterbi) {
  if (!e || !p || !t || (npairs && (!pair_profile || !pair_target || !viterbi)))
    return fail(SX_EINVAL, "sx_score_viterbi_static: NULL argument");
  if (p->eng != e || t->eng != e)
    return fail(SX_EINVAL, "sx_score_viterbi_static: profiles/targets belong to another engine");
  if (npairs > kStaticMaxPairs)
    return fail(SX_EINVAL, "sx_score_viterbi_static: " + std::to_string(npairs) + " pairs exceed the fixed limit of " +
                               std::to_string(kStaticMaxPairs) + " per call");
  std::lock_guard<std::mutex> lk(e->mu);
  const size_t np = p->h.size(), nt = t->len.size();
  StaticLayout lay{};
  for (size_t i = 0; i < npairs; i++) {
    if (pair_profile[i] < 0 || (size_t)pair_profile[i] >= np || pair_target[i] < 0 || (size_t)pair_target[i] >= nt)
      return fail(SX_EINVAL, "sx_score_viterbi_static: pair " + std::to_string(i) + " out of range");
    if (p->dp[pair_profile[i]].vbin < 0)
      return fail(SX_EINVAL, "sx_score_viterbi_static: profiles of M > " + std::to_string(kMaxM) + " are not supported");
    lay.n[p->dp[pair_profile[i]].vbin]++;
  }
  if (!npairs) return SX_OK;
  for (int b = 1; b < kNumVbins; b++) lay.off[b] = lay.off[b - 1] + lay.n[b - 1];
  try {
    CK(cudaSetDevice(e->device));
    unsigned char* scratch = nullptr;
    const int rc = static_scratch_ptr(e->device, &scratch);
    if (rc) return rc;
    cudaStream_t s = e->stream;
    CK(cudaMemcpyAsync(scratch + kStaticPairIdxOff, pair_profile, npairs * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(scratch + kStaticPairIdxOff + kStaticMaxPairs * sizeof(int32_t), pair_target,
                       npairs * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(scratch + kStaticFlagOff, 0, sizeof(unsigned), s));
    static_bucket_kernel<<<1, 1024, 0, s>>>(scratch, (int)npairs, p->d_prof.p, lay);
    const auto& K = kernels();
    const PairRec* recs = reinterpret_cast<const PairRec*>(scratch + kStaticRecOff);
    const BinRegion* bins = reinterpret_cast<const BinRegion*>(scratch + kStaticBinOff);
    const unsigned* counts = reinterpret_cast<const unsigned*>(scratch + kStaticCountOff);
    unsigned* flag = reinterpret_cast<unsigned*>(scratch + kStaticFlagOff);
    float* scores = reinterpret_cast<float*>(scratch + kStaticScoreOff);
    for (int b = 0; b < kNumVbins; b++) {
      if (!lay.n[b]) continue;
      const int blocks = (int)std::min<int64_t>((lay.n[b] + 7) / 8, (int64_t)e->num_sms * 16);
      K.vit[b]<<<blocks, 256, 0, s>>>(recs, counts, bins, b, nullptr, nullptr, nullptr, flag, p->d_prof.p, nullptr,
                                      p->d_vfb.p, t->d_res.p, t->d_off.p, t->d_len.p, t->d_xsc.p, 0.f, scores);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(viterbi, scores, npairs * sizeof(float), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  } catch (const CudaError& ce) {
    return fail(ce.code, ce.msg);
  }
  return SX_OK;
}
