// Plain one-pair-per-block kernels: the straightforward GPU formulation the
// batched cascade is measured against.  One CTA of kPlainThreads threads per
// (profile, target) pair; thread t owns columns k = t+1, t+1+kPlainThreads, ...;
// the previous row is exchanged through shared memory with __syncthreads,
// row maxima are block reductions, the profile is read from a plain
// [row][M+1] layout in global memory.  Same arithmetic as the batched kernels
// (and the reference), so the scores are identical; only the organisation
// differs.
#pragma once
#include "kernels.cuh"

namespace sxk {

constexpr int kPlainThreads = 128;
constexpr int kPlainMaxCols = 16;  // columns per thread: M <= 2048

// plain image per profile: 25 msc rows then 8 log transitions
// (mm mi md im ii dm dd bm), each of length M+1 (index k).
struct PlainProfile {
  int64_t off;  // float offset
  int32_t m, pad;
};

__device__ __forceinline__ float block_max(float v, float* red) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  float r = red[0];
#pragma unroll
  for (int q = 1; q < kPlainThreads / 32; q++) r = fmaxf(r, red[q]);
  __syncthreads();
  return r;
}

// MSV (src/hmmer/dp.rs:92-145) for pairs p = first_p + blockIdx.x / nt, t = blockIdx.x % nt.
static __global__ void __launch_bounds__(kPlainThreads) plain_msv_kernel(
    int64_t first_pair, int nt, const PlainProfile* __restrict__ pprof, const float* __restrict__ pimg,
    const DevProfile* __restrict__ profs, const Thresholds* __restrict__ thr, const uint8_t* __restrict__ res,
    const int64_t* __restrict__ toff, const int32_t* __restrict__ tlen, const float4* __restrict__ tpar,
    PairRec* __restrict__ surv, const BinRegion* __restrict__ bins, unsigned* __restrict__ counts,
    unsigned* __restrict__ overflow) {
  __shared__ float row[2048 + 1];
  __shared__ float red[kPlainThreads / 32];
  const int64_t pair = first_pair + blockIdx.x;
  const int p = (int)(pair / nt), t = (int)(pair % nt);
  if (!thr[p].exact) return;
  const PlainProfile pp = pprof[p];
  const int M = pp.m;
  const float* msc = pimg + pp.off;
  const float tbm = profs[p].msv_tbm;
  const uint8_t* s = res + toff[t];
  const int L = tlen[t];
  const float4 tp = tpar[t];
  const float tloop = tp.x, tmove = tp.y, nullsc = tp.z;
  float prev[kPlainMaxCols];
#pragma unroll
  for (int q = 0; q < kPlainMaxCols; q++) prev[q] = SX_NEG_INF;
  float xn = 0.f, xb = tmove, xj = SX_NEG_INF, xc = SX_NEG_INF;
  for (int i = 0; i < L; i++) {
    const int x = s[i];
    // publish the previous row so column k can read k-1
#pragma unroll
    for (int q = 0; q < kPlainMaxCols; q++) {
      const int k = threadIdx.x + 1 + q * kPlainThreads;
      if (k <= M) row[k] = prev[q];
    }
    if (threadIdx.x == 0) row[0] = SX_NEG_INF;
    __syncthreads();
    const float be = fadd(xb, tbm);
    float xe = SX_NEG_INF;
#pragma unroll
    for (int q = 0; q < kPlainMaxCols; q++) {
      const int k = threadIdx.x + 1 + q * kPlainThreads;
      if (k <= M) {
        const float v = fadd(msc[x * (M + 1) + k], fmx(row[k - 1], be));
        prev[q] = v;
        xe = fmx(xe, v);
      }
    }
    xe = block_max(xe, red);  // also orders the row reads before the next row's writes
    xj = fmx(fadd(xj, tloop), fadd(xe, -kLn2));
    xc = fmx(fadd(xc, tloop), fadd(xe, -kLn2));
    xn = fadd(xn, tloop);
    xb = fmx(fadd(xn, tmove), fadd(xj, tmove));
  }
  if (threadIdx.x == 0) {
    const float usc = (L > 0 && M > 0) ? fadd(xc, tmove) : SX_NEG_INF;
    if (bits_stat(usc, nullsc) >= thr[p].s1) {
      PairRec r;
      r.p = p; r.t = t; r.usc = usc; r.filtersc = 0.f; r.vsc = 0.f; r.fwd = 0.f; r.slot = -1; r.pad = 0;
      push_pair(r, profs[p].vbin, surv, bins, counts, overflow);
    }
  }
}

// Viterbi (src/hmmer/dp.rs:152-189), one CTA per pair of the input list; the
// row's D chain is run serially by thread 0.
static __global__ void __launch_bounds__(kPlainThreads) plain_viterbi_kernel(
    const PairRec* __restrict__ in, const unsigned* __restrict__ in_counts, const BinRegion* __restrict__ in_bins,
    int bin, PairRec* __restrict__ out, const BinRegion* __restrict__ out_bins, unsigned* __restrict__ out_counts,
    unsigned* __restrict__ overflow, const PlainProfile* __restrict__ pprof, const float* __restrict__ pimg,
    const Thresholds* __restrict__ thr, const uint8_t* __restrict__ res, const int64_t* __restrict__ toff,
    const int32_t* __restrict__ tlen, const float4* __restrict__ xsc, float slack,
    const DevProfile* __restrict__ profs) {
  __shared__ float sm[2049], si[2049], sd[2049], mc[2049], dcur[2049];
  __shared__ float red[kPlainThreads / 32];
  const unsigned n = min(in_counts[bin], in_bins[bin].cap);
  for (unsigned w = blockIdx.x; w < n; w += gridDim.x) {
    PairRec r = in[in_bins[bin].off + w];
    const PlainProfile pp = pprof[r.p];
    const int M = pp.m, W = M + 1;
    const float* msc = pimg + pp.off;
    const float* tv = msc + 25 * W;  // mm mi md im ii dm dd bm
    const uint8_t* s = res + toff[r.t];
    const int L = tlen[r.t];
    const float4 xs = xsc[r.t];
    for (int k = threadIdx.x; k <= M; k += kPlainThreads) sm[k] = si[k] = sd[k] = SX_NEG_INF;
    __syncthreads();
    float xn = 0.f, xb = xs.y, xj = SX_NEG_INF, xc = SX_NEG_INF;
    for (int i = 0; i < L; i++) {
      const int x = s[i];
      const bool ins_ok = x != 24;
      float newi[kPlainMaxCols];
#pragma unroll
      for (int q = 0; q < kPlainMaxCols; q++) {
        const int k = threadIdx.x + 1 + q * kPlainThreads;
        newi[q] = SX_NEG_INF;
        if (k <= M) {
          const float sc = fmx(fmx(fadd(sm[k - 1], tv[0 * W + k - 1]), fadd(si[k - 1], tv[3 * W + k - 1])),
                               fmx(fadd(xb, tv[7 * W + k]), fadd(sd[k - 1], tv[5 * W + k - 1])));
          mc[k] = fadd(sc, msc[x * W + k]);
          if (k < M && ins_ok) newi[q] = fmx(fadd(sm[k], tv[1 * W + k]), fadd(si[k], tv[4 * W + k]));
        }
      }
      if (threadIdx.x == 0) mc[0] = SX_NEG_INF;
      __syncthreads();
      if (threadIdx.x == 0) {  // D chain, sequential in k
        float d = SX_NEG_INF;
        for (int k = 1; k <= M; k++) {
          d = fmx(fadd(mc[k - 1], tv[2 * W + k - 1]), fadd(d, tv[6 * W + k - 1]));
          dcur[k] = d;
        }
      }
      __syncthreads();
      float xe = SX_NEG_INF;
#pragma unroll
      for (int q = 0; q < kPlainMaxCols; q++) {
        const int k = threadIdx.x + 1 + q * kPlainThreads;
        if (k <= M) {
          xe = fmx(xe, fmx(mc[k], dcur[k]));
          sm[k] = mc[k];
          si[k] = newi[q];
          sd[k] = dcur[k];
        }
      }
      xe = block_max(xe, red);
      xj = fmx(fadd(xj, xs.x), fadd(xe, -kLn2));
      xc = fmx(fadd(xc, xs.x), fadd(xe, -kLn2));
      xn = fadd(xn, xs.x);
      xb = fmx(fadd(xn, xs.y), fadd(xj, xs.y));
    }
    if (threadIdx.x == 0) {
      r.vsc = (L > 0 && M > 0) ? fadd(xc, xs.y) : SX_NEG_INF;
      if (bits_stat(r.vsc, r.filtersc) >= thr[r.p].s2 - slack)
        push_pair(r, profs[r.p].vbin, out, out_bins, out_counts, overflow);
    }
    __syncthreads();
  }
}

}  // namespace sxk
