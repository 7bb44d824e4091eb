// Profiles longer than the warp-chunked kernels' 32 x 64 = 2048 columns
// (marker models of long proteins).  One CTA of kPlainThreads threads per
// (profile, target) pair; thread t owns columns k = t+1, t+1+kPlainThreads, ...;
// the rows live in a per-CTA slice of global scratch (L1/L2 resident), and the
// sequential parts of a row (the Viterbi and Forward/Backward D chains, the
// Forward row sum and the Backward B sum) are run in order by thread 0.  The
// arithmetic is the reference's, operation for operation, as in the
// warp-chunked kernels, so the scores and raw rows are identical.
//
// Profile image (the plain layout extended): rows of M+1 floats indexed by k,
//   0..24  msc[x][k]       25..32 log transitions  mm mi md im ii dm dd bm
//   33..57 mo[x][k]        58..65 probabilities    mm mi md im ii dm dd bm
#pragma once
#include "plain.cuh"

namespace sxk {

constexpr int kLongRows = 66;
enum { kLT = 25, kLMo = 33, kLP = 58 };  // first rows of log transitions, odds, probabilities
enum { kQMM = 0, kQMI, kQMD, kQIM, kQII, kQDM, kQDD, kQBM };
constexpr int kLongArrays = 6;  // scratch rows of M+1 floats per CTA

struct LongPair {
  int32_t p, t;
};

// MSV (src/hmmer/dp.rs:92-145): score of every pair.
static __global__ void __launch_bounds__(kPlainThreads) long_msv_kernel(
    const LongPair* __restrict__ pairs, int n, const PlainProfile* __restrict__ pprof, const float* __restrict__ pimg,
    const DevProfile* __restrict__ profs, const uint8_t* __restrict__ res, const int64_t* __restrict__ toff,
    const int32_t* __restrict__ tlen, const float4* __restrict__ tpar, float* __restrict__ scratch, int64_t stride,
    float* __restrict__ out) {
  __shared__ float red[kPlainThreads / 32];
  float* A = scratch + (int64_t)blockIdx.x * stride;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const LongPair q = pairs[w];
    const PlainProfile pp = pprof[q.p];
    const int M = pp.m, W = M + 1;
    const float* img = pimg + pp.off;
    const float tbm = profs[q.p].msv_tbm;
    const uint8_t* s = res + toff[q.t];
    const int L = tlen[q.t];
    const float4 tp = tpar[q.t];
    const float tloop = tp.x, tmove = tp.y;
    float* prev = A;
    float* cur = A + W;
    for (int k = threadIdx.x; k <= M; k += kPlainThreads) prev[k] = cur[k] = SX_NEG_INF;
    __syncthreads();
    float xn = 0.f, xb = tmove, xj = SX_NEG_INF, xc = SX_NEG_INF;
    for (int i = 0; i < L; i++) {
      const float* e = img + (int64_t)__ldg(s + i) * W;
      const float be = fadd(xb, tbm);
      float xe = SX_NEG_INF;
      for (int k = threadIdx.x + 1; k <= M; k += kPlainThreads) {
        const float v = fadd(__ldg(e + k), fmx(prev[k - 1], be));
        cur[k] = v;
        xe = fmx(xe, v);
      }
      xe = block_max(xe, red);  // also orders this row's writes before the next row's reads
      xj = fmx(fadd(xj, tloop), fadd(xe, -kLn2));
      xc = fmx(fadd(xc, tloop), fadd(xe, -kLn2));
      xn = fadd(xn, tloop);
      xb = fmx(fadd(xn, tmove), fadd(xj, tmove));
      float* t = prev;
      prev = cur;
      cur = t;
    }
    if (threadIdx.x == 0) out[w] = (L > 0 && M > 0) ? fadd(xc, tmove) : SX_NEG_INF;
    __syncthreads();
  }
}

// Viterbi filter (src/hmmer/dp.rs:152-189): score of every pair.
static __global__ void __launch_bounds__(kPlainThreads) long_viterbi_kernel(
    const LongPair* __restrict__ pairs, int n, const PlainProfile* __restrict__ pprof, const float* __restrict__ pimg,
    const uint8_t* __restrict__ res, const int64_t* __restrict__ toff, const int32_t* __restrict__ tlen,
    const float4* __restrict__ xsc, float* __restrict__ scratch, int64_t stride, float* __restrict__ out) {
  __shared__ float red[kPlainThreads / 32];
  float* A = scratch + (int64_t)blockIdx.x * stride;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const LongPair q = pairs[w];
    const PlainProfile pp = pprof[q.p];
    const int M = pp.m, W = M + 1;
    const float* img = pimg + pp.off;
    const float* tv = img + kLT * W;
    const uint8_t* s = res + toff[q.t];
    const int L = tlen[q.t];
    const float4 xs = xsc[q.t];
    float *sm = A, *si = A + W, *sd = A + 2 * W, *mc = A + 3 * W, *ni = A + 4 * W, *dc = A + 5 * W;
    for (int k = threadIdx.x; k <= M; k += kPlainThreads) sm[k] = si[k] = sd[k] = mc[k] = ni[k] = dc[k] = SX_NEG_INF;
    __syncthreads();
    float xn = 0.f, xb = xs.y, xj = SX_NEG_INF, xc = SX_NEG_INF;
    for (int i = 0; i < L; i++) {
      const int x = __ldg(s + i);
      const bool ins_ok = x != 24;
      const float* e = img + (int64_t)x * W;
      for (int k = threadIdx.x + 1; k <= M; k += kPlainThreads) {
        const float sc = fmx(fmx(fadd(sm[k - 1], __ldg(tv + kQMM * W + k - 1)), fadd(si[k - 1], __ldg(tv + kQIM * W + k - 1))),
                             fmx(fadd(xb, __ldg(tv + kQBM * W + k)), fadd(sd[k - 1], __ldg(tv + kQDM * W + k - 1))));
        mc[k] = fadd(sc, __ldg(e + k));
        ni[k] = (k < M && ins_ok) ? fmx(fadd(sm[k], __ldg(tv + kQMI * W + k)), fadd(si[k], __ldg(tv + kQII * W + k)))
                                  : SX_NEG_INF;
      }
      __syncthreads();
      if (threadIdx.x == 0) {  // D chain, sequential in k
        float d = SX_NEG_INF;
        for (int k = 1; k <= M; k++) {
          d = fmx(fadd(mc[k - 1], __ldg(tv + kQMD * W + k - 1)), fadd(d, __ldg(tv + kQDD * W + k - 1)));
          dc[k] = d;
        }
      }
      __syncthreads();
      float xe = SX_NEG_INF;
      for (int k = threadIdx.x + 1; k <= M; k += kPlainThreads) {
        xe = fmx(xe, fmx(mc[k], dc[k]));
        sm[k] = mc[k];
        si[k] = ni[k];
        sd[k] = dc[k];
      }
      xe = block_max(xe, red);
      xj = fmx(fadd(xj, xs.x), fadd(xe, -kLn2));
      xc = fmx(fadd(xc, xs.x), fadd(xe, -kLn2));
      xn = fadd(xn, xs.x);
      xb = fmx(fadd(xn, xs.y), fadd(xj, xs.y));
    }
    if (threadIdx.x == 0) out[w] = (L > 0 && M > 0) ? fadd(xc, xs.y) : SX_NEG_INF;
    __syncthreads();
  }
}

// Forward (src/hmmer/dp.rs:229-298) then Backward (dp.rs:301-392) of every
// pair, multihit, writing the raw special rows exactly as forward_kernel and
// backward_kernel do: fwd rows 1..L (N B E J C, rescale factor or 0); bwd
// row L (E, C), rows L-1..1 (N B E J C, factor) and the B sum in slot 1 of row 0.
static __global__ void __launch_bounds__(kPlainThreads) long_rows_kernel(
    const LongPair* __restrict__ pairs, int n, const PlainProfile* __restrict__ pprof, const float* __restrict__ pimg,
    const uint8_t* __restrict__ res, const int64_t* __restrict__ toff, const int32_t* __restrict__ tlen,
    const float4* __restrict__ xsc, float* __restrict__ scratch, int64_t stride, float* __restrict__ rows_f,
    float* __restrict__ rows_b, const int64_t* __restrict__ row_off) {
  __shared__ float red[kPlainThreads / 32];
  __shared__ float sx[6];
  float* A = scratch + (int64_t)blockIdx.x * stride;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const LongPair q = pairs[w];
    const PlainProfile pp = pprof[q.p];
    const int M = pp.m, W = M + 1;
    const float* img = pimg + pp.off;
    const float* pv = img + kLP * W;  // probabilities mm mi md im ii dm dd bm
    auto P = [&](int r, int k) { return __ldg(pv + r * W + k); };
    const uint8_t* s = res + toff[q.t];
    const int L = tlen[q.t];
    const float4 xs = xsc[q.t];
    const float ploop = xs.z, pmove = xs.w;
    float* fo = rows_f + row_off[w];
    float* bo = rows_b + row_off[w];
    // ---- Forward
    float *mp = A, *ip = A + W, *dp = A + 2 * W, *mc = A + 3 * W, *ic = A + 4 * W, *dc = A + 5 * W;
    for (int k = threadIdx.x; k <= M; k += kPlainThreads) mp[k] = ip[k] = dp[k] = mc[k] = ic[k] = dc[k] = 0.f;
    __syncthreads();
    float xn = 1.f, xb = pmove, xj = 0.f, xc = 0.f;
    for (int i = 0; i < L; i++) {
      const int x = __ldg(s + i);
      const float ins = x != 24 ? 1.f : 0.f;
      const float* eo = img + (int64_t)(kLMo + x) * W;
      for (int k = threadIdx.x + 1; k <= M; k += kPlainThreads) {
        float t = fmul(xb, P(kQBM, k));
        t = fadd(t, fmul(mp[k - 1], P(kQMM, k - 1)));
        t = fadd(t, fmul(ip[k - 1], P(kQIM, k - 1)));
        t = fadd(t, fmul(dp[k - 1], P(kQDM, k - 1)));
        mc[k] = fmul(t, __ldg(eo + k));
        ic[k] = k < M ? fmul(fadd(fmul(mp[k], P(kQMI, k)), fmul(ip[k], P(kQII, k))), ins) : 0.f;
      }
      __syncthreads();
      if (threadIdx.x == 0) {  // D chain and row sum, in order of k
        float dcar = 0.f, xe = 0.f;
        for (int k = 1; k <= M; k++) {
          const float d = fadd(fmul(mc[k - 1], P(kQMD, k - 1)), fmul(dcar, P(kQDD, k - 1)));
          dc[k] = d;
          xe = fadd(xe, fadd(mc[k], d));
          dcar = d;
        }
        sx[0] = xe;
      }
      __syncthreads();
      float xe = sx[0];
      xj = fadd(fmul(xj, ploop), fmul(xe, 0.5f));
      xc = fadd(fmul(xc, ploop), fmul(xe, 0.5f));
      xn = fmul(xn, ploop);
      xb = fadd(fmul(xn, pmove), fmul(xj, pmove));
      float scale = 0.f;
      if (xe > 1.0e4f) {
        const float inv = __fdiv_rn(1.0f, xe);
        for (int k = threadIdx.x + 1; k <= M; k += kPlainThreads) {
          mc[k] = fmul(mc[k], inv);
          ic[k] = fmul(ic[k], inv);
          dc[k] = fmul(dc[k], inv);
        }
        xn = fmul(xn, inv);
        xb = fmul(xb, inv);
        xj = fmul(xj, inv);
        xc = fmul(xc, inv);
        scale = xe;
        xe = 1.0f;
      }
      if (threadIdx.x == 0) {
        float* o = fo + 6 * (int64_t)(i + 1);
        o[0] = xn; o[1] = xb; o[2] = xe; o[3] = xj; o[4] = xc; o[5] = scale;
      }
      __syncthreads();
      float* t;
      t = mp; mp = mc; mc = t;
      t = ip; ip = ic; ic = t;
      t = dp; dp = dc; dc = t;
    }
    __syncthreads();
    // ---- Backward: mn/in hold row i+1, me = mn*eo and bt = B terms of row i
    float *mn = A, *in_ = A + W, *me = A + 2 * W, *bt = A + 3 * W, *ivv = A + 4 * W, *dd = A + 5 * W;
    xc = pmove;
    float xe = fmul(xc, 0.5f);
    xj = 0.f;
    xn = 0.f;
    for (int k = threadIdx.x; k <= M; k += kPlainThreads) in_[k] = 0.f;
    if (threadIdx.x == 0 && M > 0) {  // row L: M and D from the E state, descending
      mn[M] = dd[M] = xe;
      float dcar = xe;
      for (int k = M - 1; k >= 1; k--) {
        mn[k] = fadd(xe, fmul(dcar, P(kQMD, k)));
        dd[k] = fadd(xe, fmul(dcar, P(kQDD, k)));
        dcar = dd[k];
      }
      mn[0] = 0.f;
    }
    if (threadIdx.x == 0 && L > 0) {
      float* o = bo + 6 * (int64_t)L;
      o[0] = 0.f; o[1] = 0.f; o[2] = xe; o[3] = 0.f; o[4] = xc; o[5] = 0.f;
    }
    __syncthreads();
    for (int i = L - 1; i >= 1; i--) {
      const int x = __ldg(s + i);
      const float ins = x != 24 ? 1.f : 0.f;
      const float* eo = img + (int64_t)(kLMo + x) * W;
      for (int k = threadIdx.x + 1; k <= M; k += kPlainThreads) {
        const float e = __ldg(eo + k);
        me[k] = fmul(mn[k], e);
        bt[k] = fmul(fmul(mn[k], P(kQBM, k)), e);
        ivv[k] = fmul(in_[k], ins);
      }
      __syncthreads();
      if (threadIdx.x == 0) {  // B sum ascending, specials, D chain descending
        float b = 0.f;
        for (int k = 1; k <= M; k++) b = fadd(b, bt[k]);
        const float xb0 = b;
        xj = fadd(fmul(xj, ploop), fmul(xb0, pmove));
        xc = fmul(xc, ploop);
        xe = fadd(fmul(xj, 0.5f), fmul(xc, 0.5f));
        xn = fadd(fmul(xn, ploop), fmul(xb0, pmove));
        if (M > 0) {
          dd[M] = xe;
          float dcar = xe;
          for (int k = M - 1; k >= 1; k--) {
            dd[k] = fadd(fadd(fmul(me[k + 1], P(kQDM, k)), fmul(dcar, P(kQDD, k))), xe);
            dcar = dd[k];
          }
        }
        sx[0] = xb0; sx[1] = xe; sx[2] = xn; sx[3] = xj; sx[4] = xc;
      }
      __syncthreads();
      const float xb0 = sx[0];
      xe = sx[1]; xn = sx[2]; xj = sx[3]; xc = sx[4];
      // M and I of row i in place of row i+1 (each k reads me/ivv/dd, not mn/in_)
      float rowmax = fmaxf(fmaxf(fmaxf(fmaxf(xb0, xe), xn), xj), xc);
      for (int k = threadIdx.x + 1; k <= M; k += kPlainThreads) {
        if (k < M) {
          const float mv = fadd(fadd(fadd(fmul(me[k + 1], P(kQMM, k)), fmul(ivv[k], P(kQMI, k))), xe),
                                fmul(dd[k + 1], P(kQMD, k)));
          mn[k] = mv;
          in_[k] = fadd(fmul(me[k + 1], P(kQIM, k)), fmul(ivv[k], P(kQII, k)));
          rowmax = fmaxf(rowmax, mv);
        } else {
          mn[k] = xe;
          in_[k] = 0.f;
        }
      }
      rowmax = block_max(rowmax, red);
      float scale = 0.f, xb_o = xb0;
      if (rowmax > 1.0e4f) {
        const float inv = __fdiv_rn(1.0f, rowmax);
        for (int k = threadIdx.x + 1; k <= M; k += kPlainThreads) {
          mn[k] = fmul(mn[k], inv);
          in_[k] = fmul(in_[k], inv);
        }
        xb_o = fmul(xb0, inv);
        xe = fmul(xe, inv);
        xn = fmul(xn, inv);
        xj = fmul(xj, inv);
        xc = fmul(xc, inv);
        scale = rowmax;
      }
      if (threadIdx.x == 0) {
        float* o = bo + 6 * (int64_t)i;
        o[0] = xn; o[1] = xb_o; o[2] = xe; o[3] = xj; o[4] = xc; o[5] = scale;
      }
      __syncthreads();
    }
    if (L > 0) {  // row 0: B sum with residue 1
      const float* eo = img + (int64_t)(kLMo + __ldg(s)) * W;
      for (int k = threadIdx.x + 1; k <= M; k += kPlainThreads) bt[k] = fmul(fmul(mn[k], P(kQBM, k)), __ldg(eo + k));
      __syncthreads();
      if (threadIdx.x == 0) {
        float b = 0.f;
        for (int k = 1; k <= M; k++) b = fadd(b, bt[k]);
        bo[0] = 0.f; bo[1] = b; bo[2] = 0.f; bo[3] = 0.f; bo[4] = 0.f; bo[5] = 0.f;
      }
    }
    __syncthreads();
  }
}

}  // namespace sxk
