// Envelope rescoring on the device: the full-matrix passes of
// rescore_isolated_domain (src/hmmer/pipeline.rs:545-591) for a batch of
// envelopes, one warp per envelope.
//
//   env_forward_kernel   forward_matrix  (src/hmmer/dp.rs:442-513)
//   env_backward_kernel  backward_matrix (src/hmmer/dp.rs:516-601)
//   env_post_kernel      decode (dp.rs:1278-1306) fused with the sums of
//                        null2_from_posterior (dp.rs:1310-1350) and the
//                        optimal-accuracy DP and traceback (dp.rs:1355-1564)
//
// The arithmetic is the reference's, operation for operation (no FMA, the D
// chains and row sums in order by lane batons), so the matrices, posteriors
// and coordinates equal the host's bit for bit.  Every log/exp stays on the
// host: the forward and backward kernels write raw scaled special rows and
// rescale factors, the host turns them into the per-row posterior factor
// exp(lnF + lnB - lnZ) and the N/J/C posteriors, and the post kernel reads
// those back.
#pragma once
#include "kernels.cuh"

namespace sxk {

// One envelope: residues i0 .. i0+lr-1 (0-based) of target t against profile p,
// with the unihit special transitions of the whole target's length.
struct EnvRec {
  int32_t p, t;
  int32_t i0, lr;
  float ploop, pmove, pe_loop, pe_move;
  int64_t plane_off;  // float offset: 5 planes of (lr+1) rows x 32*VC columns (FM FI BM BI OD)
  int64_t row_off;    // float offset: forward raw rows 6(lr+1), then backward raw rows 6(lr+1)
  int64_t aux_off;    // float offset: pn pj pc (inputs), then OA specials xe xn xj xb xc; (lr+1) each
  int64_t fac_off;    // double offset: posterior factor per row (lr+1)
  int64_t out_off;    // float offset of kEnvOut outputs
};
// Outputs: [0,20) sum_k (sm[k]*norm)*mo[x][k] for x < 20, [20] si (the row-major
// sum of insert posteriors), [21] found (1/0), [22..25] i0 i1 k0 k1 (as floats).
constexpr int kEnvOut = 32;

// Plane element of column k (1-based) in the lane-major layout: lane (k-1)/VC,
// chunk slot (k-1)%VC.
template <int VC>
__device__ __forceinline__ int64_t plane_at(int64_t row, int k) {
  return row * (32 * VC) + (int64_t)(((k - 1) % VC) * 32 + (k - 1) / VC);
}

// forward_matrix: M/I planes (scaled, after each row's rescaling) and the raw
// special rows N B E J C scale for rows 1..lr.
template <int VC>
__global__ void __launch_bounds__(32) env_forward_kernel(const EnvRec* __restrict__ recs, int n,
                                                         const DevProfile* __restrict__ profs,
                                                         const float* __restrict__ vfb,
                                                         const uint8_t* __restrict__ res,
                                                         const int64_t* __restrict__ toff, float* __restrict__ planes,
                                                         float* __restrict__ rows) {
  constexpr int RS = 32 * VC;
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += warps) {
    const EnvRec r = recs[w];
    const DevProfile P = profs[r.p];
    const Img<VC> img{vfb + P.vfb_off};
    const int M = P.m;
    const int nl = (M + VC - 1) / VC;
    const uint8_t* s = res + toff[r.t] + r.i0;
    const int L = r.lr;
    const float ploop = r.ploop, pmove = r.pmove, pe_loop = r.pe_loop, pe_move = r.pe_move;
    float* FM = planes + r.plane_off;
    float* FI = FM + (int64_t)(L + 1) * RS;
    float* orow = rows + r.row_off;
    TransRows<VC> tr;
    tr.load(img, kRowFwd, lane);
    float mp[VC], ip[VC], dp[VC], eo[VC];
#pragma unroll
    for (int c = 0; c < VC; c++) mp[c] = ip[c] = dp[c] = 0.f;
    float xn = 1.f, xb = pmove, xj = 0.f, xc = 0.f;
    int x = L > 0 ? __ldg(s) : 24;
#pragma unroll
    for (int c = 0; c < VC; c++) eo[c] = img.at(kRowMo + x, c, lane);
    for (int i = 0; i < L; i++) {
      const int xnext = (i + 1 < L) ? __ldg(s + i + 1) : 24;
      float eon[VC];
#pragma unroll
      for (int c = 0; c < VC; c++) eon[c] = img.at(kRowMo + xnext, c, lane);
      const float ins = x != 24 ? 1.f : 0.f;
      const float mpl0 = __shfl_up_sync(kFull, mp[VC - 1], 1);
      const float ipl0 = __shfl_up_sync(kFull, ip[VC - 1], 1);
      const float dpl0 = __shfl_up_sync(kFull, dp[VC - 1], 1);
      const float mpl = lane ? mpl0 : 0.f, ipl = lane ? ipl0 : 0.f, dpl = lane ? dpl0 : 0.f;
      float mv[VC], iv[VC], a[VC], dv[VC], pdd[VC];
#pragma unroll
      for (int c = 0; c < VC; c++) {
        const int k = lane * VC + c + 1;
        const float mpv = c ? mp[c - 1] : mpl, ipv = c ? ip[c - 1] : ipl, dpv = c ? dp[c - 1] : dpl;
        float t = fmul(xb, tr.get(img, kRowFwd, 0, c, lane));
        t = fadd(t, fmul(mpv, tr.get(img, kRowFwd, 1, c, lane)));
        t = fadd(t, fmul(ipv, tr.get(img, kRowFwd, 2, c, lane)));
        t = fadd(t, fmul(dpv, tr.get(img, kRowFwd, 3, c, lane)));
        mv[c] = fmul(t, eo[c]);
        iv[c] = k < M ? fmul(fadd(fmul(mp[c], tr.get(img, kRowFwd, 4, c, lane)),
                                  fmul(ip[c], tr.get(img, kRowFwd, 5, c, lane))), ins)
                      : 0.f;
      }
      const float mcl0 = __shfl_up_sync(kFull, mv[VC - 1], 1);
      const float mcl = lane ? mcl0 : 0.f;
#pragma unroll
      for (int c = 0; c < VC; c++) {
        a[c] = fmul(c ? mv[c - 1] : mcl, tr.get(img, kRowFwd, 6, c, lane));
        pdd[c] = tr.get(img, kRowFwd, 7, c, lane);
      }
      // ordered D chain and row sum: dc[k] = a_k + dc[k-1]*p_dd[k-1]; xe += mv + dc
      float dcar = 0.f, xe = 0.f;
      for (int sl = 0; sl < nl; sl++) {
        if (lane == sl) {
#pragma unroll
          for (int c = 0; c < VC; c++) {
            const float d = fadd(a[c], fmul(dcar, pdd[c]));
            dv[c] = d;
            xe = fadd(xe, fadd(mv[c], d));
            dcar = d;
          }
        }
        dcar = __shfl_sync(kFull, dcar, sl);
        xe = __shfl_sync(kFull, xe, sl);
      }
      if (lane >= nl) {
#pragma unroll
        for (int c = 0; c < VC; c++) dv[c] = 0.f;
      }
      xj = fadd(fmul(xj, ploop), fmul(xe, pe_loop));
      xc = fadd(fmul(xc, ploop), fmul(xe, pe_move));
      xn = fmul(xn, ploop);
      xb = fadd(fmul(xn, pmove), fmul(xj, pmove));
      float scale = 0.f;
      if (xe > 1.0e4f) {
        const float inv = __fdiv_rn(1.0f, xe);
#pragma unroll
        for (int c = 0; c < VC; c++) {
          mv[c] = fmul(mv[c], inv);
          iv[c] = fmul(iv[c], inv);
          dv[c] = fmul(dv[c], inv);
        }
        xn = fmul(xn, inv);
        xb = fmul(xb, inv);
        xj = fmul(xj, inv);
        xc = fmul(xc, inv);
        scale = xe;
        xe = 1.0f;
      }
      if (lane == 0) {
        float* o = orow + 6 * (i + 1);
        o[0] = xn; o[1] = xb; o[2] = xe; o[3] = xj; o[4] = xc; o[5] = scale;
      }
#pragma unroll
      for (int c = 0; c < VC; c++) {
        FM[(int64_t)(i + 1) * RS + c * 32 + lane] = mv[c];
        FI[(int64_t)(i + 1) * RS + c * 32 + lane] = iv[c];
        mp[c] = mv[c];
        ip[c] = iv[c];
        dp[c] = dv[c];
        eo[c] = eon[c];
      }
      x = xnext;
    }
  }
}

// backward_matrix: M/I planes for rows lr..1 and the raw special rows (row lr:
// E and C; rows lr-1..1: N B E J C scale; row 0: the B sum in slot 1).
template <int VC>
__global__ void __launch_bounds__(32) env_backward_kernel(const EnvRec* __restrict__ recs, int n,
                                                          const DevProfile* __restrict__ profs,
                                                          const float* __restrict__ vfb,
                                                          const uint8_t* __restrict__ res,
                                                          const int64_t* __restrict__ toff, float* __restrict__ planes,
                                                          float* __restrict__ rows) {
  constexpr int RS = 32 * VC;
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += warps) {
    const EnvRec r = recs[w];
    const DevProfile P = profs[r.p];
    const Img<VC> img{vfb + P.vfb_off};
    const int M = P.m;
    const int nl = (M + VC - 1) / VC;
    const int lM = (M - 1) / VC;  // lane holding column M
    const uint8_t* s = res + toff[r.t] + r.i0;
    const int L = r.lr;
    const float ploop = r.ploop, pmove = r.pmove, pe_loop = r.pe_loop, pe_move = r.pe_move;
    float* BM = planes + r.plane_off + 2 * (int64_t)(L + 1) * RS;
    float* BI = BM + (int64_t)(L + 1) * RS;
    float* orow = rows + r.row_off + 6 * (int64_t)(L + 1);
    float mn[VC], in_[VC], dn[VC];
    // row L
    float xc = pmove;
    float xe = fmul(xc, pe_move);
    float xj = 0.f, xn = 0.f;
    {
      float pmd0[VC], pdd0[VC];
#pragma unroll
      for (int c = 0; c < VC; c++) {
        pmd0[c] = img.at(kRowBwd + 2, c, lane);
        pdd0[c] = img.at(kRowBwd + 6, c, lane);
      }
      float dcar = 0.f;
      for (int sl = lM; sl >= 0; sl--) {
        if (lane == sl) {
#pragma unroll
          for (int c = VC - 1; c >= 0; c--) {
            const int k = lane * VC + c + 1;
            if (k > M) {
              mn[c] = dn[c] = 0.f;
            } else if (k == M) {
              mn[c] = dn[c] = xe;
              dcar = xe;
            } else {
              mn[c] = fadd(xe, fmul(dcar, pmd0[c]));
              dn[c] = fadd(xe, fmul(dcar, pdd0[c]));
              dcar = dn[c];
            }
          }
        }
        dcar = __shfl_sync(kFull, dcar, sl);
      }
      if (lane > lM) {
#pragma unroll
        for (int c = 0; c < VC; c++) mn[c] = dn[c] = 0.f;
      }
#pragma unroll
      for (int c = 0; c < VC; c++) in_[c] = 0.f;
    }
    if (L > 0) {
#pragma unroll
      for (int c = 0; c < VC; c++) {
        BM[(int64_t)L * RS + c * 32 + lane] = mn[c];
        BI[(int64_t)L * RS + c * 32 + lane] = 0.f;
      }
    }
    if (lane == 0 && L > 0) {
      float* o = orow + 6 * L;
      o[0] = 0.f; o[1] = 0.f; o[2] = xe; o[3] = 0.f; o[4] = xc; o[5] = 0.f;
    }
    for (int i = L - 1; i >= 1; i--) {
      const int x = __ldg(s + i);
      const float ins = x != 24 ? 1.f : 0.f;
      float eo[VC], me[VC], bt[VC];
#pragma unroll
      for (int c = 0; c < VC; c++) {
        eo[c] = img.at(kRowMo + x, c, lane);
        me[c] = fmul(mn[c], eo[c]);
        bt[c] = fmul(fmul(mn[c], img.at(kRowBwd + 7, c, lane)), eo[c]);
      }
      // B sum, ascending k
      float b = 0.f;
      for (int sl = 0; sl < nl; sl++) {
        if (lane == sl) {
#pragma unroll
          for (int c = 0; c < VC; c++) b = fadd(b, bt[c]);
        }
        b = __shfl_sync(kFull, b, sl);
      }
      const float xb = b;
      xj = fadd(fmul(xj, ploop), fmul(xb, pmove));
      xc = fmul(xc, ploop);
      xe = fadd(fmul(xj, pe_loop), fmul(xc, pe_move));
      xn = fadd(fmul(xn, ploop), fmul(xb, pmove));
      float rowmax = fmaxf(fmaxf(fmaxf(fmaxf(xb, xe), xn), xj), xc);
      const float me_up = __shfl_down_sync(kFull, me[0], 1);
      float mnext[VC], iv[VC], mc[VC], ic[VC], dc[VC];
#pragma unroll
      for (int c = 0; c < VC; c++) {
        mnext[c] = c < VC - 1 ? me[c + 1] : (lane < 31 ? me_up : 0.f);
        iv[c] = fmul(in_[c], ins);
      }
      float pdm[VC], pdd[VC];
#pragma unroll
      for (int c = 0; c < VC; c++) {
        pdm[c] = img.at(kRowBwd + 5, c, lane);
        pdd[c] = img.at(kRowBwd + 6, c, lane);
      }
      // D chain, descending k
      float dcar = 0.f;
      for (int sl = lM; sl >= 0; sl--) {
        if (lane == sl) {
#pragma unroll
          for (int c = VC - 1; c >= 0; c--) {
            const int k = lane * VC + c + 1;
            if (k > M) {
              dc[c] = 0.f;
            } else if (k == M) {
              dc[c] = xe;
              dcar = xe;
            } else {
              dc[c] = fadd(fadd(fmul(mnext[c], pdm[c]), fmul(dcar, pdd[c])), xe);
              dcar = dc[c];
            }
          }
        }
        dcar = __shfl_sync(kFull, dcar, sl);
      }
      if (lane > lM) {
#pragma unroll
        for (int c = 0; c < VC; c++) dc[c] = 0.f;
      }
      const float dc_up = __shfl_down_sync(kFull, dc[0], 1);
#pragma unroll
      for (int c = 0; c < VC; c++) {
        const int k = lane * VC + c + 1;
        const float dnext = c < VC - 1 ? dc[c + 1] : (lane < 31 ? dc_up : 0.f);
        if (k < M) {
          const float mv = fadd(fadd(fadd(fmul(mnext[c], img.at(kRowBwd + 0, c, lane)),
                                          fmul(iv[c], img.at(kRowBwd + 1, c, lane))), xe),
                                fmul(dnext, img.at(kRowBwd + 2, c, lane)));
          mc[c] = mv;
          ic[c] = fadd(fmul(mnext[c], img.at(kRowBwd + 3, c, lane)), fmul(iv[c], img.at(kRowBwd + 4, c, lane)));
          rowmax = fmaxf(rowmax, mv);
        } else if (k == M) {
          mc[c] = xe;
          ic[c] = 0.f;
        } else {
          mc[c] = 0.f;
          ic[c] = 0.f;
        }
      }
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) rowmax = fmaxf(rowmax, __shfl_xor_sync(kFull, rowmax, o));
      float scale = 0.f;
      float xb_o = xb;
      if (rowmax > 1.0e4f) {
        const float inv = __fdiv_rn(1.0f, rowmax);
#pragma unroll
        for (int c = 0; c < VC; c++) {
          mc[c] = fmul(mc[c], inv);
          ic[c] = fmul(ic[c], inv);
          dc[c] = fmul(dc[c], inv);
        }
        xb_o = fmul(xb, inv);
        xe = fmul(xe, inv);
        xn = fmul(xn, inv);
        xj = fmul(xj, inv);
        xc = fmul(xc, inv);
        scale = rowmax;
      }
      if (lane == 0) {
        float* o = orow + 6 * i;
        o[0] = xn; o[1] = xb_o; o[2] = xe; o[3] = xj; o[4] = xc; o[5] = scale;
      }
#pragma unroll
      for (int c = 0; c < VC; c++) {
        BM[(int64_t)i * RS + c * 32 + lane] = mc[c];
        BI[(int64_t)i * RS + c * 32 + lane] = ic[c];
        mn[c] = mc[c];
        in_[c] = ic[c];
        dn[c] = dc[c];
      }
    }
    // row 0: B sum with residue 1
    if (L > 0) {
      const int x0 = __ldg(s);
      float bt[VC];
#pragma unroll
      for (int c = 0; c < VC; c++) bt[c] = fmul(fmul(mn[c], img.at(kRowBwd + 7, c, lane)), img.at(kRowMo + x0, c, lane));
      float b = 0.f;
      for (int sl = 0; sl < nl; sl++) {
        if (lane == sl) {
#pragma unroll
          for (int c = 0; c < VC; c++) b = fadd(b, bt[c]);
        }
        b = __shfl_sync(kFull, b, sl);
      }
      if (lane == 0) {
        float* o = orow;
        o[0] = 0.f; o[1] = b; o[2] = 0.f; o[3] = 0.f; o[4] = 0.f; o[5] = 0.f;
      }
    }
  }
}

__device__ __forceinline__ float oa_gate(float t, float v) { return t > 0.0f ? v : 0.0f; }
__device__ __forceinline__ float oa_dis(float t, float v) { return t == 0.0f ? SX_NEG_INF : v; }

// decode + null2 sums + optimal-accuracy DP and traceback.  Reads the forward
// and backward M/I planes, the host's per-row factor exp(lnF + lnB - lnZ) and
// N/J/C posteriors; overwrites the backward planes with the OA M/I matrices
// (each backward row is read before its OA row is written) and fills the OD
// plane and the OA special arrays, which the traceback (lane 0) reads.
template <int VC>
__global__ void __launch_bounds__(32) env_post_kernel(const EnvRec* __restrict__ recs, int n,
                                                      const DevProfile* __restrict__ profs,
                                                      const float* __restrict__ vfb, float* __restrict__ planes,
                                                      float* __restrict__ aux, const double* __restrict__ facs,
                                                      float* __restrict__ outs) {
  constexpr int RS = 32 * VC;
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += warps) {
    const EnvRec r = recs[w];
    const DevProfile P = profs[r.p];
    const Img<VC> img{vfb + P.vfb_off};
    const int M = P.m;
    const int nl = (M + VC - 1) / VC;
    const int L = r.lr;
    const int64_t PL = (int64_t)(L + 1) * RS;
    const float* FM = planes + r.plane_off;
    const float* FI = FM + PL;
    float* OM = planes + r.plane_off + 2 * PL;  // backward M, then OA M
    float* OI = OM + PL;                        // backward I, then OA I
    float* OD = OI + PL;
    float* ab = aux + r.aux_off;
    const float* pn = ab;
    const float* pj = ab + (L + 1);
    const float* pc = ab + 2 * (L + 1);
    float* sxe = ab + 3 * (L + 1);
    float* sxn = sxe + (L + 1);
    float* sxj = sxn + (L + 1);
    float* sxb = sxj + (L + 1);
    float* sxc = sxb + (L + 1);
    const double* fac = facs + r.fac_off;
    float* out = outs + r.out_off;
    const bool ploop0 = r.ploop == 0.0f, pe_loop0 = r.pe_loop == 0.0f, pe_move0 = r.pe_move == 0.0f,
               pmove0 = r.pmove == 0.0f;
    // probability transitions at column k: p_bm[k], p_mm[k-1], p_im[k-1], p_dm[k-1],
    // p_mi[k], p_ii[k], p_md[k-1], p_dd[k-1]
    float tp[8][VC];
#pragma unroll
    for (int q = 0; q < 8; q++)
#pragma unroll
      for (int c = 0; c < VC; c++) tp[q][c] = img.at(kRowFwd + q, c, lane);
    float sm[VC], omp[VC], oip[VC], odp[VC];
#pragma unroll
    for (int c = 0; c < VC; c++) {
      sm[c] = 0.f;
      omp[c] = oip[c] = odp[c] = SX_NEG_INF;
      OM[c * 32 + lane] = SX_NEG_INF;
      OI[c * 32 + lane] = SX_NEG_INF;
      OD[c * 32 + lane] = SX_NEG_INF;
    }
    float si = 0.f;
    float xbp = 0.f, xnp = 0.f, xjp = SX_NEG_INF, xcp = SX_NEG_INF;
    if (lane == 0) {
      sxe[0] = SX_NEG_INF; sxn[0] = 0.f; sxj[0] = SX_NEG_INF; sxb[0] = 0.f; sxc[0] = SX_NEG_INF;
    }
    for (int i = 1; i <= L; i++) {
      const double f = fac[i];
      float pm[VC], pi[VC];
#pragma unroll
      for (int c = 0; c < VC; c++) {
        const int k = lane * VC + c + 1;
        const int64_t e = (int64_t)i * RS + c * 32 + lane;
        pm[c] = k <= M ? (float)__dmul_rn(__dmul_rn((double)FM[e], (double)OM[e]), f) : 0.f;
        pi[c] = k < M ? (float)__dmul_rn(__dmul_rn((double)FI[e], (double)OI[e]), f) : 0.f;
        if (k <= M) sm[c] = fadd(sm[c], pm[c]);
      }
      // si: every insert posterior, row-major in k
      for (int sl = 0; sl < nl; sl++) {
        if (lane == sl) {
#pragma unroll
          for (int c = 0; c < VC; c++)
            if (lane * VC + c + 1 <= M) si = fadd(si, pi[c]);
        }
        si = __shfl_sync(kFull, si, sl);
      }
      // OA row: M and I from the previous row, then the D chain in order
      const float oml0 = __shfl_up_sync(kFull, omp[VC - 1], 1);
      const float oil0 = __shfl_up_sync(kFull, oip[VC - 1], 1);
      const float odl0 = __shfl_up_sync(kFull, odp[VC - 1], 1);
      float om[VC], oi[VC], od[VC];
      float emax = SX_NEG_INF;
#pragma unroll
      for (int c = 0; c < VC; c++) {
        const int k = lane * VC + c + 1;
        om[c] = oi[c] = SX_NEG_INF;
        if (k <= M) {
          float sv = oa_gate(tp[0][c], xbp);
          if (k >= 2) {
            const float omv = c ? omp[c - 1] : oml0, oiv = c ? oip[c - 1] : oil0, odv = c ? odp[c - 1] : odl0;
            sv = fmaxf(sv, oa_gate(tp[1][c], omv));
            sv = fmaxf(sv, oa_gate(tp[2][c], oiv));
            sv = fmaxf(sv, oa_gate(tp[3][c], odv));
          } else {
            sv = fmaxf(sv, 0.0f);
          }
          om[c] = fadd(sv, pm[c]);
          emax = fmaxf(emax, om[c]);
          oi[c] = fadd(fmaxf(oa_gate(tp[4][c], omp[c]), oa_gate(tp[5][c], oip[c])), pi[c]);
        }
      }
      const float omleft0 = __shfl_up_sync(kFull, om[VC - 1], 1);
      float dcar = SX_NEG_INF;
      for (int sl = 0; sl < nl; sl++) {
        if (lane == sl) {
#pragma unroll
          for (int c = 0; c < VC; c++) {
            const int k = lane * VC + c + 1;
            if (k > M) {
              od[c] = SX_NEG_INF;
            } else if (k == 1) {
              od[c] = SX_NEG_INF;
              dcar = SX_NEG_INF;
            } else {
              const float omk1 = c ? om[c - 1] : omleft0;
              od[c] = fmaxf(oa_gate(tp[6][c], omk1), oa_gate(tp[7][c], dcar));
              dcar = od[c];
              emax = fmaxf(emax, od[c]);
            }
          }
        }
        dcar = __shfl_sync(kFull, dcar, sl);
      }
      if (lane >= nl) {
#pragma unroll
        for (int c = 0; c < VC; c++) od[c] = SX_NEG_INF;
      }
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) emax = fmaxf(emax, __shfl_xor_sync(kFull, emax, o));
      const float xe_i = emax;
      float t1 = ploop0 ? 0.0f : fadd(xjp, pj[i]);
      float t2 = pe_loop0 ? 0.0f : xe_i;
      const float xj_i = fmaxf(t1, t2);
      t1 = ploop0 ? 0.0f : fadd(xcp, pc[i]);
      t2 = pe_move0 ? 0.0f : xe_i;
      const float xc_i = fmaxf(t1, t2);
      const float xn_i = ploop0 ? 0.0f : fadd(xnp, pn[i]);
      t1 = pmove0 ? 0.0f : xn_i;
      t2 = pmove0 ? 0.0f : xj_i;
      const float xb_i = fmaxf(t1, t2);
#pragma unroll
      for (int c = 0; c < VC; c++) {
        const int64_t e = (int64_t)i * RS + c * 32 + lane;
        OM[e] = om[c];
        OI[e] = oi[c];
        OD[e] = od[c];
        omp[c] = om[c];
        oip[c] = oi[c];
        odp[c] = od[c];
      }
      if (lane == 0) {
        sxe[i] = xe_i; sxn[i] = xn_i; sxj[i] = xj_i; sxb[i] = xb_i; sxc[i] = xc_i;
      }
      xbp = xb_i;
      xnp = xn_i;
      xjp = xj_i;
      xcp = xc_i;
    }
    // null2 column sums: v[x] = sum_k (sm[k] * norm) * mo[x][k], k ascending
    const float norm = __fdiv_rn(1.0f, (float)max(L, 1));
    for (int x = 0; x < 20; x++) {
      float v = 0.f;
      for (int sl = 0; sl < nl; sl++) {
        if (lane == sl) {
#pragma unroll
          for (int c = 0; c < VC; c++)
            if (lane * VC + c + 1 <= M) v = fadd(v, fmul(fmul(sm[c], norm), img.at(kRowMo + x, c, lane)));
        }
        v = __shfl_sync(kFull, v, sl);
      }
      if (lane == 0) out[x] = v;
    }
    __syncwarp();  // the OA planes written by every lane, read by lane 0 below
    if (lane == 0) {
      out[20] = si;
      // traceback (optimal_accuracy_coords, dp.rs:1420-1564)
      auto TP = [&](int q, int k) { return img.at(kRowFwd + q, (k - 1) % VC, (k - 1) / VC); };
      auto at = [&](const float* pl, int row, int k) { return pl[plane_at<VC>(row, k)]; };
      enum St { SC, SE, SM, SI, SD, SB, SJ, SN };
      St s0 = SC;
      const int q_stripes = max(2, (M - 1) / 4 + 1);
      int i = L, k = 0;
      bool got_first = false, got_last = false;
      int ci0 = 0, ci1 = 0, ck0 = 0, ck1 = 0;
      const int64_t limit = 8LL * (L + 2) * (M + 2) + 64;
      for (int64_t guard = 1; guard <= limit; guard++) {
        St s1;
        if (s0 == SC) {
          if (i == 0) break;
          const float a = ploop0 ? SX_NEG_INF : fadd(sxc[i - 1], pc[i]);
          const float b = pe_move0 ? SX_NEG_INF : sxe[i];
          s1 = a > b ? SC : SE;
        } else if (s0 == SE) {
          float mx = SX_NEG_INF;
          int pick = 0;
          St pst = SM;
          for (int q = 0; q < q_stripes; q++) {
            for (int rr = 0; rr < 4; rr++) {
              const int kk = rr * q_stripes + q + 1;
              if (kk <= M && at(OM, i, kk) >= mx) { mx = at(OM, i, kk); pick = kk; pst = SM; }
            }
            for (int rr = 0; rr < 4; rr++) {
              const int kk = rr * q_stripes + q + 1;
              if (kk <= M && at(OD, i, kk) > mx) { mx = at(OD, i, kk); pick = kk; pst = SD; }
            }
          }
          if (pick == 0) break;
          k = pick;
          s1 = pst;
        } else if (s0 == SM) {
          if (i < 1 || k < 1) break;  // no predecessor left (reachable only when every path is -inf)
          if (!got_last) { got_last = true; ci1 = i; ck1 = k; }
          got_first = true;
          ci0 = i;
          ck0 = k;
          float path[4] = {SX_NEG_INF, SX_NEG_INF, SX_NEG_INF, oa_dis(TP(0, k), sxb[i - 1])};
          if (k >= 2) {
            path[0] = oa_dis(TP(1, k), at(OM, i - 1, k - 1));
            path[1] = oa_dis(TP(2, k), at(OI, i - 1, k - 1));
            path[2] = oa_dis(TP(3, k), at(OD, i - 1, k - 1));
          }
          int best = 0;
          for (int t = 1; t < 4; t++)
            if (path[t] > path[best]) best = t;
          k -= 1;
          i -= 1;
          s1 = best == 0 ? SM : best == 1 ? SI : best == 2 ? SD : SB;
        } else if (s0 == SD) {
          if (k < 1) break;
          float a = SX_NEG_INF, b = SX_NEG_INF;
          if (k >= 2) {
            a = oa_dis(TP(6, k), at(OM, i, k - 1));
            b = oa_dis(TP(7, k), at(OD, i, k - 1));
          }
          k -= 1;
          s1 = a >= b ? SM : SD;
        } else if (s0 == SI) {
          if (i < 1 || k < 1) break;
          const float a = oa_dis(TP(4, k), at(OM, i - 1, k));
          const float b = oa_dis(TP(5, k), at(OI, i - 1, k));
          i -= 1;
          s1 = a >= b ? SM : SI;
        } else if (s0 == SB) {
          const float a = pmove0 ? SX_NEG_INF : sxn[i];
          const float b = pmove0 ? SX_NEG_INF : sxj[i];
          if (a > b) s1 = SN;
          else break;
        } else {
          break;
        }
        if ((s1 == SN || s1 == SJ || s1 == SC) && s1 == s0) i -= 1;
        if (s1 == SN) break;
        s0 = s1;
      }
      const bool found = got_first && got_last;
      out[21] = found ? 1.f : 0.f;
      out[22] = (float)ci0;
      out[23] = (float)ci1;
      out[24] = (float)ck0;
      out[25] = (float)ck1;
    }
  }
}

}  // namespace sxk
