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

// Diagonal layout of a region's M/I/D planes for the stochastic traceback:
// cell (i, k), 1 <= i <= lr, 1 <= k <= M, at (i - k + M - 1) * M + (k - 1), so
// the cells of a run of match states, (i, k) -> (i-1, k-1), are adjacent.
__host__ __device__ __forceinline__ int64_t diag_at(int64_t i, int k, int M) {
  return (i - k + M - 1) * (int64_t)M + (k - 1);
}
__host__ __device__ __forceinline__ int64_t diag_plane(int64_t lr, int M) { return (lr + M - 1) * (int64_t)M; }

// forward_matrix: M/I planes (scaled, after each row's rescaling) and the raw
// special rows N B E J C scale for rows 1..lr.  DIAG writes the M, I and D
// planes in the diagonal layout instead (the stochastic traceback's input).
template <int VC, bool DIAG = false>
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
    float* FI = FM + (DIAG ? diag_plane(L, M) : (int64_t)(L + 1) * RS);
    float* FD = FI + diag_plane(L, M);
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
        if (DIAG) {
          const int k = lane * VC + c + 1;
          if (k <= M) {
            const int64_t at = diag_at(i + 1, k, M);
            FM[at] = mv[c];
            FI[at] = iv[c];
            FD[at] = dv[c];
          }
        } else {
          FM[(int64_t)(i + 1) * RS + c * 32 + lane] = mv[c];
          FI[(int64_t)(i + 1) * RS + c * 32 + lane] = iv[c];
        }
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

// Per-lane column arrays of a warp-per-envelope kernel: registers for narrow
// profiles, shared memory for wide ones (VC >= kPostSmemVC), where holding
// the post kernel's 17 arrays of VC floats in registers spills to local memory.
// In shared memory element c of a lane's array sits at s[32 * c]: a warp's
// access to one c is one conflict-free wavefront.
template <int VC, bool SH>
struct Cols {
  float r[SH ? 1 : VC];
  float* s;
  __device__ __forceinline__ float& operator[](int c) {
    if constexpr (SH) return s[c * 32];
    else return r[c];
  }
};
constexpr int kPostSmemVC = 16;
constexpr int kPostArrays = 17;  // tp[8], sm, omp, oip, odp, pm, pi, om, oi, od
// Dynamic shared memory of env_post_kernel<VC> (one warp per CTA): the row
// buffer of the insert-posterior sum, then the column arrays when they live
// in shared memory.
__host__ __device__ constexpr size_t env_post_smem(int vc) {
  return ((vc >= kPostSmemVC ? (size_t)kPostArrays : 0) + 1) * 32 * vc * sizeof(float);
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
    constexpr bool SH = VC >= kPostSmemVC;
    extern __shared__ float post_smem[];
    Cols<VC, SH> tp[8], sm, omp, oip, odp, pm, pi, om, oi, od;
    float* sirow = post_smem;  // the row's insert posteriors, element (c, lane) at c * 32 + lane
    if constexpr (SH) {
      float* b = post_smem + 32 * VC + lane;
#pragma unroll
      for (int q = 0; q < 8; q++) tp[q].s = b + q * 32 * VC;
      sm.s = b + 8 * 32 * VC;
      omp.s = b + 9 * 32 * VC;
      oip.s = b + 10 * 32 * VC;
      odp.s = b + 11 * 32 * VC;
      pm.s = b + 12 * 32 * VC;
      pi.s = b + 13 * 32 * VC;
      om.s = b + 14 * 32 * VC;
      oi.s = b + 15 * 32 * VC;
      od.s = b + 16 * 32 * VC;
    }
#pragma unroll
    for (int q = 0; q < 8; q++)
#pragma unroll
      for (int c = 0; c < VC; c++) tp[q][c] = img.at(kRowFwd + q, c, lane);
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
#pragma unroll
      for (int c = 0; c < VC; c++) {
        const int k = lane * VC + c + 1;
        const int64_t e = (int64_t)i * RS + c * 32 + lane;
        pm[c] = k <= M ? (float)__dmul_rn(__dmul_rn((double)FM[e], (double)OM[e]), f) : 0.f;
        pi[c] = k < M ? (float)__dmul_rn(__dmul_rn((double)FI[e], (double)OI[e]), f) : 0.f;
        if (k <= M) sm[c] = fadd(sm[c], pm[c]);
      }
      // si: every insert posterior, row-major in k.  The row's values go to
      // shared memory and lane 0 adds them in column order (the same order
      // and roundings as a lane-to-lane baton, without its 32 shuffle hops).
#pragma unroll
      for (int c = 0; c < VC; c++) sirow[c * 32 + lane] = pi[c];
      __syncwarp();
      if (lane == 0) {
        int c = 0, l = 0;
        for (int k = 1; k <= M; k++) {
          si = fadd(si, sirow[c * 32 + l]);
          if (++c == VC) {
            c = 0;
            l++;
          }
        }
      }
      __syncwarp();
      // OA row: M and I from the previous row, then the D chain in order
      const float oml0 = __shfl_up_sync(kFull, omp[VC - 1], 1);
      const float oil0 = __shfl_up_sync(kFull, oip[VC - 1], 1);
      const float odl0 = __shfl_up_sync(kFull, odp[VC - 1], 1);
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
      // The D chain od[k] = max(gate(t_md, om[k-1]), gate(t_dd, od[k-1])) only
      // selects and takes maxima of non-negative values (or -inf), exact in
      // any order, so it runs as a scan.  Column k maps the chain value v to
      // max(a_k, v) when t_dd > 0 and to the constant max(a_k, 0) otherwise
      // (k = 1: the constant -inf; k > M: the identity).  Each lane composes
      // its columns' maps, the composites are scanned across lanes (5 shuffle
      // rounds), and each lane replays its columns from its carry.
      bool lc = false;          // the lane's composite: constant (true) or v -> max(lv, v)
      float lv = SX_NEG_INF;
#pragma unroll
      for (int c = 0; c < VC; c++) {
        const int k = lane * VC + c + 1;
        if (k > M) continue;
        if (k == 1) {
          lc = true;
          lv = SX_NEG_INF;
          continue;
        }
        const float a = oa_gate(tp[6][c], c ? om[c - 1] : omleft0);
        if (tp[7][c] > 0.0f) {
          lv = fmaxf(lv, a);
        } else {
          lc = true;
          lv = fmaxf(a, 0.0f);
        }
      }
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {  // inclusive scan: earlier lanes' composite, then this lane's
        const int pc = __shfl_up_sync(kFull, (int)lc, o);
        const float pv = __shfl_up_sync(kFull, lv, o);
        if (lane >= o && !lc) {
          lv = fmaxf(pv, lv);
          lc = pc != 0;
        }
      }
      float dcar = __shfl_up_sync(kFull, lv, 1);  // chain value entering this lane's first column
      if (lane == 0) dcar = SX_NEG_INF;
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


// ---- stochastic traceback ensembles of multi-domain regions ------------------
// region_trace_ensemble (src/hmmer/pipeline.rs:360-477) up to the clustering:
// kTraceSamples sampled traces (stochastic_trace, src/hmmer/dp.rs:1075-1258)
// through the region's multihit Forward matrix (env_forward_kernel<VC, true>,
// diagonal layout), one Easel LCG stream per region, the per-trace null2 of
// every sampled domain and its per-position sums.  The host clusters the
// samples and takes the logs.

constexpr int kTraceSamples = 200;
constexpr int kTraceDoms = 32;   // sampled domains of one trace held in shared memory
constexpr int kTraceRecord = 6;  // region, trace, sqfrom, sqto, hmmfrom, hmmto (target coordinates)
constexpr int kTraceRes = 20;    // canonical residues; codes 20..23 degenerate, 24 '*'
// Per profile column k (1-based), kTraceCol floats at (k-1)*kTraceCol:
// p_bm[k] p_mm[k-1] p_im[k-1] p_dm[k-1] p_mi[k] p_ii[k] p_md[k-1] p_dd[k-1],
// then the match odds mo[x][k] of the 20 canonical residues.
constexpr int kTraceCol = 28;

struct TraceRec {
  int32_t m, t;        // profile length, target
  int32_t i0, lr;      // region residues i0 .. i0+lr-1 (0-based)
  float ploop, pmove;  // multihit special transitions of the target's length
  float pe_loop, pe_move;
  int64_t plane_off;   // diagonal M I D planes of env_forward_kernel<VC, true>
  int64_t row_off;     // its raw special rows, 6 (lr+1)
  int64_t n2_off;      // per-position null2 sums, lr+1 floats (slot 0 unused)
  int64_t col_off;     // the profile's column table (kTraceCol floats per column)
};

struct TraceConsts {
  uint32_t lcg0;        // LCG state after seeding (esl_mix3 of seed 42)
  int32_t deg_n[4];     // member counts of the degenerate codes B J Z X
  int8_t deg_m[4][20];  // their members (esl_abc_FAvgScVec order)
};

__device__ __forceinline__ double trace_uniform(uint32_t& rng) {
  rng = rng * 69069u + 1u;
  return (double)rng * 2.3283064365386962890625e-10;  // / 2^32, exact
}

// esl_vec_FNorm (Kahan) then esl_rnd_FChoose (src/hmmer/dp.rs:1026-1059); the
// quotients acc/norm are independent, so all are formed before the first test.
// The last candidate needs none: with no earlier hit the choice is N-1 whether
// or not its test passes.
template <int N>
__device__ __forceinline__ int trace_choose(uint32_t& rng, float (&v)[N]) {
  float s = 0.f, comp = 0.f;
#pragma unroll
  for (int i = 0; i < N; i++) {
    const float y = __fsub_rn(v[i], comp);
    const float t = __fadd_rn(s, y);
    comp = __fsub_rn(__fsub_rn(t, s), y);
    s = t;
  }
#pragma unroll
  for (int i = 0; i < N; i++) v[i] = s != 0.f ? __fdiv_rn(v[i], s) : 1.f / (float)N;
  double norm = 0.0, acc[N];
#pragma unroll
  for (int i = 0; i < N; i++) norm = __dadd_rn(norm, (double)v[i]);
  double a = 0.0;
#pragma unroll
  for (int i = 0; i < N; i++) acc[i] = a = __dadd_rn(a, (double)v[i]);
  const double roll = trace_uniform(rng);
  int pick = N - 1;
#pragma unroll
  for (int i = N - 2; i >= 0; i--)
    if (roll < __ddiv_rn(acc[i], norm)) pick = i;
  return pick;
}

// One warp per region; every lane follows the same trace (same loads, same LCG
// draws), lanes 0..19 carry the null2 sums of the residues, the warp scans the
// E-state entry candidates 32 at a time (each lane forms the running sum up to
// its candidate, in order) and all lanes update the per-position sums.  A
// region that leaves the matrix, or whose samples overflow the pool or the
// per-trace buffer, is flagged (status 1) for the host to redo.  Pool records
// carry the region's index `first + w` within the caller's batch.
static __global__ void __launch_bounds__(128) env_trace_kernel(const TraceRec* __restrict__ recs, int n,
                                                        const float* __restrict__ cols,
                                                        const uint8_t* __restrict__ res,
                                                        const int64_t* __restrict__ toff,
                                                        const float* __restrict__ planes,
                                                        const float* __restrict__ rows, float* __restrict__ n2sum,
                                                        int32_t* __restrict__ pool, int32_t* __restrict__ pool_count,
                                                        int32_t pool_cap, int32_t first, int32_t* __restrict__ status,
                                                        TraceConsts tc) {
  __shared__ float sn2[4][32];
  __shared__ int4 sdom[4][kTraceDoms];
  const int lane = threadIdx.x & 31;
  const int wib = (threadIdx.x >> 5) & 3;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  enum { SC, SE, SM, SI, SD, SB, SJ, SN };
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += warps) {
    const TraceRec r = recs[w];
    const int M = r.m;
    const int L = r.lr;
    const int64_t PL = diag_plane(L, M);
    const float* FM = planes + r.plane_off;
    const float* FI = FM + PL;
    const float* FD = FI + PL;
    const float* xr = rows + r.row_off;
    const float* col = cols + r.col_off;
    const uint8_t* s = res + toff[r.t] + r.i0;
    float* ns = n2sum + r.n2_off;
    bool bad = L < 1 || M < 1;
    for (int pos = lane; pos <= L; pos += 32) ns[pos] = 0.f;
    __syncwarp();
    // planes at (row, k), 1 <= k <= M; row 0 of the matrix is all zero
    auto plane = [&](const float* X, int row, int k) { return row ? __ldg(X + diag_at(row, k, M)) : 0.f; };
    auto prob = [&](int q, int k) { return __ldg(col + (k - 1) * kTraceCol + q); };
    const float pmove = r.pmove, ploop = r.ploop;
    // special row i, slots N B E J C and the rescale factor (1 when the row was
    // not rescaled); row 0 is the start state N = 1, B = pmove
    auto spec = [&](int slot, int i) -> float {
      if (i == 0) return slot == 0 || slot == 5 ? 1.f : slot == 1 ? pmove : 0.f;
      const float v = __ldg(xr + 6 * (int64_t)i + slot);
      return slot == 5 && !(v > 0.f) ? 1.f : v;
    };
    const int q_stripes = max(2, (M - 1) / 4 + 1);
    const int ncand = 8 * q_stripes;
    // entry candidate c of the E-state scan (the reference's striped order):
    // stripe c/8, M (c%8 < 4) or D, node (c%4)*q_stripes + c/8 + 1
    auto cand_k = [&](int c) { return (c & 3) * q_stripes + (c >> 3) + 1; };
    const int64_t limit = 8 * (int64_t)(L + 2) * (int64_t)(M + 2) + 64;
    uint32_t rng = tc.lcg0;
    for (int tr = 0; tr < kTraceSamples && !bad; tr++) {
      int s0 = SC;
      int i = L, k = 0;
      bool have = false;
      int sqfrom = 0, sqto = 0, hmmfrom = 0, hmmto = 0, nn = 0;
      float vs = 0.f;  // lane x < 20: sum of mo[x][node] over the domain's nodes
      int hi = L + 1;  // positions >= hi have their sum for this trace
      int nd = 0;      // domains of this trace so far (in discovery order: last first)
      for (int64_t guard = 1; guard <= limit; guard++) {
        int s1;
        if (s0 == SC) {
          if (i == 0) break;
          float path[2] = {fmul(spec(4, i - 1), ploop), fmul(fmul(spec(2, i), r.pe_move), spec(5, i))};
          s1 = trace_choose(rng, path) == 0 ? SC : SE;
        } else if (s0 == SE) {
          const double roll = trace_uniform(rng);
          const float norm = (float)__ddiv_rn(1.0, (double)spec(2, i));
          double acc = 0.0;
          int pick = 0, pst = SM;
          for (int pass = 0; pick == 0 && pass < 1000; pass++) {
            auto load = [&](int c) {
              const int kk = cand_k(c);
              return c < ncand && kk <= M ? (double)fmul(plane((c & 4) ? FD : FM, i, kk), norm) : 0.0;
            };
            double val = load(lane);
            for (int c0 = 0; c0 < ncand; c0 += 32) {
              const double nxt = c0 + 32 < ncand ? load(c0 + 32 + lane) : 0.0;
              // lane j: the running sum through candidate c0 + j, in order;
              // a skipped candidate adds +0, which leaves the sum unchanged
              double run = acc;
              for (int j = 0; j < 32; j++) {
                const double v = __shfl_sync(kFull, val, j);
                if (j <= lane) run = __dadd_rn(run, v);
              }
              const unsigned hit = __ballot_sync(kFull, roll < run);
              if (hit) {
                const int j = __ffs(hit) - 1;
                pick = cand_k(c0 + j);
                pst = ((c0 + j) & 4) ? SD : SM;
                break;
              }
              acc = __shfl_sync(kFull, run, 31);
              val = nxt;
            }
            if (pick == 0 && acc <= 0.0) break;
          }
          if (pick == 0) break;
          k = pick;
          have = true;
          sqfrom = sqto = hmmfrom = hmmto = nn = 0;
          vs = 0.f;
          s1 = pst;
        } else if (s0 == SM) {
          if (i < 1 || k < 1 || k > M) { bad = true; break; }
          if (have) {
            if (sqto == 0) { sqto = i; hmmto = k; }
            sqfrom = i;
            hmmfrom = k;
            nn++;
            if (lane < kTraceRes) vs = __fadd_rn(vs, prob(8 + lane, k));
          }
          float path[4] = {fmul(spec(1, i - 1), prob(0, k)), 0.f, 0.f, 0.f};
          if (k >= 2) {
            path[1] = fmul(plane(FM, i - 1, k - 1), prob(1, k));
            path[2] = fmul(plane(FI, i - 1, k - 1), prob(2, k));
            path[3] = fmul(plane(FD, i - 1, k - 1), prob(3, k));
          }
          const int c = trace_choose(rng, path);
          k -= 1;
          i -= 1;
          s1 = c == 0 ? SB : c == 1 ? SM : c == 2 ? SI : SD;
        } else if (s0 == SD) {
          float path[2] = {0.f, 0.f};
          if (k >= 2) {
            if (k > M) { bad = true; break; }
            path[0] = fmul(plane(FM, i, k - 1), prob(6, k));
            path[1] = fmul(plane(FD, i, k - 1), prob(7, k));
          }
          const int c = trace_choose(rng, path);
          k -= 1;
          s1 = c == 0 ? SM : SD;
        } else if (s0 == SI) {
          if (i < 1 || k < 1 || k > M) { bad = true; break; }
          if (have) {
            nn++;
            if (lane < kTraceRes) vs = __fadd_rn(vs, prob(8 + lane, k));
          }
          float path[2] = {fmul(plane(FM, i - 1, k), prob(4, k)), fmul(plane(FI, i - 1, k), prob(5, k))};
          const int c = trace_choose(rng, path);
          i -= 1;
          s1 = c == 0 ? SM : SI;
        } else if (s0 == SB) {
          if (have) {  // a sampled domain is complete: its null2 and its positions' sums
            if (nd >= kTraceDoms) { bad = true; break; }
            const float ld = (float)max(nn, 1);
            if (lane < kTraceRes) sn2[wib][lane] = __fdiv_rn(vs, ld);
            __syncwarp();
            if (lane >= kTraceRes && lane < kTraceRes + 4) {
              const int d = lane - kTraceRes;
              float a = 0.f;
              for (int q = 0; q < tc.deg_n[d]; q++) a = __fadd_rn(a, sn2[wib][tc.deg_m[d][q]]);
              sn2[wib][lane] = __fdiv_rn(a, (float)tc.deg_n[d]);
            } else if (lane == kTraceRes + 4) {
              sn2[wib][lane] = 1.f;
            }
            __syncwarp();
            for (int pos = sqto + 1 + lane; pos < hi; pos += 32) ns[pos] = __fadd_rn(ns[pos], 1.f);
            for (int pos = sqfrom + 1 + lane; pos <= sqto; pos += 32)
              ns[pos] = __fadd_rn(ns[pos], sn2[wib][__ldg(s + pos - 1)]);
            __syncwarp();
            hi = sqfrom + 1;
            if (lane == 0) sdom[wib][nd] = make_int4(sqfrom, sqto, hmmfrom, hmmto);
            nd++;
            have = false;
          }
          float path[2] = {fmul(spec(0, i), pmove), fmul(spec(3, i), pmove)};
          s1 = trace_choose(rng, path) == 0 ? SN : SJ;
        } else if (s0 == SJ) {
          if (i == 0) break;
          float path[2] = {fmul(spec(3, i - 1), ploop), fmul(fmul(spec(2, i), r.pe_loop), spec(5, i))};
          s1 = trace_choose(rng, path) == 0 ? SJ : SE;
        } else {
          if (i == 0) break;
          s1 = SN;
        }
        if ((s1 == SN || s1 == SJ || s1 == SC) && s1 == s0) i -= 1;
        s0 = s1;
      }
      if (bad) break;
      for (int pos = 1 + lane; pos < hi; pos += 32) ns[pos] = __fadd_rn(ns[pos], 1.f);
      __syncwarp();
      // this trace's domains in sequence order, as one block of the pool
      int base = 0;
      if (lane == 0 && nd > 0) base = atomicAdd(pool_count, nd);
      base = __shfl_sync(kFull, base, 0);
      if (nd > 0 && (int64_t)base + nd > (int64_t)pool_cap) {  // mark the reserved slots that exist as unused
        for (int q = lane; q < nd && base + q < pool_cap; q += 32) pool[(int64_t)(base + q) * kTraceRecord] = -1;
        bad = true;
        break;
      }
      for (int q = lane; q < nd; q += 32) {
        const int4 d = sdom[wib][nd - 1 - q];
        int32_t* o = pool + (int64_t)(base + q) * kTraceRecord;
        o[0] = first + w;
        o[1] = tr;
        o[2] = d.x + r.i0;
        o[3] = d.y + r.i0;
        o[4] = d.z;
        o[5] = d.w;
      }
      __syncwarp();
    }
    if (lane == 0) status[w] = bad ? 1 : 0;
  }
}

}  // namespace sxk
