// Adjoint of the Forward score: gradients of lnZ (multihit, target-length
// config; src/hmmer/dp.rs:229-298) with respect to every log-space emission
// and transition score of the profile, i.e. the posterior expected counts
// that posterior decoding (src/hmmer/dp.rs:1278-1306) sums for domain
// definition.
//
// One warp per pair, lane l holding columns l*VC+1 .. l*VC+VC.  Kernel A runs
// Forward and keeps every S-th scaled row (S = ceil(sqrt(L))) plus the scaled
// special rows; kernel B runs Backward from row L down and, segment by
// segment, recomputes the S Forward rows it needs from the segment's
// checkpoint, so device scratch per pair is O(M sqrt(L)).  For each row i it
// accumulates, with per-row scale factors exp(lnF_a + lnB_b - lnZ) in f64:
//   emissions  F_M(i,k) B_M(i,k), F_I(i,k) B_I(i,k)
//   into row i F(i-1,k-1) t e(k,x_i) B_M(i,k)   (MM IM DM)  and  F_B(i-1) t_bm e B_M(i,k)
//   within i   F_M/F_D(i,k-1) t B_D(i,k)        (MD DD)
//   to row i+1 F_M/F_I(i,k) t ins(x_{i+1}) B_I(i+1,k)  (MI II)
// Every accumulator slot is written by exactly one lane (the owner of the
// transition's target column), so no atomics are needed.
#pragma once
#include "kernels.cuh"

namespace sxk {

struct AdjPair {
  int32_t p, t;
  int32_t S;        // checkpoint interval
  int32_t pad;
  int64_t ck_off;   // float offset: ceil(L/S)+1 checkpoint rows x 3 x 32*VC
  int64_t seg_off;  // float offset: (S+1) rows x 3 x 32*VC
  int64_t sp_off;   // float offset: (L+1) x 6 scaled specials (xn xb xe xj xc scale)
  int64_t ls_off;   // double offset: (L+1) cumulative Forward ln scale
  int64_t out_off;  // float offset in the output buffer: d_msc[25][M+1], d_isc[25][M+1], d_tr[8][M+1]
};

// One Forward row (dp.rs:254-296) for a warp: updates (mp, ip, dp) in place to
// row i and the specials; returns the row's rescale factor (0 if none).
template <int VC>
__device__ __forceinline__ float adj_fwd_row(const Img<VC>& img, int lane, int M, int nl, int x, float (&mp)[VC],
                                             float (&ip)[VC], float (&dp)[VC], float& xn, float& xb, float& xj,
                                             float& xc, float& xe_out, float ploop, float pmove) {
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
    float t = fmul(xb, img.at(kRowFwd + 0, c, lane));
    t = fadd(t, fmul(mpv, img.at(kRowFwd + 1, c, lane)));
    t = fadd(t, fmul(ipv, img.at(kRowFwd + 2, c, lane)));
    t = fadd(t, fmul(dpv, img.at(kRowFwd + 3, c, lane)));
    mv[c] = fmul(t, img.at(kRowMo + x, c, lane));
    iv[c] = k < M ? fmul(fadd(fmul(mp[c], img.at(kRowFwd + 4, c, lane)), fmul(ip[c], img.at(kRowFwd + 5, c, lane))), ins)
                  : 0.f;
  }
  const float mcl0 = __shfl_up_sync(kFull, mv[VC - 1], 1);
  const float mcl = lane ? mcl0 : 0.f;
#pragma unroll
  for (int c = 0; c < VC; c++) {
    a[c] = fmul(c ? mv[c - 1] : mcl, img.at(kRowFwd + 6, c, lane));
    pdd[c] = img.at(kRowFwd + 7, c, lane);
  }
  // D chain D[k] = a_k + D[k-1] p_k as an affine scan across lanes, row sum as
  // a butterfly (the adjoint is checked against FP64, not bit for bit)
  float A = 0.f, B = 1.f;
#pragma unroll
  for (int c = 0; c < VC; c++) {
    A = fadd(a[c], fmul(A, pdd[c]));
    B = fmul(B, pdd[c]);
  }
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const float Au = __shfl_up_sync(kFull, A, o), Bu = __shfl_up_sync(kFull, B, o);
    if (lane >= o) {
      A = fadd(A, fmul(B, Au));
      B = fmul(B, Bu);
    }
  }
  const float din = __shfl_up_sync(kFull, A, 1);
  float dcar = lane ? din : 0.f, xe = 0.f;
#pragma unroll
  for (int c = 0; c < VC; c++) {
    const float d = fadd(a[c], fmul(dcar, pdd[c]));
    dv[c] = d;
    xe = fadd(xe, fadd(mv[c], d));
    dcar = d;
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) xe = fadd(xe, __shfl_xor_sync(kFull, xe, o));
  if (lane >= nl) {
#pragma unroll
    for (int c = 0; c < VC; c++) dv[c] = 0.f;
  }
  xj = fadd(fmul(xj, ploop), fmul(xe, 0.5f));
  xc = fadd(fmul(xc, ploop), fmul(xe, 0.5f));
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
#pragma unroll
  for (int c = 0; c < VC; c++) {
    mp[c] = mv[c];
    ip[c] = iv[c];
    dp[c] = dv[c];
  }
  xe_out = xe;
  return scale;
}

template <int VC>
__device__ __forceinline__ void adj_store_row(float* base, int lane, const float (&m)[VC], const float (&i)[VC],
                                              const float (&d)[VC]) {
#pragma unroll
  for (int c = 0; c < VC; c++) {
    base[(0 * VC + c) * 32 + lane] = m[c];
    base[(1 * VC + c) * 32 + lane] = i[c];
    base[(2 * VC + c) * 32 + lane] = d[c];
  }
}
template <int VC>
__device__ __forceinline__ void adj_load_row(const float* base, int lane, float (&m)[VC], float (&i)[VC],
                                             float (&d)[VC]) {
#pragma unroll
  for (int c = 0; c < VC; c++) {
    m[c] = base[(0 * VC + c) * 32 + lane];
    i[c] = base[(1 * VC + c) * 32 + lane];
    d[c] = base[(2 * VC + c) * 32 + lane];
  }
}

// Kernel A: Forward with checkpoints every S rows; writes lnZ.
template <int VC>
__global__ void __launch_bounds__(128) adjoint_forward_kernel(const AdjPair* __restrict__ pairs, int npairs,
                                                              const DevProfile* __restrict__ profs,
                                                              const float* __restrict__ vfb,
                                                              const uint8_t* __restrict__ res,
                                                              const int64_t* __restrict__ toff,
                                                              const int32_t* __restrict__ tlen,
                                                              const float4* __restrict__ xsc, float* __restrict__ fbuf,
                                                              double* __restrict__ dbuf, double* __restrict__ lnz) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < npairs; w += warps) {
    const AdjPair A = pairs[w];
    const DevProfile P = profs[A.p];
    const Img<VC> img{vfb + P.vfb_off};
    const int M = P.m, nl = (M + VC - 1) / VC, L = tlen[A.t], S = A.S;
    const uint8_t* s = res + toff[A.t];
    const float4 xs = xsc[A.t];
    const float ploop = xs.z, pmove = xs.w;
    float* ck = fbuf + A.ck_off;
    float* sp = fbuf + A.sp_off;
    double* ls = dbuf + A.ls_off;
    float mp[VC], ip[VC], dp[VC];
#pragma unroll
    for (int c = 0; c < VC; c++) mp[c] = ip[c] = dp[c] = 0.f;
    float xn = 1.f, xb = pmove, xj = 0.f, xc = 0.f, xe = 0.f;
    double lnscale = 0.0;
    adj_store_row<VC>(ck, lane, mp, ip, dp);
    if (lane == 0) {
      sp[0] = xn; sp[1] = xb; sp[2] = 0.f; sp[3] = xj; sp[4] = xc; sp[5] = 0.f;
      ls[0] = 0.0;
    }
    for (int i = 1; i <= L; i++) {
      const float scale = adj_fwd_row<VC>(img, lane, M, nl, __ldg(s + i - 1), mp, ip, dp, xn, xb, xj, xc, xe, ploop, pmove);
      if (scale > 0.f) lnscale += log((double)scale);
      if (lane == 0) {
        float* o = sp + 6 * i;
        o[0] = xn; o[1] = xb; o[2] = xe; o[3] = xj; o[4] = xc; o[5] = scale;
        ls[i] = lnscale;
      }
      if (i % S == 0) adj_store_row<VC>(ck + (size_t)(i / S) * 3 * 32 * VC, lane, mp, ip, dp);
    }
    if (lane == 0) {
      const float v = fmul(xc, pmove);
      lnz[w] = (v > 0.f ? log((double)v) : -INFINITY) + lnscale;
    }
  }
}

// Kernel B: Backward sweep with segment recomputation and count accumulation.
template <int VC>
__global__ void __launch_bounds__(128) adjoint_backward_kernel(const AdjPair* __restrict__ pairs, int npairs,
                                                               const DevProfile* __restrict__ profs,
                                                               const float* __restrict__ vfb,
                                                               const uint8_t* __restrict__ res,
                                                               const int64_t* __restrict__ toff,
                                                               const int32_t* __restrict__ tlen,
                                                               const float4* __restrict__ xsc,
                                                               float* __restrict__ fbuf, const double* __restrict__ dbuf,
                                                               const double* __restrict__ lnz, float* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < npairs; w += warps) {
    const AdjPair A = pairs[w];
    const DevProfile P = profs[A.p];
    const Img<VC> img{vfb + P.vfb_off};
    const int M = P.m, nl = (M + VC - 1) / VC, lM = (M - 1) / VC, L = tlen[A.t], S = A.S;
    const uint8_t* s = res + toff[A.t];
    const float4 xs = xsc[A.t];
    const float ploop = xs.z, pmove = xs.w;
    const float* ck = fbuf + A.ck_off;
    float* seg = fbuf + A.seg_off;
    const float* sp = fbuf + A.sp_off;
    const double* lsf = dbuf + A.ls_off;
    const double lz = lnz[w];
    const int W = M + 1;
    float* __restrict__ o_msc = out + A.out_off;  // the three count arrays never overlap
    float* __restrict__ o_isc = out + A.out_off + 25 * W;
    float* __restrict__ o_tr = out + A.out_off + 50 * W;
    if (L <= 0 || !(lz > -INFINITY)) continue;
    const int rowf = 3 * 32 * VC;  // floats per stored row
    // Backward state: row i+1 (mn, inx, dn) and the specials
    float mn[VC], inx[VC], dn[VC];
    float bxc = pmove, bxe = fmul(pmove, 0.5f), bxj = 0.f, bxn = 0.f;
    double lnsb = 0.0;  // cumulative Backward ln scale of the current row
    int seg_lo = -1;    // first row held in `seg` (rows seg_lo .. seg_lo+S)
    for (int i = L; i >= 1; i--) {
      // ---- Backward row i ----
      float mc[VC], ic[VC], dc[VC];
      float bxb = 0.f;
      const double lnsb_next = lnsb;  // ln scale of row i+1
      double lnsb_i = lnsb;
      if (i == L) {
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
                mc[c] = dc[c] = 0.f;
              } else if (k == M) {
                mc[c] = dc[c] = bxe;
                dcar = bxe;
              } else {
                mc[c] = fadd(bxe, fmul(dcar, pmd0[c]));
                dc[c] = fadd(bxe, fmul(dcar, pdd0[c]));
                dcar = dc[c];
              }
            }
          }
          dcar = __shfl_sync(kFull, dcar, sl);
        }
        if (lane > lM) {
#pragma unroll
          for (int c = 0; c < VC; c++) mc[c] = dc[c] = 0.f;
        }
#pragma unroll
        for (int c = 0; c < VC; c++) ic[c] = 0.f;
      } else {
        const int x = __ldg(s + i);  // residue i+1
        const float ins = x != 24 ? 1.f : 0.f;
        float eo[VC], me[VC], bt[VC], pdm[VC], pdd[VC];
#pragma unroll
        for (int c = 0; c < VC; c++) {
          eo[c] = img.at(kRowMo + x, c, lane);
          me[c] = fmul(mn[c], eo[c]);
          bt[c] = fmul(fmul(mn[c], img.at(kRowBwd + 7, c, lane)), eo[c]);
          pdm[c] = img.at(kRowBwd + 5, c, lane);
          pdd[c] = img.at(kRowBwd + 6, c, lane);
        }
        float b = 0.f;
#pragma unroll
        for (int c = 0; c < VC; c++) b = fadd(b, bt[c]);
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) b = fadd(b, __shfl_xor_sync(kFull, b, o));
        bxb = b;
        bxj = fadd(fmul(bxj, ploop), fmul(bxb, pmove));
        bxc = fmul(bxc, ploop);
        bxe = fadd(fmul(bxj, 0.5f), fmul(bxc, 0.5f));
        bxn = fadd(fmul(bxn, ploop), fmul(bxb, pmove));
        float rowmax = fmaxf(fmaxf(fmaxf(fmaxf(bxb, bxe), bxn), bxj), bxc);
        const float me_up = __shfl_down_sync(kFull, me[0], 1);
        float mnext[VC], iv[VC];
#pragma unroll
        for (int c = 0; c < VC; c++) {
          mnext[c] = c < VC - 1 ? me[c + 1] : (lane < 31 ? me_up : 0.f);
          iv[c] = fmul(inx[c], ins);
        }
        // D chain, descending: D[k] = (mnext_k p_dm + bxe) + p_dd D[k+1], D[M] = bxe,
        // as an affine scan from the top lane down
        float A = 0.f, B = 1.f;
#pragma unroll
        for (int c = VC - 1; c >= 0; c--) {
          const int k = lane * VC + c + 1;
          const float al = k < M ? fadd(fmul(mnext[c], pdm[c]), bxe) : (k == M ? bxe : 0.f);
          const float be = k < M ? pdd[c] : 0.f;
          A = fadd(al, fmul(be, A));
          B = fmul(be, B);
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const float Ad = __shfl_down_sync(kFull, A, o), Bd = __shfl_down_sync(kFull, B, o);
          if (lane + o < 32) {
            A = fadd(A, fmul(B, Ad));
            B = fmul(B, Bd);
          }
        }
        const float dtop = __shfl_down_sync(kFull, A, 1);
        float dcar = lane < 31 ? dtop : 0.f;
#pragma unroll
        for (int c = VC - 1; c >= 0; c--) {
          const int k = lane * VC + c + 1;
          if (k > M) {
            dc[c] = 0.f;
          } else if (k == M) {
            dc[c] = bxe;
            dcar = bxe;
          } else {
            dc[c] = fadd(fadd(fmul(mnext[c], pdm[c]), fmul(dcar, pdd[c])), bxe);
            dcar = dc[c];
          }
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
            mc[c] = fadd(fadd(fadd(fmul(mnext[c], img.at(kRowBwd + 0, c, lane)), fmul(iv[c], img.at(kRowBwd + 1, c, lane))), bxe),
                         fmul(dnext, img.at(kRowBwd + 2, c, lane)));
            ic[c] = fadd(fmul(mnext[c], img.at(kRowBwd + 3, c, lane)), fmul(iv[c], img.at(kRowBwd + 4, c, lane)));
            rowmax = fmaxf(rowmax, mc[c]);
          } else if (k == M) {
            mc[c] = bxe;
            ic[c] = 0.f;
          } else {
            mc[c] = ic[c] = 0.f;
          }
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) rowmax = fmaxf(rowmax, __shfl_xor_sync(kFull, rowmax, o));
        if (rowmax > 1.0e4f) {
          const float inv = __fdiv_rn(1.0f, rowmax);
#pragma unroll
          for (int c = 0; c < VC; c++) {
            mc[c] = fmul(mc[c], inv);
            ic[c] = fmul(ic[c], inv);
            dc[c] = fmul(dc[c], inv);
          }
          bxe = fmul(bxe, inv);
          bxn = fmul(bxn, inv);
          bxj = fmul(bxj, inv);
          bxc = fmul(bxc, inv);
          lnsb += log((double)rowmax);
        }
        lnsb_i = lnsb;
      }
      // ---- Forward rows i-1 and i from the current segment ----
      if (seg_lo < 0 || i - 1 < seg_lo) {
        const int j = (i - 1) / S;
        seg_lo = j * S;
        float fm[VC], fi[VC], fd[VC];
        adj_load_row<VC>(ck + (size_t)j * rowf, lane, fm, fi, fd);
        adj_store_row<VC>(seg, lane, fm, fi, fd);
        const float* q = sp + 6 * seg_lo;
        float xn = q[0], xb = q[1], xj = q[3], xc = q[4], xe;
        const int hi = min(seg_lo + S, L);
        for (int r = seg_lo + 1; r <= hi; r++) {
          adj_fwd_row<VC>(img, lane, M, nl, __ldg(s + r - 1), fm, fi, fd, xn, xb, xj, xc, xe, ploop, pmove);
          adj_store_row<VC>(seg + (size_t)(r - seg_lo) * rowf, lane, fm, fi, fd);
        }
        __syncwarp();
      }
      float fm0[VC], fi0[VC], fd0[VC], fm1[VC], fi1[VC], fd1[VC];
      adj_load_row<VC>(seg + (size_t)(i - 1 - seg_lo) * rowf, lane, fm0, fi0, fd0);  // row i-1
      adj_load_row<VC>(seg + (size_t)(i - seg_lo) * rowf, lane, fm1, fi1, fd1);      // row i
      // ---- accumulate counts ----
      const int x = __ldg(s + i - 1);
      const float fb0 = sp[6 * (i - 1) + 1];
      // scale factors of the scaled cell products, exponents formed in f64
      const float f_ii = expf((float)(lsf[i] + lnsb_i - lz));        // F(i) . B(i)
      const float f_i0 = expf((float)(lsf[i - 1] + lnsb_i - lz));    // F(i-1) . B(i)
      const float f_i1 = expf((float)(lsf[i] + lnsb_next - lz));     // F(i) . B(i+1)
      const float fm0l0 = __shfl_up_sync(kFull, fm0[VC - 1], 1), fi0l0 = __shfl_up_sync(kFull, fi0[VC - 1], 1);
      const float fd0l0 = __shfl_up_sync(kFull, fd0[VC - 1], 1), fm1l0 = __shfl_up_sync(kFull, fm1[VC - 1], 1);
      const float fd1l0 = __shfl_up_sync(kFull, fd1[VC - 1], 1);
#pragma unroll
      for (int c = 0; c < VC; c++) {
        const int k = lane * VC + c + 1;
        if (k > M) continue;
        const float e = img.at(kRowMo + x, c, lane);
        o_msc[x * W + k] += fm1[c] * mc[c] * f_ii;
        if (k < M) o_isc[x * W + k] += fi1[c] * ic[c] * f_ii;
        const float bme = e * mc[c] * f_i0;
        o_tr[7 * W + k] += fb0 * img.at(kRowFwd + 0, c, lane) * bme;  // B -> M_k
        if (k >= 2) {
          const float m0 = c ? fm0[c - 1] : fm0l0, i0 = c ? fi0[c - 1] : fi0l0, d0 = c ? fd0[c - 1] : fd0l0;
          const float m1 = c ? fm1[c - 1] : fm1l0, d1 = c ? fd1[c - 1] : fd1l0;
          o_tr[0 * W + k - 1] += m0 * img.at(kRowFwd + 1, c, lane) * bme;    // MM
          o_tr[3 * W + k - 1] += i0 * img.at(kRowFwd + 2, c, lane) * bme;    // IM
          o_tr[5 * W + k - 1] += d0 * img.at(kRowFwd + 3, c, lane) * bme;    // DM
          o_tr[2 * W + k - 1] += m1 * img.at(kRowFwd + 6, c, lane) * dc[c] * f_ii;  // MD
          o_tr[6 * W + k - 1] += d1 * img.at(kRowFwd + 7, c, lane) * dc[c] * f_ii;  // DD
        }
        if (k < M && i < L) {
          const int xn1 = __ldg(s + i);
          if (xn1 != 24) {
            o_tr[1 * W + k] += fm1[c] * img.at(kRowFwd + 4, c, lane) * inx[c] * f_i1;  // MI
            o_tr[4 * W + k] += fi1[c] * img.at(kRowFwd + 5, c, lane) * inx[c] * f_i1;  // II
          }
        }
      }
      __syncwarp();
      // advance: row i becomes "next"
#pragma unroll
      for (int c = 0; c < VC; c++) {
        mn[c] = mc[c];
        inx[c] = ic[c];
        dn[c] = dc[c];
      }
    }
  }
}

}  // namespace sxk
