// sm_100a kernels of the sxhmm engine: the hmmsearch filter cascade and the
// Forward/Backward passes over (profile, target) pairs.
//
// Exactness contract.  Every score-producing operation is an explicit
// round-to-nearest f32 add/mul (__fadd_rn/__fmul_rn; the build also passes
// -fmad=false) or an exact max, applied in the association order of the
// reference (src/hmmer/dp.rs).  MSV and Viterbi therefore return the
// reference's scores bit for bit, and Forward/Backward produce bit-identical
// scaled rows; the only transcendental work on the device (f64 log of the
// rescale factors, f32 log of the final Forward value, the f64 logs of the
// composition-bias filter) feeds conservative filter decisions only, which the
// host re-checks exactly with the reference's libm.
#pragma once
#include <cstdint>

namespace sxk {

#define SX_NEG_INF (__int_as_float(0xff800000))
constexpr float kLn2 = 0.693147182464599609375f;
constexpr unsigned kFull = 0xffffffffu;

// ---- device records ------------------------------------------------------
struct DevProfile {  // 88 bytes
  int32_t m;
  int32_t vc;        // columns per lane in the warp-chunked layout (32 lanes)
  int32_t vbin;      // survivor-list bin of vc
  int32_t msv_g;     // MSV lanes per target
  int32_t msv_c;     // MSV columns per lane
  int32_t q_cap;     // packed pre-screen: row maxima above this (int16 units) pass at once
  int64_t msv_off;   // float4 offset of the MSV shared-memory image
  int64_t vfb_off;   // float offset of the warp-chunked image (kImgRows rows of 32*vc)
  float msv_tbm;
  int32_t vshape;    // Viterbi lane-group shape (index into the engine's shape table)
  int64_t vit_off;   // float4 offset of the Viterbi image (33 rows, lane-major for that shape)
  int64_t q_off;     // uint2 offset of the quantized MSV image; -1: the profile is not pre-screened
  int32_t q_tbm;     // msv_tbm rounded up, units of 2^-20 nat (pre-screen entry constant)
  int32_t qv_shape;  // packed Viterbi pre-screen shape; -1: the profile is not pre-screened
  int64_t qv_off;    // uint4 offset of its quantized Viterbi image
  int32_t qv_cap;    // its row maxima above this (int16 units) pass at once
  int32_t pad2;
};
struct Thresholds {  // per profile, per search: pass iff statistic >= threshold (bits)
  float s1, s2, s3;
  int32_t exact;     // 1: thresholds are exact (monotone tails); 0: filtering disabled
};
struct PairRec {  // 32 bytes
  int32_t p, t;
  float usc, filtersc, vsc, fwd;
  int32_t slot;   // caller's slot (explicit-pair mode) or -1
  int32_t pad;
};
struct BinRegion {
  int64_t off;
  uint32_t cap;
  uint32_t pad;
};
struct MsvTile {
  int32_t p, begin, end, pad;
};

// warp-chunked image row indices
enum : int {
  kRowMsc = 0,    // 25 rows: log-odds match scores msc[x][k]
  kRowVit = 25,   // 8 rows: t_mm[k-1], t_im[k-1], t_dm[k-1], t_bm[k], t_mi[k], t_ii[k], t_md[k-1], t_dd[k-1]
  kRowMo = 33,    // 25 rows: match odds mo[x][k]
  kRowFwd = 58,   // 8 rows: p_bm[k], p_mm[k-1], p_im[k-1], p_dm[k-1], p_mi[k], p_ii[k], p_md[k-1], p_dd[k-1]
  kRowBwd = 66,   // 8 rows: p_mm[k], p_mi[k], p_md[k], p_im[k], p_ii[k], p_dm[k], p_dd[k], p_bm[k]
  kImgRows = 74
};

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fmx(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ float fmx3(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
// Maximum over the full warp in one redux: the map f -> bits ^ (sign ? 0x7fffffff : 0)
// is an order-preserving bijection from non-NaN f32 to int32 and its own inverse,
// so the result is exactly the f32 maximum (only -0 and +0 are told apart,
// with -0 below +0, which fmaxf may order either way).
__device__ __forceinline__ float warp_max_f32(float v) {
  int k = __float_as_int(v);
  k ^= (k >> 31) & 0x7fffffff;
  k = __reduce_max_sync(kFull, k);
  k ^= (k >> 31) & 0x7fffffff;
  return __int_as_float(k);
}
// Maximum of v[0..N) with the fewest ALU instructions: three-input maxes level
// by level with the remainders carried up, so at most the last step is a
// two-input max — floor(N/2) instructions.  Overwrites v; max is exact in any
// order.
template <int N>
__device__ __forceinline__ float max_tree(float* v) {
  if constexpr (N == 1) {
    return v[0];
  } else if constexpr (N == 2) {
    return fmx(v[0], v[1]);
  } else {
    constexpr int T = N / 3, R = N % 3;
#pragma unroll
    for (int i = 0; i < T; i++) v[i] = fmx3(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
#pragma unroll
    for (int i = 0; i < R; i++) v[T + i] = v[3 * T + i];
    return max_tree<T + R>(v);
  }
}
__device__ __forceinline__ float bits_stat(float sc, float ref) { return __fdiv_rn(__fsub_rn(sc, ref), kLn2); }

__device__ __forceinline__ void push_pair(const PairRec& r, int bin, PairRec* lists, const BinRegion* bins,
                                          unsigned* counts, unsigned* overflow) {
  const unsigned pos = atomicAdd(&counts[bin], 1u);
  if (pos < bins[bin].cap) lists[bins[bin].off + pos] = r;
  else atomicOr(overflow, 1u);
}

// ===========================================================================
// MSV filter (src/hmmer/dp.rs:92-145).
//
// A CTA owns one tile = (profile, slice of a target list).  The profile's
// match-score rows are staged once in shared memory in a lane-major float4
// layout; each warp is split into groups of G lanes, every group scores one
// target at a time and pulls the next target from the slice with a shared
// atomic.  Lane j of a group holds columns k = j*C + c + 1 (c < C) of the DP
// row in registers; the diagonal dependency needs one shuffle per row and the
// row maximum a log2(G)-step butterfly.  Rows are consumed four at a time from
// 16-byte residue words prefetched one word ahead.  A group that runs past
// its target keeps computing on throw-away rows so the warp never diverges
// inside the row loop; the score is latched at row L.
// ===========================================================================
template <int G, int C>
__global__ void __launch_bounds__(256, 2) msv_kernel(const MsvTile* __restrict__ tiles, const DevProfile* __restrict__ profs,
                                                  const Thresholds* __restrict__ thr,
                                                  const float4* __restrict__ msv_img, const uint8_t* __restrict__ res,
                                                  const int64_t* __restrict__ toff, const int32_t* __restrict__ tlen,
                                                  const float4* __restrict__ tpar, const int32_t* __restrict__ list,
                                                  float* __restrict__ score_out, const int32_t* __restrict__ slot,
                                                  PairRec* __restrict__ surv, const BinRegion* __restrict__ bins,
                                                  unsigned* __restrict__ counts, unsigned* __restrict__ overflow,
                                                  const unsigned* __restrict__ rcount, unsigned rcap, int p0) {
  static_assert(C % 4 == 0 && (G & (G - 1)) == 0 && G <= 32, "bad MSV shape");
  constexpr int NC4 = C / 4;
  constexpr int ROW4 = NC4 * G;  // float4 per residue row
  // A quarter-warp (8 lanes) issues one LDS.128 wavefront: with G < 8 it holds
  // 8/G groups reading rows of different residues.  Each of those groups reads
  // its own copy of the image, copy q shifted by q*G float4 (q*16G bytes)
  // inside the 128-byte bank window, so their chunks never share a bank.
  constexpr int NCOPY = G < 8 ? 8 / G : 1;
  constexpr int ROWP = (ROW4 + 7) & ~7;            // row stride padded to 128 bytes
  constexpr int COPY4 = 25 * ROWP + 8;             // float4 per copy, +8 keeps copies 128-byte aligned
  extern __shared__ float4 sm_rows[];
  __shared__ int s_next;
  const MsvTile tile = tiles[blockIdx.x];
  const DevProfile P = profs[tile.p];
  {
    const float4* src = msv_img + P.msv_off;
    for (int q = threadIdx.x; q < 25 * ROW4; q += blockDim.x) {
      const int x = q / ROW4, e = q - x * ROW4;
      const float4 v = src[q];
#pragma unroll
      for (int cp = 0; cp < NCOPY; cp++) sm_rows[cp * COPY4 + cp * G + x * ROWP + e] = v;
    }
  }
  // Targets of the tile: list[first + k * stride] for first + k * stride < last.
  // A rescoring tile (rcount != null) takes the pre-screen's survivors of its
  // profile, region (p - p0) * rcap of the list, every `end`-th one from `begin`.
  int first = tile.begin, last = tile.end, stride = 1;
  if (rcount) {
    const int q = tile.p - p0;
    first = q * (int)rcap + tile.begin;
    last = q * (int)rcap + (int)min(rcount[q], rcap);
    stride = tile.end;
  }
  if (threadIdx.x == 0) s_next = 0;
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const int j = lane & (G - 1);
  const float4* my_rows = sm_rows + ((lane >> 0) / G % NCOPY) * (COPY4 + G);
  const int gl = lane - j;
  const unsigned gmask = (G == 32) ? kFull : (((1u << G) - 1u) << gl);
  const float tbm = P.msv_tbm;
  const float s1 = thr[tile.p].s1;
  const int bin = P.vbin;

  float prev[C];
#pragma unroll
  for (int c = 0; c < C; c++) prev[c] = SX_NEG_INF;
  float xn = 0.f, xb = 0.f, xj = SX_NEG_INF, tloop = 0.f, tmove = 0.f, nullsc = 0.f, fin = SX_NEG_INF;
  int entry = -1, tgt = 0, L = 0, row = 0, boff = 0;
  const uint8_t* seq = res;
  uint4 rcur = make_uint4(0x18181818u, 0x18181818u, 0x18181818u, 0x18181818u), rnext = rcur;
  bool active = false, done = false;

  for (;;) {
    if (!done && row >= L) {  // group-uniform: finish the current target, fetch the next
      if (active && j == 0) {
        const int p = tile.p;
        fin = fadd(fin, tmove);  // xc at row L, then C->T
        if (score_out) score_out[slot ? slot[entry] : entry] = fin;
        if (surv && bits_stat(fin, nullsc) >= s1) {
          PairRec r;
          r.p = p; r.t = tgt; r.usc = fin; r.filtersc = 0.f; r.vsc = 0.f; r.fwd = 0.f;
          r.slot = slot ? slot[entry] : -1; r.pad = 0;
          push_pair(r, bin, surv, bins, counts, overflow);
        }
      }
      int e = 0;
      if (j == 0) e = first + atomicAdd(&s_next, 1) * stride;
      e = __shfl_sync(gmask, e, gl);
      if (e < last) {
        entry = e;
        tgt = list[e];
        L = tlen[tgt];
        seq = res + toff[tgt];
        const float4 tp = tpar[tgt];
        tloop = tp.x; tmove = tp.y; nullsc = tp.z;
        xn = 0.f; xb = tmove; xj = SX_NEG_INF; fin = SX_NEG_INF;
#pragma unroll
        for (int c = 0; c < C; c++) prev[c] = SX_NEG_INF;
        row = 0;
        boff = 0;
        rcur = __ldg(reinterpret_cast<const uint4*>(seq));
        rnext = __ldg(reinterpret_cast<const uint4*>(seq + 16));
        active = true;
        if (L <= 0) { fin = SX_NEG_INF; }
      } else {
        active = false;
        done = true;
        L = 0;
      }
    }
    if (__all_sync(kFull, done)) break;

    const int q = (row - boff) >> 2;
    const int rem = L - row;  // rows left in the target; the score is latched when it reaches 0
    uint32_t w = q == 0 ? rcur.x : q == 1 ? rcur.y : q == 2 ? rcur.z : rcur.w;
    if (done) w = 0x18181818u;  // '*' rows: all -inf, never read back
    float xjr[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int x = (w >> (8 * r)) & 0xff;
      const float4* rowp = my_rows + x * ROWP + j;
      float4 rv[NC4];
#pragma unroll
      for (int c4 = 0; c4 < NC4; c4++) rv[c4] = rowp[c4 * G];
      const float be = fadd(xb, tbm);
      float left = __shfl_up_sync(kFull, prev[C - 1], 1, G);
      if (j == 0) left = SX_NEG_INF;
      // new row in place, highest column first so prev[c-1] is still the old value
#pragma unroll
      for (int c = C - 1; c >= 1; c--) {
        const float4& a4 = rv[c >> 2];
        const float ra = (c & 3) == 0 ? a4.x : (c & 3) == 1 ? a4.y : (c & 3) == 2 ? a4.z : a4.w;
        prev[c] = fadd(ra, fmx(prev[c - 1], be));
      }
      prev[0] = fadd(rv[0].x, fmx(left, be));
      // row maximum: a tree of 3-input maxes over the lane's C columns
      float tv[C];
#pragma unroll
      for (int c = 0; c < C; c++) tv[c] = prev[c];
      float xe = max_tree<C>(tv);
#pragma unroll
      for (int o = G / 2; o >= 1; o >>= 1) xe = fmx(xe, __shfl_xor_sync(kFull, xe, o, G));
      // J and C follow the same recurrence from the same start (E->J and E->C
      // are both ln 1/2, J->J and C->C both tloop), so xc == xj on every row;
      // and max(xn+t, xj+t) == max(xn, xj)+t because f32 addition rounds
      // monotonically.  Both rewrites are exact.
      xj = fmx(fadd(xj, tloop), fadd(xe, -kLn2));
      xn = fadd(xn, tloop);
      xb = fadd(fmx(xn, xj), tmove);
      xjr[r] = xj;
    }
    // the target's last row falls in this block: latch J (= C) at row L
    if (rem >= 1 && rem <= 4) fin = rem == 1 ? xjr[0] : rem == 2 ? xjr[1] : rem == 3 ? xjr[2] : xjr[3];
    row += 4;
    if (row - boff == 16) {
      boff += 16;
      rcur = rnext;
      if (active) rnext = __ldg(reinterpret_cast<const uint4*>(seq + boff + 16));
    }
  }
}

// ===========================================================================
// Composition-bias filter score (src/hmmer/pipeline.rs:107-150), one thread per
// pair, in f64 with the device log.  Decision on the F1 threshold with slack;
// the host re-checks survivors with the exact libm value.
// btab per profile: eo0[25], eo1[25], t00, t01, t10, t11  (54 doubles)
// With `vlist`, the survivors of profiles that have a packed Viterbi
// pre-screen image go to their profile's list (region (p - p0) * vcap, count
// vcount[p - p0]) instead of the Viterbi lists.
// ===========================================================================
static __global__ void __launch_bounds__(256) bias_kernel(const PairRec* __restrict__ in, const unsigned* __restrict__ in_counts,
                                                   const BinRegion* __restrict__ in_bins, PairRec* __restrict__ out,
                                                   const BinRegion* __restrict__ out_bins, unsigned* __restrict__ out_counts,
                                                   unsigned* __restrict__ overflow, const double* __restrict__ btab,
                                                   const Thresholds* __restrict__ thr, const uint8_t* __restrict__ res,
                                                   const int64_t* __restrict__ toff, const int32_t* __restrict__ tlen,
                                                   float slack, float* __restrict__ score_out,
                                                   const DevProfile* __restrict__ profs,
                                                   PairRec* __restrict__ vlist = nullptr, unsigned vcap = 0,
                                                   unsigned* __restrict__ vcount = nullptr, int p0 = 0) {
  const int bin = blockIdx.y;
  const unsigned n = min(in_counts[bin], in_bins[bin].cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    PairRec r = in[in_bins[bin].off + i];
    const double* bt = btab + (size_t)r.p * 54;
    const double t00 = bt[50], t01 = bt[51], t10 = bt[52], t11 = bt[53];
    const uint8_t* s = res + toff[r.t];
    const int L = tlen[r.t];
    const double tiny = 2.2250738585072014e-308;
    double logsc = 0.0;
    int x = s[0];
    double d0 = __dmul_rn(bt[x], 0.999), d1 = __dmul_rn(bt[25 + x], 0.001);
    double mx = fmax(fmax(d0, d1), tiny);
    d0 = __ddiv_rn(d0, mx);
    d1 = __ddiv_rn(d1, mx);
    logsc = __dadd_rn(logsc, log(mx));
    for (int q = 1; q < L; q++) {
      x = s[q];
      const double n0 = __dmul_rn(__dadd_rn(__dmul_rn(d0, t00), __dmul_rn(d1, t10)), bt[x]);
      const double n1 = __dmul_rn(__dadd_rn(__dmul_rn(d0, t01), __dmul_rn(d1, t11)), bt[25 + x]);
      mx = fmax(fmax(n0, n1), tiny);
      d0 = __ddiv_rn(n0, mx);
      d1 = __ddiv_rn(n1, mx);
      logsc = __dadd_rn(logsc, log(mx));
    }
    logsc = __dadd_rn(logsc, log(__dadd_rn(d0, d1)));
    const double p1 = __ddiv_rn((double)L, __dadd_rn((double)L, 1.0));
    const float fsc = (float)__dadd_rn(__dadd_rn(logsc, __dmul_rn((double)L, log(p1))), log(__dsub_rn(1.0, p1)));
    r.filtersc = fsc;
    if (score_out) {
      score_out[r.slot] = fsc;
      continue;
    }
    if (bits_stat(r.usc, fsc) >= thr[r.p].s1 - slack) {
      if (vlist && profs[r.p].qv_shape >= 0) {
        const unsigned pos = atomicAdd(&vcount[r.p - p0], 1u);
        if (pos < vcap) vlist[(int64_t)(r.p - p0) * vcap + pos] = r;
        else atomicOr(overflow, 1u);
      } else {
        push_pair(r, profs[r.p].vshape, out, out_bins, out_counts, overflow);
      }
    }
  }
}

// DP cells (sum of M * L) of the pairs in the per-bin lists (grid.y = bin):
// the work a stage receives, for its GCUPS.  Double atomics per warp; the
// order of the additions (and so the last bits) may vary between runs.
static __global__ void __launch_bounds__(256) stage_cells_kernel(const PairRec* __restrict__ lists,
                                                          const unsigned* __restrict__ counts,
                                                          const BinRegion* __restrict__ bins,
                                                          const DevProfile* __restrict__ profs,
                                                          const int32_t* __restrict__ tlen, double* __restrict__ out) {
  const int b = blockIdx.y;
  const unsigned n = min(counts[b], bins[b].cap);
  double acc = 0.0;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const PairRec r = lists[bins[b].off + i];
    acc += (double)profs[r.p].m * (double)tlen[r.t];
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) acc += __shfl_down_sync(kFull, acc, o);
  if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(out, acc);
}

// Lane-chunked access to the warp-chunked profile image: column k = lane*VC + c + 1.
template <int VC>
struct Img {
  const float* base;
  __device__ __forceinline__ float at(int row, int c, int lane) const { return __ldg(base + ((row * VC + c) << 5) + lane); }
};

// Eight per-column transition rows of the image starting at `row0`: held in
// registers for the whole pair when VC is small (M <= 128), re-read from the
// (L1-cached) image otherwise.
template <int VC, bool kHold = (VC <= 4)>
struct TransRows {
  float t[8][VC];
  __device__ __forceinline__ void load(const Img<VC>& img, int row0, int lane) {
#pragma unroll
    for (int q = 0; q < 8; q++)
#pragma unroll
      for (int c = 0; c < VC; c++) t[q][c] = img.at(row0 + q, c, lane);
  }
  __device__ __forceinline__ float get(const Img<VC>&, int, int q, int c, int) const { return t[q][c]; }
};
template <int VC>
struct TransRows<VC, false> {
  __device__ __forceinline__ void load(const Img<VC>&, int, int) {}
  __device__ __forceinline__ float get(const Img<VC>& img, int row0, int q, int c, int lane) const {
    return img.at(row0 + q, c, lane);
  }
};

// ===========================================================================
// Viterbi filter (src/hmmer/dp.rs:152-189), one warp per pair, lane l holding
// columns l*VC+1 .. l*VC+VC.  M and I cells of a row are independent; the
// D chain D[k] = max(M[k-1]+t_md, D[k-1]+t_dd) is resolved lazily: each lane
// runs its chunk with carry -inf, then carries are pushed across lanes until
// no value changes.  fl(x+t) is monotone in x, so the fixed point equals the
// sequential recurrence exactly.
// ===========================================================================
template <int VC>
__global__ void __launch_bounds__(256) viterbi_kernel(
    const PairRec* __restrict__ in, const unsigned* __restrict__ in_counts, const BinRegion* __restrict__ in_bins,
    int bin, PairRec* __restrict__ out, const BinRegion* __restrict__ out_bins, unsigned* __restrict__ out_counts,
    unsigned* __restrict__ overflow, const DevProfile* __restrict__ profs, const Thresholds* __restrict__ thr,
    const float* __restrict__ vfb, const uint8_t* __restrict__ res, const int64_t* __restrict__ toff,
    const int32_t* __restrict__ tlen, const float4* __restrict__ xsc, float slack, float* __restrict__ score_out) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const unsigned n = min(in_counts[bin], in_bins[bin].cap);
  for (unsigned w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += warps) {
    PairRec r = in[in_bins[bin].off + w];
    const DevProfile P = profs[r.p];
    const Img<VC> img{vfb + P.vfb_off};
    const int M = P.m;
    const uint8_t* s = res + toff[r.t];
    const int L = tlen[r.t];
    const float4 xs = xsc[r.t];  // loop, move (log), ploop, pmove
    TransRows<VC> tr;
    tr.load(img, kRowVit, lane);
    float mp[VC], ip[VC], dp[VC], rs[VC];
#pragma unroll
    for (int c = 0; c < VC; c++) mp[c] = ip[c] = dp[c] = SX_NEG_INF;
    float xn = 0.f, xb = xs.y, xj = SX_NEG_INF, xc = SX_NEG_INF;
    int x = L > 0 ? __ldg(s) : 24;
#pragma unroll
    for (int c = 0; c < VC; c++) rs[c] = img.at(kRowMsc + x, c, lane);
    for (int i = 0; i < L; i++) {
      // prefetch the next row's residue and match scores
      const int xnext = (i + 1 < L) ? __ldg(s + i + 1) : 24;
      float rsn[VC];
#pragma unroll
      for (int c = 0; c < VC; c++) rsn[c] = img.at(kRowMsc + xnext, c, lane);
      const bool ins_ok = x != 24;
      const float mpl0 = __shfl_up_sync(kFull, mp[VC - 1], 1);
      const float ipl0 = __shfl_up_sync(kFull, ip[VC - 1], 1);
      const float dpl0 = __shfl_up_sync(kFull, dp[VC - 1], 1);
      const float mpl = lane ? mpl0 : SX_NEG_INF, ipl = lane ? ipl0 : SX_NEG_INF, dpl = lane ? dpl0 : SX_NEG_INF;
      float mv[VC], iv[VC], dv[VC];
#pragma unroll
      for (int c = 0; c < VC; c++) {
        const int k = lane * VC + c + 1;
        const float mpv = c ? mp[c - 1] : mpl, ipv = c ? ip[c - 1] : ipl, dpv = c ? dp[c - 1] : dpl;
        const float sc = fmx(fmx(fadd(mpv, tr.get(img, kRowVit, 0, c, lane)), fadd(ipv, tr.get(img, kRowVit, 1, c, lane))),
                             fmx(fadd(xb, tr.get(img, kRowVit, 3, c, lane)), fadd(dpv, tr.get(img, kRowVit, 2, c, lane))));
        mv[c] = fadd(sc, rs[c]);
        iv[c] = (k < M && ins_ok)
                    ? fmx(fadd(mp[c], tr.get(img, kRowVit, 4, c, lane)), fadd(ip[c], tr.get(img, kRowVit, 5, c, lane)))
                    : SX_NEG_INF;
      }
      // D chain, first pass with carry -inf
      const float mcl0 = __shfl_up_sync(kFull, mv[VC - 1], 1);
      float d = SX_NEG_INF;
#pragma unroll
      for (int c = 0; c < VC; c++) {
        const float mcv = c ? mv[c - 1] : (lane ? mcl0 : SX_NEG_INF);
        d = fmx(fadd(mcv, tr.get(img, kRowVit, 6, c, lane)), fadd(d, tr.get(img, kRowVit, 7, c, lane)));
        dv[c] = d;
      }
      // push carries across lanes until nothing changes (at most 31 rounds)
      for (int it = 0; it < 32; it++) {
        const float cin0 = __shfl_up_sync(kFull, dv[VC - 1], 1);
        float cin = lane ? cin0 : SX_NEG_INF;
        bool go = true, changed = false;
#pragma unroll
        for (int c = 0; c < VC; c++) {
          if (go) {
            const float cand = fadd(cin, tr.get(img, kRowVit, 7, c, lane));
            if (cand > dv[c]) {
              dv[c] = cand;
              cin = cand;
              changed = true;
            } else {
              go = false;
            }
          }
        }
        if (!__any_sync(kFull, changed)) break;
      }
      float xe = SX_NEG_INF;
#pragma unroll
      for (int c = 0; c < VC; c++) xe = fmx3(xe, mv[c], dv[c]);
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) xe = fmx(xe, __shfl_xor_sync(kFull, xe, o));
      xj = fmx(fadd(xj, xs.x), fadd(xe, -kLn2));
      xc = fmx(fadd(xc, xs.x), fadd(xe, -kLn2));
      xn = fadd(xn, xs.x);
      xb = fmx(fadd(xn, xs.y), fadd(xj, xs.y));
#pragma unroll
      for (int c = 0; c < VC; c++) {
        mp[c] = mv[c];
        ip[c] = iv[c];
        dp[c] = dv[c];
        rs[c] = rsn[c];
      }
      x = xnext;
    }
    const float vsc = (L > 0 && M > 0) ? fadd(xc, xs.y) : SX_NEG_INF;
    if (lane == 0) {
      r.vsc = vsc;
      if (score_out) score_out[r.slot] = vsc;
      else if (bits_stat(vsc, r.filtersc) >= thr[r.p].s2 - slack) push_pair(r, bin, out, out_bins, out_counts, overflow);
    }
  }
}

// ===========================================================================
// Forward (src/hmmer/dp.rs:229-298), one warp per pair, probability space with
// the reference's sparse rescaling.  M and I cells are computed in parallel;
// the D chain and the row sum xe (both sequential in k in the reference) are
// evaluated in order by passing a baton from lane to lane, so every rounding
// matches.  Modes: rows != null writes the raw special rows (N B E J C, rescale
// factor) per row i = 1..L; otherwise the pair passes when the device estimate
// of the F3 statistic clears the threshold minus `slack`.
//
// SCAN (the F3 pre-screen only): the D chain is an affine recurrence
// D[k] = a_k + D[k-1] p_k, so each lane forms its transfer (A, B) over its
// columns, a Kogge-Stone scan of 5 shuffles composes them across lanes, each
// lane re-runs its columns from the true carry-in, and the row sum is a
// butterfly.  A row's dependent depth falls from ~2M to ~6 VC operations.  The
// rounding differs from the reference's order, so the pass test adds a bound
// on the difference: for sums and products of non-negative numbers the
// relative errors of two evaluation orders add up along their longest paths,
// at most 2^-24 per operation, i.e. |ln F_scan - ln F_ref| <=
// (L+1)(2M + 6 VC + 64) 2^-24, taken twice.  The pre-screen therefore passes
// every pair the exact F3 test (on the host, from exact rows) passes.
// ===========================================================================
template <int VC, bool SCAN = false>
__global__ void __launch_bounds__(256) forward_kernel(
    const PairRec* __restrict__ in, const unsigned* __restrict__ in_counts, const BinRegion* __restrict__ in_bins,
    int bin, PairRec* __restrict__ out, const BinRegion* __restrict__ out_bins, unsigned* __restrict__ out_counts,
    unsigned* __restrict__ overflow, const DevProfile* __restrict__ profs, const Thresholds* __restrict__ thr,
    const float* __restrict__ vfb, const uint8_t* __restrict__ res, const int64_t* __restrict__ toff,
    const int32_t* __restrict__ tlen, const float4* __restrict__ xsc, float slack, float* __restrict__ rows,
    const int64_t* __restrict__ row_off) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const unsigned n = min(in_counts[bin], in_bins[bin].cap);
  for (unsigned w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += warps) {
    PairRec r = in[in_bins[bin].off + w];
    const DevProfile P = profs[r.p];
    const Img<VC> img{vfb + P.vfb_off};
    const int M = P.m;
    const int nl = (M + VC - 1) / VC;  // lanes holding columns 1..M
    const uint8_t* s = res + toff[r.t];
    const int L = tlen[r.t];
    const float4 xs = xsc[r.t];
    const float ploop = xs.z, pmove = xs.w;
    float* orow = rows ? rows + row_off[in_bins[bin].off + w] : nullptr;
    TransRows<VC> tr;
    tr.load(img, kRowFwd, lane);
    float mp[VC], ip[VC], dp[VC], eo[VC];
#pragma unroll
    for (int c = 0; c < VC; c++) mp[c] = ip[c] = dp[c] = 0.f;
    float xn = 1.f, xb = pmove, xj = 0.f, xc = 0.f;
    double lnscale = 0.0;
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
        iv[c] = k < M ? fmul(fadd(fmul(mp[c], tr.get(img, kRowFwd, 4, c, lane)), fmul(ip[c], tr.get(img, kRowFwd, 5, c, lane))), ins)
                      : 0.f;
      }
      const float mcl0 = __shfl_up_sync(kFull, mv[VC - 1], 1);
      const float mcl = lane ? mcl0 : 0.f;
#pragma unroll
      for (int c = 0; c < VC; c++) {
        a[c] = fmul(c ? mv[c - 1] : mcl, tr.get(img, kRowFwd, 6, c, lane));
        pdd[c] = tr.get(img, kRowFwd, 7, c, lane);
      }
      float dcar = 0.f, xe = 0.f;
      if constexpr (SCAN) {
        // lane transfer D_out = A + B D_in, then an inclusive scan over lanes
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
        dcar = lane ? din : 0.f;
        float xl = 0.f;
#pragma unroll
        for (int c = 0; c < VC; c++) {
          const float d = fadd(a[c], fmul(dcar, pdd[c]));
          dv[c] = d;
          xl = fadd(xl, fadd(mv[c], d));
          dcar = d;
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) xl = fadd(xl, __shfl_xor_sync(kFull, xl, o));
        xe = xl;
      } else {
        // ordered D chain and row sum: dc[k] = a_k + dc[k-1]*p_dd[k-1]; xe += mv + dc
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
      }
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
        lnscale += log((double)xe);
        scale = xe;
        xe = 1.0f;
      }
      if (orow && lane == 0) {
        float* o = orow + 6 * (i + 1);
        o[0] = xn; o[1] = xb; o[2] = xe; o[3] = xj; o[4] = xc; o[5] = scale;
      }
#pragma unroll
      for (int c = 0; c < VC; c++) {
        mp[c] = mv[c];
        ip[c] = iv[c];
        dp[c] = dv[c];
        eo[c] = eon[c];
      }
      x = xnext;
    }
    if (lane == 0) {
      const float v = fmul(xc, pmove);
      const float fsc = (L > 0 && M > 0) ? (float)((double)(v > 0.f ? logf(v) : SX_NEG_INF) + lnscale) : SX_NEG_INF;
      r.fwd = fsc;
      const float sl = SCAN ? slack + 2.0f * (float)(L + 1) * (float)(2 * M + 6 * VC + 64) * 5.9604645e-8f / kLn2 : slack;
      if (!rows && bits_stat(fsc, r.filtersc) >= thr[r.p].s3 - sl) push_pair(r, bin, out, out_bins, out_counts, overflow);
    }
  }
}

// ===========================================================================
// Backward (src/hmmer/dp.rs:301-392), one warp per pair.  The B sum (ascending
// in k) and the D chain (descending in k) are sequential in the reference and
// are evaluated by lane batons; every other cell is parallel.  Writes the raw
// special rows: row L (E, C), rows L-1..1 (N B E J C, rescale factor) and the
// row-0 B sum in slot 1 of row 0.
// ===========================================================================
template <int VC>
__global__ void __launch_bounds__(256) backward_kernel(
    const PairRec* __restrict__ in, const unsigned* __restrict__ in_counts, const BinRegion* __restrict__ in_bins,
    int bin, const DevProfile* __restrict__ profs, const float* __restrict__ vfb, const uint8_t* __restrict__ res,
    const int64_t* __restrict__ toff, const int32_t* __restrict__ tlen, const float4* __restrict__ xsc,
    float* __restrict__ rows, const int64_t* __restrict__ row_off) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const unsigned n = min(in_counts[bin], in_bins[bin].cap);
  for (unsigned w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += warps) {
    const PairRec r = in[in_bins[bin].off + w];
    const DevProfile P = profs[r.p];
    const Img<VC> img{vfb + P.vfb_off};
    const int M = P.m;
    const int nl = (M + VC - 1) / VC;
    const int lM = (M - 1) / VC;  // lane holding column M
    const uint8_t* s = res + toff[r.t];
    const int L = tlen[r.t];
    const float4 xs = xsc[r.t];
    const float ploop = xs.z, pmove = xs.w;
    float* orow = rows + row_off[in_bins[bin].off + w];
    float mn[VC], in_[VC], dn[VC];
    // row L
    float xc = pmove;
    float xe = fmul(xc, 0.5f);
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
    if (lane == 0 && L > 0) {
      float* o = orow + 6 * L;
      o[0] = 0.f; o[1] = 0.f; o[2] = xe; o[3] = 0.f; o[4] = xc; o[5] = 0.f;
    }
    double lnscale = 0.0;
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
      xe = fadd(fmul(xj, 0.5f), fmul(xc, 0.5f));
      xn = fadd(fmul(xn, ploop), fmul(xb, pmove));
      float rowmax = fmaxf(fmaxf(fmaxf(fmaxf(xb, xe), xn), xj), xc);
      // mnext[k] = mn[k+1]*eo[k+1]
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
          const float mv = fadd(fadd(fadd(fmul(mnext[c], img.at(kRowBwd + 0, c, lane)), fmul(iv[c], img.at(kRowBwd + 1, c, lane))), xe),
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
        lnscale += log((double)rowmax);
        scale = rowmax;
      }
      if (lane == 0) {
        float* o = orow + 6 * i;
        o[0] = xn; o[1] = xb_o; o[2] = xe; o[3] = xj; o[4] = xc; o[5] = scale;
      }
#pragma unroll
      for (int c = 0; c < VC; c++) {
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
        orow[0] = 0.f; orow[1] = b; orow[2] = 0.f; orow[3] = 0.f; orow[4] = 0.f; orow[5] = 0.f;
      }
    }
  }
}

}  // namespace sxk

namespace sxk {

// ===========================================================================
// Viterbi filter, lane-group form (src/hmmer/dp.rs:152-189).  A warp holds
// 32/G pairs; a group of G lanes scores one pair, lane j holding columns
// j*C+1 .. j*C+C.  The profile's 33 score rows (25 log-odds, 8 transitions
// shifted so column k reads its own slot) are a lane-major float4 image read
// through L1, four columns per 16-byte load.  A row is updated in place: M and
// I descending (each needs the old values at k and k-1), then the D chain
// ascending with carry -inf at the lane boundary, then carries are pushed
// across the group's lanes until nothing changes (exact, as fl(x+t) is
// monotone in x).  All groups step rows in lock step; a group that finishes a
// pair takes the next one, and the score is latched at its last row.
// ===========================================================================
template <int G, int C, bool RT>
__global__ void __launch_bounds__(256, (C <= 16 && !(RT && C > 8)) ? 2 : 1) viterbi_g_kernel(
    const PairRec* __restrict__ in, const unsigned* __restrict__ in_counts, const BinRegion* __restrict__ in_bins,
    int bin, PairRec* __restrict__ out, const BinRegion* __restrict__ out_bins, unsigned* __restrict__ out_counts,
    unsigned* __restrict__ overflow, const DevProfile* __restrict__ profs, const Thresholds* __restrict__ thr,
    const float4* __restrict__ vimg, const uint8_t* __restrict__ res, const int64_t* __restrict__ toff,
    const int32_t* __restrict__ tlen, const float4* __restrict__ xsc, float slack, float* __restrict__ score_out,
    unsigned* __restrict__ cursor) {
  static_assert(C % 8 == 0 && (G & (G - 1)) == 0 && G <= 32, "bad Viterbi shape");
  constexpr int NC4 = C / 4;
  constexpr int ROW4 = NC4 * G;
  const int lane = threadIdx.x & 31;
  const int j = lane & (G - 1);
  const int gl = lane - j;
  const unsigned gmask = (G == 32) ? kFull : (((1u << G) - 1u) << gl);
  const unsigned n = min(in_counts[bin], in_bins[bin].cap);
  const int64_t base = in_bins[bin].off;

  float mp[C], ip[C], dp[C], pre[C];
  // RT: the pair's 8 transition rows for this lane's columns live in
  // registers (loaded once per pair); otherwise they are re-read every row
  float4 trr[RT ? 8 : 1][RT ? C / 4 : 1];
  float xn = 0.f, xb = 0.f, xj = SX_NEG_INF, fin = SX_NEG_INF;
  float lloop = 0.f, lmove = 0.f;
  int L = 0, row = 0, boff = 0;
  bool active = false, done = false;
  PairRec r{};
  const float4* img = vimg;
  const uint8_t* s = res;
  // residues 16 at a time from 16-byte words, one word fetched ahead (targets
  // are 16-byte aligned with slack after the last one)
  uint4 rcur = make_uint4(0x18181818u, 0x18181818u, 0x18181818u, 0x18181818u), rnext = rcur;
  float dpl = SX_NEG_INF;  // left lane's D at its last column, previous row
  int xcur = 24;           // residue of the current row ('*' past the end)
  float4 scur[NC4];        // its score chunks for this lane's columns
  auto residue_at = [](const uint4& w4, int q, bool valid) -> int {
    if (!valid) return 24;
    const uint32_t w = (q >> 2) == 0 ? w4.x : (q >> 2) == 1 ? w4.y : (q >> 2) == 2 ? w4.z : w4.w;
    return (w >> (8 * (q & 3))) & 0xff;
  };
  auto load_scores = [&](int xr) {
    const float4* rowx = img + xr * ROW4 + j;
#pragma unroll
    for (int c4 = 0; c4 < NC4; c4++) scur[c4] = rowx[c4 * G];
  };
  load_scores(24);
  for (;;) {
    if (!done && row >= L) {  // group-uniform: finish the pair, take the next one
      if (active && j == 0) {
        r.vsc = fin;
        if (score_out) score_out[r.slot] = fin;
        else if (bits_stat(fin, r.filtersc) >= thr[r.p].s2 - slack)
          push_pair(r, profs[r.p].vbin, out, out_bins, out_counts, overflow);
      }
      // pairs are handed out in list order, so the groups resident on an SM
      // work on neighbouring pairs (mostly one profile: its image stays in L1)
      unsigned e = 0;
      if (j == 0) e = atomicAdd(cursor + bin, 1u);
      e = __shfl_sync(gmask, e, gl);
      if (e < n) {
        r = in[base + e];
        const DevProfile P = profs[r.p];
        img = vimg + P.vit_off;
        L = tlen[r.t];
        s = res + toff[r.t];
        const float4 xs = xsc[r.t];
        lloop = xs.x;
        lmove = xs.y;
        xn = 0.f; xb = lmove; xj = SX_NEG_INF;
        fin = SX_NEG_INF;
#pragma unroll
        for (int c = 0; c < C; c++) mp[c] = ip[c] = dp[c] = pre[c] = SX_NEG_INF;
        row = 0;
        boff = 0;
        rcur = __ldg(reinterpret_cast<const uint4*>(s));
        rnext = __ldg(reinterpret_cast<const uint4*>(s + 16));
        dpl = SX_NEG_INF;
        xcur = residue_at(rcur, 0, L > 0);
        load_scores(xcur);
        if constexpr (RT) {
          const float4* t0 = img + 25 * ROW4 + j;
#pragma unroll
          for (int q = 0; q < 8; q++)
#pragma unroll
            for (int c4 = 0; c4 < NC4; c4++) trr[q][c4] = __ldg(t0 + (q * NC4 + c4) * G);
        }
        active = true;
      } else {
        active = false;
        done = true;
        L = 0;
      }
    }
    if (__all_sync(kFull, done)) break;
    const int x = xcur;
    const float4* tr = img + 25 * ROW4 + j;  // transition rows: mm im dm bm mi ii md dd
    auto T = [&](int q, int c4) -> float4 {
      if constexpr (RT) return trr[q][c4];
      else return tr[(q * NC4 + c4) * G];
    };
    auto pick = [](const float4& v, int e) { return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w; };
    // ip holds this row's I, computed during the previous row; a '*' residue
    // has no insert emission (rare: a group-uniform branch)
    if (x == 24) {
#pragma unroll
      for (int c = 0; c < C; c++) ip[c] = SX_NEG_INF;
    }
    // ---- M: max(pre, D[k-1] + t_dm, B + t_bm) + msc; pre = max(M[k-1] + t_mm,
    // I[k-1] + t_im) of the previous row, computed during that row; dpl is
    // the left lane's final D at its last column, from the carry loop ----
#pragma unroll
    for (int c4 = 0; c4 < NC4; c4++) {
      const float4 tdm = T(2, c4), tbm = T(3, c4);
      const float4 sc4 = scur[c4];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int c = 4 * c4 + e;
        const float dpv = c ? dp[c - 1] : dpl;
        mp[c] = fadd(fmx3(pre[c], fadd(dpv, pick(tdm, e)), fadd(xb, pick(tbm, e))), pick(sc4, e));
      }
    }
    // ---- D chain (ascending, carry -inf at the lane boundary) and, in the
    // same block so the scheduler can fill the chain's latency, the next
    // row's pre and I from this row's M and I (I descending, in place) ----
    const float mcl0 = __shfl_up_sync(kFull, mp[C - 1], 1, G);
    const float ipl0 = __shfl_up_sync(kFull, ip[C - 1], 1, G);
    const float mcl = j ? mcl0 : SX_NEG_INF, ipl = j ? ipl0 : SX_NEG_INF;
    float d = SX_NEG_INF;
#pragma unroll
    for (int c4 = 0; c4 < NC4; c4++) {
      const float4 tmd = T(6, c4), tdd = T(7, c4);
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int c = 4 * c4 + e;
        const float mcv = c ? mp[c - 1] : mcl;
        d = fmx(fadd(mcv, pick(tmd, e)), fadd(d, pick(tdd, e)));
        dp[c] = d;
      }
    }
#pragma unroll
    for (int c4 = NC4 - 1; c4 >= 0; c4--) {
      const float4 tmm = T(0, c4), tim = T(1, c4), tmi = T(4, c4), tii = T(5, c4);
#pragma unroll
      for (int e = 3; e >= 0; e--) {
        const int c = 4 * c4 + e;
        const float mpv = c ? mp[c - 1] : mcl, ipv = c ? ip[c - 1] : ipl;
        pre[c] = fmx(fadd(mpv, pick(tmm, e)), fadd(ipv, pick(tim, e)));
        // I of the next row (t_mi, t_ii are -inf from column M on, so I_M.. stay -inf)
        ip[c] = fmx(fadd(mp[c], pick(tmi, e)), fadd(ip[c], pick(tii, e)));
      }
    }
    // ---- push carries across the group's lanes (at most G-1 rounds); a
    // round runs only when some lane's first column improves ----
    // Every improving round moves the carries one lane on, so the loop ends
    // by the vote within G rounds; its last shuffle is the next row's dpl.
    bool settled = false;
    for (int it = 0; it < G; it++) {
      const float cin0 = __shfl_up_sync(kFull, dp[C - 1], 1, G);
      float cin = j ? cin0 : SX_NEG_INF;
      const bool need = fadd(cin, pick(T(7, 0), 0)) > dp[0];
      if (!__any_sync(kFull, need)) {
        dpl = cin;
        settled = true;
        break;
      }
      bool go = true;
#pragma unroll
      for (int c4 = 0; c4 < NC4; c4++) {
        if (go) {
          const float4 tdd = T(7, c4);
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const int c = 4 * c4 + e;
            if (go) {
              const float cand = fadd(cin, pick(tdd, e));
              if (cand > dp[c]) {
                dp[c] = cand;
                cin = cand;
              } else {
                go = false;
              }
            }
          }
        }
      }
    }
    if (!settled) {
      const float d0 = __shfl_up_sync(kFull, dp[C - 1], 1, G);
      dpl = j ? d0 : SX_NEG_INF;
    }
    // ---- row maximum and special states ----
    float blk[C / 8];
#pragma unroll
    for (int b = 0; b < C / 8; b++) {
      const float* mv = mp + 8 * b;
      const float* dv = dp + 8 * b;
      blk[b] = fmx3(fmx3(fmx3(mv[0], mv[1], mv[2]), fmx3(mv[3], mv[4], mv[5]), fmx(mv[6], mv[7])),
                    fmx3(dv[0], dv[1], dv[2]), fmx3(fmx3(dv[3], dv[4], dv[5]), dv[6], dv[7]));
    }
    float xe = blk[0];
#pragma unroll
    for (int b = 1; b < C / 8; b++) xe = fmx(xe, blk[b]);
    if constexpr (G == 32) {
      xe = warp_max_f32(xe);
    } else {
#pragma unroll
      for (int o = G / 2; o >= 1; o >>= 1) xe = fmx(xe, __shfl_xor_sync(kFull, xe, o, G));
    }
    // xc == xj and max(xn+t, xj+t) == max(xn, xj)+t, exactly (as in msv_kernel)
    xj = fmx(fadd(xj, lloop), fadd(xe, -kLn2));
    xn = fadd(xn, lloop);
    xb = fadd(fmx(xn, xj), lmove);
    row++;
    if (row == L) fin = fadd(xj, lmove);
    if (row - boff == 16) {
      boff += 16;
      rcur = rnext;
      if (active) rnext = __ldg(reinterpret_cast<const uint4*>(s + boff + 16));
    }
    // the next row's residue and score chunks, loaded a row ahead
    xcur = residue_at(rcur, row - boff, active && row < L);
    load_scores(xcur);
  }
}

}  // namespace sxk
