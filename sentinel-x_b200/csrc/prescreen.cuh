// Packed-integer MSV pre-screen: an upper bound of the reference's f32 MSV
// score (src/hmmer/dp.rs:92-145) for two profiles at once, in int16x2 lanes.
//
// Why: the exact f32 MSV kernel is bound by its ALU pipe and by the 4 bytes of
// shared memory each DP cell reads.  Here every 32-bit word carries the same
// column of two profiles (profile a in the low half, b in the high half), so
// one LDS.128 feeds 8 cells, one max.s16x2 / add.s16x2 pair does 2 cells, and
// the pair shares the target's residues and the diagonal shuffle.
//
// Exactness.  The pre-screen never decides a pair; it only rejects pairs whose
// bound fails F1, and every pair it passes is rescored by the exact kernel.
// The bound holds by construction:
//   * cells are integers in units of q = 2^-9 nat.  Every match score is
//     rounded up (e_u = ceil((e + rho)/q), rho = 2^-12 nat, which exceeds the
//     f32 rounding of one addition for |value| < 4096 nats) and clamped up to
//     -16 nats; the entry score is rounded up the same way and clamped up to
//     -32 nats.  Integer max-plus over rounded-up scores is >= the real-valued
//     recurrence, which is >= the f32 recurrence minus its rounding, so by
//     induction every integer cell is >= the f32 cell (max is exact and
//     monotone; raising an input only raises the result);
//   * the row maximum is an int16 max, exact; it enters the special states,
//     kept as int32 in units of 2^-20 nat with every constant (tloop, tmove,
//     tbm, -ln 2) rounded up after adding 2^-17 nat, the f32 rounding bound of
//     one addition for |value| <= 128 nats; the specials are therefore upper
//     bounds of the reference's f32 specials row by row;
//   * the final bound (xC + tmove, rounded up to f32) goes through the same
//     f32 bit statistic as the exact kernel, which is monotone.
// int16 headroom: cells stay in [-32768, cap + emax]; a row maximum above the
// profile's cap (32767 minus its largest rounded score) marks the pair as
// passing before any cell can wrap, and the flag is sticky.
#pragma once
#include <cstdint>

#include "kernels.cuh"

namespace sxk {

constexpr int kQ16Shift = 9;        // cells: units of 2^-9 nat
constexpr int kQ32Shift = 20;       // specials: units of 2^-20 nat
constexpr int kQ32Rho = 8;          // 2^-17 nat in units of 2^-20
constexpr int kQ16EFloor = -8192;   // -16 nats: lowest match score of a real column
constexpr int kQ16EPad = -16384;    // columns past M
constexpr int kQ16BeFloor = -16384; // -32 nats: lowest entry score
constexpr int kQ32Neg = -(1 << 30); // f32 -inf of the special states
constexpr unsigned kQ16Neg2 = 0x80008000u;  // (-32768, -32768)

// A pair of profiles of one MSV shape x a slice [begin, end) of the target list
// (pb = -1: the high half is padding and produces no decisions).
struct PackedTile {
  int32_t pa, pb, begin, end;
};

__device__ __forceinline__ unsigned max2s16(unsigned a, unsigned b) {
  unsigned d;
  asm("max.s16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
__device__ __forceinline__ unsigned add2s16(unsigned a, unsigned b) {
  unsigned d;
  asm("add.s16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
// f32 constant in units of 2^-20 nat, plus rho, rounded up (exact: x * 2^20 is
// exact in f32 and the integers involved stay below 2^24 in magnitude).
__device__ __forceinline__ int q32_up(float x) {
  return (int)ceilf(__fmul_rn(x, 1048576.0f)) + kQ32Rho;
}

// Bound of a profile pair against a slice of targets.  Each profile has its
// own quantized image (25 rows of int16, the lane-major chunk layout of its
// f32 MSV image, 4 columns per uint2); the CTA interleaves the two into words
// while staging them in shared memory.  Per target and half: with `rlist`,
// a pair whose bound passes F1 (or hit the cap) is appended to its profile's
// rescoring list (region (p - p0) * rcap); with `bound_out`, the bound
// (f32 nats, +inf when capped) is written at slot[entry] (profile a) and
// bound_stride + slot[entry] (profile b).
template <int G, int C>
__global__ void __launch_bounds__(256, 2) msv16_kernel(
    const PackedTile* __restrict__ tiles, const DevProfile* __restrict__ profs, const Thresholds* __restrict__ thr,
    const uint2* __restrict__ qimg, const uint8_t* __restrict__ res, const int64_t* __restrict__ toff,
    const int32_t* __restrict__ tlen, const float4* __restrict__ tpar, const int32_t* __restrict__ list,
    int32_t* __restrict__ rlist, unsigned rcap, unsigned* __restrict__ rcount, int p0, unsigned* __restrict__ overflow,
    float* __restrict__ bound_out, const int32_t* __restrict__ slot, int64_t bound_stride) {
  static_assert(C % 4 == 0 && (G & (G - 1)) == 0 && G <= 32, "bad MSV shape");
  constexpr int NC4 = C / 4;
  constexpr int ROW4 = NC4 * G;
  constexpr int NCOPY = G < 8 ? 8 / G : 1;   // bank-conflict-free copies, as in msv_kernel
  constexpr int ROWP = (ROW4 + 7) & ~7;
  constexpr int COPY4 = 25 * ROWP + 8;
  extern __shared__ uint4 sm_img[];
  __shared__ int s_next;
  const PackedTile tile = tiles[blockIdx.x];
  const DevProfile PA = profs[tile.pa];
  const bool has_b = tile.pb >= 0;
  const DevProfile PB = profs[has_b ? tile.pb : tile.pa];
  {
    const uint2* sa = qimg + PA.q_off;
    const uint2* sb = qimg + PB.q_off;
    for (int q = threadIdx.x; q < 25 * ROW4; q += blockDim.x) {
      const int x = q / ROW4, e = q - x * ROW4;
      const uint2 va = sa[q];
      const uint2 vb = has_b ? sb[q] : make_uint2(0xc000c000u, 0xc000c000u);
      const uint4 v = make_uint4(__byte_perm(va.x, vb.x, 0x5410), __byte_perm(va.x, vb.x, 0x7632),
                                 __byte_perm(va.y, vb.y, 0x5410), __byte_perm(va.y, vb.y, 0x7632));
#pragma unroll
      for (int cp = 0; cp < NCOPY; cp++) sm_img[cp * COPY4 + cp * G + x * ROWP + e] = v;
    }
  }
  if (threadIdx.x == 0) s_next = tile.begin;
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const int j = lane & (G - 1);
  const uint4* my_rows = sm_img + (lane / G % NCOPY) * (COPY4 + G);
  const int gl = lane - j;
  const unsigned gmask = (G == 32) ? kFull : (((1u << G) - 1u) << gl);
  const float s1a = thr[tile.pa].s1;
  const float s1b = has_b ? thr[tile.pb].s1 : 0.f;
  const int cap_a = PA.q_cap, cap_b = has_b ? PB.q_cap : 32767;
  const int tbm_a = PA.q_tbm, tbm_b = PB.q_tbm;
  const int nln2 = (int)ceilf(-0.693147182464599609375f * 1048576.0f) + kQ32Rho;

  unsigned prev[C];
#pragma unroll
  for (int c = 0; c < C; c++) prev[c] = kQ16Neg2;
  int xn = 0, xja = kQ32Neg, xjb = kQ32Neg, tloop = 0, tmove = 0;
  unsigned bew = kQ16Neg2;
  int fina = kQ32Neg, finb = kQ32Neg;
  bool biga = false, bigb = false;
  float nullsc = 0.f;
  int entry = -1, tgt = 0, L = 0, row = 0, boff = 0;
  const uint8_t* seq = res;
  uint4 rcur = make_uint4(0x18181818u, 0x18181818u, 0x18181818u, 0x18181818u), rnext = rcur;
  bool active = false, done = false;

  for (;;) {
    if (!done && row >= L) {  // group-uniform: finish the current target, fetch the next
      if (active && j == 0) {
        const float uba = biga ? __int_as_float(0x7f800000) : __fmul_rn(__int2float_ru(fina + tmove), 9.5367431640625e-7f);
        const float ubb = bigb ? __int_as_float(0x7f800000) : __fmul_rn(__int2float_ru(finb + tmove), 9.5367431640625e-7f);
        const bool pa_ok = biga || bits_stat(uba, nullsc) >= s1a;
        const bool pb_ok = has_b && (bigb || bits_stat(ubb, nullsc) >= s1b);
        if (bound_out) {
          const int64_t o = slot ? slot[entry] : entry;
          bound_out[o] = uba;
          if (has_b) bound_out[bound_stride + o] = ubb;
        }
        if (rlist) {
          if (pa_ok) {
            const unsigned pos = atomicAdd(&rcount[tile.pa - p0], 1u);
            if (pos < rcap) rlist[(int64_t)(tile.pa - p0) * rcap + pos] = tgt;
            else atomicOr(overflow, 1u);
          }
          if (pb_ok) {
            const unsigned pos = atomicAdd(&rcount[tile.pb - p0], 1u);
            if (pos < rcap) rlist[(int64_t)(tile.pb - p0) * rcap + pos] = tgt;
            else atomicOr(overflow, 1u);
          }
        }
      }
      int e = 0;
      if (j == 0) e = atomicAdd(&s_next, 1);
      e = __shfl_sync(gmask, e, gl);
      if (e < tile.end) {
        entry = e;
        tgt = list[e];
        L = tlen[tgt];
        seq = res + toff[tgt];
        const float4 tp = tpar[tgt];
        tloop = q32_up(tp.x);
        tmove = q32_up(tp.y);
        nullsc = tp.z;
        xn = 0;
        xja = xjb = kQ32Neg;
        fina = finb = kQ32Neg;
        biga = bigb = false;
        {  // entry score of row 1 from xB = tmove
          const int bea = max((tmove + tbm_a + 2047) >> (kQ32Shift - kQ16Shift), kQ16BeFloor);
          const int beb = max((tmove + tbm_b + 2047) >> (kQ32Shift - kQ16Shift), kQ16BeFloor);
          bew = __byte_perm((unsigned)bea, (unsigned)beb, 0x5410);
        }
#pragma unroll
        for (int c = 0; c < C; c++) prev[c] = kQ16Neg2;
        row = 0;
        boff = 0;
        rcur = __ldg(reinterpret_cast<const uint4*>(seq));
        rnext = __ldg(reinterpret_cast<const uint4*>(seq + 16));
        active = L > 0;
      } else {
        active = false;
        done = true;
        L = 0;
      }
    }
    if (__all_sync(kFull, done)) break;

    const int q = (row - boff) >> 2;
    const int rem = L - row;
    uint32_t w = q == 0 ? rcur.x : q == 1 ? rcur.y : q == 2 ? rcur.z : rcur.w;
    if (done) w = 0x18181818u;
    int xjra[4], xjrb[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int x = (w >> (8 * r)) & 0xff;
      const uint4* rowp = my_rows + x * ROWP + j;
      uint4 rv[NC4];
#pragma unroll
      for (int c4 = 0; c4 < NC4; c4++) rv[c4] = rowp[c4 * G];
      unsigned left = __shfl_up_sync(kFull, prev[C - 1], 1, G);
      if (j == 0) left = kQ16Neg2;
#pragma unroll
      for (int c = C - 1; c >= 1; c--) {
        const uint4& a4 = rv[c >> 2];
        const unsigned ra = (c & 3) == 0 ? a4.x : (c & 3) == 1 ? a4.y : (c & 3) == 2 ? a4.z : a4.w;
        prev[c] = add2s16(max2s16(prev[c - 1], bew), ra);
      }
      prev[0] = add2s16(max2s16(left, bew), rv[0].x);
      // row maximum: a tree of packed maxes, then a butterfly over the group
      unsigned tv[C];
#pragma unroll
      for (int c = 0; c < C; c++) tv[c] = prev[c];
#pragma unroll
      for (int span = 1; span < C; span <<= 1)
#pragma unroll
        for (int c = 0; c + span < C; c += 2 * span) tv[c] = max2s16(tv[c], tv[c + span]);
      unsigned xe = tv[0];
#pragma unroll
      for (int o = G / 2; o >= 1; o >>= 1) xe = max2s16(xe, __shfl_xor_sync(kFull, xe, o, G));
      const int ea = (int)(short)(xe & 0xffffu), eb = (int)xe >> 16;
      biga |= ea > cap_a;
      bigb |= eb > cap_b;
      // special states, int32 upper bounds of the reference's f32 N/J/C/B
      // (J and C follow the same recurrence, as in msv_kernel)
      xja = max(xja + tloop, ea * 2048 + nln2);
      xjb = max(xjb + tloop, eb * 2048 + nln2);
      xn += tloop;
      const int xba = max(xn, xja) + tmove, xbb = max(xn, xjb) + tmove;
      const int bea = max((xba + tbm_a + 2047) >> (kQ32Shift - kQ16Shift), kQ16BeFloor);
      const int beb = max((xbb + tbm_b + 2047) >> (kQ32Shift - kQ16Shift), kQ16BeFloor);
      bew = __byte_perm((unsigned)bea, (unsigned)beb, 0x5410);
      xjra[r] = xja;
      xjrb[r] = xjb;
    }
    if (rem >= 1 && rem <= 4) {
      fina = rem == 1 ? xjra[0] : rem == 2 ? xjra[1] : rem == 3 ? xjra[2] : xjra[3];
      finb = rem == 1 ? xjrb[0] : rem == 2 ? xjrb[1] : rem == 3 ? xjrb[2] : xjrb[3];
    }
    row += 4;
    if (row - boff == 16) {
      boff += 16;
      rcur = rnext;
      if (active) rnext = __ldg(reinterpret_cast<const uint4*>(seq + boff + 16));
    }
  }
}

}  // namespace sxk

namespace sxk {

// ---------------------------------------------------------------------------
// Packed-integer Viterbi pre-screen: an upper bound of the reference's f32
// Viterbi score (src/hmmer/dp.rs:152-189) for two targets of one profile at
// once, in int16x2 lanes (target a in the low half, b in the high half).
//
// Why: the exact lane-group kernel (viterbi_g_kernel) is bound by the
// latency of each row's sequential parts -- the D chain, the carry vote, the
// row-maximum butterfly, the special states -- and by the per-row control
// around them, which a lane group pays once per pair.  Here one pass of all
// of that serves two pairs: every 32-bit word holds the same column of two
// DP rows, one max.s16x2 / add.s16x2 updates both, and the carry vote, the
// butterfly and the loop control are shared.
//
// Exactness.  As for the MSV pre-screen, the bound never decides a pair: a
// pair passes when its bound passes F2 (with the exact kernel's slack), and
// every passing pair is rescored by viterbi_g_kernel, so the survivors of
// the stage are exactly the reference's.  The bound holds by construction:
//   * cells are integers in units of q = 2^-9 nat.  Match scores are rounded
//     up after adding 2^-12 nat (more than the f32 rounding of one addition
//     for |value| < 4096 nats) and clamped up to -8 nats; transition scores
//     the same way, clamped up to -8 nats (t_bm: -16 nats) and down to 0 --
//     a transition t <= 0 never raises a value (fl(a + t) <= a), so 0 bounds
//     any t in [-2^-12, 0]; -inf scores become the floor.  Integer max-plus
//     over rounded-up scores is >= the real-valued recurrence, which is >=
//     the f32 recurrence minus its rounding; by induction every integer cell
//     is >= the f32 cell (max is exact and monotone; raising an input only
//     raises the result).  The insert rows ignore the '*' residue's
//     insert-state cut (dp.rs:172), which only raises I;
//   * the row maximum is taken over M alone: with every transition <= 0,
//     D[k] <= max over k' < k of M[k'] in f32 and in the integers alike;
//   * the specials are int32 in units of 2^-20 nat with every constant
//     rounded up after adding 2^-17 nat, as in the MSV pre-screen;
//   * the final bound (xJ + tmove at row L, rounded up to f32) goes through
//     the exact kernel's f32 bit statistic, which is monotone.
// int16 range: the floors keep every sum >= -28672 (B + t_bm >= -12 nats so
// M >= -32 nats, D, I >= -40 nats, pre >= -48 nats, plus one more
// transition); every value is <= the previous rows' maximum plus the largest
// match score, so a row maximum above the profile's cap (32767 minus that
// score) marks the pair as passing before anything can wrap (sticky).
// Columns past M carry the floor scores; the profile's quantized image has
// the kernel's width G*C and the CPU model follows the same columns.
// ---------------------------------------------------------------------------
constexpr int kV16TFloor = -4096;    // -8 nats: lowest transition score (t_bm excepted)
constexpr int kV16BmFloor = -8192;   // -16 nats: lowest t_bm
constexpr int kV16EFloor = -4096;    // -8 nats: lowest match score, and columns past M
constexpr int kV16BFloor = -4096;    // -8 nats: lowest B state
constexpr unsigned kV16Init2 = 0xc000c000u;  // (-16384, -16384): -inf before row 1 / left of column 1
constexpr unsigned kV16Low2 = 0xa000a000u;   // (-24576, -24576): provisional D carry into a lane

// One profile x every nsub-th entry (from sub) of its Viterbi pre-screen list.
struct VitTile {
  int32_t p, sub, nsub, pad;
};

// int16x2 helpers: replace one half of a word by the same half of v.
__device__ __forceinline__ unsigned set_half(unsigned w, int h, unsigned v) {
  return h ? __byte_perm(w, v, 0x7610) : __byte_perm(w, v, 0x3254);
}

// Bound of pairs of one profile (tile.p) against the targets of its list
// (region (p - p0) * vcap of `vlist`, vcount[p - p0] entries).  The profile's
// quantized image (qv_off, uint4 units): 8 transition rows of W/4 uint4 (each
// column's score in both halves: t_mm t_im t_dm at k-1, t_bm t_mi t_ii at k,
// t_md t_dd at k-1), then 25 match-score rows of W/4 uint2 (4 columns of
// int16), both in the lane-major chunk layout of the f32 Viterbi image.
// Per pair: with `score_out`, the bound (f32 nats; +inf when capped, NaN for
// an empty target) goes to score_out[slot]; otherwise a pair whose bound
// passes F2 is appended to the exact Viterbi's list (bin vshape).  stats[0..2]
// accumulate the DP cells bounded, the cells of the passing pairs and the
// passing pairs.
template <int G, int C>
__global__ void __launch_bounds__(128, (C <= 8 ? 4 : 3)) vit16_kernel(
    const VitTile* __restrict__ tiles, const DevProfile* __restrict__ profs, const Thresholds* __restrict__ thr,
    const uint4* __restrict__ qvimg, const uint8_t* __restrict__ res, const int64_t* __restrict__ toff,
    const int32_t* __restrict__ tlen, const float4* __restrict__ xsc, const PairRec* __restrict__ vlist,
    unsigned vcap, const unsigned* __restrict__ vcount, int p0, PairRec* __restrict__ out,
    const BinRegion* __restrict__ out_bins, unsigned* __restrict__ out_counts, unsigned* __restrict__ overflow,
    float slack, float* __restrict__ score_out, double* __restrict__ stats) {
  static_assert(C % 4 == 0 && (G & (G - 1)) == 0 && G <= 32, "bad packed Viterbi shape");
  constexpr int NC4 = C / 4;
  constexpr int ROW4 = NC4 * G;  // uint4 per transition row, uint2 per score row
  static_assert(ROW4 % 2 == 0, "score rows must fill whole uint4");
  constexpr int NIMG4 = 8 * ROW4 + 25 * ROW4 / 2;
  extern __shared__ uint4 sm_v[];
  __shared__ unsigned s_next;
  const VitTile tile = tiles[blockIdx.x];
  const DevProfile P = profs[tile.p];
  {
    const uint4* src = qvimg + P.qv_off;
    for (int q = threadIdx.x; q < NIMG4; q += blockDim.x) sm_v[q] = src[q];
  }
  if (threadIdx.x == 0) s_next = 0;
  __syncthreads();
  const uint4* Ts = sm_v;
  const uint2* Es = reinterpret_cast<const uint2*>(sm_v + 8 * ROW4);

  const int lane = threadIdx.x & 31;
  const int j = lane & (G - 1);
  const int gl = lane - j;
  const unsigned gmask = (G == 32) ? kFull : (((1u << G) - 1u) << gl);
  const int pl = tile.p - p0;
  const unsigned n = min(vcount[pl], vcap);
  const PairRec* lst = vlist + (int64_t)pl * vcap;
  const int cap = P.qv_cap;
  const float s2 = thr[tile.p].s2;
  const int nln2 = (int)ceilf(-0.693147182464599609375f * 1048576.0f) + kQ32Rho;
  const uint4* tr = Ts + j;
  auto T = [&](int q, int c4) -> uint4 { return tr[(q * NC4 + c4) * G]; };
  auto pick = [](const uint4& v, int e) -> unsigned { return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w; };

  unsigned mp[C], ip[C], dp[C], pre[C];
#pragma unroll
  for (int c = 0; c < C; c++) mp[c] = ip[c] = dp[c] = pre[c] = kV16Init2;
  unsigned bw = kV16Init2;   // B of both halves for the row being computed
  unsigned dpl = kV16Init2;  // left lane's D at its last column, previous row
  // per half: pair state
  int L[2] = {0, 0}, row[2] = {0, 0}, boff[2] = {0, 0}, idx[2] = {0, 0};
  int xn[2] = {0, 0}, xj[2] = {kQ32Neg, kQ32Neg}, fin[2] = {kQ32Neg, kQ32Neg}, tl[2] = {0, 0}, tm[2] = {0, 0};
  bool act[2] = {false, false}, big[2] = {false, false}, dn[2] = {false, false};
  const uint8_t* seq[2] = {res, res};
  // residues: 16-byte words, the next one prefetched; wc = the current 4
  // bytes, consumed from the low byte up (targets are padded with '*' to a
  // 16-byte boundary and followed by 64 bytes of slack, so every byte read is
  // a valid residue code)
  uint4 rc[2], rn[2];
  uint32_t wc[2] = {0x18181818u, 0x18181818u};
#pragma unroll
  for (int h = 0; h < 2; h++) rc[h] = rn[h] = make_uint4(0x18181818u, 0x18181818u, 0x18181818u, 0x18181818u);
  double cells_in = 0.0, cells_pass = 0.0, npass = 0.0;

  for (;;) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (!dn[h] && row[h] >= L[h]) {  // group-uniform: finish this half's pair, take the next one
        if (act[h] && j == 0) {
          const PairRec r = lst[idx[h]];
          const float ub = L[h] == 0 ? __int_as_float(0x7fc00000)
                           : big[h]  ? __int_as_float(0x7f800000)
                                     : __fmul_rn(__int2float_ru(fin[h]), 9.5367431640625e-7f);
          if (score_out) {
            score_out[r.slot] = ub;
          } else if (L[h] > 0) {
            const double cells = (double)P.m * (double)L[h];
            cells_in += cells;
            if (big[h] || bits_stat(ub, r.filtersc) >= s2 - slack) {
              push_pair(r, P.vshape, out, out_bins, out_counts, overflow);
              cells_pass += cells;
              npass += 1.0;
            }
          }
        }
        unsigned k = 0;
        if (j == 0) k = atomicAdd(&s_next, 1u);
        k = __shfl_sync(gmask, k, gl);
        const unsigned e = (unsigned)tile.sub + k * (unsigned)tile.nsub;
        if (k < n && e < n) {
          idx[h] = (int)e;
          const int t = lst[e].t;
          L[h] = tlen[t];
          seq[h] = res + toff[t];
          const float4 xs = xsc[t];
          tl[h] = q32_up(xs.x);
          tm[h] = q32_up(xs.y);
          xn[h] = 0;
          xj[h] = kQ32Neg;
          fin[h] = kQ32Neg;
          big[h] = false;
          row[h] = 0;
          boff[h] = 0;
          rc[h] = __ldg(reinterpret_cast<const uint4*>(seq[h]));
          rn[h] = __ldg(reinterpret_cast<const uint4*>(seq[h] + 16));
          wc[h] = rc[h].x;
          act[h] = true;
#pragma unroll
          for (int c = 0; c < C; c++) {
            mp[c] = set_half(mp[c], h, kV16Init2);
            ip[c] = set_half(ip[c], h, kV16Init2);
            dp[c] = set_half(dp[c], h, kV16Init2);
            pre[c] = set_half(pre[c], h, kV16Init2);
          }
          dpl = set_half(dpl, h, kV16Init2);
          // B of row 1: xB = tmove
          const int b16 = max((tm[h] + 2047) >> (kQ32Shift - kQ16Shift), kV16BFloor);
          bw = set_half(bw, h, ((unsigned)b16 & 0xffffu) * 0x10001u);
        } else {
          act[h] = false;
          dn[h] = true;
          L[h] = 0;
        }
      }
    }
    if (__all_sync(kFull, dn[0] && dn[1])) break;

    // this row's residue of each half (idle halves compute on stale ones)
    int x[2];
#pragma unroll
    for (int h = 0; h < 2; h++) x[h] = (int)(wc[h] & 0xffu);
    // match scores of both halves, interleaved into words
    unsigned ew[C];
    {
      const uint2* ea = Es + x[0] * ROW4 + j;
      const uint2* eb = Es + x[1] * ROW4 + j;
#pragma unroll
      for (int c4 = 0; c4 < NC4; c4++) {
        const uint2 a = ea[c4 * G], b = eb[c4 * G];
        ew[4 * c4 + 0] = __byte_perm(a.x, b.x, 0x5410);
        ew[4 * c4 + 1] = __byte_perm(a.x, b.x, 0x7632);
        ew[4 * c4 + 2] = __byte_perm(a.y, b.y, 0x5410);
        ew[4 * c4 + 3] = __byte_perm(a.y, b.y, 0x7632);
      }
    }
    // ---- M: max(pre, D[k-1] + t_dm, B + t_bm) + msc (dp.rs:167-169) ----
#pragma unroll
    for (int c4 = 0; c4 < NC4; c4++) {
      const uint4 tdm = T(2, c4), tbm = T(3, c4);
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int c = 4 * c4 + e;
        const unsigned dpv = c ? dp[c - 1] : dpl;
        mp[c] = add2s16(max2s16(max2s16(pre[c], add2s16(dpv, pick(tdm, e))), add2s16(bw, pick(tbm, e))), ew[c]);
      }
    }
    // ---- D chain (ascending; provisional carry into lanes other than the
    // first), then the next row's pre and I (descending, in place) ----
    const unsigned mcl0 = __shfl_up_sync(kFull, mp[C - 1], 1, G);
    const unsigned ipl0 = __shfl_up_sync(kFull, ip[C - 1], 1, G);
    const unsigned mcl = j ? mcl0 : kV16Init2, ipl = j ? ipl0 : kV16Init2;
    {
      unsigned d = j ? kV16Low2 : kV16Init2;
#pragma unroll
      for (int c4 = 0; c4 < NC4; c4++) {
        const uint4 tmd = T(6, c4), tdd = T(7, c4);
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int c = 4 * c4 + e;
          const unsigned mcv = c ? mp[c - 1] : mcl;
          d = max2s16(add2s16(mcv, pick(tmd, e)), add2s16(d, pick(tdd, e)));
          dp[c] = d;
        }
      }
    }
#pragma unroll
    for (int c4 = NC4 - 1; c4 >= 0; c4--) {
      const uint4 tmm = T(0, c4), tim = T(1, c4), tmi = T(4, c4), tii = T(5, c4);
#pragma unroll
      for (int e = 3; e >= 0; e--) {
        const int c = 4 * c4 + e;
        const unsigned mpv = c ? mp[c - 1] : mcl, ipv = c ? ip[c - 1] : ipl;
        pre[c] = max2s16(add2s16(mpv, pick(tmm, e)), add2s16(ipv, pick(tim, e)));
        ip[c] = max2s16(add2s16(mp[c], pick(tmi, e)), add2s16(ip[c], pick(tii, e)));
      }
    }
    // ---- carries across the group's lanes until nothing changes (exact:
    // max-plus is monotone and the provisional carry is below every D) ----
    bool settled = false;
    for (int it = 0; it < G; it++) {
      const unsigned c0 = __shfl_up_sync(kFull, dp[C - 1], 1, G);
      unsigned cin = j ? c0 : kV16Init2;
      const unsigned tdd0 = T(7, 0).x;
      const bool need = max2s16(add2s16(cin, tdd0), dp[0]) != dp[0];
      if (!__any_sync(kFull, need)) {
        dpl = cin;
        settled = true;
        break;
      }
      bool go = true;
#pragma unroll
      for (int c4 = 0; c4 < NC4; c4++) {
        if (go) {
          const uint4 tdd = T(7, c4);
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const int c = 4 * c4 + e;
            if (go) {
              const unsigned nd = max2s16(dp[c], add2s16(cin, pick(tdd, e)));
              if (nd == dp[c]) {
                go = false;
              } else {
                dp[c] = nd;
                cin = nd;
              }
            }
          }
        }
      }
    }
    if (!settled) {
      const unsigned d0 = __shfl_up_sync(kFull, dp[C - 1], 1, G);
      dpl = j ? d0 : kV16Init2;
    }
    // ---- row maximum over M (D never exceeds it), per half ----
    unsigned tv[C];
#pragma unroll
    for (int c = 0; c < C; c++) tv[c] = mp[c];
#pragma unroll
    for (int span = 1; span < C; span <<= 1)
#pragma unroll
      for (int c = 0; c + span < C; c += 2 * span) tv[c] = max2s16(tv[c], tv[c + span]);
    unsigned xe = tv[0];
#pragma unroll
    for (int o = G / 2; o >= 1; o >>= 1) xe = max2s16(xe, __shfl_xor_sync(kFull, xe, o, G));
    // ---- special states per half (xC == xJ, as in the exact kernel) ----
    int b16[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int eh = h ? ((int)xe >> 16) : (int)(short)(xe & 0xffffu);
      big[h] |= eh > cap;
      xj[h] = max(xj[h] + tl[h], eh * 2048 + nln2);
      xn[h] += tl[h];
      const int xb = max(xn[h], xj[h]) + tm[h];
      b16[h] = max((xb + 2047) >> (kQ32Shift - kQ16Shift), kV16BFloor);
      row[h]++;
      if (row[h] == L[h]) fin[h] = xj[h] + tm[h];
      if ((row[h] & 3) == 0) {
        if (row[h] - boff[h] == 16) {
          boff[h] += 16;
          rc[h] = rn[h];
          if (act[h]) rn[h] = __ldg(reinterpret_cast<const uint4*>(seq[h] + boff[h] + 16));
        }
        const int q = (row[h] - boff[h]) >> 2;
        wc[h] = q == 0 ? rc[h].x : q == 1 ? rc[h].y : q == 2 ? rc[h].z : rc[h].w;
      } else {
        wc[h] >>= 8;
      }
    }
    bw = __byte_perm((unsigned)b16[0], (unsigned)b16[1], 0x5410);
  }
  // stats: one atomic per warp
  if (stats) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
      cells_in += __shfl_xor_sync(kFull, cells_in, o);
      cells_pass += __shfl_xor_sync(kFull, cells_pass, o);
      npass += __shfl_xor_sync(kFull, npass, o);
    }
    if (lane == 0 && cells_in != 0.0) {
      atomicAdd(stats + 0, cells_in);
      atomicAdd(stats + 1, cells_pass);
      atomicAdd(stats + 2, npass);
    }
  }
}

}  // namespace sxk
