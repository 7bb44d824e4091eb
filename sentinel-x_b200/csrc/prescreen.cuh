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
