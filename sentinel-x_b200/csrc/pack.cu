// Kernel-shape choice, the device images of profiles and targets, and the
// per-profile filter thresholds of a search.
#include "engine.hpp"
#include "long.cuh"
#include "tuned_shapes.inc"

namespace sxe {


// Pick the MSV shape with the fewest issued instructions per useful DP cell.
// Per row a warp issues about 2.75*C instructions of cell work (FADD, FMNMX,
// a share of FMNMX3 and LDS.128) plus ~44 of per-row overhead (residue
// extraction, shuffles, specials) and 2 per butterfly step; it advances 32/G
// targets by M cells each (fitted to ncu instruction counts on B200).
int choose_msv_shape(int m) {
  int best = -1;
  double best_cost = 1e30;
  for (int s = 0; s < kNumMsvShapes; s++) {
    const int g = kMsvShapes[s].g, c = kMsvShapes[s].c;
    if (g * c < m) continue;
    const double instr = 2.75 * c + 44.0 + 2.0 * std::log2((double)g);
    const double cost = instr / ((32.0 / g) * m);
    if (cost < best_cost * 0.999) {
      best_cost = cost;
      best = s;
    }
  }
  return best;
}
// Viterbi shape: per row a lane does ~19 instructions per column (16 lane-ops
// plus 9 loads per 4 columns) and ~50 of overhead; lanes per pair cost
// lazy-F carry rounds and butterfly steps; C >= 24 halves occupancy.
int choose_vit_shape(int m) {
  int best = -1;
  double best_cost = 1e30;
  for (int s = 0; s < kNumVitShapes; s++) {
    const int g = kVitShapes[s].g, c = kVitShapes[s].c;
    if (g * c < m) continue;
    // per-row lane instructions; register-held transitions save the 8 loads per 4 columns
    const double per_row = (kVitShapes[s].rt ? 9.0 : 19.0) * c + 50.0 + 12.0 * std::log2((double)g);
    const double occ = vit_ctas_per_sm(kVitShapes[s]) == 2 ? 1.0 : 0.5;
    const double cost = per_row * g / (32.0 * m) / occ;
    if (cost < best_cost * 0.999) {
      best_cost = cost;
      best = s;
    }
  }
  return best;
}
// Persistent grid for a lane-group Viterbi launch of `n` pairs: the CTAs that
// fit on the GPU at once (two per SM for C <= 16, whose registers are capped
// at 128, one otherwise), fewer if the pairs need fewer groups.
int vit_blocks(int num_sms, int shape, unsigned n) {
  const int g = kVitShapes[shape].g, per_sm = vit_ctas_per_sm(kVitShapes[shape]);
  return (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)n * g + 255) / 256, (int64_t)num_sms * per_sm));
}

// Packed Viterbi pre-screen shape of a profile: the narrowest that covers M;
// -1 when none does.
int choose_vit16_shape(int m) {
  for (int s = 0; s < kNumVit16Shapes; s++)
    if (kVit16Shapes[s].g * kVit16Shapes[s].c >= m) return s;
  return -1;
}

// Forward/Backward pass kernels run one warp per pair in one-warp CTAs, so a
// warp that finishes frees its SM slot at once instead of holding it until
// the longest pair of a larger CTA is done.
int warp_ctas(int num_sms, unsigned n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)n, (int64_t)num_sms * 32));
}

int choose_vbin(int m) {
  const int need = (m + 31) / 32;
  for (int b = 0; b < kNumVbins; b++)
    if (kVcBins[b] >= need) return b;
  return -1;
}


// The built-in shape table of a kind: for Viterbi the shapes measured fastest
// per range of M on B200 (tuned_shapes.inc, written by sxhmm/tune.py); none for
// MSV, whose cost model was fitted to ncu instruction counts.
std::vector<int16_t> default_shape_table(int kind) {
  std::vector<int16_t> t;
  if (kind != 1) return t;
  t.assign(kMaxM + 1, -1);
  for (const auto& r : kTunedVit) {
    int idx = -1;
    for (int s = 0; s < kNumVitShapes; s++)
      if (kVitShapes[s].g == r[2] && kVitShapes[s].c == r[3] && kVitShapes[s].rt == r[4]) idx = s;
    if (idx < 0 || kVitShapes[idx].g * kVitShapes[idx].c < r[1]) continue;
    for (int m = std::max(r[0], 0); m <= r[1] && m <= kMaxM; m++) t[(size_t)m] = (int16_t)idx;
  }
  return t;
}

// Kernel shape for a profile of length m: the engine's table where it has an
// entry, else the cost model (kind 0 MSV, 1 Viterbi).
int shape_for(const sx_engine* E, int kind, int m) {
  const auto& t = E->shape_table[kind];
  if (m >= 0 && (size_t)m < t.size() && t[(size_t)m] >= 0) return t[(size_t)m];
  return kind == 0 ? choose_msv_shape(m) : choose_vit_shape(m);
}

// ---- profile packing --------------------------------------------------------
// The images of a profile the warp-chunked and lane-group kernels read.
void pack_images(const ProfileHost& h, const DevProfile& d, float4* msv, float4* vit, float* vfb) {
  const int m = h.m;
  // MSV image: residue row x, float4 chunk c4 of lane j at (x*NC4 + c4)*G + j;
  // lane j's column c is k = j*C + c + 1.
  {
    const int G = d.msv_g, C = d.msv_c, NC4 = C / 4;
    float4* base = msv + d.msv_off;
    for (int x = 0; x < 25; x++)
      for (int j = 0; j < G; j++)
        for (int c4 = 0; c4 < NC4; c4++) {
          float v[4];
          for (int e = 0; e < 4; e++) {
            const int k = j * C + c4 * 4 + e + 1;
            v[e] = k <= m ? h.msc_row(x)[k] : kNegInf;
          }
          base[((size_t)x * NC4 + c4) * G + j] = make_float4(v[0], v[1], v[2], v[3]);
        }
  }
  // Viterbi image: rows 0..24 log-odds, 25..32 transitions (mm im dm at k-1, bm mi ii at k,
  // md dd at k-1), lane-major float4 chunks as for MSV
  {
    const int G = kVitShapes[d.vshape].g, C = kVitShapes[d.vshape].c, NC4 = C / 4;
    float4* base = vit + d.vit_off;
    auto row = [&](int r, const std::function<float(int)>& f, float pad) {
      for (int j = 0; j < G; j++)
        for (int c4 = 0; c4 < NC4; c4++) {
          float v[4];
          for (int e = 0; e < 4; e++) {
            const int k = j * C + c4 * 4 + e + 1;
            v[e] = k <= m ? f(k) : pad;
          }
          base[((size_t)r * NC4 + c4) * G + j] = make_float4(v[0], v[1], v[2], v[3]);
        }
    };
    for (int x = 0; x < 25; x++) row(x, [&](int k) { return h.msc_row(x)[k]; }, kNegInf);
    const auto& t = h.t;
    row(25, [&](int k) { return t[TMM][k - 1]; }, kNegInf);
    row(26, [&](int k) { return t[TIM][k - 1]; }, kNegInf);
    row(27, [&](int k) { return t[TDM][k - 1]; }, kNegInf);
    row(28, [&](int k) { return t[TBM][k]; }, kNegInf);
    // no insert state at node M: -inf from k = M on keeps I_M.. at -inf
    row(29, [&](int k) { return k < m ? t[TMI][k] : kNegInf; }, kNegInf);
    row(30, [&](int k) { return k < m ? t[TII][k] : kNegInf; }, kNegInf);
    row(31, [&](int k) { return t[TMD][k - 1]; }, kNegInf);
    row(32, [&](int k) { return t[TDD][k - 1]; }, kNegInf);
  }
  // warp-chunked image: row r, lane l, column c (k = l*vc + c + 1) at (r*vc + c)*32 + l
  {
    const int vc = d.vc;
    float* base = vfb + d.vfb_off;
    auto put = [&](int r, const std::function<float(int)>& f, float pad) {
      for (int l = 0; l < 32; l++)
        for (int c = 0; c < vc; c++) {
          const int k = l * vc + c + 1;
          base[((size_t)r * vc + c) * 32 + l] = k <= m ? f(k) : pad;
        }
    };
    for (int x = 0; x < 25; x++) {
      put(sxk::kRowMsc + x, [&](int k) { return h.msc_row(x)[k]; }, kNegInf);
      put(sxk::kRowMo + x, [&](int k) { return h.mo_row(x)[k]; }, 0.0f);
    }
    const auto& t = h.t;
    const auto& p = h.p;
    auto shl = [&](const std::vector<float>& v) { return [&v](int k) { return v[k - 1]; }; };
    auto at = [&](const std::vector<float>& v) { return [&v](int k) { return v[k]; }; };
    put(sxk::kRowVit + 0, shl(t[TMM]), kNegInf);
    put(sxk::kRowVit + 1, shl(t[TIM]), kNegInf);
    put(sxk::kRowVit + 2, shl(t[TDM]), kNegInf);
    put(sxk::kRowVit + 3, at(t[TBM]), kNegInf);
    put(sxk::kRowVit + 4, at(t[TMI]), kNegInf);
    put(sxk::kRowVit + 5, at(t[TII]), kNegInf);
    put(sxk::kRowVit + 6, shl(t[TMD]), kNegInf);
    put(sxk::kRowVit + 7, shl(t[TDD]), kNegInf);
    put(sxk::kRowFwd + 0, at(p[TBM]), 0.0f);
    put(sxk::kRowFwd + 1, shl(p[TMM]), 0.0f);
    put(sxk::kRowFwd + 2, shl(p[TIM]), 0.0f);
    put(sxk::kRowFwd + 3, shl(p[TDM]), 0.0f);
    put(sxk::kRowFwd + 4, at(p[TMI]), 0.0f);
    put(sxk::kRowFwd + 5, at(p[TII]), 0.0f);
    put(sxk::kRowFwd + 6, shl(p[TMD]), 0.0f);
    put(sxk::kRowFwd + 7, shl(p[TDD]), 0.0f);
    put(sxk::kRowBwd + 0, at(p[TMM]), 0.0f);
    put(sxk::kRowBwd + 1, at(p[TMI]), 0.0f);
    put(sxk::kRowBwd + 2, at(p[TMD]), 0.0f);
    put(sxk::kRowBwd + 3, at(p[TIM]), 0.0f);
    put(sxk::kRowBwd + 4, at(p[TII]), 0.0f);
    put(sxk::kRowBwd + 5, at(p[TDM]), 0.0f);
    put(sxk::kRowBwd + 6, at(p[TDD]), 0.0f);
    put(sxk::kRowBwd + 7, at(p[TBM]), 0.0f);
  }
}

// Quantized MSV image of the packed pre-screen (prescreen.cuh): the match
// scores in units of 2^-9 nat rounded up after adding 2^-12 nat, clamped up to
// -16 nats (-inf included), -32 nats past column M, in the lane-major chunk
// layout of the profile's f32 MSV image (4 columns per uint2).  Returns the
// largest rounded score of a real column; the profile's cap is 32767 minus it.
int pack_qimage(const ProfileHost& h, const DevProfile& d, uint2* out) {
  const int m = h.m, G = d.msv_g, C = d.msv_c, NC4 = C / 4;
  int emax = sxk::kQ16EFloor;
  auto q = [&](int x, int k) -> int {
    if (k > m) return sxk::kQ16EPad;
    const float e = h.msc_row(x)[k];
    if (!(e > -1e30f)) return sxk::kQ16EFloor;  // -inf (and NaN, which no configured profile has)
    const double u = std::ceil(((double)e + std::ldexp(1.0, -12)) * 512.0);
    const int v = (int)std::max<double>(u, (double)sxk::kQ16EFloor);
    emax = std::max(emax, v);
    return v;
  };
  uint2* base = out + d.q_off;
  for (int x = 0; x < 25; x++)
    for (int j = 0; j < G; j++)
      for (int c4 = 0; c4 < NC4; c4++) {
        int v[4];
        for (int e = 0; e < 4; e++) v[e] = q(x, j * C + c4 * 4 + e + 1);
        uint2 w;
        w.x = (uint32_t)(v[0] & 0xffff) | ((uint32_t)(v[1] & 0xffff) << 16);
        w.y = (uint32_t)(v[2] & 0xffff) | ((uint32_t)(v[3] & 0xffff) << 16);
        base[((size_t)x * NC4 + c4) * G + j] = w;
      }
  return emax;
}

// Quantized Viterbi image of the packed pre-screen (prescreen.cuh
// vit16_kernel), in units of 2^-9 nat: every score rounded up after adding
// 2^-12 nat; match scores clamped up to -8 nats, transitions clamped to
// [-8 nats, 0] (t_bm to [-16 nats, 0]); -inf scores and columns past M take
// the floor.  8 transition rows (each column's score in both int16 halves of
// a word, 4 columns per uint4), then 25 match-score rows (4 columns per
// uint2), lane-major like the f32 Viterbi image, at width G*C of the
// profile's pre-screen shape.  Returns the largest rounded match score.
int pack_qvimage(const ProfileHost& h, const DevProfile& d, uint4* out) {
  const int m = h.m, G = kVit16Shapes[d.qv_shape].g, C = kVit16Shapes[d.qv_shape].c, NC4 = C / 4;
  auto up = [](float v) { return std::ceil(((double)v + std::ldexp(1.0, -12)) * 512.0); };
  int emax = sxk::kV16EFloor;
  auto em = [&](int x, int k) -> int {
    if (k > m) return sxk::kV16EFloor;
    const float e = h.msc_row(x)[k];
    if (!(e > -1e30f)) return sxk::kV16EFloor;
    const int v = (int)std::max<double>(up(e), (double)sxk::kV16EFloor);
    emax = std::max(emax, v);
    return v;
  };
  auto tq = [&](float t, int floor) -> int {
    if (!(t > -1e30f)) return floor;
    return (int)std::max<double>(std::min<double>(up(t), 0.0), (double)floor);
  };
  const auto& t = h.t;
  // transition row q of column k (the f32 Viterbi image's rows 25..32)
  auto tr = [&](int q, int k) -> int {
    if (k > m) return q == 3 ? sxk::kV16BmFloor : sxk::kV16TFloor;
    switch (q) {
      case 0: return tq(t[TMM][k - 1], sxk::kV16TFloor);
      case 1: return tq(t[TIM][k - 1], sxk::kV16TFloor);
      case 2: return tq(t[TDM][k - 1], sxk::kV16TFloor);
      case 3: return tq(t[TBM][k], sxk::kV16BmFloor);
      case 4: return k < m ? tq(t[TMI][k], sxk::kV16TFloor) : sxk::kV16TFloor;
      case 5: return k < m ? tq(t[TII][k], sxk::kV16TFloor) : sxk::kV16TFloor;
      case 6: return tq(t[TMD][k - 1], sxk::kV16TFloor);
      default: return tq(t[TDD][k - 1], sxk::kV16TFloor);
    }
  };
  auto dup = [](int v) { return ((uint32_t)v & 0xffffu) * 0x10001u; };
  uint4* base = out + d.qv_off;
  const size_t row4 = (size_t)NC4 * G;
  for (int q = 0; q < 8; q++)
    for (int j = 0; j < G; j++)
      for (int c4 = 0; c4 < NC4; c4++) {
        const int k = j * C + c4 * 4 + 1;
        base[(q * NC4 + c4) * G + j] = make_uint4(dup(tr(q, k)), dup(tr(q, k + 1)), dup(tr(q, k + 2)), dup(tr(q, k + 3)));
      }
  uint2* es = reinterpret_cast<uint2*>(base + 8 * row4);
  for (int x = 0; x < 25; x++)
    for (int j = 0; j < G; j++)
      for (int c4 = 0; c4 < NC4; c4++) {
        int v[4];
        for (int e = 0; e < 4; e++) v[e] = em(x, j * C + c4 * 4 + e + 1);
        uint2 w;
        w.x = (uint32_t)(v[0] & 0xffff) | ((uint32_t)(v[1] & 0xffff) << 16);
        w.y = (uint32_t)(v[2] & 0xffff) | ((uint32_t)(v[3] & 0xffff) << 16);
        es[((size_t)x * NC4 + c4) * G + j] = w;
      }
  return emax;
}
// uint4 entries of a quantized Viterbi image of shape s
int64_t qvimage_size(int s) {
  const int64_t row4 = (int64_t)(kVit16Shapes[s].c / 4) * kVit16Shapes[s].g;
  return 8 * row4 + 25 * row4 / 2;
}

// Composition-bias filter table (src/hmmer/pipeline.rs:110-131): 54 doubles.
void pack_bias(const ProfileHost& h, double* b) {
  const int m = h.m;
  for (int x = 0; x < 25; x++) b[x] = b[25 + x] = 1.0;
  for (int x = 0; x < NRES; x++) b[25 + x] = (double)h.compo[x] / (double)kBackground[x];
  for (int code = 20; code <= 23; code++) {
    const Degenerate& dg = degenerate(code);
    double e0 = 0, e1 = 0, z = 0;
    for (int q = 0; q < dg.n; q++) {
      e0 += (double)kBackground[dg.members[q]];
      e1 += (double)h.compo[dg.members[q]];
      z += (double)kBackground[dg.members[q]];
    }
    b[code] = e0 / z;
    b[25 + code] = e1 / z;
  }
  const double l0 = 400.0, l1 = (double)m / 8.0;
  b[50] = l0 / (l0 + 1.0);
  b[51] = 1.0 / (l0 + 1.0);
  b[52] = 1.0 / (l1 + 1.0);
  b[53] = l1 / (l1 + 1.0);
}

void pack_profiles(sx_profiles* P) {
  const size_t np = P->h.size();
  P->dp.resize(np);
  P->msv_shape.resize(np);
  int64_t msv_total = 0, vfb_total = 0, vit_total = 0, q_total = 0, qv_total = 0;
  for (size_t i = 0; i < np; i++) {
    const ProfileHost& h = P->h[i];
    DevProfile& d = P->dp[i];
    memset(&d, 0, sizeof d);
    d.m = h.m;
    d.msv_tbm = h.msv_tbm;
    if (is_long(h.m)) {  // no warp-chunked, MSV or Viterbi images: the long kernels read the plain image
      P->msv_shape[i] = -1;
      d.vbin = d.vshape = -1;
      d.msv_off = msv_total;
      d.vfb_off = vfb_total;
      d.vit_off = vit_total;
      d.q_off = -1;
      d.qv_shape = -1;
      d.qv_off = -1;
      continue;
    }
    const int s = shape_for(P->eng, 0, h.m);
    const int vb = choose_vbin(h.m);
    if (s < 0 || vb < 0) throw CudaError{SX_EINVAL, "profile '" + h.name + "': no kernel shape for M=" + std::to_string(h.m)};
    P->msv_shape[i] = s;
    d.msv_g = kMsvShapes[s].g;
    d.msv_c = kMsvShapes[s].c;
    d.vbin = vb;
    d.vc = kVcBins[vb];
    d.msv_off = msv_total;
    msv_total += 25LL * (d.msv_c / 4) * d.msv_g;
    d.q_off = q_total;
    q_total += 25LL * (d.msv_c / 4) * d.msv_g;
    d.q_tbm = (int32_t)std::ceil(((double)h.msv_tbm + std::ldexp(1.0, -17)) * 1048576.0);
    d.vfb_off = vfb_total;
    vfb_total += (int64_t)sxk::kImgRows * 32 * d.vc;
    d.vshape = shape_for(P->eng, 1, h.m);
    if (d.vshape < 0) throw CudaError{SX_EINVAL, "profile '" + h.name + "' too long for the Viterbi shapes"};
    d.vit_off = vit_total;
    vit_total += 33LL * (kVitShapes[d.vshape].c / 4) * kVitShapes[d.vshape].g;
    d.qv_shape = choose_vit16_shape(h.m);
    d.qv_off = -1;
    if (d.qv_shape >= 0) {
      d.qv_off = qv_total;
      qv_total += qvimage_size(d.qv_shape);
    }
  }
  std::vector<float4> msv((size_t)msv_total);
  std::vector<float4> vit((size_t)std::max<int64_t>(vit_total, 1));
  std::vector<float> vfb((size_t)vfb_total);
  std::vector<double> bias(np * 54);
  std::vector<uint2> qimg((size_t)std::max<int64_t>(q_total, 1));
  std::vector<uint4> qvimg((size_t)std::max<int64_t>(qv_total, 1));
  for (size_t i = 0; i < np; i++) {
    if (P->dp[i].vbin >= 0) {
      pack_images(P->h[i], P->dp[i], msv.data(), vit.data(), vfb.data());
      // a profile whose rounded scores leave less than half of the int16
      // range as headroom (scores above +16 nats) stays on the exact kernel
      const int emax = pack_qimage(P->h[i], P->dp[i], qimg.data());
      if (emax < 8192) P->dp[i].q_cap = 32767 - emax;
      else P->dp[i].q_off = -1;
      // the Viterbi pre-screen takes the MSV pre-screen's profiles (whose
      // bias-filter survivors fit the per-profile lists of the MSV rescoring)
      // whose rounded match scores leave at least half of the int16 range
      DevProfile& d = P->dp[i];
      if (d.qv_shape >= 0 && d.q_off >= 0) {
        const int vmax = pack_qvimage(P->h[i], d, qvimg.data());
        if (vmax < 8192) d.qv_cap = 32767 - vmax;
        else d.qv_shape = -1;
      } else {
        d.qv_shape = -1;
      }
    }
    pack_bias(P->h[i], bias.data() + i * 54);
  }
  // plain layout: 25 msc rows then mm mi md im ii dm dd bm, each M+1 long;
  // long profiles add the 25 odds rows and the 8 probability rows (same order),
  // the image of the long kernels
  std::vector<sxk::PlainProfile> pprof(np);
  int64_t plain_total = 0;
  for (size_t i = 0; i < np; i++) {
    pprof[i].off = plain_total;
    pprof[i].m = P->h[i].m;
    pprof[i].pad = 0;
    plain_total += (is_long(P->h[i].m) ? (int64_t)sxk::kLongRows : 33LL) * (P->h[i].m + 1);
  }
  std::vector<float> plain((size_t)std::max<int64_t>(plain_total, 1));
  for (size_t i = 0; i < np; i++) {
    const ProfileHost& h = P->h[i];
    const size_t w = (size_t)h.m + 1;
    float* b = plain.data() + pprof[i].off;
    memcpy(b, h.msc.data(), sizeof(float) * 25 * w);
    const int order[8] = {TMM, TMI, TMD, TIM, TII, TDM, TDD, TBM};
    for (int q = 0; q < 8; q++) memcpy(b + (25 + q) * w, h.t[order[q]].data(), sizeof(float) * w);
    if (is_long(h.m)) {
      memcpy(b + sxk::kLMo * w, h.mo.data(), sizeof(float) * 25 * w);
      for (int q = 0; q < 8; q++) memcpy(b + (sxk::kLP + q) * w, h.p[order[q]].data(), sizeof(float) * w);
    }
  }
  cudaStream_t s = P->eng->stream;
  P->d_pprof.upload(pprof.data(), np, s);
  P->d_plain.upload(plain.data(), plain.size(), s);
  P->d_prof.upload(P->dp.data(), np, s);
  P->d_msv.upload(msv.data(), msv.size(), s);
  P->d_qimg.upload(qimg.data(), qimg.size(), s);
  P->d_qvimg.upload(qvimg.data(), qvimg.size(), s);
  P->d_vit.upload(vit.data(), vit.size(), s);
  P->d_vfb.upload(vfb.data(), vfb.size(), s);
  P->d_bias.upload(bias.data(), bias.size(), s);
  CK(cudaStreamSynchronize(s));
}

// ---- target packing ---------------------------------------------------------
void pack_targets(sx_targets* T) {
  const size_t n = T->len.size();
  std::vector<float4> tpar(n), xsc(n);
  T->residues = 0;
  // the length constants depend on L alone: computed once per distinct length
  std::unordered_map<int64_t, std::pair<float4, float4>> by_len;
  for (size_t i = 0; i < n; i++) {
    const int64_t l = T->len[i];
    auto it = by_len.find(l);
    if (it == by_len.end()) {
      const float lf = (float)l;
      // MSV length model (src/hmmer/dp.rs:98-100) and the multihit Xsc (model.rs:284-312)
      const float tloop = std::log(lf / (lf + 3.0f));
      const float tmove = std::log(3.0f / (lf + 3.0f));
      const SpecialTr st = special_transitions(l, true);
      it = by_len.emplace(l, std::make_pair(make_float4(tloop, tmove, null1_score(l), 0.0f),
                                            make_float4(st.loop, st.move, st.ploop, st.pmove))).first;
    }
    tpar[i] = it->second.first;
    xsc[i] = it->second.second;
    T->residues += (double)l;
  }
  // indices by length, longest first, ties in input order (a counting sort
  // when the lengths allow one)
  T->order.resize(n);
  int32_t mx = 0;
  for (size_t i = 0; i < n; i++) mx = std::max(mx, T->len[i]);
  if (mx <= (1 << 22)) {
    std::vector<int32_t> start((size_t)mx + 2, 0);
    for (size_t i = 0; i < n; i++) start[(size_t)(mx - T->len[i]) + 1]++;
    for (size_t k = 1; k < start.size(); k++) start[k] += start[k - 1];
    for (size_t i = 0; i < n; i++) T->order[(size_t)start[(size_t)(mx - T->len[i])]++] = (int32_t)i;
  } else {
    std::iota(T->order.begin(), T->order.end(), 0);
    std::stable_sort(T->order.begin(), T->order.end(), [&](int a, int b) { return T->len[a] > T->len[b]; });
  }
  cudaStream_t s = T->eng->stream;
  // all arrays in one pooled block, each 256-byte aligned
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t o_res = 0, o_off = o_res + up(T->dsq.size()), o_len = o_off + up(8 * n), o_tpar = o_len + up(4 * n);
  const size_t o_xsc = o_tpar + up(16 * n), o_order = o_xsc + up(16 * n), total = o_order + up(4 * n);
  if (T->block) T->eng->target_blocks.give(T->block, T->block_bytes);
  T->block = T->eng->target_blocks.take(total, T->block_bytes);
  char* b = static_cast<char*>(T->block);
  T->d_res.view(b + o_res, T->dsq.size());
  T->d_off.view(b + o_off, n);
  T->d_len.view(b + o_len, n);
  T->d_tpar.view(b + o_tpar, n);
  T->d_xsc.view(b + o_xsc, n);
  T->d_order.view(b + o_order, n);
  auto put = [&](void* dst, const void* src, size_t bytes) {
    if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
  };
  put(T->d_res.p, T->dsq.data(), T->dsq.size());
  put(T->d_off.p, T->off.data(), 8 * n);
  put(T->d_len.p, T->len.data(), 4 * n);
  put(T->d_tpar.p, tpar.data(), 16 * n);
  put(T->d_xsc.p, xsc.data(), 16 * n);
  put(T->d_order.p, T->order.data(), 4 * n);
  CK(cudaStreamSynchronize(s));
}

void append_target(sx_targets* T, const uint8_t* dig, size_t l) {
  const int64_t o = (int64_t)T->dsq.size();
  T->off.push_back(o);
  T->len.push_back((int32_t)l);
  T->dsq.insert(T->dsq.end(), dig, dig + l);
  // pad to a 16-byte boundary; kernels read up to 48 bytes past a target
  size_t padded = (T->dsq.size() + 15) & ~(size_t)15;
  T->dsq.resize(padded, SYM_STAR);
}

// ---- thresholds ---------------------------------------------------------------
// Per profile, the smallest f32 bit statistic that passes each filter
// (pipeline.rs:164-183).  The tails are monotone in the statistic, except the
// Gumbel survival around its branch at 1e-5; a threshold within 2% of that
// point disables device filtering for the stage (the host still decides).
std::vector<Thresholds> make_thresholds(const std::vector<ProfileHost>& H, const SearchOpts& o) {
  std::vector<Thresholds> th(H.size());
  auto near_branch = [](double f) { return f > 0.98e-5 && f < 1.02e-5; };
  for (size_t i = 0; i < H.size(); i++) {
    const ProfileHost& h = H[i];
    Thresholds& t = th[i];
    if (!o.filters || !h.calibrated()) {
      t.s1 = t.s2 = t.s3 = -INFINITY;
      t.exact = 0;
      continue;
    }
    t.exact = 1;
    const double mmu = h.msv[0], mlam = h.msv[1], vmu = h.vit[0], vlam = h.vit[1], ftau = h.fwd[0], flam = h.fwd[1];
    t.s1 = near_branch(o.f1) ? -INFINITY : f32_boundary([&](float s) { return !(gumbel_survival((double)s, mmu, mlam) > o.f1); });
    t.s2 = near_branch(o.f2) ? -INFINITY : f32_boundary([&](float s) { return !(gumbel_survival((double)s, vmu, vlam) > o.f2); });
    t.s3 = f32_boundary([&](float s) { return !(std::exp(exp_tail_logsurv((double)s, ftau, flam)) > o.f3); });
    if (std::isnan(t.s1)) t.s1 = -INFINITY;
    if (std::isnan(t.s2)) t.s2 = -INFINITY;
    if (std::isnan(t.s3)) t.s3 = -INFINITY;
  }
  return th;
}

}  // namespace sxe
