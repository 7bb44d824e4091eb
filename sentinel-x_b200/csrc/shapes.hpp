// Kernel shapes compiled into the library and the per-shape launch tables.
//
// The template instantiations live in their own translation units
// (k_msv.cu, k_msv16.cu, k_vit.cu, k_vit16.cu, k_vbin.cu, k_env.cu) so the library builds in
// parallel; the host translation units launch them through the function-pointer tables
// filled here.
#pragma once
#include <cstdint>

#include "kernels.cuh"
#include "adjoint.cuh"
#include "envelope.cuh"
#include "prescreen.cuh"

namespace sx {

using sxk::BinRegion;
using sxk::DevProfile;
using sxk::MsvTile;
using sxk::PairRec;
using sxk::Thresholds;

// MSV (G lanes per target, C columns per lane) shapes compiled into the library.
struct MsvShape {
  int g, c;
};
constexpr MsvShape kMsvShapes[] = {
    {1, 8}, {1, 16}, {1, 24}, {1, 32}, {1, 40}, {1, 48}, {1, 56}, {1, 64},
    {2, 8}, {2, 16}, {2, 24}, {2, 32}, {2, 40}, {2, 48}, {2, 56}, {2, 64},
    {4, 8}, {4, 16}, {4, 24}, {4, 32}, {4, 40}, {4, 48}, {4, 56}, {4, 64},
    {8, 8}, {8, 16}, {8, 24}, {8, 32}, {8, 40}, {8, 48}, {8, 56}, {8, 64},
    {16, 8}, {16, 16}, {16, 24}, {16, 32}, {16, 40}, {16, 48}, {16, 56}, {16, 64},
    {32, 8}, {32, 16}, {32, 24}, {32, 32}, {32, 40}, {32, 48}, {32, 56}, {32, 64},
    // intermediate widths for the common range of M: half the column padding
    {2, 36}, {2, 44}, {2, 52}, {2, 60}, {4, 36}, {4, 44}, {4, 52}, {4, 60},
    {8, 36}, {8, 44}, {8, 52}, {8, 60}};
constexpr int kNumMsvShapes = sizeof(kMsvShapes) / sizeof(kMsvShapes[0]);
constexpr int kMaxM = 2048;  // columns of the warp-chunked and lane-group kernels
// Longer profiles (marker models of long proteins) run through the long kernels.
inline bool is_long(int m) { return m > kMaxM; }
// Viterbi lane-group shapes: G lanes per pair, C columns per lane, rt = the
// transition rows held in registers for the whole pair (C <= 16).
struct VitShape {
  int g, c, rt;
};
constexpr VitShape kVitShapes[] = {{1, 8, 0},   {2, 8, 0},   {4, 8, 0},   {8, 8, 0},   {16, 8, 0},  {32, 8, 0},
                                   {1, 16, 0},  {2, 16, 0},  {4, 16, 0},  {8, 16, 0},  {16, 16, 0}, {32, 16, 0},
                                   {4, 24, 0},  {8, 24, 0},  {16, 24, 0}, {32, 24, 0}, {32, 32, 0}, {32, 48, 0},
                                   {32, 64, 0}, {4, 8, 1},   {8, 8, 1},   {16, 8, 1},  {32, 8, 1},  {32, 16, 1}};
// CTAs of one shape resident per SM: registers are capped at 128 for C <= 16
// (two 256-thread CTAs) except with 16 register-held transition columns.
constexpr int vit_ctas_per_sm(const VitShape& v) { return (v.c <= 16 && !(v.rt && v.c > 8)) ? 2 : 1; }
constexpr int kNumVitShapes = sizeof(kVitShapes) / sizeof(kVitShapes[0]);
constexpr int kMaxBins = 32;  // survivor lists per stage (vbins or Viterbi shapes)
static_assert(kNumVitShapes <= kMaxBins, "too many Viterbi shapes");

// Packed Viterbi pre-screen shapes (prescreen.cuh vit16_kernel): G lanes per
// pair of targets, C columns per lane; a profile takes the narrowest that
// covers M, profiles wider than the last one are not pre-screened.  Above 64
// columns 16 columns a lane beat 8 (Viterbi pre-screen of the Pfam-scale
// search 65 -> 59 ms): the row's per-lane overhead is shared by twice the
// cells, at 163 registers and three 128-thread CTAs per SM.
struct Vit16Shape {
  int g, c;
};
constexpr Vit16Shape kVit16Shapes[] = {{4, 8}, {8, 8}, {8, 16}, {16, 16}, {32, 16}};
constexpr int kNumVit16Shapes = sizeof(kVit16Shapes) / sizeof(kVit16Shapes[0]);
// dynamic shared memory of one tile: 8 transition rows of 4 bytes per column
// and 25 score rows of 2 bytes per column
constexpr int vit16_smem(const Vit16Shape& v) { return 82 * v.g * v.c; }
// threads per CTA: the kernel's launch bounds give 128 registers a thread
// for C <= 8 (four 128-thread CTAs per SM), 168 for C = 16 (three)
constexpr int vit16_threads(const Vit16Shape&) { return 128; }

// Warp-chunked column counts (columns per lane, 32 lanes per pair).
constexpr int kVcBins[] = {1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64};
constexpr int kNumVbins = sizeof(kVcBins) / sizeof(kVcBins[0]);

typedef void (*MsvFn)(const MsvTile*, const DevProfile*, const Thresholds*, const float4*, const uint8_t*,
                      const int64_t*, const int32_t*, const float4*, const int32_t*, float*, const int32_t*, PairRec*,
                      const BinRegion*, unsigned*, unsigned*, const unsigned*, unsigned, int);
typedef void (*Msv16Fn)(const sxk::PackedTile*, const DevProfile*, const Thresholds*, const uint2*, const uint8_t*,
                        const int64_t*, const int32_t*, const float4*, const int32_t*, int32_t*, unsigned, unsigned*,
                        int, unsigned*, float*, const int32_t*, int64_t);
typedef void (*Vit16Fn)(const sxk::VitTile*, const DevProfile*, const Thresholds*, const uint4*, const uint8_t*,
                        const int64_t*, const int32_t*, const float4*, const PairRec*, unsigned, const unsigned*, int,
                        PairRec*, const BinRegion*, unsigned*, unsigned*, float, float*, double*);
typedef void (*VitFn)(const PairRec*, const unsigned*, const BinRegion*, int, PairRec*, const BinRegion*, unsigned*,
                      unsigned*, const DevProfile*, const Thresholds*, const float*, const uint8_t*, const int64_t*,
                      const int32_t*, const float4*, float, float*);
typedef void (*VitGFn)(const PairRec*, const unsigned*, const BinRegion*, int, PairRec*, const BinRegion*, unsigned*,
                       unsigned*, const DevProfile*, const Thresholds*, const float4*, const uint8_t*, const int64_t*,
                       const int32_t*, const float4*, float, float*, unsigned*);
typedef void (*FwdFn)(const PairRec*, const unsigned*, const BinRegion*, int, PairRec*, const BinRegion*, unsigned*,
                      unsigned*, const DevProfile*, const Thresholds*, const float*, const uint8_t*, const int64_t*,
                      const int32_t*, const float4*, float, float*, const int64_t*);
typedef void (*BwdFn)(const PairRec*, const unsigned*, const BinRegion*, int, const DevProfile*, const float*,
                      const uint8_t*, const int64_t*, const int32_t*, const float4*, float*, const int64_t*);
typedef void (*AdjFFn)(const sxk::AdjPair*, int, const DevProfile*, const float*, const uint8_t*, const int64_t*,
                       const int32_t*, const float4*, float*, double*, double*);
typedef void (*AdjBFn)(const sxk::AdjPair*, int, const DevProfile*, const float*, const uint8_t*, const int64_t*,
                       const int32_t*, const float4*, float*, const double*, const double*, float*);
typedef void (*EnvPassFn)(const sxk::EnvRec*, int, const DevProfile*, const float*, const uint8_t*, const int64_t*,
                          float*, float*);
typedef void (*EnvPostFn)(const sxk::EnvRec*, int, const DevProfile*, const float*, float*, float*, const double*,
                          float*);

struct KernelTables {
  MsvFn msv[kNumMsvShapes];
  Msv16Fn msv16[kNumMsvShapes];  // the packed pre-screen, same shapes
  EnvPassFn envf[kNumVbins], envb[kNumVbins];
  EnvPostFn envp[kNumVbins];
  EnvPassFn regf[kNumVbins];
  VitFn vit[kNumVbins];
  FwdFn fwd[kNumVbins];
  FwdFn fwd_scan[kNumVbins];  // the F3 pre-screen
  BwdFn bwd[kNumVbins];
  AdjFFn adjf[kNumVbins];
  AdjBFn adjb[kNumVbins];
  VitGFn vitg[kNumVitShapes];
  Vit16Fn vit16[kNumVit16Shapes];  // the packed Viterbi pre-screen
};

// Filled by the kernel translation units.
void fill_msv_tables(KernelTables& t);
void fill_msv16_tables(KernelTables& t);
void fill_vit_tables(KernelTables& t);
void fill_vit16_tables(KernelTables& t);
void fill_vbin_tables(KernelTables& t);
void fill_env_tables(KernelTables& t);

}  // namespace sx
