// Instantiations of the warp-chunked kernels (warp-per-pair Viterbi, Forward,
// the Forward pre-screen, Backward, the adjoint passes), one per column width.
#include "shapes.hpp"

namespace sx {
namespace {
template <int I>
struct VbinTable {
  static void fill(KernelTables& t) {
    t.vit[I] = sxk::viterbi_kernel<kVcBins[I]>;
    t.fwd[I] = sxk::forward_kernel<kVcBins[I]>;
    t.fwd_scan[I] = sxk::forward_kernel<kVcBins[I], true>;
    t.bwd[I] = sxk::backward_kernel<kVcBins[I]>;
    t.adjf[I] = sxk::adjoint_forward_kernel<kVcBins[I]>;
    t.adjb[I] = sxk::adjoint_backward_kernel<kVcBins[I]>;
    VbinTable<I + 1>::fill(t);
  }
};
template <>
struct VbinTable<kNumVbins> {
  static void fill(KernelTables&) {}
};
}  // namespace

void fill_vbin_tables(KernelTables& t) { VbinTable<0>::fill(t); }

}  // namespace sx
