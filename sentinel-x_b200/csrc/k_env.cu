// Instantiations of the envelope-rescoring and region kernels, one per
// column width.
#include "shapes.hpp"

namespace sx {
namespace {
template <int I>
struct EnvTable {
  static void fill(KernelTables& t) {
    t.envf[I] = sxk::env_forward_kernel<kVcBins[I]>;
    t.envb[I] = sxk::env_backward_kernel<kVcBins[I]>;
    t.envp[I] = sxk::env_post_kernel<kVcBins[I]>;
    t.regf[I] = sxk::env_forward_kernel<kVcBins[I], true>;
    EnvTable<I + 1>::fill(t);
  }
};
template <>
struct EnvTable<kNumVbins> {
  static void fill(KernelTables&) {}
};
}  // namespace

void fill_env_tables(KernelTables& t) { EnvTable<0>::fill(t); }

}  // namespace sx
