// Instantiations of the lane-group Viterbi kernels, one per shape.
#include "shapes.hpp"

namespace sx {
namespace {
template <int I>
struct VitGTable {
  static void fill(VitGFn* t) {
    t[I] = sxk::viterbi_g_kernel<kVitShapes[I].g, kVitShapes[I].c, kVitShapes[I].rt != 0>;
    VitGTable<I + 1>::fill(t);
  }
};
template <>
struct VitGTable<kNumVitShapes> {
  static void fill(VitGFn*) {}
};
}  // namespace

void fill_vit_tables(KernelTables& t) { VitGTable<0>::fill(t.vitg); }

}  // namespace sx
