// Instantiations of the MSV kernels, one per lane-group shape.
#include "shapes.hpp"

namespace sx {
namespace {
template <int I>
struct MsvTable {
  static void fill(MsvFn* t) {
    t[I] = sxk::msv_kernel<kMsvShapes[I].g, kMsvShapes[I].c>;
    MsvTable<I + 1>::fill(t);
  }
};
template <>
struct MsvTable<kNumMsvShapes> {
  static void fill(MsvFn*) {}
};
}  // namespace

void fill_msv_tables(KernelTables& t) { MsvTable<0>::fill(t.msv); }

}  // namespace sx
