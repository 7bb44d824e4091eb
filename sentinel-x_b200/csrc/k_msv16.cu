// Instantiations of the packed MSV pre-screen, one per lane-group shape.
#include "shapes.hpp"

namespace sx {
namespace {
template <int I>
struct Msv16Table {
  static void fill(Msv16Fn* t) {
    t[I] = sxk::msv16_kernel<kMsvShapes[I].g, kMsvShapes[I].c>;
    Msv16Table<I + 1>::fill(t);
  }
};
template <>
struct Msv16Table<kNumMsvShapes> {
  static void fill(Msv16Fn*) {}
};
}  // namespace

void fill_msv16_tables(KernelTables& t) { Msv16Table<0>::fill(t.msv16); }

}  // namespace sx
