// Instantiations of the packed Viterbi pre-screen, one per lane-group shape.
#include "shapes.hpp"

namespace sx {
namespace {
template <int I>
struct Vit16Table {
  static void fill(Vit16Fn* t) {
    t[I] = sxk::vit16_kernel<kVit16Shapes[I].g, kVit16Shapes[I].c>;
    Vit16Table<I + 1>::fill(t);
  }
};
template <>
struct Vit16Table<kNumVit16Shapes> {
  static void fill(Vit16Fn*) {}
};
}  // namespace

void fill_vit16_tables(KernelTables& t) { Vit16Table<0>::fill(t.vit16); }

}  // namespace sx
