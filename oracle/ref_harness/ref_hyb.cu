// Test-only harness around the reference's own FP64 GPU repulsion
// (code/cuda/SG-tSNE-HYB/sgtsnepi/src/cuda/Frep.cu:142-175), compiled in
// place from the reference tree by oracle/build_ref.sh.  Used to produce
// golden vectors of the reference itself; never part of the product.
#include <vector>
#include "../types.hpp"

coord computeFrepulsive_GPU(coord *Freph, coord *yh, int n, int d, double h, double *timeInfo);

extern "C" double ref_hyb_repulsive(int n, int d, double h, const double *y_point_major, double *F) {
  std::vector<double> y(y_point_major, y_point_major + (size_t)n * d);  // the call shifts its copy
  double time_info[16] = {0};
  return computeFrepulsive_GPU(F, y.data(), n, d, h, time_info);
}
