// Instantiations of the LG particle-filter kernels (compiled in parallel).
#include "gf_pf_lg.cuh"

namespace gf {
void register_lg_f64(std::vector<PfLgKernels>& v, bool guided) {
  v.push_back(guided ? make_lg<double, 1, 1, true>() : make_lg<double, 1, 1, false>());
  v.push_back(guided ? make_lg<double, 2, 2, true>() : make_lg<double, 2, 2, false>());
  v.push_back(guided ? make_lg<double, 4, 4, true>() : make_lg<double, 4, 4, false>());
  v.push_back(guided ? make_lg<double, 8, 8, true>() : make_lg<double, 8, 8, false>());
  v.push_back(guided ? make_lg<double, 16, 16, true>() : make_lg<double, 16, 16, false>());
}
}  // namespace gf
