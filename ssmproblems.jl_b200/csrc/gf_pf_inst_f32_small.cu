// Instantiations of the LG particle-filter kernels (compiled in parallel).
#include "gf_pf_lg.cuh"

namespace gf {
void register_lg_f32_small(std::vector<PfLgKernels>& v, bool guided) {
  v.push_back(guided ? make_lg<float, 1, 1, true>() : make_lg<float, 1, 1, false>());
  v.push_back(guided ? make_lg<float, 2, 2, true>() : make_lg<float, 2, 2, false>());
  v.push_back(guided ? make_lg<float, 4, 4, true>() : make_lg<float, 4, 4, false>());
  v.push_back(guided ? make_lg<float, 8, 4, true>() : make_lg<float, 8, 4, false>());
  v.push_back(guided ? make_lg<float, 8, 8, true>() : make_lg<float, 8, 8, false>());
}
}  // namespace gf
