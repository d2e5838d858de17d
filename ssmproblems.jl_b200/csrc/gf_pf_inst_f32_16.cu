// Instantiations of the LG particle-filter kernels (compiled in parallel).
#include "gf_pf_lg.cuh"

namespace gf {
void register_lg_f32_16(std::vector<PfLgKernels>& v, bool guided) {
  v.push_back(guided ? make_lg<float, 16, 8, true>() : make_lg<float, 16, 8, false>());
  v.push_back(guided ? make_lg<float, 16, 16, true>() : make_lg<float, 16, 16, false>());
}
}  // namespace gf
