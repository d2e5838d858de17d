// Instantiations of the LG particle-filter kernels (compiled in parallel).
#include "gf_pf_lg.cuh"

namespace gf {
void register_lg_f32_32(std::vector<PfLgKernels>& v, bool guided) {
  v.push_back(guided ? make_lg<float, 32, 16, true>() : make_lg<float, 32, 16, false>());
  v.push_back(guided ? make_lg<float, 32, 32, true>() : make_lg<float, 32, 32, false>());
}
}  // namespace gf
