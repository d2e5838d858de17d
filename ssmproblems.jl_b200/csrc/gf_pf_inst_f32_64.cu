// gf_pf_inst_f32_64.cu -- FP32 linear-Gaussian PF kernels for state dimension 33..64.
// The bootstrap filter takes the tensor-core propagation (one block per SM at
// this size: its operand tiles fill the shared memory); the CUDA-core variant
// serves guided proposals and GF_PLAN_SIMT.
#include "gf_pf_lg.cuh"

namespace gf {

void register_lg_f32_64(std::vector<PfLgKernels>& v, bool guided) {
  v.push_back(guided ? make_lg<float, 64, 32, true>() : make_lg<float, 64, 32, false>());
}

}  // namespace gf
