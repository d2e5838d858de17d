// gf_pf_inst_f32_64.cu -- FP32 linear-Gaussian PF kernels for state dimension 33..64.
// The bootstrap filter takes the tensor-core propagation (one block per SM at
// this size: its operand tiles fill the shared memory); the CUDA-core variant
// serves guided proposals and GF_PLAN_SIMT.  The guided instance compiles in
// gf_pf_inst_f32_64g.cu (in parallel: both are the build's slowest units).
#include "gf_pf_lg.cuh"

namespace gf {

PfLgKernels make_lg_f32_64_guided();

void register_lg_f32_64(std::vector<PfLgKernels>& v, bool guided) {
  v.push_back(guided ? make_lg_f32_64_guided() : make_lg<float, 64, 32, false>());
}

}  // namespace gf
