// gf_pf_inst_f32_64g.cu -- the guided-proposal FP32 PF kernels for state
// dimension 33..64 (registered by gf_pf_inst_f32_64.cu).
#include "gf_pf_lg.cuh"

namespace gf {

PfLgKernels make_lg_f32_64_guided() { return make_lg<float, 64, 32, true>(); }

}  // namespace gf
