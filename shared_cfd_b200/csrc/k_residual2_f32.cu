// k_residual2_f32.cu -- the FP32 (mixed path) instantiations of the fused residual kernel.
#include "k_residual2.cuh"

namespace scfd {

bool launch_residual2_f32(const View& v, cudaStream_t s, int mode) { return launch_residual2_rt<float>(v, s, mode); }

}  // namespace scfd
