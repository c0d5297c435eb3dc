// k_residual2_f64.cu -- the FP64 instantiations of the fused residual kernel.
#include "k_residual2.cuh"

namespace scfd {

bool launch_residual2_f64(const View& v, cudaStream_t s, int mode) { return launch_residual2_rt<double>(v, s, mode); }

}  // namespace scfd
