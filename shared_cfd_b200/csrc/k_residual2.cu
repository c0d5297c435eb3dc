// k_residual2.cu -- dispatch of the fused residual kernel (k_residual2.cuh) by
// record precision, and the list of its tile shapes.
#include "k_residual2.cuh"

namespace scfd {

bool launch_residual2(const View& v, cudaStream_t s, int mode) {
    return v.precision == SCFD_PREC_MIXED ? launch_residual2_f32(v, s, mode) : launch_residual2_f64(v, s, mode);
}

int residual2_tiles(int* tx, int* ty) {
    const int t[4][2] = {{Tile0::TX, Tile0::TY}, {Tile1::TX, Tile1::TY}, {Tile2::TX, Tile2::TY}, {Tile3::TX, Tile3::TY}};
    for (int k = 0; k < 4; ++k) {
        if (tx) tx[k] = t[k][0];
        if (ty) ty[k] = t[k][1];
    }
    return 4;
}

}  // namespace scfd
