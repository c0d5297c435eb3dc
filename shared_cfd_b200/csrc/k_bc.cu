// k_bc.cu -- set_BC on the device.
//
// The reference fills ghost cells in this order (store/cond/no-nV/condition.tail.f90
// and the generated condition.f90): section_exchange (block-interface halo,
// lines 2-70) -> user i-boundaries -> user j-boundaries -> set_corners
// (lines 331-356).  Every ghost write of the first three phases reads only
// interior cells, so the host expands them into one list of ghost-cell
// operations, keeps the last writer of each ghost cell in reference order, and
// a single launch applies them all.  set_corners reads ghost cells and runs as
// a second launch.
#include "scfd_internal.h"

namespace scfd {



__global__ void k_ghost(View v, const GhostOp* ops, int nops, const double* bcval, int valstride) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nops) return;
    const GhostOp op = ops[t];
    const long long N = v.ncell;
    const int W = v.W, nY = v.nY;
    double* w = v.w;
    double* vhi = v.vhi;
    const long long d = op.dst, s = op.src;
    const double* val = bcval + (long long)op.bc * valstride;
    switch (op.kind) {
        case SCFD_BC_FIXED:
            for (int k = 0; k < W; ++k) w[k * N + d] = val[k];
            for (int k = 0; k < nY; ++k) vhi[k * N + d] = val[W + k];
            return;
        case SCFD_BC_FIXED_PIN: {
            const double pin = w[3 * N + s];
            for (int k = 0; k < W; ++k) w[k * N + d] = val[k];
            for (int k = 0; k < nY; ++k) vhi[k * N + d] = val[W + k];
            w[d] = pin * val[W + nY] / val[W + nY + 1];
            w[3 * N + d] = pin;
            return;
        }
        default:
            break;
    }
    for (int k = 0; k < W; ++k) w[k * N + d] = w[k * N + s];
    for (int k = 0; k < nY; ++k) vhi[k * N + d] = vhi[k * N + s];
    if (op.kind == SCFD_BC_OUTFLOW_P) {
        w[3 * N + d] = val[0];
    } else if (op.kind == SCFD_BC_SLIP) {
        const double u = w[N + s], vv = w[2 * N + s];
        const double un = u * op.n1 + vv * op.n2;
        w[N + d] = u - 2.0 * un * op.n1;
        w[2 * N + d] = vv - 2.0 * un * op.n2;
    } else if (op.kind == SCFD_BC_NOSLIP) {
        w[N + d] = val[0] * 2.0 - w[N + s];
        w[2 * N + d] = val[1] * 2.0 - w[2 * N + s];
    }
}

__global__ void k_corners(View v) {
    const int t = threadIdx.x;
    if ((t >> 2) >= v.P.nact) return;
    const int p = v.P.act[t >> 2];
    const int pi = (t & 1) ? 1 : -1, pj = (t & 2) ? 1 : -1;
    const int i = pi < 0 ? 1 : v.P.ni[p];
    const int j = pj < 0 ? 1 : v.P.nj[p];
    const long long N = v.ncell;
    const long long a = cidx(v.P, p, i, j), b = cidx(v.P, p, i, j + pj), c = cidx(v.P, p, i + pi, j);
    const long long d = cidx(v.P, p, i + pi, j + pj);
    for (int k = 0; k < v.W; ++k)
        v.w[k * N + d] = 1.0 / 3.0 * (v.w[k * N + a] + v.w[k * N + b] + v.w[k * N + c]);
    for (int k = 0; k < v.nY; ++k)
        v.vhi[k * N + d] = 1.0 / 3.0 * (v.vhi[k * N + a] + v.vhi[k * N + b] + v.vhi[k * N + c]);
}

// the ghost-cell writes without set_corners (for stencils that never read corners)
int launch_ghost_ops(const View& v, cudaStream_t s, const GhostOp* ops, int nops, const double* bcval, int valstride) {
    if (nops <= 0) return 0;
    k_ghost<<<(nops + 127) / 128, 128, 0, s>>>(v, ops, nops, bcval, valstride);
    return 1;
}

int launch_ghosts(const View& v, cudaStream_t s, const GhostOp* ops, int nops, const double* bcval, int valstride) {
    int n = 0;
    if (nops > 0) {
        k_ghost<<<(nops + 127) / 128, 128, 0, s>>>(v, ops, nops, bcval, valstride);
        ++n;
    }
    if (v.P.nact == 0) return n;
    k_corners<<<1, 4 * v.P.nact, 0, s>>>(v);
    return n + 1;
}

}  // namespace scfd
