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



// One thread per (ghost op, component): component m < W of w, then vhi.
__global__ void k_ghost(View v, const GhostOp* ops, int nops, const double* bcval, int valstride) {
    const int W = v.W, nY = v.nY, NC = W + nY;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)nops * NC) return;
    const int m = (int)(t / nops), o = (int)(t - (long long)m * nops);
    const GhostOp op = ops[o];
    const long long N = v.ncell;
    const long long d = op.dst, s = op.src;
    const double* val = bcval + (long long)op.bc * valstride;
    if (m >= W) {  // vhi
        const int k = m - W;
        v.vhi[k * N + d] = (op.kind == SCFD_BC_FIXED || op.kind == SCFD_BC_FIXED_PIN) ? val[W + k] : v.vhi[k * N + s];
        return;
    }
    const double* w = v.w;
    double r;
    switch (op.kind) {
        case SCFD_BC_FIXED:
            r = val[m];
            break;
        case SCFD_BC_FIXED_PIN: {
            const double pin = w[3 * N + s];
            r = m == 0 ? pin * val[W + nY] / val[W + nY + 1] : (m == 3 ? pin : val[m]);
            break;
        }
        case SCFD_BC_OUTFLOW_P:
            r = m == 3 ? val[0] : w[m * N + s];
            break;
        case SCFD_BC_SLIP:
            if (m == 1 || m == 2) {
                const double u = w[N + s], vv = w[2 * N + s];
                const double un = u * op.n1 + vv * op.n2;
                r = m == 1 ? u - 2.0 * un * op.n1 : vv - 2.0 * un * op.n2;
            } else {
                r = w[m * N + s];
            }
            break;
        case SCFD_BC_NOSLIP:
            r = (m == 1 || m == 2) ? val[m - 1] * 2.0 - w[m * N + s] : w[m * N + s];
            break;
        default:
            r = w[m * N + s];
            break;
    }
    v.w[m * N + d] = r;
}

// set_corners (condition.tail.f90:331-356): one thread per (plane, corner, component)
__global__ void k_corners(View v) {
    const int NC = v.W + v.nY;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * v.P.nact * NC) return;
    const int m = t % NC, pc = t / NC;
    const int p = v.P.act[pc >> 2];
    const int pi = (pc & 1) ? 1 : -1, pj = (pc & 2) ? 1 : -1;
    const int i = pi < 0 ? 1 : v.P.ni[p];
    const int j = pj < 0 ? 1 : v.P.nj[p];
    const long long N = v.ncell;
    const long long a = cidx(v.P, p, i, j), b = cidx(v.P, p, i, j + pj), c = cidx(v.P, p, i + pi, j);
    const long long d = cidx(v.P, p, i + pi, j + pj);
    double* f = m < v.W ? v.w + m * N : v.vhi + (m - v.W) * N;
    f[d] = 1.0 / 3.0 * (f[a] + f[b] + f[c]);
}

// the ghost-cell writes without set_corners (for stencils that never read corners)
int launch_ghost_ops(const View& v, cudaStream_t s, const GhostOp* ops, int nops, const double* bcval, int valstride) {
    if (nops <= 0) return 0;
    const long long nt = (long long)nops * (v.W + v.nY);
    k_ghost<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(v, ops, nops, bcval, valstride);
    return 1;
}

int launch_ghosts(const View& v, cudaStream_t s, const GhostOp* ops, int nops, const double* bcval, int valstride) {
    int n = 0;
    if (nops > 0) {
        const long long nt = (long long)nops * (v.W + v.nY);
        k_ghost<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(v, ops, nops, bcval, valstride);
        ++n;
    }
    if (v.P.nact == 0) return n;
    const int nc = 4 * v.P.nact * (v.W + v.nY);
    k_corners<<<(nc + 127) / 128, 128, 0, s>>>(v);
    return n + 1;
}

}  // namespace scfd
