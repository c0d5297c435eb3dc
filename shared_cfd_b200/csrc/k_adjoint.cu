// k_adjoint.cu -- device kernels of the discrete adjoint of the explicit
// ideal-gas step (scfd_adjoint_run): q^{n+1} = q^n + dt/Vol R(w(q^n)) with R
// the inviscid MUSCL + SLAU residual of a 2d case
// (time_scheme/euler/time_euler_viscous.raw.f90:1-23, core/scheme.f90).
//
// One reverse step takes lam = dJ/dq^{n+1} and, with w^n recomputed from q^n
// (thermo and ghost cells), forms
//   Rb_c = dt/Vol_c lam_c                         (interior cells)
//   per face f between L and R: Fb = ds_f (Rb_R - Rb_L); the reverse of SLAU and
//     of the MUSCL states adds the adjoint of w to the 4 cells of the stencil
//   the reverse of the ghost writes moves ghost adjoints to the interior cells
//     they copy and to the boundary values (the parameter gradient)
//   lam_c += (dw/dq)^T wb_c + [c on the objective boundary] ds dp/dq
// so that lam becomes dJ/dq^n.  dt is the fixed time step (no derivative).
// wb starts at zero once per run: every step's consumers clear what they read
// (each ghost cell has one ghost write; the inviscid stencils never reach the
// corner cells).
#include "adj_face.cuh"
#include "scfd_internal.h"

namespace scfd {

namespace {
constexpr int NY1 = 1;           // the ideal gas carries one species
constexpr int NC = 6 + NY1;      // rho, u, v, p, Y, gamma, h_t
constexpr int DD = NY1 + 3;      // conserved components
}  // namespace

// w component of the m-th SLAU state entry
__device__ __forceinline__ int wcomp(int m, int D) { return m < 4 + NY1 ? m : (m == 4 + NY1 ? D + 1 : D + 2); }

__global__ void __launch_bounds__(128, 3) k_adj_faces(View v, const double* __restrict__ lam, double* __restrict__ wbar,
                                                     double dt) {
    const int p = v.P.act[blockIdx.y];
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    const int nfi = (ni + 1) * nj, nfj = ni * (nj + 1);
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfi + nfj) return;
    const bool iface = f < nfi;
    int i, j;
    if (iface) {
        i = f % (ni + 1);
        j = f / (ni + 1) + 1;
    } else {
        const int g = f - nfi;
        i = g % ni + 1;
        j = g / ni;
    }
    const long long N = v.ncell;
    const int D = DD;
    long long c[4];
    for (int s = 0; s < 4; ++s)
        c[s] = iface ? cidx(v.P, p, i - 1 + s, j) : cidx(v.P, p, i, j - 1 + s);
    // interior test of L (stencil 1) and R (stencil 2)
    const bool inL = iface ? i >= 1 : j >= 1;
    const bool inR = iface ? i + 1 <= ni : j + 1 <= nj;
    const double ds = iface ? v.dsi[c[1]] : v.dsj[c[1]];
    double tgb[DD];
    bool any = false;
#pragma unroll
    for (int k = 0; k < DD; ++k) {
        const double rl = inL ? dt / v.Vol[c[1]] * lam[k * N + c[1]] : 0.0;
        const double rr = inR ? dt / v.Vol[c[2]] * lam[k * N + c[2]] : 0.0;
        tgb[k] = ds * (rr - rl);
        any = any || tgb[k] != 0.0;
    }
    if (!any) return;
    const double phi = v.recon == SCFD_RECON_MUSCL ? v.phi_mus : 0.0, km = v.k_mus;
    // face states first; the stencil is read again (from L1) for the reverse of MUSCL
    double wl[NC], wr[NC];
#pragma unroll
    for (int m = 0; m < NC; ++m) {
        const double* wk = v.w + wcomp(m, D) * N;
        adj::muscl_fwd(__ldg(wk + c[0]), __ldg(wk + c[1]), __ldg(wk + c[2]), __ldg(wk + c[3]), phi, km, wl[m], wr[m]);
    }
    const double* vn = iface ? v.vni : v.vnj;
    const double n1 = vn[c[1]], n2 = vn[N + c[1]];
    double wlb[NC] = {0}, wrb[NC] = {0};
    adj::slau_rev(NY1, wl, wr, n1, n2, tgb, wlb, wrb);
#pragma unroll
    for (int m = 0; m < NC; ++m) {
        const double* wk = v.w + wcomp(m, D) * N;
        double b[4] = {0, 0, 0, 0};
        adj::muscl_rev(__ldg(wk + c[0]), __ldg(wk + c[1]), __ldg(wk + c[2]), __ldg(wk + c[3]), phi, km, wlb[m], wrb[m],
                       b[0], b[1], b[2], b[3]);
        double* wb = wbar + wcomp(m, D) * N;
#pragma unroll
        for (int s = 0; s < 4; ++s)
            if (b[s] != 0.0) atomicAdd(wb + c[s], b[s]);
    }
}

// Reverse of k_ghost (k_bc.cu): every op reads interior cells only, so the
// ghost adjoints move to the copied cells and, for value-setting kinds, to the
// gradient of descriptor param_bc's values.
__global__ void k_adj_ghost(View v, const GhostOp* __restrict__ ops, int nops, const double* __restrict__ bcval,
                            int valstride, double* __restrict__ wbar, double* __restrict__ grad, int param_bc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nops) return;
    const GhostOp op = ops[t];
    const long long N = v.ncell, d = op.dst, s = op.src;
    const int W = v.W, nY = v.nY;
    const double* val = bcval + (long long)op.bc * valstride;
    const bool mine = op.kind >= 0 && op.bc == param_bc;
    auto to_src = [&](int k, double x) {
        if (x != 0.0) atomicAdd(wbar + k * N + s, x);
    };
    auto to_grad = [&](int k, double x) {
        if (mine && x != 0.0) atomicAdd(grad + k, x);
    };
    // the ghost's adjoint is consumed here: clear it for the next step
    auto clear = [&]() {
        for (int k = 0; k < W; ++k) wbar[k * N + d] = 0.0;
    };
    switch (op.kind) {
        case SCFD_BC_FIXED:
            for (int k = 0; k < W; ++k) to_grad(k, wbar[k * N + d]);
            clear();
            return;
        case SCFD_BC_FIXED_PIN: {
            // w_d = value except rho = pin value[W+nY] / value[W+nY+1], p = pin = w_s(p)
            const double pin = v.w[3 * N + s], a = val[W + nY], b = val[W + nY + 1];
            const double rb = wbar[d], pb = wbar[3 * N + d];
            for (int k = 0; k < W; ++k)
                if (k != 0 && k != 3) to_grad(k, wbar[k * N + d]);
            to_src(3, pb + rb * a / b);
            to_grad(W + nY, rb * pin / b);
            to_grad(W + nY + 1, -rb * pin * a / (b * b));
            clear();
            return;
        }
        default:
            break;
    }
    for (int k = 0; k < W; ++k) {
        if (op.kind == SCFD_BC_OUTFLOW_P && k == 3) continue;
        if ((op.kind == SCFD_BC_SLIP || op.kind == SCFD_BC_NOSLIP) && (k == 1 || k == 2)) continue;
        to_src(k, wbar[k * N + d]);
    }
    if (op.kind == SCFD_BC_OUTFLOW_P) {
        to_grad(0, wbar[3 * N + d]);
    } else if (op.kind == SCFD_BC_SLIP) {
        // u_d = u - 2 un n1, v_d = v - 2 un n2, un = u n1 + v n2
        const double ub = wbar[N + d], vb = wbar[2 * N + d];
        const double n1 = op.n1, n2 = op.n2;
        to_src(1, ub * (1.0 - 2.0 * n1 * n1) + vb * (-2.0 * n1 * n2));
        to_src(2, ub * (-2.0 * n1 * n2) + vb * (1.0 - 2.0 * n2 * n2));
    } else if (op.kind == SCFD_BC_NOSLIP) {
        // u_d = 2 value[0] - u, v_d = 2 value[1] - v
        to_src(1, -wbar[N + d]);
        to_src(2, -wbar[2 * N + d]);
        to_grad(0, 2.0 * wbar[N + d]);
        to_grad(1, 2.0 * wbar[2 * N + d]);
    }
    clear();
}

// lam_c += (dw/dq)^T wb_c over the interior cells (ideal gas: set_w and the
// ideal thermal model; gamma, R and mu do not depend on q here)
__global__ void k_adj_prim(View v, double* __restrict__ wbar, double* __restrict__ lam) {
    const int p = v.P.act[blockIdx.y];
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= ni * nj) return;
    const long long N = v.ncell;
    const long long c = cidx(v.P, p, idx % ni + 1, idx / ni + 1);
    constexpr int D = DD;
    double q[DD], qb[DD] = {0};
#pragma unroll
    for (int k = 0; k < D; ++k) q[k] = v.q[k * N + c];
    double Yb[NY1];
#pragma unroll
    for (int k = 0; k < NY1; ++k) Yb[k] = wbar[(4 + k) * N + c];
    adj::ideal_prim_rev(NY1, q, v.kappa, wbar[c], wbar[N + c], wbar[2 * N + c], wbar[3 * N + c], Yb,
                        wbar[(D + 2) * N + c], qb);
#pragma unroll
    for (int k = 0; k < D; ++k) lam[k * N + c] += qb[k];
    // consumed: clear the components the faces add to (gamma's adjoint has no use here)
#pragma unroll
    for (int m = 0; m < NC; ++m) wbar[wcomp(m, D) * N + c] = 0.0;
}

// the objective's term of one state: J += sum_c wt_c p(q_c), in a fixed order
// (one CTA, pairwise tree), and lam_c += wt_c dp/dq_c
__global__ void k_adj_objective(View v, const long long* __restrict__ cells, const double* __restrict__ wt, int n,
                                double* J, double* lam, int grad_only) {
    __shared__ double sh[256];
    const long long N = v.ncell;
    constexpr int D = DD;
    double acc = 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const long long c = cells[t];
        double q[DD];
#pragma unroll
        for (int k = 0; k < D; ++k) q[k] = v.q[k * N + c];
        if (lam) {
            double qb[DD] = {0};
            adj::ideal_p_rev(NY1, q, v.kappa, wt[t], qb);
#pragma unroll
            for (int k = 0; k < D; ++k) lam[k * N + c] += qb[k];
        }
        if (!grad_only) acc += wt[t] * adj::ideal_p(NY1, q, v.kappa);
    }
    if (grad_only) return;
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *J += sh[0];
}

int launch_adj_faces(const View& v, cudaStream_t s, const double* lam, double* wbar, double dt) {
    int mx = 0;
    for (int a = 0; a < v.P.nact; ++a) {
        const int p = v.P.act[a];
        const int nf = (v.P.ni[p] + 1) * v.P.nj[p] + v.P.ni[p] * (v.P.nj[p] + 1);
        mx = nf > mx ? nf : mx;
    }
    if (v.P.nact == 0 || mx == 0) return 0;
    k_adj_faces<<<dim3((mx + 127) / 128, v.P.nact), 128, 0, s>>>(v, lam, wbar, dt);
    return 1;
}

int launch_adj_ghost(const View& v, cudaStream_t s, const GhostOp* ops, int nops, const double* bcval, int valstride,
                     double* wbar, double* grad, int param_bc) {
    if (nops <= 0) return 0;
    k_adj_ghost<<<(nops + 127) / 128, 128, 0, s>>>(v, ops, nops, bcval, valstride, wbar, grad, param_bc);
    return 1;
}

int launch_adj_prim(const View& v, cudaStream_t s, double* wbar, double* lam) {
    int mx = 0;
    for (int a = 0; a < v.P.nact; ++a) {
        const int p = v.P.act[a];
        mx = v.P.ni[p] * v.P.nj[p] > mx ? v.P.ni[p] * v.P.nj[p] : mx;
    }
    if (v.P.nact == 0) return 0;
    k_adj_prim<<<dim3((mx + 255) / 256, v.P.nact), 256, 0, s>>>(v, wbar, lam);
    return 1;
}

int launch_adj_objective(const View& v, cudaStream_t s, const long long* cells, const double* wt, int n, double* J,
                         double* lam, int grad_only) {
    if (n <= 0) return 0;
    k_adj_objective<<<1, 256, 0, s>>>(v, cells, wt, n, J, lam, grad_only);
    return 1;
}

}  // namespace scfd
