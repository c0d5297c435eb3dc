// scfd_api.cu -- the C ABI of include/scfd_b200.h: context, device arena,
// metrics, boundary expansion, state transfer and the per-step kernel sequence.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "chem_tables.h"
#include "scfd_internal.h"

using namespace scfd;

// bytes of each pinned chunk of the host <-> device copies (two chunks per context)
constexpr size_t kRingChunk = 32ull << 20;

struct scfd_ctx {
    scfd_desc d{};
    std::string err;
    int np = 0, nY = 0, D = 0, W = 0, nimax = 0, njmax = 0;
    Planes P{};
    long long ncell = 0;
    std::vector<std::vector<double>> xh, rh;
    std::vector<int> geo_set;
    bool committed = false, have_chem = false, uploaded = false;
    std::vector<int32_t> cut;
    std::vector<scfd_bc> bcs;
    scfd_chem chem{};
    cudaStream_t stream = nullptr;
    int device = 0, nsm = 148;
    char* arena = nullptr;
    size_t arena_bytes = 0;
    View v{};
    DevScalars* d_sc = nullptr;
    DevScalars* h_sc = nullptr;  // pinned
    // sweeps
    int nsf = 0, nsb = 0;
    int* d_strips_f = nullptr;
    int* d_strips_b = nullptr;
    double* d_xfer = nullptr;
    int* d_progress = nullptr;
    int* d_tickets = nullptr;
    double* d_partials = nullptr;
    // boundaries
    GhostOp* d_ops = nullptr;
    int nops = 0;
    double* d_bcval = nullptr;
    int valstride = SCFD_BC_MAXVAL + 2;
    // cluster-wavefront sweeps over strip records (k_wave.cu)
    bool use_sw3 = false;
    Wave sw3{};
    // chemistry
    unsigned long long* d_counter = nullptr;
    ChemQueue dq{};  // cells whose chemistry interval goes to DVODE
    // rms
    double* d_rms_partial = nullptr;
    double* d_rms_out = nullptr;
    // pinned staging for transfers
    double* d_ref = nullptr;  // device staging of one field in the reference layout
    void* h_ring[2] = {nullptr, nullptr};  // pinned chunks of the host <-> device copies
    cudaEvent_t ring_ev[2] = {nullptr, nullptr};
    long long launches = 0;
    int cells_max = 0;
    // per-kernel timing
    bool profiling = false;
    // the whole physical step as one CUDA graph (captured at the second step)
    bool use_graph = true;
    int eager_steps = 0;
    cudaGraphExec_t graph = nullptr;
    long long graph_launches = 0;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<std::pair<int, size_t>> ev_marks;  // kind, index of the start event
    double kind_ms[SCFD_K_COUNT] = {0};
    long long kind_n[SCFD_K_COUNT] = {0};
    // block sharding: planes of this rank, the cells it exports to other
    // ranks' ghost copies, the cells it imports, exchange and reduction
    // buffers, and the position of a staged step (scfd_dstep)
    int nranks = 1, rank = 0;
    std::vector<int> owner;
    long long* d_exp = nullptr;
    int nexp = 0;
    HaloImport* d_imp = nullptr;
    int nimp = 0;
    double* d_halo = nullptr;
    long long seg = 0;
    double* d_red = nullptr;
    int ds_stage = 0, ds_j = 0;
    long long ds_att0 = 0, ds_fb0 = 0;
    bool own(int p) const { return owner.empty() || owner[p] == rank; }  // p 0-based
    // discrete adjoint (scfd_adjoint_run): face lengths on the host, and the
    // device buffers and reverse-step graphs kept from one run to the next
    std::vector<double> h_dsi, h_dsj;
    struct AdjCache {
        double* slots = nullptr;
        int nslots = 0;
        double* lam = nullptr;
        double* wbar = nullptr;
        double* dgrad = nullptr;
        double* dJ = nullptr;
        long long* ocells = nullptr;
        double* owt = nullptr;
        cudaGraphExec_t rev_graph[2] = {nullptr, nullptr};
        int key_obj = -2, key_param = -2;
        std::vector<std::vector<int>> best_split;  // checkpoint plan of the last (nsteps, snapshots)
        int plan_n = -1, plan_s = -1;
    } adj;
    // autotuner (launch shapes of the residual and thermo kernels)
    bool tuned = false;
    std::string tune_report = "{}";

    int fail(int code, const std::string& m) {
        err = m;
        return code;
    }
};

namespace {

#define CK(x)                                                                               \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) return c->fail(SCFD_E_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

inline double sq(double a) { return a * a; }

// ---------------------------------------------------------------------------
// Metrics on the host in FP64 (store/dim/{2d,q2d}/geometry.f90, LU-SGS set_vnc_dsc,
// viscous set_geojac), written straight into the device slot layout.
// ---------------------------------------------------------------------------
struct HostGeo {
    std::vector<double> Vol, Area, dsi, dsj, vni, vnj, x, r, gjc, gji, gjj, dsci, dscj, vnci, vncj;
};

void build_geometry(scfd_ctx* c, HostGeo& g) {
    const long long N = c->ncell;
    auto z = [&](std::vector<double>& a, int k) { a.assign((size_t)(k * N), 0.0); };
    z(g.Vol, 1); z(g.Area, 1); z(g.dsi, 1); z(g.dsj, 1); z(g.vni, 2); z(g.vnj, 2); z(g.x, 1); z(g.r, 1);
    z(g.gjc, 4); z(g.gji, 4); z(g.gjj, 4); z(g.dsci, 1); z(g.dscj, 1); z(g.vnci, 2); z(g.vncj, 2);
    const bool q2d = c->d.dim == SCFD_DIM_Q2D;
    const bool quirk = c->d.quirk_q1 != 0;
    for (int p = 0; p < c->np; ++p) {
        const int ni = c->P.ni[p], nj = c->P.nj[p];
        const std::vector<double>& XH = c->xh[p];
        const std::vector<double>& RH = c->rh[p];
        auto xh = [&](int i, int j) { return XH[i + (ni + 1) * j]; };
        auto rh = [&](int i, int j) { return RH[i + (ni + 1) * j]; };
        auto C = [&](int i, int j) { return cidx(c->P, p, i, j); };
        // cell centres with ghost extrapolation (set_xr, geometry.f90:79-106)
        auto X = [&](int i, int j) -> double& { return g.x[C(i, j)]; };
        auto R = [&](int i, int j) -> double& { return g.r[C(i, j)]; };
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                X(i, j) = 1.0 / 4.0 * (xh(i - 1, j - 1) + xh(i, j - 1) + xh(i - 1, j) + xh(i, j));
                R(i, j) = 1.0 / 4.0 * (rh(i - 1, j - 1) + rh(i, j - 1) + rh(i - 1, j) + rh(i, j));
            }
        // The reference writes x(ni(k)+1, j) for EVERY plane k here (ni is the
        // per-plane array: a vector subscript); with quirk_q1 this is kept.
        std::vector<int> icols, jrows;
        if (quirk) {
            for (int k = 0; k < c->np; ++k) {
                icols.push_back(c->P.ni[k]);
                jrows.push_back(c->P.nj[k]);
            }
        } else {
            icols.push_back(ni);
            jrows.push_back(nj);
        }
        for (int j = 1; j <= nj; ++j) {
            X(0, j) = 2.0 * X(1, j) - X(2, j);
            R(0, j) = 2.0 * R(1, j) - R(2, j);
            std::vector<double> vx, vr;
            for (int n : icols) {
                // out-of-plane columns (n >= this plane's ni + 2) fall into the
                // padding of the reference's nimax-wide array; they are read
                // nowhere, so only columns inside this plane's slots are kept
                vx.push_back(n + 1 <= ni + 1 && n - 1 >= 0 ? 2.0 * X(n, j) - X(n - 1, j) : 0.0);
                vr.push_back(n + 1 <= ni + 1 && n - 1 >= 0 ? 2.0 * R(n, j) - R(n - 1, j) : 0.0);
            }
            for (size_t k = 0; k < icols.size(); ++k)
                if (icols[k] + 1 <= ni + 1) X(icols[k] + 1, j) = vx[k];
            for (size_t k = 0; k < icols.size(); ++k)
                if (icols[k] + 1 <= ni + 1) R(icols[k] + 1, j) = vr[k];
        }
        for (int i = 0; i <= ni + 1; ++i) {
            X(i, 0) = 2.0 * X(i, 1) - X(i, 2);
            R(i, 0) = 2.0 * R(i, 1) - R(i, 2);
            std::vector<double> vx, vr;
            for (int n : jrows) {
                vx.push_back(n + 1 <= nj + 1 ? 2.0 * X(i, n) - X(i, n - 1) : 0.0);
                vr.push_back(n + 1 <= nj + 1 ? 2.0 * R(i, n) - R(i, n - 1) : 0.0);
            }
            for (size_t k = 0; k < jrows.size(); ++k)
                if (jrows[k] + 1 <= nj + 1) X(i, jrows[k] + 1) = vx[k];
            for (size_t k = 0; k < jrows.size(); ++k)
                if (jrows[k] + 1 <= nj + 1) R(i, jrows[k] + 1) = vr[k];
        }
        auto tri = [](double a1, double a2, double b1, double b2, double c1, double c2) {
            return 1.0 / 2.0 * (a1 * (b2 - c2) + b1 * (c2 - a2) + c1 * (a2 - b2));
        };
        auto dist = [](double x1, double y1, double x2, double y2) { return std::sqrt(sq(x1 - x2) + sq(y1 - y2)); };
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                const double A1 = tri(xh(i - 1, j - 1), rh(i - 1, j - 1), xh(i, j - 1), rh(i, j - 1), xh(i - 1, j), rh(i - 1, j));
                const double A2 = tri(xh(i, j - 1), rh(i, j - 1), xh(i, j), rh(i, j), xh(i - 1, j), rh(i - 1, j));
                const long long cc = C(i, j);
                if (q2d) {
                    g.Area[cc] = A1 + A2;
                    g.Vol[cc] = (rh(i - 1, j - 1) + rh(i, j - 1) + rh(i - 1, j)) * A1 / 3.0 +
                                (rh(i, j - 1) + rh(i, j) + rh(i - 1, j)) * A2 / 3.0;
                } else {
                    g.Area[cc] = 0.0;
                    g.Vol[cc] = A1 + A2;
                }
            }
        for (int j = 0; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                double ds = dist(xh(i - 1, j), rh(i - 1, j), xh(i, j), rh(i, j));
                if (q2d) ds = ds * (rh(i - 1, j) + rh(i, j)) / 2.0;
                g.dsj[C(i, j)] = ds;
                const double nx = -(rh(i, j) - rh(i - 1, j)), nr = xh(i, j) - xh(i - 1, j);
                const double sd = std::sqrt(sq(nx) + sq(nr));
                g.vnj[C(i, j)] = nx / sd;
                g.vnj[N + C(i, j)] = nr / sd;
            }
        for (int j = 1; j <= nj; ++j)
            for (int i = 0; i <= ni; ++i) {
                double ds = dist(xh(i, j - 1), rh(i, j - 1), xh(i, j), rh(i, j));
                if (q2d) ds = ds * (rh(i, j - 1) + rh(i, j)) / 2.0;
                g.dsi[C(i, j)] = ds;
                const double nx = rh(i, j) - rh(i, j - 1), nr = -(xh(i, j) - xh(i, j - 1));
                const double sd = std::sqrt(sq(nx) + sq(nr));
                g.vni[C(i, j)] = nx / sd;
                g.vni[N + C(i, j)] = nr / sd;
            }
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i) {
                const double a1 = (xh(i - 1, j - 1) + xh(i, j - 1)) * 0.5, a2 = (rh(i - 1, j - 1) + rh(i, j - 1)) * 0.5;
                const double b1 = (xh(i, j - 1) + xh(i, j)) * 0.5, b2 = (rh(i, j - 1) + rh(i, j)) * 0.5;
                const double c1 = (xh(i - 1, j) + xh(i, j)) * 0.5, c2 = (rh(i - 1, j) + rh(i, j)) * 0.5;
                const double d1 = (xh(i - 1, j - 1) + xh(i - 1, j)) * 0.5, d2 = (rh(i - 1, j - 1) + rh(i - 1, j)) * 0.5;
                double dci = std::sqrt(sq(c1 - a1) + sq(c2 - a2));
                double dcj = std::sqrt(sq(b1 - d1) + sq(b2 - d2));
                const long long cc = C(i, j);
                g.vnci[cc] = (b1 - d1) / dcj;
                g.vnci[N + cc] = (b2 - d2) / dcj;
                g.vncj[cc] = (c1 - a1) / dci;
                g.vncj[N + cc] = (c2 - a2) / dci;
                if (q2d) {
                    dci = dci * (c2 + a2) * 0.5;
                    dcj = dcj * (b2 + d2) * 0.5;
                }
                g.dsci[cc] = dci;
                g.dscj[cc] = dcj;
            }
        auto put = [&](std::vector<double>& a, long long cc, double dxdxi, double dydxi, double dxdeta, double dydeta) {
            const double det = dxdxi * dydeta - dydxi * dxdeta;
            a[cc] = dydeta / det;
            a[N + cc] = -dxdeta / det;
            a[2 * N + cc] = -dydxi / det;
            a[3 * N + cc] = dxdxi / det;
        };
        for (int j = 1; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i)
                put(g.gjc, C(i, j), (X(i + 1, j) - X(i - 1, j)) * 0.5, (R(i + 1, j) - R(i - 1, j)) * 0.5,
                    (X(i, j + 1) - X(i, j - 1)) * 0.5, (R(i, j + 1) - R(i, j - 1)) * 0.5);
        for (int j = 1; j <= nj; ++j)
            for (int i = 0; i <= ni; ++i)
                put(g.gji, C(i, j), X(i + 1, j) - X(i, j), R(i + 1, j) - R(i, j),
                    (X(i + 1, j + 1) + X(i, j + 1) - X(i + 1, j - 1) - X(i, j - 1)) * 0.25,
                    (R(i + 1, j + 1) + R(i, j + 1) - R(i + 1, j - 1) - R(i, j - 1)) * 0.25);
        for (int j = 0; j <= nj; ++j)
            for (int i = 1; i <= ni; ++i)
                put(g.gjj, C(i, j), (X(i + 1, j + 1) + X(i + 1, j) - X(i - 1, j + 1) - X(i - 1, j)) * 0.25,
                    (R(i + 1, j + 1) + R(i + 1, j) - R(i - 1, j + 1) - R(i - 1, j)) * 0.25, X(i, j + 1) - X(i, j),
                    R(i, j + 1) - R(i, j));
    }
}

// ---------------------------------------------------------------------------
// set_BC expansion: halo copies (section_exchange), then the i- and j-boundary
// descriptors, de-duplicated so the last writer of each ghost cell wins.
// ---------------------------------------------------------------------------
int build_ghost_ops(scfd_ctx* c, const HostGeo& g, std::vector<GhostOp>& out) {
    std::vector<GhostOp> ops;
    auto inside = [&](int p, int i, int j) {
        return p >= 0 && p < c->np && i >= -1 && i <= c->P.ni[p] + 2 && j >= -1 && j <= c->P.nj[p] + 2;
    };
    auto interior = [&](int p, int i, int j) {
        return p >= 0 && p < c->np && i >= 1 && i <= c->P.ni[p] && j >= 1 && j <= c->P.nj[p];
    };
    auto add = [&](int pd, int id, int jd, int ps, int is, int js, int kind, int bc, double n1, double n2) -> bool {
        if (!inside(pd, id, jd) || !interior(ps, is, js) || interior(pd, id, jd)) return false;
        GhostOp o;
        o.dst = cidx(c->P, pd, id, jd);
        o.src = cidx(c->P, ps, is, js);
        o.kind = kind;
        o.bc = bc;
        o.n1 = n1;
        o.n2 = n2;
        ops.push_back(o);
        return true;
    };
    const size_t nrec = c->cut.size() / 11;
    for (size_t n = 0; n < nrec; ++n) {
        const int32_t* r = &c->cut[n * 11];
        const int geo = r[0], width = r[1], order = r[2], p1 = r[3] - 1, c1 = r[4], s1 = r[5], pm1 = r[6],
                  p2 = r[7] - 1, c2 = r[8], s2 = r[9], pm2 = r[10];
        if (geo < 1 || geo > 4 || width < 0 || (order != 1 && order != -1) || (pm1 != 1 && pm1 != -1) ||
            (pm2 != 1 && pm2 != -1))
            return c->fail(SCFD_E_CONNECT, "bad connectivity record " + std::to_string(n + 1));
        bool ok = true;
        for (int inc = 0; inc < width && ok; ++inc) {
            const int a = s1 + inc, b = s2 + inc * order;
            switch (geo) {
                case 1:
                    ok = add(p1, c1 + pm1, a, p2, c2, b, -1, 0, 0, 0) && add(p1, c1 + 2 * pm1, a, p2, c2 - pm2, b, -1, 0, 0, 0) &&
                         add(p2, c2 + pm2, b, p1, c1, a, -1, 0, 0, 0) && add(p2, c2 + 2 * pm2, b, p1, c1 - pm1, a, -1, 0, 0, 0);
                    break;
                case 2:
                    ok = add(p1, c1 + pm1, a, p2, b, c2, -1, 0, 0, 0) && add(p1, c1 + 2 * pm1, a, p2, b, c2 - pm2, -1, 0, 0, 0) &&
                         add(p2, b, c2 + pm2, p1, c1, a, -1, 0, 0, 0) && add(p2, b, c2 + 2 * pm2, p1, c1 - pm1, a, -1, 0, 0, 0);
                    break;
                case 3:
                    ok = add(p1, a, c1 + pm1, p2, c2, b, -1, 0, 0, 0) && add(p1, a, c1 + 2 * pm1, p2, c2 - pm2, b, -1, 0, 0, 0) &&
                         add(p2, c2 + pm2, b, p1, a, c1, -1, 0, 0, 0) && add(p2, c2 + 2 * pm2, b, p1, a, c1 - pm1, -1, 0, 0, 0);
                    break;
                default:
                    ok = add(p1, a, c1 + pm1, p2, b, c2, -1, 0, 0, 0) && add(p1, a, c1 + 2 * pm1, p2, b, c2 - pm2, -1, 0, 0, 0) &&
                         add(p2, b, c2 + pm2, p1, a, c1, -1, 0, 0, 0) && add(p2, b, c2 + 2 * pm2, p1, a, c1 - pm1, -1, 0, 0, 0);
                    break;
            }
        }
        if (!ok) return c->fail(SCFD_E_CONNECT, "connectivity record " + std::to_string(n + 1) + " leaves the planes");
    }
    const long long N = c->ncell;
    for (int phase = 0; phase < 2; ++phase)
        for (size_t k = 0; k < c->bcs.size(); ++k) {
            const scfd_bc& b = c->bcs[k];
            const bool iside = b.side == SCFD_SIDE_ILO || b.side == SCFD_SIDE_IHI;
            if ((phase == 0) != iside) continue;
            const int p = b.plane - 1, ni = c->P.ni[p], nj = c->P.nj[p];
            for (int s = b.first; s <= b.last; ++s) {
                int ib, jb, i1, j1, i2, j2;
                long long fc;
                const std::vector<double>* nv;
                switch (b.side) {
                    case SCFD_SIDE_ILO: ib = 1; jb = s; i1 = 0; j1 = s; i2 = -1; j2 = s; fc = cidx(c->P, p, 0, s); nv = &g.vni; break;
                    case SCFD_SIDE_IHI: ib = ni; jb = s; i1 = ni + 1; j1 = s; i2 = ni + 2; j2 = s; fc = cidx(c->P, p, ni, s); nv = &g.vni; break;
                    case SCFD_SIDE_JLO: ib = s; jb = 1; i1 = s; j1 = 0; i2 = s; j2 = -1; fc = cidx(c->P, p, s, 0); nv = &g.vnj; break;
                    default: ib = s; jb = nj; i1 = s; j1 = nj + 1; i2 = s; j2 = nj + 2; fc = cidx(c->P, p, s, nj); nv = &g.vnj; break;
                }
                const double n1 = (*nv)[fc], n2 = (*nv)[N + fc];
                add(p, i1, j1, p, ib, jb, b.kind, (int)k, n1, n2);
                add(p, i2, j2, p, ib, jb, b.kind, (int)k, n1, n2);
            }
        }
    std::unordered_map<long long, size_t> last;
    for (size_t k = 0; k < ops.size(); ++k) last[ops[k].dst] = k;
    out.clear();
    for (size_t k = 0; k < ops.size(); ++k)
        if (last[ops[k].dst] == k) out.push_back(ops[k]);
    return 0;
}

template <typename T>
T* carve(char*& p, size_t n) {
    T* r = reinterpret_cast<T*>(p);
    size_t bytes = (n * sizeof(T) + 255) & ~(size_t)255;
    p += bytes;
    return r;
}
template <typename T>
size_t need(size_t n) {
    return (n * sizeof(T) + 255) & ~(size_t)255;
}

int sync_scalars(scfd_ctx* c) {
    CK(cudaMemcpyAsync(c->h_sc, c->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

// Runs f() (which enqueues one kernel of the given kind) between two CUDA
// events when profiling is on.
template <typename Fn>
int timed(scfd_ctx* c, int kind, Fn f) {
    if (!c->profiling) return f();
    while (c->ev_pool.size() < c->ev_used + 2) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        c->ev_pool.push_back(e);
    }
    const size_t k = c->ev_used;
    c->ev_used += 2;
    cudaEventRecord(c->ev_pool[k], c->stream);
    const int n = f();
    cudaEventRecord(c->ev_pool[k + 1], c->stream);
    c->ev_marks.push_back({kind, k});
    return n;
}

void collect_events(scfd_ctx* c) {
    if (!c->profiling || c->ev_marks.empty()) return;
    cudaStreamSynchronize(c->stream);
    for (auto& m : c->ev_marks) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev_pool[m.second], c->ev_pool[m.second + 1]);
        c->kind_ms[m.first] += ms;
        c->kind_n[m.first] += 1;
    }
    c->ev_marks.clear();
    c->ev_used = 0;
}

// Whether the residual runs the fused kernel (k_residual2.cuh) rather than the
// generic one (the conditions of launch_residual and launch_residual2).
bool fused_residual(const scfd_ctx* c) {
    const int sch = c->d.scheme;
    if (sch == SCFD_SCHEME_DUAL || precon_scheme(sch)) return false;
    if (sch != SCFD_SCHEME_EULER && !c->use_sw3) return false;
    return c->nY == 1 || c->nY == 8 || c->nY == 9;
}

// The kernels of one physical step, stage by stage; n counts the launches.
struct Seq {
    scfd_ctx* c;
    const View& v;
    cudaStream_t s;
    long long n = 0;
    explicit Seq(scfd_ctx* ctx) : c(ctx), v(ctx->v), s(ctx->stream) {}

    void primitive() { n += timed(c, SCFD_K_THERMO, [&] { return launch_thermo(v, s, c->cells_max); }); }
    void bc() {
        n += timed(c, SCFD_K_BC, [&] { return launch_ghosts(v, s, c->d_ops, c->nops, c->d_bcval, c->valstride); });
        // FP32 copies of w and vhi for the generic residual kernel (the fused one
        // rounds its tile from the FP64 state itself)
        if (v.precision == SCFD_PREC_MIXED && !fused_residual(c))
            n += timed(c, SCFD_K_OTHER, [&] { return launch_to_f32(v, s); });
    }
    void chem() {
        n += timed(c, SCFD_K_CHEM,
                   [&] { return launch_chem_impl(v, s, c->d.chem_max_substeps, c->d_counter, c->nsm, c->dq); });
    }
    void setdt() { n += timed(c, SCFD_K_DT, [&] { return launch_set_dt(v, s); }); }
    void copyq(double* dst, const double* src) {
        const long long qbytes = sizeof(double) * (long long)c->D * c->ncell;
        timed(c, SCFD_K_COPY, [&] { return (int)(cudaMemcpyAsync(dst, src, qbytes, cudaMemcpyDeviceToDevice, s) ? 0 : 0); });
    }
    void residual(int mode) {
        if (mode == RES_NR && c->d.scheme == SCFD_SCHEME_DUAL) mode = RES_DUAL;
        if (mode == RES_NR && c->d.scheme == SCFD_SCHEME_PRECON) mode = RES_PRECON;
        if (mode == RES_LUSGS && c->d.scheme == SCFD_SCHEME_PRECON_LUSGS) mode = RES_PRECON_LUSGS;
        const bool coeffs = mode != RES_EULER && !c->use_sw3;
        n += timed(c, SCFD_K_RESIDUAL, [&] { return launch_residual(v, s, mode, coeffs); });
    }
    void sweeps() {
        if (c->nsf == 0) return;  // a rank without planes
        launch_sweep_reset(s, c->d_progress, c->d_tickets, c->nsf, c->nsb);
        if (c->use_sw3) {
            n += timed(c, SCFD_K_PACK, [&] { return launch_wave(v, s, c->sw3, 0, 0); });
            n += timed(c, SCFD_K_SWEEP_FWD, [&] { return launch_wave(v, s, c->sw3, 1, 0); });
            n += timed(c, SCFD_K_SWEEP_BWD, [&] { return launch_wave(v, s, c->sw3, 2, 0); });
            if (c->d.scheme == SCFD_SCHEME_NR) n += timed(c, SCFD_K_UPDATE, [&] { return launch_wave(v, s, c->sw3, 4, 0); });
            return;
        }
        n += timed(c, SCFD_K_SWEEP_FWD, [&] {
            return launch_sweep(v, s, 0, c->d_xfer, c->d_progress, c->d_partials, c->d_tickets, c->nsf, c->nsb,
                                c->d_strips_f, c->d_strips_b);
        });
        n += timed(c, SCFD_K_SWEEP_BWD, [&] {
            return launch_sweep(v, s, 1, c->d_xfer, c->d_progress, c->d_partials, c->d_tickets, c->nsf, c->nsb,
                                c->d_strips_f, c->d_strips_b);
        });
    }
    // the (res, omega) partials of the last backward sweep: per pack block
    // (k_omega) on the wavefront path, per strip on the one-warp-per-strip path
    const double* partials() const { return c->use_sw3 ? c->sw3.partials : c->d_partials; }
    int nstrips() const { return c->use_sw3 ? c->sw3.nstrips : c->nsb; }
    // q update after the sweeps: NR relaxes with the omega reduced from
    // `part` (nparts strip partials); LU-SGS (inner = 1) adds Dq
    void update(int inner, const double* part, int nparts) {
        if (c->use_sw3) {
            if (c->nsf == 0) return;
            Wave w3 = c->sw3;
            w3.partials = const_cast<double*>(part);
            w3.nstrips = nparts;
            n += timed(c, SCFD_K_UPDATE, [&] { return launch_wave(v, s, w3, 3, inner); });
        } else if (dual_time_scheme(c->d.scheme)) {
            n += timed(c, SCFD_K_UPDATE, [&] { return launch_nr_update(v, s, part, nparts, inner); });
        }
    }
    void step_end() {
        n += timed(c, SCFD_K_OTHER, [&] { return launch_step_end(v, s, c->d.res_rate_warn, c->d.res_rate_err); });
    }
};

// the kernel sequence of one physical step
int enqueue_step(scfd_ctx* c) {
    Seq q(c);
    const View& v = c->v;
    const bool reactive = c->d.thermo == SCFD_THERMO_CHEMKIN_REACTIVE;
    if (dual_time_scheme(c->d.scheme)) {
        q.primitive();
        q.setdt();
        if (reactive) q.chem();
        q.copyq(v.qpp, v.qp);
        q.copyq(v.qp, v.q);
        for (int j = 1; j < c->d.num_internal_loop; ++j) {
            q.primitive();
            q.bc();
            q.residual(RES_NR);
            q.sweeps();
            q.update(j, q.partials(), q.nstrips());
        }
        q.step_end();
    } else {
        if (reactive) {
            q.primitive();
            q.setdt();
            q.chem();
            q.copyq(v.qp, v.q);
            q.primitive();
        } else {
            q.copyq(v.qp, v.q);
            q.primitive();
            q.setdt();
        }
        q.bc();
        if (c->d.scheme == SCFD_SCHEME_EULER) {
            q.residual(RES_EULER);
        } else {
            q.residual(RES_LUSGS);
            q.sweeps();
            q.update(1, q.partials(), q.nstrips());
        }
    }
    CK(cudaGetLastError());
    c->launches += q.n;
    return 0;
}

int fill_stats(scfd_ctx* c, scfd_stats* st, long long att0, long long fb0) {
    const DevScalars& h = *c->h_sc;
    if (st) {
        std::memset(st, 0, sizeof(*st));
        st->dt_grbl = h.dt_grbl;
        st->tt = h.tt;
        st->res = h.res;
        st->res1 = h.res1;
        st->omega = h.omega;
        st->status = h.status;
        st->inner_iters = dual_time_scheme(c->d.scheme) ? std::max(0, c->d.num_internal_loop - 1) : 0;
        st->chem_attempts = h.chem_attempts - att0;
        st->chem_fallback_cells = h.chem_fallback - fb0;
        st->res_warn = (dual_time_scheme(c->d.scheme) && h.res / h.res1 > c->d.res_rate_warn) ? 1 : 0;
    }
    return h.status;
}

}  // namespace

extern "C" {

int scfd_abi_version(void) { return SCFD_ABI_VERSION; }

int scfd_create(const scfd_desc* d, scfd_ctx** out) {
    if (!d || !out) return SCFD_E_ARG;
    if (d->abi_version != SCFD_ABI_VERSION) return SCFD_E_ARG;
    if (d->nplane < 1 || d->nplane > SCFD_MAX_PLANES || d->ny < 1 || d->ny > SCFD_MAX_SPECIES) return SCFD_E_ARG;
    if (d->scheme != SCFD_SCHEME_EULER && d->scheme != SCFD_SCHEME_LUSGS && d->scheme != SCFD_SCHEME_NR &&
        d->scheme != SCFD_SCHEME_DUAL && !precon_scheme(d->scheme))
        return SCFD_E_UNSUPPORTED;
    // precon / preconLU-SGS: 2d only, local time step (checkout_flow.py:154-160,171-177)
    if (precon_scheme(d->scheme) &&
        (d->dim != SCFD_DIM_2D || d->dt_mode != SCFD_DT_LOCAL || d->thermo == SCFD_THERMO_CHEMKIN_REACTIVE))
        return SCFD_E_UNSUPPORTED;
    if (d->scheme == SCFD_SCHEME_DUAL) {  // checkout_flow.py:159-168; no reacting variant of dual
        if (d->dim != SCFD_DIM_2D || d->dt_mode == SCFD_DT_LOCAL || d->thermo == SCFD_THERMO_CHEMKIN_REACTIVE)
            return SCFD_E_UNSUPPORTED;
        if (!(d->cfl_tau > 0.0)) return SCFD_E_ARG;
    }
    if (d->thermo == SCFD_THERMO_IDEAL && d->ny != 1) return SCFD_E_ARG;
    if (d->thermo == SCFD_THERMO_CHEMKIN_REACTIVE && d->dt_mode == SCFD_DT_LOCAL) return SCFD_E_UNSUPPORTED;
    auto* c = new scfd_ctx();
    c->d = *d;
    c->np = d->nplane;
    c->nY = d->ny;
    c->D = c->nY + 3;
    c->W = c->D + 5;
    c->P.np = c->np;
    long long base = 0;
    for (int p = 0; p < c->np; ++p) {
        const int ni = d->ni[p], nj = d->nj[p];
        if (ni < 2 || nj < 2) {
            delete c;
            return SCFD_E_ARG;
        }
        c->P.ni[p] = ni;
        c->P.nj[p] = nj;
        c->P.pitch[p] = (ni + 4 + 31) / 32 * 32;
        c->P.base[p] = base;
        base += (long long)(nj + 4) * c->P.pitch[p];
        base = (base + 31) / 32 * 32;
        c->nimax = std::max(c->nimax, ni);
        c->njmax = std::max(c->njmax, nj);
        c->cells_max = std::max(c->cells_max, ni * nj);
    }
    c->ncell = base;
    c->xh.resize(c->np);
    c->rh.resize(c->np);
    c->geo_set.assign(c->np, 0);
    *out = c;
    return 0;
}

int scfd_destroy(scfd_ctx* c) {
    if (!c) return SCFD_E_ARG;
    for (auto& g : c->adj.rev_graph)
        if (g) cudaGraphExecDestroy(g);
    for (void* b : {(void*)c->adj.slots, (void*)c->adj.lam, (void*)c->adj.wbar, (void*)c->adj.dgrad, (void*)c->adj.dJ,
                    (void*)c->adj.ocells, (void*)c->adj.owt})
        if (b) cudaFree(b);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    for (int b = 0; b < 2; ++b) {
        if (c->h_ring[b]) cudaFreeHost(c->h_ring[b]);
        if (c->ring_ev[b]) cudaEventDestroy(c->ring_ev[b]);
    }
    for (auto e : c->ev_pool) cudaEventDestroy(e);
    if (c->arena) cudaFree(c->arena);
    if (c->h_sc) cudaFreeHost(c->h_sc);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return 0;
}

int scfd_last_error(const scfd_ctx* c, char* buf, int len) {
    if (!c || !buf || len <= 0) return SCFD_E_ARG;
    std::snprintf(buf, (size_t)len, "%s", c->err.c_str());
    return 0;
}

int scfd_set_geometry(scfd_ctx* c, int plane, const double* xh, const double* rh) {
    if (!c || plane < 1 || plane > c->np || !xh || !rh) return SCFD_E_ARG;
    if (c->committed) return c->fail(SCFD_E_STATE, "geometry after commit");
    const size_t n = (size_t)(c->P.ni[plane - 1] + 1) * (c->P.nj[plane - 1] + 1);
    c->xh[plane - 1].assign(xh, xh + n);
    c->rh[plane - 1].assign(rh, rh + n);
    c->geo_set[plane - 1] = 1;
    return 0;
}

int scfd_set_connectivity(scfd_ctx* c, const int32_t* recs, int n) {
    if (!c || n < 0 || (n > 0 && !recs)) return SCFD_E_ARG;
    if (c->committed) return c->fail(SCFD_E_STATE, "connectivity after commit");
    c->cut.assign(recs, recs + 11 * (size_t)n);
    return 0;
}

int scfd_set_bc(scfd_ctx* c, const scfd_bc* b, int n) {
    if (!c || n < 0 || (n > 0 && !b)) return SCFD_E_ARG;
    if (c->committed) return c->fail(SCFD_E_STATE, "boundaries after commit");
    for (int k = 0; k < n; ++k) {
        const scfd_bc& x = b[k];
        if (x.plane < 1 || x.plane > c->np || x.side < 0 || x.side > 3 || x.kind < 0 || x.kind > SCFD_BC_FIXED_PIN)
            return c->fail(SCFD_E_ARG, "bad boundary descriptor " + std::to_string(k));
        const int len = (x.side <= SCFD_SIDE_IHI) ? c->P.nj[x.plane - 1] : c->P.ni[x.plane - 1];
        if (x.first < 1 || x.last > len || x.first > x.last)
            return c->fail(SCFD_E_ARG, "boundary descriptor range " + std::to_string(k));
    }
    c->bcs.assign(b, b + n);
    return 0;
}

int scfd_set_chem(scfd_ctx* c, const scfd_chem* ch) {
    if (!c || !ch) return SCFD_E_ARG;
    if (ch->ns != c->nY || ch->nr < 1 || ch->nr > SCFD_MAX_REACTIONS || ch->nt < 0 || ch->nt > ch->ns)
        return c->fail(SCFD_E_ARG, "chemistry tables do not match nY");
    c->chem = *ch;
    c->have_chem = true;
    return 0;
}

int scfd_commit(scfd_ctx* c) {
    if (!c) return SCFD_E_ARG;
    if (c->committed) return c->fail(SCFD_E_STATE, "commit called twice");
    for (int p = 0; p < c->np; ++p)
        if (!c->geo_set[p]) return c->fail(SCFD_E_STATE, "geometry of plane " + std::to_string(p + 1) + " not set");
    if (c->d.thermo != SCFD_THERMO_IDEAL && !c->have_chem) return c->fail(SCFD_E_STATE, "chemistry tables not set");
    CK(cudaGetDevice(&c->device));
    CK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    HostGeo g;
    build_geometry(c, g);
    c->h_dsi = g.dsi;
    c->h_dsj = g.dsj;
    std::vector<GhostOp> ops;
    int st = build_ghost_ops(c, g, ops);
    if (st) return st;
    // planes this rank updates
    c->P.nact = 0;
    for (int p = 0; p < c->np; ++p)
        if (c->own(p)) c->P.act[c->P.nact++] = p;
    // Block sharding: every rank keeps the ghost writes of its own planes.  The
    // halo copies among them whose source cell lies on another rank's plane
    // read that cell from the exchange buffer: rank q exports, in slot order,
    // every cell of its planes that a halo copy onto another rank's plane
    // reads; each rank imports the exported cells its own copies read.
    std::vector<long long> exp_cells;
    std::vector<HaloImport> imps;
    if (!c->owner.empty()) {
        auto plane_of = [&](long long slot) {
            int p = 0;
            while (p + 1 < c->np && c->P.base[p + 1] <= slot) ++p;
            return p;
        };
        std::vector<std::vector<long long>> ex(c->nranks);
        for (const GhostOp& o : ops) {
            if (o.kind != -1) continue;
            const int q = c->owner[plane_of(o.src)];
            if (c->owner[plane_of(o.dst)] != q) ex[q].push_back(o.src);
        }
        size_t mx = 0;
        for (auto& e : ex) {
            std::sort(e.begin(), e.end());
            e.erase(std::unique(e.begin(), e.end()), e.end());
            mx = std::max(mx, e.size());
        }
        c->seg = (long long)mx * (c->W + c->nY);
        exp_cells = ex[c->rank];
        std::vector<GhostOp> mine;
        std::vector<long long> reads;
        for (const GhostOp& o : ops)
            if (c->own(plane_of(o.dst))) {
                mine.push_back(o);
                reads.push_back(o.src);
            }
        ops.swap(mine);
        std::sort(reads.begin(), reads.end());
        for (int q = 0; q < c->nranks; ++q) {
            if (q == c->rank) continue;
            const long long n = (long long)ex[q].size();
            for (long long t = 0; t < n; ++t)
                if (std::binary_search(reads.begin(), reads.end(), ex[q][t]))
                    imps.push_back(HaloImport{ex[q][t], q * c->seg + t, n});
        }
    }
    c->nexp = (int)exp_cells.size();
    c->nimp = (int)imps.size();
    c->nops = (int)ops.size();
    // strips for the sweeps
    std::vector<int> sf, sb;
    for (int p = 0; p < c->np; ++p) {
        if (!c->own(p)) continue;
        const int ns = (c->P.nj[p] + 31) / 32;
        for (int s = 0; s < ns; ++s) {
            sf.push_back(p);
            sf.push_back(s);
        }
    }
    sb = sf;
    c->nsf = (int)sf.size() / 2;
    c->nsb = c->nsf;
    const long long N = c->ncell;
    const int D = c->D, W = c->W, nY = c->nY;
    const bool mixed = c->d.precision == SCFD_PREC_MIXED;
    const bool impl = c->d.scheme != SCFD_SCHEME_EULER;
    // chemistry tables, compact
    const ChemTables tabs = c->have_chem ? ChemTables(c->chem) : ChemTables();
    const int nrec = 64 * c->np;
    // strip records for the cluster-wavefront sweeps
    // the dual and precon schemes take the generic residual and sweeps
    const bool dual = c->d.scheme == SCFD_SCHEME_DUAL || precon_scheme(c->d.scheme);
    const WaveSizes wz = impl && !dual ? wave_sizes(nY, mixed) : WaveSizes{0, 0, 0, 0};
    const size_t esz3 = mixed ? sizeof(float) : sizeof(double);
    const bool legacy = std::getenv("SCFD_SWEEP_LEGACY") != nullptr;
    const char* graph_env = std::getenv("SCFD_GRAPH");
    c->use_graph = !(graph_env && std::strcmp(graph_env, "0") == 0);
    const int ncl_max = wz.xs > 0 && !legacy ? wave_max_clusters(nY, mixed) : 0;
    c->use_sw3 = wz.xs > 0 && !legacy && ncl_max > 0;
    std::vector<long long> step_off;
    std::vector<int> blks3, strips3, tasksf, tasksb;
    long long steps_total = 0;
    if (c->use_sw3) {
        const int pad = wave_pad_steps(), tpc = wave_strips_per_task();
        int fs = 0;
        for (int pl = 0; pl < c->np; ++pl) {
            if (!c->own(pl)) continue;
            const int ns = (c->P.nj[pl] + 31) / 32, steps = c->P.ni[pl] + 31;
            const int fs_plane = fs;
            for (int st3 = 0; st3 < ns; ++st3, ++fs) {
                step_off.push_back(steps_total);
                steps_total += steps + 2 * pad;
                for (int t0 = 0; t0 < steps; t0 += 32) {
                    blks3.push_back(fs);
                    blks3.push_back(t0);
                }
                strips3.insert(strips3.end(), {pl, st3, fs, 0});
            }
            // tasks of up to tpc strips: forward from the bottom, backward from the top
            for (int s0 = 0; s0 < ns; s0 += tpc) tasksf.insert(tasksf.end(), {pl, s0, std::min(tpc, ns - s0), fs_plane});
            for (int s0 = ns - 1; s0 >= 0; s0 -= tpc) tasksb.insert(tasksb.end(), {pl, s0, std::min(tpc, s0 + 1), fs_plane});
        }
    }
    const int ntasks = (int)tasksf.size() / 4;
    const int hk = wave_handoff_chunk();
    const long long xstride3 = (long long)wave_chunks(c->nimax) * hk * std::max(1, wz.d4);
    // arena size
    size_t bytes = 0;
    bytes += 3 * need<double>(D * N);                         // q, qp, qpp
    bytes += need<double>(W * N) + 2 * need<double>(nY * N);  // w, vhi, DHi
    bytes += need<double>(D * N);                             // Dq
    bytes += 4 * need<double>(N);                             // dt_mat, alpha, nuA, nuB
    if (dual) bytes += need<double>(4 * N);                   // pre_sca
    bytes += 8 * need<double>(N) + 4 * need<double>(2 * N) + 3 * need<double>(4 * N);  // geometry
    if (mixed) bytes += need<float>(W * N) + need<float>(nY * N);
    bytes += need<DevScalars>(1);
    bytes += 2 * need<int>(2 * c->nsf);
    bytes += need<double>((size_t)c->nsf * (c->nimax + 8) * D);
    bytes += need<int>(c->nsf + c->nsb) + need<int>(2) + need<double>(2 * std::max<size_t>(c->nsb, blks3.size() / 2));
    bytes += need<GhostOp>(std::max(1, c->nops)) + need<double>(std::max<size_t>(1, c->bcs.size()) * c->valstride);
    bytes += need<long long>(std::max(1, c->nexp)) + need<HaloImport>(std::max(1, c->nimp)) +
             need<double>(std::max<long long>(1, c->seg * c->nranks)) + need<double>(8);
    bytes += need<unsigned long long>(1) + need<double>(nrec) + need<double>(1);
    bytes += tabs.bytes();
    long long dq_cap = 0;  // interior cells of the updated planes
    for (int a = 0; a < c->P.nact; ++a) dq_cap += (long long)c->P.ni[c->P.act[a]] * c->P.nj[c->P.act[a]];
    if (c->have_chem)
        bytes += need<long long>(dq_cap) + need<double>(dq_cap) + need<double>((size_t)dq_cap * (c->chem.ns + 1)) +
                 need<unsigned long long>(2);
    const size_t nref = (size_t)(c->nimax + 4) * (c->njmax + 4) * c->np;
    bytes += need<double>((size_t)std::max(std::max(W, D), nY) * nref);
    if (c->use_sw3)
        bytes += need<char>(steps_total * wz.xs * esz3) + need<char>(steps_total * wz.cs * esz3) +
                 need<long long>(step_off.size()) + need<int>(blks3.size()) + need<int>(strips3.size()) +
                 need<int>(tasksf.size()) + need<int>(tasksb.size()) + need<double>((size_t)ntasks * xstride3);
    bytes += 64 * 256;
    c->arena_bytes = bytes;
    CK(cudaMalloc(&c->arena, bytes));
    CK(cudaMemsetAsync(c->arena, 0, bytes, c->stream));
    char* p = c->arena;
    View& v = c->v;
    v.base = reinterpret_cast<double*>(c->arena);
    v.P = c->P;
    v.ncell = N;
    v.nY = nY; v.D = D; v.W = W;
    v.dim = c->d.dim; v.viscous = c->d.viscous; v.recon = c->d.recon; v.thermo = c->d.thermo;
    v.mu_model = c->d.mu_model; v.scheme = c->d.scheme; v.dt_mode = c->d.dt_mode; v.precision = c->d.precision;
    v.phi_mus = c->d.phi_mus; v.k_mus = c->d.k_mus; v.kappa = c->d.kappa; v.rgas = c->d.rgas; v.nu_gas = c->d.nu_gas;
    v.suth_mu0 = c->d.suth_mu0; v.suth_t0 = c->d.suth_t0; v.suth_s = c->d.suth_s;
    v.prandtl = c->d.prandtl; v.schmidt = c->d.schmidt; v.cfl = c->d.cfl; v.dt_fixed = c->d.dt_fixed;
    v.omega_max = c->d.omega_max; v.omega_min = c->d.omega_min; v.dq_max = c->d.dq_max;
    v.q = carve<double>(p, D * N); v.qp = carve<double>(p, D * N); v.qpp = carve<double>(p, D * N);
    v.w = carve<double>(p, W * N); v.vhi = carve<double>(p, nY * N); v.DHi = carve<double>(p, nY * N);
    v.Dq = carve<double>(p, D * N);
    v.dt_mat = carve<double>(p, N); v.alpha = carve<double>(p, N); v.nuA = carve<double>(p, N); v.nuB = carve<double>(p, N);
    v.pre = dual ? carve<double>(p, 4 * N) : nullptr;
    v.cfl_tau = c->d.cfl_tau;
    v.res_tile = 0;
    v.thermo_block = 128;
    v.Vol = carve<double>(p, N); v.Area = carve<double>(p, N); v.dsi = carve<double>(p, N); v.dsj = carve<double>(p, N);
    v.x = carve<double>(p, N); v.r = carve<double>(p, N); v.dsci = carve<double>(p, N); v.dscj = carve<double>(p, N);
    v.vni = carve<double>(p, 2 * N); v.vnj = carve<double>(p, 2 * N); v.vnci = carve<double>(p, 2 * N); v.vncj = carve<double>(p, 2 * N);
    v.gjc = carve<double>(p, 4 * N); v.gji = carve<double>(p, 4 * N); v.gjj = carve<double>(p, 4 * N);
    if (mixed) {
        v.w32 = carve<float>(p, W * N);
        v.vhi32 = carve<float>(p, nY * N);
    }
    c->d_sc = carve<DevScalars>(p, 1);
    v.sc = c->d_sc;
    c->d_strips_f = carve<int>(p, 2 * c->nsf);
    c->d_strips_b = carve<int>(p, 2 * c->nsb);
    c->d_xfer = carve<double>(p, (size_t)c->nsf * (c->nimax + 8) * D);
    c->d_progress = carve<int>(p, c->nsf + c->nsb);
    c->d_tickets = carve<int>(p, 2);
    c->d_partials = carve<double>(p, 2 * std::max<size_t>(c->nsb, blks3.size() / 2));
    c->d_ops = carve<GhostOp>(p, std::max(1, c->nops));
    c->d_exp = carve<long long>(p, std::max(1, c->nexp));
    c->d_imp = carve<HaloImport>(p, std::max(1, c->nimp));
    c->d_halo = carve<double>(p, std::max<long long>(1, c->seg * c->nranks));
    c->d_red = carve<double>(p, 8);
    c->d_bcval = carve<double>(p, std::max<size_t>(1, c->bcs.size()) * c->valstride);
    c->d_counter = carve<unsigned long long>(p, 1);
    if (c->have_chem) {
        c->dq.cell = carve<long long>(p, dq_cap);
        c->dq.tt = carve<double>(p, dq_cap);
        c->dq.y = carve<double>(p, (size_t)dq_cap * (c->chem.ns + 1));
        c->dq.count = carve<unsigned long long>(p, 2);
        c->dq.capacity = dq_cap;
        c->dq.warp_doubles = (int)chem_dvode_warp_doubles(c->chem.ns, c->chem.nr);
        const int e = chem_dvode_setup(c->chem.ns, c->chem.nr, &c->dq.warps_per_block);
        if (e) return c->fail(SCFD_E_CUDA, std::string("DVODE kernel setup: ") + cudaGetErrorString((cudaError_t)e));
    }
    c->d_rms_partial = carve<double>(p, nrec);
    c->d_rms_out = carve<double>(p, 1);
    c->d_ref = carve<double>(p, (size_t)std::max(std::max(W, D), nY) * nref);
    for (int b = 0; b < 2; ++b) {
        CK(cudaMallocHost(&c->h_ring[b], kRingChunk));
        CK(cudaEventCreateWithFlags(&c->ring_ev[b], cudaEventDisableTiming));
    }
    if (c->use_sw3) {
        Wave& w3 = c->sw3;
        w3.X = carve<char>(p, steps_total * wz.xs * esz3);
        w3.C = carve<char>(p, steps_total * wz.cs * esz3);
        long long* so = carve<long long>(p, step_off.size());
        int* bk = carve<int>(p, blks3.size());
        int* sp = carve<int>(p, strips3.size());
        int* tf = carve<int>(p, tasksf.size());
        int* tb = carve<int>(p, tasksb.size());
        w3.xfer = carve<double>(p, (size_t)ntasks * xstride3);
        CK(cudaMemcpyAsync(so, step_off.data(), step_off.size() * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(bk, blks3.data(), blks3.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(sp, strips3.data(), strips3.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(tf, tasksf.data(), tasksf.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(tb, tasksb.data(), tasksb.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        w3.step_off = so;
        w3.blk = reinterpret_cast<const int2*>(bk);
        w3.nblk = (int)blks3.size() / 2;
        w3.strips = reinterpret_cast<const int4*>(sp);
        w3.nstrips = w3.nblk;  // k_omega's partials: one per pack block
        w3.tasks_f = reinterpret_cast<const int4*>(tf);
        w3.tasks_b = reinterpret_cast<const int4*>(tb);
        w3.ntasks = ntasks;
        w3.nclusters = std::min(ntasks, ncl_max);
        w3.xstride = xstride3;
        w3.progress = c->d_progress;
        w3.tickets = c->d_tickets;
        w3.partials = c->d_partials;
        CK(cudaStreamSynchronize(c->stream));
    }
    if (p > c->arena + c->arena_bytes) return c->fail(SCFD_E_CUDA, "arena overflow");
    // geometry upload
    auto up = [&](double* d, const std::vector<double>& h) {
        return cudaMemcpyAsync(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    };
    CK(up(v.Vol, g.Vol)); CK(up(v.Area, g.Area)); CK(up(v.dsi, g.dsi)); CK(up(v.dsj, g.dsj));
    CK(up(v.vni, g.vni)); CK(up(v.vnj, g.vnj)); CK(up(v.x, g.x)); CK(up(v.r, g.r));
    CK(up(v.gjc, g.gjc)); CK(up(v.gji, g.gji)); CK(up(v.gjj, g.gjj)); CK(up(v.dsci, g.dsci)); CK(up(v.dscj, g.dscj));
    CK(up(v.vnci, g.vnci)); CK(up(v.vncj, g.vncj));
    CK(cudaMemcpyAsync(c->d_strips_f, sf.data(), sf.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_strips_b, sb.data(), sb.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    if (c->nops)
        CK(cudaMemcpyAsync(c->d_ops, ops.data(), ops.size() * sizeof(GhostOp), cudaMemcpyHostToDevice, c->stream));
    if (c->nexp)
        CK(cudaMemcpyAsync(c->d_exp, exp_cells.data(), exp_cells.size() * sizeof(long long), cudaMemcpyHostToDevice,
                           c->stream));
    if (c->nimp)
        CK(cudaMemcpyAsync(c->d_imp, imps.data(), imps.size() * sizeof(HaloImport), cudaMemcpyHostToDevice, c->stream));
    if (!c->bcs.empty()) {
        std::vector<double> val(c->bcs.size() * c->valstride);
        for (size_t k = 0; k < c->bcs.size(); ++k)
            std::memcpy(&val[k * c->valstride], c->bcs[k].value, sizeof(double) * c->valstride);
        CK(cudaMemcpyAsync(c->d_bcval, val.data(), val.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    if (c->have_chem) {
        CK(tabs.upload(v.chem, p, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    if (p > c->arena + c->arena_bytes) return c->fail(SCFD_E_CUDA, "arena overflow");
    CK(cudaMallocHost(&c->h_sc, sizeof(DevScalars)));
    CK(cudaStreamSynchronize(c->stream));
    (void)impl;
    c->committed = true;
    return 0;
}

// reference layout f(k, -1:nimax+2, -1:njmax+2, plane) <-> SoA slots
// Host <-> device copies of the caller's arrays.  Page-locked arrays (the
// caller's cudaHostRegister or cudaMallocHost memory) are moved by the DMA
// engine directly; pageable ones go through two pinned chunks: the host threads
// copy one chunk while the DMA engine moves the other.

// true when [p, p + bytes) starts and ends in page-locked host memory
static bool page_locked(const void* p, size_t bytes) {
    if (!p || bytes == 0) return false;
    for (const char* q : {static_cast<const char*>(p), static_cast<const char*>(p) + bytes - 1}) {
        cudaPointerAttributes a{};
        if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
            cudaGetLastError();  // an unknown pointer is pageable memory, not an error
            return false;
        }
        if (a.type != cudaMemoryTypeHost) return false;
    }
    return true;
}

static void par_copy(void* dst, const void* src, size_t bytes) {
    const size_t piece = 1ull << 20;
    const long long n = (long long)((bytes + piece - 1) / piece);
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < n; ++k) {
        const size_t off = (size_t)k * piece, len = std::min(piece, bytes - off);
        std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, len);
    }
}

static int h2d_pipelined(scfd_ctx* c, void* dev, const void* host, size_t bytes) {
    if (page_locked(host, bytes)) {
        CK(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, c->stream));
        return 0;
    }
    size_t off = 0;
    for (int k = 0; off < bytes; ++k) {
        const int b = k & 1;
        const size_t len = std::min(kRingChunk, bytes - off);
        CK(cudaEventSynchronize(c->ring_ev[b]));  // the copy that last read chunk b has finished
        par_copy(c->h_ring[b], static_cast<const char*>(host) + off, len);
        CK(cudaMemcpyAsync(static_cast<char*>(dev) + off, c->h_ring[b], len, cudaMemcpyHostToDevice, c->stream));
        CK(cudaEventRecord(c->ring_ev[b], c->stream));
        off += len;
    }
    return 0;
}

static int d2h_pipelined(scfd_ctx* c, void* host, const void* dev, size_t bytes) {
    if (page_locked(host, bytes)) {
        CK(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return 0;
    }
    size_t off = 0, prev_off = 0, prev_len = 0;
    int k = 0;
    for (; off < bytes; ++k) {
        const int b = k & 1;
        const size_t len = std::min(kRingChunk, bytes - off);
        CK(cudaMemcpyAsync(c->h_ring[b], static_cast<const char*>(dev) + off, len, cudaMemcpyDeviceToHost,
                           c->stream));
        CK(cudaEventRecord(c->ring_ev[b], c->stream));
        if (k > 0) {  // the previous chunk has landed: copy it out while this one moves
            CK(cudaEventSynchronize(c->ring_ev[b ^ 1]));
            par_copy(static_cast<char*>(host) + prev_off, c->h_ring[b ^ 1], prev_len);
        }
        prev_off = off;
        prev_len = len;
        off += len;
    }
    if (k > 0) {
        CK(cudaEventSynchronize(c->ring_ev[(k - 1) & 1]));
        par_copy(static_cast<char*>(host) + prev_off, c->h_ring[(k - 1) & 1], prev_len);
    }
    return 0;
}

// The reference-layout arrays cross PCIe unchanged into a device staging
// buffer (d_ref) and are transposed to / from the cell slots on the GPU.
static int upload_field(scfd_ctx* c, const double* ref, int nk, double* dev) {
    const int IX = c->nimax + 4, JX = c->njmax + 4;
    const size_t bytes = sizeof(double) * (size_t)nk * IX * JX * c->np;
    int st = h2d_pipelined(c, c->d_ref, ref, bytes);
    if (st) return st;
    launch_ref_soa(c->v, c->stream, nk, IX, JX, c->d_ref, dev, nullptr, 0);
    CK(cudaGetLastError());
    return 0;
}
static int download_field(scfd_ctx* c, const double* dev, int nk, double* ref) {
    const int IX = c->nimax + 4, JX = c->njmax + 4;
    const size_t bytes = sizeof(double) * (size_t)nk * IX * JX * c->np;
    launch_ref_soa(c->v, c->stream, nk, IX, JX, nullptr, const_cast<double*>(dev), c->d_ref, 1);
    CK(cudaGetLastError());
    return d2h_pipelined(c, ref, c->d_ref, bytes);
}

int scfd_upload(scfd_ctx* c, const double* q, const double* w, const double* vhi, double tt) {
    if (!c || !q || !w) return SCFD_E_ARG;
    if (!c->committed) return c->fail(SCFD_E_STATE, "upload before commit");
    int st;
    if ((st = upload_field(c, q, c->D, c->v.q))) return st;
    if ((st = upload_field(c, w, c->W, c->v.w))) return st;
    if (vhi && (st = upload_field(c, vhi, c->nY, c->v.vhi))) return st;
    const long long qb = sizeof(double) * (long long)c->D * c->ncell;
    CK(cudaMemcpyAsync(c->v.qp, c->v.q, qb, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->v.qpp, c->v.q, qb, cudaMemcpyDeviceToDevice, c->stream));
    DevScalars h{};
    h.tt = tt;
    h.first_dual = 1;
    h.res1 = 1.0;
    CK(cudaMemcpyAsync(c->d_sc, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->uploaded = true;
    c->ds_stage = 0;
    return 0;
}

int scfd_prepare(scfd_ctx* c, int step) {
    if (!c || !c->committed || !c->uploaded) return c ? c->fail(SCFD_E_STATE, "prepare before upload") : SCFD_E_ARG;
    (void)step;
    c->launches = 0;
    c->launches += launch_thermo(c->v, c->stream, c->cells_max);
    c->launches += launch_ghosts(c->v, c->stream, c->d_ops, c->nops, c->d_bcval, c->valstride);
    CK(cudaGetLastError());
    int st = sync_scalars(c);
    if (st) return st;
    return c->h_sc->status;
}

// ---------------------------------------------------------------------------
// Autotuner: picks the residual tile shape and the thermo CTA size for this
// context by timing every candidate (CUDA events, 1 warm-up + 3 timed launches)
// on the context's state.  The kernels under test overwrite q..nuB and the
// scalars, which are saved first and restored after.  Runs once, before the
// first step is enqueued (so a captured graph holds the chosen shapes).
// ---------------------------------------------------------------------------
static int autotune(scfd_ctx* c) {
    c->tuned = true;
    View& v = c->v;
    v.res_tile = 0;
    v.thermo_block = 128;
    const char* env = std::getenv("SCFD_AUTOTUNE");
    if (env && std::strcmp(env, "0") == 0) {
        c->tune_report = "{\"enabled\": false, \"residual_tile\": \"32x8\", \"thermo_block\": 128}";
        return 0;
    }
    cudaStream_t s = c->stream;
    const size_t bytes = (size_t)((char*)v.Vol - (char*)v.q);
    char* save = nullptr;
    if (cudaMalloc(&save, bytes + sizeof(DevScalars)) != cudaSuccess) {
        cudaGetLastError();
        c->tune_report = "{\"enabled\": false, \"reason\": \"no memory for the state copy\"}";
        return 0;
    }
    CK(cudaMemcpyAsync(save, v.q, bytes, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(save + bytes, v.sc, sizeof(DevScalars), cudaMemcpyDeviceToDevice, s));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto time3 = [&](auto launch) {
        launch();
        cudaEventRecord(e0, s);
        for (int r = 0; r < 3; ++r) launch();
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms / 3.0f;
    };
    char buf[512];
    std::string rep = "{\"enabled\": true";
    // residual: the fused kernel of the strip-record path (not the generic one)
    const int mode = c->d.scheme == SCFD_SCHEME_EULER ? RES_EULER : c->d.scheme == SCFD_SCHEME_LUSGS ? RES_LUSGS : RES_NR;
    const bool fused = c->d.scheme != SCFD_SCHEME_DUAL && !precon_scheme(c->d.scheme) &&
                       (mode == RES_EULER || c->use_sw3) &&
                       (c->nY == 1 || c->nY == 8 || c->nY == 9) && c->P.nact > 0;
    const char* force = std::getenv("SCFD_RES_TILE");  // pins the tile (index), e.g. for profiling
    int tx[8], ty[8];
    const int nt = residual2_tiles(tx, ty);
    if (fused && force && std::atoi(force) >= 0 && std::atoi(force) < nt) {
        v.res_tile = std::atoi(force);
        std::snprintf(buf, sizeof(buf), ", \"residual_tile\": \"%dx%d\", \"residual_forced\": true", tx[v.res_tile],
                      ty[v.res_tile]);
        rep += buf;
    } else if (fused) {
        if (v.precision == SCFD_PREC_MIXED) launch_to_f32(v, s);
        float best = 1e30f;
        int pick = 0;
        rep += ", \"residual_ms\": {";
        for (int k = 0; k < nt; ++k) {
            v.res_tile = k;
            const float ms = time3([&] { launch_residual2(v, s, mode); });
            std::snprintf(buf, sizeof(buf), "%s\"%dx%d\": %.4f", k ? ", " : "", tx[k], ty[k], ms);
            rep += buf;
            if (ms < best) {
                best = ms;
                pick = k;
            }
        }
        v.res_tile = pick;
        std::snprintf(buf, sizeof(buf), "}, \"residual_tile\": \"%dx%d\"", tx[pick], ty[pick]);
        rep += buf;
    }
    if (c->P.nact > 0) {
        const int cand[3] = {64, 128, 256};
        float best = 1e30f;
        int pick = 128;
        rep += ", \"thermo_ms\": {";
        for (int k = 0; k < 3; ++k) {
            v.thermo_block = cand[k];
            const float ms = time3([&] { launch_thermo(v, s, c->cells_max); });
            std::snprintf(buf, sizeof(buf), "%s\"%d\": %.4f", k ? ", " : "", cand[k], ms);
            rep += buf;
            if (ms < best) {
                best = ms;
                pick = cand[k];
            }
        }
        v.thermo_block = pick;
        std::snprintf(buf, sizeof(buf), "}, \"thermo_block\": %d", pick);
        rep += buf;
    }
    rep += "}";
    CK(cudaMemcpyAsync(v.q, save, bytes, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(v.sc, save + bytes, sizeof(DevScalars), cudaMemcpyDeviceToDevice, s));
    CK(cudaStreamSynchronize(s));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(save);
    CK(cudaGetLastError());
    c->tune_report = rep;
    return 0;
}

// One physical step.  The first step of a context runs eagerly (it also sets
// the kernels' shared-memory attributes); the second is captured into a CUDA
// graph, which every later step replays with one launch.  The graph holds
// device pointers and host constants of the context only: dt, time and status
// live on the device.  Profiled steps run eagerly (their events are recorded
// between the kernels).
int step_once(scfd_ctx* c) {
    if (!c->tuned) {
        const int st = autotune(c);
        if (st) return st;
    }
    if (c->profiling || !c->use_graph || c->eager_steps < 1) {
        ++c->eager_steps;
        return enqueue_step(c);
    }
    if (!c->graph) {
        const long long before = c->launches;
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const int st = enqueue_step(c);
        const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (st) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return c->fail(SCFD_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        const cudaError_t ei = cudaGraphInstantiate(&c->graph, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            c->graph = nullptr;
            return c->fail(SCFD_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
        }
        c->graph_launches = c->launches - before;
        c->launches = before;
    }
    CK(cudaGraphLaunch(c->graph, c->stream));
    c->launches += c->graph_launches;
    return 0;
}

int scfd_step(scfd_ctx* c, int step, scfd_stats* stats) {
    if (!c || !c->committed || !c->uploaded) return c ? c->fail(SCFD_E_STATE, "step before upload") : SCFD_E_ARG;
    if (c->nranks > 1) return c->fail(SCFD_E_STATE, "partitioned context: step through scfd_dstep");
    (void)step;
    int st = sync_scalars(c);
    if (st) return st;
    const long long att0 = c->h_sc->chem_attempts, fb0 = c->h_sc->chem_fallback;
    c->launches = 0;
    if ((st = step_once(c))) return st;
    if ((st = sync_scalars(c))) return st;
    collect_events(c);
    return fill_stats(c, stats, att0, fb0);
}

int scfd_run(scfd_ctx* c, int step, int nsteps, scfd_stats* stats) {
    if (!c || !c->committed || !c->uploaded) return c ? c->fail(SCFD_E_STATE, "run before upload") : SCFD_E_ARG;
    if (c->nranks > 1) return c->fail(SCFD_E_STATE, "partitioned context: step through scfd_dstep");
    (void)step;
    int st = sync_scalars(c);
    if (st) return st;
    const long long att0 = c->h_sc->chem_attempts, fb0 = c->h_sc->chem_fallback;
    c->launches = 0;
    for (int n = 0; n < nsteps; ++n) {
        if ((st = step_once(c))) return st;
        if (c->profiling && c->ev_used > 4096) collect_events(c);
    }
    if ((st = sync_scalars(c))) return st;
    collect_events(c);
    // the chemistry counts of the last step (a run of no step reports none)
    const DevScalars& h = *c->h_sc;
    const bool any = nsteps > 0 && (h.chem_attempts != att0 || h.chem_fallback != fb0);
    return fill_stats(c, stats, any ? h.chem_attempts - h.chem_attempts_last : h.chem_attempts,
                      any ? h.chem_fallback - h.chem_fallback_last : h.chem_fallback);
}

int scfd_set_partition(scfd_ctx* c, const int32_t* owner, int nranks, int rank) {
    if (!c || !owner || nranks < 1 || nranks > SCFD_MAX_RANKS || rank < 0 || rank >= nranks) return SCFD_E_ARG;
    if (c->committed) return c->fail(SCFD_E_STATE, "partition after commit");
    for (int p = 0; p < c->np; ++p)
        if (owner[p] < 0 || owner[p] >= nranks) return c->fail(SCFD_E_ARG, "plane owner out of range");
    c->owner.assign(owner, owner + c->np);
    c->nranks = nranks;
    c->rank = rank;
    return 0;
}

// Stages of scfd_dstep: the kernel sequence of enqueue_step cut at the points
// where the ranks exchange halo cells or reduce scalars.  The device carries
// on whatever the status; every rank issues the same requests.
enum { DS_BEGIN = 0, DS_AFTER_DT, DS_INNER, DS_AFTER_HALO_NR, DS_AFTER_RES, DS_AFTER_HALO, DS_AFTER_STATUS };

int scfd_dstep(scfd_ctx* c, int step, scfd_dreq* req, scfd_stats* stats) {
    if (!c || !req) return SCFD_E_ARG;
    req->kind = SCFD_DREQ_DONE;
    req->buf = nullptr;
    if (!c->committed || !c->uploaded) return c->fail(SCFD_E_STATE, "dstep before upload");
    (void)step;
    const bool nr = dual_time_scheme(c->d.scheme);
    const bool reactive = c->d.thermo == SCFD_THERMO_CHEMKIN_REACTIVE;
    const View& v = c->v;
    cudaStream_t s = c->stream;
    Seq q(c);
    auto reduce = [&](int nsum, int nmin, int next) {
        req->kind = SCFD_DREQ_REDUCE;
        req->nsum = nsum;
        req->nmin = nmin;
        req->buf = c->d_red;
        c->ds_stage = next;
    };
    auto exchange = [&](int next) {
        q.n += launch_halo_pack(v, s, c->d_exp, c->nexp, c->d_halo + (long long)c->rank * c->seg);
        req->kind = SCFD_DREQ_HALO;
        req->nranks = c->nranks;
        req->seg = c->seg;
        req->buf = c->d_halo;
        c->ds_stage = next;
    };
    bool finished = false;
    for (bool more = true; more;) {
        more = false;
        switch (c->ds_stage) {
            case DS_BEGIN: {
                if (!c->tuned) {
                    const int st0 = autotune(c);
                    if (st0) return st0;
                }
                const int st = sync_scalars(c);
                if (st) return st;
                c->ds_att0 = c->h_sc->chem_attempts;
                c->ds_fb0 = c->h_sc->chem_fallback;
                c->launches = 0;
                if (!nr && !reactive) q.copyq(v.qp, v.q);
                q.primitive();
                q.n += timed(c, SCFD_K_DT, [&] { return launch_set_dt_cells(v, s); });
                q.n += launch_dt_export(v, s, c->d_red);
                reduce(0, 2, DS_AFTER_DT);
                break;
            }
            case DS_AFTER_DT:
                q.n += launch_dt_import(v, s, c->d_red);
                if (reactive) q.chem();
                if (nr) {
                    q.copyq(v.qpp, v.qp);
                    q.copyq(v.qp, v.q);
                    c->ds_j = 1;
                    c->ds_stage = DS_INNER;
                    more = true;
                    break;
                }
                if (reactive) {
                    q.copyq(v.qp, v.q);
                    q.primitive();
                }
                exchange(DS_AFTER_HALO);
                break;
            case DS_INNER:
                if (c->ds_j >= c->d.num_internal_loop) {
                    q.step_end();
                    finished = true;
                    break;
                }
                q.primitive();
                exchange(DS_AFTER_HALO_NR);
                break;
            case DS_AFTER_HALO_NR:
                q.n += launch_halo_unpack(v, s, c->d_imp, c->nimp, c->d_halo);
                q.bc();
                q.residual(RES_NR);
                q.sweeps();
                q.n += launch_res_export(v, s, q.partials(), c->nsf == 0 ? 0 : q.nstrips(), c->d_red);
                reduce(1, 2, DS_AFTER_RES);
                break;
            case DS_AFTER_RES:
                q.n += launch_res_import(v, s, c->d_red, c->ds_j);
                q.update(c->ds_j, c->d_red, 1);
                ++c->ds_j;
                c->ds_stage = DS_INNER;
                more = true;
                break;
            case DS_AFTER_HALO:
                q.n += launch_halo_unpack(v, s, c->d_imp, c->nimp, c->d_halo);
                q.bc();
                if (c->d.scheme == SCFD_SCHEME_EULER) {
                    q.residual(RES_EULER);
                } else {
                    q.residual(RES_LUSGS);
                    q.sweeps();
                    q.update(1, q.partials(), q.nstrips());
                }
                q.n += launch_status_export(v, s, c->d_red);
                reduce(0, 1, DS_AFTER_STATUS);
                break;
            default:  // DS_AFTER_STATUS
                q.n += launch_status_import(v, s, c->d_red);
                finished = true;
                break;
        }
    }
    CK(cudaGetLastError());
    c->launches += q.n;
    if (!finished) return 0;
    c->ds_stage = DS_BEGIN;
    req->kind = SCFD_DREQ_DONE;
    req->buf = nullptr;
    const int st = sync_scalars(c);
    if (st) return st;
    collect_events(c);
    return fill_stats(c, stats, c->ds_att0, c->ds_fb0);
}

int scfd_set_bc_values(scfd_ctx* c, int bc, const double* value) {
    if (!c || !value || bc < 0 || bc >= (int)c->bcs.size()) return SCFD_E_ARG;
    if (!c->committed) return c->fail(SCFD_E_STATE, "set_bc_values before commit");
    std::memcpy(c->bcs[bc].value, value, sizeof(double) * c->valstride);
    CK(cudaMemcpyAsync(c->d_bcval + (size_t)bc * c->valstride, value, sizeof(double) * c->valstride,
                       cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

// ---------------------------------------------------------------------------
// Discrete adjoint of the explicit ideal-gas step with binomial checkpointing.
// ---------------------------------------------------------------------------
namespace {

// binomial(s + t, t): steps reversible with s stored states and t sweeps
long long binom_steps(int s, int t) {
    long double r = 1.0L;
    for (int k = 1; k <= t; ++k) r = r * (long double)(s + k) / (long double)k;
    return r > 4e18L ? (long long)4e18 : (long long)(r + 0.5L);
}

struct AdjRun {
    scfd_ctx* c;
    const scfd_adj_desc* d;
    double dt = 0.0;
    size_t qsz = 0;            // doubles per stored state (q, all slots)
    double* slots = nullptr;   // [snapshots + 1][qsz]
    int nslots = 0;
    std::vector<int> free_slot;
    double* lam = nullptr;     // dJ/dq, D components per slot
    double* wbar = nullptr;    // adjoint of w, W components per slot
    double* dgrad = nullptr;   // [valstride]
    double* dJ = nullptr;
    long long* ocells = nullptr;
    double* owt = nullptr;
    int nobj = 0;
    long long fwd = 0, rev = 0;
    int visited = 0;           // highest step index whose state has been formed
    cudaGraphExec_t* rev_graph = nullptr;  // [2]: reverse step without / with the objective term (context-owned)

    bool in_window(int n) const { return n >= d->win_first && n <= d->win_last; }
    int save(int slot) {
        CK(cudaMemcpyAsync(slots + (size_t)slot * qsz, c->v.q, qsz * sizeof(double), cudaMemcpyDeviceToDevice,
                           c->stream));
        return 0;
    }
    int restore(int slot) {
        CK(cudaMemcpyAsync(c->v.q, slots + (size_t)slot * qsz, qsz * sizeof(double), cudaMemcpyDeviceToDevice,
                           c->stream));
        return 0;
    }
    // q^a in the context -> q^b; adds the objective of states formed for the first time
    int advance(int a, int b) {
        for (int k = a; k < b; ++k) {
            int st = step_once(c);
            if (st) return st;
            ++fwd;
            if (k + 1 > visited) {
                visited = k + 1;
                if (in_window(k + 1)) launch_adj_objective(c->v, c->stream, ocells, owt, nobj, dJ, nullptr, 0);
            }
        }
        return 0;
    }
    // the kernels of one reverse step (captured once per variant into a CUDA graph)
    void enqueue_back(bool obj) {
        const View& v = c->v;
        cudaStream_t s = c->stream;
        launch_thermo(v, s, c->cells_max);
        launch_ghost_ops(v, s, c->d_ops, c->nops, c->d_bcval, c->valstride);
        launch_adj_faces(v, s, lam, wbar, dt);
        launch_adj_ghost(v, s, c->d_ops, c->nops, c->d_bcval, c->valstride, wbar, dgrad, d->param_bc);
        launch_adj_prim(v, s, wbar, lam);
        if (obj) launch_adj_objective(v, s, ocells, owt, nobj, nullptr, lam, 1);
    }
    // q^n in the context; lam = dJ/dq^{n+1} -> dJ/dq^n
    int step_back(int n) {
        const int var = in_window(n) ? 1 : 0;
        if (!rev_graph[var]) {
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            enqueue_back(var == 1);
            const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
            if (e != cudaSuccess) return c->fail(SCFD_E_CUDA, std::string("adjoint graph capture: ") + cudaGetErrorString(e));
            const cudaError_t ei = cudaGraphInstantiate(&rev_graph[var], g, 0);
            cudaGraphDestroy(g);
            if (ei != cudaSuccess) {
                rev_graph[var] = nullptr;
                return c->fail(SCFD_E_CUDA, std::string("adjoint graph instantiate: ") + cudaGetErrorString(ei));
            }
        }
        CK(cudaGraphLaunch(rev_graph[var], c->stream));
        c->launches += 6 + var;
        ++rev;
        return 0;
    }
    // optimal first stored state of a segment (dynamic programming over the cost
    // F(l, s) = min over l1 of l1 + F(l - l1, s - 1) + F(l1, s) of this
    // recursion, in forward steps), when the table is affordable
    std::vector<std::vector<int>> best_split;
    void plan(int n, int S) {
        // with a stored state per step (or none) the split rule below is already optimal
        if (S < 1 || S >= n - 1 || (double)n * n * S > 2e9) return;
        std::vector<std::vector<long long>> F(S + 1, std::vector<long long>(n + 1, 0));
        best_split.assign(S + 1, std::vector<int>(n + 1, 1));
        for (int l = 1; l <= n; ++l) F[0][l] = (long long)l * (l - 1) / 2;
        for (int sf = 1; sf <= S; ++sf)
            for (int l = 2; l <= n; ++l) {
                long long bestc = -1;
                for (int l1 = 1; l1 < l; ++l1) {
                    const long long cst = l1 + F[sf - 1][l - l1] + F[sf][l1];
                    if (bestc < 0 || cst < bestc) {
                        bestc = cst;
                        best_split[sf][l] = l1;
                    }
                }
                F[sf][l] = bestc;
            }
    }
    int split(int a, int b, int sfree) const {
        const int n = b - a;
        if (sfree < (int)best_split.size() && n < (int)best_split[sfree].size()) return a + best_split[sfree][n];
        int t = 1;
        while (binom_steps(sfree, t) < n) ++t;
        const long long tail = binom_steps(sfree - 1, t);
        const int m = b - (int)std::min<long long>(tail, n - 1);
        return std::max(m, a + 1);
    }
    // precondition: the context holds q^a, stored in slot sa; lam = dJ/dq^b
    int revolve(int a, int b, int sa) {
        int st;
        if (b - a == 1) return step_back(a);
        if (free_slot.empty()) {
            for (int k = b - 1; k >= a; --k) {
                if ((st = restore(sa)) || (st = advance(a, k)) || (st = step_back(k))) return st;
            }
            return 0;
        }
        const int m = split(a, b, (int)free_slot.size());
        if ((st = advance(a, m))) return st;
        const int sm = free_slot.back();
        free_slot.pop_back();
        if ((st = save(sm))) return st;
        if ((st = revolve(m, b, sm))) return st;
        free_slot.push_back(sm);
        if ((st = restore(sa))) return st;
        return revolve(a, m, sa);
    }
};

}  // namespace

int scfd_adjoint_run(scfd_ctx* c, const scfd_adj_desc* d, double* J, double* grad, int64_t* counts) {
    if (!c || !d || !J) return SCFD_E_ARG;
    if (!c->committed || !c->uploaded) return c->fail(SCFD_E_STATE, "adjoint before upload");
    if (d->abi_version != SCFD_ABI_VERSION || d->nsteps < 1 || d->snapshots < 0 || d->win_first < 0 ||
        d->win_first > d->win_last || d->win_last >= d->nsteps || d->obj_bc < 0 || d->obj_bc >= (int)c->bcs.size() ||
        d->param_bc < -1 || d->param_bc >= (int)c->bcs.size() || (!d->forward_only && d->param_bc >= 0 && !grad))
        return c->fail(SCFD_E_ARG, "bad adjoint descriptor");
    const scfd_desc& cd = c->d;
    if (cd.scheme != SCFD_SCHEME_EULER || cd.thermo != SCFD_THERMO_IDEAL || cd.dim != SCFD_DIM_2D || cd.viscous ||
        cd.dt_mode != SCFD_DT_FIXED || cd.precision != SCFD_PREC_FP64 || c->nranks > 1 || c->nY != 1)
        return c->fail(SCFD_E_UNSUPPORTED, "the adjoint covers the 2d inviscid ideal-gas explicit step (FP64, fixed dt)");
    AdjRun r;
    r.c = c;
    r.d = d;
    r.dt = cd.dt_fixed;
    r.qsz = (size_t)c->D * c->ncell;
    auto& A = c->adj;
    const int S = d->forward_only ? 0 : std::min(d->snapshots, d->nsteps);
    // buffers: allocated once per context (the state slots grow when a run needs more)
    if (!A.lam) {
        int mx = 1;
        for (int p = 0; p < c->np; ++p) mx = std::max(mx, std::max(c->P.ni[p], c->P.nj[p]));
        if (cudaMalloc(&A.lam, sizeof(double) * r.qsz) != cudaSuccess ||
            cudaMalloc(&A.wbar, sizeof(double) * (size_t)c->W * c->ncell) != cudaSuccess ||
            cudaMalloc(&A.dgrad, sizeof(double) * c->valstride) != cudaSuccess ||
            cudaMalloc(&A.dJ, sizeof(double)) != cudaSuccess ||
            cudaMalloc(&A.ocells, sizeof(long long) * mx) != cudaSuccess ||
            cudaMalloc(&A.owt, sizeof(double) * mx) != cudaSuccess) {
            cudaGetLastError();
            return c->fail(SCFD_E_CUDA, "no device memory for the adjoint");
        }
    }
    if (A.nslots < S + 1) {
        if (A.slots) cudaFree(A.slots);
        A.slots = nullptr;
        A.nslots = 0;
        if (cudaMalloc(&A.slots, sizeof(double) * r.qsz * (S + 1)) != cudaSuccess) {
            cudaGetLastError();
            return c->fail(SCFD_E_CUDA, "no device memory for the adjoint's stored states");
        }
        A.nslots = S + 1;
    }
    r.slots = A.slots;
    r.nslots = S + 1;
    r.lam = A.lam;
    r.wbar = A.wbar;
    r.dgrad = A.dgrad;
    r.dJ = A.dJ;
    r.ocells = A.ocells;
    r.owt = A.owt;
    // objective cells: the first interior cells along the descriptor's range, weighted by the face length
    {
        const scfd_bc& b = c->bcs[d->obj_bc];
        const int p = b.plane - 1, ni = c->P.ni[p], nj = c->P.nj[p];
        std::vector<long long> cells;
        std::vector<double> wt;
        for (int sx = b.first; sx <= b.last; ++sx) {
            switch (b.side) {
                case SCFD_SIDE_ILO: cells.push_back(cidx(c->P, p, 1, sx)); wt.push_back(c->h_dsi[cidx(c->P, p, 0, sx)]); break;
                case SCFD_SIDE_IHI: cells.push_back(cidx(c->P, p, ni, sx)); wt.push_back(c->h_dsi[cidx(c->P, p, ni, sx)]); break;
                case SCFD_SIDE_JLO: cells.push_back(cidx(c->P, p, sx, 1)); wt.push_back(c->h_dsj[cidx(c->P, p, sx, 0)]); break;
                default: cells.push_back(cidx(c->P, p, sx, nj)); wt.push_back(c->h_dsj[cidx(c->P, p, sx, nj)]); break;
            }
        }
        r.nobj = (int)cells.size();
        CK(cudaMemcpyAsync(r.ocells, cells.data(), sizeof(long long) * cells.size(), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(r.owt, wt.data(), sizeof(double) * wt.size(), cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    // the reverse-step graphs bake the descriptor indices in: rebuild them when those change
    if (A.key_obj != d->obj_bc || A.key_param != d->param_bc) {
        for (auto& g : A.rev_graph)
            if (g) cudaGraphExecDestroy(g);
        A.rev_graph[0] = A.rev_graph[1] = nullptr;
        A.key_obj = d->obj_bc;
        A.key_param = d->param_bc;
    }
    r.rev_graph = A.rev_graph;
    int st = 0;
    for (int k = S; k >= 1; --k) r.free_slot.push_back(k);
    if (!d->forward_only) {
        if (A.plan_n != d->nsteps || A.plan_s != S) {
            r.plan(d->nsteps, S);
            A.best_split = std::move(r.best_split);
            A.plan_n = d->nsteps;
            A.plan_s = S;
        }
        r.best_split = A.best_split;
    }
    DevScalars sc0;
    if ((st = sync_scalars(c))) return st;
    sc0 = *c->h_sc;
    CK(cudaMemsetAsync(r.dJ, 0, sizeof(double), c->stream));
    CK(cudaMemsetAsync(r.dgrad, 0, sizeof(double) * c->valstride, c->stream));
    if (!d->forward_only) {
        CK(cudaMemsetAsync(r.lam, 0, sizeof(double) * r.qsz, c->stream));
        CK(cudaMemsetAsync(r.wbar, 0, sizeof(double) * (size_t)c->W * c->ncell, c->stream));
    }
    c->launches = 0;
    if ((st = r.save(0))) return st;
    if (r.in_window(0)) launch_adj_objective(c->v, c->stream, r.ocells, r.owt, r.nobj, r.dJ, nullptr, 0);
    if (d->forward_only)
        st = r.advance(0, d->win_last);
    else
        st = r.revolve(0, d->nsteps, 0);
    if (st) return st;
    // the uploaded state back: q, qp, qpp and the scalars
    if ((st = r.restore(0))) return st;
    const size_t qb = sizeof(double) * r.qsz;
    CK(cudaMemcpyAsync(c->v.qp, c->v.q, qb, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->v.qpp, c->v.q, qb, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_sc, &sc0, sizeof(DevScalars), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(J, r.dJ, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (grad) CK(cudaMemcpyAsync(grad, r.dgrad, sizeof(double) * c->valstride, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (counts) {
        counts[0] = r.fwd;
        counts[1] = r.rev;
    }
    return 0;
}

int scfd_tuning(scfd_ctx* c, char* json, int len) {
    if (!c || !json || len <= 0) return SCFD_E_ARG;
    // the autotuner's report plus the sweep implementation the context runs
    std::string rep = c->tune_report;
    char sw[160];
    if (c->use_sw3)
        std::snprintf(sw, sizeof(sw), "\"sweep\": {\"kind\": \"cluster wavefront\", \"tasks\": %d, \"clusters\": %d}",
                      c->sw3.ntasks, c->sw3.nclusters);
    else
        std::snprintf(sw, sizeof(sw), "\"sweep\": {\"kind\": \"%s\"}",
                      c->d.scheme == SCFD_SCHEME_EULER ? "none" : "generic");
    const size_t close = rep.rfind('}');
    if (close != std::string::npos) rep = rep.substr(0, close) + (rep.size() > 2 ? ", " : "") + sw + "}";
    std::snprintf(json, (size_t)len, "%s", rep.c_str());
    return (int)rep.size() < len ? 0 : SCFD_E_ARG;
}

int scfd_rms(scfd_ctx* c, double* rms) {
    if (!c || !rms || !c->committed) return SCFD_E_ARG;
    launch_rms(c->v, c->stream, c->d_rms_partial, c->d_rms_out);
    CK(cudaMemcpyAsync(rms, c->d_rms_out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return (*rms != *rms) ? SCFD_E_NAN : 0;
}

int scfd_inner_log(scfd_ctx* c, double* omega, double* res, int n) {
    if (!c || !c->committed || n < 0) return -SCFD_E_ARG;
    if (!dual_time_scheme(c->d.scheme)) return 0;
    if (int st = sync_scalars(c)) return -st;
    int m = std::min(std::min(n, std::max(0, c->d.num_internal_loop - 1)), SCFD_INNER_LOG);
    for (int k = 0; k < m; ++k) {
        if (omega) omega[k] = c->h_sc->il_omega[k];
        if (res) res[k] = c->h_sc->il_res[k];
    }
    return m;
}

int scfd_download(scfd_ctx* c, double* q, double* w, double* vhi, double* tt) {
    if (!c || !c->committed) return SCFD_E_ARG;
    int st;
    if (q && (st = download_field(c, c->v.q, c->D, q))) return st;
    if (w && (st = download_field(c, c->v.w, c->W, w))) return st;
    if (vhi && (st = download_field(c, c->v.vhi, c->nY, vhi))) return st;
    if (tt) {
        if ((st = sync_scalars(c))) return st;
        *tt = c->h_sc->tt;
    }
    return 0;
}

// ---- restart.bin (store/core/inout.f90) -----------------------------------
// Fortran sequential unformatted, big-endian (the reference compiles with
// -fconvert=big-endian): every record is [int32 n][n bytes][int32 n].
static void put_be(std::string& out, const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t k = 0; k < n; ++k) out.push_back((char)b[n - 1 - k]);
}
static void get_be(const char* in, void* p, size_t n) {
    unsigned char* b = static_cast<unsigned char*>(p);
    for (size_t k = 0; k < n; ++k) b[n - 1 - k] = (unsigned char)in[k];
}
static void put_record(std::string& out, const std::string& payload) {
    const int32_t n = (int32_t)payload.size();
    put_be(out, &n, 4);
    out += payload;
    put_be(out, &n, 4);
}

int scfd_write_restart(scfd_ctx* c, const char* path, int step) {
    if (!c || !path) return SCFD_E_ARG;
    if (!c->committed) return c->fail(SCFD_E_STATE, "write_restart before commit");
    const int D = c->D, W = c->W, nY = c->nY, IX = c->nimax + 4, JX = c->njmax + 4;
    const size_t cells = (size_t)IX * JX * c->np;
    std::vector<double> q(cells * D), w(cells * W);
    double tt = 0.0;
    int st = scfd_download(c, q.data(), w.data(), nullptr, &tt);
    if (st) return st;
    auto at = [&](int p, int i, int j) { return (size_t)(i + 1) + (size_t)IX * ((size_t)(j + 1) + (size_t)JX * p); };
    const int ig = D + 1, iht = D + 2, iR = D + 3;  // 0-based indxg, indxht, indxR
    // set_bc_q: the first ghost layer of q from w (inout.f90:151-198)
    auto bc_q = [&](int p, int i, int j) {
        const size_t c0 = at(p, i, j);
        const double* wc = &w[c0 * W];
        double* qc = &q[c0 * D];
        const double tmp = wc[0];
        for (int k = 0; k < nY; ++k) qc[k] = tmp * wc[k + 4];
        qc[nY] = tmp * wc[1];
        qc[nY + 1] = tmp * wc[2];
        qc[nY + 2] = tmp * wc[iht] - wc[3];
    };
    for (int p = 0; p < c->np; ++p) {
        const int ni = c->P.ni[p], nj = c->P.nj[p];
        for (int j = 1; j <= nj; ++j) {
            bc_q(p, 0, j);
            bc_q(p, ni + 1, j);
        }
        for (int i = 0; i <= ni + 1; ++i) {
            bc_q(p, i, 0);
            bc_q(p, i, nj + 1);
        }
    }
    std::string field;
    for (int p = 0; p < c->np; ++p)
        for (int j = 0; j <= c->P.nj[p] + 1; ++j)
            for (int i = 0; i <= c->P.ni[p] + 1; ++i) {
                const size_t c0 = at(p, i, j);
                for (int k = 0; k < D; ++k) put_be(field, &q[c0 * D + k], 8);
                put_be(field, &w[c0 * W + iR], 8);
                put_be(field, &w[c0 * W + ig], 8);
                put_be(field, &w[c0 * W + 3], 8);
            }
    std::string out, rec;
    const int32_t s32 = step;
    put_be(rec, &s32, 4);
    put_record(out, rec);
    rec.clear();
    put_be(rec, &tt, 8);
    put_record(out, rec);
    put_record(out, field);
    FILE* f = std::fopen(path, "wb");
    if (!f) return c->fail(SCFD_E_IO, std::string("cannot open ") + path);
    const size_t wr = std::fwrite(out.data(), 1, out.size(), f);
    const int cl = std::fclose(f);
    if (wr != out.size() || cl != 0) return c->fail(SCFD_E_IO, std::string("cannot write ") + path);
    return 0;
}

int scfd_write_geometry(scfd_ctx* c, const char* path) {
    if (!c || !path) return SCFD_E_ARG;
    for (int p = 0; p < c->np; ++p)
        if (!c->geo_set[p]) return c->fail(SCFD_E_STATE, "geometry of plane " + std::to_string(p + 1) + " not set");
    std::string out, rec;
    for (int p = 0; p < c->np; ++p) {
        const int32_t ni = c->P.ni[p], nj = c->P.nj[p];
        for (const int32_t n : {ni, nj}) {
            rec.clear();
            put_be(rec, &n, 4);
            put_record(out, rec);
        }
        rec.clear();
        for (int j = 0; j <= nj; ++j)
            for (int i = 0; i <= ni; ++i) {
                const size_t k = (size_t)i + (size_t)(ni + 1) * j;
                put_be(rec, &c->xh[p][k], 8);
                put_be(rec, &c->rh[p][k], 8);
            }
        put_record(out, rec);
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) return c->fail(SCFD_E_IO, std::string("cannot open ") + path);
    const size_t wr = std::fwrite(out.data(), 1, out.size(), f);
    const int cl = std::fclose(f);
    if (wr != out.size() || cl != 0) return c->fail(SCFD_E_IO, std::string("cannot write ") + path);
    return 0;
}

int scfd_read_restart(scfd_ctx* c, const char* path, int* step, double* tt) {
    if (!c || !path || !step) return SCFD_E_ARG;
    if (!c->committed) return c->fail(SCFD_E_STATE, "read_restart before commit");
    FILE* f = std::fopen(path, "rb");
    if (!f) return c->fail(SCFD_E_IO, std::string("cannot open ") + path);
    std::string buf;
    char tmp[1 << 16];
    size_t n;
    while ((n = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.append(tmp, n);
    std::fclose(f);
    std::vector<std::pair<size_t, size_t>> recs;  // offset, length
    for (size_t pos = 0; pos < buf.size();) {
        int32_t a = 0, b = 0;
        if (pos + 4 > buf.size()) return c->fail(SCFD_E_IO, "truncated record marker");
        get_be(&buf[pos], &a, 4);
        if (a < 0 || pos + 8 + (size_t)a > buf.size()) return c->fail(SCFD_E_IO, "truncated record");
        get_be(&buf[pos + 4 + a], &b, 4);
        if (a != b) return c->fail(SCFD_E_IO, "record markers disagree");
        recs.push_back({pos + 4, (size_t)a});
        pos += 8 + (size_t)a;
    }
    const int D = c->D, W = c->W, IX = c->nimax + 4, JX = c->njmax + 4;
    size_t need = 0;
    for (int p = 0; p < c->np; ++p) need += (size_t)(c->P.ni[p] + 2) * (c->P.nj[p] + 2) * (D + 3) * 8;
    if (recs.size() != 3 || recs[0].second != 4 || recs[1].second != 8 || recs[2].second != need)
        return c->fail(SCFD_E_IO, "restart file does not match the case");
    int32_t s32 = 0;
    double t = 0.0;
    get_be(&buf[recs[0].first], &s32, 4);
    get_be(&buf[recs[1].first], &t, 8);
    const size_t cells = (size_t)IX * JX * c->np;
    std::vector<double> q(cells * D), w(cells * W);
    int st = scfd_download(c, q.data(), w.data(), nullptr, nullptr);
    if (st) return st;
    const char* fp = &buf[recs[2].first];
    const int ig = D + 1, iR = D + 3;
    for (int p = 0; p < c->np; ++p)
        for (int j = 0; j <= c->P.nj[p] + 1; ++j)
            for (int i = 0; i <= c->P.ni[p] + 1; ++i) {
                const size_t c0 = (size_t)(i + 1) + (size_t)IX * ((size_t)(j + 1) + (size_t)JX * p);
                for (int k = 0; k < D; ++k, fp += 8) get_be(fp, &q[c0 * D + k], 8);
                get_be(fp, &w[c0 * W + iR], 8);
                get_be(fp + 8, &w[c0 * W + ig], 8);
                get_be(fp + 16, &w[c0 * W + 3], 8);
                fp += 24;
            }
    if ((st = scfd_upload(c, q.data(), w.data(), nullptr, t))) return st;
    *step = s32;
    if (tt) *tt = t;
    return 0;
}

int scfd_download_qp(scfd_ctx* c, double* qp) {
    if (!c || !c->committed || !qp) return SCFD_E_ARG;
    return download_field(c, c->v.qp, c->D, qp);
}

int scfd_get_stream(scfd_ctx* c, void** s) {
    if (!c || !s) return SCFD_E_ARG;
    *s = (void*)c->stream;
    return 0;
}

int scfd_launch_count(const scfd_ctx* c, int64_t* n) {
    if (!c || !n) return SCFD_E_ARG;
    *n = c->launches;
    return 0;
}

int scfd_profile(scfd_ctx* c, int enable) {
    if (!c) return SCFD_E_ARG;
    c->profiling = enable != 0;
    for (int k = 0; k < SCFD_K_COUNT; ++k) {
        c->kind_ms[k] = 0.0;
        c->kind_n[k] = 0;
    }
    c->ev_marks.clear();
    c->ev_used = 0;
    return 0;
}

int scfd_kernel_stats(scfd_ctx* c, int kind, double* total_ms, int64_t* launches, char* name, int namelen) {
    static const char* names[SCFD_K_COUNT] = {"thermo", "bc", "set_dt", "chemistry", "residual", "sweep_fwd",
                                              "sweep_bwd", "update", "copy", "other", "pack"};
    if (!c || kind < 0 || kind >= SCFD_K_COUNT) return SCFD_E_ARG;
    if (total_ms) *total_ms = c->kind_ms[kind];
    if (launches) *launches = c->kind_n[kind];
    if (name && namelen > 0) std::snprintf(name, (size_t)namelen, "%s", names[kind]);
    return 0;
}

}  // extern "C"
