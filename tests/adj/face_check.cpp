// Test driver (CPU): the reverse of the MUSCL face states, of the SLAU flux and
// of the ideal-gas primitive map in adj_face.cuh against central differences
// of the forward functions on seeded random states.  Prints the largest
// relative mismatch of each check.
#include <cstdio>
#include <cmath>
#include <random>
#include <vector>

#include "adj_face.cuh"

using namespace scfd::adj;

// largest |a - b| over the largest |b| of a gradient vector
static double vrel(const std::vector<double>& a, const std::vector<double>& b) {
    double e = 0.0, m = 1e-300;
    for (size_t k = 0; k < a.size(); ++k) {
        e = std::fmax(e, std::fabs(a[k] - b[k]));
        m = std::fmax(m, std::fabs(b[k]));
    }
    return e / m;
}

int main() {
    std::mt19937_64 rng(20240713);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    const int nY = 1, nc = 6 + nY;
    double worst_muscl = 0.0, worst_slau = 0.0, worst_prim = 0.0, worst_p = 0.0;
    for (int trial = 0; trial < 400; ++trial) {
        // MUSCL
        const double phi = 1.0, km = 1.0 / 3.0;
        double w[4];
        for (double& x : w) x = 1.0 + 0.3 * U(rng);
        const double wlb = U(rng), wrb = U(rng);
        double b[4] = {0, 0, 0, 0};
        muscl_rev(w[0], w[1], w[2], w[3], phi, km, wlb, wrb, b[0], b[1], b[2], b[3]);
        std::vector<double> ad4(b, b + 4), fd4(4);
        for (int k = 0; k < 4; ++k) {
            const double h = 1e-6;
            double wp[4], wm[4];
            for (int m = 0; m < 4; ++m) wp[m] = wm[m] = w[m];
            wp[k] += h;
            wm[k] -= h;
            double lp, rp, lm, rm;
            muscl_fwd(wp[0], wp[1], wp[2], wp[3], phi, km, lp, rp);
            muscl_fwd(wm[0], wm[1], wm[2], wm[3], phi, km, lm, rm);
            fd4[k] = (wlb * (lp - lm) + wrb * (rp - rm)) / (2 * h);
        }
        worst_muscl = std::fmax(worst_muscl, vrel(ad4, fd4));
        // SLAU: states with Mach numbers around 0-2 in both directions
        std::vector<double> wl(nc), wr(nc), tgb(nY + 3), wlb2(nc, 0.0), wrb2(nc, 0.0);
        auto state = [&](std::vector<double>& s) {
            s[0] = 1.0 + 0.5 * U(rng);
            s[1] = 300.0 * U(rng);
            s[2] = 150.0 * U(rng);
            s[3] = 1e5 * (1.0 + 0.5 * U(rng));
            s[4] = 1.0;
            s[4 + nY] = 1.4;
            s[5 + nY] = 3.5 * s[3] / s[0] + 0.5 * (s[1] * s[1] + s[2] * s[2]);
        };
        state(wl);
        state(wr);
        const double th = 3.14159265 * U(rng);
        const double n1 = std::cos(th), n2 = std::sin(th);
        for (double& x : tgb) x = U(rng);
        slau_rev(nY, wl.data(), wr.data(), n1, n2, tgb.data(), wlb2.data(), wrb2.data());
        for (int side = 0; side < 2; ++side) {
            // each input scaled by its magnitude, so that the vector is comparable
            std::vector<double> ads(nc), fds(nc);
            for (int k = 0; k < nc; ++k) {
                std::vector<double>& s = side ? wr : wl;
                const double mag = std::fabs(s[k]) + 1.0;
                const double h = 1e-5 * mag;
                const double keep = s[k];
                std::vector<double> tp(nY + 3), tm(nY + 3);
                s[k] = keep + h;
                slau_fwd(nY, wl.data(), wr.data(), n1, n2, tp.data());
                s[k] = keep - h;
                slau_fwd(nY, wl.data(), wr.data(), n1, n2, tm.data());
                s[k] = keep;
                double fd = 0.0;
                for (int m = 0; m < nY + 3; ++m) fd += tgb[m] * (tp[m] - tm[m]) / (2 * h);
                fds[k] = fd * mag;
                ads[k] = (side ? wrb2[k] : wlb2[k]) * mag;
            }
            worst_slau = std::fmax(worst_slau, vrel(ads, fds));
        }
        // ideal primitive map and the objective pressure
        std::vector<double> q(nY + 3), qb(nY + 3, 0.0), qb2(nY + 3, 0.0);
        q[0] = 1.0 + 0.5 * U(rng);
        q[1] = q[0] * 200 * U(rng);
        q[2] = q[0] * 100 * U(rng);
        q[3] = 2.5e5 * (1.0 + 0.3 * U(rng)) + 0.5 * (q[1] * q[1] + q[2] * q[2]) / q[0];
        const double kappa = 1.4;
        double rb = U(rng), ub = U(rng), vb = U(rng), pb = U(rng), hb = U(rng), Yb = U(rng);
        ideal_prim_rev(nY, q.data(), kappa, rb, ub, vb, pb, &Yb, hb, qb.data());
        const double pbo = U(rng);
        ideal_p_rev(nY, q.data(), kappa, pbo, qb2.data());
        auto prim = [&](const std::vector<double>& x) {
            const double rho = x[0], u = x[1] / rho, v = x[2] / rho, Y = x[0] / rho;
            const double ei = x[3] / rho - 0.5 * (u * u + v * v);
            const double p = rho * (kappa - 1.0) * ei;
            const double ht = (x[3] + p) / rho;
            return rb * rho + ub * u + vb * v + pb * p + Yb * Y + hb * ht;
        };
        std::vector<double> fdq(nY + 3), fdp(nY + 3), adq(nY + 3), adp(nY + 3);
        for (int k = 0; k < nY + 3; ++k) {
            const double h = 1e-4 * std::fabs(q[k]) + 1e-9;
            std::vector<double> a = q, c = q;
            a[k] += h;
            c[k] -= h;
            fdq[k] = (prim(a) - prim(c)) / (2 * h) * std::fabs(q[k]);
            fdp[k] = pbo * (ideal_p(nY, a.data(), kappa) - ideal_p(nY, c.data(), kappa)) / (2 * h) * std::fabs(q[k]);
            adq[k] = qb[k] * std::fabs(q[k]);
            adp[k] = qb2[k] * std::fabs(q[k]);
        }
        worst_prim = std::fmax(worst_prim, vrel(adq, fdq));
        worst_p = std::fmax(worst_p, vrel(adp, fdp));
    }
    std::printf("muscl %.3e\nslau %.3e\nprim %.3e\npressure %.3e\n", worst_muscl, worst_slau, worst_prim, worst_p);
    return 0;
}
