// Host build of the exact per-node collision (particuology_hydraulic_penalty_b200/csrc/collide.cuh)
// so its operation order can be checked against the NumPy oracle on a CPU.
// Built by tests/test_collide_host.py with g++ -O2 -ffp-contract=off.
#include <cstddef>

#include "collide.cuh"

extern "C" void exact_collide_cells(const double* f_in, const double* solid, const double* us, int moving, double tau,
                                    double fx, double fy, double fz, int ncell, double* f_out, double* imb_out,
                                    double* mom_out) {
    using namespace psc;
    const double hfx = xmul(0.5, fx), hfy = xmul(0.5, fy), hfz = xmul(0.5, fz);
    for (int c = 0; c < ncell; ++c) {
        double f[Q];
        for (int i = 0; i < Q; ++i) f[i] = f_in[(size_t)i * ncell + c];
        const ExactMoments mo = moments_exact(f, hfx, hfy, hfz);
        double imb[3];
        const double usx = moving ? us[c] : 0.0, usy = moving ? us[ncell + c] : 0.0, usz = moving ? us[2 * ncell + c] : 0.0;
        collide_exact(f, mo, solid[c], moving != 0, usx, usy, usz, tau, fx, fy, fz, hfx, hfy, hfz, imb);
        for (int i = 0; i < Q; ++i) f_out[(size_t)i * ncell + c] = f[i];
        for (int k = 0; k < 3; ++k) imb_out[(size_t)k * ncell + c] = imb[k];
        mom_out[c] = mo.rho;
        mom_out[ncell + c] = mo.ux;
        mom_out[2 * ncell + c] = mo.uy;
        mom_out[3 * ncell + c] = mo.uz;
    }
}

extern "C" void fast_collide_cells(const double* g_in, const double* solid, const double* us, int moving, double tau,
                                   double fx, double fy, double fz, int ncell, double* g_out, double* imb_out) {
    using namespace psc;
    FastParams<double> p;
    p.inv_tau = 1.0 / tau;
    p.pref = 1.0 - 0.5 / tau;
    p.fx = fx;
    p.fy = fy;
    p.fz = fz;
    for (int c = 0; c < ncell; ++c) {
        double g[Q];
        for (int i = 0; i < Q; ++i) g[i] = g_in[(size_t)i * ncell + c];
        const FastMoments<double> mo = moments_fast(g);
        const double al = solid[c];
        const double B = al / (al + tau * (1.0 - al) + 1.0e-14);
        double imb[3];
        if (moving)
            collide_fast<double, true, true>(g, mo, 1.0 / mo.rho, B, us[c], us[ncell + c], us[2 * ncell + c], p, imb);
        else
            collide_fast<double, false, true>(g, mo, 1.0 / mo.rho, B, 0.0, 0.0, 0.0, p, imb);
        for (int i = 0; i < Q; ++i) g_out[(size_t)i * ncell + c] = g[i];
        for (int k = 0; k < 3; ++k) imb_out[(size_t)k * ncell + c] = imb[k];
    }
}

// The per-window-constant form run by the throughput kernels (collide_fast2):
// BGK when tau_minus is 0, else TRT.
extern "C" void fast2_collide_cells(const double* g_in, const double* solid, const double* us, int moving, double tau,
                                    double tau_minus, double fx, double fy, double fz, int ncell, double* g_out,
                                    double* imb_out) {
    using namespace psc;
    WinConst<double> wc;
    make_win_const(wc, tau, fx, fy, fz, tau_minus);
    for (int c = 0; c < ncell; ++c) {
        double g[Q];
        for (int i = 0; i < Q; ++i) g[i] = g_in[(size_t)i * ncell + c];
        const double al = solid[c];
        const double B = al / (al + tau * (1.0 - al) + 1.0e-14);
        const double kb = (1.0 - B) / tau;
        double imb[3], mom[4];
        const double usx = moving ? us[c] : 0.0, usy = moving ? us[ncell + c] : 0.0, usz = moving ? us[2 * ncell + c] : 0.0;
        if (tau_minus > 0.0) {
            if (moving) collide_fast2<double, true, true, true>(g, wc, B, kb, usx, usy, usz, 0.0, mom, imb);
            else collide_fast2<double, false, true, true>(g, wc, B, kb, usx, usy, usz, 0.0, mom, imb);
        } else {
            if (moving) collide_fast2<double, true, true>(g, wc, B, kb, usx, usy, usz, 0.0, mom, imb);
            else collide_fast2<double, false, true>(g, wc, B, kb, usx, usy, usz, 0.0, mom, imb);
        }
        for (int i = 0; i < Q; ++i) g_out[(size_t)i * ncell + c] = g[i];
        for (int k = 0; k < 3; ++k) imb_out[(size_t)k * ncell + c] = imb[k];
    }
}
