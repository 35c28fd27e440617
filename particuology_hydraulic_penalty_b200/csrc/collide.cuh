// Per-node PSC-IMB collision: moments, Noble-Torczynski solid weighting, Guo
// forcing and the node IMB momentum.  Host+device so that the exact variant
// can be unit-tested on a CPU against the NumPy oracle.
//
// Two formulations of the same step (src/lbm_dem/psc3d.py:211-236):
//  * exact   -- absolute FP64 populations, every rounding in the reference's
//               order (NumPy evaluates one IEEE operation per ufunc call),
//               no FMA: bit-identical to the reference.
//  * fast<R> -- populations stored as deviations g_i = f_i - w_i (rho0 = 1),
//               arithmetic in R (double or float) with FMAs and reciprocal
//               multiplies.  The rest-weight offsets cancel in every
//               difference the step takes, so small deviations keep full
//               relative precision.
//
// Reference quirks reproduced by both (they are the method as published):
//  * moment velocity u = (m + F/2) / rho, and the collision uses a second
//    shift u_eff = u + F/(2 rho) = (m + F) / rho          (psc3d.py:214, 219)
//  * Guo forcing added at every node, not weighted by 1 - B  (psc3d.py:230-232)
//  * B = alpha / (alpha + tau (1 - alpha) + 1e-14)          (psc3d.py:229)
#pragma once

#include "d3q19.cuh"

namespace psc {

// ===========================================================================
// exact FP64
// ===========================================================================
struct ExactMoments {
    double rho, ux, uy, uz;
    Divisor by_rho;  // rho with its reciprocal
};

// x / c_s^2 and x / c_s^4, correctly rounded (Markstein's correction, d3q19.cuh)
PSC_HD double div_cs2(double x) { return xdiv_r(x, CS2, RCS2); }
PSC_HD double div_cs2sq(double x) { return xdiv_r(x, CS2SQ, RCS2SQ); }

// rho and u = (m + F/2)/rho of absolute populations f, psc3d.py:211-214.
PSC_HD ExactMoments moments_exact(const double* f, double hfx, double hfy, double hfz) {
    ExactMoments m;
    double rho = f[0];
#pragma unroll
    for (int i = 1; i < Q; ++i) rho = xadd(rho, f[i]);
    m.rho = rho;
    m.by_rho = make_divisor(rho);
    m.ux = xdiv_d(xadd(seq_moment_exact<0>(f), hfx), m.by_rho);
    m.uy = xdiv_d(xadd(seq_moment_exact<1>(f), hfy), m.by_rho);
    m.uz = xdiv_d(xadd(seq_moment_exact<2>(f), hfz), m.by_rho);
    return m;
}

PSC_HD double cm(int c, double x) { return c == 0 ? 0.0 : (c > 0 ? x : -x); }

// Velocity inlet by moving-wall bounce-back (Ladd 1994): the population i
// entering x = 0 from outside is the node's post-collision population opp(i)
// plus 2 w_i rho_in (c_i . u_in) / cs^2, which injects rho_in u_in per unit
// face area.  This is that term, in the operation order of the oracle.
PSC_HD double inlet_correction_exact(int i, double r, double x, double y, double z) {
    const double cu = xadd(xadd(cm(cxv(i), x), cm(cyv(i), y)), cm(czv(i), z));
    return div_cs2(xmul(xmul(2.0, xmul(wgt(i), r)), cu));
}

// The directions entering x = 0 from outside (c_x = +1).
PSC_HD constexpr bool enters_x0(int i) { return i == 1 || i == 7 || i == 9 || i == 11 || i == 13; }

// Collide f in place.  solid: clipped solid fraction.  moving: use (usx, usy,
// usz), else the solid velocity is zero.  imb receives sum_i c_i B Omega_s,i in
// the reference's sequential order (psc3d.py:234-236).
PSC_HD void collide_exact(double* f, const ExactMoments& mo, double solid, bool moving, double usx, double usy,
                          double usz, double tau, double fx, double fy, double fz, double hfx, double hfy,
                          double hfz, double* imb) {
    const double rho = mo.rho;
    const Divisor by_tau = make_divisor(tau);
    // u_eff = u + 0.5 F / rho   (psc3d.py:217-219)
    const double uex = xadd(mo.ux, xdiv_d(hfx, mo.by_rho));
    const double uey = xadd(mo.uy, xdiv_d(hfy, mo.by_rho));
    const double uez = xadd(mo.uz, xdiv_d(hfz, mo.by_rho));
    // equilibrium pieces shared by all directions (psc3d.py:98, :102)
    const double uu = xadd(xadd(xmul(uex, uex), xmul(uey, uey)), xmul(uez, uez));
    const double ct = div_cs2(xmul(0.5, uu));
    double uus = 0.0, cts = 0.0;
    if (moving) {
        uus = xadd(xadd(xmul(usx, usx), xmul(usy, usy)), xmul(usz, usz));
        cts = div_cs2(xmul(0.5, uus));
    }
    // B (psc3d.py:228-229)
    const double al = solid < 0.0 ? 0.0 : (solid > 1.0 ? 1.0 : solid);
    const double B = xdiv(al, xadd(xadd(al, xmul(tau, xsub(1.0, al))), 1.0e-14));
    const double omB = xsub(1.0, B);
    // Guo prefactor and u.F (psc3d.py:108-109)
    const double pref = xsub(1.0, xdiv_d(0.5, by_tau));
    const double uf = xadd(xadd(xmul(uex, fx), xmul(uey, fy)), xmul(uez, fz));

    double ix = 0.0, iy = 0.0, iz = 0.0;  // imb accumulators, index order from +0

    // rest population: cu = 0, cf = 0
    {
        const double wr = xmul(W0, rho);
        const double feqf = xmul(wr, xsub(1.0, ct));
        const double feqs = moving ? xmul(wr, xsub(1.0, cts)) : wr;
        const double f0 = f[0];
        const double os = xsub(feqs, feqf);  // (f0 - f0) + feqs - feqf
        const double obgk = -xdiv_d(xsub(f0, feqf), by_tau);
        const double coll = xadd(xmul(omB, obgk), xmul(B, os));
        const double g = xmul(xmul(pref, W0), div_cs2(-uf));
        f[0] = xadd(f0, xadd(coll, g));
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const int i = 2 * k + 1, j = i + 1;  // c_j = -c_i
        const double w = wgt(i);
        const double wr = xmul(w, rho);
        // feq with u_eff: cu_j = -cu_i exactly, so q_j = -q_i and b_j = b_i
        const double cu = xadd(xadd(cm(cxv(i), uex), cm(cyv(i), uey)), cm(czv(i), uez));
        const double q = div_cs2(cu);
        const double b = div_cs2sq(xmul(xmul(0.5, cu), cu));
        const double feqf_i = xmul(wr, xsub(xadd(xadd(1.0, q), b), ct));
        const double feqf_j = xmul(wr, xsub(xadd(xadd(1.0, -q), b), ct));
        double feqs_i = wr, feqs_j = wr;  // u_s = 0: feq = w rho exactly
        if (moving) {
            const double cus = xadd(xadd(cm(cxv(i), usx), cm(cyv(i), usy)), cm(czv(i), usz));
            const double qs = div_cs2(cus);
            const double bs = div_cs2sq(xmul(xmul(0.5, cus), cus));
            feqs_i = xmul(wr, xsub(xadd(xadd(1.0, qs), bs), cts));
            feqs_j = xmul(wr, xsub(xadd(xadd(1.0, -qs), bs), cts));
        }
        const double fi = f[i], fj = f[j];
        // Omega_s = f_opp - f + feq_s - feq_f[opp]   (psc3d.py:223-226)
        const double os_i = xsub(xadd(xsub(fj, fi), feqs_i), feqf_j);
        const double os_j = xsub(xadd(xsub(fi, fj), feqs_j), feqf_i);
        // Omega_bgk = -(f - feq_f) / tau   (psc3d.py:221)
        const double ob_i = -xdiv_d(xsub(fi, feqf_i), by_tau);
        const double ob_j = -xdiv_d(xsub(fj, feqf_j), by_tau);
        const double coll_i = xadd(xmul(omB, ob_i), xmul(B, os_i));
        const double coll_j = xadd(xmul(omB, ob_j), xmul(B, os_j));
        // Guo: pref W ((cf - uf)/cs2 + cu cf / cs2^2), cf_j = -cf_i   (psc3d.py:110-113)
        const double cf = xadd(xadd(cm(cxv(i), fx), cm(cyv(i), fy)), cm(czv(i), fz));
        const double pw = xmul(pref, w);
        const double t2 = div_cs2sq(xmul(cu, cf));
        const double g_i = xmul(pw, xadd(div_cs2(xsub(cf, uf)), t2));
        const double g_j = xmul(pw, xadd(div_cs2(xsub(-cf, uf)), t2));
        f[i] = xadd(fi, xadd(coll_i, g_i));
        f[j] = xadd(fj, xadd(coll_j, g_j));
        // node IMB momentum, sequential in index order (i then j)
        const double bo_i = xmul(B, os_i), bo_j = xmul(B, os_j);
        ix = cxv(i) > 0 ? xadd(ix, bo_i) : (cxv(i) < 0 ? xsub(ix, bo_i) : ix);
        ix = cxv(j) > 0 ? xadd(ix, bo_j) : (cxv(j) < 0 ? xsub(ix, bo_j) : ix);
        iy = cyv(i) > 0 ? xadd(iy, bo_i) : (cyv(i) < 0 ? xsub(iy, bo_i) : iy);
        iy = cyv(j) > 0 ? xadd(iy, bo_j) : (cyv(j) < 0 ? xsub(iy, bo_j) : iy);
        iz = czv(i) > 0 ? xadd(iz, bo_i) : (czv(i) < 0 ? xsub(iz, bo_i) : iz);
        iz = czv(j) > 0 ? xadd(iz, bo_j) : (czv(j) < 0 ? xsub(iz, bo_j) : iz);
    }
    imb[0] = ix;
    imb[1] = iy;
    imb[2] = iz;
}

// ===========================================================================
// fast deviation form, arithmetic type R
// ===========================================================================
template <typename R>
struct FastMoments {
    R drho, rho, mx, my, mz;
};

template <typename R>
PSC_HD FastMoments<R> moments_fast(const R* g) {
    FastMoments<R> m;
    m.drho = (((g[0] + g[1]) + (g[2] + g[3])) + ((g[4] + g[5]) + (g[6] + g[7]))) +
             (((g[8] + g[9]) + (g[10] + g[11])) + ((g[12] + g[13]) + (g[14] + g[15]))) + ((g[16] + g[17]) + g[18]);
    m.rho = R(1) + m.drho;
    m.mx = ((g[1] - g[2]) + (g[7] - g[8])) + ((g[9] - g[10]) + (g[11] - g[12])) + (g[13] - g[14]);
    m.my = ((g[3] - g[4]) + (g[7] - g[8])) + ((g[10] - g[9]) + (g[15] - g[16])) + (g[17] - g[18]);
    m.mz = ((g[5] - g[6]) + (g[11] - g[12])) + ((g[14] - g[13]) + (g[15] - g[16])) + (g[18] - g[17]);
    return m;
}

template <typename R>
struct FastParams {
    R inv_tau, pref, fx, fy, fz;
};

// c * x for a lattice component c in {-1, 0, 1} (folded once loops unroll).
template <typename R>
PSC_HD R csel(int c, R x) {
    return c == 0 ? R(0) : (c > 0 ? x : -x);
}

// Collide deviations g in place; irho = 1 / rho; B solid weight.  imb gets
// sum_i c_i B Omega_s,i.  Returns nothing else: the caller owns the moments.
template <typename R, bool MOVING, bool IMB>
PSC_HD void collide_fast(R* g, const FastMoments<R>& mo, R irho, R B, R usx, R usy, R usz,
                         const FastParams<R>& p, R* imb) {
    const R rho = mo.rho, drho = mo.drho;
    const R uex = (mo.mx + p.fx) * irho;
    const R uey = (mo.my + p.fy) * irho;
    const R uez = (mo.mz + p.fz) * irho;
    const R uu = uex * uex + uey * uey + uez * uez;
    const R uf = uex * p.fx + uey * p.fy + uez * p.fz;
    const R omB = R(1) - B;
    const R kb = omB * p.inv_tau;  // (1 - B) / tau
    R uus = R(0);
    if (MOVING) uus = usx * usx + usy * usy + usz * usz;
    const R r15 = R(1.5) * rho;
    R ax = R(0), ay = R(0), az = R(0);
    {
        const R geq = R(W0) * (drho - r15 * uu);
        const R os = R(W0) * r15 * (uu - uus);
        const R G = R(-3) * p.pref * R(W0) * uf;
        g[0] = g[0] - kb * (g[0] - geq) + B * os + G;
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const int i = 2 * k + 1, j = i + 1;
        const R w = R(wgt(i));
        const R cu = csel(cxv(i), uex) + csel(cyv(i), uey) + csel(czv(i), uez);
        const R cF = csel(cxv(i), p.fx) + csel(cyv(i), p.fy) + csel(czv(i), p.fz);
        const R sym = w * (drho + rho * (R(4.5) * cu * cu - R(1.5) * uu));
        const R asym = R(3) * w * rho * cu;
        R ssym, sasym;
        if (MOVING) {
            const R cus = csel(cxv(i), usx) + csel(cyv(i), usy) + csel(czv(i), usz);
            ssym = w * (drho + rho * (R(4.5) * cus * cus - R(1.5) * uus));
            sasym = R(3) * w * rho * cus;
        } else {
            ssym = w * drho;
            sasym = R(0);
        }
        const R gi = g[i], gj = g[j];
        const R d = gj - gi;
        const R e = ssym - sym;
        const R h = sasym + asym;
        const R os_i = d + e + h;
        const R os_j = e - d - h;
        const R pw = p.pref * w;
        const R t9 = R(9) * cu * cF;
        const R G_i = pw * (R(3) * (cF - uf) + t9);
        const R G_j = pw * (R(3) * (-cF - uf) + t9);
        g[i] = gi - kb * (gi - (sym + asym)) + B * os_i + G_i;
        g[j] = gj - kb * (gj - (sym - asym)) + B * os_j + G_j;
        if (IMB) {
            const R dm = B * (os_i - os_j);  // c_i B os_i + c_j B os_j = c_i B (os_i - os_j)
            ax += csel(cxv(i), dm);
            ay += csel(cyv(i), dm);
            az += csel(czv(i), dm);
        }
    }
    if (IMB) {
        imb[0] = ax;
        imb[1] = ay;
        imb[2] = az;
    }
}

}  // namespace psc

namespace psc {

// ===========================================================================
// fast deviation form with per-window constants hoisted (throughput kernels)
// ===========================================================================
// Everything that depends only on the window (tau, F) is computed once per
// window: (1 - B)/tau comes from a per-level table, the Guo terms are split
// into per-direction constants A_k = 3 pref w_k (c_k . F) and
// K_k = 9 pref w_k (c_k . F) so that G_i = K_k cu - 3 pref w uF +- A_k.
template <typename R>
struct WinConst {
    R inv_tau;
    R trt_ratio;  // omega- / omega+ (1 for BGK)
    R fx, fy, fz;
    R pw3[3];  // 3 pref w for the rest, axis and diagonal weights
    R A[9];    // 3 pref w_k (c_k . F) for the nine direction pairs
    R K[9];    // 9 pref w_k (c_k . F)
};

// tau_minus > 0 selects two-relaxation-time collision (symmetric parts relax
// with 1/tau, antisymmetric with 1/tau_minus; Guo's antisymmetric term takes
// the prefactor 1 - 1/(2 tau_minus)).  tau_minus = tau is BGK.
template <typename R>
PSC_HD void make_win_const(WinConst<R>& c, double tau, double fx, double fy, double fz, double tau_minus = 0.0) {
    const double pref = 1.0 - 0.5 / tau;
    const double tm = tau_minus > 0.0 ? tau_minus : tau;
    const double pref_m = 1.0 - 0.5 / tm;
    c.inv_tau = (R)(1.0 / tau);
    c.trt_ratio = (R)(tau / tm);
    c.fx = (R)fx;
    c.fy = (R)fy;
    c.fz = (R)fz;
    c.pw3[0] = (R)(3.0 * pref * W0);
    c.pw3[1] = (R)(3.0 * pref * W1);
    c.pw3[2] = (R)(3.0 * pref * W2);
    for (int k = 0; k < 9; ++k) {
        const int i = 2 * k + 1;
        const double w = wgt(i);
        const double cf = cxv(i) * fx + cyv(i) * fy + czv(i) * fz;
        c.A[k] = (R)(3.0 * pref_m * w * cf);
        c.K[k] = (R)(9.0 * pref * w * cf);
    }
}

// Collide deviations g in place.  B solid weight, kb = (1 - B) / tau.
// mom receives rho - 1 and the moment velocity u = (m + F/2)/rho of the
// incoming state; imb the node IMB momentum when IMB.
template <typename R, bool MOVING, bool IMB, bool TRT = false>
PSC_HD void collide_fast2(R* g, const WinConst<R>& c, R B, R kb, R usx, R usy, R usz, R irho_hint, R* mom,
                          R* imb, bool want_mom = true) {
    const R kbm = kb * c.trt_ratio;
    (void)kbm;
    const R drho = (((g[0] + g[1]) + (g[2] + g[3])) + ((g[4] + g[5]) + (g[6] + g[7]))) +
                   (((g[8] + g[9]) + (g[10] + g[11])) + ((g[12] + g[13]) + (g[14] + g[15]))) +
                   ((g[16] + g[17]) + g[18]);
    const R rho = R(1) + drho;
    const R irho = irho_hint > R(0) ? irho_hint : R(1) / rho;
    const R mx = ((g[1] - g[2]) + (g[7] - g[8])) + ((g[9] - g[10]) + (g[11] - g[12])) + (g[13] - g[14]);
    const R my = ((g[3] - g[4]) + (g[7] - g[8])) + ((g[10] - g[9]) + (g[15] - g[16])) + (g[17] - g[18]);
    const R mz = ((g[5] - g[6]) + (g[11] - g[12])) + ((g[14] - g[13]) + (g[15] - g[16])) + (g[18] - g[17]);
    if (want_mom) {  // (plain steps of the throughput kernels store no moments)
        mom[0] = drho;
        mom[1] = (mx + R(0.5) * c.fx) * irho;
        mom[2] = (my + R(0.5) * c.fy) * irho;
        mom[3] = (mz + R(0.5) * c.fz) * irho;
    }
    const R uex = (mx + c.fx) * irho, uey = (my + c.fy) * irho, uez = (mz + c.fz) * irho;
    const R uu15 = R(1.5) * (uex * uex + uey * uey + uez * uez);
    const R uF = uex * c.fx + uey * c.fy + uez * c.fz;
    const R omk = R(1) - kb;
    R uus15 = R(0);
    if (MOVING) uus15 = R(1.5) * (usx * usx + usy * usy + usz * usz);
    R ax = R(0), ay = R(0), az = R(0);
    {
        const R w = R(W0);
        const R geq = w * (drho - rho * uu15);
        const R os = w * rho * (uu15 - uus15);
        g[0] = omk * g[0] + kb * geq + B * os - c.pw3[0] * uF;
    }
    // The collision regrouped per population pair.  With geq = w drho + wrq +- asym, the solid
    // terms os_i = (g_j - g_i) + e + h, os_j = (g_i - g_j) + e - h (e = -wrq + e_s,
    // h = asym + h_s, e_s and h_s from the solid velocity), Guo's G = K cu - 3 pref w uF +- A,
    // and the fluid part relaxing the pair's symmetric half with kb and its antisymmetric half
    // with kbm (= kb for BGK; TRT: kb omega-/omega+):
    //   g_i' = a g_i + b g_j + S + T,   g_j' = a g_j + b g_i + S - T,
    //   a = 1 - (kb + kbm)/2 - B,  b = B + (kbm - kb)/2   (BGK: 1 - kb - B and B),
    //   S = K cu + (kb - B) wrq + (kb w drho - 3 pref w uF) + B e_s,
    //   T = 3 (kbm + B) w rho cu + B h_s + A,
    // and the pair's IMB momentum B (os_i - os_j) = 2 B ((g_j - g_i) + h).  With
    // wrq = w rho (4.5 cu^2 - 1.5 u^2), S without e_s is the quadratic cu (q cu + K) + b,
    // q = 4.5 (kb - B) w rho, b = kb w drho - 3 pref w uF - (kb - B) w rho 1.5 u^2: two FMAs per
    // pair.  The per-weight factors are computed once per cell.
    const R omB = TRT ? R(1) - R(0.5) * (kb + kbm) - B : omk - B;
    const R bB = TRT ? B + R(0.5) * (kbm - kb) : B;
    const R kmB = kb - B, B2 = B + B;
    const R kbd = kb * drho;
    const R wr1 = R(W1) * rho, wr2 = R(W2) * rho;
    const R m1 = kmB * wr1, m2 = kmB * wr2;
    const R q1 = R(4.5) * m1, q2 = R(4.5) * m2;
    const R b1 = (R(W1) * kbd - c.pw3[1] * uF) - m1 * uu15, b2 = (R(W2) * kbd - c.pw3[2] * uF) - m2 * uu15;
    const R kp3 = R(3) * ((TRT ? kbm : kb) + B);
    const R t1 = kp3 * wr1, t2 = kp3 * wr2;
    const R a1 = R(3) * wr1, a2 = R(3) * wr2;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const int i = 2 * k + 1, j = i + 1;
        const bool axis = i < 7;
        const R wr = axis ? wr1 : wr2;
        const R cu = csel(cxv(i), uex) + csel(cyv(i), uey) + csel(czv(i), uez);
        R S = cu * ((axis ? q1 : q2) * cu + c.K[k]) + (axis ? b1 : b2);
        R T = (axis ? t1 : t2) * cu + c.A[k];
        R h = (axis ? a1 : a2) * cu;
        if (MOVING) {
            const R cus = csel(cxv(i), usx) + csel(cyv(i), usy) + csel(czv(i), usz);
            S += B * (wr * (R(4.5) * cus * cus - uus15));
            const R hs = R(3) * wr * cus;
            T += B * hs;
            h += hs;
        }
        const R gi = g[i], gj = g[j];
        g[i] = omB * gi + (bB * gj + (S + T));
        g[j] = omB * gj + (bB * gi + (S - T));
        if (IMB) {
            const R dm = B2 * ((gj - gi) + h);
            ax += csel(cxv(i), dm);
            ay += csel(cyv(i), dm);
            az += csel(czv(i), dm);
        }
    }
    if (IMB) {
        imb[0] = ax;
        imb[1] = ay;
        imb[2] = az;
    }
}

}  // namespace psc

namespace psc {

// ===========================================================================
// voxel bounce-back D3Q19 (scripts/run_3d_window_lbm.py:95-146), exact FP64
// ===========================================================================
// At a solid node the reference overwrites populations in index order,
// f[i] = f[OPP[i]] for i = 0..18 (:117-119); because f[2k+1] is overwritten
// before f[2k+2] reads it, both members of each pair end up holding the old
// f[2k+2].  Reproduced as written.
PSC_HD void bounce_solid_as_reference(double* f) {
#pragma unroll
    for (int k = 0; k < 9; ++k) f[2 * k + 1] = f[2 * k + 2];
}

// BGK + Guo with the single half-force shift of run_3d_window_lbm.py:106-114:
// u = (m + F/2)/rho, u = 0 at solid nodes, f <- f - (f - feq)/tau + guo(u).
PSC_HD void collide_bb_exact(double* f, bool solid, double tau, double fx, double fy, double fz, double* mom) {
    const double hfx = xmul(0.5, fx), hfy = xmul(0.5, fy), hfz = xmul(0.5, fz);
    ExactMoments mo = moments_exact(f, hfx, hfy, hfz);
    if (solid) {
        mo.ux = 0.0;
        mo.uy = 0.0;
        mo.uz = 0.0;
    }
    mom[0] = mo.rho;
    mom[1] = mo.ux;
    mom[2] = mo.uy;
    mom[3] = mo.uz;
    const double rho = mo.rho, ux = mo.ux, uy = mo.uy, uz = mo.uz;
    const Divisor by_tau = make_divisor(tau);
    const double uu = xadd(xadd(xmul(ux, ux), xmul(uy, uy)), xmul(uz, uz));
    const double ct = div_cs2(xmul(0.5, uu));
    const double pref = xsub(1.0, xdiv_d(0.5, by_tau));
    const double uf = xadd(xadd(xmul(ux, fx), xmul(uy, fy)), xmul(uz, fz));
    {
        const double feq = xmul(xmul(W0, rho), xsub(1.0, ct));
        const double g = xmul(xmul(pref, W0), div_cs2(-uf));
        f[0] = xadd(xsub(f[0], xdiv_d(xsub(f[0], feq), by_tau)), g);
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const int i = 2 * k + 1, j = i + 1;
        const double w = wgt(i);
        const double wr = xmul(w, rho);
        const double cu = xadd(xadd(cm(cxv(i), ux), cm(cyv(i), uy)), cm(czv(i), uz));
        const double q = div_cs2(cu);
        const double b = div_cs2sq(xmul(xmul(0.5, cu), cu));
        const double feq_i = xmul(wr, xsub(xadd(xadd(1.0, q), b), ct));
        const double feq_j = xmul(wr, xsub(xadd(xadd(1.0, -q), b), ct));
        const double cf = xadd(xadd(cm(cxv(i), fx), cm(cyv(i), fy)), cm(czv(i), fz));
        const double pw = xmul(pref, w);
        const double t2 = div_cs2sq(xmul(cu, cf));
        const double g_i = xmul(pw, xadd(div_cs2(xsub(cf, uf)), t2));
        const double g_j = xmul(pw, xadd(div_cs2(xsub(-cf, uf)), t2));
        f[i] = xadd(xsub(f[i], xdiv_d(xsub(f[i], feq_i), by_tau)), g_i);
        f[j] = xadd(xsub(f[j], xdiv_d(xsub(f[j], feq_j), by_tau)), g_j);
    }
}

}  // namespace psc
