// Per-window set-up and per-cell work shared by the deviation-storage
// kernels (k_step_fast: one cell per thread at a time; k_step_pair: two
// consecutive z cells per thread with paired loads and stores), so both run
// the same arithmetic on every cell.
#pragma once

#include "step_common.cuh"

namespace psc {

template <typename T, typename R, typename O>
struct FastWin {
    const T* src;
    T* dst;
    const uint8_t* level;
    const double* solid;
    const O* us;
    O* imb;
    O* mom;
    double* partials;
    int64_t tile_begin;
    int64_t tile_end;
    uint32_t nx, ny, nz, N;
    uint32_t step_x, step_y, step_z;     // blockDim cells as a mixed-radix (x, y, z) increment
    uint32_t tstep_x, tstep_y, tstep_z;  // tile_cells cells (one tile on) likewise
    int32_t tile_cells;
    int32_t moving;
    int32_t inactive;
    int32_t trt;
    int32_t open_x;  // PSC_WIN_OPEN_X
    R scale, inv_scale;
    WinConst<R> c;
    R corr[Q];       // open_x: bounce-back inlet term 2 w_i rho_in (c_i . u_in) / cs^2
    R Blut[256];
    R kblut[256];
    R alut[256];  // clipped solid fraction per level
    R tau;
};

template <typename T, typename R, typename O>
__device__ void load_fast_win(FastWin<T, R, O>& s, const psc_window& W, bool moving_launch) {
    // one warp fills the scalar part, all threads the level tables
    if (threadIdx.x == 0) {
        s.src = reinterpret_cast<const T*>(W.f_src);
        s.dst = reinterpret_cast<T*>(W.f_dst);
        s.level = W.level;
        s.solid = W.solid;
        s.us = reinterpret_cast<const O*>(W.us);
        s.imb = reinterpret_cast<O*>(W.imb);
        s.mom = reinterpret_cast<O*>(W.moments);
        s.partials = W.partials;
        s.tile_begin = W.tile_begin;
        s.tile_end = W.tile_begin + W.tile_count;
        s.nx = W.nx;
        s.ny = W.ny;
        s.nz = W.nz;
        s.N = (uint32_t)W.nx * W.ny * W.nz;
        const uint32_t q = blockDim.x / (uint32_t)W.nz;
        s.step_z = blockDim.x % (uint32_t)W.nz;
        s.step_y = q % (uint32_t)W.ny;
        s.step_x = q / (uint32_t)W.ny;
        const uint32_t tc = W.tile_cells > 0 ? (uint32_t)W.tile_cells : 0u;
        const uint32_t tq = tc / (uint32_t)W.nz;
        s.tstep_z = tc % (uint32_t)W.nz;
        s.tstep_y = tq % (uint32_t)W.ny;
        s.tstep_x = tq / (uint32_t)W.ny;
        s.tile_cells = W.tile_cells;
        s.moving = (moving_launch && (W.flags & PSC_WIN_MOVING) && W.us != nullptr) ? 1 : 0;
        s.inactive = (W.flags & PSC_WIN_INACTIVE) ? 1 : 0;
        s.scale = (R)W.store_scale;
        s.inv_scale = (R)(1.0 / W.store_scale);
        s.tau = (R)W.tau;
        make_win_const(s.c, W.tau, W.force[0], W.force[1], W.force[2], W.tau_minus);
        s.trt = W.tau_minus > 0.0 ? 1 : 0;
        s.open_x = (W.flags & PSC_WIN_OPEN_X) ? 1 : 0;
    }
    if ((W.flags & PSC_WIN_OPEN_X) && threadIdx.x < Q) {
        const int i = threadIdx.x;
        s.corr[i] = (R)inlet_correction_exact(i, W.inlet_rho, W.inlet_u[0], W.inlet_u[1], W.inlet_u[2]);
    }
    const int S = W.subsamples;
    const int S3 = S * S * S;
    if (W.level) {
        for (int l = threadIdx.x; l <= S3 && l < 256; l += blockDim.x) {
            const double al = (double)l / (double)S3;
            const double B = al / (al + W.tau * (1.0 - al) + 1.0e-14);
            s.Blut[l] = (R)B;
            s.kblut[l] = (R)((1.0 - B) / W.tau);
            s.alut[l] = (R)al;
        }
    }
}

// RED: PSC_STEP_REDUCE as a compile-time switch, so launches without
// reductions carry no loop-carried FP64 accumulators.
// The per-cell work after the pulls (psc3d.py:211-246): inlet fix-up at an
// open x = 0, solid weight from the level tables, collision (or the moments
// only), and this thread's reduction sums.  g holds the pulled populations in
// stored units on entry and the post-collision deviations on exit; mom and
// imb receive the cell's moments (rho - 1, u) and IMB momentum.  The caller
// stores g, imb and mom.
template <typename TR, bool MOVING, bool RED>
__device__ __forceinline__ void fast_cell(const FastWin<typename TR::T, typename TR::R, typename TR::O>& sw,
                                          typename TR::R (&g)[Q], uint32_t c, uint32_t N, bool inlet, bool do_collide,
                                          bool do_imb, typename TR::R (&mom)[4], typename TR::R (&imb)[3],
                                          double (&red)[PSC_NRED], bool do_mom = true) {
    using R = typename TR::R;
    constexpr bool do_red = RED;
    if (TR::scaled) {
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] *= sw.inv_scale;
    }
    if (inlet) {  // velocity inlet at x = 0 (the x = 0 plane only): bounce-back of the node's own
                     // opp(i) + 2 w_i rho_in (c_i . u_in) / cs^2
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            if (!enters_x0(i)) continue;
            R back = ld_pop(sw.src + (size_t)opp(i) * N + c);
            if (TR::scaled) back *= sw.inv_scale;
            g[i] = back + sw.corr[i];
        }
    }
    R B, kb, al;
    if (sw.level) {
        const uint8_t lv = sw.level[c];
        B = sw.Blut[lv];
        kb = sw.kblut[lv];
        al = sw.alut[lv];
    } else {
        al = (R)sw.solid[c];
        B = al * fast_rcp<R>(al + sw.tau * (R(1) - al) + R(1.0e-14));
        kb = (R(1) - B) * sw.c.inv_tau;
    }
    R usx = R(0), usy = R(0), usz = R(0);
    const bool moving = MOVING && sw.moving;
    if (moving) {
        usx = (R)sw.us[c];
        usy = (R)sw.us[(size_t)N + c];
        usz = (R)sw.us[2 * (size_t)N + c];
    }
    imb[0] = imb[1] = imb[2] = R(0);
    const R drho = (((g[0] + g[1]) + (g[2] + g[3])) + ((g[4] + g[5]) + (g[6] + g[7]))) +
                   (((g[8] + g[9]) + (g[10] + g[11])) + ((g[12] + g[13]) + (g[14] + g[15]))) +
                   ((g[16] + g[17]) + g[18]);
    const R irho = fast_rcp<R>(R(1) + drho);
    const bool want_mom = do_mom || RED;
    if (do_collide) {
        if (sw.trt) {
            if (moving) collide_fast2<R, MOVING, true, true>(g, sw.c, B, kb, usx, usy, usz, irho, mom, imb, want_mom);
            else collide_fast2<R, false, true, true>(g, sw.c, B, kb, usx, usy, usz, irho, mom, imb, want_mom);
        } else if (do_imb || do_red) {
            if (moving) collide_fast2<R, MOVING, true>(g, sw.c, B, kb, usx, usy, usz, irho, mom, imb, want_mom);
            else collide_fast2<R, false, true>(g, sw.c, B, kb, usx, usy, usz, irho, mom, imb, want_mom);
        } else {
            if (moving) collide_fast2<R, MOVING, false>(g, sw.c, B, kb, usx, usy, usz, irho, mom, imb, want_mom);
            else collide_fast2<R, false, false>(g, sw.c, B, kb, usx, usy, usz, irho, mom, imb, want_mom);
        }
    } else {
        const R mx = ((g[1] - g[2]) + (g[7] - g[8])) + ((g[9] - g[10]) + (g[11] - g[12])) + (g[13] - g[14]);
        const R my = ((g[3] - g[4]) + (g[7] - g[8])) + ((g[10] - g[9]) + (g[15] - g[16])) + (g[17] - g[18]);
        const R mz = ((g[5] - g[6]) + (g[11] - g[12])) + ((g[14] - g[13]) + (g[15] - g[16])) + (g[18] - g[17]);
        mom[0] = drho;
        mom[1] = (mx + R(0.5) * sw.c.fx) * irho;
        mom[2] = (my + R(0.5) * sw.c.fy) * irho;
        mom[3] = (mz + R(0.5) * sw.c.fz) * irho;
    }
    if (do_red) {
        const double solid = (double)al;
        const double fl = 1.0 - solid;
        const double rho_d = 1.0 + (double)mom[0];
        const double ux = (double)mom[1], uy = (double)mom[2], uz = (double)mom[3];
        red[PSC_RED_RHO] += rho_d;
        red[PSC_RED_UX] += ux;
        red[PSC_RED_UY] += uy;
        red[PSC_RED_UZ] += uz;
        red[PSC_RED_FLUID_UX] += fl * ux;
        red[PSC_RED_FLUID_UY] += fl * uy;
        red[PSC_RED_FLUID_UZ] += fl * uz;
        red[PSC_RED_FLUID] += fl;
        red[PSC_RED_IMBX] += (double)imb[0];
        red[PSC_RED_IMBY] += (double)imb[1];
        red[PSC_RED_IMBZ] += (double)imb[2];
        red[PSC_RED_NONFINITE] += (isfinite(rho_d) && isfinite(ux) && isfinite(uy) && isfinite(uz)) ? 0.0 : 1.0;
        red[PSC_RED_SOLID] += solid;
    }
}

}  // namespace psc
