// Voxel bounce-back D3Q19 window LBM (the reference's second, simpler
// solver: scripts/run_3d_window_lbm.py, voxelize :73-92, run_lbm :95-146).
//
// Binary solid from sphere centres (cell-centre inside test), then per step,
// fused in one pull pass over post-collision populations:
//   pull f(x) = fpost(x - c)          (the reference's np.roll push, :115-116)
//   solid x: in-place pair overwrite   (:117-119, reproduced as written)
//   moments, u = 0 at solid nodes      (:104-110)
//   BGK + Guo, single half-force shift (:113-114)
// Exact FP64 arithmetic in the reference's operation order.
#include "collide.cuh"
#include "internal.cuh"

namespace psc {

// One block per sphere: cells of its clamped box whose centre lies inside.
__global__ void k_vox_spheres(const double* __restrict__ pts, int M, double lox, double loy, double loz, double dxx,
                              double dxy, double dxz, double radius, int nx, int ny, int nz, uint8_t* solid) {
    const int m = blockIdx.x;
    if (m >= M) return;
    const double x = pts[3 * m], y = pts[3 * m + 1], z = pts[3 * m + 2];
    // box clamp [max(0, floor((c - r - lo)/dx)), min(n - 1, ceil((c + r - lo)/dx))]
    const int ix0 = max(0, (int)floor(xdiv(xsub(xsub(x, radius), lox), dxx)));
    const int ix1 = min(nx - 1, (int)ceil(xdiv(xsub(xadd(x, radius), lox), dxx)));
    const int iy0 = max(0, (int)floor(xdiv(xsub(xsub(y, radius), loy), dxy)));
    const int iy1 = min(ny - 1, (int)ceil(xdiv(xsub(xadd(y, radius), loy), dxy)));
    const int iz0 = max(0, (int)floor(xdiv(xsub(xsub(z, radius), loz), dxz)));
    const int iz1 = min(nz - 1, (int)ceil(xdiv(xsub(xadd(z, radius), loz), dxz)));
    if (ix1 < ix0 || iy1 < iy0 || iz1 < iz0) return;
    const int ex = ix1 - ix0 + 1, ey = iy1 - iy0 + 1, ez = iz1 - iz0 + 1;
    const double rr = xmul(radius, radius);
    for (int e = threadIdx.x; e < ex * ey * ez; e += blockDim.x) {
        const int a = e / (ey * ez), rem = e - a * ey * ez, b = rem / ez, c = rem - b * ez;
        const int ix = ix0 + a, iy = iy0 + b, iz = iz0 + c;
        // cell centre lo + (i + 0.5) dx (:77), distance test (:91)
        const double cx = xadd(lox, xmul((double)ix + 0.5, dxx));
        const double cy = xadd(loy, xmul((double)iy + 0.5, dxy));
        const double cz = xadd(loz, xmul((double)iz + 0.5, dxz));
        const double ddx = xsub(cx, x), ddy = xsub(cy, y), ddz = xsub(cz, z);
        if (xadd(xadd(xmul(ddx, ddx), xmul(ddy, ddy)), xmul(ddz, ddz)) <= rr)
            solid[((size_t)ix * ny + iy) * nz + iz] = 1;
    }
}

__global__ void __launch_bounds__(256) k_bb_step(const double* __restrict__ src, double* __restrict__ dst,
                                                  const uint8_t* __restrict__ solid, int nx, int ny, int nz,
                                                  double tau, double fx, double fy, double fz, unsigned flags,
                                                  double* __restrict__ mom) {
    const uint32_t N = (uint32_t)nx * ny * nz;
    const bool do_collide = flags & PSC_STEP_COLLIDE;
    const bool do_mom = flags & PSC_STEP_MOMENTS;
    for (uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x; cell < N; cell += gridDim.x * blockDim.x) {
        const uint32_t iz = cell % nz, r = cell / nz, iy = r % ny, ix = r / ny;
        const int32_t nyz = ny * nz;
        const int32_t xm = ix == 0 ? (nx - 1) * nyz : -nyz, xp = ix == (uint32_t)(nx - 1) ? -(nx - 1) * nyz : nyz;
        const int32_t ym = iy == 0 ? (ny - 1) * nz : -nz, yp = iy == (uint32_t)(ny - 1) ? -(ny - 1) * nz : nz;
        const int32_t zm = iz == 0 ? nz - 1 : -1, zp = iz == (uint32_t)(nz - 1) ? -(nz - 1) : 1;
        double f[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int32_t o = (cxv(i) == 1 ? xm : (cxv(i) == -1 ? xp : 0)) +
                              (cyv(i) == 1 ? ym : (cyv(i) == -1 ? yp : 0)) +
                              (czv(i) == 1 ? zm : (czv(i) == -1 ? zp : 0));
            f[i] = src[(size_t)i * N + (size_t)((int64_t)cell + o)];
        }
        const bool s = solid[cell] != 0;
        if (s) bounce_solid_as_reference(f);
        double m[4];
        if (do_collide) {
            collide_bb_exact(f, s, tau, fx, fy, fz, m);
#pragma unroll
            for (int i = 0; i < Q; ++i) dst[(size_t)i * N + cell] = f[i];
        } else {
            ExactMoments mo = moments_exact(f, xmul(0.5, fx), xmul(0.5, fy), xmul(0.5, fz));
            m[0] = mo.rho;
            m[1] = s ? 0.0 : mo.ux;
            m[2] = s ? 0.0 : mo.uy;
            m[3] = s ? 0.0 : mo.uz;
        }
        if (do_mom) {
#pragma unroll
            for (int k = 0; k < 4; ++k) mom[(size_t)k * N + cell] = m[k];
        }
    }
}

cudaError_t launch_vox_spheres(const double* pts, int M, const double* lo, const double* dx, double radius, int nx,
                               int ny, int nz, uint8_t* solid, cudaStream_t s) {
    if (M <= 0) return cudaSuccess;
    k_vox_spheres<<<M, 256, 0, s>>>(pts, M, lo[0], lo[1], lo[2], dx[0], dx[1], dx[2], radius, nx, ny, nz, solid);
    return cudaGetLastError();
}

cudaError_t launch_bb_step(const double* src, double* dst, const uint8_t* solid, int nx, int ny, int nz, double tau,
                           double fx, double fy, double fz, unsigned flags, double* mom, cudaStream_t s) {
    const int64_t N = (int64_t)nx * ny * nz;
    int64_t g = (N + 255) / 256;
    const int64_t cap = (int64_t)sm_count() * 8;
    if (g > cap) g = cap;
    k_bb_step<<<(unsigned)g, 256, 0, s>>>(src, dst, solid, nx, ny, nz, tau, fx, fy, fz, flags, mom);
    return cudaGetLastError();
}

}  // namespace psc

namespace psc {

// Element-wise equilibrium (src/lbm_dem/psc3d.py:97-103) and Guo forcing
// (:106-114) in the reference's operation order, for the module-level helpers.
__global__ void k_equilibrium(const double* rho, const double* ux, const double* uy, const double* uz, double* out,
                              int64_t n) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const double r = rho[c], x = ux[c], y = uy[c], z = uz[c];
        const double uu = xadd(xadd(xmul(x, x), xmul(y, y)), xmul(z, z));
        const double ct = xdiv(xmul(0.5, uu), CS2);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const double cu = xadd(xadd(cm(cxv(i), x), cm(cyv(i), y)), cm(czv(i), z));
            const double a = xadd(1.0, xdiv(cu, CS2));
            const double b = xdiv(xmul(xmul(0.5, cu), cu), CS2SQ);
            out[(size_t)i * n + c] = xmul(xmul(wgt(i), r), xsub(xadd(a, b), ct));
        }
    }
}

__global__ void k_guo(double fx, double fy, double fz, const double* ux, const double* uy, const double* uz,
                      double tau, double* out, int64_t n) {
    const double pref = xsub(1.0, xdiv(0.5, tau));
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const double x = ux[c], y = uy[c], z = uz[c];
        const double uf = xadd(xadd(xmul(x, fx), xmul(y, fy)), xmul(z, fz));
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const double cu = xadd(xadd(cm(cxv(i), x), cm(cyv(i), y)), cm(czv(i), z));
            const double cf = xadd(xadd(cm(cxv(i), fx), cm(cyv(i), fy)), cm(czv(i), fz));
            out[(size_t)i * n + c] =
                xmul(xmul(pref, wgt(i)), xadd(xdiv(xsub(cf, uf), CS2), xdiv(xmul(cu, cf), CS2SQ)));
        }
    }
}

cudaError_t launch_equilibrium(const double* rho, const double* ux, const double* uy, const double* uz, double* out,
                               int64_t n, cudaStream_t s) {
    int64_t g = (n + 255) / 256;
    const int64_t cap = (int64_t)sm_count() * 8;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    k_equilibrium<<<(unsigned)g, 256, 0, s>>>(rho, ux, uy, uz, out, n);
    return cudaGetLastError();
}

cudaError_t launch_guo(double fx, double fy, double fz, const double* ux, const double* uy, const double* uz,
                       double tau, double* out, int64_t n, cudaStream_t s) {
    int64_t g = (n + 255) / 256;
    const int64_t cap = (int64_t)sm_count() * 8;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    k_guo<<<(unsigned)g, 256, 0, s>>>(fx, fy, fz, ux, uy, uz, tau, out, n);
    return cudaGetLastError();
}

}  // namespace psc
