// Discrete adjoint of the Darcy permeability with respect to the particles'
// centres and radii (no counterpart in the reference; it differentiates the
// reference's step, src/lbm_dem/psc3d.py:208-246, and the caller-side K of
// scripts/run_psc_permeability_resolution.py:144-150).
//
// Forward model: static particles, deviation storage (F64 or F32), smooth
// solid fraction (psc_geometry.smooth_eps > 0), pull streaming with stored
// post-collision states S_t, f_t = pull(S_t), S_{t+1} = C(f_t; B).
// K = kappa * sum_x (1 - solid) u.dir of pull(S_T), u = (m + F/2) / rho.
//
// Reverse pass, one launch per step (t = T-1 .. 0):
//   mu(x)            = J_C(f_t(x))^T lambda_{t+1}(x)      (local 19x19, by hand)
//   lambda_t(x - c_i) = mu_i(x)                          (pull^T = push; one
//                                                         store per element)
//   dK/dB(x)        += lambda_{t+1}(x) . dC/dB(f_t(x))
// Each reverse step reads S_t (pulled) and lambda_{t+1}, writes lambda_t and
// updates one FP64 accumulator per cell: ~1.6x the bytes of a forward step.
#include "collide.cuh"
#include "internal.cuh"

namespace psc {

namespace {

template <typename R>
struct Pull19 {
    R v[Q];
};

__device__ __forceinline__ void decode(uint32_t cell, int nx, int ny, int nz, uint32_t& ix, uint32_t& iy,
                                       uint32_t& iz) {
    iz = cell % (uint32_t)nz;
    const uint32_t r = cell / (uint32_t)nz;
    iy = r % (uint32_t)ny;
    ix = r / (uint32_t)ny;
}

// offset from x to x - c_i (periodic)
template <int I>
__device__ __forceinline__ int32_t src_off(int32_t xm, int32_t xp, int32_t ym, int32_t yp, int32_t zm, int32_t zp) {
    return (cxv(I) == 1 ? xm : (cxv(I) == -1 ? xp : 0)) + (cyv(I) == 1 ? ym : (cyv(I) == -1 ? yp : 0)) +
           (czv(I) == 1 ? zm : (czv(I) == -1 ? zp : 0));
}

template <int I = 0>
__device__ __forceinline__ void offsets(int32_t* off, int32_t xm, int32_t xp, int32_t ym, int32_t yp, int32_t zm,
                                        int32_t zp) {
    if constexpr (I < Q) {
        off[I] = src_off<I>(xm, xp, ym, yp, zm, zp);
        offsets<I + 1>(off, xm, xp, ym, yp, zm, zp);
    }
}

__device__ __forceinline__ void coord_offsets(uint32_t ix, uint32_t iy, uint32_t iz, int nx, int ny, int nz,
                                              int32_t* off) {
    const int32_t nyz = ny * nz;
    const int32_t xm = ix == 0 ? (nx - 1) * nyz : -nyz;
    const int32_t xp = ix == (uint32_t)(nx - 1) ? -(nx - 1) * nyz : nyz;
    const int32_t ym = iy == 0 ? (ny - 1) * nz : -nz;
    const int32_t yp = iy == (uint32_t)(ny - 1) ? -(ny - 1) * nz : nz;
    const int32_t zm = iz == 0 ? nz - 1 : -1;
    const int32_t zp = iz == (uint32_t)(nz - 1) ? -(nz - 1) : 1;
    offsets(off, xm, xp, ym, yp, zm, zp);
}

__device__ __forceinline__ void cell_offsets(uint32_t cell, int nx, int ny, int nz, int32_t* off) {
    uint32_t ix, iy, iz;
    decode(cell, nx, ny, nz, ix, iy, iz);
    coord_offsets(ix, iy, iz, nx, ny, nz, off);
}

// Cell coordinates of a grid-stride loop: decoded once, then advanced by the
// stride's own (x, y, z) digits with carries (no division per cell).
struct StrideWalk {
    uint32_t ix, iy, iz, sx, sy, sz, ny, nz;
    __device__ __forceinline__ StrideWalk(uint32_t cell, uint32_t stride, int nx, int ny_, int nz_) {
        ny = (uint32_t)ny_;
        nz = (uint32_t)nz_;
        decode(cell, nx, ny_, nz_, ix, iy, iz);
        sz = stride % nz;
        const uint32_t q = stride / nz;
        sy = q % ny;
        sx = q / ny;
    }
    __device__ __forceinline__ void next() {
        iz += sz;
        const uint32_t cz = iz >= nz;
        iz -= cz ? nz : 0u;
        iy += sy + cz;
        const uint32_t cy = iy >= ny;
        iy -= cy ? ny : 0u;
        ix += sx + cy;
    }
};

}  // namespace

// lambda_T(x - c_i) = dK/df_i(x) = kappa (1 - solid) (c_i.dir - u.dir) / rho ; dK/dsolid = -kappa u.dir
template <typename R>
__global__ void k_adjoint_seed(psc_adjoint_args a) {
    const uint32_t N = (uint32_t)a.nx * a.ny * a.nz;
    const R* S = reinterpret_cast<const R*>(a.state);
    R* lam = reinterpret_cast<R*>(a.lam_out);
    const R dx = (R)a.dir[0], dy = (R)a.dir[1], dz = (R)a.dir[2];
    const R fx = (R)a.force[0], fy = (R)a.force[1], fz = (R)a.force[2];
    for (uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x; cell < N; cell += gridDim.x * blockDim.x) {
        int32_t off[Q];
        cell_offsets(cell, a.nx, a.ny, a.nz, off);
        R g[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] = S[(size_t)i * N + (size_t)((int64_t)cell + off[i])];
        const FastMoments<R> mo = moments_fast(g);
        const R irho = R(1) / mo.rho;
        const R uF = ((mo.mx + R(0.5) * fx) * dx + (mo.my + R(0.5) * fy) * dy + (mo.mz + R(0.5) * fz) * dz) * irho;
        const double solid = a.solid[cell];
        const R w = (R)(a.kappa * (1.0 - solid));
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const R cd = (R)cxv(i) * dx + (R)cyv(i) * dy + (R)czv(i) * dz;
            lam[(size_t)i * N + (size_t)((int64_t)cell + off[i])] = w * (cd - uF) * irho;
        }
        a.dKdsolid[cell] = -a.kappa * (double)uF;
        a.dKdB[cell] = 0.0;
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_adjoint_step(psc_adjoint_args a) {
    const uint32_t N = (uint32_t)a.nx * a.ny * a.nz;
    const R* S = reinterpret_cast<const R*>(a.state);
    const R* lin = reinterpret_cast<const R*>(a.lam_in);
    R* lout = reinterpret_cast<R*>(a.lam_out);
    const R tau = (R)a.tau, inv_tau = R(1) / tau, pref = R(1) - R(0.5) / tau;
    const R Fx = (R)a.force[0], Fy = (R)a.force[1], Fz = (R)a.force[2];
    const uint32_t stride = gridDim.x * blockDim.x;
    StrideWalk at(blockIdx.x * blockDim.x + threadIdx.x, stride, a.nx, a.ny, a.nz);
    for (uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x; cell < N; cell += stride, at.next()) {
        int32_t off[Q];
        coord_offsets(at.ix, at.iy, at.iz, a.nx, a.ny, a.nz, off);
        R g[Q], lam[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            g[i] = S[(size_t)i * N + (size_t)((int64_t)cell + off[i])];
            lam[i] = lin[(size_t)i * N + cell];
        }
        const R al = (R)a.solid[cell];
        const R B = al / (al + tau * (R(1) - al) + R(1.0e-14));
        const FastMoments<R> mo = moments_fast(g);
        const R rho = mo.rho, drho = mo.drho, irho = R(1) / rho;
        const R uex = (mo.mx + Fx) * irho, uey = (mo.my + Fy) * irho, uez = (mo.mz + Fz) * irho;
        const R uu = uex * uex + uey * uey + uez * uez;
        const R kb = (R(1) - B) * inv_tau;
        const R direct = R(1) - kb - B;
        R mu[Q];
        R dB = R(0), drho_bar = R(0), s1 = R(0), s2 = R(0);
        R Vx = R(0), Vy = R(0), Vz = R(0);
        {  // rest population
            const R w = R(W0);
            const R geq = w * (drho - R(1.5) * rho * uu);
            const R os = w * drho - geq;
            dB += lam[0] * ((g[0] - geq) * inv_tau + os);
            const R a0 = (kb - B) * lam[0];
            mu[0] = (R(1) - kb) * lam[0];
            drho_bar += B * w * lam[0] + a0 * w * (R(1) - R(1.5) * uu);
            s1 += R(3) * w * rho * a0;
            s2 += R(3) * pref * w * lam[0];
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const int i = 2 * k + 1, j = i + 1;
            const R w = R(wgt(i));
            const R cu = csel(cxv(i), uex) + csel(cyv(i), uey) + csel(czv(i), uez);
            const R cF = csel(cxv(i), Fx) + csel(cyv(i), Fy) + csel(czv(i), Fz);
            const R q2 = R(4.5) * cu * cu - R(1.5) * uu;
            const R sym = w * (drho + rho * q2);
            const R asym = R(3) * w * rho * cu;
            const R geq_i = sym + asym, geq_j = sym - asym;
            const R os_i = g[j] - g[i] + w * drho - geq_j;
            const R os_j = g[i] - g[j] + w * drho - geq_i;
            const R li = lam[i], lj = lam[j];
            dB += li * ((g[i] - geq_i) * inv_tau + os_i) + lj * ((g[j] - geq_j) * inv_tau + os_j);
            const R ai = kb * li - B * lj, aj = kb * lj - B * li;
            mu[i] = direct * li + B * lj;
            mu[j] = direct * lj + B * li;
            drho_bar += B * w * (li + lj) + w * (ai * (R(1) + R(3) * cu + q2) + aj * (R(1) - R(3) * cu + q2));
            const R vc = w * rho * (ai * (R(3) + R(9) * cu) - aj * (R(3) - R(9) * cu)) + R(9) * pref * w * cF * (li + lj);
            Vx += csel(cxv(i), vc);
            Vy += csel(cyv(i), vc);
            Vz += csel(czv(i), vc);
            s1 += R(3) * w * rho * (ai + aj);
            s2 += R(3) * pref * w * (li + lj);
        }
        const R ubx = Vx - s1 * uex - s2 * Fx;
        const R uby = Vy - s1 * uey - s2 * Fy;
        const R ubz = Vz - s1 * uez - s2 * Fz;
        const R mbx = ubx * irho, mby = uby * irho, mbz = ubz * irho;
        drho_bar -= (ubx * uex + uby * uey + ubz * uez) * irho;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const R v = mu[i] + drho_bar + csel(cxv(i), mbx) + csel(cyv(i), mby) + csel(czv(i), mbz);
            lout[(size_t)i * N + (size_t)((int64_t)cell + off[i])] = v;
        }
        a.dKdB[cell] += (double)dB;
    }
}

// Per-cell dK/d(alpha_sum) = (dK/dB dB/dalpha + dK/dsolid) [0 < alpha_sum < 1], then
// per-particle sums over bbox entries of dK/dalpha_sum * d alpha_p / d(x, y, z, r).
constexpr int GRAD_THREADS = 256;

__global__ void __launch_bounds__(GRAD_THREADS) k_adjoint_geom_chunks(psc_geometry g, psc_adjoint_args a,
                                                                       double* part) {
    __shared__ double s[GRAD_THREADS / 32][4];
    const int64_t C = g.totals[1];
    const int S = g.subsamples;
    const double Sd = (double)S, eps = g.smooth_eps, tau = a.tau;
    const double inv_s3 = 1.0 / (Sd * Sd * Sd);
    for (int64_t chunk = blockIdx.x; chunk < C; chunk += gridDim.x) {
        // owner particle of this chunk (largest p with chunk_off[p] <= chunk)
        int lo = 0, hi = g.nparticles - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (g.chunk_off[mid] <= chunk) lo = mid;
            else hi = mid - 1;
        }
        const int p = lo;
        const int64_t e0 = g.ent_off[p] + (chunk - g.chunk_off[p]) * g.chunk_entries;
        const int64_t e1 = min(e0 + (int64_t)g.chunk_entries, g.ent_off[p + 1]);
        const double* q = g.particles + (size_t)p * 10;
        const int32_t* bb = g.bbox + (size_t)p * 6;
        const int64_t eyz = (int64_t)bb[4] * bb[5];
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
            const int64_t local = e - g.ent_off[p];
            const int32_t ia = (int32_t)(local / eyz);
            const int64_t rem = local - (int64_t)ia * eyz;
            const int32_t ib = (int32_t)(rem / bb[5]);
            const int32_t ic = (int32_t)(rem - (int64_t)ib * bb[5]);
            const int32_t ix = bb[0] + ia, iy = bb[1] + ib, iz = bb[2] + ic;
            const uint32_t cell = ((uint32_t)ix * g.ny + iy) * g.nz + iz;
            const double as = g.alpha_sum[cell];
            if (!(as > 0.0 && as < 1.0)) continue;  // clip: zero derivative outside (0, 1)
            const double D = as + tau * (1.0 - as) + 1.0e-14;
            const double gcell = a.dKdB[cell] * (tau + 1.0e-14) / (D * D) + a.dKdsolid[cell];
            double gx = 0.0, gy = 0.0, gz = 0.0, gr = 0.0;
            for (int sa = 0; sa < S; ++sa) {
                const double dx = ((double)ix + ((double)sa + 0.5) / Sd) - q[0];
                for (int sb = 0; sb < S; ++sb) {
                    const double dy = ((double)iy + ((double)sb + 0.5) / Sd) - q[1];
                    for (int sc = 0; sc < S; ++sc) {
                        const double dz = ((double)iz + ((double)sc + 0.5) / Sd) - q[2];
                        const double d = sqrt(dx * dx + dy * dy + dz * dz);
                        const double sg = 0.5 * (1.0 + tanh(0.5 * (q[3] - d) / eps));
                        const double ds = sg * (1.0 - sg) / eps;
                        const double dinv = d > 1.0e-12 ? 1.0 / d : 0.0;
                        gr += ds;
                        gx += ds * dx * dinv;
                        gy += ds * dy * dinv;
                        gz += ds * dz * dinv;
                    }
                }
            }
            const double f = gcell * inv_s3;
            acc[0] += f * gx;
            acc[1] += f * gy;
            acc[2] += f * gz;
            acc[3] += f * gr;
        }
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            double x = acc[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (lane == 0) s[warp][k] = x;
        }
        __syncthreads();
        if (threadIdx.x < 4) {
            double t = 0.0;
            for (int w = 0; w < nw; ++w) t += s[w][threadIdx.x];
            part[chunk * 4 + threadIdx.x] = t;
        }
        __syncthreads();
    }
}

__global__ void k_adjoint_geom_final(psc_geometry g, const double* part, double* grad) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.nparticles; p += gridDim.x * blockDim.x) {
        double t[4] = {0.0, 0.0, 0.0, 0.0};
        for (int64_t c = g.chunk_off[p]; c < g.chunk_off[p + 1]; ++c)
            for (int k = 0; k < 4; ++k) t[k] += part[c * 4 + k];
        for (int k = 0; k < 4; ++k) grad[(size_t)p * 4 + k] = t[k];
    }
}

static unsigned cap_grid(int64_t work, int threads, int per_sm) {
    int64_t g = (work + threads - 1) / threads;
    const int64_t cap = (int64_t)sm_count() * per_sm;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (unsigned)g;
}

cudaError_t launch_adjoint_seed(const psc_adjoint_args& a, cudaStream_t stream) {
    const int64_t N = (int64_t)a.nx * a.ny * a.nz;
    if (a.store == PSC_STORE_F64) k_adjoint_seed<double><<<cap_grid(N, 256, 8), 256, 0, stream>>>(a);
    else k_adjoint_seed<float><<<cap_grid(N, 256, 8), 256, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_step(const psc_adjoint_args& a, cudaStream_t stream) {
    const int64_t N = (int64_t)a.nx * a.ny * a.nz;
    if (a.store == PSC_STORE_F64) k_adjoint_step<double><<<cap_grid(N, 256, 8), 256, 0, stream>>>(a);
    else k_adjoint_step<float><<<cap_grid(N, 256, 8), 256, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_geometry_grad(const psc_geometry& g, const psc_adjoint_args& a, double* part,
                                         double* grad, cudaStream_t stream) {
    if (g.nparticles <= 0) return cudaSuccess;
    if (g.capacity_chunks > 0) {
        const int64_t cap = (int64_t)sm_count() * 8;
        const unsigned grid = (unsigned)(g.capacity_chunks < cap ? g.capacity_chunks : cap);
        k_adjoint_geom_chunks<<<grid, GRAD_THREADS, 0, stream>>>(g, a, part);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    k_adjoint_geom_final<<<cap_grid(g.nparticles, 256, 4), 256, 0, stream>>>(g, part, grad);
    return cudaGetLastError();
}

}  // namespace psc
