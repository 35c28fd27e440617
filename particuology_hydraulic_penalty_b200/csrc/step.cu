// Fused pull-stream + PSC-IMB collide kernel over a list of lattice windows.
//
// One launch = one lattice step of every window (src/lbm_dem/psc3d.py:208-246):
//   pull      f_i(x) = f*_i(x - c_i)   (periodic; equivalent to the
//             reference's push np.roll(f*_i, c_i) at :239-242)
//   moments   rho, u of the pulled (post-stream) state           (:211-214)
//   collide   Noble-Torczynski PSC + Guo forcing                  (:215-232)
//   write     f*_i(x) to the other buffer, optional IMB momentum   (:234-236)
//   reduce    per-tile FP64 partial sums (flux, porosity, IMB, NaN count)
//
// Work decomposition: each window is cut into tiles of STEP_THREADS
// consecutive cells (flat index (ix*ny + iy)*nz + iz), and a persistent grid
// (a multiple of the SM count) walks the global tile list.  One thread owns
// one cell of a tile: every population plane is read and written with
// consecutive addresses (the +-z pulls are off by one element and hit L1),
// so each population crosses HBM exactly once per step.
#include "collide.cuh"
#include "internal.cuh"
#include "step_common.cuh"

namespace psc {

// The exact FP64 variant is bound by its FP64 dependency chains: two CTAs per SM
// (at most 128 registers) hide their latency better than one.
template <int STORE, bool MOVING>
__global__ void __launch_bounds__(STEP_THREADS, STORE == PSC_STORE_F64_EXACT ? 2 : 1)
    k_step(const psc_window* __restrict__ wins, int nwin,
                                                        int64_t total_tiles, unsigned flags) {
    using TR = StoreTraits<STORE>;
    using T = typename TR::T;
    using R = typename TR::R;
    using O = typename TR::O;
    __shared__ int64_t s_begin[MAX_SMEM_WINDOWS];
    static_assert(STEP_THREADS / 32 == PSC_PARTIAL_ROWS, "one partial row per warp");
    const bool in_smem = nwin <= MAX_SMEM_WINDOWS;
    if (in_smem) {
        for (int i = threadIdx.x; i < nwin; i += blockDim.x) s_begin[i] = wins[i].tile_begin;
    }
    __syncthreads();
    const bool do_collide = flags & PSC_STEP_COLLIDE;
    const bool do_imb = do_collide && (flags & PSC_STEP_IMB);
    const bool do_mom = flags & PSC_STEP_MOMENTS;
    const bool do_red = flags & PSC_STEP_REDUCE;

    for (int64_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        const int wi = find_window(wins, in_smem ? s_begin : nullptr, nwin, t);
        const psc_window& W = wins[wi];
        if (W.flags & PSC_WIN_INACTIVE) continue;  // block-uniform
        const int nx = W.nx, ny = W.ny, nz = W.nz;
        const uint32_t N = (uint32_t)nx * (uint32_t)ny * (uint32_t)nz;
        const int64_t local_tile = t - W.tile_begin;
        const uint32_t cell = (uint32_t)(local_tile * W.tile_cells) + threadIdx.x;
        const bool valid = cell < N;
        double red[PSC_NRED];
#pragma unroll
        for (int k = 0; k < PSC_NRED; ++k) red[k] = 0.0;

        if (valid) {
            const uint32_t iz = cell % (uint32_t)nz;
            const uint32_t rr = cell / (uint32_t)nz;
            const uint32_t iy = rr % (uint32_t)ny;
            const uint32_t ix = rr / (uint32_t)ny;
            const bool open_x = (W.flags & PSC_WIN_OPEN_X) != 0;
            const NbrOffsets nb = nbr_offsets(ix, iy, iz, nx, ny, nz, open_x);
            const bool moving = MOVING && (W.flags & PSC_WIN_MOVING) && W.us != nullptr;
            R f[Q];
            const R scale = TR::scaled ? (R)W.store_scale : R(1);
            PullLoop<T, R, Q>::run(f, reinterpret_cast<const T*>(W.f_src), N, cell, nb, R(1) / scale, TR::scaled);
            if (open_x && ix == 0) {  // velocity inlet: bounce-back of the node's own opp(i) + momentum term
                const T* srcT = reinterpret_cast<const T*>(W.f_src);
#pragma unroll
                for (int i = 0; i < Q; ++i) {
                    if (!enters_x0(i)) continue;
                    const R back = ld_pop(srcT + (size_t)opp(i) * N + cell);
                    const double corr =
                        inlet_correction_exact(i, W.inlet_rho, W.inlet_u[0], W.inlet_u[1], W.inlet_u[2]);
                    if constexpr (TR::exact) f[i] = xadd((double)back, corr);
                    else f[i] = (TR::scaled ? back / scale : back) + (R)corr;
                }
            }
            O* mom = reinterpret_cast<O*>(W.moments);
            O* imbp = reinterpret_cast<O*>(W.imb);
            const O* usp = reinterpret_cast<const O*>(W.us);
            double rho_d, ux_d, uy_d, uz_d, solid_d;
            double imb_d[3] = {0.0, 0.0, 0.0};
            if constexpr (TR::exact) {
                const double hfx = xmul(0.5, W.force[0]), hfy = xmul(0.5, W.force[1]), hfz = xmul(0.5, W.force[2]);
                const ExactMoments mo = moments_exact(f, hfx, hfy, hfz);
                rho_d = mo.rho;
                ux_d = mo.ux;
                uy_d = mo.uy;
                uz_d = mo.uz;
                solid_d = W.solid[cell];
                if (do_collide) {
                    double usx = 0.0, usy = 0.0, usz = 0.0;
                    if (moving) {
                        usx = usp[cell];
                        usy = usp[(size_t)N + cell];
                        usz = usp[2 * (size_t)N + cell];
                    }
                    collide_exact(f, mo, solid_d, moving, usx, usy, usz, W.tau, W.force[0], W.force[1], W.force[2],
                                  hfx, hfy, hfz, imb_d);
                }
            } else {
                const FastMoments<R> mo = moments_fast(f);
                const R irho = R(1) / mo.rho;
                const R fx = (R)W.force[0], fy = (R)W.force[1], fz = (R)W.force[2];
                const R ux = (mo.mx + R(0.5) * fx) * irho;
                const R uy = (mo.my + R(0.5) * fy) * irho;
                const R uz = (mo.mz + R(0.5) * fz) * irho;
                rho_d = (double)mo.rho;
                ux_d = (double)ux;
                uy_d = (double)uy;
                uz_d = (double)uz;
                const int s = W.subsamples;
                const int s3 = s * s * s;
                // uint8 clipped sample level; without one (smooth geometry) the FP64 solid field
                const R al = W.level ? (R)W.level[cell] / (R)s3 : (R)W.solid[cell];
                solid_d = (double)al;
                if (do_collide) {
                    const R tau = (R)W.tau;
                    const R B = al / (al + tau * (R(1) - al) + R(1.0e-14));
                    FastParams<R> p;
                    p.inv_tau = R(1) / tau;
                    p.pref = R(1) - R(0.5) / tau;
                    p.fx = fx;
                    p.fy = fy;
                    p.fz = fz;
                    R usx = R(0), usy = R(0), usz = R(0);
                    if (moving) {
                        usx = (R)usp[cell];
                        usy = (R)usp[(size_t)N + cell];
                        usz = (R)usp[2 * (size_t)N + cell];
                    }
                    R im[3];
                    if (do_imb || do_red) {
                        if (moving) collide_fast<R, MOVING, true>(f, mo, irho, B, usx, usy, usz, p, im);
                        else collide_fast<R, false, true>(f, mo, irho, B, usx, usy, usz, p, im);
                        imb_d[0] = (double)im[0];
                        imb_d[1] = (double)im[1];
                        imb_d[2] = (double)im[2];
                    } else {
                        if (moving) collide_fast<R, MOVING, false>(f, mo, irho, B, usx, usy, usz, p, im);
                        else collide_fast<R, false, false>(f, mo, irho, B, usx, usy, usz, p, im);
                    }
                }
            }
            if (do_mom) {
                mom[cell] = (O)rho_d;
                mom[(size_t)N + cell] = (O)ux_d;
                mom[2 * (size_t)N + cell] = (O)uy_d;
                mom[3 * (size_t)N + cell] = (O)uz_d;
            }
            if (do_collide) {
                T* dst = reinterpret_cast<T*>(W.f_dst);
#pragma unroll
                for (int i = 0; i < Q; ++i) st_pop(dst + (size_t)i * N + cell, TR::scaled ? f[i] * scale : f[i]);
                if (do_imb) {
                    imbp[cell] = (O)imb_d[0];
                    imbp[(size_t)N + cell] = (O)imb_d[1];
                    imbp[2 * (size_t)N + cell] = (O)imb_d[2];
                }
            }
            if (do_red) {
                const double fl = 1.0 - solid_d;
                red[PSC_RED_RHO] = rho_d;
                red[PSC_RED_UX] = ux_d;
                red[PSC_RED_UY] = uy_d;
                red[PSC_RED_UZ] = uz_d;
                red[PSC_RED_FLUID_UX] = fl * ux_d;
                red[PSC_RED_FLUID_UY] = fl * uy_d;
                red[PSC_RED_FLUID_UZ] = fl * uz_d;
                red[PSC_RED_FLUID] = fl;
                red[PSC_RED_IMBX] = imb_d[0];
                red[PSC_RED_IMBY] = imb_d[1];
                red[PSC_RED_IMBZ] = imb_d[2];
                red[PSC_RED_NONFINITE] =
                    (isfinite(rho_d) && isfinite(ux_d) && isfinite(uy_d) && isfinite(uz_d)) ? 0.0 : 1.0;
                red[PSC_RED_SOLID] = solid_d;
            }
        }
        if (do_red) {  // one row per warp and tile; the block of local tile 0 writes the header
            warp_reduce_store<PSC_NRED>(red, W.partials + (1 + local_tile * PSC_PARTIAL_ROWS) * PSC_NRED);
            if (local_tile == 0 && threadIdx.x == 0) W.partials[0] = (double)(W.tile_count * PSC_PARTIAL_ROWS);
        }
    }
}

// Window sums of the partial rows (header row: element 0 = row count; the
// rows follow it), deterministic, in two launches:
//  1. k_reduce_segments: blockIdx.y = window; blocks stride over segments of
//     REDUCE_SEG consecutive rows; each segment is summed by a fixed tree and
//     its sum written over the segment's first row (the partials are consumed);
//  2. k_reduce_windows: one block per window sums the segment rows in order.
constexpr int REDUCE_SEG = STEP_THREADS;

// Row count from the header, clamped to the window's capacity.
__device__ __forceinline__ int64_t partial_rows(const psc_window& W) {
    const double h = W.partials[0];
    const int64_t cap = W.tile_count * PSC_PARTIAL_ROWS;
    if (!(h > 0.0)) return 0;
    const int64_t r = (int64_t)h;
    return r < cap ? r : cap;
}
constexpr int REDUCE_SEG_BLOCKS = 64;  // blocks per window in launch 1

__global__ void __launch_bounds__(STEP_THREADS) k_reduce_segments(const psc_window* __restrict__ wins) {
    __shared__ double s_red[STEP_THREADS / 32][PSC_NRED];
    __shared__ double s_out[PSC_NRED];
    const psc_window& W = wins[blockIdx.y];
    const int64_t rows = partial_rows(W);
    const int64_t nseg = (rows + REDUCE_SEG - 1) / REDUCE_SEG;
    double* body = W.partials + PSC_NRED;
    for (int64_t sg = blockIdx.x; sg < nseg; sg += gridDim.x) {  // block-uniform
        const int64_t r = sg * REDUCE_SEG + threadIdx.x;
        double v[PSC_NRED];
        if (r < rows) {
            const double* p = body + r * PSC_NRED;
#pragma unroll
            for (int k = 0; k < PSC_NRED; ++k) v[k] = p[k];
        } else {
#pragma unroll
            for (int k = 0; k < PSC_NRED; ++k) v[k] = 0.0;
        }
        block_reduce_store<PSC_NRED>(v, s_red, s_out);  // every read of the segment precedes its barrier
        if (threadIdx.x < PSC_NRED) body[sg * REDUCE_SEG * PSC_NRED + threadIdx.x] = s_out[threadIdx.x];
    }
}

__global__ void __launch_bounds__(STEP_THREADS) k_reduce_windows(const psc_window* __restrict__ wins,
                                                                 double* __restrict__ out) {
    __shared__ double s_red[STEP_THREADS / 32][PSC_NRED];
    const psc_window& W = wins[blockIdx.x];
    const int64_t rows = partial_rows(W);
    const int64_t nseg = (rows + REDUCE_SEG - 1) / REDUCE_SEG;
    double acc[PSC_NRED];
#pragma unroll
    for (int k = 0; k < PSC_NRED; ++k) acc[k] = 0.0;
    for (int64_t sg = threadIdx.x; sg < nseg; sg += blockDim.x) {
        const double* p = W.partials + PSC_NRED + sg * REDUCE_SEG * PSC_NRED;
#pragma unroll
        for (int k = 0; k < PSC_NRED; ++k) acc[k] += p[k];
    }
    block_reduce_store<PSC_NRED>(acc, s_red, out + (size_t)blockIdx.x * PSC_NRED);
}

template <int STORE>
__global__ void k_init_eq(void* f, int64_t ncells) {
    using T = typename StoreTraits<STORE>::T;
    T* p = reinterpret_cast<T*>(f);
    const int64_t total = ncells * Q;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / ncells);
        // equilibrium(rho=1, u=0) = w_i exactly (psc3d.py:136-140); deviation 0
        if constexpr (StoreTraits<STORE>::exact) st_pop(p + e, wgt(i));
        else st_pop(p + e, 0.0f);
    }
}

__device__ __forceinline__ double to_double(double v) { return v; }
__device__ __forceinline__ double to_double(float v) { return (double)v; }
__device__ __forceinline__ double to_double(__half v) { return (double)__half2float(v); }
__device__ __forceinline__ double to_double(__nv_bfloat16 v) { return (double)__bfloat162float(v); }

template <typename T>
__device__ __forceinline__ double to_abs(T v, int i, bool exact, bool scaled, double inv_scale) {
    double d = to_double(v);
    if (exact) return d;
    if (scaled) d *= inv_scale;
    return d + wgt(i);
}

// dst_i(x) = src_i(x - c_i) in absolute FP64 (the reference's post-stream f);
// with open_x the x faces follow PSC_WIN_OPEN_X (bounce-back velocity inlet
// at x = 0, zero-gradient outflow at x = nx - 1).
template <int STORE>
__global__ void k_stream_push(const void* src, double* dst, int nx, int ny, int nz, double scale, bool open_x,
                              double in_rho, double in_ux, double in_uy, double in_uz) {
    using TR = StoreTraits<STORE>;
    using T = typename TR::T;
    const uint32_t N = (uint32_t)nx * ny * nz;
    const T* s = reinterpret_cast<const T*>(src);
    for (uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x; cell < N; cell += gridDim.x * blockDim.x) {
        const uint32_t iz = cell % nz, rr = cell / nz, iy = rr % ny, ix = rr / ny;
        const NbrOffsets nb = nbr_offsets(ix, iy, iz, nx, ny, nz, open_x);
        int32_t off[Q];
        off[0] = 0;
        off[1] = pull_offset<1>(nb); off[2] = pull_offset<2>(nb); off[3] = pull_offset<3>(nb);
        off[4] = pull_offset<4>(nb); off[5] = pull_offset<5>(nb); off[6] = pull_offset<6>(nb);
        off[7] = pull_offset<7>(nb); off[8] = pull_offset<8>(nb); off[9] = pull_offset<9>(nb);
        off[10] = pull_offset<10>(nb); off[11] = pull_offset<11>(nb); off[12] = pull_offset<12>(nb);
        off[13] = pull_offset<13>(nb); off[14] = pull_offset<14>(nb); off[15] = pull_offset<15>(nb);
        off[16] = pull_offset<16>(nb); off[17] = pull_offset<17>(nb); off[18] = pull_offset<18>(nb);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const T v = s[(size_t)i * N + (size_t)((int64_t)cell + off[i])];
            double a = to_abs(v, i, TR::exact, TR::scaled, 1.0 / scale);
            if (open_x && ix == 0 && enters_x0(i)) {  // inlet: bounce-back of opp(i) at the node + momentum term
                const double back = to_abs(s[(size_t)opp(i) * N + cell], opp(i), TR::exact, TR::scaled, 1.0 / scale);
                a = xadd(back, inlet_correction_exact(i, in_rho, in_ux, in_uy, in_uz));
            }
            dst[(size_t)i * N + cell] = a;
        }
    }
}

// dst_i(y) = store(src_i(y + c_i)): inverse of k_stream_push.
template <int STORE>
__global__ void k_stream_pull_store(const double* src, void* dst, int nx, int ny, int nz, double scale) {
    using TR = StoreTraits<STORE>;
    using T = typename TR::T;
    const uint32_t N = (uint32_t)nx * ny * nz;
    T* d = reinterpret_cast<T*>(dst);
    for (uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x; cell < N; cell += gridDim.x * blockDim.x) {
        const uint32_t iz = cell % nz, rr = cell / nz, iy = rr % ny, ix = rr / ny;
        const NbrOffsets nb = nbr_offsets(ix, iy, iz, nx, ny, nz);
        // y + c_i is the pull source of direction opp(i)
        int32_t off[Q];
        off[0] = 0;
        off[1] = pull_offset<2>(nb); off[2] = pull_offset<1>(nb); off[3] = pull_offset<4>(nb);
        off[4] = pull_offset<3>(nb); off[5] = pull_offset<6>(nb); off[6] = pull_offset<5>(nb);
        off[7] = pull_offset<8>(nb); off[8] = pull_offset<7>(nb); off[9] = pull_offset<10>(nb);
        off[10] = pull_offset<9>(nb); off[11] = pull_offset<12>(nb); off[12] = pull_offset<11>(nb);
        off[13] = pull_offset<14>(nb); off[14] = pull_offset<13>(nb); off[15] = pull_offset<16>(nb);
        off[16] = pull_offset<15>(nb); off[17] = pull_offset<18>(nb); off[18] = pull_offset<17>(nb);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            double v = src[(size_t)i * N + (size_t)((int64_t)cell + off[i])];
            if (!TR::exact) {
                v -= wgt(i);
                if (TR::scaled) v *= scale;
            }
            if constexpr (sizeof(T) == 8) d[(size_t)i * N + cell] = (T)v;
            else if constexpr (sizeof(T) == 4) d[(size_t)i * N + cell] = (T)v;
            else st_pop(d + (size_t)i * N + cell, (float)v);
        }
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <int STORE, bool MOVING>
static cudaError_t launch_step_t(const psc_window* d_windows, int nwin, int64_t total_tiles, unsigned flags,
                                 int grid_ctas, cudaStream_t stream) {
    if (grid_ctas <= 0) {
        static int per_sm[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int dev = 0;
        cudaGetDevice(&dev);
        int& occ = per_sm[dev & 7];
        if (occ == 0) {
            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_step<STORE, MOVING>, STEP_THREADS, 0);
            if (e != cudaSuccess) return e;
            if (occ <= 0) occ = 1;
        }
        const int64_t g = (int64_t)sm_count() * occ;
        grid_ctas = (int)(total_tiles < g ? total_tiles : g);
    }
    if ((int64_t)grid_ctas > total_tiles) grid_ctas = (int)total_tiles;
    if (grid_ctas <= 0) return cudaSuccess;
    k_step<STORE, MOVING><<<grid_ctas, STEP_THREADS, 0, stream>>>(d_windows, nwin, total_tiles, flags);
    return cudaGetLastError();
}

cudaError_t launch_step(int store, const psc_window* d_windows, int nwin, int64_t total_tiles, unsigned flags,
                        bool moving, int grid_ctas, cudaStream_t stream) {
#define PSC_STEP_CASE(S)                                                                                          \
    case S:                                                                                                       \
        return moving ? launch_step_t<S, true>(d_windows, nwin, total_tiles, flags, grid_ctas, stream)           \
                      : launch_step_t<S, false>(d_windows, nwin, total_tiles, flags, grid_ctas, stream);
    switch (store) {
        PSC_STEP_CASE(PSC_STORE_F64_EXACT)
        PSC_STEP_CASE(PSC_STORE_F64)
        PSC_STEP_CASE(PSC_STORE_F32)
        PSC_STEP_CASE(PSC_STORE_F16)
        PSC_STEP_CASE(PSC_STORE_BF16)
        default:
            return cudaErrorInvalidValue;
    }
#undef PSC_STEP_CASE
}

cudaError_t launch_reduce_windows(const psc_window* d_windows, int nwin, double* out, cudaStream_t stream) {
    k_reduce_segments<<<dim3(REDUCE_SEG_BLOCKS, (unsigned)nwin), STEP_THREADS, 0, stream>>>(d_windows);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_reduce_windows<<<nwin, STEP_THREADS, 0, stream>>>(d_windows, out);
    return cudaGetLastError();
}

static int grid_for(int64_t work, int threads) {
    int64_t g = (work + threads - 1) / threads;
    const int64_t cap = (int64_t)sm_count() * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

cudaError_t launch_init_equilibrium(int store, double scale, void* f, int64_t ncells, cudaStream_t stream) {
    (void)scale;
    const int g = grid_for(ncells * Q, 256);
    switch (store) {
        case PSC_STORE_F64_EXACT: k_init_eq<PSC_STORE_F64_EXACT><<<g, 256, 0, stream>>>(f, ncells); break;
        case PSC_STORE_F64: k_init_eq<PSC_STORE_F64><<<g, 256, 0, stream>>>(f, ncells); break;
        case PSC_STORE_F32: k_init_eq<PSC_STORE_F32><<<g, 256, 0, stream>>>(f, ncells); break;
        case PSC_STORE_F16: k_init_eq<PSC_STORE_F16><<<g, 256, 0, stream>>>(f, ncells); break;
        case PSC_STORE_BF16: k_init_eq<PSC_STORE_BF16><<<g, 256, 0, stream>>>(f, ncells); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_stream_push(int store, double scale, const void* src, double* dst, int nx, int ny, int nz,
                               cudaStream_t stream, bool open_x, const double* inlet) {
    const int g = grid_for((int64_t)nx * ny * nz, 256);
    const double r = open_x ? inlet[0] : 1.0, ux = open_x ? inlet[1] : 0.0, uy = open_x ? inlet[2] : 0.0,
                 uz = open_x ? inlet[3] : 0.0;
#define PSC_PUSH_CASE(S) \
    case S: k_stream_push<S><<<g, 256, 0, stream>>>(src, dst, nx, ny, nz, scale, open_x, r, ux, uy, uz); break;
    switch (store) {
        PSC_PUSH_CASE(PSC_STORE_F64_EXACT)
        PSC_PUSH_CASE(PSC_STORE_F64)
        PSC_PUSH_CASE(PSC_STORE_F32)
        PSC_PUSH_CASE(PSC_STORE_F16)
        PSC_PUSH_CASE(PSC_STORE_BF16)
        default: return cudaErrorInvalidValue;
    }
#undef PSC_PUSH_CASE
    return cudaGetLastError();
}

// Open-x inverse at the inlet plane: the populations that only the inlet's
// bounce-back reads (c_x = -1 at x = 0) are set so that the pulled value of
// the entering direction i = opp(j) is f_i(0): stored_j = f_i - term_i (to
// rounding in the exact mode).
template <int STORE>
__global__ void k_open_x_unpull(const double* src, void* dst, int nx, int ny, int nz, double scale, double in_rho,
                                double in_ux, double in_uy, double in_uz) {
    using TR = StoreTraits<STORE>;
    using T = typename TR::T;
    const uint32_t N = (uint32_t)nx * ny * nz;
    const uint32_t plane = (uint32_t)ny * nz;  // the cells of x = 0
    T* d = reinterpret_cast<T*>(dst);
    for (uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x; cell < plane; cell += gridDim.x * blockDim.x) {
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            if (!enters_x0(i)) continue;
            const int j = opp(i);
            double v = xsub(src[(size_t)i * N + cell], inlet_correction_exact(i, in_rho, in_ux, in_uy, in_uz));
            if (!TR::exact) {
                v -= wgt(j);
                if (TR::scaled) v *= scale;
            }
            if constexpr (sizeof(T) == 8) d[(size_t)j * N + cell] = (T)v;
            else if constexpr (sizeof(T) == 4) d[(size_t)j * N + cell] = (T)v;
            else st_pop(d + (size_t)j * N + cell, (float)v);
        }
    }
}

cudaError_t launch_stream_pull_store(int store, double scale, const double* src, void* dst, int nx, int ny, int nz,
                                     cudaStream_t stream, bool open_x, const double* inlet) {
    const int g = grid_for((int64_t)nx * ny * nz, 256);
    switch (store) {
        case PSC_STORE_F64_EXACT: k_stream_pull_store<PSC_STORE_F64_EXACT><<<g, 256, 0, stream>>>(src, dst, nx, ny, nz, scale); break;
        case PSC_STORE_F64: k_stream_pull_store<PSC_STORE_F64><<<g, 256, 0, stream>>>(src, dst, nx, ny, nz, scale); break;
        case PSC_STORE_F32: k_stream_pull_store<PSC_STORE_F32><<<g, 256, 0, stream>>>(src, dst, nx, ny, nz, scale); break;
        case PSC_STORE_F16: k_stream_pull_store<PSC_STORE_F16><<<g, 256, 0, stream>>>(src, dst, nx, ny, nz, scale); break;
        case PSC_STORE_BF16: k_stream_pull_store<PSC_STORE_BF16><<<g, 256, 0, stream>>>(src, dst, nx, ny, nz, scale); break;
        default: return cudaErrorInvalidValue;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !open_x) return e;
    const int gp = grid_for((int64_t)ny * nz, 256);
    const double r = inlet[0], ux = inlet[1], uy = inlet[2], uz = inlet[3];
#define PSC_UNPULL_CASE(S) \
    case S: k_open_x_unpull<S><<<gp, 256, 0, stream>>>(src, dst, nx, ny, nz, scale, r, ux, uy, uz); break;
    switch (store) {
        PSC_UNPULL_CASE(PSC_STORE_F64_EXACT)
        PSC_UNPULL_CASE(PSC_STORE_F64)
        PSC_UNPULL_CASE(PSC_STORE_F32)
        PSC_UNPULL_CASE(PSC_STORE_F16)
        PSC_UNPULL_CASE(PSC_STORE_BF16)
        default: return cudaErrorInvalidValue;
    }
#undef PSC_UNPULL_CASE
    return cudaGetLastError();
}

}  // namespace psc
