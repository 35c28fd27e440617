// TMA-staged throughput kernel for the deviation storage modes.
//
// Same step as k_step_fast (src/lbm_dem/psc3d.py:208-246); what changes is how
// the 19 pulled populations reach the SM.  A tile is TY whole z-rows of one
// x-plane (cells ((ix*ny + y0 .. y0+TY-1)*nz + 0 .. nz-1)).  For population
// i the pull sources of that tile are TY consecutive rows of plane i at
// x - c_ix, y - c_iy: one contiguous run of TY*nz elements (two when the
// y-range wraps), so a producer warp fetches each with one cp.async.bulk
// (the TMA engine) into a shared-memory stage and signals an mbarrier.
// Consumer warps read the stage with the z-shift (and the z wrap) applied
// in shared memory, collide and store coalesced.  STAGES stages are kept in
// flight per CTA, so the SM has tens of kB of HBM reads outstanding without
// spending registers or issue slots on global loads.
//
// The tile's uint8 solid level (or FP64 smooth solid fraction) rides in the
// same stage, so the consumers touch global memory only to store.
//
// Every mbarrier wait is bounded: after PSC_WAIT_LIMIT polls the kernel
// records an error in psc_device_status (read with psc_device_status()),
// stops issuing work, waits (bounded) for its own copies in flight and returns.
#include "step_common.cuh"

namespace psc {

__device__ int g_psc_status = 0;

constexpr int TMA_CONSUMERS = 256;
constexpr int TMA_THREADS = TMA_CONSUMERS + 32;  // + one producer warp
constexpr long long PSC_WAIT_LIMIT = 1ll << 26;   // polls before a wait is declared stuck

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait; false (and a recorded error) when the limit is hit.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int code) {
    for (long long it = 0; it < PSC_WAIT_LIMIT; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
    }
    atomicCAS(&g_psc_status, 0, code);
    return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(TMA_CONSUMERS) : "memory"); }

template <typename T, typename R, typename O>
struct TmaWin {
    const T* src;
    T* dst;
    const uint8_t* level;
    const double* solid;
    const O* us;
    O* imb;
    O* mom;
    double* partials;
    int64_t tile_begin, tile_end;
    uint32_t nx, ny, nz, N, ty, nyb;
    int32_t moving;
    int32_t inactive;
    int32_t trt;
    R scale, inv_scale, tau;
    WinConst<R> c;
    R Blut[256];
    R kblut[256];
    R alut[256];
};

// tile t of window W -> (ix, y0, rows)
__device__ __forceinline__ void row_tile(const psc_window& W, int64_t t, uint32_t& ix, uint32_t& y0,
                                         uint32_t& rows) {
    const uint32_t ty = (uint32_t)(W.tile_cells / W.nz);
    const uint32_t nyb = ((uint32_t)W.ny + ty - 1) / ty;
    const uint32_t local = (uint32_t)(t - W.tile_begin);
    ix = local / nyb;
    y0 = (local - ix * nyb) * ty;
    rows = min(ty, (uint32_t)W.ny - y0);
}

template <int STORE, bool MOVING, int STAGES, bool RED>
__global__ void __launch_bounds__(TMA_THREADS, 2) k_step_tma(const psc_window* __restrict__ wins, int nwin,
                                                           int64_t total_tiles, unsigned flags, uint32_t stage_bytes) {
    using TR = StoreTraits<STORE>;
    using T = typename TR::T;
    using R = typename TR::R;
    using O = typename TR::O;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t full[STAGES], empty[STAGES];
    __shared__ TmaWin<T, R, O> sw;
    static_assert(TMA_CONSUMERS / 32 == PSC_PARTIAL_ROWS, "one partial row per consumer warp");
    __shared__ int s_abort;

    const int64_t t0 = (total_tiles * (int64_t)blockIdx.x) / gridDim.x;
    const int64_t t1 = (total_tiles * ((int64_t)blockIdx.x + 1)) / gridDim.x;
    const bool producer = threadIdx.x >= TMA_CONSUMERS;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], TMA_CONSUMERS / 32);
        }
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (producer) {
        // The whole producer warp works each tile: lane 0 arms the stage's
        // mbarrier with the byte count, then lane i < 19 issues the bulk copy
        // (or two, across a y wrap) of population i and lane 19 the tile's
        // solid level, so no lane does more than a few address computations.
        const int lane = threadIdx.x - TMA_CONSUMERS;
        int64_t win_end = -1;
        int wi = 0;
        uint32_t issued = 0;
        bool stop = false;
        for (int64_t t = t0; t < t1; ++t) {
            if (t >= win_end) {
                wi = find_window(wins, nullptr, nwin, t);
                win_end = wins[wi].tile_begin + wins[wi].tile_count;
            }
            if (wins[wi].flags & PSC_WIN_INACTIVE) continue;  // the consumers skip the same tiles
            const int s = (int)(issued % STAGES);
            if (issued >= (uint32_t)STAGES) {
                int ok = 1;
                if (lane == 0) ok = mbar_wait(&empty[s], ((issued / STAGES) - 1) & 1, 0x101) && !s_abort;
                ok = __shfl_sync(0xffffffffu, ok, 0);
                if (!ok) {
                    if (lane == 0) s_abort = 1;
                    stop = true;
                    break;
                }
            }
            const psc_window& W = wins[wi];
            uint32_t ix, y0, rows;
            row_tile(W, t, ix, y0, rows);
            const uint32_t nx = W.nx, ny = W.ny, nz = W.nz;
            const uint32_t row_bytes = nz * (uint32_t)sizeof(T);
            const uint32_t pop_bytes = (uint32_t)(W.tile_cells) * (uint32_t)sizeof(T);  // ty * nz * sizeof(T)
            unsigned char* stage = smem + (size_t)s * stage_bytes;
            if (lane == 0) mbar_expect_tx(&full[s], 19u * rows * row_bytes + rows * nz * (W.level ? 1u : 8u));
            __syncwarp();
            if (lane < Q) {
                const int i = lane;
                const int cx = cxv_rt(i), cy = cyv_rt(i);
                const uint32_t xs = cx == 1 ? (ix == 0 ? nx - 1 : ix - 1) : (cx == -1 ? (ix + 1 == nx ? 0 : ix + 1) : ix);
                int ys = (int)y0 - cy;
                unsigned char* dst = stage + (size_t)i * pop_bytes;
                const T* plane = reinterpret_cast<const T*>(W.f_src) + (size_t)i * ((size_t)nx * ny * nz) +
                                 (size_t)xs * ny * nz;
                uint32_t r0 = 0;
                if (ys < 0) {  // first row wraps to ny - 1
                    bulk_g2s(dst, plane + (size_t)(ny - 1) * nz, row_bytes, &full[s]);
                    r0 = 1;
                    ys = 0;
                }
                uint32_t n_in = rows - r0;
                if ((uint32_t)ys + n_in > ny) n_in = ny - (uint32_t)ys;  // rows before the top wrap
                if (n_in) bulk_g2s(dst + (size_t)r0 * row_bytes, plane + (size_t)ys * nz, n_in * row_bytes, &full[s]);
                const uint32_t rest = rows - r0 - n_in;  // rows wrapping to y = 0
                if (rest) bulk_g2s(dst + (size_t)(r0 + n_in) * row_bytes, plane, rest * row_bytes, &full[s]);
            } else if (lane == Q) {
                // the tile's own solid level (uint8) or smooth solid fraction (double), no shift
                const size_t base = ((size_t)ix * ny + y0) * nz;
                unsigned char* gdst = stage + (size_t)19 * pop_bytes;
                if (W.level) bulk_g2s(gdst, W.level + base, rows * nz, &full[s]);
                else bulk_g2s(gdst, W.solid + base, rows * nz * 8u, &full[s]);
            }
            ++issued;
        }
        (void)stop;
        // drain: wait (bounded) for every issued stage to land before the CTA may exit
        if (lane == 0) {
            const uint32_t n_issued = issued;
            for (uint32_t k = (n_issued > (uint32_t)STAGES ? n_issued - STAGES : 0); k < n_issued; ++k)
                mbar_wait(&full[k % STAGES], (k / STAGES) & 1, 0x102);
        }
        return;
    }

    // ---------------- consumers ----------------
    const bool do_collide = flags & PSC_STEP_COLLIDE;
    const bool do_imb = do_collide && (flags & PSC_STEP_IMB);
    const bool do_mom = flags & PSC_STEP_MOMENTS;
    constexpr bool do_red = RED;
    int64_t win_end = -1;
    uint32_t k = 0;
    bool aborted = false;  // after a stuck wait: keep joining the barriers, skip the work
    double red[PSC_NRED];  // this thread's sums over the CTA's cells of the current window
#pragma unroll
    for (int q = 0; q < PSC_NRED; ++q) red[q] = 0.0;
    bool have = false;
    for (int64_t t = t0; t < t1; ++t) {
        if (t >= win_end) {
            if (do_red && have)
                flush_segment<PSC_NRED>(red, sw.partials, sw.tile_begin, sw.tile_end - sw.tile_begin, total_tiles,
                                        gridDim.x);
            have = false;
            consumer_sync();
            if (threadIdx.x == 0) {
                const int wi = find_window(wins, nullptr, nwin, t);
                const psc_window& W = wins[wi];
                sw.src = reinterpret_cast<const T*>(W.f_src);
                sw.dst = reinterpret_cast<T*>(W.f_dst);
                sw.level = W.level;
                sw.solid = W.solid;
                sw.us = reinterpret_cast<const O*>(W.us);
                sw.imb = reinterpret_cast<O*>(W.imb);
                sw.mom = reinterpret_cast<O*>(W.moments);
                sw.partials = W.partials;
                sw.tile_begin = W.tile_begin;
                sw.tile_end = W.tile_begin + W.tile_count;
                sw.nx = W.nx;
                sw.ny = W.ny;
                sw.nz = W.nz;
                sw.N = (uint32_t)W.nx * W.ny * W.nz;
                sw.ty = (uint32_t)(W.tile_cells / W.nz);
                sw.nyb = ((uint32_t)W.ny + sw.ty - 1) / sw.ty;
                sw.moving = (MOVING && (W.flags & PSC_WIN_MOVING) && W.us != nullptr) ? 1 : 0;
                sw.inactive = (W.flags & PSC_WIN_INACTIVE) ? 1 : 0;
                sw.scale = (R)W.store_scale;
                sw.inv_scale = (R)(1.0 / W.store_scale);
                sw.tau = (R)W.tau;
                make_win_const(sw.c, W.tau, W.force[0], W.force[1], W.force[2], W.tau_minus);
                sw.trt = W.tau_minus > 0.0 ? 1 : 0;
            }
            consumer_sync();
            {
                const psc_window& W = wins[find_window(wins, nullptr, nwin, t)];
                const int S3 = W.subsamples * W.subsamples * W.subsamples;
                if (W.level) {
                    for (int l = threadIdx.x; l <= S3 && l < 256; l += TMA_CONSUMERS) {
                        const double al = (double)l / (double)S3;
                        const double B = al / (al + W.tau * (1.0 - al) + 1.0e-14);
                        sw.Blut[l] = (R)B;
                        sw.kblut[l] = (R)((1.0 - B) / W.tau);
                        sw.alut[l] = (R)al;
                    }
                }
            }
            consumer_sync();
            win_end = sw.tile_end;
        }
        if (sw.inactive) continue;  // uniform over consumers; the producer issued nothing for it
        have = true;
        const int s = (int)(k % STAGES);
        if (!aborted && !mbar_wait(&full[s], (k / STAGES) & 1, 0x103)) {
            aborted = true;
            s_abort = 1;
        }
        const uint32_t N = sw.N, nz = sw.nz, ny = sw.ny;
        const uint32_t local = (uint32_t)(t - sw.tile_begin);
        const uint32_t ix = local / sw.nyb;
        const uint32_t y0 = (local - ix * sw.nyb) * sw.ty;
        const uint32_t rows = min(sw.ty, ny - y0);
        const uint32_t ncell = rows * nz;
        const uint32_t pop_elems = sw.ty * nz;
        const T* st = reinterpret_cast<const T*>(smem + (size_t)s * stage_bytes);
        const unsigned char* st_geo = smem + (size_t)s * stage_bytes + (size_t)19 * pop_elems * sizeof(T);
        const uint32_t base = (ix * ny + y0) * nz;
        const uint32_t dyy = TMA_CONSUMERS / nz, dz = TMA_CONSUMERS - dyy * nz;
        uint32_t yy = threadIdx.x / nz, iz = threadIdx.x - yy * nz;
        for (uint32_t c = threadIdx.x; c < (aborted ? 0u : ncell); c += TMA_CONSUMERS) {
            if (c != threadIdx.x) {  // carry-add (yy, iz) by TMA_CONSUMERS cells
                iz += dz;
                const uint32_t cz = iz >= nz;
                iz -= cz ? nz : 0;
                yy += dyy + cz;
            }
            const uint32_t zrow = yy * nz;
            const uint32_t zm = iz == 0 ? nz - 1 : iz - 1;  // z - 1 (pull for c_z = +1)
            const uint32_t zp = iz == nz - 1 ? 0 : iz + 1;  // z + 1 (pull for c_z = -1)
            R g[Q];
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                const uint32_t zz = czv(i) == 1 ? zm : (czv(i) == -1 ? zp : iz);
                const R v = ld_smem_pop(st + (size_t)i * pop_elems + zrow + zz);
                g[i] = TR::scaled ? v * sw.inv_scale : v;
            }
            const uint32_t cell = base + c;
            R B, kb, al;
            if (sw.level) {
                const uint8_t lv = st_geo[c];
                B = sw.Blut[lv];
                kb = sw.kblut[lv];
                al = sw.alut[lv];
            } else {
                al = (R)reinterpret_cast<const double*>(st_geo)[c];
                B = al * fast_rcp<R>(al + sw.tau * (R(1) - al) + R(1.0e-14));
                kb = (R(1) - B) * sw.c.inv_tau;
            }
            R usx = R(0), usy = R(0), usz = R(0);
            const bool moving = MOVING && sw.moving;
            if (moving) {
                usx = (R)sw.us[cell];
                usy = (R)sw.us[(size_t)N + cell];
                usz = (R)sw.us[2 * (size_t)N + cell];
            }
            R mom[4], imb[3] = {R(0), R(0), R(0)};
            if (do_collide) {
                if (sw.trt) {
                    if (moving) collide_fast2<R, MOVING, true, true>(g, sw.c, B, kb, usx, usy, usz, R(0), mom, imb);
                    else collide_fast2<R, false, true, true>(g, sw.c, B, kb, usx, usy, usz, R(0), mom, imb);
                } else if (do_imb || do_red) {
                    if (moving) collide_fast2<R, MOVING, true>(g, sw.c, B, kb, usx, usy, usz, R(0), mom, imb);
                    else collide_fast2<R, false, true>(g, sw.c, B, kb, usx, usy, usz, R(0), mom, imb);
                } else {
                    if (moving) collide_fast2<R, MOVING, false>(g, sw.c, B, kb, usx, usy, usz, R(0), mom, imb);
                    else collide_fast2<R, false, false>(g, sw.c, B, kb, usx, usy, usz, R(0), mom, imb);
                }
                T* dst = sw.dst + cell;
                uint32_t plane = 0;
#pragma unroll
                for (int i = 0; i < Q; ++i) {
                    st_pop(dst + plane, TR::scaled ? g[i] * sw.scale : g[i]);
                    plane += N;
                }
                if (do_imb) {
                    sw.imb[cell] = (O)imb[0];
                    sw.imb[(size_t)N + cell] = (O)imb[1];
                    sw.imb[2 * (size_t)N + cell] = (O)imb[2];
                }
            } else {
                const FastMoments<R> mo = moments_fast(g);
                const R irho = R(1) / mo.rho;
                mom[0] = mo.drho;
                mom[1] = (mo.mx + R(0.5) * sw.c.fx) * irho;
                mom[2] = (mo.my + R(0.5) * sw.c.fy) * irho;
                mom[3] = (mo.mz + R(0.5) * sw.c.fz) * irho;
            }
            if (do_mom) {
                sw.mom[cell] = (O)(R(1) + mom[0]);
                sw.mom[(size_t)N + cell] = (O)mom[1];
                sw.mom[2 * (size_t)N + cell] = (O)mom[2];
                sw.mom[3 * (size_t)N + cell] = (O)mom[3];
            }
            if (do_red) {
                const double solid = (double)al, fl = 1.0 - solid;
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
        // this warp is done reading stage s
        __syncwarp();
        if ((threadIdx.x & 31) == 0) mbar_arrive(&empty[s]);
        ++k;
    }
    if (do_red && have)
        flush_segment<PSC_NRED>(red, sw.partials, sw.tile_begin, sw.tile_end - sw.tile_begin, total_tiles, gridDim.x);
}

template <int STORE, bool MOVING, int STAGES, bool RED>
static cudaError_t launch_tma_t(const psc_window* d, int nwin, int64_t tiles, unsigned flags, int grid,
                                uint32_t stage_bytes, cudaStream_t s) {
    const size_t smem = (size_t)STAGES * stage_bytes;
    auto kern = k_step_tma<STORE, MOVING, STAGES, RED>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (grid <= 0) {
        int occ = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, TMA_THREADS, smem);
        if (e != cudaSuccess) return e;
        if (occ <= 0) return cudaErrorInvalidConfiguration;
        const int64_t g = (int64_t)sm_count() * occ;
        grid = (int)(tiles < g ? tiles : g);
    }
    if ((int64_t)grid > tiles) grid = (int)tiles;  // every CTA owns >= 1 tile
    if (grid <= 0) return cudaSuccess;
    kern<<<grid, TMA_THREADS, smem, s>>>(d, nwin, tiles, flags, stage_bytes);
    return cudaGetLastError();
}

template <int STORE, bool MOVING, bool RED>
static cudaError_t launch_tma_r(const psc_window* d, int nwin, int64_t tiles, unsigned flags, int grid, int stages,
                                uint32_t stage_bytes, cudaStream_t s) {
    switch (stages) {
        case 2: return launch_tma_t<STORE, MOVING, 2, RED>(d, nwin, tiles, flags, grid, stage_bytes, s);
        case 3: return launch_tma_t<STORE, MOVING, 3, RED>(d, nwin, tiles, flags, grid, stage_bytes, s);
        case 4: return launch_tma_t<STORE, MOVING, 4, RED>(d, nwin, tiles, flags, grid, stage_bytes, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int STORE, bool MOVING>
static cudaError_t launch_tma_m(const psc_window* d, int nwin, int64_t tiles, unsigned flags, int grid, int stages,
                                uint32_t stage_bytes, cudaStream_t s) {
    return (flags & PSC_STEP_REDUCE) ? launch_tma_r<STORE, MOVING, true>(d, nwin, tiles, flags, grid, stages, stage_bytes, s)
                                     : launch_tma_r<STORE, MOVING, false>(d, nwin, tiles, flags, grid, stages, stage_bytes, s);
}

template <int STORE>
static cudaError_t launch_tma_s(const psc_window* d, int nwin, int64_t tiles, unsigned flags, bool moving, int grid,
                                int stages, uint32_t stage_bytes, cudaStream_t s) {
    return moving ? launch_tma_m<STORE, true>(d, nwin, tiles, flags, grid, stages, stage_bytes, s)
                  : launch_tma_m<STORE, false>(d, nwin, tiles, flags, grid, stages, stage_bytes, s);
}

cudaError_t launch_step_tma(int store, const psc_window* d_windows, int nwin, int64_t total_tiles, unsigned flags,
                            bool moving, int grid_ctas, int stages, uint32_t stage_bytes, cudaStream_t stream) {
    switch (store) {
        case PSC_STORE_F64: return launch_tma_s<PSC_STORE_F64>(d_windows, nwin, total_tiles, flags, moving, grid_ctas, stages, stage_bytes, stream);
        case PSC_STORE_F32: return launch_tma_s<PSC_STORE_F32>(d_windows, nwin, total_tiles, flags, moving, grid_ctas, stages, stage_bytes, stream);
        case PSC_STORE_F16: return launch_tma_s<PSC_STORE_F16>(d_windows, nwin, total_tiles, flags, moving, grid_ctas, stages, stage_bytes, stream);
        case PSC_STORE_BF16: return launch_tma_s<PSC_STORE_BF16>(d_windows, nwin, total_tiles, flags, moving, grid_ctas, stages, stage_bytes, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t read_device_status(int* out, bool clear) {
    cudaError_t e = cudaMemcpyFromSymbol(out, g_psc_status, sizeof(int));
    if (e != cudaSuccess || !clear) return e;
    const int zero = 0;
    return cudaMemcpyToSymbol(g_psc_status, &zero, sizeof(int));
}

}  // namespace psc
