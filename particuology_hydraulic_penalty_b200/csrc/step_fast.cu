// Throughput kernel for the deviation storage modes (F64 / F32 / F16 / BF16).
//
// Same step as k_step (pull-stream + PSC-IMB collide, src/lbm_dem/psc3d.py:
// 208-246), organised to keep the SM's issue slots for the collision:
//  * each persistent CTA owns a CONTIGUOUS run of tiles, so it meets a new
//    window only a few times; per-window constants (Guo terms, 1/tau, the
//    solid-level -> B and (1-B)/tau tables, mixed-radix tile stride) are built
//    once in shared memory when the window changes;
//  * a tile is CPT x 256 consecutive cells; a thread owns CPT of them,
//    issues all 19 x CPT pulls before computing, and advances its (ix, iy, iz)
//    between cells by a carry-add instead of integer division;
//  * 32-bit population offsets, reciprocal instead of division.
#include "fast_cell.cuh"

namespace psc {

// Resident CTAs the register allocation aims for: four (64 registers) for
// FP32/FP16/BF16 storage, three with moving particles (the solid-velocity
// terms), two for FP64, whose arithmetic needs about twice the registers, and
// two with reductions (13 FP64 accumulators per thread).  An explicit target
// matters: ptxas allocates differently without one.
template <int STORE, bool MOVING, bool RED>
struct StepOccupancy {
    static constexpr int value = (STORE == PSC_STORE_F64 || RED) ? 2 : (MOVING ? 3 : 4);
};

template <int STORE, bool MOVING, int CPT, bool RED>
__global__ void __launch_bounds__(STEP_THREADS, (StepOccupancy<STORE, MOVING, RED>::value)) k_step_fast(const psc_window* __restrict__ wins, int nwin,
                                                             int64_t total_tiles, unsigned flags) {
    using TR = StoreTraits<STORE>;
    using T = typename TR::T;
    using R = typename TR::R;
    using O = typename TR::O;
    __shared__ FastWin<T, R, O> sw;
    static_assert(STEP_THREADS / 32 == PSC_PARTIAL_ROWS, "one partial row per warp");
    const bool do_collide = flags & PSC_STEP_COLLIDE;
    const bool do_imb = do_collide && (flags & PSC_STEP_IMB);
    const bool do_mom = flags & PSC_STEP_MOMENTS;
    constexpr bool do_red = RED;
    const int64_t t0 = (total_tiles * (int64_t)blockIdx.x) / gridDim.x;
    const int64_t t1 = (total_tiles * ((int64_t)blockIdx.x + 1)) / gridDim.x;
    int64_t win_end = -1;
    double red[PSC_NRED];  // this thread's sums over the CTA's cells of the current window
#pragma unroll
    for (int q = 0; q < PSC_NRED; ++q) red[q] = 0.0;
    bool have = false;  // block-uniform: red holds cells of the window in sw
    for (int64_t t = t0; t < t1; ++t) {
        if (t >= win_end) {  // block-uniform: entering a new window
            if (do_red && have)
                flush_segment<PSC_NRED>(red, sw.partials, sw.tile_begin, sw.tile_end - sw.tile_begin, total_tiles,
                                        gridDim.x);
            have = false;
            __syncthreads();
            const int wi = find_window(wins, nullptr, nwin, t);
            load_fast_win(sw, wins[wi], MOVING);
            __syncthreads();
            win_end = sw.tile_end;
        }
        if (sw.inactive) continue;  // block-uniform
        have = true;
        const uint32_t N = sw.N, nx = sw.nx, ny = sw.ny, nz = sw.nz;
        const uint32_t base = (uint32_t)((t - sw.tile_begin) * sw.tile_cells);
        uint32_t cell = base + threadIdx.x;
        uint32_t iz = cell % nz, rr = cell / nz, iy = rr % ny, ix = rr / ny;
        const T* src = sw.src;
        R f[CPT][Q];
        uint32_t cells[CPT];
        bool inlet[CPT];
        const bool open_x = sw.open_x;
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            cells[k] = cell;
            inlet[k] = open_x && ix == 0;
            if (cell < N) {
                const int32_t nyz = (int32_t)(ny * nz);
                // open x: the x faces read the cell's own plane (zero-gradient outflow)
                const int32_t xm = ix == 0 ? (open_x ? 0 : (int32_t)(nx - 1) * nyz) : -nyz;
                const int32_t xp = ix == nx - 1 ? (open_x ? 0 : -(int32_t)(nx - 1) * nyz) : nyz;
                const int32_t ym = iy == 0 ? (int32_t)(ny - 1) * (int32_t)nz : -(int32_t)nz;
                const int32_t yp = iy == ny - 1 ? -(int32_t)(ny - 1) * (int32_t)nz : (int32_t)nz;
                const int32_t zm = iz == 0 ? (int32_t)nz - 1 : -1;
                const int32_t zp = iz == nz - 1 ? -(int32_t)(nz - 1) : 1;
                const T* sc = src + cell;
                uint32_t plane = 0;
#pragma unroll
                for (int i = 0; i < Q; ++i) {
                    const int32_t o = (cxv(i) == 1 ? xm : (cxv(i) == -1 ? xp : 0)) +
                                      (cyv(i) == 1 ? ym : (cyv(i) == -1 ? yp : 0)) +
                                      (czv(i) == 1 ? zm : (czv(i) == -1 ? zp : 0));
                    f[k][i] = ld_pop(sc + (int64_t)(int32_t)(plane + (uint32_t)o));
                    plane += N;
                }
            }
            // advance (ix, iy, iz) by blockDim cells with carries
            cell += blockDim.x;
            iz += sw.step_z;
            const uint32_t cz = iz >= nz;
            iz -= cz ? nz : 0;
            iy += sw.step_y + cz;
            const uint32_t cy = iy >= ny;
            iy -= cy ? ny : 0;
            ix += sw.step_x + cy;
        }
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const uint32_t c = cells[k];
            if (c >= N) continue;
            R* g = f[k];
            R mom[4], imb[3];
            fast_cell<TR, MOVING, RED>(sw, f[k], c, N, inlet[k], do_collide, do_imb, mom, imb, red, do_mom);
            if (do_collide) {
                T* dst = sw.dst + c;
                uint32_t plane = 0;
#pragma unroll
                for (int i = 0; i < Q; ++i) {
                    st_pop(dst + plane, TR::scaled ? g[i] * sw.scale : g[i]);
                    plane += N;
                }
                if (do_imb) {
                    sw.imb[c] = (O)imb[0];
                    sw.imb[(size_t)N + c] = (O)imb[1];
                    sw.imb[2 * (size_t)N + c] = (O)imb[2];
                }
            }
            if (do_mom) {
                sw.mom[c] = (O)(R(1) + mom[0]);
                sw.mom[(size_t)N + c] = (O)mom[1];
                sw.mom[2 * (size_t)N + c] = (O)mom[2];
                sw.mom[3 * (size_t)N + c] = (O)mom[3];
            }
        }
    }
    if (do_red && have)
        flush_segment<PSC_NRED>(red, sw.partials, sw.tile_begin, sw.tile_end - sw.tile_begin, total_tiles, gridDim.x);
}

template <int STORE, bool MOVING, int CPT, bool RED>
static cudaError_t launch_fast_t(const psc_window* d_windows, int nwin, int64_t total_tiles, unsigned flags,
                                 int grid_ctas, cudaStream_t stream) {
    if (grid_ctas <= 0) {
        static int per_sm[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int dev = 0;
        cudaGetDevice(&dev);
        int& occ = per_sm[dev & 7];
        if (occ == 0) {
            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_step_fast<STORE, MOVING, CPT, RED>,
                                                                          STEP_THREADS, 0);
            if (e != cudaSuccess) return e;
            if (occ <= 0) occ = 1;
        }
        const int64_t g = (int64_t)sm_count() * occ;
        grid_ctas = (int)(total_tiles < g ? total_tiles : g);
    }
    if ((int64_t)grid_ctas > total_tiles) grid_ctas = (int)total_tiles;  // every CTA owns >= 1 tile
    if (grid_ctas <= 0) return cudaSuccess;
    k_step_fast<STORE, MOVING, CPT, RED><<<grid_ctas, STEP_THREADS, 0, stream>>>(d_windows, nwin, total_tiles, flags);
    return cudaGetLastError();
}

template <int STORE, bool RED>
static cudaError_t launch_fast_r(const psc_window* d, int nwin, int64_t tiles, unsigned flags, bool moving, int cpt,
                                 int grid, cudaStream_t s) {
    switch (cpt) {
        case 1: return moving ? launch_fast_t<STORE, true, 1, RED>(d, nwin, tiles, flags, grid, s)
                              : launch_fast_t<STORE, false, 1, RED>(d, nwin, tiles, flags, grid, s);
        case 2: return moving ? launch_fast_t<STORE, true, 2, RED>(d, nwin, tiles, flags, grid, s)
                              : launch_fast_t<STORE, false, 2, RED>(d, nwin, tiles, flags, grid, s);
        case 4: return moving ? launch_fast_t<STORE, true, 4, RED>(d, nwin, tiles, flags, grid, s)
                              : launch_fast_t<STORE, false, 4, RED>(d, nwin, tiles, flags, grid, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int STORE>
static cudaError_t launch_fast_s(const psc_window* d, int nwin, int64_t tiles, unsigned flags, bool moving, int cpt,
                                 int grid, cudaStream_t s) {
    return (flags & PSC_STEP_REDUCE) ? launch_fast_r<STORE, true>(d, nwin, tiles, flags, moving, cpt, grid, s)
                                     : launch_fast_r<STORE, false>(d, nwin, tiles, flags, moving, cpt, grid, s);
}

cudaError_t launch_step_fast(int store, const psc_window* d_windows, int nwin, int64_t total_tiles, unsigned flags,
                             bool moving, int cpt, int grid_ctas, cudaStream_t stream) {
    switch (store) {
        case PSC_STORE_F64: return launch_fast_s<PSC_STORE_F64>(d_windows, nwin, total_tiles, flags, moving, cpt, grid_ctas, stream);
        case PSC_STORE_F32: return launch_fast_s<PSC_STORE_F32>(d_windows, nwin, total_tiles, flags, moving, cpt, grid_ctas, stream);
        case PSC_STORE_F16: return launch_fast_s<PSC_STORE_F16>(d_windows, nwin, total_tiles, flags, moving, cpt, grid_ctas, stream);
        case PSC_STORE_BF16: return launch_fast_s<PSC_STORE_BF16>(d_windows, nwin, total_tiles, flags, moving, cpt, grid_ctas, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace psc
