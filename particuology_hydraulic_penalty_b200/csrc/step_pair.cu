// Pair kernel for the deviation storage modes: the step of k_step_fast
// (pull-stream + PSC-IMB collide, src/lbm_dem/psc3d.py:208-246) with each
// thread owning two consecutive z cells (c, c + 1), c even.
//
// With nz even a pair never crosses a z row, so the nine directions with
// c_z = 0 pull both cells with one aligned 2-element load, and all nineteen
// populations (and the IMB / moment fields) are written with 2-element
// stores; the ten z-shifted directions pull two scalars.  Measured on the
// bare access pattern (19 planes read + 19 written, 33 M cells): 2-element
// accesses at two CTAs per SM move 6.5 TB/s against 5.1-5.9 TB/s for scalar
// ones.  The per-cell arithmetic is fast_cell(), the same function as the
// one-cell kernel's, so both produce identical populations.
#include "fast_cell.cuh"
#include "internal.cuh"

namespace psc {

// Set (once) when a launch met a window it cannot run: 0x201 odd nz,
// 0x202 tiles not planned by psc_plan_pair_tiles.  Such windows are skipped.
__device__ int g_pair_status = 0;

constexpr int PAIR_CELLS = 2;

__device__ __forceinline__ void ld_pair(const float* p, float& a, float& b) {
    asm volatile("ld.global.nc.L2::256B.v2.f32 {%0, %1}, [%2];" : "=f"(a), "=f"(b) : "l"(p));
}
__device__ __forceinline__ void ld_pair(const double* p, double& a, double& b) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    a = v.x;
    b = v.y;
}
__device__ __forceinline__ void ld_pair(const __half* p, float& a, float& b) {
    const float2 v = __half22float2(__ldg(reinterpret_cast<const __half2*>(p)));
    a = v.x;
    b = v.y;
}
__device__ __forceinline__ void ld_pair(const __nv_bfloat16* p, float& a, float& b) {
    const float2 v = __bfloat1622float2(__ldg(reinterpret_cast<const __nv_bfloat162*>(p)));
    a = v.x;
    b = v.y;
}

__device__ __forceinline__ void st_pair(float* p, float a, float b) {
    *reinterpret_cast<float2*>(p) = make_float2(a, b);
}
__device__ __forceinline__ void st_pair(double* p, double a, double b) {
    *reinterpret_cast<double2*>(p) = make_double2(a, b);
}
// 16-bit pairs stream (evict-first) like the one-cell stores; the same round-to-nearest conversion
__device__ __forceinline__ void st_pair(__half* p, float a, float b) {
    __stcs(reinterpret_cast<__half2*>(p), __floats2half2_rn(a, b));
}
__device__ __forceinline__ void st_pair(__nv_bfloat16* p, float a, float b) {
    __stcs(reinterpret_cast<__nv_bfloat162*>(p), __floats2bfloat162_rn(a, b));
}

// Resident CTAs the register allocation aims for: two cells per thread need
// about twice the registers of the one-cell kernel.
template <int STORE, bool MOVING, bool RED>
struct PairOccupancy {
    static constexpr int value = (STORE == PSC_STORE_F64) ? 1 : 2;
};

template <int STORE, bool MOVING, bool RED>
__global__ void __launch_bounds__(STEP_THREADS, (PairOccupancy<STORE, MOVING, RED>::value))
    k_step_pair(const psc_window* __restrict__ wins, int nwin, int64_t total_tiles, unsigned flags) {
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
    double red[PSC_NRED];
#pragma unroll
    for (int q = 0; q < PSC_NRED; ++q) red[q] = 0.0;
    bool have = false;
    bool skip = false;  // block-uniform: the window in sw cannot run here
    // this thread's first cell (ix, iy, iz) in the current tile: divided out when the CTA enters a
    // window, then advanced tile by tile (consecutive tiles, tile_cells apart) by a carry-add
    bool fresh = true;
    uint32_t ix = 0, iy = 0, iz = 0;
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
            skip = (sw.nz & 1u) != 0 || sw.tile_cells != PAIR_CELLS * (int32_t)blockDim.x;
            fresh = true;
            if (skip && threadIdx.x == 0) atomicCAS(&g_pair_status, 0, (sw.nz & 1u) ? 0x201 : 0x202);
        }
        if (sw.inactive || skip) continue;  // block-uniform
        have = true;
        const uint32_t N = sw.N, nx = sw.nx, ny = sw.ny, nz = sw.nz;
        const uint32_t c0 = (uint32_t)((t - sw.tile_begin) * sw.tile_cells) + PAIR_CELLS * threadIdx.x;
        if (fresh) {
            iz = c0 % nz;
            const uint32_t rr = c0 / nz;
            iy = rr % ny;
            ix = rr / ny;
            fresh = false;
        } else {  // one tile on: += the tile step, single carries (each step component < its extent)
            iz += sw.tstep_z;
            const uint32_t cz = iz >= nz;
            iz -= cz ? nz : 0u;
            iy += sw.tstep_y + cz;
            const uint32_t cy = iy >= ny;
            iy -= cy ? ny : 0u;
            ix += sw.tstep_x + cy;
        }
        if (c0 >= N) continue;  // N is even: c0 + 1 < N as well (the window's last tile)
        const uint32_t c1 = c0 + 1;
        const bool open_x = sw.open_x;
        const bool inlet = open_x && ix == 0;
        const int32_t nyz = (int32_t)(ny * nz);
        const int32_t xm = ix == 0 ? (open_x ? 0 : (int32_t)(nx - 1) * nyz) : -nyz;
        const int32_t xp = ix == nx - 1 ? (open_x ? 0 : -(int32_t)(nx - 1) * nyz) : nyz;
        const int32_t ym = iy == 0 ? (int32_t)(ny - 1) * (int32_t)nz : -(int32_t)nz;
        const int32_t yp = iy == ny - 1 ? -(int32_t)(ny - 1) * (int32_t)nz : (int32_t)nz;
        // z sources: c0 pulls z - 1 (wraps at iz = 0) and z + 1 (iz + 1 <= nz - 1); c1 pulls z (= iz) and
        // z + 2 (wraps when iz + 1 == nz - 1)
        const int32_t zm0 = iz == 0 ? (int32_t)nz - 1 : -1;
        const int32_t zp1 = iz + 2 == nz ? -(int32_t)(nz - 1) : 1;
        const T* src = sw.src;
        R g0[Q], g1[Q];
        uint32_t plane = 0;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int32_t oxy = (cxv(i) == 1 ? xm : (cxv(i) == -1 ? xp : 0)) + (cyv(i) == 1 ? ym : (cyv(i) == -1 ? yp : 0));
            const T* p = src + (int64_t)(int32_t)(plane + c0 + (uint32_t)oxy);
            if (czv(i) == 0) {
                ld_pair(p, g0[i], g1[i]);  // c0 even, oxy a multiple of nz (even): aligned
            } else if (czv(i) == 1) {
                g0[i] = ld_pop(p + zm0);
                g1[i] = ld_pop(p);
            } else {
                g0[i] = ld_pop(p + 1);
                g1[i] = ld_pop(p + 1 + zp1);
            }
            plane += N;
        }
        R mom0[4], imb0[3], mom1[4], imb1[3];
        fast_cell<TR, MOVING, RED>(sw, g0, c0, N, inlet, do_collide, do_imb, mom0, imb0, red, do_mom);
        fast_cell<TR, MOVING, RED>(sw, g1, c1, N, inlet, do_collide, do_imb, mom1, imb1, red, do_mom);
        if (do_collide) {
            T* dst = sw.dst + c0;
            uint32_t pl = 0;
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                if (TR::scaled) st_pair(dst + pl, g0[i] * sw.scale, g1[i] * sw.scale);
                else st_pair(dst + pl, g0[i], g1[i]);
                pl += N;
            }
            if (do_imb) {
#pragma unroll
                for (int k = 0; k < 3; ++k) st_pair(sw.imb + (size_t)k * N + c0, (O)imb0[k], (O)imb1[k]);
            }
        }
        if (do_mom) {
            st_pair(sw.mom + c0, (O)(R(1) + mom0[0]), (O)(R(1) + mom1[0]));
#pragma unroll
            for (int k = 1; k < 4; ++k) st_pair(sw.mom + (size_t)k * N + c0, (O)mom0[k], (O)mom1[k]);
        }
    }
    if (do_red && have)
        flush_segment<PSC_NRED>(red, sw.partials, sw.tile_begin, sw.tile_end - sw.tile_begin, total_tiles, gridDim.x);
}

template <int STORE, bool MOVING, bool RED>
static cudaError_t launch_pair_t(const psc_window* d_windows, int nwin, int64_t total_tiles, unsigned flags,
                                 int grid_ctas, cudaStream_t stream) {
    if (grid_ctas <= 0) {
        static int per_sm[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int dev = 0;
        cudaGetDevice(&dev);
        int& occ = per_sm[dev & 7];
        if (occ == 0) {
            cudaError_t e =
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_step_pair<STORE, MOVING, RED>, STEP_THREADS, 0);
            if (e != cudaSuccess) return e;
            if (occ <= 0) occ = 1;
        }
        const int64_t g = (int64_t)sm_count() * occ;
        grid_ctas = (int)(total_tiles < g ? total_tiles : g);
    }
    if ((int64_t)grid_ctas > total_tiles) grid_ctas = (int)total_tiles;  // every CTA owns >= 1 tile
    if (grid_ctas <= 0) return cudaSuccess;
    k_step_pair<STORE, MOVING, RED><<<grid_ctas, STEP_THREADS, 0, stream>>>(d_windows, nwin, total_tiles, flags);
    return cudaGetLastError();
}

template <int STORE>
static cudaError_t launch_pair_s(const psc_window* d, int nwin, int64_t tiles, unsigned flags, bool moving, int grid,
                                 cudaStream_t s) {
    const bool red = (flags & PSC_STEP_REDUCE) != 0;
    if (moving) return red ? launch_pair_t<STORE, true, true>(d, nwin, tiles, flags, grid, s)
                           : launch_pair_t<STORE, true, false>(d, nwin, tiles, flags, grid, s);
    return red ? launch_pair_t<STORE, false, true>(d, nwin, tiles, flags, grid, s)
               : launch_pair_t<STORE, false, false>(d, nwin, tiles, flags, grid, s);
}

cudaError_t launch_step_pair(int store, const psc_window* d_windows, int nwin, int64_t total_tiles, unsigned flags,
                             bool moving, int grid_ctas, cudaStream_t stream) {
    switch (store) {
        case PSC_STORE_F64: return launch_pair_s<PSC_STORE_F64>(d_windows, nwin, total_tiles, flags, moving, grid_ctas, stream);
        case PSC_STORE_F32: return launch_pair_s<PSC_STORE_F32>(d_windows, nwin, total_tiles, flags, moving, grid_ctas, stream);
        case PSC_STORE_F16: return launch_pair_s<PSC_STORE_F16>(d_windows, nwin, total_tiles, flags, moving, grid_ctas, stream);
        case PSC_STORE_BF16: return launch_pair_s<PSC_STORE_BF16>(d_windows, nwin, total_tiles, flags, moving, grid_ctas, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t read_pair_status(int* out, bool clear) {
    cudaError_t e = cudaMemcpyFromSymbol(out, g_pair_status, sizeof(int));
    if (e != cudaSuccess || !clear) return e;
    const int zero = 0;
    return cudaMemcpyToSymbol(g_pair_status, &zero, sizeof(int));
}

}  // namespace psc
