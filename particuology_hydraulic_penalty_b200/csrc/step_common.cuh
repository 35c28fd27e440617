// Storage traits and population-access helpers shared by the step kernels.
#pragma once

#include "collide.cuh"
#include "internal.cuh"

namespace psc {

template <int STORE>
struct StoreTraits;
template <>
struct StoreTraits<PSC_STORE_F64_EXACT> {
    using T = double;
    using R = double;
    using O = double;
    static constexpr bool exact = true;
    static constexpr bool scaled = false;
};
template <>
struct StoreTraits<PSC_STORE_F64> {
    using T = double;
    using R = double;
    using O = double;
    static constexpr bool exact = false;
    static constexpr bool scaled = false;
};
template <>
struct StoreTraits<PSC_STORE_F32> {
    using T = float;
    using R = float;
    using O = float;
    static constexpr bool exact = false;
    static constexpr bool scaled = false;
};
template <>
struct StoreTraits<PSC_STORE_F16> {
    using T = __half;
    using R = float;
    using O = float;
    static constexpr bool exact = false;
    static constexpr bool scaled = true;
};
template <>
struct StoreTraits<PSC_STORE_BF16> {
    using T = __nv_bfloat16;
    using R = float;
    using O = float;
    static constexpr bool exact = false;
    static constexpr bool scaled = true;
};

__device__ __forceinline__ double ld_pop(const double* p) { return __ldg(p); }
// FP32 pulls ask L2 to fetch the whole 256-byte line pair: consecutive tiles of
// a CTA read consecutive rows, so the neighbouring sectors are used next
// (measured +1.3 % on the 24-window batch).
__device__ __forceinline__ float ld_pop(const float* p) {
    float v;
    asm volatile("ld.global.nc.L2::256B.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ float ld_pop(const __half* p) { return __half2float(__ldg(p)); }
__device__ __forceinline__ float ld_pop(const __nv_bfloat16* p) { return __bfloat162float(__ldg(p)); }

template <typename R>
__device__ __forceinline__ R fast_rcp(R x);
template <>
__device__ __forceinline__ float fast_rcp<float>(float x) {
    return __frcp_rn(x);
}
template <>
__device__ __forceinline__ double fast_rcp<double>(double x) {
    return __drcp_rn(x);
}

// plain (shared-memory) reads of a stored population
__device__ __forceinline__ double ld_smem_pop(const double* p) { return *p; }
__device__ __forceinline__ float ld_smem_pop(const float* p) { return *p; }
__device__ __forceinline__ float ld_smem_pop(const __half* p) { return __half2float(*p); }
__device__ __forceinline__ float ld_smem_pop(const __nv_bfloat16* p) { return __bfloat162float(*p); }

__device__ __forceinline__ void st_pop(double* p, double v) { *p = v; }
__device__ __forceinline__ void st_pop(float* p, float v) { *p = v; }
// 16-bit stores stream (evict-first): measured +7 % for FP16 storage.
__device__ __forceinline__ void st_pop(__half* p, float v) { __stcs(p, __float2half_rn(v)); }
__device__ __forceinline__ void st_pop(__nv_bfloat16* p, float v) { __stcs(p, __float2bfloat16_rn(v)); }

// Offset (in cells) from x to x - c_i for direction i, given the wrapped
// neighbour offsets of this cell.
struct NbrOffsets {
    int32_t xm, xp, ym, yp, zm, zp;  // to ix-1, ix+1, iy-1, iy+1, iz-1, iz+1
};

// Offsets to the six face neighbours, periodic; with open_x the x faces
// point at the cell's own plane instead of wrapping (zero-gradient outflow at
// x = nx - 1; at x = 0 the inlet replaces the pulled values afterwards).
__device__ __forceinline__ NbrOffsets nbr_offsets(uint32_t ix, uint32_t iy, uint32_t iz, int nx, int ny, int nz,
                                                  bool open_x = false) {
    NbrOffsets o;
    const int32_t nyz = ny * nz;
    o.xm = ix == 0 ? (open_x ? 0 : (nx - 1) * nyz) : -nyz;
    o.xp = ix == (uint32_t)(nx - 1) ? (open_x ? 0 : -(nx - 1) * nyz) : nyz;
    o.ym = iy == 0 ? (ny - 1) * nz : -nz;
    o.yp = iy == (uint32_t)(ny - 1) ? -(ny - 1) * nz : nz;
    o.zm = iz == 0 ? nz - 1 : -1;
    o.zp = iz == (uint32_t)(nz - 1) ? -(nz - 1) : 1;
    return o;
}

template <int I>
__device__ __forceinline__ int32_t pull_offset(const NbrOffsets& o) {
    // source of direction I at x is x - c_I
    return (cxv(I) == 1 ? o.xm : (cxv(I) == -1 ? o.xp : 0)) + (cyv(I) == 1 ? o.ym : (cyv(I) == -1 ? o.yp : 0)) +
           (czv(I) == 1 ? o.zm : (czv(I) == -1 ? o.zp : 0));
}

template <typename T, typename R, int I>
struct PullLoop {
    __device__ __forceinline__ static void run(R* f, const T* src, size_t N, uint32_t cell, const NbrOffsets& o,
                                               R inv_scale, bool scaled) {
        PullLoop<T, R, I - 1>::run(f, src, N, cell, o, inv_scale, scaled);
        const R v = ld_pop(src + (size_t)(I - 1) * N + (size_t)((int64_t)cell + pull_offset<I - 1>(o)));
        f[I - 1] = scaled ? v * inv_scale : v;
    }
};
template <typename T, typename R>
struct PullLoop<T, R, 0> {
    __device__ __forceinline__ static void run(R*, const T*, size_t, uint32_t, const NbrOffsets&, R, bool) {}
};

__device__ __forceinline__ int find_window(const psc_window* wins, const int64_t* s_begin, int nwin, int64_t t) {
    int lo = 0, hi = nwin - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int64_t b = s_begin ? s_begin[mid] : wins[mid].tile_begin;
        if (b <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Warp sums of v, written as this warp's row of a tile's partials:
// rows[warp][k] for k < NV (lane k stores value k).  No block barrier.
template <int NV>
__device__ __forceinline__ void warp_reduce_store(double (&v)[NV], double* rows) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* out = rows + (size_t)warp * NV;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = v[k];
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) x += __shfl_xor_sync(0xffffffffu, x, s);
        if (lane == k) out[k] = x;
    }
}

// The CTA of a persistent grid of `grid` CTAs over `total` tiles (CTA b owns
// [total * b / grid, total * (b + 1) / grid)) that owns tile t.
__device__ __forceinline__ int64_t cta_of_tile(int64_t t, int64_t total, int64_t grid) {
    return ((t + 1) * grid - 1) / total;
}

// End of this CTA's run of tiles inside one window: each warp writes the sums
// of its threads' accumulators as row (b - b_first) * PSC_PARTIAL_ROWS + warp
// of the window's partials (after the header row), and the window's first
// CTA writes the row count into the header.  Resets the accumulators.
template <int NV>
__device__ __forceinline__ void flush_segment(double (&red)[NV], double* partials, int64_t tile_begin,
                                              int64_t tile_count, int64_t total, int64_t grid) {
    const int64_t bf = cta_of_tile(tile_begin, total, grid);
    const int64_t bl = cta_of_tile(tile_begin + tile_count - 1, total, grid);
    const int64_t row = ((int64_t)blockIdx.x - bf) * PSC_PARTIAL_ROWS;
    warp_reduce_store<NV>(red, partials + (1 + row) * NV);
    if ((int64_t)blockIdx.x == bf && threadIdx.x == 0) partials[0] = (double)((bl - bf + 1) * PSC_PARTIAL_ROWS);
#pragma unroll
    for (int k = 0; k < NV; ++k) red[k] = 0.0;
}

template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double (*s_red)[NV], double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = v[k];
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) x += __shfl_xor_sync(0xffffffffu, x, s);
        if (lane == 0) s_red[warp][k] = x;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double acc = 0.0;
        const int nw = blockDim.x >> 5;
        for (int w = 0; w < nw; ++w) acc += s_red[w][threadIdx.x];
        out[threadIdx.x] = acc;
    }
    __syncthreads();
}

}  // namespace psc
