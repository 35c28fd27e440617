// Particle geometry on the GPU: sub-sampled solid fraction (K1), solid
// velocity, and per-particle IMB force / torque (K3).
//
// Reference: src/lbm_dem/psc3d.py
//   bbox + S^3 inside count      :60-94 (sparse task), :151-173 (dense)
//   alpha sum / solid             :174-175, :339-344
//   solid velocity                :181-206, :347-373
//   particle loads                :255-281, :375-407
//
// Data flow (all device-resident, no host round trip except the entry total
// that sizes the caller's buffers):
//   plan     one block: clipped bbox per particle, entry offsets (sum of bbox
//            volumes) and load-chunk offsets by block scans
//   count    one thread per (particle, bbox cell): S^3 inside tests in FP64
//            with the reference's rounding (no FMA) -> uint16 count; bump the
//            per-cell particle counter
//   scan     counters -> per-cell list offsets
//   fill     scatter (particle, count) into the cell lists
//   final    per cell: sort its list by particle id, sum alpha = count / S^3 in
//            that order from 0.0 (bit-identical to NumPy's sequential sums),
//            clip to the solid fraction, clipped integer level
//   loads    chunks of bbox entries per particle, deterministic block sums,
//            then a fixed-order per-particle sum of the chunk partials
#include "collide.cuh"
#include "internal.cuh"

namespace psc {

constexpr int PF = 10;  // particle fields: x y z r vx vy vz wx wy wz

// Clipped [lo, hi) box per axis: lo = max(0, floor(c - r - 1)),
// hi = min(n, ceil(c + r + 1))  (psc3d.py:73-78).
__device__ __forceinline__ void axis_box(double c, double r, int n, int32_t& lo, int32_t& ext) {
    double a = floor(xsub(xsub(c, r), 1.0));
    double b = ceil(xadd(xadd(c, r), 1.0));
    if (!(a > 0.0)) a = 0.0;  // also maps NaN to 0 (rejected on the host)
    if (!(b < (double)n)) b = (double)n;
    if (a > (double)n) a = (double)n;
    if (b < 0.0) b = 0.0;
    lo = (int32_t)a;
    const int32_t hi = (int32_t)b;
    ext = hi > lo ? hi - lo : 0;
}

template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* s_warp, T& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    T x = v;
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, x, s);
        if (lane >= s) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T w = lane < nw ? s_warp[lane] : T(0);
#pragma unroll
        for (int s = 1; s < 32; s <<= 1) {
            const T y = __shfl_up_sync(0xffffffffu, w, s);
            if (lane >= s) w += y;
        }
        if (lane < nw) s_warp[lane] = w;
    }
    __syncthreads();
    const T warp_prefix = warp > 0 ? s_warp[warp - 1] : T(0);
    total = s_warp[nw - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

// One block: boxes, entry offsets, chunk offsets, totals.
__global__ void __launch_bounds__(1024) k_geometry_plan(psc_geometry g) {
    __shared__ int64_t s_warp[32];
    __shared__ int64_t s_carry[2];
    const int P = g.nparticles;
    if (threadIdx.x == 0) {
        s_carry[0] = 0;
        s_carry[1] = 0;
    }
    __syncthreads();
    const int64_t ch = g.chunk_entries;
    for (int base = 0; base < P; base += blockDim.x) {
        const int p = base + threadIdx.x;
        int64_t vol = 0;
        if (p < P) {
            const double* q = g.particles + (size_t)p * PF;
            int32_t lo[3], ex[3];
            axis_box(q[0], q[3], g.nx, lo[0], ex[0]);
            axis_box(q[1], q[3], g.ny, lo[1], ex[1]);
            axis_box(q[2], q[3], g.nz, lo[2], ex[2]);
            int32_t* bb = g.bbox + (size_t)p * 6;
            bb[0] = lo[0];
            bb[1] = lo[1];
            bb[2] = lo[2];
            bb[3] = ex[0];
            bb[4] = ex[1];
            bb[5] = ex[2];
            vol = (int64_t)ex[0] * ex[1] * ex[2];
        }
        const int64_t nch = (vol + ch - 1) / ch;
        int64_t tot_e, tot_c;
        const int64_t pe = block_exclusive_scan<int64_t>(vol, s_warp, tot_e);
        const int64_t pc = block_exclusive_scan<int64_t>(nch, s_warp, tot_c);
        if (p < P) {
            g.ent_off[p] = s_carry[0] + pe;
            g.chunk_off[p] = s_carry[1] + pc;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_carry[0] += tot_e;
            s_carry[1] += tot_c;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        g.ent_off[P] = s_carry[0];
        g.chunk_off[P] = s_carry[1];
        g.totals[0] = s_carry[0];
        g.totals[1] = s_carry[1];
        g.totals[2] = 0;
        g.totals[3] = (s_carry[0] > g.capacity_entries || s_carry[1] > g.capacity_chunks) ? 1 : 0;
    }
}

// Largest p with off[p] <= e (off has P+1 non-decreasing entries, off[0] = 0).
__device__ __forceinline__ int owner_of(const int64_t* off, int P, int64_t e) {
    int lo = 0, hi = P - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= e) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Inside-sample count of one cell: offsets (k + 0.5)/S, d = (i + o) - c,
// (dx*dx + dy*dy) + dz*dz <= r*r, every operation rounded once
// (psc3d.py:72, :86-89).
__device__ __forceinline__ int sample_count(int32_t ix, int32_t iy, int32_t iz, double px, double py, double pz,
                                            double rr, int S) {
    const double Sd = (double)S;
    int cnt = 0;
    for (int a = 0; a < S; ++a) {
        const double dx = xsub(xadd((double)ix, xdiv((double)a + 0.5, Sd)), px);
        const double dx2 = xmul(dx, dx);
        for (int b = 0; b < S; ++b) {
            const double dy = xsub(xadd((double)iy, xdiv((double)b + 0.5, Sd)), py);
            const double dxy = xadd(dx2, xmul(dy, dy));
            for (int c = 0; c < S; ++c) {
                const double dz = xsub(xadd((double)iz, xdiv((double)c + 0.5, Sd)), pz);
                cnt += xadd(dxy, xmul(dz, dz)) <= rr ? 1 : 0;
            }
        }
    }
    return cnt;
}

// Smooth surrogate of sample_count / S^3: every sample contributes
// sigma((r - d_s) / eps) (logistic via tanh), the differentiable solid
// fraction used by the adjoint.  Same boxes and sample offsets as the count.
__device__ __forceinline__ double smooth_alpha(int32_t ix, int32_t iy, int32_t iz, double px, double py, double pz,
                                               double r, int S, double eps) {
    const double Sd = (double)S;
    double acc = 0.0;
    for (int a = 0; a < S; ++a) {
        const double dx = ((double)ix + ((double)a + 0.5) / Sd) - px;
        for (int b = 0; b < S; ++b) {
            const double dy = ((double)iy + ((double)b + 0.5) / Sd) - py;
            for (int c = 0; c < S; ++c) {
                const double dz = ((double)iz + ((double)c + 0.5) / Sd) - pz;
                const double d = sqrt(dx * dx + dy * dy + dz * dz);
                acc += 0.5 * (1.0 + tanh(0.5 * (r - d) / eps));
            }
        }
    }
    return acc / (Sd * Sd * Sd);
}

// Descriptor of one load-reduction chunk, computed by k_chunk_desc (one
// thread per chunk, so the lookups of many chunks overlap) into the chunk's
// own partial row (6 doubles); every thread of the chunk's block reads it
// before the chunk's last warp overwrites the row with the sums.
struct ChunkDesc {
    int64_t e0, e1;       // entry range
    int32_t p;            // particle
    int32_t local0;       // e0 - ent_off[p]
    int32_t x0, y0, z0;   // clipped box origin
    int32_t ey, ez;       // box extents in y and z
    int32_t pad;
};
static_assert(sizeof(ChunkDesc) == 6 * sizeof(double), "a chunk descriptor fills one partial row");

__device__ __forceinline__ ChunkDesc make_chunk_desc(const psc_geometry& g, int64_t c) {
    const int p = owner_of(g.chunk_off, g.nparticles, c);
    const int64_t eb = g.ent_off[p];
    ChunkDesc d;
    d.e0 = eb + (c - g.chunk_off[p]) * g.chunk_entries;
    d.e1 = min(d.e0 + (int64_t)g.chunk_entries, g.ent_off[p + 1]);
    d.p = p;
    d.local0 = (int32_t)(d.e0 - eb);
    const int32_t* bb = g.bbox + (size_t)p * 6;
    d.x0 = bb[0];
    d.y0 = bb[1];
    d.z0 = bb[2];
    d.ey = bb[4];
    d.ez = bb[5];
    d.pad = 0;
    return d;
}

// sample_count for a compile-time S: the same IEEE operations on the same
// operands, with the sample offsets (k + 0.5) / S computed once per thread and
// each axis's squared distances once per cell (S values per axis), so a
// sample costs one addition and one comparison: (dx2 + dy2) + dz2 <= r^2.
template <int S>
__device__ __forceinline__ int sample_count_t(int32_t ix, int32_t iy, int32_t iz, double px, double py, double pz,
                                              double rr, const double (&o)[S]) {
    double dy2[S], dz2[S];
#pragma unroll
    for (int k = 0; k < S; ++k) {
        const double dy = xsub(xadd((double)iy, o[k]), py);
        const double dz = xsub(xadd((double)iz, o[k]), pz);
        dy2[k] = xmul(dy, dy);
        dz2[k] = xmul(dz, dz);
    }
    int cnt = 0;
#pragma unroll
    for (int a = 0; a < S; ++a) {
        const double dx = xsub(xadd((double)ix, o[a]), px);
        const double dx2 = xmul(dx, dx);
#pragma unroll
        for (int b = 0; b < S; ++b) {
            const double dxy = xadd(dx2, dy2[b]);
#pragma unroll
            for (int c = 0; c < S; ++c) cnt += xadd(dxy, dz2[c]) <= rr ? 1 : 0;
        }
    }
    return cnt;
}

// Inside-sample count of every bbox entry (S: the subsample count as a
// compile-time constant, or 0: the general loop) and the per-cell entry counts
// of the cell lists.
//
// One block per load chunk (its particle and entry range from the chunk
// offsets, one lookup per chunk instead of one per entry); thread t takes the
// chunk's entries t, t + blockDim.x, ... and steps their bbox-local
// coordinates by a carry-add.
template <int S>
__global__ void __launch_bounds__(256, 2) k_geometry_count(psc_geometry g) {
    const int64_t E = min(g.totals[0], g.capacity_entries);
    const int64_t C = g.totals[1];
    const bool smooth = g.smooth_eps > 0.0;
    double o[S > 0 ? S : 1];
#pragma unroll
    for (int k = 0; k < (S > 0 ? S : 1); ++k) o[k] = xdiv((double)k + 0.5, (double)(S > 0 ? S : 1));  // (k + 0.5) / S
    const uint32_t ny = (uint32_t)g.ny, nz = (uint32_t)g.nz;
    for (int64_t chunk = blockIdx.x; chunk < C; chunk += gridDim.x) {
        const ChunkDesc dsc = make_chunk_desc(g, chunk);
        const int64_t e1 = min(dsc.e1, E);
        int64_t e = dsc.e0 + threadIdx.x;
        if (e >= e1) continue;
        const double* q = g.particles + (size_t)dsc.p * PF;
        const double px = q[0], py = q[1], pz = q[2], r = q[3], rr = xmul(r, r);
        const uint32_t ey = (uint32_t)dsc.ey, ez = (uint32_t)dsc.ez, eyz = ey * ez;
        const uint32_t local = (uint32_t)dsc.local0 + threadIdx.x;
        uint32_t a = local / eyz;
        const uint32_t rem = local - a * eyz;
        uint32_t b = rem / ez;
        uint32_t k = rem - b * ez;
        const uint32_t step_k = blockDim.x % ez;
        const uint32_t step_q = blockDim.x / ez;
        const uint32_t step_b = step_q % ey;
        const uint32_t step_a = step_q / ey;
        for (; e < e1; e += blockDim.x) {
            const int32_t ix = dsc.x0 + (int32_t)a, iy = dsc.y0 + (int32_t)b, iz = dsc.z0 + (int32_t)k;
            int cnt;
            if (smooth) {
                const double al = smooth_alpha(ix, iy, iz, px, py, pz, r, g.subsamples, g.smooth_eps);
                g.ent_alpha[e] = al;
                cnt = al > 0.0 ? 1 : 0;  // membership of the cell list
            } else if constexpr (S > 0) {
                cnt = sample_count_t<S>(ix, iy, iz, px, py, pz, rr, o);
            } else {
                cnt = sample_count(ix, iy, iz, px, py, pz, rr, g.subsamples);
            }
            g.ent_cnt[e] = (uint16_t)cnt;
            if (cnt > 0) atomicAdd(g.cell_n + (((uint32_t)ix * ny + (uint32_t)iy) * nz + (uint32_t)iz), 1);
            // next entry of this thread: (a, b, k) += (step_a, step_b, step_k) with carries
            k += step_k;
            const uint32_t ck = k >= ez;
            k -= ck ? ez : 0u;
            b += step_b + ck;
            const uint32_t cb = b >= ey;
            b -= cb ? ey : 0u;
            a += step_a + cb;
        }
    }
}

// The cell lists: every entry with a non-zero count appends (particle, count)
// to its cell's list (the order within a list is fixed by k_geometry_final's
// sort).  Walks the chunks as k_geometry_count does.
__global__ void __launch_bounds__(256) k_geometry_fill(psc_geometry g) {
    const int64_t E = min(g.totals[0], g.capacity_entries);
    const int64_t C = g.totals[1];
    const uint32_t ny = (uint32_t)g.ny, nz = (uint32_t)g.nz;
    for (int64_t chunk = blockIdx.x; chunk < C; chunk += gridDim.x) {
        const ChunkDesc dsc = make_chunk_desc(g, chunk);
        const int64_t e1 = min(dsc.e1, E);
        int64_t e = dsc.e0 + threadIdx.x;
        if (e >= e1) continue;
        const uint32_t ey = (uint32_t)dsc.ey, ez = (uint32_t)dsc.ez, eyz = ey * ez;
        const uint32_t local = (uint32_t)dsc.local0 + threadIdx.x;
        uint32_t a = local / eyz;
        const uint32_t rem = local - a * eyz;
        uint32_t b = rem / ez;
        uint32_t k = rem - b * ez;
        const uint32_t step_k = blockDim.x % ez;
        const uint32_t step_q = blockDim.x / ez;
        const uint32_t step_b = step_q % ey;
        const uint32_t step_a = step_q / ey;
        for (; e < e1; e += blockDim.x) {
            const uint16_t cnt = g.ent_cnt[e];
            if (cnt != 0) {
                const uint32_t cell = (((uint32_t)dsc.x0 + a) * ny + ((uint32_t)dsc.y0 + b)) * nz + ((uint32_t)dsc.z0 + k);
                const int32_t pos = atomicAdd(g.cell_n + cell, 1);
                const int64_t idx = (int64_t)g.cell_off[cell] + pos;
                if (idx < g.capacity_entries) {
                    g.cl_pid[idx] = dsc.p;
                    g.cl_cnt[idx] = cnt;
                    if (g.cl_ent) g.cl_ent[idx] = (int32_t)e;
                }
            }
            k += step_k;
            const uint32_t ck = k >= ez;
            k -= ck ? ez : 0u;
            b += step_b + ck;
            const uint32_t cb = b >= ey;
            b -= cb ? ey : 0u;
            a += step_a + cb;
        }
    }
}

__global__ void k_geometry_final(psc_geometry g) {
    const uint32_t N = (uint32_t)g.nx * g.ny * g.nz;
    const int S = g.subsamples;
    const int S3 = S * S * S;
    const double S3d = (double)S3;
    int local_max = 0;
    for (uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x; cell < N; cell += gridDim.x * blockDim.x) {
        const int32_t b = g.cell_off[cell], e = g.cell_off[cell + 1];
        const int L = e - b;
        local_max = max(local_max, L);
        // insertion sort by particle id (lists are a handful long)
        const bool smooth = g.smooth_eps > 0.0;
        for (int i = b + 1; i < e; ++i) {
            const int32_t kp = g.cl_pid[i];
            const uint16_t kc = g.cl_cnt[i];
            const int32_t ke = smooth ? g.cl_ent[i] : 0;
            int j = i - 1;
            while (j >= b && g.cl_pid[j] > kp) {
                g.cl_pid[j + 1] = g.cl_pid[j];
                g.cl_cnt[j + 1] = g.cl_cnt[j];
                if (smooth) g.cl_ent[j + 1] = g.cl_ent[j];
                --j;
            }
            g.cl_pid[j + 1] = kp;
            g.cl_cnt[j + 1] = kc;
            if (smooth) g.cl_ent[j + 1] = ke;
        }
        double asum = 0.0;
        int csum = 0;
        for (int i = b; i < e; ++i) {
            const int c = g.cl_cnt[i];
            asum = smooth ? asum + g.ent_alpha[g.cl_ent[i]] : xadd(asum, xdiv((double)c, S3d));
            csum += c;
        }
        g.alpha_sum[cell] = asum;
        g.solid[cell] = asum < 0.0 ? 0.0 : (asum > 1.0 ? 1.0 : asum);
        if (g.level) g.level[cell] = (uint8_t)(csum < S3 ? csum : S3);
    }
    // warp max then one atomic per warp
    for (int s = 16; s > 0; s >>= 1) local_max = max(local_max, __shfl_xor_sync(0xffffffffu, local_max, s));
    if ((threadIdx.x & 31) == 0 && local_max > 0)
        atomicMax(reinterpret_cast<unsigned long long*>(g.totals + 2), (unsigned long long)local_max);
}

template <typename O>
__global__ void k_solid_velocity(psc_geometry g, O* us) {
    const uint32_t N = (uint32_t)g.nx * g.ny * g.nz;
    const double S3d = (double)(g.subsamples * g.subsamples * g.subsamples);
    for (uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x; cell < N; cell += gridDim.x * blockDim.x) {
        const int32_t b = g.cell_off[cell], e = g.cell_off[cell + 1];
        double ux = 0.0, uy = 0.0, uz = 0.0;
        if (e > b) {
            const uint32_t iz = cell % g.nz, rr = cell / g.nz, iy = rr % g.ny, ix = rr / g.ny;
            const double xn = xadd((double)ix, 0.5), yn = xadd((double)iy, 0.5), zn = xadd((double)iz, 0.5);
            for (int i = b; i < e; ++i) {
                const double* q = g.particles + (size_t)g.cl_pid[i] * PF;
                const double al = xdiv((double)g.cl_cnt[i], S3d);
                const double rx = xsub(xn, q[0]), ry = xsub(yn, q[1]), rz = xsub(zn, q[2]);
                // v = V + w x r in the reference's term order (psc3d.py:362-364)
                const double vx = xsub(xadd(q[4], xmul(q[8], rz)), xmul(q[9], ry));
                const double vy = xsub(xadd(q[5], xmul(q[9], rx)), xmul(q[7], rz));
                const double vz = xsub(xadd(q[6], xmul(q[7], ry)), xmul(q[8], rx));
                ux = xadd(ux, xmul(al, vx));
                uy = xadd(uy, xmul(al, vy));
                uz = xadd(uz, xmul(al, vz));
            }
            const double as = g.alpha_sum[cell];
            if (as > 1.0e-14) {
                ux = xdiv(ux, as);
                uy = xdiv(uy, as);
                uz = xdiv(uz, as);
            }
        }
        us[cell] = (O)ux;
        us[(size_t)N + cell] = (O)uy;
        us[2 * (size_t)N + cell] = (O)uz;
    }
}

constexpr int LOAD_THREADS = 256;
constexpr int LOAD_WARPS = LOAD_THREADS / 32;

// Chunk sums without a block barrier per chunk.  Every warp of a block visits
// the block's chunks in the same order (its threads' columns of each), adds
// its 32 threads' sums by an xor-shuffle tree and leaves the warp sum in a
// ring slot of the chunk; the warp that completes the slot's count adds the
// LOAD_WARPS warp sums in warp order from 0.0 and writes the chunk row (the
// order of a block reduction through shared memory by thread 0).  A warp runs up
// to CHUNK_RING chunks ahead of the slowest warp of its block before it waits
// for a slot.  The slowest warp never waits, so every wait ends; the wait is
// bounded all the same (status 0x301, psc_device_status).
//
// With a barrier per chunk the block moved at the pace of its slowest warp
// (threads own 0 to 16 list entries of a chunk, one or two staging passes)
// and ncu counted 4.2 barrier stalls per issue on the list kernel; without
// it the 24-window batch's list reduction took 318 us instead of 427.
constexpr int CHUNK_RING = 4;
__device__ int g_loads_status = 0;

struct ChunkRing {
    double v[CHUNK_RING][LOAD_WARPS][6];
    int count[CHUNK_RING];
    long long done[CHUNK_RING];  // block-local index of the chunk last written from the slot
};

__device__ __forceinline__ void chunk_ring_init(ChunkRing& r) {
    if (threadIdx.x < CHUNK_RING) {
        r.count[threadIdx.x] = 0;
        r.done[threadIdx.x] = (long long)threadIdx.x - CHUNK_RING;
    }
    __syncthreads();
}

// Warp-level end of the block's j-th chunk: acc (this thread's sums) joins
// the chunk's row once every warp of the block has finished the chunk.
__device__ __forceinline__ void chunk_ring_finish(ChunkRing& r, long long j, double (&acc)[6], double* row) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = (int)(j % CHUNK_RING);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        double x = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        acc[k] = x;
    }
    if (lane == 0) {
        volatile long long* done = r.done;
        uint32_t spins = 0;
        while (done[slot] != j - CHUNK_RING) {  // the slot's previous chunk is written out
            if (++spins > (1u << 24)) {
                atomicCAS(&g_loads_status, 0, 0x301);
                break;
            }
            __nanosleep(64);
        }
        volatile double* v = &r.v[slot][warp][0];
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] = acc[k];
        __threadfence_block();
        if (atomicAdd(&r.count[slot], 1) == LOAD_WARPS - 1) {  // the chunk's last warp
            __threadfence_block();
            volatile const double* all = &r.v[slot][0][0];
            double out[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                double s = 0.0;
                for (int w = 0; w < LOAD_WARPS; ++w) s += all[w * 6 + k];
                out[k] = s;
            }
#pragma unroll
            for (int k = 0; k < 6; ++k) row[k] = out[k];
            atomicExch(&r.count[slot], 0);
            __threadfence_block();
            done[slot] = j;
        }
    }
    __syncwarp();
}

__global__ void __launch_bounds__(256) k_chunk_desc(psc_geometry g, double* part) {
    const int64_t C = g.totals[1];
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C; c += (int64_t)gridDim.x * blockDim.x)
        *reinterpret_cast<ChunkDesc*>(part + c * 6) = make_chunk_desc(g, c);
}

// The block's table of inside / S^3 for every sample count (S <= 16) holds
// the exact IEEE quotients of psc3d.py:88, computed once per block.
//
// The gathers are latency-bound: an entry's five loads (count, alpha sum,
// three IMB components) go to cells spread over its bounding box, and with
// the loads of one pass per thread in flight the kernel kept DRAM at 13 % of
// its bandwidth (ncu: 55 % of stalls on long scoreboard).  So each thread
// copies the data of its entries LOAD_STAGES - 1 passes ahead into its own
// shared-memory slots (cp.async, no registers held) and computes from there;
// the arithmetic and its order per thread are those of a one-entry loop.
// On the 24-window batch (57.5 M entries) the all-windows chunk kernel took
// 504 us with four stages against 581 us with the loads in registers; three
// stages ran as fast as four, two slower than none.  What is left is issue-
// and conversion-bound (FP64 division and conversions per entry): exact
// integer-path conversions cut the conversion-unit load but added more
// instructions than they saved.
#ifndef PSC_LOADS_STAGES
#define PSC_LOADS_STAGES 4
#endif
constexpr int LOAD_STAGES = PSC_LOADS_STAGES;
static_assert(LOAD_STAGES >= 2, "the staging ring needs two slots");
// Resident blocks per SM the register allocation of the chunk kernels aims for.
#ifndef PSC_LOADS_MIN_BLOCKS
#define PSC_LOADS_MIN_BLOCKS 3
#endif

// One block's staging ring, structure of arrays over the threads (thread t
// owns column t of every row: no bank conflicts, no barriers).
template <typename I>
struct LoadRing {
    double alpha[LOAD_STAGES][LOAD_THREADS];
    I imb[LOAD_STAGES][3][LOAD_THREADS];
    uint32_t cnt[LOAD_STAGES][LOAD_THREADS];  // the aligned pair of uint16 counts holding the entry's
};

template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(dst), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}

// This thread's share of one chunk's sums (force, torque).  A thread visits the
// entries e0 + tid, e0 + tid + 256, ...; their bbox coordinates advance by a
// fixed mixed-radix stride with carries (one 32-bit division per chunk).
// s_al holds count / S^3 for every count; cap_entries is the length of
// ent_cnt (the count pairs are read as aligned 32-bit words inside it).
// (The path of a geometry without a loads list.)
template <typename I>
__device__ __forceinline__ void chunk_thread_sums(const ChunkDesc& dsc, const double* particles,
                                                  const uint16_t* ent_cnt, int64_t cap_entries,
                                                  const double* alpha_sum, const I* imb, uint32_t N, uint32_t ny,
                                                  uint32_t nz, const double* s_al, LoadRing<I>& ring,
                                                  double (&acc)[6]) {
    const int64_t e0 = dsc.e0, e1 = dsc.e1;
    const int tid = threadIdx.x;
    if (e0 + tid >= e1) return;
    const double* q = particles + (size_t)dsc.p * PF;
    const uint32_t ey = (uint32_t)dsc.ey, ez = (uint32_t)dsc.ez;
    // bbox-local coordinates of this thread's first entry, and the stride
    const uint32_t local = (uint32_t)dsc.local0 + tid;
    const uint32_t eyz = ey * ez;
    uint32_t a = local / eyz;
    const uint32_t rem = local - a * eyz;
    uint32_t b = rem / ez;
    uint32_t k = rem - b * ez;
    const uint32_t step_k = blockDim.x % ez;
    const uint32_t step_q = blockDim.x / ez;
    const uint32_t step_b = step_q % ey;
    const uint32_t step_a = step_q / ey;
    const uint32_t bx = (uint32_t)dsc.x0, by = (uint32_t)dsc.y0, bz = (uint32_t)dsc.z0;
    // prefetch cursor: entry ep at bbox-local (pa, pb, pk)
    int64_t ep = e0 + tid;
    uint32_t pa = a, pb = b, pk = k;
    auto prefetch = [&](int slot) {
        if (ep < e1) {  // the cell lies in the clipped box, so it exists even where the count is 0
            const uint32_t cell = ((bx + pa) * ny + (by + pb)) * nz + (bz + pk);
            cp_async<8>(&ring.alpha[slot][tid], alpha_sum + cell);
            cp_async<sizeof(I)>(&ring.imb[slot][0][tid], imb + cell);
            cp_async<sizeof(I)>(&ring.imb[slot][1][tid], imb + (size_t)N + cell);
            cp_async<sizeof(I)>(&ring.imb[slot][2][tid], imb + 2 * (size_t)N + cell);
            const int64_t even = ep & ~(int64_t)1;
            if (even + 1 < cap_entries) cp_async<4>(&ring.cnt[slot][tid], ent_cnt + even);
            else ring.cnt[slot][tid] = ent_cnt[ep];  // last entry of the array at an even index
        }
        cp_async_commit();  // one group per pass, empty past the end
        ep += blockDim.x;
        pk += step_k;
        const uint32_t ck = pk >= ez;
        pk -= ck ? ez : 0u;
        pb += step_b + ck;
        const uint32_t cb = pb >= ey;
        pb -= cb ? ey : 0u;
        pa += step_a + cb;
    };
#pragma unroll
    for (int s = 0; s < LOAD_STAGES - 1; ++s) prefetch(s);
    const double qx = q[0], qy = q[1], qz = q[2];
    int slot = 0;
    for (int64_t e = e0 + tid; e < e1; e += blockDim.x) {
        cp_async_wait<LOAD_STAGES - 2>();  // the group of this pass has landed
        const uint32_t pair = ring.cnt[slot][tid];
        const uint32_t cnt = (e & 1) ? pair >> 16 : pair & 0xffffu;
        if (cnt != 0) {
            const double as = ring.alpha[slot][tid];
            const double mx = (double)ring.imb[slot][0][tid];
            const double my = (double)ring.imb[slot][1][tid];
            const double mz = (double)ring.imb[slot][2][tid];
            // owner weight alpha_p / max(alpha_sum, 1e-14)   (psc3d.py:386)
            const double al = s_al[cnt];
            const double ow = xdiv(al, as > 1.0e-14 ? as : 1.0e-14);
            const double nfx = -xmul(ow, mx);
            const double nfy = -xmul(ow, my);
            const double nfz = -xmul(ow, mz);
            // torque arm (i + 0.5) - X, no periodic wrap   (psc3d.py:397-402)
            const double rx = xsub(xadd((double)(bx + a), 0.5), qx);
            const double ry = xsub(xadd((double)(by + b), 0.5), qy);
            const double rz = xsub(xadd((double)(bz + k), 0.5), qz);
            acc[0] += nfx;
            acc[1] += nfy;
            acc[2] += nfz;
            acc[3] += xsub(xmul(ry, nfz), xmul(rz, nfy));
            acc[4] += xsub(xmul(rz, nfx), xmul(rx, nfz));
            acc[5] += xsub(xmul(rx, nfy), xmul(ry, nfx));
        }
        // refill the slot consumed in the previous pass (its values are used above)
        prefetch(slot == 0 ? LOAD_STAGES - 1 : slot - 1);
        slot = slot == LOAD_STAGES - 1 ? 0 : slot + 1;
        // next entry of this thread: (a, b, k) += (step_a, step_b, step_k) with carries
        k += step_k;
        const uint32_t ck = k >= ez;
        k -= ck ? ez : 0u;
        b += step_b + ck;
        const uint32_t cb = b >= ey;
        b -= cb ? ey : 0u;
        a += step_a + cb;
    }
    cp_async_wait<0>();  // nothing in flight into the ring when the next chunk starts
}

// One block per chunk of one particle's bbox entries.
template <typename I>
__global__ void __launch_bounds__(LOAD_THREADS, PSC_LOADS_MIN_BLOCKS) k_loads_chunks(psc_geometry g, const I* imb,
                                                                                 double* part) {
    __shared__ ChunkRing rows;
    __shared__ LoadRing<I> ring;
    extern __shared__ double s_al[];  // S^3 + 1 entries (dynamic)
    const int64_t C = g.totals[1];
    const uint32_t N = (uint32_t)g.nx * g.ny * g.nz;
    const int S3 = g.subsamples * g.subsamples * g.subsamples;
    const double S3d = (double)S3;
    for (int c = threadIdx.x; c <= S3; c += blockDim.x) s_al[c] = xdiv((double)c, S3d);
    chunk_ring_init(rows);  // (its barrier also publishes s_al)
    long long j = 0;
    for (int64_t chunk = blockIdx.x; chunk < C; chunk += gridDim.x, ++j) {  // every warp, in this order
        // every thread reads the chunk's descriptor before the chunk's last warp overwrites the row
        const ChunkDesc dsc = *reinterpret_cast<const ChunkDesc*>(part + chunk * 6);
        double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        chunk_thread_sums<I>(dsc, g.particles, g.ent_cnt, g.capacity_entries, g.alpha_sum, imb, N, (uint32_t)g.ny,
                             (uint32_t)g.nz, s_al, ring, acc);
        chunk_ring_finish(rows, j, acc, part + chunk * 6);
    }
}

// The list path: the chunk's sums from its loads list (chunk_list_build, run
// by the first loads call on a geometry).  Thread t reduces its slots
// slot0 + k * blockDim.x, k < its count, in order; gone are the zero-count
// entries, the count and alpha-sum gathers and the FP64 division.
//
// The gathers are latency-bound, so a chunk is staged in two asynchronous
// copies into the thread's own shared-memory column (cp.async, no registers
// held, no barrier: a thread reads only what it copied): first every list
// entry of the thread (weight and cell), then the IMB momentum of those cells;
// the next chunk's descriptor and counts are loaded meanwhile.  Two memory
// round trips per chunk instead of one per dependent load.
constexpr int LIST_STAGE_K = 6;  // list entries per thread staged at a time (a column holds up to 16: three passes)
static_assert(LOAD_THREADS == PSC_LOAD_THREADS, "the loads list layout assumes PSC_LOAD_THREADS threads per chunk");

template <typename I>
constexpr size_t list_stage_bytes() {
    return (size_t)LIST_STAGE_K * LOAD_THREADS * (sizeof(double) + sizeof(uint32_t) + 3 * sizeof(I));
}

struct ListCursor {
    ChunkDesc dsc;
    uint32_t n_t;
};

// Asynchronous copy of list entries k0 .. k0 + m - 1 of this thread's column
// (weight and cell) into its stage slots 0 .. m - 1.
__device__ __forceinline__ void list_issue(int64_t slot0, const double* lw, const uint32_t* labk, uint32_t k0,
                                           uint32_t m, unsigned char* stage) {
    const int t = threadIdx.x;
    double* s_w = reinterpret_cast<double*>(stage);
    uint32_t* s_abk = reinterpret_cast<uint32_t*>(s_w + LIST_STAGE_K * LOAD_THREADS);
    const int64_t stride = blockDim.x;
    for (uint32_t k = 0; k < m; ++k) {
        cp_async<8>(&s_w[k * LOAD_THREADS + t], lw + slot0 + (int64_t)(k0 + k) * stride);
        cp_async<4>(&s_abk[k * LOAD_THREADS + t], labk + slot0 + (int64_t)(k0 + k) * stride);
    }
    cp_async_commit();
}

__device__ __forceinline__ uint32_t list_pass_size(uint32_t n_t, uint32_t k0) {
    return n_t - k0 < (uint32_t)LIST_STAGE_K ? n_t - k0 : (uint32_t)LIST_STAGE_K;
}

// One chunk's sums of this thread from its list column, LIST_STAGE_K entries
// at a time, in list order.  The first pass's list copy was issued already
// (list_issue with k0 = 0); each pass waits for its list entries, copies the
// IMB momentum of their cells, waits again and adds them up.
template <typename I>
__device__ __forceinline__ void list_chunk_sums(const ListCursor& cur, int64_t slot0, const double* particles,
                                                const double* lw, const uint32_t* labk, const I* imb, uint32_t N,
                                                uint32_t ny, uint32_t nz, unsigned char* stage, double (&acc)[6]) {
    const int t = threadIdx.x;
    const uint32_t n_t = cur.n_t;
    if (n_t == 0) return;
    double* s_w = reinterpret_cast<double*>(stage);
    uint32_t* s_abk = reinterpret_cast<uint32_t*>(s_w + LIST_STAGE_K * LOAD_THREADS);
    I* s_imb = reinterpret_cast<I*>(s_abk + LIST_STAGE_K * LOAD_THREADS);
    const uint32_t bx = (uint32_t)cur.dsc.x0, by = (uint32_t)cur.dsc.y0, bz = (uint32_t)cur.dsc.z0;
    const double* q = particles + (size_t)cur.dsc.p * PF;
    const double qx = q[0], qy = q[1], qz = q[2];
    for (uint32_t k0 = 0; k0 < n_t; k0 += LIST_STAGE_K) {
        const uint32_t m = list_pass_size(n_t, k0);
        if (k0 > 0) list_issue(slot0, lw, labk, k0, m, stage);
        cp_async_wait<0>();
        for (uint32_t k = 0; k < m; ++k) {
            const uint32_t abk = s_abk[k * LOAD_THREADS + t];
            const uint32_t a = abk & 0x7ffu, b = (abk >> 11) & 0x7ffu, kz = abk >> 22;
            const uint32_t cell = ((bx + a) * ny + (by + b)) * nz + (bz + kz);
            cp_async<sizeof(I)>(&s_imb[(k * 3 + 0) * LOAD_THREADS + t], imb + cell);
            cp_async<sizeof(I)>(&s_imb[(k * 3 + 1) * LOAD_THREADS + t], imb + (size_t)N + cell);
            cp_async<sizeof(I)>(&s_imb[(k * 3 + 2) * LOAD_THREADS + t], imb + 2 * (size_t)N + cell);
        }
        cp_async_commit();
        cp_async_wait<0>();
        for (uint32_t k = 0; k < m; ++k) {
            const uint32_t abk = s_abk[k * LOAD_THREADS + t];
            const uint32_t a = abk & 0x7ffu, b = (abk >> 11) & 0x7ffu, kz = abk >> 22;
            const double ow = s_w[k * LOAD_THREADS + t];
            const double nfx = -xmul(ow, (double)s_imb[(k * 3 + 0) * LOAD_THREADS + t]);
            const double nfy = -xmul(ow, (double)s_imb[(k * 3 + 1) * LOAD_THREADS + t]);
            const double nfz = -xmul(ow, (double)s_imb[(k * 3 + 2) * LOAD_THREADS + t]);
            // torque arm (i + 0.5) - X, no periodic wrap   (psc3d.py:397-402)
            const double rx = xsub(xadd((double)(bx + a), 0.5), qx);
            const double ry = xsub(xadd((double)(by + b), 0.5), qy);
            const double rz = xsub(xadd((double)(bz + kz), 0.5), qz);
            acc[0] += nfx;
            acc[1] += nfy;
            acc[2] += nfz;
            acc[3] += xsub(xmul(ry, nfz), xmul(rz, nfy));
            acc[4] += xsub(xmul(rz, nfx), xmul(rx, nfz));
            acc[5] += xsub(xmul(rx, nfy), xmul(ry, nfx));
        }
    }
}

// A chunk's list entries overlap the previous chunk's sums: each thread issues
// the next chunk's first list copy as soon as its own sums are done (its stage
// slots are free then), before its warp's sum.
template <typename I>
__global__ void __launch_bounds__(LOAD_THREADS, 3) k_loads_chunks_list(psc_geometry g, const I* imb, double* part) {
    __shared__ ChunkRing rows;
    extern __shared__ __align__(16) unsigned char list_stage[];
    chunk_ring_init(rows);
    const int64_t C = g.totals[1];
    const uint32_t N = (uint32_t)g.nx * g.ny * g.nz;
    ListCursor cur{};
    int64_t chunk = blockIdx.x;
    if (chunk < C) {
        cur.dsc = *reinterpret_cast<const ChunkDesc*>(part + chunk * 6);
        cur.n_t = g.load_n[chunk * LOAD_THREADS + threadIdx.x];
        list_issue(chunk * g.chunk_entries + threadIdx.x, g.load_w, g.load_abk, 0, list_pass_size(cur.n_t, 0),
                   list_stage);
    }
    for (long long j = 0; chunk < C; chunk += gridDim.x, ++j) {  // every warp, in this order
        // the next chunk's descriptor (its row is overwritten only when this block reduces it) and counts
        const int64_t nxt = chunk + gridDim.x;
        ListCursor nc{};
        if (nxt < C) {
            nc.dsc = *reinterpret_cast<const ChunkDesc*>(part + nxt * 6);
            nc.n_t = g.load_n[nxt * LOAD_THREADS + threadIdx.x];
        }
        double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        list_chunk_sums<I>(cur, chunk * g.chunk_entries + threadIdx.x, g.particles, g.load_w, g.load_abk, imb, N,
                           (uint32_t)g.ny, (uint32_t)g.nz, list_stage, acc);
        if (nxt < C)
            list_issue(nxt * g.chunk_entries + threadIdx.x, g.load_w, g.load_abk, 0, list_pass_size(nc.n_t, 0),
                       list_stage);
        chunk_ring_finish(rows, j, acc, part + chunk * 6);
        cur = nc;
    }
}

// The loads list of one chunk, built warp by warp.  Warp w of the block owns
// the chunk's bbox entries 32w + l + PSC_LOAD_THREADS j (lane l, j <
// chunk_entries / PSC_LOAD_THREADS), visited in that order; its entries with a
// non-zero count are numbered c = 0, 1, ... in that order and dealt round-robin
// to its lanes: entry c goes to slot k = c / 32 of lane c % 32, i.e. list slot
// chunk * chunk_entries + k * PSC_LOAD_THREADS + 32w + c % 32, with its owner
// weight alpha_p / max(alpha_sum, 1e-14) (psc3d.py:386) and its bbox-local
// cell.  So neighbouring lanes reduce neighbouring cells (the IMB gathers of a
// warp touch few lines) and a warp's lanes own counts that differ by at most one.
__device__ __forceinline__ void chunk_list_build(const ChunkDesc& dsc, const uint16_t* ent_cnt, int64_t E,
                                                 const double* alpha_sum, uint32_t ny, uint32_t nz,
                                                 const double* s_al, int32_t chunk_entries, double* lw,
                                                 uint32_t* labk, int64_t slot_chunk, uint8_t* load_n_chunk) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t ey = (uint32_t)dsc.ey, ez = (uint32_t)dsc.ez, eyz = ey * ez;
    const int passes = chunk_entries / LOAD_THREADS;
    const int64_t e1 = min(dsc.e1, E);
    const uint32_t below = (1u << lane) - 1u;  // lanes before this one
    uint32_t base = 0;                          // non-zero entries of the warp so far
#pragma unroll 4
    for (int j = 0; j < passes; ++j) {  // warp-uniform
        const uint32_t off = warp * 32u + lane + (uint32_t)j * LOAD_THREADS;  // entry offset in the chunk
        const int64_t e = dsc.e0 + off;
        const uint32_t cnt = e < e1 ? (uint32_t)ent_cnt[e] : 0u;
        const uint32_t mask = __ballot_sync(0xffffffffu, cnt != 0u);
        if (cnt != 0u) {
            const uint32_t local = (uint32_t)dsc.local0 + off;
            const uint32_t a = local / eyz;
            const uint32_t rem = local - a * eyz;
            const uint32_t b = rem / ez;
            const uint32_t k = rem - b * ez;
            const uint32_t cell = (((uint32_t)dsc.x0 + a) * ny + ((uint32_t)dsc.y0 + b)) * nz + ((uint32_t)dsc.z0 + k);
            const double as = alpha_sum[cell];
            const double ow = xdiv(s_al[cnt], as > 1.0e-14 ? as : 1.0e-14);
            const uint32_t c = base + __popc(mask & below);
            const int64_t slot = slot_chunk + (int64_t)(c >> 5) * LOAD_THREADS + warp * 32u + (c & 31u);
            lw[slot] = ow;
            labk[slot] = a | (b << 11) | (k << 22);
        }
        base += __popc(mask);
    }
    load_n_chunk[warp * 32u + lane] = (uint8_t)(base > lane ? (base - lane + 31u) >> 5 : 0u);
}

// The loads list of every chunk of one geometry (descriptors in the partial rows).
__global__ void __launch_bounds__(LOAD_THREADS) k_loads_list_build(const __grid_constant__ psc_geometry g,
                                                                   const double* part) {
    extern __shared__ double s_al[];  // S^3 + 1 entries (dynamic)
    const int S3 = g.subsamples * g.subsamples * g.subsamples;
    const double S3d = (double)S3;
    for (int c = threadIdx.x; c <= S3; c += blockDim.x) s_al[c] = xdiv((double)c, S3d);
    __syncthreads();
    const int64_t C = g.totals[1];
    const int64_t E = min(g.totals[0], g.capacity_entries);
    for (int64_t chunk = blockIdx.x; chunk < C; chunk += gridDim.x) {
        const ChunkDesc dsc = *reinterpret_cast<const ChunkDesc*>(part + chunk * 6);
        chunk_list_build(dsc, g.ent_cnt, E, g.alpha_sum, (uint32_t)g.ny, (uint32_t)g.nz, s_al, g.chunk_entries,
                         g.load_w, g.load_abk, chunk * g.chunk_entries, g.load_n + chunk * LOAD_THREADS);
    }
}

// The loads lists of the jobs whose list is not current, in one launch.
__global__ void __launch_bounds__(LOAD_THREADS) k_loads_list_build_multi(const LoadsJob* jobs,
                                                                         const int64_t* chunk_base, int njobs,
                                                                         const double* part) {
    extern __shared__ double s_al[];  // S^3 + 1 entries for the largest S of the jobs (dynamic)
    const int64_t C = chunk_base[njobs];
    int cur_S = 0;  // S of the table in s_al (block-uniform: every thread visits the same chunks)
    for (int64_t chunk = blockIdx.x; chunk < C; chunk += gridDim.x) {
        const ChunkDesc dsc = *reinterpret_cast<const ChunkDesc*>(part + chunk * 6);
        const psc_geometry& g = jobs[dsc.pad].g;
        if (g.list_ready) continue;  // block-uniform
        const int S = g.subsamples;
        if (S != cur_S) {
            __syncthreads();  // no thread reads the old table any more
            const int S3 = S * S * S;
            const double S3d = (double)S3;
            for (int c = threadIdx.x; c <= S3; c += blockDim.x) s_al[c] = xdiv((double)c, S3d);
            __syncthreads();
            cur_S = S;
        }
        const int64_t local = chunk - chunk_base[dsc.pad];
        chunk_list_build(dsc, g.ent_cnt, min(g.totals[0], g.capacity_entries), g.alpha_sum, (uint32_t)g.ny,
                         (uint32_t)g.nz, s_al, g.chunk_entries, g.load_w, g.load_abk, local * g.chunk_entries,
                         g.load_n + local * LOAD_THREADS);
    }
}

// Per-particle sums of the chunk partials c0 .. c1-1: one warp per particle,
// lane l sums chunks c0 + l, c0 + l + 32, ... in order, then a fixed shuffle tree.
__device__ __forceinline__ void particle_sums(const double* part, int64_t c0, int64_t c1, double* force,
                                              double* torque) {
    const int lane = threadIdx.x & 31;
    double F[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int64_t c = c0 + lane; c < c1; c += 32) {
#pragma unroll
        for (int k = 0; k < 6; ++k) F[k] += part[c * 6 + k];
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) F[k] += __shfl_xor_sync(0xffffffffu, F[k], o);
    }
    if (lane < 3) {
        force[lane] = F[lane];
        torque[lane] = F[3 + lane];
    }
}

__global__ void __launch_bounds__(256) k_loads_particles(psc_geometry g, const double* part, double* forces,
                                                         double* torques) {
    const int p = (int)(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
    if (p >= g.nparticles) return;  // warp-uniform
    particle_sums(part, g.chunk_off[p], g.chunk_off[p + 1], forces + (size_t)p * 3, torques + (size_t)p * 3);
}

// One block: the closure residual |sum_p F_p + sum_x imb| and the max force /
// torque norms (psc3d.py:247-253, :280-281) from the per-particle loads.
__device__ __forceinline__ void loads_diag_block(int P, const double* imb_sums, const double* forces,
                                                 const double* torques, double* diag) {
    __shared__ double s[32][5];
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // sum Fx, Fy, Fz, max |F|^2, max |T|^2
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        const double* F = forces + (size_t)p * 3;
        const double* T = torques + (size_t)p * 3;
        v[0] += F[0];
        v[1] += F[1];
        v[2] += F[2];
        v[3] = fmax(v[3], F[0] * F[0] + F[1] * F[1] + F[2] * F[2]);
        v[4] = fmax(v[4], T[0] * T[0] + T[1] * T[1] + T[2] * T[2]);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, x, o);
            x = k < 3 ? x + y : fmax(x, y);
        }
        if (lane == 0) s[warp][k] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int w = 0; w < nw; ++w) {
            for (int k = 0; k < 3; ++k) r[k] += s[w][k];
            r[3] = fmax(r[3], s[w][3]);
            r[4] = fmax(r[4], s[w][4]);
        }
        const double cx = r[0] + imb_sums[0], cy = r[1] + imb_sums[1], cz = r[2] + imb_sums[2];
        diag[PSC_DIAG_MOMENTUM_RESIDUAL] = sqrt(cx * cx + cy * cy + cz * cz);
        diag[PSC_DIAG_MAX_FORCE] = sqrt(r[3]);
        diag[PSC_DIAG_MAX_TORQUE] = sqrt(r[4]);
        diag[PSC_DIAG_FORCE_SUM_X] = r[0];
        diag[PSC_DIAG_FORCE_SUM_Y] = r[1];
        diag[PSC_DIAG_FORCE_SUM_Z] = r[2];
    }
}

__global__ void __launch_bounds__(1024) k_loads_diag(psc_geometry g, const double* imb_sums, const double* forces,
                                                     const double* torques, double* diag) {
    loads_diag_block(g.nparticles, imb_sums, forces, torques, diag);
}

// ---------------------------------------------------------------------------
// particle loads of many windows in one launch sequence
// ---------------------------------------------------------------------------
// The chunks of all jobs form one index space (job k owns chunks
// chunk_base[k] .. chunk_base[k+1]-1, its particles particle_base[k] ..),
// so the small windows of a batch fill the GPU together instead of one
// launch each.  Every per-chunk, per-particle and per-window sum runs the
// single-window arithmetic in the same order: the results are bitwise those
// of one launch_particle_loads per window.

__global__ void __launch_bounds__(256) k_chunk_desc_multi(const LoadsJob* jobs, const int64_t* chunk_base, int njobs,
                                                          double* part) {
    const int64_t C = chunk_base[njobs];
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C; c += (int64_t)gridDim.x * blockDim.x) {
        const int k = owner_of(chunk_base, njobs, c);
        ChunkDesc d = make_chunk_desc(jobs[k].g, c - chunk_base[k]);
        d.pad = k;  // the chunk's job
        *reinterpret_cast<ChunkDesc*>(part + c * 6) = d;
    }
}

template <typename I>
__global__ void __launch_bounds__(LOAD_THREADS, PSC_LOADS_MIN_BLOCKS)
    k_loads_chunks_multi(const LoadsJob* jobs, const int64_t* chunk_base, int njobs, double* part) {
    __shared__ ChunkRing rows;
    __shared__ LoadRing<I> ring;
    extern __shared__ double s_al[];  // S^3 + 1 entries for the largest S of the jobs (dynamic)
    chunk_ring_init(rows);
    const int64_t C = chunk_base[njobs];
    int cur_S = 0;  // S of the table in s_al (the same in every warp: all visit the same chunks)
    long long j = 0;
    for (int64_t chunk = blockIdx.x; chunk < C; chunk += gridDim.x, ++j) {  // every warp, in this order
        const ChunkDesc dsc = *reinterpret_cast<const ChunkDesc*>(part + chunk * 6);
        const psc_geometry& g = jobs[dsc.pad].g;
        const int S = g.subsamples;
        if (S != cur_S) {  // every warp at the same chunk: the barriers are block-uniform
            __syncthreads();  // no warp reads the old table any more
            const int S3 = S * S * S;
            const double S3d = (double)S3;
            for (int c = threadIdx.x; c <= S3; c += blockDim.x) s_al[c] = xdiv((double)c, S3d);
            __syncthreads();
            cur_S = S;
        }
        double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        chunk_thread_sums<I>(dsc, g.particles, g.ent_cnt, g.capacity_entries, g.alpha_sum,
                             reinterpret_cast<const I*>(jobs[dsc.pad].imb), (uint32_t)g.nx * g.ny * g.nz,
                             (uint32_t)g.ny, (uint32_t)g.nz, s_al, ring, acc);
        chunk_ring_finish(rows, j, acc, part + chunk * 6);
    }
}

// The list path for many windows: every job's loads list is current.
template <typename I>
__global__ void __launch_bounds__(LOAD_THREADS, 3) k_loads_chunks_list_multi(const LoadsJob* jobs,
                                                                           const int64_t* chunk_base, int njobs,
                                                                           double* part) {
    __shared__ ChunkRing rows;
    extern __shared__ __align__(16) unsigned char list_stage[];
    chunk_ring_init(rows);
    const int64_t C = chunk_base[njobs];
    ListCursor cur{};
    int64_t chunk = blockIdx.x;
    if (chunk < C) {
        cur.dsc = *reinterpret_cast<const ChunkDesc*>(part + chunk * 6);
        const psc_geometry& g0 = jobs[cur.dsc.pad].g;
        const int64_t local0 = chunk - chunk_base[cur.dsc.pad];
        cur.n_t = g0.load_n[local0 * LOAD_THREADS + threadIdx.x];
        list_issue(local0 * g0.chunk_entries + threadIdx.x, g0.load_w, g0.load_abk, 0, list_pass_size(cur.n_t, 0),
                   list_stage);
    }
    for (long long j = 0; chunk < C; chunk += gridDim.x, ++j) {  // every warp, in this order
        const int64_t nxt = chunk + gridDim.x;
        ListCursor nc{};
        if (nxt < C) {
            nc.dsc = *reinterpret_cast<const ChunkDesc*>(part + nxt * 6);
            nc.n_t = jobs[nc.dsc.pad].g.load_n[(nxt - chunk_base[nc.dsc.pad]) * LOAD_THREADS + threadIdx.x];
        }
        const LoadsJob& J = jobs[cur.dsc.pad];
        const int64_t local = chunk - chunk_base[cur.dsc.pad];
        double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        list_chunk_sums<I>(cur, local * J.g.chunk_entries + threadIdx.x, J.g.particles, J.g.load_w, J.g.load_abk,
                           reinterpret_cast<const I*>(J.imb), (uint32_t)J.g.nx * J.g.ny * J.g.nz, (uint32_t)J.g.ny,
                           (uint32_t)J.g.nz, list_stage, acc);
        if (nxt < C) {  // the next chunk's first list copy, overlapping this chunk's warp sums
            const psc_geometry& gn = jobs[nc.dsc.pad].g;
            list_issue((nxt - chunk_base[nc.dsc.pad]) * gn.chunk_entries + threadIdx.x, gn.load_w, gn.load_abk, 0,
                       list_pass_size(nc.n_t, 0), list_stage);
        }
        chunk_ring_finish(rows, j, acc, part + chunk * 6);
        cur = nc;
    }
}

__global__ void __launch_bounds__(256) k_loads_particles_multi(const LoadsJob* jobs, const int64_t* chunk_base,
                                                               const int64_t* particle_base, int njobs,
                                                               const double* part) {
    const int64_t gp = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (gp >= particle_base[njobs]) return;  // warp-uniform
    const int k = owner_of(particle_base, njobs, gp);
    const LoadsJob& J = jobs[k];
    const int p = (int)(gp - particle_base[k]);
    particle_sums(part + chunk_base[k] * 6, J.g.chunk_off[p], J.g.chunk_off[p + 1], J.forces + (size_t)p * 3,
                  J.torques + (size_t)p * 3);
}

__global__ void __launch_bounds__(1024) k_loads_diag_multi(const LoadsJob* jobs) {
    const LoadsJob& J = jobs[blockIdx.x];
    loads_diag_block(J.g.nparticles, J.imb_sums, J.forces, J.torques, J.diag);
}

// ---------------------------------------------------------------------------
// exclusive scan (int32), three passes over blocks of SCAN_ITEMS elements
// ---------------------------------------------------------------------------
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_PER_THREAD = 8;
constexpr int SCAN_ITEMS = SCAN_THREADS * SCAN_PER_THREAD;

size_t scan_tmp_bytes(int64_t n) {
    const int64_t nb = (n + SCAN_ITEMS - 1) / SCAN_ITEMS;
    return (size_t)(nb + 1) * sizeof(int32_t) + 256;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_partial(const int32_t* in, int64_t n, int32_t* bsum) {
    __shared__ int32_t s_warp[32];
    const int64_t base = (int64_t)blockIdx.x * SCAN_ITEMS + (int64_t)threadIdx.x * SCAN_PER_THREAD;
    int32_t acc = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER_THREAD; ++k)
        if (base + k < n) acc += in[base + k];
    int32_t total;
    block_exclusive_scan<int32_t>(acc, s_warp, total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_top(int32_t* bsum, int64_t nb) {
    __shared__ int32_t s_warp[32];
    __shared__ int32_t s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < nb; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const int32_t v = i < nb ? bsum[i] : 0;
        int32_t total;
        const int32_t ex = block_exclusive_scan<int32_t>(v, s_warp, total);
        if (i < nb) bsum[i] = s_carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) s_carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) bsum[nb] = s_carry;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_apply(const int32_t* in, int32_t* out, int64_t n,
                                                             const int32_t* bsum, int64_t nb) {
    __shared__ int32_t s_warp[32];
    const int64_t base = (int64_t)blockIdx.x * SCAN_ITEMS + (int64_t)threadIdx.x * SCAN_PER_THREAD;
    int32_t v[SCAN_PER_THREAD];
    int32_t acc = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER_THREAD; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        acc += v[k];
    }
    int32_t total;
    int32_t run = block_exclusive_scan<int32_t>(acc, s_warp, total) + bsum[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_PER_THREAD; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = bsum[nb];
}

cudaError_t scan_exclusive_i32(const int32_t* in, int32_t* out, int64_t n, void* tmp, cudaStream_t stream) {
    const int64_t nb = (n + SCAN_ITEMS - 1) / SCAN_ITEMS;
    int32_t* bsum = reinterpret_cast<int32_t*>(tmp);
    if (nb == 0) {
        return cudaMemsetAsync(out, 0, sizeof(int32_t), stream);
    }
    k_scan_partial<<<(unsigned)nb, SCAN_THREADS, 0, stream>>>(in, n, bsum);
    k_scan_top<<<1, 1024, 0, stream>>>(bsum, nb);
    k_scan_apply<<<(unsigned)nb, SCAN_THREADS, 0, stream>>>(in, out, n, bsum, nb);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static unsigned grid_cap(int64_t work, int threads) {
    int64_t gsz = (work + threads - 1) / threads;
    const int64_t cap = (int64_t)sm_count() * 32;
    if (gsz > cap) gsz = cap;
    if (gsz < 1) gsz = 1;
    return (unsigned)gsz;
}

cudaError_t launch_geometry_plan(const psc_geometry& g, cudaStream_t stream) {
    k_geometry_plan<<<1, 1024, 0, stream>>>(g);
    return cudaGetLastError();
}

cudaError_t launch_geometry_build(const psc_geometry& g, cudaStream_t stream) {
    const int64_t N = (int64_t)g.nx * g.ny * g.nz;
    cudaError_t e = cudaMemsetAsync(g.cell_n, 0, (size_t)N * sizeof(int32_t), stream);
    if (e != cudaSuccess) return e;
    if (g.capacity_entries > 0) {
        const unsigned grid = grid_cap(g.capacity_entries, g.chunk_entries > 0 ? g.chunk_entries : 4096);  // ~ one block per chunk
        switch (g.smooth_eps > 0.0 ? 0 : g.subsamples) {  // the count kernel for a compile-time S
            case 1: k_geometry_count<1><<<grid, 256, 0, stream>>>(g); break;
            case 2: k_geometry_count<2><<<grid, 256, 0, stream>>>(g); break;
            case 3: k_geometry_count<3><<<grid, 256, 0, stream>>>(g); break;
            case 4: k_geometry_count<4><<<grid, 256, 0, stream>>>(g); break;
            case 5: k_geometry_count<5><<<grid, 256, 0, stream>>>(g); break;
            case 6: k_geometry_count<6><<<grid, 256, 0, stream>>>(g); break;
            default: k_geometry_count<0><<<grid, 256, 0, stream>>>(g); break;
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if ((e = scan_exclusive_i32(g.cell_n, g.cell_off, N, g.scan_tmp, stream)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(g.cell_n, 0, (size_t)N * sizeof(int32_t), stream)) != cudaSuccess) return e;
    if (g.capacity_entries > 0) {
        k_geometry_fill<<<grid_cap(g.capacity_entries, g.chunk_entries > 0 ? g.chunk_entries : 4096), 256, 0,
                          stream>>>(g);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    k_geometry_final<<<grid_cap(N, 256), 256, 0, stream>>>(g);
    return cudaGetLastError();
}

cudaError_t read_loads_status(int* out, bool clear) {
    cudaError_t e = cudaMemcpyFromSymbol(out, g_loads_status, sizeof(int));
    if (e != cudaSuccess || !clear) return e;
    const int zero = 0;
    return cudaMemcpyToSymbol(g_loads_status, &zero, sizeof(int));
}

cudaError_t launch_solid_velocity(const psc_geometry& g, int us_type, void* us, cudaStream_t stream) {
    const int64_t N = (int64_t)g.nx * g.ny * g.nz;
    if (us_type == 0) k_solid_velocity<double><<<grid_cap(N, 256), 256, 0, stream>>>(g, reinterpret_cast<double*>(us));
    else k_solid_velocity<float><<<grid_cap(N, 256), 256, 0, stream>>>(g, reinterpret_cast<float*>(us));
    return cudaGetLastError();
}

// The chunk kernels hold a static staging ring and a dynamic count table of
// up to 16^3 + 1 doubles; for FP64 fields the sum can pass the default 48 KB
// of shared memory per block, so every device gets the opt-in once.
static cudaError_t loads_smem_optin() {
    constexpr int kMaxDev = 64;
    static int done[kMaxDev];  // benign race: setting the attribute twice is harmless
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDev || done[dev]) return e;
    const int lut = (16 * 16 * 16 + 1) * (int)sizeof(double);
    if ((e = cudaFuncSetAttribute(k_loads_chunks_list<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)list_stage_bytes<float>())) ||
        (e = cudaFuncSetAttribute(k_loads_chunks_list<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)list_stage_bytes<double>())) ||
        (e = cudaFuncSetAttribute(k_loads_chunks_list_multi<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)list_stage_bytes<float>())) ||
        (e = cudaFuncSetAttribute(k_loads_chunks_list_multi<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)list_stage_bytes<double>())) ||
        (e = cudaFuncSetAttribute(k_loads_chunks<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, lut)) ||
        (e = cudaFuncSetAttribute(k_loads_chunks<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, lut)) ||
        (e = cudaFuncSetAttribute(k_loads_chunks_multi<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, lut)) ||
        (e = cudaFuncSetAttribute(k_loads_chunks_multi<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, lut)))
        return e;
    done[dev] = 1;
    return cudaSuccess;
}

cudaError_t launch_particle_loads(const psc_geometry& g, int imb_type, const void* imb, double* chunk_partials,
                                  const double* imb_sums, double* forces, double* torques, double* diag,
                                  cudaStream_t stream) {
    if (g.capacity_chunks > 0 && g.nparticles > 0) {
        const int64_t cap = (int64_t)sm_count() * 16;
        const unsigned grid = (unsigned)(g.capacity_chunks < cap ? g.capacity_chunks : cap);
        const size_t lut = (size_t)(g.subsamples * g.subsamples * g.subsamples + 1) * sizeof(double);
        const int64_t cg = (g.capacity_chunks + 255) / 256;
        cudaError_t e0 = loads_smem_optin();
        if (e0 != cudaSuccess) return e0;
        k_chunk_desc<<<(unsigned)(cg < cap ? cg : cap), 256, 0, stream>>>(g, chunk_partials);
        if (g.load_w && g.load_abk && g.load_n) {  // the list path: the list first, unless it is current
            if (!g.list_ready) k_loads_list_build<<<grid, LOAD_THREADS, lut, stream>>>(g, chunk_partials);
            if (imb_type == 0)
                k_loads_chunks_list<double><<<grid, LOAD_THREADS, list_stage_bytes<double>(), stream>>>(
                    g, reinterpret_cast<const double*>(imb), chunk_partials);
            else
                k_loads_chunks_list<float><<<grid, LOAD_THREADS, list_stage_bytes<float>(), stream>>>(
                    g, reinterpret_cast<const float*>(imb), chunk_partials);
        } else if (imb_type == 0) {  // no loads list: the whole boxes
            k_loads_chunks<double><<<grid, LOAD_THREADS, lut, stream>>>(g, reinterpret_cast<const double*>(imb),
                                                                        chunk_partials);
        } else {
            k_loads_chunks<float><<<grid, LOAD_THREADS, lut, stream>>>(g, reinterpret_cast<const float*>(imb),
                                                                       chunk_partials);
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (g.nparticles > 0) {
        k_loads_particles<<<(g.nparticles + 7) / 8, 256, 0, stream>>>(g, chunk_partials, forces, torques);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    k_loads_diag<<<1, 1024, 0, stream>>>(g, imb_sums, forces, torques, diag);
    return cudaGetLastError();
}

cudaError_t launch_particle_loads_multi(const LoadsJob* d_jobs, const int64_t* d_chunk_base,
                                        const int64_t* d_particle_base, int njobs, int64_t total_chunks,
                                        int64_t total_particles, int imb_type, int max_subsamples,
                                        bool all_lists, bool list_ready, double* part, cudaStream_t stream) {
    if (njobs <= 0) return cudaSuccess;
    const int64_t cap = (int64_t)sm_count() * 16;
    if (total_chunks > 0) {
        const int64_t cg = (total_chunks + 255) / 256;
        cudaError_t e0 = loads_smem_optin();
        if (e0 != cudaSuccess) return e0;
        k_chunk_desc_multi<<<(unsigned)(cg < cap ? cg : cap), 256, 0, stream>>>(d_jobs, d_chunk_base, njobs, part);
        const unsigned grid = (unsigned)(total_chunks < cap ? total_chunks : cap);
        const size_t lut = (size_t)(max_subsamples * max_subsamples * max_subsamples + 1) * sizeof(double);
        // every job has a loads list: the lists that are not current first, then the list path
        if (all_lists && !list_ready)
            k_loads_list_build_multi<<<grid, LOAD_THREADS, lut, stream>>>(d_jobs, d_chunk_base, njobs, part);
        if (all_lists && imb_type == 0)
            k_loads_chunks_list_multi<double><<<grid, LOAD_THREADS, list_stage_bytes<double>(), stream>>>(
                d_jobs, d_chunk_base, njobs, part);
        else if (all_lists)
            k_loads_chunks_list_multi<float><<<grid, LOAD_THREADS, list_stage_bytes<float>(), stream>>>(
                d_jobs, d_chunk_base, njobs, part);
        else if (imb_type == 0)
            k_loads_chunks_multi<double><<<grid, LOAD_THREADS, lut, stream>>>(d_jobs, d_chunk_base, njobs, part);
        else
            k_loads_chunks_multi<float><<<grid, LOAD_THREADS, lut, stream>>>(d_jobs, d_chunk_base, njobs, part);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (total_particles > 0) {
        k_loads_particles_multi<<<(unsigned)((total_particles + 7) / 8), 256, 0, stream>>>(
            d_jobs, d_chunk_base, d_particle_base, njobs, part);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    k_loads_diag_multi<<<(unsigned)njobs, 1024, 0, stream>>>(d_jobs);
    return cudaGetLastError();
}

}  // namespace psc
