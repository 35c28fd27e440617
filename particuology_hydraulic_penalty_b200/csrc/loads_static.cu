// Particle force / torque for callers that cannot allocate device memory.
//
// psc_particle_loads() reduces each particle's IMB momentum in chunks and
// needs a caller-provided buffer for the per-chunk partial sums.  Some
// callers have no way to provide one: a solver embedded in another program
// that owns the whole device memory budget (for example a DEM code's coupling
// hook that only receives the IMB field and the particle arrays), or a
// coupling loop that must not call cudaMalloc after start-up because an
// allocation there synchronises the device and stalls the exchange.
// psc_particle_loads_static() computes the same loads with the partial sums
// kept in a fixed array inside this library instead.
//
// The array is a file-scope static __device__ buffer of
// PSC_LOADS_STATIC_MAX_CHUNKS x 6 doubles (768 KiB); every GPU that loads the
// library holds it until the process exits.  Its device address is looked up
// once per device (cudaGetSymbolAddress) on the first call made while that
// device is current, so make that first call before any stream capture.
// All calls share the one array: each call writes every partial it later
// reads (nothing has to start at zero), and calls that overlap on the GPU --
// two streams, or two host threads -- race on it and must be serialised.
#include <mutex>

#include "collide.cuh"
#include "internal.cuh"

namespace psc {
namespace {

constexpr int64_t kMaxChunks = PSC_LOADS_STATIC_MAX_CHUNKS;
constexpr int kMaxDevices = 64;
constexpr int kThreads = 256;

static __device__ __align__(256) double g_loads_scratch[kMaxChunks * 6];

double* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

// Device address of g_loads_scratch on the current device (looked up once).
cudaError_t scratch_address(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_loads_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

__device__ __forceinline__ int chunk_owner(const int64_t* off, int P, int64_t c) {
    int lo = 0, hi = P - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= c) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Same per-entry terms as the caller-scratch kernels: owner weight
// alpha_p / max(alpha_sum, 1e-14), node force -w * imb, torque arm
// (i + 0.5) - X without periodic wrap (src/lbm_dem/psc3d.py:375-407).
template <typename I>
__global__ void __launch_bounds__(kThreads) k_static_chunks(psc_geometry g, const I* imb, double* part,
                                                             int64_t max_chunks) {
    __shared__ double s[kThreads / 32][6];
    const int64_t C = min(g.totals[1], max_chunks);
    const uint32_t N = (uint32_t)g.nx * g.ny * g.nz;
    const double S3d = (double)(g.subsamples * g.subsamples * g.subsamples);
    for (int64_t chunk = blockIdx.x; chunk < C; chunk += gridDim.x) {
        const int p = chunk_owner(g.chunk_off, g.nparticles, chunk);
        const int64_t e0 = g.ent_off[p] + (chunk - g.chunk_off[p]) * g.chunk_entries;
        const int64_t e1 = min(e0 + (int64_t)g.chunk_entries, g.ent_off[p + 1]);
        const double* q = g.particles + (size_t)p * 10;
        const int32_t* bb = g.bbox + (size_t)p * 6;
        const int64_t eyz = (int64_t)bb[4] * bb[5];
        double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
            const uint16_t cnt = g.ent_cnt[e];
            if (cnt == 0) continue;
            const int64_t local = e - g.ent_off[p];
            const int32_t a = (int32_t)(local / eyz);
            const int64_t rem = local - (int64_t)a * eyz;
            const int32_t b = (int32_t)(rem / bb[5]);
            const int32_t k = (int32_t)(rem - (int64_t)b * bb[5]);
            const int32_t ix = bb[0] + a, iy = bb[1] + b, iz = bb[2] + k;
            const uint32_t cell = ((uint32_t)ix * g.ny + iy) * g.nz + iz;
            const double al = xdiv((double)cnt, S3d);
            const double as = g.alpha_sum[cell];
            const double ow = xdiv(al, as > 1.0e-14 ? as : 1.0e-14);
            const double nfx = -xmul(ow, (double)imb[cell]);
            const double nfy = -xmul(ow, (double)imb[(size_t)N + cell]);
            const double nfz = -xmul(ow, (double)imb[2 * (size_t)N + cell]);
            const double rx = xsub(xadd((double)ix, 0.5), q[0]);
            const double ry = xsub(xadd((double)iy, 0.5), q[1]);
            const double rz = xsub(xadd((double)iz, 0.5), q[2]);
            acc[0] += nfx;
            acc[1] += nfy;
            acc[2] += nfz;
            acc[3] += xsub(xmul(ry, nfz), xmul(rz, nfy));
            acc[4] += xsub(xmul(rz, nfx), xmul(rx, nfz));
            acc[5] += xsub(xmul(rx, nfy), xmul(ry, nfx));
        }
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
        for (int v = 0; v < 6; ++v) {
            double x = acc[v];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (lane == 0) s[warp][v] = x;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll
            for (int v = 0; v < 6; ++v) {
                double t = 0.0;
                for (int w = 0; w < nw; ++w) t += s[w][v];
                part[chunk * 6 + v] = t;
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(1024) k_static_final(psc_geometry g, const double* part, int64_t max_chunks,
                                                       const double* imb_sums, double* forces, double* torques,
                                                       double* diag) {
    __shared__ double s[32][5];
    const int P = g.nparticles;
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        double F[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        const int64_t c1 = min(g.chunk_off[p + 1], max_chunks);
        for (int64_t c = g.chunk_off[p]; c < c1; ++c) {
#pragma unroll
            for (int k = 0; k < 6; ++k) F[k] += part[c * 6 + k];
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            forces[(size_t)p * 3 + k] = F[k];
            torques[(size_t)p * 3 + k] = F[3 + k];
        }
        v[0] += F[0];
        v[1] += F[1];
        v[2] += F[2];
        v[3] = fmax(v[3], F[0] * F[0] + F[1] * F[1] + F[2] * F[2]);
        v[4] = fmax(v[4], F[3] * F[3] + F[4] * F[4] + F[5] * F[5]);
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

}  // namespace
}  // namespace psc

using namespace psc;

extern "C" int psc_particle_loads_static(const psc_geometry* h_geo, int imb_type, const void* imb,
                                         const double* imb_sums, double* forces, double* torques, double* diag,
                                         void* stream) {
    if (!h_geo) return fail(PSC_E_INVALID, "psc_particle_loads_static: null geometry");
    const psc_geometry& g = *h_geo;
    if (g.nx <= 0 || g.ny <= 0 || g.nz <= 0 || (int64_t)g.nx * g.ny * g.nz >= (1ll << 31))
        return fail(PSC_E_INVALID, "psc_particle_loads_static: bad lattice extents");
    if (g.subsamples < 1 || g.subsamples > 16 || g.nparticles < 0 || g.chunk_entries <= 0)
        return fail(PSC_E_INVALID, "psc_particle_loads_static: bad geometry fields");
    if (imb_type != 0 && imb_type != 1)
        return fail(PSC_E_INVALID, "psc_particle_loads_static: imb_type must be 0 (double) or 1 (float)");
    if (!imb_sums || !diag || !g.ent_off || !g.chunk_off || !g.totals)
        return fail(PSC_E_INVALID, "psc_particle_loads_static: null array");
    if (g.capacity_chunks > kMaxChunks)
        return fail(PSC_E_CAPACITY, "psc_particle_loads_static: the geometry allows " +
                                        std::to_string(g.capacity_chunks) + " load chunks; the built-in scratch holds " +
                                        std::to_string(kMaxChunks) + " (use psc_particle_loads with your own buffer)");
    if (g.nparticles > 0 && (!imb || !forces || !torques || !g.ent_cnt || !g.alpha_sum || !g.particles || !g.bbox))
        return fail(PSC_E_INVALID, "psc_particle_loads_static: null array");
    double* part = nullptr;
    cudaError_t e = scratch_address(&part);
    if (e != cudaSuccess) return cuda_fail(e, "psc_particle_loads_static: scratch address");
    const cudaStream_t s = as_stream(stream);
    // the kernels never read more chunks than the geometry's declared capacity
    const int64_t cap = g.capacity_chunks;
    if (cap > 0 && g.nparticles > 0) {
        const int64_t most = (int64_t)sm_count() * 8;
        const unsigned grid = (unsigned)(cap < most ? cap : most);
        if (imb_type == 0)
            k_static_chunks<double><<<grid, kThreads, 0, s>>>(g, static_cast<const double*>(imb), part, cap);
        else
            k_static_chunks<float><<<grid, kThreads, 0, s>>>(g, static_cast<const float*>(imb), part, cap);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "psc_particle_loads_static");
    }
    k_static_final<<<1, 1024, 0, s>>>(g, part, cap, imb_sums, forces, torques, diag);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "psc_particle_loads_static");
    return PSC_OK;
}
