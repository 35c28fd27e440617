// GPU check of xdiv_r (csrc/d3q19.cuh) against __ddiv_rn, bit for bit.
// Built by tests/test_gpu_exact_div.py with nvcc for sm_100a; test helper only.
#include <cstdint>

#include <cuda_runtime.h>

#include "d3q19.cuh"

namespace {

__device__ __forceinline__ uint64_t mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// x_i: random sign and significand, exponent uniform in [emin, emax].
__global__ void k_div_random(double y, uint64_t n, uint64_t seed, int emin, int emax, unsigned long long* bad,
                             double* first) {
    const psc::Divisor d = psc::make_divisor(y);
    const uint64_t span = (uint64_t)(emax - emin + 1);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned long long mine = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t r = mix(seed + 0x9e3779b97f4a7c15ull * (2 * i + 1));
        const uint64_t e = (uint64_t)(emin + 1023 + (int64_t)(mix(r + 0x632be59bd9b4e019ull) % span));
        const double x = __longlong_as_double((long long)((r & 0x800fffffffffffffull) | (e << 52)));
        const double a = psc::xdiv_d(x, d);
        const double b = __ddiv_rn(x, y);
        if (__double_as_longlong(a) != __double_as_longlong(b)) {
            if (mine == 0) *first = x;  // any one of them
            ++mine;
        }
    }
    if (mine) atomicAdd(bad, mine);
}

__global__ void k_div_list(double y, const double* xs, int n, double* out, double* ref) {
    const psc::Divisor d = psc::make_divisor(y);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        out[i] = psc::xdiv_d(xs[i], d);
        ref[i] = __ddiv_rn(xs[i], y);
    }
}

}  // namespace

extern "C" {

// Number of x (of n random ones) whose xdiv_r result differs from __ddiv_rn; -1 on a CUDA error.
long long div_check_gpu(double y, unsigned long long n, unsigned long long seed, int emin, int emax,
                        double* h_first) {
    unsigned long long* bad = nullptr;
    double* first = nullptr;
    if (cudaMalloc(&bad, sizeof(*bad)) != cudaSuccess) return -1;
    if (cudaMalloc(&first, sizeof(*first)) != cudaSuccess) return -1;
    cudaMemset(bad, 0, sizeof(*bad));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    k_div_random<<<sms * 8, 256>>>(y, n, seed, emin, emax, bad, first);
    unsigned long long h_bad = 0;
    cudaError_t e = cudaMemcpy(&h_bad, bad, sizeof(h_bad), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && h_bad && h_first) e = cudaMemcpy(h_first, first, sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(bad);
    cudaFree(first);
    return e == cudaSuccess ? (long long)h_bad : -1;
}

// out[i] = xdiv_r path, ref[i] = __ddiv_rn for host arrays xs[n]; 0 or -1 on a CUDA error.
int div_list_gpu(double y, const double* h_xs, int n, double* h_out, double* h_ref) {
    double *xs = nullptr, *out = nullptr, *ref = nullptr;
    const size_t b = (size_t)n * sizeof(double);
    if (cudaMalloc(&xs, b) != cudaSuccess || cudaMalloc(&out, b) != cudaSuccess || cudaMalloc(&ref, b) != cudaSuccess)
        return -1;
    cudaMemcpy(xs, h_xs, b, cudaMemcpyHostToDevice);
    k_div_list<<<1, 256>>>(y, xs, n, out, ref);
    cudaError_t e = cudaMemcpy(h_out, out, b, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(h_ref, ref, b, cudaMemcpyDeviceToHost);
    cudaFree(xs);
    cudaFree(out);
    cudaFree(ref);
    return e == cudaSuccess ? 0 : -1;
}

}  // extern "C"
