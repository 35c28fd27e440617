// Internal declarations shared by the .cu translation units of libpscb200.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>

#include <string>

#include "../../include/psc_b200.h"

namespace psc {

// Thread-local last-error slot behind psc_last_error(), and the number of
// errors set on this thread (a handle copies the message when it changes).
void set_error(const std::string& msg);
uint64_t error_seq();
const std::string& last_error_string();
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t err, const char* what);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Number of SMs of the current device (cached per device).
int sm_count();

constexpr int STEP_THREADS = 256;
constexpr int MAX_SMEM_WINDOWS = 256;

// launchers (return cudaError_t of the launch)
cudaError_t launch_step(int store, const psc_window* d_windows, int nwin, int64_t total_tiles, unsigned flags,
                        bool moving, int grid_ctas, cudaStream_t stream);
cudaError_t launch_step_fast(int store, const psc_window* d_windows, int nwin, int64_t total_tiles, unsigned flags,
                             bool moving, int cpt, int grid_ctas, cudaStream_t stream);
cudaError_t launch_step_tma(int store, const psc_window* d_windows, int nwin, int64_t total_tiles, unsigned flags,
                            bool moving, int grid_ctas, int stages, uint32_t stage_bytes, cudaStream_t stream);
cudaError_t launch_step_pair(int store, const psc_window* d_windows, int nwin, int64_t total_tiles, unsigned flags,
                             bool moving, int grid_ctas, cudaStream_t stream);
cudaError_t read_device_status(int* out, bool clear);
cudaError_t read_pair_status(int* out, bool clear);
cudaError_t read_loads_status(int* out, bool clear);
cudaError_t launch_reduce_windows(const psc_window* d_windows, int nwin, double* out, cudaStream_t stream);
cudaError_t launch_init_equilibrium(int store, double scale, void* f, int64_t ncells, cudaStream_t stream);
// inlet = {rho, ux, uy, uz} when open_x (PSC_WIN_OPEN_X faces), else unused
cudaError_t launch_stream_push(int store, double scale, const void* src, double* dst, int nx, int ny, int nz,
                               cudaStream_t stream, bool open_x = false, const double* inlet = nullptr);
cudaError_t launch_stream_pull_store(int store, double scale, const double* src, void* dst, int nx, int ny, int nz,
                                     cudaStream_t stream, bool open_x = false, const double* inlet = nullptr);

cudaError_t launch_geometry_plan(const psc_geometry& g, cudaStream_t stream);
cudaError_t launch_geometry_build(const psc_geometry& g, cudaStream_t stream);
cudaError_t launch_solid_velocity(const psc_geometry& g, int us_type, void* us, cudaStream_t stream);
cudaError_t launch_particle_loads(const psc_geometry& g, int imb_type, const void* imb, double* chunk_partials,
                                  const double* imb_sums, double* forces, double* torques, double* diag,
                                  cudaStream_t stream);

// One window of a many-window particle-loads launch (a device table).
struct LoadsJob {
    psc_geometry g;
    const void* imb;          // IMB field [3][N] of the window (one imb_type for all jobs)
    const double* imb_sums;   // sum of the IMB field (3)
    double* forces;           // [P][3]
    double* torques;          // [P][3]
    double* diag;             // [PSC_NDIAG]
};
// Particle loads and load diagnostics of njobs windows in four launches.
// d_chunk_base / d_particle_base: [njobs + 1] exclusive prefix sums of the
// jobs' chunk and particle counts (the totals are their last entries, also
// passed by value); part: total_chunks rows of 6 doubles.  all_lists: every
// job gives loads-list arrays (the list path: the lists of the jobs whose list
// is not current are built first); list_ready: every job's list is current.
// Without all_lists the loads are reduced over the whole boxes.
cudaError_t launch_particle_loads_multi(const LoadsJob* d_jobs, const int64_t* d_chunk_base,
                                        const int64_t* d_particle_base, int njobs, int64_t total_chunks,
                                        int64_t total_particles, int imb_type, int max_subsamples,
                                        bool all_lists, bool list_ready, double* part, cudaStream_t stream);

cudaError_t launch_adjoint_seed(const psc_adjoint_args& a, cudaStream_t stream);
cudaError_t launch_adjoint_step(const psc_adjoint_args& a, cudaStream_t stream);
cudaError_t launch_adjoint_geometry_grad(const psc_geometry& g, const psc_adjoint_args& a, double* part,
                                         double* grad, cudaStream_t stream);

cudaError_t launch_vox_spheres(const double* pts, int M, const double* lo, const double* dx, double radius, int nx,
                               int ny, int nz, uint8_t* solid, cudaStream_t s);
cudaError_t launch_bb_step(const double* src, double* dst, const uint8_t* solid, int nx, int ny, int nz, double tau,
                           double fx, double fy, double fz, unsigned flags, double* mom, cudaStream_t s);

cudaError_t launch_equilibrium(const double* rho, const double* ux, const double* uy, const double* uz, double* out,
                               int64_t n, cudaStream_t s);
cudaError_t launch_guo(double fx, double fy, double fz, const double* ux, const double* uy, const double* uz,
                       double tau, double* out, int64_t n, cudaStream_t s);

// exclusive scan of int32 counts -> int32 offsets, out has n + 1 entries
size_t scan_tmp_bytes(int64_t n);
cudaError_t scan_exclusive_i32(const int32_t* in, int32_t* out, int64_t n, void* tmp, cudaStream_t stream);

}  // namespace psc
