/*
 * psc_b200.h -- C ABI of libpscb200.so: the D3Q19 partially-saturated-cell
 * immersed-boundary (PSC-IMB) lattice-Boltzmann step on one NVIDIA B200
 * (sm_100a).
 *
 * The reference implementation is pure NumPy (src/lbm_dem/psc3d.py of
 * wangjianfttt/particuology_Hydraulic-penalty-) and has no FFI of its own.
 * These entry points are what a ctypes binding of that module's hot path
 * needs; each cites the reference function it replaces.  The Python package
 * particuology_hydraulic_penalty_b200 binds them with ctypes.
 *
 * Conventions
 *  - Every function returns PSC_OK (0) or a negative PSC_E* code; the message
 *    of the last failure on the calling thread is psc_last_error().
 *  - All array pointers are DEVICE pointers unless the parameter name starts
 *    with "h_".  Two layers:
 *      descriptor layer (psc_window / psc_geometry / psc_adjoint_args): the
 *        caller allocates every buffer and no entry point allocates device
 *        memory; sizes come from the *_bytes / plan queries;
 *      handle layer (psc_solver / psc_batch, at the end of this file): the
 *        reference's solver object -- the handle owns its device memory,
 *        stream and CUDA graphs and takes and returns HOST arrays.
 *  - "stream" is a cudaStream_t passed as void* (NULL = legacy default stream).
 *    Work is enqueued asynchronously; nothing synchronises unless stated.
 *  - Lattice layout: structure of arrays, population plane i of a window is
 *    f[i * N + (ix * ny + iy) * nz + iz], N = nx * ny * nz, iz contiguous --
 *    the reference's f[i, ix, iy, iz] (psc3d.py:140) flattened.
 *  - The velocity set, its index order and weights are those of
 *    psc3d.py:17-43 (rest, +-x, +-y, +-z, then 12 diagonals in +- pairs).
 *  - Stored populations are POST-COLLISION values (pull streaming): a step
 *    reads f*_i(x - c_i), collides at x and writes f*_i(x).  The reference's
 *    post-stream state is recovered by psc_stream_push().
 *  - Handles are not thread-safe; distinct windows / buffers are independent.
 */
#ifndef PSC_B200_H
#define PSC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSC_ABI_VERSION 5

/* ---- status codes ------------------------------------------------------- */
#define PSC_OK 0
#define PSC_E_INVALID -1     /* bad argument (null pointer, size, mode) */
#define PSC_E_CUDA -2        /* a CUDA runtime call failed */
#define PSC_E_UNSUPPORTED -3 /* valid but not supported by the library or the device */
#define PSC_E_CAPACITY -4    /* a caller buffer is too small (see plan queries) */

/* ---- storage / arithmetic modes of the populations ---------------------- */
#define PSC_STORE_F64_EXACT 0 /* absolute f in FP64, reference operation order: bit-exact */
#define PSC_STORE_F64 1       /* deviation f - w*rho0 in FP64, FMA arithmetic */
#define PSC_STORE_F32 2       /* deviation in FP32, FP32 arithmetic */
#define PSC_STORE_F16 3       /* deviation * store_scale in FP16, FP32 arithmetic */
#define PSC_STORE_BF16 4      /* deviation * store_scale in BF16, FP32 arithmetic */

/* ---- per-step flags ----------------------------------------------------- */
#define PSC_STEP_COLLIDE 1u /* collide and write f_dst; without it: moments only */
#define PSC_STEP_IMB 2u     /* write the node IMB momentum (psc3d.py:234-236) */
#define PSC_STEP_MOMENTS 4u /* write rho, ux, uy, uz of the pulled state */
#define PSC_STEP_REDUCE 8u  /* write per-tile FP64 reduction partials */
#define PSC_STEP_MOVING 16u /* some window has PSC_WIN_MOVING: compile in the u_s path */

/* ---- kernel variants of the deviation modes ----------------------------- */
#define PSC_KERNEL_AUTO 0   /* psc_step_windows_ex: the direct kernel; the handle layer picks the pair
                               kernel for FP32/FP16/BF16 storage when every window has an even nz */
#define PSC_KERNEL_DIRECT 1 /* per-thread coalesced pulls (any window) */
#define PSC_KERNEL_TMA 2    /* bulk-copy (TMA) row staging in shared memory */
#define PSC_KERNEL_PAIR 3   /* two consecutive z cells per thread, 2-element loads and stores; windows planned
                               by psc_plan_pair_tiles (nz even, population buffers 16-byte aligned) */

/* Launch configuration of psc_step_windows_ex(). */
typedef struct psc_launch {
    int32_t grid_ctas;        /* persistent grid size; 0 = SM count x occupancy */
    int32_t cells_per_thread; /* 1, 2 or 4; the windows must be planned with tile_cells = 256 x this */
    int32_t kernel;           /* PSC_KERNEL_* (PSC_STORE_F64_EXACT always runs its own kernel) */
    int32_t stages;           /* TMA pipeline depth: 2, 3 or 4 (0 = 3) */
    int32_t stage_bytes;      /* TMA: shared-memory bytes per stage, from psc_plan_row_tiles */
} psc_launch;

/* ---- per-window flags --------------------------------------------------- */
#define PSC_WIN_MOVING 1   /* read the solid velocity field us (else u_s = 0) */
#define PSC_WIN_INACTIVE 2 /* skip the window's tiles: state frozen (e.g. converged); no partials written */
/* Open along x (no counterpart in the reference, which is periodic in every
 * direction, psc3d.py:239-242).  Velocity inlet at x = 0 by moving-wall
 * bounce-back: a population entering from outside (c_x = +1) is the node's
 * own post-collision population of the opposite direction plus
 * 2 w_i inlet_rho (c_i . inlet_u) / cs^2 (mass flux inlet_rho * inlet_u per
 * unit face area).  Zero-gradient outflow at x = nx - 1: a population
 * entering from outside (c_x = -1) is the post-collision value of the plane
 * x = nx - 1 itself.  y and z stay periodic.  Honoured by the exact and the
 * direct kernels; psc_plan_row_tiles rejects such windows. */
#define PSC_WIN_OPEN_X 4

/* Reduction slots written per tile with PSC_STEP_REDUCE and summed per window
 * by psc_reduce_windows().  Velocities are the stored-moment velocities
 * u = (m + F/2) / rho of the PULLED state (psc3d.py:211-214 / 243-246). */
#define PSC_RED_RHO 0
#define PSC_RED_UX 1
#define PSC_RED_UY 2
#define PSC_RED_UZ 3
#define PSC_RED_FLUID_UX 4 /* sum (1 - solid) * ux */
#define PSC_RED_FLUID_UY 5
#define PSC_RED_FLUID_UZ 6
#define PSC_RED_FLUID 7 /* sum (1 - solid) */
#define PSC_RED_IMBX 8  /* sum of this step's IMB momentum (collide only) */
#define PSC_RED_IMBY 9
#define PSC_RED_IMBZ 10
#define PSC_RED_NONFINITE 11 /* number of cells with a non-finite moment */
#define PSC_RED_SOLID 12     /* sum of the clipped solid fraction (solid_volume_lu) */
#define PSC_NRED 13
/* Reduction partials of one window: a header row (element 0 = number of
 * rows that follow, written by the step kernel) and up to
 * tile_count * PSC_PARTIAL_ROWS rows of PSC_NRED doubles.  The persistent
 * kernels accumulate each thread's cells over the CTA's whole run of tiles
 * inside the window and write one row per warp and CTA (no per-tile
 * reduction, no block barrier); the exact kernel writes one row per warp and
 * tile.  Sums are deterministic for a given launch configuration. */
#define PSC_PARTIAL_ROWS 8

/* Diagnostics written by psc_particle_loads() (psc3d.py:247-253). */
#define PSC_DIAG_MOMENTUM_RESIDUAL 0
#define PSC_DIAG_MAX_FORCE 1
#define PSC_DIAG_MAX_TORQUE 2
#define PSC_DIAG_FORCE_SUM_X 3
#define PSC_DIAG_FORCE_SUM_Y 4
#define PSC_DIAG_FORCE_SUM_Z 5
#define PSC_NDIAG 6

/* One lattice window of a (batched) launch.  Lives in device memory; the
 * array of windows handed to psc_step_windows() is a device pointer.  All windows of
 * one launch share the storage mode. */
typedef struct psc_window {
    int32_t nx, ny, nz;    /* lattice extent (the reference's n, n, n) */
    int32_t subsamples;    /* S: solid fraction from S^3 samples per cell */
    int32_t flags;         /* PSC_WIN_* */
    int32_t tile_cells;    /* cells per tile (set by psc_plan_tiles) */
    int64_t tile_begin;    /* first global tile index of this window */
    int64_t tile_count;    /* number of tiles of this window */
    double tau;            /* BGK relaxation time */
    double force[3];       /* body force; the reference is (0, 0, body_force_z) */
    double store_scale;    /* F16/BF16: stored = deviation * store_scale; else 1 */
    const void* f_src;     /* populations read this step [19][N] */
    void* f_dst;           /* populations written this step [19][N] */
    const double* solid;   /* PSC_STORE_F64_EXACT: clipped solid fraction [N] */
    const uint8_t* level;  /* other modes: clipped inside-sample count [N] */
    const void* us;        /* solid velocity [3][N] (double in F64 modes, float otherwise) */
    void* imb;             /* IMB momentum [3][N] (double in F64 modes, float otherwise) */
    void* moments;         /* rho, ux, uy, uz [4][N] (same element type as imb) */
    double* partials;      /* [1 + tile_count * PSC_PARTIAL_ROWS][PSC_NRED] (header row first) */
    double tau_minus;      /* TRT: antisymmetric relaxation time (0 = BGK, the reference's collision);
                              deviation storage modes only */
    double inlet_rho;      /* PSC_WIN_OPEN_X: inlet density */
    double inlet_u[3];     /* PSC_WIN_OPEN_X: inlet velocity */
} psc_window;

/* Particle-derived geometry of ONE window (device arrays, caller-owned).
 * Particles are [P][10] float64: x, y, z, r, vx, vy, vz, wx, wy, wz in
 * lattice units -- the fields of the reference's Particle3D (psc3d.py:46-57). */
typedef struct psc_geometry {
    int32_t nx, ny, nz;
    int32_t subsamples;
    int32_t nparticles;
    int32_t chunk_entries;    /* bbox entries per load-reduction chunk (power of 2) */
    int64_t capacity_entries; /* length of ent_cnt / cl_pid / cl_cnt */
    int64_t capacity_chunks;  /* rows of the chunk partial buffer of psc_particle_loads */
    const double* particles;  /* [P][10] */
    int32_t* bbox;            /* [P][6]: x0, y0, z0, ex, ey, ez (clipped box) */
    int64_t* ent_off;         /* [P+1] bbox-entry offsets */
    int64_t* chunk_off;       /* [P+1] load-chunk offsets */
    int64_t* totals;          /* [4]: entries, chunks, max particles per cell, overflow flag */
    uint16_t* ent_cnt;        /* [capacity_entries] inside-sample count per bbox entry */
    int32_t* cell_n;          /* [N] scratch counter */
    int32_t* cell_off;        /* [N+1] cell -> particle list offsets */
    int32_t* cl_pid;          /* [capacity_entries] particle ids per cell, ascending */
    uint16_t* cl_cnt;         /* [capacity_entries] their sample counts */
    double* alpha_sum;        /* [N] unclipped alpha sum (psc3d.py:174 / 339-341) */
    double* solid;            /* [N] clip(alpha_sum, 0, 1) (psc3d.py:175 / 344) */
    uint8_t* level;           /* [N] min(sum of counts, S^3), or NULL; needs S^3 <= 255 */
    void* scan_tmp;           /* scratch of psc_scan_tmp_bytes(N + 1) bytes */
    /* Smooth solid fraction (the differentiable surrogate used by the
     * adjoint): when smooth_eps > 0 every sample contributes
     * sigma((r - |x_s - X|) / smooth_eps) instead of the 0/1 inside test. */
    double smooth_eps;
    double* ent_alpha;        /* [capacity_entries] smooth alpha per entry (smooth mode) */
    int32_t* cl_ent;          /* [capacity_entries] entry index per cell-list slot (smooth mode) */
    /* Loads list, for a geometry used by more than one loads call (static
     * particles).  Every load chunk is reduced by PSC_LOAD_THREADS threads (warps
     * of 32).  Warp w owns the chunk's entries 32w + l + j * PSC_LOAD_THREADS
     * (lane l, in order of j then l); its entries with a non-zero sample count are
     * numbered c = 0, 1, ... in that order and dealt round-robin to its lanes:
     * entry c is slot k = c / 32 of thread t = 32w + c % 32, at list index
     * chunk * chunk_entries + k * PSC_LOAD_THREADS + t, holding the entry's owner
     * weight alpha_p / max(alpha_sum, 1e-14) (load_w) and its bbox-local cell
     * a | b << 11 | k << 22 (load_abk); load_n[chunk * PSC_LOAD_THREADS + t]
     * counts thread t's slots.  With the three arrays set, psc_particle_loads
     * reduces from the list, building it first when list_ready == 0 (so every
     * call on a geometry gives the same sums, bit for bit); the caller sets
     * list_ready after a call on the same geometry.  Without the arrays it
     * reduces over the whole boxes (the same loads to round-off).  Needs
     * chunk_entries a multiple of PSC_LOAD_THREADS, at most 16 of them, and
     * nx, ny <= 2048, nz <= 1024; NULL arrays = no list. */
    double* load_w;           /* [capacity_chunks * chunk_entries] or NULL */
    uint32_t* load_abk;       /* [capacity_chunks * chunk_entries] or NULL */
    uint8_t* load_n;          /* [capacity_chunks * PSC_LOAD_THREADS] or NULL */
    int32_t list_ready;
    int32_t reserved;
} psc_geometry;

#define PSC_LOAD_THREADS 256 /* threads reducing one load chunk */

/* Arguments of the adjoint kernels (one window, deviation storage F64/F32).
 * The adjoint state lambda has the arithmetic type of the storage mode
 * (double for PSC_STORE_F64, float for PSC_STORE_F32). */
typedef struct psc_adjoint_args {
    int32_t nx, ny, nz;
    int32_t store;          /* PSC_STORE_F64 or PSC_STORE_F32 */
    double tau;
    double force[3];
    double kappa;           /* nu / (|F| N): K = kappa * sum (1 - solid) u.dir */
    double dir[3];          /* unit vector along the body force */
    const void* state;      /* stored post-collision populations S_t [19][N] */
    const double* solid;    /* clipped solid fraction [N] */
    const void* lam_in;     /* dK/dS_{t+1} [19][N] */
    void* lam_out;          /* dK/dS_t [19][N] (written, one store per element) */
    double* dKdB;           /* [N] accumulated dK/dB */
    double* dKdsolid;       /* [N] direct dK/dsolid (written by the seed) */
} psc_adjoint_args;

/* ---- library ------------------------------------------------------------ */
int psc_abi_version(void);
const char* psc_last_error(void);
/* sizeof(psc_window) and sizeof(psc_geometry) as compiled into the library,
 * so bindings can check their struct layout. */
size_t psc_window_size(void);
size_t psc_geometry_size(void);
size_t psc_adjoint_args_size(void);
/* Bytes of scan scratch needed for n elements. */
size_t psc_scan_tmp_bytes(int64_t n);

/* ---- tiles and windows -------------------------------------------------- */
/* Fill tile_cells / tile_begin / tile_count of h_windows (HOST array) and
 * return the total tile count in *h_total_tiles.  tile_cells: 0 (= 256),
 * 256, 512 or 1024 (256 x cells per thread).  A window must hold fewer than
 * 2^31 / 19 cells (32-bit population offsets). */
int psc_plan_tiles(struct psc_window* h_windows, int nwin, int tile_cells, int64_t* h_total_tiles);

/* Row tiles for PSC_KERNEL_TMA: a tile is `rows` whole z-rows of one x-plane
 * (rows = 0: chosen per window for ~48 kB of populations per stage; rows =
 * -1: each window keeps the rows preset as tile_cells = rows * nz).  elem_bytes is
 * the storage element size; every window needs nz * elem_bytes % 16 == 0 and
 * 16-byte aligned population buffers (bulk-copy rule).  Returns the total
 * tile count and the shared-memory bytes one stage needs. */
int psc_plan_row_tiles(struct psc_window* h_windows, int nwin, int rows, int elem_bytes, int64_t* h_total_tiles,
                       int32_t* h_stage_bytes);
/* Tiles for PSC_KERNEL_PAIR: 512-cell tiles (two cells per thread); every
 * window needs an even nz (a cell pair never crosses a z row). */
int psc_plan_pair_tiles(struct psc_window* h_windows, int nwin, int64_t* h_total_tiles);
/* Device-side status word: non-zero after a kernel gave up a bounded wait
 * (0x101 producer, 0x102 drain, 0x103 consumer of the TMA kernel; 0x301 a
 * load-chunk kernel's wait for a partial-sum slot) or skipped a window it
 * cannot run (0x201 odd nz, 0x202 tiles not planned for the pair kernel).
 * Synchronises. */
int psc_device_status(int* h_status, int clear);

/* Equilibrium at rho = 1, u = 0 in the given storage mode
 * (the reference's initial state, psc3d.py:136-140). */
int psc_init_equilibrium(int store, double store_scale, void* f, int64_t ncells, void* stream);

/* ---- geometry (psc3d.py:60-94, 151-179, 328-345) ------------------------ */
/* Clipped bounding boxes, entry and chunk offsets, totals.  The caller reads
 * totals[0] (entries) and totals[1] (chunks) to size ent_cnt / cl_* and the
 * load partials before psc_geometry_build. */
int psc_geometry_plan(const psc_geometry* h_geo, void* stream);
/* Inside-sample counts, per-cell particle lists (ascending id), alpha_sum,
 * solid and level.  Bit-exact with the reference (no FMA contraction). */
int psc_geometry_build(const psc_geometry* h_geo, void* stream);
/* alpha-weighted rigid-body velocity u_s = sum_p alpha_p (V_p + w_p x r) /
 * sum alpha (psc3d.py:181-206 / 347-373), written as [3][N] of us_type
 * (0 = float64, 1 = float32). */
int psc_solid_velocity(const psc_geometry* h_geo, int us_type, void* us, void* stream);

/* ---- the step (psc3d.py:208-246) ---------------------------------------- */
/* One pull-stream + collide pass over every tile of every window.
 * d_windows: device array of nwin windows; total_tiles from psc_plan_tiles;
 * grid_ctas = 0 picks a persistent grid (a multiple of the SM count). */
int psc_step_windows(int store, const struct psc_window* d_windows, int nwin, int64_t total_tiles,
             unsigned flags, int grid_ctas, void* stream);
/* psc_step_windows with an explicit launch configuration (kernel variant, cells per
 * thread, grid); cfg may be NULL for the defaults. */
int psc_step_windows_ex(int store, const struct psc_window* d_windows, int nwin, int64_t total_tiles, unsigned flags,
                const psc_launch* cfg, void* stream);
/* Sum the per-tile partials of each window in a fixed order (deterministic)
 * into out[nwin][PSC_NRED] (device).  The partials are consumed: segment sums
 * are written over them, so reduce once per PSC_STEP_REDUCE pass.  nwin must
 * not exceed 65535. */
int psc_reduce_windows(const struct psc_window* d_windows, int nwin, double* out, void* stream);

/* ---- particle loads (psc3d.py:255-281 / 375-407) ------------------------ */
/* Per-particle force and torque from the node IMB momentum imb [3][N]
 * (imb_type 0 = float64, 1 = float32), owner weights alpha_p / alpha_sum
 * (computed per bbox entry, or read from the geometry's loads list when
 * list_ready).
 * chunk_partials: [capacity_chunks][6] scratch.  imb_sums: device [3] sum of
 * the node IMB momentum (PSC_RED_IMB* of the same step).  Writes forces
 * [P][3], torques [P][3] and diag [PSC_NDIAG]. */
int psc_particle_loads(const psc_geometry* h_geo, int imb_type, const void* imb, double* chunk_partials,
                       const double* imb_sums, double* forces, double* torques, double* diag, void* stream);

/* ---- element-wise helpers of the reference module ----------------------- */
/* out[i][c] = equilibrium of (rho, u) at n cells, exact FP64 in the
 * reference's operation order (equilibrium, psc3d.py:97-103). */
int psc_equilibrium(const double* rho, const double* ux, const double* uy, const double* uz, double* out, int64_t n,
                    void* stream);
/* out[i][c] = Guo forcing term for force (fx, fy, fz) (guo_force, psc3d.py:106-114). */
int psc_guo_force(double fx, double fy, double fz, const double* ux, const double* uy, const double* uz, double tau,
                  double* out, int64_t n, void* stream);

/* ---- voxel bounce-back window LBM (scripts/run_3d_window_lbm.py) -------- */
/* solid[(ix*ny + iy)*nz + iz] = 1 where the cell centre lo + (i + 0.5) dx lies
 * inside any sphere of the given radius (voxelize, run_3d_window_lbm.py:73-92).
 * d_points [M][3] device; h_lo, h_dx HOST double[3].  solid is OR-ed into
 * (clear it first). */
int psc_voxelize_spheres(const double* d_points, int M, const double* h_lo, const double* h_dx, double radius,
                         int nx, int ny, int nz, uint8_t* solid, void* stream);
/* One step of run_lbm (:100-119) on post-collision FP64 populations (pull,
 * solid-node pair overwrite as in the reference, moments with u = 0 at solid
 * nodes, BGK + Guo with force (fx, fy, fz)); flags PSC_STEP_COLLIDE and/or
 * PSC_STEP_MOMENTS (rho, ux, uy, uz [4][N]). */
int psc_bounceback_step(const double* f_src, double* f_dst, const uint8_t* solid, int nx, int ny, int nz, double tau,
                        double fx, double fy, double fz, unsigned flags, double* moments, void* stream);

/* ---- particle loads without caller scratch (no counterpart in the reference)
 * For callers that cannot allocate device memory -- a solver embedded in a
 * program that owns the device memory budget, or a coupling loop that must
 * not call cudaMalloc after start-up (it synchronises the device).  The same
 * loads as psc_particle_loads() to round-off (its per-particle sums add the
 * chunk partials in another order), but the per-chunk partial sums live in a
 * fixed array inside the library: PSC_LOADS_STATIC_MAX_CHUNKS x 6 doubles
 * (768 KiB) held by every GPU that loads the library until exit.
 * h_geo->capacity_chunks must not exceed PSC_LOADS_STATIC_MAX_CHUNKS
 * (PSC_E_CAPACITY otherwise).  The first call on a device looks the array's
 * address up (cudaGetSymbolAddress) -- make it before any stream capture.
 * All calls share the array: calls that overlap on the GPU race. */
#define PSC_LOADS_STATIC_MAX_CHUNKS 16384
int psc_particle_loads_static(const psc_geometry* h_geo, int imb_type, const void* imb, const double* imb_sums,
                              double* forces, double* torques, double* diag, void* stream);

/* ---- adjoint of the permeability (no counterpart in the reference) ------- */
/* Seed: lambda_T = dK/dS_T for K = kappa sum (1 - solid) u.dir of the
 * post-stream state pull(S_T); also the direct term dK/dsolid. */
int psc_adjoint_seed(const psc_adjoint_args* h_args, void* stream);
/* One reverse step: lambda_t = pull^T (J_t^T lambda_{t+1}) with J_t the
 * collision Jacobian at pull(S_t); dKdB += lambda_{t+1} . dC/dB. */
int psc_adjoint_step(const psc_adjoint_args* h_args, void* stream);
/* dK/d(x, y, z, r) per particle through the smooth solid fraction:
 * grad[P][4]; chunk_partials [capacity_chunks][4] scratch. */
int psc_adjoint_geometry_grad(const psc_geometry* h_geo, const psc_adjoint_args* h_args, double* chunk_partials,
                              double* grad, void* stream);

/* ---- population layout conversions -------------------------------------- */
/* dst_i(x + c_i) = src_i(x): turns the stored post-collision populations into
 * the reference's post-stream f (psc3d.py:239-242); returns absolute FP64
 * populations for every storage mode. */
int psc_stream_push(int store, double store_scale, const void* src, double* dst, int nx, int ny, int nz,
                    void* stream);
/* psc_stream_push for a PSC_WIN_OPEN_X window (bounce-back velocity inlet of
 * (inlet_rho, h_inlet_u[3]) at x = 0, zero-gradient outflow at x = nx - 1;
 * no counterpart in the reference). */
int psc_stream_push_open(int store, double store_scale, const void* src, double* dst, int nx, int ny, int nz,
                         double inlet_rho, const double* h_inlet_u, void* stream);
/* Inverse: absolute FP64 post-stream f -> stored representation. */
int psc_stream_pull_store(int store, double store_scale, const double* src, void* dst, int nx, int ny, int nz,
                          void* stream);
/* psc_stream_pull_store for a PSC_WIN_OPEN_X window: also sets the stored
 * populations that only the inlet's bounce-back reads, so the next pull
 * reproduces src at x = 0 (to rounding in the exact mode). */
int psc_stream_pull_store_open(int store, double store_scale, const double* src, void* dst, int nx, int ny, int nz,
                               double inlet_rho, const double* h_inlet_u, void* stream);

/* ======================================================================== *
 * Handle layer: the reference's solver object (PscD3Q19 / SparsePscD3Q19,  *
 * psc3d.py:117-407) and batches of windows.  A handle owns its device      *
 * memory (allocated at creation and when a geometry grows), its stream and *
 * its CUDA graphs; every array argument is a HOST array.  Functions that   *
 * return data synchronise the handle's stream.  Handles are not            *
 * thread-safe; distinct handles are independent.                           *
 * ======================================================================== */

/* Configuration of one lattice window (PscD3Q19.__init__, psc3d.py:120-147). */
typedef struct psc_config {
    int32_t nx, ny, nz;       /* lattice extent (the reference's n, n, n) */
    int32_t subsamples;       /* S (the reference's default: 4 dense, 3 sparse) */
    int32_t store;            /* PSC_STORE_* */
    int32_t static_geometry;  /* 0: voxelise again whenever the particles changed (psc3d.py:209-210) */
    int32_t device;           /* CUDA device ordinal */
    int32_t conv_min_steps;   /* PSC_RUN_CONVERGE: never stop before this step of the call (>= 1) */
    double tau;               /* BGK relaxation time (default 0.72 in the reference) */
    double tau_minus;         /* TRT antisymmetric relaxation time; 0 = BGK, the reference's collision */
    double force[3];          /* body force; the reference: (0, 0, body_force_z) */
    double store_scale;       /* PSC_STORE_F16 / BF16 stored-deviation scale; 0 = the mode's default */
    double conv_tol;          /* PSC_RUN_CONVERGE tolerance; 0 = 1e-8 (couple_psc_liggghts.py:168) */
    void* stream;             /* cudaStream_t for all work of the handle; NULL = a stream of its own */
    int32_t open_x;           /* 1: velocity inlet at x = 0, zero-gradient outflow at x = nx - 1
                                 (PSC_WIN_OPEN_X; not in the reference); 0: periodic */
    int32_t conv_check_every; /* PSC_RUN_CONVERGE: evaluate the criterion every k steps (on steps k - 1 and
                                 k); 0 or 1 = every step, as the reference's loop does */
    double inlet_rho;         /* open_x: inlet density */
    double inlet_u[3];        /* open_x: inlet velocity */
} psc_config;

/* Diagnostics of one step.  The first five are the reference's dictionary
 * (psc3d.py:247-253); the rest are the Darcy quantities its callers derive
 * (run_psc_permeability_resolution.py:144-160).  Moments are those of the
 * post-stream state. */
typedef struct psc_diag {
    double solid_volume_lu;   /* sum of the clipped solid fraction */
    double mean_uz;           /* mean post-stream u_z */
    double momentum_residual; /* |sum_p F_p + sum_x imb| */
    double max_force;         /* max_p |F_p| (0 without particles) */
    double max_torque;        /* max_p |T_p| */
    double mean_u[3];         /* mean post-stream velocity */
    double superficial_u[3];  /* sum (1 - solid) u / N */
    double fluid_volume_lu;   /* sum (1 - solid) */
    double imb_sum[3];        /* sum of the node IMB momentum of the step */
    double force_sum[3];      /* sum_p F_p */
    double permeability;      /* nu (superficial_u . F) / |F|^2, nu = (tau - 1/2) / 3; 0 when F = 0 */
    double nonfinite_cells;   /* cells with a non-finite moment (0 for a healthy run) */
} psc_diag;

typedef struct psc_status {
    int32_t steps_done;       /* steps taken by this call */
    int32_t converged;        /* PSC_RUN_CONVERGE / psc_batch_converge: criterion met */
    double residual;          /* last relative change of the convergence quantity (inf if none) */
    psc_diag diag;            /* diagnostics of the last step (PSC_RUN_DIAG / PSC_RUN_CONVERGE) */
} psc_status;

/* psc_step() flags */
#define PSC_RUN_DIAG 1u     /* diagnostics and particle loads of the final step */
#define PSC_RUN_CONVERGE 2u /* stop at the first step k >= conv_min_steps, k a multiple of
                               conv_check_every, with |mean_uz_k - mean_uz_{k-1}| / |mean_uz_k| < conv_tol
                               (lbm_converge, couple_psc_liggghts.py:284-296; the criterion is evaluated on
                               the device, the host reads its outcome once per block of steps); particle
                               loads and diagnostics of the final step only; implies PSC_RUN_DIAG */
#define PSC_RUN_FIELDS 4u   /* also write the rho / u fields of the final state (else made on demand) */

/* psc_get_fields() selectors; every field is returned as float64 */
#define PSC_FIELD_RHO 0       /* [N] post-stream density (1 before the first step, psc3d.py:136) */
#define PSC_FIELD_UX 1        /* [N] */
#define PSC_FIELD_UY 2        /* [N] */
#define PSC_FIELD_UZ 3        /* [N] (m_z + F_z/2) / rho, psc3d.py:243-246 */
#define PSC_FIELD_SOLID 4     /* [N] clipped solid fraction */
#define PSC_FIELD_IMB_X 5     /* [N] IMB momentum of the last step */
#define PSC_FIELD_IMB_Y 6
#define PSC_FIELD_IMB_Z 7
#define PSC_FIELD_ALPHA_SUM 8 /* [N] unclipped alpha sum (alpha_sum_flat) */
#define PSC_FIELD_US_X 9      /* [N] solid velocity (solid_velocity(), psc3d.py:181-206) */
#define PSC_FIELD_US_Y 10
#define PSC_FIELD_US_Z 11
#define PSC_FIELD_F 12        /* [19][N] post-stream populations, absolute (PscD3Q19.f) */

typedef struct psc_solver psc_solver;

/* PscD3Q19(n, particles, tau, subsamples, body_force_z, static_geometry):
 * populations at the rest equilibrium, no particles yet. */
int psc_create(const psc_config* h_cfg, psc_solver** out);
int psc_destroy(psc_solver* h);
/* h_particles [P][10] (x, y, z, r, vx, vy, vz, wx, wy, wz: Particle3D).  Copied;
 * read by the next step.  A changed array triggers a new voxelisation unless
 * static_geometry is set (the reference re-reads positions and velocities
 * every step for the solid velocity and torque arms in either case). */
int psc_set_particles(psc_solver* h, const double* h_particles, int nparticles);
/* rebuild_geometry() (psc3d.py:151-179 / 328-345), now. */
int psc_rebuild_geometry(psc_solver* h);
/* nsteps calls of collide_stream_psc() (psc3d.py:208-253).  h_status may be
 * NULL.  Without PSC_RUN_DIAG the intermediate steps skip the reductions
 * (they change no state); the IMB field of the final step is always written.
 * psc_step(h, 1, PSC_RUN_DIAG) (one drop-in call) replays its launches from a
 * CUDA graph, one per population buffer and kind of call, recorded on the
 * second call whose launch arguments (buffers, sizes, kernel, descriptor
 * version) match the previous call's; on a stream the caller is capturing it
 * runs its launches directly, so they go into the caller's graph.  Such a call
 * takes its post-stream sums from the next step, run ahead into the other
 * population buffer and a second IMB field, when the step inputs (geometry,
 * solid velocity, descriptors) are those of the previous such call; the next
 * such call takes that step as its own if the inputs still match, and any
 * other stepping or state-setting call drops it.  Results are the same bits
 * as with a reduction-only pass. */
int psc_step(psc_solver* h, int nsteps, unsigned flags, psc_status* h_status);
/* Field `which` (PSC_FIELD_*) as float64 into h_dst ([N], or [19][N] for PSC_FIELD_F). */
int psc_get_fields(psc_solver* h, int which, double* h_dst);
/* Message of the last failed call on this handle ("" if none).  A call that
 * fails also sets the calling thread's psc_last_error(); psc_create reports
 * there only (it returns no handle on failure).  Valid until the next failing
 * call on the handle or psc_destroy. */
const char* psc_solver_last_error(const psc_solver* h);
/* lbm_converge (coupling_sync/couple_psc_liggghts.py:284-296) as one call: up to max_steps steps,
 * stopping at the first step k >= min_steps (k a multiple of check_every, or max_steps) with
 * |mean_uz_k - mean_uz_{k-1}| / max(|mean_uz_k|, 1e-30) < tol.  check_every = 1 evaluates every
 * step, as the reference does (same iterations and residual); a larger k takes the criterion on
 * steps k - 1 and k only and runs the steps in between without reductions.  The criterion runs on
 * the device; the state, loads and diagnostics returned are those of the stopping step
 * (h_status: steps_done = iterations, residual, converged, diag).  flags: 0 or PSC_RUN_FIELDS. */
int psc_converge(psc_solver* h, int max_steps, double tol, int min_steps, int check_every, unsigned flags,
                 psc_status* h_status);
/* Set the post-stream populations (PscD3Q19.f = ...), absolute float64 [19][N]. */
int psc_set_populations(psc_solver* h, const double* h_f);
/* hydro_forces / hydro_torques [P][3] of the last step (accumulate_particle_loads,
 * psc3d.py:255-281, computed here if the last step did not). */
int psc_get_loads(psc_solver* h, double* h_forces, double* h_torques);
/* accumulate_particle_loads() (psc3d.py:255-281): loads and diagnostics again
 * from the last step's IMB field with the current geometry and particle
 * state (torque arms use the current positions). */
int psc_accumulate_particle_loads(psc_solver* h);
/* Diagnostics of the last step (computed here if the last step did not). */
int psc_get_diag(psc_solver* h, psc_diag* h_diag);
/* Sparse solid fractions per particle (SparsePscD3Q19.node_ids / alpha_vals,
 * psc3d.py:328-345): h_offsets [P+1] is always written; the ascending node
 * ids and alphas of particle p go to h_ids / h_vals [h_offsets[p] ..
 * h_offsets[p+1]) when capacity >= h_offsets[P] (else only the offsets,
 * PSC_E_CAPACITY). */
int psc_get_sparse_alpha(psc_solver* h, int64_t* h_offsets, int64_t* h_ids, double* h_vals, int64_t capacity);
/* Particle count and lattice cells of the handle. */
int psc_solver_info(psc_solver* h, int* h_nparticles, int64_t* h_cells);
/* ---- adjoint handle: K and dK/d(x, y, z, r) of every particle (no counterpart
 * in the reference) ---------------------------------------------------------
 * One static periodic BGK window in PSC_STORE_F32 or F64 deviation storage,
 * run from rest for `steps` steps with the smooth solid fraction (each
 * sub-sample contributes sigma((r - d) / smooth_eps)); checkpoints every
 * `checkpoint_every` steps; the backward pass recomputes each segment from its
 * checkpoint and runs the reverse steps (psc_adjoint_seed / psc_adjoint_step)
 * and the geometry gradient (psc_adjoint_geometry_grad).  K = nu (sum
 * (1 - solid) u . d) / N / |F|, d = F / |F|.  Device memory: the two
 * population buffers, ceil(steps / checkpoint_every) checkpoints and
 * checkpoint_every recomputed states. */
typedef struct psc_adjoint psc_adjoint;
int psc_adjoint_create(const psc_config* h_cfg, double smooth_eps, int steps, int checkpoint_every,
                       psc_adjoint** out);
int psc_adjoint_destroy(psc_adjoint* a);
/* Message of the last failed call on this adjoint handle ("" if none), as psc_solver_last_error. */
const char* psc_adjoint_last_error(const psc_adjoint* a);
/* K after the forward run with h_particles [P][10] (velocities ignored: static particles). */
int psc_adjoint_forward(psc_adjoint* a, const double* h_particles, int nparticles, double* h_K);
/* h_grad [P][4] = dK/d(x, y, z, r) of every particle for the last forward run. */
int psc_adjoint_backward(psc_adjoint* a, double* h_grad);

/* sizeof of the handle-layer structs as compiled into the library. */
size_t psc_config_size(void);
size_t psc_diag_size(void);
size_t psc_status_size(void);

/* ---- batches: many windows of uneven size, one persistent launch per step */
typedef struct psc_batch psc_batch;

/* nwin windows (all with the same store, device and stream).  launch may be
 * NULL (direct kernel, one cell per thread, automatic grid); graph_steps
 * (even, >= 2; 0 = none) steps are captured per CUDA graph and replayed. */
int psc_batch_create(const psc_config* h_cfgs, int nwin, const psc_launch* h_launch, int graph_steps,
                     psc_batch** out);
int psc_batch_destroy(psc_batch* b);
/* Message of the last failed call on this batch ("" if none), as psc_solver_last_error. */
const char* psc_batch_last_error(const psc_batch* b);
/* Particles of window `win`; a changed array re-voxelises that window before the next step. */
int psc_batch_set_particles(psc_batch* b, int win, const double* h_particles, int nparticles);
/* psc_batch_set_particles for every window in one call: h_particles[k] is window k's [P_k][10]
 * array (may be NULL when nparticles[k] is 0).  All windows are staged in one host buffer and
 * uploaded with one copy on the batch's own upload stream, beside the step kernels (they do not
 * read particles); whatever does read them waits for the copy.  Every window is checked before
 * any takes its new state: if one is rejected (NaN / Inf, null array) the call returns the error
 * and every window keeps its previous state. */
int psc_batch_set_particles_all(psc_batch* b, const double* const* h_particles, const int* h_nparticles);
/* nsteps steps of every active window.  PSC_RUN_DIAG: diagnostics and loads
 * of every window at the final step into h_status[nwin] (may be NULL).
 * The post-stream sums of a PSC_RUN_DIAG call are the moment sums of the next
 * step's pull.  With the pair kernel, without PSC_RUN_FIELDS and with the step
 * inputs (geometry, solid velocity, descriptors, frozen set) unchanged since
 * the previous PSC_RUN_DIAG call, the call runs that next step (into the other
 * population buffer and a second IMB field per window; the current state is
 * untouched) instead of a reduction-only pass, and the next call takes it as
 * its first step if the inputs are still the same.  Results are the same bits
 * either way. */
int psc_batch_step(psc_batch* b, int nsteps, unsigned flags, psc_status* h_status);
/* Step until every window's Darcy permeability changes by less than tol per
 * step, checked on a pair of consecutive steps every check_every steps; a
 * converged window is frozen (its tiles skipped) when `freeze` is set.
 * h_status[nwin]: steps to convergence (steps_done), converged flag, residual
 * and the diagnostics of the reductions-only pass at the end. */
int psc_batch_converge(psc_batch* b, double tol, int check_every, int max_steps, int min_steps, int freeze,
                       psc_status* h_status);
int psc_batch_get_diag(psc_batch* b, int win, psc_diag* h_diag);
int psc_batch_get_loads(psc_batch* b, int win, double* h_forces, double* h_torques);
int psc_batch_get_fields(psc_batch* b, int win, int which, double* h_dst);

#ifdef __cplusplus
}
#endif

#endif /* PSC_B200_H */
