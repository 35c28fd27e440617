// extern "C" entry points of libpscb200.so (declared in include/psc_b200.h).
//
// Every entry point validates its arguments on the host, enqueues work on the
// caller's stream and returns a status code; no exception crosses the ABI and
// nothing here allocates device memory.
#include <cstdio>
#include <string>

#include "internal.cuh"

namespace psc {

static thread_local std::string g_last_error;
static thread_local uint64_t g_error_seq = 0;  // errors set on this thread so far

void set_error(const std::string& msg) {
    g_last_error = msg;
    ++g_error_seq;
}

uint64_t error_seq() { return g_error_seq; }
const std::string& last_error_string() { return g_last_error; }

int fail(int code, const std::string& msg) {
    set_error(msg);
    return code;
}

int cuda_fail(cudaError_t err, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) + ")";
    return fail(PSC_E_CUDA, m);
}

int sm_count() {
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    int& c = cache[dev & 63];
    if (c == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        c = v;
    }
    return c;
}

static bool valid_store(int s) { return s >= PSC_STORE_F64_EXACT && s <= PSC_STORE_BF16; }

static int check_extent(int nx, int ny, int nz, const char* who) {
    if (nx <= 0 || ny <= 0 || nz <= 0) return fail(PSC_E_INVALID, std::string(who) + ": lattice extents must be > 0");
    const long long n = (long long)nx * ny * nz;
    if (n >= (1ll << 31)) return fail(PSC_E_UNSUPPORTED, std::string(who) + ": a window must have < 2^31 cells");
    return PSC_OK;
}

static int check_geometry(const psc_geometry* g, const char* who) {
    if (!g) return fail(PSC_E_INVALID, std::string(who) + ": null geometry");
    int st = check_extent(g->nx, g->ny, g->nz, who);
    if (st) return st;
    if (g->subsamples < 1 || g->subsamples > 16)
        return fail(PSC_E_INVALID, std::string(who) + ": subsamples must be in [1, 16]");
    if (g->nparticles < 0) return fail(PSC_E_INVALID, std::string(who) + ": negative particle count");
    if (g->chunk_entries <= 0) return fail(PSC_E_INVALID, std::string(who) + ": chunk_entries must be > 0");
    if (g->capacity_entries < 0 || g->capacity_chunks < 0 || g->capacity_entries >= (1ll << 31))
        return fail(PSC_E_INVALID, std::string(who) + ": capacities must be in [0, 2^31)");
    if (g->nparticles > 0 && (!g->particles || !g->bbox))
        return fail(PSC_E_INVALID, std::string(who) + ": null particle or bbox array");
    if (!g->ent_off || !g->chunk_off || !g->totals)
        return fail(PSC_E_INVALID, std::string(who) + ": null offsets/totals array");
    return PSC_OK;
}

}  // namespace psc

using namespace psc;

extern "C" {

int psc_abi_version(void) { return PSC_ABI_VERSION; }

const char* psc_last_error(void) { return g_last_error.c_str(); }

size_t psc_window_size(void) { return sizeof(psc_window); }

size_t psc_geometry_size(void) { return sizeof(psc_geometry); }

size_t psc_adjoint_args_size(void) { return sizeof(psc_adjoint_args); }

size_t psc_scan_tmp_bytes(int64_t n) { return scan_tmp_bytes(n < 0 ? 0 : n); }

int psc_plan_tiles(psc_window* h_windows, int nwin, int tile_cells, int64_t* h_total_tiles) {
    if (!h_windows || nwin <= 0 || !h_total_tiles) return fail(PSC_E_INVALID, "psc_plan_tiles: bad arguments");
    if (tile_cells == 0) tile_cells = STEP_THREADS;
    if (tile_cells != STEP_THREADS && tile_cells != 2 * STEP_THREADS && tile_cells != 4 * STEP_THREADS)
        return fail(PSC_E_UNSUPPORTED, "psc_plan_tiles: tile_cells must be 0, 256, 512 or 1024");
    int64_t begin = 0;
    for (int w = 0; w < nwin; ++w) {
        psc_window& W = h_windows[w];
        int st = check_extent(W.nx, W.ny, W.nz, "psc_plan_tiles");
        if (st) return st;
        const int64_t n = (int64_t)W.nx * W.ny * W.nz;
        if (n * 19 >= (1ll << 31))
            return fail(PSC_E_UNSUPPORTED, "psc_plan_tiles: a window must hold fewer than 2^31/19 cells");
        W.tile_cells = tile_cells;
        W.tile_begin = begin;
        W.tile_count = (n + tile_cells - 1) / tile_cells;
        begin += W.tile_count;
    }
    *h_total_tiles = begin;
    return PSC_OK;
}

int psc_plan_row_tiles(psc_window* h_windows, int nwin, int rows, int elem_bytes, int64_t* h_total_tiles,
                       int32_t* h_stage_bytes) {
    if (!h_windows || nwin <= 0 || !h_total_tiles || !h_stage_bytes || rows < -1)
        return fail(PSC_E_INVALID, "psc_plan_row_tiles: bad arguments");
    if (elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8)
        return fail(PSC_E_INVALID, "psc_plan_row_tiles: elem_bytes must be 2, 4 or 8");
    int64_t begin = 0;
    int64_t stage = 0;
    for (int w = 0; w < nwin; ++w) {
        psc_window& W = h_windows[w];
        int st = check_extent(W.nx, W.ny, W.nz, "psc_plan_row_tiles");
        if (st) return st;
        if (W.flags & PSC_WIN_OPEN_X)
            return fail(PSC_E_UNSUPPORTED, "psc_plan_row_tiles: the TMA kernel runs periodic windows only (window " +
                                               std::to_string(w) + " has PSC_WIN_OPEN_X)");
        const int64_t n = (int64_t)W.nx * W.ny * W.nz;
        if (n * 19 >= (1ll << 31))
            return fail(PSC_E_UNSUPPORTED, "psc_plan_row_tiles: a window must hold fewer than 2^31/19 cells");
        if (((int64_t)W.nz * elem_bytes) % 16 != 0)
            return fail(PSC_E_UNSUPPORTED, "psc_plan_row_tiles: nz * elem_bytes must be a multiple of 16 (window " +
                                               std::to_string(w) + ")");
        const int geo_bytes = W.level ? 1 : 8;  // uint8 level or FP64 solid rides in the stage
        if (!W.level && !W.solid) return fail(PSC_E_INVALID, "psc_plan_row_tiles: window without level or solid");
        if (((int64_t)W.nz * geo_bytes) % 16 != 0)
            return fail(PSC_E_UNSUPPORTED, std::string("psc_plan_row_tiles: the ") + (W.level ? "uint8 level" : "FP64 solid") +
                                               " rows need nz * " + std::to_string(geo_bytes) +
                                               " to be a multiple of 16 (window " + std::to_string(w) + ")");
        if ((reinterpret_cast<uintptr_t>(W.level ? (const void*)W.level : (const void*)W.solid)) % 16 != 0)
            return fail(PSC_E_UNSUPPORTED, "psc_plan_row_tiles: level / solid buffers must be 16-byte aligned");
        if ((reinterpret_cast<uintptr_t>(W.f_src) | reinterpret_cast<uintptr_t>(W.f_dst)) % 16 != 0)
            return fail(PSC_E_UNSUPPORTED, "psc_plan_row_tiles: population buffers must be 16-byte aligned");
        int ty = rows;
        if (ty == -1) {  // keep the rows preset in tile_cells (= rows * nz)
            if (W.tile_cells <= 0 || W.tile_cells % W.nz != 0)
                return fail(PSC_E_INVALID, "psc_plan_row_tiles: rows = -1 needs tile_cells = rows * nz preset");
            ty = W.tile_cells / W.nz;
        }
        if (ty == 0) {  // ~24 kB per stage: three stages and two CTAs fit on one SM
            ty = (int)((24 * 1024) / ((int64_t)W.nz * (19 * elem_bytes + geo_bytes)));
            if (ty < 1) ty = 1;
        }
        if (ty > W.ny) ty = W.ny;
        const int64_t bytes = (int64_t)ty * W.nz * (19 * elem_bytes + geo_bytes);
        if (bytes > 96 * 1024)
            return fail(PSC_E_UNSUPPORTED, "psc_plan_row_tiles: a row tile needs more than 96 kB of shared memory");
        if (ty * W.nz > 4096)
            return fail(PSC_E_UNSUPPORTED, "psc_plan_row_tiles: more than 4096 cells per row tile");
        W.tile_cells = ty * W.nz;
        W.tile_begin = begin;
        W.tile_count = (int64_t)W.nx * ((W.ny + ty - 1) / ty);
        begin += W.tile_count;
        if (bytes > stage) stage = bytes;
    }
    *h_total_tiles = begin;
    *h_stage_bytes = (int32_t)((stage + 127) / 128 * 128);
    return PSC_OK;
}

int psc_device_status(int* h_status, int clear) {
    if (!h_status) return fail(PSC_E_INVALID, "psc_device_status: null output");
    int tma = 0, pair = 0, loads = 0;
    cudaError_t e = read_device_status(&tma, clear != 0);
    if (e == cudaSuccess) e = read_pair_status(&pair, clear != 0);
    if (e == cudaSuccess) e = read_loads_status(&loads, clear != 0);
    *h_status = tma ? tma : (pair ? pair : loads);
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_device_status");
}

int psc_plan_pair_tiles(psc_window* h_windows, int nwin, int64_t* h_total_tiles) {
    if (!h_windows || nwin <= 0 || !h_total_tiles) return fail(PSC_E_INVALID, "psc_plan_pair_tiles: bad arguments");
    for (int w = 0; w < nwin; ++w)
        if (h_windows[w].nz % 2 != 0)
            return fail(PSC_E_UNSUPPORTED, "psc_plan_pair_tiles: the pair kernel needs an even nz (window " +
                                               std::to_string(w) + ")");
    return psc_plan_tiles(h_windows, nwin, 2 * STEP_THREADS, h_total_tiles);
}

int psc_init_equilibrium(int store, double store_scale, void* f, int64_t ncells, void* stream) {
    if (!valid_store(store)) return fail(PSC_E_INVALID, "psc_init_equilibrium: unknown storage mode");
    if (!f || ncells <= 0) return fail(PSC_E_INVALID, "psc_init_equilibrium: null buffer or empty lattice");
    cudaError_t e = launch_init_equilibrium(store, store_scale, f, ncells, as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_init_equilibrium");
}

int psc_geometry_plan(const psc_geometry* h_geo, void* stream) {
    int st = check_geometry(h_geo, "psc_geometry_plan");
    if (st) return st;
    cudaError_t e = launch_geometry_plan(*h_geo, as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_geometry_plan");
}

int psc_geometry_build(const psc_geometry* h_geo, void* stream) {
    int st = check_geometry(h_geo, "psc_geometry_build");
    if (st) return st;
    const psc_geometry& g = *h_geo;
    if (!g.cell_n || !g.cell_off || !g.alpha_sum || !g.solid || !g.scan_tmp)
        return fail(PSC_E_INVALID, "psc_geometry_build: null cell array");
    if (g.capacity_entries > 0 && (!g.ent_cnt || !g.cl_pid || !g.cl_cnt))
        return fail(PSC_E_INVALID, "psc_geometry_build: null entry array");
    if (g.level && g.subsamples * g.subsamples * g.subsamples > 255)
        return fail(PSC_E_UNSUPPORTED, "psc_geometry_build: the uint8 level field needs subsamples <= 6");
    if (g.smooth_eps < 0.0 || !(g.smooth_eps == g.smooth_eps))
        return fail(PSC_E_INVALID, "psc_geometry_build: smooth_eps must be >= 0");
    if (g.smooth_eps > 0.0 && g.capacity_entries > 0 && (!g.ent_alpha || !g.cl_ent))
        return fail(PSC_E_INVALID, "psc_geometry_build: smooth mode needs ent_alpha and cl_ent");
    if (g.smooth_eps > 0.0 && g.level)
        return fail(PSC_E_INVALID, "psc_geometry_build: smooth mode has no integer level (pass level = NULL)");
    cudaError_t e = launch_geometry_build(g, as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_geometry_build");
}

int psc_solid_velocity(const psc_geometry* h_geo, int us_type, void* us, void* stream) {
    int st = check_geometry(h_geo, "psc_solid_velocity");
    if (st) return st;
    if (!us || (us_type != 0 && us_type != 1)) return fail(PSC_E_INVALID, "psc_solid_velocity: bad output");
    cudaError_t e = launch_solid_velocity(*h_geo, us_type, us, as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_solid_velocity");
}

int psc_step_windows_ex(int store, const psc_window* d_windows, int nwin, int64_t total_tiles, unsigned flags,
                const psc_launch* cfg, void* stream) {
    if (!valid_store(store)) return fail(PSC_E_INVALID, "psc_step_windows: unknown storage mode");
    if (!d_windows || nwin <= 0 || total_tiles < 0) return fail(PSC_E_INVALID, "psc_step_windows: bad window list");
    psc_launch c = {0, 1, PSC_KERNEL_AUTO, 0, 0};
    if (cfg) c = *cfg;
    if (c.grid_ctas < 0) return fail(PSC_E_INVALID, "psc_step_windows: grid_ctas must be >= 0");
    if (c.cells_per_thread != 1 && c.cells_per_thread != 2 && c.cells_per_thread != 4)
        return fail(PSC_E_INVALID, "psc_step_windows: cells_per_thread must be 1, 2 or 4");
    const bool moving = (flags & PSC_STEP_MOVING) != 0;
    cudaError_t e;
    if (store == PSC_STORE_F64_EXACT) {
        // (TRT windows are rejected by the hosts that build tables; the exact kernel runs BGK)
        if (c.cells_per_thread != 1)
            return fail(PSC_E_UNSUPPORTED, "psc_step_windows: PSC_STORE_F64_EXACT runs one cell per thread");
        e = launch_step(store, d_windows, nwin, total_tiles, flags, moving, c.grid_ctas, as_stream(stream));
    } else if (c.kernel == PSC_KERNEL_AUTO || c.kernel == PSC_KERNEL_DIRECT) {
        e = launch_step_fast(store, d_windows, nwin, total_tiles, flags, moving, c.cells_per_thread, c.grid_ctas,
                             as_stream(stream));
    } else if (c.kernel == PSC_KERNEL_PAIR) {
        e = launch_step_pair(store, d_windows, nwin, total_tiles, flags, moving, c.grid_ctas, as_stream(stream));
    } else if (c.kernel == PSC_KERNEL_TMA) {
        const int stages = c.stages == 0 ? 3 : c.stages;
        if (stages < 2 || stages > 4) return fail(PSC_E_INVALID, "psc_step_windows: TMA stages must be 2, 3 or 4");
        if (c.stage_bytes <= 0 || c.stage_bytes % 16 != 0 || (int64_t)stages * c.stage_bytes > 200 * 1024)
            return fail(PSC_E_INVALID, "psc_step_windows: bad TMA stage_bytes (use psc_plan_row_tiles)");
        e = launch_step_tma(store, d_windows, nwin, total_tiles, flags, moving, c.grid_ctas, stages,
                            (uint32_t)c.stage_bytes, as_stream(stream));
    } else {
        return fail(PSC_E_UNSUPPORTED, "psc_step_windows: unknown kernel variant");
    }
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_step_windows");
}

int psc_step_windows(int store, const psc_window* d_windows, int nwin, int64_t total_tiles, unsigned flags, int grid_ctas,
             void* stream) {
    psc_launch c = {grid_ctas, 1, PSC_KERNEL_AUTO, 0, 0};
    return psc_step_windows_ex(store, d_windows, nwin, total_tiles, flags, &c, stream);
}

int psc_reduce_windows(const psc_window* d_windows, int nwin, double* out, void* stream) {
    if (!d_windows || nwin <= 0 || !out) return fail(PSC_E_INVALID, "psc_reduce_windows: bad arguments");
    if (nwin > 65535) return fail(PSC_E_UNSUPPORTED, "psc_reduce_windows: at most 65535 windows per call");
    cudaError_t e = launch_reduce_windows(d_windows, nwin, out, as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_reduce_windows");
}

int psc_particle_loads(const psc_geometry* h_geo, int imb_type, const void* imb, double* chunk_partials,
                       const double* imb_sums, double* forces, double* torques, double* diag, void* stream) {
    int st = check_geometry(h_geo, "psc_particle_loads");
    if (st) return st;
    if (imb_type != 0 && imb_type != 1) return fail(PSC_E_INVALID, "psc_particle_loads: imb_type must be 0 or 1");
    if (!imb_sums || !diag) return fail(PSC_E_INVALID, "psc_particle_loads: null imb_sums / diag");
    if (h_geo->nparticles > 0 && (!imb || !forces || !torques || !h_geo->ent_cnt || !h_geo->alpha_sum))
        return fail(PSC_E_INVALID, "psc_particle_loads: null array");
    if (h_geo->nparticles > 0 && h_geo->capacity_chunks > 0 && !chunk_partials)
        return fail(PSC_E_INVALID, "psc_particle_loads: null chunk partials");
    // the entry gathers are asynchronous copies of whole elements (counts as aligned pairs)
    if (h_geo->nparticles > 0 &&
        ((uintptr_t)h_geo->ent_cnt % 4 || (uintptr_t)h_geo->alpha_sum % 8 || (uintptr_t)imb % (imb_type == 0 ? 8 : 4)))
        return fail(PSC_E_INVALID,
                    "psc_particle_loads: ent_cnt must be 4-byte aligned, alpha_sum and the IMB field element-aligned");
    const int lists = (h_geo->load_w != nullptr) + (h_geo->load_abk != nullptr) + (h_geo->load_n != nullptr);
    if (lists != 0 && lists != 3)
        return fail(PSC_E_INVALID, "psc_particle_loads: give all three loads-list arrays or none");
    if (lists == 3 && (h_geo->chunk_entries % PSC_LOAD_THREADS != 0 || h_geo->chunk_entries / PSC_LOAD_THREADS > 16 ||
                       h_geo->nx > 2048 || h_geo->ny > 2048 || h_geo->nz > 1024))
        return fail(PSC_E_INVALID, "psc_particle_loads: the loads list needs chunk_entries a multiple of "
                                   "PSC_LOAD_THREADS (at most 16 of them) and nx, ny <= 2048, nz <= 1024");
    if (lists == 0 && h_geo->list_ready)
        return fail(PSC_E_INVALID, "psc_particle_loads: list_ready without the loads-list arrays");
    cudaError_t e = launch_particle_loads(*h_geo, imb_type, imb, chunk_partials, imb_sums, forces, torques, diag,
                                          as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_particle_loads");
}

static int check_adjoint(const psc_adjoint_args* a, const char* who, bool need_in) {
    if (!a) return fail(PSC_E_INVALID, std::string(who) + ": null args");
    int st = check_extent(a->nx, a->ny, a->nz, who);
    if (st) return st;
    if (a->store != PSC_STORE_F64 && a->store != PSC_STORE_F32)
        return fail(PSC_E_UNSUPPORTED, std::string(who) + ": the adjoint supports PSC_STORE_F64 and PSC_STORE_F32");
    if (!(a->tau > 0.5)) return fail(PSC_E_INVALID, std::string(who) + ": tau must exceed 0.5");
    if (!a->state || !a->solid || !a->lam_out || !a->dKdB || !a->dKdsolid || (need_in && !a->lam_in))
        return fail(PSC_E_INVALID, std::string(who) + ": null array");
    if (need_in && a->lam_in == a->lam_out)
        return fail(PSC_E_INVALID, std::string(who) + ": lam_in and lam_out must differ (scattered stores)");
    return PSC_OK;
}

int psc_adjoint_seed(const psc_adjoint_args* h_args, void* stream) {
    int st = check_adjoint(h_args, "psc_adjoint_seed", false);
    if (st) return st;
    cudaError_t e = launch_adjoint_seed(*h_args, as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_adjoint_seed");
}

int psc_adjoint_step(const psc_adjoint_args* h_args, void* stream) {
    int st = check_adjoint(h_args, "psc_adjoint_step", true);
    if (st) return st;
    cudaError_t e = launch_adjoint_step(*h_args, as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_adjoint_step");
}

int psc_adjoint_geometry_grad(const psc_geometry* h_geo, const psc_adjoint_args* h_args, double* chunk_partials,
                              double* grad, void* stream) {
    int st = check_geometry(h_geo, "psc_adjoint_geometry_grad");
    if (st) return st;
    if (!(h_geo->smooth_eps > 0.0))
        return fail(PSC_E_INVALID, "psc_adjoint_geometry_grad: needs a smooth geometry (smooth_eps > 0)");
    if (!h_args || !h_args->dKdB || !h_args->dKdsolid || !h_geo->alpha_sum)
        return fail(PSC_E_INVALID, "psc_adjoint_geometry_grad: null array");
    if (h_geo->nparticles > 0 && (!grad || (h_geo->capacity_chunks > 0 && !chunk_partials)))
        return fail(PSC_E_INVALID, "psc_adjoint_geometry_grad: null output");
    cudaError_t e = launch_adjoint_geometry_grad(*h_geo, *h_args, chunk_partials, grad, as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_adjoint_geometry_grad");
}

int psc_equilibrium(const double* rho, const double* ux, const double* uy, const double* uz, double* out, int64_t n,
                    void* stream) {
    if (n < 0 || (n > 0 && (!rho || !ux || !uy || !uz || !out)))
        return fail(PSC_E_INVALID, "psc_equilibrium: bad arguments");
    if (n == 0) return PSC_OK;
    cudaError_t e = launch_equilibrium(rho, ux, uy, uz, out, n, as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_equilibrium");
}

int psc_guo_force(double fx, double fy, double fz, const double* ux, const double* uy, const double* uz, double tau,
                  double* out, int64_t n, void* stream) {
    if (n < 0 || (n > 0 && (!ux || !uy || !uz || !out))) return fail(PSC_E_INVALID, "psc_guo_force: bad arguments");
    if (n == 0) return PSC_OK;
    cudaError_t e = launch_guo(fx, fy, fz, ux, uy, uz, tau, out, n, as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_guo_force");
}

int psc_voxelize_spheres(const double* d_points, int M, const double* h_lo, const double* h_dx, double radius,
                         int nx, int ny, int nz, uint8_t* solid, void* stream) {
    int st = check_extent(nx, ny, nz, "psc_voxelize_spheres");
    if (st) return st;
    if (M < 0 || (M > 0 && !d_points) || !h_lo || !h_dx || !solid)
        return fail(PSC_E_INVALID, "psc_voxelize_spheres: bad arguments");
    if (!(h_dx[0] > 0.0 && h_dx[1] > 0.0 && h_dx[2] > 0.0) || !(radius == radius))
        return fail(PSC_E_INVALID, "psc_voxelize_spheres: cell sizes must be > 0");
    cudaError_t e = launch_vox_spheres(d_points, M, h_lo, h_dx, radius, nx, ny, nz, solid, as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_voxelize_spheres");
}

int psc_bounceback_step(const double* f_src, double* f_dst, const uint8_t* solid, int nx, int ny, int nz, double tau,
                        double fx, double fy, double fz, unsigned flags, double* moments, void* stream) {
    int st = check_extent(nx, ny, nz, "psc_bounceback_step");
    if (st) return st;
    if (!f_src || !solid || ((flags & PSC_STEP_COLLIDE) && (!f_dst || f_dst == f_src)) ||
        ((flags & PSC_STEP_MOMENTS) && !moments))
        return fail(PSC_E_INVALID, "psc_bounceback_step: bad buffers");
    if (!(tau > 0.5)) return fail(PSC_E_INVALID, "psc_bounceback_step: tau must exceed 0.5");
    cudaError_t e = launch_bb_step(f_src, f_dst, solid, nx, ny, nz, tau, fx, fy, fz, flags, moments,
                                   as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_bounceback_step");
}

int psc_stream_push(int store, double store_scale, const void* src, double* dst, int nx, int ny, int nz,
                    void* stream) {
    if (!valid_store(store) || !src || !dst) return fail(PSC_E_INVALID, "psc_stream_push: bad arguments");
    int st = check_extent(nx, ny, nz, "psc_stream_push");
    if (st) return st;
    if (store_scale == 0.0) return fail(PSC_E_INVALID, "psc_stream_push: zero store_scale");
    cudaError_t e = launch_stream_push(store, store_scale, src, dst, nx, ny, nz, as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_stream_push");
}

int psc_stream_push_open(int store, double store_scale, const void* src, double* dst, int nx, int ny, int nz,
                         double inlet_rho, const double* h_inlet_u, void* stream) {
    if (!valid_store(store) || !src || !dst || !h_inlet_u)
        return fail(PSC_E_INVALID, "psc_stream_push_open: bad arguments");
    int st = check_extent(nx, ny, nz, "psc_stream_push_open");
    if (st) return st;
    if (store_scale == 0.0) return fail(PSC_E_INVALID, "psc_stream_push_open: zero store_scale");
    const double inlet[4] = {inlet_rho, h_inlet_u[0], h_inlet_u[1], h_inlet_u[2]};
    cudaError_t e = launch_stream_push(store, store_scale, src, dst, nx, ny, nz, as_stream(stream), true, inlet);
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_stream_push_open");
}

int psc_stream_pull_store(int store, double store_scale, const double* src, void* dst, int nx, int ny, int nz,
                          void* stream) {
    if (!valid_store(store) || !src || !dst) return fail(PSC_E_INVALID, "psc_stream_pull_store: bad arguments");
    int st = check_extent(nx, ny, nz, "psc_stream_pull_store");
    if (st) return st;
    cudaError_t e = launch_stream_pull_store(store, store_scale, src, dst, nx, ny, nz, as_stream(stream));
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_stream_pull_store");
}

int psc_stream_pull_store_open(int store, double store_scale, const double* src, void* dst, int nx, int ny, int nz,
                               double inlet_rho, const double* h_inlet_u, void* stream) {
    if (!valid_store(store) || !src || !dst || !h_inlet_u)
        return fail(PSC_E_INVALID, "psc_stream_pull_store_open: bad arguments");
    int st = check_extent(nx, ny, nz, "psc_stream_pull_store_open");
    if (st) return st;
    const double inlet[4] = {inlet_rho, h_inlet_u[0], h_inlet_u[1], h_inlet_u[2]};
    cudaError_t e =
        launch_stream_pull_store(store, store_scale, src, dst, nx, ny, nz, as_stream(stream), true, inlet);
    return e == cudaSuccess ? PSC_OK : cuda_fail(e, "psc_stream_pull_store_open");
}

}  // extern "C"
