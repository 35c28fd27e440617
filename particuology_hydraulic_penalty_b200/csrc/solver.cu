// Handle layer of libpscb200.so: the reference's solver object
// (PscD3Q19 / SparsePscD3Q19, src/lbm_dem/psc3d.py:117-407) and batches of
// windows stepped by one persistent launch, written as a native runtime.
//
// A handle owns its device buffers, its stream and its CUDA graphs, and
// drives the descriptor-layer kernels (geometry, step, reductions, loads) in
// the order of collide_stream_psc (psc3d.py:208-253):
//   voxelise (if the particles changed and the geometry is not static)
//   -> solid velocity (if a particle moves)
//   -> fused pull-stream + collide (+ IMB momentum, + per-tile reductions)
//   -> particle loads -> reductions of the post-stream state -> diagnostics.
// One call runs any number of steps with no host work between them except
// where the caller asks for per-step diagnostics (the lbm_converge loop).
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "internal.cuh"

namespace psc {
namespace {

#define PSC_TRY(expr)                  \
    do {                               \
        int psc_try_st_ = (expr);      \
        if (psc_try_st_ != PSC_OK) return psc_try_st_; \
    } while (0)
#define PSC_CUDA(expr, what)                             \
    do {                                                 \
        cudaError_t psc_cuda_e_ = (expr);                \
        if (psc_cuda_e_ != cudaSuccess) return cuda_fail(psc_cuda_e_, what); \
    } while (0)

constexpr int kQ = 19;
constexpr int kChunkEntries = 4096;  // bbox entries per load-reduction chunk
static_assert(kChunkEntries % PSC_LOAD_THREADS == 0 && kChunkEntries / PSC_LOAD_THREADS <= 16,
              "the loads list holds at most 16 entries per thread and chunk");
constexpr int kOutLen = 2 * PSC_NRED + PSC_NDIAG;  // [red_pre][red_post][diag]

// Owned device array (contents are not kept when it grows).  A grow allocates
// the new block before it frees the old one, so a failed grow leaves the array
// (and every pointer to it) as it was.
template <class T>
struct DArray {
    T* p = nullptr;
    int64_t n = 0;
    DArray() = default;
    DArray(const DArray&) = delete;
    DArray& operator=(const DArray&) = delete;
    ~DArray() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t ensure(int64_t m, bool zero, cudaStream_t s) {
        if (m < 1) m = 1;
        if (p && m <= n) return cudaSuccess;
        T* q = nullptr;
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&q), (size_t)m * sizeof(T));
        if (e != cudaSuccess) return e;
        release();
        p = q;
        n = m;
        return zero ? cudaMemsetAsync(p, 0, (size_t)m * sizeof(T), s) : cudaSuccess;
    }
};

// Owned page-locked host array.
template <class T>
struct HArray {
    T* p = nullptr;
    int64_t n = 0;
    HArray() = default;
    HArray(const HArray&) = delete;
    HArray& operator=(const HArray&) = delete;
    ~HArray() {
        if (p) cudaFreeHost(p);
    }
    cudaError_t ensure(int64_t m) {
        if (m < 1) m = 1;
        if (p && m <= n) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&p), (size_t)m * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            return e;
        }
        n = m;
        return cudaSuccess;
    }
};

// Makes the handle's device current for the duration of a call.
struct DeviceScope {
    int prev = -1;
    bool changed = false;
    cudaError_t err = cudaSuccess;
    explicit DeviceScope(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) {
            err = cudaSetDevice(dev);
            changed = err == cudaSuccess;
        }
    }
    ~DeviceScope() {
        if (changed && prev >= 0) cudaSetDevice(prev);
    }
};

// Keeps a handle's last error: every error set on this thread while the
// guard lives (one call on the handle) is copied into the handle's message.
struct ErrorCapture {
    std::string* dst;
    uint64_t seq0;
    explicit ErrorCapture(std::string& d) : dst(&d), seq0(error_seq()) {}
    ~ErrorCapture() {
        if (error_seq() != seq0) *dst = last_error_string();
    }
};

// Auxiliary streams of a handle for work of one step that is independent of
// the main stream's (particle loads beside the post-stream reduction pass):
// begin() makes every lane wait for the main stream's work so far, end()
// makes the main stream wait for every lane.
struct Lanes {
    static constexpr int kMax = 4;
    int n = 0;
    cudaStream_t s[kMax] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[kMax] = {};
    Lanes() = default;
    Lanes(const Lanes&) = delete;
    Lanes& operator=(const Lanes&) = delete;
    ~Lanes() {
        for (int i = 0; i < n; ++i) {
            if (s[i]) cudaStreamDestroy(s[i]);
            if (join[i]) cudaEventDestroy(join[i]);
        }
        if (fork) cudaEventDestroy(fork);
    }
    cudaError_t init(int count) {
        cudaError_t e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
        for (int i = 0; i < count && i < kMax && e == cudaSuccess; ++i) {
            e = cudaStreamCreateWithFlags(&s[i], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming);
            if (e == cudaSuccess) n = i + 1;
        }
        return e;
    }
    cudaStream_t lane(int k) const { return s[k % n]; }
    cudaError_t begin(cudaStream_t main) {
        cudaError_t e = cudaEventRecord(fork, main);
        for (int i = 0; i < n && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(s[i], fork, 0);
        return e;
    }
    cudaError_t end(cudaStream_t main) {
        cudaError_t e = cudaSuccess;
        for (int i = 0; i < n && e == cudaSuccess; ++i) {
            e = cudaEventRecord(join[i], s[i]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(main, join[i], 0);
        }
        return e;
    }
};

int store_elem_bytes(int store) {
    switch (store) {
        case PSC_STORE_F64_EXACT:
        case PSC_STORE_F64: return 8;
        case PSC_STORE_F32: return 4;
        default: return 2;
    }
}

double default_store_scale(int store) { return store == PSC_STORE_F16 ? 1048576.0 : 1.0; }  // FP16: 2^20

bool finite3(const double* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

int check_config(const psc_config& c, const char* who) {
    const std::string w(who);
    if (c.nx <= 0 || c.ny <= 0 || c.nz <= 0) return fail(PSC_E_INVALID, w + ": lattice extents must be > 0");
    const long long n = (long long)c.nx * c.ny * c.nz;
    if (n * kQ >= (1ll << 31)) return fail(PSC_E_UNSUPPORTED, w + ": a window must hold fewer than 2^31 / 19 cells");
    if (c.store < PSC_STORE_F64_EXACT || c.store > PSC_STORE_BF16) return fail(PSC_E_INVALID, w + ": unknown store");
    if (c.subsamples < 1 || c.subsamples > 16) return fail(PSC_E_INVALID, w + ": subsamples must be in [1, 16]");
    if (c.store != PSC_STORE_F64_EXACT && c.subsamples > 6)
        return fail(PSC_E_UNSUPPORTED, w + ": the deviation storage modes keep the solid level as uint8 (subsamples <= 6)");
    if (!(std::isfinite(c.tau) && c.tau > 0.0)) return fail(PSC_E_INVALID, w + ": tau must be a positive number");
    if (!(std::isfinite(c.tau_minus) && c.tau_minus >= 0.0)) return fail(PSC_E_INVALID, w + ": tau_minus must be >= 0");
    if (c.tau_minus > 0.0 && c.store == PSC_STORE_F64_EXACT)
        return fail(PSC_E_UNSUPPORTED, w + ": TRT runs in the deviation storage modes only");
    if (!finite3(c.force)) return fail(PSC_E_INVALID, w + ": the body force must be finite");
    if (!(std::isfinite(c.store_scale) && c.store_scale >= 0.0))
        return fail(PSC_E_INVALID, w + ": store_scale must be >= 0 (0 = default)");
    if (!(std::isfinite(c.conv_tol) && c.conv_tol >= 0.0)) return fail(PSC_E_INVALID, w + ": conv_tol must be >= 0");
    if (c.conv_check_every < 0) return fail(PSC_E_INVALID, w + ": conv_check_every must be >= 0");
    if (c.device < 0) return fail(PSC_E_INVALID, w + ": negative device ordinal");
    if (c.open_x != 0 && c.open_x != 1) return fail(PSC_E_INVALID, w + ": open_x must be 0 or 1");
    if (c.open_x && !(std::isfinite(c.inlet_rho) && c.inlet_rho > 0.0 && finite3(c.inlet_u)))
        return fail(PSC_E_INVALID, w + ": open_x needs a positive inlet_rho and a finite inlet_u");
    return PSC_OK;
}

// ---------------------------------------------------------------------------
// one window: populations, per-cell fields and particle geometry
// ---------------------------------------------------------------------------
struct Window {
    psc_config cfg{};
    int64_t N = 0;
    int elem = 8;          // bytes per stored population
    bool fdouble = true;   // imb / moments / us element type: double (FP64 modes) or float
    double scale = 1.0;
    bool want_level = false;
    DArray<unsigned char> f[2];
    int cur = 0;           // buffer holding the current post-collision populations
    DArray<unsigned char> imb, moments, us;
    // A batch window keeps one IMB field per buffer parity: a step into buffer
    // c writes imb_for(c), so the IMB of the current state (imb_for(cur))
    // survives a step run ahead into the other buffer.  A solver window keeps one.
    DArray<unsigned char> imb_alt;
    bool imb_dual = false;
    int imb_par = 0;  // imb_dual: parity of the IMB field of the last step that wrote one
    unsigned char* imb_for(int c) const { return (imb_dual && c == 1) ? imb_alt.p : imb.p; }
    DArray<double> partials;
    int64_t partials_cap = 0;  // tiles the partial buffer holds
    int64_t solo_tiles = 0;
    DArray<psc_window> solo[2];  // single-window descriptor table per parity
    int solo_kernel = PSC_KERNEL_AUTO;  // kernel of the single-window launches
    bool solo_dirty = true;
    uint64_t desc_version = 1;   // bumped whenever a descriptor field changes
    // particles and geometry
    int P = 0;
    std::vector<double> hp;
    HArray<double> pinned;
    cudaEvent_t upload_done = nullptr;
    DArray<double> particles;
    const double* ext_particles = nullptr;  // a batch's shared upload buffer (psc_batch_set_particles_all)
    DArray<int32_t> bbox;
    DArray<int64_t> ent_off, chunk_off, totals;
    DArray<uint16_t> ent_cnt, cl_cnt;
    DArray<int32_t> cell_n, cell_off, cl_pid;
    DArray<double> alpha_sum, solid;
    DArray<uint8_t> level;
    DArray<unsigned char> scan_tmp;
    DArray<double> chunk_partials;
    double smooth_eps = 0.0;  // > 0: smooth solid fraction (the adjoint's differentiable surrogate)
    DArray<double> ent_alpha;
    DArray<int32_t> cl_ent;
    // loads list (owner weights and cells of the non-zero bbox entries), written
    // by the first loads call on a geometry and read by the later ones
    // (list_version == built_version); kept only where the list's packing fits
    DArray<double> load_w;
    DArray<uint32_t> load_abk;
    DArray<uint8_t> load_n;
    uint64_t list_version = 0;
    int64_t cap_entries = 0, cap_chunks = 0, n_entries = 0, n_chunks = 0;
    DArray<double> forces, torques;
    uint64_t pversion = 1, built_version = 0, us_version = 0;
    bool built = false;
    bool moving = false;
    // state of the last step's results
    bool stepped = false, moments_ready = false, loads_ready = false, diag_ready = false;
    DArray<double> out;  // [red_pre][red_post][diag]
    psc_diag last{};

    ~Window() {
        if (upload_done) cudaEventDestroy(upload_done);
    }

    void touch() {
        solo_dirty = true;
        ++desc_version;
    }
    size_t field_bytes() const { return fdouble ? 8 : 4; }
    int field_type() const { return fdouble ? 0 : 1; }  // imb_type / us_type of the descriptor layer

    psc_geometry geometry() const {
        psc_geometry g{};
        g.nx = cfg.nx;
        g.ny = cfg.ny;
        g.nz = cfg.nz;
        g.subsamples = cfg.subsamples;
        g.nparticles = P;
        g.chunk_entries = kChunkEntries;
        g.capacity_entries = cap_entries;
        g.capacity_chunks = cap_chunks;
        g.particles = P ? (ext_particles ? ext_particles : particles.p) : nullptr;
        g.bbox = bbox.p;
        g.ent_off = ent_off.p;
        g.chunk_off = chunk_off.p;
        g.totals = totals.p;
        g.ent_cnt = cap_entries ? ent_cnt.p : nullptr;
        g.cell_n = cell_n.p;
        g.cell_off = cell_off.p;
        g.cl_pid = cap_entries ? cl_pid.p : nullptr;
        g.cl_cnt = cap_entries ? cl_cnt.p : nullptr;
        g.alpha_sum = alpha_sum.p;
        g.solid = solid.p;
        g.level = want_level ? level.p : nullptr;
        g.scan_tmp = scan_tmp.p;
        g.smooth_eps = smooth_eps;
        g.ent_alpha = smooth_eps > 0.0 && cap_entries ? ent_alpha.p : nullptr;
        g.cl_ent = smooth_eps > 0.0 && cap_entries ? cl_ent.p : nullptr;
        const bool list = list_allowed() && cap_chunks && load_n.p;
        g.load_w = list ? load_w.p : nullptr;
        g.load_abk = list ? load_abk.p : nullptr;
        g.load_n = list ? load_n.p : nullptr;
        g.list_ready = list && built && list_version == built_version ? 1 : 0;
        return g;
    }
    // The loads list packs bbox-local cells into 11 + 11 + 10 bits.
    bool list_allowed() const { return !(smooth_eps > 0.0) && cfg.nx <= 2048 && cfg.ny <= 2048 && cfg.nz <= 1024; }
    // A loads launch with geometry() has been enqueued: the list it writes is
    // what the next launches on this geometry read (stream order).
    void loads_enqueued() {
        if (load_n.p && built) list_version = built_version;
    }

    // Descriptor reading buffer `src` (tile fields unset).
    psc_window descriptor(int src) const {
        psc_window d{};
        d.nx = cfg.nx;
        d.ny = cfg.ny;
        d.nz = cfg.nz;
        d.subsamples = cfg.subsamples;
        d.flags = (moving ? PSC_WIN_MOVING : 0) | (cfg.open_x ? PSC_WIN_OPEN_X : 0);
        d.tau = cfg.tau;
        d.force[0] = cfg.force[0];
        d.force[1] = cfg.force[1];
        d.force[2] = cfg.force[2];
        d.store_scale = scale;
        d.f_src = f[src].p;
        d.f_dst = f[1 - src].p;
        d.solid = solid.p;
        d.level = want_level ? level.p : nullptr;
        d.us = moving ? us.p : nullptr;
        d.imb = imb_for(1 - src);
        d.moments = moments.p;
        d.partials = partials.p;
        d.tau_minus = cfg.tau_minus;
        d.inlet_rho = cfg.open_x ? cfg.inlet_rho : 1.0;
        d.inlet_u[0] = cfg.open_x ? cfg.inlet_u[0] : 0.0;
        d.inlet_u[1] = cfg.open_x ? cfg.inlet_u[1] : 0.0;
        d.inlet_u[2] = cfg.open_x ? cfg.inlet_u[2] : 0.0;
        return d;
    }
};

int window_init(Window& w, const psc_config& c, cudaStream_t s, const char* who) {
    PSC_TRY(check_config(c, who));
    w.cfg = c;
    w.N = (int64_t)c.nx * c.ny * c.nz;
    w.elem = store_elem_bytes(c.store);
    w.fdouble = c.store == PSC_STORE_F64_EXACT || c.store == PSC_STORE_F64;
    w.scale = c.store_scale > 0.0 ? c.store_scale : default_store_scale(c.store);
    w.want_level = c.store != PSC_STORE_F64_EXACT && !(w.smooth_eps > 0.0);
    const int64_t N = w.N;
    PSC_CUDA(w.f[0].ensure(kQ * N * w.elem, false, s), who);
    PSC_CUDA(w.f[1].ensure(kQ * N * w.elem, false, s), who);
    PSC_TRY(psc_init_equilibrium(c.store, w.scale, w.f[0].p, N, s));
    PSC_CUDA(w.cell_n.ensure(N, true, s), who);
    PSC_CUDA(w.cell_off.ensure(N + 1, true, s), who);
    PSC_CUDA(w.alpha_sum.ensure(N, true, s), who);
    PSC_CUDA(w.solid.ensure(N, true, s), who);
    if (w.want_level) PSC_CUDA(w.level.ensure(N, true, s), who);
    PSC_CUDA(w.scan_tmp.ensure((int64_t)scan_tmp_bytes(N + 1), false, s), who);
    PSC_CUDA(w.totals.ensure(4, true, s), who);
    PSC_CUDA(w.ent_off.ensure(1, true, s), who);
    PSC_CUDA(w.chunk_off.ensure(1, true, s), who);
    PSC_CUDA(w.bbox.ensure(6, true, s), who);
    PSC_CUDA(w.out.ensure(kOutLen, true, s), who);
    // per-tile partials, sized once for any tiling of the window: 256-cell
    // tiles (ceil(N / 256)) or row tiles (at most nx * ny); descriptor tables
    // keep this pointer, so it never moves
    w.partials_cap = std::max<int64_t>((N + 255) / 256, (int64_t)c.nx * c.ny);
    PSC_CUDA(w.partials.ensure((1 + w.partials_cap * PSC_PARTIAL_ROWS) * PSC_NRED, true, s), who);
    PSC_CUDA(cudaEventCreateWithFlags(&w.upload_done, cudaEventDisableTiming), who);
    return PSC_OK;
}

int window_ensure_imb(Window& w, cudaStream_t s) {
    if (w.imb.p && (!w.imb_dual || w.imb_alt.p)) return PSC_OK;
    PSC_CUDA(w.imb.ensure(3 * w.N * (int64_t)w.field_bytes(), true, s), "imb field");
    if (w.imb_dual) PSC_CUDA(w.imb_alt.ensure(3 * w.N * (int64_t)w.field_bytes(), true, s), "imb field");
    w.touch();
    return PSC_OK;
}

int window_ensure_moments(Window& w, cudaStream_t s) {
    if (w.moments.p) return PSC_OK;
    PSC_CUDA(w.moments.ensure(4 * w.N * (int64_t)w.field_bytes(), true, s), "moment fields");
    w.touch();
    return PSC_OK;
}

// Validation and bookkeeping of a new particle state (no upload): per-P
// buffers, the host copy, the change version and the moving flag.
// Copies n doubles from src to dst and reports whether src equals ref bit for
// bit: the staging copy and the unchanged-state test in one pass.
bool copy_same(double* dst, const double* src, const double* ref, size_t n) {
    uint64_t diff = 0;
    for (size_t i = 0; i < n; ++i) {
        uint64_t v, r;
        std::memcpy(&v, src + i, sizeof(v));
        std::memcpy(&r, ref + i, sizeof(r));
        std::memcpy(dst + i, &v, sizeof(v));
        diff |= v ^ r;
    }
    return diff == 0;
}

// Finiteness of a particle state (the reference fails on NaN / Inf) as one
// sum: v * 0 is NaN exactly for non-finite v.
bool particles_finite(const double* hp, size_t n) {
    double probe = 0.0;
    for (size_t i = 0; i < n; ++i) probe += hp[i] * 0.0;
    return probe == 0.0;
}

// Every fallible step a particle count of P needs (the per-particle device and
// pinned buffers), taken before any window takes a new state.  A buffer that had
// to move loses its contents, so the window's geometry and loads are made again
// from its accepted state at the next step.
int window_reserve_particles(Window& w, int P, cudaStream_t s, const char* who) {
    if (P == w.P && w.particles.p) return PSC_OK;
    PSC_CUDA(cudaEventSynchronize(w.upload_done), who);  // the old staging buffer may still be read
    const void* before[7] = {w.particles.p, w.bbox.p, w.ent_off.p, w.chunk_off.p, w.forces.p, w.torques.p, w.pinned.p};
    cudaError_t e = w.particles.ensure((int64_t)P * 10, true, s);
    if (e == cudaSuccess) e = w.bbox.ensure((int64_t)std::max(P, 1) * 6, true, s);
    if (e == cudaSuccess) e = w.ent_off.ensure((int64_t)P + 1, true, s);
    if (e == cudaSuccess) e = w.chunk_off.ensure((int64_t)P + 1, true, s);
    if (e == cudaSuccess) e = w.forces.ensure((int64_t)P * 3, true, s);
    if (e == cudaSuccess) e = w.torques.ensure((int64_t)P * 3, true, s);
    if (e == cudaSuccess) e = w.pinned.ensure((int64_t)P * 10);
    const void* after[7] = {w.particles.p, w.bbox.p, w.ent_off.p, w.chunk_off.p, w.forces.p, w.torques.p, w.pinned.p};
    if (std::memcmp(before, after, sizeof(before)) != 0) {
        w.built = false;
        w.loads_ready = false;
        w.diag_ready = false;
        w.touch();
    }
    if (e != cudaSuccess) return cuda_fail(e, who);
    return PSC_OK;
}

// known: 0 nothing known; 1 hp equals the last accepted state bit for bit
// (same count); 2 hp differs from it and is known to be finite.  With the
// buffers reserved (window_reserve_particles) and known != 0 nothing here fails.
int window_accept_particles(Window& w, const double* hp, int P, cudaStream_t s, const char* who, int known = 0) {
    if (P < 0) return fail(PSC_E_INVALID, std::string(who) + ": negative particle count");
    if (P > 0 && !hp) return fail(PSC_E_INVALID, std::string(who) + ": null particle array");
    // unchanged (bitwise) since the last upload: nothing to validate or record again
    const size_t n10 = (size_t)P * 10;
    const bool same_size = P == w.P && w.hp.size() == n10;
    const bool differs = known == 2 || !same_size ||
                         (known != 1 && n10 && std::memcmp(w.hp.data(), hp, n10 * sizeof(double)) != 0);
    bool mv = w.moving;
    if (differs) {
        if (known != 2 && !particles_finite(hp, n10))
            return fail(PSC_E_INVALID, std::string(who) + ": particle state contains NaN or Inf");
        // whether any particle moves
        mv = false;
        for (int p = 0; p < P && !mv; ++p)
            for (int k = 4; k < 10; ++k) mv = mv || hp[(size_t)p * 10 + k] != 0.0;
    }
    const bool changed = differs;
    PSC_TRY(window_reserve_particles(w, P, s, who));
    if (P != w.P) {
        w.built = false;
        w.loads_ready = false;
        w.diag_ready = false;
        w.P = P;
    }
    if (changed) {
        w.hp.assign(hp, hp + (size_t)P * 10);
        ++w.pversion;
    }
    if (mv != w.moving) {
        w.moving = mv;
        w.touch();
    }
    return PSC_OK;
}

int window_set_particles(Window& w, const double* hp, int P, cudaStream_t s, const char* who) {
    PSC_TRY(window_accept_particles(w, hp, P, s, who));
    w.ext_particles = nullptr;
    if (P > 0) {
        // every step reads the caller's current state (psc3d.py re-reads the
        // Particle3D objects each call); staged through page-locked memory
        PSC_CUDA(cudaEventSynchronize(w.upload_done), who);
        std::memcpy(w.pinned.p, hp, (size_t)P * 10 * sizeof(double));
        PSC_CUDA(cudaMemcpyAsync(w.particles.p, w.pinned.p, (size_t)P * 10 * sizeof(double), cudaMemcpyHostToDevice, s),
                 who);
        PSC_CUDA(cudaEventRecord(w.upload_done, s), who);
    }
    return PSC_OK;
}

// A geometry rebuild in two halves, so that a batch reads the entry and chunk
// counts of all its windows after one synchronisation: the plan (bounding
// boxes, entry and chunk offsets, totals) with the totals copied into the
// pinned slot tot4[0..3], then, once the copy has landed, the buffers grown
// to the counts and the build enqueued.
int window_rebuild_plan(Window& w, cudaStream_t s, int64_t* tot4, const char* who) {
    psc_geometry g = w.geometry();
    w.built = false;  // the plan overwrites the current geometry's offsets
    PSC_TRY(psc_geometry_plan(&g, s));
    PSC_CUDA(cudaMemcpyAsync(tot4, w.totals.p, 4 * sizeof(int64_t), cudaMemcpyDeviceToHost, s), who);
    return PSC_OK;
}

int window_rebuild_finish(Window& w, cudaStream_t s, const int64_t* tot4, const char* who) {
    w.n_entries = tot4[0];
    w.n_chunks = tot4[1];
    if (w.n_entries >= (1ll << 31) - 1)
        return fail(PSC_E_CAPACITY, std::string(who) + ": too many bounding-box entries (>= 2^31) for one window");
    if (w.n_entries > w.cap_entries) {
        const int64_t cap = std::min<int64_t>(w.n_entries + w.n_entries / 4 + 1024, (1ll << 31) - 2);
        PSC_CUDA(w.ent_cnt.ensure(cap, false, s), who);
        PSC_CUDA(w.cl_pid.ensure(cap, false, s), who);
        PSC_CUDA(w.cl_cnt.ensure(cap, false, s), who);
        if (w.smooth_eps > 0.0) {
            PSC_CUDA(w.ent_alpha.ensure(cap, false, s), who);
            PSC_CUDA(w.cl_ent.ensure(cap, false, s), who);
        }
        w.cap_entries = cap;
    }
    if (w.n_chunks > w.cap_chunks) {
        const int64_t cap = w.n_chunks + w.n_chunks / 4 + 16;
        PSC_CUDA(w.chunk_partials.ensure(cap * 6, false, s), who);
        if (w.list_allowed()) {
            PSC_CUDA(w.load_w.ensure(cap * kChunkEntries, false, s), who);
            PSC_CUDA(w.load_abk.ensure(cap * kChunkEntries, false, s), who);
            PSC_CUDA(w.load_n.ensure(cap * PSC_LOAD_THREADS, false, s), who);
        }
        w.cap_chunks = cap;
    }
    psc_geometry g = w.geometry();
    PSC_TRY(psc_geometry_build(&g, s));
    w.built = true;
    w.built_version = w.pversion;
    w.list_version = 0;
    w.us_version = 0;
    w.loads_ready = false;
    w.diag_ready = false;
    return PSC_OK;
}

int window_rebuild(Window& w, cudaStream_t s, HArray<int64_t>& tot, const char* who) {
    PSC_CUDA(tot.ensure(4), who);
    PSC_TRY(window_rebuild_plan(w, s, tot.p, who));
    PSC_CUDA(cudaStreamSynchronize(s), who);
    return window_rebuild_finish(w, s, tot.p, who);
}

int window_solid_velocity(Window& w, cudaStream_t s) {
    if (!w.us.p) {
        PSC_CUDA(w.us.ensure(3 * w.N * (int64_t)w.field_bytes(), true, s), "solid velocity");
        w.touch();
    }
    psc_geometry g = w.geometry();
    PSC_TRY(psc_solid_velocity(&g, w.field_type(), w.us.p, s));
    w.us_version = w.pversion;
    return PSC_OK;
}

// Geometry and solid velocity up to date for the next step (psc3d.py:209-210, :215).
bool window_needs_rebuild(const Window& w) {
    return !w.built || (!w.cfg.static_geometry && w.built_version != w.pversion);
}
bool window_needs_solid_velocity(const Window& w) { return w.moving && w.us_version != w.pversion; }

// Whether window_prepare will launch work that reads the particle array.
bool window_prepare_reads_particles(const Window& w) {
    return window_needs_rebuild(w) || window_needs_solid_velocity(w);
}

int window_prepare(Window& w, cudaStream_t s, HArray<int64_t>& tot, const char* who) {
    if (window_needs_rebuild(w)) PSC_TRY(window_rebuild(w, s, tot, who));
    if (window_needs_solid_velocity(w)) PSC_TRY(window_solid_velocity(w, s));
    return PSC_OK;
}

int window_upload_solo(Window& w, cudaStream_t s) {
    if (!w.solo_dirty) return PSC_OK;
    psc_window d[2] = {w.descriptor(0), w.descriptor(1)};
    int64_t total = 0;
    // FP32/FP16/BF16 storage with an even nz: the pair kernel (two z cells per thread)
    w.solo_kernel = (w.cfg.store >= PSC_STORE_F32 && w.cfg.nz % 2 == 0) ? PSC_KERNEL_PAIR : PSC_KERNEL_AUTO;
    if (w.solo_kernel == PSC_KERNEL_PAIR) {
        PSC_TRY(psc_plan_pair_tiles(d, 1, &total));
        PSC_TRY(psc_plan_pair_tiles(d + 1, 1, &total));
    } else {
        PSC_TRY(psc_plan_tiles(d, 1, 0, &total));
        PSC_TRY(psc_plan_tiles(d + 1, 1, 0, &total));
    }
    if (total > w.partials_cap) return fail(PSC_E_CAPACITY, "window descriptor: tile partials too small");
    d[0].partials = w.partials.p;
    d[1].partials = w.partials.p;
    w.solo_tiles = total;
    for (int p = 0; p < 2; ++p) {
        PSC_CUDA(w.solo[p].ensure(1, false, s), "window descriptor");
        PSC_CUDA(cudaMemcpyAsync(w.solo[p].p, &d[p], sizeof(psc_window), cudaMemcpyHostToDevice, s), "window descriptor");
    }
    PSC_CUDA(cudaStreamSynchronize(s), "window descriptor");  // d lives on this stack frame
    w.solo_dirty = false;
    return PSC_OK;
}

int launch_solo(Window& w, unsigned flags, cudaStream_t s) {
    PSC_TRY(window_upload_solo(w, s));
    if (w.moving) flags |= PSC_STEP_MOVING;
    psc_launch c = {0, 1, w.solo_kernel, 0, 0};
    return psc_step_windows_ex(w.cfg.store, w.solo[w.cur].p, 1, w.solo_tiles, flags, &c, s);
}

double* red_pre(Window& w) { return w.out.p; }
double* red_post(Window& w) { return w.out.p + PSC_NRED; }
double* diag_dev(Window& w) { return w.out.p + 2 * PSC_NRED; }

int window_loads(Window& w, cudaStream_t s) {
    psc_geometry g = w.geometry();
    PSC_TRY(psc_particle_loads(&g, w.field_type(), w.imb_for(w.imb_par), w.chunk_partials.p,
                               red_pre(w) + PSC_RED_IMBX, w.forces.p, w.torques.p, diag_dev(w), s));
    w.loads_enqueued();
    w.loads_ready = true;
    return PSC_OK;
}

// Darcy permeability along the body force from one window's post-stream
// reductions: K = nu * (sum (1 - solid) u . d) / N / |F| with d = F / |F| and
// nu = (tau - 1/2) / 3 (run_psc_permeability_resolution.py:144-150, where
// F = (0, 0, Fz) and d = e_z); 0 without a body force.
double row_permeability(const Window& w, const double* row) {
    const double* F = w.cfg.force;
    const double fmag = std::sqrt(F[0] * F[0] + F[1] * F[1] + F[2] * F[2]);
    if (!(fmag > 0.0)) return 0.0;
    const double d0 = F[0] / fmag, d1 = F[1] / fmag, d2 = F[2] / fmag;
    const double flux = d0 * row[PSC_RED_FLUID_UX] + d1 * row[PSC_RED_FLUID_UY] + d2 * row[PSC_RED_FLUID_UZ];
    const double superficial = flux / (double)w.N;
    const double nu = (w.cfg.tau - 0.5) / 3.0;
    return nu * superficial / fmag;
}

void fill_diag(const Window& w, const double* host_out, psc_diag& d) {
    const double* pre = host_out;
    const double* post = host_out + PSC_NRED;
    const double* dg = host_out + 2 * PSC_NRED;
    const double N = (double)w.N;
    std::memset(&d, 0, sizeof(d));
    d.solid_volume_lu = post[PSC_RED_SOLID];
    d.mean_uz = post[PSC_RED_UZ] / N;
    d.momentum_residual = dg[PSC_DIAG_MOMENTUM_RESIDUAL];
    d.max_force = w.P ? dg[PSC_DIAG_MAX_FORCE] : 0.0;
    d.max_torque = w.P ? dg[PSC_DIAG_MAX_TORQUE] : 0.0;
    for (int k = 0; k < 3; ++k) {
        d.mean_u[k] = post[PSC_RED_UX + k] / N;
        d.superficial_u[k] = post[PSC_RED_FLUID_UX + k] / N;
        d.imb_sum[k] = pre[PSC_RED_IMBX + k];
        d.force_sum[k] = dg[PSC_DIAG_FORCE_SUM_X + k];
    }
    d.fluid_volume_lu = post[PSC_RED_FLUID];
    d.permeability = row_permeability(w, post);
    d.nonfinite_cells = post[PSC_RED_NONFINITE];
}

// Copy a [count] field of the window's field type to float64 host memory.
int field_to_host(const Window& w, const void* src, int64_t count, double* dst, cudaStream_t s, const char* who) {
    if (w.fdouble) {
        PSC_CUDA(cudaMemcpyAsync(dst, src, (size_t)count * 8, cudaMemcpyDeviceToHost, s), who);
        PSC_CUDA(cudaStreamSynchronize(s), who);
        return PSC_OK;
    }
    std::vector<float> tmp((size_t)count);
    PSC_CUDA(cudaMemcpyAsync(tmp.data(), src, (size_t)count * 4, cudaMemcpyDeviceToHost, s), who);
    PSC_CUDA(cudaStreamSynchronize(s), who);
    for (int64_t i = 0; i < count; ++i) dst[i] = (double)tmp[(size_t)i];
    return PSC_OK;
}

int window_get_field(Window& w, int which, double* dst, cudaStream_t s, HArray<int64_t>& tot, const char* who) {
    if (!dst) return fail(PSC_E_INVALID, std::string(who) + ": null output");
    const int64_t N = w.N;
    switch (which) {
        case PSC_FIELD_RHO:
        case PSC_FIELD_UX:
        case PSC_FIELD_UY:
        case PSC_FIELD_UZ: {
            if (!w.stepped) {  // the reference starts from rho = 1, u = 0 arrays (psc3d.py:136-139)
                std::fill(dst, dst + N, which == PSC_FIELD_RHO ? 1.0 : 0.0);
                return PSC_OK;
            }
            if (!w.moments_ready) {
                PSC_TRY(window_ensure_moments(w, s));
                PSC_TRY(launch_solo(w, PSC_STEP_MOMENTS, s));
                w.moments_ready = true;
            }
            return field_to_host(w, w.moments.p + (size_t)which * N * w.field_bytes(), N, dst, s, who);
        }
        case PSC_FIELD_SOLID:
        case PSC_FIELD_ALPHA_SUM: {
            if (!w.built) {
                std::fill(dst, dst + N, 0.0);
                return PSC_OK;
            }
            const double* src = which == PSC_FIELD_SOLID ? w.solid.p : w.alpha_sum.p;
            PSC_CUDA(cudaMemcpyAsync(dst, src, (size_t)N * 8, cudaMemcpyDeviceToHost, s), who);
            PSC_CUDA(cudaStreamSynchronize(s), who);
            return PSC_OK;
        }
        case PSC_FIELD_IMB_X:
        case PSC_FIELD_IMB_Y:
        case PSC_FIELD_IMB_Z: {
            if (!w.stepped || !w.imb.p) {
                std::fill(dst, dst + N, 0.0);
                return PSC_OK;
            }
            const int k = which - PSC_FIELD_IMB_X;
            return field_to_host(w, w.imb_for(w.imb_par) + (size_t)k * N * w.field_bytes(), N, dst, s, who);
        }
        case PSC_FIELD_US_X:
        case PSC_FIELD_US_Y:
        case PSC_FIELD_US_Z: {
            if (!w.built) PSC_TRY(window_rebuild(w, s, tot, who));
            if (w.us_version != w.pversion || !w.us.p) PSC_TRY(window_solid_velocity(w, s));
            const int k = which - PSC_FIELD_US_X;
            return field_to_host(w, w.us.p + (size_t)k * N * w.field_bytes(), N, dst, s, who);
        }
        case PSC_FIELD_F: {
            double* tmp = nullptr;
            PSC_CUDA(cudaMalloc(reinterpret_cast<void**>(&tmp), (size_t)kQ * N * 8), who);
            int st = w.cfg.open_x ? psc_stream_push_open(w.cfg.store, w.scale, w.f[w.cur].p, tmp, w.cfg.nx, w.cfg.ny,
                                                         w.cfg.nz, w.cfg.inlet_rho, w.cfg.inlet_u, s)
                                  : psc_stream_push(w.cfg.store, w.scale, w.f[w.cur].p, tmp, w.cfg.nx, w.cfg.ny,
                                                    w.cfg.nz, s);
            cudaError_t e = cudaSuccess;
            if (st == PSC_OK) e = cudaMemcpyAsync(dst, tmp, (size_t)kQ * N * 8, cudaMemcpyDeviceToHost, s);
            if (st == PSC_OK && e == cudaSuccess) e = cudaStreamSynchronize(s);
            cudaFree(tmp);
            if (st != PSC_OK) return st;
            if (e != cudaSuccess) return cuda_fail(e, who);
            return PSC_OK;
        }
        default: return fail(PSC_E_INVALID, std::string(who) + ": unknown field selector");
    }
}

int window_set_populations(Window& w, const double* hf, cudaStream_t s, const char* who) {
    if (!hf) return fail(PSC_E_INVALID, std::string(who) + ": null populations");
    const int64_t n = kQ * w.N;
    double* tmp = nullptr;
    PSC_CUDA(cudaMalloc(reinterpret_cast<void**>(&tmp), (size_t)n * 8), who);
    cudaError_t e = cudaMemcpyAsync(tmp, hf, (size_t)n * 8, cudaMemcpyHostToDevice, s);
    int st = PSC_OK;
    if (e == cudaSuccess)
        st = w.cfg.open_x ? psc_stream_pull_store_open(w.cfg.store, w.scale, tmp, w.f[w.cur].p, w.cfg.nx, w.cfg.ny,
                                                       w.cfg.nz, w.cfg.inlet_rho, w.cfg.inlet_u, s)
                          : psc_stream_pull_store(w.cfg.store, w.scale, tmp, w.f[w.cur].p, w.cfg.nx, w.cfg.ny,
                                                  w.cfg.nz, s);
    if (e == cudaSuccess && st == PSC_OK) e = cudaStreamSynchronize(s);
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail(e, who);
    if (st != PSC_OK) return st;
    w.moments_ready = false;
    w.diag_ready = false;
    return PSC_OK;
}

int window_sparse_alpha(Window& w, int64_t* offsets, int64_t* ids, double* vals, int64_t capacity, cudaStream_t s,
                        const char* who) {
    if (!offsets) return fail(PSC_E_INVALID, std::string(who) + ": null offsets");
    const int P = w.P;
    offsets[0] = 0;
    if (!w.built || P == 0) {
        for (int p = 0; p <= P; ++p) offsets[p] = 0;
        return PSC_OK;
    }
    std::vector<uint16_t> cnt((size_t)w.n_entries);
    std::vector<int64_t> off((size_t)P + 1);
    std::vector<int32_t> box((size_t)P * 6);
    if (w.n_entries)
        PSC_CUDA(cudaMemcpyAsync(cnt.data(), w.ent_cnt.p, (size_t)w.n_entries * 2, cudaMemcpyDeviceToHost, s), who);
    PSC_CUDA(cudaMemcpyAsync(off.data(), w.ent_off.p, (size_t)(P + 1) * 8, cudaMemcpyDeviceToHost, s), who);
    PSC_CUDA(cudaMemcpyAsync(box.data(), w.bbox.p, (size_t)P * 6 * 4, cudaMemcpyDeviceToHost, s), who);
    PSC_CUDA(cudaStreamSynchronize(s), who);
    int64_t total = 0;
    for (int p = 0; p < P; ++p) {
        for (int64_t e = off[p]; e < off[p + 1]; ++e) total += cnt[(size_t)e] != 0;
        offsets[p + 1] = total;
    }
    if (!ids || !vals || capacity < total) {
        if (total == 0) return PSC_OK;
        return fail(PSC_E_CAPACITY, std::string(who) + ": capacity below the entry count in offsets[P]");
    }
    const double s3 = (double)w.cfg.subsamples * w.cfg.subsamples * w.cfg.subsamples;
    const int64_t ny = w.cfg.ny, nz = w.cfg.nz;
    int64_t k = 0;
    for (int p = 0; p < P; ++p) {
        const int64_t x0 = box[(size_t)p * 6], y0 = box[(size_t)p * 6 + 1], z0 = box[(size_t)p * 6 + 2];
        const int64_t ey = box[(size_t)p * 6 + 4], ez = box[(size_t)p * 6 + 5];
        for (int64_t e = off[p]; e < off[p + 1]; ++e) {
            const uint16_t c = cnt[(size_t)e];
            if (!c) continue;
            const int64_t loc = e - off[p];
            const int64_t a = loc / (ey * ez);
            const int64_t rem = loc - a * ey * ez;
            const int64_t b = rem / ez;
            const int64_t z = rem - b * ez;
            ids[k] = ((a + x0) * ny + (b + y0)) * nz + (z + z0);
            vals[k] = (double)c / s3;  // inside / S^3 (psc3d.py:88)
            ++k;
        }
    }
    return PSC_OK;
}

}  // namespace
}  // namespace psc

using namespace psc;

// ---------------------------------------------------------------------------
// single-window solver
// ---------------------------------------------------------------------------
struct psc_solver {
    std::string last_error;  // message of the last failed call on this handle
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    Lanes lanes;  // one lane: particle loads beside the post-stream reduction pass
    Window w;
    HArray<int64_t> tot;
    HArray<double> host_out;
    // The single reporting step (psc_step(h, 1, PSC_RUN_DIAG), one drop-in
    // collide_stream_psc() call) as a CUDA graph per buffer parity, keyed by
    // every pointer, size and version its launches capture: captured on the
    // second call with an unchanged key, replayed while the key holds.
    // One graph per buffer parity and kind of call (kReportAhead: the next step is run ahead;
    // kReportCommit: this call's step was run ahead by the previous call).
    cudaGraphExec_t report_graph[2][4] = {{nullptr, nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr, nullptr}};
    std::vector<unsigned char> report_key[2][4];   // key of report_graph[parity][kind]
    std::vector<unsigned char> report_seen[2][4];  // key of the last eager run of that parity and kind
    // The step run ahead: the post-stream sums of a reporting call are the moment sums of the next
    // step's pull (the same per-cell arithmetic and tile rows in every kernel), so when the step
    // inputs are those of the previous reporting call, the call runs the next step into the other
    // buffer and IMB field instead of a reduction-only pass; the next reporting call takes it as
    // its step when its inputs are still the same.  Every other call that steps or sets the state
    // drops it (the current state is untouched by it).
    DArray<double> ahead_red;             // reductions of the step run ahead
    bool ahead_ready = false;
    std::vector<uint64_t> ahead_inputs;   // step inputs it ran with
    std::vector<uint64_t> report_inputs;  // step inputs of the last reporting call
    // device-side convergence (psc_converge): criterion state [kConvState] + reductions snapshot,
    // and two pinned status slots the host polls
    DArray<double> conv;
    HArray<double> conv_host;
    cudaEvent_t conv_ev[2] = {nullptr, nullptr};

    ~psc_solver() {
        for (auto& row : report_graph)
            for (auto& g : row)
                if (g) cudaGraphExecDestroy(g);
        for (auto& e : conv_ev)
            if (e) cudaEventDestroy(e);
    }
};

namespace psc {
namespace {

// The reductions of the post-stream state and the diagnostics of the step just
// taken, copied to the host (psc3d.py:243-253).
int solver_report(psc_solver& h, bool loads, bool fields, bool post = true) {
    Window& w = h.w;
    cudaStream_t s = h.stream;
    if (fields) PSC_TRY(window_ensure_moments(w, s));
    if (post || fields) PSC_TRY(window_upload_solo(w, s));  // (synchronises when a descriptor changed)
    if (loads) {  // the loads read the IMB field and geometry only: beside the reduction pass
        PSC_CUDA(h.lanes.begin(s), "psc_step");
        PSC_TRY(window_loads(w, h.lanes.lane(0)));
    }
    if (post || fields) {
        // the step's own partials (pre-collision state) were reduced into red_pre already
        PSC_TRY(launch_solo(w, PSC_STEP_REDUCE | (fields ? PSC_STEP_MOMENTS : 0u), s));
        PSC_TRY(psc_reduce_windows(w.solo[w.cur].p, 1, red_post(w), s));
    }
    if (loads) PSC_CUDA(h.lanes.end(s), "psc_step");
    PSC_CUDA(h.host_out.ensure(kOutLen), "psc_step");
    PSC_CUDA(cudaMemcpyAsync(h.host_out.p, w.out.p, kOutLen * sizeof(double), cudaMemcpyDeviceToHost, s), "psc_step");
    PSC_CUDA(cudaStreamSynchronize(s), "psc_step");
    if (fields) w.moments_ready = true;
    fill_diag(w, h.host_out.p, w.last);
    w.diag_ready = loads;
    return PSC_OK;
}

// ---------------------------------------------------------------------------
// lbm_converge on the device (couple_psc_liggghts.py:284-296)
// ---------------------------------------------------------------------------
// Criterion state, doubles: [0] mean_uz of the last check, [1] its step,
// [2] converged flag, [3] stopping step, [4] residual of the last check;
// [kConvState ..) the out row (red_pre, red_post) of the stopping step.
constexpr int kConvState = 8;

// One check after step `step` of the call: out holds red_pre (the reductions
// of the state before the step, i.e. the previous step's post-stream state)
// and red_post (the post-stream state of the step).  mean_uz of the previous
// step is the value this kernel kept when it checked that step (every step
// checked: the reference's sequence of values), else red_pre's.  Step 1 has
// no previous value (residual inf, as the reference's first iteration).  On
// convergence the out row is kept and the window is marked inactive in both
// descriptor tables, so the launches already enqueued after it do nothing.
__global__ void k_converge_check(const double* out, double* cs, psc_window* tab0, psc_window* tab1, int step,
                                 int min_steps, double tol, double N) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || cs[2] != 0.0) return;
    const double now = out[PSC_NRED + PSC_RED_UZ] / N;
    double resid = __longlong_as_double(0x7ff0000000000000ll);  // +inf
    if (step > 1) {
        const double prev = cs[1] == (double)(step - 1) ? cs[0] : out[PSC_RED_UZ] / N;
        const double a = fabs(now);
        resid = fabs(now - prev) / (a < 1.0e-30 ? 1.0e-30 : a);
    }
    cs[0] = now;
    cs[1] = (double)step;
    cs[4] = resid;
    if (step >= min_steps && resid < tol) {
        cs[2] = 1.0;
        cs[3] = (double)step;
        for (int k = 0; k < 2 * PSC_NRED; ++k) cs[kConvState + k] = out[k];
        tab0->flags |= PSC_WIN_INACTIVE;
        tab1->flags |= PSC_WIN_INACTIVE;
    }
}

// One collide_stream_psc step; `imb` writes the IMB field and reduces the
// step's partials into red_pre.
int solver_collide(psc_solver& h, bool imb) {
    Window& w = h.w;
    cudaStream_t s = h.stream;
    unsigned flags = PSC_STEP_COLLIDE;
    if (imb) {
        PSC_TRY(window_ensure_imb(w, s));
        flags |= PSC_STEP_IMB | PSC_STEP_REDUCE;
    }
    PSC_TRY(launch_solo(w, flags, s));
    w.cur ^= 1;
    if (imb) w.imb_par = w.cur;
    w.stepped = true;
    w.moments_ready = false;
    w.loads_ready = false;
    w.diag_ready = false;
    if (imb) PSC_TRY(psc_reduce_windows(w.solo[w.cur].p, 1, red_pre(w), s));
    return PSC_OK;
}

constexpr int kReportAhead = 1;   // the call runs the next step ahead (instead of a reduction pass)
constexpr int kReportCommit = 2;  // the call's step was run ahead by the previous reporting call

// Everything the launches of one reporting step from buffer parity `par`
// capture: a graph recorded under one key replays correctly under the same key.
std::vector<unsigned char> report_key(const psc_solver& h, int par, int kind) {
    const Window& w = h.w;
    struct Key {
        psc_geometry g;
        const void* desc[2];
        const void* imb[2];
        const void* out;
        const void* ahead;
        const void* host;
        const void* chunks;
        const void* forces;
        const void* torques;
        uint64_t desc_version;
        int64_t tiles;
        int32_t kernel, store, moving, par, field_type, kind;
    } k;
    std::memset(&k, 0, sizeof(k));  // padding too: keys compare bytewise
    k.g = w.geometry();
    k.desc[0] = w.solo[0].p;
    k.desc[1] = w.solo[1].p;
    k.imb[0] = w.imb_for(0);
    k.imb[1] = w.imb_for(1);
    k.out = w.out.p;
    k.ahead = h.ahead_red.p;
    k.host = h.host_out.p;
    k.chunks = w.chunk_partials.p;
    k.forces = w.forces.p;
    k.torques = w.torques.p;
    k.desc_version = w.desc_version;
    k.tiles = w.solo_tiles;
    k.kernel = w.solo_kernel;
    k.store = w.cfg.store;
    k.moving = w.moving ? 1 : 0;
    k.par = par;
    k.field_type = w.field_type();
    k.kind = kind;
    const unsigned char* b = reinterpret_cast<const unsigned char*>(&k);
    return std::vector<unsigned char>(b, b + sizeof(k));
}

// Everything a step reads besides the populations.
std::vector<uint64_t> solver_step_inputs(const psc_solver& h) {
    const Window& w = h.w;
    return {w.built_version, w.moving ? w.us_version : 0, w.desc_version, (uint64_t)(w.moving ? 1 : 0),
            (uint64_t)w.solo_kernel, (uint64_t)w.solo_tiles};
}

// The GPU work of one reporting step from buffer parity `par` (the launches of
// solver_collide(imb) + solver_report(loads, post) without their host-side
// bookkeeping), ending with the read-back into host_out.  kReportCommit: the
// step from `par` is in place already (buffer par ^ 1, its IMB field and its
// reductions in ahead_red).  kReportAhead: the post-stream sums come from the
// next step, run from par ^ 1 into buffer par and IMB field par.
int report_step_work(psc_solver& h, int par, int kind) {
    Window& w = h.w;
    cudaStream_t s = h.stream;
    const unsigned mv = w.moving ? PSC_STEP_MOVING : 0u;
    const psc_launch c = {0, 1, w.solo_kernel, 0, 0};
    const unsigned full = PSC_STEP_COLLIDE | PSC_STEP_IMB | PSC_STEP_REDUCE | mv;
    if (kind & kReportCommit) {
        PSC_CUDA(cudaMemcpyAsync(red_pre(w), h.ahead_red.p, PSC_NRED * sizeof(double), cudaMemcpyDeviceToDevice, s),
                 "psc_step");
    } else {
        PSC_TRY(psc_step_windows_ex(w.cfg.store, w.solo[par].p, 1, w.solo_tiles, full, &c, s));
        PSC_TRY(psc_reduce_windows(w.solo[par ^ 1].p, 1, red_pre(w), s));
    }
    PSC_CUDA(h.lanes.begin(s), "psc_step");  // the loads on a lane; the main stream's kernel first
    if (kind & kReportAhead) {
        PSC_TRY(psc_step_windows_ex(w.cfg.store, w.solo[par ^ 1].p, 1, w.solo_tiles, full, &c, s));
        PSC_TRY(psc_reduce_windows(w.solo[par].p, 1, h.ahead_red.p, s));
        PSC_CUDA(cudaMemcpyAsync(red_post(w), h.ahead_red.p, PSC_NRED * sizeof(double), cudaMemcpyDeviceToDevice, s),
                 "psc_step");
    } else {
        PSC_TRY(psc_step_windows_ex(w.cfg.store, w.solo[par ^ 1].p, 1, w.solo_tiles, PSC_STEP_REDUCE | mv, &c, s));
        PSC_TRY(psc_reduce_windows(w.solo[par ^ 1].p, 1, red_post(w), s));
    }
    psc_geometry g = w.geometry();
    PSC_TRY(psc_particle_loads(&g, w.field_type(), w.imb_for(par ^ 1), w.chunk_partials.p, red_pre(w) + PSC_RED_IMBX,
                               w.forces.p, w.torques.p, diag_dev(w), h.lanes.lane(0)));
    w.loads_enqueued();
    PSC_CUDA(h.lanes.end(s), "psc_step");
    PSC_CUDA(cudaMemcpyAsync(h.host_out.p, w.out.p, kOutLen * sizeof(double), cudaMemcpyDeviceToHost, s), "psc_step");
    return PSC_OK;
}

// One collide_stream_psc() step with its loads and diagnostics (the work of
// solver_collide(imb) + solver_report(loads)), replayed from a CUDA graph
// when nothing it captures has changed since the previous call of its kind.
int solver_report_step(psc_solver& h) {
    Window& w = h.w;
    cudaStream_t s = h.stream;
    // everything that may allocate, upload or synchronise happens here, outside any capture
    PSC_TRY(window_ensure_imb(w, s));
    PSC_TRY(window_upload_solo(w, s));
    PSC_CUDA(h.host_out.ensure(kOutLen), "psc_step");
    PSC_CUDA(h.ahead_red.ensure(PSC_NRED, true, s), "psc_step");
    const std::vector<uint64_t> inputs = solver_step_inputs(h);
    int kind = 0;
    if (h.ahead_ready && inputs == h.ahead_inputs) kind |= kReportCommit;
    if (inputs == h.report_inputs) kind |= kReportAhead;
    h.ahead_ready = false;
    const int par = w.cur;
    std::vector<unsigned char> key = report_key(h, par, kind);
    cudaGraphExec_t& graph = h.report_graph[par][kind];
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    PSC_CUDA(cudaStreamIsCapturing(s, &cap), "psc_step");
    if (cap != cudaStreamCaptureStatusNone) {
        kind = 0;  // the caller records this step into its own graph: no step run ahead
        PSC_TRY(report_step_work(h, par, kind));
    } else if (graph && key == h.report_key[par][kind]) {
        PSC_CUDA(cudaGraphLaunch(graph, s), "psc_step");
    } else if (key == h.report_seen[par][kind]) {
        // the same launches as the previous call of this parity and kind: record them once, then replay
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
            h.report_key[par][kind].clear();
        }
        PSC_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "psc_step");
        const int st = report_step_work(h, par, kind);
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(s, &g);
        if (st != PSC_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (ec != cudaSuccess) return cuda_fail(ec, "psc_step: capturing the reporting step");
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) return cuda_fail(ei, "psc_step: instantiating the reporting step");
        graph = exec;
        h.report_key[par][kind] = key;
        PSC_CUDA(cudaGraphLaunch(exec, s), "psc_step");
    } else {
        PSC_TRY(report_step_work(h, par, kind));
        h.report_seen[par][kind] = std::move(key);
    }
    w.cur ^= 1;
    w.imb_par = w.cur;
    w.stepped = true;
    w.moments_ready = false;
    w.loads_ready = true;
    PSC_CUDA(cudaStreamSynchronize(s), "psc_step");
    if (kind & kReportAhead) {  // the step run ahead added its own IMB; a reduction pass adds none
        for (int q = PSC_RED_IMBX; q <= PSC_RED_IMBZ; ++q) h.host_out.p[PSC_NRED + q] = 0.0;
        h.ahead_ready = true;
        h.ahead_inputs = inputs;
    }
    h.report_inputs = inputs;
    fill_diag(w, h.host_out.p, w.last);
    w.diag_ready = true;
    return PSC_OK;
}

// lbm_converge as one call (psc_converge, PSC_RUN_CONVERGE): steps are
// enqueued in blocks with the criterion evaluated on the device at every
// check step (a multiple of check_every, and the last step); the host reads
// the criterion state once per block, one block behind, and stops enqueuing
// once it reports convergence.  Steps enqueued after the stopping step find
// the window inactive and do nothing, so the populations stay those of the
// stopping step: buffer parity start ^ (steps & 1).
int solver_converge(psc_solver& h, int nsteps, double tol, int min_steps, int check_every, bool fields,
                    psc_status& st) {
    Window& w = h.w;
    cudaStream_t s = h.stream;
    const char* who = "psc_converge";
    PSC_TRY(window_ensure_imb(w, s));
    PSC_TRY(window_upload_solo(w, s));
    // from here on the device may mark the window inactive in its descriptor tables: whatever
    // path leaves this function, the next launch uploads them afresh
    w.solo_dirty = true;
    PSC_CUDA(h.conv.ensure(kConvState + 2 * PSC_NRED, false, s), who);
    PSC_CUDA(h.conv_host.ensure(2 * kConvState), who);
    for (auto& e : h.conv_ev)
        if (!e) PSC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), who);
    PSC_CUDA(cudaMemsetAsync(h.conv.p, 0, kConvState * sizeof(double), s), who);
    const unsigned mv = w.moving ? PSC_STEP_MOVING : 0u;
    const psc_launch c = {0, 1, w.solo_kernel, 0, 0};
    const int start = w.cur;
    // steps per poll: ~3e7 lattice updates (about a millisecond of the step kernel), 4 .. 256 steps
    const int64_t per = std::max<int64_t>(4, std::min<int64_t>(256, 30000000 / std::max<int64_t>(w.N, 1)));
    const int block = (int)std::max<int64_t>(check_every, per);
    int t = 0, polls = 0, pending = -1;
    bool stop = false;
    while (t < nsteps && !stop) {
        const int end = (int)std::min<int64_t>(nsteps, (int64_t)t + block);
        for (int u = t + 1; u <= end; ++u) {
            const int par = start ^ ((u - 1) & 1);
            if (u % check_every != 0 && u != nsteps) {
                PSC_TRY(psc_step_windows_ex(w.cfg.store, w.solo[par].p, 1, w.solo_tiles, PSC_STEP_COLLIDE | mv, &c, s));
                continue;
            }
            PSC_TRY(psc_step_windows_ex(w.cfg.store, w.solo[par].p, 1, w.solo_tiles,
                                        PSC_STEP_COLLIDE | PSC_STEP_IMB | PSC_STEP_REDUCE | mv, &c, s));
            PSC_TRY(psc_reduce_windows(w.solo[par ^ 1].p, 1, red_pre(w), s));
            PSC_TRY(psc_step_windows_ex(w.cfg.store, w.solo[par ^ 1].p, 1, w.solo_tiles, PSC_STEP_REDUCE | mv, &c, s));
            PSC_TRY(psc_reduce_windows(w.solo[par ^ 1].p, 1, red_post(w), s));
            k_converge_check<<<1, 32, 0, s>>>(w.out.p, h.conv.p, w.solo[0].p, w.solo[1].p, u, min_steps, tol,
                                              (double)w.N);
            PSC_CUDA(cudaGetLastError(), who);
        }
        t = end;
        const int slot = polls & 1;
        PSC_CUDA(cudaMemcpyAsync(h.conv_host.p + slot * kConvState, h.conv.p, kConvState * sizeof(double),
                                 cudaMemcpyDeviceToHost, s),
                 who);
        PSC_CUDA(cudaEventRecord(h.conv_ev[slot], s), who);
        if (pending >= 0) {
            PSC_CUDA(cudaEventSynchronize(h.conv_ev[pending]), who);
            stop = h.conv_host.p[pending * kConvState + 2] != 0.0;
        }
        pending = slot;
        ++polls;
    }
    PSC_CUDA(cudaStreamSynchronize(s), who);
    const double* cs = h.conv_host.p + pending * kConvState;  // covers every enqueued step
    const bool converged = cs[2] != 0.0;
    const int done = converged ? (int)cs[3] : nsteps;
    st.converged = converged ? 1 : 0;
    st.steps_done = done;
    st.residual = cs[4];
    w.cur = start ^ (done & 1);
    w.imb_par = w.cur;  // the last step that ran wrote its IMB field (a check step)
    w.stepped = true;
    w.moments_ready = false;
    w.loads_ready = false;
    w.diag_ready = false;
    if (converged)  // the reductions of the stopping step (later enqueued reductions read no new partials)
        PSC_CUDA(cudaMemcpyAsync(w.out.p, h.conv.p + kConvState, 2 * PSC_NRED * sizeof(double),
                                 cudaMemcpyDeviceToDevice, s),
                 who);
    PSC_TRY(window_upload_solo(w, s));  // the descriptor tables without the inactive flag
    // loads and diagnostics of the stopping step (its IMB field; the post-stream reductions are
    // taken already unless the fields are wanted)
    PSC_TRY(solver_report(h, true, fields, fields));
    st.diag = w.last;
    return PSC_OK;
}

}  // namespace
}  // namespace psc

extern "C" {

int psc_create(const psc_config* h_cfg, psc_solver** out) {
    if (!h_cfg || !out) return fail(PSC_E_INVALID, "psc_create: null argument");
    *out = nullptr;
    PSC_TRY(check_config(*h_cfg, "psc_create"));
    DeviceScope ds(h_cfg->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "psc_create: cudaSetDevice");
    std::unique_ptr<psc_solver> h(new (std::nothrow) psc_solver());
    if (!h) return fail(PSC_E_CAPACITY, "psc_create: out of host memory");
    h->device = h_cfg->device;
    if (h_cfg->stream) {
        h->stream = as_stream(h_cfg->stream);
    } else {
        PSC_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "psc_create");
        h->own_stream = true;
    }
    h->w.imb_dual = true;  // a reporting call may run the next step ahead (solver_report_step)
    int st = window_init(h->w, *h_cfg, h->stream, "psc_create");
    if (st == PSC_OK) {
        cudaError_t e = h->lanes.init(1);
        if (e != cudaSuccess) st = cuda_fail(e, "psc_create");
    }
    if (st == PSC_OK) st = window_set_particles(h->w, nullptr, 0, h->stream, "psc_create");
    if (st == PSC_OK) {
        cudaError_t e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) st = cuda_fail(e, "psc_create");
    }
    if (st != PSC_OK) {
        psc_destroy(h.release());
        return st;
    }
    *out = h.release();
    return PSC_OK;
}

int psc_destroy(psc_solver* h) {
    if (!h) return PSC_OK;
    {
        DeviceScope ds(h->device);
        cudaStreamSynchronize(h->stream);
        cudaStream_t s = h->stream;
        bool own = h->own_stream;
        delete h;  // frees the device buffers on the handle's device
        if (own) cudaStreamDestroy(s);
    }
    return PSC_OK;
}

int psc_set_particles(psc_solver* h, const double* h_particles, int nparticles) {
    if (!h) return fail(PSC_E_INVALID, "psc_set_particles: null handle");
    ErrorCapture errors_(h->last_error);
    DeviceScope ds(h->device);
    return window_set_particles(h->w, h_particles, nparticles, h->stream, "psc_set_particles");
}

int psc_rebuild_geometry(psc_solver* h) {
    if (!h) return fail(PSC_E_INVALID, "psc_rebuild_geometry: null handle");
    ErrorCapture errors_(h->last_error);
    DeviceScope ds(h->device);
    return window_rebuild(h->w, h->stream, h->tot, "psc_rebuild_geometry");
}

int psc_step(psc_solver* h, int nsteps, unsigned flags, psc_status* h_status) {
    if (!h) return fail(PSC_E_INVALID, "psc_step: null handle");
    ErrorCapture errors_(h->last_error);
    if (nsteps < 0) return fail(PSC_E_INVALID, "psc_step: negative step count");
    if (flags & ~(PSC_RUN_DIAG | PSC_RUN_CONVERGE | PSC_RUN_FIELDS)) return fail(PSC_E_INVALID, "psc_step: unknown flags");
    DeviceScope ds(h->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "psc_step: cudaSetDevice");
    Window& w = h->w;
    const bool converge = (flags & PSC_RUN_CONVERGE) != 0;
    const bool diag = converge || (flags & PSC_RUN_DIAG) != 0;
    const bool fields = (flags & PSC_RUN_FIELDS) != 0;
    const double tol = w.cfg.conv_tol > 0.0 ? w.cfg.conv_tol : 1.0e-8;
    const int min_steps = std::max(1, w.cfg.conv_min_steps);
    psc_status st{};
    st.residual = INFINITY;
    if (nsteps > 0) PSC_TRY(window_prepare(w, h->stream, h->tot, "psc_step"));
    if (nsteps == 1 && diag && !converge && !fields) {  // one collide_stream_psc() call
        PSC_TRY(solver_report_step(*h));
        st.steps_done = 1;
        st.diag = w.last;
        if (h_status) *h_status = st;
        return PSC_OK;
    }
    if (nsteps > 0) h->ahead_ready = false;  // these steps overwrite the other buffer
    if (converge && nsteps > 0) {
        PSC_TRY(solver_converge(*h, nsteps, tol, min_steps, std::max(1, w.cfg.conv_check_every), fields, st));
        if (h_status) *h_status = st;
        return PSC_OK;
    }
    for (int k = 1; k <= nsteps; ++k) PSC_TRY(solver_collide(*h, k == nsteps));
    st.steps_done = nsteps;
    if (nsteps > 0 && (diag || fields)) {
        PSC_TRY(solver_report(*h, diag, fields));
        if (diag) st.diag = w.last;
    } else if (nsteps > 0) {
        PSC_CUDA(cudaGetLastError(), "psc_step");
    }
    if (h_status) *h_status = st;
    return PSC_OK;
}

int psc_converge(psc_solver* h, int max_steps, double tol, int min_steps, int check_every, unsigned flags,
                 psc_status* h_status) {
    if (!h) return fail(PSC_E_INVALID, "psc_converge: null handle");
    ErrorCapture errors_(h->last_error);
    if (max_steps < 1 || check_every < 1 || !(tol >= 0.0) || !std::isfinite(tol))
        return fail(PSC_E_INVALID, "psc_converge: need max_steps >= 1, check_every >= 1 and a finite tol >= 0");
    if (flags & ~PSC_RUN_FIELDS) return fail(PSC_E_INVALID, "psc_converge: unknown flags");
    DeviceScope ds(h->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "psc_converge: cudaSetDevice");
    psc_status st{};
    st.residual = INFINITY;
    h->ahead_ready = false;
    PSC_TRY(window_prepare(h->w, h->stream, h->tot, "psc_converge"));
    PSC_TRY(solver_converge(*h, max_steps, tol, std::max(1, min_steps), check_every, (flags & PSC_RUN_FIELDS) != 0,
                            st));
    if (h_status) *h_status = st;
    return PSC_OK;
}

int psc_get_fields(psc_solver* h, int which, double* h_dst) {
    if (!h) return fail(PSC_E_INVALID, "psc_get_fields: null handle");
    ErrorCapture errors_(h->last_error);
    DeviceScope ds(h->device);
    return window_get_field(h->w, which, h_dst, h->stream, h->tot, "psc_get_fields");
}

int psc_set_populations(psc_solver* h, const double* h_f) {
    if (!h) return fail(PSC_E_INVALID, "psc_set_populations: null handle");
    ErrorCapture errors_(h->last_error);
    DeviceScope ds(h->device);
    h->ahead_ready = false;  // the state changes
    return window_set_populations(h->w, h_f, h->stream, "psc_set_populations");
}

int psc_get_loads(psc_solver* h, double* h_forces, double* h_torques) {
    if (!h) return fail(PSC_E_INVALID, "psc_get_loads: null handle");
    ErrorCapture errors_(h->last_error);
    Window& w = h->w;
    if (w.P > 0 && (!h_forces || !h_torques)) return fail(PSC_E_INVALID, "psc_get_loads: null output");
    if (w.P == 0) return PSC_OK;
    DeviceScope ds(h->device);
    if (!w.stepped) {  // hydro_forces / hydro_torques start as zeros (psc3d.py:146-147)
        std::fill(h_forces, h_forces + 3 * (size_t)w.P, 0.0);
        std::fill(h_torques, h_torques + 3 * (size_t)w.P, 0.0);
        return PSC_OK;
    }
    if (!w.loads_ready) {  // accumulate_particle_loads() with the current geometry (psc3d.py:255-281)
        if (!w.imb.p) return fail(PSC_E_INVALID, "psc_get_loads: no IMB field (no step has run)");
        PSC_TRY(window_loads(w, h->stream));
    }
    PSC_CUDA(cudaMemcpyAsync(h_forces, w.forces.p, (size_t)w.P * 24, cudaMemcpyDeviceToHost, h->stream),
             "psc_get_loads");
    PSC_CUDA(cudaMemcpyAsync(h_torques, w.torques.p, (size_t)w.P * 24, cudaMemcpyDeviceToHost, h->stream),
             "psc_get_loads");
    PSC_CUDA(cudaStreamSynchronize(h->stream), "psc_get_loads");
    return PSC_OK;
}

int psc_accumulate_particle_loads(psc_solver* h) {
    if (!h) return fail(PSC_E_INVALID, "psc_accumulate_particle_loads: null handle");
    ErrorCapture errors_(h->last_error);
    Window& w = h->w;
    if (!w.stepped || !w.imb.p) return fail(PSC_E_INVALID, "psc_accumulate_particle_loads: no step has run");
    DeviceScope ds(h->device);
    if (!w.built) PSC_TRY(window_rebuild(w, h->stream, h->tot, "psc_accumulate_particle_loads"));
    PSC_TRY(solver_report(*h, true, false));
    w.diag_ready = true;
    return PSC_OK;
}

int psc_get_diag(psc_solver* h, psc_diag* h_diag) {
    if (!h || !h_diag) return fail(PSC_E_INVALID, "psc_get_diag: null argument");
    Window& w = h->w;
    if (!w.stepped) {
        std::memset(h_diag, 0, sizeof(psc_diag));
        return PSC_OK;
    }
    DeviceScope ds(h->device);
    if (!w.diag_ready) {
        if (!w.imb.p) return fail(PSC_E_INVALID, "psc_get_diag: no IMB field (no step has run)");
        PSC_TRY(solver_report(*h, true, false));
    }
    *h_diag = w.last;
    return PSC_OK;
}

int psc_get_sparse_alpha(psc_solver* h, int64_t* h_offsets, int64_t* h_ids, double* h_vals, int64_t capacity) {
    if (!h) return fail(PSC_E_INVALID, "psc_get_sparse_alpha: null handle");
    ErrorCapture errors_(h->last_error);
    DeviceScope ds(h->device);
    return window_sparse_alpha(h->w, h_offsets, h_ids, h_vals, capacity, h->stream, "psc_get_sparse_alpha");
}

const char* psc_solver_last_error(const psc_solver* h) { return h ? h->last_error.c_str() : ""; }

size_t psc_config_size(void) { return sizeof(psc_config); }

size_t psc_diag_size(void) { return sizeof(psc_diag); }

size_t psc_status_size(void) { return sizeof(psc_status); }

int psc_solver_info(psc_solver* h, int* h_nparticles, int64_t* h_cells) {
    if (!h) return fail(PSC_E_INVALID, "psc_solver_info: null handle");
    if (h_nparticles) *h_nparticles = h->w.P;
    if (h_cells) *h_cells = h->w.N;
    return PSC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// batches
// ---------------------------------------------------------------------------
struct psc_batch {
    std::string last_error;  // message of the last failed call on this handle
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int store = PSC_STORE_F32;
    psc_launch launch{0, 1, PSC_KERNEL_AUTO, 0, 0};
    int graph_steps = 0;
    std::vector<std::unique_ptr<Window>> w;
    DArray<psc_window> table[2];
    int64_t total_tiles = 0;
    bool tables_dirty = true;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int parity = 0;
    std::vector<int> frozen;  // -1 active, else the buffer parity holding the frozen state
    std::vector<double> frozen_red;  // [nwin][NRED] post-stream reductions at freezing
    DArray<double> red_pre, red_post, diag;
    // Step run ahead.  A reporting step needs the post-stream sums of its state, i.e. the
    // moment sums that the next step's pull computes (the same per-cell arithmetic in the pair
    // kernel, the same tile order: the same bits).  When the step inputs did not change since
    // the previous reporting call, the reporting call runs that next step (into the other buffer
    // and IMB field; the current state stays as it is) instead of a reduction-only pass, and the
    // next call takes it as its first step when its inputs are still the same.
    DArray<double> red_next;            // reductions of the step run ahead
    bool ahead_ready = false;           // a step run ahead is waiting in the other buffer
    std::vector<uint64_t> ahead_inputs;  // the step inputs it ran with
    std::vector<uint64_t> report_inputs;  // the step inputs of the last reporting call
    uint64_t tables_version = 0;
    HArray<double> host;
    HArray<int64_t> tot;
    std::vector<psc_diag> last;
    std::vector<char> have_diag;
    std::vector<uint64_t> built_desc;  // descriptor versions the tables were built from
    bool moving_any = false;
    Lanes lanes;  // particle loads of the windows beside the post-stream reduction pass
    HArray<double> up_host;    // every window's particles, staged for one upload
    DArray<double> up_dev;
    // The upload runs on its own stream beside the step kernels, which do not
    // read particles: up_ready (on the main stream) orders it after every
    // earlier reader of up_dev, up_done ends it.  Until the main stream has
    // waited for up_done (up_pending), whatever reads particles waits first.
    cudaStream_t up_stream = nullptr;
    cudaEvent_t up_ready = nullptr;
    cudaEvent_t up_done = nullptr;
    bool up_pending = false;
    std::vector<int64_t> staged;  // per window: offset of its accepted state in up_host, or -1
    // particle loads of all active windows in one launch sequence: job table
    // [LoadsJob x n][chunk bases n+1][particle bases n+1], as last uploaded
    // one table per buffer parity (a job names the IMB field of its window's current buffer)
    std::vector<unsigned char> jobs_last[2];
    HArray<unsigned char> jobs_host[2];
    DArray<unsigned char> jobs_dev[2];
    int jobs_par = 0;  // the table of the last batch_loads_table
    DArray<double> loads_part;  // chunk partials of all jobs
    int jobs_n = 0, jobs_max_s = 1;
    int64_t jobs_chunks = 0, jobs_particles = 0;
    bool jobs_list_ready = false;  // every job's loads list is current
    bool jobs_all_lists = false;   // every job has loads-list arrays (the list path of the loads)

    ~psc_batch() {
        for (auto& g : graph)
            if (g) cudaGraphExecDestroy(g);
        if (up_done) cudaEventDestroy(up_done);
        if (up_ready) cudaEventDestroy(up_ready);
        if (up_stream) cudaStreamDestroy(up_stream);
    }
};

namespace psc {
namespace {

// Job table of the particle loads of every active window (one
// launch_particle_loads_multi per reporting step).  Built on the host each
// time and uploaded only when it changed (new geometry, buffers, frozen set).
int batch_loads_table(psc_batch& b, const char* who) {
    const int nwin = (int)b.w.size();
    std::vector<LoadsJob> jobs;
    std::vector<int64_t> cb(1, 0), pb(1, 0);
    int max_s = 1;
    bool ready = true, lists = true;
    for (int k = 0; k < nwin; ++k) {
        if (b.frozen[(size_t)k] >= 0) continue;
        const Window& w = *b.w[(size_t)k];
        LoadsJob j;
        std::memset(&j, 0, sizeof(j));  // padding too: the table is compared bytewise
        j.g = w.geometry();
        ready = ready && (w.P == 0 || j.g.list_ready);
        lists = lists && (w.P == 0 || (j.g.load_w && j.g.load_abk && j.g.load_n));
        j.imb = w.imb_for(w.cur);
        j.imb_sums = b.red_pre.p + (size_t)k * PSC_NRED + PSC_RED_IMBX;
        j.forces = w.forces.p;
        j.torques = w.torques.p;
        j.diag = b.diag.p + (size_t)k * PSC_NDIAG;
        jobs.push_back(j);
        cb.push_back(cb.back() + (w.P > 0 ? w.n_chunks : 0));
        pb.push_back(pb.back() + w.P);
        max_s = std::max(max_s, w.cfg.subsamples);
    }
    const size_t n = jobs.size();
    const size_t jb = n * sizeof(LoadsJob), bb = (n + 1) * sizeof(int64_t);
    std::vector<unsigned char> bytes(jb + 2 * bb);
    if (jb) std::memcpy(bytes.data(), jobs.data(), jb);
    std::memcpy(bytes.data() + jb, cb.data(), bb);
    std::memcpy(bytes.data() + jb + bb, pb.data(), bb);
    b.jobs_n = (int)n;
    b.jobs_max_s = max_s;
    b.jobs_chunks = cb.back();
    b.jobs_particles = pb.back();
    b.jobs_list_ready = ready;
    b.jobs_all_lists = lists;
    const int t = b.parity;
    b.jobs_par = t;
    if (bytes == b.jobs_last[t]) return PSC_OK;
    // No wait is needed before the rewrite: only reporting calls use the table, its pinned copy and
    // the partials, and every reporting call ends with a stream synchronisation, so nothing of an
    // earlier call still reads them (a buffer that grows is freed by cudaFree, which waits anyway).
    PSC_CUDA(b.loads_part.ensure(std::max<int64_t>(b.jobs_chunks, 1) * 6, false, b.stream), who);
    PSC_CUDA(b.jobs_dev[t].ensure((int64_t)bytes.size(), false, b.stream), who);
    PSC_CUDA(b.jobs_host[t].ensure((int64_t)bytes.size()), who);
    std::memcpy(b.jobs_host[t].p, bytes.data(), bytes.size());
    PSC_CUDA(cudaMemcpyAsync(b.jobs_dev[t].p, b.jobs_host[t].p, bytes.size(), cudaMemcpyHostToDevice, b.stream),
             who);
    b.jobs_last[t].swap(bytes);
    return PSC_OK;
}

const LoadsJob* batch_jobs(const psc_batch& b) { return reinterpret_cast<const LoadsJob*>(b.jobs_dev[b.jobs_par].p); }

const int64_t* batch_chunk_base(const psc_batch& b) {
    return reinterpret_cast<const int64_t*>(b.jobs_dev[b.jobs_par].p + (size_t)b.jobs_n * sizeof(LoadsJob));
}

const int64_t* batch_particle_base(const psc_batch& b) {
    return batch_chunk_base(b) + b.jobs_n + 1;
}

void batch_drop_graphs(psc_batch& b) {
    for (auto& g : b.graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

int batch_build_tables(psc_batch& b) {
    const int nwin = (int)b.w.size();
    std::vector<psc_window> tab[2];
    b.moving_any = false;
    for (int p = 0; p < 2; ++p) {
        tab[p].resize((size_t)nwin);
        for (int k = 0; k < nwin; ++k) {
            Window& w = *b.w[(size_t)k];
            tab[p][(size_t)k] = w.descriptor(p);
            if (b.frozen[(size_t)k] >= 0) tab[p][(size_t)k].flags |= PSC_WIN_INACTIVE;
            b.moving_any = b.moving_any || w.moving;
        }
        int64_t total = 0;
        if (b.launch.kernel == PSC_KERNEL_TMA) {
            int32_t sb = 0;
            PSC_TRY(psc_plan_row_tiles(tab[p].data(), nwin, 0, store_elem_bytes(b.store), &total, &sb));
            b.launch.stage_bytes = sb;
        } else if (b.launch.kernel == PSC_KERNEL_PAIR) {
            PSC_TRY(psc_plan_pair_tiles(tab[p].data(), nwin, &total));
        } else {
            PSC_TRY(psc_plan_tiles(tab[p].data(), nwin, 256 * b.launch.cells_per_thread, &total));
        }
        b.total_tiles = total;
        for (int k = 0; k < nwin; ++k) {
            Window& w = *b.w[(size_t)k];
            if (tab[p][(size_t)k].tile_count > w.partials_cap)
                return fail(PSC_E_CAPACITY, "batch tables: tile partials too small");
            tab[p][(size_t)k].partials = w.partials.p;
        }
    }
    for (int p = 0; p < 2; ++p) {
        PSC_CUDA(b.table[p].ensure(nwin, false, b.stream), "batch tables");
        PSC_CUDA(cudaMemcpyAsync(b.table[p].p, tab[p].data(), (size_t)nwin * sizeof(psc_window),
                                 cudaMemcpyHostToDevice, b.stream),
                 "batch tables");
    }
    PSC_CUDA(cudaStreamSynchronize(b.stream), "batch tables");
    for (int k = 0; k < nwin; ++k) b.built_desc[(size_t)k] = b.w[(size_t)k]->desc_version;
    b.tables_dirty = false;
    ++b.tables_version;
    batch_drop_graphs(b);
    return PSC_OK;
}

void batch_sync_cur(psc_batch& b) {
    for (size_t k = 0; k < b.w.size(); ++k) b.w[k]->cur = b.frozen[k] >= 0 ? b.frozen[k] : b.parity;
}

// Everything a step reads besides the populations: each window's geometry,
// solid velocity, descriptor and frozen state, and the launch tables.
std::vector<uint64_t> batch_step_inputs(const psc_batch& b) {
    std::vector<uint64_t> v;
    v.reserve(b.w.size() * 5 + 1);
    v.push_back(b.tables_version);
    for (size_t k = 0; k < b.w.size(); ++k) {
        const Window& w = *b.w[k];
        v.push_back(w.built_version);
        v.push_back(w.moving ? w.us_version : 0);
        v.push_back(w.desc_version);
        v.push_back((uint64_t)(int64_t)b.frozen[k]);
        v.push_back(w.moving ? 1 : 0);
    }
    return v;
}

// A reporting step may run the next step ahead (instead of the reduction-only
// pass) in the pair kernel, without field output, and when its inputs are
// those of the previous reporting call (a static geometry; moved particles
// rebuild it, so such calls keep the reduction pass).
bool batch_may_run_ahead(const psc_batch& b, bool fields, const std::vector<uint64_t>& inputs) {
    return b.launch.kernel == PSC_KERNEL_PAIR && !fields && inputs == b.report_inputs;
}

int batch_launch(psc_batch& b, unsigned flags) {
    if (b.moving_any) flags |= PSC_STEP_MOVING;
    return psc_step_windows_ex(b.store, b.table[b.parity].p, (int)b.w.size(), b.total_tiles, flags, &b.launch,
                               b.stream);
}

// The main stream waits for a pending particle upload (psc_batch_set_particles_all):
// everything queued on it afterwards, lanes forked from it included, sees the new state.
int batch_upload_join(psc_batch& b, const char* who) {
    if (!b.up_pending) return PSC_OK;
    PSC_CUDA(cudaStreamWaitEvent(b.stream, b.up_done, 0), who);
    b.up_pending = false;
    return PSC_OK;
}

// Everything the next step reads is on the device and described by the tables.
int batch_prepare(psc_batch& b, bool imb, bool moments) {
    // geometry rebuilds: every window's plan, one synchronisation for all their counts, the builds
    const char* who = "psc_batch_step";
    std::vector<size_t> plan;
    for (size_t k = 0; k < b.w.size(); ++k)
        if (window_needs_rebuild(*b.w[k])) plan.push_back(k);
    if (!plan.empty()) {
        PSC_TRY(batch_upload_join(b, who));
        PSC_CUDA(b.tot.ensure(4 * (int64_t)b.w.size()), who);
        for (size_t k : plan) PSC_TRY(window_rebuild_plan(*b.w[k], b.stream, b.tot.p + 4 * k, who));
        PSC_CUDA(cudaStreamSynchronize(b.stream), who);
        for (size_t k : plan) PSC_TRY(window_rebuild_finish(*b.w[k], b.stream, b.tot.p + 4 * k, who));
    }
    for (size_t k = 0; k < b.w.size(); ++k) {
        Window& w = *b.w[k];
        if (window_prepare_reads_particles(w)) PSC_TRY(batch_upload_join(b, "psc_batch_step"));
        PSC_TRY(window_prepare(w, b.stream, b.tot, "psc_batch_step"));
        if (imb) PSC_TRY(window_ensure_imb(w, b.stream));
        if (moments) PSC_TRY(window_ensure_moments(w, b.stream));
        if (w.desc_version != b.built_desc[k]) b.tables_dirty = true;
    }
    if (b.tables_dirty) PSC_TRY(batch_build_tables(b));
    return PSC_OK;
}

int batch_capture(psc_batch& b, int parity) {
    const int saved = b.parity;
    b.parity = parity;
    PSC_CUDA(cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal), "graph capture");
    int st = PSC_OK;
    for (int i = 0; i < b.graph_steps && st == PSC_OK; ++i) {
        st = batch_launch(b, PSC_STEP_COLLIDE);
        b.parity ^= 1;
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b.stream, &g);
    b.parity = saved;
    if (st != PSC_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return cuda_fail(e, "graph capture");
    e = cudaGraphInstantiate(&b.graph[parity], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        b.graph[parity] = nullptr;
        return cuda_fail(e, "graph instantiate");
    }
    return PSC_OK;
}

int batch_plain_steps(psc_batch& b, int n) {
    if (b.graph_steps > 0 && n >= b.graph_steps) {
        if (!b.graph[b.parity]) PSC_TRY(batch_capture(b, b.parity));
        const int reps = n / b.graph_steps;
        for (int r = 0; r < reps; ++r) PSC_CUDA(cudaGraphLaunch(b.graph[b.parity], b.stream), "graph launch");
        n -= reps * b.graph_steps;  // an even graph length returns to this parity
    }
    for (int i = 0; i < n; ++i) {
        PSC_TRY(batch_launch(b, PSC_STEP_COLLIDE));
        b.parity ^= 1;
    }
    batch_sync_cur(b);
    for (auto& wp : b.w) {
        wp->stepped = true;
        wp->moments_ready = false;
        wp->loads_ready = false;
        wp->diag_ready = false;
    }
    return PSC_OK;
}

// Reductions of every window's current post-stream state into red_post
// (host copy in b.host + nwin * NRED); frozen windows report their rows at freezing.
int batch_observe(psc_batch& b, double* host_rows) {
    const int nwin = (int)b.w.size();
    PSC_TRY(batch_launch(b, PSC_STEP_REDUCE));
    PSC_TRY(psc_reduce_windows(b.table[b.parity].p, nwin, b.red_post.p, b.stream));
    PSC_CUDA(cudaMemcpyAsync(host_rows, b.red_post.p, (size_t)nwin * PSC_NRED * 8, cudaMemcpyDeviceToHost, b.stream),
             "batch reductions");
    PSC_CUDA(cudaStreamSynchronize(b.stream), "batch reductions");
    for (int k = 0; k < nwin; ++k)
        if (b.frozen[(size_t)k] >= 0)
            std::memcpy(host_rows + (size_t)k * PSC_NRED, b.frozen_red.data() + (size_t)k * PSC_NRED,
                        PSC_NRED * sizeof(double));
    return PSC_OK;
}

int batch_freeze(psc_batch& b, int k, const double* row) {
    b.frozen[(size_t)k] = b.parity;
    std::memcpy(b.frozen_red.data() + (size_t)k * PSC_NRED, row, PSC_NRED * sizeof(double));
    // set the flag in both device tables in place: captured graphs stay valid
    const size_t off = (size_t)k * sizeof(psc_window) + offsetof(psc_window, flags);
    int32_t flags = (b.w[(size_t)k]->moving ? PSC_WIN_MOVING : 0) | (b.w[(size_t)k]->cfg.open_x ? PSC_WIN_OPEN_X : 0);
    flags |= PSC_WIN_INACTIVE;
    for (int p = 0; p < 2; ++p)
        PSC_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(b.table[p].p) + off, &flags, sizeof(flags),
                                 cudaMemcpyHostToDevice, b.stream),
                 "freeze");
    PSC_CUDA(cudaStreamSynchronize(b.stream), "freeze");
    b.w[(size_t)k]->cur = b.parity;
    return PSC_OK;
}

}  // namespace
}  // namespace psc

extern "C" {

int psc_batch_create(const psc_config* h_cfgs, int nwin, const psc_launch* h_launch, int graph_steps, psc_batch** out) {
    if (!h_cfgs || !out || nwin <= 0) return fail(PSC_E_INVALID, "psc_batch_create: bad arguments");
    *out = nullptr;
    if (graph_steps < 0 || graph_steps % 2)
        return fail(PSC_E_INVALID, "psc_batch_create: graph_steps must be even and >= 0");
    for (int k = 0; k < nwin; ++k) {
        PSC_TRY(check_config(h_cfgs[k], "psc_batch_create"));
        if (h_cfgs[k].store != h_cfgs[0].store || h_cfgs[k].device != h_cfgs[0].device ||
            h_cfgs[k].stream != h_cfgs[0].stream)
            return fail(PSC_E_INVALID, "psc_batch_create: all windows need the same store, device and stream");
    }
    psc_launch lc = {0, 1, PSC_KERNEL_AUTO, 0, 0};
    if (h_launch) lc = *h_launch;
    if (lc.grid_ctas < 0) return fail(PSC_E_INVALID, "psc_batch_create: grid_ctas must be >= 0");
    if (lc.cells_per_thread != 1 && lc.cells_per_thread != 2 && lc.cells_per_thread != 4)
        return fail(PSC_E_INVALID, "psc_batch_create: cells_per_thread must be 1, 2 or 4");
    if (h_cfgs[0].store == PSC_STORE_F64_EXACT &&
        (lc.cells_per_thread != 1 || lc.kernel == PSC_KERNEL_TMA || lc.kernel == PSC_KERNEL_PAIR))
        return fail(PSC_E_UNSUPPORTED, "psc_batch_create: PSC_STORE_F64_EXACT runs the one-cell-per-thread kernel");
    if (lc.kernel == PSC_KERNEL_TMA && lc.stages == 0) lc.stages = 3;
    if (lc.kernel == PSC_KERNEL_AUTO && h_cfgs[0].store >= PSC_STORE_F32 && lc.cells_per_thread == 1) {
        // the pair kernel when every window has an even nz (as the Python batch decides)
        bool even = true;
        for (int k = 0; k < nwin; ++k) even = even && h_cfgs[k].nz % 2 == 0;
        if (even) lc.kernel = PSC_KERNEL_PAIR;
    }
    DeviceScope ds(h_cfgs[0].device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "psc_batch_create: cudaSetDevice");
    std::unique_ptr<psc_batch> b(new (std::nothrow) psc_batch());
    if (!b) return fail(PSC_E_CAPACITY, "psc_batch_create: out of host memory");
    b->device = h_cfgs[0].device;
    b->store = h_cfgs[0].store;
    b->launch = lc;
    b->graph_steps = graph_steps;
    if (h_cfgs[0].stream) {
        b->stream = as_stream(h_cfgs[0].stream);
    } else {
        PSC_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "psc_batch_create");
        b->own_stream = true;
    }
    int st = PSC_OK;
    for (int k = 0; k < nwin && st == PSC_OK; ++k) {
        b->w.emplace_back(new (std::nothrow) Window());
        if (!b->w.back()) {
            st = fail(PSC_E_CAPACITY, "psc_batch_create: out of host memory");
            break;
        }
        b->w.back()->imb_dual = true;
        st = window_init(*b->w.back(), h_cfgs[k], b->stream, "psc_batch_create");
        if (st == PSC_OK) st = window_set_particles(*b->w.back(), nullptr, 0, b->stream, "psc_batch_create");
    }
    b->frozen.assign((size_t)nwin, -1);
    b->staged.assign((size_t)nwin, -1);
    b->frozen_red.assign((size_t)nwin * PSC_NRED, 0.0);
    b->last.assign((size_t)nwin, psc_diag{});
    b->have_diag.assign((size_t)nwin, 0);
    b->built_desc.assign((size_t)nwin, 0);
    if (st == PSC_OK) {
        cudaError_t e = b->red_pre.ensure((int64_t)nwin * PSC_NRED, true, b->stream);
        if (e == cudaSuccess) e = b->red_post.ensure((int64_t)nwin * PSC_NRED, true, b->stream);
        if (e == cudaSuccess) e = b->red_next.ensure((int64_t)nwin * PSC_NRED, true, b->stream);
        if (e == cudaSuccess) e = b->diag.ensure((int64_t)nwin * PSC_NDIAG, true, b->stream);
        if (e == cudaSuccess) e = b->host.ensure((int64_t)nwin * kOutLen);
        if (e == cudaSuccess) e = b->lanes.init(1);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->up_done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->up_ready, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->up_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) st = cuda_fail(e, "psc_batch_create");
    }
    if (st != PSC_OK) {
        psc_batch_destroy(b.release());
        return st;
    }
    *out = b.release();
    return PSC_OK;
}

int psc_batch_destroy(psc_batch* b) {
    if (!b) return PSC_OK;
    DeviceScope ds(b->device);
    cudaStreamSynchronize(b->stream);
    if (b->up_stream) cudaStreamSynchronize(b->up_stream);
    cudaStream_t s = b->stream;
    bool own = b->own_stream;
    delete b;
    if (own) cudaStreamDestroy(s);
    return PSC_OK;
}

int psc_batch_set_particles(psc_batch* b, int win, const double* h_particles, int nparticles) {
    if (!b || win < 0 || win >= (int)b->w.size()) return fail(PSC_E_INVALID, "psc_batch_set_particles: bad window");
    ErrorCapture errors_(b->last_error);
    DeviceScope ds(b->device);
    PSC_TRY(batch_upload_join(*b, "psc_batch_set_particles"));
    b->staged[(size_t)win] = -1;  // the staging buffer no longer holds its accepted state
    return window_set_particles(*b->w[(size_t)win], h_particles, nparticles, b->stream, "psc_batch_set_particles");
}

int psc_batch_set_particles_all(psc_batch* b, const double* const* h_particles, const int* h_nparticles) {
    if (!b || !h_particles || !h_nparticles) return fail(PSC_E_INVALID, "psc_batch_set_particles_all: null argument");
    ErrorCapture errors_(b->last_error);
    DeviceScope ds(b->device);
    const char* who = "psc_batch_set_particles_all";
    const size_t nwin = b->w.size();
    int64_t total = 0;
    for (size_t k = 0; k < nwin; ++k) {
        if (h_nparticles[k] < 0) return fail(PSC_E_INVALID, std::string(who) + ": negative particle count");
        total += (int64_t)h_nparticles[k] * 10;
    }
    // one staging buffer and one host-to-device copy for all windows
    PSC_CUDA(cudaEventSynchronize(b->up_done), who);  // the previous upload has left the staging buffer
    const int64_t cap = b->up_dev.n < total ? total + total / 4 + 64 : b->up_dev.n;
    const double* const host_before = b->up_host.p;
    PSC_CUDA(b->up_host.ensure(cap), who);
    // where the staging buffer still holds a window's accepted state (the previous call's copy);
    // unknown from here until this call succeeds
    std::vector<int64_t> staged(nwin, -1);
    if (b->up_host.p == host_before) staged.swap(b->staged);
    b->staged.assign(nwin, -1);
    // pass 1: stage every window (an unchanged state is found in the same pass) and validate the
    // changed ones; one rejected window leaves every window as it was
    std::vector<int> known(nwin, 0);
    std::vector<int64_t> offs(nwin + 1, 0);
    for (size_t k = 0; k < nwin; ++k) {
        if (h_nparticles[k] > 0 && !h_particles[k])
            return fail(PSC_E_INVALID, std::string(who) + ": null particle array (window " + std::to_string(k) + ")");
        offs[k + 1] = offs[k] + (int64_t)h_nparticles[k] * 10;
    }
    // window k: copy into the staging buffer, note whether it equals the accepted state, check a
    // changed one for NaN / Inf (known[k] = 1 same, 2 changed and finite, -1 non-finite)
    // (where the buffer holds the accepted state at the same place, a read-only comparison: an
    // unchanged state is not written again)
    auto stage = [&](int k) {
        const Window& w = *b->w[(size_t)k];
        const int P = h_nparticles[k];
        const size_t n10 = (size_t)P * 10;
        double* dst = b->up_host.p + offs[(size_t)k];
        bool same = P == 0 && w.P == 0 && w.hp.empty();  // (empty before and now)
        if (P > 0 && P == w.P && w.hp.size() == n10 && staged[(size_t)k] == offs[(size_t)k]) {
            same = std::memcmp(dst, h_particles[k], n10 * sizeof(double)) == 0;
            if (!same) std::memcpy(dst, h_particles[k], n10 * sizeof(double));
        } else if (P > 0 && P == w.P && w.hp.size() == n10) {
            same = copy_same(dst, h_particles[k], w.hp.data(), n10);
        } else if (P > 0) {
            std::memcpy(dst, h_particles[k], n10 * sizeof(double));
        }
        known[(size_t)k] = same ? 1 : (particles_finite(h_particles[k], n10) ? 2 : -1);
    };
    for (size_t k = 0; k < nwin; ++k) stage((int)k);
    for (size_t k = 0; k < nwin; ++k)
        if (known[k] < 0)
            return fail(PSC_E_INVALID,
                        std::string(who) + ": particle state contains NaN or Inf (window " + std::to_string(k) + ")");
    // every fallible step of the windows that change their particle count, before any window
    // takes its new state
    for (size_t k = 0; k < nwin; ++k) PSC_TRY(window_reserve_particles(*b->w[k], h_nparticles[k], b->stream, who));
    // the device buffer grows only now: until every window is accepted the windows keep reading
    // the current one (a failed grow leaves it in place)
    if (b->up_dev.n < total) {
        PSC_CUDA(cudaStreamSynchronize(b->stream), who);  // kernels may still read the old buffer
        PSC_CUDA(b->up_dev.ensure(cap, false, b->stream), who);
    }
    // pass 2: every window takes its staged state (nothing here fails: validated and reserved above)
    int64_t off = 0;
    for (size_t k = 0; k < nwin; ++k) {
        Window& w = *b->w[k];
        const int P = h_nparticles[k];
        PSC_TRY(window_accept_particles(w, h_particles[k], P, b->stream, who, known[k]));
        w.ext_particles = b->up_dev.p + off;
        off += (int64_t)P * 10;
    }
    // after every kernel queued so far (they may read up_dev), on the upload stream
    PSC_CUDA(cudaEventRecord(b->up_ready, b->stream), who);
    PSC_CUDA(cudaStreamWaitEvent(b->up_stream, b->up_ready, 0), who);
    if (off > 0)
        PSC_CUDA(cudaMemcpyAsync(b->up_dev.p, b->up_host.p, (size_t)off * sizeof(double), cudaMemcpyHostToDevice,
                                 b->up_stream),
                 who);
    PSC_CUDA(cudaEventRecord(b->up_done, b->up_stream), who);
    b->up_pending = true;
    b->staged.assign(offs.begin(), offs.end() - 1);
    return PSC_OK;
}

int psc_batch_step(psc_batch* b, int nsteps, unsigned flags, psc_status* h_status) {
    if (!b) return fail(PSC_E_INVALID, "psc_batch_step: null handle");
    ErrorCapture errors_(b->last_error);
    if (nsteps < 0) return fail(PSC_E_INVALID, "psc_batch_step: negative step count");
    if (flags & ~(PSC_RUN_DIAG | PSC_RUN_FIELDS)) return fail(PSC_E_INVALID, "psc_batch_step: unknown flags");
    DeviceScope ds(b->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "psc_batch_step: cudaSetDevice");
    const bool diag = (flags & PSC_RUN_DIAG) != 0;
    const bool fields = (flags & PSC_RUN_FIELDS) != 0;
    const int nwin = (int)b->w.size();
    if (nsteps == 0) return PSC_OK;
    PSC_TRY(batch_prepare(*b, diag, fields));
    const size_t rows = (size_t)nwin * PSC_NRED;
    const std::vector<uint64_t> inputs = batch_step_inputs(*b);
    // a step run ahead by the previous reporting call with these inputs is this call's first step
    int remaining = nsteps;
    bool final_done = false;  // the final step's populations, IMB field and red_pre are in place
    if (b->ahead_ready) {
        b->ahead_ready = false;
        if (inputs == b->ahead_inputs) {
            b->parity ^= 1;
            batch_sync_cur(*b);
            --remaining;
            if (remaining == 0 && diag) {
                PSC_CUDA(cudaMemcpyAsync(b->red_pre.p, b->red_next.p, rows * 8, cudaMemcpyDeviceToDevice, b->stream),
                         "psc_batch_step");
                for (int k = 0; k < nwin; ++k)
                    if (b->frozen[(size_t)k] < 0) b->w[(size_t)k]->imb_par = b->w[(size_t)k]->cur;
                final_done = true;
            }
        }
    }
    PSC_TRY(batch_plain_steps(*b, diag && !final_done ? remaining - 1 : remaining));
    if (diag) {
        if (!final_done) {  // final step: IMB and partials
            PSC_TRY(batch_launch(*b, PSC_STEP_COLLIDE | PSC_STEP_IMB | PSC_STEP_REDUCE));
            b->parity ^= 1;
            batch_sync_cur(*b);
            PSC_TRY(psc_reduce_windows(b->table[b->parity].p, nwin, b->red_pre.p, b->stream));
            for (int k = 0; k < nwin; ++k)
                if (b->frozen[(size_t)k] < 0) b->w[(size_t)k]->imb_par = b->w[(size_t)k]->cur;
        }
        // the loads of every active window in one launch sequence read the IMB field and geometry
        // only: on a lane, beside the post-stream reductions, which come from the next step run
        // ahead (it writes the other buffer and IMB field only) or from a reduction-only pass.  The
        // main stream's kernel is launched first: the loads wait for the particle upload anyway.
        PSC_TRY(batch_loads_table(*b, "psc_batch_step"));
        PSC_CUDA(b->lanes.begin(b->stream), "psc_batch_step");
        const bool ahead = batch_may_run_ahead(*b, fields, inputs);
        const double* post_rows = ahead ? b->red_next.p : b->red_post.p;
        if (ahead) {
            PSC_TRY(batch_launch(*b, PSC_STEP_COLLIDE | PSC_STEP_IMB | PSC_STEP_REDUCE));
            PSC_TRY(psc_reduce_windows(b->table[b->parity ^ 1].p, nwin, b->red_next.p, b->stream));
        } else {
            PSC_TRY(batch_launch(*b, PSC_STEP_REDUCE | (fields ? PSC_STEP_MOMENTS : 0u)));
            PSC_TRY(psc_reduce_windows(b->table[b->parity].p, nwin, b->red_post.p, b->stream));
        }
        if (b->up_pending)  // the loads read the particles: after their upload
            PSC_CUDA(cudaStreamWaitEvent(b->lanes.lane(0), b->up_done, 0), "psc_batch_step");
        PSC_CUDA(launch_particle_loads_multi(batch_jobs(*b), batch_chunk_base(*b),
                                             batch_particle_base(*b), b->jobs_n, b->jobs_chunks, b->jobs_particles,
                                             b->w[0]->field_type(), b->jobs_max_s, b->jobs_all_lists,
                                             b->jobs_list_ready,
                                             b->loads_part.p, b->lanes.lane(0)),
                 "psc_batch_step: particle loads");
        for (int k = 0; k < nwin; ++k)
            if (b->frozen[(size_t)k] < 0) {
                b->w[(size_t)k]->loads_enqueued();
                b->w[(size_t)k]->loads_ready = true;
            }
        PSC_CUDA(b->lanes.end(b->stream), "psc_batch_step");
        double* host = b->host.p;
        PSC_CUDA(cudaMemcpyAsync(host, b->red_pre.p, rows * 8, cudaMemcpyDeviceToHost, b->stream), "psc_batch_step");
        PSC_CUDA(cudaMemcpyAsync(host + rows, post_rows, rows * 8, cudaMemcpyDeviceToHost, b->stream),
                 "psc_batch_step");
        PSC_CUDA(cudaMemcpyAsync(host + 2 * rows, b->diag.p, (size_t)nwin * PSC_NDIAG * 8, cudaMemcpyDeviceToHost,
                                 b->stream),
                 "psc_batch_step");
        PSC_CUDA(cudaStreamSynchronize(b->stream), "psc_batch_step");
        if (ahead) {
            b->ahead_ready = true;
            b->ahead_inputs = inputs;
        }
        b->report_inputs = inputs;
        for (int k = 0; k < nwin; ++k) {
            Window& w = *b->w[(size_t)k];
            if (b->frozen[(size_t)k] >= 0) continue;
            double row[kOutLen];
            std::memcpy(row, host + (size_t)k * PSC_NRED, PSC_NRED * 8);
            std::memcpy(row + PSC_NRED, host + rows + (size_t)k * PSC_NRED, PSC_NRED * 8);
            std::memcpy(row + 2 * PSC_NRED, host + 2 * rows + (size_t)k * PSC_NDIAG, PSC_NDIAG * 8);
            if (ahead)  // the step run ahead added its own IMB; a reduction pass adds none
                for (int q = PSC_RED_IMBX; q <= PSC_RED_IMBZ; ++q) row[PSC_NRED + q] = 0.0;
            fill_diag(w, row, b->last[(size_t)k]);
            b->have_diag[(size_t)k] = 1;
            w.stepped = true;
            w.moments_ready = fields;
            w.diag_ready = true;
        }
    } else if (fields) {
        PSC_TRY(batch_launch(*b, PSC_STEP_MOMENTS));
        for (auto& wp : b->w) wp->moments_ready = true;
        PSC_CUDA(cudaStreamSynchronize(b->stream), "psc_batch_step");
    } else {
        PSC_CUDA(cudaGetLastError(), "psc_batch_step");
    }
    PSC_TRY(batch_upload_join(*b, "psc_batch_step"));  // later calls see the main stream after the upload
    if (h_status)
        for (int k = 0; k < nwin; ++k) {
            h_status[k] = psc_status{};
            h_status[k].steps_done = b->frozen[(size_t)k] >= 0 ? 0 : nsteps;
            h_status[k].residual = INFINITY;
            h_status[k].diag = b->last[(size_t)k];
        }
    return PSC_OK;
}

int psc_batch_converge(psc_batch* b, double tol, int check_every, int max_steps, int min_steps, int freeze,
                       psc_status* h_status) {
    if (!b) return fail(PSC_E_INVALID, "psc_batch_converge: null handle");
    ErrorCapture errors_(b->last_error);
    if (!(tol > 0.0) || check_every < 2 || max_steps < 2 || min_steps < 0)
        return fail(PSC_E_INVALID, "psc_batch_converge: need tol > 0, check_every >= 2, max_steps >= 2");
    DeviceScope ds(b->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "psc_batch_converge: cudaSetDevice");
    const int nwin = (int)b->w.size();
    PSC_TRY(batch_upload_join(*b, "psc_batch_converge"));
    b->ahead_ready = false;  // its own loop of plain steps and observations
    PSC_TRY(batch_prepare(*b, false, false));
    std::vector<double> r1((size_t)nwin * PSC_NRED), r2((size_t)nwin * PSC_NRED);
    std::vector<int> conv((size_t)nwin, -1);
    std::vector<double> resid((size_t)nwin, INFINITY);
    int done = 0;
    while (done < max_steps) {
        const int n = std::max(0, std::min(check_every - 1, max_steps - done - 1));
        PSC_TRY(batch_plain_steps(*b, n));
        done += n;
        PSC_TRY(batch_observe(*b, r1.data()));
        PSC_TRY(batch_plain_steps(*b, 1));
        done += 1;
        PSC_TRY(batch_observe(*b, r2.data()));
        bool all = true;
        for (int k = 0; k < nwin; ++k) {
            const Window& w = *b->w[(size_t)k];
            const double* row2 = r2.data() + (size_t)k * PSC_NRED;
            if (row2[PSC_RED_NONFINITE] > 0.0)
                return fail(PSC_E_INVALID, "psc_batch_converge: non-finite moments in window " + std::to_string(k));
            const double k1 = row_permeability(w, r1.data() + (size_t)k * PSC_NRED);
            const double k2 = row_permeability(w, row2);
            if (conv[(size_t)k] < 0) {
                resid[(size_t)k] = std::fabs(k2 - k1) / std::max(std::fabs(k2), 1e-300);
                if (resid[(size_t)k] < tol && done >= min_steps) {
                    conv[(size_t)k] = done;
                    if (freeze) PSC_TRY(batch_freeze(*b, k, row2));
                }
            }
            all = all && conv[(size_t)k] >= 0;
        }
        if (all) break;
    }
    PSC_TRY(batch_observe(*b, r2.data()));
    for (int k = 0; k < nwin; ++k) {
        Window& w = *b->w[(size_t)k];
        double row[kOutLen] = {0};
        std::memcpy(row + PSC_NRED, r2.data() + (size_t)k * PSC_NRED, PSC_NRED * 8);
        psc_diag d{};
        fill_diag(w, row, d);
        if (h_status) {
            h_status[k] = psc_status{};
            h_status[k].steps_done = conv[(size_t)k] >= 0 ? conv[(size_t)k] : done;
            h_status[k].converged = conv[(size_t)k] >= 0;
            h_status[k].residual = resid[(size_t)k];
            h_status[k].diag = d;
        }
    }
    return PSC_OK;
}

const char* psc_batch_last_error(const psc_batch* b) { return b ? b->last_error.c_str() : ""; }

int psc_batch_get_diag(psc_batch* b, int win, psc_diag* h_diag) {
    if (!b || !h_diag || win < 0 || win >= (int)b->w.size())
        return fail(PSC_E_INVALID, "psc_batch_get_diag: bad arguments");
    ErrorCapture errors_(b->last_error);
    if (!b->have_diag[(size_t)win])
        return fail(PSC_E_INVALID, "psc_batch_get_diag: no PSC_RUN_DIAG step has run for this window");
    *h_diag = b->last[(size_t)win];
    return PSC_OK;
}

int psc_batch_get_loads(psc_batch* b, int win, double* h_forces, double* h_torques) {
    if (!b || win < 0 || win >= (int)b->w.size()) return fail(PSC_E_INVALID, "psc_batch_get_loads: bad window");
    ErrorCapture errors_(b->last_error);
    Window& w = *b->w[(size_t)win];
    if (w.P == 0) return PSC_OK;
    if (!h_forces || !h_torques) return fail(PSC_E_INVALID, "psc_batch_get_loads: null output");
    if (!w.loads_ready) return fail(PSC_E_INVALID, "psc_batch_get_loads: no PSC_RUN_DIAG step has run since the last step");
    DeviceScope ds(b->device);
    PSC_CUDA(cudaMemcpyAsync(h_forces, w.forces.p, (size_t)w.P * 24, cudaMemcpyDeviceToHost, b->stream),
             "psc_batch_get_loads");
    PSC_CUDA(cudaMemcpyAsync(h_torques, w.torques.p, (size_t)w.P * 24, cudaMemcpyDeviceToHost, b->stream),
             "psc_batch_get_loads");
    PSC_CUDA(cudaStreamSynchronize(b->stream), "psc_batch_get_loads");
    return PSC_OK;
}

int psc_batch_get_fields(psc_batch* b, int win, int which, double* h_dst) {
    if (!b || win < 0 || win >= (int)b->w.size()) return fail(PSC_E_INVALID, "psc_batch_get_fields: bad window");
    ErrorCapture errors_(b->last_error);
    DeviceScope ds(b->device);
    Window& w = *b->w[(size_t)win];
    batch_sync_cur(*b);
    PSC_TRY(batch_upload_join(*b, "psc_batch_get_fields"));
    return window_get_field(w, which, h_dst, b->stream, b->tot, "psc_batch_get_fields");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// adjoint of the permeability (no counterpart in the reference)
// ---------------------------------------------------------------------------
struct psc_adjoint {
    std::string last_error;  // message of the last failed call on this handle
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    Window w;  // smooth geometry, PSC_STORE_F32 / F64 deviation storage
    HArray<int64_t> tot;
    HArray<double> host;
    int steps = 0, every = 0;
    std::vector<std::unique_ptr<DArray<unsigned char>>> ckpt;  // S_t at t = 0, every, 2 every, ...
    DArray<unsigned char> states;                              // one segment's recomputed states
    DArray<psc_window> seg_tab;                                // their step descriptors
    DArray<unsigned char> lam[2];
    DArray<double> dKdB, dKds, red, gpart, grad;
    bool forward_done = false;
    double K = 0.0;
};

namespace psc {
namespace {

size_t adj_state_bytes(const psc_adjoint& a) { return (size_t)19 * a.w.N * a.w.elem; }

psc_adjoint_args adj_args(const psc_adjoint& a) {
    const Window& w = a.w;
    const double* F = w.cfg.force;
    const double fmag = std::sqrt(F[0] * F[0] + F[1] * F[1] + F[2] * F[2]);
    psc_adjoint_args r{};
    r.nx = w.cfg.nx;
    r.ny = w.cfg.ny;
    r.nz = w.cfg.nz;
    r.store = w.cfg.store;
    r.tau = w.cfg.tau;
    r.force[0] = F[0];
    r.force[1] = F[1];
    r.force[2] = F[2];
    r.kappa = (w.cfg.tau - 0.5) / 3.0 / (fmag * (double)w.N);
    r.dir[0] = F[0] / fmag;
    r.dir[1] = F[1] / fmag;
    r.dir[2] = F[2] / fmag;
    r.solid = w.solid.p;
    r.dKdB = a.dKdB.p;
    r.dKdsolid = a.dKds.p;
    return r;
}

// States S_t0 .. S_{t1-1} of one segment, recomputed from its checkpoint.
int adj_segment(psc_adjoint& a, int t0, int t1) {
    Window& w = a.w;
    cudaStream_t s = a.stream;
    const size_t sb = adj_state_bytes(a);
    const int L = t1 - t0;
    PSC_CUDA(cudaMemcpyAsync(a.states.p, a.ckpt[(size_t)(t0 / a.every)]->p, sb, cudaMemcpyDeviceToDevice, s),
             "psc_adjoint_backward");
    if (L < 2) return PSC_OK;
    std::vector<psc_window> tab((size_t)(L - 1));
    for (int k = 0; k < L - 1; ++k) {
        psc_window d = w.descriptor(0);
        d.f_src = a.states.p + (size_t)k * sb;
        d.f_dst = a.states.p + (size_t)(k + 1) * sb;
        d.imb = nullptr;
        d.moments = nullptr;
        d.flags &= ~PSC_WIN_MOVING;
        int64_t total = 0;
        PSC_TRY(psc_plan_tiles(&d, 1, 0, &total));
        tab[(size_t)k] = d;
    }
    PSC_CUDA(a.seg_tab.ensure(L - 1, false, s), "psc_adjoint_backward");
    PSC_CUDA(cudaMemcpyAsync(a.seg_tab.p, tab.data(), (size_t)(L - 1) * sizeof(psc_window), cudaMemcpyHostToDevice, s),
             "psc_adjoint_backward");
    psc_launch c = {0, 1, PSC_KERNEL_AUTO, 0, 0};
    for (int k = 0; k < L - 1; ++k)
        PSC_TRY(psc_step_windows_ex(w.cfg.store, a.seg_tab.p + k, 1, tab[(size_t)k].tile_count, PSC_STEP_COLLIDE, &c, s));
    PSC_CUDA(cudaStreamSynchronize(s), "psc_adjoint_backward");  // tab lives on this frame
    return PSC_OK;
}

}  // namespace
}  // namespace psc

extern "C" {

int psc_adjoint_create(const psc_config* h_cfg, double smooth_eps, int steps, int checkpoint_every,
                       psc_adjoint** out) {
    if (!h_cfg || !out) return fail(PSC_E_INVALID, "psc_adjoint_create: null argument");
    *out = nullptr;
    PSC_TRY(check_config(*h_cfg, "psc_adjoint_create"));
    if (h_cfg->store != PSC_STORE_F32 && h_cfg->store != PSC_STORE_F64)
        return fail(PSC_E_UNSUPPORTED, "psc_adjoint_create: the adjoint runs in PSC_STORE_F32 or PSC_STORE_F64");
    if (!(smooth_eps > 0.0) || !std::isfinite(smooth_eps))
        return fail(PSC_E_INVALID, "psc_adjoint_create: smooth_eps must be > 0");
    if (steps < 1 || checkpoint_every < 1) return fail(PSC_E_INVALID, "psc_adjoint_create: steps and checkpoint_every must be >= 1");
    if (!(h_cfg->tau > 0.5)) return fail(PSC_E_INVALID, "psc_adjoint_create: tau must exceed 0.5");
    if (h_cfg->tau_minus > 0.0 || h_cfg->open_x)
        return fail(PSC_E_UNSUPPORTED, "psc_adjoint_create: the adjoint runs BGK on periodic windows");
    const double* F = h_cfg->force;
    if (!(F[0] * F[0] + F[1] * F[1] + F[2] * F[2] > 0.0))
        return fail(PSC_E_INVALID, "psc_adjoint_create: the permeability needs a non-zero body force");
    DeviceScope ds(h_cfg->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "psc_adjoint_create: cudaSetDevice");
    std::unique_ptr<psc_adjoint> a(new (std::nothrow) psc_adjoint());
    if (!a) return fail(PSC_E_CAPACITY, "psc_adjoint_create: out of host memory");
    a->device = h_cfg->device;
    a->steps = steps;
    a->every = checkpoint_every;
    if (h_cfg->stream) {
        a->stream = as_stream(h_cfg->stream);
    } else {
        PSC_CUDA(cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking), "psc_adjoint_create");
        a->own_stream = true;
    }
    psc_config c = *h_cfg;
    c.static_geometry = 1;
    a->w.smooth_eps = smooth_eps;
    int st = window_init(a->w, c, a->stream, "psc_adjoint_create");
    if (st == PSC_OK) st = window_set_particles(a->w, nullptr, 0, a->stream, "psc_adjoint_create");
    if (st != PSC_OK) {
        psc_adjoint_destroy(a.release());
        return st;
    }
    *out = a.release();
    return PSC_OK;
}

const char* psc_adjoint_last_error(const psc_adjoint* a) { return a ? a->last_error.c_str() : ""; }

int psc_adjoint_destroy(psc_adjoint* a) {
    if (!a) return PSC_OK;
    DeviceScope ds(a->device);
    cudaStreamSynchronize(a->stream);
    cudaStream_t s = a->stream;
    bool own = a->own_stream;
    delete a;
    if (own) cudaStreamDestroy(s);
    return PSC_OK;
}

int psc_adjoint_forward(psc_adjoint* a, const double* h_particles, int nparticles, double* h_K) {
    if (!a || !h_K) return fail(PSC_E_INVALID, "psc_adjoint_forward: null argument");
    ErrorCapture errors_(a->last_error);
    DeviceScope ds(a->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "psc_adjoint_forward: cudaSetDevice");
    Window& w = a->w;
    cudaStream_t s = a->stream;
    const char* who = "psc_adjoint_forward";
    // the particles are static for the run: their velocities do not enter
    PSC_TRY(window_set_particles(w, h_particles, nparticles, s, who));
    PSC_TRY(window_rebuild(w, s, a->tot, who));
    if (w.moving) {
        w.moving = false;
        w.touch();
    }
    PSC_TRY(psc_init_equilibrium(w.cfg.store, w.scale, w.f[0].p, w.N, s));
    w.cur = 0;
    const size_t sb = adj_state_bytes(*a);
    const int nck = (a->steps + a->every - 1) / a->every;
    while ((int)a->ckpt.size() < nck) a->ckpt.emplace_back(new DArray<unsigned char>());
    for (int t = 0; t < a->steps; ++t) {
        if (t % a->every == 0) {
            DArray<unsigned char>& ck = *a->ckpt[(size_t)(t / a->every)];
            PSC_CUDA(ck.ensure((int64_t)sb, false, s), who);
            PSC_CUDA(cudaMemcpyAsync(ck.p, w.f[w.cur].p, sb, cudaMemcpyDeviceToDevice, s), who);
        }
        PSC_TRY(launch_solo(w, PSC_STEP_COLLIDE, s));
        w.cur ^= 1;
    }
    PSC_TRY(launch_solo(w, PSC_STEP_REDUCE, s));
    PSC_CUDA(a->red.ensure(PSC_NRED, true, s), who);
    PSC_TRY(psc_reduce_windows(w.solo[w.cur].p, 1, a->red.p, s));
    PSC_CUDA(a->host.ensure(PSC_NRED), who);
    PSC_CUDA(cudaMemcpyAsync(a->host.p, a->red.p, PSC_NRED * sizeof(double), cudaMemcpyDeviceToHost, s), who);
    PSC_CUDA(cudaStreamSynchronize(s), who);
    a->K = row_permeability(w, a->host.p);
    a->forward_done = true;
    *h_K = a->K;
    return PSC_OK;
}

int psc_adjoint_backward(psc_adjoint* a, double* h_grad) {
    if (!a) return fail(PSC_E_INVALID, "psc_adjoint_backward: null handle");
    ErrorCapture errors_(a->last_error);
    if (!a->forward_done) return fail(PSC_E_INVALID, "psc_adjoint_backward: call psc_adjoint_forward first");
    Window& w = a->w;
    if (w.P > 0 && !h_grad) return fail(PSC_E_INVALID, "psc_adjoint_backward: null output");
    DeviceScope ds(a->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "psc_adjoint_backward: cudaSetDevice");
    cudaStream_t s = a->stream;
    const char* who = "psc_adjoint_backward";
    const size_t sb = adj_state_bytes(*a);
    PSC_CUDA(a->lam[0].ensure((int64_t)sb, false, s), who);
    PSC_CUDA(a->lam[1].ensure((int64_t)sb, false, s), who);
    PSC_CUDA(a->dKdB.ensure(w.N, false, s), who);
    PSC_CUDA(a->dKds.ensure(w.N, false, s), who);
    PSC_CUDA(cudaMemsetAsync(a->dKdB.p, 0, (size_t)w.N * 8, s), who);
    PSC_CUDA(cudaMemsetAsync(a->dKds.p, 0, (size_t)w.N * 8, s), who);
    PSC_CUDA(a->states.ensure((int64_t)sb * std::min(a->every, a->steps), false, s), who);
    psc_adjoint_args args = adj_args(*a);
    args.state = w.f[w.cur].p;
    args.lam_out = a->lam[0].p;
    PSC_TRY(psc_adjoint_seed(&args, s));
    int cur = 0;
    const int nseg = (a->steps + a->every - 1) / a->every;
    for (int seg = nseg - 1; seg >= 0; --seg) {
        const int t0 = seg * a->every;
        const int t1 = std::min(t0 + a->every, a->steps);
        PSC_TRY(adj_segment(*a, t0, t1));
        for (int t = t1 - 1; t >= t0; --t) {
            args.state = a->states.p + (size_t)(t - t0) * sb;
            args.lam_in = a->lam[cur].p;
            args.lam_out = a->lam[1 - cur].p;
            PSC_TRY(psc_adjoint_step(&args, s));
            cur = 1 - cur;
        }
    }
    psc_geometry g = w.geometry();
    PSC_CUDA(a->gpart.ensure(std::max<int64_t>(w.cap_chunks, 1) * 4, false, s), who);
    PSC_CUDA(a->grad.ensure((int64_t)std::max(w.P, 1) * 4, true, s), who);
    PSC_TRY(psc_adjoint_geometry_grad(&g, &args, a->gpart.p, a->grad.p, s));
    if (w.P > 0)
        PSC_CUDA(cudaMemcpyAsync(h_grad, a->grad.p, (size_t)w.P * 4 * sizeof(double), cudaMemcpyDeviceToHost, s), who);
    PSC_CUDA(cudaStreamSynchronize(s), who);
    return PSC_OK;
}

}  // extern "C"
