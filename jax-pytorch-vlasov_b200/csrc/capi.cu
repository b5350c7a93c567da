// C ABI of the Vlasov-Poisson library: argument checks, workspace layout and
// the launch sequence of one Strang step. Declarations and the reference
// functions each entry point replaces: include/vlasov_b200.h.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>

#include "common.cuh"
#include "launch.h"

namespace vp {

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

int set_error(int code, const char* msg) {
    g_last_error = msg ? msg : "";
    return code;
}

int set_cuda_error(const char* what) {
    const cudaError_t e = cudaGetLastError();
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return VP_ERR_CUDA;
}

int check_launch(const char* what) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return VP_OK;
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return VP_ERR_CUDA;
}

int sm_count() {
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cache[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = n > 0 ? n : 148;
    }
    return cache[dev];
}

int occupancy_raw(const void* kern, int block, size_t smem) {
    struct Entry {
        const void* k;
        int block;
        size_t smem;
        int dev;
        int occ;
    };
    static Entry cache[128];
    static int used = 0;
    static std::mutex mu;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    for (int i = 0; i < used; ++i)
        if (cache[i].k == kern && cache[i].block == block && cache[i].smem == smem && cache[i].dev == dev)
            return cache[i].occ;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, block, smem) != cudaSuccess) {
        cudaGetLastError();
        n = 1;
    }
    if (n < 1) n = 1;
    if (used < 128) cache[used++] = Entry{kern, block, smem, dev, n};
    return n;
}

// Optional timing events around the phases of a step (events[2p], events[2p+1]).
struct Marks {
    void* const* ev;
    cudaStream_t st;
    int rec(int i) const {
        if (!ev || !ev[i]) return VP_OK;
        if (cudaEventRecord(static_cast<cudaEvent_t>(ev[i]), st) != cudaSuccess)
            return set_cuda_error("cudaEventRecord(timing event)");
        return VP_OK;
    }
    int begin(int p) const { return rec(2 * p); }
    int end(int p) const { return rec(2 * p + 1); }
};

static size_t al(size_t b) { return (b + 255) & ~size_t(255); }

static bool dtype_ok(int d) { return d == VP_F32 || d == VP_F64 || d == VP_BF16; }

static size_t drift_rho_part_bytes(int64_t n_outer, int64_t n_line, int64_t n_inner) {
    const int64_t tiles = (n_inner + 127) / 128;  // worst case: one column per thread, 128 threads per tile
    return al((size_t)n_outer * tiles * n_line * sizeof(double));
}

size_t step2d_layout(int64_t nx, int64_t ny, int64_t nvx, int64_t nvy, char* base, Step2dWs* w) {
    size_t off = 0;
    auto take = [&](size_t b) {
        char* p = base ? base + off : nullptr;
        off += al(b);
        return p;
    };
    Step2dWs t;
    // density partials: per 128-column tile of the y sweep, or per
    // 32-column group of the fused (x, y) pass
    const size_t part_sweep = drift_rho_part_bytes(nx, ny, nvx * nvy);
    const size_t part_plane = al((size_t)nx * ny * (size_t)plane_part_tiles(nvx, nvy) * sizeof(double));
    t.part = reinterpret_cast<double*>(take(std::max(part_sweep, part_plane)));
    t.rho = reinterpret_cast<double*>(take((size_t)nx * ny * sizeof(double)));
    t.ex = reinterpret_cast<double*>(take((size_t)nx * ny * sizeof(double)));
    t.ey = reinterpret_cast<double*>(take((size_t)nx * ny * sizeof(double)));
    t.moments = reinterpret_cast<double*>(take((size_t)nx * ny * 4 * sizeof(double)));
    t.pois = take(poisson2d_ws_bytes(nx, ny));
    if (w) *w = t;
    return off;
}

struct Step1dWs {
    double *part, *n, *e, *parts;
};

static size_t step1d_layout(int64_t nx, int64_t nv, char* base, Step1dWs* w) {
    size_t off = 0;
    auto take = [&](size_t b) {
        char* p = base ? base + off : nullptr;
        off += al(b);
        return p;
    };
    Step1dWs t;
    t.part = reinterpret_cast<double*>(take(drift_rho_part_bytes(1, nx, nv)));
    t.n = reinterpret_cast<double*>(take((size_t)nx * sizeof(double)));
    t.e = reinterpret_cast<double*>(take((size_t)nx * sizeof(double)));
    t.parts = reinterpret_cast<double*>(take(4 * sizeof(double)));
    if (w) *w = t;
    return off;
}

}  // namespace vp

using namespace vp;

#define VP_CHECK(cond, msg) \
    do {                    \
        if (!(cond)) return set_error(VP_ERR_ARG, msg); \
    } while (0)

static cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

extern "C" {

const char* vp_version(void) { return "vlasov_b200 0.1 (sm_100a)"; }
const char* vp_last_error(void) { return g_last_error.c_str(); }
uint64_t vp_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int vp_drift(const void* f_in, void* f_out, int dtype, int64_t n_outer, int64_t n_line, int64_t n_inner,
             int64_t sel_div, int64_t sel_mod, const int32_t* shift, int32_t shift_spread, const void* W,
             void* stream) {
    if (!dtype_ok(dtype)) return set_error(VP_ERR_DTYPE, "vp_drift: unknown dtype");
    VP_CHECK(f_in && f_out && shift && W, "vp_drift: null pointer");
    VP_CHECK(f_in != f_out, "vp_drift: f_out must not alias f_in");
    VP_CHECK(n_outer > 0 && n_line > 0 && n_inner > 0 && sel_div > 0 && sel_mod > 0, "vp_drift: bad size");
    VP_CHECK(n_line < (1 << 30), "vp_drift: line too long");
    return run_strided(dtype, f_in, f_out, n_outer, n_line, n_inner, false, sel_div, sel_mod, shift_spread, shift, W, nullptr, 0,
                       1, 0.0, 1.0, -1, nullptr, nullptr, EQ_NONE, S(stream));
}

size_t vp_drift_rho_workspace_bytes(int64_t n_outer, int64_t n_line, int64_t n_inner) {
    return drift_rho_part_bytes(n_outer, n_line, n_inner);
}

int vp_drift_rho(const void* f_in, void* f_out, int dtype, int64_t n_outer, int64_t n_line, int64_t n_inner,
                 int64_t sel_div, int64_t sel_mod, const int32_t* shift, int32_t shift_spread, const void* W,
                 double scale, double* rho,
                 void* workspace, size_t workspace_bytes, void* stream) {
    if (!dtype_ok(dtype)) return set_error(VP_ERR_DTYPE, "vp_drift_rho: unknown dtype");
    VP_CHECK(f_in && f_out && shift && W && rho, "vp_drift_rho: null pointer");
    VP_CHECK(f_in != f_out, "vp_drift_rho: f_out must not alias f_in");
    VP_CHECK(n_outer > 0 && n_line > 0 && n_inner > 0 && sel_div > 0 && sel_mod > 0, "vp_drift_rho: bad size");
    VP_CHECK(n_line < (1 << 30), "vp_drift_rho: line too long");
    if (!workspace || workspace_bytes < drift_rho_part_bytes(n_outer, n_line, n_inner))
        return set_error(VP_ERR_WORKSPACE, "vp_drift_rho: workspace too small");
    int tiles = 0;
    double* part = static_cast<double*>(workspace);
    int rc = run_strided(dtype, f_in, f_out, n_outer, n_line, n_inner, false, sel_div, sel_mod, shift_spread, shift, W, nullptr,
                         0, 1, 0.0, 1.0, -1, part, &tiles, EQ_NONE, S(stream));
    if (rc) return rc;
    return run_rho_finalize(part, n_outer, n_line, tiles, scale, 0.0, rho, S(stream));
}

size_t vp_drift_pair_workspace_bytes(int64_t nx, int64_t ny, int64_t nvx, int64_t nvy) {
    if (nx <= 0 || ny <= 0 || nvx <= 0 || nvy <= 0) return 0;
    return (size_t)nx * (size_t)plane_part_tiles(nvx, nvy) * (size_t)ny * sizeof(double);
}

int vp_drift_pair(const void* f_in, void* f_out, int dtype, int64_t nx, int64_t ny, int64_t nvx, int64_t nvy,
                  int32_t xfirst, int64_t x_begin, int64_t x_count, const int32_t* shift_x, const void* W_x,
                  const int32_t* shift_y, const void* W_y, double scale, double* rho, void* workspace,
                  size_t workspace_bytes, void* stream) {
    if (!dtype_ok(dtype)) return set_error(VP_ERR_DTYPE, "vp_drift_pair: unknown dtype");
    VP_CHECK(f_in && f_out && shift_x && W_x && shift_y && W_y, "vp_drift_pair: null pointer");
    VP_CHECK(f_in != f_out, "vp_drift_pair: f_out must not alias f_in");
    VP_CHECK(nx > 0 && ny > 0 && nvx > 0 && nvy > 0, "vp_drift_pair: bad size");
    VP_CHECK(x_begin >= 0 && x_count > 0 && x_begin + x_count <= nx, "vp_drift_pair: output rows outside [0, nx)");
    VP_CHECK(!rho || xfirst, "vp_drift_pair: the density comes with the x-then-y order");
    if (!plane_fits(dtype, nx, ny, nvx, nvy, f_in) || !plane_fits(dtype, nx, ny, nvx, nvy, f_out))
        return set_error(VP_ERR_UNSUPPORTED,
                         "vp_drift_pair: needs FP32, 16 <= ny <= 128, nvy % 32 == 0 and 16-byte aligned buffers");
    double* part = nullptr;
    if (rho) {
        if (!workspace || workspace_bytes < vp_drift_pair_workspace_bytes(nx, ny, nvx, nvy))
            return set_error(VP_ERR_WORKSPACE, "vp_drift_pair: workspace too small");
        part = static_cast<double*>(workspace);
    }
    int tiles = 0;
    int rc = run_plane(dtype, xfirst != 0, f_in, f_out, nx, ny, nvx, nvy, x_begin, x_count, shift_x, W_x, shift_y,
                       W_y, part, &tiles, EQ_NONE, nullptr, 0, S(stream));
    if (rc || !rho) return rc;
    // the partials are [nx][tiles][ny]: the range's rows are contiguous
    return run_rho_finalize(part + x_begin * tiles * ny, x_count, ny, tiles, scale, 0.0, rho + x_begin * ny, S(stream));
}

int vp_kick(const void* f_in, void* f_out, int dtype, int64_t n_outer, int64_t n_line, int64_t n_inner,
            const void* E, int e_dtype, int64_t e_div, double dt, double dv, int32_t window, void* stream) {
    if (!dtype_ok(dtype)) return set_error(VP_ERR_DTYPE, "vp_kick: unknown dtype");
    VP_CHECK(f_in && f_out && E, "vp_kick: null pointer");
    VP_CHECK(f_in != f_out, "vp_kick: f_out must not alias f_in");
    VP_CHECK(n_outer > 0 && n_line > 0 && n_inner > 0 && e_div > 0, "vp_kick: bad size");
    VP_CHECK(e_dtype == VP_F32 || e_dtype == VP_F64, "vp_kick: E must be float32 or float64");
    VP_CHECK(dv != 0.0, "vp_kick: dv == 0");
    VP_CHECK(n_line < (1 << 30), "vp_kick: line too long");
    const int e_f64 = e_dtype == VP_F64;
    if (n_inner == 1)
        return run_kick_contig(dtype, f_in, f_out, n_outer, n_line, E, e_f64, e_div, dt, dv, window, EQ_NONE,
                               S(stream));
    return run_strided(dtype, f_in, f_out, n_outer, n_line, n_inner, true, 1, 1, -1, nullptr, nullptr, E, e_f64, e_div,
                       dt, dv, window, nullptr, nullptr, EQ_NONE, S(stream));
}

int vp_kick2d(const void* f_in, void* f_out, int dtype, int64_t n_planes, int64_t nvx, int64_t nvy,
              const double* Ex, const double* Ey, double dt, double dvx, double dvy, int32_t window,
              const double* vx, const double* vy, double* moments, void* stream) {
    if (!dtype_ok(dtype)) return set_error(VP_ERR_DTYPE, "vp_kick2d: unknown dtype");
    VP_CHECK(f_in && f_out && Ex && Ey, "vp_kick2d: null pointer");
    VP_CHECK(f_in != f_out, "vp_kick2d: f_out must not alias f_in");
    VP_CHECK(n_planes > 0 && nvx > 0 && nvy > 0, "vp_kick2d: bad size");
    VP_CHECK(dvx != 0.0 && dvy != 0.0, "vp_kick2d: zero velocity spacing");
    VP_CHECK(!moments || (vx && vy), "vp_kick2d: moments need vx and vy");
    const int rc = run_kick2d(dtype, f_in, f_out, n_planes, nvx, nvy, Ex, Ey, dt, dvx, dvy, window, vx, vy, moments,
                              EQ_NONE, S(stream));
    if (rc == VP_ERR_UNSUPPORTED) return set_error(rc, "vp_kick2d: nvy too wide for one warp per plane row");
    return rc;
}

int vp_advect_gather(const void* f_in, void* f_out, int dtype, int64_t n_outer, int64_t n_line, int64_t n_inner,
                     const void* vel, int64_t vs_outer, int64_t vs_line, int64_t vs_inner, double dt, double dx,
                     int periodic, void* stream) {
    if (!dtype_ok(dtype)) return set_error(VP_ERR_DTYPE, "vp_advect_gather: unknown dtype");
    VP_CHECK(f_in && f_out && vel, "vp_advect_gather: null pointer");
    VP_CHECK(f_in != f_out, "vp_advect_gather: f_out must not alias f_in");
    VP_CHECK(n_outer > 0 && n_line > 0 && n_inner > 0, "vp_advect_gather: bad size");
    VP_CHECK(dx != 0.0, "vp_advect_gather: dx == 0");
    return run_gather(dtype, f_in, f_out, n_outer, n_line, n_inner, vel, vs_outer, vs_line, vs_inner, dt, dx,
                      periodic, S(stream));
}

int vp_rho(const void* f, int dtype, int64_t n_points, int64_t n_v, double dvx, double dvy, void* rho,
           int out_dtype, void* stream) {
    if (!dtype_ok(dtype)) return set_error(VP_ERR_DTYPE, "vp_rho: unknown dtype");
    VP_CHECK(f && rho, "vp_rho: null pointer");
    VP_CHECK(n_points > 0 && n_v > 0, "vp_rho: bad size");
    VP_CHECK(out_dtype == VP_F32 || out_dtype == VP_F64, "vp_rho: out_dtype must be float32 or float64");
    return run_rho(dtype, f, n_points, n_v, dvx, dvy, rho, out_dtype, S(stream));
}

int vp_lagrange_interp(const void* alpha, const void* vals, void* out, int dtype, int64_t n, void* stream) {
    VP_CHECK(n >= 0, "vp_lagrange_interp: negative size");
    VP_CHECK(n == 0 || (alpha && vals && out), "vp_lagrange_interp: null pointer");
    return run_lagrange(dtype, alpha, vals, out, n, 0, S(stream));
}

int vp_lagrange_weights(const void* alpha, void* weights, int dtype, int64_t n, void* stream) {
    VP_CHECK(n >= 0, "vp_lagrange_weights: negative size");
    VP_CHECK(n == 0 || (alpha && weights), "vp_lagrange_weights: null pointer");
    return run_lagrange(dtype, alpha, nullptr, weights, n, 1, S(stream));
}

int vp_init_product(const double* space, const double* vel, void* f, int dtype, int64_t n_points, int64_t n_v,
                    void* stream) {
    if (!dtype_ok(dtype)) return set_error(VP_ERR_DTYPE, "vp_init_product: unknown dtype");
    VP_CHECK(n_points >= 0 && n_v >= 0, "vp_init_product: negative size");
    if (n_points == 0 || n_v == 0) return VP_OK;
    VP_CHECK(space && vel && f, "vp_init_product: null pointer");
    return run_init_product(dtype, space, vel, f, n_points, n_v, S(stream));
}

size_t vp_poisson2d_workspace_bytes(int64_t nx, int64_t ny) { return poisson2d_ws_bytes(nx, ny); }

int vp_poisson2d(const double* rho, int64_t nx, int64_t ny, const double* kx, const double* ky,
                 const double* inv_ksq, double dx, double dy, double* ex, double* ey, double* drho, double* phi,
                 double* energy, void* workspace, size_t workspace_bytes, void* stream) {
    VP_CHECK(rho && kx && ky && inv_ksq && ex && ey, "vp_poisson2d: null pointer");
    VP_CHECK(nx > 0 && ny > 0 && nx <= 4096 && ny <= 4096, "vp_poisson2d: sizes must be in [1, 4096]");
    if (!poisson2d_fits(nx, ny))
        return set_error(VP_ERR_UNSUPPORTED, "vp_poisson2d: the transforms need more shared memory than a block "
                                             "has (nx above about 1800 or ny above about 3600)");
    if (!workspace || workspace_bytes < poisson2d_ws_bytes(nx, ny))
        return set_error(VP_ERR_WORKSPACE, "vp_poisson2d: workspace too small");
    Pois2dWsView v{};
    int rc = run_poisson2d(rho, nx, ny, kx, ky, inv_ksq, ex, ey, drho, phi, workspace, &v, S(stream));
    if (rc) return rc;
    if (!energy) return VP_OK;
    return run_diag_finalize(v, nullptr, 0, dx * dy, 0.5 * dx * dy, 0.0, 0.0, 0.0, energy, nullptr, S(stream));
}

int vp_poisson2d_static(const double* rho, int64_t nx, int64_t ny, const double* kx, const double* ky,
                        const double* inv_ksq, double dx, double dy, double* ex, double* ey, double* drho,
                        double* phi, double* energy, void* stream) {
    VP_CHECK(rho && kx && ky && inv_ksq && ex && ey, "vp_poisson2d_static: null pointer");
    VP_CHECK(nx > 0 && ny > 0, "vp_poisson2d_static: sizes must be positive");
    if (nx > VP_POISSON2D_STATIC_MAX_N || ny > VP_POISSON2D_STATIC_MAX_N)
        return set_error(VP_ERR_UNSUPPORTED, "vp_poisson2d_static: nx and ny must be <= VP_POISSON2D_STATIC_MAX_N");
    return run_poisson2d_static(rho, nx, ny, kx, ky, inv_ksq, dx, dy, ex, ey, drho, phi, energy, S(stream));
}

size_t vp_poisson1d_workspace_bytes(int64_t nx) { return poisson1d_ws_bytes(nx); }

int vp_poisson1d(const double* n, int64_t nx, const double* inv_kx, const double* inv_kx_sq, double dx, double* e,
                 double* rho, double* phi, double* energy, void* workspace, size_t workspace_bytes, void* stream) {
    VP_CHECK(n && inv_kx && inv_kx_sq && e, "vp_poisson1d: null pointer");
    VP_CHECK(nx > 0, "vp_poisson1d: bad size");
    if (!workspace || workspace_bytes < poisson1d_ws_bytes(nx))
        return set_error(VP_ERR_WORKSPACE, "vp_poisson1d: workspace too small");
    double* parts = static_cast<double*>(workspace);
    int rc = run_poisson1d(n, nx, inv_kx, inv_kx_sq, e, rho, phi, parts, S(stream));
    if (rc || !energy) return rc;
    Pois2dWsView v{parts, parts + 1, nullptr, 1};
    return run_diag_finalize(v, nullptr, 0, dx, 0.5 * dx, 0.0, 0.0, 0.0, energy, nullptr, S(stream));
}

size_t vp_step2d_workspace_bytes(int64_t nx, int64_t ny, int64_t nvx, int64_t nvy) {
    return step2d_layout(nx, ny, nvx, nvy, nullptr, nullptr);
}

// the position drifts go through the fused (x, y) plane passes
static bool step2d_planar(const vp_step2d_desc* d) {
    return !d->sweeps_only && plane_fits(d->dtype, d->nx, d->ny, d->nvx, d->nvy, d->f_in) &&
           plane_fits(d->dtype, d->nx, d->ny, d->nvx, d->nvy, d->f_out) &&
           plane_fits(d->dtype, d->nx, d->ny, d->nvx, d->nvy, d->f_tmp);
}

int vp_step2d_passes(const vp_step2d_desc* d, int32_t* plane_fused) {
    VP_CHECK(d, "vp_step2d_passes: null descriptor");
    if (!dtype_ok(d->dtype)) return set_error(VP_ERR_DTYPE, "vp_step2d_passes: unknown dtype");
    const bool phys = d->physics_mode != 0;
    const bool fused = kick2d_fits(d->dtype, d->nvy, d->f_in, d->f_out, d->f_tmp);
    const bool planar = step2d_planar(d);
    if (plane_fused) *plane_fused = planar ? 1 : 0;
    return (phys ? (fused ? 1 : 2) : 0) + (planar ? 2 : 4);
}

int vp_step2d(const vp_step2d_desc* d, void* stream) {
    VP_CHECK(d, "vp_step2d: null descriptor");
    if (!dtype_ok(d->dtype)) return set_error(VP_ERR_DTYPE, "vp_step2d: unknown dtype");
    VP_CHECK(d->f_in && d->f_out && d->f_tmp, "vp_step2d: null f buffer");
    VP_CHECK(d->f_in != d->f_out && d->f_in != d->f_tmp && d->f_out != d->f_tmp,
             "vp_step2d: f_in, f_out and f_tmp must be distinct");
    VP_CHECK(d->nx > 0 && d->ny > 0 && d->nvx > 1 && d->nvy > 1, "vp_step2d: bad size");
    VP_CHECK(d->nx < (1 << 30) && d->ny < (1 << 30) && d->nvx < (1 << 30) && d->nvy < (1 << 30),
             "vp_step2d: axis too long");
    VP_CHECK(d->shift_x && d->W_x && d->shift_y && d->W_y, "vp_step2d: null drift table");
    VP_CHECK(!d->physics_mode || (d->kx && d->ky && d->inv_ksq), "vp_step2d: null spectral arrays");
    VP_CHECK(!d->diagnostics || !d->diag || (d->vx && d->vy), "vp_step2d: diagnostics need vx and vy");
    VP_CHECK(d->dvx != 0.0 && d->dvy != 0.0, "vp_step2d: zero velocity spacing");
    if (d->physics_mode && !poisson2d_fits(d->nx, d->ny))
        return set_error(VP_ERR_UNSUPPORTED, "vp_step2d: the field solve's transforms need nx below about 1800 "
                                             "and ny below about 3600 (shared memory)");
    const size_t need = step2d_layout(d->nx, d->ny, d->nvx, d->nvy, nullptr, nullptr);
    if (!d->workspace || d->workspace_bytes < need) return set_error(VP_ERR_WORKSPACE, "vp_step2d: workspace too small");
    Step2dWs w;
    step2d_layout(d->nx, d->ny, d->nvx, d->nvy, static_cast<char*>(d->workspace), &w);
    cudaStream_t st = S(stream);
    const int64_t nx = d->nx, ny = d->ny, nvx = d->nvx, nvy = d->nvy;
    const bool phys = d->physics_mode != 0;
    const bool want_diag = d->diagnostics && d->diag;
    const bool want_rho = phys || want_diag;
    // both kicks in one pass when a plane row fits one warp, else two sweeps
    const bool fused = kick2d_fits(d->dtype, nvy, d->f_in, d->f_out, d->f_tmp);
    const bool eq_on = d->eq_vx || d->eq_vy;
    VP_CHECK(!eq_on || (d->eq_vx && d->eq_vy), "vp_step2d: the equilibrium split needs eq_vx and eq_vy");
    if (eq_on && phys && !fused)
        return set_error(VP_ERR_UNSUPPORTED, "vp_step2d: the equilibrium split needs the fused kick (nvy <= 128)");
    const EqSplit eqs{d->eq_vx, d->eq_vy, nvx, nvy};
    const EqSplit* EQ = eq_on ? &eqs : EQ_NONE;
    // The position drifts in pairs through the (x, y) plane when the layout
    // allows (one pass over f each, intermediate on chip, bit-identical);
    // otherwise one sweep per axis. The fused passes are timed under the x
    // phases, the y phases then stay empty.
    const bool planar = step2d_planar(d);
    const int n_sweeps = (phys ? (fused ? 3 : 4) : 2) + (planar ? 0 : 2);
    int i = 0;
    auto dst_of = [&](int k) -> void* { return ((n_sweeps - 1 - k) % 2 == 0) ? d->f_out : d->f_tmp; };
    const void* src = d->f_in;
    int rc;
    Marks mk{d->events, st};
    void* dst;
    if (planar) {
        // x then y drift (dt/2 each), with the density when needed
        if ((rc = mk.begin(VP_PHASE_DRIFT_X1))) return rc;
        dst = dst_of(i++);
        int tiles = 0;
        rc = run_plane(d->dtype, true, src, dst, nx, ny, nvx, nvy, 0, nx, d->shift_x, d->W_x, d->shift_y, d->W_y,
                       want_rho ? w.part : nullptr, &tiles, EQ, d->status, d->test_stall, st);
        if (rc || (rc = mk.end(VP_PHASE_DRIFT_X1))) return rc;
        // the density partials' sum, timed as its own phase
        if ((rc = mk.begin(VP_PHASE_DRIFT_Y1))) return rc;
        if (want_rho &&
            (rc = run_rho_finalize(w.part, nx, ny, tiles, d->dvx * d->dvy, eq_on ? d->eq_moment : 0.0, w.rho, st)))
            return rc;
        if ((rc = mk.end(VP_PHASE_DRIFT_Y1))) return rc;
        src = dst;
    } else {
    // x drift (dt/2)
    if ((rc = mk.begin(VP_PHASE_DRIFT_X1))) return rc;
    dst = dst_of(i++);
    rc = run_strided(d->dtype, src, dst, 1, nx, ny * nvx * nvy, false, nvy, nvx, d->shift_spread_x, d->shift_x, d->W_x, nullptr, 0, 1,
                     0.0, 1.0, -1, nullptr, nullptr, EQ, st);
    if (rc || (rc = mk.end(VP_PHASE_DRIFT_X1))) return rc;
    src = dst;
    // y drift (dt/2), fused with rho when needed
    if ((rc = mk.begin(VP_PHASE_DRIFT_Y1))) return rc;
    dst = dst_of(i++);
    if (want_rho) {
        int tiles = 0;
        rc = run_strided(d->dtype, src, dst, nx, ny, nvx * nvy, false, 1, nvy, d->shift_spread_y, d->shift_y, d->W_y, nullptr, 0, 1, 0.0,
                         1.0, -1, w.part, &tiles, EQ, st);
        if (rc) return rc;
        rc = run_rho_finalize(w.part, nx, ny, tiles, d->dvx * d->dvy, eq_on ? d->eq_moment : 0.0, w.rho, st);
    } else {
        rc = run_strided(d->dtype, src, dst, nx, ny, nvx * nvy, false, 1, nvy, d->shift_spread_y, d->shift_y, d->W_y, nullptr, 0, 1, 0.0,
                         1.0, -1, nullptr, nullptr, EQ, st);
    }
    if (rc || (rc = mk.end(VP_PHASE_DRIFT_Y1))) return rc;
    src = dst;
    }
    Pois2dWsView pv{};
    double* moments = nullptr;
    if ((rc = mk.begin(VP_PHASE_FIELD))) return rc;
    if (phys) {
        double* ex = d->ex ? d->ex : w.ex;
        double* ey = d->ey ? d->ey : w.ey;
        rc = run_poisson2d(w.rho, nx, ny, d->kx, d->ky, d->inv_ksq, ex, ey, d->drho, d->phi, w.pois, &pv, st);
        if (rc || (rc = mk.end(VP_PHASE_FIELD)) || (rc = mk.begin(VP_PHASE_KICK))) return rc;
        if (fused) {
            moments = (want_diag && d->diagnostics >= 2) ? w.moments : nullptr;
            dst = dst_of(i++);
            rc = run_kick2d(d->dtype, src, dst, nx * ny, nvx, nvy, ex, ey, d->dt, d->dvx, d->dvy, d->window, d->vx,
                            d->vy, moments, EQ, st);
            if (rc) return rc;
            src = dst;
        } else {
            dst = dst_of(i++);
            rc = run_strided(d->dtype, src, dst, nx * ny, nvx, nvy, true, 1, 1, -1, nullptr, nullptr, ex, 1, 1, d->dt,
                             d->dvx, d->window, nullptr, nullptr, EQ_NONE, st);
            if (rc) return rc;
            src = dst;
            dst = dst_of(i++);
            rc = run_kick_contig(d->dtype, src, dst, nx * ny * nvx, nvy, ey, 1, nvx, d->dt, d->dvy, d->window,
                                 EQ_NONE, st);
            if (rc) return rc;
            src = dst;
        }
        if ((rc = mk.end(VP_PHASE_KICK))) return rc;
    } else {
        if (d->drho && cudaMemsetAsync(d->drho, 0, nx * ny * sizeof(double), st) != cudaSuccess)
            return set_cuda_error("cudaMemsetAsync(drho)");
        if (d->phi && cudaMemsetAsync(d->phi, 0, nx * ny * sizeof(double), st) != cudaSuccess)
            return set_cuda_error("cudaMemsetAsync(phi)");
        if (d->ex && cudaMemsetAsync(d->ex, 0, nx * ny * sizeof(double), st) != cudaSuccess)
            return set_cuda_error("cudaMemsetAsync(ex)");
        if (d->ey && cudaMemsetAsync(d->ey, 0, nx * ny * sizeof(double), st) != cudaSuccess)
            return set_cuda_error("cudaMemsetAsync(ey)");
        if ((rc = mk.end(VP_PHASE_FIELD)) || (rc = mk.begin(VP_PHASE_KICK)) || (rc = mk.end(VP_PHASE_KICK)))
            return rc;
    }
    if (planar) {
        // y then x drift (dt/2 each)
        if ((rc = mk.begin(VP_PHASE_DRIFT_Y2)) || (rc = mk.end(VP_PHASE_DRIFT_Y2))) return rc;
        if ((rc = mk.begin(VP_PHASE_DRIFT_X2))) return rc;
        dst = dst_of(i++);
        rc = run_plane(d->dtype, false, src, dst, nx, ny, nvx, nvy, 0, nx, d->shift_x, d->W_x, d->shift_y, d->W_y,
                       nullptr, nullptr, EQ, d->status, d->test_stall, st);
        if (rc || (rc = mk.end(VP_PHASE_DRIFT_X2)) || (rc = mk.begin(VP_PHASE_DIAG))) return rc;
    } else {
    // y drift (dt/2)
    if ((rc = mk.begin(VP_PHASE_DRIFT_Y2))) return rc;
    dst = dst_of(i++);
    rc = run_strided(d->dtype, src, dst, nx, ny, nvx * nvy, false, 1, nvy, d->shift_spread_y, d->shift_y, d->W_y, nullptr, 0, 1, 0.0,
                     1.0, -1, nullptr, nullptr, EQ, st);
    if (rc || (rc = mk.end(VP_PHASE_DRIFT_Y2))) return rc;
    src = dst;
    // x drift (dt/2)
    if ((rc = mk.begin(VP_PHASE_DRIFT_X2))) return rc;
    dst = dst_of(i++);
    rc = run_strided(d->dtype, src, dst, 1, nx, ny * nvx * nvy, false, nvy, nvx, d->shift_spread_x, d->shift_x, d->W_x, nullptr, 0, 1,
                     0.0, 1.0, -1, nullptr, nullptr, EQ, st);
    if (rc || (rc = mk.end(VP_PHASE_DRIFT_X2)) || (rc = mk.begin(VP_PHASE_DIAG))) return rc;
    }
    if (want_diag) {
        const double dV = d->dx * d->dy * d->dvx * d->dvy;
        if (!phys) {
            // mass straight from rho: sum rho * dx * dy (rho already carries dvx*dvy)
            Pois2dWsView mv{w.rho, nullptr, nullptr, (int)(nx * ny)};
            rc = run_diag_finalize(mv, nullptr, 0, d->dx * d->dy, 0.0, dV, 0.0, 0.0, nullptr, d->diag, st, d->status);
        } else {
            // without the fused kick the L2 / kinetic moments are not computed (NaN)
            rc = run_diag_finalize(pv, moments, nx * ny, d->dx * d->dy, 0.5 * d->dx * d->dy, dV, d->dt / d->dvx,
                                   d->dt / d->dvy, nullptr, d->diag, st, d->status);
        }
        if (rc) return rc;
    }
    return mk.end(VP_PHASE_DIAG);
}

size_t vp_step1d_workspace_bytes(int64_t nx, int64_t nv) { return step1d_layout(nx, nv, nullptr, nullptr); }

int vp_step1d(const vp_step1d_desc* d, void* stream) {
    VP_CHECK(d, "vp_step1d: null descriptor");
    if (!dtype_ok(d->dtype)) return set_error(VP_ERR_DTYPE, "vp_step1d: unknown dtype");
    VP_CHECK(d->f_in && d->f_out && d->f_tmp, "vp_step1d: null f buffer");
    VP_CHECK(d->f_in != d->f_out && d->f_in != d->f_tmp && d->f_out != d->f_tmp,
             "vp_step1d: f_in, f_out and f_tmp must be distinct");
    VP_CHECK(d->nx > 0 && d->nv > 1 && d->nx < (1 << 30) && d->nv < (1 << 30), "vp_step1d: bad size");
    VP_CHECK(d->shift && d->W, "vp_step1d: null drift table");
    VP_CHECK(!d->physics_mode || (d->inv_kx && d->inv_kx_sq), "vp_step1d: null spectral arrays");
    VP_CHECK(d->dv != 0.0, "vp_step1d: dv == 0");
    const size_t need = step1d_layout(d->nx, d->nv, nullptr, nullptr);
    if (!d->workspace || d->workspace_bytes < need) return set_error(VP_ERR_WORKSPACE, "vp_step1d: workspace too small");
    Step1dWs w;
    step1d_layout(d->nx, d->nv, static_cast<char*>(d->workspace), &w);
    cudaStream_t st = S(stream);
    const int64_t nx = d->nx, nv = d->nv;
    const bool phys = d->physics_mode != 0;
    const bool want_diag = d->diagnostics && d->diag;
    const int n_sweeps = phys ? 3 : 2;
    const bool eq_on = d->eq_v != nullptr;
    const EqSplit eqs{nullptr, d->eq_v, 1, nv};
    const EqSplit* EQ = eq_on ? &eqs : EQ_NONE;
    int i = 0;
    auto dst_of = [&](int k) -> void* { return ((n_sweeps - 1 - k) % 2 == 0) ? d->f_out : d->f_tmp; };
    const void* src = d->f_in;
    int rc;
    Marks mk{d->events, st};
    if ((rc = mk.begin(VP_PHASE_DRIFT_X1))) return rc;
    void* dst = dst_of(i++);
    // power-of-two nx: the field solve also writes the diagnostics (summing
    // the density partials there instead of in k_rho_finalize was slower:
    // one CTA would wait on all their loads)
    const bool fused_field = phys && poisson1d_fuses(nx);
    if (phys || want_diag) {
        int tiles = 0;
        rc = run_strided(d->dtype, src, dst, 1, nx, nv, false, 1, nv, d->shift_spread, d->shift, d->W, nullptr, 0, 1, 0.0, 1.0, -1,
                         w.part, &tiles, EQ, st);
        if (rc) return rc;
        rc = run_rho_finalize(w.part, 1, nx, tiles, d->dv, eq_on ? d->eq_moment : 0.0, w.n, st);
    } else {
        rc = run_strided(d->dtype, src, dst, 1, nx, nv, false, 1, nv, d->shift_spread, d->shift, d->W, nullptr, 0, 1, 0.0, 1.0, -1,
                         nullptr, nullptr, EQ, st);
    }
    if (rc || (rc = mk.end(VP_PHASE_DRIFT_X1))) return rc;
    if ((rc = mk.begin(VP_PHASE_DRIFT_Y1)) || (rc = mk.end(VP_PHASE_DRIFT_Y1))) return rc;
    src = dst;
    if ((rc = mk.begin(VP_PHASE_FIELD))) return rc;
    if (phys) {
        double* e = d->e ? d->e : w.e;
        if (fused_field)
            rc = run_poisson1d_fused(w.n, nullptr, 0, 0.0, 0.0, nx, d->inv_kx, d->inv_kx_sq, e, d->rho, d->phi,
                                     w.parts, want_diag ? d->diag : nullptr, d->dx, 0.5 * d->dx, d->dt / d->dv,
                                     d->status, st);
        else
            rc = run_poisson1d(w.n, nx, d->inv_kx, d->inv_kx_sq, e, d->rho, d->phi, w.parts, st);
        if (rc || (rc = mk.end(VP_PHASE_FIELD)) || (rc = mk.begin(VP_PHASE_KICK))) return rc;
        dst = dst_of(i++);
        rc = run_kick_contig(d->dtype, src, dst, nx, nv, e, 1, 1, d->dt, d->dv, d->window, EQ, st);
        if (rc || (rc = mk.end(VP_PHASE_KICK))) return rc;
        src = dst;
    } else {
        if (d->rho && cudaMemsetAsync(d->rho, 0, nx * sizeof(double), st) != cudaSuccess)
            return set_cuda_error("cudaMemsetAsync(rho)");
        if (d->phi && cudaMemsetAsync(d->phi, 0, nx * sizeof(double), st) != cudaSuccess)
            return set_cuda_error("cudaMemsetAsync(phi)");
        if (d->e && cudaMemsetAsync(d->e, 0, nx * sizeof(double), st) != cudaSuccess)
            return set_cuda_error("cudaMemsetAsync(e)");
        if ((rc = mk.end(VP_PHASE_FIELD)) || (rc = mk.begin(VP_PHASE_KICK)) || (rc = mk.end(VP_PHASE_KICK)))
            return rc;
    }
    if ((rc = mk.begin(VP_PHASE_DRIFT_Y2)) || (rc = mk.end(VP_PHASE_DRIFT_Y2))) return rc;
    if ((rc = mk.begin(VP_PHASE_DRIFT_X2))) return rc;
    dst = dst_of(i++);
    rc = run_strided(d->dtype, src, dst, 1, nx, nv, false, 1, nv, d->shift_spread, d->shift, d->W, nullptr, 0, 1, 0.0, 1.0, -1, nullptr,
                     nullptr, EQ, st);
    if (rc || (rc = mk.end(VP_PHASE_DRIFT_X2)) || (rc = mk.begin(VP_PHASE_DIAG))) return rc;
    if (want_diag && !fused_field) {
        if (phys) {
            // parts = {sum n, sum e^2, max|e|, 0}: the emax pair reads (max|e|, 0)
            Pois2dWsView v{w.parts, w.parts + 1, w.parts + 2, 1};
            rc = run_diag_finalize(v, nullptr, 0, d->dx, 0.5 * d->dx, 0.0, d->dt / d->dv, 0.0, nullptr, d->diag, st,
                                   d->status);
        } else {
            Pois2dWsView v{w.n, nullptr, nullptr, (int)nx};
            rc = run_diag_finalize(v, nullptr, 0, d->dx, 0.0, 0.0, 0.0, 0.0, nullptr, d->diag, st, d->status);
        }
        if (rc) return rc;
    }
    return mk.end(VP_PHASE_DIAG);
}

}  // extern "C"
