// Host-side plumbing shared by the kernel files: error state, device
// properties, occupancy, and the internal launchers behind the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace vp {

int set_error(int code, const char* msg);
int set_cuda_error(const char* what);
int check_launch(const char* what);
int sm_count();
int occupancy_raw(const void* kern, int block, size_t smem);

template <typename K>
inline int occupancy(K kern, int block, size_t smem) {
    return occupancy_raw(reinterpret_cast<const void*>(kern), block, smem);
}

// Separable equilibrium of the split storage f = feq + g:
// feq(ivx, ivy) = A[ivx] * B[ivy] (A == NULL: factor 1, the 1D1V case).
struct EqSplit {
    const double* A;
    const double* B;
    int64_t nvx, nvy;
};
#define EQ_NONE static_cast<const EqSplit*>(nullptr)

// ---------------------------------------------------------------------------
// Kernel argument blocks (plain data, also stored in device-resident tables
// by the batched step)
// ---------------------------------------------------------------------------
struct StridedArgs {
    const void* in;
    void* out;
    int64_t n_outer;
    int n_line;
    int64_t n_inner;
    int64_t ncg;    // column groups (of VEC elements) per outer row
    int tiles;      // ceil(ncg / blockDim.x)
    int seg;        // outputs per line segment
    int nseg;       // segments per line
    int64_t items;  // n_outer * tiles * nseg
    // drift table
    int64_t sel_div;
    int sel_mod;
    const int32_t* shift;
    const void* W;
    // kick field
    const void* E;
    int e_f64;
    int64_t e_div;
    double dt, dv;
    int window;
    // fused moment partials [n_outer][tiles][n_line]
    double* part;
    // equilibrium split (drifts): column c has feq = eqA[(c / eq_nvy) % eq_nvx] * eqB[c % eq_nvy]
    const double* eqA;  // NULL: factor 1
    const double* eqB;  // NULL: no split
    int64_t eq_nvx, eq_nvy;
};

struct Kick2dArgs {
    const void* in;
    void* out;
    int64_t n_planes;
    int nvx, nvy;
    int team;   // lanes per plane (power of two, <= 32)
    int groups; // nvy / VEC
    const double* Ex;
    const double* Ey;
    double dt, dvx, dvy;
    int window;
    const double* vx;
    const double* vy;
    double* moments;
    // equilibrium split: feq = eqA[ivx] * eqB[ivy] (both NULL: off)
    const double* eqA;
    const double* eqB;
};

// Poisson solve of one run (workspace pointers from the 2D layout).
struct Pois2dRun {
    const double* rho;
    int nx, ny;
    const double *kx, *ky, *inv_ksq;
    double *drho, *phi, *ex, *ey;
    double2 *R, *Zp, *Zx, *Zy;
    double *mass_part, *we_part, *emax_part;
};

// rho[o*n_line + l] = scale * sum_t part[o][t][l] + offset for one run.
struct RhoFinRun {
    const double* part;
    int64_t n_outer;
    int n_line, tiles;
    double scale, offset;
    double* rho;
};

struct DiagArgs {
    const double* mass_part;  // [n_mass]
    int n_mass;
    const double* we_part;  // [n_we]
    int n_we;
    const double* emax_part;  // [n_emax][2]
    int n_emax;
    const double* moments;  // [n_mom][4]
    int64_t n_mom;
    double mass_scale, we_scale, dv_scale;  // dx*dy, 0.5*dx*dy, dV
    double shift_x, shift_y;                // dt/dvx, dt/dvy
    double* energy;                         // optional [2]: {W_E, mass}
    double* diag;                           // optional [VP_DIAG_COUNT]
    int64_t slot_stride;                    // batched form: doubles between history slots
    int* status;                            // optional: VP_STATUS_NONFINITE ORed in
};

struct Pois2dWsView {
    const double* mass_part;
    const double* we_part;
    const double* emax_part;
    int n_lines;
};

// Workspace of one 2D2V step (capi.cu): rho partials, rho, fields, kick
// moments, Poisson scratch.
struct Step2dWs {
    double *part, *rho, *ex, *ey, *moments;
    void* pois;
};
size_t step2d_layout(int64_t nx, int64_t ny, int64_t nvx, int64_t nvy, char* base, Step2dWs* w);

// sweeps.cu
int run_strided(int dtype, const void* in, void* out, int64_t n_outer, int64_t n_line, int64_t n_inner, bool kick,
                int64_t sel_div, int64_t sel_mod, int spread, const int32_t* shift, const void* W, const void* E, int e_f64,
                int64_t e_div, double dt, double dv, int window, double* part, int* tiles_out, const EqSplit* eq,
                cudaStream_t st);
int run_rho_finalize(const double* part, int64_t n_outer, int64_t n_line, int tiles, double scale, double offset,
                     double* rho,
                     cudaStream_t st);
int run_kick2d(int dtype, const void* in, void* out, int64_t n_planes, int64_t nvx, int64_t nvy, const double* Ex,
               const double* Ey, double dt, double dvx, double dvy, int window, const double* vx,
               const double* vy, double* moments, const EqSplit* eq, cudaStream_t st);
bool kick2d_fits(int dtype, int64_t nvy, const void* a, const void* b, const void* c);
// f[p][v] = S[p] * V[v] (FP64 product, rounded once to the storage type)
int run_init_product(int dtype, const double* S, const double* V, void* f, int64_t n_points, int64_t n_v,
                     cudaStream_t st);
// Both position drifts of f[nx][ny][nvx][nvy] in one pass (x then y, or y
// then x), with the density row sums of x-then-y into part
// ([nx][plane_part_tiles][ny], tiles returned) when part is not null. With
// eq (equilibrium split, eq->A and eq->B both set) each drift of the stored
// perturbation g adds feq * (sum of the column's weights - 1), as the
// single-axis sweeps do.
bool plane_fits(int dtype, int64_t nx, int64_t ny, int64_t nvx, int64_t nvy, const void* in);
int64_t plane_part_tiles(int64_t nvx, int64_t nvy);
// Only the output rows x_begin .. x_begin + x_count - 1 are written (their
// density partials too); the inputs wrap around nx.
int run_plane(int dtype, bool xfirst, const void* in, void* out, int64_t nx, int64_t ny, int64_t nvx, int64_t nvy,
              int64_t x_begin, int64_t x_count, const int* shift_x, const void* W_x, const int* shift_y,
              const void* W_y, double* part, int* tiles, const EqSplit* eq, int* status, int stall, cudaStream_t st);
// Batched drift pairs (runs of up to 64 rows, a multiple of 8, FP32,
// nvy % 16 == 0, aligned): one record of plane_run_bytes() per fused run and
// pass in the device table (64-byte aligned, in any order), filled on the host by
// plane_batch_run (in -> out; part: the density partials
// [nx][nvx*nvy/32][ny] of the x-first pass, or NULL); items = the run's
// items (x first: packs of groups of 32 columns; y first: groups), start[r]
// the prefix sums of the items; slab_rows the rows of one ring slab of the
// run, the launch takes the largest over its runs.
size_t plane_run_bytes();
bool plane_batch_fits(int dtype, int64_t nx, int64_t ny, int64_t nvx, int64_t nvy, const void* a, const void* b,
                      const void* c);
int plane_batch_run(void* record, bool xfirst, const void* in, void* out, int64_t nx, int64_t ny, int64_t nvx,
                    int64_t nvy, const int* shift_x, const void* W_x, const int* shift_y, const void* W_y,
                    double* part, int* status, int stall, int64_t* items, int* slab_rows);
// runs_host / start_host: the host copies of the records and prefix sums
// (the x-first pass takes the runs' tensor maps as a kernel parameter)
// records 0 .. n_full - 1 hold runs with nvy % 32 == 0 (whole 32-column TMA
// boxes), the rest runs whose groups come in half boxes of 16 (one launch each)
int launch_plane_batch(bool xfirst, bool rho, const void* runs, const void* runs_host, const int64_t* start,
                       const int64_t* start_host, int n_full, int n_runs, int64_t items, int slab_rows,
                       cudaStream_t st);
int run_kick_contig(int dtype, const void* in, void* out, int64_t n_rows, int64_t n, const void* E, int e_f64,
                    int64_t e_div, double dt, double dv, int window, const EqSplit* eq, cudaStream_t st);
int run_gather(int dtype, const void* in, void* out, int64_t n_outer, int64_t n, int64_t n_inner, const void* vel,
               int64_t vso, int64_t vsl, int64_t vsc, double dt, double dx, int periodic, cudaStream_t st);
int run_rho(int dtype, const void* f, int64_t n_points, int64_t n_v, double dvx, double dvy, void* rho,
            int out_dtype, cudaStream_t st);
int run_lagrange(int dtype, const void* alpha, const void* vals, void* out, int64_t n, int mode, cudaStream_t st);

// batched step (sweeps.cu)
int strided_batch_args(int dtype, const void* in, void* out, int64_t n_outer, int64_t n_line, int64_t n_inner,
                       int64_t sel_div, int64_t sel_mod, int spread, const int32_t* shift, const void* W,
                       double* part, int block, StridedArgs* a, int* vec, int* nt);
void strided_batch_finish(StridedArgs* a, int vec, int block);
int strided_batch_pref_vec(int dtype);
// pdl: launch as a programmatic dependent of the kernel before it on st (a
// plane pass over the batch's other runs, which must not share a buffer with
// these sweeps)
int launch_strided_batch(int dtype, int vec, int nt, bool rho, bool wrap, const StridedArgs* runs,
                         const int64_t* start, int n_runs, int block, int grid_cap, int max_line, bool pdl,
                         cudaStream_t st);
int launch_rho_finalize_batch(const RhoFinRun* runs, int n_runs, int max_outer, int max_line, cudaStream_t st);
int kick2d_batch_args(int dtype, const void* in, void* out, int64_t n_planes, int64_t nvx, int64_t nvy,
                      const double* Ex, const double* Ey, double dt, double dvx, double dvy, int window,
                      Kick2dArgs* a, int* vec);
int64_t kick2d_batch_finish(Kick2dArgs* a, int dtype, int vec, int block, int64_t* items);
int launch_kick2d_batch(int dtype, int vec, const Kick2dArgs* runs, const int64_t* start, int n_runs, int block,
                        int grid_cap, size_t smem, cudaStream_t st);

// mlp.cu (learned drift correction)
size_t mlp_smem_bytes(bool train);
int mlp_net_elems();
int mlp_grad_elems();
struct MlpSweepArgs;
int run_mlp_sweep(bool train, bool kick, const MlpSweepArgs& args, cudaStream_t st);

// poisson.cu
size_t poisson2d_ws_bytes(int64_t nx, int64_t ny);
// the 2D solve's transform kernels fit the per-block shared memory
bool poisson2d_fits(int64_t nx, int64_t ny);
int run_poisson2d(const double* rho, int64_t nx, int64_t ny, const double* kx, const double* ky,
                  const double* inv_ksq, double* ex, double* ey, double* drho, double* phi, void* ws,
                  Pois2dWsView* view, cudaStream_t st);
int run_diag_finalize(const Pois2dWsView& pv, const double* moments, int64_t n_mom, double mass_scale,
                      double we_scale, double dv_scale, double shift_x, double shift_y, double* energy,
                      double* diag, cudaStream_t st, int* status = nullptr);
int run_poisson2d_static(const double* rho, int64_t nx, int64_t ny, const double* kx, const double* ky,
                         const double* inv_ksq, double dx, double dy, double* ex, double* ey, double* drho,
                         double* phi, double* energy, cudaStream_t st);
void pois2d_run_args(const double* rho, int64_t nx, int64_t ny, const double* kx, const double* ky,
                     const double* inv_ksq, double* ex, double* ey, double* drho, double* phi, void* ws,
                     Pois2dRun* a, Pois2dWsView* view);
int launch_poisson2d_batch(const Pois2dRun* runs, int n_runs, int max_nx, int max_ny, cudaStream_t st);
int launch_diag_finalize_batch(const DiagArgs* runs, int n_runs, int slot, cudaStream_t st);
size_t poisson1d_ws_bytes(int64_t nx);
int run_poisson1d(const double* n, int64_t nx, const double* inv_kx, const double* inv_kx_sq, double* e,
                  double* rho, double* phi, double* parts, cudaStream_t st);
// The 1D solve that also writes the diagnostics (optional), its density
// given (n) or summed from per-tile partials (n null); only for
// poisson1d_fuses(nx).
bool poisson1d_fuses(int64_t nx);
int run_poisson1d_fused(const double* n, const double* part, int tiles, double scale, double offset, int64_t nx,
                        const double* inv_kx, const double* inv_kx_sq, double* e, double* rho, double* phi,
                        double* parts, double* diag, double mass_scale, double we_scale, double shift,
                        int* status, cudaStream_t st);

}  // namespace vp
