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

struct Pois2dWsView {
    const double* mass_part;
    const double* we_part;
    const double* emax_part;
    int n_lines;
};

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
int run_kick_contig(int dtype, const void* in, void* out, int64_t n_rows, int64_t n, const void* E, int e_f64,
                    int64_t e_div, double dt, double dv, int window, const EqSplit* eq, cudaStream_t st);
int run_gather(int dtype, const void* in, void* out, int64_t n_outer, int64_t n, int64_t n_inner, const void* vel,
               int64_t vso, int64_t vsl, int64_t vsc, double dt, double dx, int periodic, cudaStream_t st);
int run_rho(int dtype, const void* f, int64_t n_points, int64_t n_v, double dvx, double dvy, void* rho,
            int out_dtype, cudaStream_t st);

// poisson.cu
size_t poisson2d_ws_bytes(int64_t nx, int64_t ny);
int run_poisson2d(const double* rho, int64_t nx, int64_t ny, const double* kx, const double* ky,
                  const double* inv_ksq, double* ex, double* ey, double* drho, double* phi, void* ws,
                  Pois2dWsView* view, cudaStream_t st);
int run_diag_finalize(const Pois2dWsView& pv, const double* moments, int64_t n_mom, double mass_scale,
                      double we_scale, double dv_scale, double shift_x, double shift_y, double* energy,
                      double* diag, cudaStream_t st);
int run_poisson2d_static(const double* rho, int64_t nx, int64_t ny, const double* kx, const double* ky,
                         const double* inv_ksq, double dx, double dy, double* ex, double* ey, double* drho,
                         double* phi, double* energy, cudaStream_t st);
size_t poisson1d_ws_bytes(int64_t nx);
int run_poisson1d(const double* n, int64_t nx, const double* inv_kx, const double* inv_kx_sq, double* e,
                  double* rho, double* phi, double* parts, cudaStream_t st);

}  // namespace vp
