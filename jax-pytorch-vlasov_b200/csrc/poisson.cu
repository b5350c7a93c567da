// FP64 periodic Poisson solves of the Vlasov-Poisson step.
//
// 2D (compute_poisson_real, vlasov2D2V.py:488-517): three small kernels,
//   rows:    delta = rho - 1, real DFT along y      -> R[x][ky]     (ky <= Ny/2)
//   columns: DFT along x, phi_k = R_k*inv_ksq, E_k = -i k phi_k,
//            inverse DFT along x of phi_k, Ex_k, Ey_k -> Z*[x][ky]
//   rows:    complex-to-real inverse along y (imaginary parts of the DC and
//            Nyquist bins ignored, like torch.fft.irfft2) -> phi, Ex, Ey
// Each line transform is a direct DFT over a shared-memory twiddle table
// (sincospi of exact fractions), O(N) per output, any N. At 128x128 the whole
// solve is ~1 MFLOP per launch and not worth an FFT.
//
// 1D (solve_poisson_real, vlasov1D1V.py:538-572): one block. Power-of-two
// lengths use an in-shared-memory radix-2 FFT (Nx = 4096 would cost ~17
// MFLOP as a DFT); E and phi come out of ONE inverse transform of
// E_k + i*phi_k (both are real signals).
//
// Reductions (field energy, mass) use per-line partials summed in a fixed
// order by one block: results are bitwise reproducible run to run.
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "launch.h"

namespace vp {

constexpr int kPBlock = 256;

// twiddle table tw[j] = exp(+2 pi i j / n), j < n
__device__ __forceinline__ void fill_twiddles(double2* tw, int n) {
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)j / (double)n, &s, &c);
        tw[j] = make_double2(c, s);
    }
}

// Fixed-order block reductions (blockDim.x a multiple of 32, at most 1024;
// scratch >= 32 doubles): a shuffle tree in each warp, then one over the
// warps' results in warp 0. Every thread gets the result.
template <bool MAX>
__device__ double block_reduce(double v, double* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double o = __shfl_xor_sync(0xffffffffu, v, off);
        v = MAX ? fmax(v, o) : v + o;
    }
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < nw ? scratch[lane] : (MAX ? -INFINITY : 0.0);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_xor_sync(0xffffffffu, v, off);
            v = MAX ? fmax(v, o) : v + o;
        }
        if (lane == 0) scratch[0] = v;
    }
    __syncthreads();
    const double r = scratch[0];
    __syncthreads();
    return r;
}

__device__ double block_sum(double v, double* scratch) { return block_reduce<false>(v, scratch); }
__device__ double block_max(double v, double* scratch) { return block_reduce<true>(v, scratch); }

// ---- 2D ----------------------------------------------------------------------
// The three transforms are direct DFTs over shared-memory twiddle tables
// (any size). Each output's sum is cut into H = max(1, threads / outputs)
// consecutive slices so that every thread of the block works; the slices'
// partial sums are added in slice order (a fixed order).
__host__ __device__ constexpr int p2_slices(int outputs, int threads) {
    return outputs >= threads ? 1 : threads / outputs;
}
__host__ __device__ constexpr size_t p2_parts(int outputs, int threads) {
    return (size_t)(outputs > threads ? outputs : threads);  // >= outputs * slices
}
__host__ __device__ constexpr size_t p2_fwd_smem(int ny) {
    return (size_t)ny * sizeof(double2) + (size_t)(ny + 1) * sizeof(double) + kPBlock * sizeof(double) +
           p2_parts(ny / 2 + 1, kPBlock) * sizeof(double2);
}
__host__ __device__ constexpr size_t p2_cols_smem(int nx) {
    return 5 * (size_t)nx * sizeof(double2) + 3 * p2_parts(nx, kPBlock) * sizeof(double2);
}
__host__ __device__ constexpr size_t p2_inv_smem(int ny) {
    return (size_t)ny * sizeof(double2) + 3 * (size_t)(ny / 2 + 1) * sizeof(double2) + kPBlock * sizeof(double) +
           3 * p2_parts(ny, kPBlock) * sizeof(double);
}

// the three transform kernels' shared memory against the sm_100 opt-in limit
// of 227 KB per block (the column transform's grows as 128 nx bytes, the
// inverse rows' as 64 ny: nx up to about 1800, ny up to about 3600)
constexpr size_t kSmemOptin = 232448;
bool poisson2d_fits(int64_t nx, int64_t ny) {
    if (nx <= 0 || ny <= 0 || nx > 4096 || ny > 4096) return false;
    return p2_fwd_smem((int)ny) <= kSmemOptin && p2_cols_smem((int)nx) <= kSmemOptin &&
           p2_inv_smem((int)ny) <= kSmemOptin;
}

// ---- 2D: rows, forward ------------------------------------------------------
__device__ __forceinline__ void p2_rows_fwd(const double* __restrict__ rho, int nx, int ny, double* __restrict__ drho,
                                            double2* __restrict__ R, double* __restrict__ mass_part, const int ix,
                                            unsigned char* smem_raw) {
    double2* tw = reinterpret_cast<double2*>(smem_raw);
    double* row = reinterpret_cast<double*>(tw + ny);
    double* scratch = row + ny + (ny & 1);  // even: part stays 16-byte aligned
    double2* part = reinterpret_cast<double2*>(scratch + kPBlock);
    const int nyh = ny / 2 + 1;
    fill_twiddles(tw, ny);
    double m = 0.0;
    for (int iy = threadIdx.x; iy < ny; iy += blockDim.x) {
        const double v = rho[(int64_t)ix * ny + iy];
        const double d = v - 1.0;
        row[iy] = d;
        if (drho) drho[(int64_t)ix * ny + iy] = d;
        m += v;
    }
    m = block_sum(m, scratch);  // its barriers also publish row and tw
    if (threadIdx.x == 0 && mass_part) mass_part[ix] = m;
    const int H = p2_slices(nyh, blockDim.x);
    for (int t = threadIdx.x; t < nyh * H; t += blockDim.x) {
        const int ky = t % nyh, h = t / nyh;
        const int i0 = h * ny / H, i1 = (h + 1) * ny / H;
        double re = 0.0, im = 0.0;
        int idx = (int)(((int64_t)ky * i0) % ny);
        for (int iy = i0; iy < i1; ++iy) {
            const double2 w = tw[idx];
            re = fma(row[iy], w.x, re);
            im = fma(-row[iy], w.y, im);
            idx += ky;
            if (idx >= ny) idx -= ny;
        }
        part[t] = make_double2(re, im);
    }
    __syncthreads();
    for (int ky = threadIdx.x; ky < nyh; ky += blockDim.x) {
        double2 acc = part[ky];
        for (int h = 1; h < H; ++h) {
            const double2 q = part[h * nyh + ky];
            acc.x += q.x;
            acc.y += q.y;
        }
        R[(int64_t)ix * nyh + ky] = acc;
    }
}

__global__ void __launch_bounds__(kPBlock) k_p2_rows_fwd(const double* __restrict__ rho, int nx, int ny,
                                                       double* __restrict__ drho, double2* __restrict__ R,
                                                       double* __restrict__ mass_part) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    p2_rows_fwd(rho, nx, ny, drho, R, mass_part, blockIdx.x, smem_raw);
}

// ---- 2D: columns ------------------------------------------------------------
__device__ __forceinline__ void p2_cols(const double2* __restrict__ R, int nx, int ny, const double* __restrict__ kx,
                                        const double* __restrict__ ky, const double* __restrict__ inv_ksq,
                                        double2* __restrict__ Zp, double2* __restrict__ Zx, double2* __restrict__ Zy,
                                        const int k, unsigned char* smem_raw) {
    const int nyh = ny / 2 + 1;
    double2* tw = reinterpret_cast<double2*>(smem_raw);
    double2* col = tw + nx;
    double2* P = col + nx;
    double2* X = P + nx;
    double2* Y = X + nx;
    const size_t np = p2_parts(nx, blockDim.x);
    double2* part = Y + nx;  // [3][np]
    fill_twiddles(tw, nx);
    for (int ix = threadIdx.x; ix < nx; ix += blockDim.x) col[ix] = R[(int64_t)ix * nyh + k];
    __syncthreads();
    const int H = p2_slices(nx, blockDim.x);
    for (int t = threadIdx.x; t < nx * H; t += blockDim.x) {
        const int q = t % nx, h = t / nx;
        const int i0 = h * nx / H, i1 = (h + 1) * nx / H;
        double re = 0.0, im = 0.0;
        int idx = (int)(((int64_t)q * i0) % nx);
        for (int ix = i0; ix < i1; ++ix) {
            const double2 w = tw[idx];
            const double2 c = col[ix];
            // c * conj(w)
            re = fma(c.x, w.x, fma(c.y, w.y, re));
            im = fma(c.y, w.x, fma(-c.x, w.y, im));
            idx += q;
            if (idx >= nx) idx -= nx;
        }
        part[t] = make_double2(re, im);
    }
    __syncthreads();
    const double kyv = ky[k];
    for (int q = threadIdx.x; q < nx; q += blockDim.x) {
        double re = part[q].x, im = part[q].y;
        for (int h = 1; h < H; ++h) {
            re += part[h * nx + q].x;
            im += part[h * nx + q].y;
        }
        const double inv = inv_ksq[(int64_t)q * nyh + k];
        const double pr = re * inv, pi = im * inv;
        const double kxv = kx[q];
        P[q] = make_double2(pr, pi);
        X[q] = make_double2(pi * kxv, -pr * kxv);
        Y[q] = make_double2(pi * kyv, -pr * kyv);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nx * H; t += blockDim.x) {
        const int ix = t % nx, h = t / nx;
        const int q0 = h * nx / H, q1 = (h + 1) * nx / H;
        double pr = 0.0, pi = 0.0, xr = 0.0, xi = 0.0, yr = 0.0, yi = 0.0;
        int idx = (int)(((int64_t)ix * q0) % nx);
        for (int q = q0; q < q1; ++q) {
            const double2 w = tw[idx];
            const double2 a = P[q], b = X[q], c = Y[q];
            pr = fma(a.x, w.x, fma(-a.y, w.y, pr));
            pi = fma(a.y, w.x, fma(a.x, w.y, pi));
            xr = fma(b.x, w.x, fma(-b.y, w.y, xr));
            xi = fma(b.y, w.x, fma(b.x, w.y, xi));
            yr = fma(c.x, w.x, fma(-c.y, w.y, yr));
            yi = fma(c.y, w.x, fma(c.x, w.y, yi));
            idx += ix;
            if (idx >= nx) idx -= nx;
        }
        part[t] = make_double2(pr, pi);
        part[np + t] = make_double2(xr, xi);
        part[2 * np + t] = make_double2(yr, yi);
    }
    __syncthreads();
    const double sc = 1.0 / (double)nx;
    for (int ix = threadIdx.x; ix < nx; ix += blockDim.x) {
        double2 p = part[ix], x = part[np + ix], y = part[2 * np + ix];
        for (int h = 1; h < H; ++h) {
            const double2 a = part[h * nx + ix], b = part[np + h * nx + ix], c = part[2 * np + h * nx + ix];
            p.x += a.x;
            p.y += a.y;
            x.x += b.x;
            x.y += b.y;
            y.x += c.x;
            y.y += c.y;
        }
        const int64_t o = (int64_t)ix * nyh + k;
        Zp[o] = make_double2(p.x * sc, p.y * sc);
        Zx[o] = make_double2(x.x * sc, x.y * sc);
        Zy[o] = make_double2(y.x * sc, y.y * sc);
    }
}

__global__ void __launch_bounds__(kPBlock) k_p2_cols(const double2* __restrict__ R, int nx, int ny,
                                                   const double* __restrict__ kx, const double* __restrict__ ky,
                                                   const double* __restrict__ inv_ksq, double2* __restrict__ Zp,
                                                   double2* __restrict__ Zx, double2* __restrict__ Zy) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    p2_cols(R, nx, ny, kx, ky, inv_ksq, Zp, Zx, Zy, blockIdx.x, smem_raw);  // block = ky index
}

// ---- 2D: rows, complex-to-real inverse ------------------------------------------
__device__ __forceinline__ void p2_rows_inv(const double2* __restrict__ Zp, const double2* __restrict__ Zx,
                                            const double2* __restrict__ Zy, int nx, int ny, double* __restrict__ phi,
                                            double* __restrict__ ex, double* __restrict__ ey,
                                            double* __restrict__ we_part, double* __restrict__ emax_part,
                                            const int ix, unsigned char* smem_raw) {
    const int nyh = ny / 2 + 1;
    double2* tw = reinterpret_cast<double2*>(smem_raw);
    double2* zp = tw + ny;
    double2* zx = zp + nyh;
    double2* zy = zx + nyh;
    double* scratch = reinterpret_cast<double*>(zy + nyh);
    const size_t np = p2_parts(ny, blockDim.x);
    double* part = scratch + kPBlock;  // [3][np]
    fill_twiddles(tw, ny);
    for (int q = threadIdx.x; q < nyh; q += blockDim.x) {
        const int64_t o = (int64_t)ix * nyh + q;
        zp[q] = Zp[o];
        zx[q] = Zx[o];
        zy[q] = Zy[o];
    }
    __syncthreads();
    const bool even = (ny % 2) == 0;
    const int last = (ny - 1) / 2;  // last bin that appears twice
    // sums over the bins 1..last, cut into H slices
    const int H = p2_slices(ny, blockDim.x);
    for (int t = threadIdx.x; t < ny * H; t += blockDim.x) {
        const int iy = t % ny, h = t / ny;
        const int q0 = 1 + h * last / H, q1 = 1 + (h + 1) * last / H;
        double sp = 0.0, sx = 0.0, sy = 0.0;
        int idx = (int)(((int64_t)iy * q0) % ny);
        for (int q = q0; q < q1; ++q) {
            const double2 w = tw[idx];
            sp = fma(zp[q].x, w.x, fma(-zp[q].y, w.y, sp));
            sx = fma(zx[q].x, w.x, fma(-zx[q].y, w.y, sx));
            sy = fma(zy[q].x, w.x, fma(-zy[q].y, w.y, sy));
            idx += iy;
            if (idx >= ny) idx -= ny;
        }
        part[t] = sp;
        part[np + t] = sx;
        part[2 * np + t] = sy;
    }
    __syncthreads();
    const double sc = 1.0 / (double)ny;
    double we = 0.0, exm = 0.0, eym = 0.0;
    for (int iy = threadIdx.x; iy < ny; iy += blockDim.x) {
        double sp = part[iy], sx = part[np + iy], sy = part[2 * np + iy];
        for (int h = 1; h < H; ++h) {
            sp += part[h * ny + iy];
            sx += part[np + h * ny + iy];
            sy += part[2 * np + h * ny + iy];
        }
        double vp = zp[0].x + 2.0 * sp, vx = zx[0].x + 2.0 * sx, vy = zy[0].x + 2.0 * sy;
        if (even) {
            const double sgn = (iy & 1) ? -1.0 : 1.0;
            vp += sgn * zp[ny / 2].x;
            vx += sgn * zx[ny / 2].x;
            vy += sgn * zy[ny / 2].x;
        }
        vp *= sc;
        vx *= sc;
        vy *= sc;
        const int64_t o = (int64_t)ix * ny + iy;
        if (phi) phi[o] = vp;
        if (ex) ex[o] = vx;
        if (ey) ey[o] = vy;
        we = fma(vx, vx, fma(vy, vy, we));
        exm = fmax(exm, fabs(vx));
        eym = fmax(eym, fabs(vy));
    }
    we = block_sum(we, scratch);
    exm = block_max(exm, scratch);
    eym = block_max(eym, scratch);
    if (threadIdx.x == 0) {
        if (we_part) we_part[ix] = we;
        if (emax_part) {
            emax_part[2 * ix] = exm;
            emax_part[2 * ix + 1] = eym;
        }
    }
}

__global__ void __launch_bounds__(kPBlock) k_p2_rows_inv(const double2* __restrict__ Zp,
                                                       const double2* __restrict__ Zx,
                                                       const double2* __restrict__ Zy, int nx, int ny,
                                                       double* __restrict__ phi, double* __restrict__ ex,
                                                       double* __restrict__ ey, double* __restrict__ we_part,
                                                       double* __restrict__ emax_part) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    p2_rows_inv(Zp, Zx, Zy, nx, ny, phi, ex, ey, we_part, emax_part, blockIdx.x, smem_raw);
}

// ---- 2D, many runs: blockIdx.y = run, blockIdx.x = line (blocks past the
// run's line count leave at once) --------------------------------------------
__global__ void __launch_bounds__(kPBlock) k_p2_rows_fwd_batch(const Pois2dRun* __restrict__ runs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Pois2dRun a = runs[blockIdx.y];
    if ((int)blockIdx.x >= a.nx) return;
    p2_rows_fwd(a.rho, a.nx, a.ny, a.drho, a.R, a.mass_part, blockIdx.x, smem_raw);
}

__global__ void __launch_bounds__(kPBlock) k_p2_cols_batch(const Pois2dRun* __restrict__ runs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Pois2dRun a = runs[blockIdx.y];
    if ((int)blockIdx.x >= a.ny / 2 + 1) return;
    p2_cols(a.R, a.nx, a.ny, a.kx, a.ky, a.inv_ksq, a.Zp, a.Zx, a.Zy, blockIdx.x, smem_raw);
}

__global__ void __launch_bounds__(kPBlock) k_p2_rows_inv_batch(const Pois2dRun* __restrict__ runs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Pois2dRun a = runs[blockIdx.y];
    if ((int)blockIdx.x >= a.nx) return;
    p2_rows_inv(a.Zp, a.Zx, a.Zy, a.nx, a.ny, a.phi, a.ex, a.ey, a.we_part, a.emax_part, blockIdx.x, smem_raw);
}

// ---- diagnostics finalize (one block, fixed order) -------------------------------
__device__ __forceinline__ void diag_finalize(const DiagArgs& a, double* scratch) {
    double m = 0.0, w = 0.0, ex = 0.0, ey = 0.0, pre = 0.0, post = 0.0, l2 = 0.0;
    for (int i = threadIdx.x; i < a.n_mass; i += blockDim.x) m += a.mass_part[i];
    for (int i = threadIdx.x; i < a.n_we; i += blockDim.x) w += a.we_part[i];
    for (int i = threadIdx.x; i < a.n_emax; i += blockDim.x) {
        ex = fmax(ex, a.emax_part[2 * i]);
        ey = fmax(ey, a.emax_part[2 * i + 1]);
    }
    for (int64_t i = threadIdx.x; i < a.n_mom; i += blockDim.x) {
        pre += a.moments[4 * i + 0];
        post += a.moments[4 * i + 1];
        l2 += a.moments[4 * i + 2];
    }
    m = block_sum(m, scratch);
    w = block_sum(w, scratch);
    ex = block_max(ex, scratch);
    ey = block_max(ey, scratch);
    pre = block_sum(pre, scratch);
    post = block_sum(post, scratch);
    l2 = block_sum(l2, scratch);
    if (threadIdx.x == 0) {
        const double we = w * a.we_scale, mass = m * a.mass_scale;
        if (a.status && ((a.n_we && !isfinite(we)) || (a.n_mass && !isfinite(mass))))
            atomicOr(a.status, VP_STATUS_NONFINITE);
        if (a.energy) {
            a.energy[0] = we;
            a.energy[1] = mass;
        }
        if (a.diag) {
            const double nan = __longlong_as_double(0x7ff8000000000000ULL);
            a.diag[VP_DIAG_FIELD_ENERGY] = a.n_we ? we : 0.0;
            a.diag[VP_DIAG_MASS] = a.n_mass ? mass : nan;
            a.diag[VP_DIAG_L2] = a.n_mom ? l2 * a.dv_scale : nan;
            a.diag[VP_DIAG_KINETIC] = a.n_mom ? 0.5 * post * a.dv_scale : nan;
            a.diag[VP_DIAG_KINETIC_PRE] = a.n_mom ? 0.5 * pre * a.dv_scale : nan;
            a.diag[VP_DIAG_MAX_SHIFT] = a.n_emax ? fmax(ex * a.shift_x, ey * a.shift_y) : 0.0;
            a.diag[6] = 0.0;
            a.diag[7] = 0.0;
        }
    }
}

__global__ void __launch_bounds__(kPBlock) k_diag_finalize(const __grid_constant__ DiagArgs a) {
    __shared__ double scratch[kPBlock];
    diag_finalize(a, scratch);
}

// one block per run; run r's diagnostics land at diag + slot * slot_stride
__global__ void __launch_bounds__(kPBlock) k_diag_finalize_batch(const DiagArgs* __restrict__ runs, int slot) {
    __shared__ double scratch[kPBlock];
    DiagArgs a = runs[blockIdx.x];
    if (a.diag) a.diag += (int64_t)slot * a.slot_stride;
    diag_finalize(a, scratch);
}

// ---- 2D host ------------------------------------------------------------------
struct Pois2dWs {
    double2 *R, *Zp, *Zx, *Zy;
    double *mass_part, *we_part, *emax_part;
};

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

static size_t pois2d_layout(int64_t nx, int64_t ny, char* base, Pois2dWs* w) {
    const int64_t nyh = ny / 2 + 1;
    const size_t cplx = align256((size_t)nx * nyh * sizeof(double2));
    const size_t line = align256((size_t)nx * sizeof(double));
    size_t off = 0;
    auto take = [&](size_t b) {
        char* p = base ? base + off : nullptr;
        off += b;
        return p;
    };
    Pois2dWs t;
    t.R = reinterpret_cast<double2*>(take(cplx));
    t.Zp = reinterpret_cast<double2*>(take(cplx));
    t.Zx = reinterpret_cast<double2*>(take(cplx));
    t.Zy = reinterpret_cast<double2*>(take(cplx));
    t.mass_part = reinterpret_cast<double*>(take(line));
    t.we_part = reinterpret_cast<double*>(take(line));
    t.emax_part = reinterpret_cast<double*>(take(2 * line));
    if (w) *w = t;
    return off;
}

size_t poisson2d_ws_bytes(int64_t nx, int64_t ny) { return pois2d_layout(nx, ny, nullptr, nullptr); }

static int set_smem(const void* kern, size_t smem) {
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return set_cuda_error("cudaFuncSetAttribute(poisson)");
    return VP_OK;
}

// Launches the three transform kernels; partials stay in the workspace.
int run_poisson2d(const double* rho, int64_t nx, int64_t ny, const double* kx, const double* ky,
                  const double* inv_ksq, double* ex, double* ey, double* drho, double* phi, void* ws,
                  Pois2dWsView* view, cudaStream_t st) {
    Pois2dWs w;
    pois2d_layout(nx, ny, static_cast<char*>(ws), &w);
    const int64_t nyh = ny / 2 + 1;
    int rc;
    const size_t s1 = p2_fwd_smem((int)ny);
    if ((rc = set_smem((const void*)k_p2_rows_fwd, s1))) return rc;
    k_p2_rows_fwd<<<(unsigned)nx, kPBlock, s1, st>>>(rho, (int)nx, (int)ny, drho, w.R, w.mass_part);
    if ((rc = check_launch("k_p2_rows_fwd"))) return rc;
    const size_t s2 = p2_cols_smem((int)nx);
    if ((rc = set_smem((const void*)k_p2_cols, s2))) return rc;
    k_p2_cols<<<(unsigned)nyh, kPBlock, s2, st>>>(w.R, (int)nx, (int)ny, kx, ky, inv_ksq, w.Zp, w.Zx, w.Zy);
    if ((rc = check_launch("k_p2_cols"))) return rc;
    const size_t s3 = p2_inv_smem((int)ny);
    if ((rc = set_smem((const void*)k_p2_rows_inv, s3))) return rc;
    k_p2_rows_inv<<<(unsigned)nx, kPBlock, s3, st>>>(w.Zp, w.Zx, w.Zy, (int)nx, (int)ny, phi, ex, ey, w.we_part,
                                                     w.emax_part);
    if ((rc = check_launch("k_p2_rows_inv"))) return rc;
    if (view) {
        view->mass_part = w.mass_part;
        view->we_part = w.we_part;
        view->emax_part = w.emax_part;
        view->n_lines = (int)nx;
    }
    return VP_OK;
}

// Poisson arguments of one run of a batch (workspace of poisson2d_ws_bytes).
void pois2d_run_args(const double* rho, int64_t nx, int64_t ny, const double* kx, const double* ky,
                     const double* inv_ksq, double* ex, double* ey, double* drho, double* phi, void* ws,
                     Pois2dRun* a, Pois2dWsView* view) {
    Pois2dWs w;
    pois2d_layout(nx, ny, static_cast<char*>(ws), &w);
    *a = Pois2dRun{};
    a->rho = rho;
    a->nx = (int)nx;
    a->ny = (int)ny;
    a->kx = kx;
    a->ky = ky;
    a->inv_ksq = inv_ksq;
    a->drho = drho;
    a->phi = phi;
    a->ex = ex;
    a->ey = ey;
    a->R = w.R;
    a->Zp = w.Zp;
    a->Zx = w.Zx;
    a->Zy = w.Zy;
    a->mass_part = w.mass_part;
    a->we_part = w.we_part;
    a->emax_part = w.emax_part;
    if (view) {
        view->mass_part = w.mass_part;
        view->we_part = w.we_part;
        view->emax_part = w.emax_part;
        view->n_lines = (int)nx;
    }
}

int launch_poisson2d_batch(const Pois2dRun* runs, int n_runs, int max_nx, int max_ny, cudaStream_t st) {
    const int max_nyh = max_ny / 2 + 1;
    int rc;
    const size_t s1 = p2_fwd_smem(max_ny);
    if ((rc = set_smem((const void*)k_p2_rows_fwd_batch, s1))) return rc;
    k_p2_rows_fwd_batch<<<dim3((unsigned)max_nx, (unsigned)n_runs), kPBlock, s1, st>>>(runs);
    if ((rc = check_launch("k_p2_rows_fwd_batch"))) return rc;
    const size_t s2 = p2_cols_smem(max_nx);
    if ((rc = set_smem((const void*)k_p2_cols_batch, s2))) return rc;
    k_p2_cols_batch<<<dim3((unsigned)max_nyh, (unsigned)n_runs), kPBlock, s2, st>>>(runs);
    if ((rc = check_launch("k_p2_cols_batch"))) return rc;
    const size_t s3 = p2_inv_smem(max_ny);
    if ((rc = set_smem((const void*)k_p2_rows_inv_batch, s3))) return rc;
    k_p2_rows_inv_batch<<<dim3((unsigned)max_nx, (unsigned)n_runs), kPBlock, s3, st>>>(runs);
    return check_launch("k_p2_rows_inv_batch");
}

int launch_diag_finalize_batch(const DiagArgs* runs, int n_runs, int slot, cudaStream_t st) {
    k_diag_finalize_batch<<<(unsigned)n_runs, kPBlock, 0, st>>>(runs, slot);
    return check_launch("k_diag_finalize_batch");
}

int run_diag_finalize(const Pois2dWsView& pv, const double* moments, int64_t n_mom, double mass_scale,
                      double we_scale, double dv_scale, double shift_x, double shift_y, double* energy,
                      double* diag, cudaStream_t st, int* status) {
    DiagArgs a{};
    a.mass_part = pv.mass_part;
    a.n_mass = pv.mass_part ? pv.n_lines : 0;
    a.we_part = pv.we_part;
    a.n_we = pv.we_part ? pv.n_lines : 0;
    a.emax_part = pv.emax_part;
    a.n_emax = pv.emax_part ? pv.n_lines : 0;
    a.moments = moments;
    a.n_mom = moments ? n_mom : 0;
    a.mass_scale = mass_scale;
    a.we_scale = we_scale;
    a.dv_scale = dv_scale;
    a.shift_x = shift_x;
    a.shift_y = shift_y;
    a.energy = energy;
    a.diag = diag;
    a.status = status;
    k_diag_finalize<<<1, kPBlock, 0, st>>>(a);
    return check_launch("k_diag_finalize");
}

// ---- 1D ----------------------------------------------------------------------
// In-place radix-2 complex FFT of x[0..n) in shared memory, sign = -1 forward
// (exp(-2 pi i jk/n)), +1 inverse (unscaled). tw[j] = exp(+2 pi i j/n), j < n/2.
__device__ void fft_radix2(double2* x, const double2* tw, int n, int logn, int sign) {
    if (logn == 0) return;  // length 1: identity
    // bit-reversal permutation
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int j = (int)(__brev((unsigned)i) >> (32 - logn));
        if (j > i) {
            const double2 t = x[i];
            x[i] = x[j];
            x[j] = t;
        }
    }
    __syncthreads();
    for (int s = 1; s <= logn; ++s) {
        const int m = 1 << s, half = m >> 1;
        const int tstride = n / m;
        for (int b = threadIdx.x; b < n / 2; b += blockDim.x) {
            const int grp = b / half, pos = b % half;
            const int i0 = grp * m + pos, i1 = i0 + half;
            double2 t = tw[pos * tstride];
            t.y *= sign;
            const double2 u = x[i0], v = x[i1];
            const double2 tv = make_double2(v.x * t.x - v.y * t.y, v.x * t.y + v.y * t.x);
            x[i0] = make_double2(u.x + tv.x, u.y + tv.y);
            x[i1] = make_double2(u.x - tv.x, u.y - tv.y);
        }
        __syncthreads();
    }
}

// Direct DFT variant for lengths that are not powers of two: y = sum x w^(sign jk)
__device__ void dft_direct(const double2* x, double2* y, const double2* tw, int n, int sign) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double re = 0.0, im = 0.0;
        int idx = 0;
        for (int j = 0; j < n; ++j) {
            double2 t = tw[idx];
            t.y *= sign;
            re = fma(x[j].x, t.x, fma(-x[j].y, t.y, re));
            im = fma(x[j].y, t.x, fma(x[j].x, t.y, im));
            idx += k;
            if (idx >= n) idx -= n;
        }
        y[k] = make_double2(re, im);
    }
}

__global__ void __launch_bounds__(1024) k_p1(const double* __restrict__ nrho, int nx,
                                            const double* __restrict__ inv_kx,
                                            const double* __restrict__ inv_kx_sq, double* __restrict__ e,
                                            double* __restrict__ rho_out, double* __restrict__ phi,
                                            double* __restrict__ parts /* [3]: mass, we, emax */) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* tw = reinterpret_cast<double2*>(smem_raw);  // n entries
    double2* a = tw + nx;
    double2* b = a + nx;
    double* scratch = reinterpret_cast<double*>(b + nx);
    const int n = nx;
    int logn = 0;
    while ((1 << logn) < n) ++logn;
    const bool pow2 = (1 << logn) == n;
    fill_twiddles(tw, n);
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = nrho[i];
        m += v;
        const double r = v - 1.0;
        if (rho_out) rho_out[i] = r;
        a[i] = make_double2(r, 0.0);
    }
    m = block_sum(m, scratch);
    __syncthreads();
    double2* spec;
    if (pow2) {
        fft_radix2(a, tw, n, logn, -1);
        spec = a;
    } else {
        dft_direct(a, b, tw, n, -1);
        __syncthreads();
        spec = b;
    }
    // Build the hermitian spectrum of E_k + i*phi_k (bins 0..n/2 from the
    // half spectrum, imaginary parts of DC and Nyquist dropped as c2r does).
    double2* z = (spec == a) ? b : a;
    const int nh = n / 2 + 1;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int kk = k < nh ? k : n - k;  // mirror
        const double2 r = spec[kk];
        // E_k = (im*ik, -re*ik); phi_k = (re*ik2, im*ik2)
        double er = r.y * inv_kx[kk], ei = -r.x * inv_kx[kk];
        double pr = r.x * inv_kx_sq[kk], pi = r.y * inv_kx_sq[kk];
        if (kk == 0 || (n % 2 == 0 && kk == n / 2)) {
            ei = 0.0;
            pi = 0.0;
        }
        if (k >= nh) {  // conjugate of the mirrored bin
            ei = -ei;
            pi = -pi;
        }
        // Z = E + i*phi
        z[k] = make_double2(er - pi, ei + pr);
    }
    __syncthreads();
    double2* res;
    if (pow2) {
        fft_radix2(z, tw, n, logn, +1);
        res = z;
    } else {
        double2* y = (z == a) ? b : a;
        dft_direct(z, y, tw, n, +1);
        __syncthreads();
        res = y;
    }
    const double sc = 1.0 / (double)n;
    double we = 0.0, em = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double ev = res[i].x * sc, pv = res[i].y * sc;
        e[i] = ev;
        if (phi) phi[i] = pv;
        we = fma(ev, ev, we);
        em = fmax(em, fabs(ev));
    }
    we = block_sum(we, scratch);
    em = block_max(em, scratch);
    if (threadIdx.x == 0 && parts) {
        parts[0] = m;
        parts[1] = we;
        parts[2] = em;
        parts[3] = 0.0;
    }
}

// ---- 1D, power-of-two lengths ------------------------------------------------
// The same solve for n = 2^k <= 8192 as a Stockham autosort FFT (radix-16
// passes, then one radix-2/4/8 pass for the remainder) in one block of
// max(32, n/16) threads. Pass with span p and radix R: butterfly b takes
// x_j = a[b + j n/R] (j < R), multiplies x_j by w^j (w = exp(-+2 pi i k/(pR)),
// k = b mod p), applies the R-point DFT in registers and stores its output m
// at (b - k) R + k + m p; after the last pass the array is in natural order.
// Each thread keeps 16 values per pass, every pass reads its inputs, waits for
// the block, then overwrites the same buffer, and the buffer is padded by one
// entry every 16 so that the strided accesses of every pass spread over all
// shared-memory banks. The R-point DFT is a radix-2 decimation in frequency
// over registers with the 16th roots of unity as constants.
namespace p1 {
constexpr int kMaxN = 8192;
constexpr int kMaxThreads = kMaxN / 16;

__host__ __device__ __forceinline__ int pad(int i) { return i + (i >> 4); }

__device__ __forceinline__ double2 cmul(double2 a, double2 w) {
    return make_double2(fma(a.x, w.x, -a.y * w.y), fma(a.x, w.y, a.y * w.x));
}

// cos and sin of 2 pi q / 16
__host__ __device__ constexpr double cos16(int q) {
    constexpr double C = 0.92387953251128675613, S = 0.38268343236508977173, H = 0.70710678118654752440;
    switch (q & 15) {
        case 0: return 1.0;
        case 1: return C;
        case 2: return H;
        case 3: return S;
        case 4: return 0.0;
        case 5: return -S;
        case 6: return -H;
        case 7: return -C;
        case 8: return -1.0;
        case 9: return -C;
        case 10: return -H;
        case 11: return -S;
        case 12: return 0.0;
        case 13: return S;
        case 14: return H;
        default: return C;
    }
}
__host__ __device__ constexpr double sin16(int q) { return cos16(q - 4); }

// a * exp(-+2 pi i q/16) (minus for the forward transform); q is a constant
// once the calling loops are unrolled
template <bool INV>
__device__ __forceinline__ double2 rot16(double2 a, int q) {
    q &= 15;
    if (q == 0) return a;
    if (q == 8) return make_double2(-a.x, -a.y);
    if (q == 4) return INV ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
    if (q == 12) return INV ? make_double2(a.y, -a.x) : make_double2(-a.y, a.x);
    return cmul(a, make_double2(cos16(q), INV ? sin16(q) : -sin16(q)));
}

__host__ __device__ constexpr int bitrev(int m, int bits) {
    int r = 0;
    for (int i = 0; i < bits; ++i) r |= ((m >> i) & 1) << (bits - 1 - i);
    return r;
}

// R-point DFT of x in place, natural order in and out
template <int R, bool INV>
__device__ __forceinline__ void dft(double2* x) {
    constexpr int bits = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4;
#pragma unroll
    for (int len = R; len >= 2; len >>= 1) {
#pragma unroll
        for (int s = 0; s < R; s += len) {
#pragma unroll
            for (int j = 0; j < len / 2; ++j) {
                const double2 a = x[s + j], b = x[s + j + len / 2];
                x[s + j] = make_double2(a.x + b.x, a.y + b.y);
                x[s + j + len / 2] = rot16<INV>(make_double2(a.x - b.x, a.y - b.y), j * (16 / len));
            }
        }
    }
    double2 y[R];
#pragma unroll
    for (int m = 0; m < R; ++m) y[bitrev(m, bits)] = x[m];
#pragma unroll
    for (int m = 0; m < R; ++m) x[m] = y[m];
}

// x[j] *= w^j (j < R), the powers from a product tree of depth log2(R)
template <int R>
__device__ __forceinline__ void twiddle(double2* x, double2 w) {
    x[1] = cmul(x[1], w);
    if constexpr (R > 2) {
        const double2 w2 = cmul(w, w);
        x[2] = cmul(x[2], w2);
        x[3] = cmul(x[3], cmul(w2, w));
        if constexpr (R > 4) {
            const double2 w4 = cmul(w2, w2);
            x[4] = cmul(x[4], w4);
#pragma unroll
            for (int j = 5; j < 8; ++j) x[j] = cmul(x[j], cmul(w4, j == 5 ? w : j == 6 ? w2 : cmul(w2, w)));
            if constexpr (R > 8) {
                const double2 w8 = cmul(w4, w4);
                x[8] = cmul(x[8], w8);
                const double2 w3 = cmul(w2, w);
                const double2 lo[8] = {w, w, w2, w3, w4, cmul(w4, w), cmul(w4, w2), cmul(w4, w3)};
#pragma unroll
                for (int j = 9; j < 16; ++j) x[j] = cmul(x[j], cmul(w8, lo[j - 8]));
            }
        }
    }
}

template <int R, bool INV>
__device__ __forceinline__ void pass(double2* buf, int n, int p) {
    constexpr int NB = 16 / R;
    const int nb = n / R, T = blockDim.x;
    double2 x[NB][R];
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int b = threadIdx.x + q * T;
        if (b < nb) {
#pragma unroll
            for (int j = 0; j < R; ++j) x[q][j] = buf[pad(b + j * nb)];
        }
    }
    __syncthreads();
    const double inv_pr = 2.0 / (double)(p * R);  // a power of two: exact
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int b = threadIdx.x + q * T;
        if (b < nb) {
            const int k = b & (p - 1);
            if (k) {
                double sn, cs;
                sincospi((double)k * inv_pr, &sn, &cs);
                twiddle<R>(x[q], make_double2(cs, INV ? sn : -sn));
            }
            dft<R, INV>(x[q]);
            const int base = (b - k) * R + k;
#pragma unroll
            for (int m = 0; m < R; ++m) buf[pad(base + m * p)] = x[q][m];
        }
    }
    __syncthreads();
}

template <bool INV>
__device__ void fft(double2* buf, int n) {
    int p = 1;
    while (p * 16 <= n) {
        pass<16, INV>(buf, n, p);
        p *= 16;
    }
    const int r = n / p;
    if (r == 2) pass<2, INV>(buf, n, p);
    else if (r == 4) pass<4, INV>(buf, n, p);
    else if (r == 8) pass<8, INV>(buf, n, p);
}

// deterministic block reduction (sum, or max of non-negative values); the
// result is valid in thread 0
template <bool MAX>
__device__ double reduce(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double o = __shfl_xor_sync(0xffffffffu, v, off);
        v = MAX ? fmax(v, o) : v + o;
    }
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < nw ? red[lane] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_xor_sync(0xffffffffu, v, off);
            v = MAX ? fmax(v, o) : v + o;
        }
    }
    return v;
}
}  // namespace p1

// Arguments of k_p1_pow2. The density is either given (nrho) or summed from
// per-tile partials as k_rho_finalize does (t = 0, 1, ... in order, then
// * scale + offset); the diagnostics (optional) are those k_diag_finalize
// writes for one line of partials {mass, we, max |E|, 0}.
struct P1Args {
    const double* nrho;
    const double* part;
    int tiles;
    double scale, offset;
    int n;
    const double* inv_kx;
    const double* inv_kx_sq;
    double* e;
    double* rho_out;
    double* phi;
    double* parts;  // [4]: mass, we, emax, 0
    double* diag;   // [VP_DIAG_COUNT]
    double mass_scale, we_scale, shift;
    int* status;    // optional: VP_STATUS_NONFINITE ORed in
};

__global__ void __launch_bounds__(p1::kMaxThreads) k_p1_pow2(const __grid_constant__ P1Args a) {
    using namespace p1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = a.n;
    double2* buf = reinterpret_cast<double2*>(smem_raw);  // pad(n) entries
    double* red = reinterpret_cast<double*>(buf + pad(n));  // 3 x 32
    const int T = blockDim.x, t = threadIdx.x;
    double* __restrict__ rho_out = a.rho_out;
    double* __restrict__ e = a.e;
    double* __restrict__ phi = a.phi;
    const double* __restrict__ inv_kx = a.inv_kx;
    const double* __restrict__ inv_kx_sq = a.inv_kx_sq;
    // the thread's (at most 16) densities, all loads issued before any store
    double dens[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int i = t + q * T;
        double v = 0.0;
        if (i < n) {
            if (a.nrho) {
                v = __ldg(a.nrho + i);
            } else {
                double acc = 0.0;
                for (int k = 0; k < a.tiles; ++k) acc += __ldg(a.part + (int64_t)k * n + i);
                v = acc * a.scale + a.offset;
            }
        }
        dens[q] = v;
    }
    double m = 0.0;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int i = t + q * T;
        if (i >= n) break;
        const double v = dens[q];
        m += v;
        const double r = v - 1.0;
        if (rho_out) rho_out[i] = r;
        buf[pad(i)] = make_double2(r, 0.0);
    }
    m = reduce<false>(m, red);
    __syncthreads();
    fft<false>(buf, n);
    // the hermitian spectrum of Z = E + i phi from the bins 0..n/2 (imaginary
    // parts of the DC and Nyquist bins dropped, as a c2r transform does)
    const int nh = n / 2 + 1;
    double2 z[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int k = t + q * T;
        if (k < n) {
            const int kk = k < nh ? k : n - k;
            const double2 r = buf[pad(kk)];
            const double ik = __ldg(inv_kx + kk), ik2 = __ldg(inv_kx_sq + kk);
            double er = r.y * ik, ei = -r.x * ik;
            double pr = r.x * ik2, pi = r.y * ik2;
            if (kk == 0 || kk == n / 2) {
                ei = 0.0;
                pi = 0.0;
            }
            if (k >= nh) {
                ei = -ei;
                pi = -pi;
            }
            z[q] = make_double2(er - pi, ei + pr);
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int k = t + q * T;
        if (k < n) buf[pad(k)] = z[q];
    }
    __syncthreads();
    fft<true>(buf, n);
    const double sc = 1.0 / (double)n;
    double we = 0.0, em = 0.0;
    for (int i = t; i < n; i += T) {
        const double2 v = buf[pad(i)];
        const double ev = v.x * sc, pv = v.y * sc;
        e[i] = ev;
        if (phi) phi[i] = pv;
        we = fma(ev, ev, we);
        em = fmax(em, fabs(ev));
    }
    we = reduce<false>(we, red + 32);
    em = reduce<true>(em, red + 64);
    if (t == 0) {
        if (a.parts) {
            a.parts[0] = m;
            a.parts[1] = we;
            a.parts[2] = em;
            a.parts[3] = 0.0;
        }
        if (a.diag) {
            const double nan = __longlong_as_double(0x7ff8000000000000ULL);
            if (a.status && (!isfinite(we * a.we_scale) || !isfinite(m * a.mass_scale)))
                atomicOr(a.status, VP_STATUS_NONFINITE);
            a.diag[VP_DIAG_FIELD_ENERGY] = we * a.we_scale;
            a.diag[VP_DIAG_MASS] = m * a.mass_scale;
            a.diag[VP_DIAG_L2] = nan;
            a.diag[VP_DIAG_KINETIC] = nan;
            a.diag[VP_DIAG_KINETIC_PRE] = nan;
            a.diag[VP_DIAG_MAX_SHIFT] = fmax(em * a.shift, 0.0 * 0.0);
            a.diag[6] = 0.0;
            a.diag[7] = 0.0;
        }
    }
}

static bool p1_pow2(int64_t nx) { return nx >= 2 && nx <= p1::kMaxN && (nx & (nx - 1)) == 0; }

static int launch_p1_pow2(const P1Args& a, cudaStream_t st) {
    const size_t smem = (size_t)p1::pad(a.n) * sizeof(double2) + 96 * sizeof(double);
    int rc;
    if ((rc = set_smem((const void*)k_p1_pow2, smem))) return rc;
    k_p1_pow2<<<1, std::max(32, a.n / 16), smem, st>>>(a);
    return check_launch("k_p1_pow2");
}

bool poisson1d_fuses(int64_t nx) { return p1_pow2(nx); }

int run_poisson1d_fused(const double* n, const double* part, int tiles, double scale, double offset, int64_t nx,
                        const double* inv_kx, const double* inv_kx_sq, double* e, double* rho, double* phi,
                        double* parts, double* diag, double mass_scale, double we_scale, double shift,
                        int* status, cudaStream_t st) {
    if (!p1_pow2(nx)) return set_error(VP_ERR_UNSUPPORTED, "1D Poisson: fused form needs a power-of-two nx <= 8192");
    P1Args a{};
    a.nrho = n;
    a.part = part;
    a.tiles = tiles;
    a.scale = scale;
    a.offset = offset;
    a.n = (int)nx;
    a.inv_kx = inv_kx;
    a.inv_kx_sq = inv_kx_sq;
    a.e = e;
    a.rho_out = rho;
    a.phi = phi;
    a.parts = parts;
    a.diag = diag;
    a.mass_scale = mass_scale;
    a.we_scale = we_scale;
    a.shift = shift;
    a.status = status;
    return launch_p1_pow2(a, st);
}

size_t poisson1d_ws_bytes(int64_t nx) {
    (void)nx;
    return 256;
}

int run_poisson1d(const double* n, int64_t nx, const double* inv_kx, const double* inv_kx_sq, double* e,
                  double* rho, double* phi, double* parts, cudaStream_t st) {
    int rc;
    if (p1_pow2(nx)) {
        P1Args a{};
        a.nrho = n;
        a.n = (int)nx;
        a.inv_kx = inv_kx;
        a.inv_kx_sq = inv_kx_sq;
        a.e = e;
        a.rho_out = rho;
        a.phi = phi;
        a.parts = parts;
        return launch_p1_pow2(a, st);
    }
    const size_t smem = 3 * (size_t)nx * sizeof(double2) + 1024 * sizeof(double);
    if (smem > 220 * 1024) return set_error(VP_ERR_UNSUPPORTED, "1D Poisson: nx too large for one block");
    if ((rc = set_smem((const void*)k_p1, smem))) return rc;
    k_p1<<<1, 1024, smem, st>>>(n, (int)nx, inv_kx, inv_kx_sq, e, rho, phi, parts);
    return check_launch("k_p1");
}

}  // namespace vp

// ---- 2D, allocation-free variant ---------------------------------------------
// Scratch of vp_poisson2d_static: a file-scope device array sized for the
// largest grid that entry point accepts (VP_POISSON2D_STATIC_MAX_N in each
// direction). Every GPU that loads the library holds it until the process
// exits. Host code cannot use the symbol as an address: the device address is
// looked up once per device with cudaGetSymbolAddress and cached.
namespace vp {

constexpr size_t kStaticAlign(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kPoisStaticBytes =
    4 * kStaticAlign((size_t)VP_POISSON2D_STATIC_MAX_N * (VP_POISSON2D_STATIC_MAX_N / 2 + 1) * sizeof(double2)) +
    4 * kStaticAlign((size_t)VP_POISSON2D_STATIC_MAX_N * sizeof(double));

static __device__ __align__(256) unsigned char g_poisson2d_scratch[kPoisStaticBytes];

static std::mutex g_poisson2d_scratch_mu;
static void* g_poisson2d_scratch_ptr[64] = {nullptr};

// Device address of the scratch on the current device (looked up on the
// first call per device, which therefore should not happen inside a stream
// capture).
static int poisson2d_static_scratch(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return set_cuda_error("cudaGetDevice");
    if (dev < 0 || dev >= 64) return set_error(VP_ERR_UNSUPPORTED, "vp_poisson2d_static: device index >= 64");
    std::lock_guard<std::mutex> lock(g_poisson2d_scratch_mu);
    if (!g_poisson2d_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_poisson2d_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return set_error(VP_ERR_CUDA, "vp_poisson2d_static: cudaGetSymbolAddress of the scratch array failed");
        }
        g_poisson2d_scratch_ptr[dev] = p;
    }
    *out = g_poisson2d_scratch_ptr[dev];
    return VP_OK;
}

int run_poisson2d_static(const double* rho, int64_t nx, int64_t ny, const double* kx, const double* ky,
                         const double* inv_ksq, double dx, double dy, double* ex, double* ey, double* drho,
                         double* phi, double* energy, cudaStream_t st) {
    if (poisson2d_ws_bytes(nx, ny) > kPoisStaticBytes)
        return set_error(VP_ERR_UNSUPPORTED, "vp_poisson2d_static: grid larger than the static scratch");
    void* ws = nullptr;
    int rc = poisson2d_static_scratch(&ws);
    if (rc) return rc;
    // every kernel below writes its part of the scratch before reading it,
    // so nothing has to be cleared between calls
    Pois2dWsView v{};
    rc = run_poisson2d(rho, nx, ny, kx, ky, inv_ksq, ex, ey, drho, phi, ws, &v, st);
    if (rc || !energy) return rc;
    return run_diag_finalize(v, nullptr, 0, dx * dy, 0.5 * dx * dy, 0.0, 0.0, 0.0, energy, nullptr, st);
}

}  // namespace vp
