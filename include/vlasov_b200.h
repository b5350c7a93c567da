/*
 * vlasov_b200.h - C ABI of the B200 (sm_100a) Vlasov-Poisson library.
 *
 * Plain pointers and sizes only. Every array argument is a DEVICE pointer
 * unless its comment says "host". Every entry point enqueues work on the
 * given CUDA stream (a cudaStream_t passed as void*, NULL = legacy default
 * stream), returns immediately, and reports argument errors synchronously
 * through its return value. The library never allocates device memory inside
 * these calls: the caller owns every buffer, including the scratch
 * "workspace" whose size the *_workspace_bytes() queries return.
 *
 * Data layout: the distribution function f is a contiguous row-major array.
 * 2D2V: f[Nx][Ny][Nvx][Nvy] (vy fastest). 1D1V: f[Nx][Nv].
 * The sweep entry points view any such array as [n_outer][n_line][n_inner],
 * where n_line is the advected axis (n_outer = product of the dims before it,
 * n_inner = product of the dims after it).
 *
 * Each entry point cites the function of the reference PyTorch solver
 * (simulations/vlasov2d_2v/pytorch/src/vlasov2D2V.py and
 * simulations/vlasov1d_1v/pytorch/src/vlasov1D1V.py of
 * yasahi-hpc/JAX-PyTorch-Vlasov) whose result it reproduces.
 */
#ifndef VLASOV_B200_H
#define VLASOV_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define VP_OK 0
#define VP_ERR_ARG 1         /* null pointer, non-positive size, aliasing buffers */
#define VP_ERR_DTYPE 2       /* unknown storage type */
#define VP_ERR_WORKSPACE 3   /* workspace missing or smaller than required */
#define VP_ERR_CUDA 4        /* a CUDA call or kernel launch failed (see vp_last_error) */
#define VP_ERR_UNSUPPORTED 5 /* shape outside what the kernels implement */

/* Bits a step ORs into its device status word (vp_step2d_desc.status,
 * vp_step1d_desc.status) while it runs; the caller reads and clears it when
 * it synchronises (the launch itself has returned VP_OK by then). */
#define VP_STATUS_WAIT_TIMEOUT 1 /* a bounded device wait (TMA load completion) ran out after 1 s;
                                    the CTA filled its share of f (and of the density) with NaN */
#define VP_STATUS_NONFINITE 2    /* the step's field energy or mass is not finite */

/* ---- storage types of f ------------------------------------------------ */
#define VP_F32 0  /* float storage, float arithmetic */
#define VP_F64 1  /* double storage, double arithmetic */
#define VP_BF16 2 /* bfloat16 storage, float arithmetic */

/* The "compute type" of a storage type is double for VP_F64 and float
 * otherwise; drift weight tables and gather velocities use it. */

/* Library version string and the message of the last failed call on this
 * host thread. */
const char* vp_version(void);
const char* vp_last_error(void);

/* Number of kernels this process has launched through the library so far
 * (host-side count, all devices). No reference counterpart: it lets a
 * benchmark state how many of its own kernels ran in a timed region. */
uint64_t vp_launch_count(void);

/* ---- sweeps ------------------------------------------------------------ */

/* Periodic drift with static per-velocity shifts (the x and y drifts).
 * Replaces advect_x_static (vlasov2D2V.py:756-819; vlasov1D1V.py:408-448)
 * with the shift/weight tables of precompute_x_drift (vlasov2D2V.py:670-714):
 *   out[o,l,c] = sum_k W[k*sel_mod + j] * in[o, (l - shift[j] - (k-2)) mod n_line, c]
 * for k = 0..5, where j = (c / sel_div) % sel_mod.
 * shift: int32[sel_mod]; W: compute type [6][sel_mod]. f_out must not
 * overlap f_in.
 * shift_spread: an upper bound, supplied by the caller from the host copy of
 * the table, of max(shift) - min(shift) over every aligned group of 4 table
 * entries (4q .. 4q+3), or -1 if unknown. With sel_div == 1 (the y drift,
 * whose shift follows the contiguous vy index) a bound of 0 or 1 lets each
 * thread move 4 columns at once; otherwise the sweep uses scalar columns. */
int vp_drift(const void* f_in, void* f_out, int dtype, int64_t n_outer, int64_t n_line,
             int64_t n_inner, int64_t sel_div, int64_t sel_mod, const int32_t* shift,
             int32_t shift_spread, const void* W, void* stream);

/* The same drift fused with the velocity moment of its output (the y drift
 * before the field solve, vlasov2D2V.py:1064 followed by compute_rho :416-431;
 * 1D1V: the x drift and n = sum(f,1)*dv, vlasov1D1V.py:685,521):
 *   rho[o*n_line + l] = (sum_c out[o,l,c]) * scale      (FP64, deterministic)
 * workspace: vp_drift_rho_workspace_bytes() bytes of scratch. */
int vp_drift_rho(const void* f_in, void* f_out, int dtype, int64_t n_outer, int64_t n_line,
                 int64_t n_inner, int64_t sel_div, int64_t sel_mod, const int32_t* shift,
                 int32_t shift_spread, const void* W, double scale, double* rho, void* workspace,
                 size_t workspace_bytes, void* stream);
size_t vp_drift_rho_workspace_bytes(int64_t n_outer, int64_t n_line, int64_t n_inner);

/* Both position drifts of f[nx][ny][nvx][nvy] in one pass over f, the
 * intermediate on chip: x then y (xfirst = 1) or y then x (xfirst = 0), each
 * drift as vp_drift with its own table (shift_x/W_x indexed by vx, shift_y/
 * W_y by vy; W in FP32). Replaces the pairs advect_x_static(axis 0) +
 * advect_x_static(axis 1) of vlasov_step_gather_free_impl
 * (vlasov2D2V.py:1063-1064 and :1079-1080); f is the same bits as the two
 * sweeps give. Only the output rows x_begin .. x_begin + x_count - 1 are
 * written (the input rows wrap around nx), so a caller can compute the rows
 * that need fresh neighbour data apart from the others. With xfirst and rho
 * != NULL the pass also forms the density of its rows,
 *   rho[x*ny + y] = scale * sum_{vx,vy} out[x,y,vx,vy]   (FP64, deterministic),
 * for x in the range; workspace: vp_drift_pair_workspace_bytes() bytes
 * (the density partials; may be NULL without rho).
 * Needs FP32, 16 <= ny <= 128, nvy a multiple of 32 and 16-byte aligned
 * buffers; VP_ERR_UNSUPPORTED otherwise (the caller then runs two vp_drift
 * sweeps). */
int vp_drift_pair(const void* f_in, void* f_out, int dtype, int64_t nx, int64_t ny, int64_t nvx,
                  int64_t nvy, int32_t xfirst, int64_t x_begin, int64_t x_count, const int32_t* shift_x,
                  const void* W_x, const int32_t* shift_y, const void* W_y, double scale, double* rho,
                  void* workspace, size_t workspace_bytes, void* stream);
size_t vp_drift_pair_workspace_bytes(int64_t nx, int64_t ny, int64_t nvx, int64_t nvy);

/* Dirichlet kick along n_line with a field constant over each outer row
 * (the vx or vy kick). Replaces advect_v_static with build_v_tap_weights
 * (vlasov2D2V.py:822-913; vlasov1D1V.py:450-501): outer row o uses the field
 * value E[o / e_div] (e_dtype VP_F32 or VP_F64), d = E*dt/dv, s = floor(d),
 * alpha = d - s, and
 *   out[o,l,c] = sum_k w_k(alpha) * in[o, l - s - (k-2), c]   (zero outside [0, n_line)).
 * window >= 0 drops the taps with |s + k - 2| > window + 2, as the
 * reference's static window S does; window < 0 keeps every tap (exact for
 * any |d|). */
int vp_kick(const void* f_in, void* f_out, int dtype, int64_t n_outer, int64_t n_line,
            int64_t n_inner, const void* E, int e_dtype, int64_t e_div, double dt, double dv,
            int32_t window, void* stream);

/* Both kicks of one 2D2V Strang step in one pass over each (x, y) plane:
 * the vx kick with Ex, then the vy kick with Ey (vlasov2D2V.py:1076-1077).
 * f is [n_planes][nvx][nvy]; Ex, Ey: double[n_planes].
 * moments (optional, NULL to skip): double[n_planes][4] per-plane sums
 *   { sum f_in*(vx^2+vy^2), sum f_out*(vx^2+vy^2), sum f_out^2, sum f_out }
 * with vx, vy the velocity grids (double[nvx], double[nvy]; required only
 * with moments). */
int vp_kick2d(const void* f_in, void* f_out, int dtype, int64_t n_planes, int64_t nvx,
              int64_t nvy, const double* Ex, const double* Ey, double dt, double dvx,
              double dvy, int32_t window, const double* vx, const double* vy, double* moments,
              void* stream);

/* General semi-Lagrangian sweep with a per-element departure point.
 * Replaces advect_1d / advect_1d_vectorized (vlasov2D2V.py:287-413;
 * vlasov1D1V.py:212-256): depart = l - (v*dt)/dx, floor/fraction in the
 * compute type, taps floor+k-2 taken mod n_line (periodic != 0) or masked
 * to zero outside [0, n_line). The velocity of element (o,l,c) is
 * vel[o*vs_outer + l*vs_line + c*vs_inner] (compute type). */
int vp_advect_gather(const void* f_in, void* f_out, int dtype, int64_t n_outer, int64_t n_line,
                     int64_t n_inner, const void* vel, int64_t vs_outer, int64_t vs_line,
                     int64_t vs_inner, double dt, double dx, int periodic, void* stream);

/* ---- initial conditions ---------------------------------------------------- */

/* f[p][v] = space[p] * vel[v] for p < n_points, v < n_v (f row-major,
 * space and vel FP64 on the device), the product rounded once to dtype: the
 * initial conditions of Vlasov.initialize (vlasov2D2V.py:1319-1355, Landau:
 * space = 1 + eps cos(kx x) cos(ky y), vel = exp(-|v|^2/2)/sqrt(2 pi);
 * vlasov1D1V.py:881-911), which the reference builds as a broadcast tensor
 * product; the result has the same bits as that product rounded by
 * .to(dtype). */
int vp_init_product(const double* space, const double* vel, void* f, int dtype, int64_t n_points, int64_t n_v,
                    void* stream);

/* ---- interpolation helpers ---------------------------------------------- */

/* The 6-point Lagrange sum of lagrange5_interp_sum (vlasov2D2V.py:238-260;
 * vlasov1D1V.py, same function): out[i] = sum_k w_k(alpha[i]) vals[6 i + k]
 * with the closed-form weights of the nodes -2..3, each product rounded and
 * the terms summed left to right. dtype VP_F32 or VP_F64. */
int vp_lagrange_interp(const void* alpha, const void* vals, void* out, int dtype, int64_t n, void* stream);
/* The product-form weights of get_lagrange5_weights (vlasov2D2V.py:210-235):
 * weights[6 i + j] = prod_{m != j} (alpha[i] - x_m) / (x_j - x_m). */
int vp_lagrange_weights(const void* alpha, void* weights, int dtype, int64_t n, void* stream);

/* ---- moments and field ------------------------------------------------- */

/* Velocity moment. Replaces compute_rho (vlasov2D2V.py:416-431):
 *   rho[p] = (sum_{c < n_v} f[p*n_v + c]) * dvx * dvy,
 * summed in FP64 in a fixed order; written as out_dtype (VP_F32/VP_F64). */
int vp_rho(const void* f, int dtype, int64_t n_points, int64_t n_v, double dvx, double dvy,
           void* rho, int out_dtype, void* stream);

/* Periodic 2D Poisson solve in FP64. Replaces compute_poisson_real
 * (vlasov2D2V.py:488-517): delta = rho - 1, phi_k = rfft2(delta)*inv_ksq,
 * E_k = -i k phi_k, then irfft2 of size (nx, ny) (imaginary parts of the
 * DC and Nyquist bins of the last axis ignored, as torch.fft does).
 * kx: double[nx]; ky: double[ny/2+1]; inv_ksq: double[nx][ny/2+1].
 * Outputs (any may be NULL except ex, ey): ex, ey, drho, phi: double[nx][ny].
 * energy (optional): double[2] = { 1/2 sum(ex^2+ey^2) dx dy, sum(rho) dx dy }.
 * Sizes: 1 <= nx, ny <= 4096, and the transforms' shared memory (about
 * 128 nx bytes for the columns, 64 ny for the inverse rows) within the
 * 227 KB a block may hold, i.e. nx up to about 1800 and ny up to about
 * 3600; larger sizes return VP_ERR_UNSUPPORTED (so do vp_step2d and
 * vp_batch2d_plan in physics mode). */
int vp_poisson2d(const double* rho, int64_t nx, int64_t ny, const double* kx, const double* ky,
                 const double* inv_ksq, double dx, double dy, double* ex, double* ey,
                 double* drho, double* phi, double* energy, void* workspace,
                 size_t workspace_bytes, void* stream);
size_t vp_poisson2d_workspace_bytes(int64_t nx, int64_t ny);

/* vp_poisson2d for callers that cannot allocate device memory. No
 * counterpart in the reference (whose field solve allocates through
 * torch.fft): this entry point serves hosts that must not call cudaMalloc or
 * any allocating routine at the point of the call, such as a foreign runtime
 * that hands over only its own pre-registered input and output buffers and
 * owns all other device memory, or an embedded solver that may not grow its
 * device footprint after start-up.
 * The caller passes inputs and outputs exactly as for vp_poisson2d; the
 * scratch comes from a file-scope device array of the library, sized for
 * nx, ny <= VP_POISSON2D_STATIC_MAX_N (about 2 MiB, held on every GPU that
 * loads the library until the process exits). Larger grids are rejected with
 * VP_ERR_UNSUPPORTED. The first call on a device looks up that array's
 * device address (cudaGetSymbolAddress); make that first call before any
 * stream capture. All calls share the one array and it keeps the last call's
 * contents (nothing in it has to start at zero): calls that overlap on the
 * GPU, e.g. on two streams at once, race with each other. */
#define VP_POISSON2D_STATIC_MAX_N 256
int vp_poisson2d_static(const double* rho, int64_t nx, int64_t ny, const double* kx, const double* ky,
                        const double* inv_ksq, double dx, double dy, double* ex, double* ey,
                        double* drho, double* phi, double* energy, void* stream);

/* Periodic 1D Poisson solve in FP64 from the density n = sum(f,1)*dv.
 * Replaces solve_poisson_real (vlasov1D1V.py:538-572) after its sum:
 * rho = n - 1, E_k = -i rho_k inv_kx, phi_k = rho_k inv_kx_sq, irfft(nx).
 * inv_kx, inv_kx_sq: double[nx/2+1]. e, rho, phi: double[nx] (rho, phi may
 * be NULL). energy (optional): double[2] = { 1/2 sum(e^2) dx, sum(n) dx }. */
int vp_poisson1d(const double* n, int64_t nx, const double* inv_kx, const double* inv_kx_sq,
                 double dx, double* e, double* rho, double* phi, double* energy,
                 void* workspace, size_t workspace_bytes, void* stream);
size_t vp_poisson1d_workspace_bytes(int64_t nx);

/* ---- one Strang step ---------------------------------------------------- */

/* Diagnostics written by the step functions (double[VP_DIAG_COUNT]). */
#define VP_DIAG_FIELD_ENERGY 0 /* 1/2 sum |E|^2 dx (dy): mid-step field */
#define VP_DIAG_MASS 1         /* sum n dx (dy), n the mid-step density */
#define VP_DIAG_L2 2           /* sum f^2 dV after the kick(s) */
#define VP_DIAG_KINETIC 3      /* 1/2 sum f |v|^2 dV after the kick(s) */
#define VP_DIAG_KINETIC_PRE 4  /* 1/2 sum f |v|^2 dV before the kick(s) */
#define VP_DIAG_MAX_SHIFT 5    /* max |E| dt/dv over both kicks, in cells */
#define VP_DIAG_COUNT 8

/* Phases of a step, for the optional timing events of the step descriptors:
 * events[2p] is recorded on the stream before phase p, events[2p+1] after
 * it (cudaEvent_t handles created by the caller; both at the same point
 * when a phase does not run). */
#define VP_PHASE_DRIFT_X1 0  /* 1D1V: the first x drift fused with n; 2D2V fused
                                pair: the x-then-y pass with its density partials */
#define VP_PHASE_DRIFT_Y1 1  /* y drift fused with rho (2D2V only); fused pair:
                                the sum of the density partials */
#define VP_PHASE_FIELD 2     /* Poisson solve */
#define VP_PHASE_KICK 3      /* vx+vy kick (2D2V), v kick (1D1V) */
#define VP_PHASE_DRIFT_Y2 4  /* 2D2V only */
#define VP_PHASE_DRIFT_X2 5
#define VP_PHASE_DIAG 6
#define VP_PHASE_COUNT 7

/* One Strang step of the 2D2V system, the schedule of
 * vlasov_step_gather_free_impl (vlasov2D2V.py:1043-1083):
 * x(dt/2), y(dt/2) fused with rho, Poisson, vx(dt)+vy(dt) fused,
 * y(dt/2), x(dt/2). Where the layout allows (FP32, 16 <= ny <= 128, nvy a
 * multiple of 32, 16-byte aligned buffers, sweeps_only == 0; with or
 * without the equilibrium split) each pair of position drifts runs as one pass over f
 * with the intermediate on chip: f is the same bits, rho is summed in
 * another (fixed) order. With physics_mode == 0 the field is zero, the
 * kicks are the identity and are skipped, and drho/phi are zeroed (as the
 * reference returns zeros). f_in is read only; the result is written to
 * f_out; f_tmp is a third buffer of the same size. Buffers must not
 * overlap. */
typedef struct vp_step2d_desc {
    int32_t dtype;
    int64_t nx, ny, nvx, nvy;
    double dt, dx, dy, dvx, dvy;
    int32_t physics_mode;
    int32_t window;        /* kick window S (<0: exact kick) */
    int32_t diagnostics;   /* 0: none; 1: field energy, mass, max shift; 2: also the
                              L2 / kinetic moments (an FP64 epilogue in the kick) */
    int32_t shift_spread_x; /* see vp_drift (tables of the x and y drifts) */
    int32_t shift_spread_y;
    const void* f_in;
    void* f_out;
    void* f_tmp;
    const int32_t* shift_x; /* [nvx] */
    const void* W_x;        /* compute type [6][nvx] */
    const int32_t* shift_y; /* [nvy] */
    const void* W_y;        /* compute type [6][nvy] */
    const double* kx;       /* [nx] */
    const double* ky;       /* [ny/2+1] */
    const double* inv_ksq;  /* [nx][ny/2+1] */
    const double* vx;       /* [nvx] (diagnostics only) */
    const double* vy;       /* [nvy] (diagnostics only) */
    double* drho;           /* [nx][ny] mid-step rho - 1 (may be NULL) */
    double* phi;            /* [nx][ny] mid-step potential (may be NULL) */
    double* ex;             /* [nx][ny] mid-step field (may be NULL) */
    double* ey;             /* [nx][ny] (may be NULL) */
    double* diag;           /* [VP_DIAG_COUNT] (may be NULL) */
    void* workspace;
    size_t workspace_bytes;
    void* const* events;    /* optional [2*VP_PHASE_COUNT] cudaEvent_t, NULL to skip */
    /* Equilibrium split (optional, both NULL to disable): f = feq + g with a
     * separable equilibrium feq(vx, vy) = eq_vx[ivx] * eq_vy[ivy] (double).
     * f_in / f_out / f_tmp then hold g, and every sweep advances g so that
     * feq + g follows the unsplit step exactly in exact arithmetic (the
     * drifts add feq*(sum of weights - 1), the kicks add the kicked
     * equilibrium minus feq). The stored precision then applies to the
     * perturbation instead of f. eq_moment = sum(eq_vx)*dvx * sum(eq_vy)*dvy
     * (the equilibrium's density, added to rho). Needs the fused kick (a
     * plane row of at most 128 elements per warp). No reference counterpart:
     * the reference stores the full f. */
    const double* eq_vx;
    const double* eq_vy;
    double eq_moment;
    /* nonzero: the position drifts run as one sweep per axis even where the
     * fused (x, y) plane passes apply; f is the same either way, the
     * density then also has the single-axis sweeps' summation order. */
    int32_t sweeps_only;
    /* optional device int32 (NULL to skip): VP_STATUS_* bits ORed in. */
    int32_t* status;
    /* test hook, 0 in normal use: nonzero makes the first TMA load of every
     * fused-plane CTA expect 16 more bytes than it brings, so that its wait
     * runs out (after 1 s) and the timeout path is exercised. */
    int32_t test_stall;
} vp_step2d_desc;

int vp_step2d(const vp_step2d_desc* desc, void* stream);
size_t vp_step2d_workspace_bytes(int64_t nx, int64_t ny, int64_t nvx, int64_t nvy);
/* How vp_step2d runs this descriptor, without GPU work: returns the number
 * of passes over f (each reads and writes f once; < 0 on a bad descriptor)
 * and sets *plane_fused (may be NULL) to 1 when the position drifts go in
 * pairs through the fused (x, y) plane passes (FP32 storage, 16 <= ny <=
 * 128, nvy a multiple of 32, 16-byte aligned buffers). No counterpart in the reference, whose drifts are separate tensor
 * operations; it tells a caller how much HBM traffic one step moves. */
int vp_step2d_passes(const vp_step2d_desc* desc, int32_t* plane_fused);

/* One Strang step of the 1D1V system, the schedule of
 * vlasov_step_gather_free_impl (vlasov1D1V.py:668-701): x(dt/2) fused with
 * n, Poisson, v(dt), x(dt/2). rho, phi, e are the mid-step fields. */
typedef struct vp_step1d_desc {
    int32_t dtype;
    int64_t nx, nv;
    double dt, dx, dv;
    int32_t physics_mode;
    int32_t window;
    int32_t diagnostics;
    int32_t shift_spread; /* see vp_drift */
    const void* f_in;
    void* f_out;
    void* f_tmp;
    const int32_t* shift; /* [nv] */
    const void* W;        /* compute type [6][nv] */
    const double* inv_kx;    /* [nx/2+1] */
    const double* inv_kx_sq; /* [nx/2+1] */
    const double* v;         /* [nv] (diagnostics only) */
    double* rho;
    double* phi;
    double* e;
    double* diag;
    void* workspace;
    size_t workspace_bytes;
    void* const* events; /* optional [2*VP_PHASE_COUNT] cudaEvent_t */
    /* Equilibrium split (optional): f = eq_v[iv] + g, as in vp_step2d_desc;
     * eq_moment = sum(eq_v) * dv. */
    const double* eq_v;
    double eq_moment;
    int32_t* status; /* optional device int32: VP_STATUS_* bits ORed in */
} vp_step1d_desc;

int vp_step1d(const vp_step1d_desc* desc, void* stream);
size_t vp_step1d_workspace_bytes(int64_t nx, int64_t nv);

/* ---- batched 2D2V steps ---------------------------------------------------
 * Many independent runs of uneven sizes and parameters advanced together,
 * one launch per substep for all of them (no reference counterpart: the
 * reference advances one run per Vlasov object, vlasov2D2V.py:1392-1435;
 * each run of a batch follows vp_step2d's schedule and arithmetic).
 *
 * Usage: fill one vp_batch2d_run per run; vp_batch2d_plan writes a table of
 * vp_batch2d_table_bytes(n) bytes into host memory; copy it unchanged to a
 * device buffer aligned to 64 bytes; then every vp_batch2d_step(table,
 * table_dev, slot, stream) advances all runs by one step. The step only
 * launches kernels (no copies, no allocation), so a sequence of steps can be
 * captured in a CUDA graph; it reads the host table too (the fused runs' TMA
 * descriptors go to the kernels as parameters), which must stay as planned.
 * Each run's state is advanced in place: f -> s2 -> s1 -> f for the runs
 * whose drift pairs are fused (FP32, 32 <= ny <= 64 with ny % 8 == 0,
 * nvy % 16 == 0 and nvx * nvy % 32 == 0, 16-byte aligned buffers, unless
 * vp_batch_tiles.sweeps_only),
 * else f -> s1 -> s2 -> s1 -> s2 -> f. */
typedef struct vp_batch2d_run {
    int32_t nx, ny, nvx, nvy;
    double dt, dx, dy, dvx, dvy;
    int32_t window;         /* kick window S (<0: exact kick) */
    int32_t shift_spread_x; /* see vp_drift */
    int32_t shift_spread_y;
    int32_t segments_x;     /* CTAs per x line of this run: 1, 2, 4 (0: the batch's tile shape) */
    int32_t segments_y;     /* CTAs per y line of this run (0: the batch's tile shape) */
    int32_t test_stall;     /* test hook: 1 makes the first TMA completion wait of each CTA of the fused
                               passes on this run run out (1 s), as vp_step2d_desc.test_stall; 0 */
    void* f;                /* [nx][ny][nvx][nvy] state, advanced in place */
    void* s1;               /* scratch of the size of f */
    void* s2;               /* scratch of the size of f */
    const int32_t* shift_x; /* [nvx] */
    const void* W_x;        /* compute type [6][nvx] */
    const int32_t* shift_y; /* [nvy] */
    const void* W_y;        /* compute type [6][nvy] */
    const double* kx;       /* [nx] */
    const double* ky;       /* [ny/2+1] */
    const double* inv_ksq;  /* [nx][ny/2+1] */
    double* drho;           /* [nx][ny] mid-step rho - 1 (may be NULL) */
    double* phi;            /* [nx][ny] (may be NULL) */
    double* diag;           /* VP_DIAG_COUNT doubles at diag + slot * diag_slot_stride (may be NULL) */
    int64_t diag_slot_stride;
    void* workspace;        /* vp_step2d_workspace_bytes(nx, ny, nvx, nvy) bytes */
    size_t workspace_bytes;
    int32_t* status;        /* optional device int32: VP_STATUS_* bits ORed in for this run (a wait of a
                               fused pass that ran out: the CTA's share of every run it served, this
                               one included, is NaN; non-finite diagnostics) */
} vp_batch2d_run;

/* Tile shapes of the batched sweeps, per sweep kind (0: x drifts, 1: y
 * drifts, 2: fused kick). Zeros select the defaults. */
#define VP_BATCH_KINDS 3
typedef struct vp_batch_tiles {
    int32_t block[VP_BATCH_KINDS];       /* threads per CTA (one tile of columns): 128 or 256 */
    int32_t ctas_per_sm[VP_BATCH_KINDS]; /* persistent CTAs per SM, <= the occupancy limit */
    int32_t segments[VP_BATCH_KINDS];    /* CTAs per line of the drifts: 1, 2 or 4 (ignored for the kick) */
    int32_t sweeps_only;                 /* 1: one sweep per axis for every run, even those the fused
                                            drift pairs take (FP32, 32 <= ny <= 64, ny % 8 == 0,
                                            nvy % 16 == 0, nvx * nvy % 32 == 0) */
} vp_batch_tiles;

size_t vp_batch2d_table_bytes(int32_t n_runs);
/* physics_mode must be 1 when diagnostics is 1; diagnostics: 0 or 1 (field
 * energy, mass, max shift). All runs share dtype. */
int vp_batch2d_plan(int32_t dtype, int32_t physics_mode, int32_t diagnostics, const vp_batch2d_run* runs,
                    int32_t n_runs, const vp_batch_tiles* tiles, void* table, size_t table_bytes);
/* events: optional [2*VP_PHASE_COUNT] cudaEvent_t around the substeps of
 * all runs (VP_PHASE_DRIFT_Y1 includes the rho finalize), NULL to skip. */
int vp_batch2d_step(const void* table, const void* table_dev, int32_t slot, void* const* events, void* stream);

/* ---- learned interpolation correction (BF16 tensor cores) ----------------
 * No reference counterpart. A per-cell network corrects the 6 Lagrange
 * weights of a periodic drift (the sweep of vp_drift, FP32 storage) or of a
 * kick (the sweep of vp_kick with the exact window):
 *   x  = [f_k / max|f| (k < 6), alpha - 1/2, 1, 0...]  (16 inputs)
 *   h1 = relu(W1 x), h2 = relu(W2 [h1, 1, 0...]), o = W3 [h2, 1, 0...]
 *   out = sum_k (W[k][j] + o_k - mean(o_0..o_5)) f_k
 * with f_k the stencil values of vp_drift, j the table column of the cell
 * and alpha[j] its fractional shift. When n_line and n_inner are both powers
 * of two the correction is projected line by line,
 *   out_l -= mean over the line of (out_l - sum_k W[k][j] f_k),
 * so that every line (o, c) keeps the plain sweep's sum (the drift conserves
 * it, the kick changes it only by what leaves the velocity range); the
 * training passes differentiate through the projection. Matrix products run
 * on tcgen05 tensor cores with BF16 operands and FP32 accumulation.
 * net: bf16 row-major, packed W1 [64][16] (column 7 = bias), W2 [64][80]
 * (column 64 = bias), W3 [16][80] (rows 6..15 zero), then the transposed
 * copies W3T [64][16] (W3T[h][o] = W3[o][h]) and W2T [64][64]
 * (W2T[i][m] = W2[m][i]) used by the backward pass.
 * status: device int32, set to 1 when a tensor-core completion wait timed out
 * (the results are then invalid). */
#define VP_MLP_NET_ELEMS (64 * 16 + 64 * 80 + 16 * 80 + 64 * 16 + 64 * 64)
#define VP_MLP_GRAD_ELEMS (64 * 16 + 64 * 80 + 16 * 80)
int vp_mlp_drift(const float* f_in, float* f_out, int64_t n_outer, int64_t n_line, int64_t n_inner,
                 int64_t sel_div, int64_t sel_mod, const int32_t* shift, const float* W,
                 const float* alpha, const void* net, int32_t* status, void* stream);
/* Training pass over every cell of one drift: r = (out - target) * inv_scale;
 * *loss += sum r^2 and grad (float [VP_MLP_GRAD_ELEMS]: dW1, dW2, dW3 in the
 * layout of net) += the gradient of sum r^2 (both accumulated, not
 * overwritten). */
int vp_mlp_train(const float* f_in, const float* target, int64_t n_outer, int64_t n_line,
                 int64_t n_inner, int64_t sel_div, int64_t sel_mod, const int32_t* shift,
                 const float* W, const float* alpha, const void* net, double inv_scale, float* grad,
                 double* loss, int32_t* status, void* stream);
/* The same correction applied to the kick of vp_kick (window < 0): row o of
 * [n_outer][n_line][n_inner] moves by E[o / e_div] * dt / dv cells, zero
 * outside the line; the shift, the fraction alpha and the plain weights
 * follow vp_kick's formulas, evaluated in FP32. */
int vp_mlp_kick(const float* f_in, float* f_out, int64_t n_outer, int64_t n_line, int64_t n_inner,
                const double* E, int64_t e_div, double dt, double dv, const void* net, int32_t* status,
                void* stream);
int vp_mlp_train_kick(const float* f_in, const float* target, int64_t n_outer, int64_t n_line,
                      int64_t n_inner, const double* E, int64_t e_div, double dt, double dv,
                      const void* net, double inv_scale, float* grad, double* loss, int32_t* status,
                      void* stream);

#ifdef __cplusplus
}
#endif
#endif /* VLASOV_B200_H */
