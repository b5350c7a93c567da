/*
 * Body of the CPU oracle, instantiated once per real type (REAL / SFX are
 * defined by vp_oracle.c before each inclusion).
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product links or calls this code;
 * it is the checker the CUDA kernels are compared against, and the timed CPU
 * baseline of bench.py.
 *
 * Every routine restates one function of the reference's PyTorch solver
 * (simulations/vlasov2d_2v/pytorch/src/vlasov2D2V.py and
 * simulations/vlasov1d_1v/pytorch/src/vlasov1D1V.py) with the same operation
 * order and the same working precision, so that an FP64 run reproduces the
 * reference to round-off and an FP32 run follows the reference's own FP32
 * arithmetic (multiply then add, no fused multiply-add: build with
 * -ffp-contract=off).
 *
 * Layout convention shared with the CUDA library: an N-d contiguous array is
 * viewed as [n_outer][n_line][n_inner] where n_line is the advected axis.
 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)

/* Lagrange 6-point weights, reference vlasov2D2V.py:263-285
 * (lagrange5_weights) - the same closed-form polynomials evaluated left to
 * right, each product and quotient rounded in REAL. */
static inline void CAT(lag5_, SFX)(REAL a, REAL w[6]) {
    REAL a2 = a * a;
    REAL a3 = a2 * a;
    REAL a4 = a3 * a;
    REAL a5 = a4 * a;
    w[0] = (a / (REAL)20.0) - (a2 / (REAL)24.0) - (a3 / (REAL)24.0) + (a4 / (REAL)24.0) - (a5 / (REAL)120.0);
    w[1] = -(a / (REAL)2.0) + ((REAL)2.0 * a2 / (REAL)3.0) - (a3 / (REAL)24.0) - (a4 / (REAL)6.0) + (a5 / (REAL)24.0);
    w[2] = (REAL)1.0 - (a / (REAL)3.0) - ((REAL)5.0 * a2 / (REAL)4.0) + ((REAL)5.0 * a3 / (REAL)12.0) + (a4 / (REAL)4.0) - (a5 / (REAL)12.0);
    w[3] = a + ((REAL)2.0 * a2 / (REAL)3.0) - ((REAL)7.0 * a3 / (REAL)12.0) - (a4 / (REAL)6.0) + (a5 / (REAL)12.0);
    w[4] = -(a / (REAL)4.0) - (a2 / (REAL)24.0) + ((REAL)7.0 * a3 / (REAL)24.0) + (a4 / (REAL)24.0) - (a5 / (REAL)24.0);
    w[5] = (a / (REAL)30.0) - (a3 / (REAL)24.0) + (a5 / (REAL)120.0);
}

void CAT(or_lagrange5_weights_, SFX)(const REAL* alpha, int64_t n, REAL* w /* [6][n] */) {
    for (int64_t i = 0; i < n; ++i) {
        REAL t[6];
        CAT(lag5_, SFX)(alpha[i], t);
        for (int k = 0; k < 6; ++k) w[k * n + i] = t[k];
    }
}

/* Periodic drift with per-velocity static shift and weights.
 * Reference: advect_x_static, vlasov2D2V.py:756-819 (and vlasov1D1V.py:408-448):
 *   out = 0; for k: out = out + f[(i - s_j - o_k) mod N] * W[k, j]
 * with o_k = k - 2. The table index of column c is j = (c / sel_div) % sel_mod. */
void CAT(or_drift_static_, SFX)(const REAL* in, REAL* out, int64_t n_outer, int64_t n_line,
                                int64_t n_inner, int64_t sel_div, int64_t sel_mod,
                                const int64_t* shift, const REAL* W /* [6][sel_mod] */) {
    /* Columns with the same table entry j form runs of sel_div contiguous
     * elements; per output row the 6 source rows of each j are resolved
     * once, and the arithmetic of every element is the reference's. */
    const int64_t period = sel_div * sel_mod;
    const int blocked = (n_inner % period) == 0;
#pragma omp parallel
    {
        int64_t* rows = (int64_t*)malloc(sizeof(int64_t) * 6 * (size_t)sel_mod);
#pragma omp for collapse(2) schedule(static)
        for (int64_t o = 0; o < n_outer; ++o) {
            for (int64_t l = 0; l < n_line; ++l) {
                const REAL* src = in + o * n_line * n_inner;
                REAL* dst = out + (o * n_line + l) * n_inner;
                for (int64_t j = 0; j < sel_mod; ++j) {
                    for (int k = 0; k < 6; ++k) {
                        int64_t r = (l - shift[j] - (k - 2)) % n_line;
                        rows[j * 6 + k] = (r < 0 ? r + n_line : r) * n_inner;
                    }
                }
                if (blocked) {
                    for (int64_t q = 0; q < n_inner; q += period) {
                        for (int64_t j = 0; j < sel_mod; ++j) {
                            const int64_t* rj = rows + j * 6;
                            const REAL w0 = W[0 * sel_mod + j], w1 = W[1 * sel_mod + j], w2 = W[2 * sel_mod + j];
                            const REAL w3 = W[3 * sel_mod + j], w4 = W[4 * sel_mod + j], w5 = W[5 * sel_mod + j];
                            const int64_t c0 = q + j * sel_div;
                            const REAL *s0 = src + rj[0], *s1 = src + rj[1], *s2 = src + rj[2];
                            const REAL *s3 = src + rj[3], *s4 = src + rj[4], *s5 = src + rj[5];
                            for (int64_t c = c0; c < c0 + sel_div; ++c) {
                                REAL acc = (REAL)0;
                                acc = acc + s0[c] * w0;
                                acc = acc + s1[c] * w1;
                                acc = acc + s2[c] * w2;
                                acc = acc + s3[c] * w3;
                                acc = acc + s4[c] * w4;
                                acc = acc + s5[c] * w5;
                                dst[c] = acc;
                            }
                        }
                    }
                } else {
                    for (int64_t c = 0; c < n_inner; ++c) {
                        const int64_t j = (c / sel_div) % sel_mod;
                        REAL acc = (REAL)0;
                        for (int k = 0; k < 6; ++k) acc = acc + src[rows[j * 6 + k] + c] * W[k * sel_mod + j];
                        dst[c] = acc;
                    }
                }
            }
        }
        free(rows);
    }
}

/* Dirichlet kick with a per-point field E.
 * Reference: build_v_tap_weights + advect_v_static, vlasov2D2V.py:822-913
 * (vlasov1D1V.py:450-501): d = (E*dt)/dv, s = floor(d), alpha = d - s,
 * W6 = lagrange5_weights(alpha); the taps m = s + o_k inside the static window
 * [-S-2, S+2] are summed in ascending m over the zero-padded line.
 * window < 0 keeps every tap (exact kick for any |d|; equals the reference
 * whenever |d| < S). E index of outer row o is o / e_div. */
void CAT(or_kick_static_, SFX)(const REAL* in, REAL* out, int64_t n_outer, int64_t n_line,
                               int64_t n_inner, const REAL* E, int64_t e_div, double dt,
                               double dv, int64_t window) {
#pragma omp parallel for schedule(static)
    for (int64_t o = 0; o < n_outer; ++o) {
        REAL d = (E[o / e_div] * (REAL)dt) / (REAL)dv;
        REAL sf = (REAL)floor((double)d);
        REAL alpha = d - sf;
        int64_t s = (int64_t)sf;
        REAL w[6];
        CAT(lag5_, SFX)(alpha, w);
        const REAL* src = in + o * n_line * n_inner;
        REAL* dst = out + o * n_line * n_inner;
        for (int64_t l = 0; l < n_line; ++l) {
            REAL* drow = dst + l * n_inner;
            for (int64_t c = 0; c < n_inner; ++c) drow[c] = (REAL)0;
            /* taps in ascending order; a tap outside the line reads the zero
             * padding and leaves every element unchanged */
            for (int k = 0; k < 6; ++k) {
                const int64_t m = s + (k - 2);
                if (window >= 0 && (m < -window - 2 || m > window + 2)) continue;
                const int64_t r = l - m;
                if (r < 0 || r >= n_line) continue;
                const REAL* srow = src + r * n_inner;
                const REAL wk = w[k];
                for (int64_t c = 0; c < n_inner; ++c) drow[c] = drow[c] + wk * srow[c];
            }
        }
    }
}

/* General semi-Lagrangian sweep with a per-element departure point.
 * Reference: advect_1d_vectorized, vlasov2D2V.py:287-353 (vlasov1D1V.py:212-256):
 *   depart = i - (v*dt)/dx, idx = floor(depart), alpha = depart - idx,
 *   taps idx + o_k (mod N, or clamped and masked to zero), then
 *   lagrange5_interp_sum: w0*g0 + w1*g1 + ... + w5*g5 left to right.
 * The velocity of element (o, l, c) is vel[o*vso + l*vsl + c*vsc]. */
void CAT(or_advect_gather_, SFX)(const REAL* in, REAL* out, int64_t n_outer, int64_t n_line,
                                 int64_t n_inner, const REAL* vel, int64_t vso, int64_t vsl,
                                 int64_t vsc, double dt, double dx, int periodic) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t o = 0; o < n_outer; ++o) {
        for (int64_t l = 0; l < n_line; ++l) {
            const REAL* src = in + o * n_line * n_inner;
            REAL* dst = out + (o * n_line + l) * n_inner;
            for (int64_t c = 0; c < n_inner; ++c) {
                REAL v = vel[o * vso + l * vsl + c * vsc];
                REAL disp = (v * (REAL)dt) / (REAL)dx;
                REAL depart = (REAL)l - disp;
                REAL fl = (REAL)floor((double)depart);
                REAL a = depart - fl;
                int64_t il = (int64_t)fl;
                REAL g[6];
                for (int k = 0; k < 6; ++k) {
                    int64_t r = il + (k - 2);
                    if (periodic) {
                        r %= n_line;
                        if (r < 0) r += n_line;
                        g[k] = src[r * n_inner + c];
                    } else {
                        int valid = (r >= 0 && r < n_line);
                        int64_t rc = r < 0 ? 0 : (r > n_line - 1 ? n_line - 1 : r);
                        g[k] = src[rc * n_inner + c] * (valid ? (REAL)1 : (REAL)0);
                    }
                }
                REAL w[6];
                CAT(lag5_, SFX)(a, w);
                dst[c] = w[0] * g[0] + w[1] * g[1] + w[2] * g[2] + w[3] * g[3] + w[4] * g[4] + w[5] * g[5];
            }
        }
    }
}

/* Charge density. Reference: compute_rho, vlasov2D2V.py:416-431
 * (sum over the trailing n_v elements, then * dvx * dvy); the 1D1V form
 * (vlasov1D1V.py:521) passes dvy = 1. The sum is accumulated in FP64 and
 * rounded to REAL once, as a stand-in for torch's pairwise reduction. */
void CAT(or_rho_, SFX)(const REAL* f, int64_t n_xy, int64_t n_v, double dvx, double dvy,
                       REAL* rho) {
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n_xy; ++p) {
        double s = 0.0;
        const REAL* src = f + p * n_v;
        for (int64_t c = 0; c < n_v; ++c) s += (double)src[c];
        REAL r = (REAL)s;
        r = r * (REAL)dvx;
        r = r * (REAL)dvy;
        rho[p] = r;
    }
}

#undef CAT
#undef CAT2
