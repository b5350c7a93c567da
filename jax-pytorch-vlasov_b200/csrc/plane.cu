// Two drifts in the (x, y) plane of f[x][y][vx][vy] in one pass over HBM.
//
// The position half-steps of the Strang step come in pairs: x then y before
// the field solve (the y drift also yields the charge density), y then x
// after the kick. As two sweeps, each pair writes and re-reads a full
// intermediate copy of f; this kernel keeps the intermediate on chip.
//
//  * A CTA owns a group of 32 consecutive columns of the (vx, vy) plane
//    (lane <-> column; the group sits inside one vx, so it shares one x
//    shift) over all y, 8 y rows per thread, and walks x.
//  * Each x row of the group (ny rows of 32 contiguous floats, 128 B) comes
//    in as one TMA box into a ring of DEPTH shared-memory slabs, completion
//    on one mbarrier per slab (waits are bounded). x first stages its output
//    rows in shared memory (its density sums read them there) and writes
//    them by TMA stores; y first stores them from registers (a warp writes
//    128 contiguous bytes per row) and needs a block barrier only to hand
//    back slabs, which it does every second row.
//  * The x drift is a 6-row sliding window in registers. The y drift (shift
//    per vy, i.e. per lane) reads 13 consecutive rows of a whole row plane
//    in shared memory: the slab itself (y first) or a double-buffered plane
//    of x-drifted rows (x first). Slabs and planes carry 16 halo rows after
//    row ny (copies of rows 0..15), so the periodic window never wraps.
//  * The row loop is unrolled by DEPTH = 6 = the window length, so ring
//    slots, buffer parities and window registers are fixed per unrolled
//    step; pairs of y rows go through the paired FP32 FMA of sm_100.
//  * Every element goes through the same FMA chain as in the single-axis
//    sweep (k_strided: round(w5 g5), then fma down to tap 0) and the
//    intermediate is kept in FP32 as that sweep stores it, so f is
//    bit-identical to the two-sweep path.
//  * x first runs its y drift one row behind the x drift (the plane of row
//    k is complete at the barrier of step k), so every row costs one
//    barrier. It can also sum each output row over its 32 columns in FP64
//    (from the staged output, one step later still: four threads per y row,
//    8 columns each, then two shuffles) into per-group partials of the
//    charge density, [nx][groups][ny], reduced in a fixed order by
//    k_rho_finalize_wide.
//  * Above 112 rows the x-first pair runs as k_plane_xr instead: 16 y rows
//    per thread, the x window of the 21 rows its y drift reads kept in
//    registers (the 5 rows past a warp's own are recomputed), so neither a
//    plane exchange nor a per-row barrier is needed; same partials layout.
//  * Equilibrium split (EQ; the state holds g = f - A(vx) B(vy)): each drift
//    adds the per-column constant feq * (sum of the column's 6 weights - 1)
//    after its 6 taps, in the same operations as the single-axis sweep, so
//    the split passes stay bit-identical to the split sweeps.
// A wait that runs out (1 s) makes the CTA wait for its stores, fill its
// whole share of the output (and its density partials) with NaN, wait
// (bounded) for its loads in flight and leave, so a failure shows in the
// results.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>
#include <cmath>

#include "common.cuh"
#include "launch.h"

namespace vp {
namespace plane {

constexpr int CG = 32;                   // columns per group (= lanes)
constexpr int YT = 8;                    // y rows per thread
constexpr int MAXW = 16;                 // warps per CTA
constexpr int YMAX = MAXW * YT;          // ny <= 128
constexpr int YMIN = 16;                 // ny >= 16: the halo copies 16 real rows
constexpr int DEPTH = 6;                 // slabs in flight = unroll of the row loop
constexpr int HALO = 16;                 // rows after row ny: copies of rows 0..15
// floats per slab or plane, and per output staging buffer, of a kernel
// built for at most ym rows (64 or 128: two CTAs or one per SM)
__host__ __device__ constexpr int buf_floats(int ym) { return (ym + HALO) * CG; }
__host__ __device__ constexpr int stage_floats(int ym) { return ym * CG; }

struct Args {
    float* out;
    int nx, ny, nvx, nvy;
    int xb, xc;         // the output rows: xb .. xb + xc - 1 (all: 0, nx)
    int64_t m;          // columns per (x, y) point: nvx * nvy
    int n_cg;           // column groups: m / CG
    const int* shift_x;
    const float* W_x;   // [6][nvx] tap weights
    const int* shift_y;
    const float* W_y;   // [6][nvy]
    double* part;       // [nx][n_cg][ny] FP64 row sums (x first with the density)
    const double* eqA;  // equilibrium split feq = eqA[vx] * eqB[vy] (EQ kernels)
    const double* eqB;
    int* status;        // optional: VP_STATUS_WAIT_TIMEOUT ORed in by a CTA whose wait ran out
    int stall;          // test hook: the first load of each CTA expects 16 bytes too many
};

// The rows a CTA loads. Work comes in segments (one group, output rows
// xa .. xa+n-1 of the launch's range xb .. xb+xc-1; a line is the whole
// range), each loading the rows xa - s - 3 + q, q = 0 .. n + 4, of its group
// (s: the group's x shift; rows wrap around nx). CTA b of G first takes whole lines of
// the groups b, b + G, b + 2G, ... (neighbouring groups then stream the same
// x rows at the same time, so HBM sees long runs of each (x, y) point's
// columns), then an even share of the rows of the n_cg % G groups left.
struct Seq {
    int w, full, b, G;  // whole-line rounds: done, total; this CTA; CTAs
    int t, t1;          // share of the remaining lines' rows (n_cg * xc < 2^31)
    int cg, xa, n, q, r0;
    __device__ __forceinline__ void init(const Args& a, int b_, int G_) {
        b = b_;
        G = G_;
        full = a.n_cg / G;
        w = 0;
        const int64_t rest = (int64_t)(a.n_cg - full * G) * a.xc;
        t = (int)(rest * b / G);
        t1 = (int)(rest * (b + 1) / G);
        if (valid()) start(a);
    }
    __device__ __forceinline__ void start(const Args& a) {
        if (w < full) {
            cg = w * G + b;
            xa = a.xb;
            n = a.xc;
        } else {
            cg = full * G + t / a.xc;
            const int o = t % a.xc;
            xa = a.xb + o;
            n = min(t1 - t, a.xc - o);
        }
        const int jx = (cg * CG / a.nvy) % a.nvx;
        r0 = xa - __ldg(a.shift_x + jx) - 3;
        q = 0;
    }
    __device__ __forceinline__ bool valid() const { return w < full || t < t1; }
    __device__ __forceinline__ int row(int nx) const {
        const int r = (r0 + q) % nx;
        return r < 0 ? r + nx : r;
    }
    __device__ __forceinline__ void next(const Args& a) {
        if (__builtin_expect(++q == n + 5, 0)) {
            if (w < full)
                ++w;
            else
                t += n;
            if (valid()) start(a);
        }
    }
};

// producer state in shared memory (only thread 0 touches it)
struct Producer {
    Seq seq;
    long long issued;
};

template <int P> struct Step { static constexpr int value = P; };

__device__ __forceinline__ void bar_init(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void expect_bytes(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// box at (column c0, row r0) of the [nx*ny][m] view of f into dst
__device__ __forceinline__ void tma_load(const CUtensorMap* tm, uint32_t dst, uint32_t bar, int c0, int r0) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(r0), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma_store(const CUtensorMap* tm, uint32_t src, int c0, int r0) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                     reinterpret_cast<uint64_t>(tm)),
                 "r"(c0), "r"(r0), "r"(src)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// the bulk stores issued so far have read their shared memory / are done
__device__ __forceinline__ void stores_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void stores_done() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// mbarrier phase wait that sleeps between polls; false after ~1 s
__device__ __forceinline__ bool wait_phase(uint32_t bar, uint32_t parity) {
    const uint64_t t0 = now_ns();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity), "r"(20000u)
            : "memory");
        if (ok) return true;
        if (now_ns() - t0 > 1000000000ull) return false;
    }
}

// 6-tap drift of a pair of rows: round(w5 t5), then fma down to tap 0
__device__ __forceinline__ float2 taps(const float2 (&w)[6], float2 t0, float2 t1, float2 t2, float2 t3, float2 t4,
                                       float2 t5) {
    float2 acc = __fmul2_rn(w[5], t5);
    acc = __ffma2_rn(w[4], t4, acc);
    acc = __ffma2_rn(w[3], t3, acc);
    acc = __ffma2_rn(w[2], t2, acc);
    acc = __ffma2_rn(w[1], t1, acc);
    return __ffma2_rn(w[0], t0, acc);
}

// the split's constant after the taps (a plain FP32 add per row, as the
// single-axis sweep adds it)
template <bool EQ>
__device__ __forceinline__ float2 plus(float2 o, float b) {
    if constexpr (EQ) {
        o.x += b;
        o.y += b;
    }
    return o;
}

// the split's constant of a lane's column: feq * (sum of its 6 weights - 1),
// the weights summed from tap 5 down to tap 0 in FP64, rounded once
__device__ __forceinline__ float split_bias(double feq, const float2 (&w)[6]) {
    double s = -1.0;
#pragma unroll
    for (int j = 0; j < 6; ++j) s += (double)w[j].x;
    return (float)(feq * s);
}

// y drift of the thread's 8 rows from 13 consecutive rows of a buffer
// (g: row y0 - s - 3 of the lane's column, halo included)
template <bool EQ>
__device__ __forceinline__ void y_drift(const float* g, const float2 (&wy)[6], float by, float2 (&o)[YT / 2]) {
    float r[YT + 5];
#pragma unroll
    for (int k = 0; k < YT + 5; ++k) r[k] = g[k * CG];
#pragma unroll
    for (int p = 0; p < YT / 2; ++p) {
        const int i = 2 * p;
        o[p] = plus<EQ>(taps(wy, make_float2(r[i], r[i + 1]), make_float2(r[i + 1], r[i + 2]),
                             make_float2(r[i + 2], r[i + 3]), make_float2(r[i + 3], r[i + 4]),
                             make_float2(r[i + 4], r[i + 5]), make_float2(r[i + 5], r[i + 6])),
                        by);
    }
}

// FULL: ny is a multiple of 8, every thread row is a real row.
// YM: the most rows the buffers hold (ny <= YM); 64 halves the shared memory
// so that two CTAs share an SM.
template <bool XFIRST, bool RHO, bool FULL, int YM, bool EQ>
__global__ void __launch_bounds__(YM / YT * 32, YMAX / YM)
    k_plane(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap thalo,
            const __grid_constant__ CUtensorMap tout, const __grid_constant__ Args a) {
    static_assert(!RHO || XFIRST, "the density comes with the x-first order");
    constexpr int BUF = buf_floats(YM), STG = stage_floats(YM);
    extern __shared__ __align__(1024) unsigned char smem[];
    float* slabs = reinterpret_cast<float*>(smem);  // [DEPTH][BUF]
    float* stage = slabs + DEPTH * BUF;             // [2][STG] (x first)
    float* planes = stage + (XFIRST ? 2 * STG : 0); // [2][BUF] (x first)
    uint64_t* bars = reinterpret_cast<uint64_t*>(planes + (XFIRST ? 2 * BUF : 0));
    Producer* prod = reinterpret_cast<Producer*>(bars + DEPTH);
    const int nx = a.nx, ny = a.ny;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int y0 = warp * YT;
    Seq cons;
    cons.init(a, blockIdx.x, gridDim.x);
    if (!cons.valid()) return;
    const uint32_t slab0 = smem_u32(slabs), stage0 = smem_u32(stage), bar0 = smem_u32(bars);
    const uint32_t in_bytes = (uint32_t)((ny + (XFIRST ? 0 : HALO)) * CG * 4);
    // the producer's current row into slab d
    uint32_t extra = a.stall ? 16u : 0u;  // test hook, first load only
    auto issue = [&](int d, const Seq& s) {
        const uint32_t dst = slab0 + (uint32_t)(d * BUF * 4), bar = bar0 + 8 * d;
        const int r = s.row(nx) * ny;
        expect_bytes(bar, in_bytes + extra);
        tma_load(&tin, dst, bar, s.cg * CG, r);
        if constexpr (!XFIRST) tma_load(&thalo, dst + (uint32_t)(ny * CG * 4), bar, s.cg * CG, r);
    };
    if (tid == 0) {
        for (int d = 0; d < DEPTH; ++d) bar_init(bar0 + 8 * d);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        Seq p = cons;
        long long n = 0;
        for (; n < DEPTH && p.valid(); ++n) {
            issue((int)n, p);
            extra = 0;
            p.next(a);
        }
        prod->seq = p;
        prod->issued = n;
    }
    __syncthreads();

    float2 win[YT / 2][6];
#pragma unroll
    for (int p = 0; p < YT / 2; ++p)
#pragma unroll
        for (int s = 0; s < 6; ++s) win[p][s] = make_float2(0.f, 0.f);
    float2 wx[6], wy[6];
    float bx = 0.f, by = 0.f;  // the split's constants of the lane's column (EQ)
    int yoff = 0;           // float offset of row y0 - sy - 3 (mod ny), column lane
    uint32_t parity = 0;    // of the current pass over the ring
    long long L = 0;        // loads consumed
    bool pend = false;      // x first: a row waiting for its y drift
    int pend_x = 0, pend_cg = 0;
    bool failed = false;
    bool okacc = true;  // y first: waits since the last barrier all ended
    int last = 0;

    // x first: y drift of the pending row from plane PL into stage PL
    auto y_pending = [&](auto pl) {
        constexpr int PL = decltype(pl)::value;
        float2 o[YT / 2];
        y_drift<EQ>(planes + PL * BUF + yoff, wy, by, o);
        float* st = stage + PL * STG;
#pragma unroll
        for (int p = 0; p < YT / 2; ++p) {
            const int y = y0 + 2 * p;
            if (FULL || y < ny) st[y * CG + lane] = o[p].x;
            if (FULL || y + 1 < ny) st[(y + 1) * CG + lane] = o[p].y;
        }
    };
    // x first: density partials of row rx of group rcg from its complete
    // stage SP (thread: y row tid / 4, columns 8 (tid % 4) .. + 7)
    const int rrow = tid >> 2, rq = tid & 3;
    auto rho_row = [&](auto sp, bool on, int rx, int rcg) {
        constexpr int SP = decltype(sp)::value;
        const float4* src = reinterpret_cast<const float4*>(stage + SP * STG + rrow * CG) + 2 * rq;
        // odd rows read their second chunk first: neighbouring rows then
        // never hit the same banks
        const int odd = rrow & 1;
        const float4 u = src[odd], v = src[1 - odd];
        const double s = (((double)u.x + (double)u.y) + ((double)u.z + (double)u.w)) +
                         (((double)v.x + (double)v.y) + ((double)v.z + (double)v.w));
        double t = s + __shfl_xor_sync(0xffffffffu, s, 1);
        t += __shfl_xor_sync(0xffffffffu, t, 2);
        if (on && rq == 0 && rrow < ny) a.part[((int64_t)rx * a.n_cg + rcg) * ny + rrow] = t;
    };
    bool rho_on = false;    // x first: a stored row waiting for its density
    int rho_x = 0, rho_cg = 0;

    // the weights and y window of the consumer's current group
    auto tables = [&]() {
        const int jx = (int)(((int64_t)cons.cg * CG / a.nvy) % a.nvx);
        const int jy = (int)(((int64_t)cons.cg * CG) % a.nvy) + lane;
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            const float u = __ldg(a.W_x + (5 - j) * a.nvx + jx), v = __ldg(a.W_y + (5 - j) * a.nvy + jy);
            wx[j] = make_float2(u, u);
            wy[j] = make_float2(v, v);
        }
        if constexpr (EQ) {
            const double feq = __ldg(a.eqA + jx) * __ldg(a.eqB + jy);
            bx = split_bias(feq, wx);
            by = split_bias(feq, wy);
        }
        int r = (y0 - __ldg(a.shift_y + jy) - 3) % ny;
        if (r < 0) r += ny;
        yoff = r * CG + lane;
    };
    tables();

    auto body = [&](auto step) -> bool {
        constexpr int P = decltype(step)::value;
        if constexpr (XFIRST) {
            // both unconditional (their buffers are free when nothing is
            // pending); only the writes that leave the CTA are predicated
            if constexpr (RHO) rho_row(Step<P & 1>{}, rho_on, rho_x, rho_cg);
            y_pending(Step<(P + 1) & 1>{});
        }
        const bool ok = wait_phase(bar0 + 8 * P, parity);
        const bool emit = cons.q >= 5;
        const float* sl = slabs + P * BUF;
        float2 nv[YT / 2];
        if constexpr (XFIRST) {
            // x drift: window slots hold loads L-5 .. L-1, the new row is L
#pragma unroll
            for (int p = 0; p < YT / 2; ++p)
                nv[p] = make_float2(sl[(y0 + 2 * p) * CG + lane], sl[(y0 + 2 * p + 1) * CG + lane]);
            {  // unconditional: a plane written without output is never read
                float* pl = planes + (P & 1) * BUF;
#pragma unroll
                for (int p = 0; p < YT / 2; ++p) {
                    const float2 o = plus<EQ>(taps(wx, win[p][(P + 1) % 6], win[p][(P + 2) % 6], win[p][(P + 3) % 6],
                                                   win[p][(P + 4) % 6], win[p][(P + 5) % 6], nv[p]),
                                              bx);
                    const int y = y0 + 2 * p;
                    if (FULL || y < ny) pl[y * CG + lane] = o.x;
                    if (FULL || y + 1 < ny) pl[(y + 1) * CG + lane] = o.y;
                    if (y0 < HALO) {  // warp-uniform: the rows copied after row ny
                        pl[(ny + y) * CG + lane] = o.x;
                        pl[(ny + y + 1) * CG + lane] = o.y;
                    }
                }
            }
        } else {
            // y drift of the new row from its slab, then the x drift
            y_drift<EQ>(sl + yoff, wy, by, nv);
            if (emit) {
                float* dst = a.out + ((int64_t)(cons.xa + cons.q - 5) * ny + y0) * a.m + (int64_t)cons.cg * CG + lane;
#pragma unroll
                for (int p = 0; p < YT / 2; ++p) {
                    const float2 o = plus<EQ>(taps(wx, win[p][(P + 1) % 6], win[p][(P + 2) % 6], win[p][(P + 3) % 6],
                                                   win[p][(P + 4) % 6], win[p][(P + 5) % 6], nv[p]),
                                              bx);
                    const int y = y0 + 2 * p;
                    if (FULL || y < ny) dst[(int64_t)(2 * p) * a.m] = o.x;
                    if (FULL || y + 1 < ny) dst[(int64_t)(2 * p + 1) * a.m] = o.y;
                }
            }
        }
#pragma unroll
        for (int p = 0; p < YT / 2; ++p) win[p][P] = nv[p];
        if constexpr (XFIRST) {
        // staged rows become visible to the TMA store; the previous store
        // has read its stage before that buffer is written again
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (tid == 0) stores_read();
        if (__syncthreads_or(!ok)) {
            failed = true;
            return false;
        }
        if (P == DEPTH - 1) parity ^= 1u;
        ++L;
        if (tid == 0) {
            if (pend) tma_store(&tout, stage0 + (uint32_t)(((P + 1) & 1) * STG * 4), pend_cg * CG, pend_x * ny);
            Seq& p = prod->seq;
            if (p.valid()) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue(P, p);
                p.next(a);
                prod->issued += 1;
            }
        }
        } else {
            okacc = okacc && ok;
            if (P & 1) {  // slabs P-1 and P are free once every warp is past both
                if (__syncthreads_or(!okacc)) {
                    failed = true;
                    return false;
                }
                if (tid == 0) {
                    Seq& p = prod->seq;
#pragma unroll
                    for (int d = P - 1; d <= P; ++d)
                        if (p.valid()) {
                            issue(d, p);
                            p.next(a);
                            prod->issued += 1;
                        }
                }
            }
            if (P == DEPTH - 1) parity ^= 1u;
            ++L;
        }
        if constexpr (XFIRST) {
            rho_on = pend;
            rho_x = pend_x;
            rho_cg = pend_cg;
            pend = emit;
            pend_x = cons.xa + cons.q - 5;
            pend_cg = cons.cg;
        }
        cons.next(a);
        last = P;
        // a new group: its tables after the pending row of the last one
        // went through (x first: one step into the group, before any
        // output row; y first: before its first row)
        if (cons.valid() && cons.q == (XFIRST ? 1 : 0)) tables();
        return cons.valid();
    };

    while (body(Step<0>{}) && body(Step<1>{}) && body(Step<2>{}) && body(Step<3>{}) && body(Step<4>{}) &&
           body(Step<5>{})) {
    }
    if constexpr (!XFIRST) {
        // a wait on a last, even row has had no barrier vote yet
        if (!failed && __syncthreads_or(!okacc)) failed = true;
    }

    if constexpr (XFIRST) {
        if (!failed) {
            // the rows still in the pipeline: the density of the row stored
            // at the last step, then the last row (its plane is complete)
            if (RHO) {
                if (last & 1)
                    rho_row(Step<0>{}, rho_on, rho_x, rho_cg);
                else
                    rho_row(Step<1>{}, rho_on, rho_x, rho_cg);
            }
            if (pend) {
                if (last & 1)
                    y_pending(Step<1>{});
                else
                    y_pending(Step<0>{});
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                if (tid == 0) stores_read();
                __syncthreads();
                if (tid == 0) tma_store(&tout, stage0 + (uint32_t)((last & 1) * STG * 4), pend_cg * CG, pend_x * ny);
                if (RHO) {
                    if (last & 1)
                        rho_row(Step<1>{}, true, pend_x, pend_cg);
                    else
                        rho_row(Step<0>{}, true, pend_x, pend_cg);
                }
            }
        }
    }
    if (tid == 0) stores_done();
    if (failed) {
        // no store lands after this point: the whole share reads NaN, then
        // the loads in flight land
        __syncthreads();
        Seq z;
        z.init(a, blockIdx.x, gridDim.x);
        while (z.valid()) {
            if (z.q >= 5) {
                const int x = z.xa + z.q - 5;
                for (int i = 0; i < YT && y0 + i < ny; ++i) {
                    a.out[((int64_t)x * ny + y0 + i) * a.m + (int64_t)z.cg * CG + lane] = NAN;
                    if (RHO && lane == 0) a.part[((int64_t)x * a.n_cg + z.cg) * ny + y0 + i] = (double)NAN;
                }
            }
            z.next(a);
        }
        if (tid == 0) {
            if (a.status) atomicOr(a.status, VP_STATUS_WAIT_TIMEOUT);
            for (long long k = L; k < prod->issued; ++k)
                wait_phase(bar0 + 8 * (int)(k % DEPTH), (uint32_t)((k / DEPTH) & 1));
        }
    }
}

// ---- x then y with the x window in registers --------------------------------
// The x-first pair without a plane exchange: a thread owns 16 y rows and
// keeps the x window of the 21 rows its y drift reads (its 16 rows shifted by
// its lane's y shift, plus the 5 more the 6 taps reach; neighbouring warps
// recompute the x drift of those 5 rows for themselves). Slabs carry 20 halo
// rows, the x-drifted rows stay in registers for the y drift, outputs leave
// from registers (a warp writes 128 contiguous bytes per row), and a block
// barrier is needed only to hand back slabs, every second row, as in the
// y-first kernel. The density sums each output row over the group's 32
// columns in FP64 with a butterfly reduce-scatter over the warp's lanes.
// The FMA chains are those of k_plane, so f is bit-identical to it.
constexpr int YT2 = 16;             // y rows per thread
constexpr int WR = YT2 + 5;         // rows of the x window per thread
constexpr int HALO2 = 20;           // rows after row ny: copies of rows 0..19
__host__ __device__ constexpr int buf2_floats(int ym) { return (ym + HALO2) * CG; }

// the 6-tap chain of taps() for one row
__device__ __forceinline__ float tap1(const float2 (&w)[6], float t0, float t1, float t2, float t3, float t4,
                                      float t5) {
    float acc = __fmul_rn(w[5].x, t5);
    acc = __fmaf_rn(w[4].x, t4, acc);
    acc = __fmaf_rn(w[3].x, t3, acc);
    acc = __fmaf_rn(w[2].x, t2, acc);
    acc = __fmaf_rn(w[1].x, t1, acc);
    return __fmaf_rn(w[0].x, t0, acc);
}

// density staging: per warp and buffer, 16 rows of 32 columns, rows padded
// to 36 floats so that the 16-byte reads of 8 lanes (4 rows, 2 halves) hit
// distinct banks
constexpr int RSTRIDE = CG + 4;
constexpr int RFLOATS = YT2 * RSTRIDE;

template <bool RHO, bool FULL, int YM, bool EQ>
__global__ void __launch_bounds__(YM / YT2 * 32, YMAX / YM)
    k_plane_xr(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap thalo,
               const __grid_constant__ Args a) {
    constexpr int BUF = buf2_floats(YM), NW = YM / YT2;
    extern __shared__ __align__(1024) unsigned char smem[];
    float* slabs = reinterpret_cast<float*>(smem);  // [DEPTH][BUF]
    float* red = slabs + DEPTH * BUF;               // [2][NW][RFLOATS] (density)
    uint64_t* bars = reinterpret_cast<uint64_t*>(red + (RHO ? 2 * NW * RFLOATS : 0));
    Producer* prod = reinterpret_cast<Producer*>(bars + DEPTH);
    const int nx = a.nx, ny = a.ny;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int y0 = warp * YT2;
    Seq cons;
    cons.init(a, blockIdx.x, gridDim.x);
    if (!cons.valid()) return;
    const uint32_t slab0 = smem_u32(slabs), bar0 = smem_u32(bars);
    const uint32_t in_bytes = (uint32_t)((ny + HALO2) * CG * 4);
    uint32_t extra = a.stall ? 16u : 0u;  // test hook, first load only
    auto issue = [&](int d, const Seq& s) {
        const uint32_t dst = slab0 + (uint32_t)(d * BUF * 4), bar = bar0 + 8 * d;
        const int r = s.row(nx) * ny;
        expect_bytes(bar, in_bytes + extra);
        tma_load(&tin, dst, bar, s.cg * CG, r);
        tma_load(&thalo, dst + (uint32_t)(ny * CG * 4), bar, s.cg * CG, r);
    };
    if (tid == 0) {
        for (int d = 0; d < DEPTH; ++d) bar_init(bar0 + 8 * d);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        Seq p = cons;
        long long n = 0;
        for (; n < DEPTH && p.valid(); ++n) {
            issue((int)n, p);
            extra = 0;
            p.next(a);
        }
        prod->seq = p;
        prod->issued = n;
    }
    __syncthreads();

    float2 win[WR / 2][6];  // rows 0..19 of the window, in pairs
    float wl[6];            // row 20
#pragma unroll
    for (int s = 0; s < 6; ++s) {
#pragma unroll
        for (int p = 0; p < WR / 2; ++p) win[p][s] = make_float2(0.f, 0.f);
        wl[s] = 0.f;
    }
    float2 wx[6], wy[6];
    float bx = 0.f, by = 0.f;  // the split's constants of the lane's column (EQ)
    int yoff = 0;  // float offset of row y0 - sy - 3 (mod ny), column lane
    uint32_t parity = 0;
    long long L = 0;
    bool failed = false, okacc = true;
    bool rho_on = false;  // a staged row waiting for its density
    int rho_x = 0, rho_cg = 0;
    // density of the row staged in buffer SP: lanes 2r and 2r + 1 add the
    // two halves of row r in FP64, then each other's sums
    auto rho_flush = [&](auto sp) {
        constexpr int SP = decltype(sp)::value;
        __syncwarp();
        const float4* src =
            reinterpret_cast<const float4*>(red + (SP * NW + warp) * RFLOATS + (lane >> 1) * RSTRIDE + (lane & 1) * 16);
        const float4 q0 = src[0], q1 = src[1], q2 = src[2], q3 = src[3];
        const double s0 = ((double)q0.x + (double)q0.y) + ((double)q0.z + (double)q0.w);
        const double s1 = ((double)q1.x + (double)q1.y) + ((double)q1.z + (double)q1.w);
        const double s2 = ((double)q2.x + (double)q2.y) + ((double)q2.z + (double)q2.w);
        const double s3 = ((double)q3.x + (double)q3.y) + ((double)q3.z + (double)q3.w);
        double t = (s0 + s1) + (s2 + s3);
        t += __shfl_xor_sync(0xffffffffu, t, 1);
        const int yr = y0 + (lane >> 1);
        if (rho_on && !(lane & 1) && yr < ny) a.part[((int64_t)rho_x * a.n_cg + rho_cg) * ny + yr] = t;
    };

    auto tables = [&]() {
        const int jx = (int)(((int64_t)cons.cg * CG / a.nvy) % a.nvx);
        const int jy = (int)(((int64_t)cons.cg * CG) % a.nvy) + lane;
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            const float u = __ldg(a.W_x + (5 - j) * a.nvx + jx), v = __ldg(a.W_y + (5 - j) * a.nvy + jy);
            wx[j] = make_float2(u, u);
            wy[j] = make_float2(v, v);
        }
        if constexpr (EQ) {
            const double feq = __ldg(a.eqA + jx) * __ldg(a.eqB + jy);
            bx = split_bias(feq, wx);
            by = split_bias(feq, wy);
        }
        int r = (y0 - __ldg(a.shift_y + jy) - 3) % ny;
        if (r < 0) r += ny;
        yoff = r * CG + lane;
    };
    tables();

    auto body = [&](auto step) -> bool {
        constexpr int P = decltype(step)::value;
        const bool ok = wait_phase(bar0 + 8 * P, parity);
        // the previous row's density goes along with this row's drifts
        if constexpr (RHO) rho_flush(Step<(P + 1) & 1>{});
        const float* sl = slabs + P * BUF + yoff;
        // the new row replaces the oldest (load L - 6) in slot P
#pragma unroll
        for (int p = 0; p < WR / 2; ++p) win[p][P] = make_float2(sl[(2 * p) * CG], sl[(2 * p + 1) * CG]);
        wl[P] = sl[(WR - 1) * CG];
        if (cons.q >= 5) {
            float xd[WR];
#pragma unroll
            for (int p = 0; p < WR / 2; ++p) {
                const float2 o = plus<EQ>(taps(wx, win[p][(P + 1) % 6], win[p][(P + 2) % 6], win[p][(P + 3) % 6],
                                               win[p][(P + 4) % 6], win[p][(P + 5) % 6], win[p][P]),
                                          bx);
                xd[2 * p] = o.x;
                xd[2 * p + 1] = o.y;
            }
            xd[WR - 1] = tap1(wx, wl[(P + 1) % 6], wl[(P + 2) % 6], wl[(P + 3) % 6], wl[(P + 4) % 6],
                              wl[(P + 5) % 6], wl[P]);
            if constexpr (EQ) xd[WR - 1] += bx;
            float o16[YT2];
#pragma unroll
            for (int p = 0; p < YT2 / 2; ++p) {
                const int i = 2 * p;
                const float2 o = plus<EQ>(taps(wy, make_float2(xd[i], xd[i + 1]), make_float2(xd[i + 1], xd[i + 2]),
                                               make_float2(xd[i + 2], xd[i + 3]), make_float2(xd[i + 3], xd[i + 4]),
                                               make_float2(xd[i + 4], xd[i + 5]), make_float2(xd[i + 5], xd[i + 6])),
                                          by);
                o16[i] = o.x;
                o16[i + 1] = o.y;
            }
            const int x = cons.xa + cons.q - 5;
            float* dst = a.out + ((int64_t)x * ny + y0) * a.m + (int64_t)cons.cg * CG + lane;
#pragma unroll
            for (int e = 0; e < YT2; ++e)
                if (FULL || y0 + e < ny) dst[(int64_t)e * a.m] = o16[e];
            if constexpr (RHO) {
                // stage the row for its density (rows past ny add zero)
                float* rb = red + ((P & 1) * NW + warp) * RFLOATS + lane;
                __syncwarp();
#pragma unroll
                for (int e = 0; e < YT2; ++e) rb[e * RSTRIDE] = (FULL || y0 + e < ny) ? o16[e] : 0.f;
                rho_x = x;
                rho_cg = cons.cg;
            }
        }
        if constexpr (RHO) rho_on = cons.q >= 5;
        okacc = okacc && ok;
        if (P & 1) {  // slabs P-1 and P are free once every warp is past both
            if (__syncthreads_or(!okacc)) {
                failed = true;
                return false;
            }
            if (tid == 0) {
                Seq& p = prod->seq;
#pragma unroll
                for (int d = P - 1; d <= P; ++d)
                    if (p.valid()) {
                        issue(d, p);
                        p.next(a);
                        prod->issued += 1;
                    }
            }
        }
        if (P == DEPTH - 1) parity ^= 1u;
        ++L;
        cons.next(a);
        if (cons.valid() && cons.q == 0) tables();
        return cons.valid();
    };

    while (body(Step<0>{}) && body(Step<1>{}) && body(Step<2>{}) && body(Step<3>{}) && body(Step<4>{}) &&
           body(Step<5>{})) {
    }
    // a wait on a last, even row has had no barrier vote yet
    if (!failed && __syncthreads_or(!okacc)) failed = true;
    if (RHO && !failed) {  // the density of the last row
        if (L & 1)
            rho_flush(Step<0>{});
        else
            rho_flush(Step<1>{});
    }
    if (failed) {
        // the whole share reads NaN, then the loads in flight land
        __syncthreads();
        Seq z;
        z.init(a, blockIdx.x, gridDim.x);
        while (z.valid()) {
            if (z.q >= 5) {
                const int x = z.xa + z.q - 5;
                for (int i = 0; i < YT2 && y0 + i < ny; ++i) {
                    a.out[((int64_t)x * ny + y0 + i) * a.m + (int64_t)z.cg * CG + lane] = NAN;
                    if (RHO && lane == 0) a.part[((int64_t)x * a.n_cg + z.cg) * ny + y0 + i] = (double)NAN;
                }
            }
            z.next(a);
        }
        if (tid == 0) {
            if (a.status) atomicOr(a.status, VP_STATUS_WAIT_TIMEOUT);
            for (long long k = L; k < prod->issued; ++k)
                wait_phase(bar0 + 8 * (int)(k % DEPTH), (uint32_t)((k / DEPTH) & 1));
        }
    }
}

// ---- x then y with the density on its own warpgroup ---------------------------
// The x-first pair of k_plane_xr for 113..128 rows when the density is wanted.
// Warps 0..7 (the drift warps, 16 y rows each) only stage every output row in
// shared memory next to its global store; warps 8..11 (the density warps, one
// thread per y row) sum each staged row over its 32 columns in FP64 and store
// the per-group partial. The FP64 conversions and sums thus run beside the
// drifts instead of inside their dependency chains. The block barrier that
// hands back slabs every second row also hands over the staged rows: rows of
// pair j are staged between barriers j-1 and j and summed between barriers j
// and j+1 while the drift warps stage pair j+1 into the other two slots.
// Registers: launched at 168 a thread (384 threads fill the register file);
// setmaxnreg then gives the drift warpgroups 216 and the density warpgroup 72
// (256 * 216 + 128 * 72 = 64512 = 384 * 168: the density warps' release
// covers the drift warps' increase exactly). Each role's code, its tail
// included, stays inside its own branch so that it is compiled to its own
// budget. The producer (TMA issue) is the first density thread.
constexpr int XRD_CW = 8;                // drift warps
constexpr int XRD_THREADS = 32 * (XRD_CW + 4);
constexpr int DSTRIDE = CG + 4;          // staged row: 32 floats + 4 of padding (conflict-free 16-byte reads)
constexpr int DSLOTS = 4;                // staged rows: two pairs
struct RowMeta {
    int x, cg, valid, pad;
};
__host__ __device__ constexpr size_t xrd_smem_bytes() {
    return (size_t)(DEPTH * buf2_floats(YMAX) + DSLOTS * YMAX * DSTRIDE) * 4 + DSLOTS * sizeof(RowMeta) + DEPTH * 8 +
           sizeof(Producer);
}

template <bool FULL, bool EQ>
__global__ void __launch_bounds__(XRD_THREADS, 1)
    k_plane_xrd(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap thalo,
                const __grid_constant__ Args a) {
    constexpr int YM = YMAX, BUF = buf2_floats(YM);
    extern __shared__ __align__(1024) unsigned char smem[];
    float* slabs = reinterpret_cast<float*>(smem);            // [DEPTH][BUF]
    float* stage = slabs + DEPTH * BUF;                        // [DSLOTS][YM][DSTRIDE]
    RowMeta* meta = reinterpret_cast<RowMeta*>(stage + DSLOTS * YM * DSTRIDE);
    uint64_t* bars = reinterpret_cast<uint64_t*>(meta + DSLOTS);
    Producer* prod = reinterpret_cast<Producer*>(bars + DEPTH);
    const int nx = a.nx, ny = a.ny;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool drift = warp < XRD_CW;
    constexpr int PTID = XRD_CW * 32;  // producer: the first density thread
    const int dy = tid - PTID;         // density thread: its y row
    const int y0 = warp * YT2;
    Seq cons;
    cons.init(a, blockIdx.x, gridDim.x);
    if (!cons.valid()) return;
    const uint32_t slab0 = smem_u32(slabs), bar0 = smem_u32(bars);
    const uint32_t in_bytes = (uint32_t)((ny + HALO2) * CG * 4);
    uint32_t extra = a.stall ? 16u : 0u;  // test hook, first load only
    auto issue = [&](int d, const Seq& s) {
        const uint32_t dst = slab0 + (uint32_t)(d * BUF * 4), bar = bar0 + 8 * d;
        const int r = s.row(nx) * ny;
        expect_bytes(bar, in_bytes + extra);
        tma_load(&tin, dst, bar, s.cg * CG, r);
        tma_load(&thalo, dst + (uint32_t)(ny * CG * 4), bar, s.cg * CG, r);
    };
    if (tid == PTID) {
        for (int d = 0; d < DEPTH; ++d) bar_init(bar0 + 8 * d);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        Seq p = cons;
        long long n = 0;
        for (; n < DEPTH && p.valid(); ++n) {
            issue((int)n, p);
            extra = 0;
            p.next(a);
        }
        prod->seq = p;
        prod->issued = n;
    }
    if (tid < DSLOTS) meta[tid].valid = 0;
    __syncthreads();

    uint32_t parity = 0;
    long long L = 0;
    bool failed = false, okacc = true;
    int pp = 0;  // which pair of staging slots the current two rows use

    // density threads: sum the staged rows of slot pair q in FP64 (fixed order)
    auto density = [&](int q) {
#pragma unroll 1
        for (int h = 0; h < 2; ++h) {
            const int slot = 2 * q + h;
            const RowMeta m = meta[slot];
            if (m.valid && dy < ny) {
                const float4* r = reinterpret_cast<const float4*>(stage + ((size_t)slot * YM + dy) * DSTRIDE);
                double t[2];
#pragma unroll
                for (int k = 0; k < 2; ++k) {  // two halves of 16 columns, each a fixed tree
                    const float4 u0 = r[4 * k], u1 = r[4 * k + 1], u2 = r[4 * k + 2], u3 = r[4 * k + 3];
                    t[k] = ((((double)u0.x + (double)u0.y) + ((double)u0.z + (double)u0.w)) +
                            (((double)u1.x + (double)u1.y) + ((double)u1.z + (double)u1.w))) +
                           ((((double)u2.x + (double)u2.y) + ((double)u2.z + (double)u2.w)) +
                            (((double)u3.x + (double)u3.y) + ((double)u3.z + (double)u3.w)));
                }
                a.part[((int64_t)m.x * a.n_cg + m.cg) * ny + dy] = t[0] + t[1];
            }
        }
    };

    // the register budget of each role holds inside its own branch
    if (drift) {
        asm volatile("setmaxnreg.inc.sync.aligned.u32 216;" ::: "memory");
        float2 win[WR / 2][6];  // rows 0..19 of the window, in pairs
        float wl[6];            // row 20
#pragma unroll
        for (int s = 0; s < 6; ++s) {
#pragma unroll
            for (int p = 0; p < WR / 2; ++p) win[p][s] = make_float2(0.f, 0.f);
            wl[s] = 0.f;
        }
        float2 wx[6], wy[6];
        float bx = 0.f, by = 0.f;
        int yoff = 0;
        auto tables = [&]() {
            const int jx = (cons.cg * CG / a.nvy) % a.nvx;
            const int jy = (cons.cg * CG) % a.nvy + lane;
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                const float u = __ldg(a.W_x + (5 - j) * a.nvx + jx), v = __ldg(a.W_y + (5 - j) * a.nvy + jy);
                wx[j] = make_float2(u, u);
                wy[j] = make_float2(v, v);
            }
            if constexpr (EQ) {
                const double feq = __ldg(a.eqA + jx) * __ldg(a.eqB + jy);
                bx = split_bias(feq, wx);
                by = split_bias(feq, wy);
            }
            int r = (y0 - __ldg(a.shift_y + jy) - 3) % ny;
            if (r < 0) r += ny;
            yoff = r * CG + lane;
        };
        tables();

        auto body = [&](auto step) -> bool {
            constexpr int P = decltype(step)::value;
            const bool ok = wait_phase(bar0 + 8 * P, parity);
            const float* sl = slabs + P * BUF + yoff;
#pragma unroll
            for (int p = 0; p < WR / 2; ++p) win[p][P] = make_float2(sl[(2 * p) * CG], sl[(2 * p + 1) * CG]);
            wl[P] = sl[(WR - 1) * CG];
            const bool emit = cons.q >= 5;
            const int slot = 2 * pp + (P & 1);
            const int x = cons.xa + cons.q - 5;
            if (emit) {
                float xd[WR];
#pragma unroll
                for (int p = 0; p < WR / 2; ++p) {
                    const float2 o = plus<EQ>(taps(wx, win[p][(P + 1) % 6], win[p][(P + 2) % 6], win[p][(P + 3) % 6],
                                                   win[p][(P + 4) % 6], win[p][(P + 5) % 6], win[p][P]),
                                              bx);
                    xd[2 * p] = o.x;
                    xd[2 * p + 1] = o.y;
                }
                xd[WR - 1] = tap1(wx, wl[(P + 1) % 6], wl[(P + 2) % 6], wl[(P + 3) % 6], wl[(P + 4) % 6],
                                  wl[(P + 5) % 6], wl[P]);
                if constexpr (EQ) xd[WR - 1] += bx;
                float o16[YT2];
#pragma unroll
                for (int p = 0; p < YT2 / 2; ++p) {
                    const int i = 2 * p;
                    const float2 o =
                        plus<EQ>(taps(wy, make_float2(xd[i], xd[i + 1]), make_float2(xd[i + 1], xd[i + 2]),
                                      make_float2(xd[i + 2], xd[i + 3]), make_float2(xd[i + 3], xd[i + 4]),
                                      make_float2(xd[i + 4], xd[i + 5]), make_float2(xd[i + 5], xd[i + 6])),
                                 by);
                    o16[i] = o.x;
                    o16[i + 1] = o.y;
                }
                float* dst = a.out + ((int64_t)x * ny + y0) * a.m + (int64_t)cons.cg * CG + lane;
                float* st = stage + ((size_t)slot * YM + y0) * DSTRIDE + lane;
#pragma unroll
                for (int e = 0; e < YT2; ++e)
                    if (FULL || y0 + e < ny) {
                        dst[(int64_t)e * a.m] = o16[e];
                        st[e * DSTRIDE] = o16[e];
                    }
            }
            if (tid == 0) {
                meta[slot] = RowMeta{x, cons.cg, emit ? 1 : 0, 0};
                if (!(P & 1)) meta[slot + 1].valid = 0;  // a pair may end after one row
            }
            okacc = okacc && ok;
            if (P & 1) {
                if (__syncthreads_or(!okacc)) {
                    failed = true;
                    return false;
                }
                pp ^= 1;
            }
            if (P == DEPTH - 1) parity ^= 1u;
            ++L;
            cons.next(a);
            if (__builtin_expect(cons.q == 0, 0) && cons.valid()) tables();
            return cons.valid();
        };
        while (body(Step<0>{}) && body(Step<1>{}) && body(Step<2>{}) && body(Step<3>{}) && body(Step<4>{}) &&
               body(Step<5>{})) {
        }
        // a wait on a last, even row has had no barrier vote yet
        if (!failed && __syncthreads_or(!okacc)) failed = true;
        if (failed) {
            // the whole share reads NaN (after this barrier no store of a
            // row lands any more)
            __syncthreads();
            Seq z;
            z.init(a, blockIdx.x, gridDim.x);
            while (z.valid()) {
                if (z.q >= 5) {
                    const int x = z.xa + z.q - 5;
                    for (int i = 0; i < YT2 && y0 + i < ny; ++i) {
                        a.out[((int64_t)x * ny + y0 + i) * a.m + (int64_t)z.cg * CG + lane] = NAN;
                        if (lane == 0) a.part[((int64_t)x * a.n_cg + z.cg) * ny + y0 + i] = (double)NAN;
                    }
                }
                z.next(a);
            }
        }
    } else {
        asm volatile("setmaxnreg.dec.sync.aligned.u32 72;" ::: "memory");
        // the density warpgroup: the same steps and barriers, no waits
        auto body = [&](auto step) -> bool {
            constexpr int P = decltype(step)::value;
            if (P & 1) {
                if (__syncthreads_or(0)) {
                    failed = true;
                    return false;
                }
                if (tid == PTID) {  // slabs P-1 and P are free
                    Seq& p = prod->seq;
#pragma unroll
                    for (int d = P - 1; d <= P; ++d)
                        if (p.valid()) {
                            issue(d, p);
                            p.next(a);
                            prod->issued += 1;
                        }
                }
                density(pp);
                pp ^= 1;
            }
            if (P == DEPTH - 1) parity ^= 1u;
            ++L;
            cons.next(a);
            return cons.valid();
        };
        while (body(Step<0>{}) && body(Step<1>{}) && body(Step<2>{}) && body(Step<3>{}) && body(Step<4>{}) &&
               body(Step<5>{})) {
        }
        // the drift warps' last vote (the same barrier, reached from their branch)
        if (!failed && __syncthreads_or(0)) failed = true;
        if (!failed && (L & 1)) density(pp);  // the last, single row
        if (failed) {
            __syncthreads();  // pairs with the drift warps' barrier before their NaN fill
            if (tid == PTID) {
                if (a.status) atomicOr(a.status, VP_STATUS_WAIT_TIMEOUT);
                // the loads in flight land before the block leaves
                for (long long k = L; k < prod->issued; ++k)
                    wait_phase(bar0 + 8 * (int)(k % DEPTH), (uint32_t)((k / DEPTH) & 1));
            }
        }
    }
}

// ---- many runs in one launch ------------------------------------------------
// The batched form of k_plane for runs of up to 64 rows (the 64-run batch of
// uneven grids): one persistent launch per drift pair for every run whose
// layout fits, each CTA walking whole lines (one group of 32 columns over all
// x) of the runs in order. Each run's tensor maps live in the batch's device
// table next to its arguments. The arithmetic of every element is that of
// k_plane (same FMA chains, FP32 intermediate), so f is bit-identical to the
// run stepped alone; outputs leave by direct stores, and the x-first pass
// stages its rows only for the FP64 density sums (four threads per y row,
// the order of k_plane's). Blocks have 8 warps; the warps past a run's rows
// compute nothing that is stored.
struct alignas(64) PlaneRun {
    CUtensorMap tin;    // [nx*ny][m] FP32, box {32, ny}
    CUtensorMap thalo;  // box {32, HALO}: y rows 0..15 of an x row, after row ny
    Args a;
};

// Whole lines of the batch's items, item g = (run r, group g - start[r]),
// for CTA b of G: items b, b + G, ...; loads q = 0 .. nx + 4 of the group's
// rows -s - 3 + q (mod nx), s the group's x shift.
struct BSeq {
    int64_t g, total, stride;
    int r, cg, nx, ny, q, r0;
    __device__ __forceinline__ void init(const PlaneRun* runs, const int64_t* start, int n_runs, int64_t b,
                                         int64_t G) {
        g = b;
        stride = G;
        total = start[n_runs];
        r = 0;
        if (valid()) begin(runs, start, n_runs);
    }
    __device__ __forceinline__ void begin(const PlaneRun* runs, const int64_t* start, int n_runs) {
        while (r + 1 < n_runs && start[r + 1] <= g) ++r;
        const Args& a = runs[r].a;
        cg = (int)(g - start[r]);
        nx = a.nx;
        ny = a.ny;
        const int jx = (int)(((int64_t)cg * CG / a.nvy) % a.nvx);
        r0 = -__ldg(a.shift_x + jx) - 3;
        q = 0;
    }
    __device__ __forceinline__ bool valid() const { return g < total; }
    __device__ __forceinline__ int row() const {
        const int v = (r0 + q) % nx;
        return v < 0 ? v + nx : v;
    }
    __device__ __forceinline__ void next(const PlaneRun* runs, const int64_t* start, int n_runs) {
        if (++q == nx + 5) {
            g += stride;
            if (valid()) begin(runs, start, n_runs);
        }
    }
};

struct BProducer {
    BSeq seq;
    long long issued;
    int fenced;  // the last run whose tensor maps this CTA has acquired
};

__host__ __device__ constexpr size_t batch_smem_bytes(bool xfirst, bool rho) {
    return (size_t)(DEPTH * buf_floats(YMAX / 2) + (rho ? 2 * stage_floats(YMAX / 2) : 0) +
                    (xfirst ? 2 * buf_floats(YMAX / 2) : 0)) * 4 +
           DEPTH * 8 + sizeof(BProducer);
}

template <bool XFIRST, bool RHO>
__global__ void __launch_bounds__(YMAX / 2 / YT * 32, 2)
    k_plane_batch(const PlaneRun* __restrict__ runs, const int64_t* __restrict__ start, int n_runs) {
    static_assert(!RHO || XFIRST, "the density comes with the x-first order");
    constexpr int YM = YMAX / 2, BUF = buf_floats(YM), STG = stage_floats(YM);
    extern __shared__ __align__(1024) unsigned char smem[];
    float* slabs = reinterpret_cast<float*>(smem);    // [DEPTH][BUF]
    float* stage = slabs + DEPTH * BUF;                // [2][STG] (the density's staged rows)
    float* planes = stage + (RHO ? 2 * STG : 0);       // [2][BUF] (x first)
    uint64_t* bars = reinterpret_cast<uint64_t*>(planes + (XFIRST ? 2 * BUF : 0));
    BProducer* prod = reinterpret_cast<BProducer*>(bars + DEPTH);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int y0 = warp * YT;
    BSeq cons;
    cons.init(runs, start, n_runs, blockIdx.x, gridDim.x);
    if (!cons.valid()) return;
    const uint32_t slab0 = smem_u32(slabs), bar0 = smem_u32(bars);
    auto issue = [&](int d, const BSeq& s) {
        const PlaneRun* pr = runs + s.r;
        if (prod->fenced != s.r) {
            // the run's tensor maps reached global memory by a copy from the host
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&pr->tin) : "memory");
            if constexpr (!XFIRST)
                asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&pr->thalo) : "memory");
            prod->fenced = s.r;
        }
        const uint32_t dst = slab0 + (uint32_t)(d * BUF * 4), bar = bar0 + 8 * d;
        const int rr = s.row() * s.ny;
        expect_bytes(bar, (uint32_t)((s.ny + (XFIRST ? 0 : HALO)) * CG * 4));
        tma_load(&pr->tin, dst, bar, s.cg * CG, rr);
        if constexpr (!XFIRST) tma_load(&pr->thalo, dst + (uint32_t)(s.ny * CG * 4), bar, s.cg * CG, rr);
    };
    if (tid == 0) {
        prod->fenced = -1;
        for (int d = 0; d < DEPTH; ++d) bar_init(bar0 + 8 * d);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        BSeq p = cons;
        long long n = 0;
        for (; n < DEPTH && p.valid(); ++n) {
            issue((int)n, p);
            p.next(runs, start, n_runs);
        }
        prod->seq = p;
        prod->issued = n;
    }
    __syncthreads();

    float2 win[YT / 2][6];
#pragma unroll
    for (int p = 0; p < YT / 2; ++p)
#pragma unroll
        for (int s = 0; s < 6; ++s) win[p][s] = make_float2(0.f, 0.f);
    float2 wx[6], wy[6];
    int yoff = 0, ny = cons.ny, n_cg = 0;
    float* out = nullptr;
    double* part = nullptr;
    int64_t m = 0;
    uint32_t parity = 0;
    long long L = 0;
    bool failed = false, okacc = true;
    bool pend = false;  // x first: a row waiting for its y drift
    int pend_x = 0, pend_cg = 0;
    bool rho_on = false;  // x first: a staged row waiting for its density
    int rho_x = 0, rho_cg = 0, rho_ny = 0, rho_ncg = 0;
    double* rho_part = nullptr;

    // the weights, y window and run of the consumer's current group
    auto tables = [&]() {
        const Args& a = runs[cons.r].a;
        out = a.out;
        m = a.m;
        ny = cons.ny;
        part = a.part;
        n_cg = a.n_cg;
        const int jx = (int)(((int64_t)cons.cg * CG / a.nvy) % a.nvx);
        const int jy = (int)(((int64_t)cons.cg * CG) % a.nvy) + lane;
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            const float u = __ldg(a.W_x + (5 - j) * a.nvx + jx), v = __ldg(a.W_y + (5 - j) * a.nvy + jy);
            wx[j] = make_float2(u, u);
            wy[j] = make_float2(v, v);
        }
        int r = (y0 - __ldg(a.shift_y + jy) - 3) % ny;
        if (r < 0) r += ny;
        yoff = r * CG + lane;
    };
    tables();

    // x first: y drift of the pending row from plane PL; stored, and staged
    // in PL for its density
    auto y_pending = [&](auto pl) {
        constexpr int PL = decltype(pl)::value;
        float2 o[YT / 2];
        y_drift<false>(planes + PL * BUF + yoff, wy, 0.f, o);
        if (pend) {
            float* dst = out + ((int64_t)pend_x * ny + y0) * m + (int64_t)pend_cg * CG + lane;
#pragma unroll
            for (int p = 0; p < YT / 2; ++p) {
                const int y = y0 + 2 * p;
                if (y < ny) dst[(int64_t)(2 * p) * m] = o[p].x;
                if (y + 1 < ny) dst[(int64_t)(2 * p + 1) * m] = o[p].y;
            }
        }
        if constexpr (RHO) {
            float* st = stage + PL * STG;
#pragma unroll
            for (int p = 0; p < YT / 2; ++p) {
                const int y = y0 + 2 * p;
                if (y < ny) st[y * CG + lane] = o[p].x;
                if (y + 1 < ny) st[(y + 1) * CG + lane] = o[p].y;
            }
        }
    };
    // x first: density partials of the row staged in SP (thread: y row
    // tid / 4, columns 8 (tid % 4) .. + 7; the sums of k_plane's order)
    const int rrow = tid >> 2, rq = tid & 3;
    auto rho_row = [&](auto sp) {
        constexpr int SP = decltype(sp)::value;
        const float4* src = reinterpret_cast<const float4*>(stage + SP * STG + rrow * CG) + 2 * rq;
        const int odd = rrow & 1;
        const float4 u = src[odd], v = src[1 - odd];
        const double s = (((double)u.x + (double)u.y) + ((double)u.z + (double)u.w)) +
                         (((double)v.x + (double)v.y) + ((double)v.z + (double)v.w));
        double t = s + __shfl_xor_sync(0xffffffffu, s, 1);
        t += __shfl_xor_sync(0xffffffffu, t, 2);
        if (rho_on && rq == 0 && rrow < rho_ny) rho_part[((int64_t)rho_x * rho_ncg + rho_cg) * rho_ny + rrow] = t;
    };

    auto body = [&](auto step) -> bool {
        constexpr int P = decltype(step)::value;
        if constexpr (XFIRST) {
            if constexpr (RHO) rho_row(Step<P & 1>{});
            y_pending(Step<(P + 1) & 1>{});
        }
        const bool ok = wait_phase(bar0 + 8 * P, parity);
        const bool emit = cons.q >= 5;
        const float* sl = slabs + P * BUF;
        float2 nv[YT / 2];
        if constexpr (XFIRST) {
            // x drift of the new row into plane P & 1 (read one step later)
#pragma unroll
            for (int p = 0; p < YT / 2; ++p)
                nv[p] = make_float2(sl[(y0 + 2 * p) * CG + lane], sl[(y0 + 2 * p + 1) * CG + lane]);
            float* pl = planes + (P & 1) * BUF;
#pragma unroll
            for (int p = 0; p < YT / 2; ++p) {
                const float2 o = taps(wx, win[p][(P + 1) % 6], win[p][(P + 2) % 6], win[p][(P + 3) % 6],
                                      win[p][(P + 4) % 6], win[p][(P + 5) % 6], nv[p]);
                const int y = y0 + 2 * p;
                if (y < ny) pl[y * CG + lane] = o.x;
                if (y + 1 < ny) pl[(y + 1) * CG + lane] = o.y;
                if (y0 < HALO) {  // warp-uniform: the rows copied after row ny
                    pl[(ny + y) * CG + lane] = o.x;
                    pl[(ny + y + 1) * CG + lane] = o.y;
                }
            }
        } else {
            // y drift of the new row from its slab, then the x drift
            y_drift<false>(sl + yoff, wy, 0.f, nv);
            if (emit) {
                float* dst = out + ((int64_t)(cons.q - 5) * ny + y0) * m + (int64_t)cons.cg * CG + lane;
#pragma unroll
                for (int p = 0; p < YT / 2; ++p) {
                    const float2 o = taps(wx, win[p][(P + 1) % 6], win[p][(P + 2) % 6], win[p][(P + 3) % 6],
                                          win[p][(P + 4) % 6], win[p][(P + 5) % 6], nv[p]);
                    const int y = y0 + 2 * p;
                    if (y < ny) dst[(int64_t)(2 * p) * m] = o.x;
                    if (y + 1 < ny) dst[(int64_t)(2 * p + 1) * m] = o.y;
                }
            }
        }
#pragma unroll
        for (int p = 0; p < YT / 2; ++p) win[p][P] = nv[p];
        okacc = okacc && ok;
        if (XFIRST || (P & 1)) {
            // x first: every row (its plane and staged row change hands);
            // y first: every second row (slabs P-1 and P are free)
            if (__syncthreads_or(!okacc)) {
                failed = true;
                return false;
            }
            if (tid == 0) {
                BSeq& p = prod->seq;
#pragma unroll
                for (int d = XFIRST ? P : P - 1; d <= P; ++d)
                    if (p.valid()) {
                        issue(d, p);
                        p.next(runs, start, n_runs);
                        prod->issued += 1;
                    }
            }
        }
        if (P == DEPTH - 1) parity ^= 1u;
        ++L;
        if constexpr (XFIRST) {
            // the row y_pending staged this step belongs to the consumer's run
            rho_on = pend;
            rho_x = pend_x;
            rho_cg = pend_cg;
            rho_ny = ny;
            rho_ncg = n_cg;
            rho_part = part;
            pend = emit;
            pend_x = cons.q - 5;
            pend_cg = cons.cg;
        }
        cons.next(runs, start, n_runs);
        // a new group: its tables after the pending row of the last one went
        // through (x first: one step into the group; y first: before its first row)
        if (cons.valid() && cons.q == (XFIRST ? 1 : 0)) tables();
        return cons.valid();
    };

    while (body(Step<0>{}) && body(Step<1>{}) && body(Step<2>{}) && body(Step<3>{}) && body(Step<4>{}) &&
           body(Step<5>{})) {
    }
    if constexpr (!XFIRST) {
        // a wait on a last, even row has had no barrier vote yet
        if (!failed && __syncthreads_or(!okacc)) failed = true;
    } else if (!failed) {
        // the rows still in the pipeline: the density of the row staged at
        // the last step, then the last row (its plane is complete)
        const int last = (int)((L - 1) % DEPTH);
        if constexpr (RHO) {
            if (last & 1)
                rho_row(Step<0>{});
            else
                rho_row(Step<1>{});
        }
        if (pend) {
            if (last & 1)
                y_pending(Step<1>{});
            else
                y_pending(Step<0>{});
            if constexpr (RHO) {
                __syncthreads();
                rho_on = true;
                rho_x = pend_x;
                rho_cg = pend_cg;
                rho_ny = ny;
                rho_ncg = n_cg;
                rho_part = part;
                if (last & 1)
                    rho_row(Step<1>{});
                else
                    rho_row(Step<0>{});
            }
        }
    }
    if (failed) {
        // the whole share reads NaN, then the loads in flight land
        __syncthreads();
        BSeq z;
        z.init(runs, start, n_runs, blockIdx.x, gridDim.x);
        while (z.valid()) {
            if (z.q >= 5) {
                const Args& za = runs[z.r].a;
                const int x = z.q - 5;
                for (int i = 0; i < YT && y0 + i < z.ny; ++i) {
                    za.out[((int64_t)x * z.ny + y0 + i) * za.m + (int64_t)z.cg * CG + lane] = NAN;
                    if (RHO && lane == 0) za.part[((int64_t)x * za.n_cg + z.cg) * z.ny + y0 + i] = (double)NAN;
                }
            }
            z.next(runs, start, n_runs);
        }
        if (tid == 0)
            for (long long k = L; k < prod->issued; ++k)
                wait_phase(bar0 + 8 * (int)(k % DEPTH), (uint32_t)((k / DEPTH) & 1));
    }
}

// cuTensorMapEncodeTiled from the driver, looked up once
static PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    }
    return fn;
}

// [nx*ny][m] FP32 view of f with a {CG, rows} box
static bool make_map(CUtensorMap* tm, const void* base, int64_t m, int64_t rows_total, int box_rows) {
    const cuuint64_t dims[2] = {(cuuint64_t)m, (cuuint64_t)rows_total};
    const cuuint64_t strides[1] = {(cuuint64_t)(m * sizeof(float))};
    const cuuint32_t box[2] = {(cuuint32_t)CG, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return encoder()(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static constexpr size_t smem_bytes(bool xfirst, int ym) {
    return (size_t)(DEPTH * buf_floats(ym) + (xfirst ? 2 * stage_floats(ym) + 2 * buf_floats(ym) : 0)) * 4 +
           DEPTH * 8 + sizeof(Producer);
}

template <bool XFIRST, bool RHO, bool FULL, int YM, bool EQ>
static int launch_t(const CUtensorMap& tin, const CUtensorMap& thalo, const CUtensorMap& tout, const Args& a,
                    cudaStream_t st) {
    auto kern = k_plane<XFIRST, RHO, FULL, YM, EQ>;
    constexpr size_t smem = smem_bytes(XFIRST, YM);
    const int block = 32 * ((a.ny + YT - 1) / YT);
    static int raised[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return set_error(VP_ERR_CUDA, "run_plane: device index out of range");
    if (!raised[dev]) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return set_cuda_error("cudaFuncSetAttribute(k_plane)");
        raised[dev] = 1;
    }
    const int occ = occupancy(kern, block, smem);
    const int64_t total = (int64_t)a.n_cg * a.xc;
    const int64_t grid = std::min<int64_t>(total, (int64_t)sm_count() * occ);
    kern<<<(unsigned)grid, block, smem, st>>>(tin, thalo, tout, a);
    return check_launch("k_plane");
}

template <bool FULL, bool EQ>
static int launch_xrd(const CUtensorMap& tin, const CUtensorMap& thalo, const Args& a, cudaStream_t st) {
    auto kern = k_plane_xrd<FULL, EQ>;
    constexpr size_t smem = xrd_smem_bytes();
    static int raised[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return set_error(VP_ERR_CUDA, "run_plane: device index out of range");
    if (!raised[dev]) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return set_cuda_error("cudaFuncSetAttribute(k_plane_xrd)");
        raised[dev] = 1;
    }
    const int occ = occupancy(kern, XRD_THREADS, smem);
    if (occ < 1) return set_error(VP_ERR_UNSUPPORTED, "run_plane: the density pass does not fit an SM");
    const int64_t total = (int64_t)a.n_cg * a.xc;
    const int64_t grid = std::min<int64_t>(total, (int64_t)sm_count() * occ);
    kern<<<(unsigned)grid, XRD_THREADS, smem, st>>>(tin, thalo, a);
    return check_launch("k_plane_xrd");
}

template <bool RHO, bool FULL, int YM, bool EQ>
static int launch_xr(const CUtensorMap& tin, const CUtensorMap& thalo, const Args& a, cudaStream_t st) {
    auto kern = k_plane_xr<RHO, FULL, YM, EQ>;
    constexpr size_t smem = (size_t)(DEPTH * buf2_floats(YM) + (RHO ? 2 * (YM / YT2) * RFLOATS : 0)) * 4 +
                            DEPTH * 8 + sizeof(Producer);
    const int block = 32 * ((a.ny + YT2 - 1) / YT2);
    static int raised[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return set_error(VP_ERR_CUDA, "run_plane: device index out of range");
    if (!raised[dev]) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return set_cuda_error("cudaFuncSetAttribute(k_plane_xr)");
        raised[dev] = 1;
    }
    const int occ = occupancy(kern, block, smem);
    const int64_t total = (int64_t)a.n_cg * a.xc;
    const int64_t grid = std::min<int64_t>(total, (int64_t)sm_count() * occ);
    kern<<<(unsigned)grid, block, smem, st>>>(tin, thalo, a);
    return check_launch("k_plane_xr");
}

template <bool XFIRST, bool RHO>
static int launch_batch_t(const PlaneRun* runs, const int64_t* start, int n_runs, int64_t items, cudaStream_t st) {
    auto kern = k_plane_batch<XFIRST, RHO>;
    constexpr size_t smem = batch_smem_bytes(XFIRST, RHO);
    constexpr int block = YMAX / 2 / YT * 32;
    static int raised[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return set_error(VP_ERR_CUDA, "plane batch: device index out of range");
    if (!raised[dev]) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return set_cuda_error("cudaFuncSetAttribute(k_plane_batch)");
        raised[dev] = 1;
    }
    const int occ = occupancy(kern, block, smem);
    if (occ < 1) return set_error(VP_ERR_UNSUPPORTED, "plane batch: the kernel does not fit an SM");
    const int64_t grid = std::min<int64_t>(items, (int64_t)sm_count() * occ);
    kern<<<(unsigned)grid, block, smem, st>>>(runs, start, n_runs);
    return check_launch("k_plane_batch");
}

}  // namespace plane

size_t plane_run_bytes() { return sizeof(plane::PlaneRun); }

// Runs of 49..64 rows. Measured on B200 (batches of one run size, FP32): the
// fused pairs beat the sweeps for 64-row runs (64^4: 1.575 against 1.839 ms a
// step) but not below (48 rows: 1.740 against 1.584; 16 rows: 2.4x slower):
// a smaller run's TMA row boxes keep too few bytes in flight in the 6-slab
// ring, and most of the block's warps have no rows.
bool plane_batch_fits(int dtype, int64_t nx, int64_t ny, int64_t nvx, int64_t nvy, const void* a, const void* b,
                      const void* c) {
    return plane_fits(dtype, nx, ny, nvx, nvy, a) && plane_fits(dtype, nx, ny, nvx, nvy, b) &&
           plane_fits(dtype, nx, ny, nvx, nvy, c) && ny > 48 && ny <= plane::YMAX / 2;
}

int plane_batch_run(void* record, const void* in, void* out, int64_t nx, int64_t ny, int64_t nvx, int64_t nvy,
                    const int* shift_x, const void* W_x, const int* shift_y, const void* W_y, double* part,
                    int64_t* items) {
    using namespace plane;
    // encoded in an aligned local record, then copied into the (host) table
    PlaneRun rec;
    std::memset(static_cast<void*>(&rec), 0, sizeof(PlaneRun));
    PlaneRun* pr = &rec;
    Args& a = pr->a;
    a.out = static_cast<float*>(out);
    a.nx = (int)nx;
    a.ny = (int)ny;
    a.nvx = (int)nvx;
    a.nvy = (int)nvy;
    a.xb = 0;
    a.xc = (int)nx;
    a.m = nvx * nvy;
    a.n_cg = (int)(a.m / CG);
    a.shift_x = shift_x;
    a.W_x = static_cast<const float*>(W_x);
    a.shift_y = shift_y;
    a.W_y = static_cast<const float*>(W_y);
    a.part = part;
    if (!make_map(&pr->tin, in, a.m, nx * ny, (int)ny) || !make_map(&pr->thalo, in, a.m, nx * ny, HALO))
        return set_error(VP_ERR_CUDA, "plane batch: cuTensorMapEncodeTiled failed");
    std::memcpy(record, &rec, sizeof(PlaneRun));
    *items = a.n_cg;
    return VP_OK;
}

int launch_plane_batch(bool xfirst, bool rho, const void* runs, const int64_t* start, int n_runs, int64_t items,
                       cudaStream_t st) {
    using namespace plane;
    if (items <= 0) return VP_OK;
    const PlaneRun* pr = static_cast<const PlaneRun*>(runs);
    if (!xfirst) return launch_batch_t<false, false>(pr, start, n_runs, items, st);
    return rho ? launch_batch_t<true, true>(pr, start, n_runs, items, st)
               : launch_batch_t<true, false>(pr, start, n_runs, items, st);
}

bool plane_fits(int dtype, int64_t nx, int64_t ny, int64_t nvx, int64_t nvy, const void* f) {
    using namespace plane;
    if (dtype != VP_F32) return false;
    if (ny < YMIN || ny > YMAX || nvy % CG != 0 || nvx < 1 || nx < 1) return false;
    if ((int64_t)nx * ny >= (1ll << 31) || nvx * nvy >= (1ll << 31)) return false;
    if (nvx * nvy / CG * nx >= (1ll << 31)) return false;  // column groups x rows: 32-bit work counters
    if (reinterpret_cast<uintptr_t>(f) % 16 != 0) return false;
    return encoder() != nullptr;
}

int64_t plane_part_tiles(int64_t nvx, int64_t nvy) { return nvx * nvy / plane::CG; }

int run_plane(int dtype, bool xfirst, const void* in, void* out, int64_t nx, int64_t ny, int64_t nvx, int64_t nvy,
              int64_t x_begin, int64_t x_count, const int* shift_x, const void* W_x, const int* shift_y,
              const void* W_y, double* part, int* tiles, const EqSplit* eq, int* status, int stall, cudaStream_t st) {
    using namespace plane;
    if (!plane_fits(dtype, nx, ny, nvx, nvy, in) || !plane_fits(dtype, nx, ny, nvx, nvy, out))
        return set_error(VP_ERR_UNSUPPORTED, "run_plane: layout not fused");
    if (x_begin < 0 || x_count < 1 || x_begin + x_count > nx)
        return set_error(VP_ERR_ARG, "run_plane: output rows outside [0, nx)");
    Args a{};
    a.out = static_cast<float*>(out);
    a.nx = (int)nx;
    a.xb = (int)x_begin;
    a.xc = (int)x_count;
    a.ny = (int)ny;
    a.nvx = (int)nvx;
    a.nvy = (int)nvy;
    a.m = nvx * nvy;
    a.n_cg = (int)(a.m / CG);
    a.shift_x = shift_x;
    a.W_x = static_cast<const float*>(W_x);
    a.shift_y = shift_y;
    a.W_y = static_cast<const float*>(W_y);
    a.part = part;
    const bool eq_on = eq && eq->A && eq->B;
    if (eq && !eq_on && (eq->A || eq->B))
        return set_error(VP_ERR_UNSUPPORTED, "run_plane: the split needs both equilibrium factors");
    a.eqA = eq_on ? eq->A : nullptr;
    a.eqB = eq_on ? eq->B : nullptr;
    a.status = status;
    a.stall = stall;
    if (tiles) *tiles = a.n_cg;
    CUtensorMap tin, thalo, tout;
    if (xfirst && ny > YMAX - YT2) {
        // x then y with the window in registers: 8 warps per CTA. With
        // fewer rows (fewer warps, one CTA per SM) the plane exchange of
        // k_plane is faster.
        if (!make_map(&tin, in, a.m, nx * ny, (int)ny) || !make_map(&thalo, in, a.m, nx * ny, HALO2))
            return set_error(VP_ERR_CUDA, "run_plane: cuTensorMapEncodeTiled failed");
        const bool full2 = ny % YT2 == 0;
        auto go2 = [&](auto eqc) {
            constexpr bool E = decltype(eqc)::value != 0;
            if (part)  // the density on its own warpgroup
                return full2 ? launch_xrd<true, E>(tin, thalo, a, st) : launch_xrd<false, E>(tin, thalo, a, st);
            return full2 ? launch_xr<false, true, YMAX, E>(tin, thalo, a, st)
                         : launch_xr<false, false, YMAX, E>(tin, thalo, a, st);
        };
        return eq_on ? go2(Step<1>{}) : go2(Step<0>{});
    }
    if (!make_map(&tin, in, a.m, nx * ny, (int)ny) || !make_map(&thalo, in, a.m, nx * ny, HALO) ||
        !make_map(&tout, out, a.m, nx * ny, (int)ny))
        return set_error(VP_ERR_CUDA, "run_plane: cuTensorMapEncodeTiled failed");
    const bool full = ny % YT == 0;
    auto go = [&](auto ym, auto eqc) {
        constexpr int YM = decltype(ym)::value;
        constexpr bool E = decltype(eqc)::value != 0;
        if (xfirst) {
            if (part)
                return full ? launch_t<true, true, true, YM, E>(tin, thalo, tout, a, st)
                            : launch_t<true, true, false, YM, E>(tin, thalo, tout, a, st);
            return full ? launch_t<true, false, true, YM, E>(tin, thalo, tout, a, st)
                        : launch_t<true, false, false, YM, E>(tin, thalo, tout, a, st);
        }
        return full ? launch_t<false, false, true, YM, E>(tin, thalo, tout, a, st)
                    : launch_t<false, false, false, YM, E>(tin, thalo, tout, a, st);
    };
    if (ny <= YMAX / 2) return eq_on ? go(Step<YMAX / 2>{}, Step<1>{}) : go(Step<YMAX / 2>{}, Step<0>{});
    return eq_on ? go(Step<YMAX>{}, Step<1>{}) : go(Step<YMAX>{}, Step<0>{});
}

}  // namespace vp
