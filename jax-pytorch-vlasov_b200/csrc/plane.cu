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
#include <cstddef>
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
    // the next row of the segment; false at its end (then next_seg)
    __device__ __forceinline__ bool step_on() { return ++q < n + 5; }
    __device__ __forceinline__ void next_seg(const Args& a) {
        if (w < full)
            ++w;
        else
            t += n;
        if (valid()) start(a);
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

// body(Step<P>) for P = p0, p0 + 1, ... around the ring until it returns
// false; the step it stopped at. One copy of each unrolled step: a pack's
// end leaves the loop instead of being handled inside every step.
template <typename Body>
__device__ __forceinline__ int run_steps(Body& body, int p0) {
    for (;;) {
        switch (p0) {
            case 0:
                if (!body(Step<0>{})) return 0;
                [[fallthrough]];
            case 1:
                if (!body(Step<1>{})) return 1;
                [[fallthrough]];
            case 2:
                if (!body(Step<2>{})) return 2;
                [[fallthrough]];
            case 3:
                if (!body(Step<3>{})) return 3;
                [[fallthrough]];
            case 4:
                if (!body(Step<4>{})) return 4;
                [[fallthrough]];
            default:
                if (!body(Step<5>{})) return 5;
        }
        p0 = 0;
    }
}

// y drift of the thread's 8 rows from 13 consecutive rows of a buffer
// (g: row y0 - s - 3 of the lane's column, halo included)
template <bool EQ, int RS = CG>
__device__ __forceinline__ void y_drift(const float* g, const float2 (&wy)[6], float by, float2 (&o)[YT / 2]) {
    float r[YT + 5];
#pragma unroll
    for (int k = 0; k < YT + 5; ++k) r[k] = g[k * RS];
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
            return cons.step_on();
        };
        for (int p0 = 0;;) {
            const int pe = run_steps(body, p0);
            if (failed) break;
            cons.next_seg(a);
            if (!cons.valid()) break;
            tables();
            p0 = (pe + 1) % DEPTH;
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
            return cons.step_on();
        };
        for (int p0 = 0;;) {
            const int pe = run_steps(body, p0);
            if (failed) break;
            cons.next_seg(a);
            if (!cons.valid()) break;
            p0 = (pe + 1) % DEPTH;
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
// The batched drift pairs for runs of up to 64 rows (the 64-run batch of
// uneven grids): one persistent launch per pair for every run whose layout
// fits, each CTA walking whole lines (column groups over all x) of the runs
// in order, several groups of one run at a time. The runs' arguments live in
// the batch's device table; their tensor maps go to the kernel as a
// parameter (up to XB_MAXR runs a launch), so that TMA reads its
// descriptors from the parameter space as in the single-run kernels (with
// the maps in the device table the same kernels ran at about half the
// speed). The arithmetic of every element is that of the single-run passes
// (same FMA chains, FP32 intermediate), so f is bit-identical to the run
// stepped alone.
struct alignas(64) PlaneRun {
    CUtensorMap tin;    // [nx*ny][m] FP32, box {32, ny}
    CUtensorMap thalo;  // box {32, halo rows}: y rows 0.. of an x row, after row ny
    Args a;
    int k_pack;         // column groups stepped together by one CTA
    int slab_rows;      // rows of one ring slab: k_pack boxes of ny + halo rows
};

// ---- many runs, x then y, register window ---------------------------------
// The batched x-first pass in the form of k_plane_xrd (setmaxnreg 216 / 72,
// 208 / 88 with half boxes: the issuers' second x row): 8 drift
// warps of 16 y rows with the 21-row x window in registers, and a warpgroup
// of 4 density warps (the FP64 row sums of the staged output, one thread a row, in
// k_plane_xrd's order; its first thread issues the TMA loads). A CTA steps a
// pack of K column groups of one run through x together, K = 8 / ceil(ny /
// 16) (two groups of up to 64 rows, four of up to 32): warp w works on group
// w / wpg, rows 16 (w % wpg) .. +15. Each step loads K boxes of ny + 20 rows,
// one per group (the groups of a pack lie in different vx, so their x rows
// differ). The K ny <= 128 output rows of a step are staged for the density
// warps without padding, 16-byte chunks swizzled by row (chunk ^ row % 8;
// ny is a multiple of 8, so a warp's rows start on a multiple of 8). Every
// element takes k_plane_xrd's FMA chains and every density partial its sum
// order, so f and rho are bit-identical to the run stepped alone.
constexpr int XB_SROWS = 128;  // staged rows per slot
// columns per TMA box of the packed x-first pass: a group of 32 columns comes
// in as two boxes of 16 (each at the x row of its own vx, so that groups
// which span two vx of a run with nvy % 32 != 0 work too); in shared memory a
// group is [half][ny + 20][16]
constexpr int HB = 16;
// packs per ny: up to 32 rows four groups of ny + 20 rows, up to 64 two
constexpr int xb_pack(int ny) { return XRD_CW / ((ny + YT2 - 1) / YT2); }
constexpr int XB_MAX_SLAB_ROWS = 4 * (32 + HALO2);
struct PackMeta {
    int x, r, cg0, kv, ny, valid, pad0, pad1;
};

// Whole lines of the batch's packs, pack g = (run r, groups k_pack (g -
// start[r]) ..), for CTA b of G: packs b, b + G, ...; step q = 0 .. nx + 4
// loads, for each group k of the pack, x row r0_k + q (mod nx).
struct PSeq {
    int g, total, stride;
    int r, K, kv, cg0, nx, ny, q;
    __device__ __forceinline__ void init(const PlaneRun* runs, const int64_t* start, int n_runs, int b, int G) {
        g = (int)start[0] + b;  // start[] holds the prefix sums of the whole batch
        stride = G;
        total = (int)start[n_runs];
        r = 0;
        if (valid()) begin(runs, start, n_runs);
    }
    __device__ __forceinline__ void begin(const PlaneRun* runs, const int64_t* start, int n_runs) {
        while (r + 1 < n_runs && start[r + 1] <= g) ++r;
        const PlaneRun& pr = runs[r];
        K = pr.k_pack;
        cg0 = (g - (int)start[r]) * K;
        kv = min(K, pr.a.n_cg - cg0);
        nx = pr.a.nx;
        ny = pr.a.ny;
        q = 0;
    }
    __device__ __forceinline__ bool valid() const { return g < total; }
    // the next step of the pack; false at its end (then next_pack)
    __device__ __forceinline__ bool step_on() { return ++q < nx + 5; }
    __device__ __forceinline__ void next_pack(const PlaneRun* runs, const int64_t* start, int n_runs) {
        g += stride;
        if (valid()) begin(runs, start, n_runs);
    }
    __device__ __forceinline__ void next(const PlaneRun* runs, const int64_t* start, int n_runs) {
        if (!step_on()) next_pack(runs, start, n_runs);
    }
};

struct XBProducer {
    PSeq seq;
    int r0[8];  // the current pack's group halves (x first) or groups: -(x shift) - 3
    long long issued;  // loads issued (steps)
};

// the tensor maps of up to XB_MAXR runs as a kernel parameter (16 KB): TMA
// reads its descriptors from the parameter space, as the single-run kernels
// do; batches of more runs launch once per XB_MAXR runs
constexpr int XB_MAXR = 64;
struct XBMaps {
    CUtensorMap tin[XB_MAXR];
    CUtensorMap thalo[XB_MAXR];
};

__host__ __device__ constexpr size_t xrd_batch_smem_bytes(int slab_rows) {
    return (size_t)(DEPTH * slab_rows * CG + DSLOTS * XB_SROWS * CG) * 4 + DSLOTS * sizeof(PackMeta) + DEPTH * 8 +
           sizeof(XBProducer);
}

// The launches of one plane pass (the whole-box and half-box classes, more
// than 64 runs, then the x sweep of the batch's other runs) follow each other
// as programmatic dependents (pdl_release / pdl_hold): they work on different
// runs, so each starts its CTAs on the SMs the launch before it leaves.
template <bool RHO, bool HALF>
__device__ __forceinline__ void xrd_batch_body(const XBMaps& maps, const PlaneRun* __restrict__ runs,
                                               const int64_t* __restrict__ start, int n_runs, int slab_floats) {
    extern __shared__ __align__(1024) unsigned char smem[];
    float* slabs = reinterpret_cast<float*>(smem);                 // [DEPTH][slab_floats]
    float* stage = slabs + DEPTH * slab_floats;                     // [DSLOTS][XB_SROWS][CG], swizzled
    PackMeta* meta = reinterpret_cast<PackMeta*>(stage + DSLOTS * XB_SROWS * CG);
    uint64_t* bars = reinterpret_cast<uint64_t*>(meta + DSLOTS);
    XBProducer* prod = reinterpret_cast<XBProducer*>(bars + DEPTH);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool drift = warp < XRD_CW;
    constexpr int PTID = XRD_CW * 32;  // producer: the first density thread
    const int dy = tid - PTID;         // density thread: its staged row
    PSeq cons;
    cons.init(runs, start, n_runs, (int)blockIdx.x, (int)gridDim.x);
    if (!cons.valid()) return;
    const uint32_t slab0 = smem_u32(slabs), bar0 = smem_u32(bars);
    const uint32_t slab_bytes = (uint32_t)slab_floats * 4u;
    constexpr int BW = HALF ? HB : CG, NB = CG / BW;  // box columns, boxes per group
    // producers: thread PTID issues the first DEPTH steps; then the first lane
    // of density warp k issues group k's loads of every step (a step's 2K TMA
    // operations on one thread had put that thread's warp on the path to each
    // barrier). Each keeps its copy of the sequence and of its groups' x-row
    // offsets in registers; across the role split they pass through shared
    // memory.
    XBProducer pr{};
    auto pack_rows = [&]() {
        const Args& a = runs[pr.seq.r].a;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k < pr.seq.kv) {
#pragma unroll
                for (int h = 0; h < NB; ++h)
                    pr.r0[2 * k + h] = -__ldg(a.shift_x + (((pr.seq.cg0 + k) * CG + h * BW) / a.nvy) % a.nvx) - 3;
            }
    };
    // the loads of groups k0 .. k1 - 1 of the sequence's current step into
    // slab d; group 0's issuer arms the barrier with the step's bytes (extra:
    // the test hook's 16 bytes too many on the CTA's first load). Loads that
    // complete before the arming leave the barrier's byte count negative for
    // a while; the phase cannot complete before its one arrival.
    auto issue = [&](int d, uint32_t extra) {
        const PSeq& ps = pr.seq;
        const CUtensorMap* tin = &maps.tin[ps.r];
        const CUtensorMap* thalo = &maps.thalo[ps.r];
        const uint32_t box = (uint32_t)((ps.ny + HALO2) * CG * 4), bar = bar0 + 8 * d;
        expect_bytes(bar, box * (uint32_t)ps.kv + extra);
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k < ps.kv) {
#pragma unroll
                for (int h = 0; h < NB; ++h) {
                    int v = (pr.r0[2 * k + h] + ps.q) % ps.nx;
                    if (v < 0) v += ps.nx;
                    const uint32_t dst = slab0 + (uint32_t)d * slab_bytes + (uint32_t)k * box + (uint32_t)h * box / NB;
                    const int c0 = (ps.cg0 + k) * CG + h * BW;
                    tma_load(tin, dst, bar, c0, v * ps.ny);
                    tma_load(thalo, dst + (uint32_t)(ps.ny * BW * 4), bar, c0, v * ps.ny);
                }
            }
        pr.issued += 1;
    };
    auto advance = [&]() {
        if (!pr.seq.step_on()) {
            pr.seq.next_pack(runs, start, n_runs);
            if (pr.seq.valid()) pack_rows();
        }
    };
    if (tid == PTID) {
        for (int d = 0; d < DEPTH; ++d) bar_init(bar0 + 8 * d);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        pr.seq = cons;
        pr.issued = 0;
        pack_rows();
        for (int n = 0; n < DEPTH && pr.seq.valid(); ++n) {
            issue(n, n == 0 && runs[cons.r].a.stall ? 16u : 0u);
            advance();
        }
        *prod = pr;
    }
    if (tid < DSLOTS) meta[tid].valid = 0;
    __syncthreads();

    uint32_t parity = 0;
    long long L = 0;
    bool failed = false, okacc = true;
    int pp = 0;  // which pair of staging slots the current two rows use

    // density threads: sum the staged rows of slot pair q in FP64 (fixed
    // order); the run's partials and the thread's (group, row) are cached
    int c_r = -1, c_ny = -1, c_ncg = 0, kd = 0, yd = 0;
    double* c_part = nullptr;
    auto density = [&](int q) {
#pragma unroll 1
        for (int h = 0; h < 2; ++h) {
            const int slot = 2 * q + h;
            const PackMeta m = meta[slot];
            if (m.valid && dy < m.kv * m.ny) {
                if (m.r != c_r) {
                    c_r = m.r;
                    c_part = runs[m.r].a.part;
                    c_ncg = runs[m.r].a.n_cg;
                }
                if (m.ny != c_ny) {
                    c_ny = m.ny;
                    kd = dy / m.ny;
                    yd = dy - kd * m.ny;
                }
                const float4* rw = reinterpret_cast<const float4*>(stage + ((size_t)slot * XB_SROWS + dy) * CG);
                const int sw = dy & 7;
                double t[2];
#pragma unroll
                for (int k = 0; k < 2; ++k) {  // two halves of 16 columns, each a fixed tree
                    const float4 u0 = rw[(4 * k) ^ sw], u1 = rw[(4 * k + 1) ^ sw], u2 = rw[(4 * k + 2) ^ sw],
                                 u3 = rw[(4 * k + 3) ^ sw];
                    t[k] = ((((double)u0.x + (double)u0.y) + ((double)u0.z + (double)u0.w)) +
                            (((double)u1.x + (double)u1.y) + ((double)u1.z + (double)u1.w))) +
                           ((((double)u2.x + (double)u2.y) + ((double)u2.z + (double)u2.w)) +
                            (((double)u3.x + (double)u3.y) + ((double)u3.z + (double)u3.w)));
                }
                c_part[((int64_t)m.x * c_ncg + m.cg0 + kd) * m.ny + yd] = t[0] + t[1];
            }
        }
    };

    // the register budget of each role holds inside its own branch
    if (drift) {
        // the half-box issuers' second x row needs the larger density budget
        if constexpr (HALF)
            asm volatile("setmaxnreg.inc.sync.aligned.u32 208;" ::: "memory");
        else
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
        int yoff = 0, y0 = 0, kg = 0, ny = 0;
        bool act = false;  // this warp has rows of a valid group of the pack
        float* outp = nullptr;
        int64_t m = 0;
        auto tables = [&]() {
            const Args& a = runs[cons.r].a;
            ny = cons.ny;
            const int wpg = (ny + YT2 - 1) / YT2;
            kg = warp / wpg;
            y0 = (warp - kg * wpg) * YT2;
            act = kg < cons.kv;
            outp = a.out;
            m = a.m;
            if (act) {
                const int cg = cons.cg0 + kg;
                const int jx = ((cg * CG + lane) / a.nvy) % a.nvx;  // per lane: a group may span two vx
                const int jy = (cg * CG + lane) % a.nvy;
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    const float u = __ldg(a.W_x + (5 - j) * a.nvx + jx), v = __ldg(a.W_y + (5 - j) * a.nvy + jy);
                    wx[j] = make_float2(u, u);
                    wy[j] = make_float2(v, v);
                }
                int r = (y0 - __ldg(a.shift_y + jy) - 3) % ny;
                if (r < 0) r += ny;
                // the lane's box (BW columns, rows BW floats apart)
                yoff = kg * (ny + HALO2) * CG + (lane / BW) * (ny + HALO2) * BW + r * BW + (lane % BW);
            }
        };
        tables();

        auto body = [&](auto step) -> bool {
            constexpr int P = decltype(step)::value;
            bool ok = true;
            const bool emit = cons.q >= 5;
            const int slot = 2 * pp + (P & 1);
            const int x = cons.q - 5;
            if (act) {
                ok = wait_phase(bar0 + 8 * P, parity);
                const float* sl = slabs + P * slab_floats + yoff;
#pragma unroll
                for (int p = 0; p < WR / 2; ++p) win[p][P] = make_float2(sl[(2 * p) * BW], sl[(2 * p + 1) * BW]);
                wl[P] = sl[(WR - 1) * BW];
                if (emit) {
                    float xd[WR];
#pragma unroll
                    for (int p = 0; p < WR / 2; ++p) {
                        const float2 o = taps(wx, win[p][(P + 1) % 6], win[p][(P + 2) % 6], win[p][(P + 3) % 6],
                                              win[p][(P + 4) % 6], win[p][(P + 5) % 6], win[p][P]);
                        xd[2 * p] = o.x;
                        xd[2 * p + 1] = o.y;
                    }
                    xd[WR - 1] = tap1(wx, wl[(P + 1) % 6], wl[(P + 2) % 6], wl[(P + 3) % 6], wl[(P + 4) % 6],
                                      wl[(P + 5) % 6], wl[P]);
                    float o16[YT2];
#pragma unroll
                    for (int p = 0; p < YT2 / 2; ++p) {
                        const int i = 2 * p;
                        const float2 o = taps(wy, make_float2(xd[i], xd[i + 1]), make_float2(xd[i + 1], xd[i + 2]),
                                              make_float2(xd[i + 2], xd[i + 3]), make_float2(xd[i + 3], xd[i + 4]),
                                              make_float2(xd[i + 4], xd[i + 5]), make_float2(xd[i + 5], xd[i + 6]));
                        o16[i] = o.x;
                        o16[i + 1] = o.y;
                    }
                    float* dst = outp + ((int64_t)x * ny + y0) * m + (int64_t)(cons.cg0 + kg) * CG + lane;
                    float* st = stage + ((size_t)slot * XB_SROWS + kg * ny + y0) * CG;
                    (void)st;
                    if (y0 + YT2 <= ny) {  // warp-uniform: all 16 rows are real
#pragma unroll
                        for (int e = 0; e < YT2; ++e) {
                            dst[(int64_t)e * m] = o16[e];
                            if constexpr (RHO) st[e * CG + (lane ^ ((e & 7) << 2))] = o16[e];
                        }
                    } else {
#pragma unroll
                        for (int e = 0; e < YT2; ++e)
                            if (y0 + e < ny) {
                                dst[(int64_t)e * m] = o16[e];
                                if constexpr (RHO) st[e * CG + (lane ^ ((e & 7) << 2))] = o16[e];
                            }
                    }
                }
            }
            if (tid == 0) {
                meta[slot] = PackMeta{x, cons.r, cons.cg0, cons.kv, cons.ny, emit ? 1 : 0, 0, 0};
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
            return cons.step_on();
        };
        for (int p0 = 0;;) {
            const int pe = run_steps(body, p0);
            if (failed) break;
            cons.next_pack(runs, start, n_runs);
            if (!cons.valid()) break;
            tables();
            p0 = (pe + 1) % DEPTH;
        }
        // a wait on a last, even row has had no barrier vote yet
        if (!failed && __syncthreads_or(!okacc)) failed = true;
        if (failed) {
            // the whole share reads NaN (after this barrier no store of a
            // row lands any more)
            __syncthreads();
            PSeq z;
            z.init(runs, start, n_runs, (int)blockIdx.x, (int)gridDim.x);
            while (z.valid()) {
                const int wpg = (z.ny + YT2 - 1) / YT2;
                const int zk = warp / wpg, zy0 = (warp - zk * wpg) * YT2;
                if (tid == 0 && z.q == 0 && runs[z.r].a.status)  // every run this CTA served
                    atomicOr(runs[z.r].a.status, VP_STATUS_WAIT_TIMEOUT);
                if (z.q >= 5 && zk < z.kv) {
                    const Args& za = runs[z.r].a;
                    const int x = z.q - 5;
                    for (int i = 0; i < YT2 && zy0 + i < z.ny; ++i) {
                        za.out[((int64_t)x * z.ny + zy0 + i) * za.m + (int64_t)(z.cg0 + zk) * CG + lane] = NAN;
                        if (RHO && lane == 0)
                            za.part[((int64_t)x * za.n_cg + z.cg0 + zk) * z.ny + zy0 + i] = (double)NAN;
                    }
                }
                z.next(runs, start, n_runs);
            }
        }
    } else {
        if constexpr (HALF)
            asm volatile("setmaxnreg.dec.sync.aligned.u32 88;" ::: "memory");
        else
            asm volatile("setmaxnreg.dec.sync.aligned.u32 72;" ::: "memory");
        const bool issuer = (dy & 31) == 0;  // first lane of density warp kq issues group kq
        const int kq = dy >> 5;
        PSeq qs{};                  // the issuer's copy of the sequence
        int q_r0 = 0, q_r1 = 0;     // its group's halves: -(x shift) - 3
        long long q_issued = 0;
        if (issuer) {
            qs = prod->seq;
            q_r0 = kq < 4 ? prod->r0[2 * kq] : 0;
            q_r1 = kq < 4 ? prod->r0[2 * kq + 1] : 0;
            q_issued = prod->issued;
        }
        auto issue_q = [&](int d) {
            const uint32_t box = (uint32_t)((qs.ny + HALO2) * CG * 4), bar = bar0 + 8 * d;
            if (kq == 0) expect_bytes(bar, box * (uint32_t)qs.kv);
            if (kq < qs.kv) {
#pragma unroll
                for (int h = 0; h < NB; ++h) {
                    int v = ((h ? q_r1 : q_r0) + qs.q) % qs.nx;
                    if (v < 0) v += qs.nx;
                    const uint32_t dst = slab0 + (uint32_t)d * slab_bytes + (uint32_t)kq * box + (uint32_t)h * box / NB;
                    const int c0 = (qs.cg0 + kq) * CG + h * BW;
                    tma_load(&maps.tin[qs.r], dst, bar, c0, v * qs.ny);
                    tma_load(&maps.thalo[qs.r], dst + (uint32_t)(qs.ny * BW * 4), bar, c0, v * qs.ny);
                }
            }
            q_issued += 1;
            if (!qs.step_on()) {
                qs.next_pack(runs, start, n_runs);
                if (qs.valid() && kq < qs.kv) {
                    const Args& a = runs[qs.r].a;
                    const int c0 = (qs.cg0 + kq) * CG;
                    q_r0 = -__ldg(a.shift_x + (c0 / a.nvy) % a.nvx) - 3;
                    if (HALF) q_r1 = -__ldg(a.shift_x + ((c0 + HB) / a.nvy) % a.nvx) - 3;
                }
            }
        };
        // the density warpgroup: the same steps and barriers, no waits
        auto body = [&](auto step) -> bool {
            constexpr int P = decltype(step)::value;
            if (P & 1) {
                if (__syncthreads_or(0)) {
                    failed = true;
                    return false;
                }
                if (issuer) {  // slabs P-1 and P are free
#pragma unroll
                    for (int d = P - 1; d <= P; ++d)
                        if (qs.valid()) issue_q(d);
                }
                if constexpr (RHO) density(pp);
                pp ^= 1;
            }
            if (P == DEPTH - 1) parity ^= 1u;
            ++L;
            return cons.step_on();
        };
        for (int p0 = 0;;) {
            const int pe = run_steps(body, p0);
            if (failed) break;
            cons.next_pack(runs, start, n_runs);
            if (!cons.valid()) break;
            p0 = (pe + 1) % DEPTH;
        }
        // the drift warps' last vote (the same barrier, reached from their branch)
        if (!failed && __syncthreads_or(0)) failed = true;
        if constexpr (RHO)
            if (!failed && (L & 1)) density(pp);  // the last, single row
        if (failed) {
            __syncthreads();  // pairs with the drift warps' barrier before their NaN fill
            if (tid == PTID) {
                // the loads in flight land before the block leaves
                for (long long k = L; k < q_issued; ++k)
                    wait_phase(bar0 + 8 * (int)(k % DEPTH), (uint32_t)((k / DEPTH) & 1));
            }
        }
    }
}

template <bool RHO, bool HALF>
__global__ void __launch_bounds__(XRD_THREADS, 1)
    k_plane_xrd_batch(const __grid_constant__ XBMaps maps, const PlaneRun* __restrict__ runs,
                      const int64_t* __restrict__ start, int n_runs, int slab_floats) {
    pdl_release();
    xrd_batch_body<RHO, HALF>(maps, runs, start, n_runs, slab_floats);
    pdl_hold();
}

// ---- many runs, y then x ---------------------------------------------------
// The batched y-first pass in the form of k_plane<0>: 8 warps of 8 y rows, each
// thread's y drift from 13 rows of the slab, then the 6-row x window of
// y-drifted rows in registers; two CTAs per SM. A CTA steps a pack of K =
// 8 / ceil(ny / 8) column groups of one run through x together (two groups
// of up to 32 rows, else one), warp w on group w / wpg, rows 8 (w % wpg) ..
// +7; each step loads K boxes of ny + 16 rows. The first thread issues the
// loads, two slabs after every second row's block barrier.
constexpr int YB_MAX_SLAB_ROWS = 2 * (32 + HALO);
constexpr int yb_pack(int ny) { return 8 / ((ny + YT - 1) / YT); }

__host__ __device__ constexpr size_t yx_batch_smem_bytes(int slab_rows) {
    return (size_t)DEPTH * slab_rows * CG * 4 + DEPTH * 8 + 2 * sizeof(XBProducer);
}

template <bool HALF>
__device__ __forceinline__ void yx_batch_body(const XBMaps& maps, const PlaneRun* __restrict__ runs,
                                              const int64_t* __restrict__ start, int n_runs, int slab_floats) {
    extern __shared__ __align__(1024) unsigned char smem[];
    float* slabs = reinterpret_cast<float*>(smem);  // [DEPTH][slab_floats]
    uint64_t* bars = reinterpret_cast<uint64_t*>(slabs + DEPTH * slab_floats);
    XBProducer* prod = reinterpret_cast<XBProducer*>(bars + DEPTH);  // [2]: one per issuer
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    PSeq cons;
    cons.init(runs, start, n_runs, (int)blockIdx.x, (int)gridDim.x);
    if (!cons.valid()) return;
    const uint32_t slab0 = smem_u32(slabs), bar0 = smem_u32(bars);
    const uint32_t slab_bytes = (uint32_t)slab_floats * 4u;
    constexpr int BW = HALF ? HB : CG, NB = CG / BW;  // box columns, boxes per group
    auto pack_rows = [&]() {
        const PSeq& s = prod->seq;
        const Args& a = runs[s.r].a;
        for (int k = 0; k < s.kv; ++k)
            for (int h = 0; h < NB; ++h)
                prod->r0[2 * k + h] = -__ldg(a.shift_x + (((s.cg0 + k) * CG + h * BW) / a.nvy) % a.nvx) - 3;
    };
    uint32_t extra = 0;  // test hook: the first load of the CTA expects 16 bytes too many
    auto issue = [&](int d) {
        const PSeq& s = prod->seq;
        const CUtensorMap* tin = &maps.tin[s.r];
        const CUtensorMap* thalo = &maps.thalo[s.r];
        const uint32_t box = (uint32_t)((s.ny + HALO) * CG * 4), bar = bar0 + 8 * d;
        expect_bytes(bar, box * (uint32_t)s.kv + extra);
        extra = 0;
        for (int k = 0; k < s.kv; ++k)
            for (int h = 0; h < NB; ++h) {
                int v = (prod->r0[2 * k + h] + s.q) % s.nx;
                if (v < 0) v += s.nx;
                const uint32_t dst = slab0 + (uint32_t)d * slab_bytes + (uint32_t)k * box + (uint32_t)h * box / NB;
                const int c0 = (s.cg0 + k) * CG + h * BW;
                tma_load(tin, dst, bar, c0, v * s.ny);
                tma_load(thalo, dst + (uint32_t)(s.ny * BW * 4), bar, c0, v * s.ny);
            }
    };
    auto advance = [&]() {
        prod->seq.next(runs, start, n_runs);
        if (prod->seq.valid() && prod->seq.q == 0) pack_rows();
    };
    // after the first DEPTH steps: the first lane of warp 7 - k issues group
    // k's loads (k < 2), warp 7's arming the barrier with the step's bytes;
    // each issuer steps its own copy of the sequence (in shared memory). One
    // thread issuing a step's four loads had put its warp on the path to
    // every second row's barrier.
    auto issue_q = [&](XBProducer& q, int kq, int d) {
        const PSeq& qs = q.seq;
        const uint32_t box = (uint32_t)((qs.ny + HALO) * CG * 4), bar = bar0 + 8 * d;
        if (kq == 0) expect_bytes(bar, box * (uint32_t)qs.kv);
        if (kq < qs.kv)
            for (int h = 0; h < NB; ++h) {
                int v = (q.r0[2 * kq + h] + qs.q) % qs.nx;
                if (v < 0) v += qs.nx;
                const uint32_t dst = slab0 + (uint32_t)d * slab_bytes + (uint32_t)kq * box + (uint32_t)h * box / NB;
                const int c0 = (qs.cg0 + kq) * CG + h * BW;
                tma_load(&maps.tin[qs.r], dst, bar, c0, v * qs.ny);
                tma_load(&maps.thalo[qs.r], dst + (uint32_t)(qs.ny * BW * 4), bar, c0, v * qs.ny);
            }
        q.issued += 1;
        if (!q.seq.step_on()) {
            q.seq.next_pack(runs, start, n_runs);
            if (q.seq.valid() && kq < q.seq.kv) {
                const Args& a = runs[q.seq.r].a;
                for (int h = 0; h < NB; ++h)
                    q.r0[2 * kq + h] = -__ldg(a.shift_x + (((q.seq.cg0 + kq) * CG + h * BW) / a.nvy) % a.nvx) - 3;
            }
        }
    };
    if (tid == 0) {
        for (int d = 0; d < DEPTH; ++d) bar_init(bar0 + 8 * d);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        prod->seq = cons;
        extra = runs[cons.r].a.stall ? 16u : 0u;
        pack_rows();
        long long n = 0;
        for (; n < DEPTH && prod->seq.valid(); ++n) {
            issue((int)n);
            advance();
        }
        prod->issued = n;
        prod[1] = prod[0];
    }
    __syncthreads();

    float2 win[YT / 2][6];
#pragma unroll
    for (int p = 0; p < YT / 2; ++p)
#pragma unroll
        for (int s = 0; s < 6; ++s) win[p][s] = make_float2(0.f, 0.f);
    float2 wx[6], wy[6];
    int yoff = 0, y0 = 0, kg = 0, ny = 0;
    bool act = false;
    float* outp = nullptr;
    int64_t m = 0;
    uint32_t parity = 0;
    long long L = 0;
    bool failed = false, okacc = true;
    auto tables = [&]() {
        const Args& a = runs[cons.r].a;
        ny = cons.ny;
        const int wpg = (ny + YT - 1) / YT;
        kg = warp / wpg;
        y0 = (warp - kg * wpg) * YT;
        act = kg < cons.kv;
        outp = a.out;
        m = a.m;
        if (act) {
            const int cg = cons.cg0 + kg;
            const int jx = ((cg * CG + lane) / a.nvy) % a.nvx;  // per lane: a group may span two vx
            const int jy = (cg * CG + lane) % a.nvy;
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                const float u = __ldg(a.W_x + (5 - j) * a.nvx + jx), v = __ldg(a.W_y + (5 - j) * a.nvy + jy);
                wx[j] = make_float2(u, u);
                wy[j] = make_float2(v, v);
            }
            int r = (y0 - __ldg(a.shift_y + jy) - 3) % ny;
            if (r < 0) r += ny;
            // the lane's box (BW columns, rows BW floats apart)
            yoff = kg * (ny + HALO) * CG + (lane / BW) * (ny + HALO) * BW + r * BW + (lane % BW);
        }
    };
    tables();

    auto body = [&](auto step) -> bool {
        constexpr int P = decltype(step)::value;
        bool ok = true;
        if (act) {
            ok = wait_phase(bar0 + 8 * P, parity);
            float2 nv[YT / 2];
            y_drift<false, BW>(slabs + P * slab_floats + yoff, wy, 0.f, nv);
            if (cons.q >= 5) {
                float* dst = outp + ((int64_t)(cons.q - 5) * ny + y0) * m + (int64_t)(cons.cg0 + kg) * CG + lane;
                float2 o[YT / 2];
#pragma unroll
                for (int p = 0; p < YT / 2; ++p)
                    o[p] = taps(wx, win[p][(P + 1) % 6], win[p][(P + 2) % 6], win[p][(P + 3) % 6],
                                win[p][(P + 4) % 6], win[p][(P + 5) % 6], nv[p]);
                if (y0 + YT <= ny) {  // warp-uniform: all 8 rows are real
#pragma unroll
                    for (int p = 0; p < YT / 2; ++p) {
                        dst[(int64_t)(2 * p) * m] = o[p].x;
                        dst[(int64_t)(2 * p + 1) * m] = o[p].y;
                    }
                } else {
#pragma unroll
                    for (int p = 0; p < YT / 2; ++p) {
                        const int y = y0 + 2 * p;
                        if (y < ny) dst[(int64_t)(2 * p) * m] = o[p].x;
                        if (y + 1 < ny) dst[(int64_t)(2 * p + 1) * m] = o[p].y;
                    }
                }
            }
#pragma unroll
            for (int p = 0; p < YT / 2; ++p) win[p][P] = nv[p];
        }
        okacc = okacc && ok;
        if (P & 1) {
            // slabs P-1 and P are free
            if (__syncthreads_or(!okacc)) {
                failed = true;
                return false;
            }
            if (lane == 0 && warp >= 6) {
                const int kq = 7 - warp;
                XBProducer& q = prod[kq];
#pragma unroll
                for (int d = P - 1; d <= P; ++d)
                    if (q.seq.valid()) issue_q(q, kq, d);
            }
        }
        if (P == DEPTH - 1) parity ^= 1u;
        ++L;
        return cons.step_on();
    };

    for (int p0 = 0;;) {
        const int pe = run_steps(body, p0);
        if (failed) break;
        cons.next_pack(runs, start, n_runs);
        if (!cons.valid()) break;
        tables();
        p0 = (pe + 1) % DEPTH;
    }
    // a wait on a last, even row has had no barrier vote yet
    if (!failed && __syncthreads_or(!okacc)) failed = true;
    if (failed) {
        // the whole share reads NaN, then the loads in flight land
        __syncthreads();
        PSeq z;
        z.init(runs, start, n_runs, (int)blockIdx.x, (int)gridDim.x);
        while (z.valid()) {
            const int wpg = (z.ny + YT - 1) / YT;
            const int zk = warp / wpg, zy0 = (warp - zk * wpg) * YT;
            if (tid == 0 && z.q == 0 && runs[z.r].a.status)  // every run this CTA served
                atomicOr(runs[z.r].a.status, VP_STATUS_WAIT_TIMEOUT);
            if (z.q >= 5 && zk < z.kv) {
                const Args& za = runs[z.r].a;
                const int x = z.q - 5;
                for (int i = 0; i < YT && zy0 + i < z.ny; ++i)
                    za.out[((int64_t)x * z.ny + zy0 + i) * za.m + (int64_t)(z.cg0 + zk) * CG + lane] = NAN;
            }
            z.next(runs, start, n_runs);
        }
        if (tid == 0)
            for (long long k = L; k < prod->issued; ++k)
                wait_phase(bar0 + 8 * (int)(k % DEPTH), (uint32_t)((k / DEPTH) & 1));
    }
}

template <bool HALF>
__global__ void __launch_bounds__(8 * 32, 2)
    k_plane_yx_batch(const __grid_constant__ XBMaps maps, const PlaneRun* __restrict__ runs,
                     const int64_t* __restrict__ start, int n_runs, int slab_floats) {
    pdl_release();
    yx_batch_body<HALF>(maps, runs, start, n_runs, slab_floats);
    pdl_hold();
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
static bool make_map(CUtensorMap* tm, const void* base, int64_t m, int64_t rows_total, int box_rows,
                     int box_cols = CG) {
    const cuuint64_t dims[2] = {(cuuint64_t)m, (cuuint64_t)rows_total};
    const cuuint64_t strides[1] = {(cuuint64_t)(m * sizeof(float))};
    const cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
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


// the parameter copies of the runs' tensor maps, launched per XB_MAXR runs
template <typename Kern>
static int launch_runs(Kern kern, int block, size_t smem, const PlaneRun* runs, const PlaneRun* runs_host,
                       const int64_t* start, const int64_t* start_host, int n_runs, int per_sm, int slab_rows,
                       bool* first, cudaStream_t st, const char* name) {
    XBMaps maps;  // host staging of the parameter (the launch copies it)
    std::memset(static_cast<void*>(&maps), 0, sizeof(maps));
    const char* hb = reinterpret_cast<const char*>(runs_host);  // the host table need not be 64-byte aligned
    for (int r0 = 0; r0 < n_runs; r0 += XB_MAXR) {
        const int nr = std::min(XB_MAXR, n_runs - r0);
        const int64_t items = start_host[r0 + nr] - start_host[r0];
        if (items <= 0) continue;
        for (int i = 0; i < nr; ++i) {
            const char* rec = hb + (size_t)(r0 + i) * sizeof(PlaneRun);
            std::memcpy(static_cast<void*>(&maps.tin[i]), rec + offsetof(PlaneRun, tin), sizeof(CUtensorMap));
            std::memcpy(static_cast<void*>(&maps.thalo[i]), rec + offsetof(PlaneRun, thalo), sizeof(CUtensorMap));
        }
        const int64_t grid = std::min<int64_t>(items, (int64_t)sm_count() * per_sm);
        // every launch of the pass after its first one as a programmatic
        // dependent of the launch before it
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)grid);
        cfg.blockDim = dim3((unsigned)block);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cfg.attrs = attr;
        cfg.numAttrs = *first ? 0 : 1;
        *first = false;
        const cudaError_t le = cudaLaunchKernelEx(&cfg, kern, maps, runs + r0, start + r0, nr, slab_rows * CG);
        int rc = check_launch(name);
        if (!rc && le != cudaSuccess) rc = set_error(VP_ERR_CUDA, "plane batch: cudaLaunchKernelEx failed");
        if (rc) return rc;
    }
    return VP_OK;
}

template <bool HALF>
static int launch_yx_batch(const PlaneRun* runs, const PlaneRun* runs_host, const int64_t* start,
                           const int64_t* start_host, int n_runs, int slab_rows, bool* first, cudaStream_t st) {
    auto kern = k_plane_yx_batch<HALF>;
    const size_t smem = yx_batch_smem_bytes(slab_rows);
    static int raised[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return set_error(VP_ERR_CUDA, "plane batch: device index out of range");
    if (!raised[dev]) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)yx_batch_smem_bytes(YB_MAX_SLAB_ROWS)) != cudaSuccess)
            return set_cuda_error("cudaFuncSetAttribute(k_plane_yx_batch)");
        raised[dev] = 1;
    }
    if (slab_rows < 1 || slab_rows > YB_MAX_SLAB_ROWS) return set_error(VP_ERR_ARG, "plane batch: bad slab rows");
    const int occ = occupancy(kern, 8 * 32, smem);
    if (occ < 1) return set_error(VP_ERR_UNSUPPORTED, "plane batch: the kernel does not fit an SM");
    return launch_runs(kern, 8 * 32, smem, runs, runs_host, start, start_host, n_runs, occ, slab_rows, first, st,
                       "k_plane_yx_batch");
}

template <bool RHO, bool HALF>
static int launch_xrd_batch_t(const PlaneRun* runs, const PlaneRun* runs_host, const int64_t* start,
                              const int64_t* start_host, int n_runs, int slab_rows, bool* first, cudaStream_t st) {
    auto kern = k_plane_xrd_batch<RHO, HALF>;
    const size_t smem = xrd_batch_smem_bytes(slab_rows);
    static int raised[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return set_error(VP_ERR_CUDA, "plane batch: device index out of range");
    if (!raised[dev]) {
        // once, for the largest layout any batch can ask for
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)xrd_batch_smem_bytes(XB_MAX_SLAB_ROWS)) != cudaSuccess)
            return set_cuda_error("cudaFuncSetAttribute(k_plane_xrd_batch)");
        raised[dev] = 1;
    }
    if (slab_rows < 1 || slab_rows > XB_MAX_SLAB_ROWS) return set_error(VP_ERR_ARG, "plane batch: bad slab rows");
    return launch_runs(kern, XRD_THREADS, smem, runs, runs_host, start, start_host, n_runs, 1, slab_rows, first,
                       st, "k_plane_xrd_batch");
}

}  // namespace plane

size_t plane_run_bytes() { return sizeof(plane::PlaneRun); }

// Runs of 32..64 rows, a multiple of 8 (the packs of the x-first pass stage
// whole 8-row swizzle blocks), nvy a multiple of 16. The packed passes take
// 20..64 rows; below 32 they lose to the sweeps (24^4 batches: 1.565 against
// 1.135 ms a step), the x window's 5 warm-up rows of every line adding a
// fifth to the loads.
bool plane_batch_fits(int dtype, int64_t nx, int64_t ny, int64_t nvx, int64_t nvy, const void* a, const void* b,
                      const void* c) {
    using namespace plane;
    if (dtype != VP_F32 || ny < 32 || ny > YMAX / 2 || ny % 8 != 0 || nx < 1 || nvx < 1) return false;
    // groups of 32 columns in half boxes of 16, each inside one vx
    if (nvy % HB != 0 || (nvx * nvy) % CG != 0) return false;
    if ((int64_t)nx * ny >= (1ll << 31) || nvx * nvy >= (1ll << 31) || nvx * nvy / CG * nx >= (1ll << 31)) return false;
    for (const void* p : {a, b, c})
        if (reinterpret_cast<uintptr_t>(p) % 16 != 0) return false;
    return encoder() != nullptr;
}

int plane_batch_run(void* record, bool xfirst, const void* in, void* out, int64_t nx, int64_t ny, int64_t nvx,
                    int64_t nvy, const int* shift_x, const void* W_x, const int* shift_y, const void* W_y,
                    double* part, int* status, int stall, int64_t* items, int* slab_rows) {
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
    a.status = status;
    a.stall = stall;
    // x first: packs of xb_pack(ny) groups, boxes of ny + 20 rows; y first:
    // packs of yb_pack(ny) groups, boxes of ny + 16 rows
    const int halo = xfirst ? HALO2 : HALO;
    pr->k_pack = xfirst ? xb_pack((int)ny) : yb_pack((int)ny);
    pr->slab_rows = pr->k_pack * ((int)ny + halo);
    if (ny < HALO2 || ny % 8 != 0 || pr->slab_rows > (xfirst ? XB_MAX_SLAB_ROWS : YB_MAX_SLAB_ROWS))
        return set_error(VP_ERR_UNSUPPORTED, "plane batch: rows outside the packed layouts");
    // runs whose 32-column groups may span two vx (nvy % 32 != 0) take their
    // groups in two half boxes, each at its own x row
    const int bc = nvy % CG ? HB : CG;
    if (!make_map(&pr->tin, in, a.m, nx * ny, (int)ny, bc) || !make_map(&pr->thalo, in, a.m, nx * ny, halo, bc))
        return set_error(VP_ERR_CUDA, "plane batch: cuTensorMapEncodeTiled failed");
    std::memcpy(record, &rec, sizeof(PlaneRun));
    *items = (a.n_cg + pr->k_pack - 1) / pr->k_pack;
    *slab_rows = pr->slab_rows;
    return VP_OK;
}

int launch_plane_batch(bool xfirst, bool rho, const void* runs, const void* runs_host, const int64_t* start,
                       const int64_t* start_host, int n_full, int n_runs, int64_t items, int slab_rows,
                       cudaStream_t st) {
    using namespace plane;
    if (items <= 0) return VP_OK;
    const PlaneRun* pr = static_cast<const PlaneRun*>(runs);
    const PlaneRun* ph = static_cast<const PlaneRun*>(runs_host);
    // records 0 .. n_full - 1 in whole 32-column boxes, the rest in half boxes;
    // the launches after the first start as its CTAs leave the SMs
    bool first = true;
    for (int half = 0; half < 2; ++half) {
        const int r0 = half ? n_full : 0, nr = half ? n_runs - n_full : n_full;
        if (nr <= 0 || start_host[r0 + nr] == start_host[r0]) continue;
        const PlaneRun *q = pr + r0, *qh = ph + r0;
        const int64_t *sq = start + r0, *sqh = start_host + r0;
        int rc;
        if (!xfirst)
            rc = half ? launch_yx_batch<true>(q, qh, sq, sqh, nr, slab_rows, &first, st)
                      : launch_yx_batch<false>(q, qh, sq, sqh, nr, slab_rows, &first, st);
        else if (rho)
            rc = half ? launch_xrd_batch_t<true, true>(q, qh, sq, sqh, nr, slab_rows, &first, st)
                      : launch_xrd_batch_t<true, false>(q, qh, sq, sqh, nr, slab_rows, &first, st);
        else
            rc = half ? launch_xrd_batch_t<false, true>(q, qh, sq, sqh, nr, slab_rows, &first, st)
                      : launch_xrd_batch_t<false, false>(q, qh, sq, sqh, nr, slab_rows, &first, st);
        if (rc) return rc;
    }
    return VP_OK;
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
