// Semi-Lagrangian sweeps of the Vlasov-Poisson step on sm_100a.
//
// Every sweep is HBM-bound (6 FMAs per element against 2 x sizeof(f) bytes),
// so the kernels are written to move each element of f exactly once in and
// once out, with wide coalesced accesses on the contiguous axis:
//
//  * k_strided: sweep along a strided axis (x, y, vx of 2D2V; x of 1D1V).
//    Lanes run across the contiguous columns; each thread walks its column
//    down the advected axis with a 6-row sliding window held in registers,
//    loading U rows per chunk so that U independent 4/8/16-byte loads per
//    thread are in flight. A full periodic line re-uses its first 5 rows for
//    the wrap instead of reading them twice. No shared-memory staging is
//    needed: the window is the halo. Optional epilogue: FP64 sum over the
//    columns of every output row (the charge density), reduced through a
//    small per-warp transpose in shared memory, deterministic.
//  * k_kick2d: both velocity kicks of a 2D2V step in one pass over each
//    (x, y) plane: the vx kick is the strided sliding window, its rows go
//    through a per-team shared-memory row buffer for the vy kick.
//  * k_kick_contig: a kick along the contiguous axis (vy alone, v of 1D1V).
//  * k_gather: the general per-element-departure sweep (advect_1d semantics).
//  * k_rho: compute_rho as a standalone reduction.
#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "launch.h"

namespace vp {

constexpr int kU = 8;        // rows per chunk of the sliding window
constexpr int kBlock = 256;  // threads per block of the sweep kernels


// NT = rows of the interpolation window of one output: 6 when the VEC
// columns of a thread share one shift, 7 when their shifts differ by at most
// one (the y drift, whose shift follows vy, the contiguous index): each
// element then gets its own 7-tap weight vector with one zero tap.
// One work item of a strided sweep: a segment of output rows of one tile of
// blockDim.x * VEC columns of one outer row. All threads of the block call it
// with the same item (the moment epilogue synchronises the block).
// KU: rows per chunk of the sliding window (KU loads in flight per thread).
// The 2-byte storage type uses 16 so that a thread keeps as many bytes in
// flight as the 4-byte one (its held rows stay packed, 2 registers per 4
// values); the moment epilogue reduces 8 rows at a time.
template <typename TS, int NT, bool RHO>
__host__ __device__ constexpr int chunk_rows() {
    return sizeof(TS) == 2 ? 16 : kU;
}

template <typename TS, int VEC, int NT, bool KICK, bool RHO, bool WRAPREUSE, bool EQ, int KU = kU>
__device__ __forceinline__ void strided_item(const StridedArgs& a, const int64_t item, unsigned char* smem_raw) {
    using C = compute_t<TS>;
    using V = Vec<TS, VEC>;
    constexpr int NW = NT - 1;  // window rows carried from chunk to chunk
    constexpr int WV = NT == 6 ? 1 : VEC;  // distinct weight vectors per thread
    static_assert(NT == 6 || (NT == 7 && !KICK), "7-row windows are for drifts");
    static_assert(!RHO || KU % 8 == 0, "the moment epilogue reduces 8 rows at a time");
    const TS* __restrict__ in = static_cast<const TS*>(a.in);
    TS* __restrict__ out = static_cast<TS*>(a.out);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5;
    double* wpart = reinterpret_cast<double*>(smem_raw);  // [nwarps][seg] per-warp row sums
    const int n = a.n_line;
    const int64_t ni = a.n_inner;
    {
        int64_t t_ = item;
        const int sg = (int)(t_ % a.nseg);
        t_ /= a.nseg;
        const int tl = (int)(t_ % a.tiles);
        const int64_t o = t_ / a.tiles;
        const int64_t cg = (int64_t)tl * blockDim.x + threadIdx.x;
        const bool active = cg < a.ncg;
        const int l0 = sg * a.seg;
        const int l_end = min(l0 + a.seg, n);
        const int64_t col = active ? cg * VEC : 0;

        // wt[e][j]: weight of window row j (base row l - s_hi - 3) for element e
        C wt[WV][NT];
        int s_hi;
        if constexpr (KICK) {
            C w[6];
            const int64_t ei = o / a.e_div;
            if (a.e_f64)
                s_hi = kick_weights<double, C>(static_cast<const double*>(a.E)[ei], a.dt, a.dv, a.window, w);
            else
                s_hi = kick_weights<float, C>(static_cast<const float*>(a.E)[ei], a.dt, a.dv, a.window, w);
            s_hi = max(-(1 << 28), min(1 << 28, s_hi));
#pragma unroll
            for (int j = 0; j < 6; ++j) wt[0][j] = w[5 - j];
        } else if constexpr (NT == 6) {
            const int jt = (int)((col / a.sel_div) % a.sel_mod);
            s_hi = a.shift[jt];
            const C* Wt = static_cast<const C*>(a.W);
#pragma unroll
            for (int j = 0; j < 6; ++j) wt[0][j] = Wt[(5 - j) * a.sel_mod + jt];
        } else {
            int se[VEC];
            s_hi = -(1 << 30);
#pragma unroll
            for (int e = 0; e < VEC; ++e) {
                const int jt = (int)(((col + e) / a.sel_div) % a.sel_mod);
                se[e] = a.shift[jt];
                s_hi = max(s_hi, se[e]);
            }
            const C* Wt = static_cast<const C*>(a.W);
#pragma unroll
            for (int e = 0; e < VEC; ++e) {
                const int jt = (int)(((col + e) / a.sel_div) % a.sel_mod);
                const bool lo = se[e] != s_hi;  // shift one below the group maximum
#pragma unroll
                for (int j = 0; j < NT; ++j) {
                    // tap k sits at row j = (s_hi - s_e) + 5 - k
                    const C w_same = j <= 5 ? Wt[(5 - j) * a.sel_mod + jt] : C(0);
                    const C w_lo = j >= 1 ? Wt[(6 - j) * a.sel_mod + jt] : C(0);
                    wt[e][j] = lo ? w_lo : w_same;
                }
            }
        }
        // equilibrium split: the drift of feq + g leaves g + feq*(sum w - 1)
        C bias[EQ ? VEC : 1];
        if constexpr (EQ && !KICK) {
            {
#pragma unroll
                for (int e = 0; e < VEC; ++e) {
                    const int64_t c = col + e;
                    const double feq = (a.eqA ? a.eqA[(c / a.eq_nvy) % a.eq_nvx] : 1.0) * a.eqB[c % a.eq_nvy];
                    double wsum = -1.0;
#pragma unroll
                    for (int j = 0; j < NT; ++j) wsum += (double)wt[NT == 6 ? 0 : e][j];
                    bias[e] = C(feq * wsum);
                }
            }
        }
        const TS* src = in + (o * n) * ni + col;
        TS* dst = out + (o * n) * ni + col;
        // FP32 compute: neighbouring elements go through the paired FMA of
        // sm_100 (per lane the same IEEE operations); wp[h][j] holds the tap
        // weights of elements 2h and 2h+1. Not for the 7-row FP32 windows,
        // whose per-element weight pairs would spill (and which are
        // memory-bound anyway); BF16 storage, bound by instructions, pairs both.
        constexpr bool PAIRS = std::is_same<C, float>::value && VEC % 2 == 0 && (NT == 6 || sizeof(TS) == 2);
        float2 wp[PAIRS ? VEC / 2 : 1][NT];
        if constexpr (PAIRS) {
#pragma unroll
            for (int h = 0; h < VEC / 2; ++h)
#pragma unroll
                for (int j = 0; j < NT; ++j)
                    wp[h][j] = make_float2(wt[NT == 6 ? 0 : 2 * h][j], wt[NT == 6 ? 0 : 2 * h + 1][j]);
        }

        using R = typename Raw<TS, VEC>::type;  // a held row (packed for 4 x bf16)
        const R rzero = raw_zero<TS, VEC>();

        V win[NW];
        R first[WRAPREUSE ? NW : 1];
        int rnext;
        if constexpr (!KICK) {
            int64_t r64 = ((int64_t)l0 - s_hi - 3) % n;
            int r = (int)(r64 < 0 ? r64 + n : r64);
#pragma unroll
            for (int j = 0; j < NW; ++j) {
                const R w = active ? ldraw<TS, VEC>(src + (int64_t)r * ni) : rzero;
                win[j] = raw_vec<TS, VEC>(w);
                if constexpr (WRAPREUSE) first[j] = w;
                r = wrap_up(r + 1, n);
            }
            rnext = r;
        } else {
            const int r = l0 - s_hi - 3;
#pragma unroll
            for (int j = 0; j < NW; ++j) {
                const int rr = r + j;
                win[j] = raw_vec<TS, VEC>((active && rr >= 0 && rr < n) ? ldraw<TS, VEC>(src + (int64_t)rr * ni)
                                                                          : rzero);
            }
            rnext = r + NW;
        }

        // rows of the chunk whose first output row is lc (KU loads in flight)
        R nx[KU];
        auto load_chunk = [&](int lc) {
            // whole lines of a multiple of KU rows end on the rows they began with
            const bool last = WRAPREUSE && a.nseg == 1 && (n % KU) == 0 && (lc + KU >= l_end);
#pragma unroll
            for (int u = 0; u < KU; ++u) {
                if constexpr (!KICK) {
                    const int rr = wrap_up(rnext + u, n);
                    if (WRAPREUSE && last && u >= KU - NW)
                        nx[u] = first[WRAPREUSE ? u - (KU - NW) : 0];
                    else
                        nx[u] = active ? ldraw<TS, VEC>(src + (int64_t)rr * ni) : rzero;
                } else {
                    const int rr = rnext + u;
                    nx[u] = (active && rr >= 0 && rr < n) ? ldraw<TS, VEC>(src + (int64_t)rr * ni) : rzero;
                }
            }
            rnext = KICK ? rnext + KU : wrap_up(rnext + KU, n);
        };
        load_chunk(l0);

        // reduce-scatter of 8 row sums over the 32 lanes (fixed order): lane
        // ends with row ((lane>>4)&1)*4 + ((lane>>3)&1)*2 + ((lane>>2)&1) of
        // the 8 rows from l + row0, written to the warp's row partials
        auto reduce8 = [&](const double (&r8)[8], int l, int row0) {
            const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
            double t4[4], t2[2];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const double send = h16 ? r8[i] : r8[i + 4];
                const double keep = h16 ? r8[i + 4] : r8[i];
                t4[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
            }
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const double send = h8 ? t4[i] : t4[i + 2];
                const double keep = h8 ? t4[i + 2] : t4[i];
                t2[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
            }
            double t1;
            {
                const double send = h4 ? t2[0] : t2[1];
                const double keep = h4 ? t2[1] : t2[0];
                t1 = keep + __shfl_xor_sync(0xffffffffu, send, 4);
            }
            t1 += __shfl_xor_sync(0xffffffffu, t1, 2);
            t1 += __shfl_xor_sync(0xffffffffu, t1, 1);
            const int row = row0 + (h16 ? 4 : 0) + (h8 ? 2 : 0) + (h4 ? 1 : 0);
            if ((lane & 3) == 0 && l + row < l_end) wpart[warp * a.seg + (l - l0) + row] = t1;
        };

        for (int l = l0; l < l_end; l += KU) {
            double rs[RHO ? 8 : 1];
            // each output row is stored (and summed) as soon as it is formed
#pragma unroll
            for (int u = 0; u < KU; ++u) {
                V res;
                if constexpr (PAIRS) {
#pragma unroll
                    for (int h = 0; h < VEC / 2; ++h) {
                        auto g2 = [&](int j) -> float2 {
                            return j < NW ? make_float2(win[j].v[2 * h], win[j].v[2 * h + 1])
                                          : make_float2(raw_get<TS, VEC>(nx[j - NW], 2 * h),
                                                        raw_get<TS, VEC>(nx[j - NW], 2 * h + 1));
                        };
                        float2 acc = __fmul2_rn(wp[h][NT - 1], g2(u + NT - 1));
#pragma unroll
                        for (int j = NT - 2; j >= 0; --j) acc = __ffma2_rn(wp[h][j], g2(u + j), acc);
                        if constexpr (EQ) {
                            acc.x += bias[2 * h];
                            acc.y += bias[2 * h + 1];
                        }
                        res.v[2 * h] = acc.x;
                        res.v[2 * h + 1] = acc.y;
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < VEC; ++e) {
                        auto g = [&](int j) -> C { return j < NW ? win[j].v[e] : raw_get<TS, VEC>(nx[j - NW], e); };
                        const int we = NT == 6 ? 0 : e;
                        // ascending stencil tap k = descending window row j
                        C acc = wt[we][NT - 1] * g(u + NT - 1);
#pragma unroll
                        for (int j = NT - 2; j >= 0; --j) acc = fma(wt[we][j], g(u + j), acc);
                        if constexpr (EQ) acc += bias[e];
                        res.v[e] = acc;
                    }
                }
                const bool row_ok = active && l + u < l_end;
                if (row_ok) stv<TS, VEC>(dst + (int64_t)(l + u) * ni, res);
                if constexpr (RHO) {
                    double acc = 0.0;
                    if (row_ok) {
#pragma unroll
                        for (int e = 0; e < VEC; ++e) acc += (double)as_stored<TS>(res.v[e]);
                    }
                    rs[u & 7] = acc;
                    // every completed group of 8 rows but the chunk's last is
                    // reduced at once (the last waits for the next loads)
                    if ((u & 7) == 7 && u + 1 < KU) reduce8(rs, l, u - 7);
                }
            }
#pragma unroll
            for (int j = 0; j < NW; ++j) win[j] = raw_vec<TS, VEC>(nx[KU - NW + j]);
            // next chunk's loads go out before the moment epilogue
            if (l + KU < l_end) load_chunk(l + KU);

            if constexpr (RHO) reduce8(rs, l, KU - 8);
        }

        if constexpr (RHO) {
            __syncthreads();
            for (int ll = threadIdx.x; ll < l_end - l0; ll += blockDim.x) {
                double acc = 0.0;
                for (int wq = 0; wq < nwarps; ++wq) acc += wpart[wq * a.seg + ll];
                a.part[(o * a.tiles + tl) * (int64_t)n + l0 + ll] = acc;
            }
            __syncthreads();
        }
    }
}

template <typename TS, int VEC, int NT, bool KICK, bool RHO, bool WRAPREUSE, bool EQ>
__global__ void __launch_bounds__(kBlock, 2) k_strided(const __grid_constant__ StridedArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    for (int64_t item = blockIdx.x; item < a.items; item += gridDim.x)
        strided_item<TS, VEC, NT, KICK, RHO, WRAPREUSE, EQ, chunk_rows<TS, NT, RHO>()>(a, item, smem_raw);
}

// The same sweep over the items of many runs: run r owns the global items
// [start[r], start[r+1]); a block's items only increase, so its run index
// only moves forward. Launched as a programmatic dependent of a plane pass
// over the batch's other runs, it holds its completion until the pass's.
template <typename TS, int VEC, int NT, bool RHO, bool WRAPREUSE>
__global__ void __launch_bounds__(kBlock, 2)
    k_strided_batch(const StridedArgs* __restrict__ runs, const int64_t* __restrict__ start, int n_runs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int64_t total = start[n_runs];
    int r = 0;
    for (int64_t g = blockIdx.x; g < total; g += gridDim.x) {
        while (r + 1 < n_runs && start[r + 1] <= g) ++r;
        const StridedArgs a = runs[r];
        strided_item<TS, VEC, NT, false, RHO, WRAPREUSE, false, chunk_rows<TS, NT, RHO>()>(a, g - start[r], smem_raw);
    }
    pdl_hold();
}

// rho[o*n + l] = scale * sum_t part[o][t][l]
__global__ void k_rho_finalize(const double* __restrict__ part, int64_t n_outer, int n_line, int tiles,
                               double scale, double offset, double* __restrict__ rho) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_outer * n_line) return;
    const int64_t o = i / n_line;
    const int l = (int)(i % n_line);
    double acc = 0.0;
    for (int t = 0; t < tiles; ++t) acc += part[(o * tiles + t) * (int64_t)n_line + l];
    rho[i] = acc * scale + offset;
}

// ---------------------------------------------------------------------------
// host side of the strided sweeps
// ---------------------------------------------------------------------------
struct StridedPlan {
    int vec, nt;
    int tiles, seg, nseg;
    int64_t ncg, items;
};

// Elements per thread (VEC) and window rows (NT). The VEC consecutive columns
// of a thread share one shift when the table index changes only every sel_div
// columns (and always in a kick); when it changes with every column
// (sel_div == 1), a 7-row window covers groups whose shifts differ by at most
// one, which the caller certifies through `spread` (max over aligned groups of
// 4 table entries of max shift - min shift; negative = unknown).
static void pick_vec(int dtype, int64_t n_inner, int64_t sel_div, int64_t sel_mod, bool kick, int spread,
                     const void* in, const void* out, int* vec, int* nt) {
    const int64_t esz = dtype == VP_F64 ? 8 : (dtype == VP_F32 ? 4 : 2);
    const int v = dtype == VP_F64 ? 2 : 4;
    *vec = 1;
    *nt = 6;
    if (n_inner % v) return;
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) % (v * esz)) return;
    if (kick || sel_div % v == 0) {
        *vec = v;
        return;
    }
    // every column has its own weights here, so the per-element (7-row) form
    // is used even when the integer shifts of a group coincide
    if (sel_div == 1 && sel_mod % 4 == 0 && spread >= 0 && spread <= 1) {
        *vec = v;
        *nt = 7;
    }
}

static StridedPlan plan_strided(int64_t n_outer, int64_t n_line, int64_t n_inner, int vec, int nt,
                                int occ_blocks, int sms, bool rho) {
    StridedPlan p;
    p.vec = vec;
    p.nt = nt;
    p.ncg = n_inner / vec;
    p.tiles = (int)((p.ncg + kBlock - 1) / kBlock);
    // Lines may be split into segments (each costs NT-1 extra halo rows).
    // The number of segments per line minimises waves x (segment + halo)
    // rows, the time of the busiest block slot, with items handed out in
    // waves over the resident slots; ties keep fewer segments.
    const int64_t slots = (int64_t)sms * std::max(occ_blocks, 1);
    const int64_t base = n_outer * p.tiles;
    int seg = (int)n_line;
    int64_t best = -1;
    for (int64_t k = 1; k <= std::min<int64_t>(n_line, 4 * slots); ++k) {
        const int s = (int)((n_line + k - 1) / k);
        if (s < 16 && k > 1) break;
        const int64_t items = base * ((n_line + s - 1) / s);
        const int64_t cost = ((items + slots - 1) / slots) * (s + (k > 1 ? nt - 1 : 0));
        if (best < 0 || cost < best) {
            best = cost;
            seg = s;
        }
    }
    if (rho) seg = std::min(seg, 1024);
    p.seg = seg;
    p.nseg = (int)((n_line + seg - 1) / seg);
    p.items = base * p.nseg;
    return p;
}

template <typename TS, int VEC, int NT, bool KICK, bool RHO, bool EQ>
static int launch_strided_t(StridedArgs a, int sms, cudaStream_t st) {
    // whole periodic lines reuse their first rows for the wrap (not with the
    // moment epilogue, whose prefetched chunk needs the registers)
    constexpr int KU = chunk_rows<TS, NT, RHO>();
    const bool full = (a.nseg == 1) && (a.n_line % KU == 0) && (a.n_line >= KU) && !RHO;
    const size_t smem = RHO ? (size_t)(kBlock / 32) * a.seg * sizeof(double) : 0;
    auto kern = (!KICK && full) ? k_strided<TS, VEC, NT, KICK, RHO, true, EQ>
                                : k_strided<TS, VEC, NT, KICK, RHO, false, EQ>;
    if (smem > 48 * 1024) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return set_cuda_error("cudaFuncSetAttribute(k_strided)");
    }
    const int occ = occupancy(kern, kBlock, smem);
    const int64_t grid = std::min<int64_t>(a.items, (int64_t)sms * occ);
    kern<<<(unsigned)std::max<int64_t>(grid, 1), kBlock, smem, st>>>(a);
    return check_launch("k_strided");
}

template <typename TS, bool KICK, bool RHO, bool EQ>
static int launch_strided_vec(StridedArgs a, int vec, int nt, int sms, cudaStream_t st) {
    constexpr int V = sizeof(TS) == 8 ? 2 : 4;
    if (vec == V) {
        if constexpr (!KICK) {
            if (nt == 7) return launch_strided_t<TS, V, 7, KICK, RHO, EQ>(a, sms, st);
        }
        return launch_strided_t<TS, V, 6, KICK, RHO, EQ>(a, sms, st);
    }
    return launch_strided_t<TS, 1, 6, KICK, RHO, EQ>(a, sms, st);
}

template <bool KICK, bool RHO, bool EQ>
static int launch_strided(int dtype, StridedArgs a, int vec, int nt, int sms, cudaStream_t st) {
    switch (dtype) {
        case VP_F32: return launch_strided_vec<float, KICK, RHO, EQ>(a, vec, nt, sms, st);
        case VP_F64: return launch_strided_vec<double, KICK, RHO, EQ>(a, vec, nt, sms, st);
        case VP_BF16: return launch_strided_vec<__nv_bfloat16, KICK, RHO, EQ>(a, vec, nt, sms, st);
    }
    return set_error(VP_ERR_DTYPE, "unknown dtype");
}

int run_strided(int dtype, const void* in, void* out, int64_t n_outer, int64_t n_line, int64_t n_inner,
                bool kick, int64_t sel_div, int64_t sel_mod, int spread, const int32_t* shift, const void* W,
                const void* E, int e_f64, int64_t e_div, double dt, double dv, int window, double* part,
                int* tiles_out, const EqSplit* eq, cudaStream_t st) {
    const int sms = sm_count();
    const bool rho = part != nullptr || tiles_out != nullptr;
    int vec, nt;
    pick_vec(dtype, n_inner, sel_div, sel_mod, kick, spread, in, out, &vec, &nt);
    const int occ_est = vec > 1 ? 2 : 4;
    StridedPlan p = plan_strided(n_outer, n_line, n_inner, vec, nt, occ_est, sms, rho);
    if (tiles_out) *tiles_out = p.tiles;
    if (tiles_out && !part) return VP_OK;  // plan query only
    StridedArgs a{};
    a.in = in;
    a.out = out;
    a.n_outer = n_outer;
    a.n_line = (int)n_line;
    a.n_inner = n_inner;
    a.ncg = p.ncg;
    a.tiles = p.tiles;
    a.seg = p.seg;
    a.nseg = p.nseg;
    a.items = p.items;
    a.sel_div = sel_div;
    a.sel_mod = (int)sel_mod;
    a.shift = shift;
    a.W = W;
    a.E = E;
    a.e_f64 = e_f64;
    a.e_div = e_div;
    a.dt = dt;
    a.dv = dv;
    a.window = window;
    a.part = part;
    if (eq && eq->B) {
        if (kick) return set_error(VP_ERR_UNSUPPORTED, "equilibrium split: the strided kick has no split form");
        a.eqA = eq->A;
        a.eqB = eq->B;
        a.eq_nvx = eq->nvx > 0 ? eq->nvx : 1;
        a.eq_nvy = eq->nvy;
    }
    if (kick) return launch_strided<true, false, false>(dtype, a, vec, nt, sms, st);
    if (a.eqB) {
        if (rho) return launch_strided<false, true, true>(dtype, a, vec, nt, sms, st);
        return launch_strided<false, false, true>(dtype, a, vec, nt, sms, st);
    }
    if (rho) return launch_strided<false, true, false>(dtype, a, vec, nt, sms, st);
    return launch_strided<false, false, false>(dtype, a, vec, nt, sms, st);
}

// The same sum for many tiles (the fused plane pass writes one partial per
// 32 columns): block (32 lines, 8 slices); slice s adds the tiles
// t = s (mod 8) with four running sums (t = s, s+8, s+16, s+24 mod 32),
// then the 8 slices are added in order. Fixed order, so deterministic.
// The density from many tiles' partials [n_outer][tiles][n_line]: 32 points
// of a line per block, 16 slices of the tiles per point (slice s adds tiles
// s, s + 16, ... into 8 accumulators in turn, so that 8 loads are in flight
// per thread), then the accumulators and the slices in a fixed order.
constexpr int kFinSlices = 16;
__global__ void __launch_bounds__(32 * kFinSlices) k_rho_finalize_wide(const double* __restrict__ part, int n_line,
                                                                      int tiles, double scale, double offset,
                                                                      double* __restrict__ rho) {
    __shared__ double sl[kFinSlices][33];
    const int l = blockIdx.x * 32 + threadIdx.x;
    const int64_t o = blockIdx.y;
    const int sidx = threadIdx.y;
    double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (l < n_line) {
        const double* p = part + (o * tiles) * (int64_t)n_line + l;
        int t = sidx;
        for (; t + 7 * kFinSlices < tiles; t += 8 * kFinSlices) {
            double v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = __ldcs(p + (int64_t)(t + k * kFinSlices) * n_line);
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] += v[k];
        }
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (t + k * kFinSlices < tiles) acc[k] += __ldcs(p + (int64_t)(t + k * kFinSlices) * n_line);
    }
    sl[sidx][threadIdx.x] = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
    __syncthreads();
    if (sidx == 0 && l < n_line) {
        double a = sl[0][threadIdx.x];
#pragma unroll
        for (int k = 1; k < kFinSlices; ++k) a += sl[k][threadIdx.x];
        rho[o * n_line + l] = a * scale + offset;
    }
}

int run_rho_finalize(const double* part, int64_t n_outer, int64_t n_line, int tiles, double scale, double offset,
                     double* rho,
                     cudaStream_t st) {
    if (tiles > 32 && n_outer <= 65535) {
        const dim3 grid((unsigned)((n_line + 31) / 32), (unsigned)n_outer);
        k_rho_finalize_wide<<<grid, dim3(32, kFinSlices), 0, st>>>(part, (int)n_line, tiles, scale, offset, rho);
        return check_launch("k_rho_finalize_wide");
    }
    const int64_t total = n_outer * n_line;
    k_rho_finalize<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(part, n_outer, (int)n_line, tiles, scale, offset,
                                                                      rho);
    return check_launch("k_rho_finalize");
}

// ---------------------------------------------------------------------------
// fused vx + vy kick over [n_planes][nvx][nvy]
// ---------------------------------------------------------------------------

// 4 consecutive compute-type values from shared memory (16-byte aligned)
template <typename C>
__device__ __forceinline__ void lds4(const C* p, C (&v)[4]) {
    if constexpr (sizeof(C) == 4) {
        const float4 t = *reinterpret_cast<const float4*>(p);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else {
        const double2 t = reinterpret_cast<const double2*>(p)[0];
        const double2 u = reinterpret_cast<const double2*>(p)[1];
        v[0] = t.x; v[1] = t.y; v[2] = u.x; v[3] = u.y;
    }
}

template <typename C>
__device__ __forceinline__ void sts4(C* p, const C (&v)[4]) {
    if constexpr (sizeof(C) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
        reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
    }
}

// vy kick of 4 elements from the 12 row values t[0..11] that start at the
// element offset R (static) before the window of the first element
template <int R, typename C>
__device__ __forceinline__ void vy_taps(const C (&t)[12], const C (&wy)[6], C (&o)[4]) {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        C acc = wy[0] * t[R + e + 5];
        acc = fma(wy[1], t[R + e + 4], acc);
        acc = fma(wy[2], t[R + e + 3], acc);
        acc = fma(wy[3], t[R + e + 2], acc);
        acc = fma(wy[4], t[R + e + 1], acc);
        acc = fma(wy[5], t[R + e + 0], acc);
        o[e] = acc;
    }
}

// Rows of a plane per chunk of the fused kick: 4 for 4 doubles per lane (the
// same 128 bytes in flight per thread as 8 rows of 4 floats, in half the
// registers), else 8.
template <typename TS, int VEC>
__host__ __device__ constexpr int kick2d_rows() {
    return (sizeof(TS) == 8 && VEC == 4) ? 4 : kU;
}

// Planes [base, base + teams per block) of a fused kick: one team of lanes
// per plane. All threads of the block call it with the same base.
template <typename TS, int VEC, bool DIAG, bool EQ>
__device__ __forceinline__ void kick2d_item(const Kick2dArgs& a, const int64_t base, unsigned char* smem_raw) {
    using C = compute_t<TS>;
    using V = Vec<TS, VEC>;
    constexpr int KK = kick2d_rows<TS, VEC>();
    const TS* __restrict__ in = static_cast<const TS*>(a.in);
    TS* __restrict__ out = static_cast<TS*>(a.out);
    const int team = a.team;
    const int teams_per_block = blockDim.x / team;
    const int tid_team = threadIdx.x / team;
    const int li = threadIdx.x % team;
    const bool lane_ok = li < a.groups;
    const int nvx = a.nvx, nvy = a.nvy, groups = a.groups;
    C* rowbuf = reinterpret_cast<C*>(smem_raw) + (size_t)tid_team * KK * nvy;
    // equilibrium split: the team's tables of (Kx A - A)(vx) for its plane
    // and of A(vx), after all teams' row buffers
    C* dAt = reinterpret_cast<C*>(smem_raw) + (size_t)teams_per_block * KK * nvy + (size_t)tid_team * 2 * nvx;
    C* At = dAt + nvx;
    // and the block's copy of the equilibrium factors (FP64), after the tables
    const double* eqA = reinterpret_cast<const double*>(reinterpret_cast<C*>(smem_raw) +
                                                        (size_t)teams_per_block * (KK * nvy + 2 * nvx));
    const double* eqB = eqA + nvx;

    double vy2[VEC];
    if constexpr (DIAG) {
#pragma unroll
        for (int e = 0; e < VEC; ++e) {
            const int iv = li * VEC + e;
            const double v = (lane_ok && iv < nvy) ? a.vy[iv] : 0.0;
            vy2[e] = v * v;
        }
    }
    V zero;
#pragma unroll
    for (int e = 0; e < VEC; ++e) zero.v[e] = C(0);

    (void)teams_per_block;
    {
        const int64_t p = base + tid_team;
        const bool pv = p < a.n_planes;
        const bool active = pv && lane_ok;
        C wx[6], wy[6];
        double wxd[6], wyd[6];
        int sx = 0, sy = 0;
        if (pv) {
            sx = kick_weights<double, double>(a.Ex[p], a.dt, a.dvx, a.window, wxd);
            sy = kick_weights<double, double>(a.Ey[p], a.dt, a.dvy, a.window, wyd);
        } else {
#pragma unroll
            for (int k = 0; k < 6; ++k) wxd[k] = wyd[k] = 0.0;
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            wx[k] = C(wxd[k]);
            wy[k] = C(wyd[k]);
        }
        sx = max(-(1 << 28), min(1 << 28, sx));
        sy = max(-(1 << 28), min(1 << 28, sy));
        float2 wx2[6];  // the vx weights paired, for the paired FMA (FP32 compute)
#pragma unroll
        for (int k = 0; k < 6; ++k) wx2[k] = make_float2((float)wx[k], (float)wx[k]);
        // equilibrium split: the kicks of feq = A(vx) B(vy) add
        // (Kx A - A)(vx) B(vy) after the vx kick and A(vx) (Ky B - B)(vy) after
        // the vy kick (K: the plane's kick operator, zero outside the grid).
        // Both factors are evaluated in FP64 and rounded to the compute type;
        // each term is one more FMA after the element's 6 taps.
        double Be[EQ ? VEC : 1], dBe[EQ ? VEC : 1];
        C Bc[EQ ? VEC : 1], dBc[EQ ? VEC : 1];
        auto eq_factors = [&]() {
#pragma unroll
            for (int e = 0; e < VEC; ++e) {
                const int iv = li * VEC + e;
                Be[e] = (lane_ok && iv < nvy) ? eqB[iv] : 0.0;
                double k_b = 0.0;
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    const int j = iv - sy + 2 - k;
                    if (lane_ok && j >= 0 && j < nvy) k_b = fma(wyd[k], eqB[j], k_b);
                }
                dBe[e] = k_b - Be[e];
                Bc[e] = C(Be[e]);
                dBc[e] = C(dBe[e]);
            }
        };
        auto dA_row = [&](int row) -> double {
            double k_a = 0.0;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                const int j = row - sx + 2 - k;
                if (j >= 0 && j < nvx) k_a = fma(wxd[k], eqA[j], k_a);
            }
            return k_a - eqA[row];
        };
        // the split's factors: before the first loads when the moments need
        // them there, else after the first loads are in flight
        auto eq_setup = [&]() {
            eq_factors();
            // the previous plane's readers of the table are past the
            // warp barrier that ends its last chunk
            for (int row = li; row < nvx; row += team) {
                dAt[row] = pv ? C(dA_row(row)) : C(0);
                At[row] = C(eqA[row]);
            }
            __syncwarp();
        };
        if constexpr (EQ && DIAG) eq_setup();
        // vy window of the lane's first element starts gshift elements away:
        // group offset gd (floor division) and element remainder r in [0, 4)
        const int gshift = -sy - 3;
        const int gd = gshift >= 0 ? gshift / 4 : -((-gshift + 3) / 4);
        const int r = gshift - 4 * gd;
        const TS* src = in + p * (int64_t)nvx * nvy + li * VEC;
        TS* dst = out + p * (int64_t)nvx * nvy + li * VEC;
        double m_pre = 0.0, m_post = 0.0, m_l2 = 0.0, m_sum = 0.0;

        using R = typename Raw<TS, VEC>::type;  // a held row (packed for 4 x bf16)
        auto load_row = [&](int rr) -> R {
            R v = (active && rr >= 0 && rr < nvx) ? ldraw<TS, VEC>(src + (int64_t)rr * nvy) : raw_zero<TS, VEC>();
            if constexpr (DIAG) {
                if (active && rr >= 0 && rr < nvx) {
                    const double vx2 = a.vx[rr] * a.vx[rr];
#pragma unroll
                    for (int e = 0; e < VEC; ++e) {
                        double fv = (double)raw_get<TS, VEC>(v, e);
                        if constexpr (EQ) fv += eqA[rr] * Be[e];
                        m_pre += fv * (vx2 + vy2[e]);
                    }
                }
            }
            return v;
        };

        V win[5];
        const int r0 = -sx - 3;
#pragma unroll
        for (int j = 0; j < 5; ++j) win[j] = raw_vec<TS, VEC>(load_row(r0 + j));
        int rnext = r0 + 5;
        // 4-byte and 2-byte storage load each chunk's rows one chunk ahead
        // (under the previous chunk's vy kick); 8-byte storage and the
        // moment variant would spill and load them in place
        constexpr bool AHEAD = sizeof(TS) <= 4 && !DIAG;
        R nx[KK];
        if constexpr (AHEAD) {
#pragma unroll
            for (int u = 0; u < KK; ++u) nx[u] = load_row(rnext + u);
            rnext += KK;
        }
        if constexpr (EQ && !DIAG) eq_setup();

        for (int l = 0; l < nvx; l += KK) {
            if constexpr (!AHEAD) {
#pragma unroll
                for (int u = 0; u < KK; ++u) nx[u] = load_row(rnext + u);
                rnext += KK;
            }
            // vx kick of rows l..l+KK-1 into the team's row buffer (rounded to
            // the storage type, as the reference stores f between the kicks)
#pragma unroll
            for (int u = 0; u < KK; ++u) {
                C rv[VEC];
                C dA = C(0);
                if constexpr (EQ) dA = dAt[min(l + u, nvx - 1)];
                if constexpr (std::is_same<C, float>::value && VEC % 2 == 0 && !DIAG) {
                    // pairs of elements through the paired FMA (same IEEE
                    // operations per lane)
#pragma unroll
                    for (int h = 0; h < VEC / 2; ++h) {
                        auto g2 = [&](int j) -> float2 {
                            return j < 5 ? make_float2(win[j].v[2 * h], win[j].v[2 * h + 1])
                                         : make_float2(raw_get<TS, VEC>(nx[j - 5], 2 * h),
                                                       raw_get<TS, VEC>(nx[j - 5], 2 * h + 1));
                        };
                        float2 acc = __fmul2_rn(wx2[0], g2(u + 5));
                        acc = __ffma2_rn(wx2[1], g2(u + 4), acc);
                        acc = __ffma2_rn(wx2[2], g2(u + 3), acc);
                        acc = __ffma2_rn(wx2[3], g2(u + 2), acc);
                        acc = __ffma2_rn(wx2[4], g2(u + 1), acc);
                        acc = __ffma2_rn(wx2[5], g2(u + 0), acc);
                        if constexpr (EQ) acc = __ffma2_rn(make_float2(dA, dA), make_float2(Bc[2 * h], Bc[2 * h + 1]), acc);
                        rv[2 * h] = as_stored<TS>(acc.x);
                        rv[2 * h + 1] = as_stored<TS>(acc.y);
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < VEC; ++e) {
                        auto g = [&](int j) -> C { return j < 5 ? win[j].v[e] : raw_get<TS, VEC>(nx[j - 5], e); };
                        C acc = wx[0] * g(u + 5);
                        acc = fma(wx[1], g(u + 4), acc);
                        acc = fma(wx[2], g(u + 3), acc);
                        acc = fma(wx[3], g(u + 2), acc);
                        acc = fma(wx[4], g(u + 1), acc);
                        acc = fma(wx[5], g(u + 0), acc);
                        if constexpr (EQ) acc = fma(dA, Bc[e], acc);
                        rv[e] = as_stored<TS>(acc);
                    }
                }
                if (lane_ok) {
                    if constexpr (VEC == 4) {
                        sts4<C>(rowbuf + u * nvy + li * 4, rv);
                    } else {
#pragma unroll
                        for (int e = 0; e < VEC; ++e) rowbuf[u * nvy + li * VEC + e] = rv[e];
                    }
                }
            }
            // the window moves on (the last 5 rows of [win; nx], KK may be
            // < 5) and the next chunk's loads go out before the vy kick,
            // which then hides their latency
#pragma unroll
            for (int j = 0; j < 5; ++j) {
                const int idx = j + KK;
                if (idx < 5) win[j] = win[idx];
                else win[j] = raw_vec<TS, VEC>(nx[idx - 5]);
            }
            if constexpr (AHEAD) {
                if (l + KK < nvx) {
#pragma unroll
                    for (int u = 0; u < KK; ++u) nx[u] = load_row(rnext + u);
                    rnext += KK;
                }
            }
            __syncwarp();
            // vy kick of the buffered rows
#pragma unroll
            for (int u = 0; u < KK; ++u) {
                V rres;
                if constexpr (VEC == 4) {
                    C t[12];
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        const int gi = li + gd + j;
                        C q[4] = {C(0), C(0), C(0), C(0)};
                        if (gi >= 0 && gi < groups) lds4<C>(rowbuf + u * nvy + gi * 4, q);
#pragma unroll
                        for (int e = 0; e < 4; ++e) t[4 * j + e] = q[e];
                    }
                    C o4[4];
                    switch (r) {
                        case 0: vy_taps<0, C>(t, wy, o4); break;
                        case 1: vy_taps<1, C>(t, wy, o4); break;
                        case 2: vy_taps<2, C>(t, wy, o4); break;
                        default: vy_taps<3, C>(t, wy, o4); break;
                    }
#pragma unroll
                    for (int e = 0; e < 4; ++e) rres.v[e] = o4[e];
                } else {
#pragma unroll
                    for (int e = 0; e < VEC; ++e) {
                        const int iv = li * VEC + e;
                        auto g = [&](int k) -> C {
                            const int j = iv - sy + 2 - k;
                            return (j >= 0 && j < nvy) ? rowbuf[u * nvy + j] : C(0);
                        };
                        C acc = wy[0] * g(0);
                        acc = fma(wy[1], g(1), acc);
                        acc = fma(wy[2], g(2), acc);
                        acc = fma(wy[3], g(3), acc);
                        acc = fma(wy[4], g(4), acc);
                        acc = fma(wy[5], g(5), acc);
                        rres.v[e] = acc;
                    }
                }
                if constexpr (EQ) {
                    const C A = At[min(l + u, nvx - 1)];
#pragma unroll
                    for (int e = 0; e < VEC; ++e) rres.v[e] = fma(A, dBc[e], rres.v[e]);
                }
                if (active && l + u < nvx) {
                    stv<TS, VEC>(dst + (int64_t)(l + u) * nvy, rres);
                    if constexpr (DIAG) {
                        const double vx2 = a.vx[l + u] * a.vx[l + u];
#pragma unroll
                        for (int e = 0; e < VEC; ++e) {
                            double fv = (double)as_stored<TS>(rres.v[e]);
                            if constexpr (EQ) fv += eqA[l + u] * Be[e];
                            m_post += fv * (vx2 + vy2[e]);
                            m_l2 += fv * fv;
                            m_sum += fv;
                        }
                    }
                }
            }
            __syncwarp();
        }
        if constexpr (DIAG) {
            for (int off = team >> 1; off > 0; off >>= 1) {
                m_pre += __shfl_xor_sync(0xffffffffu, m_pre, off, team);
                m_post += __shfl_xor_sync(0xffffffffu, m_post, off, team);
                m_l2 += __shfl_xor_sync(0xffffffffu, m_l2, off, team);
                m_sum += __shfl_xor_sync(0xffffffffu, m_sum, off, team);
            }
            if (pv && li == 0) {
                a.moments[p * 4 + 0] = m_pre;
                a.moments[p * 4 + 1] = m_post;
                a.moments[p * 4 + 2] = m_l2;
                a.moments[p * 4 + 3] = m_sum;
            }
        }
    }
}

template <typename TS, int VEC, bool DIAG, bool EQ>
__global__ void __launch_bounds__(kBlock, 2) k_kick2d(const __grid_constant__ Kick2dArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int teams_per_block = blockDim.x / a.team;
    if constexpr (EQ) {
        // the equilibrium factors, read by every plane, once per block
        double* eq = reinterpret_cast<double*>(reinterpret_cast<compute_t<TS>*>(smem_raw) +
                                               (size_t)teams_per_block * (kick2d_rows<TS, VEC>() * a.nvy + 2 * a.nvx));
        for (int i = threadIdx.x; i < a.nvx + a.nvy; i += blockDim.x)
            eq[i] = i < a.nvx ? a.eqA[i] : a.eqB[i - a.nvx];
        __syncthreads();
    }
    const int64_t stride = (int64_t)gridDim.x * teams_per_block;
    for (int64_t base = (int64_t)blockIdx.x * teams_per_block; base < a.n_planes; base += stride)
        kick2d_item<TS, VEC, DIAG, EQ>(a, base, smem_raw);
}

// The fused kick over the planes of many runs: item g of run r (start[r] <=
// g < start[r+1]) covers planes [(g - start[r]) * teams, ...) of that run,
// teams = blockDim.x / team of the run.
template <typename TS, int VEC>
__global__ void __launch_bounds__(kBlock, 2)
    k_kick2d_batch(const Kick2dArgs* __restrict__ runs, const int64_t* __restrict__ start, int n_runs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int64_t total = start[n_runs];
    int r = 0;
    for (int64_t g = blockIdx.x; g < total; g += gridDim.x) {
        while (r + 1 < n_runs && start[r + 1] <= g) ++r;
        const Kick2dArgs a = runs[r];
        // runs differ in team width, so a warp's row buffers move between
        // items: every warp must be done with the previous item's buffers
        __syncthreads();
        const int64_t teams = blockDim.x / a.team;
        kick2d_item<TS, VEC, false, false>(a, (g - start[r]) * teams, smem_raw);
    }
}

template <typename TS, int VEC, bool DIAG, bool EQ>
static int launch_kick2d_t(Kick2dArgs a, cudaStream_t st) {
    const int teams = kBlock / a.team;
    const size_t smem =
        (size_t)teams * (kick2d_rows<TS, VEC>() * a.nvy + (EQ ? 2 * a.nvx : 0)) * sizeof(compute_t<TS>) +
        (EQ ? (size_t)(a.nvx + a.nvy) * sizeof(double) : 0);
    auto kern = k_kick2d<TS, VEC, DIAG, EQ>;
    if (smem > 48 * 1024) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return set_cuda_error("cudaFuncSetAttribute(k_kick2d)");
    }
    const int occ = occupancy(kern, kBlock, smem);
    const int64_t blocks_needed = (a.n_planes + teams - 1) / teams;
    const int64_t grid = std::min<int64_t>(blocks_needed, (int64_t)sm_count() * occ);
    kern<<<(unsigned)std::max<int64_t>(grid, 1), kBlock, smem, st>>>(a);
    return check_launch("k_kick2d");
}

template <typename TS, bool DIAG>
static int launch_kick2d_vec(Kick2dArgs a, int vec, cudaStream_t st) {
    const bool eq = a.eqB != nullptr;
    if (vec == 4) return eq ? launch_kick2d_t<TS, 4, DIAG, true>(a, st) : launch_kick2d_t<TS, 4, DIAG, false>(a, st);
    if constexpr (sizeof(TS) == 8) {
        if (vec == 2)
            return eq ? launch_kick2d_t<TS, 2, DIAG, true>(a, st) : launch_kick2d_t<TS, 2, DIAG, false>(a, st);
    }
    return eq ? launch_kick2d_t<TS, 1, DIAG, true>(a, st) : launch_kick2d_t<TS, 1, DIAG, false>(a, st);
}

// Elements per lane of the fused kick: 4 when rows and buffers allow it (one
// 128-element row per warp), else 2 (FP64), else 1.
static int kick2d_vec(int dtype, int64_t nvy, uintptr_t addr_or) {
    const int64_t esz = dtype == VP_F64 ? 8 : (dtype == VP_F32 ? 4 : 2);
    // FP64 prefers 2 per lane (4 doubles per lane spill registers) while a
    // plane row still fits one warp
    const bool f64_narrow = dtype == VP_F64 && nvy <= 64;
    for (int vec : {4, 2}) {
        if (vec == 2 && dtype != VP_F64) continue;
        if (vec == 4 && f64_narrow) continue;
        if (nvy % vec == 0 && addr_or % (vec * esz) == 0) return vec;
    }
    return 1;
}

bool kick2d_fits(int dtype, int64_t nvy, const void* a, const void* b, const void* c) {
    const uintptr_t o = reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) | reinterpret_cast<uintptr_t>(c);
    return nvy / kick2d_vec(dtype, nvy, o) <= 32;
}

int run_kick2d(int dtype, const void* in, void* out, int64_t n_planes, int64_t nvx, int64_t nvy,
               const double* Ex, const double* Ey, double dt, double dvx, double dvy, int window,
               const double* vx, const double* vy, double* moments, const EqSplit* eq, cudaStream_t st) {
    const int vec = kick2d_vec(dtype, nvy, reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out));
    const int groups = (int)(nvy / vec);
    if (groups > 32) {
        // wider rows: more groups per lane would be needed; run the two kicks apart
        return VP_ERR_UNSUPPORTED;
    }
    int team = 1;
    while (team < groups) team <<= 1;
    Kick2dArgs a{};
    a.in = in;
    a.out = out;
    a.n_planes = n_planes;
    a.nvx = (int)nvx;
    a.nvy = (int)nvy;
    a.team = team;
    a.groups = groups;
    a.Ex = Ex;
    a.Ey = Ey;
    a.dt = dt;
    a.dvx = dvx;
    a.dvy = dvy;
    a.window = window;
    a.vx = vx;
    a.vy = vy;
    a.moments = moments;
    if (eq && eq->B) {
        a.eqA = eq->A;
        a.eqB = eq->B;
    }
    const bool diag = moments != nullptr;
    switch (dtype) {
        case VP_F32: return diag ? launch_kick2d_vec<float, true>(a, vec, st) : launch_kick2d_vec<float, false>(a, vec, st);
        case VP_F64: return diag ? launch_kick2d_vec<double, true>(a, vec, st) : launch_kick2d_vec<double, false>(a, vec, st);
        case VP_BF16:
            return diag ? launch_kick2d_vec<__nv_bfloat16, true>(a, vec, st)
                        : launch_kick2d_vec<__nv_bfloat16, false>(a, vec, st);
    }
    return set_error(VP_ERR_DTYPE, "unknown dtype");
}

// ---------------------------------------------------------------------------
// many runs per launch (the batched step): argument blocks of every run live
// in a device table; one launch per sweep covers the items of all runs
// ---------------------------------------------------------------------------
// The density of every run of a batch: block (line chunk, outer row o, run);
// each run's partials are summed in the order the single-run step uses for
// its tile count (k_rho_finalize_wide above 32 tiles, k_rho_finalize else),
// so a run of a batch has the density of the same run stepped alone.
__global__ void __launch_bounds__(32 * kFinSlices) k_rho_finalize_batch(const RhoFinRun* __restrict__ runs) {
    __shared__ double sl[kFinSlices][33];
    const RhoFinRun a = runs[blockIdx.z];
    const int64_t o = blockIdx.y;
    const int l = blockIdx.x * 32 + threadIdx.x;
    if (o >= a.n_outer || blockIdx.x * 32 >= a.n_line) return;  // uniform over the block
    const int sidx = threadIdx.y;
    const bool ok = l < a.n_line;
    const double* p = a.part + (o * a.tiles) * (int64_t)a.n_line + l;
    if (a.tiles <= 32) {
        if (sidx == 0 && ok) {
            double acc = 0.0;
            for (int t = 0; t < a.tiles; ++t) acc += p[(int64_t)t * a.n_line];
            a.rho[o * a.n_line + l] = acc * a.scale + a.offset;
        }
        return;
    }
    double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (ok) {
        int t = sidx;
        for (; t + 7 * kFinSlices < a.tiles; t += 8 * kFinSlices) {
            double v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = __ldcs(p + (int64_t)(t + k * kFinSlices) * a.n_line);
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[k] += v[k];
        }
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (t + k * kFinSlices < a.tiles) acc[k] += __ldcs(p + (int64_t)(t + k * kFinSlices) * a.n_line);
    }
    sl[sidx][threadIdx.x] = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
    __syncthreads();
    if (sidx == 0 && ok) {
        double s = sl[0][threadIdx.x];
#pragma unroll
        for (int k = 1; k < kFinSlices; ++k) s += sl[k][threadIdx.x];
        a.rho[o * a.n_line + l] = s * a.scale + a.offset;
    }
}

int strided_batch_args(int dtype, const void* in, void* out, int64_t n_outer, int64_t n_line, int64_t n_inner,
                       int64_t sel_div, int64_t sel_mod, int spread, const int32_t* shift, const void* W,
                       double* part, int block, StridedArgs* a, int* vec, int* nt) {
    pick_vec(dtype, n_inner, sel_div, sel_mod, false, spread, in, out, vec, nt);
    *a = StridedArgs{};
    a->in = in;
    a->out = out;
    a->n_outer = n_outer;
    a->n_line = (int)n_line;
    a->n_inner = n_inner;
    a->sel_div = sel_div;
    a->sel_mod = (int)sel_mod;
    a->shift = shift;
    a->W = W;
    a->part = part;
    a->e_div = 1;
    a->dv = 1.0;
    a->window = -1;
    a->seg = (int)n_line;  // whole lines
    a->nseg = 1;
    (void)block;
    return VP_OK;
}

void strided_batch_finish(StridedArgs* a, int vec, int block) {
    a->ncg = a->n_inner / vec;
    a->tiles = (int)((a->ncg + block - 1) / block);
    a->items = a->n_outer * a->tiles;
}

int strided_batch_pref_vec(int dtype) { return dtype == VP_F64 ? 2 : 4; }

template <typename TS, int VEC, int NT, bool RHO, bool WRAP>
static int launch_sb_t(const StridedArgs* runs, const int64_t* start, int n_runs, int block, int grid_cap,
                       size_t smem, bool pdl, cudaStream_t st) {
    auto kern = k_strided_batch<TS, VEC, NT, RHO, WRAP>;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return set_cuda_error("cudaFuncSetAttribute(k_strided_batch)");
    const int occ = occupancy(kern, block, smem);
    const int grid = std::max(1, std::min(grid_cap, sm_count() * occ));
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    const cudaError_t le = cudaLaunchKernelEx(&cfg, kern, runs, start, n_runs);
    int rc = check_launch("k_strided_batch");
    if (!rc && le != cudaSuccess) rc = set_error(VP_ERR_CUDA, "k_strided_batch: cudaLaunchKernelEx failed");
    return rc;
}

template <typename TS, bool RHO, bool WRAP>
static int launch_sb_v(int vec, int nt, const StridedArgs* runs, const int64_t* start, int n_runs, int block,
                       int grid_cap, size_t smem, bool pdl, cudaStream_t st) {
    constexpr int V = sizeof(TS) == 8 ? 2 : 4;
    if (vec == V && nt == 7)
        return launch_sb_t<TS, V, 7, RHO, WRAP>(runs, start, n_runs, block, grid_cap, smem, pdl, st);
    if (vec == V) return launch_sb_t<TS, V, 6, RHO, WRAP>(runs, start, n_runs, block, grid_cap, smem, pdl, st);
    return launch_sb_t<TS, 1, 6, RHO, WRAP>(runs, start, n_runs, block, grid_cap, smem, pdl, st);
}

template <bool RHO, bool WRAP>
static int launch_sb_d(int dtype, int vec, int nt, const StridedArgs* runs, const int64_t* start, int n_runs,
                       int block, int grid_cap, size_t smem, bool pdl, cudaStream_t st) {
    switch (dtype) {
        case VP_F32:
            return launch_sb_v<float, RHO, WRAP>(vec, nt, runs, start, n_runs, block, grid_cap, smem, pdl, st);
        case VP_F64:
            return launch_sb_v<double, RHO, WRAP>(vec, nt, runs, start, n_runs, block, grid_cap, smem, pdl, st);
        case VP_BF16:
            return launch_sb_v<__nv_bfloat16, RHO, WRAP>(vec, nt, runs, start, n_runs, block, grid_cap, smem, pdl,
                                                          st);
    }
    return set_error(VP_ERR_DTYPE, "unknown dtype");
}

int launch_strided_batch(int dtype, int vec, int nt, bool rho, bool wrap, const StridedArgs* runs,
                         const int64_t* start, int n_runs, int block, int grid_cap, int max_line, bool pdl,
                         cudaStream_t st) {
    if (block != 128 && block != 256) return set_error(VP_ERR_ARG, "batched sweep: block must be 128 or 256");
    if (rho) {
        const size_t smem = (size_t)(block / 32) * max_line * sizeof(double);
        return launch_sb_d<true, false>(dtype, vec, nt, runs, start, n_runs, block, grid_cap, smem, pdl, st);
    }
    if (wrap) return launch_sb_d<false, true>(dtype, vec, nt, runs, start, n_runs, block, grid_cap, 0, pdl, st);
    return launch_sb_d<false, false>(dtype, vec, nt, runs, start, n_runs, block, grid_cap, 0, pdl, st);
}

int launch_rho_finalize_batch(const RhoFinRun* runs, int n_runs, int max_outer, int max_line, cudaStream_t st) {
    const dim3 grid((unsigned)((max_line + 31) / 32), (unsigned)max_outer, (unsigned)n_runs);
    k_rho_finalize_batch<<<grid, dim3(32, kFinSlices), 0, st>>>(runs);
    return check_launch("k_rho_finalize_batch");
}

int kick2d_batch_args(int dtype, const void* in, void* out, int64_t n_planes, int64_t nvx, int64_t nvy,
                      const double* Ex, const double* Ey, double dt, double dvx, double dvy, int window,
                      Kick2dArgs* a, int* vec) {
    *vec = kick2d_vec(dtype, nvy, reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out));
    *a = Kick2dArgs{};
    a->in = in;
    a->out = out;
    a->n_planes = n_planes;
    a->nvx = (int)nvx;
    a->nvy = (int)nvy;
    a->Ex = Ex;
    a->Ey = Ey;
    a->dt = dt;
    a->dvx = dvx;
    a->dvy = dvy;
    a->window = window;
    return VP_OK;
}

// team and item count of a run once the batch's common VEC is known;
// returns the run's shared-memory need per block
int64_t kick2d_batch_finish(Kick2dArgs* a, int dtype, int vec, int block, int64_t* items) {
    a->groups = a->nvy / vec;
    int team = 1;
    while (team < a->groups) team <<= 1;
    a->team = team;
    const int teams = block / team;
    *items = (a->n_planes + teams - 1) / teams;
    const int64_t csz = dtype == VP_F64 ? 8 : 4;
    const int rows = (dtype == VP_F64 && vec == 4) ? kick2d_rows<double, 4>() : kU;
    return (int64_t)teams * rows * a->nvy * csz;
}

template <typename TS, int VEC>
static int launch_kb_t(const Kick2dArgs* runs, const int64_t* start, int n_runs, int block, int grid_cap,
                       size_t smem, cudaStream_t st) {
    auto kern = k_kick2d_batch<TS, VEC>;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return set_cuda_error("cudaFuncSetAttribute(k_kick2d_batch)");
    const int occ = occupancy(kern, block, smem);
    const int grid = std::max(1, std::min(grid_cap, sm_count() * occ));
    kern<<<grid, block, smem, st>>>(runs, start, n_runs);
    return check_launch("k_kick2d_batch");
}

template <typename TS>
static int launch_kb_v(int vec, const Kick2dArgs* runs, const int64_t* start, int n_runs, int block, int grid_cap,
                       size_t smem, cudaStream_t st) {
    if (vec == 4) return launch_kb_t<TS, 4>(runs, start, n_runs, block, grid_cap, smem, st);
    if constexpr (sizeof(TS) == 8) {
        if (vec == 2) return launch_kb_t<TS, 2>(runs, start, n_runs, block, grid_cap, smem, st);
    }
    return launch_kb_t<TS, 1>(runs, start, n_runs, block, grid_cap, smem, st);
}

int launch_kick2d_batch(int dtype, int vec, const Kick2dArgs* runs, const int64_t* start, int n_runs, int block,
                        int grid_cap, size_t smem, cudaStream_t st) {
    if (block != 128 && block != 256) return set_error(VP_ERR_ARG, "batched kick: block must be 128 or 256");
    switch (dtype) {
        case VP_F32: return launch_kb_v<float>(vec, runs, start, n_runs, block, grid_cap, smem, st);
        case VP_F64: return launch_kb_v<double>(vec, runs, start, n_runs, block, grid_cap, smem, st);
        case VP_BF16: return launch_kb_v<__nv_bfloat16>(vec, runs, start, n_runs, block, grid_cap, smem, st);
    }
    return set_error(VP_ERR_DTYPE, "unknown dtype");
}

// ---------------------------------------------------------------------------
// kick along the contiguous axis: rows of n_line elements, one field value
// per row. Each group of tpr threads owns one row, staged in shared memory.
// ---------------------------------------------------------------------------
template <typename TS>
__global__ void __launch_bounds__(kBlock) k_kick_contig(const TS* __restrict__ in, TS* __restrict__ out,
                                                      int64_t n_rows, int n, const void* E, int e_f64,
                                                      int64_t e_div, double dt, double dv, int window, int tpr,
                                                      const double* __restrict__ eqA,
                                                      const double* __restrict__ eqB, int64_t eq_arows) {
    using C = compute_t<TS>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int rpb = blockDim.x / tpr;
    const int g = threadIdx.x / tpr, li = threadIdx.x % tpr;
    C* row = reinterpret_cast<C*>(smem_raw) + (size_t)g * n;
    for (int64_t base = (int64_t)blockIdx.x * rpb; base < n_rows; base += (int64_t)gridDim.x * rpb) {
        const int64_t o = base + g;
        const bool ok = o < n_rows;
        C w[6];
        double wd[6];
        int s = 0;
        if (ok) {
            const int64_t ei = o / e_div;
            s = e_f64 ? kick_weights<double, double>(static_cast<const double*>(E)[ei], dt, dv, window, wd)
                      : kick_weights<float, double>(static_cast<const float*>(E)[ei], dt, dv, window, wd);
#pragma unroll
            for (int k = 0; k < 6; ++k) w[k] = C(wd[k]);
            s = max(-(1 << 28), min(1 << 28, s));
            for (int i = li; i < n; i += tpr) row[i] = to_c(in[o * n + i]);
        }
        __syncthreads();
        if (ok) {
            for (int i = li; i < n; i += tpr) {
                auto gv = [&](int k) -> C {
                    const int j = i - s + 2 - k;
                    return (j >= 0 && j < n) ? row[j] : C(0);
                };
                C acc = w[0] * gv(0);
                acc = fma(w[1], gv(1), acc);
                acc = fma(w[2], gv(2), acc);
                acc = fma(w[3], gv(3), acc);
                acc = fma(w[4], gv(4), acc);
                acc = fma(w[5], gv(5), acc);
                if (eqB) {
                    // equilibrium split: add the kicked equilibrium minus itself
                    double kb = 0.0;
#pragma unroll
                    for (int k = 0; k < 6; ++k) {
                        const int j = i - s + 2 - k;
                        if (j >= 0 && j < n) kb = fma(wd[k], eqB[j], kb);
                    }
                    const double Ao = eqA ? eqA[o % eq_arows] : 1.0;
                    acc += C(Ao * (kb - eqB[i]));
                }
                out[o * n + i] = from_c<TS>(acc);
            }
        }
        __syncthreads();
    }
}

// The same kick for rows whose length is a multiple of 4 (4- and 2-byte
// storage, no equilibrium split): a thread owns groups of 4 elements (16- or
// 8-byte accesses), the block walks rows through a double-buffered
// shared-memory row while the next row's loads are in flight, one thread per
// row evaluates the weights, and the 6 taps of a group come from 3 aligned
// 4-element reads (vy_taps: the same operations, in the same order, as the
// scalar kernel's, zero outside the row).
constexpr int kContigGroups = 8;  // groups of 4 per thread: rows up to 8192

template <typename TS>
__global__ void __launch_bounds__(kBlock) k_kick_contig4(const TS* __restrict__ in, TS* __restrict__ out,
                                                         int64_t n_rows, int n, const void* E, int e_f64,
                                                         int64_t e_div, double dt, double dv, int window) {
    using C = compute_t<TS>;
    static_assert(sizeof(C) == 4, "4- and 2-byte storage");
    using R = typename Raw<TS, 4>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* rows = reinterpret_cast<C*>(smem_raw);          // [2][n]
    float* wts = reinterpret_cast<float*>(rows + 2 * n);  // [2][8]: 6 weights, the shift's bits
    const int groups = n / 4, tid = threadIdx.x;
    R cur[kContigGroups];
    auto load = [&](int64_t o) {
#pragma unroll
        for (int k = 0; k < kContigGroups; ++k) {
            const int g = tid + k * kBlock;
            cur[k] = (o < n_rows && g < groups) ? ldraw<TS, 4>(in + o * n + g * 4) : raw_zero<TS, 4>();
        }
    };
    int b = 0;
    load(blockIdx.x);
    for (int64_t o = blockIdx.x; o < n_rows; o += gridDim.x, b ^= 1) {
        C* row = rows + b * n;
#pragma unroll
        for (int k = 0; k < kContigGroups; ++k) {
            const int g = tid + k * kBlock;
            if (g < groups) {
                C v[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) v[e] = raw_get<TS, 4>(cur[k], e);
                sts4<C>(row + g * 4, v);
            }
        }
        if (tid == 0) {
            double wd[6];
            const int64_t ei = o / e_div;
            int sh = e_f64 ? kick_weights<double, double>(static_cast<const double*>(E)[ei], dt, dv, window, wd)
                           : kick_weights<float, double>(static_cast<const float*>(E)[ei], dt, dv, window, wd);
            sh = max(-(1 << 28), min(1 << 28, sh));
#pragma unroll
            for (int k = 0; k < 6; ++k) wts[b * 8 + k] = (float)C(wd[k]);
            wts[b * 8 + 6] = __int_as_float(sh);
        }
        load(o + gridDim.x);  // the next row's loads go out before the kick
        __syncthreads();
        C w[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) w[k] = wts[b * 8 + k];
        const int sh = __float_as_int(wts[b * 8 + 6]);
        // the window of a group's first element starts gshift elements away:
        // group offset gd (floor division) and remainder r in [0, 4)
        const int gshift = -sh - 3;
        const int gd = gshift >= 0 ? gshift / 4 : -((-gshift + 3) / 4);
        const int r = gshift - 4 * gd;
#pragma unroll
        for (int k = 0; k < kContigGroups; ++k) {
            const int g = tid + k * kBlock;
            if (g >= groups) continue;
            C t[12];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const int gi = g + gd + j;
                C q[4] = {C(0), C(0), C(0), C(0)};
                if (gi >= 0 && gi < groups) lds4<C>(row + gi * 4, q);
#pragma unroll
                for (int e = 0; e < 4; ++e) t[4 * j + e] = q[e];
            }
            Vec<TS, 4> res;
            switch (r) {
                case 0: vy_taps<0, C>(t, w, res.v); break;
                case 1: vy_taps<1, C>(t, w, res.v); break;
                case 2: vy_taps<2, C>(t, w, res.v); break;
                default: vy_taps<3, C>(t, w, res.v); break;
            }
            stv<TS, 4>(out + o * n + g * 4, res);
        }
        // one barrier per row: buffer b is written again two rows on, after
        // the next row's barrier, when every thread is done reading it
    }
}

template <typename TS>
static int launch_kick_contig_t(const void* in, void* out, int64_t n_rows, int64_t n, const void* E, int e_f64,
                                int64_t e_div, double dt, double dv, int window, const EqSplit* eq,
                                cudaStream_t st) {
    if constexpr (sizeof(TS) <= 4) {
        const size_t align = sizeof(TS) * 4;
        if (n % 4 == 0 && n / 4 <= kBlock * kContigGroups && !(eq && eq->B) &&
            reinterpret_cast<uintptr_t>(in) % align == 0 && reinterpret_cast<uintptr_t>(out) % align == 0) {
            const size_t smem = 2 * (size_t)n * sizeof(compute_t<TS>) + 16 * sizeof(float);
            auto kern = k_kick_contig4<TS>;
            if (smem > 48 * 1024 &&
                cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
                return set_cuda_error("cudaFuncSetAttribute(k_kick_contig4)");
            const int occ = occupancy(kern, kBlock, smem);
            const int64_t grid = std::min<int64_t>(n_rows, (int64_t)sm_count() * occ);
            kern<<<(unsigned)std::max<int64_t>(grid, 1), kBlock, smem, st>>>(
                static_cast<const TS*>(in), static_cast<TS*>(out), n_rows, (int)n, E, e_f64, e_div, dt, dv, window);
            return check_launch("k_kick_contig4");
        }
    }
    int tpr = 32;
    while (tpr < n && tpr < kBlock) tpr <<= 1;
    const int rpb = kBlock / tpr;
    const size_t smem = (size_t)rpb * n * sizeof(compute_t<TS>);
    if (smem > 200 * 1024) return set_error(VP_ERR_UNSUPPORTED, "kick row too long for shared memory");
    auto kern = k_kick_contig<TS>;
    if (smem > 48 * 1024) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return set_cuda_error("cudaFuncSetAttribute(k_kick_contig)");
    }
    const int occ = occupancy(kern, kBlock, smem);
    const int64_t grid = std::min<int64_t>((n_rows + rpb - 1) / rpb, (int64_t)sm_count() * occ);
    const bool eqon = eq && eq->B;
    kern<<<(unsigned)std::max<int64_t>(grid, 1), kBlock, smem, st>>>(
        static_cast<const TS*>(in), static_cast<TS*>(out), n_rows, (int)n, E, e_f64, e_div, dt, dv, window, tpr,
        eqon ? eq->A : nullptr, eqon ? eq->B : nullptr, eqon && eq->nvx > 0 ? eq->nvx : 1);
    return check_launch("k_kick_contig");
}

int run_kick_contig(int dtype, const void* in, void* out, int64_t n_rows, int64_t n, const void* E, int e_f64,
                    int64_t e_div, double dt, double dv, int window, const EqSplit* eq, cudaStream_t st) {
    switch (dtype) {
        case VP_F32:
            return launch_kick_contig_t<float>(in, out, n_rows, n, E, e_f64, e_div, dt, dv, window, eq, st);
        case VP_F64:
            return launch_kick_contig_t<double>(in, out, n_rows, n, E, e_f64, e_div, dt, dv, window, eq, st);
        case VP_BF16:
            return launch_kick_contig_t<__nv_bfloat16>(in, out, n_rows, n, E, e_f64, e_div, dt, dv, window, eq, st);
    }
    return set_error(VP_ERR_DTYPE, "unknown dtype");
}

// ---------------------------------------------------------------------------
// general sweep with a per-element departure point (advect_1d semantics)
// ---------------------------------------------------------------------------
template <typename TS>
__global__ void k_gather(const TS* __restrict__ in, TS* __restrict__ out, int64_t n_outer, int n,
                         int64_t n_inner, const compute_t<TS>* __restrict__ vel, int64_t vso, int64_t vsl,
                         int64_t vsc, double dt, double dx, int periodic) {
    using C = compute_t<TS>;
    using R = Rn<C>;
    const int64_t total = n_outer * n * n_inner;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = i % n_inner;
        const int64_t ol = i / n_inner;
        const int l = (int)(ol % n);
        const int64_t o = ol / n;
        const C v = vel[o * vso + (int64_t)l * vsl + c * vsc];
        const C disp = R::div(R::mul(v, C(dt)), C(dx));
        const C depart = R::sub(C(l), disp);
        const C fl = floor(depart);
        const C al = R::sub(depart, fl);
        const int64_t il = (int64_t)fl;
        C w[6];
        lagrange6<C>(al, w);
        const TS* src = in + o * n * n_inner + c;
        C acc = C(0);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            int64_t r = il + k - 2;
            C gv;
            if (periodic) {
                r %= n;
                if (r < 0) r += n;
                gv = to_c(src[r * n_inner]);
            } else {
                const bool valid = r >= 0 && r < n;
                const int64_t rc = r < 0 ? 0 : (r > n - 1 ? n - 1 : r);
                gv = R::mul(to_c(src[rc * n_inner]), valid ? C(1) : C(0));
            }
            const C t = R::mul(w[k], gv);
            acc = k == 0 ? t : R::add(acc, t);
        }
        out[i] = from_c<TS>(acc);
    }
}

int run_gather(int dtype, const void* in, void* out, int64_t n_outer, int64_t n, int64_t n_inner, const void* vel,
               int64_t vso, int64_t vsl, int64_t vsc, double dt, double dx, int periodic, cudaStream_t st) {
    const int64_t total = n_outer * n * n_inner;
    const int64_t grid = std::min<int64_t>((total + 255) / 256, (int64_t)sm_count() * 16);
    switch (dtype) {
        case VP_F32:
            k_gather<float><<<(unsigned)grid, 256, 0, st>>>(static_cast<const float*>(in), static_cast<float*>(out),
                                                            n_outer, (int)n, n_inner, static_cast<const float*>(vel),
                                                            vso, vsl, vsc, dt, dx, periodic);
            break;
        case VP_F64:
            k_gather<double><<<(unsigned)grid, 256, 0, st>>>(static_cast<const double*>(in), static_cast<double*>(out),
                                                             n_outer, (int)n, n_inner, static_cast<const double*>(vel),
                                                             vso, vsl, vsc, dt, dx, periodic);
            break;
        case VP_BF16:
            k_gather<__nv_bfloat16><<<(unsigned)grid, 256, 0, st>>>(
                static_cast<const __nv_bfloat16*>(in), static_cast<__nv_bfloat16*>(out), n_outer, (int)n, n_inner,
                static_cast<const float*>(vel), vso, vsl, vsc, dt, dx, periodic);
            break;
        default: return set_error(VP_ERR_DTYPE, "unknown dtype");
    }
    return check_launch("k_gather");
}

// ---------------------------------------------------------------------------
// compute_rho: one warp per point, FP64 accumulation, fixed order
// ---------------------------------------------------------------------------
template <typename TS, typename TO>
__global__ void k_rho(const TS* __restrict__ f, int64_t n_points, int64_t n_v, double dvx, double dvy,
                      TO* __restrict__ rho) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t p = wid; p < n_points; p += nw) {
        double acc = 0.0;
        const TS* src = f + p * n_v;
        for (int64_t c = lane; c < n_v; c += 32) acc += (double)to_c(src[c]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (lane == 0) rho[p] = (TO)((acc * dvx) * dvy);
    }
}

int run_rho(int dtype, const void* f, int64_t n_points, int64_t n_v, double dvx, double dvy, void* rho,
            int out_dtype, cudaStream_t st) {
    const int64_t grid = std::min<int64_t>((n_points * 32 + 255) / 256, (int64_t)sm_count() * 16);
    const unsigned gb = (unsigned)std::max<int64_t>(grid, 1);
#define VP_RHO_CASE(TS_)                                                                                      \
    if (out_dtype == VP_F64)                                                                                  \
        k_rho<TS_, double><<<gb, 256, 0, st>>>(static_cast<const TS_*>(f), n_points, n_v, dvx, dvy,          \
                                                static_cast<double*>(rho));                                   \
    else                                                                                                      \
        k_rho<TS_, float><<<gb, 256, 0, st>>>(static_cast<const TS_*>(f), n_points, n_v, dvx, dvy,           \
                                               static_cast<float*>(rho));
    switch (dtype) {
        case VP_F32: VP_RHO_CASE(float) break;
        case VP_F64: VP_RHO_CASE(double) break;
        case VP_BF16: VP_RHO_CASE(__nv_bfloat16) break;
        default: return set_error(VP_ERR_DTYPE, "unknown dtype");
    }
#undef VP_RHO_CASE
    return check_launch("k_rho");
}

}  // namespace vp

// ---------------------------------------------------------------------------
// Lagrange helpers of the interpolation API: the 6-point sum with the
// closed-form weights (lagrange5_interp_sum, vlasov2D2V.py:238-260: each
// product rounded, summed left to right) and the product-form weights
// (get_lagrange5_weights, :210-235: w_j = prod_{m != j} (a - x_m)/(x_j - x_m)
// over the nodes x = -2..3, in that order), every operation rounded on its
// own so the results equal the reference's eager evaluation bit for bit.
// ---------------------------------------------------------------------------
namespace vp {

template <typename T>
__global__ void k_lagrange(const T* __restrict__ alpha, const T* __restrict__ vals, T* __restrict__ out, int64_t n,
                           int mode) {
    using R = Rn<T>;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const T a = alpha[i];
    if (mode == 0) {
        T w[6];
        lagrange6<T>(a, w);
        T acc = R::mul(w[0], vals[6 * i]);
#pragma unroll
        for (int k = 1; k < 6; ++k) acc = R::add(acc, R::mul(w[k], vals[6 * i + k]));
        out[i] = acc;
    } else {
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            const T xj = T(j - 2);
            T w = T(1);
#pragma unroll
            for (int m = 0; m < 6; ++m) {
                if (m == j) continue;
                const T xm = T(m - 2);
                w = R::div(R::mul(w, R::sub(a, xm)), R::sub(xj, xm));
            }
            out[6 * i + j] = w;
        }
    }
}

int run_lagrange(int dtype, const void* alpha, const void* vals, void* out, int64_t n, int mode, cudaStream_t st) {
    if (n == 0) return VP_OK;
    const unsigned grid = (unsigned)((n + 255) / 256);
    if (dtype == VP_F64)
        k_lagrange<double><<<grid, 256, 0, st>>>(static_cast<const double*>(alpha), static_cast<const double*>(vals),
                                                 static_cast<double*>(out), n, mode);
    else if (dtype == VP_F32)
        k_lagrange<float><<<grid, 256, 0, st>>>(static_cast<const float*>(alpha), static_cast<const float*>(vals),
                                                static_cast<float*>(out), n, mode);
    else
        return set_error(VP_ERR_DTYPE, "vp_lagrange: float32 or float64 only");
    return check_launch("k_lagrange");
}

}  // namespace vp
