// Learned correction of the drift interpolation weights on tensor cores.
//
// A per-cell network proposes a correction dw to the 6 Lagrange weights of
// a sweep: a periodic drift (x / y, shift and weights from the drift table)
// or a Dirichlet kick (vx / vy, shift and weights from the plane's field E,
// the formulas of the plain kick evaluated in FP32):
//   x  = [f_k / s (k < 6), alpha - 1/2, 1, 0 x 8]          s = max_k |f_k|
//   h1 = relu(W1 x)            W1: [64][16]  (column 7 = bias)
//   h2 = relu(W2 [h1, 1, 0])   W2: [64][80]  (column 64 = bias)
//   o  = W3 [h2, 1, 0]         W3: [16][80]  (rows >= 6 zero)
//   dw = o[0:6] - mean(o[0:6])        (the weights keep summing to one)
//   out = sum_k (w_k + dw_k) f_k
// When the line length n and n_inner are powers of two the correction is
// projected, line by line, to zero sum:
//   out_l -= mean_l (out_l - plain_l),  plain_l = sum_k w_k f_k
// so each line's sum changes exactly as in the plain sweep (the periodic
// drift keeps it, the kick loses what leaves the velocity range). The tiles
// of a CTA then run in super-tiles of P tiles that hold whole lines (a lane
// keeps to one line in all P tiles); the line sums are reduced at the end of
// the super-tile and subtracted from the outputs it wrote, which are still
// in L2.
// x, h1, h2 and the weights are BF16 operands of tcgen05.mma (kind::f16,
// FP32 accumulators in tensor memory); dw and the output are FP32.
//
// Each tile is 128 consecutive cells of the flattened
// [n_outer][n_line][n_inner] array (the MMA M), thread <-> cell <->
// accumulator lane, one tile per CTA of 128 threads at a time. Inference
// CTAs hold 128 tensor-memory columns and ~48 KB of shared memory, so four
// share an SM and overlap one another's MMA waits; training CTAs hold all 512
// columns (the weight gradients live there). Every operand lives in shared
// memory in the canonical K-major layout without swizzle (8 x 16-byte core
// matrices, K chunks 128 bytes apart, 8-row groups (K/8)*128 bytes apart).
// A single thread issues the MMAs; completion is signalled through one
// mbarrier (tcgen05.commit) that every thread waits on, with a time limit:
// a wait that runs out sets *status and the kernel leaves after releasing
// its tensor memory.
//
// Training (TRAIN = true) adds, per tile, the residual against a target,
//   r = (out - target) * inv_scale,  loss += sum r^2,
// the backward deltas on tensor cores
//   do  = P (gy f),  gy = 2 r inv_scale (less its line mean when projected)
//                                       (P: the zero-mean projection)
//   dz2 = (do  W3)[0:64] * [z2 > 0]     (MMA with W3 transposed)
//   dz1 = (dz2 W2)[0:64] * [z1 > 0]     (MMA with W2 transposed)
// and the weight gradients accumulated in tensor memory over all tiles of
// the CTA (reduction over cells = the MMA K):
//   [dW2; dW1] = [dz2^T; dz1^T] [h1', x]      (one M=128, N=96 chain)
//   dW3^T      = h2'^T do                     (M=128, N=16)
// added to the global FP32 gradient once per CTA. A projected training
// sweep runs the forward layers twice per super-tile: the first pass sums
// (out - plain) and (plain - target) over each line, the second uses their
// means: out' = out - mean(out - plain) and, since mean(out') = mean(plain),
//   mean_l(gy) = 2 inv_scale^2 (mean(plain) - mean(target)).
#include <stdint.h>

#include <algorithm>

#include "common.cuh"
#include "launch.h"

namespace vp {
namespace mlp {

constexpr int TM = 128;  // cells per tile = MMA M
// tiles per CTA and MMA round trip (one: independent CTAs interleave their
// MMA waits with each other's epilogues)
__host__ __device__ constexpr int subtiles(bool) { return 1; }
constexpr int XS = TM * 16 * 2;  // bytes of one tile's layer-1 input [TM][16]
constexpr int HS = TM * 80 * 2;  // bytes of one tile's hidden layer [TM][80]
constexpr int K1 = 16;   // layer-1 input width
constexpr int HID = 64;  // hidden width
constexpr int K2 = 80;   // hidden + constant + zero pad
constexpr int NO = 16;   // layer-3 outputs (6 used)
constexpr int KW = 128;  // cells per weight-gradient chain (= TM)

// bf16 element offsets of the packed network (see include/vlasov_b200.h)
constexpr int OFF_W1 = 0;
constexpr int OFF_W2 = OFF_W1 + HID * K1;
constexpr int OFF_W3 = OFF_W2 + HID * K2;
constexpr int OFF_W3T = OFF_W3 + NO * K2;
constexpr int OFF_W2T = OFF_W3T + HID * NO;
constexpr int NET_ELEMS = OFF_W2T + HID * HID;
// FP32 gradient offsets
constexpr int G_W1 = 0;
constexpr int G_W2 = G_W1 + HID * K1;
constexpr int G_W3 = G_W2 + HID * K2;
constexpr int GRAD_ELEMS = G_W3 + NO * K2;

// ---------------------------------------------------------------------------
// tcgen05 / mbarrier primitives (inline PTX)
// ---------------------------------------------------------------------------
// byte offset of element (r, k) of a [R][K] K-major bf16 matrix
__device__ __forceinline__ uint32_t kmaj(int r, int k, int K) {
    return (uint32_t)(((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory descriptor of the 16-wide K slice starting at k0
__device__ __forceinline__ uint64_t kdesc(uint32_t base, int k0, int K) {
    const uint32_t start = base + (uint32_t)(k0 >> 3) * 128u;
    const uint64_t lbo = 128u >> 4;                          // next 8-wide K chunk
    const uint64_t sbo = ((uint32_t)(K >> 3) * 128u) >> 4;  // next 8-row group
    return (uint64_t)((start >> 4) & 0x3FFFu) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// instruction descriptor: BF16 x BF16 -> F32, A and B K-major, M x N
__host__ __device__ constexpr uint32_t idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(id), "r"(acc)
        : "memory");
}

// D[TM][N] (+)= A[TM][K] B[N][K]^T, K a multiple of 16
__device__ __forceinline__ void gemm(uint32_t d_tmem, uint32_t a_base, uint32_t b_base, int K, int N,
                                     bool accumulate) {
    const uint32_t id = idesc(TM, N);
    for (int k0 = 0; k0 < K; k0 += 16)
        mma(d_tmem, kdesc(a_base, k0, K), kdesc(b_base, k0, K), id, (accumulate || k0 > 0) ? 1u : 0u);
}

__device__ __forceinline__ void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's accumulator lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void st_bf16(unsigned char* base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // a in the low half
    return *reinterpret_cast<const uint32_t*>(&h);
}

// 8 consecutive K elements of one row (one 16-byte row of a core matrix)
__device__ __forceinline__ void st8_bf16(unsigned char* base, uint32_t off, const float* v) {
    *reinterpret_cast<uint4*>(base + off) =
        make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
}

// the stencil, plain weights and fraction of one cell
struct CellData {
    float f[6], w[6];
    float al;
    int64_t cell;
    bool act;
};

// ---------------------------------------------------------------------------
// shared-memory plan (bytes)
// ---------------------------------------------------------------------------
struct Smem {
    uint32_t x, h1, h2, w1, w2, w3, w3t, w2t;  // both modes
    uint32_t dO, dz2, aw, bw, h2t, doT;        // training only
    uint32_t bar, tslot, loss, line, total;
};

__host__ __device__ constexpr uint32_t al128(uint32_t b) { return (b + 127u) & ~127u; }

__host__ __device__ constexpr Smem plan(bool train) {
    Smem s{};
    uint32_t o = 0;
    auto take = [&](uint32_t b) {
        const uint32_t r = o;
        o += al128(b);
        return r;
    };
    const uint32_t sub = (uint32_t)subtiles(train);
    s.x = take(sub * XS);
    s.h1 = take(sub * HS);
    // inference: layer 2's output overwrites layer 1's (no longer read once
    // the layer-2 MMA has completed); training keeps both for the gradients
    s.h2 = train ? take(sub * HS) : s.h1;
    s.w1 = take(HID * K1 * 2);
    s.w2 = take(HID * K2 * 2);
    s.w3 = take(NO * K2 * 2);
    if (train) {
        s.w3t = take(HID * NO * 2);
        s.w2t = take(HID * HID * 2);
        s.dO = take(TM * NO * 2);    // [cell][16]   A of dh2
        s.dz2 = take(TM * HID * 2);  // [cell][64]   A of dh1
        s.aw = take(128 * KW * 2);   // [dz2^T; dz1^T] [128][cells]
        s.bw = take(96 * KW * 2);    // [h1'^T; x^T]   [96][cells]
        s.h2t = take(128 * KW * 2);  // h2'^T (80 rows, rest zero) [128][cells]
        s.doT = take(NO * KW * 2);   // do^T [16][cells]
    }
    s.bar = take(8);
    s.tslot = take(4);
    s.loss = take(sub * TM * 8);
    s.line = take(2 * TM * 4);  // line sums of the projection
    s.total = o;
    return s;
}

// tensor-memory columns
constexpr uint32_t T_D1 = 0, T_D2 = 64, T_D3 = 128;  // forward (D3: 16 used of 32)
constexpr uint32_t T_G2 = 160, T_G1 = 224;           // backward deltas
constexpr uint32_t T_WA = 288, T_WB = 384;           // [dW2 | dW1] (96), dW3^T (16)
constexpr uint32_t TMEM_TRAIN = 512, TMEM_INFER = 128;

}  // namespace mlp

struct MlpSweepArgs {
    const float* in;
    const float* target;  // training only
    float* out;           // inference only
    int64_t n_outer, n_inner;
    int n_line;
    // drift: table column j = (c / sel_div) % sel_mod
    int64_t sel_div;
    int sel_mod;
    const int32_t* shift;
    const float* W;      // [6][sel_mod] Lagrange weights
    const float* alpha;  // [sel_mod] fractional shifts
    // kick: field E[o / e_div], shift (E dt) / dv
    const double* E;
    int64_t e_div;
    double dt, dv;
    const __nv_bfloat16* net;
    float* grad;      // training: [GRAD_ELEMS]
    double* loss;     // training: sum of r^2
    float inv_scale;  // training: residual scale
    int64_t cells;    // n_outer * n_line * n_inner
    // line projection (set by run_mlp_sweep): with nb = 2^st_lg, super-tile
    // st holds the tiles (st / nb) * per_st * nb + k * nb + st % nb,
    // k < per_st; in each tile q lanes, qstride apart, belong to one line
    // (q, qstride powers of two)
    int proj, per_st, q, qstride, st_lg;
    int* status;
};

namespace mlp {
using SweepArgs = MlpSweepArgs;

// copy a row-major [R][K] bf16 matrix from global into the K-major layout
__device__ void load_matrix(unsigned char* sm, uint32_t dst, const __nv_bfloat16* src, int R, int K) {
    for (int i = threadIdx.x; i < R * K; i += blockDim.x) {
        const int r = i / K, k = i % K;
        *reinterpret_cast<__nv_bfloat16*>(sm + dst + kmaj(r, k, K)) = src[i];
    }
}

template <bool TRAIN, bool KICK>
__global__ void __launch_bounds__(TM * subtiles(TRAIN), TRAIN ? 1 : 4) k_mlp_sweep(const __grid_constant__ SweepArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    constexpr Smem S = plan(TRAIN);
    constexpr int SUB = subtiles(TRAIN);
    constexpr int NT = TM * SUB;
    static_assert(SUB == 1, "the super-tile loop takes one tile per item");
    constexpr uint32_t TD3 = TRAIN ? T_D3 : T_D1;  // inference: layer 3 reuses layer 1's columns
    const int t = threadIdx.x;
    const int u = t / TM;        // this thread's tile of the CTA
    const int tl = t % TM;       // its cell (row) within the tile
    const uint32_t ux = (uint32_t)u * XS, uh = (uint32_t)u * HS;
    const uint32_t base = smem_u32(sm);
    const uint32_t bar = base + S.bar;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + S.tslot);
    const uint32_t ncols = TRAIN ? TMEM_TRAIN : TMEM_INFER;

    // zero every operand buffer once: padding rows / columns stay zero
    for (uint32_t i = t * 16; i < S.bar; i += NT * 16) *reinterpret_cast<uint4*>(sm + i) = make_uint4(0, 0, 0, 0);
    __syncthreads();
    load_matrix(sm, S.w1, a.net + OFF_W1, HID, K1);
    load_matrix(sm, S.w2, a.net + OFF_W2, HID, K2);
    load_matrix(sm, S.w3, a.net + OFF_W3, NO, K2);
    if (TRAIN) {
        load_matrix(sm, S.w3t, a.net + OFF_W3T, HID, NO);
        load_matrix(sm, S.w2t, a.net + OFF_W2T, HID, HID);
    }
    // constant-one columns of the layer inputs (bias columns)
    st_bf16(sm, S.x + ux + kmaj(tl, 7, K1), 1.0f);
    st_bf16(sm, S.h1 + uh + kmaj(tl, HID, K2), 1.0f);
    st_bf16(sm, S.h2 + uh + kmaj(tl, HID, K2), 1.0f);
    if (TRAIN) {
        // the transposed copies hold the constant rows: h1'^T row 64 and h2'^T row 64
        st_bf16(sm, S.bw + kmaj(HID, t, KW), 1.0f);
        st_bf16(sm, S.h2t + kmaj(HID, t, KW), 1.0f);
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (t < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tm = *tslot;
    // this warp's 32 lanes, in this tile's 128 columns
    const uint32_t lane_base = tm + ((uint32_t)(tl & ~31) << 16) + (uint32_t)u * 128u;
    uint32_t phase = 0;
    bool ok = true;
    double loss_acc = 0.0;
    bool wacc = false;  // weight-gradient accumulators hold data

    // one MMA group issued by thread 0, completion awaited by all threads;
    // `work` runs on every thread while the tensor cores compute
    auto run_with = [&](auto&& issue, auto&& work) -> bool {
        fence_async_smem();
        fence_before();
        __syncthreads();
        fence_after();
        if (t == 0) {
            issue();
            commit(bar);
        }
        work();
        const bool done = mbar_wait(bar, phase & 1u);
        phase++;
        const bool all = __syncthreads_and(done) != 0;  // every thread takes the same exit
        fence_after();
        return all;
    };
    auto run = [&](auto&& issue) -> bool { return run_with(issue, [] {}); };

    const int64_t tiles = (a.cells + TM - 1) / TM;
    const int n = a.n_line;
    // stencil of a cell: f_k = in[o, l - s - (k - 2), c], taken mod n (drift)
    // or zero outside [0, n) (kick)
    auto gather = [&](int64_t tile) {
        CellData d;
        d.cell = (tile + u) * TM + tl;  // = (o * n + l) * n_inner + c
        d.act = tile < tiles && d.cell < a.cells;
        d.al = 0.0f;
#pragma unroll
        for (int k = 0; k < 6; ++k) d.f[k] = d.w[k] = 0.0f;
        if (d.act) {
            const int64_t c = d.cell % a.n_inner;
            const int l = (int)((d.cell / a.n_inner) % n);
            const int64_t o = d.cell / (a.n_inner * n);
            const float* col = a.in + (o * n) * a.n_inner + c;
            if constexpr (KICK) {
                // shift and weights in FP32 (the network corrects them anyway;
                // FP64 divisions per cell would dominate the kernel)
                const float e = (float)a.E[o / a.e_div];
                int s = kick_weights<float, float>(e, a.dt, a.dv, -1, d.w);
                s = max(-(1 << 28), min(1 << 28, s));
                const float dd = __fdiv_rn(__fmul_rn(e, (float)a.dt), (float)a.dv);
                d.al = __fsub_rn(dd, floorf(dd));
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    const int64_t r = (int64_t)l - s + 2 - k;
                    d.f[k] = (r >= 0 && r < n) ? col[r * a.n_inner] : 0.0f;
                }
            } else {
                const int j = (int)((c / a.sel_div) % a.sel_mod);
                const int s = a.shift[j];
                d.al = a.alpha[j];
                int r = (int)(((int64_t)l - s + 2) % n);
                if (r < 0) r += n;
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    d.f[k] = col[(int64_t)r * a.n_inner];
                    d.w[k] = a.W[k * a.sel_mod + j];
                    r = r == 0 ? n - 1 : r - 1;
                }
            }
        }
        return d;
    };

    // super-tiles: P tiles holding whole lines (one tile without projection);
    // training with projection passes over them twice (line sums, then the
    // forward + backward pass)
    const int P = a.per_st;
    const int npass = (TRAIN && a.proj) ? 2 : 1;
    const int items = npass * P;
    const int64_t n_super = tiles / P;
    auto tile_of = [&](int64_t st, int k) -> int64_t {
        return (((st >> a.st_lg) * P + k) << a.st_lg) + (st & ((1ll << a.st_lg) - 1));
    };
    float* lred = reinterpret_cast<float*>(sm + S.line);
    // a line's lanes: within a warp they are combined by shuffles (offsets
    // qstride, 2 qstride, ... < 32), across warps through shared memory
    // (cnt partials, xs apart, from gx)
    const int qspan = a.q * a.qstride;
    const int xs = max(a.qstride, 32);
    const int cnt = qspan / xs;
    const int gx = (tl / qspan) * qspan + tl % xs;
    const float inv_n = 1.0f / (float)n;  // exact: n is a power of two when projecting
    float lsum_c = 0.0f, lsum_d = 0.0f;   // this lane's share of its line's sums
    float mc = 0.0f, md = 0.0f;           // line means of (out - plain), (plain - target)

    int64_t st = blockIdx.x;
    int j = 0;
    CellData nxt = gather(st < n_super ? tile_of(st, 0) : tiles);
    while (st < n_super && ok) {
        const int pass = j / P, k_st = j - (j / P) * P;
        int64_t st2 = st;
        int j2 = j + 1;
        if (j2 == items) {
            st2 += gridDim.x;
            j2 = 0;
        }
        const int64_t tile2 = st2 < n_super ? tile_of(st2, j2 % P) : tiles;
        const bool last_pass = pass == npass - 1;
        const CellData cur = nxt;
        const bool act = cur.act;
        const int64_t cell = cur.cell;
        const float* f = cur.f;
        const float* w = cur.w;
        float sc = 0.0f;
#pragma unroll
        for (int k = 0; k < 6; ++k) sc = fmaxf(sc, fabsf(f[k]));
        const float inv = sc > 0.0f ? 1.0f / sc : 0.0f;
        {
            float xv[8];
#pragma unroll
            for (int k = 0; k < 6; ++k) xv[k] = f[k] * inv;
            xv[6] = act ? cur.al - 0.5f : 0.0f;
            xv[7] = 1.0f;
            st8_bf16(sm, S.x + ux + kmaj(tl, 0, K1), xv);
        }
        if (TRAIN) {
#pragma unroll
            for (int k = 0; k < 6; ++k) st_bf16(sm, S.bw + kmaj(K2 + k, t, KW), f[k] * inv);
            st_bf16(sm, S.bw + kmaj(K2 + 6, t, KW), act ? cur.al - 0.5f : 0.0f);
            st_bf16(sm, S.bw + kmaj(K2 + 7, t, KW), act ? 1.0f : 0.0f);
        }
        // layer 1
        if (!(ok = run_with(
                  [&] {
                      for (int v = 0; v < SUB; ++v)
                          gemm(tm + v * 128 + T_D1, base + S.x + v * XS, base + S.w1, K1, HID, false);
                  },
                  [&] { nxt = gather(tile2); })))
            break;
        uint32_t m1[2] = {0u, 0u}, m2[2] = {0u, 0u};  // relu masks of z1, z2
#pragma unroll
        for (int q = 0; q < HID / 16; q += 2) {  // two loads in flight per wait
            float v[32];
            tmem_ld16(lane_base + T_D1 + q * 16, *reinterpret_cast<float(*)[16]>(v));
            tmem_ld16(lane_base + T_D1 + q * 16 + 16, *reinterpret_cast<float(*)[16]>(v + 16));
            tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const int h = q * 16 + i;
                const bool pos = v[i] > 0.0f;
                if (TRAIN && pos) m1[h >> 5] |= 1u << (h & 31);
                v[i] = act && pos ? v[i] : 0.0f;
                if (TRAIN) st_bf16(sm, S.bw + kmaj(h, t, KW), v[i]);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) st8_bf16(sm, S.h1 + uh + kmaj(tl, q * 16 + 8 * i, K2), v + 8 * i);
        }
        // layer 2
        if (!(ok = run([&] {
                  for (int v = 0; v < SUB; ++v)
                      gemm(tm + v * 128 + T_D2, base + S.h1 + v * HS, base + S.w2, K2, HID, false);
              })))
            break;
#pragma unroll
        for (int q = 0; q < HID / 16; q += 2) {  // two loads in flight per wait
            float v[32];
            tmem_ld16(lane_base + T_D2 + q * 16, *reinterpret_cast<float(*)[16]>(v));
            tmem_ld16(lane_base + T_D2 + q * 16 + 16, *reinterpret_cast<float(*)[16]>(v + 16));
            tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const int h = q * 16 + i;
                const bool pos = v[i] > 0.0f;
                if (TRAIN && pos) m2[h >> 5] |= 1u << (h & 31);
                v[i] = act && pos ? v[i] : 0.0f;
                if (TRAIN) st_bf16(sm, S.h2t + kmaj(h, t, KW), v[i]);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) st8_bf16(sm, S.h2 + uh + kmaj(tl, q * 16 + 8 * i, K2), v + 8 * i);
        }
        if (TRAIN) st_bf16(sm, S.h2t + kmaj(HID, t, KW), act ? 1.0f : 0.0f);
        // layer 3
        if (!(ok = run([&] {
                  for (int v = 0; v < SUB; ++v)
                      gemm(tm + v * 128 + TD3, base + S.h2 + v * HS, base + S.w3, K2, NO, false);
              })))
            break;
        float ov[16];
        tmem_ld16(lane_base + TD3, ov);
        tmem_wait_ld();
        float mean = 0.0f;
#pragma unroll
        for (int k = 0; k < 6; ++k) mean += ov[k];
        mean *= (1.0f / 6.0f);
        float y = 0.0f, yp = 0.0f;
#pragma unroll
        for (int k = 0; k < 6; ++k) y = fmaf(w[k] + (ov[k] - mean), f[k], y);
        if (a.proj) {
#pragma unroll
            for (int k = 0; k < 6; ++k) yp = fmaf(w[k], f[k], yp);
        }
        if (!TRAIN) {
            if (act) {
                a.out[cell] = y;
                lsum_c += y - yp;
            }
        } else if (!last_pass) {
            if (act) {
                const float tg = a.target[cell];
                lsum_c += y - yp;
                lsum_d += yp - tg;
            }
        } else {
            // ---- training: residual, deltas, weight gradients ----
            const float tg = act ? a.target[cell] : 0.0f;
            const float r = act ? (y - mc - tg) * a.inv_scale : 0.0f;
            loss_acc += (double)r * r;
            const float gy = act ? 2.0f * (r - md * a.inv_scale) * a.inv_scale : 0.0f;  // dL/dy, less its line mean
            float g6[6], gm = 0.0f;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                g6[k] = gy * f[k];
                gm += g6[k];
            }
            gm *= (1.0f / 6.0f);
            {
                float dv8[8];
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    dv8[k] = act ? g6[k] - gm : 0.0f;
                    st_bf16(sm, S.doT + kmaj(k, t, KW), dv8[k]);
                }
                dv8[6] = dv8[7] = 0.0f;
                st8_bf16(sm, S.dO + kmaj(t, 0, NO), dv8);
            }
            // dh2 = do W3 (B = W3^T [64][16])
            if (!(ok = run([&] { gemm(tm + T_G2, base + S.dO, base + S.w3t, NO, HID, false); }))) break;
#pragma unroll
            for (int q = 0; q < HID / 16; ++q) {
                float v[16];
                tmem_ld16(lane_base + T_G2 + q * 16, v);
                tmem_wait_ld();
                float dz[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int h = q * 16 + i;
                    dz[i] = act && ((m2[h >> 5] >> (h & 31)) & 1u) ? v[i] : 0.0f;
                    st_bf16(sm, S.aw + kmaj(h, t, KW), dz[i]);
                }
                st8_bf16(sm, S.dz2 + kmaj(t, q * 16, HID), dz);
                st8_bf16(sm, S.dz2 + kmaj(t, q * 16 + 8, HID), dz + 8);
            }
            // dh1 = dz2 W2 (B = W2^T [64][64])
            if (!(ok = run([&] { gemm(tm + T_G1, base + S.dz2, base + S.w2t, HID, HID, false); }))) break;
#pragma unroll
            for (int q = 0; q < HID / 16; ++q) {
                float v[16];
                tmem_ld16(lane_base + T_G1 + q * 16, v);
                tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int h = q * 16 + i;
                    const float d = (m1[h >> 5] >> (h & 31)) & 1u ? v[i] : 0.0f;
                    st_bf16(sm, S.aw + kmaj(HID + h, t, KW), act ? d : 0.0f);
                }
            }
            // weight gradients over this tile's cells (K = the 128 cells)
            const bool acc_w = wacc;
            if (!(ok = run([&] {
                      gemm(tm + T_WA, base + S.aw, base + S.bw, KW, 96, acc_w);
                      gemm(tm + T_WB, base + S.h2t, base + S.doT, KW, NO, acc_w);
                  })))
                break;
            wacc = true;
        }
        // end of the super-tile's first pass: line means, then (inference)
        // the outputs it wrote are moved onto the plain sweep's line sums
        if (a.proj && pass == 0 && k_st == P - 1) {
            for (int off = a.qstride; off < 32 && off < qspan; off <<= 1) {
                lsum_c += __shfl_xor_sync(0xffffffffu, lsum_c, off);
                lsum_d += __shfl_xor_sync(0xffffffffu, lsum_d, off);
            }
            if (cnt > 1) {
                lred[tl] = lsum_c;
                lred[TM + tl] = lsum_d;
                __syncthreads();
                lsum_c = lsum_d = 0.0f;
                for (int m = 0; m < cnt; ++m) {
                    lsum_c += lred[gx + m * xs];
                    lsum_d += lred[TM + gx + m * xs];
                }
                __syncthreads();
            }
            mc = lsum_c * inv_n;
            md = lsum_d * inv_n;
            lsum_c = lsum_d = 0.0f;
            if (!TRAIN) {
                for (int k = 0; k < P; ++k) {
                    const int64_t c2 = tile_of(st, k) * TM + tl;
                    if (c2 < a.cells) a.out[c2] -= mc;
                }
            }
        }
        st = st2;
        j = j2;
    }

    if (TRAIN && ok && wacc) {
        // lanes 0-63: dW2 (columns 0-79 of WA); lanes 64-127: dW1 (columns 80-95)
        if (t < HID) {
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                float v[16];
                tmem_ld16(lane_base + T_WA + q * 16, v);
                tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) atomicAdd(&a.grad[G_W2 + t * K2 + q * 16 + i], v[i]);
            }
        } else {
            float v[16];
            tmem_ld16(lane_base + T_WA + 80, v);
            tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 16; ++i) atomicAdd(&a.grad[G_W1 + (t - HID) * K1 + i], v[i]);
        }
        // dW3^T: lane h (< 80) holds dW3[o][h] in column o
        {
            float v[16];
            tmem_ld16(lane_base + T_WB, v);
            tmem_wait_ld();
            if (t < K2) {
#pragma unroll
                for (int i = 0; i < 6; ++i) atomicAdd(&a.grad[G_W3 + i * K2 + t], v[i]);
            }
        }
    }
    if (TRAIN) {
        double* red = reinterpret_cast<double*>(sm + S.loss);
        red[t] = loss_acc;
        __syncthreads();
        if (t == 0) {
            double sum = 0.0;
            for (int i = 0; i < NT; ++i) sum += red[i];
            atomicAdd(a.loss, sum);
        }
    }
    if (!ok && t == 0) atomicExch(a.status, 1);
    fence_before();
    __syncthreads();
    fence_after();
    if (t < 32) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(ncols) : "memory");
    }
}

}  // namespace mlp

size_t mlp_smem_bytes(bool train) { return mlp::plan(train).total; }

int run_mlp_sweep(bool train, bool kick, const MlpSweepArgs& args, cudaStream_t st) {
    MlpSweepArgs a = args;
    a.cells = a.n_outer * a.n_line * a.n_inner;
    const int64_t tiles = (a.cells + mlp::TM - 1) / mlp::TM;
    // line projection when n_line and n_inner are powers of two; a line
    // (o, c) of n cells n_inner apart occupies
    //   n_inner >= TM:      one lane in each of n tiles (n_inner / TM tiles apart)
    //   n * n_inner >= TM:  TM / n_inner lanes in each of n * n_inner / TM consecutive tiles
    //   n * n_inner <  TM:  n lanes of one tile
    auto pow2 = [](int64_t v) { return v > 0 && (v & (v - 1)) == 0; };
    const int64_t n = a.n_line, ni = a.n_inner;
    a.proj = pow2(n) && pow2(ni) ? 1 : 0;
    a.per_st = 1;
    a.q = 1;
    a.qstride = 1;
    a.st_lg = 0;
    if (a.proj) {
        if (ni >= mlp::TM) {
            a.per_st = (int)n;
            while ((mlp::TM << a.st_lg) < ni) a.st_lg++;
        } else if (n * ni >= mlp::TM) {
            a.q = (int)(mlp::TM / ni);
            a.qstride = (int)ni;
            a.per_st = (int)(n * ni / mlp::TM);
        } else {
            a.q = (int)n;
            a.qstride = (int)ni;
        }
    }
    // inference asks for at least 48 KB so that no more than four CTAs (4 x 128
    // tensor-memory columns) share an SM
    const size_t smem = train ? mlp_smem_bytes(true) : std::max<size_t>(mlp_smem_bytes(false), 48 * 1024);
    auto kern = train ? (kick ? mlp::k_mlp_sweep<true, true> : mlp::k_mlp_sweep<true, false>)
                      : (kick ? mlp::k_mlp_sweep<false, true> : mlp::k_mlp_sweep<false, false>);
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return set_cuda_error("cudaFuncSetAttribute(k_mlp_sweep)");
    // training holds all 512 tensor-memory columns: one CTA per SM;
    // inference holds 128: four CTAs per SM
    const int64_t per_sm = train ? 1 : 4;
    const int64_t n_super = tiles / a.per_st;  // super-tiles (tiles without projection)
    const int64_t grid = std::min<int64_t>(n_super, (int64_t)sm_count() * per_sm);
    kern<<<(unsigned)std::max<int64_t>(grid, 1), mlp::TM * mlp::subtiles(train), smem, st>>>(a);
    return check_launch("k_mlp_sweep");
}

int mlp_net_elems() { return mlp::NET_ELEMS; }
int mlp_grad_elems() { return mlp::GRAD_ELEMS; }

}  // namespace vp

using namespace vp;

extern "C" {

static int mlp_sizes(int64_t n_outer, int64_t n_line, int64_t n_inner) {
    if (n_outer <= 0 || n_line <= 0 || n_inner <= 0 || n_line >= (1 << 30) || n_outer * n_line * n_inner < 0)
        return set_error(VP_ERR_ARG, "vp_mlp: bad size");
    return VP_OK;
}

static MlpSweepArgs drift_args(const float* f_in, int64_t n_outer, int64_t n_line, int64_t n_inner, int64_t sel_div,
                               int64_t sel_mod, const int32_t* shift, const float* W, const float* alpha,
                               const void* net, int32_t* status) {
    MlpSweepArgs a{};
    a.in = f_in;
    a.n_outer = n_outer;
    a.n_line = (int)n_line;
    a.n_inner = n_inner;
    a.sel_div = sel_div;
    a.sel_mod = (int)sel_mod;
    a.shift = shift;
    a.W = W;
    a.alpha = alpha;
    a.e_div = 1;
    a.dv = 1.0;
    a.net = static_cast<const __nv_bfloat16*>(net);
    a.inv_scale = 1.0f;
    a.status = reinterpret_cast<int*>(status);
    return a;
}

static MlpSweepArgs kick_args(const float* f_in, int64_t n_outer, int64_t n_line, int64_t n_inner, const double* E,
                              int64_t e_div, double dt, double dv, const void* net, int32_t* status) {
    MlpSweepArgs a{};
    a.in = f_in;
    a.n_outer = n_outer;
    a.n_line = (int)n_line;
    a.n_inner = n_inner;
    a.sel_div = 1;
    a.sel_mod = 1;
    a.E = E;
    a.e_div = e_div;
    a.dt = dt;
    a.dv = dv;
    a.net = static_cast<const __nv_bfloat16*>(net);
    a.inv_scale = 1.0f;
    a.status = reinterpret_cast<int*>(status);
    return a;
}

int vp_mlp_drift(const float* f_in, float* f_out, int64_t n_outer, int64_t n_line, int64_t n_inner, int64_t sel_div,
                 int64_t sel_mod, const int32_t* shift, const float* W, const float* alpha, const void* net,
                 int32_t* status, void* stream) {
    if (!f_in || !net || !shift || !W || !alpha || !status) return set_error(VP_ERR_ARG, "vp_mlp_drift: null pointer");
    if (!f_out || f_out == f_in) return set_error(VP_ERR_ARG, "vp_mlp_drift: f_out null or aliasing f_in");
    if (sel_div <= 0 || sel_mod <= 0) return set_error(VP_ERR_ARG, "vp_mlp_drift: bad table size");
    int rc = mlp_sizes(n_outer, n_line, n_inner);
    if (rc) return rc;
    MlpSweepArgs a = drift_args(f_in, n_outer, n_line, n_inner, sel_div, sel_mod, shift, W, alpha, net, status);
    a.out = f_out;
    return run_mlp_sweep(false, false, a, static_cast<cudaStream_t>(stream));
}

int vp_mlp_train(const float* f_in, const float* target, int64_t n_outer, int64_t n_line, int64_t n_inner,
                 int64_t sel_div, int64_t sel_mod, const int32_t* shift, const float* W, const float* alpha,
                 const void* net, double inv_scale, float* grad, double* loss, int32_t* status, void* stream) {
    if (!f_in || !net || !shift || !W || !alpha || !status) return set_error(VP_ERR_ARG, "vp_mlp_train: null pointer");
    if (!target || !grad || !loss) return set_error(VP_ERR_ARG, "vp_mlp_train: null target, grad or loss");
    if (sel_div <= 0 || sel_mod <= 0) return set_error(VP_ERR_ARG, "vp_mlp_train: bad table size");
    int rc = mlp_sizes(n_outer, n_line, n_inner);
    if (rc) return rc;
    MlpSweepArgs a = drift_args(f_in, n_outer, n_line, n_inner, sel_div, sel_mod, shift, W, alpha, net, status);
    a.target = target;
    a.grad = grad;
    a.loss = loss;
    a.inv_scale = (float)inv_scale;
    return run_mlp_sweep(true, false, a, static_cast<cudaStream_t>(stream));
}

int vp_mlp_kick(const float* f_in, float* f_out, int64_t n_outer, int64_t n_line, int64_t n_inner, const double* E,
                int64_t e_div, double dt, double dv, const void* net, int32_t* status, void* stream) {
    if (!f_in || !E || !net || !status) return set_error(VP_ERR_ARG, "vp_mlp_kick: null pointer");
    if (!f_out || f_out == f_in) return set_error(VP_ERR_ARG, "vp_mlp_kick: f_out null or aliasing f_in");
    if (e_div <= 0 || n_outer % e_div || dv == 0.0) return set_error(VP_ERR_ARG, "vp_mlp_kick: bad e_div or dv");
    int rc = mlp_sizes(n_outer, n_line, n_inner);
    if (rc) return rc;
    MlpSweepArgs a = kick_args(f_in, n_outer, n_line, n_inner, E, e_div, dt, dv, net, status);
    a.out = f_out;
    return run_mlp_sweep(false, true, a, static_cast<cudaStream_t>(stream));
}

int vp_mlp_train_kick(const float* f_in, const float* target, int64_t n_outer, int64_t n_line, int64_t n_inner,
                      const double* E, int64_t e_div, double dt, double dv, const void* net, double inv_scale,
                      float* grad, double* loss, int32_t* status, void* stream) {
    if (!f_in || !E || !net || !status) return set_error(VP_ERR_ARG, "vp_mlp_train_kick: null pointer");
    if (!target || !grad || !loss) return set_error(VP_ERR_ARG, "vp_mlp_train_kick: null target, grad or loss");
    if (e_div <= 0 || n_outer % e_div || dv == 0.0) return set_error(VP_ERR_ARG, "vp_mlp_train_kick: bad e_div or dv");
    int rc = mlp_sizes(n_outer, n_line, n_inner);
    if (rc) return rc;
    MlpSweepArgs a = kick_args(f_in, n_outer, n_line, n_inner, E, e_div, dt, dv, net, status);
    a.target = target;
    a.grad = grad;
    a.loss = loss;
    a.inv_scale = (float)inv_scale;
    return run_mlp_sweep(true, true, a, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
