// Initial conditions of the drivers: f[p][v] = S[p] * V[v], a spatial profile
// times a velocity profile, both FP64, the product rounded once to the
// storage type. The reference builds the same tensors with broadcasting
// products in the run's device memory (Landau: (1 + eps cos kx cos ky) times
// exp(-|v|^2/2)/sqrt(2 pi), vlasov2D2V.py:1319-1355; 1D: vlasov1D1V.py:881-911);
// one product in FP64 and one rounding give the same bits as torch's
// broadcast multiply followed by .to(dtype).
//
// Write-bound: each thread stores 4 consecutive v of one point (one 16-byte
// FP32 store, 8 bytes in BF16, two 16-byte stores in FP64) in a grid-stride
// loop sized to the SM count.
#include <algorithm>

#include "common.cuh"
#include "launch.h"

namespace vp {

__device__ __forceinline__ void store_rounded(float* p, double v) { *p = (float)v; }
__device__ __forceinline__ void store_rounded(double* p, double v) { *p = v; }
__device__ __forceinline__ void store_rounded(__nv_bfloat16* p, double v) { *p = __double2bfloat16(v); }

template <typename TS>
__global__ void __launch_bounds__(256) k_init_product(const double* __restrict__ S, const double* __restrict__ V,
                                                      TS* __restrict__ f, int64_t n_points, int64_t n_v) {
    const int64_t per = n_v / 4;  // groups of 4 v per point (n_v % 4 == 0 on this path)
    const int64_t total = n_points * per;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = i / per;
        const int64_t v = (i - p * per) * 4;
        const double s = __ldg(S + p);
        TS* dst = f + p * n_v + v;
        if constexpr (sizeof(TS) == 4) {
            *reinterpret_cast<float4*>(dst) = make_float4((float)(s * __ldg(V + v)), (float)(s * __ldg(V + v + 1)),
                                                          (float)(s * __ldg(V + v + 2)), (float)(s * __ldg(V + v + 3)));
        } else if constexpr (sizeof(TS) == 8) {
            reinterpret_cast<double2*>(dst)[0] = make_double2(s * __ldg(V + v), s * __ldg(V + v + 1));
            reinterpret_cast<double2*>(dst)[1] = make_double2(s * __ldg(V + v + 2), s * __ldg(V + v + 3));
        } else {
            __nv_bfloat16 h[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) h[e] = __double2bfloat16(s * __ldg(V + v + e));
            *reinterpret_cast<uint2*>(dst) = *reinterpret_cast<const uint2*>(h);
        }
    }
}

// any n_v, any alignment: one element per thread
template <typename TS>
__global__ void __launch_bounds__(256) k_init_product_scalar(const double* __restrict__ S,
                                                             const double* __restrict__ V, TS* __restrict__ f,
                                                             int64_t n_points, int64_t n_v) {
    const int64_t total = n_points * n_v;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = i / n_v;
        store_rounded(f + i, __ldg(S + p) * __ldg(V + (i - p * n_v)));
    }
}

template <typename TS>
static int launch_init(const double* S, const double* V, void* f, int64_t n_points, int64_t n_v, cudaStream_t st) {
    const size_t align = sizeof(TS) == 2 ? 8 : 16;
    const bool vec = n_v % 4 == 0 && reinterpret_cast<uintptr_t>(f) % align == 0;
    const int64_t work = vec ? n_points * (n_v / 4) : n_points * n_v;
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, (int64_t)sm_count() * 8));
    if (vec)
        k_init_product<TS><<<(unsigned)grid, 256, 0, st>>>(S, V, static_cast<TS*>(f), n_points, n_v);
    else
        k_init_product_scalar<TS><<<(unsigned)grid, 256, 0, st>>>(S, V, static_cast<TS*>(f), n_points, n_v);
    return check_launch("k_init_product");
}

int run_init_product(int dtype, const double* S, const double* V, void* f, int64_t n_points, int64_t n_v,
                     cudaStream_t st) {
    if (dtype == VP_F32) return launch_init<float>(S, V, f, n_points, n_v, st);
    if (dtype == VP_F64) return launch_init<double>(S, V, f, n_points, n_v, st);
    return launch_init<__nv_bfloat16>(S, V, f, n_points, n_v, st);
}

}  // namespace vp
