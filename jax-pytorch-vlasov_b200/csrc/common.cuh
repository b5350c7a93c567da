// Shared device helpers of the Vlasov-Poisson library (sm_100a).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/vlasov_b200.h"

namespace vp {

// ---------------------------------------------------------------------------
// storage type -> compute type
// ---------------------------------------------------------------------------
template <typename TS> struct Compute;
template <> struct Compute<float> { using type = float; };
template <> struct Compute<double> { using type = double; };
template <> struct Compute<__nv_bfloat16> { using type = float; };
template <typename TS> using compute_t = typename Compute<TS>::type;

__device__ __forceinline__ float to_c(float v) { return v; }
__device__ __forceinline__ double to_c(double v) { return v; }
__device__ __forceinline__ float to_c(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename TS> __device__ __forceinline__ TS from_c(compute_t<TS> v);
template <> __device__ __forceinline__ float from_c<float>(float v) { return v; }
template <> __device__ __forceinline__ double from_c<double>(double v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_c<__nv_bfloat16>(float v) {
    return __float2bfloat16_rn(v);
}

// VEC consecutive storage elements moved as one aligned access
// (16 B for 4 x float, 8 B for 4 x bf16, 32 B as two 16 B for 4 x double).
template <typename TS, int VEC> struct Vec { compute_t<TS> v[VEC]; };

template <typename TS, int VEC>
__device__ __forceinline__ Vec<TS, VEC> ldv(const TS* __restrict__ p) {
    Vec<TS, VEC> r;
    if constexpr (VEC == 1) {
        r.v[0] = to_c(__ldg(p));
    } else if constexpr (VEC == 4 && sizeof(TS) == 4) {
        float4 t = __ldg(reinterpret_cast<const float4*>(p));
        r.v[0] = t.x; r.v[1] = t.y; r.v[2] = t.z; r.v[3] = t.w;
    } else if constexpr (VEC == 4 && sizeof(TS) == 2) {
        uint2 t = __ldg(reinterpret_cast<const uint2*>(p));
        __nv_bfloat162 a = *reinterpret_cast<__nv_bfloat162*>(&t.x);
        __nv_bfloat162 b = *reinterpret_cast<__nv_bfloat162*>(&t.y);
        float2 fa = __bfloat1622float2(a), fb = __bfloat1622float2(b);
        r.v[0] = fa.x; r.v[1] = fa.y; r.v[2] = fb.x; r.v[3] = fb.y;
    } else if constexpr (VEC == 2 && sizeof(TS) == 8) {
        double2 t = __ldg(reinterpret_cast<const double2*>(p));
        r.v[0] = t.x; r.v[1] = t.y;
    } else if constexpr (VEC == 4 && sizeof(TS) == 8) {
        double2 t = __ldg(reinterpret_cast<const double2*>(p));
        double2 u = __ldg(reinterpret_cast<const double2*>(p) + 1);
        r.v[0] = t.x; r.v[1] = t.y; r.v[2] = u.x; r.v[3] = u.y;
    } else if constexpr (VEC == 2 && sizeof(TS) == 4) {
        float2 t = __ldg(reinterpret_cast<const float2*>(p));
        r.v[0] = t.x; r.v[1] = t.y;
    } else {
#pragma unroll
        for (int e = 0; e < VEC; ++e) r.v[e] = to_c(__ldg(p + e));
    }
    return r;
}

template <typename TS, int VEC>
__device__ __forceinline__ void stv(TS* __restrict__ p, const Vec<TS, VEC>& r) {
    if constexpr (VEC == 1) {
        p[0] = from_c<TS>(r.v[0]);
    } else if constexpr (VEC == 4 && sizeof(TS) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(r.v[0], r.v[1], r.v[2], r.v[3]);
    } else if constexpr (VEC == 4 && sizeof(TS) == 2) {
        __nv_bfloat162 a = __floats2bfloat162_rn(r.v[0], r.v[1]);
        __nv_bfloat162 b = __floats2bfloat162_rn(r.v[2], r.v[3]);
        uint2 t;
        t.x = *reinterpret_cast<uint32_t*>(&a);
        t.y = *reinterpret_cast<uint32_t*>(&b);
        *reinterpret_cast<uint2*>(p) = t;
    } else if constexpr (VEC == 2 && sizeof(TS) == 8) {
        *reinterpret_cast<double2*>(p) = make_double2(r.v[0], r.v[1]);
    } else if constexpr (VEC == 4 && sizeof(TS) == 8) {
        reinterpret_cast<double2*>(p)[0] = make_double2(r.v[0], r.v[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2(r.v[2], r.v[3]);
    } else if constexpr (VEC == 2 && sizeof(TS) == 4) {
        *reinterpret_cast<float2*>(p) = make_float2(r.v[0], r.v[1]);
    } else {
#pragma unroll
        for (int e = 0; e < VEC; ++e) p[e] = from_c<TS>(r.v[e]);
    }
}

// A chunk row as it is held between its load and its use: the packed
// storage bits for 4 x bf16 (2 registers; unpacked where the stencil reads
// them, so the loads of a whole chunk stay in flight together), the compute
// vector itself for every other case.
template <typename TS, int VEC>
struct Raw {
    static constexpr bool packed = sizeof(TS) == 2 && VEC == 4;
    using type = Vec<TS, VEC>;
};
template <>
struct Raw<__nv_bfloat16, 4> {
    static constexpr bool packed = true;
    using type = uint2;
};

template <typename TS, int VEC>
__device__ __forceinline__ typename Raw<TS, VEC>::type ldraw(const TS* __restrict__ p) {
    if constexpr (Raw<TS, VEC>::packed) {
        return __ldg(reinterpret_cast<const uint2*>(p));
    } else {
        return ldv<TS, VEC>(p);
    }
}

template <typename TS, int VEC>
__device__ __forceinline__ typename Raw<TS, VEC>::type raw_zero() {
    if constexpr (Raw<TS, VEC>::packed) {
        return make_uint2(0u, 0u);
    } else {
        Vec<TS, VEC> z;
#pragma unroll
        for (int e = 0; e < VEC; ++e) z.v[e] = compute_t<TS>(0);
        return z;
    }
}

// element e (a compile-time index after unrolling) of a held row
template <typename TS, int VEC>
__device__ __forceinline__ compute_t<TS> raw_get(const typename Raw<TS, VEC>::type& r, int e) {
    if constexpr (Raw<TS, VEC>::packed) {
        const uint32_t w = (e < 2) ? r.x : r.y;
        return __uint_as_float((e & 1) ? (w & 0xFFFF0000u) : (w << 16));  // bf16 -> f32 is exact
    } else {
        return r.v[e];
    }
}

template <typename TS, int VEC>
__device__ __forceinline__ Vec<TS, VEC> raw_vec(const typename Raw<TS, VEC>::type& r) {
    if constexpr (Raw<TS, VEC>::packed) {
        Vec<TS, VEC> v;
#pragma unroll
        for (int e = 0; e < VEC; ++e) v.v[e] = raw_get<TS, VEC>(r, e);
        return v;
    } else {
        return r;
    }
}

// The value a stored element reads back as (rounding of the storage type).
template <typename TS> __device__ __forceinline__ compute_t<TS> as_stored(compute_t<TS> v) {
    return to_c(from_c<TS>(v));
}

// ---------------------------------------------------------------------------
// Lagrange weights of the 6-point stencil (nodes -2..3), evaluated with the
// reference's closed-form polynomials (lagrange5_weights,
// vlasov2D2V.py:263-285) term by term, each operation rounded on its own
// (explicit _rn intrinsics keep the compiler from contracting into FMAs), so
// a double evaluation matches the reference's FP64 weights bit for bit.
// ---------------------------------------------------------------------------
struct RnD {
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
};
struct RnF {
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
};
template <typename C> struct Rn;
template <> struct Rn<double> : RnD {};
template <> struct Rn<float> : RnF {};

template <typename C>
__device__ __forceinline__ void lagrange6(C a, C w[6]) {
    using R = Rn<C>;
    const C a2 = R::mul(a, a), a3 = R::mul(a2, a), a4 = R::mul(a3, a), a5 = R::mul(a4, a);
    // w0 = a/20 - a2/24 - a3/24 + a4/24 - a5/120
    w[0] = R::sub(R::add(R::sub(R::sub(R::div(a, C(20)), R::div(a2, C(24))), R::div(a3, C(24))),
                         R::div(a4, C(24))),
                  R::div(a5, C(120)));
    // w1 = -(a/2) + (2 a2)/3 - a3/24 - a4/6 + a5/24
    w[1] = R::add(R::sub(R::sub(R::add(-R::div(a, C(2)), R::div(R::mul(C(2), a2), C(3))),
                                R::div(a3, C(24))),
                         R::div(a4, C(6))),
                  R::div(a5, C(24)));
    // w2 = 1 - a/3 - (5 a2)/4 + (5 a3)/12 + a4/4 - a5/12
    w[2] = R::sub(R::add(R::add(R::sub(R::sub(C(1), R::div(a, C(3))), R::div(R::mul(C(5), a2), C(4))),
                                R::div(R::mul(C(5), a3), C(12))),
                         R::div(a4, C(4))),
                  R::div(a5, C(12)));
    // w3 = a + (2 a2)/3 - (7 a3)/12 - a4/6 + a5/12
    w[3] = R::add(R::sub(R::sub(R::add(a, R::div(R::mul(C(2), a2), C(3))),
                                R::div(R::mul(C(7), a3), C(12))),
                         R::div(a4, C(6))),
                  R::div(a5, C(12)));
    // w4 = -(a/4) - a2/24 + (7 a3)/24 + a4/24 - a5/24
    w[4] = R::sub(R::add(R::add(R::sub(-R::div(a, C(4)), R::div(a2, C(24))),
                                R::div(R::mul(C(7), a3), C(24))),
                         R::div(a4, C(24))),
                  R::div(a5, C(24)));
    // w5 = a/30 - a3/24 + a5/120
    w[5] = R::add(R::sub(R::div(a, C(30)), R::div(a3, C(24))), R::div(a5, C(120)));
}

// Shift and weights of a kick with field value e: d = (e*dt)/dv, s = floor(d),
// alpha = d - s (build_v_tap_weights, vlasov2D2V.py:852-856), evaluated in
// the field's precision F and handed to the sweep in the compute type C.
// window >= 0 zeroes the taps outside the reference's static window.
template <typename F, typename C>
__device__ __forceinline__ int kick_weights(F e, double dt, double dv, int window, C w[6]) {
    using R = Rn<F>;
    const F d = R::div(R::mul(e, F(dt)), F(dv));
    const F fl = floor(d);
    const F alpha = R::sub(d, fl);
    F wf[6];
    lagrange6<F>(alpha, wf);
    const int s = (int)fl;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const int m = s + k - 2;
        const bool keep = window < 0 || (m >= -window - 2 && m <= window + 2);
        w[k] = keep ? C(wf[k]) : C(0);
    }
    return s;
}

__device__ __forceinline__ int wrap_up(int r, int n) {
    while (r >= n) r -= n;
    return r;
}

// ---------------------------------------------------------------------------
// shared-memory addresses, the global timer, mbarrier waits with a limit
// ---------------------------------------------------------------------------
// Programmatic dependent launch. pdl_release (at a kernel's start) lets the
// next launch on the stream, made with the programmatic-serialization
// attribute, start its CTAs while this grid still runs; pdl_hold (before a
// kernel exits) waits until the launch before it has completed and its
// writes are visible, and returns at once for a launch made without the
// attribute. A dependent launch must not touch what its predecessor touches;
// holding before exit makes its completion imply the predecessor's, so the
// ordinary launches after it see both.
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_hold() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t now_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// wait for the mbarrier phase with the given parity; false after ~1 s
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    const uint64_t t0 = now_ns();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (now_ns() - t0 > 1000000000ull) return false;
    }
}

}  // namespace vp
