// pushmath.cuh — the velocity factor 1 - Vx of the plasma push in the form
// the fast push kernels use, shared by the push kernels (push.cuh) and the
// push adjoint's recompute (adjoint.cu), so that the adjoint recomputes
// exactly the push the forward ran; and the cell index helpers and value
// pairs both use.
//
// The push divides by 1 - Vx (movepart_splitlayer.cpp:1258-1371: the kicks
// q2m hx/2 E/(1-Vx), the deposits w dJ V/(1-Vx), the transverse move
// V hx/h/(1-Vx)).  For an electron moving forward fast (px > 0, Vx -> 1) the
// difference 1 - px/gamma cancels: in FP32 its relative error grows as
// 6e-8 / (1 - Vx).  The fast kernels therefore use the equal form
//     1 - px/g = (g - px)/g = (1 + py^2 + pz^2) / (g (g + px)),   g = sqrt(1 + p^2),
// for px > 0, which has no cancellation, and 1 - px/g itself for px <= 0
// (no cancellation there either): in FP32, and in FP64 for the grouped push
// of the FP64 path on FFT transforms.  The plain FP64 path keeps the
// reference's own expression order for bit-exact parity.
#pragma once
#include <cuda_runtime.h>

namespace qs {

// Approximate reciprocal: PTX rcp.approx.ftz.f32, one special-function
// instruction, at most 1 ulp from 1/x (PTX ISA), in place of the correctly
// rounded reciprocal's refinement sequence.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// 1 - px / g for momentum (px, py, pz) with inv_g = 1 / sqrt(1 + p^2)
__device__ __forceinline__ float one_minus_vx(float px, float py, float pz, float inv_g) {
    const float pt2 = fmaf(py, py, pz * pz);                   // py^2 + pz^2
    const float g = (1.f + fmaf(px, px, pt2)) * inv_g;         // sqrt(1 + p^2)
    const float fwd = (1.f + pt2) * inv_g * rcp_approx(g + px);
    const float bwd = fmaf(-px, inv_g, 1.f);
    return px > 0.f ? fwd : bwd;
}

__device__ __forceinline__ double one_minus_vx(double px, double py, double pz, double inv_g) {
    const double pt2 = fma(py, py, pz * pz);
    const double g = (1.0 + fma(px, px, pt2)) * inv_g;
    const double fwd = (1.0 + pt2) * inv_g / (g + px);
    const double bwd = fma(-px, inv_g, 1.0);
    return px > 0.0 ? fwd : bwd;
}

// j within one period of [0, M) (a shift of at most one period): no loop
__device__ __forceinline__ int wrap1(int j, int M) {
    j += (j < 0) ? M : 0;
    return j - ((j >= M) ? M : 0);
}

// k = cell / My, j = cell % My through a float reciprocal with correction
// (exact for cell < 2^24)
__device__ __forceinline__ void cell_jk(int cell, int My, float invMy, int& j, int& k) {
    int q = (int)((float)cell * invMy);
    int r = cell - q * My;
    if (r < 0) { q -= 1; r += My; }
    else if (r >= My) { q += 1; r -= My; }
    j = r;
    k = q;
}

// Value pairs: the field pairs of the grouped push's tile, (Ex, Ey), (Ez,
// Bx), (By, Bz), and the push adjoint's field-adjoint pairs.  In FP32 the
// packed instructions of sm_100 (__ffma2_rn and friends: two FP32 lanes,
// each rounded as fmaf, so the sums are those of the scalar chain), in FP64
// two FMAs.
template <class T>
struct FPair;
template <>
struct FPair<float> {
    using type = float2;
    static __device__ __forceinline__ float2 make(float x, float y) { return make_float2(x, y); }
    static __device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
    static __device__ __forceinline__ float2 mul(float s, float2 v) {
        return __fmul2_rn(make_float2(s, s), v);
    }
    static __device__ __forceinline__ float2 fma(float s, float2 v, float2 c) {
        return __ffma2_rn(make_float2(s, s), v, c);
    }
};
template <>
struct FPair<double> {
    using type = double2;
    static __device__ __forceinline__ double2 make(double x, double y) { return make_double2(x, y); }
    static __device__ __forceinline__ double2 add(double2 a, double2 b) {
        return make_double2(a.x + b.x, a.y + b.y);
    }
    static __device__ __forceinline__ double2 mul(double s, double2 v) {
        return make_double2(s * v.x, s * v.y);
    }
    static __device__ __forceinline__ double2 fma(double s, double2 v, double2 c) {
        return make_double2(::fma(s, v.x, c.x), ::fma(s, v.y, c.y));
    }
};

}  // namespace qs
