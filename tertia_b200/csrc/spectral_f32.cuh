// spectral_f32.cuh — the fast per-mode predictor / corrector maps
// (GuessFieldsHydroLinLayerSplit, movefieldshydrolinlayersplit.cpp:808-900;
// IterateFieldsHydroLinLayerSplit, :1374-1477) on two adjacent modes, shared
// by the FP32 map kernels (spectral_f32.cu) and the kernels that apply them
// between the two halves of a transform (dtt_fft.cu: FP32, and FP64 on the
// FFT path).  R is the real type.
//
// Same algebra as predictor_kernel / corrector_kernel in spectral.cu, arranged
// for the GPU rather than for bit-exact agreement with the oracle: the five
// divisions of a mode become two reciprocals, 1/k^2 and 1/(k^2 + density),
// plus uniform constants; beam-spectrum terms whose xi-interpolation weight
// is zero are not read; FMA contraction is allowed.  The results differ from
// the literal forms by a few ulp.
#pragma once
#include "qs_common.cuh"
#include "qs_internal.h"

namespace qs {
namespace specf32 {

template <class R> struct Pair2;
template <> struct Pair2<float> { using type = float2; };
template <> struct Pair2<double> { using type = double2; };
template <class R> using pair_t = typename Pair2<R>::type;

template <class R>
__device__ __forceinline__ pair_t<R> ld2(const R* p, size_t n) {
    return __ldg(reinterpret_cast<const pair_t<R>*>(p + n));
}
template <class R>
__device__ __forceinline__ void st2(R* p, size_t n, R a, R b) {
    pair_t<R> v;
    v.x = a;
    v.y = b;
    *reinterpret_cast<pair_t<R>*>(p + n) = v;
}

// beam terms of two modes; layers whose weight is zero are not read
template <class R>
struct BeamPair { R rb[2], rbp[2], jxb[2]; };

template <class R>
__device__ __forceinline__ BeamPair<R> beam_pair(const SpecArgs<R>& a, size_t n) {
    BeamPair<R> b;
    pair_t<R> r = ld2(a.Rb0, n), jx = ld2(a.Jxb0, n);
    b.rb[0] = a.wb0 * r.x; b.rb[1] = a.wb0 * r.y;
    b.jxb[0] = a.wb0 * jx.x; b.jxb[1] = a.wb0 * jx.y;
    if (a.wb1 != R(0)) {
        r = ld2(a.Rb1, n);
        jx = ld2(a.Jxb1, n);
        b.rb[0] += a.wb1 * r.x; b.rb[1] += a.wb1 * r.y;
        b.jxb[0] += a.wb1 * jx.x; b.jxb[1] += a.wb1 * jx.y;
    }
    b.rbp[0] = b.rbp[1] = R(0);
    if (a.wp0 != R(0)) {
        r = ld2(a.Rbp0, n);
        b.rbp[0] = a.wp0 * r.x; b.rbp[1] = a.wp0 * r.y;
    }
    if (a.wp1 != R(0)) {
        r = ld2(a.Rbp1, n);
        b.rbp[0] += a.wp1 * r.x; b.rbp[1] += a.wp1 * r.y;
    }
    return b;
}

// clear two modes of the 4 deposit planes the next push adds to
template <class R>
__device__ __forceinline__ void zero_src2(const SpecArgs<R>& a, size_t n) {
    if (a.zero_src) {
        const size_t N = (size_t)a.ny * a.nz;
#pragma unroll
        for (int q = 0; q < 4; q++) st2(a.zero_src + q * N, n, R(0), R(0));
    }
}

// outputs of the maps on two modes
template <class R>
struct Modes2 {
    R rho[2], ex[2], ey[2], ez[2], bx[2], by[2], bz[2];
};

// Guess (:843-872) on modes (j, k), (j+1, k); n = j + ny k
template <class R>
__device__ __forceinline__ Modes2<R> predictor_modes2(const SpecArgs<R>& a, int j, int k,
                                                      size_t n) {
    const R d = *a.dens_p, hx = a.hx;
    const R dh2 = d * hx * hx;
    const R inv_den = R(1) / (R(4) + dh2);
    const R propagator = (R(4) - dh2) * inv_den;
    const R c_rb = dh2 * inv_den;            // (rb + rbp) d hx^2 / denominator
    const R c_ex = R(4) * hx * inv_den;      // 4 Ex hx (k^2 + d) / denominator
    const R c_rho = R(2) * d * hx * inv_den; // 2 (2 rp + rb + rbp) d hx / ((k^2+d) den)
    const R akz = a.piZ * ((R)k + R(0.5));
    const pair_t<R> rp2 = ld2(a.RhoP, n), jxp2 = ld2(a.JxP, n), jyp2 = ld2(a.JyP, n),
                    jzp2 = ld2(a.JzP, n), exp2 = ld2(a.ExP, n), eyp2 = ld2(a.EyP, n),
                    ezp2 = ld2(a.EzP, n);
    const BeamPair<R> b = beam_pair(a, n);
    const R rp_[2] = {rp2.x, rp2.y}, jxp_[2] = {jxp2.x, jxp2.y}, jyp_[2] = {jyp2.x, jyp2.y},
            jzp_[2] = {jzp2.x, jzp2.y}, exp_[2] = {exp2.x, exp2.y},
            eyp_[2] = {eyp2.x, eyp2.y}, ezp_[2] = {ezp2.x, ezp2.y};
    Modes2<R> o;
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const R aky = a.piY * ((R)(j + q) + R(0.5));
        const R ak2 = aky * aky + akz * akz;
        const R inv_ak2 = R(1) / ak2;
        const R inv_dk = R(1) / (d + ak2);
        const R rp = rp_[q], rbs = b.rb[q] + b.rbp[q];
        o.rho[q] = propagator * rp - rbs * c_rb + c_ex * exp_[q] * (ak2 + d);
        o.ex[q] = propagator * exp_[q] - (R(2) * rp + rbs) * c_rho * inv_dk;
        const R srcE = (rbs + rp + o.rho[q]) * inv_dk;
        o.ey[q] = -eyp_[q] + aky * srcE;
        o.ez[q] = -ezp_[q] + akz * srcE;
        const R jy = jyp_[q] + R(0.5) * hx * d * (o.ey[q] + eyp_[q]);
        const R jz = jzp_[q] + R(0.5) * hx * d * (o.ez[q] + ezp_[q]);
        const R jx = jxp_[q] + R(0.5) * hx * d * (o.ex[q] + exp_[q]);
        o.bx[q] = (akz * jy - aky * jz) * inv_ak2;
        o.by[q] = (-akz * (jx + b.jxb[q]) + d * o.ez[q]) * inv_ak2;
        o.bz[q] = (aky * (jx + b.jxb[q]) - d * o.ey[q]) * inv_ak2;
    }
    return o;
}

// Iterate (:1419-1466) on modes (j, k), (j+1, k) with the C-deposit spectra
// jx2, jy2, jz2 of the two modes
template <class R>
__device__ __forceinline__ Modes2<R> corrector_modes2(const SpecArgs<R>& a, int j, int k,
                                                      size_t n, pair_t<R> jx2, pair_t<R> jy2,
                                                      pair_t<R> jz2) {
    const R d = *a.dens_p, hx = a.hx;
    const R akz = a.piZ * ((R)k + R(0.5));
    const pair_t<R> rp2 = ld2(a.RhoP, n), jxp2 = ld2(a.JxP, n), jyp2 = ld2(a.JyP, n),
                    jzp2 = ld2(a.JzP, n), eyp2 = ld2(a.EyP, n), ezp2 = ld2(a.EzP, n),
                    rold2 = ld2(a.Rho, n);
    const BeamPair<R> b = beam_pair(a, n);
    const R rp_[2] = {rp2.x, rp2.y}, jx_[2] = {jx2.x, jx2.y}, jy_[2] = {jy2.x, jy2.y},
            jz_[2] = {jz2.x, jz2.y}, jxp_[2] = {jxp2.x, jxp2.y}, jyp_[2] = {jyp2.x, jyp2.y},
            jzp_[2] = {jzp2.x, jzp2.y}, eyp_[2] = {eyp2.x, eyp2.y},
            ezp_[2] = {ezp2.x, ezp2.y}, rold_[2] = {rold2.x, rold2.y};
    Modes2<R> o;
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const R aky = a.piY * ((R)(j + q) + R(0.5));
        const R ak2 = aky * aky + akz * akz;
        const R inv_ak2 = R(1) / ak2;
        const R inv_dk = R(1) / (d + ak2);
        const R jx = jx_[q], jy = jy_[q], jz = jz_[q];
        o.rho[q] = rp_[q] + jx - jxp_[q] - R(0.5) * hx * (aky * (jy + jyp_[q]) + akz * (jz + jzp_[q]));
        o.ex[q] = -(aky * jy + akz * jz) * inv_ak2;
        const R srcE = (b.rb[q] + b.rbp[q] + rp_[q] + rold_[q]) * inv_dk;
        o.ey[q] = -eyp_[q] + aky * srcE;
        o.ez[q] = -ezp_[q] + akz * srcE;
        o.bx[q] = (akz * jy - aky * jz) * inv_ak2;
        o.by[q] = (-akz * (jx + b.jxb[q]) + d * o.ez[q]) * inv_ak2;
        o.bz[q] = (aky * (jx + b.jxb[q]) - d * o.ey[q]) * inv_ak2;
    }
    return o;
}

// Rho, Ex, Ey, Ez (and B when kept) into the spectral bank, and the two modes
// of the next push's deposit planes cleared
template <class R>
__device__ __forceinline__ void store_modes2(const SpecArgs<R>& a, size_t n, const Modes2<R>& o) {
    st2(a.Rho, n, o.rho[0], o.rho[1]);
    st2(a.Ex, n, o.ex[0], o.ex[1]);
    st2(a.Ey, n, o.ey[0], o.ey[1]);
    st2(a.Ez, n, o.ez[0], o.ez[1]);
    zero_src2(a, n);
    if (a.write_b) {
        st2(a.Bx, n, o.bx[0], o.bx[1]);
        st2(a.By, n, o.by[0], o.by[1]);
        st2(a.Bz, n, o.bz[0], o.bz[1]);
    }
}

}  // namespace specf32
}  // namespace qs
