// spectral_f32.cu — FP32 fast forms of the per-mode predictor / corrector maps
// (GuessFieldsHydroLinLayerSplit, movefieldshydrolinlayersplit.cpp:808-900;
// IterateFieldsHydroLinLayerSplit, :1374-1477).
//
// Same algebra as predictor_kernel / corrector_kernel in spectral.cu, arranged
// for the GPU rather than for bit-exact agreement with the oracle:
//   * two adjacent modes per thread (float2 loads and stores; the split
//     operand of the tensor-core transforms is stored as bf16x2 / float2),
//   * a 2-D grid (blockIdx.y = z-mode row), so no integer division,
//   * the five divisions of a mode become two reciprocals, 1/k^2 and
//     1/(k^2 + density), plus uniform constants,
//   * beam-spectrum terms whose xi-interpolation weight is zero are not read
//     (the second layer when NxSplit = 1, the previous-layer beam at the head),
//   * FMA contraction allowed (this file is not built with -fmad=false).
// The results differ from the literal forms by a few FP32 ulp.
#include <cuda_bf16.h>

#include "qs_common.cuh"
#include "qs_internal.h"
#include "split.cuh"
#include "pdl.cuh"

namespace qs {
namespace {

constexpr int kThreads = 128;   // threads per block; 2 modes each

__device__ __forceinline__ float2 ld2(const float* p, size_t n) {
    return __ldg(reinterpret_cast<const float2*>(p + n));
}
__device__ __forceinline__ void st2(float* p, size_t n, float a, float b) {
    *reinterpret_cast<float2*>(p + n) = make_float2(a, b);
}

// beam terms of two modes; layers whose weight is zero are not read
struct BeamPair { float rb[2], rbp[2], jxb[2]; };

__device__ __forceinline__ BeamPair beam_pair(const SpecArgs<float>& a, size_t n) {
    BeamPair b;
    float2 r = ld2(a.Rb0, n), jx = ld2(a.Jxb0, n);
    b.rb[0] = a.wb0 * r.x; b.rb[1] = a.wb0 * r.y;
    b.jxb[0] = a.wb0 * jx.x; b.jxb[1] = a.wb0 * jx.y;
    if (a.wb1 != 0.f) {
        r = ld2(a.Rb1, n);
        jx = ld2(a.Jxb1, n);
        b.rb[0] += a.wb1 * r.x; b.rb[1] += a.wb1 * r.y;
        b.jxb[0] += a.wb1 * jx.x; b.jxb[1] += a.wb1 * jx.y;
    }
    b.rbp[0] = b.rbp[1] = 0.f;
    if (a.wp0 != 0.f) {
        r = ld2(a.Rbp0, n);
        b.rbp[0] = a.wp0 * r.x; b.rbp[1] = a.wp0 * r.y;
    }
    if (a.wp1 != 0.f) {
        r = ld2(a.Rbp1, n);
        b.rbp[0] += a.wp1 * r.x; b.rbp[1] += a.wp1 * r.y;
    }
    return b;
}

// clear two modes of the 4 deposit planes the next push adds to
__device__ __forceinline__ void zero_src2(const SpecArgs<float>& a, size_t n) {
    if (a.zero_src) {
        const size_t N = (size_t)a.ny * a.nz;
#pragma unroll
        for (int q = 0; q < 4; q++) st2(a.zero_src + q * N, n, 0.f, 0.f);
    }
}

// split terms of two adjacent values into NSPLIT term planes (KIND 0: bf16,
// KIND 1: tf32 in float storage); idx is even
template <int KIND, int NSPLIT>
__device__ __forceinline__ void put_split2(const SpecArgs<float>& a, int slot, size_t n, float v0,
                                           float v1) {
    if constexpr (NSPLIT > 0) {
        const size_t idx = (size_t)slot * a.ny * a.nz + n;
        float t0[3], t1[3];
        split_value<KIND>(v0, NSPLIT, t0);
        split_value<KIND>(v1, NSPLIT, t1);
#pragma unroll
        for (int s = 0; s < NSPLIT; s++) {
            if constexpr (KIND == 0) {
                __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(
                    (__nv_bfloat16*)a.split + (size_t)s * a.tstride + idx);
                *o = __floats2bfloat162_rn(t0[s], t1[s]);   // exact: terms are bf16 values
            } else {
                st2((float*)a.split + (size_t)s * a.tstride, idx, t0[s], t1[s]);
            }
        }
    }
}

template <int KIND, int NSPLIT>
__global__ void __launch_bounds__(kThreads) predictor_f32_kernel(SpecArgs<float> a) {
    const int j = 2 * (blockIdx.x * kThreads + threadIdx.x);
    const int k = blockIdx.y;
    if (j >= a.ny) return;
    pdl_wait();
    const size_t n = (size_t)j + (size_t)a.ny * k;
    const float d = *a.dens_p, hx = a.hx;
    const float dh2 = d * hx * hx;
    const float inv_den = 1.f / (4.f + dh2);
    const float propagator = (4.f - dh2) * inv_den;
    const float c_rb = dh2 * inv_den;            // (rb + rbp) d hx^2 / denominator
    const float c_ex = 4.f * hx * inv_den;       // 4 Ex hx (k^2 + d) / denominator
    const float c_rho = 2.f * d * hx * inv_den;  // 2 (2 rp + rb + rbp) d hx / ((k^2+d) den)
    const float akz = a.piZ * ((float)k + 0.5f);
    const float2 rp2 = ld2(a.RhoP, n), jxp2 = ld2(a.JxP, n), jyp2 = ld2(a.JyP, n),
                 jzp2 = ld2(a.JzP, n), exp2 = ld2(a.ExP, n), eyp2 = ld2(a.EyP, n),
                 ezp2 = ld2(a.EzP, n);
    const BeamPair b = beam_pair(a, n);
    pdl_trigger();
    const float rp_[2] = {rp2.x, rp2.y}, jxp_[2] = {jxp2.x, jxp2.y}, jyp_[2] = {jyp2.x, jyp2.y},
                jzp_[2] = {jzp2.x, jzp2.y}, exp_[2] = {exp2.x, exp2.y},
                eyp_[2] = {eyp2.x, eyp2.y}, ezp_[2] = {ezp2.x, ezp2.y};
    float rho[2], ex[2], ey[2], ez[2], bx[2], by[2], bz[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const float aky = a.piY * ((float)(j + q) + 0.5f);
        const float ak2 = aky * aky + akz * akz;
        const float inv_ak2 = 1.f / ak2;
        const float inv_dk = 1.f / (d + ak2);
        const float rp = rp_[q], rbs = b.rb[q] + b.rbp[q];
        rho[q] = propagator * rp - rbs * c_rb + c_ex * exp_[q] * (ak2 + d);
        ex[q] = propagator * exp_[q] - (2.f * rp + rbs) * c_rho * inv_dk;
        const float srcE = (rbs + rp + rho[q]) * inv_dk;
        ey[q] = -eyp_[q] + aky * srcE;
        ez[q] = -ezp_[q] + akz * srcE;
        const float jy = jyp_[q] + 0.5f * hx * d * (ey[q] + eyp_[q]);
        const float jz = jzp_[q] + 0.5f * hx * d * (ez[q] + ezp_[q]);
        const float jx = jxp_[q] + 0.5f * hx * d * (ex[q] + exp_[q]);
        bx[q] = (akz * jy - aky * jz) * inv_ak2;
        by[q] = (-akz * (jx + b.jxb[q]) + d * ez[q]) * inv_ak2;
        bz[q] = (aky * (jx + b.jxb[q]) - d * ey[q]) * inv_ak2;
    }
    st2(a.Rho, n, rho[0], rho[1]);
    st2(a.Ex, n, ex[0], ex[1]);
    st2(a.Ey, n, ey[0], ey[1]);
    st2(a.Ez, n, ez[0], ez[1]);
    zero_src2(a, n);
    if (a.write_b) {
        st2(a.Bx, n, bx[0], bx[1]);
        st2(a.By, n, by[0], by[1]);
        st2(a.Bz, n, bz[0], bz[1]);
    }
    put_split2<KIND, NSPLIT>(a, 0, n, ex[0], ex[1]);
    put_split2<KIND, NSPLIT>(a, 1, n, ey[0], ey[1]);
    put_split2<KIND, NSPLIT>(a, 2, n, ez[0], ez[1]);
    put_split2<KIND, NSPLIT>(a, 3, n, bx[0], bx[1]);
    put_split2<KIND, NSPLIT>(a, 4, n, by[0], by[1]);
    put_split2<KIND, NSPLIT>(a, 5, n, bz[0], bz[1]);
}

template <int KIND, int NSPLIT>
__global__ void __launch_bounds__(kThreads) corrector_f32_kernel(SpecArgs<float> a) {
    const int j = 2 * (blockIdx.x * kThreads + threadIdx.x);
    const int k = blockIdx.y;
    if (j >= a.ny) return;
    pdl_wait();
    const size_t n = (size_t)j + (size_t)a.ny * k;
    const float d = *a.dens_p, hx = a.hx;
    const float akz = a.piZ * ((float)k + 0.5f);
    const float2 rp2 = ld2(a.RhoP, n), jx2 = ld2(a.Jx, n), jy2 = ld2(a.Jy, n), jz2 = ld2(a.Jz, n),
                 jxp2 = ld2(a.JxP, n), jyp2 = ld2(a.JyP, n), jzp2 = ld2(a.JzP, n),
                 eyp2 = ld2(a.EyP, n), ezp2 = ld2(a.EzP, n), rold2 = ld2(a.Rho, n);
    const BeamPair b = beam_pair(a, n);
    pdl_trigger();
    const float rp_[2] = {rp2.x, rp2.y}, jx_[2] = {jx2.x, jx2.y}, jy_[2] = {jy2.x, jy2.y},
                jz_[2] = {jz2.x, jz2.y}, jxp_[2] = {jxp2.x, jxp2.y}, jyp_[2] = {jyp2.x, jyp2.y},
                jzp_[2] = {jzp2.x, jzp2.y}, eyp_[2] = {eyp2.x, eyp2.y},
                ezp_[2] = {ezp2.x, ezp2.y}, rold_[2] = {rold2.x, rold2.y};
    float rho[2], ex[2], ey[2], ez[2], bx[2], by[2], bz[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const float aky = a.piY * ((float)(j + q) + 0.5f);
        const float ak2 = aky * aky + akz * akz;
        const float inv_ak2 = 1.f / ak2;
        const float inv_dk = 1.f / (d + ak2);
        const float jx = jx_[q], jy = jy_[q], jz = jz_[q];
        rho[q] = rp_[q] + jx - jxp_[q] - 0.5f * hx * (aky * (jy + jyp_[q]) + akz * (jz + jzp_[q]));
        ex[q] = -(aky * jy + akz * jz) * inv_ak2;
        const float srcE = (b.rb[q] + b.rbp[q] + rp_[q] + rold_[q]) * inv_dk;
        ey[q] = -eyp_[q] + aky * srcE;
        ez[q] = -ezp_[q] + akz * srcE;
        bx[q] = (akz * jy - aky * jz) * inv_ak2;
        by[q] = (-akz * (jx + b.jxb[q]) + d * ez[q]) * inv_ak2;
        bz[q] = (aky * (jx + b.jxb[q]) - d * ey[q]) * inv_ak2;
    }
    st2(a.Ey, n, ey[0], ey[1]);
    st2(a.Ez, n, ez[0], ez[1]);
    st2(a.Rho, n, rho[0], rho[1]);
    st2(a.Ex, n, ex[0], ex[1]);
    zero_src2(a, n);
    if (a.write_b) {
        st2(a.Bx, n, bx[0], bx[1]);
        st2(a.By, n, by[0], by[1]);
        st2(a.Bz, n, bz[0], bz[1]);
    }
    put_split2<KIND, NSPLIT>(a, 0, n, ex[0], ex[1]);
    put_split2<KIND, NSPLIT>(a, 1, n, ey[0], ey[1]);
    put_split2<KIND, NSPLIT>(a, 2, n, ez[0], ez[1]);
    put_split2<KIND, NSPLIT>(a, 3, n, bx[0], bx[1]);
    put_split2<KIND, NSPLIT>(a, 4, n, by[0], by[1]);
    put_split2<KIND, NSPLIT>(a, 5, n, bz[0], bz[1]);
    if (NSPLIT > 0 && a.split_rho) put_split2<KIND, NSPLIT>(a, 6, n, rho[0], rho[1]);
}

// (kind, nsplit) of the operand; -1 when there is none or it is not handled
int split_case(const SpecArgs<float>& a) {
    if (!a.split) return 0;
    if (a.tstride % 2) return -1;
    if (a.split_kind == 0 && a.nsplit == 2) return 1;
    if (a.split_kind == 1 && a.nsplit == 2) return 2;
    if (a.split_kind == 0 && a.nsplit == 3) return 3;
    return -1;
}

}  // namespace

int launch_predictor_fast(const SpecArgs<float>& a, cudaStream_t st) {
    const int c = split_case(a);
    if (a.ny % 2 || c < 0) return 0;
    const dim3 g((unsigned)((a.ny / 2 + kThreads - 1) / kThreads), (unsigned)a.nz);
    switch (c) {
        case 0: launch_pdl(predictor_f32_kernel<0, 0>, g, dim3(kThreads), 0, st, a); break;
        case 1: launch_pdl(predictor_f32_kernel<0, 2>, g, dim3(kThreads), 0, st, a); break;
        case 2: launch_pdl(predictor_f32_kernel<1, 2>, g, dim3(kThreads), 0, st, a); break;
        default: launch_pdl(predictor_f32_kernel<0, 3>, g, dim3(kThreads), 0, st, a); break;
    }
    return 1;
}

int launch_corrector_fast(const SpecArgs<float>& a, cudaStream_t st) {
    const int c = split_case(a);
    if (a.ny % 2 || c < 0) return 0;
    const dim3 g((unsigned)((a.ny / 2 + kThreads - 1) / kThreads), (unsigned)a.nz);
    switch (c) {
        case 0: launch_pdl(corrector_f32_kernel<0, 0>, g, dim3(kThreads), 0, st, a); break;
        case 1: launch_pdl(corrector_f32_kernel<0, 2>, g, dim3(kThreads), 0, st, a); break;
        case 2: launch_pdl(corrector_f32_kernel<1, 2>, g, dim3(kThreads), 0, st, a); break;
        default: launch_pdl(corrector_f32_kernel<0, 3>, g, dim3(kThreads), 0, st, a); break;
    }
    return 1;
}

}  // namespace qs
