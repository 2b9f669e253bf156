// spectral_f32.cu — kernels of the FP32 per-mode predictor / corrector maps
// (spectral_f32.cuh holds the per-mode algebra): two adjacent modes per
// thread (float2 loads and stores; the split operand of the tensor-core
// transforms is stored as bf16x2 / float2), a 2-D grid (blockIdx.y = z-mode
// row), so no integer division.
#include <cuda_bf16.h>

#include "qs_common.cuh"
#include "qs_internal.h"
#include "split.cuh"
#include "pdl.cuh"
#include "spectral_f32.cuh"
#include "charge.cuh"

namespace qs {
namespace {

using namespace specf32;

constexpr int kThreads = 128;   // threads per block; 2 modes each

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
    const Modes2<float> o = predictor_modes2(a, j, k, n);
    pdl_trigger();
    store_modes2(a, n, o);
    put_split2<KIND, NSPLIT>(a, 0, n, o.ex[0], o.ex[1]);
    put_split2<KIND, NSPLIT>(a, 1, n, o.ey[0], o.ey[1]);
    put_split2<KIND, NSPLIT>(a, 2, n, o.ez[0], o.ez[1]);
    put_split2<KIND, NSPLIT>(a, 3, n, o.bx[0], o.bx[1]);
    put_split2<KIND, NSPLIT>(a, 4, n, o.by[0], o.by[1]);
    put_split2<KIND, NSPLIT>(a, 5, n, o.bz[0], o.bz[1]);
}

template <int KIND, int NSPLIT>
__global__ void __launch_bounds__(kThreads) corrector_f32_kernel(SpecArgs<float> a) {
    const int j = 2 * (blockIdx.x * kThreads + threadIdx.x);
    const int k = blockIdx.y;
    double qr = 0.0, qj = 0.0;
    pdl_wait();
    if (j < a.ny) {
        const size_t n = (size_t)j + (size_t)a.ny * k;
        const float2 jx2 = ld2(a.Jx, n);
        const Modes2<float> o = corrector_modes2(a, j, k, n, jx2, ld2(a.Jy, n), ld2(a.Jz, n));
        pdl_trigger();
        store_modes2(a, n, o);
        put_split2<KIND, NSPLIT>(a, 0, n, o.ex[0], o.ex[1]);
        put_split2<KIND, NSPLIT>(a, 1, n, o.ey[0], o.ey[1]);
        put_split2<KIND, NSPLIT>(a, 2, n, o.ez[0], o.ez[1]);
        put_split2<KIND, NSPLIT>(a, 3, n, o.bx[0], o.bx[1]);
        put_split2<KIND, NSPLIT>(a, 4, n, o.by[0], o.by[1]);
        put_split2<KIND, NSPLIT>(a, 5, n, o.bz[0], o.bz[1]);
        if (NSPLIT > 0 && a.split_rho) put_split2<KIND, NSPLIT>(a, 6, n, o.rho[0], o.rho[1]);
        if (a.qsum) {
            const double cz = a.qcz[k], c0 = a.qcy[j] * cz, c1 = a.qcy[j + 1] * cz;
            qr = (double)o.rho[0] * c0 + (double)o.rho[1] * c1;
            qj = (double)jx2.x * c0 + (double)jx2.y * c1;
        }
    }
    if (a.qsum)
        charge_block_sum(qr, qj, a.qsum + 2 * ((size_t)blockIdx.y * gridDim.x + blockIdx.x));
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
