// split.cuh — splitting an FP32 value into low-precision terms for the
// split-precision tensor-core transforms: v ~ t0 + t1 (+ t2) with each term
// rounded to BF16 (KIND 0) or TF32 (KIND 1) and the next term taken from the
// FP32 remainder.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace qs {

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

template <int KIND>
__device__ __forceinline__ void split_value(float v, int n, float (&t)[3]) {
    float r = v;
#pragma unroll
    for (int s = 0; s < 3; s++) {
        if (s < n) {
            const float h = (KIND == 0) ? __bfloat162float(__float2bfloat16_rn(r)) : tf32_rna(r);
            t[s] = h;
            r = __fsub_rn(r, h);
        } else {
            t[s] = 0.f;
        }
    }
}

// store the nsplit terms of v at element `idx` of term planes `tstride` apart
template <int KIND>
__device__ __forceinline__ void store_split(void* base, size_t tstride, size_t idx, float v,
                                            int nsplit) {
    float t[3];
    split_value<KIND>(v, nsplit, t);
    if (KIND == 0) {
        __nv_bfloat16* o = (__nv_bfloat16*)base;
        for (int s = 0; s < nsplit; s++) o[(size_t)s * tstride + idx] = __float2bfloat16_rn(t[s]);
    } else {
        float* o = (float*)base;
        for (int s = 0; s < nsplit; s++) o[(size_t)s * tstride + idx] = t[s];
    }
}

}  // namespace qs
