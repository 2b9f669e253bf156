// charge.cuh — FP64 global charge sums of every layer.
//
// Per layer, the sums over the transverse plane of the corrected density
// (f_Dens after the layer's last Iterate, movefieldshydrolinlayersplit.cpp:
// 1545-1602), of the Jx deposit of its full push, and of the beam's RhoBeam.
// They are accumulated in FP64 whatever the precision of the march.
//
// The plasma sums come from the spectra inside the last corrector of a
// layer: a plane x is the inverse REDFT11 x REDFT11 transform of its
// spectrum X divided by 4 ny nz, and
//   sum_{n=0}^{N-1} 2 cos(pi (n + 1/2)(k + 1/2) / N) = (-1)^k / sin(pi (2k+1) / (4N)),
// so sum_n x(n) = (1 / (4 ny nz)) sum_k X(k) c_ky(ny) c_kz(nz) with
// c_k(N) = (-1)^k / sin(pi (2k+1) / (4N)).  Each block writes its partial sums
// (a fixed order inside the block) and a last kernel adds the partials of a
// layer in index order, so the sums are the same from run to run.
#pragma once
#include "qs_common.cuh"

namespace qs {

// Sum (r, j) over the block; thread 0 writes out[0] = sum r, out[1] = sum j.
// Every thread of the block must call it.
__device__ __forceinline__ void charge_block_sum(double r, double j, double* out) {
    const unsigned full = 0xffffffffu;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        r += __shfl_down_sync(full, r, o);
        j += __shfl_down_sync(full, j, o);
    }
    __shared__ double sh_charge[2][32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int nw = (blockDim.x + 31) >> 5;
    if (l == 0) {
        sh_charge[0][w] = r;
        sh_charge[1][w] = j;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int i = 0; i < nw; i++) {
            a += sh_charge[0][i];
            b += sh_charge[1][i];
        }
        out[0] = a;
        out[1] = b;
    }
}

}  // namespace qs
