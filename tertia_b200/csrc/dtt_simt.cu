// dtt_simt.cu — half-integer DCT-IV / DST-IV transforms as batched dense
// GEMMs on the CUDA cores, exact FP32 or FP64.
//
// Replaces the reference's FFTW REDFT11/RODFT11 plans
// (movefieldshydrolinlayersplit.cpp:389-427) and the dead cuFFT twin
// CUDA_WRAP_fourierHalfInteger2D (half_integer2D.cu:583).  The design is the
// reference's own dense-matrix attempt (surfaceFFT.cu:108-164) scaled up:
// Y = A_z X A_y, computed as two passes of out = (in . A)^T so each pass
// reads its operand row-major and the transpose lands in the epilogue.
// This is the plain FP64 path and the exact-FP32 path; the split-precision
// tensor-core path is dtt_tc.cu.
#include "qs_common.cuh"
#include "qs_internal.h"

namespace qs {

template <class T, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__(256) dtt_pass_simt(DttPassArgs<T> a) {
    static_assert((BM / TM) * (BN / TN) == 256, "256 threads");
    constexpr int TX = BM / TM;   // threads along M
    __shared__ __align__(16) T As[2][BK][BM];
    __shared__ __align__(16) T Bs[2][BK][BN];
    const int f = blockIdx.z;
    const T* __restrict__ A = a.in[f];
    const T* __restrict__ B = a.mat[f];
    T* __restrict__ O = a.out[f];
    const int R = a.R, K = a.K;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;

    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++) acc[i][j] = T(0);

    // global -> smem loaders: A tile BM x BK (rows of in), B tile BK x BN
    constexpr int A_ELEMS = BM * BK / 256;
    constexpr int B_ELEMS = BK * BN / 256;
    T ra[A_ELEMS], rb[B_ELEMS];
    auto load_tiles = [&](int k0) {
#pragma unroll
        for (int e = 0; e < A_ELEMS; e++) {
            int idx = tid * A_ELEMS + e;       // row-major over (BM, BK)
            int mm = idx / BK, kk = idx % BK;
            int gm = m0 + mm, gk = k0 + kk;
            ra[e] = (gm < R && gk < K) ? A[(size_t)gm * K + gk] : T(0);
        }
#pragma unroll
        for (int e = 0; e < B_ELEMS; e++) {
            int idx = tid * B_ELEMS + e;       // row-major over (BK, BN)
            int kk = idx / BN, nn = idx % BN;
            int gk = k0 + kk, gn = n0 + nn;
            rb[e] = (gk < K && gn < K) ? B[(size_t)gk * K + gn] : T(0);
        }
    };
    auto store_tiles = [&](int buf) {
#pragma unroll
        for (int e = 0; e < A_ELEMS; e++) {
            int idx = tid * A_ELEMS + e;
            As[buf][idx % BK][idx / BK] = ra[e];
        }
#pragma unroll
        for (int e = 0; e < B_ELEMS; e++) {
            int idx = tid * B_ELEMS + e;
            Bs[buf][idx / BN][idx % BN] = rb[e];
        }
    };

    const int nk = (K + BK - 1) / BK;
    load_tiles(0);
    store_tiles(0);
    __syncthreads();
    for (int kt = 0; kt < nk; kt++) {
        const int buf = kt & 1;
        if (kt + 1 < nk) load_tiles((kt + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            T av[TM], bv[TN];
#pragma unroll
            for (int i = 0; i < TM; i++) av[i] = As[buf][kk][tx * TM + i];
#pragma unroll
            for (int j = 0; j < TN; j++) bv[j] = Bs[buf][kk][ty * TN + j];
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int j = 0; j < TN; j++) acc[i][j] += av[i] * bv[j];
        }
        if (kt + 1 < nk) store_tiles(buf ^ 1);
        __syncthreads();
    }
    // epilogue: out[n][m] (transposed), consecutive threads cover consecutive m
    const T s = a.scale;
#pragma unroll
    for (int j = 0; j < TN; j++) {
        int gn = n0 + ty * TN + j;
        if (gn >= K) continue;
#pragma unroll
        for (int i = 0; i < TM; i++) {
            int gm = m0 + tx * TM + i;
            if (gm < R) O[(size_t)gn * R + gm] = acc[i][j] * s;
        }
    }
}

template <class T>
static void launch_pass(const DttPassArgs<T>& a, int nf, cudaStream_t st);

template <>
void launch_pass<float>(const DttPassArgs<float>& a, int nf, cudaStream_t st) {
    dim3 grid((a.R + 127) / 128, (a.K + 127) / 128, nf);
    dtt_pass_simt<float, 128, 128, 8, 8, 8><<<grid, 256, 0, st>>>(a);
}

template <>
void launch_pass<double>(const DttPassArgs<double>& a, int nf, cudaStream_t st) {
    dim3 grid((a.R + 63) / 64, (a.K + 63) / 64, nf);
    dtt_pass_simt<double, 64, 64, 8, 4, 4><<<grid, 256, 0, st>>>(a);
}

template <class T>
int run_dtt_simt_pass(int pass, const DttJob<T>& job, int ny, int nz, const DttMats<T>& my,
                      const DttMats<T>& mz, T* scratch, cudaStream_t st) {
    if (job.nf <= 0) return 0;
    const size_t plane = (size_t)ny * nz;
    DttPassArgs<T> a{};
    for (int f = 0; f < job.nf; f++) {
        if (pass == 0) {
            a.in[f] = job.in[f];
            a.mat[f] = my.m[job.ky[f]];
            a.out[f] = scratch + f * plane;
        } else {
            a.in[f] = scratch + f * plane;
            a.mat[f] = mz.m[job.kz[f]];
            a.out[f] = job.out[f];
        }
    }
    if (pass == 0) { a.R = nz; a.K = ny; a.scale = T(1); }
    else { a.R = ny; a.K = nz; a.scale = job.scale; }
    launch_pass<T>(a, job.nf, st);
    return 1;
}

template <class T>
int run_dtt_simt(const DttJob<T>& job, int ny, int nz, const DttMats<T>& my,
                 const DttMats<T>& mz, T* scratch, cudaStream_t st) {
    return run_dtt_simt_pass<T>(0, job, ny, nz, my, mz, scratch, st) +
           run_dtt_simt_pass<T>(1, job, ny, nz, my, mz, scratch, st);
}

template int run_dtt_simt_pass<float>(int, const DttJob<float>&, int, int, const DttMats<float>&,
                                      const DttMats<float>&, float*, cudaStream_t);
template int run_dtt_simt_pass<double>(int, const DttJob<double>&, int, int,
                                       const DttMats<double>&, const DttMats<double>&, double*,
                                       cudaStream_t);
template int run_dtt_simt<float>(const DttJob<float>&, int, int, const DttMats<float>&,
                                 const DttMats<float>&, float*, cudaStream_t);
template int run_dtt_simt<double>(const DttJob<double>&, int, int, const DttMats<double>&,
                                  const DttMats<double>&, double*, cudaStream_t);

}  // namespace qs
