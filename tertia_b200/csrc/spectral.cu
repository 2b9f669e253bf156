// spectral.cu — per-mode maps of the half-integer spectral field solve and
// the small per-layer kernels around them.
//
// Predictor: GuessFieldsHydroLinLayerSplit's linearised step
// (movefieldshydrolinlayersplit.cpp:808-900; dead GPU twin
// linearized_kernel, linearized.cu:11-103).  Corrector:
// IterateFieldsHydroLinLayerSplit (:1374-1477; twin
// linearizedIteratekernel, linearized.cu:105-209).  The expression order is
// the reference's and the file is compiled with -fmad=false.
//
// The P-layer spectra (RhoP, E*P, J*P) are the previous layer's final
// spectra carried in HBM: the reference recomputes them by transforming the
// P layer's real planes (:569-623, :717-743), which are the inverse
// transforms of exactly those spectra, so the forward-of-inverse is skipped.
#include <cmath>

#include "qs_common.cuh"
#include "qs_internal.h"
#include "split.cuh"
#include "density.cuh"
#include "charge.cuh"

namespace qs {

template <class T>
__device__ __forceinline__ void put_split(const SpecArgs<T>& a, int slot, int n1, T v) {
    const size_t idx = (size_t)slot * a.ny * a.nz + n1;
    if (a.split_kind == 0) store_split<0>(a.split, a.tstride, idx, (float)v, a.nsplit);
    else store_split<1>(a.split, a.tstride, idx, (float)v, a.nsplit);
}

template <class T>
__device__ __forceinline__ void beam_terms(const SpecArgs<T>& a, int n1, T& rb, T& rbp, T& jxb) {
    rb = a.wb0 * a.Rb0[n1] + a.wb1 * a.Rb1[n1];
    jxb = a.wb0 * a.Jxb0[n1] + a.wb1 * a.Jxb1[n1];
    rbp = a.wp0 * a.Rbp0[n1] + a.wp1 * a.Rbp1[n1];
}

template <class T>
__global__ void predictor_kernel(SpecArgs<T> a) {
    const int n1 = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = a.ny * a.nz;
    if (n1 >= N) return;
    const int j = n1 % a.ny, k = n1 / a.ny;
    const T d = *a.dens_p, hx = a.hx;
    const T akz = a.piZ * (T(k) + T(0.5));
    const T aky = a.piY * (T(j) + T(0.5));
    const T ak2 = aky * aky + akz * akz;
    const T rp = a.RhoP[n1];
    const T jxp = a.JxP[n1], jyp = a.JyP[n1], jzp = a.JzP[n1];
    const T exp_ = a.ExP[n1], eyp = a.EyP[n1], ezp = a.EzP[n1];
    T rb, rbp, jxb;
    beam_terms(a, n1, rb, rbp, jxb);
    const T propagator = (T(4) - d * hx * hx) / (T(4) + d * hx * hx);
    const T denominator = T(4) + d * hx * hx;
    const T rho = propagator * rp - (rb + rbp) * d * hx * hx / denominator +
                  T(4) * exp_ * hx * (ak2 + d) / denominator;
    const T ex = propagator * exp_ - T(2) * (T(2) * rp + rb + rbp) * d * hx / ((ak2 + d) * denominator);
    const T ey = -eyp + aky * (rb + rbp + rp + rho) / (d + ak2);
    const T ez = -ezp + akz * (rb + rbp + rp + rho) / (d + ak2);
    const T jy = jyp + hx * d * (ey + eyp) / T(2);
    const T jz = jzp + hx * d * (ez + ezp) / T(2);
    const T jx = jxp + hx * d * (ex + exp_) / T(2);
    const T bx = -aky / ak2 * jz + akz / ak2 * jy;
    const T by = (-akz * (jx + jxb) + d * ez) / ak2;
    const T bz = (aky * (jx + jxb) - d * ey) / ak2;
    a.Rho[n1] = rho;
    a.Ex[n1] = ex;
    a.Ey[n1] = ey;
    a.Ez[n1] = ez;
    if (a.zero_src)
        for (int q = 0; q < 4; q++) a.zero_src[(size_t)q * N + n1] = T(0);
    if (a.write_b) {
        a.Bx[n1] = bx;
        a.By[n1] = by;
        a.Bz[n1] = bz;
    }
    if (a.split) {
        put_split(a, 0, n1, ex);
        put_split(a, 1, n1, ey);
        put_split(a, 2, n1, ez);
        put_split(a, 3, n1, bx);
        put_split(a, 4, n1, by);
        put_split(a, 5, n1, bz);
    }
}

template <class T>
__device__ __forceinline__ void corrector_mode(const SpecArgs<T>& a, int n1, double& qr,
                                               double& qj);

template <class T>
__global__ void corrector_kernel(SpecArgs<T> a) {
    const int n1 = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = a.ny * a.nz;
    double qr = 0.0, qj = 0.0;
    if (n1 < N) corrector_mode(a, n1, qr, qj);
    if (a.qsum) charge_block_sum(qr, qj, a.qsum + 2 * (size_t)blockIdx.x);
}

template <class T>
__device__ __forceinline__ void corrector_mode(const SpecArgs<T>& a, int n1, double& qr,
                                               double& qj) {
    const int N = a.ny * a.nz;
    const int j = n1 % a.ny, k = n1 / a.ny;
    const T d = *a.dens_p, hx = a.hx;
    const T akz = a.piZ * (T(k) + T(0.5));
    const T aky = a.piY * (T(j) + T(0.5));
    const T ak2 = aky * aky + akz * akz;
    const T rp = a.RhoP[n1];
    const T jx = a.Jx[n1], jy = a.Jy[n1], jz = a.Jz[n1];
    const T rho = rp + jx - a.JxP[n1] - hx * (aky * (jy + a.JyP[n1]) + akz * (jz + a.JzP[n1])) / T(2);
    T rb, rbp, jxb;
    beam_terms(a, n1, rb, rbp, jxb);
    const T eyp = a.EyP[n1], ezp = a.EzP[n1];
    const T rho_old = a.Rho[n1];
    const T newEx = -(aky * jy + akz * jz) / ak2;
    const T newEy = -eyp + aky * (rb + rbp + rp + rho_old) / (d + ak2);
    const T newEz = -ezp + akz * (rb + rbp + rp + rho_old) / (d + ak2);
    const T bx = -aky / ak2 * jz + akz / ak2 * jy;
    const T by = (-akz * (jx + jxb) + d * newEz) / ak2;
    const T bz = (aky * (jx + jxb) - d * newEy) / ak2;
    a.Ey[n1] = newEy;
    a.Ez[n1] = newEz;
    a.Rho[n1] = rho;
    a.Ex[n1] = newEx;
    if (a.qsum) {
        const double c = a.qcy[j] * a.qcz[k];
        qr = (double)rho * c;
        qj = (double)jx * c;
    }
    if (a.zero_src)
        for (int q = 0; q < 4; q++) a.zero_src[(size_t)q * N + n1] = T(0);
    if (a.write_b) {
        a.Bx[n1] = bx;
        a.By[n1] = by;
        a.Bz[n1] = bz;
    }
    if (a.split) {
        put_split(a, 0, n1, newEx);
        put_split(a, 1, n1, newEy);
        put_split(a, 2, n1, newEz);
        put_split(a, 3, n1, bx);
        put_split(a, 4, n1, by);
        put_split(a, 5, n1, bz);
        if (a.split_rho) put_split(a, 6, n1, rho);
    }
}

template <class T>
int launch_predictor(const SpecArgs<T>& a, cudaStream_t st) {
    if constexpr (sizeof(T) == 4) {
        if (launch_predictor_fast(a, st)) return 1;
    }
    const int N = a.ny * a.nz;
    predictor_kernel<T><<<(N + 255) / 256, 256, 0, st>>>(a);
    return 1;
}
template <class T>
int launch_corrector(const SpecArgs<T>& a, cudaStream_t st) {
    if constexpr (sizeof(T) == 4) {
        if (launch_corrector_fast(a, st)) return 1;
    }
    const int N = a.ny * a.nz;
    corrector_kernel<T><<<(N + 255) / 256, 256, 0, st>>>(a);
    return 1;
}

// out[0] = RhoBeam, out[1] = JxBeam of the C layer.
template <class T>
__global__ void beam_layer_kernel(const T* __restrict__ cur, const T* __restrict__ nxt, int S,
                                  int s, T* __restrict__ out, size_t plane, int* err) {
    const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= plane) return;
    T r, jx;
    if (S == 1) {
        r = cur[n];
        jx = cur[plane + n];
    } else {
        const T Sd = T(S);
        r = (cur[n] * (Sd - T(s)) + nxt[n] * T(s)) / Sd;
        jx = (cur[plane + n] * (Sd - T(s)) + nxt[plane + n] * T(s)) / Sd;
    }
    out[n] = r;
    out[plane + n] = jx;
    if (fabs((double)jx) > 10.0) atomicOr(err, DEV_ERR_BEAM_CURRENT);
}

template <class T>
int launch_beam_layer(const T* cur, const T* nxt, int S, int s, T* out, size_t plane, int* err,
                      cudaStream_t st) {
    beam_layer_kernel<T><<<(unsigned)((plane + 255) / 256), 256, 0, st>>>(cur, nxt, S, s, out,
                                                                          plane, err);
    return 1;
}

// kBeamSumParts blocks per layer (blockIdx.y): the |JxBeam| > 10 check of
// :618-621 and the block's FP64 partial sum of RhoBeam
template <class T>
__global__ void __launch_bounds__(256) beam_check_kernel(const T* __restrict__ b3, int nlayers,
                                                         size_t plane, int* err, double* part) {
    const int i = blockIdx.y;
    const T* rb = b3 + (size_t)i * 2 * plane;
    const T* jxb = rb + plane;
    double s = 0.0;
    bool bad = false;
    for (size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x; n < plane;
         n += (size_t)gridDim.x * blockDim.x) {
        s += (double)rb[n];
        bad |= fabs((double)jxb[n]) > 10.0;
    }
    if (bad) atomicOr(err, DEV_ERR_BEAM_CURRENT);
    charge_block_sum(s, 0.0, part + 2 * ((size_t)i * gridDim.x + blockIdx.x));
}

template <class T>
int launch_beam_check(const T* b3, int nlayers, size_t plane, int* err, double* part,
                      cudaStream_t st) {
    dim3 g((unsigned)kBeamSumParts, nlayers);
    beam_check_kernel<T><<<g, 256, 0, st>>>(b3, nlayers, plane, err, part);
    return 1;
}

__global__ void charge_reduce_kernel(const double* __restrict__ part, int nparts, int nlayers,
                                     double scale, double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * nlayers) return;
    const int layer = t >> 1, q = t & 1;
    const double* p = part + 2 * (size_t)layer * nparts + q;
    double s = 0.0;
    for (int i = 0; i < nparts; i++) s += p[2 * (size_t)i];
    out[t] = scale * s;
}

int launch_charge_reduce(const double* part, int nparts, int nlayers, double scale, double* out,
                         cudaStream_t st) {
    charge_reduce_kernel<<<(2 * nlayers + 127) / 128, 128, 0, st>>>(part, nparts, nlayers, scale,
                                                                   out);
    return 1;
}

template <class T>
__global__ void onaxis_kernel(const T* __restrict__ f3, int L, size_t plane, size_t idx,
                              T* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L) out[i] = f3[(size_t)i * 6 * plane + idx];
}

template <class T>
int launch_onaxis(const T* fields3d, int L, size_t plane, size_t idx, T* out, cudaStream_t st) {
    onaxis_kernel<T><<<(L + 255) / 256, 256, 0, st>>>(fields3d, L, plane, idx, out);
    return 1;
}

// ---- front-layer seeding with a counter-based generator.
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): 10 rounds of the
// published multiply-xor bijection with Weyl key schedule.
struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox_round(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t lo0 = M0 * c.x, hi0 = __umulhi(M0, c.x);
    const uint32_t lo1 = M1 * c.z, hi1 = __umulhi(M1, c.z);
    return U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
}

__device__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        c = philox_round(c, k0, k1);
        k0 += W0;
        k1 += W1;
    }
    return c;
}

__device__ __forceinline__ void box_muller(uint32_t a, uint32_t b, double& n0, double& n1) {
    const double u1 = ((double)a + 0.5) * 2.3283064365386963e-10;  // 2^-32
    const double u2 = ((double)b + 0.5) * 2.3283064365386963e-10;
    const double r = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    n0 = r * c;
    n1 = r * s;
}

template <class T>
__global__ void seed_front_kernel(SeedFront s, int32_t* cell, T* y, T* z, T* px, T* py, T* pz,
                                  T* w) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = (int64_t)s.My * s.Mz * s.ppc;
    if (p >= n) return;
    const int c = (int)(p / s.ppc), is = (int)(p % s.ppc);
    const uint32_t k0 = (uint32_t)s.seed, k1 = (uint32_t)(s.seed >> 32);
    // counter = (particle index, step): one block of 4 words gives 4 normals
    const U4 r0 = philox4x32_10(
        U4{(uint32_t)p, (uint32_t)(p >> 32), (uint32_t)s.step, (uint32_t)(s.step >> 32)}, k0, k1);
    double g0, g1, g2, g3;
    box_muller(r0.x, r0.y, g0, g1);
    box_muller(r0.z, r0.w, g2, g3);
    double weight = s.weight;
    if (s.use_profile) {
        // Density at the cell's corner (mesh.cpp:415-417), GetWeight()*dens (:471)
        const int j = c % s.My, k = c / s.My;
        const double dens = profile_density(s.prof, s.x_front, s.hy * j - s.y_half,
                                            s.hz * k - s.z_half);
        weight = dens > 0.0 ? (1. / s.ppc) * dens : 0.0;
    }
    cell[p] = c;
    y[p] = (T)s.offs_y[is];
    z[p] = (T)s.offs_z[is];
    px[p] = (T)(s.px0 + s.sx * g0);
    py[p] = (T)(s.py0 + s.sy * g1);
    pz[p] = (T)(s.pz0 + s.sz * g2);
    w[p] = (T)weight;
}

template <class T>
int launch_seed_front(const SeedFront& s, int32_t* cell, T* y, T* z, T* px, T* py, T* pz, T* w,
                      cudaStream_t st) {
    const int64_t n = (int64_t)s.My * s.Mz * s.ppc;
    seed_front_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(s, cell, y, z, px, py, pz, w);
    return 1;
}

template <class T>
__global__ void set_value_kernel(T* dst, T v) {
    *dst = v;
}
template <class T>
int launch_set_value(T* dst, T v, cudaStream_t st) {
    set_value_kernel<T><<<1, 1, 0, st>>>(dst, v);
    return 1;
}

template <class T>
__global__ void convert_kernel(const void* __restrict__ src, int is_double, T* __restrict__ dst,
                               size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst[i] = is_double ? (T)((const double*)src)[i] : (T)((const float*)src)[i];
}
template <class T>
__global__ void convert_back_kernel(const T* __restrict__ src, double* __restrict__ dst, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = (double)src[i];
}
template <class T>
int launch_convert(const void* src, int src_is_double, T* dst, size_t n, cudaStream_t st) {
    if (!n) return 0;
    convert_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(src, src_is_double, dst, n);
    return 1;
}
template <class T>
int launch_convert_back(const T* src, double* dst, size_t n, cudaStream_t st) {
    if (!n) return 0;
    convert_back_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(src, dst, n);
    return 1;
}

// ---- layer output: a block of the 3-D store in x-fastest order
// out[i + L (jj + nj kk)] = base[i * layer_stride + (j0 + jj) + My (k0 + kk)]
template <class T>
__global__ void gather_xfast_kernel(const T* __restrict__ base, size_t layer_stride, int L,
                                    int My, int j0, int nj, int k0, int nk,
                                    double* __restrict__ out) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t total = (size_t)L * nj * nk;
    if (idx >= total) return;
    const int i = (int)(idx % L);
    const size_t rest = idx / L;
    const int jj = (int)(rest % nj), kk = (int)(rest / nj);
    out[idx] = (double)base[(size_t)i * layer_stride + (size_t)(j0 + jj) + (size_t)My * (k0 + kk)];
}
template <class T>
int launch_gather_xfast(const T* base, size_t layer_stride, int L, int My, int j0, int nj, int k0,
                        int nk, double* out, cudaStream_t st) {
    const size_t total = (size_t)L * nj * nk;
    if (!total) return 0;
    gather_xfast_kernel<T><<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
        base, layer_stride, L, My, j0, nj, k0, nk, out);
    return 1;
}

// ---- the FP32 attribution study of the FP64 engine (see api.cu)
__global__ void round_f32_kernel(double* __restrict__ x, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = (double)(float)x[i];
}
int launch_round_f32(double* x, size_t n, cudaStream_t st) {
    if (!n) return 0;
    round_f32_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, n);
    return 1;
}
__global__ void add_widened_kernel(double* __restrict__ dst, const float* __restrict__ src,
                                   size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] += (double)src[i];
}
// dst += (double)now - (double)before; in-cell fractions (frac) kept in [0, 1]
__global__ void add_increment_kernel(double* __restrict__ dst, const float* __restrict__ now,
                                     const float* __restrict__ before, size_t n, int frac) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = dst[i] + ((double)now[i] - (double)before[i]);
    if (frac) v = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
    dst[i] = v;
}
int launch_add_increment(double* dst, const float* now, const float* before, size_t n, int frac,
                         cudaStream_t st) {
    if (!n) return 0;
    add_increment_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dst, now, before, n, frac);
    return 1;
}
int launch_add_widened(double* dst, const float* src, size_t n, cudaStream_t st) {
    if (!n) return 0;
    add_widened_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dst, src, n);
    return 1;
}

#define QS_INST(T)                                                                              \
    template int launch_predictor<T>(const SpecArgs<T>&, cudaStream_t);                         \
    template int launch_corrector<T>(const SpecArgs<T>&, cudaStream_t);                         \
    template int launch_beam_layer<T>(const T*, const T*, int, int, T*, size_t, int*,           \
                                      cudaStream_t);                                            \
    template int launch_onaxis<T>(const T*, int, size_t, size_t, T*, cudaStream_t);            \
    template int launch_gather_xfast<T>(const T*, size_t, int, int, int, int, int, int, double*, \
                                        cudaStream_t);                                          \
    template int launch_beam_check<T>(const T*, int, size_t, int*, double*, cudaStream_t);     \
    template int launch_seed_front<T>(const SeedFront&, int32_t*, T*, T*, T*, T*, T*, T*,       \
                                      cudaStream_t);                                            \
    template int launch_set_value<T>(T*, T, cudaStream_t);                                      \
    template int launch_convert<T>(const void*, int, T*, size_t, cudaStream_t);                 \
    template int launch_convert_back<T>(const T*, double*, size_t, cudaStream_t);
QS_INST(float)
QS_INST(double)
#undef QS_INST

}  // namespace qs
