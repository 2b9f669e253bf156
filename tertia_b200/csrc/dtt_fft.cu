// dtt_fft.cu — FP32 half-integer transforms (FFTW REDFT11 / RODFT11, the
// reference's plans at movefieldshydrolinlayersplit.cpp:389-427) through a
// complex FFT of half the length, for power-of-two sizes 32 .. 2048.
//
// A DCT-IV of length n is an n/2-point complex FFT between a pre- and a
// post-twiddle (the standard reduction; e.g. Britanak, Yip and Rao,
// "Discrete Cosine and Sine Transforms", 2007):
//   z_i = (x[2i] + i x[n-1-2i]) e^{-i pi i/n},   Z = FFT_{n/2}(z),
//   s_i = Z_i e^{-i pi (i+1/4)/n},   y[2i] = 2 Re s_i,   y[n-1-2i] = -2 Im s_i.
// A DST-IV is the DCT-IV of the reversed input with the odd outputs negated.
// The FFT is the Stockham autosort formulation of Govindaraju et al.
// ("High performance discrete Fourier transforms on graphics processors",
// SC 2008): a radix-V pass in registers (V values per thread: 8 for
// n <= 256, 16 above), then Stockham passes of radix V (and the remaining
// factor) through shared memory, each thread holding one butterfly group in
// registers and the sequence in shared memory between passes.  Every twiddle
// comes from one table of e^{-2 pi i k/(n/2)} built in FP64 on the host, so
// the error is that of an FP32 FFT (a few 1e-7 relative), well below the
// split-precision GEMMs'.
//
// A 2-D transform is two kernels over a batch of planes (nz rows of ny, y
// fastest): rows along y into a scratch plane, then columns along z into the
// destination with the output scale.  Both read and write each plane once.
#include <cmath>
#include <vector>

#include "qs_common.cuh"
#include "qs_internal.h"
#include "pdl.cuh"
#include "spectral_f32.cuh"
#include "adjoint_maps.cuh"
#include "charge.cuh"
#include "trace.cuh"

namespace qs {
namespace fft {

// The FFT machinery is written once for a complex type C: float2 for the FP32
// transforms, double2 for the FP64 ones (the same algorithm in FP64).
template <class C> struct Cx;
template <> struct Cx<float2> {
    using Real = float;
    __device__ __host__ static float2 make(float x, float y) { return make_float2(x, y); }
};
template <> struct Cx<double2> {
    using Real = double;
    __device__ __host__ static double2 make(double x, double y) { return make_double2(x, y); }
};

template <class C>
__device__ __forceinline__ C cmul(C a, C b) {
    return Cx<C>::make(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class C>
__device__ __forceinline__ C cadd(C a, C b) { return Cx<C>::make(a.x + b.x, a.y + b.y); }
template <class C>
__device__ __forceinline__ C csub(C a, C b) { return Cx<C>::make(a.x - b.x, a.y - b.y); }

template <int R>
__device__ __forceinline__ int bitrev(int i) {
    constexpr int B = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4;
    return (int)(__brev((unsigned)i) >> (32 - B));
}

// e^{-2 pi i k/16} for k = 0..7 (cos and sin of multiples of pi/8)
constexpr double kC8 = 0.923879532511286756;   // cos(pi/8)
constexpr double kS8 = 0.382683432365089772;   // sin(pi/8)
constexpr double kR2 = 0.707106781186547524;   // cos(pi/4)

// x * e^{-2 pi i k/16}, with the multiplications by 1 and -i left out
template <int K, class C>
__device__ __forceinline__ C rot16(C x) {
    static_assert(K >= 0 && K < 8, "rot16");
    using Real = typename Cx<C>::Real;
    constexpr Real r2 = (Real)kR2;
    if constexpr (K == 0) return x;
    else if constexpr (K == 4) return Cx<C>::make(x.y, -x.x);
    else if constexpr (K == 2) return Cx<C>::make(r2 * (x.x + x.y), r2 * (x.y - x.x));
    else if constexpr (K == 6) return Cx<C>::make(r2 * (x.y - x.x), -r2 * (x.x + x.y));
    else {
        constexpr Real c = (Real)(K == 1 ? kC8 : K == 3 ? kS8 : K == 5 ? -kS8 : -kC8);
        constexpr Real s = (Real)(K == 1 ? kS8 : K == 3 ? kC8 : K == 5 ? kC8 : kS8);
        return Cx<C>::make(c * x.x + s * x.y, c * x.y - s * x.x);
    }
}

// one radix-2 stage of butterflies of length LEN over the R registers
template <int R, int LEN, int T, class C>
__device__ __forceinline__ void dit_stage_t(C (&v)[R]) {
    if constexpr (T < LEN / 2) {
#pragma unroll
        for (int s = 0; s < R; s += LEN) {
            const C u = v[s + T];
            const C x = rot16<T * (16 / LEN)>(v[s + T + LEN / 2]);
            v[s + T] = cadd(u, x);
            v[s + T + LEN / 2] = csub(u, x);
        }
        dit_stage_t<R, LEN, T + 1>(v);
    }
}
template <int R, int LEN, class C>
__device__ __forceinline__ void dit_stages(C (&v)[R]) {
    if constexpr (LEN <= R) {
        dit_stage_t<R, LEN, 0>(v);
        dit_stages<R, 2 * LEN>(v);
    }
}

// R-point forward DFT in registers (radix-2, decimation in time, R <= 16,
// constant twiddles).  The input is loaded in bit-reversed order
// (v[i] = x[bitrev(i)]), so only memory addresses are permuted and every
// register index is static; the output is in natural order.
template <int R, class C>
__device__ __forceinline__ void dft(C (&v)[R]) {
    dit_stages<R, 2>(v);
}

// Exchanges between passes: a sequence whose threads share one warp only
// needs the warp to meet; wider ones need the whole block.
template <bool WARP>
__device__ __forceinline__ void seq_sync() {
    if constexpr (WARP) __syncwarp();
    else __syncthreads();
}

// load, twiddle and transform butterfly group j of a pass (registers only)
template <int M, int R, int NS, class C, class At>
__device__ __forceinline__ void stockham_group(C (&v)[R], const C* W, At at, int j, const C* tw) {
#pragma unroll
    for (int i = 0; i < R; i++) {
        const int r = bitrev<R>(i);
        v[i] = W[at(j + r * (M / R))];
        if (i) v[i] = cmul(v[i], tw[(j % NS) * r * (M / (NS * R))]);
    }
    dft<R>(v);
}

template <int R, int NS, class C, class At>
__device__ __forceinline__ void stockham_store(const C (&v)[R], C* W, At at, int j) {
    const int d = (j / NS) * NS * R + (j % NS);
#pragma unroll
    for (int r = 0; r < R; r++) W[at(d + r * NS)] = v[r];
}

// One Stockham pass of radix R after NS points have been combined: every
// thread of a sequence (T = M/V of them, V values each) does (M/R)/T
// butterfly groups (1, 2, 4 or 8).  `at(e)` maps element e of this thread's
// sequence to its shared-memory slot.
template <int M, int V, int R, int NS, bool WARP, class C, class At>
__device__ __forceinline__ void stockham_pass(C* W, At at, int jt, const C* tw) {
    constexpr int T = M / V;
    constexpr int G = (M / R) / T;
    static_assert(G == 1 || G == 2 || G == 4 || G == 8, "groups per thread");
    if constexpr (G == 1) {
        C v[R];
        stockham_group<M, R, NS>(v, W, at, jt, tw);
        seq_sync<WARP>();
        stockham_store<R, NS>(v, W, at, jt);
    } else {
        C v[G][R];
#pragma unroll
        for (int g = 0; g < G; g++) stockham_group<M, R, NS>(v[g], W, at, jt + g * T, tw);
        seq_sync<WARP>();
#pragma unroll
        for (int g = 0; g < G; g++) stockham_store<R, NS>(v[g], W, at, jt + g * T);
    }
    seq_sync<WARP>();
}

// The last pass keeps its butterfly groups in registers: thread jt ends up
// with Z_q for q = jt + T*m in slot m (m < V), and Z_{M-1-q} sits in slot
// V-1-m of thread T-1-jt.
template <int M, int V, int R, int NS, class C, class At>
__device__ __forceinline__ void final_pass(const C* W, At at, int jt, const C* tw, C (&fin)[V]) {
    constexpr int T = M / V;
    constexpr int G = (M / R) / T;
    static_assert(NS * R == M && G * R == V, "final pass");
#pragma unroll
    for (int g = 0; g < G; g++) {
        C v[R];
        stockham_group<M, R, NS>(v, W, at, jt + g * T, tw);
#pragma unroll
        for (int r = 0; r < R; r++) fin[g + G * r] = v[r];
    }
}

// the passes after the first radix-V one (radix V, then the remaining factor)
template <int M, int V, int NS, bool WARP>
struct Passes {
    static constexpr int R = (M / NS) >= V ? V : (M / NS);
    template <class C, class At>
    __device__ __forceinline__ static void run(C* W, At at, int jt, const C* tw, C (&fin)[V]) {
        if constexpr (NS * R == M) {
            final_pass<M, V, R, NS>(W, at, jt, tw, fin);
        } else {
            stockham_pass<M, V, R, NS, WARP>(W, at, jt, tw);
            Passes<M, V, NS * R, WARP>::run(W, at, jt, tw, fin);
        }
    }
};

// values per thread: 8 on the small grids (more threads in flight, measured
// faster at n = 256), 16 from n = 512 on (fewer passes; as fast or faster)
template <int M>
__host__ __device__ constexpr int vpt() {
    return M <= 128 ? 8 : 16;
}
// values per thread of the FP64 transforms: 8 (twice the registers per value)
template <int M, class C>
__host__ __device__ constexpr int vpt_c() {
    return sizeof(C) == sizeof(float2) ? vpt<M>() : 8;
}
// values per thread of the map kernels' row transforms: 8 on the 512-wide
// FP32 grid, so that a transform group is one whole warp, every thread of the
// CTA takes part in the transforms and the CTA needs fewer registers (four
// CTAs per SM: the 512 z-mode rows run in one wave); elsewhere those of the
// plain row transforms
template <int M, class C = float2>
__host__ __device__ constexpr int spec_vpt() {
    return (sizeof(C) == sizeof(float2) && M == 256) ? 8 : vpt_c<M, C>();
}
template <class Real> struct CxOf;
template <> struct CxOf<float> { using type = float2; };
template <> struct CxOf<double> { using type = double2; };

template <class Real>
struct RowArgsT {
    const Real* in[kMaxXfFields];
    Real* out[kMaxXfFields];
    int kind[kMaxXfFields];   // QS_REDFT11 / QS_RODFT11 of each field
    int nrows;                // rows per plane
    int total;                // nf * nrows
    Real scale;
    const typename CxOf<Real>::type* tab;   // tw[M], pre[M], post[M]
};
using RowArgs = RowArgsT<float>;

template <int M, class C = float2>
__host__ __device__ constexpr int row_threads() {
    return (M / vpt_c<M, C>()) > 64 ? (M / vpt_c<M, C>()) : 64;
}

// Transform along the contiguous axis: each sequence of T = M/V threads
// takes one row of n = 2M values (small blocks, so that the rows of a batch
// spread evenly over the SMs).  Thread jt holds the pairs P[jt + T*b]
// (P[i] = (x[2i], x[2i+1])); the mirrored element x[n-1-2i] of the
// pre-twiddle and the mirrored output of the post-twiddle belong to thread
// T-1-jt, a shuffle away when a row lies within one warp.  Shared slot of
// element e: e + e/V (one pad per V keeps the stride-V stores of the first
// pass free of bank conflicts).
template <int M, class C>
__global__ void __launch_bounds__(row_threads<M, C>())
    fft_rows_kernel(RowArgsT<typename Cx<C>::Real> a) {
    using Real = typename Cx<C>::Real;
    constexpr int V = vpt_c<M, C>();
    constexpr int T = M / V;
    constexpr int NT = row_threads<M, C>();
    constexpr int SEQ = NT / T;
    constexpr int LD = M + M / V;
    constexpr bool WARP = T <= 32;
    __shared__ C W[SEQ * LD];
    __shared__ C tws[M];
    __shared__ C posts[M];
    for (int i = threadIdx.x; i < M; i += NT) {
        tws[i] = a.tab[i];
        posts[i] = a.tab[2 * M + i];
    }
    const int s = threadIdx.x / T, jt = threadIdx.x % T;
    const int row = blockIdx.x * SEQ + s;
    const bool valid = row < a.total;
    const int f = valid ? row / a.nrows : 0, k = valid ? row % a.nrows : 0;
    C* Ws = W + s * LD;
    auto at = [](int e) { return e + e / V; };
    QS_TRACE_ENTRY();
    pdl_wait();
    QS_TRACE_WAITED();
    const Real* inf = a.in[0];
    Real* outf = a.out[0];
    int kind = a.kind[0];
#pragma unroll
    for (int q = 1; q < kMaxXfFields; q++)
        if (q == f) { inf = a.in[q]; outf = a.out[q]; kind = a.kind[q]; }
    const C* P = reinterpret_cast<const C*>(inf + (size_t)k * 2 * M);
    const C* pre = a.tab + M;
    // the V pairs of this thread in bit-reversed order, the pre-twiddle
    C p[V], w[V];
#pragma unroll
    for (int b = 0; b < V; b++) {
        const int i = jt + bitrev<V>(b) * T;
        p[b] = valid ? P[i] : Cx<C>::make(Real(0), Real(0));
        w[b] = __ldg(pre + i);
    }
    C v[V];
    if constexpr (WARP) {
        // x[n-1-2i] = P[M-1-i].y: slot V-1-b of thread T-1-jt
#pragma unroll
        for (int b = 0; b < V; b++) {
            const Real mirror = __shfl_xor_sync(0xffffffffu, p[V - 1 - b].y, T - 1);
            const C z = kind == QS_REDFT11 ? Cx<C>::make(p[b].x, mirror)
                                           : Cx<C>::make(mirror, p[b].x);
            v[b] = cmul(z, w[b]);
        }
    } else {
#pragma unroll
        for (int b = 0; b < V; b++) {
            const int i = jt + bitrev<V>(b) * T;
            const Real mirror = valid ? P[M - 1 - i].y : Real(0);
            const C z = kind == QS_REDFT11 ? Cx<C>::make(p[b].x, mirror)
                                           : Cx<C>::make(mirror, p[b].x);
            v[b] = cmul(z, w[b]);
        }
    }
    __syncthreads();   // twiddle tables in place
    dft<V>(v);
    C fin[V];
    if constexpr (T == 1) {
        // one pass: Z_r in slot r, the thread owns the whole sequence
#pragma unroll
        for (int r = 0; r < V; r++) fin[r] = v[r];
    } else {
#pragma unroll
        for (int r = 0; r < V; r++) Ws[at(jt * V + r)] = v[r];
        seq_sync<WARP>();
        Passes<M, V, V, WARP>::run(Ws, at, jt, tws, fin);
    }
    pdl_trigger();
    // s_q = Z_q e^{-i pi (q+1/4)/n}; out pair q = (2 Re s_q, -+2 Im s_{M-1-q})
    Real im[V];
#pragma unroll
    for (int m = 0; m < V; m++) {
        const int q = jt + T * m;
        const C sq = cmul(fin[m], posts[q]);
        fin[m] = sq;
        im[m] = sq.y;
    }
    Real mirror[V];
    if constexpr (WARP) {
#pragma unroll
        for (int m = 0; m < V; m++) mirror[m] = __shfl_xor_sync(0xffffffffu, im[V - 1 - m], T - 1);
    } else {
        // rows wider than a warp: the mirrored parts through shared memory
        __syncthreads();
        Real* ims = reinterpret_cast<Real*>(Ws);
#pragma unroll
        for (int m = 0; m < V; m++) ims[jt + T * m] = im[m];
        __syncthreads();
#pragma unroll
        for (int m = 0; m < V; m++) mirror[m] = ims[M - 1 - (jt + T * m)];
    }
    QS_TRACE_END(trace::K_YPASS);
    if (!valid) return;
    C* O = reinterpret_cast<C*>(outf + (size_t)k * 2 * M);
    const Real c2 = Real(2) * a.scale;
    const Real sgn = kind == QS_REDFT11 ? -c2 : c2;
#pragma unroll
    for (int m = 0; m < V; m++) O[jt + T * m] = Cx<C>::make(c2 * fin[m].x, sgn * mirror[m]);
}

template <class Real>
struct ColArgsT {
    const Real* in[kMaxXfFields];
    Real* out[kMaxXfFields];
    Real* acc[kMaxXfFields];    // optional: the input is also added here
    Real* clr[kMaxXfFields];    // optional: the input planes, zeroed once read
    int kind[kMaxXfFields];
    int ncols;                // row length of the planes (the y size)
    Real scale;
    const typename CxOf<Real>::type* tab;
};
using ColArgs = ColArgsT<float>;

// Transform along the strided axis: a CTA takes TJ adjacent columns of one
// plane (TJ floats = whole 32-byte sectors per row); column c's sequence
// lives at W[e * TJ + c], its T threads are TJ lanes apart.
template <int M, int TJ, class C>
__global__ void __launch_bounds__(TJ * (M / vpt_c<M, C>()))
    fft_cols_kernel(ColArgsT<typename Cx<C>::Real> a) {
    using Real = typename Cx<C>::Real;
    constexpr int V = vpt_c<M, C>();
    constexpr int T = M / V;
    constexpr int NT = TJ * T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tws = reinterpret_cast<C*>(smem_raw);
    C* posts = tws + M;
    C* W = tws + 2 * M;
    for (int i = threadIdx.x; i < M; i += NT) {
        tws[i] = a.tab[i];
        posts[i] = a.tab[2 * M + i];
    }
    const int c = threadIdx.x % TJ, jt = threadIdx.x / TJ;
    const int f = blockIdx.y;
    const int col = blockIdx.x * TJ + c;
    const size_t ld = (size_t)a.ncols;
    auto at = [c](int e) { return e * TJ + c; };
    QS_TRACE_ENTRY();
    pdl_wait();
    QS_TRACE_WAITED();
    const Real* inf = a.in[0];
    Real* outf = a.out[0];
    Real* accf = a.acc[0];
    Real* clrf = a.clr[0];
    int kind = a.kind[0];
#pragma unroll
    for (int q = 1; q < kMaxXfFields; q++)
        if (q == f) {
            inf = a.in[q]; outf = a.out[q]; accf = a.acc[q]; clrf = a.clr[q]; kind = a.kind[q];
        }
    const C* pre = a.tab + M;
    Real lo[V], hi[V];
    C w[V];
#pragma unroll
    for (int b = 0; b < V; b++) {
        const int i = jt + bitrev<V>(b) * T;
        lo[b] = inf[(size_t)(2 * i) * ld + col];
        hi[b] = inf[(size_t)(2 * M - 1 - 2 * i) * ld + col];
        w[b] = __ldg(pre + i);
    }
    if (accf || clrf) {   // the same for the whole CTA
#pragma unroll
        for (int b = 0; b < V; b++) {
            const int i = jt + bitrev<V>(b) * T;
            const size_t olo = (size_t)(2 * i) * ld + col;
            const size_t ohi = (size_t)(2 * M - 1 - 2 * i) * ld + col;
            if (accf) {
                accf[olo] += lo[b];
                accf[ohi] += hi[b];
            }
            if (clrf) {
                clrf[olo] = Real(0);
                clrf[ohi] = Real(0);
            }
        }
    }
    C v[V];
#pragma unroll
    for (int b = 0; b < V; b++) {
        const C z = kind == QS_REDFT11 ? Cx<C>::make(lo[b], hi[b]) : Cx<C>::make(hi[b], lo[b]);
        v[b] = cmul(z, w[b]);
    }
    __syncthreads();
    dft<V>(v);
    C fin[V];
    if constexpr (T == 1) {
#pragma unroll
        for (int r = 0; r < V; r++) fin[r] = v[r];
    } else {
#pragma unroll
        for (int r = 0; r < V; r++) W[at(jt * V + r)] = v[r];
        __syncthreads();
        Passes<M, V, V, false>::run(W, at, jt, tws, fin);
    }
    pdl_trigger();
    Real im[V];
#pragma unroll
    for (int m = 0; m < V; m++) {
        const int q = jt + T * m;
        fin[m] = cmul(fin[m], posts[q]);
        im[m] = fin[m].y;
    }
    __syncthreads();
    Real* ims = reinterpret_cast<Real*>(W);
#pragma unroll
    for (int m = 0; m < V; m++) ims[(jt + T * m) * TJ + c] = im[m];
    __syncthreads();
    const Real c2 = Real(2) * a.scale;
    const Real sgn = kind == QS_REDFT11 ? -c2 : c2;
#pragma unroll
    for (int m = 0; m < V; m++) {
        const int q = jt + T * m;
        outf[(size_t)(2 * q) * ld + col] = c2 * fin[m].x;
        outf[(size_t)(2 * q + 1) * ld + col] = sgn * ims[(M - 1 - q) * TJ + c];
    }
    QS_TRACE_END(trace::K_ZPASS);
}

template <int M, class C = float2>
__host__ __device__ constexpr int cols_tj() {
    return (M / vpt_c<M, C>()) >= 16 ? 8 : (M / vpt_c<M, C>()) >= 4 ? 16 : 32;
}

template <int M, class C = float2>
size_t cols_smem() {
    return sizeof(C) * (size_t)M * (2 + cols_tj<M, C>());
}

template <int M, class C = float2>
cudaError_t set_cols_smem() {
    return cudaFuncSetAttribute(fft_cols_kernel<M, cols_tj<M, C>(), C>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)cols_smem<M, C>());
}

template <int M, class C = float2>
cudaError_t launch_rows(const RowArgsT<typename Cx<C>::Real>& a, cudaStream_t st) {
    constexpr int SEQ = row_threads<M, C>() / (M / vpt_c<M, C>());
    const int blocks = (a.total + SEQ - 1) / SEQ;
    return launch_pdl(fft_rows_kernel<M, C>, dim3((unsigned)blocks), dim3(row_threads<M, C>()), 0,
                      st, a);
}

template <int M, class C = float2>
cudaError_t launch_cols(const ColArgsT<typename Cx<C>::Real>& a, int nf, cudaStream_t st) {
    constexpr int TJ = cols_tj<M, C>();
    return launch_pdl(fft_cols_kernel<M, TJ, C>, dim3((unsigned)(a.ncols / TJ), (unsigned)nf),
                      dim3(TJ * (M / vpt_c<M, C>())), cols_smem<M, C>(), st, a);
}

// ---------------------------------------------------------------------------
// The per-mode Guess / Iterate maps between the two halves of a transform.
// The march transforms along z first (column kernel), so that one kernel can
// take a z-mode row k through [forward y-transform of the deposit J] ->
// [corrector or predictor on the row's modes] -> [inverse y-transform of E, B
// (and Rho)], with the row in shared memory in between; the column kernel
// then finishes the inverse along z.  A CTA holds one row: 8 groups of
// T = M/V lanes (one warp holds whole groups), each group taking one plane's
// row through a transform; groups without a plane run it on zeros, so that
// every lane meets every shuffle.

// one row of n = 2M values through the half-integer transform of `kind` by
// the T lanes of a group: in_pair(i) = (x[2i], x[2i+1]); out_pair(q, v) gets
// the output pair q; `valid` false runs the group on zeros and stores nothing
template <int M, class C = float2, int V = vpt_c<M, C>(), class InPair, class OutPair>
__device__ __forceinline__ void row_dtt_group(InPair in_pair, OutPair out_pair, int kind,
                                              typename Cx<C>::Real scale, bool valid, int jt,
                                              C* Wg, const C* tws, const C* posts,
                                              const C* pre) {
    using Real = typename Cx<C>::Real;
    constexpr int T = M / V;
    static_assert(T >= 1 && T <= 32, "a group within one warp");
    auto at = [](int e) { return e + e / V; };
    C p[V], w[V];
#pragma unroll
    for (int b = 0; b < V; b++) {
        const int i = jt + bitrev<V>(b) * T;
        p[b] = valid ? in_pair(i) : Cx<C>::make(Real(0), Real(0));
        w[b] = __ldg(pre + i);
    }
    C v[V];
#pragma unroll
    for (int b = 0; b < V; b++) {
        const Real mirror = __shfl_xor_sync(0xffffffffu, p[V - 1 - b].y, T - 1);
        const C z = kind == QS_REDFT11 ? Cx<C>::make(p[b].x, mirror)
                                       : Cx<C>::make(mirror, p[b].x);
        v[b] = cmul(z, w[b]);
    }
    dft<V>(v);
    C fin[V];
    if constexpr (T == 1) {
#pragma unroll
        for (int r = 0; r < V; r++) fin[r] = v[r];
    } else {
#pragma unroll
        for (int r = 0; r < V; r++) Wg[at(jt * V + r)] = v[r];
        __syncwarp();
        Passes<M, V, V, true>::run(Wg, at, jt, tws, fin);
    }
    Real im[V];
#pragma unroll
    for (int m = 0; m < V; m++) {
        fin[m] = cmul(fin[m], posts[jt + T * m]);
        im[m] = fin[m].y;
    }
    const Real c2 = Real(2) * scale;
    const Real sgn = kind == QS_REDFT11 ? -c2 : c2;
#pragma unroll
    for (int m = 0; m < V; m++) {
        const Real mirror = __shfl_xor_sync(0xffffffffu, im[V - 1 - m], T - 1);
        if (valid) out_pair(jt + T * m, Cx<C>::make(c2 * fin[m].x, sgn * mirror));
    }
    __syncwarp();   // Wg is free again
}

template <class Real>
struct SpecRowArgsT {
    const Real* jin;      // corrector: Jx, Jy, Jz after the z-pass (stride `plane`)
    Real* out;            // Ex, Ey, Ez, Bx, By, Bz (, Rho) after the inverse y-pass
    int nout;             // 6, or 7 with Rho
    const typename CxOf<Real>::type* tab;   // tables of the y size
    Real* out_next;       // with the next layer's predictor: its Ex..Bz after the y-pass
    int avg_next;         // out_next gets (this layer's E, B + the predicted ones) / 2
};
using SpecRowArgs = SpecRowArgsT<float>;

constexpr int kSpecGroups = 8;
// one transform group per plane of a row: Ex..Bz and Rho out of the map
// kernel, the six field adjoints into its adjoint
static_assert(kSpecGroups >= 7, "a transform group per plane");

template <int M, class C = float2>
__host__ __device__ constexpr size_t spec_rows_smem() {
    // tables, FFT work of each group, the row's J spectra and E, B, Rho spectra
    return sizeof(C) * (2 * (size_t)M + (size_t)kSpecGroups * (M + M / spec_vpt<M, C>())) +
           sizeof(typename Cx<C>::Real) * (3 + 7) * (size_t)(2 * M);
}

// threads of a map CTA: the transform groups, or one per mode pair if more
template <int M, class C = float2>
__host__ __device__ constexpr int spec_threads() {
    return kSpecGroups * (M / spec_vpt<M, C>()) > M ? kSpecGroups * (M / spec_vpt<M, C>()) : M;
}

// PRED_NEXT (with CORRECT): the layer's last corrector, then the next
// layer's predictor (`an`, whose P bank is the bank the corrector has just
// written) on the same row, and its inverse y-pass into r.out_next.  The maps
// are per mode and each thread keeps its mode pairs in both loops, so the
// predictor reads what the same thread stored; it overwrites the corrector's
// P bank (no longer needed) only at those modes.  C: float2 (FP32) or
// double2 (FP64 on FFT transforms).
template <int M, bool CORRECT, bool PRED_NEXT, class C>
__device__ __forceinline__ void spectral_rows_body(SpecArgs<typename Cx<C>::Real> a,
                                                   SpecRowArgsT<typename Cx<C>::Real> r,
                                                   SpecArgs<typename Cx<C>::Real> an) {
    static_assert(CORRECT || !PRED_NEXT, "the next layer's predictor follows a corrector");
    using namespace specf32;
    using Real = typename Cx<C>::Real;
    constexpr int V = spec_vpt<M, C>();
    constexpr int T = M / V;
    constexpr int NTF = kSpecGroups * T;   // the transform groups (whole warps)
    constexpr int NT = spec_threads<M, C>();
    static_assert(NTF % 32 == 0, "transform groups fill whole warps");
    constexpr int N = 2 * M;
    constexpr int LD = M + M / V;
    extern __shared__ __align__(16) unsigned char smem_spec[];
    C* tws = reinterpret_cast<C*>(smem_spec);
    C* posts = tws + M;
    C* W = posts + M;
    Real* J = reinterpret_cast<Real*>(W + kSpecGroups * LD);   // 3 x N
    Real* EB = J + 3 * N;                                       // 7 x N
    for (int i = threadIdx.x; i < M; i += NT) {
        tws[i] = r.tab[i];
        posts[i] = r.tab[2 * M + i];
    }
    const int k = blockIdx.x;
    const int g = threadIdx.x / T, jt = threadIdx.x % T;
    // the first group of this thread's warp: a warp whose groups all lack a
    // plane skips the transform (its lanes meet no shuffle of another warp)
    const int wg0 = (threadIdx.x / 32) * (32 / T);
    C* Wg = W + g * LD;
    const C* pre = r.tab + M;
    const size_t plane = (size_t)N * a.nz;
    QS_TRACE_ENTRY();
    pdl_wait();
    QS_TRACE_WAITED();
    __syncthreads();
    if constexpr (CORRECT) {
        // forward y-transform of the deposit rows (Jx REDFT11, Jy RODFT11, Jz REDFT11)
        if (threadIdx.x < NTF && wg0 < 3) {
            const bool valid = g < 3;
            const int gg = valid ? g : 0;
            const C* src = reinterpret_cast<const C*>(r.jin + gg * plane + (size_t)k * N);
            C* dst = reinterpret_cast<C*>(J + gg * N);
            row_dtt_group<M, C, V>([src](int i) { return src[i]; },
                                [dst](int q, C v) { dst[q] = v; },
                                gg == 1 ? QS_RODFT11 : QS_REDFT11, Real(1), valid, jt, Wg, tws,
                                posts, pre);
        }
        __syncthreads();
    }
    auto to_eb = [&](int j, const Modes2<Real>& o) {
        *reinterpret_cast<C*>(EB + 0 * N + j) = Cx<C>::make(o.ex[0], o.ex[1]);
        *reinterpret_cast<C*>(EB + 1 * N + j) = Cx<C>::make(o.ey[0], o.ey[1]);
        *reinterpret_cast<C*>(EB + 2 * N + j) = Cx<C>::make(o.ez[0], o.ez[1]);
        *reinterpret_cast<C*>(EB + 3 * N + j) = Cx<C>::make(o.bx[0], o.bx[1]);
        *reinterpret_cast<C*>(EB + 4 * N + j) = Cx<C>::make(o.by[0], o.by[1]);
        *reinterpret_cast<C*>(EB + 5 * N + j) = Cx<C>::make(o.bz[0], o.bz[1]);
        *reinterpret_cast<C*>(EB + 6 * N + j) = Cx<C>::make(o.rho[0], o.rho[1]);
    };
    // the maps on the row's modes, two per thread
    double qr = 0.0, qj = 0.0;   // FP64 charge sums (charge.cuh)
    for (int pj = threadIdx.x; pj < M; pj += NT) {
        const int j = 2 * pj;
        const size_t n = (size_t)j + (size_t)N * k;
        Modes2<Real> o;
        if constexpr (CORRECT) {
            const C jx2 = *reinterpret_cast<const C*>(J + j);
            const C jy2 = *reinterpret_cast<const C*>(J + N + j);
            const C jz2 = *reinterpret_cast<const C*>(J + 2 * N + j);
            st2(const_cast<Real*>(a.Jx), n, jx2.x, jx2.y);   // the bank keeps the deposit spectra
            st2(const_cast<Real*>(a.Jy), n, jy2.x, jy2.y);
            st2(const_cast<Real*>(a.Jz), n, jz2.x, jz2.y);
            o = corrector_modes2(a, j, k, n, jx2, jy2, jz2);
            if (a.qsum) {
                const double c0 = a.qcy[j], c1 = a.qcy[j + 1];
                qr += (double)o.rho[0] * c0 + (double)o.rho[1] * c1;
                qj += (double)jx2.x * c0 + (double)jx2.y * c1;
            }
        } else {
            o = predictor_modes2(a, j, k, n);
        }
        store_modes2(a, n, o);
        to_eb(j, o);
    }
    if (CORRECT && a.qsum) {
        const double cz = a.qcz[k];
        charge_block_sum(qr * cz, qj * cz, a.qsum + 2 * (size_t)k);
    }
    __syncthreads();
    if constexpr (!PRED_NEXT) pdl_trigger();
    // inverse y-transform of Ex Ey Ez Bx By Bz Rho (y kinds C S C S C S C)
    if (threadIdx.x < NTF && wg0 < r.nout) {
        const bool valid = g < r.nout;
        const int gg = valid ? g : 0;
        const C* src = reinterpret_cast<const C*>(EB + gg * N);
        C* dst = reinterpret_cast<C*>(r.out + gg * plane + (size_t)k * N);
        row_dtt_group<M, C, V>([src](int i) { return src[i]; },
                            [dst](int q, C v) { dst[q] = v; },
                            (gg & 1) ? QS_RODFT11 : QS_REDFT11, Real(1), valid, jt, Wg, tws, posts,
                            pre);
    }
    if constexpr (PRED_NEXT) {
        __syncthreads();   // EB is free again
        for (int pj = threadIdx.x; pj < M; pj += NT) {
            const int j = 2 * pj;
            const size_t n = (size_t)j + (size_t)N * k;
            const Modes2<Real> o = predictor_modes2(an, j, k, n);
            store_modes2(an, n, o);
            if (r.avg_next) {
                // the fields the next layer's first push gathers: this
                // layer's (still in EB) and the predicted ones, averaged
                const Real h = Real(0.5);
                C* eb = reinterpret_cast<C*>(EB + j);
                const Real v[6][2] = {{o.ex[0], o.ex[1]}, {o.ey[0], o.ey[1]}, {o.ez[0], o.ez[1]},
                                      {o.bx[0], o.bx[1]}, {o.by[0], o.by[1]}, {o.bz[0], o.bz[1]}};
#pragma unroll
                for (int f = 0; f < 6; f++) {
                    const C e = eb[f * (N / 2)];
                    eb[f * (N / 2)] = Cx<C>::make(h * (e.x + v[f][0]), h * (e.y + v[f][1]));
                }
            } else {
                to_eb(j, o);
            }
        }
        __syncthreads();
        pdl_trigger();
        if (threadIdx.x < NTF && wg0 < 6) {
            const bool valid = g < 6;
            const int gg = valid ? g : 0;
            const C* src = reinterpret_cast<const C*>(EB + gg * N);
            C* dst = reinterpret_cast<C*>(r.out_next + gg * plane + (size_t)k * N);
            row_dtt_group<M, C, V>([src](int i) { return src[i]; },
                                [dst](int q, C v) { dst[q] = v; },
                                (gg & 1) ? QS_RODFT11 : QS_REDFT11, Real(1), valid, jt, Wg, tws,
                                posts, pre);
        }
    }
    QS_TRACE_END(PRED_NEXT ? trace::K_MAP_CORR_PRED
                           : (CORRECT ? trace::K_MAP_CORR : trace::K_MAP_PRED));
}

// On the 1024-wide FP32 grid (M = 512): 512 threads at most 64 registers, two
// CTAs per SM (their shared memory, 84 KB each, fits twice).
template <int M, bool CORRECT, bool PRED_NEXT, class C = float2>
__global__ void __launch_bounds__(spec_threads<M, C>(),
                                  (M == 512 && sizeof(C) == sizeof(float2)) ? 2 : 1)
    spectral_rows_kernel(SpecArgs<typename Cx<C>::Real> a, SpecRowArgsT<typename Cx<C>::Real> r,
                         SpecArgs<typename Cx<C>::Real> an) {
    spectral_rows_body<M, CORRECT, PRED_NEXT, C>(a, r, an);
}

// The same map kernel compiled for four CTAs per SM (at most 64 registers):
// on the 512-wide FP32 grid its 512 z-mode rows then run in one wave on the
// 148 SMs, where three CTAs per SM leave 68 rows for a second one.
template <int M, bool CORRECT, bool PRED_NEXT, class C = float2>
__global__ void __launch_bounds__(spec_threads<M, C>(), 4)
    spectral_rows_wave_kernel(SpecArgs<typename Cx<C>::Real> a,
                              SpecRowArgsT<typename Cx<C>::Real> r,
                              SpecArgs<typename Cx<C>::Real> an) {
    spectral_rows_body<M, CORRECT, PRED_NEXT, C>(a, r, an);
}

template <int M, class C>
constexpr bool spec_one_wave() {
    return sizeof(C) == sizeof(float2) && M == 256;
}

template <int M, bool CORRECT, bool PRED_NEXT, class C>
constexpr auto spec_rows_fn() {
    if constexpr (spec_one_wave<M, C>()) return spectral_rows_wave_kernel<M, CORRECT, PRED_NEXT, C>;
    else return spectral_rows_kernel<M, CORRECT, PRED_NEXT, C>;
}

template <int M, class C = float2>
cudaError_t set_spec_rows_smem() {
    cudaError_t e = cudaFuncSetAttribute(spec_rows_fn<M, true, false, C>(),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)spec_rows_smem<M, C>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(spec_rows_fn<M, false, false, C>(),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)spec_rows_smem<M, C>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(spec_rows_fn<M, true, true, C>(),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)spec_rows_smem<M, C>());
    return e;
}

template <int M, class C = float2>
cudaError_t launch_spec_rows(const SpecArgs<typename Cx<C>::Real>& a,
                             const SpecRowArgsT<typename Cx<C>::Real>& r, bool correct,
                             const SpecArgs<typename Cx<C>::Real>* next, cudaStream_t st) {
    const dim3 grid((unsigned)a.nz), block(spec_threads<M, C>());
    const size_t sm = spec_rows_smem<M, C>();
    if (next)
        return launch_pdl(spec_rows_fn<M, true, true, C>(), grid, block, sm, st, a, r, *next);
    if (correct)
        return launch_pdl(spec_rows_fn<M, true, false, C>(), grid, block, sm, st, a, r, a);
    return launch_pdl(spec_rows_fn<M, false, false, C>(), grid, block, sm, st, a, r, a);
}

// The adjoints of the maps in the same arrangement (the transforms are their
// own transposes): a CTA takes z-mode row k of the six field adjoints (after
// their z-pass) through the y-pass, the corrector's (or predictor's) adjoint
// on the row's modes, one mode per thread, and for the corrector the y-pass
// of the three current adjoints.
struct AdjRowArgs {
    const float* in;      // the 6 field adjoints after the z-pass (stride `plane`)
    float* out;           // corrector: the 3 current adjoints after the y-pass
    const float2* tab;
};

// values per thread of the adjoint map kernel's row transforms: as in the
// forward map kernel, 8 on the 512-wide grid (a group is one warp and every
// thread of the CTA transforms), else those of the plain row transforms
template <int M>
__host__ __device__ constexpr int adj_vpt() {
    return M == 256 ? 8 : vpt<M>();
}

template <int M>
__host__ __device__ constexpr size_t adj_rows_smem() {
    return sizeof(float2) * (2 * (size_t)M + (size_t)kSpecGroups * (M + M / adj_vpt<M>())) +
           sizeof(float) * (6 + 3) * (size_t)(2 * M);
}

template <int M>
__host__ __device__ constexpr int adj_threads() {
    // the transform groups on the 512-wide grid (two modes per thread, four
    // CTAs per SM); elsewhere one mode per thread, at most 512 (the rest loop)
    return M == 256 ? kSpecGroups * (M / adj_vpt<M>())
           : kSpecGroups * (M / vpt<M>()) > 2 * M ? kSpecGroups * (M / vpt<M>())
                                                  : (2 * M > 512 ? 512 : 2 * M);
}

template <int M, bool CORRECT>
__device__ __forceinline__ void adjoint_rows_body(AdjSpecArgs<float> a, AdjRowArgs r) {
    using namespace adjmaps;
    constexpr int V = adj_vpt<M>();
    constexpr int T = M / V;
    constexpr int NTF = kSpecGroups * T;
    constexpr int NT = adj_threads<M>();
    constexpr int N = 2 * M;
    constexpr int LD = M + M / V;
    static_assert(NTF % 32 == 0, "transform groups fill whole warps");
    extern __shared__ float2 smem_f2[];
    float2* tws = smem_f2;
    float2* posts = tws + M;
    float2* W = posts + M;
    float* IN = reinterpret_cast<float*>(W + kSpecGroups * LD);   // 6 x N
    float* OUT = IN + 6 * N;                                       // 3 x N
    for (int i = threadIdx.x; i < M; i += NT) {
        tws[i] = r.tab[i];
        posts[i] = r.tab[2 * M + i];
    }
    const int k = blockIdx.x;
    const int g = threadIdx.x / T, jt = threadIdx.x % T;
    const int wg0 = (threadIdx.x / 32) * (32 / T);   // a warp without planes skips a transform
    float2* Wg = W + g * LD;
    const float2* pre = r.tab + M;
    const size_t plane = (size_t)N * a.nz;
    pdl_wait();
    __syncthreads();
    if (threadIdx.x < NTF && wg0 < 6) {   // y-pass of the field adjoints (y kinds C S C S C S)
        const bool valid = g < 6;
        const int gg = valid ? g : 0;
        const float2* src = reinterpret_cast<const float2*>(r.in + gg * plane + (size_t)k * N);
        float2* dst = reinterpret_cast<float2*>(IN + gg * N);
        row_dtt_group<M, float2, V>([src](int i) { return src[i]; },
                         [dst](int q, float2 v) { dst[q] = v; },
                         (gg & 1) ? QS_RODFT11 : QS_REDFT11, 1.f, valid, jt, Wg, tws, posts, pre);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < N; j += NT) {
        const size_t n = (size_t)j + (size_t)N * k;
        const float le[3] = {IN[j], IN[N + j], IN[2 * N + j]};
        const float lb[3] = {IN[3 * N + j], IN[4 * N + j], IN[5 * N + j]};
        if constexpr (CORRECT) {
            float lj[3];
            corrector_adjoint_mode(a, j, k, n, le, lb, lj);
            OUT[j] = lj[0];
            OUT[N + j] = lj[1];
            OUT[2 * N + j] = lj[2];
        } else {
            predictor_adjoint_mode(a, j, k, n, le, lb);
        }
    }
    pdl_trigger();
    if constexpr (CORRECT) {
        __syncthreads();
        if (threadIdx.x < NTF && wg0 < 3) {   // y-pass of the current adjoints (y kinds C S C)
            const bool valid = g < 3;
            const int gg = valid ? g : 0;
            const float2* src = reinterpret_cast<const float2*>(OUT + gg * N);
            float2* dst = reinterpret_cast<float2*>(r.out + gg * plane + (size_t)k * N);
            row_dtt_group<M, float2, V>([src](int i) { return src[i]; },
                             [dst](int q, float2 v) { dst[q] = v; },
                             gg == 1 ? QS_RODFT11 : QS_REDFT11, 1.f, valid, jt, Wg, tws, posts,
                             pre);
        }
    }
}

// On the 1024-wide grid (M = 512): 512 threads at most 64 registers, two CTAs
// per SM (their shared memory, 80 KB each, fits twice).
template <int M, bool CORRECT>
__global__ void __launch_bounds__(adj_threads<M>(), M == 512 ? 2 : 1)
    adjoint_rows_kernel(AdjSpecArgs<float> a, AdjRowArgs r) {
    adjoint_rows_body<M, CORRECT>(a, r);
}

// The same compiled for four CTAs per SM (at most 64 registers): the 512
// z-mode rows of the 512-wide grid in one wave on the 148 SMs.
template <int M, bool CORRECT>
__global__ void __launch_bounds__(adj_threads<M>(), 4)
    adjoint_rows_wave_kernel(AdjSpecArgs<float> a, AdjRowArgs r) {
    adjoint_rows_body<M, CORRECT>(a, r);
}

template <int M, bool CORRECT>
constexpr auto adj_rows_fn() {
    if constexpr (M == 256) return adjoint_rows_wave_kernel<M, CORRECT>;
    else return adjoint_rows_kernel<M, CORRECT>;
}

template <int M>
cudaError_t set_adj_rows_smem() {
    cudaError_t e = cudaFuncSetAttribute(adj_rows_fn<M, true>(),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)adj_rows_smem<M>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(adj_rows_fn<M, false>(),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)adj_rows_smem<M>());
    return e;
}

template <int M>
cudaError_t launch_adj_rows(const AdjSpecArgs<float>& a, const AdjRowArgs& r, bool correct,
                            cudaStream_t st) {
    const dim3 grid((unsigned)a.nz), block(adj_threads<M>());
    if (correct)
        return launch_pdl(adj_rows_fn<M, true>(), grid, block, adj_rows_smem<M>(), st, a, r);
    return launch_pdl(adj_rows_fn<M, false>(), grid, block, adj_rows_smem<M>(), st, a, r);
}

}  // namespace fft

namespace {

bool fft_size_ok(int n) { return n >= 32 && n <= 2048 && (n & (n - 1)) == 0; }

// table of one size n: tw[M] = e^{-2 pi i k/M}, pre[M] = e^{-i pi i/n},
// post[M] = e^{-i pi (i+1/4)/n}, M = n/2, built in FP64
template <class C>
std::vector<C> fft_table(int n) {
    using Real = typename fft::Cx<C>::Real;
    const int M = n / 2;
    std::vector<C> t(3 * (size_t)M);
    for (int k = 0; k < M; k++) {
        const double a = -2.0 * M_PI * k / M;
        t[k] = fft::Cx<C>::make((Real)std::cos(a), (Real)std::sin(a));
        const double b = -M_PI * k / n;
        t[M + k] = fft::Cx<C>::make((Real)std::cos(b), (Real)std::sin(b));
        const double c = -M_PI * (k + 0.25) / n;
        t[2 * M + k] = fft::Cx<C>::make((Real)std::cos(c), (Real)std::sin(c));
    }
    return t;
}

}  // namespace

DttFft::~DttFft() {
    if (tab_y) cudaFree(tab_y);
    if (tab_z && tab_z != tab_y) cudaFree(tab_z);
}

DttFft* DttFft::create(int ny, int nz) {
    if (!fft_size_ok(ny) || !fft_size_ok(nz)) return nullptr;
    auto* d = new DttFft();
    d->ny = ny;
    d->nz = nz;
    auto up = [](int n, float2** dst) {
        std::vector<float2> t = fft_table<float2>(n);
        if (cudaMalloc(dst, t.size() * sizeof(float2)) != cudaSuccess) return false;
        return cudaMemcpy(*dst, t.data(), t.size() * sizeof(float2), cudaMemcpyHostToDevice) ==
               cudaSuccess;
    };
    bool ok = up(ny, &d->tab_y);
    if (ok) {
        if (nz == ny) d->tab_z = d->tab_y;
        else ok = up(nz, &d->tab_z);
    }
    cudaError_t e = cudaSuccess;
    // the maps between the two halves of a transform (rows within one warp)
    if (ok && ny >= 128 && ny <= 1024) {
        switch (ny / 2) {
            case 512: e = fft::set_spec_rows_smem<512>(); if (e == cudaSuccess) e = fft::set_adj_rows_smem<512>(); break;
            case 256: e = fft::set_spec_rows_smem<256>(); if (e == cudaSuccess) e = fft::set_adj_rows_smem<256>(); break;
            case 128: e = fft::set_spec_rows_smem<128>(); if (e == cudaSuccess) e = fft::set_adj_rows_smem<128>(); break;
            default: e = fft::set_spec_rows_smem<64>(); if (e == cudaSuccess) e = fft::set_adj_rows_smem<64>(); break;
        }
        d->spec_rows = e == cudaSuccess;
        e = cudaSuccess;
    }
    for (int n : {ny, nz}) {
        switch (n / 2) {
            case 1024: e = fft::set_cols_smem<1024>(); break;
            case 512: e = fft::set_cols_smem<512>(); break;
            case 256: e = fft::set_cols_smem<256>(); break;
            case 128: e = fft::set_cols_smem<128>(); break;
            case 64: e = fft::set_cols_smem<64>(); break;
            case 32: e = fft::set_cols_smem<32>(); break;
            default: e = fft::set_cols_smem<16>(); break;
        }
        if (e != cudaSuccess) ok = false;
    }
    if (!ok) {
        delete d;
        return nullptr;
    }
    return d;
}

int DttFft::run_cols(int nf, const float* const* in, float* const* out, const int* kind,
                     float scale, cudaStream_t st, float* const* acc, float* const* clr) const {
    if (nf <= 0 || nf > kMaxXfFields) return 0;
    fft::ColArgs a{};
    for (int f = 0; f < nf; f++) {
        a.in[f] = in[f];
        a.out[f] = out[f];
        a.acc[f] = acc ? acc[f] : nullptr;
        a.clr[f] = clr ? clr[f] : nullptr;
        a.kind[f] = kind[f];
    }
    a.ncols = ny;
    a.scale = scale;
    a.tab = tab_z;
    cudaError_t e;
    switch (nz / 2) {
        case 1024: e = fft::launch_cols<1024>(a, nf, st); break;
        case 512: e = fft::launch_cols<512>(a, nf, st); break;
        case 256: e = fft::launch_cols<256>(a, nf, st); break;
        case 128: e = fft::launch_cols<128>(a, nf, st); break;
        case 64: e = fft::launch_cols<64>(a, nf, st); break;
        case 32: e = fft::launch_cols<32>(a, nf, st); break;
        default: e = fft::launch_cols<16>(a, nf, st); break;
    }
    return e == cudaSuccess ? 1 : 0;
}

int DttFft::run_spectral_rows(const SpecArgs<float>& a, bool correct, const float* jin,
                              float* out, int nout, cudaStream_t st,
                              const SpecArgs<float>* next, float* out_next,
                              bool avg_next) const {
    if (!spec_rows) return 0;
    if (next && (!correct || !out_next || nout != 6)) return 0;
    fft::SpecRowArgs r{};
    r.jin = jin;
    r.out = out;
    r.nout = nout;
    r.tab = tab_y;
    r.out_next = out_next;
    r.avg_next = (next && avg_next) ? 1 : 0;
    cudaError_t e;
    switch (ny / 2) {
        case 512: e = fft::launch_spec_rows<512>(a, r, correct, next, st); break;
        case 256: e = fft::launch_spec_rows<256>(a, r, correct, next, st); break;
        case 128: e = fft::launch_spec_rows<128>(a, r, correct, next, st); break;
        default: e = fft::launch_spec_rows<64>(a, r, correct, next, st); break;
    }
    return e == cudaSuccess ? 1 : 0;
}

int DttFft::run_adjoint_rows(const AdjSpecArgs<float>& a, bool correct, const float* in,
                             float* out, cudaStream_t st) const {
    if (!spec_rows) return 0;
    fft::AdjRowArgs r{};
    r.in = in;
    r.out = out;
    r.tab = tab_y;
    cudaError_t e;
    switch (ny / 2) {
        case 512: e = fft::launch_adj_rows<512>(a, r, correct, st); break;
        case 256: e = fft::launch_adj_rows<256>(a, r, correct, st); break;
        case 128: e = fft::launch_adj_rows<128>(a, r, correct, st); break;
        default: e = fft::launch_adj_rows<64>(a, r, correct, st); break;
    }
    return e == cudaSuccess ? 1 : 0;
}

int DttFft::run_pass(int pass, const DttJob<float>& job, float* scratch, cudaStream_t st) const {
    if (job.nf <= 0 || job.nf > kMaxXfFields) return 0;
    const size_t plane = (size_t)ny * nz;
    cudaError_t e = cudaSuccess;
    if (pass == 0) {   // along y: in -> scratch
        fft::RowArgs a{};
        for (int f = 0; f < job.nf; f++) {
            a.in[f] = job.in[f];
            a.out[f] = scratch + f * plane;
            a.kind[f] = job.ky[f];
        }
        a.nrows = nz;
        a.total = job.nf * nz;
        a.scale = 1.f;
        a.tab = tab_y;
        switch (ny / 2) {
            case 1024: e = fft::launch_rows<1024>(a, st); break;
            case 512: e = fft::launch_rows<512>(a, st); break;
            case 256: e = fft::launch_rows<256>(a, st); break;
            case 128: e = fft::launch_rows<128>(a, st); break;
            case 64: e = fft::launch_rows<64>(a, st); break;
            case 32: e = fft::launch_rows<32>(a, st); break;
            default: e = fft::launch_rows<16>(a, st); break;
        }
    } else {           // along z: scratch -> out, scaled
        fft::ColArgs a{};
        for (int f = 0; f < job.nf; f++) {
            a.in[f] = scratch + f * plane;
            a.out[f] = job.out[f];
            a.kind[f] = job.kz[f];
        }
        a.ncols = ny;
        a.scale = job.scale;
        a.tab = tab_z;
        switch (nz / 2) {
            case 1024: e = fft::launch_cols<1024>(a, job.nf, st); break;
            case 512: e = fft::launch_cols<512>(a, job.nf, st); break;
            case 256: e = fft::launch_cols<256>(a, job.nf, st); break;
            case 128: e = fft::launch_cols<128>(a, job.nf, st); break;
            case 64: e = fft::launch_cols<64>(a, job.nf, st); break;
            case 32: e = fft::launch_cols<32>(a, job.nf, st); break;
            default: e = fft::launch_cols<16>(a, job.nf, st); break;
        }
    }
    return e == cudaSuccess ? 1 : 0;
}

// ---------------------------------------------------------------- FP64
namespace {
bool fft64_size_ok(int n) { return n >= 32 && n <= 1024 && (n & (n - 1)) == 0; }
}  // namespace

DttFft64::~DttFft64() {
    if (tab_y) cudaFree(tab_y);
    if (tab_z && tab_z != tab_y) cudaFree(tab_z);
}

DttFft64* DttFft64::create(int ny, int nz) {
    if (!fft64_size_ok(ny) || !fft64_size_ok(nz)) return nullptr;
    auto* d = new DttFft64();
    d->ny = ny;
    d->nz = nz;
    auto up = [](int n, double2** dst) {
        std::vector<double2> t = fft_table<double2>(n);
        if (cudaMalloc(dst, t.size() * sizeof(double2)) != cudaSuccess) return false;
        return cudaMemcpy(*dst, t.data(), t.size() * sizeof(double2), cudaMemcpyHostToDevice) ==
               cudaSuccess;
    };
    bool ok = up(ny, &d->tab_y);
    if (ok) {
        if (nz == ny) d->tab_z = d->tab_y;
        else ok = up(nz, &d->tab_z);
    }
    for (int n : {ny, nz}) {
        if (!ok) break;
        cudaError_t e;
        switch (n / 2) {
            case 512: e = fft::set_cols_smem<512, double2>(); break;
            case 256: e = fft::set_cols_smem<256, double2>(); break;
            case 128: e = fft::set_cols_smem<128, double2>(); break;
            case 64: e = fft::set_cols_smem<64, double2>(); break;
            case 32: e = fft::set_cols_smem<32, double2>(); break;
            default: e = fft::set_cols_smem<16, double2>(); break;
        }
        if (e != cudaSuccess) ok = false;
    }
    if (!ok) {
        delete d;
        return nullptr;
    }
    // the map kernels between the halves: a row group must fit in one warp
    // (8 values per thread), so ny up to 512
    if (ny >= 128 && ny <= 512) {
        cudaError_t e;
        switch (ny / 2) {
            case 256: e = fft::set_spec_rows_smem<256, double2>(); break;
            case 128: e = fft::set_spec_rows_smem<128, double2>(); break;
            default: e = fft::set_spec_rows_smem<64, double2>(); break;
        }
        d->spec_rows = e == cudaSuccess;
        cudaGetLastError();
    }
    return d;
}

int DttFft64::run_cols(int nf, const double* const* in, double* const* out, const int* kind,
                       double scale, cudaStream_t st) const {
    if (nf <= 0 || nf > kMaxXfFields) return 0;
    fft::ColArgsT<double> a{};
    for (int f = 0; f < nf; f++) {
        a.in[f] = in[f];
        a.out[f] = out[f];
        a.kind[f] = kind[f];
    }
    a.ncols = ny;
    a.scale = scale;
    a.tab = tab_z;
    cudaError_t e;
    switch (nz / 2) {
        case 512: e = fft::launch_cols<512, double2>(a, nf, st); break;
        case 256: e = fft::launch_cols<256, double2>(a, nf, st); break;
        case 128: e = fft::launch_cols<128, double2>(a, nf, st); break;
        case 64: e = fft::launch_cols<64, double2>(a, nf, st); break;
        case 32: e = fft::launch_cols<32, double2>(a, nf, st); break;
        default: e = fft::launch_cols<16, double2>(a, nf, st); break;
    }
    return e == cudaSuccess ? 1 : 0;
}

int DttFft64::run_spectral_rows(const SpecArgs<double>& a, bool correct, const double* jin,
                                double* out, int nout, cudaStream_t st,
                                const SpecArgs<double>* next, double* out_next,
                                bool avg_next) const {
    if (!spec_rows) return 0;
    if (next && (!correct || !out_next || nout != 6)) return 0;
    fft::SpecRowArgsT<double> r{};
    r.jin = jin;
    r.out = out;
    r.nout = nout;
    r.tab = tab_y;
    r.out_next = out_next;
    r.avg_next = (next && avg_next) ? 1 : 0;
    cudaError_t e;
    switch (ny / 2) {
        case 256: e = fft::launch_spec_rows<256, double2>(a, r, correct, next, st); break;
        case 128: e = fft::launch_spec_rows<128, double2>(a, r, correct, next, st); break;
        default: e = fft::launch_spec_rows<64, double2>(a, r, correct, next, st); break;
    }
    return e == cudaSuccess ? 1 : 0;
}

int DttFft64::run_pass(int pass, const DttJob<double>& job, double* scratch,
                       cudaStream_t st) const {
    if (job.nf <= 0 || job.nf > kMaxXfFields) return 0;
    const size_t plane = (size_t)ny * nz;
    cudaError_t e = cudaSuccess;
    if (pass == 0) {   // along y: in -> scratch
        fft::RowArgsT<double> a{};
        for (int f = 0; f < job.nf; f++) {
            a.in[f] = job.in[f];
            a.out[f] = scratch + f * plane;
            a.kind[f] = job.ky[f];
        }
        a.nrows = nz;
        a.total = job.nf * nz;
        a.scale = 1.0;
        a.tab = tab_y;
        switch (ny / 2) {
            case 512: e = fft::launch_rows<512, double2>(a, st); break;
            case 256: e = fft::launch_rows<256, double2>(a, st); break;
            case 128: e = fft::launch_rows<128, double2>(a, st); break;
            case 64: e = fft::launch_rows<64, double2>(a, st); break;
            case 32: e = fft::launch_rows<32, double2>(a, st); break;
            default: e = fft::launch_rows<16, double2>(a, st); break;
        }
    } else {           // along z: scratch -> out, scaled
        fft::ColArgsT<double> a{};
        for (int f = 0; f < job.nf; f++) {
            a.in[f] = scratch + f * plane;
            a.out[f] = job.out[f];
            a.kind[f] = job.kz[f];
        }
        a.ncols = ny;
        a.scale = job.scale;
        a.tab = tab_z;
        switch (nz / 2) {
            case 512: e = fft::launch_cols<512, double2>(a, job.nf, st); break;
            case 256: e = fft::launch_cols<256, double2>(a, job.nf, st); break;
            case 128: e = fft::launch_cols<128, double2>(a, job.nf, st); break;
            case 64: e = fft::launch_cols<64, double2>(a, job.nf, st); break;
            case 32: e = fft::launch_cols<32, double2>(a, job.nf, st); break;
            default: e = fft::launch_cols<16, double2>(a, job.nf, st); break;
        }
    }
    return e == cudaSuccess ? 1 : 0;
}

}  // namespace qs

QS_TRACE_UNIT(fft)
