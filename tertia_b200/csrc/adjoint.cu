// adjoint.cu — reverse-mode (adjoint) kernels of the xi-march.
//
// The march maps the driver-beam currents (RhoBeam, JxBeam of every layer)
// to the fields of every layer through, per layer, a linear spectral
// predictor, inverse transforms, the plasma push with its current deposit,
// forward transforms of the currents and the linear spectral corrector
// (Mesh::MoveSplitLayer, movepart_splitlayer.cpp:561-778).  These kernels are
// the transposes of those steps; the transforms are their own transposes
// (the REDFT11 / RODFT11 matrices are symmetric), so the adjoint of a
// transform is the same transform and the adjoint of the inverse is the
// transform times 1/(4 ny nz).
//
// NGP plasma push (the reference's live shape): a particle keeps its seeded
// cell, the field gather is at that cell and the deposit cells come from
// floor() of the sub-cycled position, so positions carry no derivative; the
// adjoint state of a particle is the adjoint of its momentum.  The push
// adjoint recomputes the particle's forward update from the stored
// layer-entry state and back-propagates through it by hand.
#include <cmath>

#include "qs_common.cuh"
#include "qs_internal.h"
#include "pushmath.cuh"
#include "pdl.cuh"
#include "adjoint_maps.cuh"

namespace qs {

namespace {

template <class T>
__device__ __forceinline__ T ldg_(const T* p) { return __ldg(p); }

__device__ __forceinline__ int wrap_m(int j, int M) {
    while (j >= M) j -= M;
    while (j < 0) j += M;
    return j;
}

}  // namespace

// ---------------------------------------------------------------------------
// 1 - Vx of momentum p with inv_g = 1/gamma, and 1 - (Vxm + Vxp)/2 from the
// two: FP32 in the push kernels' cancellation-free forms (pushmath.cuh), FP64
// in the reference's expression order, as the forward ran them
template <class T>
__device__ __forceinline__ T omv(T px, T, T, T inv_g) { return T(1) - px * inv_g; }
template <>
__device__ __forceinline__ float omv<float>(float px, float py, float pz, float inv_g) {
    return one_minus_vx(px, py, pz, inv_g);
}
template <class T>
__device__ __forceinline__ T omv_mean(T vxm, T vxp, T, T) { return T(1) - T(0.5) * (vxm + vxp); }
template <>
__device__ __forceinline__ float omv_mean<float>(float, float, float omm, float omp) {
    return 0.5f * (omm + omp);
}

// push adjoint: one thread per particle
template <class T>
__global__ void __launch_bounds__(256) push_adjoint_kernel(PushAdjArgs<T> a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    pdl_wait();
    const int My = a.My, Mz = a.Mz;
    const int cell = a.cell[i];
    const int j = cell % My, k = cell / My;
    const T one = T(1), half = T(0.5);
    const T yp = a.y[i], zp = a.z[i];
    if (!(yp >= T(0) && yp <= one && zp >= T(0) && zp <= one)) return;   // forward skipped it
    const T px0 = a.px[i], py0 = a.py[i], pz0 = a.pz[i];
    const T w = a.w[i];
    const size_t plane = a.plane, n = (size_t)cell;
    T E[3], B[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        E[c] = ldg_(a.F + c * plane + n);
        B[c] = ldg_(a.F + (3 + c) * plane + n);
    }
    B[0] += a.bxe; B[1] += a.bye; B[2] += a.bze;

    // ---- forward recompute (the factored form of the push)
    const T p[3] = {px0, py0, pz0};
    const T s0 = one + p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
    const T r0 = one / sqrt(s0);
    const T Vp[3] = {p[0] * r0, p[1] * r0, p[2] * r0};
    const T av = omv(p[0], p[1], p[2], r0);
    const T ia = one / av;
    const T kE = a.sE * ia;
    const T e[3] = {E[0] * kE, E[1] * kE, E[2] * kE};
    const T p1[3] = {p[0] + e[0], p[1] + e[1], p[2] + e[2]};
    const T s1 = one + p1[0] * p1[0] + p1[1] * p1[1] + p1[2] * p1[2];
    const T r1 = one / sqrt(s1);
    const T kB = r1 * kE;
    const T b[3] = {B[0] * kB, B[1] * kB, B[2] * kB};
    const T q = one + b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
    const T co = T(2) / q;
    const T u[3] = {p1[0] + (p1[1] * b[2] - p1[2] * b[1]), p1[1] + (p1[2] * b[0] - p1[0] * b[2]),
                    p1[2] + (p1[0] * b[1] - p1[1] * b[0])};
    const T p3[3] = {u[0] * co, u[1] * co, u[2] * co};
    const T p2[3] = {p1[0] + e[0] + (p3[1] * b[2] - p3[2] * b[1]),
                     p1[1] + e[1] + (p3[2] * b[0] - p3[0] * b[2]),
                     p1[2] + e[2] + (p3[0] * b[1] - p3[1] * b[0])};
    const T s2 = one + p2[0] * p2[0] + p2[1] * p2[1] + p2[2] * p2[2];
    const T r2 = one / sqrt(s2);
    const T Vm[3] = {p2[0] * r2, p2[1] * r2, p2[2] * r2};
    const T V[3] = {half * (Vm[0] + Vp[0]), half * (Vm[1] + Vp[1]), half * (Vm[2] + Vp[2])};
    const T cv = omv_mean(Vm[0], Vp[0], omv(p2[0], p2[1], p2[2], r2), av);
    const T inv2 = one / cv;
    const T wq = w * inv2;
    const T dJ0[3] = {a.djx0, a.djy0, a.djz0};
    const T dy = V[1] * a.hxhy * inv2, dz = V[2] * a.hxhz * inv2;

    // ---- G = sum over sub-steps of part_step * lambda_J(deposit cell)
    T G[3] = {T(0), T(0), T(0)};
    {
        T partdx = T(0), step = one;
        const T ady = dy < T(0) ? -dy : dy, adz = dz < T(0) ? -dz : dz;
        if (ady > one || adz > one) step = partdx = (ady > adz ? ady : adz);
        if (partdx < one) partdx = step = one;
        T ytmp = yp, ztmp = zp;
        const T MyT = T(My), MzT = T(Mz);
        int jj = j, kk = k;
        while (partdx > T(0)) {
            T ps;
            if (partdx > one) { partdx -= one; ps = one / step; }
            else { ps = partdx / step; partdx = T(0); }
            if (a.precise) {
                const T uy = ytmp + dy * ps, uz = ztmp + dz * ps;
                const T fy = floor(uy), fz = floor(uz);
                T ry = uy - fy, rz = uz - fz;
                int sy = (int)fy, sz = (int)fz;
                if (ry >= one) { ry = T(0); sy += 1; }
                if (rz >= one) { rz = T(0); sz += 1; }
                jj = wrap_m(j + sy, My);
                kk = wrap_m(k + sz, Mz);
                ytmp = ry;
                ztmp = rz;
            } else {
                ytmp += dy * ps + T(j);
                ztmp += dz * ps + T(k);
                while (ytmp > MyT) ytmp -= MyT;
                while (ytmp < T(0)) ytmp += MyT;
                while (ztmp > MzT) ztmp -= MzT;
                while (ztmp < T(0)) ztmp += MzT;
                jj = (int)ytmp;
                kk = (int)ztmp;
                ytmp -= T(jj);
                ztmp -= T(kk);
            }
            const size_t m = (size_t)wrap_m(jj, My) + (size_t)My * wrap_m(kk, Mz);
#pragma unroll
            for (int c = 0; c < 3; c++) G[c] += ps * ldg_(a.lamD + c * plane + m);
        }
    }

    // ---- backward
    T bp2[3] = {T(0), T(0), T(0)};
    if (a.full) {
        bp2[0] = a.lamPm[i];
        bp2[1] = a.lamPm[a.n + i];
        bp2[2] = a.lamPm[2 * a.n + i];
    }
    // dj_c = wq dJ0_c Vm_c
    T bVm[3], bwq = T(0);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        bVm[c] = wq * dJ0[c] * G[c];
        bwq += G[c] * dJ0[c] * Vm[c];
    }
    const T binv2 = w * bwq;
    const T bcv = -inv2 * inv2 * binv2;
    const T bVx = -bcv;                    // cv = 1 - Vx
    bVm[0] += half * bVx;
    T bVp[3] = {half * bVx, T(0), T(0)};
    // Vm = p2 r2
    {
        const T br2 = bVm[0] * p2[0] + bVm[1] * p2[1] + bVm[2] * p2[2];
        const T f = -r2 * r2 * r2 * br2;
#pragma unroll
        for (int c = 0; c < 3; c++) bp2[c] += r2 * bVm[c] + f * p2[c];
    }
    // p2 = p1 + e + p3 x b
    T bp1[3] = {bp2[0], bp2[1], bp2[2]};
    T be[3] = {bp2[0], bp2[1], bp2[2]};
    const T bp3[3] = {b[1] * bp2[2] - b[2] * bp2[1], b[2] * bp2[0] - b[0] * bp2[2],
                      b[0] * bp2[1] - b[1] * bp2[0]};
    T bb[3] = {bp2[1] * p3[2] - bp2[2] * p3[1], bp2[2] * p3[0] - bp2[0] * p3[2],
               bp2[0] * p3[1] - bp2[1] * p3[0]};
    // p3 = co u
    const T bco = bp3[0] * u[0] + bp3[1] * u[1] + bp3[2] * u[2];
    const T bu[3] = {co * bp3[0], co * bp3[1], co * bp3[2]};
    // u = p1 + p1 x b
    bp1[0] += bu[0] + (b[1] * bu[2] - b[2] * bu[1]);
    bp1[1] += bu[1] + (b[2] * bu[0] - b[0] * bu[2]);
    bp1[2] += bu[2] + (b[0] * bu[1] - b[1] * bu[0]);
    bb[0] += bu[1] * p1[2] - bu[2] * p1[1];
    bb[1] += bu[2] * p1[0] - bu[0] * p1[2];
    bb[2] += bu[0] * p1[1] - bu[1] * p1[0];
    // co = 2 / q, q = 1 + b.b
    const T bq = -co * co * T(0.5) * bco;
#pragma unroll
    for (int c = 0; c < 3; c++) bb[c] += T(2) * b[c] * bq;
    // b = B kB
    T bB[3];
    T bkB = T(0);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        bB[c] = kB * bb[c];
        bkB += B[c] * bb[c];
    }
    // kB = r1 kE
    const T br1 = kE * bkB;
    T bkE = r1 * bkB;
    {
        const T f = -r1 * r1 * r1 * br1;
#pragma unroll
        for (int c = 0; c < 3; c++) bp1[c] += f * p1[c];
    }
    // p1 = p + e
    T bp[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        bp[c] = bp1[c];
        be[c] += bp1[c];
    }
    // e = E kE
    T bE[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        bE[c] = kE * be[c];
        bkE += E[c] * be[c];
    }
    // kE = sE / (1 - Vp_x)
    const T bia = a.sE * bkE;
    const T bav = -ia * ia * bia;
    bVp[0] += -bav;
    // Vp = p r0
    {
        const T br0 = bVp[0] * p[0] + bVp[1] * p[1] + bVp[2] * p[2];
        const T f = -r0 * r0 * r0 * br0;
#pragma unroll
        for (int c = 0; c < 3; c++) bp[c] += r0 * bVp[c] + f * p[c];
    }
    // momenta adjoint: the full push sets it, the half pushes add to it
    if (a.full) {
        a.lamPm[i] = bp[0];
        a.lamPm[a.n + i] = bp[1];
        a.lamPm[2 * a.n + i] = bp[2];
    } else {
        a.lamPm[i] += bp[0];
        a.lamPm[a.n + i] += bp[1];
        a.lamPm[2 * a.n + i] += bp[2];
    }
    // fields: E = (P + C)/2 and B = (P + C)/2 + external
#pragma unroll
    for (int c = 0; c < 3; c++) {
        atomicAdd(a.lamFC + c * plane + n, half * bE[c]);
        atomicAdd(a.lamFC + (3 + c) * plane + n, half * bB[c]);
    }
}

template <class T>
int launch_push_adjoint(const PushAdjArgs<T>& a, cudaStream_t st) {
    if (a.n <= 0) return 0;
    launch_pdl(push_adjoint_kernel<T>, dim3((unsigned)((a.n + 255) / 256)), dim3(256), 0, st, a);
    return 1;
}

// ---------------------------------------------------------------------------
// CIC push adjoint: one thread per particle.  The bilinear gather weights
// depend on the in-cell position (y, z) and the deposit weights on the
// position after the move, so besides the momentum adjoint the particle
// carries the adjoint of its position (lamPos); cells come from floor() and
// carry none.  The sub-step fractions are differentiated through the step
// length when |dy| or |dz| exceeds one cell per layer (the number of
// sub-steps is piecewise constant).  Up to kMaxSub sub-steps are followed.
constexpr int kMaxSub = 8;

// FP32 uses the forward push's fast forms (rsqrt, approximate reciprocal,
// fast divide), so that the recomputed push is the one the forward ran
template <class T>
__device__ __forceinline__ T rsq(T x) { return T(1) / sqrt(x); }
template <>
__device__ __forceinline__ float rsq<float>(float x) { return rsqrtf(x); }
template <class T>
__device__ __forceinline__ T rcp(T x) { return T(1) / x; }
template <>
__device__ __forceinline__ float rcp<float>(float x) { return rcp_approx(x); }
template <class T>
__device__ __forceinline__ T fdiv(T a, T b) { return a / b; }
template <>
__device__ __forceinline__ float fdiv<float>(float a, float b) { return __fdividef(a, b); }

// The adjoint of particle i: its momentum and position adjoints are stored,
// the adjoint of the fields it gathered (6 fields x 4 corners of its cell, as
// pairs: lf[2f] = corners 0 and 1 of field f, lf[2f + 1] = corners 2 and 3)
// goes to lf, and its cell is returned (-1, lf unset, when the forward
// skipped the particle).
// Offsets into the planes and the per-particle arrays are 32-bit (the
// adjoint's set-up checks 6 ny nz and 3 n below 2^31), so that an address is
// one wide multiply-add from its plane's base.  (j, k) of the cell is
// returned too.
// The gathered fields' y and z slopes, needed only at the end, wait in
// shared memory (sg: 12 x blockDim values, this thread's column) instead of
// 12 registers through the recompute and the backward.
template <class T>
__device__ __forceinline__ int push_adjoint_cic_one(const PushAdjArgs<T>& a, uint32_t i,
                                                    typename FPair<T>::type (&lf)[12], int& jo,
                                                    int& ko, T* sg) {
    using P = FPair<T>;
    const int My = a.My, Mz = a.Mz;
    const int cell = a.cell[i];
    int j, k;
    cell_jk(cell, My, a.invMy, j, k);
    jo = j;
    ko = k;
    const T one = T(1), half = T(0.5);
    const T yp = a.y[i], zp = a.z[i];
    if (!(yp >= T(0) && yp <= one && zp >= T(0) && zp <= one)) return -1;   // forward skipped it
    const T px0 = a.px[i], py0 = a.py[i], pz0 = a.pz[i];
    const T w = a.w[i];
    const uint32_t plane = (uint32_t)a.plane, un = (uint32_t)a.n;
    const int j1 = wrap1(j + 1, My), k1 = wrap1(k + 1, Mz);
    const uint32_t row0 = (uint32_t)My * (uint32_t)k, row1 = (uint32_t)My * (uint32_t)k1;
    const uint32_t nn[4] = {(uint32_t)j + row0, (uint32_t)j1 + row0, (uint32_t)j + row1,
                            (uint32_t)j1 + row1};
    const int tid = threadIdx.x, nt = blockDim.x;
    // the gathered fields g and their derivatives in y and z (kept instead of
    // the 24 corner values for the position adjoint of the gather)
    T g[6];
    {
        const T wg[4] = {(one - yp) * (one - zp), yp * (one - zp), (one - yp) * zp, yp * zp};
        const T* Fb = a.F;
#pragma unroll
        for (int f = 0; f < 6; f++, Fb += plane) {
            T F[4];
            g[f] = T(0);
#pragma unroll
            for (int r = 0; r < 4; r++) {
                F[r] = ldg_(Fb + nn[r]);
                g[f] += wg[r] * F[r];
            }
            sg[f * nt + tid] = (one - zp) * (F[1] - F[0]) + zp * (F[3] - F[2]);
            sg[(6 + f) * nt + tid] = (one - yp) * (F[2] - F[0]) + yp * (F[3] - F[1]);
        }
    }
    const T E[3] = {g[0], g[1], g[2]};
    const T B[3] = {g[3] + a.bxe, g[4] + a.bye, g[5] + a.bze};

    // ---- forward recompute of the push (as in push_adjoint_kernel)
    const T p[3] = {px0, py0, pz0};
    const T s0 = one + p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
    const T r0 = rsq(s0);
    const T Vp[3] = {p[0] * r0, p[1] * r0, p[2] * r0};
    const T omp = omv(p[0], p[1], p[2], r0);
    const T ia = rcp(omp);
    const T kE = a.sE * ia;
    const T e[3] = {E[0] * kE, E[1] * kE, E[2] * kE};
    const T p1[3] = {p[0] + e[0], p[1] + e[1], p[2] + e[2]};
    const T r1 = rsq(one + p1[0] * p1[0] + p1[1] * p1[1] + p1[2] * p1[2]);
    const T kB = r1 * kE;
    const T b[3] = {B[0] * kB, B[1] * kB, B[2] * kB};
    const T co = fdiv(T(2), one + b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
    const T u[3] = {p1[0] + (p1[1] * b[2] - p1[2] * b[1]), p1[1] + (p1[2] * b[0] - p1[0] * b[2]),
                    p1[2] + (p1[0] * b[1] - p1[1] * b[0])};
    const T p3[3] = {u[0] * co, u[1] * co, u[2] * co};
    const T p2[3] = {p1[0] + e[0] + (p3[1] * b[2] - p3[2] * b[1]),
                     p1[1] + e[1] + (p3[2] * b[0] - p3[0] * b[2]),
                     p1[2] + e[2] + (p3[0] * b[1] - p3[1] * b[0])};
    const T r2 = rsq(one + p2[0] * p2[0] + p2[1] * p2[1] + p2[2] * p2[2]);
    const T Vm[3] = {p2[0] * r2, p2[1] * r2, p2[2] * r2};
    const T V[3] = {half * (Vm[0] + Vp[0]), half * (Vm[1] + Vp[1]), half * (Vm[2] + Vp[2])};
    const T inv2 = rcp(omv_mean(Vm[0], Vp[0], omv(p2[0], p2[1], p2[2], r2), omp));
    const T wq = w * inv2;
    const T dJ0[3] = {a.djx0, a.djy0, a.djz0};
    const T dq[3] = {wq * dJ0[0] * Vm[0], wq * dJ0[1] * Vm[1], wq * dJ0[2] * Vm[2]};
    const T dy = V[1] * a.hxhy * inv2, dz = V[2] * a.hxhz * inv2;

    // ---- sub-steps (cell-relative moves), kept for the backward pass.  With
    // |dy| or |dz| above one cell the step is the larger of the two and each
    // sub-step's fraction ps depends on it: d ps / d step is -1/step^2 for the
    // full sub-steps and nfull/step^2 for the last one.  The first sub-step
    // stays in registers (the only one unless the particle crosses more than
    // one cell per layer), the others go to the arrays.
    T sry[kMaxSub], srz[kMaxSub], sps[kMaxSub], sdps[kMaxSub];
    int sjb[kMaxSub], skb[kMaxSub];
    T ry0 = T(0), rz0 = T(0), ps0 = T(0), dps0 = T(0);
    int jb0 = 0, kb0 = 0;
    int ns = 0;
    T dstep_dy = T(0), dstep_dz = T(0), step = one;
    {
        T partdx = T(0);
        const T ady = dy < T(0) ? -dy : dy, adz = dz < T(0) ? -dz : dz;
        if (ady > one || adz > one) {
            step = partdx = (ady > adz ? ady : adz);
            if (ady > adz) dstep_dy = dy < T(0) ? -one : one;
            else dstep_dz = dz < T(0) ? -one : one;
        }
        if (partdx < one) {
            partdx = step = one;
            dstep_dy = dstep_dz = T(0);
        }
        T ytmp = yp, ztmp = zp;
        int jb = j, kb = k;
        int nfull = 0;
        while (partdx > T(0) && ns < kMaxSub) {
            T ps, dps;
            if (partdx > one) {
                partdx -= one;
                ps = rcp(step);
                dps = -ps * ps;
                nfull++;
            } else {
                ps = fdiv(partdx, step);
                partdx = T(0);
                dps = fdiv(T(nfull), step * step);
            }
            const T uy = ytmp + dy * ps, uz = ztmp + dz * ps;
            const T fy = floor(uy), fz = floor(uz);
            T ry = uy - fy, rz = uz - fz;
            int sy = (int)fy, sz = (int)fz;
            if (ry >= one) { ry = T(0); sy += 1; }
            if (rz >= one) { rz = T(0); sz += 1; }
            jb = wrap1(jb + sy, My);     // |sy|, |sz| <= 2: a sub-step moves at most a cell
            kb = wrap1(kb + sz, Mz);
            ytmp = ry;
            ztmp = rz;
            if (ns == 0) {
                ry0 = ry; rz0 = rz; ps0 = ps; dps0 = dps; jb0 = jb; kb0 = kb;
            } else {
                sry[ns] = ry; srz[ns] = rz; sps[ns] = ps; sdps[ns] = dps;
                sjb[ns] = jb; skb[ns] = kb;
            }
            ns++;
        }
    }

    // ---- backward through the sub-steps: deposits and position chain
    T lyc = a.full ? a.lamPos[i] : T(0), lzc = a.full ? a.lamPos[un + i] : T(0);
    T ldy = T(0), ldz = T(0), lstep = T(0);
    T ldq[3] = {T(0), T(0), T(0)};
    auto back = [&](T ry, T rz, T ps, T dps, int jb, int kb) {
        T lps = T(0);
        const int jb1 = wrap1(jb + 1, My), kb1 = wrap1(kb + 1, Mz);
        const uint32_t rb0 = (uint32_t)My * (uint32_t)kb, rb1 = (uint32_t)My * (uint32_t)kb1;
        const uint32_t nd[4] = {(uint32_t)jb + rb0, (uint32_t)jb1 + rb0, (uint32_t)jb + rb1,
                                (uint32_t)jb1 + rb1};
        const T wc[4] = {(one - ry) * (one - rz), ry * (one - rz), (one - ry) * rz, ry * rz};
        T acc[4] = {T(0), T(0), T(0), T(0)};
        const T* Db = a.lamD;
#pragma unroll
        for (int d = 0; d < 3; d++, Db += plane) {
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const T G = ldg_(Db + nd[r]);
                ldq[d] += ps * wc[r] * G;
                acc[r] += dq[d] * G;
            }
        }
        T lwc[4];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            lwc[r] = ps * acc[r];
            lps += wc[r] * acc[r];
        }
        const T lry = lyc + (one - rz) * (lwc[1] - lwc[0]) + rz * (lwc[3] - lwc[2]);
        const T lrz = lzc + (one - ry) * (lwc[2] - lwc[0]) + ry * (lwc[3] - lwc[1]);
        ldy += lry * ps;
        ldz += lrz * ps;
        lps += lry * dy + lrz * dz;      // u = y + d ps
        lstep += lps * dps;
        lyc = lry;      // the position before this sub-step
        lzc = lrz;
    };
    for (int q = ns - 1; q >= 1; q--) back(sry[q], srz[q], sps[q], sdps[q], sjb[q], skb[q]);
    if (ns > 0) back(ry0, rz0, ps0, dps0, jb0, kb0);
    T lyp = lyc, lzp = lzc;
    ldy += lstep * dstep_dy;
    ldz += lstep * dstep_dz;

    // ---- backward through the push
    T bp2[3] = {T(0), T(0), T(0)};
    if (a.full) {
        bp2[0] = a.lamPm[i];
        bp2[1] = a.lamPm[un + i];
        bp2[2] = a.lamPm[2 * un + i];
    }
    T bVm[3], bwq = T(0);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        bVm[c] = wq * dJ0[c] * ldq[c];
        bwq += ldq[c] * dJ0[c] * Vm[c];
    }
    // dy = Vy hxhy inv2, dz = Vz hxhz inv2
    const T bVy = ldy * a.hxhy * inv2, bVz = ldz * a.hxhz * inv2;
    const T binv2 = w * bwq + ldy * V[1] * a.hxhy + ldz * V[2] * a.hxhz;
    const T bVx = inv2 * inv2 * binv2;    // inv2 = 1/(1 - Vx)
    const T bV[3] = {bVx, bVy, bVz};
    T bVp[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        bVm[c] += half * bV[c];
        bVp[c] = half * bV[c];
    }
    {
        const T br2 = bVm[0] * p2[0] + bVm[1] * p2[1] + bVm[2] * p2[2];
        const T f = -r2 * r2 * r2 * br2;
#pragma unroll
        for (int c = 0; c < 3; c++) bp2[c] += r2 * bVm[c] + f * p2[c];
    }
    T bp1[3] = {bp2[0], bp2[1], bp2[2]};
    T be[3] = {bp2[0], bp2[1], bp2[2]};
    const T bp3[3] = {b[1] * bp2[2] - b[2] * bp2[1], b[2] * bp2[0] - b[0] * bp2[2],
                      b[0] * bp2[1] - b[1] * bp2[0]};
    T bb[3] = {bp2[1] * p3[2] - bp2[2] * p3[1], bp2[2] * p3[0] - bp2[0] * p3[2],
               bp2[0] * p3[1] - bp2[1] * p3[0]};
    const T bco = bp3[0] * u[0] + bp3[1] * u[1] + bp3[2] * u[2];
    const T bu[3] = {co * bp3[0], co * bp3[1], co * bp3[2]};
    bp1[0] += bu[0] + (b[1] * bu[2] - b[2] * bu[1]);
    bp1[1] += bu[1] + (b[2] * bu[0] - b[0] * bu[2]);
    bp1[2] += bu[2] + (b[0] * bu[1] - b[1] * bu[0]);
    bb[0] += bu[1] * p1[2] - bu[2] * p1[1];
    bb[1] += bu[2] * p1[0] - bu[0] * p1[2];
    bb[2] += bu[0] * p1[1] - bu[1] * p1[0];
    const T bq = -co * co * T(0.5) * bco;
#pragma unroll
    for (int c = 0; c < 3; c++) bb[c] += T(2) * b[c] * bq;
    T bB[3];
    T bkB = T(0);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        bB[c] = kB * bb[c];
        bkB += B[c] * bb[c];
    }
    const T br1 = kE * bkB;
    T bkE = r1 * bkB;
    {
        const T f = -r1 * r1 * r1 * br1;
#pragma unroll
        for (int c = 0; c < 3; c++) bp1[c] += f * p1[c];
    }
    T bp[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        bp[c] = bp1[c];
        be[c] += bp1[c];
    }
    T bE[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        bE[c] = kE * be[c];
        bkE += E[c] * be[c];
    }
    const T bia = a.sE * bkE;
    bVp[0] += ia * ia * bia;              // ia = 1/(1 - Vp_x)
    {
        const T br0 = bVp[0] * p[0] + bVp[1] * p[1] + bVp[2] * p[2];
        const T f = -r0 * r0 * r0 * br0;
#pragma unroll
        for (int c = 0; c < 3; c++) bp[c] += r0 * bVp[c] + f * p[c];
    }
    // ---- backward through the gather g_f = sum_r wg_r F_f,r
    const T bg[6] = {bE[0], bE[1], bE[2], bB[0], bB[1], bB[2]};
    const auto w01 = P::make((one - yp) * (one - zp), yp * (one - zp));
    const auto w23 = P::make((one - yp) * zp, yp * zp);
#pragma unroll
    for (int f = 0; f < 6; f++) {
        lyp += bg[f] * sg[f * nt + tid];
        lzp += bg[f] * sg[(6 + f) * nt + tid];
        const T hb = half * bg[f];
        lf[2 * f] = P::mul(hb, w01);
        lf[2 * f + 1] = P::mul(hb, w23);
    }
    if (a.full) {
        a.lamPm[i] = bp[0];
        a.lamPm[un + i] = bp[1];
        a.lamPm[2 * un + i] = bp[2];
        a.lamPos[i] = lyp;
        a.lamPos[un + i] = lzp;
    } else {
        a.lamPm[i] += bp[0];
        a.lamPm[un + i] += bp[1];
        a.lamPm[2 * un + i] += bp[2];
        a.lamPos[i] += lyp;
        a.lamPos[un + i] += lzp;
    }
    return cell;
}

// Sums of v over runs of lanes with equal key (the particles of a warp are
// grouped by cell): the first lane of each run gets its run's sum and true.
// The values are pairs (two shuffles, one packed add in FP32).
template <int NV, class V>
__device__ __forceinline__ bool warp_run_sums(V (&v)[NV], int key) {
    using P = FPair<decltype(v[0].x)>;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int prevKey = __shfl_up_sync(full, key, 1);
    const unsigned starts = __ballot_sync(full, lane == 0 || prevKey != key);
    const int rs = 31 - __clz(starts & (0xffffffffu >> (31 - lane)));   // run start
    const unsigned after = starts & ~(0xffffffffu >> (31 - lane));       // starts > lane
    const int re = after ? __ffs(after) - 2 : 31;                        // run end
    const int maxrun = (int)__reduce_max_sync(full, key >= 0 ? (unsigned)(re - rs + 1) : 1u);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        if (maxrun > d) {   // the same for every lane
            const bool take = lane + d <= re && ((lane - rs) & (2 * d - 1)) == 0;
#pragma unroll
            for (int q = 0; q < NV; q++) {
                V o;
                o.x = __shfl_down_sync(full, v[q].x, d);
                o.y = __shfl_down_sync(full, v[q].y, d);
                if (take) v[q] = P::add(v[q], o);
            }
        }
    }
    return key >= 0 && lane == rs;
}

// FP32: 4 blocks per SM (64 registers and a few spills; the latency of the
// gathers hidden by more warps, measured faster than 2 or 3 blocks); FP64 as
// many registers as it takes
template <class T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 1)
    push_adjoint_cic_kernel(PushAdjArgs<T> a) {
    __shared__ T sg[12 * 256];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    pdl_wait();
    typename FPair<T>::type lf[12];
    int j = 0, k = 0;
    const int cell = i < (uint32_t)a.n ? push_adjoint_cic_one(a, i, lf, j, k, sg) : -1;
    if (cell < 0) {
#pragma unroll
        for (int q = 0; q < 12; q++) lf[q] = FPair<T>::make(T(0), T(0));
    }
    // the field adjoints of a cell's particles summed in the warp, then one
    // atomic per field and corner
    if (warp_run_sums<12>(lf, cell)) {
        const int My = a.My, Mz = a.Mz;
        const uint32_t plane = (uint32_t)a.plane;
        const int j1 = wrap1(j + 1, My), k1 = wrap1(k + 1, Mz);
        const uint32_t row0 = (uint32_t)My * (uint32_t)k, row1 = (uint32_t)My * (uint32_t)k1;
        const uint32_t nn[4] = {(uint32_t)j + row0, (uint32_t)j1 + row0, (uint32_t)j + row1,
                                (uint32_t)j1 + row1};
        T* Lb = a.lamFC;
#pragma unroll
        for (int f = 0; f < 6; f++, Lb += plane) {
            atomicAdd(Lb + nn[0], lf[2 * f].x);
            atomicAdd(Lb + nn[1], lf[2 * f].y);
            atomicAdd(Lb + nn[2], lf[2 * f + 1].x);
            atomicAdd(Lb + nn[3], lf[2 * f + 1].y);
        }
    }
}

template <class T>
int launch_push_adjoint_cic(const PushAdjArgs<T>& a, cudaStream_t st) {
    if (a.n <= 0) return 0;
    launch_pdl(push_adjoint_cic_kernel<T>, dim3((unsigned)((a.n + 255) / 256)), dim3(256), 0, st,
               a);
    return 1;
}

__global__ void invert_ids_kernel(const int32_t* __restrict__ id, int64_t n,
                                  int32_t* __restrict__ inv) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) {
        const int32_t v = id[p];
        if (v >= 0 && v < n) inv[v] = (int32_t)p;
    }
}

template <class T>
__global__ void permute_kernel(const int32_t* __restrict__ id_to, const int32_t* __restrict__ inv,
                               int64_t n, const T* __restrict__ src, T* __restrict__ dst,
                               int narr) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int32_t v = id_to[q];
    const int32_t p = (v >= 0 && v < n) ? inv[v] : -1;
    for (int c = 0; c < narr; c++)
        dst[(size_t)c * n + q] = (p >= 0 && p < n) ? src[(size_t)c * n + p] : T(0);
}

template <class T>
int launch_permute_adjoint(const int32_t* id_from, const int32_t* id_to, int64_t n, int32_t* inv,
                           const T* src, T* dst, int narr, cudaStream_t st) {
    if (n <= 0) return 0;
    const unsigned g = (unsigned)((n + 255) / 256);
    invert_ids_kernel<<<g, 256, 0, st>>>(id_from, n, inv);
    permute_kernel<T><<<g, 256, 0, st>>>(id_to, inv, n, src, dst, narr);
    return 2;
}

// ---------------------------------------------------------------------------
// per-mode adjoints of the spectral maps

template <class T>
__global__ void corrector_adjoint_kernel(AdjSpecArgs<T> a) {
    using namespace adjmaps;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (j >= a.ny) return;
    pdl_wait();
    const size_t n = (size_t)j + (size_t)a.ny * k;
    const T le[3] = {opt(a.lE[0], n), opt(a.lE[1], n), opt(a.lE[2], n)};
    const T lb[3] = {opt(a.lB[0], n), opt(a.lB[1], n), opt(a.lB[2], n)};
    T lj[3];
    corrector_adjoint_mode(a, j, k, n, le, lb, lj);
    a.lJ[0][n] = lj[0];
    a.lJ[1][n] = lj[1];
    a.lJ[2][n] = lj[2];
}

template <class T>
__global__ void predictor_adjoint_kernel(AdjSpecArgs<T> a) {
    using namespace adjmaps;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (j >= a.ny) return;
    pdl_wait();
    const size_t n = (size_t)j + (size_t)a.ny * k;
    const T le[3] = {opt(a.lE[0], n), opt(a.lE[1], n), opt(a.lE[2], n)};
    const T lb[3] = {opt(a.lB[0], n), opt(a.lB[1], n), opt(a.lB[2], n)};
    predictor_adjoint_mode(a, j, k, n, le, lb);
}

template <class T>
int launch_corrector_adjoint(const AdjSpecArgs<T>& a, cudaStream_t st) {
    const dim3 g((unsigned)((a.ny + 127) / 128), (unsigned)a.nz);
    launch_pdl(corrector_adjoint_kernel<T>, g, dim3(128), 0, st, a);
    return 1;
}

template <class T>
int launch_predictor_adjoint(const AdjSpecArgs<T>& a, cudaStream_t st) {
    const dim3 g((unsigned)((a.ny + 127) / 128), (unsigned)a.nz);
    launch_pdl(predictor_adjoint_kernel<T>, g, dim3(128), 0, st, a);
    return 1;
}

// ---------------------------------------------------------------------------
// acc += x over n values (the P-field adjoint gathers every push's share)
template <class T>
__global__ void add_planes_kernel(T* __restrict__ acc, const T* __restrict__ x, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pdl_wait();
    acc[i] += x[i];
}

template <class T>
int launch_add_planes(T* acc, const T* x, size_t n, cudaStream_t st) {
    if (!n) return 0;
    launch_pdl(add_planes_kernel<T>, dim3((unsigned)((n + 255) / 256)), dim3(256), 0, st, acc, x,
               n);
    return 1;
}

// out = (P + C) / 2, the push's gathered fields (the same expression as the
// push, so the adjoint recomputes the push the forward ran)
template <class T>
__global__ void avg_planes_kernel(const T* __restrict__ P, const T* __restrict__ C,
                                  T* __restrict__ out, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pdl_wait();
    out[i] = T(0.5) * (P[i] + C[i]);
}

template <class T>
int launch_avg_planes(const T* P, const T* C, T* out, size_t n, cudaStream_t st) {
    if (!n) return 0;
    launch_pdl(avg_planes_kernel<T>, dim3((unsigned)((n + 255) / 256)), dim3(256), 0, st, P, C,
               out, n);
    return 1;
}

// ---------------------------------------------------------------------------
// out[idx] += v[layer] for the on-axis loss gradient of one layer
template <class T>
__global__ void add_point_kernel(T* plane_ex, size_t idx, const T* v, int layer) {
    if (threadIdx.x == 0 && blockIdx.x == 0) plane_ex[idx] += v[layer];
}

template <class T>
int launch_add_point(T* plane_ex, size_t idx, const T* v, int layer, cudaStream_t st) {
    add_point_kernel<T><<<1, 32, 0, st>>>(plane_ex, idx, v, layer);
    return 1;
}

// ---------------------------------------------------------------------------
// d loss / d w_p of every beam particle: the transpose of the 3-D CIC deposit
// of the last beam push (movebeam.cpp:662-774): drho = w polarity,
// djx = w polarity Vx at the 8 corners of the particle's post-push cell.
template <class T>
__global__ void __launch_bounds__(256) beam_weight_grad_kernel(BeamGradArgs<T> a) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const int L = a.L, My = a.My, Mz = a.Mz;
    const int i = a.bi[p], j = a.bj[p], k = a.bk[p];
    double g = 0.0;
    if (i >= 0 && i < L && j >= 0 && j < My && k >= 0 && k < Mz) {
        const double px = a.px[p], py = a.py[p], pz = a.pz[p];
        const double Vx = px / sqrt(1. + px * px + py * py + pz * pz);
        const double ax1 = a.x[p], ax0 = 1. - ax1, ay1 = a.y[p], ay0 = 1. - ay1, az1 = a.z[p],
                     az0 = 1. - az1;
        const size_t plane = a.plane;
        for (int di = 0; di < 2; di++)
            for (int dj = 0; dj < 2; dj++)
                for (int dk = 0; dk < 2; dk++) {
                    const int ii = i + di, jj = j + dj, kk = k + dk;
                    if (ii > L || ii < a.lo || jj >= My || kk >= Mz) continue;   // zero below lo
                    const double wc = (di ? ax1 : ax0) * (dj ? ay1 : ay0) * (dk ? az1 : az0);
                    const size_t m = (size_t)jj + (size_t)My * kk;
                    const size_t l = (size_t)(ii - a.lo);
                    g += wc * ((double)a.lb3[(l * 2 + 0) * plane + m] +
                               Vx * (double)a.lb3[(l * 2 + 1) * plane + m]);
                }
    }
    a.out[p] = g * a.polarity;
}

template <class T>
int launch_beam_weight_grad(const BeamGradArgs<T>& a, cudaStream_t st) {
    if (a.n <= 0) return 0;
    beam_weight_grad_kernel<T><<<(unsigned)((a.n + 255) / 256), 256, 0, st>>>(a);
    return 1;
}

template <class T>
__global__ void __launch_bounds__(256) save_state_kernel(StateCopy<T> c) {
    pdl_wait();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < c.n;
         i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int q = 0; q < 5; q++) c.dst[q][i] = c.src[q][i];
        if (c.csrc) c.cdst[i] = c.csrc[i];
    }
}

template <class T>
int launch_save_state(const StateCopy<T>& c, cudaStream_t st) {
    if (c.n <= 0) return 0;
    const int64_t blocks = std::min<int64_t>((c.n + 255) / 256, 148 * 8);
    launch_pdl(save_state_kernel<T>, dim3((unsigned)blocks), dim3(256), 0, st, c);
    return 1;
}

#define QS_ADJ_INST(T)                                                                   \
    template int launch_push_adjoint<T>(const PushAdjArgs<T>&, cudaStream_t);            \
    template int launch_push_adjoint_cic<T>(const PushAdjArgs<T>&, cudaStream_t);        \
    template int launch_permute_adjoint<T>(const int32_t*, const int32_t*, int64_t,      \
                                           int32_t*, const T*, T*, int, cudaStream_t);   \
    template int launch_corrector_adjoint<T>(const AdjSpecArgs<T>&, cudaStream_t);       \
    template int launch_predictor_adjoint<T>(const AdjSpecArgs<T>&, cudaStream_t);       \
    template int launch_add_point<T>(T*, size_t, const T*, int, cudaStream_t);           \
    template int launch_add_planes<T>(T*, const T*, size_t, cudaStream_t);               \
    template int launch_avg_planes<T>(const T*, const T*, T*, size_t, cudaStream_t);     \
    template int launch_save_state<T>(const StateCopy<T>&, cudaStream_t);                \
    template int launch_beam_weight_grad<T>(const BeamGradArgs<T>&, cudaStream_t);
QS_ADJ_INST(float)
QS_ADJ_INST(double)

}  // namespace qs
