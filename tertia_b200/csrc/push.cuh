// push.cu — plasma macro-particle push across one xi-layer with current /
// density deposit (reference Mesh::MoveParticlesLayerSplit,
// movepart_splitlayer.cpp:781-1544, DepositCurrentsInCellSplit :1547-1655,
// ExchangeCurrentsSplit :1685-1711; dead GPU twin cuMoveSplitParticles,
// plasma_particles.cu:72-863).
//
// Layout: particles are SoA (y, z, px, py, pz, w, cell) grouped by cell in
// ascending cell order, one thread per particle.  In the reference's live
// NGP path a particle never leaves its seeded cell (the full-step relink at
// :1507 uses the outer jtmp = j), so the grouping is permanent and the 4-8
// particles of a cell sit in consecutive lanes: their deposits are summed
// with a warp-segmented reduction over runs of equal destination cell and a
// single lane per run issues the global atomics.  The guard-ring fold of
// ExchangeCurrentsSplit is done by depositing at (j mod My, k mod Mz).
//
// The FP64 kernel (push_f64.cu, compiled with -fmad=false) follows the
// reference's expression order without contraction and reproduces the oracle
// bit for bit on identical inputs, cell indices included.  The FP32 kernel
// (push_f32.cu) uses the same physics with the divisions factored into six
// reciprocals and FMA contraction allowed: it is instruction bound, not
// memory bound, and this halves its instruction count.
#pragma once
#include "qs_common.cuh"
#include "qs_internal.h"
#include "pdl.cuh"
#include "pushmath.cuh"
#include "trace.cuh"

namespace qs {

template <class T>
__device__ __forceinline__ T ld(const T* p) { return __ldg(p); }

template <class T>
__device__ __forceinline__ T sqrt_t(T x);
template <>
__device__ __forceinline__ float sqrt_t<float>(float x) { return __fsqrt_rn(x); }
template <>
__device__ __forceinline__ double sqrt_t<double>(double x) { return __dsqrt_rn(x); }

template <class T>
__device__ __forceinline__ T floor_t(T x);
template <>
__device__ __forceinline__ float floor_t<float>(float x) { return floorf(x); }
template <>
__device__ __forceinline__ double floor_t<double>(double x) { return floor(x); }

template <class T>
__device__ __forceinline__ T fabs_t(T x) { return x < T(0) ? -x : x; }

__device__ __forceinline__ int wrap_idx(int j, int M) {
    // shifts are small (|shift| <= a few cells): avoid the integer modulo
    while (j >= M) j -= M;
    while (j < 0) j += M;
    return j;
}


// Sub-cycled transverse move and deposit of one particle (:1389-1479 with
// DepositCurrentsInCellSplit :1547-1615 or the CIC of MoveInCell), then the
// full-step store (:1501-1512).  The first sub-step's deposit is returned in
// (key, v) for the warp-level reduction; later sub-steps deposit directly.
template <class T, int SHAPE, bool PRECISE, int NV>
__device__ __forceinline__ void move_and_deposit(const PushArgs<T>& a, int64_t i, int j, int k,
                                                 T yp, T zp, T px, T py, T pz, T djx, T djy,
                                                 T djz, T drho, T dy, T dz, int& key, T (&v)[NV]) {
    const T one = T(1);
    const int My = a.My, Mz = a.Mz;
    const size_t plane = a.plane;
    T partdx = T(0), step = one;
    if (fabs_t(dy) > one || fabs_t(dz) > one) {
        if (fabs_t(dy) > fabs_t(dz)) step = partdx = fabs_t(dy);
        else step = partdx = fabs_t(dz);
    }
    if (partdx < one) partdx = step = one;
    const T MyT = T(My), MzT = T(Mz);
    T ytmp = yp, ztmp = zp;
    int jb = j, kb = k, jj = j, kk = k;
    bool first = true;
    while (partdx > T(0)) {
        T part_step;
        if (partdx > one) {
            partdx -= one;
            part_step = one / step;
        } else {
            part_step = partdx / step;
            partdx = T(0);
        }
        if (SHAPE == QS_SHAPE_NGP && !PRECISE) {
            // reference form (:1420-1437); the added j is the outer j_jump
            ytmp += dy * part_step + T(j);
            ztmp += dz * part_step + T(k);
            while (ytmp > MyT) ytmp -= MyT;
            while (ytmp < T(0)) ytmp += MyT;
            while (ztmp > MzT) ztmp -= MzT;
            while (ztmp < T(0)) ztmp += MzT;
            jj = (int)ytmp;
            kk = (int)ztmp;
            ytmp -= T(jj);
            ztmp -= T(kk);
        } else {
            const T uy = ytmp + dy * part_step;
            const T uz = ztmp + dz * part_step;
            const T fy = floor_t<T>(uy), fz = floor_t<T>(uz);
            T ry = uy - fy, rz = uz - fz;
            int sy = (int)fy, sz = (int)fz;
            if (ry >= one) { ry = T(0); sy += 1; }
            if (rz >= one) { rz = T(0); sz += 1; }
            const int bj = (SHAPE == QS_SHAPE_NGP) ? j : jb;
            const int bk = (SHAPE == QS_SHAPE_NGP) ? k : kb;
            jj = wrap_idx(bj + sy, My);
            kk = wrap_idx(bk + sz, Mz);
            ytmp = ry;
            ztmp = rz;
            jb = jj;
            kb = kk;
        }
        const T s = part_step;
        const int fj = wrap_idx(jj, My), fk = wrap_idx(kk, Mz);
        if (SHAPE == QS_SHAPE_NGP) {
            const T d0 = djx * s, d1 = djy * s, d2 = djz * s, d3 = drho * s;
            if (first) {
                key = fj + My * fk;
                v[0] = d0; v[1] = d1; v[2] = d2; v[3] = d3;
            } else {
                const size_t n = (size_t)fj + (size_t)My * fk;
                atomicAdd(a.dep + 0 * plane + n, d0);
                atomicAdd(a.dep + 1 * plane + n, d1);
                atomicAdd(a.dep + 2 * plane + n, d2);
                atomicAdd(a.dep + 3 * plane + n, d3);
            }
        } else {
            const T ayp = ytmp, ayc = one - ayp, azp = ztmp, azc = one - azp;
            const T w00 = ayc * azc, w10 = ayp * azc, w01 = ayc * azp, w11 = ayp * azp;
            const T q[4] = {djx * s, djy * s, djz * s, drho * s};
            const T wc[4] = {w00, w10, w01, w11};
            if (first) {
                key = fj + My * fk;
#pragma unroll
                for (int cnr = 0; cnr < 4; cnr++)
#pragma unroll
                    for (int qq = 0; qq < 4; qq++) v[cnr * 4 + qq] = q[qq] * wc[cnr];
            } else {
                const int j1 = wrap_idx(fj + 1, My), k1 = wrap_idx(fk + 1, Mz);
                const size_t nn[4] = {(size_t)fj + (size_t)My * fk,
                                      (size_t)j1 + (size_t)My * fk,
                                      (size_t)fj + (size_t)My * k1,
                                      (size_t)j1 + (size_t)My * k1};
#pragma unroll
                for (int cnr = 0; cnr < 4; cnr++)
#pragma unroll
                    for (int qq = 0; qq < 4; qq++)
                        atomicAdd(a.dep + qq * plane + nn[cnr], q[qq] * wc[cnr]);
            }
        }
        first = false;
    }
    const int jf = wrap_idx(jj, My), kf = wrap_idx(kk, Mz);
    if (a.dep_cell) a.dep_cell[i] = jf + My * kf;
    if (a.full) {
        a.px[i] = px;
        a.py[i] = py;
        a.pz[i] = pz;
        a.y[i] = ytmp;
        a.z[i] = ztmp;
        if (SHAPE == QS_SHAPE_CIC) a.cell_out[i] = jf + My * kf;
    }
}

// SHAPE: QS_SHAPE_NGP / QS_SHAPE_CIC.  PRECISE: cell-relative position
// update (u = frac + d*part_step measured from the base cell) instead of the
// reference's ytmp + j form; the FP32 kernels use it to keep the in-cell
// fraction at full float precision.
template <class T, int SHAPE, bool PRECISE, bool FAST>
__global__ void __launch_bounds__(256) push_kernel(PushArgs<T> a) {
    constexpr int NV = (SHAPE == QS_SHAPE_NGP) ? 4 : 16;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int My = a.My, Mz = a.Mz;
    int key = -1;          // base cell of the first sub-step deposit
    T v[NV];
#pragma unroll
    for (int c = 0; c < NV; c++) v[c] = T(0);

    if (i < a.n) {
        const T one = T(1), two = T(2), half = T(0.5);
        const int cell = a.cell[i];
        int j, k;
        if (FAST) cell_jk(cell, My, a.invMy, j, k);
        else { j = cell % My; k = cell / My; }
        const T yp = a.y[i], zp = a.z[i];
        T px = a.px[i], py = a.py[i], pz = a.pz[i];
        const T weight = a.w[i];
        if (!(yp >= T(0) && yp <= one && zp >= T(0) && zp <= one)) {
            atomicOr(a.err, DEV_ERR_RANGE);
        } else {
            if constexpr (FAST) {
            // ---- FP32: the same update with the divisions factored out, and
            // 1 - Vx in its cancellation-free form (pushmath.cuh)
            const T inv_gp = one / sqrt_t<T>(one + px * px + py * py + pz * pz);
            const T Vxp = px * inv_gp, Vyp = py * inv_gp, Vzp = pz * inv_gp;
            const T q2m = a.q2m;
            const size_t plane = a.plane;
            T ex, ey, ez, bx, by, bz;
            if (SHAPE == QS_SHAPE_NGP) {
                const size_t n = (size_t)cell;
                ex = half * (ld(a.P + 0 * plane + n) + ld(a.C + 0 * plane + n));
                ey = half * (ld(a.P + 1 * plane + n) + ld(a.C + 1 * plane + n));
                ez = half * (ld(a.P + 2 * plane + n) + ld(a.C + 2 * plane + n));
                bx = half * (ld(a.P + 3 * plane + n) + ld(a.C + 3 * plane + n));
                by = half * (ld(a.P + 4 * plane + n) + ld(a.C + 4 * plane + n));
                bz = half * (ld(a.P + 5 * plane + n) + ld(a.C + 5 * plane + n));
            } else {
                const T ayc = one - yp, ayp = yp, azc = one - zp, azp = zp;
                const T acc = ayc * azc, apc = ayp * azc, acp = ayc * azp, app = ayp * azp;
                const int j1 = wrap_idx(j + 1, My), k1 = wrap_idx(k + 1, Mz);
                const size_t n00 = (size_t)j + (size_t)My * k, n10 = (size_t)j1 + (size_t)My * k,
                             n01 = (size_t)j + (size_t)My * k1, n11 = (size_t)j1 + (size_t)My * k1;
                T g[6];
#pragma unroll
                for (int c = 0; c < 6; c++) {
                    const T* Pc = a.P + c * plane;
                    const T* Cc = a.C + c * plane;
                    T vp = acc * ld(Pc + n00) + apc * ld(Pc + n10) + acp * ld(Pc + n01) +
                           app * ld(Pc + n11);
                    T vc = acc * ld(Cc + n00) + apc * ld(Cc + n10) + acp * ld(Cc + n01) +
                           app * ld(Cc + n11);
                    g[c] = half * (vp + vc);
                }
                ex = g[0]; ey = g[1]; ez = g[2]; bx = g[3]; by = g[4]; bz = g[5];
            }
            const T omp = one_minus_vx(px, py, pz, inv_gp);   // 1 - Vx before the kick
            const T inv1 = one / omp;
            const T kE = a.sE * inv1;                 // q2m*hx/2 / (1 - Vx)
            ex *= kE;
            ey *= kE;
            ez *= kE;
            px += ex;
            py += ey;
            pz += ez;
            const T gamma_r = one / sqrt_t<T>(one + px * px + py * py + pz * pz);
            const T kB = gamma_r * kE;               // gamma_r*q2m/(1-Vx)*hx/2
            bx = (bx + a.bxe) * kB;
            by = (by + a.bye) * kB;
            bz = (bz + a.bze) * kB;
            const T co = two / (one + bx * bx + by * by + bz * bz);
            const T p3x = (py * bz - pz * by + px) * co;
            const T p3y = (pz * bx - px * bz + py) * co;
            const T p3z = (px * by - py * bx + pz) * co;
            px += ex + (p3y * bz - p3z * by);
            py += ey + (p3z * bx - p3x * bz);
            pz += ez + (p3x * by - p3y * bx);
            const T inv_g = one / sqrt_t<T>(one + px * px + py * py + pz * pz);
            const T Vxm = px * inv_g, Vym = py * inv_g, Vzm = pz * inv_g;
            const T Vy = half * (Vym + Vyp);
            const T Vz = half * (Vzm + Vzp);
            // 1 - (Vxm + Vxp)/2 = ((1 - Vxm) + (1 - Vxp))/2
            const T inv2 = one / (half * (one_minus_vx(px, py, pz, inv_g) + omp));
            const T wq = weight * inv2;
            const T djx = wq * a.djx0 * Vxm;
            const T djy = wq * a.djy0 * Vym;
            const T djz = wq * a.djz0 * Vzm;
            const T drho = wq * a.drho0;
            const T dy = Vy * a.hxhy * inv2;
            const T dz = Vz * a.hxhz * inv2;
            move_and_deposit<T, SHAPE, PRECISE, NV>(a, i, j, k, yp, zp, px, py, pz, djx, djy, djz,
                                                   drho, dy, dz, key, v);
            } else {
            T gammap = sqrt_t<T>(one + px * px + py * py + pz * pz);
            T Vx = px / gammap;
            const T Vxp = Vx, Vyp = py / gammap, Vzp = pz / gammap;
            const T q2m = a.q2m;
            const size_t plane = a.plane;
            T ex, ey, ez, bx, by, bz;
            if (SHAPE == QS_SHAPE_NGP) {
                const size_t n = (size_t)cell;
                ex = half * (ld(a.P + 0 * plane + n) + ld(a.C + 0 * plane + n));
                ey = half * (ld(a.P + 1 * plane + n) + ld(a.C + 1 * plane + n));
                ez = half * (ld(a.P + 2 * plane + n) + ld(a.C + 2 * plane + n));
                bx = half * (ld(a.P + 3 * plane + n) + ld(a.C + 3 * plane + n));
                by = half * (ld(a.P + 4 * plane + n) + ld(a.C + 4 * plane + n));
                bz = half * (ld(a.P + 5 * plane + n) + ld(a.C + 5 * plane + n));
            } else {
                const T ayc = one - yp, ayp = yp, azc = one - zp, azp = zp;
                const T acc = ayc * azc, apc = ayp * azc, acp = ayc * azp, app = ayp * azp;
                const int j1 = wrap_idx(j + 1, My), k1 = wrap_idx(k + 1, Mz);
                const size_t n00 = (size_t)j + (size_t)My * k, n10 = (size_t)j1 + (size_t)My * k,
                             n01 = (size_t)j + (size_t)My * k1, n11 = (size_t)j1 + (size_t)My * k1;
                T g[6];
#pragma unroll
                for (int c = 0; c < 6; c++) {
                    const T* Pc = a.P + c * plane;
                    const T* Cc = a.C + c * plane;
                    T vp = acc * ld(Pc + n00) + apc * ld(Pc + n10) + acp * ld(Pc + n01) +
                           app * ld(Pc + n11);
                    T vc = acc * ld(Cc + n00) + apc * ld(Cc + n10) + acp * ld(Cc + n01) +
                           app * ld(Cc + n11);
                    g[c] = half * (vp + vc);
                }
                ex = g[0]; ey = g[1]; ez = g[2]; bx = g[3]; by = g[4]; bz = g[5];
            }
            const T hx = a.hx;
            const T sE = q2m * hx / two;
            ex *= sE;
            ey *= sE;
            ez *= sE;
            px += ex / (one - Vx);
            py += ey / (one - Vx);
            pz += ez / (one - Vx);
            T gamma = sqrt_t<T>(one + px * px + py * py + pz * pz);
            const T gamma_r = one / gamma;
            bx += a.bxe;
            by += a.bye;
            bz += a.bze;
            bx = bx * gamma_r * q2m / (one - Vx) * hx / two;
            by = by * gamma_r * q2m / (one - Vx) * hx / two;
            bz = bz * gamma_r * q2m / (one - Vx) * hx / two;
            const T co = two / (one + (bx * bx) + (by * by) + (bz * bz));
            T p3x = py * bz - pz * by + px;
            T p3y = pz * bx - px * bz + py;
            T p3z = px * by - py * bx + pz;
            p3x *= co;
            p3y *= co;
            p3z *= co;
            const T px_new = p3y * bz - p3z * by;
            const T py_new = p3z * bx - p3x * bz;
            const T pz_new = p3x * by - p3y * bx;
            px += ex / (one - Vx) + px_new;
            py += ey / (one - Vx) + py_new;
            pz += ez / (one - Vx) + pz_new;
            gamma = sqrt_t<T>(one + px * px + py * py + pz * pz);
            const T Vxm = px / gamma, Vym = py / gamma, Vzm = pz / gamma;
            Vx = half * (Vxm + Vxp);
            const T Vy = half * (Vym + Vyp);
            const T Vz = half * (Vzm + Vzp);
            T djx = weight * a.djx0 * Vxm;
            T djy = weight * a.djy0 * Vym;
            T djz = weight * a.djz0 * Vzm;
            T drho = weight * a.drho0;
            djx *= one / (one - Vx);
            djy *= one / (one - Vx);
            djz *= one / (one - Vx);
            drho *= one / (one - Vx);
            T dy = Vy * hx / a.hy;
            T dz = Vz * hx / a.hz;
            dy = dy / (one - Vx);
            dz = dz / (one - Vx);
            move_and_deposit<T, SHAPE, PRECISE, NV>(a, i, j, k, yp, zp, px, py, pz, djx, djy, djz,
                                                   drho, dy, dz, key, v);
            }
        }
    }

    // warp-segmented sum over runs of equal first-deposit cell
    const unsigned full = 0xffffffffu;
    const int nextKey = __shfl_down_sync(full, key, 1);
    const int prevKey = __shfl_up_sync(full, key, 1);
    const bool last = (lane == 31) || (nextKey != key);
    const unsigned lastMask = __ballot_sync(full, last);
    const int end = __ffs(lastMask & (full << lane)) - 1;
    const bool head = (lane == 0) || (prevKey != key);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
#pragma unroll
        for (int c = 0; c < NV; c++) {
            const T o = __shfl_down_sync(full, v[c], d);
            if (lane + d <= end) v[c] += o;
        }
    }
    if (head && key >= 0) {
        const size_t plane = a.plane;
        if (SHAPE == QS_SHAPE_NGP) {
            const size_t n = (size_t)key;
#pragma unroll
            for (int qq = 0; qq < 4; qq++) atomicAdd(a.dep + qq * plane + n, v[qq]);
        } else {
            const int fj = key % My, fk = key / My;
            const int j1 = wrap_idx(fj + 1, My), k1 = wrap_idx(fk + 1, Mz);
            const size_t nn[4] = {(size_t)fj + (size_t)My * fk, (size_t)j1 + (size_t)My * fk,
                                  (size_t)fj + (size_t)My * k1, (size_t)j1 + (size_t)My * k1};
#pragma unroll
            for (int cnr = 0; cnr < 4; cnr++)
#pragma unroll
                for (int qq = 0; qq < 4; qq++)
                    atomicAdd(a.dep + qq * plane + nn[cnr], v[cnr * 4 + qq]);
        }
    }
}

// ---------------------------------------------------------------------------
// FP32 NGP push, one thread per cell, for the uniform lattice layout
// (particle p of the layer sits in cell p / PPC): in the live reference path a
// particle never leaves its seeded cell, so this layout is permanent.  The
// cell's fields are gathered once, its PPC particles are read and written as
// float4 vectors, deposits into the cell itself are summed in registers and
// flushed with 4 atomics; deposits that land in another cell go straight to
// global atomics.  Same physics as push_kernel<float, NGP, precise, fast>,
// with approximate reciprocals (a few ulp) for the divisions.
template <int PPC>
__global__ void __launch_bounds__(128) push_cell_kernel(PushArgs<float> a) {
    static_assert(PPC == 4, "float4 particle vectors");
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    const int My = a.My, Mz = a.Mz;
    if (cell >= My * Mz) return;
    pdl_wait();
    int j, k;
    cell_jk(cell, My, a.invMy, j, k);
    const size_t plane = a.plane;
    const size_t n = (size_t)cell;
    const float ex0 = 0.5f * (ld(a.P + 0 * plane + n) + ld(a.C + 0 * plane + n));
    const float ey0 = 0.5f * (ld(a.P + 1 * plane + n) + ld(a.C + 1 * plane + n));
    const float ez0 = 0.5f * (ld(a.P + 2 * plane + n) + ld(a.C + 2 * plane + n));
    const float bx0 = 0.5f * (ld(a.P + 3 * plane + n) + ld(a.C + 3 * plane + n)) + a.bxe;
    const float by0 = 0.5f * (ld(a.P + 4 * plane + n) + ld(a.C + 4 * plane + n)) + a.bye;
    const float bz0 = 0.5f * (ld(a.P + 5 * plane + n) + ld(a.C + 5 * plane + n)) + a.bze;
    const size_t base = (size_t)cell * PPC;
    float4 Y = *(const float4*)(a.y + base), Z = *(const float4*)(a.z + base);
    float4 PX = *(const float4*)(a.px + base), PY = *(const float4*)(a.py + base);
    float4 PZ = *(const float4*)(a.pz + base);
    const float4 W = *(const float4*)(a.w + base);
    float* yv = &Y.x; float* zv = &Z.x; float* pxv = &PX.x; float* pyv = &PY.x;
    float* pzv = &PZ.x; const float* wv = &W.x;
    float own0 = 0.f, own1 = 0.f, own2 = 0.f, own3 = 0.f;
#pragma unroll
    for (int q = 0; q < PPC; q++) {
        const float yp = yv[q], zp = zv[q];
        if (!(yp >= 0.f && yp <= 1.f && zp >= 0.f && zp <= 1.f)) {
            atomicOr(a.err, DEV_ERR_RANGE);
            continue;
        }
        float px = pxv[q], py = pyv[q], pz = pzv[q];
        const float inv_gp = rsqrtf(1.f + px * px + py * py + pz * pz);
        const float Vyp = py * inv_gp, Vzp = pz * inv_gp;
        const float omp = one_minus_vx(px, py, pz, inv_gp);   // 1 - Vx before the kick
        const float kE = a.sE * rcp_approx(omp);
        const float ex = ex0 * kE, ey = ey0 * kE, ez = ez0 * kE;
        px += ex; py += ey; pz += ez;
        const float kB = rsqrtf(1.f + px * px + py * py + pz * pz) * kE;
        const float bx = bx0 * kB, by = by0 * kB, bz = bz0 * kB;
        const float co = __fdividef(2.f, 1.f + bx * bx + by * by + bz * bz);
        const float p3x = (py * bz - pz * by + px) * co;
        const float p3y = (pz * bx - px * bz + py) * co;
        const float p3z = (px * by - py * bx + pz) * co;
        px += ex + (p3y * bz - p3z * by);
        py += ey + (p3z * bx - p3x * bz);
        pz += ez + (p3x * by - p3y * bx);
        const float inv_g = rsqrtf(1.f + px * px + py * py + pz * pz);
        const float Vxm = px * inv_g, Vym = py * inv_g, Vzm = pz * inv_g;
        const float Vy = 0.5f * (Vym + Vyp), Vz = 0.5f * (Vzm + Vzp);
        const float inv2 = rcp_approx(0.5f * (one_minus_vx(px, py, pz, inv_g) + omp));
        const float wq = wv[q] * inv2;
        const float djx = wq * a.djx0 * Vxm, djy = wq * a.djy0 * Vym, djz = wq * a.djz0 * Vzm;
        const float drho = wq * a.drho0;
        const float dy = Vy * a.hxhy * inv2, dz = Vz * a.hxhz * inv2;
        float partdx = 0.f, step = 1.f;
        if (fabsf(dy) > 1.f || fabsf(dz) > 1.f) step = partdx = fmaxf(fabsf(dy), fabsf(dz));
        if (partdx < 1.f) partdx = step = 1.f;
        float ytmp = yp, ztmp = zp;
        while (partdx > 0.f) {
            float ps;
            if (partdx > 1.f) { partdx -= 1.f; ps = rcp_approx(step); }
            else { ps = __fdividef(partdx, step); partdx = 0.f; }
            // cell-relative update; the base cell stays the seeded cell (the
            // reference adds the outer j_jump = j at every sub-step)
            const float uy = ytmp + dy * ps, uz = ztmp + dz * ps;
            const float fy = floorf(uy), fz = floorf(uz);
            float ry = uy - fy, rz = uz - fz;
            int sy = (int)fy, sz = (int)fz;
            if (ry >= 1.f) { ry = 0.f; sy += 1; }
            if (rz >= 1.f) { rz = 0.f; sz += 1; }
            ytmp = ry;
            ztmp = rz;
            const float d0 = djx * ps, d1 = djy * ps, d2 = djz * ps, d3 = drho * ps;
            if (sy == 0 && sz == 0) {
                own0 += d0; own1 += d1; own2 += d2; own3 += d3;
            } else {
                const int jj = wrap_idx(j + sy, My), kk = wrap_idx(k + sz, Mz);
                const size_t m = (size_t)jj + (size_t)My * kk;
                atomicAdd(a.dep + 0 * plane + m, d0);
                atomicAdd(a.dep + 1 * plane + m, d1);
                atomicAdd(a.dep + 2 * plane + m, d2);
                atomicAdd(a.dep + 3 * plane + m, d3);
            }
        }
        yv[q] = ytmp; zv[q] = ztmp; pxv[q] = px; pyv[q] = py; pzv[q] = pz;
    }
    pdl_trigger();
    atomicAdd(a.dep + 0 * plane + n, own0);
    atomicAdd(a.dep + 1 * plane + n, own1);
    atomicAdd(a.dep + 2 * plane + n, own2);
    atomicAdd(a.dep + 3 * plane + n, own3);
    if (a.full) {
        *(float4*)(a.y + base) = Y; *(float4*)(a.z + base) = Z;
        *(float4*)(a.px + base) = PX; *(float4*)(a.py + base) = PY;
        *(float4*)(a.pz + base) = PZ;
    }
}

// ---------------------------------------------------------------------------
// CIC push over particles grouped by cell (the counting sort in sort.cu
// regroups them every few full pushes), FP32, or FP64 with FMA contraction
// for the FP64 path on FFT transforms.  A block owns a tile of 32 x TY cells
// and stages the fields (P and C averaged) of the tile's cells plus one row
// and column in shared memory for the gather.  A warp owns one row of 32
// cells for the whole launch and lane l owns cell c0 + l.  The row's
// particles are processed in windows of WIN slots:
//  - phase 1, particle-parallel (lane = particle, the next one prefetched):
//    the push; the first sub-step's charges q = dq * ps, its in-cell position
//    and its cell (and the final cell) are staged in shared memory, further
//    sub-steps (|dy| or |dz| above a cell, rare) deposit by global atomics;
//  - phase 2, cell-parallel (lane = cell): each lane walks the slots of its
//    own cell inside the window (regrouped, they are [offset(c),
//    offset(c + 1))), rebuilds the 4 corner weights and adds the 4 x ND
//    corner values to registers.  A particle whose first sub-step ended in
//    another cell (it moved since the last regrouping) is added by global
//    atomics instead; on a full push followed by a regrouping the lane counts
//    the particles that stay in its cell and adds one count per cell.
// No shuffles or matches sum the deposits.  The window's slots carry one pad
// word per 32, so that lanes reading slots about ppc apart hit distinct
// banks.  At the end each lane spreads its cell's corner sums (the right-hand
// corners through a shuffle to the next lane), the warps combine their rows
// in the block tile in two ordered phases, and the tile is flushed with one
// global atomic per touched cell and current.  Particles gathered outside
// the tile (moved since the regrouping) read the fields from global memory.
// ND = 3 leaves out the density deposit, which the march does not read.  The
// full push stores the particles in place with their new cell.  Same physics
// as push_kernel<T, CIC, precise, fast> (movepart_layer_CIC.cpp:165-193,
// 449-496 weights), the divisions factored into reciprocals.
template <class T>
__device__ __forceinline__ int cell_offset(const PushArgs<T>& a, int c) {
    return a.loff[c] + a.bpref[c >> 10];
}

// the reciprocal forms of the grouped push: approximate in FP32, IEEE in FP64
template <class T>
struct RowMath;
template <>
struct RowMath<float> {
    static __device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }
    static __device__ __forceinline__ float rcp(float x) { return rcp_approx(x); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdividef(a, b); }
};
template <>
struct RowMath<double> {
    static __device__ __forceinline__ double rsq(double x) { return rsqrt(x); }
    static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
    static __device__ __forceinline__ double div(double a, double b) { return a / b; }
};

// one CIC sub-step of a particle (cell-relative move from base cell (jb, kb),
// periodic wrap, the 4 corner weights of the new position)
template <class T>
__device__ __forceinline__ void cic_substep(T dy, T dz, T ps, T& ytmp, T& ztmp, int& jb, int& kb,
                                            int My, int Mz, T (&wc)[4]) {
    const T one = T(1);
    const T uy = ytmp + dy * ps, uz = ztmp + dz * ps;
    const T fy = floor_t<T>(uy), fz = floor_t<T>(uz);
    T ry = uy - fy, rz = uz - fz;
    int sy = (int)fy, sz = (int)fz;
    if (ry >= one) { ry = T(0); sy += 1; }
    if (rz >= one) { rz = T(0); sz += 1; }
    jb = wrap1(jb + sy, My);   // |dy * ps| <= 1: the shift is at most one cell
    kb = wrap1(kb + sz, Mz);
    ytmp = ry;
    ztmp = rz;
    wc[0] = (one - ry) * (one - rz);
    wc[1] = ry * (one - rz);
    wc[2] = (one - ry) * rz;
    wc[3] = ry * rz;
}

template <int TY, int ND, int WIN, class T>
__global__ void __launch_bounds__(32 * TY) push_cic_row_kernel(PushArgs<T> a) {
    using M = RowMath<T>;
    using FP = FPair<T>;
    using P2 = typename FP::type;
    constexpr int TX = 32, W = TX + 1, H = TY + 1;
    constexpr int NS = ND + 2;           // staged per slot: ND charges, in-cell y and z
    constexpr int WP = WIN + WIN / 32;   // one pad word per 32 slots
    static_assert(WIN % 32 == 0, "whole warps per window");
    const T one = T(1), zero = T(0), half = T(0.5);
    __shared__ P2 Fs[3][H][W];           // field pairs of the tile cells + one row/column (P, C averaged)
    __shared__ T Tt[ND][H][W];           // block deposit tile [current][row][col]
    __shared__ T S[TY][NS][WP];          // staged deposits of the window
    __shared__ int K[TY][2][WP];         // [0]: first sub-step's cell (-1: none); [1]: final cell
    const int lane = threadIdx.x & 31, wr = threadIdx.x >> 5;
    const int My = a.My, Mz = a.Mz;
    const size_t plane = a.plane;
    const int tiles_x = My / TX;
    const int j0 = (blockIdx.x % tiles_x) * TX, k0 = (blockIdx.x / tiles_x) * TY;
    for (int i = threadIdx.x; i < ND * H * W; i += 32 * TY) (&Tt[0][0][0])[i] = zero;
    QS_TRACE_ENTRY();
    pdl_wait();
    QS_TRACE_WAITED();
    for (int i = threadIdx.x; i < H * W; i += 32 * TY) {
        const int r = i / W, cc = i - r * W;
        const size_t m = (size_t)wrap1(j0 + cc, My) + (size_t)My * wrap1(k0 + r, Mz);
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const P2 pp = FP::make(ld(a.P + 2 * q * plane + m), ld(a.P + (2 * q + 1) * plane + m));
            const P2 cp = FP::make(ld(a.C + 2 * q * plane + m), ld(a.C + (2 * q + 1) * plane + m));
            Fs[q][r][cc] = FP::mul(half, FP::add(pp, cp));
        }
    }
    __syncthreads();
    // the tile's own cells of the gathered fields, for the push adjoint (the
    // march, which skips the density deposit, is what the adjoint recomputes)
    if constexpr (ND == 3)
        if (a.favg)
            for (int i = threadIdx.x; i < TY * TX; i += 32 * TY) {
                const int r = i / TX, cc = i - r * TX;
                const size_t m = (size_t)(j0 + cc) + (size_t)My * (k0 + r);
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    a.favg[2 * q * plane + m] = Fs[q][r][cc].x;
                    a.favg[(2 * q + 1) * plane + m] = Fs[q][r][cc].y;
                }
            }
    const int c0 = j0 + My * (k0 + wr);   // this warp's 32 cells: c0 .. c0+31
    const int mycell = c0 + lane;
    const int lo = cell_offset(a, mycell);
    const int hi = (size_t)(mycell + 1) < plane ? cell_offset(a, mycell + 1) : (int)a.n;
    const int pbeg = __shfl_sync(0xffffffffu, lo, 0);
    const int pend = __shfl_sync(0xffffffffu, hi, 31);
    const bool count = a.full && a.cnt;
    int stay = 0;                        // particles that end the full push in mycell
    // the cell's sums of current d at its corners (0, 1) and (2, 3)
    P2 acc[ND][2];
#pragma unroll
    for (int d = 0; d < ND; d++) acc[d][0] = acc[d][1] = FP::make(zero, zero);
    // the particle of the next pass is loaded while this one is pushed
    int nx_cell = 0;
    T nx_y = zero, nx_z = zero, nx_px = zero, nx_py = zero, nx_pz = zero, nx_w = zero;
    if (pbeg + lane < pend) {
        const int q = pbeg + lane;
        nx_cell = a.cell[q]; nx_y = a.y[q]; nx_z = a.z[q];
        nx_px = a.px[q]; nx_py = a.py[q]; nx_pz = a.pz[q]; nx_w = a.w[q];
    }
    for (int wbase = pbeg; wbase < pend; wbase += WIN) {
        const int wend = min(pend, wbase + WIN);
        // phase 1: lane = particle
        for (int base = wbase; base < wend; base += 32) {
            const int p = base + lane;
            const int cell = nx_cell;
            const T yp = nx_y, zp = nx_z, w = nx_w;
            T px = nx_px, py = nx_py, pz = nx_pz;
            if (p + 32 < pend) {
                const int q = p + 32;
                nx_cell = a.cell[q]; nx_y = a.y[q]; nx_z = a.z[q];
                nx_px = a.px[q]; nx_py = a.py[q]; nx_pz = a.pz[q]; nx_w = a.w[q];
            }
            int key = -1, last = cell;
            T qv[ND], ay = zero, az = zero;
#pragma unroll
            for (int d = 0; d < ND; d++) qv[d] = zero;
            if (p < pend) {
                if (!(yp >= zero && yp <= one && zp >= zero && zp <= one)) {
                    atomicOr(a.err, DEV_ERR_RANGE);   // no deposit; it stays in its cell
                } else {
                    int j, k;
                    cell_jk(cell, My, a.invMy, j, k);
                    const T wg[4] = {(one - yp) * (one - zp), yp * (one - zp), (one - yp) * zp,
                                     yp * zp};
                    T g[6];
                    const int tj = j - j0, tk = k - k0;
                    if (tj >= 0 && tj < TX && tk >= 0 && tk < TY) {
#pragma unroll
                        for (int q = 0; q < 3; q++) {
                            P2 gq = FP::mul(wg[0], Fs[q][tk][tj]);
                            gq = FP::fma(wg[1], Fs[q][tk][tj + 1], gq);
                            gq = FP::fma(wg[2], Fs[q][tk + 1][tj], gq);
                            gq = FP::fma(wg[3], Fs[q][tk + 1][tj + 1], gq);
                            g[2 * q] = gq.x;
                            g[2 * q + 1] = gq.y;
                        }
                    } else {
                        const int j1 = wrap1(j + 1, My), k1 = wrap1(k + 1, Mz);
                        const size_t nn[4] = {(size_t)j + (size_t)My * k,
                                              (size_t)j1 + (size_t)My * k,
                                              (size_t)j + (size_t)My * k1,
                                              (size_t)j1 + (size_t)My * k1};
#pragma unroll
                        for (int f = 0; f < 6; f++) {
                            T s = zero;
#pragma unroll
                            for (int r = 0; r < 4; r++)
                                s += wg[r] * half * (ld(a.P + f * plane + nn[r]) +
                                                     ld(a.C + f * plane + nn[r]));
                            g[f] = s;
                        }
                    }
                    const T inv_gp = M::rsq(one + px * px + py * py + pz * pz);
                    const T Vyp = py * inv_gp, Vzp = pz * inv_gp;
                    const T omp = one_minus_vx(px, py, pz, inv_gp);   // 1 - Vx before the kick
                    const T kE = a.sE * M::rcp(omp);
                    const T ex = g[0] * kE, ey = g[1] * kE, ez = g[2] * kE;
                    px += ex; py += ey; pz += ez;
                    const T kB = M::rsq(one + px * px + py * py + pz * pz) * kE;
                    const T bx = (g[3] + a.bxe) * kB, by = (g[4] + a.bye) * kB,
                            bz = (g[5] + a.bze) * kB;
                    const T co = M::div(T(2), one + bx * bx + by * by + bz * bz);
                    const T p3x = (py * bz - pz * by + px) * co;
                    const T p3y = (pz * bx - px * bz + py) * co;
                    const T p3z = (px * by - py * bx + pz) * co;
                    px += ex + (p3y * bz - p3z * by);
                    py += ey + (p3z * bx - p3x * bz);
                    pz += ez + (p3x * by - p3y * bx);
                    const T inv_g = M::rsq(one + px * px + py * py + pz * pz);
                    const T Vxm = px * inv_g, Vym = py * inv_g, Vzm = pz * inv_g;
                    const T Vy = half * (Vym + Vyp), Vz = half * (Vzm + Vzp);
                    const T inv2 = M::rcp(half * (one_minus_vx(px, py, pz, inv_g) + omp));
                    const T wq = w * inv2;
                    const T dq[4] = {wq * a.djx0 * Vxm, wq * a.djy0 * Vym, wq * a.djz0 * Vzm,
                                     wq * a.drho0};
                    const T dy = Vy * a.hxhy * inv2, dz = Vz * a.hxhz * inv2;
                    // sub-steps of at most one cell: the first covers 1/step of
                    // the move, partdx what remains of it after the first
                    const T ady = fabs_t(dy), adz = fabs_t(dz);
                    const T mx = ady > adz ? ady : adz;
                    T partdx = zero, step = one, ps = one;
                    if (mx > one) { step = mx; partdx = mx - one; ps = M::rcp(step); }
                    T ytmp = yp, ztmp = zp;
                    int jb = j, kb = k;
                    // first sub-step: staged for the cell-parallel sum
                    T wc[4];
                    cic_substep<T>(dy, dz, ps, ytmp, ztmp, jb, kb, My, Mz, wc);
                    key = jb + My * kb;
#pragma unroll
                    for (int d = 0; d < ND; d++) qv[d] = dq[d] * ps;
                    ay = ytmp;
                    az = ztmp;
                    // further sub-steps: direct atomics
                    while (partdx > zero) {
                        if (partdx > one) { partdx -= one; ps = M::rcp(step); }
                        else { ps = M::div(partdx, step); partdx = zero; }
                        cic_substep<T>(dy, dz, ps, ytmp, ztmp, jb, kb, My, Mz, wc);
                        const int jb1 = wrap1(jb + 1, My), kb1 = wrap1(kb + 1, Mz);
                        const size_t nd[4] = {(size_t)jb + (size_t)My * kb,
                                              (size_t)jb1 + (size_t)My * kb,
                                              (size_t)jb + (size_t)My * kb1,
                                              (size_t)jb1 + (size_t)My * kb1};
#pragma unroll
                        for (int r = 0; r < 4; r++)
#pragma unroll
                            for (int d = 0; d < ND; d++)
                                atomicAdd(a.dep + d * plane + nd[r], dq[d] * ps * wc[r]);
                    }
                    last = jb + My * kb;
                    if (a.full) {
                        a.y[p] = ytmp; a.z[p] = ztmp; a.px[p] = px; a.py[p] = py; a.pz[p] = pz;
                        a.cell_out[p] = last;
                    }
                }
            }
            const int s = base - wbase + lane, sp = s + (s >> 5);
            K[wr][0][sp] = key;
            if (count) K[wr][1][sp] = last;
#pragma unroll
            for (int d = 0; d < ND; d++) S[wr][d][sp] = qv[d];
            S[wr][ND][sp] = ay;
            S[wr][ND + 1][sp] = az;
        }
        __syncwarp();
        // phase 2: lane = cell
        const int qa = max(lo, wbase), qb = min(hi, wend);
        for (int q = qa; q < qb; q++) {
            const int s = q - wbase, sp = s + (s >> 5);
            const int key = K[wr][0][sp];
            if (count) {
                const int last = K[wr][1][sp];
                if (last == mycell) stay++;
                else atomicAdd(a.cnt + last, 1);
            }
            if (key < 0) continue;
            const T ry = S[wr][ND][sp], rz = S[wr][ND + 1][sp];
            T qv[ND];
#pragma unroll
            for (int d = 0; d < ND; d++) qv[d] = S[wr][d][sp];
            if (key == mycell) {
                // corner weights in pairs: (1 - rz) (1 - ry, ry) and rz (1 - ry, ry)
                const P2 wy = FP::make(one - ry, ry);
                const P2 w01 = FP::mul(one - rz, wy), w23 = FP::mul(rz, wy);
#pragma unroll
                for (int d = 0; d < ND; d++) {
                    acc[d][0] = FP::fma(qv[d], w01, acc[d][0]);
                    acc[d][1] = FP::fma(qv[d], w23, acc[d][1]);
                }
            } else {
                const T wc[4] = {(one - ry) * (one - rz), ry * (one - rz), (one - ry) * rz,
                                 ry * rz};
                int kj, kk;
                cell_jk(key, My, a.invMy, kj, kk);
                const int kj1 = wrap1(kj + 1, My), kk1 = wrap1(kk + 1, Mz);
                const size_t nd[4] = {(size_t)kj + (size_t)My * kk, (size_t)kj1 + (size_t)My * kk,
                                      (size_t)kj + (size_t)My * kk1, (size_t)kj1 + (size_t)My * kk1};
#pragma unroll
                for (int r = 0; r < 4; r++)
#pragma unroll
                    for (int d = 0; d < ND; d++) atomicAdd(a.dep + d * plane + nd[r], qv[d] * wc[r]);
            }
        }
        __syncwarp();
    }
    if (stay) atomicAdd(a.cnt + mycell, stay);
    pdl_trigger();
    // spread the per-cell sums to the corners: the lane of cell (l, row) owns
    // column l of rows row and row+1; the right-hand corners go to lane l+1
    const unsigned full = 0xffffffffu;
    T row0[ND], row1[ND], edge0[ND], edge1[ND];
#pragma unroll
    for (int d = 0; d < ND; d++) {
        const T c00 = acc[d][0].x, c10 = acc[d][0].y;
        const T c01 = acc[d][1].x, c11 = acc[d][1].y;
        const T l10 = __shfl_up_sync(full, c10, 1), l11 = __shfl_up_sync(full, c11, 1);
        row0[d] = c00 + (lane > 0 ? l10 : zero);
        row1[d] = c01 + (lane > 0 ? l11 : zero);
        edge0[d] = c10;   // used by lane 31 only: column 32
        edge1[d] = c11;
    }
#pragma unroll
    for (int d = 0; d < ND; d++) {
        Tt[d][wr][lane] += row0[d];
        if (lane == 31) Tt[d][wr][TX] += edge0[d];
    }
    __syncthreads();
#pragma unroll
    for (int d = 0; d < ND; d++) {
        Tt[d][wr + 1][lane] += row1[d];
        if (lane == 31) Tt[d][wr + 1][TX] += edge1[d];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < H * W; i += 32 * TY) {
        const int r = i / W, cc = i - r * W;
        const size_t m = (size_t)wrap1(j0 + cc, My) + (size_t)My * wrap1(k0 + r, Mz);
#pragma unroll
        for (int d = 0; d < ND; d++) {
            const T x = Tt[d][r][cc];
            if (x != zero) atomicAdd(a.dep + d * plane + m, x);
        }
    }
    QS_TRACE_END(a.full ? trace::K_PUSH_FULL : trace::K_PUSH_HALF);
}

// the grouped CIC push (both widths): 0 when the layout does not fit it
template <class T>
int launch_push_rows(const PushArgs<T>& a, cudaStream_t st) {
    constexpr int TY = 4, WIN = 128;
    if (!a.loff || a.dep_cell) return 0;   // grouped by cell with offsets (the engine checks the shape)
    const dim3 grid((a.My / 32) * (a.Mz / TY));
    if (a.skip_dens)
        launch_pdl(push_cic_row_kernel<TY, 3, WIN, T>, grid, dim3(32 * TY), 0, st, a);
    else
        launch_pdl(push_cic_row_kernel<TY, 4, WIN, T>, grid, dim3(32 * TY), 0, st, a);
    return 1;
}

int launch_push_rows_f64(const PushArgs<double>& a, cudaStream_t st);   // push_f64fma.cu

template <class T>
int launch_push(const PushArgs<T>& a, int shape, bool precise, cudaStream_t st) {
    if (a.n <= 0) return 0;
    constexpr bool F32 = sizeof(T) == 4;
    const int threads = 256;
    const unsigned blocks = (unsigned)((a.n + threads - 1) / threads);
    if (shape == QS_SHAPE_NGP) {
        if constexpr (F32) {
            if (a.uniform_ppc == 4 && a.n == (int64_t)a.My * a.Mz * 4 && !a.dep_cell) {
                const int cells = a.My * a.Mz;
                launch_pdl(push_cell_kernel<4>, dim3((cells + 127) / 128), dim3(128), 0, st, a);
                return 1;
            }
            push_kernel<T, QS_SHAPE_NGP, true, true><<<blocks, threads, 0, st>>>(a);
        } else {
            if (precise) push_kernel<T, QS_SHAPE_NGP, true, false><<<blocks, threads, 0, st>>>(a);
            else push_kernel<T, QS_SHAPE_NGP, false, false><<<blocks, threads, 0, st>>>(a);
        }
    } else {
        if constexpr (F32) {
            if (launch_push_rows<float>(a, st)) return 1;
        } else {
            if (a.loff && !a.dep_cell) return launch_push_rows_f64(a, st);
        }
        push_kernel<T, QS_SHAPE_CIC, true, F32><<<blocks, threads, 0, st>>>(a);
    }
    return 1;
}

}  // namespace qs
