// adjoint_maps.cuh — per-mode adjoints (transposes) of the Guess / Iterate
// spectral maps, shared by the adjoint's map kernels (adjoint.cu) and the
// FP32 kernels that apply them between the halves of a transform
// (dtt_fft.cu).
#pragma once
#include "qs_common.cuh"
#include "qs_internal.h"

namespace qs {
namespace adjmaps {

template <class T>
__device__ __forceinline__ void beam_adj(const AdjSpecArgs<T>& a, size_t n, T lrb, T lrbp,
                                         T ljxb) {
    if (a.wb0 != T(0)) {
        a.lRb0[n] += a.wb0 * lrb;
        a.lJxb0[n] += a.wb0 * ljxb;
    }
    if (a.wb1 != T(0)) {
        a.lRb1[n] += a.wb1 * lrb;
        a.lJxb1[n] += a.wb1 * ljxb;
    }
    if (a.wp0 != T(0)) a.lRbp0[n] += a.wp0 * lrbp;
    if (a.wp1 != T(0)) a.lRbp1[n] += a.wp1 * lrbp;
}

template <class T>
__device__ __forceinline__ T opt(const T* p, size_t n) { return p ? p[n] : T(0); }

template <class T>
__device__ __forceinline__ void put_lp(const AdjSpecArgs<T>& a, int f, size_t n, T v) {
    if (a.lP_set) a.lP[f][n] = v;
    else a.lP[f][n] += v;
}

// Transpose of corrector_kernel (IterateFieldsHydroLinLayerSplit's per-mode
// update, movefieldshydrolinlayersplit.cpp:1419-1466) at mode (j, k): le, lb
// are the adjoints of its spectral E, B outputs; lj gets the adjoint of its
// J input; the other adjoints go to the planes of `a`.
template <class T>
__device__ __forceinline__ void corrector_adjoint_mode(const AdjSpecArgs<T>& a, int j, int k,
                                                       size_t n, const T (&le)[3],
                                                       const T (&lb)[3], T (&lj)[3]) {
    const T d = *a.dens_p, hx = a.hx;
    const T akz = a.piZ * (T(k) + T(0.5));
    const T aky = a.piY * (T(j) + T(0.5));
    const T k2 = aky * aky + akz * akz;
    const T lrho = opt(a.lRho, n);
    const T lex = le[0] + opt(a.lEb[0], n);
    T ley = le[1] + opt(a.lEb[1], n);
    T lez = le[2] + opt(a.lEb[2], n);
    const T lbx = lb[0], lby = lb[1], lbz = lb[2];
    // by = (-akz (jx + jxb) + d ez)/k2, bz = (aky (jx + jxb) - d ey)/k2
    lez += d * lby / k2;
    ley -= d * lbz / k2;
    const T ljxs = (-akz * lby + aky * lbz) / k2;          // d(by,bz)/d(jx + jxb)
    T ljx = lrho + ljxs + opt(a.lJb[0], n);
    T ljy = -hx * T(0.5) * aky * lrho - aky / k2 * lex + akz / k2 * lbx + opt(a.lJb[1], n);
    T ljz = -hx * T(0.5) * akz * lrho - akz / k2 * lex - aky / k2 * lbx + opt(a.lJb[2], n);
    const T lsrc = (aky * ley + akz * lez) / (d + k2);     // src = rb + rbp + rp + rho_old
    lj[0] = ljx;
    lj[1] = ljy;
    lj[2] = ljz;
    a.lRhoOld[n] = lsrc;
    // P-bank inputs: 0 RhoP, 1 ExP, 2 EyP, 3 EzP, 4 JxP, 5 JyP, 6 JzP
    put_lp(a, 0, n, lrho + lsrc);
    if (a.lP_set) a.lP[1][n] = T(0);
    put_lp(a, 2, n, -ley);
    put_lp(a, 3, n, -lez);
    put_lp(a, 4, n, -lrho);
    put_lp(a, 5, n, -hx * T(0.5) * aky * lrho);
    put_lp(a, 6, n, -hx * T(0.5) * akz * lrho);
    beam_adj(a, n, lsrc, lsrc, ljxs);
}

// Transpose of predictor_kernel (GuessFieldsHydroLinLayerSplit's per-mode
// update, movefieldshydrolinlayersplit.cpp:843-872) at mode (j, k): le, lb
// are the adjoints of its spectral E, B outputs.
template <class T>
__device__ __forceinline__ void predictor_adjoint_mode(const AdjSpecArgs<T>& a, int j, int k,
                                                       size_t n, const T (&le)[3],
                                                       const T (&lb)[3]) {
    const T d = *a.dens_p, hx = a.hx;
    const T akz = a.piZ * (T(k) + T(0.5));
    const T aky = a.piY * (T(j) + T(0.5));
    const T k2 = aky * aky + akz * akz;
    const T den = T(4) + d * hx * hx;
    const T prop = (T(4) - d * hx * hx) / den;
    const T lrho = opt(a.lRho, n);
    T lex = le[0], ley = le[1], lez = le[2];
    const T lbx = lb[0], lby = lb[1], lbz = lb[2];
    // b from the predicted currents and fields
    const T ljx = (-akz * lby + aky * lbz) / k2;   // also the jxb adjoint
    const T ljy = akz * lbx / k2;
    const T ljz = -aky * lbx / k2;
    lez += d * lby / k2;
    ley -= d * lbz / k2;
    // jx = jxp + hx d (ex + exp)/2 (and y, z)
    const T hd2 = hx * d * T(0.5);
    lex += hd2 * ljx;
    ley += hd2 * ljy;
    lez += hd2 * ljz;
    T lexp = hd2 * ljx, leyp = hd2 * ljy, lezp = hd2 * ljz;
    // ey = -eyp + aky src/(d + k2), src = rb + rbp + rp + rho
    const T lsrc = (aky * ley + akz * lez) / (d + k2);
    leyp -= ley;
    lezp -= lez;
    const T lrho_t = lrho + lsrc;
    // rho = prop rp - (rb + rbp) d hx^2/den + 4 exp hx (k2 + d)/den
    // ex  = prop exp - 2 (2 rp + rb + rbp) d hx / ((k2 + d) den)
    const T cex = T(2) * d * hx / ((k2 + d) * den);
    const T lrp = lsrc + prop * lrho_t - T(2) * cex * lex;
    const T lrb = lsrc - d * hx * hx / den * lrho_t - cex * lex;
    lexp += T(4) * hx * (k2 + d) / den * lrho_t + prop * lex;
    put_lp(a, 0, n, lrp);
    put_lp(a, 1, n, lexp);
    put_lp(a, 2, n, leyp);
    put_lp(a, 3, n, lezp);
    put_lp(a, 4, n, ljx);
    put_lp(a, 5, n, ljy);
    put_lp(a, 6, n, ljz);
    beam_adj(a, n, lrb, lrb, ljx);
}

}  // namespace adjmaps
}  // namespace qs
