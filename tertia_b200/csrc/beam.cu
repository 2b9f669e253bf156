// beam.cu — driver-beam push and 3-D CIC deposit (reference
// Mesh::MoveBeamParticles, movebeam.cpp:14-659, and Mesh::MoveBeamInCell,
// :662-774; dead GPU twin moveBeamKernel, cuBeam.cu:106-690).
//
// One thread per beam macro-particle.  The particle state (cell, in-cell
// fraction, momentum, weight) stays FP64 across beam steps; the fields are
// read from the per-layer field store in the march's real type.  The
// expression order is the reference's (compiled with -fmad=false), including
// the unscaled E kick (:334-336, the q2m*Ts/2 scaling is commented out at
// :301-316) and the synchrotron momentum loss (:449-491; the photon
// histogram is a diagnostic and is not kept).  Beam currents deposited
// outside the interior planes of layers 0..nx are dropped: the reference
// deposits them into guard cells that its solve never reads.
#include "qs_common.cuh"
#include "qs_internal.h"

namespace qs {

template <class T>
__device__ __forceinline__ double fget(const T* f3, size_t plane, int i, int f, int j, int k,
                                       int My, int Mz) {
    if (j == My) j = 0;   // periodic guard copy (ExchangeFieldsSplit)
    if (k == Mz) k = 0;
    return (double)__ldg(f3 + ((size_t)i * 6 + f) * plane + (size_t)j + (size_t)My * k);
}

template <class T>
__device__ __forceinline__ void bdep(T* b3, size_t plane, int L, int My, int Mz, int i, int j,
                                     int k, double rho, double jx) {
    if (i < 0 || i > L || j < 0 || j >= My || k < 0 || k >= Mz) return;
    const size_t n = (size_t)j + (size_t)My * k;
    atomicAdd(b3 + ((size_t)i * 2 + 0) * plane + n, (T)rho);
    atomicAdd(b3 + ((size_t)i * 2 + 1) * plane + n, (T)jx);
}

template <class T>
__global__ void __launch_bounds__(256) beam_push_kernel(BeamArgs<T> a) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const int L = a.L, My = a.My, Mz = a.Mz;
    const int i = a.bi[p], j = a.bj[p], k = a.bk[p];
    if (i < 0 || i >= L || j < 0 || j >= My || k < 0 || k >= Mz) return;  // frozen particle
    const double weight = a.w[p];
    const double x = a.x[p], y = a.y[p], z = a.z[p];
    double px = a.px[p], py = a.py[p], pz = a.pz[p];
    const double pxn = px, pyn = py, pzn = pz;
    const double q2m = a.q2m;
    if (x < 0 || x > 1 || y < 0 || y > 1 || z < 0 || z > 1) {
        atomicOr(a.err, DEV_ERR_RANGE);
        return;
    }
    const double axc = 1. - x, axp = x, ayc = 1. - y, ayp = y, azc = 1. - z, azp = z;
    const double accc = axc * ayc * azc, acpc = axc * ayp * azc, accp = axc * ayc * azp,
                 acpp = axc * ayp * azp, apcc = axp * ayc * azc, appc = axp * ayp * azc,
                 apcp = axp * ayc * azp, appp = axp * ayp * azp;
    const T* f3 = a.fields3d;
    const size_t plane = a.plane;
    double g[6];
#pragma unroll
    for (int f = 0; f < 6; f++) {
        g[f] = accc * fget(f3, plane, i, f, j, k, My, Mz) +
               acpc * fget(f3, plane, i, f, j + 1, k, My, Mz) +
               accp * fget(f3, plane, i, f, j, k + 1, My, Mz) +
               acpp * fget(f3, plane, i, f, j + 1, k + 1, My, Mz) +
               apcc * fget(f3, plane, i + 1, f, j, k, My, Mz) +
               appc * fget(f3, plane, i + 1, f, j + 1, k, My, Mz) +
               apcp * fget(f3, plane, i + 1, f, j, k + 1, My, Mz) +
               appp * fget(f3, plane, i + 1, f, j + 1, k + 1, My, Mz);
    }
    const double ex = g[0], ey = g[1], ez = g[2];
    double bx = g[3] + a.bxe, by = g[4] + a.bye, bz = g[5] + a.bze;
    const double ts = a.ts;
    px += ex;
    py += ey;
    pz += ez;
    double gamma = sqrt(1. + px * px + py * py + pz * pz);
    const double gamma_r = 1. / gamma;
    bx = bx * gamma_r * q2m * ts / 2.;
    by = by * gamma_r * q2m * ts / 2.;
    bz = bz * gamma_r * q2m * ts / 2.;
    const double co = 2. / (1. + (bx * bx) + (by * by) + (bz * bz));
    double p3x = py * bz - pz * by + px;
    double p3y = pz * bx - px * bz + py;
    double p3z = px * by - py * bx + pz;
    p3x *= co;
    p3y *= co;
    p3z *= co;
    const double px_new = p3y * bz - p3z * by;
    const double py_new = p3z * bx - p3x * bz;
    const double pz_new = p3x * by - p3y * bx;
    px += (ex + px_new);
    py += (ey + py_new);
    pz += (ez + pz_new);
    const double p2 = px * px + py * py + pz * pz;
    if (a.synchrotron && 1. + p2 > a.syn_min * a.syn_min) {
        double dpx = px - pxn, dpy = py - pyn, dpz = pz - pzn;
        const double pdp = px * dpx + py * dpy + pz * dpz;
        dpx -= px * (pdp / p2);
        dpy -= py * (pdp / p2);
        dpz -= pz * (pdp / p2);
        const double p2absrev = 1.0 / sqrt(p2);
        const double nx = px * p2absrev, nyv = py * p2absrev, nzv = pz * p2absrev;
        const double dpabs = sqrt(dpx * dpx + dpy * dpy + dpz * dpz);
        const double Gamma2 = 1. + p2;
        const double omega_c = 3. * Gamma2 * dpabs / (4. * 3.1415927 * ts);
        const double Ephoton = a.elaser_photon * omega_c;
        const double alfa = 1. / 137.;
        const double nph = 4. / 9. * alfa * dpabs;
        px -= (nph * Ephoton * nx / 511000.0);
        py -= (nph * Ephoton * nyv / 511000.0);
        pz -= (nph * Ephoton * nzv / 511000.0);
    }
    gamma = 1. / sqrt(1. + px * px + py * py + pz * pz);
    const double Vx = px * gamma, Vy = py * gamma;
    const double polarity = a.polarity;
    const double djx = weight * polarity * Vx;
    const double drho = weight * polarity;
    (void)Vy;
    const double dx = (px * gamma - 1.) * ts / a.hx;
    const double dy = py * gamma * ts / a.hy;
    const double dz = pz * gamma * ts / a.hz;
    double xtmp = x + dx, ytmp = y + dy, ztmp = z + dz;
    int i_jump = (int)xtmp, j_jump = (int)ytmp, k_jump = (int)ztmp;
    if (xtmp < 0.) i_jump--;
    if (ytmp < 0.) j_jump--;
    if (ztmp < 0.) k_jump--;
    int itmp = i + i_jump, jtmp = j + j_jump, ktmp = k + k_jump;
    if (itmp < 0) itmp = -1;
    if (itmp > L - 1) itmp = L;
    if (jtmp < 0) jtmp = -1;
    if (jtmp > My - 1) jtmp = My;
    if (ktmp < 0) ktmp = -1;
    if (ktmp > Mz - 1) ktmp = Mz;
    xtmp -= i_jump;
    ytmp -= j_jump;
    ztmp -= k_jump;
    while (xtmp < 0.) xtmp += 1.;
    while (xtmp > 1.) xtmp -= 1.;
    while (ytmp < 0.) ytmp += 1.;
    while (ytmp > 1.) ytmp -= 1.;
    while (ztmp < 0.) ztmp += 1.;
    while (ztmp > 1.) ztmp -= 1.;
    a.px[p] = px;
    a.py[p] = py;
    a.pz[p] = pz;
    a.x[p] = xtmp;
    a.y[p] = ytmp;
    a.z[p] = ztmp;
    a.bi[p] = itmp;
    a.bj[p] = jtmp;
    a.bk[p] = ktmp;
    const double ax1 = xtmp, ax0 = 1. - ax1, ay1 = ytmp, ay0 = 1. - ay1, az1 = ztmp,
                 az0 = 1. - az1;
    T* b3 = a.beam3d;
#pragma unroll
    for (int di = 0; di < 2; di++)
#pragma unroll
        for (int dj = 0; dj < 2; dj++)
#pragma unroll
            for (int dk = 0; dk < 2; dk++) {
                const double wx = di ? ax1 : ax0, wy = dj ? ay1 : ay0, wz = dk ? az1 : az0;
                bdep(b3, plane, L, My, Mz, itmp + di, jtmp + dj, ktmp + dk,
                     drho * wx * wy * wz, djx * wx * wy * wz);
            }
}

template <class T>
int launch_beam_push(const BeamArgs<T>& a, cudaStream_t st) {
    if (a.n <= 0) return 0;
    beam_push_kernel<T><<<(unsigned)((a.n + 255) / 256), 256, 0, st>>>(a);
    return 1;
}

template int launch_beam_push<float>(const BeamArgs<float>&, cudaStream_t);
template int launch_beam_push<double>(const BeamArgs<double>&, cudaStream_t);

}  // namespace qs
