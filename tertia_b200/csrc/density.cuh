// density.cuh — plasma density profiles of Specie::Density (plasma.cpp:6-399)
// as one __host__ __device__ function: the front-seeding kernel evaluates it
// per cell, the host once per march for the density of the Guess/Iterate maps.
//
// Differences from the reference, all without effect on the steady result:
//   * the reference replaces non-positive radii (and Scale) by defaults in the
//     Specie members on its first call; here the defaults are taken locally
//     on every call, which is what the reference computes from its second
//     call on (its very first COS-GAUSS call reads RadiusX before defaulting);
//   * the periodic reductions (plasma.cpp:47-52, 98-114) subtract a whole
//     number of periods at once instead of one period per loop pass, so a
//     coordinate many periods away may differ by rounding; the loops'
//     end intervals ((0, P] and [0, P) for x, (-P/2, P/2] for y and z) are kept.
#pragma once
#include <math.h>

#include "../../include/qsb200.h"

#if defined(__CUDACC__)
#define QS_HD __host__ __device__
#else
#define QS_HD
#endif

namespace qs {

constexpr double kRefPi = 3.1415927;   // the reference's PI (domain.h:10)

// x reduced like `while (x > P) x -= P; while (x < 0) x += P;` (P > 0)
QS_HD inline double reduce_period(double x, double P) {
    if (x > P) {
        x -= P * (ceil(x / P) - 1.0);
        for (int i = 0; i < 2 && x > P; i++) x -= P;
        for (int i = 0; i < 2 && x <= 0.0; i++) x += P;
    } else if (x < 0.0) {
        x += P * ceil(-x / P);
        for (int i = 0; i < 2 && x < 0.0; i++) x += P;
        for (int i = 0; i < 2 && x >= P; i++) x -= P;
    }
    return x;
}

// v reduced like `while (v > P/2) v -= P; while (v <= -P/2) v += P;` (P > 0)
QS_HD inline double reduce_half_period(double v, double P) {
    if (v > 0.5 * P || v <= -0.5 * P) {
        v -= P * floor(v / P + 0.5);
        for (int i = 0; i < 2 && v > 0.5 * P; i++) v -= P;
        for (int i = 0; i < 2 && v <= -0.5 * P; i++) v += P;
    }
    return v;
}

// ramps of the trapezoid-like profiles: rising over [begin, plateau_begin],
// falling over [plateau_end, end]
QS_HD inline double up_ramp(const qs_density_profile& p, double x) {
    return (x - p.begin) / (p.plateau_begin - p.begin);
}
QS_HD inline double down_ramp(const qs_density_profile& p, double x) {
    return (p.end - x) / (p.end - p.plateau_end);
}

// Specie::Density(xco, yco, zco); the expression order of each case follows
// the reference so that the host and the device agree to the last bits of
// the math library.
QS_HD inline double profile_density(const qs_density_profile& p, double x, double y, double z) {
    const double n0 = p.density;
    const double R = p.radius <= 0.0 ? 1.0 : p.radius;
    switch (p.distribution) {
    case 12: {   // periodic (:30-58)
        if (x < p.begin || x > p.end) return 0.0;
        if (x < p.plateau_begin) {
            const double sc = p.scale <= 0.0 ? 1.0 : p.scale;
            return n0 * exp((x - p.plateau_begin) / sc);
        }
        if (x > p.plateau_end) return n0 * (p.end - x) / (p.end - p.plateau_end);
        const double n1 = p.density1 < 0.0 ? 0.0 : p.density1;
        const double xt = reduce_period(x, p.xperiod);
        return xt > p.xperiod - p.delta ? n1 : n0;
    }
    case 11:     // gradient (:60-73)
        if (x < 0.0 || x < p.begin || x > p.end) return 0.0;
        if (x < p.plateau_begin) return n0 * (x - p.begin) / (p.plateau_begin - p.begin);
        if (x < p.plateau_end) return n0 * exp((x - p.plateau_begin) / p.delta);
        if (x > p.plateau_end) return n0 * (p.end - x) / (p.end - p.plateau_end);
        return 0.0;
    case 10:     // linear step (:74-90)
        if (x < 0.0 || x < p.begin || x > p.end) return 0.0;
        if (x < p.plateau_begin) return n0;
        if (x < p.plateau_end)
            return n0 + n0 * p.delta * (x - p.plateau_begin) / (p.plateau_end - p.plateau_begin);
        if (x > p.plateau_end) return n0 * (1. + p.delta);
        return 0.0;
    case 9: {    // round and gophered rod (:91-141)
        if (x < p.begin || x > p.end) return 0.0;
        y = y + p.angle_y * (x - p.begin);
        if (p.yperiod > 0.0) y = reduce_half_period(y, p.yperiod);
        if (p.zperiod > 0.0) z = reduce_half_period(z, p.zperiod);
        const double ry = p.radius_y == 0.0 ? R : p.radius_y;
        const double rz = p.radius_z == 0.0 ? R : p.radius_z;
        double arg = (y - p.y0) * (y - p.y0) / ry / ry + (z - p.z0) * (z - p.z0) / rz / rz;
        if (p.xperiod > 0.0) arg *= 1 + p.delta * sin(2. * kRefPi * x / p.xperiod);
        if ((ry > 0 || rz > 0) && arg > 1) return 0.0;
        if ((ry < 0 || rz < 0) && arg < 1) return 0.0;
        return n0;
    }
    case 8: {    // tanh step (:142-160)
        if (x < 0.0 || x < p.begin || x > p.end) return 0.0;
        const double r2 = y * y + z * z;
        if (r2 > p.radius * p.radius) return 0.0;
        const double rx = p.radius_x <= 0.0 ? 1.0 : p.radius_x;
        return n0 * (0.5 * (1. - tanh((x - p.x0) / rx)));
    }
    case 7: {    // COS-GAUSS (:161-223)
        if (x < 0.0 || x < p.begin || x > p.end) return 0.0;
        const double rx = p.radius_x <= 0.0 ? R : p.radius_x;
        const double ry0 = p.radius_y <= 0.0 ? R : p.radius_y;
        const double rz0 = p.radius_z <= 0.0 ? R : p.radius_z;
        double front = p.end - p.x0;
        front = front < rx ? 1.0 : rx * 100.;
        double arg_front = 0.0;
        if (x > p.x0) arg_front = (x - p.x0) / front;
        arg_front *= arg_front / 2.;
        double arg = (x - p.x0) / rx;
        if (fabs(arg) > sqrt(2. * kRefPi)) return 0.0;
        double dn = 0.5 * (1 + cos(sqrt(kRefPi / 2.) * arg));
        double mod = p.xperiod != 0.0 ? 1. + p.delta * cos(2 * kRefPi * x / p.xperiod) : 1.;
        if (mod <= 0.0) mod = 1.;
        const double ry = ry0 * mod, rz = rz0 * mod;
        dn = dn / (mod * mod);
        arg = 0.5 * (y - p.y0) * (y - p.y0) / ry / ry + 0.5 * (z - p.z0) * (z - p.z0) / rz / rz;
        if (arg > 4) return 0.0;
        dn *= exp(-arg - arg_front);
        if (x > p.plateau_end && x < p.end) {
            const double xmid = (p.end + p.plateau_end) / 2.;
            const double width = p.end - p.plateau_end;
            dn *= 0.5 * (1. - tanh(4. * (x - xmid) / width));
        }
        return n0 * dn;
    }
    case 6: {    // empty channel (:224-251)
        if (x < 0.0 || x < p.begin || x > p.end) return 0.0;
        const double r2 = (y - p.y0) * (y - p.y0) + (z - p.z0) * (z - p.z0);
        double d = n0;
        if (r2 < R * R) d *= p.delta;
        if (x < p.plateau_begin) return d * up_ramp(p, x);
        if (x > p.plateau_end) return d * down_ramp(p, x);
        return d;
    }
    case 5:      // exponential (:252-266)
        if (x < 0.0 || x < p.begin || x > p.end) return 0.0;
        if (x < p.plateau_begin)
            return 0.5 * n0 * (1. + tanh(5. * (x - p.begin) / (p.plateau_begin - p.begin)));
        if (x > p.plateau_end) return n0 * (1. + p.delta) * (p.end - x) / (p.end - p.plateau_end);
        return n0 * (1. + p.delta * (x - p.plateau_begin) / (p.plateau_end - p.plateau_begin));
    case 4: {    // parallelepiped (:267-287)
        const double rx = p.radius_x <= 0.0 ? R : p.radius_x;
        const double ry = p.radius_y <= 0.0 ? R : p.radius_y;
        const double rz = p.radius_z <= 0.0 ? R : p.radius_z;
        if (fabs(x - p.x0) > rx || fabs(y - p.y0) > ry || fabs(z - p.z0) > rz) return 0.0;
        return n0;
    }
    case 3: {    // curved Gaussian channel (:288-322)
        if (x < 0.0 || x < p.begin || x > p.end) return 0.0;
        double yc = p.y0, zc = p.z0;
        if (p.xperiod > 0.0 && x > p.curvature_begin && x < p.curvature_end) {
            yc = p.y0 + p.y_curvature * sin(2. * kRefPi * x / p.xperiod);
            zc = p.z0 + p.z_curvature * cos(2. * kRefPi * x / p.xperiod);
        }
        const double r2 = (y - yc) * (y - yc) + (z - zc) * (z - zc);
        const double arg = r2 / R / R;
        double t = 0.0;
        if (arg < 2) t = p.delta * exp(-arg);
        if (t < 0) t = 0.0;
        if (t > 1) t = 1.0;
        const double d = n0 * (1. - t);
        if (x < p.plateau_begin) return d * up_ramp(p, x);
        if (x > p.plateau_end) return d * down_ramp(p, x);
        return d;
    }
    case 2: {    // Gaussian channel (:323-350)
        if (x < 0.0 || x < p.begin || x > p.end) return 0.0;
        const double r2 = (y - p.y0) * (y - p.y0) + (z - p.z0) * (z - p.z0);
        const double arg = r2 / R / R;
        double t = 0.0;
        if (arg < 10) t = p.delta * exp(-arg);
        if (t < 0) t = 0.0;
        if (t > 1) t = 1.0;
        if (x < p.plateau_begin)
            return n0 * (x - p.begin) / (p.plateau_begin - p.begin) * (1. - t);
        if (x > p.plateau_end)
            return p.density1 * (p.end - x) / (p.end - p.plateau_end) * (1. - t);
        return (1. - t) * (n0 * (p.plateau_end - x) + p.density1 * (x - p.plateau_begin)) /
               (p.plateau_end - p.plateau_begin);
    }
    case 1: {    // Gaussian ellipsoid (:351-379)
        if (x < p.begin || x > p.end) return 0.0;
        const double rx = p.radius_x <= 0.0 ? R : p.radius_x;
        const double ry = p.radius_y <= 0.0 ? R : p.radius_y;
        const double rz = p.radius_z <= 0.0 ? R : p.radius_z;
        const double arg = (x - p.x0) * (x - p.x0) / rx / rx + (y - p.y0) * (y - p.y0) / ry / ry +
                           (z - p.z0) * (z - p.z0) / rz / rz;
        if (arg > 16) return 0.0;
        const double xp = p.xperiod <= 0.0 ? 1.0 : p.xperiod;
        return n0 * exp(-arg) * (1. + p.delta * cos(2 * kRefPi * (x - p.x0) / xp));
    }
    default:     // trapezoid (:380-392), also for unknown numbers
        if (x < 0.0 || x < p.begin || x > p.end) return 0.0;
        if (x < p.plateau_begin) return n0 * (x - p.begin) / (p.plateau_begin - p.begin);
        if (x > p.plateau_end) return n0 * (p.end - x) / (p.end - p.plateau_end);
        return n0;
    }
}

}  // namespace qs
