// qs_oracle.cpp — CPU oracle of the quasi-static xi-layer loop.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker that the GPU product
// path is compared against (tests, smoke check, CPU baseline of the bench).
// It is a literal FP64 restatement of the reference's live host path; each
// function cites the reference lines it follows.  Parity status is stated
// in qs_oracle.h.
#include "qs_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef std::complex<double> cplx;

// ---------------------------------------------------------------------------
// Half-integer transforms: FFTW REDFT11 / RODFT11 (the kinds the reference
// plans at movefieldshydrolinlayersplit.cpp:389-427).
//   REDFT11: Y_k = 2 sum_j X_j cos(pi (j+1/2)(k+1/2)/n)
//   RODFT11: Y_k = 2 sum_j X_j sin(pi (j+1/2)(k+1/2)/n)
// Fast form (n a power of two, n >= 2): the DCT-IV through an n/2-point
// complex FFT,  z_m = (x_{2m} + i x_{n-1-2m}) e^{-i pi m/n},
// S_p = e^{-i pi (p+1/4)/n} FFT_{n/2}(z)_p,  Y_{2p} = 2 Re S_p,
// Y_{n-1-2p} = -2 Im S_p.  The DST-IV follows from
// DST-IV(x)_k = (-1)^k DCT-IV(reverse x)_k.
// ---------------------------------------------------------------------------
struct Dtt1Plan {
    int n = 0;
    bool fast = false;
    int m = 0;                       // n/2
    std::vector<cplx> pre, post, tw;  // pre[m], post[p], FFT twiddles
    std::vector<int> rev;
    std::vector<double> cosTab, sinTab;  // direct tables (n*n)
};

std::mutex g_plan_mutex;
std::map<int, std::shared_ptr<Dtt1Plan>> g_plans;

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

std::shared_ptr<Dtt1Plan> get_plan(int n) {
    std::lock_guard<std::mutex> lock(g_plan_mutex);
    auto it = g_plans.find(n);
    if (it != g_plans.end()) return it->second;
    auto p = std::make_shared<Dtt1Plan>();
    p->n = n;
    p->fast = is_pow2(n) && n >= 2;
    if (p->fast) {
        int m = n / 2;
        p->m = m;
        p->pre.resize(m);
        p->post.resize(m);
        for (int i = 0; i < m; i++) {
            p->pre[i] = std::polar(1.0, -M_PI * i / n);
            p->post[i] = std::polar(1.0, -M_PI * (i + 0.25) / n);
        }
        p->tw.resize(m > 1 ? m / 2 : 1);
        for (int i = 0; i < (int)p->tw.size(); i++)
            p->tw[i] = std::polar(1.0, -2.0 * M_PI * i / m);
        p->rev.resize(m);
        int bits = 0;
        while ((1 << bits) < m) bits++;
        for (int i = 0; i < m; i++) {
            int r = 0;
            for (int b = 0; b < bits; b++)
                if (i & (1 << b)) r |= 1 << (bits - 1 - b);
            p->rev[i] = r;
        }
    }
    // direct tables are kept for every n (tests use them as the O(N^2) sums)
    if (n <= 4096) {
        p->cosTab.resize((size_t)n * n);
        p->sinTab.resize((size_t)n * n);
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++) {
                double a = M_PI * (j + 0.5) * (k + 0.5) / n;
                p->cosTab[(size_t)k * n + j] = std::cos(a);
                p->sinTab[(size_t)k * n + j] = std::sin(a);
            }
    }
    g_plans[n] = p;
    return p;
}

void fft_inplace(const Dtt1Plan& p, cplx* a) {
    const int m = p.m;
    for (int i = 0; i < m; i++)
        if (i < p.rev[i]) std::swap(a[i], a[p.rev[i]]);
    for (int len = 2; len <= m; len <<= 1) {
        const int half = len >> 1, step = m / len;
        for (int s = 0; s < m; s += len)
            for (int t = 0; t < half; t++) {
                cplx w = p.tw[t * step];
                cplx u = a[s + t], v = a[s + t + half] * w;
                a[s + t] = u + v;
                a[s + t + half] = u - v;
            }
    }
}

void dct4_fast(const Dtt1Plan& p, const double* x, double* y, cplx* work) {
    const int n = p.n, m = p.m;
    for (int i = 0; i < m; i++) work[i] = cplx(x[2 * i], x[n - 1 - 2 * i]) * p.pre[i];
    fft_inplace(p, work);
    for (int i = 0; i < m; i++) {
        cplx s = work[i] * p.post[i];
        y[2 * i] = 2.0 * s.real();
        y[n - 1 - 2 * i] = -2.0 * s.imag();
    }
}

void dtt1(const Dtt1Plan& p, int kind, const double* x, double* y, bool direct,
          std::vector<double>& tmp, std::vector<cplx>& work) {
    const int n = p.n;
    if (direct || !p.fast) {
        const std::vector<double>& tab = (kind == QS_REDFT11) ? p.cosTab : p.sinTab;
        if (tab.empty()) {  // very large non power of two: compute on the fly
            for (int k = 0; k < n; k++) {
                double s = 0.0;
                for (int j = 0; j < n; j++) {
                    double a = M_PI * (j + 0.5) * (k + 0.5) / n;
                    s += x[j] * (kind == QS_REDFT11 ? std::cos(a) : std::sin(a));
                }
                y[k] = 2.0 * s;
            }
            return;
        }
        for (int k = 0; k < n; k++) {
            const double* row = &tab[(size_t)k * n];
            double s = 0.0;
            for (int j = 0; j < n; j++) s += x[j] * row[j];
            y[k] = 2.0 * s;
        }
        return;
    }
    work.resize(p.m);
    if (kind == QS_REDFT11) {
        dct4_fast(p, x, y, work.data());
    } else {
        tmp.resize(n);
        for (int j = 0; j < n; j++) tmp[j] = x[n - 1 - j];
        dct4_fast(p, tmp.data(), y, work.data());
        for (int k = 1; k < n; k += 2) y[k] = -y[k];
    }
}

// 2-D transform of one nz x ny plane (y fastest), like
// fftw_plan_r2r_2d(nz, ny, in, out, kind_z, kind_y).
void r2r_2d(int nz, int ny, int kind_z, int kind_y, const double* in, double* out,
            bool direct = false) {
    auto py = get_plan(ny);
    auto pz = get_plan(nz);
    std::vector<double> mid((size_t)nz * ny);
#pragma omp parallel
    {
        std::vector<double> tmp;
        std::vector<cplx> work;
#pragma omp for schedule(static)
        for (int k = 0; k < nz; k++)
            dtt1(*py, kind_y, in + (size_t)k * ny, &mid[(size_t)k * ny], direct, tmp, work);
        std::vector<double> col(nz), res(nz);
#pragma omp for schedule(static)
        for (int j = 0; j < ny; j++) {
            for (int k = 0; k < nz; k++) col[k] = mid[(size_t)k * ny + j];
            dtt1(*pz, kind_z, col.data(), res.data(), direct, tmp, work);
            for (int k = 0; k < nz; k++) out[(size_t)k * ny + j] = res[k];
        }
    }
}

// ---------------------------------------------------------------------------
// Plasma sub-push of one particle (MoveParticlesLayerSplit,
// movepart_splitlayer.cpp:882-1522, reference live NGP path) and the CIC
// variant (weights of movepart_layer_CIC.cpp:165-193 / 449-496).
// The arithmetic follows the reference expression by expression; T is
// double for the oracle proper and float for the FP32 bit-exactness check.
// ---------------------------------------------------------------------------
template <class T>
struct PushParams {
    int My, Mz;
    T hx, hy, hz;              // hx = HxSplit*part
    T q2m, djx0, djy0, djz0, drho0;
    T bXext, bYext, bZext;
    int shape;                 // qs_shape
    bool precise;              // cell-relative position update (FP32 path form)
};

template <class T>
PushParams<T> make_params(const qs_config* c) {
    PushParams<T> p;
    p.My = c->ny;
    p.Mz = c->nz;
    p.hx = (T)(c->hx / (c->nx_split > 0 ? c->nx_split : 1));
    p.hy = (T)c->hy;
    p.hz = (T)c->hz;
    p.q2m = (T)c->plasma_q2m;
    p.djx0 = (T)c->plasma_djx0;
    p.djy0 = (T)c->plasma_djy0;
    p.djz0 = (T)c->plasma_djz0;
    p.drho0 = (T)c->plasma_drho0;
    p.bXext = (T)c->bx_ext;
    p.bYext = (T)c->by_ext;
    p.bZext = (T)c->bz_ext;
    p.shape = c->shape;
    p.precise = false;
    return p;
}

// Field access on interior planes with periodic wrap (the guard copies of
// ExchangeFieldsSplit, movepart_splitlayer.cpp:1659-1682).
template <class T>
struct PlaneSet {
    const T* f[6];
    int My, Mz;
    T at(int c, int j, int k) const {
        j %= My; if (j < 0) j += My;
        k %= Mz; if (k < 0) k += Mz;
        return f[c][(size_t)j + (size_t)My * k];
    }
};

template <class T>
struct DepositSink {
    T* d[4];  // Jx, Jy, Jz, Dens (interior, periodic fold applied)
    int My, Mz;
    void add(int j, int k, T jx, T jy, T jz, T rho) {
        j %= My; if (j < 0) j += My;
        k %= Mz; if (k < 0) k += Mz;
        size_t n = (size_t)j + (size_t)My * k;
        d[0][n] += jx; d[1][n] += jy; d[2][n] += jz; d[3][n] += rho;
    }
};

// Returns the folded cell of the last deposit.  j,k: the particle's cell.
template <class T>
int push_one(const PushParams<T>& pp, const PlaneSet<T>& P, const PlaneSet<T>& C,
             DepositSink<T>& dep, int& j_io, int& k_io, T& y_io, T& z_io, T& px_io,
             T& py_io, T& pz_io, T weight, bool full) {
    const int j = j_io, k = k_io;
    const T one = (T)1, two = (T)2, half = (T)0.5;
    const T yp = y_io, zp = z_io;
    T px = px_io, py = py_io, pz = pz_io;
    T gammap = std::sqrt(one + px * px + py * py + pz * pz);
    T Vx = px / gammap;
    T Vxp = Vx, Vyp = py / gammap, Vzp = pz / gammap;
    T q2m = pp.q2m;
    T ex, ey, ez, bx, by, bz;
    if (pp.shape == QS_SHAPE_NGP) {
        // :1100-1217 NGP gather at the particle's cell from P and C, averaged
        ex = half * (P.at(0, j, k) + C.at(0, j, k));
        ey = half * (P.at(1, j, k) + C.at(1, j, k));
        ez = half * (P.at(2, j, k) + C.at(2, j, k));
        bx = half * (P.at(3, j, k) + C.at(3, j, k));
        by = half * (P.at(4, j, k) + C.at(4, j, k));
        bz = half * (P.at(5, j, k) + C.at(5, j, k));
    } else {
        // bilinear weights of movepart_layer_CIC.cpp:165-193 at the particle
        T ayc = one - yp, ayp = yp, azc = one - zp, azp = zp;
        T acc = ayc * azc, apc = ayp * azc, acp = ayc * azp, app = ayp * azp;
        T g[6];
        for (int c = 0; c < 6; c++) {
            T vp = acc * P.at(c, j, k) + apc * P.at(c, j + 1, k) + acp * P.at(c, j, k + 1) +
                   app * P.at(c, j + 1, k + 1);
            T vc = acc * C.at(c, j, k) + apc * C.at(c, j + 1, k) + acp * C.at(c, j, k + 1) +
                   app * C.at(c, j + 1, k + 1);
            g[c] = half * (vp + vc);
        }
        ex = g[0]; ey = g[1]; ez = g[2]; bx = g[3]; by = g[4]; bz = g[5];
    }
    const T hx = pp.hx;
    // :1245-1247
    T sE = q2m * hx / two;
    ex *= sE;
    ey *= sE;
    ez *= sE;
    // :1260-1262
    px += ex / (one - Vx);
    py += ey / (one - Vx);
    pz += ez / (one - Vx);
    T gamma = std::sqrt(one + px * px + py * py + pz * pz);
    T gamma_r = one / gamma;
    bx += pp.bXext;
    by += pp.bYext;
    bz += pp.bZext;
    // :1282-1284
    bx = bx * gamma_r * q2m / (one - Vx) * hx / two;
    by = by * gamma_r * q2m / (one - Vx) * hx / two;
    bz = bz * gamma_r * q2m / (one - Vx) * hx / two;
    T co = two / (one + (bx * bx) + (by * by) + (bz * bz));
    T p3x = py * bz - pz * by + px;
    T p3y = pz * bx - px * bz + py;
    T p3z = px * by - py * bx + pz;
    p3x *= co;
    p3y *= co;
    p3z *= co;
    T px_new = p3y * bz - p3z * by;
    T py_new = p3z * bx - p3x * bz;
    T pz_new = p3x * by - p3y * bx;
    // :1314-1316
    px += ex / (one - Vx) + px_new;
    py += ey / (one - Vx) + py_new;
    pz += ez / (one - Vx) + pz_new;
    gamma = std::sqrt(one + px * px + py * py + pz * pz);
    T Vxm = px / gamma, Vym = py / gamma, Vzm = pz / gamma;
    Vx = half * (Vxm + Vxp);
    T Vy = half * (Vym + Vyp);
    T Vz = half * (Vzm + Vzp);
    // :1337-1340
    T djx = weight * pp.djx0 * Vxm;
    T djy = weight * pp.djy0 * Vym;
    T djz = weight * pp.djz0 * Vzm;
    T drho = weight * pp.drho0;
    // :1356-1359
    djx *= one / (one - Vx);
    djy *= one / (one - Vx);
    djz *= one / (one - Vx);
    drho *= one / (one - Vx);
    // :1365-1371
    T dy = Vy * hx / pp.hy;
    T dz = Vz * hx / pp.hz;
    dy = dy / (one - Vx);
    dz = dz / (one - Vx);
    // :1389-1404 sub-cycling set-up
    T partdx = 0, step = one;
    if (std::fabs(dy) > one || std::fabs(dz) > one) {
        if (std::fabs(dy) > std::fabs(dz)) step = partdx = std::fabs(dy);
        else step = partdx = std::fabs(dz);
    }
    if (partdx < one) partdx = step = one;
    const T My = (T)pp.My, Mz = (T)pp.Mz;
    T ytmp = yp, ztmp = zp;
    int jb = j, kb = k;   // base cell used by the position update
    int jj = j, kk = k;   // cell of the last deposit
    while (partdx > 0) {
        T part_step;
        if (partdx > one) {
            partdx -= one;
            part_step = one / step;
        } else {
            part_step = partdx / step;
            partdx = 0;
        }
        if (pp.shape == QS_SHAPE_NGP && !pp.precise) {
            // :1420-1437 the reference form.  j_jump here is the OUTER
            // variable (= j, :1380): the inner `int j_jump` of :1434 is
            // declared after this statement.
            ytmp += dy * part_step + (T)j;
            ztmp += dz * part_step + (T)k;
            while (ytmp > My) ytmp -= My;
            while (ytmp < 0) ytmp += My;
            while (ztmp > Mz) ztmp -= Mz;
            while (ztmp < 0) ztmp += Mz;
            jj = (int)ytmp;
            kk = (int)ztmp;
            ytmp -= (T)jj;
            ztmp -= (T)kk;
        } else {
            // cell-relative form: u = frac + d*part_step measured from the
            // base cell; NGP keeps the reference's base cell j (see above),
            // CIC moves the base cell with the particle.
            T uy = ytmp + dy * part_step;
            T uz = ztmp + dz * part_step;
            T fy = std::floor(uy), fz = std::floor(uz);
            T ry = uy - fy, rz = uz - fz;
            int sy = (int)fy, sz = (int)fz;
            if (ry >= one) { ry = 0; sy += 1; }
            if (rz >= one) { rz = 0; sz += 1; }
            int base_j = (pp.shape == QS_SHAPE_NGP) ? j : jb;
            int base_k = (pp.shape == QS_SHAPE_NGP) ? k : kb;
            jj = (base_j + sy) % pp.My; if (jj < 0) jj += pp.My;
            kk = (base_k + sz) % pp.Mz; if (kk < 0) kk += pp.Mz;
            ytmp = ry;
            ztmp = rz;
            jb = jj;
            kb = kk;
        }
        // DepositCurrentsInCellSplit :1547-1615 (NGP, live lines :1612-1615)
        // or the 4-point CIC of MoveInCell, movepart_layer_CIC.cpp:449-496
        T s = part_step;
        if (pp.shape == QS_SHAPE_NGP) {
            dep.add(jj, kk, djx * s, djy * s, djz * s, drho * s);
        } else {
            T ayp = ytmp, ayc = one - ayp, azp = ztmp, azc = one - azp;
            T w00 = ayc * azc, w10 = ayp * azc, w01 = ayc * azp, w11 = ayp * azp;
            T a = djx * s, b = djy * s, c = djz * s, r = drho * s;
            dep.add(jj, kk, a * w00, b * w00, c * w00, r * w00);
            dep.add(jj + 1, kk, a * w10, b * w10, c * w10, r * w10);
            dep.add(jj, kk + 1, a * w01, b * w01, c * w01, r * w01);
            dep.add(jj + 1, kk + 1, a * w11, b * w11, c * w11, r * w11);
        }
    }
    int jf = jj % pp.My; if (jf < 0) jf += pp.My;
    int kf = kk % pp.Mz; if (kf < 0) kf += pp.Mz;
    if (full) {
        // :1501-1512: p <- (px,py,pz), x <- (0, ytmp, ztmp); relinked to
        // GetNyz(jtmp,ktmp) with the OUTER jtmp = j, ktmp = k (:1348-1350):
        // in the live path a particle keeps its cell.
        px_io = px;
        py_io = py;
        pz_io = pz;
        y_io = ytmp;
        z_io = ztmp;
        if (pp.shape == QS_SHAPE_CIC) {
            j_io = jf;
            k_io = kf;
        }
    }
    return jf + pp.My * kf;
}

template <class T>
int push_layer_arrays(const qs_config* cfg, int64_t n, int32_t* cell, T* y, T* z, T* px,
                      T* py, T* pz, const T* w, const T* P, const T* C, T* dep,
                      int32_t* dep_cell, int full, int precise) {
    if (!cfg || n < 0) return QS_ERR_INVALID;
    PushParams<T> pp = make_params<T>(cfg);
    pp.precise = precise != 0;
    const size_t plane = (size_t)cfg->ny * cfg->nz;
    PlaneSet<T> Ps, Cs;
    Ps.My = Cs.My = cfg->ny;
    Ps.Mz = Cs.Mz = cfg->nz;
    for (int c = 0; c < 6; c++) {
        Ps.f[c] = P + c * plane;
        Cs.f[c] = C + c * plane;
    }
    DepositSink<T> sink;
    sink.My = cfg->ny;
    sink.Mz = cfg->nz;
    for (int c = 0; c < 4; c++) sink.d[c] = dep + c * plane;
    for (int64_t i = 0; i < n; i++) {
        if (!(y[i] >= 0 && y[i] <= 1 && z[i] >= 0 && z[i] <= 1)) return QS_ERR_PARTICLE_RANGE;
        int jc = cell[i] % cfg->ny, kc = cell[i] / cfg->ny;
        int dc = push_one<T>(pp, Ps, Cs, sink, jc, kc, y[i], z[i], px[i], py[i], pz[i], w[i],
                             full != 0);
        if (dep_cell) dep_cell[i] = dc;
        if (full) cell[i] = jc + cfg->ny * kc;
    }
    return QS_OK;
}

// ---------------------------------------------------------------------------
// The oracle mesh: P/C transverse layers with a guard ring of 2 cells
// (l_dMy = l_dMz = 2, domain.cpp:140-145), the 3-D layer array, the
// spectral work arrays of the Guess/Iterate solve, plasma and beam particles.
// ---------------------------------------------------------------------------
enum { NPL = 12 };  // Ex Ey Ez Bx By Bz Jx Jy Jz Dens RhoBeam JxBeam

// Per-mode linear predictor of GuessFieldsHydroLinLayerSplit
// (movefieldshydrolinlayersplit.cpp:808-900; the same formulas as the
// reference's CUDA twin linearized_kernel, CUDA_WRAP/linearized.cu:11-103).
// Inputs: P-layer spectra and beam spectra; outputs: C-layer spectra.
extern "C" void qso_predictor_modes(int ny, int nz, double hx, double d, double Ylength,
                                    double Zlength, const double* fRhoP, const double* fJxP,
                                    const double* fJyP, const double* fJzP, const double* fExP,
                                    const double* fEyP, const double* fEzP,
                                    const double* fRhoBeam, const double* fRhoBeamP,
                                    const double* fJxBeam, double* fRho, double* fEx,
                                    double* fEy, double* fEz, double* fJx, double* fJy,
                                    double* fJz, double* fBx, double* fBy, double* fBz) {
    const double hxs = hx;
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++) {
            double akz = M_PI / Zlength * (k + 0.5);
            double aky = M_PI / Ylength * (j + 0.5);
            double ak2 = aky * aky + akz * akz;
            size_t n1 = (size_t)j + (size_t)ny * k;
            double rp = fRhoP[n1];
            double jxp = fJxP[n1];
            double jyp = fJyP[n1];
            double jzp = fJzP[n1];
            double exp_ = fExP[n1];
            double eyp = fEyP[n1];
            double ezp = fEzP[n1];
            double rb = fRhoBeam[n1];
            double rbp = fRhoBeamP[n1];
            double propagator = (4. - d * hxs * hxs) / (4. + d * hxs * hxs);
            double denominator = 4. + d * hxs * hxs;
            fRho[n1] = propagator * rp - (rb + rbp) * d * hxs * hxs / denominator +
                       4. * exp_ * hxs * (ak2 + d) / denominator;
            fEx[n1] = propagator * exp_ -
                      2. * (2. * rp + rb + rbp) * d * hxs / ((ak2 + d) * denominator);
            fEy[n1] = -eyp + aky * (rb + rbp + rp + fRho[n1]) / (d + ak2);
            fEz[n1] = -ezp + akz * (rb + rbp + rp + fRho[n1]) / (d + ak2);
            fJy[n1] = jyp + hxs * d * (fEy[n1] + eyp) / 2.;
            fJz[n1] = jzp + hxs * d * (fEz[n1] + ezp) / 2.;
            fJx[n1] = jxp + hxs * d * (fEx[n1] + exp_) / 2.;
            fBx[n1] = -aky / ak2 * fJz[n1] + akz / ak2 * fJy[n1];
            fBy[n1] = (-akz * (fJx[n1] + fJxBeam[n1]) + d * fEz[n1]) / ak2;
            fBz[n1] = (aky * (fJx[n1] + fJxBeam[n1]) - d * fEy[n1]) / ak2;
        }
}

// Per-mode corrector of IterateFieldsHydroLinLayerSplit
// (movefieldshydrolinlayersplit.cpp:1374-1477; the same formulas as the
// reference's CUDA twin linearizedIteratekernel, CUDA_WRAP/linearized.cu:105-209).
// fRho holds rho_old on entry and the new rho on exit.
extern "C" void qso_corrector_modes(int ny, int nz, double hx, double d, double Ylength,
                                    double Zlength, const double* fRhoP, const double* fJxP,
                                    const double* fJyP, const double* fJzP, const double* fEyP,
                                    const double* fEzP, const double* fRhoBeam,
                                    const double* fRhoBeamP, const double* fJxBeam,
                                    const double* fJx, const double* fJy, const double* fJz,
                                    double* fRho, double* fEx, double* fEy, double* fEz,
                                    double* fBx, double* fBy, double* fBz) {
    const double hxs = hx;
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++) {
            double akz = M_PI / Zlength * (k + 0.5);
            double aky = M_PI / Ylength * (j + 0.5);
            double ak2 = aky * aky + akz * akz;
            size_t n1 = (size_t)j + (size_t)ny * k;
            double rp = fRhoP[n1];
            double jy = fJy[n1];
            double jz = fJz[n1];
            double rho = rp + fJx[n1] - fJxP[n1] -
                         hxs * (aky * (jy + fJyP[n1]) + akz * (jz + fJzP[n1])) / 2.;
            double rb = fRhoBeam[n1];
            double rbp = fRhoBeamP[n1];
            double eyp = fEyP[n1];
            double ezp = fEzP[n1];
            double newEx = -(aky * jy + akz * jz) / ak2;
            double newEy = -eyp + aky * (rb + rbp + rp + fRho[n1]) / (d + ak2);
            double newEz = -ezp + akz * (rb + rbp + rp + fRho[n1]) / (d + ak2);
            fEy[n1] = newEy;
            fEz[n1] = newEz;
            fRho[n1] = rho;
            fEx[n1] = newEx;
            fBx[n1] = -aky / ak2 * fJz[n1] + akz / ak2 * fJy[n1];
            fBy[n1] = (-akz * (fJx[n1] + fJxBeam[n1]) + d * newEz) / ak2;
            fBz[n1] = (aky * (fJx[n1] + fJxBeam[n1]) - d * newEy) / ak2;
        }
}

// ---- Specie::Density (plasma.cpp:6-399).  The Specie members the reference
// defaults on the fly (Radius, RadiusX/Y/Z, Scale) are defaulted in a copy
// first, as after the reference's first call; the periodic reductions are
// the reference's loops (bounded).
struct SpecieProfile {
    qs_density_profile q;
    explicit SpecieProfile(const qs_density_profile& p) : q(p) {}

    static double wrap_up(double v, double P, long cap = 100000000L) {
        while (v > P && cap-- > 0) v -= P;
        while (v < 0. && cap-- > 0) v += P;
        return v;
    }
    static double wrap_mid(double v, double P, long cap = 100000000L) {
        while (v > P / 2. && cap-- > 0) v -= P;
        while (v <= -P / 2. && cap-- > 0) v += P;
        return v;
    }

    double operator()(double xco, double yco, double zco) {
        const double PI_ = 3.1415927;  // domain.h:10
        double tmp = 0.;
        double density = q.density, density1 = q.density1;
        double arg, r2;
        switch (q.distribution) {
        case 12:
            if (xco < q.begin || xco > q.end) return tmp;
            if (xco < q.plateau_begin) {
                if (q.scale <= 0) q.scale = 1;
                return density * exp((xco - q.plateau_begin) / q.scale);
            }
            if (xco > q.plateau_end) return density * (q.end - xco) / (q.end - q.plateau_end);
            if (density1 < 0) density1 = 0.;
            return wrap_up(xco, q.xperiod) > q.xperiod - q.delta ? density1 : density;
        case 11:
            if (xco < 0. || xco < q.begin || xco > q.end) return 0.;
            if (xco < q.plateau_begin) return density * (xco - q.begin) / (q.plateau_begin - q.begin);
            if (xco < q.plateau_end) return density * exp((xco - q.plateau_begin) / q.delta);
            if (xco > q.plateau_end) return density * (q.end - xco) / (q.end - q.plateau_end);
            return 0.;
        case 10:
            if (xco < 0. || xco < q.begin || xco > q.end) return tmp;
            if (xco < q.plateau_begin) return q.density;
            if (xco < q.plateau_end)
                return density + density * q.delta * (xco - q.plateau_begin) /
                                     (q.plateau_end - q.plateau_begin);
            if (xco > q.plateau_end) return density * (1. + q.delta);
            return 0.;
        case 9:
            if (xco < q.begin || xco > q.end) return 0.;
            yco = yco + q.angle_y * (xco - q.begin);
            if (q.yperiod > 0.) yco = wrap_mid(yco, q.yperiod);
            if (q.zperiod > 0.) zco = wrap_mid(zco, q.zperiod);
            if (q.radius <= 0.) q.radius = 1.;
            if (q.radius_x <= 0.) q.radius_x = q.radius;
            if (q.radius_y == 0.) q.radius_y = q.radius;
            if (q.radius_z == 0.) q.radius_z = q.radius;
            arg = (yco - q.y0) * (yco - q.y0) / q.radius_y / q.radius_y +
                  (zco - q.z0) * (zco - q.z0) / q.radius_z / q.radius_z;
            if (q.xperiod > 0.) arg *= 1 + q.delta * sin(2. * PI_ * xco / q.xperiod);
            if ((q.radius_y > 0 || q.radius_z > 0) && arg > 1) return 0.;
            if ((q.radius_y < 0 || q.radius_z < 0) && arg < 1) return 0.;
            return q.density;
        case 8:
            if (xco < 0. || xco < q.begin || xco > q.end) return tmp;
            r2 = yco * yco + zco * zco;
            if (r2 > q.radius * q.radius) return tmp;
            if (q.radius_x <= 0.) q.radius_x = 1.;
            density = 0.5 * (1. - tanh((xco - q.x0) / q.radius_x));
            return q.density * density;
        case 7: {
            if (xco < 0. || xco < q.begin || xco > q.end) return tmp;
            if (q.radius <= 0.) q.radius = 1.;
            if (q.radius_x <= 0.) q.radius_x = q.radius;
            if (q.radius_y <= 0.) q.radius_y = q.radius;
            if (q.radius_z <= 0.) q.radius_z = q.radius;
            double front = q.end - q.x0;
            front = front < q.radius_x ? 1 : q.radius_x * 100.;
            double arg_front = 0.;
            if (xco > q.x0) arg_front = (xco - q.x0) / front;
            arg_front *= arg_front / 2.;
            arg = (xco - q.x0) / q.radius_x;
            if (fabs(arg) > sqrt(2. * PI_)) return tmp;
            density = 0.5 * (1 + cos(sqrt(PI_ / 2.) * arg));
            double modulation = q.xperiod != 0. ? 1. + q.delta * cos(2 * PI_ * xco / q.xperiod) : 1.;
            if (modulation <= 0.) modulation = 1.;
            const double Ry = q.radius_y * modulation, Rz = q.radius_z * modulation;
            density = density / (modulation * modulation);
            arg = 0.5 * (yco - q.y0) * (yco - q.y0) / Ry / Ry + 0.5 * (zco - q.z0) * (zco - q.z0) / Rz / Rz;
            if (arg > 4) return tmp;
            density *= exp(-arg - arg_front);
            if (xco > q.plateau_end && xco < q.end) {
                const double xmid = (q.end + q.plateau_end) / 2.;
                const double width = q.end - q.plateau_end;
                density *= 0.5 * (1. - tanh(4. * (xco - xmid) / width));
            }
            return q.density * density;
        }
        case 6:
            if (xco < 0. || xco < q.begin || xco > q.end) return tmp;
            r2 = (yco - q.y0) * (yco - q.y0) + (zco - q.z0) * (zco - q.z0);
            if (q.radius <= 0.) q.radius = 1.;
            if (r2 < q.radius * q.radius) density *= q.delta;
            if (xco < q.plateau_begin) {
                density *= (xco - q.begin) / (q.plateau_begin - q.begin);
                return density;
            }
            if (xco > q.plateau_end) {
                density *= (q.end - xco) / (q.end - q.plateau_end);
                return density;
            }
            return density;
        case 5:
            if (xco < 0. || xco < q.begin || xco > q.end) return tmp;
            if (xco < q.plateau_begin)
                return 0.5 * density * (1. + tanh(5. * (xco - q.begin) / (q.plateau_begin - q.begin)));
            if (xco > q.plateau_end)
                return density * (1. + q.delta) * (q.end - xco) / (q.end - q.plateau_end);
            return q.density * (1. + q.delta * (xco - q.plateau_begin) / (q.plateau_end - q.plateau_begin));
        case 4:
            if (q.radius <= 0.) q.radius = 1.;
            if (q.radius_x <= 0.) q.radius_x = q.radius;
            if (q.radius_y <= 0.) q.radius_y = q.radius;
            if (q.radius_z <= 0.) q.radius_z = q.radius;
            if (fabs(xco - q.x0) > q.radius_x) return 0.;
            if (fabs(yco - q.y0) > q.radius_y) return 0.;
            if (fabs(zco - q.z0) > q.radius_z) return 0.;
            return density;
        case 3: {
            if (xco < 0. || xco < q.begin || xco > q.end) return tmp;
            double y0 = q.y0, z0 = q.z0;
            if (q.xperiod > 0. && xco > q.curvature_begin && xco < q.curvature_end) {
                y0 = q.y0 + q.y_curvature * sin(2. * PI_ * xco / q.xperiod);
                z0 = q.z0 + q.z_curvature * cos(2. * PI_ * xco / q.xperiod);
            }
            r2 = (yco - y0) * (yco - y0) + (zco - z0) * (zco - z0);
            if (q.radius <= 0.) q.radius = 1.;
            arg = r2 / q.radius / q.radius;
            if (arg < 2) tmp = q.delta * exp(-arg);
            if (tmp < 0) tmp = 0.;
            if (tmp > 1) tmp = 1.;
            density *= (1. - tmp);
            if (xco < q.plateau_begin) {
                density *= (xco - q.begin) / (q.plateau_begin - q.begin);
                return density;
            }
            if (xco > q.plateau_end) {
                density *= (q.end - xco) / (q.end - q.plateau_end);
                return density;
            }
            return density;
        }
        case 2:
            if (xco < 0. || xco < q.begin || xco > q.end) return tmp;
            r2 = (yco - q.y0) * (yco - q.y0) + (zco - q.z0) * (zco - q.z0);
            if (q.radius <= 0.) q.radius = 1.;
            arg = r2 / q.radius / q.radius;
            if (arg < 10) tmp = q.delta * exp(-arg);
            if (tmp < 0) tmp = 0.;
            if (tmp > 1) tmp = 1.;
            if (xco < q.plateau_begin)
                return density * (xco - q.begin) / (q.plateau_begin - q.begin) * (1. - tmp);
            if (xco > q.plateau_end)
                return density1 * (q.end - xco) / (q.end - q.plateau_end) * (1. - tmp);
            return (1. - tmp) * (q.density * (q.plateau_end - xco) + q.density1 * (xco - q.plateau_begin)) /
                   (q.plateau_end - q.plateau_begin);
        case 1:
            if (xco < q.begin || xco > q.end) return 0.;
            if (q.radius <= 0.) q.radius = 1.;
            if (q.radius_x <= 0.) q.radius_x = q.radius;
            if (q.radius_y <= 0.) q.radius_y = q.radius;
            if (q.radius_z <= 0.) q.radius_z = q.radius;
            arg = (xco - q.x0) * (xco - q.x0) / q.radius_x / q.radius_x +
                  (yco - q.y0) * (yco - q.y0) / q.radius_y / q.radius_y +
                  (zco - q.z0) * (zco - q.z0) / q.radius_z / q.radius_z;
            if (arg > 16) return tmp;
            if (q.xperiod <= 0.) q.xperiod = 1.;
            return q.density * exp(-arg) * (1. + q.delta * cos(2 * PI_ * (xco - q.x0) / q.xperiod));
        default:
        case 0:
            if (xco < 0. || xco < q.begin || xco > q.end) return tmp;
            if (xco < q.plateau_begin) return density * (xco - q.begin) / (q.plateau_begin - q.begin);
            if (xco > q.plateau_end) return density * (q.end - xco) / (q.end - q.plateau_end);
            return q.density;
        }
    }
};

struct Oracle {
    qs_config cfg;
    int My = 0, Mz = 0, L = 0, NxSplit = 1, nIter = 1;
    static const int G = 2;
    int sy = 0, sz = 0;
    size_t nyz = 0;       // guarded plane size
    size_t nI = 0;        // interior plane size
    double hx = 0, hy = 0, hz = 0, Ylength = 0, Zlength = 0, ts = 0;
    double phase = 0;
    bool have_profile = false;
    qs_density_profile profile{};

    std::vector<double> P[NPL], C[NPL];
    std::vector<double> A;          // layers 0..L, 10 planes each (fields, currents)
    std::vector<double> Bm[4];      // JxBeam JyBeam JzBeam RhoBeam, layers -1..L+1

    // plasma particles (id-indexed); lists per interior cell, head first
    std::vector<double> ppy, ppz, ppx_, ppy_, ppz_, pw;
    std::vector<int> pcell;
    std::map<int, std::vector<std::vector<int>>> stored;   // layer -> lists
    std::vector<std::vector<int>> listsP, listsC;
    bool haveFront = false;
    // a layer received from the rank ahead (UnpackLayer, para.cpp:175-285):
    // fields and sources (A plane order, interior nI) and beam spectra
    bool recvPending = false, recvActive = false;
    std::vector<double> recvPlanes, recvJxB, recvRhoB;
    std::vector<std::vector<int>> frontLists;

    // beam particles
    std::vector<int> bi, bj, bk;
    std::vector<double> bx, by, bz, bpx, bpy, bpz, bw;

    // spectral and real work arrays (ny*nz), names of the reference
    bool firstCall = true;
    std::vector<double> rEx, rEy, rEz, rBx, rBy, rBz, rJx, rJy, rJz, rRho, rJxBeam, rRhoBeam;
    std::vector<double> fEx, fEy, fEz, fBx, fBy, fBz, fJx, fJy, fJz, fRho;
    std::vector<double> fExP, fEyP, fEzP, fJxP, fJyP, fJzP, fRhoP;
    std::vector<double> fJxBeam, fRhoBeam, fJxBeamP, fRhoBeamP;

    std::vector<double> onaxis;

    size_t gidx(int j, int k) const { return (size_t)(j + G) + (size_t)sy * (k + G); }
    size_t aidx(int i, int f, int j, int k) const {
        return ((size_t)i * 10 + f) * nyz + gidx(j, k);
    }
    size_t bidx(int i, int j, int k) const { return (size_t)(i + 1) * nyz + gidx(j, k); }

    bool init(const qs_config* c) {
        cfg = *c;
        My = c->ny; Mz = c->nz; L = c->nx;
        NxSplit = c->nx_split < 1 ? 1 : c->nx_split;
        nIter = c->n_iter < 0 ? 0 : c->n_iter;
        if (My < 2 || Mz < 2 || L < 1) return false;
        sy = My + 2 * G;
        sz = Mz + 2 * G;
        nyz = (size_t)sy * sz;
        nI = (size_t)My * Mz;
        hx = c->hx / NxSplit;  // HxSplit (domain.cpp:124-125)
        hy = c->hy;
        hz = c->hz;
        Ylength = My * hy;     // f_Ylength = l_Ysize*f_Hy (domain.cpp:138-141)
        Zlength = Mz * hz;
        ts = c->ts;
        for (int f = 0; f < NPL; f++) {
            P[f].assign(nyz, 0.0);
            C[f].assign(nyz, 0.0);
        }
        A.assign((size_t)(L + 1) * 10 * nyz, 0.0);
        for (int f = 0; f < 4; f++) Bm[f].assign((size_t)(L + 3) * nyz, 0.0);
        listsP.assign(nI, {});
        listsC.assign(nI, {});
        onaxis.assign(L, 0.0);
        return true;
    }

    double density_at(double xco, double yco, double zco) const {
        if (!have_profile) return cfg.plasma_density;
        SpecieProfile sp(profile);
        return sp(xco, yco, zco);
    }
    double dens() const {
        // :236-252 |Density*q2m| of the plasma electrons at the head layer
        // i = l_Mx-1, on axis (j = l_My/2., k = l_Mz/2.); 0 -> 1
        const int i = L - 1, j = (int)(My / 2.), k = (int)(Mz / 2.);
        const double xco = cfg.hx * i + phase;   // X(i) = Hx()*i
        const double yco = hy * j - Ylength / 2.;
        const double zco = hz * k - Zlength / 2.;
        double d = std::fabs(density_at(xco, yco, zco) * cfg.plasma_q2m);
        if (d == 0.0) d = 1.0;
        return d;
    }

    // ---- ExchangeFieldsSplit / ExchangeCurrentsSplit (:1659-1711)
    void exchange_fields() {
        for (int k = -1; k < Mz + 1; k++)
            for (int f = 0; f < 6; f++) {
                C[f][gidx(-1, k)] = C[f][gidx(My - 1, k)];
                C[f][gidx(My, k)] = C[f][gidx(0, k)];
            }
        for (int j = -1; j < My + 1; j++)
            for (int f = 0; f < 6; f++) {
                C[f][gidx(j, -1)] = C[f][gidx(j, Mz - 1)];
                C[f][gidx(j, Mz)] = C[f][gidx(j, 0)];
            }
    }
    void exchange_currents() {
        for (int k = -1; k < Mz + 1; k++)
            for (int f = 6; f < 10; f++) {
                C[f][gidx(0, k)] += C[f][gidx(My, k)];
                C[f][gidx(My - 1, k)] += C[f][gidx(-1, k)];
                C[f][gidx(My, k)] = C[f][gidx(-1, k)] = 0.0;
            }
        for (int j = -1; j < My + 1; j++)
            for (int f = 6; f < 10; f++) {
                C[f][gidx(j, 0)] += C[f][gidx(j, Mz)];
                C[f][gidx(j, Mz - 1)] += C[f][gidx(j, -1)];
                C[f][gidx(j, Mz)] = C[f][gidx(j, -1)] = 0.0;
            }
    }
    void clear_currents_split() {  // ClearCurrentsSplit, mesh.cpp:692-701 (incl. Dens)
        for (int f = 6; f < 10; f++) std::fill(C[f].begin(), C[f].end(), 0.0);
    }
    void clear_rho_split() { std::fill(C[9].begin(), C[9].end(), 0.0); }

    void alloc_spectral() {
        auto z = [&](std::vector<double>& v) { v.assign(nI, 0.0); };
        for (auto* v : {&rEx, &rEy, &rEz, &rBx, &rBy, &rBz, &rJx, &rJy, &rJz, &rRho, &rJxBeam,
                        &rRhoBeam, &fEx, &fEy, &fEz, &fBx, &fBy, &fBz, &fJx, &fJy, &fJz, &fRho,
                        &fExP, &fEyP, &fEzP, &fJxP, &fJyP, &fJzP, &fRhoP, &fJxBeam, &fRhoBeam,
                        &fJxBeamP, &fRhoBeamP})
            z(*v);
    }

    void fwd(const std::vector<double>& in, std::vector<double>& out, int kz, int ky) {
        r2r_2d(Mz, My, kz, ky, in.data(), out.data());
    }

    bool beam_current_ok() const {
        for (int k = 0; k < Mz; k++)
            for (int j = 0; j < My; j++)
                if (std::fabs(C[11][gidx(j, k)]) > 10) return false;
        return true;
    }

    // ---- GuessFieldsHydroLinLayerSplit (movefieldshydrolinlayersplit.cpp:222-1169)
    int guess(int iLayer, int iSplit) {
        const double d = dens();
        const int ny = My, nz = Mz;
        if (firstCall) {
            firstCall = false;
            alloc_spectral();
        }
        if (iLayer > L - 2 && !recvActive) {  // :430-445, the last rank: the head layer
            for (auto* v : {&fEx, &fEy, &fEz, &fBx, &fBy, &fBz, &fJx, &fJy, &fJz, &fRho, &fJxP,
                            &fJyP, &fJzP, &fRhoP, &fExP, &fEyP, &fEzP, &fJxBeam, &fRhoBeam,
                            &fJxBeamP, &fRhoBeamP})
                std::fill(v->begin(), v->end(), 0.0);
        }
        if (recvActive && iLayer == L - 1 && iSplit == 0) {
            // :547-551 below the first rank: the received beam spectra
            fJxBeam = recvJxB;
            fRhoBeam = recvRhoB;
        }
        // :552-558
        fRhoBeamP = fRhoBeam;
        fJxBeamP = fJxBeam;
        // :569-623 gather P (sources, fields) and C (beam)
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++) {
                size_t n = (size_t)j + (size_t)ny * k, g = gidx(j, k);
                rRho[n] = P[9][g];
                rEx[n] = P[0][g];
                rEy[n] = P[1][g];
                rEz[n] = P[2][g];
                rJx[n] = P[6][g];
                rJy[n] = P[7][g];
                rJz[n] = P[8][g];
                rJxBeam[n] = C[11][g];
                rRhoBeam[n] = C[10][g];
            }
        if (!beam_current_ok()) return QS_ERR_BEAM_CURRENT;
        // :717-743
        fwd(rRhoBeam, fRhoBeam, QS_REDFT11, QS_REDFT11);
        fwd(rJxBeam, fJxBeam, QS_REDFT11, QS_REDFT11);
        fwd(rRho, fRho, QS_REDFT11, QS_REDFT11);
        fwd(rEx, fEx, QS_REDFT11, QS_REDFT11);
        fwd(rEy, fEy, QS_REDFT11, QS_RODFT11);
        fwd(rEz, fEz, QS_RODFT11, QS_REDFT11);
        fwd(rJx, fJx, QS_REDFT11, QS_REDFT11);
        fwd(rJy, fJy, QS_REDFT11, QS_RODFT11);
        fwd(rJz, fJz, QS_RODFT11, QS_REDFT11);
        // :808-900 linear predictor per mode (P spectra taken from the C arrays)
        fRhoP = fRho; fJxP = fJx; fJyP = fJy; fJzP = fJz;
        fExP = fEx; fEyP = fEy; fEzP = fEz;
        qso_predictor_modes(ny, nz, hx, d, Ylength, Zlength, fRhoP.data(), fJxP.data(),
                            fJyP.data(), fJzP.data(), fExP.data(), fEyP.data(), fEzP.data(),
                            fRhoBeam.data(), fRhoBeamP.data(), fJxBeam.data(), fRho.data(),
                            fEx.data(), fEy.data(), fEz.data(), fJx.data(), fJy.data(),
                            fJz.data(), fBx.data(), fBy.data(), fBz.data());
        // :946-967 inverse transforms
        fwd(fRho, rRho, QS_REDFT11, QS_REDFT11);
        fwd(fEx, rEx, QS_REDFT11, QS_REDFT11);
        fwd(fEy, rEy, QS_REDFT11, QS_RODFT11);
        fwd(fEz, rEz, QS_RODFT11, QS_REDFT11);
        fwd(fJx, rJx, QS_REDFT11, QS_REDFT11);
        fwd(fJy, rJy, QS_REDFT11, QS_RODFT11);
        fwd(fJz, rJz, QS_RODFT11, QS_REDFT11);
        fwd(fBx, rBx, QS_RODFT11, QS_RODFT11);
        fwd(fBy, rBy, QS_RODFT11, QS_REDFT11);
        fwd(fBz, rBz, QS_REDFT11, QS_RODFT11);
        // :1004-1061 normalise and store into C
        const double norm = 4. * ny * nz;
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++) {
                size_t n = (size_t)j + (size_t)ny * k, g = gidx(j, k);
                C[9][g] = rRho[n] / norm;
                C[6][g] = rJx[n] / norm;
                C[7][g] = rJy[n] / norm;
                C[8][g] = rJz[n] / norm;
                C[0][g] = rEx[n] / norm;
                C[1][g] = rEy[n] / norm;
                C[2][g] = rEz[n] / norm;
                C[3][g] = rBx[n] / norm;
                C[4][g] = rBy[n] / norm;
                C[5][g] = rBz[n] / norm;
            }
        return QS_OK;
    }

    // ---- IterateFieldsHydroLinLayerSplit (movefieldshydrolinlayersplit.cpp:1173-1671)
    int iterate(int /*iLayer*/, int /*iSplit*/, int /*iter*/, double* rel_err) {
        const double d = dens();
        const int ny = My, nz = Mz;
        if (firstCall) return QS_ERR_STATE;  // :1229-1233
        // :1252-1305 gather C deposit currents (rRho = Dens+1 is dead)
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++) {
                size_t n = (size_t)j + (size_t)ny * k, g = gidx(j, k);
                rJx[n] = C[6][g];
                rJy[n] = C[7][g];
                rJz[n] = C[8][g];
            }
        if (!beam_current_ok()) return QS_ERR_BEAM_CURRENT;
        // :1343-1345
        fwd(rJx, fJx, QS_REDFT11, QS_REDFT11);
        fwd(rJy, fJy, QS_REDFT11, QS_RODFT11);
        fwd(rJz, fJz, QS_RODFT11, QS_REDFT11);
        // :1374-1477 corrector per mode
        qso_corrector_modes(ny, nz, hx, d, Ylength, Zlength, fRhoP.data(), fJxP.data(),
                            fJyP.data(), fJzP.data(), fEyP.data(), fEzP.data(),
                            fRhoBeam.data(), fRhoBeamP.data(), fJxBeam.data(), fJx.data(),
                            fJy.data(), fJz.data(), fRho.data(), fEx.data(), fEy.data(),
                            fEz.data(), fBx.data(), fBy.data(), fBz.data());
        // :1517-1533
        fwd(fRho, rRho, QS_REDFT11, QS_REDFT11);
        fwd(fEx, rEx, QS_REDFT11, QS_REDFT11);
        fwd(fEy, rEy, QS_REDFT11, QS_RODFT11);
        fwd(fEz, rEz, QS_RODFT11, QS_REDFT11);
        fwd(fBx, rBx, QS_RODFT11, QS_RODFT11);
        fwd(fBy, rBy, QS_RODFT11, QS_REDFT11);
        fwd(fBz, rBz, QS_REDFT11, QS_RODFT11);
        // :1545-1602 normalise, store into C, relative change of E
        const double norm = 4. * ny * nz;
        double maxEx = 1e-5, maxEy = 1e-5, maxEz = 1e-5;
        double difEx = 0, difEy = 0, difEz = 0;
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++) {
                size_t n = (size_t)j + (size_t)ny * k, g = gidx(j, k);
                double vRho = rRho[n] / norm, vEx = rEx[n] / norm, vEy = rEy[n] / norm,
                       vEz = rEz[n] / norm;
                maxEx = std::max(maxEx, std::fabs(vEx));
                maxEy = std::max(maxEy, std::fabs(vEy));
                maxEz = std::max(maxEz, std::fabs(vEz));
                difEx = std::max(difEx, std::fabs(C[0][g] - vEx));
                difEy = std::max(difEy, std::fabs(C[1][g] - vEy));
                difEz = std::max(difEz, std::fabs(C[2][g] - vEz));
                C[9][g] = vRho;
                C[0][g] = vEx;
                C[1][g] = vEy;
                C[2][g] = vEz;
                C[3][g] = rBx[n] / norm;
                C[4][g] = rBy[n] / norm;
                C[5][g] = rBz[n] / norm;
            }
        double e = std::max(difEx / maxEx, difEy / maxEy);
        e = std::max(e, difEz / maxEz);
        if (rel_err) *rel_err = e;
        return QS_OK;
    }

    // ---- MoveParticlesLayerSplit over the P-cell lists (:781-1544)
    int push(int iLayer, int /*iSplit*/, int iFullStep) {
        (void)iLayer;
        PushParams<double> pp = make_params<double>(&cfg);
        std::vector<double> Pi[6], Ci[6], D[4];
        for (int f = 0; f < 6; f++) {
            Pi[f].resize(nI);
            Ci[f].resize(nI);
        }
        for (int f = 0; f < 4; f++) D[f].assign(nI, 0.0);
        for (int k = 0; k < Mz; k++)
            for (int j = 0; j < My; j++) {
                size_t n = (size_t)j + (size_t)My * k, g = gidx(j, k);
                for (int f = 0; f < 6; f++) {
                    Pi[f][n] = P[f][g];
                    Ci[f][n] = C[f][g];
                }
            }
        PlaneSet<double> Ps, Cs;
        Ps.My = Cs.My = My;
        Ps.Mz = Cs.Mz = Mz;
        for (int f = 0; f < 6; f++) {
            Ps.f[f] = Pi[f].data();
            Cs.f[f] = Ci[f].data();
        }
        // The reference deposits into the guard ring and folds it in
        // ExchangeCurrentsSplit; depositing with the periodic fold directly
        // is the same sum.  Rows of cells are pushed in parallel with
        // thread-private deposit planes; the relinks are applied afterwards
        // in the reference's processing order (cells k-major, list order).
        int nthreads = 1;
#ifdef _OPENMP
        nthreads = omp_get_max_threads();
#endif
        std::vector<std::vector<double>> Dt((size_t)nthreads);
        std::vector<std::vector<std::pair<int, int>>> moves((size_t)Mz);
        int bad = 0;
#pragma omp parallel
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            std::vector<double>& Dl = Dt[(size_t)t];
            Dl.assign(4 * nI, 0.0);
            DepositSink<double> sink;
            sink.My = My;
            sink.Mz = Mz;
            for (int f = 0; f < 4; f++) sink.d[f] = Dl.data() + f * nI;
#pragma omp for schedule(static)
            for (int k = 0; k < Mz; k++) {
                for (int j = 0; j < My; j++) {
                    size_t c = (size_t)j + (size_t)My * k;
                    for (int id : listsP[c]) {
                        double& y = ppy[id];
                        double& z = ppz[id];
                        if (!(y >= 0 && y <= 1 && z >= 0 && z <= 1)) {
#pragma omp atomic write
                            bad = 1;
                            continue;
                        }
                        int jc = j, kc = k;
                        push_one<double>(pp, Ps, Cs, sink, jc, kc, y, z, ppx_[id], ppy_[id],
                                         ppz_[id], pw[id], iFullStep != 0);
                        if (iFullStep) moves[(size_t)k].push_back({id, jc + My * kc});
                    }
                }
            }
        }
        if (bad) return QS_ERR_PARTICLE_RANGE;
        for (int t = 0; t < nthreads; t++) {
            if (Dt[(size_t)t].empty()) continue;
            for (int f = 0; f < 4; f++)
                for (size_t n = 0; n < nI; n++) D[f][n] += Dt[(size_t)t][f * nI + n];
        }
        if (iFullStep) {
            std::vector<std::vector<int>> newC = listsC;
            for (int k = 0; k < Mz; k++)
                for (auto& mv : moves[(size_t)k]) {
                    newC[(size_t)mv.second].insert(newC[(size_t)mv.second].begin(), mv.first);
                    pcell[mv.first] = mv.second;   // p->p_Next = cnew.p_Particles
                }
            for (auto& l : listsP) l.clear();    // pcc.p_Particles = p_next
            listsC.swap(newC);
        }
        for (int k = 0; k < Mz; k++)
            for (int j = 0; j < My; j++) {
                size_t n = (size_t)j + (size_t)My * k, g = gidx(j, k);
                for (int f = 0; f < 4; f++) C[6 + f][g] += D[f][n];
            }
        return QS_OK;
    }

    // ---- MoveSplitLayer (:561-778)
    int move_split_layer(int iLayer, int iSplit) {
        int st = guess(iLayer, iSplit);
        if (st) return st;
        exchange_fields();
        for (int iter = 0; iter < nIter; iter++) {
            clear_currents_split();
            clear_rho_split();
            st = push(iLayer, iSplit, 0);
            if (st) return st;
            exchange_currents();
            st = iterate(iLayer, iSplit, iter, nullptr);
            if (st) return st;
            exchange_fields();
        }
        clear_currents_split();
        st = push(iLayer, iSplit, 1);
        if (st) return st;
        exchange_currents();
        st = iterate(iLayer, iSplit, -1, nullptr);
        if (st) return st;
        exchange_fields();
        return QS_OK;
    }

    // Cell::operator= (cells.cpp:25-47) over the copy range of the march
    // loops (k in [-2, Mz+1), j in [-2, My+1)): fields and currents copied,
    // beam members untouched, the particle list moved.
    void copy_layer_in(std::vector<double>* dst, int iLayer) {  // dst <- A[iLayer]
        for (int k = -G; k < Mz + G - 1; k++)
            for (int j = -G; j < My + G - 1; j++)
                for (int f = 0; f < 10; f++) dst[f][gidx(j, k)] = A[aidx(iLayer, f, j, k)];
    }
    void copy_layer_out(int iLayer, const std::vector<double>* src) {  // A[iLayer] <- src
        for (int k = -G; k < Mz + G - 1; k++)
            for (int j = -G; j < My + G - 1; j++)
                for (int f = 0; f < 10; f++) A[aidx(iLayer, f, j, k)] = src[f][gidx(j, k)];
    }

    // ---- MoveAllSplitLayers pieces (:25-558)
    int begin_march() {
        // :38-42 zero every current of the 3-D array
        for (int i = 0; i <= L; i++)
            for (int f = 6; f < 10; f++)
                std::fill(A.begin() + aidx(i, f, -G, -G), A.begin() + aidx(i, f, -G, -G) + nyz,
                          0.0);
        // :105-151 below the first rank the received layer is set into layer
        // l_Mx (CUDA_WRAP_setLayerToMesh, paraCPUlayers.cu:178-285).  The
        // reference writes its interior cells only; the guard ring is filled
        // periodically here, as ExchangeFieldsSplit does for every marched layer.
        recvActive = recvPending;
        recvPending = false;
        if (recvActive) {
            for (int f = 0; f < 10; f++)
                for (int k = -G; k < Mz + G - 1; k++)
                    for (int j = -G; j < My + G - 1; j++) {
                        const int jj = (j + My) % My, kk = (k + Mz) % Mz;
                        A[aidx(L, f, j, k)] = recvPlanes[(size_t)f * nI + jj + (size_t)My * kk];
                    }
        } else {
            for (int f = 0; f < 10; f++)
                std::fill(A.begin() + aidx(L, f, -G, -G), A.begin() + aidx(L, f, -G, -G) + nyz,
                          0.0);
        }
        // :63 SeedFrontParticles: the loaded front lists live at layer L
        if (!haveFront) return QS_ERR_STATE;
        stored.clear();
        stored[L] = frontLists;
        for (size_t c = 0; c < nI; c++)
            for (int id : frontLists[c]) pcell[id] = (int)c;
        haveFront = false;
        return QS_OK;
    }

    int layer_begin(int iLayer, int iSplit) {
        if (iLayer < 0 || iLayer >= L || iSplit < 0 || iSplit >= NxSplit) return QS_ERR_INVALID;
        if (iSplit == 0) {
            // :170-187 P <- Array[iLayer+1]
            copy_layer_in(P, iLayer + 1);
            auto it = stored.find(iLayer + 1);
            if (it != stored.end()) {
                listsP = std::move(it->second);
                stored.erase(it);
            } else {
                listsP.assign(nI, {});
            }
        }
        // :330-348 beam currents interpolated in xi into C and P
        const double S = NxSplit;
        for (int k = -G; k < Mz + G - 1; k++)
            for (int j = -G; j < My + G - 1; j++) {
                size_t g = gidx(j, k);
                double rc = Bm[3][bidx(iLayer, j, k)], rpv = Bm[3][bidx(iLayer + 1, j, k)];
                double jc = Bm[0][bidx(iLayer, j, k)], jpv = Bm[0][bidx(iLayer + 1, j, k)];
                C[10][g] = (rc * (S - iSplit) + rpv * iSplit) / S;
                P[10][g] = (rc * (S - iSplit - 1.) + rpv * (iSplit + 1.)) / S;
                C[11][g] = (jc * (S - iSplit) + jpv * iSplit) / S;
                P[11][g] = (jc * (S - iSplit - 1.) + jpv * (iSplit + 1.)) / S;
            }
        return QS_OK;
    }

    int layer_end(int iLayer, int iSplit) {
        // :423-428 P <- C (fields, currents, particles)
        for (int k = -G; k < Mz + G - 1; k++)
            for (int j = -G; j < My + G - 1; j++) {
                size_t g = gidx(j, k);
                for (int f = 0; f < 10; f++) P[f][g] = C[f][g];
            }
        listsP = std::move(listsC);
        listsC.assign(nI, {});
        if (iSplit == NxSplit - 1) {
            // :467-473 Array[iLayer] <- P
            copy_layer_out(iLayer, P);
            stored[iLayer] = std::move(listsP);
            listsP.assign(nI, {});
            onaxis[iLayer] = A[aidx(iLayer, 0, My / 2, Mz / 2)];
        }
        return QS_OK;
    }

    int move_all_split_layers() {
        int st = begin_march();
        if (st) return st;
        for (int iLayer = L - 1; iLayer > -1; iLayer--)
            for (int iSplit = 0; iSplit < NxSplit; iSplit++) {
                st = layer_begin(iLayer, iSplit);
                if (st) return st;
                st = move_split_layer(iLayer, iSplit);
                if (st) return st;
                st = layer_end(iLayer, iSplit);
                if (st) return st;
            }
        return QS_OK;
    }

    // ---- MoveBeamParticles + MoveBeamInCell (movebeam.cpp:14-774)
    double fld(int f, int i, int j, int k) const { return A[aidx(i, f, j, k)]; }

    int move_beam() {
        // ClearBeamCurrents (mesh.cpp:648-663)
        for (int f = 0; f < 4; f++) std::fill(Bm[f].begin(), Bm[f].end(), 0.0);
        const double ts_ = ts, hx_ = cfg.hx, hy_ = hy, hz_ = hz;
        const double PI_ = 3.1415927;  // domain.h:10
        const double ElaserPhoton = 1.2398e-4 / cfg.wavelength;
        const double eSynMin = cfg.syn_min;
        const int64_t nb = (int64_t)bi.size();
        for (int64_t p = 0; p < nb; p++) {
            int i = bi[p], j = bj[p], k = bk[p];
            // the reference loops i in [0,l_Mx), j in [0,l_My), k in [0,l_Mz)
            if (i < 0 || i >= L || j < 0 || j >= My || k < 0 || k >= Mz) continue;
            double weight = bw[p];
            double x = bx[p], y = by[p], z = bz[p];
            double px = bpx[p], py = bpy[p], pz = bpz[p];
            double pxn = px, pyn = py, pzn = pz;
            double q2m = cfg.beam_q2m;
            if (x < 0 || x > 1 || y < 0 || y > 1 || z < 0 || z > 1) return QS_ERR_PARTICLE_RANGE;
            double axc = 1. - x, axp = x, ayc = 1. - y, ayp = y, azc = 1. - z, azp = z;
            double accc = axc * ayc * azc, acpc = axc * ayp * azc, accp = axc * ayc * azp,
                   acpp = axc * ayp * azp, apcc = axp * ayc * azc, appc = axp * ayp * azc,
                   apcp = axp * ayc * azp, appp = axp * ayp * azp;
            auto g8 = [&](int f) {
                return accc * fld(f, i, j, k) + acpc * fld(f, i, j + 1, k) +
                       accp * fld(f, i, j, k + 1) + acpp * fld(f, i, j + 1, k + 1) +
                       apcc * fld(f, i + 1, j, k) + appc * fld(f, i + 1, j + 1, k) +
                       apcp * fld(f, i + 1, j, k + 1) + appp * fld(f, i + 1, j + 1, k + 1);
            };
            double ex = g8(0), ey = g8(1), ez = g8(2);
            double bxf = g8(3), byf = g8(4), bzf = g8(5);
            bxf += cfg.bx_ext;
            byf += cfg.by_ext;
            bzf += cfg.bz_ext;
            // :334-336 E added unscaled (the q2m*ts/2 scaling is commented out)
            px += ex;
            py += ey;
            pz += ez;
            double gamma = std::sqrt(1. + px * px + py * py + pz * pz);
            double gamma_r = 1. / gamma;
            bxf = bxf * gamma_r * q2m * ts_ / 2.;
            byf = byf * gamma_r * q2m * ts_ / 2.;
            bzf = bzf * gamma_r * q2m * ts_ / 2.;
            double co = 2. / (1. + (bxf * bxf) + (byf * byf) + (bzf * bzf));
            double p3x = py * bzf - pz * byf + px;
            double p3y = pz * bxf - px * bzf + py;
            double p3z = px * byf - py * bxf + pz;
            p3x *= co;
            p3y *= co;
            p3z *= co;
            double px_new = p3y * bzf - p3z * byf;
            double py_new = p3z * bxf - p3x * bzf;
            double pz_new = p3x * byf - p3y * bxf;
            px += (ex + px_new);
            py += (ey + py_new);
            pz += (ez + pz_new);
            // :449-491 synchrotron radiation reaction (photon histogram omitted)
            double p2 = px * px + py * py + pz * pz;
            if (cfg.synchrotron && 1. + p2 > eSynMin * eSynMin) {
                double dpx = px - pxn, dpy = py - pyn, dpz = pz - pzn;
                double pdp = px * dpx + py * dpy + pz * dpz;
                dpx -= px * (pdp / p2);
                dpy -= py * (pdp / p2);
                dpz -= pz * (pdp / p2);
                double p2absrev = 1.0 / std::sqrt(p2);
                double nx = px * p2absrev, nyv = py * p2absrev, nzv = pz * p2absrev;
                double dpabs = std::sqrt(dpx * dpx + dpy * dpy + dpz * dpz);
                double Gamma2 = 1. + p2;
                double omega_c = 3. * Gamma2 * dpabs / (4. * PI_ * ts_);
                double Ephoton = ElaserPhoton * omega_c;
                double alfa = 1. / 137.;
                double nph = 4. / 9. * alfa * dpabs;
                px -= (nph * Ephoton * nx / 511000.0);
                py -= (nph * Ephoton * nyv / 511000.0);
                pz -= (nph * Ephoton * nzv / 511000.0);
            }
            // :496-529
            gamma = 1. / std::sqrt(1. + px * px + py * py + pz * pz);
            double Vx = px * gamma, Vy = py * gamma, Vz = pz * gamma;
            double polarity = cfg.beam_polarity;
            double djx = weight * polarity * Vx;
            double djy = weight * polarity * Vy;
            double djz = weight * polarity * Vz;
            double drho = weight * polarity;
            double dx = (px * gamma - 1.) * ts_ / hx_;
            double dy = py * gamma * ts_ / hy_;
            double dz = pz * gamma * ts_ / hz_;
            double xtmp = x + dx, ytmp = y + dy, ztmp = z + dz;
            // :542-605
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
            bpx[p] = px;
            bpy[p] = py;
            bpz[p] = pz;
            bx[p] = xtmp;
            by[p] = ytmp;
            bz[p] = ztmp;
            bi[p] = itmp;
            bj[p] = jtmp;
            bk[p] = ktmp;
            // MoveBeamInCell :662-774 (8-point CIC of w*v and w)
            double ax1 = xtmp, ax0 = 1. - ax1, ay1 = ytmp, ay0 = 1. - ay1, az1 = ztmp,
                   az0 = 1. - az1;
            for (int di = 0; di < 2; di++)
                for (int dj = 0; dj < 2; dj++)
                    for (int dk = 0; dk < 2; dk++) {
                        const double wx = di ? ax1 : ax0, wy = dj ? ay1 : ay0,
                                     wz = dk ? az1 : az0;
                        size_t b = bidx(itmp + di, jtmp + dj, ktmp + dk);
                        Bm[0][b] += djx * wx * wy * wz;
                        Bm[1][b] += djy * wx * wy * wz;
                        Bm[2][b] += djz * wx * wy * wz;
                        Bm[3][b] += drho * wx * wy * wz;
                    }
        }
        return QS_OK;
    }
};

int g_threads = 1;

}  // namespace

struct qso {
    Oracle o;
};

extern "C" {

void qso_set_threads(int n) {
    g_threads = n < 1 ? 1 : n;
#ifdef _OPENMP
    omp_set_num_threads(g_threads);
#endif
}
int qso_get_threads(void) { return g_threads; }

int qso_create(const qs_config* cfg, qso** out) {
    if (!cfg || !out) return QS_ERR_INVALID;
    qso* h = new (std::nothrow) qso;
    if (!h) return QS_ERR_OOM;
    try {
        if (!h->o.init(cfg)) {
            delete h;
            return QS_ERR_INVALID;
        }
    } catch (const std::bad_alloc&) {
        delete h;
        return QS_ERR_OOM;
    }
    *out = h;
    return QS_OK;
}

void qso_destroy(qso* o) { delete o; }

double qso_density(const qs_density_profile* p, double x, double y, double z) {
    if (!p) return 0.0;
    SpecieProfile sp(*p);
    return sp(x, y, z);
}

int qso_set_density_profile(qso* h, const qs_density_profile* p) {
    if (!h) return QS_ERR_INVALID;
    h->o.have_profile = p != nullptr;
    if (p) h->o.profile = *p;
    return QS_OK;
}

int qso_set_phase(qso* h, double phase) {
    if (!h) return QS_ERR_INVALID;
    h->o.phase = phase;
    return QS_OK;
}

// ---- PackLayer / UnpackLayer (para.cpp:94-285): 12 planes (Bx, By, Bz, Ex,
// Ey, Ez, Jx, Jy, Jz, Rho, fftJxBeamHydro, fftRhoBeamHydro) then 12 particle
// blocks (Px, Py, Pz, X, Y, Z, Q2m, Weight, i_X, i_Y, i_Z, isort)
int64_t qso_layer_pack_size(const qso* h) {
    return h ? 12 * (int64_t)h->o.nI + 12 * (int64_t)h->o.ppy.size() : -1;
}

int qso_pack_layer(qso* h, double* buf, int64_t n) {
    if (!h || !buf || n != qso_layer_pack_size(h)) return QS_ERR_INVALID;
    Oracle& o = h->o;
    auto it = o.stored.find(0);
    if (it == o.stored.end()) return QS_ERR_STATE;   // no complete march
    const size_t nI = o.nI;
    const int order[10] = {3, 4, 5, 0, 1, 2, 6, 7, 8, 9};   // A planes in pack order
    for (int k = 0; k < o.Mz; k++)
        for (int j = 0; j < o.My; j++) {
            const size_t n1 = (size_t)j + (size_t)o.My * k;
            for (int f = 0; f < 10; f++) buf[f * nI + n1] = o.A[o.aidx(0, order[f], j, k)];
            buf[10 * nI + n1] = o.fJxBeam[n1];
            buf[11 * nI + n1] = o.fRhoBeam[n1];
        }
    const int64_t m = (int64_t)o.ppy.size();
    double* pb = buf + 12 * nI;
    int64_t r = 0;
    for (int k = 0; k < o.Mz; k++)           // the layer walk of paraCPUlayers.cu:76-113
        for (int j = 0; j < o.My; j++)
            for (int id : it->second[(size_t)j + (size_t)o.My * k]) {
                if (r >= m) return QS_ERR_STATE;
                pb[r] = o.ppx_[id];
                pb[r + m] = o.ppy_[id];
                pb[r + 2 * m] = o.ppz_[id];
                pb[r + 3 * m] = 0.0;
                pb[r + 4 * m] = o.ppy[id];
                pb[r + 5 * m] = o.ppz[id];
                pb[r + 6 * m] = o.cfg.plasma_q2m;
                pb[r + 7 * m] = o.pw[id];
                pb[r + 8 * m] = 0.0;
                pb[r + 9 * m] = j;
                pb[r + 10 * m] = k;
                pb[r + 11 * m] = 0.0;
                r++;
            }
    return r == m ? QS_OK : QS_ERR_STATE;
}

int qso_unpack_layer(qso* h, const double* buf, int64_t n) {
    if (!h || !buf) return QS_ERR_INVALID;
    Oracle& o = h->o;
    const int64_t fixed = 12 * (int64_t)o.nI;
    if (n < fixed || (n - fixed) % 12) return QS_ERR_INVALID;
    const int64_t m = (n - fixed) / 12;
    const size_t nI = o.nI;
    const int order[10] = {3, 4, 5, 0, 1, 2, 6, 7, 8, 9};
    o.recvPlanes.assign(10 * nI, 0.0);
    for (int f = 0; f < 10; f++)
        std::copy(buf + f * nI, buf + (f + 1) * nI, o.recvPlanes.begin() + (size_t)order[f] * nI);
    o.recvJxB.assign(buf + 10 * nI, buf + 11 * nI);
    o.recvRhoB.assign(buf + 11 * nI, buf + 12 * nI);
    // CUDA_WRAP_setLayerToMesh appends each particle to the list of its cell
    const double* pb = buf + fixed;
    std::vector<int64_t> ord(m);
    std::vector<int32_t> cell(m);
    for (int64_t r = 0; r < m; r++) {
        const int j = (int)pb[r + 9 * m], k = (int)pb[r + 10 * m];
        if (j < 0 || j >= o.My || k < 0 || k >= o.Mz) return QS_ERR_INVALID;
        cell[r] = j + o.My * k;
        ord[r] = r;
    }
    std::stable_sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) { return cell[a] < cell[b]; });
    std::vector<int32_t> c(m);
    std::vector<double> y(m), z(m), px(m), py(m), pz(m), w(m);
    for (int64_t r = 0; r < m; r++) {
        const int64_t q = ord[r];
        c[r] = cell[q];
        px[r] = pb[q];
        py[r] = pb[q + m];
        pz[r] = pb[q + 2 * m];
        y[r] = pb[q + 4 * m];
        z[r] = pb[q + 5 * m];
        w[r] = pb[q + 7 * m];
    }
    int st = qso_load_front_plasma(h, m, c.data(), y.data(), z.data(), px.data(), py.data(),
                                   pz.data(), w.data());
    if (st) return st;
    o.recvPending = true;
    return QS_OK;
}

int qso_front_weights(qso* h, double* out) {
    // Mesh::SeedParticles (mesh.cpp:413-471): xco = X(l_Mx) + phase, the
    // cell's corner in y and z, weight GetWeight()*dens = dens/ppc, no
    // particle (weight 0 here) where dens <= 0
    if (!h || !out) return QS_ERR_INVALID;
    const Oracle& o = h->o;
    const double xco = o.cfg.hx * o.L + o.phase;
    for (int k = 0; k < o.Mz; k++)
        for (int j = 0; j < o.My; j++) {
            const double yco = o.hy * j - o.Ylength / 2.;
            const double zco = o.hz * k - o.Zlength / 2.;
            const double dens = o.density_at(xco, yco, zco);
            out[j + (size_t)o.My * k] = dens > 0. ? 1. / o.cfg.ppc * dens : 0.0;
        }
    return QS_OK;
}

int qso_load_beam(qso* h, int64_t n, const int32_t* i, const int32_t* j, const int32_t* k,
                  const double* x, const double* y, const double* z, const double* px,
                  const double* py, const double* pz, const double* w) {
    if (!h || n < 0) return QS_ERR_INVALID;
    Oracle& o = h->o;
    o.bi.assign(i, i + n);
    o.bj.assign(j, j + n);
    o.bk.assign(k, k + n);
    o.bx.assign(x, x + n);
    o.by.assign(y, y + n);
    o.bz.assign(z, z + n);
    o.bpx.assign(px, px + n);
    o.bpy.assign(py, py + n);
    o.bpz.assign(pz, pz + n);
    o.bw.assign(w, w + n);
    return QS_OK;
}

int qso_get_beam(qso* h, int64_t n, int32_t* i, int32_t* j, int32_t* k, double* x, double* y,
                 double* z, double* px, double* py, double* pz, double* w) {
    if (!h || n != (int64_t)h->o.bi.size()) return QS_ERR_INVALID;
    Oracle& o = h->o;
    for (int64_t p = 0; p < n; p++) {
        if (i) i[p] = o.bi[p];
        if (j) j[p] = o.bj[p];
        if (k) k[p] = o.bk[p];
        if (x) x[p] = o.bx[p];
        if (y) y[p] = o.by[p];
        if (z) z[p] = o.bz[p];
        if (px) px[p] = o.bpx[p];
        if (py) py[p] = o.bpy[p];
        if (pz) pz[p] = o.bpz[p];
        if (w) w[p] = o.bw[p];
    }
    return QS_OK;
}

int64_t qso_beam_count(const qso* h) { return h ? (int64_t)h->o.bi.size() : -1; }

int qso_load_front_plasma(qso* h, int64_t n, const int32_t* cell, const double* y,
                          const double* z, const double* px, const double* py,
                          const double* pz, const double* w) {
    if (!h || n < 0) return QS_ERR_INVALID;
    Oracle& o = h->o;
    o.ppy.assign(y, y + n);
    o.ppz.assign(z, z + n);
    o.ppx_.assign(px, px + n);
    o.ppy_.assign(py, py + n);
    o.ppz_.assign(pz, pz + n);
    o.pw.assign(w, w + n);
    o.pcell.assign(cell, cell + n);
    o.frontLists.assign(o.nI, {});
    int32_t prev = -1;
    for (int64_t p = 0; p < n; p++) {
        if (cell[p] < 0 || (size_t)cell[p] >= o.nI || cell[p] < prev) return QS_ERR_INVALID;
        prev = cell[p];
        o.frontLists[cell[p]].push_back((int)p);   // given order = list order
    }
    o.haveFront = true;
    return QS_OK;
}

int64_t qso_plasma_count(const qso* h) { return h ? (int64_t)h->o.ppy.size() : -1; }

int qso_get_plasma(qso* h, int64_t n, int32_t* cell, double* y, double* z, double* px,
                   double* py, double* pz, double* w) {
    if (!h || n != (int64_t)h->o.ppy.size()) return QS_ERR_INVALID;
    Oracle& o = h->o;
    for (int64_t p = 0; p < n; p++) {
        if (cell) cell[p] = o.pcell[p];
        if (y) y[p] = o.ppy[p];
        if (z) z[p] = o.ppz[p];
        if (px) px[p] = o.ppx_[p];
        if (py) py[p] = o.ppy_[p];
        if (pz) pz[p] = o.ppz_[p];
        if (w) w[p] = o.pw[p];
    }
    return QS_OK;
}

int qso_set_layer(qso* h, int which, int field, const double* data) {
    if (!h || !data || field < 0 || field >= NPL || (which != 0 && which != 1))
        return QS_ERR_INVALID;
    Oracle& o = h->o;
    std::vector<double>* L = which == QS_LAYER_P ? o.P : o.C;
    for (int k = 0; k < o.Mz; k++)
        for (int j = 0; j < o.My; j++) L[field][o.gidx(j, k)] = data[(size_t)j + (size_t)o.My * k];
    if (field < 6 && which == QS_LAYER_C) o.exchange_fields();
    return QS_OK;
}

int qso_get_layer(qso* h, int which, int field, double* out) {
    if (!h || !out || field < 0 || field >= NPL || (which != 0 && which != 1))
        return QS_ERR_INVALID;
    Oracle& o = h->o;
    std::vector<double>* L = which == QS_LAYER_P ? o.P : o.C;
    for (int k = 0; k < o.Mz; k++)
        for (int j = 0; j < o.My; j++) out[(size_t)j + (size_t)o.My * k] = L[field][o.gidx(j, k)];
    return QS_OK;
}

int qso_get_field3d(qso* h, int field, int layer, double* out) {
    if (!h || !out || field < 0 || field >= 10 || layer < 0 || layer > h->o.L)
        return QS_ERR_INVALID;
    Oracle& o = h->o;
    for (int k = 0; k < o.Mz; k++)
        for (int j = 0; j < o.My; j++)
            out[(size_t)j + (size_t)o.My * k] = o.A[o.aidx(layer, field, j, k)];
    return QS_OK;
}

static int beam_plane(int field) {
    if (field == QS_F_RHOBEAM) return 3;
    if (field == QS_F_JXBEAM) return 0;
    return -1;
}

int qso_set_beam_currents(qso* h, int field, int layer, const double* data) {
    int b = beam_plane(field);
    if (!h || !data || b < 0 || layer < 0 || layer > h->o.L) return QS_ERR_INVALID;
    Oracle& o = h->o;
    for (int k = 0; k < o.Mz; k++)
        for (int j = 0; j < o.My; j++)
            o.Bm[b][o.bidx(layer, j, k)] = data[(size_t)j + (size_t)o.My * k];
    return QS_OK;
}

int qso_get_beam_currents(qso* h, int field, int layer, double* out) {
    int b = beam_plane(field);
    if (!h || !out || b < 0 || layer < 0 || layer > h->o.L) return QS_ERR_INVALID;
    Oracle& o = h->o;
    for (int k = 0; k < o.Mz; k++)
        for (int j = 0; j < o.My; j++)
            out[(size_t)j + (size_t)o.My * k] = o.Bm[b][o.bidx(layer, j, k)];
    return QS_OK;
}

int qso_get_onaxis_ex(qso* h, double* out) {
    if (!h || !out) return QS_ERR_INVALID;
    std::copy(h->o.onaxis.begin(), h->o.onaxis.end(), out);
    return QS_OK;
}

int qso_set_field3d(qso* h, int field, int layer, const double* data) {
    if (!h || !data || field < 0 || field > 5 || layer < 0 || layer > h->o.L) return QS_ERR_INVALID;
    Oracle& o = h->o;
    // interior and the whole guard ring, periodic in y and z
    for (int k = -o.G; k < o.Mz + o.G; k++)
        for (int j = -o.G; j < o.My + o.G; j++) {
            const int jj = (j + o.My) % o.My, kk = (k + o.Mz) % o.Mz;
            o.A[o.aidx(layer, field, j, k)] = data[(size_t)jj + (size_t)o.My * kk];
        }
    return QS_OK;
}

int qso_get_psi(qso* h, double* out) {
    if (!h || !out) return QS_ERR_INVALID;
    const Oracle& o = h->o;
    // psi(nx) = 0 ahead of the box, trapezoid of on-axis Ex towards the tail
    double psi = 0.0, prev = 0.0;
    for (int i = o.L - 1; i >= 0; i--) {
        psi += o.cfg.hx * 0.5 * (o.onaxis[(size_t)i] + prev);
        out[i] = psi;
        prev = o.onaxis[(size_t)i];
    }
    return QS_OK;
}

int qso_get_charge_sums(qso* h, double* rho, double* jx, double* rho_beam) {
    if (!h) return QS_ERR_INVALID;
    const Oracle& o = h->o;
    // stored layer i: plane 9 is f_Dens after the layer's last Iterate (the
    // corrected density, :1545-1602), plane 6 the Jx deposit of its full push
    for (int i = 0; i < o.L; i++) {
        double sr = 0.0, sj = 0.0;
        for (int k = 0; k < o.Mz; k++)
            for (int j = 0; j < o.My; j++) {
                sr += o.A[o.aidx(i, 9, j, k)];
                sj += o.A[o.aidx(i, 6, j, k)];
            }
        if (rho) rho[i] = sr;
        if (jx) jx[i] = sj;
    }
    if (rho_beam)
        for (int i = 0; i <= o.L; i++) {
            double sb = 0.0;
            for (int k = 0; k < o.Mz; k++)
                for (int j = 0; j < o.My; j++) sb += o.Bm[3][o.bidx(i, j, k)];
            rho_beam[i] = sb;
        }
    return QS_OK;
}

int qso_step(qso* h) {
    if (!h) return QS_ERR_INVALID;
    h->o.phase += h->o.ts;  // step.cpp:33
    int st = h->o.move_beam();
    if (st) return st;
    return h->o.move_all_split_layers();
}
int qso_move_beam_particles(qso* h) { return h ? h->o.move_beam() : QS_ERR_INVALID; }
int qso_move_all_split_layers(qso* h) { return h ? h->o.move_all_split_layers() : QS_ERR_INVALID; }
int qso_begin_march(qso* h) { return h ? h->o.begin_march() : QS_ERR_INVALID; }
int qso_layer_begin(qso* h, int iLayer, int iSplit) {
    return h ? h->o.layer_begin(iLayer, iSplit) : QS_ERR_INVALID;
}
int qso_move_split_layer(qso* h, int iLayer, int iSplit) {
    return h ? h->o.move_split_layer(iLayer, iSplit) : QS_ERR_INVALID;
}
int qso_guess_fields(qso* h, int iLayer, int iSplit) {
    if (!h) return QS_ERR_INVALID;
    int st = h->o.guess(iLayer, iSplit);
    if (!st) h->o.exchange_fields();
    return st;
}
int qso_move_particles_layer(qso* h, int iLayer, int iSplit, int iFullStep) {
    if (!h) return QS_ERR_INVALID;
    h->o.clear_currents_split();
    int st = h->o.push(iLayer, iSplit, iFullStep);
    if (!st) h->o.exchange_currents();
    return st;
}
int qso_iterate_fields(qso* h, int iLayer, int iSplit, int iter, double* rel_err) {
    if (!h) return QS_ERR_INVALID;
    int st = h->o.iterate(iLayer, iSplit, iter, rel_err);
    if (!st) h->o.exchange_fields();
    return st;
}
int qso_layer_end(qso* h, int iLayer, int iSplit) {
    return h ? h->o.layer_end(iLayer, iSplit) : QS_ERR_INVALID;
}

int qso_dtt1d(int n, int kind, const double* in, double* out, int direct) {
    if (n < 1 || !in || !out || (kind != QS_REDFT11 && kind != QS_RODFT11)) return QS_ERR_INVALID;
    auto p = get_plan(n);
    std::vector<double> tmp;
    std::vector<cplx> work;
    dtt1(*p, kind, in, out, direct != 0, tmp, work);
    return QS_OK;
}

int qso_transform2d(int nz, int ny, int kind_z, int kind_y, int batch, const double* in,
                    double* out, int direct) {
    if (nz < 1 || ny < 1 || batch < 0 || !in || !out) return QS_ERR_INVALID;
    if ((kind_z != QS_REDFT11 && kind_z != QS_RODFT11) ||
        (kind_y != QS_REDFT11 && kind_y != QS_RODFT11))
        return QS_ERR_INVALID;
    const size_t plane = (size_t)nz * ny;
    for (int b = 0; b < batch; b++)
        r2r_2d(nz, ny, kind_z, kind_y, in + b * plane, out + b * plane, direct != 0);
    return QS_OK;
}

int qso_push_layer_f64(const qs_config* cfg, int64_t n, int32_t* cell, double* y, double* z,
                       double* px, double* py, double* pz, const double* w, const double* P,
                       const double* C, double* dep, int32_t* dep_cell, int full, int precise) {
    return push_layer_arrays<double>(cfg, n, cell, y, z, px, py, pz, w, P, C, dep, dep_cell, full,
                                     precise);
}

int qso_push_layer_f32(const qs_config* cfg, int64_t n, int32_t* cell, float* y, float* z,
                       float* px, float* py, float* pz, const float* w, const float* P,
                       const float* C, float* dep, int32_t* dep_cell, int full, int precise) {
    return push_layer_arrays<float>(cfg, n, cell, y, z, px, py, pz, w, P, C, dep, dep_cell, full,
                                    precise);
}

}  // extern "C"
