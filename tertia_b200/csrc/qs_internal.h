// qs_internal.h — host-side launchers shared by the CUDA translation units.
#pragma once
#include "qs_common.cuh"

namespace qs {

// Per-mode spectral maps of the Guess / Iterate solve.
template <class T>
struct SpecArgs {
    int ny, nz;
    T piY, piZ;          // M_PI/Ylength, M_PI/Zlength
    T hx;
    // |Density*q2m| of the maps, in device memory so that a captured march
    // follows a density that changes from step to step
    const T* dens_p;
    const T *RhoP, *ExP, *EyP, *EzP, *JxP, *JyP, *JzP;   // P spectral state
    // beam spectra of this (layer, split): w0*X0 + w1*X1 (the xi-interpolation
    // of movepart_splitlayer.cpp:330-348 applied to the spectra), and of the
    // previous (layer, split) for RhoBeamP (weights 0 at the head layer)
    const T *Rb0, *Rb1, *Jxb0, *Jxb1;
    T wb0, wb1;
    const T *Rbp0, *Rbp1;
    T wp0, wp1;
    const T *Jx, *Jy, *Jz;                                // forward of the C deposit
    T* Rho;                                               // in/out spectral rho
    T *Ex, *Ey, *Ez, *Bx, *By, *Bz;                       // spectral outputs
    int write_b;         // store Bx, By, Bz spectra (exact-GEMM transforms read them)
    // split-precision operand of the inverse transform: slots 0..5 = Ex,Ey,Ez,
    // Bx,By,Bz, slot 6 = Rho when split_rho; term s of slot f at
    // split + s*tstride + f*ny*nz (bf16 for split_kind 0, tf32 for 1)
    void* split;
    int nsplit, split_kind, split_rho;
    size_t tstride;
    // optional: 4 planes (the C-layer deposit) cleared by the kernel for the
    // push that follows it (ClearCurrentsSplit without a separate memset)
    T* zero_src;
    // optional (correctors): FP64 charge sums (charge.cuh); each block writes
    // its partial sums of rho c_ky c_kz and Jx c_ky c_kz to qsum[2 * block]
    double* qsum;
    const double *qcy, *qcz;   // c_k(ny), c_k(nz)
};

template <class T>
int launch_predictor(const SpecArgs<T>& a, cudaStream_t st);
template <class T>
int launch_corrector(const SpecArgs<T>& a, cudaStream_t st);
// FP32 forms (spectral_f32.cu); return 0 when the shape is not handled
int launch_predictor_fast(const SpecArgs<float>& a, cudaStream_t st);
int launch_corrector_fast(const SpecArgs<float>& a, cudaStream_t st);

// C-layer beam currents for (iLayer, iSplit): the xi-interpolation of
// movepart_splitlayer.cpp:330-348 plus the |JxBeam| > 10 check.
template <class T>
int launch_beam_layer(const T* cur, const T* nxt, int S, int s, T* out, size_t plane, int* err,
                      cudaStream_t st);
// |JxBeam| > 10 anywhere in the beam-current store (layers x [RhoBeam, JxBeam]),
// and the FP64 partial sums of each layer's RhoBeam: part[2 * (layer *
// kBeamSumParts + b)] for the kBeamSumParts blocks b of a layer
constexpr int kBeamSumParts = 32;
template <class T>
int launch_beam_check(const T* b3, int nlayers, size_t plane, int* err, double* part,
                      cudaStream_t st);
// out[layer * 2 + q] = scale * sum over p < nparts of part[2 * (layer * nparts + p) + q]
// (q = 0, 1; in index order)
int launch_charge_reduce(const double* part, int nparts, int nlayers, double scale, double* out,
                         cudaStream_t st);

template <class T>
int launch_onaxis(const T* fields3d, int L, size_t plane, size_t idx, T* out, cudaStream_t st);
// a block of a 3-D store (L layers, `layer_stride` values apart, planes of
// rows of My) in x-fastest order, widened to double:
// out[i + L (jj + nj kk)] = base[i * layer_stride + (j0 + jj) + My (k0 + kk)]
template <class T>
int launch_gather_xfast(const T* base, size_t layer_stride, int L, int My, int j0, int nj, int k0,
                        int nk, double* out, cudaStream_t st);

// Front-layer seeding (Mesh::SeedParticles, mesh.cpp:413-548): ppc
// particles per cell on the in-cell lattice, thermal momenta from a
// counter-based generator, weight from the uniform density or the profile.
struct SeedFront {
    int My, Mz, ppc;
    double offs_y[16], offs_z[16];
    double px0, py0, pz0, sx, sy, sz;
    double weight;               // uniform: Density/ppc
    int use_profile;             // 1: weight (1/ppc)*Density(x_front, y_j, z_k), 0 where <= 0
    qs_density_profile prof;
    double x_front, hy, hz, y_half, z_half;
    uint64_t seed, step;
};
template <class T>
int launch_seed_front(const SeedFront& s, int32_t* cell, T* y, T* z, T* px, T* py, T* pz, T* w,
                      cudaStream_t st);
// one value into device memory, in stream order
template <class T>
int launch_set_value(T* dst, T v, cudaStream_t st);

template <class T>
int launch_convert(const void* src, int src_is_double, T* dst, size_t n, cudaStream_t st);
// x = (double)(float)x over n values (the FP32 attribution study)
int launch_round_f32(double* x, size_t n, cudaStream_t st);
// dst += (double)src over n values
int launch_add_widened(double* dst, const float* src, size_t n, cudaStream_t st);
// dst += (double)now - (double)before over n values; with frac, dst stays in [0, 1]
int launch_add_increment(double* dst, const float* now, const float* before, size_t n, int frac,
                         cudaStream_t st);
template <class T>
int launch_convert_back(const T* src, double* dst, size_t n, cudaStream_t st);

// Transforms.
template <class T>
int run_dtt_simt(const DttJob<T>& job, int ny, int nz, const DttMats<T>& my,
                 const DttMats<T>& mz, T* scratch, cudaStream_t st);
// FP32 half-integer transforms through half-length complex FFTs
// (dtt_fft.cu), for power-of-two ny, nz in [32, 2048]: pass 0 along y from
// the job's inputs into `scratch` (same layout), pass 1 along z from there
// into the job's outputs with its scale.
template <class T>
struct AdjSpecArgs;

struct DttFft {
    int ny = 0, nz = 0;
    float2* tab_y = nullptr;   // twiddle tables of each size
    float2* tab_z = nullptr;
    bool spec_rows = false;    // run_spectral_rows available (ny in [128, 1024])
    static DttFft* create(int ny, int nz);   // nullptr when a size is not handled
    int run_pass(int pass, const DttJob<float>& job, float* scratch, cudaStream_t st) const;
    // the z-pass alone: nf planes in -> out, y-spectral or real alike; with
    // `acc` each input plane is also added to acc[f], with `clr` the planes
    // clr[f] (the inputs) are zeroed once read
    int run_cols(int nf, const float* const* in, float* const* out, const int* kind, float scale,
                 cudaStream_t st, float* const* acc = nullptr,
                 float* const* clr = nullptr) const;
    // one z-mode row per CTA: [forward y-pass of the 3 z-transformed deposit
    // planes at jin, when `correct`] -> corrector (or predictor) of `a` ->
    // inverse y-pass of Ex Ey Ez Bx By Bz (, Rho when nout = 7) into `out`
    // (planes of ny*nz, unscaled); jin and out may be the same planes
    // with `next` (the layer's last corrector, nout = 6): the next layer's
    // predictor too, its E, B after the y-pass into out_next, or with
    // avg_next the average of this layer's E, B and the predicted ones
    int run_spectral_rows(const SpecArgs<float>& a, bool correct, const float* jin, float* out,
                          int nout, cudaStream_t st, const SpecArgs<float>* next = nullptr,
                          float* out_next = nullptr, bool avg_next = false) const;
    // the same for the adjoints of the maps: y-pass of the 6 z-transformed
    // field adjoints at `in`, the corrector's (predictor's) adjoint, and for
    // the corrector the y-pass of the 3 current adjoints into `out`
    int run_adjoint_rows(const AdjSpecArgs<float>& a, bool correct, const float* in, float* out,
                         cudaStream_t st) const;
    ~DttFft();
};

// FP64 half-integer transforms through half-length complex FFTs: the same
// algorithm and kernels as DttFft in FP64, for power-of-two ny, nz in
// [32, 1024] (pass 0 along y into `scratch`, pass 1 along z with the scale)
struct DttFft64 {
    int ny = 0, nz = 0;
    double2* tab_y = nullptr;
    double2* tab_z = nullptr;
    bool spec_rows = false;    // run_spectral_rows available (ny in [128, 512])
    static DttFft64* create(int ny, int nz);   // nullptr when a size is not handled
    int run_pass(int pass, const DttJob<double>& job, double* scratch, cudaStream_t st) const;
    // as DttFft's, in FP64
    int run_cols(int nf, const double* const* in, double* const* out, const int* kind,
                 double scale, cudaStream_t st) const;
    int run_spectral_rows(const SpecArgs<double>& a, bool correct, const double* jin, double* out,
                          int nout, cudaStream_t st, const SpecArgs<double>* next = nullptr,
                          double* out_next = nullptr, bool avg_next = false) const;
    ~DttFft64();
};

template <class T>
int run_dtt_simt_pass(int pass, const DttJob<T>& job, int ny, int nz, const DttMats<T>& my,
                      const DttMats<T>& mz, T* scratch, cudaStream_t st);

// kernel classes of the per-kernel timing (qs_profile_read)
enum KernelClass {
    KC_PUSH = 0, KC_GEMM = 1, KC_SPLIT = 2, KC_SPECTRAL = 3, KC_BEAM_SPECTRA = 4,
    KC_BEAM_PUSH = 5, KC_SEED = 6, KC_MISC = 7, KC_SORT = 8, KC_N = 9
};

template <class T>
int launch_push(const PushArgs<T>& a, int shape, bool precise, cudaStream_t st);

// Beam push + 3-D CIC deposit (movebeam.cpp:14-774).
template <class T>
struct BeamArgs {
    int64_t n;
    int L, My, Mz;
    int32_t *bi, *bj, *bk;
    double *x, *y, *z, *px, *py, *pz;
    const double* w;
    const T* fields3d;    // (L+1) layers x 6 planes
    T* beam3d;            // (L+1) layers x 2 planes (RhoBeam, JxBeam)
    size_t plane;
    double ts, hx, hy, hz, q2m, polarity, bxe, bye, bze;
    double syn_min, elaser_photon;
    int synchrotron;
    int* err;
};
template <class T>
int launch_beam_push(const BeamArgs<T>& a, cudaStream_t st);

// ---- grouping the plasma by cell (sort.cu)
template <class T>
struct PlasmaSet {
    int32_t* cell;
    T *y, *z, *px, *py, *pz, *w;
    int32_t* id;
};
int scan_blocks_count(int ncell);
int launch_count_cells(const int32_t* cell, int64_t n, int ncell, int* cnt, int* err,
                       cudaStream_t st);
int launch_cell_offsets(int* cnt, int ncell, int* loff, int* bsum, int* bpref,
                        unsigned* ticket, int clear, cudaStream_t st);
template <class T>
int launch_scatter(const PlasmaSet<T>& in, const PlasmaSet<T>& out, int64_t n, int ncell,
                   int* cnt, const int* loff, const int* bpref, int* err, cudaStream_t st);
int launch_iota(int32_t* id, int64_t n, cudaStream_t st);

// ---- adjoint (adjoint.cu)

// Push adjoint of one layer: the particles' layer-entry state, the P and C
// fields the push gathered, and the adjoint of its deposit (Jx, Jy, Jz) in;
// the adjoint of the momenta (3 x n, in/out: set by the full push, added to
// by the half pushes) and of the P and C fields (added to) out.
template <class T>
struct PushAdjArgs {
    int64_t n;
    int My, Mz;
    const int32_t* cell;
    const T *y, *z, *px, *py, *pz, *w;
    const T* F;           // 6 planes: the fields the push gathered, (P + C) / 2
    const T* lamD;        // 3 planes
    T* lamPm;             // 3 x n
    T* lamFC;             // 6 planes: the field adjoint of this push (added to)
    T* lamPos;            // CIC: 2 x n adjoint of the in-cell positions y, z (like lamPm)
    size_t plane;
    T sE, hxhy, hxhz, djx0, djy0, djz0, bxe, bye, bze;
    int full, precise;
    float invMy;          // 1 / My (cell -> (j, k) without an integer division)
};
template <class T>
int launch_push_adjoint(const PushAdjArgs<T>& a, cudaStream_t st);
template <class T>
int launch_push_adjoint_cic(const PushAdjArgs<T>& a, cudaStream_t st);
// dst[q] = src[inv[id_to[q]]] for `narr` arrays of n values (T), after
// inv[id_from[p]] = p: carries per-particle adjoints from one particle order
// to another
template <class T>
int launch_permute_adjoint(const int32_t* id_from, const int32_t* id_to, int64_t n, int32_t* inv,
                           const T* src, T* dst, int narr, cudaStream_t st);

// Per-mode adjoint of the predictor / corrector.  Inputs (any may be null =
// zero): lRho, lE (+ lEb, a second contribution), lB, lJb (adjoint of the
// corrector's J input that reaches it from the bank).  Outputs: lJ (total
// adjoint of the corrector's J input), lRhoOld (adjoint of its rho_old), lP
// (adjoint of the 7 P-bank inputs RhoP, ExP, EyP, EzP, JxP, JyP, JzP; set
// when lP_set, else added to) and the beam spectra (added to, with the
// xi-interpolation weights of the forward).
template <class T>
struct AdjSpecArgs {
    int ny, nz;
    T piY, piZ, hx;
    const T* dens_p;
    const T* lRho;
    const T* lE[3];
    const T* lEb[3];
    const T* lB[3];
    const T* lJb[3];
    T* lJ[3];
    T* lRhoOld;
    T* lP[7];
    int lP_set;
    T *lRb0, *lRb1, *lJxb0, *lJxb1;
    T wb0, wb1;
    T *lRbp0, *lRbp1;
    T wp0, wp1;
};
template <class T>
int launch_corrector_adjoint(const AdjSpecArgs<T>& a, cudaStream_t st);
template <class T>
int launch_predictor_adjoint(const AdjSpecArgs<T>& a, cudaStream_t st);
template <class T>
int launch_add_point(T* plane_ex, size_t idx, const T* v, int layer, cudaStream_t st);
// acc += x over n values
template <class T>
int launch_add_planes(T* acc, const T* x, size_t n, cudaStream_t st);
// The particle blocks of the hand-off buffer (pack.cu): the m particles
// ordered by cell, load order within a cell (key = load ids, or null when the
// device order is the load order), as 12 double rows at out.  Scratch: cnt
// and fill (ncell ints, zeroed by the caller), start (ncell + 1), ord (m).
template <class T>
struct PackArgs {
    int64_t m;
    int My, ncell;
    const int32_t* cell;
    const int32_t* key;
    const T *y, *z, *px, *py, *pz, *w;
    double q2m;
    int *cnt, *start, *fill;
    int32_t* ord;
    double* out;
    int* err;
};
template <class T>
int launch_pack_particles(const PackArgs<T>& a, cudaStream_t st);
// UnpackLayer's particle blocks on the device (pack.cu): `buf` holds the 12
// double rows of m particles.  launch_unpack_check gives every row its cell
// (key_cell; -1 for a bad row), counts the cells into cnt (ncell ints, zeroed
// by the caller) and lowers *bad (set to m by the caller) to the lowest bad
// row.  launch_unpack_order (after a clean check) orders the rows by cell,
// buffer order within a cell (start: ncell + 1, fill: ncell zeroed, ord: m),
// and writes them into the plasma arrays; *nonuniform is set unless row r
// lies in cell r / ppc for every r.
template <class T>
struct UnpackArgs {
    int64_t m;
    int My, Mz, ncell, ppc;
    const double* buf;
    double q2m;
    int32_t* key_cell;
    int *cnt, *start, *fill;
    int32_t* ord;
    unsigned long long* bad;
    int* nonuniform;
    int32_t* cell;
    T *y, *z, *px, *py, *pz, *w;
    int* err;
};
template <class T>
int launch_unpack_check(const UnpackArgs<T>& a, cudaStream_t st);
template <class T>
int launch_unpack_order(const UnpackArgs<T>& a, cudaStream_t st);
// out = w0 a + w1 b over n values, in double
template <class T>
int launch_pack_mix(const T* a, const T* b, double w0, double w1, size_t n, double* out,
                    cudaStream_t st);

// out = (P + C) / 2 over n values: the fields a push gathers, kept for its adjoint
template <class T>
int launch_avg_planes(const T* P, const T* C, T* out, size_t n, cudaStream_t st);

// dst[q][i] = src[q][i] for the 5 particle arrays (y, z, px, py, pz) and
// cdst[i] = csrc[i] when csrc is set, i < n: a layer's entry state, saved by
// the adjoint's recomputation in one launch
template <class T>
struct StateCopy {
    const T* src[5];
    T* dst[5];
    const int32_t* csrc;
    int32_t* cdst;
    int64_t n;
};
template <class T>
int launch_save_state(const StateCopy<T>& c, cudaStream_t st);

// d loss / d (beam macro-particle weight) from the adjoint of the real beam
// currents (lb3: layers lo .. L x 2 planes RhoBeam, JxBeam; zero below lo).
template <class T>
struct BeamGradArgs {
    int64_t n;
    int L, My, Mz;
    int lo;
    const int32_t *bi, *bj, *bk;
    const double *x, *y, *z, *px, *py, *pz;
    const T* lb3;
    size_t plane;
    double polarity;
    double* out;
};
template <class T>
int launch_beam_weight_grad(const BeamGradArgs<T>& a, cudaStream_t st);

}  // namespace qs
