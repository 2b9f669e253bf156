/*
 * qs_oracle.h — CPU oracle of the quasi-static xi-layer loop (TEST
 * INFRASTRUCTURE ONLY: the checker the GPU path is compared against; never
 * part of the product path).
 *
 * A plain FP64 C++ restatement of the reference's live host path:
 *   movepart_splitlayer.cpp:25-1711   (march, layer, plasma push, deposit,
 *                                      guard exchange)
 *   movefieldshydrolinlayersplit.cpp:222-1671 (Guess / Iterate spectral solve)
 *   movebeam.cpp:14-774               (beam push + 3-D CIC deposit)
 * with its own half-integer transforms implementing the FFTW REDFT11 /
 * RODFT11 definitions (FFTW 3 is a system library of the reference, not
 * vendored, version unpinned).
 *
 * Parity status (the pins, each run by the tests):
 *  - the plasma push with its deposit and guard fold, and the beam push with
 *    its synchrotron loss and 3-D deposit, against the reference's own host
 *    code (movepart_splitlayer.cpp:781-1544, 1685-1711; movebeam.cpp:14-774)
 *    compiled from the reference checkout (oracle/ref_pin.cpp, make refpin):
 *    particle states and cells bit for bit, deposits to the order of the
 *    additions;
 *  - the per-mode predictor and corrector against the reference's CUDA twins
 *    of them (CUDA_WRAP/linearized.cu, oracle/ref_harness.cu, make ref);
 *  - the transforms against scipy.fft dct/dst type 4 (FFTW's published
 *    REDFT11 / RODFT11 definitions) and direct O(N^2) sums, FFTW itself being
 *    a system dependency of the reference that is not present here;
 *  - the march's orchestration (gathers, normalisation, the P / C layer
 *    swaps) by its line-cited restatement and known answers: zero beam, the
 *    linear response of the predictor's propagator, charge bookkeeping.
 */
#ifndef QS_ORACLE_H
#define QS_ORACLE_H

#include <stdint.h>
#include "../include/qsb200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qso qso;

/* Per-mode spectral maps (FP64), in the argument convention of the
 * reference's CUDA twins linearized_kernel / linearizedIteratekernel. */
void qso_predictor_modes(int ny, int nz, double hx, double d, double Ylength,
                         double Zlength, const double* fRhoP, const double* fJxP,
                         const double* fJyP, const double* fJzP, const double* fExP,
                         const double* fEyP, const double* fEzP, const double* fRhoBeam,
                         const double* fRhoBeamP, const double* fJxBeam, double* fRho,
                         double* fEx, double* fEy, double* fEz, double* fJx, double* fJy,
                         double* fJz, double* fBx, double* fBy, double* fBz);
void qso_corrector_modes(int ny, int nz, double hx, double d, double Ylength,
                         double Zlength, const double* fRhoP, const double* fJxP,
                         const double* fJyP, const double* fJzP, const double* fEyP,
                         const double* fEzP, const double* fRhoBeam, const double* fRhoBeamP,
                         const double* fJxBeam, const double* fJx, const double* fJy,
                         const double* fJz, double* fRho, double* fEx, double* fEy,
                         double* fEz, double* fBx, double* fBy, double* fBz);

void qso_set_threads(int n);
int qso_get_threads(void);

int qso_create(const qs_config* cfg, qso** out);
void qso_destroy(qso* o);

int qso_load_beam(qso* o, int64_t n, const int32_t* i, const int32_t* j,
                  const int32_t* k, const double* x, const double* y,
                  const double* z, const double* px, const double* py,
                  const double* pz, const double* w);
int qso_get_beam(qso* o, int64_t n, int32_t* i, int32_t* j, int32_t* k,
                 double* x, double* y, double* z, double* px, double* py,
                 double* pz, double* w);
int64_t qso_beam_count(const qso* o);

int qso_load_front_plasma(qso* o, int64_t n, const int32_t* cell,
                          const double* y, const double* z, const double* px,
                          const double* py, const double* pz, const double* w);
int64_t qso_plasma_count(const qso* o);
/* Particles of the layer in flight, reported in the order they were loaded
 * (particle id order), with their current cell. */
int qso_get_plasma(qso* o, int64_t n, int32_t* cell, double* y, double* z,
                   double* px, double* py, double* pz, double* w);

int qso_set_layer(qso* o, int which, int field, const double* data);
int qso_get_layer(qso* o, int which, int field, double* out);
int qso_get_field3d(qso* o, int field, int layer, double* out);
int qso_set_beam_currents(qso* o, int field, int layer, const double* data);
int qso_get_beam_currents(qso* o, int field, int layer, double* out);
int qso_get_onaxis_ex(qso* o, double* out);

/* Fields (Ex..Bz, field 0..5) of stored layer 0..nx: the interior plane and
 * its periodic guard ring, as the march leaves them for the beam push. */
int qso_set_field3d(qso* o, int field, int layer, const double* data);
/* Wake potential on axis (a derived quantity the reference does not
 * compute): psi(nx) = 0, psi(i) = psi(i+1) + hx (Ex_i + Ex_{i+1})/2 over the
 * on-axis Ex of the last march. */
int qso_get_psi(qso* o, double* out);
/* FP64 sums over the interior cells of every layer of the last march:
 * rho[nx] of f_Dens after the layer's last Iterate (the corrected density,
 * movefieldshydrolinlayersplit.cpp:1545-1602), jx[nx] of the Jx deposit of
 * its full push, rho_beam[nx+1] of RhoBeam of the beam-current store.  Any
 * pointer may be NULL. */
int qso_get_charge_sums(qso* o, double* rho, double* jx, double* rho_beam);
int qso_step(qso* o);
/* Specie::Density (plasma.cpp:6-399) of a profile at (x, y, z). */
double qso_density(const qs_density_profile* p, double x, double y, double z);
/* The plasma profile (NULL: uniform cfg.plasma_density) and the phase. */
int qso_set_density_profile(qso* o, const qs_density_profile* p);
int qso_set_phase(qso* o, double phase);
/* Weights Mesh::SeedParticles gives the front particles of each cell
 * (j + ny*k), 0 where it seeds none. */
int qso_front_weights(qso* o, double* out);
/* PackLayer / UnpackLayer (para.cpp:94-285) in the reference's buffer
 * layout; the unpacked layer is the front of the next march. */
int64_t qso_layer_pack_size(const qso* o);
int qso_pack_layer(qso* o, double* buf, int64_t n);
int qso_unpack_layer(qso* o, const double* buf, int64_t n);
int qso_move_beam_particles(qso* o);
int qso_move_all_split_layers(qso* o);
int qso_begin_march(qso* o);
int qso_layer_begin(qso* o, int iLayer, int iSplit);
int qso_move_split_layer(qso* o, int iLayer, int iSplit);
int qso_guess_fields(qso* o, int iLayer, int iSplit);
int qso_move_particles_layer(qso* o, int iLayer, int iSplit, int iFullStep);
int qso_iterate_fields(qso* o, int iLayer, int iSplit, int iter,
                       double* rel_err);
int qso_layer_end(qso* o, int iLayer, int iSplit);

/* 1-D and 2-D half-integer transforms, unnormalised FFTW definitions.
 * 2-D: nz x ny planes (y fastest), kind_z along z, kind_y along y.
 * direct != 0 selects the O(N^2) sums instead of the FFT algorithm. */
int qso_dtt1d(int n, int kind, const double* in, double* out, int direct);
int qso_transform2d(int nz, int ny, int kind_z, int kind_y, int batch,
                    const double* in, double* out, int direct);

/* Kernel-level oracle of one plasma sub-push over a particle array
 * (MoveParticlesLayerSplit + DepositCurrentsInCellSplit + the periodic fold
 * of ExchangeCurrentsSplit).  P and C hold 6 interior planes each
 * (Ex,Ey,Ez,Bx,By,Bz); dep holds 4 planes (Jx,Jy,Jz,Dens) that are ADDED to;
 * dep_cell receives the cell (j + ny*k, folded) of each particle's last
 * deposit; on full != 0 the particle state is updated in place (and in CIC
 * mode cell[] too).  The f32 variant runs the same arithmetic in float;
 * precise != 0 selects the cell-relative position update (the FP32 path's
 * form) instead of the reference's ytmp + j form. */
int qso_push_layer_f64(const qs_config* cfg, int64_t n, int32_t* cell,
                       double* y, double* z, double* px, double* py,
                       double* pz, const double* w, const double* P,
                       const double* C, double* dep, int32_t* dep_cell,
                       int full, int precise);
int qso_push_layer_f32(const qs_config* cfg, int64_t n, int32_t* cell,
                       float* y, float* z, float* px, float* py, float* pz,
                       const float* w, const float* P, const float* C,
                       float* dep, int32_t* dep_cell, int full, int precise);

#ifdef __cplusplus
}
#endif
#endif
