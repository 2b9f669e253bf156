/*
 * mesh_qs.h — a C++ adapter over qsb200.h that keeps the method names of the
 * reference's class Mesh (mesh.h:55-76) for the hot path, so that
 * Domain::Step (step.cpp:63-105) can call
 *     meshqs->MoveBeamParticles(); meshqs->MoveAllSplitLayers();
 * in place of the Mesh members.  Header only; link with -lqsb200.
 *
 * Every library status other than QS_OK becomes a std::runtime_error with
 * the library's message (the reference calls exit() at those sites).
 */
#ifndef MESH_QS_H
#define MESH_QS_H

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "qsb200.h"

class MeshQS {
 public:
  // The geometry and namelist values of Domain/Mesh/Specie the hot path uses
  // (domain.cpp:42-57, elements.cpp:11-67).
  MeshQS(int My, int Mz, int Mx, double Hx, double Hy, double Hz, double Ts, int nIter,
         int NxSplit, int ppc, double density, double wavelength,
         int precision = QS_PREC_FP32, int shape = QS_SHAPE_CIC) {
    qs_config c;
    qs_config_default(&c);
    c.ny = My; c.nz = Mz; c.nx = Mx;
    c.hx = Hx; c.hy = Hy; c.hz = Hz; c.ts = Ts;
    c.n_iter = nIter; c.nx_split = NxSplit; c.ppc = ppc;
    c.plasma_density = density; c.wavelength = wavelength;
    c.precision = precision;   // QS_PREC_FP32 (FFT transforms) is the measured default;
                               // QS_PREC_FP64 the plain FP64 path
    c.shape = shape;           // QS_SHAPE_CIC, or QS_SHAPE_NGP (the reference's live path)
    check(qs_create(&c, &h_), nullptr);
  }
  ~MeshQS() { qs_destroy(h_); }
  MeshQS(const MeshQS&) = delete;
  MeshQS& operator=(const MeshQS&) = delete;

  // Mesh::SeedBeamParticles (mesh.cpp:108-234): the caller's sampled beam
  void LoadBeam(int64_t n, const int32_t* i, const int32_t* j, const int32_t* k,
                const double* x, const double* y, const double* z, const double* px,
                const double* py, const double* pz, const double* w) {
    check(qs_load_beam(h_, n, i, j, k, x, y, z, px, py, pz, w), h_);
  }
  // Mesh::SeedFrontParticles (mesh.cpp:98-106) from host arrays, grouped by cell
  void LoadFrontParticles(int64_t n, const int32_t* cell, const double* y, const double* z,
                          const double* px, const double* py, const double* pz,
                          const double* w) {
    check(qs_load_front_plasma(h_, n, cell, y, z, px, py, pz, w), h_);
  }
  // ... or seeded on the device
  void SeedFrontParticles(uint64_t step) { check(qs_seed_front_plasma(h_, step), h_); }

  void MoveBeamParticles() { check(qs_move_beam_particles(h_), h_); }
  void MoveAllSplitLayers() { check(qs_move_all_split_layers(h_), h_); }
  void MoveSplitLayer(int iLayer, int iSplit) {
    check(qs_layer_begin(h_, iLayer, iSplit), h_);
    check(qs_move_split_layer(h_, iLayer, iSplit), h_);
    check(qs_layer_end(h_, iLayer, iSplit), h_);
  }
  void GuessFieldsHydroLinLayerSplit(int iLayer, int iSplit) {
    check(qs_guess_fields(h_, iLayer, iSplit), h_);
  }
  void MoveParticlesLayerSplit(int iLayer, int iSplit, int iFullStep) {
    check(qs_move_particles_layer(h_, iLayer, iSplit, iFullStep), h_);
  }
  double IterateFieldsHydroLinLayerSplit(int iLayer, int iSplit, int N_iter) {
    double err = 0;
    check(qs_iterate_fields(h_, iLayer, iSplit, N_iter, &err), h_);
    return err;
  }

  // the longitudinal field on axis of every layer (reading Cell::f_Ex)
  std::vector<double> OnAxisEx(int Mx) {
    std::vector<double> ex((size_t)Mx);
    check(qs_get_onaxis_ex(h_, ex.data()), h_);
    return ex;
  }
  qs_handle* handle() { return h_; }

 private:
  static void check(qs_status s, qs_handle* h) {
    if (s != QS_OK)
      throw std::runtime_error(std::string(qs_status_string(s)) + ": " + qs_last_error(h));
  }
  qs_handle* h_ = nullptr;
};

#endif /* MESH_QS_H */
