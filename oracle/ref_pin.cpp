// ref_pin.cpp — TEST INFRASTRUCTURE ONLY: the pin of the oracle against the
// reference itself, never part of the product.
//
// It drives the reference's own plasma push, Mesh::MoveParticlesLayerSplit
// (movepart_splitlayer.cpp:781-1544) with its guard fold ExchangeCurrentsSplit
// (:1685-1711), and its beam push, Mesh::MoveBeamParticles with MoveBeamInCell
// (movebeam.cpp:14-774), on decks and particles handed in as plain arrays, so
// that the oracle's restatements of them (oracle/qs_oracle.cpp) can be
// compared with the reference bit for bit (tests/test_oracle_pin.py).  The
// reference files are compiled where they lie by oracle/Makefile (target
// refpin, output oracle/_ref/librefpin.so) together with the reference's
// cells.cpp, particles.cpp, elements.cpp and plasma.cpp; stub headers in
// oracle/ref_stubs/ give the type names of FFTW, MPI and HDF5, which those
// files name but do not call on these paths.
//
// The reference's Domain, Mesh and Controls constructors read namelist files
// and set up MPI, HDF5 and the CUDA plug-ins, so those objects are laid out
// field by field here (the access specifiers are opened for this file only);
// Cell, Specie and the particles are built by the reference's own
// constructors.  The functions those files call outside them are stand-ins:
//   - the CUDA_WRAP diagnostics and layer copies do nothing (the reference's
//     run_control.h selects the host computation for both pushes);
//   - one MPI rank (GetRank 0, GetSize 1);
//   - the namelist reader hands every entry its default (no file);
//   - Mesh::ClearBeamCurrents zeroes the four beam currents of every cell, as
//     mesh.cpp:648-663 does;
//   - the synchrotron photon histogram is not recorded (the momentum loss,
//     movebeam.cpp:446-491, is the reference's);
//   - the Domain accessors the files call out of line return its fields.
#include <cassert>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>
#include <math.h>
#include <memory.h>
#include <stdio.h>
#include <stdlib.h>
#include <sys/time.h>
#include <cuda.h>
#include <cublas_v2.h>
#include <driver_types.h>

#include "../include/qsb200.h"

#define private public
#define protected public
#include "vlpl3d.h"
#include "run_control.h"
#include "CUDA_WRAP/beam_copy.h"
#include "CUDA_WRAP/cuBeam.h"
#include "CUDA_WRAP/cuBeamValues.h"
#include "CUDA_WRAP/cuLayers.h"
#include "CUDA_WRAP/paraLayers.h"
#include "CUDA_WRAP/paraCPUlayers.h"
#include "CUDA_WRAP/plasma_particles.h"
#include "CUDA_WRAP/diagnostic_print.h"
#include "CUDA_WRAP/cuParticles.h"
#include "para.h"
#undef private
#undef protected

// ----------------------------------------------------------- stand-ins
int CUDA_WRAP_write_beam_value(int, int, int, double*, double) { return 0; }
int CUDA_WRAP_write_plasma_value(int, int, int, double) { return 0; }
void getLayersPC(cudaLayer**, cudaLayer**) {}
int ReceiveLayer(cudaLayer*, int, int, int) { return 0; }
int SendLayer(cudaLayer*, int, int, int) { return 0; }
int cuLayerPrintCentre(cudaLayer*, int, Mesh*, Cell*, char*) { return 0; }
void cuMoveSplitParticles(int, int, cudaLayer*, cudaLayer*, int, int, double, double, double,
                          double*, double*, double*, double*, int, int) {}
int CUDA_WRAP_copy3Dfields(Mesh*, Cell*, int, int, int) { return 0; }
int CUDA_WRAP_alloc3Dfields(int, int, int) { return 0; }
int CUDA_WRAP_clearCurrents(int, int, int) { return 0; }
int CUDA_WRAP_createNewLayer(cudaLayer**, cudaLayer*) { return 0; }
int CUDA_WRAP_setLayerToMesh(Mesh*, Cell*, int, int, int, cudaLayer*, int) { return 0; }
int CUDA_WRAP_alloc3Dcurrents(int, int, int) { return 0; }
int CUDA_WRAP_copyLayerFrom3D(int, int, int, int, cudaLayer**) { return 0; }
int CUDA_WRAP_allocLayerOnHost(cudaLayer**, int, int, int) { return 0; }
int CUDA_WRAP_getLayerFromMesh(Mesh*, Cell*, int, int, int, cudaLayer**) { return 0; }
int CUDA_WRAP_copyLayerToDevice(Mesh*, Cell*, int, int, int, cudaLayer**) { return 0; }
int CUDA_WRAP_printBeamDensity3D(Mesh*, int, char*) { return 0; }
int CUDA_DEBUG_print3DmatrixLayer(double*, int, int, int, char*) { return 0; }
int CUDA_WRAP_printLayerParticles(cudaLayer*, char*) { return 0; }
int CUDA_WRAP_check_all_hidden_fields(Mesh*, int, int, int, Cell*, Cell*, cudaLayer*,
                                      cudaLayer*) {
    return 0;
}
int CUDA_WRAP_copyLayerDeviceToDevice(int, int, int, cudaLayer*, cudaLayer*) { return 0; }
int CUDA_WRAP_getLayerParticlesNumber(Mesh*, Cell*, int, int, int, char*) { return 0; }
int CUDA_WRAP_printParticleListFromHost(Mesh*, Cell*, int, int, int, char*) { return 0; }
double* d_Ey3D = nullptr;
double* h_beam_values = nullptr;
int GetRank() { return 0; }
int GetSize() { return 1; }

NList::NList(const char*) : head(nullptr), tail(nullptr) {}
NList_Entry* NList::AddEntry(char*, int* ptr, int v) { *ptr = v; return nullptr; }
NList_Entry* NList::AddEntry(char*, long* ptr, long v) { *ptr = v; return nullptr; }
NList_Entry* NList::AddEntry(char*, double* ptr, double v) { *ptr = v; return nullptr; }
int NList::read(FILE*) { return 0; }
long Specie::Save(FILE*) { return 0; }
long Specie::Load(FILE*) { return 0; }
long IonSpecie::Save(FILE*) { return 0; }
long IonSpecie::Load(FILE*) { return 0; }
double IonSpecie::GetADKprob(double, int) { return 0.0; }
void Synchrotron::AddParticle(Particle*, double, double, double, double) {}
Particle* Boundary::AddZombie(Particle* p, Cell*) { return p; }

Domain* Domain::p_D = nullptr;
Specie* Domain::GetSpecie(int sort) { return pa_Species[sort]; }
double Domain::GetTs() { return f_Ts; }
long Domain::Add2Specie(int) { return 0; }
long Domain::RemoveFromSpecie(int) { return 0; }

void Mesh::ClearBeamCurrents() {
    for (long n = 0; n < l_sizeXYZ; n++) {
        Cell& c = p_CellArray[n];
        c.f_JxBeam = c.f_JyBeam = c.f_JzBeam = c.f_RhoBeam = 0.;
    }
}
[[noreturn]] static void not_on_the_pinned_paths(const char* what) {
    std::fprintf(stderr, "ref_pin: %s is not on the pinned paths\n", what);
    std::abort();
}
void Mesh::ClearCurrentsSplit() { not_on_the_pinned_paths("ClearCurrentsSplit"); }
void Mesh::ClearRhoSplit() { not_on_the_pinned_paths("ClearRhoSplit"); }
void Mesh::SeedFrontParticles() { not_on_the_pinned_paths("SeedFrontParticles"); }
void Mesh::GuessFieldsHydroLinLayerSplit(int, int) { not_on_the_pinned_paths("Guess"); }
double Mesh::IterateFieldsHydroLinLayerSplit(int, int, int) { not_on_the_pinned_paths("Iterate"); }

// ------------------------------------------------------------- set-up
namespace {

template <class T>
T* raw_object() {
    void* p = ::operator new(sizeof(T));
    std::memset(p, 0, sizeof(T));
    return static_cast<T*>(p);
}

struct World {
    Domain* d = nullptr;
    Controls* cntrl = nullptr;
    UnitsCGS* cgs = nullptr;
    Synchrotron* syn = nullptr;
    Specie* electrons = nullptr;
    Specie* beam = nullptr;
    Specie* species[2] = {nullptr, nullptr};
};

// the Domain, Controls, units and the plasma electrons of a deck
World make_world(const qs_config* c, int nx) {
    World w;
    w.cgs = raw_object<UnitsCGS>();
    w.cgs->f_Qe = 1.;
    w.cgs->f_Me = 1.;
    w.cgs->f_Clight = 1.;
    w.cgs->f_Wavelength = c->wavelength;
    w.cntrl = raw_object<Controls>();
    w.syn = raw_object<Synchrotron>();
    w.syn->f_SynMin = c->syn_min;
    w.d = raw_object<Domain>();
    new (&w.d->out_Flog) std::ofstream();
    new (&w.d->out_Fig8) std::ofstream();
    Domain* d = w.d;
    d->f_Ts = c->ts;
    d->f_Hx = c->hx;
    d->i_NxSplit = c->nx_split;
    d->f_HxSplit = c->hx / c->nx_split;
    d->f_Hy = c->hy;
    d->f_Hz = c->hz;
    d->i_nIter = c->n_iter;
    d->f_Xlength = c->hx * nx;
    d->f_Ylength = c->hy * c->ny;
    d->f_Zlength = c->hz * c->nz;
    d->f_Wavelength = c->wavelength;
    d->i_Nsorts = 2;
    d->f_BxExternal = c->bx_ext;
    d->f_ByExternal = c->by_ext;
    d->f_BzExternal = c->bz_ext;
    d->p_CGS = w.cgs;
    d->p_Cntrl = w.cntrl;
    d->p_Synchrotron = w.syn;
    d->pa_Species = w.species;
    Domain::p_D = d;
    // the plasma electrons through the reference's constructor (namelist
    // defaults), then the deck's values
    w.electrons = new Specie((char*)"Electrons", nullptr);
    Specie* s = w.electrons;
    s->l_perCell = c->ppc;
    s->f_q2m = c->plasma_q2m;
    s->f_dJx = c->plasma_djx0;
    s->f_dJy = c->plasma_djy0;
    s->f_dJz = c->plasma_djz0;
    s->f_dRho = c->plasma_drho0;
    s->f_Narb = c->plasma_density;
    s->f_Begin = -1e30;
    s->f_End = 1e30;
    s->f_PlateauBegin = -1e30;
    s->f_PlateauEnd = 1e30;
    s->i_ScatterFlag = 0;
    s->i_BeamFlag = 0;
    w.species[0] = s;
    // the driver: a beam species (sort 1), electrons of the deck's q/m
    w.beam = new Specie((char*)"Beam", nullptr);
    w.beam->i_Sort = 1;
    w.beam->f_q2m = c->beam_q2m;
    w.beam->i_BeamFlag = 1;
    w.beam->i_ScatterFlag = 0;
    w.species[1] = w.beam;
    return w;
}

void free_world(World& w) {
    delete w.electrons;
    delete w.beam;
    w.d->out_Flog.~basic_ofstream();
    w.d->out_Fig8.~basic_ofstream();
    ::operator delete(w.d);
    ::operator delete(w.cntrl);
    ::operator delete(w.cgs);
    ::operator delete(w.syn);
    Domain::p_D = nullptr;
}

Mesh* make_mesh(int nx, int ny, int nz) {
    Mesh* m = raw_object<Mesh>();
    m->SetSizes(nx, ny, nz, 2, 2, 2);
    return m;
}

}  // namespace

// ---------------------------------------------------------- entry points
extern "C" {

// One sub-push of the plasma over a P and a C layer: the reference's
// MoveParticlesLayerSplit(iLayer = 0, iSplit = 0, iFullStep = full) and its
// ExchangeCurrentsSplit.  Particles are given grouped by cell (cell = j + ny
// k, in list order within a cell); P and C hold 6 interior planes (Ex, Ey,
// Ez, Bx, By, Bz), periodic in the guard ring.  Out: dep = 4 interior planes
// Jx, Jy, Jz, Dens of the C layer; on a full push the particles' new state and
// cell (the layer they were relinked into), in input order.
int refpin_push_layer(const qs_config* c, int64_t n, const int32_t* cell, double* y, double* z,
                      double* px, double* py, double* pz, const double* w, const double* P,
                      const double* C, double* dep, int32_t* cell_out, int full) {
    const int My = c->ny, Mz = c->nz;
    World world = make_world(c, 4);
    Mesh* m = make_mesh(4, My, Mz);
    const long nyz = m->l_sizeY * m->l_sizeZ;
    m->p_CellLayerP = new Cell[nyz];
    m->p_CellLayerC = new Cell[nyz];
    const size_t pl = (size_t)My * Mz;
    for (int k = -2; k < Mz + 2; k++)
        for (int j = -2; j < My + 2; j++) {
            const size_t s = (size_t)((j + My) % My) + (size_t)My * ((k + Mz) % Mz);
            Cell& pc = m->p_CellLayerP[m->GetNyz(j, k)];
            Cell& cc = m->p_CellLayerC[m->GetNyz(j, k)];
            for (int f = 0; f < 6; f++) {
                pc.f_Fields[f] = P[f * pl + s];
                cc.f_Fields[f] = C[f * pl + s];
            }
        }
    // the particles of each cell, created last first so that the head-first
    // lists hold them in input order
    std::vector<Particle*> parts((size_t)n, nullptr);
    for (int64_t q = n - 1; q >= 0; q--) {
        const int j = cell[q] % My, k = cell[q] / My;
        parts[(size_t)q] = new Electron(&m->p_CellLayerP[m->GetNyz(j, k)], w[q], 0., y[q], z[q],
                                        px[q], py[q], pz[q], c->plasma_q2m, 0);
    }
    m->MoveParticlesLayerSplit(0, 0, full, 1.);
    m->ExchangeCurrentsSplit(0);
    for (int k = 0; k < Mz; k++)
        for (int j = 0; j < My; j++) {
            const Cell& cc = m->p_CellLayerC[m->GetNyz(j, k)];
            const size_t s = (size_t)j + (size_t)My * k;
            dep[s] = cc.f_Jx;
            dep[pl + s] = cc.f_Jy;
            dep[2 * pl + s] = cc.f_Jz;
            dep[3 * pl + s] = cc.f_Dens;
        }
    if (full) {
        std::unordered_map<const Particle*, int32_t> where;
        for (int k = 0; k < Mz; k++)
            for (int j = 0; j < My; j++)
                for (Particle* p = m->p_CellLayerC[m->GetNyz(j, k)].p_Particles; p; p = p->p_Next)
                    where[p] = j + My * k;
        for (int64_t q = 0; q < n; q++) {
            const Particle* p = parts[(size_t)q];
            y[q] = p->f_Y;
            z[q] = p->f_Z;
            px[q] = p->f_Px;
            py[q] = p->f_Py;
            pz[q] = p->f_Pz;
            auto it = where.find(p);
            cell_out[q] = it == where.end() ? -1 : it->second;
        }
    }
    for (Particle* p : parts) delete p;
    delete[] m->p_CellLayerP;
    delete[] m->p_CellLayerC;
    ::operator delete(m);
    free_world(world);
    return 0;
}

// The beam push over the 3-D field array: the reference's MoveBeamParticles.
// fields: (nx+1) layers x 6 interior planes, periodic in y and z; the beam
// particles with their cells (i, j, k), fractions and momenta (input order).
// Out: the particles' new state and cells, and cur = (nx+1) layers x 4
// interior planes JxBeam, JyBeam, JzBeam, RhoBeam.
int refpin_beam_push(const qs_config* c, int64_t nb, int32_t* bi, int32_t* bj, int32_t* bk,
                     double* x, double* y, double* z, double* px, double* py, double* pz,
                     const double* w, const double* fields, double* cur) {
    const int L = c->nx, My = c->ny, Mz = c->nz;
    World world = make_world(c, L);
    world.syn->f_SynMin = c->synchrotron ? c->syn_min : 1e300;
    Mesh* m = make_mesh(L, My, Mz);
    m->p_CellArray = new Cell[m->l_sizeXYZ];
    // each cell's per-species density (MoveBeamInCell adds the beam's into
    // it); the Cell destructor frees it
    for (long n = 0; n < m->l_sizeXYZ; n++) m->p_CellArray[n].f_DensArray = new double[2]();
    const size_t pl = (size_t)My * Mz;
    for (int i = 0; i <= L; i++)
        for (int k = -2; k < Mz + 2; k++)
            for (int j = -2; j < My + 2; j++) {
                const size_t s = (size_t)((j + My) % My) + (size_t)My * ((k + Mz) % Mz);
                Cell& cc = m->p_CellArray[m->GetN(i, j, k)];
                for (int f = 0; f < 6; f++) cc.f_Fields[f] = fields[((size_t)i * 6 + f) * pl + s];
            }
    std::vector<Particle*> parts((size_t)nb, nullptr);
    for (int64_t q = nb - 1; q >= 0; q--) {
        Particle* p = new Particle(nullptr, w[q], x[q], y[q], z[q], px[q], py[q], pz[q],
                                   c->beam_q2m, 1);
        m->p_CellArray[m->GetN(bi[q], bj[q], bk[q])].AddBeamParticle(p);
        parts[(size_t)q] = p;
    }
    m->MoveBeamParticles();
    std::unordered_map<const Particle*, long> where;
    for (long n = 0; n < m->l_sizeXYZ; n++)
        for (Particle* p = m->p_CellArray[n].p_BeamParticles; p; p = p->p_Next) where[p] = n;
    for (int64_t q = 0; q < nb; q++) {
        const Particle* p = parts[(size_t)q];
        x[q] = p->f_X;
        y[q] = p->f_Y;
        z[q] = p->f_Z;
        px[q] = p->f_Px;
        py[q] = p->f_Py;
        pz[q] = p->f_Pz;
        auto it = where.find(p);
        if (it == where.end()) {
            bi[q] = bj[q] = bk[q] = -9;
        } else {   // n = i + dMx + sizeX (j + dMy + sizeY (k + dMz))
            long n = it->second;
            const long i = n % m->l_sizeX - m->l_dMx;
            n /= m->l_sizeX;
            bj[q] = (int32_t)(n % m->l_sizeY - m->l_dMy);
            bk[q] = (int32_t)(n / m->l_sizeY - m->l_dMz);
            bi[q] = (int32_t)i;
        }
    }
    for (int i = 0; i <= L; i++)
        for (int k = 0; k < Mz; k++)
            for (int j = 0; j < My; j++) {
                const Cell& cc = m->p_CellArray[m->GetN(i, j, k)];
                const size_t s = (size_t)j + (size_t)My * k;
                cur[((size_t)i * 4 + 0) * pl + s] = cc.f_JxBeam;
                cur[((size_t)i * 4 + 1) * pl + s] = cc.f_JyBeam;
                cur[((size_t)i * 4 + 2) * pl + s] = cc.f_JzBeam;
                cur[((size_t)i * 4 + 3) * pl + s] = cc.f_RhoBeam;
            }
    for (Particle* p : parts) delete p;
    delete[] m->p_CellArray;
    ::operator delete(m);
    free_world(world);
    return 0;
}

}  // extern "C"
