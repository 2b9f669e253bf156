/*
 * qsb200.h — C ABI of the B200-native quasi-static xi-layer loop.
 *
 * The library replaces the hot path of the snytav/tertia quasi-static
 * plasma-wakefield code: the xi-march over transverse layers (plasma push +
 * deposit, spectral half-integer field solve) and the driver-beam push.
 * Every entry point below names the reference function or plug-in
 * (CUDA_WRAP_*) it replaces.  All calls return qs_status; nothing calls
 * exit().  Pointers are HOST pointers unless the name ends in _dev.
 * A handle owns all device memory and one CUDA stream; use one handle per
 * host thread.
 *
 * Geometry (reference Mesh, mesh.h:10-160):
 *   ny = l_My, nz = l_Mz transverse cells; nx = l_Mx xi-layers.
 *   Layer i = 0 .. nx-1; layer nx is the front layer where fresh plasma is
 *   seeded (Mesh::SeedFrontParticles, mesh.cpp:98-106).
 *   A transverse plane is stored row-major with y fastest:
 *   index = j + ny*k  (the reference's spectral index n = j + ny*k,
 *   movefieldshydrolinlayersplit.cpp:577).
 *   "Ex" is the reference's longitudinal field (x is the xi axis).
 */
#ifndef QSB200_H
#define QSB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum qs_status {
    QS_OK = 0,
    QS_ERR_INVALID = 1,        /* bad argument or configuration              */
    QS_ERR_CUDA = 2,           /* CUDA runtime / driver error                */
    QS_ERR_OOM = 3,            /* device allocation failed                   */
    QS_ERR_DEVICE = 4,         /* device-side error flag raised (see below)  */
    QS_ERR_BEAM_CURRENT = 5,   /* |JxBeam| > 10 in a layer: the reference's
                                  "Too large beam current" exit(20),
                                  movefieldshydrolinlayersplit.cpp:618-621    */
    QS_ERR_PARTICLE_RANGE = 6, /* particle fraction outside [0,1]: the
                                  reference's exit(-212) / exit(-12),
                                  movepart_splitlayer.cpp:945-951,
                                  movebeam.cpp:201-207                        */
    QS_ERR_UNSUPPORTED = 7,    /* valid request this build does not handle  */
    QS_ERR_TIMEOUT = 8,        /* a bounded device wait gave up              */
    QS_ERR_STATE = 9           /* call out of sequence                       */
} qs_status;

/* Arithmetic of the layer loop. */
typedef enum qs_precision {
    QS_PREC_FP64 = 0,    /* plain FP64 everywhere (the FP64 GPU path)               */
    QS_PREC_FP32 = 1,    /* FP32 push/deposit, FP32 transforms: half-length complex
                            FFTs for power-of-two sizes, else FP32 matrix passes */
    QS_PREC_TF32X3 = 2,  /* FP32 push/deposit, transforms as 3-term TF32 split
                            products on the tcgen05 tensor cores, FP32 accumulate   */
    QS_PREC_BF16X3 = 3,  /* as above with 3-term BF16 split products               */
    QS_PREC_BF16X6 = 4,  /* as above with 6-term BF16 split products (3-way split)  */
    QS_PREC_FP64_FFT = 5 /* FP64 everywhere, with the FFT transforms of the FP32 path
                            computed in FP64 (power-of-two ny, nz in [32, 1024]):
                            the reference's FFTW algorithm class on the GPU; with
                            CIC the plasma is grouped by cell as in FP32 and the
                            push uses FMA (not bit-identical to QS_PREC_FP64)    */
} qs_precision;

/* Plasma particle shape. */
typedef enum qs_shape {
    QS_SHAPE_NGP = 0,    /* reference live path: NGP gather at the particle's cell
                            from P and C averaged, NGP deposit, particles keep
                            their seeded cell (movepart_splitlayer.cpp:1101-1615) */
    QS_SHAPE_CIC = 1     /* bilinear gather / 4-point CIC deposit with the weights
                            of movepart_layer_CIC.cpp:165-193,449-496, particles
                            relinked to the cell they move into                  */
} qs_shape;

/* Transform kinds (FFTW r2r kinds used by the reference). */
typedef enum qs_dtt_kind {
    QS_REDFT11 = 0,      /* Y_k = 2 sum_j X_j cos(pi (j+1/2)(k+1/2) / n) */
    QS_RODFT11 = 1       /* Y_k = 2 sum_j X_j sin(pi (j+1/2)(k+1/2) / n) */
} qs_dtt_kind;

/* Layer planes (reference Cell members, cells.h:42-62). */
typedef enum qs_field {
    QS_F_EX = 0, QS_F_EY = 1, QS_F_EZ = 2,
    QS_F_BX = 3, QS_F_BY = 4, QS_F_BZ = 5,
    QS_F_JX = 6, QS_F_JY = 7, QS_F_JZ = 8,
    QS_F_DENS = 9,
    QS_F_RHOBEAM = 10, QS_F_JXBEAM = 11
} qs_field;

typedef enum qs_layer_sel {
    QS_LAYER_P = 0,      /* Mesh::p_CellLayerP, the previous (already solved) layer */
    QS_LAYER_C = 1       /* Mesh::p_CellLayerC, the layer being solved              */
} qs_layer_sel;

/*
 * Run configuration: the hot-path keys of the reference namelists
 * (Domain: domain.cpp:42-57; Specie: elements.cpp:11-67;
 *  Synchrotron: synchrotron.cpp:13).  Fill with qs_config_default() first.
 */
typedef struct qs_config {
    int32_t ny, nz, nx;         /* l_My, l_Mz, l_Mx                                  */
    int32_t nx_split;           /* NxSplit (default 1)                               */
    int32_t n_iter;             /* nIter   (default 1)                               */
    int32_t ppc;                /* P_perCell of the plasma electrons (default 4)     */
    double hx, hy, hz;          /* Hx, Hy, Hz                                        */
    double ts;                  /* Ts, the beam time step                            */
    double plasma_density;      /* Density of the uniform plasma electrons           */
    double plasma_q2m;          /* f_q2m of the plasma electrons (-1)                */
    double plasma_djx0, plasma_djy0, plasma_djz0, plasma_drho0; /* GetdJ (-1 each)   */
    double plasma_px0, plasma_py0, plasma_pz0;                  /* Px0, Py0, Pz0     */
    double pspread_x, pspread_y, pspread_z;  /* PspreadX/Y/Z (thermal sigma, m c)    */
    double bx_ext, by_ext, bz_ext;           /* BxExternal, ByExternal, BzExternal   */
    double beam_q2m;            /* q/m of the driver macro-particles (-1: electrons) */
    double beam_polarity;       /* charge sign used by the beam deposit (Polarity)   */
    double syn_min;             /* Synchrotron SynMin (gamma threshold, default 100) */
    double wavelength;          /* Domain Wavelength in cm (default 0.001)           */
    int32_t synchrotron;        /* 1: apply the radiation-reaction momentum loss     */
    int32_t precision;          /* qs_precision                                      */
    int32_t shape;              /* qs_shape                                          */
    int32_t device;             /* CUDA device ordinal                               */
    int32_t store_sources;      /* 1: also keep Dens/Jx/Jy/Jz of every layer         */
    int32_t use_graph;          /* 1: replay the march as one captured CUDA graph    */
    uint64_t seed;              /* seed of the front-layer thermal momenta           */
} qs_config;

typedef struct qs_handle qs_handle;

/* ---------------------------------------------------------------- lifecycle */

/* Reference defaults (Domain/Specie/Synchrotron namelist defaults) for a
 * 128x128x256 uniform-plasma deck with 4 ppc and cell 0.05. */
qs_status qs_config_default(qs_config* cfg);

/* Domain::Domain + Mesh::Mesh (domain.cpp:14-216, mesh.cpp:12-32) and the
 * lazy device allocations of the CUDA_WRAP plug-ins
 * (plasma_particles.cu:770-811, half_integer2D.cu:600-604). */
qs_status qs_create(const qs_config* cfg, qs_handle** out);
qs_status qs_destroy(qs_handle* h);

/* Text of the last error on this handle (or of the last failed qs_create on
 * this thread when h is NULL). */
const char* qs_last_error(const qs_handle* h);
const char* qs_status_string(qs_status s);

/* Synchronise the handle's stream and report any device-side error flag. */
qs_status qs_sync(qs_handle* h);
/* The handle's cudaStream_t, for callers that enqueue around the library. */
qs_status qs_get_stream(qs_handle* h, void** stream);

/* ------------------------------------------------------------- state in/out */

/* Driver beam macro-particles: cell (i = xi layer, j, k) and in-cell
 * fractions x,y,z in [0,1], momenta, weight.  Replaces the lattice seeding of
 * Mesh::SeedBeamParticles (mesh.cpp:108-234): the caller samples the beam. */
qs_status qs_load_beam(qs_handle* h, int64_t n,
                       const int32_t* i, const int32_t* j, const int32_t* k,
                       const double* x, const double* y, const double* z,
                       const double* px, const double* py, const double* pz,
                       const double* w);
qs_status qs_get_beam(qs_handle* h, int64_t n,
                      int32_t* i, int32_t* j, int32_t* k,
                      double* x, double* y, double* z,
                      double* px, double* py, double* pz, double* w);
int64_t qs_beam_count(const qs_handle* h);

/* Front-layer plasma (Mesh::SeedFrontParticles / SeedParticles,
 * mesh.cpp:98-106,413-548).  cell = j + ny*k; particles must be grouped by
 * cell in ascending cell order.  The arrays are used by the next march. */
qs_status qs_load_front_plasma(qs_handle* h, int64_t n, const int32_t* cell,
                               const double* y, const double* z,
                               const double* px, const double* py,
                               const double* pz, const double* w);
/* Seed the front layer on the device: ppc particles per cell on the
 * reference lattice (mesh.cpp:455-459), weight Density/ppc, momenta
 * P0 + N(0, Pspread) from a counter-based generator keyed by (seed, step). */
qs_status qs_seed_front_plasma(qs_handle* h, uint64_t step);
int64_t qs_plasma_count(const qs_handle* h);

/* Plasma density profile: Specie::Density (plasma.cpp:6-399) with the
 * namelist values of Specie (elements.cpp:11-58).  Coordinates as in the
 * reference: x from the left X boundary plus the phase (the distance the box
 * has moved), y and z from the axis.  distribution (i_Distribution):
 *   0 trapezoid, 1 Gaussian ellipsoid, 2 Gaussian channel, 3 curved Gaussian
 *   channel, 4 parallelepiped, 5 exponential, 6 empty channel, 7 COS-GAUSS,
 *   8 tanh step, 9 rod, 10 linear step, 11 gradient, 12 periodic. */
typedef struct qs_density_profile {
    int32_t distribution;
    int32_t reserved;                            /* 0                          */
    double density, density1;                    /* Density, Density1          */
    double begin, end, plateau_begin, plateau_end;
    double scale, delta;                         /* Scale, Delta               */
    double radius, radius_x, radius_y, radius_z;
    double x0, y0, z0;
    double xperiod, yperiod, zperiod;
    double angle_y;                              /* AngleY                     */
    double y_curvature, z_curvature;             /* Ycurvature, Zcurvature     */
    double curvature_begin, curvature_end;       /* CurvatureBegin/End         */
} qs_density_profile;

/* A uniform profile: distribution 0 with density 1 from x = 0 on. */
qs_status qs_density_profile_default(qs_density_profile* p);
/* Set the plasma profile (NULL: the uniform cfg.plasma_density again).  With
 * a profile, qs_seed_front_plasma gives the particles of cell (j, k) the
 * weight Density(x_front, y_j, z_k)/ppc at the front x = Hx*nx + phase
 * (mesh.cpp:413-431,471) and weight 0 where the density is not positive (the
 * reference seeds no particle there; a zero weight deposits exact zeros), and
 * the Guess/Iterate maps take |Density*q2m| on axis at the head layer
 * x = Hx*(nx-1) + phase (movefieldshydrolinlayersplit.cpp:236-250; 0 -> 1).
 * Distribution 12 needs xperiod > 0 (the reference loops forever otherwise). */
qs_status qs_set_density_profile(qs_handle* h, const qs_density_profile* p);
/* Specie::Density of the profile set on h at (x, y, z), evaluated on the host
 * (the uniform density when none is set). */
qs_status qs_plasma_density(qs_handle* h, double x, double y, double z, double* out);
/* Phase (Controls f_Phase): the distance the box has moved; qs_step adds Ts
 * before its beam push (step.cpp:33). */
qs_status qs_set_phase(qs_handle* h, double phase);
qs_status qs_get_phase(qs_handle* h, double* phase);

/* xi-pipeline hand-off in the reference's wire format (PackLayer /
 * UnpackLayer, para.cpp:94-285; LAYER_ATTRIBUTE_NUMBER = 12 and
 * BEAM_PARTICLE_ATTRIBUTE_NUMBER = 12, CUDA_WRAP/paraLayers.h:4-5): one
 * double buffer of 12 planes of ny*nz (n = j + ny*k) in the order Bx, By, Bz,
 * Ex, Ey, Ez, Jx, Jy, Jz, Rho, fftJxBeamHydro, fftRhoBeamHydro, then 12
 * blocks of Np particle attributes Px, Py, Pz, X, Y, Z, Q2m, Weight, i_X,
 * i_Y, i_Z, isort, particles cell by cell.  Size 12*ny*nz + 12*Np. */
int64_t qs_layer_pack_size(const qs_handle* h);
/* PackLayer + SendLayer's device read (para.cpp:94-150, 286-330): after a
 * march, the tail layer (layer 0: fields, the currents of its last push, the
 * corrected Rho, the beam spectra of its last split) and the plasma in
 * flight, particles cell by cell and in load order within a cell.  n must be
 * qs_layer_pack_size(h).  The buffer is assembled in device memory and copied
 * to buf once (synchronous on return); pinned host memory gives the full
 * copy rate. */
qs_status qs_pack_layer(qs_handle* h, double* buf, int64_t n);
/* ReceiveLayer + UnpackLayer + CUDA_WRAP_setLayerToMesh (para.cpp:332-412,
 * 175-285; paraCPUlayers.cu:178-297): the received layer becomes the front
 * (layer nx) of the next march, as below the first rank of the reference's
 * pipeline (movepart_splitlayer.cpp:105-151): its fields and sources are the
 * head layer's P, its beam spectra the head's RhoBeamP (:547-551), and its
 * particles the front plasma.  It serves that one march. */
qs_status qs_unpack_layer(qs_handle* h, const double* buf, int64_t n);
/* Drop a received layer that no march has used yet (empty front again). */
qs_status qs_clear_front_layer(qs_handle* h);
/* Plasma particles of the layer in flight (after a march: layer 0). */
qs_status qs_get_plasma(qs_handle* h, int64_t n, int32_t* cell,
                        double* y, double* z, double* px, double* py,
                        double* pz, double* w);

/* Transverse layers P / C (interior ny*nz, periodic guards implied). */
qs_status qs_set_layer(qs_handle* h, int which, int field, const double* data);
qs_status qs_get_layer(qs_handle* h, int which, int field, double* out);

/* 3-D per-layer storage (Mesh::p_CellArray): E, B of every layer (and
 * Dens/J when store_sources), beam currents RhoBeam/JxBeam. */
qs_status qs_get_field3d(qs_handle* h, int field, int layer, double* out);
qs_status qs_set_beam_currents(qs_handle* h, int field, int layer,
                               const double* data);
qs_status qs_get_beam_currents(qs_handle* h, int field, int layer, double* out);

/* On-axis longitudinal field: reference Ex at (My/2, Mz/2) of layers
 * 0..nx-1 of the field store (after the last march, or the layers a march
 * driven through the fine-grained entry points has finished so far). */
qs_status qs_get_onaxis_ex(qs_handle* h, double* out);
/* Wake potential psi(xi_i), a derived quantity the reference does not
 * compute: psi(nx) = 0, psi(i) = psi(i+1) + hx (Ex_i + Ex_{i+1})/2 on axis. */
qs_status qs_get_psi(qs_handle* h, double* out);

/* Layer output.  The reference writes HDF5 (Mesh::Save's field file,
 * save.cpp:520-838, vsNNN_3d_fields.h5; Mesh::SaveCadrMovie2's frames,
 * mesh.cpp:976-1090); HDF5 is not part of this library, so the same datasets
 * go into a plain self-describing file, QSF1 (little-endian):
 *   bytes 0-7   "QSF1" and four zero bytes
 *   int32 ndatasets, int32 0
 *   ndatasets entries of 72 bytes: char name[32] (zero padded), int32 dtype
 *   (1 int32, 2 float64), int32 rank, int64 dims[3] (fastest first, unused
 *   ones 1), int64 byte offset of the data in the file
 *   the data blocks (8-byte aligned)
 * qs_save_fields: "meshinfo" (16 int32: Mx, 0, Mx, 0, My, 0, My, 0, Mz, 0,
 * Mz, 0 and four zeros, the reference's l_Mx, l_dMx, l_sizeX, l_offsetX ...
 * without guard cells), "phase", the axes "X" (i hx + phase), "Y"
 * (j hy - Ylength/2), "Z", and the 3-D arrays "Ex" "Ey" "Ez" "Bx" "By" "Bz"
 * (and "Jx" "Jy" "Jz" "Dens" with store_sources = 1) of the field store, dims
 * (nx, ny, nz), the layer index fastest as in the reference's files.
 * qs_save_movie_frame: the same axes and, for each of those quantities, its
 * plane through the axis in (x, y) at z = nz/2 ("Ex_xy", dims (nx, ny)) and
 * in (x, z) at y = ny/2 ("Ex_xz", dims (nx, nz)).  Both are synchronous. */
qs_status qs_save_fields(qs_handle* h, const char* path);
qs_status qs_save_movie_frame(qs_handle* h, const char* path);

/* No counterpart in the reference (which has no such diagnostic; the planes
 * summed are those its Cell array stores).  FP64 global charge sums of every
 * layer of the last march, computed on the device in FP64 whatever the
 * precision of the march: the sum over the transverse plane of
 *   rho[nx]        the corrected density (the Cell's f_Dens after the layer's
 *                  last Iterate, movefieldshydrolinlayersplit.cpp:1545-1602),
 *   jx[nx]         the Jx deposit of the layer's full push,
 *   rho_beam[nx+1] RhoBeam of the beam-current store after the last beam push
 *                  (MoveBeamInCell, movebeam.cpp:662-774).
 * Any pointer may be NULL. */
qs_status qs_get_charge_sums(qs_handle* h, double* rho, double* jx, double* rho_beam);

/* No counterpart in the reference.  A self-test of the bounded device waits
 * (the waits of the tensor-core transform kernel give up after a fixed number
 * of tries, set QS_ERR_TIMEOUT's device flag, release what they hold and
 * return): one CTA waits, through the same wait routine, on a barrier that
 * nothing completes, for `tries` tries (1 .. 2^22).  Returns QS_ERR_TIMEOUT
 * when the limit and the error path work (the flag is then cleared and the
 * handle stays usable), an earlier pending error first. */
qs_status qs_selftest_wait_limit(qs_handle* h, unsigned tries);

/* --------------------------------------------------------------- the path */

/* Domain::Step (step.cpp:24-122): phase += Ts, beam push, xi-march. */
qs_status qs_step(qs_handle* h);
/* Mesh::MoveBeamParticles (movebeam.cpp:14-659) incl. MoveBeamInCell. */
qs_status qs_move_beam_particles(qs_handle* h);
/* Mesh::MoveAllSplitLayers (movepart_splitlayer.cpp:25-558). */
qs_status qs_move_all_split_layers(qs_handle* h);

/* Fine-grained pieces of the march, in the order MoveAllSplitLayers runs
 * them.  qs_begin_march: zero the 3-D currents and take the front layer
 * (movepart_splitlayer.cpp:38-63).  qs_layer_begin: P <- layer iLayer+1 on
 * iSplit 0 and the xi-interpolation of the beam currents into C
 * (:170-187, :330-348).  qs_layer_end: P <- C and, on the last split,
 * layer iLayer <- P (:423-428, :467-473). */
qs_status qs_begin_march(qs_handle* h);
qs_status qs_layer_begin(qs_handle* h, int iLayer, int iSplit);
/* Mesh::MoveSplitLayer (movepart_splitlayer.cpp:561-778). */
qs_status qs_move_split_layer(qs_handle* h, int iLayer, int iSplit);
/* Mesh::GuessFieldsHydroLinLayerSplit (movefieldshydrolinlayersplit.cpp:222)
 * = CUDA_WRAP_linearized_loop (linearized.h:4) + its transforms. */
qs_status qs_guess_fields(qs_handle* h, int iLayer, int iSplit);
/* Mesh::MoveParticlesLayerSplit (movepart_splitlayer.cpp:781) =
 * cuMoveSplitParticles (plasma_particles.h:15-16), deposit included. */
qs_status qs_move_particles_layer(qs_handle* h, int iLayer, int iSplit,
                                  int iFullStep);
/* Mesh::IterateFieldsHydroLinLayerSplit (movefieldshydrolinlayersplit.cpp:1173)
 * = CUDA_WRAP_linearizedIterateloop (linearized.h:27).  rel_err (may be NULL)
 * receives max(|dE|/max|E|) over Ex,Ey,Ez as the reference returns it. */
qs_status qs_iterate_fields(qs_handle* h, int iLayer, int iSplit, int iter,
                            double* rel_err);
qs_status qs_layer_end(qs_handle* h, int iLayer, int iSplit);

/* CUDA_WRAP_fourierHalfInteger2D (half_integer2D.h:8): batch of nz x ny
 * real planes, unnormalised FFTW REDFT11/RODFT11 along z (kind_z) and y
 * (kind_y), computed in the handle's precision mode.  Host pointers. */
qs_status qs_transform2d(qs_handle* h, int kind_z, int kind_y, int batch,
                         const double* in, double* out);
/* Same on device memory in the handle's real type (float, or double in
 * QS_PREC_FP64), enqueued on the handle's stream. */
qs_status qs_transform2d_dev(qs_handle* h, int kind_z, int kind_y, int batch,
                             const void* d_in, void* d_out);

/* No counterpart in the reference.  The FP64 transform of qs_transform2d_dev
 * for callers that cannot allocate device memory (a plugin that may only use
 * buffers its host framework's allocator hands it, so it cannot hold a
 * qs_handle, whose creation allocates).  No handle: it runs on the current
 * device, enqueued on `stream` (a cudaStream_t; NULL = legacy default stream),
 * and calls no cudaMalloc, cudaFree or other allocating routine.  d_in and
 * d_out are device arrays of batch nz x ny double planes.  Its only other
 * memory is a fixed 6 MiB scratch array inside the library's CUDA module,
 * which each GPU that loads the module holds until the process exits; it
 * limits ny and nz to 512 (each a multiple of 8): larger sizes return
 * QS_ERR_INVALID with the reason in qs_last_error(NULL).  The first call on a
 * device looks up the array's device address (again only after the device's
 * context has changed, e.g. after cudaDeviceReset), so make that first call
 * before any stream capture.  A CUDA error already pending on the calling
 * thread is reported as QS_ERR_CUDA and left in place; nothing is launched.
 * All calls on a device share the array: calls whose GPU work overlaps
 * (other streams, other host threads) race and must be ordered by the
 * caller. */
qs_status qs_transform2d_noalloc(int kind_z, int kind_y, int ny, int nz, int batch,
                                 const double* d_in, double* d_out, void* stream);

/* ------------------------------------------------------------ the adjoint
 *
 * Reverse-mode gradient of a loss on the on-axis longitudinal field with
 * respect to the driver-beam macro-particle weights (no counterpart in the
 * reference, which has no adjoint; the forward it differentiates is
 * Mesh::MoveAllSplitLayers, movepart_splitlayer.cpp:25-558, with the beam
 * currents deposited by the last beam push, movebeam.cpp:662-774).
 *
 * qs_adjoint_checkpoints(h, K): from the next march on, store the plasma
 * particles and the P-bank spectra every K layers (K = 0 turns it off and
 * frees the storage).  Call it after the front plasma is loaded or seeded.
 * Supported for the NGP and CIC shapes and NxSplit = 1. */
qs_status qs_adjoint_checkpoints(qs_handle* h, int every);
/* Given dloss_donaxis_ex[nx] = d loss / d (on-axis Ex of layer i) for the last
 * march (which must have stored checkpoints, with no beam change since),
 * recompute each K-layer segment from its checkpoint and sweep it in reverse;
 * writes dloss_dbeam_weight[n_beam] = d loss / d w_p for every beam particle
 * at its post-push position (particles outside the box get 0).  The sweep
 * starts at the lowest layer with a nonzero dloss entry.  It reuses the
 * march's working state: afterwards the plasma arrays are undefined and the
 * field store may differ from the march's in the last bits (atomic order). */
qs_status qs_adjoint(qs_handle* h, const double* dloss_donaxis_ex,
                     double* dloss_dbeam_weight);

/* One step through host buffers (the e2e entry point): copies the beam in
 * from host, seeds the front plasma, runs qs_step, copies the beam and the
 * on-axis Ex back.  Any out pointer may be NULL to skip that copy. */
qs_status qs_step_host(qs_handle* h, int64_t n_beam,
                       const int32_t* i, const int32_t* j, const int32_t* k,
                       const double* x, const double* y, const double* z,
                       const double* px, const double* py, const double* pz,
                       const double* w,
                       int32_t* i_out, int32_t* j_out, int32_t* k_out,
                       double* x_out, double* y_out, double* z_out,
                       double* px_out, double* py_out, double* pz_out,
                       double* onaxis_ex_out);

/* Number of kernel launches the library issued on this handle so far
 * (graph replays count their nodes). */
int64_t qs_kernel_launches(const qs_handle* h);

/* Per-kernel timing, the counterpart of the reference's stage timers
 * (timeBegin/timeEnd/timePrint, CUDA_WRAP/cuda_wrap_control.cu:74-116, and
 * GUESS_TIME_PRINT, movefieldshydrolinlayersplit.cpp:1159-1168).  While
 * enabled, the march runs launch by launch (no graph replay) with a CUDA event
 * pair around every kernel on the handle's stream. */
qs_status qs_profile_enable(qs_handle* h, int on);
/* Milliseconds and launch counts per kernel class since the last read:
 * 0 push/deposit, 1 transform GEMM, 2 transform operand split, 3 spectral
 * maps, 4 beam-current spectra, 5 beam push, 6 front seeding, 7 other,
 * 8 regrouping of the CIC plasma by cell.
 * Resets the counters. */
qs_status qs_profile_read(qs_handle* h, double* ms, int64_t* launches, int n);

#ifdef __cplusplus
}
#endif
#endif /* QSB200_H */
