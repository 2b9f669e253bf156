// api.cu — the C ABI of include/qsb200.h and the engine that runs the
// quasi-static xi-march on one GPU.
//
// Data layout in HBM (T = float, or double in QS_PREC_FP64):
//   f3   : (nx+1) layers x 6 planes (Ex,Ey,Ez,Bx,By,Bz)    Mesh::p_CellArray fields
//   b3   : (nx+1) layers x 2 planes (RhoBeam, JxBeam)      beam currents; after the
//          beam push's check and sums they are transformed in place into their
//          REDFT11 x REDFT11 spectra, which the march reads
//   src3 : (nx+1) layers x 4 planes (Jx,Jy,Jz,Dens)        only with store_sources
//   P / C layer fields alias f3 during the march: C of the last split of layer
//   i is f3[i] and P of layer i is f3[i+1], so the reference's copies
//   P <- Array[i+1], P <- C, Array[i] <- P (movepart_splitlayer.cpp:170-187,
//   423-428, 467-473) cost nothing.
//   Spectral state: two banks of 12 planes [Rho,Ex,Ey,Ez,Bx,By,Bz,Jx,Jy,Jz,
//   Rb,Jxb]; the bank of the previous (layer, split) is the P state
//   (RhoP, E*P, J*P, RhoBeamP), swapped at every layer end.
//   Plasma particles: SoA grouped by cell; beam particles: SoA, FP64.
// A plane is ny*nz values, index j + ny*k.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <new>
#include <string>
#include <vector>

#include "qs_common.cuh"
#include "qs_internal.h"
#include "dtt_tc.h"
#include "density.cuh"

namespace qs {

static thread_local std::string g_create_error;
thread_local bool g_pdl = false;

// error text of calls made without a handle (read by qs_last_error(NULL))
void set_unbound_error(const std::string& why) { g_create_error = why; }

struct EngineBase {
    qs_config cfg{};
    int My = 0, Mz = 0, L = 0, S = 1, nIter = 1;
    size_t plane = 0;
    int dev = 0;
    cudaStream_t st = nullptr;
    int* d_err = nullptr;
    std::string err;
    int64_t launches = 0;
    uint64_t step_count = 0;
    double phase = 0;
    // plasma density profile (Specie::Density); uniform cfg.plasma_density
    // when none is set
    bool have_profile = false;
    qs_density_profile profile{};
    bool capturing = false;
    int64_t capture_count = 0;
    // per-kernel timing (qs_profile_*): an event pair around every launch
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_next = 0;
    std::vector<std::pair<int, size_t>> prof_recs;
    double prof_ms[KC_N] = {};
    int64_t prof_n[KC_N] = {};
    virtual ~EngineBase() {
        for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
    }

    void count(int n) {
        if (capturing) capture_count += n;
        else launches += n;
    }
    cudaEvent_t ev_get() {
        if (ev_next == ev_pool.size()) {
            cudaEvent_t e = nullptr;
            cudaEventCreate(&e);
            ev_pool.push_back(e);
        }
        return ev_pool[ev_next++];
    }
    // launch through f() (returns the kernels it launched) as class cls
    template <class F>
    int klaunch(int cls, F&& f) {
        if (prof && !capturing) {
            const size_t i0 = ev_next;
            cudaEventRecord(ev_get(), st);
            const int n = f();
            cudaEventRecord(ev_get(), st);
            prof_recs.push_back({cls, i0});
            prof_n[cls] += n;
            count(n);
            return n;
        }
        const int n = f();
        count(n);
        return n;
    }
    qs_status resolve_profile() {
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "profile synchronize");
        for (auto& r : prof_recs) {
            float ms = 0.f;
            e = cudaEventElapsedTime(&ms, ev_pool[r.second], ev_pool[r.second + 1]);
            if (e != cudaSuccess) return cuda_fail(e, "profile event");
            prof_ms[r.first] += ms;
        }
        prof_recs.clear();
        ev_next = 0;
        return QS_OK;
    }

    qs_status fail(qs_status s, const char* fmt, ...) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        err = buf;
        return s;
    }
    qs_status cuda_fail(cudaError_t e, const char* what) {
        return fail(e == cudaErrorMemoryAllocation ? QS_ERR_OOM : QS_ERR_CUDA, "%s: %s", what,
                    cudaGetErrorString(e));
    }

    // Specie::Density of the plasma electrons at (x, y, z)
    double density_at(double x, double y, double z) const {
        if (!have_profile) return cfg.plasma_density;
        return profile_density(profile, x, y, z);
    }
    // the density of the Guess/Iterate maps: |Density*q2m| on axis at the
    // head layer i = l_Mx-1 (movefieldshydrolinlayersplit.cpp:236-250), 1 when 0
    double march_density() const {
        const int j = My / 2, k = Mz / 2;
        const double x = cfg.hx * (L - 1) + phase;
        const double y = cfg.hy * j - My * cfg.hy / 2.;
        const double z = cfg.hz * k - Mz * cfg.hz / 2.;
        double d = std::fabs(density_at(x, y, z) * cfg.plasma_q2m);
        if (d == 0.0) d = 1.0;
        return d;
    }

    virtual qs_status init() = 0;
    virtual qs_status load_beam(int64_t, const int32_t*, const int32_t*, const int32_t*,
                                const double*, const double*, const double*, const double*,
                                const double*, const double*, const double*) = 0;
    virtual qs_status get_beam(int64_t, int32_t*, int32_t*, int32_t*, double*, double*, double*,
                               double*, double*, double*, double*) = 0;
    virtual int64_t beam_count() const = 0;
    virtual qs_status load_front(int64_t, const int32_t*, const double*, const double*,
                                 const double*, const double*, const double*, const double*) = 0;
    virtual qs_status seed_front(uint64_t) = 0;
    virtual int64_t plasma_count() const = 0;
    virtual qs_status get_plasma(int64_t, int32_t*, double*, double*, double*, double*, double*,
                                 double*) = 0;
    virtual qs_status set_layer(int, int, const double*) = 0;
    virtual qs_status get_layer(int, int, double*) = 0;
    virtual qs_status get_field3d(int, int, double*) = 0;
    virtual qs_status set_beam_currents(int, int, const double*) = 0;
    virtual qs_status get_beam_currents(int, int, double*) = 0;
    virtual qs_status get_onaxis(double*) = 0;
    virtual qs_status move_beam() = 0;
    virtual qs_status march() = 0;
    virtual qs_status begin_march() = 0;
    virtual qs_status layer_begin(int, int) = 0;
    virtual qs_status move_split_layer(int, int) = 0;
    virtual qs_status guess(int, int) = 0;
    virtual qs_status push(int, int, int) = 0;
    virtual qs_status iterate(int, int, int, double*) = 0;
    virtual qs_status layer_end(int, int) = 0;
    virtual qs_status transform2d(int, int, int, const double*, double*) = 0;
    virtual qs_status transform2d_dev(int, int, int, const void*, void*) = 0;
    virtual qs_status adjoint_checkpoints(int) = 0;
    virtual qs_status adjoint(const double*, double*) = 0;
    virtual int64_t pack_size() const = 0;
    virtual qs_status pack_layer(double*, int64_t) = 0;
    virtual qs_status unpack_layer(const double*, int64_t) = 0;
    virtual qs_status clear_front_layer() = 0;
    virtual qs_status get_charge_sums(double*, double*, double*) = 0;
    virtual qs_status save_output(const char*, bool movie) = 0;

    qs_status check_device() {
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "stream synchronize");
        int h = 0;
        e = cudaMemcpy(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "error flag read");
        if (h) {
            cudaMemset(d_err, 0, sizeof(int));
            if (h & DEV_ERR_BEAM_CURRENT)
                return fail(QS_ERR_BEAM_CURRENT, "Too large beam current (|JxBeam| > 10)");
            if (h & DEV_ERR_RANGE)
                return fail(QS_ERR_PARTICLE_RANGE, "particle in-cell fraction outside [0,1]");
            if (h & DEV_ERR_TIMEOUT) return fail(QS_ERR_TIMEOUT, "bounded device wait gave up");
            if (h & DEV_ERR_INTERNAL)
                return fail(QS_ERR_DEVICE, "internal consistency check failed on the device "
                                           "(plasma regrouping)");
            return fail(QS_ERR_DEVICE, "device error flag 0x%x", h);
        }
        return QS_OK;
    }
};

#define CK(x)                                              \
    do {                                                   \
        cudaError_t e_ = (x);                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, #x);   \
    } while (0)

// transform kinds
constexpr int CC = QS_REDFT11, SS = QS_RODFT11;
// spectral bank planes
enum { SP_RHO = 0, SP_EX, SP_EY, SP_EZ, SP_BX, SP_BY, SP_BZ, SP_JX, SP_JY, SP_JZ, SP_RB, SP_JXB,
       SP_N };

template <class T>
struct Engine : EngineBase {
    bool tc = false;            // split-precision tensor-core transforms
    int tc_mode = 0;
    T* f3 = nullptr;
    T* b3 = nullptr;
    T* src3 = nullptr;
    T* splitbuf = nullptr;      // 2 x 6 planes (NxSplit > 1 and stand-alone use)
    T* srcbuf = nullptr;        // 2 x 4 planes (P and C sources)
    T* Pf = nullptr;
    T* Cf = nullptr;
    T* Psrc = nullptr;
    T* Csrc = nullptr;
    T* Cbeam = nullptr;         // 2 planes (C-layer beam currents, on request)
    T* sb3 = nullptr;           // the spectra of RhoBeam, JxBeam: b3 itself, transformed in place
    bool sb3_valid = false;
    bool b3_spec = false;       // b3 holds the spectra (else the real beam currents)
    bool in_march = false;      // inside MoveAllSplitLayers (skip output-only work)
    int cur_layer = -1, cur_split = 0;
    T* bank = nullptr;          // 2 x SP_N planes
    int cur = 0;                // bank index of the current (layer, split)
    bool p_valid = true;        // P-bank spectra match the P real planes
    T* scratch = nullptr;       // transform intermediate, 8 planes
    // Side streams of the march.  [0]: the last z-pass of a layer (its real
    // E, B, read by the next layer's pushes) runs beside the next layer's
    // predictor, which then writes its half-transformed E, B into scratch2;
    // [1]: the plasma regrouping after a full push runs beside the Iterate
    // and Guess that follow.  Every reader of their outputs joins first.
    cudaStream_t st_side[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork[2] = {nullptr, nullptr}, ev_join[2] = {nullptr, nullptr};
    bool side_pending[2] = {false, false};
    bool side_z = false, side_sort = false;   // set for one march
    T* scratch2 = nullptr;      // 6 planes
    // the layer whose predictor the previous layer's last corrector kernel
    // has already run (its E, B after the y-pass in scratch2), or -1
    int pred_next = -1;
    // next_avg: the fused predictor wrote the average of the layer's E, B and
    // the predicted ones; half_avg: the C layer holds that average after the
    // next Guess, so its first push gathers from C alone and does not wait for
    // the layer's last z-pass (side stream 0)
    bool next_avg = false, half_avg = false;
    int fuse_lo = 0;            // lowest layer of the march (or recomputed segment)
    // adjoint sweep: the predictor adjoint of a layer runs on side stream 0
    // beside the next layer's first field z-pass (which then uses scratch2)
    bool side_adj = false, adj_pred_pending = false;
    T* push_favg = nullptr;     // the next push writes its gathered fields here
    // The adjoint's store of the fields every push of the last march gathered,
    // (nIter + 1) x 6 planes per layer, kept when checkpoints are on and the
    // push is the grouped CIC one, for the fstore_n layers nearest the head
    // that fit in free device memory (all of them where they fit): the adjoint
    // recomputes a segment whose layers are all stored by its full pushes
    // alone, each gathering the stored fields (the march's pushes, bit for
    // bit), instead of by the whole march.  The adjoint sweeps from the head
    // down to the loss window, so the head layers are the ones it reads.
    // QS_ADJ_FIELDS=n stores at most n layers (0: no store).
    T* fstore = nullptr;
    int fstore_n = 0;
    long fstore_cap = getenv("QS_ADJ_FIELDS") ? atol(getenv("QS_ADJ_FIELDS")) : -1;
    const T* push_fields = nullptr;   // the next push gathers these planes alone
    T* mats = nullptr;          // transform matrices
    DttMats<T> my, mz;
    TcTransformer* tcx = nullptr;
    DttFft* fftx = nullptr;     // FP32 transforms through FFTs (power-of-two sizes)
    DttFft64* fftx64 = nullptr; // QS_PREC_FP64_FFT: the same FFTs in FP64
    T* onaxis_d = nullptr;
    T* dens_dev = nullptr;      // |Density*q2m| of the march in flight (spectral maps)
    double dens_set = -1.0;     // the value dens_dev holds (-1: none yet)
    T* stage = nullptr;         // conversion staging, 8 planes
    double* stage_d = nullptr;  // double staging, 8 planes
    // plasma
    int64_t np = 0, np_cap = 0;
    int32_t* pcell = nullptr;
    T *py = nullptr, *pz = nullptr, *ppx = nullptr, *ppy = nullptr, *ppz = nullptr, *pw = nullptr;
    bool front_pending = false;
    // xi-pipeline hand-off: a layer received from the rank ahead
    // (UnpackLayer, para.cpp:175-285) is the front (layer nx) of the next
    // march: its E, B in field-store layer nx, its sources and beam spectra here
    bool front_layer = false;
    bool front_used = false;    // a march has started from it (it serves one march)
    bool graph_front = false;   // the captured march was built with a received front
    T* front_src = nullptr;     // Jx, Jy, Jz, Rho of the received layer
    T* front_beam = nullptr;    // RhoBeam, JxBeam spectra of the received layer
    // CIC in FP32, and in FP64 on FFT transforms, keeps the plasma grouped by
    // cell (sort.cu): a second set of particle arrays for the regrouping
    // scatter, load-order ids, per-cell counts and offsets, and where the
    // grouping stands
    bool cic_sort = false;
    int32_t *acell = nullptr, *pid = nullptr, *apid = nullptr;
    T *ay = nullptr, *az = nullptr, *apx = nullptr, *apy = nullptr, *apz = nullptr, *aw = nullptr;
    int *cic_cnt = nullptr, *cic_loff = nullptr, *cic_bsum = nullptr, *cic_bpref = nullptr;
    unsigned* cic_ticket = nullptr;
    struct Grouping {
        bool grouped = true, off_valid = false, counted = false, flip = false;
        int since = 0;   // full pushes since the last regrouping
    } grp;
    // regroup after every cic_every-th full push (particles drift about 1% of
    // a cell per layer, so the push's global-memory fallback for the few that
    // left their row stays cheap in between); QS_CIC_REGROUP overrides
    int cic_every = getenv("QS_CIC_REGROUP") ? std::max(1, atoi(getenv("QS_CIC_REGROUP"))) : 2;
    // programmatic dependent launch inside the march (QS_PDL=0 turns it off)
    bool use_pdl = !(getenv("QS_PDL") && getenv("QS_PDL")[0] == '0');
    bool uniform_layout = false;   // particle p in cell p / ppc (lattice seeding)
    // beam
    int64_t nb = 0, nb_cap = 0;
    int32_t *bi = nullptr, *bj = nullptr, *bk = nullptr;
    double *bx = nullptr, *by = nullptr, *bz = nullptr, *bpx = nullptr, *bpy = nullptr,
           *bpz = nullptr, *bw = nullptr;
    // graph of the march
    cudaGraphExec_t gexec = nullptr;
    int64_t graph_kernels = 0;
    struct HostState { T *Pf, *Cf, *Psrc, *Csrc; int cur; Grouping grp; } graph_end{}, adj_end{};
    bool marched = false;
    bool tail_ready = false;    // layer 0 of a complete march is in place (qs_pack_layer)
    // adjoint: layer checkpoints of the last march and the reverse sweep's buffers
    int ck_every = 0;           // checkpoint every ck_every layers (0: off)
    bool ck_valid = false;      // the last march stored checkpoints for the current beam
    int ck_count = 0;
    T* ck = nullptr;            // ck_count x (5 np + 7 planes)
    T* seg = nullptr;           // ck_every x (5 np + (nIter+1) x 6 planes)
    T* lam = nullptr;           // adjoint work planes (see adjoint())
    T* lam_pm = nullptr;        // 3 x np momentum adjoint
    T* lam_sb = nullptr;        // layers lam_lo..nx x 2 planes: adjoint of the beam spectra, then
                                // (in place) of the real beam currents
    int lam_lo = -1;            // first layer lam_sb holds (the lowest one a sweep reaches)
    T* d_dloss = nullptr;       // nx: d loss / d on-axis Ex of each layer
    double* d_gradw = nullptr;  // nb: d loss / d beam weight
    // CIC adjoint: checkpointed cells and ids, the cells entering each layer of
    // a segment, the position adjoint, and the reorder between checkpoints
    bool cic_adj = false;
    bool adj_recompute = false;   // recomputing a segment: keep the particle order
    int32_t *ck_cell = nullptr, *ck_id = nullptr, *seg_cell = nullptr, *adj_inv = nullptr;
    T* lam_pos = nullptr;
    T* adj_tmp = nullptr;
    cudaGraphExec_t adj_exec = nullptr;   // captured sweep for the layers adj_lo .. head
    int adj_lo = -1;
    int64_t adj_graph_nb = -1;
    int64_t adj_kernels = 0;
    int64_t adj_np = 0, adj_nb = 0;

    // FP64 charge sums (charge.cuh): weight tables c_k(ny), c_k(nz), the
    // partial sums of the correctors (L x q_nparts x 2) and of the beam check
    // ((L+1) x kBeamSumParts x 2), and the sums (L x 2 plasma, (L+1) x 2 beam)
    double *q_cy = nullptr, *q_cz = nullptr, *q_part = nullptr, *qb_part = nullptr;
    double* q_sums = nullptr;
    int q_nparts = 0;

    // FP32 attribution study of the FP64 engine (bitmask QS_FP32_STUDY, read
    // at creation): one part of the march computed or stored in FP32 and the
    // rest in FP64, to measure what each FP32 quantity adds to the error of
    // the FP32 march
    //    1  every transform through the FP32 FFT kernels
    //    2  the spectral state carried from layer to layer (and the beam
    //       spectra) rounded to float after each map
    //    4  the plasma push and deposit through the FP32 push kernel (float
    //       particle state, float fields and deposit)
    //    8  the real field planes of each layer rounded to float
    //   16  the beam currents rounded to float after the beam deposit
    //   32  the front plasma (positions, momenta, weights) rounded to float
    //       when it is seeded or loaded: the FP32 path's starting state
    //   64  the plasma state rounded to float after every full push (its
    //       storage in FP32, the push arithmetic in FP64)
    //  128  the push through the FP32 push kernel as with 4, but the FP64
    //       state takes the push's increments (its arithmetic in FP32, its
    //       storage in FP64)
    //  256  as 64 for the in-cell positions only
    //  512  as 64 for the momenta only
    int fp32_study = 0;
    DttFft* study_fft = nullptr;
    float* study_f = nullptr;   // 40 planes: transform in / out / scratch, P and C fields, deposit
    float* study_p = nullptr;   // 11 x np_cap: 6 particle values, 5 of them before the push

    // the hand-off buffer assembled on the device, and its ordering scratch
    double* d_pack = nullptr;
    int* d_pack_i = nullptr;
    size_t pack_cap = 0, pack_icap = 0;

    T* bankp(int b, int p) { return bank + ((size_t)b * SP_N + p) * plane; }
    T* f3layer(int i) { return f3 + (size_t)i * 6 * plane; }

    ~Engine() override {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (adj_exec) cudaGraphExecDestroy(adj_exec);
        delete tcx;
        delete fftx;
        delete fftx64;
        delete study_fft;
        void* ptrs[] = {f3, b3, src3, splitbuf, srcbuf, Cbeam, bank, scratch, mats, onaxis_d,
                        stage, stage_d, pcell, py, pz, ppx, ppy, ppz, pw, bi, bj, bk, bx, by, bz,
                        bpx, bpy, bpz, bw, d_err, dens_dev, front_src, front_beam, ck, seg, lam, lam_pm, lam_sb,
                        d_dloss, d_gradw, acell, pid, apid, ay, az, apx, apy, apz, aw, cic_cnt,
                        cic_loff, cic_bsum, cic_bpref, cic_ticket, ck_cell, ck_id, seg_cell,
                        adj_inv, lam_pos, adj_tmp, d_pack, d_pack_i, q_cy, q_cz, q_part,
                        qb_part, q_sums, study_f, study_p, scratch2, fstore};
        for (void* p : ptrs)
            if (p) cudaFree(p);
        for (int k = 0; k < 2; k++) {
            if (ev_fork[k]) cudaEventDestroy(ev_fork[k]);
            if (ev_join[k]) cudaEventDestroy(ev_join[k]);
            if (st_side[k]) cudaStreamDestroy(st_side[k]);
        }
        if (st) cudaStreamDestroy(st);
    }

    template <class U>
    qs_status alloc(U** p, size_t n, const char* what) {
        cudaError_t e = cudaMalloc((void**)p, n * sizeof(U) + 16);
        if (e != cudaSuccess) return cuda_fail(e, what);
        return QS_OK;
    }

    qs_status init() override {
        plane = (size_t)My * Mz;
        CK(cudaSetDevice(dev));
        // the march's chain runs at the highest stream priority and its side
        // work (the last z-pass of a layer, the plasma regrouping) at the
        // lowest, so that the CTA scheduler gives free SM slots to the chain
        int prio_lo = 0, prio_hi = 0;
        CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
        CK(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio_hi));
        for (int k = 0; k < 2; k++) {
            CK(cudaStreamCreateWithPriority(&st_side[k], cudaStreamNonBlocking, prio_lo));
            CK(cudaEventCreateWithFlags(&ev_fork[k], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ev_join[k], cudaEventDisableTiming));
        }
        qs_status s;
        if ((s = alloc(&d_err, 1, "error flag"))) return s;
        CK(cudaMemset(d_err, 0, sizeof(int)));
        if ((s = alloc(&f3, (size_t)(L + 1) * 6 * plane, "field store"))) return s;
        CK(cudaMemset(f3, 0, (size_t)(L + 1) * 6 * plane * sizeof(T)));
        if ((s = alloc(&b3, (size_t)(L + 1) * 2 * plane, "beam current store"))) return s;
        CK(cudaMemset(b3, 0, (size_t)(L + 1) * 2 * plane * sizeof(T)));
        if (cfg.store_sources) {
            if ((s = alloc(&src3, (size_t)(L + 1) * 4 * plane, "source store"))) return s;
            CK(cudaMemset(src3, 0, (size_t)(L + 1) * 4 * plane * sizeof(T)));
        }
        if ((s = alloc(&splitbuf, 12 * plane, "split layers"))) return s;
        CK(cudaMemset(splitbuf, 0, 12 * plane * sizeof(T)));
        if ((s = alloc(&srcbuf, 8 * plane, "source layers"))) return s;
        CK(cudaMemset(srcbuf, 0, 8 * plane * sizeof(T)));
        if ((s = alloc(&Cbeam, 2 * plane, "beam layer"))) return s;
        CK(cudaMemset(Cbeam, 0, 2 * plane * sizeof(T)));
        cic_sort = cfg.shape == QS_SHAPE_CIC &&
                   (sizeof(T) == 4 || cfg.precision == QS_PREC_FP64_FFT) && My % 32 == 0 &&
                   Mz % 4 == 0;
        if (cic_sort) {
            const int nb_scan = scan_blocks_count((int)plane);
            if ((s = alloc(&cic_cnt, plane, "cell counts"))) return s;
            if ((s = alloc(&cic_loff, plane, "cell offsets"))) return s;
            if ((s = alloc(&cic_bsum, (size_t)nb_scan, "cell offsets"))) return s;
            if ((s = alloc(&cic_bpref, (size_t)nb_scan + 1, "cell offsets"))) return s;
            if ((s = alloc(&cic_ticket, 1, "cell offsets"))) return s;
            CK(cudaMemset(cic_cnt, 0, plane * sizeof(int)));
            CK(cudaMemset(cic_ticket, 0, sizeof(unsigned)));
        }
        sb3 = b3;   // zero currents have zero spectra
        b3_spec = true;
        sb3_valid = true;
        if ((s = alloc(&bank, 2 * SP_N * plane, "spectral banks"))) return s;
        CK(cudaMemset(bank, 0, 2 * SP_N * plane * sizeof(T)));
        if ((s = alloc(&scratch, 8 * plane, "transform scratch"))) return s;
        if ((s = alloc(&stage, 8 * plane, "staging"))) return s;
        if ((s = alloc(&stage_d, 8 * plane, "staging"))) return s;
        if ((s = alloc(&onaxis_d, (size_t)L, "on-axis"))) return s;
        CK(cudaMemset(onaxis_d, 0, L * sizeof(T)));
        if ((s = alloc(&dens_dev, 1, "density"))) return s;
        if ((s = set_march_density())) return s;
        // charge sums: one partial per corrector block (the largest grid of
        // the corrector kernels: one block per z-mode row, 256 modes per block,
        // or 256 mode pairs per row)
        q_nparts = std::max(Mz, std::max((int)((plane + 255) / 256), ((My / 2 + 127) / 128) * Mz));
        if ((s = alloc(&q_part, (size_t)L * 2 * q_nparts, "charge sums"))) return s;
        CK(cudaMemset(q_part, 0, (size_t)L * 2 * q_nparts * sizeof(double)));
        if ((s = alloc(&qb_part, (size_t)(L + 1) * 2 * kBeamSumParts, "charge sums"))) return s;
        CK(cudaMemset(qb_part, 0, (size_t)(L + 1) * 2 * kBeamSumParts * sizeof(double)));
        if ((s = alloc(&q_sums, (size_t)2 * L + 2 * (L + 1), "charge sums"))) return s;
        CK(cudaMemset(q_sums, 0, ((size_t)2 * L + 2 * (L + 1)) * sizeof(double)));
        {
            // c_k(N) = (-1)^k / sin(pi (2k+1) / (4N)): the plane sum of the
            // inverse REDFT11 basis function k
            std::vector<double> cy(My), cz(Mz);
            auto fillc = [](std::vector<double>& c, int N) {
                for (int k = 0; k < N; k++)
                    c[k] = (k % 2 ? -1.0 : 1.0) / std::sin(M_PI * (2.0 * k + 1.0) / (4.0 * N));
            };
            fillc(cy, My);
            fillc(cz, Mz);
            if ((s = alloc(&q_cy, (size_t)My, "charge sums"))) return s;
            if ((s = alloc(&q_cz, (size_t)Mz, "charge sums"))) return s;
            CK(cudaMemcpy(q_cy, cy.data(), My * sizeof(double), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(q_cz, cz.data(), Mz * sizeof(double), cudaMemcpyHostToDevice));
        }
        // transform matrices 2 cos / 2 sin (pi (j+1/2)(k+1/2)/n); the angle is
        // reduced exactly in integers: (2j+1)(2k+1) mod 8n in units of pi/(4n)
        const size_t ny2 = (size_t)My * My, nz2 = (size_t)Mz * Mz;
        if ((s = alloc(&mats, 2 * ny2 + 2 * nz2, "transform matrices"))) return s;
        std::vector<T> hm(2 * ny2 + 2 * nz2);
        auto fill = [&](T* out, int n, int kind) {
            for (int k = 0; k < n; k++)
                for (int j = 0; j < n; j++) {
                    long long q = ((long long)(2 * j + 1) * (2 * k + 1)) % (8LL * n);
                    double a = M_PI * (double)q / (4.0 * n);
                    out[(size_t)k * n + j] = (T)(2.0 * (kind == CC ? std::cos(a) : std::sin(a)));
                }
        };
        fill(hm.data(), My, CC);
        fill(hm.data() + ny2, My, SS);
        fill(hm.data() + 2 * ny2, Mz, CC);
        fill(hm.data() + 2 * ny2 + nz2, Mz, SS);
        CK(cudaMemcpy(mats, hm.data(), hm.size() * sizeof(T), cudaMemcpyHostToDevice));
        my.m[CC] = mats;
        my.m[SS] = mats + ny2;
        mz.m[CC] = mats + 2 * ny2;
        mz.m[SS] = mats + 2 * ny2 + nz2;
        if (tc) {
            std::string msg;
            tcx = TcTransformer::create(tc_mode, My, Mz, d_err, msg);
            if (!tcx) return fail(QS_ERR_UNSUPPORTED, "tensor-core transform: %s", msg.c_str());
        } else if (sizeof(T) == 4) {
            fftx = DttFft::create(My, Mz);   // other sizes keep the FP32 matrix passes
            CK(cudaGetLastError());
            if (fftx && (s = alloc(&scratch2, 6 * plane, "transform scratch"))) return s;
        } else if (cfg.precision == QS_PREC_FP64_FFT) {
            fftx64 = DttFft64::create(My, Mz);
            CK(cudaGetLastError());
            if (!fftx64)
                return fail(QS_ERR_UNSUPPORTED, "FP64 FFT transforms need power-of-two ny, nz "
                                                "in [32, 1024]");
            if ((s = alloc(&scratch2, 6 * plane, "transform scratch"))) return s;
        }
        if (sizeof(T) == 8 && getenv("QS_FP32_STUDY")) {
            fp32_study = atoi(getenv("QS_FP32_STUDY")) & 1023;
            if (fp32_study & 1) {
                study_fft = DttFft::create(My, Mz);
                CK(cudaGetLastError());
                if (!study_fft)
                    return fail(QS_ERR_UNSUPPORTED, "FP32 study: the FFT transforms need "
                                                    "power-of-two ny, nz in [32, 2048]");
            }
            if ((s = alloc(&study_f, 40 * plane, "FP32 study"))) return s;
        }
        Pf = splitbuf;
        Cf = splitbuf + 6 * plane;
        Psrc = srcbuf;
        Csrc = srcbuf + 4 * plane;
        cur = 0;
        CK(cudaStreamSynchronize(st));
        return QS_OK;
    }

    // ------------------------------------------- the FP32 attribution study
    // the job's transforms through the FP32 FFT kernels: inputs rounded to
    // float, outputs widened back
    void study_xform(const DttJob<T>& job) {
        if constexpr (sizeof(T) == 8) {
            float* fin = study_f;
            float* fout = study_f + 8 * plane;
            float* fscr = study_f + 16 * plane;
            DttJob<float> jf;
            jf.nf = job.nf;
            jf.scale = (float)job.scale;
            for (int f = 0; f < job.nf; f++) {
                klaunch(KC_MISC, [&] {
                    return launch_convert<float>(job.in[f], 1, fin + (size_t)f * plane, plane, st);
                });
                jf.in[f] = fin + (size_t)f * plane;
                jf.out[f] = fout + (size_t)f * plane;
                jf.kz[f] = job.kz[f];
                jf.ky[f] = job.ky[f];
            }
            for (int pass = 0; pass < 2; pass++)
                klaunch(KC_GEMM, [&] { return study_fft->run_pass(pass, jf, fscr, st); });
            for (int f = 0; f < job.nf; f++)
                klaunch(KC_MISC, [&] {
                    return launch_convert_back<float>(fout + (size_t)f * plane, job.out[f], plane,
                                                      st);
                });
        }
    }
    // the plasma arrays (with the weights when `weights`) rounded to float:
    // positions and momenta, or with bit 256 / 512 the positions / momenta only
    void study_round_plasma(int bit, bool weights) {
        T* arr[6] = {py, pz, ppx, ppy, ppz, pw};
        for (int c = 0; c < (weights ? 6 : 5); c++) {
            study_round(arr[c], (size_t)np, bit);
            if (bit == 64) study_round(arr[c], (size_t)np, c < 2 ? 256 : (c < 5 ? 512 : 0));
        }
    }
    void study_round(T* x, size_t n, int bit) {
        if constexpr (sizeof(T) == 8) {
            if (fp32_study & bit) klaunch(KC_MISC, [&] { return launch_round_f32(x, n, st); });
        }
    }
    // the push through the FP32 kernel on float copies of the particles and
    // the P, C fields; its deposit is added to the double C sources
    qs_status study_push(int full) {
        if constexpr (sizeof(T) == 8) {
            if (!clear_by_maps()) CK(cudaMemsetAsync(Csrc, 0, 4 * plane * sizeof(T), st));
            if (!np) return QS_OK;
            float* fP = study_f + 24 * plane;
            float* fC = fP + 6 * plane;
            float* fdep = fC + 6 * plane;
            klaunch(KC_MISC, [&] { return launch_convert<float>(Pf, 1, fP, 6 * plane, st); });
            klaunch(KC_MISC, [&] { return launch_convert<float>(Cf, 1, fC, 6 * plane, st); });
            CK(cudaMemsetAsync(fdep, 0, 4 * plane * sizeof(float), st));
            T* dsrc[6] = {py, pz, ppx, ppy, ppz, pw};
            float* fp[6];
            for (int c = 0; c < 6; c++) {
                fp[c] = study_p + (size_t)c * np_cap;
                klaunch(KC_MISC, [&] { return launch_convert<float>(dsrc[c], 1, fp[c], np, st); });
            }
            PushArgs<float> a{};
            a.n = np;
            a.My = My; a.Mz = Mz;
            a.cell = pcell;
            a.y = fp[0]; a.z = fp[1]; a.px = fp[2]; a.py = fp[3]; a.pz = fp[4]; a.w = fp[5];
            a.P = fP; a.C = fC; a.dep = fdep;
            a.cell_out = pcell;
            a.dep_cell = nullptr;
            a.plane = plane;
            a.hx = (float)(cfg.hx / S); a.hy = (float)cfg.hy; a.hz = (float)cfg.hz;
            a.q2m = (float)cfg.plasma_q2m;
            a.djx0 = (float)cfg.plasma_djx0; a.djy0 = (float)cfg.plasma_djy0;
            a.djz0 = (float)cfg.plasma_djz0; a.drho0 = (float)cfg.plasma_drho0;
            a.bxe = (float)cfg.bx_ext; a.bye = (float)cfg.by_ext; a.bze = (float)cfg.bz_ext;
            a.sE = (float)(cfg.plasma_q2m * (cfg.hx / S) / 2.0);
            a.hxhy = (float)((cfg.hx / S) / cfg.hy);
            a.hxhz = (float)((cfg.hx / S) / cfg.hz);
            a.invMy = 1.0f / (float)My;
            a.full = full;
            a.err = d_err;
            float* before = study_p + 6 * (size_t)np_cap;   // the float state before the push
            if ((fp32_study & 128) && full)
                CK(cudaMemcpyAsync(before, study_p, 5 * (size_t)np_cap * sizeof(float),
                                   cudaMemcpyDeviceToDevice, st));
            klaunch(KC_PUSH, [&] { return launch_push<float>(a, cfg.shape, true, st); });
            klaunch(KC_MISC, [&] { return launch_add_widened(Csrc, fdep, 4 * plane, st); });
            if (full)
                for (int c = 0; c < 5; c++) {
                    if (fp32_study & 128)   // the FP64 state takes the increment
                        klaunch(KC_MISC, [&] {
                            return launch_add_increment(dsrc[c], fp[c], before + (size_t)c * np_cap,
                                                        np, c < 2, st);
                        });
                    else
                        klaunch(KC_MISC, [&] {
                            return launch_convert_back<float>(fp[c], dsrc[c], np, st);
                        });
                }
            CK(cudaGetLastError());
        }
        return QS_OK;
    }

    // ---------------------------------------------------------- transforms
    void xform(const DttJob<T>& job, T* work = nullptr) {
        if (!work) work = scratch;
        if (fp32_study & 1) {
            study_xform(job);
            return;
        }
        if (tc) {
            for (int stage = 0; stage < 3; stage++)
                klaunch(stage == 0 ? KC_SPLIT : KC_GEMM, [&] {
                    return tcx->run_stage(stage, job.nf, (const void* const*)job.in,
                                          (void* const*)job.out, job.kz, job.ky,
                                          (double)job.scale, st);
                });
        } else if (fftx) {
            if constexpr (sizeof(T) == 4)
                for (int pass = 0; pass < 2; pass++)
                    klaunch(KC_GEMM, [&] { return fftx->run_pass(pass, job, work, st); });
        } else if (fftx64) {
            if constexpr (sizeof(T) == 8)
                for (int pass = 0; pass < 2; pass++)
                    klaunch(KC_GEMM, [&] { return fftx64->run_pass(pass, job, work, st); });
        } else {
            for (int pass = 0; pass < 2; pass++)
                klaunch(KC_GEMM, [&] {
                    return run_dtt_simt_pass<T>(pass, job, My, Mz, my, mz, work, st);
                });
        }
    }

    DttJob<T> job_stack(const T* in_stack, int nf, T* const* outs, const int* kz, const int* ky,
                        T scale) {
        DttJob<T> j;
        j.nf = nf;
        for (int f = 0; f < nf; f++) {
            j.in[f] = in_stack + (size_t)f * plane;
            j.out[f] = outs[f];
            j.kz[f] = kz[f];
            j.ky[f] = ky[f];
        }
        j.scale = scale;
        return j;
    }

    T inv_scale() const { return (T)(1.0 / (4.0 * (double)My * (double)Mz)); }

    // ------------------------------------------------------------ particles
    PlasmaSet<T> cur_set() { return PlasmaSet<T>{pcell, py, pz, ppx, ppy, ppz, pw, pid}; }
    PlasmaSet<T> alt_set() { return PlasmaSet<T>{acell, ay, az, apx, apy, apz, aw, apid}; }
    void swap_sets() {
        std::swap(pcell, acell); std::swap(py, ay); std::swap(pz, az); std::swap(ppx, apx);
        std::swap(ppy, apy); std::swap(ppz, apz); std::swap(pw, aw); std::swap(pid, apid);
        grp.flip = !grp.flip;
    }
    // a fresh front layer: grouped by cell in load order, counts cleared
    qs_status cic_fresh_front() {
        if (!cic_sort || !np) return QS_OK;
        klaunch(KC_MISC, [&] { return launch_iota(pid, np, st); });
        CK(cudaMemsetAsync(cic_cnt, 0, plane * sizeof(int), st));
        grp.grouped = true;
        grp.off_valid = false;
        grp.counted = false;
        grp.since = 0;
        return QS_OK;
    }
    // make the cell offsets valid for the arrays the next push reads:
    // regroup after a full push, or count and scan a freshly loaded layer
    qs_status cic_prepare() {
        const int ncell = (int)plane;
        if (!grp.grouped) {
            klaunch(KC_SORT, [&] {
                return launch_cell_offsets(cic_cnt, ncell, cic_loff, cic_bsum, cic_bpref, cic_ticket, 0,
                                           st);
            });
            klaunch(KC_SORT, [&] {
                return launch_scatter<T>(cur_set(), alt_set(), np, ncell, cic_cnt, cic_loff,
                                         cic_bpref, d_err, st);
            });
            swap_sets();
            // the scatter rebuilt the arrays in cell order: the offsets hold
            grp.grouped = true;
            grp.off_valid = true;
            grp.counted = false;
        } else if (!grp.off_valid) {
            if (!grp.counted)
                klaunch(KC_SORT, [&] {
                    return launch_count_cells(pcell, np, ncell, cic_cnt, d_err, st);
                });
            klaunch(KC_SORT, [&] {
                return launch_cell_offsets(cic_cnt, ncell, cic_loff, cic_bsum, cic_bpref, cic_ticket, 1,
                                           st);
            });
            grp.off_valid = true;
            grp.counted = false;
        }
        CK(cudaGetLastError());
        return QS_OK;
    }

    qs_status ensure_plasma(int64_t n) {
        if (n <= np_cap) return QS_OK;
        if (grp.flip) swap_sets();
        void* old[] = {pcell, py, pz, ppx, ppy, ppz, pw, acell, ay, az, apx, apy, apz, aw, pid,
                       apid};
        for (void* p : old)
            if (p) cudaFree(p);
        acell = pid = apid = nullptr;
        ay = az = apx = apy = apz = aw = nullptr;
        qs_status s;
        if ((s = alloc(&pcell, n, "plasma"))) return s;
        if ((s = alloc(&py, n, "plasma"))) return s;
        if ((s = alloc(&pz, n, "plasma"))) return s;
        if ((s = alloc(&ppx, n, "plasma"))) return s;
        if ((s = alloc(&ppy, n, "plasma"))) return s;
        if ((s = alloc(&ppz, n, "plasma"))) return s;
        if ((s = alloc(&pw, n, "plasma"))) return s;
        if (cic_sort) {
            if ((s = alloc(&acell, n, "plasma"))) return s;
            if ((s = alloc(&ay, n, "plasma"))) return s;
            if ((s = alloc(&az, n, "plasma"))) return s;
            if ((s = alloc(&apx, n, "plasma"))) return s;
            if ((s = alloc(&apy, n, "plasma"))) return s;
            if ((s = alloc(&apz, n, "plasma"))) return s;
            if ((s = alloc(&aw, n, "plasma"))) return s;
            if ((s = alloc(&pid, n, "plasma"))) return s;
            if ((s = alloc(&apid, n, "plasma"))) return s;
        }
        if (fp32_study & (4 | 128)) {
            if (study_p) cudaFree(study_p);
            study_p = nullptr;
            if ((s = alloc(&study_p, 11 * (size_t)n, "FP32 study"))) return s;
        }
        np_cap = n;
        if (gexec) {  // the captured march baked the old pointers
            cudaGraphExecDestroy(gexec);
            gexec = nullptr;
        }
        drop_adjoint_graph();
        return QS_OK;
    }

    void drop_adjoint_graph() {
        if (adj_exec) cudaGraphExecDestroy(adj_exec);
        adj_exec = nullptr;
        adj_lo = -1;
    }

    qs_status ensure_beam(int64_t n) {
        if (n <= nb_cap) return QS_OK;
        void* old[] = {bi, bj, bk, bx, by, bz, bpx, bpy, bpz, bw};
        for (void* p : old)
            if (p) cudaFree(p);
        qs_status s;
        if ((s = alloc(&bi, n, "beam"))) return s;
        if ((s = alloc(&bj, n, "beam"))) return s;
        if ((s = alloc(&bk, n, "beam"))) return s;
        if ((s = alloc(&bx, n, "beam"))) return s;
        if ((s = alloc(&by, n, "beam"))) return s;
        if ((s = alloc(&bz, n, "beam"))) return s;
        if ((s = alloc(&bpx, n, "beam"))) return s;
        if ((s = alloc(&bpy, n, "beam"))) return s;
        if ((s = alloc(&bpz, n, "beam"))) return s;
        if ((s = alloc(&bw, n, "beam"))) return s;
        nb_cap = n;
        drop_adjoint_graph();   // it baked the old beam arrays
        return QS_OK;
    }

    qs_status load_beam(int64_t n, const int32_t* i, const int32_t* j, const int32_t* k,
                        const double* x, const double* y, const double* z, const double* px,
                        const double* py_, const double* pz_, const double* w) override {
        if (n < 0 || (n > 0 && (!i || !j || !k || !x || !y || !z || !px || !py_ || !pz_ || !w)))
            return fail(QS_ERR_INVALID, "qs_load_beam: bad arguments");
        qs_status s = ensure_beam(n);
        if (s) return s;
        nb = n;
        if (!n) return QS_OK;
        CK(cudaMemcpyAsync(bi, i, n * 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(bj, j, n * 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(bk, k, n * 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(bx, x, n * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(by, y, n * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(bz, z, n * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(bpx, px, n * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(bpy, py_, n * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(bpz, pz_, n * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(bw, w, n * 8, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        return QS_OK;
    }

    qs_status get_beam(int64_t n, int32_t* i, int32_t* j, int32_t* k, double* x, double* y,
                       double* z, double* px, double* py_, double* pz_, double* w) override {
        if (n != nb) return fail(QS_ERR_INVALID, "qs_get_beam: n=%lld, beam has %lld",
                                 (long long)n, (long long)nb);
        if (!n) return QS_OK;
        struct { void* h; const void* d; size_t sz; } c[] = {
            {i, bi, 4}, {j, bj, 4}, {k, bk, 4}, {x, bx, 8}, {y, by, 8}, {z, bz, 8},
            {px, bpx, 8}, {py_, bpy, 8}, {pz_, bpz, 8}, {w, bw, 8}};
        for (auto& e : c)
            if (e.h) CK(cudaMemcpyAsync(e.h, e.d, n * e.sz, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return QS_OK;
    }
    int64_t beam_count() const override { return nb; }

    qs_status load_front(int64_t n, const int32_t* cell, const double* y, const double* z,
                         const double* px, const double* py_, const double* pz_,
                         const double* w) override {
        if (n < 0 || (n > 0 && (!cell || !y || !z || !px || !py_ || !pz_ || !w)))
            return fail(QS_ERR_INVALID, "qs_load_front_plasma: bad arguments");
        int32_t prev = -1;
        for (int64_t p = 0; p < n; p++) {
            if (cell[p] < 0 || (size_t)cell[p] >= plane || cell[p] < prev)
                return fail(QS_ERR_INVALID, "qs_load_front_plasma: cells must be grouped in "
                                            "ascending order within [0, ny*nz)");
            prev = cell[p];
        }
        qs_status s = ensure_plasma(n);
        if (s) return s;
        if (grp.flip) swap_sets();   // the march graph starts from the first set
        np = n;
        uniform_layout = (n == (int64_t)plane * cfg.ppc);
        for (int64_t p = 0; p < n && uniform_layout; p++)
            if (cell[p] != (int32_t)(p / cfg.ppc)) uniform_layout = false;
        if (n) {
            CK(cudaMemcpyAsync(pcell, cell, n * 4, cudaMemcpyHostToDevice, st));
            const double* src[6] = {y, z, px, py_, pz_, w};
            T* dst[6] = {py, pz, ppx, ppy, ppz, pw};
            for (int c = 0; c < 6; c++) {
                // stage through stage_d in chunks of 8 planes
                size_t chunk = 8 * plane;
                for (int64_t o = 0; o < n; o += (int64_t)chunk) {
                    size_t m = (size_t)std::min<int64_t>((int64_t)chunk, n - o);
                    CK(cudaMemcpyAsync(stage_d, src[c] + o, m * 8, cudaMemcpyHostToDevice, st));
                    klaunch(KC_MISC, [&] { return launch_convert<T>(stage_d, 1, dst[c] + o, m, st); });
                }
            }
            CK(cudaStreamSynchronize(st));
        }
        study_round_plasma(32, true);
        if ((s = cic_fresh_front())) return s;
        front_pending = true;
        return QS_OK;
    }

    qs_status seed_front(uint64_t step) override {
        const int ppc = cfg.ppc;
        if (ppc < 1 || ppc > 16) return fail(QS_ERR_INVALID, "ppc must be in [1,16]");
        qs_status s = ensure_plasma((int64_t)plane * ppc);
        if (s) return s;
        if (grp.flip) swap_sets();   // the march graph starts from the first set
        np = (int64_t)plane * ppc;
        uniform_layout = true;
        // in-cell lattice of Mesh::SeedParticles (mesh.cpp:436-470), head first
        double oy[16], oz[16];
        int iside = (int)(std::pow((double)(ppc - 1), 0.5) + 1.0);
        for (int is = 0; is < ppc; is++) {
            double y, z;
            if (ppc == 1 || ppc == 2 || ppc == 3) {
                y = z = 0.5;
            } else if (ppc == 4) {
                y = 1. / 3. * (1. + is % 2);
                z = 1. / 3. * (1. + is / 2);
            } else {
                int iz = is / iside, iy = is - iside * iz;
                y = 1. / iside * (iy + .5);
                z = 1. / iside * (iz + .5);
            }
            oy[is] = y;
            oz[is] = z;
        }
        SeedFront sf{};
        sf.My = My; sf.Mz = Mz; sf.ppc = ppc;
        for (int is = 0; is < ppc; is++) {
            sf.offs_y[is] = oy[is];
            sf.offs_z[is] = oz[is];
        }
        sf.px0 = cfg.plasma_px0; sf.py0 = cfg.plasma_py0; sf.pz0 = cfg.plasma_pz0;
        sf.sx = cfg.pspread_x; sf.sy = cfg.pspread_y; sf.sz = cfg.pspread_z;
        sf.weight = cfg.plasma_density / ppc;   // Specie::GetWeight()*dens
        sf.use_profile = have_profile ? 1 : 0;
        sf.prof = profile;
        // the front layer i = l_Mx and the cell corners (mesh.cpp:415-417)
        sf.x_front = cfg.hx * L + phase;
        sf.hy = cfg.hy; sf.hz = cfg.hz;
        sf.y_half = My * cfg.hy / 2.;
        sf.z_half = Mz * cfg.hz / 2.;
        sf.seed = cfg.seed; sf.step = step;
        klaunch(KC_SEED, [&] {
            return launch_seed_front<T>(sf, pcell, py, pz, ppx, ppy, ppz, pw, st);
        });
        CK(cudaGetLastError());
        study_round_plasma(32, true);
        if ((s = cic_fresh_front())) return s;
        front_pending = true;
        return QS_OK;
    }

    int64_t plasma_count() const override { return np; }

    qs_status get_plasma(int64_t n, int32_t* cell, double* y, double* z, double* px,
                         double* py_, double* pz_, double* w) override {
        if (n != np) return fail(QS_ERR_INVALID, "qs_get_plasma: n mismatch");
        if (!n) return QS_OK;
        if (cic_sort) return get_plasma_by_id(n, cell, y, z, px, py_, pz_, w);
        if (cell) CK(cudaMemcpyAsync(cell, pcell, n * 4, cudaMemcpyDeviceToHost, st));
        double* dst[6] = {y, z, px, py_, pz_, w};
        T* src[6] = {py, pz, ppx, ppy, ppz, pw};
        for (int c = 0; c < 6; c++) {
            if (!dst[c]) continue;
            size_t chunk = 8 * plane;
            for (int64_t o = 0; o < n; o += (int64_t)chunk) {
                size_t m = (size_t)std::min<int64_t>((int64_t)chunk, n - o);
                klaunch(KC_MISC, [&] { return launch_convert_back<T>(src[c] + o, stage_d, m, st); });
                CK(cudaMemcpyAsync(dst[c] + o, stage_d, m * 8, cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
            }
        }
        CK(cudaStreamSynchronize(st));
        return QS_OK;
    }

    // the regrouped plasma back in load order (each particle carries its id)
    qs_status get_plasma_by_id(int64_t n, int32_t* cell, double* y, double* z, double* px,
                               double* py_, double* pz_, double* w) {
        std::vector<int32_t> id(n), ci(n);
        CK(cudaMemcpyAsync(id.data(), pid, n * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(ci.data(), pcell, n * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (cell)
            for (int64_t p = 0; p < n; p++) cell[id[p]] = ci[p];
        double* dst[6] = {y, z, px, py_, pz_, w};
        T* src[6] = {py, pz, ppx, ppy, ppz, pw};
        std::vector<double> tmp(n);
        for (int c = 0; c < 6; c++) {
            if (!dst[c]) continue;
            size_t chunk = 8 * plane;
            for (int64_t o = 0; o < n; o += (int64_t)chunk) {
                size_t m = (size_t)std::min<int64_t>((int64_t)chunk, n - o);
                klaunch(KC_MISC, [&] { return launch_convert_back<T>(src[c] + o, stage_d, m, st); });
                CK(cudaMemcpyAsync(tmp.data() + o, stage_d, m * 8, cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
            }
            for (int64_t p = 0; p < n; p++) dst[c][id[p]] = tmp[p];
        }
        return QS_OK;
    }

    // --------------------------------------------------------- plane I/O
    qs_status put_plane(T* dst, const double* src) {
        CK(cudaMemcpyAsync(stage_d, src, plane * 8, cudaMemcpyHostToDevice, st));
        klaunch(KC_MISC, [&] { return launch_convert<T>(stage_d, 1, dst, plane, st); });
        CK(cudaStreamSynchronize(st));
        return QS_OK;
    }
    qs_status get_plane(const T* src, double* dst) {
        klaunch(KC_MISC, [&] { return launch_convert_back<T>(src, stage_d, plane, st); });
        CK(cudaMemcpyAsync(dst, stage_d, plane * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return QS_OK;
    }

    T* layer_plane(int which, int field) {
        T* F = which == QS_LAYER_P ? Pf : Cf;
        T* Sr = which == QS_LAYER_P ? Psrc : Csrc;
        if (field >= QS_F_EX && field <= QS_F_BZ) return F + (size_t)field * plane;
        if (field >= QS_F_JX && field <= QS_F_JZ) return Sr + (size_t)(field - QS_F_JX) * plane;
        if (field == QS_F_DENS) return Sr + 3 * plane;
        return nullptr;
    }

    qs_status set_layer(int which, int field, const double* data) override {
        if ((which != QS_LAYER_P && which != QS_LAYER_C) || !data)
            return fail(QS_ERR_INVALID, "qs_set_layer: bad arguments");
        T* p = layer_plane(which, field);
        if (!p)
            return fail(QS_ERR_INVALID,
                        "qs_set_layer: field %d is not settable (the C-layer beam currents derive "
                        "from the beam-current store: use qs_set_beam_currents)", field);
        if (which == QS_LAYER_P) p_valid = false;
        return put_plane(p, data);
    }

    qs_status get_layer(int which, int field, double* out) override {
        if ((which != QS_LAYER_P && which != QS_LAYER_C) || !out)
            return fail(QS_ERR_INVALID, "qs_get_layer: bad arguments");
        if (which == QS_LAYER_C && (field == QS_F_RHOBEAM || field == QS_F_JXBEAM)) {
            // derived from the beam-current store at the current (layer, split)
            const int i = cur_layer < 0 ? L - 1 : cur_layer;
            const T* cur_b = b3 + (size_t)i * 2 * plane;
            const T* nxt_b = b3 + (size_t)(i + 1) * 2 * plane;
            if (b3_spec) {   // the real planes of layers i and i+1 from their spectra
                beam_real(cur_b, stage, 2);
                beam_real(nxt_b, stage + 2 * plane, 2);
                cur_b = stage;
                nxt_b = stage + 2 * plane;
            }
            klaunch(KC_MISC, [&] {
                return launch_beam_layer<T>(cur_b, nxt_b, S, cur_split, Cbeam, plane, d_err, st);
            });
            return get_plane(Cbeam + (field == QS_F_JXBEAM ? plane : 0), out);
        }
        T* p = layer_plane(which, field);
        if (!p) return fail(QS_ERR_INVALID, "qs_get_layer: field %d not readable", field);
        return get_plane(p, out);
    }

    qs_status get_field3d(int field, int layer, double* out) override {
        if (!out || layer < 0 || layer > L) return fail(QS_ERR_INVALID, "qs_get_field3d: bad layer");
        if (field >= QS_F_EX && field <= QS_F_BZ)
            return get_plane(f3layer(layer) + (size_t)field * plane, out);
        if (field >= QS_F_JX && field <= QS_F_DENS) {
            if (!src3) return fail(QS_ERR_STATE, "sources are stored only with store_sources=1");
            int q = field == QS_F_DENS ? 3 : field - QS_F_JX;
            return get_plane(src3 + ((size_t)layer * 4 + q) * plane, out);
        }
        return fail(QS_ERR_INVALID, "qs_get_field3d: bad field");
    }

    T* beam_plane(int field, int layer) {
        int q = field == QS_F_RHOBEAM ? 0 : (field == QS_F_JXBEAM ? 1 : -1);
        if (q < 0 || layer < 0 || layer > L) return nullptr;
        return b3 + ((size_t)layer * 2 + q) * plane;
    }
    qs_status set_beam_currents(int field, int layer, const double* data) override {
        T* p = beam_plane(field, layer);
        if (!p || !data) return fail(QS_ERR_INVALID, "qs_set_beam_currents: bad arguments");
        if (b3_spec) {   // the whole store back to real currents first
            batched_cc(b3, b3, 2 * (L + 1), KC_GEMM, inv_scale());
            b3_spec = false;
        }
        sb3_valid = false;
        ck_valid = false;
        return put_plane(p, data);
    }

    // nplanes real beam-current planes from their spectra at `spec` into `out`
    void beam_real(const T* spec, T* out, int nplanes) {
        T* outs[kMaxXfFields];
        int kz[kMaxXfFields], ky[kMaxXfFields];
        for (int f = 0; f < nplanes; f++) {
            outs[f] = out + (size_t)f * plane;
            kz[f] = ky[f] = CC;
        }
        xform(job_stack(spec, nplanes, outs, kz, ky, inv_scale()));
    }

    // Spectra of every layer's beam currents (RhoBeam, JxBeam: REDFT11 x
    // REDFT11, movefieldshydrolinlayersplit.cpp:717-718) in large batches,
    // once per beam push instead of once per layer; plus the |JxBeam| > 10
    // check of :618-621.
    // REDFT11 x REDFT11 transforms of np contiguous planes in large batches
    // (in place when in_planes == out_planes: every batch is read into the
    // transform's scratch before its output is written)
    void batched_cc(const T* in_planes, T* out_planes, int np, int cls, T scale = T(1)) {
        if (tc) {
            for (int b0 = 0; b0 < np; b0 += 64) {
                const int nf = std::min(64, np - b0);
                const float* in = (const float*)(in_planes + (size_t)b0 * plane);
                float* out = (float*)(out_planes + (size_t)b0 * plane);
                const double sc = (double)scale;
                klaunch(KC_SPLIT, [&] { return tcx->run_batched(in, out, nf, sc, 0, st); });
                klaunch(cls, [&] { return tcx->run_batched(in, out, nf, sc, 1, st); });
                klaunch(cls, [&] { return tcx->run_batched(in, out, nf, sc, 2, st); });
            }
        } else {
            for (int b0 = 0; b0 < np; b0 += kMaxXfFields) {
                const int nf = std::min(kMaxXfFields, np - b0);
                T* outs[kMaxXfFields];
                int kz[kMaxXfFields], ky[kMaxXfFields];
                for (int f = 0; f < nf; f++) {
                    outs[f] = out_planes + (size_t)(b0 + f) * plane;
                    kz[f] = ky[f] = CC;
                }
                xform(job_stack(in_planes + (size_t)b0 * plane, nf, outs, kz, ky, scale));
            }
        }
    }

    qs_status beam_spectra() {
        klaunch(KC_BEAM_SPECTRA, [&] {
            return launch_beam_check<T>(b3, L + 1, plane, d_err, qb_part, st);
        });
        klaunch(KC_MISC, [&] {
            return launch_charge_reduce(qb_part, kBeamSumParts, L + 1, 1.0, q_sums + 2 * (size_t)L,
                                        st);
        });
        batched_cc(b3, b3, 2 * (L + 1), KC_GEMM);   // in place: b3 now holds the spectra
        b3_spec = true;
        study_round(sb3, (size_t)(L + 1) * 2 * plane, 2);
        CK(cudaGetLastError());
        sb3_valid = true;
        return QS_OK;
    }
    qs_status get_beam_currents(int field, int layer, double* out) override {
        T* p = beam_plane(field, layer);
        if (!p || !out) return fail(QS_ERR_INVALID, "qs_get_beam_currents: bad arguments");
        if (b3_spec) {   // the real plane from its spectrum
            beam_real(p, stage, 1);
            return get_plane(stage, out);
        }
        return get_plane(p, out);
    }

    qs_status get_onaxis(double* out) override {
        if (!out) return fail(QS_ERR_INVALID, "qs_get_onaxis_ex: null");
        // from the field store, so that a march driven layer by layer through
        // the fine-grained entry points is read the same way
        klaunch(KC_MISC, [&] {
            return launch_onaxis<T>(f3, L, plane, (size_t)(My / 2) + (size_t)My * (Mz / 2), onaxis_d,
                                    st);
        });
        std::vector<T> h(L);
        CK(cudaMemcpyAsync(h.data(), onaxis_d, L * sizeof(T), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int i = 0; i < L; i++) out[i] = (double)h[i];
        return QS_OK;
    }

    // ------------------------------------------------------------- beam push
    qs_status move_beam() override {
        ck_valid = false;
        CK(cudaMemsetAsync(b3, 0, (size_t)(L + 1) * 2 * plane * sizeof(T), st));
        b3_spec = false;
        sb3_valid = false;
        BeamArgs<T> a{};
        a.n = nb;
        a.L = L; a.My = My; a.Mz = Mz;
        a.bi = bi; a.bj = bj; a.bk = bk;
        a.x = bx; a.y = by; a.z = bz; a.px = bpx; a.py = bpy; a.pz = bpz; a.w = bw;
        a.fields3d = f3;
        a.beam3d = b3;
        a.plane = plane;
        a.ts = cfg.ts; a.hx = cfg.hx; a.hy = cfg.hy; a.hz = cfg.hz;
        a.q2m = cfg.beam_q2m; a.polarity = cfg.beam_polarity;
        a.bxe = cfg.bx_ext; a.bye = cfg.by_ext; a.bze = cfg.bz_ext;
        a.syn_min = cfg.syn_min;
        a.elaser_photon = 1.2398e-4 / cfg.wavelength;
        a.synchrotron = cfg.synchrotron;
        a.err = d_err;
        klaunch(KC_BEAM_PUSH, [&] { return launch_beam_push<T>(a, st); });
        CK(cudaGetLastError());
        study_round(b3, (size_t)(L + 1) * 2 * plane, 16);
        return beam_spectra();
    }

    // --------------------------------------------------------- the march
    T* sbp(int layer, int q) { return sb3 + ((size_t)layer * 2 + q) * plane; }

    SpecArgs<T> spec_args(int iLayer, int iSplit) {
        SpecArgs<T> a{};
        a.ny = My; a.nz = Mz;
        const double Ylength = My * cfg.hy, Zlength = Mz * cfg.hz;
        a.piY = (T)(M_PI / Ylength);
        a.piZ = (T)(M_PI / Zlength);
        a.hx = (T)(cfg.hx / S);
        a.dens_p = dens_dev;
        const int pb = cur ^ 1, cb = cur;
        a.RhoP = bankp(pb, SP_RHO); a.ExP = bankp(pb, SP_EX); a.EyP = bankp(pb, SP_EY);
        a.EzP = bankp(pb, SP_EZ); a.JxP = bankp(pb, SP_JX); a.JyP = bankp(pb, SP_JY);
        a.JzP = bankp(pb, SP_JZ);
        // beam of this (layer, split): layers iLayer and iLayer+1 weighted (S-s)/S, s/S
        a.Rb0 = sbp(iLayer, 0); a.Rb1 = sbp(iLayer + 1, 0);
        a.Jxb0 = sbp(iLayer, 1); a.Jxb1 = sbp(iLayer + 1, 1);
        a.wb0 = (T)((double)(S - iSplit) / S);
        a.wb1 = (T)((double)iSplit / S);
        // beam of the previous (layer, split); zero on the head layer (:430-445)
        a.Rbp0 = a.Rb0; a.Rbp1 = a.Rb1; a.wp0 = T(0); a.wp1 = T(0);
        if (iLayer == L - 1 && iSplit == 0 && front_layer) {
            // below the first rank the head's RhoBeamP is the received layer's
            // beam spectrum (CUDA_WRAP_setBeamFFT, :547-551)
            a.Rbp0 = front_beam;
            a.wp0 = T(1);
        } else if (iLayer < L - 1 || front_layer) {
            if (iSplit > 0) {
                a.wp0 = (T)((double)(S - iSplit + 1) / S);
                a.wp1 = (T)((double)(iSplit - 1) / S);
            } else {
                a.Rbp0 = sbp(iLayer + 1, 0);
                a.Rbp1 = sbp(std::min(iLayer + 2, L), 0);
                a.wp0 = (T)(1.0 / S);
                a.wp1 = (T)((double)(S - 1) / S);
            }
        }
        a.Jx = bankp(cb, SP_JX); a.Jy = bankp(cb, SP_JY); a.Jz = bankp(cb, SP_JZ);
        a.Rho = bankp(cb, SP_RHO);
        a.Ex = bankp(cb, SP_EX); a.Ey = bankp(cb, SP_EY); a.Ez = bankp(cb, SP_EZ);
        a.Bx = bankp(cb, SP_BX); a.By = bankp(cb, SP_BY); a.Bz = bankp(cb, SP_BZ);
        a.write_b = tc ? 0 : 1;
        if (tc) {
            int ns = 0, kd = 0;
            size_t ts = 0;
            void* base = nullptr;
            tcx->split_target(&base, &ns, &kd, &ts);
            a.split = base; a.nsplit = ns; a.split_kind = kd; a.tstride = ts;
        }
        return a;
    }

    // inverse transforms of the spectral E, B (+ Rho) into the C layer
    void inverse_EB(bool with_rho, T* work = nullptr) {
        const int cb = cur;
        const int nf = with_rho ? 7 : 6;
        T* outs[7] = {Cf, Cf + plane, Cf + 2 * plane, Cf + 3 * plane, Cf + 4 * plane,
                      Cf + 5 * plane, Csrc + 3 * plane};
        const int kz[7] = {CC, CC, SS, SS, SS, CC, CC};
        const int ky[7] = {CC, SS, CC, SS, CC, SS, CC};
        if (tc) {   // the spectral kernel already wrote the split operand
            for (int stage = 1; stage <= 2; stage++)
                klaunch(KC_GEMM, [&] {
                    return tcx->run_stage(stage, nf, nullptr, (void* const*)outs, kz, ky,
                                          (double)inv_scale(), st);
                });
        } else {
            DttJob<T> j;
            j.nf = nf;
            const int src[7] = {SP_EX, SP_EY, SP_EZ, SP_BX, SP_BY, SP_BZ, SP_RHO};
            for (int f = 0; f < nf; f++) {
                j.in[f] = bankp(cb, src[f]);
                j.out[f] = outs[f];
                j.kz[f] = kz[f];
                j.ky[f] = ky[f];
            }
            j.scale = inv_scale();
            xform(j, work);
        }
    }

    qs_status begin_march() override {
        ck_valid = false;   // a march driven piece by piece keeps no checkpoints
        if (qs_status s0 = set_march_density()) return s0;
        if (qs_status s0 = take_front_layer()) return s0;
        if (!front_pending) {
            qs_status s = seed_front(step_count);
            if (s) return s;
        }
        front_pending = false;
        return begin_march_device();
    }

    // the device part of MoveAllSplitLayers' set-up (capturable)
    qs_status begin_march_device() {
        if (src3) CK(cudaMemsetAsync(src3, 0, (size_t)(L + 1) * 4 * plane * sizeof(T), st));
        CK(cudaMemsetAsync(q_part, 0, (size_t)L * 2 * q_nparts * sizeof(double), st));
        Psrc = srcbuf;
        Csrc = srcbuf + 4 * plane;
        CK(cudaMemsetAsync(srcbuf, 0, 8 * plane * sizeof(T), st));
        cur = 0;
        p_valid = true;
        if (front_layer) {
            // the received layer is P of the head layer; its spectra are
            // forward transforms of its planes, as Guess computes them (:717-743)
            CK(cudaMemcpyAsync(Psrc, front_src, 4 * plane * sizeof(T), cudaMemcpyDeviceToDevice,
                               st));
            p_valid = false;
        }
        Pf = f3layer(L);
        Cf = f3layer(L - 1);
        cur_layer = -1;
        cur_split = 0;
        marched = true;
        tail_ready = false;
        return QS_OK;
    }

    qs_status layer_begin(int iLayer, int iSplit) override {
        if (iLayer < 0 || iLayer >= L || iSplit < 0 || iSplit >= S)
            return fail(QS_ERR_INVALID, "qs_layer_begin: bad layer/split");
        if (iSplit == 0) Pf = f3layer(iLayer + 1);
        else Pf = Cf;
        Cf = (iSplit == S - 1) ? f3layer(iLayer) : splitbuf + (size_t)(iSplit & 1) * 6 * plane;
        cur_layer = iLayer;
        cur_split = iSplit;
        return QS_OK;
    }

    qs_status guess(int iLayer, int iSplit) override {
        const int pb = cur ^ 1;
        if (!sb3_valid || !p_valid) join_sides();   // these transforms use scratch
        if (!sb3_valid) {
            qs_status s = beam_spectra();
            if (s) return s;
        }
        if (iLayer == L - 1 && iSplit == 0 && p_valid) {
            // :430-445 the head layer starts from zero spectra (P is layer nx = 0)
            CK(cudaMemsetAsync(bankp(pb, 0), 0, (size_t)SP_RB * plane * sizeof(T), st));
        }
        if (!p_valid) {
            // P planes were set from outside: transform them like :717-743
            T* outs[7] = {bankp(pb, SP_RHO), bankp(pb, SP_EX), bankp(pb, SP_EY),
                          bankp(pb, SP_EZ), bankp(pb, SP_JX), bankp(pb, SP_JY),
                          bankp(pb, SP_JZ)};
            const T* ins[7] = {Psrc + 3 * plane, Pf, Pf + plane, Pf + 2 * plane, Psrc,
                               Psrc + plane, Psrc + 2 * plane};
            const int kz[7] = {CC, CC, CC, SS, CC, CC, SS};
            const int ky[7] = {CC, CC, SS, CC, CC, SS, CC};
            for (int f = 0; f < 7; f++)
                CK(cudaMemcpyAsync(stage + (size_t)f * plane, ins[f], plane * sizeof(T),
                                   cudaMemcpyDeviceToDevice, st));
            xform(job_stack(stage, 7, outs, kz, ky, T(1)));
            p_valid = true;
        }
        if (fft_maps() && pred_next == iLayer && iSplit == 0 && p_valid && sb3_valid) {
            // the previous layer's last corrector kernel ran this predictor
            pred_next = -1;
            half_avg = next_avg;
            next_avg = false;
            eb_zpass(6, scratch2);
            CK(cudaGetLastError());
            return QS_OK;
        }
        pred_next = -1;
        next_avg = half_avg = false;
        if (fft_maps()) {
            // predictor and the inverse y-pass of E, B in one kernel, then the z-pass
            SpecArgs<T> a = spec_args(iLayer, iSplit);
            a.zero_src = clear_by_maps() ? Csrc : nullptr;
            a.write_b = 0;
            // beside a pending last z-pass of the previous layer (reading
            // scratch) the map writes scratch2
            T* out = side_z ? scratch2 : scratch;
            klaunch(KC_SPECTRAL, [&] { return spec_rows_run(a, false, nullptr, out, 6); });
            eb_zpass(6, out);
            CK(cudaGetLastError());
            return QS_OK;
        }
        {
            SpecArgs<T> a = spec_args(iLayer, iSplit);
            a.zero_src = clear_by_maps() ? Csrc : nullptr;   // for the push that follows
            klaunch(KC_SPECTRAL, [&] { return launch_predictor<T>(a, st); });
            study_round(bankp(cur, 0), (size_t)SP_RB * plane, 2);
        }
        // :946-967, :1004-1061: E, B into C (the predicted Rho and J planes are
        // cleared before any use by the push that follows)
        inverse_EB(false);
        study_round(Cf, 6 * plane, 8);
        CK(cudaGetLastError());
        return QS_OK;
    }

    // FP32 FFT transforms with the Guess / Iterate maps between their halves
    bool fft_maps() const {
        // (the precision study rounds the state between separate map kernels)
        return (fftx && fftx->spec_rows) || (fftx64 && fftx64->spec_rows && !fp32_study);
    }
    // the adjoint's maps between the halves of its transforms (FP32)
    bool adj_fused() const { return fftx && fftx->spec_rows; }
    int spec_rows_run(const SpecArgs<T>& a, bool correct, const T* jin, T* out, int nout,
                      const SpecArgs<T>* next = nullptr, T* out_next = nullptr,
                      bool avg_next = false) {
        if constexpr (sizeof(T) == 4)
            return fftx->run_spectral_rows(a, correct, jin, out, nout, st, next, out_next,
                                           avg_next);
        else
            return fftx64->run_spectral_rows(a, correct, jin, out, nout, st, next, out_next,
                                             avg_next);
    }
    int cols_run(int nf, const T* const* in, T* const* out, const int* kind, T scale) {
        if constexpr (sizeof(T) == 4) return fftx->run_cols(nf, in, out, kind, scale, st);
        else return fftx64->run_cols(nf, in, out, kind, scale, st);
    }

    // z-pass of the E, B (and Rho) planes the map kernel left in `from`:
    // E, B into the C layer, Rho into the density plane of the C sources
    void eb_zpass(int nout, const T* from) {
        const T* ins[7];
        T* outs[7] = {Cf, Cf + plane, Cf + 2 * plane, Cf + 3 * plane, Cf + 4 * plane,
                      Cf + 5 * plane, Csrc + 3 * plane};
        const int kz[7] = {CC, CC, SS, SS, SS, CC, CC};
        for (int f = 0; f < nout; f++) ins[f] = from + (size_t)f * plane;
        klaunch(KC_GEMM, [&] { return cols_run(nout, ins, outs, kz, inv_scale()); });
    }

    // Inside the march (no source store) the deposit planes are cleared by
    // the spectral kernel that precedes each push instead of by a memset.
    bool clear_by_maps() const { return in_march && !src3; }

    qs_status push(int iLayer, int iSplit, int full) override {
        (void)iLayer; (void)iSplit;
        // the fields and the plasma this push reads: with the averaged fields
        // in C the previous layer's last z-pass (side 0) is not among them
        const bool from_avg = !full && half_avg;
        half_avg = false;
        if (from_avg) join_side(1);
        else join_sides();
        if (fp32_study & (4 | 128)) return study_push(full);
        // ClearCurrentsSplit: inside the march the preceding spectral kernel
        // already cleared Csrc
        if (!clear_by_maps()) CK(cudaMemsetAsync(Csrc, 0, 4 * plane * sizeof(T), st));
        if (cic_sort) {
            qs_status s = cic_prepare();
            if (s) return s;
        }
        PushArgs<T> a{};
        a.n = np;
        a.My = My; a.Mz = Mz;
        a.cell = pcell;
        a.y = py; a.z = pz; a.px = ppx; a.py = ppy; a.pz = ppz; a.w = pw;
        a.P = from_avg ? Cf : Pf;   // (C + C) / 2 = C exactly
        a.C = Cf;
        if (push_fields) {   // the adjoint's recomputation: the stored gathered fields
            a.P = a.C = push_fields;
            push_fields = nullptr;
        }
        a.dep = Csrc;
        a.cell_out = pcell;
        a.dep_cell = nullptr;
        a.plane = plane;
        a.hx = (T)(cfg.hx / S); a.hy = (T)cfg.hy; a.hz = (T)cfg.hz;
        a.q2m = (T)cfg.plasma_q2m;
        a.djx0 = (T)cfg.plasma_djx0; a.djy0 = (T)cfg.plasma_djy0; a.djz0 = (T)cfg.plasma_djz0;
        a.drho0 = (T)cfg.plasma_drho0;
        a.bxe = (T)cfg.bx_ext; a.bye = (T)cfg.by_ext; a.bze = (T)cfg.bz_ext;
        a.sE = (T)(cfg.plasma_q2m * (cfg.hx / S) / 2.0);
        a.hxhy = (T)((cfg.hx / S) / cfg.hy);
        a.hxhz = (T)((cfg.hx / S) / cfg.hz);
        a.invMy = 1.0f / (float)My;
        // lattice order (particle p seeded in cell p / ppc): the NGP
        // one-thread-per-cell kernel relies on it
        a.uniform_ppc = uniform_layout ? cfg.ppc : 0;
        a.full = full;
        a.err = d_err;
        a.skip_dens = clear_by_maps() ? 1 : 0;   // the march never reads the density deposit
        a.favg = push_favg;
        push_favg = nullptr;
        bool regroup = false;
        if (cic_sort) {
            a.loff = cic_loff;
            a.bpref = cic_bpref;
            regroup = full && !adj_recompute && grp.since + 1 >= cic_every;
            a.cnt = regroup ? cic_cnt : nullptr;   // the full push builds the histogram
        }
        const bool precise = sizeof(T) == 4;
        klaunch(KC_PUSH, [&] { return launch_push<T>(a, cfg.shape, precise, st); });
        CK(cudaGetLastError());
        if (full) study_round_plasma(64, false);
        if (cic_sort && full && !adj_recompute) {
            if (regroup) {   // regroup before the next push
                grp.grouped = false;
                grp.off_valid = false;
                grp.counted = true;
                grp.since = 0;
            } else {
                grp.since++;
            }
        }
        if (regroup && side_sort) {   // beside the Iterate and Guess that follow
            qs_status s = QS_OK;
            const cudaError_t e = on_side(1, [&] { s = cic_prepare(); });
            if (e != cudaSuccess) return cuda_fail(e, "side stream");
            if (s) return s;
        }
        return QS_OK;
    }

    // run f() on side stream k after the work queued so far on st; the
    // launches inside f() go to the side stream
    template <class F>
    cudaError_t on_side(int k, F&& f) {
        cudaError_t e = cudaEventRecord(ev_fork[k], st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st_side[k], ev_fork[k], 0);
        if (e != cudaSuccess) return e;
        std::swap(st, st_side[k]);
        f();
        std::swap(st, st_side[k]);
        side_pending[k] = true;
        return cudaEventRecord(ev_join[k], st_side[k]);
    }
    // make st wait for side stream k's pending work
    void join_side(int k) {
        if (side_pending[k]) {
            cudaStreamWaitEvent(st, ev_join[k], 0);
            side_pending[k] = false;
        }
    }
    // make st wait for the side streams' pending work
    void join_sides() {
        for (int k = 0; k < 2; k++)
            if (side_pending[k]) {
                cudaStreamWaitEvent(st, ev_join[k], 0);
                side_pending[k] = false;
            }
    }

    qs_status iterate(int iLayer, int iSplit, int iter, double* rel_err) override {
        const int cb = cur;
        std::vector<double> oldE;
        if (rel_err) {
            CK(cudaStreamSynchronize(st));
            oldE.resize(3 * plane);
            for (int c = 0; c < 3; c++) {
                qs_status s = get_plane(Cf + c * plane, oldE.data() + c * plane);
                if (s) return s;
            }
        }
        // the last iterate stores Dens too (:1517-1602); inside the march that
        // real-space density is output only, so it is kept when sources are stored
        const bool want_rho = iter < 0 && (!in_march || src3 != nullptr);
        if (fft_maps()) {
            // :1343-1345 along z, then the y-pass of J, the corrector and the
            // inverse y-pass of E, B (, Rho) in one kernel, then their z-pass
            {
                join_side(0);   // a pending last z-pass of the previous layer reads scratch
                const T* ins[3] = {Csrc, Csrc + plane, Csrc + 2 * plane};
                T* outs[3] = {scratch, scratch + plane, scratch + 2 * plane};
                const int kz[3] = {CC, CC, SS};
                klaunch(KC_GEMM, [&] { return cols_run(3, ins, outs, kz, T(1)); });
                SpecArgs<T> a = spec_args(iLayer, iSplit);
                a.write_b = 0;
                a.zero_src = (clear_by_maps() && iter >= 0) ? Csrc : nullptr;
                charge_args(a, iLayer, iSplit, iter);
                const int nout = want_rho ? 7 : 6;
                // the layer's last corrector also runs the next layer's
                // predictor on its rows (the next Guess then only z-passes)
                const bool fuse = side_z && iter < 0 && nout == 6 && iLayer > fuse_lo && S == 1;
                SpecArgs<T> an{};
                if (fuse) {
                    cur ^= 1;   // the banks as layer_end leaves them
                    an = spec_args(iLayer - 1, 0);
                    cur ^= 1;
                    an.zero_src = clear_by_maps() ? Psrc : nullptr;   // the next push's deposit
                    an.write_b = 0;
                }
                // the next layer's first push gathers the average of this
                // layer's fields and the predicted ones: with the grouped CIC
                // push (whose gathered fields the adjoint reads) the map
                // kernel forms it, so that push needs one z-pass, not two
                const bool avg = fuse && cic_sort && clear_by_maps();
                klaunch(KC_SPECTRAL, [&] {
                    return spec_rows_run(a, true, scratch, scratch, nout, fuse ? &an : nullptr,
                                         fuse ? scratch2 : nullptr, avg);
                });
                pred_next = fuse ? iLayer - 1 : -1;
                next_avg = avg;
                if (side_z && iter < 0 && nout == 6) {
                    // the layer's last z-pass: only the next layer's pushes read it
                    const cudaError_t e = on_side(0, [&] { eb_zpass(nout, scratch); });
                    if (e != cudaSuccess) return cuda_fail(e, "side stream");
                } else {
                    eb_zpass(nout, scratch);
                }
            }
            CK(cudaGetLastError());
        } else {
            {   // :1343-1345
                T* outs[3] = {bankp(cb, SP_JX), bankp(cb, SP_JY), bankp(cb, SP_JZ)};
                const int kz[3] = {CC, CC, SS}, ky[3] = {CC, SS, CC};
                xform(job_stack(Csrc, 3, outs, kz, ky, T(1)));
            }
            SpecArgs<T> a = spec_args(iLayer, iSplit);
            a.split_rho = want_rho ? 1 : 0;
            charge_args(a, iLayer, iSplit, iter);
            // a push follows every Iterate but the last: clear its deposit planes
            // (the forward J transform above has consumed them)
            a.zero_src = (clear_by_maps() && iter >= 0) ? Csrc : nullptr;
            klaunch(KC_SPECTRAL, [&] { return launch_corrector<T>(a, st); });
            study_round(bankp(cb, 0), (size_t)SP_RB * plane, 2);
            if (side_z && iter < 0 && !want_rho) {
                // the layer's last inverse transform: only the next layer's
                // pushes read it, and nothing writes its bank before them
                const cudaError_t e = on_side(0, [&] { inverse_EB(false, scratch2); });
                if (e != cudaSuccess) return cuda_fail(e, "side stream");
            } else {
                inverse_EB(want_rho);
            }
            study_round(Cf, 6 * plane, 8);
            CK(cudaGetLastError());
        }
        if (rel_err) {
            std::vector<double> nw(plane);
            double mx[3] = {1e-5, 1e-5, 1e-5}, df[3] = {0, 0, 0};
            for (int c = 0; c < 3; c++) {
                qs_status s = get_plane(Cf + c * plane, nw.data());
                if (s) return s;
                for (size_t n = 0; n < plane; n++) {
                    mx[c] = std::max(mx[c], std::fabs(nw[n]));
                    df[c] = std::max(df[c], std::fabs(oldE[c * plane + n] - nw[n]));
                }
            }
            *rel_err = std::max(std::max(df[0] / mx[0], df[1] / mx[1]), df[2] / mx[2]);
        }
        return QS_OK;
    }

    // the last corrector of a layer writes its FP64 charge partials (not while
    // the adjoint recomputes a segment: the march's sums stand)
    void charge_args(SpecArgs<T>& a, int iLayer, int iSplit, int iter) {
        if (iter >= 0 || iSplit != S - 1 || adj_recompute) return;
        a.qsum = q_part + (size_t)iLayer * 2 * q_nparts;
        a.qcy = q_cy;
        a.qcz = q_cz;
    }

    // ------------------------------------------------------- layer output
    // Mesh::Save's field file (save.cpp:520-838) and Mesh::SaveCadrMovie2's
    // central slices (mesh.cpp:976-1090), in the QSF1 layout of qsb200.h:
    // the reference's dataset names, x (the layer index) fastest.
    qs_status save_output(const char* path, bool movie) override {
        if (!path) return fail(QS_ERR_INVALID, "qs_save: null path");
        struct Set {
            std::string name;
            int dtype;               // 1 int32, 2 float64
            int64_t d[3];
            std::function<qs_status(FILE*)> write;
        };
        std::vector<Set> sets;
        auto host_set = [&](const char* name, std::vector<double> v) {
            const int64_t n = (int64_t)v.size();
            sets.push_back({name, 2, {n, 1, 1}, [v](FILE* f) {
                                return fwrite(v.data(), sizeof(double), v.size(), f) == v.size()
                                           ? QS_OK : QS_ERR_INVALID;
                            }});
        };
        {
            // meshinfo: l_Mx, l_dMx, l_sizeX, l_offsetX and the same for y and
            // z (no guard cells here), then four zeros
            std::vector<int32_t> mi = {L, 0, L, 0, My, 0, My, 0, Mz, 0, Mz, 0, 0, 0, 0, 0};
            sets.push_back({"meshinfo", 1, {16, 1, 1}, [mi](FILE* f) {
                                return fwrite(mi.data(), sizeof(int32_t), mi.size(), f) ==
                                               mi.size() ? QS_OK : QS_ERR_INVALID;
                            }});
        }
        host_set("phase", {phase});
        {
            std::vector<double> X(L), Y(My), Z(Mz);
            for (int i = 0; i < L; i++) X[i] = cfg.hx * i + phase;
            for (int j = 0; j < My; j++) Y[j] = cfg.hy * j - My * cfg.hy / 2.;
            for (int k = 0; k < Mz; k++) Z[k] = cfg.hz * k - Mz * cfg.hz / 2.;
            host_set("X", X);
            host_set("Y", Y);
            host_set("Z", Z);
        }
        // a block of the store in x-fastest order through the staging buffer
        const size_t cap = 8 * plane;
        auto gathered = [this, cap](const T* base, size_t stride, int j0, int nj, int k0, int nk,
                                    FILE* f) -> qs_status {
            std::vector<double> h;
            const size_t row = (size_t)L * nj;           // one kk of the block
            for (int kk = 0; kk < nk;) {
                int nkc = (int)std::max<size_t>(1, cap / std::max<size_t>(row, 1));
                nkc = std::min(nkc, nk - kk);
                if (row > cap) {                          // a row in pieces of whole x runs
                    const int njc = (int)std::max<size_t>(1, cap / L);
                    for (int jj = 0; jj < nj; jj += njc) {
                        const int n = std::min(njc, nj - jj);
                        klaunch(KC_MISC, [&] {
                            return launch_gather_xfast<T>(base, stride, L, My, j0 + jj, n,
                                                          k0 + kk, 1, stage_d, st);
                        });
                        h.resize((size_t)L * n);
                        CK(cudaMemcpyAsync(h.data(), stage_d, h.size() * 8, cudaMemcpyDeviceToHost,
                                           st));
                        CK(cudaStreamSynchronize(st));
                        if (fwrite(h.data(), 8, h.size(), f) != h.size()) return QS_ERR_INVALID;
                    }
                    kk += 1;
                    continue;
                }
                klaunch(KC_MISC, [&] {
                    return launch_gather_xfast<T>(base, stride, L, My, j0, nj, k0 + kk, nkc,
                                                  stage_d, st);
                });
                h.resize(row * nkc);
                CK(cudaMemcpyAsync(h.data(), stage_d, h.size() * 8, cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                if (fwrite(h.data(), 8, h.size(), f) != h.size()) return QS_ERR_INVALID;
                kk += nkc;
            }
            return QS_OK;
        };
        struct Src { const char* name; const T* base; size_t stride; };
        std::vector<Src> srcs = {{"Ex", f3, 6 * plane}, {"Ey", f3 + plane, 6 * plane},
                                 {"Ez", f3 + 2 * plane, 6 * plane}, {"Bx", f3 + 3 * plane, 6 * plane},
                                 {"By", f3 + 4 * plane, 6 * plane}, {"Bz", f3 + 5 * plane, 6 * plane}};
        if (src3) {   // the sources of every layer (kept with store_sources = 1)
            srcs.push_back({"Jx", src3, 4 * plane});
            srcs.push_back({"Jy", src3 + plane, 4 * plane});
            srcs.push_back({"Jz", src3 + 2 * plane, 4 * plane});
            srcs.push_back({"Dens", src3 + 3 * plane, 4 * plane});
        }
        for (const Src& q : srcs) {
            if (!movie) {
                sets.push_back({q.name, 2, {L, My, Mz}, [=](FILE* f) {
                                    return gathered(q.base, q.stride, 0, My, 0, Mz, f);
                                }});
            } else {   // the (x, y) plane through the axis and the (x, z) plane
                sets.push_back({std::string(q.name) + "_xy", 2, {L, My, 1}, [=](FILE* f) {
                                    return gathered(q.base, q.stride, 0, My, Mz / 2, 1, f);
                                }});
                sets.push_back({std::string(q.name) + "_xz", 2, {L, Mz, 1}, [=](FILE* f) {
                                    return gathered(q.base, q.stride, My / 2, 1, 0, Mz, f);
                                }});
            }
        }
        // header: magic, count, then one 72-byte entry per set (name[32],
        // dtype, rank, dims[3] fastest first, byte offset of the data)
        const int64_t hdr = 16 + 72 * (int64_t)sets.size();
        std::vector<int64_t> off(sets.size());
        int64_t pos = hdr;
        for (size_t d = 0; d < sets.size(); d++) {
            off[d] = pos;
            const int64_t n = sets[d].d[0] * sets[d].d[1] * sets[d].d[2];
            pos += n * (sets[d].dtype == 1 ? 4 : 8);
            pos = (pos + 7) & ~(int64_t)7;
        }
        FILE* f = fopen(path, "wb");
        if (!f) return fail(QS_ERR_INVALID, "qs_save: cannot open %s", path);
        bool ok = fwrite("QSF1\0\0\0\0", 1, 8, f) == 8;
        const int32_t cnt[2] = {(int32_t)sets.size(), 0};
        ok = ok && fwrite(cnt, 4, 2, f) == 2;
        for (size_t d = 0; d < sets.size() && ok; d++) {
            char name[32] = {};
            std::strncpy(name, sets[d].name.c_str(), 31);
            const int rank = sets[d].d[2] > 1 ? 3 : (sets[d].d[1] > 1 ? 2 : 1);
            const int32_t ty[2] = {sets[d].dtype, rank};
            ok = fwrite(name, 1, 32, f) == 32 && fwrite(ty, 4, 2, f) == 2 &&
                 fwrite(sets[d].d, 8, 3, f) == 3 && fwrite(&off[d], 8, 1, f) == 1;
        }
        qs_status s = ok ? QS_OK : QS_ERR_INVALID;
        for (size_t d = 0; d < sets.size() && !s; d++) {
            if (fseek(f, (long)off[d], SEEK_SET) != 0) s = QS_ERR_INVALID;
            else s = sets[d].write(f);
        }
        if (fclose(f) != 0 && !s) s = QS_ERR_INVALID;
        if (s == QS_ERR_INVALID) return fail(s, "qs_save: write to %s failed", path);
        if (s) return s;
        return check_device();
    }

    qs_status get_charge_sums(double* rho, double* jx, double* rho_beam) override {
        // the plasma sums of the layers marched so far (the march also runs
        // this reduction at its end)
        klaunch(KC_MISC, [&] {
            return launch_charge_reduce(q_part, q_nparts, L, 1.0 / (4.0 * My * Mz), q_sums, st);
        });
        std::vector<double> h((size_t)2 * L + 2 * (L + 1));
        CK(cudaMemcpyAsync(h.data(), q_sums, h.size() * sizeof(double), cudaMemcpyDeviceToHost,
                           st));
        CK(cudaStreamSynchronize(st));
        for (int i = 0; i < L; i++) {
            if (rho) rho[i] = h[2 * (size_t)i];
            if (jx) jx[i] = h[2 * (size_t)i + 1];
        }
        if (rho_beam)
            for (int i = 0; i <= L; i++) rho_beam[i] = h[2 * (size_t)L + 2 * (size_t)i];
        return QS_OK;
    }

    qs_status move_split_layer(int iLayer, int iSplit) override {
        // with the adjoint's field store, each push leaves its gathered fields there
        const bool keep = in_march && !adj_recompute && fstored(iLayer);
        qs_status s = guess(iLayer, iSplit);
        if (s) return s;
        for (int it = 0; it < nIter; it++) {
            if (keep) push_favg = fstore_at(iLayer, it);
            if ((s = push(iLayer, iSplit, 0))) return s;
            if ((s = iterate(iLayer, iSplit, it, nullptr))) return s;
        }
        if (keep) push_favg = fstore_at(iLayer, nIter);
        if ((s = push(iLayer, iSplit, 1))) return s;
        return iterate(iLayer, iSplit, -1, nullptr);
    }

    qs_status layer_end(int iLayer, int iSplit) override {
        if (iLayer == 0 && iSplit == S - 1) tail_ready = true;
        cur ^= 1;
        std::swap(Psrc, Csrc);
        if (iSplit == S - 1 && src3)
            CK(cudaMemcpyAsync(src3 + (size_t)iLayer * 4 * plane, Psrc, 4 * plane * sizeof(T),
                               cudaMemcpyDeviceToDevice, st));
        return QS_OK;
    }

    qs_status march_device() {
        in_march = true;
        g_pdl = use_pdl && !prof;   // event pairs between kernels would break the chain
        // side streams: not under per-kernel event timing or the precision study
        const bool side = !prof && !fp32_study;
        side_z = side && (fft_maps() || fftx64) && S == 1 && !src3;
        side_sort = side && cic_sort;
        pred_next = -1;
        next_avg = half_avg = false;
        fuse_lo = 0;
        qs_status s = march_device_body();
        join_sides();
        side_z = side_sort = false;
        pred_next = -1;
        next_avg = half_avg = false;
        g_pdl = false;
        in_march = false;
        return s;
    }

    qs_status march_device_body() {
        qs_status s = begin_march_device();
        if (s) return s;
        for (int i = L - 1; i >= 0; i--)
            for (int sp = 0; sp < S; sp++) {
                if (ck_every > 0 && sp == 0 && (L - 1 - i) % ck_every == 0)
                    if ((s = save_checkpoint((L - 1 - i) / ck_every))) return s;
                if ((s = layer_begin(i, sp))) return s;
                if ((s = move_split_layer(i, sp))) return s;
                if ((s = layer_end(i, sp))) return s;
            }
        join_sides();
        klaunch(KC_MISC, [&] {
            return launch_onaxis<T>(f3, L, plane, (size_t)(My / 2) + (size_t)My * (Mz / 2), onaxis_d,
                                    st);
        });
        klaunch(KC_MISC, [&] {
            return launch_charge_reduce(q_part, q_nparts, L, 1.0 / (4.0 * My * Mz), q_sums, st);
        });
        return QS_OK;
    }

    // ------------------------------------------------- xi-pipeline hand-off
    // PackLayer / UnpackLayer (para.cpp:94-285).  A received layer serves the
    // one march that follows it; the march after that starts from the empty
    // front again unless another layer arrives (the reference receives one
    // every step, para.cpp:346-412, movepart_splitlayer.cpp:105-151).
    qs_status take_front_layer() {
        if (front_layer && front_used) return clear_front_layer();
        if (front_layer) front_used = true;
        return QS_OK;
    }

    qs_status clear_front_layer() override {
        if (front_layer) CK(cudaMemsetAsync(f3layer(L), 0, 6 * plane * sizeof(T), st));
        front_layer = false;
        front_used = false;
        return QS_OK;
    }

    int64_t pack_size() const override { return 12 * (int64_t)plane + 12 * np; }

    // Plane order of the hand-off buffer (para.cpp:108-120): Bx, By, Bz, Ex,
    // Ey, Ez, Jx, Jy, Jz, Rho, fftJxBeamHydro, fftRhoBeamHydro; particle
    // blocks (:135-146): Px, Py, Pz, X, Y, Z, Q2m, Weight, i_X, i_Y, i_Z, isort.
    qs_status pack_layer(double* buf, int64_t n) override {
        if (!buf || n != pack_size())
            return fail(QS_ERR_INVALID, "qs_pack_layer: n must be qs_layer_pack_size (%lld)",
                        (long long)pack_size());
        if (!tail_ready) return fail(QS_ERR_STATE, "qs_pack_layer: no complete march to pack");
        {
            const qs_status s0 = check_device();   // the march's own errors come first
            if (s0) return s0;
        }
        // the buffer is assembled in device memory and leaves in one copy
        {
            qs_status s = ensure_pack_space(n, np);
            if (s) return s;
        }
        const size_t P = plane;
        double* dp = d_pack;
        // the tail layer's fields
        const int fsrc[6] = {3, 4, 5, 0, 1, 2};
        for (int f = 0; f < 6; f++)
            klaunch(KC_MISC, [&] {
                return launch_convert_back<T>(f3layer(0) + (size_t)fsrc[f] * P, dp + (size_t)f * P,
                                              P, st);
            });
        // its currents: the deposit of its last push, kept as the P sources
        for (int f = 0; f < 3; f++)
            klaunch(KC_MISC, [&] {
                return launch_convert_back<T>(Psrc + (size_t)f * P, dp + (size_t)(6 + f) * P, P,
                                              st);
            });
        // its Rho: the corrected spectral rho, inverse-transformed and
        // normalised as the Iterate store does (:1546-1602)
        {
            T* outs[1] = {stage};
            const int kz[1] = {CC}, ky[1] = {CC};
            xform(job_stack(bankp(cur ^ 1, SP_RHO), 1, outs, kz, ky, inv_scale()));
            klaunch(KC_MISC, [&] { return launch_convert_back<T>(stage, dp + 9 * P, P, st); });
        }
        // the beam spectra of its last split (fft_of_JxBeam, fft_of_RhoBeam)
        {
            const double w0 = 1.0 / S, w1 = (double)(S - 1) / S;
            for (int q = 0; q < 2; q++) {
                double* out = dp + (q == 0 ? 11 : 10) * P;
                if (S > 1)
                    klaunch(KC_MISC, [&] {
                        return launch_pack_mix<T>(sbp(0, q), sbp(1, q), w0, w1, P, out, st);
                    });
                else
                    klaunch(KC_MISC, [&] { return launch_convert_back<T>(sbp(0, q), out, P, st); });
            }
        }
        // the plasma in flight, cell by cell, load order within a cell
        if (np > 0) {
            int* cnt = d_pack_i;
            int* fill = cnt + P;
            int* start = fill + P;
            int32_t* ord = start + P + 1;
            CK(cudaMemsetAsync(cnt, 0, 2 * P * sizeof(int), st));
            PackArgs<T> a{};
            a.m = np; a.My = My; a.ncell = (int)P;
            a.cell = pcell;
            a.key = cic_sort ? pid : nullptr;   // regrouped: the load ids give the order
            a.y = py; a.z = pz; a.px = ppx; a.py = ppy; a.pz = ppz; a.w = pw;
            a.q2m = cfg.plasma_q2m;
            a.cnt = cnt; a.start = start; a.fill = fill; a.ord = ord;
            a.out = dp + 12 * P;
            a.err = d_err;
            klaunch(KC_MISC, [&] { return launch_pack_particles<T>(a, st); });
        }
        CK(cudaMemcpyAsync(buf, dp, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaGetLastError());
        return check_device();
    }

    qs_status unpack_layer(const double* buf, int64_t n) override {
        const int64_t fixed = 12 * (int64_t)plane;
        if (!buf || n < fixed || (n - fixed) % 12)
            return fail(QS_ERR_INVALID, "qs_unpack_layer: n must be 12*ny*nz + 12*Np");
        const int64_t m = (n - fixed) / 12;
        if (m > INT32_MAX) return fail(QS_ERR_INVALID, "qs_unpack_layer: too many particles");
        // the buffer enters the device in one copy; the particle rows are
        // checked there, and only a clean buffer changes the handle's state
        qs_status s = ensure_pack_space(n, m);
        if (s) return s;
        const size_t P = plane;
        int* cnt = d_pack_i;
        int* fill = cnt + P;
        int* start = fill + P;
        int32_t* ord = start + P + 1;
        int32_t* key_cell = ord + m;
        unsigned long long* bad = (unsigned long long*)(key_cell + m + 1);   // 8-byte aligned below
        bad = (unsigned long long*)(((uintptr_t)bad + 7) & ~(uintptr_t)7);
        int* nonuniform = (int*)(bad + 1);
        CK(cudaMemcpyAsync(d_pack, buf, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(cnt, 0, 2 * P * sizeof(int), st));
        const unsigned long long none = (unsigned long long)m;
        CK(cudaMemcpyAsync(bad, &none, sizeof(none), cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(nonuniform, 0, sizeof(int), st));
        UnpackArgs<T> a{};
        a.m = m; a.My = My; a.Mz = Mz; a.ncell = (int)P; a.ppc = cfg.ppc;
        a.buf = d_pack + fixed;
        a.q2m = cfg.plasma_q2m;
        a.key_cell = key_cell;
        a.cnt = cnt; a.start = start; a.fill = fill; a.ord = ord;
        a.bad = bad; a.nonuniform = nonuniform;
        a.err = d_err;
        klaunch(KC_MISC, [&] { return launch_unpack_check<T>(a, st); });
        unsigned long long first_bad = none;
        CK(cudaMemcpyAsync(&first_bad, bad, sizeof(first_bad), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (first_bad < (unsigned long long)m) {
            // the lowest bad row, reported as the reference-format check of it
            const int64_t r = (int64_t)first_bad;
            const double* pb = buf + fixed;
            const double jd = pb[r + 9 * m], kd = pb[r + 10 * m];
            if (!(jd >= 0 && jd < My && kd >= 0 && kd < Mz) || jd != (double)(int)jd ||
                kd != (double)(int)kd)
                return fail(QS_ERR_INVALID, "qs_unpack_layer: particle %lld has cell (%g, %g) "
                                            "outside the layer", (long long)r, jd, kd);
            const double yy = pb[r + 4 * m], zz = pb[r + 5 * m];
            if (!(yy >= 0 && yy <= 1 && zz >= 0 && zz <= 1))
                return fail(QS_ERR_PARTICLE_RANGE, "qs_unpack_layer: particle %lld has in-cell "
                                                   "position outside [0,1]", (long long)r);
            return fail(QS_ERR_UNSUPPORTED, "qs_unpack_layer: particle %lld is not of the "
                                            "plasma electron species", (long long)r);
        }
        if (!front_src && (s = alloc(&front_src, 4 * plane, "received layer"))) return s;
        if (!front_beam && (s = alloc(&front_beam, 2 * plane, "received layer"))) return s;
        if ((s = ensure_plasma(m))) return s;
        if (grp.flip) swap_sets();   // the march graph starts from the first set
        a.cell = pcell;
        a.y = py; a.z = pz; a.px = ppx; a.py = ppy; a.pz = ppz; a.w = pw;
        klaunch(KC_MISC, [&] { return launch_unpack_order<T>(a, st); });
        // the planes: Bx By Bz Ex Ey Ez into the front layer's fields, Jx Jy
        // Jz Rho into its sources, fftJxBeamHydro / fftRhoBeamHydro
        const int fdst[6] = {3, 4, 5, 0, 1, 2};
        for (int f = 0; f < 6; f++)
            klaunch(KC_MISC, [&] {
                return launch_convert<T>(d_pack + (size_t)f * P, 1, f3layer(L) + (size_t)fdst[f] * P,
                                         P, st);
            });
        klaunch(KC_MISC, [&] {
            return launch_convert<T>(d_pack + 6 * P, 1, front_src, 4 * P, st);
        });
        klaunch(KC_MISC, [&] { return launch_convert<T>(d_pack + 11 * P, 1, front_beam, P, st); });
        klaunch(KC_MISC, [&] {
            return launch_convert<T>(d_pack + 10 * P, 1, front_beam + P, P, st);
        });
        int nonu = 1;
        CK(cudaMemcpyAsync(&nonu, nonuniform, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        {
            const qs_status s0 = check_device();
            if (s0) return s0;
        }
        np = m;
        uniform_layout = m == (int64_t)plane * cfg.ppc && !nonu;
        if ((s = cic_fresh_front())) return s;
        front_pending = true;
        front_layer = true;
        front_used = false;
        return QS_OK;
    }

    // device space of the hand-off buffer (n doubles) and its ordering
    // scratch for m particles: counts, fill cursors, offsets, order, the
    // rows' cells and two status words
    qs_status ensure_pack_space(int64_t n, int64_t m) {
        const size_t ints = 3 * plane + 1 + 2 * (size_t)m + 8;
        if ((size_t)n > pack_cap || ints > pack_icap) {
            if (d_pack) cudaFree(d_pack);
            if (d_pack_i) cudaFree(d_pack_i);
            d_pack = nullptr;
            d_pack_i = nullptr;
            pack_cap = pack_icap = 0;
            qs_status s = alloc(&d_pack, (size_t)n, "hand-off buffer");
            if (!s) s = alloc(&d_pack_i, ints, "hand-off buffer order");
            if (s) return s;
            pack_cap = (size_t)n;
            pack_icap = ints;
        }
        return QS_OK;
    }

    // Write the density of the spectral maps for the march that follows into
    // dens_dev (in stream order, outside any captured graph).
    qs_status set_march_density() {
        const double d = march_density();
        if (d == dens_set) return QS_OK;
        klaunch(KC_MISC, [&] { return launch_set_value<T>(dens_dev, (T)d, st); });
        CK(cudaGetLastError());
        dens_set = d;
        return QS_OK;
    }

    qs_status march() override {
        if (qs_status s0 = set_march_density()) return s0;
        if (qs_status s0 = take_front_layer()) return s0;
        if (!front_pending) {
            qs_status s = seed_front(step_count);
            if (s) return s;
        }
        front_pending = false;
        if (!sb3_valid) {
            qs_status s = beam_spectra();
            if (s) return s;
        }
        if (!cfg.use_graph || prof) {
            qs_status s = march_device();
            ck_valid = !s && ck_every > 0 && !front_layer;
            return s;
        }
        if (gexec && graph_front != front_layer) {   // the head layer's set-up differs
            cudaGraphExecDestroy(gexec);
            gexec = nullptr;
        }
        if (!gexec) {
            graph_front = front_layer;
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            capturing = true;
            capture_count = 0;
            qs_status s = march_device();
            capturing = false;
            cudaError_t e = cudaStreamEndCapture(st, &g);
            if (s) {
                if (g) cudaGraphDestroy(g);
                return s;
            }
            if (e != cudaSuccess) return cuda_fail(e, "march capture");
            e = cudaGraphInstantiate(&gexec, g, cudaGraphInstantiateFlagUseNodePriority);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                gexec = nullptr;
                return cuda_fail(e, "march graph instantiate");
            }
            graph_kernels = capture_count;
            graph_end = HostState{Pf, Cf, Psrc, Csrc, cur, grp};
        }
        CK(cudaGraphLaunch(gexec, st));
        ck_valid = ck_every > 0 && !front_layer;
        launches += graph_kernels;
        Pf = graph_end.Pf; Cf = graph_end.Cf; Psrc = graph_end.Psrc; Csrc = graph_end.Csrc;
        cur = graph_end.cur;
        if (graph_end.grp.flip != grp.flip) swap_sets();
        grp = graph_end.grp;
        p_valid = true;
        marched = true;
        tail_ready = true;
        return QS_OK;
    }

    // ------------------------------------------------------------ adjoint
    // Checkpoint m holds the state entering layer L-1-m*K: the plasma
    // particles (y, z, px, py, pz, and their weights, which the regrouping
    // carries along) and the P-bank spectra (Rho, Ex, Ey, Ez, Jx, Jy, Jz);
    // the P-layer fields are layer L-m*K of the field store.
    size_t ck_stride() const { return 6 * (size_t)adj_np + 7 * plane; }
    size_t seg_stride() const { return 5 * (size_t)adj_np + (size_t)(nIter + 1) * 6 * plane; }
    T* particle_arrays(int c) { T* a[5] = {py, pz, ppx, ppy, ppz}; return a[c]; }

    qs_status save_checkpoint(int m) {
        if (m >= ck_count || np != adj_np) return fail(QS_ERR_STATE, "checkpoint storage");
        join_sides();   // the regrouped plasma
        T* dst = ck + (size_t)m * ck_stride();
        for (int c = 0; c < 5; c++)
            CK(cudaMemcpyAsync(dst + (size_t)c * np, particle_arrays(c), np * sizeof(T),
                               cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(dst + 5 * (size_t)np, pw, np * sizeof(T), cudaMemcpyDeviceToDevice,
                           st));
        const int pb = cur ^ 1;
        T* b = dst + 6 * (size_t)np;
        CK(cudaMemcpyAsync(b, bankp(pb, SP_RHO), 4 * plane * sizeof(T), cudaMemcpyDeviceToDevice,
                           st));
        CK(cudaMemcpyAsync(b + 4 * plane, bankp(pb, SP_JX), 3 * plane * sizeof(T),
                           cudaMemcpyDeviceToDevice, st));
        if (cic_adj) {   // CIC: the cells move, and the plasma is regrouped (ids)
            CK(cudaMemcpyAsync(ck_cell + (size_t)m * np, pcell, np * sizeof(int32_t),
                               cudaMemcpyDeviceToDevice, st));
            if (cic_sort)
                CK(cudaMemcpyAsync(ck_id + (size_t)m * np, pid, np * sizeof(int32_t),
                                   cudaMemcpyDeviceToDevice, st));
        }
        return QS_OK;
    }

    qs_status restore_checkpoint(int m) {
        const T* src = ck + (size_t)m * ck_stride();
        for (int c = 0; c < 5; c++)
            CK(cudaMemcpyAsync(particle_arrays(c), src + (size_t)c * np, np * sizeof(T),
                               cudaMemcpyDeviceToDevice, st));
        // the weights in this checkpoint's particle order (the plasma may
        // have been regrouped since)
        CK(cudaMemcpyAsync(pw, src + 5 * (size_t)np, np * sizeof(T), cudaMemcpyDeviceToDevice,
                           st));
        const int pb = cur ^ 1;
        const T* b = src + 6 * (size_t)np;
        CK(cudaMemcpyAsync(bankp(pb, SP_RHO), b, 4 * plane * sizeof(T), cudaMemcpyDeviceToDevice,
                           st));
        CK(cudaMemcpyAsync(bankp(pb, SP_JX), b + 4 * plane, 3 * plane * sizeof(T),
                           cudaMemcpyDeviceToDevice, st));
        if (cic_adj) {
            CK(cudaMemcpyAsync(pcell, ck_cell + (size_t)m * np, np * sizeof(int32_t),
                               cudaMemcpyDeviceToDevice, st));
            if (cic_sort) {
                CK(cudaMemcpyAsync(pid, ck_id + (size_t)m * np, np * sizeof(int32_t),
                                   cudaMemcpyDeviceToDevice, st));
                // the recomputation keeps this order (no regrouping): fresh
                // counts and offsets for it
                CK(cudaMemsetAsync(cic_cnt, 0, plane * sizeof(int), st));
                grp.grouped = true;
                grp.off_valid = false;
                grp.counted = false;
                grp.since = 0;
            }
        }
        return QS_OK;
    }

    qs_status adjoint_checkpoints(int every) override {
        if (every < 0) return fail(QS_ERR_INVALID, "qs_adjoint_checkpoints: every must be >= 0");
        if (every > 0 && S != 1)
            return fail(QS_ERR_UNSUPPORTED, "the adjoint supports NxSplit = 1");
        // the push adjoint indexes the planes and per-particle arrays with 32-bit offsets
        if (every > 0 && (6 * (uint64_t)plane >= (1ull << 31) || 3 * (uint64_t)np >= (1ull << 31)))
            return fail(QS_ERR_UNSUPPORTED, "the adjoint needs 6 ny nz and 3 x the particle count "
                                            "below 2^31");
        CK(cudaStreamSynchronize(st));
        void* old[] = {ck, seg, lam, lam_pm, lam_sb, d_dloss, ck_cell, ck_id, seg_cell,
                       lam_pos, adj_inv, adj_tmp, fstore};
        for (void* p : old)
            if (p) cudaFree(p);
        ck = seg = lam = lam_pm = lam_sb = d_dloss = lam_pos = adj_tmp = fstore = nullptr;
        lam_lo = -1;
        ck_cell = ck_id = seg_cell = adj_inv = nullptr;
        ck_every = 0;
        ck_valid = false;
        if (gexec) {   // the captured march has (or lacks) the checkpoint copies
            cudaGraphExecDestroy(gexec);
            gexec = nullptr;
        }
        drop_adjoint_graph();
        if (every == 0) return QS_OK;
        if (np <= 0) return fail(QS_ERR_STATE, "qs_adjoint_checkpoints: no plasma loaded");
        const int K = std::min(every, L);
        adj_np = np;
        ck_count = (L + K - 1) / K;
        qs_status s;
        if ((s = alloc(&ck, (size_t)ck_count * ck_stride(), "adjoint checkpoints"))) return s;
        if ((s = alloc(&seg, (size_t)K * seg_stride(), "adjoint segment"))) return s;
        if ((s = alloc(&lam, (size_t)LAM_N * plane, "adjoint planes"))) return s;
        if ((s = alloc(&lam_pm, 3 * (size_t)np, "adjoint momenta"))) return s;
        if ((s = alloc(&d_dloss, (size_t)L, "loss gradient"))) return s;
        cic_adj = cfg.shape == QS_SHAPE_CIC;
        if (cic_adj) {
            if ((s = alloc(&ck_cell, (size_t)ck_count * np, "adjoint checkpoints"))) return s;
            if ((s = alloc(&seg_cell, (size_t)K * np, "adjoint segment"))) return s;
            if ((s = alloc(&lam_pos, 2 * (size_t)np, "adjoint positions"))) return s;
            if (cic_sort) {
                if ((s = alloc(&ck_id, (size_t)ck_count * np, "adjoint checkpoints"))) return s;
                if ((s = alloc(&adj_inv, (size_t)np, "adjoint reorder"))) return s;
                if ((s = alloc(&adj_tmp, 5 * (size_t)np, "adjoint reorder"))) return s;
            }
        }
        fstore_n = 0;
        if (cic_sort && fstore_cap != 0 && !fp32_study) {
            // as many head layers as leave a sixteenth of the device free
            // (for the adjoint's own buffers, allocated when it first runs)
            const size_t per = (size_t)(nIter + 1) * 6 * plane * sizeof(T);
            size_t fr = 0, tot = 0;
            if (cudaMemGetInfo(&fr, &tot) == cudaSuccess && fr > tot / 16) {
                const size_t fit = (fr - tot / 16) / per;
                size_t cap = std::min<size_t>((size_t)L, fit);
                if (fstore_cap > 0) cap = std::min<size_t>(cap, (size_t)fstore_cap);
                const int n = (int)cap;
                if (n >= K) {   // at least one whole segment
                    if ((s = alloc(&fstore, (size_t)n * per / sizeof(T), "adjoint field store")))
                        return s;
                    fstore_n = n;
                }
            }
        }
        ck_every = K;
        return QS_OK;
    }

    bool fstore_ok() const { return fstore && ck_every > 0 && cic_sort && !src3 && !fp32_study; }
    // the store holds layers L - fstore_n .. L - 1, the head layer first
    bool fstored(int layer) const { return fstore_ok() && layer >= L - fstore_n; }
    T* fstore_at(int layer, int q) {
        return fstore + ((size_t)(L - 1 - layer) * (nIter + 1) + q) * 6 * plane;
    }

    // adjoint work planes
    enum { LAM_C = 0,          // 7: adjoint of this layer's final bank (Rho, Ex..Ez, Jx..Jz)
           LAM_P = 7,          // 7: adjoint of this layer's P-bank inputs
           LAM_CF = 14,        // 6: adjoint of this layer's final fields (field store layer i)
           LAM_PF = 20,        // 6: adjoint of the P-layer fields (layer i+1)
           LAM_CX = 26,        // 6: adjoint of an intermediate C-layer field set
           LAM_SPEC = 32,      // 6: adjoint of E, B spectra
           LAM_J = 38,         // 3: adjoint of the J spectra
           LAM_D = 41,         // 3: adjoint of the real deposit Jx, Jy, Jz
           LAM_RHO0 = 44,      // 2: adjoint of rho_old along the corrector chain
           LAM_N = 46 };
    // The C and P banks (and the CF and PF field sets) swap roles from one
    // layer to the next: the P side of layer i is the C side of layer i+1.
    int adj_par = 0;
    T* lamp(int i) {
        if (adj_par) {
            if (i < LAM_P) i += 7;
            else if (i < LAM_CF) i -= 7;
            else if (i < LAM_PF) i += 6;
            else if (i < LAM_CX) i -= 6;
        }
        return lam + (size_t)i * plane;
    }
    T* lam_sbp(int layer, int q) { return lam_sb + ((size_t)(layer - lam_lo) * 2 + q) * plane; }

    // save the particles (and cells) entering layer i into the segment's slot
    void save_entry(T* slot, int i, int c) {
        StateCopy<T> sc{};
        for (int q = 0; q < 5; q++) {
            sc.src[q] = particle_arrays(q);
            sc.dst[q] = slot + (size_t)q * np;
        }
        if (cic_adj) {
            sc.csrc = pcell;
            sc.cdst = seg_cell + (size_t)(c - i) * np;
        }
        sc.n = np;
        klaunch(KC_MISC, [&] { return launch_save_state<T>(sc, st); });
    }

    // with the field store: recompute the particles entering layers c .. lo
    // of one segment from its checkpoint by the full pushes alone, each
    // gathering the fields the march stored for it (its deposit is not read)
    qs_status recompute_states(int m, int c, int lo) {
        in_march = true;
        adj_recompute = true;
        qs_status s = restore_checkpoint(m);
        for (int i = c; !s && i >= lo; i--) {
            save_entry(seg + (size_t)(c - i) * seg_stride(), i, c);
            if (i > lo) {
                push_fields = fstore_at(i, nIter);
                s = push(i, 0, 1);
            }
        }
        push_fields = nullptr;
        in_march = false;
        adj_recompute = false;
        return s;
    }

    // recompute the layers c .. lo of one segment from its checkpoint, storing
    // each layer's entry particles and intermediate C fields
    qs_status recompute_segment(int m, int c, int lo) {
        in_march = true;
        adj_recompute = true;
        // the forward's side stream for the last z-pass of a layer and its
        // fused next predictor (the plasma is not regrouped here)
        side_z = !prof && !fp32_study && (fft_maps() || fftx64) && S == 1 && !src3;
        pred_next = -1;
        next_avg = half_avg = false;
        fuse_lo = lo;
        qs_status s = restore_checkpoint(m);
        for (int i = c; !s && i >= lo; i--) {
            T* slot = seg + (size_t)(c - i) * seg_stride();
            save_entry(slot, i, c);   // the layer's entry particles (and cells), in one launch
            T* fs = slot + 5 * (size_t)np;
            if ((s = layer_begin(i, 0))) break;
            if ((s = guess(i, 0))) break;
            join_sides();   // P: the previous layer's last z-pass
            // each push's gathered fields (P + C) / 2, for its adjoint: the
            // grouped push writes them itself
            auto gathered = [&](T* out) {
                if (cic_sort && clear_by_maps()) push_favg = out;
                else klaunch(KC_MISC, [&] { return launch_avg_planes<T>(Pf, Cf, out, 6 * plane, st); });
            };
            gathered(fs);
            for (int it = 0; it < nIter && !s; it++) {
                if ((s = push(i, 0, 0))) break;
                if ((s = iterate(i, 0, it, nullptr))) break;
                gathered(fs + (size_t)(it + 1) * 6 * plane);
            }
            if (s) break;
            if ((s = push(i, 0, 1))) break;
            if ((s = iterate(i, 0, -1, nullptr))) break;
            if ((s = layer_end(i, 0))) break;
        }
        join_sides();
        side_z = false;
        pred_next = -1;
        next_avg = half_avg = false;
        fuse_lo = 0;
        push_favg = nullptr;
        in_march = false;
        adj_recompute = false;
        return s;
    }

    // transform `nf` adjoint planes in place of the spectral adjoint: out = scale T(in)
    void adj_xform(const T* in, T* out, int nf, const int* kz, const int* ky, T scale) {
        T* outs[6];
        for (int f = 0; f < nf; f++) outs[f] = out + (size_t)f * plane;
        xform(job_stack(in, nf, outs, kz, ky, scale));
    }

    AdjSpecArgs<T> adj_args(int iLayer) {
        const SpecArgs<T> f = spec_args(iLayer, 0);
        AdjSpecArgs<T> a{};
        a.ny = My; a.nz = Mz;
        a.piY = f.piY; a.piZ = f.piZ; a.hx = f.hx; a.dens_p = f.dens_p;
        a.lRb0 = lam_sbp(iLayer, 0); a.lRb1 = lam_sbp(iLayer + 1, 0);
        a.lJxb0 = lam_sbp(iLayer, 1); a.lJxb1 = lam_sbp(iLayer + 1, 1);
        a.wb0 = f.wb0; a.wb1 = f.wb1;
        a.lRbp0 = lam_sbp(std::min(iLayer + 1, L), 0);
        a.lRbp1 = lam_sbp(std::min(iLayer + 2, L), 0);
        a.wp0 = f.wp0; a.wp1 = f.wp1;
        return a;
    }

    PushAdjArgs<T> push_adj_args(const T* slot, const int32_t* slot_cell, const T* fields,
                                 int full) {
        PushAdjArgs<T> a{};
        a.n = np; a.My = My; a.Mz = Mz;
        a.invMy = 1.0f / (float)My;
        a.cell = cic_adj ? slot_cell : pcell;   // NGP: the seeded cells never change
        a.lamPos = lam_pos;
        a.y = slot; a.z = slot + np; a.px = slot + 2 * np; a.py = slot + 3 * np;
        a.pz = slot + 4 * np; a.w = pw;
        a.F = fields;
        a.lamD = lamp(LAM_D);
        a.lamPm = lam_pm;
        a.lamFC = lamp(LAM_CX);
        a.plane = plane;
        a.sE = (T)(cfg.plasma_q2m * cfg.hx / 2.0);
        a.hxhy = (T)(cfg.hx / cfg.hy); a.hxhz = (T)(cfg.hx / cfg.hz);
        a.djx0 = (T)cfg.plasma_djx0; a.djy0 = (T)cfg.plasma_djy0; a.djz0 = (T)cfg.plasma_djz0;
        a.bxe = (T)cfg.bx_ext; a.bye = (T)cfg.by_ext; a.bze = (T)cfg.bz_ext;
        a.full = full;
        a.precise = sizeof(T) == 4;
        return a;
    }

    // reverse sweep over one layer (the transpose of move_split_layer)
    int push_adjoint(const PushAdjArgs<T>& a) {
        return cic_adj ? launch_push_adjoint_cic<T>(a, st) : launch_push_adjoint<T>(a, st);
    }

    // the adjoint of [inverse transforms of E, B] <- map <- [forward transform
    // of J] with the map between the halves of the transforms: z-pass of the
    // six field adjoints at `lf`, y-pass + the map's adjoint (+ the y-pass of
    // the current adjoints) per z-mode row, then their z-pass into LAM_D
    // In the z-pass that reads the field adjoints at lf: with `push_share`
    // (lf is a push's LAM_CX) they are also added to LAM_PF, the P layer's
    // share; with `clear` lf is zeroed once read (LAM_CX for the next push,
    // LAM_CF for its turn as the next layer's LAM_PF).
    void adj_map_fused(T* lf, const AdjSpecArgs<T>& a, bool correct, bool push_share, bool clear) {
        adj_zpass_fields(lf, push_share, clear, scratch);
        adj_rows_then_j(a, correct, scratch);
    }
    // its first part: the z-pass of the six field adjoints into `work`
    void adj_zpass_fields(T* lf, bool push_share, bool clear, T* work) {
        if constexpr (sizeof(T) == 4) {
            const int EBz[6] = {CC, CC, SS, SS, SS, CC};
            const float* ins[6];
            float* outs[6];
            float* acc[6];
            float* clr[6];
            for (int f = 0; f < 6; f++) {
                ins[f] = lf + (size_t)f * plane;
                outs[f] = work + (size_t)f * plane;
                acc[f] = lamp(LAM_PF + f);
                clr[f] = lf + (size_t)f * plane;
            }
            klaunch(KC_GEMM, [&] {
                return fftx->run_cols(6, ins, outs, EBz, inv_scale(), st, push_share ? acc : nullptr,
                                      clear ? clr : nullptr);
            });
        }
    }
    // its second part: the map adjoint rows on `work` and the z-pass of the
    // current adjoints into LAM_D
    void adj_rows_then_j(const AdjSpecArgs<T>& a, bool correct, T* work) {
        if constexpr (sizeof(T) == 4) {
            const int Jz[3] = {CC, CC, SS};
            klaunch(KC_SPECTRAL, [&] { return fftx->run_adjoint_rows(a, correct, work, work, st); });
            if (correct) {
                const float* ji[3] = {work, work + plane, work + 2 * plane};
                float* jo[3] = {lamp(LAM_D), lamp(LAM_D + 1), lamp(LAM_D + 2)};
                klaunch(KC_GEMM, [&] { return fftx->run_cols(3, ji, jo, Jz, 1.f, st); });
            }
        }
    }

    // fs: the fields each push of the layer gathered, 6 planes per push
    qs_status adjoint_layer(int i, const T* slot, const int32_t* slot_cell, const T* fs) {
        const int EBz[6] = {CC, CC, SS, SS, SS, CC}, EBy[6] = {CC, SS, CC, SS, CC, SS};
        const int Jz[3] = {CC, CC, SS}, Jy[3] = {CC, SS, CC};
        const T sc = inv_scale();
        Pf = f3layer(i + 1);
        // LAM_PF gathers this layer's shares from zero (on the fused path the
        // first map cleared it in the previous layer, as its LAM_CF)
        if (!adj_fused()) CK(cudaMemsetAsync(lamp(LAM_PF), 0, 6 * plane * sizeof(T), st));
        klaunch(KC_MISC, [&] {
            return launch_add_point<T>(lamp(LAM_CF), (size_t)(My / 2) + (size_t)My * (Mz / 2),
                                       d_dloss, i, st);
        });
        // final Iterate: C fields <- inverse transforms of its E, B
        if (!adj_fused()) adj_xform(lamp(LAM_CF), lamp(LAM_SPEC), 6, EBz, EBy, sc);
        {
            AdjSpecArgs<T> a = adj_args(i);
            a.lRho = lamp(LAM_C + 0);
            for (int c = 0; c < 3; c++) {
                a.lE[c] = lamp(LAM_SPEC + c);
                a.lEb[c] = lamp(LAM_C + 1 + c);
                a.lB[c] = lamp(LAM_SPEC + 3 + c);
                a.lJb[c] = lamp(LAM_C + 4 + c);
                a.lJ[c] = lamp(LAM_J + c);
            }
            a.lRhoOld = lamp(LAM_RHO0);
            for (int f = 0; f < 7; f++) a.lP[f] = lamp(LAM_P + f);
            a.lP_set = 1;
            if (adj_fused()) {
                // beside a pending predictor adjoint of the previous layer
                // (on the side stream, in scratch) the field z-pass uses
                // scratch2; the rows need that predictor adjoint's LAM_C
                T* work = adj_pred_pending ? scratch2 : scratch;
                adj_pred_pending = false;
                adj_zpass_fields(lamp(LAM_CF), false, true, work);
                join_sides();
                adj_rows_then_j(a, true, work);
            } else {
                klaunch(KC_SPECTRAL, [&] { return launch_corrector_adjoint<T>(a, st); });
                adj_xform(lamp(LAM_J), lamp(LAM_D), 3, Jz, Jy, T(1));
            }
        }
        // the push field adjoints (LAM_CX) start from zero; on the fused path
        // the z-pass that reads them clears them and adds the P layer's share
        if (!adj_fused()) CK(cudaMemsetAsync(lamp(LAM_CX), 0, 6 * plane * sizeof(T), st));
        klaunch(KC_PUSH, [&] {
            return push_adjoint(push_adj_args(slot, slot_cell, fs + (size_t)nIter * 6 * plane, 1));
        });
        // the P layer's field adjoint gathers every push's share
        if (!adj_fused())
            klaunch(KC_MISC, [&] {
                return launch_add_planes<T>(lamp(LAM_PF), lamp(LAM_CX), 6 * plane, st);
            });
        int rho_in = LAM_RHO0;
        for (int it = nIter - 1; it >= 0; it--) {
            if (!adj_fused()) adj_xform(lamp(LAM_CX), lamp(LAM_SPEC), 6, EBz, EBy, sc);
            AdjSpecArgs<T> a = adj_args(i);
            a.lRho = lamp(rho_in);
            const int rho_out = rho_in == LAM_RHO0 ? LAM_RHO0 + 1 : LAM_RHO0;
            for (int c = 0; c < 3; c++) {
                a.lE[c] = lamp(LAM_SPEC + c);
                a.lB[c] = lamp(LAM_SPEC + 3 + c);
                a.lJ[c] = lamp(LAM_J + c);
            }
            a.lRhoOld = lamp(rho_out);
            for (int f = 0; f < 7; f++) a.lP[f] = lamp(LAM_P + f);
            a.lP_set = 0;
            if (adj_fused()) {
                adj_map_fused(lamp(LAM_CX), a, true, true, true);
            } else {
                klaunch(KC_SPECTRAL, [&] { return launch_corrector_adjoint<T>(a, st); });
                adj_xform(lamp(LAM_J), lamp(LAM_D), 3, Jz, Jy, T(1));
            }
            rho_in = rho_out;
            if (!adj_fused()) CK(cudaMemsetAsync(lamp(LAM_CX), 0, 6 * plane * sizeof(T), st));
            klaunch(KC_PUSH, [&] {
                return push_adjoint(push_adj_args(slot, slot_cell, fs + (size_t)it * 6 * plane, 0));
            });
            if (!adj_fused())
                klaunch(KC_MISC, [&] {
                    return launch_add_planes<T>(lamp(LAM_PF), lamp(LAM_CX), 6 * plane, st);
                });
        }
        // Guess: C fields <- inverse transforms of the predicted E, B
        if (!adj_fused()) adj_xform(lamp(LAM_CX), lamp(LAM_SPEC), 6, EBz, EBy, sc);
        {
            AdjSpecArgs<T> a = adj_args(i);
            a.lRho = lamp(rho_in);
            for (int c = 0; c < 3; c++) {
                a.lE[c] = lamp(LAM_SPEC + c);
                a.lB[c] = lamp(LAM_SPEC + 3 + c);
            }
            for (int f = 0; f < 7; f++) a.lP[f] = lamp(LAM_P + f);
            a.lP_set = 0;
            if (adj_fused()) {
                adj_zpass_fields(lamp(LAM_CX), true, true, scratch);
                if (side_adj) {   // beside the next layer's add_point and field z-pass
                    const cudaError_t e = on_side(0, [&] { adj_rows_then_j(a, false, scratch); });
                    if (e != cudaSuccess) return cuda_fail(e, "side stream");
                    adj_pred_pending = true;
                } else {
                    adj_rows_then_j(a, false, scratch);
                }
            } else {
                klaunch(KC_SPECTRAL, [&] { return launch_predictor_adjoint<T>(a, st); });
            }
        }
        // hand the P-side adjoints to layer i+1 (its final bank and fields)
        adj_par ^= 1;
        CK(cudaGetLastError());
        return QS_OK;
    }

    // the device part of the adjoint (capturable): clear the adjoints, sweep
    // the segments from layer lo to the head, then d loss / d beam weight
    qs_status adjoint_device(int lo) {
        adj_par = 0;
        CK(cudaMemsetAsync(lam, 0, (size_t)LAM_N * plane * sizeof(T), st));
        CK(cudaMemsetAsync(lam_pm, 0, 3 * (size_t)np * sizeof(T), st));
        if (lam_pos) CK(cudaMemsetAsync(lam_pos, 0, 2 * (size_t)np * sizeof(T), st));
        CK(cudaMemsetAsync(lam_sb, 0, (size_t)(L + 1 - lam_lo) * 2 * plane * sizeof(T), st));
        int first = L + 1;   // lowest beam-spectrum layer the sweep touches
        if (lo >= 0) {
            const int K = ck_every;
            const int mlo = (L - 1 - lo) / K;
            for (int m = mlo; m >= 0; m--) {
                const int c = L - 1 - m * K;
                const int end = std::max(c - K + 1, lo);
                if (m < mlo && cic_adj && cic_sort) {
                    // the particle adjoints are in checkpoint m+1's order (the
                    // forward regrouped the plasma since checkpoint m): carry
                    // them to checkpoint m's order, which the recomputation keeps
                    CK(cudaMemcpyAsync(adj_tmp, lam_pm, 3 * (size_t)np * sizeof(T),
                                       cudaMemcpyDeviceToDevice, st));
                    CK(cudaMemcpyAsync(adj_tmp + 3 * (size_t)np, lam_pos,
                                       2 * (size_t)np * sizeof(T), cudaMemcpyDeviceToDevice, st));
                    klaunch(KC_MISC, [&] {
                        return launch_permute_adjoint<T>(ck_id + (size_t)(m + 1) * np,
                                                         ck_id + (size_t)m * np, np, adj_inv,
                                                         adj_tmp, lam_pm, 3, st);
                    });
                    klaunch(KC_MISC, [&] {
                        return launch_permute_adjoint<T>(ck_id + (size_t)(m + 1) * np,
                                                         ck_id + (size_t)m * np, np, adj_inv,
                                                         adj_tmp + 3 * (size_t)np, lam_pos, 2,
                                                         st);
                    });
                }
                cur = 0;
                const bool stored = fstored(end);   // then every layer of the segment
                qs_status s = stored ? recompute_states(m, c, end) : recompute_segment(m, c, end);
                if (s) return s;
                side_adj = !prof && !fp32_study && adj_fused();
                adj_pred_pending = false;
                for (int i = end; i <= c && !s; i++) {
                    const int32_t* sc = cic_adj ? seg_cell + (size_t)(c - i) * np : nullptr;
                    const T* slot = seg + (size_t)(c - i) * seg_stride();
                    s = adjoint_layer(i, slot, sc, stored ? fstore_at(i, 0) : slot + 5 * (size_t)np);
                }
                join_sides();   // the next recomputation rewrites what the sweep reads
                side_adj = adj_pred_pending = false;
                if (s) return s;
            }
            first = lo;
        }
        // beam spectra adjoint -> real beam-current adjoint (layers first..L;
        // the rest is zero) -> d loss / d w
        // (in place: lam_sb holds layers lam_lo..L; the sweep wrote layers
        // first..L, and every layer below lam_lo is zero)
        if (first <= L)
            batched_cc(lam_sbp(first, 0), lam_sbp(first, 0), 2 * (L + 1 - first), KC_GEMM);
        BeamGradArgs<T> g{};
        g.n = nb; g.L = L; g.My = My; g.Mz = Mz;
        g.lo = first <= L ? lam_lo : L + 1;
        g.bi = bi; g.bj = bj; g.bk = bk;
        g.x = bx; g.y = by; g.z = bz; g.px = bpx; g.py = bpy; g.pz = bpz;
        g.lb3 = lam_sb;
        g.plane = plane;
        g.polarity = cfg.beam_polarity;
        g.out = d_gradw;
        klaunch(KC_BEAM_PUSH, [&] { return launch_beam_weight_grad<T>(g, st); });
        CK(cudaGetLastError());
        return QS_OK;
    }

    qs_status adjoint(const double* dloss, double* dw) override {
        if (!dloss || !dw) return fail(QS_ERR_INVALID, "qs_adjoint: null pointer");
        if (ck_every <= 0) return fail(QS_ERR_STATE, "qs_adjoint: checkpoints are off");
        if (front_layer)
            return fail(QS_ERR_UNSUPPORTED, "qs_adjoint: the march started from a received layer; "
                                            "the adjoint starts from the empty front");
        if (!ck_valid || np != adj_np)
            return fail(QS_ERR_STATE, "qs_adjoint: the last march did not store checkpoints "
                                      "for the current beam");
        int lo = -1;
        for (int i = 0; i < L && lo < 0; i++)
            if (dloss[i] != 0.0) lo = i;
        if (nb > adj_nb) {
            if (d_gradw) cudaFree(d_gradw);
            d_gradw = nullptr;
            qs_status s = alloc(&d_gradw, (size_t)nb, "beam weight gradient");
            if (s) return s;
            adj_nb = nb;
            drop_adjoint_graph();
        }
        if (nb != adj_graph_nb) drop_adjoint_graph();   // the beam count is baked in
        {
            // the beam-spectrum adjoint covers the layers the sweep reaches
            // (from the lowest layer with a nonzero loss entry to the head)
            const int need_lo = lo >= 0 ? lo : L;
            if (!lam_sb || need_lo < lam_lo) {
                if (lam_sb) cudaFree(lam_sb);
                lam_sb = nullptr;
                qs_status s = alloc(&lam_sb, (size_t)(L + 1 - need_lo) * 2 * plane,
                                    "adjoint beam spectra");
                if (s) return s;
                lam_lo = need_lo;
                drop_adjoint_graph();   // it baked the old array
            }
        }
        {
            std::vector<T> h(L);
            for (int i = 0; i < L; i++) h[i] = (T)dloss[i];
            CK(cudaMemcpyAsync(d_dloss, h.data(), L * sizeof(T), cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
        }
        if (cfg.use_graph && !prof) {
            // the sweep for this range of layers is captured once and replayed
            if (!adj_exec || adj_lo != lo) {
                if (adj_exec) cudaGraphExecDestroy(adj_exec);
                adj_exec = nullptr;
                cudaGraph_t g = nullptr;
                CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                capturing = true;
                capture_count = 0;
                g_pdl = use_pdl;
                qs_status s = adjoint_device(lo);
                g_pdl = false;
                capturing = false;
                cudaError_t e = cudaStreamEndCapture(st, &g);
                if (s) {
                    if (g) cudaGraphDestroy(g);
                    return s;
                }
                if (e != cudaSuccess) return cuda_fail(e, "adjoint capture");
                e = cudaGraphInstantiate(&adj_exec, g, cudaGraphInstantiateFlagUseNodePriority);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) {
                    adj_exec = nullptr;
                    return cuda_fail(e, "adjoint graph instantiate");
                }
                adj_lo = lo;
                adj_graph_nb = nb;
                adj_kernels = capture_count;
                adj_end = HostState{Pf, Cf, Psrc, Csrc, cur, grp};
            }
            CK(cudaGraphLaunch(adj_exec, st));
            launches += adj_kernels;
            Pf = adj_end.Pf; Cf = adj_end.Cf; Psrc = adj_end.Psrc; Csrc = adj_end.Csrc;
            cur = adj_end.cur;
        } else {
            qs_status s = adjoint_device(lo);
            if (s) return s;
        }
        if (nb > 0)
            CK(cudaMemcpyAsync(dw, d_gradw, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        ck_valid = false;   // the recomputation reused the march's working state
        return QS_OK;
    }

    // ------------------------------------------------------ raw transforms
    qs_status transform2d(int kz, int ky, int batch, const double* in, double* out) override {
        if (batch < 0 || !in || !out || (kz != CC && kz != SS) || (ky != CC && ky != SS))
            return fail(QS_ERR_INVALID, "qs_transform2d: bad arguments");
        for (int b0 = 0; b0 < batch; b0 += 4) {
            int nf = std::min(4, batch - b0);
            CK(cudaMemcpyAsync(stage_d, in + (size_t)b0 * plane, nf * plane * 8,
                               cudaMemcpyHostToDevice, st));
            klaunch(KC_MISC, [&] { return launch_convert<T>(stage_d, 1, stage, nf * plane, st); });
            T* outs[4];
            int kza[4], kya[4];
            for (int f = 0; f < nf; f++) {
                outs[f] = stage + (size_t)(4 + f) * plane;
                kza[f] = kz;
                kya[f] = ky;
            }
            xform(job_stack(stage, nf, outs, kza, kya, T(1)));
            klaunch(KC_MISC, [&] { return launch_convert_back<T>(stage + 4 * plane, stage_d, nf * plane, st); });
            CK(cudaMemcpyAsync(out + (size_t)b0 * plane, stage_d, nf * plane * 8,
                               cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        }
        CK(cudaGetLastError());
        return QS_OK;
    }

    qs_status transform2d_dev(int kz, int ky, int batch, const void* d_in, void* d_out) override {
        if (batch < 0 || !d_in || !d_out || (kz != CC && kz != SS) || (ky != CC && ky != SS))
            return fail(QS_ERR_INVALID, "qs_transform2d_dev: bad arguments");
        const T* in = (const T*)d_in;
        T* out = (T*)d_out;
        for (int b0 = 0; b0 < batch; b0 += kMaxXfFields) {
            int nf = std::min(kMaxXfFields, batch - b0);
            T* outs[kMaxXfFields];
            int kza[kMaxXfFields], kya[kMaxXfFields];
            for (int f = 0; f < nf; f++) {
                outs[f] = out + (size_t)(b0 + f) * plane;
                kza[f] = kz;
                kya[f] = ky;
            }
            xform(job_stack(in + (size_t)b0 * plane, nf, outs, kza, kya, T(1)));
        }
        CK(cudaGetLastError());
        return QS_OK;
    }
};

}  // namespace qs

using namespace qs;

struct qs_handle {
    EngineBase* e;
};

static qs_status validate(const qs_config* c, std::string& why) {
    if (!c) { why = "null config"; return QS_ERR_INVALID; }
    if (c->ny < 8 || c->nz < 8 || c->nx < 1) { why = "need ny, nz >= 8 and nx >= 1"; return QS_ERR_INVALID; }
    if (c->ny % 8 || c->nz % 8) { why = "ny and nz must be multiples of 8"; return QS_ERR_INVALID; }
    if (c->nx_split < 1 || c->n_iter < 0) { why = "nx_split >= 1 and n_iter >= 0"; return QS_ERR_INVALID; }
    if (c->ppc < 1 || c->ppc > 16) { why = "ppc must be in [1,16]"; return QS_ERR_INVALID; }
    if (!(c->hx > 0) || !(c->hy > 0) || !(c->hz > 0)) { why = "cell sizes must be > 0"; return QS_ERR_INVALID; }
    if (c->shape != QS_SHAPE_NGP && c->shape != QS_SHAPE_CIC) { why = "bad shape"; return QS_ERR_INVALID; }
    if (c->precision < QS_PREC_FP64 || c->precision > QS_PREC_FP64_FFT) { why = "bad precision"; return QS_ERR_INVALID; }
    if (!(c->wavelength > 0)) { why = "wavelength must be > 0"; return QS_ERR_INVALID; }
    return QS_OK;
}

extern "C" {

qs_status qs_config_default(qs_config* c) {
    if (!c) return QS_ERR_INVALID;
    memset(c, 0, sizeof *c);
    c->ny = c->nz = 128;
    c->nx = 256;
    c->nx_split = 1;
    c->n_iter = 1;
    c->ppc = 4;
    c->hx = c->hy = c->hz = 0.05;
    c->ts = 1.0;
    c->plasma_density = 1.0;
    c->plasma_q2m = -1.0;
    c->plasma_djx0 = c->plasma_djy0 = c->plasma_djz0 = c->plasma_drho0 = -1.0;
    c->beam_q2m = -1.0;
    c->beam_polarity = -1.0;
    c->syn_min = 100.0;
    c->wavelength = 0.001;
    c->synchrotron = 1;
    c->precision = QS_PREC_FP32;
    c->shape = QS_SHAPE_NGP;
    c->device = 0;
    c->store_sources = 0;
    c->use_graph = 1;
    c->seed = 12345;
    return QS_OK;
}

qs_status qs_create(const qs_config* cfg, qs_handle** out) {
    if (!out) return QS_ERR_INVALID;
    *out = nullptr;
    std::string why;
    qs_status s = validate(cfg, why);
    if (s) {
        g_create_error = why;
        return s;
    }
    EngineBase* e = nullptr;
    bool tc = cfg->precision >= QS_PREC_TF32X3 && cfg->precision <= QS_PREC_BF16X6;
    if (cfg->precision == QS_PREC_FP64 || cfg->precision == QS_PREC_FP64_FFT)
        e = new (std::nothrow) Engine<double>();
    else {
        auto* ef = new (std::nothrow) Engine<float>();
        if (ef) {
            ef->tc = tc;
            ef->tc_mode = cfg->precision;
        }
        e = ef;
    }
    if (!e) {
        g_create_error = "out of host memory";
        return QS_ERR_OOM;
    }
    e->cfg = *cfg;
    e->My = cfg->ny;
    e->Mz = cfg->nz;
    e->L = cfg->nx;
    e->S = cfg->nx_split;
    e->nIter = cfg->n_iter;
    e->dev = cfg->device;
    s = e->init();
    if (s) {
        g_create_error = e->err;
        delete e;
        return s;
    }
    qs_handle* h = new (std::nothrow) qs_handle{e};
    if (!h) {
        delete e;
        g_create_error = "out of host memory";
        return QS_ERR_OOM;
    }
    *out = h;
    return QS_OK;
}

qs_status qs_destroy(qs_handle* h) {
    if (!h) return QS_ERR_INVALID;
    if (h->e) {
        cudaSetDevice(h->e->dev);
        delete h->e;
    }
    delete h;
    return QS_OK;
}

const char* qs_last_error(const qs_handle* h) {
    if (!h) return g_create_error.c_str();
    return h->e->err.c_str();
}

const char* qs_status_string(qs_status s) {
    switch (s) {
        case QS_OK: return "ok";
        case QS_ERR_INVALID: return "invalid argument";
        case QS_ERR_CUDA: return "CUDA error";
        case QS_ERR_OOM: return "out of device memory";
        case QS_ERR_DEVICE: return "device error flag";
        case QS_ERR_BEAM_CURRENT: return "too large beam current";
        case QS_ERR_PARTICLE_RANGE: return "particle outside its cell";
        case QS_ERR_UNSUPPORTED: return "unsupported";
        case QS_ERR_TIMEOUT: return "device wait timed out";
        case QS_ERR_STATE: return "call out of sequence";
    }
    return "unknown status";
}

#define H_OR_INVALID(h)                   \
    if (!(h) || !(h)->e) return QS_ERR_INVALID; \
    EngineBase* E = (h)->e;               \
    if (cudaSetDevice(E->dev) != cudaSuccess) return E->fail(QS_ERR_CUDA, "cudaSetDevice failed");

qs_status qs_sync(qs_handle* h) {
    H_OR_INVALID(h);
    return E->check_device();
}

qs_status qs_get_stream(qs_handle* h, void** stream) {
    if (!h || !stream) return QS_ERR_INVALID;
    *stream = (void*)h->e->st;
    return QS_OK;
}

qs_status qs_load_beam(qs_handle* h, int64_t n, const int32_t* i, const int32_t* j,
                       const int32_t* k, const double* x, const double* y, const double* z,
                       const double* px, const double* py, const double* pz, const double* w) {
    H_OR_INVALID(h);
    return E->load_beam(n, i, j, k, x, y, z, px, py, pz, w);
}

qs_status qs_get_beam(qs_handle* h, int64_t n, int32_t* i, int32_t* j, int32_t* k, double* x,
                      double* y, double* z, double* px, double* py, double* pz, double* w) {
    H_OR_INVALID(h);
    return E->get_beam(n, i, j, k, x, y, z, px, py, pz, w);
}

int64_t qs_beam_count(const qs_handle* h) { return h ? h->e->beam_count() : -1; }

qs_status qs_load_front_plasma(qs_handle* h, int64_t n, const int32_t* cell, const double* y,
                               const double* z, const double* px, const double* py,
                               const double* pz, const double* w) {
    H_OR_INVALID(h);
    return E->load_front(n, cell, y, z, px, py, pz, w);
}

qs_status qs_seed_front_plasma(qs_handle* h, uint64_t step) {
    H_OR_INVALID(h);
    qs_status s = E->seed_front(step);
    if (s) return s;
    return E->check_device();
}

int64_t qs_plasma_count(const qs_handle* h) { return h ? h->e->plasma_count() : -1; }

qs_status qs_density_profile_default(qs_density_profile* p) {
    if (!p) return QS_ERR_INVALID;
    std::memset(p, 0, sizeof *p);
    p->distribution = 0;
    p->density = 1.0;
    p->plateau_end = p->end = 1e30;
    p->curvature_end = 1e20;   // the namelist default (elements.cpp:53)
    return QS_OK;
}

qs_status qs_set_density_profile(qs_handle* h, const qs_density_profile* p) {
    H_OR_INVALID(h);
    if (!p) {
        E->have_profile = false;
        return QS_OK;
    }
    if (p->distribution == 12 && !(p->xperiod > 0.0))
        return E->fail(QS_ERR_INVALID, "the periodic profile needs xperiod > 0");
    E->profile = *p;
    E->have_profile = true;
    return QS_OK;
}

qs_status qs_plasma_density(qs_handle* h, double x, double y, double z, double* out) {
    H_OR_INVALID(h);
    if (!out) return E->fail(QS_ERR_INVALID, "out is NULL");
    *out = E->density_at(x, y, z);
    return QS_OK;
}

qs_status qs_set_phase(qs_handle* h, double phase) {
    H_OR_INVALID(h);
    if (!std::isfinite(phase)) return E->fail(QS_ERR_INVALID, "phase must be finite");
    E->phase = phase;
    return QS_OK;
}

int64_t qs_layer_pack_size(const qs_handle* h) { return h && h->e ? h->e->pack_size() : -1; }

qs_status qs_pack_layer(qs_handle* h, double* buf, int64_t n) {
    H_OR_INVALID(h);
    qs_status s = E->pack_layer(buf, n);
    if (s) return s;
    return E->check_device();
}

qs_status qs_unpack_layer(qs_handle* h, const double* buf, int64_t n) {
    H_OR_INVALID(h);
    qs_status s = E->unpack_layer(buf, n);
    if (s) return s;
    return E->check_device();
}

qs_status qs_clear_front_layer(qs_handle* h) {
    H_OR_INVALID(h);
    qs_status s = E->clear_front_layer();
    if (s) return s;
    return E->check_device();
}

qs_status qs_get_phase(qs_handle* h, double* phase) {
    H_OR_INVALID(h);
    if (!phase) return E->fail(QS_ERR_INVALID, "phase is NULL");
    *phase = E->phase;
    return QS_OK;
}

qs_status qs_get_plasma(qs_handle* h, int64_t n, int32_t* cell, double* y, double* z, double* px,
                        double* py, double* pz, double* w) {
    H_OR_INVALID(h);
    return E->get_plasma(n, cell, y, z, px, py, pz, w);
}

qs_status qs_set_layer(qs_handle* h, int which, int field, const double* data) {
    H_OR_INVALID(h);
    return E->set_layer(which, field, data);
}
qs_status qs_get_layer(qs_handle* h, int which, int field, double* out) {
    H_OR_INVALID(h);
    return E->get_layer(which, field, out);
}
qs_status qs_get_field3d(qs_handle* h, int field, int layer, double* out) {
    H_OR_INVALID(h);
    return E->get_field3d(field, layer, out);
}
qs_status qs_set_beam_currents(qs_handle* h, int field, int layer, const double* data) {
    H_OR_INVALID(h);
    return E->set_beam_currents(field, layer, data);
}
qs_status qs_get_beam_currents(qs_handle* h, int field, int layer, double* out) {
    H_OR_INVALID(h);
    return E->get_beam_currents(field, layer, out);
}
qs_status qs_get_onaxis_ex(qs_handle* h, double* out) {
    H_OR_INVALID(h);
    return E->get_onaxis(out);
}
qs_status qs_save_fields(qs_handle* h, const char* path) {
    H_OR_INVALID(h);
    return E->save_output(path, false);
}
qs_status qs_save_movie_frame(qs_handle* h, const char* path) {
    H_OR_INVALID(h);
    return E->save_output(path, true);
}

qs_status qs_get_charge_sums(qs_handle* h, double* rho, double* jx, double* rho_beam) {
    H_OR_INVALID(h);
    return E->get_charge_sums(rho, jx, rho_beam);
}

qs_status qs_selftest_wait_limit(qs_handle* h, unsigned tries) {
    H_OR_INVALID(h);
    if (tries == 0 || tries > (1u << 22))
        return E->fail(QS_ERR_INVALID, "qs_selftest_wait_limit: tries must be in [1, 2^22]");
    qs_status s = E->check_device();   // earlier errors first
    if (s) return s;
    launch_wait_limit_probe(E->d_err, tries, E->st);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return E->cuda_fail(e, "wait-limit probe launch");
    return E->check_device();          // QS_ERR_TIMEOUT, and the flag cleared
}

qs_status qs_get_psi(qs_handle* h, double* out) {
    H_OR_INVALID(h);
    if (!out) return QS_ERR_INVALID;
    std::vector<double> ex(E->L);
    qs_status s = E->get_onaxis(ex.data());
    if (s) return s;
    // psi(nx) = 0 ahead of the box; trapezoid in xi towards the tail
    double psi = 0.0, prev = 0.0;
    for (int i = E->L - 1; i >= 0; i--) {
        psi += E->cfg.hx * 0.5 * (ex[i] + prev);
        out[i] = psi;
        prev = ex[i];
    }
    return QS_OK;
}

qs_status qs_step(qs_handle* h) {
    H_OR_INVALID(h);
    E->phase += E->cfg.ts;   // step.cpp:33
    qs_status s = E->move_beam();
    if (s) return s;
    s = E->march();
    if (s) return s;
    E->step_count++;
    return E->check_device();
}

qs_status qs_move_beam_particles(qs_handle* h) {
    H_OR_INVALID(h);
    qs_status s = E->move_beam();
    if (s) return s;
    return E->check_device();
}

qs_status qs_move_all_split_layers(qs_handle* h) {
    H_OR_INVALID(h);
    qs_status s = E->march();
    if (s) return s;
    E->step_count++;
    return E->check_device();
}

qs_status qs_begin_march(qs_handle* h) {
    H_OR_INVALID(h);
    qs_status s = E->begin_march();
    if (s) return s;
    return E->check_device();
}
qs_status qs_layer_begin(qs_handle* h, int iLayer, int iSplit) {
    H_OR_INVALID(h);
    qs_status s = E->layer_begin(iLayer, iSplit);
    if (s) return s;
    return E->check_device();
}
qs_status qs_move_split_layer(qs_handle* h, int iLayer, int iSplit) {
    H_OR_INVALID(h);
    if (iLayer < 0 || iLayer >= E->L || iSplit < 0 || iSplit >= E->S) return QS_ERR_INVALID;
    qs_status s = E->move_split_layer(iLayer, iSplit);
    if (s) return s;
    return E->check_device();
}
qs_status qs_guess_fields(qs_handle* h, int iLayer, int iSplit) {
    H_OR_INVALID(h);
    if (iLayer < 0 || iLayer >= E->L || iSplit < 0 || iSplit >= E->S) return QS_ERR_INVALID;
    qs_status s = E->guess(iLayer, iSplit);
    if (s) return s;
    return E->check_device();
}
qs_status qs_move_particles_layer(qs_handle* h, int iLayer, int iSplit, int iFullStep) {
    H_OR_INVALID(h);
    qs_status s = E->push(iLayer, iSplit, iFullStep);
    if (s) return s;
    return E->check_device();
}
qs_status qs_iterate_fields(qs_handle* h, int iLayer, int iSplit, int iter, double* rel_err) {
    H_OR_INVALID(h);
    qs_status s = E->iterate(iLayer, iSplit, iter, rel_err);
    if (s) return s;
    return E->check_device();
}
qs_status qs_layer_end(qs_handle* h, int iLayer, int iSplit) {
    H_OR_INVALID(h);
    if (iLayer < 0 || iLayer >= E->L || iSplit < 0 || iSplit >= E->S) return QS_ERR_INVALID;
    qs_status s = E->layer_end(iLayer, iSplit);
    if (s) return s;
    return E->check_device();
}

qs_status qs_transform2d(qs_handle* h, int kind_z, int kind_y, int batch, const double* in,
                         double* out) {
    H_OR_INVALID(h);
    qs_status s = E->transform2d(kind_z, kind_y, batch, in, out);
    if (s) return s;
    return E->check_device();
}

qs_status qs_transform2d_dev(qs_handle* h, int kind_z, int kind_y, int batch, const void* d_in,
                             void* d_out) {
    H_OR_INVALID(h);
    return E->transform2d_dev(kind_z, kind_y, batch, d_in, d_out);
}

qs_status qs_adjoint_checkpoints(qs_handle* h, int every) {
    H_OR_INVALID(h);
    return E->adjoint_checkpoints(every);
}

qs_status qs_adjoint(qs_handle* h, const double* dloss_donaxis_ex, double* dloss_dbeam_weight) {
    H_OR_INVALID(h);
    qs_status s = E->adjoint(dloss_donaxis_ex, dloss_dbeam_weight);
    if (s) return s;
    return E->check_device();
}

qs_status qs_step_host(qs_handle* h, int64_t n_beam, const int32_t* i, const int32_t* j,
                       const int32_t* k, const double* x, const double* y, const double* z,
                       const double* px, const double* py, const double* pz, const double* w,
                       int32_t* i_out, int32_t* j_out, int32_t* k_out, double* x_out,
                       double* y_out, double* z_out, double* px_out, double* py_out,
                       double* pz_out, double* onaxis_ex_out) {
    H_OR_INVALID(h);
    qs_status s = E->load_beam(n_beam, i, j, k, x, y, z, px, py, pz, w);
    if (s) return s;
    s = qs_step(h);
    if (s) return s;
    if (i_out || j_out || k_out || x_out || y_out || z_out || px_out || py_out || pz_out) {
        s = E->get_beam(n_beam, i_out, j_out, k_out, x_out, y_out, z_out, px_out, py_out, pz_out,
                        nullptr);
        if (s) return s;
    }
    if (onaxis_ex_out) return E->get_onaxis(onaxis_ex_out);
    return QS_OK;
}

int64_t qs_kernel_launches(const qs_handle* h) { return h ? h->e->launches : -1; }

qs_status qs_profile_enable(qs_handle* h, int on) {
    H_OR_INVALID(h);
    qs_status s = E->resolve_profile();
    if (s) return s;
    E->prof = on != 0;
    for (int c = 0; c < KC_N; c++) {
        E->prof_ms[c] = 0;
        E->prof_n[c] = 0;
    }
    return QS_OK;
}

qs_status qs_profile_read(qs_handle* h, double* ms, int64_t* launches, int n) {
    H_OR_INVALID(h);
    if (n < 0 || (n > 0 && (!ms || !launches))) return QS_ERR_INVALID;
    qs_status s = E->resolve_profile();
    if (s) return s;
    for (int c = 0; c < n && c < KC_N; c++) {
        ms[c] = E->prof_ms[c];
        launches[c] = E->prof_n[c];
        E->prof_ms[c] = 0;
        E->prof_n[c] = 0;
    }
    for (int c = KC_N; c < n; c++) {
        ms[c] = 0;
        launches[c] = 0;
    }
    return QS_OK;
}

}  // extern "C"
