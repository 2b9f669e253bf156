// qs_common.cuh — shared types of the B200 quasi-static layer loop.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

#include "../../include/qsb200.h"

namespace qs {

// Device-side error bits (the reference's exit() sites become flags the
// host turns into qs_status values).
enum DevErr : int {
    DEV_ERR_RANGE = 1,         // particle fraction outside [0,1] (exit(-212)/exit(-12))
    DEV_ERR_BEAM_CURRENT = 2,  // |JxBeam| > 10 (exit(20))
    DEV_ERR_TIMEOUT = 4,       // a bounded device wait gave up
    DEV_ERR_INTERNAL = 8,      // an internal consistency check failed (access skipped)
};

constexpr int kMaxXfFields = 8;

// One pass of a batched half-integer transform: for every field f,
// out_f[c][r] = scale * sum_k in_f[r][k] * mat_f[k][c]  (out = (in . mat)^T),
// in_f is R x K row-major, mat_f K x K symmetric, out_f K x R row-major.
template <class T>
struct DttPassArgs {
    const T* in[kMaxXfFields];
    const T* mat[kMaxXfFields];
    T* out[kMaxXfFields];
    int R, K;
    T scale;
};

// A batched 2-D transform request (both passes).
template <class T>
struct DttJob {
    int nf = 0;
    const T* in[kMaxXfFields] = {};
    T* out[kMaxXfFields] = {};
    int kz[kMaxXfFields] = {};
    int ky[kMaxXfFields] = {};
    T scale = T(1);
};

// Transform matrices of one size n: 2 cos / 2 sin (pi (j+1/2)(k+1/2) / n).
template <class T>
struct DttMats {
    const T* m[2] = {nullptr, nullptr};  // [QS_REDFT11], [QS_RODFT11]
};

// Plasma push arguments.
template <class T>
struct PushArgs {
    int64_t n;
    int My, Mz;
    const int32_t* cell;
    T *y, *z, *px, *py, *pz;
    const T* w;
    const T* P;     // 6 planes Ex..Bz of the P layer
    const T* C;     // 6 planes Ex..Bz of the C layer
    T* dep;         // 4 planes Jx, Jy, Jz, Dens (added to)
    int32_t* cell_out;    // CIC: new cell on the full step (may alias cell)
    int32_t* dep_cell;    // optional: folded cell of the last deposit
    size_t plane;
    T hx, hy, hz, q2m, djx0, djy0, djz0, drho0, bxe, bye, bze;
    T sE, hxhy, hxhz;     // q2m*hx/2, hx/hy, hx/hz (factored FP32 form)
    float invMy;          // 1/My for the cell index split
    int uniform_ppc;      // >0: particle p sits in cell p / uniform_ppc (lattice layout)
    // FP32 CIC over particles grouped by cell: cell c holds particles
    // loff[c] + bpref[c / 1024] .. (next cell's offset) - 1; the full push
    // counts the new cells into cnt
    const int* loff;
    const int* bpref;
    int* cnt;
    int skip_dens;        // 1: leave out the density deposit (plane 3), unused by the caller
    T* favg;              // grouped CIC without the density deposit: when set, the fields
                          // the push gathers, (P + C) / 2, are written here (6 planes),
                          // for the push adjoint
    int full;
    int* err;
};

}  // namespace qs
