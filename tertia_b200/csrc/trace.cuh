// trace.cuh — an opt-in device timeline of the march's kernels.
//
// Compiled in only with -DQS_TRACE (the separate libqsb200_trace.so that
// tertia_b200/build.py links beside libqsb200.so): thread 0 of every CTA of
// an instrumented kernel stamps %globaltimer (ns) when the CTA starts, when
// its programmatic-dependency wait returns (the predecessor has finished) and
// when it ends, and appends the three stamps with the kernel kind, the grid's
// y size, blockIdx and the SM to a ring buffer in device memory.  The ring is
// attached with qs_trace_attach (include/qsb200_trace.h); the host side that
// reads and summarises it is tertia_b200/trace.py.  Without QS_TRACE the
// macros are empty and the kernels are those of libqsb200.so.
//
// Record layout (4 x u64): t_entry, t_waited, t_end,
//   kind << 56 | gridDim.y << 48 | blockIdx.y << 40 | smid << 32 | blockIdx.x
#pragma once
#include <cuda_runtime.h>

namespace qs {
namespace trace {

// kernel kinds of the records
enum Kind : unsigned {
    K_PUSH_HALF = 1,      // grouped CIC push without particle stores
    K_PUSH_FULL = 2,      // grouped CIC push that stores the particles
    K_ZPASS = 3,          // transform along z (fft_cols_kernel)
    K_YPASS = 4,          // transform along y (fft_rows_kernel)
    K_MAP_PRED = 5,       // map kernel: predictor
    K_MAP_CORR = 6,       // map kernel: corrector
    K_MAP_CORR_PRED = 8,  // map kernel: corrector and the next layer's predictor
    K_SCAN = 10,          // regrouping: cell offsets
    K_SCATTER = 11,       // regrouping: particle scatter
};

}  // namespace trace
}  // namespace qs

#ifdef QS_TRACE
namespace qs {
namespace trace {

struct Ring {
    unsigned long long* rec;   // 4 words per record
    unsigned* pos;             // records appended so far (wraps at mask + 1)
    unsigned mask;             // ring size - 1 (a power of two)
};
// one per translation unit, set by that unit's qs_trace_set_* (below)
static __device__ Ring g_ring;

__device__ __forceinline__ unsigned long long now() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned smid() {
    unsigned s;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(s));
    return s;
}
__device__ __forceinline__ void record(unsigned kind, unsigned long long t0,
                                       unsigned long long t1) {
    if (threadIdx.x != 0 || g_ring.rec == nullptr) return;
    const unsigned p = atomicAdd(g_ring.pos, 1u) & g_ring.mask;
    unsigned long long* r = g_ring.rec + 4ull * p;
    r[0] = t0;
    r[1] = t1;
    r[2] = now();
    r[3] = ((unsigned long long)(kind & 0xffu) << 56) |
           ((unsigned long long)(gridDim.y & 0xffu) << 48) |
           ((unsigned long long)(blockIdx.y & 0xffu) << 40) |
           ((unsigned long long)(smid() & 0xffu) << 32) | (unsigned long long)blockIdx.x;
}

}  // namespace trace
}  // namespace qs

#define QS_TRACE_ENTRY() const unsigned long long qs_trace_t0 = ::qs::trace::now()
#define QS_TRACE_WAITED() const unsigned long long qs_trace_t1 = ::qs::trace::now()
#define QS_TRACE_END(kind) ::qs::trace::record((kind), qs_trace_t0, qs_trace_t1)
// the setter of a translation unit's ring (called by qs_trace_attach)
#define QS_TRACE_UNIT(name)                                                             \
    extern "C" int qs_trace_set_##name(void* rec, void* pos, unsigned mask) {           \
        const ::qs::trace::Ring r{(unsigned long long*)rec, (unsigned*)pos, mask};       \
        return (int)cudaMemcpyToSymbol(::qs::trace::g_ring, &r, sizeof(r));             \
    }
#else
#define QS_TRACE_ENTRY() \
    do {                 \
    } while (0)
#define QS_TRACE_WAITED() \
    do {                  \
    } while (0)
#define QS_TRACE_END(kind) \
    do {                   \
    } while (0)
#define QS_TRACE_UNIT(name)
#endif
