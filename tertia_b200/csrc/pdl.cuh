// pdl.cuh — programmatic dependent launch for the kernels of the xi-march.
//
// A march is a long chain of dependent kernels (about 17 per layer), each
// short (5-12 us).  Launched with the programmatic-stream-serialisation
// attribute, a kernel may be scheduled before its predecessor has finished:
// its prologue (barrier set-up, TMEM allocation, descriptor prefetch, index
// math) overlaps the predecessor's tail, and pdl_wait() then blocks until the
// predecessor has completed and its memory is visible.  Every kernel launched
// through launch_pdl() calls pdl_wait() before it touches memory that an
// earlier kernel writes or reads, so the ordering is that of a plain stream.
// pdl_trigger() lets the successor be scheduled; every thread of the kernel
// calls it once its own share of the main work is issued.  Without the
// attribute both instructions are no-ops.
#pragma once
#include <cuda_runtime.h>

namespace qs {

// set by the engine around the launches of a march (per host thread)
extern thread_local bool g_pdl;

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    unsigned n = 0;
    if (g_pdl) {
        attr[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[n].val.programmaticStreamSerializationAllowed = 1;
        n++;
    }
    // the stream's priority, also as a node attribute when the launch is
    // captured into a graph
    int prio = 0;
    if (cudaStreamGetPriority(st, &prio) == cudaSuccess && prio != 0) {
        attr[n].id = cudaLaunchAttributePriority;
        attr[n].val.priority = prio;
        n++;
    }
    cfg.attrs = n ? attr : nullptr;
    cfg.numAttrs = n;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

}  // namespace qs
