// noalloc.cu — the FP64 2-D half-integer transform with no device allocation.
//
// Some callers cannot call cudaMalloc.  A solver plugin that lives inside a
// host framework's process often may only use device memory the framework
// hands it: the framework's caching allocator has to account for every byte,
// an allocation the plugin makes on its own can fail or evict the
// framework's cache, and cudaMalloc / cudaFree synchronise the device in the
// middle of the framework's own stream work.  qs_create allocates its
// working set, so such a caller cannot hold a qs_handle.
//
// qs_transform2d_noalloc serves them: the caller passes its input and output
// planes, and the only other device memory used is g_noalloc_scratch below,
// a fixed array of kScratchDoubles doubles (6 MiB) that the CUDA module itself
// carries.  It holds the two transform matrices and one intermediate plane,
// which bounds ny and nz to kNoAllocMaxN.  Every GPU on which this library's
// module is loaded holds that array until the process exits.
//
// In host code g_noalloc_scratch is only a host-side stand-in for the device
// array, not a device address: the device address is looked up with
// cudaGetSymbolAddress, with the device current, on the first call made on a
// device, and again only when the device's context has changed since (a
// cudaDeviceReset between calls makes the runtime load the module, and so the
// array, afresh).  A CUDA error that is already pending on the calling thread
// when the call starts belongs to the caller: the call reports it without
// clearing it and does nothing.  Every call on a device shares the one
// array, and the array keeps whatever the last call left in it.  Nothing in it
// needs to start at zero: each call writes every element it later reads
// (both matrices, then the whole intermediate plane of each batch plane).
// Calls whose GPU work overlaps (two streams, or two host threads on one
// device) race on the array and give wrong results; callers must order them.
#include <cuda.h>            // CUcontext / CUresult types only: the driver calls are
#include <cuda_runtime.h>    // fetched through cudaGetDriverEntryPointByVersion

#include <mutex>
#include <string>

#include "qs_common.cuh"
#include "qs_internal.h"

namespace qs {

void set_unbound_error(const std::string& why);   // qs_last_error(NULL) text (api.cu)

namespace {

constexpr int kNoAllocMaxN = 512;
// two matrices (ny^2 + nz^2) and one nz x ny plane at the largest size
constexpr size_t kScratchDoubles = 3 * (size_t)kNoAllocMaxN * kNoAllocMaxN;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_setup_mu;
double* g_scratch_dev[kMaxDevices] = {};          // device address per device ordinal
unsigned long long g_scratch_ctx[kMaxDevices] = {};   // id of the context it was looked up in

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

// unique id of the calling thread's current context (0 when it cannot be read)
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_cur = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {   // under g_setup_mu
        looked_up = true;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", (void**)&get_cur, 12000,
                                             cudaEnableDefault, &q1) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess)
            get_cur = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", (void**)&get_id, 12000,
                                             cudaEnableDefault, &q2) != cudaSuccess ||
            q2 != cudaDriverEntryPointSuccess)
            get_id = nullptr;
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_cur && get_id && get_cur(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, &id) == CUDA_SUCCESS)
        return id;
    return 0;
}

// 2 cos / 2 sin (pi (j+1/2)(k+1/2) / n), angle reduced exactly in integers:
// (2j+1)(2k+1) mod 8n in units of pi/(4n) (the same table the handle builds)
__global__ void noalloc_matrix_kernel(double* m, int n, int kind) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * n) return;
    const int k = idx / n, j = idx - k * n;
    const long long q = ((long long)(2 * j + 1) * (2 * k + 1)) % (8LL * n);
    const double x = (double)q / (4.0 * n);   // angle / pi, in [0, 2)
    m[idx] = 2.0 * (kind == QS_REDFT11 ? cospi(x) : sinpi(x));
}

qs_status fail(qs_status s, const std::string& why) {
    set_unbound_error("qs_transform2d_noalloc: " + why);
    return s;
}

// device address of the scratch array on the current device (set-up on the
// first call per device)
qs_status scratch_on_current_device(double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(QS_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(QS_ERR_DEVICE, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    // look the address up again when the current context is not the one it
    // was found in (or cannot be identified: 0)
    const unsigned long long ctx = current_context_id();
    if (!g_scratch_dev[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
        double* p = nullptr;
        e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(QS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_dev[dev] = p;
        g_scratch_ctx[dev] = current_context_id();   // the lookup made the context current
    }
    *out = g_scratch_dev[dev];
    return QS_OK;
}

}  // namespace
}  // namespace qs

using namespace qs;

extern "C" qs_status qs_transform2d_noalloc(int kind_z, int kind_y, int ny, int nz, int batch,
                                            const double* d_in, double* d_out, void* stream) {
    if ((kind_z != QS_REDFT11 && kind_z != QS_RODFT11) ||
        (kind_y != QS_REDFT11 && kind_y != QS_RODFT11))
        return fail(QS_ERR_INVALID, "kinds must be QS_REDFT11 or QS_RODFT11");
    if (ny < 8 || nz < 8 || ny % 8 || nz % 8)
        return fail(QS_ERR_INVALID, "ny and nz must be multiples of 8, at least 8");
    if (ny > kNoAllocMaxN || nz > kNoAllocMaxN)
        return fail(QS_ERR_INVALID, "ny = " + std::to_string(ny) + ", nz = " + std::to_string(nz) +
                                        " exceed the fixed scratch limit of " +
                                        std::to_string(kNoAllocMaxN) + " per dimension");
    if (batch < 0) return fail(QS_ERR_INVALID, "batch must be >= 0");
    if (batch == 0) return QS_OK;
    if (!d_in || !d_out) return fail(QS_ERR_INVALID, "null plane pointer");
    {
        // an error left by the caller's own earlier CUDA work stays the
        // caller's: report it, leave it in place, launch nothing
        const cudaError_t pending = cudaPeekAtLastError();
        if (pending != cudaSuccess)
            return fail(QS_ERR_CUDA, std::string("a CUDA error was already pending on this thread "
                                                 "before the call (left in place): ") +
                                         cudaGetErrorString(pending));
    }
    double* scratch = nullptr;
    qs_status s = scratch_on_current_device(&scratch);
    if (s) return s;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t plane = (size_t)ny * nz;
    double* mat_y = scratch;
    double* mat_z = mat_y + (size_t)ny * ny;
    double* inter = mat_z + (size_t)nz * nz;
    noalloc_matrix_kernel<<<(ny * ny + 255) / 256, 256, 0, st>>>(mat_y, ny, kind_y);
    noalloc_matrix_kernel<<<(nz * nz + 255) / 256, 256, 0, st>>>(mat_z, nz, kind_z);
    DttMats<double> my, mz;
    my.m[QS_REDFT11] = my.m[QS_RODFT11] = mat_y;
    mz.m[QS_REDFT11] = mz.m[QS_RODFT11] = mat_z;
    for (int b = 0; b < batch; b++) {   // one intermediate plane: one batch plane at a time
        DttJob<double> job;
        job.nf = 1;
        job.in[0] = d_in + (size_t)b * plane;
        job.out[0] = d_out + (size_t)b * plane;
        job.kz[0] = kind_z;
        job.ky[0] = kind_y;
        job.scale = 1.0;
        run_dtt_simt<double>(job, ny, nz, my, mz, inter, st);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(QS_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return QS_OK;
}
