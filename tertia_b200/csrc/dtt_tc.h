// dtt_tc.h — split-precision half-integer transforms on the tcgen05 tensor
// cores (host interface).
#pragma once
#include <cuda_runtime.h>
#include <string>

namespace qs {

// the bounded-wait self-test (dtt_tc.cu): sets DEV_ERR_TIMEOUT in *err after
// `limit` tries of an mbarrier wait nothing completes
int launch_wait_limit_probe(int* err, unsigned limit, cudaStream_t st);

class TcTransformer {
public:
    // mode: QS_PREC_TF32X3 / QS_PREC_BF16X3 / QS_PREC_BF16X6.  Returns nullptr
    // (with a reason) when the sizes or the mode are not supported.
    static TcTransformer* create(int mode, int ny, int nz, int* err_flag, std::string& why);
    virtual ~TcTransformer() {}
    // nf fields: out_f = scale * A_z(kz_f) in_f A_y(ky_f); in_f are nz x ny
    // planes stored consecutively from in[0]; returns the kernels launched.
    virtual int run(int nf, const void* const* in, void* const* out, const int* kz,
                    const int* ky, double scale, int elem_size, cudaStream_t st) = 0;
    // the three launches of run(), separately (for per-kernel timing):
    // stage 0 splits the inputs, stage 1 is the y pass, stage 2 the z pass.
    virtual int run_stage(int stage, int nf, const void* const* in, void* const* out,
                          const int* kz, const int* ky, double scale, cudaStream_t st) = 0;
    // operand buffer a producer may fill directly before run_stage(1..2):
    // term s of field f at base + (s * term_stride + f * ny*nz) elements,
    // element type bf16 (kind 0) or tf32-in-float (kind 1)
    virtual void split_target(void** base, int* nsplit, int* kind, size_t* term_stride) = 0;
    // REDFT11 x REDFT11 transform of nplanes contiguous planes in batches;
    // stage < 0 runs all three launches of every batch
    virtual int run_batched(const float* in, float* out, int nplanes, double scale, int stage,
                            cudaStream_t st) = 0;
};

}  // namespace qs
