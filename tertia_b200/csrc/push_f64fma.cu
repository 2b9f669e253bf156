// push_f64fma.cu — the grouped CIC push (push.cuh) in FP64 with FMA
// contraction, for the FP64 path on FFT transforms.  push_f64.cu, compiled
// without contraction, keeps the reference's expression order for the plain
// FP64 path.
#include "push.cuh"

namespace qs {
int launch_push_rows_f64(const PushArgs<double>& a, cudaStream_t st) {
    return launch_push_rows<double>(a, st);
}
}  // namespace qs

QS_TRACE_UNIT(push64)
