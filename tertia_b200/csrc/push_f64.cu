// push_f64.cu — the FP64 plasma push (see push.cuh).  Compiled with
// -fmad=false: the reference's expression order without contraction.
#include "push.cuh"

namespace qs {
template int launch_push<double>(const PushArgs<double>&, int, bool, cudaStream_t);
}  // namespace qs
