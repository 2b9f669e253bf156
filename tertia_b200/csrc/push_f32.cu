// push_f32.cu — the FP32 plasma push (see push.cuh): factored divisions,
// FMA contraction allowed.
#include "push.cuh"

namespace qs {
template int launch_push<float>(const PushArgs<float>&, int, bool, cudaStream_t);
}  // namespace qs

QS_TRACE_UNIT(push)
