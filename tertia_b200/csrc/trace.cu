// trace.cu — qs_trace_attach of the traced library (see trace.cuh); linked
// only into libqsb200_trace.so, whose instrumented units are compiled with
// -DQS_TRACE.
#include "trace.cuh"
#include "../../include/qsb200.h"
#include "../../include/qsb200_trace.h"

extern "C" int qs_trace_set_push(void* rec, void* pos, unsigned mask);
extern "C" int qs_trace_set_push64(void* rec, void* pos, unsigned mask);
extern "C" int qs_trace_set_fft(void* rec, void* pos, unsigned mask);
extern "C" int qs_trace_set_sort(void* rec, void* pos, unsigned mask);

extern "C" int qs_trace_attach(void* rec, unsigned* pos, unsigned nrec) {
    if (rec && (nrec == 0 || (nrec & (nrec - 1)) != 0 || !pos)) return QS_ERR_INVALID;
    const unsigned mask = rec ? nrec - 1 : 0;
    int (*set[])(void*, void*, unsigned) = {qs_trace_set_push, qs_trace_set_push64,
                                            qs_trace_set_fft, qs_trace_set_sort};
    for (auto f : set)
        if (f(rec, pos, mask) != 0) return QS_ERR_CUDA;
    return QS_OK;
}
