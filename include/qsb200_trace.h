/* qsb200_trace.h — the device timeline of the traced build.
 *
 * libqsb200_trace.so exports everything qsb200.h declares plus the entry
 * below; its march kernels (the grouped CIC push, the z- and y-passes of the
 * transforms, the map kernels and the plasma regrouping) stamp, per CTA, when
 * the CTA started, when its wait on the preceding kernel returned and when it
 * ended, into a ring of records in device memory.  libqsb200.so has neither
 * the entry nor the stamps.  It plays the part of the reference's wall-clock
 * stamps around the phases of a layer (gettimeofday in MoveAllSplitLayers and
 * MoveSplitLayer, movepart_splitlayer.cpp:28-554, 574-732) at the
 * granularity of kernels and CTAs.
 *
 * A record is four 64-bit words:
 *   [0] %globaltimer (ns) at the CTA's start,
 *   [1] when its dependency wait returned,
 *   [2] at its end,
 *   [3] kind << 56 | gridDim.y << 48 | blockIdx.y << 40 | SM << 32 | blockIdx.x,
 * with kind 1 / 2 the push without / with particle stores, 3 a z-pass, 4 a
 * y-pass, 5 / 6 / 8 the map kernel (predictor / corrector / corrector with
 * the next layer's predictor), 10 / 11 the regrouping's offsets / scatter.
 */
#ifndef QSB200_TRACE_H
#define QSB200_TRACE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Attach a ring of nrec records (nrec a power of two; rec: 4 * nrec
 * uint64 of device memory, pos: one uint32 of device memory, zeroed by the
 * caller) to the instrumented kernels, or detach with rec = NULL.  Records
 * past nrec overwrite the oldest; *pos counts every record appended.  Kernels
 * already launched or captured write to the ring that is attached when they
 * run.  Returns QS_OK, QS_ERR_INVALID or QS_ERR_CUDA. */
int qs_trace_attach(void* rec, unsigned* pos, unsigned nrec);

#ifdef __cplusplus
}
#endif
#endif
