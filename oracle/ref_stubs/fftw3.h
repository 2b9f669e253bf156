/* Stand-in for FFTW 3's header when the reference's push and beam files are
 * compiled for the oracle pin (oracle/ref_pin.cpp): those files need only the
 * type names, no FFTW call is linked. */
#ifndef QS_PIN_FFTW3_STUB_H
#define QS_PIN_FFTW3_STUB_H
typedef double fftw_complex[2];
typedef struct fftw_plan_s* fftw_plan;
typedef int fftw_r2r_kind;
#endif
