/* Stand-in for HDF5's header (oracle pin build): the type names the
 * reference's declarations use; no HDF5 call is linked. */
#ifndef QS_PIN_HDF5_STUB_H
#define QS_PIN_HDF5_STUB_H
typedef long long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
#endif
