/* Stand-in for MPI's header (oracle pin build): type names only; the pin
 * runs one rank and its harness supplies GetRank / GetSize. */
#ifndef QS_PIN_MPI_STUB_H
#define QS_PIN_MPI_STUB_H
typedef int MPI_Comm;
typedef int MPI_Status;
typedef int MPI_Request;
#endif
