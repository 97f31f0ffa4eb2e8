/* Stand-in for the MPI types named by CarpetLib's dist.hh, for a build
 * without MPI.  Only declarations; no MPI call is ever made. */
#ifndef CGX_SHIM_NOMPI_H
#define CGX_SHIM_NOMPI_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
typedef long MPI_Aint;
#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_CHAR 3
#define MPI_BYTE 4
#define MPI_SHORT 5
#define MPI_UNSIGNED 6
#define MPI_UNSIGNED_CHAR 7
#define MPI_UNSIGNED_SHORT 8
#define MPI_LONG 9
#define MPI_UNSIGNED_LONG 10
#define MPI_LONG_LONG_INT 11
#define MPI_FLOAT 12
#define MPI_LONG_DOUBLE 13
#define MPI_REQUEST_NULL 0
#endif
