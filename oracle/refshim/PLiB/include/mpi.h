/* Project-written single-rank stand-in for <mpi.h>. Test infrastructure only:
 * the oracle harness compiles the reference's CPU hot path as one rank, where
 * every collective is a local copy and point-to-point calls are never made.
 * Symbol list: the MPI_* names used under PLiB/, Iterators/ and HiDEMLib/. */
#ifndef HIDEM_REFSHIM_MPI_H
#define HIDEM_REFSHIM_MPI_H
#include <cstring>
#include <cstddef>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1
#define MPI_COMM_TYPE_SHARED 0
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_MAX_PROCESSOR_NAME 64
#define MPI_SUCCESS 0

#define MPI_BYTE 1
#define MPI_CHAR 1
#define MPI_C_BOOL 1
#define MPI_INT 4
#define MPI_UINT 4
#define MPI_UNSIGNED 4
#define MPI_FLOAT 4
#define MPI_DOUBLE 8
#define MPI_LONG_LONG_INT 8
#define MPI_LONG_LONG 8
#define MPI_UNSIGNED_LONG 8
#define MPI_INT64_T 8
#define MPI_UINT64_T 8
#define MPI_UINT32_T 4
#define MPI_INT32_T 4
#define MPI_UINT8_T 1
#define MPI_INT8_T 1

#define MPI_SUM 0
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_LOR 3

inline int hidem_shim_copy(const void *s, void *r, int n, MPI_Datatype t) {
    if (s != MPI_IN_PLACE && s != r && n > 0) std::memcpy(r, s, (size_t)n * (size_t)t);
    return 0;
}
inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) { return hidem_shim_copy(s, r, n, t); }
inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) { return hidem_shim_copy(s, r, n, t); }
inline int MPI_Allgather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, MPI_Comm) { return hidem_shim_copy(s, r, n, t); }
inline int MPI_Gather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, int, MPI_Comm) { return hidem_shim_copy(s, r, n, t); }
inline int MPI_Gatherv(const void *s, int n, MPI_Datatype t, void *r, const int *, const int *, MPI_Datatype, int, MPI_Comm) { return hidem_shim_copy(s, r, n, t); }
inline int MPI_Alltoall(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, MPI_Comm) { return hidem_shim_copy(s, r, n, t); }
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Exscan(const void *, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) { if (n > 0) std::memset(r, 0, (size_t)n * (size_t)t); return 0; }
inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return 0; }
inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return 0; }
inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }
inline int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }
inline int MPI_Info_create(MPI_Info *) { return 0; }
inline int MPI_Comm_split_type(MPI_Comm c, int, int, MPI_Info, MPI_Comm *n) { *n = c; return 0; }
inline int MPI_Get_processor_name(char *name, int *len) { std::strcpy(name, "local"); *len = 5; return 0; }
#endif
